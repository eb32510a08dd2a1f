/*
C entry points of the CPU oracle, shared by the two oracle libraries:
  oracle/_build/liboracle.so   - the restated solvers of mhd_oracle.hpp
  oracle/_ref/libpamhd_ref.so  - the reference's own solver headers
Both drive them with the same grid restatements: Mode C (mode_c.hpp) and
the staggered-field step (mode_s.hpp).

TEST INFRASTRUCTURE - see mhd_oracle.hpp for who may use this.

The including file defines ORACLE_API(name) (the exported symbol name),
ORACLE_FLUX (the solver dispatch functor type) and ORACLE_SPLIT (the
two-population split solver functor type).
*/
#include <cstdio>
#include <cstring>
#include <vector>

#include "mode_s.hpp"
#include "n_solve.hpp"
#include "substep.hpp"

namespace {

using Grid = oracle::Mode_C_Grid<ORACLE_FLUX>;
using SGrid = oracle::Mode_S_Grid<ORACLE_FLUX>;
using NGrid = oracle::N_Grid<ORACLE_SPLIT>;
using LGrid = oracle::Substep_Grid<ORACLE_FLUX>;

thread_local std::string last_error;

int fail_with(const char* what)
{
	last_error = what;
	return PAMHD_ERR_ARGUMENT;
}

} // namespace

extern "C" {

// text of the last argument error of this thread
const char* ORACLE_API(last_error)(void)
{
	return last_error.c_str();
}

/*
Face fluxes of n independent face problems in the face frame; see
pamhd_gpu_face_flux in include/pamhd_gpu.h for the layout.  flags[i]
receives the PAMHD_FLAG_* of the exception the solver threw, or 0.
Returns the number of failed faces.
*/
int64_t ORACLE_API(face_flux)(
	int32_t solver, int64_t n, const double* neg, const double* pos, const double* bg,
	double gamma, double mu0, double* flux, double* speed, uint32_t* flags)
{
	const ORACLE_FLUX solve{};
	int64_t failed = 0;
	for (int64_t i = 0; i < n; i++) {
		oracle::MHD a, b;
		const double* x = neg + 8 * i;
		const double* y = pos + 8 * i;
		a.rho = x[0]; a.mom = {x[1], x[2], x[3]}; a.nrj = x[4]; a.mag = {x[5], x[6], x[7]};
		b.rho = y[0]; b.mom = {y[1], y[2], y[3]}; b.nrj = y[4]; b.mag = {y[5], y[6], y[7]};
		oracle::Vec3 g{0, 0, 0};
		if (bg != nullptr) g = {bg[3 * i], bg[3 * i + 1], bg[3 * i + 2]};
		double* out = flux + 8 * i;
		try {
			const oracle::Face_Flux r = solve(solver, a, b, g, gamma, mu0);
			const double row[8] = {
				r.flux.rho, r.flux.mom[0], r.flux.mom[1], r.flux.mom[2],
				r.flux.nrj, r.flux.mag[0], r.flux.mag[1], r.flux.mag[2]};
			std::memcpy(out, row, sizeof row);
			speed[i] = r.speed;
			flags[i] = 0;
		} catch (const oracle::Domain_Error& e) {
			for (int k = 0; k < 8; k++) out[k] = 0;
			speed[i] = 0;
			flags[i] = e.flag;
			failed++;
		} catch (const std::exception&) {
			for (int k = 0; k < 8; k++) out[k] = 0;
			speed[i] = 0;
			flags[i] = 0x80000000u;
			failed++;
		}
	}
	return failed;
}

// a Mode C grid; returns NULL on an invalid configuration
void* ORACLE_API(grid_create)(const pamhd_cfg* cfg)
{
	try {
		return new Grid(*cfg);
	} catch (const std::exception& e) {
		last_error = e.what();
		return nullptr;
	}
}

void ORACLE_API(grid_destroy)(void* grid)
{
	delete static_cast<Grid*>(grid);
}

void ORACLE_API(grid_set_threads)(void* grid, int32_t threads)
{
	static_cast<Grid*>(grid)->threads = threads < 1 ? 1 : threads;
}

int ORACLE_API(grid_set_state)(void* grid, const double* const soa[8])
{
	try {
		static_cast<Grid*>(grid)->set_interior(soa);
	} catch (const std::exception& e) {
		return fail_with(e.what());
	}
	return PAMHD_OK;
}

int ORACLE_API(grid_get_state)(void* grid, double* const soa[8])
{
	static_cast<Grid*>(grid)->get_interior(soa);
	return PAMHD_OK;
}

/*
One step (see Mode_C_Grid::step).  On a solver failure returns
PAMHD_ERR_PHYSICS with the flag, the failing cell (interior coordinates;
ghosts are -1 or n) and the face direction (+1..+3); the state is left as
it was before the step's update.
*/
int ORACLE_API(grid_step)(void* grid, double max_dt, double* dt_taken,
                          uint32_t* flag, int32_t cell[3], int32_t* dir)
{
	Grid& g = *static_cast<Grid*>(grid);
	*flag = 0;
	try {
		*dt_taken = g.step(max_dt);
	} catch (const oracle::Domain_Error& e) {
		*flag = e.flag;
		int c[3];
		g.coords(size_t(g.failure.cell), c);
		for (int d = 0; d < 3; d++) cell[d] = c[d];
		*dir = g.failure.dir;
		return PAMHD_ERR_PHYSICS;
	} catch (const std::exception& e) {
		return fail_with(e.what());
	}
	return PAMHD_OK;
}

/*
Largest face signal speed of the last step per dimension: the maximum of
Max_v over the cells the step visited (mhd/solve.hpp:319-322 stores each
face's speed in both cells' slots).
*/
int ORACLE_API(grid_max_signal)(void* grid, double out[3])
{
	const Grid& g = *static_cast<const Grid*>(grid);
	for (int d = 0; d < 3; d++) out[d] = 0.0;
	for (size_t idx = 0; idx < g.U.size(); idx++) {
		if (g.CType[idx] < 0) continue;
		for (int d = 0; d < 3; d++) {
			out[d] = std::max(out[d], std::max(g.Max_v[idx][2 * d], g.Max_v[idx][2 * d + 1]));
		}
	}
	return PAMHD_OK;
}

/*
Time-stamped inflow of a VALUE side (see Mode_C_Grid::set_inflow): count
timestamps and count + 1 states of 8 doubles.
*/
int ORACLE_API(grid_set_inflow)(void* grid, int32_t dim, int32_t side, int32_t count, const double* times,
                                const double* states)
{
	if (count < 0 or (count > 0 and times == nullptr) or states == nullptr) return fail_with("inflow arguments");
	std::vector<double> t(times, times + count);
	std::vector<std::array<double, 8>> u(size_t(count) + 1);
	for (size_t i = 0; i < u.size(); i++) {
		for (int v = 0; v < 8; v++) u[i][v] = states[8 * i + v];
	}
	try {
		static_cast<Grid*>(grid)->set_inflow(dim, side, t, u);
	} catch (const std::exception& e) {
		return fail_with(e.what());
	}
	return PAMHD_OK;
}

// one step with a prescribed dt (see Mode_C_Grid::step_with)
int ORACLE_API(grid_step_dt)(void* grid, double dt, uint32_t* flag)
{
	Grid& g = *static_cast<Grid*>(grid);
	*flag = 0;
	try {
		g.step_with(dt);
	} catch (const oracle::Domain_Error& e) {
		*flag = e.flag;
		return PAMHD_ERR_PHYSICS;
	} catch (const std::exception& e) {
		return fail_with(e.what());
	}
	return PAMHD_OK;
}

// runs steps until t reaches t_end or max_steps steps were taken; returns steps taken or -1
int64_t ORACLE_API(grid_run)(void* grid, double t_start, double t_end, int64_t max_steps,
                             double* t_reached, double* dt_history)
{
	Grid& g = *static_cast<Grid*>(grid);
	double t = t_start;
	int64_t steps = 0;
	try {
		while (t < t_end and steps < max_steps) {
			const double dt = g.step(t_end - t);
			if (dt_history != nullptr) dt_history[steps] = dt;
			t += dt;
			steps++;
		}
	} catch (const std::exception& e) {
		last_error = e.what();
		*t_reached = t;
		return -1;
	}
	*t_reached = t;
	return steps;
}

// a staggered-field grid (periodic, COPY or VALUE sides); NULL on an invalid configuration
void* ORACLE_API(sgrid_create)(const pamhd_cfg* cfg)
{
	try {
		return new SGrid(*cfg);
	} catch (const std::exception& e) {
		last_error = e.what();
		return nullptr;
	}
}

void ORACLE_API(sgrid_destroy)(void* grid)
{
	delete static_cast<SGrid*>(grid);
}

// cell state (8 arrays) and the normal field of every cell's -x, -y, -z face (3 arrays; along a
// bounded dimension n + 1 faces, the high wall included)
int ORACLE_API(sgrid_set_state)(void* grid, const double* const soa[8], const double* const faces[3])
{
	try {
		static_cast<SGrid*>(grid)->set_state(soa, faces);
	} catch (const std::exception& e) {
		return fail_with(e.what());
	}
	return PAMHD_OK;
}

// background field: bg[3 d + c] = component c at every cell's -d face; NULL clears it
int ORACLE_API(sgrid_set_background)(void* grid, const double* const bg[9])
{
	static_cast<SGrid*>(grid)->set_background(bg);
	return PAMHD_OK;
}

int ORACLE_API(sgrid_get_state)(void* grid, double* const soa[8], double* const faces[3])
{
	static_cast<SGrid*>(grid)->get_state(soa, faces);
	return PAMHD_OK;
}

// time-stamped states of the staggered grid's VALUE side, as grid_set_inflow
int ORACLE_API(sgrid_set_inflow)(void* grid, int32_t dim, int32_t side, int32_t count, const double* times,
                                 const double* states)
{
	if (count < 0 or (count > 0 and times == nullptr) or states == nullptr) return fail_with("inflow arguments");
	std::vector<double> t(times, times + count);
	std::vector<std::array<double, 8>> u(size_t(count) + 1);
	for (size_t i = 0; i < u.size(); i++) {
		for (int v = 0; v < 8; v++) u[i][v] = states[8 * i + v];
	}
	try {
		static_cast<SGrid*>(grid)->set_inflow(dim, side, t, u);
	} catch (const std::exception& e) {
		return fail_with(e.what());
	}
	return PAMHD_OK;
}

// one staggered step (see Mode_S_Grid::step); failures as grid_step
int ORACLE_API(sgrid_step)(void* grid, double max_dt, double* dt_taken,
                           uint32_t* flag, int32_t cell[3], int32_t* dir)
{
	SGrid& g = *static_cast<SGrid*>(grid);
	*flag = 0;
	try {
		*dt_taken = g.step(max_dt);
	} catch (const oracle::Domain_Error& e) {
		*flag = e.flag;
		int c[3];
		g.coords(size_t(g.failure.cell), c);
		for (int d = 0; d < 3; d++) cell[d] = c[d];
		*dir = g.failure.dir;
		return PAMHD_ERR_PHYSICS;
	} catch (const std::exception& e) {
		return fail_with(e.what());
	}
	return PAMHD_OK;
}

/*
Split fluxes of n two-population face problems (total states, face frame):
neg, pos n x 8; flux_neg, flux_pos n x 8 (already times area and dt);
speed n; flags n.  Returns the number of failed faces.
*/
int64_t ORACLE_API(face_flux_N)(
	int32_t solver, int64_t n, const double* neg, const double* pos, double area, double dt,
	double gamma, double mu0, double* flux_neg, double* flux_pos, double* speed, uint32_t* flags)
{
	const ORACLE_SPLIT split{};
	int64_t failed = 0;
	for (int64_t i = 0; i < n; i++) {
		oracle::MHD a, b;
		const double* x = neg + 8 * i;
		const double* y = pos + 8 * i;
		a.rho = x[0]; a.mom = {x[1], x[2], x[3]}; a.nrj = x[4]; a.mag = {x[5], x[6], x[7]};
		b.rho = y[0]; b.mom = {y[1], y[2], y[3]}; b.nrj = y[4]; b.mag = {y[5], y[6], y[7]};
		double* on = flux_neg + 8 * i;
		double* op = flux_pos + 8 * i;
		try {
			const oracle::Split_Flux r = split(solver, a, b, oracle::Vec3{0, 0, 0}, area, dt, gamma, mu0);
			const double rn[8] = {r.neg.rho, r.neg.mom[0], r.neg.mom[1], r.neg.mom[2],
			                      r.neg.nrj, r.neg.mag[0], r.neg.mag[1], r.neg.mag[2]};
			const double rp[8] = {r.pos.rho, r.pos.mom[0], r.pos.mom[1], r.pos.mom[2],
			                      r.pos.nrj, r.pos.mag[0], r.pos.mag[1], r.pos.mag[2]};
			std::memcpy(on, rn, sizeof rn);
			std::memcpy(op, rp, sizeof rp);
			speed[i] = r.speed;
			flags[i] = 0;
		} catch (const oracle::Domain_Error& e) {
			for (int k = 0; k < 8; k++) on[k] = op[k] = 0;
			speed[i] = 0;
			flags[i] = e.flag;
			failed++;
		} catch (const std::exception&) {
			for (int k = 0; k < 8; k++) on[k] = op[k] = 0;
			speed[i] = 0;
			flags[i] = 0x80000000u;
			failed++;
		}
	}
	return failed;
}

/*
The scheme of tests/mhd/two_reference.cpp (see oracle::reference_2pop_1d)
with this library's split solvers; returns the number of steps or -1.
*/
int32_t ORACLE_API(reference_2pop_1d)(int32_t solver, int32_t cells, double t_end, double length, double* out)
{
	try {
		return oracle::reference_2pop_1d(ORACLE_SPLIT{}, solver, cells, t_end, length, out);
	} catch (const std::exception& e) {
		last_error = e.what();
		return -1;
	}
}

// a two-population grid (periodic); NULL on an invalid configuration
void* ORACLE_API(ngrid_create)(const int32_t n[3], const double len[3], int32_t solver, double gamma, double mu0,
                               double min_pressure)
{
	try {
		return new NGrid(n[0], n[1], n[2], len[0], len[1], len[2], solver, gamma, mu0, min_pressure);
	} catch (const std::exception& e) {
		last_error = e.what();
		return nullptr;
	}
}

void ORACLE_API(ngrid_destroy)(void* grid)
{
	delete static_cast<NGrid*>(grid);
}

// 13 arrays: rho1, mom1 xyz, E1, rho2, mom2 xyz, E2, B xyz
int ORACLE_API(ngrid_set_state)(void* grid, const double* const a[13])
{
	static_cast<NGrid*>(grid)->set_state(a);
	return PAMHD_OK;
}

int ORACLE_API(ngrid_get_state)(void* grid, double* const a[13])
{
	static_cast<NGrid*>(grid)->get_state(a);
	return PAMHD_OK;
}

// one step of length dt; *max_dt receives the next step's limit; failures as grid_step
int ORACLE_API(ngrid_step)(void* grid, double dt, double* max_dt, uint32_t* flag, int32_t cell[3], int32_t* dir)
{
	NGrid& g = *static_cast<NGrid*>(grid);
	*flag = 0;
	try {
		*max_dt = g.step(dt);
	} catch (const oracle::Domain_Error& e) {
		*flag = e.flag;
		if (g.failure.cell >= 0) {
			const int64_t c = g.failure.cell;
			cell[0] = int32_t(c % g.n[0]);
			cell[1] = int32_t((c / g.n[0]) % g.n[1]);
			cell[2] = int32_t(c / (int64_t(g.n[0]) * g.n[1]));
			*dir = g.failure.dir;
		}
		return PAMHD_ERR_PHYSICS;
	} catch (const std::exception& e) {
		return fail_with(e.what());
	}
	return PAMHD_OK;
}

// a grid with local time stepping (periodic); NULL on an invalid configuration
void* ORACLE_API(lgrid_create)(const pamhd_cfg* cfg)
{
	try {
		return new LGrid(*cfg);
	} catch (const std::exception& e) {
		last_error = e.what();
		return nullptr;
	}
}

void ORACLE_API(lgrid_destroy)(void* grid)
{
	delete static_cast<LGrid*>(grid);
}

int ORACLE_API(lgrid_set_state)(void* grid, const double* const soa[8])
{
	try {
		static_cast<LGrid*>(grid)->set_interior(soa);
	} catch (const std::exception& e) {
		return fail_with(e.what());
	}
	return PAMHD_OK;
}

int ORACLE_API(lgrid_get_state)(void* grid, double* const soa[8])
{
	static_cast<LGrid*>(grid)->get_interior(soa);
	return PAMHD_OK;
}

// the substep exponents' bounds of every cell (the options substep-min / substep-max)
int ORACLE_API(lgrid_set_exponents)(void* grid, const int32_t* mins, const int32_t* maxs)
{
	try {
		static_cast<LGrid*>(grid)->set_exponents(mins, maxs);
	} catch (const std::exception& e) {
		return fail_with(e.what());
	}
	return PAMHD_OK;
}

/*
The substep plan from given per-cell CFL limits (x fastest) on the grid's
exponent bounds (lgrid_set_exponents first): every cell's period, the
substep length and the largest period.  Returns PAMHD_OK, or
PAMHD_ERR_PHYSICS where the reference aborts on unexpected substeps.
*/
int ORACLE_API(lgrid_plan)(void* grid, const double* limits, double max_dt, int32_t* periods, double* substep,
                           int32_t* max_period)
{
	LGrid& g = *static_cast<LGrid*>(grid);
	try {
		g.plan_from_limits(limits, max_dt);
	} catch (const std::exception& e) {
		last_error = e.what();
		return PAMHD_ERR_PHYSICS;
	}
	for (size_t c = 0; c < g.U.size(); c++) periods[c] = g.period[c];
	*substep = g.substep;
	*max_period = g.max_substep;
	return PAMHD_OK;
}

// one step with substeps; *dt_taken its length, *substeps their number, periods[c] each cell's period
int ORACLE_API(lgrid_step)(void* grid, double max_dt, double* dt_taken, int32_t* substeps, int32_t* periods,
                           uint32_t* flag)
{
	LGrid& g = *static_cast<LGrid*>(grid);
	*flag = 0;
	try {
		*dt_taken = g.step(max_dt);
	} catch (const oracle::Domain_Error& e) {
		*flag = e.flag;
		return PAMHD_ERR_PHYSICS;
	} catch (const std::exception& e) {
		return fail_with(e.what());
	}
	*substeps = g.max_substep;
	if (periods != nullptr) {
		for (size_t c = 0; c < g.U.size(); c++) periods[c] = g.period[c];
	}
	return PAMHD_OK;
}

} // extern "C"
