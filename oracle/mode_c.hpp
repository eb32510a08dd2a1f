/*
CPU oracle, L3: the cell-centred ("Mode C") MHD step on a uniform grid and
the 1-D scheme of the reference's golden generator.

TEST INFRASTRUCTURE - see mhd_oracle.hpp for who may use this.

Mode_C_Grid<Flux> restates, for a uniform Cartesian grid with one ghost
layer on non-periodic sides:
  - cell classes of mhd/boundaries.hpp:79-236: interior cells are 1
    (solve), ghosts that touch the interior through a face are 0
    (boundary, read-only), edge and corner ghosts are -1 (dont_solve);
  - get_fluxes, mhd/solve.hpp:217-392 without the staggered parts: for
    every cell of class >= 0 and each +d face neighbour of class >= 0, the
    two states are rotated into the face frame (:106-118), solved
    (:135-154), the speed stored on both sides (:319-322) and dt * F added
    to the cell's +d and the neighbour's -d flux slots (:375-392);
  - update_mhd_state, mhd/solve.hpp:1543-1602, Mode C part: for class > 0
    cells U += (F(-d) - F(+d)) / d_len for x, then y, then z, with the
    momentum and field terms multiplied by 1/d_len as the reference does,
    and the field updated from the solver's field flux (:1578-1587);
  - minimize_timestep, mhd/solve.hpp:1933-2007, and the global rule of
    substepping.hpp:285-338 without substeps: dt_cell = min over the faces
    of CFL * d_len / max(Max_v) (0 if that speed <= 0), global dt = the
    minimum over cells of class >= 0, replaced by max_dt when
    max_dt <= that minimum;
  - ghost refresh after each step, as tests/mhd/test.cpp:559 applies the
    boundaries: COPY copies density, velocity, thermal pressure and field
    of the inward face neighbour (mhd/boundaries.hpp:818-1030, the
    constant-pressure field copy of update_vol_B, solve.hpp:1648-1672);
    VALUE sets a fixed conservative state.
A dimension with one cell is inactive (no faces).  The step parallelises
over cells with std::thread: every face writes only its own two slots.

reference_1d() restates tests/mhd/reference.cpp:189-440 and :833-877 (hydro
fluxes from the solver, field from the upwind E = -v x B, apply_fluxes with
its positivity checks), the scheme its mhd_*.ref goldens were made with.
*/
#ifndef PAMHD_ORACLE_MODE_C_HPP
#define PAMHD_ORACLE_MODE_C_HPP

#include <atomic>
#include <cstring>
#include <functional>
#include <mutex>

#include "mhd_oracle.hpp"

namespace oracle {

// apply_fluxes of mhd/common.hpp:707-743 (state += flux * factor, then checks)
inline void apply_fluxes(MHD& u, const MHD& f, const double factor, const double gamma, const double mu0)
{
	u.rho += f.rho * factor;
	for (int i = 0; i < 3; i++) u.mom[i] = u.mom[i] + f.mom[i] * factor;
	u.nrj += f.nrj * factor;
	for (int i = 0; i < 3; i++) u.mag[i] = u.mag[i] + f.mag[i] * factor;
	if (u.rho <= 0) {
		throw Domain_Error(PAMHD_FLAG_NEW_STATE, "New state has negative mass density");
	}
	const double p = get_pressure(u.rho, u.mom, u.nrj, u.mag, gamma, mu0);
	if (p <= 0) {
		throw Domain_Error(PAMHD_FLAG_NEW_STATE, "New state has negative pressure");
	}
}

// the first face at which a step failed, in the reference's iteration order
struct Failure {
	uint32_t flag = 0;
	int64_t cell = -1; // linear index in the extended grid
	int dir = 0;
	std::string what;
};

template <class Flux> class Mode_C_Grid {
public:
	pamhd_cfg cfg;
	Flux flux;
	int n[3], ext[3], N[3];
	bool active[3], periodic[3];
	std::vector<MHD> U;
	std::vector<std::array<MHD, 6>> F;     // dt-scaled flux per face slot (-x,+x,-y,+y,-z,+z)
	std::vector<std::array<double, 6>> Max_v;
	std::vector<double> Timestep;
	std::vector<int8_t> CType;
	int threads = 1;
	Failure failure;
	/*
	Time-stamped inflow of VALUE sides, as the solar-wind boundary of
	mhd/solar_wind_box.hpp:227-268: states[i] holds while i timestamps are
	<= the simulation time (states has one more entry than times).  Empty:
	the side keeps cfg.value_lo / value_hi.
	*/
	struct Inflow {
		std::vector<double> times;
		std::vector<std::array<double, 8>> states;
	};
	Inflow inflow[3][2];
	double time = 0;  // simulation time since set_interior

	explicit Mode_C_Grid(const pamhd_cfg& c) : cfg(c)
	{
		if (cfg.solver != PAMHD_RUSANOV and cfg.solver != PAMHD_HLL_ATHENA
			and cfg.solver != PAMHD_HLLD_ATHENA and cfg.solver != PAMHD_ROE_ATHENA) {
			throw std::invalid_argument("invalid solver");
		}
		for (int d = 0; d < 3; d++) {
			n[d] = cfg.n[d];
			if (n[d] < 1) throw std::invalid_argument("cell count must be >= 1");
			active[d] = n[d] > 1;
			periodic[d] = cfg.bc_lo[d] == PAMHD_BC_PERIODIC and cfg.bc_hi[d] == PAMHD_BC_PERIODIC;
			if (active[d] and not periodic[d]
				and (cfg.bc_lo[d] == PAMHD_BC_PERIODIC or cfg.bc_hi[d] == PAMHD_BC_PERIODIC)) {
				throw std::invalid_argument("periodic must be given on both sides");
			}
			ext[d] = (active[d] and not periodic[d]) ? 1 : 0;
			N[d] = n[d] + 2 * ext[d];
		}
		const size_t total = size_t(N[0]) * N[1] * N[2];
		U.resize(total);
		F.assign(total, {});
		Max_v.assign(total, {0, 0, 0, 0, 0, 0});
		Timestep.assign(total, 0);
		CType.resize(total);
		for (int k = -ext[2]; k < n[2] + ext[2]; k++)
		for (int j = -ext[1]; j < n[1] + ext[1]; j++)
		for (int i = -ext[0]; i < n[0] + ext[0]; i++) {
			const int c[3] = {i, j, k};
			int outside = 0;
			for (int d = 0; d < 3; d++) outside += (c[d] < 0 or c[d] >= n[d]) ? 1 : 0;
			CType[index(i, j, k)] = outside == 0 ? 1 : (outside == 1 ? 0 : -1);
		}
	}

	size_t index(const int i, const int j, const int k) const
	{
		return size_t(i + ext[0]) + size_t(N[0]) * (size_t(j + ext[1]) + size_t(N[1]) * size_t(k + ext[2]));
	}

	void coords(const size_t idx, int c[3]) const
	{
		c[0] = int(idx % N[0]) - ext[0];
		c[1] = int((idx / N[0]) % N[1]) - ext[1];
		c[2] = int(idx / (size_t(N[0]) * N[1])) - ext[2];
	}

	// linear index of the +d face neighbour of cell c, or -1 if none
	int64_t plus_neighbor(const int c[3], const int d) const
	{
		if (not active[d]) return -1;
		int m[3] = {c[0], c[1], c[2]};
		m[d] += 1;
		if (periodic[d] and m[d] == n[d]) m[d] = 0;
		if (m[d] >= n[d] + ext[d]) return -1;
		return int64_t(index(m[0], m[1], m[2]));
	}

	int64_t minus_neighbor(const int c[3], const int d) const
	{
		if (not active[d]) return -1;
		int m[3] = {c[0], c[1], c[2]};
		m[d] -= 1;
		if (periodic[d] and m[d] < 0) m[d] = n[d] - 1;
		if (m[d] < -ext[d]) return -1;
		return int64_t(index(m[0], m[1], m[2]));
	}

	void set_interior(const double* const soa[8])
	{
		for (int k = 0; k < n[2]; k++)
		for (int j = 0; j < n[1]; j++)
		for (int i = 0; i < n[0]; i++) {
			const size_t src = size_t(i) + size_t(n[0]) * (size_t(j) + size_t(n[1]) * k);
			MHD& u = U[index(i, j, k)];
			u.rho = soa[0][src];
			u.mom = {soa[1][src], soa[2][src], soa[3][src]};
			u.nrj = soa[4][src];
			u.mag = {soa[5][src], soa[6][src], soa[7][src]};
		}
		for (auto& m: Max_v) m = {0, 0, 0, 0, 0, 0};
		failure = Failure();
		time = 0;
		apply_boundaries();
	}

	// the value of a VALUE side at the current time
	const double* value_of(const int d, const bool lo) const
	{
		const Inflow& t = inflow[d][lo ? 0 : 1];
		if (t.states.empty()) return lo ? cfg.value_lo[d] : cfg.value_hi[d];
		size_t i = 0;
		while (i < t.times.size() and time >= t.times[i]) i++;
		return t.states[i].data();
	}

	void set_inflow(const int d, const int side, const std::vector<double>& times,
	                const std::vector<std::array<double, 8>>& states)
	{
		if (d < 0 or d > 2 or (side != 0 and side != 1)) throw std::invalid_argument("side");
		if ((side == 0 ? cfg.bc_lo[d] : cfg.bc_hi[d]) != PAMHD_BC_VALUE) {
			throw std::invalid_argument("inflow tables are for VALUE sides");
		}
		if (states.size() != times.size() + 1) throw std::invalid_argument("states: one more than times");
		inflow[d][side] = {times, states};
		apply_boundaries();
	}

	void get_interior(double* const soa[8]) const
	{
		for (int k = 0; k < n[2]; k++)
		for (int j = 0; j < n[1]; j++)
		for (int i = 0; i < n[0]; i++) {
			const size_t dst = size_t(i) + size_t(n[0]) * (size_t(j) + size_t(n[1]) * k);
			const MHD& u = U[index(i, j, k)];
			soa[0][dst] = u.rho;
			soa[1][dst] = u.mom[0]; soa[2][dst] = u.mom[1]; soa[3][dst] = u.mom[2];
			soa[4][dst] = u.nrj;
			soa[5][dst] = u.mag[0]; soa[6][dst] = u.mag[1]; soa[7][dst] = u.mag[2];
		}
	}

	// runs body(first, last) over [0, count) on `threads` threads
	void parallel(const size_t count, const std::function<void(size_t, size_t)>& body) const
	{
		if (threads <= 1 or count < 4096) {
			body(0, count);
			return;
		}
		std::vector<std::thread> pool;
		const size_t chunk = (count + threads - 1) / threads;
		for (int t = 0; t < threads; t++) {
			const size_t a = std::min(count, t * chunk), b = std::min(count, a + chunk);
			if (a < b) pool.emplace_back(body, a, b);
		}
		for (auto& th: pool) th.join();
	}

	// copy of a ghost from its inward neighbour (mhd/boundaries.hpp:818-1030)
	MHD copy_of(const MHD& src) const
	{
		const double g = cfg.adiabatic_index, mu0 = cfg.vacuum_permeability;
		MHD out;
		out.rho = src.rho / 1.0;
		const Vec3 v = get_velocity(src.mom, src.rho);
		for (int i = 0; i < 3; i++) out.mom[i] = out.rho * v[i];
		out.mag = src.mag;
		const double p = get_pressure(src.rho, src.mom, src.nrj, src.mag, g, mu0) / 1.0;
		out.nrj = get_total_energy_density(out.rho, get_velocity(out.mom, out.rho), p, out.mag, g, mu0);
		return out;
	}

	void apply_boundaries()
	{
		for (size_t idx = 0; idx < U.size(); idx++) {
			if (CType[idx] != 0) continue;
			int c[3];
			coords(idx, c);
			int d = 0, outside = 0;
			while (c[d] >= 0 and c[d] < n[d]) d++;
			for (int e = 0; e < 3; e++) outside += (c[e] < 0 or c[e] >= n[e]) ? 1 : 0;
			// edge and vertex cells of the staggered grid's layer (class 0 there) are its own to fill
			if (outside > 1) continue;
			const bool lo = c[d] < 0;
			const int kind = lo ? cfg.bc_lo[d] : cfg.bc_hi[d];
			if (kind == PAMHD_BC_VALUE) {
				const double* v = value_of(d, lo);
				MHD& u = U[idx];
				u.rho = v[0];
				u.mom = {v[1], v[2], v[3]};
				u.nrj = v[4];
				u.mag = {v[5], v[6], v[7]};
			} else {
				int m[3] = {c[0], c[1], c[2]};
				m[d] = lo ? 0 : n[d] - 1;
				U[idx] = copy_of(U[index(m[0], m[1], m[2])]);
			}
		}
	}

	// minimize_timestep + set_minmax_substepping_period, no substeps
	double timestep(const double max_dt)
	{
		const double cfl = cfg.time_step_factor;
		parallel(U.size(), [&](size_t a, size_t b) {
			for (size_t idx = a; idx < b; idx++) {
				if (CType[idx] < 0) continue;
				int c[3];
				coords(idx, c);
				double t = std::numeric_limits<double>::max();
				bool zero = false;
				for (int d = 0; d < 3; d++) {
					const int64_t up = plus_neighbor(c, d), down = minus_neighbor(c, d);
					if (up >= 0 and CType[up] >= 0) {
						const double v = std::max(Max_v[idx][2 * d + 1], Max_v[up][2 * d]);
						if (v <= 0) zero = true; else t = std::min(cfl * cfg.cell_length[d] / v, t);
					}
					if (down >= 0 and CType[down] >= 0) {
						const double v = std::max(Max_v[down][2 * d + 1], Max_v[idx][2 * d]);
						if (v <= 0) zero = true; else t = std::min(cfl * cfg.cell_length[d] / v, t);
					}
				}
				Timestep[idx] = zero ? 0.0 : t;
			}
		});
		double smallest = std::numeric_limits<double>::max();
		for (size_t idx = 0; idx < U.size(); idx++) {
			if (CType[idx] >= 0) smallest = std::min(Timestep[idx], smallest);
		}
		return (max_dt <= smallest) ? max_dt : smallest;
	}

	// the solve of one face in the frame of dimension d (mhd/solve.hpp:80-188)
	Face_Flux solve_face(const MHD& a, const MHD& b, const int d) const
	{
		MHD neg = a, pos = b;
		neg.mom = get_rotated_vector(a.mom, d + 1);
		neg.mag = get_rotated_vector(a.mag, d + 1);
		pos.mom = get_rotated_vector(b.mom, d + 1);
		pos.mag = get_rotated_vector(b.mag, d + 1);
		const Vec3 bg{0, 0, 0};
		Face_Flux r = flux(cfg.solver, neg, pos, bg, cfg.adiabatic_index, cfg.vacuum_permeability);
		r.flux.mom = get_rotated_vector(r.flux.mom, -(d + 1));
		r.flux.mag = get_rotated_vector(r.flux.mag, -(d + 1));
		return r;
	}

	// one step; returns dt taken; throws Domain_Error at the first failing face
	double step(const double max_dt)
	{
		return step_with(timestep(max_dt));
	}

	/*
	One step with a given dt instead of the CFL rule (a frozen dt schedule, for
	the perturbed runs that check the GPU adjoint); the face speeds are still
	recorded as in step().
	*/
	double step_with(const double dt)
	{
		failure = Failure();
		std::mutex fail_lock;
		parallel(U.size(), [&](size_t a, size_t b) {
			for (size_t idx = a; idx < b; idx++) {
				if (CType[idx] < 0) continue;
				int c[3];
				coords(idx, c);
				for (int d = 0; d < 3; d++) {
					const int64_t up = plus_neighbor(c, d);
					if (up < 0 or CType[up] < 0) continue;
					Face_Flux r;
					try {
						r = solve_face(U[idx], U[up], d);
					} catch (const Domain_Error& e) {
						std::lock_guard<std::mutex> g(fail_lock);
						const bool first = failure.flag == 0
							or int64_t(idx) < failure.cell
							or (int64_t(idx) == failure.cell and d + 1 < failure.dir);
						if (first) failure = {e.flag, int64_t(idx), d + 1, e.what()};
						continue;
					}
					Max_v[idx][2 * d + 1] = r.speed;
					Max_v[up][2 * d] = r.speed;
					MHD& fc = F[idx][2 * d + 1];
					MHD& fn = F[up][2 * d];
					fc.rho = 0 + dt * r.flux.rho;
					fn.rho = 0 + dt * r.flux.rho;
					fc.nrj = 0 + dt * r.flux.nrj;
					fn.nrj = 0 + dt * r.flux.nrj;
					for (int i = 0; i < 3; i++) {
						fc.mom[i] = 0 + dt * r.flux.mom[i];
						fn.mom[i] = 0 + dt * r.flux.mom[i];
						fc.mag[i] = 0 + dt * r.flux.mag[i];
						fn.mag[i] = 0 + dt * r.flux.mag[i];
					}
				}
			}
		});
		if (failure.flag != 0) {
			throw Domain_Error(failure.flag, failure.what);
		}
		update();
		time += dt;
		apply_boundaries();
		return dt;
	}

	// update_mhd_state, Mode C part (solve.hpp:1543-1602)
	void update()
	{
		double inv_len[3];
		for (int d = 0; d < 3; d++) inv_len[d] = 1 / cfg.cell_length[d];
		parallel(U.size(), [&](size_t a, size_t b) {
			for (size_t idx = a; idx < b; idx++) {
				if (CType[idx] > 0) {
					MHD& u = U[idx];
					const auto& f = F[idx];
					for (int d = 0; d < 3; d++) {
						if (not active[d]) continue;
						u.rho += (f[2 * d].rho - f[2 * d + 1].rho) / cfg.cell_length[d];
					}
					for (int d = 0; d < 3; d++) {
						if (not active[d]) continue;
						for (int i = 0; i < 3; i++) {
							u.mom[i] = u.mom[i] + inv_len[d] * (f[2 * d].mom[i] + (-f[2 * d + 1].mom[i]));
						}
					}
					for (int d = 0; d < 3; d++) {
						if (not active[d]) continue;
						u.nrj += (f[2 * d].nrj - f[2 * d + 1].nrj) / cfg.cell_length[d];
					}
					for (int d = 0; d < 3; d++) {
						if (not active[d]) continue;
						for (int i = 0; i < 3; i++) {
							u.mag[i] = u.mag[i] + inv_len[d] * (f[2 * d].mag[i] + (-f[2 * d + 1].mag[i]));
						}
					}
				}
				F[idx] = {};
			}
		});
	}
};

/*
tests/mhd/reference.cpp, restated: 1-D grid of `cells` cells (the first and
last are the fixed boundary cells), x in [0, length], the SI Brio-Wu-like
tube of its initialize_mhd (:189-265), stepped with CFL 0.5 and the lagged
rule time_step = min(CFL * max_dt, until_end) (:833-843) until t_end.
Returns the number of steps; `out` receives cells * 8 values
(rho, mom, E, B) as the program's save_mhd writes them (:596-616).
*/
template <class Flux>
int reference_1d(const Flux& flux, const int solver, const int cells, const double t_end,
                 const double length, double* out)
{
	const double gamma = 5.0 / 3.0, mu0 = 4e-7 * M_PI, proton_mass = 1.672621777e-27;
	const double cell_size = length / cells;
	std::vector<MHD> U(cells), Fl(cells);
	std::vector<Vec3> Bflux(cells, Vec3{0, 0, 0});
	std::vector<Vec3> E(cells, Vec3{0, 0, 0});
	for (int c = 0; c < cells; c++) {
		MHD& u = U[c];
		const double center = (0.5 + c) * cell_size;
		double p;
		u.mag = {1.5e-9, 0, 0};
		if (center < length / 2) {
			u.rho = proton_mass * 3e6;
			u.mag[1] = 1e-9;
			p = 3e-12;
		} else {
			u.rho = proton_mass * 1e6;
			u.mag[1] = -1e-9;
			p = 1e-12;
		}
		if (cells % 2 == 0 and c == cells / 2 - 1) u.mag[1] = 0;
		if (cells % 2 == 1 and c == cells / 2) {
			u.rho = proton_mass * 2e6;
			p = 2e-12;
		}
		u.nrj = get_total_energy_density(u.rho, u.mom, p, u.mag, gamma, mu0);
	}

	double max_dt = 0, time = 0;
	int steps = 0;
	while (time < t_end) {
		const double cfl = 0.5, until_end = t_end - time;
		const double dt = std::min(cfl * max_dt, until_end);
		max_dt = std::numeric_limits<double>::max();
		const double area = 1.0;
		for (int c = 0; c < cells - 1; c++) {
			MHD& a = U[c];
			MHD& b = U[c + 1];
			Face_Flux r = flux(solver, a, b, Vec3{0, 0, 0}, gamma, mu0);
			r.flux.rho *= area * dt;
			for (int i = 0; i < 3; i++) r.flux.mom[i] = r.flux.mom[i] * (area * dt);
			r.flux.nrj *= area * dt;
			max_dt = std::min(max_dt, cell_size / r.speed);
			if (c > 0) {
				Fl[c].rho -= r.flux.rho;
				for (int i = 0; i < 3; i++) Fl[c].mom[i] = Fl[c].mom[i] + (-r.flux.mom[i]);
				Fl[c].nrj -= r.flux.nrj;
			}
			if (c < cells - 2) {
				Fl[c + 1].rho += r.flux.rho;
				for (int i = 0; i < 3; i++) Fl[c + 1].mom[i] = Fl[c + 1].mom[i] + r.flux.mom[i];
				Fl[c + 1].nrj += r.flux.nrj;
			}
			// upwind E = -v x B (reference.cpp:393-413)
			const double ia = 1 / a.rho, ib = 1 / b.rho;
			const Vec3 vc{a.mom[0] * ia, a.mom[1] * ia, a.mom[2] * ia};
			const Vec3 vn{b.mom[0] * ib, b.mom[1] * ib, b.mom[2] * ib};
			E[c][0] = 0;
			if (vc[0] + vn[0] > 0) {
				E[c][1] = vc[0] * a.mag[2] - vc[2] * a.mag[0];
				E[c][2] = vc[1] * a.mag[0] - vc[0] * a.mag[1];
			} else {
				E[c][1] = vn[0] * b.mag[2] - vn[2] * a.mag[0];
				E[c][2] = vn[1] * a.mag[0] - vn[0] * b.mag[1];
			}
			Vec3& bf = Bflux[c];
			bf = {0, E[c][2], -E[c][1]};
			if (c > 0) {
				bf[1] -= E[c - 1][2];
				bf[2] += E[c - 1][1];
			}
			for (int i = 0; i < 3; i++) bf[i] = bf[i] * dt;
		}
		const double inverse_volume = 1.0 / (area * cell_size);
		for (int c = 0; c < cells; c++) {
			MHD f = Fl[c];
			f.mag = Bflux[c];
			apply_fluxes(U[c], f, inverse_volume, gamma, mu0);
			Fl[c] = MHD();
			Bflux[c] = {0, 0, 0};
		}
		time += dt;
		steps++;
	}
	for (int c = 0; c < cells; c++) {
		const MHD& u = U[c];
		const double row[8] = {u.rho, u.mom[0], u.mom[1], u.mom[2], u.nrj, u.mag[0], u.mag[1], u.mag[2]};
		std::memcpy(out + 8 * size_t(c), row, sizeof row);
	}
	return steps;
}

} // namespace oracle

#endif
