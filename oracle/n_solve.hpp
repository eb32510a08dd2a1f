/*
CPU oracle, L3: the two-population ("N") MHD step.

TEST INFRASTRUCTURE - see mhd_oracle.hpp for who may use this.

Two fluid populations share one magnetic field.  A face is solved for the
total state (the populations' mass, momentum and energy summed, the shared
field) with a split solver that returns the flux leaving the negative side
and the flux entering from the positive side separately, already scaled by
area and dt:
  - get_flux_N_rusanov (mhd/N_rusanov.hpp:61-170);
  - get_flux_N_hll (mhd/N_hll_athena.hpp:47-231), including two
    statements of the reference kept as it computes them: the positive
    side's momentum flux is scaled a second time by its factor, and its
    field flux is left as the unscaled physical flux (:224-227);
both on N_get_flux (mhd/common.hpp:500-549, the physical flux of each side).
Each side's mass, momentum and energy flux is shared between the
populations by that side's mass fractions; the field flux is the sum of
the two sides' (mhd/N_solve.hpp:354-437).

reference_2pop_1d() restates tests/mhd/two_reference.cpp (its grid,
initialize_mhd :220-289, solve_mhd :297-477, the time loop and
apply_fluxes_N of mhd/common.hpp:743-780), the scheme of the reference's
golden files tests/mhd/2mhd_*.ref.

N_Grid restates N_solve + apply_fluxes_N (mhd/N_solve.hpp:79-446, :457-587)
on a uniform grid periodic in every dimension (dimensions of one cell have
no faces): every face is solved once, its contributions added to its two
cells in the fixed order -x, +x, -y, +y, -z, +z of each cell's faces; each
population's state += flux / volume; where the total thermal pressure falls
below min_pressure, the total energy is reset to that pressure and shared
by mass fraction.  step(dt) returns the largest dt the faces allow for the
next step, min over faces of d_len / max_signal (mhd/N_solve.hpp:345).
*/
#ifndef PAMHD_ORACLE_N_SOLVE_HPP
#define PAMHD_ORACLE_N_SOLVE_HPP

#include <limits>
#include <tuple>
#include <vector>

#include "mode_c.hpp"

namespace oracle {

struct Split_Flux {
	MHD neg, pos;
	double speed = 0;
};

// mhd/N_rusanov.hpp:61-170
inline Split_Flux get_flux_N_rusanov(const MHD& L, const MHD& R, const Vec3& bg, const double area,
                                     const double dt, const double gamma, const double mu0)
{
	if (not std::isnormal(L.rho) or L.rho < 0) {
		throw Domain_Error(PAMHD_FLAG_DENSITY, "Invalid mass density in state_neg");
	}
	if (not std::isnormal(R.rho) or R.rho < 0) {
		throw Domain_Error(PAMHD_FLAG_DENSITY, "Invalid mass density in state_pos");
	}
	const double
		fast_neg = get_fast_magnetosonic_speed(L.rho, L.mom, L.nrj, L.mag, bg, gamma, mu0),
		fast_pos = get_fast_magnetosonic_speed(R.rho, R.mom, R.nrj, R.mag, bg, gamma, mu0),
		max_fast = std::max(fast_neg, fast_pos),
		s = std::max(std::abs(get_velocity(L.mom, L.rho)[0]) + max_fast,
		             std::abs(get_velocity(R.mom, R.rho)[0]) + max_fast);
	MHD fn = get_flux(L, bg, gamma, mu0);
	MHD fp = get_flux(R, bg, gamma, mu0);
	const double c = 0.5 * area * dt;
	Split_Flux out;
	out.neg.rho = c * (fn.rho + L.rho * s);
	for (int i = 0; i < 3; i++) out.neg.mom[i] = c * (fn.mom[i] + L.mom[i] * s);
	out.neg.nrj = c * (fn.nrj + L.nrj * s);
	for (int i = 0; i < 3; i++) out.neg.mag[i] = c * (fn.mag[i] + L.mag[i] * s);
	out.pos.rho = c * (fp.rho - R.rho * s);
	for (int i = 0; i < 3; i++) out.pos.mom[i] = c * (fp.mom[i] + R.mom[i] * -s);
	out.pos.nrj = c * (fp.nrj - R.nrj * s);
	for (int i = 0; i < 3; i++) out.pos.mag[i] = c * (fp.mag[i] + R.mag[i] * -s);
	out.speed = s;
	return out;
}

// mhd/N_hll_athena.hpp:47-231
inline Split_Flux get_flux_N_hll(const MHD& L, const MHD& R, const Vec3& bg, const double area,
                                 const double dt, const double gamma, const double mu0)
{
	const Vec3 vn = get_velocity(L.mom, L.rho), vp = get_velocity(R.mom, R.rho);
	const double
		p_neg = get_pressure(L.rho, L.mom, L.nrj, L.mag, gamma, mu0),
		p_pos = get_pressure(R.rho, R.mom, R.nrj, R.mag, gamma, mu0),
		pb_neg = (L.mag[0] * L.mag[0] + L.mag[1] * L.mag[1] + L.mag[2] * L.mag[2]) / (2 * mu0),
		pb_pos = (R.mag[0] * R.mag[0] + R.mag[1] * R.mag[1] + R.mag[2] * R.mag[2]) / (2 * mu0),
		fast_neg = get_fast_magnetosonic_speed(L.rho, L.mom, L.nrj, L.mag, bg, gamma, mu0),
		fast_pos = get_fast_magnetosonic_speed(R.rho, R.mom, R.nrj, R.mag, bg, gamma, mu0),
		max_signal = std::max(fast_neg, fast_pos),
		s_neg = (vn[0] <= vp[0]) ? vn[0] - max_signal : vp[0] - max_signal,
		s_pos = (vn[0] <= vp[0]) ? vp[0] + max_signal : vn[0] + max_signal,
		bm = std::min(s_neg, 0.0),
		bp = std::max(s_pos, 0.0);
	if (not std::isnormal(p_neg) or p_neg < 0) {
		throw Domain_Error(PAMHD_FLAG_PRESSURE, "Invalid thermal pressure in state_neg");
	}
	if (not std::isfinite(pb_neg) or pb_neg < 0) {
		throw Domain_Error(PAMHD_FLAG_PRESSURE, "Invalid magnetic pressure in state_neg");
	}
	if (not std::isfinite(s_neg)) {
		throw Domain_Error(PAMHD_FLAG_WAVE_SPEED, "Invalid max signal speed in state_neg");
	}
	if (not std::isnormal(p_pos) or p_pos < 0) {
		throw Domain_Error(PAMHD_FLAG_PRESSURE, "Invalid thermal pressure in state_pos");
	}
	if (not std::isfinite(pb_pos) or pb_pos < 0) {
		throw Domain_Error(PAMHD_FLAG_PRESSURE, "Invalid magnetic pressure in state_pos");
	}
	if (not std::isfinite(s_pos)) {
		throw Domain_Error(PAMHD_FLAG_WAVE_SPEED, "Invalid max signal speed in state_pos");
	}
	Split_Flux out;
	if (not std::isnormal(bp - bm) or bp - bm < 0) {
		return out;   // zero fluxes and speed
	}
	MHD fn = get_flux(L, bg, gamma, mu0);
	MHD fp = get_flux(R, bg, gamma, mu0);
	const double
		neg_factor = bp / (bp - bm) * area * dt,
		pos_factor = bm / (bm - bp) * area * dt;
	out.neg.rho = neg_factor * (fn.rho - L.rho * bm);
	for (int i = 0; i < 3; i++) out.neg.mom[i] = neg_factor * (fn.mom[i] + L.mom[i] * -bm);
	out.neg.nrj = neg_factor * (fn.nrj - L.nrj * bm);
	for (int i = 0; i < 3; i++) out.neg.mag[i] = neg_factor * (fn.mag[i] + L.mag[i] * -bm);
	out.pos.rho = pos_factor * (fp.rho - R.rho * bp);
	for (int i = 0; i < 3; i++) out.pos.mom[i] = pos_factor * (fp.mom[i] + R.mom[i] * -bp);
	out.pos.nrj = pos_factor * (fp.nrj - R.nrj * bp);
	// the reference scales the positive side's momentum flux again and keeps its field flux unscaled
	for (int i = 0; i < 3; i++) out.pos.mom[i] = pos_factor * (out.pos.mom[i] + R.mom[i] * -bp);
	out.pos.mag = fp.mag;
	out.speed = std::max(std::fabs(bp), std::fabs(bm));
	return out;
}

// the split solver of a solver id (PAMHD_RUSANOV or PAMHD_HLL_ATHENA)
struct Restated_Split_Solvers {
	Split_Flux operator()(const int solver, const MHD& L, const MHD& R, const Vec3& bg, const double area,
	                      const double dt, const double gamma, const double mu0) const
	{
		if (solver == PAMHD_RUSANOV) return get_flux_N_rusanov(L, R, bg, area, dt, gamma, mu0);
		if (solver == PAMHD_HLL_ATHENA) return get_flux_N_hll(L, R, bg, area, dt, gamma, mu0);
		throw std::invalid_argument("the two-population step has Rusanov and HLL only");
	}
};

// the two populations and the shared field of a cell
struct Two_Pop {
	double rho1 = 0, rho2 = 0, nrj1 = 0, nrj2 = 0;
	Vec3 mom1{0, 0, 0}, mom2{0, 0, 0}, mag{0, 0, 0};
};

// one face's contribution to each population and to the field (mhd/N_solve.hpp:354-382)
struct Two_Pop_Flux {
	double rho1 = 0, rho2 = 0, nrj1 = 0, nrj2 = 0;
	Vec3 mom1{0, 0, 0}, mom2{0, 0, 0}, mag{0, 0, 0};
};

inline MHD total_state(const Two_Pop& c)
{
	MHD s;
	s.rho = c.rho1 + c.rho2;
	for (int i = 0; i < 3; i++) s.mom[i] = c.mom1[i] + c.mom2[i];
	s.nrj = c.nrj1 + c.nrj2;
	s.mag = c.mag;
	return s;
}

/*
The populations' shares of a split face flux (mhd/N_solve.hpp:354-382 and
tests/mhd/two_reference.cpp:417-475): population k receives
frac_k,neg * flux_neg + frac_k,pos * flux_pos, frac the mass fractions of
the face's negative and positive cells; the field receives
flux_neg + flux_pos.
*/
inline Two_Pop_Flux share(const Split_Flux& f, const Two_Pop& a, const Two_Pop& b)
{
	const double
		f1n = a.rho1 / (a.rho1 + a.rho2), f2n = a.rho2 / (a.rho1 + a.rho2),
		f1p = b.rho1 / (b.rho1 + b.rho2), f2p = b.rho2 / (b.rho1 + b.rho2);
	Two_Pop_Flux o;
	o.rho1 = f1n * f.neg.rho + f1p * f.pos.rho;
	o.rho2 = f2n * f.neg.rho + f2p * f.pos.rho;
	o.nrj1 = f1n * f.neg.nrj + f1p * f.pos.nrj;
	o.nrj2 = f2n * f.neg.nrj + f2p * f.pos.nrj;
	for (int i = 0; i < 3; i++) {
		o.mom1[i] = f1n * f.neg.mom[i] + f1p * f.pos.mom[i];
		o.mom2[i] = f2n * f.neg.mom[i] + f2p * f.pos.mom[i];
		o.mag[i] = f.neg.mag[i] + f.pos.mag[i];
	}
	return o;
}

/*
tests/mhd/two_reference.cpp restated: cells cells on x in [0, length]
(the first and last are fixed), SI units, gamma 5/3, mu0 4 pi 1e-7,
Bx 1.5e-9; population 1 (3e6 protons/m^3, By 1e-9, p 3e-12) fills the left
half, population 2 (1e6 protons/m^3, By -1e-9, p 1e-12) the right half,
each with the other population absent; the lagged rule
dt = min(CFL max_dt, until_end), CFL 0.5, until t_end.  out receives
cells x 13 values: rho1, mom1 xyz, E1, rho2, mom2 xyz, E2, B xyz.
Returns the number of steps.
*/
template <class Split>
int reference_2pop_1d(const Split& split, const int solver, const int cells, const double t_end,
                      const double length, double* out)
{
	const double gamma = 5.0 / 3.0, mu0 = 4e-7 * M_PI, proton_mass = 1.672621777e-27;
	const double cell_size = length / cells;
	std::vector<Two_Pop> U(cells);
	std::vector<Two_Pop_Flux> Fl(cells);
	for (int c = 0; c < cells; c++) {
		Two_Pop& u = U[c];
		u.mag = {1.5e-9, 0, 0};
		const double center = (0.5 + c) * cell_size;
		if (center < length / 2) {
			u.rho1 = proton_mass * 3e6;
			u.mag[1] = 1e-9;
			u.nrj1 = get_total_energy_density(u.rho1, u.mom1, 3e-12, u.mag, gamma, mu0);
		} else {
			u.rho2 = proton_mass * 1e6;
			u.mag[1] = -1e-9;
			u.nrj2 = get_total_energy_density(u.rho2, u.mom2, 1e-12, u.mag, gamma, mu0);
		}
	}
	double max_dt = 0, time = 0;
	int steps = 0;
	while (time < t_end) {
		const double cfl = 0.5, until_end = t_end - time;
		const double dt = std::min(cfl * max_dt, until_end);
		max_dt = std::numeric_limits<double>::max();
		double step_max = std::numeric_limits<double>::max();
		for (int c = 0; c < cells - 1; c++) {
			const Two_Pop& a = U[c];
			const Two_Pop& b = U[c + 1];
			const Split_Flux f = split(solver, total_state(a), total_state(b), Vec3{0, 0, 0}, 1.0, dt, gamma, mu0);
			step_max = std::min(step_max, cell_size / f.speed);
			const double
				f1n = a.rho1 / (a.rho1 + a.rho2), f2n = a.rho2 / (a.rho1 + a.rho2),
				f1p = b.rho1 / (b.rho1 + b.rho2), f2p = b.rho2 / (b.rho1 + b.rho2);
			if (c > 0) {
				Two_Pop_Flux& o = Fl[c];
				for (int i = 0; i < 3; i++) o.mag[i] = o.mag[i] + -(f.neg.mag[i] + f.pos.mag[i]);
				o.rho1 -= f1n * f.neg.rho + f1p * f.pos.rho;
				for (int i = 0; i < 3; i++) o.mom1[i] = o.mom1[i] + -(f1n * f.neg.mom[i] + f1p * f.pos.mom[i]);
				o.nrj1 -= f1n * f.neg.nrj + f1p * f.pos.nrj;
				o.rho2 -= f2n * f.neg.rho + f2p * f.pos.rho;
				for (int i = 0; i < 3; i++) o.mom2[i] = o.mom2[i] + -(f2n * f.neg.mom[i] + f2p * f.pos.mom[i]);
				o.nrj2 -= f2n * f.neg.nrj + f2p * f.pos.nrj;
			}
			if (c < cells - 2) {
				Two_Pop_Flux& o = Fl[c + 1];
				for (int i = 0; i < 3; i++) o.mag[i] = (o.mag[i] + f.neg.mag[i]) + f.pos.mag[i];
				o.rho1 += f1n * f.neg.rho + f1p * f.pos.rho;
				for (int i = 0; i < 3; i++) o.mom1[i] = (o.mom1[i] + f1n * f.neg.mom[i]) + f1p * f.pos.mom[i];
				o.nrj1 += f1n * f.neg.nrj + f1p * f.pos.nrj;
				o.rho2 += f2n * f.neg.rho + f2p * f.pos.rho;
				for (int i = 0; i < 3; i++) o.mom2[i] = (o.mom2[i] + f2n * f.neg.mom[i]) + f2p * f.pos.mom[i];
				o.nrj2 += f2n * f.neg.nrj + f2p * f.pos.nrj;
			}
		}
		max_dt = std::min(max_dt, step_max);
		const double inverse_volume = 1.0 / (1.0 * cell_size);
		for (int c = 0; c < cells; c++) {
			Two_Pop& u = U[c];
			Two_Pop_Flux& o = Fl[c];
			for (int i = 0; i < 3; i++) u.mag[i] = u.mag[i] + o.mag[i] * inverse_volume;
			u.rho1 += o.rho1 * inverse_volume;
			for (int i = 0; i < 3; i++) u.mom1[i] = u.mom1[i] + o.mom1[i] * inverse_volume;
			u.nrj1 += o.nrj1 * inverse_volume;
			u.rho2 += o.rho2 * inverse_volume;
			for (int i = 0; i < 3; i++) u.mom2[i] = u.mom2[i] + o.mom2[i] * inverse_volume;
			u.nrj2 += o.nrj2 * inverse_volume;
			o = Two_Pop_Flux();
		}
		time += dt;
		steps++;
	}
	for (int c = 0; c < cells; c++) {
		const Two_Pop& u = U[c];
		const double row[13] = {u.rho1, u.mom1[0], u.mom1[1], u.mom1[2], u.nrj1,
		                        u.rho2, u.mom2[0], u.mom2[1], u.mom2[2], u.nrj2,
		                        u.mag[0], u.mag[1], u.mag[2]};
		for (int v = 0; v < 13; v++) out[13 * size_t(c) + v] = row[v];
	}
	return steps;
}

/*
N_solve + apply_fluxes_N on a uniform grid periodic in every dimension (see
the file comment).  Cells x fastest; dimensions of one cell are inactive.
*/
template <class Split> class N_Grid {
public:
	int n[3];
	bool active[3];
	double len[3];
	int solver;
	double gamma, mu0, min_pressure;
	Split split;
	std::vector<Two_Pop> U;
	std::vector<Two_Pop_Flux> X[3];   // contribution of every cell's -d face
	Failure failure;

	N_Grid(const int nx, const int ny, const int nz, const double lx, const double ly, const double lz,
	       const int solver_, const double gamma_, const double mu0_, const double min_pressure_)
		: n{nx, ny, nz}, len{lx, ly, lz}, solver(solver_), gamma(gamma_), mu0(mu0_), min_pressure(min_pressure_)
	{
		if (solver != PAMHD_RUSANOV and solver != PAMHD_HLL_ATHENA) {
			throw std::invalid_argument("the two-population step has Rusanov and HLL only");
		}
		for (int d = 0; d < 3; d++) {
			if (n[d] < 1 or not (len[d] > 0)) throw std::invalid_argument("grid size");
			active[d] = n[d] > 1;
		}
		const size_t N = size_t(n[0]) * n[1] * n[2];
		U.resize(N);
		for (int d = 0; d < 3; d++) X[d].assign(N, Two_Pop_Flux());
	}

	size_t at(int i, int j, int k) const
	{
		i = (i % n[0] + n[0]) % n[0];
		j = (j % n[1] + n[1]) % n[1];
		k = (k % n[2] + n[2]) % n[2];
		return size_t(i) + size_t(n[0]) * (size_t(j) + size_t(n[1]) * k);
	}

	// the solve of the face between cell a (negative side) and b along axis d (mhd/N_solve.hpp:204-352)
	Split_Flux solve(const Two_Pop& a, const Two_Pop& b, const int d, const double area, const double dt) const
	{
		MHD L = total_state(a), R = total_state(b);
		L.mom = get_rotated_vector(L.mom, d + 1);
		L.mag = get_rotated_vector(L.mag, d + 1);
		R.mom = get_rotated_vector(R.mom, d + 1);
		R.mag = get_rotated_vector(R.mag, d + 1);
		Split_Flux f = split(solver, L, R, Vec3{0, 0, 0}, area, dt, gamma, mu0);
		f.neg.mom = get_rotated_vector(f.neg.mom, -(d + 1));
		f.pos.mom = get_rotated_vector(f.pos.mom, -(d + 1));
		f.neg.mag = get_rotated_vector(f.neg.mag, -(d + 1));
		f.pos.mag = get_rotated_vector(f.pos.mag, -(d + 1));
		return f;
	}

	// one step of length dt; returns min over faces of d_len / max_signal (the next step's limit)
	double step(const double dt)
	{
		failure = Failure();
		const double area[3] = {len[1] * len[2], len[0] * len[2], len[0] * len[1]};
		double max_dt = std::numeric_limits<double>::max();
		// each cell's +d faces in cell order, as N_solve visits them (mhd/N_solve.hpp:127-172)
		for (int k = 0; k < n[2]; k++)
		for (int j = 0; j < n[1]; j++)
		for (int i = 0; i < n[0]; i++) {
			const size_t m = at(i, j, k);
			for (int d = 0; d < 3; d++) {
				if (not active[d]) continue;
				const size_t c = at(i + (d == 0), j + (d == 1), k + (d == 2));
				Split_Flux f;
				try {
					f = solve(U[m], U[c], d, area[d], dt);
				} catch (const Domain_Error& e) {
					if (failure.flag == 0) failure = {e.flag, int64_t(m), d + 1, e.what()};
					continue;
				}
				max_dt = std::min(max_dt, len[d] / f.speed);
				X[d][c] = share(f, U[m], U[c]);
			}
		}
		if (failure.flag != 0) throw Domain_Error(failure.flag, failure.what);
		const double inverse_volume = 1.0 / (len[0] * len[1] * len[2]);
		std::vector<Two_Pop> next(U.size());
		for (int k = 0; k < n[2]; k++)
		for (int j = 0; j < n[1]; j++)
		for (int i = 0; i < n[0]; i++) {
			const size_t c = at(i, j, k);
			Two_Pop_Flux f;
			for (int d = 0; d < 3; d++) {
				if (not active[d]) continue;
				const Two_Pop_Flux& lo = X[d][c];
				const Two_Pop_Flux& hi = X[d][at(i + (d == 0), j + (d == 1), k + (d == 2))];
				f.rho1 += lo.rho1; f.rho1 -= hi.rho1;
				f.rho2 += lo.rho2; f.rho2 -= hi.rho2;
				f.nrj1 += lo.nrj1; f.nrj1 -= hi.nrj1;
				f.nrj2 += lo.nrj2; f.nrj2 -= hi.nrj2;
				for (int v = 0; v < 3; v++) {
					f.mom1[v] += lo.mom1[v]; f.mom1[v] -= hi.mom1[v];
					f.mom2[v] += lo.mom2[v]; f.mom2[v] -= hi.mom2[v];
					f.mag[v] += lo.mag[v]; f.mag[v] -= hi.mag[v];
				}
			}
			Two_Pop u = U[c];
			// apply_fluxes_N, mhd/N_solve.hpp:505-546
			u.rho1 += f.rho1 * inverse_volume;
			u.rho2 += f.rho2 * inverse_volume;
			for (int v = 0; v < 3; v++) u.mom1[v] += f.mom1[v] * inverse_volume;
			for (int v = 0; v < 3; v++) u.mom2[v] += f.mom2[v] * inverse_volume;
			u.nrj1 += f.nrj1 * inverse_volume;
			u.nrj2 += f.nrj2 * inverse_volume;
			for (int v = 0; v < 3; v++) u.mag[v] += f.mag[v] * inverse_volume;
			// minimum pressure (:553-583)
			const double total_mass = u.rho1 + u.rho2, total_energy = u.nrj1 + u.nrj2;
			const Vec3 total_mom{u.mom1[0] + u.mom2[0], u.mom1[1] + u.mom2[1], u.mom1[2] + u.mom2[2]};
			const double p = get_pressure(total_mass, total_mom, total_energy, u.mag, gamma, mu0);
			if (not (p >= min_pressure)) {
				const double e = get_total_energy_density(total_mass, get_velocity(total_mom, total_mass),
				                                          min_pressure, u.mag, gamma, mu0);
				u.nrj1 = u.rho1 / total_mass * e;
				u.nrj2 = u.rho2 / total_mass * e;
			}
			next[c] = u;
		}
		U.swap(next);
		return max_dt;
	}

	// 13 arrays of n0 n1 n2 doubles: rho1, mom1 xyz, E1, rho2, mom2 xyz, E2, B xyz
	void set_state(const double* const a[13])
	{
		for (size_t c = 0; c < U.size(); c++) {
			Two_Pop& u = U[c];
			u.rho1 = a[0][c]; u.mom1 = {a[1][c], a[2][c], a[3][c]}; u.nrj1 = a[4][c];
			u.rho2 = a[5][c]; u.mom2 = {a[6][c], a[7][c], a[8][c]}; u.nrj2 = a[9][c];
			u.mag = {a[10][c], a[11][c], a[12][c]};
		}
	}

	void get_state(double* const a[13]) const
	{
		for (size_t c = 0; c < U.size(); c++) {
			const Two_Pop& u = U[c];
			const double row[13] = {u.rho1, u.mom1[0], u.mom1[1], u.mom1[2], u.nrj1,
			                        u.rho2, u.mom2[0], u.mom2[1], u.mom2[2], u.nrj2,
			                        u.mag[0], u.mag[1], u.mag[2]};
			for (int v = 0; v < 13; v++) a[v][c] = row[v];
		}
	}
};

} // namespace oracle

#endif
