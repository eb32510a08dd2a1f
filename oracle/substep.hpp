/*
CPU oracle, L3: the cell-centred step with local time stepping (substeps).

TEST INFRASTRUCTURE - see mhd_oracle.hpp for who may use this.

The reference's timestep() (mhd/solve.hpp:1837-1924) lets cells advance
with periods of 2^k substeps of one common substep length:
  - set_minmax_substepping_period with the options (substepping.hpp:
    195-257): every cell's smallest and largest exponent (the caller's
    substep-min / substep-max, evaluated per cell), the smallest minimum
    subtracted from all minima when it is above 0;
  - minimize_timestep (mhd/solve.hpp:1933-2007): each cell's CFL limit from
    the previous step's face speeds;
  - set_minmax_substepping_period with the limits (substepping.hpp:
    259-394): if max_dt is at most the smallest limit, every exponent is 0
    and the substep is max_dt; else the substep is the smallest
    limit / 2^min over cells, and each cell's largest exponent drops to
    floor(log2(min(limit, max_dt) / substep));
  - restrict_substepping_period (substepping.hpp:104-176): a cell's exponent
    is at most 1 above any face or edge neighbour's (the largest such
    assignment, reached by repeated passes);
  - update_substeps (:58-98): periods 2^exponent, the step has as many
    substeps as the largest period;
  - per substep s: get_fluxes (mhd/solve.hpp:254-392) solves a cell's +d faces
    when s is a multiple of the smallest period among the cell and its face
    and edge neighbours, M, and adds (substep M) F to both sides' flux slots;
    update_mhd_state (:1543-1602) updates the cells whose period divides s
    and zeroes their slots; the other cells keep accumulating.
The step's length is the substep added once per substep.  Grids periodic in
every dimension; dimensions of one cell are inactive (the reference's
one-cell periodic dimension makes a cell its own neighbour, which neither
changes a period minimum nor the update).
*/
#ifndef PAMHD_ORACLE_SUBSTEP_HPP
#define PAMHD_ORACLE_SUBSTEP_HPP

#include <cmath>

#include "mode_c.hpp"

namespace oracle {

template <class Flux> class Substep_Grid : public Mode_C_Grid<Flux> {
public:
	using Base = Mode_C_Grid<Flux>;
	using Base::cfg;
	using Base::n;
	using Base::U;
	using Base::F;
	using Base::Max_v;
	using Base::Timestep;
	using Base::active;
	using Base::failure;
	using Base::time;

	std::vector<int> user_min, user_max;   // the options' exponents per cell
	std::vector<int> S;                    // exponents of the current step
	std::vector<int> period;               // 2^S
	int max_substep = 1;
	double substep = 0;

	explicit Substep_Grid(const pamhd_cfg& c) : Base(c)
	{
		for (int d = 0; d < 3; d++) {
			if (cfg.bc_lo[d] != PAMHD_BC_PERIODIC or cfg.bc_hi[d] != PAMHD_BC_PERIODIC) {
				throw std::invalid_argument("local time stepping needs a periodic grid");
			}
		}
		user_min.assign(U.size(), 0);
		user_max.assign(U.size(), 0);
		S.assign(U.size(), 0);
		period.assign(U.size(), 1);
	}

	size_t at(int i, int j, int k) const
	{
		i = (i % n[0] + n[0]) % n[0];
		j = (j % n[1] + n[1]) % n[1];
		k = (k % n[2] + n[2]) % n[2];
		return this->index(i, j, k);
	}

	void set_exponents(const int32_t* mins, const int32_t* maxs)
	{
		for (size_t c = 0; c < U.size(); c++) {
			if (mins[c] < 0 or maxs[c] < 0 or mins[c] > 30 or maxs[c] > 30) {
				throw std::invalid_argument("substep exponents must be in 0 .. 30");
			}
			user_min[c] = mins[c];
			user_max[c] = maxs[c];
		}
	}

	// the face and edge neighbours of a cell in the active dimensions
	template <class Body> void for_neighbours(const size_t c, Body body) const
	{
		int p[3];
		this->coords(c, p);
		for (int dz = -1; dz <= 1; dz++)
		for (int dy = -1; dy <= 1; dy++)
		for (int dx = -1; dx <= 1; dx++) {
			const int o[3] = {dx, dy, dz};
			int nonzero = 0;
			bool ok = true;
			for (int d = 0; d < 3; d++) {
				if (o[d] != 0) {
					nonzero++;
					if (not active[d]) ok = false;
				}
			}
			if (not ok or nonzero == 0 or nonzero == 3) continue;
			body(at(p[0] + dx, p[1] + dy, p[2] + dz));
		}
	}

	// the exponents and the substep of a step capped by max_dt (substepping.hpp:195-394)
	void plan(const double max_dt)
	{
		this->timestep(std::numeric_limits<double>::max());  // fills Timestep[] (minimize_timestep)
		plan_from_limits(max_dt);
	}

	// the same from given CFL limits, one per cell (the reference functions' pin)
	void plan_from_limits(const double* limits, const double max_dt)
	{
		for (size_t c = 0; c < U.size(); c++) Timestep[c] = limits[c];
		plan_from_limits(max_dt);
	}

	// the plan from the limits in Timestep[]
	void plan_from_limits(const double max_dt)
	{
		const size_t N = U.size();
		std::vector<int> smin(user_min), smax(user_max);
		int lowest = std::numeric_limits<int>::max();
		for (size_t c = 0; c < N; c++) lowest = std::min(smin[c], lowest);
		if (lowest > 0) {
			for (size_t c = 0; c < N; c++) smin[c] -= lowest;
		}
		double smallest = std::numeric_limits<double>::max();
		for (size_t c = 0; c < N; c++) smallest = std::min(Timestep[c], smallest);
		if (max_dt <= smallest) {
			for (size_t c = 0; c < N; c++) smin[c] = smax[c] = 0;
			substep = max_dt;
		} else {
			double ret = std::numeric_limits<double>::max();
			for (size_t c = 0; c < N; c++) ret = std::min(ret, Timestep[c] / (1 << smin[c]));
			for (size_t c = 0; c < N; c++) {
				const double dt = Timestep[c];
				if (dt > 0) {
					const int step = std::max(0, int(std::floor(std::log2(std::min(dt, max_dt) / ret))));
					if (smax[c] > step) smax[c] = step;
					if (smin[c] > smax[c]) throw std::runtime_error("unexpected substeps");
				} else {
					smin[c] = smax[c] = 0;
				}
			}
			substep = ret;
		}
		// restrict_substepping_period
		S = smax;
		bool modified = true;
		while (modified) {
			modified = false;
			for (size_t c = 0; c < N; c++) {
				for_neighbours(c, [&](const size_t m) {
					if (S[c] > S[m] + 1) {
						S[c] = S[m] + 1;
						modified = true;
					}
				});
			}
		}
		max_substep = 1;
		for (size_t c = 0; c < N; c++) {
			period[c] = 1 << S[c];
			max_substep = std::max(period[c], max_substep);
		}
	}

	// one step (timestep() with substeps); returns its length
	double step(const double max_dt)
	{
		plan(max_dt);
		const size_t N = U.size();
		std::vector<int> M(N);
		for (size_t c = 0; c < N; c++) {
			int m = period[c];
			for_neighbours(c, [&](const size_t q) { m = std::min(m, period[q]); });
			M[c] = m;
		}
		failure = Failure();
		double total = 0;
		for (int s = 1; s <= max_substep; s++) {
			total += substep;
			for (size_t c = 0; c < N; c++) {
				if (s % M[c] != 0) continue;
				int p[3];
				this->coords(c, p);
				const double min_dt = substep * M[c];
				for (int d = 0; d < 3; d++) {
					if (not active[d]) continue;
					const size_t up = at(p[0] + (d == 0), p[1] + (d == 1), p[2] + (d == 2));
					Face_Flux r;
					try {
						r = this->solve_face(U[c], U[up], d);
					} catch (const Domain_Error& e) {
						if (failure.flag == 0) failure = {e.flag, int64_t(c), d + 1, e.what()};
						continue;
					}
					Max_v[c][2 * d + 1] = r.speed;
					Max_v[up][2 * d] = r.speed;
					MHD& fc = F[c][2 * d + 1];
					MHD& fn = F[up][2 * d];
					fc.rho += min_dt * r.flux.rho;
					fn.rho += min_dt * r.flux.rho;
					fc.nrj += min_dt * r.flux.nrj;
					fn.nrj += min_dt * r.flux.nrj;
					for (int v = 0; v < 3; v++) {
						fc.mom[v] = fc.mom[v] + min_dt * r.flux.mom[v];
						fn.mom[v] = fn.mom[v] + min_dt * r.flux.mom[v];
						fc.mag[v] = fc.mag[v] + min_dt * r.flux.mag[v];
						fn.mag[v] = fn.mag[v] + min_dt * r.flux.mag[v];
					}
				}
			}
			if (failure.flag != 0) throw Domain_Error(failure.flag, failure.what);
			update(s);
		}
		time += total;
		return total;
	}

	// update_mhd_state for the cells whose period divides s (mhd/solve.hpp:1543-1602)
	void update(const int s)
	{
		double inv_len[3];
		for (int d = 0; d < 3; d++) inv_len[d] = 1 / cfg.cell_length[d];
		for (size_t c = 0; c < U.size(); c++) {
			if (s % period[c] != 0) continue;
			MHD& u = U[c];
			auto& f = F[c];
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
			f = {};
		}
	}
};

} // namespace oracle

#endif
