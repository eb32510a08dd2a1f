/*
CPU oracle, L3: the staggered-field ("Mode S") MHD step on a uniform,
periodic Cartesian grid.

TEST INFRASTRUCTURE - see mhd_oracle.hpp for who may use this.

The reference's timestep (mhd/solve.hpp:1837-1924) keeps, besides the
cell-centred state, the normal magnetic field of every cell face (Face_B)
and advances it by constrained transport.  Mode_S_Grid<Flux> restates it
for a uniform grid that is periodic in every dimension, where a dimension
of one cell is its own neighbour (the reference's emulated 1-D and 2-D runs
keep those dimensions, tests/mhd/config_files/.../Alfvén_wave):
  - face fluxes and Max_v of every cell's +d faces as Mode C
    (mhd/solve.hpp:217-392), including a cell's face with itself in a
    dimension of one cell;
  - the face-B changes of assign_face_dBs_f{x,y,z} (mhd/solve.hpp:587-1494)
    on equal-size neighbours: a d-directed face flux F gives the edge
    terms E_b = ((F[B_a] dt) L_b) / 4 and E_a = -((F[B_b] dt) L_a) / 4
    (a = d+1, b = d+2 cyclically; :610-612, :925-927, the z form), which
    change the normal field of the faces around the flux face's four edges
    and never the flux face itself.  Every face is stored once here (the
    reference stores both sides' copies and makes them agree in
    sync_magnetic_field, common_functions.hpp:191-269), and its change is
    the sum of its twelve terms in the fixed order of face_dB() below;
  - update_mhd_state (mhd/solve.hpp:1543-1602): the Mode C update of the
    cell state, volume field included, then Face_B += Face_dB / area;
  - update_vol_B with constant thermal pressure (mhd/solve.hpp:1631-1683),
    called twice as timestep() does (inside the substep loop and after
    sync_magnetic_field, :1895-1918): the pressure from the current
    state, the volume field the mean of the cell's two faces per
    dimension, the total energy recomputed from that pressure;
  - the lagged CFL rule and the time cap as Mode C.
Face storage: Bf[d][cell] is the normal field of the cell's -d face; the
+d face of a cell is the -d face of its +d neighbour.

Background field (optional): Bg[d][cell] is the background field vector at
the cell's -d face (the reference's Bg_B of the face, integrated over it at
initialisation, mhd/initialize.hpp:517-530).  The face between a cell and its
+d neighbour is solved with that face's vector, rotated into the face frame
(mhd/solve.hpp:120-121); the solvers use it as the reference's do (Rusanov
and HLL in the flux and the fast speeds, HLLD and Roe not at all).  The cell
state and Face_B hold the field without the background, as in the reference.
*/
#ifndef PAMHD_ORACLE_MODE_S_HPP
#define PAMHD_ORACLE_MODE_S_HPP

#include "mode_c.hpp"

namespace oracle {

template <class Flux> class Mode_S_Grid : public Mode_C_Grid<Flux> {
public:
	using Base = Mode_C_Grid<Flux>;
	using Base::cfg;
	using Base::n;
	using Base::U;
	using Base::F;
	using Base::Max_v;
	using Base::active;
	using Base::failure;
	using Base::time;

	std::vector<double> Bf[3];   // normal field of each cell's -d face
	std::vector<MHD> FF[3];      // raw flux through each cell's -d face, unrotated
	std::vector<Vec3> Bg[3];     // background field at each cell's -d face (empty: none)

	explicit Mode_S_Grid(const pamhd_cfg& c) : Base(c)
	{
		for (int d = 0; d < 3; d++) {
			if (cfg.bc_lo[d] != PAMHD_BC_PERIODIC or cfg.bc_hi[d] != PAMHD_BC_PERIODIC) {
				throw std::invalid_argument("the staggered step needs a periodic grid");
			}
			// a dimension of one cell is its own neighbour
			active[d] = true;
		}
		for (int d = 0; d < 3; d++) {
			Bf[d].assign(U.size(), 0.0);
			FF[d].assign(U.size(), MHD());
		}
	}

	size_t at(const int i, const int j, const int k) const
	{
		const int c[3] = {(i % n[0] + n[0]) % n[0], (j % n[1] + n[1]) % n[1], (k % n[2] + n[2]) % n[2]};
		return this->index(c[0], c[1], c[2]);
	}

	// cell state (8 SoA arrays, x fastest) and face field (3 arrays, -d face of every cell)
	void set_state(const double* const soa[8], const double* const faces[3])
	{
		this->set_interior(soa);
		for (int d = 0; d < 3; d++) {
			for (int k = 0; k < n[2]; k++)
			for (int j = 0; j < n[1]; j++)
			for (int i = 0; i < n[0]; i++) {
				Bf[d][this->index(i, j, k)] = faces[d][size_t(i) + size_t(n[0]) * (size_t(j) + size_t(n[1]) * k)];
			}
		}
	}

	// bg[3 d + c]: component c of the background field at every cell's -d face; nullptr clears it
	void set_background(const double* const bg[9])
	{
		for (int d = 0; d < 3; d++) {
			Bg[d].clear();
			if (bg == nullptr) continue;
			Bg[d].resize(U.size());
			for (int k = 0; k < n[2]; k++)
			for (int j = 0; j < n[1]; j++)
			for (int i = 0; i < n[0]; i++) {
				const size_t src = size_t(i) + size_t(n[0]) * (size_t(j) + size_t(n[1]) * k);
				Bg[d][this->index(i, j, k)] = {bg[3 * d][src], bg[3 * d + 1][src], bg[3 * d + 2][src]};
			}
		}
	}

	// the face of cell a with its +d neighbour b, with the face's background field (mhd/solve.hpp:80-188)
	Face_Flux solve_face_bg(const MHD& a, const MHD& b, const int d, const Vec3& bg) const
	{
		MHD neg = a, pos = b;
		neg.mom = get_rotated_vector(a.mom, d + 1);
		neg.mag = get_rotated_vector(a.mag, d + 1);
		pos.mom = get_rotated_vector(b.mom, d + 1);
		pos.mag = get_rotated_vector(b.mag, d + 1);
		const Vec3 rbg = get_rotated_vector(bg, d + 1);
		Face_Flux r = this->flux(cfg.solver, neg, pos, rbg, cfg.adiabatic_index, cfg.vacuum_permeability);
		r.flux.mom = get_rotated_vector(r.flux.mom, -(d + 1));
		r.flux.mag = get_rotated_vector(r.flux.mag, -(d + 1));
		return r;
	}

	void get_state(double* const soa[8], double* const faces[3]) const
	{
		this->get_interior(soa);
		if (faces == nullptr) return;
		for (int d = 0; d < 3; d++) {
			for (int k = 0; k < n[2]; k++)
			for (int j = 0; j < n[1]; j++)
			for (int i = 0; i < n[0]; i++) {
				faces[d][size_t(i) + size_t(n[0]) * (size_t(j) + size_t(n[1]) * k)] = Bf[d][this->index(i, j, k)];
			}
		}
	}

	/*
	Change of the normal field of the -d face of cell (i, j, k), times the
	face area, from the raw face fluxes FF and dt: the twelve edge terms of
	assign_face_dBs_f{x,y,z} that reach this face, summed in this order:
	d-directed fluxes of the faces one cell away along a and along b, then
	the a-directed and the b-directed fluxes of the faces that share an
	edge with it.
	*/
	double face_dB(const int d, const int i, const int j, const int k, const double dt) const
	{
		const int a = (d + 1) % 3, b = (d + 2) % 3;
		const double La = cfg.cell_length[a], Lb = cfg.cell_length[b];
		int c[3] = {i, j, k};
		const auto cell = [&](const int da, const int db, const int dd) {
			int m[3] = {c[0], c[1], c[2]};
			m[a] += da;
			m[b] += db;
			m[d] += dd;
			return at(m[0], m[1], m[2]);
		};
		const auto bcomp = [](const MHD& f, const int comp) { return f.mag[comp]; };
		// E_b of a d-flux: ((F[B_a] dt) L_b) / 4; E_a: -((F[B_b] dt) L_a) / 4
		const auto e1 = [&](const MHD& f) { return bcomp(f, a) * dt * Lb / 4; };
		const auto e2 = [&](const MHD& f) { return -(bcomp(f, b) * dt * La / 4); };
		// the a-flux's E on the edge along b: -((F[B_d] dt) L_b) / 4
		const auto e3 = [&](const MHD& f) { return -(bcomp(f, d) * dt * Lb / 4); };
		// the b-flux's E on the edge along a: ((F[B_d] dt) L_a) / 4
		const auto e4 = [&](const MHD& f) { return bcomp(f, d) * dt * La / 4; };

		double dB = 0;
		dB += e1(FF[d][cell(+1, 0, 0)]);
		dB -= e1(FF[d][cell(-1, 0, 0)]);
		dB -= e2(FF[d][cell(0, +1, 0)]);
		dB += e2(FF[d][cell(0, -1, 0)]);
		dB += e3(FF[a][cell(+1, 0, 0)]);
		dB += e3(FF[a][cell(+1, 0, -1)]);
		dB -= e3(FF[a][cell(0, 0, 0)]);
		dB -= e3(FF[a][cell(0, 0, -1)]);
		dB -= e4(FF[b][cell(0, +1, 0)]);
		dB -= e4(FF[b][cell(0, +1, -1)]);
		dB += e4(FF[b][cell(0, 0, 0)]);
		dB += e4(FF[b][cell(0, 0, -1)]);
		return dB;
	}

	// update_vol_B with constant thermal pressure (mhd/solve.hpp:1631-1683) for one cell
	void update_vol_B(const size_t idx, const Vec3& mean)
	{
		const double g = cfg.adiabatic_index, mu0 = cfg.vacuum_permeability;
		MHD& u = U[idx];
		if (u.rho <= 0) return;
		const double p = get_pressure(u.rho, u.mom, u.nrj, u.mag, g, mu0);
		u.mag = mean;
		const double inv = 1 / u.rho;
		const Vec3 vel{u.mom[0] * inv, u.mom[1] * inv, u.mom[2] * inv};
		u.nrj = get_total_energy_density(u.rho, vel, p, u.mag, g, mu0);
	}

	// mean of the two faces of a cell per dimension
	Vec3 face_mean(const std::vector<double>* B, const int i, const int j, const int k) const
	{
		const size_t idx = this->index(i, j, k);
		return {0.5 * (B[0][idx] + B[0][at(i + 1, j, k)]),
		        0.5 * (B[1][idx] + B[1][at(i, j + 1, k)]),
		        0.5 * (B[2][idx] + B[2][at(i, j, k + 1)])};
	}

	// one staggered step (timestep(), mhd/solve.hpp:1837-1924, one substep); returns dt
	double step(const double max_dt)
	{
		return step_with(this->timestep(max_dt));
	}

	double step_with(const double dt)
	{
		failure = Failure();
		// fluxes of every cell's +d faces, in the reference's order of cells and faces
		for (size_t idx = 0; idx < U.size(); idx++) {
			int c[3];
			this->coords(idx, c);
			for (int d = 0; d < 3; d++) {
				const int64_t up = this->plus_neighbor(c, d);
				Face_Flux r;
				try {
					r = Bg[d].empty() ? this->solve_face(U[idx], U[up], d)
					                  : solve_face_bg(U[idx], U[up], d, Bg[d][up]);
				} catch (const Domain_Error& e) {
					if (failure.flag == 0) failure = {e.flag, int64_t(idx), d + 1, e.what()};
					continue;
				}
				Max_v[idx][2 * d + 1] = r.speed;
				Max_v[up][2 * d] = r.speed;
				FF[d][up] = r.flux;
				MHD& fc = F[idx][2 * d + 1];
				MHD& fn = F[up][2 * d];
				fc.rho = 0 + dt * r.flux.rho;
				fn.rho = 0 + dt * r.flux.rho;
				fc.nrj = 0 + dt * r.flux.nrj;
				fn.nrj = 0 + dt * r.flux.nrj;
				for (int v = 0; v < 3; v++) {
					fc.mom[v] = 0 + dt * r.flux.mom[v];
					fn.mom[v] = 0 + dt * r.flux.mom[v];
					fc.mag[v] = 0 + dt * r.flux.mag[v];
					fn.mag[v] = 0 + dt * r.flux.mag[v];
				}
			}
		}
		if (failure.flag != 0) throw Domain_Error(failure.flag, failure.what);

		// new face field from the old one and the edge terms
		std::vector<double> nb[3];
		for (int d = 0; d < 3; d++) {
			nb[d].resize(U.size());
			const int a = (d + 1) % 3, b = (d + 2) % 3;
			const double area = cfg.cell_length[a] * cfg.cell_length[b];
			for (int k = 0; k < n[2]; k++)
			for (int j = 0; j < n[1]; j++)
			for (int i = 0; i < n[0]; i++) {
				const size_t idx = this->index(i, j, k);
				nb[d][idx] = Bf[d][idx] + face_dB(d, i, j, k, dt) / area;
			}
		}
		// cell state as Mode C, the volume field included
		this->update();
		for (int d = 0; d < 3; d++) Bf[d].swap(nb[d]);
		// update_vol_B twice with constant thermal pressure
		for (int pass = 0; pass < 2; pass++) {
			for (int k = 0; k < n[2]; k++)
			for (int j = 0; j < n[1]; j++)
			for (int i = 0; i < n[0]; i++) {
				update_vol_B(this->index(i, j, k), face_mean(Bf, i, j, k));
			}
		}
		time += dt;
		return dt;
	}
};

} // namespace oracle

#endif
