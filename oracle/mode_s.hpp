/*
CPU oracle, L3: the staggered-field ("Mode S") MHD step on a uniform
Cartesian grid, periodic or bounded in each dimension.

TEST INFRASTRUCTURE - see mhd_oracle.hpp for who may use this.

The reference's timestep (mhd/solve.hpp:1837-1924) keeps, besides the
cell-centred state, the normal magnetic field of every cell face (Face_B)
and advances it by constrained transport.  Mode_S_Grid<Flux> restates it
for a uniform grid where a periodic dimension of one cell is its own
neighbour (the reference's emulated 1-D and 2-D runs keep those dimensions,
tests/mhd/config_files/.../Alfvén_wave):
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

Bounded dimensions (COPY or VALUE sides, two cells or more) follow the
solar-wind box (tests/mhd/solar_wind_box.cpp), the reference's driver of
staggered runs with open sides.  Its grid has one layer of boundary cells
around the box, and prepare_grid (grid/solar_wind_box.hpp:268-376) makes
every cell of that layer a boundary cell (class 0), faces, edges and
vertices alike; here the layer is a ghost layer outside the n cells.  So:
  - every face between two cells of the extended grid is solved and its
    speed enters the timestep (get_fluxes and minimize_timestep take every
    cell of class >= 0, solve.hpp:254-262, :1965-2003), the ghost-ghost
    faces of the layer included;
  - update_mhd_state changes the state and the face copies of class 1
    cells only (solve.hpp:1544): a face between two interior cells gets its
    twelve terms on both copies; a wall face (between an interior cell and
    the layer) on the interior cell's copy only, and sync_magnetic_field,
    which visits the cells in index order and moves each pair of copies to
    their mean (common_functions.hpp:216-251), then leaves it about half
    way: wall_sync() below repeats its two visits;
  - after the step's time advances (solar_wind_box.cpp:541-553),
    apply_boundaries_sw_box (mhd/solar_wind_box.hpp:328-573) refills the
    layer: each layer cell takes density and momentum of the interior cell
    it touches through a face, an edge or a vertex (:386-537), the normal
    field of its faces from that cell's faces, mirrored across the walls
    it lies behind (the face on the far side of the cell from a wall takes
    the value of the face on the near side), its volume field the mean of
    its two faces per dimension, and its total energy from the source
    cell's thermal pressure;
  - a VALUE side is the solar-wind plane (apply_solar_wind_boundaries,
    :227-306): its cells take the side's state (a time-stamped table,
    selected by the new time) with every face at the state's field, and
    the cell on the inner side of each of them gets the state's normal
    field on the shared face, the mean of its two faces along that
    dimension (each half added) as its volume field, and its total energy
    from its thermal pressure before the change.  One VALUE side at most,
    as the reference's single wind direction.
The face arrays of set_state / get_state hold n + 1 faces along a bounded
dimension (its two walls included) and n along a periodic one.

Background field (optional, periodic grids): Bg[d][cell] is the background
field vector at the cell's -d face (the reference's Bg_B of the face,
integrated over it at initialisation, mhd/initialize.hpp:517-530).  The
face between a cell and its +d neighbour is solved with that face's vector,
rotated into the face frame (mhd/solve.hpp:120-121); the solvers use it as
the reference's do (Rusanov and HLL in the flux and the fast speeds, HLLD
and Roe not at all).  The cell state and Face_B hold the field without the
background, as in the reference.
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
	using Base::ext;
	using Base::U;
	using Base::F;
	using Base::Max_v;
	using Base::CType;
	using Base::active;
	using Base::periodic;
	using Base::failure;
	using Base::time;

	std::vector<double> Bf[3];   // normal field of each cell's -d face
	std::vector<MHD> FF[3];      // raw flux through each cell's -d face, unrotated
	std::vector<Vec3> Bg[3];     // background field at each cell's -d face (empty: none)
	int value_dim = -1, value_side = 0;  // the VALUE side, if any
	bool loaded = false;                 // a state was set (the layer can be filled)

	explicit Mode_S_Grid(const pamhd_cfg& c) : Base(c)
	{
		for (int d = 0; d < 3; d++) {
			if (n[d] == 1 and not periodic[d]) {
				throw std::invalid_argument("a dimension of one cell must be periodic in the staggered step");
			}
			for (int side = 0; side < 2; side++) {
				const int kind = side == 0 ? cfg.bc_lo[d] : cfg.bc_hi[d];
				if (kind == PAMHD_BC_VALUE and n[d] > 1) {
					if (value_dim >= 0) throw std::invalid_argument("one VALUE side at most in the staggered step");
					value_dim = d;
					value_side = side;
				} else if (kind != PAMHD_BC_PERIODIC and kind != PAMHD_BC_COPY and n[d] > 1) {
					throw std::invalid_argument("staggered sides are PERIODIC, COPY or VALUE");
				}
			}
			// a dimension of one cell is its own neighbour
			active[d] = true;
		}
		// every cell of the boundary layer is a boundary cell (class 0), edges and vertices included
		for (size_t idx = 0; idx < U.size(); idx++) {
			int cc[3];
			this->coords(idx, cc);
			bool inside = true;
			for (int d = 0; d < 3; d++) inside = inside and cc[d] >= 0 and cc[d] < n[d];
			CType[idx] = inside ? 1 : 0;
		}
		for (int d = 0; d < 3; d++) {
			Bf[d].assign(U.size(), 0.0);
			FF[d].assign(U.size(), MHD());
		}
	}

	bool bounded(const int d) const { return ext[d] == 1; }

	// index of cell (i, j, k): periodic dimensions wrap, bounded ones reach one cell past the walls
	size_t at(const int i, const int j, const int k) const
	{
		int c[3] = {i, j, k};
		for (int d = 0; d < 3; d++) {
			if (not bounded(d)) c[d] = (c[d] % n[d] + n[d]) % n[d];
		}
		return this->index(c[0], c[1], c[2]);
	}

	// faces along dimension e of the face arrays of dimension d (walls included when bounded)
	int face_extent(const int d, const int e) const { return n[e] + ((e == d and bounded(d)) ? 1 : 0); }

	// cell state (8 SoA arrays, x fastest) and face field (3 arrays, the -d face of every cell, and
	// along a bounded dimension the high wall too), then the boundary layer
	void set_state(const double* const soa[8], const double* const faces[3])
	{
		this->set_interior(soa);
		for (int d = 0; d < 3; d++) {
			const int fx = face_extent(d, 0), fy = face_extent(d, 1), fz = face_extent(d, 2);
			for (int k = 0; k < fz; k++)
			for (int j = 0; j < fy; j++)
			for (int i = 0; i < fx; i++) {
				Bf[d][this->index(i, j, k)] = faces[d][size_t(i) + size_t(fx) * (size_t(j) + size_t(fy) * k)];
			}
		}
		loaded = true;
		fill_boundaries();
	}

	void set_inflow(const int d, const int side, const std::vector<double>& times,
	                const std::vector<std::array<double, 8>>& states)
	{
		Base::set_inflow(d, side, times, states);
		if (loaded) fill_boundaries();
	}

	// bg[3 d + c]: component c of the background field at every cell's -d face; nullptr clears it
	void set_background(const double* const bg[9])
	{
		for (int d = 0; d < 3; d++) {
			Bg[d].clear();
			if (bg == nullptr) continue;
			for (int e = 0; e < 3; e++) {
				if (bounded(e)) throw std::invalid_argument("the background field needs a periodic grid");
			}
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
			const int fx = face_extent(d, 0), fy = face_extent(d, 1), fz = face_extent(d, 2);
			for (int k = 0; k < fz; k++)
			for (int j = 0; j < fy; j++)
			for (int i = 0; i < fx; i++) {
				faces[d][size_t(i) + size_t(fx) * (size_t(j) + size_t(fy) * k)] = Bf[d][this->index(i, j, k)];
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

	/*
	sync_magnetic_field (common_functions.hpp:216-251) on a wall face: the
	boundary cell's copy keeps the old value `old` (its Face_dB is not
	applied), the interior cell's copy has `updated`; the cells are visited
	in index order, and each visit moves the visiting cell's copy down by
	half the difference and the other's up by the same.  lo_wall: the
	boundary cell comes first (a wall at the low end of a dimension).
	Returns the interior cell's copy.
	*/
	static double wall_sync(const double old, const double updated, const bool lo_wall)
	{
		if (lo_wall) {
			const double diff1 = old - updated;
			const double g1 = old - diff1 / 2, p1 = updated + diff1 / 2;
			const double diff2 = p1 - g1;
			return p1 - diff2 / 2;
		}
		const double diff1 = updated - old;
		const double p1 = updated - diff1 / 2, g1 = old + diff1 / 2;
		const double diff2 = g1 - p1;
		return p1 + diff2 / 2;
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

	/*
	The boundary layer from the interior (apply_boundaries_sw_box,
	mhd/solar_wind_box.hpp:386-537, then apply_solar_wind_boundaries
	:227-306 on the VALUE side), as described above.  The layer's cells
	read interior cells only, so their order does not matter; the VALUE
	plane comes after them.
	*/
	void fill_boundaries()
	{
		const double g = cfg.adiabatic_index, mu0 = cfg.vacuum_permeability;
		for (size_t idx = 0; idx < U.size(); idx++) {
			if (CType[idx] != 0) continue;
			int c[3], s[3];
			this->coords(idx, c);
			bool shell[3];
			for (int d = 0; d < 3; d++) {
				shell[d] = c[d] < 0 or c[d] >= n[d];
				s[d] = c[d] < 0 ? 0 : (c[d] >= n[d] ? n[d] - 1 : c[d]);
			}
			const size_t src = this->index(s[0], s[1], s[2]);
			const MHD& su = U[src];
			const double p = get_pressure(su.rho, su.mom, su.nrj, su.mag, g, mu0);
			MHD& u = U[idx];
			u.rho = su.rho;
			u.mom = su.mom;
			Vec3 mean;
			for (int e = 0; e < 3; e++) {
				int up[3] = {s[0], s[1], s[2]};
				up[e] += 1;
				const double lo = Bf[e][src], hi = Bf[e][at(up[0], up[1], up[2])];
				// the -e face of this cell: the source's +e face behind a low wall, else the face at
				// the same place along e (a high wall's own face when the cell lies behind it)
				int f[3] = {s[0], s[1], s[2]};
				f[e] = (shell[e] and c[e] < 0) ? 1 : c[e];
				Bf[e][idx] = Bf[e][at(f[0], f[1], f[2])];
				// the cell's two faces along e are the source's two, swapped behind a wall
				mean[e] = shell[e] ? 0.5 * (hi + lo) : 0.5 * (lo + hi);
			}
			u.mag = mean;
			const double inv = 1 / u.rho;
			u.nrj = get_total_energy_density(u.rho, Vec3{u.mom[0] * inv, u.mom[1] * inv, u.mom[2] * inv}, p,
			                                 u.mag, g, mu0);
		}
		if (value_dim < 0) return;
		const int d = value_dim, a = (d + 1) % 3, b = (d + 2) % 3;
		const bool lo = value_side == 0;
		const double* v = this->value_of(d, lo);
		const int plane = lo ? -1 : n[d], inner = lo ? 0 : n[d] - 1;
		for (int tb = -ext[b]; tb < n[b] + ext[b]; tb++)
		for (int ta = -ext[a]; ta < n[a] + ext[a]; ta++) {
			int c[3];
			c[d] = plane;
			c[a] = ta;
			c[b] = tb;
			const size_t idx = this->index(c[0], c[1], c[2]);
			MHD& u = U[idx];
			u.rho = v[0];
			u.mom = {v[1], v[2], v[3]};
			u.nrj = v[4];
			u.mag = {v[5], v[6], v[7]};
			for (int e = 0; e < 3; e++) Bf[e][idx] = v[5 + e];
			// the inner neighbour: the shared face at the state's normal field
			int q[3] = {c[0], c[1], c[2]};
			q[d] = inner;
			const size_t qi = this->index(q[0], q[1], q[2]);
			MHD& w = U[qi];
			const double p = get_pressure(w.rho, w.mom, w.nrj, w.mag, g, mu0);
			int qu[3] = {q[0], q[1], q[2]};
			qu[d] += 1;
			const size_t shared = lo ? qi : this->index(qu[0], qu[1], qu[2]);
			const size_t other = lo ? this->index(qu[0], qu[1], qu[2]) : qi;
			Bf[d][shared] = v[5 + d];
			w.mag[d] = Bf[d][shared] / 2 + Bf[d][other] / 2;
			const double inv = 1 / w.rho;
			w.nrj = get_total_energy_density(w.rho, Vec3{w.mom[0] * inv, w.mom[1] * inv, w.mom[2] * inv}, p,
			                                 w.mag, g, mu0);
		}
	}

	// one staggered step (timestep(), mhd/solve.hpp:1837-1924, one substep); returns dt
	double step(const double max_dt)
	{
		return step_with(this->timestep(max_dt));
	}

	double step_with(const double dt)
	{
		failure = Failure();
		// fluxes of every +d face between two cells of class >= 0, in the reference's order of cells and faces
		for (size_t idx = 0; idx < U.size(); idx++) {
			if (CType[idx] < 0) continue;
			int c[3];
			this->coords(idx, c);
			for (int d = 0; d < 3; d++) {
				const int64_t up = this->plus_neighbor(c, d);
				if (up < 0 or CType[up] < 0) continue;
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

		// new face field of the interior cells' faces (walls included) from the edge terms
		std::vector<double> nb[3], old[3];
		for (int d = 0; d < 3; d++) {
			nb[d] = Bf[d];
			old[d] = Bf[d];
			const int a = (d + 1) % 3, b = (d + 2) % 3;
			const double area = cfg.cell_length[a] * cfg.cell_length[b];
			const int fx = face_extent(d, 0), fy = face_extent(d, 1), fz = face_extent(d, 2);
			for (int k = 0; k < fz; k++)
			for (int j = 0; j < fy; j++)
			for (int i = 0; i < fx; i++) {
				const size_t idx = this->index(i, j, k);
				nb[d][idx] = Bf[d][idx] + face_dB(d, i, j, k, dt) / area;
			}
		}
		// cell state as Mode C, the volume field included
		this->update();
		for (int d = 0; d < 3; d++) Bf[d].swap(nb[d]);
		// update_vol_B inside the substep loop, with the interior cells' own copies of the walls
		for (int k = 0; k < n[2]; k++)
		for (int j = 0; j < n[1]; j++)
		for (int i = 0; i < n[0]; i++) {
			update_vol_B(this->index(i, j, k), face_mean(Bf, i, j, k));
		}
		// sync_magnetic_field on the walls, then update_vol_B again
		for (int d = 0; d < 3; d++) {
			if (not bounded(d)) continue;
			const int a = (d + 1) % 3, b = (d + 2) % 3;
			for (int tb = 0; tb < n[b]; tb++)
			for (int ta = 0; ta < n[a]; ta++) {
				for (const int w: {0, n[d]}) {
					int c[3];
					c[d] = w;
					c[a] = ta;
					c[b] = tb;
					const size_t idx = this->index(c[0], c[1], c[2]);
					Bf[d][idx] = wall_sync(old[d][idx], Bf[d][idx], w == 0);
				}
			}
		}
		for (int k = 0; k < n[2]; k++)
		for (int j = 0; j < n[1]; j++)
		for (int i = 0; i < n[0]; i++) {
			update_vol_B(this->index(i, j, k), face_mean(Bf, i, j, k));
		}
		time += dt;
		fill_boundaries();
		return dt;
	}
};

} // namespace oracle

#endif
