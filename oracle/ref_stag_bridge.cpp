/*
libstag_ref.so: the reference's OWN staggered-field step (and, below, its
cell-centred subset), compiled
unchanged from the reference tree by oracle/Makefile on a one-rank box
stand-in for dccrg (ref_shim/box_grid.hpp): timestep() of mhd/solve.hpp
(get_fluxes with assign_face_dBs_f{x,y,z}, update_mhd_state, update_vol_B,
sync_magnetic_field of common_functions.hpp), and on a bounded box the
solar-wind box's apply_boundaries_sw_box (mhd/solar_wind_box.hpp) with the
program's loop around them (tests/mhd/solar_wind_box.cpp:446-553).  The C
entry point below runs that loop on a given state, so that the oracle's
restatement (oracle/mode_s.hpp) and through it the GPU step can be held to
the reference's own arithmetic.

The box: the given n cells, plus along each bounded dimension one layer of
boundary cells on both sides, as the solar-wind box's grid carries them;
the cell classes and the face / edge / vertex / wind cell lists are made as
prepare_grid (grid/solar_wind_box.hpp:268-376) makes them for a box with no
planet and no refinement.  Periodic dimensions wrap and carry no layer.

TEST INFRASTRUCTURE - see mhd_oracle.hpp for who may use this.
*/
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

// the grid and mhd option parsers (muparserx, rapidjson) are not needed: the functions used take
// their options as template parameters or as the plain structure below; their include guards keep
// them out
#define PAMHD_MHD_OPTIONS_HPP
#define PAMHD_GRID_AMR_HPP
#define PAMHD_SOLAR_WIND_BOX_OPTIONS_HPP
#define PAMHD_BACKGROUND_MAGNETIC_FIELD_HPP

#include <functional>

#include "single_rank_mpi.hpp"
#include "box_grid.hpp"

// the two refinement-level variables that grid/amr.hpp defines for the MHD cell (same names and
// data types, so that mhd/variables.hpp builds its cell type unchanged)
namespace pamhd {
namespace grid {
struct Target_Refinement_Level_Min {
	static bool is_stale;
	using data_type = int;
};
struct Target_Refinement_Level_Max {
	static bool is_stale;
	using data_type = int;
};
}

// the background field's interface that initialize_plasma names (background_magnetic_field.hpp:
// 331-334); no background field here
template <class Scalar, class Vector> class Background_Magnetic_Field {
public:
	Vector get_background_field(const Vector&, const Scalar&) const { return Vector{0, 0, 0}; }
};

// the solar-wind options the boundary functions read (solar_wind_box_options.hpp:50-66)
struct Solar_Wind_Box_Options {
	int sw_dir{0};
	size_t sw_dim{3};
	double inner_radius{-1}, inner_nr_density{-1}, inner_pressure{-1};
	std::array<double, 3> inner_velocity{0, 0, 0}, inner_magnetic_field{0, 0, 0};
	std::vector<double> sw_nr_density, sw_pressure, sw_timestamps;
	std::vector<std::array<double, 3>> sw_velocity, sw_magnetic_field;
};
}

// where the reference stops the program (abort() after its diagnostic), stop this call instead
[[noreturn]] inline void reference_stopped()
{
	throw std::runtime_error("the reference aborted");
}
#define abort() reference_stopped()
#include "mhd/variables.hpp"
#include "variable_getter.hpp"
#include "common_functions.hpp"
#include "mhd/solve.hpp"
#include "mhd/solar_wind_box.hpp"
#undef abort

bool pamhd::grid::Target_Refinement_Level_Min::is_stale = true;
bool pamhd::grid::Target_Refinement_Level_Max::is_stale = true;
bool pamhd::Bg_Magnetic_Field::is_stale = true;
bool pamhd::mhd::Mass_Density::is_stale = true;
bool pamhd::mhd::Momentum_Density::is_stale = true;
bool pamhd::mhd::Total_Energy_Density::is_stale = true;
bool pamhd::Magnetic_Field::is_stale = true;
bool pamhd::Face_Magnetic_Field::is_stale = true;
bool pamhd::Cell_Type::is_stale = true;
bool pamhd::Substepping_Period::is_stale = true;
bool pamhd::Substep_Min::is_stale = true;
bool pamhd::Substep_Max::is_stale = true;
bool pamhd::Timestep::is_stale = true;
bool pamhd::mhd::Max_Velocity::is_stale = true;

namespace {

using Cell = pamhd::mhd::Cell;
using Grid = oracle_shim::Box_Grid<Cell>;

// the program's variable getters (tests/mhd/solar_wind_box.cpp:84-144)
const auto Bg_B = pamhd::Variable_Getter<pamhd::Bg_Magnetic_Field>();
const auto Mas = pamhd::Variable_Getter<pamhd::mhd::Mass_Density>();
const auto Mom = pamhd::Variable_Getter<pamhd::mhd::Momentum_Density>();
const auto Nrj = pamhd::Variable_Getter<pamhd::mhd::Total_Energy_Density>();
const auto Vol_B = pamhd::Variable_Getter<pamhd::Magnetic_Field>();
const auto Face_B = pamhd::Variable_Getter<pamhd::Face_Magnetic_Field>();
const auto Face_dB = pamhd::Variable_Getter<pamhd::Face_dB>();
const auto Berror = pamhd::Variable_Getter<pamhd::Face_B_Error>();
const auto CType = pamhd::Variable_Getter<pamhd::Cell_Type>();
const auto Substep = pamhd::Variable_Getter<pamhd::Substepping_Period>();
const auto Substep_Min = pamhd::Variable_Getter<pamhd::Substep_Min>();
const auto Substep_Max = pamhd::Variable_Getter<pamhd::Substep_Max>();
const auto Timestep = pamhd::Variable_Getter<pamhd::Timestep>();
const auto Max_v = pamhd::Variable_Getter<pamhd::mhd::Max_Velocity>();
const auto MHDF = pamhd::Variable_Getter<pamhd::mhd::MHD_Flux>();
const auto Mas_f = [](Cell& cell_data, const int dir)->auto& {
	return MHDF.data(cell_data)(dir)[pamhd::mhd::Mass_Density()];
};
const auto Mom_f = [](Cell& cell_data, const int dir)->auto& {
	return MHDF.data(cell_data)(dir)[pamhd::mhd::Momentum_Density()];
};
const auto Nrj_f = [](Cell& cell_data, const int dir)->auto& {
	return MHDF.data(cell_data)(dir)[pamhd::mhd::Total_Energy_Density()];
};
const auto Mag_f = [](Cell& cell_data, const int dir)->auto& {
	return MHDF.data(cell_data)(dir)[pamhd::Magnetic_Field()];
};

// substepping options: every cell's exponent bounds from a per-cell table (x fastest) looked up at
// the cell's centre, as the options' expressions are evaluated there (substepping.hpp:213-228), or
// 0 everywhere (no substeps) without a table
struct Per_Cell_Exponent {
	const Grid* grid = nullptr;
	const int32_t* values = nullptr;
	double evaluate(double, const double x, const double y, const double z, double, double, double) const
	{
		if (values == nullptr) return 0;
		const auto& g = grid->geometry;
		const int i = int(std::floor(x / g.len[0])), j = int(std::floor(y / g.len[1])),
			k = int(std::floor(z / g.len[2]));
		return values[i + size_t(g.n[0]) * (j + size_t(g.n[1]) * k)];
	}
};
struct Sim_Options {
	int substep_min_i = 0, substep_max_i = 0;
	Per_Cell_Exponent substep_min_e, substep_max_e;
};

using Cell_List = std::vector<Grid::Cell>;

} // namespace

/*
Runs the solar-wind box's loop for nsteps steps (the first the dt = 0
priming step) on a box of n cells per dimension (bc: 0 periodic, 1 COPY,
2 VALUE; a bounded dimension gets a layer of boundary cells on both
sides).  cells: 8 arrays of the n cells (x fastest); faces: the normal
field of every cell's -d face, n + 1 faces along a bounded dimension (the
high wall last), the three arrays one after another.  value_prim: the VALUE
side's number density (proton mass 1), velocity xyz, pressure and field
xyz.  Writes the state after the steps in the same layout, every step's dt,
and the conservative state the wind cells took (8 values).  Returns 0, or
1 with the message of a thrown exception (the reference's domain errors and
stops).
*/
extern "C" int ref_stag_run(const int32_t n[3], const double cell_length[3], const int32_t bc_lo[3],
                            const int32_t bc_hi[3], const int32_t solver_id, const double gamma, const double mu0,
                            const double cfl, const double* cells, const double* faces, const double* value_prim,
                            const int32_t nsteps, double* cells_out, double* faces_out, double* dts,
                            double* value_out)
{
	try {
		std::array<int, 3> ext{}, E{};
		std::array<bool, 3> periodic{};
		pamhd::Solar_Wind_Box_Options box;
		for (int d = 0; d < 3; d++) {
			periodic[d] = bc_lo[d] == 0 and bc_hi[d] == 0;
			ext[d] = (n[d] > 1 and not periodic[d]) ? 1 : 0;
			E[d] = n[d] + 2 * ext[d];
			if (ext[d] and bc_lo[d] == 2) box.sw_dir = -(d + 1);
			if (ext[d] and bc_hi[d] == 2) box.sw_dir = +(d + 1);
		}
		Grid grid(E, {cell_length[0], cell_length[1], cell_length[2]}, periodic);
		if (box.sw_dir != 0) {
			box.sw_dim = size_t(std::abs(box.sw_dir) - 1);
			box.sw_nr_density = {value_prim[0]};
			box.sw_velocity = {{value_prim[1], value_prim[2], value_prim[3]}};
			box.sw_pressure = {value_prim[4]};
			box.sw_magnetic_field = {{value_prim[5], value_prim[6], value_prim[7]}};
		}
		const auto index = [&](const int i, const int j, const int k) {
			return size_t(i + ext[0]) + size_t(E[0]) * (size_t(j + ext[1]) + size_t(E[1]) * size_t(k + ext[2]));
		};
		// classes and boundary lists as prepare_grid (grid/solar_wind_box.hpp:283-376)
		Cell_List sw_cells, vert_cells, planet_cells;
		pamhd::Face_Type<Cell_List> face_cells;
		pamhd::Edge_Type<Cell_List> edge_cells;
		for (const auto& cell: grid.local_cells()) {
			const auto idx = grid.mapping.get_indices(cell.id);
			int s[3];
			for (int d = 0; d < 3; d++) {
				s[d] = 0;
				if (ext[d] and idx[d] == 0) s[d] = -1;
				else if (ext[d] and int(idx[d]) == E[d] - 1) s[d] = +1;
			}
			CType.data(*cell.data) = (s[0] == 0 and s[1] == 0 and s[2] == 0) ? 1 : 0;
			if (box.sw_dir != 0 and s[box.sw_dim] == (box.sw_dir < 0 ? -1 : +1)) sw_cells.push_back(cell);
			const int x = s[0], y = s[1], z = s[2];
			if (x != 0 and y != 0 and z != 0) vert_cells.push_back(cell);
			else if (y != 0 and z != 0) edge_cells(0, y, z).push_back(cell);
			else if (x != 0 and z != 0) edge_cells(1, x, z).push_back(cell);
			else if (x != 0 and y != 0) edge_cells(2, x, y).push_back(cell);
			else if (x != 0) face_cells(x).push_back(cell);
			else if (y != 0) face_cells(2 * y).push_back(cell);
			else if (z != 0) face_cells(3 * z).push_back(cell);
		}
		// the state: interior cells, each cell's copies of its faces
		const size_t cells_n = size_t(n[0]) * n[1] * n[2];
		size_t fofs[3], at = 0;
		int fext[3][3];
		for (int d = 0; d < 3; d++) {
			fofs[d] = at;
			for (int e = 0; e < 3; e++) fext[d][e] = n[e] + ((e == d and ext[d]) ? 1 : 0);
			at += size_t(fext[d][0]) * fext[d][1] * fext[d][2];
		}
		const auto face_at = [&](const int d, const int i, const int j, const int k) {
			return fofs[d] + size_t(i) + size_t(fext[d][0]) * (size_t(j) + size_t(fext[d][1]) * k);
		};
		for (int k = 0; k < n[2]; k++)
		for (int j = 0; j < n[1]; j++)
		for (int i = 0; i < n[0]; i++) {
			const size_t src = size_t(i) + size_t(n[0]) * (size_t(j) + size_t(n[1]) * k);
			Cell& c = grid.data[index(i, j, k)];
			Mas.data(c) = cells[src];
			Mom.data(c) = {cells[cells_n + src], cells[2 * cells_n + src], cells[3 * cells_n + src]};
			Nrj.data(c) = cells[4 * cells_n + src];
			Vol_B.data(c) = {cells[5 * cells_n + src], cells[6 * cells_n + src], cells[7 * cells_n + src]};
			const int ijk[3] = {i, j, k};
			for (int d = 0; d < 3; d++) {
				int up[3] = {i, j, k};
				up[d] += 1;
				if (not ext[d]) up[d] %= n[d];
				Face_B.data(c)(d, -1) = faces[face_at(d, ijk[0], ijk[1], ijk[2])];
				Face_B.data(c)(d, +1) = faces[face_at(d, up[0], up[1], up[2])];
			}
		}
		for (auto& c: grid.data) {
			Substep.data(c) = Substep_Min.data(c) = Substep_Max.data(c) = 1;
			Max_v.data(c) = {-1, -1, -1, -1, -1, -1};
			Berror.data(c) = 0;
			for (int dir: {-3, -2, -1, +1, +2, +3}) Bg_B.data(c)(dir) = {0, 0, 0};
		}
		Sim_Options options;
		const pamhd::mhd::Solver solver = solver_id == 0 ? pamhd::mhd::Solver::rusanov
			: solver_id == 2 ? pamhd::mhd::Solver::hll_athena
			: solver_id == 3 ? pamhd::mhd::Solver::hlld_athena
			: pamhd::mhd::Solver::roe_athena;
		// the program's start and loop (tests/mhd/solar_wind_box.cpp:446-553)
		double t = 0;
		pamhd::mhd::update_vol_B(0, grid.local_cells(), Mas, Mom, Nrj, Vol_B, Face_B, CType, Substep, gamma, mu0,
		                         true);
		pamhd::mhd::apply_boundaries_sw_box(grid, t, box, sw_cells, face_cells, edge_cells, vert_cells,
		                                    planet_cells, gamma, mu0, 1.0, Mas, Mom, Nrj, Vol_B, Face_B, Face_dB,
		                                    CType);
		pamhd::sync_magnetic_field(grid, Face_B, Vol_B, Berror, CType);
		if (box.sw_dir != 0) {
			Cell& w = *sw_cells.front().data;
			const double v[8] = {Mas.data(w), Mom.data(w)[0], Mom.data(w)[1], Mom.data(w)[2], Nrj.data(w),
			                     Vol_B.data(w)[0], Vol_B.data(w)[1], Vol_B.data(w)[2]};
			std::memcpy(value_out, v, sizeof v);
		}
		for (int s = 0; s < nsteps; s++) {
			const double cap = s == 0 ? 0.0 : std::numeric_limits<double>::max();
			const auto [dt, max_sub, calcs] = pamhd::mhd::timestep(
				solver, grid, options, t, cap, cfl, gamma, mu0, Mas, Mom, Nrj, Vol_B, Face_B, Face_dB, Berror, Bg_B,
				Mas_f, Mom_f, Nrj_f, Mag_f, CType, Timestep, Substep, Substep_Min, Substep_Max, Max_v);
			(void)max_sub;
			(void)calcs;
			dts[s] = dt;
			t += dt;
			pamhd::mhd::apply_boundaries_sw_box(grid, t, box, sw_cells, face_cells, edge_cells, vert_cells,
			                                    planet_cells, gamma, mu0, 1.0, Mas, Mom, Nrj, Vol_B, Face_B,
			                                    Face_dB, CType);
			pamhd::sync_magnetic_field(grid, Face_B, Vol_B, Berror, CType);
		}
		for (int k = 0; k < n[2]; k++)
		for (int j = 0; j < n[1]; j++)
		for (int i = 0; i < n[0]; i++) {
			const size_t dst = size_t(i) + size_t(n[0]) * (size_t(j) + size_t(n[1]) * k);
			Cell& c = grid.data[index(i, j, k)];
			cells_out[dst] = Mas.data(c);
			for (int e = 0; e < 3; e++) cells_out[(1 + e) * cells_n + dst] = Mom.data(c)[e];
			cells_out[4 * cells_n + dst] = Nrj.data(c);
			for (int e = 0; e < 3; e++) cells_out[(5 + e) * cells_n + dst] = Vol_B.data(c)[e];
		}
		// every face from the copy of the cell above it, the high walls from the last cells' copies
		for (int d = 0; d < 3; d++) {
			for (int k = 0; k < fext[d][2]; k++)
			for (int j = 0; j < fext[d][1]; j++)
			for (int i = 0; i < fext[d][0]; i++) {
				const int c[3] = {i, j, k};
				const bool wall = ext[d] and c[d] == n[d];
				int m[3] = {i, j, k};
				if (wall) m[d] -= 1;
				Cell& cell = grid.data[index(m[0], m[1], m[2])];
				faces_out[face_at(d, i, j, k)] = Face_B.data(cell)(d, wall ? +1 : -1);
			}
		}
		return 0;
	} catch (const std::exception& e) {
		std::cerr << e.what() << std::endl;
		return 1;
	}
}

/*
The cell-centred step on a periodic box (a dimension of one cell not
periodic: it has no faces, as the reference's 2-D grids with periodic
{true, true, false}), from the reference's own functions
in timestep()'s order without its face-field parts (mhd/solve.hpp:1865-1902:
set_minmax_substepping_period, minimize_timestep, the substep plan,
get_all_fluxes, update_mhd_state; no update_vol_B and no sync, so the cell's
volume field keeps the flux update): nsteps steps, the first the dt = 0
priming step.  cells as ref_stag_run; writes the state after the steps and
every step's dt.  Returns 0, or 1 with the message of a thrown exception.
*/
extern "C" int ref_cell_centred_substep_run(const int32_t n[3], const double cell_length[3],
                                            const int32_t solver_id, const double gamma, const double mu0,
                                            const double cfl, const double* cells, const int32_t* smin,
                                            const int32_t* smax, const int32_t nsteps, double* cells_out,
                                            double* dts, int32_t* max_periods);

extern "C" int ref_cell_centred_run(const int32_t n[3], const double cell_length[3], const int32_t solver_id,
                                    const double gamma, const double mu0, const double cfl, const double* cells,
                                    const int32_t nsteps, double* cells_out, double* dts)
{
	return ref_cell_centred_substep_run(n, cell_length, solver_id, gamma, mu0, cfl, cells, nullptr, nullptr,
	                                    nsteps, cells_out, dts, nullptr);
}

/*
As ref_cell_centred_run with local time stepping: smin, smax the smallest
and largest substep exponent of every cell (the options' substep-min and
substep-max, x fastest), or nullptr for 0.  Writes each step's largest
period too (max_periods, or nullptr).
*/
extern "C" int ref_cell_centred_substep_run(const int32_t n[3], const double cell_length[3],
                                            const int32_t solver_id, const double gamma, const double mu0,
                                            const double cfl, const double* cells, const int32_t* smin,
                                            const int32_t* smax, const int32_t nsteps, double* cells_out,
                                            double* dts, int32_t* max_periods)
{
	try {
		const std::array<int, 3> N{n[0], n[1], n[2]};
		Grid grid(N, {cell_length[0], cell_length[1], cell_length[2]}, {n[0] > 1, n[1] > 1, n[2] > 1});
		const size_t count = size_t(n[0]) * n[1] * n[2];
		for (size_t i = 0; i < count; i++) {
			Cell& c = grid.data[i];
			Mas.data(c) = cells[i];
			Mom.data(c) = {cells[count + i], cells[2 * count + i], cells[3 * count + i]};
			Nrj.data(c) = cells[4 * count + i];
			Vol_B.data(c) = {cells[5 * count + i], cells[6 * count + i], cells[7 * count + i]};
			CType.data(c) = 1;
			Substep.data(c) = Substep_Min.data(c) = Substep_Max.data(c) = 1;
			Max_v.data(c) = {-1, -1, -1, -1, -1, -1};
			for (int dir: {-3, -2, -1, +1, +2, +3}) {
				Bg_B.data(c)(dir) = {0, 0, 0};
				Face_B.data(c)(dir) = 0;
			}
		}
		Sim_Options options;
		if (smin != nullptr and smax != nullptr) {
			options.substep_min_i = options.substep_max_i = -1;
			options.substep_min_e = {&grid, smin};
			options.substep_max_e = {&grid, smax};
		}
		const pamhd::mhd::Solver solver = solver_id == 0 ? pamhd::mhd::Solver::rusanov
			: solver_id == 2 ? pamhd::mhd::Solver::hll_athena
			: solver_id == 3 ? pamhd::mhd::Solver::hlld_athena
			: pamhd::mhd::Solver::roe_athena;
		double t = 0;
		for (int s = 0; s < nsteps; s++) {
			const double cap = s == 0 ? 0.0 : std::numeric_limits<double>::max();
			pamhd::set_minmax_substepping_period(t, grid, options, Substep_Min, Substep_Max);
			pamhd::mhd::minimize_timestep(grid, cfl, CType, Timestep, Max_v);
			const double sub_dt = pamhd::set_minmax_substepping_period(grid, cap, CType, Timestep, Substep_Min,
			                                                           Substep_Max);
			pamhd::restrict_substepping_period(grid, Substep, Substep_Max, CType);
			const int max_substep = pamhd::update_substeps(grid, CType, Substep);
			double total_dt = 0;
			for (int substep = 1; substep <= max_substep; substep++) {
				total_dt += sub_dt;
				pamhd::mhd::get_all_fluxes(sub_dt, solver, grid, substep, gamma, mu0, Mas, Mom, Nrj, Vol_B, Face_B,
				                           Face_dB, Bg_B, Mas_f, Mom_f, Nrj_f, Mag_f, CType, Substep, Max_v);
				pamhd::mhd::update_mhd_state(grid.local_cells(), grid, substep, Face_B, Face_dB, CType, Substep,
				                             Mas, Mom, Nrj, Vol_B, Mas_f, Mom_f, Nrj_f, Mag_f);
			}
			dts[s] = total_dt;
			if (max_periods != nullptr) max_periods[s] = max_substep;
			t += total_dt;
		}
		for (size_t i = 0; i < count; i++) {
			Cell& c = grid.data[i];
			cells_out[i] = Mas.data(c);
			for (int e = 0; e < 3; e++) cells_out[(1 + e) * count + i] = Mom.data(c)[e];
			cells_out[4 * count + i] = Nrj.data(c);
			for (int e = 0; e < 3; e++) cells_out[(5 + e) * count + i] = Vol_B.data(c)[e];
		}
		return 0;
	} catch (const std::exception& e) {
		std::cerr << e.what() << std::endl;
		return 1;
	}
}

