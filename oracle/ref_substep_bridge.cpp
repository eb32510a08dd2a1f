/*
libsubstep_ref.so: the reference's OWN temporal substepping functions
(substepping.hpp: set_minmax_substepping_period, both forms;
restrict_substepping_period; update_substeps), compiled unchanged from the
reference tree by oracle/Makefile, on a single-rank uniform-grid stand-in
for dccrg (ref_shim/uniform_grid.hpp, ref_shim/single_rank_mpi.hpp).  The
C entry point runs them in the order of the reference's timestep()
(mhd/solve.hpp:1865-1884) on given per-cell CFL limits, so that the
oracle's restatement of the substep plan (oracle/substep.hpp) can be held
to them bit for bit.

TEST INFRASTRUCTURE - see mhd_oracle.hpp for who may use this.
*/
#include <cmath>
#include <cstdint>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>

// mhd/options.hpp (the options parser: rapidjson, muparserx) is not needed: the functions below
// take the options object as a template parameter; its include guard keeps it out
#define PAMHD_MHD_OPTIONS_HPP
#include "single_rank_mpi.hpp"
#include "uniform_grid.hpp"

// where the reference stops the program (abort() after its diagnostic), stop this call instead, so
// that a test can see the stop and go on
[[noreturn]] inline void reference_stopped()
{
	throw std::runtime_error("the reference aborted");
}
#define abort() reference_stopped()
#include "substepping.hpp"
#undef abort

namespace {

struct Stale {
	bool is_stale = false;
};

struct Cell_Data {
	int ctype = 1;
	double timestep = 0;
	int substep = 0, substep_min = 0, substep_max = 0;
	static void set_transfer_all(bool, const Stale&) {}
};

// accessors with the reference's data()/type() interface
template <class T, T Cell_Data::*Member> struct Getter {
	Stale* stale;
	T& data(Cell_Data& c) const { return c.*Member; }
	Stale& type() const { return *stale; }
};

using Grid = oracle_shim::Uniform_Grid<Cell_Data>;

// the options' per-cell exponents: an expression evaluated at a cell's centre, here a lookup
struct Per_Cell_Expression {
	const Grid* grid;
	const int32_t* values;
	double evaluate(double, const double x, const double y, const double z, double, double, double) const
	{
		const auto& g = grid->geometry;
		const int i = int(std::floor(x / g.len[0])), j = int(std::floor(y / g.len[1])),
			k = int(std::floor(z / g.len[2]));
		return values[i + size_t(g.n[0]) * (j + size_t(g.n[1]) * k)];
	}
};

struct Options {
	int substep_min_i = -1, substep_max_i = -1;
	Per_Cell_Expression substep_min_e, substep_max_e;
};

} // namespace

/*
The substep plan of one step: per-cell CFL limits (Timestep), the options'
smallest and largest exponent per cell (x fastest), the step's cap max_dt.
Writes every cell's period (2^exponent), the substep length and the
largest period.  Returns 0, or 1 with the message of a thrown exception
(the reference aborts on unexpected substeps).
*/
extern "C" int ref_substep_plan(const int32_t n[3], const double cell_length[3], const double* limits,
                                const int32_t* smin, const int32_t* smax, const double max_dt,
                                int32_t* periods, double* substep, int32_t* max_period)
{
	try {
		Grid grid({n[0], n[1], n[2]}, {cell_length[0], cell_length[1], cell_length[2]});
		Stale s_type, s_step, s_min, s_max, s_dt;
		const Getter<int, &Cell_Data::ctype> CType{&s_type};
		const Getter<double, &Cell_Data::timestep> Timestep{&s_dt};
		const Getter<int, &Cell_Data::substep> Substep{&s_step};
		const Getter<int, &Cell_Data::substep_min> Substep_Min{&s_min};
		const Getter<int, &Cell_Data::substep_max> Substep_Max{&s_max};
		Options options;
		options.substep_min_e = {&grid, smin};
		options.substep_max_e = {&grid, smax};
		pamhd::set_minmax_substepping_period(0.0, grid, options, Substep_Min, Substep_Max);
		for (size_t c = 0; c < grid.data.size(); c++) grid.data[c].timestep = limits[c];
		*substep = pamhd::set_minmax_substepping_period(grid, max_dt, CType, Timestep, Substep_Min, Substep_Max);
		pamhd::restrict_substepping_period(grid, Substep, Substep_Max, CType);
		*max_period = pamhd::update_substeps(grid, CType, Substep);
		for (size_t c = 0; c < grid.data.size(); c++) periods[c] = grid.data[c].substep;
		return 0;
	} catch (const std::exception& e) {
		std::cerr << e.what() << std::endl;
		return 1;
	}
}
