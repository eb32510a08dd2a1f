/*
Stand-in for the variable tags of the reference's mhd/variables.hpp,
force-included (g++ -include) before the reference sources so that the real
header's include guard skips it.  The real header pulls in the AMR and grid
option headers, which need muparserx and rapidjson (absent here).

TEST INFRASTRUCTURE ONLY (oracle build recipe).

The tags below carry the same names and data types as the reference's
(mhd/variables.hpp:57-135 for the scalar/vector tags, :151-176 for the HD
containers, :240 for detail::MHD) because the reference solver templates
index cells by these exact types.  Nothing else from that header is needed
by the solver headers or by tests/mhd/reference.cpp.
*/
#ifndef ORACLE_REF_VARIABLES_STANDIN_HPP
#define ORACLE_REF_VARIABLES_STANDIN_HPP

// make the reference's own mhd/variables.hpp a no-op
#define PAMHD_MHD_VARIABLES_HPP

// standard headers the reference sources use without including them
// (in the full build they arrive through dccrg and boost)
#include <algorithm>
#include <array>
#include <cmath>
#include <functional>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "gensimcell.hpp"
#include "common_variables.hpp"

namespace pamhd {
namespace mhd {

struct Mass_Density { using data_type = double; };
struct Momentum_Density { using data_type = std::array<double, 3>; };
struct Total_Energy_Density { using data_type = double; };
struct Velocity { using data_type = std::array<double, 3>; };
struct Pressure { using data_type = double; };
struct Number_Density { using data_type = double; };

using HD_Conservative = gensimcell::Cell<
	gensimcell::Always_Transfer,
	Mass_Density, Momentum_Density, Total_Energy_Density>;

using HD_Primitive = gensimcell::Cell<
	gensimcell::Never_Transfer,
	Mass_Density, Velocity, Pressure>;

struct HD_State_Conservative { using data_type = HD_Conservative; };
struct HD_Flux_Conservative { using data_type = HD_Conservative; };
// the second population of tests/mhd/two_reference.cpp (mhd/variables.hpp:163-164)
struct HD2_State_Conservative { using data_type = HD_Conservative; };
struct HD2_Flux_Conservative { using data_type = HD_Conservative; };

namespace detail {
using MHD = gensimcell::Cell<
	gensimcell::Never_Transfer,
	pamhd::mhd::Mass_Density,
	pamhd::mhd::Momentum_Density,
	pamhd::mhd::Total_Energy_Density,
	pamhd::Magnetic_Field>;
}

}} // namespaces

#endif
