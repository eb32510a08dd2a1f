/*
liboracle.so: the restated solvers (mhd_oracle.hpp) behind the oracle C
entry points (capi_body.hpp), plus the restated 1-D golden generator.

TEST INFRASTRUCTURE - see mhd_oracle.hpp for who may use this.
*/
#define ORACLE_API(name) oracle_##name
#define ORACLE_FLUX oracle::Restated_Solvers
#define ORACLE_SPLIT oracle::Restated_Split_Solvers
#include "capi_body.hpp"

extern "C" {

/*
The scheme of tests/mhd/reference.cpp (see oracle::reference_1d); returns
the number of steps or -1 when a solver or the positivity check threw.
*/
int32_t oracle_reference_1d(int32_t solver, int32_t cells, double t_end, double length, double* out)
{
	try {
		return oracle::reference_1d(oracle::Restated_Solvers{}, solver, cells, t_end, length, out);
	} catch (const std::exception& e) {
		last_error = e.what();
		return -1;
	}
}

}
