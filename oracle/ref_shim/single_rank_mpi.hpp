/*
Stand-in for the few MPI calls of the reference's substepping.hpp, for one
rank: a reduction over one rank is a copy.  Interface only, no arithmetic.
TEST INFRASTRUCTURE (oracle/ref_substep_bridge.cpp).
*/
#ifndef PAMHD_ORACLE_SINGLE_RANK_MPI_HPP
#define PAMHD_ORACLE_SINGLE_RANK_MPI_HPP

#include <cstdint>
#include <cstring>

using MPI_Comm = int;
enum MPI_Datatype { MPI_INT, MPI_UINT64_T, MPI_DOUBLE };
enum MPI_Op { MPI_MAX, MPI_MIN, MPI_SUM };
constexpr int MPI_SUCCESS = 0;

inline int MPI_Allreduce(const void* in, void* out, const int count, const MPI_Datatype type, MPI_Op, MPI_Comm)
{
	const size_t size = type == MPI_INT ? sizeof(int) : (type == MPI_UINT64_T ? sizeof(uint64_t) : sizeof(double));
	std::memcpy(out, in, size * size_t(count));
	return MPI_SUCCESS;
}

inline int MPI_Comm_free(MPI_Comm*)
{
	return MPI_SUCCESS;
}

#endif
