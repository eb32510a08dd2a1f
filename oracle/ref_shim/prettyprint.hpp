/*
Stand-in for the prettyprint library header (a submodule absent from the
reference tree) so that tests/mhd/two_reference.cpp compiles unchanged:
stream output of std::array, which the program prints in its diagnostics.
No arithmetic.  TEST INFRASTRUCTURE.
*/
#ifndef ORACLE_SHIM_PRETTYPRINT_HPP
#define ORACLE_SHIM_PRETTYPRINT_HPP

#include <array>
#include <cstddef>
#include <ostream>

namespace std {
template <class T, size_t N>
ostream& operator<<(ostream& os, const array<T, N>& a)
{
	os << "(";
	for (size_t i = 0; i < N; i++) os << (i ? ", " : "") << a[i];
	return os << ")";
}
}

#endif
