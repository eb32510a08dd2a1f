/*
Minimal stand-in for the gensimcell cell container, written for this
project so that the reference's header-only MHD solvers can be compiled
without the (empty) gensimcell submodule.

TEST INFRASTRUCTURE ONLY: it is used by the oracle build recipe
(oracle/Makefile) and by nothing that ships.

A cell is a tuple of tagged variables; cell[Tag()] returns a reference to
the value of type Tag::data_type.  Storage and indexing only: there is no
arithmetic, no MPI transfer logic (set_transfer_all does nothing) and no
I/O.
*/
#ifndef ORACLE_GENSIMCELL_STANDIN_HPP
#define ORACLE_GENSIMCELL_STANDIN_HPP

#include <cstddef>
#include <tuple>
#include <type_traits>

namespace gensimcell {

struct Never_Transfer {};
struct Always_Transfer {};
struct Optional_Transfer {};

namespace standin {
template <class Wanted, class... Tags> struct position;
template <class Wanted, class... Rest>
struct position<Wanted, Wanted, Rest...> : std::integral_constant<std::size_t, 0> {};
template <class Wanted, class First, class... Rest>
struct position<Wanted, First, Rest...>
	: std::integral_constant<std::size_t, 1 + position<Wanted, Rest...>::value> {};
}

template <class Transfer_Policy, class... Tags> class Cell {
	std::tuple<typename Tags::data_type...> values{};

public:
	// which variables MPI would transfer: nothing to transfer on one rank
	template <class... Variables> static void set_transfer_all(const bool, const Variables&...) {}

	template <class Tag> typename Tag::data_type& operator[](const Tag&)
	{
		return std::get<standin::position<Tag, Tags...>::value>(values);
	}

	template <class Tag> const typename Tag::data_type& operator[](const Tag&) const
	{
		return std::get<standin::position<Tag, Tags...>::value>(values);
	}
};

} // namespace gensimcell

#endif
