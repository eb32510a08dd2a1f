/*
Empty stand-in for boost/lexical_cast.hpp: tests/mhd/reference.cpp includes
it but calls nothing from it.  TEST INFRASTRUCTURE ONLY.
*/
#ifndef ORACLE_BOOST_LEXICAL_CAST_STANDIN_HPP
#define ORACLE_BOOST_LEXICAL_CAST_STANDIN_HPP
#endif
