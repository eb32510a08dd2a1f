/*
Stand-in for the dccrg header the reference's solver sources include: the
one-rank uniform box of box_grid.hpp is the grid they are instantiated
with.  TEST INFRASTRUCTURE (oracle/ref_stag_bridge.cpp).
*/
#ifndef PAMHD_ORACLE_DCCRG_STANDIN_HPP
#define PAMHD_ORACLE_DCCRG_STANDIN_HPP
#include "box_grid.hpp"
#endif
