/*
Empty stand-in for the rapidjson header that mhd/solar_wind_box.hpp
includes: the functions of that header used by oracle/ref_stag_bridge.cpp
take their options as plain structures and parse nothing.
TEST INFRASTRUCTURE (oracle/ref_stag_bridge.cpp).
*/
#ifndef PAMHD_ORACLE_RAPIDJSON_STANDIN_HPP
#define PAMHD_ORACLE_RAPIDJSON_STANDIN_HPP
namespace rapidjson {}
#endif
