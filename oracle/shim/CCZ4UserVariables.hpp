/* Test infrastructure (oracle reference build): the 25 CCZ4 evolution
 * variables in the order the CCZ4-geometry operator reads them (chi,
 * h_ij, K, A_ij, Theta, Gamma^i, lapse, shift^i, B^i); the GRHD
 * components follow them in the tests' UserVariables.hpp. */
#ifndef SHIM_CCZ4USERVARIABLES_HPP_
#define SHIM_CCZ4USERVARIABLES_HPP_
#include <array>
#include <string>
enum
{
    c_chi,
    c_h11,
    c_h12,
    c_h13,
    c_h22,
    c_h23,
    c_h33,
    c_K,
    c_A11,
    c_A12,
    c_A13,
    c_A22,
    c_A23,
    c_A33,
    c_Theta,
    c_Gamma1,
    c_Gamma2,
    c_Gamma3,
    c_lapse,
    c_shift1,
    c_shift2,
    c_shift3,
    c_B1,
    c_B2,
    c_B3,
    NUM_CCZ4_VARS
};
namespace CCZ4Variables
{
static const std::array<std::string, NUM_CCZ4_VARS> names = {
    "chi",    "h11",    "h12",    "h13",    "h22", "h23", "h33",
    "K",      "A11",    "A12",    "A13",    "A22", "A23", "A33",
    "Theta",  "Gamma1", "Gamma2", "Gamma3", "lapse", "shift1", "shift2",
    "shift3", "B1",     "B2",     "B3"};
}
static const std::array<std::string, NUM_CCZ4_VARS> ccz4_variable_names =
    CCZ4Variables::names;
#endif
