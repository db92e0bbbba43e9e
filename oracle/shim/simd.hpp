/* Test infrastructure (oracle reference build): scalar code only. */
#ifndef SHIM_SIMD_HPP_
#define SHIM_SIMD_HPP_
struct disable_simd
{
};
#endif
