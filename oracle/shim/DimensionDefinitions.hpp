/* Test infrastructure (oracle reference build): the dimension macros the
 * GRHD headers use.  Three dimensions only. */
#ifndef SHIM_DIMENSIONDEFINITIONS_HPP_
#define SHIM_DIMENSIONDEFINITIONS_HPP_

#ifndef CH_SPACEDIM
#define CH_SPACEDIM 3
#endif
#define SpaceDim CH_SPACEDIM
#define DEFAULT_TENSOR_DIM CH_SPACEDIM
#define D_DECL(a, b, c) a, b, c

/* FOR(i), FOR(i, j), FOR(i, j, k), FOR(i, j, k, l): nested loops over
 * 0..CH_SPACEDIM-1, the first index outermost; FOR1..FOR4 the same by
 * count. */
#define FOR1(i) for (int i = 0; i < CH_SPACEDIM; ++i)
#define FOR2(i, j) FOR1(i) FOR1(j)
#define FOR3(i, j, k) FOR2(i, j) FOR1(k)
#define FOR4(i, j, k, l) FOR3(i, j, k) FOR1(l)
#define SHIM_FOR_PICK(_1, _2, _3, _4, NAME, ...) NAME
#define FOR(...)                                                              \
    SHIM_FOR_PICK(__VA_ARGS__, FOR4, FOR3, FOR2, FOR1, unused)(__VA_ARGS__)

#endif
