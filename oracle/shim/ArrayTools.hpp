/* Test infrastructure (oracle reference build): concatenation of two
 * std::arrays (variable-name tables). */
#ifndef SHIM_ARRAYTOOLS_HPP_
#define SHIM_ARRAYTOOLS_HPP_
#include <array>
#include <cstddef>
namespace ArrayTools
{
template <class T, std::size_t N, std::size_t M>
std::array<T, N + M> concatenate(const std::array<T, N> &a,
                                 const std::array<T, M> &b)
{
    std::array<T, N + M> out;
    for (std::size_t i = 0; i < N; ++i)
        out[i] = a[i];
    for (std::size_t i = 0; i < M; ++i)
        out[N + i] = b[i];
    return out;
}
} // namespace ArrayTools
#endif
