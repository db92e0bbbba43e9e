/* Test infrastructure (oracle reference build): the TensorAlgebra
 * functions the GRHD headers and backgrounds call, restated from their
 * mathematics with the same operation order as the oracle's restatement
 * (oracle/grhd_oracle.c: det_sym, inverse_sym, christoffel_ULL, trace_sym,
 * dot_metric): symmetric 3x3 determinant and inverse by cofactors,
 * Christoffel symbols of the first and second kind, traces and
 * contractions with a metric. */
#ifndef SHIM_TENSORALGEBRA_HPP_
#define SHIM_TENSORALGEBRA_HPP_

#include "DimensionDefinitions.hpp"
#include "Tensor.hpp"

template <class data_t> struct chris_t
{
    Tensor<3, data_t> ULL; /* Gamma^i_jk */
    Tensor<3, data_t> LLL; /* Gamma_ijk */
    Tensor<1, data_t> contracted;
};

namespace TensorAlgebra
{
inline double delta(int i, int j) { return i == j ? 1.0 : 0.0; }

template <class data_t>
data_t compute_determinant_sym(const Tensor<2, data_t> &m)
{
    return m[0][0] * m[1][1] * m[2][2] + 2 * m[0][1] * m[0][2] * m[1][2] -
           m[0][0] * m[1][2] * m[1][2] - m[1][1] * m[0][2] * m[0][2] -
           m[2][2] * m[0][1] * m[0][1];
}

template <class data_t>
Tensor<2, data_t> compute_inverse_sym(const Tensor<2, data_t> &m)
{
    const data_t det = compute_determinant_sym(m);
    Tensor<2, data_t> out;
    out[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[1][2]) / det;
    out[0][1] = (m[0][2] * m[1][2] - m[0][1] * m[2][2]) / det;
    out[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) / det;
    out[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[0][2]) / det;
    out[1][2] = (m[0][1] * m[0][2] - m[0][0] * m[1][2]) / det;
    out[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[0][1]) / det;
    out[1][0] = out[0][1];
    out[2][0] = out[0][2];
    out[2][1] = out[1][2];
    return out;
}

/* sum_ij m_ij g^ij (either argument order: both are symmetric) */
template <class data_t>
data_t compute_trace(const Tensor<2, data_t> &a, const Tensor<2, data_t> &b)
{
    data_t t = 0;
    FOR(i, j) { t += b[i][j] * a[i][j]; }
    return t;
}

/* sum_ij a^i b^j g_ij */
template <class data_t>
data_t compute_dot_product(const Tensor<1, data_t> &a,
                           const Tensor<1, data_t> &b,
                           const Tensor<2, data_t> &g)
{
    data_t d = 0;
    FOR(i, j) { d += a[i] * b[j] * g[i][j]; }
    return d;
}

/* v_i = g_ij v^j */
template <class data_t>
Tensor<1, data_t> lower_all(const Tensor<1, data_t> &v,
                            const Tensor<2, data_t> &g)
{
    Tensor<1, data_t> out;
    FOR(i)
    {
        out[i] = 0;
        FOR(j) { out[i] += g[i][j] * v[j]; }
    }
    return out;
}

/* Gamma_ijk = 1/2 (d_k g_ij + d_j g_ik - d_i g_jk), d1[i][j][k] = d_k g_ij;
 * Gamma^i_jk = g^il Gamma_ljk */
template <class data_t>
chris_t<data_t>
compute_christoffel(const Tensor<2, Tensor<1, data_t>> &d1,
                    const Tensor<2, data_t> &gUU)
{
    chris_t<data_t> out;
    FOR(i, j, k)
    {
        out.LLL[i][j][k] =
            0.5 * (d1[j][i][k] + d1[k][i][j] - d1[j][k][i]);
    }
    FOR(i, j, k)
    {
        out.ULL[i][j][k] = 0;
        FOR(l) { out.ULL[i][j][k] += gUU[i][l] * out.LLL[l][j][k]; }
    }
    FOR(i)
    {
        out.contracted[i] = 0;
        FOR(j, k) { out.contracted[i] += gUU[j][k] * out.ULL[i][j][k]; }
    }
    return out;
}
} // namespace TensorAlgebra

#endif
