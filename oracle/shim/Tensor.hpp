/* Test infrastructure (oracle reference build): Tensor<rank, T> as nested
 * fixed-size arrays indexed with [].  Constructed unset (the GRHD headers
 * initialise every tensor they accumulate into), from one value (every
 * entry set to it: `Tensor<2, double> h = 0.0;`), or a rank-1 tensor from
 * a list of its entries (`{a, b, c}`). */
#ifndef SHIM_TENSOR_HPP_
#define SHIM_TENSOR_HPP_

#include "DimensionDefinitions.hpp"
#include <initializer_list>

template <int rank, class data_t, int size = DEFAULT_TENSOR_DIM> class Tensor
{
  public:
    Tensor() {}
    Tensor(const data_t &v)
    {
        for (int i = 0; i < size; ++i)
            arr[i] = v;
    }
    Tensor<rank - 1, data_t, size> &operator[](int i) { return arr[i]; }
    const Tensor<rank - 1, data_t, size> &operator[](int i) const
    {
        return arr[i];
    }

  private:
    Tensor<rank - 1, data_t, size> arr[size];
};

template <class data_t, int size> class Tensor<1, data_t, size>
{
  public:
    Tensor() {}
    Tensor(const data_t &v)
    {
        for (int i = 0; i < size; ++i)
            arr[i] = v;
    }
    Tensor(std::initializer_list<data_t> list)
    {
        int i = 0;
        for (const data_t &v : list)
            if (i < size)
                arr[i++] = v;
    }
    data_t &operator[](int i) { return arr[i]; }
    const data_t &operator[](int i) const { return arr[i]; }

  private:
    data_t arr[size];
};

#endif
