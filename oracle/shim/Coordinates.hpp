/* Test infrastructure (oracle reference build): cell-centred coordinates
 * relative to a centre, x = (i + 1/2) dx - centre_x, and the coordinate
 * radius clamped below at 1e-6 (the convention the reference's recorded
 * golden values confirm through the oracle). */
#ifndef SHIM_COORDINATES_HPP_
#define SHIM_COORDINATES_HPP_

#include "Cell.hpp"
#include "DimensionDefinitions.hpp"
#include "IntVect.H"
#include <algorithm>
#include <array>
#include <cmath>

template <class data_t> class Coordinates
{
  public:
    data_t x;
    double y, z;

    Coordinates(const IntVect &iv, double dx,
                const std::array<double, CH_SPACEDIM> &center)
    {
        x = (iv[0] + 0.5) * dx - center[0];
        y = (iv[1] + 0.5) * dx - center[1];
        z = (iv[2] + 0.5) * dx - center[2];
    }

    Coordinates(const Cell<data_t> &cell, double dx,
                const std::array<double, CH_SPACEDIM> &center)
        : Coordinates(cell.get_int_vect(), dx, center)
    {
    }

    data_t get_radius() const
    {
        const data_t r = std::sqrt(x * x + y * y + z * z);
        return std::max(r, data_t(1.0e-6));
    }
};

#endif
