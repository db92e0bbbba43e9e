/* Test infrastructure (oracle reference build): the cell handle the
 * backgrounds' compute(Cell) methods take.  Those methods are not on the
 * operator path; the handle only has to carry its index. */
#ifndef SHIM_CELL_HPP_
#define SHIM_CELL_HPP_

#include "IntVect.H"

template <class data_t> class Cell
{
  public:
    explicit Cell(const IntVect &iv) : m_iv(iv) {}
    const IntVect &get_int_vect() const { return m_iv; }
    template <class value_t> void store_vars(const value_t &, int) const {}
    template <class vars_t> void store_vars(const vars_t &) const {}

  private:
    IntVect m_iv;
};

#endif
