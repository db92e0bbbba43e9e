/* Test infrastructure (oracle reference build): the Chombo names the GRHD
 * operator headers and the reference's tests use, for one process holding
 * every box of a level:
 *   IntVect, Box (inclusive cell ranges), BoxIterator (x fastest),
 *   FArrayBox (components of a box in Fortran order, filled with NaN at
 *   construction so that nothing relies on unset data), ProblemDomain
 *   (non-periodic), DisjointBoxLayout / DataIterator / DataIndex,
 *   LevelData<FArrayBox> with exchange() (ghost cells from the other
 *   boxes' valid regions) and copyTo() (the source's valid regions into
 *   the destination's boxes grown by its ghosts), Vector, Real, MayDay,
 *   pout.
 * Written from the call sites, not from Chombo. */
#ifndef SHIM_CHOMBO_H_
#define SHIM_CHOMBO_H_

#include "DimensionDefinitions.hpp"
#include <algorithm>
#include <cstdio>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

typedef double Real;

template <class T> class Vector : public std::vector<T>
{
  public:
    Vector() {}
    explicit Vector(std::size_t n) : std::vector<T>(n) {}
    Vector(std::size_t n, const T &v) : std::vector<T>(n, v) {}
};

class IntVect
{
  public:
    IntVect() : v{0, 0, 0} {}
    IntVect(int a, int b, int c) : v{a, b, c} {}
    int &operator[](int d) { return v[d]; }
    const int &operator[](int d) const { return v[d]; }
    IntVect operator+(const IntVect &o) const
    {
        return IntVect(v[0] + o.v[0], v[1] + o.v[1], v[2] + o.v[2]);
    }
    IntVect operator-(const IntVect &o) const
    {
        return IntVect(v[0] - o.v[0], v[1] - o.v[1], v[2] - o.v[2]);
    }
    IntVect operator-() const { return IntVect(-v[0], -v[1], -v[2]); }
    IntVect operator*(int s) const
    {
        return IntVect(v[0] * s, v[1] * s, v[2] * s);
    }
    IntVect &operator+=(const IntVect &o)
    {
        for (int d = 0; d < 3; ++d)
            v[d] += o.v[d];
        return *this;
    }
    IntVect &operator-=(const IntVect &o)
    {
        for (int d = 0; d < 3; ++d)
            v[d] -= o.v[d];
        return *this;
    }
    bool operator==(const IntVect &o) const
    {
        return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2];
    }
    bool operator!=(const IntVect &o) const { return !(*this == o); }
    static const IntVect Zero;
    static const IntVect Unit;

  private:
    int v[3];
};
inline IntVect operator*(int s, const IntVect &a) { return a * s; }
inline std::ostream &operator<<(std::ostream &os, const IntVect &a)
{
    return os << "(" << a[0] << "," << a[1] << "," << a[2] << ")";
}
inline const IntVect IntVect::Zero = IntVect(0, 0, 0);
inline const IntVect IntVect::Unit = IntVect(1, 1, 1);
inline IntVect BASISV(int d)
{
    IntVect e;
    e[d] = 1;
    return e;
}

class Box
{
  public:
    Box() : m_lo(0, 0, 0), m_hi(-1, -1, -1) {}
    Box(const IntVect &lo, const IntVect &hi) : m_lo(lo), m_hi(hi) {}
    const IntVect &smallEnd() const { return m_lo; }
    const IntVect &bigEnd() const { return m_hi; }
    int smallEnd(int d) const { return m_lo[d]; }
    int bigEnd(int d) const { return m_hi[d]; }
    bool isEmpty() const
    {
        return m_hi[0] < m_lo[0] || m_hi[1] < m_lo[1] || m_hi[2] < m_lo[2];
    }
    bool ok() const { return !isEmpty(); }
    long long numPts() const
    {
        return isEmpty() ? 0
                         : (long long)(m_hi[0] - m_lo[0] + 1) *
                               (m_hi[1] - m_lo[1] + 1) *
                               (m_hi[2] - m_lo[2] + 1);
    }
    int size(int d) const { return m_hi[d] - m_lo[d] + 1; }
    bool contains(const IntVect &p) const
    {
        for (int d = 0; d < 3; ++d)
            if (p[d] < m_lo[d] || p[d] > m_hi[d])
                return false;
        return true;
    }
    bool contains(const Box &b) const
    {
        return b.isEmpty() || (contains(b.m_lo) && contains(b.m_hi));
    }
    Box &grow(int n) { return grow(IntVect(n, n, n)); }
    Box &grow(const IntVect &n)
    {
        m_lo -= n;
        m_hi += n;
        return *this;
    }
    Box &grow(int d, int n)
    {
        m_lo[d] -= n;
        m_hi[d] += n;
        return *this;
    }
    Box &growLo(int d, int n)
    {
        m_lo[d] -= n;
        return *this;
    }
    Box &growHi(int d, int n)
    {
        m_hi[d] += n;
        return *this;
    }
    Box &shift(const IntVect &s)
    {
        m_lo += s;
        m_hi += s;
        return *this;
    }
    Box operator&(const Box &o) const
    {
        IntVect lo, hi;
        for (int d = 0; d < 3; ++d)
        {
            lo[d] = std::max(m_lo[d], o.m_lo[d]);
            hi[d] = std::min(m_hi[d], o.m_hi[d]);
        }
        return Box(lo, hi);
    }
    Box &operator&=(const Box &o) { return *this = *this & o; }
    bool operator==(const Box &o) const
    {
        return m_lo == o.m_lo && m_hi == o.m_hi;
    }

  private:
    IntVect m_lo, m_hi;
};
inline Box grow(const Box &b, int n)
{
    Box g = b;
    return g.grow(n);
}
inline Box grow(const Box &b, const IntVect &n)
{
    Box g = b;
    return g.grow(n);
}

class BoxIterator
{
  public:
    BoxIterator() {}
    explicit BoxIterator(const Box &b) : m_box(b) { begin(); }
    void define(const Box &b)
    {
        m_box = b;
        begin();
    }
    void begin() { m_cur = m_box.smallEnd(); }
    bool ok() const
    {
        return !m_box.isEmpty() && m_cur[2] <= m_box.bigEnd(2);
    }
    void operator++()
    {
        if (++m_cur[0] > m_box.bigEnd(0))
        {
            m_cur[0] = m_box.smallEnd(0);
            if (++m_cur[1] > m_box.bigEnd(1))
            {
                m_cur[1] = m_box.smallEnd(1);
                ++m_cur[2];
            }
        }
    }
    const IntVect &operator()() const { return m_cur; }

  private:
    Box m_box;
    IntVect m_cur;
};

class Interval
{
  public:
    Interval(int a, int b) : m_a(a), m_b(b) {}
    int begin() const { return m_a; }
    int end() const { return m_b; }
    int size() const { return m_b - m_a + 1; }

  private:
    int m_a, m_b;
};

class FArrayBox
{
  public:
    FArrayBox() : m_ncomp(0) {}
    FArrayBox(const Box &b, int ncomp) { define(b, ncomp); }
    void define(const Box &b, int ncomp)
    {
        m_box = b;
        m_ncomp = ncomp;
        m_data.assign((std::size_t)b.numPts() * ncomp,
                      std::numeric_limits<double>::quiet_NaN());
    }
    const Box &box() const { return m_box; }
    int nComp() const { return m_ncomp; }
    long long index(const IntVect &p) const
    {
        const Box &b = m_box;
        return (long long)(p[0] - b.smallEnd(0)) +
               (long long)b.size(0) *
                   ((p[1] - b.smallEnd(1)) +
                    (long long)b.size(1) * (p[2] - b.smallEnd(2)));
    }
    Real &operator()(const IntVect &p, int comp = 0)
    {
        return m_data[index(p) + (std::size_t)comp * m_box.numPts()];
    }
    const Real &operator()(const IntVect &p, int comp = 0) const
    {
        return m_data[index(p) + (std::size_t)comp * m_box.numPts()];
    }
    void setVal(Real v) { std::fill(m_data.begin(), m_data.end(), v); }
    void setVal(Real v, int comp)
    {
        std::fill(m_data.begin() + (std::size_t)comp * m_box.numPts(),
                  m_data.begin() + (std::size_t)(comp + 1) * m_box.numPts(),
                  v);
    }
    void setVal(Real v, const Box &region, int comp, int ncomp = 1)
    {
        const Box r = region & m_box;
        for (BoxIterator bit(r); bit.ok(); ++bit)
            for (int c = comp; c < comp + ncomp; ++c)
                (*this)(bit(), c) = v;
    }
    /* the components of src over the overlap of the two boxes */
    void copy(const FArrayBox &src)
    {
        copy(src, m_box & src.m_box, 0, 0, std::min(m_ncomp, src.m_ncomp));
    }
    void copy(const FArrayBox &src, const Box &region, int src_comp,
              int dst_comp, int ncomp)
    {
        const Box r = region & m_box & src.m_box;
        for (BoxIterator bit(r); bit.ok(); ++bit)
            for (int c = 0; c < ncomp; ++c)
                (*this)(bit(), dst_comp + c) = src(bit(), src_comp + c);
    }
    Real *dataPtr(int comp = 0)
    {
        return m_data.data() + (std::size_t)comp * m_box.numPts();
    }
    const Real *dataPtr(int comp = 0) const
    {
        return m_data.data() + (std::size_t)comp * m_box.numPts();
    }

  private:
    Box m_box;
    int m_ncomp;
    std::vector<Real> m_data;
};

class ProblemDomain
{
  public:
    ProblemDomain() {}
    explicit ProblemDomain(const Box &b) : m_box(b) {}
    const Box &domainBox() const { return m_box; }
    bool isPeriodic(int) const { return false; }
    bool isPeriodic() const { return false; }
    bool contains(const IntVect &p) const { return m_box.contains(p); }

  private:
    Box m_box;
};

class DataIndex
{
  public:
    DataIndex() : m_i(0) {}
    explicit DataIndex(int i) : m_i(i) {}
    int intCode() const { return m_i; }
    bool operator==(const DataIndex &o) const { return m_i == o.m_i; }

  private:
    int m_i;
};

class DataIterator
{
  public:
    DataIterator() : m_n(0), m_i(0) {}
    explicit DataIterator(int n) : m_n(n), m_i(0) {}
    void begin() { m_i = 0; }
    bool ok() const { return m_i < m_n; }
    void operator++() { ++m_i; }
    DataIndex operator()() const { return DataIndex(m_i); }
    operator DataIndex() const { return DataIndex(m_i); }
    void reset() { begin(); }

  private:
    int m_n, m_i;
};
typedef DataIterator LayoutIterator;

class DisjointBoxLayout
{
  public:
    DisjointBoxLayout() {}
    DisjointBoxLayout(const Vector<Box> &boxes, const Vector<int> &,
                      const ProblemDomain &domain)
        : m_boxes(boxes.begin(), boxes.end()), m_domain(domain)
    {
    }
    DisjointBoxLayout(const Vector<Box> &boxes, const Vector<int> &)
        : m_boxes(boxes.begin(), boxes.end())
    {
    }
    void close() {}
    DataIterator dataIterator() const { return DataIterator(size()); }
    LayoutIterator layoutIterator() const { return DataIterator(size()); }
    int size() const { return (int)m_boxes.size(); }
    const Box &operator[](const DataIndex &i) const
    {
        return m_boxes[i.intCode()];
    }
    const Box &operator[](const DataIterator &i) const
    {
        return (*this)[i()];
    }
    const ProblemDomain &physDomain() const { return m_domain; }
    int procID(const DataIndex &) const { return 0; }

  private:
    std::vector<Box> m_boxes;
    ProblemDomain m_domain;
};

template <class T> class LevelData
{
  public:
    LevelData() : m_ncomp(0) {}
    LevelData(const DisjointBoxLayout &grids, int ncomp,
              const IntVect &ghost = IntVect::Zero)
    {
        define(grids, ncomp, ghost);
    }
    void define(const DisjointBoxLayout &grids, int ncomp,
                const IntVect &ghost = IntVect::Zero)
    {
        m_grids = grids;
        m_ncomp = ncomp;
        m_ghost = ghost;
        m_fabs.clear();
        m_fabs.resize(grids.size());
        for (int i = 0; i < grids.size(); ++i)
            m_fabs[i].define(::grow(grids[DataIndex(i)], ghost), ncomp);
    }
    const DisjointBoxLayout &disjointBoxLayout() const { return m_grids; }
    const DisjointBoxLayout &getBoxes() const { return m_grids; }
    DataIterator dataIterator() const { return m_grids.dataIterator(); }
    const IntVect &ghostVect() const { return m_ghost; }
    int nComp() const { return m_ncomp; }
    T &operator[](const DataIndex &i) { return m_fabs[i.intCode()]; }
    const T &operator[](const DataIndex &i) const
    {
        return m_fabs[i.intCode()];
    }
    T &operator[](const DataIterator &i) { return (*this)[i()]; }
    const T &operator[](const DataIterator &i) const { return (*this)[i()]; }

    /* ghost cells of every box from the other boxes' valid regions */
    void exchange()
    {
        for (int i = 0; i < m_grids.size(); ++i)
            for (int j = 0; j < m_grids.size(); ++j)
            {
                if (i == j)
                    continue;
                const Box overlap = m_fabs[i].box() & m_grids[DataIndex(j)];
                if (!overlap.isEmpty())
                    m_fabs[i].copy(m_fabs[j], overlap, 0, 0, m_ncomp);
            }
    }
    /* the valid regions of this into dest's boxes grown by its ghosts */
    void copyTo(LevelData<T> &dest) const
    {
        const int nc = std::min(m_ncomp, dest.m_ncomp);
        for (int i = 0; i < dest.m_grids.size(); ++i)
            for (int j = 0; j < m_grids.size(); ++j)
            {
                const Box overlap =
                    dest.m_fabs[i].box() & m_grids[DataIndex(j)];
                if (!overlap.isEmpty())
                    dest.m_fabs[i].copy(m_fabs[j], overlap, 0, 0, nc);
            }
    }

  private:
    DisjointBoxLayout m_grids;
    int m_ncomp;
    IntVect m_ghost;
    std::vector<T> m_fabs;
};

namespace MayDay
{
[[noreturn]] inline void Error(const char *msg = "MayDay::Error")
{
    throw std::runtime_error(msg);
}
[[noreturn]] inline void Abort(const char *msg = "MayDay::Abort")
{
    throw std::runtime_error(msg);
}
inline void Warning(const char *msg) { std::cerr << msg << "\n"; }
} // namespace MayDay

inline std::ostream &pout() { return std::cout; }
inline int procID() { return 0; }
inline int numProc() { return 1; }

#endif
