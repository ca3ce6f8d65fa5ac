// Test infrastructure only: a stand-in for the subset of the schnek grid
// library that MPulse's sources use (schnek is not vendored with MPulse and
// its version is unpinned).  Only the behaviour MPulse relies on is provided:
//   * inclusive index ranges [low, high] per dimension (mpulse.h:13-26,
//     globals.cpp:74-75, storage.cpp:30-46);
//   * C order, i.e. the LAST index runs fastest, which matches the k-innermost
//     loops of fdtd_plrc.t:221-233;
//   * resize(), element access by operator(), assignment of a scalar to every
//     element, getLow()/getHigh()/getDims().
// No bounds checks: MPulse is built with -DNDEBUG for the oracle.
#ifndef MPB_REFSHIM_SCHNEK_GRID_HPP
#define MPB_REFSHIM_SCHNEK_GRID_HPP

#include "array.hpp"
#include <cstddef>
#include <vector>

namespace schnek {

template <int Rank> struct GridNoArgCheck {};
template <int Rank> struct GridAssertCheck {};

template <class T, int Rank, template <int> class Checker = GridNoArgCheck>
class Grid {
 public:
  typedef Array<int, Rank> IndexType;
  typedef T value_type;

  Grid() { IndexType z(0); resize(z, z); }
  Grid(const IndexType &lo, const IndexType &hi) { resize(lo, hi); }
  explicit Grid(const IndexType &dims) { resize(dims); }

  void resize(const IndexType &lo, const IndexType &hi) {
    lo_ = lo;
    hi_ = hi;
    std::size_t total = 1;
    for (int d = 0; d < Rank; ++d) {
      ext_[d] = hi[d] - lo[d] + 1;
      if (ext_[d] < 0) ext_[d] = 0;
      total *= std::size_t(ext_[d]);
    }
    // stride of the last dimension is 1 (C order)
    std::size_t s = 1;
    for (int d = Rank - 1; d >= 0; --d) {
      stride_[d] = s;
      s *= std::size_t(ext_[d]);
    }
    data_.assign(total, T());
  }
  void resize(const IndexType &dims) {
    IndexType lo(0), hi;
    for (int d = 0; d < Rank; ++d) hi[d] = dims[d] - 1;
    resize(lo, hi);
  }

  Grid &operator=(const T &v) {
    for (std::size_t n = 0; n < data_.size(); ++n) data_[n] = v;
    return *this;
  }

  T &operator()(int i) { return data_[lin1(i)]; }
  const T &operator()(int i) const { return data_[lin1(i)]; }
  T &operator()(int i, int j) { return data_[lin2(i, j)]; }
  const T &operator()(int i, int j) const { return data_[lin2(i, j)]; }
  T &operator()(int i, int j, int k) { return data_[lin3(i, j, k)]; }
  const T &operator()(int i, int j, int k) const { return data_[lin3(i, j, k)]; }
  T &operator[](const IndexType &ix) { return data_[linN(ix)]; }
  const T &operator[](const IndexType &ix) const { return data_[linN(ix)]; }

  const IndexType &getLow() const { return lo_; }
  const IndexType &getHigh() const { return hi_; }
  const IndexType &getDims() const { return ext_; }
  int getLow(int d) const { return lo_[d]; }
  int getHigh(int d) const { return hi_[d]; }
  int getDims(int d) const { return ext_[d]; }

  T *getRawData() { return data_.empty() ? 0 : &data_[0]; }
  const T *getRawData() const { return data_.empty() ? 0 : &data_[0]; }
  std::size_t getSize() const { return data_.size(); }

  typename std::vector<T>::iterator begin() { return data_.begin(); }
  typename std::vector<T>::iterator end() { return data_.end(); }
  typename std::vector<T>::const_iterator cbegin() const { return data_.begin(); }
  typename std::vector<T>::const_iterator cend() const { return data_.end(); }

 private:
  std::size_t lin1(int i) const { return std::size_t(i - lo_[0]); }
  std::size_t lin2(int i, int j) const {
    return std::size_t(i - lo_[0]) * stride_[0] + std::size_t(j - lo_[1]);
  }
  std::size_t lin3(int i, int j, int k) const {
    return std::size_t(i - lo_[0]) * stride_[0] +
           std::size_t(j - lo_[1]) * stride_[1] + std::size_t(k - lo_[2]);
  }
  std::size_t linN(const IndexType &ix) const {
    std::size_t o = 0;
    for (int d = 0; d < Rank; ++d) o += std::size_t(ix[d] - lo_[d]) * stride_[d];
    return o;
  }

  IndexType lo_, hi_, ext_;
  std::size_t stride_[Rank];
  std::vector<T> data_;
};

}  // namespace schnek

#endif
