// Test infrastructure only: stand-in for schnek::Array, a fixed-size value
// array used by MPulse as grid index and 3-vector (mpulse.h:17-26).
#ifndef MPB_REFSHIM_SCHNEK_ARRAY_HPP
#define MPB_REFSHIM_SCHNEK_ARRAY_HPP

namespace schnek {

template <class T, int N>
class Array {
 public:
  Array() { for (int n = 0; n < N; ++n) v_[n] = T(); }
  Array(T a) {  // implicit: MPulse passes plain ints as 1-D indices (cpml_border.cpp:308)
    for (int n = 0; n < N; ++n) v_[n] = a; }
  Array(T a, T b) { fill(); v_[0] = a; if (N > 1) v_[1] = b; }
  Array(T a, T b, T c) { fill(); v_[0] = a; if (N > 1) v_[1] = b; if (N > 2) v_[2] = c; }

  T &operator[](int n) { return v_[n]; }
  const T &operator[](int n) const { return v_[n]; }

  bool operator==(const Array &o) const {
    for (int n = 0; n < N; ++n)
      if (!(v_[n] == o.v_[n])) return false;
    return true;
  }
  bool operator!=(const Array &o) const { return !(*this == o); }

 private:
  void fill() { for (int n = 0; n < N; ++n) v_[n] = T(); }
  T v_[N];
};

}  // namespace schnek

#endif
