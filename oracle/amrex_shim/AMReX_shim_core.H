// Minimal host-only stand-in for the handful of AMReX names that CAMR's
// hydro kernels use (Array4, Box, IntVect, GpuArray, FArrayBox, ParallelFor,
// Math::copysign/abs, min/max, grow/growHi/surroundingNodes, Geometry::Domain).
//
// This header is test infrastructure for the oracle: it lets the reference's
// own hot-path sources (Source/Hydro/**, Source/EOS/GammaLaw/EOS.H) compile
// unmodified on the CPU so that their output can pin the CPU restatement and
// the CUDA kernels.  It is written from AMReX's documented semantics:
//   * Array4 indexing: (i-lo.x) + (j-lo.y)*jstride + (k-lo.z)*kstride + n*nstride
//   * ParallelFor on the CPU: k outermost, i innermost
//   * freshly allocated FArrayBox data is NOT initialised; this shim fills it
//     with quiet NaN so that any read of a never-written slot shows up.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <type_traits>
#include <vector>

#ifndef AMREX_SPACEDIM
#define AMREX_SPACEDIM 3
#endif

#define AMREX_GPU_DEVICE
#define AMREX_GPU_HOST
#define AMREX_GPU_HOST_DEVICE
#define AMREX_FORCE_INLINE inline
#define AMREX_INLINE inline
#define AMREX_D_DECL(a, b, c) a, b, c
#define AMREX_D_TERM(a, b, c) a b c
#define AMREX_D_PICK(a, b, c) c
#define BL_PROFILE(x)
#define BL_PROFILE_VAR(x, y)
#define BL_PROFILE_VAR_STOP(x)
#define AMREX_ASSERT(x) ((void)0)
#define AMREX_ALWAYS_ASSERT(x)                                                 \
  do {                                                                         \
    if (!(x)) amrex::shim_assert_failed(#x, __FILE__, __LINE__);               \
  } while (0)
#define AMREX_ALWAYS_ASSERT_WITH_MESSAGE(x, m) AMREX_ALWAYS_ASSERT(x)

#ifdef CAMR_FLOP_COUNT
#include "camr_counted_real.H"
#endif

namespace amrex {

#ifdef CAMR_FLOP_COUNT
using Real = camr_flops::CountedReal;
#else
using Real = double;
#endif

// Assertion failures in the reference kernels are counted, not fatal, so that
// the oracle never aborts the test process; the count is read by the glue.
inline long& shim_assert_count() {
  static thread_local long c = 0;
  return c;
}
inline void shim_assert_failed(const char*, const char*, int) {
  ++shim_assert_count();
}

inline void Error(const char* msg) {
  std::fprintf(stderr, "amrex::Error (shim): %s\n", msg);
  ++shim_assert_count();
}
inline void Error(const std::string& msg) { Error(msg.c_str()); }
inline void Error() { Error("unspecified"); }
inline void Abort(const char* msg) { Error(msg); }

template <class... Ts>
inline void ignore_unused(const Ts&...) {}

template <class T>
inline const T& min(const T& a, const T& b) { return std::min(a, b); }
template <class T>
inline const T& max(const T& a, const T& b) { return std::max(a, b); }
#ifdef CAMR_FLOP_COUNT
inline Real min(Real a, Real b) { return std::min(a, b); }
inline Real max(Real a, Real b) { return std::max(a, b); }
#endif

namespace Math {
inline double copysign(double a, double b) { return std::copysign(a, b); }
inline double abs(double a) { return std::fabs(a); }
#ifdef CAMR_FLOP_COUNT
inline Real copysign(Real a, Real b) { return camr_flops::copysign(a, b); }
inline Real abs(Real a) { return camr_flops::abs(a); }
#endif
}  // namespace Math

template <class T, int N>
struct GpuArray {
  T arr[N];
  T& operator[](int i) { return arr[i]; }
  const T& operator[](int i) const { return arr[i]; }
  T* data() { return arr; }
  const T* data() const { return arr; }
};

struct IntVect {
  int v[3] = {0, 0, 0};
  IntVect() = default;
  IntVect(int a, int b, int c) { v[0] = a; v[1] = b; v[2] = c; }
  explicit IntVect(int a) { v[0] = v[1] = v[2] = a; }
  int& operator[](int i) { return v[i]; }
  int operator[](int i) const { return v[i]; }
  static IntVect TheDimensionVector(int d) {
    IntVect r; r.v[d] = 1; return r;
  }
  IntVect operator+(const IntVect& o) const {
    return IntVect(v[0] + o.v[0], v[1] + o.v[1], v[2] + o.v[2]);
  }
  IntVect operator-(const IntVect& o) const {
    return IntVect(v[0] - o.v[0], v[1] - o.v[1], v[2] - o.v[2]);
  }
};
inline IntVect operator*(int s, const IntVect& a) {
  return IntVect(s * a[0], s * a[1], s * a[2]);
}

template <class T>
struct Array4;

struct Box {
  IntVect lo, hi;
  int nodal[3] = {0, 0, 0};
  Box() = default;
  Box(const IntVect& l, const IntVect& h) : lo(l), hi(h) {}
  // The index range of an array (cell-centred).
  template <class T>
  explicit Box(const Array4<T>& a);
  Box& grow(int n) {
    for (int d = 0; d < 3; ++d) { lo[d] -= n; hi[d] += n; }
    return *this;
  }
  Box& grow(const IntVect& n) {
    for (int d = 0; d < 3; ++d) { lo[d] -= n[d]; hi[d] += n[d]; }
    return *this;
  }
  // grow by n in direction d only
  Box& grow(int d, int n) {
    lo[d] -= n;
    hi[d] += n;
    return *this;
  }
  Box& surroundingNodes() {
    for (int d = 0; d < 3; ++d)
      if (!nodal[d]) { hi[d] += 1; nodal[d] = 1; }
    return *this;
  }
  Box& operator&=(const Box& o) {
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::max(lo[d], o.lo[d]);
      hi[d] = std::min(hi[d], o.hi[d]);
    }
    return *this;
  }
  bool contains(const IntVect& p) const {
    return p[0] >= lo[0] && p[0] <= hi[0] && p[1] >= lo[1] && p[1] <= hi[1] &&
           p[2] >= lo[2] && p[2] <= hi[2];
  }
  const int* loVect() const { return lo.v; }
  const int* hiVect() const { return hi.v; }
  GpuArray<int, 3> loVect3d() const { return {{lo[0], lo[1], lo[2]}}; }
  GpuArray<int, 3> hiVect3d() const { return {{hi[0], hi[1], hi[2]}}; }
  const IntVect& smallEnd() const { return lo; }
  const IntVect& bigEnd() const { return hi; }
  long numPts() const {
    return long(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
  }
};

inline Box grow(const Box& b, int n) {
  Box r = b;
  for (int d = 0; d < 3; ++d) { r.lo[d] -= n; r.hi[d] += n; }
  return r;
}
inline Box grow(const Box& b, int d, int n) {
  Box r = b; r.lo[d] -= n; r.hi[d] += n; return r;
}
inline Box growHi(const Box& b, int d, int n) {
  Box r = b; r.hi[d] += n; return r;
}
// Face-centred box in direction d: one more point on the high side.
inline Box surroundingNodes(const Box& b, int d) {
  Box r = b;
  if (!r.nodal[d]) { r.hi[d] += 1; r.nodal[d] = 1; }
  return r;
}
inline Box surroundingNodes(const Box& b) {
  Box r = b;
  for (int d = 0; d < 3; ++d) r = surroundingNodes(r, d);
  return r;
}

template <class T>
struct Array4 {
  T* p = nullptr;
  long long jstride = 0, kstride = 0, nstride = 0;
  IntVect begin, end;  // end is one past hi
  int ncomp = 0;

  Array4() = default;
  Array4(T* ptr, const IntVect& lo, const IntVect& hi_plus_1, int nc)
      : p(ptr), begin(lo), end(hi_plus_1), ncomp(nc) {
    jstride = end[0] - begin[0];
    kstride = jstride * (end[1] - begin[1]);
    nstride = kstride * (end[2] - begin[2]);
  }
  template <class U, class = typename std::enable_if<
                         std::is_same<const U, T>::value && !std::is_same<U, T>::value>::type>
  Array4(const Array4<U>& o)
      : p(o.p), jstride(o.jstride), kstride(o.kstride), nstride(o.nstride),
        begin(o.begin), end(o.end), ncomp(o.ncomp) {}

  explicit operator bool() const { return p != nullptr; }
  T& operator()(int i, int j, int k, int n = 0) const {
    return p[(i - begin[0]) + (j - begin[1]) * jstride +
             (k - begin[2]) * kstride + n * nstride];
  }
  T& operator()(const IntVect& iv, int n = 0) const {
    return (*this)(iv[0], iv[1], iv[2], n);
  }
  bool contains(int i, int j, int k) const {
    return i >= begin[0] && i < end[0] && j >= begin[1] && j < end[1] &&
           k >= begin[2] && k < end[2];
  }
};

template <class T>
Box::Box(const Array4<T>& a)
    : lo(a.begin), hi(IntVect(a.end[0] - 1, a.end[1] - 1, a.end[2] - 1)) {}

// Node-centred version of a cell box (every direction of `t` that is 1).
inline Box convert(const Box& b, const IntVect& t) {
  Box r = b;
  for (int d = 0; d < 3; ++d)
    if (t[d] && !r.nodal[d]) { r.hi[d] += 1; r.nodal[d] = 1; }
  return r;
}

// Types named only in declarations of the reference's EB entry points.
class MFIter;
class EBFArrayBoxFactory;

struct Arena {};
inline Arena* The_Async_Arena() { return nullptr; }
inline Arena* The_Arena() { return nullptr; }

enum class RunOn { Host, Device, Gpu, Cpu };

class FArrayBox {
 public:
  FArrayBox() = default;
  FArrayBox(const Box& b, int nc, Arena* = nullptr) { resize(b, nc); }
  void resize(const Box& b, int nc, Arena* = nullptr) {
    bx_ = b; nc_ = nc;
    data_.assign(size_t(b.numPts()) * nc, Real(std::numeric_limits<double>::quiet_NaN()));
  }
  Array4<Real> array() {
    return Array4<Real>(data_.data(), bx_.lo,
                        IntVect(bx_.hi[0] + 1, bx_.hi[1] + 1, bx_.hi[2] + 1), nc_);
  }
  Array4<const Real> const_array() { return Array4<const Real>(array()); }
  template <RunOn R = RunOn::Host>
  void setVal(Real v) { std::fill(data_.begin(), data_.end(), v); }
  void clear() { data_.clear(); data_.shrink_to_fit(); }
  const Box& box() const { return bx_; }
  int nComp() const { return nc_; }

 private:
  Box bx_;
  int nc_ = 0;
  std::vector<Real> data_;
};

class Geometry {
 public:
  Geometry() = default;
  explicit Geometry(const Box& dom, const int* periodic = nullptr) : dom_(dom) {
    for (int d = 0; d < 3; ++d) per_[d] = periodic ? periodic[d] : 0;
  }
  const Box& Domain() const { return dom_; }
  bool isPeriodic(int d) const { return per_[d] != 0; }
  // The domain grown by n in its periodic directions.
  Box growPeriodicDomain(int n) const {
    Box r = dom_;
    for (int d = 0; d < 3; ++d)
      if (per_[d]) { r.lo[d] -= n; r.hi[d] += n; }
    return r;
  }
 private:
  Box dom_;
  int per_[3] = {0, 0, 0};
};

struct BCRec {
  int bc[6] = {0, 0, 0, 0, 0, 0};
  const int* lo() const { return bc; }
  const int* hi() const { return bc + 3; }
  const int* data() const { return bc; }
};

template <class F>
inline void ParallelFor(const Box& b, F&& f) {
  for (int k = b.lo[2]; k <= b.hi[2]; ++k)
    for (int j = b.lo[1]; j <= b.hi[1]; ++j)
      for (int i = b.lo[0]; i <= b.hi[0]; ++i) f(i, j, k);
}
template <class F>
inline void Loop(const Box& b, F&& f) { ParallelFor(b, f); }
template <class F>
inline void ParallelFor(const Box& b, int ncomp, F&& f) {
  for (int n = 0; n < ncomp; ++n)
    for (int k = b.lo[2]; k <= b.hi[2]; ++k)
      for (int j = b.lo[1]; j <= b.hi[1]; ++j)
        for (int i = b.lo[0]; i <= b.hi[0]; ++i) f(i, j, k, n);
}

namespace Gpu {
inline void streamSynchronize() {}
inline bool notInLaunchRegion() { return true; }
}  // namespace Gpu

}  // namespace amrex
