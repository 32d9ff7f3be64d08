// clg_common.cuh -- shared device types for the B200 fermion hot path.
//
// Data layout in HBM (all fields even-odd split, structure of arrays):
//   site s = ((x*Ly + y)*Lz + z)*Lt + t (the reference's order, Data/CCommonData.h:274-277),
//   parity p = (x+y+z+t)&1, checkerboard index h = s >> 1 (Lt even), V_h = V/2.
//   Wilson spinor, per parity and right-hand side, "chunk-major" [chunk][h]:
//     FP64 : 12 x double2            (192 B / site)
//     FP32 :  6 x float4             ( 96 B / site)
//     FP16 :  3 x uint4 (4 half2)    ( 48 B / site) + float norm per site (4 B)
//   staggered vector: FP64 3 x double2, FP32 3 x float2 (24 B), FP16 3 x half2 + norm.
//   Gauge links, per parity p and direction mu, [chunk][h]:
//     FP64 : 9 x double2 (18 reals)
//     FP32 : 3 x float4 (12 reals: rows 0,1; row 2 = conj(row0 x row1))   or 9 x float2 (18 reals)
//     FP16 : uint4 + uint2 (12 reals as 6 half2)
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace clg {

enum Prec : int { P64 = 0, P32 = 1, P16 = 2 };

// Unsigned 32-bit division by a divisor fixed per lattice: one multiply-high,
// a subtraction and two shifts instead of a division sequence (T. Granlund and
// P. L. Montgomery, "Division by invariant integers using multiplication",
// PLDI 1994, Fig. 4.1).  Exact for every n < 2^32 and 1 <= d < 2^31.
struct FastDiv {
  unsigned m = 1, s1 = 0, s2 = 0;
  void set(unsigned d) {
    unsigned l = 0;
    while ((1ull << l) < d) ++l;
    m = (unsigned)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
    s1 = l < 1 ? l : 1;
    s2 = l > 0 ? l - 1 : 0;
  }
  __device__ __forceinline__ unsigned div(unsigned n) const {
    const unsigned t = __umulhi(m, n);
    return (t + ((n - t) >> s1)) >> s2;
  }
};

struct Geom {
  int L[4];      // Lx Ly Lz Lt
  int bc[4];     // fermion boundary signs
  int64_t V;     // volume
  int64_t Vh;    // V/2
  FastDiv dL[4]; // division by L[mu]
};

// ---------------------------------------------------------------- complex helpers
template <typename T> struct cpx;
template <> struct cpx<double> { double x, y; };
template <> struct cpx<float> { float x, y; };

template <typename T> __host__ __device__ __forceinline__ cpx<T> mk(T a, T b) { cpx<T> r; r.x = a; r.y = b; return r; }
template <typename T> __device__ __forceinline__ cpx<T> operator+(cpx<T> a, cpx<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ cpx<T> operator-(cpx<T> a, cpx<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T> __device__ __forceinline__ cpx<T> operator*(cpx<T> a, cpx<T> b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T> __device__ __forceinline__ cpx<T> operator*(T s, cpx<T> a) { return mk<T>(s * a.x, s * a.y); }
template <typename T> __device__ __forceinline__ cpx<T> cj(cpx<T> a) { return mk<T>(a.x, -a.y); }
// acc + s * a, one fused multiply-add per real component
template <typename T> __device__ __forceinline__ cpx<T> cfma(T s, cpx<T> a, cpx<T> acc) {
  if constexpr (sizeof(T) == 4)
    return mk<T>(fmaf(s, a.x, acc.x), fmaf(s, a.y, acc.y));
  else
    return mk<T>(fma(s, a.x, acc.x), fma(s, a.y, acc.y));
}
// conj(a) * b
template <typename T> __device__ __forceinline__ cpx<T> cjmul(cpx<T> a, cpx<T> b) {
  return mk<T>(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
// multiply by i^b (b known at compile time after unrolling)
template <typename T> __device__ __forceinline__ cpx<T> mul_i(cpx<T> a, int b) {
  switch (b & 3) {
    case 0: return a;
    case 1: return mk<T>(-a.y, a.x);
    case 2: return mk<T>(-a.x, -a.y);
    default: return mk<T>(a.y, -a.x);
  }
}

// ---------------------------------------------------------------- geometry
// Coordinates of the checkerboard site (parity p, index h).
// 32-bit index arithmetic: lattices are limited to V < 2^31 sites (checked when
// the lattice is created), and 64-bit integer division is emulated on the GPU.
__device__ __forceinline__ void eo_coords(const Geom& g, int p, int64_t h, int c[4]) {
  const unsigned s0 = 2u * (unsigned)h;
  const unsigned Lt = (unsigned)g.L[3], Lz = (unsigned)g.L[2], Ly = (unsigned)g.L[1];
  unsigned r = g.dL[3].div(s0);
  const int t0 = (int)(s0 - r * Lt);
  unsigned q = g.dL[2].div(r);
  c[2] = (int)(r - q * Lz);
  r = g.dL[1].div(q);
  c[1] = (int)(q - r * Ly);
  c[0] = (int)r;
  c[3] = t0 + ((c[0] + c[1] + c[2] + p) & 1);
}
__device__ __forceinline__ int64_t site_index(const Geom& g, const int c[4]) {
  return (int64_t)((((unsigned)c[0] * (unsigned)g.L[1] + (unsigned)c[1]) * (unsigned)g.L[2] + (unsigned)c[2]) *
                       (unsigned)g.L[3] + (unsigned)c[3]);
}

// ---------------------------------------------------------------- programmatic dependent launch
// A kernel launched with programmatic stream serialization may start while
// the previous kernel in the stream is still draining.  The hot kernels
// (hops, site functors) therefore
//   1. let their own dependents launch as soon as every one of their blocks
//      has started (pdl_launch_dependents at block start), and
//   2. call pdl_wait() -- a hardware wait for the previous grid's completion
//      and memory flush -- before reading or writing anything that kernel
//      may touch; only index arithmetic and reads of constant data (links,
//      geometry) come before it.
// Both are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;\n" ::); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

// ---------------------------------------------------------------- errors
#define CLG_CUDA_OK(expr)                                   \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) return clg::cuda_status(_e);     \
  } while (0)

}  // namespace clg
