// field_io.cuh -- per-site loads and stores of spinors / colour vectors and
// SU(3) links in the structure-of-arrays layouts described in clg_common.cuh.
//
// A site vector holds NC complex numbers (12 for Wilson, 3 for staggered).
// Every chunk [k][h] is a naturally aligned vector type, so a warp reading
// consecutive h issues fully coalesced 8/16-byte loads.
#pragma once
#include "clg_common.cuh"

namespace clg {

template <int P> struct AccT { using T = float; };
template <> struct AccT<P64> { using T = double; };

// bytes per complex number stored
template <int P> constexpr int cbytes() { return P == P64 ? 16 : (P == P32 ? 8 : 4); }
// bytes per site of the data array (excluding the FP16 norm)
template <int P, int NC> constexpr int site_bytes() { return NC * cbytes<P>(); }

__device__ __forceinline__ float2 h2f(uint32_t u) {
  __half2 h = *reinterpret_cast<__half2*>(&u);
  return __half22float2(h);
}
__device__ __forceinline__ uint32_t f2h(float a, float b) {
  __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

// ------------------------------------------------------------------ site vectors
template <int P, int NC, typename AT>
__device__ __forceinline__ void load_site(const void* __restrict__ base, const float* __restrict__ nrm,
                                          int64_t Vh, int64_t h, cpx<AT> v[NC]) {
  if constexpr (P == P64) {
    const double2* b = reinterpret_cast<const double2*>(base);
#pragma unroll
    for (int k = 0; k < NC; ++k) {
      const double2 d = __ldg(b + k * Vh + h);
      v[k] = mk<AT>((AT)d.x, (AT)d.y);
    }
  } else if constexpr (P == P32) {
    if constexpr (NC % 2 == 0) {
      const float4* b = reinterpret_cast<const float4*>(base);
#pragma unroll
      for (int k = 0; k < NC / 2; ++k) {
        const float4 d = __ldg(b + k * Vh + h);
        v[2 * k] = mk<AT>((AT)d.x, (AT)d.y);
        v[2 * k + 1] = mk<AT>((AT)d.z, (AT)d.w);
      }
    } else {
      const float2* b = reinterpret_cast<const float2*>(base);
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        const float2 d = __ldg(b + k * Vh + h);
        v[k] = mk<AT>((AT)d.x, (AT)d.y);
      }
    }
  } else {
    const float n = __ldg(nrm + h);
    if constexpr (NC == 12) {
      // spin-planar words (spinor_word): word 6q + 2c + ri holds part ri of
      // colour c of spins 2q (low half) and 2q + 1 (high half)
      const uint4* b = reinterpret_cast<const uint4*>(base);
      uint32_t w[12];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const uint4 d = __ldg(b + k * Vh + h);
        w[4 * k] = d.x; w[4 * k + 1] = d.y; w[4 * k + 2] = d.z; w[4 * k + 3] = d.w;
      }
#pragma unroll
      for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float2 re = h2f(w[6 * q + 2 * c]), im = h2f(w[6 * q + 2 * c + 1]);
          v[(2 * q) * 3 + c] = mk<AT>(n * re.x, n * im.x);
          v[(2 * q + 1) * 3 + c] = mk<AT>(n * re.y, n * im.y);
        }
    } else if constexpr (NC % 4 == 0) {
      const uint4* b = reinterpret_cast<const uint4*>(base);
#pragma unroll
      for (int k = 0; k < NC / 4; ++k) {
        const uint4 d = __ldg(b + k * Vh + h);
        float2 f;
        f = h2f(d.x); v[4 * k + 0] = mk<AT>(n * f.x, n * f.y);
        f = h2f(d.y); v[4 * k + 1] = mk<AT>(n * f.x, n * f.y);
        f = h2f(d.z); v[4 * k + 2] = mk<AT>(n * f.x, n * f.y);
        f = h2f(d.w); v[4 * k + 3] = mk<AT>(n * f.x, n * f.y);
      }
    } else {
      const uint32_t* b = reinterpret_cast<const uint32_t*>(base);
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        const float2 f = h2f(__ldg(b + k * Vh + h));
        v[k] = mk<AT>(n * f.x, n * f.y);
      }
    }
  }
}

template <int P, int NC, typename AT>
__device__ __forceinline__ void store_site(void* __restrict__ base, float* __restrict__ nrm, int64_t Vh, int64_t h,
                                           const cpx<AT> v[NC]) {
  if constexpr (P == P64) {
    double2* b = reinterpret_cast<double2*>(base);
#pragma unroll
    for (int k = 0; k < NC; ++k) b[k * Vh + h] = make_double2((double)v[k].x, (double)v[k].y);
  } else if constexpr (P == P32) {
    if constexpr (NC % 2 == 0) {
      float4* b = reinterpret_cast<float4*>(base);
#pragma unroll
      for (int k = 0; k < NC / 2; ++k)
        b[k * Vh + h] = make_float4((float)v[2 * k].x, (float)v[2 * k].y, (float)v[2 * k + 1].x, (float)v[2 * k + 1].y);
    } else {
      float2* b = reinterpret_cast<float2*>(base);
#pragma unroll
      for (int k = 0; k < NC; ++k) b[k * Vh + h] = make_float2((float)v[k].x, (float)v[k].y);
    }
  } else {
    float m = 0.f;
#pragma unroll
    for (int k = 0; k < NC; ++k) m = fmaxf(m, fmaxf(fabsf((float)v[k].x), fabsf((float)v[k].y)));
    // a site whose largest component is below 1e-30 is stored as exact zero:
    // 1/m of a float denormal overflows to inf and would turn the site into NaN
    // (point sources produce such sites after a few hops)
    if (!(m > 1e-30f)) m = 0.f;
    const float inv = m > 0.f ? __frcp_rn(m) : 0.f;  // the correctly rounded 1/m
    nrm[h] = m;
    if constexpr (NC == 12) {
      uint32_t w[12];
#pragma unroll
      for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const cpx<AT> lo = v[(2 * q) * 3 + c], hi = v[(2 * q + 1) * 3 + c];
          w[6 * q + 2 * c] = f2h((float)lo.x * inv, (float)hi.x * inv);
          w[6 * q + 2 * c + 1] = f2h((float)lo.y * inv, (float)hi.y * inv);
        }
      uint4* b = reinterpret_cast<uint4*>(base);
#pragma unroll
      for (int k = 0; k < 3; ++k) b[k * Vh + h] = make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
    } else if constexpr (NC % 4 == 0) {
      uint4* b = reinterpret_cast<uint4*>(base);
#pragma unroll
      for (int k = 0; k < NC / 4; ++k) {
        uint4 d;
        d.x = f2h((float)v[4 * k + 0].x * inv, (float)v[4 * k + 0].y * inv);
        d.y = f2h((float)v[4 * k + 1].x * inv, (float)v[4 * k + 1].y * inv);
        d.z = f2h((float)v[4 * k + 2].x * inv, (float)v[4 * k + 2].y * inv);
        d.w = f2h((float)v[4 * k + 3].x * inv, (float)v[4 * k + 3].y * inv);
        b[k * Vh + h] = d;
      }
    } else {
      uint32_t* b = reinterpret_cast<uint32_t*>(base);
#pragma unroll
      for (int k = 0; k < NC; ++k) b[k * Vh + h] = f2h((float)v[k].x * inv, (float)v[k].y * inv);
    }
  }
}

// ------------------------------------------------------------------ SU(3) links
// Link arrays per parity: [mu][chunk][h].  RECON = 18 (full) or 12 (rows 0,1).
template <int P, int RECON> constexpr int link_chunks() {
  return P == P64 ? (RECON == 18 ? 9 : 6) : (P == P32 ? (RECON == 18 ? 9 : 3) : 2);
}
template <int P, int RECON> constexpr int link_bytes() {
  return P == P64 ? RECON * 8 : (P == P32 ? RECON * 4 : RECON * 2);
}

template <typename AT>
__device__ __forceinline__ void reconstruct_row2(cpx<AT> u[9]) {
  // row2 = conj(row0 x row1), exact for det U = 1
  u[6] = cj(u[1] * u[5] - u[2] * u[4]);
  u[7] = cj(u[2] * u[3] - u[0] * u[5]);
  u[8] = cj(u[0] * u[4] - u[1] * u[3]);
}

template <int P, int RECON, typename AT>
__device__ __forceinline__ void load_link(const void* __restrict__ base, int mu, int64_t Vh, int64_t h, cpx<AT> u[9]) {
  constexpr int NCH = link_chunks<P, RECON>();
  const int64_t off = (int64_t)mu * NCH * Vh + h;
  if constexpr (P == P64) {
    const double2* b = reinterpret_cast<const double2*>(base) + off;
    constexpr int N = RECON == 18 ? 9 : 6;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const double2 d = __ldg(b + k * Vh);
      u[k] = mk<AT>((AT)d.x, (AT)d.y);
    }
    if constexpr (RECON == 12) reconstruct_row2(u);
  } else if constexpr (P == P32) {
    if constexpr (RECON == 18) {
      const float2* b = reinterpret_cast<const float2*>(base) + off;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const float2 d = __ldg(b + k * Vh);
        u[k] = mk<AT>((AT)d.x, (AT)d.y);
      }
    } else {
      const float4* b = reinterpret_cast<const float4*>(base) + off;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float4 d = __ldg(b + k * Vh);
        u[2 * k] = mk<AT>((AT)d.x, (AT)d.y);
        u[2 * k + 1] = mk<AT>((AT)d.z, (AT)d.w);
      }
      reconstruct_row2(u);
    }
  } else {
    // FP16, 12 reals: chunk 0 = uint4 (u0..u3), chunk 1 = uint2 (u4,u5); the two
    // chunks live in separate arrays: [mu][h] uint4 followed by [mu][h] uint2.
    const uint4* b4 = reinterpret_cast<const uint4*>(base);
    const uint2* b2 = reinterpret_cast<const uint2*>(b4 + 4 * Vh);
    const uint4 d = __ldg(b4 + (int64_t)mu * Vh + h);
    const uint2 e = __ldg(b2 + (int64_t)mu * Vh + h);
    float2 f;
    f = h2f(d.x); u[0] = mk<AT>(f.x, f.y);
    f = h2f(d.y); u[1] = mk<AT>(f.x, f.y);
    f = h2f(d.z); u[2] = mk<AT>(f.x, f.y);
    f = h2f(d.w); u[3] = mk<AT>(f.x, f.y);
    f = h2f(e.x); u[4] = mk<AT>(f.x, f.y);
    f = h2f(e.y); u[5] = mk<AT>(f.x, f.y);
    reconstruct_row2(u);
  }
}

// ------------------------------------------------------------------ packed FP16 (load now, unpack later)
// An FP16 Wilson spinor is 12 half2 words (3 uint4 chunks) in spin-planar
// order: word 6q + 2c + ri holds part ri (0 real, 1 imaginary) of colour c of
// spin 2q in its low half and of spin 2q + 1 in its high half.  The hop's spin
// projection pairs spins (0, 1) with (2, 3) or (3, 2), so it takes its half2
// planes from these words as they are (at most a swap of halves).
__host__ __device__ constexpr int spinor_word(int q, int c, int ri) { return 6 * q + 2 * c + ri; }
struct Packed16 {
  uint4 c[3];
  float n;
};
struct PackedLink16 {
  uint4 a;
  uint2 b;
};
__device__ __forceinline__ void load_packed16(const void* __restrict__ base, const float* __restrict__ nrm, int64_t Vh,
                                              int64_t h, Packed16& p) {
  const uint4* b = reinterpret_cast<const uint4*>(base);
  p.c[0] = __ldg(b + h);
  p.c[1] = __ldg(b + Vh + h);
  p.c[2] = __ldg(b + 2 * Vh + h);
  p.n = __ldg(nrm + h);
}
__device__ __forceinline__ void load_packed_link16(const void* __restrict__ base, int mu, int64_t Vh, int64_t h,
                                                   PackedLink16& l) {
  const uint4* b4 = reinterpret_cast<const uint4*>(base);
  const uint2* b2 = reinterpret_cast<const uint2*>(b4 + 4 * Vh);
  l.a = __ldg(b4 + (int64_t)mu * Vh + h);
  l.b = __ldg(b2 + (int64_t)mu * Vh + h);
}

// bytes of one parity's link array
template <int P, int RECON> constexpr int64_t link_parity_bytes(int64_t Vh) { return 4 * Vh * (int64_t)link_bytes<P, RECON>(); }

}  // namespace clg
