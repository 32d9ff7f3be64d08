// dslash.cuh -- Wilson and staggered hopping stencils on one checkerboard.
//
// Wilson (restating _kernelDFermionWilsonSquareSU3,
// Data/Field/WilsonDirac/CFieldFermionWilsonSquareSU3.cu:32-163, as a hop):
//   H psi(x)   = sum_mu [ s+ (1 - g_mu) U_mu(x) psi(x+mu) + s- (1 + g_mu) U_mu(x-mu)^+ psi(x-mu) ]
//   H^+ psi(x) = the same with (1 -/+ g_mu) swapped   (D^+ = g5 D g5, :53-56, :149-152)
// evaluated with spin projection: (1 -/+ g_mu) has rank two in the chiral basis of
// Tools/Math/GammaMatrix.h:447-478, so two colour vectors are multiplied by the
// link instead of four and the lower spin components are rebuilt by a phase.
// D = 1 - kappa H on the full lattice is two checkerboard launches with
// out_p = in_p - kappa H in_(1-p);  M_ee = 1 - kappa^2 H_eo H_oe (Docs/SparseLinearAlgebra/evenodd.tex:11-16).
//
// Staggered (restating _kernelDFermionKS, Data/Field/Staggered/CFieldFermionKSSU3.cu:33-117):
//   H chi(x) = sum_mu eta_mu(x) [ s+ U_mu(x) chi(x+mu) - s- U_mu(x-mu)^+ chi(x-mu) ],
//   D = 2am + H, D^+ = 2am - H, eta_mu(x) = (-1)^(x_0+..+x_(mu-1)) (Data/CCommonData.h:228-236).
//
// The epilogue computes out = xa * x + a * (H in), optionally times a real
// device-resident scalar (used for lazily normalised Krylov vectors).
#pragma once
#include "field_io.cuh"
#include "reduce.cuh"

namespace clg {

// One right-hand side of a batch of lattices: its lattice's geometry and link
// arrays ([precision][parity]; FP64 18-real, FP32 and FP16 12-real).
struct HopSeg {
  Geom g;
  const void* u[3][2];
};

struct HopArgs {
  Geom g;
  int out_parity;
  const void* in;      // input spinors at parity 1-out_parity (rhs 0)
  const float* in_norm;
  void* out;           // output at out_parity
  float* out_norm;
  const void* x;       // xpay source at out_parity (nullable)
  const float* x_norm;
  const void* U_here;  // links of parity out_parity
  const void* U_there; // links of parity 1-out_parity
  int64_t in_stride;   // bytes between right-hand sides
  int64_t out_stride;
  int64_t x_stride;
  int64_t in_nstride;  // floats between right-hand sides of the FP16 norms
  int64_t out_nstride;
  int64_t x_nstride;
  double2 a;           // multiplies H in
  double2 xa;          // multiplies x
  const double* scale_dev;  // optional: whole result times scale_dev[rhs * scale_stride]
  int scale_stride;
  const int* skip_dev;      // optional: rhs with skip_dev[rhs * skip_stride] != 0 are not computed
  int skip_stride;
  int nrhs;                 // right-hand sides (interleaved in blockIdx.x)
  // a batch of lattices (nullable): right-hand side r lives on lattice seg[r]
  // (geometry and links, checkerboard size seg_vh[r]); g.Vh is then the
  // fields' chunk stride, the largest checkerboard of the batch, and sites
  // h >= seg_vh[r] are padding
  const HopSeg* seg;
  const int64_t* seg_vh;
  // the tile hops' block order (wilson_hop_tile16_kernel): 0 = tiles in site
  // order, else the rows y are walked in chunks of tile_rows (tile16_index)
  int tile_rows;
  // a batch of lattices, tile form: lattice l's tiles are the blocks
  // [btile[l].tile0, btile[l + 1].tile0), its right-hand sides
  // [rhs0, rhs0 + nrhs), its geometry and links those of seg[btile[l].seg]
  const struct BatchTile* btile;
  int nbtile;
  int64_t btiles;  // blocks of the batch (all lattices' tiles)
};
struct BatchTile {
  int64_t tile0;
  int rhs0, nrhs, seg;
};
// the lattice of batch block b (a handful of lattices: a linear scan)
__device__ __forceinline__ BatchTile batch_tile(const HopArgs& a) {
  int l = 0;
  while (l + 1 < a.nbtile && a.btile[l + 1].tile0 <= (int64_t)blockIdx.x) ++l;
  return a.btile[l];
}

// chiral gamma tables (GammaMatrix.h:447-478): row r -> column perm[r] with phase i^z4[r]
__device__ __forceinline__ constexpr int gperm(int mu, int r) {
  return (mu < 2) ? (3 - r) : ((r + 2) & 3);
}
__device__ __forceinline__ constexpr int gz4(int mu, int r) {
  // mu=0: {3,3,1,1}; mu=1: {2,0,0,2}; mu=2: {3,1,1,3}; mu=3: {0,0,0,0}
  return mu == 0 ? (r < 2 ? 3 : 1) : mu == 1 ? ((r == 0 || r == 3) ? 2 : 0) : mu == 2 ? ((r == 0 || r == 3) ? 3 : 1) : 0;
}

template <typename AT, bool DAG>
__device__ __forceinline__ void su3_mv(const cpx<AT> u[9], const cpx<AT> v[3], cpx<AT> o[3]) {
  if constexpr (!DAG) {
#pragma unroll
    for (int r = 0; r < 3; ++r) o[r] = u[3 * r] * v[0] + u[3 * r + 1] * v[1] + u[3 * r + 2] * v[2];
  } else {
#pragma unroll
    for (int r = 0; r < 3; ++r) o[r] = cjmul(u[r], v[0]) + cjmul(u[3 + r], v[1]) + cjmul(u[6 + r], v[2]);
  }
}

// acc += s * P^{SGN}_mu (Udag? U^+ : U) psi   with P^{SGN} = (1 + SGN g_mu)
template <typename AT, int MU, int SGN, bool UDAG>
__device__ __forceinline__ void wilson_hop_dir(cpx<AT> acc[12], const cpx<AT> psi[12], const cpx<AT> u[9], AT s) {
  constexpr int add = SGN < 0 ? 2 : 0;
  cpx<AT> h0[3], h1[3], g0[3], g1[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    h0[c] = psi[c] + mul_i(psi[3 * gperm(MU, 0) + c], gz4(MU, 0) + add);
    h1[c] = psi[3 + c] + mul_i(psi[3 * gperm(MU, 1) + c], gz4(MU, 1) + add);
  }
  su3_mv<AT, UDAG>(u, h0, g0);
  su3_mv<AT, UDAG>(u, h1, g1);
  // each accumulator row takes s * (phase * g) as one fused multiply-add per
  // real component: the phase is a swap / negation (operand modifiers), and s
  // is never applied to g separately
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    acc[c] = cfma(s, g0[c], acc[c]);
    acc[3 + c] = cfma(s, g1[c], acc[3 + c]);
    // rows 2,3: coefficient SGN*i^z4[r] times the projected row perm[r] (in {0,1})
    acc[6 + c] = cfma(s, mul_i(gperm(MU, 2) == 0 ? g0[c] : g1[c], gz4(MU, 2) + add), acc[6 + c]);
    acc[9 + c] = cfma(s, mul_i(gperm(MU, 3) == 0 ? g0[c] : g1[c], gz4(MU, 3) + add), acc[9 + c]);
  }
}

// ---------------------------------------------------------------- FP16 arithmetic in half2 words
// A word holds one complex number, real part in the low half.  Multiplying by
// a phase i^Z is a swap of the halves and/or a sign-bit flip.
__device__ __forceinline__ uint32_t h2_swap(uint32_t a) { return __byte_perm(a, 0, 0x1032); }
template <int Z>
__device__ __forceinline__ uint32_t h2_mul_i(uint32_t a) {
  if constexpr ((Z & 3) == 0) return a;
  if constexpr ((Z & 3) == 1) return h2_swap(a) ^ 0x00008000u;  // (-im, re)
  if constexpr ((Z & 3) == 2) return a ^ 0x80008000u;           // (-re, -im)
  return h2_swap(a) ^ 0x80000000u;                               // (im, -re)
}
__device__ __forceinline__ __half2 as_h2(uint32_t a) { return *reinterpret_cast<__half2*>(&a); }
__device__ __forceinline__ uint32_t as_u32(__half2 a) { return *reinterpret_cast<uint32_t*>(&a); }
// o + u * v   (UDAG: o + conj(u) * v), u given as its broadcast real / imaginary parts
template <bool UDAG>
__device__ __forceinline__ __half2 h2_cmac(__half2 ur, __half2 ui, uint32_t v, __half2 o) {
  o = __hfma2(ur, as_h2(v), o);
  return __hfma2(ui, as_h2(UDAG ? h2_mul_i<3>(v) : h2_mul_i<1>(v)), o);
}

// The third row of an FP16 12-real link, row2 = conj(row0 x row1), on half2
// words: u[0..5] are rows 0 and 1 (one complex number per word), u[6..8] are
// written.
__device__ __forceinline__ void link16_third_row(uint32_t u[9]) {
  // u6 = conj(u1 u5 - u2 u4), u7 = conj(u2 u3 - u0 u5), u8 = conj(u0 u4 - u1 u3)
  const __half2 zero = __float2half2_rn(0.f);
  auto cross = [&](int a, int b, int c, int d) -> uint32_t {
    __half2 t = h2_cmac<false>(__low2half2(as_h2(u[a])), __high2half2(as_h2(u[a])), u[b], zero);
    const uint32_t nd = u[d] ^ 0x80008000u;  // -u[d]
    t = h2_cmac<false>(__low2half2(as_h2(u[c])), __high2half2(as_h2(u[c])), nd, t);
    return as_u32(t) ^ 0x80000000u;  // conjugate
  };
  // u6 and u7 together, "planar" across the two: lane 0 carries u1 u5 - u2 u4,
  // lane 1 u2 u3 - u0 u5, so the products need no broadcasts or swaps
  const __half2 X = as_h2(__byte_perm(u[1], u[2], 0x5410)), Xi = as_h2(__byte_perm(u[1], u[2], 0x7632));
  const __half2 Y = as_h2(__byte_perm(u[5], u[3], 0x5410)), Yi = as_h2(__byte_perm(u[5], u[3], 0x7632));
  const __half2 Z = as_h2(__byte_perm(u[2], u[0], 0x5410)), Zi = as_h2(__byte_perm(u[2], u[0], 0x7632));
  const __half2 W = as_h2(__byte_perm(u[4], u[5], 0x5410)), Wi = as_h2(__byte_perm(u[4], u[5], 0x7632));
  __half2 re = __hmul2(X, Y);
  re = __hfma2(__hneg2(Xi), Yi, re);
  re = __hfma2(__hneg2(Z), W, re);
  re = __hfma2(Zi, Wi, re);
  __half2 nim = __hmul2(Z, Wi);  // minus the imaginary parts: the conjugate directly
  nim = __hfma2(Zi, W, nim);
  nim = __hfma2(__hneg2(X), Yi, nim);
  nim = __hfma2(__hneg2(Xi), Y, nim);
  u[6] = __byte_perm(as_u32(re), as_u32(nim), 0x5410);
  u[7] = __byte_perm(as_u32(re), as_u32(nim), 0x7632);
  u[8] = cross(0, 4, 1, 3);
}

// FP16 hop accumulators, "planar" over pairs of spin rows: r[c] holds the real
// parts of rows (0, 1) of colour c, r[3 + c] those of rows (2, 3); i[] the
// imaginary parts.  acc16_out gives the usual interleaved acc[12].
struct Acc16 {
  float2 r[6], i[6];
};
__device__ __forceinline__ void acc16_zero(Acc16& A) {
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    A.r[k] = make_float2(0.f, 0.f);
    A.i[k] = make_float2(0.f, 0.f);
  }
}
__device__ __forceinline__ void acc16_out(const Acc16& A, cpx<float> acc[12]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    acc[c] = mk<float>(A.r[c].x, A.i[c].x);
    acc[3 + c] = mk<float>(A.r[c].y, A.i[c].y);
    acc[6 + c] = mk<float>(A.r[3 + c].x, A.i[3 + c].x);
    acc[9 + c] = mk<float>(A.r[3 + c].y, A.i[3 + c].y);
  }
}

// a + (P0 ? +b.lo : -b.lo, P1 ? +b.hi : -b.hi), one half2 instruction
template <bool P0, bool P1>
__device__ __forceinline__ __half2 h2_add_signed(__half2 a, __half2 b) {
  if constexpr (P0 && P1) return __hadd2(a, b);
  else if constexpr (!P0 && !P1) return __hsub2(a, b);
  else return __hfma2(__floats2half2_rn(P0 ? 1.f : -1.f, P1 ? 1.f : -1.f), b, a);
}
// acc + (S0 ? s : -s, S1 ? s : -s) * f, one packed f32x2 FMA
template <bool S0, bool S1>
__device__ __forceinline__ float2 f2_fma_signed(float s, float2 f, float2 acc) {
  return __ffma2_rn(make_float2(S0 ? s : -s, S1 ? s : -s), f, acc);
}

// The FP16 counterpart of wilson_hop_dir with the whole link given (u[9], one
// complex number per half2 word), planar over the two projected spin rows:
// the spin projection forms, per colour, one half2 of the real parts of both
// projected rows and one of the imaginary parts; every HFMA2 of the colour
// mat-vec then serves both rows with no swap or sign flip of its operands
// (the link element's real / imaginary part is the broadcast operand), and
// the phases of the rebuilt rows 2, 3 are per-lane signs of one packed f32x2
// FMA.  The accumulation is in FP32 with the factor s (boundary sign times
// the neighbour's site norm).  Every rounding step is the one of the
// interleaved formulation (projection a + i^z b, U h as (re, im) pairs,
// s * g + acc per real component), so results are bit-identical to it.
// Both projected rows' phases i^z have the same parity for every direction
// of the chiral basis (gz4), which is what lets one plane select serve both.
template <int MU, int SGN, bool UDAG>
__device__ __forceinline__ void wilson_hop_dir16_u(Acc16& A, const Packed16& p, const uint32_t (&u)[9], float s) {
  constexpr int add = SGN < 0 ? 2 : 0;
  constexpr int z0 = (gz4(MU, 0) + add) & 3, z1 = (gz4(MU, 1) + add) & 3;
  static_assert(((z0 ^ z1) & 1) == 0, "projected rows with phases of different parity");
  uint32_t w[12];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    w[4 * k + 0] = p.c[k].x;
    w[4 * k + 1] = p.c[k].y;
    w[4 * k + 2] = p.c[k].z;
    w[4 * k + 3] = p.c[k].w;
  }
  // projected rows j = 0, 1:  h_j[c] = psi_j[c] + i^z_j psi_perm(j)[c].  The
  // spin-planar storage (spinor_word) holds spins (0, 1) and (2, 3) as planes:
  // rows (0, 1) are the q = 0 words, rows perm = (2, 3) the q = 1 words and
  // perm = (3, 2) the same with their halves swapped.
  static_assert(gperm(MU, 0) + gperm(MU, 1) == 5 && gperm(MU, 0) >= 2, "perm pairs spins 2 and 3");
  __half2 hR[3], hI[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const __half2 Ar = as_h2(w[spinor_word(0, c, 0)]), Ai = as_h2(w[spinor_word(0, c, 1)]);
    uint32_t br = w[spinor_word(1, c, 0)], bi = w[spinor_word(1, c, 1)];
    if constexpr (gperm(MU, 0) == 3) {
      br = h2_swap(br);
      bi = h2_swap(bi);
    }
    const __half2 Br = as_h2(br), Bi = as_h2(bi);
    if constexpr ((z0 & 1) == 0) {  // i^z = +-1
      hR[c] = h2_add_signed<z0 == 0, z1 == 0>(Ar, Br);
      hI[c] = h2_add_signed<z0 == 0, z1 == 0>(Ai, Bi);
    } else {  // i^z b = (-b.im, b.re) for z = 1, (b.im, -b.re) for z = 3
      hR[c] = h2_add_signed<z0 == 3, z1 == 3>(Ar, Bi);
      hI[c] = h2_add_signed<z0 == 1, z1 == 1>(Ai, Br);
    }
  }
  // g_j = U h_j (UDAG: U^+ h_j), both rows per instruction
  const __half2 zero = __float2half2_rn(0.f);
  __half2 gR[3] = {zero, zero, zero}, gI[3] = {zero, zero, zero};
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      // U: row r, column k;  U^+: conj of row k, column r
      const uint32_t e = UDAG ? u[3 * k + r] : u[3 * r + k];
      const __half2 er = __low2half2(as_h2(e)), ei = __high2half2(as_h2(e));
      gR[r] = __hfma2(er, hR[k], gR[r]);
      gI[r] = __hfma2(er, hI[k], gI[r]);
      if constexpr (UDAG) {  // conj(e) h: re += ei h.im, im -= ei h.re
        gR[r] = __hfma2(ei, hI[k], gR[r]);
        gI[r] = __hfma2(__hneg2(ei), hR[k], gI[r]);
      } else {               // e h: re -= ei h.im, im += ei h.re
        gR[r] = __hfma2(__hneg2(ei), hI[k], gR[r]);
        gI[r] = __hfma2(ei, hR[k], gI[r]);
      }
    }
  // FP32 accumulation.  Rows 0, 1 take s g_0, s g_1; rows 2, 3 take
  // s i^z_r g_perm(r), perm = (1, 0) for mu < 2 (the lanes swapped) and (0, 1)
  // for mu >= 2, with z_2, z_3 of equal parity as well.
  constexpr int z2 = (gz4(MU, 2) + add) & 3, z3 = (gz4(MU, 3) + add) & 3;
  static_assert(((z2 ^ z3) & 1) == 0, "rebuilt rows with phases of different parity");
  constexpr bool swp = gperm(MU, 2) == 1;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float2 fr = __half22float2(gR[c]), fi = __half22float2(gI[c]);
    A.r[c] = f2_fma_signed<true, true>(s, fr, A.r[c]);
    A.i[c] = f2_fma_signed<true, true>(s, fi, A.i[c]);
    const float2 gr = swp ? make_float2(fr.y, fr.x) : fr;
    const float2 gi = swp ? make_float2(fi.y, fi.x) : fi;
    if constexpr ((z2 & 1) == 0) {
      A.r[3 + c] = f2_fma_signed<z2 == 0, z3 == 0>(s, gr, A.r[3 + c]);
      A.i[3 + c] = f2_fma_signed<z2 == 0, z3 == 0>(s, gi, A.i[3 + c]);
    } else {
      A.r[3 + c] = f2_fma_signed<z2 == 3, z3 == 3>(s, gi, A.r[3 + c]);
      A.i[3 + c] = f2_fma_signed<z2 == 1, z3 == 1>(s, gr, A.i[3 + c]);
    }
  }
}

// The same with the link as stored (12-real): the third row is rebuilt first.
template <int MU, int SGN, bool UDAG>
__device__ __forceinline__ void wilson_hop_dir16(Acc16& A, const Packed16& p, const PackedLink16& l, float s) {
  uint32_t u[9] = {l.a.x, l.a.y, l.a.z, l.a.w, l.b.x, l.b.y, 0u, 0u, 0u};
  link16_third_row(u);
  wilson_hop_dir16_u<MU, SGN, UDAG>(A, p, u, s);
}

struct NbrInfo {
  int hf[4], hb[4];   // checkerboard index of x+mu, x-mu (V < 2^31)
  float sf[4], sb[4]; // boundary signs
};

__device__ __forceinline__ void neighbours(const Geom& g, int p, int64_t h, NbrInfo& nb, int c[4]) {
  eo_coords(g, p, h, c);
  const int s = (int)site_index(g, c);
  int st[4];
  st[3] = 1;
  st[2] = g.L[3];
  st[1] = g.L[2] * g.L[3];
  st[0] = g.L[1] * st[1];
#pragma unroll
  for (int mu = 0; mu < 4; ++mu) {
    int sf = s + st[mu], sb = s - st[mu];
    float bf = 1.f, bb = 1.f;
    if (c[mu] == g.L[mu] - 1) { sf -= g.L[mu] * st[mu]; bf = (float)g.bc[mu]; }
    if (c[mu] == 0) { sb += g.L[mu] * st[mu]; bb = (float)g.bc[mu]; }
    nb.hf[mu] = sf >> 1;
    nb.hb[mu] = sb >> 1;
    nb.sf[mu] = bf;
    nb.sb[mu] = bb;
  }
}

// acc <- [scale_dev[rhs] *] (a * acc + xa * x) at (rhs, h)
template <int P, typename AT>
__device__ __forceinline__ void wilson_hop_finish(const HopArgs& a, int rhs, int64_t h, cpx<AT> acc[12]) {
  const int64_t Vh = a.g.Vh;
  // the coefficients of the operators are real (-kappa, -kappa^2, 1): a real
  // fast path (uniform branch) takes half the multiplies, packed f32x2 in FP32
  if (a.a.y == 0.0 && a.a.x == 1.0) {
    // the plain hop (a = 1): nothing to scale (x * 1 is exact, so skipping it changes no bit)
  } else if (a.a.y == 0.0) {
    const AT ar = (AT)a.a.x;
    if constexpr (sizeof(AT) == 4) {
      float2* av = reinterpret_cast<float2*>(acc);
      const float2 s2 = make_float2(ar, ar);
#pragma unroll
      for (int k = 0; k < 12; ++k) av[k] = __fmul2_rn(s2, av[k]);
    } else {
#pragma unroll
      for (int k = 0; k < 12; ++k) acc[k] = ar * acc[k];
    }
  } else {
    const cpx<AT> ca = mk<AT>((AT)a.a.x, (AT)a.a.y);
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = ca * acc[k];
  }
  if (a.x) {
    cpx<AT> xv[12];
    const char* xp = reinterpret_cast<const char*>(a.x) + rhs * a.x_stride;
    load_site<P, 12, AT>(xp, a.x_norm ? a.x_norm + rhs * a.x_nstride : nullptr, Vh, h, xv);
    if (a.xa.y == 0.0) {
      const AT xr = (AT)a.xa.x;
      if constexpr (sizeof(AT) == 4) {
        float2* av = reinterpret_cast<float2*>(acc);
        const float2* xw = reinterpret_cast<const float2*>(xv);
        const float2 s2 = make_float2(xr, xr);
#pragma unroll
        for (int k = 0; k < 12; ++k) av[k] = __ffma2_rn(s2, xw[k], av[k]);
      } else {
#pragma unroll
        for (int k = 0; k < 12; ++k) acc[k] = cfma(xr, xv[k], acc[k]);
      }
    } else {
      const cpx<AT> cx = mk<AT>((AT)a.xa.x, (AT)a.xa.y);
#pragma unroll
      for (int k = 0; k < 12; ++k) acc[k] = acc[k] + cx * xv[k];
    }
  }
  if (a.scale_dev) {
    const AT sc = (AT)a.scale_dev[rhs * a.scale_stride];
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = sc * acc[k];
  }
}

template <int P, typename AT>
__device__ __forceinline__ void wilson_hop_store(const HopArgs& a, int rhs, int64_t h, const cpx<AT> acc[12]) {
  store_site<P, 12, AT>(reinterpret_cast<char*>(a.out) + rhs * a.out_stride,
                        a.out_norm ? a.out_norm + rhs * a.out_nstride : nullptr, a.g.Vh, h, acc);
}

// The whole stencil for output site (rhs, h): acc = [scale *] (a H in + xa x),
// on the lattice g with links U_here (parity out_parity) and U_there.  The
// spinors' chunk stride is a.g.Vh (equal to g.Vh except in a batch of lattices).
template <int P, int RECON, bool DAGGER, bool SEG, typename AT>
__device__ __forceinline__ void wilson_hop_site_on(const HopArgs& a, const Geom& g, const void* U_here,
                                                   const void* U_there, int rhs, int64_t h, cpx<AT> acc[12]) {
  const int64_t Vh = a.g.Vh;
  const int64_t lVh = SEG ? g.Vh : Vh;  // the links' stride: the lattice's own checkerboard
  const void* const Uh = SEG ? U_here : a.U_here;
  const void* const Ut = SEG ? U_there : a.U_there;
  const char* in = reinterpret_cast<const char*>(a.in) + rhs * a.in_stride;
  const float* in_norm = a.in_norm ? a.in_norm + rhs * a.in_nstride : nullptr;

  NbrInfo nb;
  int c[4];
  if constexpr (SEG)
    neighbours(g, a.out_parity, h, nb, c);
  else
    neighbours(a.g, a.out_parity, h, nb, c);

#pragma unroll
  for (int k = 0; k < 12; ++k) acc[k] = mk<AT>(0, 0);

  // D: forward (1 - g), backward (1 + g); D^+: swapped
  constexpr int SF = DAGGER ? 1 : -1;
  constexpr int SB = -SF;
  if constexpr (P == P16) {
    // FP16: both neighbours' packed data (19 registers each) are loaded before
    // either is used, so twice the bytes are in flight per thread.  The spin
    // projection, the third link row and the link products run on half2 words
    // (wilson_hop_dir16); the projection and the link product are linear, so
    // the neighbour's site norm is applied with the boundary sign to the 6
    // projected products when they are accumulated in FP32.
    Acc16 A;
    acc16_zero(A);
#define CLG_WILSON_DIR16(MU)                                                            \
  {                                                                                     \
    Packed16 pf, pb;                                                                    \
    PackedLink16 lf, lb;                                                                \
    load_packed16(in, in_norm, Vh, nb.hf[MU], pf);                                      \
    load_packed_link16(Uh, MU, lVh, h, lf);                                             \
    load_packed16(in, in_norm, Vh, nb.hb[MU], pb);                                      \
    load_packed_link16(Ut, MU, lVh, nb.hb[MU], lb);                                     \
    wilson_hop_dir16<MU, SF, false>(A, pf, lf, nb.sf[MU] * pf.n);                       \
    wilson_hop_dir16<MU, SB, true>(A, pb, lb, nb.sb[MU] * pb.n);                        \
  }
    CLG_WILSON_DIR16(0)
    CLG_WILSON_DIR16(1)
    CLG_WILSON_DIR16(2)
    CLG_WILSON_DIR16(3)
#undef CLG_WILSON_DIR16
    acc16_out(A, acc);
  } else {
#define CLG_WILSON_DIR(MU)                                                              \
  {                                                                                     \
    cpx<AT> psi[12], u[9];                                                              \
    load_site<P, 12, AT>(in, in_norm, Vh, nb.hf[MU], psi);                              \
    load_link<P, RECON, AT>(Uh, MU, lVh, h, u);                                         \
    wilson_hop_dir<AT, MU, SF, false>(acc, psi, u, (AT)nb.sf[MU]);                      \
    load_site<P, 12, AT>(in, in_norm, Vh, nb.hb[MU], psi);                              \
    load_link<P, RECON, AT>(Ut, MU, lVh, nb.hb[MU], u);                                 \
    wilson_hop_dir<AT, MU, SB, true>(acc, psi, u, (AT)nb.sb[MU]);                       \
  }
    CLG_WILSON_DIR(0)
    CLG_WILSON_DIR(1)
    CLG_WILSON_DIR(2)
    CLG_WILSON_DIR(3)
#undef CLG_WILSON_DIR
  }
  wilson_hop_finish<P>(a, rhs, h, acc);
}

template <int P, int RECON, bool DAGGER, typename AT>
__device__ __forceinline__ void wilson_hop_site(const HopArgs& a, int rhs, int64_t h, cpx<AT> acc[12]) {
  wilson_hop_site_on<P, RECON, DAGGER, false>(a, a.g, a.U_here, a.U_there, rhs, h, acc);
}

// The precision index of the batch link table (HopSeg::u)
template <int P> constexpr int seg_prec() { return P == P64 ? 0 : (P == P32 ? 1 : 2); }

// Right-hand side rhs of a batch of lattices: its own geometry and links.
// False for a padding site (h beyond that lattice's checkerboard).
template <int P, int RECON, bool DAGGER, typename AT>
__device__ __forceinline__ bool wilson_hop_site_batch(const HopArgs& a, int rhs, int64_t h, cpx<AT> acc[12]) {
  const HopSeg& sg = a.seg[rhs];
  if (h >= sg.g.Vh) return false;
  wilson_hop_site_on<P, RECON, DAGGER, true>(a, sg.g, sg.u[seg_prec<P>()][a.out_parity], sg.u[seg_prec<P>()][1 - a.out_parity],
                                       rhs, h, acc);
  return true;
}

// Register caps through the launch bounds (the autotuner picks per operator):
// (256, 3) caps at 80 registers (24 resident warps per SM instead of 16): the
// hop is latency-bound on its gathers, and the low-precision variants fit in
// 80 registers without spilling.  (64, 14) caps at 72 registers, 28 warps per
// SM: one rhs of a 32^3 x 16 checkerboard (262144 threads) then runs in two
// full waves instead of 2.3.
template <int P, int RECON, bool DAGGER, int MAXT = 256, int MINB = 1>
__global__ void __launch_bounds__(MAXT, MINB) wilson_hop_kernel(HopArgs a) {
  using AT = typename AccT<P>::T;
  // right-hand sides are interleaved in blockIdx.x so that the CTAs of all rhs
  // for the same sites run back to back and share the links through L2
  const int rhs = (int)(blockIdx.x % (unsigned)a.nrhs);
  const int64_t h = (int64_t)(blockIdx.x / (unsigned)a.nrhs) * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait();
  if (h >= a.g.Vh) return;
  if (a.skip_dev && a.skip_dev[(int64_t)rhs * a.skip_stride]) return;
  cpx<AT> acc[12];
  wilson_hop_site<P, RECON, DAGGER>(a, rhs, h, acc);
  wilson_hop_store<P>(a, rhs, h, acc);
}

// The hop over a batch of lattices (HopArgs::seg): right-hand side r on its own
// lattice, the grid spanning the largest checkerboard.
// (the register caps of the tuned one-lattice kernels: 80 for FP32 / FP16,
// 128 for FP64)
template <int P, int RECON, bool DAGGER>
__global__ void __launch_bounds__(256, P == P64 ? 2 : 3) wilson_hop_batch_kernel(HopArgs a) {
  using AT = typename AccT<P>::T;
  const int rhs = (int)(blockIdx.x % (unsigned)a.nrhs);
  const int64_t h = (int64_t)(blockIdx.x / (unsigned)a.nrhs) * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait();
  if (h >= a.g.Vh) return;
  if (a.skip_dev && a.skip_dev[(int64_t)rhs * a.skip_stride]) return;
  cpx<AT> acc[12];
  if (wilson_hop_site_batch<P, RECON, DAGGER>(a, rhs, h, acc)) wilson_hop_store<P>(a, rhs, h, acc);
}

// The hop with a fused epilogue E (used by the Krylov solvers):
//   E::STORE      the result is stored to a.out (else it only feeds E::site)
//   E::NRED       doubles reduced over the grid per rhs, E::finalize(rhs, tot)
//                 runs on the device in the last block (grid_reduce_finalize2)
//   E::site(rhs, h, acc, red)   per-site work on the result in registers
// Every thread reaches the block reduction: out-of-range sites contribute
// zero; a block of a skipped (finished) right-hand side only takes its ticket,
// and E::finalize ignores such right-hand sides.
template <int P, int RECON, bool DAGGER, int MAXT, int MINB, class E, bool BATCH = false>
__global__ void __launch_bounds__(MAXT, MINB) wilson_hop_epi_kernel(HopArgs a, E e, double* partials,
                                                                    double* gpart, unsigned* counter,
                                                                    unsigned group) {
  using AT = typename AccT<P>::T;
  const int rhs = (int)(blockIdx.x % (unsigned)a.nrhs);
  const unsigned slot = blockIdx.x / (unsigned)a.nrhs;
  const int64_t h = (int64_t)slot * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait();
  // in a batch of lattices a block wholly in this rhs's padding reduces nothing
  const bool skipped = (a.skip_dev && a.skip_dev[(int64_t)rhs * a.skip_stride]) ||
                       (BATCH && (int64_t)slot * blockDim.x >= a.seg_vh[rhs]);
  double red[E::NRED];
#pragma unroll
  for (int k = 0; k < E::NRED; ++k) red[k] = 0.0;
  if (!skipped && h < a.g.Vh) {
    cpx<AT> acc[12];
    bool valid = true;
    if constexpr (BATCH)
      valid = wilson_hop_site_batch<P, RECON, DAGGER>(a, rhs, h, acc);
    else
      wilson_hop_site<P, RECON, DAGGER>(a, rhs, h, acc);
    if (valid) {
      if constexpr (E::STORE) wilson_hop_store<P>(a, rhs, h, acc);
      e.site(rhs, h, acc, red);
    }
  }
  const int rr[1] = {rhs};
  const bool cc[1] = {!skipped}, hh[1] = {true};
  grid_reduce_finalize2<E::NRED, 1>(red, e, rr, cc, hh, (unsigned)rhs, (unsigned)a.nrhs, slot,
                                    gridDim.x / (unsigned)a.nrhs, a.nrhs, group, partials, gpart, counter,
                                    BATCH ? a.seg_vh : nullptr);
}

// ---------------------------------------------------------------- FP16, two right-hand sides per thread
// The multi-right-hand-side form of the FP16 hop (the batched solves of many
// sources on one gauge field): one thread computes one output site for a pair
// of right-hand sides (rhs0, rhs1).  The link of each direction is loaded and
// its third row rebuilt once for both, the neighbour indices and boundary
// signs are computed once, and the two spinors are held "planar": one half2
// word carries the real parts of the same component of rhs0 and rhs1, another
// the imaginary parts.  The spin projection's phases then cost nothing (they
// select a plane and a sign), every HFMA2 of the colour product does useful
// work for both right-hand sides, and the FP32 accumulation is one packed
// f32x2 FMA per component pair.  Each product is evaluated with the same
// operands in the same order as the one-rhs kernel (wilson_hop_dir16), so the
// two kernels give bit-identical results.
template <int MU, int SGN, bool UDAG>
__device__ __forceinline__ void wilson_hop_dir16_pair(float2 accR[12], float2 accI[12], const Packed16& p0,
                                                      const Packed16& p1, const PackedLink16& l, float s0, float s1) {
  constexpr int add = SGN < 0 ? 2 : 0;
  uint32_t w0[12], w1[12];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    w0[4 * k + 0] = p0.c[k].x; w0[4 * k + 1] = p0.c[k].y; w0[4 * k + 2] = p0.c[k].z; w0[4 * k + 3] = p0.c[k].w;
    w1[4 * k + 0] = p1.c[k].x; w1[4 * k + 1] = p1.c[k].y; w1[4 * k + 2] = p1.c[k].z; w1[4 * k + 3] = p1.c[k].w;
  }
  // planar spin projection: h_j[c] = psi[j][c] + i^z_j psi[perm_j][c], j = 0, 1
  __half2 hR[2][3], hI[2][3];
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      // spin s of colour c: half (s & 1) of the spin-planar words of pair s >> 1
      const int sa = j, sb = gperm(MU, j);
      const int ar = spinor_word(sa >> 1, c, 0), ai = spinor_word(sa >> 1, c, 1);
      const int br = spinor_word(sb >> 1, c, 0), bi = spinor_word(sb >> 1, c, 1);
      const unsigned sela = (sa & 1) ? 0x7632 : 0x5410, selb = (sb & 1) ? 0x7632 : 0x5410;
      const __half2 aR = as_h2(__byte_perm(w0[ar], w1[ar], sela)), aI = as_h2(__byte_perm(w0[ai], w1[ai], sela));
      const __half2 bR = as_h2(__byte_perm(w0[br], w1[br], selb)), bI = as_h2(__byte_perm(w0[bi], w1[bi], selb));
      const int z = (gz4(MU, j) + add) & 3;
      if (z == 0) { hR[j][c] = __hadd2(aR, bR); hI[j][c] = __hadd2(aI, bI); }
      else if (z == 1) { hR[j][c] = __hsub2(aR, bI); hI[j][c] = __hadd2(aI, bR); }
      else if (z == 2) { hR[j][c] = __hsub2(aR, bR); hI[j][c] = __hsub2(aI, bI); }
      else { hR[j][c] = __hadd2(aR, bI); hI[j][c] = __hsub2(aI, bR); }
    }
  // the link (rows 0, 1 stored; row 2 = conj(row0 x row1)), as in wilson_hop_dir16
  uint32_t u[9] = {l.a.x, l.a.y, l.a.z, l.a.w, l.b.x, l.b.y, 0u, 0u, 0u};
  {
    const __half2 zero = __float2half2_rn(0.f);
    auto cross = [&](int a, int b, int c, int d) -> uint32_t {
      __half2 t = h2_cmac<false>(__low2half2(as_h2(u[a])), __high2half2(as_h2(u[a])), u[b], zero);
      const uint32_t nd = u[d] ^ 0x80008000u;
      t = h2_cmac<false>(__low2half2(as_h2(u[c])), __high2half2(as_h2(u[c])), nd, t);
      return as_u32(t) ^ 0x80000000u;
    };
    const __half2 X = as_h2(__byte_perm(u[1], u[2], 0x5410)), Xi = as_h2(__byte_perm(u[1], u[2], 0x7632));
    const __half2 Y = as_h2(__byte_perm(u[5], u[3], 0x5410)), Yi = as_h2(__byte_perm(u[5], u[3], 0x7632));
    const __half2 Z = as_h2(__byte_perm(u[2], u[0], 0x5410)), Zi = as_h2(__byte_perm(u[2], u[0], 0x7632));
    const __half2 W = as_h2(__byte_perm(u[4], u[5], 0x5410)), Wi = as_h2(__byte_perm(u[4], u[5], 0x7632));
    __half2 re = __hmul2(X, Y);
    re = __hfma2(__hneg2(Xi), Yi, re);
    re = __hfma2(__hneg2(Z), W, re);
    re = __hfma2(Zi, Wi, re);
    __half2 nim = __hmul2(Z, Wi);
    nim = __hfma2(Zi, W, nim);
    nim = __hfma2(__hneg2(X), Yi, nim);
    nim = __hfma2(__hneg2(Xi), Y, nim);
    u[6] = __byte_perm(as_u32(re), as_u32(nim), 0x5410);
    u[7] = __byte_perm(as_u32(re), as_u32(nim), 0x7632);
    u[8] = cross(0, 4, 1, 3);
  }
  // colour products on the planar pair: g = U h (UDAG: U^+ h), with the real
  // part of the link element first, as h2_cmac does
  const __half2 zero = __float2half2_rn(0.f);
  __half2 gR[2][3], gI[2][3];
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int r = 0; r < 3; ++r) { gR[j][r] = zero; gI[j][r] = zero; }
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const uint32_t e = UDAG ? u[3 * k + r] : u[3 * r + k];
      const __half2 er = __low2half2(as_h2(e)), ei = __high2half2(as_h2(e));
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        gR[j][r] = __hfma2(er, hR[j][k], gR[j][r]);
        gI[j][r] = __hfma2(er, hI[j][k], gI[j][r]);
        if (UDAG) {  // conj(e) h: re += ei hI, im -= ei hR
          gR[j][r] = __hfma2(ei, hI[j][k], gR[j][r]);
          gI[j][r] = __hfma2(ei, __hneg2(hR[j][k]), gI[j][r]);
        } else {     // e h: re -= ei hI, im += ei hR
          gR[j][r] = __hfma2(ei, __hneg2(hI[j][k]), gR[j][r]);
          gI[j][r] = __hfma2(ei, hR[j][k], gI[j][r]);
        }
      }
    }
  // FP32 accumulation, packed over the pair
  const float2 ss = make_float2(s0, s1), sn = make_float2(-s0, -s1);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float2 fR[2], fI[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      fR[j] = __half22float2(gR[j][c]);
      fI[j] = __half22float2(gI[j][c]);
      accR[3 * j + c] = __ffma2_rn(ss, fR[j], accR[3 * j + c]);
      accI[3 * j + c] = __ffma2_rn(ss, fI[j], accI[3 * j + c]);
    }
#pragma unroll
    for (int row = 2; row < 4; ++row) {
      const int z = (gz4(MU, row) + add) & 3;
      const int j = gperm(MU, row);
      float2& aR = accR[3 * row + c];
      float2& aI = accI[3 * row + c];
      if (z == 0) { aR = __ffma2_rn(ss, fR[j], aR); aI = __ffma2_rn(ss, fI[j], aI); }
      else if (z == 1) { aR = __ffma2_rn(sn, fI[j], aR); aI = __ffma2_rn(ss, fR[j], aI); }
      else if (z == 2) { aR = __ffma2_rn(sn, fR[j], aR); aI = __ffma2_rn(sn, fI[j], aI); }
      else { aR = __ffma2_rn(ss, fI[j], aR); aI = __ffma2_rn(sn, fR[j], aI); }
    }
  }
}

// H in for output site h of the right-hand sides rhs0 and rhs1 (FP16 storage,
// 12-real links), then the finish (a H in + xa x, optional scale) per rhs.
template <bool DAGGER>
__device__ __forceinline__ void wilson_hop_site_pair16(const HopArgs& a, int rhs0, int rhs1, int64_t h,
                                                       cpx<float> acc0[12], cpx<float> acc1[12]) {
  const int64_t Vh = a.g.Vh;
  const char* in0 = reinterpret_cast<const char*>(a.in) + rhs0 * a.in_stride;
  const char* in1 = reinterpret_cast<const char*>(a.in) + rhs1 * a.in_stride;
  const float* n0 = a.in_norm + rhs0 * a.in_nstride;
  const float* n1 = a.in_norm + rhs1 * a.in_nstride;
  NbrInfo nb;
  int c[4];
  neighbours(a.g, a.out_parity, h, nb, c);
  float2 accR[12], accI[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    accR[k] = make_float2(0.f, 0.f);
    accI[k] = make_float2(0.f, 0.f);
  }
  constexpr int SF = DAGGER ? 1 : -1;
  constexpr int SB = -SF;
#define CLG_WILSON_DIR16_PAIR(MU)                                                                         \
  {                                                                                                       \
    Packed16 pf0, pf1;                                                                                    \
    PackedLink16 lf;                                                                                      \
    load_packed16(in0, n0, Vh, nb.hf[MU], pf0);                                                           \
    load_packed16(in1, n1, Vh, nb.hf[MU], pf1);                                                           \
    load_packed_link16(a.U_here, MU, Vh, h, lf);                                                          \
    wilson_hop_dir16_pair<MU, SF, false>(accR, accI, pf0, pf1, lf, nb.sf[MU] * pf0.n, nb.sf[MU] * pf1.n); \
    Packed16 pb0, pb1;                                                                                    \
    PackedLink16 lb;                                                                                      \
    load_packed16(in0, n0, Vh, nb.hb[MU], pb0);                                                           \
    load_packed16(in1, n1, Vh, nb.hb[MU], pb1);                                                           \
    load_packed_link16(a.U_there, MU, Vh, nb.hb[MU], lb);                                                 \
    wilson_hop_dir16_pair<MU, SB, true>(accR, accI, pb0, pb1, lb, nb.sb[MU] * pb0.n, nb.sb[MU] * pb1.n);  \
  }
  CLG_WILSON_DIR16_PAIR(0)
  CLG_WILSON_DIR16_PAIR(1)
  CLG_WILSON_DIR16_PAIR(2)
  CLG_WILSON_DIR16_PAIR(3)
#undef CLG_WILSON_DIR16_PAIR
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    acc0[k] = mk<float>(accR[k].x, accI[k].x);
    acc1[k] = mk<float>(accR[k].y, accI[k].y);
  }
  wilson_hop_finish<P16>(a, rhs0, h, acc0);
  wilson_hop_finish<P16>(a, rhs1, h, acc1);
}

// Pairs of right-hand sides are interleaved in blockIdx.x (pair = blockIdx.x %
// npairs).  With an odd count the last pair's second member repeats the first
// and is neither stored nor reduced.
__device__ __forceinline__ void pair_of(const HopArgs& a, unsigned npairs, int& rhs0, int& rhs1, bool& has1,
                                        unsigned& slot) {
  const unsigned q = blockIdx.x % npairs;
  slot = blockIdx.x / npairs;
  rhs0 = 2 * (int)q;
  has1 = rhs0 + 1 < a.nrhs;
  rhs1 = has1 ? rhs0 + 1 : rhs0;
}

template <bool DAGGER, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) wilson_hop_pair_kernel(HopArgs a) {
  const unsigned npairs = (unsigned)(a.nrhs + 1) / 2u;
  int rhs0, rhs1;
  bool has1;
  unsigned slot;
  pair_of(a, npairs, rhs0, rhs1, has1, slot);
  const int64_t h = (int64_t)slot * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait();
  if (h >= a.g.Vh) return;
  const bool run0 = !(a.skip_dev && a.skip_dev[(int64_t)rhs0 * a.skip_stride]);
  const bool run1 = has1 && !(a.skip_dev && a.skip_dev[(int64_t)rhs1 * a.skip_stride]);
  if (!run0 && !run1) return;
  cpx<float> acc0[12], acc1[12];
  wilson_hop_site_pair16<DAGGER>(a, rhs0, rhs1, h, acc0, acc1);
  if (run0) wilson_hop_store<P16>(a, rhs0, h, acc0);
  if (run1) wilson_hop_store<P16>(a, rhs1, h, acc1);
}

// The pair form of wilson_hop_epi_kernel: E::site runs once per right-hand
// side of the pair; the block reduces both right-hand sides' values.
template <bool DAGGER, int MAXT, int MINB, class E>
__global__ void __launch_bounds__(MAXT, MINB) wilson_hop_pair_epi_kernel(HopArgs a, E e, double* partials,
                                                                         double* gpart, unsigned* counter,
                                                                         unsigned group) {
  const unsigned npairs = (unsigned)(a.nrhs + 1) / 2u;
  int rhs0, rhs1;
  bool has1;
  unsigned slot;
  pair_of(a, npairs, rhs0, rhs1, has1, slot);
  const int64_t h = (int64_t)slot * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait();
  const bool run0 = !(a.skip_dev && a.skip_dev[(int64_t)rhs0 * a.skip_stride]);
  const bool run1 = has1 && !(a.skip_dev && a.skip_dev[(int64_t)rhs1 * a.skip_stride]);
  double red[2 * E::NRED];
#pragma unroll
  for (int k = 0; k < 2 * E::NRED; ++k) red[k] = 0.0;
  if ((run0 || run1) && h < a.g.Vh) {
    cpx<float> acc0[12], acc1[12];
    wilson_hop_site_pair16<DAGGER>(a, rhs0, rhs1, h, acc0, acc1);
    if (run0) {
      if constexpr (E::STORE) wilson_hop_store<P16>(a, rhs0, h, acc0);
      e.site(rhs0, h, acc0, red);
    }
    if (run1) {
      if constexpr (E::STORE) wilson_hop_store<P16>(a, rhs1, h, acc1);
      e.site(rhs1, h, acc1, red + E::NRED);
    }
  }
  const int rr[2] = {rhs0, rhs1};
  const bool cc[2] = {run0, run1}, hh[2] = {true, has1};
  grid_reduce_finalize2<E::NRED, 2>(red, e, rr, cc, hh, (unsigned)(rhs0 / 2), npairs, slot, gridDim.x / npairs,
                                    a.nrhs, group, partials, gpart, counter);
}

// ---------------------------------------------------------------- FP16, a tile of sites for every right-hand side
// The multi-right-hand-side FP16 hop with the links of a tile of 32 output
// sites loaded and completed (third row) once for all right-hand sides.  The
// block first stages, for its 32 sites, the neighbour indices with the
// boundary signs and the 8 links of each site (U_mu(x), U_mu(x - mu)) as
// 18-real half2 words in shared memory; then its warps loop over the
// right-hand sides (warp w takes rhs w, w + nwarps, ...), each lane computing
// one output site per right-hand side with the links read from shared memory.
// Per site and rhs this drops the link loads from global memory, the third-row
// rebuild and the neighbour arithmetic of the one-rhs kernel, and each link
// crosses DRAM once per launch whatever the L2 holds.  The arithmetic per site
// and rhs is wilson_hop_dir16_u's, so the results are bit-identical to the
// one-rhs kernel.
constexpr int TILE16 = 32;
// the y-rows per chunk of the blocked tile order for this lattice, rhs count
// and tile size (dslash.cu)
int tile_rows(const Geom& g, int nrhs, int ts = TILE16, int sbytes = 52);
// bytes of one Wilson spinor per site and rhs (FP16: with its norm)
template <int P> constexpr int spinor_bytes() { return P == P64 ? 192 : (P == P32 ? 96 : 52); }
struct Tile16 {
  uint4 la[8][TILE16];     // link words 0-3; direction d < 4: U_d(x), d >= 4: U_(d-4)(x - mu)
  uint4 lb[8][TILE16];     // words 4-7
  uint32_t lc[8][TILE16];  // word 8
  int nb[8][TILE16];       // checkerboard index of x + mu (d < 4), of x - mu (d >= 4)
  uint32_t neg[TILE16];    // bit d: the boundary sign of direction d is -1
};

// The tile of block blockIdx.x.  In site order a spinor is read by the tiles
// of its x-neighbours a whole (y, z, t) volume apart, so the L2 would have to
// hold about three such slabs of every right-hand side.  With tile_rows > 0
// (the lattice's z-t planes a whole number of tiles, L_y a multiple of
// tile_rows) the blocks instead walk chunk after chunk of tile_rows y-rows,
// x slowest within a chunk: the slabs shrink by L_y / tile_rows, and only the
// y-neighbours across a chunk's edge are read from DRAM a second time.
template <int TS>
__device__ __forceinline__ int64_t tile_index(const HopArgs& a) {
  const int64_t b = blockIdx.x;
  if (a.tile_rows <= 0) return b;
  const int64_t np = (int64_t)a.g.L[2] * a.g.L[3] / (2 * TS);  // tiles per (x, y) plane
  const int64_t per_x = a.tile_rows * np, per_chunk = a.g.L[0] * per_x;
  const int64_t yc = b / per_chunk, r = b - yc * per_chunk;
  const int64_t x = r / per_x, r2 = r - x * per_x;
  const int64_t yi = r2 / np, k = r2 - yi * np;
  return (x * a.g.L[1] + yc * a.tile_rows + yi) * np + k;
}
__device__ __forceinline__ int64_t tile16_index(const HopArgs& a) { return tile_index<TILE16>(a); }

// The neighbours of the tile's sites (geometry only: no memory is read, so
// this runs before the wait on the previous kernel)
template <class T>
__device__ __forceinline__ void tile16_neighbours(const Geom& g, int parity, int64_t h0, T& t) {
  for (int i = threadIdx.x; i < TILE16; i += blockDim.x) {
    const int64_t h = h0 + i;
    uint32_t neg = 0;
    if (h < g.Vh) {
      NbrInfo nb;
      int c[4];
      neighbours(g, parity, h, nb, c);
#pragma unroll
      for (int mu = 0; mu < 4; ++mu) {
        t.nb[mu][i] = nb.hf[mu];
        t.nb[4 + mu][i] = nb.hb[mu];
        neg |= (nb.sf[mu] < 0.f ? 1u : 0u) << mu;
        neg |= (nb.sb[mu] < 0.f ? 1u : 0u) << (4 + mu);
      }
    } else {
#pragma unroll
      for (int d = 0; d < 8; ++d) t.nb[d][i] = 0;
    }
    t.neg[i] = neg;
  }
}

// The tile's links, third row rebuilt (after tile16_neighbours and a barrier);
// Uh / Ut the link arrays of the output / input parity, Vh the lattice's
// checkerboard size (their stride)
__device__ __forceinline__ void tile16_links(const void* Uh, const void* Ut, int64_t Vh, int64_t h0, Tile16& t) {
  for (int k = threadIdx.x; k < 8 * TILE16; k += blockDim.x) {
    const int d = k / TILE16, i = k % TILE16;
    const int64_t h = h0 + i;
    uint32_t u[9] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
    if (h < Vh) {
      PackedLink16 l;
      if (d < 4)
        load_packed_link16(Uh, d, Vh, h, l);
      else
        load_packed_link16(Ut, d - 4, Vh, t.nb[d][i], l);
      u[0] = l.a.x; u[1] = l.a.y; u[2] = l.a.z; u[3] = l.a.w; u[4] = l.b.x; u[5] = l.b.y;
      link16_third_row(u);
    }
    t.la[d][i] = make_uint4(u[0], u[1], u[2], u[3]);
    t.lb[d][i] = make_uint4(u[4], u[5], u[6], u[7]);
    t.lc[d][i] = u[8];
  }
}

__device__ __forceinline__ void tile16_link(const Tile16& t, int d, int i, uint32_t (&u)[9]) {
  const uint4 x = t.la[d][i], y = t.lb[d][i];
  u[0] = x.x; u[1] = x.y; u[2] = x.z; u[3] = x.w;
  u[4] = y.x; u[5] = y.y; u[6] = y.z; u[7] = y.w;
  u[8] = t.lc[d][i];
}

// H in at tile site i (output site h) of right-hand side rhs, then the finish
template <bool DAGGER>
__device__ __forceinline__ void wilson_hop_site_tile16(const HopArgs& a, const Tile16& t, int i, int rhs, int64_t h,
                                                       cpx<float> acc[12]) {
  const int64_t Vh = a.g.Vh;
  const char* in = reinterpret_cast<const char*>(a.in) + rhs * a.in_stride;
  const float* in_norm = a.in_norm + rhs * a.in_nstride;
  Acc16 A;
  acc16_zero(A);
  const uint32_t neg = t.neg[i];
  constexpr int SF = DAGGER ? 1 : -1;
  constexpr int SB = -SF;
#define CLG_TILE_DIR16(MU)                                                   \
  {                                                                          \
    Packed16 pf, pb;                                                         \
    load_packed16(in, in_norm, Vh, t.nb[MU][i], pf);                         \
    load_packed16(in, in_norm, Vh, t.nb[4 + MU][i], pb);                     \
    uint32_t u[9];                                                           \
    tile16_link(t, MU, i, u);                                                \
    wilson_hop_dir16_u<MU, SF, false>(A, pf, u, (neg >> MU) & 1u ? -pf.n : pf.n);         \
    tile16_link(t, 4 + MU, i, u);                                            \
    wilson_hop_dir16_u<MU, SB, true>(A, pb, u, (neg >> (4 + MU)) & 1u ? -pb.n : pb.n);    \
  }
  CLG_TILE_DIR16(0)
  CLG_TILE_DIR16(1)
  CLG_TILE_DIR16(2)
  CLG_TILE_DIR16(3)
#undef CLG_TILE_DIR16
  acc16_out(A, acc);
  wilson_hop_finish<P16>(a, rhs, h, acc);
}

// Whether any of the right-hand sides [r0, r1) still needs work (uniform over
// the block; after the wait on the previous kernel, which may have set skips).
// A block whose right-hand sides have all finished stages nothing.
__device__ __forceinline__ bool tile_any_live(const HopArgs& a, int r0, int r1) {
  if (!a.skip_dev) return r1 > r0;
  for (int r = r0; r < r1; ++r)
    if (!a.skip_dev[(int64_t)r * a.skip_stride]) return true;
  return false;
}

// The work of one tile block: lattice g (links Uh, Ut), output sites
// [h0, h0 + 32), right-hand sides [r0, r1).  In a batch of lattices g is one
// lattice of the batch and a.g.Vh the fields' (padded) chunk stride.
template <bool DAGGER>
__device__ __forceinline__ void tile16_body(const HopArgs& a, Tile16& t, const Geom& g, const void* Uh,
                                            const void* Ut, int64_t h0, int r0, int r1) {
  pdl_launch_dependents();
  tile16_neighbours(g, a.out_parity, h0, t);
  pdl_wait();
  if (!tile_any_live(a, r0, r1)) return;  // no barrier has been passed yet: uniform
  __syncthreads();
  tile16_links(Uh, Ut, g.Vh, h0, t);
  __syncthreads();
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int64_t h = h0 + lane;
  if (h >= g.Vh) return;  // no barrier follows
  for (int rhs = r0 + (threadIdx.x >> 5); rhs < r1; rhs += nw) {
    if (a.skip_dev && a.skip_dev[(int64_t)rhs * a.skip_stride]) continue;
    cpx<float> acc[12];
    wilson_hop_site_tile16<DAGGER>(a, t, lane, rhs, h, acc);
    wilson_hop_store<P16>(a, rhs, h, acc);
  }
}

// One block per tile of 32 output sites, blockDim = 32 x (warps sharing the
// right-hand sides); MINB 2 leaves the registers uncapped (128), 3 caps at 80;
// MAXT 128 with MINB 7 caps at 72 (7 blocks of 4 warps per SM).
// BATCH: a batch of lattices, one block per tile of one lattice (btile).
template <bool DAGGER, int MINB, bool BATCH = false, int MAXT = 256>
__global__ void __launch_bounds__(MAXT, MINB) wilson_hop_tile16_kernel(HopArgs a) {
  __shared__ Tile16 t;
  if constexpr (BATCH) {
    const BatchTile bt = batch_tile(a);
    const HopSeg& sg = a.seg[bt.seg];
    const Geom g = sg.g;
    tile16_body<DAGGER>(a, t, g, sg.u[2][a.out_parity], sg.u[2][1 - a.out_parity],
                        ((int64_t)blockIdx.x - bt.tile0) * TILE16, bt.rhs0, bt.rhs0 + bt.nrhs);
  } else {
    tile16_body<DAGGER>(a, t, a.g, a.U_here, a.U_there, tile16_index(a) * TILE16, 0, a.nrhs);
  }
}

// The epilogue form of tile16_body: per right-hand side the warp reduces its
// 32 sites and writes the tile's partial (slot = block); in a batch the block
// writes zero partials for the other lattices' right-hand sides.  The blocks
// then reduce in two levels (tile_reduce_finalize).
template <bool DAGGER, class E>
__device__ __forceinline__ void tile16_epi_body(const HopArgs& a, const E& e, Tile16& t, const Geom& g,
                                                const void* Uh, const void* Ut, int64_t h0, int r0, int r1,
                                                double* partials, double* gpart, unsigned* counter,
                                                unsigned group) {
  pdl_launch_dependents();
  tile16_neighbours(g, a.out_parity, h0, t);
  pdl_wait();
  const bool any = tile_any_live(a, r0, r1);
  __syncthreads();
  if (any) tile16_links(Uh, Ut, g.Vh, h0, t);
  __syncthreads();
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int64_t h = h0 + lane;
  const unsigned nslots = gridDim.x;
  for (int rhs = r0 + (threadIdx.x >> 5); any && rhs < r1; rhs += nw) {
    if (a.skip_dev && a.skip_dev[(int64_t)rhs * a.skip_stride]) continue;
    double red[E::NRED];
#pragma unroll
    for (int k = 0; k < E::NRED; ++k) red[k] = 0.0;
    if (h < g.Vh) {
      cpx<float> acc[12];
      wilson_hop_site_tile16<DAGGER>(a, t, lane, rhs, h, acc);
      if constexpr (E::STORE) wilson_hop_store<P16>(a, rhs, h, acc);
      e.site(rhs, h, acc, red);
    }
#pragma unroll
    for (int k = 0; k < E::NRED; ++k) {
      double v = red[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) partials[((int64_t)rhs * nslots + blockIdx.x) * E::NRED + k] = v;
    }
    if (lane == 0) __threadfence();
  }
  if (r0 > 0 || r1 < a.nrhs) {
    for (int q = threadIdx.x; q < a.nrhs * E::NRED; q += blockDim.x) {
      const int rhs = q / E::NRED;
      if (rhs < r0 || rhs >= r1) partials[((int64_t)rhs * nslots + blockIdx.x) * E::NRED + q % E::NRED] = 0.0;
    }
    __threadfence();
  }
  tile_reduce_finalize<E::NRED>(e, nslots, a.nrhs, group, partials, gpart, counter);
}

template <bool DAGGER, int MINB, class E, bool BATCH = false, int MAXT = 256>
__global__ void __launch_bounds__(MAXT, MINB) wilson_hop_tile16_epi_kernel(HopArgs a, E e, double* partials,
                                                                          double* gpart, unsigned* counter,
                                                                          unsigned group) {
  __shared__ Tile16 t;
  if constexpr (BATCH) {
    const BatchTile bt = batch_tile(a);
    const HopSeg& sg = a.seg[bt.seg];
    const Geom g = sg.g;
    tile16_epi_body<DAGGER>(a, e, t, g, sg.u[2][a.out_parity], sg.u[2][1 - a.out_parity],
                            ((int64_t)blockIdx.x - bt.tile0) * TILE16, bt.rhs0, bt.rhs0 + bt.nrhs, partials,
                            gpart, counter, group);
  } else {
    tile16_epi_body<DAGGER>(a, e, t, a.g, a.U_here, a.U_there, tile16_index(a) * TILE16, 0, a.nrhs, partials,
                            gpart, counter, group);
  }
}

// ---------------------------------------------------------------- FP64 / FP32, a tile of sites for every right-hand side
// The tile form of the FP64 and FP32 hops: the block stages the 8 links of its
// 32 sites once (complete, as load_link gives them: 18-real, or 12-real with
// the third row rebuilt) as complex numbers in shared memory, then loops over
// the right-hand sides like wilson_hop_tile16_kernel.  The FP64 hop of a
// batched solve's outer residual re-reads 1152 link bytes per site and rhs
// through L2 in the one-rhs form; here each link crosses DRAM once per
// launch.  Arithmetic per site and rhs is wilson_hop_dir's (bit-identical).
template <typename AT>
struct TileN {
  cpx<AT> u[8][9][TILE16];  // direction d < 4: U_d(x), d >= 4: U_(d-4)(x - mu)
  int nb[8][TILE16];
  uint32_t neg[TILE16];
};

template <int P, int RECON, typename AT>
__device__ __forceinline__ void tileN_links(const void* Uh, const void* Ut, int64_t Vh, int64_t h0, TileN<AT>& t) {
  for (int k = threadIdx.x; k < 8 * TILE16; k += blockDim.x) {
    const int d = k / TILE16, i = k % TILE16;
    const int64_t h = h0 + i;
    cpx<AT> u[9];
    if (h < Vh) {
      if (d < 4)
        load_link<P, RECON, AT>(Uh, d, Vh, h, u);
      else
        load_link<P, RECON, AT>(Ut, d - 4, Vh, t.nb[d][i], u);
    } else {
#pragma unroll
      for (int w = 0; w < 9; ++w) u[w] = mk<AT>(0, 0);
    }
#pragma unroll
    for (int w = 0; w < 9; ++w) t.u[d][w][i] = u[w];
  }
}

template <int P, bool DAGGER, typename AT>
__device__ __forceinline__ void wilson_hop_site_tileN(const HopArgs& a, const TileN<AT>& t, int i, int rhs, int64_t h,
                                                      cpx<AT> acc[12]) {
  const int64_t Vh = a.g.Vh;
  const char* in = reinterpret_cast<const char*>(a.in) + rhs * a.in_stride;
  const float* in_norm = a.in_norm ? a.in_norm + rhs * a.in_nstride : nullptr;
#pragma unroll
  for (int k = 0; k < 12; ++k) acc[k] = mk<AT>(0, 0);
  const uint32_t neg = t.neg[i];
  constexpr int SF = DAGGER ? 1 : -1;
  constexpr int SB = -SF;
#define CLG_TILEN_DIR(MU)                                                              \
  {                                                                                    \
    cpx<AT> psi[12], u[9];                                                             \
    load_site<P, 12, AT>(in, in_norm, Vh, t.nb[MU][i], psi);                           \
    _Pragma("unroll") for (int w = 0; w < 9; ++w) u[w] = t.u[MU][w][i];                \
    wilson_hop_dir<AT, MU, SF, false>(acc, psi, u, (neg >> MU) & 1u ? (AT)-1 : (AT)1); \
    load_site<P, 12, AT>(in, in_norm, Vh, t.nb[4 + MU][i], psi);                       \
    _Pragma("unroll") for (int w = 0; w < 9; ++w) u[w] = t.u[4 + MU][w][i];            \
    wilson_hop_dir<AT, MU, SB, true>(acc, psi, u, (neg >> (4 + MU)) & 1u ? (AT)-1 : (AT)1); \
  }
  CLG_TILEN_DIR(0)
  CLG_TILEN_DIR(1)
  CLG_TILEN_DIR(2)
  CLG_TILEN_DIR(3)
#undef CLG_TILEN_DIR
  wilson_hop_finish<P>(a, rhs, h, acc);
}

template <int P, int RECON, bool DAGGER, typename AT>
__device__ __forceinline__ void tileN_body(const HopArgs& a, TileN<AT>& t, const Geom& g, const void* Uh,
                                           const void* Ut, int64_t h0, int r0, int r1) {
  pdl_launch_dependents();
  tile16_neighbours(g, a.out_parity, h0, t);
  pdl_wait();
  if (!tile_any_live(a, r0, r1)) return;  // no barrier has been passed yet: uniform
  __syncthreads();
  tileN_links<P, RECON>(Uh, Ut, g.Vh, h0, t);
  __syncthreads();
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int64_t h = h0 + lane;
  if (h >= g.Vh) return;  // no barrier follows
  for (int rhs = r0 + (threadIdx.x >> 5); rhs < r1; rhs += nw) {
    if (a.skip_dev && a.skip_dev[(int64_t)rhs * a.skip_stride]) continue;
    cpx<AT> acc[12];
    wilson_hop_site_tileN<P, DAGGER>(a, t, lane, rhs, h, acc);
    wilson_hop_store<P>(a, rhs, h, acc);
  }
}

template <int P, int RECON, bool DAGGER, int MINB, bool BATCH = false>
__global__ void __launch_bounds__(256, MINB) wilson_hop_tileN_kernel(HopArgs a) {
  using AT = typename AccT<P>::T;
  __shared__ TileN<AT> t;
  if constexpr (BATCH) {
    const BatchTile bt = batch_tile(a);
    const HopSeg& sg = a.seg[bt.seg];
    const Geom g = sg.g;
    tileN_body<P, RECON, DAGGER>(a, t, g, sg.u[seg_prec<P>()][a.out_parity], sg.u[seg_prec<P>()][1 - a.out_parity],
                                 ((int64_t)blockIdx.x - bt.tile0) * TILE16, bt.rhs0, bt.rhs0 + bt.nrhs);
  } else {
    tileN_body<P, RECON, DAGGER>(a, t, a.g, a.U_here, a.U_there, tile16_index(a) * TILE16, 0, a.nrhs);
  }
}

template <int P, int RECON, bool DAGGER, class E, typename AT>
__device__ __forceinline__ void tileN_epi_body(const HopArgs& a, const E& e, TileN<AT>& t, const Geom& g,
                                               const void* Uh, const void* Ut, int64_t h0, int r0, int r1,
                                               double* partials, double* gpart, unsigned* counter, unsigned group) {
  pdl_launch_dependents();
  tile16_neighbours(g, a.out_parity, h0, t);
  pdl_wait();
  const bool any = tile_any_live(a, r0, r1);
  __syncthreads();
  if (any) tileN_links<P, RECON>(Uh, Ut, g.Vh, h0, t);
  __syncthreads();
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int64_t h = h0 + lane;
  const unsigned nslots = gridDim.x;
  for (int rhs = r0 + (threadIdx.x >> 5); any && rhs < r1; rhs += nw) {
    if (a.skip_dev && a.skip_dev[(int64_t)rhs * a.skip_stride]) continue;
    double red[E::NRED];
#pragma unroll
    for (int k = 0; k < E::NRED; ++k) red[k] = 0.0;
    if (h < g.Vh) {
      cpx<AT> acc[12];
      wilson_hop_site_tileN<P, DAGGER>(a, t, lane, rhs, h, acc);
      if constexpr (E::STORE) wilson_hop_store<P>(a, rhs, h, acc);
      e.site(rhs, h, acc, red);
    }
#pragma unroll
    for (int k = 0; k < E::NRED; ++k) {
      double v = red[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) partials[((int64_t)rhs * nslots + blockIdx.x) * E::NRED + k] = v;
    }
    if (lane == 0) __threadfence();
  }
  if (r0 > 0 || r1 < a.nrhs) {
    for (int q = threadIdx.x; q < a.nrhs * E::NRED; q += blockDim.x) {
      const int rhs = q / E::NRED;
      if (rhs < r0 || rhs >= r1) partials[((int64_t)rhs * nslots + blockIdx.x) * E::NRED + q % E::NRED] = 0.0;
    }
    __threadfence();
  }
  tile_reduce_finalize<E::NRED>(e, nslots, a.nrhs, group, partials, gpart, counter);
}

template <int P, int RECON, bool DAGGER, int MINB, class E, bool BATCH = false>
__global__ void __launch_bounds__(256, MINB) wilson_hop_tileN_epi_kernel(HopArgs a, E e, double* partials,
                                                                         double* gpart, unsigned* counter,
                                                                         unsigned group) {
  using AT = typename AccT<P>::T;
  __shared__ TileN<AT> t;
  if constexpr (BATCH) {
    const BatchTile bt = batch_tile(a);
    const HopSeg& sg = a.seg[bt.seg];
    const Geom g = sg.g;
    tileN_epi_body<P, RECON, DAGGER>(a, e, t, g, sg.u[seg_prec<P>()][a.out_parity],
                                     sg.u[seg_prec<P>()][1 - a.out_parity], ((int64_t)blockIdx.x - bt.tile0) * TILE16,
                                     bt.rhs0, bt.rhs0 + bt.nrhs, partials, gpart, counter, group);
  } else {
    tileN_epi_body<P, RECON, DAGGER>(a, e, t, a.g, a.U_here, a.U_there, tile16_index(a) * TILE16, 0, a.nrhs, partials,
                                     gpart, counter, group);
  }
}

// ---------------------------------------------------------------- FP16 with the colour products on the tensor cores
// The multi-right-hand-side FP16 hop as small matrix products (mma.sync
// m16n8k16, FP16 operands, FP32 accumulation).  For output site x, with
// directions d = 2 mu + (0 forward, 1 backward), the hop is
//   out_s = sum_d U_d ( c_{d,s} h_d^(j_{d,s}) ),   s = 0..3,
// where h_d^(0,1) are the two spin-projected rows of the neighbour's spinor,
// rows 0, 1 take c = 1, j = s, and the rebuilt rows 2, 3 take the phase
// i^z and row perm of the chiral basis (linearity moves the phase before the
// link).  So per site, with one column per (right-hand side, output row s)
// holding the 8 directions' 3 colours (re, im) of c h (K = 8 x 8, 6 used), the
// whole hop of all right-hand sides is one product
//   OUT^T [columns x (colour, re/im)] = COL^T [columns x K] . E^T [K x 6]
// with E the real 6 x 6 embedding of each direction's link (U, or U^+
// backward).  A block takes a tile of MMA_TS sites and the right-hand sides in
// groups of MMA_G:
//   1. staging (all threads, lanes over sites: coalesced): for each (site,
//      rhs) the 8 neighbour norms give nmax; each neighbour spinor is
//      projected, scaled by sign * norm / nmax (<= 1, so FP16 cannot overflow)
//      and its four columns' K-blocks are stored to shared memory;
//   2. products (warp w = site w): per mu one k-step; the A fragments
//      (columns) by ldmatrix, the B fragment (the link embedding) built in
//      registers from the staged links; the FP32 accumulators hold the sums
//      over all 8 directions;
//   3. finish (thread per (site, rhs)): times nmax, then the usual epilogue
//      and store.
// The FP16 rounding differs from wilson_hop_kernel's (the projected rows are
// rounded once more when scaled; the colour sums are exact products summed in
// FP32 instead of HFMA2 chains), within the FP16 storage's precision.
constexpr int MMA_TS = 8;                       // sites per tile
constexpr int MMA_G = 16;                       // right-hand sides per group
constexpr int MMA_CS = 72;                      // halves per column: 8 x 8 + 8 pad (144 B: ldmatrix rows conflict-free)
constexpr int MMA_SS = 4 * MMA_G * MMA_CS + 8;  // halves per site (+16 B: staging stores conflict-free)
constexpr int MMA_CB = MMA_G * 12 + 2;          // float2 per site of the result buffer (+16 B)
struct Mma16Smem {
  __half col[MMA_TS * MMA_SS];  // per site: column (rhs_local * 4 + s), K = d * 8 + colour * 2 + re/im
  float2 res[MMA_TS * MMA_CB];  // per site: [rhs_local][s * 3 + colour] / nmax
  uint32_t u[8][9][MMA_TS];     // links as 9 half2 words, direction d = 2 mu + backward
  int nb[8][MMA_TS];            // neighbour checkerboard index per direction
  uint32_t neg[MMA_TS];         // bit d: boundary sign -1
  float nmax[MMA_TS][MMA_G];
};

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void* p) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}
__device__ __forceinline__ void mma_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// the tile's geometry and links (staged once per tile)
__device__ __forceinline__ void mma16_stage_geometry(const HopArgs& a, int64_t h0, Mma16Smem& t) {
  for (int i = threadIdx.x; i < MMA_TS; i += blockDim.x) {
    const int64_t h = h0 + i;
    uint32_t neg = 0;
    if (h < a.g.Vh) {
      NbrInfo nb;
      int c[4];
      neighbours(a.g, a.out_parity, h, nb, c);
#pragma unroll
      for (int mu = 0; mu < 4; ++mu) {
        t.nb[2 * mu][i] = nb.hf[mu];
        t.nb[2 * mu + 1][i] = nb.hb[mu];
        neg |= (nb.sf[mu] < 0.f ? 1u : 0u) << (2 * mu);
        neg |= (nb.sb[mu] < 0.f ? 1u : 0u) << (2 * mu + 1);
      }
    } else {
#pragma unroll
      for (int d = 0; d < 8; ++d) t.nb[d][i] = 0;
    }
    t.neg[i] = neg;
  }
}
__device__ __forceinline__ void mma16_stage_links(const HopArgs& a, int64_t h0, Mma16Smem& t) {
  for (int k = threadIdx.x; k < 8 * MMA_TS; k += blockDim.x) {
    const int d = k / MMA_TS, i = k % MMA_TS;
    const int64_t h = h0 + i;
    uint32_t u[9] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
    if (h < a.g.Vh) {
      PackedLink16 l;
      if ((d & 1) == 0)
        load_packed_link16(a.U_here, d >> 1, a.g.Vh, h, l);
      else
        load_packed_link16(a.U_there, d >> 1, a.g.Vh, t.nb[d][i], l);
      u[0] = l.a.x; u[1] = l.a.y; u[2] = l.a.z; u[3] = l.a.w; u[4] = l.b.x; u[5] = l.b.y;
      link16_third_row(u);
    }
#pragma unroll
    for (int w = 0; w < 9; ++w) t.u[d][w][i] = u[w];
  }
}

// One direction's four columns for (site i, rhs_local rl): the projected rows
// of the neighbour spinor p, scaled by r2, with the rebuilt rows' phases.
template <int MU, int SGN>
__device__ __forceinline__ void mma16_columns(__half* colsite, int rl, int d, const Packed16& p, __half2 r2) {
  constexpr int add = SGN < 0 ? 2 : 0;
  uint32_t sp[12];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    sp[4 * k + 0] = p.c[k].x;
    sp[4 * k + 1] = p.c[k].y;
    sp[4 * k + 2] = p.c[k].z;
    sp[4 * k + 3] = p.c[k].w;
  }
  // w[3 s + c]: spin s, colour c as one (re, im) word, from the spin-planar storage
  uint32_t w[12];
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      w[3 * s + c] = __byte_perm(sp[spinor_word(s >> 1, c, 0)], sp[spinor_word(s >> 1, c, 1)],
                                 (s & 1) ? 0x7632 : 0x5410);
  uint32_t h[2][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    h[0][c] = as_u32(__hmul2(__hadd2(as_h2(w[c]), as_h2(h2_mul_i<gz4(MU, 0) + add>(w[3 * gperm(MU, 0) + c]))), r2));
    h[1][c] = as_u32(__hmul2(__hadd2(as_h2(w[3 + c]), as_h2(h2_mul_i<gz4(MU, 1) + add>(w[3 * gperm(MU, 1) + c]))), r2));
  }
  constexpr int j2 = gperm(MU, 2), j3 = gperm(MU, 3);
  uint4* base = reinterpret_cast<uint4*>(colsite + (rl * 4) * MMA_CS + d * 8);
  constexpr int CS4 = MMA_CS / 8;  // uint4 per column
  base[0] = make_uint4(h[0][0], h[0][1], h[0][2], 0u);
  base[CS4] = make_uint4(h[1][0], h[1][1], h[1][2], 0u);
  base[2 * CS4] = make_uint4(h2_mul_i<gz4(MU, 2) + add>(h[j2][0]), h2_mul_i<gz4(MU, 2) + add>(h[j2][1]),
                             h2_mul_i<gz4(MU, 2) + add>(h[j2][2]), 0u);
  base[3 * CS4] = make_uint4(h2_mul_i<gz4(MU, 3) + add>(h[j3][0]), h2_mul_i<gz4(MU, 3) + add>(h[j3][1]),
                             h2_mul_i<gz4(MU, 3) + add>(h[j3][2]), 0u);
}

// Phase 1 for right-hand sides [r0, r0 + MMA_G): thread t stages site t % 8,
// rhs_local (t / 8) % 16, directions mu in {0, 1} (t < 128) or {2, 3}.
template <bool DAGGER>
__device__ __forceinline__ void mma16_stage_columns(const HopArgs& a, int64_t h0, int r0, Mma16Smem& t) {
  const int i = threadIdx.x % MMA_TS, rl = (threadIdx.x / MMA_TS) % MMA_G, dh = threadIdx.x / (MMA_TS * MMA_G);
  const int rhs = r0 + rl;
  const int64_t h = h0 + i;
  const bool valid = h < a.g.Vh && rhs < a.nrhs && !(a.skip_dev && a.skip_dev[(int64_t)rhs * a.skip_stride]);
  __half* colsite = t.col + i * MMA_SS;
  if (!valid) {
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
    for (int d = 0; d < 4; ++d)
#pragma unroll
      for (int s = 0; s < 4; ++s)
        reinterpret_cast<uint4*>(colsite + (rl * 4 + s) * MMA_CS + (4 * dh + d) * 8)[0] = z;
    if (dh == 0) t.nmax[i][rl] = 0.f;
    return;
  }
  const char* in = reinterpret_cast<const char*>(a.in) + rhs * a.in_stride;
  const float* in_norm = a.in_norm + rhs * a.in_nstride;
  float nm = 0.f;
#pragma unroll
  for (int d = 0; d < 8; ++d) nm = fmaxf(nm, __ldg(in_norm + t.nb[d][i]));
  if (dh == 0) t.nmax[i][rl] = nm;
  const float inv = nm > 0.f ? 1.f / nm : 0.f;
  const uint32_t neg = t.neg[i];
  constexpr int SF = DAGGER ? 1 : -1;
  constexpr int SB = -SF;
#define CLG_MMA_DIR(MU)                                                                          \
  {                                                                                              \
    Packed16 pf, pb;                                                                             \
    load_packed16(in, in_norm, a.g.Vh, t.nb[2 * MU][i], pf);                                     \
    load_packed16(in, in_norm, a.g.Vh, t.nb[2 * MU + 1][i], pb);                                 \
    const float rf = ((neg >> (2 * MU)) & 1u ? -pf.n : pf.n) * inv;                              \
    const float rb = ((neg >> (2 * MU + 1)) & 1u ? -pb.n : pb.n) * inv;                          \
    mma16_columns<MU, SF>(colsite, rl, 2 * MU, pf, __float2half2_rn(rf));                        \
    mma16_columns<MU, SB>(colsite, rl, 2 * MU + 1, pb, __float2half2_rn(rb));                    \
  }
  if (dh == 0) {
    CLG_MMA_DIR(0)
    CLG_MMA_DIR(1)
  } else {
    CLG_MMA_DIR(2)
    CLG_MMA_DIR(3)
  }
#undef CLG_MMA_DIR
}

// Phase 2: warp w multiplies site w's columns (ncols_tiles m-tiles of 16
// columns) by its links' embedding; results to t.res.
__device__ __forceinline__ void mma16_products(Mma16Smem& t, int mtiles) {
  const int lane = threadIdx.x & 31, i = threadIdx.x >> 5;
  if (i >= MMA_TS) return;
  const int g = lane >> 2, q = lane & 3;
  // the B fragment (E^T): lane holds E[n = g][k = 2q, 2q + 1] (forward link,
  // k < 8) and E[g][2q + 8, 2q + 9] (backward), n = colour a * 2 + re/im of
  // the output, k = colour b = q of the input (re, im)
  uint32_t bf[4][2];
  const int ca = g >> 1, ri = g & 1;
  const bool live = g < 6 && q < 3;
#pragma unroll
  for (int mu = 0; mu < 4; ++mu) {
    const uint32_t m = live ? t.u[2 * mu][3 * ca + q][i] : 0u;      // U[a][b]
    const uint32_t w = live ? t.u[2 * mu + 1][3 * q + ca][i] : 0u;  // U^+[a][b] = conj(U[b][a])
    bf[mu][0] = ri == 0 ? (m ^ 0x80000000u) : h2_swap(m);             // (Re M, -Im M) | (Im M, Re M)
    bf[mu][1] = ri == 0 ? w : (h2_swap(w) ^ 0x00008000u);            // M = conj(W): (Re W, Im W) | (-Im W, Re W)
  }
  const __half* colsite = t.col + i * MMA_SS;
  float2* res = t.res + i * MMA_CB;
  // ldmatrix.x4 rows: lanes 0-7 matrix 0 (columns 0-7, k 0-7), 8-15 matrix 1
  // (columns 8-15, k 0-7), 16-23 matrix 2 (columns 0-7, k 8-15), 24-31 matrix 3
  const int lrow = (lane & 7) + ((lane >> 3) & 1) * 8, lk = (lane >> 4) * 8;
  for (int mt = 0; mt < mtiles; ++mt) {
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    const __half* cp = colsite + (mt * 16 + lrow) * MMA_CS + lk;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
      uint32_t af[4];
      ldsm_x4(af, cp + mu * 16);
      mma_16816(acc, af, bf[mu][0], bf[mu][1]);
    }
    // acc[0, 1]: column mt * 16 + g, output colour q (re, im); acc[2, 3]: column + 8
    if (q < 3) {
      const int c0 = mt * 16 + g, c1 = c0 + 8;  // column = rhs_local * 4 + s
      res[(c0 >> 2) * 12 + (c0 & 3) * 3 + q] = make_float2(acc[0], acc[1]);
      res[(c1 >> 2) * 12 + (c1 & 3) * 3 + q] = make_float2(acc[2], acc[3]);
    }
  }
}

template <bool DAGGER, int MINB>
__global__ void __launch_bounds__(256, MINB) wilson_hop_mma16_kernel(HopArgs a) {
  extern __shared__ __align__(16) unsigned char mma_smem[];
  Mma16Smem& t = *reinterpret_cast<Mma16Smem*>(mma_smem);
  const int64_t h0 = tile_index<MMA_TS>(a) * MMA_TS;
  pdl_launch_dependents();
  mma16_stage_geometry(a, h0, t);
  pdl_wait();
  __syncthreads();
  mma16_stage_links(a, h0, t);
  for (int r0 = 0; r0 < a.nrhs; r0 += MMA_G) {
    mma16_stage_columns<DAGGER>(a, h0, r0, t);
    __syncthreads();
    mma16_products(t, (min(MMA_G, a.nrhs - r0) + 3) / 4);
    __syncthreads();
    if (threadIdx.x < MMA_TS * MMA_G) {
      const int i = threadIdx.x % MMA_TS, rl = threadIdx.x / MMA_TS, rhs = r0 + rl;
      const int64_t h = h0 + i;
      if (h < a.g.Vh && rhs < a.nrhs && !(a.skip_dev && a.skip_dev[(int64_t)rhs * a.skip_stride])) {
        const float nm = t.nmax[i][rl];
        const float2* rp = t.res + i * MMA_CB + rl * 12;
        cpx<float> acc[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) {
          const float2 v = rp[k];
          acc[k] = mk<float>(v.x * nm, v.y * nm);
        }
        wilson_hop_finish<P16>(a, rhs, h, acc);
        wilson_hop_store<P16>(a, rhs, h, acc);
      }
    }
    __syncthreads();
  }
}

// The epilogue form: per right-hand side the 8 sites of the tile reduce in
// groups of 8 lanes and write the tile's partial; tile_reduce_finalize after.
template <bool DAGGER, int MINB, class E>
__global__ void __launch_bounds__(256, MINB) wilson_hop_mma16_epi_kernel(HopArgs a, E e, double* partials,
                                                                         double* gpart, unsigned* counter,
                                                                         unsigned group) {
  extern __shared__ __align__(16) unsigned char mma_smem[];
  Mma16Smem& t = *reinterpret_cast<Mma16Smem*>(mma_smem);
  const int64_t h0 = tile_index<MMA_TS>(a) * MMA_TS;
  pdl_launch_dependents();
  mma16_stage_geometry(a, h0, t);
  pdl_wait();
  __syncthreads();
  mma16_stage_links(a, h0, t);
  const unsigned nslots = gridDim.x;
  for (int r0 = 0; r0 < a.nrhs; r0 += MMA_G) {
    mma16_stage_columns<DAGGER>(a, h0, r0, t);
    __syncthreads();
    mma16_products(t, (min(MMA_G, a.nrhs - r0) + 3) / 4);
    __syncthreads();
    if (threadIdx.x < MMA_TS * MMA_G) {
      const int i = threadIdx.x % MMA_TS, rl = threadIdx.x / MMA_TS, rhs = r0 + rl;
      const int64_t h = h0 + i;
      // uniform over the 8 lanes of (rl): rhs and its skip flag
      const bool live = rhs < a.nrhs && !(a.skip_dev && a.skip_dev[(int64_t)rhs * a.skip_stride]);
      double red[E::NRED];
#pragma unroll
      for (int k = 0; k < E::NRED; ++k) red[k] = 0.0;
      if (live && h < a.g.Vh) {
        const float nm = t.nmax[i][rl];
        const float2* rp = t.res + i * MMA_CB + rl * 12;
        cpx<float> acc[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) {
          const float2 v = rp[k];
          acc[k] = mk<float>(v.x * nm, v.y * nm);
        }
        wilson_hop_finish<P16>(a, rhs, h, acc);
        if constexpr (E::STORE) wilson_hop_store<P16>(a, rhs, h, acc);
        e.site(rhs, h, acc, red);
      }
#pragma unroll
      for (int k = 0; k < E::NRED; ++k) {
        double v = red[k];
#pragma unroll
        for (int o = MMA_TS / 2; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o, MMA_TS);
        if (live && i == 0) partials[((int64_t)rhs * nslots + blockIdx.x) * E::NRED + k] = v;
      }
      if (live && i == 0) __threadfence();
    }
    __syncthreads();
  }
  tile_reduce_finalize<E::NRED>(e, nslots, a.nrhs, group, partials, gpart, counter);
}

// The FP16 staggered direction on half2 words: o = U chi (UDAG: U^+ chi) with
// the link's third row rebuilt on half2 words and 2 HFMA2 per complex
// multiply-add (as wilson_hop_dir16), then acc += s o in packed FP32 (s = eta
// x boundary sign x the neighbour's site norm; the mat-vec is linear, so the
// norm is applied once to its result).
template <bool UDAG>
__device__ __forceinline__ void staggered_dir16(float2 acc[3], const uint32_t (&v)[3], const PackedLink16& l, float s) {
  uint32_t u[9] = {l.a.x, l.a.y, l.a.z, l.a.w, l.b.x, l.b.y, 0u, 0u, 0u};
  link16_third_row(u);
  const __half2 zero = __float2half2_rn(0.f);
  __half2 g[3] = {zero, zero, zero};
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const uint32_t e = UDAG ? u[3 * k + r] : u[3 * r + k];
      g[r] = h2_cmac<UDAG>(__low2half2(as_h2(e)), __high2half2(as_h2(e)), v[k], g[r]);
    }
  const float2 ss = make_float2(s, s);
#pragma unroll
  for (int c = 0; c < 3; ++c) acc[c] = __ffma2_rn(ss, __half22float2(g[c]), acc[c]);
}
__device__ __forceinline__ float load_color16(const void* __restrict__ base, const float* __restrict__ nrm, int64_t Vh,
                                              int64_t h, uint32_t (&v)[3]) {
  const uint32_t* b = reinterpret_cast<const uint32_t*>(base);
#pragma unroll
  for (int k = 0; k < 3; ++k) v[k] = __ldg(b + k * Vh + h);
  return __ldg(nrm + h);
}

// out = [scale *] (a H in + xa x) at (rhs, h), stored
template <int P, typename AT>
__device__ __forceinline__ void staggered_finish_store(const HopArgs& a, int rhs, int64_t h, cpx<AT> acc[3]) {
  const int64_t Vh = a.g.Vh;
  const cpx<AT> ca = mk<AT>((AT)a.a.x, (AT)a.a.y);
#pragma unroll
  for (int k = 0; k < 3; ++k) acc[k] = ca * acc[k];
  if (a.x) {
    cpx<AT> xv[3];
    const char* xp = reinterpret_cast<const char*>(a.x) + rhs * a.x_stride;
    load_site<P, 3, AT>(xp, a.x_norm ? a.x_norm + rhs * a.x_nstride : nullptr, Vh, h, xv);
    const cpx<AT> cx = mk<AT>((AT)a.xa.x, (AT)a.xa.y);
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[k] = acc[k] + cx * xv[k];
  }
  if (a.scale_dev) {
    const AT sc = (AT)a.scale_dev[rhs * a.scale_stride];
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[k] = sc * acc[k];
  }
  store_site<P, 3, AT>(reinterpret_cast<char*>(a.out) + rhs * a.out_stride,
                       a.out_norm ? a.out_norm + rhs * a.out_nstride : nullptr, Vh, h, acc);
}

// H in at output site h of right-hand side rhs (the sum over the 8 links,
// before the coefficients of the finish)
template <int P, int RECON>
__device__ __forceinline__ void staggered_hop_site(const HopArgs& a, int rhs, int64_t h,
                                                   cpx<typename AccT<P>::T> acc[3]) {
  using AT = typename AccT<P>::T;
  const int64_t Vh = a.g.Vh;
  const char* in = reinterpret_cast<const char*>(a.in) + rhs * a.in_stride;
  const float* in_norm = a.in_norm ? a.in_norm + rhs * a.in_nstride : nullptr;

  NbrInfo nb;
  int c[4];
  neighbours(a.g, a.out_parity, h, nb, c);

#pragma unroll
  for (int k = 0; k < 3; ++k) acc[k] = mk<AT>(0, 0);
  if constexpr (P == P16) {
    float2 a16[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
      int es = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (k < mu) es += c[k];
      const float eta = (es & 1) ? -1.f : 1.f;
      uint32_t vf[3], vb[3];
      PackedLink16 lf, lb;
      const float nf = load_color16(in, in_norm, Vh, nb.hf[mu], vf);
      load_packed_link16(a.U_here, mu, Vh, h, lf);
      const float nbn = load_color16(in, in_norm, Vh, nb.hb[mu], vb);
      load_packed_link16(a.U_there, mu, Vh, nb.hb[mu], lb);
      staggered_dir16<false>(a16, vf, lf, eta * nb.sf[mu] * nf);
      staggered_dir16<true>(a16, vb, lb, -eta * nb.sb[mu] * nbn);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[k] = mk<AT>(a16[k].x, a16[k].y);
  } else {
#pragma unroll
  for (int mu = 0; mu < 4; ++mu) {
    int es = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k < mu) es += c[k];
    const AT eta = (es & 1) ? (AT)-1 : (AT)1;
    cpx<AT> v[3], u[9], o[3];
    load_site<P, 3, AT>(in, in_norm, Vh, nb.hf[mu], v);
    load_link<P, RECON, AT>(a.U_here, mu, Vh, h, u);
    su3_mv<AT, false>(u, v, o);
    const AT sf = eta * (AT)nb.sf[mu];
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[k] = acc[k] + sf * o[k];
    load_site<P, 3, AT>(in, in_norm, Vh, nb.hb[mu], v);
    load_link<P, RECON, AT>(a.U_there, mu, Vh, nb.hb[mu], u);
    su3_mv<AT, true>(u, v, o);
    const AT sb = -eta * (AT)nb.sb[mu];
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[k] = acc[k] + sb * o[k];
  }
  }
}

template <int P, int RECON>
__device__ __forceinline__ void staggered_hop_body(const HopArgs& a) {
  using AT = typename AccT<P>::T;
  // right-hand sides are interleaved in blockIdx.x so that the CTAs of all rhs
  // for the same sites run back to back and share the links through L2
  const int rhs = (int)(blockIdx.x % (unsigned)a.nrhs);
  const int64_t h = (int64_t)(blockIdx.x / (unsigned)a.nrhs) * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait();
  if (h >= a.g.Vh) return;
  if (a.skip_dev && a.skip_dev[(int64_t)rhs * a.skip_stride]) return;
  cpx<AT> acc[3];
  staggered_hop_site<P, RECON>(a, rhs, h, acc);
  staggered_finish_store<P>(a, rhs, h, acc);
}

// The staggered hop of one right-hand side with its xpay source x and a fused
// reduction: out = a H in + xa x is stored, and the last block hands
// Re sum_h <x(h), out(h)> (FP64 over the grid, out as stored: FP64 / FP32) to
// E::finalize(0, tot) / E::finalize_warp on the device.  The second hop of the
// Schur operator (2am)^2 p - H_eo H_oe p then yields (p, A p) of a CG
// iteration without a separate pass over p and A p.  Every thread reaches the
// reduction; a skipped right-hand side (skip_dev) contributes zero, and E's
// finalize still runs.
template <int P, int RECON, int MINB, class E>
__global__ void __launch_bounds__(256, MINB) staggered_hop_xdot_kernel(HopArgs a, E e, double* partials,
                                                                      unsigned* counter) {
  static_assert(P != P16, "the FP16 result is rounded when stored: reduce it from memory");
  using AT = typename AccT<P>::T;
  const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait();
  double red[1] = {0.0};
  if (!(a.skip_dev && a.skip_dev[0]) && h < a.g.Vh) {
    cpx<AT> acc[3], xv[3];
    staggered_hop_site<P, RECON>(a, 0, h, acc);
    load_site<P, 3, AT>(reinterpret_cast<const char*>(a.x), nullptr, a.g.Vh, h, xv);
    const cpx<AT> ca = mk<AT>((AT)a.a.x, (AT)a.a.y), cx = mk<AT>((AT)a.xa.x, (AT)a.xa.y);
    AT re = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      acc[k] = ca * acc[k] + cx * xv[k];
      re += xv[k].x * acc[k].x + xv[k].y * acc[k].y;
    }
    store_site<P, 3, AT>(reinterpret_cast<char*>(a.out), nullptr, a.g.Vh, h, acc);
    red[0] = (double)re;
  }
  grid_reduce_finalize<1>(red, e, 0, blockIdx.x, gridDim.x, 1, partials, counter);
}

// __launch_bounds__(256): the FP64 kernel takes 90 registers (22 warps per
// SM); the capped form (256, 3) holds it to 80 (24 warps).  The autotuner
// picks per operator and lattice.
template <int P, int RECON>
__global__ void __launch_bounds__(256) staggered_hop_kernel(HopArgs a) {
  staggered_hop_body<P, RECON>(a);
}
template <int P, int RECON>
__global__ void __launch_bounds__(256, 3) staggered_hop_kernel_capped(HopArgs a) {
  staggered_hop_body<P, RECON>(a);
}

// The tile form of the FP64 / FP32 staggered hop for several right-hand sides
// (the batched per-shift refinement of a multi-shift solve): the block stages
// the 8 links of its 32 sites once (TileN, complete as load_link gives them)
// with the neighbour indices and the signs eta_mu(x) x boundary (forward) and
// -eta_mu(x) x boundary (backward), then its warps loop over the right-hand
// sides.  A staggered link is 8 times the bytes of the colour vector it acts
// on, so staging it once per tile saves most of the traffic of a one-rhs
// launch per rhs.  Per site and rhs the arithmetic of staggered_hop_body.
template <int P, int RECON, int MINB>
__global__ void __launch_bounds__(256, MINB) staggered_tile_kernel(HopArgs a) {
  using AT = typename AccT<P>::T;
  __shared__ TileN<AT> t;
  const int64_t h0 = tile16_index(a) * TILE16;
  pdl_launch_dependents();
  for (int i = threadIdx.x; i < TILE16; i += blockDim.x) {
    const int64_t h = h0 + i;
    uint32_t neg = 0;
    if (h < a.g.Vh) {
      NbrInfo nb;
      int c[4];
      neighbours(a.g, a.out_parity, h, nb, c);
#pragma unroll
      for (int mu = 0; mu < 4; ++mu) {
        int es = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (k < mu) es += c[k];
        const float eta = (es & 1) ? -1.f : 1.f;
        t.nb[mu][i] = nb.hf[mu];
        t.nb[4 + mu][i] = nb.hb[mu];
        neg |= (eta * nb.sf[mu] < 0.f ? 1u : 0u) << mu;
        neg |= (-eta * nb.sb[mu] < 0.f ? 1u : 0u) << (4 + mu);
      }
    } else {
#pragma unroll
      for (int d = 0; d < 8; ++d) t.nb[d][i] = 0;
    }
    t.neg[i] = neg;
  }
  pdl_wait();
  if (!tile_any_live(a, 0, a.nrhs)) return;  // no barrier has been passed yet: uniform
  __syncthreads();
  tileN_links<P, RECON>(a.U_here, a.U_there, a.g.Vh, h0, t);
  __syncthreads();
  const int i = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int64_t h = h0 + i;
  if (h >= a.g.Vh) return;  // no barrier follows
  const int64_t Vh = a.g.Vh;
  const uint32_t neg = t.neg[i];
  for (int rhs = threadIdx.x >> 5; rhs < a.nrhs; rhs += nw) {
    if (a.skip_dev && a.skip_dev[(int64_t)rhs * a.skip_stride]) continue;
    const char* in = reinterpret_cast<const char*>(a.in) + rhs * a.in_stride;
    const float* in_norm = a.in_norm ? a.in_norm + rhs * a.in_nstride : nullptr;
    cpx<AT> acc[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[k] = mk<AT>(0, 0);
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
      cpx<AT> v[3], u[9], o[3];
      load_site<P, 3, AT>(in, in_norm, Vh, t.nb[mu][i], v);
#pragma unroll
      for (int w = 0; w < 9; ++w) u[w] = t.u[mu][w][i];
      su3_mv<AT, false>(u, v, o);
      const AT sf = (neg >> mu) & 1u ? (AT)-1 : (AT)1;
#pragma unroll
      for (int k = 0; k < 3; ++k) acc[k] = acc[k] + sf * o[k];
      load_site<P, 3, AT>(in, in_norm, Vh, t.nb[4 + mu][i], v);
#pragma unroll
      for (int w = 0; w < 9; ++w) u[w] = t.u[4 + mu][w][i];
      su3_mv<AT, true>(u, v, o);
      const AT sb = (neg >> (4 + mu)) & 1u ? (AT)-1 : (AT)1;
#pragma unroll
      for (int k = 0; k < 3; ++k) acc[k] = acc[k] + sb * o[k];
    }
    staggered_finish_store<P>(a, rhs, h, acc);
  }
}

}  // namespace clg
