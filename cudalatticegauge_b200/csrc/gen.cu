// gen.cu -- seeded field generation on the device, CLGBin / Bridge++ import and
// export (reordering into the even-odd structure-of-arrays layout), the
// plaquette and the unitarity check of the gauge field.
//
// Generator (published methods):
//   Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), key = {seed_lo, seed_hi ^ field_id},
//   counter = {index_lo, index_hi, sub, tag}; Box-Muller Gaussians from two 53-bit
//   uniforms; Haar SU(3) by Gram-Schmidt QR of a complex Gaussian matrix (Mezzadri,
//   Notices AMS 54, 2007) with det fixed to 1; exp(i eps H) by a scaled Taylor series
//   and squaring, re-unitarised.  Field indices follow the reference's site order so a
//   field generated here equals the same field generated on the host.
#include <cstring>

#include "blas.cuh"

namespace clg {

namespace {

constexpr uint32_t TAG_GAUGE = 0x47415547u, TAG_SPINOR = 0x5350494eu, TAG_Z2 = 0x5a324e53u, TAG_Z4 = 0x5a344e53u;

__device__ __forceinline__ void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
  const uint64_t x = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);
  return ((double)x + 0.5) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ void gauss2(uint64_t seed, uint32_t fid, uint64_t index, uint32_t sub, uint32_t tag,
                                       double& g1, double& g2) {
  uint32_t c[4] = {(uint32_t)index, (uint32_t)(index >> 32), sub, tag};
  philox(c, (uint32_t)seed, (uint32_t)(seed >> 32) ^ fid);
  const double v1 = u53(c[0], c[1]), v2 = u53(c[2], c[3]);
  const double r = sqrt(-2.0 * log(v1));
  double sn, cs;
  sincospi(2.0 * v2, &sn, &cs);
  g1 = r * cs;
  g2 = r * sn;
}

using C = cpx<double>;

__device__ void haar(uint64_t seed, uint32_t fid, uint64_t link, C z[9]) {
  const double isq2 = 0.70710678118654752440084436210485;
  for (int k = 0; k < 9; ++k) {
    double a, b;
    gauss2(seed, fid, link, (uint32_t)k, TAG_GAUGE, a, b);
    z[k] = mk<double>(a * isq2, b * isq2);
  }
  for (int c = 0; c < 3; ++c) {
    for (int p = 0; p < c; ++p) {
      C d = mk<double>(0, 0);
      for (int r = 0; r < 3; ++r) d = d + cjmul(z[3 * r + p], z[3 * r + c]);
      for (int r = 0; r < 3; ++r) z[3 * r + c] = z[3 * r + c] - d * z[3 * r + p];
    }
    double nn = 0;
    for (int r = 0; r < 3; ++r) nn += z[3 * r + c].x * z[3 * r + c].x + z[3 * r + c].y * z[3 * r + c].y;
    const double inv = 1.0 / sqrt(nn);
    for (int r = 0; r < 3; ++r) z[3 * r + c] = inv * z[3 * r + c];
  }
  const C det = z[0] * (z[4] * z[8] - z[5] * z[7]) - z[1] * (z[3] * z[8] - z[5] * z[6]) + z[2] * (z[3] * z[7] - z[4] * z[6]);
  const C f = cj(det);
  for (int r = 0; r < 3; ++r) z[3 * r + 2] = z[3 * r + 2] * f;
}

__device__ void reunitarise(C m[9]) {
  double n0 = 0;
  for (int k = 0; k < 3; ++k) n0 += m[k].x * m[k].x + m[k].y * m[k].y;
  n0 = 1.0 / sqrt(n0);
  for (int k = 0; k < 3; ++k) m[k] = n0 * m[k];
  C d = mk<double>(0, 0);
  for (int k = 0; k < 3; ++k) d = d + cjmul(m[k], m[3 + k]);
  for (int k = 0; k < 3; ++k) m[3 + k] = m[3 + k] - d * m[k];
  double n1 = 0;
  for (int k = 0; k < 3; ++k) n1 += m[3 + k].x * m[3 + k].x + m[3 + k].y * m[3 + k].y;
  n1 = 1.0 / sqrt(n1);
  for (int k = 0; k < 3; ++k) m[3 + k] = n1 * m[3 + k];
  reconstruct_row2(m);
}

__device__ void expH(uint64_t seed, uint32_t fid, uint64_t link, double eps, C E[9]) {
  double h[8];
  for (int k = 0; k < 4; ++k) gauss2(seed, fid, link, (uint32_t)k, TAG_GAUGE, h[2 * k], h[2 * k + 1]);
  const double is3 = 0.57735026918962576450914878050196;
  C H[9];
  H[0] = mk<double>(0.5 * (h[2] + h[7] * is3), 0);
  H[4] = mk<double>(0.5 * (-h[2] + h[7] * is3), 0);
  H[8] = mk<double>(0.5 * (-2.0 * h[7] * is3), 0);
  H[1] = mk<double>(0.5 * h[0], -0.5 * h[1]);
  H[3] = cj(H[1]);
  H[2] = mk<double>(0.5 * h[3], -0.5 * h[4]);
  H[6] = cj(H[2]);
  H[5] = mk<double>(0.5 * h[5], -0.5 * h[6]);
  H[7] = cj(H[5]);
  C A[9];
  double fn = 0;
  for (int k = 0; k < 9; ++k) {
    A[k] = mk<double>(-eps * H[k].y, eps * H[k].x);  // i eps H
    fn += A[k].x * A[k].x + A[k].y * A[k].y;
  }
  fn = sqrt(fn);
  int s = 0;
  while (fn > 0.25) {
    fn *= 0.5;
    ++s;
  }
  const double scale = ldexp(1.0, -s);
  for (int k = 0; k < 9; ++k) A[k] = scale * A[k];
  for (int k = 0; k < 9; ++k) E[k] = mk<double>((k % 4 == 0) ? 1.0 : 0.0, 0);
  for (int n = 18; n >= 1; --n) {
    C P[9];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) P[3 * r + c] = A[3 * r] * E[c] + A[3 * r + 1] * E[3 + c] + A[3 * r + 2] * E[6 + c];
    const double inv = 1.0 / (double)n;
    for (int k = 0; k < 9; ++k) E[k] = mk<double>(((k % 4 == 0) ? 1.0 : 0.0) + P[k].x * inv, P[k].y * inv);
  }
  for (int q = 0; q < s; ++q) {
    C T[9];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) T[3 * r + c] = E[3 * r] * E[c] + E[3 * r + 1] * E[3 + c] + E[3 * r + 2] * E[6 + c];
    for (int k = 0; k < 9; ++k) E[k] = T[k];
  }
  reunitarise(E);
}

struct SiteIdx {
  int c[4];
  int64_t s;
  int p;
  int64_t h;
};
__device__ __forceinline__ SiteIdx site_from_linear(const Geom& g, int64_t s) {
  // V < 2^31: 32-bit multiply-high divisions by the extents
  SiteIdx r;
  unsigned t = (unsigned)s;
  unsigned q = g.dL[3].div(t);
  r.c[3] = (int)(t - q * (unsigned)g.L[3]);
  t = q;
  q = g.dL[2].div(t);
  r.c[2] = (int)(t - q * (unsigned)g.L[2]);
  t = q;
  q = g.dL[1].div(t);
  r.c[1] = (int)(t - q * (unsigned)g.L[1]);
  r.c[0] = (int)q;
  r.s = s;
  r.p = (r.c[0] + r.c[1] + r.c[2] + r.c[3]) & 1;
  r.h = s >> 1;
  return r;
}

__device__ __forceinline__ void store_link64(double2* const* u, int p, int mu, int64_t Vh, int64_t h, const C m[9]) {
  double2* b = u[p] + (int64_t)mu * 9 * Vh + h;
  for (int k = 0; k < 9; ++k) b[k * Vh] = make_double2(m[k].x, m[k].y);
}
__device__ __forceinline__ void load_link64(double2* const* u, int p, int mu, int64_t Vh, int64_t h, C m[9]) {
  const double2* b = u[p] + (int64_t)mu * 9 * Vh + h;
  for (int k = 0; k < 9; ++k) {
    const double2 d = b[k * Vh];
    m[k] = mk<double>(d.x, d.y);
  }
}

struct LinkPtrs {
  double2* u[2];
};

__global__ void gauge_gen_kernel(Geom g, LinkPtrs L, int init, uint64_t seed, uint32_t fid, double eps) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= 4 * g.V) return;
  const int64_t s = l >> 2;
  const int mu = (int)(l & 3);
  const SiteIdx si = site_from_linear(g, s);
  C m[9];
  if (init == CLG_GAUGE_HAAR)
    haar(seed, fid, (uint64_t)l, m);
  else if (init == CLG_GAUGE_EXPH)
    expH(seed, fid, (uint64_t)l, eps, m);
  else if (init == CLG_GAUGE_ZERO)
    for (int k = 0; k < 9; ++k) m[k] = mk<double>(0, 0);
  else
    for (int k = 0; k < 9; ++k) m[k] = mk<double>((k % 4 == 0) ? 1.0 : 0.0, 0);
  store_link64(L.u, si.p, mu, g.Vh, si.h, m);
}

// CLGBin (link = s*4+mu) or Bridge++ (site x-fastest) <-> even-odd SoA
__global__ void gauge_reorder_kernel(Geom g, LinkPtrs L, double* buf, int layout, int to_device) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= 4 * g.V) return;
  const int64_t s = l >> 2;
  const int mu = (int)(l & 3);
  const SiteIdx si = site_from_linear(g, s);
  int64_t src = l;
  if (layout == CLG_LAYOUT_BRIDGEPP) {
    const int64_t bs = si.c[0] + (int64_t)si.c[1] * g.L[0] + (int64_t)si.c[2] * g.L[0] * g.L[1] +
                       (int64_t)si.c[3] * g.L[0] * g.L[1] * g.L[2];
    src = bs * 4 + mu;
  }
  double* b = buf + 18 * src;
  C m[9];
  if (to_device) {
    for (int k = 0; k < 9; ++k) m[k] = mk<double>(b[2 * k], b[2 * k + 1]);
    store_link64(L.u, si.p, mu, g.Vh, si.h, m);
  } else {
    load_link64(L.u, si.p, mu, g.Vh, si.h, m);
    for (int k = 0; k < 9; ++k) {
      b[2 * k] = m[k].x;
      b[2 * k + 1] = m[k].y;
    }
  }
}

// full-lattice CLGBin field data (nc complex per site) <-> one rhs of a field
template <int P, int NC>
__global__ void field_reorder_kernel(Geom g, DField f, int nparity, int rhs, double* buf, int to_device) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const SiteIdx si = site_from_linear(g, s);
  double* b = buf + 2 * NC * s;
  const bool held = nparity == 2 || si.p == f.first_parity;
  C v[NC];
  if (to_device) {
    if (!held) return;
    for (int k = 0; k < NC; ++k) v[k] = mk<double>(b[2 * k], b[2 * k + 1]);
    store_site<P, NC, double>(f.base(rhs, si.p), f.nbase(rhs, si.p), f.Vh, si.h, v);
  } else {
    if (held)
      load_site<P, NC, double>(f.base(rhs, si.p), f.nbase(rhs, si.p), f.Vh, si.h, v);
    else
      for (int k = 0; k < NC; ++k) v[k] = mk<double>(0, 0);
    for (int k = 0; k < NC; ++k) {
      b[2 * k] = v[k].x;
      b[2 * k + 1] = v[k].y;
    }
  }
}

// The same reorder with the FP64 lexicographic data in mapped pinned host
// memory, read or written by the SMs over the host link (zero copy).  It runs
// on the copy stream beside a solve, so it is built not to disturb one:
//   - a block moves tiles of XS sites; the host side as consecutive 16-byte
//     chunks (whole, contiguous link requests, all a thread's loads issued
//     before the first is used), the device side one site per thread through
//     a shared tile padded to NC + 1 chunks per site (conflict-free);
//   - every access is a streaming one (ld/st .cs, evict-first in L2), so the
//     transfer's bytes do not displace the solve's L2 working set;
//   - a small grid-stride grid: a few blocks keep the link busy, and the SMs
//     stay with the solve.
// Used for FP64 fields only (the transfer format); others take the staging path.
template <int NC>
__global__ void __launch_bounds__(256) field_stream_kernel(Geom g, DField f, int nparity, int rhs, double2* host,
                                                           int to_device) {
  constexpr int XS = 128, ROW = NC + 1, CH = XS * NC, PER = (CH + 255) / 256;
  __shared__ double2 tile[XS * ROW];
  const int64_t ntiles = (g.V + XS - 1) / XS;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t s0 = t * XS;
    const int ns = (int)min((int64_t)XS, g.V - s0);
    double2* hb = host + s0 * NC;
    const int j = threadIdx.x;
    SiteIdx si;
    bool held = false;
    if (j < ns) {
      si = site_from_linear(g, s0 + j);
      held = nparity == 2 || si.p == f.first_parity;
    }
    if (to_device) {
      double2 r[PER];
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        const int i = j + q * 256;
        if (i < ns * NC) r[q] = __ldcs(hb + i);
      }
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        const int i = j + q * 256;
        if (i < ns * NC) tile[i + i / NC] = r[q];
      }
      __syncthreads();
      if (held) {
        double2* b = reinterpret_cast<double2*>(f.base(rhs, si.p));
#pragma unroll
        for (int k = 0; k < NC; ++k) __stcs(b + k * f.Vh + si.h, tile[j * ROW + k]);
      }
    } else {
      if (j < ns) {
        const double2* b = reinterpret_cast<const double2*>(f.base(rhs, held ? si.p : f.first_parity));
#pragma unroll
        for (int k = 0; k < NC; ++k) tile[j * ROW + k] = held ? __ldcs(b + k * f.Vh + si.h) : make_double2(0.0, 0.0);
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        const int i = j + q * 256;
        if (i < ns * NC) __stcs(hb + i, tile[i + i / NC]);
      }
    }
    __syncthreads();  // the tile is refilled by the next iteration
  }
}

template <int P, int NC>
struct SourceF {
  DField f;
  Geom g;
  int rhs0;
  int kind;
  uint64_t seed;
  uint32_t fid;
  int64_t site;
  int comp;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int r, int p, int64_t h, double*) const {
    // full-lattice index of checkerboard site (p, h)
    int c[4];
    eo_coords(g, p, h, c);
    const int64_t s = site_index(g, c);
    C v[NC];
    const double isq2 = 0.70710678118654752440084436210485;
    if (kind == CLG_SOURCE_GAUSS) {
      for (int k = 0; k < NC; ++k) {
        double a, b;
        gauss2(seed, fid, (uint64_t)s, (uint32_t)k, TAG_SPINOR, a, b);
        v[k] = mk<double>(a * isq2, b * isq2);
      }
    } else if (kind == CLG_SOURCE_Z2) {
      uint32_t w[4] = {(uint32_t)s, (uint32_t)((uint64_t)s >> 32), 0u, TAG_Z2};
      philox(w, (uint32_t)seed, (uint32_t)(seed >> 32) ^ fid);
      for (int k = 0; k < NC; ++k) {
        const int b0 = 2 * k, b1 = 2 * k + 1;
        const uint32_t x0 = w[b0 >> 5] >> (b0 & 31), x1 = w[b1 >> 5] >> (b1 & 31);
        v[k] = mk<double>((x0 & 1u) ? -isq2 : isq2, (x1 & 1u) ? -isq2 : isq2);
      }
    } else if (kind == CLG_SOURCE_Z4) {
      // i^b, b = bits 2k, 2k+1 of one Philox output
      uint32_t w[4] = {(uint32_t)s, (uint32_t)((uint64_t)s >> 32), 0u, TAG_Z4};
      philox(w, (uint32_t)seed, (uint32_t)(seed >> 32) ^ fid);
      for (int k = 0; k < NC; ++k) {
        const uint32_t b = (w[(2 * k) >> 5] >> ((2 * k) & 31)) & 3u;
        v[k] = mk<double>(b == 0 ? 1.0 : (b == 2 ? -1.0 : 0.0), b == 1 ? 1.0 : (b == 3 ? -1.0 : 0.0));
      }
    } else {
      for (int k = 0; k < NC; ++k) v[k] = mk<double>((kind == CLG_SOURCE_POINT && s == site && k == comp) ? 1.0 : 0.0, 0);
    }
    store_site<P, NC, double>(f.base(rhs0 + r, p), f.nbase(rhs0 + r, p), f.Vh, h, v);
  }
  __device__ void finalize(int, const double*) const {}
};

struct PlaqF {
  Geom g;
  LinkPtrs L;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int, int p, int64_t h, double* acc) const {
    int c[4];
    eo_coords(g, p, h, c);
    double tot = 0;
    for (int mu = 0; mu < 4; ++mu)
      for (int nu = mu + 1; nu < 4; ++nu) {
        int a[4] = {c[0], c[1], c[2], c[3]}, b[4] = {c[0], c[1], c[2], c[3]};
        a[mu] = (a[mu] + 1) % g.L[mu];
        b[nu] = (b[nu] + 1) % g.L[nu];
        const int pa = (a[0] + a[1] + a[2] + a[3]) & 1, pb = (b[0] + b[1] + b[2] + b[3]) & 1;
        C u1[9], u2[9], u3[9], u4[9], P[9], Q[9];
        load_link64(L.u, p, mu, g.Vh, h, u1);
        load_link64(L.u, pa, nu, g.Vh, site_index(g, a) >> 1, u2);
        load_link64(L.u, pb, mu, g.Vh, site_index(g, b) >> 1, u3);
        load_link64(L.u, p, nu, g.Vh, h, u4);
        for (int r = 0; r < 3; ++r)
          for (int cc = 0; cc < 3; ++cc) {
            P[3 * r + cc] = u1[3 * r] * u2[cc] + u1[3 * r + 1] * u2[3 + cc] + u1[3 * r + 2] * u2[6 + cc];
            Q[3 * r + cc] = u4[3 * r] * u3[cc] + u4[3 * r + 1] * u3[3 + cc] + u4[3 * r + 2] * u3[6 + cc];
          }
        for (int k = 0; k < 9; ++k) tot += P[k].x * Q[k].x + P[k].y * Q[k].y;
      }
    acc[0] += tot / 3.0;
  }
  __device__ void finalize(int, const double* s) const {}
};

struct PlaqOut {
  PlaqF f;
  double* out;
  __device__ bool active(int r) const { return f.active(r); }
  __device__ void operator()(int r, int p, int64_t h, double* acc) const { f(r, p, h, acc); }
  __device__ void finalize(int, const double* s) const { out[0] = s[0]; }
};

__global__ void unitarity_kernel(Geom g, LinkPtrs L, unsigned long long* worst) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double w = 0;
  if (l < 4 * g.V) {
    const int64_t s = l >> 2;
    const int mu = (int)(l & 3);
    const int64_t t = s;
    int c[4];
    int64_t q = t;
    c[3] = (int)(q % g.L[3]); q /= g.L[3];
    c[2] = (int)(q % g.L[2]); q /= g.L[2];
    c[1] = (int)(q % g.L[1]); c[0] = (int)(q / g.L[1]);
    const int p = (c[0] + c[1] + c[2] + c[3]) & 1;
    C m[9];
    load_link64(L.u, p, mu, g.Vh, s >> 1, m);
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 3; ++cc) {
        C d = mk<double>(0, 0);
        for (int k = 0; k < 3; ++k) d = d + m[3 * r + k] * cj(m[3 * cc + k]);
        const double e = hypot(d.x - (r == cc ? 1.0 : 0.0), d.y);
        w = fmax(w, e);
      }
    const C det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
    w = fmax(w, hypot(det.x - 1.0, det.y));
    if (!(w == w)) w = 1e300;  // NaN counts as not unitary
  }
  for (int o = 16; o > 0; o >>= 1) w = fmax(w, __shfl_down_sync(0xffffffffu, w, o));
  if ((threadIdx.x & 31) == 0) atomicMax(worst, (unsigned long long)__double_as_longlong(w));
}

}  // namespace

// ---------------------------------------------------------------- host entry points
clg_status gauge_generate(clg_gauge_s* U, int init, uint64_t seed, uint32_t fid, double eps) {
  clg_context_s* ctx = U->lat->ctx;
  const Geom& g = U->lat->g;
  LinkPtrs L{{(double2*)U->u64[0], (double2*)U->u64[1]}};
  const int64_t n = 4 * g.V;
  gauge_gen_kernel<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(g, L, init, seed, fid, eps);
  ctx->kernels++;
  CLG_CUDA_OK(cudaGetLastError());
  U->dirty_lowp = true;
  return CLG_SUCCESS;
}

clg_status gauge_reorder(clg_gauge_s* U, double* dev_buf, int layout, int to_device) {
  clg_context_s* ctx = U->lat->ctx;
  const Geom& g = U->lat->g;
  LinkPtrs L{{(double2*)U->u64[0], (double2*)U->u64[1]}};
  const int64_t n = 4 * g.V;
  gauge_reorder_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(g, L, dev_buf, layout, to_device);
  ctx->kernels++;
  CLG_CUDA_OK(cudaGetLastError());
  if (to_device) U->dirty_lowp = true;
  return CLG_SUCCESS;
}

clg_status field_reorder(clg_field_s* f, int rhs, double* dev_buf, int to_device) {
  clg_context_s* ctx = f->lat->ctx;
  const Geom& g = f->lat->g;
  const FieldRef r = f->ref();
  return with_pn(f->prec, f->nc(), [&](auto P, auto NC) -> clg_status {
    field_reorder_kernel<P.value, NC.value>
        <<<(unsigned)((g.V + 255) / 256), 256, 0, ctx->stream>>>(g, dfield(r), r.nparity, rhs, dev_buf, to_device);
    ctx->kernels++;
    CLG_CUDA_OK(cudaGetLastError());
    return CLG_SUCCESS;
  });
}

clg_status field_stream(clg_field_s* f, int rhs, double* host_dev, int to_device, cudaStream_t s) {
  clg_context_s* ctx = f->lat->ctx;
  const Geom& g = f->lat->g;
  if (f->prec != CLG_PREC_DOUBLE) return CLG_ERR_BAD_ARG;
  const FieldRef r = f->ref();
  const int64_t tiles = (g.V + 127) / 128;
  const unsigned grid = (unsigned)std::min<int64_t>(tiles, ctx->xfer_blocks);
  double2* h = reinterpret_cast<double2*>(host_dev);
  if (f->nc() == 12)
    field_stream_kernel<12><<<grid, 256, 0, s>>>(g, dfield(r), r.nparity, rhs, h, to_device);
  else
    field_stream_kernel<3><<<grid, 256, 0, s>>>(g, dfield(r), r.nparity, rhs, h, to_device);
  ctx->kernels++;
  CLG_CUDA_OK(cudaGetLastError());
  return CLG_SUCCESS;
}

clg_status field_source(clg_field_s* f, int rhs, int kind, uint64_t seed, uint32_t fid, int64_t site, int comp) {
  clg_context_s* ctx = f->lat->ctx;
  const FieldRef r = f->ref();
  return with_pn(f->prec, f->nc(), [&](auto P, auto NC) {
    SourceF<P.value, NC.value> fn{dfield(r), f->lat->g, rhs, kind, seed, fid, site, comp};
    return launch_sites<0>(ctx, fn, r.first_parity, r.nparity, r.Vh, 1);
  });
}

clg_status gauge_plaquette(clg_gauge_s* U, double* host_out) {
  clg_context_s* ctx = U->lat->ctx;
  const Geom& g = U->lat->g;
  double* d = nullptr;
  clg_status st = dalloc(ctx, (void**)&d, sizeof(double));
  if (st) return st;
  PlaqOut fn{PlaqF{g, LinkPtrs{{(double2*)U->u64[0], (double2*)U->u64[1]}}}, d};
  st = launch_sites<1>(ctx, fn, 0, 2, g.Vh, 1);
  if (!st) {
    cudaError_t e = cudaMemcpyAsync(host_out, d, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) st = ctx->fail(cuda_status(e), cudaGetErrorString(e));
    *host_out /= (6.0 * (double)g.V);
  }
  dfree(d);
  return st;
}

clg_status gauge_unitarity(clg_gauge_s* U, double* host_out) {
  clg_context_s* ctx = U->lat->ctx;
  const Geom& g = U->lat->g;
  unsigned long long* d = nullptr;
  clg_status st = dalloc(ctx, (void**)&d, sizeof(unsigned long long));
  if (st) return st;
  cudaError_t e = cudaMemsetAsync(d, 0, sizeof(unsigned long long), ctx->stream);
  const int64_t n = 4 * g.V;
  if (e == cudaSuccess) {
    unitarity_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(
        g, LinkPtrs{{(double2*)U->u64[0], (double2*)U->u64[1]}}, d);
    ctx->kernels++;
    e = cudaGetLastError();
  }
  unsigned long long bits = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, d, sizeof(bits), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  dfree(d);
  if (e != cudaSuccess) return ctx->fail(cuda_status(e), cudaGetErrorString(e));
  double w;
  memcpy(&w, &bits, sizeof(w));
  *host_out = w;
  return CLG_SUCCESS;
}

}  // namespace clg
