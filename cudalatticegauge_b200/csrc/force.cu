// force.cu -- the Wilson fermion force on the gauge links (the HMC
// pseudofermion force), FP64, and the whole force step of
// CFieldFermionWilsonSquareSU3::CalculateForceS
// (Data/Field/WilsonDirac/CFieldFermionWilsonSquareSU3.cu:1016-1100).
//
// With X = (D D^+)^-1 phi and Y = D^+ X, _kernelDWilsonForceSU3 (same file,
// :170-231) adds to every link
//   F_mu(x) += s_+ kappa Ta(U_mu(x) mid),
//   mid = sum_s [(1 - g_mu) Y(x+mu)]_s X(x)_s^+  +  X(x+mu)_s [(1 + g_mu) Y(x)]_s^+
// (colour outer products summed over spin, makeSU3Contract, SU3.h:395-500;
// Ta the traceless anti-hermitian part, SU3.h:953-980; s_+ the fermion
// boundary sign of the hop x -> x+mu).
//
// In the chiral basis (1 -+ g_mu) has rank 2: rows 2, 3 of a projected spinor
// are phases times rows 0, 1, and the same phases pair the rows of the other
// factor, so each spin sum collapses onto the two upper rows of BOTH factors
// projected with the same sign:
//   mid = sum_{j<2} [(1-g)Y(x+mu)]_j [(1-g)X(x)]_j^+ + [(1+g)X(x+mu)]_j [(1+g)Y(x)]_j^+
// -- 36 complex multiply-adds instead of 72.
//
// Layout and traffic.  A block of 128 threads is four warps over the same 32
// checkerboard sites, warp w taking direction mu = w (warp-uniform, so the
// gamma structure is compile-time and nothing diverges).  Blocks alternate
// parity (blockIdx.x = 2 * site block + parity) so both checkerboards of a
// field region are read while the region is in L2.  Compulsory DRAM traffic
// per site: X and Y (2 x 192 B per right-hand side), U (4 x 144 B), F read and
// written (4 x 288 B) = 2112 B for one right-hand side.  Several right-hand
// sides (pseudofermions) are summed into mid before the one F update.
#include "clg_common.cuh"
#include "dslash.cuh"
#include "internal.h"

namespace clg {

namespace {

using C = cpx<double>;

struct ForceArgs {
  Geom g;
  const double2* U[2];  // per parity, [mu][9][Vh]
  double2* F[2];
  const char* X;        // rhs 0, parity 0 ([rhs][parity][12][Vh] double2)
  const char* Y;
  int64_t blk;          // bytes of one parity block
  int64_t rstride;      // bytes between right-hand sides
  int nrhs;
  double kappa;
};

// ------------------------------------------------------------------ shared-memory staging
// One block = TILE checkerboard sites of one parity x 4 directions.  Every
// operand of the block (spinors here and at the four forward neighbours, the
// links and the force links) is requested at the start with 16-byte cp.async
// copies into shared memory -- 96 KB in flight per block, two blocks per SM,
// instead of the few hundred bytes a thread can hold in registers -- then
// computed from there.  On 32^3 x 16 this took the kernel from 0.51 to 0.82 of
// the measured copy bandwidth (331 -> 207 us; staging all but F: 440 us; a
// persistent form with one block per SM double-buffering its tiles: 217 us).
constexpr int TILE = 32;
constexpr int E_HERE = 2 * 12 * TILE;    // X(x), Y(x)           [field][k][site]
constexpr int E_NBR = 4 * 2 * 12 * TILE; // X(x+mu), Y(x+mu)     [mu][field][k][site]
constexpr int E_LINK = 4 * 9 * TILE;     // U_mu(x) or F_mu(x)   [mu][k][site]
constexpr size_t FORCE_SMEM = sizeof(double2) * (E_HERE + E_NBR + 2 * E_LINK);  // 96 KB

__device__ __forceinline__ void cp_async16(double2* smem, const double2* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// the two upper rows of (1 + SGN g_mu) v, v = 12 complex at stride TILE in shared memory
template <int MU, int SGN>
__device__ __forceinline__ void proj_smem(const double2* v0, C out[6]) {
  C v[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    const double2 d = v0[k * TILE];
    v[k] = mk<double>(d.x, d.y);
  }
  constexpr int add = SGN < 0 ? 2 : 0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    out[c] = v[c] + mul_i(v[3 * gperm(MU, 0) + c], gz4(MU, 0) + add);
    out[3 + c] = v[3 + c] + mul_i(v[3 * gperm(MU, 1) + c], gz4(MU, 1) + add);
  }
}

// mid[a][b] += sum_j l_j[a] conj(r_j[b])
__device__ __forceinline__ void outer_acc(C mid[9], const C l[6], const C r[6]) {
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      C m = mid[3 * a + b];
      m.x = fma(l[a].x, r[b].x, fma(l[a].y, r[b].y, m.x));
      m.y = fma(l[a].y, r[b].x, fma(-l[a].x, r[b].y, m.y));
      m.x = fma(l[3 + a].x, r[3 + b].x, fma(l[3 + a].y, r[3 + b].y, m.x));
      m.y = fma(l[3 + a].y, r[3 + b].x, fma(-l[3 + a].x, r[3 + b].y, m.y));
      mid[3 * a + b] = m;
    }
}

// forward neighbour (checkerboard index) of site h of parity p in direction mu
// and the fermion boundary sign of that hop
__device__ __forceinline__ int64_t forward_nbr(const Geom& g, int p, int64_t h, int mu, double& sg) {
  int c[4];
  eo_coords(g, p, h, c);
  const int64_t s = site_index(g, c);
  // mu is a run-time value: select its extent, coordinate and sign with
  // static indices (no local-memory array)
  int cm = 0, lm = 1, bm = 1;
  int64_t st = 1;
#pragma unroll
  for (int k = 3; k >= 0; --k) {
    if (k == mu) {
      cm = c[k];
      lm = g.L[k];
      bm = g.bc[k];
    }
    if (k > mu) st *= g.L[k];
  }
  int64_t sf = s + st;
  sg = 1.0;
  if (cm == lm - 1) {
    sf -= (int64_t)lm * st;
    sg = (double)bm;
  }
  return sf >> 1;
}

template <int MU>
__device__ __forceinline__ void force_compute(const ForceArgs& a, const double2* sm, int p, int lane, int64_t h,
                                              double sg, const C mid_in[9]) {
  const int64_t Vh = a.g.Vh;
  const double2* s_link = sm + E_HERE + E_NBR + MU * 9 * TILE + lane;
  // m = U_mu(x) mid
  C m[9];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    C u[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double2 d = s_link[(3 * i + k) * TILE];
      u[k] = mk<double>(d.x, d.y);
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) m[3 * i + j] = u[0] * mid_in[j] + u[1] * mid_in[3 + j] + u[2] * mid_in[6 + j];
  }
  // F += s_+ kappa Ta(m)
  const double w = sg * a.kappa;
  double2* fb = (p ? a.F[1] : a.F[0]) + (int64_t)MU * 9 * Vh + h;
  const double2* s_f = s_link + E_LINK;
  const double tr = (m[0].y + m[4].y + m[8].y) * (1.0 / 3.0);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      C t;
      if (i == j) {
        t = mk<double>(0.0, m[4 * i].y - tr);
      } else {
        // (m_ij - conj(m_ji)) / 2
        t = mk<double>(0.5 * (m[3 * i + j].x - m[3 * j + i].x), 0.5 * (m[3 * i + j].y + m[3 * j + i].y));
      }
      double2 f = s_f[(3 * i + j) * TILE];
      f.x = fma(w, t.x, f.x);
      f.y = fma(w, t.y, f.y);
      fb[(3 * i + j) * Vh] = f;
    }
}

template <int MU>
__device__ __forceinline__ void force_mid(const double2* sm, int lane, C mid[9]) {
  const double2* xh = sm + lane;
  const double2* yh = xh + 12 * TILE;
  const double2* xn = sm + E_HERE + MU * 24 * TILE + lane;
  const double2* yn = xn + 12 * TILE;
  C l[6], q[6];
  proj_smem<MU, -1>(yn, l);
  proj_smem<MU, -1>(xh, q);
  outer_acc(mid, l, q);
  proj_smem<MU, +1>(xn, l);
  proj_smem<MU, +1>(yh, q);
  outer_acc(mid, l, q);
}

// blockIdx.x = 2 * tile + parity; threadIdx.x = 32 * mu + lane
__global__ void __launch_bounds__(128) wilson_force_kernel(ForceArgs a) {
  extern __shared__ double2 sm[];
  const int p = (int)(blockIdx.x & 1);
  const int lane = (int)(threadIdx.x & 31), mu = (int)(threadIdx.x >> 5);
  const int64_t h = (int64_t)(blockIdx.x >> 1) * TILE + lane;
  const int64_t Vh = a.g.Vh;
  const bool live = h < Vh;
  double sg = 1.0;
  const int64_t hn = live ? forward_nbr(a.g, p, h, mu, sg) : 0;
  const int64_t here = (int64_t)p * a.blk, there = (int64_t)(1 - p) * a.blk;

  if (live) {
    const double2* ub = (p ? a.U[1] : a.U[0]) + (int64_t)mu * 9 * Vh + h;
    double2* su = sm + E_HERE + E_NBR + mu * 9 * TILE + lane;
#pragma unroll
    for (int k = 0; k < 9; ++k) cp_async16(su + k * TILE, ub + k * Vh);
    const double2* fb = (p ? a.F[1] : a.F[0]) + (int64_t)mu * 9 * Vh + h;
#pragma unroll
    for (int k = 0; k < 9; ++k) cp_async16(su + E_LINK + k * TILE, fb + k * Vh);
  }
  C mid[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) mid[k] = mk<double>(0, 0);
  for (int r = 0; r < a.nrhs; ++r) {
    if (live) {
      const int64_t ro = (int64_t)r * a.rstride;
      // here: the 24 complex of X(x), Y(x), six per warp
#pragma unroll
      for (int e = 0; e < 6; ++e) {
        const int f = mu * 6 + e;  // 0..23: X k = f, Y k = f - 12
        const double2* src = reinterpret_cast<const double2*>((f < 12 ? a.X : a.Y) + ro + here) + (f % 12) * Vh + h;
        cp_async16(sm + f * TILE + lane, src);
      }
      const double2* xs = reinterpret_cast<const double2*>(a.X + ro + there) + hn;
      const double2* ys = reinterpret_cast<const double2*>(a.Y + ro + there) + hn;
      double2* dn = sm + E_HERE + mu * 24 * TILE + lane;
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        cp_async16(dn + k * TILE, xs + k * Vh);
        cp_async16(dn + (12 + k) * TILE, ys + k * Vh);
      }
    }
    cp_async_wait_all();
    __syncthreads();
    if (live) {
      switch (mu) {
        case 0: force_mid<0>(sm, lane, mid); break;
        case 1: force_mid<1>(sm, lane, mid); break;
        case 2: force_mid<2>(sm, lane, mid); break;
        default: force_mid<3>(sm, lane, mid); break;
      }
    }
    if (r + 1 < a.nrhs) __syncthreads();  // the next right-hand side overwrites the spinors
  }
  if (!live) return;
  switch (mu) {
    case 0: force_compute<0>(a, sm, p, lane, h, sg, mid); break;
    case 1: force_compute<1>(a, sm, p, lane, h, sg, mid); break;
    case 2: force_compute<2>(a, sm, p, lane, h, sg, mid); break;
    default: force_compute<3>(a, sm, p, lane, h, sg, mid); break;
  }
}

// ------------------------------------------------------------------ staggered rational force
// _kernelDFermionKSForce (Staggered/CFieldFermionKSSU3.cu:216-262): with
// phi_i = (D D^+ + b_i)^-1 phi and phi_id = D0 phi_i (the massless D),
//   F_mu(x) -= Ta(s_+ eta_mu(x) [U_mu(x) A + B U_mu(x)^+]),
//   A = sum_i a_i phi_i(x+mu) phi_id(x)^+,   B = sum_i a_i phi_i(x) phi_id(x+mu)^+
// (the reference's two contractions per pole, makeSU3ContractV; Ta is linear, so
// the poles are summed before the one Ta and the one F update).  Same block
// shape as the Wilson force: 32 sites x 4 direction warps, parity-interleaved
// blocks.  The poles are streamed through a ring of cp.async stages (the
// copies of pole i+1 are in flight while pole i is contracted); U and F are
// staged once.  Compulsory DRAM traffic per site: 2 x 48 B per pole, U 576 B,
// F 1152 B.  With 12 poles on 32^3 x 16 the kernel runs at 0.57 of the copy
// bandwidth: each pole is a short contraction between two block barriers, and
// the per-pole copy issue and barrier waits, not DRAM, set the pace.
constexpr int KS_FORCE_MAX = 64;
constexpr int KS_HERE = 2 * 3 * TILE;     // phi_i(x), phi_id(x)        [field][k][site]
constexpr int KS_NBR = 4 * 2 * 3 * TILE;  // phi_i(x+mu), phi_id(x+mu)  [mu][field][k][site]
constexpr int KS_STAGE = KS_HERE + KS_NBR;
constexpr size_t ks_force_smem(int nstage) { return sizeof(double2) * (nstage * KS_STAGE + 2 * E_LINK); }

struct KsForceArgs {
  Geom g;
  const double2* U[2];
  double2* F[2];
  int64_t blk;  // bytes of one parity block of a field
  int n;
  const char* phi_i[KS_FORCE_MAX];
  const char* phi_id[KS_FORCE_MAX];
  double a[KS_FORCE_MAX];
};


// m[r][q] += w * l[r] conj(r[q])
__device__ __forceinline__ void outer3_acc(C m[9], double w, const double2* l, const double2* r) {
  C lv[3], rv[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double2 x = l[k * TILE], y = r[k * TILE];
    lv[k] = mk<double>(w * x.x, w * x.y);
    rv[k] = mk<double>(y.x, y.y);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      C t = m[3 * i + j];
      t.x = fma(lv[i].x, rv[j].x, fma(lv[i].y, rv[j].y, t.x));
      t.y = fma(lv[i].y, rv[j].x, fma(-lv[i].x, rv[j].y, t.y));
      m[3 * i + j] = t;
    }
}

template <int NSTAGE>
__global__ void __launch_bounds__(128) ks_force_kernel(KsForceArgs a) {
  extern __shared__ double2 sm[];
  const int p = (int)(blockIdx.x & 1);
  const int lane = (int)(threadIdx.x & 31), mu = (int)(threadIdx.x >> 5);
  const int64_t h = (int64_t)(blockIdx.x >> 1) * TILE + lane;
  const int64_t Vh = a.g.Vh;
  const bool live = h < Vh;
  double sg = 1.0, eta = 1.0;
  int64_t hn = 0;
  if (live) {
    hn = forward_nbr(a.g, p, h, mu, sg);
    int c[4];
    eo_coords(a.g, p, h, c);
    int cs = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (k < mu) cs += c[k];
    eta = (cs & 1) ? -1.0 : 1.0;
  }
  // byte offsets of this thread's site and forward neighbour in a field, and
  // of one colour component; per pole only the field base changes
  const int64_t off_here = (int64_t)p * a.blk + h * 16, off_nbr = (int64_t)(1 - p) * a.blk + hn * 16;
  const int64_t kstride = Vh * 16;
  double2* s_link = sm + NSTAGE * KS_STAGE;

  // copies of pole i into ring stage i % NSTAGE
  auto issue = [&](int i) {
    if (!live || i >= a.n) return;
    double2* st = sm + (i % NSTAGE) * KS_STAGE;
    const char* fi = a.phi_i[i];
    const char* fd = a.phi_id[i];
    // here: the 6 components f (phi_i k = f for f < 3, phi_id k = f - 3) over
    // the 4 warps, warp mu taking f = mu and f = mu + 4
    cp_async16(st + mu * TILE + lane,
               reinterpret_cast<const double2*>((mu == 3 ? fd : fi) + off_here + (mu == 3 ? 0 : mu) * kstride));
    if (mu < 2)
      cp_async16(st + (mu + 4) * TILE + lane, reinterpret_cast<const double2*>(fd + off_here + (mu + 1) * kstride));
    double2* dn = st + KS_HERE + mu * 6 * TILE + lane;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      cp_async16(dn + k * TILE, reinterpret_cast<const double2*>(fi + off_nbr + k * kstride));
      cp_async16(dn + (3 + k) * TILE, reinterpret_cast<const double2*>(fd + off_nbr + k * kstride));
    }
  };

  if (live) {
    const double2* ub = (p ? a.U[1] : a.U[0]) + (int64_t)mu * 9 * Vh + h;
    const double2* fb = (p ? a.F[1] : a.F[0]) + (int64_t)mu * 9 * Vh + h;
    double2* su = s_link + mu * 9 * TILE + lane;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      cp_async16(su + k * TILE, ub + k * Vh);
      cp_async16(su + E_LINK + k * TILE, fb + k * Vh);
    }
  }
  // prologue: poles 0 .. NSTAGE-2 in flight, one commit group each (group 0
  // also holds the links); every thread commits every group, empty or not
#pragma unroll
  for (int j = 0; j < NSTAGE - 1; ++j) {
    issue(j);
    cp_async_commit();
  }

  C A[9], B[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) A[k] = B[k] = mk<double>(0, 0);
  for (int i = 0; i < a.n; ++i) {
    issue(i + NSTAGE - 1);  // into the stage pole i - 1 used (released by the barrier below)
    cp_async_commit();
    cp_async_wait<NSTAGE - 1>();  // this thread's copies of pole i (and the links) landed
    __syncthreads();              // everyone's did
    if (live) {
      const double2* st = sm + (i % NSTAGE) * KS_STAGE;
      const double2* nb = st + KS_HERE + mu * 6 * TILE + lane;
      const double w = a.a[i];
      outer3_acc(A, w, nb, st + 3 * TILE + lane);  // phi_i(x+mu) phi_id(x)^+
      outer3_acc(B, w, st + lane, nb + 3 * TILE);  // phi_i(x) phi_id(x+mu)^+
    }
    __syncthreads();  // pole i's stage is free for pole i + NSTAGE
  }
  cp_async_wait<0>();
  __syncthreads();
  if (!live) return;

  // m = U A + B U^+
  const double2* su = s_link + mu * 9 * TILE + lane;
  C u[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double2 d = su[k * TILE];
    u[k] = mk<double>(d.x, d.y);
  }
  C m[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      C t = u[3 * i] * A[j] + u[3 * i + 1] * A[3 + j] + u[3 * i + 2] * A[6 + j];
      // (B U^+)_ij = sum_k B_ik conj(U_jk)
      t = t + B[3 * i] * cj(u[3 * j]) + B[3 * i + 1] * cj(u[3 * j + 1]) + B[3 * i + 2] * cj(u[3 * j + 2]);
      m[3 * i + j] = t;
    }
  // F -= s_+ eta Ta(m)
  const double w = -sg * eta;
  double2* fb = (p ? a.F[1] : a.F[0]) + (int64_t)mu * 9 * Vh + h;
  const double2* s_f = su + E_LINK;
  const double tr = (m[0].y + m[4].y + m[8].y) * (1.0 / 3.0);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      C t;
      if (i == j)
        t = mk<double>(0.0, m[4 * i].y - tr);
      else
        t = mk<double>(0.5 * (m[3 * i + j].x - m[3 * j + i].x), 0.5 * (m[3 * i + j].y + m[3 * j + i].y));
      double2 f = s_f[(3 * i + j) * TILE];
      f.x = fma(w, t.x, f.x);
      f.y = fma(w, t.y, f.y);
      fb[(3 * i + j) * Vh] = f;
    }
}

clg_status force_check(clg_gauge F, clg_gauge U, clg_field X, clg_field Y) {
  if (!F || !U || !X || !Y) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = U->lat->ctx;
  if (F->lat != U->lat || X->lat != U->lat || Y->lat != U->lat)
    return ctx->fail(CLG_ERR_BAD_ARG, "force: fields on different lattices");
  if (F == U) return ctx->fail(CLG_ERR_BAD_ARG, "force: the force field must not be the gauge field");
  if (X->kind != CLG_FERMION_WILSON || Y->kind != CLG_FERMION_WILSON)
    return ctx->fail(CLG_ERR_BAD_ARG, "force: Wilson fermion fields expected");
  if (X->subset != CLG_SUBSET_FULL || Y->subset != CLG_SUBSET_FULL)
    return ctx->fail(CLG_ERR_BAD_ARG, "force: FULL fields expected");
  if (X->prec != CLG_PREC_DOUBLE || Y->prec != CLG_PREC_DOUBLE)
    return ctx->fail(CLG_ERR_BAD_ARG, "force: FP64 fields expected");
  if (X->nrhs != Y->nrhs) return ctx->fail(CLG_ERR_BAD_ARG, "force: X and Y hold different numbers of right-hand sides");
  if (!U->u64[0] || !F->u64[0]) return ctx->fail(CLG_ERR_BAD_ARG, "force: gauge field without data");
  return CLG_SUCCESS;
}

}  // namespace

}  // namespace clg

using namespace clg;

extern "C" {

clg_status clg_wilson_force(clg_gauge F, clg_gauge U, clg_field X, clg_field Y) {
  clg_status st = force_check(F, U, X, Y);
  if (st) return st;
  if ((st = settle(X)) || (st = settle(Y))) return st;
  clg_context_s* ctx = U->lat->ctx;
  const Geom& g = U->lat->g;
  ForceArgs a;
  a.g = g;
  for (int p = 0; p < 2; ++p) {
    a.U[p] = reinterpret_cast<const double2*>(U->u64[p]);
    a.F[p] = reinterpret_cast<double2*>(F->u64[p]);
  }
  const FieldRef xr = X->ref(), yr = Y->ref();
  a.X = xr.data;
  a.Y = yr.data;
  a.blk = xr.blk;
  a.rstride = xr.rstride;
  a.nrhs = X->nrhs;
  a.kappa = X->param;
  const int64_t nblk = (g.Vh + TILE - 1) / TILE;
  const size_t smem = FORCE_SMEM;
  cudaError_t e = cudaFuncSetAttribute(wilson_force_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    wilson_force_kernel<<<(unsigned)(2 * nblk), 128, smem, ctx->stream>>>(a);
    ctx->kernels++;
    e = cudaPeekAtLastError();
  }
  if (e != cudaSuccess) return ctx->fail(cuda_status(e), cudaGetErrorString(e));
  F->su3 = false;
  F->unitarity = -1.0;
  F->dirty_lowp = true;
  return CLG_SUCCESS;
}

clg_status clg_wilson_fermion_force(clg_solver S, clg_gauge F, clg_gauge U, clg_field phi, clg_field cache,
                                    clg_solve_info* info) {
  if (!S || !F || !U || !phi || !info) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = S->ctx;
  if (phi->kind != CLG_FERMION_WILSON || phi->subset != CLG_SUBSET_FULL || phi->prec != CLG_PREC_DOUBLE)
    return ctx->fail(CLG_ERR_BAD_ARG, "fermion force: phi must be a FULL FP64 Wilson field");
  if (cache && (cache->lat != phi->lat || cache->kind != phi->kind || cache->subset != phi->subset ||
                cache->nrhs != phi->nrhs))
    return ctx->fail(CLG_ERR_BAD_ARG, "fermion force: the cache field differs from phi in shape");
  clg_status st = CLG_SUCCESS;
  // X and Y live with the solver between calls (one HMC trajectory calls this
  // once per molecular-dynamics step)
  for (clg_field* t : {&S->force_x, &S->force_y}) {
    clg_field f = *t;
    if (f && (f->lat != phi->lat || f->nrhs != phi->nrhs)) {
      clg_field_destroy(f);
      *t = f = nullptr;
    }
    if (!f) {
      st = clg_field_create(phi->lat, CLG_FERMION_WILSON, CLG_SUBSET_FULL, CLG_PREC_DOUBLE, phi->nrhs, phi->param, t);
      if (st) return st;
    }
    if ((st = clg_field_set_param(*t, phi->param))) return st;
  }
  clg_field X = S->force_x, Y = S->force_y;
  // a failed solve adds nothing to F (the reference returns FALSE before the force)
  if ((st = clg_solve(S, X, phi, U, CLG_OP_DDDAG, cache, info))) return st;
  if (cache && (st = clg_field_copy(cache, X))) return st;
  if ((st = clg_apply_to(CLG_OP_DDAG, Y, X, U, CLG_COEFF_NONE, 0.0, 0.0))) return st;
  return clg_wilson_force(F, U, X, Y);
}

clg_status clg_ks_force(clg_gauge F, clg_gauge U, int n, const clg_field* phi_i, const clg_field* phi_id,
                        const double* a) {
  if (!F || !U || !phi_i || !phi_id || !a) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = U->lat->ctx;
  if (n < 1 || n > KS_FORCE_MAX) return ctx->fail(CLG_ERR_BAD_ARG, "staggered force: 1 to 64 poles");
  if (F->lat != U->lat) return ctx->fail(CLG_ERR_BAD_ARG, "staggered force: fields on different lattices");
  if (F == U) return ctx->fail(CLG_ERR_BAD_ARG, "force: the force field must not be the gauge field");
  if (!U->u64[0] || !F->u64[0]) return ctx->fail(CLG_ERR_BAD_ARG, "force: gauge field without data");
  KsForceArgs k;
  k.g = U->lat->g;
  for (int p = 0; p < 2; ++p) {
    k.U[p] = reinterpret_cast<const double2*>(U->u64[p]);
    k.F[p] = reinterpret_cast<double2*>(F->u64[p]);
  }
  k.n = n;
  for (int i = 0; i < n; ++i) {
    for (clg_field f : {phi_i[i], phi_id[i]}) {
      if (!f || f->lat != U->lat || f->kind != CLG_FERMION_STAGGERED || f->subset != CLG_SUBSET_FULL ||
          f->prec != CLG_PREC_DOUBLE || f->nrhs != 1)
        return ctx->fail(CLG_ERR_BAD_ARG, "staggered force: FULL FP64 staggered fields of one right-hand side expected");
      if (clg_status st = settle(f)) return st;
    }
    k.phi_i[i] = phi_i[i]->data;
    k.phi_id[i] = phi_id[i]->data;
    k.a[i] = a[i];
  }
  for (int i = n; i < KS_FORCE_MAX; ++i) {
    k.phi_i[i] = k.phi_id[i] = nullptr;
    k.a[i] = 0.0;
  }
  k.blk = phi_i[0]->blk;
  const int64_t nblk = (k.g.Vh + TILE - 1) / TILE;
  // ring depth 2: 3, 4 and 5 stages (fewer blocks per SM) measured no faster,
  // nor did two or three poles per stage (409 / 606 us against 403); a
  // barrier-free form with the poles loaded through registers by four
  // direction threads per site in one warp ran at 782 us; U and F read from
  // global memory at the end instead of staged (4 blocks per SM at 128
  // registers, against 3 with staging) ran at 551 us against 399
  constexpr int nstage = 2;
  void (*kern)(KsForceArgs) = ks_force_kernel<nstage>;
  const size_t smem = ks_force_smem(nstage);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    kern<<<(unsigned)(2 * nblk), 128, smem, ctx->stream>>>(k);
    ctx->kernels++;
    e = cudaPeekAtLastError();
  }
  if (e != cudaSuccess) return ctx->fail(cuda_status(e), cudaGetErrorString(e));
  F->su3 = false;
  F->unitarity = -1.0;
  F->dirty_lowp = true;
  return CLG_SUCCESS;
}

clg_status clg_ks_fermion_force(clg_solver S, clg_gauge F, clg_gauge U, clg_field phi, int degree, const double* a,
                                const double* b, clg_solve_info* info) {
  if (!S || !F || !U || !phi || !a || !b || !info) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = S->ctx;
  if (degree < 1 || degree > KS_FORCE_MAX) return ctx->fail(CLG_ERR_BAD_ARG, "staggered force: 1 to 64 poles");
  if (phi->kind != CLG_FERMION_STAGGERED || phi->subset != CLG_SUBSET_FULL || phi->prec != CLG_PREC_DOUBLE ||
      phi->nrhs != 1)
    return ctx->fail(CLG_ERR_BAD_ARG, "staggered force: phi must be a FULL FP64 staggered field");
  clg_status st = CLG_SUCCESS;
  // phi_i and phi_id live with the solver between calls
  auto& fi = S->ks_phi_i;
  auto& fd = S->ks_phi_id;
  if (!fi.empty() && (fi[0]->lat != phi->lat || (int)fi.size() < degree)) {
    for (clg_field f : fi) clg_field_destroy(f);
    for (clg_field f : fd) clg_field_destroy(f);
    fi.clear();
    fd.clear();
  }
  while ((int)fi.size() < degree) {
    clg_field x = nullptr, y = nullptr;
    if ((st = clg_field_create(phi->lat, CLG_FERMION_STAGGERED, CLG_SUBSET_FULL, CLG_PREC_DOUBLE, 1, 0.0, &x)))
      return st;
    fi.push_back(x);
    if ((st = clg_field_create(phi->lat, CLG_FERMION_STAGGERED, CLG_SUBSET_FULL, CLG_PREC_DOUBLE, 1, 0.0, &y)))
      return st;
    fd.push_back(y);
  }
  std::vector<double> shifts(2 * degree);
  for (int i = 0; i < degree; ++i) {
    shifts[2 * i] = b[i];
    shifts[2 * i + 1] = 0.0;
  }
  // phi_i = (D D^+ + b_i)^-1 phi; a failed solve adds nothing to F
  if ((st = clg_solve_multishift(S, fi.data(), degree, shifts.data(), phi, U, CLG_OP_DDDAG, info))) return st;
  // phi_id = D0 phi_i: the fields carry mass 0, so D is the massless operator
  for (int i = 0; i < degree; ++i)
    if ((st = clg_apply_to(CLG_OP_D, fd[i], fi[i], U, CLG_COEFF_NONE, 0.0, 0.0))) return st;
  return clg_ks_force(F, U, degree, fi.data(), fd.data(), a);
}

}  // extern "C"
