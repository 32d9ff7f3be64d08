// krylov.cuh -- device-resident Krylov state and the fused site functors used
// by the solvers (solvers.cu).  All scalars of a right-hand side live in
// device memory; the finalize step of each reduction (run by the last block,
// one thread per right-hand side) updates them, so an iteration needs no
// host round trip (the reference reads every dot product back with a blocking
// copy: Core/CudaHelper.cu:697-710).
#pragma once
#include "blas.cuh"

namespace clg {

constexpr int GM_MAXK = 16;  // longest GMRES cycle kept on the device

enum : int { ST_RUNNING = 0, ST_CONVERGED = 1, ST_BREAKDOWN = 2 };

struct KState {
  // BiCGStab / CG scalars
  double2 rho, alpha, omega, beta;
  double rr, rr0, tol2;
  int done;      // this rhs needs no more work in the current inner solve
  int skip;      // kernels skip this rhs (done, or converged mid-iteration)
  int conv_s;    // BiCGStab: |s| small, finish with x += alpha p
  int status;
  int iters;     // operator applications
  int j;         // GMRES: columns built in this cycle
  int since;     // device-side inner loop: chunks without improving `best`
  int pad;
  // GMRES cycle
  double2 H[(GM_MAXK + 1) * GM_MAXK];  // H[i*GM_MAXK + j]
  double2 cs[GM_MAXK], sn[GM_MAXK];
  double2 g[GM_MAXK + 1];
  double2 y[GM_MAXK];
  double s[GM_MAXK + 1];   // lazy normalisation: v_i = s_i * V'_i
  double beta0;            // |r| at the start of the cycle
  double resid_est;        // |g_(j+1)| estimate
  double best;             // device-side inner loop: smallest residual seen (stagnation guard)
};

__device__ __forceinline__ bool bad(double v) { return !(v == v) || isinf(v); }

// ------------------------------------------------------------------ BiCGStab
// F_rv: (r^, v) -> alpha = rho / (r^, v)
template <int P, int NC>
struct BiAlpha {
  DField rh, v;
  KState* st;
  __device__ bool active(int r) const { return !st[r].skip; }
  __device__ void operator()(int rhs, int p, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> a[NC], b[NC];
    ldv<P, NC, AT>(rh, rhs, p, h, a);
    ldv<P, NC, AT>(v, rhs, p, h, b);
    acc_dot<NC, AT>(a, b, acc);
  }
  __device__ void finalize(int r, const double* s) const {
    KState& k = st[r];
    if (k.skip) return;
    const double2 d = make_double2(s[0], s[1]);
    if ((d.x == 0.0 && d.y == 0.0) || bad(d.x) || bad(d.y)) {
      k.status = ST_BREAKDOWN;
      k.done = k.skip = 1;
      return;
    }
    k.alpha = cdiv(k.rho, d);
    k.iters += 1;
  }
};

// r <- r - alpha v ; |r|^2 -> conv_s
template <int P, int NC>
struct BiS {
  DField r, v;
  KState* st;
  __device__ bool active(int q) const { return !st[q].skip; }
  __device__ void operator()(int rhs, int p, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> a[NC], b[NC];
    ldv<P, NC, AT>(r, rhs, p, h, a);
    ldv<P, NC, AT>(v, rhs, p, h, b);
    const double2 al = st[rhs].alpha;
    const cpx<AT> ca = mk<AT>((AT)al.x, (AT)al.y);
#pragma unroll
    for (int k = 0; k < NC; ++k) a[k] = a[k] - ca * b[k];
    stv<P, NC, AT>(r, rhs, p, h, a);
    acc[0] += site_norm2<NC, AT>(a);
  }
  __device__ void finalize(int q, const double* s) const {
    KState& k = st[q];
    if (k.skip) return;
    if (bad(s[0])) {
      k.status = ST_BREAKDOWN;
      k.done = k.skip = 1;
      return;
    }
    if (s[0] <= k.tol2 * k.rr0) {
      k.conv_s = 1;
      k.skip = 1;
    }
  }
};

// (t, s), (t, t) -> omega = (t, s) / (t, t)   [s stored in r]
template <int P, int NC>
struct BiOmega {
  DField t, r;
  KState* st;
  __device__ bool active(int q) const { return !st[q].skip; }
  __device__ void operator()(int rhs, int p, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> a[NC], b[NC];
    ldv<P, NC, AT>(t, rhs, p, h, a);
    ldv<P, NC, AT>(r, rhs, p, h, b);
    acc_dot<NC, AT>(a, b, acc);
    acc[2] += site_norm2<NC, AT>(a);
  }
  __device__ void finalize(int q, const double* s) const {
    KState& k = st[q];
    if (k.skip) return;
    k.iters += 1;
    if (!(s[2] > 0.0) || bad(s[2])) {
      k.status = ST_BREAKDOWN;
      k.done = k.skip = 1;
      return;
    }
    k.omega = make_double2(s[0] / s[2], s[1] / s[2]);
  }
};

// x += alpha p + omega s ; r = s - omega t ; (r^, r), |r|^2 -> beta, rho
// (or, when |s| was already small: x += alpha p and stop)
template <int P, int NC>
struct BiUpdate {
  DField x, p, r, t, rh;
  KState* st;
  __device__ bool active(int q) const { return !st[q].done; }
  __device__ void operator()(int rhs, int par, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    const KState& k = st[rhs];
    cpx<AT> vx[NC], vp[NC];
    ldv<P, NC, AT>(x, rhs, par, h, vx);
    ldv<P, NC, AT>(p, rhs, par, h, vp);
    const cpx<AT> ca = mk<AT>((AT)k.alpha.x, (AT)k.alpha.y);
    if (k.conv_s) {
#pragma unroll
      for (int i = 0; i < NC; ++i) vx[i] = vx[i] + ca * vp[i];
      stv<P, NC, AT>(x, rhs, par, h, vx);
      return;
    }
    cpx<AT> vr[NC], vt[NC], vh[NC];
    ldv<P, NC, AT>(r, rhs, par, h, vr);
    ldv<P, NC, AT>(t, rhs, par, h, vt);
    ldv<P, NC, AT>(rh, rhs, par, h, vh);
    const cpx<AT> co = mk<AT>((AT)k.omega.x, (AT)k.omega.y);
#pragma unroll
    for (int i = 0; i < NC; ++i) {
      vx[i] = vx[i] + ca * vp[i] + co * vr[i];
      vr[i] = vr[i] - co * vt[i];
    }
    stv<P, NC, AT>(x, rhs, par, h, vx);
    stv<P, NC, AT>(r, rhs, par, h, vr);
    acc_dot<NC, AT>(vh, vr, acc);
    acc[2] += site_norm2<NC, AT>(vr);
  }
  __device__ void finalize(int q, const double* s) const {
    KState& k = st[q];
    if (k.done) return;
    if (k.conv_s) {
      k.status = ST_CONVERGED;
      k.done = k.skip = 1;
      return;
    }
    const double2 rho_new = make_double2(s[0], s[1]);
    k.rr = s[2];
    if (bad(s[2]) || bad(rho_new.x)) {
      k.status = ST_BREAKDOWN;
      k.done = k.skip = 1;
      return;
    }
    if (s[2] <= k.tol2 * k.rr0) {
      k.status = ST_CONVERGED;
      k.done = k.skip = 1;
      return;
    }
    if ((rho_new.x == 0.0 && rho_new.y == 0.0) || (k.omega.x == 0.0 && k.omega.y == 0.0)) {
      k.status = ST_BREAKDOWN;
      k.done = k.skip = 1;
      return;
    }
    k.beta = cmul(cdiv(rho_new, k.rho), cdiv(k.alpha, k.omega));
    k.rho = rho_new;
  }
};

// p = r + beta (p - omega v)
template <int P, int NC>
struct BiP {
  DField p, r, v;
  KState* st;
  __device__ bool active(int q) const { return !st[q].skip; }
  __device__ void operator()(int rhs, int par, int64_t h, double*) const {
    using AT = typename AccT<P>::T;
    const KState& k = st[rhs];
    cpx<AT> vp[NC], vr[NC], vv[NC];
    ldv<P, NC, AT>(p, rhs, par, h, vp);
    ldv<P, NC, AT>(r, rhs, par, h, vr);
    ldv<P, NC, AT>(v, rhs, par, h, vv);
    const cpx<AT> cb = mk<AT>((AT)k.beta.x, (AT)k.beta.y), co = mk<AT>((AT)k.omega.x, (AT)k.omega.y);
#pragma unroll
    for (int i = 0; i < NC; ++i) vp[i] = vr[i] + cb * (vp[i] - co * vv[i]);
    stv<P, NC, AT>(p, rhs, par, h, vp);
  }
  __device__ void finalize(int, const double*) const {}
};

// start: r = b (x = 0), r^ = r, p = r, rho = |r|^2
template <int P, int NC>
struct BiInit {
  DField b, x, r, rh, p;
  KState* st;
  const double* tolv;  // relative tolerance per right-hand side
  __device__ bool active(int q) const { return !st[q].done; }
  __device__ void operator()(int rhs, int par, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> vb[NC], z[NC];
    ldv<P, NC, AT>(b, rhs, par, h, vb);
#pragma unroll
    for (int i = 0; i < NC; ++i) z[i] = mk<AT>(0, 0);
    stv<P, NC, AT>(x, rhs, par, h, z);
    stv<P, NC, AT>(r, rhs, par, h, vb);
    stv<P, NC, AT>(rh, rhs, par, h, vb);
    stv<P, NC, AT>(p, rhs, par, h, vb);
    acc[0] += site_norm2<NC, AT>(vb);
  }
  __device__ void finalize(int q, const double* s) const {
    KState& k = st[q];
    if (k.done) return;
    k.rr0 = k.rr = s[0];
    k.rho = make_double2(s[0], 0.0);
    k.tol2 = tolv[q] * tolv[q];
    k.conv_s = 0;
    k.status = ST_RUNNING;
    if (!(s[0] > 0.0)) {  // zero right-hand side: x = 0 is exact
      k.status = ST_CONVERGED;
      k.done = k.skip = 1;
    }
  }
};

// ------------------------------------------------------------------ CG (Hermitian positive definite)
// start: r = b, p = b, x = 0, rr = |b|^2
template <int P, int NC>
struct CgInit {
  DField b, x, r, p;
  KState* st;
  const double* tolv;  // relative tolerance per right-hand side
  __device__ bool active(int q) const { return !st[q].done; }
  __device__ void operator()(int rhs, int par, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> vb[NC], z[NC];
    ldv<P, NC, AT>(b, rhs, par, h, vb);
#pragma unroll
    for (int i = 0; i < NC; ++i) z[i] = mk<AT>(0, 0);
    stv<P, NC, AT>(x, rhs, par, h, z);
    stv<P, NC, AT>(r, rhs, par, h, vb);
    stv<P, NC, AT>(p, rhs, par, h, vb);
    acc[0] += site_norm2<NC, AT>(vb);
  }
  __device__ void finalize(int q, const double* s) const {
    KState& k = st[q];
    if (k.done) return;
    k.rr0 = k.rr = s[0];
    k.tol2 = tolv[q] * tolv[q];
    k.status = ST_RUNNING;
    if (!(s[0] > 0.0)) {
      k.status = ST_CONVERGED;
      k.done = k.skip = 1;
    }
  }
};
// pAp = (p, A p) -> alpha = rr / pAp; counts `weight` operator applications
__device__ __forceinline__ void cg_alpha_finalize(KState& k, double pAp, int weight) {
  if (k.skip) return;
  k.iters += weight;
  if (!(pAp > 0.0) || bad(pAp)) {
    k.status = ST_BREAKDOWN;
    k.done = k.skip = 1;
    return;
  }
  k.alpha = make_double2(k.rr / pAp, 0.0);
}
// rr_new = |r|^2 after the update -> beta, convergence
__device__ __forceinline__ void cg_update_finalize(KState& k, double rr_new) {
  if (k.skip) return;
  if (bad(rr_new)) {
    k.status = ST_BREAKDOWN;
    k.done = k.skip = 1;
    return;
  }
  k.beta = make_double2(rr_new / k.rr, 0.0);
  k.rr = rr_new;
  if (rr_new <= k.tol2 * k.rr0) {
    k.status = ST_CONVERGED;
    k.done = k.skip = 1;
  }
}

// (p, q) -> alpha = rr / (p, q)
template <int P, int NC>
struct CgAlpha {
  DField p, q;
  KState* st;
  int weight;  // operator applications per Krylov-operator application (2 for M M^+)
  __device__ bool active(int r) const { return !st[r].skip; }
  __device__ void operator()(int rhs, int par, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> a[NC], b[NC];
    ldv<P, NC, AT>(p, rhs, par, h, a);
    ldv<P, NC, AT>(q, rhs, par, h, b);
    acc_dot<NC, AT>(a, b, acc);
  }
  __device__ void finalize(int r, const double* s) const { cg_alpha_finalize(st[r], s[0], weight); }
};
// x += alpha p ; r -= alpha q ; rr_new -> beta
template <int P, int NC>
struct CgUpdate {
  DField x, r, p, q;
  KState* st;
  __device__ bool active(int w) const { return !st[w].skip; }
  __device__ void operator()(int rhs, int par, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    const AT al = (AT)st[rhs].alpha.x;
    cpx<AT> vx[NC], vr[NC], vp[NC], vq[NC];
    ldv<P, NC, AT>(x, rhs, par, h, vx);
    ldv<P, NC, AT>(r, rhs, par, h, vr);
    ldv<P, NC, AT>(p, rhs, par, h, vp);
    ldv<P, NC, AT>(q, rhs, par, h, vq);
#pragma unroll
    for (int i = 0; i < NC; ++i) {
      vx[i] = vx[i] + al * vp[i];
      vr[i] = vr[i] - al * vq[i];
    }
    stv<P, NC, AT>(x, rhs, par, h, vx);
    stv<P, NC, AT>(r, rhs, par, h, vr);
    acc[0] += site_norm2<NC, AT>(vr);
  }
  __device__ void finalize(int w, const double* s) const { cg_update_finalize(st[w], s[0]); }
};

// CG on A = M M^+ (or M^+ M) with the vector work fused into the Schur hops
// (wilson_hop_epi_kernel).  The second hop of the first factor produces
// q = M^+ p (or M p), stores it and reduces |q|^2 = (p, A p) -> alpha; the
// second hop of the second factor produces A p in registers only and applies
//   x += alpha p,  r -= alpha A p,  |r|^2 -> beta
// at its own site, so A p is never written and the separate (p, A p) and
// update passes disappear.  Both act on the even checkerboard (parity 0).
template <int P>
struct CgHopAlpha {
  static constexpr int NRED = 1;
  static constexpr bool STORE = true;
  KState* st;
  int weight;
  template <typename AT>
  __device__ void site(int, int64_t, const cpx<AT> q[12], double* red) const {
    red[0] += site_norm2<12, AT>(q);
  }
  __device__ void finalize(int r, const double* s) const { cg_alpha_finalize(st[r], s[0], weight); }
};
template <int P>
struct CgHopUpdate {
  static constexpr int NRED = 1;
  static constexpr bool STORE = false;
  DField x, r, p;
  KState* st;
  template <typename AT>
  __device__ void site(int rhs, int64_t h, const cpx<AT> ap[12], double* red) const {
    const AT al = (AT)st[rhs].alpha.x;
    cpx<AT> vx[12], vr[12], vp[12];
    ldv<P, 12, AT>(x, rhs, 0, h, vx);
    ldv<P, 12, AT>(r, rhs, 0, h, vr);
    ldv<P, 12, AT>(p, rhs, 0, h, vp);
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      vx[i] = vx[i] + al * vp[i];
      vr[i] = vr[i] - al * ap[i];
    }
    stv<P, 12, AT>(x, rhs, 0, h, vx);
    stv<P, 12, AT>(r, rhs, 0, h, vr);
    red[0] += site_norm2<12, AT>(vr);
  }
  __device__ void finalize(int w, const double* s) const { cg_update_finalize(st[w], s[0]); }
};
// p = r + beta p
template <int P, int NC>
struct CgP {
  DField p, r;
  KState* st;
  __device__ bool active(int w) const { return !st[w].skip; }
  __device__ void operator()(int rhs, int par, int64_t h, double*) const {
    using AT = typename AccT<P>::T;
    const AT be = (AT)st[rhs].beta.x;
    cpx<AT> vp[NC], vr[NC];
    ldv<P, NC, AT>(p, rhs, par, h, vp);
    ldv<P, NC, AT>(r, rhs, par, h, vr);
#pragma unroll
    for (int i = 0; i < NC; ++i) vp[i] = vr[i] + be * vp[i];
    stv<P, NC, AT>(p, rhs, par, h, vp);
  }
  __device__ void finalize(int, const double*) const {}
};

// ------------------------------------------------------------------ GMRES(k)
// V' vectors are stored un-normalised; v_i = s_i V'_i (s_i in KState).
struct VList {
  DField v[GM_MAXK + 1];
};

// cycle start: V'_0 = b - (K x) [w holds K x, or nothing for x = 0]; beta = |V'_0|
template <int P, int NC>
struct GmStart {
  DField b, w, v0;
  KState* st;
  int have_x;
  const double* tolv;  // relative to |b| of the inner solve (stored in rr0 at first cycle)
  int first;
  __device__ bool active(int q) const { return !st[q].done; }
  __device__ void operator()(int rhs, int par, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> vb[NC];
    ldv<P, NC, AT>(b, rhs, par, h, vb);
    if (have_x) {
      cpx<AT> vw[NC];
      ldv<P, NC, AT>(w, rhs, par, h, vw);
#pragma unroll
      for (int i = 0; i < NC; ++i) vb[i] = vb[i] - vw[i];
    }
    stv<P, NC, AT>(v0, rhs, par, h, vb);
    acc[0] += site_norm2<NC, AT>(vb);
  }
  __device__ void finalize(int q, const double* s) const {
    KState& k = st[q];
    if (k.done) return;
    if (first) {
      k.rr0 = s[0];
      k.tol2 = tolv[q] * tolv[q];
      k.status = ST_RUNNING;
    }
    k.skip = 0;
    k.j = 0;
    const double beta = sqrt(s[0]);
    k.beta0 = beta;
    k.resid_est = beta;
    if (bad(beta)) {
      k.status = ST_BREAKDOWN;
      k.done = k.skip = 1;
      return;
    }
    if (s[0] <= k.tol2 * k.rr0) {
      k.status = ST_CONVERGED;
      k.done = k.skip = 1;
      return;
    }
    k.g[0] = make_double2(beta, 0.0);
    k.s[0] = 1.0 / beta;
  }
};

// h_ij = s_i <V'_i, w>, i <= J: J+1 dot products (2(J+1) reductions) in one pass;
// J is a template argument so the reduction width matches the column
template <int P, int NC, int J>
struct GmDotsJ {
  VList V;
  DField w;
  KState* st;
  __device__ bool active(int q) const { return !st[q].skip; }
  __device__ void operator()(int rhs, int par, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> vw[NC];
    ldv<P, NC, AT>(w, rhs, par, h, vw);
#pragma unroll
    for (int i = 0; i <= J; ++i) {
      cpx<AT> vi[NC];
      ldv<P, NC, AT>(V.v[i], rhs, par, h, vi);
      acc_dot<NC, AT>(vi, vw, acc + 2 * i);
    }
  }
  __device__ void finalize(int q, const double* s) const {
    KState& k = st[q];
    if (k.skip) return;
    k.iters += 1;
    for (int i = 0; i <= J; ++i) k.H[i * GM_MAXK + J] = make_double2(k.s[i] * s[2 * i], k.s[i] * s[2 * i + 1]);
  }
};

// V'_{j+1} = w - sum_i h_ij v_i ; h_{j+1,j} = |V'_{j+1}| ; Givens rotation of column j
template <int P, int NC>
struct GmOrtho {
  VList V;
  DField w;
  KState* st;
  int j;
  __device__ bool active(int q) const { return !st[q].skip; }
  __device__ void operator()(int rhs, int par, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    const KState& k = st[rhs];
    cpx<AT> vw[NC];
    ldv<P, NC, AT>(w, rhs, par, h, vw);
#pragma unroll
    for (int i = 0; i < GM_MAXK; ++i) {
      if (i > j) break;
      cpx<AT> vi[NC];
      ldv<P, NC, AT>(V.v[i], rhs, par, h, vi);
      const double2 c = k.H[i * GM_MAXK + j];
      const cpx<AT> cc = mk<AT>((AT)(c.x * k.s[i]), (AT)(c.y * k.s[i]));
#pragma unroll
      for (int m = 0; m < NC; ++m) vw[m] = vw[m] - cc * vi[m];
    }
    stv<P, NC, AT>(V.v[j + 1], rhs, par, h, vw);
    acc[0] += site_norm2<NC, AT>(vw);
  }
  __device__ void finalize(int q, const double* s) const {
    KState& k = st[q];
    if (k.skip) return;
    const double hn = sqrt(s[0]);
    double2* H = k.H;
    H[(j + 1) * GM_MAXK + j] = make_double2(hn, 0.0);
    k.s[j + 1] = hn > 0.0 ? 1.0 / hn : 0.0;
    // apply the previous rotations to column j (RotateH, CSolverGMRES.cpp:262-327, incrementally)
    for (int i = 0; i < j; ++i) {
      const double2 hij = H[i * GM_MAXK + j], hi1 = H[(i + 1) * GM_MAXK + j];
      H[i * GM_MAXK + j] = make_double2(0, 0);
      const double2 a = cmul(cconj(k.cs[i]), hij), b = cmul(cconj(k.sn[i]), hi1);
      H[i * GM_MAXK + j] = make_double2(a.x + b.x, a.y + b.y);
      const double2 c = cmul(k.cs[i], hi1), d = cmul(k.sn[i], hij);
      H[(i + 1) * GM_MAXK + j] = make_double2(c.x - d.x, c.y - d.y);
    }
    const double2 hjj = H[j * GM_MAXK + j], hj1 = H[(j + 1) * GM_MAXK + j];
    const double den = sqrt(hjj.x * hjj.x + hjj.y * hjj.y + hj1.x * hj1.x + hj1.y * hj1.y);
    if (!(den > 0.0) || bad(den)) {
      k.status = ST_BREAKDOWN;
      k.skip = 1;
      return;
    }
    const double2 cs = make_double2(hjj.x / den, hjj.y / den), sn = make_double2(hj1.x / den, hj1.y / den);
    k.cs[j] = cs;
    k.sn[j] = sn;
    H[j * GM_MAXK + j] = make_double2(den, 0.0);
    H[(j + 1) * GM_MAXK + j] = make_double2(0.0, 0.0);
    const double2 gj = k.g[j];
    const double2 m = cmul(sn, gj);
    k.g[j + 1] = make_double2(-m.x, -m.y);
    k.g[j] = cmul(cconj(cs), gj);
    k.j = j + 1;
    const double2 gn = k.g[j + 1];
    k.resid_est = sqrt(gn.x * gn.x + gn.y * gn.y);
    // happy breakdown or converged: stop extending this cycle
    if (k.resid_est * k.resid_est <= k.tol2 * k.rr0 || hn == 0.0) k.skip = 1;
  }
};

// back substitution of the j x j triangle (SolveY, CSolverGMRES.cpp:329-358); coefficients y_i s_i
__global__ void gm_solve_y(KState* st, int nrhs);

// x += sum_i (y_i s_i) V'_i over the columns built in this cycle
template <int P, int NC>
struct GmUpdate {
  VList V;
  DField x;
  KState* st;
  int kmax;
  __device__ bool active(int q) const { return !st[q].done && st[q].j > 0; }
  __device__ void operator()(int rhs, int par, int64_t h, double*) const {
    using AT = typename AccT<P>::T;
    const KState& k = st[rhs];
    cpx<AT> vx[NC];
    ldv<P, NC, AT>(x, rhs, par, h, vx);
    for (int i = 0; i < k.j; ++i) {
      cpx<AT> vi[NC];
      ldv<P, NC, AT>(V.v[i], rhs, par, h, vi);
      const double2 c = k.y[i];
      const cpx<AT> cc = mk<AT>((AT)c.x, (AT)c.y);
#pragma unroll
      for (int m = 0; m < NC; ++m) vx[m] = vx[m] + cc * vi[m];
    }
    stv<P, NC, AT>(x, rhs, par, h, vx);
  }
  __device__ void finalize(int, const double*) const {}
};

}  // namespace clg
