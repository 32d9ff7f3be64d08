// multishift.cu -- CMultiShiftSolver::Solve (SparseLinearAlgebra/CMultiShiftSolver.h:38-47):
// (op + c_n) x_n = b for n < nshift, and CFieldFermion::RationalApproximation
// (Data/Field/CField.cpp:114-145).
//
// CLG_SOLVER_CGM (Hermitian positive operators, real shifts >= 0): multi-shift
// CG (B. Jegerlehner, hep-lat/9612014) shares one Krylov space for all shifts in
// the inner precision; every shift is then refined to the FP64 true residual by
// the batched defect-correction loop with the shifts as right-hand sides.
// The reference has no CG-M; its multi-shift family (CMultiShiftFOM,
// CMultiShiftGMRES, CMultiShiftBiCGStab, CMultiShiftNested) shares the interface.
//
// CLG_SOLVER_FOM_MS (any operator, complex shifts): CMultiShiftFOM's restarted
// FOM over one Krylov space in FP64 (mskrylov.cu), then the batched FP64
// defect correction checks (and if needed refines) every shift.
//
// CLG_SOLVER_NESTED_MS (any operator, complex shifts): all shifts are solved as
// one batch of right-hand sides (one launch per step covers every shift) by
// GMRES in the inner precision inside FP64 defect correction, the batched
// counterpart of CMultiShiftNested::Solve (CMultiShiftNested.cpp:69-145).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "dslash.cuh"
#include "krylov.cuh"

namespace clg {

clg_status fom_ms_run(clg_context_s* ctx, std::unique_ptr<SolveCacheBase>& cache, const clg_gauge_s* U, int kind,
                      double param, int op, const FieldRef& b, const std::vector<double2>& shifts, int m,
                      int restart, double tol, const FieldRef** X_out, int* apps_out, int* cycles_out);

clg_status bicgstab_ms_run(clg_context_s* ctx, std::unique_ptr<SolveCacheBase>& cache, const clg_gauge_s* U, int kind,
                           double param, int op, const FieldRef& b, const std::vector<double2>& shifts, int dev_step,
                           int max_step, double tol, const FieldRef** X_out, int* apps_out, int* iters_out);

clg_status gmres_ms_run(clg_context_s* ctx, std::unique_ptr<SolveCacheBase>& cache, const clg_gauge_s* U, int kind,
                        double param, int op, const FieldRef& b, const std::vector<double2>& shifts, int m, int restart,
                        double tol, const FieldRef** X_out, int* apps_out, int* cycles_out);

constexpr int CGM_MAXSHIFT = 64;
constexpr int CGM_RING_MAX = 8;

// Ring length M of the deferred shift updates: the flush holds M residuals of
// a site in registers (M * NC complex doubles).
constexpr int cgm_ring(int nc) { return nc == 3 ? 8 : 2; }

// Device state of a multi-shift CG.  The shifted vectors x_k, p_k are not
// touched every iteration: within a block of M iterations starting at s they
// are kept as coefficients over the materialised p_k^s and the block's
// residuals r_{s+1..s+M} (the base residual ring),
//   p_k^j = cg_k p_k^s + sum_u cc_k[u] r_{s+u},
//   x_k^j = x_k^s + ch_k p_k^s + sum_u ce_k[u] r_{s+u},
// and one flush per block writes x_k^{s+M}, p_k^{s+M}.
struct CgmState {
  double rr, bb, tol2, alpha, alpha_old, beta, pq;
  int iters, done, nshift, nvalid;  // nvalid: residuals of the current block in the ring
  double shift[CGM_MAXSHIFT];
  double zeta[CGM_MAXSHIFT], zeta_old[CGM_MAXSHIFT], zeta_new[CGM_MAXSHIFT];
  double alpha_k[CGM_MAXSHIFT];
  int active[CGM_MAXSHIFT];
  int pend_x[CGM_MAXSHIFT];  // x_k has updates in this block
  int pend_p[CGM_MAXSHIFT];  // p_k is needed after this block (shift still iterating)
  double cg[CGM_MAXSHIFT], ch[CGM_MAXSHIFT];
  double cc[CGM_MAXSHIFT][CGM_RING_MAX + 1], ce[CGM_MAXSHIFT][CGM_RING_MAX + 1];
};

namespace {

// (p, q) -> alpha and the shifted alpha_k (Jegerlehner eq. for zeta_{n+1});
// x_k^{j+1} = x_k^j + alpha_k p_k^j goes into the block coefficients.  t is
// the iteration's position in its block (t = 0 opens a block: the previous
// one was flushed).
template <int P, int NC>
struct CgmAlpha {
  DField p, q;
  CgmState* st;
  int t;
  __device__ bool active(int) const { return !st->done; }
  __device__ void operator()(int, int par, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> a[NC], b[NC];
    ldv<P, NC, AT>(p, 0, par, h, a);
    ldv<P, NC, AT>(q, 0, par, h, b);
    AT re = 0;
#pragma unroll
    for (int k = 0; k < NC; ++k) re += a[k].x * b[k].x + a[k].y * b[k].y;
    acc[0] += (double)re;
  }
  // shift k's part of the finalize; every load comes before the first store,
  // so one round of memory latency covers them
  __device__ void shift_alpha(CgmState& c, int k, bool go, double alpha, double beta, double aold) const {
    constexpr int R = CGM_RING_MAX;
    const int act = c.active[k];
    const double zn = c.zeta[k], zo = c.zeta_old[k], sh = c.shift[k];
    double cg = 1.0, ch = 0.0, cc[R + 1], ce[R + 1];
#pragma unroll
    for (int u = 1; u <= R; ++u) cc[u] = ce[u] = 0.0;
    if (t > 0) {
      cg = c.cg[k];
      ch = c.ch[k];
#pragma unroll
      for (int u = 1; u <= R; ++u)
        if (u <= t) {
          cc[u] = c.cc[k][u];
          ce[u] = c.ce[k][u];
        }
    } else {
      // a block opens: the previous one was flushed
      c.pend_x[k] = c.pend_p[k] = 0;
      c.cg[k] = 1.0;
      c.ch[k] = 0.0;
#pragma unroll
      for (int u = 0; u <= R; ++u) c.cc[k][u] = c.ce[k][u] = 0.0;
    }
    if (!go || !act) return;
    const double den = alpha * beta * (zo - zn) + zo * aold * (1.0 + sh * alpha);
    const double znew = zn * zo * aold / den;
    const double ak = alpha * znew / zn;
    c.zeta_new[k] = znew;
    c.alpha_k[k] = ak;
    c.ch[k] = ch + ak * cg;
#pragma unroll
    for (int u = 1; u <= R; ++u)
      if (u <= t) c.ce[k][u] = ce[u] + ak * cc[u];
    c.pend_x[k] = 1;
  }
  // warp 0 of the last block: lane l owns the shifts k = l, l + 32.  Runs on
  // every replayed iteration, also once all shifts are done, so a flushed
  // block is never applied twice.
  __device__ void finalize_warp(int, const double* s, int lane) const {
    CgmState& c = *st;
    const int ns = c.nshift, done = c.done;
    const double rr = c.rr, beta = c.beta, aold = c.alpha_old;
    const bool ok = s[0] > 0.0 && !bad(s[0]);
    const bool go = !done && ok;
    const double alpha = rr / s[0];
    if (lane < ns) shift_alpha(c, lane, go, alpha, beta, aold);
    if (lane + 32 < ns) shift_alpha(c, lane + 32, go, alpha, beta, aold);
    __syncwarp();
    if (lane == 0) {
      if (t == 0) c.nvalid = 0;
      if (!done) {
        c.iters += 1;
        if (ok) c.alpha = alpha;
        else c.done = 2;
      }
    }
  }
};

// r_{j+1} = r_j - alpha q (ring slots t -> t + 1 mod M); |r|^2 -> beta,
// beta_k, p_k^{j+1} = zeta_k r_{j+1} + beta_k p_k^j into the coefficients,
// convergence per shift
template <int P, int NC>
struct CgmR {
  DField ring, q;
  CgmState* st;
  int t, M;
  __device__ bool active(int) const { return !st->done; }
  __device__ void operator()(int, int par, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> vr[NC], vq[NC];
    ldv<P, NC, AT>(ring, t, par, h, vr);
    ldv<P, NC, AT>(q, 0, par, h, vq);
    const AT a = (AT)st->alpha;
#pragma unroll
    for (int i = 0; i < NC; ++i) vr[i] = vr[i] - a * vq[i];
    stv<P, NC, AT>(ring, (t + 1) % M, par, h, vr);
    acc[0] += site_norm2<NC, AT>(vr);
  }
  // shift k's part; loads before stores (one round of memory latency).
  // Returns whether shift k still iterates.
  __device__ int shift_r(CgmState& c, int k, double beta, double s0, double lim) const {
    constexpr int R = CGM_RING_MAX;
    const int act = c.active[k];
    const double znew = c.zeta_new[k], z = c.zeta[k], cg = c.cg[k];
    double cc[R + 1];
#pragma unroll
    for (int u = 1; u <= R; ++u) cc[u] = u <= t ? c.cc[k][u] : 0.0;
    if (!act) return 0;
    const double ratio = znew / z;
    const double bk = beta * ratio * ratio;
    c.zeta_old[k] = z;
    c.zeta[k] = znew;
    c.cg[k] = cg * bk;
#pragma unroll
    for (int u = 1; u <= R; ++u)
      if (u <= t) c.cc[k][u] = cc[u] * bk;
    c.cc[k][t + 1] = znew;
    const bool conv = znew * znew * s0 <= lim;
    if (conv) c.active[k] = 0;
    c.pend_p[k] = conv ? 0 : 1;
    return conv ? 0 : 1;
  }
  // warp 0 of the last block: lane l owns the shifts k = l, l + 32
  __device__ void finalize_warp(int, const double* s, int lane) const {
    CgmState& c = *st;
    const int ns = c.nshift, done = c.done;
    const double rr = c.rr, lim = c.tol2 * c.bb;
    if (done) return;
    if (bad(s[0])) {
      __syncwarp();
      if (lane == 0) c.done = 2;
      return;
    }
    const double beta = s[0] / rr;
    int nact = 0;
    if (lane < ns) nact += shift_r(c, lane, beta, s[0], lim);
    if (lane + 32 < ns) nact += shift_r(c, lane + 32, beta, s[0], lim);
    nact = __reduce_add_sync(0xffffffffu, nact);
    __syncwarp();  // every lane has read rr before lane 0 replaces it
    if (lane == 0) {
      c.nvalid = t + 1;
      c.alpha_old = c.alpha;
      c.beta = beta;
      c.rr = s[0];
      if (nact == 0) c.done = 1;
    }
  }
};

// p = r_{j+1} + beta p (ring slot `slot`), inside a block
template <int P, int NC>
struct CgmP {
  DField ring, p;
  CgmState* st;
  int slot;
  __device__ bool active(int) const { return !st->done; }
  __device__ void operator()(int, int par, int64_t h, double*) const {
    using AT = typename AccT<P>::T;
    cpx<AT> vr[NC], vp[NC];
    ldv<P, NC, AT>(ring, slot, par, h, vr);
    ldv<P, NC, AT>(p, 0, par, h, vp);
    const AT b = (AT)st->beta;
#pragma unroll
    for (int i = 0; i < NC; ++i) vp[i] = vr[i] + b * vp[i];
    stv<P, NC, AT>(p, 0, par, h, vp);
  }
  __device__ void finalize(int, const double*) const {}
};

// The block's last iteration: p = r_{s+M} + beta p, and every shift with
// pending updates takes them from the M residuals r_{s+u} (ring slot u mod M,
// only the nvalid written in this block):
//   x_k += ch_k p_k + sum_u ce_k[u] r_{s+u};  p_k = cg_k p_k + sum_u cc_k[u] r_{s+u}
// Each site's residuals are read once for all shifts.
// The ring and p are in the iteration precision PR; x_k, p_k are FP64.
template <int PR, int NC, int M>
struct CgmFlush {
  DField ring, x, pk, p;
  CgmState* st;
  int nshift;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int, int par, int64_t h, double*) const {
    using AT = double;
    const int nv = st->nvalid;
    cpx<AT> rv[M][NC];
#pragma unroll
    for (int u = 0; u < M; ++u) {
      if (u < nv) {
        ldv<PR, NC, AT>(ring, (u + 1) % M, par, h, rv[u]);
      } else {
#pragma unroll
        for (int i = 0; i < NC; ++i) rv[u][i] = mk<AT>(0, 0);
      }
    }
    if (!st->done) {
      cpx<AT> vp[NC];
      ldv<PR, NC, AT>(p, 0, par, h, vp);
      const AT b = st->beta;
#pragma unroll
      for (int i = 0; i < NC; ++i) vp[i] = rv[M - 1][i] + b * vp[i];
      stv<PR, NC, AT>(p, 0, par, h, vp);
    }
    for (int k = 0; k < nshift; ++k) {
      const bool px = st->pend_x[k], pp = st->pend_p[k];
      if (!px && !pp) continue;
      cpx<AT> vk[NC];
      ldv<P64, NC, AT>(pk, k, par, h, vk);
      if (px) {
        cpx<AT> vx[NC];
        ldv<P64, NC, AT>(x, k, par, h, vx);
        const AT a = st->ch[k];
#pragma unroll
        for (int i = 0; i < NC; ++i) vx[i] = vx[i] + a * vk[i];
#pragma unroll
        for (int u = 0; u < M - 1; ++u) {
          const AT e = st->ce[k][u + 1];
#pragma unroll
          for (int i = 0; i < NC; ++i) vx[i] = vx[i] + e * rv[u][i];
        }
        stv<P64, NC, AT>(x, k, par, h, vx);
      }
      if (pp) {
        const AT g = st->cg[k];
#pragma unroll
        for (int i = 0; i < NC; ++i) vk[i] = g * vk[i];
#pragma unroll
        for (int u = 0; u < M; ++u) {
          const AT cu = st->cc[k][u + 1];
#pragma unroll
          for (int i = 0; i < NC; ++i) vk[i] = vk[i] + cu * rv[u][i];
        }
        stv<P64, NC, AT>(pk, k, par, h, vk);
      }
    }
  }
  __device__ void finalize(int, const double*) const {}
};

// start (FP64): r_0 = p = b (ring slot 0), x_k = 0, p_k = b, |b|^2
template <int P, int NC>
struct CgmInit {
  DField b, ring, p, x, pk;
  CgmState* st;
  int nshift;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int, int par, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> vb[NC], z[NC];
    ldv<P, NC, AT>(b, 0, par, h, vb);
#pragma unroll
    for (int i = 0; i < NC; ++i) z[i] = mk<AT>(0, 0);
    stv<P, NC, AT>(ring, 0, par, h, vb);
    stv<P, NC, AT>(p, 0, par, h, vb);
    for (int k = 0; k < nshift; ++k) {
      stv<P, NC, AT>(x, k, par, h, z);
      stv<P, NC, AT>(pk, k, par, h, vb);
    }
    acc[0] += site_norm2<NC, AT>(vb);
  }
  __device__ void finalize(int, const double* s) const {
    CgmState& c = *st;
    c.rr = c.bb = s[0];
    c.alpha_old = 1.0;
    c.beta = 0.0;
    c.iters = 0;
    c.nvalid = 0;
    c.done = s[0] > 0.0 ? 0 : 1;
    for (int k = 0; k < c.nshift; ++k) {
      c.zeta[k] = c.zeta_old[k] = 1.0;
      c.active[k] = c.done ? 0 : 1;
      c.pend_x[k] = c.pend_p[k] = 0;
    }
  }
};

// A mixed solve leaves FP64 for the inner precision PR at a chunk boundary
// (every shift vector flushed, the residual in ring slot 0): r and p change
// precision, the iteration goes on.
template <int PR, int NC>
struct CgmSwitch {
  DField ring64, p64, ring, p;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int, int par, int64_t h, double*) const {
    cpx<double> v[NC];
    ldv<P64, NC, double>(ring64, 0, par, h, v);
    stv<PR, NC, double>(ring, 0, par, h, v);
    ldv<P64, NC, double>(p64, 0, par, h, v);
    stv<PR, NC, double>(p, 0, par, h, v);
  }
  __device__ void finalize(int, const double*) const {}
};

struct OwnedF {
  FieldRef ref;
  void* data = nullptr;
  float* norm = nullptr;
  ~OwnedF() {
    dfree(data);
    dfree(norm);
  }
  clg_status alloc(clg_context_s* ctx, int prec, int nc, int nparity, int fp, int nrhs, int64_t Vh) {
    const int64_t blk = Vh * site_bytes_of(prec, nc);
    clg_status st = dalloc(ctx, &data, (size_t)blk * nparity * nrhs);
    if (st) return st;
    if (prec == CLG_PREC_HALF && (st = dalloc(ctx, (void**)&norm, (size_t)Vh * nparity * nrhs * sizeof(float)))) return st;
    ref.data = (char*)data;
    ref.norm = norm;
    ref.blk = blk;
    ref.rstride = blk * nparity;
    ref.nrstride = norm ? Vh * nparity : 0;
    ref.nparity = nparity;
    ref.first_parity = fp;
    ref.prec = prec;
    ref.nc = nc;
    ref.nrhs = nrhs;
    ref.Vh = Vh;
    return CLG_SUCCESS;
  }
};

// The vectors of the shared iteration in one precision: the residual ring,
// p, q = A p and the operator's temporaries.
struct CgmIter {
  OwnedF ring, p, q, t_odd, t_full;
  cudaGraphExec_t exec = nullptr;  // a captured chunk of iterations
  int64_t graph_kernels = 0;
  bool tuned = false;  // one chunk ran eagerly (its launches are tuned)
  ~CgmIter() {
    if (exec) cudaGraphExecDestroy(exec);
  }
  clg_status alloc(clg_context_s* ctx, int P, int nc, int np, int fp, int M, int64_t Vh, int op) {
    clg_status s;
    if ((s = ring.alloc(ctx, P, nc, np, fp, M, Vh)) || (s = p.alloc(ctx, P, nc, np, fp, 1, Vh)) ||
        (s = q.alloc(ctx, P, nc, np, fp, 1, Vh)) || (s = t_odd.alloc(ctx, P, nc, 1, 1, 1, Vh)))
      return s;
    if (op == CLG_OP_DDDAG && (s = t_full.alloc(ctx, P, nc, 2, 0, 1, Vh))) return s;
    return CLG_SUCCESS;
  }
};

// Buffers, device state, pinned summary and the captured iteration graphs of a
// multi-shift CG, kept in the solver between calls with the same shape and
// gauge arrays (a call then costs the solve, not cudaMalloc/cudaFree, pinned
// allocations and a graph capture).  The solutions x_k, the shifted p_k and
// the start vector are FP64; it[0] iterates in FP64, it[1] (mixed solves) in
// the inner precision.
struct CgmWork : SolveCacheBase {
  std::string key;
  OwnedF X, bP, pk;
  CgmIter it[2];
  int M = 1;  // ring length (residuals per flush block)
  CgmState* st = nullptr;
  CgmState* hs = nullptr;  // pinned copy read per chunk
  ~CgmWork() {
    dfree(st);
    if (hs) cudaFreeHost(hs);
  }
  clg_status alloc(clg_context_s* ctx, int P, int nc, int np, int fp, int ns, int64_t Vh, int op) {
    clg_status s;
    M = cgm_ring(nc);
    if ((s = X.alloc(ctx, CLG_PREC_DOUBLE, nc, np, fp, ns, Vh)) ||
        (s = bP.alloc(ctx, CLG_PREC_DOUBLE, nc, np, fp, 1, Vh)) ||
        (s = pk.alloc(ctx, CLG_PREC_DOUBLE, nc, np, fp, ns, Vh)) ||
        (s = it[0].alloc(ctx, CLG_PREC_DOUBLE, nc, np, fp, M, Vh, op)))
      return s;
    if (P != CLG_PREC_DOUBLE && (s = it[1].alloc(ctx, P, nc, np, fp, M, Vh, op))) return s;
    if ((s = dalloc(ctx, (void**)&st, sizeof(CgmState)))) return s;
    if (cudaMallocHost((void**)&hs, sizeof(CgmState)) != cudaSuccess) {
      hs = nullptr;
      return ctx->fail(CLG_ERR_OOM, "multi-shift: pinned state");
    }
    return CLG_SUCCESS;
  }
};

// q = (DD^+)_ee p = (2am)^2 p - H_eo H_oe p for the staggered Schur operator
// (FP64 / FP32) with (p, q) -> alpha (CgmAlpha) reduced in the second hop's
// epilogue: the iteration needs no separate pass over p and q.
template <int PR, int NC>
clg_status cgm_schur_alpha(clg_context_s* ctx, CgmIter& I, clg_gauge_s* U, int kind, double param, CgmState* st,
                           int t) {
  HopSpec s1;
  s1.kind = kind;
  s1.prec = PR;
  s1.dagger = false;
  s1.out_parity = 1;
  s1.in = I.p.ref;
  s1.out = I.t_odd.ref;
  s1.x = nullptr;
  s1.a = make_double2(1, 0);
  s1.xa = make_double2(0, 0);
  s1.scale_dev = nullptr;
  s1.scale_stride = 0;
  s1.skip_dev = &st->done;
  s1.skip_stride = 0;
  s1.nrhs = 1;
  if (clg_status e = hop(ctx, U, s1)) return e;
  HopSpec s2 = s1;
  s2.out_parity = 0;
  s2.in = I.t_odd.ref;
  s2.out = I.q.ref;
  s2.x = &I.p.ref;
  s2.a = make_double2(-1, 0);
  s2.xa = make_double2(param * param, 0);
  HopArgs a;
  if (clg_status e = make_hop_args(ctx, U, s2, a)) return e;
  const int bs = 256;
  const int64_t nb = (a.g.Vh + bs - 1) / bs;
  if (clg_status e = ensure_reduction(ctx, nb)) return e;
  const CgmAlpha<PR, NC> f{dfield(I.p.ref), dfield(I.q.ref), st, t};
  cudaError_t err;
  if constexpr (PR == P64)
    err = launch_pdl(ctx, staggered_hop_xdot_kernel<P64, 18, 3, CgmAlpha<PR, NC>>, dim3((unsigned)nb), dim3(bs), 0, a,
                     f, ctx->red_partials, ctx->red_counter);
  else if (U->recon32 == 12)
    err = launch_pdl(ctx, staggered_hop_xdot_kernel<P32, 12, 4, CgmAlpha<PR, NC>>, dim3((unsigned)nb), dim3(bs), 0, a,
                     f, ctx->red_partials, ctx->red_counter);
  else
    err = launch_pdl(ctx, staggered_hop_xdot_kernel<P32, 18, 4, CgmAlpha<PR, NC>>, dim3((unsigned)nb), dim3(bs), 0, a,
                     f, ctx->red_partials, ctx->red_counter);
  if (err != cudaSuccess) return ctx->fail(cuda_status(err), std::string("multi-shift hop: ") + cudaGetErrorString(err));
  return CLG_SUCCESS;
}

// One chunk of multi-shift CG iterations on the vectors I (precision PR);
// iteration i sits at position t = i mod M of its flush block (a chunk holds
// whole blocks, so every chunk ends with a flush).
template <int PR, int NC>
clg_status cgm_chunk(clg_context_s* ctx, CgmWork& W, CgmIter& I, clg_gauge_s* U, int kind, double param, int op,
                     int fp, int np, int64_t Vh, int ns, int chunk) {
  constexpr int MV = cgm_ring(NC);
  CgmState* st = W.st;
  const double2 one = make_double2(1, 0);
  const int* skip = &st->done;
  const FieldRef* tmp = (op == CLG_OP_DDDAG) ? &I.t_full.ref : &I.t_odd.ref;
  for (int i = 0; i < chunk; ++i) {
    const int t = i % MV;
    clg_status e;
    bool fused = false;
    if constexpr (PR != P16 && NC == 3) fused = op == CLG_OP_DDDAG_EE && ctx->fused_cg;
    if (fused) {
      if constexpr (PR != P16 && NC == 3)
        if ((e = cgm_schur_alpha<PR, NC>(ctx, I, U, kind, param, st, t))) return e;
    } else {
      if ((e = apply_op(ctx, op, U, kind, param, I.q.ref, I.p.ref, tmp, one, 1, nullptr, 0, skip, 0))) return e;
      if ((e = launch_sites<1>(ctx, CgmAlpha<PR, NC>{dfield(I.p.ref), dfield(I.q.ref), st, t}, fp, np, Vh, 1)))
        return e;
    }
    if ((e = launch_sites<1>(ctx, CgmR<PR, NC>{dfield(I.ring.ref), dfield(I.q.ref), st, t, MV}, fp, np, Vh, 1)))
      return e;
    if (t + 1 < MV)
      e = launch_sites<0>(ctx, CgmP<PR, NC>{dfield(I.ring.ref), dfield(I.p.ref), st, t + 1}, fp, np, Vh, 1);
    else
      e = launch_sites<0>(
          ctx, CgmFlush<PR, NC, MV>{dfield(I.ring.ref), dfield(W.X.ref), dfield(W.pk.ref), dfield(I.p.ref), st, ns},
          fp, np, Vh, 1);
    if (e) return e;
  }
  return CLG_SUCCESS;
}

// Multi-shift CG on a Hermitian positive operator to the recursive target
// tol for every shift; W.X receives the nshift FP64 solutions.  The shared
// iteration runs in FP64 until |r| <= lo_from |b| and in the inner precision P
// after that (P = FP64: FP64 throughout).  The shifted residuals are
// collinear with the shared one only up to the rounding of the iterations
// that made them, so the early iterations, where |r| is large, are the FP64
// ones.
clg_status cgm_run(clg_context_s* ctx, CgmWork& W, clg_gauge_s* U, int kind, double param, int op, const FieldRef& b,
                   const std::vector<double>& shifts, int P, double tol, double lo_from, int max_iter,
                   int* iters_out) {
  const int nc = W.X.ref.nc, np = b.nparity, fp = b.first_parity;
  const int64_t Vh = b.Vh;
  const int ns = (int)shifts.size();
  clg_status s;
  if ((s = blas_copy(ctx, W.bP.ref, b))) return s;
  CgmState* st = W.st;
  CgmState h;
  std::memset(&h, 0, sizeof(h));
  h.nshift = ns;
  h.tol2 = tol * tol;
  for (int k = 0; k < ns; ++k) h.shift[k] = shifts[k];
  if (cudaMemcpyAsync(st, &h, sizeof(h), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
    return ctx->fail(CLG_ERR_CUDA, "multi-shift: state upload");
  const bool mixed = P != CLG_PREC_DOUBLE;
  return with_pn(P, nc, [&](auto PP, auto NN) -> clg_status {
    constexpr int PV = PP.value, NV = NN.value;
    CgmIter& I64 = W.it[0];
    clg_status e = launch_sites<1>(ctx, CgmInit<P64, NV>{dfield(W.bP.ref), dfield(I64.ring.ref), dfield(I64.p.ref),
                                                          dfield(W.X.ref), dfield(W.pk.ref), st, ns},
                                   fp, np, Vh, 1);
    if (e) return e;
    int phase = 0;  // 0: FP64 iterations, 1: inner precision
    auto to_lo = [&]() -> clg_status {
      phase = 1;
      CgmIter& IL = W.it[1];
      return launch_sites<0>(ctx, CgmSwitch<PV, NV>{dfield(I64.ring.ref), dfield(I64.p.ref), dfield(IL.ring.ref),
                                                    dfield(IL.p.ref)},
                             fp, np, Vh, 1);
    };
    if (mixed && !(lo_from < 1.0) && (e = to_lo())) return e;
    const int chunk = 16;
    int done = 0, it = 0;
    for (int c = 0; c * chunk < max_iter + chunk; ++c) {
      CgmIter& I = W.it[phase];
      auto run = [&]() -> clg_status {
        if (phase == 0) return cgm_chunk<P64, NV>(ctx, W, I, U, kind, param, op, fp, np, Vh, ns, chunk);
        return cgm_chunk<PV, NV>(ctx, W, I, U, kind, param, op, fp, np, Vh, ns, chunk);
      };
      // a phase's first chunk runs eagerly (it tunes the launches); its second
      // captures the chunk, later chunks and calls replay it
      if (!I.exec && I.tuned && ctx->stream) {
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
          const int64_t k0 = ctx->kernels;  // captured launches are counted per replay
          e = run();
          I.graph_kernels = ctx->kernels - k0;
          ctx->kernels = k0;
          if (cudaStreamEndCapture(ctx->stream, &g) == cudaSuccess && g && !e) cudaGraphInstantiate(&I.exec, g, 0);
          if (g) cudaGraphDestroy(g);
          cudaGetLastError();
        }
      }
      if (e) break;
      if (I.exec) {
        if (cudaGraphLaunch(I.exec, ctx->stream) != cudaSuccess) {
          e = ctx->fail(CLG_ERR_CUDA, "multi-shift graph launch");
          break;
        }
        ctx->kernels += I.graph_kernels;
      } else {
        if ((e = run())) break;
        I.tuned = true;
      }
      if (cudaMemcpyAsync(W.hs, st, sizeof(CgmState), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
          cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        e = ctx->fail(CLG_ERR_CUDA, "multi-shift sync");
        break;
      }
      done = W.hs->done;
      it = W.hs->iters;
      if (done || it >= max_iter) break;
      if (mixed && phase == 0 && W.hs->rr <= lo_from * lo_from * W.hs->bb && (e = to_lo())) break;
    }
    *iters_out = it;
    return e;
  });
}

}  // namespace
}  // namespace clg

using namespace clg;

extern "C" {

clg_status clg_solve_multishift(clg_solver S, clg_field* x, int nshift, const double* shifts, clg_field b, clg_gauge g,
                                int op, clg_solve_info* info) {
  if (!S || !x || !b || !g || !shifts || !info || nshift < 1) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = S->ctx;
  if (nshift > CGM_MAXSHIFT) return ctx->fail(CLG_ERR_UNSUPPORTED, "at most 64 shifts");
  if (b->nrhs != 1) return ctx->fail(CLG_ERR_BAD_ARG, "multi-shift solves take one right-hand side");
  for (int k = 0; k < nshift; ++k) {
    if (!x[k] || x[k]->lat != b->lat || x[k]->kind != b->kind || x[k]->subset != b->subset || x[k]->nrhs != 1)
      return ctx->fail(CLG_ERR_BAD_ARG, "multi-shift: solution fields must match b");
    if (x[k]->data == b->data) return ctx->fail(CLG_ERR_BAD_ARG, "multi-shift: x must not alias b (CMultiShiftSolver.h:35)");
  }
  if (clg_status st = settle(b)) return st;
  for (int k = 0; k < nshift; ++k)
    if (clg_status st = settle(x[k])) return st;
  if (S->p.kind != CLG_SOLVER_CGM && S->p.kind != CLG_SOLVER_FOM_MS && S->p.kind != CLG_SOLVER_NESTED_MS &&
      S->p.kind != CLG_SOLVER_BICGSTAB_MS && S->p.kind != CLG_SOLVER_GMRES_MS)
    return ctx->fail(CLG_ERR_BAD_ARG,
                     "clg_solve_multishift needs a CGM, FOM_MS, GMRES_MS, BICGSTAB_MS or NESTED_MS solver");
  std::vector<double2> sh(nshift);
  for (int k = 0; k < nshift; ++k) sh[k] = make_double2(shifts[2 * k], shifts[2 * k + 1]);
  const bool hermitian = op == CLG_OP_DDDAG || op == CLG_OP_DDDAG_EE || op == CLG_OP_MEE_MEEDAG;
  // CG needs op + c_n Hermitian positive: real shifts >= 0 (complex shifts take GMRES)
  bool real_nonneg = true;
  for (int k = 0; k < nshift; ++k) real_nonneg = real_nonneg && sh[k].y == 0.0 && sh[k].x >= 0.0;
  clg_solver_params prm = S->p;
  clg_status s = CLG_SUCCESS;
  const int P = prm.inner_precision;
  const int nc = b->nc();
  const int64_t Vh = b->lat->g.Vh;
  CgmWork* W = nullptr;
  int cgm_iters = 0;
  const FieldRef* fom_x = nullptr;
  int fom_apps = 0, fom_cycles = 0;
  const bool use_cgm = S->p.kind == CLG_SOLVER_CGM;
  if (use_cgm) {
    if (!hermitian) return ctx->fail(CLG_ERR_BAD_ARG, "CG-M needs a Hermitian positive operator (DDdagger forms)");
    std::vector<double> real(nshift);
    for (int k = 0; k < nshift; ++k) {
      if (sh[k].y != 0.0 || sh[k].x < 0.0) return ctx->fail(CLG_ERR_BAD_ARG, "CG-M shifts must be real and >= 0");
      real[k] = sh[k].x;
    }
    if ((s = gauge_prepare(g, P))) return s;
    const L2LinkWindow l2(ctx, g, P);
    if (op == CLG_OP_MEE_MEEDAG) return ctx->fail(CLG_ERR_UNSUPPORTED, "CG-M on MEE_MEEDAG: use FOM_MS");
    // workspace reused while lattice, kind, parity layout, precision, shift
    // count, operator and the gauge arrays stay the same
    const std::string key = std::to_string((uintptr_t)b->lat) + "/" + std::to_string(b->kind) + "/" +
                            std::to_string(b->subset) + "/" + std::to_string(P) + "/" + std::to_string(nshift) + "/" +
                            std::to_string(op) + "/" + std::to_string((uintptr_t)g) + "/" +
                            std::to_string((uintptr_t)g->u64[0]) + "/" + std::to_string((uintptr_t)g->u32[0]) + "/" +
                            std::to_string((uintptr_t)g->u16[0]) + "/" + std::to_string(b->param);
    W = dynamic_cast<CgmWork*>(S->cache_cgm.get());
    if (!W || W->key != key) {
      cudaStreamSynchronize(ctx->stream);
      S->cache_cgm.reset();
      W = new CgmWork();
      S->cache_cgm.reset(W);
      if ((s = W->alloc(ctx, P, nc, b->nparity(), 0, nshift, Vh, op))) {
        S->cache_cgm.reset();
        return s;
      }
      W->key = key;
    }
    // every shift to half the FP64 tolerance in the shared iteration; a
    // mixed solve leaves FP64 once |r| <= inner_tol |b|
    if ((s = cgm_run(ctx, *W, g, b->kind, b->param, op, b->ref(), real, P, prm.tol_true_rel * 0.5, prm.inner_tol,
                     prm.max_iterations, &cgm_iters)))
      return s;
    prm.kind = CLG_SOLVER_CG;  // per-shift refinement
  } else if (S->p.kind == CLG_SOLVER_FOM_MS || S->p.kind == CLG_SOLVER_BICGSTAB_MS ||
             S->p.kind == CLG_SOLVER_GMRES_MS) {
    if (b->prec != CLG_PREC_DOUBLE)
      return ctx->fail(CLG_ERR_BAD_ARG, "multi-shift FOM / BiCGStab work on FP64 fields");
    for (int k = 0; k < nshift; ++k)
      if (x[k]->prec != CLG_PREC_DOUBLE)
        return ctx->fail(CLG_ERR_BAD_ARG, "multi-shift FOM / BiCGStab work on FP64 fields");
    if ((s = gauge_prepare(g, CLG_PREC_DOUBLE))) return s;
    if (S->p.kind == CLG_SOLVER_FOM_MS)
      s = fom_ms_run(ctx, S->cache_fom, g, b->kind, b->param, op, b->ref(), sh, prm.max_dim, prm.restart,
                     prm.tol_true_rel * 0.5, &fom_x, &fom_apps, &fom_cycles);
    else if (S->p.kind == CLG_SOLVER_GMRES_MS)
      s = gmres_ms_run(ctx, S->cache_fom, g, b->kind, b->param, op, b->ref(), sh, prm.max_dim, prm.restart,
                       prm.tol_true_rel * 0.5, &fom_x, &fom_apps, &fom_cycles);
    else
      s = bicgstab_ms_run(ctx, S->cache_fom, g, b->kind, b->param, op, b->ref(), sh, std::max(1, prm.deviation_step),
                          std::max(1, prm.max_step), prm.tol_true_rel * 0.5, &fom_x, &fom_apps, &fom_cycles);
    if (s) return s;
    // the FP64 check / refinement of every shift (GMRES at most 16 deep on the device)
    prm.kind = hermitian && real_nonneg ? CLG_SOLVER_CG : CLG_SOLVER_GMRES;
    prm.max_dim = std::min(prm.max_dim, (int)GM_MAXK);
  } else {
    prm.kind = hermitian && real_nonneg ? CLG_SOLVER_CG : CLG_SOLVER_GMRES;
  }
  SolveReq q;
  q.cache = &S->cache_shift;
  q.ctx = ctx;
  q.prm = &prm;
  q.U = g;
  q.lat = b->lat;
  q.kind = b->kind;
  q.param = b->param;
  q.op = op;
  q.subset = b->subset;
  q.nrhs = nshift;
  q.b = b->ref();
  q.b_broadcast = true;
  if (use_cgm) q.x0 = &W->X.ref;
  if (fom_x) q.x0 = fom_x;
  q.shifts = sh.data();
  for (int k = 0; k < nshift; ++k) q.xout.push_back(x[k]->ref());
  q.info = info;
  s = solve_core(q);
  for (int k = 0; k < nshift; ++k) {
    info[k].iterations += cgm_iters + fom_apps;
    info[k].restarts += fom_cycles;
  }
  return s;
}

clg_status clg_rational_apply(clg_solver S, clg_field f, clg_gauge g, int op, int degree, double c, const double* a,
                              const double* bsh, clg_solve_info* info) {
  if (!S || !f || !g || !a || !bsh || !info || degree < 1) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = S->ctx;
  if (f->nrhs != 1) return ctx->fail(CLG_ERR_BAD_ARG, "rational approximation acts on one field");
  if (clg_status st = settle(f)) return st;
  std::vector<clg_field> xs(degree, nullptr);
  clg_status s = CLG_SUCCESS;
  for (int i = 0; i < degree && !s; ++i) s = clg_field_create(f->lat, f->kind, f->subset, f->prec, 1, f->param, &xs[i]);
  std::vector<double> sh(2 * degree, 0.0);
  for (int i = 0; i < degree; ++i) sh[2 * i] = bsh[i];
  if (!s) s = clg_solve_multishift(S, xs.data(), degree, sh.data(), f, g, op, info);
  // f <- c f + sum_i a_i x_i   (CField.cpp:140-146)
  if (!s || s == CLG_ERR_NOT_CONVERGED) {
    clg_status t = blas_axpby(ctx, f->ref(), make_double2(0, 0), f->ref(), make_double2(c, 0));
    for (int i = 0; i < degree && !t; ++i) t = blas_axpby(ctx, f->ref(), make_double2(a[i], 0), xs[i]->ref(), make_double2(1, 0));
    if (t) s = t;
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess && !s) s = ctx->fail(CLG_ERR_CUDA, "rational sync");
  }
  for (auto x : xs)
    if (x) clg_field_destroy(x);
  return s;
}

}  // extern "C"
