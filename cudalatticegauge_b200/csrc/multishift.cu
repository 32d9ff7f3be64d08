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

struct CgmState {
  double rr, bb, tol2, alpha, alpha_old, beta, pq;
  int iters, done, nshift, pad;
  double shift[CGM_MAXSHIFT];
  double zeta[CGM_MAXSHIFT], zeta_old[CGM_MAXSHIFT], zeta_new[CGM_MAXSHIFT];
  double alpha_k[CGM_MAXSHIFT], beta_k[CGM_MAXSHIFT];
  int active[CGM_MAXSHIFT];
  int upd_x[CGM_MAXSHIFT];  // x_k takes alpha_k p_k in this iteration (active when alpha_k was formed)
};

namespace {

// (p, q) -> alpha and the shifted alpha_k (Jegerlehner eq. for zeta_{n+1})
template <int P, int NC>
struct CgmAlpha {
  DField p, q;
  CgmState* st;
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
  __device__ void finalize(int, const double* s) const {
    CgmState& c = *st;
    // runs on every replayed iteration, also once all shifts are done, so a
    // finished solve never repeats its last x update
    for (int k = 0; k < c.nshift; ++k) c.upd_x[k] = 0;
    if (c.done) return;
    c.iters += 1;
    if (!(s[0] > 0.0) || bad(s[0])) {
      c.done = 2;
      return;
    }
    const double alpha = c.rr / s[0];
    for (int k = 0; k < c.nshift; ++k) {
      c.upd_x[k] = c.active[k];
      if (!c.active[k]) continue;
      const double zn = c.zeta[k], zo = c.zeta_old[k];
      const double den = alpha * c.beta * (zo - zn) + zo * c.alpha_old * (1.0 + c.shift[k] * alpha);
      const double znew = zn * zo * c.alpha_old / den;
      c.zeta_new[k] = znew;
      c.alpha_k[k] = alpha * znew / zn;
    }
    c.alpha = alpha;
  }
};

// r -= alpha q ; |r|^2 -> beta, beta_k, convergence per shift
template <int P, int NC>
struct CgmR {
  DField r, q;
  CgmState* st;
  __device__ bool active(int) const { return !st->done; }
  __device__ void operator()(int, int par, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> vr[NC], vq[NC];
    ldv<P, NC, AT>(r, 0, par, h, vr);
    ldv<P, NC, AT>(q, 0, par, h, vq);
    const AT a = (AT)st->alpha;
#pragma unroll
    for (int i = 0; i < NC; ++i) vr[i] = vr[i] - a * vq[i];
    stv<P, NC, AT>(r, 0, par, h, vr);
    acc[0] += site_norm2<NC, AT>(vr);
  }
  __device__ void finalize(int, const double* s) const {
    CgmState& c = *st;
    if (c.done) return;
    if (bad(s[0])) {
      c.done = 2;
      return;
    }
    const double beta = s[0] / c.rr;
    int nact = 0;
    for (int k = 0; k < c.nshift; ++k) {
      if (!c.active[k]) continue;
      const double ratio = c.zeta_new[k] / c.zeta[k];
      c.beta_k[k] = beta * ratio * ratio;
      c.zeta_old[k] = c.zeta[k];
      c.zeta[k] = c.zeta_new[k];
      if (c.zeta[k] * c.zeta[k] * s[0] <= c.tol2 * c.bb)
        c.active[k] = 0;
      else
        ++nact;
    }
    c.alpha_old = c.alpha;
    c.beta = beta;
    c.rr = s[0];
    if (nact == 0) c.done = 1;
  }
};

// One pass after the residual update, grid.y = nshift + 1:
//   shift k < nshift:  x_k += alpha_k p_k ; p_k = zeta_k r + beta_k p_k
//                      (both from the same, old p_k: the x update of the
//                      shift loop deferred past r's update, as the algebra allows)
//   y = nshift:        p = r + beta p
template <int P, int NC>
struct CgmUpdate {
  DField x, pk, p, r;
  CgmState* st;
  int nshift;
  __device__ bool active(int k) const {
    if (k == nshift) return !st->done;
    return st->upd_x[k] || (!st->done && st->active[k]);
  }
  __device__ void operator()(int k, int par, int64_t h, double*) const {
    using AT = typename AccT<P>::T;
    cpx<AT> vp[NC], vr[NC];
    ldv<P, NC, AT>(r, 0, par, h, vr);
    if (k == nshift) {
      ldv<P, NC, AT>(p, 0, par, h, vp);
      const AT b = (AT)st->beta;
#pragma unroll
      for (int i = 0; i < NC; ++i) vp[i] = vr[i] + b * vp[i];
      stv<P, NC, AT>(p, 0, par, h, vp);
      return;
    }
    ldv<P, NC, AT>(pk, k, par, h, vp);
    if (st->upd_x[k]) {
      cpx<AT> vx[NC];
      ldv<P, NC, AT>(x, k, par, h, vx);
      const AT a = (AT)st->alpha_k[k];
#pragma unroll
      for (int i = 0; i < NC; ++i) vx[i] = vx[i] + a * vp[i];
      stv<P, NC, AT>(x, k, par, h, vx);
    }
    if (!st->done && st->active[k]) {
      const AT z = (AT)st->zeta[k], b = (AT)st->beta_k[k];
#pragma unroll
      for (int i = 0; i < NC; ++i) vp[i] = z * vr[i] + b * vp[i];
      stv<P, NC, AT>(pk, k, par, h, vp);
    }
  }
  __device__ void finalize(int, const double*) const {}
};

// start: r = p = b, x_k = 0, p_k = b, |b|^2
template <int P, int NC>
struct CgmInit {
  DField b, r, p, x, pk;
  CgmState* st;
  int nshift;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int, int par, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> vb[NC], z[NC];
    ldv<P, NC, AT>(b, 0, par, h, vb);
#pragma unroll
    for (int i = 0; i < NC; ++i) z[i] = mk<AT>(0, 0);
    stv<P, NC, AT>(r, 0, par, h, vb);
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
    c.done = s[0] > 0.0 ? 0 : 1;
    for (int k = 0; k < c.nshift; ++k) {
      c.zeta[k] = c.zeta_old[k] = 1.0;
      c.active[k] = c.done ? 0 : 1;
      c.upd_x[k] = 0;
    }
  }
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

// Buffers, device state, pinned summary and the captured iteration graph of a
// multi-shift CG, kept in the solver between calls with the same shape and
// gauge arrays (a call then costs the solve, not cudaMalloc/cudaFree, pinned
// allocations and a graph capture).
struct CgmWork : SolveCacheBase {
  std::string key;
  OwnedF X, bP, r, p, q, pk, t_odd, t_full;
  CgmState* st = nullptr;
  CgmState* hs = nullptr;  // pinned copy read per chunk
  cudaGraphExec_t exec = nullptr;
  int64_t graph_kernels = 0;
  ~CgmWork() {
    if (exec) cudaGraphExecDestroy(exec);
    dfree(st);
    if (hs) cudaFreeHost(hs);
  }
  clg_status alloc(clg_context_s* ctx, int P, int nc, int np, int fp, int ns, int64_t Vh, int op) {
    clg_status s;
    if ((s = X.alloc(ctx, P, nc, np, fp, ns, Vh)) || (s = bP.alloc(ctx, P, nc, np, fp, 1, Vh)) ||
        (s = r.alloc(ctx, P, nc, np, fp, 1, Vh)) || (s = p.alloc(ctx, P, nc, np, fp, 1, Vh)) ||
        (s = q.alloc(ctx, P, nc, np, fp, 1, Vh)) || (s = pk.alloc(ctx, P, nc, np, fp, ns, Vh)) ||
        (s = t_odd.alloc(ctx, P, nc, 1, 1, 1, Vh)))
      return s;
    if (op == CLG_OP_DDDAG && (s = t_full.alloc(ctx, P, nc, 2, 0, 1, Vh))) return s;
    if ((s = dalloc(ctx, (void**)&st, sizeof(CgmState)))) return s;
    if (cudaMallocHost((void**)&hs, sizeof(CgmState)) != cudaSuccess) {
      hs = nullptr;
      return ctx->fail(CLG_ERR_OOM, "multi-shift: pinned state");
    }
    return CLG_SUCCESS;
  }
};

// Multi-shift CG in precision P on a Hermitian positive operator; W.X receives
// the nshift solutions.
clg_status cgm_run(clg_context_s* ctx, CgmWork& W, clg_gauge_s* U, int kind, double param, int op, const FieldRef& b,
                   const std::vector<double>& shifts, double tol, int max_iter, int* iters_out) {
  const FieldRef& X = W.X.ref;
  const int P = X.prec, nc = X.nc, np = b.nparity, fp = b.first_parity;
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
  const double2 one = make_double2(1, 0);
  const int* skip = &st->done;
  return with_pn(P, nc, [&](auto PP, auto NN) -> clg_status {
    constexpr int PV = PP.value, NV = NN.value;
    clg_status e = launch_sites<1>(ctx, CgmInit<PV, NV>{dfield(W.bP.ref), dfield(W.r.ref), dfield(W.p.ref), dfield(X),
                                                         dfield(W.pk.ref), st, ns},
                                   fp, np, Vh, 1);
    if (e) return e;
    const int chunk = 16;
    auto body = [&]() -> clg_status {
      clg_status e2;
      const FieldRef* tmp = (op == CLG_OP_DDDAG) ? &W.t_full.ref : &W.t_odd.ref;
      if ((e2 = apply_op(ctx, op, U, kind, param, W.q.ref, W.p.ref, tmp, one, 1, nullptr, 0, skip, 0))) return e2;
      if ((e2 = launch_sites<1>(ctx, CgmAlpha<PV, NV>{dfield(W.p.ref), dfield(W.q.ref), st}, fp, np, Vh, 1))) return e2;
      if ((e2 = launch_sites<1>(ctx, CgmR<PV, NV>{dfield(W.r.ref), dfield(W.q.ref), st}, fp, np, Vh, 1))) return e2;
      CgmUpdate<PV, NV> up{dfield(X), dfield(W.pk.ref), dfield(W.p.ref), dfield(W.r.ref), st, ns};
      return launch_sites<0>(ctx, up, fp, np, Vh, ns + 1);
    };
    int done = 0, it = 0;
    e = CLG_SUCCESS;
    for (int c = 0; c * chunk < max_iter + chunk; ++c) {
      // the first chunk of the first call runs eagerly (it tunes the launches);
      // the second captures the chunk, later chunks and calls replay it
      if (c == 1 && !W.exec && ctx->stream) {
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
          const int64_t k0 = ctx->kernels;  // captured launches are counted per replay
          for (int i = 0; i < chunk && !e; ++i) e = body();
          W.graph_kernels = ctx->kernels - k0;
          ctx->kernels = k0;
          if (cudaStreamEndCapture(ctx->stream, &g) == cudaSuccess && g && !e) cudaGraphInstantiate(&W.exec, g, 0);
          if (g) cudaGraphDestroy(g);
          cudaGetLastError();
        }
      }
      if (e) break;
      if (W.exec) {
        if (cudaGraphLaunch(W.exec, ctx->stream) != cudaSuccess) {
          e = ctx->fail(CLG_ERR_CUDA, "multi-shift graph launch");
          break;
        }
        ctx->kernels += W.graph_kernels;
      } else {
        for (int i = 0; i < chunk && !e; ++i) e = body();
        if (e) break;
      }
      if (cudaMemcpyAsync(W.hs, st, sizeof(CgmState), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
          cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        e = ctx->fail(CLG_ERR_CUDA, "multi-shift sync");
        break;
      }
      done = W.hs->done;
      it = W.hs->iters;
      if (done || it >= max_iter) break;
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
    // recursive-residual target of the multi-shift phase: the FP64 tolerance
    // itself in FP64; inner_tol (floored where the precision's recurrences
    // stop tracking the true residual) in FP32 / FP16
    const double itol = P == CLG_PREC_DOUBLE ? prm.tol_true_rel * 0.5
                                             : std::max(prm.inner_tol, P == CLG_PREC_SINGLE ? 1e-9 : 1e-4);
    if ((s = cgm_run(ctx, *W, g, b->kind, b->param, op, b->ref(), real, itol, prm.max_iterations, &cgm_iters)))
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
