// gcrodr.cu -- GCRO-DR: GMRES with deflated restarting and a recycled
// subspace kept between solves (CSLASolverGCRODR,
// SparseLinearAlgebra/CSolverGCRODR.cpp:196-911; Parks, de Sturler, Mackey,
// Johnson & Maiti, SIAM J. Sci. Comput. 28 (2006) 1651).
//
// Each cycle works in [U_k, V_{m-k}] with A U_k = C_k, C_k^+ C_k = 1 and the
// Arnoldi vectors V orthogonal to C_k, so that
//   A [U_k, V_{m-k}] = [C_k, V_{m-k+1}] G,  G = [[D_k, B], [0, Hbar]]
// (D_k the norms that make U_k unit vectors).  The correction minimises the
// residual over that space; then k vectors of the cycle's space become the
// next U_k (the deflation space: the reference's default EEDT_SVD, the k
// smallest eigenpairs of G^+ G p = l blockdiag(U^+ U, 1) p; or EEDT_REV Ritz
// or EEDT_HEV harmonic Ritz vectors, clg_deflation):
//   U_k = [U_k, V] P R^-1, C_k = [C_k, V] Q with G P = Q R.
// The first solve starts with one GMRES(m) cycle whose Hbar gives the first
// U_k; later solves (the same operator, e.g. successive molecular-dynamics
// steps or right-hand sides) start from the kept U_k: C_k = A U_k, QR,
// U_k R^-1 (GenerateCUFirstTime).  clg_solver_reset drops U_k (the
// reference's start of a trajectory).
//
// B200 form: FP64 vectors on the device, one right-hand side; every
// orthogonalisation is one multi-dot launch (up to 16 inner products per
// pass, classical Gram-Schmidt applied twice) and one linear-combination
// launch, so a cycle costs (m - k) operator applications, one explicit
// residual b - A x (the reference's RecalculateR option, which it calls "the
// accurate result") and O(m) small launches with one host read each.  The
// small dense problems (least squares, QR, generalized eigenproblem, order
// <= 33) run on the host (dense.h); the reference runs them on the device.
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "hostkrylov.cuh"

namespace clg {

namespace {

using dense::Mat;
using dense::Z;
using hk::MD;
using hk::MAXV;

// the recycled subspace and the per-solve vectors, kept by the solver
struct GcroWork : hk::HostVecs {
  const void* lat = nullptr;
  int kind = -1, subset = -1, op = -1, m = 0, k = 0;
  std::vector<FieldRef> U, C, V, Tu, Tc;
  FieldRef x, r, w, t;
  bool u_valid = false;
};

struct Gcro : hk::HostKrylov {
  GcroWork& G;
  Gcro(clg_context_s* c, GcroWork& w, const clg_gauge_s* u, int kd, int o, int n, double prm, int64_t vh)
      : hk::HostKrylov{c, w, u, kd, o, n, prm, vh}, G(w) {}
  // r = b - A x
  clg_status residual(const FieldRef& b, const FieldRef& x, const FieldRef& r) {
    if (clg_status st = apply(G.t, x)) return st;
    return lincomb(r, Z(0.0, 0.0), {&b, &G.t}, {Z(1.0, 0.0), Z(-1.0, 0.0)});
  }
  // U = T R^-1 for upper triangular R (k x k) (FieldSolveY, CSolverGCRODR.cpp:763-780)
  clg_status solve_r(std::vector<FieldRef>& T, const Mat& R, int k) {
    for (int i = 0; i < k; ++i) {
      std::vector<const FieldRef*> vs;
      std::vector<Z> c;
      for (int j = 0; j < i; ++j) {
        vs.push_back(&T[j]);
        c.push_back(-R(j, i) / R(i, i));
      }
      if (clg_status st = lincomb(T[i], Z(1.0, 0.0) / R(i, i), vs, c)) return st;
    }
    return CLG_SUCCESS;
  }
};

double now_s() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

}  // namespace

clg_status gcrodr_solve(::clg_solver_s* S, clg_field_s* X, clg_field_s* B, clg_gauge_s* Ug, int op, clg_field_s* X0,
                        clg_solve_info* info) {
  clg_context_s* ctx = S->ctx;
  const double t0 = now_s();
  if (B->nrhs != 1) return ctx->fail(CLG_ERR_UNSUPPORTED, "GCRO-DR solves one right-hand side at a time");
  if (B->prec != CLG_PREC_DOUBLE || X->prec != CLG_PREC_DOUBLE || (X0 && X0->prec != CLG_PREC_DOUBLE))
    return ctx->fail(CLG_ERR_BAD_ARG, "GCRO-DR works on FP64 fields");
  const bool even = B->subset == CLG_SUBSET_EVEN;
  const bool even_op = op == CLG_OP_MEE || op == CLG_OP_MEE_DAG || op == CLG_OP_MEE_MEEDAG || op == CLG_OP_DDDAG_EE;
  const bool full_op = op == CLG_OP_D || op == CLG_OP_DDAG || op == CLG_OP_DDDAG || op == CLG_OP_DD;
  if (!(even ? even_op : full_op)) return ctx->fail(CLG_ERR_BAD_ARG, "GCRO-DR: operator and field subset do not match");
  if (clg_status st = gauge_prepare(Ug, CLG_PREC_DOUBLE)) return st;
  const int m = S->p.max_dim, k = S->p.kdim > 0 ? S->p.kdim : S->p.max_dim - 2;
  const int defl = S->p.deflation;
  const bool mdr = S->p.kind == CLG_SOLVER_GMRESMDR;

  // workspace (and the recycled U_k) for this lattice / operator / sizes
  auto* Wp = dynamic_cast<GcroWork*>(S->cache_gcro.get());
  if (!Wp || Wp->lat != B->lat || Wp->kind != B->kind || Wp->subset != B->subset || Wp->op != op || Wp->m != m ||
      Wp->k != k) {
    S->cache_gcro.reset();
    auto nw = std::make_unique<GcroWork>();
    nw->ctx = ctx;
    nw->proto = B->ref();
    nw->lat = B->lat;
    nw->kind = B->kind;
    nw->subset = B->subset;
    nw->op = op;
    nw->m = m;
    nw->k = k;
    clg_status st = CLG_SUCCESS;
    nw->U.resize(k);
    nw->C.resize(k);
    nw->Tu.resize(k);
    nw->Tc.resize(k);
    nw->V.resize(m - k + 1);
    for (auto* vv : {&nw->U, &nw->C, &nw->Tu, &nw->Tc, &nw->V})
      for (FieldRef& f : *vv)
        if (!st) st = nw->vec(f);
    for (FieldRef* f : {&nw->x, &nw->r, &nw->w, &nw->t})
      if (!st) st = nw->vec(*f);
    if (!st) {  // the operator's temporary: a full field
      FieldRef full = nw->proto;
      full.nparity = 2;
      full.first_parity = 0;
      full.rstride = full.blk * 2;
      nw->proto = full;
      st = nw->vec(nw->tmp);
      nw->proto = B->ref();
    }
    if (!st) {
      void* p = nullptr;
      st = dalloc(ctx, &p, sizeof(double) * 2 * MD);
      if (!st) {
        nw->allocs.push_back(p);
        nw->dev_out = static_cast<double*>(p);
      }
    }
    if (st) return st;
    Wp = nw.get();
    S->cache_gcro = std::move(nw);
  }
  GcroWork& W = *Wp;
  for (clg_field f : {X, B, X0})
    if (f)
      if (clg_status st = settle(f)) return st;
  Gcro g{ctx, W, Ug, B->kind, op, B->nc(), B->param, B->lat->g.Vh};
  const FieldRef b = B->ref();
  const double tol = S->p.tol_true_rel;
  clg_status st = CLG_SUCCESS;
  std::memset(info, 0, sizeof(*info));

  const double bnorm = g.norm(b);
  if (bnorm < 0) return ctx->fail(CLG_ERR_CUDA, "GCRO-DR: reading |b|");
  // x0 = the start vector, or b (CSolverGCRODR.cpp:216-223)
  if ((st = g.copy(W.x, X0 ? X0->ref() : b))) return st;
  if (bnorm == 0.0) {
    if ((st = g.copy(X->ref(), b))) return st;
    info->true_rel_residual = 0.0;
    info->seconds = now_s() - t0;
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? CLG_SUCCESS : ctx->fail(cuda_status(e), cudaGetErrorString(e));
  }

  auto Wvec = [&](int j) -> FieldRef& { return j < k ? W.C[j] : W.V[j - k]; };  // GetW
  double rnorm = 0.0;
  int cycles = 0;
  auto finish = [&](clg_status s) -> clg_status {
    // the true residual before x is written (X may alias B)
    if (!s) s = g.residual(b, W.x, W.r);
    const double tr = s ? -1.0 : g.norm(W.r) / bnorm;
    if (!s) s = g.copy(X->ref(), W.x);
    info->iterations = g.apps;
    info->restarts = cycles;
    info->outer = 1;
    info->true_rel_residual = tr;
    info->seconds = now_s() - t0;
    if (!s && !(tr <= tol)) s = CLG_ERR_NOT_CONVERGED;
    info->status = s;
    if (tr < 0) info->true_rel_residual = NAN;
    return s;
  };

  bool c_ready = false;  // C = A U already (the GMRES-MDR start)
  if (W.u_valid && mdr) {
    // GMRES-MDR's start (CSLASolverGMRESMDR::GenerateCUFirstTime,
    // CSolverGMRESMDR.cpp:16-135): Q R = U (QRFactorizationOfUk, :140-170),
    // C = A Q, the k x k problem of the deflation type on span Q (REV: Q^+ A Q;
    // HEV: Q^+ A^+ A Q p = l Q^+ A^+ Q p; SVD: Q^+ A^+ A Q), U = Q P.  The
    // reference leaves C = A Q there, which breaks A U = C for the cycles that
    // follow; here C = A Q P (no extra application) and the QR below makes it
    // orthonormal with U rescaled to match, as the recycled start requires.
    for (int i = 0; i < k && W.u_valid; ++i) {
      std::vector<const FieldRef*> prev;
      for (int j = 0; j < i; ++j) prev.push_back(&W.U[j]);
      std::vector<Z> h;
      if (i && (st = g.orthogonalise(W.U[i], prev, h))) return finish(st);
      const double n = g.norm(W.U[i]);
      if (!(n > 0)) W.u_valid = false;
      else if ((st = g.scale(W.U[i], Z(1.0 / n, 0.0)))) return finish(st);
    }
    if (W.u_valid) {
      for (int i = 0; i < k; ++i)
        if ((st = g.apply(W.C[i], W.U[i]))) return finish(st);
      Mat M(k, k), B(k, k);
      for (int j = 0; j < k; ++j) {
        std::vector<const FieldRef*> vs;
        for (int i = 0; i < k; ++i) vs.push_back(defl == CLG_DEFLATION_REV ? &W.U[i] : &W.C[i]);
        std::vector<Z> d;
        if ((st = g.dots(W.C[j], vs, d))) return finish(st);  // d[i] = <v_i, C_j>
        for (int i = 0; i < k; ++i) M(i, j) = d[i];
        if (defl == CLG_DEFLATION_HEV) {
          std::vector<Z> e;
          std::vector<const FieldRef*> cs;
          for (int i = 0; i < k; ++i) cs.push_back(&W.C[i]);
          if ((st = g.dots(W.U[j], cs, e))) return finish(st);  // <C_i, Q_j>
          for (int i = 0; i < k; ++i) B(i, j) = e[i];
        }
      }
      std::vector<Z> ev;
      Mat P;
      const bool ok = defl == CLG_DEFLATION_HEV ? dense::geig(M, B, ev, P) : dense::eig(M, ev, P);
      if (ok) {
        // U = Q P, C = (A Q) P through the Tu / Tc scratch vectors
        for (int j = 0; j < k; ++j) {
          std::vector<const FieldRef*> qs, cs;
          std::vector<Z> c;
          for (int i = 0; i < k; ++i) {
            qs.push_back(&W.U[i]);
            cs.push_back(&W.C[i]);
            c.push_back(P(i, j));
          }
          if ((st = g.lincomb(W.Tu[j], Z(0.0, 0.0), qs, c)) || (st = g.lincomb(W.Tc[j], Z(0.0, 0.0), cs, c)))
            return finish(st);
        }
        for (int j = 0; j < k; ++j)
          if ((st = g.copy(W.U[j], W.Tu[j])) || (st = g.copy(W.C[j], W.Tc[j]))) return finish(st);
      }
      c_ready = true;
    }
  }
  if (W.u_valid) {
    // C = A U, QR, U = U R^-1 (GenerateCUFirstTime / QRFactorAY, CSolverGCRODR.cpp:501-539, 817-841)
    Mat R(k, k);
    for (int i = 0; i < k && !c_ready; ++i)
      if ((st = g.apply(W.C[i], W.U[i]))) return finish(st);
    for (int i = 0; i < k; ++i) {
      std::vector<const FieldRef*> prev;
      for (int j = 0; j < i; ++j) prev.push_back(&W.C[j]);
      std::vector<Z> h;
      if (i && (st = g.orthogonalise(W.C[i], prev, h))) return finish(st);
      for (int j = 0; j < i; ++j) R(j, i) = h[j];
      const double n = g.norm(W.C[i]);
      if (!(n > 0)) {
        W.u_valid = false;
        break;
      }
      R(i, i) = n;
      if ((st = g.scale(W.C[i], Z(1.0 / n, 0.0)))) return finish(st);
    }
    if (W.u_valid && (st = g.solve_r(W.U, R, k))) return finish(st);
  }
  if ((st = g.residual(b, W.x, W.r))) return finish(st);
  rnorm = g.norm(W.r);

  if (!W.u_valid) {
    // one GMRES(m) cycle (FirstTimeGMERESSolve, :400-499), its Hbar gives the first U_k
    const double beta = rnorm;
    if (beta <= tol * bnorm) return finish(CLG_SUCCESS);
    if ((st = g.lincomb(Wvec(0), Z(0.0, 0.0), {&W.r}, {Z(1.0 / beta, 0.0)}))) return finish(st);
    Mat H(m + 1, m);
    int mm = m;
    for (int j = 0; j < m; ++j) {
      if ((st = g.apply(Wvec(j + 1), Wvec(j)))) return finish(st);
      std::vector<const FieldRef*> vs;
      for (int l = 0; l <= j; ++l) vs.push_back(&Wvec(l));
      std::vector<Z> h;
      if ((st = g.orthogonalise(Wvec(j + 1), vs, h))) return finish(st);
      for (int l = 0; l <= j; ++l) H(l, j) = h[l];
      const double hn = g.norm(Wvec(j + 1));
      H(j + 1, j) = hn;
      if (!(hn > 1e-14 * beta)) {  // invariant subspace: the solution is in span(W_0..W_j)
        mm = j + 1;
        break;
      }
      if ((st = g.scale(Wvec(j + 1), Z(1.0 / hn, 0.0)))) return finish(st);
    }
    Mat Hs(mm + 1, mm);
    for (int i = 0; i <= mm; ++i)
      for (int j = 0; j < mm; ++j) Hs(i, j) = H(i, j);
    std::vector<Z> c(mm + 1, Z(0.0, 0.0)), y;
    c[0] = beta;
    if (!dense::lstsq(Hs, c, y)) return finish(ctx->fail(CLG_ERR_BREAKDOWN, "GCRO-DR: least squares"));
    {
      std::vector<const FieldRef*> vs;
      for (int j = 0; j < mm; ++j) vs.push_back(&Wvec(j));
      if ((st = g.lincomb(W.x, Z(1.0, 0.0), vs, y))) return finish(st);
    }
    if ((st = g.residual(b, W.x, W.r))) return finish(st);
    rnorm = g.norm(W.r);
    cycles = 1;
    if (mm == m) {
      // FindPk1 (:541-570): SVD the k smallest eigenpairs of Hbar^+ Hbar; REV
      // the k smallest of the square H_m; HEV the k largest of H_m p = l Hbar^+ Hbar p
      std::vector<Z> ev;
      Mat X;
      Mat Hm(m, m);
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) Hm(i, j) = H(i, j);
      bool ok;
      if (defl == CLG_DEFLATION_REV) ok = dense::eig(Hm, ev, X);
      else if (defl == CLG_DEFLATION_HEV) ok = dense::geig(Hm, dense::mul_dag(H, H), ev, X);
      else ok = dense::eig(dense::mul_dag(H, H), ev, X);
      if (ok) {
        const Mat P = dense::select(ev, X, k, defl != CLG_DEFLATION_HEV);
        Mat Q, R;
        if (dense::qr_thin(dense::mul(H, P), Q, R)) {
          // GenerateCU right after GMRES: U = W_m P R^-1, C = W_{m+1} Q
          std::vector<const FieldRef*> wm, wm1;
          for (int j = 0; j < m; ++j) wm.push_back(&Wvec(j));
          for (int j = 0; j <= m; ++j) wm1.push_back(&Wvec(j));
          for (int j = 0; j < k && !st; ++j) {
            std::vector<Z> cp(m), cq(m + 1);
            for (int i = 0; i < m; ++i) cp[i] = P(i, j);
            for (int i = 0; i <= m; ++i) cq[i] = Q(i, j);
            st = g.lincomb(W.Tu[j], Z(0.0, 0.0), wm, cp);
            if (!st) st = g.lincomb(W.Tc[j], Z(0.0, 0.0), wm1, cq);
          }
          if (!st) st = g.solve_r(W.Tu, R, k);
          if (st) return finish(st);
          std::swap(W.U, W.Tu);
          std::swap(W.C, W.Tc);
          W.u_valid = true;
        }
      }
    }
    // without a deflation space from this cycle (an invariant subspace was
    // found, or the small problems failed) the loop below runs GMRES(m) cycles
  }

  while (!(rnorm <= tol * bnorm) && cycles < S->p.restart && g.apps < S->p.max_iterations) {
    ++cycles;
    if (!W.u_valid) {
      // plain GMRES(m) cycle
      const double beta = rnorm;
      if ((st = g.lincomb(Wvec(0), Z(0.0, 0.0), {&W.r}, {Z(1.0 / beta, 0.0)}))) return finish(st);
      Mat H(m + 1, m);
      int mm = m;
      for (int j = 0; j < m; ++j) {
        if ((st = g.apply(Wvec(j + 1), Wvec(j)))) return finish(st);
        std::vector<const FieldRef*> vs;
        for (int l = 0; l <= j; ++l) vs.push_back(&Wvec(l));
        std::vector<Z> h;
        if ((st = g.orthogonalise(Wvec(j + 1), vs, h))) return finish(st);
        for (int l = 0; l <= j; ++l) H(l, j) = h[l];
        const double hn = g.norm(Wvec(j + 1));
        H(j + 1, j) = hn;
        if (!(hn > 1e-14 * beta)) {
          mm = j + 1;
          break;
        }
        if ((st = g.scale(Wvec(j + 1), Z(1.0 / hn, 0.0)))) return finish(st);
      }
      Mat Hs(mm + 1, mm);
      for (int i = 0; i <= mm; ++i)
        for (int j = 0; j < mm; ++j) Hs(i, j) = H(i, j);
      std::vector<Z> c(mm + 1, Z(0.0, 0.0)), y;
      c[0] = beta;
      if (!dense::lstsq(Hs, c, y)) return finish(ctx->fail(CLG_ERR_BREAKDOWN, "GCRO-DR: least squares"));
      std::vector<const FieldRef*> vs;
      for (int j = 0; j < mm; ++j) vs.push_back(&Wvec(j));
      if ((st = g.lincomb(W.x, Z(1.0, 0.0), vs, y))) return finish(st);
      if ((st = g.residual(b, W.x, W.r))) return finish(st);
      rnorm = g.norm(W.r);
      continue;
    }
    // x += U C^+ r, r -= C C^+ r (OrthognalXR, :860-875)
    {
      std::vector<const FieldRef*> cs, us;
      for (int i = 0; i < k; ++i) {
        cs.push_back(&W.C[i]);
        us.push_back(&W.U[i]);
      }
      std::vector<Z> d;
      if ((st = g.dots(W.r, cs, d))) return finish(st);
      std::vector<Z> nd(k);
      for (int i = 0; i < k; ++i) nd[i] = -d[i];
      if ((st = g.lincomb(W.x, Z(1.0, 0.0), us, d))) return finish(st);
      if ((st = g.lincomb(W.r, Z(1.0, 0.0), cs, nd))) return finish(st);
    }
    // unit U_i, G_ii = 1/|U_i| (NormUkAndSetD, :843-858)
    Mat G(m + 1, m);
    for (int i = 0; i < k; ++i) {
      const double n = g.norm(W.U[i]);
      if (!(n > 0)) return finish(ctx->fail(CLG_ERR_BREAKDOWN, "GCRO-DR: zero recycled vector"));
      G(i, i) = 1.0 / n;
      if ((st = g.scale(W.U[i], Z(1.0 / n, 0.0)))) return finish(st);
    }
    const double beta = g.norm(W.r);
    if ((st = g.lincomb(W.V[0], Z(0.0, 0.0), {&W.r}, {Z(1.0 / beta, 0.0)}))) return finish(st);
    // Arnoldi with (1 - C C^+) A on the V (:259-301)
    int mm = m;
    for (int j = k; j < m; ++j) {
      const int jj = j - k;
      if ((st = g.apply(W.V[jj + 1], W.V[jj]))) return finish(st);
      std::vector<const FieldRef*> vs;
      for (int i = 0; i < k; ++i) vs.push_back(&W.C[i]);
      for (int l = 0; l <= jj; ++l) vs.push_back(&W.V[l]);
      std::vector<Z> h;
      if ((st = g.orthogonalise(W.V[jj + 1], vs, h))) return finish(st);
      for (int i = 0; i < k; ++i) G(i, j) = h[i];
      for (int l = 0; l <= jj; ++l) G(k + l, j) = h[k + l];
      const double hn = g.norm(W.V[jj + 1]);
      G(j + 1, j) = hn;
      if (!(hn > 1e-14 * beta)) {
        mm = j + 1;
        break;
      }
      if ((st = g.scale(W.V[jj + 1], Z(1.0 / hn, 0.0)))) return finish(st);
    }
    Mat Gs(mm + 1, mm);
    for (int i = 0; i <= mm; ++i)
      for (int j = 0; j < mm; ++j) Gs(i, j) = G(i, j);
    std::vector<Z> c(mm + 1, Z(0.0, 0.0)), y;
    c[k] = beta;
    if (!dense::lstsq(Gs, c, y)) return finish(ctx->fail(CLG_ERR_BREAKDOWN, "GCRO-DR: least squares"));
    {
      std::vector<const FieldRef*> vs;
      for (int i = 0; i < k; ++i) vs.push_back(&W.U[i]);
      for (int j = k; j < mm; ++j) vs.push_back(&W.V[j - k]);
      if ((st = g.lincomb(W.x, Z(1.0, 0.0), vs, y))) return finish(st);
    }
    if ((st = g.residual(b, W.x, W.r))) return finish(st);
    rnorm = g.norm(W.r);
    if (mm < m) continue;  // invariant subspace: keep U_k as it is
    const bool converged = rnorm <= tol * bnorm;
    // FindPk2 (:572-760), with W = [U, V_{m-k}], What = [C, V_{m-k+1}], A W = What G:
    //   SVD  G^+ G p = l B p, k smallest, B = W^+ W = [[U^+ U, U^+ V], [V^+ U, 1]]
    //        with the U^+ V blocks taken as 0 (the reference's B for SVD);
    //   REV  (W^+ What) G p = l B p, k smallest;
    //   HEV  G^+ (What^+ W) p = l G^+ G p, k largest.
    Mat Bm(m, m);
    for (int i = 0; i < m; ++i) Bm(i, i) = 1.0;
    for (int i = 0; i < k; ++i) {
      std::vector<const FieldRef*> us;
      for (int j = 0; j < k; ++j) us.push_back(&W.U[j]);
      std::vector<Z> d;
      if ((st = g.dots(W.U[i], us, d))) return finish(st);
      for (int j = 0; j < k; ++j)
        if (j != i) Bm(j, i) = d[j];  // (U_j^+ U_i)
    }
    std::vector<Z> ev;
    Mat Xv;
    bool ok;
    if (defl == CLG_DEFLATION_SVD) {
      ok = dense::geig(dense::mul_dag(G, G), Bm, ev, Xv);
    } else {
      // E(l, i) = What_l^+ U_i, i < k (the U columns of What^+ W; the V
      // columns of W are the unit vectors e_j there, V being orthonormal and
      // orthogonal to C)
      std::vector<const FieldRef*> hat;
      for (int i = 0; i < k; ++i) hat.push_back(&W.C[i]);
      for (int j = 0; j <= m - k; ++j) hat.push_back(&W.V[j]);
      Mat E(m + 1, k);
      for (int i = 0; i < k; ++i) {
        std::vector<Z> d;
        if ((st = g.dots(W.U[i], hat, d))) return finish(st);
        for (int l = 0; l <= m; ++l) E(l, i) = d[l];
      }
      if (defl == CLG_DEFLATION_REV) {
        Mat AL(m, m + 1);  // W^+ What
        for (int i = 0; i < k; ++i)
          for (int j = 0; j <= m; ++j) AL(i, j) = std::conj(E(j, i));
        for (int i = k; i < m; ++i) AL(i, i) = 1.0;
        for (int i = 0; i < k; ++i)
          for (int j = k; j < m; ++j) {
            Bm(i, j) = AL(i, j);  // U_i^+ V_{j-k}
            Bm(j, i) = std::conj(AL(i, j));
          }
        ok = dense::geig(dense::mul(AL, G), Bm, ev, Xv);
      } else {
        Mat AL(m + 1, m);  // What^+ W
        for (int l = 0; l <= m; ++l)
          for (int j = 0; j < k; ++j) AL(l, j) = E(l, j);
        for (int j = k; j < m; ++j) AL(j, j) = 1.0;
        ok = dense::geig(dense::mul_dag(G, AL), dense::mul_dag(G, G), ev, Xv);
      }
    }
    if (!ok) continue;  // keep U_k
    const Mat P = dense::select(ev, Xv, k, defl != CLG_DEFLATION_HEV);
    Mat Q, R;
    if (!dense::qr_thin(dense::mul(G, P), Q, R)) continue;
    // GenerateCU (:782-815): U = [U, V] P R^-1, C = [C, V] Q (C only while unconverged)
    std::vector<const FieldRef*> yv, wv;
    for (int i = 0; i < k; ++i) {
      yv.push_back(&W.U[i]);
      wv.push_back(&W.C[i]);
    }
    for (int j = 0; j < m - k; ++j) yv.push_back(&W.V[j]);
    for (int j = 0; j <= m - k; ++j) wv.push_back(&W.V[j]);
    for (int j = 0; j < k && !st; ++j) {
      std::vector<Z> cp(m), cq(m + 1);
      for (int i = 0; i < m; ++i) cp[i] = P(i, j);
      for (int i = 0; i <= m; ++i) cq[i] = Q(i, j);
      st = g.lincomb(W.Tu[j], Z(0.0, 0.0), yv, cp);
      if (!st && !converged) st = g.lincomb(W.Tc[j], Z(0.0, 0.0), wv, cq);
    }
    if (!st) st = g.solve_r(W.Tu, R, k);
    if (st) return finish(st);
    std::swap(W.U, W.Tu);
    if (!converged) std::swap(W.C, W.Tc);
  }
  return finish(CLG_SUCCESS);
}

}  // namespace clg

extern "C" clg_status clg_solver_reset(clg_solver s) {
  if (!s) return CLG_ERR_BAD_ARG;
  if (auto* w = dynamic_cast<clg::GcroWork*>(s->cache_gcro.get())) w->u_valid = false;
  return CLG_SUCCESS;
}
