// mskrylov.cu -- the reference's multi-shift solvers that share one Krylov
// space of A over every shift c_n of (A + c_n) x_n = b: CMultiShiftFOM::Solve
// (SparseLinearAlgebra/CMultiShiftFOM.cpp:97-270), CMultiShiftGMRES::Solve
// (CMultiShiftGMRES.cpp:113-330) and CMultiShiftBiCGStab::Solve
// (CMultiShiftBiCGStab.cpp:73-437), the latter two at the end of this file.
//
// Restarted FOM(m) (the full orthogonalisation method): the Arnoldi relation
// A V_m = V_m H_m + h_{m+1,m} v_{m+1} e_m^T holds for A + c_n with H_m + c_n,
// so one Arnoldi cycle serves every shift.  Shift n solves the square system
// (H_m + c_n) y_n = beta_n e_1 (the reference rotates the Hessenberg with
// Givens and back-substitutes; the same solution), adds V_m y_n to x_n, and its
// residual is beta_n' v_{m+1} with beta_n' = -h_{m+1,m} y_n[m-1]: the residuals
// of all shifts stay collinear, and the next cycle starts from v_{m+1}.  The
// solve stops when every |beta_n| is below the target.
//
// B200 form: FP64 vectors on the device (the reference's precision for this
// solver), the Arnoldi orthogonalisation by classical Gram-Schmidt applied
// twice (one multi-dot and one linear-combination launch per pass; the
// reference uses modified Gram-Schmidt with one launch per inner product), the
// m x m shifted systems on the host.  A final batched FP64 defect correction
// (the shifts as right-hand sides, GMRES inside) checks every shift's true
// residual and refines any shift the recurrence left above tol_true_rel.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "hostkrylov.cuh"

namespace clg {

namespace {

using dense::Mat;
using dense::Z;

constexpr int FOM_MAXDIM = 32;  // vectors of one cycle (the linear combinations take up to 34)

struct FomWork : hk::HostVecs {
  std::string key;
  std::vector<FieldRef> V;  // the cycle's basis v_0 .. v_{m-1}
  FieldRef w, R;            // Arnoldi workspace, the next start vector v_m
  FieldRef X;               // the nshift solutions (FP64, right-hand sides = shifts)
};

template <int NC>
struct ConjF {  // y = conj(y), elementwise (CField::Dagger)
  DField y;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int, int p, int64_t h, double*) const {
    cpx<double> v[NC];
    ldv<P64, NC, double>(y, 0, p, h, v);
#pragma unroll
    for (int c = 0; c < NC; ++c) v[c].y = -v[c].y;
    stv<P64, NC, double>(y, 0, p, h, v);
  }
  __device__ void finalize(int, const double*) const {}
};

clg_status conj_field(clg_context_s* ctx, const FieldRef& y) {
  if (y.nc == 12) return launch_sites<0>(ctx, ConjF<12>{dfield(y)}, y.first_parity, y.nparity, y.Vh, 1);
  return launch_sites<0>(ctx, ConjF<3>{dfield(y)}, y.first_parity, y.nparity, y.Vh, 1);
}

}  // namespace

// The FOM phase: X[n] = (A + c_n)^-1 b to |beta_n| <= tol |b| (or restart
// cycles); returns the operator applications.
clg_status fom_ms_run(clg_context_s* ctx, std::unique_ptr<SolveCacheBase>& cache, const clg_gauge_s* U, int kind,
                      double param, int op, const FieldRef& b, const std::vector<double2>& shifts, int m,
                      int restart, double tol, const FieldRef** X_out, int* apps_out, int* cycles_out) {
  const int ns = (int)shifts.size();
  const int nc = b.nc;
  const int64_t Vh = b.Vh;
  const std::string key = std::to_string((uintptr_t)b.data) + "/" + std::to_string(b.nparity) + "/" +
                          std::to_string(b.first_parity) + "/" + std::to_string(nc) + "/" + std::to_string(Vh) +
                          "/" + std::to_string(m) + "/" + std::to_string(ns);
  auto* W = dynamic_cast<FomWork*>(cache.get());
  if (!W || W->key != key) {
    cudaStreamSynchronize(ctx->stream);
    cache.reset();
    auto nw = std::make_unique<FomWork>();
    nw->ctx = ctx;
    nw->proto = b;
    nw->proto.nrhs = 1;
    nw->proto.rstride = nw->proto.blk * nw->proto.nparity;
    nw->V.resize(m);
    clg_status st = CLG_SUCCESS;
    for (FieldRef& f : nw->V)
      if (!st) st = nw->vec(f);
    if (!st) st = nw->vec(nw->w);
    if (!st) st = nw->vec(nw->R);
    if (!st) st = nw->full_vec(nw->tmp);
    if (!st) st = nw->out_buffer();
    if (!st) {  // the solutions: one allocation, shift k is right-hand side k
      void* p = nullptr;
      st = dalloc(ctx, &p, (size_t)nw->proto.rstride * ns);
      if (!st) {
        nw->allocs.push_back(p);
        nw->X = nw->proto;
        nw->X.data = static_cast<char*>(p);
        nw->X.nrhs = ns;
      }
    }
    if (st) return st;
    nw->key = key;
    W = nw.get();
    cache = std::move(nw);
  }
  hk::HostKrylov K{ctx, *W, U, kind, op, nc, param, Vh};
  auto xk = [&](int k) {
    FieldRef f = W->X;
    f.data = W->X.data + (int64_t)k * W->X.rstride;
    f.nrhs = 1;
    return f;
  };
  clg_status st;
  for (int k = 0; k < ns; ++k)
    if ((st = K.scale(xk(k), Z(0.0, 0.0)))) return st;
  *X_out = &W->X;
  *apps_out = 0;
  *cycles_out = 0;
  const double bnorm = K.norm(b);
  if (bnorm < 0) return ctx->fail(CLG_ERR_CUDA, "multi-shift FOM: reading |b|");
  if (bnorm == 0.0) return CLG_SUCCESS;
  // v_0 = b / |b|, beta_n = |b| for every shift (CMultiShiftFOM.cpp:141-160)
  if ((st = K.lincomb(W->R, Z(0.0, 0.0), {&b}, {Z(1.0 / bnorm, 0.0)}))) return st;
  std::vector<Z> beta(ns, Z(bnorm, 0.0));
  std::vector<int> active(ns, 1);
  for (int cyc = 0; cyc < restart; ++cyc) {
    ++*cycles_out;
    if ((st = K.copy(W->V[0], W->R))) return st;
    Mat H(m + 1, m);
    int dim = m;
    for (int j = 0; j < m; ++j) {
      if ((st = K.apply(W->w, W->V[j]))) return st;
      std::vector<const FieldRef*> vs;
      for (int i = 0; i <= j; ++i) vs.push_back(&W->V[i]);
      std::vector<Z> h;
      if ((st = K.orthogonalise(W->w, vs, h))) return st;
      for (int i = 0; i <= j; ++i) H(i, j) = h[i];
      const double hn = K.norm(W->w);
      if (hn < 0) return ctx->fail(CLG_ERR_CUDA, "multi-shift FOM: reading |w|");
      H(j + 1, j) = Z(hn, 0.0);
      if (hn <= 1e-300 * bnorm) {  // invariant subspace: the solution lies in V_{j+1}
        dim = j + 1;
        break;
      }
      const FieldRef& next = (j + 1 < m) ? W->V[j + 1] : W->R;
      if ((st = K.lincomb(next, Z(0.0, 0.0), {&W->w}, {Z(1.0 / hn, 0.0)}))) return st;
    }
    double worst = 0.0;
    for (int n = 0; n < ns; ++n) {
      if (!active[n]) continue;
      Mat Hc(dim, dim);
      for (int r = 0; r < dim; ++r)
        for (int c = 0; c < dim; ++c) Hc(r, c) = H(r, c) + (r == c ? Z(shifts[n].x, shifts[n].y) : Z(0.0, 0.0));
      std::vector<Z> g(dim, Z(0.0, 0.0)), y;
      g[0] = beta[n];
      if (!dense::lstsq(Hc, g, y)) return ctx->fail(CLG_ERR_BREAKDOWN, "multi-shift FOM: singular shifted Hessenberg");
      std::vector<const FieldRef*> vs;
      for (int i = 0; i < dim; ++i) vs.push_back(&W->V[i]);
      const FieldRef x = xk(n);
      if ((st = K.lincomb(x, Z(1.0, 0.0), vs, y))) return st;
      // the next residual of this shift: beta_n v_m (CMultiShiftFOM.cpp:227-229)
      beta[n] = (dim == m) ? -H(m, m - 1).real() * y[m - 1] : Z(0.0, 0.0);
      const double bl = std::abs(beta[n]);
      if (!(bl == bl)) return ctx->fail(CLG_ERR_BREAKDOWN, "multi-shift FOM: NaN in the recurrence");
      if (bl <= tol * bnorm) active[n] = 0;
      worst = std::max(worst, bl);
    }
    *apps_out += dim;
    if (worst <= tol * bnorm || dim < m) break;
  }
  return CLG_SUCCESS;
}

// CMultiShiftGMRES::Solve (SparseLinearAlgebra/CMultiShiftGMRES.cpp:113-330;
// A. Frommer and U. Glaessner, SIAM J. Sci. Comput. 19 (1998) 15): restarted
// GMRES(m) on the unshifted seed system; every shift keeps its residual
// collinear with the seed's, r_n = beta_n r_seed: with z = beta e_1 - Hbar y
// (the seed's residual in the cycle's basis), shift n solves the square system
// [Hbar + c_n I~ | z] [y_n; beta_n'] = beta_n beta e_1 and adds V y_n to x_n.
// The next cycle restarts from the seed's true residual b - A x_seed.  Stop
// when every |beta_n| |z| (the shifted residual norms) is below tol |b|.
clg_status gmres_ms_run(clg_context_s* ctx, std::unique_ptr<SolveCacheBase>& cache, const clg_gauge_s* U, int kind,
                        double param, int op, const FieldRef& b, const std::vector<double2>& shifts, int m, int restart,
                        double tol, const FieldRef** X_out, int* apps_out, int* cycles_out) {
  const int ns = (int)shifts.size();
  const int nc = b.nc;
  const int64_t Vh = b.Vh;
  const std::string key = "gmres-m/" + std::to_string((uintptr_t)b.data) + "/" + std::to_string(b.nparity) + "/" +
                          std::to_string(b.first_parity) + "/" + std::to_string(nc) + "/" + std::to_string(Vh) +
                          "/" + std::to_string(m) + "/" + std::to_string(ns);
  auto* W = dynamic_cast<FomWork*>(cache.get());
  if (!W || W->key != key) {
    cudaStreamSynchronize(ctx->stream);
    cache.reset();
    auto nw = std::make_unique<FomWork>();
    nw->ctx = ctx;
    nw->proto = b;
    nw->proto.nrhs = 1;
    nw->proto.rstride = nw->proto.blk * nw->proto.nparity;
    nw->V.resize(m + 1);  // V[m] holds the seed solution
    clg_status st = CLG_SUCCESS;
    for (FieldRef& f : nw->V)
      if (!st) st = nw->vec(f);
    if (!st) st = nw->vec(nw->w);
    if (!st) st = nw->vec(nw->R);
    if (!st) st = nw->full_vec(nw->tmp);
    if (!st) st = nw->out_buffer();
    if (!st) {
      void* p = nullptr;
      st = dalloc(ctx, &p, (size_t)nw->proto.rstride * ns);
      if (!st) {
        nw->allocs.push_back(p);
        nw->X = nw->proto;
        nw->X.data = static_cast<char*>(p);
        nw->X.nrhs = ns;
      }
    }
    if (st) return st;
    nw->key = key;
    W = nw.get();
    cache = std::move(nw);
  }
  hk::HostKrylov K{ctx, *W, U, kind, op, nc, param, Vh};
  auto xk = [&](int k) {
    FieldRef f = W->X;
    f.data = W->X.data + (int64_t)k * W->X.rstride;
    f.nrhs = 1;
    return f;
  };
  const Z zero(0.0, 0.0), one(1.0, 0.0);
  FieldRef& xs = W->V[m];
  clg_status st;
  for (int k = 0; k < ns; ++k)
    if ((st = K.scale(xk(k), zero))) return st;
  if ((st = K.scale(xs, zero))) return st;
  *X_out = &W->X;
  *apps_out = 0;
  *cycles_out = 0;
  const double bnorm = K.norm(b);
  if (bnorm < 0) return ctx->fail(CLG_ERR_CUDA, "multi-shift GMRES: reading |b|");
  if (bnorm == 0.0) return CLG_SUCCESS;
  std::vector<Z> beta0(ns, one);
  for (int cyc = 0; cyc < restart; ++cyc) {
    ++*cycles_out;
    // the seed residual: b, then b - A x_seed (CMultiShiftGMRES.cpp:158-172)
    if (cyc == 0) {
      if ((st = K.copy(W->R, b))) return st;
    } else {
      if ((st = K.apply(W->w, xs)) || (st = K.lincomb(W->R, zero, {&b, &W->w}, {one, -one}))) return st;
    }
    const double beta = K.norm(W->R);
    if (beta < 0) return ctx->fail(CLG_ERR_CUDA, "multi-shift GMRES: reading |r|");
    if (beta == 0.0) break;
    if ((st = K.lincomb(W->V[0], zero, {&W->R}, {Z(1.0 / beta, 0.0)}))) return st;
    Mat H(m + 1, m);
    int dim = m;
    for (int j = 0; j < m; ++j) {
      if ((st = K.apply(W->w, W->V[j]))) return st;
      std::vector<const FieldRef*> vs;
      for (int i = 0; i <= j; ++i) vs.push_back(&W->V[i]);
      std::vector<Z> h;
      if ((st = K.orthogonalise(W->w, vs, h))) return st;
      for (int i = 0; i <= j; ++i) H(i, j) = h[i];
      const double hn = K.norm(W->w);
      if (hn < 0) return ctx->fail(CLG_ERR_CUDA, "multi-shift GMRES: reading |w|");
      H(j + 1, j) = Z(hn, 0.0);
      if (hn <= 1e-300 * bnorm) {
        dim = j + 1;
        break;
      }
      if (j + 1 < m && (st = K.lincomb(W->V[j + 1], zero, {&W->w}, {Z(1.0 / hn, 0.0)}))) return st;
    }
    *apps_out += dim + (cyc > 0 ? 1 : 0);
    // the seed system: y = argmin |beta e_1 - Hbar y|, z = beta e_1 - Hbar y
    Mat Hb(dim + 1, dim);
    for (int r = 0; r <= dim; ++r)
      for (int c = 0; c < dim; ++c) Hb(r, c) = H(r, c);
    std::vector<Z> g(dim + 1, zero), y;
    g[0] = Z(beta, 0.0);
    if (!dense::lstsq(Hb, g, y)) return ctx->fail(CLG_ERR_BREAKDOWN, "multi-shift GMRES: seed least squares");
    std::vector<const FieldRef*> vs;
    for (int i = 0; i < dim; ++i) vs.push_back(&W->V[i]);
    if ((st = K.lincomb(xs, one, vs, y))) return st;
    std::vector<Z> z(dim + 1);
    for (int r = 0; r <= dim; ++r) {
      Z hy = zero;
      for (int c = 0; c < dim; ++c) hy += Hb(r, c) * y[c];
      z[r] = g[r] - hy;
    }
    double zn = 0.0;
    for (const Z& v : z) zn += std::norm(v);
    zn = std::sqrt(zn);
    double worst = 0.0;
    for (int n = 0; n < ns; ++n) {
      // [Hbar + c_n I~ | z] [y_n; beta_n'] = beta_n beta e_1
      Mat Hh(dim + 1, dim + 1);
      for (int r = 0; r <= dim; ++r) {
        for (int c = 0; c < dim; ++c)
          Hh(r, c) = Hb(r, c) + (r == c ? Z(shifts[n].x, shifts[n].y) : zero);
        Hh(r, dim) = z[r];
      }
      std::vector<Z> gn(dim + 1, zero), w;
      gn[0] = beta0[n] * beta;
      if (!dense::lstsq(Hh, gn, w)) return ctx->fail(CLG_ERR_BREAKDOWN, "multi-shift GMRES: shifted system");
      std::vector<Z> yn(w.begin(), w.begin() + dim);
      if ((st = K.lincomb(xk(n), one, vs, yn))) return st;
      beta0[n] = w[dim];
      const double e = std::abs(beta0[n]) * zn;
      if (!(e == e)) return ctx->fail(CLG_ERR_BREAKDOWN, "multi-shift GMRES: NaN in the recurrence");
      worst = std::max(worst, e);
    }
    if (worst <= tol * bnorm) break;
  }
  return CLG_SUCCESS;
}

// CMultiShiftBiCGStab::Solve (SparseLinearAlgebra/CMultiShiftBiCGStab.cpp:73-437;
// B. Jegerlehner, hep-lat/9612014): the BiCGStab recurrences of A with the
// shadow residual conj(b), every shift's iterate and shifted residual s_n
// updated from the shared vectors through the zeta / beta_n / alpha_n
// recurrences; every `dev_step` iterations |s| and every |s_n| are compared
// with tol |b|.  FP64 vectors; the scalars on the host.
clg_status bicgstab_ms_run(clg_context_s* ctx, std::unique_ptr<SolveCacheBase>& cache, const clg_gauge_s* U, int kind,
                           double param, int op, const FieldRef& b, const std::vector<double2>& shifts, int dev_step,
                           int max_step, double tol, const FieldRef** X_out, int* apps_out, int* iters_out) {
  const int ns = (int)shifts.size();
  const int nc = b.nc;
  const int64_t Vh = b.Vh;
  const std::string key = "bicgstab-m/" + std::to_string((uintptr_t)b.data) + "/" + std::to_string(b.nparity) + "/" +
                          std::to_string(b.first_parity) + "/" + std::to_string(nc) + "/" + std::to_string(Vh) +
                          "/" + std::to_string(ns);
  auto* W = dynamic_cast<FomWork*>(cache.get());
  if (!W || W->key != key) {
    cudaStreamSynchronize(ctx->stream);
    cache.reset();
    auto nw = std::make_unique<FomWork>();
    nw->ctx = ctx;
    nw->proto = b;
    nw->proto.nrhs = 1;
    nw->proto.rstride = nw->proto.blk * nw->proto.nparity;
    nw->V.resize(6 + ns);  // R, W, W0, S, SA, WA, then s_n per shift
    clg_status st = CLG_SUCCESS;
    for (FieldRef& f : nw->V)
      if (!st) st = nw->vec(f);
    if (!st) st = nw->full_vec(nw->tmp);
    if (!st) st = nw->out_buffer();
    if (!st) {
      void* p = nullptr;
      st = dalloc(ctx, &p, (size_t)nw->proto.rstride * ns);
      if (!st) {
        nw->allocs.push_back(p);
        nw->X = nw->proto;
        nw->X.data = static_cast<char*>(p);
        nw->X.nrhs = ns;
      }
    }
    if (st) return st;
    nw->key = key;
    W = nw.get();
    cache = std::move(nw);
  }
  hk::HostKrylov K{ctx, *W, U, kind, op, nc, param, Vh};
  auto xk = [&](int k) {
    FieldRef f = W->X;
    f.data = W->X.data + (int64_t)k * W->X.rstride;
    f.nrhs = 1;
    return f;
  };
  FieldRef &R = W->V[0], &Wv = W->V[1], &W0 = W->V[2], &S = W->V[3], &SA = W->V[4], &WA = W->V[5];
  auto Ss = [&](int k) -> FieldRef& { return W->V[6 + k]; };
  const Z one(1.0, 0.0), zero(0.0, 0.0);
  clg_status st;
  *X_out = &W->X;
  *apps_out = 0;
  *iters_out = 0;
  for (int k = 0; k < ns; ++k)
    if ((st = K.scale(xk(k), zero)) || (st = K.copy(Ss(k), b))) return st;
  const double blen = K.norm(b);
  if (blen < 0) return ctx->fail(CLG_ERR_CUDA, "multi-shift BiCGStab: reading |b|");
  if (blen == 0.0) return CLG_SUCCESS;
  auto dot = [&](const FieldRef& a, const FieldRef& c, Z& out) -> clg_status {
    std::vector<Z> d;
    if (clg_status e = K.dots(c, {&a}, d)) return e;
    out = d[0];
    return CLG_SUCCESS;
  };
  if ((st = K.copy(R, b)) || (st = K.copy(S, b)) || (st = K.copy(W0, b))) return st;
  if ((st = conj_field(ctx, W0))) return st;  // the shadow residual conj(b)
  Z delta, phi, t;
  if ((st = dot(W0, R, delta))) return st;
  if ((st = K.apply(SA, b))) return st;
  if ((st = dot(W0, SA, t))) return st;
  phi = t / delta;
  Z beta = zero, alpha = zero;
  std::vector<Z> betas(ns, one), zeta(ns, one), zetaold(ns, one), rho(ns, one);
  std::vector<double> sl(ns, 1.0);
  auto live = [&](int k) { return !(sl[k] < tol * blen); };
  for (int it = 0; it < max_step * dev_step; ++it) {
    ++*iters_out;
    const Z newbeta = -one / phi;
    for (int k = 0; k < ns; ++k) {
      if (!live(k)) continue;
      const Z c(shifts[k].x, shifts[k].y);
      if (it == 0) {
        zeta[k] = one / (one - c * newbeta);
        betas[k] = newbeta * zeta[k];
      } else {
        const Z znm1 = zetaold[k];
        zetaold[k] = zeta[k];
        const Z zb = znm1 * beta;
        zeta[k] = (zetaold[k] * zb) / (alpha * (newbeta * (znm1 - zetaold[k])) + zb * (one - c * newbeta));
        betas[k] = newbeta * zeta[k] / zetaold[k];
      }
    }
    beta = newbeta;
    // w = r + beta SA ; WA = A w ; chi = <WA, w> / |WA|^2
    if ((st = K.lincomb(Wv, zero, {&R, &SA}, {one, beta})) || (st = K.apply(WA, Wv))) return st;
    Z wa_w, wa_wa;
    if ((st = dot(WA, Wv, wa_w)) || (st = dot(WA, WA, wa_wa))) return st;
    const Z chi = wa_w / wa_wa.real();
    for (int k = 0; k < ns; ++k) {
      if (!live(k)) continue;
      const Z c(shifts[k].x, shifts[k].y);
      const Z dinom = one + c * chi;
      const Z chirho = chi / dinom * rho[k];
      const Z crz = chirho * zeta[k];
      // x_n += -beta_n s_n + crz w ;  s_n += -(crz / beta_n) w + (chirho zeta_n / beta_n) r
      const FieldRef xn = xk(k);
      if ((st = K.lincomb(xn, one, {&Ss(k), &Wv}, {-betas[k], crz}))) return st;
      if ((st = K.lincomb(Ss(k), one, {&Wv, &R}, {-(crz / betas[k]), chirho * zetaold[k] / betas[k]}))) return st;
      rho[k] = rho[k] / dinom;
    }
    // r = w - chi WA ; delta' = <w0, r> ; alpha = -beta delta' / (chi delta)
    if ((st = K.lincomb(R, zero, {&Wv, &WA}, {one, -chi}))) return st;
    Z newdelta;
    if ((st = dot(W0, R, newdelta))) return st;
    alpha = (beta * (-newdelta)) / (chi * delta);
    delta = newdelta;
    for (int k = 0; k < ns; ++k) {
      if (!live(k)) continue;
      const Z an = (alpha * zeta[k] * betas[k]) / (zetaold[k] * beta);
      if ((st = K.lincomb(Ss(k), an, {&R}, {zeta[k] * rho[k]}))) return st;
    }
    // s = alpha (s - chi SA) + r ; SA = A s ; phi = <w0, SA> / delta
    if ((st = K.lincomb(S, alpha, {&SA, &R}, {-alpha * chi, one}))) return st;
    if ((st = K.apply(SA, S))) return st;
    if ((st = dot(W0, SA, t))) return st;
    phi = t / delta;
    if (!(std::abs(phi) == std::abs(phi)) || std::abs(delta) == 0.0)
      return ctx->fail(CLG_ERR_BREAKDOWN, "multi-shift BiCGStab: breakdown");
    if ((it + 1) % dev_step == 0) {
      double worst = K.norm(S);
      for (int k = 0; k < ns; ++k) {
        if (!live(k)) continue;
        sl[k] = K.norm(Ss(k));
        worst = std::max(worst, sl[k]);
      }
      if (worst < tol * blen) break;
    }
  }
  *apps_out = K.apps;
  return CLG_SUCCESS;
}

}  // namespace clg
