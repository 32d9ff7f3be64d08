// measure.cu -- measurements on top of the batched solves: the meson
// correlator of 12 point-source propagators and the stochastic (Z4-noise)
// condensate traces.
//
// Meson correlator (CMeasureMesonCorrelator::CalculateCorrelator,
// Measurement/CMeasureMesonCorrelator.cu:254-411): the 12 spin-colour point
// sources at the origin are solved in ONE batched call (12 right-hand sides
// of one field), then for every requested gamma the per-site contraction of
// _kernelCalculateCorrelatorSU3 (:26-174) and the spatial sum per time slice
// times 2/sqrt(V) (:366-380).  One pass over the propagators serves up to 8
// gammas; the per-site values go to a [gamma][t][xyz] buffer and a second
// kernel sums each (gamma, t) row in a fixed order (deterministic).
//
// Condensate (CMeasureChiralCondensate::OnConfigurationAcceptedZ4SingleField,
// Measurement/CMeasureChiralCondensate.cu:236-290, _kernelDotMeasureAll
// :38-100): (1/V) sum_x eta(x)^+ Gamma_k psi(x) for the nine measurement kinds
// (1, gamma1..gamma5, gamma4 gamma5, and the rotating-frame gamma1 + y omega
// gamma4, gamma2 - x omega gamma4, which are gamma1 and gamma2 here: omega = 0)
// of every right-hand side, psi = D^-1 eta with the noise sources solved in
// one batched call.  One site kernel with 18 FP64 reductions per right-hand side.
//
// Gamma matrices: the chiral set and the products of
// gammaMatrixSet::CreateGammaMatrix (Tools/Math/GammaMatrix.h:405-511) built
// on the host by the same rules (row r -> column idx[r], phase i^z[r]).
#include <cmath>
#include <vector>

#include "blas.cuh"

namespace clg {

namespace {

struct GammaT {
  int idx[4];
  int z[4];
  int ns;  // CalculateNextSymmetricIndex
};

enum {
  G_UNITY = 0, G_1, G_2, G_3, G_4, G_5, G_51, G_52, G_53, G_54, G_15, G_25, G_35, G_45, S_12, S_23, S_31, S_41, S_42,
  S_43, S_12E, S_23E, S_31E, G_C, G_MAX
};

GammaT gmult(const GammaT& a, const GammaT& b, int extra_i) {
  GammaT o{};
  for (int r = 0; r < 4; ++r) {
    o.idx[r] = b.idx[a.idx[r]];
    o.z[r] = (a.z[r] + b.z[a.idx[r]] + extra_i) & 3;
  }
  return o;
}

std::vector<GammaT> gamma_table() {
  std::vector<GammaT> g(G_MAX);
  auto set = [&](int w, int r, int c, int z) {
    g[w].idx[r] = c;
    g[w].z[r] = z;
  };
  for (int r = 0; r < 4; ++r) set(G_UNITY, r, r, 0);
  const int t1[4][2] = {{3, 3}, {2, 3}, {1, 1}, {0, 1}}, t2[4][2] = {{3, 2}, {2, 0}, {1, 0}, {0, 2}},
            t3[4][2] = {{2, 3}, {3, 1}, {0, 1}, {1, 3}}, t4[4][2] = {{2, 0}, {3, 0}, {0, 0}, {1, 0}},
            t5[4][2] = {{0, 0}, {1, 0}, {2, 2}, {3, 2}};
  for (int r = 0; r < 4; ++r) {
    set(G_1, r, t1[r][0], t1[r][1]);
    set(G_2, r, t2[r][0], t2[r][1]);
    set(G_3, r, t3[r][0], t3[r][1]);
    set(G_4, r, t4[r][0], t4[r][1]);
    set(G_5, r, t5[r][0], t5[r][1]);
  }
  g[G_51] = gmult(g[G_5], g[G_1], 0);
  g[G_52] = gmult(g[G_5], g[G_2], 0);
  g[G_53] = gmult(g[G_5], g[G_3], 0);
  g[G_54] = gmult(g[G_5], g[G_4], 0);
  g[G_15] = gmult(g[G_1], g[G_5], 0);
  g[G_25] = gmult(g[G_2], g[G_5], 0);
  g[G_35] = gmult(g[G_3], g[G_5], 0);
  g[G_45] = gmult(g[G_4], g[G_5], 0);
  g[S_12] = gmult(g[G_2], g[G_1], 1);
  g[S_23] = gmult(g[G_3], g[G_2], 1);
  g[S_31] = gmult(g[G_1], g[G_3], 1);
  g[S_12E] = gmult(g[G_1], g[G_2], 1);
  g[S_23E] = gmult(g[G_2], g[G_3], 1);
  g[S_31E] = gmult(g[G_3], g[G_1], 1);
  g[S_41] = gmult(g[G_1], g[G_4], 1);
  g[S_42] = gmult(g[G_2], g[G_4], 1);
  g[S_43] = gmult(g[G_3], g[G_4], 1);
  g[G_C] = gmult(g[G_4], g[G_2], 0);
  static const int nsi[4] = {0, 2, 3, 1};
  for (auto& x : g) x.ns = nsi[x.idx[0]];
  return g;
}

// ------------------------------------------------------------------ meson correlator
constexpr int MESON_CHUNK = 8;

struct MesonArgs {
  Geom g;
  DField prop;  // FP64 Wilson, 12 right-hand sides r = spin * 3 + colour
  int ng;
  GammaT gm[MESON_CHUNK];
  double* out;  // [ng][Lt][Vxyz]
  int64_t Vxyz;
};

// sum_{a, b} Re(conj(S(j,a)_{i,b}) S(pj,a)_{pi,b}) at checkerboard site (p, h)
__device__ __forceinline__ double meson_term(const MesonArgs& m, int p, int64_t h, int i, int j, int pi, int pj) {
  const int64_t Vh = m.g.Vh;
  double t = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double2* x = reinterpret_cast<const double2*>(m.prop.base(3 * j + a, p)) + (int64_t)(3 * i) * Vh + h;
    const double2* y = reinterpret_cast<const double2*>(m.prop.base(3 * pj + a, p)) + (int64_t)(3 * pi) * Vh + h;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const double2 u = __ldg(x + b * Vh), v = __ldg(y + b * Vh);
      t = fma(u.x, v.x, fma(u.y, v.y, t));
    }
  }
  return t;
}

__global__ void __launch_bounds__(256) meson_site_kernel(MesonArgs m) {
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i0 >= 2 * m.g.Vh) return;
  const int p = (int)(i0 / m.g.Vh);
  const int64_t h = i0 - (int64_t)p * m.g.Vh;
  int c[4];
  eo_coords(m.g, p, h, c);
  const int64_t s = site_index(m.g, c);
  const int Lt = m.g.L[3];
  const int64_t xyz = s / Lt;
  for (int k = 0; k < m.ng; ++k) {
    const GammaT& G = m.gm[k];
    double res = 0.0;
    for (int i = 1; i < 4; ++i)
      for (int j = i + 1; j < 4; ++j) {
        // i^(z_i + conj(z_j)) is real: +1 for 0 mod 4, -1 for 2 mod 4
        const int zz = G.z[i] + (((G.z[j] & 1) << 1) + G.z[j]);
        res += (1.0 - (double)(zz & 2)) * meson_term(m, p, h, i, j, G.idx[i], G.idx[j]);
      }
    if (G.ns == 0) {
      for (int i = 0; i < 4; ++i) res += 0.5 * meson_term(m, p, h, i, i, i, i);
    } else {
      res += meson_term(m, p, h, 0, 0, G.idx[0], G.idx[0]);
      res += meson_term(m, p, h, G.ns, G.ns, G.idx[G.ns], G.idx[G.ns]);
    }
    m.out[((int64_t)k * Lt + c[3]) * m.Vxyz + xyz] = res;
  }
}

// C[k][t] = scale * sum_xyz buf[k][t][xyz], one block per (t, k), fixed order
__global__ void __launch_bounds__(256) row_sum_kernel(const double* buf, int64_t n, double scale, double* out) {
  const int64_t row = (int64_t)blockIdx.y * gridDim.x + blockIdx.x;
  const double* r = buf + row * n;
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += r[i];
  __shared__ double sm[256];
  sm[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[row] = scale * sm[0];
}

// ------------------------------------------------------------------ condensate
constexpr int COND_KINDS = 9;

struct CondF {
  DField eta, psi;  // FP64 Wilson, nrhs each
  GammaT gm[COND_KINDS];
  double* out;      // [rhs][kind] complex
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int rhs, int p, int64_t h, double* acc) const {
    cpx<double> e[12], q[12];
    ldv<P64, 12, double>(eta, rhs, p, h, e);
    ldv<P64, 12, double>(psi, rhs, p, h, q);
#pragma unroll
    for (int k = 0; k < COND_KINDS; ++k) {
      double re = 0.0, im = 0.0;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        // (Gamma psi)_{r, c} = i^z[r] psi_{idx[r], c}
        const int z = gm[k].z[r], src = gm[k].idx[r];
        double sr = 0.0, si = 0.0;  // sum_c conj(eta_{r,c}) psi_{src,c}
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          cpx<double> v = q[0];
          // select psi_{src, c} without dynamic register indexing
#pragma unroll
          for (int t = 0; t < 4; ++t)
            if (t == src) v = q[3 * t + c];
          const cpx<double> a = e[3 * r + c];
          sr = fma(a.x, v.x, fma(a.y, v.y, sr));
          si = fma(a.x, v.y, fma(-a.y, v.x, si));
        }
        // times i^z
        const double xr = (z == 0) ? sr : (z == 1) ? -si : (z == 2) ? -sr : si;
        const double xi = (z == 0) ? si : (z == 1) ? sr : (z == 2) ? -si : -sr;
        re += xr;
        im += xi;
      }
      acc[2 * k] += re;
      acc[2 * k + 1] += im;
    }
  }
  __device__ void finalize(int rhs, const double* s) const {
    for (int k = 0; k < 2 * COND_KINDS; ++k) out[2 * COND_KINDS * rhs + k] = s[k];
  }
};

clg_status check_prop(clg_field f, int nrhs_min, const char* what) {
  if (!f) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = f->lat->ctx;
  if (f->kind != CLG_FERMION_WILSON || f->subset != CLG_SUBSET_FULL || f->prec != CLG_PREC_DOUBLE ||
      f->nrhs < nrhs_min)
    return ctx->fail(CLG_ERR_BAD_ARG, std::string(what) + ": a FULL FP64 Wilson field is required");
  return CLG_SUCCESS;
}

clg_status sync_fail(clg_context_s* ctx) {
  const cudaError_t e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? CLG_SUCCESS : ctx->fail(cuda_status(e), cudaGetErrorString(e));
}

}  // namespace

}  // namespace clg

using namespace clg;

extern "C" {

clg_status clg_meson_contract(clg_field prop, int ngamma, const int* gammas, double* corr) {
  if (clg_status st = check_prop(prop, 12, "meson correlator")) return st;
  clg_context_s* ctx = prop->lat->ctx;
  if (prop->nrhs != 12) return ctx->fail(CLG_ERR_BAD_ARG, "meson correlator: the propagator field holds 12 right-hand sides");
  if (ngamma < 1 || !gammas || !corr) return ctx->fail(CLG_ERR_BAD_ARG, "meson correlator: no gamma matrices");
  for (int k = 0; k < ngamma; ++k)
    if (gammas[k] < 0 || gammas[k] >= G_MAX) return ctx->fail(CLG_ERR_BAD_ARG, "meson correlator: unknown gamma matrix");
  if (clg_status st = settle(prop)) return st;
  const Geom& g = prop->lat->g;
  const int Lt = g.L[3];
  const int64_t Vxyz = g.V / Lt;
  const std::vector<GammaT> tab = gamma_table();
  const int chunk = std::min(ngamma, MESON_CHUNK);
  double *buf = nullptr, *dout = nullptr;
  clg_status st = dalloc(ctx, (void**)&buf, (size_t)chunk * g.V * sizeof(double));
  if (st) return st;
  if ((st = dalloc(ctx, (void**)&dout, (size_t)ngamma * Lt * sizeof(double)))) {
    dfree(buf);
    return st;
  }
  const double scale = 2.0 / std::sqrt((double)g.V);
  for (int k0 = 0; k0 < ngamma && !st; k0 += MESON_CHUNK) {
    MesonArgs m;
    m.g = g;
    m.prop = dfield(prop->ref());
    m.ng = std::min(MESON_CHUNK, ngamma - k0);
    for (int k = 0; k < m.ng; ++k) m.gm[k] = tab[gammas[k0 + k]];
    m.out = buf;
    m.Vxyz = Vxyz;
    meson_site_kernel<<<(unsigned)((2 * g.Vh + 255) / 256), 256, 0, ctx->stream>>>(m);
    row_sum_kernel<<<dim3((unsigned)Lt, (unsigned)m.ng), 256, 0, ctx->stream>>>(buf, Vxyz, scale, dout + (int64_t)k0 * Lt);
    ctx->kernels += 2;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) st = ctx->fail(cuda_status(e), cudaGetErrorString(e));
  }
  if (!st) {
    const cudaError_t e = cudaMemcpyAsync(corr, dout, (size_t)ngamma * Lt * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    st = e == cudaSuccess ? sync_fail(ctx) : ctx->fail(cuda_status(e), cudaGetErrorString(e));
  }
  dfree(buf);
  dfree(dout);
  return st;
}

clg_status clg_meson_correlator(clg_solver S, clg_gauge U, clg_field prop, int ngamma, const int* gammas, double* corr,
                                clg_solve_info* info) {
  if (!S || !U || !info) return CLG_ERR_BAD_ARG;
  if (clg_status st = check_prop(prop, 12, "meson correlator")) return st;
  clg_context_s* ctx = S->ctx;
  if (prop->nrhs != 12) return ctx->fail(CLG_ERR_BAD_ARG, "meson correlator: the propagator field holds 12 right-hand sides");
  clg_field b = nullptr;
  clg_status st = clg_field_create(prop->lat, CLG_FERMION_WILSON, CLG_SUBSET_FULL, CLG_PREC_DOUBLE, 12, prop->param, &b);
  if (st) return st;
  // point sources at the origin, source spin s colour c in right-hand side 3 s + c
  for (int r = 0; r < 12 && !st; ++r) st = clg_field_random(b, r, CLG_SOURCE_POINT, 0, 0, 0, r);
  if (!st) st = clg_solve(S, prop, b, U, CLG_OP_D, nullptr, info);
  clg_field_destroy(b);
  if (st) return st;
  return clg_meson_contract(prop, ngamma, gammas, corr);
}

clg_status clg_condensate_contract(clg_field eta, clg_field psi, double* re_im) {
  if (clg_status st = check_prop(eta, 1, "condensate")) return st;
  if (clg_status st = check_prop(psi, 1, "condensate")) return st;
  clg_context_s* ctx = eta->lat->ctx;
  if (!re_im || eta->lat != psi->lat || eta->nrhs != psi->nrhs)
    return ctx->fail(CLG_ERR_BAD_ARG, "condensate: eta and psi differ in shape");
  if (clg_status st = settle(eta)) return st;
  if (clg_status st = settle(psi)) return st;
  const std::vector<GammaT> tab = gamma_table();
  const int kinds[COND_KINDS] = {G_UNITY, G_1, G_2, G_3, G_4, G_5, G_45, G_1, G_2};
  CondF f;
  f.eta = dfield(eta->ref());
  f.psi = dfield(psi->ref());
  for (int k = 0; k < COND_KINDS; ++k) f.gm[k] = tab[kinds[k]];
  const int nrhs = eta->nrhs;
  double* dout = nullptr;
  clg_status st = dalloc(ctx, (void**)&dout, (size_t)nrhs * 2 * COND_KINDS * sizeof(double));
  if (st) return st;
  f.out = dout;
  st = launch_sites<2 * COND_KINDS>(ctx, f, 0, 2, eta->lat->g.Vh, nrhs);
  std::vector<double> h((size_t)nrhs * 2 * COND_KINDS);
  if (!st) {
    const cudaError_t e = cudaMemcpyAsync(h.data(), dout, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    st = e == cudaSuccess ? sync_fail(ctx) : ctx->fail(cuda_status(e), cudaGetErrorString(e));
  }
  dfree(dout);
  if (st) return st;
  const double iv = 1.0 / (double)eta->lat->g.V;
  for (size_t i = 0; i < h.size(); ++i) re_im[i] = h[i] * iv;
  return CLG_SUCCESS;
}

clg_status clg_chiral_condensate(clg_solver S, clg_gauge U, clg_field eta, clg_field psi, uint64_t seed,
                                 double* re_im, clg_solve_info* info) {
  if (!S || !U || !re_im || !info) return CLG_ERR_BAD_ARG;
  if (clg_status st = check_prop(eta, 1, "condensate")) return st;
  if (clg_status st = check_prop(psi, 1, "condensate")) return st;
  clg_context_s* ctx = S->ctx;
  if (eta->lat != psi->lat || eta->nrhs != psi->nrhs)
    return ctx->fail(CLG_ERR_BAD_ARG, "condensate: eta and psi differ in shape");
  const int n = eta->nrhs;
  clg_status st = CLG_SUCCESS;
  // one Z4 noise vector per right-hand side (EFIT_RandomZ4), all solved in one call
  for (int r = 0; r < n && !st; ++r) st = clg_field_random(eta, r, CLG_SOURCE_Z4, seed, (uint32_t)(r + 1), 0, 0);
  if (!st) st = clg_solve(S, psi, eta, U, CLG_OP_D, nullptr, info);
  if (st) return st;
  std::vector<double> per((size_t)n * 2 * COND_KINDS);
  if ((st = clg_condensate_contract(eta, psi, per.data()))) return st;
  // average over the noise vectors
  for (int k = 0; k < 2 * COND_KINDS; ++k) {
    double s = 0.0;
    for (int r = 0; r < n; ++r) s += per[(size_t)r * 2 * COND_KINDS + k];
    re_im[k] = s / n;
  }
  return CLG_SUCCESS;
}

}  // extern "C"
