// hostkrylov.cuh -- FP64 Krylov building blocks driven from the host: one
// right-hand side, the small dense algebra on the host (dense.h), every
// orthogonalisation one multi-dot launch (up to MD inner products, read back)
// and one linear-combination launch.  Used by the recycled solver (GCRO-DR)
// and by the multi-shift solvers that share one Krylov space over all shifts
// (multi-shift FOM and BiCGStab-M), whose per-cycle work is dominated by the
// operator applications, not by these launches.
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

#include "blas.cuh"
#include "dense.h"

namespace clg {
namespace hk {

using dense::Z;

constexpr int MD = 16;    // inner products per multi-dot launch
constexpr int MAXV = 34;  // vectors per linear combination (m + 1 <= 33, + 1)

template <int NC>
struct MultiDotF {  // out[i] = sum_x conj(v_i(x)) w(x), i < n
  DField w;
  DField v[MD];
  int n;
  double* out;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int, int p, int64_t h, double* acc) const {
    cpx<double> wv[NC];
    ldv<P64, NC, double>(w, 0, p, h, wv);
#pragma unroll
    for (int i = 0; i < MD; ++i) {
      if (i >= n) break;
      cpx<double> a[NC];
      ldv<P64, NC, double>(v[i], 0, p, h, a);
      double re = 0.0, im = 0.0;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        re = fma(a[c].x, wv[c].x, fma(a[c].y, wv[c].y, re));
        im = fma(a[c].x, wv[c].y, fma(-a[c].y, wv[c].x, im));
      }
      acc[2 * i] += re;
      acc[2 * i + 1] += im;
    }
  }
  __device__ void finalize(int, const double* s) const {
    for (int k = 0; k < 2 * n; ++k) out[k] = s[k];
  }
};

template <int NC>
struct LinCombF {  // out = beta out + sum_i c_i v_i
  DField out;
  DField v[MAXV];
  double2 c[MAXV];
  double2 beta;
  int n;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int, int p, int64_t h, double*) const {
    cpx<double> o[NC];
    if (beta.x != 0.0 || beta.y != 0.0) {
      ldv<P64, NC, double>(out, 0, p, h, o);
      const cpx<double> b = mk<double>(beta.x, beta.y);
#pragma unroll
      for (int k = 0; k < NC; ++k) o[k] = b * o[k];
    } else {
#pragma unroll
      for (int k = 0; k < NC; ++k) o[k] = mk<double>(0, 0);
    }
    for (int i = 0; i < n; ++i) {
      cpx<double> a[NC];
      ldv<P64, NC, double>(v[i], 0, p, h, a);
      const cpx<double> ci = mk<double>(c[i].x, c[i].y);
#pragma unroll
      for (int k = 0; k < NC; ++k) o[k] = o[k] + ci * a[k];
    }
    stv<P64, NC, double>(out, 0, p, h, o);
  }
  __device__ void finalize(int, const double*) const {}
};

// device vectors of one shape owned by a solver cache
struct HostVecs : SolveCacheBase {
  clg_context_s* ctx = nullptr;
  std::vector<void*> allocs;
  FieldRef proto;
  FieldRef tmp;  // the operators' temporary (a full field)
  double* dev_out = nullptr;
  ~HostVecs() override {
    for (void* p : allocs) dfree(p);
  }
  clg_status vec(FieldRef& f) {
    void* p = nullptr;
    const size_t bytes = (size_t)proto.blk * proto.nparity;
    if (clg_status st = dalloc(ctx, &p, bytes)) return st;
    allocs.push_back(p);
    f = proto;
    f.data = static_cast<char*>(p);
    return CLG_SUCCESS;
  }
  // a full (both parities) field of the proto's shape: the operators' temporary
  clg_status full_vec(FieldRef& f) {
    const FieldRef keep = proto;
    proto.nparity = 2;
    proto.first_parity = 0;
    proto.rstride = proto.blk * 2;
    const clg_status st = vec(f);
    proto = keep;
    return st;
  }
  clg_status out_buffer() {
    void* p = nullptr;
    if (clg_status st = dalloc(ctx, &p, sizeof(double) * 2 * MD)) return st;
    allocs.push_back(p);
    dev_out = static_cast<double*>(p);
    return CLG_SUCCESS;
  }
};

struct HostKrylov {
  clg_context_s* ctx;
  HostVecs& W;
  const clg_gauge_s* Ug;
  int kind, op, nc;
  double param;
  int64_t Vh;
  int apps = 0;

  clg_status apply(const FieldRef& out, const FieldRef& in) {
    ++apps;
    return apply_op(ctx, op, Ug, kind, param, out, in, &W.tmp, make_double2(1.0, 0.0), 1);
  }
  // out[i] = v_i^+ w for the n vectors vs (n arbitrary), read to the host
  clg_status dots(const FieldRef& w, const std::vector<const FieldRef*>& vs, std::vector<Z>& out) {
    out.assign(vs.size(), Z(0.0, 0.0));
    for (size_t i0 = 0; i0 < vs.size(); i0 += MD) {
      const int n = (int)std::min<size_t>(MD, vs.size() - i0);
      clg_status st;
      if (nc == 12) {
        MultiDotF<12> f;
        f.w = dfield(w);
        for (int i = 0; i < MD; ++i) f.v[i] = dfield(*vs[i0 + std::min(i, n - 1)]);
        f.n = n;
        f.out = W.dev_out;
        st = launch_sites<2 * MD>(ctx, f, W.proto.first_parity, W.proto.nparity, Vh, 1);
      } else {
        MultiDotF<3> f;
        f.w = dfield(w);
        for (int i = 0; i < MD; ++i) f.v[i] = dfield(*vs[i0 + std::min(i, n - 1)]);
        f.n = n;
        f.out = W.dev_out;
        st = launch_sites<2 * MD>(ctx, f, W.proto.first_parity, W.proto.nparity, Vh, 1);
      }
      if (st) return st;
      double h[2 * MD];
      cudaError_t e = cudaMemcpyAsync(h, W.dev_out, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, ctx->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
      if (e != cudaSuccess) return ctx->fail(cuda_status(e), cudaGetErrorString(e));
      for (int i = 0; i < n; ++i) out[i0 + i] = Z(h[2 * i], h[2 * i + 1]);
    }
    return CLG_SUCCESS;
  }
  double norm(const FieldRef& a) {
    std::vector<Z> d;
    if (dots(a, {&a}, d)) return -1.0;
    return std::sqrt(std::max(d[0].real(), 0.0));
  }
  // out = beta out + sum_i c_i v_i
  clg_status lincomb(const FieldRef& out, Z beta, const std::vector<const FieldRef*>& vs, const std::vector<Z>& c) {
    if (vs.size() > (size_t)MAXV) return ctx->fail(CLG_ERR_UNSUPPORTED, "too many vectors in one linear combination");
    auto fill = [&](auto& f) {
      f.out = dfield(out);
      f.n = (int)vs.size();
      f.beta = make_double2(beta.real(), beta.imag());
      for (size_t i = 0; i < vs.size(); ++i) {
        f.v[i] = dfield(*vs[i]);
        f.c[i] = make_double2(c[i].real(), c[i].imag());
      }
    };
    if (nc == 12) {
      LinCombF<12> f;
      fill(f);
      return launch_sites<0>(ctx, f, W.proto.first_parity, W.proto.nparity, Vh, 1);
    }
    LinCombF<3> f;
    fill(f);
    return launch_sites<0>(ctx, f, W.proto.first_parity, W.proto.nparity, Vh, 1);
  }
  clg_status copy(const FieldRef& dst, const FieldRef& src) { return lincomb(dst, Z(0.0, 0.0), {&src}, {Z(1.0, 0.0)}); }
  clg_status scale(const FieldRef& a, Z s) { return lincomb(a, s, {}, {}); }
  // w <- w - sum_i (v_i^+ w) v_i, twice; the coefficients of both passes summed into h
  clg_status orthogonalise(const FieldRef& w, const std::vector<const FieldRef*>& vs, std::vector<Z>& h) {
    h.assign(vs.size(), Z(0.0, 0.0));
    for (int pass = 0; pass < 2; ++pass) {
      std::vector<Z> d;
      if (clg_status st = dots(w, vs, d)) return st;
      std::vector<Z> neg(d.size());
      for (size_t i = 0; i < d.size(); ++i) {
        h[i] += d[i];
        neg[i] = -d[i];
      }
      if (clg_status st = lincomb(w, Z(1.0, 0.0), vs, neg)) return st;
    }
    return CLG_SUCCESS;
  }
};

}  // namespace hk
}  // namespace clg
