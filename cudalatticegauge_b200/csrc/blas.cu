// blas.cu -- field BLAS of CField (Data/Field/CField.h:127-201) on the
// even-odd structure-of-arrays layout: Dot (sum conj(a) b, FP64 accumulate),
// norm, axpby, precision-converting copy, zero.
#include "blas.cuh"

namespace clg {

namespace {

template <int P, int NC>
struct DotF {
  DField a, b;
  double* out;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int rhs, int p, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> va[NC], vb[NC];
    ldv<P, NC, AT>(a, rhs, p, h, va);
    ldv<P, NC, AT>(b, rhs, p, h, vb);
    acc_dot<NC, AT>(va, vb, acc);
  }
  __device__ void finalize(int rhs, const double* s) const {
    out[2 * rhs] = s[0];
    out[2 * rhs + 1] = s[1];
  }
};

template <int P, int NC>
struct Norm2F {
  DField a;
  double* out;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int rhs, int p, int64_t h, double* acc) const {
    using AT = typename AccT<P>::T;
    cpx<AT> va[NC];
    ldv<P, NC, AT>(a, rhs, p, h, va);
    acc[0] += site_norm2<NC, AT>(va);
  }
  __device__ void finalize(int rhs, const double* s) const { out[rhs] = s[0]; }
};

template <int P, int NC>
struct AxpbyF {
  DField y, x;
  double2 a, b;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int rhs, int p, int64_t h, double*) const {
    using AT = typename AccT<P>::T;
    cpx<AT> vy[NC], vx[NC];
    ldv<P, NC, AT>(x, rhs, p, h, vx);
    ldv<P, NC, AT>(y, rhs, p, h, vy);
    const cpx<AT> ca = mk<AT>((AT)a.x, (AT)a.y), cb = mk<AT>((AT)b.x, (AT)b.y);
#pragma unroll
    for (int k = 0; k < NC; ++k) vy[k] = ca * vx[k] + cb * vy[k];
    stv<P, NC, AT>(y, rhs, p, h, vy);
  }
  __device__ void finalize(int, const double*) const {}
};

template <int PD, int PS, int NC>
struct CopyF {
  DField d, s;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int rhs, int p, int64_t h, double*) const {
    cpx<double> v[NC];
    load_site<PS, NC, double>(s.base(rhs, p), s.nbase(rhs, p), s.Vh, h, v);
    store_site<PD, NC, double>(d.base(rhs, p), d.nbase(rhs, p), d.Vh, h, v);
  }
  __device__ void finalize(int, const double*) const {}
};

template <int P, int NC>
struct ZeroF {
  DField y;
  __device__ bool active(int) const { return true; }
  __device__ void operator()(int rhs, int p, int64_t h, double*) const {
    using AT = typename AccT<P>::T;
    cpx<AT> v[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) v[k] = mk<AT>(0, 0);
    stv<P, NC, AT>(y, rhs, p, h, v);
  }
  __device__ void finalize(int, const double*) const {}
};

bool same_shape(const FieldRef& a, const FieldRef& b) {
  return a.nc == b.nc && a.nrhs == b.nrhs && a.Vh == b.Vh && a.first_parity == b.first_parity && a.nparity == b.nparity;
}

}  // namespace

clg_status blas_copy_strided(clg_context_s* ctx, const FieldRef& d, const FieldRef& s) {
  if (d.nc != s.nc || d.nrhs != s.nrhs || d.first_parity != s.first_parity || d.nparity != s.nparity)
    return ctx->fail(CLG_ERR_BAD_ARG, "strided copy: field shapes differ");
  const int64_t vh = d.Vh < s.Vh ? d.Vh : s.Vh;
  auto go = [&](auto PD, auto PS, auto NC) {
    CopyF<PD.value, PS.value, NC.value> f{dfield(d), dfield(s)};
    return launch_sites<0>(ctx, f, d.first_parity, d.nparity, vh, d.nrhs);
  };
  if (d.prec != CLG_PREC_DOUBLE || s.prec != CLG_PREC_DOUBLE)
    return ctx->fail(CLG_ERR_BAD_ARG, "strided copy: FP64 fields");
  return d.nc == 12 ? go(std::integral_constant<int, P64>{}, std::integral_constant<int, P64>{}, std::integral_constant<int, 12>{})
                    : go(std::integral_constant<int, P64>{}, std::integral_constant<int, P64>{}, std::integral_constant<int, 3>{});
}

clg_status blas_dot(clg_context_s* ctx, const FieldRef& a, const FieldRef& b, double* dev_out) {
  if (!same_shape(a, b) || a.prec != b.prec) return ctx->fail(CLG_ERR_BAD_ARG, "dot: field shapes differ");
  return with_pn(a.prec, a.nc, [&](auto P, auto NC) {
    DotF<P.value, NC.value> f{dfield(a), dfield(b), dev_out};
    return launch_sites<2>(ctx, f, a.first_parity, a.nparity, a.Vh, a.nrhs);
  });
}

clg_status blas_norm2(clg_context_s* ctx, const FieldRef& a, double* dev_out) {
  return with_pn(a.prec, a.nc, [&](auto P, auto NC) {
    Norm2F<P.value, NC.value> f{dfield(a), dev_out};
    return launch_sites<1>(ctx, f, a.first_parity, a.nparity, a.Vh, a.nrhs);
  });
}

clg_status blas_axpby(clg_context_s* ctx, const FieldRef& y, double2 a, const FieldRef& x, double2 b) {
  if (!same_shape(x, y) || x.prec != y.prec) return ctx->fail(CLG_ERR_BAD_ARG, "axpby: field shapes differ");
  return with_pn(y.prec, y.nc, [&](auto P, auto NC) {
    AxpbyF<P.value, NC.value> f{dfield(y), dfield(x), a, b};
    return launch_sites<0>(ctx, f, y.first_parity, y.nparity, y.Vh, y.nrhs);
  });
}

clg_status blas_copy(clg_context_s* ctx, const FieldRef& d, const FieldRef& s) {
  if (!same_shape(d, s)) return ctx->fail(CLG_ERR_BAD_ARG, "copy: field shapes differ");
  auto go = [&](auto PD, auto PS, auto NC) {
    CopyF<PD.value, PS.value, NC.value> f{dfield(d), dfield(s)};
    return launch_sites<0>(ctx, f, d.first_parity, d.nparity, d.Vh, d.nrhs);
  };
  using I0 = std::integral_constant<int, 0>;
  using I1 = std::integral_constant<int, 1>;
  using I2 = std::integral_constant<int, 2>;
  auto by_src = [&](auto PD, auto NC) -> clg_status {
    if (s.prec == 0) return go(PD, I0{}, NC);
    if (s.prec == 1) return go(PD, I1{}, NC);
    return go(PD, I2{}, NC);
  };
  return with_pn(d.prec, d.nc, by_src);
}

clg_status blas_zero(clg_context_s* ctx, const FieldRef& y) {
  return with_pn(y.prec, y.nc, [&](auto P, auto NC) {
    ZeroF<P.value, NC.value> f{dfield(y)};
    return launch_sites<0>(ctx, f, y.first_parity, y.nparity, y.Vh, y.nrhs);
  });
}

}  // namespace clg
