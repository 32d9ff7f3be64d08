// fileio.cu -- gauge-configuration and fermion-field files in the reference's
// formats, with the MD5 of every file written.
//
//   CLGBin double / float    18 reals per link (9 complex, row-major), links
//                            l = site*4 + mu in CLGBin site order
//                            (CFieldGaugeSU3::InitialFieldWithFile / SaveToFile,
//                            Data/Field/Gauge/CFieldGaugeSU3.cu:1080-1222,
//                            Data/Field/CField.cpp:32-72); fermion fields 24
//                            (Wilson) or 6 (staggered) reals per site.
//   CLGBin compressed        9 reals per link: the logarithm A = log U
//                            (anti-hermitian) as A01, A02, A12 (re, im) and the
//                            imaginary diagonal (SaveToCompressedFile,
//                            CFieldGaugeSU3.cu:1651-1690; InitialWithByteCompressed
//                            :1224-1265 reads it back through U = exp A).
//                            The reference writes its build's Real: double,
//                            or float in a single-precision build.
//   Bridge++ binary / text   18 doubles per link in Bridge++ site order
//                            (x fastest), big-endian in the binary file, one
//                            value per line in the text file (:1089-1125).
//
// log and exp of a link run on the device: a cyclic complex Jacobi
// eigensolver for 3x3 hermitian matrices (Golub & Van Loan, Matrix
// Computations, 8.5; the complex rotation is the real one after a phase that
// makes the pivot real).  exp(A) = V diag(exp(i w)) V^+ with -iA = V diag(w) V^+;
// log(U) = V diag(i theta) V^+ with V the eigenvectors of the hermitian
// (U + U^+)/2 + c (U - U^+)/(2i) (which commutes with U and has distinct
// eigenvalues for distinct eigenphases unless c is unlucky: a second c is tried)
// and theta the principal arguments of V^+ U V.
//
// MD5 follows RFC 1321.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace clg {

namespace {

// ------------------------------------------------------------------ MD5 (RFC 1321)
struct Md5 {
  uint32_t s[4] = {0x67452301u, 0xefcdab89u, 0x98badcfeu, 0x10325476u};
  uint64_t len = 0;
  unsigned char buf[64];
  size_t fill = 0;

  static uint32_t rotl(uint32_t x, int c) { return (x << c) | (x >> (32 - c)); }

  void block(const unsigned char* p) {
    // per-round shift amounts and the sine table K[i] = floor(2^32 |sin(i + 1)|)
    static const int R[64] = {7, 12, 17, 22, 7, 12, 17, 22, 7, 12, 17, 22, 7, 12, 17, 22,
                              5, 9,  14, 20, 5, 9,  14, 20, 5, 9,  14, 20, 5, 9,  14, 20,
                              4, 11, 16, 23, 4, 11, 16, 23, 4, 11, 16, 23, 4, 11, 16, 23,
                              6, 10, 15, 21, 6, 10, 15, 21, 6, 10, 15, 21, 6, 10, 15, 21};
    static const std::array<uint32_t, 64> K = [] {
      std::array<uint32_t, 64> k{};
      for (int i = 0; i < 64; ++i) k[i] = (uint32_t)(uint64_t)std::floor(std::fabs(std::sin((double)(i + 1))) * 4294967296.0);
      return k;
    }();
    uint32_t M[16];
    for (int i = 0; i < 16; ++i)
      M[i] = (uint32_t)p[4 * i] | ((uint32_t)p[4 * i + 1] << 8) | ((uint32_t)p[4 * i + 2] << 16) |
             ((uint32_t)p[4 * i + 3] << 24);
    uint32_t a = s[0], b = s[1], c = s[2], d = s[3];
    for (int i = 0; i < 64; ++i) {
      uint32_t f;
      int g;
      if (i < 16) {
        f = (b & c) | (~b & d);
        g = i;
      } else if (i < 32) {
        f = (d & b) | (~d & c);
        g = (5 * i + 1) & 15;
      } else if (i < 48) {
        f = b ^ c ^ d;
        g = (3 * i + 5) & 15;
      } else {
        f = c ^ (b | ~d);
        g = (7 * i) & 15;
      }
      const uint32_t t = d;
      d = c;
      c = b;
      b = b + rotl(a + f + K[i] + M[g], R[i]);
      a = t;
    }
    s[0] += a;
    s[1] += b;
    s[2] += c;
    s[3] += d;
  }
  void update(const void* data, size_t n) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    len += n;
    while (n) {
      const size_t k = std::min(n, 64 - fill);
      memcpy(buf + fill, p, k);
      fill += k;
      p += k;
      n -= k;
      if (fill == 64) {
        block(buf);
        fill = 0;
      }
    }
  }
  std::string hex() {
    const uint64_t bits = len * 8;
    const unsigned char one = 0x80, zero = 0;
    update(&one, 1);
    while (fill != 56) update(&zero, 1);
    unsigned char L[8];
    for (int i = 0; i < 8; ++i) L[i] = (unsigned char)(bits >> (8 * i));
    update(L, 8);
    char out[33];
    for (int i = 0; i < 16; ++i) snprintf(out + 2 * i, 3, "%02x", (s[i / 4] >> (8 * (i % 4))) & 0xffu);
    return std::string(out, 32);
  }
};

std::string md5_hex(const void* data, size_t n) {
  Md5 m;
  m.update(data, n);
  return m.hex();
}

// ------------------------------------------------------------------ files
bool read_file(const char* path, std::vector<char>& out) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  fseek(f, 0, SEEK_END);
  const long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  if (n < 0) {
    fclose(f);
    return false;
  }
  out.resize((size_t)n);
  const size_t got = n ? fread(out.data(), 1, (size_t)n, f) : 0;
  fclose(f);
  return got == (size_t)n;
}

bool write_file(const char* path, const void* data, size_t n) {
  FILE* f = fopen(path, "wb");
  if (!f) return false;
  const size_t put = n ? fwrite(data, 1, n, f) : 0;
  const bool ok = fclose(f) == 0 && put == n;
  return ok;
}

void byteswap8(char* p, size_t count) {
  for (size_t i = 0; i < count; ++i) {
    char* q = p + 8 * i;
    for (int j = 0; j < 4; ++j) std::swap(q[j], q[7 - j]);
  }
}

// ------------------------------------------------------------------ link log / exp
using Z = cpx<double>;

__device__ __forceinline__ Z zconj(Z a) { return mk<double>(a.x, -a.y); }

__device__ void mat3_mul(const Z a[9], const Z b[9], Z o[9]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) o[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
}
// o = a^+ b
__device__ void mat3_dag_mul(const Z a[9], const Z b[9], Z o[9]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      o[3 * i + j] = zconj(a[i]) * b[j] + zconj(a[3 + i]) * b[3 + j] + zconj(a[6 + i]) * b[6 + j];
}

// a (hermitian, overwritten) = V diag(w) V^+; bounded number of sweeps
__device__ void herm3_eig(Z a[9], Z v[9], double w[3]) {
  for (int k = 0; k < 9; ++k) v[k] = mk<double>((k % 4 == 0) ? 1.0 : 0.0, 0.0);
  for (int sweep = 0; sweep < 24; ++sweep) {
    const double off = a[1].x * a[1].x + a[1].y * a[1].y + a[2].x * a[2].x + a[2].y * a[2].y + a[5].x * a[5].x +
                       a[5].y * a[5].y;
    const double dg = a[0].x * a[0].x + a[4].x * a[4].x + a[8].x * a[8].x;
    if (off <= 1e-34 * dg || off < 1e-300) break;
    for (int pq = 0; pq < 3; ++pq) {
      const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
      const Z apq = a[3 * p + q];
      const double r = sqrt(apq.x * apq.x + apq.y * apq.y);
      if (r < 1e-300) continue;
      const Z e = mk<double>(apq.x / r, apq.y / r);  // a_pq = r e
      const double tau = (a[4 * q].x - a[4 * p].x) / (2.0 * r);
      const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
      const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
      // J = D G: D = diag(1, .., conj(e) at q), G the real rotation (c, s; -s, c) in (p, q)
      Z J[9];
      for (int k = 0; k < 9; ++k) J[k] = mk<double>((k % 4 == 0) ? 1.0 : 0.0, 0.0);
      J[3 * p + p] = mk<double>(c, 0.0);
      J[3 * p + q] = mk<double>(s, 0.0);
      J[3 * q + p] = (-s) * zconj(e);
      J[3 * q + q] = c * zconj(e);
      Z t1[9], t2[9];
      mat3_mul(a, J, t1);
      mat3_dag_mul(J, t1, t2);
      for (int k = 0; k < 9; ++k) a[k] = t2[k];
      // keep a exactly hermitian against rounding
      for (int i = 0; i < 3; ++i) {
        a[4 * i].y = 0.0;
        for (int j = i + 1; j < 3; ++j) a[3 * j + i] = zconj(a[3 * i + j]);
      }
      mat3_mul(v, J, t1);
      for (int k = 0; k < 9; ++k) v[k] = t1[k];
    }
  }
  for (int i = 0; i < 3; ++i) w[i] = a[4 * i].x;
}

// U = exp(A), A anti-hermitian given by its 9 stored reals
__global__ void link_exp_kernel(const double* __restrict__ in9, double* __restrict__ out18, int64_t nlinks) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nlinks) return;
  const double* o = in9 + 9 * l;
  // H = -i A: H_ij = (A_ij.y, -A_ij.x)
  Z A[9];
  A[1] = mk<double>(o[0], o[1]);
  A[3] = mk<double>(-o[0], o[1]);
  A[2] = mk<double>(o[2], o[3]);
  A[6] = mk<double>(-o[2], o[3]);
  A[5] = mk<double>(o[4], o[5]);
  A[7] = mk<double>(-o[4], o[5]);
  A[0] = mk<double>(0.0, o[6]);
  A[4] = mk<double>(0.0, o[7]);
  A[8] = mk<double>(0.0, o[8]);
  Z H[9], V[9];
  for (int k = 0; k < 9; ++k) H[k] = mk<double>(A[k].y, -A[k].x);
  double w[3];
  herm3_eig(H, V, w);
  Z E[3];
  for (int k = 0; k < 3; ++k) {
    double sn, cs;
    sincos(w[k], &sn, &cs);
    E[k] = mk<double>(cs, sn);
  }
  double* u = out18 + 18 * l;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      Z acc = mk<double>(0, 0);
      for (int k = 0; k < 3; ++k) acc = acc + V[3 * i + k] * E[k] * zconj(V[3 * j + k]);
      u[2 * (3 * i + j)] = acc.x;
      u[2 * (3 * i + j) + 1] = acc.y;
    }
}

// A = log(U) (principal branch), stored as 9 reals; *fail counts links whose
// eigenvectors could not be separated.  With V from the hermitian above,
// D = V^+ U V = Lambda + N, N the small off-diagonal part left by rounding
// (large when two eigenphases give close eigenvalues of that hermitian: then
// another c is tried).  log(Lambda + N) = log Lambda + L(N) to first order in N,
// L the Frechet derivative of the logarithm at a diagonal matrix:
// L(N)_jk = N_jk (log l_j - log l_k) / (l_j - l_k), = N_jk / l_j for l_j = l_k.
__global__ void link_log_kernel(const double* __restrict__ in18, double* __restrict__ out9, int64_t nlinks,
                                unsigned int* fail) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nlinks) return;
  const double* u = in18 + 18 * l;
  Z U[9];
  for (int k = 0; k < 9; ++k) U[k] = mk<double>(u[2 * k], u[2 * k + 1]);
  const double cs[3] = {0.6180339887498949, -1.3247179572447460, 2.7182818284590452};
  Z Vb[9], Db[9];
  double best = 1e300;
  for (int attempt = 0; attempt < 3 && best > 1e-20; ++attempt) {
    const double c = cs[attempt];
    Z M[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        const Z a = U[3 * i + j], b = zconj(U[3 * j + i]);
        // (a + b)/2 + c (a - b)/(2i) = (a + b)/2 - i c (a - b)/2
        const Z s = mk<double>(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
        const Z d = mk<double>(0.5 * (a.x - b.x), 0.5 * (a.y - b.y));
        M[3 * i + j] = mk<double>(s.x + c * d.y, s.y - c * d.x);
      }
    Z V[9], T[9], D[9];
    double w[3];
    herm3_eig(M, V, w);
    mat3_mul(U, V, T);
    mat3_dag_mul(V, T, D);
    double off = 0.0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        if (i != j) off += D[3 * i + j].x * D[3 * i + j].x + D[3 * i + j].y * D[3 * i + j].y;
    if (off < best) {
      best = off;
      for (int k = 0; k < 9; ++k) {
        Vb[k] = V[k];
        Db[k] = D[k];
      }
    }
  }
  double* o = out9 + 9 * l;
  if (!(best <= 1e-12)) {
    atomicAdd(fail, 1u);
    for (int k = 0; k < 9; ++k) o[k] = 0.0;
    return;
  }
  double th[3];
  Z lam[3];
  for (int k = 0; k < 3; ++k) {
    th[k] = atan2(Db[4 * k].y, Db[4 * k].x);
    double sn, cn;
    sincos(th[k], &sn, &cn);
    lam[k] = mk<double>(cn, sn);
  }
  Z B[9];
  for (int j = 0; j < 3; ++j)
    for (int k = 0; k < 3; ++k) {
      if (j == k) {
        B[4 * j] = mk<double>(0.0, th[j]);
        continue;
      }
      const Z dl = lam[j] - lam[k];
      const double dl2 = dl.x * dl.x + dl.y * dl.y;
      Z f;
      if (dl2 > 1e-16) {
        // i (th_j - th_k) / dl
        const Z num = mk<double>(0.0, th[j] - th[k]);
        f = mk<double>((num.x * dl.x + num.y * dl.y) / dl2, (num.y * dl.x - num.x * dl.y) / dl2);
      } else {
        f = zconj(lam[j]);  // 1 / l_j
      }
      B[3 * j + k] = f * Db[3 * j + k];
    }
  Z T[9], A[9];
  // A = V B V^+
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) T[3 * i + k] = Vb[3 * i] * B[k] + Vb[3 * i + 1] * B[3 + k] + Vb[3 * i + 2] * B[6 + k];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      A[3 * i + j] = T[3 * i] * zconj(Vb[3 * j]) + T[3 * i + 1] * zconj(Vb[3 * j + 1]) + T[3 * i + 2] * zconj(Vb[3 * j + 2]);
  // stored as the anti-hermitian part (the upper triangle and the imaginary diagonal)
  o[0] = 0.5 * (A[1].x - A[3].x);
  o[1] = 0.5 * (A[1].y + A[3].y);
  o[2] = 0.5 * (A[2].x - A[6].x);
  o[3] = 0.5 * (A[2].y + A[6].y);
  o[4] = 0.5 * (A[5].x - A[7].x);
  o[5] = 0.5 * (A[5].y + A[7].y);
  o[6] = A[0].y;
  o[7] = A[4].y;
  o[8] = A[8].y;
}

clg_status copy_status(clg_context_s* ctx, cudaError_t e) {
  return e == cudaSuccess ? CLG_SUCCESS : ctx->fail(cuda_status(e), cudaGetErrorString(e));
}

void put_md5(const std::string& h, char* md5_hex_out) {
  if (md5_hex_out) {
    memcpy(md5_hex_out, h.data(), 32);
    md5_hex_out[32] = 0;
  }
}

}  // namespace

}  // namespace clg

using namespace clg;

extern "C" {

clg_status clg_md5(const void* data, size_t bytes, char* md5_hex_out) {
  if ((!data && bytes) || !md5_hex_out) return CLG_ERR_BAD_ARG;
  put_md5(md5_hex(data, bytes), md5_hex_out);
  return CLG_SUCCESS;
}

clg_status clg_gauge_save(clg_gauge g, const char* path, int format, char* md5_hex_out) {
  if (!g || !path) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = g->lat->ctx;
  const int64_t nl = 4 * g->lat->g.V;
  std::vector<double> u18((size_t)nl * 18);
  std::vector<char> bytes;
  clg_status st = CLG_SUCCESS;
  switch (format) {
    case CLG_FILE_CLGBIN_DOUBLE:
    case CLG_FILE_CLGBIN_FLOAT:
    case CLG_FILE_BRIDGEPP_BIN:
    case CLG_FILE_BRIDGEPP_TXT: {
      if ((st = clg_gauge_export(g, u18.data(), 0))) return st;
      if (format == CLG_FILE_CLGBIN_DOUBLE) {
        bytes.resize(u18.size() * 8);
        memcpy(bytes.data(), u18.data(), bytes.size());
      } else if (format == CLG_FILE_CLGBIN_FLOAT) {
        bytes.resize(u18.size() * 4);
        float* f = reinterpret_cast<float*>(bytes.data());
        for (size_t i = 0; i < u18.size(); ++i) f[i] = (float)u18[i];
      } else {
        // CLGBin -> Bridge++ site order (x fastest)
        const int* L = g->lat->g.L;
        std::vector<double> b(u18.size());
        for (int x = 0; x < L[0]; ++x)
          for (int y = 0; y < L[1]; ++y)
            for (int z = 0; z < L[2]; ++z)
              for (int t = 0; t < L[3]; ++t) {
                const int64_t s = (((int64_t)x * L[1] + y) * L[2] + z) * L[3] + t;
                const int64_t sb = x + (int64_t)L[0] * (y + (int64_t)L[1] * (z + (int64_t)L[2] * t));
                memcpy(&b[(size_t)sb * 72], &u18[(size_t)s * 72], 72 * sizeof(double));
              }
        if (format == CLG_FILE_BRIDGEPP_BIN) {
          bytes.resize(b.size() * 8);
          memcpy(bytes.data(), b.data(), bytes.size());
          byteswap8(bytes.data(), b.size());
        } else {
          std::string txt;
          txt.reserve(b.size() * 26);
          char line[40];
          for (double v : b) {
            const int n = snprintf(line, sizeof line, "%.17g\n", v);
            txt.append(line, (size_t)n);
          }
          bytes.assign(txt.begin(), txt.end());
        }
      }
      break;
    }
    case CLG_FILE_CLGBIN_COMPRESSED:
    case CLG_FILE_CLGBIN_COMPRESSED_FLOAT: {
      if (!g->su3) return ctx->fail(CLG_ERR_BAD_ARG, "compressed files hold SU(3) links (log U)");
      double *d18 = nullptr, *d9 = nullptr;
      unsigned int* dfail = nullptr;
      if ((st = dalloc(ctx, (void**)&d18, (size_t)nl * 18 * 8))) return st;
      if ((st = dalloc(ctx, (void**)&d9, (size_t)nl * 9 * 8 + 16))) {
        dfree(d18);
        return st;
      }
      dfail = reinterpret_cast<unsigned int*>(d9 + nl * 9);
      std::vector<double> h9((size_t)nl * 9);
      unsigned int nfail = 0;
      st = clg_gauge_export(g, d18, 1);
      if (!st) st = copy_status(ctx, cudaMemsetAsync(dfail, 0, sizeof(unsigned int), ctx->stream));
      if (!st) {
        link_log_kernel<<<(unsigned)((nl + 127) / 128), 128, 0, ctx->stream>>>(d18, d9, nl, dfail);
        ctx->kernels++;
        st = copy_status(ctx, cudaGetLastError());
      }
      if (!st) st = copy_status(ctx, cudaMemcpyAsync(h9.data(), d9, h9.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
      if (!st) st = copy_status(ctx, cudaMemcpyAsync(&nfail, dfail, sizeof nfail, cudaMemcpyDeviceToHost, ctx->stream));
      if (!st) st = copy_status(ctx, cudaStreamSynchronize(ctx->stream));
      dfree(d18);
      dfree(d9);
      if (st) return st;
      if (nfail) return ctx->fail(CLG_ERR_BAD_ARG, "compressed save: " + std::to_string(nfail) + " links without a logarithm");
      if (format == CLG_FILE_CLGBIN_COMPRESSED) {
        bytes.resize(h9.size() * 8);
        memcpy(bytes.data(), h9.data(), bytes.size());
      } else {
        bytes.resize(h9.size() * 4);
        float* f = reinterpret_cast<float*>(bytes.data());
        for (size_t i = 0; i < h9.size(); ++i) f[i] = (float)h9[i];
      }
      break;
    }
    default:
      return ctx->fail(CLG_ERR_BAD_ARG, "unknown gauge file format");
  }
  if (!write_file(path, bytes.data(), bytes.size()))
    return ctx->fail(CLG_ERR_BAD_ARG, std::string("cannot write ") + path);
  put_md5(md5_hex(bytes.data(), bytes.size()), md5_hex_out);
  return CLG_SUCCESS;
}

clg_status clg_gauge_load(clg_gauge g, const char* path, int format) {
  if (!g || !path) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = g->lat->ctx;
  const int64_t nl = 4 * g->lat->g.V;
  std::vector<char> bytes;
  if (!read_file(path, bytes)) return ctx->fail(CLG_ERR_BAD_ARG, std::string("cannot read ") + path);
  auto size_error = [&](size_t want) {
    return ctx->fail(CLG_ERR_BAD_ARG, std::string(path) + ": " + std::to_string(bytes.size()) + " bytes, expected " +
                                          std::to_string(want) + " for this lattice and format");
  };
  std::vector<double> u;
  switch (format) {
    case CLG_FILE_CLGBIN_DOUBLE:
    case CLG_FILE_BRIDGEPP_BIN: {
      if (bytes.size() != (size_t)nl * 18 * 8) return size_error((size_t)nl * 18 * 8);
      if (format == CLG_FILE_BRIDGEPP_BIN) byteswap8(bytes.data(), (size_t)nl * 18);
      u.resize((size_t)nl * 18);
      memcpy(u.data(), bytes.data(), bytes.size());
      return clg_gauge_import(g, u.data(), format == CLG_FILE_BRIDGEPP_BIN ? CLG_LAYOUT_BRIDGEPP : CLG_LAYOUT_CLGBIN, 0);
    }
    case CLG_FILE_CLGBIN_FLOAT: {
      if (bytes.size() != (size_t)nl * 18 * 4) return size_error((size_t)nl * 18 * 4);
      u.resize((size_t)nl * 18);
      const float* f = reinterpret_cast<const float*>(bytes.data());
      for (size_t i = 0; i < u.size(); ++i) u[i] = (double)f[i];
      return clg_gauge_import(g, u.data(), CLG_LAYOUT_CLGBIN, 0);
    }
    case CLG_FILE_BRIDGEPP_TXT: {
      bytes.push_back(0);
      u.reserve((size_t)nl * 18);
      const char* p = bytes.data();
      char* end = nullptr;
      for (;;) {
        const double v = strtod(p, &end);
        if (end == p) break;
        u.push_back(v);
        p = end;
      }
      while (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t') ++p;
      if (*p != 0 || u.size() != (size_t)nl * 18)
        return ctx->fail(CLG_ERR_BAD_ARG, std::string(path) + ": " + std::to_string(u.size()) +
                                              " numbers read, expected " + std::to_string(nl * 18));
      return clg_gauge_import(g, u.data(), CLG_LAYOUT_BRIDGEPP, 0);
    }
    case CLG_FILE_CLGBIN_COMPRESSED:
    case CLG_FILE_CLGBIN_COMPRESSED_FLOAT: {
      const size_t rs = format == CLG_FILE_CLGBIN_COMPRESSED ? 8 : 4;
      if (bytes.size() != (size_t)nl * 9 * rs) return size_error((size_t)nl * 9 * rs);
      std::vector<double> h9((size_t)nl * 9);
      if (rs == 8) {
        memcpy(h9.data(), bytes.data(), bytes.size());
      } else {
        const float* f = reinterpret_cast<const float*>(bytes.data());
        for (size_t i = 0; i < h9.size(); ++i) h9[i] = (double)f[i];
      }
      double *d9 = nullptr, *d18 = nullptr;
      clg_status st = dalloc(ctx, (void**)&d9, h9.size() * 8);
      if (st) return st;
      if ((st = dalloc(ctx, (void**)&d18, (size_t)nl * 18 * 8))) {
        dfree(d9);
        return st;
      }
      st = copy_status(ctx, cudaMemcpyAsync(d9, h9.data(), h9.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
      if (!st) {
        link_exp_kernel<<<(unsigned)((nl + 127) / 128), 128, 0, ctx->stream>>>(d9, d18, nl);
        ctx->kernels++;
        st = copy_status(ctx, cudaGetLastError());
      }
      if (!st) st = clg_gauge_import(g, d18, CLG_LAYOUT_CLGBIN, 1);
      if (!st) st = copy_status(ctx, cudaStreamSynchronize(ctx->stream));
      dfree(d9);
      dfree(d18);
      return st;
    }
    default:
      return ctx->fail(CLG_ERR_BAD_ARG, "unknown gauge file format");
  }
}

clg_status clg_field_save(clg_field f, int rhs, const char* path, int format, char* md5_hex_out) {
  if (!f || !path || rhs < 0 || rhs >= f->nrhs) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = f->lat->ctx;
  if (format != CLG_FILE_CLGBIN_DOUBLE && format != CLG_FILE_CLGBIN_FLOAT)
    return ctx->fail(CLG_ERR_BAD_ARG, "fermion fields are saved as CLGBin double or float");
  const size_t n = (size_t)f->lat->g.V * 2 * f->nc();
  std::vector<double> d(n);
  clg_status st = clg_field_export(f, rhs, d.data(), 0);
  if (st) return st;
  std::vector<char> bytes;
  if (format == CLG_FILE_CLGBIN_DOUBLE) {
    bytes.resize(n * 8);
    memcpy(bytes.data(), d.data(), bytes.size());
  } else {
    bytes.resize(n * 4);
    float* p = reinterpret_cast<float*>(bytes.data());
    for (size_t i = 0; i < n; ++i) p[i] = (float)d[i];
  }
  if (!write_file(path, bytes.data(), bytes.size()))
    return ctx->fail(CLG_ERR_BAD_ARG, std::string("cannot write ") + path);
  put_md5(md5_hex(bytes.data(), bytes.size()), md5_hex_out);
  return CLG_SUCCESS;
}

clg_status clg_field_load(clg_field f, int rhs, const char* path, int format) {
  if (!f || !path || rhs < 0 || rhs >= f->nrhs) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = f->lat->ctx;
  if (format != CLG_FILE_CLGBIN_DOUBLE && format != CLG_FILE_CLGBIN_FLOAT)
    return ctx->fail(CLG_ERR_BAD_ARG, "fermion fields are read as CLGBin double or float");
  const size_t n = (size_t)f->lat->g.V * 2 * f->nc();
  const size_t rs = format == CLG_FILE_CLGBIN_DOUBLE ? 8 : 4;
  std::vector<char> bytes;
  if (!read_file(path, bytes)) return ctx->fail(CLG_ERR_BAD_ARG, std::string("cannot read ") + path);
  if (bytes.size() != n * rs)
    return ctx->fail(CLG_ERR_BAD_ARG, std::string(path) + ": " + std::to_string(bytes.size()) + " bytes, expected " +
                                          std::to_string(n * rs));
  std::vector<double> d(n);
  if (rs == 8) {
    memcpy(d.data(), bytes.data(), bytes.size());
  } else {
    const float* p = reinterpret_cast<const float*>(bytes.data());
    for (size_t i = 0; i < n; ++i) d[i] = (double)p[i];
  }
  return clg_field_import(f, rhs, d.data(), 0);
}

}  // extern "C"
