// dslash.cu -- launchers for the checkerboard hopping kernels and the
// low-precision link copies (12-real reconstruction) they read.
#include <algorithm>
#include <string>

#include "dslash.cuh"
#include "internal.h"

namespace clg {

namespace {

// the launch is idempotent (safe to repeat while timing block sizes) unless
// the output aliases the xpay source
bool idempotent(const HopArgs& a) { return a.x == nullptr || a.x != a.out; }

// FP64 / FP32 Wilson hop over a tile of 32 sites for all right-hand sides
// (wilson_hop_tileN_kernel); config = block size | (16 + v) << 16, v & 1 =
// the register cap (128 for FP64, 80 for FP32), v & 2 = the blocked tile order
template <int P, int RECON>
cudaError_t launch_wilson_tileN(clg_context_s* ctx, const HopArgs& a0, bool dagger, int cfg) {
  constexpr int CAP = P == P64 ? 2 : 3;
  const int bs = cfg & 0xffff;
  HopArgs a = a0;
  a.tile_rows = ((cfg >> 16) & 2) ? tile_rows(a.g, a.nrhs, TILE16, spinor_bytes<P>()) : 0;
  dim3 grid((unsigned)((a.g.Vh + TILE16 - 1) / TILE16));
  if ((cfg >> 16) & 1)
    return dagger ? launch_pdl(ctx, wilson_hop_tileN_kernel<P, RECON, true, CAP>, grid, dim3(bs), 0, a)
                  : launch_pdl(ctx, wilson_hop_tileN_kernel<P, RECON, false, CAP>, grid, dim3(bs), 0, a);
  return dagger ? launch_pdl(ctx, wilson_hop_tileN_kernel<P, RECON, true, 1>, grid, dim3(bs), 0, a)
                : launch_pdl(ctx, wilson_hop_tileN_kernel<P, RECON, false, 1>, grid, dim3(bs), 0, a);
}

std::vector<int> tile_warps(int nrhs);

template <int P, int RECON>
cudaError_t launch_wilson(clg_context_s* ctx, const HopArgs& a, bool dagger, int nrhs, const std::string& key) {
  // config = block size | (variant << 16): 0 plain, 1 capped at 80 registers,
  // 2 capped at 72 registers (64-thread blocks only), 3 capped at 128 (FP64:
  // the uncapped FP64 kernel takes 254 registers, 8 warps per SM)
  auto go = [&](int cfg) {
    const int bs = cfg & 0xffff;
    const int variant = cfg >> 16;
    if constexpr (P != P16) {
      if (variant >= 16) return launch_wilson_tileN<P, RECON>(ctx, a, dagger, cfg);
    }
    dim3 grid((unsigned)(((a.g.Vh + bs - 1) / bs) * nrhs));
    if constexpr (P == P64) {
      if (variant == 3)
        return dagger ? launch_pdl(ctx, wilson_hop_kernel<P, RECON, true, 256, 2>, grid, dim3(bs), 0, a)
                      : launch_pdl(ctx, wilson_hop_kernel<P, RECON, false, 256, 2>, grid, dim3(bs), 0, a);
    }
    if constexpr (P != P64) {
      if (variant == 1)
        return dagger ? launch_pdl(ctx, wilson_hop_kernel<P, RECON, true, 256, 3>, grid, dim3(bs), 0, a)
                      : launch_pdl(ctx, wilson_hop_kernel<P, RECON, false, 256, 3>, grid, dim3(bs), 0, a);
      if (variant == 2 && bs == 64)
        return dagger ? launch_pdl(ctx, wilson_hop_kernel<P, RECON, true, 64, 14>, grid, dim3(bs), 0, a)
                      : launch_pdl(ctx, wilson_hop_kernel<P, RECON, false, 64, 14>, grid, dim3(bs), 0, a);
    }
    return dagger ? launch_pdl(ctx, wilson_hop_kernel<P, RECON, true>, grid, dim3(bs), 0, a)
                  : launch_pdl(ctx, wilson_hop_kernel<P, RECON, false>, grid, dim3(bs), 0, a);
  };
  if (ctx->hop_config >= 0) {
    ctx->tuned[key] = ctx->hop_config;  // the fused epilogue launches follow the pinned form
    return go(ctx->hop_config);
  }
  // __launch_bounds__(256, ...) caps the block at 256 threads
  std::vector<int> cand = {64, 128, 256};
  if (P != P64)
    for (int bs : {64, 128, 256}) cand.push_back(bs | (1 << 16));
  if (P != P64) cand.push_back(64 | (2 << 16));
  if (P == P64)
    for (int bs : {64, 128, 256}) cand.push_back(bs | (3 << 16));
  // several right-hand sides: the tile form (links staged once per tile)
  if (P != P16 && nrhs >= 2)
    for (int w : tile_warps(nrhs))
      for (int v = 0; v < (tile_rows(a.g, nrhs, TILE16, spinor_bytes<P>()) ? 4 : 2); ++v)
        cand.push_back((32 * w) | ((16 + v) << 16));
  return go(tune_block(ctx, key, idempotent(a), go, cand));
}

// FP16 Wilson hop with the right-hand sides in pairs (wilson_hop_pair_kernel);
// config = block size | (variant << 16): 0 caps at 128 registers, 1 at 96
cudaError_t launch_wilson_pair(clg_context_s* ctx, const HopArgs& a, bool dagger, const std::string& key) {
  const unsigned npairs = (unsigned)(a.nrhs + 1) / 2u;
  auto go = [&](int cfg) {
    const int bs = cfg & 0xffff;
    const int variant = cfg >> 16;
    dim3 grid((unsigned)(((a.g.Vh + bs - 1) / bs) * npairs));
    if (variant == 1)
      return dagger ? launch_pdl(ctx, wilson_hop_pair_kernel<true, 256, 2>, grid, dim3(bs), 0, a)
                    : launch_pdl(ctx, wilson_hop_pair_kernel<false, 256, 2>, grid, dim3(bs), 0, a);
    return dagger ? launch_pdl(ctx, wilson_hop_pair_kernel<true, 256, 1>, grid, dim3(bs), 0, a)
                  : launch_pdl(ctx, wilson_hop_pair_kernel<false, 256, 1>, grid, dim3(bs), 0, a);
  };
  if (ctx->hop_pair_config >= 0) {
    ctx->tuned[key + "_pair"] = ctx->hop_pair_config;  // the fused epilogue launches follow it
    return go(ctx->hop_pair_config);
  }
  std::vector<int> cand;
  for (int bs : {64, 128, 256}) {
    cand.push_back(bs);
    cand.push_back(bs | (1 << 16));
  }
  return go(tune_block(ctx, key + "_pair", idempotent(a), go, cand));
}

// a batch of lattices: one right-hand side per lattice segment, untuned
template <int P, int RECON>
cudaError_t launch_wilson_batch(clg_context_s* ctx, const HopArgs& a, bool dagger) {
  if (a.btile) {
    // the tile form, one block per tile of 32 sites of one lattice (4 warps;
    // FP16 / FP32 capped at 80 registers, FP64 at 128)
    constexpr int CAP = P == P64 ? 2 : 3;
    const dim3 grid((unsigned)a.btiles), block(128);
    if constexpr (P == P16)
      return dagger ? launch_pdl(ctx, wilson_hop_tile16_kernel<true, CAP, true>, grid, block, 0, a)
                    : launch_pdl(ctx, wilson_hop_tile16_kernel<false, CAP, true>, grid, block, 0, a);
    else
      return dagger ? launch_pdl(ctx, wilson_hop_tileN_kernel<P, RECON, true, CAP, true>, grid, block, 0, a)
                    : launch_pdl(ctx, wilson_hop_tileN_kernel<P, RECON, false, CAP, true>, grid, block, 0, a);
  }
  const int bs = P == P64 ? 64 : 128;
  dim3 grid((unsigned)(((a.g.Vh + bs - 1) / bs) * a.nrhs));
  return dagger ? launch_pdl(ctx, wilson_hop_batch_kernel<P, RECON, true>, grid, dim3(bs), 0, a)
                : launch_pdl(ctx, wilson_hop_batch_kernel<P, RECON, false>, grid, dim3(bs), 0, a);
}

}  // namespace

// The y-rows per chunk of the tile hops' blocked order (0: site order): the
// largest divisor of L_y whose three x-slabs of input spinors (sbytes per
// site and rhs: 52 FP16 with its norm, 96 FP32, 192 FP64), over all
// right-hand sides, take at most 24 MB of L2; 0 when the z-t planes are not a
// whole number of tiles or no chunk smaller than L_y qualifies.
int tile_rows(const Geom& g, int nrhs, int ts, int sbytes) {
  const int64_t plane = (int64_t)g.L[2] * g.L[3];
  if (plane % (2 * ts)) return 0;
  const int64_t slab_row = plane / 2 * nrhs * sbytes;  // spinor bytes of one y-row, all rhs
  int best = 0;
  for (int by = 1; by < g.L[1]; ++by)
    if (g.L[1] % by == 0 && 3 * by * slab_row <= (int64_t)24 << 20) best = by;
  return best;
}

namespace {

// FP16 Wilson hop with the colour products on the tensor cores
// (wilson_hop_mma16_kernel, 256 threads, a tile of MMA_TS sites); config
// variant 24 + v, v & 1 = at most 128 registers (two blocks per SM), v & 2 =
// the blocked tile order
cudaError_t launch_wilson_mma(clg_context_s* ctx, const HopArgs& a0, bool dagger, int cfg) {
  HopArgs a = a0;
  const int v = (cfg >> 16) - 24;
  a.tile_rows = (v & 2) ? tile_rows(a.g, a.nrhs, MMA_TS) : 0;
  dim3 grid((unsigned)((a.g.Vh + MMA_TS - 1) / MMA_TS));
  const size_t smem = sizeof(Mma16Smem);
  auto go = [&](void (*kernel)(HopArgs)) {
    if (const cudaError_t e = opt_in_smem((const void*)kernel, smem)) return e;
    return launch_pdl(ctx, kernel, grid, dim3(256), smem, a);
  };
  if (v & 1) return dagger ? go(wilson_hop_mma16_kernel<true, 2>) : go(wilson_hop_mma16_kernel<false, 2>);
  return dagger ? go(wilson_hop_mma16_kernel<true, 1>) : go(wilson_hop_mma16_kernel<false, 1>);
}

// FP16 Wilson hop over a tile of 32 sites for all right-hand sides
// (wilson_hop_tile16_kernel); config = block size | (16 + v) << 16 with v & 1
// = the 80-register cap and v & 2 = the blocked tile order (tile_rows);
// variants from 24 on are the tensor-core form (launch_wilson_mma)
cudaError_t launch_wilson_tile(clg_context_s* ctx, const HopArgs& a0, bool dagger, int cfg) {
  if ((cfg >> 16) >= 24) return launch_wilson_mma(ctx, a0, dagger, cfg);
  const int bs = cfg & 0xffff;
  HopArgs a = a0;
  a.tile_rows = ((cfg >> 16) & 2) ? tile_rows(a.g, a.nrhs) : 0;
  dim3 grid((unsigned)((a.g.Vh + TILE16 - 1) / TILE16));
  const int v = cfg >> 16;
  if (v >= 20) {  // blocks of at most 128 threads: 72 (v & 1 == 0) or 64 registers
    if (bs > 128) return cudaErrorInvalidConfiguration;
    if (v & 1)
      return dagger ? launch_pdl(ctx, wilson_hop_tile16_kernel<true, 8, false, 128>, grid, dim3(bs), 0, a)
                    : launch_pdl(ctx, wilson_hop_tile16_kernel<false, 8, false, 128>, grid, dim3(bs), 0, a);
    return dagger ? launch_pdl(ctx, wilson_hop_tile16_kernel<true, 7, false, 128>, grid, dim3(bs), 0, a)
                  : launch_pdl(ctx, wilson_hop_tile16_kernel<false, 7, false, 128>, grid, dim3(bs), 0, a);
  }
  if (v & 1)
    return dagger ? launch_pdl(ctx, wilson_hop_tile16_kernel<true, 3>, grid, dim3(bs), 0, a)
                  : launch_pdl(ctx, wilson_hop_tile16_kernel<false, 3>, grid, dim3(bs), 0, a);
  return dagger ? launch_pdl(ctx, wilson_hop_tile16_kernel<true, 2>, grid, dim3(bs), 0, a)
                : launch_pdl(ctx, wilson_hop_tile16_kernel<false, 2>, grid, dim3(bs), 0, a);
}

// warps per tile block worth timing for nrhs right-hand sides: 4 and 8, and
// the divisors of nrhs between 3 and 8 (no warp idles at the end)
std::vector<int> tile_warps(int nrhs) {
  std::vector<int> w = {4, 8};
  for (int d = 3; d <= 8; ++d)
    if (nrhs % d == 0 && d != 4 && d != 8) w.push_back(d);
  if (nrhs < 4) w = {nrhs};
  return w;
}

// The autotuner's choice of the FP16 Wilson hop's form for two or more
// right-hand sides: one rhs per thread (config variants 0..2), two per thread
// (variant 8 + the pair variant) or a tile of sites for all rhs (variants 16,
// 17).  The winner is recorded under the keys the fused epilogue launches
// look up (key, key_pair, key_tile).
cudaError_t launch_wilson_auto(clg_context_s* ctx, const HopArgs& a, bool dagger, int nrhs, const std::string& key) {
  auto it = ctx->tuned.find(key + "_auto");
  int cfg;
  if (it != ctx->tuned.end()) {
    cfg = it->second;
  } else {
    auto go = [&](int c) -> cudaError_t {
      const int v = c >> 16;
      if (v >= 16) return launch_wilson_tile(ctx, a, dagger, c);
      if (v >= 8) {
        ctx->tuned[key + "_pair"] = (c & 0xffff) | ((v - 8) << 16);
        return launch_wilson_pair(ctx, a, dagger, key);
      }
      ctx->tuned[key] = c;
      return launch_wilson<P16, 12>(ctx, a, dagger, nrhs, key);
    };
    std::vector<int> cand;
    for (int bs : {64, 128, 256}) {
      cand.push_back(bs);
      cand.push_back(bs | (1 << 16));
      cand.push_back(bs | (8 << 16));
      cand.push_back(bs | (9 << 16));
    }
    cand.push_back(64 | (2 << 16));
    for (int w : tile_warps(nrhs)) {
      const int nv = tile_rows(a.g, nrhs) ? 4 : 2;
      for (int v = 0; v < nv; ++v) cand.push_back((32 * w) | ((16 + v) << 16));
      if (w <= 4)  // the 72- and 64-register caps (more resident blocks of at most 4 warps)
        for (int v = 0; v < nv; ++v) cand.push_back((32 * w) | ((20 + v) << 16));
    }
    if (ctx->hop_mma)
      for (int v = 0; v < (tile_rows(a.g, nrhs, MMA_TS) ? 4 : 2); ++v) cand.push_back(256 | ((24 + v) << 16));
    // untuned (inside a capture, or the output aliases the xpay source): the
    // one-rhs kernel, and nothing is cached
    if (!ctx->tuning_enabled || !idempotent(a) || stream_capturing(ctx->stream))
      return launch_wilson<P16, 12>(ctx, a, dagger, nrhs, key);
    std::map<int, float> times;
    cfg = tune_block(ctx, key + "_auto", true, go, cand, 128, &times);
    // a tile form in site order that the blocked order matches within 3 %:
    // take the blocked one, whose fewer DRAM bytes help the fused epilogue
    // hops (more memory traffic than the plain hop timed here) that follow
    // this choice
    if ((cfg >> 16) == 16 || (cfg >> 16) == 17 || (cfg >> 16) == 20 || (cfg >> 16) == 21) {
      const int blocked = cfg + (2 << 16);
      auto a = times.find(cfg), b = times.find(blocked);
      if (a != times.end() && b != times.end() && b->second <= 1.03f * a->second) {
        cfg = blocked;
        ctx->tuned[key + "_auto"] = cfg;
      }
    }
    ctx->tuned.erase(key);
    ctx->tuned.erase(key + "_pair");
    ctx->tuned.erase(key + "_tile");
    const int v = cfg >> 16;
    if (v >= 16) ctx->tuned[key + "_tile"] = cfg;
    else if (v >= 8) ctx->tuned[key + "_pair"] = (cfg & 0xffff) | ((v - 8) << 16);
    else ctx->tuned[key] = cfg;
  }
  if ((cfg >> 16) >= 16) return launch_wilson_tile(ctx, a, dagger, cfg);
  if ((cfg >> 16) >= 8) return launch_wilson_pair(ctx, a, dagger, key);
  return launch_wilson<P16, 12>(ctx, a, dagger, nrhs, key);
}

template <int P, int RECON>
cudaError_t launch_staggered(clg_context_s* ctx, const HopArgs& a, int nrhs, const std::string& key) {
  // config = block size | (variant << 16): 0 uncapped, 1 capped at 80 registers
  // variants 16..19 (FP64 / FP32, several rhs): the tile form, v & 1 the
  // register cap (128 FP64, 80 FP32), v & 2 the blocked tile order
  auto go = [&](int cfg) {
    const int bs = cfg & 0xffff;
    const int v = cfg >> 16;
    if constexpr (P != P16) {
      if (v >= 16) {
        constexpr int CAP = P == P64 ? 2 : 3;
        HopArgs at = a;
        at.tile_rows = (v & 2) ? tile_rows(a.g, a.nrhs, TILE16, P == P64 ? 48 : 24) : 0;
        dim3 tg((unsigned)((a.g.Vh + TILE16 - 1) / TILE16));
        if (v & 1) return launch_pdl(ctx, staggered_tile_kernel<P, RECON, CAP>, tg, dim3(bs), 0, at);
        return launch_pdl(ctx, staggered_tile_kernel<P, RECON, 1>, tg, dim3(bs), 0, at);
      }
    }
    dim3 grid((unsigned)(((a.g.Vh + bs - 1) / bs) * nrhs));
    if (v == 1) return launch_pdl(ctx, staggered_hop_kernel_capped<P, RECON>, grid, dim3(bs), 0, a);
    return launch_pdl(ctx, staggered_hop_kernel<P, RECON>, grid, dim3(bs), 0, a);
  };
  if (ctx->hop_config >= 0 && (P != P16 || (ctx->hop_config >> 16) < 16)) return go(ctx->hop_config);
  std::vector<int> cand = {64, 128, 256};
  if (P == P64)
    for (int bs : {64, 128, 256}) cand.push_back(bs | (1 << 16));
  if (P != P16 && nrhs >= 2)
    for (int w : tile_warps(nrhs))
      for (int v = 0; v < (tile_rows(a.g, nrhs, TILE16, P == P64 ? 48 : 24) ? 4 : 2); ++v)
        cand.push_back((32 * w) | ((16 + v) << 16));
  return go(tune_block(ctx, key, idempotent(a), go, cand));
}

// FP64 [mu][9][h] double2 -> FP32 12-real [mu][3][h] float4 or 18-real [mu][9][h] float2
__global__ void links_to_fp32(const double2* __restrict__ u64, void* out, int64_t Vh, int recon) {
  const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (h >= Vh) return;
  const double2* src = u64 + (int64_t)mu * 9 * Vh + h;
  if (recon == 12) {
    float4* dst = reinterpret_cast<float4*>(out) + (int64_t)mu * 3 * Vh + h;
    for (int k = 0; k < 3; ++k) {
      const double2 a = src[(2 * k) * Vh], b = src[(2 * k + 1) * Vh];
      dst[k * Vh] = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
    }
  } else {
    float2* dst = reinterpret_cast<float2*>(out) + (int64_t)mu * 9 * Vh + h;
    for (int k = 0; k < 9; ++k) {
      const double2 a = src[k * Vh];
      dst[k * Vh] = make_float2((float)a.x, (float)a.y);
    }
  }
}

// FP64 -> FP16 12-real: [mu][h] uint4 (u0..u3) then [mu][h] uint2 (u4, u5)
__global__ void links_to_fp16(const double2* __restrict__ u64, void* out, int64_t Vh) {
  const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (h >= Vh) return;
  const double2* src = u64 + (int64_t)mu * 9 * Vh + h;
  uint32_t w[6];
  for (int k = 0; k < 6; ++k) {
    const double2 a = src[k * Vh];
    __half2 hv = __floats2half2_rn((float)a.x, (float)a.y);
    w[k] = *reinterpret_cast<uint32_t*>(&hv);
  }
  uint4* d4 = reinterpret_cast<uint4*>(out);
  uint2* d2 = reinterpret_cast<uint2*>(d4 + 4 * Vh);
  d4[(int64_t)mu * Vh + h] = make_uint4(w[0], w[1], w[2], w[3]);
  d2[(int64_t)mu * Vh + h] = make_uint2(w[4], w[5]);
}

}  // namespace

clg_status gauge_prepare(clg_gauge_s* U, int prec) {
  if (prec == CLG_PREC_DOUBLE || U->seg) return CLG_SUCCESS;  // a batch's lattices are prepared when it is built
  clg_context_s* ctx = U->lat->ctx;
  const int64_t Vh = U->lat->g.Vh;
  if (U->dirty_lowp) {
    // both parities of a low-precision copy live in one allocation ([0] first)
    dfree(U->u32[0]);
    dfree(U->u16[0]);
    U->u32[0] = U->u32[1] = U->u16[0] = U->u16[1] = nullptr;
    U->dirty_lowp = false;
  }
  if (prec == CLG_PREC_HALF && !U->su3)
    return ctx->fail(CLG_ERR_UNSUPPORTED, "half-precision links need SU(3) links (12-real reconstruction)");
  dim3 grid((unsigned)((Vh + 255) / 256), 4);
  if (prec == CLG_PREC_SINGLE && !U->u32[0]) {
    U->recon32 = U->su3 ? 12 : 18;
    const size_t bytes = (size_t)4 * Vh * U->recon32 * 4;  // one parity
    clg_status st = dalloc(ctx, &U->u32[0], 2 * bytes);
    if (st) return st;
    U->u32[1] = static_cast<char*>(U->u32[0]) + bytes;
    for (int p = 0; p < 2; ++p) {
      links_to_fp32<<<grid, 256, 0, ctx->stream>>>((const double2*)U->u64[p], U->u32[p], Vh, U->recon32);
      ctx->kernels++;
      CLG_CUDA_OK(cudaGetLastError());
    }
  }
  if (prec == CLG_PREC_HALF && !U->u16[0]) {
    const size_t bytes = (size_t)4 * Vh * 24;  // one parity
    clg_status st = dalloc(ctx, &U->u16[0], 2 * bytes);
    if (st) return st;
    U->u16[1] = static_cast<char*>(U->u16[0]) + bytes;
    for (int p = 0; p < 2; ++p) {
      links_to_fp16<<<grid, 256, 0, ctx->stream>>>((const double2*)U->u64[p], U->u16[p], Vh);
      ctx->kernels++;
      CLG_CUDA_OK(cudaGetLastError());
    }
  }
  return CLG_SUCCESS;
}

L2LinkWindow::L2LinkWindow(clg_context_s* c, const clg_gauge_s* U, int prec) : ctx(c) {
  if (!ctx->l2_window || ctx->max_window == 0 || ctx->max_persist == 0) return;
  const void* base = nullptr;
  size_t bytes = 0;
  gauge_link_range(U, prec, &base, &bytes);
  // only a link copy that leaves most of the L2 to the vectors: the 100 MB
  // FP32 copy of a 32^3x16 lattice made the FP32 solve 13 % slower, the 50 MB
  // FP16 copy made the FP16 solve 5 % faster
  if (!base || bytes > ctx->l2_bytes / 2 || stream_capturing(ctx->stream)) return;
  const size_t win = std::min(bytes, ctx->max_window);
  const size_t carve = std::min(win, ctx->max_persist);
  if (ctx->persist_set < carve) {
    if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, carve) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    ctx->persist_set = carve;
  }
  cudaStreamAttrValue v = {};
  v.accessPolicyWindow.base_ptr = const_cast<void*>(base);
  v.accessPolicyWindow.num_bytes = win;
  v.accessPolicyWindow.hitRatio = (float)std::min(1.0, (double)ctx->persist_set / (double)win);
  v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
  v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  set = cudaStreamSetAttribute(ctx->stream, cudaStreamAttributeAccessPolicyWindow, &v) == cudaSuccess;
  cudaGetLastError();
}

L2LinkWindow::~L2LinkWindow() {
  if (!set) return;
  cudaStreamAttrValue v = {};
  v.accessPolicyWindow.num_bytes = 0;
  cudaStreamSetAttribute(ctx->stream, cudaStreamAttributeAccessPolicyWindow, &v);
  cudaGetLastError();
}

// The link copy the hops of precision `prec` read (both parities, one range).
void gauge_link_range(const clg_gauge_s* U, int prec, const void** base, size_t* bytes) {
  const int64_t Vh = U->lat->g.Vh;
  if (prec == CLG_PREC_SINGLE && U->u32[0]) {
    *base = U->u32[0];
    *bytes = (size_t)2 * 4 * Vh * U->recon32 * 4;
  } else if (prec == CLG_PREC_HALF && U->u16[0]) {
    *base = U->u16[0];
    *bytes = (size_t)2 * 4 * Vh * 24;
  } else {
    *base = nullptr;
    *bytes = 0;
  }
}

clg_status make_hop_args(clg_context_s* ctx, const clg_gauge_s* U, const HopSpec& s, HopArgs& a) {
  const int p = s.out_parity;
  if (!s.in.has_parity(1 - p) || !s.out.has_parity(p) || (s.x && !s.x->has_parity(p)))
    return ctx->fail(CLG_ERR_BAD_ARG, "hop: field does not hold the required checkerboard");
  if (s.in.prec != s.prec || s.out.prec != s.prec || (s.x && s.x->prec != s.prec))
    return ctx->fail(CLG_ERR_BAD_ARG, "hop: precision mismatch");
  a.g = U->lat->g;
  a.out_parity = p;
  a.in = s.in.base(0, 1 - p);
  a.in_norm = s.in.nbase(0, 1 - p);
  a.out = s.out.base(0, p);
  a.out_norm = s.out.nbase(0, p);
  a.x = s.x ? s.x->base(0, p) : nullptr;
  a.x_norm = s.x ? s.x->nbase(0, p) : nullptr;
  a.in_stride = s.in.rstride;
  a.out_stride = s.out.rstride;
  a.x_stride = s.x ? s.x->rstride : 0;
  a.in_nstride = s.in.nrstride;
  a.out_nstride = s.out.nrstride;
  a.x_nstride = s.x ? s.x->nrstride : 0;
  a.a = s.a;
  a.xa = s.xa;
  a.scale_dev = s.scale_dev;
  a.scale_stride = s.scale_stride;
  a.skip_dev = s.skip_dev;
  a.skip_stride = s.skip_stride;
  a.nrhs = s.nrhs > 0 ? s.nrhs : 1;
  a.seg = U->seg;
  a.seg_vh = U->seg_vh;
  a.tile_rows = 0;
  a.btile = U->btile;
  a.nbtile = U->nbtile;
  a.btiles = U->btiles;
  if (U->seg) {
    if (s.kind != CLG_FERMION_WILSON) return ctx->fail(CLG_ERR_UNSUPPORTED, "a batch of lattices takes Wilson fermions");
    a.U_here = a.U_there = nullptr;
    return CLG_SUCCESS;
  }
  if (s.prec == CLG_PREC_DOUBLE) {
    a.U_here = U->u64[p];
    a.U_there = U->u64[1 - p];
  } else if (s.prec == CLG_PREC_SINGLE) {
    a.U_here = U->u32[p];
    a.U_there = U->u32[1 - p];
    if (!a.U_here || !a.U_there) return ctx->fail(CLG_ERR_BAD_ARG, "hop: FP32 links not prepared");
  } else {
    a.U_here = U->u16[p];
    a.U_there = U->u16[1 - p];
    if (!a.U_here || !a.U_there) return ctx->fail(CLG_ERR_BAD_ARG, "hop: FP16 links not prepared");
  }
  return CLG_SUCCESS;
}

static std::string hop_key(const clg_gauge_s* U, const HopSpec& s) {
  const bool wilson = s.kind == CLG_FERMION_WILSON;
  return std::string(wilson ? "wilson" : "ks") + "_p" + std::to_string(s.prec) + "_d" + std::to_string((int)s.dagger) +
         "_V" + std::to_string((long long)U->lat->g.Vh) + "_n" + std::to_string(s.nrhs) + "_r" +
         std::to_string(s.prec == CLG_PREC_SINGLE ? U->recon32 : 0);
}

int tuned_hop_pair_config(clg_context_s* ctx, const clg_gauge_s* U, const HopSpec& s, int fallback) {
  auto it = ctx->tuned.find(hop_key(U, s) + "_pair");
  return it == ctx->tuned.end() ? fallback : it->second;
}

int tuned_hop_tile_config(clg_context_s* ctx, const clg_gauge_s* U, const HopSpec& s, int fallback) {
  if (ctx->hop_pair_mode == 3) return ctx->hop_tile_config;
  auto it = ctx->tuned.find(hop_key(U, s) + "_tile");
  return it == ctx->tuned.end() ? fallback : it->second;
}

int tuned_hop_config(clg_context_s* ctx, const clg_gauge_s* U, const HopSpec& s, int fallback) {
  auto it = ctx->tuned.find(hop_key(U, s));
  return it == ctx->tuned.end() ? fallback : it->second;
}

int tuned_hop_block(clg_context_s* ctx, const clg_gauge_s* U, const HopSpec& s, int fallback) {
  auto it = ctx->tuned.find(hop_key(U, s));
  if (it == ctx->tuned.end()) return fallback;
  return it->second & 0xffff;
}

clg_status hop(clg_context_s* ctx, const clg_gauge_s* U, const HopSpec& s) {
  HopArgs a;
  if (clg_status st = make_hop_args(ctx, U, s, a)) return st;
  const bool wilson = s.kind == CLG_FERMION_WILSON;
  const std::string key = hop_key(U, s);
  cudaError_t e = cudaSuccess;
  if (a.seg) {
    e = s.prec == CLG_PREC_DOUBLE   ? launch_wilson_batch<P64, 18>(ctx, a, s.dagger)
        : s.prec == CLG_PREC_SINGLE ? launch_wilson_batch<P32, 12>(ctx, a, s.dagger)
                                    : launch_wilson_batch<P16, 12>(ctx, a, s.dagger);
  } else if (s.prec == CLG_PREC_DOUBLE) {
    e = wilson ? launch_wilson<P64, 18>(ctx, a, s.dagger, s.nrhs, key) : launch_staggered<P64, 18>(ctx, a, s.nrhs, key);
  } else if (s.prec == CLG_PREC_SINGLE) {
    if (U->recon32 == 12)
      e = wilson ? launch_wilson<P32, 12>(ctx, a, s.dagger, s.nrhs, key) : launch_staggered<P32, 12>(ctx, a, s.nrhs, key);
    else
      e = wilson ? launch_wilson<P32, 18>(ctx, a, s.dagger, s.nrhs, key) : launch_staggered<P32, 18>(ctx, a, s.nrhs, key);
  } else if (wilson && s.nrhs >= 2 && ctx->hop_pair_mode == 3) {
    e = launch_wilson_tile(ctx, a, s.dagger, ctx->hop_tile_config);
  } else if (wilson && s.nrhs >= 2 && ctx->hop_pair_mode == 1) {
    e = launch_wilson_pair(ctx, a, s.dagger, key);
  } else if (wilson && s.nrhs >= 2 && ctx->hop_pair_mode == 2 && ctx->hop_config < 0) {
    e = launch_wilson_auto(ctx, a, s.dagger, s.nrhs, key);
  } else {
    e = wilson ? launch_wilson<P16, 12>(ctx, a, s.dagger, s.nrhs, key) : launch_staggered<P16, 12>(ctx, a, s.nrhs, key);
  }
  if (e != cudaSuccess) return ctx->fail(cuda_status(e), std::string("hop launch: ") + cudaGetErrorString(e));
  return CLG_SUCCESS;
}

}  // namespace clg
