// batch.cu -- clg_solve_lattices: right-hand sides on several lattices of
// uneven volume (each with its own gauge field) solved together.
//
// The reference holds one lattice per process (extents in __constant__ memory,
// Core/CudaHelper.cu:14-25; appQuitCLG / appInitialCLG to change them,
// Core/CLGLibManager.cpp:1131-1162), so a set of lattices is a sequence of
// processes there.  Here the right-hand sides of all lattices become the
// right-hand sides of one solve on a padded "batch lattice": every field of the
// solve holds, per right-hand side, its lattice's checkerboards in the
// structure-of-arrays layout with the chunk stride of the largest checkerboard
// of the set; the sites past a lattice's own checkerboard are padding that
// stays zero.  The hop kernels take the lattice of each right-hand side from a
// device table (HopSeg: geometry and link arrays per right-hand side; the tile
// form's blocks are the tiles of 32 sites of each lattice in turn, BatchTile,
// so no block works on padding and each lattice's links are staged once per
// tile for all its right-hand sides), and the
// vector kernels skip the padding (site_reduce_batch_kernel with the per-rhs
// checkerboard sizes; the padding is zero either way).  So one iteration of the
// inner Krylov method is the same fixed number of launches whatever the number
// of lattices, and it is captured and replayed as a CUDA graph like any other
// solve.
#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "dslash.cuh"
#include "internal.h"

namespace clg {
namespace {

struct BatchWork : SolveCacheBase {
  std::string key;
  clg_context_s* ctx = nullptr;
  clg_lattice_s vlat;        // the padded batch lattice
  clg_gauge_s vgauge;        // its "gauge field": the per-rhs HopSeg table
  HopSeg* seg_dev = nullptr;
  int64_t* vh_dev = nullptr;  // per-rhs checkerboard sizes
  BatchTile* tile_dev = nullptr;  // per lattice: its tiles of 32 sites and right-hand sides
  void* b_data = nullptr;
  void* x_data = nullptr;
  FieldRef B, X;             // FP64 full fields, padded
  std::unique_ptr<SolveCacheBase> solve_cache;
  ~BatchWork() override {
    if (ctx) cudaStreamSynchronize(ctx->stream);
    solve_cache.reset();
    dfree(seg_dev);
    dfree(vh_dev);
    dfree(tile_dev);
    dfree(b_data);
    dfree(x_data);
  }
};

FieldRef padded_full(char* data, int nc, int nrhs, int64_t Vh) {
  FieldRef f;
  f.data = data;
  f.norm = nullptr;
  f.blk = Vh * (int64_t)nc * 16;
  f.rstride = 2 * f.blk;
  f.nrstride = 0;
  f.nparity = 2;
  f.first_parity = 0;
  f.prec = CLG_PREC_DOUBLE;
  f.nc = nc;
  f.nrhs = nrhs;
  f.Vh = Vh;
  return f;
}

}  // namespace
}  // namespace clg

using namespace clg;

extern "C" clg_status clg_solve_lattices(clg_solver S, int n, clg_field* x, clg_field* b, clg_gauge* U, int op,
                                         clg_solve_info* info) {
  if (!S || n < 1 || !x || !b || !U || !info) return CLG_ERR_BAD_ARG;
  clg_context_s* ctx = S->ctx;
  if (op != CLG_OP_D && op != CLG_OP_DDAG)
    return ctx->fail(CLG_ERR_UNSUPPORTED, "solve_lattices: D or D^+ on full fields");
  if (S->p.kind != CLG_SOLVER_GMRES && S->p.kind != CLG_SOLVER_BICGSTAB && S->p.kind != CLG_SOLVER_CG)
    return ctx->fail(CLG_ERR_BAD_ARG, "solve_lattices: GMRES, BiCGStab or CG");
  int total = 0;
  int64_t vh_max = 0;
  int largest = 0;
  for (int i = 0; i < n; ++i) {
    if (!x[i] || !b[i] || !U[i]) return CLG_ERR_BAD_ARG;
    if (b[i]->lat->ctx != ctx || U[i]->lat != b[i]->lat || x[i]->lat != b[i]->lat)
      return ctx->fail(CLG_ERR_BAD_ARG, "solve_lattices: x, b and U of a lattice must share it (and the context)");
    if (b[i]->kind != CLG_FERMION_WILSON || b[i]->subset != CLG_SUBSET_FULL || b[i]->prec != CLG_PREC_DOUBLE ||
        x[i]->kind != b[i]->kind || x[i]->subset != b[i]->subset || x[i]->prec != b[i]->prec ||
        x[i]->nrhs != b[i]->nrhs)
      return ctx->fail(CLG_ERR_BAD_ARG, "solve_lattices: FP64 full Wilson fields, x shaped as b");
    if (b[i]->param != b[0]->param) return ctx->fail(CLG_ERR_BAD_ARG, "solve_lattices: one hopping parameter");
    if (S->p.inner_precision != CLG_PREC_DOUBLE && !U[i]->su3)
      return ctx->fail(CLG_ERR_UNSUPPORTED, "solve_lattices: low-precision inner solves need SU(3) links");
    total += b[i]->nrhs;
    if (b[i]->lat->g.Vh > vh_max) {
      vh_max = b[i]->lat->g.Vh;
      largest = i;
    }
  }
  for (int i = 0; i < n; ++i) {
    if (clg_status st = settle(b[i])) return st;
    if (clg_status st = settle(x[i])) return st;
    if (clg_status st = gauge_prepare(U[i], S->p.inner_precision)) return st;
  }
  const int nc = 12;
  // the batch (table, padded fields, the solve's workspace) is kept while the
  // set of lattices, gauge arrays and right-hand-side counts stays the same
  std::string key = std::to_string(n) + "/" + std::to_string(op);
  for (int i = 0; i < n; ++i)
    key += "/" + std::to_string((uintptr_t)b[i]->lat) + ":" + std::to_string(b[i]->nrhs) + ":" +
           std::to_string((uintptr_t)U[i]->u64[0]) + ":" + std::to_string((uintptr_t)U[i]->u32[0]) + ":" +
           std::to_string((uintptr_t)U[i]->u16[0]);
  auto* W = dynamic_cast<BatchWork*>(S->cache_batch.get());
  if (!W || W->key != key) {
    cudaStreamSynchronize(ctx->stream);
    S->cache_batch.reset();
    auto nw = std::make_unique<BatchWork>();
    nw->ctx = ctx;
    nw->vlat.ctx = ctx;
    nw->vlat.g = b[largest]->lat->g;  // geometry unused by the batch kernels; Vh = the padded chunk stride
    nw->vgauge.lat = &nw->vlat;
    nw->vgauge.su3 = true;
    nw->vgauge.dirty_lowp = false;
    std::vector<HopSeg> segs;
    std::vector<int64_t> vhs;
    std::vector<BatchTile> tiles;
    int64_t ntiles = 0;
    for (int i = 0; i < n; ++i) {
      BatchTile bt;
      bt.tile0 = ntiles;
      bt.rhs0 = (int)segs.size();
      bt.nrhs = b[i]->nrhs;
      bt.seg = (int)segs.size();
      tiles.push_back(bt);
      ntiles += (b[i]->lat->g.Vh + TILE16 - 1) / TILE16;
      for (int r = 0; r < b[i]->nrhs; ++r) {
        HopSeg sg;
        sg.g = b[i]->lat->g;
        for (int p = 0; p < 2; ++p) {
          sg.u[0][p] = U[i]->u64[p];
          sg.u[1][p] = U[i]->u32[p];
          sg.u[2][p] = U[i]->u16[p];
        }
        segs.push_back(sg);
        vhs.push_back(b[i]->lat->g.Vh);
      }
    }
    const size_t fbytes = (size_t)vh_max * nc * 16 * 2 * total;
    clg_status st;
    if ((st = dalloc(ctx, (void**)&nw->seg_dev, sizeof(HopSeg) * segs.size())) ||
        (st = dalloc(ctx, (void**)&nw->vh_dev, sizeof(int64_t) * vhs.size())) ||
        (st = dalloc(ctx, (void**)&nw->tile_dev, sizeof(BatchTile) * tiles.size())) ||
        (st = dalloc(ctx, &nw->b_data, fbytes)) || (st = dalloc(ctx, &nw->x_data, fbytes)))
      return st;
    cudaMemsetAsync(nw->b_data, 0, fbytes, ctx->stream);
    cudaMemsetAsync(nw->x_data, 0, fbytes, ctx->stream);
    if (cudaMemcpyAsync(nw->seg_dev, segs.data(), sizeof(HopSeg) * segs.size(), cudaMemcpyHostToDevice, ctx->stream) !=
            cudaSuccess ||
        cudaMemcpyAsync(nw->vh_dev, vhs.data(), sizeof(int64_t) * vhs.size(), cudaMemcpyHostToDevice, ctx->stream) !=
            cudaSuccess ||
        cudaMemcpyAsync(nw->tile_dev, tiles.data(), sizeof(BatchTile) * tiles.size(), cudaMemcpyHostToDevice,
                        ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess)
      return ctx->fail(CLG_ERR_CUDA, "solve_lattices: table upload");
    nw->vgauge.seg = nw->seg_dev;
    nw->vgauge.seg_vh = nw->vh_dev;
    nw->vgauge.btile = nw->tile_dev;
    nw->vgauge.nbtile = (int)tiles.size();
    nw->vgauge.btiles = ntiles;
    nw->B = padded_full(static_cast<char*>(nw->b_data), nc, total, vh_max);
    nw->X = padded_full(static_cast<char*>(nw->x_data), nc, total, vh_max);
    nw->key = key;
    W = nw.get();
    S->cache_batch = std::move(nw);
  }
  // the right-hand sides in, lattice by lattice
  int off = 0;
  for (int i = 0; i < n; ++i) {
    const FieldRef bi = b[i]->ref();
    if (clg_status st = blas_copy_strided(ctx, W->B.rhs_view(off, bi.nrhs), bi)) return st;
    off += bi.nrhs;
  }
  SolveReq q;
  q.cache = &W->solve_cache;
  q.ctx = ctx;
  q.prm = &S->p;
  q.U = &W->vgauge;
  q.lat = &W->vlat;
  q.kind = CLG_FERMION_WILSON;
  q.param = b[0]->param;
  q.op = op;
  q.subset = CLG_SUBSET_FULL;
  q.nrhs = total;
  q.b = W->B;
  q.xout.push_back(W->X);
  q.info = info;
  // the solve's site kernels skip each right-hand side's padding
  ctx->batch_vh = W->vh_dev;
  ctx->batch_vh_stride = vh_max;
  ctx->batch_nrhs = total;
  const clg_status s = solve_core(q);
  ctx->batch_vh = nullptr;
  ctx->batch_vh_stride = 0;
  ctx->batch_nrhs = 0;
  if (s && s != CLG_ERR_NOT_CONVERGED && s != CLG_ERR_BREAKDOWN) return s;
  off = 0;
  for (int i = 0; i < n; ++i) {
    const FieldRef xi = x[i]->ref();
    if (clg_status st = blas_copy_strided(ctx, xi, W->X.rhs_view(off, xi.nrhs))) return st;
    off += xi.nrhs;
  }
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return ctx->fail(CLG_ERR_CUDA, "solve_lattices: sync");
  return s;
}
