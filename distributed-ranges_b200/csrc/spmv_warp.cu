// spmv_warp.cu -- plan, dispatch and autotuning of the persistent
// warp-granular SpMV (kernels in spmv_warp.cuh, instantiated per storage type
// in spmv_warp_f32.cu, spmv_warp_f64.cu and spmv_warp_bf16.cu).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "spmv_warp.cuh"

namespace drb {

using warpk::kRows;
using warpk::WarpResid;

// Kernel variant: item span 128, 256 or 512 nonzeros, skewed or plain product
// layout (128: 40-48 registers instead of 64, so 5-6 CTAs per SM instead of 4,
// for storage whose 16-byte group is at most 4 elements), and | 2 for the
// two-slot pipelined kernel of the plain product (128 or 256, skewed).  Encoded as tile | (skew ? 1 : 0) in build_pipe_plan's `tile`
// argument (0 = choose).  The choice does not change results beyond the
// summation order of a chunked row, which is the same for both layouts.
//
// Default (measured on B200, random columns, 336M nonzeros, 64 MB x):
// 256-nonzero items with the skewed layout are fastest or tied at every row
// length (fixed rows of 16..4096 nonzeros: 1.33-1.49 ms; the bench's
// power-law: 1.61 ms against 1.97 ms for 512-nonzero items) once chunked
// rows finish in a separate pass.  The environment variable
// DRB_SPMV_VARIANT="tile,skew" (e.g. "512,0") overrides it for handles
// created afterwards ("128,1,1": the two-slot kernel); drb_csr_autotune
// measures them all instead.
int choose_pipe_variant(int64_t, const void *, int) {
  if (const char *e = std::getenv("DRB_SPMV_VARIANT")) {
    const int t = std::atoi(e);
    const char *c = std::strchr(e, ',');
    const int sk = c ? std::atoi(c + 1) : 0;
    const char *c2 = c ? std::strchr(c + 1, ',') : nullptr;
    const int two = c2 ? std::atoi(c2 + 1) : 0;
    if (t == 128 || t == 256 || t == 512)
      return t | (sk ? 1 : 0) | (two ? 2 : 0);
  }
  return 256 | 1;
}

drb_status build_pipe_plan(PipePlan &plan, int64_t m, const void *rowptr_host,
                           int rbytes, int group, int tile, int rows) {
  plan.gen++; // graphs captured over the old items are stale
  if (tile == 0)
    tile = choose_pipe_variant(m, rowptr_host, rbytes);
  plan.skew = (tile & 1) != 0;
  plan.two_slot = (tile & 2) != 0;
  tile &= ~3;
  if (tile != 128 && tile != 256 && tile != 512)
    tile = 256;
  if (tile == 128 && group > 4) // a 128-nonzero item holds 32 groups of at most 4
    tile = 256;
  if (plan.two_slot) {
    plan.skew = true; // the pipelined kernel uses the skewed layout only
    if (tile == 512)
      plan.two_slot = false;
  }
  if (rows <= 0 || rows > kRows)
    rows = kRows;
  plan.tile = tile;
  plan.rows = rows;
  plan.group = group;
  auto RP = [&](int64_t i) -> int64_t {
    return rbytes == 4 ? (int64_t)((const int32_t *)rowptr_host)[i]
                       : ((const int64_t *)rowptr_host)[i];
  };
  const int64_t G = group;
  std::vector<Item> longi, tiles;
  std::vector<Chunk> chunks;
  std::vector<int4> splits;
  int64_t nsplit = 0;
  int64_t r = 0;
  while (r < m) {
    const int64_t p0 = RP(r), a0 = p0 & ~(G - 1), p1 = RP(r + 1);
    if (p1 - a0 > tile) {
      // a row wider than one item: aligned chunks of `tile` elements
      const int64_t nch = (p1 - a0 + tile - 1) / tile;
      const int first = (int)chunks.size();
      for (int64_t i = 0; i < nch; i++) {
        Chunk c;
        c.p0 = std::max(p0, a0 + i * tile);
        c.p1 = std::min(p1, a0 + (i + 1) * tile);
        c.row = (int32_t)r;
        c.first = first;
        c.count = (int32_t)nch;
        c.counter = (int32_t)nsplit;
        chunks.push_back(c);
        Item it{};
        it.p0 = c.p0;
        it.len = (int32_t)(c.p1 - c.p0);
        it.r0 = (int32_t)r;
        it.nrows = 0;
        it.chunk = first + (int32_t)i;
        longi.push_back(it);
      }
      splits.push_back(make_int4((int)r, first, (int)nch, 0));
      nsplit++;
      r++;
      continue;
    }
    int64_t r1 = r + 1;
    while (r1 < m && r1 - r < rows && RP(r1 + 1) - a0 <= tile)
      r1++;
    Item it{};
    it.p0 = p0;
    it.len = (int32_t)(RP(r1) - p0);
    it.r0 = (int32_t)r;
    it.nrows = (int32_t)(r1 - r);
    it.chunk = -1;
    tiles.push_back(it);
    r = r1;
  }
  // Interleave chunk items with whole-row items so every warp's share mixes
  // both kinds.
  std::vector<Item> all;
  all.reserve(longi.size() + tiles.size());
  size_t a = 0, b = 0;
  const double ratio = tiles.empty() ? 0.0 : (double)longi.size() / (double)tiles.size();
  double acc = 0.0;
  while (a < longi.size() || b < tiles.size()) {
    if (b < tiles.size()) {
      all.push_back(tiles[b++]);
      acc += ratio;
    }
    while (a < longi.size() && (acc >= 1.0 || b >= tiles.size())) {
      all.push_back(longi[a++]);
      acc -= 1.0;
    }
  }
  plan.seg_items.release(); // the row-segment order is rebuilt on demand
  plan.seg_c0.clear();
  plan.seg_blk.clear();
  plan.seg_i0.clear();
  plan.seg_r0.clear();
  plan.nitems = (int64_t)all.size();
  plan.nchunks = (int64_t)chunks.size();
  plan.nsplit = nsplit;
  DRB_TRY(plan.items.alloc(sizeof(Item) * std::max<size_t>(all.size(), 1)));
  if (!all.empty())
    DRB_CUDA_TRY(cudaMemcpy(plan.items.p, all.data(), sizeof(Item) * all.size(),
                            cudaMemcpyHostToDevice));
  DRB_TRY(plan.chunks.alloc(sizeof(Chunk) * std::max<size_t>(chunks.size(), 1)));
  if (!chunks.empty())
    DRB_CUDA_TRY(cudaMemcpy(plan.chunks.p, chunks.data(), sizeof(Chunk) * chunks.size(),
                            cudaMemcpyHostToDevice));
  DRB_TRY(plan.splits.alloc(sizeof(int4) * std::max<size_t>(splits.size(), 1)));
  if (!splits.empty())
    DRB_CUDA_TRY(cudaMemcpy(plan.splits.p, splits.data(), sizeof(int4) * splits.size(),
                            cudaMemcpyHostToDevice));
  plan.split_first.resize(splits.size());
  for (size_t i = 0; i < splits.size(); i++)
    plan.split_first[i] = splits[i].y;
  DRB_TRY(plan.partials.alloc(sizeof(double) * std::max<size_t>(chunks.size(), 1)));
  DRB_TRY(plan.counters.alloc(sizeof(int) * std::max<int64_t>(nsplit, 1)));
  DRB_CUDA_TRY(cudaMemset(plan.counters.p, 0, plan.counters.bytes));
  DRB_TRY(plan.err.alloc(sizeof(int) * 4));
  DRB_CUDA_TRY(cudaMemset(plan.err.p, 0, plan.err.bytes));
  return DRB_OK;
}

drb_status spmv_pipe_launch(Csr &A, const void *x, void *y, cudaStream_t s) {
  if (A.sell.on)
    return sell_launch(A, x, y, nullptr, 0, A.sell.nslices, s);
  switch (A.storage) {
  case DRB_F32:
    return warp_launch_f32(A, x, y, nullptr, (A.flags & DRB_FLAG_COMPENSATED) != 0, s);
  case DRB_F64:
    return warp_launch_f64(A, x, y, nullptr, s);
  case DRB_BF16:
    return warp_launch_bf16(A, x, y, (A.flags & DRB_FLAG_BF16_X_F32) != 0, s);
  }
  set_error("spmv: storage type not handled");
  return DRB_ERR_UNSUPPORTED;
}

drb_status fused_scratch(Csr &A) {
  PipePlan &P = A.pipe;
  int sms = 0;
  DRB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, A.device));
  // [per-CTA partials][ticket, 16 bytes][per-item partials]
  const size_t bytes = sizeof(double) * ((size_t)sms * 32 + (size_t)P.nitems) + 16;
  if (!P.red.p || P.red.bytes < bytes) {
    DRB_TRY(P.red.alloc(bytes));
    DRB_CUDA_TRY(cudaMemset(P.red.p, 0, P.red.bytes));
  }
  return DRB_OK;
}

namespace {
// y = A x with a fused row reduction into *out (see WarpResid).
drb_status fused_pipe_launch(Csr &A, const void *x, const void *b, void *y, double *out,
                             bool dot, const int *stop, cudaStream_t s) {
  PipePlan &P = A.pipe;
  if (P.nitems == 0) {
    DRB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double), s));
    return DRB_OK;
  }
  int sms = 0;
  DRB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, A.device));
  const size_t slots = (size_t)sms * 32;
  DRB_TRY(fused_scratch(A));
  WarpResid ra;
  ra.b = b;
  ra.partials = P.red.as<double>();
  ra.ticket = reinterpret_cast<int *>(P.red.as<double>() + slots);
  ra.ipart = P.red.as<double>() + slots + 2;
  ra.out = out;
  ra.stop = stop;
  ra.dot = dot ? 1 : 0;
  if (A.sell.on)
    return sell_launch(A, x, y, &ra, 0, A.sell.nslices, s);
  if (A.storage == DRB_F32)
    return warp_launch_f32(A, x, y, &ra, false, s);
  if (A.storage == DRB_F64)
    return warp_launch_f64(A, x, y, &ra, s);
  set_error("fused SpMV reduction: storage type not handled");
  return DRB_ERR_UNSUPPORTED;
}
} // namespace

drb_status residual_pipe_launch(Csr &A, const void *x, const void *b, void *y,
                                double *out, cudaStream_t s) {
  return fused_pipe_launch(A, x, b, y, out, false, nullptr, s);
}

drb_status rowdot_pipe_launch(Csr &A, const void *x, const void *w, void *y,
                              double *out, const int *stop, cudaStream_t s) {
  return fused_pipe_launch(A, x, w, y, out, true, stop, s);
}

int plan_group(int vbytes, int cbytes);

// Times the single-RHS row-block variants (128-, 256- and 512-nonzero items,
// skewed or plain layout; 128 only for 4-byte groups), and the sliced-ELL copy when
// the matrix qualifies for one, on this matrix's sparsity pattern (x = 0,
// three launches each after one warm-up) and keeps the fastest.  Returns the
// chosen variant (tile | skew, or kVariantSell) in *chosen.
drb_status autotune_pipe(Csr &A, cudaStream_t s, int *chosen) {
  const int vb = dtype_bytes(A.storage);
  const int group = plan_group(vb, A.cbytes);
  std::vector<char> rp((size_t)A.rbytes * (A.m + 1));
  if (A.m >= 0)
    DRB_CUDA_TRY(cudaMemcpy(rp.data(), A.rowptr.p, rp.size(), cudaMemcpyDeviceToHost));
  DevBuf xb, yb;
  DRB_TRY(xb.alloc((size_t)vb * (A.n + 1)));
  DRB_TRY(yb.alloc((size_t)8 * (A.m + 1)));
  DRB_CUDA_TRY(cudaMemsetAsync(xb.p, 0, xb.bytes, s));
  cudaEvent_t e0, e1;
  DRB_CUDA_TRY(cudaEventCreate(&e0));
  DRB_CUDA_TRY(cudaEventCreate(&e1));
  // the row-block variants, then the sliced-ELL copy when the rows allow one
  if (!A.sell.built)
    DRB_TRY(sell_build(A, rp.data(), A.rbytes, s));
  std::vector<int> variants = {256 | 1, 256, 512 | 1, 512, 256 | 3};
  if (group <= 4) { // 128-nonzero items: fewer registers, more warps per SM
    variants.push_back(128 | 1);
    variants.push_back(128);
    variants.push_back(128 | 3);
  }
  if (A.sell.built)
    variants.push_back(kVariantSell);
  const int nvar = (int)variants.size();
  std::vector<float> vms(nvar, 3.4e38f);
  drb_status st = DRB_OK;
  // Two rounds over the variants, each variant's best kept, after ~30 ms of
  // warm-up launches: a first variant timed while the clocks still ramp up
  // from idle would otherwise lose to a slower one timed later.
  A.sell.on = false;
  st = build_pipe_plan(A.pipe, A.m, rp.data(), A.rbytes, group, variants[0], 0);
  float warm = 0.f;
  for (int w = 0; w < 50 && st == DRB_OK; w++) {
    cudaEventRecord(e0, s);
    st = spmv_pipe_launch(A, xb.p, yb.p, s);
    cudaEventRecord(e1, s);
    float ms = 0.f;
    if (st != DRB_OK || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
      break;
    warm += ms;
    if (w >= 4 && warm >= 30.f)
      break;
  }
  for (int round = 0; round < 2 && st == DRB_OK; round++) {
    for (int iv = 0; iv < nvar; iv++) {
      const int v = variants[iv];
      A.sell.on = v == kVariantSell;
      if (!A.sell.on)
        st = build_pipe_plan(A.pipe, A.m, rp.data(), A.rbytes, group, v, 0);
      if (st != DRB_OK)
        break;
      if ((st = spmv_pipe_launch(A, xb.p, yb.p, s)) != DRB_OK)
        break;
      // the fastest of five separately timed launches: variants differ by a
      // few percent, less than the spread of a sum of launches
      for (int i = 0; i < 5 && st == DRB_OK; i++) {
        cudaEventRecord(e0, s);
        st = spmv_pipe_launch(A, xb.p, yb.p, s);
        cudaEventRecord(e1, s);
        float ms = 0.f;
        if (st != DRB_OK || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
          if (st == DRB_OK)
            st = DRB_ERR_CUDA;
          break;
        }
        vms[iv] = std::min(vms[iv], ms);
      }
    }
  }
  int best = variants[0], best_rb = variants[0];
  float best_ms = 3.4e38f, best_rb_ms = 3.4e38f;
  for (int iv = 0; iv < nvar; iv++) {
    if (vms[iv] < best_ms) {
      best_ms = vms[iv];
      best = variants[iv];
    }
    if (variants[iv] != kVariantSell && vms[iv] < best_rb_ms) {
      best_rb_ms = vms[iv];
      best_rb = variants[iv];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  DRB_TRY(st);
  A.sell.on = best == kVariantSell;
  // the row-block plan stays built (the multi-RHS and adjoint paths use it);
  // its rebuild also marks captured graphs stale
  DRB_TRY(build_pipe_plan(A.pipe, A.m, rp.data(), A.rbytes, group, best_rb, 0));
  if (!A.sell.on)
    sell_release(A);
  if (chosen)
    *chosen = best;
  return DRB_OK;
}

// Reads and clears the handle's device error word (set by kernels whose
// bounded device-side waits expired).
drb_status pipe_check(Csr &A, cudaStream_t s) {
  if (!A.pipe.err.p)
    return DRB_OK;
  int e = 0;
  DRB_CUDA_TRY(cudaMemcpyAsync(&e, A.pipe.err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  DRB_CUDA_TRY(cudaStreamSynchronize(s));
  if (e != 0) {
    DRB_CUDA_TRY(cudaMemsetAsync(A.pipe.err.p, 0, sizeof(int), s));
    set_error("a device-side wait timed out");
    return DRB_ERR_TIMEOUT;
  }
  return DRB_OK;
}

} // namespace drb
