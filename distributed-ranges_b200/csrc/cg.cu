// cg.cu -- unpreconditioned conjugate gradients with every vector and scalar
// on the device.
//
// The reference gives the pieces -- gemv (include/dr/mp/algorithms/matrix/
// gemv.hpp:16-27), reduce over a distributed_vector (reduce.hpp:58-181) and
// element-wise transforms -- and leaves the loop to the caller, who would pay
// a host round trip per reduction.  Here one iteration is three launches:
//
//   1. the persistent SpMV, q = A p, with p.q summed in its row epilogue
//      (rowdot_pipe_launch; the same deterministic per-CTA partials + last-CTA
//      combine as the fused residual);
//   2. cg_update: alpha = rr / p.q from device memory, x += alpha p,
//      r -= alpha q, and r.r summed on the way (the last CTA stores rr, beta,
//      the iteration count and the stop word);
//   3. cg_pupdate: p = r + beta p.
//
// kCgBlock iterations are captured once into a CUDA graph and replayed; after
// each replay the state word is copied to pinned host memory behind an event
// while the next replay is already queued, so the host never stalls the GPU.
// Once the stop word is set every kernel of the remaining iterations returns
// at its first instruction.  Vectors are the matrix's value type (f32 / f64);
// the scalars are f64.
#include <cmath>

#include "drb_internal.cuh"

namespace drb {

namespace {
constexpr int kCgNT = 256;
// 3 CTAs per SM, all resident at once (the kernels are bounded to fit);
// fixed, so the sums are deterministic
constexpr int kCgGrid = 148 * 3;
constexpr int kCgMinBlocks = 3;
constexpr int kCgBlock = 8;  // iterations per graph replay

enum : int { kRunning = 0, kConverged = 1, kBreakdown = 2, kMaxIters = 3 };

struct CgState {
  double rr;   // r.r of the current residual
  double pq;   // p.Ap of the current iteration (written by the SpMV)
  double beta; // rr' / rr of the last update
  double bb;   // b.b
  double tol2; // rtol^2 * b.b
  int64_t iters, max_iters;
  int done; // kRunning, kConverged, kBreakdown, kMaxIters
  int pad;
};
} // namespace

struct CgPlan {
  DevBuf r, p, q, state, scratch; // scratch: double[2 * kCgGrid] + ticket
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const void *gx = nullptr; // the x the graph was captured with
  uint64_t gen = 0;         // and the SpMV plan generation
  CgState *host = nullptr;  // two pinned slots
  cudaEvent_t ev[2] = {nullptr, nullptr};
  ~CgPlan() {
    if (exec)
      cudaGraphExecDestroy(exec);
    if (graph)
      cudaGraphDestroy(graph);
    for (cudaEvent_t e : ev)
      if (e)
        cudaEventDestroy(e);
    if (host)
      cudaFreeHost(host);
  }
};

void CgPlanDeleter::operator()(CgPlan *p) const { delete p; }

namespace {

__device__ __forceinline__ double wsum(double v) {
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Sums NV per-thread values over the grid.  Every CTA stores its NV partials;
// the last CTA to arrive (ticket) adds them in CTA order and returns true in
// its thread 0 with the totals in tot.  The ticket is re-armed.
template <int NV>
__device__ bool grid_sums(const double (&v)[NV], double *partials, int *ticket,
                          double (&tot)[NV]) {
  __shared__ double s_red[NV][kCgNT / 32];
  __shared__ int s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NV; j++) {
    const double t = wsum(v[j]);
    if (lane == 0)
      s_red[j][warp] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; j++) {
      double c = 0.0;
      for (int w = 0; w < kCgNT / 32; w++)
        c += s_red[j][w];
      partials[(size_t)j * kCgGrid + blockIdx.x] = c;
    }
    __threadfence();
    s_last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last)
    return false;
  __threadfence();
#pragma unroll
  for (int j = 0; j < NV; j++) {
    double c = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += kCgNT)
      c += __ldcg(&partials[(size_t)j * kCgGrid + i]);
    c = wsum(c);
    __syncthreads();
    if (lane == 0)
      s_red[j][warp] = c;
  }
  __syncthreads();
  if (threadIdx.x != 0)
    return false;
#pragma unroll
  for (int j = 0; j < NV; j++) {
    double c = 0.0;
    for (int w = 0; w < kCgNT / 32; w++)
      c += s_red[j][w];
    tot[j] = c;
  }
  *ticket = 0;
  return true;
}

// r = b - q (q = A x0), p = r; rr = r.r, bb = b.b; the stop word starts the
// loop (or ends it at once when x0 already meets the tolerance).
template <class T>
__global__ void __launch_bounds__(kCgNT, kCgMinBlocks)
    cg_init(int64_t n, const T *__restrict__ b, const T *__restrict__ q, T *__restrict__ r,
            T *__restrict__ p, CgState *st, double rtol, int64_t max_iters,
            double *partials, int *ticket) {
  double acc[2] = {0.0, 0.0};
  const int64_t nth = (int64_t)gridDim.x * kCgNT;
  for (int64_t i = (int64_t)blockIdx.x * kCgNT + threadIdx.x; i < n; i += nth) {
    const T bi = b[i];
    const T ri = bi - q[i];
    r[i] = ri;
    p[i] = ri;
    acc[0] += (double)ri * (double)ri;
    acc[1] += (double)bi * (double)bi;
  }
  double tot[2];
  if (grid_sums<2>(acc, partials, ticket, tot)) {
    st->rr = tot[0];
    st->bb = tot[1];
    st->tol2 = rtol * rtol * tot[1];
    st->pq = 0.0;
    st->beta = 0.0;
    st->iters = 0;
    st->max_iters = max_iters;
    st->done = tot[0] <= st->tol2 ? kConverged : (max_iters <= 0 ? kMaxIters : kRunning);
  }
}

// 16 bytes of T (two doubles or four floats).
template <class T> union Vec16T {
  uint4 u;
  T t[16 / sizeof(T)];
};

// alpha = rr / p.q; x += alpha p; r -= alpha q; rr' = r.r; beta = rr' / rr.
// With VEC (x, r, p, q all 16-byte aligned) every thread moves 16-byte
// vectors, two of them per loop trip, so enough bytes are in flight to
// stream at the HBM rate; the scalar tail follows.
template <class T, bool VEC>
__global__ void __launch_bounds__(kCgNT, kCgMinBlocks)
    cg_update(int64_t n, T *__restrict__ x, T *__restrict__ r, const T *__restrict__ p,
              const T *__restrict__ q, CgState *st, double *partials, int *ticket) {
  const volatile CgState *vs = st;
  if (vs->done != kRunning)
    return; // uniform over the grid
  const double rr = vs->rr, pq = vs->pq;
  const double alpha = rr / pq;
  if (!(pq > 0.0) || !isfinite(alpha)) {
    // every CTA sees the same scalars and leaves x and r as they were
    if (blockIdx.x == 0 && threadIdx.x == 0)
      st->done = kBreakdown;
    return;
  }
  double acc[1] = {0.0};
  const int64_t tid = (int64_t)blockIdx.x * kCgNT + threadIdx.x;
  const int64_t nth = (int64_t)gridDim.x * kCgNT;
  int64_t done = 0;
  if (VEC) {
    constexpr int PER = 16 / sizeof(T);
    const int64_t nv = n / PER;
    auto step = [&](int64_t i, Vec16T<T> &vx, Vec16T<T> &vr, const Vec16T<T> &vp,
                    const Vec16T<T> &vq) {
#pragma unroll
      for (int e = 0; e < PER; e++) {
        vx.t[e] = (T)((double)vx.t[e] + alpha * (double)vp.t[e]);
        vr.t[e] = (T)((double)vr.t[e] - alpha * (double)vq.t[e]);
        acc[0] += (double)vr.t[e] * (double)vr.t[e];
      }
      reinterpret_cast<uint4 *>(x)[i] = vx.u;
      reinterpret_cast<uint4 *>(r)[i] = vr.u;
    };
    for (int64_t i = tid; i < nv; i += 2 * nth) {
      const int64_t j = i + nth;
      Vec16T<T> x0, r0, p0, q0, x1, r1, p1, q1;
      x0.u = reinterpret_cast<const uint4 *>(x)[i];
      r0.u = reinterpret_cast<const uint4 *>(r)[i];
      p0.u = __ldg(reinterpret_cast<const uint4 *>(p) + i);
      q0.u = __ldg(reinterpret_cast<const uint4 *>(q) + i);
      if (j < nv) {
        x1.u = reinterpret_cast<const uint4 *>(x)[j];
        r1.u = reinterpret_cast<const uint4 *>(r)[j];
        p1.u = __ldg(reinterpret_cast<const uint4 *>(p) + j);
        q1.u = __ldg(reinterpret_cast<const uint4 *>(q) + j);
      }
      step(i, x0, r0, p0, q0);
      if (j < nv)
        step(j, x1, r1, p1, q1);
    }
    done = nv * PER;
  }
  for (int64_t i = done + tid; i < n; i += nth) {
    const T xi = (T)((double)x[i] + alpha * (double)p[i]);
    const T ri = (T)((double)r[i] - alpha * (double)q[i]);
    x[i] = xi;
    r[i] = ri;
    acc[0] += (double)ri * (double)ri;
  }
  double tot[1];
  if (grid_sums<1>(acc, partials, ticket, tot)) {
    const double rr1 = tot[0];
    const int64_t it = st->iters + 1;
    st->iters = it;
    st->beta = rr1 / rr;
    st->rr = rr1;
    st->done = rr1 <= st->tol2 ? kConverged : (it >= st->max_iters ? kMaxIters : kRunning);
  }
}

// p = r + beta p (r and p are the plan's own, 16-byte aligned buffers).
template <class T>
__global__ void __launch_bounds__(kCgNT, kCgMinBlocks)
    cg_pupdate(int64_t n, const T *__restrict__ r, T *__restrict__ p, const CgState *st) {
  const volatile CgState *vs = st;
  if (vs->done != kRunning)
    return;
  const double beta = vs->beta;
  constexpr int PER = 16 / sizeof(T);
  const int64_t tid = (int64_t)blockIdx.x * kCgNT + threadIdx.x;
  const int64_t nth = (int64_t)gridDim.x * kCgNT;
  const int64_t nv = n / PER;
  for (int64_t i = tid; i < nv; i += 2 * nth) {
    const int64_t j = i + nth;
    Vec16T<T> r0, p0, r1, p1;
    r0.u = __ldg(reinterpret_cast<const uint4 *>(r) + i);
    p0.u = reinterpret_cast<const uint4 *>(p)[i];
    if (j < nv) {
      r1.u = __ldg(reinterpret_cast<const uint4 *>(r) + j);
      p1.u = reinterpret_cast<const uint4 *>(p)[j];
    }
#pragma unroll
    for (int e = 0; e < PER; e++)
      p0.t[e] = (T)((double)r0.t[e] + beta * (double)p0.t[e]);
    reinterpret_cast<uint4 *>(p)[i] = p0.u;
    if (j < nv) {
#pragma unroll
      for (int e = 0; e < PER; e++)
        p1.t[e] = (T)((double)r1.t[e] + beta * (double)p1.t[e]);
      reinterpret_cast<uint4 *>(p)[j] = p1.u;
    }
  }
  for (int64_t i = nv * PER + tid; i < n; i += nth)
    p[i] = (T)((double)r[i] + beta * (double)p[i]);
}

int cg_grid(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>(kCgGrid, (n + kCgNT - 1) / kCgNT));
}

template <class T>
drb_status enqueue_iterations(Csr &A, CgPlan &C, T *x, int iters, cudaStream_t s) {
  const int64_t n = A.n;
  const int grid = cg_grid(n);
  auto *st = C.state.as<CgState>();
  double *partials = C.scratch.as<double>();
  int *ticket = reinterpret_cast<int *>(partials + 2 * kCgGrid);
  // x is the caller's buffer: the 16-byte path needs it aligned (r, p and q
  // are the plan's own allocations)
  const bool vec = reinterpret_cast<uintptr_t>(x) % 16 == 0;
  for (int k = 0; k < iters; k++) {
    DRB_TRY(rowdot_pipe_launch(A, C.p.p, C.p.p, C.q.p, &st->pq, &st->done, s));
    if (vec)
      cg_update<T, true><<<grid, kCgNT, 0, s>>>(n, x, C.r.as<T>(), C.p.as<T>(), C.q.as<T>(),
                                                st, partials, ticket);
    else
      cg_update<T, false><<<grid, kCgNT, 0, s>>>(n, x, C.r.as<T>(), C.p.as<T>(), C.q.as<T>(),
                                                 st, partials, ticket);
    cg_pupdate<T><<<grid, kCgNT, 0, s>>>(n, C.r.as<T>(), C.p.as<T>(), st);
    note_launch(2);
    DRB_CUDA_TRY(cudaGetLastError());
  }
  return DRB_OK;
}

template <class T>
drb_status capture_block(Csr &A, CgPlan &C, T *x) {
  if (C.exec) {
    cudaGraphExecDestroy(C.exec);
    C.exec = nullptr;
  }
  if (C.graph) {
    cudaGraphDestroy(C.graph);
    C.graph = nullptr;
  }
  cudaStream_t cs;
  DRB_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  drb_status st = DRB_OK;
  g_count_pause++;
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    st = enqueue_iterations<T>(A, C, x, kCgBlock, cs);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(cs, &g);
    if (e == cudaSuccess && st == DRB_OK) {
      C.graph = g;
      e = cudaGraphInstantiate(&C.exec, g, 0);
    } else if (g) {
      cudaGraphDestroy(g);
    }
  }
  g_count_pause--;
  cudaStreamDestroy(cs);
  if (st != DRB_OK)
    return st;
  DRB_CUDA_TRY(e);
  C.gx = x;
  C.gen = A.pipe.gen;
  return DRB_OK;
}

template <class T>
drb_status solve(Csr &A, const T *b, T *x, int64_t max_iters, double rtol,
                 drb_cg_info *info, cudaStream_t s) {
  if (!A.cg)
    A.cg.reset(new CgPlan);
  CgPlan &C = *A.cg;
  const int64_t n = A.n;
  const size_t vb = sizeof(T) * (size_t)std::max<int64_t>(n, 1);
  if (C.r.bytes < vb) {
    DRB_TRY(C.r.alloc(vb));
    DRB_TRY(C.p.alloc(vb));
    DRB_TRY(C.q.alloc(vb));
    C.gx = nullptr; // the graph holds the old p, q, r
  }
  if (!C.state.p) {
    DRB_TRY(C.state.alloc(sizeof(CgState)));
    DRB_TRY(C.scratch.alloc(sizeof(double) * 2 * kCgGrid + 16));
    DRB_CUDA_TRY(cudaMemset(C.scratch.p, 0, C.scratch.bytes)); // ticket = 0
    DRB_CUDA_TRY(cudaMallocHost(&C.host, 2 * sizeof(CgState)));
    for (cudaEvent_t &e : C.ev)
      DRB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  DRB_TRY(fused_scratch(A)); // allocated before any capture
  auto *st = C.state.as<CgState>();
  double *partials = C.scratch.as<double>();
  int *ticket = reinterpret_cast<int *>(partials + 2 * kCgGrid);

  // r = b - A x0, p = r
  DRB_TRY(spmv_pipe_launch(A, x, C.q.p, s));
  cg_init<T><<<cg_grid(n), kCgNT, 0, s>>>(n, b, C.q.as<T>(), C.r.as<T>(), C.p.as<T>(), st,
                                          rtol, max_iters, partials, ticket);
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  if (C.gx != x || C.gen != A.pipe.gen || !C.exec)
    DRB_TRY(capture_block<T>(A, C, x));

  // Replays run one block ahead of the host: the state after replay k is
  // read while replay k + 1 is queued.  Slot k % 2 holds the state copied
  // after the k-th enqueue (k = 0: after the init).
  DRB_CUDA_TRY(cudaMemcpyAsync(&C.host[0], st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
  DRB_CUDA_TRY(cudaEventRecord(C.ev[0], s));
  int64_t replays = 0;
  const int64_t max_replays = max_iters / kCgBlock + 2;
  for (int64_t k = 0;; k++) {
    // queue replay k + 1 behind the state copy of step k
    const int next = (int)((k + 1) & 1);
    if (replays < max_replays) {
      DRB_CUDA_TRY(cudaGraphLaunch(C.exec, s));
      note_launch(3 * kCgBlock);
      replays++;
      DRB_CUDA_TRY(cudaMemcpyAsync(&C.host[next], st, sizeof(CgState),
                                   cudaMemcpyDeviceToHost, s));
      DRB_CUDA_TRY(cudaEventRecord(C.ev[next], s));
    }
    DRB_CUDA_TRY(cudaEventSynchronize(C.ev[k & 1]));
    if (C.host[k & 1].done != kRunning || replays >= max_replays)
      break;
  }
  DRB_CUDA_TRY(cudaStreamSynchronize(s));
  CgState h;
  DRB_CUDA_TRY(cudaMemcpy(&h, st, sizeof(CgState), cudaMemcpyDeviceToHost));
  DRB_TRY(pipe_check(A, s));
  if (info) {
    info->iterations = h.iters;
    info->residual_norm = std::sqrt(h.rr);
    info->b_norm = std::sqrt(h.bb);
    info->converged = h.done == kConverged;
    info->breakdown = h.done == kBreakdown;
  }
  return DRB_OK;
}

} // namespace

drb_status cg_solve(Csr &A, const void *b, void *x, int64_t max_iters, double rtol,
                    drb_cg_info *info, cudaStream_t s) {
  if (A.storage == DRB_F32)
    return solve<float>(A, static_cast<const float *>(b), static_cast<float *>(x), max_iters,
                        rtol, info, s);
  if (A.storage == DRB_F64)
    return solve<double>(A, static_cast<const double *>(b), static_cast<double *>(x),
                         max_iters, rtol, info, s);
  set_error("drb_csr_cg: F32 or F64 storage required (BF16 storage is not supported)");
  return DRB_ERR_UNSUPPORTED;
}

} // namespace drb
