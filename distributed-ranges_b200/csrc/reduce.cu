// reduce.cu -- mp::reduce over a device vector and the element-wise fills a
// distributed_vector needs (iota, fill).
//
// mp::reduce (include/dr/mp/algorithms/reduce.hpp:58-181) reduces each rank's
// local segments, gathers one partial per rank and combines them on the root
// (or on every rank), then applies `init` last: binary_op(init, reduce(r))
// (reduce.hpp:110-120); an empty range gives init, or value_type{} without
// one (reduce.hpp:63-65).  Here every segment is on one GPU, so the reduce is
// one launch: a fixed grid of kRedGrid CTAs, each thread striding over the
// vector with 16-byte loads, a per-CTA tree, and the last CTA (completion
// ticket) combining the per-CTA partials in index order.  The grouping
// depends only on n and x's address modulo 16, so results are deterministic.
//
// Accumulation: integer sums wrap modulo 2^32 / 2^64 (two's-complement
// addition is associative, so the result equals the sequential loop's
// wrapped sum bit for bit); float sums accumulate in double and round once
// to the element type before init is applied; min and max compare in the
// element type with std::min / std::max's rule ((b < a) ? b : a and
// (a < b) ? b : a).
#include <cstdint>
#include <cstring>
#include <limits>

#include "drb_internal.cuh"

namespace drb {
namespace {

constexpr int kRedNT = 256;
constexpr int kRedGrid = 592; // fixed: the grouping must not depend on the GPU
constexpr int kRedUnroll = 4; // 16-byte loads in flight per thread

template <class T> struct SumAcc { using type = T; };
template <> struct SumAcc<float> { using type = double; };
template <> struct SumAcc<int32_t> { using type = uint32_t; };
template <> struct SumAcc<int64_t> { using type = uint64_t; };

// One reduction: accumulator type A, identity, combine, element -> A, A -> T.
template <class T, int OP> struct ROp;
template <class T> struct ROp<T, DRB_REDUCE_SUM> {
  using A = typename SumAcc<T>::type;
  __device__ static A id() { return A(0); }
  __device__ static A f(A a, A b) { return a + b; }
  __device__ static A lift(T v) { return static_cast<A>(v); }
  __device__ static T out(A a, bool has_init, T init) {
    const T t = static_cast<T>(a);
    if (!has_init)
      return t;
    if constexpr (std::is_integral<T>::value)
      return static_cast<T>(static_cast<A>(init) + static_cast<A>(t));
    else
      return init + t;
  }
};
template <class T> struct ROp<T, DRB_REDUCE_MIN> {
  using A = T;
  __device__ static A id() {
    if constexpr (std::is_integral<T>::value)
      return std::numeric_limits<T>::max();
    else
      return std::numeric_limits<T>::infinity();
  }
  __device__ static A f(A a, A b) { return (b < a) ? b : a; }
  __device__ static A lift(T v) { return v; }
  __device__ static T out(A a, bool has_init, T init) { return has_init ? f(init, a) : a; }
};
template <class T> struct ROp<T, DRB_REDUCE_MAX> {
  using A = T;
  __device__ static A id() {
    if constexpr (std::is_integral<T>::value)
      return std::numeric_limits<T>::lowest();
    else
      return -std::numeric_limits<T>::infinity();
  }
  __device__ static A f(A a, A b) { return (a < b) ? b : a; }
  __device__ static A lift(T v) { return v; }
  __device__ static T out(A a, bool has_init, T init) { return has_init ? f(init, a) : a; }
};

template <class A> __device__ __forceinline__ A shfl_down(A v, int o) {
  return __shfl_down_sync(0xffffffffu, v, o);
}

template <class T, int OP>
__global__ void __launch_bounds__(kRedNT)
    reduce_kernel(int64_t n, const T *__restrict__ x, bool has_init, T init,
                  typename ROp<T, OP>::A *partials, int *ticket, T *out) {
  using R = ROp<T, OP>;
  using A = typename R::A;
  __shared__ A s_red[kRedNT / 32];
  __shared__ int s_last;
  constexpr int PER = 16 / sizeof(T);
  const uint64_t pol = ptx::policy_evict_first();
  A acc = R::id();
  const int64_t tid = (int64_t)blockIdx.x * kRedNT + threadIdx.x;
  const int64_t nth = (int64_t)gridDim.x * kRedNT;
  int64_t head = 0; // elements before the first 16-byte boundary
  const uintptr_t mis = reinterpret_cast<uintptr_t>(x) % 16;
  if (mis % sizeof(T) == 0) {
    head = mis ? (int64_t)((16 - mis) / sizeof(T)) : 0;
    head = head < n ? head : n;
    const int64_t nv = (n - head) / PER;
    const T *xa = x + head;
    union W {
      uint4 u;
      T t[PER];
    };
    int64_t i = tid;
    // kRedUnroll grid-strided vectors per trip, all loads issued first
    for (; i + (kRedUnroll - 1) * nth < nv; i += kRedUnroll * nth) {
      W w[kRedUnroll];
#pragma unroll
      for (int u = 0; u < kRedUnroll; u++)
        w[u].u = ptx::ld_stream16(xa + (i + u * nth) * PER, pol);
#pragma unroll
      for (int u = 0; u < kRedUnroll; u++)
#pragma unroll
        for (int q = 0; q < PER; q++)
          acc = R::f(acc, R::lift(w[u].t[q]));
    }
    for (; i < nv; i += nth) {
      W w;
      w.u = ptx::ld_stream16(xa + i * PER, pol);
#pragma unroll
      for (int q = 0; q < PER; q++)
        acc = R::f(acc, R::lift(w.t[q]));
    }
    for (int64_t i = head + nv * PER + tid; i < n; i += nth)
      acc = R::f(acc, R::lift(x[i]));
    for (int64_t i = tid; i < head; i += nth)
      acc = R::f(acc, R::lift(x[i]));
  } else {
    for (int64_t i = tid; i < n; i += nth)
      acc = R::f(acc, R::lift(x[i]));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1)
    acc = R::f(acc, shfl_down(acc, o));
  if (lane == 0)
    s_red[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    A s = R::id();
    for (int w = 0; w < kRedNT / 32; w++)
      s = R::f(s, s_red[w]);
    partials[blockIdx.x] = s;
    __threadfence();
    s_last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last)
    return;
  __threadfence();
  A s = R::id();
  for (int i = threadIdx.x; i < (int)gridDim.x; i += kRedNT)
    s = R::f(s, __ldcg(&partials[i]));
  for (int o = 16; o > 0; o >>= 1)
    s = R::f(s, shfl_down(s, o));
  __syncthreads();
  if (lane == 0)
    s_red[warp] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    A t = R::id();
    for (int w = 0; w < kRedNT / 32; w++)
      t = R::f(t, s_red[w]);
    *out = n > 0 ? R::out(t, has_init, init) : (has_init ? init : T(0));
    *ticket = 0;
  }
}

template <class T, int OP>
drb_status reduce_typed(int64_t n, const void *x, const void *init, void *out,
                        cudaStream_t s) {
  using A = typename ROp<T, OP>::A;
  T iv{};
  if (init)
    std::memcpy(&iv, init, sizeof(T));
  void *scratch = nullptr;
  const size_t bytes = sizeof(A) * kRedGrid + 16;
  DRB_TRY(scratch_alloc(&scratch, bytes, s));
  A *partials = static_cast<A *>(scratch);
  int *ticket = reinterpret_cast<int *>(partials + kRedGrid);
  cudaError_t e = cudaMemsetAsync(ticket, 0, sizeof(int), s);
  if (e == cudaSuccess) {
    // small inputs take fewer CTAs; the grid is still a function of n only
    const int64_t want = (n + kRedNT * 16 - 1) / (kRedNT * 16);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(kRedGrid, want));
    reduce_kernel<T, OP><<<grid, kRedNT, 0, s>>>(n, static_cast<const T *>(x), init != nullptr,
                                                 iv, partials, ticket, static_cast<T *>(out));
    note_launch();
    e = cudaGetLastError();
  }
  scratch_free(scratch, s);
  if (e != cudaSuccess) {
    set_error("reduce launch: %s", cudaGetErrorString(e));
    return DRB_ERR_CUDA;
  }
  return DRB_OK;
}

template <class T>
drb_status reduce_op(int64_t n, const void *x, drb_reduce_op op, const void *init,
                     void *out, cudaStream_t s) {
  switch (op) {
  case DRB_REDUCE_SUM:
    return reduce_typed<T, DRB_REDUCE_SUM>(n, x, init, out, s);
  case DRB_REDUCE_MIN:
    return reduce_typed<T, DRB_REDUCE_MIN>(n, x, init, out, s);
  case DRB_REDUCE_MAX:
    return reduce_typed<T, DRB_REDUCE_MAX>(n, x, init, out, s);
  }
  set_error("reduce: op %d not supported", (int)op);
  return DRB_ERR_INVALID_ARG;
}

// ---- iota / fill -----------------------------------------------------------
template <class T>
__global__ void iota_kernel(int64_t n, T *__restrict__ x, int64_t start) {
  const int64_t nth = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += nth)
    x[i] = static_cast<T>(start + i);
}

template <class T>
__global__ void fill_kernel(int64_t n, T *__restrict__ x, T v) {
  const int64_t nth = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += nth)
    x[i] = v;
}

int fill_grid(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>(148 * 8, (n + 255) / 256));
}

} // namespace

bool elementwise_dtype(drb_dtype t) {
  return t == DRB_F32 || t == DRB_F64 || t == DRB_INT32 || t == DRB_INT64;
}

drb_status reduce_launch(int64_t n, const void *x, drb_dtype dt, drb_reduce_op op,
                         const void *init, void *out, cudaStream_t s) {
  switch (dt) {
  case DRB_F32:
    return reduce_op<float>(n, x, op, init, out, s);
  case DRB_F64:
    return reduce_op<double>(n, x, op, init, out, s);
  case DRB_INT32:
    return reduce_op<int32_t>(n, x, op, init, out, s);
  case DRB_INT64:
    return reduce_op<int64_t>(n, x, op, init, out, s);
  default:
    break;
  }
  set_error("reduce: dtype %d not supported", (int)dt);
  return DRB_ERR_UNSUPPORTED;
}

drb_status iota_launch(int64_t n, void *x, drb_dtype dt, int64_t start, cudaStream_t s) {
  if (n == 0)
    return DRB_OK;
  const int g = fill_grid(n);
  switch (dt) {
  case DRB_F32: iota_kernel<float><<<g, 256, 0, s>>>(n, (float *)x, start); break;
  case DRB_F64: iota_kernel<double><<<g, 256, 0, s>>>(n, (double *)x, start); break;
  case DRB_INT32: iota_kernel<int32_t><<<g, 256, 0, s>>>(n, (int32_t *)x, start); break;
  case DRB_INT64: iota_kernel<int64_t><<<g, 256, 0, s>>>(n, (int64_t *)x, start); break;
  default:
    set_error("iota: dtype %d not supported", (int)dt);
    return DRB_ERR_UNSUPPORTED;
  }
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}

drb_status fill_launch(int64_t n, void *x, drb_dtype dt, const void *value, cudaStream_t s) {
  if (n == 0)
    return DRB_OK;
  const int g = fill_grid(n);
  switch (dt) {
  case DRB_F32: {
    float v;
    std::memcpy(&v, value, 4);
    fill_kernel<float><<<g, 256, 0, s>>>(n, (float *)x, v);
    break;
  }
  case DRB_F64: {
    double v;
    std::memcpy(&v, value, 8);
    fill_kernel<double><<<g, 256, 0, s>>>(n, (double *)x, v);
    break;
  }
  case DRB_INT32: {
    int32_t v;
    std::memcpy(&v, value, 4);
    fill_kernel<int32_t><<<g, 256, 0, s>>>(n, (int32_t *)x, v);
    break;
  }
  case DRB_INT64: {
    int64_t v;
    std::memcpy(&v, value, 8);
    fill_kernel<int64_t><<<g, 256, 0, s>>>(n, (int64_t *)x, v);
    break;
  }
  default:
    set_error("fill: dtype %d not supported", (int)dt);
    return DRB_ERR_UNSUPPORTED;
  }
  note_launch();
  DRB_CUDA_TRY(cudaGetLastError());
  return DRB_OK;
}

} // namespace drb
