// spmv_warp_bf16.cu -- instantiates the persistent SpMV for bfloat16 values:
// x in bf16 (or in fp32 with DRB_FLAG_BF16_X_F32), two-sum compensated fp32
// sums, y in fp32.  A bf16 x bf16 product is exact in fp32; a bf16 x fp32
// product rounds once (relative 2^-24) before the compensated sum.
#include "spmv_warp.cuh"

namespace drb {
drb_status warp_launch_bf16(Csr &A, const void *x, void *y, bool x_f32, cudaStream_t s) {
  return x_f32 ? warpk::launch_typed<uint16_t, float, false, true>(A, x, y, nullptr, s)
               : warpk::launch_typed<uint16_t, uint16_t, false, true>(A, x, y, nullptr, s);
}
} // namespace drb
