// spmv_warp_f32.cu -- instantiates the persistent SpMV for float storage
// (plain, two-sum compensated, and with the fused residual).
#include "spmv_warp.cuh"

namespace drb {
drb_status warp_launch_f32(Csr &A, const void *x, void *y, const warpk::WarpResid *ra,
                           bool comp, cudaStream_t s) {
  if (ra)
    return warpk::launch_typed<float, float, true, false>(A, x, y, ra, s);
  return comp ? warpk::launch_typed<float, float, false, true>(A, x, y, nullptr, s)
              : warpk::launch_typed<float, float, false, false>(A, x, y, nullptr, s);
}
} // namespace drb
