// spmv_warp_f64.cu -- instantiates the persistent SpMV for double storage
// (plain and with the fused residual).
#include "spmv_warp.cuh"

namespace drb {
drb_status warp_launch_f64(Csr &A, const void *x, void *y, const warpk::WarpResid *ra,
                           cudaStream_t s) {
  if (ra)
    return warpk::launch_typed<double, double, true, false>(A, x, y, ra, s);
  return warpk::launch_typed<double, double, false, false>(A, x, y, nullptr, s);
}
} // namespace drb
