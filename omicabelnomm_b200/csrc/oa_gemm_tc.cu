// Mixed-precision XR'Y~ on tcgen05 tensor cores (BF16 hi/lo split, 3 products).
#include "oa_launch.h"

namespace oa {

cudaError_t oa_launch_gemm_tc(int R, const __nv_bfloat16* Xhi, const __nv_bfloat16* Xlo, int xrows,
                              const __nv_bfloat16* Yhi, const __nv_bfloat16* Ylo, int t, int n_pad,
                              const EpiArgs& E, cudaStream_t st) {
    (void)R; (void)Xhi; (void)Xlo; (void)xrows; (void)Yhi; (void)Ylo; (void)t; (void)n_pad; (void)E; (void)st;
    return cudaErrorNotSupported;
}

}  // namespace oa
