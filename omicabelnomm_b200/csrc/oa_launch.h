// Launchers of the heavy kernel templates, each compiled in its own
// translation unit (oa_stats.cu, oa_gemm_simt.cu, oa_gemm_tc.cu).
#pragma once
#include "oa_common.cuh"

namespace oa {
struct StatsArgs;
cudaError_t oa_launch_snp_stats(int R, int LP, const StatsArgs& A, int grid, size_t smem, cudaStream_t st);
cudaError_t oa_launch_gemm_simt(int R, const float* X, size_t ldx, int xrows, const float* Yt, size_t ldy, int t,
                                int K, const float* colmean, const int* has_nan, const EpiArgs& E, cudaStream_t st);
cudaError_t oa_launch_gemm_tc(int R, const __nv_bfloat16* Xhi, const __nv_bfloat16* Xlo, int xrows,
                              const __nv_bfloat16* Yhi, const __nv_bfloat16* Ylo, int t, int n_pad,
                              const EpiArgs& E, int* err, cudaStream_t st);
}  // namespace oa
