// Launchers of the heavy kernel templates, each compiled in its own
// translation unit (oa_stats.cu, oa_gemm_simt.cu, oa_gemm_tc.cu).
#pragma once
#include "oa_common.cuh"

namespace oa {
struct StatsArgs;
struct LeanArgs;
struct SchurArgs;
cudaError_t oa_launch_snp_stats(int R, int LP, const StatsArgs& A, int grid, size_t smem, cudaStream_t st);
// spb: SNPs per CTA group, a power of two <= 8 / R; threads: 256 per CTA, or 512 with one column
// per group (R = 1, spb = 1, no in-kernel covariate projection)
cudaError_t oa_launch_snp_lean(int R, int spb, const LeanArgs& A, int grid, int threads, size_t smem,
                               cudaStream_t st);
// resident CTAs of k_snp_lean per SM for this shared-memory size and thread count (0 on error)
int oa_lean_ctas_per_sm(int R, int spb, size_t smem, bool qx, int threads);
bool oa_lean_has_qx(int R, int spb);
cudaError_t oa_launch_schur(int R, const SchurArgs& S, cudaStream_t st);
// pre-GEMM C[col * ldc + row] = sum_k X[row][k] B[col][k], col < c2 (tensor-core and SIMT forms)
cudaError_t oa_launch_pre_tc(const __nv_bfloat16* Xhi, const __nv_bfloat16* Xlo, int xrows,
                             const __nv_bfloat16* Bhi, const __nv_bfloat16* Blo, int c2, int n_pad, float* C, int ldc,
                             int* err, cudaStream_t st);
// cpart (c2 * ldc floats, or null): scratch for the second K half of a split product
cudaError_t oa_launch_pre_simt(const float* X, size_t ldx, int xrows, const float* B, size_t ldb, int c2, int K,
                               const float* colmean, const int* has_nan, int center, float* C, int ldc, float* cpart,
                               cudaStream_t st);
// center: dosages taken relative to colmean (NaN -> 0); else NaN -> colmean
cudaError_t oa_launch_gemm_simt(int R, const float* X, size_t ldx, int xrows, const float* Yt, size_t ldy, int t,
                                int K, const float* colmean, const int* has_nan, int center, const EpiArgs& E,
                                cudaStream_t st);
// variant: 1 = BK 32 x 4 stages, 2 = BK 64 x 2 stages, 3 = CTA pairs (2-SM MMA) BK 32 x 6, 4 = pairs BK 64 x 3;
// raster: 1 = trait tiles inner, 2 = SNP tiles inner
// Bound (ns of %globaltimer) of the pipeline waits of the tensor-core GEMMs and of the staging waits of the
// per-SNP statistics kernels on the current device (2 s by default); the drain waits keep 2 s
cudaError_t oa_set_wait_limit_tc(unsigned long long ns);
cudaError_t oa_set_wait_limit_stats(unsigned long long ns);
cudaError_t oa_launch_gemm_tc(int R, int variant, int raster, const __nv_bfloat16* Xhi, const __nv_bfloat16* Xlo,
                              int xrows, const __nv_bfloat16* Yhi, const __nv_bfloat16* Ylo, int t, int n_pad,
                              const EpiArgs& E, int* err, cudaStream_t st);
// Fused-operand forms: X read as FP32 (columns of ldx floats, n of them valid; ldx * 4 and X 16-byte aligned)
// and split into BF16 hi / lo in shared memory, each value taken as NaN -> fill, else x - shift, with
// shift = center ? colmean : 0 and fill = center ? 0 : colmean per row (fill only when *has_nan != 0).  oa_gemm_tc_fusable: the pipeline
// variant and trait count have a fused form (at most 128 traits, or CTA pairs); the pre-GEMM's fused form
// takes at most 128 columns.
bool oa_gemm_tc_fusable(int variant, int t);
cudaError_t oa_launch_gemm_tcf(int R, int raster, const float* X, size_t ldx, int n, int xrows, const float* colmean,
                               const int* has_nan, int center, const __nv_bfloat16* Yhi, const __nv_bfloat16* Ylo, int t, int n_pad,
                               const EpiArgs& E, int* err, cudaStream_t st);
cudaError_t oa_launch_pre_tcf(const float* X, size_t ldx, int n, int xrows, const float* colmean, const int* has_nan,
                              int center,
                              const __nv_bfloat16* Bhi, const __nv_bfloat16* Blo, int c2, int n_pad, float* C, int ldc,
                              int* err, cudaStream_t st);
}  // namespace oa
