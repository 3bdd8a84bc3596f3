// Instantiations of the FP32 SIMT GEMM with fused statistics (see oa_gemm_simt.cuh).
#include <algorithm>

#include "oa_gemm_simt.cuh"
#include "oa_launch.h"

namespace oa {

template <int R>
static cudaError_t go(const float* X, size_t ldx, int xrows, const float* Yt, size_t ldy, int t, int K,
                      const float* colmean, const int* has_nan, int center, const EpiArgs& E, cudaStream_t st) {
    dim3 grid((t + SG_BN - 1) / SG_BN, (xrows + SG_BM - 1) / SG_BM);
    const bool vec = (K % 4 == 0) && (ldx % 4 == 0) && (ldy % 4 == 0) &&
                     ((reinterpret_cast<uintptr_t>(X) & 15) == 0) && ((reinterpret_cast<uintptr_t>(Yt) & 15) == 0);
    if (vec)
        k_gemm_simt<R, true, false><<<grid, 256, 0, st>>>(X, ldx, xrows, Yt, ldy, t, K, colmean, has_nan, center,
                                                          E, nullptr, 0, nullptr, 0);
    else
        k_gemm_simt<R, false, false><<<grid, 256, 0, st>>>(X, ldx, xrows, Yt, ldy, t, K, colmean, has_nan, center,
                                                           E, nullptr, 0, nullptr, 0);
    return cudaGetLastError();
}

cudaError_t oa_launch_gemm_simt(int R, const float* X, size_t ldx, int xrows, const float* Yt, size_t ldy, int t,
                                int K, const float* colmean, const int* has_nan, int center, const EpiArgs& E,
                                cudaStream_t st) {
    switch (R) {
        case 1: return go<1>(X, ldx, xrows, Yt, ldy, t, K, colmean, has_nan, center, E, st);
        case 2: return go<2>(X, ldx, xrows, Yt, ldy, t, K, colmean, has_nan, center, E, st);
        case 4: return go<4>(X, ldx, xrows, Yt, ldy, t, K, colmean, has_nan, center, E, st);
        case 8: return go<8>(X, ldx, xrows, Yt, ldy, t, K, colmean, has_nan, center, E, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t oa_launch_pre_simt(const float* X, size_t ldx, int xrows, const float* B, size_t ldb, int c2, int K,
                               const float* colmean, const int* has_nan, int center, float* C, int ldc,
                               float* cpart, cudaStream_t st) {
    // a thin product (c2 columns: one tile column) has one CTA per 128 rows; with cpart the K range is
    // split in two halves (grid z) so that two CTAs share each SM's issue slots, and the halves are
    // summed afterwards in a fixed order
    const int kspan = cpart ? (((K + 1) / 2 + SG_BK - 1) / SG_BK) * SG_BK : 0;
    dim3 grid((c2 + SG_BN - 1) / SG_BN, (xrows + SG_BM - 1) / SG_BM, cpart ? 2 : 1);
    const bool vec = (K % 4 == 0) && (ldx % 4 == 0) && (ldb % 4 == 0) &&
                     ((reinterpret_cast<uintptr_t>(X) & 15) == 0) && ((reinterpret_cast<uintptr_t>(B) & 15) == 0);
    const EpiArgs none{};
    if (vec)
        k_gemm_simt<1, true, true><<<grid, 256, 0, st>>>(X, ldx, xrows, B, ldb, c2, K, colmean, has_nan, center, none,
                                                         C, ldc, cpart, kspan);
    else
        k_gemm_simt<1, false, true><<<grid, 256, 0, st>>>(X, ldx, xrows, B, ldb, c2, K, colmean, has_nan, center,
                                                          none, C, ldc, cpart, kspan);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !cpart) return e;
    const long long n = (long long)c2 * xrows;
    k_add_partial<<<(unsigned)std::min<long long>((n + 255) / 256, 4096), 256, 0, st>>>(C, cpart, c2, xrows, ldc);
    return cudaGetLastError();
}

}  // namespace oa
