// Instantiations of the per-SNP statistics kernel (see oa_kernels.cuh).
#include "oa_stats.cuh"
#include "oa_launch.h"

namespace oa {

template <int R, int LP>
static cudaError_t go(const StatsArgs& A, int grid, size_t smem, cudaStream_t st) {
    // TMA bulk staging needs 16-byte aligned columns whose size is a multiple of 16 bytes
    const bool bulk = (A.n % 4 == 0) && (A.ldx % 4 == 0) && ((reinterpret_cast<uintptr_t>(A.X) & 15) == 0);
    // the opt-in shared-memory size is raised once per kernel and device (no
    // attribute call while a stream is being captured into a graph)
    static int set_bulk[64], set_plain[64];
    int dev = 0;
    cudaGetDevice(&dev);
    const int d = dev & 63;
    if (bulk) {
        if (set_bulk[d] < (int)smem) {
            cudaError_t e = cudaFuncSetAttribute(k_snp_stats<R, LP, true>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024 - 1024);
            if (e != cudaSuccess) return e;
            set_bulk[d] = 227 * 1024 - 1024;
        }
        k_snp_stats<R, LP, true><<<grid, OA_NTHREADS, smem, st>>>(A);
    } else {
        if (set_plain[d] < (int)smem) {
            cudaError_t e = cudaFuncSetAttribute(k_snp_stats<R, LP, false>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024 - 1024);
            if (e != cudaSuccess) return e;
            set_plain[d] = 227 * 1024 - 1024;
        }
        k_snp_stats<R, LP, false><<<grid, OA_NTHREADS, smem, st>>>(A);
    }
    return cudaGetLastError();
}

cudaError_t oa_launch_snp_stats(int R, int LP, const StatsArgs& A, int grid, size_t smem, cudaStream_t st) {
    switch (R * 100 + LP) {
        case 104: return go<1, 4>(A, grid, smem, st);
        case 108: return go<1, 8>(A, grid, smem, st);
        case 116: return go<1, 16>(A, grid, smem, st);
        case 204: return go<2, 4>(A, grid, smem, st);
        case 208: return go<2, 8>(A, grid, smem, st);
        case 216: return go<2, 16>(A, grid, smem, st);
        case 404: return go<4, 4>(A, grid, smem, st);
        case 408: return go<4, 8>(A, grid, smem, st);
        case 416: return go<4, 16>(A, grid, smem, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace oa
