// Instantiations of the per-SNP statistics kernels (oa_stats.cuh, oa_lean.cuh).
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include "oa_lean.cuh"
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

template <int R, int SPB, bool QX, int NT = 256>
static cudaError_t go_lean(const LeanArgs& A, int grid, size_t smem, cudaStream_t st) {
    const bool bulk = !A.xrows && (A.n % 4 == 0) && (A.ldx % 4 == 0) &&
                      ((reinterpret_cast<uintptr_t>(A.X) & 15) == 0);
    static int set_bulk[64], set_plain[64];
    int dev = 0;
    cudaGetDevice(&dev);
    const int d = dev & 63;
    int* done = bulk ? set_bulk : set_plain;
    if (done[d] < (int)smem) {
        cudaError_t e = bulk ? cudaFuncSetAttribute(k_snp_lean<R, SPB, true, QX, NT>,
                                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024 - 1024)
                             : cudaFuncSetAttribute(k_snp_lean<R, SPB, false, QX, NT>,
                                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024 - 1024);
        if (e != cudaSuccess) return e;
        done[d] = 227 * 1024 - 1024;
    }
    if (bulk)
        k_snp_lean<R, SPB, true, QX, NT><<<grid, NT, smem, st>>>(A);
    else
        k_snp_lean<R, SPB, false, QX, NT><<<grid, NT, smem, st>>>(A);
    return cudaGetLastError();
}

template <int R, int SPB, bool QX, int NT = 256>
static int lean_occ(size_t smem) {
    int nb = 0;
    if (cudaFuncSetAttribute(k_snp_lean<R, SPB, true, QX, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             227 * 1024 - 1024) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_snp_lean<R, SPB, true, QX, NT>, NT, smem) !=
            cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return nb;
}

// The qx kernels (all-rows covariate projection summed in the kernel) exist for groups of at most
// LEAN_QX_NC columns with two or more columns per SNP.
bool oa_lean_has_qx(int R, int spb) { return R >= 2 && R * spb <= LEAN_QX_NC; }

int oa_lean_ctas_per_sm(int R, int spb, size_t smem, bool qx, int threads) {
    // cached per (device, R, spb, qx, smem, threads): no runtime calls while a stream is captured
    static std::map<std::tuple<int, int, int, bool, size_t, int>, int> cache;
    static std::mutex mu;
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_tuple(dev, R, spb, qx, smem, threads);
    {
        std::lock_guard<std::mutex> g(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    int v = 0;
    if (threads == LEAN_MAX_THREADS) {
        v = (R == 1 && spb == 1 && !qx) ? lean_occ<1, 1, false, LEAN_MAX_THREADS>(smem) : 0;
    } else if (qx) {
        switch (R * 100 + spb) {
            case 201: v = lean_occ<2, 1, true>(smem); break;
            case 202: v = lean_occ<2, 2, true>(smem); break;
            case 401: v = lean_occ<4, 1, true>(smem); break;
            default: v = 0;
        }
    } else {
        switch (R * 100 + spb) {
            case 101: v = lean_occ<1, 1, false>(smem); break;
            case 102: v = lean_occ<1, 2, false>(smem); break;
            case 104: v = lean_occ<1, 4, false>(smem); break;
            case 108: v = lean_occ<1, 8, false>(smem); break;
            case 201: v = lean_occ<2, 1, false>(smem); break;
            case 202: v = lean_occ<2, 2, false>(smem); break;
            case 204: v = lean_occ<2, 4, false>(smem); break;
            case 401: v = lean_occ<4, 1, false>(smem); break;
            case 402: v = lean_occ<4, 2, false>(smem); break;
            case 801: v = lean_occ<8, 1, false>(smem); break;
            default: v = 0;
        }
    }
    std::lock_guard<std::mutex> g(mu);
    cache[key] = v;
    return v;
}

cudaError_t oa_launch_snp_lean(int R, int spb, const LeanArgs& A, int grid, int threads, size_t smem,
                               cudaStream_t st) {
    if (threads == LEAN_MAX_THREADS)
        return R == 1 && spb == 1 && !A.Afull ? go_lean<1, 1, false, LEAN_MAX_THREADS>(A, grid, smem, st)
                                              : cudaErrorInvalidValue;
    if (threads != 256) return cudaErrorInvalidValue;
    if (A.Afull) {
        switch (R * 100 + spb) {
            case 201: return go_lean<2, 1, true>(A, grid, smem, st);
            case 202: return go_lean<2, 2, true>(A, grid, smem, st);
            case 401: return go_lean<4, 1, true>(A, grid, smem, st);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (R * 100 + spb) {
        case 101: return go_lean<1, 1, false>(A, grid, smem, st);
        case 102: return go_lean<1, 2, false>(A, grid, smem, st);
        case 104: return go_lean<1, 4, false>(A, grid, smem, st);
        case 108: return go_lean<1, 8, false>(A, grid, smem, st);
        case 201: return go_lean<2, 1, false>(A, grid, smem, st);
        case 202: return go_lean<2, 2, false>(A, grid, smem, st);
        case 204: return go_lean<2, 4, false>(A, grid, smem, st);
        case 401: return go_lean<4, 1, false>(A, grid, smem, st);
        case 402: return go_lean<4, 2, false>(A, grid, smem, st);
        case 801: return go_lean<8, 1, false>(A, grid, smem, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t oa_set_wait_limit_stats(unsigned long long ns) {
    return cudaMemcpyToSymbol(c_st_wait_ns, &ns, sizeof ns);
}

cudaError_t oa_launch_schur(int R, const SchurArgs& S, cudaStream_t st) {
    const long long total = (long long)S.mb * (1 + S.G + S.Z);
    if (total <= 0) return cudaSuccess;
    // persistent: at most 8 resident CTAs of 256 threads per SM
    static int sms[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (!sms[dev & 63]) cudaDeviceGetAttribute(&sms[dev & 63], cudaDevAttrMultiProcessorCount, dev);
    const unsigned blocks = (unsigned)std::min<long long>((total + 255) / 256, 8LL * sms[dev & 63]);
    switch (R) {
        case 1: k_schur<1><<<blocks, 256, 0, st>>>(S); break;
        case 2: k_schur<2><<<blocks, 256, 0, st>>>(S); break;
        case 4: k_schur<4><<<blocks, 256, 0, st>>>(S); break;
        case 8: k_schur<8><<<blocks, 256, 0, st>>>(S); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace oa
