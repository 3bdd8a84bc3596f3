// Mixed-precision form of XR'Y~ (≙ the Ay_bot sgemm, src/Algorithm.cpp:705-707)
// on the 5th-generation tensor cores, with the per-test statistics fused
// into the epilogue.
//
// Each FP32 operand is split into BF16 hi + lo (x = hi + lo to ~2^-17
// relative) and the product is accumulated in FP32 TMEM as
//     C = Xhi Yhi' + Xhi Ylo' + Xlo Yhi'        (the lo*lo term, ~2^-18, is dropped)
//
// Persistent, warp-specialised kernel, one CTA per SM:
//   warp 0      TMA producer: 4 tiled loads per K-block (Xhi, Xlo, Yhi, Ylo),
//               128B-swizzled, completing on the stage's full barrier
//   warp 1      TMEM allocator and MMA issuer: 12 tcgen05.mma (kind::f16,
//               M=128, N=256, K=16) per 64-wide K-block, tcgen05.commit frees
//               the stage; a second commit hands the accumulator to the epilogue
//   warps 2..9  epilogue, two warps per TMEM lane group (32 rows), each
//               taking half of the tile's columns: tcgen05.ld of 8 columns
//               at a time, the statistics of epi_core in registers, a record
//               built only by the lanes that store one, block-reserved row
//               emission.  The epilogue of a tile must keep pace with the
//               main loop of the next; with one warp per lane group it
//               did not.
// Two 256-column accumulators (512 TMEM columns) let the epilogue of one
// tile overlap the main loop of the next.
//
// Every wait is bounded (2 s of %globaltimer); on a timeout the kernel sets
// a flag, stops issuing, waits for its own copies and MMAs in flight, frees
// its TMEM and returns.  The host turns the flag into an error.
#include <cuda.h>

#include <algorithm>

#include "oa_epilogue.cuh"
#include "oa_launch.h"

namespace oa {
namespace tc {

constexpr int BM = 128;
constexpr int EPI_WARPS = EPI_WARPS_TC;                  // two per TMEM lane group, half of the columns each
constexpr int NUM_THREADS = 64 + 32 * EPI_WARPS;         // 320
constexpr int EPI_COLS = 8;                              // accumulator columns per tcgen05.ld of the epilogue
// A-operand K-blocks prefetched into L2 ahead of the stage loads: 512 K-elements whatever the K-block
// width (16 blocks of 32, 8 of 64), so that the lines in flight (about 38 MB over 148 SMs) stay well
// inside L2 and are not evicted before their stage load reads them
template <int BK>
constexpr int pf_blocks() {
    return 512 / BK;
}
// Bound of the pipeline waits (2 s by default; oa_set_wait_limit_tc changes
// it for the device, which the timeout tests use to make the waits run out)
// and of the drain waits after an abort (own copies and MMAs in flight;
// never shortened).
__constant__ unsigned long long c_wait_ns = 2000000000ull;
constexpr unsigned long long DRAIN_NS = 2000000000ull;

// Pipeline shape: K-block width BK (64 -> 128-byte swizzle, 32 -> 64-byte
// swizzle), the number of shared-memory stages and the tile width BN.
template <int BK_, int STAGES_, int BN_ = 256>
struct Shape {
    static constexpr int BK = BK_, STAGES = STAGES_, BN = BN_;
    static constexpr int A_BYTES = BM * BK * 2;                     // one of hi / lo
    static constexpr int B_BYTES = BN * BK * 2;
    static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr size_t SMEM_BYTES = 1024 + (size_t)STAGES * STAGE_BYTES + (size_t)BN * sizeof(TraitP);
    static constexpr uint64_t LAYOUT = BK == 64 ? 2u : 4u;          // SWIZZLE_128B : SWIZZLE_64B
    static constexpr uint32_t SBO = BK == 64 ? 1024u : 512u;        // bytes between 8-row groups
    // two accumulators of BN FP32 columns (allocation: a power of two >= 32)
    static constexpr uint32_t TMEM_COLS = 2 * BN <= 128 ? 128u : (2 * BN <= 256 ? 256u : 512u);
    // instruction descriptor, kind::f16: D FP32 (bits 4-5 = 1), A and B BF16
    // (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at
    // bits 17-22, M >> 4 at bits 24-28
    static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                      ((uint32_t)(BM >> 4) << 24);
    static_assert(BN % 16 == 0 && BN >= 32 && BN <= 256, "UMMA N for M = 128");
};

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for the phase of parity `parity` to complete; false on abort/timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag) {
    if (mbar_try(b, parity)) return true;
    const unsigned long long t0 = gtimer(), lim = c_wait_ns;
    while (true) {
        if (mbar_try(b, parity)) return true;
        if (*abort_flag) return false;
        if (gtimer() - t0 > lim) {
            *abort_flag = 1;
            return false;
        }
    }
}
// Bounded wait that ignores the abort flag (draining work in flight).
__device__ __forceinline__ void mbar_drain(uint64_t* b, uint32_t parity) {
    const unsigned long long t0 = gtimer();
    while (!mbar_try(b, parity) && gtimer() - t0 < DRAIN_NS) {
    }
}

// L2 prefetch of one tile box (no shared memory, no barrier): the A operand
// streams from DRAM, and prefetching it well ahead of the stage loads keeps
// DRAM latency off the pipeline without more shared-memory stages.
__device__ __forceinline__ void tma_prefetch_2d(const CUtensorMap* map, int x, int y) {
    asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y)
                 : "memory");
}

__device__ __forceinline__ void tma_load_2d(const CUtensorMap* map, uint64_t* bar, void* dst, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            su32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(su32(bar)), "r"(x), "r"(y)
        : "memory");
}

// UMMA shared-memory descriptor, K-major swizzled operand: start address,
// leading byte offset 1 (ignored for swizzled K-major), stride byte offset
// = bytes between 8-row groups, version 1 (sm_100), layout type
// (2 = SWIZZLE_128B, 4 = SWIZZLE_64B).
template <class SH>
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;
    d |= (uint64_t)(SH::SBO >> 4) << 32;
    d |= (uint64_t)1u << 46;
    d |= SH::LAYOUT << 61;
    return d;
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Named barrier 1 of the epilogue warps, OR-reducing `flag` over them: every
// warp gets the same answer, so a decision to leave the tile loop (an abort
// seen by some warps and not yet by others) is taken by all of them together
// and none is left waiting at the next barrier.
__device__ __forceinline__ bool epi_bar_any(int flag) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.or.pred p, 1, %2, q;\n\tselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(r)
        : "r"(flag), "n"(EPI_WARPS * 32)
        : "memory");
    return r != 0;
}

// TMEM load of 8 accumulator columns without the wait; tmem_wait8 waits for
// it and hands the registers on (read-write operands, so that no use of them
// is scheduled before the wait).
__device__ __forceinline__ void tmem_ld8_async(uint32_t taddr, uint32_t (&v)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait8(uint32_t (&v)[8]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7])
                 :
                 : "memory");
}

// Statistics epilogue of one accumulator tile for one warp: lane = row
// (SNP column i of the block, `lead` on its first column), BN traits from
// TMEM at taddr (8 columns per tcgen05.ld, the next 8 loading while these are
// evaluated when PREFETCH), trait constants from tps.  FAST: no quirk terms,
// no dense outputs and no zero sets among the tile's traits (epi_decide).
template <int R, int BN, bool FAST, bool PREFETCH>
__device__ __forceinline__ void epi_columns(const EpiArgs& E, uint32_t taddr, int n0, int t, int lane, int i,
                                            bool lead, const float* vx, const TraitP* tps, int cb, int ce,
                                            Emitter& em) {
    int cg = -1;            // pattern whose Schur inverse is cached
    bool csing = true;
    double S[R * R];
    if (!(cb < ce && n0 + cb < t)) return;
    uint32_t v[EPI_COLS], vn[EPI_COLS];
    if constexpr (PREFETCH) {
        tmem_ld8_async(taddr + (uint32_t)cb, v);
        tmem_wait8(v);
    }
    for (int c0 = cb; c0 < ce && n0 + c0 < t; c0 += EPI_COLS) {
        const bool more = PREFETCH && c0 + EPI_COLS < ce && n0 + c0 + EPI_COLS < t;   // warp-uniform
        if constexpr (PREFETCH) {
            if (more) tmem_ld8_async(taddr + (uint32_t)(c0 + EPI_COLS), vn);
        } else {
            tmem_ld8(taddr + (uint32_t)c0, v);
        }
#pragma unroll
        for (int q = 0; q < EPI_COLS; ++q) {
            const int j = n0 + c0 + q;
            if (j >= t) break;   // warp-uniform
            const TraitP tp = tps[c0 + q];
            float z[R];
            if constexpr (R == 1) {
                z[0] = __uint_as_float(v[q]);
            } else {
#pragma unroll
                for (int a = 0; a < R; ++a)
                    z[a] = __shfl_sync(0xffffffffu, __uint_as_float(v[q]), (lane & ~(R - 1)) + a);
            }
            if (tp.g != cg) {    // traits are sorted by pattern: reloads are rare
                cg = tp.g;
                csing = lead ? !load_schur<R>(E, cg, i, S) : true;
            }
            EpiTest<R> o;
            bool st = false;
            if (lead) {
                if (csing) {
                    atomicAdd(E.n_singular, 1ull);
                    epi_dense_nan<R>(E, i, tp);
                } else {
                    st = epi_decide<R, FAST>(E, i, j, z, tp, S, vx, o);
                }
            }
            epi_emit_lazy<R>(E, st, em, [&](RecOf<R>* dst) { epi_write<R>(E, i, j, tp, o, dst); });
        }
        if constexpr (PREFETCH) {
            if (more) {
                tmem_wait8(vn);
#pragma unroll
                for (int q = 0; q < EPI_COLS; ++q) v[q] = vn[q];
            }
        }
    }
}

// The statistics epilogue of one tile for one warp.  With one or two columns
// per SNP a tile without quirk terms, dense outputs or zero sets takes the
// FAST evaluation; the split-copy forms also prefetch the next 8 TMEM columns
// (their register budget has room; the fused forms and r >= 4 do not).
template <int R, int BN, bool FUSED>
__device__ __forceinline__ void epi_tile(bool fast, const EpiArgs& E, uint32_t taddr, int n0, int t, int lane,
                                         int i, bool lead, const float* vx, const TraitP* tps, int cb, int ce,
                                         Emitter& em) {
    constexpr bool PF = !FUSED && R <= 2;
    if constexpr (R <= 2) {
        if (fast) {
            epi_columns<R, BN, true, PF>(E, taddr, n0, t, lane, i, lead, vx, tps, cb, ce, em);
            return;
        }
    }
    epi_columns<R, BN, false, PF>(E, taddr, n0, t, lane, i, lead, vx, tps, cb, ce, em);
}

// Trait constants of a tile's columns for the statistics epilogue (each
// epilogue thread loads its share), then one barrier of the epilogue warps
// that also tells whether any of the tile's traits has a zero set.
__device__ __forceinline__ bool epi_load_traits(const EpiArgs& E, TraitP* tps, int n0, int t, int et, int bn) {
    int zs = 0;
    for (int q = et; q < bn; q += EPI_WARPS * 32)
        if (n0 + q < t) {
            tps[q] = load_trait(E, n0 + q);
            zs |= tps[q].zs >= 0;
        }
    return epi_bar_any(zs);
}

// STORE = false: fused statistics epilogue (t = traits).  STORE = true: the
// FP32 product is written out transposed, C[col * ldc + row] (t = columns),
// for the pre-GEMM of the per-SNP covariate sums.
template <int R, class SH, bool STORE>
__global__ void __launch_bounds__(NUM_THREADS, 1)
k_gemm_tc(const __grid_constant__ CUtensorMap mAhi, const __grid_constant__ CUtensorMap mAlo,
          const __grid_constant__ CUtensorMap mBhi, const __grid_constant__ CUtensorMap mBlo, int xrows, int t,
          int nk, EpiArgs E, float* __restrict__ cout, int ldc, int raster, int* err) {
    constexpr int BK = SH::BK, STAGES = SH::STAGES, BN = SH::BN;
    constexpr uint32_t TMEM_COLS = SH::TMEM_COLS;
    constexpr int A_BYTES = SH::A_BYTES, B_BYTES = SH::B_BYTES, STAGE_BYTES = SH::STAGE_BYTES;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    TraitP* tps = reinterpret_cast<TraitP*>(smem + (size_t)STAGES * STAGE_BYTES);   // this tile's traits
    __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], acc_full[2], acc_empty[2], done_bar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ volatile int abort_sh;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m_tiles = (xrows + BM - 1) / BM, n_tiles = (t + BN - 1) / BN;
    const int ntiles = m_tiles * n_tiles;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], EPI_WARPS * 32);
        }
        mbar_init(&done_bar, 1);
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base_sh)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem_base = tmem_base_sh;

    auto stage_ptr = [&](int s, int which) -> uint8_t* {
        // which: 0 Ahi, 1 Alo, 2 Bhi, 3 Blo
        uint8_t* b = smem + (size_t)s * STAGE_BYTES;
        return which < 2 ? b + which * A_BYTES : b + 2 * A_BYTES + (which - 2) * B_BYTES;
    };

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer ----------------
            int s = 0;
            uint32_t ph = 0;
            uint32_t pend_par[STAGES];
            bool pend[STAGES];
            for (int q = 0; q < STAGES; ++q) pend[q] = false;
            bool ok = true;
            // L2 prefetch cursor, pf_blocks<BK>() K-blocks ahead of the stage loads (across tiles)
            int pt = blockIdx.x, pkb = 0;
            auto prefetch_next = [&]() {
                if (pt >= ntiles) return;
                const int pm0 = (raster == 2 ? pt % m_tiles : pt / n_tiles) * BM;
                tma_prefetch_2d(&mAhi, pkb * BK, pm0);
                tma_prefetch_2d(&mAlo, pkb * BK, pm0);
                if (++pkb == nk) {
                    pkb = 0;
                    pt += gridDim.x;
                }
            };
            for (int q = 0; q < pf_blocks<BK>(); ++q) prefetch_next();
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                const int m0 = (raster == 2 ? tile % m_tiles : tile / n_tiles) * BM;
                const int n0 = (raster == 2 ? tile / m_tiles : tile % n_tiles) * BN;
                for (int kb = 0; kb < nk; ++kb) {
                    if (!mbar_wait(&empty_bar[s], ph ^ 1u, &abort_sh)) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(&full_bar[s], STAGE_BYTES);
                    tma_load_2d(&mAhi, &full_bar[s], stage_ptr(s, 0), kb * BK, m0);
                    tma_load_2d(&mAlo, &full_bar[s], stage_ptr(s, 1), kb * BK, m0);
                    tma_load_2d(&mBhi, &full_bar[s], stage_ptr(s, 2), kb * BK, n0);
                    tma_load_2d(&mBlo, &full_bar[s], stage_ptr(s, 3), kb * BK, n0);
                    prefetch_next();
                    pend[s] = true;
                    pend_par[s] = ph;
                    if (++s == STAGES) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
            if (!ok)  // drain our own copies before the shared memory goes away
                for (int q = 0; q < STAGES; ++q)
                    if (pend[q]) mbar_drain(&full_bar[q], pend_par[q]);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer ----------------
            int s = 0, acc = 0;
            uint32_t ph = 0, aph = 0;
            bool ok = true, issued = false;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                if (!mbar_wait(&acc_empty[acc], aph ^ 1u, &abort_sh)) break;
                fence_after();
                const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
                for (int kb = 0; kb < nk; ++kb) {
                    if (!mbar_wait(&full_bar[s], ph, &abort_sh)) {
                        ok = false;
                        break;
                    }
                    fence_after();
                    const uint32_t ahi = su32(stage_ptr(s, 0)), alo = su32(stage_ptr(s, 1));
                    const uint32_t bhi = su32(stage_ptr(s, 2)), blo = su32(stage_ptr(s, 3));
#pragma unroll
                    for (int kk = 0; kk < BK / 16; ++kk) {
                        const uint32_t off = (uint32_t)kk * 32u;   // 16 BF16 along K inside the swizzled row
                        const uint64_t dah = smem_desc<SH>(ahi + off), dal = smem_desc<SH>(alo + off);
                        const uint64_t dbh = smem_desc<SH>(bhi + off), dbl = smem_desc<SH>(blo + off);
                        mma_bf16(d_tmem, dah, dbh, SH::IDESC, (kb > 0 || kk > 0) ? 1u : 0u);
                        mma_bf16(d_tmem, dah, dbl, SH::IDESC, 1u);
                        mma_bf16(d_tmem, dal, dbh, SH::IDESC, 1u);
                    }
                    issued = true;
                    mma_commit(&empty_bar[s]);
                    if (++s == STAGES) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok) break;
                mma_commit(&acc_full[acc]);
                if (++acc == 2) {
                    acc = 0;
                    aph ^= 1u;
                }
            }
            if (issued) {  // all MMAs of this CTA complete before TMEM is freed
                mma_commit(&done_bar);
                mbar_drain(&done_bar, 0);
            }
        }
    } else if constexpr (STORE) {
        // ---------------- store epilogue ----------------
        // lane = row of the tile: each tcgen05.ld column goes out as one
        // coalesced 128-byte row segment of the transposed output
        const int lg = warp & 3;
        const int cb = ((warp - 2) >> 2) * (BN / 2);   // this warp's half of the columns
        int acc = 0;
        uint32_t aph = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            if (abort_sh) break;
            const int m0 = (raster == 2 ? tile % m_tiles : tile / n_tiles) * BM;
            const int n0 = (raster == 2 ? tile / m_tiles : tile % n_tiles) * BN;
            int ok = 1;
            if (lane == 0) ok = mbar_wait(&acc_full[acc], aph, &abort_sh) ? 1 : 0;
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) break;
            mbar_try(&acc_full[acc], aph);
            fence_after();
            const int row = m0 + lg * 32 + lane;
            for (int c0 = cb; c0 < cb + BN / 2 && n0 + c0 < t; c0 += 32) {
                uint32_t v[32];
                tmem_ld32(tmem_base + ((uint32_t)(lg * 32) << 16) + (uint32_t)(acc * BN + c0), v);
                const int qmax = min(32, t - n0 - c0);
                if (row < xrows)
#pragma unroll
                    for (int q = 0; q < 32; ++q)
                        if (q < qmax) cout[(size_t)(n0 + c0 + q) * ldc + row] = __uint_as_float(v[q]);
            }
            fence_before();
            mbar_arrive(&acc_empty[acc]);
            if (++acc == 2) {
                acc = 0;
                aph ^= 1u;
            }
        }
    } else {
        // ---------------- epilogue ----------------
        // The epilogue threads synchronise among themselves with named
        // barrier 1; every decision that ends the loop is taken right after
        // it, so all of them leave together.  Two warps share each TMEM lane
        // group (32 rows), one per half of the tile's columns.
        const int ew = warp - 2;                 // 0..EPI_WARPS-1
        const int lg = warp & 3;                 // TMEM lane group this warp may access
        const int et = ew * 32 + lane;
        const int cb = (ew >> 2) * (BN / 2);
        Emitter em;
        int acc = 0;
        uint32_t aph = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            const int m0 = (raster == 2 ? tile % m_tiles : tile / n_tiles) * BM;
            const int n0 = (raster == 2 ? tile / m_tiles : tile % n_tiles) * BN;
            if (epi_bar_any(abort_sh)) break;   // previous tile's readers are done; one decision for all warps
            // trait constants of this tile (the main loop of the tile is still running)
            const bool tile_zs = epi_load_traits(E, tps, n0, t, et, BN);
            const int row = m0 + lg * 32 + lane;   // SNP column of this lane
            const bool lead = ((lane & (R - 1)) == 0) && (row < xrows);
            const int i = row / R;
            float vx[R];
#pragma unroll
            for (int a = 0; a < R; ++a) vx[a] = lead ? E.varx[(size_t)i * R + a] : 1.f;
            const bool fast = !E.qK && !E.d_r2 && !tile_zs;
            // accumulator ready (the wait is per warp: lane 0 waits, the warp follows)
            int ok = 1;
            if (lane == 0) ok = mbar_wait(&acc_full[acc], aph, &abort_sh) ? 1 : 0;
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (ok) {
                mbar_try(&acc_full[acc], aph);
                fence_after();
                epi_tile<R, BN, false>(fast, E, tmem_base + ((uint32_t)(lg * 32) << 16) + (uint32_t)(acc * BN), n0, t,
                                        lane, i, lead, vx, tps, cb, cb + BN / 2, em);
                fence_before();
                mbar_arrive(&acc_empty[acc]);
            }
            if (++acc == 2) {
                acc = 0;
                aph ^= 1u;
            }
        }
        epi_retire<R>(E, em);
    }

    fence_before();
    __syncthreads();
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
    }
    if (threadIdx.x == 0 && abort_sh) atomicExch(err, 1);
}

// ---------------------------------------------------------------------------
// 2-SM form of the statistics GEMM: a cluster of two CTAs on neighbouring SMs
// computes a 256 x 256 tile with tcgen05.mma.cta_group::2 (M = 256: each CTA
// holds 128 rows of A and of the accumulator; B is split along N, each CTA
// staging 128 of its 256 rows).  Per SM this stages a third fewer bytes for
// the same MMA work, so six 32-K stages fit where the 1-SM form has four.
//   * both CTAs' producers load their halves with cp.async.bulk.tensor
//     .cta_group::2 into their own shared memory; the bytes complete on the
//     leader CTA's full barrier, which expects both CTAs' bytes (no
//     multicast loads);
//   * the leader's MMA thread issues the MMAs and commits with
//     .multicast::cluster to both CTAs' empty / accumulator-full barriers;
//   * each CTA's epilogue reads its own TMEM rows and releases the
//     accumulator by arriving on the leader's accumulator-empty barrier.
// Every wait is bounded as in the 1-SM form.
// ---------------------------------------------------------------------------
template <int BK_, int STAGES_>
struct Shape2 {
    static constexpr int BK = BK_, STAGES = STAGES_, BN = 256;
    static constexpr int A_BYTES = BM * BK * 2;                     // this CTA's 128 rows, one of hi / lo
    static constexpr int B_BYTES = (BN / 2) * BK * 2;               // this CTA's half of B
    static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr size_t SMEM_BYTES = 1024 + (size_t)STAGES * STAGE_BYTES + (size_t)BN * sizeof(TraitP);
    static constexpr uint64_t LAYOUT = BK == 64 ? 2u : 4u;
    static constexpr uint32_t SBO = BK == 64 ? 1024u : 512u;
    static constexpr uint32_t TMEM_COLS = 512;
    // kind::f16, D FP32, A/B BF16, K-major, N = 256, M = 256 (the CTA pair)
    static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                      ((uint32_t)(256 >> 4) << 24);
};

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// shared::cluster address of the same shared variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t map_to_rank(const void* p, uint32_t rank) {
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(su32(p)), "r"(rank));
    return out;
}
__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void tma_load_2d_pair(const CUtensorMap* map, uint32_t bar_cluster, void* dst, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
        "%4}], [%2];" ::"r"(su32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar_cluster), "r"(x), "r"(y)
        : "memory");
}
__device__ __forceinline__ void mma_bf16_pair(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                              uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8, %9, %10, %11, %12}, p;\n}\n" ::"r"(
            d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u),
        "r"(0u));
}
// commit the leader's MMAs so far to the barrier at the same offset in both CTAs
__device__ __forceinline__ void mma_commit_pair(uint64_t* bar) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            su32(bar)),
        "h"((uint16_t)3)
        : "memory");
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t bar_cluster) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster) : "memory");
}

template <int R, class SH>
__global__ void __launch_bounds__(NUM_THREADS, 1)
k_gemm_tc2(const __grid_constant__ CUtensorMap mAhi, const __grid_constant__ CUtensorMap mAlo,
           const __grid_constant__ CUtensorMap mBhi, const __grid_constant__ CUtensorMap mBlo, int xrows, int t,
           int nk, EpiArgs E, int raster, int* err) {
    constexpr int BK = SH::BK, STAGES = SH::STAGES, BN = SH::BN;
    constexpr uint32_t TMEM_COLS = SH::TMEM_COLS;
    constexpr int A_BYTES = SH::A_BYTES, B_BYTES = SH::B_BYTES, STAGE_BYTES = SH::STAGE_BYTES;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    TraitP* tps = reinterpret_cast<TraitP*>(smem + (size_t)STAGES * STAGE_BYTES);
    __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], acc_full[2], acc_empty[2], done_bar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ volatile int abort_sh;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
    const int m_tiles = (xrows + 2 * BM - 1) / (2 * BM), n_tiles = (t + BN - 1) / BN;
    const int ntiles = m_tiles * n_tiles;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], 2 * EPI_WARPS);   // one arrival per epilogue warp of both CTAs (leader's copy)
        }
        mbar_init(&done_bar, 1);
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base_sh)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    cluster_sync();       // both CTAs' barriers and TMEM exist before any remote use
    fence_after();
    const uint32_t tmem_base = tmem_base_sh;

    auto stage_ptr = [&](int s, int which) -> uint8_t* {
        uint8_t* b = smem + (size_t)s * STAGE_BYTES;
        return which < 2 ? b + which * A_BYTES : b + 2 * A_BYTES + (which - 2) * B_BYTES;
    };
    auto tile_mn = [&](int tile, int& m0, int& n0) {
        m0 = (raster == 2 ? tile % m_tiles : tile / n_tiles) * 2 * BM;
        n0 = (raster == 2 ? tile / m_tiles : tile % n_tiles) * BN;
    };

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer (both CTAs) ----------------
            int s = 0;
            uint32_t ph = 0;
            bool ok = true;
            int pt = pair, pkb = 0;          // L2 prefetch cursor, pf_blocks<BK>() K-blocks ahead
            auto prefetch_next = [&]() {
                if (pt >= ntiles) return;
                int pm0, pn0;
                tile_mn(pt, pm0, pn0);
                tma_prefetch_2d(&mAhi, pkb * BK, pm0 + (int)rank * BM);
                tma_prefetch_2d(&mAlo, pkb * BK, pm0 + (int)rank * BM);
                if (++pkb == nk) {
                    pkb = 0;
                    pt += npairs;
                }
            };
            for (int q = 0; q < pf_blocks<BK>(); ++q) prefetch_next();
            for (int tile = pair; tile < ntiles && ok; tile += npairs) {
                int m0, n0;
                tile_mn(tile, m0, n0);
                const int ma = m0 + (int)rank * BM, nb = n0 + (int)rank * (BN / 2);
                for (int kb = 0; kb < nk; ++kb) {
                    if (!mbar_wait(&empty_bar[s], ph ^ 1u, &abort_sh)) {
                        ok = false;
                        break;
                    }
                    const uint32_t fb = map_to_rank(&full_bar[s], 0);
                    if (leader) mbar_expect_tx(&full_bar[s], 2 * STAGE_BYTES);
                    tma_load_2d_pair(&mAhi, fb, stage_ptr(s, 0), kb * BK, ma);
                    tma_load_2d_pair(&mAlo, fb, stage_ptr(s, 1), kb * BK, ma);
                    tma_load_2d_pair(&mBhi, fb, stage_ptr(s, 2), kb * BK, nb);
                    tma_load_2d_pair(&mBlo, fb, stage_ptr(s, 3), kb * BK, nb);
                    prefetch_next();
                    if (++s == STAGES) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
            if (!ok && leader)   // the leader's full barriers see both CTAs' copies: drain them
                for (int q = 0; q < STAGES; ++q) mbar_drain(&full_bar[q], 0), mbar_drain(&full_bar[q], 1);
        }
    } else if (warp == 1) {
        if (lane == 0 && leader) {
            // ---------------- MMA issuer (leader CTA) ----------------
            int s = 0, acc = 0;
            uint32_t ph = 0, aph = 0;
            bool ok = true, issued = false;
            for (int tile = pair; tile < ntiles && ok; tile += npairs) {
                if (!mbar_wait(&acc_empty[acc], aph ^ 1u, &abort_sh)) break;
                fence_after();
                const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
                for (int kb = 0; kb < nk; ++kb) {
                    if (!mbar_wait(&full_bar[s], ph, &abort_sh)) {
                        ok = false;
                        break;
                    }
                    fence_after();
                    const uint32_t ahi = su32(stage_ptr(s, 0)), alo = su32(stage_ptr(s, 1));
                    const uint32_t bhi = su32(stage_ptr(s, 2)), blo = su32(stage_ptr(s, 3));
#pragma unroll
                    for (int kk = 0; kk < BK / 16; ++kk) {
                        const uint32_t off = (uint32_t)kk * 32u;
                        const uint64_t dah = smem_desc<SH>(ahi + off), dal = smem_desc<SH>(alo + off);
                        const uint64_t dbh = smem_desc<SH>(bhi + off), dbl = smem_desc<SH>(blo + off);
                        mma_bf16_pair(d_tmem, dah, dbh, SH::IDESC, (kb > 0 || kk > 0) ? 1u : 0u);
                        mma_bf16_pair(d_tmem, dah, dbl, SH::IDESC, 1u);
                        mma_bf16_pair(d_tmem, dal, dbh, SH::IDESC, 1u);
                    }
                    issued = true;
                    mma_commit_pair(&empty_bar[s]);
                    if (++s == STAGES) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok) break;
                mma_commit_pair(&acc_full[acc]);
                if (++acc == 2) {
                    acc = 0;
                    aph ^= 1u;
                }
            }
            if (issued) mma_commit_pair(&done_bar);   // both CTAs learn when the last MMA has completed
        }
        if (lane == 0) mbar_drain(&done_bar, 0);      // (a CTA pair that issued nothing waits out the bound once)
    } else {
        // ---------------- epilogue (both CTAs, own 128 rows) ----------------
        const int ew = warp - 2;
        const int lg = warp & 3;
        const int et = ew * 32 + lane;
        const int cb = (ew >> 2) * (BN / 2);
        Emitter em;
        int acc = 0;
        uint32_t aph = 0;
        for (int tile = pair; tile < ntiles; tile += npairs) {
            int m0, n0;
            tile_mn(tile, m0, n0);
            m0 += (int)rank * BM;
            if (epi_bar_any(abort_sh)) break;
            const bool tile_zs = epi_load_traits(E, tps, n0, t, et, BN);
            const int row = m0 + lg * 32 + lane;
            const bool lead = ((lane & (R - 1)) == 0) && (row < xrows);
            const int i = row / R;
            float vx[R];
#pragma unroll
            for (int a = 0; a < R; ++a) vx[a] = lead ? E.varx[(size_t)i * R + a] : 1.f;
            const bool fast = !E.qK && !E.d_r2 && !tile_zs;
            int ok = 1;
            if (lane == 0) ok = mbar_wait(&acc_full[acc], aph, &abort_sh) ? 1 : 0;
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (ok) {
                mbar_try(&acc_full[acc], aph);
                fence_after();
                epi_tile<R, BN, false>(fast, E, tmem_base + ((uint32_t)(lg * 32) << 16) + (uint32_t)(acc * BN), n0, t,
                                        lane, i, lead, vx, tps, cb, cb + BN / 2, em);
                fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_cluster(map_to_rank(&acc_empty[acc], 0));
            }
            if (++acc == 2) {
                acc = 0;
                aph ^= 1u;
            }
        }
        epi_retire<R>(E, em);
    }

    fence_before();
    __syncthreads();
    cluster_sync();       // no CTA frees TMEM or leaves while its pair may still touch it
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
    }
    if (threadIdx.x == 0 && abort_sh) atomicExch(err, 1);
}

// ---------------------------------------------------------------------------
// Fused-operand forms: the X operand is read as FP32 (the SNP columns as the
// statistics kernel read them) and split into BF16 hi / lo in shared memory,
// so that no split copy of X is written to HBM or read back.
//
// The producer loads each K-block's FP32 A tile (the CTA's 128 rows x 64
// K-elements, 32 KB, rows at 256-byte strides) and B tiles (the traits' or
// the pre-GEMM columns' hi / lo, split once per trait block) into the
// K-block's stage, prefetching the FP32 tiles into L2 ahead of use as the
// split forms do; the stages' pipeline hides the load latency.  Converter
// warps then split the A tile in place.  The UMMA operands hi and lo are laid
// out as interleaved 8-row groups (K-major, 128-byte swizzle: the 16-byte
// chunk j of row r sits at chunk j ^ (r & 7) of its 128-byte row; hi of rows
// 8g..8g+7 at 2048 g, lo at 2048 g + 1024, descriptor stride 2048 bytes), so
// that the hi and lo of an 8-row group occupy exactly the 2 KB of its FP32
// rows: one warp reads a group, synchronises and writes it, with no barrier
// between warps.  Each value is formed as the statistics kernel's split
// forms it (NaN -> the column's fill value, else x - shift; shift = the
// column mean when the columns are centred, else 0; fill = 0 when centred,
// else the imputation mean) and split as hi = bf16(x), lo = bf16(x - hi):
// the results are bit-identical to the split path's.  K past n and rows past
// the last SNP column read as 0 (TMA fill); the K tail then holds -shift as
// in the split copy, against zero B rows.  The MMA issuer waits for the
// stage's bytes and for the converters.
// Warps: 0 producer, 1 MMA issuer, 2..9 epilogue, then the converters.
// Every wait is bounded as in the split forms; drains keep the 2 s bound.
// ---------------------------------------------------------------------------
// Converter warps: four with one or two columns per SNP, two with four or eight (the epilogue's
// registers bound the block: 448 threads leave 128 registers a thread, 384 leave 168)
template <int R>
constexpr int conv_warps() {
    return R <= 2 ? 4 : 2;
}
template <int R>
constexpr int threads_f() {
    return NUM_THREADS + 32 * conv_warps<R>();
}
// registers per thread of one resident CTA (a multiple of 8): the block's warps are spread
// over the SM's four sub-partitions of 16,384 registers each, so the sub-partition with the
// most warps (ceil(warps / 4)) bounds them: 128 at 448 threads (4 warps per sub-partition),
// 168 at 384 (3)
template <int R>
constexpr int regs_f() {
    return (16384 / (((threads_f<R>() / 32 + 3) / 4) * 32)) / 8 * 8;
}
static_assert(regs_f<1>() == 128 && regs_f<8>() == 168, "register caps of the fused forms");
constexpr int FBK = 64;     // K-block of the fused forms (128-byte swizzle)
constexpr int FGROUPS = BM / 8;   // 8-row groups of a CTA's A tile

template <int STAGES_, int BN_, bool PAIR>
struct ShapeF {
    static constexpr int BK = FBK, STAGES = STAGES_, BN = BN_;
    static constexpr int A_BYTES = BM * BK * 4;                         // FP32 tile = interleaved hi / lo groups
    static constexpr int B_ROWS = PAIR ? BN / 2 : BN;                   // this CTA's rows of B
    static constexpr int B_BYTES = B_ROWS * BK * 2;
    static constexpr int STAGE_BYTES = A_BYTES + 2 * B_BYTES;
    // stages, trait constants, per-row shift and fill
    static constexpr size_t SMEM_BYTES = 1024 + (size_t)STAGES * STAGE_BYTES + (size_t)BN * sizeof(TraitP) +
                                         2 * BM * sizeof(float);
    static constexpr uint64_t LAYOUT = 2u;                              // SWIZZLE_128B
    static constexpr uint32_t SBO = 1024u;                              // B: 8-row groups back to back
    static constexpr uint32_t SBO_A = 2048u;                            // A: hi and lo groups interleaved
    static constexpr uint32_t TMEM_COLS = PAIR ? 512u : (2 * BN <= 128 ? 128u : (2 * BN <= 256 ? 256u : 512u));
    static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                      ((uint32_t)((PAIR ? 256 : BM) >> 4) << 24);
    static_assert(SMEM_BYTES <= 227u * 1024u, "shared memory of the fused form");
};

// UMMA shared-memory descriptor with an explicit stride between 8-row groups
// (fields as in smem_desc).
__device__ __forceinline__ uint64_t smem_desc_sbo(uint32_t saddr, uint32_t sbo, uint64_t layout) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;
    d |= (uint64_t)(sbo >> 4) << 32;
    d |= (uint64_t)1u << 46;
    d |= layout << 61;
    return d;
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Cluster-scope acquire form of the bounded wait: the converters of both CTAs
// of a pair arrive (release, cluster scope) on the leader's barrier after
// writing their A tiles, which the leader's MMAs then read.
__device__ __forceinline__ bool mbar_try_cluster(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* b, uint32_t parity, volatile int* abort_flag) {
    if (mbar_try_cluster(b, parity)) return true;
    const unsigned long long t0 = gtimer(), lim = c_wait_ns;
    while (true) {
        if (mbar_try_cluster(b, parity)) return true;
        if (*abort_flag) return false;
        if (gtimer() - t0 > lim) {
            *abort_flag = 1;
            return false;
        }
    }
}

// In-place split of the 8-row groups g = wc, wc + NC, ... of one stage's A
// tile by converter warp wc (of NC).  Lane l takes the 16-byte chunk c = l %
// 16 of rows l / 16 + 2 u (u < 4) of a group: it reads the four FP32 chunks,
// the warp synchronises (the group's 2 KB are read), and it writes their hi
// and lo halves.  The next group's chunks are read before this group's are
// written (another 2 KB).
template <int NC, bool WITH_NAN>
__device__ __forceinline__ void convert_stage(uint8_t* a, const float* __restrict__ shift,
                                              const float* __restrict__ fill, int wc, int lane) {
    constexpr int G = FGROUPS / NC;   // groups per warp: 4 or 8
    const int c = lane & 15, r0 = lane >> 4;
    const uint32_t cin = (uint32_t)lane * 16u;   // byte offset of the lane's first chunk in a group
    float4 cur[4], nxt[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) cur[u] = *reinterpret_cast<const float4*>(a + wc * 2048 + cin + u * 512);
#pragma unroll
    for (int gi = 0; gi < G; ++gi) {
        const int g = wc + gi * NC;
        uint8_t* grp = a + g * 2048;
        if (gi + 1 < G) {
#pragma unroll
            for (int u = 0; u < 4; ++u) nxt[u] = *reinterpret_cast<const float4*>(grp + NC * 2048 + cin + u * 512);
        }
        uint2 hv[4], lv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int row = g * 8 + r0 + 2 * u;
            const float sh = shift[row];
            const float4 v = cur[u];
            float e0 = v.x - sh, e1 = v.y - sh, e2 = v.z - sh, e3 = v.w - sh;
            if constexpr (WITH_NAN) {
                const float fl = fill[row];
                e0 = isnan(v.x) ? fl : e0;
                e1 = isnan(v.y) ? fl : e1;
                e2 = isnan(v.z) ? fl : e2;
                e3 = isnan(v.w) ? fl : e3;
            }
            const __nv_bfloat162 h01 = __floats2bfloat162_rn(e0, e1), h23 = __floats2bfloat162_rn(e2, e3);
            const float2 f01 = __bfloat1622float2(h01), f23 = __bfloat1622float2(h23);
            const __nv_bfloat162 l01 = __floats2bfloat162_rn(e0 - f01.x, e1 - f01.y);
            const __nv_bfloat162 l23 = __floats2bfloat162_rn(e2 - f23.x, e3 - f23.y);
            hv[u] = make_uint2(*reinterpret_cast<const uint32_t*>(&h01), *reinterpret_cast<const uint32_t*>(&h23));
            lv[u] = make_uint2(*reinterpret_cast<const uint32_t*>(&l01), *reinterpret_cast<const uint32_t*>(&l23));
        }
        __syncwarp();   // every lane has read this group's FP32 chunks
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t rr = (uint32_t)(r0 + 2 * u);
            const uint32_t off = rr * 128u + ((((uint32_t)c >> 1) ^ rr) << 4) + (((uint32_t)c & 1u) << 3);
            *reinterpret_cast<uint2*>(grp + off) = hv[u];
            *reinterpret_cast<uint2*>(grp + 1024 + off) = lv[u];
        }
        if (gi + 1 < G) {
#pragma unroll
            for (int u = 0; u < 4; ++u) cur[u] = nxt[u];
        }
    }
}

// Converter loop shared by the fused forms: for each tile of this CTA and
// K-block in order, wait until the stage's FP32 A tile has landed (`full`,
// this CTA's barrier), split this warp's groups in place and arrive on the
// stage's convert barrier (`arrive(s)`).  tile_rows(tile) gives the CTA's
// first row of a tile.  Each warp keeps the shift and fill of its own rows;
// warps wait, leave and arrive independently.
template <int NC, class TileRows, class Arrive>
__device__ __forceinline__ void run_converters(const float* __restrict__ colmean, const int* __restrict__ has_nan,
                                               int center, int xrows, int first_tile, int tile_step, int ntiles,
                                               int nk, int stages, int stage_bytes, uint8_t* smem, uint64_t* full,
                                               float* shift, float* fill, volatile int* abort_sh,
                                               TileRows&& tile_rows, Arrive&& arrive) {
    const int lane = threadIdx.x & 31;
    const int wc = (int)(threadIdx.x >> 5) - (2 + EPI_WARPS);
    const bool any_nan = *has_nan != 0;   // written by the statistics kernel before this launch
    int s = 0;
    uint32_t ph = 0;
    for (int tile = first_tile; tile < ntiles; tile += tile_step) {
        const int r0 = tile_rows(tile);
        __syncwarp();   // this warp's reads of the previous tile's shift / fill are done
        for (int q = lane; q < 8 * FGROUPS / NC; q += 32) {   // this warp's rows: groups wc + NC i
            const int row = (wc + NC * (q >> 3)) * 8 + (q & 7);
            const float mu = r0 + row < xrows ? colmean[r0 + row] : 0.f;
            shift[row] = center ? mu : 0.f;
            fill[row] = center ? 0.f : mu;
        }
        __syncwarp();
        for (int kb = 0; kb < nk; ++kb) {
            int ok = 1;
            if (lane == 0) ok = mbar_wait(&full[s], ph, abort_sh) ? 1 : 0;
            if (!__shfl_sync(0xffffffffu, ok, 0)) return;
            mbar_try(&full[s], ph);   // this lane's own acquire of the completed phase
            uint8_t* a = smem + (size_t)s * stage_bytes;
            if (any_nan)
                convert_stage<NC, true>(a, shift, fill, wc, lane);
            else
                convert_stage<NC, false>(a, shift, fill, wc, lane);
            fence_proxy_async_smem();   // the stores reach the tensor cores' (async) view
            __syncwarp();
            if (lane == 0) arrive(s);
            if (++s == stages) {
                s = 0;
                ph ^= 1u;
            }
        }
    }
}

// 1-SM fused form.  STORE = false: statistics epilogue (t = traits); STORE =
// true: the FP32 product is written transposed, C[col * ldc + row] (the
// pre-GEMM of the per-SNP covariate sums, t = its columns).
template <int R, class SH, bool STORE>
__global__ void __launch_bounds__(threads_f<R>()) __maxnreg__(regs_f<R>())
k_gemm_tcf(const __grid_constant__ CUtensorMap mAf, const __grid_constant__ CUtensorMap mBhi,
           const __grid_constant__ CUtensorMap mBlo, const float* __restrict__ colmean,
           const int* __restrict__ has_nan, int center, int xrows, int t, int nk, EpiArgs E,
           float* __restrict__ cout, int ldc, int raster, int* err) {
    constexpr int NC = conv_warps<R>();
    constexpr int BK = SH::BK, STAGES = SH::STAGES, BN = SH::BN;
    constexpr uint32_t TMEM_COLS = SH::TMEM_COLS;
    constexpr int A_BYTES = SH::A_BYTES, B_BYTES = SH::B_BYTES, STAGE_BYTES = SH::STAGE_BYTES;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    TraitP* tps = reinterpret_cast<TraitP*>(smem + (size_t)STAGES * STAGE_BYTES);
    float* shift = reinterpret_cast<float*>(tps + BN);
    float* fill = shift + BM;
    __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], conv_bar_s[STAGES], acc_full[2],
        acc_empty[2], done_bar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ volatile int abort_sh;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m_tiles = (xrows + BM - 1) / BM, n_tiles = (t + BN - 1) / BN;
    const int ntiles = m_tiles * n_tiles;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
            mbar_init(&conv_bar_s[s], NC);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], EPI_WARPS * 32);
        }
        mbar_init(&done_bar, 1);
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base_sh)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem_base = tmem_base_sh;

    auto stage_ptr = [&](int s, int which) -> uint8_t* {   // 0 A (FP32, then hi / lo groups), 2 Bhi, 3 Blo
        uint8_t* b = smem + (size_t)s * STAGE_BYTES;
        return which < 2 ? b : b + A_BYTES + (which - 2) * B_BYTES;
    };
    auto tile_mn = [&](int tile, int& m0, int& n0) {
        m0 = (raster == 2 ? tile % m_tiles : tile / n_tiles) * BM;
        n0 = (raster == 2 ? tile / m_tiles : tile % n_tiles) * BN;
    };

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer ----------------
            int s = 0;
            uint32_t ph = 0;
            uint32_t pend_par[STAGES];
            bool pend[STAGES];
            for (int q = 0; q < STAGES; ++q) pend[q] = false;
            bool ok = true;
            int pt = blockIdx.x, pkb = 0;
            auto prefetch_next = [&]() {
                if (pt >= ntiles) return;
                int pm0, pn0;
                tile_mn(pt, pm0, pn0);
                tma_prefetch_2d(&mAf, pkb * BK, pm0);
                if (++pkb == nk) {
                    pkb = 0;
                    pt += gridDim.x;
                }
            };
            for (int q = 0; q < pf_blocks<BK>(); ++q) prefetch_next();
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                int m0, n0;
                tile_mn(tile, m0, n0);
                for (int kb = 0; kb < nk; ++kb) {
                    if (!mbar_wait(&empty_bar[s], ph ^ 1u, &abort_sh)) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(&full_bar[s], A_BYTES + 2 * B_BYTES);
                    tma_load_2d(&mAf, &full_bar[s], stage_ptr(s, 0), kb * BK, m0);
                    tma_load_2d(&mBhi, &full_bar[s], stage_ptr(s, 2), kb * BK, n0);
                    tma_load_2d(&mBlo, &full_bar[s], stage_ptr(s, 3), kb * BK, n0);
                    pend[s] = true;
                    pend_par[s] = ph;
                    prefetch_next();
                    if (++s == STAGES) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
            if (!ok) {   // drain our own copies before the shared memory goes away
                for (int q = 0; q < STAGES; ++q)
                    if (pend[q]) mbar_drain(&full_bar[q], pend_par[q]);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer ----------------
            int s = 0, acc = 0;
            uint32_t ph = 0, aph = 0;
            bool ok = true, issued = false;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                if (!mbar_wait(&acc_empty[acc], aph ^ 1u, &abort_sh)) break;
                fence_after();
                const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
                for (int kb = 0; kb < nk; ++kb) {
                    if (!mbar_wait(&full_bar[s], ph, &abort_sh) || !mbar_wait(&conv_bar_s[s], ph, &abort_sh)) {
                        ok = false;
                        break;
                    }
                    fence_after();
                    const uint32_t ahi = su32(stage_ptr(s, 0)), alo = ahi + 1024u;
                    const uint32_t bhi = su32(stage_ptr(s, 2)), blo = su32(stage_ptr(s, 3));
#pragma unroll
                    for (int kk = 0; kk < BK / 16; ++kk) {
                        const uint32_t off = (uint32_t)kk * 32u;
                        const uint64_t dah = smem_desc_sbo(ahi + off, SH::SBO_A, SH::LAYOUT);
                        const uint64_t dal = smem_desc_sbo(alo + off, SH::SBO_A, SH::LAYOUT);
                        const uint64_t dbh = smem_desc<SH>(bhi + off), dbl = smem_desc<SH>(blo + off);
                        mma_bf16(d_tmem, dah, dbh, SH::IDESC, (kb > 0 || kk > 0) ? 1u : 0u);
                        mma_bf16(d_tmem, dah, dbl, SH::IDESC, 1u);
                        mma_bf16(d_tmem, dal, dbh, SH::IDESC, 1u);
                    }
                    issued = true;
                    mma_commit(&empty_bar[s]);
                    if (++s == STAGES) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok) break;
                mma_commit(&acc_full[acc]);
                if (++acc == 2) {
                    acc = 0;
                    aph ^= 1u;
                }
            }
            if (issued) {   // all MMAs of this CTA complete before TMEM is freed
                mma_commit(&done_bar);
                mbar_drain(&done_bar, 0);
            }
        }
    } else if (warp >= 2 + EPI_WARPS) {
        // ---------------- converters ----------------
        run_converters<NC>(
            colmean, has_nan, center, xrows, blockIdx.x, gridDim.x, ntiles, nk, STAGES, STAGE_BYTES, smem, full_bar,
            shift, fill, &abort_sh,
            [&](int tile) {
                int m0, n0;
                tile_mn(tile, m0, n0);
                return m0;
            },
            [&](int s) { mbar_arrive(&conv_bar_s[s]); });
    } else if constexpr (STORE) {
        // ---------------- store epilogue ----------------
        const int lg = warp & 3;
        const int cb = ((warp - 2) >> 2) * (BN / 2);
        int acc = 0;
        uint32_t aph = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            if (epi_bar_any(abort_sh)) break;
            int m0, n0;
            tile_mn(tile, m0, n0);
            int ok = 1;
            if (lane == 0) ok = mbar_wait(&acc_full[acc], aph, &abort_sh) ? 1 : 0;
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (ok) {
                mbar_try(&acc_full[acc], aph);
                fence_after();
                const int row = m0 + lg * 32 + lane;
                for (int c0 = cb; c0 < cb + BN / 2 && n0 + c0 < t; c0 += 32) {
                    uint32_t v[32];
                    tmem_ld32(tmem_base + ((uint32_t)(lg * 32) << 16) + (uint32_t)(acc * BN + c0), v);
                    const int qmax = min(32, t - n0 - c0);
                    if (row < xrows)
#pragma unroll
                        for (int q = 0; q < 32; ++q)
                            if (q < qmax) cout[(size_t)(n0 + c0 + q) * ldc + row] = __uint_as_float(v[q]);
                }
                fence_before();
                mbar_arrive(&acc_empty[acc]);
            }
            if (++acc == 2) {
                acc = 0;
                aph ^= 1u;
            }
        }
    } else {
        // ---------------- statistics epilogue ----------------
        const int ew = warp - 2;
        const int lg = warp & 3;
        const int et = ew * 32 + lane;
        const int cb = (ew >> 2) * (BN / 2);
        Emitter em;
        int acc = 0;
        uint32_t aph = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            int m0, n0;
            tile_mn(tile, m0, n0);
            if (epi_bar_any(abort_sh)) break;
            const bool tile_zs = epi_load_traits(E, tps, n0, t, et, BN);
            const int row = m0 + lg * 32 + lane;
            const bool lead = ((lane & (R - 1)) == 0) && (row < xrows);
            const int i = row / R;
            float vx[R];
#pragma unroll
            for (int a = 0; a < R; ++a) vx[a] = lead ? E.varx[(size_t)i * R + a] : 1.f;
            const bool fast = !E.qK && !E.d_r2 && !tile_zs;
            int ok = 1;
            if (lane == 0) ok = mbar_wait(&acc_full[acc], aph, &abort_sh) ? 1 : 0;
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (ok) {
                mbar_try(&acc_full[acc], aph);
                fence_after();
                epi_tile<R, BN, true>(fast, E, tmem_base + ((uint32_t)(lg * 32) << 16) + (uint32_t)(acc * BN), n0, t,
                                        lane, i, lead, vx, tps, cb, cb + BN / 2, em);
                fence_before();
                mbar_arrive(&acc_empty[acc]);
            }
            if (++acc == 2) {
                acc = 0;
                aph ^= 1u;
            }
        }
        epi_retire<R>(E, em);
    }

    fence_before();
    __syncthreads();
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
    }
    if (threadIdx.x == 0 && abort_sh) atomicExch(err, 1);
}

// CTA-pair fused form (statistics epilogue): as k_gemm_tc2, with each CTA's
// FP32 A rows loaded on its own barrier and split in place by its converter
// warps; the leader's MMA issuer waits for the B bytes of both CTAs (leader's
// B barrier) and for the converters of both CTAs (leader's convert barrier).
// The MMA commits reach the empty barriers of both CTAs, which each CTA's
// producer waits on.
template <int R, class SH>
__global__ void __launch_bounds__(threads_f<R>()) __maxnreg__(regs_f<R>())
k_gemm_tc2f(const __grid_constant__ CUtensorMap mAf, const __grid_constant__ CUtensorMap mBhi,
            const __grid_constant__ CUtensorMap mBlo, const float* __restrict__ colmean,
            const int* __restrict__ has_nan, int center, int xrows, int t, int nk, EpiArgs E, int raster, int* err) {
    constexpr int NC = conv_warps<R>();
    constexpr int BK = SH::BK, STAGES = SH::STAGES, BN = SH::BN;
    constexpr uint32_t TMEM_COLS = SH::TMEM_COLS;
    constexpr int A_BYTES = SH::A_BYTES, B_BYTES = SH::B_BYTES, STAGE_BYTES = SH::STAGE_BYTES;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    TraitP* tps = reinterpret_cast<TraitP*>(smem + (size_t)STAGES * STAGE_BYTES);
    float* shift = reinterpret_cast<float*>(tps + BN);
    float* fill = shift + BM;
    __shared__ __align__(8) uint64_t full_a[STAGES], full_b[STAGES], empty_bar[STAGES], conv_bar_s[STAGES],
        acc_full[2], acc_empty[2], done_bar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ volatile int abort_sh;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
    const int m_tiles = (xrows + 2 * BM - 1) / (2 * BM), n_tiles = (t + BN - 1) / BN;
    const int ntiles = m_tiles * n_tiles;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full_a[s], 1);
            mbar_init(&full_b[s], 1);
            mbar_init(&empty_bar[s], 1);
            mbar_init(&conv_bar_s[s], 2 * NC);   // leader's copy: the converter warps of both CTAs
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], 2 * EPI_WARPS);
        }
        mbar_init(&done_bar, 1);
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base_sh)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    cluster_sync();
    fence_after();
    const uint32_t tmem_base = tmem_base_sh;

    auto stage_ptr = [&](int s, int which) -> uint8_t* {
        uint8_t* b = smem + (size_t)s * STAGE_BYTES;
        return which < 2 ? b : b + A_BYTES + (which - 2) * B_BYTES;
    };
    auto tile_mn = [&](int tile, int& m0, int& n0) {
        m0 = (raster == 2 ? tile % m_tiles : tile / n_tiles) * 2 * BM;
        n0 = (raster == 2 ? tile / m_tiles : tile % n_tiles) * BN;
    };

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer (both CTAs) ----------------
            int s = 0;
            uint32_t ph = 0;
            uint32_t pend_par[STAGES];
            bool pend[STAGES];
            for (int q = 0; q < STAGES; ++q) pend[q] = false;
            bool ok = true;
            int pt = pair, pkb = 0;
            auto prefetch_next = [&]() {
                if (pt >= ntiles) return;
                int pm0, pn0;
                tile_mn(pt, pm0, pn0);
                tma_prefetch_2d(&mAf, pkb * BK, pm0 + (int)rank * BM);
                if (++pkb == nk) {
                    pkb = 0;
                    pt += npairs;
                }
            };
            for (int q = 0; q < pf_blocks<BK>(); ++q) prefetch_next();
            for (int tile = pair; tile < ntiles && ok; tile += npairs) {
                int m0, n0;
                tile_mn(tile, m0, n0);
                const int ma = m0 + (int)rank * BM, nb = n0 + (int)rank * (BN / 2);
                for (int kb = 0; kb < nk; ++kb) {
                    if (!mbar_wait(&empty_bar[s], ph ^ 1u, &abort_sh)) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(&full_a[s], A_BYTES);   // own FP32 rows, own barrier (the converters')
                    tma_load_2d(&mAf, &full_a[s], stage_ptr(s, 0), kb * BK, ma);
                    pend[s] = true;
                    pend_par[s] = ph;
                    const uint32_t fb = map_to_rank(&full_b[s], 0);
                    if (leader) mbar_expect_tx(&full_b[s], 2 * 2 * B_BYTES);
                    tma_load_2d_pair(&mBhi, fb, stage_ptr(s, 2), kb * BK, nb);
                    tma_load_2d_pair(&mBlo, fb, stage_ptr(s, 3), kb * BK, nb);
                    prefetch_next();
                    if (++s == STAGES) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
            if (!ok) {   // own FP32 copies; the leader's B barriers see both CTAs' B copies
                for (int q = 0; q < STAGES; ++q)
                    if (pend[q]) mbar_drain(&full_a[q], pend_par[q]);
                if (leader)
                    for (int q = 0; q < STAGES; ++q) mbar_drain(&full_b[q], 0), mbar_drain(&full_b[q], 1);
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && leader) {
            // ---------------- MMA issuer (leader CTA) ----------------
            int s = 0, acc = 0;
            uint32_t ph = 0, aph = 0;
            bool ok = true, issued = false;
            for (int tile = pair; tile < ntiles && ok; tile += npairs) {
                if (!mbar_wait(&acc_empty[acc], aph ^ 1u, &abort_sh)) break;
                fence_after();
                const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
                for (int kb = 0; kb < nk; ++kb) {
                    if (!mbar_wait(&full_b[s], ph, &abort_sh) || !mbar_wait_cluster(&conv_bar_s[s], ph, &abort_sh)) {
                        ok = false;
                        break;
                    }
                    fence_after();
                    const uint32_t ahi = su32(stage_ptr(s, 0)), alo = ahi + 1024u;
                    const uint32_t bhi = su32(stage_ptr(s, 2)), blo = su32(stage_ptr(s, 3));
#pragma unroll
                    for (int kk = 0; kk < BK / 16; ++kk) {
                        const uint32_t off = (uint32_t)kk * 32u;
                        const uint64_t dah = smem_desc_sbo(ahi + off, SH::SBO_A, SH::LAYOUT);
                        const uint64_t dal = smem_desc_sbo(alo + off, SH::SBO_A, SH::LAYOUT);
                        const uint64_t dbh = smem_desc<SH>(bhi + off), dbl = smem_desc<SH>(blo + off);
                        mma_bf16_pair(d_tmem, dah, dbh, SH::IDESC, (kb > 0 || kk > 0) ? 1u : 0u);
                        mma_bf16_pair(d_tmem, dah, dbl, SH::IDESC, 1u);
                        mma_bf16_pair(d_tmem, dal, dbh, SH::IDESC, 1u);
                    }
                    issued = true;
                    mma_commit_pair(&empty_bar[s]);
                    if (++s == STAGES) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok) break;
                mma_commit_pair(&acc_full[acc]);
                if (++acc == 2) {
                    acc = 0;
                    aph ^= 1u;
                }
            }
            if (issued) mma_commit_pair(&done_bar);   // both CTAs learn when the last MMA has completed
        }
        if (lane == 0) mbar_drain(&done_bar, 0);      // (a CTA pair that issued nothing waits out the bound once)
    } else if (warp >= 2 + EPI_WARPS) {
        // ---------------- converters (both CTAs, own 128 rows) ----------------
        run_converters<NC>(
            colmean, has_nan, center, xrows, pair, npairs, ntiles, nk, STAGES, STAGE_BYTES, smem, full_a, shift,
            fill, &abort_sh,
            [&](int tile) {
                int m0, n0;
                tile_mn(tile, m0, n0);
                return m0 + (int)rank * BM;
            },
            [&](int s) { mbar_arrive_cluster(map_to_rank(&conv_bar_s[s], 0)); });
    } else {
        // ---------------- epilogue (both CTAs, own 128 rows) ----------------
        const int ew = warp - 2;
        const int lg = warp & 3;
        const int et = ew * 32 + lane;
        const int cb = (ew >> 2) * (BN / 2);
        Emitter em;
        int acc = 0;
        uint32_t aph = 0;
        for (int tile = pair; tile < ntiles; tile += npairs) {
            int m0, n0;
            tile_mn(tile, m0, n0);
            m0 += (int)rank * BM;
            if (epi_bar_any(abort_sh)) break;
            const bool tile_zs = epi_load_traits(E, tps, n0, t, et, BN);
            const int row = m0 + lg * 32 + lane;
            const bool lead = ((lane & (R - 1)) == 0) && (row < xrows);
            const int i = row / R;
            float vx[R];
#pragma unroll
            for (int a = 0; a < R; ++a) vx[a] = lead ? E.varx[(size_t)i * R + a] : 1.f;
            const bool fast = !E.qK && !E.d_r2 && !tile_zs;
            int ok = 1;
            if (lane == 0) ok = mbar_wait(&acc_full[acc], aph, &abort_sh) ? 1 : 0;
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (ok) {
                mbar_try(&acc_full[acc], aph);
                fence_after();
                epi_tile<R, BN, true>(fast, E, tmem_base + ((uint32_t)(lg * 32) << 16) + (uint32_t)(acc * BN), n0, t,
                                        lane, i, lead, vx, tps, cb, cb + BN / 2, em);
                fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_cluster(map_to_rank(&acc_empty[acc], 0));
            }
            if (++acc == 2) {
                acc = 0;
                aph ^= 1u;
            }
        }
        epi_retire<R>(E, em);
    }

    fence_before();
    __syncthreads();
    cluster_sync();
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
    }
    if (threadIdx.x == 0 && abort_sh) atomicExch(err, 1);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// K-major BF16 matrix of `rows` rows and k_pad (multiple of 64) columns,
// boxes of bk x box_rows with the swizzle matching the UMMA descriptor.
static bool make_map(CUtensorMap* m, const __nv_bfloat16* ptr, int rows, int k_pad, int box_rows, int bk) {
    EncodeTiledFn fn = encode_fn();
    if (!fn || rows <= 0 || (k_pad % 64) != 0 || (reinterpret_cast<uintptr_t>(ptr) & 15) != 0) return false;
    const cuuint64_t gdim[2] = {(cuuint64_t)k_pad, (cuuint64_t)rows};
    const cuuint64_t gstride[1] = {(cuuint64_t)k_pad * 2};
    const cuuint32_t box[2] = {(cuuint32_t)bk, (cuuint32_t)box_rows};
    const cuuint32_t estride[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(ptr), gdim, gstride, box, estride,
              CU_TENSOR_MAP_INTERLEAVE_NONE, bk == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static int sm_count() {
    static int sms[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (!sms[dev & 63]) cudaDeviceGetAttribute(&sms[dev & 63], cudaDevAttrMultiProcessorCount, dev);
    return sms[dev & 63];
}

template <int R, class SH, bool STORE>
static cudaError_t go(const __nv_bfloat16* Xhi, const __nv_bfloat16* Xlo, int xrows, const __nv_bfloat16* Yhi,
                      const __nv_bfloat16* Ylo, int t, int n_pad, const EpiArgs& E, float* cout, int ldc, int raster,
                      int* err, cudaStream_t st) {
    constexpr int BN = SH::BN;
    CUtensorMap a_hi, a_lo, b_hi, b_lo;
    if (!make_map(&a_hi, Xhi, xrows, n_pad, BM, SH::BK) || !make_map(&a_lo, Xlo, xrows, n_pad, BM, SH::BK) ||
        !make_map(&b_hi, Yhi, t, n_pad, BN, SH::BK) || !make_map(&b_lo, Ylo, t, n_pad, BN, SH::BK))
        return cudaErrorInvalidValue;
    static int attr_done[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (!attr_done[dev & 63]) {   // once per device, never during a stream capture
        cudaError_t e = cudaFuncSetAttribute(k_gemm_tc<R, SH, STORE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)SH::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        attr_done[dev & 63] = 1;
    }
    const int ntiles = ((xrows + BM - 1) / BM) * ((t + BN - 1) / BN);
    const int sms = sm_count();
    const int grid = ntiles < sms ? ntiles : sms;
    k_gemm_tc<R, SH, STORE><<<grid, NUM_THREADS, SH::SMEM_BYTES, st>>>(a_hi, a_lo, b_hi, b_lo, xrows, t,
                                                                        n_pad / SH::BK, E, cout, ldc, raster, err);
    return cudaGetLastError();
}

template <int R, class SH>
static cudaError_t go2(const __nv_bfloat16* Xhi, const __nv_bfloat16* Xlo, int xrows, const __nv_bfloat16* Yhi,
                       const __nv_bfloat16* Ylo, int t, int n_pad, const EpiArgs& E, int raster, int* err,
                       cudaStream_t st) {
    CUtensorMap a_hi, a_lo, b_hi, b_lo;
    if (!make_map(&a_hi, Xhi, xrows, n_pad, BM, SH::BK) || !make_map(&a_lo, Xlo, xrows, n_pad, BM, SH::BK) ||
        !make_map(&b_hi, Yhi, t, n_pad, SH::BN / 2, SH::BK) || !make_map(&b_lo, Ylo, t, n_pad, SH::BN / 2, SH::BK))
        return cudaErrorInvalidValue;
    static int attr_done[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (!attr_done[dev & 63]) {   // once per device, never during a stream capture
        cudaError_t e = cudaFuncSetAttribute(k_gemm_tc2<R, SH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)SH::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        attr_done[dev & 63] = 1;
    }
    const int ntiles = ((xrows + 2 * BM - 1) / (2 * BM)) * ((t + SH::BN - 1) / SH::BN);
    const int pairs = std::min(ntiles, sm_count() / 2);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * pairs, 1, 1);
    cfg.blockDim = dim3(NUM_THREADS, 1, 1);
    cfg.dynamicSmemBytes = SH::SMEM_BYTES;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_gemm_tc2<R, SH>, a_hi, a_lo, b_hi, b_lo, xrows, t, n_pad / SH::BK, E, raster,
                              err);
}

// Pipeline variant: 1 = BK 32 x 4 stages, 2 = BK 64 x 2 stages, 3 = CTA pairs (2-SM MMA), BK 32 x 6 stages,
// 4 = CTA pairs, BK 64 x 3 stages (128-byte rows: half the TMA requests per byte).  Trait blocks of at most
// 128 traits take a narrower N tile (64 or 128 columns, more stages) whatever the variant: a 256-column tile
// would spend most of its MMA work on absent traits.
template <int R>
static cudaError_t go_any(int variant, int raster, const __nv_bfloat16* Xhi, const __nv_bfloat16* Xlo, int xrows,
                          const __nv_bfloat16* Yhi, const __nv_bfloat16* Ylo, int t, int n_pad, const EpiArgs& E,
                          int* err, cudaStream_t st) {
    if (t <= 64)
        return go<R, Shape<64, 4, 64>, false>(Xhi, Xlo, xrows, Yhi, Ylo, t, n_pad, E, nullptr, 0, raster, err, st);
    if (t <= 128)
        return go<R, Shape<64, 3, 128>, false>(Xhi, Xlo, xrows, Yhi, Ylo, t, n_pad, E, nullptr, 0, raster, err, st);
    if (variant == 2)
        return go<R, Shape<64, 2>, false>(Xhi, Xlo, xrows, Yhi, Ylo, t, n_pad, E, nullptr, 0, raster, err, st);
    if (variant == 3) return go2<R, Shape2<32, 6>>(Xhi, Xlo, xrows, Yhi, Ylo, t, n_pad, E, raster, err, st);
    if (variant == 4) return go2<R, Shape2<64, 3>>(Xhi, Xlo, xrows, Yhi, Ylo, t, n_pad, E, raster, err, st);
    return go<R, Shape<32, 4>, false>(Xhi, Xlo, xrows, Yhi, Ylo, t, n_pad, E, nullptr, 0, raster, err, st);
}


// FP32 K-major matrix of `rows` rows of ld floats (k_valid of them read, the
// rest of each 64-wide K-block and rows past `rows` filled with zeros), boxes
// of 64 x 128, no swizzle (rows at 256-byte strides, split in place by the
// converter warps); ld * 4 and k_valid * 4 must be 16-byte multiples and the
// base 16-byte aligned.
static bool make_map_f32(CUtensorMap* m, const float* ptr, int rows, int k_valid, size_t ld) {
    EncodeTiledFn fn = encode_fn();
    if (!fn || rows <= 0 || k_valid <= 0 || (k_valid % 4) != 0 || (ld % 4) != 0 ||
        (reinterpret_cast<uintptr_t>(ptr) & 15) != 0)
        return false;
    const cuuint64_t gdim[2] = {(cuuint64_t)k_valid, (cuuint64_t)rows};
    const cuuint64_t gstride[1] = {(cuuint64_t)ld * 4};
    const cuuint32_t box[2] = {(cuuint32_t)FBK, (cuuint32_t)BM};
    const cuuint32_t estride[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(ptr), gdim, gstride, box, estride,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int R, class SH, bool STORE>
static cudaError_t go_f(const float* X, size_t ldx, int n, int xrows, const float* colmean, const int* has_nan,
                        int center,
                        const __nv_bfloat16* Bhi, const __nv_bfloat16* Blo, int t, int n_pad, const EpiArgs& E,
                        float* cout, int ldc, int raster, int* err, cudaStream_t st) {
    constexpr int BN = SH::BN;
    CUtensorMap a_f, b_hi, b_lo;
    if (!make_map_f32(&a_f, X, xrows, n, ldx) || !make_map(&b_hi, Bhi, t, n_pad, BN, SH::BK) ||
        !make_map(&b_lo, Blo, t, n_pad, BN, SH::BK))
        return cudaErrorInvalidValue;
    static int attr_done[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (!attr_done[dev & 63]) {   // once per device, never during a stream capture
        cudaError_t e = cudaFuncSetAttribute(k_gemm_tcf<R, SH, STORE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)SH::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        attr_done[dev & 63] = 1;
    }
    const int ntiles = ((xrows + BM - 1) / BM) * ((t + BN - 1) / BN);
    const int sms = sm_count();
    const int grid = ntiles < sms ? ntiles : sms;
    k_gemm_tcf<R, SH, STORE><<<grid, threads_f<R>(), SH::SMEM_BYTES, st>>>(
        a_f, b_hi, b_lo, colmean, has_nan, center, xrows, t, n_pad / SH::BK, E, cout, ldc, raster, err);
    return cudaGetLastError();
}

template <int R, class SH>
static cudaError_t go2_f(const float* X, size_t ldx, int n, int xrows, const float* colmean, const int* has_nan,
                         int center,
                         const __nv_bfloat16* Yhi, const __nv_bfloat16* Ylo, int t, int n_pad, const EpiArgs& E,
                         int raster, int* err, cudaStream_t st) {
    CUtensorMap a_f, b_hi, b_lo;
    if (!make_map_f32(&a_f, X, xrows, n, ldx) || !make_map(&b_hi, Yhi, t, n_pad, SH::BN / 2, SH::BK) ||
        !make_map(&b_lo, Ylo, t, n_pad, SH::BN / 2, SH::BK))
        return cudaErrorInvalidValue;
    static int attr_done[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (!attr_done[dev & 63]) {
        cudaError_t e = cudaFuncSetAttribute(k_gemm_tc2f<R, SH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)SH::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        attr_done[dev & 63] = 1;
    }
    const int ntiles = ((xrows + 2 * BM - 1) / (2 * BM)) * ((t + SH::BN - 1) / SH::BN);
    const int pairs = std::min(ntiles, sm_count() / 2);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * pairs, 1, 1);
    cfg.blockDim = dim3(threads_f<R>(), 1, 1);
    cfg.dynamicSmemBytes = SH::SMEM_BYTES;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_gemm_tc2f<R, SH>, a_f, b_hi, b_lo, colmean, has_nan, center, xrows, t,
                              n_pad / SH::BK, E, raster, err);
}

// the stage counts of the split forms' tiles (Shape<64, 4, 64>, Shape<64, 3, 128>, Shape2<64, 3>)
using FNarrow64 = ShapeF<4, 64, false>;
using FNarrow128 = ShapeF<3, 128, false>;
using FPair = ShapeF<3, 256, true>;

// Fused forms of the statistics GEMM: trait blocks of at most 128 traits on
// the 1-SM narrow tiles, wider ones on CTA pairs (the fused pair form serves
// pipeline variants 3 and 4).
template <int R>
static cudaError_t go_any_f(int raster, const float* X, size_t ldx, int n, int xrows, const float* colmean,
                            const int* has_nan, int center,
                            const __nv_bfloat16* Yhi, const __nv_bfloat16* Ylo, int t, int n_pad, const EpiArgs& E,
                            int* err, cudaStream_t st) {
    if (t <= 64)
        return go_f<R, FNarrow64, false>(X, ldx, n, xrows, colmean, has_nan, center, Yhi, Ylo, t, n_pad, E, nullptr, 0, raster,
                                         err, st);
    if (t <= 128)
        return go_f<R, FNarrow128, false>(X, ldx, n, xrows, colmean, has_nan, center, Yhi, Ylo, t, n_pad, E, nullptr, 0,
                                          raster, err, st);
    return go2_f<R, FPair>(X, ldx, n, xrows, colmean, has_nan, center, Yhi, Ylo, t, n_pad, E, raster, err, st);
}

}  // namespace tc

cudaError_t oa_set_wait_limit_tc(unsigned long long ns) { return cudaMemcpyToSymbol(tc::c_wait_ns, &ns, sizeof ns); }

cudaError_t oa_launch_gemm_tc(int R, int variant, int raster, const __nv_bfloat16* Xhi, const __nv_bfloat16* Xlo,
                              int xrows, const __nv_bfloat16* Yhi, const __nv_bfloat16* Ylo, int t, int n_pad,
                              const EpiArgs& E, int* err, cudaStream_t st) {
    switch (R) {
        case 1: return tc::go_any<1>(variant, raster, Xhi, Xlo, xrows, Yhi, Ylo, t, n_pad, E, err, st);
        case 2: return tc::go_any<2>(variant, raster, Xhi, Xlo, xrows, Yhi, Ylo, t, n_pad, E, err, st);
        case 4: return tc::go_any<4>(variant, raster, Xhi, Xlo, xrows, Yhi, Ylo, t, n_pad, E, err, st);
        case 8: return tc::go_any<8>(variant, raster, Xhi, Xlo, xrows, Yhi, Ylo, t, n_pad, E, err, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t oa_launch_pre_tc(const __nv_bfloat16* Xhi, const __nv_bfloat16* Xlo, int xrows,
                             const __nv_bfloat16* Bhi, const __nv_bfloat16* Blo, int c2, int n_pad, float* C, int ldc,
                             int* err, cudaStream_t st) {
    const EpiArgs none{};
    if (c2 <= 64) return tc::go<1, tc::Shape<64, 4, 64>, true>(Xhi, Xlo, xrows, Bhi, Blo, c2, n_pad, none, C, ldc, 1, err, st);
    if (c2 <= 128)
        return tc::go<1, tc::Shape<64, 3, 128>, true>(Xhi, Xlo, xrows, Bhi, Blo, c2, n_pad, none, C, ldc, 1, err, st);
    return tc::go<1, tc::Shape<64, 2, 256>, true>(Xhi, Xlo, xrows, Bhi, Blo, c2, n_pad, none, C, ldc, 1, err, st);
}


bool oa_gemm_tc_fusable(int variant, int t) { return t <= 128 || variant >= 3; }

cudaError_t oa_launch_gemm_tcf(int R, int raster, const float* X, size_t ldx, int n, int xrows, const float* colmean,
                               const int* has_nan, int center, const __nv_bfloat16* Yhi, const __nv_bfloat16* Ylo, int t, int n_pad,
                               const EpiArgs& E, int* err, cudaStream_t st) {
    switch (R) {
        case 1: return tc::go_any_f<1>(raster, X, ldx, n, xrows, colmean, has_nan, center, Yhi, Ylo, t, n_pad, E, err, st);
        case 2: return tc::go_any_f<2>(raster, X, ldx, n, xrows, colmean, has_nan, center, Yhi, Ylo, t, n_pad, E, err, st);
        case 4: return tc::go_any_f<4>(raster, X, ldx, n, xrows, colmean, has_nan, center, Yhi, Ylo, t, n_pad, E, err, st);
        case 8: return tc::go_any_f<8>(raster, X, ldx, n, xrows, colmean, has_nan, center, Yhi, Ylo, t, n_pad, E, err, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t oa_launch_pre_tcf(const float* X, size_t ldx, int n, int xrows, const float* colmean, const int* has_nan,
                              int center,
                              const __nv_bfloat16* Bhi, const __nv_bfloat16* Blo, int c2, int n_pad, float* C, int ldc,
                              int* err, cudaStream_t st) {
    const EpiArgs none{};
    if (c2 <= 64)
        return tc::go_f<1, tc::FNarrow64, true>(X, ldx, n, xrows, colmean, has_nan, center, Bhi, Blo, c2, n_pad, none, C, ldc, 1,
                                                err, st);
    if (c2 <= 128)
        return tc::go_f<1, tc::FNarrow128, true>(X, ldx, n, xrows, colmean, has_nan, center, Bhi, Blo, c2, n_pad, none, C, ldc,
                                                 1, err, st);
    return cudaErrorInvalidValue;
}

}  // namespace oa
