// Per-SNP column statistics without covariates (k_snp_lean) and the FP64
// Schur kernel (k_schur) that combines them with the pre-GEMM output.
//
// The per-SNP quantities of the reference's corrected systems
// (Str/Sbr and their missing-row downdates, src/Algorithm.cpp:633-689,
// 1260-1315) split into
//   * X'X (r x r) over all rows and over each row set (missingness pattern
//     or zero set): k_snp_lean, from the SNP columns staged in shared memory
//     (x-only gathers, no covariate loads);
//   * Q'X and (Q o m_s)'X for every row set s: a GEMM of the SNP block with
//     the column matrix B2 = [Q | Q o m_1 | ... | Q o m_S] ("pre-GEMM", on
//     the same tensor-core / SIMT kernels as the main contraction);
// and k_schur forms, per (pattern, SNP), the FP64 Schur complement
//     (D - D_g) - (A - A_g)' W_g (A - A_g)
// and its inverse, plus var_x from the all-rows complement D - A'A.
#pragma once
#include "oa_stats.cuh"

namespace oa {

struct LeanArgs {
    const float* X;       // SNP block, column c at X + c*ldx
    size_t ldx;
    const int* xrows;     // row k of a column is X[c*ldx + xrows[k]] (a row subset), or null: X[c*ldx + k]
    int n, n_pad, mb, nbuf;
    int nsets;
    const int* rows;          // flattened row lists of the row sets
    const int* item_start;    // work items: rows [item_start[i], item_start[i+1]) of one set
    const int* set_item_off;  // items of set s: [set_item_off[s], set_item_off[s+1])
    const int* pass_off;      // passes over sets [pass_off[p], pass_off[p+1]) whose items fit in shared memory
    int npass;
    int items_cap;
    float* mean;          // [mb*r] column means if center, else imputation means (0 if the column had no NaN)
    int* has_nan;
    float* D;             // [mb][r*r] X'X over all rows
    float* Dset;          // [nsets][mb][r*r] X'X over each row set
    __nv_bfloat16* Xhi;   // [mb*r][n_pad] (tensor-core form) or null
    __nv_bfloat16* Xlo;
    int write_split;
    int use_xi;           // with several columns per group: keep the row-interleaved copy for the set pass
    int center;           // take each column relative to its mean (valid when XL holds an intercept)
    int* err;
    // all-rows covariate projection A = Q'(x - shift) of every column, summed here (short FP32
    // partial sums, FP64 across warps) instead of taken from the pre-GEMM, or null: with two or
    // more columns per SNP the all-rows Schur complement D - A'A (var_x) and the pattern systems
    // cancel a large part of D, and the pre-GEMM's long FP32 / BF16-split sums of A are then the
    // largest error of the statistics (the qx kernels, at most LEAN_QX_L covariates)
    const float4* Qb;     // [n_pad / 4][l] the orthonormal covariate basis (FP32) by blocks of four
                          // rows: Qb[k4 * l + q] = rows 4 k4 .. 4 k4 + 3 of covariate q (0 past n)
    int l;
    const double* qsum;   // [l] column sums of the basis (FP64)
    double* Afull;        // [mb*R][LEAN_QX_L]: A of column c, covariate q at Afull[c * LEAN_QX_L + q]
};

// Threads per CTA (the template's NT): 256; one column per group may also run 512 (launched where
// the column fills so much shared memory that few CTAs fit on an SM).  Shared scratch is sized
// for 512.
constexpr int LEAN_MAX_THREADS = 512;
constexpr int LEAN_MAX_WARPS = LEAN_MAX_THREADS / 32;
constexpr int LEAN_ITEM_ROWS = 256;     // rows per work item of the set pass
constexpr int LEAN_STAGE_U = 8;         // elements per thread and step of the element-wise staging
constexpr int LEAN_QX_L = 8;            // covariates of the in-kernel projection (l <= 8)
constexpr int LEAN_QX_NC = 4;           // columns per group of the qx kernels

// Shared memory of k_snp_lean: nbuf column buffers (stride n_pad floats, the
// tail [n, n_pad) kept zero) | with several columns per group, the centred
// columns interleaved by row ([n_pad][spb*R], one vector load per row in the
// set pass) | per-item partial sums | reduction scratch.
__host__ __device__ inline size_t lean_smem_bytes(int R, int n_pad, int spb, int nbuf, int items_cap,
                                                  bool use_xi = true, bool qx = false) {
    const int NC = spb * R;
    const int NQ = 2 * NC + spb * R * R + (qx ? NC * LEAN_QX_L : 0);
    return (size_t)(nbuf + (NC > 1 && use_xi ? 1 : 0)) * NC * n_pad * 4 + (size_t)items_cap * spb * R * R * 4 +
           (size_t)(LEAN_MAX_WARPS + 1) * NQ * 8 + 64;
}

// Block-wide sum of NV floats per thread over NW warps: FP32 within a warp, FP64 across
// warps (warp 0, fixed order); the first NB sums are copied to out[] on every
// thread, all NV stay at red + LEAN_MAX_WARPS * NV until red is reused.
template <int NW, int NV, int NB = NV>
__device__ __forceinline__ void block_sum_fd(float (&v)[NV], double (&out)[NB], double* red /* [warps + 1][NV] */) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_sumf(v[q]);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) red[w * NV + q] = (double)v[q];
    __syncthreads();
    double* bc = red + LEAN_MAX_WARPS * NV;
    if (w == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            const double s = warp_sum(lane < NW ? red[lane * NV + q] : 0.0);
            if (lane == 0) bc[q] = s;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NB; ++q) out[q] = bc[q];
}

// BF16 hi/lo of 8 floats (x = hi + lo to ~2^-17 relative), packed
__device__ __forceinline__ void split8(const float4 p0, const float4 p1, uint4& hi, uint4& lo) {
    const float e[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
    uint32_t h[4], o[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const __nv_bfloat162 hb = __floats2bfloat162_rn(e[2 * u], e[2 * u + 1]);
        const float2 hf = __bfloat1622float2(hb);
        const __nv_bfloat162 lb = __floats2bfloat162_rn(e[2 * u] - hf.x, e[2 * u + 1] - hf.y);
        h[u] = *reinterpret_cast<const uint32_t*>(&hb);
        o[u] = *reinterpret_cast<const uint32_t*>(&lb);
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(o[0], o[1], o[2], o[3]);
}

// One CTA handles SPB SNPs (SPB*R columns) per group; a persistent loop over
// groups with the next group's columns streaming into shared memory (TMA
// bulk copies of aligned columns; 4-byte cp.async copies otherwise, which also
// gather a row subset of a resident genotype matrix) while this one is
// processed:
//   pass 1  column sums and raw cross products from float4 reads of the
//           staged columns, one block reduction (FP64 across warps); NaN
//           propagates, so a column whose sum is NaN is counted and
//           mean-imputed in place (src/Utility.cpp:302-326) and the sweep
//           repeated - rare, dosage files seldom hold NaN.  With an
//           intercept among the covariates every later sum uses x - mean
//           (the Schur complements, X'y~ and var_x do not change; the sums
//           lose their large common part); X'X of the shifted columns
//           follows from the raw sums in FP64
//   pass 2  BF16 hi/lo split of the shifted columns (tensor-core form) and,
//           with several columns per group, their row-interleaved copy
//   pass 3  X'X over each row set: work items of at most 256 rows of one set
//           (fixed on the host per trait block) go round-robin to the warps;
//           a warp's item sum (row indices prefetched, one vector load of
//           the interleaved centred columns per row, shuffle reduction)
//           lands in its own shared-memory slot, and a set's sum adds its
//           items in order.  No atomics: the sums are bit-reproducible.
template <int R, int SPB, bool BULK, bool QX = false, int NT = 256>
__global__ void __launch_bounds__(NT)
k_snp_lean(LeanArgs A) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr int NC = SPB * R;                 // columns per group
    constexpr int K2 = SPB * R * R;             // X'X entries per group
    constexpr int NWARP = NT / 32;
    const int n = A.n, nS = A.n_pad;
    const size_t buf_floats = (size_t)NC * nS;
    float* bufs = reinterpret_cast<float*>(smem_raw);                                   // [nbuf][NC][nS]
    float* xi = bufs + (size_t)A.nbuf * buf_floats;                                     // [nS][NC] if NC > 1
    const bool use_xi = NC > 1 && A.use_xi;
    float* part = xi + (use_xi ? (size_t)NC * nS : 0);                                   // [items_cap][K2]
    double* red = reinterpret_cast<double*>(
        (reinterpret_cast<uintptr_t>(part + (size_t)A.items_cap * K2) + 7) & ~(uintptr_t)7);   // [LEAN_MAX_WARPS + 1][NQ]
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ int stop;
    const int ngroups = (A.mb + SPB - 1) / SPB;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;

    auto issue = [&](int g, int b) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // earlier generic writes to the buffer
        const int i0 = g * SPB;
        const int ncol = min(SPB, A.mb - i0) * R;
        const uint32_t bytes = (uint32_t)n * 4u;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(st_su32(&mbar[b])),
                     "r"(bytes * (uint32_t)ncol)
                     : "memory");
        for (int c = 0; c < ncol; ++c) {
            const float* src = A.X + (size_t)(i0 * R + c) * A.ldx;
            float* dst = bufs + (size_t)b * buf_floats + (size_t)c * nS;
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    st_su32(dst)),
                "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(st_su32(&mbar[b]))
                : "memory");
        }
    };

    // element-wise staging (columns not 16-byte aligned, or a row subset): 4-byte
    // cp.async copies, one commit group per group of columns and thread
    auto stage = [&](int g, int b) {
        const int i0 = g * SPB;
        const int ncol = min(SPB, A.mb - i0) * R;
        for (int c = 0; c < ncol; ++c) {
            const float* src = A.X + (size_t)(i0 * R + c) * A.ldx;
            const uint32_t dst = st_su32(bufs + (size_t)b * buf_floats + (size_t)c * nS);
            // LEAN_STAGE_U elements per thread and step: the row indices of a step
            // are loaded together, so their latencies overlap
            constexpr int nt = NT;
            for (int k0 = threadIdx.x; k0 < n; k0 += LEAN_STAGE_U * nt) {
                int kk[LEAN_STAGE_U];
#pragma unroll
                for (int u = 0; u < LEAN_STAGE_U; ++u) {
                    const int k = k0 + u * nt;
                    kk[u] = k < n ? (A.xrows ? __ldg(A.xrows + k) : k) : -1;
                }
#pragma unroll
                for (int u = 0; u < LEAN_STAGE_U; ++u)
                    if (kk[u] >= 0)
                        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                                         dst + 4u * (uint32_t)(k0 + u * nt)),
                                     "l"(src + kk[u])
                                     : "memory");
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    if (!BULK && (int)blockIdx.x < ngroups) stage(blockIdx.x, 0);

    // zero the column tails [n, n_pad) once: copies write only [0, n)
    for (int q = threadIdx.x; q < A.nbuf * NC * (nS - n); q += blockDim.x) {
        const int c = q / (nS - n), k = n + q % (nS - n);
        bufs[(size_t)c * nS + k] = 0.f;
    }
    if (threadIdx.x == 0) {
        stop = 0;
        if (BULK) {
            for (int b = 0; b < 2; ++b) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(st_su32(&mbar[b])));
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            if ((int)blockIdx.x < ngroups) issue(blockIdx.x, 0);
        }
    }
    __syncthreads();

    int q = 0;
    for (int g = blockIdx.x; g < ngroups; g += gridDim.x, ++q) {
        const int gn = g + gridDim.x;
        const int b = A.nbuf == 2 ? (q & 1) : 0;
        const uint32_t par = A.nbuf == 2 ? (uint32_t)((q >> 1) & 1) : (uint32_t)(q & 1);
        float* xs = bufs + (size_t)b * buf_floats;
        const int i0 = g * SPB;
        const int nsnp = min(SPB, A.mb - i0);
        const int ncol = nsnp * R;

        if (BULK) {
            if (threadIdx.x == 0) {
                if (A.nbuf == 2 && gn < ngroups) issue(gn, b ^ 1);
                if (!st_mbar_wait(&mbar[b], par)) {
                    stop = 1;
                    atomicExch(A.err, 1);
                }
            }
            __syncthreads();
            if (stop) break;
            st_mbar_try(&mbar[b], par);
        } else {
            // the next group goes into the other buffer (read completely in the previous round)
            if (A.nbuf == 2 && gn < ngroups) {
                stage(gn, b ^ 1);
                asm volatile("cp.async.wait_group 1;" ::: "memory");
            } else {
                asm volatile("cp.async.wait_group 0;" ::: "memory");
            }
            __syncthreads();
        }
        const float4* x4 = reinterpret_cast<const float4*>(xs);
        const int nS4 = nS / 4;

        // ---- pass 1: column sums and raw cross products in one sweep (the
        // zero tail adds nothing); NaN propagates, so a column whose sum is
        // NaN is counted and mean-imputed in place (src/Utility.cpp:302-326)
        // and the sweep is repeated - rare, dosage files seldom hold NaN
        float sh[NC];                          // subtracted from every value (centring), 0 without
        bool cnan[NC];
        {
            constexpr int NQX = QX ? NC * LEAN_QX_L : 0;
            constexpr int NV = NC + K2 + NQX;  // [column sums | cross products | Q'x of the raw columns]
            constexpr int NB = NC + K2;        // sums every thread keeps (Q'x stays in shared memory)
            static_assert(!QX || NC <= LEAN_QX_NC, "columns of the qx kernels");
            float acc[NV];
            double tot[NB];
            const double* qxs = red + LEAN_MAX_WARPS * NV + NB;   // the block's Q'x sums after the last sweep
            auto sweep = [&]() {
#pragma unroll
                for (int u = 0; u < NV; ++u) acc[u] = 0.f;
                for (int k4 = threadIdx.x; k4 < nS4; k4 += blockDim.x) {
                    float4 v[NC];
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        v[c] = c < ncol ? x4[(size_t)c * nS4 + k4] : make_float4(0.f, 0.f, 0.f, 0.f);
                        acc[c] += (v[c].x + v[c].y) + (v[c].z + v[c].w);
                    }
                    if constexpr (QX) {
                        // rows 4 k4 .. 4 k4 + 3 of each covariate: one 16-byte load per covariate
#pragma unroll
                        for (int qq = 0; qq < LEAN_QX_L; ++qq) {
                            if (qq < A.l) {
                                const float4 q4 = __ldg(A.Qb + (size_t)k4 * A.l + qq);
#pragma unroll
                                for (int c = 0; c < NC; ++c) {
                                    float& a = acc[NC + K2 + c * LEAN_QX_L + qq];
                                    a = fmaf(q4.x, v[c].x, a);
                                    a = fmaf(q4.y, v[c].y, a);
                                    a = fmaf(q4.z, v[c].z, a);
                                    a = fmaf(q4.w, v[c].w, a);
                                }
                            }
                        }
                    }
#pragma unroll
                    for (int s2 = 0; s2 < SPB; ++s2)
#pragma unroll
                        for (int a = 0; a < R; ++a)
#pragma unroll
                            for (int bb = 0; bb < R; ++bb) {
                                const float4 xa = v[s2 * R + a], xb = v[s2 * R + bb];
                                float& d = acc[NC + (s2 * R + a) * R + bb];
                                d = fmaf(xa.x, xb.x, d);
                                d = fmaf(xa.y, xb.y, d);
                                d = fmaf(xa.z, xb.z, d);
                                d = fmaf(xa.w, xb.w, d);
                            }
                }
                block_sum_fd<NWARP, NV, NB>(acc, tot, red);
            };
            sweep();
            bool any_nan = false;
            float cmean[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                cnan[c] = (c < ncol) && isnan(tot[c]);
                any_nan |= cnan[c];
                cmean[c] = (float)(tot[c] / (double)n);
            }
            if (any_nan) {   // block-uniform: count and sum the observed values, impute in place
                __syncthreads();   // every thread has read the sums before the scratch is reused
                float cs[2 * NC];
                double ct[2 * NC];
#pragma unroll
                for (int u = 0; u < 2 * NC; ++u) cs[u] = 0.f;
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    if (cnan[c]) {
                        const float* col = xs + (size_t)c * nS;
                        for (int k = threadIdx.x; k < n; k += blockDim.x) {
                            const float v = col[k];
                            if (isnan(v)) cs[NC + c] += 1.f;
                            else cs[c] += v;
                        }
                    }
                }
                block_sum_fd<NWARP, 2 * NC>(cs, ct, red);
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    if (cnan[c]) {
                        cmean[c] = (float)(ct[c] / ((double)n - ct[NC + c]));
                        float* col = xs + (size_t)c * nS;
                        for (int k = threadIdx.x; k < n; k += blockDim.x)
                            if (isnan(col[k])) col[k] = cmean[c];
                    }
                }
                __syncthreads();
                sweep();
            }
#pragma unroll
            for (int c = 0; c < NC; ++c) sh[c] = A.center ? cmean[c] : 0.f;
            if constexpr (QX) {
                // A = Q'(x - shift) = Q'x - shift * (column sums of Q), in FP64; thread u writes entry u
                // (compile-time register indices)
#pragma unroll
                for (int c = 0; c < NC; ++c)
                    if ((int)threadIdx.x / LEAN_QX_L == c && c < ncol) {
                        const int qq = threadIdx.x % LEAN_QX_L;
                        A.Afull[(size_t)(i0 * R + c) * LEAN_QX_L + qq] =
                            qq < A.l ? qxs[c * LEAN_QX_L + qq] - (double)sh[c] * A.qsum[qq] : 0.0;
                    }
            }
            if (threadIdx.x == 0) {
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    if (c < ncol) {
                        A.mean[i0 * R + c] = A.center ? cmean[c] : (cnan[c] ? cmean[c] : 0.f);
                        if (cnan[c]) atomicOr(A.has_nan, 1);
                    }
                }
                // X'X of the columns taken relative to sh over the n rows:
                // sum x_a x_b - s_a sum x_b - s_b sum x_a + n s_a s_b
#pragma unroll
                for (int s2 = 0; s2 < SPB; ++s2)
#pragma unroll
                    for (int a = 0; a < R; ++a)
#pragma unroll
                        for (int bb = 0; bb < R; ++bb) {
                            const int ca = s2 * R + a, cb = s2 * R + bb, u = (s2 * R + a) * R + bb;
                            const double sa = sh[ca], sb = sh[cb];
                            const double d = tot[NC + u] - sa * tot[cb] - sb * tot[ca] + (double)n * sa * sb;
                            if (s2 < nsnp) A.D[(size_t)i0 * R * R + u] = (float)d;
                        }
            }
        }

        // ---- pass 2: BF16 hi/lo split of the centred columns (tensor-core
        // form) and, with several columns per group, the centred columns
        // interleaved by row for the set pass; 8 rows per thread and step.
        // The tail rows [n, n_pad) get -sh: the other operands of the GEMMs
        // are zero there.
        if (A.write_split || use_xi) {
            const int np8 = nS / 8;
            for (int k8 = threadIdx.x; k8 < np8; k8 += blockDim.x) {
                float e[NC][8];
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f), p1 = p0;
                    if (c < ncol) {
                        p0 = x4[(size_t)c * nS4 + 2 * k8];
                        p1 = x4[(size_t)c * nS4 + 2 * k8 + 1];
                    }
                    const float s0 = sh[c];
                    e[c][0] = p0.x - s0;
                    e[c][1] = p0.y - s0;
                    e[c][2] = p0.z - s0;
                    e[c][3] = p0.w - s0;
                    e[c][4] = p1.x - s0;
                    e[c][5] = p1.y - s0;
                    e[c][6] = p1.z - s0;
                    e[c][7] = p1.w - s0;
                    if (A.write_split && c < ncol) {
                        uint4 h, o;
                        split8(make_float4(e[c][0], e[c][1], e[c][2], e[c][3]),
                               make_float4(e[c][4], e[c][5], e[c][6], e[c][7]), h, o);
                        reinterpret_cast<uint4*>(A.Xhi + (size_t)(i0 * R + c) * A.n_pad)[k8] = h;
                        reinterpret_cast<uint4*>(A.Xlo + (size_t)(i0 * R + c) * A.n_pad)[k8] = o;
                    }
                }
                if (!use_xi) {
                } else if constexpr (NC == 2) {
                    float4* d = reinterpret_cast<float4*>(xi + (size_t)k8 * 16);
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        d[u] = make_float4(e[0][2 * u], e[1][2 * u], e[0][2 * u + 1], e[1][2 * u + 1]);
                } else if constexpr (NC == 4) {
                    float4* d = reinterpret_cast<float4*>(xi + (size_t)k8 * 32);
#pragma unroll
                    for (int u = 0; u < 8; ++u) d[u] = make_float4(e[0][u], e[1][u], e[2][u], e[3][u]);
                } else if constexpr (NC > 1) {
#pragma unroll
                    for (int u = 0; u < 8; ++u)
#pragma unroll
                        for (int c = 0; c < NC; ++c) xi[(size_t)(8 * k8 + u) * NC + c] = e[c][u];
                }
            }
            if (use_xi) __syncthreads();   // xi is read by other warps in the set pass
        }

        // ---- pass 3: X'X over each row set, by work items
        for (int ps = 0; ps < A.npass; ++ps) {
            const int s0 = __ldg(A.pass_off + ps), s1 = __ldg(A.pass_off + ps + 1);
            const int it0 = __ldg(A.set_item_off + s0), it1 = __ldg(A.set_item_off + s1);
            for (int item = it0 + w; item < it1; item += NWARP) {
                const int ra = __ldg(A.item_start + item), rb = __ldg(A.item_start + item + 1);
                float sacc[K2];
#pragma unroll
                for (int u = 0; u < K2; ++u) sacc[u] = 0.f;
                constexpr int U = LEAN_ITEM_ROWS / 32;
                int kid[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int kk = ra + 32 * u + lane;
                    kid[u] = kk < rb ? __ldg(A.rows + kk) : -1;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (kid[u] >= 0) {
                        float x[NC];
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            if (NC == 1 || !use_xi) {
                                x[c] = xs[(size_t)c * nS + kid[u]] - sh[c];
                            } else if constexpr (NC % 4 == 0) {
                                if (c % 4 == 0) {
                                    const float4 q4 = reinterpret_cast<const float4*>(xi + (size_t)kid[u] * NC)[c / 4];
                                    x[c] = q4.x;
                                    x[c + 1] = q4.y;
                                    x[c + 2] = q4.z;
                                    x[c + 3] = q4.w;
                                }
                            } else {
                                if (c % 2 == 0) {
                                    const float2 q2 = reinterpret_cast<const float2*>(xi + (size_t)kid[u] * NC)[c / 2];
                                    x[c] = q2.x;
                                    x[c + 1] = q2.y;
                                }
                            }
                        }
#pragma unroll
                        for (int s = 0; s < SPB; ++s)
#pragma unroll
                            for (int a = 0; a < R; ++a)
#pragma unroll
                                for (int bb = 0; bb < R; ++bb)
                                    sacc[(s * R + a) * R + bb] = fmaf(x[s * R + a], x[s * R + bb], sacc[(s * R + a) * R + bb]);
                    }
                }
#pragma unroll
                for (int u = 0; u < K2; ++u) {
                    const float v = warp_sumf(sacc[u]);
                    if (lane == 0) part[(size_t)(item - it0) * K2 + u] = v;
                }
            }
            __syncthreads();
            for (int u = threadIdx.x; u < (s1 - s0) * K2; u += blockDim.x) {
                const int set = s0 + u / K2, e = u % K2;
                const int s = e / (R * R), f = e % (R * R);
                const int a0 = __ldg(A.set_item_off + set), a1 = __ldg(A.set_item_off + set + 1);
                float sum = 0.f;
                for (int it = a0; it < a1; ++it) sum += part[(size_t)(it - it0) * K2 + e];
                if (s < nsnp) A.Dset[((size_t)set * A.mb + i0 + s) * R * R + f] = sum;
            }
            __syncthreads();
        }
        __syncthreads();   // every reader of this buffer is done before it is refilled
        if (BULK && A.nbuf == 1 && threadIdx.x == 0 && gn < ngroups) issue(gn, 0);
        if (!BULK && A.nbuf == 1 && gn < ngroups) stage(gn, 0);
    }
    if (!BULK) asm volatile("cp.async.wait_group 0;" ::: "memory");   // nothing in flight at exit
    if (BULK && threadIdx.x == 0 && stop) {
        st_mbar_wait(&mbar[0], 0, true);
        st_mbar_wait(&mbar[0], 1, true);
        st_mbar_wait(&mbar[1], 0, true);
        st_mbar_wait(&mbar[1], 1, true);
    }
}

// The pre-GEMM's column matrix B2 = [Q | Q o m_1 | ... | Q o m_S] (K-major:
// column c of B2 is row c of the c2 x n_pad array), FP32 and, for the
// tensor-core form, BF16 hi/lo.  Step 1 writes Q and zeros; step 2 scatters
// Q's rows into the columns of every row set that contains them.
static __global__ void k_b2_init(const float* __restrict__ Qr, int LP, int n, int n_pad, int l, int c2,
                          float* __restrict__ B2) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)c2 * n_pad) return;
    const int c = (int)(q / n_pad), k = (int)(q % n_pad);
    B2[q] = (c < l && k < n) ? Qr[(size_t)k * LP + c] : 0.f;
}

static __global__ void k_b2_scatter(const float* __restrict__ Qr, int LP, int n_pad, int l, const int* __restrict__ set_off,
                             const int* __restrict__ rows, float* __restrict__ B2) {
    const int s = blockIdx.x;
    const int r0 = set_off[s], r1 = set_off[s + 1];
    float* dst = B2 + (size_t)(l + s * l) * n_pad;
    for (int kk = r0 + threadIdx.x; kk < r1; kk += blockDim.x) {
        const int k = rows[kk];
        for (int a = 0; a < l; ++a) dst[(size_t)a * n_pad + k] = Qr[(size_t)k * LP + a];
    }
}

static __global__ void k_split_bf16(const float* __restrict__ src, long long count, __nv_bfloat16* __restrict__ hi,
                             __nv_bfloat16* __restrict__ lo) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= count) return;
    const float v = src[q];
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    hi[q] = h;
    lo[q] = __float2bfloat16_rn(v - __bfloat162float(h));
}

struct SchurArgs {
    int l, mb, G, Z, ldc;
    int rr;                  // the caller's columns per SNP; columns [rr, R) are zero padding
    const float* C2;         // pre-GEMM output, column c of SNP column x at C2[c * ldc + x]
    const float* D;          // [mb][r*r]
    const float* Dset;       // [G+Z][mb][r*r]
    const double* W;         // [G][l][l]
    const uint8_t* pat_bad;  // [G]
    double* sinv;            // [G][mb][r*r]
    uint8_t* sing;           // [G][mb]
    float* varx;             // [mb][r]
    float* aobs;             // [G][mb][l][r] or null
    float* afull;            // [mb][l][r] or null
    double* sfinv;           // [mb][r*r] or null
    float* zA;               // [Z][mb][l][r]
    float* zD;               // [Z][mb][r][r]
    // the reference's r >= 2 downdate (quirk mode, raw uncentred columns), or null:
    float* qdel;             // [G][mb][l][r] the quirk's change of Q_obs'X
    double* qK;              // [G][mb][r][r] Gram matrix term of the quirk's RSS
    // all-rows projection A of each SNP column from k_snp_lean ([mb*r][LEAN_QX_L]), or null: A from
    // the pre-GEMM's first l columns
    const double* Afull_lean;
};

// The system of (pattern g, SNP i) as the reference's r >= 2 downdate builds
// it (correct_missings_S, src/Algorithm.cpp:1370-1399, read through sposv's
// upper triangle; Sbr_corr filled only for j < min(l, r), :1300): every SNP
// column's covariate downdate Str_corr is subtracted from the first SNP
// column only, and with r > l the SNP-block downdates of rows a >= l are
// missing.  In the orthonormal covariate basis (XL = Q R, raw uncentred SNP
// columns, Str_corr = R' A_g with A_g = (Q o m_g)'X) the quirk changes the
// covariate block ao = Q_obs'X to ao + dl with
//     dl[:, 0] = -sum_{b >= 1} A_g[:, b],   dl[:, b] = A_g[:, b] (b >= 1),
// and the SNP block Dobs = X_obs'X_obs by +D_g[a][b] for min(a, b) >= l.
// The quirk's solution is the Frisch-Waugh-Lovell one of that system:
//     beta_x = Sq^-1 (z - dl' b0_j),  Sq = Dobs + dD - (ao + dl)' W_g (ao + dl),
// and the reference's explicit RSS of that beta over the observed rows is
//     RSS = RSS0_j - 2 beta_x' z + beta_x' (Schur_g + dl' W_g dl) beta_x
// (the cross terms vanish because Q_obs' y~ = 0 and Q_obs'Q_obs = W_g^-1).
// Stored per (g, i): Sq^-1 (sinv), dl (qdel), Schur_g + dl' W_g dl (qK), and
// ao + dl (aobs: the covariate fit and the rows with y == 0 use it).
template <int R>
__device__ __noinline__ void schur_quirk(const SchurArgs& S, int i, int g, size_t gi, const double* ao,
                                         const double* Dm, const double* dso, bool full_ok) {
    const int l = S.l;
    const double* Wg = S.W + (size_t)g * l * l;
    double dl[OA_MAX_L * R], aq[OA_MAX_L * R];
    for (int qq = 0; qq < l; ++qq) {
        double ag[R];
#pragma unroll
        for (int a = 0; a < R; ++a) ag[a] = (double)S.C2[(size_t)(l + g * l + qq) * S.ldc + i * R + a];
        double rest = 0.0;
#pragma unroll
        for (int b = 1; b < R; ++b) rest += ag[b];
        dl[qq * R] = -rest;
#pragma unroll
        for (int b = 1; b < R; ++b) dl[qq * R + b] = ag[b];
#pragma unroll
        for (int a = 0; a < R; ++a) aq[qq * R + a] = ao[qq * R + a] + dl[qq * R + a];
    }
    // X'W X for the three column sets this needs: (ao, ao), (aq, aq), (dl, dl)
    auto quad = [&](const double* u, double* out) {
#pragma unroll
        for (int a = 0; a < R * R; ++a) out[a] = 0.0;
        for (int qq = 0; qq < l; ++qq) {
            double wu[R];
#pragma unroll
            for (int b = 0; b < R; ++b) wu[b] = 0.0;
            for (int v = 0; v < l; ++v) {
                const double w = Wg[qq * l + v];
#pragma unroll
                for (int b = 0; b < R; ++b) wu[b] += w * u[v * R + b];
            }
#pragma unroll
            for (int a = 0; a < R; ++a)
#pragma unroll
                for (int b = 0; b < R; ++b) out[a * R + b] += u[qq * R + a] * wu[b];
        }
    };
    double Dobs[R * R], Sq[R * R], t1[R * R], t2[R * R];
#pragma unroll
    for (int u = 0; u < R * R; ++u) Dobs[u] = Dm[u] - (double)S.Dset[gi * R * R + u];
    quad(aq, t1);
#pragma unroll
    for (int a = 0; a < R; ++a)
#pragma unroll
        for (int b = 0; b < R; ++b) {
            const double dD = (a >= l && b >= l) ? (double)S.Dset[gi * R * R + a * R + b] : 0.0;
            Sq[a * R + b] = Dobs[a * R + b] + dD - t1[a * R + b];
        }
    quad(ao, t1);
    quad(dl, t2);
#pragma unroll
    for (int u = 0; u < R * R; ++u) S.qK[gi * R * R + u] = Dobs[u] - t1[u] + t2[u];
#pragma unroll
    for (int a = 0; a < R; ++a)
        if (a >= S.rr) Sq[a * R + a] = 1.0;
    const bool ok = full_ok && !S.pat_bad[g] && schur_inverse<R>(Sq, dso);
    S.sing[gi] = ok ? 0 : 1;
#pragma unroll
    for (int u = 0; u < R * R; ++u) S.sinv[gi * R * R + u] = ok ? Sq[u] : 0.0;
    for (int u = 0; u < l * R; ++u) S.qdel[gi * l * R + u] = (float)dl[u];
    if (S.aobs)
        for (int u = 0; u < l * R; ++u) S.aobs[gi * l * R + u] = (float)aq[u];
}

// All (SNP, pattern) systems of a SNP block in one persistent launch: a
// thread per (SNP, slot) work item, grid-stride over the items.  Slot 0 is
// the all-rows complement (var_x), slots 1..G the patterns, slots
// G+1..G+Z copy the zero-set sums.
template <int R>
__device__ __forceinline__ void schur_item(const SchurArgs& S, int i, int slot) {
    const int l = S.l;
    double a_full[OA_MAX_L * R];
    if (S.Afull_lean) {
        for (int qq = 0; qq < l; ++qq)
#pragma unroll
            for (int a = 0; a < R; ++a) a_full[qq * R + a] = S.Afull_lean[((size_t)i * R + a) * LEAN_QX_L + qq];
    } else {
        for (int qq = 0; qq < l; ++qq)
#pragma unroll
            for (int a = 0; a < R; ++a) a_full[qq * R + a] = (double)S.C2[(size_t)qq * S.ldc + i * R + a];
    }
    double Dm[R * R];
#pragma unroll
    for (int u = 0; u < R * R; ++u) Dm[u] = (double)S.D[(size_t)i * R * R + u];
    // all-rows Schur complement D - A'A (Q orthonormal): var_x of the SNP terms (src/Algorithm.cpp:665-670)
    double Sf[R * R];
#pragma unroll
    for (int a = 0; a < R; ++a)
#pragma unroll
        for (int b = 0; b < R; ++b) {
            double v = Dm[a * R + b];
            for (int qq = 0; qq < l; ++qq) v -= a_full[qq * R + a] * a_full[qq * R + b];
            Sf[a * R + b] = v;
        }
    double dss[R];
#pragma unroll
    for (int a = 0; a < R; ++a) dss[a] = Dm[a * R + a];
    // zero padding columns (r = 3, 5, 6, 7 run as 4 or 8): their rows and columns of every sum are
    // exactly 0; an identity block keeps them out of the other columns' solution (coefficient 0)
#pragma unroll
    for (int a = 0; a < R; ++a)
        if (a >= S.rr) Sf[a * R + a] = dss[a] = 1.0;
    const bool full_ok = schur_inverse<R>(Sf, dss);
    if (slot == 0) {
#pragma unroll
        for (int a = 0; a < R; ++a) S.varx[(size_t)i * R + a] = full_ok ? (float)Sf[a * R + a] : 0.f;
        if (S.sfinv)
#pragma unroll
            for (int u = 0; u < R * R; ++u) S.sfinv[(size_t)i * R * R + u] = full_ok ? Sf[u] : 0.0;
        if (S.afull)
            for (int u = 0; u < l * R; ++u) S.afull[(size_t)i * l * R + u] = (float)a_full[u];
        return;
    }
    if (slot > S.G) {  // zero set z: its sums go to the epilogue unchanged
        const int z = slot - 1 - S.G;
        const size_t zi = (size_t)z * S.mb + i;
        for (int qq = 0; qq < l; ++qq)
#pragma unroll
            for (int a = 0; a < R; ++a)
                S.zA[zi * l * R + qq * R + a] = S.C2[(size_t)(l + (S.G + z) * l + qq) * S.ldc + i * R + a];
#pragma unroll
        for (int u = 0; u < R * R; ++u) S.zD[zi * R * R + u] = S.Dset[((size_t)(S.G + z) * S.mb + i) * R * R + u];
        return;
    }
    const int g = slot - 1;
    const size_t gi = (size_t)g * S.mb + i;
    double ao[OA_MAX_L * R];
    for (int qq = 0; qq < l; ++qq)
#pragma unroll
        for (int a = 0; a < R; ++a)
            ao[qq * R + a] = a_full[qq * R + a] - (double)S.C2[(size_t)(l + g * l + qq) * S.ldc + i * R + a];
    double Sg[R * R];
#pragma unroll
    for (int u = 0; u < R * R; ++u) Sg[u] = Dm[u] - (double)S.Dset[gi * R * R + u];
    double dso[R];
#pragma unroll
    for (int a = 0; a < R; ++a) dso[a] = a < S.rr ? Sg[a * R + a] : 1.0;
    const double* Wg = S.W + (size_t)g * l * l;
    for (int qq = 0; qq < l; ++qq) {
        double wa[R];
#pragma unroll
        for (int b = 0; b < R; ++b) wa[b] = 0.0;
        for (int u = 0; u < l; ++u) {
            const double wq = Wg[qq * l + u];
#pragma unroll
            for (int b = 0; b < R; ++b) wa[b] += wq * ao[u * R + b];
        }
#pragma unroll
        for (int a = 0; a < R; ++a)
#pragma unroll
            for (int b = 0; b < R; ++b) Sg[a * R + b] -= ao[qq * R + a] * wa[b];
    }
    if (S.qK) {
        schur_quirk<R>(S, i, g, gi, ao, Dm, dso, full_ok);
        return;
    }
#pragma unroll
    for (int a = 0; a < R; ++a)
        if (a >= S.rr) Sg[a * R + a] = 1.0;
    const bool ok = full_ok && !S.pat_bad[g] && schur_inverse<R>(Sg, dso);
    S.sing[gi] = ok ? 0 : 1;
#pragma unroll
    for (int u = 0; u < R * R; ++u) S.sinv[gi * R * R + u] = ok ? Sg[u] : 0.0;
    if (S.aobs)
        for (int u = 0; u < l * R; ++u) S.aobs[gi * l * R + u] = (float)ao[u];
}

// Items are numbered slot-major (consecutive threads take consecutive SNPs of one slot), so that
// a warp's loads of the SNP-indexed sums (pre-GEMM columns, D, D_s) and its stores of the
// inverses are coalesced and the slot's W_g is one broadcast.
template <int R>
__global__ void __launch_bounds__(256) k_schur(SchurArgs S) {
    const int slots = 1 + S.G + S.Z;
    const long long total = (long long)S.mb * slots;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x)
        schur_item<R>(S, (int)(q % S.mb), (int)(q / S.mb));
}

}  // namespace oa
