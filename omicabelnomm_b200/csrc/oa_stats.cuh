// Per-SNP statistics kernel (k_snp_stats) and its launch geometry.
#pragma once
#include "oa_common.cuh"

namespace oa {

// Block-wide sum of NV doubles held per thread; result valid in out[] on all threads.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* red /* [8][NV] */) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) red[w * NV + q] = v[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double s = 0.0;
        for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) s += red[ww * NV + q];
        v[q] = s;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Per-SNP statistics.  One CTA handles SPB SNPs (SPB*R columns staged in
// shared memory).  Outputs per SNP i of the block and per pattern g:
//   sinv[g][i]  = (D_obs - A_obs' W_g A_obs)^-1           (r x r, FP64)
//   varx[i]     = diag((D - A'A)^-1)  (all rows; the reference's var_x of the SNP terms)
//   aobs[g][i]  = A - A_g  (Q_obs'X, only when needed)
//   afull[i], sfinv[i]  (for covariate terms)
//   zA/zD[z][i] sums over the zero rows of zero set z
// where A = Q'X (l x r), D = X'X (r x r), A_g / D_g the same sums over the
// pattern's missing rows.
// ---------------------------------------------------------------------------
struct StatsArgs {
    const float* X;      // SNP block, column c at X + c*ldx
    size_t ldx;
    int n, n_pad, l, QS, mb, spb;
    const float* Qr;     // Q row-major, row k at Qr + k*QS (FP32)
    int nsets, G, Z;     // row sets: G patterns then Z zero sets
    const int* set_off;
    const int* rows;
    const float* qrows;  // Q rows of each set's rows, gathered contiguous ([rows][QS], FP32)
    const double* W;     // [G][l][l]
    const uint8_t* pat_bad;
    int sets_per_pass;   // row sets whose sums fit in shared memory at once
    // outputs
    float* mean;         // [mb*r] column means used for NaN imputation
    int* has_nan;        // set to 1 if any NaN was imputed
    double* sinv;        // [G][mb][r*r]
    uint8_t* sing;       // [G][mb]
    float* varx;         // [mb][r]
    float* aobs;         // [G][mb][l][r] or null
    float* afull;        // [mb][l][r] or null
    double* sfinv;       // [mb][r*r] or null
    float* zA;           // [Z][mb][l][r]
    float* zD;           // [Z][mb][r][r]
    __nv_bfloat16* Xhi;  // [mb*r][n_pad] or null (tensor-core form)
    __nv_bfloat16* Xlo;
    int write_split;
    int center;          // take each column relative to its mean (valid when XL holds an intercept)
    int nbuf;            // column buffers (2: the next group streams in during this one)
    int* err;            // set if a staging copy did not complete in time
};

// Accumulators per SNP for R columns and LP (padded) covariates, and the
// largest number of SNPs a CTA handles so that they stay in registers.
__host__ __device__ constexpr int stats_na(int R, int LP) { return R * R + LP * R; }
__host__ __device__ constexpr int stats_spb_max(int R, int LP) {
    return (8 / R) < (64 / stats_na(R, LP)) ? (8 / R)
           : ((64 / stats_na(R, LP)) > 0 ? (64 / stats_na(R, LP)) : 1);
}
// Shared-memory layout of k_snp_stats: nbuf column buffers | full | red | setacc
__host__ __device__ inline size_t stats_smem_bytes(int R, int LP, int n, int spb, int nbuf, int sets_per_pass) {
    const int nS = (n + 3) & ~3;
    const int NT = spb * stats_na(R, LP);
    const int NR = NT > 16 ? NT : 16;
    return (size_t)nbuf * spb * R * nS * 4 + (size_t)NT * 8 + (size_t)8 * NR * 8 + (size_t)sets_per_pass * NT * 4;
}

__device__ __forceinline__ uint32_t st_su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool st_mbar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(st_su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bound of the staging waits (2 s by default; oa_set_wait_limit_stats
// changes it for the device, which the timeout tests use to make the waits
// run out).  The drain waits after a stop keep the 2 s bound.
static __constant__ unsigned long long c_st_wait_ns = 2000000000ull;

// Bounded wait on %globaltimer: the staging bound, or 2 s when draining.
__device__ __forceinline__ bool st_mbar_wait(uint64_t* b, uint32_t parity, bool drain = false) {
    const unsigned long long lim = drain ? 2000000000ull : c_st_wait_ns;
    unsigned long long t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    while (!st_mbar_try(b, parity)) {
        unsigned long long t1;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
        if (t1 - t0 > lim) return false;
    }
    return true;
}

template <int R, int LP, bool BULK>
__global__ void __launch_bounds__(OA_NTHREADS)
k_snp_stats(StatsArgs A) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr int NA = stats_na(R, LP);            // accumulators per SNP
    constexpr int SPBM = stats_spb_max(R, LP);
    constexpr int ACC = SPBM * NA;
    const int n = A.n, l = A.l, spb = A.spb;
    const int nS = (n + 3) & ~3;
    const int NT = spb * NA;
    const size_t buf_floats = (size_t)spb * R * nS;
    float* bufs = reinterpret_cast<float*>(smem_raw);                         // [nbuf][spb*R][nS]
    double* full = reinterpret_cast<double*>(bufs + (size_t)A.nbuf * buf_floats);  // [spb][NA]
    double* red = full + NT;                                                  // [8][max(16, NT)]
    float* setacc = reinterpret_cast<float*>(red + 8 * (NT > 16 ? NT : 16));  // [sets_per_pass][spb][NA]
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ int fsing[8];
    __shared__ float cmean[8];
    __shared__ float cshift[8];
    __shared__ int cnan[8];
    __shared__ int stop;

    const int ngroups = (A.mb + spb - 1) / spb;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;

    // TMA bulk copy of a group's columns into buffer b (thread 0)
    auto issue = [&](int g, int b) {
        const int i0 = g * spb;
        const int ncol = min(spb, A.mb - i0) * R;
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

    if (threadIdx.x == 0) {
        stop = 0;
        if (BULK) {
            for (int b = 0; b < 2; ++b) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(st_su32(&mbar[b])));
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            if ((int)blockIdx.x < ngroups) issue(blockIdx.x, 0);
        }
    }
    __syncthreads();

    int q = 0;  // groups processed by this CTA
    for (int g = blockIdx.x; g < ngroups; g += gridDim.x, ++q) {
        const int gn = g + gridDim.x;
        const int b = A.nbuf == 2 ? (q & 1) : 0;
        const uint32_t par = A.nbuf == 2 ? (uint32_t)((q >> 1) & 1) : (uint32_t)(q & 1);
        float* xs = bufs + (size_t)b * buf_floats;
        const int i0 = g * spb;
        const int nsnp = min(spb, A.mb - i0);
        const int ncol = nsnp * R;

        // 1. stage the columns
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
            st_mbar_try(&mbar[b], par);  // every thread observes the completed phase
        } else {
            for (int c = 0; c < ncol; ++c) {
                const float* src = A.X + (size_t)(i0 * R + c) * A.ldx;
                float* dst = xs + (size_t)c * nS;
#pragma unroll 4
                for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = src[k];
            }
            __syncthreads();
        }

        // NaN count and sum per column (from shared memory)
        double vs[2 * 8];
#pragma unroll
        for (int u = 0; u < 16; ++u) vs[u] = 0.0;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            if (c < ncol) {
                const float* col = xs + (size_t)c * nS;
                float s = 0.f, cnt = 0.f;
#pragma unroll 4
                for (int k = threadIdx.x; k < n; k += blockDim.x) {
                    const float v = col[k];
                    if (isnan(v)) cnt += 1.f;
                    else s += v;
                }
                vs[c] = s;
                vs[8 + c] = cnt;
            }
        }
        block_sum<16>(vs, red);
        if (threadIdx.x < ncol) {
            const int c = threadIdx.x;
            const double cnt = vs[8 + c];
            const float mean = (float)(vs[c] / ((double)n - cnt));
            cmean[c] = mean;
            cshift[c] = A.center ? mean : 0.f;
            cnan[c] = cnt > 0.0 ? 1 : 0;
            A.mean[i0 * R + c] = (A.center || cnt > 0.0) ? mean : 0.0f;
            if (cnt > 0.0) atomicOr(A.has_nan, 1);
        }
        __syncthreads();
        // 2. mean-impute NaN dosages (src/Utility.cpp:302-326)
        for (int c = 0; c < ncol; ++c) {
            if (cnan[c]) {
                float* col = xs + (size_t)c * nS;
                const float mv = cmean[c];
                for (int k = threadIdx.x; k < n; k += blockDim.x)
                    if (isnan(col[k])) col[k] = mv;
            }
        }
        __syncthreads();
        if (A.write_split) {
            // BF16 hi/lo of each column, 8 elements (two 16-byte stores) per thread and step
            const int np8 = A.n_pad / 8;
            for (int c = 0; c < ncol; ++c) {
                const float* col = xs + (size_t)c * nS;
                const float s0 = cshift[c];
                uint4* hi = reinterpret_cast<uint4*>(A.Xhi + (size_t)(i0 * R + c) * A.n_pad);
                uint4* lo = reinterpret_cast<uint4*>(A.Xlo + (size_t)(i0 * R + c) * A.n_pad);
                for (int k8 = threadIdx.x; k8 < np8; k8 += blockDim.x) {
                    uint32_t h[4], o[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int k = k8 * 8 + 2 * u;
                        const float v0 = k < n ? col[k] - s0 : 0.f, v1 = k + 1 < n ? col[k + 1] - s0 : 0.f;
                        const __nv_bfloat16 h0 = __float2bfloat16_rn(v0), h1 = __float2bfloat16_rn(v1);
                        const __nv_bfloat16 l0 = __float2bfloat16_rn(v0 - __bfloat162float(h0));
                        const __nv_bfloat16 l1 = __float2bfloat16_rn(v1 - __bfloat162float(h1));
                        h[u] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
                        o[u] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
                    }
                    hi[k8] = make_uint4(h[0], h[1], h[2], h[3]);
                    lo[k8] = make_uint4(o[0], o[1], o[2], o[3]);
                }
            }
        }

        // 3. all-rows sums: D = X'X (R x R) and A = Q'X (LP x R, zero-padded Q) per SNP
        float acc[ACC];
#pragma unroll
        for (int u = 0; u < ACC; ++u) acc[u] = 0.f;
#pragma unroll 4
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            float qk[LP];
#pragma unroll
            for (int q4 = 0; q4 < LP / 4; ++q4) {
                const float4 v = __ldg(reinterpret_cast<const float4*>(A.Qr + (size_t)k * LP + 4 * q4));
                qk[4 * q4] = v.x; qk[4 * q4 + 1] = v.y; qk[4 * q4 + 2] = v.z; qk[4 * q4 + 3] = v.w;
            }
#pragma unroll
            for (int s = 0; s < SPBM; ++s) {
                if (s < nsnp) {
                    float x[R];
#pragma unroll
                    for (int a = 0; a < R; ++a) x[a] = xs[(size_t)(s * R + a) * nS + k] - cshift[s * R + a];
                    float* ac = acc + s * NA;
#pragma unroll
                    for (int a = 0; a < R; ++a)
#pragma unroll
                        for (int bb = 0; bb < R; ++bb) ac[a * R + bb] += x[a] * x[bb];
#pragma unroll
                    for (int qq = 0; qq < LP; ++qq)
#pragma unroll
                        for (int a = 0; a < R; ++a) ac[R * R + qq * R + a] += qk[qq] * x[a];
                }
            }
        }
        {
            for (int u = 0; u < NT; ++u) {
                const double v = warp_sum((double)acc[u]);
                if (lane == 0) red[w * NT + u] = v;
            }
            __syncthreads();
            for (int u = threadIdx.x; u < NT; u += blockDim.x) {
                double s = 0.0;
                for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) s += red[ww * NT + u];
                full[u] = s;
            }
            __syncthreads();
        }

        // 4. all-rows Schur complement per SNP: var_x of the SNP terms (src/Algorithm.cpp:665-670)
        if (threadIdx.x < nsnp) {
            const int s = threadIdx.x, i = i0 + s;
            const double* f = full + s * NA;
            double S[R * R];
#pragma unroll
            for (int a = 0; a < R; ++a)
#pragma unroll
                for (int bb = 0; bb < R; ++bb) {
                    double v = f[a * R + bb];
                    for (int qq = 0; qq < l; ++qq) v -= f[R * R + qq * R + a] * f[R * R + qq * R + bb];
                    S[a * R + bb] = v;
                }
            double dss[R];
#pragma unroll
            for (int a = 0; a < R; ++a) dss[a] = f[a * R + a];
            const bool ok = schur_inverse<R>(S, dss);
            fsing[s] = ok ? 0 : 1;
#pragma unroll
            for (int a = 0; a < R; ++a) A.varx[(size_t)i * R + a] = ok ? (float)S[a * R + a] : 0.f;
            if (A.sfinv)
#pragma unroll
                for (int u = 0; u < R * R; ++u) A.sfinv[(size_t)i * R * R + u] = ok ? S[u] : 0.0;
            if (A.afull)
                for (int u = 0; u < l * R; ++u) A.afull[(size_t)i * l * R + u] = (float)f[R * R + u];
        }
        __syncthreads();

        // 5. row-set sums (missing-row downdates and zero-row sums), then Schur per (pattern, SNP)
        for (int s0 = 0; s0 < A.nsets; s0 += A.sets_per_pass) {
            const int s1 = min(A.nsets, s0 + A.sets_per_pass);
            for (int set = s0 + w; set < s1; set += (int)(blockDim.x >> 5)) {
#pragma unroll
                for (int u = 0; u < ACC; ++u) acc[u] = 0.f;
                const int r0 = A.set_off[set], r1 = A.set_off[set + 1];
#pragma unroll 4
                for (int kk = r0 + lane; kk < r1; kk += 32) {
                    const int k = __ldg(A.rows + kk);
                    float qk[LP];
#pragma unroll
                    for (int q4 = 0; q4 < LP / 4; ++q4) {
                        const float4 v = __ldg(reinterpret_cast<const float4*>(A.qrows + (size_t)kk * LP + 4 * q4));
                        qk[4 * q4] = v.x; qk[4 * q4 + 1] = v.y; qk[4 * q4 + 2] = v.z; qk[4 * q4 + 3] = v.w;
                    }
#pragma unroll
                    for (int s = 0; s < SPBM; ++s) {
                        if (s < nsnp) {
                            float x[R];
#pragma unroll
                            for (int a = 0; a < R; ++a) x[a] = xs[(size_t)(s * R + a) * nS + k] - cshift[s * R + a];
                            float* ac = acc + s * NA;
#pragma unroll
                            for (int a = 0; a < R; ++a)
#pragma unroll
                                for (int bb = 0; bb < R; ++bb) ac[a * R + bb] += x[a] * x[bb];
#pragma unroll
                            for (int qq = 0; qq < LP; ++qq)
#pragma unroll
                                for (int a = 0; a < R; ++a) ac[R * R + qq * R + a] += qk[qq] * x[a];
                        }
                    }
                }
                float* dst = setacc + (size_t)(set - s0) * NT;
                for (int u = 0; u < NT; ++u) {
                    const float v = warp_sumf(acc[u]);
                    if (lane == 0) dst[u] = v;
                }
            }
            __syncthreads();
            // Schur complements of the patterns in this pass
            const int npat = max(0, min(s1, A.G) - s0);
            for (int idx = threadIdx.x; idx < npat * nsnp; idx += blockDim.x) {
                const int g2 = s0 + idx / nsnp, s = idx % nsnp, i = i0 + s;
                const double* f = full + s * NA;
                const float* d = setacc + (size_t)(g2 - s0) * NT + s * NA;
                double ao[OA_MAX_L * R];
                for (int u = 0; u < l * R; ++u) ao[u] = f[R * R + u] - (double)d[R * R + u];
                const double* Wg = A.W + (size_t)g2 * l * l;
                double S[R * R];
#pragma unroll
                for (int a = 0; a < R; ++a)
#pragma unroll
                    for (int bb = 0; bb < R; ++bb) S[a * R + bb] = f[a * R + bb] - (double)d[a * R + bb];
                double dso[R];
#pragma unroll
                for (int a = 0; a < R; ++a) dso[a] = S[a * R + a];
                for (int qq = 0; qq < l; ++qq) {
                    double wa[R];
#pragma unroll
                    for (int bb = 0; bb < R; ++bb) wa[bb] = 0.0;
                    for (int u = 0; u < l; ++u) {
                        const double wq = Wg[qq * l + u];
#pragma unroll
                        for (int bb = 0; bb < R; ++bb) wa[bb] += wq * ao[u * R + bb];
                    }
#pragma unroll
                    for (int a = 0; a < R; ++a)
#pragma unroll
                        for (int bb = 0; bb < R; ++bb) S[a * R + bb] -= ao[qq * R + a] * wa[bb];
                }
                const bool ok = !fsing[s] && !A.pat_bad[g2] && schur_inverse<R>(S, dso);
                const size_t gi = (size_t)g2 * A.mb + i;
                A.sing[gi] = ok ? 0 : 1;
#pragma unroll
                for (int u = 0; u < R * R; ++u) A.sinv[gi * R * R + u] = ok ? S[u] : 0.0;
                if (A.aobs)
                    for (int u = 0; u < l * R; ++u) A.aobs[gi * l * R + u] = (float)ao[u];
            }
            // zero sets in this pass
            const int zlo = max(s0, A.G);
            const int nz = max(0, s1 - zlo);
            for (int idx = threadIdx.x; idx < nz * nsnp; idx += blockDim.x) {
                const int set = zlo + idx / nsnp, s = idx % nsnp, i = i0 + s;
                const int z = set - A.G;
                const float* d = setacc + (size_t)(set - s0) * NT + s * NA;
                const size_t zi = (size_t)z * A.mb + i;
                for (int u = 0; u < l * R; ++u) A.zA[zi * l * R + u] = d[R * R + u];
#pragma unroll
                for (int u = 0; u < R * R; ++u) A.zD[zi * R * R + u] = d[u];
            }
            __syncthreads();
        }
        // single buffer: the next group's copy starts once this one is done
        if (BULK && A.nbuf == 1 && threadIdx.x == 0 && gn < ngroups) issue(gn, 0);
    }
    // a stopped CTA leaves no copy in flight behind it
    if (BULK && threadIdx.x == 0 && stop) {
        st_mbar_wait(&mbar[0], 0, true);
        st_mbar_wait(&mbar[0], 1, true);
        st_mbar_wait(&mbar[1], 0, true);
        st_mbar_wait(&mbar[1], 1, true);
    }
}

}  // namespace oa
