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
};

// Accumulators per SNP for R columns and LP (padded) covariates, and the
// largest number of SNPs a CTA handles so that they stay in registers.
__host__ __device__ constexpr int stats_na(int R, int LP) { return R * R + LP * R; }
__host__ __device__ constexpr int stats_spb_max(int R, int LP) {
    return (8 / R) < (64 / stats_na(R, LP)) ? (8 / R)
           : ((64 / stats_na(R, LP)) > 0 ? (64 / stats_na(R, LP)) : 1);
}
// Shared-memory layout of k_snp_stats: xs | full | red | setacc
__host__ __device__ inline size_t stats_smem_bytes(int R, int LP, int n, int spb, int sets_per_pass) {
    const int nS = (n + 3) & ~3;
    const int NT = spb * stats_na(R, LP);
    const int NR = NT > 16 ? NT : 16;
    return (size_t)spb * R * nS * 4 + (size_t)NT * 8 + (size_t)8 * NR * 8 + (size_t)sets_per_pass * NT * 4;
}

template <int R, int LP>
__global__ void __launch_bounds__(OA_NTHREADS)
k_snp_stats(StatsArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NA = stats_na(R, LP);            // accumulators per SNP
    constexpr int SPBM = stats_spb_max(R, LP);
    constexpr int ACC = SPBM * NA;
    const int n = A.n, l = A.l, spb = A.spb;
    const int nS = (n + 3) & ~3;
    const int i0 = blockIdx.x * spb;
    const int nsnp = min(spb, A.mb - i0);
    const int ncol = nsnp * R;
    const int NT = spb * NA;
    float* xs = reinterpret_cast<float*>(smem_raw);                      // [spb*R][nS]
    double* full = reinterpret_cast<double*>(xs + (size_t)spb * R * nS);  // [spb][NA]
    double* red = full + NT;                                              // [8][max(16, NT)]
    float* setacc = reinterpret_cast<float*>(red + 8 * (NT > 16 ? NT : 16));  // [sets_per_pass][spb][NA]
    __shared__ int fsing[8];
    __shared__ float cmean[8];
    __shared__ int cnan[8];

    // 1. stage the columns; NaN count and sum per column
    double vs[2 * 8];
#pragma unroll
    for (int q = 0; q < 16; ++q) vs[q] = 0.0;
    const bool vec = (A.ldx % 4 == 0) && ((reinterpret_cast<uintptr_t>(A.X) & 15) == 0) && (n % 4 == 0);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        if (c < ncol) {
            const float* src = A.X + (size_t)(i0 * R + c) * A.ldx;
            float* dst = xs + (size_t)c * nS;
            if (vec) {
                for (int k4 = threadIdx.x; k4 < n / 4; k4 += blockDim.x) {
                    const float4 v = __ldcs(reinterpret_cast<const float4*>(src) + k4);
                    reinterpret_cast<float4*>(dst)[k4] = v;
                    const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        if (isnan(e[u])) vs[8 + c] += 1.0;
                        else vs[c] += e[u];
                    }
                }
            } else {
                for (int k = threadIdx.x; k < n; k += blockDim.x) {
                    const float v = src[k];
                    dst[k] = v;
                    if (isnan(v)) vs[8 + c] += 1.0;
                    else vs[c] += v;
                }
            }
        }
    }
    block_sum<16>(vs, red);
    if (threadIdx.x < ncol) {
        const int c = threadIdx.x;
        const double cnt = vs[8 + c];
        const float mean = (float)(vs[c] / ((double)n - cnt));
        cmean[c] = mean;
        cnan[c] = cnt > 0.0 ? 1 : 0;
        A.mean[i0 * R + c] = cnt > 0.0 ? mean : 0.0f;
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
        for (int c = 0; c < ncol; ++c) {
            const float* col = xs + (size_t)c * nS;
            __nv_bfloat16* hi = A.Xhi + (size_t)(i0 * R + c) * A.n_pad;
            __nv_bfloat16* lo = A.Xlo + (size_t)(i0 * R + c) * A.n_pad;
            for (int k = threadIdx.x; k < A.n_pad; k += blockDim.x) {
                const float v = k < n ? col[k] : 0.0f;
                const __nv_bfloat16 h = __float2bfloat16_rn(v);
                hi[k] = h;
                lo[k] = __float2bfloat16_rn(v - __bfloat162float(h));
            }
        }
    }

    // 3. all-rows sums: D = X'X (R x R) and A = Q'X (LP x R, zero-padded Q) per SNP
    float acc[ACC];
#pragma unroll
    for (int q = 0; q < ACC; ++q) acc[q] = 0.f;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        float qk[LP];
#pragma unroll
        for (int q4 = 0; q4 < LP / 4; ++q4) {
            const float4 v = *reinterpret_cast<const float4*>(A.Qr + (size_t)k * LP + 4 * q4);
            qk[4 * q4] = v.x; qk[4 * q4 + 1] = v.y; qk[4 * q4 + 2] = v.z; qk[4 * q4 + 3] = v.w;
        }
#pragma unroll
        for (int s = 0; s < SPBM; ++s) {
            if (s < nsnp) {
                float x[R];
#pragma unroll
                for (int a = 0; a < R; ++a) x[a] = xs[(size_t)(s * R + a) * nS + k];
                float* ac = acc + s * NA;
#pragma unroll
                for (int a = 0; a < R; ++a)
#pragma unroll
                    for (int b = 0; b < R; ++b) ac[a * R + b] += x[a] * x[b];
#pragma unroll
                for (int q = 0; q < LP; ++q)
#pragma unroll
                    for (int a = 0; a < R; ++a) ac[R * R + q * R + a] += qk[q] * x[a];
            }
        }
    }
    {
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        for (int q = 0; q < NT; ++q) {
            const double v = warp_sum((double)acc[q]);
            if (lane == 0) red[w * NT + q] = v;
        }
        __syncthreads();
        for (int q = threadIdx.x; q < NT; q += blockDim.x) {
            double s = 0.0;
            for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) s += red[ww * NT + q];
            full[q] = s;
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
            for (int b = 0; b < R; ++b) {
                double v = f[a * R + b];
                for (int q = 0; q < l; ++q) v -= f[R * R + q * R + a] * f[R * R + q * R + b];
                S[a * R + b] = v;
            }
        const bool ok = spd_inverse<R>(S, R, 1e-9);
        fsing[s] = ok ? 0 : 1;
#pragma unroll
        for (int a = 0; a < R; ++a) A.varx[(size_t)i * R + a] = ok ? (float)S[a * R + a] : 0.f;
        if (A.sfinv)
#pragma unroll
            for (int q = 0; q < R * R; ++q) A.sfinv[(size_t)i * R * R + q] = ok ? S[q] : 0.0;
        if (A.afull)
            for (int q = 0; q < l * R; ++q) A.afull[(size_t)i * l * R + q] = (float)f[R * R + q];
    }
    __syncthreads();

    // 5. row-set sums (missing-row downdates and zero-row sums), then Schur per (pattern, SNP)
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int s0 = 0; s0 < A.nsets; s0 += A.sets_per_pass) {
        const int s1 = min(A.nsets, s0 + A.sets_per_pass);
        for (int set = s0 + w; set < s1; set += (int)(blockDim.x >> 5)) {
#pragma unroll
            for (int q = 0; q < ACC; ++q) acc[q] = 0.f;
            const int r0 = A.set_off[set], r1 = A.set_off[set + 1];
            for (int kk = r0 + lane; kk < r1; kk += 32) {
                const int k = A.rows[kk];
                float qk[LP];
#pragma unroll
                for (int q4 = 0; q4 < LP / 4; ++q4) {
                    const float4 v = *reinterpret_cast<const float4*>(A.Qr + (size_t)k * LP + 4 * q4);
                    qk[4 * q4] = v.x; qk[4 * q4 + 1] = v.y; qk[4 * q4 + 2] = v.z; qk[4 * q4 + 3] = v.w;
                }
#pragma unroll
                for (int s = 0; s < SPBM; ++s) {
                    if (s < nsnp) {
                        float x[R];
#pragma unroll
                        for (int a = 0; a < R; ++a) x[a] = xs[(size_t)(s * R + a) * nS + k];
                        float* ac = acc + s * NA;
#pragma unroll
                        for (int a = 0; a < R; ++a)
#pragma unroll
                            for (int b = 0; b < R; ++b) ac[a * R + b] += x[a] * x[b];
#pragma unroll
                        for (int q = 0; q < LP; ++q)
#pragma unroll
                            for (int a = 0; a < R; ++a) ac[R * R + q * R + a] += qk[q] * x[a];
                    }
                }
            }
            float* dst = setacc + (size_t)(set - s0) * NT;
            for (int q = 0; q < NT; ++q) {
                const float v = warp_sumf(acc[q]);
                if (lane == 0) dst[q] = v;
            }
        }
        __syncthreads();
        // Schur complements of the patterns in this pass
        const int npat = max(0, min(s1, A.G) - s0);
        for (int idx = threadIdx.x; idx < npat * nsnp; idx += blockDim.x) {
            const int g = s0 + idx / nsnp, s = idx % nsnp, i = i0 + s;
            const double* f = full + s * NA;
            const float* d = setacc + (size_t)(g - s0) * NT + s * NA;
            double ao[OA_MAX_L * R];
            for (int q = 0; q < l * R; ++q) ao[q] = f[R * R + q] - (double)d[R * R + q];
            const double* Wg = A.W + (size_t)g * l * l;
            double S[R * R];
#pragma unroll
            for (int a = 0; a < R; ++a)
#pragma unroll
                for (int b = 0; b < R; ++b) S[a * R + b] = f[a * R + b] - (double)d[a * R + b];
            for (int q = 0; q < l; ++q) {
                double wa[R];
#pragma unroll
                for (int b = 0; b < R; ++b) wa[b] = 0.0;
                for (int u = 0; u < l; ++u) {
                    const double wq = Wg[q * l + u];
#pragma unroll
                    for (int b = 0; b < R; ++b) wa[b] += wq * ao[u * R + b];
                }
#pragma unroll
                for (int a = 0; a < R; ++a)
#pragma unroll
                    for (int b = 0; b < R; ++b) S[a * R + b] -= ao[q * R + a] * wa[b];
            }
            const bool ok = !fsing[s] && !A.pat_bad[g] && spd_inverse<R>(S, R, 1e-9);
            const size_t gi = (size_t)g * A.mb + i;
            A.sing[gi] = ok ? 0 : 1;
#pragma unroll
            for (int q = 0; q < R * R; ++q) A.sinv[gi * R * R + q] = ok ? S[q] : 0.0;
            if (A.aobs)
                for (int q = 0; q < l * R; ++q) A.aobs[gi * l * R + q] = (float)ao[q];
        }
        // zero sets in this pass
        const int zlo = max(s0, A.G);
        const int nz = max(0, s1 - zlo);
        for (int idx = threadIdx.x; idx < nz * nsnp; idx += blockDim.x) {
            const int set = zlo + idx / nsnp, s = idx % nsnp, i = i0 + s;
            const int z = set - A.G;
            const float* d = setacc + (size_t)(set - s0) * NT + s * NA;
            const size_t zi = (size_t)z * A.mb + i;
            for (int q = 0; q < l * R; ++q) A.zA[zi * l * R + q] = d[R * R + q];
#pragma unroll
            for (int q = 0; q < R * R; ++q) A.zD[zi * R * R + q] = d[q];
        }
        __syncthreads();
    }
}

}  // namespace oa
