// Plain-FP32 form of the dominant contraction, XR' Y~ (≙ the Ay_bot sgemm,
// src/Algorithm.cpp:705-707), as a SIMT FFMA GEMM with the per-test
// statistics fused into its epilogue: no SNP x trait matrix is ever written.
//
// C[c][j] = sum_k X[c][k] * Y~[j][k]: both operands are K-contiguous (the
// individual index k is contiguous in a .fvd column).  Tile 128 (SNP
// columns) x 128 (traits) x 16 (k), 256 threads, 8x8 accumulators per
// thread, register-staged double buffering through shared memory.
#pragma once
#include "oa_epilogue.cuh"

namespace oa {

constexpr int SG_BM = 128, SG_BN = 128, SG_BK = 16, SG_PAD = 4;

// Four consecutive k of row `row`.  fix: dosage columns, where NaN is the
// column mean (center = 0: NaN -> mean[row]) or every value is taken
// relative to the column mean (center = 1: x -> x - mean[row], NaN -> 0).
template <bool VEC>
__device__ __forceinline__ void sg_load(const float* __restrict__ P, size_t ld, int nrow, int K,
                                        int row, int k, const float* __restrict__ mean, bool fix, bool center,
                                        float (&v)[4]) {
    if (row < nrow) {
        const float* src = P + (size_t)row * ld + k;
        if (VEC && k + 3 < K) {
            const float4 q = __ldg(reinterpret_cast<const float4*>(src));
            v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
        } else {
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = (k + u < K) ? __ldg(src + u) : 0.f;
        }
        if (fix) {
            const float mv = mean[row];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const float c = center ? (isnan(v[u]) ? 0.f : v[u] - mv) : (isnan(v[u]) ? mv : v[u]);
                v[u] = (k + u < K) ? c : 0.f;
            }
        }
    } else {
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = 0.f;
    }
}

// STORE = false: fused statistics epilogue.  STORE = true: the product is
// written out transposed, C[col * ldc + row] (the pre-GEMM of the per-SNP
// covariate sums); with kspan > 0 the CTAs of blockIdx.z = 1 take K from
// kspan on and write their partial product to cpart (summed into cout by
// k_add_partial, in that fixed order), those of z = 0 take K below kspan.
template <int R, bool VEC, bool STORE>
__global__ void __launch_bounds__(256, 2)
k_gemm_simt(const float* __restrict__ X, size_t ldx, int xrows, const float* __restrict__ Yt, size_t ldy,
            int t, int K, const float* __restrict__ colmean, const int* __restrict__ has_nan, int center, EpiArgs E,
            float* __restrict__ cout, int ldc, float* __restrict__ cpart, int kspan) {
    __shared__ __align__(16) float As[2][SG_BK][SG_BM + SG_PAD];
    __shared__ __align__(16) float Bs[2][SG_BK][SG_BN + SG_PAD];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int m0 = blockIdx.y * SG_BM;  // first SNP column of the tile
    const int n0 = blockIdx.x * SG_BN;  // first trait of the tile
    const int lrow = tid >> 2, lk = (tid & 3) * 4;
    const bool fix = center || *has_nan != 0;
    const bool split = STORE && kspan > 0;
    const int kb = split ? (int)blockIdx.z * kspan : 0;   // this CTA's K range [kb, ke)
    const int ke = split ? min(K, kb + kspan) : K;

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

    float ra[2][4], rb[2][4];
    auto gload = [&](int k0) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            sg_load<VEC>(X, ldx, xrows, ke, m0 + lrow + 64 * h, k0 + lk, colmean, fix, center != 0, ra[h]);
            sg_load<VEC>(Yt, ldy, t, ke, n0 + lrow + 64 * h, k0 + lk, colmean, false, false, rb[h]);
        }
    };
    auto sstore = [&](int buf) {
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                As[buf][lk + u][lrow + 64 * h] = ra[h][u];
                Bs[buf][lk + u][lrow + 64 * h] = rb[h][u];
            }
    };

    const int nk = (ke - kb + SG_BK - 1) / SG_BK;
    gload(kb);
    sstore(0);
    __syncthreads();
    for (int kt = 0; kt < nk; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < nk) gload(kb + (kt + 1) * SG_BK);
#pragma unroll
        for (int kk = 0; kk < SG_BK; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][kk][64 + ty * 4]);
            const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][kk][64 + tx * 4]);
            const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        if (kt + 1 < nk) sstore(buf ^ 1);
        __syncthreads();
    }

    if constexpr (STORE) {
        float* __restrict__ out = (split && blockIdx.z == 1) ? cpart : cout;
#pragma unroll
        for (int ii = 0; ii < 8; ++ii) {
            const int row = m0 + (ii < 4 ? ty * 4 + ii : 64 + ty * 4 + (ii - 4));
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
                const int col = n0 + (jj < 4 ? tx * 4 + jj : 64 + tx * 4 + (jj - 4));
                if (row < xrows && col < t) out[(size_t)col * ldc + row] = acc[ii][jj];
            }
        }
    } else {
        // fused epilogue: rows ty*4+{0..3} and 64+ty*4+{0..3}; a SNP's R columns
        // are consecutive rows held by this thread (R divides 4), or, with
        // R = 8, by this thread (even ty) and the thread of ty + 1 (lane + 16 of
        // the same warp), whose rows come over by shuffle
        if constexpr (R <= 4) {
#pragma unroll
            for (int half = 0; half < 2; ++half) {
#pragma unroll
                for (int sg = 0; sg < 4 / R; ++sg) {
                    const int row0 = m0 + 64 * half + ty * 4 + sg * R;
                    const int i = row0 / R;  // SNP within the block
#pragma unroll
                    for (int jj = 0; jj < 8; ++jj) {
                        const int j = n0 + (jj < 4 ? tx * 4 + jj : 64 + tx * 4 + (jj - 4));
                        float z[R];
#pragma unroll
                        for (int a = 0; a < R; ++a) z[a] = acc[half * 4 + sg * R + a][jj];
                        RecOf<R> rc;
                        const bool st = epi_eval<R>(E, i, j, z, (row0 < xrows) && (j < t), rc);
                        epi_emit<R>(E, st, rc);
                    }
                }
            }
        } else {
            static_assert(R == 8, "SNP column groups of 1, 2, 4 or 8");
            const bool lead = (ty & 1) == 0;
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int row0 = m0 + 64 * half + ty * 4;
                const int i = row0 / R;
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) {
                    const int j = n0 + (jj < 4 ? tx * 4 + jj : 64 + tx * 4 + (jj - 4));
                    float z[R];
#pragma unroll
                    for (int a = 0; a < 4; ++a) {
                        z[a] = acc[half * 4 + a][jj];
                        z[4 + a] = __shfl_down_sync(0xffffffffu, acc[half * 4 + a][jj], 16);
                    }
                    RecOf<R> rc;
                    const bool st = epi_eval<R>(E, i, j, z, lead && (row0 < xrows) && (j < t), rc);
                    epi_emit<R>(E, st, rc);
                }
            }
        }
    }
}

// The second K half of a split store-form product:
// C[col * ldc + row] += Cpart[col * ldc + row] for the rows < xrows of each of
// the c2 columns (a partial last chunk leaves rows [xrows, ldc) unwritten).
__global__ void __launch_bounds__(256) k_add_partial(float* __restrict__ cout, const float* __restrict__ cpart,
                                                     int c2, int xrows, int ldc) {
    const long long n = (long long)c2 * xrows;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const long long i = (q / xrows) * ldc + q % xrows;
        cout[i] += cpart[i];
    }
}

}  // namespace oa
