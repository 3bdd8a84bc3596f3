// Covariate terms (-i / --fdcov, ≙ the h < l iterations of hpc_statistics,
// src/Algorithm.cpp:1125-1194 with start_h = 1).
//
// With the SNP coefficients beta_x of a test known, the covariate
// coefficients in the orthonormal basis are beta_q = b0_j - W_g A_obs beta_x,
// and in the original covariate basis beta_XL = R^-1 beta_q (XL = Q R).
// Their var_x, like the reference's, comes from the all-rows inverse:
// diag(R^-1 (I + A_full Sf^-1 A_full') R^-T).
#pragma once
#include "oa_common.cuh"

namespace oa {

struct CovArgs {
    int n, l, r, p, mb;
    const int* tinv;       // original -> internal trait index
    const int* pat;
    const double* b0;      // [t][l]
    const double* W;       // [G][l][l]
    const float* aobs;     // [G][mb][l][r]
    const float* afull;    // [mb][l][r]
    const double* sfinv;   // [mb][r*r]
    const double* Rinv;    // [l][l] upper triangular, row-major
    const int* nobs;       // [t] (internal order)
    float min_t;
    int store_all;
    double min_p_disp;
};

__device__ __forceinline__ double dev_pvalue(double t) {
    if (t < 1.6) {
        const float t1 = (float)(4.4 - t);
        return 0.5 - 0.1 * (double)t1 * t;
    }
    return erfc(t * 0.70710678118654752440);
}

// beta, SE, |t| of covariate terms h = 1 .. l-1 of one test (j: internal trait index).
template <int R>
__device__ __forceinline__ void cov_eval(const CovArgs& C, int i, int j, const float* bx, float sig,
                                         float* ob, float* ose, float* ot) {
    const int l = C.l;
    const int g = C.pat[j];
    const size_t gi = (size_t)g * C.mb + i;
    const float* ao = C.aobs + gi * (size_t)(l * R);
    const float* af = C.afull + (size_t)i * l * R;
    const double* Sfi = C.sfinv + (size_t)i * R * R;
    const double* Wg = C.W + (size_t)g * l * l;
    double aob[OA_MAX_L], bq[OA_MAX_L];
    for (int q = 0; q < l; ++q) {
        double s = 0.0;
#pragma unroll
        for (int a = 0; a < R; ++a) s += (double)ao[q * R + a] * (double)bx[a];
        aob[q] = s;
    }
    for (int q = 0; q < l; ++q) {
        double s = 0.0;
        for (int u = 0; u < l; ++u) s += Wg[q * l + u] * aob[u];
        bq[q] = C.b0[(size_t)j * l + q] - s;
    }
    const double vf = (double)C.nobs[j] / (double)C.n;
    for (int h = 1; h < l; ++h) {
        double b = 0.0, v = 0.0, u[R];
#pragma unroll
        for (int a = 0; a < R; ++a) u[a] = 0.0;
        for (int k = h; k < l; ++k) {
            const double rk = C.Rinv[h * l + k];
            b += rk * bq[k];
            v += rk * rk;
#pragma unroll
            for (int a = 0; a < R; ++a) u[a] += rk * (double)af[k * R + a];
        }
#pragma unroll
        for (int a = 0; a < R; ++a)
#pragma unroll
            for (int c = 0; c < R; ++c) v += u[a] * Sfi[a * R + c] * u[c];
        const double se = (double)sig * sqrt(v * vf);
        ob[h] = (float)b;
        ose[h] = (float)se;
        ot[h] = (float)fabs(b / se);
    }
}

// Fill covariate terms of one chunk's records: [*first, counters[0]) (capped
// at the record buffer), read on the device after the chunk's GEMM.
template <int R>
__global__ void __launch_bounds__(256)
k_cov_terms(const RecOf<R>* __restrict__ rec, const unsigned long long* __restrict__ first_p,
            const unsigned long long* __restrict__ counters, long long cap, int snp_base, CovArgs C,
            float* __restrict__ cov /* [rec][l][3] */) {
    const long long first = (long long)*first_p;
    const long long last = min((long long)counters[0], cap);
    for (long long idx = first + blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < last;
         idx += (long long)gridDim.x * blockDim.x) {
        const RecOf<R> rc = rec[idx];
        if (rc.trait < 0) continue;   // an unused slot of a reserved block
        float b[OA_MAX_L], se[OA_MAX_L], t[OA_MAX_L];
        cov_eval<R>(C, rc.snp - snp_base, rc.tint, rc.b, rc.sig, b, se, t);
        float* o = cov + (size_t)idx * C.l * 3;
        o[0] = o[1] = o[2] = 0.f;
        for (int h = 1; h < C.l; ++h) {
            o[h * 3] = b[h];
            o[h * 3 + 1] = se[h];
            o[h * 3 + 2] = t[h];
        }
    }
}

// Significant covariate terms (P < min_p_disp) of tests that did not yield
// a stored row: the reference counts them in total_sig_results although
// their rows are dropped (src/Algorithm.cpp:1189-1192, 1197).
template <int R>
__global__ void __launch_bounds__(256)
k_cov_count(const float* __restrict__ d_beta, const float* __restrict__ d_t, const float* __restrict__ d_r2,
            const float* __restrict__ d_sig, long long dense_ld, int snp_base, int nsnp, int t,
            float min_r2, CovArgs C, unsigned long long* __restrict__ count) {
    const long long total = (long long)t * nsnp;
    unsigned long long mine = 0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(q / nsnp), i = (int)(q % nsnp);
        const size_t o = (size_t)j * dense_ld + snp_base + i;
        const float r2 = d_r2[o];
        if (isnan(r2)) continue;                           // RSS <= 0 or singular
        if (!(r2 > min_r2 || C.store_all)) continue;
        bool row = false;
        float bx[R];
#pragma unroll
        for (int a = 0; a < R; ++a) {
            bx[a] = d_beta[o * R + a];
            row |= (d_t[o * R + a] > C.min_t) || C.store_all;
        }
        if (row) continue;                                 // counted from the stored row
        float b[OA_MAX_L], se[OA_MAX_L], tt[OA_MAX_L];
        cov_eval<R>(C, i, C.tinv[j], bx, d_sig[o], b, se, tt);
        for (int h = 1; h < C.l; ++h)
            if ((tt[h] > C.min_t || C.store_all) && C.min_p_disp > dev_pvalue((double)tt[h])) ++mine;
    }
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(count, mine);
}

}  // namespace oa
