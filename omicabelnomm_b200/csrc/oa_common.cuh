// Shared device helpers and engine-internal types of the B200 association engine.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include "omicabel_b200.h"

#define OA_NTHREADS 256

namespace oa {
constexpr int EMIT_BLOCK = 128;   // record slots a tensor-core epilogue warp reserves at a time
constexpr int EPI_WARPS_TC = 8;   // epilogue warps per tensor-core GEMM CTA (each holds one reserved block)
}
#define OA_SETS_MAX 4096   // row sets (missingness patterns + zero sets) per trait block

namespace oa {

// Per-trait constants of the epilogue, gathered once per tile.
struct TraitP {
    double rss0;
    float a_r2, inv_ncorr, vf;
    int g, zs, orig;
};

// One stored row (a (trait, SNP) test with at least one stored SNP term),
// the device form of the reference's resultH (src/Definitions.h:271-280),
// with room for K SNP terms: K = 4 (80 bytes) up to four columns per SNP,
// K = 8 (128 bytes) for five to eight.
template <int K>
struct alignas(16) RecK {
    int32_t trait;      // trait index within the trait block
    int32_t snp;        // SNP index within the SNP block
    float r2;           // R2 (src/Algorithm.cpp:1092)
    uint32_t mask;      // bit a: SNP term a (coefficient h = l + a) stored
    float sig;          // sqrt(RSS / n_corrected) (src/Algorithm.cpp:1100)
    int32_t tint;       // trait index in the engine's internal (pattern-sorted) order
    float pad[2];
    float b[K];
    float se[K];
    float t[K];
};
using Rec = RecK<4>;
static_assert(sizeof(RecK<4>) == 80 && sizeof(RecK<8>) == 128, "Rec layout");
// The record of an engine with R columns per SNP.
template <int R>
using RecOf = RecK<(R <= 4 ? 4 : 8)>;
// Rec-sized slots one record of an engine with r columns per SNP takes.
inline int rec_slots(int r) { return r <= 4 ? 1 : 2; }

// Everything the fused statistics epilogue reads, per trait and per SNP.
// Per-trait arrays are in the engine's internal trait order (traits sorted
// by missingness pattern, so consecutive traits share their Schur tables).
struct EpiArgs {
    int n, l, r, p, mb, G;
    // per trait
    const int* pat;          // missingness pattern of the trait
    const int* zset;         // zero set of the trait or -1
    const int* tperm;        // internal -> original trait index
    const double* rss0;      // RSS of the covariate-only fit over observed rows
    const float* a_r2;       // (n-1) / ((n_corr-1) SST): R2 = 1 - RSS a_r2 (src/Algorithm.cpp:1092)
    const float* inv_ncorr;  // 1 / n_corr (src/Algorithm.cpp:1100)
    const float* vf;         // (n - miss) / n, the reference's varFactor (src/Algorithm.cpp:1052)
    const double* b0;        // covariate-only coefficients in the orthonormal basis [t][l]
    // per SNP (and pattern)
    const double* sinv;      // inverse Schur complement per (pattern, SNP): [G][mb][r*r]
    const float* varx;       // diag of the all-rows inverse for the SNP terms [mb][r]
    const uint8_t* sing;     // singular flag per (pattern, SNP) [G][mb]
    const float* aobs;       // Q_obs' X per (pattern, SNP) [G][mb][l][r]  (zero-set path)
    const float* zA;         // per (zero set, SNP) sum over zero rows of q x' [Z][mb][l][r]
    const float* zD;         // per (zero set, SNP) sum over zero rows of x x' [Z][mb][r][r]
    const double* zQ;        // per zero set sum of q q' [Z][l][l]
    const double* W;         // (Q_obs'Q_obs)^-1 per pattern [G][l][l]
    const float* qdel;       // the reference's r >= 2 downdate (quirk mode) per (pattern, SNP) [G][mb][l][r], or null
    const double* qK;        // its RSS Gram term per (pattern, SNP) [G][mb][r][r], or null
    // thresholds
    float min_r2, min_t;
    int store_all;
    // outputs
    void* rec;                       // RecOf<R> records
    unsigned long long* rec_count;   // record slots handed out (written rows and unused slots of reserved blocks)
    unsigned long long* rec_valid;   // rows written (null: not counted)
    long long cap;
    unsigned long long* n_singular;
    // dense outputs (optional): beta/se/t [t][mb][r], r2 [t][mb], sig [t][mb]
    float* d_beta;
    float* d_se;
    float* d_t;
    float* d_r2;
    float* d_sig;
    uint8_t* d_flags;        // per-test status bits [t][mb] (OA_TEST_*), or null
    int t;
    int snp_base;            // index of the block's first SNP within the API call
    long long dense_ld;      // SNPs per trait row of the dense outputs
};

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    // splitmix64 finaliser (Steele, Lea, Flood 2014)
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// In-place inverse of a small SPD matrix (row-major k x k, k <= OA_MAX_R or
// OA_MAX_L) by Cholesky.  Returns false if a pivot is not positive
// relative to the diagonal scale (the system is treated as singular).
template <int K>
__device__ __host__ inline bool spd_inverse(double* A, int k, double rel_tol) {
    double L[K * K];
    double dmax = 0.0;
    for (int i = 0; i < k; ++i) dmax = fmax(dmax, fabs(A[i * k + i]));
    if (!(dmax > 0.0)) return false;
    for (int i = 0; i < k * k; ++i) L[i] = 0.0;
    for (int j = 0; j < k; ++j) {
        double s = A[j * k + j];
        for (int q = 0; q < j; ++q) s -= L[j * k + q] * L[j * k + q];
        if (!(s > rel_tol * fmax(fabs(A[j * k + j]), 1e-300))) return false;
        double d = sqrt(s);
        L[j * k + j] = d;
        for (int i = j + 1; i < k; ++i) {
            double u = A[i * k + j];
            for (int q = 0; q < j; ++q) u -= L[i * k + q] * L[j * k + q];
            L[i * k + j] = u / d;
        }
    }
    // inverse of L (lower), then A^-1 = L^-T L^-1
    double Li[K * K];
    for (int i = 0; i < k * k; ++i) Li[i] = 0.0;
    for (int i = 0; i < k; ++i) {
        Li[i * k + i] = 1.0 / L[i * k + i];
        for (int j = 0; j < i; ++j) {
            double s = 0.0;
            for (int q = j; q < i; ++q) s += L[i * k + q] * Li[q * k + j];
            Li[i * k + j] = -s / L[i * k + i];
        }
    }
    for (int i = 0; i < k; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = 0.0;
            for (int q = i; q < k; ++q) s += Li[q * k + i] * Li[q * k + j];
            A[i * k + j] = s;
            A[j * k + i] = s;
        }
    return true;
}

// A SNP column whose residual sum of squares after the covariates (the
// diagonal of its Schur complement) is below this fraction of its own sum of
// squares over the same rows is taken as collinear with the covariates: the
// test is singular.  The sums are accumulated in FP32 (relative rounding about
// 1e-7), so an exactly collinear column (monomorphic on the observed rows, or
// equal to a covariate) leaves a residual of about 1e-7 of its sum of squares,
// while a real SNP keeps almost all of it (1 - R2 of the SNP on the covariates).
constexpr double SCHUR_SING_REL = 1e-5;

// Inverse of the r x r Schur complement S of a test (in place); false if the
// system is singular: a column collinear with the covariates (S_aa at or below
// SCHUR_SING_REL of dss[a], the column's sum of squares over the same rows) or
// SNP columns collinear among themselves (a Cholesky pivot at or below 1e-9 of
// its diagonal).
template <int R>
__device__ __host__ inline bool schur_inverse(double* S, const double* dss) {
    for (int a = 0; a < R; ++a)
        if (!(S[a * R + a] > SCHUR_SING_REL * dss[a])) return false;
    return spd_inverse<R>(S, R, 1e-9);
}

}  // namespace oa
