// Trait-block and SNP-block preparation kernels (bandwidth-bound work).
//
//  k_trait_stats  per trait: missing count, sums, zero count, missing-set
//                 hashes, Q'y  (≙ replace_nans + sumSquares + XL'Y,
//                 src/Utility.cpp:329-378, src/Algorithm.cpp:558-585, 1222-1251)
//  k_trait_set_check, k_trait_masks
//                 exact check of the grouping by hash sums; row masks for
//                 the exact regrouping after a collision
//  k_set_rows     ordered row list of each row set (missing pattern / zero set)
//  k_set_gram     per pattern W = (Q_obs'Q_obs)^-1, per zero set sum q q'
//                 (≙ generate_correction_missings_Stl, src/Algorithm.cpp:1324-1362)
//  k_trait_resid  y~ = y - Q_obs W Q'y on observed rows, RSS0, SST
//  k_snp_stats    per SNP column: NaN mean-imputation, X'X diagonal block,
//                 Q'X, missing-row downdates per row set, FP64 Schur
//                 complements and their inverses per (pattern, SNP)
//                 (≙ replace_nans_avgs, Str/Sbr, var_x, Str/Sbr corrections:
//                 src/Utility.cpp:302-326, src/Algorithm.cpp:618-689, 1260-1315)
#pragma once
#include "oa_stats.cuh"

namespace oa {

struct TraitStatsOut {
    double* sums;               // [t][2 + OA_MAX_L]: sum y, sum y^2, Q'y
    int* counts;                // [t][2]: missing, observed zeros
    unsigned long long* hashes; // [t][4]: missing h1 h2, zero h1 h2
};

static __global__ void __launch_bounds__(OA_NTHREADS)
k_trait_stats(const float* __restrict__ Y, size_t ldy, int n, int l, const double* __restrict__ Q64,
              TraitStatsOut out) {
    __shared__ double red[8 * (2 + OA_MAX_L)];
    __shared__ unsigned long long hred[8 * 4];
    __shared__ int cred[8 * 2];
    const int j = blockIdx.x;
    const float* y = Y + (size_t)j * ldy;
    double v[2 + OA_MAX_L];
#pragma unroll
    for (int q = 0; q < 2 + OA_MAX_L; ++q) v[q] = 0.0;
    int miss = 0, zc = 0;
    unsigned long long h1 = 0, h2 = 0, z1 = 0, z2 = 0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const float x = y[k];
        if (isnan(x)) {
            ++miss;
            h1 += mix64((unsigned long long)k);
            h2 += mix64((unsigned long long)k ^ 0xa5a5a5a55a5a5a5aULL);
        } else {
            v[0] += (double)x;
            v[1] += (double)x * (double)x;
            if (x == 0.0f) {
                ++zc;
                z1 += mix64((unsigned long long)k);
                z2 += mix64((unsigned long long)k ^ 0xa5a5a5a55a5a5a5aULL);
            }
#pragma unroll
            for (int q = 0; q < OA_MAX_L; ++q)
                if (q < l) v[2 + q] += Q64[(size_t)q * n + k] * (double)x;
        }
    }
    block_sum<2 + OA_MAX_L>(v, red);
    // integer and hash sums (addition is order independent: deterministic)
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        miss += __shfl_xor_sync(0xffffffffu, miss, o);
        zc += __shfl_xor_sync(0xffffffffu, zc, o);
        h1 += __shfl_xor_sync(0xffffffffu, h1, o);
        h2 += __shfl_xor_sync(0xffffffffu, h2, o);
        z1 += __shfl_xor_sync(0xffffffffu, z1, o);
        z2 += __shfl_xor_sync(0xffffffffu, z2, o);
    }
    if (lane == 0) {
        cred[w * 2] = miss;
        cred[w * 2 + 1] = zc;
        hred[w * 4] = h1;
        hred[w * 4 + 1] = h2;
        hred[w * 4 + 2] = z1;
        hred[w * 4 + 3] = z2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int cm = 0, cz = 0;
        unsigned long long a = 0, b = 0, c = 0, d = 0;
        for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) {
            cm += cred[ww * 2];
            cz += cred[ww * 2 + 1];
            a += hred[ww * 4];
            b += hred[ww * 4 + 1];
            c += hred[ww * 4 + 2];
            d += hred[ww * 4 + 3];
        }
        out.counts[j * 2] = cm;
        out.counts[j * 2 + 1] = cz;
        out.hashes[j * 4] = a;
        out.hashes[j * 4 + 1] = b;
        out.hashes[j * 4 + 2] = c;
        out.hashes[j * 4 + 3] = d;
        for (int q = 0; q < 2 + OA_MAX_L; ++q) out.sums[(size_t)j * (2 + OA_MAX_L) + q] = v[q];
    }
}

// Ordered list of the rows of each row set.  kind 0: NaN rows of the
// representative trait (a missingness pattern); kind 1: observed rows
// whose value is exactly 0 (a zero set).
static __global__ void __launch_bounds__(OA_NTHREADS)
k_set_rows(const float* __restrict__ Y, size_t ldy, int n, const int* __restrict__ set_rep,
           const int* __restrict__ set_kind, const int* __restrict__ set_off, int* __restrict__ rows) {
    __shared__ int wcount[8];
    __shared__ int wbase[8];
    __shared__ int total;
    const int s = blockIdx.x;
    const float* y = Y + (size_t)set_rep[s] * ldy;
    const int kind = set_kind[s];
    int* out = rows + set_off[s];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int base = 0;
    for (int c0 = 0; c0 < n; c0 += blockDim.x) {
        const int k = c0 + threadIdx.x;
        bool pred = false;
        if (k < n) {
            const float x = y[k];
            pred = kind == 0 ? isnan(x) : (x == 0.0f);
        }
        const unsigned m = __ballot_sync(0xffffffffu, pred);
        if (lane == 0) wcount[w] = __popc(m);
        __syncthreads();
        if (threadIdx.x == 0) {
            int acc = 0;
            for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) {
                wbase[ww] = acc;
                acc += wcount[ww];
            }
            total = acc;
        }
        __syncthreads();
        if (pred) out[base + wbase[w] + __popc(m & ((1u << lane) - 1u))] = k;
        base += total;
        __syncthreads();
    }
}

// Exact check of the trait grouping by hash sums: trait j's NaN rows must be
// those of its pattern's representative rep[2 j], and when rep[2 j + 1] >= 0
// its observed exact-zero rows those of its zero set's representative.  Any
// difference sets *bad (the host then groups the traits on their row masks).
static __global__ void __launch_bounds__(OA_NTHREADS)
k_trait_set_check(const float* __restrict__ Y, size_t ldy, int n, const int* __restrict__ rep, int* bad) {
    const int j = blockIdx.x;
    const float* y = Y + (size_t)j * ldy;
    const float* yp = Y + (size_t)rep[2 * j] * ldy;
    const int zr = rep[2 * j + 1];
    const float* yz = Y + (size_t)(zr >= 0 ? zr : j) * ldy;
    int diff = 0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const float x = y[k];
        diff |= isnan(x) != isnan(yp[k]);
        if (zr >= 0) diff |= (x == 0.0f) != (yz[k] == 0.0f);
    }
    if (__syncthreads_or(diff) && threadIdx.x == 0) atomicOr(bad, 1);
}

// Row masks of each trait, 32 rows per word: masks[(2 j) nw + w] bit b set
// when row 32 w + b is NaN, masks[(2 j + 1) nw + w] when it is an observed 0.
static __global__ void __launch_bounds__(OA_NTHREADS)
k_trait_masks(const float* __restrict__ Y, size_t ldy, int n, int nw, unsigned* __restrict__ masks) {
    const int j = blockIdx.x;
    const float* y = Y + (size_t)j * ldy;
    const int lane = threadIdx.x & 31;
    for (int k0 = (threadIdx.x >> 5) * 32; k0 < nw * 32; k0 += blockDim.x) {   // one 32-row word per warp
        const int k = k0 + lane;
        const float x = k < n ? y[k] : 1.0f;
        const unsigned mn = __ballot_sync(0xffffffffu, isnan(x));
        const unsigned mz = __ballot_sync(0xffffffffu, x == 0.0f);
        if (lane == 0) {
            masks[(size_t)(2 * j) * nw + k0 / 32] = mn;
            masks[(size_t)(2 * j + 1) * nw + k0 / 32] = mz;
        }
    }
}

// Per row set: G = sum over the set's rows of q q' (FP64).  Patterns store
// W = (I - G)^-1 (Q orthonormal over all rows, so Q_obs'Q_obs = I - G);
// zero sets store G.  sing_out[s] = 1 if I - G is not positive definite.
static __global__ void __launch_bounds__(OA_NTHREADS)
k_set_gram(const double* __restrict__ Q64, int n, int l, const int* __restrict__ set_kind,
           const int* __restrict__ set_off, const int* __restrict__ rows, double* __restrict__ W,
           double* __restrict__ zQ, const int* __restrict__ set_slot, uint8_t* __restrict__ pat_bad) {
    __shared__ double G[OA_MAX_L * OA_MAX_L];
    const int s = blockIdx.x;
    const int r0 = set_off[s], r1 = set_off[s + 1];
    const int npair = l * l;
    for (int pq = threadIdx.x; pq < npair; pq += blockDim.x) {
        const int a = pq / l, b = pq % l;
        double acc = 0.0;
        if (b <= a)
            for (int k = r0; k < r1; ++k) {
                const int row = rows[k];
                acc += Q64[(size_t)a * n + row] * Q64[(size_t)b * n + row];
            }
        G[pq] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int a = 0; a < l; ++a)
            for (int b = a + 1; b < l; ++b) G[a * l + b] = G[b * l + a];
        const int slot = set_slot[s];
        if (set_kind[s] == 1) {
            for (int q = 0; q < l * l; ++q) zQ[(size_t)slot * l * l + q] = G[q];
        } else {
            double A[OA_MAX_L * OA_MAX_L];
            for (int a = 0; a < l; ++a)
                for (int b = 0; b < l; ++b) A[a * l + b] = (a == b ? 1.0 : 0.0) - G[a * l + b];
            const bool ok = spd_inverse<OA_MAX_L>(A, l, 1e-12);
            pat_bad[slot] = ok ? 0 : 1;
            for (int q = 0; q < l * l; ++q) W[(size_t)slot * l * l + q] = ok ? A[q] : 0.0;
        }
    }
}

// y~ = y - Q b0 on observed rows (0 on missing rows), b0 = W Q'y.
// Block jj builds internal trait jj = original trait tperm[jj] (traits are
// kept sorted by missingness pattern inside the engine).  Writes Y~ (FP32,
// and BF16 hi/lo for the tensor-core form), RSS0, SST and the constants the
// epilogue folds: a_r2 = (n-1)/((n_corr-1) SST), 1/n_corr, (n-miss)/n.
static __global__ void __launch_bounds__(OA_NTHREADS)
k_trait_resid(const float* __restrict__ Y, size_t ldy, int n, int n_pad, int l, int p,
              const double* __restrict__ Q64, const double* __restrict__ sums,
              const int* __restrict__ counts, const int* __restrict__ pat,
              const double* __restrict__ W, const int* __restrict__ tperm, float* __restrict__ Yt,
              __nv_bfloat16* __restrict__ Yhi, __nv_bfloat16* __restrict__ Ylo,
              double* __restrict__ rss0, float* __restrict__ sst, int* __restrict__ nobs,
              double* __restrict__ b0out, float* __restrict__ a_r2, float* __restrict__ inv_ncorr,
              float* __restrict__ vf) {
    __shared__ double b0[OA_MAX_L];
    __shared__ double red[8];
    const int jj = blockIdx.x;
    const int j = tperm[jj];
    const double* sj = sums + (size_t)j * (2 + OA_MAX_L);
    if (threadIdx.x < l) {
        const double* Wg = W + (size_t)pat[jj] * l * l;
        double acc = 0.0;
        for (int b = 0; b < l; ++b) acc += Wg[threadIdx.x * l + b] * sj[2 + b];
        b0[threadIdx.x] = acc;
        b0out[(size_t)jj * l + threadIdx.x] = acc;
    }
    __syncthreads();
    const float* y = Y + (size_t)j * ldy;
    float* out = Yt + (size_t)jj * n_pad;
    double rss = 0.0;
    for (int k = threadIdx.x; k < n_pad; k += blockDim.x) {
        float e = 0.0f;
        if (k < n) {
            const float x = y[k];
            if (!isnan(x)) {
                double fit = 0.0;
                for (int q = 0; q < l; ++q) fit += Q64[(size_t)q * n + k] * b0[q];
                const double d = (double)x - fit;
                rss += d * d;
                e = (float)d;
            }
        }
        out[k] = e;
        if (Yhi) {
            const __nv_bfloat16 hi = __float2bfloat16_rn(e);
            Yhi[(size_t)jj * n_pad + k] = hi;
            Ylo[(size_t)jj * n_pad + k] = __float2bfloat16_rn(e - __bfloat162float(hi));
        }
    }
    rss = warp_sum(rss);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = rss;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        rss0[jj] = s;
        const int no = n - counts[j * 2];
        nobs[jj] = no;
        // the reference holds SST in long double and stores it as float (src/Algorithm.cpp:1227-1240)
        const float sstf = (float)(sj[1] - sj[0] * sj[0] / (double)no);
        sst[jj] = sstf;
        const int ncorr = no - p;
        a_r2[jj] = (float)((double)(n - 1) / ((double)(ncorr - 1) * (double)sstf));
        inv_ncorr[jj] = (float)(1.0 / (double)ncorr);
        vf[jj] = (float)((double)no / (double)n);
    }
}

// Q rows of every row set's rows, stored contiguously in set order, so that
// the per-SNP downdate gathers read them with independent coalesced loads.
static __global__ void k_set_qrows(const int* __restrict__ rows, int total, const float* __restrict__ Qr, int LP,
                                   float* __restrict__ qrows) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)total * LP) return;
    const long long kk = q / LP;
    const int c = (int)(q % LP);
    qrows[q] = Qr[(size_t)rows[kk] * LP + c];
}

// Sort keys of the stored rows: (trait, SNP) -> reference output order.
// Sort keys of the stored-row slots: trait * mb + SNP, an unused slot (trait
// -1) all ones in the low `bits` bits, so that it sorts last (the sort looks
// at those bits only; 2^bits > t * mb).
template <class RecT>
static __global__ void k_rec_keys(const RecT* __restrict__ rec, long long N, long long mb, int bits,
                                  unsigned long long* __restrict__ keys, int* __restrict__ perm) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= N) return;
    const int tr = rec[q].trait;
    keys[q] = tr < 0 ? (bits >= 64 ? ~0ull : ((1ull << bits) - 1ull))
                     : (unsigned long long)tr * (unsigned long long)mb + (unsigned)rec[q].snp;
    perm[q] = (int)q;
}

// The stored rows that go back to the host, in sorted order and packed by
// field: N x {trait, snp, r2, mask} then N x R each of b, se, t (16 + 12 R
// bytes per row instead of the 80- or 128-byte record).
struct RowsSoA {
    int32_t* trait;
    int32_t* snp;
    float* r2;
    uint32_t* mask;
    float* b;
    float* se;
    float* t;
};
// Field arrays of N rows carved from `base` (at least rows_soa_bytes(N, R) bytes).
__host__ __device__ inline size_t rows_soa_bytes(long long N, int R) { return (size_t)N * (16 + 12 * (size_t)R); }
__host__ __device__ inline RowsSoA rows_soa(void* base, long long N, int R) {
    uint8_t* p = static_cast<uint8_t*>(base);
    RowsSoA s;
    s.trait = reinterpret_cast<int32_t*>(p);
    s.snp = reinterpret_cast<int32_t*>(p + 4 * (size_t)N);
    s.r2 = reinterpret_cast<float*>(p + 8 * (size_t)N);
    s.mask = reinterpret_cast<uint32_t*>(p + 12 * (size_t)N);
    s.b = reinterpret_cast<float*>(p + 16 * (size_t)N);
    s.se = s.b + (size_t)N * R;
    s.t = s.se + (size_t)N * R;
    return s;
}

template <int R>
static __global__ void k_rec_gather(const RecOf<R>* __restrict__ rec, const int* __restrict__ perm, long long N,
                                    RowsSoA out, const float* __restrict__ cov, float* __restrict__ cov_out, int l) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= N) return;
    const int src = perm[q];
    const RecOf<R>& rc = rec[src];
    out.trait[q] = rc.trait;
    out.snp[q] = rc.snp;
    out.r2[q] = rc.r2;
    out.mask[q] = rc.mask;
#pragma unroll
    for (int a = 0; a < R; ++a) {
        out.b[(size_t)q * R + a] = rc.b[a];
        out.se[(size_t)q * R + a] = rc.se[a];
        out.t[(size_t)q * R + a] = rc.t[a];
    }
    if (cov)
        for (int u = 0; u < l * 3; ++u) cov_out[(size_t)q * l * 3 + u] = cov[(size_t)src * l * 3 + u];
}

}  // namespace oa
