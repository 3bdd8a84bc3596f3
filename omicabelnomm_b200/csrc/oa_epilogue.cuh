// Per-test statistics fused into the GEMM epilogue.
//
// Given z = X_i' y~_j (the accumulator of the XR'Y~ GEMM, y~ = y with the
// covariate fit of its missingness pattern removed), this computes what the
// reference's sposv + hpc_SSY + hpc_statistics compute for one SNP x trait
// test (src/Algorithm.cpp:714-813, 896-1214):
//
//   beta_x = Sinv_g z                       (Frisch-Waugh-Lovell: the SNP block of S^-1 rhs)
//   RSS    = RSS0_j - z' beta_x              (observed rows; exact identity, FP64)
//   RSS   -= sum over observed rows with y == 0 of (x_k' beta)^2   (the y != 0 filter, :1015)
//   R2     = 1 - (RSS/(n_corr-1)) / (SST/(n-1))                       (:1092)
//   SE_h   = sqrt(RSS/n_corr) * sqrt(var_x_h * (n-miss)/n)            (:1100, :1134)
//   t_h    = |beta_h / SE_h|                                           (:1137)
//
// and applies the store filters (RSS > 0, R2 > minR2store or -f, t >
// minTstore or -f, at least one stored SNP term; :1119-1203).
#pragma once
#include "oa_common.cuh"

namespace oa {

template <int R>
__device__ __forceinline__ bool epi_eval(const EpiArgs& E, int i, int j, const float* z, bool valid,
                                         Rec& rc) {
    if (!valid) return false;
    const int g = E.pat[j];
    const size_t gi = (size_t)g * E.mb + i;
    if (E.sing[gi]) {
        atomicAdd(E.n_singular, 1ull);
        return false;
    }
    const double* S = E.sinv + gi * (R * R);
    double bx[R];
    double zz = 0.0;
#pragma unroll
    for (int a = 0; a < R; ++a) {
        double s = 0.0;
#pragma unroll
        for (int b = 0; b < R; ++b) s += S[a * R + b] * (double)z[b];
        bx[a] = s;
        zz += (double)z[a] * s;
    }
    double rss = E.rss0[j] - zz;
    const int zs = E.zset[j];
    if (zs >= 0) {
        // fitted values on the observed zero-y rows leave the RSS (src/Algorithm.cpp:1013-1020)
        const int l = E.l;
        const float* ao = E.aobs + gi * (size_t)(l * R);
        const double* W = E.W + (size_t)g * l * l;
        double bq[OA_MAX_L];
        double aob[OA_MAX_L];
        for (int q = 0; q < l; ++q) {
            double s = 0.0;
#pragma unroll
            for (int a = 0; a < R; ++a) s += (double)ao[q * R + a] * bx[a];
            aob[q] = s;
        }
        for (int q = 0; q < l; ++q) {
            double s = 0.0;
            for (int u = 0; u < l; ++u) s += W[q * l + u] * aob[u];
            bq[q] = E.b0[(size_t)j * l + q] - s;
        }
        const double* zQ = E.zQ + (size_t)zs * l * l;
        const float* zA = E.zA + ((size_t)zs * E.mb + i) * (l * R);
        const float* zD = E.zD + ((size_t)zs * E.mb + i) * (R * R);
        double c = 0.0;
        for (int q = 0; q < l; ++q) {
            double s = 0.0;
            for (int u = 0; u < l; ++u) s += zQ[q * l + u] * bq[u];
            c += bq[q] * s;
#pragma unroll
            for (int a = 0; a < R; ++a) c += 2.0 * bq[q] * (double)zA[q * R + a] * bx[a];
        }
#pragma unroll
        for (int a = 0; a < R; ++a)
#pragma unroll
            for (int b = 0; b < R; ++b) c += bx[a] * (double)zD[a * R + b] * bx[b];
        rss -= c;
    }
    const int nobs = E.nobs[j];
    const int ncorr = nobs - E.p;
    const double R2 = 1.0 - (rss / (double)(ncorr - 1)) / ((double)E.sst[j] / (double)(E.n - 1));
    const double sig = sqrt(fmax(rss, 0.0) / (double)ncorr);
    const double vf = (double)nobs / (double)E.n;
    rc.trait = j;
    rc.snp = E.snp_base + i;
    rc.r2 = (float)R2;
    rc.sig = (float)sig;
    rc.pad[0] = rc.pad[1] = rc.pad[2] = 0.f;
    uint32_t mask = 0;
#pragma unroll
    for (int a = 0; a < R; ++a) {
        const double se = sig * sqrt((double)E.varx[(size_t)i * R + a] * vf);
        const double t = fabs(bx[a] / se);
        rc.b[a] = (float)bx[a];
        rc.se[a] = (float)se;
        rc.t[a] = (float)t;
        if (t > (double)E.min_t || E.store_all) mask |= 1u << a;
    }
#pragma unroll
    for (int a = R; a < OA_MAX_R; ++a) rc.b[a] = rc.se[a] = rc.t[a] = 0.f;
    rc.mask = mask;
    const bool live = (rss > 0.0) && (R2 > (double)E.min_r2 || E.store_all);
    if (E.d_r2) {
        const size_t o = (size_t)j * E.dense_ld + E.snp_base + i;
        const float nanf_ = __int_as_float(0x7fc00000);
        E.d_r2[o] = rss > 0.0 ? (float)R2 : nanf_;
        E.d_sig[o] = rss > 0.0 ? (float)sig : nanf_;
#pragma unroll
        for (int a = 0; a < R; ++a) {
            E.d_beta[o * R + a] = rss > 0.0 ? rc.b[a] : nanf_;
            E.d_se[o * R + a] = rss > 0.0 ? rc.se[a] : nanf_;
            E.d_t[o * R + a] = rss > 0.0 ? rc.t[a] : nanf_;
        }
    }
    return live && mask != 0u;
}

// Warp-aggregated append of the stored rows (one atomic per warp and slot).
__device__ __forceinline__ void epi_emit(const EpiArgs& E, bool st, const Rec& rc) {
    const unsigned m = __ballot_sync(0xffffffffu, st);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const int lead = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == lead) base = atomicAdd(E.rec_count, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, lead);
    if (st) {
        const unsigned long long idx = base + __popc(m & ((1u << lane) - 1u));
        if ((long long)idx < E.cap) {
            float4* dst = reinterpret_cast<float4*>(E.rec + idx);
            const float4* src = reinterpret_cast<const float4*>(&rc);
#pragma unroll
            for (int q = 0; q < (int)(sizeof(Rec) / 16); ++q) dst[q] = src[q];
        }
    }
}

}  // namespace oa
