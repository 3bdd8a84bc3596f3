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
// minTstore or -f, at least one stored SNP term; :1119-1203).  The RSS
// difference is formed in FP64 (it can cancel); the rest is FP32, the
// precision the reference holds these values in, with the per-trait
// constants folded so that a test needs one reciprocal square root and no
// division.
#pragma once
#include "oa_common.cuh"

namespace oa {

__device__ __forceinline__ TraitP load_trait(const EpiArgs& E, int j) {
    TraitP p;
    p.rss0 = E.rss0[j];
    p.a_r2 = E.a_r2[j];
    p.inv_ncorr = E.inv_ncorr[j];
    p.vf = E.vf[j];
    p.g = E.pat[j];
    p.zs = E.zset[j];
    p.orig = E.tperm[j];
    return p;
}

// Status bits of an evaluated (non-singular) test (OA_TEST_*, include/omicabel_b200.h):
// RSS <= 0 skips it (src/Algorithm.cpp:1094-1099, 1119); otherwise R2 at or
// below the store threshold without -f skips its terms (:1119-1123); a test
// with a stored SNP term has a row (:1156-1157, 1197).
__device__ __forceinline__ uint8_t test_flags(const EpiArgs& E, double rss, float r2, uint32_t mask) {
    if (!(rss > 0.0)) return OA_TEST_RSS;
    if (!(r2 > E.min_r2 || E.store_all)) return OA_TEST_R2;
    return mask ? OA_TEST_STORED : 0;
}

// Schur inverse of (pattern g, SNP i); false if the system is singular.
template <int R>
__device__ __forceinline__ bool load_schur(const EpiArgs& E, int g, int i, double* S) {
    const size_t gi = (size_t)g * E.mb + i;
    if (E.sing[gi]) return false;
    const double* src = E.sinv + gi * (R * R);
#pragma unroll
    for (int q = 0; q < R * R; ++q) S[q] = src[q];
    return true;
}

// Fitted values of the observed rows whose y is exactly 0 leave the RSS
// (src/Algorithm.cpp:1013-1020).  Rare (continuous phenotypes have no exact
// zeros); reads the zero set's sums directly.
template <int R>
__device__ __noinline__ double zero_rows_rss(const EpiArgs& E, int i, int j, const TraitP& tp, const double* bx) {
    const int l = E.l;
    const size_t gi = (size_t)tp.g * E.mb + i;
    const float* ao = E.aobs + gi * (size_t)(l * R);
    const double* W = E.W + (size_t)tp.g * l * l;
    double bq[OA_MAX_L], aob[OA_MAX_L];
    for (int q = 0; q < l; ++q) {
        double s = 0.0;
        for (int a = 0; a < R; ++a) s += (double)ao[q * R + a] * bx[a];
        aob[q] = s;
    }
    for (int q = 0; q < l; ++q) {
        double s = 0.0;
        for (int u = 0; u < l; ++u) s += W[q * l + u] * aob[u];
        bq[q] = E.b0[(size_t)j * l + q] - s;
    }
    const double* zQ = E.zQ + (size_t)tp.zs * l * l;
    const float* zA = E.zA + ((size_t)tp.zs * E.mb + i) * (l * R);
    const float* zD = E.zD + ((size_t)tp.zs * E.mb + i) * (R * R);
    double c = 0.0;
    for (int q = 0; q < l; ++q) {
        double s = 0.0;
        for (int u = 0; u < l; ++u) s += zQ[q * l + u] * bq[u];
        c += bq[q] * s;
        for (int a = 0; a < R; ++a) c += 2.0 * bq[q] * (double)zA[q * R + a] * bx[a];
    }
    for (int a = 0; a < R; ++a)
        for (int b = 0; b < R; ++b) c += bx[a] * (double)zD[a * R + b] * bx[b];
    return c;
}

// SNP coefficients and RSS of the reference's r >= 2 downdate (quirk mode;
// the per-(pattern, SNP) terms come from schur_quirk in oa_lean.cuh):
//   beta_x = Sq^-1 (z - dl' b0_j),  RSS = RSS0_j - 2 beta_x' z + beta_x' K beta_x.
template <int R>
__device__ __noinline__ double quirk_beta_rss(const EpiArgs& E, int i, int j, const TraitP& tp, const double* S,
                                              const float* z, double* bx) {
    const int l = E.l;
    const size_t gi = (size_t)tp.g * E.mb + i;
    const float* dl = E.qdel + gi * (size_t)(l * R);
    const double* b0 = E.b0 + (size_t)j * l;
    double rhs[R];
    for (int a = 0; a < R; ++a) {
        double s = (double)z[a];
        for (int q = 0; q < l; ++q) s -= (double)dl[q * R + a] * b0[q];
        rhs[a] = s;
    }
    for (int a = 0; a < R; ++a) {
        double s = 0.0;
        for (int b = 0; b < R; ++b) s += S[a * R + b] * rhs[b];
        bx[a] = s;
    }
    const double* K = E.qK + gi * (size_t)(R * R);
    double zb = 0.0, quad = 0.0;
    for (int a = 0; a < R; ++a) {
        zb += (double)z[a] * bx[a];
        double s = 0.0;
        for (int b = 0; b < R; ++b) s += K[a * R + b] * bx[b];
        quad += bx[a] * s;
    }
    return tp.rss0 - 2.0 * zb + quad;
}

// One test given its trait constants, Schur inverse S and the SNP's var_x.
template <int R>
__device__ __forceinline__ bool epi_core(const EpiArgs& E, int i, int j, const float* z, const TraitP& tp,
                                         const double* S, const float* vx, RecOf<R>& rc) {
    double bx[R];
    double rss;
    if (E.qK) {
        rss = quirk_beta_rss<R>(E, i, j, tp, S, z, bx);
    } else {
        double zz = 0.0;
#pragma unroll
        for (int a = 0; a < R; ++a) {
            double s = 0.0;
#pragma unroll
            for (int b = 0; b < R; ++b) s += S[a * R + b] * (double)z[b];
            bx[a] = s;
            zz += (double)z[a] * s;
        }
        rss = tp.rss0 - zz;
    }
    if (tp.zs >= 0) rss -= zero_rows_rss<R>(E, i, j, tp, bx);
    const float rssf = (float)rss;
    const float r2 = 1.f - rssf * tp.a_r2;
    const float sig2 = rssf * tp.inv_ncorr;
    rc.trait = tp.orig;
    rc.snp = E.snp_base + i;
    rc.r2 = r2;
    rc.sig = sqrtf(fmaxf(sig2, 0.f));
    rc.tint = j;
    rc.pad[0] = rc.pad[1] = 0.f;
    uint32_t mask = 0;
#pragma unroll
    for (int a = 0; a < R; ++a) {
        const float w = sig2 * vx[a] * tp.vf;       // SE^2
        const float rs = rsqrtf(w);
        const float b = (float)bx[a];
        const float t = fabsf(b) * rs;
        rc.b[a] = b;
        rc.se[a] = w * rs;
        rc.t[a] = t;
        if (t > E.min_t || E.store_all) mask |= 1u << a;
    }
#pragma unroll
    for (int a = R; a < (int)(sizeof(rc.b) / sizeof(float)); ++a) rc.b[a] = rc.se[a] = rc.t[a] = 0.f;
    rc.mask = mask;
    const bool live = (rss > 0.0) && (r2 > E.min_r2 || E.store_all);
    if (E.d_r2) {
        const size_t o = (size_t)tp.orig * E.dense_ld + E.snp_base + i;
        const float nanf_ = __int_as_float(0x7fc00000);
        const bool pos = rss > 0.0;
        E.d_r2[o] = pos ? r2 : nanf_;
        E.d_sig[o] = pos ? rc.sig : nanf_;
#pragma unroll
        for (int a = 0; a < R; ++a) {
            E.d_beta[o * R + a] = pos ? rc.b[a] : nanf_;
            E.d_se[o * R + a] = pos ? rc.se[a] : nanf_;
            E.d_t[o * R + a] = pos ? rc.t[a] : nanf_;
        }
        if (E.d_flags) E.d_flags[o] = test_flags(E, rss, r2, mask);
    }
    return live && mask != 0u;
}

// The statistics of one test, kept in registers until the warp knows which
// of its lanes store a row (the tensor-core epilogues build a record only
// for those).  Same arithmetic as epi_core.
template <int R>
struct EpiTest {
    double rss;
    float r2, sig2;
    float b[R], se[R], t[R];
    uint32_t mask;
};

// FAST: the caller knows that neither the quirk terms nor the dense outputs
// are set and that no trait of the tile has a zero set (the common case):
// the same arithmetic without those per-test checks.
template <int R, bool FAST = false>
__device__ __forceinline__ bool epi_decide(const EpiArgs& E, int i, int j, const float* z, const TraitP& tp,
                                           const double* S, const float* vx, EpiTest<R>& o) {
    double bx[R];
    double rss;
    if (!FAST && E.qK) {
        rss = quirk_beta_rss<R>(E, i, j, tp, S, z, bx);
    } else {
        double zz = 0.0;
#pragma unroll
        for (int a = 0; a < R; ++a) {
            double s = 0.0;
#pragma unroll
            for (int b = 0; b < R; ++b) s += S[a * R + b] * (double)z[b];
            bx[a] = s;
            zz += (double)z[a] * s;
        }
        rss = tp.rss0 - zz;
    }
    if (!FAST && tp.zs >= 0) rss -= zero_rows_rss<R>(E, i, j, tp, bx);
    const float rssf = (float)rss;
    o.rss = rss;
    o.r2 = 1.f - rssf * tp.a_r2;
    o.sig2 = rssf * tp.inv_ncorr;
    uint32_t mask = 0;
#pragma unroll
    for (int a = 0; a < R; ++a) {
        const float w = o.sig2 * vx[a] * tp.vf;     // SE^2
        const float rs = rsqrtf(w);
        const float b = (float)bx[a];
        o.b[a] = b;
        o.se[a] = w * rs;
        o.t[a] = fabsf(b) * rs;
        if (o.t[a] > E.min_t || E.store_all) mask |= 1u << a;
    }
    o.mask = mask;
    if (!FAST && E.d_r2) {
        const size_t off = (size_t)tp.orig * E.dense_ld + E.snp_base + i;
        const float nanf_ = __int_as_float(0x7fc00000);
        const bool pos = rss > 0.0;
        E.d_r2[off] = pos ? o.r2 : nanf_;
        E.d_sig[off] = pos ? sqrtf(fmaxf(o.sig2, 0.f)) : nanf_;
#pragma unroll
        for (int a = 0; a < R; ++a) {
            E.d_beta[off * R + a] = pos ? o.b[a] : nanf_;
            E.d_se[off * R + a] = pos ? o.se[a] : nanf_;
            E.d_t[off * R + a] = pos ? o.t[a] : nanf_;
        }
        if (E.d_flags) E.d_flags[off] = test_flags(E, rss, o.r2, mask);
    }
    const bool live = (rss > 0.0) && (o.r2 > E.min_r2 || E.store_all);
    return live && mask != 0u;
}

// The record of a stored test (the fields epi_core fills).
template <int R>
__device__ __forceinline__ void epi_write(const EpiArgs& E, int i, int j, const TraitP& tp, const EpiTest<R>& o,
                                          RecOf<R>* dst) {
    RecOf<R> rc;
    rc.trait = tp.orig;
    rc.snp = E.snp_base + i;
    rc.r2 = o.r2;
    rc.mask = o.mask;
    rc.sig = sqrtf(fmaxf(o.sig2, 0.f));
    rc.tint = j;
    rc.pad[0] = rc.pad[1] = 0.f;
    constexpr int K = (int)(sizeof(rc.b) / sizeof(float));
#pragma unroll
    for (int a = 0; a < K; ++a) {
        rc.b[a] = a < R ? o.b[a] : 0.f;
        rc.se[a] = a < R ? o.se[a] : 0.f;
        rc.t[a] = a < R ? o.t[a] : 0.f;
    }
    float4* d = reinterpret_cast<float4*>(dst);
    const float4* src = reinterpret_cast<const float4*>(&rc);
#pragma unroll
    for (int q = 0; q < (int)(sizeof(rc) / 16); ++q) d[q] = src[q];
}

// Dense outputs of a singular test are NaN.
template <int R>
__device__ __forceinline__ void epi_dense_nan(const EpiArgs& E, int i, const TraitP& tp) {
    if (!E.d_r2) return;
    const size_t o = (size_t)tp.orig * E.dense_ld + E.snp_base + i;
    const float nanf_ = __int_as_float(0x7fc00000);
    E.d_r2[o] = nanf_;
    E.d_sig[o] = nanf_;
#pragma unroll
    for (int a = 0; a < R; ++a) E.d_beta[o * R + a] = E.d_se[o * R + a] = E.d_t[o * R + a] = nanf_;
    if (E.d_flags) E.d_flags[o] = OA_TEST_SINGULAR;
}

// Self-contained evaluation (loads its own constants): the SIMT GEMM epilogue.
template <int R>
__device__ __forceinline__ bool epi_eval(const EpiArgs& E, int i, int j, const float* z, bool valid, RecOf<R>& rc) {
    if (!valid) return false;
    const TraitP tp = load_trait(E, j);
    double S[R * R];
    if (!load_schur<R>(E, tp.g, i, S)) {
        atomicAdd(E.n_singular, 1ull);
        epi_dense_nan<R>(E, i, tp);
        return false;
    }
    float vx[R];
#pragma unroll
    for (int a = 0; a < R; ++a) vx[a] = E.varx[(size_t)i * R + a];
    return epi_core<R>(E, i, j, z, tp, S, vx, rc);
}

// Warp-aggregated append of the stored rows: one atomic on the slot counter
// per warp and step (the SIMT GEMM, whose epilogue runs a few steps per tile).
template <int R>
__device__ __forceinline__ void epi_emit(const EpiArgs& E, bool st, const RecOf<R>& rc) {
    const unsigned m = __ballot_sync(0xffffffffu, st);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const int lead = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == lead) {
        base = atomicAdd(E.rec_count, (unsigned long long)__popc(m));
        if (E.rec_valid) atomicAdd(E.rec_valid, (unsigned long long)__popc(m));
    }
    base = __shfl_sync(0xffffffffu, base, lead);
    if (st) {
        const unsigned long long idx = base + __popc(m & ((1u << lane) - 1u));
        if ((long long)idx < E.cap) {
            float4* dst = reinterpret_cast<float4*>(static_cast<RecOf<R>*>(E.rec) + idx);
            const float4* src = reinterpret_cast<const float4*>(&rc);
#pragma unroll
            for (int q = 0; q < (int)(sizeof(rc) / 16); ++q) dst[q] = src[q];
        }
    }
}

// Record slots reserved by one warp: the tensor-core epilogues emit a few rows
// at nearly every step, and one shared counter taking an atomic per warp and
// step serialises them; a warp instead reserves EMIT_BLOCK slots at a time
// (oa_common.cuh).
struct Emitter {
    unsigned long long base = 0;
    int used = 0, cap = 0;
};

// Close a warp's reserved block: unused slots are marked invalid (trait -1)
// and the rows written are counted.  All lanes of the warp take part.
template <int R>
__device__ __forceinline__ void epi_retire(const EpiArgs& E, Emitter& em) {
    if (em.cap == 0) return;
    const int lane = threadIdx.x & 31;
    for (int q = em.used + lane; q < em.cap; q += 32) {
        const unsigned long long idx = em.base + (unsigned long long)q;
        if ((long long)idx < E.cap) static_cast<RecOf<R>*>(E.rec)[idx].trait = -1;
    }
    if (lane == 0 && E.rec_valid && em.used > 0) atomicAdd(E.rec_valid, (unsigned long long)em.used);
    em.used = em.cap = 0;
}

// Block-reserved row emission for records built only by the lanes that
// store: `write` receives the slot of the calling lane's row.
template <int R, class W>
__device__ __forceinline__ void epi_emit_lazy(const EpiArgs& E, bool st, Emitter& em, W&& write) {
    if (!E.rec) return;
    const unsigned m = __ballot_sync(0xffffffffu, st);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const int k = __popc(m);
    if (em.used + k > em.cap) {   // warp-uniform
        epi_retire<R>(E, em);
        unsigned long long b = 0;
        if (lane == 0) b = atomicAdd(E.rec_count, (unsigned long long)EMIT_BLOCK);
        em.base = __shfl_sync(0xffffffffu, b, 0);
        em.used = 0;
        em.cap = EMIT_BLOCK;
    }
    if (st) {
        const unsigned long long idx = em.base + (unsigned long long)(em.used + __popc(m & ((1u << lane) - 1u)));
        if ((long long)idx < E.cap) write(static_cast<RecOf<R>*>(E.rec) + idx);
    }
    em.used += k;
}

}  // namespace oa
