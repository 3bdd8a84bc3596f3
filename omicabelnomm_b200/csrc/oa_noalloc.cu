// oa_scan_dense_noalloc: the plain-FP32 scan of one SNP block for callers
// that cannot allocate GPU memory.
//
// Some callers cannot call cudaMalloc: plug-ins inside host frameworks that
// own the device memory pool (and forbid raw allocations), and processes
// under a hard device-memory cap whose memory was reserved up front.  This
// entry point gives them the engine's plain-FP32 block scan (the SIMT GEMM
// with fused statistics, plus the small kernels that prepare its tables)
// with every intermediate buffer carved from one file-scope
// `static __device__` array of OA_NOALLOC_SCRATCH_BYTES.  It calls no
// cudaMalloc / cudaFree and no allocating library routine, and allocates no
// host heap memory either.
//
// Differences from the block engine, all to avoid allocation: the
// covariates are orthonormalised on the device (shifted CholeskyQR3) instead
// of a host Householder QR, with the same rank rule (singular values of R
// below 1e-6); every trait is its own missingness pattern (no host-side
// grouping; the math is identical); results are dense arrays.  The call
// reads two small status words back to the host and synchronises the
// caller's stream.  The scratch array is shared by every call in the process
// and keeps the last call's contents; calls that overlap on the GPU (other
// streams or host threads) race on it.  The first call on a device looks up
// the array's device address (cudaGetSymbolAddress).
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "oa_kernels.cuh"
#include "oa_launch.h"

namespace oa {
namespace na {

// The scratch every call shares (held by each GPU that loads the library until exit).
static __device__ __align__(256) unsigned char g_scratch[OA_NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
static void* g_scratch_ptr[MAX_DEVICES];
static std::mutex g_mu;

// Device address of the scratch array on the current device (looked up once per device).
static cudaError_t scratch_address(int dev, void** out) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

// Gram matrix G[a][b] = sum_k X[a][k] X[b][k] of the l columns of X (FP64).
template <class T>
__global__ void __launch_bounds__(256) k_na_gram(const T* __restrict__ X, int n, int l, double* __restrict__ G) {
    __shared__ double red[8];
    const int a = blockIdx.x, b = blockIdx.y;
    if (b > a) return;
    double s = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) s += (double)X[(size_t)a * n + k] * (double)X[(size_t)b * n + k];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += red[w];
        G[a * l + b] = t;
        G[b * l + a] = t;
    }
}

// Q = X R^-1 with R = chol(G + s I) upper triangular: one Cholesky-QR pass.
// shift_u > 0 makes it the shifted first pass of shifted CholeskyQR3
// (Fukaya, Kannan, Nakatsukasa, Yamamoto, Yanagisawa, "Shifted Cholesky QR
// for computing the QR factorization of ill-conditioned matrices", SIAM J.
// Sci. Comput. 42(1), 2020): s = shift_u * ||X||_F^2 with
// shift_u = 11 (n l + l (l + 1)) 2^-53, which keeps the factorisation from
// breaking down for condition numbers up to about 1e15; two unshifted passes
// follow.  Writes Q (FP64, column-major), R (row-major upper, l x l) and, if
// Qr is given, Q's FP32 row-major copy padded to LP columns.  flag[0] = 1 if
// G + s I is not numerically positive definite.
template <class T>
__global__ void __launch_bounds__(256) k_na_cholq(const T* __restrict__ X, int n, int l, int LP, double shift_u,
                                                 const double* __restrict__ G, double* __restrict__ Q,
                                                 double* __restrict__ Rout, float* __restrict__ Qr,
                                                 int* __restrict__ flag) {
    __shared__ double Ri[OA_MAX_L * OA_MAX_L];
    __shared__ int bad;
    if (threadIdx.x == 0) {
        double L[OA_MAX_L * OA_MAX_L];
        bad = 0;
        double fro2 = 0.0;
        for (int j = 0; j < l; ++j) fro2 += G[j * l + j];
        const double shift = shift_u * fro2;
        for (int i = 0; i < l * l; ++i) L[i] = 0.0;
        for (int j = 0; j < l && !bad; ++j) {
            double s = G[j * l + j] + shift;
            for (int q = 0; q < j; ++q) s -= L[j * l + q] * L[j * l + q];
            if (!(s > 0.0)) {
                bad = 1;
                break;
            }
            const double d = sqrt(s);
            L[j * l + j] = d;
            for (int i = j + 1; i < l; ++i) {
                double u = G[i * l + j];
                for (int q = 0; q < j; ++q) u -= L[i * l + q] * L[j * l + q];
                L[i * l + j] = u / d;
            }
        }
        // R = L' (upper); R^-1 by back substitution
        for (int i = 0; i < l * l; ++i) Ri[i] = 0.0;
        if (!bad) {
            for (int i = 0; i < l; ++i)
                for (int j = 0; j < l; ++j) Rout[i * l + j] = j >= i ? L[j * l + i] : 0.0;
            for (int i = l - 1; i >= 0; --i) {
                Ri[i * l + i] = 1.0 / L[i * l + i];
                for (int j = i + 1; j < l; ++j) {
                    double s = 0.0;
                    for (int k = i + 1; k <= j; ++k) s += L[k * l + i] * Ri[k * l + j];
                    Ri[i * l + j] = -s / L[i * l + i];
                }
            }
        }
        if (bad) *flag = 1;
    }
    __syncthreads();
    if (bad) return;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double x[OA_MAX_L];
        for (int a = 0; a < l; ++a) x[a] = (double)X[(size_t)a * n + k];
        for (int q = 0; q < l; ++q) {
            double s = 0.0;
            for (int a = 0; a <= q; ++a) s += x[a] * Ri[a * l + q];
            Q[(size_t)q * n + k] = s;
            if (Qr) Qr[(size_t)k * LP + q] = (float)s;
        }
        if (Qr)
            for (int q = l; q < LP; ++q) Qr[(size_t)k * LP + q] = 0.f;
    }
}

// Rank check of the covariates, the block engine's rule: XL = Q R3 R2 R1
// with Q orthonormal, so the singular values of XL are those of
// R = R3 R2 R1; any below 1e-6 sets flag[0] (src/Algorithm.cpp:508-522 takes
// them from sgesvd of XL).  One-sided Jacobi on R, FP64, one thread; skipped
// when an earlier pass has already flagged the matrix.
__global__ void k_na_rank(const double* __restrict__ R1, const double* __restrict__ R2, const double* __restrict__ R3,
                          int l, const int* __restrict__ broke, int* __restrict__ flag) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (broke[0] || broke[1] || broke[2]) return;
    double T[OA_MAX_L * OA_MAX_L], A[OA_MAX_L * OA_MAX_L];
    for (int i = 0; i < l; ++i)   // T = R2 R1
        for (int j = 0; j < l; ++j) {
            double s = 0.0;
            for (int k = 0; k < l; ++k) s += R2[i * l + k] * R1[k * l + j];
            T[i * l + j] = s;
        }
    for (int i = 0; i < l; ++i)   // A = R3 T
        for (int j = 0; j < l; ++j) {
            double s = 0.0;
            for (int k = 0; k < l; ++k) s += R3[i * l + k] * T[k * l + j];
            A[i * l + j] = s;
        }
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < l; ++p)
            for (int q = p + 1; q < l; ++q) {
                double a = 0.0, b = 0.0, c = 0.0;
                for (int i = 0; i < l; ++i) {
                    a += A[i * l + p] * A[i * l + p];
                    b += A[i * l + q] * A[i * l + q];
                    c += A[i * l + p] * A[i * l + q];
                }
                if (fabs(c) <= 1e-300) continue;
                off = fmax(off, fabs(c) / sqrt(a * b));
                const double zeta = (b - a) / (2.0 * c);
                const double tn = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                const double cs = 1.0 / sqrt(1.0 + tn * tn), sn = cs * tn;
                for (int i = 0; i < l; ++i) {
                    const double x = A[i * l + p], y = A[i * l + q];
                    A[i * l + p] = cs * x - sn * y;
                    A[i * l + q] = sn * x + cs * y;
                }
            }
        if (off < 1e-15) break;
    }
    for (int p = 0; p < l; ++p) {
        double a = 0.0;
        for (int i = 0; i < l; ++i) a += A[i * l + p] * A[i * l + p];
        if (!(sqrt(a) >= 1e-6)) *flag = 1;
    }
}

// Row sets with every trait its own missingness pattern, plus one zero set
// per trait that has observed values exactly 0.  counts[j] = (missing, zeros).
__global__ void k_na_sets(const int* __restrict__ counts, int t, int* __restrict__ pat, int* __restrict__ zset,
                          int* __restrict__ tperm, int* __restrict__ set_off, int* __restrict__ set_rep,
                          int* __restrict__ set_kind, int* __restrict__ set_slot,
                          int* __restrict__ info /* [0] Z, [1] rows */) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int z = 0, off = 0;
    for (int j = 0; j < t; ++j) {
        pat[j] = j;
        tperm[j] = j;
        set_off[j] = off;
        set_rep[j] = j;
        set_kind[j] = 0;
        set_slot[j] = j;
        off += counts[2 * j];
    }
    for (int j = 0; j < t; ++j) {
        if (counts[2 * j + 1] > 0) {
            const int s = t + z;
            zset[j] = z;
            set_off[s] = off;
            set_rep[s] = j;
            set_kind[s] = 1;
            set_slot[s] = z;
            off += counts[2 * j + 1];
            ++z;
        } else {
            zset[j] = -1;
        }
    }
    set_off[t + z] = off;
    info[0] = z;
    info[1] = off;
}

// Bump allocator over the scratch array (256-byte aligned pieces).
struct Carve {
    unsigned char* base;
    size_t used = 0;
    template <class T>
    T* take(size_t count) {
        used = (used + 255) & ~(size_t)255;
        T* p = reinterpret_cast<T*>(base + used);
        used += count * sizeof(T);
        return p;
    }
};

static int pad_l(int l) { return l <= 4 ? 4 : (l <= 8 ? 8 : 16); }

}  // namespace na
}  // namespace oa

extern "C" void oa__set_error(const char* msg);

namespace {
oa_status fail(oa_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    oa__set_error(buf);
    return s;
}
}  // namespace

#define NA_CU(x)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) return fail(OA_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_));   \
    } while (0)

extern "C" oa_status oa_scan_dense_noalloc(const float* xl, const float* y, const float* xr, int32_t n, int32_t l,
                                           int32_t r, int32_t t, int32_t mb, float* beta, float* se, float* tstat,
                                           float* r2, void* stream) {
    using namespace oa;
    using namespace oa::na;
    // an error still pending from the caller's own earlier work is reported, not consumed
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess)
        return fail(OA_ERR_CUDA, "a CUDA error from earlier work is pending on this thread (left in place): %s",
                    cudaGetErrorString(pending));
    if (!xl || !y || !xr || !beta || !se || !tstat || !r2) return fail(OA_ERR_ARG, "null argument");
    if (l < 1 || l > OA_MAX_L || !(r == 1 || r == 2 || r == 4) || n <= l + r || t < 1 || mb < 1 || t > 2048)
        return fail(OA_ERR_ARG, "invalid sizes n=%d l=%d r=%d t=%d mb=%d (r in {1,2,4}, t <= 2048)", n, l, r, t,
                    mb);
    int dev = 0;
    NA_CU(cudaGetDevice(&dev));
    void* sp = nullptr;
    NA_CU(scratch_address(dev, &sp));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int LP = pad_l(l), n_pad = (n + 63) & ~63;

    // fixed part of the layout (sizes known before the data is looked at)
    Carve cv{reinterpret_cast<unsigned char*>(sp)};
    unsigned long long* counters = cv.take<unsigned long long>(4);
    int* info = cv.take<int>(8);   // [0] Z, [1] set rows, [2..4] pass breakdown, [5] rank deficient
    double* G = cv.take<double>((size_t)OA_MAX_L * OA_MAX_L);
    double* Rf = cv.take<double>((size_t)3 * OA_MAX_L * OA_MAX_L);   // R of each CholeskyQR pass
    double* Q1 = cv.take<double>((size_t)n * l);
    double* Q64 = cv.take<double>((size_t)n * l);
    float* Qr = cv.take<float>((size_t)n * LP);
    double* tsums = cv.take<double>((size_t)t * (2 + OA_MAX_L));
    int* tcounts = cv.take<int>((size_t)t * 2);
    unsigned long long* thash = cv.take<unsigned long long>((size_t)t * 4);
    int* pat = cv.take<int>(t);
    int* zset = cv.take<int>(t);
    int* tperm = cv.take<int>(t);
    float* a_r2 = cv.take<float>(t);
    float* inv_ncorr = cv.take<float>(t);
    float* vf = cv.take<float>(t);
    int* set_off = cv.take<int>((size_t)2 * t + 1);
    int* set_rep = cv.take<int>((size_t)2 * t);
    int* set_kind = cv.take<int>((size_t)2 * t);
    int* set_slot = cv.take<int>((size_t)2 * t);
    double* W = cv.take<double>((size_t)t * l * l);
    double* zQ = cv.take<double>((size_t)t * l * l);
    uint8_t* pat_bad = cv.take<uint8_t>(t);
    float* Yt = cv.take<float>((size_t)t * n_pad);
    double* rss0 = cv.take<double>(t);
    float* sst = cv.take<float>(t);
    int* nobs = cv.take<int>(t);
    double* b0 = cv.take<double>((size_t)t * l);
    float* mean = cv.take<float>((size_t)mb * r);
    int* has_nan = cv.take<int>(1);
    float* varx = cv.take<float>((size_t)mb * r);
    double* sinv = cv.take<double>((size_t)t * mb * r * r);
    uint8_t* sing = cv.take<uint8_t>((size_t)t * mb);
    float* dsig = cv.take<float>((size_t)t * mb);
    if (cv.used > OA_NOALLOC_SCRATCH_BYTES)
        return fail(OA_ERR_UNSUPPORTED,
                    "oa_scan_dense_noalloc: n=%d t=%d mb=%d r=%d needs more than the %u-byte scratch array", n, t, mb,
                    r, (unsigned)OA_NOALLOC_SCRATCH_BYTES);

    // everything that must start at zero
    NA_CU(cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned long long), st));
    NA_CU(cudaMemsetAsync(info, 0, 8 * sizeof(int), st));
    NA_CU(cudaMemsetAsync(has_nan, 0, sizeof(int), st));

    // covariates: shifted CholeskyQR3 gives an orthonormal basis in FP64 (Q1 -> Q64 -> Q1), then the
    // block engine's rank rule on the singular values of R
    const double shift_u = 11.0 * ((double)n * l + (double)l * (l + 1)) * 0x1p-53;
    const int LL = OA_MAX_L * OA_MAX_L;
    k_na_gram<float><<<dim3(l, l), 256, 0, st>>>(xl, n, l, G);
    k_na_cholq<float><<<1, 256, 0, st>>>(xl, n, l, LP, shift_u, G, Q1, Rf, nullptr, info + 2);
    k_na_gram<double><<<dim3(l, l), 256, 0, st>>>(Q1, n, l, G);
    k_na_cholq<double><<<1, 256, 0, st>>>(Q1, n, l, LP, 0.0, G, Q64, Rf + LL, nullptr, info + 3);
    k_na_gram<double><<<dim3(l, l), 256, 0, st>>>(Q64, n, l, G);
    k_na_cholq<double><<<1, 256, 0, st>>>(Q64, n, l, LP, 0.0, G, Q1, Rf + 2 * LL, Qr, info + 4);
    k_na_rank<<<1, 1, 0, st>>>(Rf, Rf + LL, Rf + 2 * LL, l, info + 2, info + 5);
    Q64 = Q1;
    // traits: missing counts, sums, Q'y; one row set per trait
    TraitStatsOut tso{tsums, tcounts, thash};
    k_trait_stats<<<t, OA_NTHREADS, 0, st>>>(y, (size_t)n, n, l, Q64, tso);
    k_na_sets<<<1, 1, 0, st>>>(tcounts, t, pat, zset, tperm, set_off, set_rep, set_kind, set_slot, info);
    NA_CU(cudaGetLastError());
    int hinfo[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    NA_CU(cudaMemcpyAsync(hinfo, info, sizeof hinfo, cudaMemcpyDeviceToHost, st));
    NA_CU(cudaStreamSynchronize(st));
    if (hinfo[2] || hinfo[3] || hinfo[4])
        return fail(OA_ERR_COLLINEAR, "the covariate matrix contains linearly dependent columns (its QR broke down)");
    if (hinfo[5])
        return fail(OA_ERR_COLLINEAR,
                    "the covariate matrix contains linearly dependent columns (singular value below 1e-6)");
    const int Z = hinfo[0], nrows = hinfo[1], nsets = t + Z;
    int* set_rows = cv.take<int>((size_t)(nrows > 0 ? nrows : 1));
    float* qrows = cv.take<float>((size_t)(nrows > 0 ? nrows : 1) * LP);
    float* zA = cv.take<float>((size_t)(Z > 0 ? Z : 1) * mb * l * r);
    float* zD = cv.take<float>((size_t)(Z > 0 ? Z : 1) * mb * r * r);
    float* aobs = Z > 0 ? cv.take<float>((size_t)t * mb * l * r) : nullptr;
    if (cv.used > OA_NOALLOC_SCRATCH_BYTES)
        return fail(OA_ERR_UNSUPPORTED,
                    "oa_scan_dense_noalloc: these inputs need %zu bytes of scratch, the array holds %u", cv.used,
                    (unsigned)OA_NOALLOC_SCRATCH_BYTES);
    k_set_rows<<<nsets, OA_NTHREADS, 0, st>>>(y, (size_t)n, n, set_rep, set_kind, set_off, set_rows);
    k_set_gram<<<nsets, OA_NTHREADS, 0, st>>>(Q64, n, l, set_kind, set_off, set_rows, W, zQ, set_slot, pat_bad);
    if (nrows > 0)
        k_set_qrows<<<(unsigned)(((long long)nrows * LP + 255) / 256), 256, 0, st>>>(set_rows, nrows, Qr, LP, qrows);
    k_trait_resid<<<t, OA_NTHREADS, 0, st>>>(y, (size_t)n, n, n_pad, l, l + r, Q64, tsums, tcounts, pat, W, tperm,
                                            Yt, nullptr, nullptr, rss0, sst, nobs, b0, a_r2, inv_ncorr, vf);
    NA_CU(cudaGetLastError());

    // per-SNP statistics (same geometry rule as the block engine)
    const int nS = (n + 3) & ~3;
    const size_t limit = 227 * 1024 - 1024;
    const int NA = r * r + LP * r;
    int spb = 8 / r < 64 / NA ? 8 / r : (64 / NA > 0 ? 64 / NA : 1);
    int nbuf = 2;
    while (spb > 1 && (size_t)nbuf * spb * r * nS * 4 > 170 * 1024) --spb;
    if ((size_t)nbuf * spb * r * nS * 4 > 170 * 1024) nbuf = 1;
    const size_t base = stats_smem_bytes(r, LP, n, spb, nbuf, 0);
    if (base + (size_t)spb * NA * 4 > limit) return fail(OA_ERR_UNSUPPORTED, "n = %d is too large", n);
    int spp = (int)((limit - base) / ((size_t)spb * NA * 4));
    if (spp > nsets) spp = nsets;
    if (spp < 1) spp = 1;
    StatsArgs A{};
    A.X = xr;
    A.ldx = (size_t)n;
    A.n = n;
    A.n_pad = n_pad;
    A.l = l;
    A.QS = LP;
    A.mb = mb;
    A.spb = spb;
    A.Qr = Qr;
    A.nsets = nsets;
    A.G = t;
    A.Z = Z;
    A.set_off = set_off;
    A.rows = set_rows;
    A.qrows = qrows;
    A.W = W;
    A.pat_bad = pat_bad;
    A.sets_per_pass = spp;
    A.mean = mean;
    A.has_nan = has_nan;
    A.sinv = sinv;
    A.sing = sing;
    A.varx = varx;
    A.aobs = aobs;
    A.zA = zA;
    A.zD = zD;
    A.nbuf = nbuf;
    A.err = reinterpret_cast<int*>(counters + 3);
    int sms = 148;
    NA_CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int groups = (mb + spb - 1) / spb;
    NA_CU(oa_launch_snp_stats(r, LP, A, groups < sms ? groups : sms, stats_smem_bytes(r, LP, n, spb, nbuf, spp), st));

    // XR'Y~ with the fused statistics, dense outputs only
    EpiArgs E{};
    E.n = n;
    E.l = l;
    E.r = r;
    E.p = l + r;
    E.mb = mb;
    E.G = t;
    E.pat = pat;
    E.zset = zset;
    E.tperm = tperm;
    E.rss0 = rss0;
    E.a_r2 = a_r2;
    E.inv_ncorr = inv_ncorr;
    E.vf = vf;
    E.b0 = b0;
    E.sinv = sinv;
    E.varx = varx;
    E.sing = sing;
    E.aobs = aobs;
    E.zA = zA;
    E.zD = zD;
    E.zQ = zQ;
    E.W = W;
    E.store_all = 1;
    E.rec = nullptr;
    E.rec_count = counters;
    E.rec_valid = nullptr;
    E.cap = 0;
    E.n_singular = counters + 1;
    E.d_beta = beta;
    E.d_se = se;
    E.d_t = tstat;
    E.d_r2 = r2;
    E.d_sig = dsig;
    E.t = t;
    E.snp_base = 0;
    E.dense_ld = mb;
    NA_CU(oa_launch_gemm_simt(r, xr, (size_t)n, mb * r, Yt, (size_t)n_pad, t, n, mean, has_nan, 0, E, st));
    unsigned long long hc[4];
    NA_CU(cudaMemcpyAsync(hc, counters, sizeof hc, cudaMemcpyDeviceToHost, st));
    NA_CU(cudaStreamSynchronize(st));
    if (hc[3]) return fail(OA_ERR_CUDA, "a device staging wait timed out");
    return OA_OK;
}
