// Block engine of the B200 association engine: device memory, kernel
// sequencing and the C ABI declared in include/omicabel_b200.h.
//
// Per trait block (≙ src/Algorithm.cpp:550-595):
//   k_trait_stats -> host groups traits by missingness pattern (and by the
//   set of observed exact zeros) -> k_set_rows -> k_set_gram -> k_trait_resid
// Per SNP chunk (≙ src/Algorithm.cpp:610-813):
//   k_snp_lean -> pre-GEMM [Q | Q o m_1 | ...]'X -> k_schur   (few row sets)
//   or k_snp_stats (one kernel with row gathers; many row sets)
//   -> XR'Y~ GEMM with fused statistics epilogue -> (covariate terms)
// Per API call: sort of the stored rows into reference order (trait, SNP).
#include <algorithm>
#include <chrono>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include <cub/cub.cuh>

#include "oa_cov.cuh"
#include "oa_kernels.cuh"
#include "oa_launch.h"
#include "oa_lean.cuh"
#include "oa_trace.h"

using namespace oa;

namespace {

thread_local std::string g_err;

void set_err(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}

#define OA_CU(x)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess) {                                                              \
            set_err("%s:%d: %s: %s", __FILE__, __LINE__, #x, cudaGetErrorString(e_));         \
            return OA_ERR_CUDA;                                                               \
        }                                                                                     \
    } while (0)

// Drop an error left by an earlier runtime call whose status was already
// handled (or deliberately ignored), so that the launch checks of this entry
// point report only their own launches.
inline void clear_stale_error(const char* where) {
    const cudaError_t s = cudaGetLastError();
    if (s != cudaSuccess && getenv("OA_DEBUG")) fprintf(stderr, "[oa] stale CUDA error before %s: %s\n", where,
                                                        cudaGetErrorString(s));
}

#define OA_CHECK(x)                    \
    do {                               \
        oa_status s_ = (x);            \
        if (s_ != OA_OK) return s_;    \
    } while (0)

// Stream on which the calling thread's engine allocates: device buffers use
// the stream-ordered allocator (cudaMallocAsync / cudaFreeAsync on the
// engine's stream), so one engine growing a buffer never waits for, or
// stalls, the work of other engines on the same GPU.
thread_local cudaStream_t g_alloc_stream = nullptr;

struct AllocOn {   // scope in which an entry point allocates on its engine's stream
    cudaStream_t prev;
    explicit AllocOn(cudaStream_t s) : prev(g_alloc_stream) { g_alloc_stream = s; }
    ~AllocOn() { g_alloc_stream = prev; }
};

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    oa_status ensure(size_t cnt) {
        if (cnt <= n && p) return OA_OK;
        if (p) cudaFreeAsync(p, g_alloc_stream);
        p = nullptr;
        n = 0;
        if (cnt == 0) cnt = 1;
        if (cudaMallocAsync(reinterpret_cast<void**>(&p), cnt * sizeof(T), g_alloc_stream) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            set_err("device allocation of %zu bytes failed", cnt * sizeof(T));
            return OA_ERR_NOMEM;
        }
        n = cnt;
        return OA_OK;
    }
    void release() {
        if (p) cudaFreeAsync(p, g_alloc_stream);
        p = nullptr;
        n = 0;
    }
};

int pad_l(int l) { return l <= 4 ? 4 : (l <= 8 ? 8 : 16); }

// Page-locked host buffers shared by every engine of the process, pooled by
// size: an engine takes the smallest idle buffer that holds what it asks for
// (at most twice that) and gives its buffers back when it is destroyed.
// cudaMallocHost is slow while other engines keep the GPU busy and
// cudaFreeHost waits for the whole device, so a server that creates an
// engine per request (each with its own individuals and covariates) must not
// pay either per request.  Idle buffers beyond PINNED_KEEP bytes are freed,
// largest first.
constexpr size_t PINNED_KEEP = 16ull << 30;
struct PinnedPool {
    std::mutex mu;
    std::multimap<size_t, void*> idle;
    size_t idle_bytes = 0;
    void* take(size_t bytes, size_t* got) {
        {
            std::lock_guard<std::mutex> g(mu);
            auto it = idle.lower_bound(bytes);
            if (it != idle.end() && it->first <= 2 * bytes + (1u << 20)) {
                void* p = it->second;
                *got = it->first;
                idle_bytes -= it->first;
                idle.erase(it);
                return p;
            }
        }
        void* p = nullptr;
        if (cudaMallocHost(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        *got = bytes;
        return p;
    }
    void give(void* p, size_t bytes) {
        if (!p) return;
        std::lock_guard<std::mutex> g(mu);
        idle.emplace(bytes, p);
        idle_bytes += bytes;
        while (idle_bytes > PINNED_KEEP && !idle.empty()) {
            auto it = std::prev(idle.end());
            cudaFreeHost(it->second);
            idle_bytes -= it->first;
            idle.erase(it);
        }
    }
};
PinnedPool& pinned_pool() {
    static PinnedPool* pool = new PinnedPool();   // never destroyed: engines may outlive static destructors
    return *pool;
}

// Grow a pinned host buffer (page-locked so the device-to-host copy runs at
// full speed), doubling so that growth is rare.  Outgrown buffers go to
// `retired` (pointer, bytes) and back to the pool when the engine is
// destroyed.  Serving engines reserve their buffers up front (oa_reserve).
template <class T>
oa_status ensure_pinned(T*& p, size_t& cap, size_t want, std::vector<std::pair<void*, size_t>>& retired) {
    if (want <= cap && p) return OA_OK;
    if (p) retired.emplace_back(p, cap * sizeof(T));
    p = nullptr;
    const size_t n = std::max<size_t>({want + want / 4, 2 * cap, 1024});
    cap = 0;
    size_t got = 0;
    p = static_cast<T*>(pinned_pool().take(n * sizeof(T), &got));
    if (!p) {
        set_err("pinned host allocation of %zu bytes failed", n * sizeof(T));
        return OA_ERR_NOMEM;
    }
    cap = got / sizeof(T);
    return OA_OK;
}

// Host-to-device copies of int tables, issued from the engine's pinned
// staging area in one batch (the area is reused only after the stream has
// been synchronised).
struct H2DBatch {
    std::vector<std::pair<int*, const std::vector<int>*>> items;
    void add(int* dst, const std::vector<int>& v) { items.emplace_back(dst, &v); }
};

// Householder QR of the n x l column-major matrix A (FP64): Q (n x l,
// column-major, orthonormal columns) and R (l x l, row-major upper
// triangular) with a positive diagonal.
void householder_qr(const std::vector<double>& A, int n, int l, std::vector<double>& Q, std::vector<double>& R) {
    std::vector<double> Wm(A);
    std::vector<std::vector<double>> V(l);
    for (int k = 0; k < l; ++k) {
        double nrm = 0.0;
        for (int i = k; i < n; ++i) nrm += Wm[(size_t)k * n + i] * Wm[(size_t)k * n + i];
        nrm = std::sqrt(nrm);
        const double x0 = Wm[(size_t)k * n + k];
        const double alpha = x0 >= 0 ? -nrm : nrm;
        std::vector<double> v(n - k);
        for (int i = k; i < n; ++i) v[i - k] = Wm[(size_t)k * n + i];
        v[0] -= alpha;
        double vn = 0.0;
        for (double e : v) vn += e * e;
        vn = std::sqrt(vn);
        if (vn > 0)
            for (double& e : v) e /= vn;
        for (int c = k; c < l; ++c) {
            double d = 0.0;
            for (int i = k; i < n; ++i) d += v[i - k] * Wm[(size_t)c * n + i];
            for (int i = k; i < n; ++i) Wm[(size_t)c * n + i] -= 2.0 * d * v[i - k];
        }
        V[k] = std::move(v);
    }
    R.assign((size_t)l * l, 0.0);
    for (int i = 0; i < l; ++i)
        for (int j = i; j < l; ++j) R[(size_t)i * l + j] = Wm[(size_t)j * n + i];
    Q.assign((size_t)n * l, 0.0);
    for (int c = 0; c < l; ++c) Q[(size_t)c * n + c] = 1.0;
    for (int k = l - 1; k >= 0; --k) {
        const std::vector<double>& v = V[k];
        for (int c = 0; c < l; ++c) {
            double d = 0.0;
            for (int i = k; i < n; ++i) d += v[i - k] * Q[(size_t)c * n + i];
            for (int i = k; i < n; ++i) Q[(size_t)c * n + i] -= 2.0 * d * v[i - k];
        }
    }
    for (int i = 0; i < l; ++i)
        if (R[(size_t)i * l + i] < 0) {
            for (int j = 0; j < l; ++j) R[(size_t)i * l + j] = -R[(size_t)i * l + j];
            for (int k = 0; k < n; ++k) Q[(size_t)i * n + k] = -Q[(size_t)i * n + k];
        }
}

// Singular values of a small square matrix (one-sided Jacobi, FP64).
std::vector<double> singular_values(std::vector<double> A /* row-major k x k */, int k) {
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < k; ++p)
            for (int q = p + 1; q < k; ++q) {
                double a = 0, b = 0, c = 0;
                for (int i = 0; i < k; ++i) {
                    a += A[(size_t)i * k + p] * A[(size_t)i * k + p];
                    b += A[(size_t)i * k + q] * A[(size_t)i * k + q];
                    c += A[(size_t)i * k + p] * A[(size_t)i * k + q];
                }
                if (std::fabs(c) <= 1e-300) continue;
                off = std::max(off, std::fabs(c) / std::sqrt(a * b));
                const double zeta = (b - a) / (2 * c);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1 + zeta * zeta));
                const double cs = 1 / std::sqrt(1 + t * t), sn = cs * t;
                for (int i = 0; i < k; ++i) {
                    const double x = A[(size_t)i * k + p], y = A[(size_t)i * k + q];
                    A[(size_t)i * k + p] = cs * x - sn * y;
                    A[(size_t)i * k + q] = sn * x + cs * y;
                }
            }
        if (off < 1e-15) break;
    }
    std::vector<double> s(k);
    for (int p = 0; p < k; ++p) {
        double a = 0;
        for (int i = 0; i < k; ++i) a += A[(size_t)i * k + p] * A[(size_t)i * k + p];
        s[p] = std::sqrt(a);
    }
    return s;
}

}  // namespace

// Pieces in which the stored rows come back to the host (converted while the next piece copies).
constexpr int RESULT_PIECES = 8;

struct oa_engine {
    oa_config cfg{};
    // r: columns per SNP in the kernels (1, 2, 4 or 8); ru: the caller's (1..8, p = l + ru); columns
    // [ru, r) are zero padding added on the device
    int n = 0, l = 0, r = 0, ru = 0, p = 0, LP = 4, n_pad = 0, sm_count = 148;
    cudaStream_t st = nullptr, cp = nullptr;
    cudaEvent_t ev_copied[2]{}, ev_used[2]{}, k0 = nullptr, k1 = nullptr;
    long long launches = 0;
    float last_ms = 0.f;
    float stats_ms = 0.f;
    float block_ms = 0.f;   // device time of the last SNP block on the engine's stream (events k0, k1)
    cudaEvent_t s0 = nullptr, s1 = nullptr;
    const char* last_name = "";
    // covariates
    DBuf<double> Q64, Rinv;
    DBuf<float> Qr;
    DBuf<float> Qb;      // [n_pad / 4][l][4] the basis by blocks of four rows (k_snp_lean's projection)
    DBuf<double> qsum;   // [l] column sums of the FP32 basis
    DBuf<double> Afull_lean;   // [chunk*r][LEAN_QX_L] all-rows projection from k_snp_lean
    bool have_cov = false;
    bool center = false;   // the first covariate is constant: SNP columns are taken relative to their means
    bool fuse_split = false;  // the tensor-core GEMMs split FP32 columns in shared memory where they can
    bool fused_last = false;  // the last enqueued chunk took the fused form
    // traits
    int t = 0;
    DBuf<float> Yraw, Yt;
    DBuf<__nv_bfloat16> Yhi, Ylo;
    DBuf<double> tsums, rss0, b0, W, zQ;
    DBuf<int> tcounts, pat, zset, nobs, set_off, set_rows, set_rep, set_kind, set_slot, tperm, tinv;
    DBuf<float> a_r2, inv_ncorr, vf;
    DBuf<unsigned long long> thash;
    DBuf<int> tcheck;            // per trait: its pattern's and zero set's representatives; collision flag
    int hash_bits = 64;          // hash-sum bits used for grouping (fewer only to test the exact regrouping)
    bool trait_regrouped = false;   // the last trait block was regrouped on exact row masks
    DBuf<float> sst, qrows;
    DBuf<uint8_t> pat_bad;
    int G = 0, Z = 0, nsets = 0;
    // pre-GEMM column matrix [Q | Q o m_1 | ... | Q o m_S] (c2 = l (1 + S) rows of n_pad)
    bool use_pre = false, b2_ready = false;
    int c2 = 0;
    // tuning: requested (0 = automatic) and in effect
    oa_tuning req{};
    int variant = 1, raster = 1, lean_spb = 0;
    // statistics-kernel layout requests (environment; 0 / -1 = the plan's choice): column buffers (1, 2)
    // and the row-interleaved column copy of the set pass (0, 1)
    int lean_nbuf = 0, lean_xi = -1;
    int lean_threads_req = 0;   // 256 or 512 threads per column-statistics CTA (OA_LEAN_THREADS), 0: by n
    // work items of the lean kernel's set pass (per trait block) and its launch plan
    DBuf<int> item_start, set_item_off, pass_off;
    std::vector<int> h_set_item_off;
    struct LeanPlan {
        int spb = 0, nbuf = 0, items_cap = 0, npass = 0;
        bool xi = true;   // row-interleaved column copy for the set pass
        size_t smem = 0;
    } lp;
    long long tune_gen = 0;
    DBuf<float> B2;
    DBuf<__nv_bfloat16> B2hi, B2lo;
    std::vector<int> h_nobs;
    // SNP chunk buffers
    int chunk = 0;
    DBuf<float> Xstage[2];
    // column model (dosage models): each SNP arrives as in_cols file columns and its r columns are
    // formed on the device; in_cols = 0: the input already holds r columns per SNP
    int in_cols = 0, model_combine = 0;
    float model_w[OA_MODEL_MAX_COLS] = {};
    DBuf<float> Xmodel;
    // interaction columns (n x n_inter, the engine's rows): the model column x becomes
    // [I_1 x, ..., I_k x (, x)] (src/AIOwrapper.cpp:808-840)
    DBuf<float> inter;
    int n_inter = 0, inter_keep = 0;
    DBuf<__nv_bfloat16> Xhi, Xlo;
    DBuf<float> mean, varx, aobs, afull, zA, zD;
    DBuf<float> D, Dset, C2T;   // pre-GEMM path: X'X, per-set X'X, pre-GEMM output
    DBuf<float> C2part;         // plain pre-GEMM: partial product of the second K half
    DBuf<int> has_nan;
    DBuf<double> sinv, sfinv;
    DBuf<float> qdel;           // quirk mode: per (pattern, SNP) terms of the reference's r >= 2 downdate
    DBuf<double> qK;
    DBuf<uint8_t> sing;
    // stored rows
    DBuf<Rec> rec, rec2;
    DBuf<float> cov, cov2;
    long long cap = 0;
    DBuf<unsigned long long> counters;  // [0] record slots, [1] singular, [2] significant covariate terms,
                                        // [3] pipeline error, [4] rows written
    DBuf<unsigned long long> marks;     // stored-row count at the start of each chunk's GEMM
    DBuf<unsigned long long> keys, keys2;
    DBuf<int> perm, perm2;
    DBuf<unsigned char> cub_tmp;
    // whole-scan CUDA graph of the device-resident path
    struct GraphKey {
        const float* xr = nullptr;
        int mb = 0, t = 0, dense = 0;
        long long gen = 0, cap = 0;
        const void* rec = nullptr;
        long long tune = 0;
        bool operator==(const GraphKey& o) const {
            return xr == o.xr && mb == o.mb && t == o.t && dense == o.dense && gen == o.gen && cap == o.cap &&
                   rec == o.rec && tune == o.tune;
        }
    };
    GraphKey gkey, warm_key;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    long long graph_launches = 0;
    long long trait_gen = 0;
    std::vector<cudaEvent_t> cev0, cev1, sev0, sev1;
    bool use_graphs = true;
    // dense outputs
    bool dense_on = false;
    DBuf<float> d_beta, d_se, d_t, d_r2, d_sig;
    DBuf<uint8_t> d_flags;
    // row subset of device SNP blocks: columns of x_ld floats, rows xrows[0..n)
    DBuf<int> xrows;
    long long x_ld = 0;
    bool subset = false;
    long long dense_ld = 0;
    int last_mb = 0;
    // host results (pinned staging for the device-to-host copy)
    Rec* h_rec = nullptr;
    size_t h_rec_cap = 0;
    float* h_cov = nullptr;
    size_t h_cov_cap = 0;
    std::vector<std::pair<void*, size_t>> retired_pinned;   // outgrown pinned buffers, back to the pool at destroy
    // pinned staging of the small host <-> device transfers (trait grouping,
    // row-set tables, counters): asynchronous copies that need no driver staging
    unsigned char* stage = nullptr;
    size_t stage_cap = 0;
    unsigned long long* h_cnt = nullptr;   // 8 counters read back after each block
    size_t h_cnt_bytes = 0;
    cudaEvent_t ev_piece[RESULT_PIECES] = {};  // the stored rows' pieces have reached the host
    std::vector<int32_t> o_trait, o_snp, o_nused;
    std::vector<float> o_r2, o_b, o_se, o_t;
    std::vector<uint32_t> o_mask;
};

namespace {

// Engines alive per device (their memory stays pooled while any is alive).
int live_engines(int device, int delta) {
    static std::mutex mu;
    static int count[64];
    std::lock_guard<std::mutex> g(mu);
    count[device & 63] += delta;
    return count[device & 63];
}

// Every device buffer of an engine (release, footprint).
template <class F>
void for_each_buf(oa_engine* e, F&& f) {
    f(e->Q64); f(e->Rinv); f(e->Qr); f(e->Qb); f(e->qsum); f(e->Afull_lean);
    f(e->Yraw); f(e->Yt); f(e->Yhi); f(e->Ylo);
    f(e->tsums); f(e->rss0); f(e->b0); f(e->W); f(e->zQ);
    f(e->tcounts); f(e->pat); f(e->zset); f(e->nobs); f(e->set_off); f(e->set_rows); f(e->set_rep);
    f(e->set_kind); f(e->set_slot); f(e->tperm); f(e->tinv);
    f(e->a_r2); f(e->inv_ncorr); f(e->vf); f(e->thash); f(e->tcheck); f(e->sst); f(e->qrows); f(e->pat_bad);
    f(e->B2); f(e->B2hi); f(e->B2lo);
    f(e->Xstage[0]); f(e->Xstage[1]); f(e->Xmodel); f(e->inter); f(e->Xhi); f(e->Xlo);
    f(e->mean); f(e->varx); f(e->aobs); f(e->afull); f(e->zA); f(e->zD); f(e->D); f(e->Dset); f(e->C2T);
    f(e->C2part);
    f(e->has_nan); f(e->sinv); f(e->sfinv); f(e->sing); f(e->qdel); f(e->qK);
    f(e->rec); f(e->rec2); f(e->cov); f(e->cov2); f(e->counters); f(e->keys); f(e->keys2); f(e->perm);
    f(e->perm2); f(e->cub_tmp);
    f(e->d_beta); f(e->d_se); f(e->d_t); f(e->d_r2); f(e->d_sig); f(e->d_flags); f(e->xrows);
    f(e->item_start); f(e->set_item_off); f(e->pass_off); f(e->marks);
}

// Columns [c0, c0 + ncol) of a strided block gathered to the engine's rows.
static __global__ void k_gather_rows(const float* __restrict__ in, long long ld, const int* __restrict__ rows, int n,
                                     float* __restrict__ out) {
    const int c = blockIdx.y;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) out[(size_t)c * n + j] = __ldg(in + (size_t)c * ld + __ldg(rows + j));
}

// Device input of one chunk: the block itself, or its row-subset gather.
// The column model of one chunk (the reference's dosage models,
// src/AIOwrapper.cpp:257-340, 1213-1275): SNP i's in_cols file columns ->
// combine: one column sum_c w[c] * x_c (additive, dominant, recessive and
// custom additive models); otherwise in_cols columns w[c] * x_c (custom
// linear model).  NaN propagates (mean imputation follows, as in the reference).
struct ModelW {
    float w[OA_MODEL_MAX_COLS];
};
// SNP i's columns go to out_r columns of `out`: the model's columns first,
// zero padding after them (engines whose kernels take 4 or 8 columns per SNP
// for r = 3, 5, 6, 7).
static __global__ void k_column_model(const float* __restrict__ in, int n, int in_cols, ModelW W, int combine,
                                      const float* __restrict__ inter, int n_inter, int keep, int out_r,
                                      float* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (k >= n) return;
    const float* src = in + (size_t)i * in_cols * n + k;
    float* dst = out + (size_t)i * out_r * n + k;
    int written;
    if (combine) {   // a zero factor drops its column (the reference does not read it)
        float acc = 0.f;
        bool any = false;
        for (int c = 0; c < in_cols; ++c) {
            if (W.w[c] == 0.f) continue;
            const float x = src[(size_t)c * n];
            acc = any ? fmaf(W.w[c], x, acc) : W.w[c] * x;
            any = true;
        }
        if (n_inter == 0) {
            dst[0] = acc;
            written = 1;
        } else {   // [I_1 x, ..., I_k x (, x)] (src/AIOwrapper.cpp:808-840)
            for (int h = 0; h < n_inter; ++h) dst[(size_t)h * n] = inter[(size_t)h * n + k] * acc;
            if (keep) dst[(size_t)n_inter * n] = acc;
            written = n_inter + keep;
        }
    } else {
        for (int c = 0; c < in_cols; ++c) dst[(size_t)c * n] = W.w[c] * src[(size_t)c * n];
        written = in_cols;
    }
    for (int c = written; c < out_r; ++c) dst[(size_t)c * n] = 0.f;
}

// The reference's r >= 2 downdate is reproduced (quirk mode; with r = 1 it
// changes nothing).  It needs raw, uncentred SNP columns and the pre-GEMM
// statistics path.
bool quirk_on(const oa_engine* e) { return e->cfg.quirk_r2 && e->r >= 2; }

// Columns per SNP of the caller's SNP blocks.
int input_cols(const oa_engine* e) { return e->in_cols > 0 ? e->in_cols : e->ru; }

// The kernels take more columns per SNP than the caller's blocks hold (r = 3, 5, 6, 7): every chunk
// goes through k_column_model, which adds the zero columns.
bool padded(const oa_engine* e) { return e->ru != e->r; }

// A chunk passes through k_column_model (a dosage model, interactions or zero padding).
bool column_pass(const oa_engine* e) { return e->in_cols > 0 || padded(e); }

// Mixed form with the pre-GEMM statistics path: nothing after the column
// statistics reads the FP32 chunk (the GEMMs read its BF16 split), so a row
// subset is gathered by the statistics kernel as it stages the columns.
bool lean_gathers(const oa_engine* e) {
    return e->subset && e->use_pre && e->cfg.precision == OA_MIXED_BF16X3;
}

template <int R>
oa_status chunk_input(oa_engine* e, const float* xr, int c0, int mbc, const float** X) {
    if (!e->subset) {
        *X = xr + (size_t)c0 * R * e->n;
        return OA_OK;
    }
    dim3 grid((unsigned)((e->n + 255) / 256), (unsigned)(mbc * R));
    k_gather_rows<<<grid, 256, 0, e->st>>>(xr + (size_t)c0 * R * e->x_ld, e->x_ld, e->xrows.p, e->n, e->Xstage[0].p);
    ++e->launches;
    OA_CU(cudaGetLastError());
    *X = e->Xstage[0].p;
    return OA_OK;
}

oa_status stage_reserve(oa_engine* e, size_t bytes) {
    return ensure_pinned(e->stage, e->stage_cap, bytes, e->retired_pinned);
}

oa_status flush_h2d(oa_engine* e, const H2DBatch& b) {
    size_t total = 0;
    for (const auto& it : b.items) total += (it.second->size() + 3) & ~size_t(3);
    OA_CHECK(stage_reserve(e, total * sizeof(int)));
    int* h = reinterpret_cast<int*>(e->stage);
    for (const auto& it : b.items) {
        const size_t k = it.second->size();
        if (k == 0) continue;
        std::memcpy(h, it.second->data(), k * sizeof(int));
        OA_CU(cudaMemcpyAsync(it.first, h, k * sizeof(int), cudaMemcpyHostToDevice, e->st));
        h += (k + 3) & ~size_t(3);
    }
    return OA_OK;
}

// The traits are grouped by (count, two hash sums) of their NaN rows and of
// their observed exact-zero rows.  Equal keys are checked on the device
// against the group's representative row by row; if any trait's rows differ
// (a hash collision), the traits are regrouped on their exact row masks, with
// groups numbered in order of first appearance as the hash grouping does.
oa_status exact_trait_sets(oa_engine* e, const float* Y, int t, const std::vector<int>& counts,
                           std::vector<int>& hpat, std::vector<int>& hz, std::vector<int>& prep,
                           std::vector<int>& zrep, std::vector<int>& pcnt, std::vector<int>& zcnt) {
    const int n = e->n;
    std::vector<int> rep((size_t)2 * t);
    for (int j = 0; j < t; ++j) {
        rep[2 * j] = prep[hpat[j]];
        rep[2 * j + 1] = hz[j] >= 0 ? zrep[hz[j]] : -1;
    }
    OA_CHECK(e->tcheck.ensure((size_t)2 * t + 4));
    H2DBatch h2d;
    h2d.add(e->tcheck.p, rep);
    OA_CHECK(flush_h2d(e, h2d));
    int* bad = e->tcheck.p + 2 * t;
    OA_CU(cudaMemsetAsync(bad, 0, sizeof(int), e->st));
    k_trait_set_check<<<t, OA_NTHREADS, 0, e->st>>>(Y, (size_t)n, n, e->tcheck.p, bad);
    ++e->launches;
    OA_CU(cudaGetLastError());
    OA_CU(cudaMemcpyAsync(e->stage, bad, sizeof(int), cudaMemcpyDeviceToHost, e->st));
    OA_CU(cudaStreamSynchronize(e->st));
    int hbad = 0;
    std::memcpy(&hbad, e->stage, sizeof(int));
    e->trait_regrouped = hbad != 0;
    if (!hbad) return OA_OK;
    const int nw = (n + 31) / 32;
    const size_t words = (size_t)2 * t * nw;
    DBuf<unsigned> masks;
    struct Release {
        DBuf<unsigned>& b;
        ~Release() { b.release(); }
    } release_masks{masks};
    OA_CHECK(masks.ensure(words));
    k_trait_masks<<<t, OA_NTHREADS, 0, e->st>>>(Y, (size_t)n, n, nw, masks.p);
    ++e->launches;
    OA_CU(cudaGetLastError());
    std::vector<unsigned> hm(words);
    OA_CU(cudaMemcpyAsync(hm.data(), masks.p, words * sizeof(unsigned), cudaMemcpyDeviceToHost, e->st));
    OA_CU(cudaStreamSynchronize(e->st));
    std::map<std::vector<unsigned>, int> pmap, zmap;
    prep.clear(), zrep.clear(), pcnt.clear(), zcnt.clear();
    for (int j = 0; j < t; ++j) {
        std::vector<unsigned> pk(hm.begin() + (size_t)(2 * j) * nw, hm.begin() + (size_t)(2 * j + 1) * nw);
        auto it = pmap.find(pk);
        if (it == pmap.end()) {
            it = pmap.emplace(std::move(pk), (int)prep.size()).first;
            prep.push_back(j);
            pcnt.push_back(counts[j * 2]);
        }
        hpat[j] = it->second;
        hz[j] = -1;
        if (counts[j * 2 + 1] > 0) {
            std::vector<unsigned> zk(hm.begin() + (size_t)(2 * j + 1) * nw, hm.begin() + (size_t)(2 * j + 2) * nw);
            auto zt = zmap.find(zk);
            if (zt == zmap.end()) {
                zt = zmap.emplace(std::move(zk), (int)zrep.size()).first;
                zrep.push_back(j);
                zcnt.push_back(counts[j * 2 + 1]);
            }
            hz[j] = zt->second;
        }
    }
    return OA_OK;
}

oa_status set_traits_impl(oa_engine* e, const float* y, int32_t t, bool device_ptr) {
    OA_TRACE("oa_set_traits: grouping, row sets, residuals");
    if (!e->have_cov) {
        set_err("oa_set_traits before oa_set_covariates");
        return OA_ERR_STATE;
    }
    if (t <= 0 || t > e->cfg.max_traits) {
        set_err("trait block of %d traits (engine limit %d)", t, e->cfg.max_traits);
        return OA_ERR_ARG;
    }
    const int n = e->n, l = e->l;
    e->t = t;
    ++e->trait_gen;
    const float* Y = y;
    if (!device_ptr) {
        OA_CHECK(e->Yraw.ensure((size_t)n * t));
        OA_CU(cudaMemcpyAsync(e->Yraw.p, y, sizeof(float) * (size_t)n * t, cudaMemcpyHostToDevice, e->st));
        Y = e->Yraw.p;
    }
    OA_CHECK(e->tsums.ensure((size_t)t * (2 + OA_MAX_L)));
    OA_CHECK(e->tcounts.ensure((size_t)t * 2));
    OA_CHECK(e->thash.ensure((size_t)t * 4));
    TraitStatsOut tso{e->tsums.p, e->tcounts.p, e->thash.p};
    k_trait_stats<<<t, OA_NTHREADS, 0, e->st>>>(Y, (size_t)n, n, l, e->Q64.p, tso);
    ++e->launches;
    OA_CU(cudaGetLastError());
    std::vector<int> counts((size_t)t * 2);
    std::vector<unsigned long long> hashes((size_t)t * 4);
    {
        const size_t hb = sizeof(unsigned long long) * hashes.size(), cb = sizeof(int) * counts.size();
        OA_CHECK(stage_reserve(e, hb + cb));
        OA_CU(cudaMemcpyAsync(e->stage, e->thash.p, hb, cudaMemcpyDeviceToHost, e->st));
        OA_CU(cudaMemcpyAsync(e->stage + hb, e->tcounts.p, cb, cudaMemcpyDeviceToHost, e->st));
        OA_CU(cudaStreamSynchronize(e->st));
        std::memcpy(hashes.data(), e->stage, hb);
        std::memcpy(counts.data(), e->stage + hb, cb);
    }

    if (e->hash_bits < 64)   // test hook: hash sums cut to their low bits make patterns collide
        for (auto& h : hashes) h &= (1ull << e->hash_bits) - 1ull;
    // group traits: missingness patterns, then sets of observed exact zeros
    std::map<std::tuple<int, unsigned long long, unsigned long long>, int> pmap, zmap;
    std::vector<int> hpat(t), hz(t, -1), prep, zrep, pcnt, zcnt;
    for (int j = 0; j < t; ++j) {
        auto key = std::make_tuple(counts[j * 2], hashes[j * 4], hashes[j * 4 + 1]);
        auto it = pmap.find(key);
        if (it == pmap.end()) {
            it = pmap.emplace(key, (int)prep.size()).first;
            prep.push_back(j);
            pcnt.push_back(counts[j * 2]);
        }
        hpat[j] = it->second;
        if (counts[j * 2 + 1] > 0) {
            auto zk = std::make_tuple(counts[j * 2 + 1], hashes[j * 4 + 2], hashes[j * 4 + 3]);
            auto zt = zmap.find(zk);
            if (zt == zmap.end()) {
                zt = zmap.emplace(zk, (int)zrep.size()).first;
                zrep.push_back(j);
                zcnt.push_back(counts[j * 2 + 1]);
            }
            hz[j] = zt->second;
        }
    }
    OA_CHECK(exact_trait_sets(e, Y, t, counts, hpat, hz, prep, zrep, pcnt, zcnt));
    e->G = (int)prep.size();
    e->Z = (int)zrep.size();
    e->nsets = e->G + e->Z;
    if (e->nsets > OA_SETS_MAX) {
        set_err("%d distinct missingness/zero patterns in one trait block (limit %d)", e->nsets, OA_SETS_MAX);
        return OA_ERR_UNSUPPORTED;
    }
    std::vector<int> off(e->nsets + 1, 0), rep(e->nsets), kind(e->nsets), slot(e->nsets);
    for (int s = 0; s < e->nsets; ++s) {
        const bool isz = s >= e->G;
        rep[s] = isz ? zrep[s - e->G] : prep[s];
        kind[s] = isz ? 1 : 0;
        slot[s] = isz ? s - e->G : s;
        off[s + 1] = off[s] + (isz ? zcnt[s - e->G] : pcnt[s]);
    }
    e->h_nobs.resize(t);
    for (int j = 0; j < t; ++j) e->h_nobs[j] = n - counts[j * 2];
    // internal trait order: sorted by (pattern, zero set) so that consecutive
    // traits of a GEMM tile share their per-(pattern, SNP) Schur inverses
    std::vector<int> order(t), inv(t), ipat(t), iz(t);
    for (int j = 0; j < t; ++j) order[j] = j;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return hpat[a] != hpat[b] ? hpat[a] < hpat[b] : hz[a] < hz[b]; });
    for (int jj = 0; jj < t; ++jj) {
        inv[order[jj]] = jj;
        ipat[jj] = hpat[order[jj]];
        iz[jj] = hz[order[jj]];
    }
    OA_CHECK(e->pat.ensure(t));
    OA_CHECK(e->zset.ensure(t));
    OA_CHECK(e->tperm.ensure(t));
    OA_CHECK(e->tinv.ensure(t));
    OA_CHECK(e->set_off.ensure(e->nsets + 1));
    OA_CHECK(e->set_rep.ensure(e->nsets));
    OA_CHECK(e->set_kind.ensure(e->nsets));
    OA_CHECK(e->set_slot.ensure(e->nsets));
    OA_CHECK(e->set_rows.ensure(std::max(off[e->nsets], 1)));
    OA_CHECK(e->W.ensure((size_t)std::max(e->G, 1) * l * l));
    OA_CHECK(e->zQ.ensure((size_t)std::max(e->Z, 1) * l * l));
    OA_CHECK(e->pat_bad.ensure(std::max(e->G, 1)));
    // work items of at most LEAN_ITEM_ROWS rows of one set, tiling the flattened row lists
    std::vector<int> istart;
    e->h_set_item_off.assign(e->nsets + 1, 0);
    for (int s2 = 0; s2 < e->nsets; ++s2) {
        e->h_set_item_off[s2] = (int)istart.size();
        for (int r0 = off[s2]; r0 < off[s2 + 1]; r0 += LEAN_ITEM_ROWS) istart.push_back(r0);
    }
    e->h_set_item_off[e->nsets] = (int)istart.size();
    istart.push_back(off[e->nsets]);
    OA_CHECK(e->item_start.ensure(istart.size()));
    OA_CHECK(e->set_item_off.ensure(e->h_set_item_off.size()));
    H2DBatch h2d;
    h2d.add(e->pat.p, ipat);
    h2d.add(e->zset.p, iz);
    h2d.add(e->tperm.p, order);
    h2d.add(e->tinv.p, inv);
    h2d.add(e->set_off.p, off);
    h2d.add(e->set_rep.p, rep);
    h2d.add(e->set_kind.p, kind);
    h2d.add(e->set_slot.p, slot);
    h2d.add(e->item_start.p, istart);
    h2d.add(e->set_item_off.p, e->h_set_item_off);
    OA_CHECK(flush_h2d(e, h2d));
    k_set_rows<<<e->nsets, OA_NTHREADS, 0, e->st>>>(Y, (size_t)n, n, e->set_rep.p, e->set_kind.p, e->set_off.p,
                                                   e->set_rows.p);
    k_set_gram<<<e->nsets, OA_NTHREADS, 0, e->st>>>(e->Q64.p, n, l, e->set_kind.p, e->set_off.p, e->set_rows.p,
                                                   e->W.p, e->zQ.p, e->set_slot.p, e->pat_bad.p);
    const int total_rows = off[e->nsets];
    OA_CHECK(e->qrows.ensure((size_t)std::max(total_rows, 1) * e->LP));
    if (total_rows > 0) {
        const long long nq = (long long)total_rows * e->LP;
        k_set_qrows<<<(unsigned)((nq + 255) / 256), 256, 0, e->st>>>(e->set_rows.p, total_rows, e->Qr.p, e->LP,
                                                                      e->qrows.p);
        ++e->launches;
    }
    e->launches += 2;
    OA_CU(cudaGetLastError());
    e->c2 = l * (1 + e->nsets);
    e->b2_ready = false;
    e->lp = oa_engine::LeanPlan{};
    OA_CHECK(e->Yt.ensure((size_t)t * e->n_pad));
    if (e->cfg.precision == OA_MIXED_BF16X3) {
        OA_CHECK(e->Yhi.ensure((size_t)t * e->n_pad));
        OA_CHECK(e->Ylo.ensure((size_t)t * e->n_pad));
    }
    OA_CHECK(e->rss0.ensure(t));
    OA_CHECK(e->sst.ensure(t));
    OA_CHECK(e->nobs.ensure(t));
    OA_CHECK(e->b0.ensure((size_t)t * l));
    OA_CHECK(e->a_r2.ensure(t));
    OA_CHECK(e->inv_ncorr.ensure(t));
    OA_CHECK(e->vf.ensure(t));
    const bool mixed = e->cfg.precision == OA_MIXED_BF16X3;
    k_trait_resid<<<t, OA_NTHREADS, 0, e->st>>>(Y, (size_t)n, n, e->n_pad, l, e->p, e->Q64.p, e->tsums.p,
                                               e->tcounts.p, e->pat.p, e->W.p, e->tperm.p, e->Yt.p,
                                               mixed ? e->Yhi.p : nullptr, mixed ? e->Ylo.p : nullptr, e->rss0.p,
                                               e->sst.p, e->nobs.p, e->b0.p, e->a_r2.p, e->inv_ncorr.p, e->vf.p);
    ++e->launches;
    OA_CU(cudaGetLastError());
    OA_CU(cudaStreamSynchronize(e->st));
    return OA_OK;
}

// Resolves the tuning for the current trait block.  Per-SNP covariate sums:
// with few row sets one pre-GEMM of the SNP block with
// [Q | Q o m_1 | ... | Q o m_S] (cost c2 / t of the main GEMM); with many,
// row gathers inside k_snp_stats.  Builds the pre-GEMM's column matrix
// the first time a trait block needs it.
oa_status lean_plan(oa_engine* e);

// Default SNPs per chunk: about 16,384/r, rounded so that the tensor-core
// GEMM's 128 x 256 tiles fill whole waves of the persistent grid (one CTA
// per SM): the M-tile count is a multiple of sm_count / gcd(sm_count, N-tiles).
int wave_chunk(const oa_engine* e, int t) {
    const int r = e->r;
    const int n_tiles = std::max(1, (std::max(t, 1) + 255) / 256);
    int a = e->sm_count, b = n_tiles;
    while (b) {
        const int q = a % b;
        a = b;
        b = q;
    }
    const int unit = e->sm_count / a;                       // M-tiles per whole number of waves
    const int mt = std::max(unit, (16384 / r * r / 128 + unit - 1) / unit * unit);
    return mt * 128 / r;
}

oa_status prepare_tuning(oa_engine* e) {
    const int t = e->t, l = e->l, n = e->n;
    e->chunk = std::min(e->cfg.max_snps, e->req.chunk_snps > 0 ? e->req.chunk_snps : wave_chunk(e, e->t));
    // default pipeline: CTA pairs with 64-wide K-blocks (the fastest at wide trait blocks; blocks of
    // at most 128 traits take the 1-SM narrow tiles whatever the variant)
    e->variant = (e->req.gemm_variant >= 1 && e->req.gemm_variant <= 4) ? e->req.gemm_variant : 4;
    e->raster = e->req.gemm_raster == 2 ? 2 : 1;
    e->lean_spb = e->req.lean_spb > 0 ? std::min(e->req.lean_spb, 8 / e->r) : 0;
    // the row-gather form handles neither the quirk, nor padding columns, nor 8 columns per SNP
    e->use_pre = quirk_on(e) || padded(e) || e->r > 4 || e->req.stats_path == 1 ||
                 (e->req.stats_path != 2 && e->c2 <= std::max(t, 256));
    if (e->use_pre && !e->b2_ready) {
        const size_t nb2 = (size_t)e->c2 * e->n_pad;
        OA_CHECK(e->B2.ensure(nb2));
        k_b2_init<<<(unsigned)((nb2 + 255) / 256), 256, 0, e->st>>>(e->Qr.p, e->LP, n, e->n_pad, l, e->c2, e->B2.p);
        ++e->launches;
        if (e->nsets > 0) {
            k_b2_scatter<<<e->nsets, 256, 0, e->st>>>(e->Qr.p, e->LP, e->n_pad, l, e->set_off.p, e->set_rows.p,
                                                      e->B2.p);
            ++e->launches;
        }
        if (e->cfg.precision == OA_MIXED_BF16X3) {
            OA_CHECK(e->B2hi.ensure(nb2));
            OA_CHECK(e->B2lo.ensure(nb2));
            k_split_bf16<<<(unsigned)((nb2 + 255) / 256), 256, 0, e->st>>>(e->B2.p, (long long)nb2, e->B2hi.p,
                                                                          e->B2lo.p);
            ++e->launches;
        }
        OA_CU(cudaGetLastError());
        e->b2_ready = true;
    }
    if (e->use_pre) OA_CHECK(lean_plan(e));
    return OA_OK;
}

StatsArgs stats_args(oa_engine* e, const float* X, int mbc, int LP, int spb, int spp) {
    StatsArgs A{};
    A.X = X;
    A.ldx = (size_t)e->n;
    A.n = e->n;
    A.n_pad = e->n_pad;
    A.l = e->l;
    A.QS = LP;
    A.mb = mbc;
    A.spb = spb;
    A.Qr = e->Qr.p;
    A.nsets = e->nsets;
    A.G = e->G;
    A.Z = e->Z;
    A.set_off = e->set_off.p;
    A.rows = e->set_rows.p;
    A.qrows = e->qrows.p;
    A.W = e->W.p;
    A.pat_bad = e->pat_bad.p;
    A.sets_per_pass = spp;
    A.mean = e->mean.p;
    A.has_nan = e->has_nan.p;
    A.sinv = e->sinv.p;
    A.sing = e->sing.p;
    A.varx = e->varx.p;
    const bool need_aobs = e->cfg.disp_cov || e->Z > 0;
    A.aobs = need_aobs ? e->aobs.p : nullptr;
    A.afull = e->cfg.disp_cov ? e->afull.p : nullptr;
    A.sfinv = e->cfg.disp_cov ? e->sfinv.p : nullptr;
    A.zA = e->zA.p;
    A.zD = e->zD.p;
    A.write_split = e->cfg.precision == OA_MIXED_BF16X3;
    A.center = e->center ? 1 : 0;
    A.Xhi = e->Xhi.p;
    A.Xlo = e->Xlo.p;
    return A;
}

template <int R>
oa_status stats_gather(oa_engine* e, const float* X, int mbc) {
    // SNPs per group: as many as fit the register budget; two column buffers
    // (double-buffered TMA staging) when they fit in ~170 KB, else one
    const int nS = (e->n + 3) & ~3;
    const size_t limit = 227 * 1024 - 1024;
    auto pick = [&](auto lp_tag) -> oa_status {
        constexpr int LP = decltype(lp_tag)::value;
        int spb = stats_spb_max(R, LP);
        int nbuf = 2;
        while (spb > 1 && (size_t)nbuf * spb * R * nS * 4 > 170 * 1024) --spb;
        if ((size_t)nbuf * spb * R * nS * 4 > 170 * 1024) nbuf = 1;
        const size_t base = stats_smem_bytes(R, LP, e->n, spb, nbuf, 0);
        if (base + (size_t)spb * stats_na(R, LP) * 4 > limit) {
            set_err("n = %d is too large for one SNP column in shared memory", e->n);
            return OA_ERR_UNSUPPORTED;
        }
        int spp = (int)std::min<size_t>((size_t)std::max(e->nsets, 1),
                                        (limit - base) / ((size_t)spb * stats_na(R, LP) * 4));
        spp = std::max(spp, 1);
        const size_t smem = stats_smem_bytes(R, LP, e->n, spb, nbuf, spp);
        StatsArgs A = stats_args(e, X, mbc, LP, spb, spp);
        A.nbuf = nbuf;
        A.err = reinterpret_cast<int*>(e->counters.p + 3);
        const int groups = (mbc + spb - 1) / spb;
        const int grid = std::min(groups, e->sm_count);
        OA_CU(oa_launch_snp_stats(R, LP, A, grid, smem, e->st));
        ++e->launches;
        return OA_OK;
    };
    if (e->LP == 4) return pick(std::integral_constant<int, 4>{});
    if (e->LP == 8) return pick(std::integral_constant<int, 8>{});
    return pick(std::integral_constant<int, 16>{});
}

// Lean path: k_snp_lean (imputation, BF16 split, X'X over all rows and over
// each row set) -> pre-GEMM C2 = [Q | Q o m_1 | ...]'X -> k_schur.
// SNPs per CTA group of k_snp_lean: requested, else two CTAs per SM where a
// double-buffered group fits in half the shared memory (a power of two <= 8 / r)
// With two or more columns per SNP and at most LEAN_QX_L covariates, k_snp_lean also sums the
// all-rows covariate projection A = Q'X of every column (short FP32 partial sums, FP64 across
// warps) for k_schur: the pre-GEMM's A (FP32 sums over all n rows; BF16 hi/lo products in the mixed
// form) is the largest error of the Schur complements and of var_x when D - A'A cancels, which two
// correlated columns per SNP make likely (an interaction with a covariate).  Those kernels take
// groups of at most LEAN_QX_NC columns.
bool want_lean_qx(const oa_engine* e) { return e->ru >= 2 && e->l <= LEAN_QX_L && e->r <= LEAN_QX_NC; }

// Threads per k_snp_lean CTA, from the column length alone (so that every tuning sums in the same
// order and gives the same bits): 512 with one column per SNP where the column takes 64 KB or more
// of shared memory (n >= 16,384: at most three CTAs fit on an SM, and the plan then keeps one SNP
// per group), else 256 (more, smaller CTAs per SM with cheaper block barriers).
int lean_threads(const oa_engine* e) {
    const bool long_col = e->r == 1 && (size_t)e->n_pad * 4 >= (size_t)64 * 1024;
    if (e->lean_threads_req) return long_col ? e->lean_threads_req : 256;
    return long_col ? LEAN_MAX_THREADS : 256;
}

int lean_group(const oa_engine* e) {
    if (lean_threads(e) == LEAN_MAX_THREADS) return 1;   // the 512-thread kernel takes one SNP per group
    const int cap = want_lean_qx(e) ? LEAN_QX_NC / e->r : 8 / e->r;
    if (e->lean_spb > 0) {
        int s = 1;
        while (s * 2 <= e->lean_spb) s *= 2;
        return std::min(s, cap);
    }
    int s = 1;
    while (s * 2 <= cap && lean_smem_bytes(e->r, e->n_pad, s * 2, 2, 0, true, want_lean_qx(e)) <= 100 * 1024)
        s *= 2;
    return s;
}

// Launch plan of k_snp_lean for the current trait block and tuning: SNPs per
// group, column buffers, shared memory, and passes over the row sets whose
// work items fit in shared memory.  Host-only (runs before any capture).
oa_status lean_plan(oa_engine* e) {
    const int R = e->r;
    const size_t limit = 227 * 1024 - 1024;
    int spb = lean_group(e);
    // A set pass heavier than the column passes (more rows in the row sets than in a column) is
    // latency-bound: it runs faster with more CTAs per SM (one column buffer, no interleaved copy)
    // than with a prefetched second buffer.
    const long long set_rows = e->h_set_item_off.empty() ? 0 : (long long)e->h_set_item_off.back() * LEAN_ITEM_ROWS;
    const bool heavy_sets = set_rows > e->n;
    int nbuf = e->lean_nbuf ? e->lean_nbuf : (heavy_sets ? 1 : 2);
    const bool xi = e->lean_xi >= 0 ? e->lean_xi == 1 : !heavy_sets;
    const bool qx = want_lean_qx(e);
    while (spb > 1 && lean_smem_bytes(R, e->n_pad, spb, nbuf, 0, xi, qx) > 200 * 1024) spb /= 2;
    if (lean_smem_bytes(R, e->n_pad, spb, nbuf, 0, xi, qx) > 200 * 1024) nbuf = 1;
    const size_t base = lean_smem_bytes(R, e->n_pad, spb, nbuf, 0, xi, qx);
    const size_t per_item = (size_t)spb * R * R * 4;
    int max_items = 1;
    for (int s2 = 0; s2 < e->nsets; ++s2)
        max_items = std::max(max_items, e->h_set_item_off[s2 + 1] - e->h_set_item_off[s2]);
    if (base + per_item * max_items > limit) {
        set_err("n = %d is too large for the column-statistics kernel's shared memory", e->n);
        return OA_ERR_UNSUPPORTED;
    }
    const int total_items = std::max(1, e->h_set_item_off.empty() ? 1 : e->h_set_item_off.back());
    const int cap = (int)std::min<size_t>((size_t)total_items, (limit - base) / per_item);
    if (e->lp.spb == spb && e->lp.nbuf == nbuf && e->lp.items_cap == cap && e->lp.xi == xi) return OA_OK;
    std::vector<int> passes{0};
    for (int s0 = 0; s0 < e->nsets;) {
        int s1 = s0 + 1;
        while (s1 < e->nsets && e->h_set_item_off[s1 + 1] - e->h_set_item_off[s0] <= cap) ++s1;
        passes.push_back(s1);
        s0 = s1;
    }
    OA_CHECK(e->pass_off.ensure(passes.size()));
    H2DBatch h2d;
    h2d.add(e->pass_off.p, passes);
    OA_CHECK(flush_h2d(e, h2d));
    OA_CU(cudaStreamSynchronize(e->st));
    e->lp.spb = spb;
    e->lp.nbuf = nbuf;
    e->lp.items_cap = cap;
    e->lp.npass = e->nsets > 0 ? (int)passes.size() - 1 : 0;
    e->lp.xi = xi;
    e->lp.smem = lean_smem_bytes(R, e->n_pad, spb, nbuf, cap, xi, qx);
    return OA_OK;
}

// The tensor-core GEMMs of this chunk read its FP32 columns and split them
// into BF16 hi / lo in shared memory, so the statistics kernel writes no
// split copy to HBM: mixed form, pre-GEMM statistics path with at most 128
// pre-GEMM columns, contiguous 16-byte aligned columns of a multiple of 4
// floats, and a GEMM shape that has a fused form (OA_FUSED_SPLIT at engine
// creation: 1 takes the fused forms, 0 keeps the split copy).
bool fused_chunk(const oa_engine* e, const float* X, size_t ldx, const int* xrows) {
    return e->fuse_split && e->cfg.precision == OA_MIXED_BF16X3 && e->use_pre && e->c2 <= 128 && !xrows &&
           ldx == (size_t)e->n && e->n % 4 == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0 &&
           oa_gemm_tc_fusable(e->variant, e->t);
}

template <int R>
oa_status stats_pre(oa_engine* e, const float* X, size_t ldx, const int* xrows, int mbc, bool fused) {
    const int spb = e->lp.spb;
    const size_t smem = e->lp.smem;
    LeanArgs A{};
    A.X = X;
    A.ldx = ldx;
    A.xrows = xrows;
    A.n = e->n;
    A.n_pad = e->n_pad;
    A.mb = mbc;
    A.nbuf = e->lp.nbuf;
    A.nsets = e->nsets;
    A.rows = e->set_rows.p;
    A.item_start = e->item_start.p;
    A.set_item_off = e->set_item_off.p;
    A.pass_off = e->pass_off.p;
    A.npass = e->lp.npass;
    A.items_cap = e->lp.items_cap;
    A.mean = e->mean.p;
    A.has_nan = e->has_nan.p;
    A.D = e->D.p;
    A.Dset = e->Dset.p;
    const bool mixed = e->cfg.precision == OA_MIXED_BF16X3;
    A.write_split = mixed && !fused ? 1 : 0;
    A.use_xi = e->lp.xi ? 1 : 0;
    A.center = e->center ? 1 : 0;
    A.Xhi = e->Xhi.p;
    A.Xlo = e->Xlo.p;
    A.err = reinterpret_cast<int*>(e->counters.p + 3);
    const bool qx = want_lean_qx(e) && oa_lean_has_qx(R, spb);
    if (qx) {
        OA_CHECK(e->Afull_lean.ensure((size_t)e->chunk * R * LEAN_QX_L));
        A.Qb = reinterpret_cast<const float4*>(e->Qb.p);
        A.l = e->l;
        A.qsum = e->qsum.p;
        A.Afull = e->Afull_lean.p;
    }
    const int groups = (mbc + spb - 1) / spb;
    const int threads = lean_threads(e);
    const int per_sm = std::max(1, oa_lean_ctas_per_sm(R, spb, smem, qx, threads));
    const int grid = std::min(groups, e->sm_count * per_sm);
    OA_CU(oa_launch_snp_lean(R, spb, A, grid, threads, smem, e->st));
    ++e->launches;
    const int ldc = e->chunk * R;
    if (fused)
        OA_CU(oa_launch_pre_tcf(X, ldx, e->n, mbc * R, e->mean.p, e->has_nan.p, e->center ? 1 : 0, e->B2hi.p,
                                e->B2lo.p, e->c2,
                                e->n_pad, e->C2T.p, ldc, reinterpret_cast<int*>(e->counters.p + 3), e->st));
    else if (mixed)
        OA_CU(oa_launch_pre_tc(e->Xhi.p, e->Xlo.p, mbc * R, e->B2hi.p, e->B2lo.p, e->c2, e->n_pad, e->C2T.p, ldc,
                               reinterpret_cast<int*>(e->counters.p + 3), e->st));
    else
        OA_CU(oa_launch_pre_simt(X, (size_t)e->n, mbc * R, e->B2.p, (size_t)e->n_pad, e->c2, e->n, e->mean.p,
                                 e->has_nan.p, e->center ? 1 : 0, e->C2T.p, ldc, e->C2part.p, e->st));
    ++e->launches;
    SchurArgs S{};
    S.l = e->l;
    S.mb = mbc;
    S.G = e->G;
    S.Z = e->Z;
    S.ldc = ldc;
    S.C2 = e->C2T.p;
    S.D = e->D.p;
    S.Dset = e->Dset.p;
    S.W = e->W.p;
    S.pat_bad = e->pat_bad.p;
    S.sinv = e->sinv.p;
    S.sing = e->sing.p;
    S.varx = e->varx.p;
    const bool need_aobs = e->cfg.disp_cov || e->Z > 0;
    S.aobs = need_aobs ? e->aobs.p : nullptr;
    S.afull = e->cfg.disp_cov ? e->afull.p : nullptr;
    S.sfinv = e->cfg.disp_cov ? e->sfinv.p : nullptr;
    S.zA = e->zA.p;
    S.zD = e->zD.p;
    S.rr = e->ru;
    S.qdel = quirk_on(e) ? e->qdel.p : nullptr;
    S.qK = quirk_on(e) ? e->qK.p : nullptr;
    S.Afull_lean = qx ? e->Afull_lean.p : nullptr;
    OA_CU(oa_launch_schur(R, S, e->st));
    ++e->launches;
    return OA_OK;
}

template <int R>
oa_status stats_dispatch(oa_engine* e, const float* X, size_t ldx, const int* xrows, int mbc, bool fused) {
    if (e->use_pre) return stats_pre<R>(e, X, ldx, xrows, mbc, fused);
    if constexpr (R > 4) {
        set_err("internal: the gather-path statistics kernel takes at most 4 columns per SNP");
        return OA_ERR_STATE;
    }
    if (xrows || ldx != (size_t)e->n) {
        set_err("internal: the gather-path statistics kernel reads gathered chunks only");
        return OA_ERR_STATE;
    }
    return stats_gather<R>(e, X, mbc);
}

EpiArgs epi_args(oa_engine* e, int mbc, int snp_base) {
    EpiArgs E{};
    E.n = e->n;
    E.l = e->l;
    E.r = e->r;
    E.p = e->p;
    E.mb = mbc;
    E.G = e->G;
    E.pat = e->pat.p;
    E.zset = e->zset.p;
    E.tperm = e->tperm.p;
    E.rss0 = e->rss0.p;
    E.a_r2 = e->a_r2.p;
    E.inv_ncorr = e->inv_ncorr.p;
    E.vf = e->vf.p;
    E.b0 = e->b0.p;
    E.sinv = e->sinv.p;
    E.varx = e->varx.p;
    E.sing = e->sing.p;
    E.aobs = e->aobs.p;
    E.zA = e->zA.p;
    E.zD = e->zD.p;
    E.zQ = e->zQ.p;
    E.W = e->W.p;
    E.qdel = quirk_on(e) ? e->qdel.p : nullptr;
    E.qK = quirk_on(e) ? e->qK.p : nullptr;
    E.min_r2 = e->cfg.min_r2_store;
    E.min_t = e->cfg.min_t_store;
    E.store_all = e->cfg.store_all;
    E.rec = e->rec.p;
    E.rec_count = e->counters.p;
    E.rec_valid = e->counters.p + 4;
    E.cap = e->cap;
    E.n_singular = e->counters.p + 1;
    E.t = e->t;
    E.snp_base = snp_base;
    E.dense_ld = e->dense_ld;
    if (e->dense_on || e->cfg.disp_cov) {
        E.d_beta = e->d_beta.p;
        E.d_se = e->d_se.p;
        E.d_t = e->d_t.p;
        E.d_r2 = e->d_r2.p;
        E.d_sig = e->d_sig.p;
        E.d_flags = e->d_flags.p;
    }
    return E;
}

CovArgs cov_args(oa_engine* e, int mbc) {
    CovArgs C{};
    C.n = e->n;
    C.l = e->l;
    C.r = e->r;
    C.p = e->p;
    C.mb = mbc;
    C.tinv = e->tinv.p;
    C.pat = e->pat.p;
    C.b0 = e->b0.p;
    C.W = e->W.p;
    C.aobs = e->aobs.p;
    C.afull = e->afull.p;
    C.sfinv = e->sfinv.p;
    C.Rinv = e->Rinv.p;
    C.nobs = e->nobs.p;
    C.min_t = e->cfg.min_t_store;
    C.store_all = e->cfg.store_all;
    C.min_p_disp = (double)e->cfg.min_p_disp;
    return C;
}

template <int R>
oa_status gemm_dispatch(oa_engine* e, const float* X, int mbc, int snp_base, bool fused) {
    EpiArgs E = epi_args(e, mbc, snp_base);
    if (fused) {
        OA_CU(oa_launch_gemm_tcf(R, e->raster, X, (size_t)e->n, e->n, mbc * R, e->mean.p, e->has_nan.p,
                                 e->center ? 1 : 0,
                                 e->Yhi.p, e->Ylo.p, e->t, e->n_pad, E, reinterpret_cast<int*>(e->counters.p + 3),
                                 e->st));
        e->last_name = e->t > 128 ? "k_gemm_tc2f" : "k_gemm_tcf";
    } else if (e->cfg.precision == OA_PLAIN_FP32) {
        // X'y~ does not change when a column is shifted (y~ is orthogonal to the intercept on the
        // observed rows): the main GEMM reads the dosages as they are, imputing NaN only
        OA_CU(oa_launch_gemm_simt(R, X, (size_t)e->n, mbc * R, e->Yt.p, (size_t)e->n_pad, e->t, e->n, e->mean.p,
                                  e->has_nan.p, 0, E, e->st));
        e->last_name = "k_gemm_simt";
    } else {
        OA_CU(oa_launch_gemm_tc(R, e->variant, e->raster, e->Xhi.p, e->Xlo.p, mbc * R, e->Yhi.p, e->Ylo.p, e->t,
                                e->n_pad, E, reinterpret_cast<int*>(e->counters.p + 3), e->st));
        e->last_name = (e->t > 128 && e->variant >= 3) ? "k_gemm_tc2" : "k_gemm_tc";
    }
    ++e->launches;
    OA_CU(cudaGetLastError());
    return OA_OK;
}

oa_status ensure_chunk_buffers(oa_engine* e) {
    const size_t mb = (size_t)e->chunk, r = e->r, l = e->l;
    const size_t G = std::max(e->G, 1), Z = std::max(e->Z, 1);
    OA_CHECK(e->mean.ensure(mb * r));
    OA_CHECK(e->has_nan.ensure(1));
    OA_CHECK(e->varx.ensure(mb * r));
    OA_CHECK(e->sinv.ensure(G * mb * r * r));
    OA_CHECK(e->sing.ensure(G * mb));
    OA_CHECK(e->zA.ensure(Z * mb * l * r));
    OA_CHECK(e->zD.ensure(Z * mb * r * r));
    if (e->cfg.disp_cov || e->Z > 0) OA_CHECK(e->aobs.ensure(G * mb * l * r));
    if (quirk_on(e)) {
        OA_CHECK(e->qdel.ensure(G * mb * l * r));
        OA_CHECK(e->qK.ensure(G * mb * r * r));
    }
    if (e->cfg.disp_cov) {
        OA_CHECK(e->afull.ensure(mb * l * r));
        OA_CHECK(e->sfinv.ensure(mb * r * r));
    }
    if (e->cfg.precision == OA_MIXED_BF16X3) {
        OA_CHECK(e->Xhi.ensure(mb * r * e->n_pad));
        OA_CHECK(e->Xlo.ensure(mb * r * e->n_pad));
    }
    if (e->use_pre) {
        OA_CHECK(e->D.ensure(mb * r * r));
        OA_CHECK(e->Dset.ensure((size_t)std::max(e->nsets, 1) * mb * r * r));
        OA_CHECK(e->C2T.ensure((size_t)e->c2 * mb * r));
        if (e->cfg.precision == OA_PLAIN_FP32) OA_CHECK(e->C2part.ensure((size_t)e->c2 * mb * r));
    }
    return OA_OK;
}

oa_status ensure_cap(oa_engine* e, long long want) {
    // contents are not kept: callers grow before a block starts or before it runs again
    if (want <= e->cap) return OA_OK;
    want += want / 4;   // headroom, so that slightly larger requests reuse the buffer
    e->rec.release();
    e->cov.release();
    e->cap = 0;
    OA_CHECK(e->rec.ensure((size_t)want * rec_slots(e->r)));   // records of RecOf<r>, in Rec units
    if (e->cfg.disp_cov) OA_CHECK(e->cov.ensure((size_t)want * e->l * 3));
    e->cap = want;
    return OA_OK;
}

// Stored-row count at the start of a chunk's GEMM (the covariate-term
// kernel of that chunk reads its record range from here and the counter).
static __global__ void k_mark(const unsigned long long* __restrict__ counters, unsigned long long* __restrict__ mark) {
    *mark = counters[0];
}

// Every chunk of a SNP block enqueued on the engine's stream with no host
// synchronisation: host blocks stream through two staging buffers on the
// copy stream, device blocks are read in place (or gathered for a row
// subset).  `capture`: the events become graph nodes.
template <int R>
oa_status enqueue_block(oa_engine* e, const float* xr, int mb, bool host_input, bool capture) {
    const int nch = (mb + e->chunk - 1) / e->chunk;
    while ((int)e->cev0.size() < nch) {
        cudaEvent_t ev[4];
        for (auto& x : ev) OA_CU(cudaEventCreate(&x));
        e->cev0.push_back(ev[0]);
        e->cev1.push_back(ev[1]);
        e->sev0.push_back(ev[2]);
        e->sev1.push_back(ev[3]);
    }
    auto rec = [&](cudaEvent_t ev) -> cudaError_t {
        return capture ? cudaEventRecordWithFlags(ev, e->st, cudaEventRecordExternal) : cudaEventRecord(ev, e->st);
    };
    const int IC = input_cols(e);
    const size_t colbytes = sizeof(float) * (size_t)e->n * IC;
    auto issue_copy = [&](int c) -> oa_status {   // host chunk c -> staging buffer c & 1 (copy stream)
        const int b = c & 1;
        const int c0 = c * e->chunk, mbc = std::min(e->chunk, mb - c0);
        OA_CU(cudaStreamWaitEvent(e->cp, e->ev_used[b], 0));
        OA_CU(cudaMemcpyAsync(e->Xstage[b].p, xr + (size_t)c0 * IC * e->n, colbytes * mbc, cudaMemcpyHostToDevice,
                              e->cp));
        OA_CU(cudaEventRecord(e->ev_copied[b], e->cp));
        return OA_OK;
    };
    if (host_input) OA_CHECK(issue_copy(0));
    const bool cov = e->cfg.disp_cov != 0;   // e->marks holds nch entries (allocated before any capture)
    for (int c = 0; c < nch; ++c) {
        const int c0 = c * e->chunk, mbc = std::min(e->chunk, mb - c0);
        const float* X = nullptr;
        size_t ldx = (size_t)e->n;
        const int* xrows = nullptr;
        if (host_input) {
            if (c + 1 < nch) OA_CHECK(issue_copy(c + 1));
            OA_CU(cudaStreamWaitEvent(e->st, e->ev_copied[c & 1], 0));
            X = e->Xstage[c & 1].p;
        } else if (lean_gathers(e)) {   // the column-statistics kernel reads the subset rows itself
            X = xr + (size_t)c0 * R * e->x_ld;
            ldx = e->x_ld;
            xrows = e->xrows.p;
        } else if (column_pass(e)) {
            X = xr + (size_t)c0 * IC * e->n;
        } else {
            OA_CHECK(chunk_input<R>(e, xr, c0, mbc, &X));
        }
        if (column_pass(e)) {   // file columns -> model columns (+ zero padding)
            ModelW W;
            const bool model = e->in_cols > 0;   // else the caller's ru columns as they are
            for (int c = 0; c < OA_MODEL_MAX_COLS; ++c) W.w[c] = model ? e->model_w[c] : 1.f;
            k_column_model<<<dim3((unsigned)((e->n + 255) / 256), (unsigned)mbc), 256, 0, e->st>>>(
                X, e->n, IC, W, model ? e->model_combine : 0, e->inter.p, e->n_inter, e->inter_keep, R,
                e->Xmodel.p);
            ++e->launches;
            OA_CU(cudaGetLastError());
            X = e->Xmodel.p;
        }
        OA_TRACE("chunk: statistics and GEMM launches");
        OA_CU(cudaMemsetAsync(e->has_nan.p, 0, sizeof(int), e->st));
        OA_CU(rec(e->sev0[c]));
        const bool fused = fused_chunk(e, X, ldx, xrows);
        e->fused_last = fused;
        OA_CHECK(stats_dispatch<R>(e, X, ldx, xrows, mbc, fused));
        OA_CU(rec(e->sev1[c]));
        if (cov) {
            k_mark<<<1, 1, 0, e->st>>>(e->counters.p, e->marks.p + c);
            ++e->launches;
        }
        OA_CU(rec(e->cev0[c]));
        OA_CHECK(gemm_dispatch<R>(e, X, mbc, c0, fused));
        OA_CU(rec(e->cev1[c]));
        if (host_input) OA_CU(cudaEventRecord(e->ev_used[c & 1], e->st));
        if (cov) {
            CovArgs C = cov_args(e, mbc);
            k_cov_terms<R><<<4 * e->sm_count, 256, 0, e->st>>>(reinterpret_cast<const RecOf<R>*>(e->rec.p),
                                                             e->marks.p + c, e->counters.p, e->cap, c0, C, e->cov.p);
            k_cov_count<R><<<4 * e->sm_count, 256, 0, e->st>>>(e->d_beta.p, e->d_t.p, e->d_r2.p, e->d_sig.p,
                                                             e->dense_ld, c0, mbc, e->t, e->cfg.min_r2_store, C,
                                                             e->counters.p + 2);
            e->launches += 2;
            OA_CU(cudaGetLastError());
        }
    }
    return OA_OK;
}

void drop_graph(oa_engine* e) {
    if (e->gexec) cudaGraphExecDestroy(e->gexec);
    if (e->graph) cudaGraphDestroy(e->graph);
    e->gexec = nullptr;
    e->graph = nullptr;
    e->gkey = oa_engine::GraphKey{};
}

// One SNP block, host or device, with one host synchronisation at its end.
// A device block seen twice with the same inputs is captured as one CUDA
// graph and replayed afterwards (the first sight runs uncaptured, which also
// sets the kernels' attributes).  If the stored rows outgrow their buffer,
// the buffer grows and the block runs again.
template <int R>
oa_status run_block(oa_engine* e, const float* xr, int mb, bool host_input) {
    const int nch = (mb + e->chunk - 1) / e->chunk;
    for (int attempt = 0; attempt < 3; ++attempt) {
        OA_CU(cudaMemsetAsync(e->counters.p, 0, 8 * sizeof(unsigned long long), e->st));
        OA_CU(cudaEventRecord(e->k0, e->st));
        bool launched = false;
        if (!host_input && e->use_graphs) {
            oa_engine::GraphKey key;
            key.xr = xr;
            key.mb = mb;
            key.t = e->t;
            key.dense = e->dense_on ? 1 : 0;
            key.gen = e->trait_gen;
            key.cap = e->cap;
            key.rec = e->rec.p;
            key.tune = e->tune_gen;
            if (!(e->gexec && e->gkey == key)) {
                drop_graph(e);
                if (e->warm_key == key) {
                    const long long l0 = e->launches;
                    OA_CU(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
                    const oa_status s = enqueue_block<R>(e, xr, mb, false, true);
                    e->graph_launches = e->launches - l0;   // kernels in the graph (they run at each launch)
                    e->launches = l0;
                    cudaGraph_t g = nullptr;
                    const cudaError_t ce = cudaStreamEndCapture(e->st, &g);
                    if (s != OA_OK) {
                        if (g) cudaGraphDestroy(g);
                        return s;
                    }
                    OA_CU(ce);
                    e->graph = g;
                    OA_CU(cudaGraphInstantiate(&e->gexec, g, 0));
                    e->gkey = key;
                } else {
                    e->warm_key = key;
                }
            }
            if (e->gexec && e->gkey == key) {
                OA_CU(cudaGraphLaunch(e->gexec, e->st));
                e->launches += e->graph_launches;
                launched = true;
            }
        }
        if (!launched) OA_CHECK(enqueue_block<R>(e, xr, mb, host_input, false));
        OA_CU(cudaEventRecord(e->k1, e->st));
        const unsigned long long* cnt = e->h_cnt;
        OA_CU(cudaMemcpyAsync(e->h_cnt, e->counters.p, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, e->st));
        OA_CU(cudaStreamSynchronize(e->st));
        if (cnt[3]) {
            set_err("a device pipeline wait timed out (the kernel stopped cleanly)");
            return OA_ERR_CUDA;
        }
        if ((long long)cnt[0] > e->cap) {   // more stored rows than room: grow, run the block again
            OA_CHECK(ensure_cap(e, (long long)(cnt[0] * 1.25) + 1024));
            drop_graph(e);
            continue;
        }
        float total = 0.f, stotal = 0.f;
        for (int c = 0; c < nch; ++c) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, e->cev0[c], e->cev1[c]) == cudaSuccess) total += ms;
            if (cudaEventElapsedTime(&ms, e->sev0[c], e->sev1[c]) == cudaSuccess) stotal += ms;
        }
        cudaGetLastError();
        e->last_ms = total;
        e->stats_ms = stotal;
        float bms = 0.f;
        e->block_ms = cudaEventElapsedTime(&bms, e->k0, e->k1) == cudaSuccess ? bms : 0.f;
        cudaGetLastError();
        e->last_name = e->cfg.precision == OA_PLAIN_FP32                ? "k_gemm_simt"
                       : e->fused_last                                  ? (e->t > 128 ? "k_gemm_tc2f" : "k_gemm_tcf")
                       : (e->t > 128 && e->variant >= 3) ? "k_gemm_tc2"
                                                          : "k_gemm_tc";
        return OA_OK;
    }
    set_err("stored-row buffer could not be grown");
    return OA_ERR_NOMEM;
}

// Stored-row slots for a block of mb SNPs x t traits in chunks of `chunk`
// SNPs: the expected stored rows (the two-sided normal tail beyond the |t|
// threshold, with headroom; every test with store_all) + the unused tails
// of the epilogue warps' reserved blocks (at most one block per warp and
// launch).  A block that still overflows grows the buffer and runs again.
long long slots_needed(const oa_engine* e, long long mb, long long t, long long chunk) {
    const long long tests = mb * t;
    const double tail = std::erfc((double)e->cfg.min_t_store / std::sqrt(2.0));
    const double share = std::min(1.0, 1.5 * tail + 1e-3);
    const long long nch = (mb + chunk - 1) / chunk;
    const long long slack = nch * (long long)e->sm_count * EPI_WARPS_TC * EMIT_BLOCK;
    const long long rows = e->cfg.store_all ? tests : (long long)(tests * share);
    return std::max<long long>(1 << 16, rows + slack);
}

template <int R>
oa_status run_snps_impl(oa_engine* e, const float* xr, int32_t mb, bool host_input, bool results_on_host,
                        oa_rows* out) {
    OA_TRACE("oa_run_snps");
    if (e->t <= 0) {
        set_err("oa_run_snps before oa_set_traits");
        return OA_ERR_STATE;
    }
    if (mb <= 0 || mb > e->cfg.max_snps) {
        set_err("SNP block of %d SNPs (engine limit %d)", mb, e->cfg.max_snps);
        return OA_ERR_ARG;
    }
    if (e->in_cols > 0 && e->model_combine && (e->n_inter > 0 ? e->n_inter + e->inter_keep : 1) != e->ru) {
        set_err("a combined column model gives r = %d columns per SNP%s, the engine has r = %d",
                e->n_inter > 0 ? e->n_inter + e->inter_keep : 1, e->n_inter > 0 ? " with its interactions" : "",
                e->ru);
        return OA_ERR_STATE;
    }
    OA_CHECK(prepare_tuning(e));
    OA_CHECK(ensure_chunk_buffers(e));
    const long long tests = (long long)mb * e->t;
    OA_CHECK(ensure_cap(e, slots_needed(e, mb, e->t, e->chunk)));
    OA_CU(cudaMemsetAsync(e->counters.p, 0, 8 * sizeof(unsigned long long), e->st));
    if (e->dense_on || e->cfg.disp_cov) {
        const size_t nd = (size_t)e->t * mb;
        OA_CHECK(e->d_beta.ensure(nd * e->r));
        OA_CHECK(e->d_se.ensure(nd * e->r));
        OA_CHECK(e->d_t.ensure(nd * e->r));
        OA_CHECK(e->d_r2.ensure(nd));
        OA_CHECK(e->d_sig.ensure(nd));
        OA_CHECK(e->d_flags.ensure(nd));
        e->dense_ld = mb;
    }
    e->last_ms = 0.f;
    e->stats_ms = 0.f;
    e->last_mb = mb;
    if (e->subset) {
        if (host_input) {
            set_err("a row subset applies to device SNP blocks only (oa_run_snps_device)");
            return OA_ERR_STATE;
        }
        if (!lean_gathers(e)) OA_CHECK(e->Xstage[0].ensure((size_t)e->chunk * e->r * e->n));
    }
    if (column_pass(e)) OA_CHECK(e->Xmodel.ensure((size_t)e->chunk * e->r * e->n));
    if (host_input) {
        if (!e->cp) OA_CU(cudaStreamCreateWithFlags(&e->cp, cudaStreamNonBlocking));
        for (int b = 0; b < 2; ++b) {
            OA_CHECK(e->Xstage[b].ensure((size_t)e->chunk * input_cols(e) * e->n));
            OA_CU(cudaEventRecord(e->ev_used[b], e->st));   // the copy stream starts after the allocation
        }
    }
    if (e->cfg.disp_cov) OA_CHECK(e->marks.ensure((mb + e->chunk - 1) / e->chunk));
    {
        OA_TRACE("SNP block on the device");
        OA_CHECK(run_block<R>(e, xr, mb, host_input));
    }
    OA_TRACE("stored rows: sort, copy back, convert");
    unsigned long long cnt[5];
    OA_CU(cudaMemcpyAsync(e->h_cnt, e->counters.p, sizeof cnt, cudaMemcpyDeviceToHost, e->st));
    OA_CU(cudaStreamSynchronize(e->st));
    std::memcpy(cnt, e->h_cnt, sizeof cnt);
    std::memset(out, 0, sizeof *out);
    out->count = (int64_t)cnt[4];
    out->tests = tests;
    out->singular = (int64_t)cnt[1];
    out->sig_cov_unrowed = (int64_t)cnt[2];
    if (!results_on_host) return OA_OK;

    // sort the stored rows into reference order (trait, then SNP); unused
    // slots of the warps' reserved blocks sort last and are dropped
    const long long NS = (long long)cnt[0];   // slots handed out
    const long long N = (long long)cnt[4];    // rows written
    const int l = e->l, p = e->p;
    // the packed fields of N rows (16 + 12 R bytes each) fit in N Rec-sized slots per rec_slots(R)
    OA_CHECK(ensure_pinned(e->h_rec, e->h_rec_cap, (size_t)N * rec_slots(R), e->retired_pinned));
    if (e->cfg.disp_cov) OA_CHECK(ensure_pinned(e->h_cov, e->h_cov_cap, (size_t)N * l * 3, e->retired_pinned));
    if (N > 0) {
        OA_CHECK(e->keys.ensure(NS));
        OA_CHECK(e->keys2.ensure(NS));
        OA_CHECK(e->perm.ensure(NS));
        OA_CHECK(e->perm2.ensure(NS));
        OA_CHECK(e->rec2.ensure((size_t)N * rec_slots(R)));
        // key bits: enough for t * mb with the all-ones invalid key above every valid one
        int bits = 1;
        while (bits < 64 && (1ull << bits) <= (unsigned long long)e->t * (unsigned long long)mb) ++bits;
        k_rec_keys<<<(unsigned)((NS + 255) / 256), 256, 0, e->st>>>(reinterpret_cast<const RecOf<R>*>(e->rec.p), NS,
                                                                     mb, bits, e->keys.p, e->perm.p);
        ++e->launches;
        size_t tmp = 0;
        OA_CU(cub::DeviceRadixSort::SortPairs(nullptr, tmp, e->keys.p, e->keys2.p, e->perm.p, e->perm2.p, (int)NS, 0,
                                              bits, e->st));
        OA_CHECK(e->cub_tmp.ensure(tmp));
        OA_CU(cub::DeviceRadixSort::SortPairs(e->cub_tmp.p, tmp, e->keys.p, e->keys2.p, e->perm.p, e->perm2.p, (int)NS,
                                              0, bits, e->st));
        if (e->cfg.disp_cov) OA_CHECK(e->cov2.ensure((size_t)N * l * 3));
        const RowsSoA dsoa = rows_soa(e->rec2.p, N, R);   // the record buffer holds the packed fields
        k_rec_gather<R><<<(unsigned)((N + 255) / 256), 256, 0, e->st>>>(reinterpret_cast<const RecOf<R>*>(e->rec.p),
                                                                        e->perm2.p, N, dsoa,
                                                                        e->cfg.disp_cov ? e->cov.p : nullptr,
                                                                        e->cfg.disp_cov ? e->cov2.p : nullptr, l);
        ++e->launches;
        if (e->cfg.disp_cov)
            OA_CU(cudaMemcpyAsync(e->h_cov, e->cov2.p, sizeof(float) * N * l * 3, cudaMemcpyDeviceToHost, e->st));
        OA_CU(cudaGetLastError());
        // the rows come back in pieces, each converted on the host while the next is in flight
        const RowsSoA hsoa = rows_soa(e->h_rec, N, R);
        for (int k = 0; k < RESULT_PIECES; ++k) {
            const long long q0 = N * k / RESULT_PIECES, q1 = N * (k + 1) / RESULT_PIECES, nq = q1 - q0;
            if (nq > 0) {
                auto d2h = [&](void* dst, const void* src, size_t bytes) {
                    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, e->st);
                };
                OA_CU(d2h(hsoa.trait + q0, dsoa.trait + q0, 4 * nq));
                OA_CU(d2h(hsoa.snp + q0, dsoa.snp + q0, 4 * nq));
                OA_CU(d2h(hsoa.r2 + q0, dsoa.r2 + q0, 4 * nq));
                OA_CU(d2h(hsoa.mask + q0, dsoa.mask + q0, 4 * nq));
                OA_CU(d2h(hsoa.b + q0 * R, dsoa.b + q0 * R, 4 * R * nq));
                OA_CU(d2h(hsoa.se + q0 * R, dsoa.se + q0 * R, 4 * R * nq));
                OA_CU(d2h(hsoa.t + q0 * R, dsoa.t + q0 * R, 4 * R * nq));
            }
            OA_CU(cudaEventRecord(e->ev_piece[k], e->st));
        }
    }
    e->o_trait.resize(N);
    e->o_snp.resize(N);
    e->o_nused.resize(N);
    e->o_r2.resize(N);
    e->o_mask.resize(N);
    e->o_b.resize((size_t)N * p);
    e->o_se.resize((size_t)N * p);
    e->o_t.resize((size_t)N * p);
    const float minT = e->cfg.min_t_store;
    const bool disp_cov = e->cfg.disp_cov != 0, store_all = e->cfg.store_all != 0;
    const int ru = e->ru;   // the caller's columns: the padding columns' terms are not reported
    const RowsSoA hs = rows_soa(e->h_rec, N, R);
    auto convert = [&](long long q0, long long q1) {
        for (long long q = q0; q < q1; ++q) {
            const int32_t tr = hs.trait[q];
            e->o_trait[q] = tr;
            e->o_snp[q] = hs.snp[q];
            e->o_nused[q] = e->h_nobs[tr];
            e->o_r2[q] = hs.r2[q];
            float* ob = &e->o_b[(size_t)q * p];
            float* os = &e->o_se[(size_t)q * p];
            float* ot = &e->o_t[(size_t)q * p];
            for (int h = 0; h < l; ++h) ob[h] = os[h] = ot[h] = 0.f;
            uint32_t m = 0;
            const uint32_t rm = hs.mask[q];
            for (int a = 0; a < ru; ++a) {
                ob[l + a] = hs.b[(size_t)q * R + a];
                os[l + a] = hs.se[(size_t)q * R + a];
                ot[l + a] = hs.t[(size_t)q * R + a];
                if (rm & (1u << a)) m |= 1u << (l + a);
            }
            if (disp_cov) {
                const float* cv = e->h_cov + (size_t)q * l * 3;
                for (int h = 1; h < l; ++h) {
                    ob[h] = cv[h * 3];
                    os[h] = cv[h * 3 + 1];
                    ot[h] = cv[h * 3 + 2];
                    if (cv[h * 3 + 2] > minT || store_all) m |= 1u << h;
                }
            }
            e->o_mask[q] = m;
        }
    };
    const int nthr = N > (1 << 18) ? (int)std::min<unsigned>(32u, std::max(1u, std::thread::hardware_concurrency())) : 1;
    std::atomic<int> piece_err{0};
    auto convert_pieces = [&](int k0, int nk) {   // thread k0 of nk: its share of every piece, in piece order
        for (int k = 0; k < RESULT_PIECES; ++k) {
            if (N > 0 && cudaEventSynchronize(e->ev_piece[k]) != cudaSuccess) {
                piece_err = 1;
                return;
            }
            const long long q0 = N * k / RESULT_PIECES, q1 = N * (k + 1) / RESULT_PIECES;
            convert(q0 + (q1 - q0) * k0 / nk, q0 + (q1 - q0) * (k0 + 1) / nk);
        }
    };
    if (nthr <= 1) {
        convert_pieces(0, 1);
    } else {
        std::vector<std::thread> th;
        for (int k = 0; k < nthr; ++k) th.emplace_back(convert_pieces, k, nthr);
        for (auto& x : th) x.join();
    }
    if (piece_err) {
        cudaGetLastError();
        set_err("waiting for the stored rows failed");
        return OA_ERR_CUDA;
    }
    out->trait = e->o_trait.data();
    out->snp = e->o_snp.data();
    out->r2 = e->o_r2.data();
    out->n_used = e->o_nused.data();
    out->coef_mask = e->o_mask.data();
    out->coef_b = e->o_b.data();
    out->coef_se = e->o_se.data();
    out->coef_t = e->o_t.data();
    return OA_OK;
}

oa_status run_snps_any(oa_engine* e, const float* xr, int32_t mb, bool host_input, bool results_on_host,
                       oa_rows* out) {
    clear_stale_error("oa_run_snps");
    if (!e || !xr || !out) {
        set_err("null argument");
        return OA_ERR_ARG;
    }
    OA_CU(cudaSetDevice(e->cfg.device));
    AllocOn alloc_on(e->st);
    switch (e->r) {
        case 1: return run_snps_impl<1>(e, xr, mb, host_input, results_on_host, out);
        case 2: return run_snps_impl<2>(e, xr, mb, host_input, results_on_host, out);
        case 4: return run_snps_impl<4>(e, xr, mb, host_input, results_on_host, out);
        case 8: return run_snps_impl<8>(e, xr, mb, host_input, results_on_host, out);
        default:
            set_err("internal: %d kernel columns per SNP", e->r);
            return OA_ERR_STATE;
    }
}

// Autotuner: coordinate descent over the tuning fields, each candidate
// timed by the device time of its per-block kernels (statistics stage +
// main GEMM, CUDA events per chunk) on the caller's sample block.
oa_status autotune_impl(oa_engine* e, const float* xr, int mb, oa_tuning* best_out) {
    OA_TRACE("oa_autotune");
    if (e->t <= 0) {
        set_err("oa_autotune before oa_set_traits");
        return OA_ERR_STATE;
    }
    const int r = e->r;
    const bool mixed = e->cfg.precision == OA_MIXED_BF16X3;
    const bool graphs = e->use_graphs;
    e->use_graphs = false;
    oa_rows rows;
    auto cost = [&](const oa_tuning& c, float* ms) -> oa_status {
        e->req = c;
        ++e->tune_gen;
        float sum = 0.f;
        for (int rep = 0; rep < 3; ++rep) {   // first run: allocations and kernel attributes
            const oa_status s = run_snps_any(e, xr, mb, false, false, &rows);
            if (s != OA_OK) return s;
            if (rep > 0) sum += e->block_ms;   // the whole block on the device
        }
        *ms = sum / 2.f;
        return OA_OK;
    };
    // a chunk size set before the call is kept (the caller's block size)
    const bool fixed_chunk = e->req.chunk_snps > 0;
    oa_tuning best{};
    best.chunk_snps = fixed_chunk ? std::min(mb, e->req.chunk_snps) : std::min(mb, wave_chunk(e, e->t));
    best.gemm_variant = 4;
    best.gemm_raster = 1;
    OA_CHECK(prepare_tuning(e));
    best.stats_path = e->use_pre ? 1 : 2;
    best.lean_spb = 0;
    float best_ms = 0.f;
    oa_status s0 = cost(best, &best_ms);
    if (s0 != OA_OK) {
        e->use_graphs = graphs;
        return s0;
    }
    auto try_field = [&](int32_t oa_tuning::*f, std::vector<int> vals) {
        for (int v : vals) {
            if (v == best.*f) continue;
            oa_tuning c = best;
            c.*f = v;
            float ms = 0.f;
            if (cost(c, &ms) != OA_OK) {   // an infeasible candidate (e.g. shared memory) is skipped
                g_err.clear();
                cudaGetLastError();
                continue;
            }
            if (ms < best_ms * 0.98f) {
                best_ms = ms;
                best = c;
            }
        }
    };
    try_field(&oa_tuning::stats_path, {1, 2});
    if (best.stats_path == 1) {
        best.lean_spb = lean_group(e);
        std::vector<int> spbs;
        for (int v = 1; v <= 8 / r; v *= 2) spbs.push_back(v);
        try_field(&oa_tuning::lean_spb, spbs);
    }
    if (mixed) {
        try_field(&oa_tuning::gemm_variant, {1, 2, 3, 4});
        try_field(&oa_tuning::gemm_raster, {1, 2});
    }
    if (!fixed_chunk) {
        std::vector<int> chunks;
        const int w = wave_chunk(e, e->t);
        for (int c : {w / 2, w, 2 * w})
            if (c > 0 && c <= mb) chunks.push_back(c);
        for (int c = 2048; c <= 32768; c *= 2)
            if (c / r <= mb) chunks.push_back(c / r);
        try_field(&oa_tuning::chunk_snps, chunks);
    }
    e->req = best;
    ++e->tune_gen;
    e->use_graphs = graphs;
    OA_CHECK(prepare_tuning(e));
    if (best_out) *best_out = best;
    return OA_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* oa_last_error(void) { return g_err.c_str(); }
void oa__set_error(const char* msg) { g_err = msg ? msg : ""; }
int32_t oa_abi_version(void) { return OA_ABI_VERSION; }

// OA_TIMING: entry points that take 20 ms or more report their host time on stderr (engine
// sizes beside it), e.g. to see where a serving request's engine set-up spends its time.
struct ApiClock {
    const char* what;
    const oa_engine* e;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    ApiClock(const char* w, const oa_engine* eng) : what(w), e(eng) {}
    ~ApiClock() {
        static const bool on = getenv("OA_TIMING") != nullptr;
        if (!on) return;
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (ms >= 20.0)
            fprintf(stderr, "[oa timing] %s %.1f ms (n %d, traits %d, max SNPs %d)\n", what, ms, e ? e->n : 0,
                    e ? e->cfg.max_traits : 0, e ? e->cfg.max_snps : 0);
    }
};

oa_status oa_engine_create(const oa_config* cfg, oa_engine** out) {
    ApiClock api_clock("oa_engine_create", nullptr);
    clear_stale_error(__func__);
    if (!cfg || !out) {
        set_err("null argument");
        return OA_ERR_ARG;
    }
    *out = nullptr;
    if (cfg->l < 1 || cfg->l > OA_MAX_L || cfg->r < 1 || cfg->r > OA_MAX_R || cfg->n <= cfg->l + cfg->r ||
        cfg->max_traits < 1 || cfg->max_snps < 1) {
        set_err("invalid engine configuration (n=%d l=%d r=%d)", cfg->n, cfg->l, cfg->r);
        return OA_ERR_ARG;
    }
    if (cfg->precision != OA_PLAIN_FP32 && cfg->precision != OA_MIXED_BF16X3) {
        set_err("unknown precision %d", cfg->precision);
        return OA_ERR_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_err("no CUDA device: the engine has no CPU path");
        return OA_ERR_CUDA;
    }
    if (cfg->device < 0 || cfg->device >= ndev) {
        set_err("device %d of %d", cfg->device, ndev);
        return OA_ERR_ARG;
    }
    OA_CU(cudaSetDevice(cfg->device));
    // compute capability and SM count of the device, queried once per device: cudaGetDeviceProperties
    // took up to 0.3 s while other engines kept the device busy (a serving request's engine set-up)
    int cc_major = 0, cc_minor = 0, sm_count = 0;
    {
        static std::mutex mu;
        static int have[64], c_major[64], c_minor[64], c_sms[64];
        std::lock_guard<std::mutex> g(mu);
        const int d = cfg->device & 63;
        if (!have[d]) {
            OA_CU(cudaDeviceGetAttribute(&c_major[d], cudaDevAttrComputeCapabilityMajor, cfg->device));
            OA_CU(cudaDeviceGetAttribute(&c_minor[d], cudaDevAttrComputeCapabilityMinor, cfg->device));
            OA_CU(cudaDeviceGetAttribute(&c_sms[d], cudaDevAttrMultiProcessorCount, cfg->device));
            have[d] = 1;
        }
        cc_major = c_major[d];
        cc_minor = c_minor[d];
        sm_count = c_sms[d];
    }
    if (cc_major < 10) {
        set_err("device %d (sm_%d%d) is not a Blackwell sm_100 part", cfg->device, cc_major, cc_minor);
        return OA_ERR_UNSUPPORTED;
    }
    {   // bound of the device pipeline and staging waits, per device: 2 s, or OA_WAIT_LIMIT_NS (the
        // timeout tests shorten it so that the waits run out and the error path is exercised)
        static std::mutex mu;
        static unsigned long long cur[64];
        const char* w = getenv("OA_WAIT_LIMIT_NS");
        const unsigned long long ns = w ? std::max(1ull, strtoull(w, nullptr, 10)) : 2000000000ull;
        std::lock_guard<std::mutex> g(mu);
        unsigned long long& c = cur[cfg->device & 63];
        if (c != ns && !(c == 0 && ns == 2000000000ull)) {
            OA_CU(oa_set_wait_limit_tc(ns));
            OA_CU(oa_set_wait_limit_stats(ns));
        }
        c = ns;
    }
    oa_engine* e = new oa_engine();
    e->cfg = *cfg;
    e->sm_count = sm_count;
    e->n = cfg->n;
    e->l = cfg->l;
    e->ru = cfg->r;
    e->r = cfg->r <= 1 ? 1 : (cfg->r <= 2 ? 2 : (cfg->r <= 4 ? 4 : 8));
    e->p = cfg->l + cfg->r;
    e->LP = pad_l(cfg->l);
    e->n_pad = (cfg->n + 63) & ~63;
    // environment defaults of the tuning (oa_set_tuning overrides them)
    if (const char* v = getenv("OA_CHUNK_SNPS")) e->req.chunk_snps = std::max(1, atoi(v));
    if (const char* v = getenv("OA_STATS_PATH")) e->req.stats_path = std::string(v) == "pre" ? 1 : (std::string(v) == "gather" ? 2 : 0);
    if (const char* v = getenv("OA_TC_VARIANT")) e->req.gemm_variant = std::min(4, std::max(0, atoi(v)));
    if (const char* v = getenv("OA_LEAN_SPB")) e->req.lean_spb = std::max(0, atoi(v));
    if (const char* v = getenv("OA_LEAN_NBUF")) e->lean_nbuf = atoi(v) == 1 ? 1 : (atoi(v) == 2 ? 2 : 0);
    if (const char* v = getenv("OA_LEAN_XI")) e->lean_xi = atoi(v) == 0 ? 0 : (atoi(v) == 1 ? 1 : -1);
    if (const char* v = getenv("OA_LEAN_THREADS")) e->lean_threads_req = atoi(v) == 512 ? 512 : (atoi(v) == 256 ? 256 : 0);
    e->chunk = std::min(cfg->max_snps, e->req.chunk_snps > 0 ? e->req.chunk_snps : 16384 / e->r);
    if (const char* v = getenv("OA_FUSED_SPLIT")) e->fuse_split = v[0] != '0';
    if (const char* v = getenv("OA_TEST_HASH_BITS")) e->hash_bits = std::min(64, std::max(0, atoi(v)));
    const char* gr = getenv("OA_GRAPHS");
    e->use_graphs = !(gr && gr[0] == '0');
    // the copy stream of host SNP blocks is created on first use: a device-resident
    // scan (serving) holds one stream, so concurrent engines spread over the
    // device's hardware work queues
    if (cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) != cudaSuccess) {
        set_err("stream creation failed");
        delete e;
        return OA_ERR_CUDA;
    }
    for (int b = 0; b < 2; ++b) {
        cudaEventCreateWithFlags(&e->ev_copied[b], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&e->ev_used[b], cudaEventDisableTiming);
        cudaEventRecord(e->ev_used[b], e->st);
    }
    for (auto& ev : e->ev_piece) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    cudaEventCreate(&e->k0);
    cudaEventCreate(&e->k1);
    cudaEventCreate(&e->s0);
    cudaEventCreate(&e->s1);
    {   // freed engine memory stays in the device's pool for the next allocation (no device-wide sync)
        static std::mutex mu;
        static bool done[64];
        std::lock_guard<std::mutex> g(mu);
        if (!done[cfg->device & 63]) {
            cudaMemPool_t pool;
            uint64_t keep = ~0ull;
            if (cudaDeviceGetDefaultMemPool(&pool, cfg->device) == cudaSuccess)
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            cudaGetLastError();
            done[cfg->device & 63] = true;
        }
    }
    {
        AllocOn alloc_on(e->st);
        if (e->counters.ensure(8) != OA_OK) {
            delete e;
            return OA_ERR_NOMEM;
        }
    }
    live_engines(cfg->device, +1);
    // pinned counters and a first staging area (trait grouping of max_traits traits)
    e->h_cnt = static_cast<unsigned long long*>(pinned_pool().take(8 * sizeof(unsigned long long), &e->h_cnt_bytes));
    if (!e->h_cnt || stage_reserve(e, (size_t)48 * cfg->max_traits + 65536) != OA_OK) {
        cudaGetLastError();
        set_err("pinned host allocation failed");
        oa_engine_destroy(e);
        return OA_ERR_NOMEM;
    }
    *out = e;
    return OA_OK;
}

oa_status oa_engine_destroy(oa_engine* e) {
    ApiClock api_clock("oa_engine_destroy", nullptr);   // e is freed before the clock reports
    if (!e) return OA_OK;
    cudaSetDevice(e->cfg.device);
    if (e->cp) cudaStreamSynchronize(e->cp);
    {
        AllocOn alloc_on(e->st);
        for_each_buf(e, [](auto& b) { b.release(); });
    }
    cudaStreamSynchronize(e->st);
    if (live_engines(e->cfg.device, -1) == 0) {   // the last engine on the device returns the pool's memory
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, e->cfg.device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
        cudaGetLastError();
    }
    PinnedPool& pp = pinned_pool();
    pp.give(e->h_rec, e->h_rec_cap * sizeof(Rec));
    pp.give(e->h_cov, e->h_cov_cap * sizeof(float));
    for (const auto& q : e->retired_pinned) pp.give(q.first, q.second);
    pp.give(e->stage, e->stage_cap);
    pp.give(e->h_cnt, e->h_cnt_bytes);
    for (int b = 0; b < 2; ++b) {
        cudaEventDestroy(e->ev_copied[b]);
        cudaEventDestroy(e->ev_used[b]);
    }
    for (auto ev : e->ev_piece)
        if (ev) cudaEventDestroy(ev);
    cudaEventDestroy(e->k0);
    cudaEventDestroy(e->k1);
    cudaEventDestroy(e->s0);
    cudaEventDestroy(e->s1);
    drop_graph(e);
    for (auto* v : {&e->cev0, &e->cev1, &e->sev0, &e->sev1})
        for (auto ev : *v) cudaEventDestroy(ev);
    cudaStreamDestroy(e->st);
    if (e->cp) cudaStreamDestroy(e->cp);
    delete e;
    return OA_OK;
}

oa_status oa_set_covariates(oa_engine* e, const float* xl) {
    ApiClock api_clock("oa_set_covariates", e);
    clear_stale_error(__func__);
    OA_TRACE("oa_set_covariates: QR and rank check");
    if (!e || !xl) {
        set_err("null argument");
        return OA_ERR_ARG;
    }
    OA_CU(cudaSetDevice(e->cfg.device));
    AllocOn alloc_on(e->st);
    const int n = e->n, l = e->l;
    std::vector<double> A((size_t)n * l), Q, R;
    for (size_t q = 0; q < A.size(); ++q) {
        if (std::isnan(xl[q])) {
            set_err("covariate matrix contains NaN (the reader drops such individuals)");
            return OA_ERR_ARG;
        }
        A[q] = xl[q];
    }
    householder_qr(A, n, l, Q, R);
    // rank check: singular values of XL are those of R (src/Algorithm.cpp:508-522)
    const std::vector<double> sv = singular_values(R, l);
    for (double s : sv)
        if (!(s >= 1e-6)) {
            set_err("the covariate matrix contains linearly dependent columns (singular value %g)", s);
            return OA_ERR_COLLINEAR;
        }
    // R^-1 (upper triangular)
    std::vector<double> Ri((size_t)l * l, 0.0);
    for (int i = l - 1; i >= 0; --i) {
        Ri[(size_t)i * l + i] = 1.0 / R[(size_t)i * l + i];
        for (int j = i + 1; j < l; ++j) {
            double s = 0.0;
            for (int k = i + 1; k <= j; ++k) s += R[(size_t)i * l + k] * Ri[(size_t)k * l + j];
            Ri[(size_t)i * l + j] = -s / R[(size_t)i * l + i];
        }
    }
    std::vector<float> Qr((size_t)n * e->LP, 0.f);
    for (int k = 0; k < n; ++k)
        for (int q = 0; q < l; ++q) Qr[(size_t)k * e->LP + q] = (float)Q[(size_t)q * n + k];
    // the FP32 basis by blocks of four rows and its column sums (the lean kernel's projection)
    std::vector<float> Qb((size_t)e->n_pad * l, 0.f);
    std::vector<double> qsum(l, 0.0);
    for (int k = 0; k < n; ++k)
        for (int q = 0; q < l; ++q) {
            const float v = Qr[(size_t)k * e->LP + q];
            Qb[((size_t)(k / 4) * l + q) * 4 + k % 4] = v;
            qsum[q] += (double)v;
        }
    OA_CHECK(e->Q64.ensure((size_t)n * l));
    OA_CHECK(e->Qr.ensure(Qr.size()));
    OA_CHECK(e->Qb.ensure(Qb.size()));
    OA_CHECK(e->qsum.ensure(qsum.size()));
    OA_CHECK(e->Rinv.ensure((size_t)l * l));
    OA_CU(cudaMemcpyAsync(e->Q64.p, Q.data(), sizeof(double) * Q.size(), cudaMemcpyHostToDevice, e->st));
    OA_CU(cudaMemcpyAsync(e->Qr.p, Qr.data(), sizeof(float) * Qr.size(), cudaMemcpyHostToDevice, e->st));
    OA_CU(cudaMemcpyAsync(e->Qb.p, Qb.data(), sizeof(float) * Qb.size(), cudaMemcpyHostToDevice, e->st));
    OA_CU(cudaMemcpyAsync(e->qsum.p, qsum.data(), sizeof(double) * qsum.size(), cudaMemcpyHostToDevice, e->st));
    OA_CU(cudaMemcpyAsync(e->Rinv.p, Ri.data(), sizeof(double) * Ri.size(), cudaMemcpyHostToDevice, e->st));
    OA_CU(cudaStreamSynchronize(e->st));
    // An intercept as the first covariate makes every quantity of the scan
    // invariant to shifting a SNP column by a constant (its Q column is
    // proportional to 1 and the other Q columns are orthogonal to 1); the
    // kernels then work with x - mean, whose sums cancel far less.
    const char* ce = getenv("OA_CENTER");
    e->center = xl[0] != 0.f && !(ce && ce[0] == '0') && !quirk_on(e);
    for (int k = 1; k < n && e->center; ++k) e->center = xl[k] == xl[0];
    e->have_cov = true;
    e->t = 0;
    return OA_OK;
}

oa_status oa_set_traits(oa_engine* e, const float* y, int32_t t) {
    clear_stale_error(__func__);
    if (!e || !y) {
        set_err("null argument");
        return OA_ERR_ARG;
    }
    OA_CU(cudaSetDevice(e->cfg.device));
    AllocOn alloc_on(e->st);
    return set_traits_impl(e, y, t, false);
}

oa_status oa_set_traits_device(oa_engine* e, const float* y, int32_t t) {
    ApiClock api_clock("oa_set_traits_device", e);
    clear_stale_error(__func__);
    if (!e || !y) {
        set_err("null argument");
        return OA_ERR_ARG;
    }
    OA_CU(cudaSetDevice(e->cfg.device));
    AllocOn alloc_on(e->st);
    return set_traits_impl(e, y, t, true);
}

oa_status oa_run_snps(oa_engine* e, const float* xr, int32_t mb, oa_rows* out) {
    return run_snps_any(e, xr, mb, true, true, out);
}

oa_status oa_run_snps_device(oa_engine* e, const float* xr, int32_t mb, int32_t results_on_host, oa_rows* out) {
    ApiClock api_clock("oa_run_snps_device", e);
    return run_snps_any(e, xr, mb, false, results_on_host != 0, out);
}

oa_status oa_set_tuning(oa_engine* e, const oa_tuning* t) {
    clear_stale_error(__func__);
    if (!e || !t) {
        set_err("null argument");
        return OA_ERR_ARG;
    }
    if (t->chunk_snps < 0 || t->gemm_variant < 0 || t->gemm_variant > 4 || t->gemm_raster < 0 ||
        t->gemm_raster > 2 || t->stats_path < 0 || t->stats_path > 2 || t->lean_spb < 0 || t->lean_spb > 8) {
        set_err("tuning field out of range");
        return OA_ERR_ARG;
    }
    e->req = *t;
    ++e->tune_gen;
    return OA_OK;
}

oa_status oa_get_tuning(const oa_engine* e, oa_tuning* t) {
    if (!e || !t) {
        set_err("null argument");
        return OA_ERR_ARG;
    }
    t->chunk_snps = e->chunk;
    t->gemm_variant = e->variant;
    t->gemm_raster = e->raster;
    t->stats_path = e->t > 0 ? (e->use_pre ? 1 : 2) : e->req.stats_path;
    t->lean_spb = lean_group(e);
    return OA_OK;
}

oa_status oa_autotune(oa_engine* e, const float* xr_dev, int32_t mb, oa_tuning* best) {
    clear_stale_error(__func__);
    if (!e || !xr_dev || mb <= 0 || mb > e->cfg.max_snps) {
        set_err("invalid autotune arguments");
        return OA_ERR_ARG;
    }
    OA_CU(cudaSetDevice(e->cfg.device));
    AllocOn alloc_on(e->st);
    return autotune_impl(e, xr_dev, mb, best);
}

oa_status oa_set_column_model(oa_engine* e, int32_t in_cols, const float* weights, int32_t combine) {
    clear_stale_error(__func__);
    if (!e) {
        set_err("null engine");
        return OA_ERR_ARG;
    }
    if (in_cols == 0) {   // plain input (and no interactions)
        e->in_cols = 0;
        e->n_inter = e->inter_keep = 0;
        drop_graph(e);
        ++e->tune_gen;
        return OA_OK;
    }
    if (in_cols < 1 || in_cols > OA_MODEL_MAX_COLS || !weights) {
        set_err("column model of %d file columns per SNP (1..%d, with weights)", in_cols, OA_MODEL_MAX_COLS);
        return OA_ERR_ARG;
    }
    // a combined column without interactions yet: r = 1, or interaction columns follow (checked when a
    // block runs, so that the model and the interactions may be set in either order)
    const int want_r = combine ? (e->n_inter > 0 ? e->n_inter + e->inter_keep : 1) : in_cols;
    if ((!combine && (want_r != e->ru || e->n_inter > 0)) || (combine && e->n_inter > 0 && want_r != e->ru)) {
        set_err("column model: %s needs r = %d, the engine has r = %d",
                combine ? "a combined column" : "scaled columns (no interactions)", want_r, e->ru);
        return OA_ERR_ARG;
    }
    if (e->subset) {
        set_err("a column model does not apply to row subsets of a resident matrix");
        return OA_ERR_STATE;
    }
    e->in_cols = in_cols;
    e->model_combine = combine ? 1 : 0;
    for (int c = 0; c < OA_MODEL_MAX_COLS; ++c) e->model_w[c] = c < in_cols ? weights[c] : 0.f;
    drop_graph(e);
    ++e->tune_gen;
    return OA_OK;
}

oa_status oa_set_interactions(oa_engine* e, const float* inter, int32_t k, int32_t keep) {
    clear_stale_error(__func__);
    if (!e || (k > 0 && !inter)) {
        set_err("null argument");
        return OA_ERR_ARG;
    }
    if (k < 1 || k + (keep ? 1 : 0) != e->ru) {
        set_err("%d interaction columns%s need r = %d, the engine has r = %d", k, keep ? " + the SNP" : "",
                k + (keep ? 1 : 0), e->ru);
        return OA_ERR_ARG;
    }
    if (e->in_cols > 0 && !e->model_combine) {
        set_err("interactions apply to one model column per SNP (not the custom linear model)");
        return OA_ERR_ARG;
    }
    if (e->subset) {
        set_err("interactions do not apply to row subsets of a resident matrix");
        return OA_ERR_STATE;
    }
    OA_CU(cudaSetDevice(e->cfg.device));
    AllocOn alloc_on(e->st);
    OA_CHECK(e->inter.ensure((size_t)e->n * k));
    OA_CU(cudaMemcpyAsync(e->inter.p, inter, sizeof(float) * (size_t)e->n * k, cudaMemcpyHostToDevice, e->st));
    OA_CU(cudaStreamSynchronize(e->st));
    if (e->in_cols == 0) {   // plain single-column SNPs: the identity model
        e->in_cols = 1;
        e->model_combine = 1;
        for (int c = 0; c < OA_MODEL_MAX_COLS; ++c) e->model_w[c] = c == 0 ? 1.f : 0.f;
    }
    e->n_inter = k;
    e->inter_keep = keep ? 1 : 0;
    drop_graph(e);
    ++e->tune_gen;
    return OA_OK;
}

oa_status oa_set_snp_rows(oa_engine* e, const int32_t* rows, int32_t n_rows, int64_t ld) {
    ApiClock api_clock("oa_set_snp_rows", e);
    clear_stale_error(__func__);
    if (!e) {
        set_err("null engine");
        return OA_ERR_ARG;
    }
    if (rows && column_pass(e)) {
        set_err("a row subset does not apply with a column model or with r = %d (zero columns added)", e->ru);
        return OA_ERR_STATE;
    }
    OA_CU(cudaSetDevice(e->cfg.device));
    AllocOn alloc_on(e->st);
    drop_graph(e);
    ++e->tune_gen;
    if (!rows) {
        e->subset = false;
        e->x_ld = 0;
        return OA_OK;
    }
    if (n_rows != e->n || ld < n_rows) {
        set_err("row subset of %d rows (engine n = %d) from columns of %lld", n_rows, e->n, (long long)ld);
        return OA_ERR_ARG;
    }
    for (int j = 0; j < n_rows; ++j)
        if (rows[j] < 0 || rows[j] >= ld || (j > 0 && rows[j] <= rows[j - 1])) {
            set_err("row subset: rows must be ascending and within [0, %lld)", (long long)ld);
            return OA_ERR_ARG;
        }
    OA_CHECK(e->xrows.ensure(n_rows));
    OA_CU(cudaMemcpyAsync(e->xrows.p, rows, sizeof(int32_t) * n_rows, cudaMemcpyHostToDevice, e->st));
    OA_CU(cudaStreamSynchronize(e->st));
    e->x_ld = ld;
    e->subset = true;
    return OA_OK;
}

int64_t oa_device_bytes(const oa_engine* e) {
    if (!e) return 0;
    int64_t total = 0;
    for_each_buf(const_cast<oa_engine*>(e), [&](auto& b) { total += (int64_t)(b.n * sizeof(*b.p)); });
    return total;
}

oa_status oa_reserve(oa_engine* e, int32_t traits, int32_t snps) {
    ApiClock api_clock("oa_reserve", e);
    clear_stale_error(__func__);
    if (!e) {
        set_err("null argument");
        return OA_ERR_ARG;
    }
    if (traits < 1 || traits > e->cfg.max_traits || snps < 1 || snps > e->cfg.max_snps) {
        set_err("reservation of %d traits x %d SNPs (engine limits %d, %d)", traits, snps, e->cfg.max_traits,
                e->cfg.max_snps);
        return OA_ERR_ARG;
    }
    OA_CU(cudaSetDevice(e->cfg.device));
    AllocOn alloc_on(e->st);
    const size_t t = (size_t)std::max(traits, 1), n = (size_t)e->n, l = (size_t)e->l;
    {
        OA_CHECK(e->tsums.ensure(t * (2 + OA_MAX_L)));
        OA_CHECK(e->tcounts.ensure(t * 2));
        OA_CHECK(e->thash.ensure(t * 4));
        for (auto* b : {&e->pat, &e->zset, &e->tperm, &e->tinv}) OA_CHECK(b->ensure(t));
        OA_CHECK(e->Yt.ensure(t * e->n_pad));
        if (e->cfg.precision == OA_MIXED_BF16X3) {
            OA_CHECK(e->Yhi.ensure(t * e->n_pad));
            OA_CHECK(e->Ylo.ensure(t * e->n_pad));
        }
        OA_CHECK(e->rss0.ensure(t));
        for (auto* b : {&e->sst, &e->a_r2, &e->inv_ncorr, &e->vf}) OA_CHECK(b->ensure(t));
        OA_CHECK(e->nobs.ensure(t));
        OA_CHECK(e->b0.ensure(t * l));
        OA_CHECK(stage_reserve(e, 48 * t + 65536 + 16 * n / LEAN_ITEM_ROWS));
    }
    const auto t_traits = std::chrono::steady_clock::now();
    {
        // the smallest chunk the tuning picks by itself (narrow trait blocks give the most chunks)
        const int chunk = std::min(e->cfg.max_snps, e->req.chunk_snps > 0 ? e->req.chunk_snps : wave_chunk(e, 1));
        const long long slots = slots_needed(e, snps, traits, chunk);
        if (slots > (long long)INT32_MAX) {
            set_err("%lld stored-row slots exceed the sort's 2^31 limit", slots);
            return OA_ERR_ARG;
        }
        OA_CHECK(ensure_cap(e, slots));
        const size_t cap = (size_t)e->cap;   // slots, with the headroom ensure_cap adds
        // rows written: all slots but the block tails
        const long long tails = ((snps + chunk - 1) / chunk) * (long long)e->sm_count * EPI_WARPS_TC * EMIT_BLOCK;
        const size_t R = (size_t)std::max<long long>(1, slots - tails);
        OA_CHECK(e->keys.ensure(cap));
        OA_CHECK(e->keys2.ensure(cap));
        OA_CHECK(e->perm.ensure(cap));
        OA_CHECK(e->perm2.ensure(cap));
        OA_CHECK(e->rec2.ensure(R * rec_slots(e->r)));
        size_t tmp = 0;
        OA_CU(cub::DeviceRadixSort::SortPairs(nullptr, tmp, e->keys.p, e->keys2.p, e->perm.p, e->perm2.p, (int)cap, 0,
                                              64, e->st));
        OA_CHECK(e->cub_tmp.ensure(tmp));
        const auto t_dev = std::chrono::steady_clock::now();
        OA_CHECK(ensure_pinned(e->h_rec, e->h_rec_cap, R * rec_slots(e->r), e->retired_pinned));
        if (e->cfg.disp_cov) {
            OA_CHECK(e->cov2.ensure(R * l * 3));
            OA_CHECK(ensure_pinned(e->h_cov, e->h_cov_cap, R * l * 3, e->retired_pinned));
        }
        const auto t_pin = std::chrono::steady_clock::now();
        OA_CU(cudaStreamSynchronize(e->st));
        if (getenv("OA_TIMING")) {
            auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
                return std::chrono::duration<double, std::milli>(b - a).count();
            };
            const auto t_end = std::chrono::steady_clock::now();
            if (ms(api_clock.t0, t_end) >= 20.0)
                fprintf(stderr,
                        "[oa timing] oa_reserve: trait buffers %.1f ms, %zu row slots %.1f ms, page-locked rows "
                        "(%zu bytes) %.1f ms, stream sync %.1f ms\n",
                        ms(api_clock.t0, t_traits), cap, ms(t_traits, t_dev), (size_t)(R * rec_slots(e->r) * sizeof(Rec)),
                        ms(t_dev, t_pin), ms(t_pin, t_end));
        }
    }
    return OA_OK;
}

oa_status oa_enable_dense(oa_engine* e, int32_t on) {
    if (!e) return OA_ERR_ARG;
    e->dense_on = on != 0;
    return OA_OK;
}

oa_status oa_dense_last(oa_engine* e, float* beta, float* se, float* tstat, float* r2) {
    clear_stale_error(__func__);
    if (!e || !e->dense_on || e->last_mb == 0) {
        set_err("dense output was not enabled for the last SNP block");
        return OA_ERR_STATE;
    }
    OA_CU(cudaSetDevice(e->cfg.device));
    const size_t nd = (size_t)e->t * e->last_mb;
    // the device arrays hold r (padded) terms per test; the caller's hold ru
    std::vector<float> tmp(padded(e) ? nd * e->r : 0);
    auto get = [&](float* dst, const float* src) -> cudaError_t {
        if (!dst) return cudaSuccess;
        cudaError_t s = cudaMemcpyAsync(padded(e) ? tmp.data() : dst, src, sizeof(float) * nd * e->r,
                                        cudaMemcpyDeviceToHost, e->st);
        if (s != cudaSuccess || !padded(e)) return s;
        if ((s = cudaStreamSynchronize(e->st)) != cudaSuccess) return s;
        for (size_t q = 0; q < nd; ++q)
            for (int a = 0; a < e->ru; ++a) dst[q * e->ru + a] = tmp[q * e->r + a];
        return cudaSuccess;
    };
    OA_CU(get(beta, e->d_beta.p));
    OA_CU(get(se, e->d_se.p));
    OA_CU(get(tstat, e->d_t.p));
    if (r2) OA_CU(cudaMemcpyAsync(r2, e->d_r2.p, sizeof(float) * nd, cudaMemcpyDeviceToHost, e->st));
    OA_CU(cudaStreamSynchronize(e->st));
    return OA_OK;
}

oa_status oa_dense_flags(oa_engine* e, uint8_t* flags) {
    clear_stale_error(__func__);
    if (!e || !flags) {
        set_err("null argument");
        return OA_ERR_ARG;
    }
    if (!e->dense_on || e->last_mb == 0) {
        set_err("dense output was not enabled for the last SNP block");
        return OA_ERR_STATE;
    }
    OA_CU(cudaSetDevice(e->cfg.device));
    const size_t nd = (size_t)e->t * e->last_mb;
    OA_CU(cudaMemcpyAsync(flags, e->d_flags.p, nd, cudaMemcpyDeviceToHost, e->st));
    OA_CU(cudaStreamSynchronize(e->st));
    return OA_OK;
}

int64_t oa_kernel_launches(const oa_engine* e) { return e ? e->launches : 0; }

float oa_last_kernel_ms(const oa_engine* e, const char** name) {
    if (!e) return 0.f;
    if (name) *name = e->last_name;
    return e->last_ms;
}

float oa_last_stats_ms(const oa_engine* e) { return e ? e->stats_ms : 0.f; }
float oa_last_block_ms(const oa_engine* e) { return e ? e->block_ms : 0.f; }

}  // extern "C"
