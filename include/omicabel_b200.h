/*
 * omicabel_b200.h — C ABI of the B200 association engine.
 *
 * Drop-in for the blocked normal-equation OLS path of OmicABELnoMM
 * (Algorithm::partialNEQ_Blocked_STL_MD, src/Algorithm.cpp:322-886 of the
 * reference).  Two levels:
 *
 *  1. Whole-run entry points that replace the reference's process and
 *     solver entry:  oa_cli_main  ≙ main            (src/main.cpp:440-500)
 *                    oa_solve     ≙ Algorithm::solve(params, out, P_NEQ_B_OPT_MD)
 *                                                    (src/Algorithm.cpp:37-48)
 *     They read .fvi/.fvd inputs and write <out>_dis.txt (+ _sto.ibin and
 *     _sto.dbin with store_bin) exactly as the reference does.
 *
 *  2. A block engine for embedding, the device-side replacement of the
 *     solver's per-block work: covariates once (≙ AIOwrapper::load_AL +
 *     the Stl/rank-check steps, src/Algorithm.cpp:475-522), one trait block
 *     (≙ load_Yblock + replace_nans/sumSquares/XL'Y/Stl_corr,
 *     src/Algorithm.cpp:550-595), then SNP blocks (≙ load_ARblock through
 *     hpc_statistics, src/Algorithm.cpp:610-813).  It returns the stored
 *     results (the reference's list<resultH>) as flat arrays.
 *
 * Conventions: plain C types, column-major float32 matrices with the
 * individual (row) index contiguous — the layout of a .fvd file.  The
 * library never calls exit(); every entry point returns an oa_status and
 * oa_last_error() describes the last failure of the calling thread.  An
 * engine owns its device memory and is used from one host thread at a time.
 */
#ifndef OMICABEL_B200_H
#define OMICABEL_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OA_ABI_VERSION 1
#define OA_MAX_L 16   /* covariates, intercept included */
#define OA_MAX_R 8    /* columns per SNP (3, 5, 6 and 7 run as 4 or 8 with zero columns added on the device) */

typedef enum oa_status {
    OA_OK = 0,
    OA_ERR_ARG = 1,            /* invalid argument or size */
    OA_ERR_CUDA = 2,           /* CUDA runtime failure (message in oa_last_error) */
    OA_ERR_COLLINEAR = 3,      /* covariates linearly dependent (src/Algorithm.cpp:510-522) */
    OA_ERR_IO = 4,             /* file missing, short or malformed */
    OA_ERR_STATE = 5,          /* call out of order (e.g. SNP block before traits) */
    OA_ERR_NOMEM = 6,          /* device or host allocation failed */
    OA_ERR_UNSUPPORTED = 7,    /* sizes beyond this build's limits */
    OA_ERR_NUMERIC = 8         /* e.g. negative sum of squares (src/Algorithm.cpp:1096-1099) */
} oa_status;

typedef enum oa_precision {
    OA_PLAIN_FP32 = 0,   /* FP32 data, FP32 SIMT GEMM, FP64 small systems */
    OA_MIXED_BF16X3 = 1  /* XR'Y on tcgen05 tensor cores, BF16 hi/lo 3-product, FP32 accumulate */
} oa_precision;

/* ---------------------------------------------------------------------------
 * Block engine
 * ------------------------------------------------------------------------- */
typedef struct oa_engine oa_engine;

typedef struct oa_config {
    int32_t n;             /* individuals after exclusions (rows) */
    int32_t l;             /* covariates incl. intercept, 1..OA_MAX_L */
    int32_t r;             /* columns per SNP, 1..OA_MAX_R (r > 4 needs the SNP's 8 columns in one
                              SM's shared memory: n up to about 6,000) */
    int32_t max_traits;    /* largest trait block passed to oa_set_traits */
    int32_t max_snps;      /* largest SNP block passed to oa_run_snps* */
    int32_t precision;     /* oa_precision */
    int32_t device;        /* CUDA device ordinal */
    int32_t disp_cov;      /* -i: also report covariate terms of stored rows */
    int32_t store_all;     /* -f: store every test (thresholds ignored) */
    int32_t quirk_r2;      /* reproduce the reference's r>=2 downdate (src/Algorithm.cpp:1390-1396) */
    float min_r2_store;    /* effective R2 store threshold (src/Algorithm.cpp:338-339) */
    float min_t_store;     /* effective |t| store threshold (src/Algorithm.cpp:359) */
    float min_p_disp;      /* display P threshold, used for the significant-result count */
    int32_t real_n;        /* individuals before exclusions (nPct denominator) */
} oa_config;

/* Stored results of one SNP block, in reference output order
 * (trait, then SNP; coefficients h = p-1 .. start_h).  One row per
 * (trait, SNP) test that has at least one stored SNP term
 * (≙ resultH, src/Definitions.h:271-280); its stored coefficients are the
 * bits of coef_mask (bit h).  coef_* hold p entries per row. */
typedef struct oa_rows {
    int64_t count;             /* rows */
    const int32_t* trait;      /* trait index within the trait block */
    const int32_t* snp;        /* SNP index within the SNP block */
    const float* r2;           /* R2 of the test */
    const int32_t* n_used;     /* n - missing of the trait */
    const uint32_t* coef_mask; /* bit h set: coefficient h stored */
    const float* coef_b;       /* [count * p] beta */
    const float* coef_se;      /* [count * p] standard error */
    const float* coef_t;       /* [count * p] |t| */
    int64_t sig_cov_unrowed;   /* covariate terms with P < min_p_disp in tests without a stored row */
    int64_t tests;             /* tests evaluated */
    int64_t singular;          /* tests skipped as singular (the reference emits undefined values) */
} oa_rows;

/* Create an engine on cfg->device.  Replaces the allocations of
 * src/Algorithm.cpp:417-456 with device buffers sized by cfg. */
oa_status oa_engine_create(const oa_config* cfg, oa_engine** out);
oa_status oa_engine_destroy(oa_engine* e);

/* Covariates, host column-major n x l (NaN-free: the reader drops such rows).
 * ≙ load_AL + ssyrk Stl + sgesvd rank check (src/Algorithm.cpp:475-522). */
oa_status oa_set_covariates(oa_engine* e, const float* xl_host);

/* One trait block, host column-major n x t, NaN = missing.
 * ≙ load_Yblock, replace_nans, sumSquares, XL'Y, Stl_corr (src/Algorithm.cpp:550-595).
 * Traits are grouped by missingness pattern on the device. */
oa_status oa_set_traits(oa_engine* e, const float* y_host, int32_t t);
/* Same with a device pointer (column stride n). */
oa_status oa_set_traits_device(oa_engine* e, const float* y_dev, int32_t t);

/* One SNP block, host column-major n x (r*mb), NaN = missing dosage.
 * ≙ load_ARblock .. hpc_statistics (src/Algorithm.cpp:610-813).  Results
 * stay valid until the next call on this engine. */
oa_status oa_run_snps(oa_engine* e, const float* xr_host, int32_t mb, oa_rows* out);
/* Same with the SNP block already in device memory (column stride n).
 * With results_on_host = 0 the oa_rows pointers are device pointers and
 * are not sorted; with 1 they are host pointers in reference order. */
oa_status oa_run_snps_device(oa_engine* e, const float* xr_dev, int32_t mb,
                             int32_t results_on_host, oa_rows* out);

/* Dense per-test output for checking: beta/se/t of the r SNP terms
 * ([t][mb][r], trait-major) and R2 ([t][mb]) of the last SNP block,
 * copied to host arrays the caller provides.  Tests that are singular or
 * have RSS <= 0 hold NaN. */
oa_status oa_dense_last(oa_engine* e, float* beta, float* se, float* tstat, float* r2);
oa_status oa_enable_dense(oa_engine* e, int32_t on);

/* Status of each test of the last SNP block ([t][mb] bytes, trait-major, as
 * oa_dense_last), with dense output enabled: 0 = evaluated, no SNP term
 * passed the store filters; otherwise one of
 *   OA_TEST_SINGULAR  the (l+r) x (l+r) system is singular for this trait's
 *                     missingness pattern (monomorphic or collinear SNP);
 *                     skipped.  The reference ignores sposv's info and
 *                     prints undefined values (src/Algorithm.cpp:767-773);
 *   OA_TEST_RSS       residual sum of squares <= 0: skipped (src/Algorithm.cpp:1094-1099, 1119);
 *   OA_TEST_R2        R2 at or below the store threshold (without store_all):
 *                     no term stored (src/Algorithm.cpp:1119-1123);
 *   OA_TEST_STORED    at least one SNP term stored: the test has a row in oa_rows. */
#define OA_TEST_SINGULAR 1u
#define OA_TEST_RSS 2u
#define OA_TEST_R2 4u
#define OA_TEST_STORED 8u
oa_status oa_dense_flags(oa_engine* e, uint8_t* flags);

/* Row subset of device SNP blocks: after this call oa_run_snps_device reads
 * SNP columns of ld floats (e.g. a genotype matrix kept resident across
 * calls) and takes rows[0..n_rows) of each (ascending, n_rows = the
 * engine's n) as its individuals, gathered on the device chunk by chunk.
 * rows = NULL restores contiguous columns of n.  Not for host blocks
 * (oa_run_snps returns OA_ERR_STATE).  No counterpart in the reference
 * (its reader keeps the rows of the exclusion list's kept runs while loading a
 * SNP block, src/AIOwrapper.cpp:1098-1130). */
oa_status oa_set_snp_rows(oa_engine* e, const int32_t* rows, int32_t n_rows, int64_t ld);

/* Column model of the SNP blocks (the reference's dosage models, applied by
 * its reader, src/AIOwrapper.cpp:257-340, 1213-1275): after this call every
 * SNP of a block passed to oa_run_snps(_device) is in_cols file columns
 * (1..8), and the engine forms its r columns on the device:
 *   combine != 0: r = 1 column sum_c weights[c] * x_c  (additive: {2,1,0},
 *                 dominant: {1,1,0}, recessive: {1,0,0} on genotype
 *                 probabilities AA, AB[, BB]; custom additive: the factors file)
 *   combine == 0: r = in_cols columns weights[c] * x_c (custom linear model).
 * With interactions (oa_set_interactions, before or after this call) a
 * combined column becomes r = k (+1) columns.  in_cols = 0 restores plain
 * blocks of r columns per SNP.  Not with row subsets. */
#define OA_MODEL_MAX_COLS 8
oa_status oa_set_column_model(oa_engine* e, int32_t in_cols, const float* weights, int32_t combine);

/* Interaction columns (the reference's single-set interactions,
 * src/AIOwrapper.cpp:808-840): inter holds k columns of n values (the
 * engine's rows, column-major, no NaN); each SNP's model column x becomes the
 * r = k (+1 with keep) columns [I_1 x, ..., I_k x (, x)].  Needs one model
 * column per SNP (plain single-column SNPs or a combined dosage model) and
 * r = k + keep.  oa_set_column_model(e, 0, ...) clears them. */
oa_status oa_set_interactions(oa_engine* e, const float* inter, int32_t k, int32_t keep);

/* Device memory held by the engine's buffers, in bytes. */
int64_t oa_device_bytes(const oa_engine* e);

/* Allocates now what a trait block of up to `traits` traits and an SNP
 * block of up to `snps` SNPs need at the engine's store thresholds
 * (trait-sized device buffers, the stored-row buffers and their sort space
 * on the device, the pinned host buffer the rows come back in), so that
 * later calls within those sizes seldom allocate.  Pinned host allocations
 * are slow while other engines keep the GPU busy: a server reserves its
 * engines' buffers when it creates them.  No counterpart in the reference
 * (one scan per process). */
oa_status oa_reserve(oa_engine* e, int32_t traits, int32_t snps);

/* Size of the scratch array used by oa_scan_dense_noalloc (64 MiB).  Every
 * GPU on which the library is loaded holds this much device memory until the
 * process exits. */
#define OA_NOALLOC_SCRATCH_BYTES (64u << 20)

/* Plain-FP32 dense scan of one SNP block that allocates no memory.
 *
 * For callers that cannot call cudaMalloc: plug-ins whose host framework
 * owns the device memory pool and forbids raw allocations, and processes
 * whose device memory was reserved up front under a hard cap.  All
 * intermediates live in one static device array of OA_NOALLOC_SCRATCH_BYTES;
 * inputs and outputs are the caller's device buffers (column-major,
 * individual index contiguous): covariates n x l (NaN-free), traits n x t
 * (NaN = missing), dosages n x (r*mb) (NaN = mean-imputed); outputs
 * beta/se/|t| [t][mb][r] and R2 [t][mb] (NaN where the test is singular or
 * has RSS <= 0), the same numbers as oa_run_snps_device + oa_dense_last of
 * an engine with store_all.  Covariates are rejected with OA_ERR_COLLINEAR
 * by the engine's rule (a singular value below 1e-6), and also when their
 * condition number is beyond about 1e15 (the device QR breaks down).
 * Limits: r in {1, 2, 4}, l <= OA_MAX_L, t <= 2048, and all intermediates
 * (about 4*n*t + 9*t*mb*r*r + 8*n*l bytes) within the array; larger inputs
 * return OA_ERR_UNSUPPORTED.  Calls share the array: calls that overlap on
 * the GPU (other streams or threads) race.  The first call on a device looks
 * up the array's address.  The call reads small status words back to the
 * host and synchronises `stream` (a cudaStream_t; NULL = default stream)
 * before returning.  A CUDA error already pending on the calling thread
 * (cudaPeekAtLastError) is left in place and reported as OA_ERR_CUDA without
 * running.  No counterpart in the reference. */
oa_status oa_scan_dense_noalloc(const float* xl_dev, const float* y_dev, const float* xr_dev, int32_t n,
                                int32_t l, int32_t r, int32_t t, int32_t mb, float* beta_dev, float* se_dev,
                                float* t_dev, float* r2_dev, void* stream);

/* Launch parameters of the per-block kernels.  0 in a field = the engine's
 * own choice.  No counterpart in the reference (its block sizes mb/tb are
 * fixed at src/Algorithm.cpp:361-372). */
typedef struct oa_tuning {
    int32_t chunk_snps;    /* SNPs per device chunk: one launch of each per-block kernel */
    int32_t gemm_variant;  /* tensor-core pipeline: 1 = K-block 32 x 4 stages, 2 = K-block 64 x 2 stages,
                              3 = CTA pairs on neighbouring SMs (2-SM MMA, 256 x 256 tiles), K-block 32 x 6,
                              4 = CTA pairs, K-block 64 x 3 (the default); trait blocks of at most 128
                              traits use 1-SM tiles of 64 or 128 columns whatever the variant */
    int32_t gemm_raster;   /* GEMM tile order: 1 = trait tiles inner, 2 = SNP tiles inner */
    int32_t stats_path;    /* per-SNP sums: 1 = pre-GEMM + batched Schur kernel, 2 = row gathers */
    int32_t lean_spb;      /* SNPs per CTA group of the column-statistics kernel (1..8/r) */
} oa_tuning;

/* Set / read the tuning (oa_get_tuning reports the values in effect for
 * the current trait block, zeros resolved). */
oa_status oa_set_tuning(oa_engine* e, const oa_tuning* t);
oa_status oa_get_tuning(const oa_engine* e, oa_tuning* t);

/* Autotuner: times candidate tunings on the device SNP block xr_dev (mb
 * SNPs, a sample of the real data; after oa_set_traits*) by coordinate
 * descent over the fields of oa_tuning (device time of the per-block
 * kernels, CUDA events), keeps the fastest in the engine and returns it in
 * *best (may be NULL).  A chunk size set with oa_set_tuning before the call
 * is kept fixed.  Results of the trial runs are discarded. */
oa_status oa_autotune(oa_engine* e, const float* xr_dev, int32_t mb, oa_tuning* best);

/* Number of kernel launches this engine issued so far (instrumentation). */
int64_t oa_kernel_launches(const oa_engine* e);
/* Device time (ms) of the dominant kernel in the last SNP block and its name. */
float oa_last_kernel_ms(const oa_engine* e, const char** name);
/* Device time (ms) of the per-SNP statistics kernel in the last SNP block. */
float oa_last_stats_ms(const oa_engine* e);
/* Device time (ms) of the whole last SNP block: CUDA events on the engine's
 * stream before its first launch and after its last (the stored-row count
 * read-back and, for host results, the sort and copy not included). */
float oa_last_block_ms(const oa_engine* e);

/* ---------------------------------------------------------------------------
 * Whole-run entry points
 * ------------------------------------------------------------------------- */
typedef struct oa_settings {
    const char* fname_xl;        /* -c, without extension */
    const char* fname_xr;        /* -g */
    const char* fname_y;         /* -p */
    const char* fname_out;       /* -o */
    const char* fname_exclude;   /* -x, NULL or "" for none */
    int32_t r;                   /* -n */
    float min_p_disp;            /* -d */
    float min_p_store;           /* -s */
    float min_r2_disp;           /* -r */
    float min_r2_store;          /* -e */
    int32_t store_bin;           /* -b */
    int32_t disp_cov;            /* -i */
    int32_t store_all;           /* -f */
    int32_t precision;           /* oa_precision (default plain) */
    int32_t device;
    int32_t quirk_r2;
    int32_t verbose;             /* progress characters and messages on stdout */
    int32_t shard;               /* this process's SNP shard, 0..shards-1 (≙ mpi_id) */
    int32_t shards;              /* SNP shards (≙ mpi_num_threads, src/AIOwrapper.cpp:95-117): with
                                    shards > 1 and m >= shards, shard k scans SNPs [k*m/shards, ...)
                                    (the last shard also the remainder) and writes
                                    <out>_mpi<k+1>__dis.txt etc. with shard-local SNP indices */
    int32_t dosage_model;        /* 0 none; 1 additive (-j), 2 dominant (-k), 3 recessive (-l) on r = 2
                                    or 3 genotype-probability columns per SNP (AA, AB[, BB]);
                                    4 custom linear (-z), 5 custom additive (-y) with the factors of
                                    fname_factors (src/AIOwrapper.cpp:257-340) */
    const char* fname_factors;   /* -z / -y: whitespace-separated factors, one per file column of a SNP */
    const char* fname_interactions; /* -v: .fvi/.fvd with k interaction columns; each SNP column x
                                       becomes [I_1 x, ..., I_k x, x] (r = k + 1) and rows with a NaN
                                       interaction value are excluded (src/AIOwrapper.cpp:371-540) */
    int32_t multi_interactions;  /* -w: with fname_interactions, one analysis per interaction column h:
                                    each SNP column x becomes the r = 2 columns [I_h x, x] of its own
                                    test, k tests per SNP, output in blocks of max(1, mb/k) SNPs x k
                                    columns with the names I<h>_<SNP> and I<h>_o_<SNP>
                                    (src/AIOwrapper.cpp:441-452, 618-660, 1208-1241) */
} oa_settings;

typedef struct oa_outputs {
    uint64_t total_sig_results;  /* ≙ Outputs.total_sig_results (src/Definitions.h:256) */
    double duration_s;
    int64_t tests;
    int64_t rows_written;
    int64_t singular;
} oa_outputs;

/* Fill s with the reference defaults (src/Algorithm.cpp:277-311). */
void oa_default_settings(oa_settings* s);
/* ≙ Algorithm::solve(params, out, P_NEQ_B_OPT_MD). */
oa_status oa_solve(const oa_settings* s, oa_outputs* out);
/* ≙ main of the reference CLI: same flags, exit status 0 / 1. */
int oa_cli_main(int argc, char** argv);

/* Re-thresholds the binary outputs <source>.ibin / <source>.dbin (written
 * with store_bin / -b) into <dest>.txt: rows whose P is below min_p_disp and
 * whose R2 is above min_r2 (force_all: every stored term), covariate terms
 * only with include_cov and when the files hold them; the reference's
 * column formats.  ≙ the reference's OmicOUT tool (OmicOUT/main.cpp:227-483),
 * including its reading of at most t blocks and its 16-bit SNP indices.
 * *rows_printed (may be NULL) receives the number of rows written. */
oa_status oa_omicout(const char* source, const char* dest, float min_p_disp, float min_r2, int32_t force_all,
                     int32_t include_cov, int64_t* rows_printed);
/* ≙ main of the reference's omicout (-b <base> -o <base> -d <P> [-r <R2>]
 * [-i] [-f]; OmicOUT/main.cpp:86-227): exit status 0 / 1. */
int oa_omicout_main(int argc, char** argv);

/* SNP range [*first, *first + *count) of shard `shard` of `shards` over m
 * SNPs: the reference's MPI split (src/AIOwrapper.cpp:95-117): m / shards
 * each, the last shard also the remainder; no split when m < shards. */
oa_status oa_shard_range(int32_t m, int32_t shard, int32_t shards, int32_t* first, int32_t* count);

/* |t| -> P exactly as the reference (long double, src/Algorithm.cpp:1159-1167). */
long double oa_pvalue(float t);
/* P threshold -> |t| threshold (src/Utility.cpp:244-250). */
float oa_t_threshold(float p);

const char* oa_last_error(void);
int32_t oa_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* OMICABEL_B200_H */
