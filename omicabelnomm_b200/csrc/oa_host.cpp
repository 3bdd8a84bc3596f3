// Host side of the drop-in: .fvi/.fvd reading with the reference's row
// selection, the whole-run driver (oa_solve ≙ Algorithm::solve), the
// _dis.txt / _sto.ibin / _sto.dbin writers and the CLI (oa_cli_main ≙ main).
//
// Reference files followed: src/main.cpp (CLI), src/AIOwrapper.cpp
// (initialize, exclusion list, removeALmissings, async_io writer),
// src/Algorithm.cpp:322-886 (block loop, thresholds, hpc_statistics
// filters), src/Utility.cpp:244-268 (getTvalue, float16 truncation).
#include <getopt.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <future>
#include <sstream>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "oa_trace.h"
#include "omicabel_b200.h"

extern "C" void oa__set_error(const char* msg);  // oa_engine.cu: shared oa_last_error() text

namespace {

thread_local std::string h_err;

void herr(const char* fmt, ...) {
    char buf[2048];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    h_err = buf;
    oa__set_error(buf);
}

constexpr double ONE_OVER_SQRT2 = 0.7071067811865475244008443621048490392848359376884740;

// ---------------------------------------------------------------------------
// .fvi / .fvd (src/AIOwrapper.h:145-175, src/AIOwrapper.cpp:2294-2317)
// ---------------------------------------------------------------------------
struct Fvi {
    uint16_t type = 0;
    uint32_t nelements = 0, nobs = 0, nvar = 0, bytes_per_record = 0, bits_per_record = 0, namelength = 0;
    std::vector<char> names;  // (nobs + nvar) * namelength raw bytes
    // bytes of one stored value: 4 (float, type 5) or 8 (double, type 6)
    size_t elem_bytes() const { return type == 6 ? 8 : 4; }
    std::string obs_name(size_t i) const { return cstr(i); }
    std::string var_name(size_t i) const { return cstr(nobs + i); }
    const char* raw(size_t i) const { return names.data() + i * namelength; }
    std::string cstr(size_t i) const {
        const char* p = names.data() + i * namelength;
        size_t k = 0;
        while (k < namelength && p[k]) ++k;
        return std::string(p, k);
    }
};

bool read_fvi(const std::string& path, Fvi& f) {
    FILE* fp = fopen(path.c_str(), "rb");
    if (!fp) {
        herr("Error reading file: %s", path.c_str());
        return false;
    }
    unsigned char hdr[48];
    if (fread(hdr, 1, 48, fp) != 48) {
        fclose(fp);
        herr("%s: truncated header", path.c_str());
        return false;
    }
    auto u32 = [&](int off) {
        uint32_t v;
        memcpy(&v, hdr + off, 4);
        return v;
    };
    memcpy(&f.type, hdr, 2);
    f.nelements = u32(4);
    f.nobs = u32(8);
    f.nvar = u32(12);
    f.bytes_per_record = u32(16);
    f.bits_per_record = u32(20);
    f.namelength = u32(24);
    const size_t nb = ((size_t)f.nobs + f.nvar) * f.namelength;
    f.names.assign(nb, 0);
    const size_t got = fread(f.names.data(), 1, nb, fp);
    fclose(fp);
    if (got != nb) {
        herr("%s: %zu name bytes, header needs %zu", path.c_str(), got, nb);
        return false;
    }
    // the reference reads every .fvd as float32 and never checks `type`
    // (src/AIOwrapper.cpp:1103-1125), although its header declares the
    // DatABEL types (src/AIOwrapper.h:145-153) and a doublefileType flag
    // (src/AIOwrapper.h:41) that nothing sets.  Here float (type 5) and double
    // (type 6, converted to float as it is read) are accepted; the integer
    // types are refused.
    const bool is_float = f.type == 5 && f.bytes_per_record == 4;
    const bool is_double = f.type == 6 && f.bytes_per_record == 8;
    if (!is_float && !is_double) {
        herr("%s: data type %u with %u bytes per record: only float (type 5, 4 bytes) and double (type 6, "
             "8 bytes) are supported", path.c_str(), f.type, f.bytes_per_record);
        return false;
    }
    return true;
}

// The .fvd beside an .fvi must hold nobs * nvar values of the declared type
// (a shorter file would end in a failed read halfway through a scan).
bool check_fvd(const std::string& prefix, const Fvi& f) {
    struct stat sb;
    const std::string path = prefix + ".fvd";
    if (stat(path.c_str(), &sb) != 0) {
        herr("Error reading file: %s", path.c_str());
        return false;
    }
    const unsigned long long want = (unsigned long long)f.nobs * f.nvar * f.elem_bytes();
    if ((unsigned long long)sb.st_size < want) {
        herr("%s: %lld bytes, the header's %u x %u values of %zu bytes need %llu (truncated file)", path.c_str(),
             (long long)sb.st_size, f.nobs, f.nvar, f.elem_bytes(), want);
        return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// host threads (output formatting, genotype reading)
// ---------------------------------------------------------------------------
// All hardware threads, or OA_HOST_THREADS; at most 64.
int host_threads() {
    static const int n = [] {
        int h = (int)std::thread::hardware_concurrency();
        if (const char* v = getenv("OA_HOST_THREADS")) h = atoi(v);
        return std::max(1, std::min(h, 64));
    }();
    return n;
}

// f(part) for part = 0 .. parts-1, part 0 on the calling thread.
template <class F>
void parallel_parts(int parts, F&& f) {
    if (parts <= 1) {
        f(0);
        return;
    }
    std::vector<std::thread> th;
    th.reserve((size_t)parts - 1);
    for (int i = 1; i < parts; ++i) th.emplace_back([&f, i] { f(i); });
    f(0);
    for (auto& x : th) x.join();
}

// count values starting at value index `first` of an .fvd, as float (64-bit
// file offsets: files beyond 2^31 values, which the reference's int offsets
// cannot address, src/AIOwrapper.cpp:909-913, 1196).
bool read_values(FILE* fp, size_t elem_bytes, size_t first, size_t count, float* dst, std::vector<double>& dbl) {
    // large reads in parallel slices (pread on the file descriptor: the page cache copies with
    // several host threads)
    const int fd = fileno(fp);
    if (elem_bytes != 4) dbl.resize(count);
    char* base = elem_bytes == 4 ? reinterpret_cast<char*>(dst) : reinterpret_cast<char*>(dbl.data());
    const size_t bytes = elem_bytes * count;
    const off_t off0 = (off_t)(elem_bytes * first);
    const int parts = bytes >= ((size_t)64 << 20) ? std::min(host_threads(), 16) : 1;
    std::atomic<bool> ok{true};
    parallel_parts(parts, [&](int i) {
        size_t a = bytes * (size_t)i / parts, b = bytes * (size_t)(i + 1) / parts;
        while (a < b && ok.load(std::memory_order_relaxed)) {
            const ssize_t got = pread(fd, base + a, b - a, off0 + (off_t)a);
            if (got <= 0) {
                if (got < 0 && errno == EINTR) continue;
                ok = false;
                return;
            }
            a += (size_t)got;
        }
    });
    if (!ok) return false;
    if (elem_bytes != 4)
        parallel_parts(parts, [&](int i) {
            const size_t a = count * (size_t)i / parts, b = count * (size_t)(i + 1) / parts;
            for (size_t q = a; q < b; ++q) dst[q] = (float)dbl[q];
        });
    return true;
}

// Kept rows as (start, length) runs, the reference's exclusion list.
using Runs = std::vector<std::pair<int, int>>;

// src/AIOwrapper.cpp:2146-2233 (read_excludeList): "first [second]" per line,
// 1-based inclusive; a one-number line leaves `second` unchanged and is read
// as a single index; reading stops once a range reaches n.
bool exclusion_rows(const std::string& fname, int n, std::vector<char>& keep, int& excluded, bool verbose) {
    std::ifstream f(fname.c_str());
    if (!f) {
        herr("Error reading exclude list file.");
        return false;
    }
    std::string line;
    int first = 0, second = 0, prev_second = -1;
    excluded = 0;
    if (verbose) printf("Excluding Ids: \n");
    while (second < n && std::getline(f, line)) {
        std::istringstream iss(line);
        int a, b;
        if (iss >> a) first = a;
        if (iss >> b) second = b;
        if (prev_second > first) {
            herr("Please provide valid positive ordered indixes! %d > %d", prev_second, first);
            return false;
        }
        if (second == prev_second) {
            if (verbose) printf("%d, ", first);
            second = first;
        } else {
            if (verbose) printf("%d-%d, ", first, second);
            if (first > second) {
                herr("Please provide ordered pairs!");
                return false;
            }
            if (first < 1 || second < 1) {
                herr("Please provide valid positive indixes!");
                return false;
            }
        }
        prev_second = second;
        for (int i = first - 1; i <= second - 1; ++i)
            if (i >= 0 && i < n && keep[i]) {
                keep[i] = 0;
                ++excluded;
            }
    }
    if (excluded >= n) {
        herr("Exclusion List excluded all data! Total Ids: %d Excluded Ids: %d", n, excluded);
        return false;
    }
    if (verbose) printf("Excluded: %d Using: %d\n", excluded, n - excluded);
    return true;
}

Runs keep_runs(const std::vector<char>& keep) {
    Runs r;
    const int n = (int)keep.size();
    for (int i = 0; i < n;) {
        if (!keep[i]) {
            ++i;
            continue;
        }
        int j = i;
        while (j < n && keep[j]) ++j;
        r.emplace_back(i, j - i);
        i = j;
    }
    return r;
}

// Read variables [v0, v0+count) of a .fvd file of elem_bytes-byte values,
// keeping only the rows in `runs`, into dst (count columns of `kept` floats each).
bool read_columns(FILE* fp, size_t elem_bytes, size_t fileN, size_t v0, size_t count, const Runs& runs,
                  size_t kept, float* dst, std::vector<float>& scratch, std::vector<double>& dbl) {
    const bool all = runs.size() == 1 && runs[0].first == 0 && (size_t)runs[0].second == fileN;
    if (all) return read_values(fp, elem_bytes, fileN * v0, fileN * count, dst, dbl);
    scratch.resize(fileN * count);
    if (!read_values(fp, elem_bytes, fileN * v0, fileN * count, scratch.data(), dbl)) return false;
    for (size_t c = 0; c < count; ++c) {
        const float* src = scratch.data() + c * fileN;
        float* out = dst + c * kept;
        size_t pos = 0;
        for (const auto& run : runs) {
            memcpy(out + pos, src + run.first, sizeof(float) * run.second);
            pos += run.second;
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// statistics helpers shared with the writer
// ---------------------------------------------------------------------------
long double pvalue_ld(float tf) {
    // src/Algorithm.cpp:1159-1167: t is the float |b/SE| held in a long double
    const long double t = (long double)tf;
    if (t < 1.6) {
        const float t1 = (float)(4.4 - t);
        return 0.5 - (long double)(0.1 * (double)t1) * t;
    }
    return erfcl(t * (long double)ONE_OVER_SQRT2);
}

long double erf_inv_ld(long double z) {
    // Newton's method on erfl(x) - z, started from Winitzki's closed form
    if (z <= -1.0L) return -HUGE_VALL;
    if (z >= 1.0L) return HUGE_VALL;
    if (z == 0.0L) return 0.0L;
    const long double a = 0.147L, pi = 3.141592653589793238462643383279502884L;
    const long double ln = logl(1.0L - z * z);
    const long double t1 = 2.0L / (pi * a) + ln / 2.0L;
    long double x = sqrtl(sqrtl(t1 * t1 - ln / a) - t1);
    if (z < 0) x = -x;
    const long double c = 2.0L / sqrtl(pi);
    for (int it = 0; it < 100; ++it) {
        const long double step = (erfl(x) - z) / (c * expl(-x * x));
        x -= step;
        if (fabsl(step) <= 1e-19L * (1.0L + fabsl(x))) break;
    }
    return x;
}

uint16_t float16_trunc(float v) {
    // top 16 bits of the IEEE bits (src/Utility.cpp:261-268)
    uint32_t u;
    memcpy(&u, &v, 4);
    return (uint16_t)(u >> 16);
}

// ---------------------------------------------------------------------------
// number formatting of the text output (the same characters as printf)
// ---------------------------------------------------------------------------
// Decimal digits of v.
inline char* put_u64(char* o, uint64_t v) {
    char d[20];
    int k = 0;
    do {
        d[k++] = (char)('0' + v % 10);
        v /= 10;
    } while (v);
    while (k) *o++ = d[--k];
    return o;
}

// printf("%.Nf", (double)f), N <= 7: the float's exact binary value m 2^e scaled by 10^N and rounded
// to the nearest integer, ties to even, as glibc rounds the exact value; the sign of negative values
// and of -0 is kept.  NaN, infinities and |f| >= 2^40 go to snprintf.
inline char* put_fixed(char* o, float f, int N) {
    static constexpr uint64_t P10[8] = {1, 10, 100, 1000, 10000, 100000, 1000000, 10000000};
    uint32_t u;
    memcpy(&u, &f, 4);
    const uint32_t ex = (u >> 23) & 0xffu, fr = u & 0x7fffffu;
    if (ex == 0xffu || ex >= 127u + 40u) return o + snprintf(o, 64, "%.*f", N, (double)f);
    const uint64_t m = ex ? (fr | 0x800000u) : fr;
    const int e = ex ? (int)ex - 150 : -149;
    const unsigned __int128 num = (unsigned __int128)m * P10[N];   // < 2^48
    uint64_t q;
    if (e >= 0) {
        q = (uint64_t)(num << e);   // < 2^64 for e <= 16
    } else if (-e >= 127) {
        q = 0;
    } else {
        const int sh = -e;
        const unsigned __int128 qq = num >> sh, rem = num - (qq << sh), half = (unsigned __int128)1 << (sh - 1);
        q = (uint64_t)qq + ((rem > half || (rem == half && (qq & 1))) ? 1u : 0u);
    }
    if (u >> 31) *o++ = '-';
    o = put_u64(o, q / P10[N]);
    if (N > 0) {
        uint64_t fp = q % P10[N];
        *o++ = '.';
        for (int d = N - 1; d >= 0; --d) {
            o[d] = (char)('0' + fp % 10);
            fp /= 10;
        }
        o += N;
    }
    return o;
}

// printf("%.7Le", v) for a long double v (the P column): the exact value M 2^e (64-bit M) times
// 10^(7-d), d = floor(log10 v), in 192-bit integer arithmetic, rounded to nearest with ties to even
// as glibc rounds the exact value.  1e-30 <= v < 1 takes this path (10^(7-d) < 2^127, e <= -64);
// anything else (0, NaN, infinities, negative, smaller or larger values) goes to snprintf.
inline char* put_sci7(char* o, long double v) {
    using u128 = unsigned __int128;
    if (!(v >= 1e-30L && v < 1.0L)) return o + snprintf(o, 64, "%.7Le", v);
    int ex = 0;
    const long double fr = frexpl(v, &ex);        // v = fr 2^ex, fr in [0.5, 1)
    const uint64_t M = (uint64_t)ldexpl(fr, 64);   // the 64 mantissa bits, exactly
    const int sh = 64 - ex;                        // v = M 2^-sh, sh in [65, 164]
    static const std::vector<u128> P10 = [] {
        std::vector<u128> t(39, 1);
        for (size_t i = 1; i < t.size(); ++i) t[i] = t[i - 1] * 10;
        return t;
    }();
    // 2^(ex-1) <= v < 2^ex: d is floor(ex log10 2) or one less (the loop steps down once if needed)
    int d = (int)std::floor(ex * 0.30102999566398119521);
    for (int attempt = 0; attempt < 3; ++attempt) {
        const int k = 7 - d;
        if (k < 0 || k > 38) break;
        const u128 p = P10[(size_t)k];
        // N = M 10^k = n2 2^128 + lo
        const u128 a = (u128)M * (uint64_t)p, b = (u128)M * (uint64_t)(p >> 64);
        const u128 mid = (a >> 64) + (uint64_t)b;
        const u128 lo = (mid << 64) | (uint64_t)a;
        const uint64_t n2 = (uint64_t)((b >> 64) + (mid >> 64));
        // q = floor(N 2^-sh), the half bit and the bits below it
        const u128 q0 = sh >= 128 ? (u128)(n2 >> (sh - 128)) : (((u128)n2 << (128 - sh)) | (lo >> sh));
        const int hb = sh - 1;
        const bool half = hb < 128 ? ((lo >> hb) & 1) != 0 : ((n2 >> (hb - 128)) & 1) != 0;
        const bool sticky = hb <= 128 ? (hb == 128 ? lo != 0 : (lo & (((u128)1 << hb) - 1)) != 0)
                                      : (lo != 0 || (n2 & ((1ull << (hb - 128)) - 1)) != 0);
        const u128 q = q0 + ((half && (sticky || (q0 & 1))) ? 1 : 0);
        if (q < 10000000u) {
            --d;
            continue;
        }
        if (q >= 100000000u) {
            ++d;
            continue;
        }
        uint64_t rest = (uint64_t)q % 10000000u;
        *o++ = (char)('0' + (uint64_t)q / 10000000u);
        *o++ = '.';
        for (int i = 6; i >= 0; --i) {
            o[i] = (char)('0' + rest % 10);
            rest /= 10;
        }
        o += 7;
        *o++ = 'e';
        *o++ = d < 0 ? '-' : '+';
        const int ad = d < 0 ? -d : d;
        if (ad < 10) *o++ = '0';
        return put_u64(o, (uint64_t)ad);
    }
    return o + snprintf(o, 64, "%.7Le", v);
}

// ---------------------------------------------------------------------------
// output writer (≙ async_io's write loop, src/AIOwrapper.cpp:1440-1558)
// ---------------------------------------------------------------------------
// The stored rows of one engine call, owned by the writer, and the order in
// which the reference writes them: write block k (one trait block x one
// reference SNP block) is rows order[blk_off[k] .. blk_off[k+1]), in (trait,
// SNP) order, with its trait base and its first SNP (the AR offset).
struct RowBatch {
    int p = 0;
    std::vector<int32_t> trait, snp, n_used;   // snp: index within the shard
    std::vector<float> r2, b, se, t;           // b, se, t: [row * p + h]
    std::vector<uint32_t> mask;
    std::vector<int64_t> order, blk_off{0};
    std::vector<int32_t> blk_trait_base, blk_ar_off;

    // Copy of an engine call's rows (engine memory, valid until its next call), split into the
    // reference's SNP blocks of mb_ref SNPs starting at shard SNP s0.
    static RowBatch from_call(const oa_rows& rr, int p, int s0, int cnt, int mb_ref, int trait_base) {
        RowBatch B;
        const size_t c = (size_t)rr.count;
        B.p = p;
        B.trait.resize(c);
        B.snp.resize(c);
        B.n_used.resize(c);
        B.r2.resize(c);
        B.mask.resize(c);
        B.b.resize(c * p);
        B.se.resize(c * p);
        B.t.resize(c * p);
        // the copies of a large call on all host threads (the next engine call waits for them)
        const int parts = (int)std::max<size_t>(1, std::min<size_t>((size_t)host_threads(), c / 65536));
        parallel_parts(parts, [&](int i) {
            const size_t a = c * (size_t)i / parts, e = c * (size_t)(i + 1) / parts;
            std::copy(rr.trait + a, rr.trait + e, B.trait.begin() + a);
            for (size_t q = a; q < e; ++q) B.snp[q] = rr.snp[q] + s0;
            std::copy(rr.n_used + a, rr.n_used + e, B.n_used.begin() + a);
            std::copy(rr.r2 + a, rr.r2 + e, B.r2.begin() + a);
            std::copy(rr.coef_mask + a, rr.coef_mask + e, B.mask.begin() + a);
            std::copy(rr.coef_b + a * p, rr.coef_b + e * p, B.b.begin() + a * p);
            std::copy(rr.coef_se + a * p, rr.coef_se + e * p, B.se.begin() + a * p);
            std::copy(rr.coef_t + a * p, rr.coef_t + e * p, B.t.begin() + a * p);
        });
        // stable counting sort by reference block (rows arrive in (trait, SNP) order)
        const int nblk = (cnt + mb_ref - 1) / mb_ref;
        std::vector<int64_t> cntb((size_t)nblk + 1, 0);
        for (size_t q = 0; q < c; ++q) ++cntb[(size_t)rr.snp[q] / mb_ref + 1];
        for (int k = 0; k < nblk; ++k) cntb[(size_t)k + 1] += cntb[k];
        B.blk_off = cntb;
        B.order.resize(c);
        for (size_t q = 0; q < c; ++q) B.order[(size_t)cntb[(size_t)rr.snp[q] / mb_ref]++] = (int64_t)q;
        for (int k = 0; k < nblk; ++k) {
            B.blk_trait_base.push_back(trait_base);
            B.blk_ar_off.push_back(s0 + k * mb_ref);
        }
        return B;
    }
};

struct Writer {
    FILE* dis = nullptr;
    FILE* dbin = nullptr;
    bool store_bin = false, store_all = false, disp_cov = false;
    long double min_p_disp = 0;
    float min_r2_disp = 0;
    int l = 0, r = 0, p = 0, real_n = 0, mb_ref = 500;
    int name_base = 0;   // first SNP of this shard in the genotype file (names only; indices are shard-local)
    int name_stride = 1;           // file columns per SNP
    bool name_first_only = false;  // a combined dosage model names a SNP by its first file column
    int n_inter = 0;               // interaction columns: SNP term a < n_inter is named "I<a+1>x<SNP>"
    // one analysis per interaction column (-w): SNP indices count (SNP, column) pairs in blocks of
    // multi_fmb file SNPs x multi_k columns; term 0 is "I<h>_<SNP>", term 1 "I<h>_o_<SNP>"
    int multi_k = 0, multi_fmb = 1, multi_m = 0;
    const Fvi* fy = nullptr;
    const Fvi* fl = nullptr;
    const Fvi* fr = nullptr;
    uint64_t total_sig = 0;
    int64_t rows_written = 0;
    std::future<void> pending;   // the batch being formatted and written
    bool write_failed = false;   // an output write failed (disk full, I/O error)

    // Output of a contiguous range of a batch's write order: text, binary records, counts.
    struct Segment {
        std::string txt, bin;
        uint64_t sig = 0;
        int64_t rows = 0;
    };

    // (pointer, length) of a name of an .fvi name table (NUL-terminated or namelength bytes)
    static std::pair<const char*, int> name_of(const Fvi* f, size_t var) {
        const char* s = f->raw((size_t)f->nobs + var);
        int k = 0;
        while (k < (int)f->namelength && s[k]) ++k;
        return {s, k};
    }
    template <class T>
    static void put(std::string& out, T v) {
        out.append(reinterpret_cast<const char*>(&v), sizeof v);
    }

    // Rows order[a, b) of the batch, formatted exactly as the reference writes them: the text rows
    // of the coefficients that pass the display filters, the .dbin block headers, records and
    // stored coefficients (src/AIOwrapper.cpp:1454-1531).
    void format_range(const RowBatch& B, int64_t a, int64_t b, Segment& S) const {
        const int start_h = disp_cov ? 1 : l;
        const int nl = (int)std::max({fy->namelength, fl->namelength, fr->namelength});
        std::vector<char> line((size_t)3 * nl + 512), an((size_t)2 * nl + 64);
        size_t k = (size_t)(std::upper_bound(B.blk_off.begin(), B.blk_off.end(), a) - B.blk_off.begin()) - 1;
        for (int64_t pos = a; pos < b; ++pos) {
            while (pos >= B.blk_off[k + 1]) ++k;
            const int64_t q = B.order[(size_t)pos];
            if (pos == B.blk_off[k] && dbin && !store_all) {
                put<int32_t>(S.bin, B.blk_trait_base[k] + B.trait[(size_t)q]);
                put<int32_t>(S.bin, (int32_t)(B.blk_off[k + 1] - B.blk_off[k]));
                put<int32_t>(S.bin, B.blk_ar_off[k] * r);
            }
            const int ytr = B.blk_trait_base[k] + B.trait[(size_t)q];
            const int snp = B.snp[(size_t)q];
            const int ii = snp - B.blk_ar_off[k];
            const uint32_t mask = B.mask[(size_t)q];
            const int nused_i = B.n_used[(size_t)q];
            const uint16_t nused = (uint16_t)nused_i;
            const float npct = (float)nused_i / (float)real_n;
            const float r2 = B.r2[(size_t)q];
            if (dbin) {
                put<uint16_t>(S.bin, nused);
                put<uint16_t>(S.bin, float16_trunc(r2));
                if (!store_all) {
                    uint8_t sz = 0;
                    for (int h = p - 1; h >= start_h; --h) sz += (mask >> h) & 1u;
                    put<uint8_t>(S.bin, sz);
                }
            }
            for (int h = p - 1; h >= start_h; --h) {
                if (!((mask >> h) & 1u)) continue;
                const float Bv = B.b[(size_t)q * B.p + h];
                const float SE = B.se[(size_t)q * B.p + h];
                const float T = B.t[(size_t)q * B.p + h];
                const long double P = pvalue_ld(T);
                if (min_p_disp > P) ++S.sig;
                const int ar_idx = ii * r + (h >= l ? h - l : 0);
                const uint8_t al_idx = h >= l ? (uint8_t)255 : (uint8_t)h;
                if ((P <= min_p_disp && r2 >= min_r2_disp) || store_all) {
                    // the term's name: " " SNP term name, or AL name ":" SNP term name for a
                    // covariate term (src/AIOwrapper.cpp:1497-1504)
                    size_t an_len = 0;
                    auto add = [&](const char* s, size_t len) {
                        if (an_len + len + 1 > an.size()) an.resize(an_len + len + 64);
                        memcpy(an.data() + an_len, s, len);
                        an_len += len;
                    };
                    if (h >= l) {
                        add(" ", 1);
                    } else {
                        const auto al = name_of(fl, (size_t)h);
                        add(al.first, (size_t)al.second);
                        add(":", 1);
                    }
                    const size_t snp_g = (size_t)(name_base + snp);
                    const int term = h >= l ? h - l : 0;
                    if (multi_k > 0) {   // src/AIOwrapper.cpp:618-660
                        const std::string mn = multi_name(snp, term);
                        add(mn.data(), mn.size());
                    } else {
                        size_t var = snp_g * name_stride + (name_first_only ? 0 : (size_t)term);
                        if (n_inter > 0) {   // src/AIOwrapper.cpp:566-612
                            if (term < n_inter) {
                                const std::string pre = "I" + std::to_string(term + 1) + "x";
                                add(pre.data(), pre.size());
                            }
                            var = snp_g * name_stride;
                        }
                        const auto sn = name_of(fr, var);
                        add(sn.first, (size_t)sn.second);
                    }
                    const auto yn = name_of(fy, (size_t)ytr);
                    const size_t need = (size_t)yn.second + an_len + 512;
                    if (line.size() < need) line.resize(need);
                    // "%s\t%s\t%u\t%.2f\t%.7f\t%.4f\t%.7f\t%.7f\t%.7Le\n" (src/AIOwrapper.cpp:1509-1511)
                    char* o = line.data();
                    memcpy(o, yn.first, (size_t)yn.second);
                    o += yn.second;
                    *o++ = '\t';
                    memcpy(o, an.data(), an_len);
                    o += an_len;
                    *o++ = '\t';
                    o = put_u64(o, nused);
                    *o++ = '\t';
                    o = put_fixed(o, npct, 2);
                    *o++ = '\t';
                    o = put_fixed(o, Bv, 7);
                    *o++ = '\t';
                    o = put_fixed(o, r2, 4);
                    *o++ = '\t';
                    o = put_fixed(o, SE, 7);
                    *o++ = '\t';
                    o = put_fixed(o, T, 7);
                    *o++ = '\t';
                    o = put_sci7(o, P);
                    *o++ = '\n';
                    S.txt.append(line.data(), (size_t)(o - line.data()));
                    ++S.rows;
                }
                if (dbin) {
                    if (disp_cov && !store_all) put<uint8_t>(S.bin, al_idx);
                    if (!store_all) put<uint16_t>(S.bin, (uint16_t)ar_idx);
                    put<float>(S.bin, Bv);
                    put<float>(S.bin, SE);
                }
            }
        }
    }

    // Format a batch on all host threads (contiguous ranges of its write order, concatenated in
    // order: the bytes of a sequential pass) and write it.
    void write_batch(const RowBatch& B) {
        const int64_t total = (int64_t)B.order.size();
        if (total == 0) return;
        const int parts = (int)std::max<int64_t>(1, std::min<int64_t>(host_threads(), total / 4096));
        std::vector<Segment> seg((size_t)parts);
        parallel_parts(parts, [&](int i) {
            format_range(B, total * i / parts, total * (i + 1) / parts, seg[(size_t)i]);
        });
        for (const Segment& s : seg) {
            total_sig += s.sig;
            rows_written += s.rows;
        }
        put_segments(dis, seg, &Segment::txt);
        if (dbin) put_segments(dbin, seg, &Segment::bin);
    }

    // The segments' bytes at the file's current position, in order: written by several threads at
    // their offsets (pwrite), the file position then moved past them.
    void put_segments(FILE* f, const std::vector<Segment>& seg, std::string Segment::*part) {
        std::vector<off_t> off(seg.size() + 1, 0);
        for (size_t i = 0; i < seg.size(); ++i) off[i + 1] = off[i] + (off_t)(seg[i].*part).size();
        if (off.back() == 0) return;
        fflush(f);
        const off_t base = ftello(f);
        const int fd = fileno(f);
        std::atomic<bool> ok{base >= 0};
        parallel_parts((int)seg.size(), [&](int i) {
            const std::string& b = seg[(size_t)i].*part;
            size_t done = 0;
            while (done < b.size() && ok.load(std::memory_order_relaxed)) {
                const ssize_t w = pwrite(fd, b.data() + done, b.size() - done, base + off[(size_t)i] + (off_t)done);
                if (w < 0 && errno == EINTR) continue;
                if (w <= 0) ok = false;
                else done += (size_t)w;
            }
        });
        if (!ok || fseeko(f, base + off.back(), SEEK_SET) != 0) write_failed = true;
    }

    // Write a batch in the background (after the previous one), so that the next engine call
    // runs meanwhile.
    void submit(RowBatch&& B) {
        finish();
        auto hold = std::make_shared<RowBatch>(std::move(B));
        pending = std::async(std::launch::async, [this, hold] {
            OA_TRACE("write outputs");
            try {
                write_batch(*hold);
            } catch (...) {   // out of host memory for the formatted text: an output error, not a crash
                write_failed = true;
            }
        });
    }
    void finish() {
        if (pending.valid()) pending.get();
    }
    // File SNP (shard-local) and interaction column of a (SNP, column) pair of -w: blocks of
    // multi_fmb file SNPs, each listed once per column (src/AIOwrapper.cpp:441-452, 1208-1241).
    void multi_pair(int v, int& file_snp, int& col) const {
        const int mbv = multi_fmb * multi_k;
        const int b = v / mbv, rem = v - b * mbv;
        const int fb = std::min(multi_fmb, multi_m - b * multi_fmb);
        col = rem / fb;
        file_snp = b * multi_fmb + rem % fb;
    }
    std::string multi_name(int v, int term) const {
        int i, col;
        multi_pair(v, i, col);
        return "I" + std::to_string(col + 1) + (term == 0 ? "_" : "_o_") +
               fr->var_name((size_t)(name_base + i) * name_stride);
    }
};

// The two host buffers the SNP blocks are read into, page-locked (the engine copies them with
// cudaMemcpyAsync), or plain memory when page-locking fails.  Page-locking a buffer of about 1 GB
// takes most of half a second, so it runs on a background thread: the first buffer while the
// engine is set up, the second while the first block is read and scanned.
struct BlockBuffers {
    float* p[2] = {nullptr, nullptr};
    bool locked[2] = {false, false};
    std::shared_future<void> ready[2];
    void alloc(int b, int device, size_t floats) {
        if (cudaSetDevice(device) != cudaSuccess) cudaGetLastError();
        locked[b] = cudaMallocHost(&p[b], sizeof(float) * floats) == cudaSuccess;
        if (!locked[b]) {
            cudaGetLastError();
            p[b] = static_cast<float*>(malloc(sizeof(float) * floats));
        }
    }
    void start(int device, size_t floats) {
        ready[0] = std::async(std::launch::async, [this, device, floats] { alloc(0, device, floats); }).share();
        std::shared_future<void> first = ready[0];
        ready[1] = std::async(std::launch::async, [this, device, floats, first] {
                       first.wait();
                       alloc(1, device, floats);
                   }).share();
    }
    // buffer b, once it exists (null: out of memory)
    float* get(int b) {
        if (ready[b].valid()) ready[b].wait();
        return p[b];
    }
    ~BlockBuffers() {
        for (int b = 0; b < 2; ++b) {
            get(b);
            if (locked[b]) cudaFreeHost(p[b]);
            else free(p[b]);
        }
    }
};

// One engine call of -w: the call's cnt file SNPs (starting at shard SNP s0, a multiple of the
// reference's file block) go to the device once, then one scan per interaction column h with the
// columns [I_h x, x]; the stored rows of all columns are merged into the reference's order (block
// of file SNPs -> trait -> column -> SNP, src/AIOwrapper.cpp:1208-1241) and written.
oa_status multi_call(oa_engine* eng, const float* xr_pinned, float* xr_dev, int cnt, int s0, int file_r, int n,
                     const std::vector<float>& inter, Writer& W, int trait_base, int64_t& tests, int64_t& singular,
                     uint64_t& sig_cov) {
    if (cudaMemcpy(xr_dev, xr_pinned, sizeof(float) * (size_t)cnt * file_r * n, cudaMemcpyHostToDevice) !=
        cudaSuccess) {
        herr("copy of a SNP block: %s", cudaGetErrorString(cudaGetLastError()));
        return OA_ERR_CUDA;
    }
    const int k = W.multi_k, fmb = W.multi_fmb, p = W.p;
    struct Row {
        int32_t trait, pair;
        float r2;
        int32_t n_used;
        uint32_t mask;
        size_t coef;   // offset into the coefficient arrays
    };
    std::vector<Row> rows;
    std::vector<float> cb, cs, ct;
    for (int h = 0; h < k; ++h) {
        oa_status st = oa_set_interactions(eng, inter.data() + (size_t)h * n, 1, 1);
        if (st != OA_OK) return st;
        oa_rows rr{};
        st = oa_run_snps_device(eng, xr_dev, cnt, 1, &rr);
        if (st != OA_OK) return st;
        tests += rr.tests;
        singular += rr.singular;
        sig_cov += (uint64_t)rr.sig_cov_unrowed;
        for (int64_t q = 0; q < rr.count; ++q) {
            const int s = s0 + rr.snp[q];           // shard-local file SNP
            const int b = s / fmb;
            const int fb = std::min(fmb, W.multi_m - b * fmb);
            const int pair = b * fmb * k + h * fb + (s - b * fmb);
            rows.push_back(Row{rr.trait[q], pair, rr.r2[q], rr.n_used[q], rr.coef_mask[q], cb.size()});
            cb.insert(cb.end(), rr.coef_b + (size_t)q * p, rr.coef_b + (size_t)(q + 1) * p);
            cs.insert(cs.end(), rr.coef_se + (size_t)q * p, rr.coef_se + (size_t)(q + 1) * p);
            ct.insert(ct.end(), rr.coef_t + (size_t)q * p, rr.coef_t + (size_t)(q + 1) * p);
        }
    }
    const int mbv = fmb * k;
    std::sort(rows.begin(), rows.end(), [mbv](const Row& a, const Row& b) {
        const int ba = a.pair / mbv, bb = b.pair / mbv;
        if (ba != bb) return ba < bb;
        if (a.trait != b.trait) return a.trait < b.trait;
        return a.pair < b.pair;
    });
    const size_t cnt_rows = rows.size();
    RowBatch g;
    g.p = p;
    g.trait.resize(cnt_rows);
    g.snp.resize(cnt_rows);
    g.n_used.resize(cnt_rows);
    g.r2.resize(cnt_rows);
    g.mask.resize(cnt_rows);
    g.b.resize(cnt_rows * p);
    g.se.resize(cnt_rows * p);
    g.t.resize(cnt_rows * p);
    for (size_t q = 0; q < cnt_rows; ++q) {
        const Row& x = rows[q];
        g.trait[q] = x.trait;
        g.snp[q] = x.pair;
        g.n_used[q] = x.n_used;
        g.r2[q] = x.r2;
        g.mask[q] = x.mask;
        std::copy(cb.begin() + x.coef, cb.begin() + x.coef + p, g.b.begin() + q * p);
        std::copy(cs.begin() + x.coef, cs.begin() + x.coef + p, g.se.begin() + q * p);
        std::copy(ct.begin() + x.coef, ct.begin() + x.coef + p, g.t.begin() + q * p);
    }
    // the call covers whole reference blocks s0 / fmb .. (s0 + cnt - 1) / fmb; the sorted rows hold
    // them one after the other
    const int b_first = s0 / fmb, b_last = (s0 + cnt - 1) / fmb;
    g.order.resize(cnt_rows);
    for (size_t q = 0; q < cnt_rows; ++q) g.order[q] = (int64_t)q;
    g.blk_off.assign((size_t)(b_last - b_first) + 2, 0);
    for (size_t q = 0; q < cnt_rows; ++q) ++g.blk_off[(size_t)(g.snp[q] / mbv - b_first) + 1];
    for (int b = b_first; b <= b_last; ++b) {
        g.blk_off[(size_t)(b - b_first) + 1] += g.blk_off[(size_t)(b - b_first)];
        g.blk_trait_base.push_back(trait_base);
        g.blk_ar_off.push_back(b * mbv);
    }
    W.submit(std::move(g));
    return OA_OK;
}

}  // namespace

extern "C" {

long double oa_pvalue(float t) { return pvalue_ld(t); }

oa_status oa_shard_range(int32_t m, int32_t shard, int32_t shards, int32_t* first, int32_t* count) {
    if (!first || !count || m < 0 || shards < 1 || shard < 0 || shard >= shards) {
        herr("shard %d of %d", shard, shards);
        return OA_ERR_ARG;
    }
    *first = 0;
    *count = m;
    if (shards > 1 && m >= shards) {
        const int m_sh = m / shards;
        *first = m_sh * shard;
        *count = shard == shards - 1 ? m_sh + (m - shards * m_sh) : m_sh;
    }
    return OA_OK;
}

float oa_t_threshold(float p) {
    // src/Utility.cpp:244-250: erf_inv(1 - p) * sqrt(2), evaluated in long double
    return (float)(erf_inv_ld((long double)(1.0 - (double)p)) * sqrt(2.0));
}

void oa_default_settings(oa_settings* s) {
    memset(s, 0, sizeof *s);
    s->r = 1;
    s->min_r2_store = 0.00001f;
    s->min_r2_disp = 0.000001f;
    s->min_p_store = 0.1f;
    s->min_p_disp = 0.05f;
    s->precision = OA_PLAIN_FP32;
    s->device = 0;
    s->shard = 0;
    s->shards = 1;
}

oa_status oa_solve(const oa_settings* S, oa_outputs* out) {
    OA_TRACE("oa_solve");
    if (!S || !out) {
        herr("null argument");
        return OA_ERR_ARG;
    }
    memset(out, 0, sizeof *out);
    const auto t_start = std::chrono::steady_clock::now();
    // OA_TIMING: host phase times on stderr at the end of the run
    double tm_files = 0, tm_create = 0, tm_setup = 0, tm_pin = 0, tm_traits = 0, tm_read = 0, tm_run = 0, tm_submit = 0, tm_finish = 0;
    auto t_mark = t_start;
    auto lap = [&t_mark](double& acc) {
        const auto now = std::chrono::steady_clock::now();
        acc += std::chrono::duration<double>(now - t_mark).count();
        t_mark = now;
    };
    const bool verbose = S->verbose != 0;
    // threshold coupling (src/Algorithm.cpp:338-342)
    float min_r2_store = S->min_r2_store, min_p_store = S->min_p_store;
    if (S->min_r2_disp < min_r2_store || S->store_bin) min_r2_store = S->min_r2_disp;
    if (S->min_p_disp > min_p_store || S->store_bin) min_p_store = S->min_p_disp;
    const float min_t_store = oa_t_threshold(min_p_store);

    const std::string fxl = S->fname_xl ? S->fname_xl : "", fxr = S->fname_xr ? S->fname_xr : "",
                      fy = S->fname_y ? S->fname_y : "", fout = S->fname_out ? S->fname_out : "";
    Fvi FL, FR, FY;
    if (!read_fvi(fy + ".fvi", FY) || !read_fvi(fxl + ".fvi", FL) || !read_fvi(fxr + ".fvi", FR)) return OA_ERR_IO;
    if (!check_fvd(fy, FY) || !check_fvd(fxl, FL) || !check_fvd(fxr, FR)) return OA_ERR_IO;
    if (FL.nobs != FR.nobs || FR.nobs != FY.nobs) {
        // the reference only stops when all three differ (src/AIOwrapper.cpp:72-85); any mismatch is an error here
        herr("The number of elements/individuals from the input files do not coincide with each other! %s:%u %s:%u "
             "%s:%u",
             fy.c_str(), FY.nobs, fxl.c_str(), FL.nobs, fxr.c_str(), FR.nobs);
        return OA_ERR_IO;
    }
    // file columns per SNP (-n) and the model's columns per SNP (src/AIOwrapper.cpp:257-340)
    const int file_r = std::max(1, S->r);
    const int fileN = (int)FL.nobs;
    if (FR.nvar % file_r != 0) {
        herr("Number of elements in %s.fvi:%u is not consistent with the value of --ngpred (-n)%d provided",
             fxr.c_str(), FR.nvar, file_r);
        return OA_ERR_IO;
    }
    float model_w[OA_MODEL_MAX_COLS] = {};
    bool combine = false;
    int r = file_r;
    if (S->dosage_model < 0 || S->dosage_model > 5) {
        herr("Requested dosages model wihtout a valid model!");
        return OA_ERR_ARG;
    }
    if (S->dosage_model >= 1 && S->dosage_model <= 3) {
        static const char* kName[] = {"", "Additive", "Dominant", "Recessive"};
        static const float kW[4][3] = {{0, 0, 0}, {2, 1, 0}, {1, 1, 0}, {1, 0, 0}};
        if (file_r != 2 && file_r != 3) {
            herr("The amount of columns per Independent Variable (--ngpred) is not 2 or 3 for a valid %s Model!",
                 kName[S->dosage_model]);
            return OA_ERR_ARG;
        }
        for (int c = 0; c < file_r; ++c) model_w[c] = kW[S->dosage_model][c];
        combine = true;
        r = 1;
    } else if (S->dosage_model == 4 || S->dosage_model == 5) {
        if (file_r > OA_MODEL_MAX_COLS) {
            herr("a dosage model takes at most %d columns per SNP", OA_MODEL_MAX_COLS);
            return OA_ERR_UNSUPPORTED;
        }
        FILE* ff = S->fname_factors ? fopen(S->fname_factors, "r") : nullptr;
        if (!ff) {
            herr("Error reading dosages file.");
            return OA_ERR_IO;
        }
        int got = 0;
        while (got < file_r && fscanf(ff, "%f", &model_w[got]) == 1) ++got;
        fclose(ff);
        if (got != file_r) {
            herr("The number of factors for the dosage model! does not coincide with the source data #facctors:%d, "
                 "expected:%d",
                 got, file_r);
            return OA_ERR_IO;
        }
        combine = S->dosage_model == 5;
        r = combine ? 1 : file_r;
    }
    const bool model = S->dosage_model != 0;
    // single-set interactions: k columns, each SNP column x -> [I_1 x, ..., I_k x, x] (src/AIOwrapper.cpp:371-480)
    Fvi FI;
    const bool use_inter = S->fname_interactions && S->fname_interactions[0];
    int n_inter = 0;
    if (use_inter) {
        if (r != 1) {
            herr("Cannot use Interactions with --ngpred set to: %d. Required is 1!\nInteractions can be only of the "
                 "form y~cov+V1*X+...+Vi*X, (only with --ngpred=1 or models excluding(--mylinear)) !",
                 file_r);
            return OA_ERR_ARG;
        }
        if (!read_fvi(std::string(S->fname_interactions) + ".fvi", FI) || !check_fvd(S->fname_interactions, FI))
            return OA_ERR_IO;
        if (FI.nobs != FR.nobs) {
            herr("The number of elements/individuals from the input files do not coincide with each other! %s:%u %s:%u",
                 S->fname_interactions, FI.nobs, fxr.c_str(), FR.nobs);
            return OA_ERR_IO;
        }
        n_inter = (int)FI.nvar;
        if (n_inter < 1 || (n_inter + 1 > OA_MAX_R && !S->multi_interactions)) {
            herr("%d interaction columns: this build supports 1..%d", n_inter, OA_MAX_R - 1);
            return OA_ERR_UNSUPPORTED;
        }
        r = n_inter + 1;
    }
    // one analysis per interaction column (-w): k columns, r = 2 ([I_h x, x]) for each
    const bool multi = use_inter && S->multi_interactions;
    if (multi) r = 2;
    const int m_file = (int)(FR.nvar / file_r), t = (int)FY.nvar, l = (int)FL.nvar, p = l + r;
    // SNP shard of this process (the reference's MPI split, src/AIOwrapper.cpp:95-117)
    const int shards = std::max(1, S->shards);
    if (S->shard < 0 || S->shard >= shards) {
        herr("shard %d of %d", S->shard, shards);
        return OA_ERR_ARG;
    }
    int first = 0, m = m_file;
    oa_shard_range(m_file, S->shard, shards, &first, &m);
    const std::string fout_eff =
        (shards > 1 && m_file >= shards) ? fout + "_mpi" + std::to_string(S->shard + 1) + "_" : fout;
    if (l < 1 || l > OA_MAX_L) {
        herr("%d covariates: this build supports 1..%d", l, OA_MAX_L);
        return OA_ERR_UNSUPPORTED;
    }
    if (r > OA_MAX_R) {
        herr("%d columns per SNP: this build supports 1..%d", r, OA_MAX_R);
        return OA_ERR_UNSUPPORTED;
    }
    // ID order checks (warnings only, as in the reference, src/AIOwrapper.cpp:148-191)
    for (int i = 0; i < fileN; ++i) {
        const std::string a = FY.obs_name(i), b = FL.obs_name(i), c = FR.obs_name(i);
        if (a != b || a != c) {
            if (verbose)
                printf("Warning, ID names between input files do not coincide! The files must have the same "
                       "meaningful order\n");
            break;
        }
    }
    // row selection: exclusion list, then rows with a NaN covariate (src/AIOwrapper.cpp:229-253, 1947-1991)
    std::vector<char> keep(fileN, 1);
    int excl = 0;
    if (S->fname_exclude && S->fname_exclude[0])
        if (!exclusion_rows(S->fname_exclude, fileN, keep, excl, verbose)) return OA_ERR_IO;
    std::vector<float> xl_all((size_t)fileN * l);
    {
        FILE* fp = fopen((fxl + ".fvd").c_str(), "rb");
        if (!fp) {
            herr("Error Reading File %s", fxl.c_str());
            return OA_ERR_IO;
        }
        std::vector<double> dbl;
        const bool got = read_values(fp, FL.elem_bytes(), 0, xl_all.size(), xl_all.data(), dbl);
        fclose(fp);
        if (!got) {
            herr("%s.fvd: short read", fxl.c_str());
            return OA_ERR_IO;
        }
    }
    int almiss = 0;
    for (int h = 0; h < l; ++h)
        for (int i = 0; i < fileN; ++i)
            if (std::isnan(xl_all[(size_t)h * fileN + i]) && keep[i]) {
                keep[i] = 0;
                ++almiss;
            }
    if (almiss > 0 && verbose) printf("Excluding %d from covariate missings\n", almiss);
    std::vector<float> inter_all;
    int intermiss = 0;
    if (use_inter) {
        for (int i = 0; i < fileN; ++i)
            if (FI.obs_name(i) != FR.obs_name(i)) {
                if (verbose)
                    printf("Warning, ID names between -g file and interactions file do not coincide! The files must "
                           "have the same meaningful order!\n");
                break;
            }
        inter_all.resize((size_t)n_inter * fileN);
        FILE* fp = fopen((std::string(S->fname_interactions) + ".fvd").c_str(), "rb");
        std::vector<double> dbl;
        const bool got = fp && read_values(fp, FI.elem_bytes(), 0, inter_all.size(), inter_all.data(), dbl);
        if (fp) fclose(fp);
        if (!got) {
            herr("Error opening Interactions File %s", S->fname_interactions);
            return OA_ERR_IO;
        }
        for (int h = 0; h < n_inter; ++h)   // rows with a NaN interaction value (src/AIOwrapper.cpp:519-533)
            for (int i = 0; i < fileN; ++i)
                if (std::isnan(inter_all[(size_t)h * fileN + i]) && keep[i]) {
                    keep[i] = 0;
                    ++intermiss;
                }
        if (intermiss > 0 && verbose) printf("Excluding %d from Interaction missings\n", intermiss);
    }
    const Runs runs = keep_runs(keep);
    const int n = fileN - excl - almiss - intermiss;
    if (p >= n) {
        herr("Error! The amount of unknows (individuals|elements) must be greater than total of variables "
             "(#covariates+#ind.variables)!");
        return OA_ERR_ARG;
    }
    if ((l > 255 || p > 255 || n > 65535) && verbose)
        printf("Warning, output binary format does not yet support current problem sizes for the provided p, l, r "
               "and n.\n");
    std::vector<float> XL((size_t)n * l);
    for (int h = 0; h < l; ++h) {
        size_t pos = 0;
        for (const auto& run : runs) {
            memcpy(&XL[(size_t)h * n + pos], &xl_all[(size_t)h * fileN + run.first], sizeof(float) * run.second);
            pos += run.second;
        }
    }
    xl_all.clear();
    xl_all.shrink_to_fit();

    // outputs
    Writer W;
    W.store_bin = S->store_bin;
    W.store_all = S->store_all;
    W.disp_cov = S->disp_cov;
    W.min_p_disp = (long double)S->min_p_disp;
    W.min_r2_disp = S->min_r2_disp;
    W.l = l;
    W.r = r;
    W.p = p;
    W.real_n = fileN;
    W.fy = &FY;
    W.fl = &FL;
    W.fr = &FR;
    W.name_base = first;
    W.name_stride = file_r;
    W.name_first_only = combine;
    W.n_inter = multi ? 0 : n_inter;
    // -w: reference blocks of fmb file SNPs x k columns (src/AIOwrapper.cpp:441-452)
    const int multi_fmb = multi ? std::max(1, std::min(m, 500) / n_inter) : 1;
    if (multi) {
        W.multi_k = n_inter;
        W.multi_fmb = multi_fmb;
        W.multi_m = m;
    }
    const int m_out = multi ? m * n_inter : m;   // SNPs of the outputs: (SNP, column) pairs with -w
    W.dis = fopen((fout_eff + "_dis.txt").c_str(), "wb");
    if (!W.dis) {
        herr("Error Creating File %s_dis.txt", fout_eff.c_str());
        return OA_ERR_IO;
    }
    fputs("Phe\tSNP\tn\tnPct\tB\tR2\tSE\tT\tP\n", W.dis);
    if (S->store_bin) {
        // _sto.ibin (src/AIOwrapper.cpp:679-733)
        FILE* fi = fopen((fout_eff + "_sto.ibin").c_str(), "wb");
        if (!fi) {
            herr("Error Creating File: %s_sto.ibin", fout_eff.c_str());
            fclose(W.dis);
            return OA_ERR_IO;
        }
        const int32_t hdr[6] = {n, l, r, t, m_out, (int32_t)FR.namelength};
        fwrite(hdr, 4, 6, fi);
        const uint8_t flags[2] = {(uint8_t)(S->disp_cov ? 1 : 0), (uint8_t)(S->store_all ? 1 : 0)};
        fwrite(flags, 1, 2, fi);
        fwrite(FL.raw((size_t)FL.nobs + 1), 1, (size_t)FL.namelength * (l - 1), fi);
        if (multi) {
            // r names per (SNP, column) pair in output order, as the text output names them.  The
            // reference writes fileR * m file names here with m already multiplied by the column
            // count (src/AIOwrapper.cpp:444, 722-728), i.e. past the end of its name table; the
            // list written here matches the header's r * m instead.
            std::vector<char> nm((size_t)FR.namelength);
            for (int v = 0; v < m_out; ++v)
                for (int term = 0; term < 2; ++term) {
                    const std::string a = W.multi_name(v, term);
                    std::fill(nm.begin(), nm.end(), 0);
                    memcpy(nm.data(), a.data(), std::min(a.size(), nm.size() - 1));
                    fwrite(nm.data(), 1, nm.size(), fi);
                }
        } else if (combine) {   // one name per SNP: its first file column (src/AIOwrapper.cpp:711-721)
            for (int i = 0; i < m; ++i)
                fwrite(FR.raw((size_t)FR.nobs + (size_t)(first + i) * file_r), 1, (size_t)FR.namelength, fi);
        } else {
            // the file's names, fileR per SNP, also with interactions (src/AIOwrapper.cpp:722-728)
            fwrite(FR.raw((size_t)FR.nobs + (size_t)first * file_r), 1, (size_t)FR.namelength * file_r * m, fi);
        }
        fwrite(FY.raw(FY.nobs), 1, (size_t)FY.namelength * t, fi);
        fclose(fi);
        W.dbin = fopen((fout_eff + "_sto.dbin").c_str(), "wb");
        if (!W.dbin) {
            herr("Error Creating File %s_sto.dbin", fout_eff.c_str());
            fclose(W.dis);
            return OA_ERR_IO;
        }
    }

    // engine: one trait block of the reference's size at a time (tb = min(t, 1000))
    const int tb = std::min(t, 1000);
    const int mb_ref = multi ? multi_fmb * n_inter : std::min(m, 500);
    W.mb_ref = mb_ref;
    // SNPs per engine call: a multiple of the reference block (of its file SNPs with -w), about
    // 1 GB of genotypes
    const int mb_file = multi ? multi_fmb : mb_ref;
    int call_snps = (int)std::max<int64_t>(1, (int64_t)(1u << 28) / ((int64_t)n * file_r));
    call_snps = std::max(mb_file, call_snps / mb_file * mb_file);
    call_snps = std::min(call_snps, m);
    BlockBuffers pins;
    pins.start(S->device, (size_t)call_snps * file_r * n);
    oa_config cfg{};
    cfg.n = n;
    cfg.l = l;
    cfg.r = r;
    cfg.max_traits = tb;
    cfg.max_snps = call_snps;
    cfg.precision = S->precision;
    cfg.device = S->device;
    cfg.disp_cov = S->disp_cov;
    cfg.store_all = S->store_all;
    cfg.quirk_r2 = S->quirk_r2;
    cfg.min_r2_store = min_r2_store;
    cfg.min_t_store = min_t_store;
    cfg.min_p_disp = S->min_p_disp;
    cfg.real_n = fileN;
    oa_engine* eng = nullptr;
    lap(tm_files);
    oa_status st = oa_engine_create(&cfg, &eng);
    lap(tm_create);
    if (st != OA_OK) {
        herr("%s", oa_last_error());
        fclose(W.dis);
        if (W.dbin) fclose(W.dbin);
        return st;
    }
    auto fail = [&](oa_status s) {
        herr("%s", oa_last_error());
        oa_engine_destroy(eng);
        W.finish();
        fclose(W.dis);
        if (W.dbin) fclose(W.dbin);
        return s;
    };
    st = oa_set_covariates(eng, XL.data());
    if (st != OA_OK) return fail(st);
    std::vector<float> inter_kept;
    if (use_inter) {   // the kept rows of each interaction column
        inter_kept.resize((size_t)n_inter * n);
        for (int h = 0; h < n_inter; ++h) {
            size_t pos = 0;
            for (const auto& run : runs) {
                memcpy(&inter_kept[(size_t)h * n + pos], &inter_all[(size_t)h * fileN + run.first],
                       sizeof(float) * run.second);
                pos += run.second;
            }
        }
        // the interactions first: a combined dosage model then keeps them (r = columns + 1)
        st = multi ? oa_set_interactions(eng, inter_kept.data(), 1, 1)
                   : oa_set_interactions(eng, inter_kept.data(), n_inter, 1);
        if (st != OA_OK) return fail(st);
    }
    if (model) {
        st = oa_set_column_model(eng, file_r, model_w, combine ? 1 : 0);
        if (st != OA_OK) return fail(st);
    }
    // -w: each call's SNP block is copied to the device once and scanned once per interaction column
    float* xr_dev = nullptr;
    if (multi && (cudaSetDevice(S->device) != cudaSuccess ||
                  cudaMalloc(&xr_dev, sizeof(float) * (size_t)call_snps * file_r * n) != cudaSuccess)) {
        cudaGetLastError();
        herr("device buffer for the SNP blocks of -w: out of memory");
        oa_engine_destroy(eng);
        fclose(W.dis);
        if (W.dbin) fclose(W.dbin);
        return OA_ERR_NOMEM;
    }

    FILE* fr = fopen((fxr + ".fvd").c_str(), "rb");
    FILE* fyd = fopen((fy + ".fvd").c_str(), "rb");
    if (!fr || !fyd) {
        if (fr) fclose(fr);
        if (fyd) fclose(fyd);
        herr("Error opening File %s", !fr ? fxr.c_str() : fy.c_str());
        oa_engine_destroy(eng);
        fclose(W.dis);
        if (W.dbin) fclose(W.dbin);
        return OA_ERR_IO;
    }
    lap(tm_setup);
    // pinned double buffers for the SNP blocks (copied with cudaMemcpyAsync by the engine)
    if (!pins.get(0)) {
        fclose(fr);
        fclose(fyd);
        if (xr_dev) cudaFree(xr_dev);
        herr("host buffers for the SNP blocks: out of memory");
        oa_engine_destroy(eng);
        fclose(W.dis);
        if (W.dbin) fclose(W.dbin);
        return OA_ERR_NOMEM;
    }
    std::atomic<bool> pin_failed{false};
    lap(tm_pin);
    std::vector<float> scratch[2];
    std::vector<double> dscratch[2], ydbl;
    std::vector<float> Yblk, yscratch;
    int64_t tests = 0, singular = 0;
    uint64_t sig_cov = 0;
    bool io_ok = true;
    const int ncalls = (m + call_snps - 1) / call_snps;
    for (int y0 = 0; y0 < t && st == OA_OK && io_ok; y0 += tb) {
        const int tcur = std::min(tb, t - y0);
        Yblk.resize((size_t)tcur * n);
        if (!read_columns(fyd, FY.elem_bytes(), fileN, y0, tcur, runs, n, Yblk.data(), yscratch, ydbl)) {
            herr("Error reading file %s.fvd", fy.c_str());
            io_ok = false;
            break;
        }
        st = oa_set_traits(eng, Yblk.data(), tcur);
        lap(tm_traits);
        if (st != OA_OK) break;
        auto read_call = [&](int c, int b) {
            OA_TRACE("read SNP block (.fvd)");
            float* dst = pins.get(b);
            if (!dst) {
                pin_failed = true;
                return false;
            }
            const int s0 = c * call_snps, cnt = std::min(call_snps, m - s0);
            return read_columns(fr, FR.elem_bytes(), fileN, (size_t)(first + s0) * file_r, (size_t)cnt * file_r, runs,
                                n, dst, scratch[b], dscratch[b]);
        };
        std::future<bool> next = std::async(std::launch::async, read_call, 0, 0);
        for (int c = 0; c < ncalls; ++c) {
            const bool read_ok = next.get();
            lap(tm_read);
            if (!read_ok) {
                if (pin_failed) herr("host buffers for the SNP blocks: out of memory");
                else herr("Error reading AR File %s.fvd", fxr.c_str());
                io_ok = false;
                break;
            }
            const int b = c & 1;
            const int s0 = c * call_snps, cnt = std::min(call_snps, m - s0);
            if (c + 1 < ncalls) next = std::async(std::launch::async, read_call, c + 1, b ^ 1);
            if (multi) {
                st = multi_call(eng, pins.p[b], xr_dev, cnt, s0, file_r, n, inter_kept, W, y0, tests, singular, sig_cov);
                if (st != OA_OK) {
                    if (c + 1 < ncalls) next.wait();
                    break;
                }
                if (verbose) {
                    putchar('*');
                    fflush(stdout);
                }
                continue;
            }
            oa_rows rows{};
            st = oa_run_snps(eng, pins.p[b], cnt, &rows);
            lap(tm_run);
            if (st != OA_OK) {
                if (c + 1 < ncalls) next.wait();
                break;
            }
            tests += rows.tests;
            singular += rows.singular;
            sig_cov += (uint64_t)rows.sig_cov_unrowed;
            // the rows go to the writer, split into the reference's SNP blocks; it formats and writes
            // them while the next call runs
            W.submit(RowBatch::from_call(rows, p, s0, cnt, mb_ref, y0));
            lap(tm_submit);
            if (verbose) {
                putchar('*');
                fflush(stdout);
            }
        }
    }
    fclose(fr);
    fclose(fyd);
    if (xr_dev) cudaFree(xr_dev);
    W.finish();
    fclose(W.dis);
    if (W.dbin) fclose(W.dbin);
    oa_engine_destroy(eng);
    lap(tm_finish);
    if (getenv("OA_TIMING"))
        fprintf(stderr,
                "[oa timing] input files %.3f s, engine creation %.3f s, covariates and models %.3f s, pinned buffers %.3f s, traits %.3f s, waiting for reads %.3f s, engine "
                "calls %.3f s, handing rows to the writer %.3f s, last writes and release %.3f s (%d host threads)\n",
                tm_files, tm_create, tm_setup, tm_pin, tm_traits, tm_read, tm_run, tm_submit, tm_finish, host_threads());
    if (!io_ok) return OA_ERR_IO;
    if (st != OA_OK) {
        if (h_err.empty()) herr("%s", oa_last_error());
        return st;
    }
    if (W.write_failed) {
        herr("Error writing the output files %s*", fout_eff.c_str());
        return OA_ERR_IO;
    }
    out->total_sig_results = W.total_sig + sig_cov;
    out->tests = tests;
    out->singular = singular;
    out->rows_written = W.rows_written;
    out->duration_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    return OA_OK;
}

// ---------------------------------------------------------------------------
// CLI (src/main.cpp:102-437)
// ---------------------------------------------------------------------------
static const char* kHelp =
    "usage: omicabelnomm -c <path/fname> --geno <path/fname> -p <path/fname> -o <path/fname> -x <path/fname> "
    "-n <#SNPcols> -t <#CPUs> -d <0.0~1.0> -r <-10.0~1.0> -b -s <0.0~1.0> -e <-10.0~1.0> -i -f\n"
    "  -p --phe     phenotypes (.fvi/.fvd)      -g --geno   genotypes\n"
    "  -c --cov     covariates                  -o --out    output prefix\n"
    "  -n --ngpred  columns per SNP             -t --thr    host threads (accepted, unused)\n"
    "  -x --excl    exclusion list              -b --stobin also write _sto.ibin/_sto.dbin\n"
    "  -d --pdisp   display P threshold         -s --psto   store P threshold\n"
    "  -r --rdisp   display R2 threshold        -e --rsto   store R2 threshold\n"
    "  -i --fdcov   include covariate terms      -f --fdgen  store every result\n"
    "  --precision plain|mixed   --device <ordinal>   --quirk-r2\n";

static std::string strip_ext(const char* a) {
    std::string s(a);
    const size_t pos = s.find_last_of('.');
    if (pos != std::string::npos) s = s.substr(0, pos);
    return s;
}

int oa_cli_main(int argc, char** argv) {
    oa_settings S;
    oa_default_settings(&S);
    S.verbose = 1;
    std::string fy, fr, fl, fo, fx, ffac, finter;
    bool phe = false, snp = false, cov = false, bout = false, shard_set = false, device_set = false;
    static struct option opts[] = {{"phe", required_argument, 0, 'p'},
                                   {"geno", required_argument, 0, 'g'},
                                   {"cov", required_argument, 0, 'c'},
                                   {"out", required_argument, 0, 'o'},
                                   {"ngpred", required_argument, 0, 'n'},
                                   {"thr", required_argument, 0, 't'},
                                   {"mem", required_argument, 0, 'm'},
                                   {"excl", required_argument, 0, 'x'},
                                   {"stobin", no_argument, 0, 'b'},
                                   {"pdisp", required_argument, 0, 'd'},
                                   {"psto", required_argument, 0, 's'},
                                   {"rdisp", required_argument, 0, 'r'},
                                   {"rsto", required_argument, 0, 'e'},
                                   {"fdcov", no_argument, 0, 'i'},
                                   {"fdgen", no_argument, 0, 'f'},
                                   {"additive", no_argument, 0, 'j'},
                                   {"dominant", no_argument, 0, 'k'},
                                   {"recessive", no_argument, 0, 'l'},
                                   {"mylinear", required_argument, 0, 'z'},
                                   {"myaddit", required_argument, 0, 'y'},
                                   {"simpleinter", required_argument, 0, 'v'},
                                   {"multinter", required_argument, 0, 'w'},
                                   {"keepinter", no_argument, 0, 'u'},
                                   {"help", no_argument, 0, 'h'},
                                   {"precision", required_argument, 0, 1000},
                                   {"device", required_argument, 0, 1001},
                                   {"quirk-r2", no_argument, 0, 1002},
                                   {"shard", required_argument, 0, 1003},
                                   {0, 0, 0, 0}};
    optind = 1;
    int c, idx = 0;
    while ((c = getopt_long(argc, argv, "c:p:g:o:n:t:m:x:d:s:r:e:z:y:v:w:ufibhjkl", opts, &idx)) != -1) {
        switch (c) {
            case 'p': phe = !phe; fy = strip_ext(optarg); printf("-p Reading phenotypes from file %s\n", optarg); break;
            case 'g': snp = !snp; fr = strip_ext(optarg); printf("-g Reading with genotype data from file %s\n", optarg); break;
            case 'c': cov = !cov; fl = strip_ext(optarg); printf("-c Reading covariates from file %s\n", optarg); break;
            case 'o': bout = !bout; fo = strip_ext(optarg); printf("-o Writing output files to %s\n", optarg); break;
            case 'n': S.r = std::max(atoi(optarg), 1); printf("-n Using columns per snp as %d\n", S.r); break;
            case 't': break;   // host threads: the GPU engine does not use them
            case 'm': break;   // --mem: accepted (the reference has no handler for it)
            case 'x': fx = optarg; printf("-x Excluding ids on %s\n", optarg); break;
            case 'd': S.min_p_disp = (float)fabs(atof(optarg)); break;
            case 's': S.min_p_store = (float)fabs(atof(optarg)); break;
            case 'r': S.min_r2_disp = (float)atof(optarg); break;
            case 'e': S.min_r2_store = (float)atof(optarg); break;
            case 'i': S.disp_cov = 1; break;
            case 'f': S.store_all = 1; break;
            case 'b': S.store_bin = 1; break;
            case 'j':
                S.dosage_model = 1;
                printf("-j Using Additive Model with (2*AA, 1*AB, 0*BB) effects\n");
                break;
            case 'k':
                S.dosage_model = 2;
                printf("-k Using Dominant Model with (1*AA, 1*AB, 0*BB) effects\n");
                break;
            case 'l':
                S.dosage_model = 3;
                printf("-j Using Recessive Model with (1*AA, 0*AB, 0*BB) effects\n");
                break;
            case 'z':
                S.dosage_model = 4;
                ffac = optarg;
                printf("-z Using Custom Linear Model with parameters read from the file %s\n", optarg);
                break;
            case 'y':
                S.dosage_model = 5;
                ffac = optarg;
                printf("-z Using Custom Additive Model with parameters read from the file %s\n", optarg);
                break;
            case 'v':
                finter = optarg;
                S.multi_interactions = 0;
                printf("-v File containing single interactions %s\n", optarg);
                break;
            case 'u':
                printf("-u Keeping independent variable for interaction analysis \n");
                break;
            case 'w':
                finter = optarg;
                S.multi_interactions = 1;
                printf("-w File containing multiple interactions %s\n", optarg);
                break;
            case 'h': fputs(kHelp, stdout); return 1;
            case 1000:
                if (!strcmp(optarg, "plain")) S.precision = OA_PLAIN_FP32;
                else if (!strcmp(optarg, "mixed")) S.precision = OA_MIXED_BF16X3;
                else { printf("--precision must be plain or mixed\n"); return 1; }
                break;
            case 1001: S.device = atoi(optarg); device_set = true; break;
            case 1002: S.quirk_r2 = 1; break;
            case 1003:
                if (sscanf(optarg, "%d/%d", &S.shard, &S.shards) != 2 || S.shards < 1 || S.shard < 0 ||
                    S.shard >= S.shards) {
                    printf("--shard must be k/N with 0 <= k < N\n");
                    return 1;
                }
                shard_set = true;
                break;
            case '?': break;
            default: return 1;
        }
    }
    if (!bout || !phe || !cov || !snp) {
        printf("Missing arguments! p:%d g:%d c:%d o:%d\n", phe, snp, cov, bout);
        return 1;
    }
    // launched as one process per GPU (mpirun or torchrun): shard and device from the launcher
    if (!shard_set) {
        const char* rk = getenv("OMPI_COMM_WORLD_RANK");
        const char* sz = getenv("OMPI_COMM_WORLD_SIZE");
        if (!rk || !sz) {
            rk = getenv("RANK");
            sz = getenv("WORLD_SIZE");
        }
        if (rk && sz && atoi(sz) > 1) {
            S.shard = atoi(rk);
            S.shards = atoi(sz);
        }
    }
    if (!device_set) {
        const char* lr = getenv("OMPI_COMM_WORLD_LOCAL_RANK");
        if (!lr) lr = getenv("LOCAL_RANK");
        if (lr) S.device = atoi(lr);
    }
    S.fname_y = fy.c_str();
    S.fname_xr = fr.c_str();
    S.fname_xl = fl.c_str();
    S.fname_out = fo.c_str();
    S.fname_exclude = fx.empty() ? nullptr : fx.c_str();
    S.fname_factors = ffac.empty() ? nullptr : ffac.c_str();
    S.fname_interactions = finter.empty() ? nullptr : finter.c_str();
    printf("omicabelnomm-b200\n");
    oa_outputs out;
    const oa_status st = oa_solve(&S, &out);
    if (st != OA_OK) {
        printf("\n%s\n", h_err.c_str());
        return 1;
    }
    printf("\nNumber of Significant Results: %llu\n\n", (unsigned long long)out.total_sig_results);
    return 0;
}

}  // extern "C"
