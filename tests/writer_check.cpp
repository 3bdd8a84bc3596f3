// Host-only check of the CLI's output writer (omicabelnomm_b200/csrc/oa_host.cpp), compiled and run
// by tests/test_writer.py without a GPU:
//   1. put_fixed / put_sci7 / put_u64 give printf's characters ("%.Nf" of floats, "%.7Le" of long
//      doubles, "%u") on random bit patterns, typical magnitudes, exact decimal ties, subnormals,
//      -0, NaN and infinities;
//   2. Writer::format_range formats random stored rows exactly as a plain snprintf pass with the
//      reference's row format (src/AIOwrapper.cpp:1497-1511) and its .dbin records
//      (src/AIOwrapper.cpp:1454-1531) would, with and without covariate terms (-i), all rows (-f)
//      and interaction names (-v);
//   3. the bytes do not depend on how many parts the rows are split into, and the files the
//      background writer leaves (parallel positioned writes after a header) hold the same bytes.
//   4. the genotype reader returns the file's values from parallel slices of float and double
//      files, with and without excluded rows, and fails on a block past the end of the file.
// The engine entry points the host file calls are stubbed: nothing here touches a device.
#include "../omicabelnomm_b200/csrc/oa_host.cpp"

#include <random>

extern "C" {
void oa__set_error(const char*) {}
const char* oa_last_error(void) { return ""; }
oa_status oa_engine_destroy(oa_engine*) { return OA_OK; }
oa_status oa_engine_create(const oa_config*, oa_engine**) { return OA_ERR_STATE; }
oa_status oa_set_covariates(oa_engine*, const float*) { return OA_ERR_STATE; }
oa_status oa_set_column_model(oa_engine*, int32_t, const float*, int32_t) { return OA_ERR_STATE; }
oa_status oa_set_traits(oa_engine*, const float*, int32_t) { return OA_ERR_STATE; }
oa_status oa_set_interactions(oa_engine*, const float*, int32_t, int32_t) { return OA_ERR_STATE; }
oa_status oa_run_snps_device(oa_engine*, const float*, int32_t, int32_t, oa_rows*) { return OA_ERR_STATE; }
oa_status oa_run_snps(oa_engine*, const float*, int32_t, oa_rows*) { return OA_ERR_STATE; }
}

namespace {

long failures = 0;

void number_checks(long random_cases) {
    std::mt19937_64 g(7);
    char a[128], b[128];
    auto check = [&](float f, int N) {
        char* e = put_fixed(a, f, N);
        *e = 0;
        snprintf(b, sizeof b, "%.*f", N, (double)f);
        if (strcmp(a, b)) {
            if (failures < 10) printf("put_fixed(%a, %d) = %s, printf gives %s\n", (double)f, N, a, b);
            ++failures;
        }
    };
    const int Ns[4] = {2, 4, 7, 0};
    for (long i = 0; i < random_cases; ++i) {
        const uint32_t u = (uint32_t)g();
        float f;
        memcpy(&f, &u, 4);
        check(f, Ns[i & 3]);
    }
    std::uniform_real_distribution<double> U(-20, 20);
    for (long i = 0; i < random_cases / 4; ++i)
        check((float)std::pow(10.0, U(g)) * ((g() & 1) ? -1.f : 1.f), Ns[i & 3]);
    for (int k = -20000; k <= 20000; ++k)
        for (int s = 1; s <= 12; ++s)
            for (int N : {2, 4, 7}) check((float)k / (float)(1 << s), N);
    for (float f : {0.f, -0.f, 1e-30f, -1e-30f, 0.125f, 0.375f, 2.5e-8f, -2.5e-8f, 0.005f, 0.015f, 1099511627775.f,
                    1099511627776.f, 3.4e38f, -3.4e38f})
        for (int N : {2, 4, 7}) check(f, N);
    for (uint32_t u : {0x7fc00000u, 0xffc00000u, 0x7f800000u, 0xff800000u, 0x00000001u, 0x807fffffu}) {
        float f;
        memcpy(&f, &u, 4);
        check(f, 7);
    }
    // "%.7Le" of long doubles: random values over the fast path's range with random low mantissa
    // bits, the P values of t from 0 to 11.2, dyadic values (exact decimal ties at the eighth
    // digit), powers of ten and their neighbours, and values outside the fast path
    auto check_sci = [&](long double v) {
        char* e = put_sci7(a, v);
        *e = 0;
        snprintf(b, sizeof b, "%.7Le", v);
        if (strcmp(a, b)) {
            if (failures < 10) printf("put_sci7(%.25Lg) = %s, printf gives %s\n", v, a, b);
            ++failures;
        }
    };
    std::uniform_real_distribution<double> L(-30.5, 0.5);
    for (long i = 0; i < random_cases; ++i) {
        int ex;
        const long double fr = frexpl(powl(10.0L, (long double)L(g)), &ex);
        uint64_t M = (uint64_t)ldexpl(fr, 64) ^ (g() & 0xffffffffull);
        M |= 1ull << 63;
        check_sci(ldexpl((long double)M, ex - 64));
    }
    for (int i = 0; i < 400000; ++i) check_sci(pvalue_ld((float)(11.2 * i / 400000.0)));
    for (int sft = 1; sft <= 40; ++sft)
        for (long j = 1; j < (1L << std::min(sft, 14)); j += 2) check_sci(ldexpl((long double)j, -sft));
    for (int d = -31; d <= 1; ++d) {
        const long double p10 = powl(10.0L, d);
        long double up = p10, dn = p10;
        for (int z = 0; z < 3; ++z) {
            check_sci(up);
            check_sci(dn);
            up = nextafterl(up, 2.0L);
            dn = nextafterl(dn, 0.0L);
        }
    }
    for (long double v : {0.0L, -0.0L, 1.0L, 0.5L, 1e-31L, 1e-300L, 2.0L, -0.25L}) check_sci(v);
    for (uint64_t v : {0ull, 9ull, 10ull, 65535ull, 4294967295ull, 18446744073709551615ull}) {
        char* e = put_u64(a, v);
        *e = 0;
        snprintf(b, sizeof b, "%llu", (unsigned long long)v);
        if (strcmp(a, b)) {
            printf("put_u64(%s) = %s\n", b, a);
            ++failures;
        }
    }
}

void names(Fvi& f, int nvar, const char* pre) {
    f.nobs = 3;
    f.nvar = (uint32_t)nvar;
    f.namelength = 32;
    f.names.assign((size_t)(f.nobs + nvar) * 32, 0);
    for (int i = 0; i < nvar; ++i) snprintf(f.names.data() + (size_t)(f.nobs + i) * 32, 32, "%s%d", pre, i + 1);
}

std::string name(const Fvi& f, size_t v) { return f.var_name(v); }
template <class T>
void put_bytes(std::string& s, T v) {
    s.append(reinterpret_cast<const char*>(&v), sizeof v);
}

// The rows as a sequential snprintf pass writes them (text and .dbin).
void plain_pass(const Writer& W, const oa_rows& rr, int s0, int cnt, std::string& txt, std::string& bin) {
    const int start_h = W.disp_cov ? 1 : W.l;
    const int nblk = (cnt + W.mb_ref - 1) / W.mb_ref;
    char line[1024];
    for (int k = 0; k < nblk; ++k) {
        std::vector<int64_t> idx;
        for (int64_t q = 0; q < rr.count; ++q)
            if (rr.snp[q] / W.mb_ref == k) idx.push_back(q);
        if (idx.empty()) continue;
        if (!W.store_all) {
            put_bytes<int32_t>(bin, rr.trait[idx[0]]);
            put_bytes<int32_t>(bin, (int32_t)idx.size());
            put_bytes<int32_t>(bin, (s0 + k * W.mb_ref) * W.r);
        }
        for (int64_t q : idx) {
            const int snp = rr.snp[q] + s0, ii = snp - (s0 + k * W.mb_ref);
            const uint32_t mask = rr.coef_mask[q];
            const float npct = (float)rr.n_used[q] / (float)W.real_n;
            put_bytes<uint16_t>(bin, (uint16_t)rr.n_used[q]);
            put_bytes<uint16_t>(bin, float16_trunc(rr.r2[q]));
            if (!W.store_all) {
                uint8_t sz = 0;
                for (int h = W.p - 1; h >= start_h; --h) sz += (mask >> h) & 1u;
                put_bytes<uint8_t>(bin, sz);
            }
            for (int h = W.p - 1; h >= start_h; --h) {
                if (!((mask >> h) & 1u)) continue;
                const float B = rr.coef_b[q * W.p + h], SE = rr.coef_se[q * W.p + h], T = rr.coef_t[q * W.p + h];
                const long double P = pvalue_ld(T);
                if ((P <= W.min_p_disp && rr.r2[q] >= W.min_r2_disp) || W.store_all) {
                    const int term = h >= W.l ? h - W.l : 0;
                    std::string an = " ";
                    if (h < W.l) an = name(*W.fl, (size_t)h) + ":";
                    if (W.n_inter > 0 && term < W.n_inter) an += "I" + std::to_string(term + 1) + "x";
                    an += name(*W.fr, (size_t)snp * W.name_stride + (W.n_inter > 0 ? 0 : (size_t)term));
                    const int len = snprintf(line, sizeof line, "%s\t%s\t%u\t%.2f\t%.7f\t%.4f\t%.7f\t%.7f\t%.7Le\n",
                                             name(*W.fy, (size_t)rr.trait[q]).c_str(), an.c_str(),
                                             (unsigned)(uint16_t)rr.n_used[q], (double)npct, (double)B,
                                             (double)rr.r2[q], (double)SE, (double)T, P);
                    txt.append(line, (size_t)len);
                }
                if (W.disp_cov && !W.store_all) put_bytes<uint8_t>(bin, h >= W.l ? (uint8_t)255 : (uint8_t)h);
                if (!W.store_all) put_bytes<uint16_t>(bin, (uint16_t)(ii * W.r + (h >= W.l ? h - W.l : 0)));
                put_bytes<float>(bin, B);
                put_bytes<float>(bin, SE);
            }
        }
    }
}

void writer_checks() {
    Fvi fy, fl, fr;
    names(fy, 40, "ph");
    names(fl, 4, "cov");
    names(fr, 4000, "snp");
    std::mt19937 g(3);
    std::uniform_real_distribution<float> U(0, 1);
    const int l = 4, r = 2, p = l + r, cnt = 1700, s0 = 600, t = 40;
    std::vector<int32_t> tr, sn, nu;
    std::vector<float> r2, b, se, tt;
    std::vector<uint32_t> mask;
    for (int j = 0; j < t; ++j)
        for (int i = 0; i < cnt; ++i) {
            if (U(g) < 0.5f) continue;
            tr.push_back(j);
            sn.push_back(i);
            nu.push_back(700 + j);
            r2.push_back(U(g) * (U(g) < 0.1f ? -1.f : 1.f));
            uint32_t m = 0;
            for (int h = 1; h < p; ++h)
                if (U(g) < 0.6f) m |= 1u << h;
            mask.push_back(m);
            for (int h = 0; h < p; ++h) {
                b.push_back((U(g) - 0.5f) * std::pow(10.f, 6.f * U(g) - 3.f));
                se.push_back(U(g) * std::pow(10.f, 4.f * U(g) - 2.f));
                tt.push_back(U(g) * 9.f);
            }
        }
    oa_rows rr{};
    rr.count = (int64_t)tr.size();
    rr.trait = tr.data();
    rr.snp = sn.data();
    rr.r2 = r2.data();
    rr.n_used = nu.data();
    rr.coef_mask = mask.data();
    rr.coef_b = b.data();
    rr.coef_se = se.data();
    rr.coef_t = tt.data();
    const RowBatch B = RowBatch::from_call(rr, p, s0, cnt, 500, 0);
    for (int variant = 0; variant < 6; ++variant) {
        Writer W;
        W.l = l;
        W.r = r;
        W.p = p;
        W.real_n = 1000;
        W.fy = &fy;
        W.fl = &fl;
        W.fr = &fr;
        W.min_p_disp = 0.05L;
        W.min_r2_disp = 0.1f;
        W.disp_cov = variant & 1;
        W.store_all = (variant & 2) != 0;
        W.n_inter = variant >= 4 ? 1 : 0;
        char tname[] = "/tmp/oa_writer_txt_XXXXXX", bname[] = "/tmp/oa_writer_bin_XXXXXX";
        const int tfd = mkstemp(tname), bfd = mkstemp(bname);
        W.dis = fdopen(tfd, "wb");
        W.dbin = fdopen(bfd, "wb");
        std::string want_txt, want_bin;
        plain_pass(W, rr, s0, cnt, want_txt, want_bin);
        for (int parts : {1, 7}) {
            std::vector<Writer::Segment> seg((size_t)parts);
            const int64_t total = (int64_t)B.order.size();
            for (int i = 0; i < parts; ++i) W.format_range(B, total * i / parts, total * (i + 1) / parts, seg[(size_t)i]);
            std::string txt, bin;
            for (const auto& s : seg) {
                txt += s.txt;
                bin += s.bin;
            }
            if (txt != want_txt || bin != want_bin) {
                printf("writer variant %d, %d parts: text %s (%zu vs %zu bytes), dbin %s\n", variant, parts,
                       txt == want_txt ? "same" : "differs", txt.size(), want_txt.size(),
                       bin == want_bin ? "same" : "differs");
                ++failures;
            }
        }
        // the files as the background writer leaves them, after a header written through the stream
        fputs("Phe\tSNP\n", W.dis);
        W.submit(RowBatch(B));
        W.submit(RowBatch(B));
        W.finish();
        fclose(W.dis);
        fclose(W.dbin);
        auto slurp = [](const char* path) {
            std::string out;
            FILE* f = fopen(path, "rb");
            char buf[1 << 16];
            size_t got;
            while (f && (got = fread(buf, 1, sizeof buf, f)) > 0) out.append(buf, got);
            if (f) fclose(f);
            return out;
        };
        const std::string ftxt = slurp(tname), fbin = slurp(bname);
        unlink(tname);
        unlink(bname);
        if (W.write_failed || ftxt != "Phe\tSNP\n" + want_txt + want_txt || fbin != want_bin + want_bin) {
            printf("writer variant %d: files differ from two sequential passes (%zu text bytes)\n", variant,
                   ftxt.size());
            ++failures;
        }
    }
}

// The genotype reader: a block of columns read in parallel slices (reads of 64 MB or more) from
// float and double files, all rows or the rows of an exclusion list, against the values written;
// a block running past the end of the file is a failed read.
void reader_checks() {
    const size_t fileN = 1000, nvar = 17000;   // 17 million values: 68 MB as float, 136 MB as double
    std::vector<double> vals(fileN * nvar);
    for (size_t q = 0; q < vals.size(); ++q) vals[q] = (double)(q % 100003) * 0.001 - 7.0;
    for (int dbl_file = 0; dbl_file < 2; ++dbl_file) {
        char name[] = "/tmp/oa_reader_XXXXXX";
        const int fd = mkstemp(name);
        FILE* f = fdopen(fd, "w+b");
        const size_t eb = dbl_file ? 8 : 4;
        for (size_t q = 0; q < vals.size(); ++q) {
            if (dbl_file) fwrite(&vals[q], 8, 1, f);
            else {
                const float x = (float)vals[q];
                fwrite(&x, 4, 1, f);
            }
        }
        fflush(f);
        const Runs all{{0, (int)fileN}}, some{{0, 100}, {250, 500}, {990, 10}};
        for (const Runs* runs : {&all, &some}) {
            size_t kept = 0;
            for (const auto& r : *runs) kept += (size_t)r.second;
            const size_t v0 = 17, count = nvar - 17;
            std::vector<float> dst(kept * count), scratch;
            std::vector<double> dbl;
            if (!read_columns(f, eb, fileN, v0, count, *runs, kept, dst.data(), scratch, dbl)) {
                printf("reader: read of %zu columns failed (%s file)\n", count, dbl_file ? "double" : "float");
                ++failures;
                continue;
            }
            size_t bad = 0;
            for (size_t c = 0; c < count; ++c) {
                size_t pos = 0;
                for (const auto& r : *runs)
                    for (int k = 0; k < r.second; ++k, ++pos)
                        bad += dst[c * kept + pos] != (float)vals[(v0 + c) * fileN + (size_t)(r.first + k)];
            }
            if (bad) {
                printf("reader: %zu values differ (%s file, %zu kept rows)\n", bad, dbl_file ? "double" : "float", kept);
                ++failures;
            }
        }
        std::vector<float> dst(fileN * 2), scratch;
        std::vector<double> dbl;
        if (read_columns(f, eb, fileN, nvar - 1, 2, Runs{{0, (int)fileN}}, fileN, dst.data(), scratch, dbl)) {
            printf("reader: a block past the end of the file was read\n");
            ++failures;
        }
        fclose(f);
        unlink(name);
    }
}

}  // namespace

int main(int argc, char** argv) {
    const long cases = argc > 1 ? atol(argv[1]) : 2000000;
    number_checks(cases);
    writer_checks();
    reader_checks();
    printf("%s: %ld failures\n", failures ? "FAIL" : "ok", failures);
    return failures ? 1 : 0;
}
