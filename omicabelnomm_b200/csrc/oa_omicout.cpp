// omicout: re-thresholds the binary outputs (<base>.ibin / <base>.dbin, the
// files the engine writes with -b) into a text table, as the reference's
// OmicOUT tool does (OmicOUT/main.cpp).  Host-only: the work is one pass over
// the stored coefficients.
//
// File layouts (written by oa_host.cpp, read back here):
//   .ibin  int32 n, l, r, t, m, namelength; uint8 disp_cov, storePInd;
//          names of the covariates 1..l-1, of the r*m SNP columns and of the
//          t traits, namelength bytes each (OmicOUT/main.cpp:263-294).
//   .dbin  storePInd (-f): for each trait, for each of the m SNPs:
//          uint16 nUsed, uint16 R2 (top half of the float), then
//          r (+ l-1 with covariates) x {float B, float SE};
//          otherwise, per write block: int32 trait, int32 rows, int32 SNP
//          offset, then per row: uint16 nUsed, uint16 R2, uint8 count, and
//          count x {[uint8 covariate index if covariates], uint16 SNP index
//          within the block, float B, float SE} (OmicOUT/main.cpp:302-420).
//
// Behaviour kept from the reference because users' scripts see it:
//   * at most t blocks are read (the loop runs over trait indices, :331);
//   * SNP name indices are 16-bit and wrap like the reference's (:310, :385);
//   * -b is cut at the first '.' of the argument (:165);
//   * rows are printed when P < the -d threshold and R2 > the -r threshold,
//     with the reference's column formats (:440-445); -f prints everything;
//   * covariate terms only with -i and when the file holds them.
#include <getopt.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "omicabel_b200.h"

namespace {

// Names are fixed-width fields; a name that fills its field runs on into the
// next one when printed, as in the reference (one NUL appended at the end).
struct NameTable {
    std::vector<char> buf;
    int width = 0;
    const char* at(long long i) const { return buf.data() + (size_t)i * width; }
};

bool read_names(std::ifstream& f, NameTable& t, long long count, int width) {
    t.width = width;
    t.buf.assign((size_t)std::max<long long>(count, 0) * width + 1, '\0');
    if (count > 0) f.read(t.buf.data(), (std::streamsize)(count * width));
    return (bool)f;
}

// One stored coefficient that passes the P filter.
struct Hit {
    float t, b, se;
    long double p;
    int al, ar;   // covariate index (255 = a SNP term), SNP column index
};

// |b / SE| and P as the reference's omicout computes them (OmicOUT/main.cpp:48-83):
// float quotient, long double P with the t < 1.6 patch.
void test_stat(float b, float se, float& t_out, long double& p_out) {
    const long double t = std::fabs(b / se);
    long double p;
    if (t < 1.6) {
        const float t1 = (float)(4.4 - t);
        p = 0.5 - 0.1 * t1 * t;
    } else {
        const long double inv_sqrt2 = 0.7071067811865475244008443621048490392848359376884740;   // as a double literal
        p = std::erfc(t * inv_sqrt2);
    }
    t_out = (float)t;
    p_out = p;
}

// One printed row.
struct Line {
    int32_t y;
    uint16_t n_used;
    float r2, pct;
    Hit h;
};

constexpr size_t LINE_BATCH = 1u << 20;

// The reference's row format (OmicOUT/main.cpp:440-445): trait, [covariate:]SNP
// (a leading space without a covariate), nUsed, its share (2 decimals), B (7),
// R2 (4), SE (7), |t| (7), P (scientific, 7).
void format_line(std::ostream& o, const Line& L, const NameTable& al_names, const NameTable& ar_names,
                 const NameTable& y_names, bool show_cov) {
    constexpr int FD = std::numeric_limits<float>::digits10 + 1;
    std::string name = " ";
    if (show_cov && L.h.al != 255) name = std::string(al_names.at(L.h.al)) + ":";
    name += ar_names.at(L.h.ar);
    o << y_names.at(L.y) << "\t" << name << "\t" << std::fixed << std::setprecision(2) << L.n_used << "\t" << L.pct
      << "\t" << std::setprecision(FD) << L.h.b << "\t" << std::fixed << std::setprecision(4) << L.r2 << "\t"
      << std::setprecision(FD) << L.h.se << "\t" << L.h.t << "\t" << std::scientific << L.h.p << std::fixed
      << std::setprecision(FD) << "\n";
}

void format_lines(const std::vector<Line>& lines, const NameTable& al_names, const NameTable& ar_names,
                  const NameTable& y_names, bool show_cov, std::ostream& out) {
    if (lines.empty()) return;
    const size_t nthr = lines.size() < 4096 ? 1
                                             : std::min<size_t>(32, std::max(1u, std::thread::hardware_concurrency()));
    std::vector<std::string> parts(nthr);
    auto work = [&](size_t k) {
        std::ostringstream o;
        const size_t a = lines.size() * k / nthr, b = lines.size() * (k + 1) / nthr;
        for (size_t q = a; q < b; ++q) format_line(o, lines[q], al_names, ar_names, y_names, show_cov);
        parts[k] = o.str();
    };
    if (nthr == 1) {
        work(0);
    } else {
        std::vector<std::thread> th;
        for (size_t k = 0; k < nthr; ++k) th.emplace_back(work, k);
        for (auto& x : th) x.join();
    }
    for (const auto& p : parts) out.write(p.data(), (std::streamsize)p.size());
}

float r2_from_u16(uint16_t v) {
    uint32_t bits = ((uint32_t)v << 16) & 0xffff0000u;
    float r;
    std::memcpy(&r, &bits, sizeof r);
    return r;
}

template <class T>
bool rd(std::ifstream& f, T& v, unsigned long long& nread) {
    f.read(reinterpret_cast<char*>(&v), sizeof v);
    nread += sizeof v;
    return (bool)f;
}

}  // namespace

extern "C" oa_status oa_omicout(const char* source, const char* dest, float min_p_disp, float min_r2,
                                int32_t force_all, int32_t include_cov, int64_t* rows_printed) {
    if (rows_printed) *rows_printed = 0;
    if (!source || !dest) return OA_ERR_ARG;
    std::ifstream fd(std::string(source) + ".dbin", std::ios::in | std::ios::binary);
    if (!fd.is_open()) {
        std::cout << "Error reading File " << source << ".dbin" << std::endl;
        return OA_ERR_IO;
    }
    std::ifstream fi(std::string(source) + ".ibin", std::ios::in | std::ios::binary);
    if (!fi) {
        std::cout << "Error Creating File " << source << ".ibin" << std::endl;
        return OA_ERR_IO;
    }
    std::ofstream out(std::string(dest) + ".txt", std::ios::out | std::ios::trunc);
    if (!out) {
        std::cout << "Error Creating File " << dest << ".txt" << std::endl;
        return OA_ERR_IO;
    }
    double pmax = min_p_disp;
    float r2min = min_r2;
    if (force_all) {
        pmax = 2.0;
        r2min = -100.0f;
    }

    int32_t n = 0, l = 0, r = 0, t = 0, m = 0, width = 0;
    uint8_t disp_cov_b = 0, per_snp_b = 0;
    unsigned long long ignored = 0;
    rd(fi, n, ignored);
    rd(fi, l, ignored);
    rd(fi, r, ignored);
    rd(fi, t, ignored);
    rd(fi, m, ignored);
    rd(fi, width, ignored);
    rd(fi, disp_cov_b, ignored);
    rd(fi, per_snp_b, ignored);
    if (!(n > 0 && l > 1 && r > 0 && m > 0 && t > 0 && width > 0)) {
        std::cout << "Input data had invalid info data!" << std::endl;
        return OA_ERR_IO;
    }
    const bool disp_cov = disp_cov_b != 0, per_snp = per_snp_b != 0;
    const bool show_cov = include_cov && disp_cov;
    NameTable al_names, ar_names, y_names;
    read_names(fi, al_names, l - 1, width);
    read_names(fi, ar_names, (long long)r * m, width);
    read_names(fi, y_names, t, width);

    fd.seekg(0, fd.end);
    const unsigned long long total = (unsigned long long)fd.tellg();
    fd.seekg(0, fd.beg);
    const int coefs = r + (disp_cov ? l - 1 : 0);   // stored terms per row with -f (no intercept)

    // Rows are collected in batches and formatted by several host threads,
    // each into its own buffer, then written in order.
    std::vector<Line> lines;
    lines.reserve(LINE_BATCH);
    int64_t printed = 0;
    auto flush_lines = [&]() {
        printed += (int64_t)lines.size();
        format_lines(lines, al_names, ar_names, y_names, show_cov, out);
        lines.clear();
    };

    unsigned long long nread = 0;
    uint8_t al = 0;   // persists across terms like the reference's (unset without covariates)
    std::vector<Hit> hits;
    for (int j = 0; j < t && nread < total; ++j) {
        int32_t y_idx = j, rows = m, ar_off = 0;
        if (!per_snp) {
            rd(fd, y_idx, nread);
            rd(fd, rows, nread);
            rd(fd, ar_off, nread);
        }
        for (int i = 0; i < rows; ++i) {
            uint16_t n_used = 0, r2_bits = 0;
            rd(fd, n_used, nread);
            rd(fd, r2_bits, nread);
            const float R2 = r2_from_u16(r2_bits);
            uint8_t count = (uint8_t)coefs;
            if (!per_snp) rd(fd, count, nread);
            hits.clear();
            for (int h = 0; h < (int)count; ++h) {
                uint16_t ar = 0;
                if (!per_snp) {
                    if (disp_cov) rd(fd, al, nread);
                    rd(fd, ar, nread);
                    ar = (uint16_t)(ar + ar_off);
                } else {
                    ar = (uint16_t)(i * r + h);
                    if (disp_cov) {
                        ar = (uint16_t)(ar - (l - 1));
                        if (h < l - 1) {
                            ar = (uint16_t)(i * r);
                            al = (uint8_t)h;
                        } else {
                            al = 255;
                        }
                    }
                }
                float B = 0.f, SE = 0.f;
                rd(fd, B, nread);
                rd(fd, SE, nread);
                const bool skip_cov = !show_cov && al != 255;
                if (!disp_cov || !skip_cov) {
                    Hit x;
                    test_stat(B, SE, x.t, x.p);
                    if ((double)x.p < pmax) {
                        x.b = B;
                        x.se = SE;
                        x.al = al;
                        x.ar = ar;
                        hits.push_back(x);
                    }
                }
            }
            if (!(R2 > r2min)) continue;
            const float pct = (float)n_used / (float)n;
            for (const Hit& x : hits) {
                lines.push_back(Line{y_idx, n_used, R2, pct, x});
                if (lines.size() == LINE_BATCH) flush_lines();
            }
        }
    }
    flush_lines();
    out.flush();
    if (!out) return OA_ERR_IO;
    if (rows_printed) *rows_printed = printed;
    return OA_OK;
}

// The reference's omicout command line (OmicOUT/main.cpp:86-227): -b/--binsource
// <base>, -o/--out <base>, -d/--pdisp <P>, -r/--rdisp <R2>, -i/--fdcov,
// -f/--fdgen; -b, -o and -d are required; exit status 1 on every error.
extern "C" int oa_omicout_main(int argc, char** argv) {
    std::string source, dest;
    bool force_all = false, include_cov = false, have_out = false, have_bin = false, have_p = false;
    float min_p = 0.f, min_r2 = -100.0f;
    static const struct option longopts[] = {{"binsource", required_argument, nullptr, 'b'},
                                             {"out", required_argument, nullptr, 'o'},
                                             {"pdisp", required_argument, nullptr, 'd'},
                                             {"rdisp", required_argument, nullptr, 'r'},
                                             {"fdcov", no_argument, nullptr, 'i'},
                                             {"fdgen", no_argument, nullptr, 'f'},
                                             {nullptr, 0, nullptr, 0}};
    optind = 1;
    for (;;) {
        int idx = 0;
        const int c = getopt_long(argc, argv, "b:o:d:r:fi", longopts, &idx);
        if (c == -1) break;
        if (!optarg && c != 'f' && c != 'i') {
            std::cout << "\nerror with argument parameter " << (char)c << std::endl;
            return 1;
        }
        switch (c) {
            case 'o':
                have_out = !have_out;
                dest = optarg;
                std::cout << "-o Writing output text file to " << dest << std::endl;
                break;
            case 'b': {
                have_bin = !have_bin;
                source = optarg;
                const size_t dot = source.find('.');
                if (dot != std::string::npos) source = source.substr(0, dot);
                std::cout << "-o Reading input from file " << source << std::endl;
                break;
            }
            case 'd':
                min_p = std::fabs((float)std::atof(optarg));
                have_p = true;
                std::cout << "-d Significance to display in .txt will be P-val's below " << min_p << std::endl;
                break;
            case 'r':
                min_r2 = (float)std::atof(optarg);
                std::cout << "-r Minimum R2 to display in .txt will be above " << min_r2 << std::endl;
                break;
            case 'i':
                include_cov = true;
                std::cout << "-i Covariate results will be included in results" << std::endl;
                break;
            case 'f':
                force_all = true;
                std::cout << "-f Forcing all includec results to be considered independently of max P-val or "
                             "min R2. (Overrides -t and -d, Big file!)"
                          << std::endl;
                break;
            default:
                break;   // getopt printed the message
        }
    }
    if (optind < argc) {
        std::printf("non-option ARGV-elements: ");
        while (optind < argc) std::printf("%s ", argv[optind++]);
        std::putchar('\n');
    }
    if (!have_bin || !have_out || !have_p) {
        std::cout << "Missing arguments!:" << " o:" << have_out << " b:" << have_bin << " d:" << have_p << std::endl;
        return 1;
    }
    const oa_status s = oa_omicout(source.c_str(), dest.c_str(), min_p, min_r2, force_all, include_cov, nullptr);
    return s == OA_OK ? 0 : 1;
}
