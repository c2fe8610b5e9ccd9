// dataset.cpp -- the reference's dataset descriptor / .bin I/O and the
// seeded synthetic generator.
//
// Descriptor (src/tensor-episdet.cu:58-83): five lines -- number of SNPs,
// controls file, number of controls, cases file, number of cases -- with file
// names relative to the descriptor's directory (:64-65, :134).  Each .bin is
// the class's [SNP][g in {0,1}][ceil(n/1024)*32] uint32 words (:111-148).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "episdet.h"
#include "host_util.h"

using namespace episdet;

extern "C" int32_t episdet_class_words(int32_t n) { return ((n + 1023) / 1024) * 32; }

static std::string dir_of(const std::string& p) {
    size_t s = p.find_last_of('/');
    if (s == std::string::npos) return ".";
    if (s == 0) return "/";
    return p.substr(0, s);
}

static std::string base_of(const std::string& p) {
    size_t s = p.find_last_of('/');
    return s == std::string::npos ? p : p.substr(s + 1);
}

static bool read_line(FILE* f, std::string& out) {
    char buf[4096];
    if (!fgets(buf, sizeof(buf), f)) return false;
    out = buf;
    while (!out.empty() && (out.back() == '\n' || out.back() == '\r')) out.pop_back();
    return true;
}

static episdet_status read_bin(const std::string& path, size_t words, uint32_t** out) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return set_error(EPISDET_ERR_IO, "cannot open '%s'", path.c_str());
    uint32_t* buf = (uint32_t*)malloc(std::max<size_t>(words, 1) * sizeof(uint32_t));
    if (!buf) {
        fclose(f);
        return set_error(EPISDET_ERR_OUT_OF_MEMORY, "host allocation of %zu words failed", words);
    }
    size_t got = fread(buf, sizeof(uint32_t), words, f);
    fclose(f);
    if (got != words) {
        free(buf);
        return set_error(EPISDET_ERR_IO, "'%s' holds %zu words, expected %zu", path.c_str(), got, words);
    }
    *out = buf;
    return EPISDET_OK;
}

extern "C" episdet_status episdet_read_dataset(const char* descriptor_path, episdet_dataset* out) {
    if (!descriptor_path || !out) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "null argument");
    memset(out, 0, sizeof(*out));
    FILE* f = fopen(descriptor_path, "r");
    if (!f) return set_error(EPISDET_ERR_IO, "File '%s' does not exist!", descriptor_path);
    std::string l_snps, l_ctrl_file, l_nctrl, l_case_file, l_ncase;
    bool ok = read_line(f, l_snps) && read_line(f, l_ctrl_file) && read_line(f, l_nctrl) &&
              read_line(f, l_case_file) && read_line(f, l_ncase);
    fclose(f);
    if (!ok) return set_error(EPISDET_ERR_IO, "descriptor '%s' has fewer than 5 lines", descriptor_path);
    long m = atol(l_snps.c_str()), nctrl = atol(l_nctrl.c_str()), ncase = atol(l_ncase.c_str());
    if (m < 1 || m > (1L << 21) - 1 || nctrl < 1 || ncase < 1 || nctrl > (1L << 30) || ncase > (1L << 30))
        return set_error(EPISDET_ERR_IO, "descriptor '%s': bad sizes (snps %ld, controls %ld, cases %ld)",
                         descriptor_path, m, nctrl, ncase);
    std::string dir = dir_of(descriptor_path);
    uint32_t *cases = nullptr, *controls = nullptr;
    size_t wc = (size_t)episdet_class_words((int32_t)ncase), wn = (size_t)episdet_class_words((int32_t)nctrl);
    episdet_status s = read_bin(dir + "/" + l_case_file, (size_t)m * 2 * wc, &cases);
    if (s != EPISDET_OK) return s;
    s = read_bin(dir + "/" + l_ctrl_file, (size_t)m * 2 * wn, &controls);
    if (s != EPISDET_OK) {
        free(cases);
        return s;
    }
    out->cases = cases;
    out->controls = controls;
    out->num_snps = (int32_t)m;
    out->num_cases = (int32_t)ncase;
    out->num_controls = (int32_t)nctrl;
    out->memory = EPISDET_HOST;
    return EPISDET_OK;
}

extern "C" void episdet_free_dataset(episdet_dataset* d) {
    if (!d) return;
    free((void*)d->cases);
    free((void*)d->controls);
    d->cases = d->controls = nullptr;
}

extern "C" episdet_status episdet_write_dataset(const char* descriptor_path, const episdet_dataset* d) {
    if (!descriptor_path || !d || !d->cases || !d->controls || d->memory != EPISDET_HOST)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "write_dataset needs host arrays and a path");
    std::string desc = descriptor_path;
    std::string dir = dir_of(desc), stem = base_of(desc);
    size_t dot = stem.rfind('.');
    if (dot != std::string::npos) stem = stem.substr(0, dot);
    std::string fc = stem + ".cases.bin", fn = stem + ".controls.bin";
    struct Part {
        std::string name;
        const uint32_t* p;
        size_t words;
    } parts[2] = {{fc, d->cases, (size_t)d->num_snps * 2 * episdet_class_words(d->num_cases)},
                  {fn, d->controls, (size_t)d->num_snps * 2 * episdet_class_words(d->num_controls)}};
    for (auto& p : parts) {
        FILE* f = fopen((dir + "/" + p.name).c_str(), "wb");
        if (!f) return set_error(EPISDET_ERR_IO, "cannot create '%s'", (dir + "/" + p.name).c_str());
        size_t put = fwrite(p.p, sizeof(uint32_t), p.words, f);
        fclose(f);
        if (put != p.words) return set_error(EPISDET_ERR_IO, "short write to '%s'", p.name.c_str());
    }
    FILE* f = fopen(desc.c_str(), "w");
    if (!f) return set_error(EPISDET_ERR_IO, "cannot create '%s'", desc.c_str());
    fprintf(f, "%d\n%s\n%d\n%s\n%d\n", d->num_snps, fn.c_str(), d->num_controls, fc.c_str(), d->num_cases);
    fclose(f);
    return EPISDET_OK;
}

extern "C" uint64_t episdet_n_choose_k(uint32_t n, uint32_t k) {
    // helper.cu:758-768: nC_i from nC_{i-1}, exact at every step.
    uint64_t r = 1;
    for (uint32_t i = 1; i <= k; ++i) {
        r = r * n / i;
        n = n - 1;
    }
    return r;
}

// ------------------------------------------------------------ generator
// Counter-based: every draw is a pure function of (seed, stream, index), so
// any subset of SNPs or samples can be regenerated independently and in
// parallel.  Mixer: the SplitMix64 finaliser (Steele, Lea & Flood 2014).
static inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline uint64_t draw(uint64_t seed, uint64_t stream, uint64_t idx) {
    return mix64(mix64(seed ^ mix64(stream)) ^ idx);
}
static inline double u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

enum : uint64_t { kTagMaf = 0x4D4146ull, kTagGeno = 0x47454E4Full << 24, kTagLabel = 0x4C4142ull, kTagPerm = 0x5045524Dull };

static inline double snp_maf(uint64_t seed, int32_t snp, double lo, double hi) {
    return lo + (hi - lo) * u01(draw(seed, kTagMaf, (uint64_t)snp));
}
// Hardy-Weinberg genotype: 0 w.p. (1-p)^2, 1 w.p. 2p(1-p), 2 w.p. p^2.
static inline int genotype(uint64_t seed, int32_t snp, uint64_t ind, double p) {
    double u = u01(draw(seed, kTagGeno + (uint64_t)snp, ind));
    double q0 = (1.0 - p) * (1.0 - p);
    if (u < q0) return 0;
    if (u < 1.0 - p * p) return 1;
    return 2;
}

static void fill_planes(uint64_t seed, int32_t M, const std::vector<double>& maf, const std::vector<uint64_t>& ids,
                        uint32_t* planes) {
    int32_t n = (int32_t)ids.size();
    size_t W = (size_t)episdet_class_words(n);
    unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&, t]() {
            for (int32_t snp = (int32_t)t; snp < M; snp += (int32_t)nt) {
                uint32_t* r0 = planes + ((size_t)snp * 2 + 0) * W;
                uint32_t* r1 = r0 + W;
                memset(r0, 0, sizeof(uint32_t) * 2 * W);
                for (int32_t s = 0; s < n; ++s) {
                    int g = genotype(seed, snp, ids[s], maf[snp]);
                    if (g < 2) (g == 0 ? r0 : r1)[s / 32] |= 1u << (31 - s % 32);
                }
            }
        });
    for (auto& x : th) x.join();
}

extern "C" episdet_status episdet_generate(const episdet_synth* sp, uint32_t* cases, uint32_t* controls) {
    if (!sp || !cases || !controls || sp->num_snps < 1 || sp->num_cases < 1 || sp->num_controls < 1 ||
        sp->num_planted < 0 || sp->num_planted > 2 || !(sp->maf_min >= 0.0f) || !(sp->maf_max <= 0.5f) ||
        sp->maf_min > sp->maf_max)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "bad synthetic spec");
    int32_t M = sp->num_snps;
    int ord = sp->planted_order == 2 ? 2 : 3;
    std::vector<double> maf((size_t)M);
    for (int32_t s = 0; s < M; ++s) maf[s] = snp_maf(sp->seed, s, sp->maf_min, sp->maf_max);
    for (int q = 0; q < sp->num_planted; ++q)
        for (int e = 0; e < ord; ++e) {
            int32_t s = sp->planted[q][e];
            if (s < 0 || s >= M) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "planted SNP %d out of range", s);
            if (sp->planted_maf > 0.0f) maf[s] = sp->planted_maf;
        }
    std::vector<uint64_t> case_ids, ctrl_ids;
    case_ids.reserve(sp->num_cases);
    ctrl_ids.reserve(sp->num_controls);
    if (sp->num_planted == 0) {
        // Labels independent of genotype: individuals 0..nc-1 are cases.
        for (int32_t i = 0; i < sp->num_cases; ++i) case_ids.push_back((uint64_t)i);
        for (int32_t i = 0; i < sp->num_controls; ++i) ctrl_ids.push_back((uint64_t)(sp->num_cases + i));
    } else {
        // Individuals drawn in order; each is a case with the penetrance of
        // its planted genotypes and is kept while its class has room.
        uint64_t ind = 0;
        const uint64_t limit = 64ull * (uint64_t)(sp->num_cases + sp->num_controls) + 1000000ull;
        while ((int32_t)case_ids.size() < sp->num_cases || (int32_t)ctrl_ids.size() < sp->num_controls) {
            if (ind > limit) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "penetrance model cannot fill classes");
            double risk = sp->base_risk;
            for (int q = 0; q < sp->num_planted; ++q) {
                bool carried = true;
                for (int e = 0; e < ord; ++e) {
                    int32_t s = sp->planted[q][e];
                    carried = carried && genotype(sp->seed, s, ind, maf[s]) >= 1;
                }
                if (carried) risk += sp->effect;
            }
            bool is_case = u01(draw(sp->seed, kTagLabel, ind)) < risk;
            if (is_case && (int32_t)case_ids.size() < sp->num_cases) case_ids.push_back(ind);
            if (!is_case && (int32_t)ctrl_ids.size() < sp->num_controls) ctrl_ids.push_back(ind);
            ++ind;
        }
    }
    fill_planes(sp->seed, M, maf, case_ids, cases);
    fill_planes(sp->seed, M, maf, ctrl_ids, controls);
    return EPISDET_OK;
}

extern "C" episdet_status episdet_generate_cohort(uint64_t seed, int32_t M, int32_t n, float maf_min, float maf_max,
                                                  uint32_t* planes) {
    if (!planes || M < 1 || n < 1 || maf_min < 0.0f || maf_max > 0.5f || maf_min > maf_max)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "bad cohort spec");
    std::vector<double> maf((size_t)M);
    for (int32_t s = 0; s < M; ++s) maf[s] = snp_maf(seed, s, maf_min, maf_max);
    std::vector<uint64_t> ids((size_t)n);
    for (int32_t i = 0; i < n; ++i) ids[i] = (uint64_t)i;
    fill_planes(seed, M, maf, ids, planes);
    return EPISDET_OK;
}

extern "C" episdet_status episdet_generate_labels(uint64_t seed, int32_t n, int32_t num_cases, int32_t num_labels,
                                                  uint32_t* labels) {
    if (!labels || n < 2 || num_cases < 1 || num_cases >= n || num_labels < 1)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "bad label spec");
    size_t W = (size_t)episdet_class_words(n);
    std::vector<uint8_t> lab((size_t)n);
    for (int32_t p = 0; p < num_labels; ++p) {
        for (int32_t s = 0; s < n; ++s) lab[s] = s < num_cases ? 1 : 0;
        if (p > 0)  // Fisher-Yates with the counter-based stream of permutation p
            for (int32_t i = n - 1; i > 0; --i) {
                uint64_t h = draw(seed, kTagPerm + (uint64_t)p, (uint64_t)i);
                int32_t j = (int32_t)((unsigned __int128)h * (unsigned __int128)(uint64_t)(i + 1) >> 64);
                std::swap(lab[i], lab[j]);
            }
        uint32_t* out = labels + (size_t)p * W;
        memset(out, 0, sizeof(uint32_t) * W);
        for (int32_t s = 0; s < n; ++s)
            if (lab[s]) out[s / 32] |= 1u << (31 - s % 32);
    }
    return EPISDET_OK;
}
