// resume.cpp -- permutation significance and the resumable (checkpointed)
// search: host code over the public entry points.
//
// Neither exists in the reference, which runs one search per process and
// prints its single best set (src/tensor-episdet.cu:159-185).
//
// The resumable search splits the first-SNP range into slabs of about equal
// work and calls episdet_search on each.  Every slab returns its top_k list
// in the engines' FP32 order (score key, then set); the union of the slabs'
// lists holds the top_k of the whole range, so merging them in that order
// reproduces one uninterrupted search's list, and the FP64 optimum over it is
// the same best set.
#include <cuda_runtime.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "episdet.h"
#include "host_util.h"

using namespace episdet;

namespace {

// ------------------------------------------------------------ significance

bool as_extreme(double perm_best, double s, bool maximize) { return maximize ? perm_best >= s : perm_best <= s; }

// ------------------------------------------------------------ candidates

struct Entry {
    uint32_t snps[3];
    float fp32;
    double fp64;
};

// The engines' candidate key: lower is better for both scores.
uint32_t score_key(float s, bool maximize) {
    if (maximize) s = -s;
    uint32_t u;
    std::memcpy(&u, &s, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

bool fp32_before(const Entry& a, const Entry& b, bool maximize) {
    const uint32_t ka = score_key(a.fp32, maximize), kb = score_key(b.fp32, maximize);
    if (ka != kb) return ka < kb;
    return std::lexicographical_compare(a.snps, a.snps + 3, b.snps, b.snps + 3);
}

// ------------------------------------------------------------ checkpoint file

constexpr char kMagic[8] = {'E', 'P', 'I', 'S', 'C', 'K', 'P', '1'};

struct Header {
    char magic[8];
    int32_t num_snps, num_cases, num_controls, order, score, top_k, first_begin, first_end;
    uint64_t fingerprint;
    int32_t cursor;  // next first SNP to search
    int32_t count;   // candidates that follow
    int64_t sets_evaluated, rounds, count_kernel_launches, h2d_bytes, d2h_bytes;
    uint64_t kernel_launches;
    double seconds, device_ms, count_kernel_ms, executed_macs;
};

struct State {
    Header h;
    std::vector<Entry> cands;
};

// 64-bit fingerprint of the planes: a sum of mixed words, so it is cheap to
// accumulate chunk by chunk (splitmix64's finaliser over word ^ position).
uint64_t mix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

episdet_status fingerprint_words(const uint32_t* words, size_t n, int memory, uint64_t salt, uint64_t* acc) {
    if (memory == EPISDET_HOST) {
        for (size_t i = 0; i < n; ++i) *acc += mix(((uint64_t)words[i] << 32) ^ (uint64_t)i ^ salt);
        return EPISDET_OK;
    }
    const size_t chunk = (size_t)4 << 20;  // words
    std::vector<uint32_t> buf(std::min(n, chunk));
    for (size_t off = 0; off < n; off += chunk) {
        const size_t m = std::min(chunk, n - off);
        cudaError_t e = cudaMemcpy(buf.data(), words + off, m * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess)
            return set_error(EPISDET_ERR_CUDA, "fingerprint copy: %s", cudaGetErrorString(e));
        for (size_t i = 0; i < m; ++i) *acc += mix(((uint64_t)buf[i] << 32) ^ (uint64_t)(off + i) ^ salt);
    }
    return EPISDET_OK;
}

episdet_status read_state(const std::string& path, State* s, bool* found) {
    *found = false;
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return EPISDET_OK;
    Header h;
    if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, kMagic, 8) != 0 || h.count < 0) {
        std::fclose(f);
        return set_error(EPISDET_ERR_IO, "%s is not a search checkpoint", path.c_str());
    }
    std::vector<Entry> c((size_t)h.count);
    if (h.count && std::fread(c.data(), sizeof(Entry), c.size(), f) != c.size()) {
        std::fclose(f);
        return set_error(EPISDET_ERR_IO, "checkpoint %s is truncated", path.c_str());
    }
    std::fclose(f);
    s->h = h;
    s->cands = std::move(c);
    *found = true;
    return EPISDET_OK;
}

// Written to a temporary file, flushed to disk, then renamed over `path`.
episdet_status write_state(const std::string& path, State& s) {
    const std::string tmp = path + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return set_error(EPISDET_ERR_IO, "cannot write %s", tmp.c_str());
    s.h.count = (int32_t)s.cands.size();
    bool ok = std::fwrite(&s.h, sizeof(s.h), 1, f) == 1;
    if (ok && !s.cands.empty()) ok = std::fwrite(s.cands.data(), sizeof(Entry), s.cands.size(), f) == s.cands.size();
    ok = ok && std::fflush(f) == 0 && fsync(fileno(f)) == 0;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) {
        std::remove(tmp.c_str());
        return set_error(EPISDET_ERR_IO, "cannot write checkpoint %s", path.c_str());
    }
    return EPISDET_OK;
}

// Work of the sets whose first SNP is x.
double first_work(int64_t M, int order, int64_t x) {
    const double r = (double)(M - 1 - x);
    return order == 2 ? r : r * (r - 1.0) / 2.0;
}

// Slab ends over [fb, last): num_slabs ranges of about equal work.
std::vector<int> slab_ends(int M, int order, int fb, int last, int num_slabs) {
    double total = 0.0;
    for (int x = fb; x < last; ++x) total += first_work(M, order, x);
    std::vector<int> ends;
    double acc = 0.0;
    int k = 1;
    for (int x = fb; x < last; ++x) {
        acc += first_work(M, order, x);
        if (acc >= total * k / num_slabs && x + 1 < last) {
            ends.push_back(x + 1);
            while (k < num_slabs && acc >= total * k / num_slabs) ++k;
        }
    }
    ends.push_back(last);
    return ends;
}

}  // namespace

extern "C" episdet_status episdet_perm_pvalues(const episdet_result* results, int32_t num_labels, int32_t score,
                                               double* pvalues, int32_t capacity, int32_t* count) {
    clear_error();
    if (!results || !pvalues || !count || capacity < 1)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "null pointer or capacity < 1");
    if (num_labels < 2) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "need the observed labels and >= 1 permutation");
    if (score != EPISDET_SCORE_K2 && score != EPISDET_SCORE_MI)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "unknown score %d", score);
    const bool maximize = score == EPISDET_SCORE_MI;
    const episdet_result& obs = results[0];
    const bool list = obs.top_count > 0 && obs.top_fp64;
    const int n = list ? std::min(obs.top_count, capacity) : 1;
    for (int j = 0; j < n; ++j) {
        const double s = list ? obs.top_fp64[j] : obs.score;
        int64_t hits = 0;
        for (int i = 1; i < num_labels; ++i) hits += as_extreme(results[i].score, s, maximize) ? 1 : 0;
        pvalues[j] = (double)(1 + hits) / (double)num_labels;
    }
    *count = n;
    return EPISDET_OK;
}

extern "C" episdet_status episdet_search_resumable(const episdet_dataset* data, const episdet_options* opts,
                                                   episdet_resume* rs, episdet_result* result) {
    clear_error();
    if (!data || !rs || !result || !rs->path || !rs->path[0])
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "null dataset, resume state, result or path");
    episdet_options o;
    if (opts)
        o = *opts;
    else
        episdet_default_options(&o);
    const int M = data->num_snps;
    if (o.order != 2 && o.order != 3) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "order must be 2 or 3");
    if (o.score != EPISDET_SCORE_K2 && o.score != EPISDET_SCORE_MI)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "unknown score %d", o.score);
    if (M < o.order || data->num_cases < 1 || data->num_controls < 1 || !data->cases || !data->controls)
        return set_error(EPISDET_ERR_INVALID_ARGUMENT, "bad dataset sizes");
    if (o.top_k <= 0) o.top_k = 1024;
    const int fb = std::max(0, o.first_begin);
    const int fe = (o.first_end <= 0 || o.first_end > M) ? M : o.first_end;
    const int last = std::min(fe, M - o.order + 1);  // first SNPs with at least one set
    if (fb >= last) return set_error(EPISDET_ERR_INVALID_ARGUMENT, "first-SNP range [%d,%d) holds no set", fb, fe);
    const int num_slabs = rs->num_slabs > 0 ? rs->num_slabs : 16;
    const bool maximize = o.score == EPISDET_SCORE_MI;
    const int k = o.top_k;

    // Fingerprint of this search: sizes, options and plane contents.
    Header cur;
    std::memset(&cur, 0, sizeof(cur));
    std::memcpy(cur.magic, kMagic, 8);
    cur.num_snps = M;
    cur.num_cases = data->num_cases;
    cur.num_controls = data->num_controls;
    cur.order = o.order;
    cur.score = o.score;
    cur.top_k = k;
    cur.first_begin = fb;
    cur.first_end = fe;
    uint64_t fp = mix((uint64_t)M * 1000003ull + (uint64_t)o.order * 7 + (uint64_t)o.score) ^
                  mix(((uint64_t)data->num_cases << 32) | (uint64_t)data->num_controls) ^
                  mix(((uint64_t)k << 40) ^ ((uint64_t)fb << 20) ^ (uint64_t)fe);
    const size_t wc = (size_t)M * 2 * episdet_class_words(data->num_cases);
    const size_t wn = (size_t)M * 2 * episdet_class_words(data->num_controls);
    episdet_status st = fingerprint_words(data->cases, wc, data->memory, 0x1ull << 62, &fp);
    if (st != EPISDET_OK) return st;
    st = fingerprint_words(data->controls, wn, data->memory, 0x2ull << 62, &fp);
    if (st != EPISDET_OK) return st;
    cur.fingerprint = fp;

    const std::string path(rs->path);
    State s;
    bool found = false;
    st = read_state(path, &s, &found);
    if (st != EPISDET_OK) return st;
    if (found) {
        const Header& h = s.h;
        if (h.num_snps != cur.num_snps || h.num_cases != cur.num_cases || h.num_controls != cur.num_controls ||
            h.order != cur.order || h.score != cur.score || h.top_k != cur.top_k || h.first_begin != cur.first_begin ||
            h.first_end != cur.first_end || h.fingerprint != cur.fingerprint)
            return set_error(EPISDET_ERR_INVALID_ARGUMENT, "checkpoint %s belongs to another search", path.c_str());
        if (h.cursor < fb || h.cursor > last || h.count > k)
            return set_error(EPISDET_ERR_IO, "checkpoint %s is inconsistent", path.c_str());
    } else {
        s.h = cur;
        s.h.cursor = fb;
    }

    const std::vector<int> ends = slab_ends(M, o.order, fb, last, num_slabs);
    std::vector<uint32_t> tsnps((size_t)k * 3);
    std::vector<float> tf32((size_t)k);
    std::vector<double> tf64((size_t)k);
    rs->slabs_run = 0;
    while (s.h.cursor < last && (rs->max_slabs <= 0 || rs->slabs_run < rs->max_slabs)) {
        const int b = s.h.cursor;
        const int e = *std::upper_bound(ends.begin(), ends.end(), b);
        episdet_options so = o;
        so.first_begin = b;
        so.first_end = e;
        episdet_result r;
        std::memset(&r, 0, sizeof(r));
        r.top_capacity = k;
        r.top_snps = tsnps.data();
        r.top_fp32 = tf32.data();
        r.top_fp64 = tf64.data();
        st = episdet_search(data, &so, &r);
        if (st != EPISDET_OK) return st;  // the checkpoint keeps the last finished slab
        for (int i = 0; i < r.top_count; ++i) {
            Entry en;
            for (int c = 0; c < 3; ++c) en.snps[c] = tsnps[(size_t)i * 3 + c];
            en.fp32 = tf32[i];
            en.fp64 = tf64[i];
            s.cands.push_back(en);
        }
        std::sort(s.cands.begin(), s.cands.end(),
                  [maximize](const Entry& x, const Entry& y) { return fp32_before(x, y, maximize); });
        if ((int)s.cands.size() > k) s.cands.resize((size_t)k);
        s.h.sets_evaluated += r.sets_evaluated;
        s.h.rounds = r.rounds;  // the whole search's reference round count, the same for every slab
        s.h.count_kernel_launches += r.count_kernel_launches;
        s.h.h2d_bytes += r.h2d_bytes;
        s.h.d2h_bytes += r.d2h_bytes;
        s.h.kernel_launches += r.kernel_launches;
        s.h.seconds += r.seconds;
        s.h.device_ms += r.device_ms;
        s.h.count_kernel_ms += r.count_kernel_ms;
        s.h.executed_macs += r.executed_macs;
        s.h.cursor = e;
        st = write_state(path, s);
        if (st != EPISDET_OK) return st;
        ++rs->slabs_run;
    }
    rs->next_first = s.h.cursor;
    rs->done = s.h.cursor >= last ? 1 : 0;

    // The answer so far: FP64 optimum of the merged list, ties to the lowest set.
    int best = -1;
    for (int i = 0; i < (int)s.cands.size(); ++i) {
        if (best < 0) {
            best = i;
            continue;
        }
        const Entry& a = s.cands[i];
        const Entry& bb = s.cands[best];
        bool better = maximize ? a.fp64 > bb.fp64 : a.fp64 < bb.fp64;
        if (a.fp64 == bb.fp64) better = std::lexicographical_compare(a.snps, a.snps + 3, bb.snps, bb.snps + 3);
        if (better) best = i;
    }
    const int cap = result->top_capacity;
    uint32_t* out_snps = result->top_snps;
    float* out_f32 = result->top_fp32;
    double* out_f64 = result->top_fp64;
    std::memset(result, 0, sizeof(*result));
    result->top_capacity = cap;
    result->top_snps = out_snps;
    result->top_fp32 = out_f32;
    result->top_fp64 = out_f64;
    if (best >= 0) {
        const Entry& bst = s.cands[best];
        for (int c = 0; c < 3; ++c) result->snps[c] = bst.snps[c];
        result->packed_indices = o.order == 2
                                     ? ((uint64_t)bst.snps[0] | ((uint64_t)bst.snps[1] << 32))
                                     : ((uint64_t)bst.snps[0] | ((uint64_t)bst.snps[1] << 21) |
                                        ((uint64_t)bst.snps[2] << 42));
        result->score = bst.fp64;
        result->score_fp32 = bst.fp32;
    }
    const int n = std::min((int)s.cands.size(), std::max(cap, 0));
    for (int i = 0; i < n; ++i) {
        if (out_snps)
            for (int c = 0; c < 3; ++c) out_snps[(size_t)i * 3 + c] = s.cands[i].snps[c];
        if (out_f32) out_f32[i] = s.cands[i].fp32;
        if (out_f64) out_f64[i] = s.cands[i].fp64;
    }
    result->top_count = (out_snps || out_f32 || out_f64) ? n : 0;
    result->sets_evaluated = s.h.sets_evaluated;
    result->rounds = s.h.rounds;
    result->seconds = s.h.seconds;
    result->device_ms = s.h.device_ms;
    result->kernel_launches = s.h.kernel_launches;
    result->count_kernel_ms = s.h.count_kernel_ms;
    result->count_kernel_launches = s.h.count_kernel_launches;
    result->executed_macs = s.h.executed_macs;
    result->h2d_bytes = s.h.h2d_bytes;
    result->d2h_bytes = s.h.d2h_bytes;
    return EPISDET_OK;
}
