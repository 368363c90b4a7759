// tune.cu -- autotuner of the blind rotation and its on-disk cache.
//
// The blind rotation has two launch-form knobs on the FFT64 backend: the grouping mb (1, 2 or 3
// LWE coefficients per step, with 2^mb - 1 grouped keys, or the staged 4 = 3 + 1 with 8 keys)
// and, for a two-digit gadget with mb = 2,
// the schedule (the two digit transforms one after the other, in lockstep, or in lockstep with
// two ciphertexts per CTA at N = 2048).  The tuner times
// every candidate on a synthetic batch with CUDA events and keeps the fastest; the choice is
// stored per (GPU name, parameter set, batch bucket) in a small JSON file that every context
// reads at creation.  (The reference has no tuner of its own: ~70 environment knobs,
// examples/aes_transcipher/main.cu:107-136, and an inline timing of three block sizes,
// bitwise/src/cirbts/cirbts-batch.cu:2410-2460.)
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "common.cuh"
#include "context.cuh"

namespace cbs {

static std::string cache_file(const char* path) {
    if (path && *path) return path;
    if (const char* e = std::getenv("CBS_TUNE_CACHE"); e && *e) return e;
    if (const char* x = std::getenv("XDG_CACHE_HOME"); x && *x) return std::string(x) + "/cbs_b200/tune.json";
    if (const char* h = std::getenv("HOME"); h && *h) return std::string(h) + "/.cache/cbs_b200/tune.json";
    return "";
}

static void make_parent_dirs(const std::string& file) {
    for (size_t i = 1; i < file.size(); ++i)
        if (file[i] == '/') mkdir(file.substr(0, i).c_str(), 0755);  // existing levels fail harmlessly
}

static uint32_t batch_bucket(uint32_t batch) {
    uint32_t b = 1;
    while (b < batch && b < (1u << 30)) b <<= 1;
    return b;
}

// "<GPU name>|N=..|Q=..|n=..|g=<bits>x<digits>" (the batch bucket is a field of the entry)
static std::string param_key(const cbs_context* c) {
    cudaDeviceProp prop{};
    std::string gpu = "unknown";
    if (cudaGetDeviceProperties(&prop, c->device) == cudaSuccess) gpu = prop.name;
    for (char& ch : gpu)
        if (ch == '"' || ch == '\\' || ch == '|') ch = '_';
    std::ostringstream k;
    k << gpu << "|N=" << c->p.N << "|Q=" << c->p.Q << "|n=" << c->p.n << "|g=" << __builtin_ctz(c->p.base_g) << "x"
      << c->p.digits_g;
    return k.str();
}

// The cache holds one flat object per line:
//   {"key": "...", "bucket": B, "mb": M, "schedule": S, "us_per_bootstrap": U, "batch": T, "candidates": C}
// between a "[" and a "]" line (a JSON array); lines are rewritten whole, so the reader only
// needs to find the fields of its own format.
struct CacheEntry {
    std::string key;
    uint32_t bucket = 0;
    cbs_tune_choice choice{};
};

static bool field_num(const std::string& line, const char* name, double* out) {
    const std::string pat = std::string("\"") + name + "\":";
    const size_t at = line.find(pat);
    if (at == std::string::npos) return false;
    const char* p = line.c_str() + at + pat.size();
    char* end = nullptr;
    const double v = std::strtod(p, &end);
    if (end == p) return false;
    *out = v;
    return true;
}

static bool field_str(const std::string& line, const char* name, std::string* out) {
    const std::string pat = std::string("\"") + name + "\": \"";
    const size_t at = line.find(pat);
    if (at == std::string::npos) return false;
    const size_t from = at + pat.size(), to = line.find('"', from);
    if (to == std::string::npos) return false;
    *out = line.substr(from, to - from);
    return true;
}

static std::vector<CacheEntry> read_cache(const std::string& file) {
    std::vector<CacheEntry> out;
    std::ifstream f(file);
    std::string line;
    while (std::getline(f, line)) {
        CacheEntry e;
        double mb = 0, sch = 0, us = 0, bucket = 0, batch = 0, cand = 0;
        if (!field_str(line, "key", &e.key) || !field_num(line, "bucket", &bucket) || !field_num(line, "mb", &mb) ||
            !field_num(line, "schedule", &sch) || !field_num(line, "us_per_bootstrap", &us))
            continue;
        field_num(line, "batch", &batch);
        field_num(line, "candidates", &cand);
        if (mb < 1 || mb > 4 || sch < 0 || sch > CBS_BR_SCHEDULE_PAIRED) continue;
        e.bucket = static_cast<uint32_t>(bucket);
        e.choice.mb = static_cast<uint32_t>(mb);
        e.choice.schedule = static_cast<uint32_t>(sch);
        e.choice.us_per_bootstrap = us;
        e.choice.batch = static_cast<uint32_t>(batch);
        e.choice.candidates = static_cast<uint32_t>(cand);
        out.push_back(e);
    }
    return out;
}

static bool write_cache(const std::string& file, const std::vector<CacheEntry>& entries) {
    make_parent_dirs(file);
    const std::string tmp = file + ".tmp";
    {
        std::ofstream f(tmp, std::ios::trunc);
        if (!f) return false;
        f << "[\n";
        for (size_t i = 0; i < entries.size(); ++i) {
            const auto& e = entries[i];
            f << "{\"key\": \"" << e.key << "\", \"bucket\": " << e.bucket << ", \"mb\": " << e.choice.mb
              << ", \"schedule\": " << e.choice.schedule << ", \"us_per_bootstrap\": " << e.choice.us_per_bootstrap
              << ", \"batch\": " << e.choice.batch << ", \"candidates\": " << e.choice.candidates << "}"
              << (i + 1 < entries.size() ? "," : "") << "\n";
        }
        f << "]\n";
        if (!f) return false;
    }
    return std::rename(tmp.c_str(), file.c_str()) == 0;
}

bool tune_cache_lookup(const cbs_context* c, const char* path, cbs_tune_choice* out) {
    const std::string file = cache_file(path);
    if (file.empty()) return false;
    const std::string key = param_key(c);
    // the entry of the largest bucket within the context's max_batch, else the smallest bucket
    const uint32_t want = batch_bucket(c->max_batch);
    const CacheEntry* fit = nullptr;
    const CacheEntry* smallest = nullptr;
    const auto entries = read_cache(file);
    for (const auto& e : entries) {
        if (e.key != key) continue;
        if (e.bucket <= want && (!fit || e.bucket > fit->bucket)) fit = &e;
        if (!smallest || e.bucket < smallest->bucket) smallest = &e;
    }
    const CacheEntry* best = fit ? fit : smallest;
    if (!best) return false;
    *out = best->choice;
    return true;
}

// uniform LWE-shaped inputs (the blind rotation's cost does not depend on their values)
static void synthetic_lwe(uint32_t batch, uint32_t n, uint64_t q, std::vector<uint64_t>& a, std::vector<uint64_t>& b) {
    uint64_t x = 0x243f6a8885a308d3ull;
    auto next = [&x]() {
        x ^= x << 13;
        x ^= x >> 7;
        x ^= x << 17;
        return x;
    };
    a.resize(static_cast<size_t>(batch) * n);
    b.resize(batch);
    for (auto& v : a) v = next() % q;
    for (auto& v : b) v = next() % q;
}

}  // namespace cbs

using namespace cbs;

extern "C" {

cbs_status cbs_autotune_blind_rotation(cbs_context* ctx, uint32_t batch, const char* cache_path, cbs_tune_choice* out) {
    CBS_CHECK_ARG(ctx, "autotune: null context");
    CBS_CHECK_ARG(batch >= 1 && batch <= ctx->max_batch, "autotune: batch must lie in [1, max_batch]");
    if (ctx->br_backend != CBS_BR_FFT64) {
        set_error("autotune: the blind-rotation knobs exist on the FFT64 backend (cbs_context_set_br_backend)");
        return CBS_ERR_UNSUPPORTED;
    }
    if (!ctx->keys_ready) {
        set_error("autotune: no key material (call cbs_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    cbs_context* c = ctx;
    cudaStream_t s = c->stream;
    std::vector<uint64_t> ha, hb;
    synthetic_lwe(batch, c->p.n, c->p.q_lwe, ha, hb);
    DevBuf<uint64_t> d_a, d_b;
    CBS_CUDA_TRY(d_a.upload(ha.data(), ha.size(), s));
    CBS_CUDA_TRY(d_b.upload(hb.data(), hb.size(), s));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CBS_CUDA_TRY(cudaEventCreate(&e0));
    CBS_CUDA_TRY(cudaEventCreate(&e1));
    struct Guard {
        cudaEvent_t a, b;
        ~Guard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } guard{e0, e1};

    // candidates: every grouping the context can form keys for, and both schedules where they differ
    const uint32_t keep_mb = c->br_mb, keep_schedule = c->br_schedule;
    std::vector<uint32_t> mbs;
    if (c->has_secret) mbs = {1, 2, 3, 4};
    else mbs = {keep_mb};
    cbs_tune_choice best{};
    best.us_per_bootstrap = 1e300;
    uint32_t tried = 0;
    for (uint32_t mb : mbs) {
        if (cbs_status st = cbs_context_set_br_multibit(c, mb)) return st;
        std::vector<uint32_t> schedules = {CBS_BR_SCHEDULE_DIGITWISE};
        if (mb == 2 && c->p.digits_g == 2) schedules.push_back(CBS_BR_SCHEDULE_LOCKSTEP);
        if (mb == 2 && c->p.digits_g == 2 && c->p.N == 2048 && batch >= 2) schedules.push_back(CBS_BR_SCHEDULE_PAIRED);
        for (uint32_t sch : schedules) {
            c->br_schedule = sch;
            if (cbs_status st = run_blind_rotate(c, d_a.p, d_b.p, batch, c->p.n, c->d_mv.p, s, false)) return st;
            CBS_CUDA_TRY(cudaEventRecord(e0, s));
            for (int r = 0; r < 2; ++r)
                if (cbs_status st = run_blind_rotate(c, d_a.p, d_b.p, batch, c->p.n, c->d_mv.p, s, false)) return st;
            CBS_CUDA_TRY(cudaEventRecord(e1, s));
            CBS_CUDA_TRY(cudaEventSynchronize(e1));
            float ms = 0;
            CBS_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
            const double us = ms * 1e3 / 2.0 / batch;
            ++tried;
            if (us < best.us_per_bootstrap) {
                best.mb = mb;
                best.schedule = sch;
                best.us_per_bootstrap = us;
            }
        }
    }
    best.batch = batch;
    best.candidates = tried;
    // apply the winner (as the context's tuned choice, not as an explicit caller setting)
    c->br_schedule = keep_schedule;
    if (cbs_status st = cbs_context_set_br_multibit(c, best.mb)) return st;
    c->mb_explicit = false;
    c->has_tuned = true;
    c->tuned = best;
    if (out) *out = best;

    const std::string file = cache_file(cache_path);
    if (!file.empty()) {
        auto entries = read_cache(file);
        const std::string key = param_key(c);
        const uint32_t bucket = batch_bucket(batch);
        bool replaced = false;
        for (auto& e : entries)
            if (e.key == key && e.bucket == bucket) {
                e.choice = best;
                replaced = true;
            }
        if (!replaced) entries.push_back(CacheEntry{key, bucket, best});
        if (!write_cache(file, entries)) {
            set_error("autotune: the choice was applied but the cache " + file + " could not be written: " +
                      std::strerror(errno));
            return CBS_ERR_UNSUPPORTED;
        }
    }
    return CBS_OK;
}

}  // extern "C"
