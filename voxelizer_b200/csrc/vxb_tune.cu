// Launch-shape autotuner (see vxb_tune.h).

#include "vxb.h"
#include "vxb_host.h"
#include "vxb_tune.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>

namespace vxb {

namespace {

// Candidate k of every knob; candidate 0 is the untuned shape.
const uint32_t kSurfBlocks[kTuneCandidates] = {16, 16, 8};
const uint32_t kSurfBatch[kTuneCandidates] = {8, 8, 16};
const uint32_t kSurfQueue[kTuneCandidates] = {0, 1, 1};
const uint32_t kMerge[kTuneCandidates] = {0, 8, 4};
const uint32_t kEmit[kTuneCandidates] = {16, 8, 32};
const uint32_t kToggle[kTuneCandidates] = {3, 3, 6};
const uint32_t kToggleQueue[kTuneCandidates] = {0, 1, 1};

LaunchShape candidate(int k) {
    LaunchShape s;
    s.surfBlocksPerSm = kSurfBlocks[k];
    s.surfBatch = kSurfBatch[k];
    s.mergeBlocksPerSm = kMerge[k];
    s.emitBlocksPerSm = kEmit[k];
    s.toggleBlocksPerSm = kToggle[k];
    s.surfQueue = kSurfQueue[k];
    s.toggleQueue = kToggleQueue[k];
    return s;
}

struct Entry {
    bool settled = false;
    LaunchShape best;
    uint32_t issued = 0;
    double sum[kKnobs][kTuneCandidates] = {};
    uint32_t n[kKnobs][kTuneCandidates] = {};
    // Second phase: the settled shapes with each material-key strategy.
    bool mergePhase = false;
    uint32_t issuedMerge = 0;
    double span[kMergeCandidates] = {};
    uint32_t nSpan[kMergeCandidates] = {};
};

struct State {
    std::mutex mu;
    int mode = kTuneOff;
    std::string path;
    std::map<std::string, Entry> buckets;
};

State& state() {
    static State* s = new State;   // never destroyed (used from static destructors of callers)
    return *s;
}

constexpr int kFieldCount = 8;
const char* const kFields[kFieldCount] = {"surf_blocks_per_sm", "surf_batch", "merge_blocks_per_sm",
                                          "emit_blocks_per_sm", "toggle_blocks_per_sm", "surf_queue",
                                          "toggle_queue", "surf_merge"};

uint32_t* field(LaunchShape& s, int i) {
    uint32_t* f[kFieldCount] = {&s.surfBlocksPerSm,   &s.surfBatch, &s.mergeBlocksPerSm, &s.emitBlocksPerSm,
                                &s.toggleBlocksPerSm, &s.surfQueue, &s.toggleQueue,      &s.surfMerge};
    return f[i];
}

bool validShape(const LaunchShape& s) {
    auto in = [](uint32_t v, const uint32_t* c) {
        for (int k = 0; k < kTuneCandidates; ++k)
            if (c[k] == v) return true;
        return false;
    };
    return in(s.surfBlocksPerSm, kSurfBlocks) && in(s.surfBatch, kSurfBatch) && in(s.mergeBlocksPerSm, kMerge) &&
           in(s.emitBlocksPerSm, kEmit) && in(s.toggleBlocksPerSm, kToggle) && in(s.surfQueue, kSurfQueue) &&
           in(s.toggleQueue, kToggleQueue) && s.surfMerge < (uint32_t)kMergeCandidates;
}

std::string jsonLocked(const State& st) {
    std::string out = "{\n";
    bool first = true;
    for (const auto& kv : st.buckets) {
        if (!kv.second.settled) continue;
        LaunchShape s = kv.second.best;
        out += first ? "  \"" : ",\n  \"";
        out += kv.first + "\": {";
        for (int i = 0; i < kFieldCount; ++i) {
            char item[96];
            snprintf(item, sizeof(item), "%s\"%s\": %u", i ? ", " : "", kFields[i], *field(s, i));
            out += item;
        }
        out += "}";
        first = false;
    }
    out += "\n}\n";
    return out;
}

void saveLocked(const State& st) {
    if (st.path.empty()) return;
    FILE* f = fopen(st.path.c_str(), "w");
    if (!f) return;
    const std::string text = jsonLocked(st);
    fwrite(text.data(), 1, text.size(), f);
    fclose(f);
}

// Reads the lines `"bucket": {"field": value, ...}` of a cache file written
// by saveLocked; entries with unknown shapes are skipped.
void loadLocked(State& st) {
    if (st.path.empty()) return;
    FILE* f = fopen(st.path.c_str(), "r");
    if (!f) return;
    char line[1024];
    while (fgets(line, sizeof(line), f)) {
        const char* q0 = strchr(line, '"');
        if (!q0) continue;
        const char* q1 = strchr(q0 + 1, '"');
        if (!q1 || !strchr(q1, '{')) continue;
        const std::string key(q0 + 1, q1);
        LaunchShape s;
        bool ok = true;
        for (int i = 0; i < kFieldCount && ok; ++i) {
            const std::string name = std::string("\"") + kFields[i] + "\":";
            const char* p = strstr(q1, name.c_str());
            unsigned v = 0;
            ok = p && sscanf(p + name.size(), " %u", &v) == 1;
            if (ok) *field(s, i) = v;
        }
        if (!ok || !validShape(s)) continue;
        Entry& e = st.buckets[key];
        e.settled = true;
        e.best = s;
    }
    fclose(f);
}

}  // namespace

std::string tuneBucket(uint32_t workTriangles, uint64_t gridWords, int nodeKind, bool materials) {
    auto lg = [](uint64_t v) { return v ? (int)std::floor(std::log2((double)v)) : 0; };
    char b[64];
    snprintf(b, sizeof(b), "t%d-w%d-k%d-m%d", lg(workTriangles), lg(gridWords), nodeKind, materials ? 1 : 0);
    return b;
}

LaunchShape tunePick(const std::string& bucket, int* trial, bool allowTrial) {
    *trial = -1;
    State& st = state();
    std::lock_guard<std::mutex> lock(st.mu);
    if (st.mode == kTuneOff) return LaunchShape();
    auto it = st.buckets.find(bucket);
    if (st.mode == kTuneFrozen) return (it != st.buckets.end() && it->second.settled) ? it->second.best : LaunchShape();
    Entry& e = st.buckets[bucket];
    if (e.settled) return e.best;
    if (!allowTrial) return LaunchShape();
    if (e.mergePhase) {
        const int m = (int)(e.issuedMerge++ % kMergeCandidates);
        *trial = kTuneCandidates + m;
        LaunchShape s = e.best;
        s.surfMerge = (uint32_t)m;
        return s;
    }
    const int k = (int)(e.issued++ % kTuneCandidates);
    *trial = k;
    return candidate(k);
}

void tuneReport(const std::string& bucket, int trial, const float* ms) {
    if (trial < 0 || trial >= kTuneCandidates + kMergeCandidates) return;
    State& st = state();
    std::lock_guard<std::mutex> lock(st.mu);
    if (st.mode != kTuneOn) return;
    Entry& e = st.buckets[bucket];
    if (e.settled) return;
    if (trial >= kTuneCandidates) {
        if (!e.mergePhase) return;
        const int m = trial - kTuneCandidates;
        if (ms[kKnobSurfaceSpan] >= 0.0f) {
            e.span[m] += ms[kKnobSurfaceSpan];
            e.nSpan[m] += 1;
        }
        for (int k = 0; k < kMergeCandidates; ++k)
            if (e.nSpan[k] < (uint32_t)kTuneSamples) return;
        e.best.surfMerge = e.span[1] / e.nSpan[1] < e.span[0] / e.nSpan[0] ? 1u : 0u;
        e.settled = true;
        saveLocked(st);
        return;
    }
    if (e.mergePhase) return;
    for (int kn = 0; kn < kKnobs; ++kn)
        if (ms[kn] >= 0.0f) {
            e.sum[kn][trial] += ms[kn];
            e.n[kn][trial] += 1;
        }
    // Settled once every candidate has its samples (a knob whose kernel
    // never runs in this bucket keeps candidate 0).
    for (int k = 0; k < kTuneCandidates; ++k) {
        uint32_t most = 0;
        for (int kn = 0; kn < kKnobs; ++kn) most = std::max(most, e.n[kn][k]);
        if (most < (uint32_t)kTuneSamples) return;
    }
    LaunchShape best;
    for (int kn = 0; kn < kKnobSurfaceSpan; ++kn) {
        int arg = 0;
        double bestMs = HUGE_VAL;
        for (int k = 0; k < kTuneCandidates; ++k) {
            if (!e.n[kn][k]) continue;
            const double avg = e.sum[kn][k] / e.n[kn][k];
            if (avg < bestMs) {
                bestMs = avg;
                arg = k;
            }
        }
        const LaunchShape c = candidate(arg);
        switch (kn) {
        case kKnobSurface:
            best.surfBlocksPerSm = c.surfBlocksPerSm;
            best.surfBatch = c.surfBatch;
            best.surfQueue = c.surfQueue;
            break;
        case kKnobMerge: best.mergeBlocksPerSm = c.mergeBlocksPerSm; break;
        case kKnobEmit: best.emitBlocksPerSm = c.emitBlocksPerSm; break;
        default:
            best.toggleBlocksPerSm = c.toggleBlocksPerSm;
            best.toggleQueue = c.toggleQueue;
            break;
        }
    }
    e.best = best;
    // Buckets with a surface pass go on to the material-key strategies.
    bool surface = false;
    for (int k = 0; k < kTuneCandidates; ++k) surface |= e.n[kKnobSurfaceSpan][k] > 0;
    if (surface) {
        e.mergePhase = true;
        return;
    }
    e.settled = true;
    saveLocked(st);
}

int tuneSetMode(int mode, const char* cachePath) {
    if (mode < kTuneOff || mode > kTuneFrozen) return failf(VXB_EINVAL, "autotune mode must be 0, 1 or 2");
    State& st = state();
    std::lock_guard<std::mutex> lock(st.mu);
    st.mode = mode;
    st.path = cachePath ? cachePath : "";
    st.buckets.clear();
    loadLocked(st);
    return 0;
}

int tuneMode() {
    State& st = state();
    std::lock_guard<std::mutex> lock(st.mu);
    return st.mode;
}

uint32_t tuneSettled() {
    State& st = state();
    std::lock_guard<std::mutex> lock(st.mu);
    uint32_t n = 0;
    for (const auto& kv : st.buckets) n += kv.second.settled ? 1u : 0u;
    return n;
}

std::string tuneJson() {
    State& st = state();
    std::lock_guard<std::mutex> lock(st.mu);
    return jsonLocked(st);
}

}  // namespace vxb

extern "C" {

vxb_status vxb_set_autotune(int mode, const char* cache_path) { return vxb::tuneSetMode(mode, cache_path); }

vxb_status vxb_autotune_state(uint32_t* settled, char* json, uint64_t json_bytes) {
    if (settled) *settled = vxb::tuneSettled();
    if (json && json_bytes) {
        const std::string t = vxb::tuneJson();
        const size_t n = std::min((size_t)json_bytes - 1, t.size());
        memcpy(json, t.data(), n);
        json[n] = 0;
    }
    return VXB_OK;
}

}  // extern "C"
