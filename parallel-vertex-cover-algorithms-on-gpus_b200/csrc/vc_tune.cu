// vc_tune.cu -- the autotuner: for each size class of graphs, the launch shape
// with the highest measured tree-node rate on this device.
//
// The reference sizes its one launch with a fixed rule
// (setBlockDimAndUseGlobalMemoryAutoWorkListSize, src/auxFunctions.cpp:469-578:
// the smallest power-of-two block whose per-block arrays fit shared memory, the
// global-memory variant when none does, and a worklist size halved until it
// fits).  Here the library's built-in rules pick the kernel by graph size; the
// tuner measures, per size class, the alternatives those rules leave open:
//   * warp search units or one 512-thread CTA per search unit (the CSR class,
//     above 1024 vertices),
//   * warps per CTA (2, 4, 8; 6 stands for 8 where a 1024-vertex graph's
//     adjacency leaves no room) -- how many search units share one staged graph
//     and one CTA pool (the dense classes up to 1024 vertices),
//   * CTA pool slots per warp (1, 2, 4) -- the depth of the shared-memory stack
//     of donated subtrees,
//   * the ring threshold: work goes to the global ring while idle CTAs minus
//     the records already queued exceed -64, -16, 0, 4 or 32 (a negative
//     threshold keeps a surplus of records queued for CTAs that go idle),
//   * the donation order when an idle sibling warp and an idle CTA both wait:
//     the CTA pool first, or the ring first,
// on seeded calibration graphs of the class (G(n, p) of the batched family's
// degrees, sizes spread over the class), each candidate timed for a fixed time
// slice, and installs the winner in the device's table; later solves of that
// class use it.  vc_set_tuning installs a table saved from an earlier run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "vc_host.h"
#include "vcgpu.h"

using namespace vcg;
using namespace vch;

namespace {

// splitmix64: a small seeded generator for the calibration graphs
struct Rng {
    uint64_t s;
    uint64_t next()
    {
        uint64_t z = (s += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    uint32_t below(uint32_t n) { return (uint32_t)(uniform() * n) % n; }
};

struct CalGraph {
    uint32_t n;
    std::vector<uint32_t> rp, col;
};

// G(n, m) with m = n * d / 2 distinct edges, CSR with sorted rows.
CalGraph gnm(Rng &r, uint32_t n, double d)
{
    const uint64_t want = std::min<uint64_t>((uint64_t)(n * d / 2), (uint64_t)n * (n - 1) / 2);
    std::vector<uint64_t> keys;
    while (keys.size() < want) {  // draw pairs, drop duplicates, repeat until enough remain
        const uint64_t draw = want - keys.size() + want / 8 + 8;
        for (uint64_t i = 0; i < draw; ++i) {
            uint32_t u = r.below(n), v = r.below(n);
            if (u == v) continue;
            if (u > v) std::swap(u, v);
            keys.push_back(((uint64_t)u << 32) | v);
        }
        std::sort(keys.begin(), keys.end());
        keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    }
    keys.resize(want);
    CalGraph g;
    g.n = n;
    std::vector<uint32_t> deg(n, 0);
    for (uint64_t k : keys) { deg[k >> 32]++; deg[k & 0xffffffffu]++; }
    g.rp.assign(n + 1, 0);
    for (uint32_t v = 0; v < n; ++v) g.rp[v + 1] = g.rp[v] + deg[v];
    g.col.assign(g.rp[n], 0);
    std::vector<uint32_t> pos(g.rp.begin(), g.rp.end() - 1);
    for (uint64_t k : keys) {
        const uint32_t u = (uint32_t)(k >> 32), v = (uint32_t)k;
        g.col[pos[u]++] = v;
        g.col[pos[v]++] = u;
    }
    for (uint32_t v = 0; v < n; ++v) std::sort(g.col.begin() + g.rp[v], g.col.begin() + g.rp[v + 1]);
    return g;
}

struct ClassSpec {
    uint32_t count, n_lo, n_hi;
    double d_lo, d_hi;
};

// Calibration graphs per class: enough to occupy every SM for the time slice.
const ClassSpec kSpec[kTuneClasses] = {
    {2048, 40, 64, 3.0, 12.0}, {1024, 90, 128, 3.0, 12.0}, {512, 150, 255, 3.0, 12.0},
    {256, 300, 640, 2.5, 4.0}, {128, 700, 1024, 2.5, 4.0}, {16, 2000, 8000, 2.5, 3.5},
};

// Runs the class's calibration batch with one candidate shape for `slice_s`
// seconds (the launch's time limit; each graph also has a node limit) and
// returns its tree nodes per second.
double measure(Ctx &c, const std::vector<CalGraph> &gs, const Tune &cand, double slice_s, bool wide, bool half)
{
    uint64_t rows = 0, cols = 0;
    for (const auto &g : gs) { rows += g.n + 1; cols += g.col.size(); }
    if (c.rp.ensure(4 * rows) || c.col.ensure(4 * std::max<uint64_t>(cols, 1))) return -1;
    Job job;
    uint64_t ro = 0, co = 0;
    for (size_t i = 0; i < gs.size(); ++i) {
        const CalGraph &g = gs[i];
        cudaMemcpyAsync((uint32_t *)c.rp.p + ro, g.rp.data(), 4 * (g.n + 1), cudaMemcpyHostToDevice, c.stream);
        if (!g.col.empty())
            cudaMemcpyAsync((uint32_t *)c.col.p + co, g.col.data(), 4 * g.col.size(), cudaMemcpyHostToDevice, c.stream);
        InstDesc d;
        memset(&d, 0, sizeof(d));
        d.n = g.n;
        d.nw = (g.n + 31) / 32;
        d.row_off = ro;
        d.col_off = co;
        d.mode = kModeMVC;
        d.init_best = g.n + 1;
        d.node_limit = 1u << 18;
        d.key = (uint32_t)i;
        d.m2 = (uint32_t)g.col.size();
        job.desc.push_back(d);
        ro += g.n + 1;
        co += g.col.size();
    }
    job.d_rp = (const uint32_t *)c.rp.p;
    job.d_col = (const uint32_t *)c.col.p;
    job.time_limit_s = slice_s;
    job.wide = wide;
    job.half = half;
    job.tune = &cand;
    if (run_job(c, job, c.stream) != VC_OK) return -1;
    uint64_t nodes = 0;
    for (const auto &s : job.st) nodes += s.nodes;
    return job.kernel_ms > 0 ? nodes / (job.kernel_ms * 1e-3) : -1;
}

constexpr uint32_t kTuneWords = 7;  // per class

void pack(const Tune *t, uint32_t *w)
{
    for (int i = 0; i < kTuneClasses; ++i) {
        uint32_t *o = w + kTuneWords * i;
        o[0] = t[i].set;
        o[1] = t[i].cta_units;
        o[2] = t[i].warps;
        o[3] = t[i].pool;
        memcpy(&o[4], &t[i].ring_bias, 4);
        memcpy(&o[5], &t[i].nodes_per_s, 4);
        o[6] = t[i].ring_first;
    }
}

bool valid(const Tune &t)
{
    return (t.warps == 2 || t.warps == 4 || t.warps == 8) && (t.pool >= 1 && t.pool <= 4) && t.cta_units <= 1 &&
           t.ring_bias >= -(1 << 20) && t.ring_bias <= (1 << 20) && t.ring_first <= 1;
}

}  // namespace

// Measures launch shapes per size class on this device and installs the
// fastest (see the file comment).  slice_s is the time each candidate runs
// (0 = 0.3 s); about a dozen candidates per class.  table (optional, 42 words)
// receives the chosen shapes: per class set, cta_units, warps, pool slots per
// warp, ring threshold (int32), measured tree nodes/s (float bits), ring first.
extern "C" vc_status vc_autotune(int32_t device, double slice_s, uint32_t *table, uint32_t max_words)
{
    DeviceGuard dg;
    vc_status err;
    Ctx *c = get_ctx(device, &err);
    if (!c) return err;
    std::lock_guard<std::mutex> lk(c->mu);
    if (slice_s <= 0) slice_s = 0.3;
    Tune best_all[kTuneClasses];
    for (int k = 0; k < kTuneClasses; ++k) {
        const ClassSpec &sp = kSpec[k];
        Rng r{0x5eed0000ull + (uint64_t)k};
        std::vector<CalGraph> gs;
        for (uint32_t i = 0; i < sp.count; ++i) {
            const uint32_t n = sp.n_lo + r.below(sp.n_hi - sp.n_lo + 1);
            const double d = sp.d_lo + (sp.d_hi - sp.d_lo) * r.uniform();
            gs.push_back(gnm(r, n, d));
        }
        const bool wide = k == 3, half = k == 4;  // the kernels the class's graphs take
        std::vector<Tune> cands;
        if (k <= 4) {
            for (uint32_t w : {2u, 4u, 8u})
                for (uint32_t p : {1u, 2u, 4u}) cands.push_back(Tune{1, 0, w, p, 0, 0});
        } else {
            for (uint32_t w : {4u, 8u}) cands.push_back(Tune{1, 0, w, 2, 0, 0});
            cands.push_back(Tune{1, 1, 8, 2, 0, 0});
        }
        Tune best{};
        double best_rate = -1;
        for (Tune &t : cands) {
            const double rate = measure(*c, gs, t, slice_s, wide, half);
            if (rate > best_rate) { best_rate = rate; best = t; }
        }
        for (int32_t bias : {-64, -16, 4, 32}) {  // then the ring threshold, with the best shape
            Tune t = best;
            t.ring_bias = bias;
            const double rate = measure(*c, gs, t, slice_s, wide, half);
            if (rate > best_rate) { best_rate = rate; best = t; }
        }
        {  // then the donation order
            Tune t = best;
            t.ring_first = 1;
            const double rate = measure(*c, gs, t, slice_s, wide, half);
            if (rate > best_rate) { best_rate = rate; best = t; }
        }
        if (best_rate <= 0) return VC_ERR_CUDA;
        best.nodes_per_s = (float)best_rate;
        best_all[k] = best;
    }
    for (int k = 0; k < kTuneClasses; ++k) c->tune[k] = best_all[k];
    if (table && max_words >= kTuneWords * kTuneClasses) pack(c->tune, table);
    return VC_OK;
}

// Installs a table from an earlier vc_autotune on this device (words as
// vc_autotune writes them; a class with set = 0 goes back to the built-in rules).
extern "C" vc_status vc_set_tuning(int32_t device, const uint32_t *table, uint32_t words)
{
    DeviceGuard dg;
    if (!table || words < kTuneWords * kTuneClasses) return VC_ERR_INVALID;
    Tune t[kTuneClasses];
    for (int i = 0; i < kTuneClasses; ++i) {
        const uint32_t *w = table + kTuneWords * i;
        t[i].set = w[0] ? 1 : 0;
        t[i].cta_units = w[1];
        t[i].warps = w[2];
        t[i].pool = w[3];
        memcpy(&t[i].ring_bias, &w[4], 4);
        memcpy(&t[i].nodes_per_s, &w[5], 4);
        t[i].ring_first = w[6];
        if (t[i].set && !valid(t[i])) return VC_ERR_INVALID;
    }
    vc_status err;
    Ctx *c = get_ctx(device, &err);
    if (!c) return err;
    std::lock_guard<std::mutex> lk(c->mu);
    for (int i = 0; i < kTuneClasses; ++i) c->tune[i] = t[i];
    return VC_OK;
}
