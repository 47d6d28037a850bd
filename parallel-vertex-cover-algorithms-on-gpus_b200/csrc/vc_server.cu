// vc_server.cu -- continuous-batching server (vc_server_* in include/vcgpu.h).
//
// A server has one or two lanes.  A lane is one persistent search kernel on its
// own stream that keeps the search state of every admitted request on the
// device.  When requests may exceed 255 vertices, small requests (the dense
// bitset kernel, about three times the node rate) and large ones (the CSR
// kernel) get a lane each; the two grids are sized so that both kernels are
// resident side by side on every SM (3 dense CTAs per SM plus one CSR CTA in
// the registers and shared memory left over), and neither kernel ever waits on
// the other.  Each lane has a host thread (the request loop) that:
//   * admits submitted requests into device slots while a slot and arena memory
//     are free (admission by the request's device bytes: its CSR plus its cover
//     bitmap; the search state itself lives in the kernel's fixed per-SU
//     workspaces, sized at creation for the largest request the lane takes),
//     copies the graph and its descriptor on a copy stream, and publishes the
//     slot id on the device submission queue.  Arena space is a first-fit free
//     list: a finished request's block is reused for the next one while the
//     kernel runs (the kernels read server graphs around L1, so no SM keeps a
//     line of the block's previous graph), so a full arena only holds requests
//     back until blocks free up -- the kernel never stops to empty it;
//   * relaunches the kernel when it has exited (it exits after an idle period)
//     and work is waiting;
//   * collects results, which the SU that returns a request's last work token
//     writes into host-mapped memory, and frees the slot.
// Requests that arrive while others run are claimed by idle search units at
// once, so their work overlaps on the device with the requests in flight.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "vc_host.h"

using namespace vcg;
using namespace vch;

namespace {

struct Pending {
    uint64_t ticket;
    uint32_t n, m;
    std::vector<uint32_t> rp, col;
    vc_request req;
    std::chrono::steady_clock::time_point t_submit;
};

struct SlotInfo {
    uint64_t ticket = 0;
    uint32_t n = 0, ub = 0, mode = 0, init_best = 0;
    uint64_t arena_off = 0, arena_len = 0;  // the request's arena block (bytes)
    std::chrono::steady_clock::time_point t_submit;
};

struct Done {
    vc_status status;
    uint32_t size, decision, has_cover;
    uint64_t nodes;
    float total_ms;
    std::vector<uint8_t> cover;
};

constexpr uint32_t kSubQ = 1u << 16;  // submission queue entries (power of two)

}  // namespace

struct SrvLane {
    int dev = -1;
    Ctx *ctx = nullptr;
    cudaStream_t kstream = nullptr, cstream = nullptr;
    uint32_t slots = 0, nw_max = 0, max_n = 0;
    uint64_t arena_cap = 0;
    Plan pl;
    uint32_t q = 0;
    DevBuf desc, st, covers, ctl, seq, data, gws, subq, arena;
    uint32_t *h_res = nullptr, *d_res = nullptr;
    uint32_t res_words = 0;
    // host state (guarded by mu)
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Pending> pending;
    std::vector<uint32_t> free_slots;
    std::vector<SlotInfo> info;
    std::unordered_map<uint64_t, uint32_t> inflight;  // ticket -> slot
    std::unordered_map<uint64_t, Done> done;
    std::deque<uint64_t> ready;  // finished tickets not yet reported by vc_server_completed
    uint64_t next_ticket = 1;
    std::map<uint64_t, uint64_t> arena_free;  // free arena blocks: byte offset -> length
    uint64_t sub_tail = 0;
    bool running = false;
    bool resident = false;  // launched at creation and kept running (no idle exit)
    bool draining = false;  // a resident kernel asked to stop before its time limit
    std::chrono::steady_clock::time_point t_launch;
    bool stop = false;
    bool discard_queue = false;
    vc_status fatal = VC_OK;
    std::thread loop;
};

namespace {

vc_status launch_kernel(SrvLane *s)
{
    // fresh control words, keeping the submission queue's head and tail
    unsigned long long ctl[kCtlWords];
    memset(ctl, 0, sizeof(ctl));
    unsigned long long head = 0;
    if (cudaMemcpy(&head, (unsigned long long *)s->ctl.p + kCursor, sizeof(head), cudaMemcpyDeviceToHost) != cudaSuccess)
        return VC_ERR_CUDA;
    // after a launch stopped at its time limit, unclaimed submissions were failed
    // on the host: drop them from the queue
    ctl[kCursor] = s->discard_queue ? s->sub_tail : head;
    s->discard_queue = false;
    ctl[kSubTail] = s->sub_tail;
    if (cudaMemcpyAsync(s->ctl.p, ctl, sizeof(ctl), cudaMemcpyHostToDevice, s->cstream) != cudaSuccess) return VC_ERR_CUDA;
    std::vector<unsigned long long> seq(s->q);
    for (uint32_t i = 0; i < s->q; ++i) seq[i] = i;
    if (cudaMemcpyAsync(s->seq.p, seq.data(), sizeof(unsigned long long) * s->q, cudaMemcpyHostToDevice, s->cstream) !=
        cudaSuccess)
        return VC_ERR_CUDA;
    if (cudaStreamSynchronize(s->cstream) != cudaSuccess) return VC_ERR_CUDA;
    Params P;
    memset(&P, 0, sizeof(P));
    P.row_ptr = (const uint32_t *)s->arena.p;
    P.col = (const uint32_t *)s->arena.p;
    P.inst = (const InstDesc *)s->desc.p;
    P.st = (InstState *)s->st.p;
    P.covers = (uint32_t *)s->covers.p;
    P.count = 0;
    P.num_su = s->pl.num_su;
    P.ctl = (unsigned long long *)s->ctl.p;
    P.pool_seq = (unsigned long long *)s->seq.p;
    P.pool_data = (uint32_t *)s->data.p;
    P.q_mask = s->q - 1;
    P.stride = s->pl.stride;
    P.np = s->pl.np;
    P.su_bytes = s->pl.su_bytes;
    P.cta_slots = s->pl.cta_slots;
    P.gws = s->pl.global_ws ? (uint8_t *)s->gws.p : nullptr;
    P.stats = nullptr;
    P.time_limit_ns = 600ull * 1000000000ull;
    P.server = 1;
    P.subq_mask = kSubQ - 1;
    P.subq = (const uint32_t *)s->subq.p;
    P.hres = s->d_res;
    P.hres_words = s->res_words;
    P.idle_ns = s->resident ? (1ull << 62) : 200ull * 1000000ull;
    void *args[] = {&P};
    // the batched path may have lowered the kernel's shared-memory limit; and
    // SMs hosting this lane keep their largest shared-memory configuration, so
    // the other lanes' CTAs can be placed beside it
    if (cudaFuncSetAttribute(s->pl.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->pl.smem) != cudaSuccess ||
        cudaFuncSetAttribute(s->pl.fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess)
        return VC_ERR_CUDA;
    if (cudaLaunchCooperativeKernel(s->pl.fn, dim3(s->pl.grid), dim3(s->pl.block), args, s->pl.smem, s->kstream) !=
        cudaSuccess)
        return VC_ERR_CUDA;
    s->running = true;
    s->t_launch = std::chrono::steady_clock::now();
    return VC_OK;
}

// Waits (bounded) until every CTA of the lane's launch has started: the next
// lane's kernel is then placed in what this one leaves free on each SM.
bool wait_resident(SrvLane *s)
{
    const auto t0 = std::chrono::steady_clock::now();
    while (std::chrono::steady_clock::now() - t0 < std::chrono::seconds(5)) {
        unsigned long long n = 0;
        if (cudaMemcpy(&n, (unsigned long long *)s->ctl.p + kStarted, sizeof(n), cudaMemcpyDeviceToHost) != cudaSuccess)
            return false;
        if (n >= s->pl.grid) return true;
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
    return false;
}

// First-fit block of `bytes` (a multiple of 256) from the lane's arena; false
// if no free block is large enough.
bool arena_alloc(SrvLane *s, uint64_t bytes, uint64_t &off)
{
    for (auto it = s->arena_free.begin(); it != s->arena_free.end(); ++it) {
        if (it->second < bytes) continue;
        off = it->first;
        const uint64_t rest = it->second - bytes;
        s->arena_free.erase(it);
        if (rest) s->arena_free.emplace(off + bytes, rest);
        return true;
    }
    return false;
}

// Returns a block to the free list, merged with free neighbours.
void arena_release(SrvLane *s, uint64_t off, uint64_t len)
{
    if (!len) return;
    auto next = s->arena_free.lower_bound(off);
    if (next != s->arena_free.end() && next->first == off + len) {
        len += next->second;
        next = s->arena_free.erase(next);
    }
    if (next != s->arena_free.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == off) {
            prev->second += len;
            return;
        }
    }
    s->arena_free.emplace(off, len);
}

// Admits pending requests into free slots (called by the loop, lock held):
// copies their graphs and descriptors, then publishes their slot ids on the
// submission queue with one synchronisation.  Returns the number admitted.
uint32_t admit(SrvLane *s, std::unique_lock<std::mutex> &lk, bool &arena_full)
{
    arena_full = false;
    std::vector<Pending> batch;
    std::vector<uint32_t> published;
    std::vector<InstDesc> descs;
    while (!s->pending.empty() && !s->free_slots.empty() && batch.size() < 256) {
        Pending &p = s->pending.front();
        const uint64_t rows = p.n + 1, cols = std::max<uint64_t>(2ull * p.m, 1);
        const uint64_t bytes = ((rows + cols) * 4 + 255) / 256 * 256;
        if (bytes > s->arena_cap) {  // can never fit
            s->done.emplace(p.ticket, Done{VC_ERR_NOMEM, 0, 0, 0, 0, 0.0f, {}});
            s->ready.push_back(p.ticket);
            s->pending.pop_front();
            continue;
        }
        uint64_t boff = 0;
        if (!arena_alloc(s, bytes, boff)) { arena_full = true; break; }
        const uint32_t slot = s->free_slots.back();
        s->free_slots.pop_back();
        const uint64_t off = boff / 4;
        InstDesc d;
        memset(&d, 0, sizeof(d));
        d.n = p.n;
        d.nw = (p.n + 31) / 32;
        d.row_off = off;
        d.col_off = off + rows;
        d.mode = p.req.instance == VC_PVC ? kModePVC : kModeMVC;
        d.k = std::min<uint32_t>(p.req.k, p.n);
        const uint32_t ub = p.req.instance == VC_MVC ? p.req.ub : 0;
        d.init_best = d.mode == kModePVC ? p.n + 1 : ((ub && ub < p.n) ? ub : p.n) + 1;
        d.cover_off = slot * s->nw_max;
        d.node_limit = p.req.node_limit;
        d.key = (uint32_t)p.ticket;
        d.m2 = kNone;  // host-validated graphs
        descs.push_back(d);
        HostResult *hr = reinterpret_cast<HostResult *>(s->h_res + (size_t)slot * s->res_words);
        hr->done = 0;  // the previous occupant's record
        SlotInfo &si = s->info[slot];
        si.ticket = p.ticket;
        si.n = p.n;
        si.ub = ub;
        si.mode = d.mode;
        si.init_best = d.init_best;
        si.t_submit = p.t_submit;
        si.arena_off = boff;
        si.arena_len = bytes;
        s->inflight.emplace(p.ticket, slot);
        published.push_back(slot);
        batch.push_back(std::move(p));
        s->pending.pop_front();
    }
    if (batch.empty()) return 0;
    for (size_t i = 0; i < batch.size(); ++i) {
        const Pending &p = batch[i];
        const InstDesc &d = descs[i];
        uint32_t *base = (uint32_t *)s->arena.p + d.row_off;
        cudaMemcpyAsync(base, p.rp.data(), 4ull * (p.n + 1), cudaMemcpyHostToDevice, s->cstream);
        if (p.m) cudaMemcpyAsync((uint32_t *)s->arena.p + d.col_off, p.col.data(), 8ull * p.m, cudaMemcpyHostToDevice, s->cstream);
        cudaMemcpyAsync((InstDesc *)s->desc.p + published[i], &descs[i], sizeof(InstDesc), cudaMemcpyHostToDevice, s->cstream);
    }
    for (size_t i = 0; i < published.size(); ++i)
        cudaMemcpyAsync((uint32_t *)s->subq.p + ((s->sub_tail + i) & (kSubQ - 1)), &published[i], 4,
                        cudaMemcpyHostToDevice, s->cstream);
    // graphs, descriptors and queue entries must land before the tail that publishes them
    if (cudaStreamSynchronize(s->cstream) != cudaSuccess) { s->fatal = VC_ERR_CUDA; return 0; }
    s->sub_tail += published.size();
    unsigned long long tail = s->sub_tail;
    cudaMemcpyAsync((unsigned long long *)s->ctl.p + kSubTail, &tail, sizeof(tail), cudaMemcpyHostToDevice, s->cstream);
    if (cudaStreamSynchronize(s->cstream) != cudaSuccess) s->fatal = VC_ERR_CUDA;
    (void)lk;
    return (uint32_t)batch.size();
}

// Collects finished requests from the host-mapped records (lock held).
uint32_t collect(SrvLane *s)
{
    uint32_t got = 0;
    std::vector<uint64_t> finished;
    for (auto &kv : s->inflight) {
        const uint32_t slot = kv.second;
        const HostResult *hr = reinterpret_cast<const HostResult *>(s->h_res + (size_t)slot * s->res_words);
        const unsigned long long done = *reinterpret_cast<const volatile unsigned long long *>(&hr->done);
        if (done != (uint32_t)kv.first) continue;
        std::atomic_thread_fence(std::memory_order_acquire);
        const SlotInfo &si = s->info[slot];
        Done d;
        const uint32_t fl = hr->flags;
        if (fl & kError) d.status = VC_ERR_INTERNAL;
        else if (fl & kBudget) d.status = VC_BUDGET;
        else if ((fl & kCut) || !(fl & kDone)) d.status = VC_TIMEOUT;
        else d.status = VC_OK;
        d.nodes = hr->nodes;
        d.has_cover = hr->cover_size != kNone;
        if (si.mode == kModeMVC) {
            d.decision = 1;
            d.size = hr->best < si.init_best ? hr->best : (si.ub ? si.ub : si.n);
        } else {
            d.decision = (fl & kFound) ? 1u : 0u;
            d.size = d.decision ? hr->cover_size : 0u;
        }
        d.cover.assign(si.n, 0);
        if (d.has_cover) {
            const uint32_t *w = reinterpret_cast<const uint32_t *>(hr + 1);
            for (uint32_t v = 0; v < si.n; ++v) d.cover[v] = (uint8_t)((w[v >> 5] >> (v & 31u)) & 1u);
        }
        d.total_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - si.t_submit).count();
        s->done.emplace(kv.first, std::move(d));
        s->ready.push_back(kv.first);
        finished.push_back(kv.first);
    }
    for (uint64_t t : finished) {
        const uint32_t slot = s->inflight[t];
        s->inflight.erase(t);
        s->free_slots.push_back(slot);
        arena_release(s, s->info[slot].arena_off, s->info[slot].arena_len);
        s->info[slot].arena_len = 0;
        ++got;
    }
    return got;
}

// After an abnormal kernel exit, requests still in flight get a timeout status.
void fail_inflight(SrvLane *s, vc_status st)
{
    s->discard_queue = true;
    for (auto &kv : s->inflight) {
        Done d{st, 0, 0, 0, 0, 0.0f, {}};
        s->done.emplace(kv.first, std::move(d));
        s->ready.push_back(kv.first);
        s->free_slots.push_back(kv.second);
        arena_release(s, s->info[kv.second].arena_off, s->info[kv.second].arena_len);
        s->info[kv.second].arena_len = 0;
    }
    s->inflight.clear();
}

void request_loop(SrvLane *s)
{
    cudaSetDevice(s->dev);
    std::unique_lock<std::mutex> lk(s->mu);
    uint32_t nap_us = 20;
    while (true) {
        if (s->fatal != VC_OK) {
            fail_inflight(s, s->fatal);
            for (auto &p : s->pending) {
                s->done.emplace(p.ticket, Done{s->fatal, 0, 0, 0, 0, 0.0f, {}});
                s->ready.push_back(p.ticket);
            }
            s->pending.clear();
            s->cv.notify_all();
            if (s->stop) break;
            s->cv.wait_for(lk, std::chrono::milliseconds(5));
            continue;
        }
        bool progress = false;
        if (s->running && cudaStreamQuery(s->kstream) != cudaErrorNotReady) {
            s->running = false;
            s->draining = false;
            // the kernel exited: everything it claimed has finished unless it stopped at its limit
            collect(s);
            unsigned long long abort_flag = 0;
            cudaMemcpy(&abort_flag, (unsigned long long *)s->ctl.p + kAbort, sizeof(abort_flag), cudaMemcpyDeviceToHost);
            if (abort_flag || cudaGetLastError() != cudaSuccess) fail_inflight(s, VC_TIMEOUT);
            progress = true;
        }
        if (!s->stop) {
            // a resident kernel is restarted well before its 600 s limit: it
            // drains (no admissions) and exits, and the loop relaunches it
            if (s->resident && s->running && !s->draining &&
                std::chrono::steady_clock::now() - s->t_launch > std::chrono::seconds(480)) {
                s->draining = true;
                unsigned long long one = 1;
                cudaMemcpyAsync((unsigned long long *)s->ctl.p + kShutdown, &one, sizeof(one), cudaMemcpyHostToDevice,
                                s->cstream);
                cudaStreamSynchronize(s->cstream);
            }
            bool arena_full = false;  // requests wait for blocks to free up
            if (!s->draining && admit(s, lk, arena_full)) progress = true;
            if ((!s->inflight.empty() || s->resident) && !s->running) {
                vc_status st = launch_kernel(s);
                if (st != VC_OK) s->fatal = st;
                progress = true;
            }
        }
        if (collect(s)) progress = true;
        if (progress) s->cv.notify_all();
        if (s->stop && s->inflight.empty() && s->pending.empty()) break;
        if (s->stop && !s->running) {
            fail_inflight(s, VC_TIMEOUT);
            break;
        }
        nap_us = progress ? 20 : std::min<uint32_t>(nap_us * 2, 500);
        s->cv.wait_for(lk, std::chrono::microseconds(nap_us));
    }
    if (s->running) {  // ask the kernel to stop once idle and wait for it (bounded by its own limits)
        unsigned long long one = 1;
        cudaMemcpyAsync((unsigned long long *)s->ctl.p + kShutdown, &one, sizeof(one), cudaMemcpyHostToDevice,
                        s->cstream);
        cudaStreamSynchronize(s->cstream);
        lk.unlock();
        cudaStreamSynchronize(s->kstream);
        lk.lock();
        s->running = false;
    }
    s->cv.notify_all();
}

// Asks a lane's loop to stop; its kernel drains and exits.
void lane_stop(SrvLane *s)
{
    if (!s) return;
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv.notify_all();
}

void lane_destroy(SrvLane *s)
{
    if (!s) return;
    lane_stop(s);
    if (s->loop.joinable()) s->loop.join();
    s->desc.release();
    s->st.release();
    s->covers.release();
    s->ctl.release();
    s->seq.release();
    s->data.release();
    s->gws.release();
    s->subq.release();
    s->arena.release();
    if (s->h_res) cudaFreeHost(s->h_res);
    if (s->kstream) cudaStreamDestroy(s->kstream);
    if (s->cstream) cudaStreamDestroy(s->cstream);
    delete s;
}

// A lane for requests of at most max_n vertices with the given plan.
vc_status lane_create(Ctx *c, uint64_t budget, uint32_t slots, uint32_t max_n, const Plan &pl, bool resident,
                      SrvLane **out)
{
    SrvLane *s = new SrvLane();
    s->resident = resident;
    s->dev = c->dev;
    s->ctx = c;
    s->slots = slots;
    s->max_n = max_n;
    s->nw_max = (max_n + 31) / 32;
    s->pl = pl;
    s->q = 1024;
    while (s->q < 2 * s->pl.num_su) s->q <<= 1;
    s->res_words = (uint32_t)(sizeof(HostResult) / 4) + s->nw_max;
    s->res_words = (s->res_words + 3) / 4 * 4;
    s->arena_cap = budget;
    s->arena_free.clear();
    s->arena_free.emplace(0, budget);
    bool ok = cudaStreamCreateWithFlags(&s->kstream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s->cstream, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && !s->desc.ensure(sizeof(InstDesc) * s->slots) && !s->st.ensure(sizeof(InstState) * s->slots) &&
         !s->covers.ensure(4ull * s->slots * s->nw_max) && !s->ctl.ensure(sizeof(unsigned long long) * kCtlWords) &&
         !s->seq.ensure(sizeof(unsigned long long) * s->q) && !s->data.ensure(4ull * s->q * s->pl.stride) &&
         !s->subq.ensure(4ull * kSubQ) && !s->arena.ensure(budget) &&
         (!s->pl.global_ws || !s->gws.ensure((size_t)s->pl.num_su * s->pl.su_bytes));
    ok = ok && cudaMemset(s->ctl.p, 0, sizeof(unsigned long long) * kCtlWords) == cudaSuccess;
    const size_t res_bytes = 4ull * s->slots * s->res_words;
    ok = ok && cudaHostAlloc((void **)&s->h_res, res_bytes, cudaHostAllocMapped) == cudaSuccess;
    ok = ok && cudaHostGetDevicePointer((void **)&s->d_res, s->h_res, 0) == cudaSuccess;
    if (!ok) {
        lane_destroy(s);
        return VC_ERR_NOMEM;
    }
    memset(s->h_res, 0, res_bytes);
    s->info.resize(s->slots);
    for (uint32_t i = 0; i < s->slots; ++i) s->free_slots.push_back(s->slots - 1 - i);
    if (resident) {  // launched now, in the order the lanes are created
        vc_status e = launch_kernel(s);
        if (e != VC_OK) {
            lane_destroy(s);
            return e;
        }
        // Bounded wait for all CTAs to start, so that the next lane is placed
        // around them.  If it runs out the lane still serves; only its
        // placement is left to the block scheduler.
        wait_resident(s);
    }
    s->loop = std::thread(request_loop, s);
    *out = s;
    return VC_OK;
}

constexpr uint32_t kDenseMax = 255;  // the narrow dense lane's largest request

// A lane's kernel shape and how many of its CTAs it places on each SM.
struct LaneSpec {
    Plan pl;
    uint32_t max_n = 0;
    uint32_t per_sm = 0;
    bool resident = false;
};

struct SmRes {
    int regs = 0, smem = 0, reserved = 0, warps = 0, blocks = 0;
};

// Registers, shared memory, warps and CTAs that `per_sm` CTAs of a plan take on one SM.
bool sm_use(const Plan &pl, uint32_t per_sm, const SmRes &r, uint64_t use[4])
{
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, pl.fn) != cudaSuccess) return false;
    const uint64_t warp_regs = (uint64_t)(fa.numRegs * 32 + 255) / 256 * 256;  // per-warp allocation unit
    use[0] += per_sm * (pl.block / 32) * warp_regs;
    use[1] += per_sm * ((uint64_t)pl.smem + fa.sharedSizeBytes + (uint64_t)r.reserved);
    use[2] += per_sm * (pl.block / 32);
    use[3] += per_sm;
    return true;
}

bool fits(const uint64_t use[4], const SmRes &r)
{
    return use[0] <= (uint64_t)r.regs && use[1] <= (uint64_t)r.smem && use[2] <= (uint64_t)r.warps &&
           use[3] <= (uint64_t)r.blocks;
}

// Lanes for requests of up to max_n (> 255) vertices: the narrow dense lane
// (n <= 255), the wide dense lane (256..640 vertices, byte degrees) and a CSR
// lane for the rest, returned in that order.  Their CTAs share every SM, and
// each placement is forced by what is free on the SMs rather than left to the
// block scheduler: the wide lane's CTAs are padded to more than half an SM's
// shared memory (so one per SM) and launched first; the narrow lane, launched
// next, finds room for exactly three CTAs per SM; the CSR lane (launched on
// demand) finds registers for exactly one.  Any lane relaunched later fits the
// same way into what the others leave.  The two dense lanes stay resident.
// Returns an empty list when this does not fit the device.
std::vector<LaneSpec> plan_lanes(Ctx &c, uint32_t max_n)
{
    std::vector<LaneSpec> none;
    SmRes r;
    if (cudaDeviceGetAttribute(&r.regs, cudaDevAttrMaxRegistersPerMultiprocessor, c.dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&r.smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c.dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&r.reserved, cudaDevAttrReservedSharedMemoryPerBlock, c.dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&r.warps, cudaDevAttrMaxThreadsPerMultiProcessor, c.dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&r.blocks, cudaDevAttrMaxBlocksPerMultiprocessor, c.dev) != cudaSuccess)
        return none;
    r.warps /= 32;
    LaneSpec narrow, wide, csr;
    narrow.max_n = kDenseMax;
    narrow.per_sm = 3;
    narrow.resident = true;
    if (make_plan(c, 32 * 8, kDenseMax, narrow.pl) != cudaSuccess || !narrow.pl.dense) return none;
    wide.max_n = std::min(max_n, kWideMaxN);
    wide.per_sm = 1;
    wide.resident = true;
    PlanOpts wo;
    wo.wide = true;
    if (make_plan(c, 32 * 20, kWideMaxN, wide.pl, wo) != cudaSuccess || !wide.pl.dense) return none;
    cudaFuncAttributes fw;
    if (cudaFuncGetAttributes(&fw, wide.pl.fn) != cudaSuccess) return none;
    // padding: two of the wide CTAs must not fit on one SM
    const uint32_t half = (uint32_t)r.smem / 2 + 1 - (uint32_t)fw.sharedSizeBytes - (uint32_t)r.reserved;
    wide.pl.smem = std::max(wide.pl.smem, half);
    if (wide.pl.smem > (uint32_t)c.smem_optin) return none;
    const uint32_t np = std::max<uint32_t>(32, (max_n + 31) / 32 * 32);
    uint64_t use[4] = {0, 0, 0, 0};
    if (!sm_use(wide.pl, 1, r, use) || !sm_use(narrow.pl, narrow.per_sm, r, use) || !fits(use, r)) return none;
    {   // exactly three narrow CTAs beside the wide one: a fourth must not fit
        uint64_t u4[4] = {use[0], use[1], use[2], use[3]};
        if (sm_use(narrow.pl, 1, r, u4) && fits(u4, r)) return none;
    }
    for (uint32_t warps = 8; warps >= 1; warps >>= 1) {
        csr.max_n = max_n;
        csr.per_sm = 1;
        PlanOpts so;
        so.warp_gws = true;
        so.warp_max_np = 1u << 16;
        so.warps = warps;
        if (make_plan(c, np, max_n, csr.pl, so) != cudaSuccess || csr.pl.dense) continue;
        uint64_t u3[4] = {use[0], use[1], use[2], use[3]};
        if (!sm_use(csr.pl, 1, r, u3) || !fits(u3, r)) continue;
        uint64_t u5[4] = {u3[0], u3[1], u3[2], u3[3]};  // and a second CSR CTA must not fit
        if (sm_use(csr.pl, 1, r, u5) && fits(u5, r)) continue;
        std::vector<LaneSpec> lanes{narrow, wide, csr};
        for (LaneSpec &l : lanes) cap_plan(c, l.pl, l.per_sm);
        return lanes;
    }
    return none;
}

}  // namespace

// Public handle: the lanes; a ticket carries its lane in its low two bits.
struct vc_server {
    std::vector<SrvLane *> lanes;
    uint32_t max_n = 0;
    bool wide_lane = false;  // lanes[1] is the wide dense lane
};

namespace {
inline SrvLane *lane_of(vc_server *s, uint64_t ticket, uint64_t *lt)
{
    const uint32_t li = (uint32_t)(ticket & 3u);
    if (li >= s->lanes.size()) return nullptr;
    *lt = ticket >> 2;
    return s->lanes[li];
}
}  // namespace

extern "C" vc_status vc_server_create(int32_t device, uint64_t mem_budget_bytes, uint32_t max_requests,
                                     uint32_t max_vertices, vc_server **out)
{
    vch::DeviceGuard dg;
    if (!out) return VC_ERR_INVALID;
    *out = nullptr;
    vc_status err;
    Ctx *c = get_ctx(device, &err);
    if (!c) return err;
    const uint32_t slots = max_requests ? max_requests : 1024;
    const uint64_t budget = mem_budget_bytes ? mem_budget_bytes : (1ull << 30);
    // the largest graph a request may have: it sizes the search units'
    // workspaces and picks the kernels (dense bitsets up to 255 vertices)
    const uint32_t max_n = max_vertices ? max_vertices : 1024;
    if (max_n > kMaxVertices) return VC_ERR_TOO_LARGE;
    vc_server *s = new vc_server();
    s->max_n = max_n;
    std::vector<LaneSpec> specs;
    if (max_n > kDenseMax && !c->force_sparse) specs = plan_lanes(*c, max_n);
    if (!specs.empty()) {
        // device memory for admitted graphs: half to the narrow dense lane;
        // the wide lane is created (and launched) first, see plan_lanes
        const uint64_t share[3] = {budget / 2, budget / 4, budget - budget / 2 - budget / 4};
        SrvLane *made[3] = {nullptr, nullptr, nullptr};
        for (int i : {1, 0, 2}) {
            vc_status e = lane_create(c, share[i], slots, specs[i].max_n, specs[i].pl, specs[i].resident, &made[i]);
            if (e != VC_OK) {
                for (SrvLane *x : made) lane_stop(x);
                for (SrvLane *x : made) lane_destroy(x);
                delete s;
                return e;
            }
        }
        s->lanes = {made[0], made[1], made[2]};
        s->wide_lane = true;
    } else {
        Plan pl;
        if (make_plan(*c, std::max<uint32_t>(32, (max_n + 31) / 32 * 32), max_n, pl) != cudaSuccess) {
            delete s;
            return VC_ERR_CUDA;
        }
        SrvLane *a = nullptr;
        vc_status e = lane_create(c, budget, slots, max_n, pl, false, &a);
        if (e != VC_OK) {
            delete s;
            return e;
        }
        s->lanes = {a};
    }
    *out = s;
    return VC_OK;
}

extern "C" vc_status vc_server_submit(vc_server *s, const vc_csr *g, const vc_request *req, uint64_t *ticket)
{
    vch::DeviceGuard dg;
    if (!s || !g || !req || !ticket) return VC_ERR_INVALID;
    if (req->instance != VC_MVC && req->instance != VC_PVC) return VC_ERR_INVALID;
    if (req->flags & VC_FLAG_DEVICE_INPUT) return VC_ERR_INVALID;  // the server copies from host memory
    if (g->n == 0) return VC_ERR_INVALID;
    if (g->n > s->max_n) return VC_ERR_TOO_LARGE;
    if (!(req->flags & VC_FLAG_NO_VALIDATE)) {
        vc_status v = validate_csr(g);
        if (v != VC_OK) return v;
    }
    // lane: narrow dense, wide dense (byte degrees, up to 640 vertices), else CSR
    uint32_t li = (uint32_t)s->lanes.size() - 1u;
    if (s->lanes.size() > 1 && g->n <= kDenseMax) li = 0;
    else if (s->wide_lane && wide_ok(g->n, g->row_ptr)) li = 1;
    SrvLane *l = s->lanes[li];
    Pending p;
    p.n = g->n;
    p.m = g->m;
    p.rp.assign(g->row_ptr, g->row_ptr + g->n + 1);
    if (g->m) p.col.assign(g->col, g->col + 2ull * g->m);
    p.req = *req;
    p.t_submit = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lk(l->mu);
    if (l->stop) return VC_ERR_INVALID;
    if (l->fatal != VC_OK) return l->fatal;
    p.ticket = l->next_ticket++;
    *ticket = (p.ticket << 2) | li;
    l->pending.push_back(std::move(p));
    l->cv.notify_all();
    return VC_OK;
}

extern "C" vc_status vc_server_poll(vc_server *s, uint64_t ticket, vc_result *out)
{
    vch::DeviceGuard dg;
    if (!s || !out) return VC_ERR_INVALID;
    uint64_t lt = 0;
    SrvLane *l = lane_of(s, ticket, &lt);
    if (!l) return VC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(l->mu);
    auto it = l->done.find(lt);
    if (it == l->done.end()) {
        if (l->inflight.count(lt)) return VC_PENDING;
        for (auto &p : l->pending)
            if (p.ticket == lt) return VC_PENDING;
        return VC_ERR_INVALID;
    }
    Done &d = it->second;
    out->status = d.status;
    out->size = d.size;
    out->decision = d.decision;
    out->has_cover = d.has_cover;
    out->tree_nodes = d.nodes;
    out->kernel_ms = 0;
    out->total_ms = d.total_ms;
    out->done_ms = d.total_ms;
    if (out->cover_mask && !d.cover.empty()) memcpy(out->cover_mask, d.cover.data(), d.cover.size());
    vc_status st = d.status;
    l->done.erase(it);
    return st;
}

extern "C" vc_status vc_server_completed(vc_server *s, uint64_t *tickets, uint32_t max_tickets, uint32_t *count)
{
    vch::DeviceGuard dg;
    if (!s || !count || (max_tickets && !tickets)) return VC_ERR_INVALID;
    uint32_t k = 0;
    for (uint32_t li = 0; li < s->lanes.size(); ++li) {
        SrvLane *l = s->lanes[li];
        std::lock_guard<std::mutex> lk(l->mu);
        while (k < max_tickets && !l->ready.empty()) {
            const uint64_t t = l->ready.front();
            l->ready.pop_front();
            if (l->done.count(t)) tickets[k++] = (t << 2) | li;  // skip tickets already collected by vc_server_poll
        }
    }
    *count = k;
    return VC_OK;
}

extern "C" vc_status vc_server_shape(vc_server *s, uint32_t *shape, uint32_t max_lanes, uint32_t *lanes)
{
    if (!s || !lanes || (max_lanes && !shape)) return VC_ERR_INVALID;
    *lanes = (uint32_t)s->lanes.size();
    for (uint32_t i = 0; i < s->lanes.size() && i < max_lanes; ++i) {
        const SrvLane *l = s->lanes[i];
        uint32_t *o = shape + 6 * i;  // per lane
        o[0] = l->max_n;
        o[1] = l->pl.grid;
        o[2] = l->pl.block;
        o[3] = l->pl.num_su;
        o[4] = l->pl.smem;
        o[5] = l->pl.dense ? 1u : 0u;
    }
    return VC_OK;
}

extern "C" vc_status vc_server_destroy(vc_server *s)
{
    vch::DeviceGuard dg;
    if (!s) return VC_ERR_INVALID;
    // all lanes stop together: a lane's kernel can only finish once all its
    // CTAs have run, which may need another lane's kernel to leave its SMs
    for (SrvLane *l : s->lanes) lane_stop(l);
    for (SrvLane *l : s->lanes) lane_destroy(l);
    delete s;
    return VC_OK;
}
