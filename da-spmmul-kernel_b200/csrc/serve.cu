// serve.cu -- a serving loop for many SpMM requests over resident matrices.
//
// The reference times one problem in a loop (SpmvSpmmProblem::benchmark,
// spmvspmm.h:220-243).  A server keeps a pool of device-resident CSR
// matrices and answers requests "C = A_m * B" that arrive over time:
//
//   * admission: every request's C lives in one device arena of a fixed byte
//     budget; a request waits in FIFO order until its C fits, and a request
//     whose C alone exceeds the budget is refused at submission;
//   * continuous batching (DASPMM_SERVE_BATCHED): a dispatcher thread takes
//     everything queued (up to max_batch requests / max_items work items)
//     into one launch group -- an instance table copy, the batch plan kernel
//     and one persistent batch kernel (batch.cu) -- as soon as one of
//     max_inflight group slots is free; results of a request do not depend on
//     the group it lands in (each output row is summed by one warp in
//     nonzero order, the column tile width follows the request's own nv);
//   * DASPMM_SERVE_PLAIN: the same queue and admission, one daspmm_spmm
//     (FP32, balanced CSR) launch per request -- the baseline a caller without
//     batching has.
//
// Completion is observed by the dispatcher polling the group's event;
// latency runs from arrival (submission, or the scheduled arrival time of
// daspmm_server_replay) to that observation.
#include "daspmm.h"
#include "internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

namespace daspmm {
namespace {

using Clock = std::chrono::steady_clock;

struct Matrix {
    int nr, nc, nnz;
    const int *rowPtr, *colIdx;
    const void *values;
    BatchTile *d_tiles;  // the matrix cut once (build_tiles), server-owned
    int ntiles, npieces, nlong;
};

struct Req {
    int matrix = 0, nv = 0;
    const void *B = nullptr;
    const float *bsc = nullptr;
    double t_arr = 0, t_launch = 0, t_done = 0;  // seconds since the server's epoch
    int status = -1;                              // -1 pending
    long long off = -1, bytes = 0;                // arena slice of C
    int group = -1;
    bool released = false;
};

struct Slot {
    BatchInst *h_inst = nullptr;  // pinned
    long long *h_begin = nullptr; // pinned
    BatchInst *d_inst = nullptr;
    long long *d_begin = nullptr;
    BatchItem *d_items = nullptr;
    unsigned long long *d_head = nullptr;
    float *d_slots = nullptr;  // piece partial sums of the group
    int *d_cnt = nullptr;      // piece counters (zero between launches)
    cudaEvent_t ev = nullptr;
    bool busy = false;
};

struct Group {
    int slot;  // -1: plain mode (ev below)
    cudaEvent_t ev;
    int id;
    std::vector<long long> tickets;
};

// First-fit allocator over [0, size) with coalescing; 256-byte granules.
class Arena {
public:
    void reset(long long size)
    {
        free_.clear();
        if (size > 0) free_[0] = size;
        size_ = size;
    }
    long long alloc(long long bytes)
    {
        bytes = (long long)align256((size_t)std::max<long long>(bytes, 1));
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            const long long off = it->first, rest = it->second - bytes;
            free_.erase(it);
            if (rest) free_[off + bytes] = rest;
            used_ += bytes;
            return off;
        }
        return -1;
    }
    void release(long long off, long long bytes)
    {
        bytes = (long long)align256((size_t)std::max<long long>(bytes, 1));
        used_ -= bytes;
        auto nx = free_.lower_bound(off);
        if (nx != free_.end() && off + bytes == nx->first) {
            bytes += nx->second;
            nx = free_.erase(nx);
        }
        if (nx != free_.begin()) {
            auto pv = std::prev(nx);
            if (pv->first + pv->second == off) {
                pv->second += bytes;
                return;
            }
        }
        free_[off] = bytes;
    }
    long long used() const { return used_; }
    long long size() const { return size_; }

private:
    std::map<long long, long long> free_;
    long long size_ = 0, used_ = 0;
};

long long c_bytes(const Matrix &m, int nv) { return (long long)m.nr * nv * 4; }

int col_tiles_of(int nv) { return (nv + batch_tile_width(nv) - 1) / batch_tile_width(nv); }

// Scratch a request needs in its launch group: slot floats and counters.
long long need_slots(const Matrix &m, int nv) { return (long long)m.npieces * nv; }
long long need_cnt(const Matrix &m, int nv) { return (long long)m.nlong * col_tiles_of(nv); }

}  // namespace
}  // namespace daspmm

using namespace daspmm;

struct daspmm_server_s {
    daspmm_server_config cfg{};
    int device = 0;
    cudaStream_t stream = nullptr;
    char *arena_base = nullptr;
    Arena arena;
    long long slot_cap = 0, cnt_cap = 0;  // per launch group (floats, ints)
    std::vector<Matrix> pool;
    std::vector<Slot> slots;
    std::deque<Group> inflight;
    std::deque<long long> queue;
    std::unordered_map<long long, Req> reqs;
    long long next_ticket = 1;
    int next_group = 0;
    std::mutex mu;
    std::condition_variable cv_work;  // dispatcher: queue / release / stop
    std::condition_variable cv_done;  // waiters: a request finished
    bool stop = false;
    std::thread dispatcher;
    Clock::time_point epoch;
    // statistics
    long long n_done = 0, n_cancelled = 0, n_refused = 0, n_groups = 0, n_launched = 0;
    long long items_total = 0;
    int max_group = 0;
    daspmm_status sticky = DASPMM_OK;

    double now() const { return std::chrono::duration<double>(Clock::now() - epoch).count(); }
};

namespace {

void destroy_slots(daspmm_server_s *s)
{
    for (Slot &sl : s->slots) {
        cudaFreeHost(sl.h_inst);
        cudaFreeHost(sl.h_begin);
        cudaFree(sl.d_inst);
        cudaFree(sl.d_begin);
        cudaFree(sl.d_items);
        cudaFree(sl.d_head);
        cudaFree(sl.d_slots);
        cudaFree(sl.d_cnt);
        if (sl.ev) cudaEventDestroy(sl.ev);
    }
    s->slots.clear();
}

// Called with the lock held: finish every request of a completed group.
void finish_group(daspmm_server_s *s, const Group &g, daspmm_status st)
{
    const double t = s->now();
    for (long long tk : g.tickets) {
        auto it = s->reqs.find(tk);
        if (it == s->reqs.end()) continue;
        it->second.t_done = t;
        it->second.status = st;
        ++s->n_done;
    }
}

// Called with the lock held: pull queued requests into a group while their C
// fits the arena (FIFO: stop at the first that does not) and the group's
// limits hold.  Returns the admitted tickets.
std::vector<long long> admit(daspmm_server_s *s, int max_req, long long max_items)
{
    std::vector<long long> out;
    long long items = 0, slots = 0, cnts = 0;
    while (!s->queue.empty() && (int)out.size() < max_req) {
        const long long tk = s->queue.front();
        Req &r = s->reqs[tk];
        const Matrix &m = s->pool[r.matrix];
        if (s->cfg.mode == DASPMM_SERVE_BATCHED) {
            const long long it = (long long)m.ntiles * col_tiles_of(r.nv);
            const long long sl = need_slots(m, r.nv), cn = need_cnt(m, r.nv);
            if (!out.empty() && (items + it > max_items || slots + sl > s->slot_cap ||
                                 cnts + cn > s->cnt_cap))
                break;
            items += it;
            slots += sl;
            cnts += cn;
        }
        const long long off = s->arena.alloc(r.bytes);
        if (off < 0) break;
        r.off = off;
        s->queue.pop_front();
        out.push_back(tk);
    }
    return out;
}

daspmm_status launch_plain(daspmm_server_s *s, Req &r, cudaEvent_t ev)
{
    const Matrix &m = s->pool[r.matrix];
    float *C = reinterpret_cast<float *>(s->arena_base + r.off);
    daspmm_status st = daspmm_spmm(DASPMM_ALG_CSR_BALANCED, DASPMM_ROW_MAJOR, m.nr, m.nc, m.nnz,
                                   r.nv, m.rowPtr, nullptr, m.colIdx,
                                   static_cast<const float *>(m.values),
                                   static_cast<const float *>(r.B), C, 0.0f, s->stream);
    if (st == DASPMM_OK) {
        const cudaError_t e = cudaEventRecord(ev, s->stream);
        if (e != cudaSuccess) st = cuda_fail(e);
    }
    return st;
}

daspmm_status launch_batch(daspmm_server_s *s, Slot &sl, std::vector<Req *> &rs, long long *nitems)
{
    const int n = (int)rs.size();
    int wmode = -1;
    sl.h_begin[0] = 0;
    long long slot_off = 0, cnt_off = 0;
    for (int i = 0; i < n; ++i) {
        const Req &r = *rs[i];
        const Matrix &m = s->pool[r.matrix];
        daspmm_instance in{};
        in.nr = m.nr; in.nc = m.nc; in.nnz = m.nnz; in.nv = r.nv;
        in.rowPtr = m.rowPtr; in.colIdx = m.colIdx; in.values = m.values;
        in.val_fmt = s->cfg.val_fmt;
        in.B = r.B; in.b_fmt = s->cfg.b_fmt; in.b_scales = r.bsc;
        in.C = reinterpret_cast<float *>(s->arena_base + r.off);
        in.beta = 0.0f;
        BatchInst &bi = sl.h_inst[i];
        const daspmm_status fs = batch_fill(in, &bi);
        if (fs != DASPMM_OK) return fs;  // checked at submission; not expected
        bi.tiles = m.d_tiles;
        bi.ntiles = m.ntiles;
        bi.slots = sl.d_slots + slot_off;
        bi.cnt = sl.d_cnt + cnt_off;
        slot_off += need_slots(m, r.nv);
        cnt_off += need_cnt(m, r.nv);
        const int w = bi.W;
        wmode = (wmode < 0 || wmode == w) ? w : 0;
        sl.h_begin[i + 1] = sl.h_begin[i] + (long long)bi.ntiles * bi.col_tiles;
    }
    *nitems = sl.h_begin[n];
    cudaError_t e = cudaMemcpyAsync(sl.d_inst, sl.h_inst, sizeof(BatchInst) * n,
                                    cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(sl.d_begin, sl.h_begin, sizeof(long long) * (n + 1),
                            cudaMemcpyHostToDevice, s->stream);
    if (e != cudaSuccess) return cuda_fail(e);
    daspmm_status st = batch_plan_async(sl.d_inst, sl.d_begin, n, sl.d_items, *nitems,
                                        s->stream);
    if (st == DASPMM_OK)
        // the 32-lane kernel: groups are small at most arrival rates, and a
        // group's latency is lower at its occupancy (p50 at 20k req/s 133
        // against 202 us with the worker-group kernel for uniform-width
        // groups, 160-176 us when also every instance qualifies; throughput
        // at the tightest equal-p99 bound no higher)
        st = batch_kernel_async(s->cfg.val_fmt, s->cfg.b_fmt, std::max(wmode, 0), false,
                                sl.d_inst, sl.d_items, *nitems, sl.d_head, s->stream);
    if (st == DASPMM_OK) {
        e = cudaEventRecord(sl.ev, s->stream);
        if (e != cudaSuccess) st = cuda_fail(e);
    }
    return st;
}

void dispatcher_main(daspmm_server_s *s)
{
    cudaSetDevice(s->device);
    const bool batched = s->cfg.mode == DASPMM_SERVE_BATCHED;
    std::vector<cudaEvent_t> plain_events;  // free events for plain groups
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        bool progress = false;
        // 1. retire completed groups, oldest first
        while (!s->inflight.empty()) {
            Group &g = s->inflight.front();
            lk.unlock();
            const cudaError_t q = cudaEventQuery(g.ev);
            lk.lock();
            if (q == cudaErrorNotReady) break;
            daspmm_status st = DASPMM_OK;
            if (q != cudaSuccess) {
                st = cuda_fail(q);
                s->sticky = st;
            }
            finish_group(s, g, st);
            if (g.slot >= 0) s->slots[g.slot].busy = false;
            else plain_events.push_back(g.ev);
            s->inflight.pop_front();
            progress = true;
            s->cv_done.notify_all();
        }
        if (s->stop && s->inflight.empty()) break;
        // 2. dispatch a new group when a slot is free
        const int max_inflight = s->cfg.max_inflight;
        if (!s->stop && !s->queue.empty() && (int)s->inflight.size() < max_inflight) {
            bool hold = false;
            if (batched && s->cfg.window_us > 0 && !s->inflight.empty() &&
                (int)s->queue.size() < s->cfg.max_batch) {
                const double oldest = s->reqs[s->queue.front()].t_arr;
                hold = (s->now() - oldest) * 1e6 < s->cfg.window_us;
            }
            std::vector<long long> tk;
            if (!hold) tk = admit(s, batched ? s->cfg.max_batch : 1, s->cfg.max_items);
            if (!tk.empty()) {
                Group g;
                g.id = s->next_group++;
                g.tickets = tk;
                const double t = s->now();
                std::vector<Req *> rs;
                for (long long t1 : tk) {
                    Req &r = s->reqs[t1];
                    r.t_launch = t;
                    r.group = g.id;
                    rs.push_back(&r);
                }
                daspmm_status st = DASPMM_OK;
                long long items = 0;
                if (batched) {
                    int si = 0;
                    while (s->slots[si].busy) ++si;  // a free slot exists: inflight < slots
                    Slot &sl = s->slots[si];
                    sl.busy = true;
                    g.slot = si;
                    g.ev = sl.ev;
                    lk.unlock();
                    st = launch_batch(s, sl, rs, &items);
                    lk.lock();
                } else {
                    g.slot = -1;
                    if (plain_events.empty()) {
                        cudaEvent_t ev = nullptr;
                        const cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
                        if (e != cudaSuccess) st = cuda_fail(e);
                        plain_events.push_back(ev);
                    }
                    g.ev = plain_events.back();
                    plain_events.pop_back();
                    if (st == DASPMM_OK) {
                        lk.unlock();
                        st = launch_plain(s, *rs[0], g.ev);
                        lk.lock();
                    }
                }
                ++s->n_groups;
                s->n_launched += (long long)tk.size();
                s->items_total += items;
                s->max_group = std::max(s->max_group, (int)tk.size());
                if (st != DASPMM_OK) {  // nothing in flight for this group
                    s->sticky = st;
                    finish_group(s, g, st);
                    if (g.slot >= 0) s->slots[g.slot].busy = false;
                    else if (g.ev) plain_events.push_back(g.ev);
                    s->cv_done.notify_all();
                } else {
                    s->inflight.push_back(std::move(g));
                }
                progress = true;
            }
        }
        if (progress) continue;
        if (s->inflight.empty()) {
            // idle: sleep until a request, a release (budget) or stop
            s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
        } else {
            // the GPU is busy: poll its events without holding the lock
            lk.unlock();
            std::this_thread::yield();
            lk.lock();
        }
    }
    lk.unlock();
    for (cudaEvent_t ev : plain_events) cudaEventDestroy(ev);
}

}  // namespace

extern "C" {

daspmm_status daspmm_server_create(const daspmm_server_config *cfg, daspmm_server *out)
{
    if (!out) return DASPMM_ERR_INVALID;
    *out = nullptr;
    daspmm_server_config c{};
    if (cfg) c = *cfg;
    if (c.budget_bytes <= 0) c.budget_bytes = 1ll << 30;
    if (c.mode != DASPMM_SERVE_BATCHED && c.mode != DASPMM_SERVE_PLAIN) return DASPMM_ERR_INVALID;
    if (c.mode == DASPMM_SERVE_PLAIN) {
        if (c.val_fmt != DASPMM_F32 || c.b_fmt != DASPMM_F32) return DASPMM_ERR_UNSUPPORTED;
    } else if (!batch_formats_ok(c.val_fmt, c.b_fmt)) {
        return DASPMM_ERR_UNSUPPORTED;
    }
    if (c.chunk <= 0) c.chunk = 256;
    if (c.max_batch <= 0) c.max_batch = 1024;
    if (c.max_items <= 0) c.max_items = 1ll << 22;
    // batched: two groups in flight, so a group of requests that arrived while
    // another runs starts on the SMs it leaves free (one group in flight
    // measured a little lower p50 / p99 on the 64-matrix pool -- 0.10 / 0.40
    // against 0.13 / 0.45 ms at 20k req/s -- with the same capacity)
    if (c.max_inflight <= 0) c.max_inflight = c.mode == DASPMM_SERVE_PLAIN ? 64 : 2;
    if (c.scratch_bytes <= 0) c.scratch_bytes = 64ll << 20;
    if (c.window_us < 0) return DASPMM_ERR_INVALID;
    daspmm_server_s *s = new (std::nothrow) daspmm_server_s;
    if (!s) return DASPMM_ERR_NOMEM;
    s->cfg = c;
    s->epoch = Clock::now();
    s->slot_cap = c.scratch_bytes / 4;
    s->cnt_cap = c.scratch_bytes / 32;
    cudaGetDevice(&s->device);
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&s->arena_base, (size_t)c.budget_bytes);
    if (e == cudaSuccess && c.mode == DASPMM_SERVE_BATCHED) {
        s->slots.resize(c.max_inflight);
        for (Slot &sl : s->slots) {
            if (e == cudaSuccess) e = cudaMallocHost(&sl.h_inst, sizeof(BatchInst) * c.max_batch);
            if (e == cudaSuccess) e = cudaMallocHost(&sl.h_begin, sizeof(long long) * (c.max_batch + 1));
            if (e == cudaSuccess) e = cudaMalloc(&sl.d_inst, sizeof(BatchInst) * c.max_batch);
            if (e == cudaSuccess) e = cudaMalloc(&sl.d_begin, sizeof(long long) * (c.max_batch + 1));
            if (e == cudaSuccess) e = cudaMalloc(&sl.d_items, sizeof(BatchItem) * c.max_items);
            if (e == cudaSuccess) e = cudaMalloc(&sl.d_head, sizeof(unsigned long long));
            if (e == cudaSuccess) e = cudaMalloc(&sl.d_slots, sizeof(float) * s->slot_cap);
            if (e == cudaSuccess) e = cudaMalloc(&sl.d_cnt, sizeof(int) * s->cnt_cap);
            if (e == cudaSuccess) e = cudaMemset(sl.d_cnt, 0, sizeof(int) * s->cnt_cap);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming);
        }
    }
    if (e != cudaSuccess) {
        const daspmm_status st = e == cudaErrorMemoryAllocation ? DASPMM_ERR_NOMEM : cuda_fail(e);
        cudaGetLastError();
        destroy_slots(s);
        cudaFree(s->arena_base);
        if (s->stream) cudaStreamDestroy(s->stream);
        delete s;
        return st;
    }
    s->arena.reset(c.budget_bytes);
    s->dispatcher = std::thread(dispatcher_main, s);
    *out = s;
    return DASPMM_OK;
}

daspmm_status daspmm_server_add_matrix(daspmm_server s, int nr, int nc, int nnz,
                                       const int *rowPtr, const int *colIdx,
                                       const void *values, int *id)
{
    if (!s || !id) return DASPMM_ERR_INVALID;
    *id = -1;
    if (nr < 0 || nc < 0 || nnz < 0 || (nnz > 0 && !values)) return DASPMM_ERR_INVALID;
    int bad = -1;
    daspmm_status st = daspmm_csr_check(nr, nc, nnz, rowPtr, colIdx, 0, &bad, nullptr);
    if (st != DASPMM_OK) return st;
    Matrix m{nr, nc, nnz, rowPtr, colIdx, values, nullptr, 0, 0, 0};
    if (s->cfg.mode == DASPMM_SERVE_BATCHED && nr > 0) {  // cut it once
        std::vector<int> rp((size_t)nr + 1);
        cudaError_t e = cudaMemcpy(rp.data(), rowPtr, sizeof(int) * (nr + 1), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e);
        TilePlan plan;
        build_tiles(rp.data(), nr, s->cfg.chunk, &plan);
        m.ntiles = (int)plan.tiles.size();
        m.npieces = plan.npieces;
        m.nlong = plan.nlong;
        e = cudaMalloc(&m.d_tiles, sizeof(BatchTile) * plan.tiles.size());
        if (e == cudaSuccess)
            e = cudaMemcpy(m.d_tiles, plan.tiles.data(), sizeof(BatchTile) * plan.tiles.size(),
                           cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(m.d_tiles);
            cudaGetLastError();
            return e == cudaErrorMemoryAllocation ? DASPMM_ERR_NOMEM : cuda_fail(e);
        }
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->pool.push_back(m);
    *id = (int)s->pool.size() - 1;
    return DASPMM_OK;
}

static daspmm_status submit_at(daspmm_server s, const daspmm_request *r, double t_arr,
                               long long *ticket)
{
    if (!s || !r || !ticket) return DASPMM_ERR_INVALID;
    *ticket = 0;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->stop) return DASPMM_ERR_INVALID;
    if (r->matrix < 0 || r->matrix >= (int)s->pool.size() || r->nv < 1) return DASPMM_ERR_INVALID;
    const Matrix &m = s->pool[r->matrix];
    if (s->cfg.mode == DASPMM_SERVE_BATCHED) {
        daspmm_instance in{};
        in.nr = m.nr; in.nc = m.nc; in.nnz = m.nnz; in.nv = r->nv;
        in.rowPtr = m.rowPtr; in.colIdx = m.colIdx; in.values = m.values;
        in.val_fmt = s->cfg.val_fmt; in.B = r->B; in.b_fmt = s->cfg.b_fmt;
        in.b_scales = r->b_scales;
        in.C = reinterpret_cast<float *>(s->arena_base);  // arena slices are 256-aligned
        BatchInst probe;
        const daspmm_status fs = batch_fill(in, &probe);
        if (fs != DASPMM_OK) return fs;
        if ((long long)m.ntiles * probe.col_tiles > s->cfg.max_items ||
            need_slots(m, r->nv) > s->slot_cap || need_cnt(m, r->nv) > s->cnt_cap) {
            ++s->n_refused;
            return DASPMM_ERR_BUDGET;
        }
    } else if (m.nnz > 0 && !r->B) {
        return DASPMM_ERR_INVALID;
    }
    const long long bytes = c_bytes(m, r->nv);
    if ((long long)align256((size_t)std::max<long long>(bytes, 1)) > s->arena.size()) {
        ++s->n_refused;
        return DASPMM_ERR_BUDGET;
    }
    const long long tk = s->next_ticket++;
    Req q;
    q.matrix = r->matrix;
    q.nv = r->nv;
    q.B = r->B;
    q.bsc = r->b_scales;
    q.t_arr = t_arr < 0 ? s->now() : t_arr;
    q.bytes = bytes;
    s->reqs.emplace(tk, q);
    s->queue.push_back(tk);
    *ticket = tk;
    lk.unlock();
    s->cv_work.notify_one();
    return DASPMM_OK;
}

daspmm_status daspmm_server_submit(daspmm_server s, const daspmm_request *r, long long *ticket)
{
    return submit_at(s, r, -1.0, ticket);
}

daspmm_status daspmm_server_cancel(daspmm_server s, long long ticket)
{
    if (!s) return DASPMM_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return DASPMM_ERR_INVALID;
    auto q = std::find(s->queue.begin(), s->queue.end(), ticket);
    if (q == s->queue.end()) return DASPMM_ERR_UNSUPPORTED;  // already launched or finished
    s->queue.erase(q);
    it->second.status = DASPMM_ERR_CANCELLED;
    it->second.t_done = s->now();
    ++s->n_cancelled;
    s->cv_done.notify_all();
    s->cv_work.notify_one();  // the head of the queue may have changed
    return DASPMM_OK;
}

static void fill_result(daspmm_server s, const Req &r, daspmm_result *out)
{
    out->status = r.status;
    out->C = (r.status == DASPMM_OK && r.off >= 0 && !r.released)
                 ? reinterpret_cast<float *>(s->arena_base + r.off)
                 : nullptr;
    out->queue_us = r.t_launch > 0 ? (r.t_launch - r.t_arr) * 1e6 : 0.0;
    out->latency_us = r.status >= 0 ? (r.t_done - r.t_arr) * 1e6 : 0.0;
    out->group = r.group;
}

daspmm_status daspmm_server_wait(daspmm_server s, long long ticket, int timeout_ms,
                                 daspmm_result *out)
{
    if (!s || !out) return DASPMM_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return DASPMM_ERR_INVALID;
    const auto deadline = Clock::now() + std::chrono::milliseconds(std::max(timeout_ms, 0));
    while (it->second.status < 0) {
        if (timeout_ms >= 0) {
            if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout &&
                it->second.status < 0) {
                fill_result(s, it->second, out);
                return DASPMM_ERR_TIMEOUT;
            }
        } else {
            s->cv_done.wait(lk);
        }
        it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return DASPMM_ERR_INVALID;
    }
    fill_result(s, it->second, out);
    return DASPMM_OK;
}

daspmm_status daspmm_server_release(daspmm_server s, long long ticket)
{
    if (!s) return DASPMM_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return DASPMM_ERR_INVALID;
    if (it->second.status < 0) return DASPMM_ERR_UNSUPPORTED;  // pending: cancel or wait first
    if (it->second.off >= 0) s->arena.release(it->second.off, it->second.bytes);
    s->reqs.erase(it);
    lk.unlock();
    s->cv_work.notify_one();  // budget freed
    return DASPMM_OK;
}

daspmm_status daspmm_server_replay(daspmm_server s, const daspmm_request *reqs, int n,
                                   const double *arrival_s, int release, daspmm_result *results)
{
    if (!s || n < 0 || (n > 0 && (!reqs || !arrival_s || !results))) return DASPMM_ERR_INVALID;
    std::vector<long long> tk(n, 0);
    std::vector<daspmm_status> sub(n, DASPMM_OK);
    std::atomic<int> submitted{0};
    std::atomic<int> worst{DASPMM_OK};
    // The collector waits for results in submission order and (release != 0)
    // frees each C at once, so the arena drains while requests still arrive.
    std::thread collector([&] {
        for (int i = 0; i < n; ++i) {
            while (submitted.load(std::memory_order_acquire) <= i) std::this_thread::yield();
            daspmm_result &r = results[i];
            r = daspmm_result{};
            if (sub[i] != DASPMM_OK) {
                r.status = sub[i];
                r.group = -1;
                continue;
            }
            const daspmm_status w = daspmm_server_wait(s, tk[i], -1, &r);
            if (w != DASPMM_OK) worst.store(w);
            if (release) {
                daspmm_server_release(s, tk[i]);
                r.C = nullptr;
            }
        }
    });
    const double t0 = s->now();
    for (int i = 0; i < n; ++i) {
        const double ta = t0 + arrival_s[i];
        for (;;) {  // sleep through long gaps, spin through the last 100 us
            const double d = ta - s->now();
            if (d <= 0) break;
            if (d > 2e-4) std::this_thread::sleep_for(std::chrono::duration<double>(d - 1e-4));
        }
        sub[i] = submit_at(s, &reqs[i], ta, &tk[i]);
        submitted.store(i + 1, std::memory_order_release);
    }
    collector.join();
    return (daspmm_status)worst.load();
}

daspmm_status daspmm_server_stats(daspmm_server s, daspmm_serve_stats *out)
{
    if (!s || !out) return DASPMM_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    out->completed = s->n_done;
    out->cancelled = s->n_cancelled;
    out->refused = s->n_refused;
    out->groups = s->n_groups;
    out->launched = s->n_launched;
    out->items = s->items_total;
    out->max_group = s->max_group;
    out->queued = (long long)s->queue.size();
    out->inflight_groups = (int)s->inflight.size();
    out->arena_used = s->arena.used();
    out->arena_bytes = s->arena.size();
    out->matrices = (int)s->pool.size();
    out->error = s->sticky;
    return DASPMM_OK;
}

daspmm_status daspmm_server_destroy(daspmm_server s)
{
    if (!s) return DASPMM_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        const double t = s->now();
        for (long long tk : s->queue) {  // never launched: cancelled
            Req &r = s->reqs[tk];
            r.status = DASPMM_ERR_CANCELLED;
            r.t_done = t;
            ++s->n_cancelled;
        }
        s->queue.clear();
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();  // in-flight groups complete first
    cudaStreamSynchronize(s->stream);
    destroy_slots(s);
    for (Matrix &m : s->pool) cudaFree(m.d_tiles);
    cudaFree(s->arena_base);
    cudaStreamDestroy(s->stream);
    delete s;
    return DASPMM_OK;
}

}  // extern "C"
