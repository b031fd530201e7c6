// Request loop over one device (include/hh.h, "serving").
//
// The reference has no serving layer: its Direct_Solver solves one problem per process.  This
// loop keeps the solver's per-problem set-up resident and streams requests through it:
//  * one plan per (dim, n, order, k) stays on the device (twiddles and sine tables are shared by
//    the context, factors and Pade tables belong to the plan) and is evicted least recently used
//    when the HBM budget needs the room; a new plan takes the kernel settings of its shape from
//    the tuning cache (hh_plan_tune), if the process has tuned that shape;
//  * continuous batching: when the dispatcher picks a request it also takes every queued request
//    of the same shape (dim, n, order) at any k (small ones, up to kMergeRhs right-hand sides in
//    all) and runs them as one batched solve over several plans (one transform launch per
//    direction, one line-solve launch with a table of which right-hand sides use which plan);
//  * admission: a batch starts only while plans plus in-flight staging stay within the budget;
//    otherwise it waits for running batches to finish;
//  * batches go round-robin to several CUDA streams, so work of different requests overlaps on
//    the device; completion is signalled by a host function enqueued behind each batch.
// Every batched solve computes each right-hand side with exactly the arithmetic of a solo solve
// on its own plan (the kernels never mix right-hand sides), so results are bitwise identical.
#include "hh_internal.cuh"

#include <hh.h>

#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

namespace {

constexpr int  kMergeRhs = 64;          // right-hand sides in one merged batch at most
constexpr long kMergePoints = 1L << 22; // requests with more points than this run on their own
// memory the pool reserves at creation (up to the budget): a fresh pool grows as plans and
// staging arrive, and a growth can stall the dispatcher for tens of milliseconds
constexpr size_t kReserveBytes = 64ull << 30;

using Key = std::tuple<int, int, int, double, double>; // dim, n, order, k_re, k_im

struct Req {
    long long       id = 0;
    hh_request      r{};
    hh_request_info info{};
    bool            done = false;
    std::string     err;
};

struct PlanEntry {
    hh_plan *plan = nullptr;
    size_t   bytes = 0;
    int      inflight = 0;
    long     last_use = 0;
};

struct Batch;

} // namespace

struct hh_server {
    int                                 device = 0;
    hh_ctx                             *ctx = nullptr;
    std::vector<cudaStream_t>           streams;
    cudaStream_t                        setup = nullptr;   // plan set-up (asynchronous)
    cudaEvent_t                         ready = nullptr;   // set-up done, per plan creation
    cudaMemPool_t                       pool = nullptr;
    int                                *flags = nullptr; // pinned, one slot per stream
    // device error words, one per stream: a batch clears its stream's word first and copies it to
    // its flag slot last, so an expired wait fails only the batch whose kernel reported it
    int                                *words = nullptr;
    int                                *own_word = nullptr; // the context's own word (restored at exit)
    int                                 inject = 0;         // batches still to fail (hh_server_inject_error)
    size_t                              budget = 0, used = 0;
    std::mutex                          m;
    std::condition_variable             cv;
    std::deque<Req *>                   queue;
    std::map<long long, Req *>          reqs;
    std::map<Key, PlanEntry>            plans;
    long long                           next_id = 1, completed = 0;
    long                                tick = 0;
    int                                 inflight = 0, rr = 0;
    bool                                stop = false;
    std::thread                         worker;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

struct Batch {
    hh_server         *s = nullptr;
    std::vector<Req *> reqs;             // grouped by plan: the requests of keys[i] are consecutive
    std::vector<Key>   keys;             // the batch's plans (one per distinct k)
    std::vector<int>   counts;           // right-hand sides per plan, in keys order
    size_t             staging = 0;
    bool               reserved = false; // staging counted in s->used
    bool               plan_ref = false; // holds an in-flight reference on each of its plans
    int               *flag = nullptr;   // pinned copy of the device error word after the batch
};

Key key_of(const hh_request &r) { return Key{r.dim, r.n, r.order, r.k_re, r.k_im}; }

long points_of(const hh_request &r) {
    long p = 1;
    for (int d = 0; d < r.dim; d++) p *= r.n;
    return p;
}

size_t plan_bytes(const hh_request &r) {
    // segment pivots (2 per 16 points), row tables, multipliers: a conservative estimate
    return (size_t)(2 * points_of(r)) * 16 + (size_t)r.n * 4096 + (1 << 20);
}

// completion: runs on a CUDA host-function thread after the batch's last operation (no CUDA calls)
void batch_done(void *arg) {
    Batch     *b = static_cast<Batch *>(arg);
    hh_server *s = b->s;
    {
        std::lock_guard<std::mutex> g(s->m);
        const double t = s->now();
        const bool   bad = b->flag && *b->flag != 0; // a kernel of this context hit a bounded wait
        for (Req *q : b->reqs) {
            q->done = true;
            q->info.t_done = t;
            q->info.status = bad ? HH_ERR_DEVICE : HH_OK;
            if (bad) q->err = "a kernel reported an expired bounded wait";
        }
        s->used -= b->staging;
        s->inflight--;
        s->completed += (long long)b->reqs.size();
        for (const Key &k : b->keys) {
            auto it = s->plans.find(k);
            if (it != s->plans.end()) it->second.inflight--;
        }
    }
    s->cv.notify_all();
    delete b;
}

// the batch could not run: release what it holds and complete its requests with `rc` (lock not held)
void fail_batch(hh_server *s, Batch *b, int rc, const std::string &msg) {
    {
        std::lock_guard<std::mutex> g(s->m);
        const double t = s->now();
        for (Req *q : b->reqs) {
            q->done = true;
            q->info.t_done = t;
            q->info.status = rc;
            q->err = msg;
        }
        if (b->reserved) s->used -= b->staging;
        s->inflight--;
        if (b->plan_ref)
            for (const Key &k : b->keys) {
                auto it = s->plans.find(k);
                if (it != s->plans.end()) it->second.inflight--;
            }
    }
    s->cv.notify_all();
    delete b;
}

// idle plans to evict, least recently used first, until `need` more bytes fit; they leave the map
// and the budget here and are destroyed by the caller without the lock (destroying a plan
// synchronizes the device, which waits for completion callbacks that take the lock)
std::vector<hh_plan *> pick_victims(hh_server *s, size_t need) {
    std::vector<hh_plan *> out;
    while (s->used + need > s->budget) {
        auto victim = s->plans.end();
        for (auto it = s->plans.begin(); it != s->plans.end(); ++it)
            if (it->second.inflight == 0 && (victim == s->plans.end() || it->second.last_use < victim->second.last_use))
                victim = it;
        if (victim == s->plans.end()) break;
        out.push_back(victim->second.plan);
        s->used -= victim->second.bytes;
        s->plans.erase(victim);
    }
    return out;
}

// Enqueue the batch on the next stream.  On failure nothing of it is left in flight.
int run_batch(hh_server *s, Batch *b, const std::vector<hh_plan *> &plans, cudaEvent_t after) {
    const hh_request &r0 = b->reqs[0]->r;
    const long        field = points_of(r0);
    const int         si = s->rr++ % (int)s->streams.size();
    cudaStream_t      st = s->streams[(size_t)si];
    double2          *buf = nullptr;
    void             *tab = nullptr;
    hh::Ctx          *cx = reinterpret_cast<hh::Ctx *>(s->ctx); // Ctx is hh_ctx's first member
    std::vector<hh::Plan *> ps;
    for (hh_plan *pl : plans) ps.push_back(reinterpret_cast<hh::Plan *>(pl)); // Plan is hh_plan's first member
    bool              inject = false;
    {
        std::lock_guard<std::mutex> g(s->m);
        if (s->inject > 0) {
            s->inject--;
            inject = true;
        }
    }
    auto enqueue = [&]() -> int {
        HH_TRY(hh_ctx_set_stream(s->ctx, st));
        cx->err_word = s->words + si; // the kernels of this batch report into its stream's word
        HH_CUDA(cudaMemsetAsync(cx->err_word, 0, sizeof(int), st));
        if (after) HH_CUDA(cudaStreamWaitEvent(st, after, 0)); // the plan's set-up
        int total = 0;
        for (Req *q : b->reqs) total += q->r.nrhs;
        // the multi-plan chunk table of this batch, from the pool in stream order
        HH_CUDA(cudaMallocFromPoolAsync(&tab, hh::line_solve_multi_table_bytes((int)ps.size(), total), s->pool, st));
        if (b->staging == 0) { // straight from the caller's device buffers
            HH_TRY(hh::solve_source_multi(ps.data(), b->counts.data(), (int)ps.size(), (const double2 *)r0.f,
                                          (double2 *)r0.u, tab));
        } else {
            HH_CUDA(cudaMallocFromPoolAsync((void **)&buf, b->staging, s->pool, st));
            long off = 0;
            for (Req *q : b->reqs) {
                const size_t bytes = sizeof(double2) * (size_t)field * q->r.nrhs;
                HH_CUDA(cudaMemcpyAsync(buf + off, q->r.f, bytes,
                                        q->r.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
                off += field * q->r.nrhs;
            }
            HH_TRY(hh::solve_source_multi(ps.data(), b->counts.data(), (int)ps.size(), buf, buf, tab));
            off = 0;
            for (Req *q : b->reqs) {
                const size_t bytes = sizeof(double2) * (size_t)field * q->r.nrhs;
                HH_CUDA(cudaMemcpyAsync(q->r.u, buf + off, bytes,
                                        q->r.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
                off += field * q->r.nrhs;
            }
            HH_CUDA(cudaFreeAsync(buf, st));
            buf = nullptr;
        }
        HH_CUDA(cudaFreeAsync(tab, st));
        tab = nullptr;
        if (inject) HH_CUDA(cudaMemsetAsync(cx->err_word, 1, 1, st)); // as if a wait had expired
        b->flag = s->flags + si;
        HH_CUDA(cudaMemcpyAsync(b->flag, cx->err_word, sizeof(int), cudaMemcpyDeviceToHost, st));
        HH_CUDA(cudaLaunchHostFunc(st, batch_done, b));
        return HH_OK;
    };
    const int rc = enqueue();
    if (rc != HH_OK) {
        cudaStreamSynchronize(st); // copies already queued must not outlive the request
        if (buf) cudaFree(buf);
        if (tab) cudaFree(tab);
    }
    return rc;
}

void dispatcher(hh_server *s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->m);
    for (;;) {
        s->cv.wait(lk, [&] { return s->stop || !s->queue.empty(); });
        if (s->queue.empty()) {
            if (s->stop) break;
            continue;
        }
        // the head request and every queued small request of the same shape (dim, n, order), at any
        // k: one batch over several plans (continuous batching)
        Req       *head = s->queue.front();
        const long field = points_of(head->r);
        Batch     *b = new Batch;
        b->s = s;
        std::vector<Req *> picked{head};
        int rhs = head->r.nrhs;
        if (field * head->r.nrhs <= kMergePoints) {
            // a merged batch never needs more than the whole budget on its own: its staging plus
            // the plans it would create
            std::vector<Key> seen{key_of(head->r)};
            int fresh_plans = s->plans.count(seen[0]) ? 0 : 1;
            for (Req *q : s->queue) {
                if (q == head || rhs >= kMergeRhs) continue;
                if (q->r.dim == head->r.dim && q->r.n == head->r.n && q->r.order == head->r.order &&
                    field * q->r.nrhs <= kMergePoints && rhs + q->r.nrhs <= kMergeRhs) {
                    const Key  kq = key_of(q->r);
                    const bool add_key = std::find(seen.begin(), seen.end(), kq) == seen.end();
                    const int  fp = fresh_plans + (add_key && !s->plans.count(kq) ? 1 : 0);
                    const size_t need_q = sizeof(double2) * (size_t)field * (rhs + q->r.nrhs) + fp * plan_bytes(head->r);
                    if (need_q > s->budget) continue;
                    if (add_key) seen.push_back(kq);
                    fresh_plans = fp;
                    picked.push_back(q);
                    rhs += q->r.nrhs;
                }
            }
        }
        // group by plan (first appearance order), so that each plan's fields are consecutive
        for (Req *q : picked) {
            const Key k = key_of(q->r);
            if (std::find(b->keys.begin(), b->keys.end(), k) == b->keys.end()) {
                b->keys.push_back(k);
                b->counts.push_back(0);
            }
        }
        for (size_t i = 0; i < b->keys.size(); i++)
            for (Req *q : picked)
                if (key_of(q->r) == b->keys[i]) {
                    b->reqs.push_back(q);
                    b->counts[i] += q->r.nrhs;
                }
        const bool direct = b->reqs.size() == 1 && head->r.on_device;
        b->staging = direct ? 0 : sizeof(double2) * (size_t)field * rhs;
        auto new_plan_bytes = [&]() {
            size_t x = 0;
            for (const Key &k : b->keys)
                if (!s->plans.count(k)) x += plan_bytes(head->r);
            return x;
        };
        auto need = [&]() { return b->staging + new_plan_bytes(); };
        // admission by HBM budget: wait for running batches, then evict idle plans
        while (s->used + need() > s->budget && s->inflight > 0) s->cv.wait(lk);
        // plans of this batch are not victims: hold them while evicting
        for (const Key &k : b->keys) {
            auto it = s->plans.find(k);
            if (it != s->plans.end()) it->second.inflight++;
        }
        std::vector<hh_plan *> victims = pick_victims(s, need());
        for (const Key &k : b->keys) {
            auto it = s->plans.find(k);
            if (it != s->plans.end()) it->second.inflight--;
        }
        if (!victims.empty()) {
            lk.unlock();
            hh_ctx_set_stream(s->ctx, s->setup); // idle plans: their memory returns to the pool in order
            for (hh_plan *v : victims) hh_plan_destroy(v);
            lk.lock();
        }
        for (Req *q : b->reqs) s->queue.erase(std::find(s->queue.begin(), s->queue.end(), q));
        const double t = s->now();
        for (Req *q : b->reqs) {
            q->info.t_start = t;
            q->info.batch_rhs = rhs;
        }
        s->inflight++;
        std::vector<Key> create;
        for (const Key &k : b->keys)
            if (!s->plans.count(k)) create.push_back(k);
        const size_t pbytes = create.size() * plan_bytes(head->r);
        if (s->used + b->staging + pbytes > s->budget) {
            lk.unlock();
            fail_batch(s, b, HH_ERR_NOMEM, "request does not fit in the server's HBM budget");
            lk.lock();
            continue;
        }
        s->used += b->staging + pbytes; // staging and (reserved) plan memory
        b->reserved = true;
        bool fresh = false;
        if (!create.empty()) {
            lk.unlock();
            // asynchronous set-up on its own stream; the batch waits for it with an event
            int rc = hh_ctx_set_stream(s->ctx, s->setup);
            std::vector<hh_plan *> made;
            for (const Key &k : create) {
                if (rc != HH_OK) break;
                const int dim = std::get<0>(k), n = std::get<1>(k), order = std::get<2>(k);
                const double kr = std::get<3>(k), ki = std::get<4>(k);
                hh_plan *plan = nullptr;
                rc = dim == 2 ? hh_plan2d_create_helmholtz(s->ctx, n, order, kr, ki, &plan)
                              : hh_plan3d_create_helmholtz(s->ctx, n, order, kr, ki, &plan);
                int tuned = 0; // the kernel settings hh_plan_tune found for this shape, if any (never measures)
                if (rc == HH_OK) rc = hh_plan_apply_tuning(plan, &tuned);
                if (plan) made.push_back(plan);
            }
            if (rc == HH_OK && cudaEventRecord(s->ready, s->setup) != cudaSuccess) rc = HH_ERR_CUDA;
            const std::string msg = rc == HH_OK ? std::string() : std::string(hh_last_error());
            fresh = rc == HH_OK;
            if (rc != HH_OK)
                for (hh_plan *pl : made) hh_plan_destroy(pl);
            lk.lock();
            if (rc != HH_OK) {
                s->used -= pbytes;
                lk.unlock();
                fail_batch(s, b, rc, msg);
                lk.lock();
                continue;
            }
            for (size_t i = 0; i < create.size(); i++) {
                PlanEntry e;
                e.plan = made[i];
                e.bytes = plan_bytes(head->r);
                s->plans.emplace(create[i], e);
            }
        }
        std::vector<hh_plan *> plans;
        for (const Key &k : b->keys) {
            PlanEntry &pe = s->plans[k];
            pe.inflight++;
            pe.last_use = ++s->tick;
            plans.push_back(pe.plan);
        }
        b->plan_ref = true;
        lk.unlock();
        const int rc = run_batch(s, b, plans, fresh ? s->ready : nullptr);
        if (rc != HH_OK) fail_batch(s, b, rc, hh_last_error());
        lk.lock();
    }
}

bool valid(const hh_request *r) {
    return r && (r->dim == 2 || r->dim == 3) && r->n >= 1 && (r->order == 2 || r->order == 4 || r->order == 6) &&
           r->nrhs >= 1 && r->nrhs <= 65535 && r->f && r->u;
}

} // namespace

using hh::set_error;

extern "C" int hh_server_create(int device, size_t budget, int streams, hh_server **out) {
    if (!out || streams < 1 || streams > 64 || budget == 0) {
        set_error("hh_server_create: invalid arguments");
        return HH_ERR_INVALID;
    }
    *out = nullptr;
    hh_server *s = new hh_server;
    s->device = device;
    s->budget = budget;
    int rc = hh_ctx_create(device, nullptr, &s->ctx);
    if (rc != HH_OK) { delete s; return rc; }
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaError_t e = cudaMemPoolCreate(&s->pool, &props);
    if (e == cudaSuccess) {
        unsigned long long keep = (unsigned long long)budget; // keep freed staging in the pool up to the budget
        e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e == cudaSuccess) { // reserve the pool's memory up front: one allocation, freed at once
        cudaStream_t ws = nullptr;
        void        *w = nullptr;
        e = cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking);
        const size_t wb = std::min(budget, kReserveBytes);
        if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&w, wb, s->pool, ws);
        if (e == cudaSuccess) e = cudaFreeAsync(w, ws);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ws);
        if (ws) cudaStreamDestroy(ws);
    }
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&s->flags, sizeof(int) * 64, cudaHostAllocDefault);
    if (e == cudaSuccess) memset(s->flags, 0, sizeof(int) * 64);
    if (e == cudaSuccess) e = cudaMalloc((void **)&s->words, sizeof(int) * 64);
    if (e == cudaSuccess) e = cudaMemset(s->words, 0, sizeof(int) * 64);
    if (e == cudaSuccess) s->own_word = reinterpret_cast<hh::Ctx *>(s->ctx)->err_word;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->setup, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ready, cudaEventDisableTiming);
    if (e == cudaSuccess) reinterpret_cast<hh::Ctx *>(s->ctx)->pool = s->pool;
    for (int i = 0; i < streams && e == cudaSuccess; i++) {
        cudaStream_t st;
        e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e == cudaSuccess) s->streams.push_back(st);
    }
    if (e != cudaSuccess) {
        set_error("hh_server_create: %s", cudaGetErrorString(e));
        for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
        if (s->pool) cudaMemPoolDestroy(s->pool);
        if (s->flags) cudaFreeHost(s->flags);
        if (s->words) cudaFree(s->words);
        hh_ctx_destroy(s->ctx);
        delete s;
        return HH_ERR_CUDA;
    }
    s->worker = std::thread(dispatcher, s);
    *out = s;
    return HH_OK;
}

extern "C" int hh_server_submit(hh_server *s, const hh_request *r, long long *id) {
    if (!s || !valid(r) || !id) {
        set_error("hh_server_submit: invalid request");
        return HH_ERR_INVALID;
    }
    Req *q = new Req;
    q->r = *r;
    {
        std::lock_guard<std::mutex> g(s->m);
        if (s->stop) {
            delete q;
            set_error("hh_server_submit: server is shutting down");
            return HH_ERR_INVALID;
        }
        q->id = s->next_id++;
        q->info.t_submit = s->now();
        s->reqs[q->id] = q;
        s->queue.push_back(q);
        *id = q->id;
    }
    s->cv.notify_all();
    return HH_OK;
}

extern "C" int hh_server_wait(hh_server *s, long long id, hh_request_info *info) {
    if (!s) return HH_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->m);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) {
        set_error("hh_server_wait: unknown request %lld", id);
        return HH_ERR_INVALID;
    }
    Req *q = it->second;
    s->cv.wait(lk, [&] { return q->done; });
    if (info) *info = q->info;
    const int rc = q->info.status;
    if (rc != HH_OK) set_error("%s", q->err.c_str());
    s->reqs.erase(it);
    delete q;
    return rc;
}

extern "C" int hh_server_stats(hh_server *s, long long *done, size_t *bytes_in_use, int *plans) {
    if (!s) return HH_ERR_INVALID;
    std::lock_guard<std::mutex> g(s->m);
    if (done) *done = s->completed;
    if (bytes_in_use) *bytes_in_use = s->used;
    if (plans) *plans = (int)s->plans.size();
    return HH_OK;
}

extern "C" double hh_server_clock(hh_server *s) { return s ? s->now() : 0.0; }

extern "C" int hh_server_destroy(hh_server *s) {
    if (!s) return HH_OK;
    {
        std::lock_guard<std::mutex> g(s->m);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    // let every batch finish (their host functions touch the server)
    for (cudaStream_t st : s->streams) cudaStreamSynchronize(st);
    {
        std::unique_lock<std::mutex> lk(s->m);
        s->cv.wait(lk, [&] { return s->inflight == 0; });
    }
    for (auto &kv : s->plans) hh_plan_destroy(kv.second.plan);
    for (auto &kv : s->reqs) delete kv.second;
    cudaStreamSynchronize(s->setup);
    reinterpret_cast<hh::Ctx *>(s->ctx)->err_word = s->own_word; // the context frees its own word
    hh_ctx_destroy(s->ctx); // while its current stream (one of the server's) still exists
    for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
    cudaStreamDestroy(s->setup);
    cudaEventDestroy(s->ready);
    cudaMemPoolDestroy(s->pool);
    cudaFreeHost(s->flags);
    cudaFree(s->words);
    delete s;
    return HH_OK;
}

extern "C" int hh_server_inject_wait_expiry(hh_server *s) {
    if (!s) {
        set_error("hh_server_inject_wait_expiry: null server");
        return HH_ERR_INVALID;
    }
    // the dispatcher owns the context's stream: write the word synchronously instead
    const int one = 1;
    cudaError_t e = cudaSetDevice(s->device);
    if (e == cudaSuccess)
        e = cudaMemcpy(reinterpret_cast<hh::Ctx *>(s->ctx)->inject_word, &one, sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        set_error("hh_server_inject_wait_expiry: %s", cudaGetErrorString(e));
        return HH_ERR_CUDA;
    }
    return HH_OK;
}

extern "C" int hh_server_inject_error(hh_server *s, int batches) {
    if (!s || batches < 0) {
        set_error("hh_server_inject_error: invalid arguments");
        return HH_ERR_INVALID;
    }
    std::lock_guard<std::mutex> g(s->m);
    s->inject = batches;
    return HH_OK;
}
