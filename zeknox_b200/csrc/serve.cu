// Batched and served commits (extensions; no zeknox counterpart).
//
// zk_commit_batch: many commit jobs (coset LDE -> leaves -> Merkle forest) of
// different sizes in one call.  The caller's stream is forked onto K internal
// streams; jobs go to streams largest-first onto the least-loaded stream (LPT),
// so small jobs overlap with each other and with the latency-bound tops of
// larger trees; the internal streams join back into the caller's stream.
// Everything is stream-ordered (pool allocations included), so a batch can be
// captured into a CUDA graph once its tables exist (run it once uncaptured).
//
// ZkServer: a request loop for commits that arrive over time.  A dispatcher
// thread admits queued jobs onto free slots while their device memory fits an
// HBM budget (reserved in the server's memory pool when it starts, so an
// admitted job rarely waits for physical memory); each slot's worker thread
// allocates and launches the jobs admitted to it, and admitted jobs run
// concurrently.  Admission is first in, first out, with one exception that
// is bounded per job: every job carries a delay budget, a fraction of its own
// estimated GPU time alone (est, from its size).  A job may start ahead of
// older queued jobs, or beside running ones, only if its est fits in the
// remaining budget of every one of those jobs, and starting it charges its
// est to each of them.  So no job is delayed, by jobs that arrived after it,
// by more than its budget (a long job's latency grows by at most that
// fraction of its own service time), while short jobs start at once beside
// long ones instead of queueing behind them; among the jobs that may start,
// the shortest goes first.  Only relative sizes enter: estimates that are
// off by a common factor change nothing.  While the oldest job waits for
// memory, others are admitted
// only if they leave room for it.  Jobs under 20 ms of estimated GPU time run
// on high-priority streams, so their blocks are scheduled onto SMs ahead of
// those of larger jobs already running.  The tree (leaves + digests + cap) of
// every job stays resident on the device until the client releases it; the
// cap is also copied to the host.  Completions are queued in order for
// zk_server_wait_any.  Latency (submit to completion of the cap copy) is
// recorded for p50 / p99.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/zeknox.h"
#include "admission.h"
#include "merkle.cuh"
#include "ntt.cuh"
#include "runtime.cuh"

using namespace zk;

namespace {

RustError ok_err() { return RustError{0, nullptr}; }
RustError mk_err(int code, const char *m) { return RustError{code, m ? strdup(m) : nullptr}; }

template <class F>
RustError guard(F &&f) {
    try {
        f();
        return ok_err();
    } catch (const Error &e) {
        return mk_err(e.code, e.what());
    } catch (const std::exception &e) {
        return mk_err(-(int)cudaErrorUnknown, e.what());
    }
}

struct Shape {
    uint32_t lg_n, rate, batches, cap_h, hash;
    uint64_t N() const { return 1ull << (lg_n + rate); }
    uint64_t n() const { return 1ull << lg_n; }
    uint64_t n_caps() const { return 1ull << cap_h; }
    uint64_t n_digests() const { return 2 * (N() - n_caps()); }
    // Work estimate: permutations (leaf sponge + nodes).
    double work() const {
        const uint64_t rate_words = hash == 1 ? 17 : 8;
        return (double)N() * ((batches + rate_words - 1) / rate_words + 1);
    }
    uint64_t coeff_bytes() const { return n() * batches * 8; }
    uint64_t leaf_bytes() const { return N() * batches * 8; }
    uint64_t digest_bytes() const { return n_digests() * 32; }
    uint64_t cap_bytes() const { return n_caps() * 32; }
    uint64_t scratch_bytes() const { return ntt_leaves_scratch_elems(lg_n + rate, batches) * 8; }
};

void validate(const Shape &s) {
    require(s.lg_n >= 1 && s.rate >= 1 && s.lg_n + s.rate <= 30, "invalid LDE size");
    require(s.batches >= 1, "empty job");
    require(s.cap_h <= s.lg_n + s.rate, "cap_height larger than the tree");
    require(merkle_hash_supported(s.hash), "unsupported hash type");
}

// The Merkle forest of a commit's leaves on `st`.
void forest_on(const Shape &sh, const uint64_t *leaves, uint64_t *digests, uint64_t *cap, cudaStream_t st) {
    MerkleJob m;
    m.digests = digests;
    m.cap = cap;
    m.leaves = leaves;
    m.n_digests = sh.n_digests();
    m.n_caps = sh.n_caps();
    m.n_leaves = sh.N();
    m.leaf_size = sh.batches;
    m.cap_height = sh.cap_h;
    m.hash_type = sh.hash;
    merkle_run(m, st);
}

// The LDE in leaf layout of polynomials [b0, b0 + nb) of a commit: a column
// slice of the leaf matrix.
void lde_leaves_slice(DeviceCtx &ctx, const Shape &sh, const uint64_t *coeffs, uint64_t *leaves, uint64_t *scratch,
                      uint64_t b0, uint64_t nb, cudaStream_t st) {
    const uint32_t lg = sh.lg_n + sh.rate;
    NttJob j;
    j.src = coeffs + b0 * sh.n();
    j.src_stride = sh.n();
    j.n_valid = sh.n();
    j.dst = leaves + b0;
    j.batches = nb;
    j.leaf_stride = sh.batches;
    j.lg = lg;
    j.pre_coset = &coset_table(ctx, lg, GROUP_GENERATOR, false);
    j.to_leaves = true;
    j.scratch = scratch;
    j.scratch_elems = ntt_leaves_scratch_elems(lg, nb);
    ntt_run(j, st);
}

// One commit on `st` from host coefficients: the copy goes in groups of
// polynomials on `cs` (4 groups from 16 polynomials, 8 from 32), and each
// group's LDE starts on `st` as soon as its copy has landed, so the copy of a
// large job is hidden behind its own transform instead of preceding it.
void commit_from_host(DeviceCtx &ctx, const Shape &sh, const void *host, uint64_t *coeffs, uint64_t *leaves,
                      uint64_t *digests, uint64_t *cap, uint64_t *scratch, cudaStream_t st, cudaStream_t cs) {
    const uint64_t B = sh.batches, n = sh.n();
    const uint64_t groups = B < 16 ? 1 : (B < 32 ? 4 : 8);
    const uint64_t gsz = (B + groups - 1) / groups;
    std::vector<cudaEvent_t> ev;
    auto record = [&](cudaStream_t on) {
        cudaEvent_t e;
        ZK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ev.push_back(e);
        ZK_CUDA(cudaEventRecord(e, on));
        return e;
    };
    try {
        ZK_CUDA(cudaStreamWaitEvent(cs, record(st), 0));  // after the allocations on st
        for (uint64_t b0 = 0; b0 < B; b0 += gsz) {
            const uint64_t nb = std::min(gsz, B - b0);
            ZK_CUDA(cudaMemcpyAsync(coeffs + b0 * n, (const uint64_t *)host + b0 * n, nb * n * sizeof(uint64_t),
                                    cudaMemcpyHostToDevice, cs));
            ZK_CUDA(cudaStreamWaitEvent(st, record(cs), 0));
            lde_leaves_slice(ctx, sh, coeffs, leaves, scratch, b0, nb, st);
        }
    } catch (...) {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);  // released once their work completes
        throw;
    }
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    forest_on(sh, leaves, digests, cap, st);
}

// One commit on `st`: LDE in leaf layout (scratch supplied), then the forest.
void commit_on(DeviceCtx &ctx, const Shape &sh, const uint64_t *coeffs, uint64_t *leaves, uint64_t *digests,
               uint64_t *cap, uint64_t *scratch, cudaStream_t st) {
    lde_leaves_slice(ctx, sh, coeffs, leaves, scratch, 0, sh.batches, st);
    forest_on(sh, leaves, digests, cap, st);
}

// Per-device pool of internal streams for batches.
struct StreamSet {
    std::vector<cudaStream_t> s;
    std::vector<cudaEvent_t> ev;
};
std::mutex g_ss_mu;
std::unordered_map<int, std::unique_ptr<StreamSet>> g_ss;

StreamSet &streams_for(int dev, uint32_t k) {
    std::lock_guard<std::mutex> g(g_ss_mu);
    auto &p = g_ss[dev];
    if (!p) p = std::make_unique<StreamSet>();
    while (p->s.size() < k) {
        cudaStream_t st;
        cudaEvent_t e;
        ZK_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        ZK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        p->s.push_back(st);
        p->ev.push_back(e);
    }
    return *p;
}

}  // namespace

// ------------------------------------------------------------------- batch

extern "C" RustError zk_commit_batch(const ZkCommitJob *jobs, uint32_t n_jobs, uint32_t n_streams, void *stream) {
    return guard([&] {
        require(jobs != nullptr || n_jobs == 0, "null job list");
        if (n_jobs == 0) return;
        const int dev = current_device();
        DeviceCtx &ctx = device_ctx(dev);
        const uint32_t k = std::max<uint32_t>(1, std::min<uint32_t>(n_streams ? n_streams : 4, 16));
        std::vector<Shape> sh(n_jobs);
        for (uint32_t i = 0; i < n_jobs; i++) {
            const ZkCommitJob &J = jobs[i];
            sh[i] = Shape{J.lg_n, J.rate_bits, J.batches, J.cap_height, J.hash_type};
            validate(sh[i]);
            require(J.d_coeffs && J.d_leaves && J.d_cap && (J.d_digests || sh[i].n_digests() == 0), "null buffer");
            // Tables first, outside any stream work (creating them synchronises).
            coset_table(ctx, J.lg_n + J.rate_bits, GROUP_GENERATOR, false);
            root_table(ctx, J.lg_n + J.rate_bits, false);
        }
        line_roots(ctx, false);
        // LPT: largest job first onto the least-loaded stream.
        std::vector<uint32_t> order(n_jobs);
        for (uint32_t i = 0; i < n_jobs; i++) order[i] = i;
        std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return sh[a].work() > sh[b].work(); });
        std::vector<double> load(k, 0.0);
        std::vector<std::vector<uint32_t>> per(k);
        std::vector<uint64_t> scratch_need(k, 0);
        for (uint32_t i : order) {
            const uint32_t s = (uint32_t)(std::min_element(load.begin(), load.end()) - load.begin());
            load[s] += sh[i].work();
            per[s].push_back(i);
            scratch_need[s] = std::max(scratch_need[s], sh[i].scratch_bytes());
        }
        StreamSet &ss = streams_for(dev, k);
        cudaStream_t caller = (cudaStream_t)stream;
        cudaEvent_t fork;
        ZK_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
        ZK_CUDA(cudaEventRecord(fork, caller));
        for (uint32_t s = 0; s < k; s++) {
            if (per[s].empty()) continue;
            cudaStream_t st = ss.s[s];
            ZK_CUDA(cudaStreamWaitEvent(st, fork, 0));
            Scratch scr(scratch_need[s], st);  // one scratch per stream, reused by its jobs
            for (uint32_t i : per[s]) {
                const ZkCommitJob &J = jobs[i];
                commit_on(ctx, sh[i], (const uint64_t *)J.d_coeffs, (uint64_t *)J.d_leaves, (uint64_t *)J.d_digests,
                          (uint64_t *)J.d_cap, scr.as<uint64_t>(), st);
            }
            // scr is freed (stream-ordered) here, after this stream's jobs
        }
        for (uint32_t s = 0; s < k; s++) {
            if (per[s].empty()) continue;
            ZK_CUDA(cudaEventRecord(ss.ev[s], ss.s[s]));
            ZK_CUDA(cudaStreamWaitEvent(caller, ss.ev[s], 0));
        }
        cudaEventDestroy(fork);
    });
}

// ------------------------------------------------------------- autotuner

extern "C" RustError zk_autotune_commit(uint32_t lg_n, uint32_t rate_bits, uint32_t batches, int32_t *timed) {
    return guard([&] {
        require(lg_n >= 1 && rate_bits >= 1 && lg_n + rate_bits <= 30 && batches >= 1, "invalid shape");
        const int dev = current_device();
        DeviceCtx &ctx = device_ctx(dev);
        root_table(ctx, lg_n + rate_bits, false);
        line_roots(ctx, false);
        int n = ntt_autotune_leaves(lg_n, rate_bits, batches, ctx.stream);
        n += merkle_autotune_leaves(1ull << (lg_n + rate_bits), batches, 0, ctx.stream);  // Poseidon leaves
        if (timed) *timed = n;
    });
}

extern "C" RustError zk_autotune_reset(void) {
    return guard([&] {
        ntt_autotune_clear();
        merkle_autotune_clear();
    });
}

// ------------------------------------------------------------------ server

struct ZkServer {
    struct Job {
        uint64_t ticket;
        Shape sh;
        const void *host_coeffs;
        std::chrono::steady_clock::time_point t_submit, t_done;
        uint64_t bytes = 0;         // device bytes held while resident
        uint64_t run_bytes = 0;     // extra bytes held while running (coeffs + scratch)
        uint64_t *d_coeffs = nullptr, *d_leaves = nullptr, *d_digests = nullptr, *d_cap = nullptr;
        uint64_t *d_scratch = nullptr;
        std::vector<uint64_t> cap;  // the cap on the host, filled when the job completes
        int slot = -1;
        double est_s = 0;           // estimated GPU time alone
        std::chrono::steady_clock::time_point t_admit{};  // when the dispatcher started it
        double alloc_s = 0;         // host time its device allocations took
        uint32_t fail_at = 0;       // injected failure: the 1-based allocation made to fail (0: none)
        double budget_s = 0;        // delay it may still take from later jobs started ahead of or beside it
        bool seeded = false;        // coefficients generated on the device from `seed`
        uint64_t seed = 0;
        cudaStream_t stream = nullptr;  // the stream the job ran on
        uint64_t seq = 0;           // submission order
        int state = 0;              // 0 queued, 1 running, 2 done, 3 failed
        int err = 0;
        std::string err_msg;        // why it failed (state 3)
    };
    int dev = 0;
    uint64_t budget = 0, in_use = 0, peak = 0;
    // Every job's delay budget: this fraction of its own estimated GPU time.
    double budget_frac = 0.05;
    // The server's own memory pool (the budget is reserved in it) and an idle
    // stream that released trees are freed on.  The pool never reuses a block
    // by making the new job's stream wait for the stream that freed it (no
    // internal dependencies): freed blocks are reused only once the free has
    // executed.  A tree freed on its slot's stream, which may already run the
    // next job, would otherwise tie a later job to that unrelated job.
    cudaMemPool_t pool = nullptr;
    cudaStream_t free_stream = nullptr;
    uint64_t reserved_start = 0;  // bytes the pool had mapped when the server started
    uint64_t ahead = 0;  // jobs started ahead of an older queued job or beside a running one
    double alloc_max_s = 0;  // longest time one job's device allocations took on the host
    // [slot][0]: high priority, [1]: normal priority, [2]: the slot's host-to-device copies
    std::vector<std::vector<cudaStream_t>> slots;
    // Per slot, pinned staging for the cap's device-to-host copy (grown by the
    // dispatcher when a larger cap comes along; the completion callback copies
    // it into the job), so that no job allocates or frees pinned memory: both
    // can synchronise with the device.
    std::vector<uint64_t *> slot_cap;
    std::vector<uint64_t> slot_cap_bytes;
    std::vector<bool> slot_busy;
    std::vector<uint64_t> running;     // tickets of admitted, unfinished jobs
    std::mutex mu;
    std::condition_variable cv;        // dispatcher wake-up
    std::condition_variable work_cv;   // slot workers' wake-up
    std::vector<uint64_t> slot_job;    // per slot: the ticket handed to its worker (0: none)
    std::vector<std::thread> workers;  // one per slot
    std::condition_variable done_cv;   // completions
    std::deque<uint64_t> queue;
    std::deque<uint64_t> done_q;       // completed or failed, not yet returned by wait_any
    uint64_t n_running = 0;
    std::unordered_map<uint64_t, std::unique_ptr<Job>> jobs;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::thread dispatcher;
    std::vector<double> latencies;     // seconds, completed jobs
    double elems_done = 0;
    uint64_t max_queue = 0;
    std::chrono::steady_clock::time_point t_first{}, t_last{};
    bool any = false;
    std::string fatal;
    // Host-side fault injection (zk_server_inject_failure): the next
    // inject_jobs admitted jobs fail at their inject_step-th device allocation.
    uint32_t inject_jobs = 0, inject_step = 0;

    void run();
    void work(int s);
    void start(Job &J, DeviceCtx &ctx);
    void fail_admitted(Job &J, const char *why);
    uint64_t submit(std::unique_ptr<Job> J);
};

namespace {

struct DoneCtx {
    ZkServer *srv;
    uint64_t ticket;
};

void CUDART_CB on_done(void *p) {
    std::unique_ptr<DoneCtx> d((DoneCtx *)p);
    ZkServer *srv = d->srv;
    std::lock_guard<std::mutex> g(srv->mu);
    auto it = srv->jobs.find(d->ticket);
    if (it == srv->jobs.end()) return;
    ZkServer::Job &J = *it->second;
    J.t_done = std::chrono::steady_clock::now();
    J.cap.assign(srv->slot_cap[J.slot], srv->slot_cap[J.slot] + J.sh.cap_bytes() / sizeof(uint64_t));
    J.state = 2;
    srv->slot_busy[J.slot] = false;
    srv->running.erase(std::find(srv->running.begin(), srv->running.end(), d->ticket));
    srv->n_running--;
    srv->done_q.push_back(d->ticket);
    srv->in_use -= J.run_bytes;  // coeffs + scratch were freed on the stream before this point
    srv->latencies.push_back(std::chrono::duration<double>(J.t_done - J.t_submit).count());
    srv->elems_done += (double)J.sh.N() * J.sh.batches;
    srv->t_last = J.t_done;
    srv->cv.notify_all();
    srv->done_cv.notify_all();
}

}  // namespace

void ZkServer::run() {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        cv.wait(lk, [&] {
            if (stop) return true;
            if (queue.empty()) return false;
            return std::find(slot_busy.begin(), slot_busy.end(), false) != slot_busy.end();
        });
        if (stop) return;
        // A job larger than the whole budget can never run: fail it.
        for (auto it = queue.begin(); it != queue.end();) {
            Job &J = *jobs[*it];
            if (J.bytes + J.run_bytes > budget) {
                J.state = 3;
                J.err = (int)cudaErrorMemoryAllocation;
                J.err_msg = "job larger than the HBM budget";
                done_q.push_back(*it);
                done_cv.notify_all();
                it = queue.erase(it);
            } else {
                ++it;
            }
        }
        if (queue.empty()) continue;
        // Budget admission (admission.h): FIFO, except that a shorter job may start
        // ahead of or beside the jobs whose delay budgets its estimate fits in.
        std::vector<uint64_t> order(queue.begin(), queue.end());  // the queue is kept in submission order
        std::vector<AdmitJob> aq(order.size());
        for (size_t q = 0; q < order.size(); q++) {
            const Job &J = *jobs[order[q]];
            aq[q] = AdmitJob{J.est_s, J.budget_s, J.bytes + J.run_bytes};
        }
        std::vector<double> rb(running.size());
        for (size_t i = 0; i < running.size(); i++) rb[i] = jobs[running[i]]->budget_s;
        const long pq = admission_pick(aq, rb, in_use, budget);
        if (pq < 0) {  // nothing can go until a job completes or memory is released
            cv.wait(lk);
            continue;
        }
        if (pq > 0 || !running.empty()) ahead++;
        admission_charge(aq, rb, pq);
        for (size_t i = 0; i < running.size(); i++) jobs[running[i]]->budget_s = rb[i];
        for (long q = 0; q < pq; q++) jobs[order[(size_t)q]]->budget_s = aq[(size_t)q].budget_s;
        const uint64_t t = order[(size_t)pq];
        queue.erase(queue.begin() + pq);
        Job &J = *jobs[t];
        const int s = (int)(std::find(slot_busy.begin(), slot_busy.end(), false) - slot_busy.begin());
        slot_busy[s] = true;
        J.slot = s;
        J.state = 1;
        J.t_admit = std::chrono::steady_clock::now();
        running.push_back(t);
        n_running++;
        in_use += J.bytes + J.run_bytes;
        peak = std::max(peak, in_use);
        if (inject_jobs) {
            inject_jobs--;
            J.fail_at = inject_step;
        }
        // The slot's worker allocates and launches, so that an allocation
        // which blocks on the host (the pool waiting for outstanding frees when
        // its free memory is fragmented; measured up to ~2 s for an 80 GB tree)
        // delays only this job, not the admission of every job behind it.
        slot_job[s] = t;
        work_cv.notify_all();
    }
}

// Slot s's worker: starts each job the dispatcher hands to the slot.
void ZkServer::work(int s) {
    ZK_CUDA(cudaSetDevice(dev));
    DeviceCtx &ctx = device_ctx(dev);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        work_cv.wait(lk, [&] { return stop || slot_job[s] != 0; });
        if (stop) return;  // a job handed over but not started is dropped with the server
        Job &J = *jobs[slot_job[s]];
        slot_job[s] = 0;
        lk.unlock();
        start(J, ctx);
        lk.lock();
    }
}

// Allocate a job's buffers from the pool and launch it on its slot's streams
// (called without `mu` held); a failure releases what it took (fail_admitted).
void ZkServer::start(Job &J, DeviceCtx &ctx) {
    const int s = J.slot;
    try {
        // priority by size: < 20 ms of estimated GPU time high, everything else normal.  (A third,
        // lowest level for the large jobs measured worse: 80 jobs at 0.75x load, p99 2.66 s and
        // throughput 0.95x FIFO, against 2.11 s and 0.99x with two levels.)
        cudaStream_t st = slots[s][J.est_s < 0.02 ? 0 : 1];
        J.stream = st;
        const Shape &sh = J.sh;
        if (slot_cap_bytes[s] < sh.cap_bytes()) {
            // Rare (a larger cap than this slot has staged so far).  The slot is
            // this job's, and its previous job's completion callback has run.
            if (slot_cap[s]) cudaFreeHost(slot_cap[s]);
            slot_cap[s] = nullptr;
            slot_cap_bytes[s] = 0;
            ZK_CUDA(cudaMallocHost((void **)&slot_cap[s], sh.cap_bytes()));
            slot_cap_bytes[s] = sh.cap_bytes();
        }
        uint32_t step = 0;
        auto alloc = [&](uint64_t **p, uint64_t bytes) {
            if (++step == J.fail_at) throw Error((int)cudaErrorMemoryAllocation, "injected allocation failure");
            ZK_CUDA(cudaMallocFromPoolAsync((void **)p, bytes, pool, st));
        };
        const auto ta = std::chrono::steady_clock::now();
        alloc(&J.d_coeffs, sh.coeff_bytes());
        alloc(&J.d_leaves, sh.leaf_bytes());
        if (sh.n_digests()) alloc(&J.d_digests, sh.digest_bytes());
        alloc(&J.d_cap, sh.cap_bytes());
        if (sh.scratch_bytes()) alloc(&J.d_scratch, sh.scratch_bytes());
        J.alloc_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - ta).count();
        {
            std::lock_guard<std::mutex> g(mu);
            alloc_max_s = std::max(alloc_max_s, J.alloc_s);
        }
        if (J.seeded) {
            salt_run(J.d_coeffs, sh.n() * sh.batches, J.seed, st);  // the job's input, generated in place
            commit_on(ctx, sh, J.d_coeffs, J.d_leaves, J.d_digests, J.d_cap, J.d_scratch, st);
        } else {
            commit_from_host(ctx, sh, J.host_coeffs, J.d_coeffs, J.d_leaves, J.d_digests, J.d_cap, J.d_scratch,
                             st, slots[s][2]);
        }
        ZK_CUDA(cudaMemcpyAsync(slot_cap[s], J.d_cap, sh.cap_bytes(), cudaMemcpyDeviceToHost, st));
        ZK_CUDA(cudaFreeAsync(J.d_coeffs, st));
        J.d_coeffs = nullptr;
        if (J.d_scratch) ZK_CUDA(cudaFreeAsync(J.d_scratch, st));
        J.d_scratch = nullptr;
        ZK_CUDA(cudaLaunchHostFunc(st, on_done, new DoneCtx{this, J.ticket}));
    } catch (const Error &e) {
        J.err = e.code;
        fail_admitted(J, e.what());
    } catch (const std::exception &e) {
        J.err = -(int)cudaErrorUnknown;
        fail_admitted(J, e.what());
    }
}

// A job that failed after admission (an allocation or a launch threw): wait
// for whatever of its work was already queued on its slot's streams, free the
// allocations it made, then release its slot and its share of the budget, so
// later jobs run as if it had never been admitted.  Called without `mu` held.
void ZkServer::fail_admitted(Job &J, const char *why) {
    const int s = J.slot;
    for (cudaStream_t st : slots[s]) cudaStreamSynchronize(st);
    for (uint64_t **p : {&J.d_coeffs, &J.d_leaves, &J.d_digests, &J.d_cap, &J.d_scratch}) {
        if (*p) cudaFreeAsync(*p, J.stream ? J.stream : slots[s][1]);
        *p = nullptr;
    }
    for (cudaStream_t st : slots[s]) cudaStreamSynchronize(st);
    cudaGetLastError();  // the failure is reported through the job, not left for the next call
    std::lock_guard<std::mutex> g(mu);
    J.state = 3;
    J.err_msg = why ? why : "job failed";
    slot_busy[s] = false;
    running.erase(std::find(running.begin(), running.end(), J.ticket));
    n_running--;
    done_q.push_back(J.ticket);
    in_use -= J.bytes + J.run_bytes;
    cv.notify_all();
    done_cv.notify_all();
}

extern "C" RustError zk_server_create(int32_t device, uint64_t hbm_budget_bytes, uint32_t n_slots, ZkServer **out) {
    return guard([&] {
        require(out != nullptr && n_slots >= 1 && n_slots <= 64 && hbm_budget_bytes > 0, "invalid server arguments");
        ZK_CUDA(cudaSetDevice(device));
        device_ctx(device);
        auto srv = std::make_unique<ZkServer>();
        srv->dev = device;
        srv->budget = hbm_budget_bytes;
        // ZK_SERVER_BUDGET_FRAC overrides the delay budget (a fraction of each job's own
        // estimated GPU time; 0 = first in, first out, one job at a time).
        if (const char *e = getenv("ZK_SERVER_BUDGET_FRAC")) srv->budget_frac = std::max(0.0, atof(e));
        int least = 0, greatest = 0;
        ZK_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        const int levels[2] = {greatest, (greatest + least) / 2};  // high, normal
        for (uint32_t i = 0; i < n_slots; i++) {
            std::vector<cudaStream_t> per;
            for (int lv : levels) {
                cudaStream_t st;
                ZK_CUDA(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, lv));
                per.push_back(st);
            }
            cudaStream_t cs;
            ZK_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
            per.push_back(cs);
            srv->slots.push_back(per);
            srv->slot_busy.push_back(false);
            srv->slot_job.push_back(0);
            uint64_t *staging = nullptr;
            ZK_CUDA(cudaMallocHost((void **)&staging, 64 << 10));  // caps of up to 2^11 digests
            srv->slot_cap.push_back(staging);
            srv->slot_cap_bytes.push_back(64 << 10);
        }
        ZK_CUDA(cudaStreamCreateWithFlags(&srv->free_stream, cudaStreamNonBlocking));
        {
            cudaMemPoolProps props{};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = device;
            ZK_CUDA(cudaMemPoolCreate(&srv->pool, &props));
            uint64_t thr = UINT64_MAX;  // keep freed memory mapped
            ZK_CUDA(cudaMemPoolSetAttribute(srv->pool, cudaMemPoolAttrReleaseThreshold, &thr));
            int no = 0, yes = 1;
            ZK_CUDA(cudaMemPoolSetAttribute(srv->pool, cudaMemPoolReuseAllowInternalDependencies, &no));
            ZK_CUDA(cudaMemPoolSetAttribute(srv->pool, cudaMemPoolReuseAllowOpportunistic, &yes));
        }
        // Reserve the budget in the pool, with an eighth more for fragmentation,
        // so admitted jobs are served from mapped memory: growing the pool while
        // jobs run maps physical memory on the dispatcher thread (about a second
        // for tens of GB), which stalls every admission meanwhile.  Memory that
        // the device's default pool keeps cached from earlier calls is handed
        // back first.  If the device cannot hold the reservation, the budget
        // alone is tried, then none (jobs grow the pool).
        {
            cudaMemPool_t def;
            if (cudaDeviceGetDefaultMemPool(&def, device) == cudaSuccess) cudaMemPoolTrimTo(def, 0);
            cudaStream_t st = srv->slots[0][0];
            for (uint64_t want : {hbm_budget_bytes + hbm_budget_bytes / 8, hbm_budget_bytes}) {
                void *p = nullptr;
                if (cudaMallocFromPoolAsync(&p, want, srv->pool, st) == cudaSuccess) {
                    ZK_CUDA(cudaFreeAsync(p, st));
                    ZK_CUDA(cudaStreamSynchronize(st));
                    break;
                }
                cudaGetLastError();
            }
            cudaMemPoolGetAttribute(srv->pool, cudaMemPoolAttrReservedMemCurrent, &srv->reserved_start);
        }
        ZkServer *p = srv.get();
        auto guarded = [p](auto body) {
            try {
                body();
            } catch (const std::exception &e) {
                std::lock_guard<std::mutex> g(p->mu);
                p->fatal = e.what();
                p->done_cv.notify_all();
            }
        };
        srv->dispatcher = std::thread([p, guarded] { guarded([p] { p->run(); }); });
        for (uint32_t i = 0; i < n_slots; i++)
            srv->workers.emplace_back([p, guarded, i] { guarded([p, i] { p->work((int)i); }); });
        *out = srv.release();
    });
}

namespace {

// GPU time of a commit alone, from its size: a fixed cost per tree level
// (each level is a launch of a few microseconds of latency at least), the
// permutations at ~1.0e9 per second and the LDE at ~60e9 evaluations per
// second (B200 figures of the drop-in path; only the relative sizes matter).
double estimate_s(const Shape &sh) {
    const double levels = (double)(sh.lg_n + sh.rate);
    return 1.0e-4 + 1.5e-5 * levels + sh.work() / 1.0e9 + (double)sh.N() * sh.batches / 60e9;
}

std::unique_ptr<ZkServer::Job> new_job(ZkServer *srv, const Shape &sh) {
    validate(sh);
    {
        // Tables are created on the caller's thread, before the job can run.
        ZK_CUDA(cudaSetDevice(srv->dev));
        DeviceCtx &ctx = device_ctx(srv->dev);
        coset_table(ctx, sh.lg_n + sh.rate, GROUP_GENERATOR, false);
        root_table(ctx, sh.lg_n + sh.rate, false);
        line_roots(ctx, false);
    }
    auto J = std::make_unique<ZkServer::Job>();
    J->sh = sh;
    J->bytes = sh.leaf_bytes() + sh.digest_bytes() + sh.cap_bytes();
    J->est_s = estimate_s(sh);
    J->run_bytes = sh.coeff_bytes() + sh.scratch_bytes();
    return J;
}

}  // namespace

uint64_t ZkServer::submit(std::unique_ptr<Job> J) {
    std::lock_guard<std::mutex> g(mu);
    require(fatal.empty(), "server failed: " + fatal);
    J->ticket = next_ticket++;
    J->seq = J->ticket;
    J->t_submit = std::chrono::steady_clock::now();
    J->budget_s = budget_frac * J->est_s;
    if (!any) {
        t_first = J->t_submit;
        any = true;
    }
    const uint64_t ticket = J->ticket;
    queue.push_back(ticket);
    max_queue = std::max<uint64_t>(max_queue, queue.size());
    jobs[ticket] = std::move(J);
    cv.notify_all();
    return ticket;
}

extern "C" RustError zk_server_submit(ZkServer *srv, const void *host_coeffs, uint32_t lg_n, uint32_t rate_bits,
                                     uint32_t batches, uint32_t cap_height, uint32_t hash_type, uint64_t *ticket) {
    return guard([&] {
        require(srv && host_coeffs && ticket, "null argument");
        auto J = new_job(srv, Shape{lg_n, rate_bits, batches, cap_height, hash_type});
        J->host_coeffs = host_coeffs;
        *ticket = srv->submit(std::move(J));
    });
}

extern "C" RustError zk_server_submit_seeded(ZkServer *srv, uint64_t seed, uint32_t lg_n, uint32_t rate_bits,
                                            uint32_t batches, uint32_t cap_height, uint32_t hash_type,
                                            uint64_t *ticket) {
    return guard([&] {
        require(srv && ticket, "null argument");
        auto J = new_job(srv, Shape{lg_n, rate_bits, batches, cap_height, hash_type});
        J->seeded = true;
        J->seed = seed;
        *ticket = srv->submit(std::move(J));
    });
}

extern "C" RustError zk_server_wait(ZkServer *srv, uint64_t ticket, uint64_t *host_cap, double *latency_s) {
    return guard([&] {
        require(srv != nullptr, "null server");
        std::unique_lock<std::mutex> lk(srv->mu);
        auto it = srv->jobs.find(ticket);
        require(it != srv->jobs.end(), "unknown ticket");
        ZkServer::Job *J = it->second.get();
        srv->done_cv.wait(lk, [&] { return J->state >= 2 || !srv->fatal.empty(); });
        if (J->state == 3)
            throw Error(J->err ? J->err : -(int)cudaErrorUnknown,
                        J->err_msg.empty() ? std::string("job failed") : "job failed: " + J->err_msg);
        require(J->state == 2, "job failed: " + srv->fatal);
        if (host_cap) memcpy(host_cap, J->cap.data(), J->sh.cap_bytes());
        if (latency_s) *latency_s = std::chrono::duration<double>(J->t_done - J->t_submit).count();
    });
}

extern "C" RustError zk_server_wait_any(ZkServer *srv, uint32_t timeout_ms, uint64_t *ticket) {
    return guard([&] {
        require(srv != nullptr && ticket != nullptr, "null argument");
        *ticket = 0;
        std::unique_lock<std::mutex> lk(srv->mu);
        auto ready = [&] {
            while (!srv->done_q.empty() && !srv->jobs.count(srv->done_q.front())) srv->done_q.pop_front();
            return !srv->done_q.empty() || (srv->queue.empty() && srv->n_running == 0) || !srv->fatal.empty();
        };
        if (timeout_ms == UINT32_MAX) srv->done_cv.wait(lk, ready);
        else srv->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
        if (!srv->done_q.empty() && srv->jobs.count(srv->done_q.front())) {
            *ticket = srv->done_q.front();
            srv->done_q.pop_front();
        }
    });
}

extern "C" RustError zk_server_result(ZkServer *srv, uint64_t ticket, void **d_leaves, void **d_digests,
                                     void **d_cap) {
    return guard([&] {
        require(srv != nullptr, "null server");
        std::lock_guard<std::mutex> g(srv->mu);
        auto it = srv->jobs.find(ticket);
        require(it != srv->jobs.end() && it->second->state == 2, "ticket not completed");
        if (d_leaves) *d_leaves = it->second->d_leaves;
        if (d_digests) *d_digests = it->second->d_digests;
        if (d_cap) *d_cap = it->second->d_cap;
    });
}

extern "C" RustError zk_server_release(ZkServer *srv, uint64_t ticket) {
    return guard([&] {
        require(srv != nullptr, "null server");
        std::unique_ptr<ZkServer::Job> J;
        {
            std::lock_guard<std::mutex> g(srv->mu);
            auto it = srv->jobs.find(ticket);
            require(it != srv->jobs.end(), "unknown ticket");
            require(it->second->state >= 2, "ticket still running");
            J = std::move(it->second);
            srv->jobs.erase(it);
        }
        ZK_CUDA(cudaSetDevice(srv->dev));
        if (J->state == 2) {
            // The job's work has completed (its completion callback ran), so the
            // tree is freed on the idle stream, not behind whatever its slot runs now.
            cudaStream_t st = srv->free_stream;
            if (J->d_leaves) ZK_CUDA(cudaFreeAsync(J->d_leaves, st));
            if (J->d_digests) ZK_CUDA(cudaFreeAsync(J->d_digests, st));
            if (J->d_cap) ZK_CUDA(cudaFreeAsync(J->d_cap, st));
            std::lock_guard<std::mutex> g(srv->mu);
            srv->in_use -= J->bytes;
            srv->cv.notify_all();
        }
    });
}

extern "C" RustError zk_server_stats(ZkServer *srv, ZkServerStats *out) {
    return guard([&] {
        require(srv && out, "null argument");
        std::lock_guard<std::mutex> g(srv->mu);
        std::vector<double> l = srv->latencies;
        std::sort(l.begin(), l.end());
        auto pct = [&](double q) { return l.empty() ? 0.0 : l[std::min<size_t>(l.size() - 1, (size_t)(q * l.size()))]; };
        memset(out, 0, sizeof(*out));
        out->completed = l.size();
        out->queued = srv->queue.size();
        out->max_queue = srv->max_queue;
        out->p50_s = pct(0.50);
        out->p99_s = pct(0.99);
        out->max_s = l.empty() ? 0 : l.back();
        out->elems = srv->elems_done;
        const double span = srv->any ? std::chrono::duration<double>(srv->t_last - srv->t_first).count() : 0.0;
        out->elems_per_s = span > 0 ? srv->elems_done / span : 0.0;
        out->hbm_in_use = srv->in_use;
        out->hbm_peak = srv->peak;
        out->ahead = srv->ahead;
        out->alloc_max_s = srv->alloc_max_s;
        out->pool_reserved_start = srv->reserved_start;
        if (srv->pool) cudaMemPoolGetAttribute(srv->pool, cudaMemPoolAttrReservedMemHigh, &out->pool_reserved_high);
    });
}

extern "C" RustError zk_server_job_times(ZkServer *srv, uint64_t ticket, double *queued_s, double *run_s) {
    return guard([&] {
        require(srv != nullptr, "null server");
        std::lock_guard<std::mutex> g(srv->mu);
        auto it = srv->jobs.find(ticket);
        require(it != srv->jobs.end() && it->second->state == 2, "ticket not completed");
        const ZkServer::Job &J = *it->second;
        if (queued_s) *queued_s = std::chrono::duration<double>(J.t_admit - J.t_submit).count();
        if (run_s) *run_s = std::chrono::duration<double>(J.t_done - J.t_admit).count();
    });
}

extern "C" RustError zk_server_inject_failure(ZkServer *srv, uint32_t n_jobs, uint32_t at_allocation) {
    return guard([&] {
        require(srv != nullptr && at_allocation >= 1, "invalid arguments");
        std::lock_guard<std::mutex> g(srv->mu);
        srv->inject_jobs = n_jobs;
        srv->inject_step = at_allocation;
    });
}

extern "C" RustError zk_server_destroy(ZkServer *srv) {
    if (!srv) return ok_err();
    {
        std::lock_guard<std::mutex> g(srv->mu);
        srv->stop = true;
        srv->cv.notify_all();
        srv->work_cv.notify_all();
    }
    if (srv->dispatcher.joinable()) srv->dispatcher.join();
    for (std::thread &w : srv->workers)
        if (w.joinable()) w.join();
    RustError r = guard([&] {
        ZK_CUDA(cudaSetDevice(srv->dev));
        for (auto &per : srv->slots)
            for (cudaStream_t st : per) ZK_CUDA(cudaStreamSynchronize(st));
        for (auto &kv : srv->jobs) {
            auto &J = *kv.second;
            for (uint64_t *p : {J.d_coeffs, J.d_leaves, J.d_digests, J.d_cap, J.d_scratch})
                if (p) cudaFree(p);
        }
        for (auto &per : srv->slots)
            for (cudaStream_t st : per) cudaStreamDestroy(st);
        for (uint64_t *p : srv->slot_cap)
            if (p) cudaFreeHost(p);
        if (srv->free_stream) {
            ZK_CUDA(cudaStreamSynchronize(srv->free_stream));
            cudaStreamDestroy(srv->free_stream);
        }
        // Hand the reserved budget back to the device.
        if (srv->pool) {
            cudaMemPoolTrimTo(srv->pool, 0);
            cudaMemPoolDestroy(srv->pool);
        }
    });
    delete srv;
    return r;
}
