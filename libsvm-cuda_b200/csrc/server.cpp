// server.cpp -- the request loop: continuous batching of independent binary
// solves on one GPU (svmb_server_* in include/svm_b200.h).
//
// The reference trains one problem per process call (svm-train, reference
// svm-train/svm-train.c:92-133); there is no serving layer to mirror.  Here a
// scheduler thread keeps up to `max_inflight` persistent launches ("waves")
// running on their own streams.  Whenever a wave finishes or a request
// arrives, a leading request -- the smallest pending one (the oldest once it
// has waited 2 s), or the oldest, by policy -- and the pending ones of a
// similar size (within a factor of 4 in rows) are admitted while
//   - the device memory of the admitted work (rows + solver state with its
//     Q-row cache budget) stays within the server's budget, and
//   - the thread blocks their state needs fit in the SMs that no running wave
//     holds,
// then uploaded (stream-ordered allocations, no device-wide synchronisation)
// and launched together as one new wave next to the waves already running.
// Requests get fewer blocks than a solve alone (rows / rows_per_block): a
// solve's iterations are latency-bound, so more requests side by side give
// more throughput than more blocks per request.
// A wave's blocks are planned within the free SMs, so all of them are
// resident at once; launches are therefore plain (not cooperative) and
// several run concurrently.  When every block of one request has finished,
// the kernel sets that request's word in host-mapped memory; the scheduler
// then copies its result out and hands its SMs to the next wave while the
// rest of the launch runs on.  Rows and solver state stay on the device
// until the launch ends.  Results equal a solve of the same request
// alone: the solver's arithmetic does not depend on the number of blocks or
// on the other instances of a launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "capi_internal.hpp"
#include "engine.hpp"
#include "svm_b200.h"

namespace svmb {
namespace {

using Clock = std::chrono::steady_clock;
constexpr double kMaxWait = 2.0;    // seconds a request may wait before it leads regardless of its size

struct Job {
    long long ticket = 0;
    int n = 0, d = 0;
    std::vector<long long> rowptr;
    std::vector<int> col;
    std::vector<float> val;
    svmb_params params{};
    std::vector<double> y;      // targets of the points
    SolveParams prm;
    SubProblem sub;
    std::unique_ptr<DeviceRows> rows;
    size_t mem = 0;             // device bytes reserved while the request runs
    // result
    int state = 0;              // 0 queued, 1 running, 2 done, -1 failed (written under the server lock)
    std::string error;
    std::vector<double> alpha;
    svmb_solve_stats stats{};
    Clock::time_point t_submit, t_start, t_done;
};

struct Slot {
    bool busy = false;
    cudaStream_t stream = nullptr;
    Wave w;
    int *flags_host = nullptr;      // host-mapped completion words, one per instance of the wave
    int *flags_dev = nullptr;
    std::vector<char> delivered;    // instance results already handed out
    std::vector<Job *> jobs;
    std::vector<SubProblem> subs;
    char *dev = nullptr;
    char *host = nullptr;
    size_t host_bytes = 0;
    size_t mem = 0;
    int blocks = 0;
};

// device bytes a request holds while it runs: its rows (CSR always, a dense
// copy when that is chosen, two norm arrays) and its solver state with the
// Q-row cache budget
size_t request_bytes(int n, int d, long long nnz, double cache_mb)
{
    const size_t csr = (size_t)(n + 1) * 8 + (size_t)nnz * 8;
    const size_t dense = (size_t)n * (size_t)((std::max(d, 1) + 3) & ~3) * 4;
    return csr + std::min(dense, csr * 2) + (size_t)n * 16 + instance_bytes(n, cache_mb) + (1 << 20);
}

// the launch-wide rows of a wave whose instances all bring their own
const DeviceRows &empty_rows()
{
    static DeviceRows none;
    return none;
}

}  // namespace

struct Server {
    svmb_server_config cfg{};
    int capacity = 0;               // solver blocks the device holds at once (one per SM)
    int device = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job *> pending;
    std::map<long long, std::unique_ptr<Job>> jobs;
    std::vector<Slot> slots;
    size_t mem_used = 0, mem_peak = 0;
    int blocks_used = 0;
    long long next_ticket = 0;
    bool stop = false;
    std::thread worker;
    // statistics
    long long completed = 0, failed = 0, waves = 0, max_concurrent = 0;
    std::vector<double> latencies;
    Clock::time_point t_first, t_last;
    bool any_submit = false;

    cudaStream_t copy_stream = nullptr;

    void loop();
    void admit(Slot &slot, std::unique_lock<std::mutex> &lk);
    void collect(Slot &slot);
    void reap(Slot &slot);
    void complete_locked(Job *j, bool ok, const std::string &err);
};

// a request's final state (called with the lock held)
void Server::complete_locked(Job *j, bool ok, const std::string &err)
{
    j->t_done = Clock::now();
    j->state = ok ? 2 : -1;             // waiters read a request only once its state is final
    if (ok) {
        completed++;
        latencies.push_back(std::chrono::duration<double>(j->t_done - j->t_submit).count());
    } else {
        j->error = err;
        failed++;
    }
    t_last = j->t_done;
    cv_done.notify_all();
}

// Hand out the instances of a running wave whose blocks have all finished
// (their completion word is set) and give their SMs to new waves at once
// (called without the lock).
void Server::collect(Slot &slot)
{
    for (int k = 0; k < slot.w.count; k++) {
        if (slot.delivered[k] || *(volatile int *)(slot.flags_host + k) == 0) continue;
        Job *j = slot.jobs[k];
        SolveResult r;
        const int rc = wave_fetch(slot.w, k, r, copy_stream);
        if (rc == 0) {
            j->alpha.assign(j->n, 0.0);
            capi::finish_instance(j->params, j->sub, r, j->y.data(), j->n, j->alpha.data(), &j->stats);
        }
        const std::string err = rc ? std::string(last_error()) : std::string();
        slot.delivered[k] = 1;
        j->rows->release_async(slot.stream);    // ordered after the launch on its stream
        j->rows.reset();
        slot.jobs[k] = nullptr;                 // a waiter may free the request once it is complete
        std::lock_guard<std::mutex> g(mu);
        complete_locked(j, rc == 0, err);
        blocks_used -= slot.w.nb[k];
        slot.blocks -= slot.w.nb[k];
    }
}

// Collect a finished wave (called without the lock).
void Server::reap(Slot &slot)
{
    collect(slot);
    std::vector<SolveResult> res(slot.subs.size());
    const int rc = wave_finish(slot.w, res);
    const std::string err = rc ? std::string(last_error()) : std::string();
    cudaFreeAsync(slot.dev, slot.stream);
    slot.dev = nullptr;
    // each request by its own outcome: one instance whose group timed out
    // fails alone; a launch that failed leaves every result unfilled
    std::vector<char> ok(slot.jobs.size(), 0);
    for (size_t k = 0; k < slot.jobs.size(); k++) {
        Job *j = slot.jobs[k];
        if (slot.delivered[k]) continue;
        j->rows->release_async(slot.stream);
        ok[k] = res[k].alpha.size() == j->sub.rows.size() && res[k].out.status >= 0;
        if (ok[k]) {
            j->alpha.assign(j->n, 0.0);
            capi::finish_instance(j->params, j->sub, res[k], j->y.data(), j->n, j->alpha.data(), &j->stats);
        }
    }
    std::lock_guard<std::mutex> g(mu);
    for (size_t k = 0; k < slot.jobs.size(); k++) {
        if (slot.delivered[k]) continue;
        slot.jobs[k]->rows.reset();
        complete_locked(slot.jobs[k], ok[k] != 0, ok[k] ? std::string() : (err.empty() ? "solve failed" : err));
    }
    mem_used -= slot.mem;
    blocks_used -= slot.blocks;
    slot.jobs.clear();
    slot.subs.clear();
    slot.busy = false;
    cv_done.notify_all();
}

// Take pending requests into a new wave on `slot` (called with the lock held;
// drops it while uploading and launching).
void Server::admit(Slot &slot, std::unique_lock<std::mutex> &lk)
{
    const int free_blocks = capacity - blocks_used;
    if (free_blocks <= 0 || pending.empty()) return;
    std::vector<Job *> take;
    size_t mem = 0;
    // A leading request, then pending requests whose size is within a factor
    // of 4 of the leader's: a launch keeps its device memory until its
    // longest solve ends, so similar sizes free it sooner.
    // the leader: the oldest request, or (smallest-first policy) the smallest
    // one unless the oldest has waited longer than kMaxWait
    if (cfg.policy == SVMB_SERVE_SMALLEST_FIRST &&
        std::chrono::duration<double>(Clock::now() - pending.front()->t_submit).count() < kMaxWait) {
        auto best = std::min_element(pending.begin(), pending.end(), [](const Job *a, const Job *b) { return a->n < b->n; });
        Job *lead = *best;
        pending.erase(best);
        pending.push_front(lead);
    }
    double lead_rows = 0;
    for (auto it = pending.begin(); it != pending.end() && (int)take.size() < std::min(cfg.max_batch, free_blocks);) {
        Job *j = *it;
        if (!take.empty() && ((double)j->n > 4.0 * lead_rows || 4.0 * (double)j->n < lead_rows)) {
            ++it;
            continue;
        }
        if (mem_used + mem + j->mem > (size_t)cfg.mem_bytes) {
            // nothing running and nothing taken: this request can never fit
            if (take.empty() && blocks_used == 0 && j->mem > (size_t)cfg.mem_bytes) {
                j->state = -1;
                j->error = "request exceeds the server's device memory budget";
                j->t_done = Clock::now();
                failed++;
                it = pending.erase(it);
                cv_done.notify_all();
                continue;
            }
            if (take.empty()) break;    // the leader waits for memory; nothing overtakes it
            ++it;
            continue;
        }
        if (take.empty()) lead_rows = (double)j->n;
        take.push_back(j);
        mem += j->mem;
        it = pending.erase(it);
    }
    if (take.empty()) return;
    for (Job *j : take) j->state = 1;
    mem_used += mem;
    mem_peak = std::max(mem_peak, mem_used);
    blocks_used += free_blocks;     // provisional: the wave's plan fixes the real count
    slot.busy = true;
    lk.unlock();

    cudaSetDevice(device);
    const auto now = Clock::now();
    slot.jobs = take;
    slot.subs.clear();
    bool ok = true;
    std::string err;
    std::vector<Job *> back;
    for (Job *j : take) {
        j->t_start = now;
        j->rows.reset(new DeviceRows());
        if (upload_csr(j->rowptr.data(), j->col.data(), j->val.data(), j->n, j->d, *j->rows, -1, slot.stream, kAllocAsync) != 0 ||
            j->rows->prepare_form(j->prm.form, slot.stream) != 0) {
            ok = false;
            err = last_error();
            break;
        }
        j->sub.rows_dev = j->rows.get();
        j->sub.own = &j->prm;
        slot.subs.push_back(j->sub);
    }
    if (ok) {
        if (wave_plan(empty_rows(), slot.subs, take[0]->prm, 0, free_blocks, slot.w) != 0) {
            ok = false;
            err = last_error();
        } else if (slot.w.count < (int)take.size()) {
            // the plan holds fewer requests than admitted: the rest go back to the queue head
            back.assign(take.begin() + slot.w.count, take.end());
            take.resize(slot.w.count);
            slot.jobs = take;
            slot.subs.resize(slot.w.count);
            for (Job *j : back) {
                j->rows->release_async(slot.stream);
                j->rows.reset();
                mem -= j->mem;
            }
        }
    }
    if (ok && slot.host_bytes < slot.w.up_bytes + slot.w.down_bytes) {
        if (slot.host) cudaFreeHost(slot.host);
        slot.host = nullptr;
        slot.host_bytes = 0;
        const size_t want = (slot.w.up_bytes + slot.w.down_bytes) * 2;
        if (cudaHostAlloc((void **)&slot.host, want, cudaHostAllocDefault) == cudaSuccess) slot.host_bytes = want;
        else { ok = false; err = "page-locked staging allocation failed"; }
    }
    if (ok && cudaMallocAsync((void **)&slot.dev, slot.w.dev_bytes, slot.stream) != cudaSuccess) {
        ok = false;
        err = "device allocation for a launch failed";
        slot.dev = nullptr;
    }
    if (ok) {
        slot.w.cooperative = false;
        memset(slot.flags_host, 0, sizeof(int) * (size_t)cfg.max_batch);
        slot.w.done_flags = slot.flags_dev;
        slot.delivered.assign(slot.w.count, 0);
        if (wave_start(empty_rows(), slot.subs, take[0]->prm, slot.w, slot.dev, slot.host, slot.stream) != 0) {
            ok = false;
            err = last_error();
        }
    }
    lk.lock();
    for (auto it = back.rbegin(); it != back.rend(); ++it) {
        (*it)->state = 0;
        pending.push_front(*it);
    }
    mem_used -= [&] { size_t b = 0; for (Job *j : back) b += j->mem; return b; }();
    if (!ok) {
        for (Job *j : slot.jobs) {
            if (j->rows) j->rows->release_async(slot.stream);
            j->rows.reset();
            j->state = -1;
            j->error = err;
            j->t_done = Clock::now();
            failed++;
        }
        if (slot.dev) cudaFreeAsync(slot.dev, slot.stream);
        slot.dev = nullptr;
        mem_used -= mem;
        blocks_used -= free_blocks;
        slot.jobs.clear();
        slot.subs.clear();
        slot.busy = false;
        cv_done.notify_all();
        return;
    }
    slot.mem = mem;
    slot.blocks = slot.w.used;
    blocks_used += slot.w.used - free_blocks;
    waves++;
    int running = 0;
    for (const Slot &s : slots) running += s.busy ? 1 : 0;
    max_concurrent = std::max<long long>(max_concurrent, running);
}

void Server::loop()
{
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
        bool any_busy = false;
        for (Slot &s : slots) {
            if (!s.busy) continue;
            lk.unlock();
            if (wave_ready(s.w)) reap(s);
            else collect(s);
            lk.lock();
            if (s.busy) any_busy = true;
        }
        for (Slot &s : slots) {
            if (pending.empty()) break;
            if (s.busy) continue;
            admit(s, lk);
            if (s.busy) any_busy = true;
            else break;     // nothing admissible now
        }
        if (stop && pending.empty() && !any_busy) break;
        if (any_busy) cv_work.wait_for(lk, std::chrono::microseconds(50));
        else cv_work.wait(lk, [&] { return stop || !pending.empty(); });
    }
}

}  // namespace svmb

using svmb::Server;

extern "C" {

struct svmb_server {
    Server s;
};

int svmb_server_create(const svmb_server_config *cfg, svmb_server **out)
{
    if (!out) { svmb::set_error("NULL output"); return -1; }
    if (!svmb_device_available()) { svmb::set_error("no CUDA device"); return -1; }
    std::unique_ptr<svmb_server> h(new svmb_server());
    Server &S = h->s;
    if (cfg) S.cfg = *cfg;
    if (S.cfg.form < SVMB_FORM_EXACT || S.cfg.form > SVMB_FORM_TF32) { svmb::set_error("unknown form"); return -1; }
    cudaGetDevice(&S.device);
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    if (S.cfg.mem_bytes <= 0) S.cfg.mem_bytes = (long long)(free_b * 0.8);
    if (S.cfg.max_inflight <= 0) S.cfg.max_inflight = 8;
    if (S.cfg.max_batch <= 0) S.cfg.max_batch = 32;
    if (S.cfg.rows_per_block <= 0) S.cfg.rows_per_block = 2000;
    if (S.cfg.policy != SVMB_SERVE_ARRIVAL_ORDER) S.cfg.policy = SVMB_SERVE_SMALLEST_FIRST;
    S.capacity = svmb::device_sm_count();     // one solver block per SM at its largest shared memory
    if (S.capacity <= 0) { svmb::set_error("no CUDA device"); return -1; }
    S.slots.resize(S.cfg.max_inflight);
    if (cudaStreamCreateWithFlags(&S.copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
        svmb::set_error("stream creation failed");
        return -1;
    }
    for (auto &sl : S.slots) {
        if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess) {
            svmb::set_error("stream creation failed");
            return -1;
        }
        // completion words the kernel sets in host memory, one per instance
        if (cudaHostAlloc((void **)&sl.flags_host, sizeof(int) * (size_t)S.cfg.max_batch, cudaHostAllocMapped) != cudaSuccess ||
            cudaHostGetDevicePointer((void **)&sl.flags_dev, sl.flags_host, 0) != cudaSuccess) {
            svmb::set_error("mapped host allocation failed");
            return -1;
        }
    }
    S.worker = std::thread([&S] { S.loop(); });
    *out = h.release();
    return 0;
}

long long svmb_server_submit(svmb_server *h, int n, int d, const long long *rowptr, const int *col, const float *val,
                             const double *y, const svmb_params *params)
{
    if (!h || n <= 0 || d < 0 || !rowptr || !y || !params) { svmb::set_error("invalid request"); return -1; }
    if (svmb::capi::check_params(params) != 0) return -1;
    if (params->form != h->s.cfg.form) { svmb::set_error("the request's form differs from the server's"); return -1; }
    for (int r = 0; r < n; r++)
        if (rowptr[r + 1] < rowptr[r]) { svmb::set_error("rowptr must be non-decreasing"); return -1; }
    for (long long e = 0; e < rowptr[n]; e++)
        if (col[e] < 0 || col[e] >= d) { svmb::set_error("column index out of range"); return -1; }
    std::unique_ptr<svmb::Job> j(new svmb::Job());
    j->n = n;
    j->d = d;
    j->rowptr.assign(rowptr, rowptr + n + 1);
    j->col.assign(col, col + rowptr[n]);
    j->val.assign(val, val + rowptr[n]);
    j->params = *params;
    j->y.assign(y, y + n);
    j->prm = svmb::capi::to_solve_params(*params);
    if (j->prm.blocks_override <= 0)
        j->prm.blocks_override = std::max(1, std::min(svmb::device_sm_count(), n / h->s.cfg.rows_per_block));
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    if (svmb::capi::make_subproblem(*params, n, idx.data(), y, n, j->sub) != 0) return -1;
    j->mem = svmb::request_bytes(n, d, rowptr[n], params->cache_mb);
    j->t_submit = svmb::Clock::now();
    Server &S = h->s;
    std::lock_guard<std::mutex> g(S.mu);
    j->ticket = S.next_ticket++;
    if (!S.any_submit) { S.any_submit = true; S.t_first = j->t_submit; }
    S.pending.push_back(j.get());
    const long long t = j->ticket;
    S.jobs[t] = std::move(j);
    S.cv_work.notify_one();
    return t;
}

int svmb_server_poll(svmb_server *h, long long ticket)
{
    if (!h) return -1;
    std::lock_guard<std::mutex> g(h->s.mu);
    auto it = h->s.jobs.find(ticket);
    if (it == h->s.jobs.end()) { svmb::set_error("unknown ticket"); return -1; }
    const int st = it->second->state;
    return st == 2 || st == -1 ? 1 : 0;
}

int svmb_server_wait(svmb_server *h, long long ticket, double *alpha_out, svmb_solve_stats *stats, double *latency_s)
{
    if (!h) { svmb::set_error("NULL server"); return -1; }
    Server &S = h->s;
    std::unique_lock<std::mutex> lk(S.mu);
    auto it = S.jobs.find(ticket);
    if (it == S.jobs.end()) { svmb::set_error("unknown ticket"); return -1; }
    svmb::Job *j = it->second.get();
    S.cv_done.wait(lk, [&] { return j->state == 2 || j->state == -1; });
    int rc = 0;
    if (j->state == 2) {
        if (alpha_out) memcpy(alpha_out, j->alpha.data(), sizeof(double) * j->n);
        if (stats) *stats = j->stats;
        if (latency_s) *latency_s = std::chrono::duration<double>(j->t_done - j->t_submit).count();
    } else {
        svmb::set_error(j->error);
        rc = -1;
    }
    S.jobs.erase(it);       // a ticket is collected once
    return rc;
}

int svmb_server_get_stats(svmb_server *h, svmb_server_stats *out)
{
    if (!h || !out) { svmb::set_error("invalid arguments"); return -1; }
    Server &S = h->s;
    std::lock_guard<std::mutex> g(S.mu);
    memset(out, 0, sizeof *out);
    out->completed = S.completed;
    out->failed = S.failed;
    out->waves = S.waves;
    out->max_concurrent_waves = S.max_concurrent;
    out->peak_mem_bytes = (long long)S.mem_peak;
    out->pending = (long long)S.pending.size();
    if (!S.latencies.empty()) {
        std::vector<double> v = S.latencies;
        std::sort(v.begin(), v.end());
        auto pct = [&](double q) { return v[std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1) + 0.5))]; };
        out->p50_s = pct(0.50);
        out->p99_s = pct(0.99);
        out->max_s = v.back();
        const double span = std::chrono::duration<double>(S.t_last - S.t_first).count();
        out->solves_per_s = span > 0 ? (double)S.completed / span : 0.0;
    }
    return 0;
}

void svmb_server_destroy(svmb_server *h)
{
    if (!h) return;
    {
        std::lock_guard<std::mutex> g(h->s.mu);
        h->s.stop = true;
        h->s.cv_work.notify_all();
    }
    if (h->s.worker.joinable()) h->s.worker.join();
    for (auto &sl : h->s.slots) {
        if (sl.stream) {
            cudaStreamSynchronize(sl.stream);
            cudaStreamDestroy(sl.stream);
        }
        if (sl.host) cudaFreeHost(sl.host);
        if (sl.flags_host) cudaFreeHost(sl.flags_host);
    }
    if (h->s.copy_stream) cudaStreamDestroy(h->s.copy_stream);
    delete h;
}

}  // extern "C"
