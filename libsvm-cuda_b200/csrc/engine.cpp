// engine.cpp -- host orchestration of the device SMO solver.
//
// Replaces the reference's CudaSolver/CudaSolverNU host classes
// (reference libsvm/cuda_solver.cpp:159-555, cuda_solverNU.cpp:64-178): instead
// of launching 7-9 kernels and two blocking device->host copies per SMO
// iteration, the whole solve of every instance runs inside one persistent
// launch (smo_kernel.cu) and the host only uploads the problem and reads the
// result back.
#include "engine.hpp"

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <cstdlib>
#include <mutex>

#include "svm.h"

namespace svmb {

static thread_local std::string g_last_error;
void set_error(const std::string &msg) { g_last_error = msg; }
const char *last_error() { return g_last_error.c_str(); }

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                \
            return -1;                                                                    \
        }                                                                                 \
    } while (0)

static std::atomic<long long> g_launches{0};
static std::atomic<long long> g_h2d{0}, g_d2h{0};
void count_launch(long long n) { g_launches += n; }
long long launch_count() { return g_launches.load(); }
void transfer_bytes(long long *h2d, long long *d2h)
{
    if (h2d) *h2d = g_h2d.load();
    if (d2h) *d2h = g_d2h.load();
}

// host<->device copies, counted per direction
cudaError_t xfer_async(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s)
{
    if (kind == cudaMemcpyHostToDevice) g_h2d += (long long)bytes;
    if (kind == cudaMemcpyDeviceToHost) g_d2h += (long long)bytes;
    return cudaMemcpyAsync(dst, src, bytes, kind, s);
}
cudaError_t xfer(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind)
{
    if (kind == cudaMemcpyHostToDevice) g_h2d += (long long)bytes;
    if (kind == cudaMemcpyDeviceToHost) g_d2h += (long long)bytes;
    return cudaMemcpy(dst, src, bytes, kind);
}

// Page-locked staging for row uploads, grown on demand and reused by later
// calls (copies from it run at full PCIe/C2C bandwidth).
namespace {
std::mutex g_pin_mu;
void *g_pin[2] = {nullptr, nullptr};
size_t g_pin_bytes[2] = {0, 0};
}  // namespace
// slot 0: row uploads (under g_pin_mu); slot 1: solver state (under the arena lock)
void *pinned_staging_slot(int slot, size_t bytes)
{
    if (bytes <= g_pin_bytes[slot]) return g_pin[slot];
    if (g_pin[slot]) cudaFreeHost(g_pin[slot]);
    g_pin[slot] = nullptr;
    g_pin_bytes[slot] = 0;
    const size_t want = std::max<size_t>(bytes + bytes / 4, 1 << 20);
    if (cudaHostAlloc(&g_pin[slot], want, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        g_pin[slot] = nullptr;
        return nullptr;
    }
    g_pin_bytes[slot] = want;
    return g_pin[slot];
}
void *pinned_staging(size_t bytes) { return pinned_staging_slot(0, bytes); }

// SVMB_TRACE=1 prints host-side stage times of every solve_batch to stderr
static bool trace_on()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("SVMB_TRACE");
        on = (e && *e == '1') ? 1 : 0;
    }
    return on == 1;
}
struct StageClock {
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now(), last = t0;
    std::string log;
    void mark(const char *what)
    {
        if (!trace_on()) return;
        const auto now = std::chrono::steady_clock::now();
        char buf[96];
        snprintf(buf, sizeof buf, " %s=%.2fms", what, std::chrono::duration<double, std::milli>(now - last).count());
        log += buf;
        last = now;
    }
    ~StageClock()
    {
        if (trace_on() && !log.empty()) fprintf(stderr, "[svmb] solve_batch%s\n", log.c_str());
    }
};

int device_sm_count()
{
    static int sms = -1;
    if (sms < 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return 0;
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return 0;
        sms = p.multiProcessorCount;
    }
    return sms;
}

DeviceRows::~DeviceRows()
{
    cudaFree(X);
    cudaFree(rowptr);
    cudaFree(col);
    cudaFree(val);
    cudaFree(xsq[0]);
    cudaFree(xsq[1]);
    cudaFree(Xs);
    cudaFree(xinv);
}

int DeviceRows::prepare_form(int form, cudaStream_t s)
{
    if (!is_tc_form(form)) return 0;
    if ((Xs && split_form == form) || n == 0) return 0;
    cudaFree(Xs);
    cudaFree(xinv);
    Xs = nullptr;
    xinv = nullptr;
    split_form = -1;
    // the tensor forms read every row densely (d features, padded to 64)
    const int nc = std::max(1, (d + kSplitChunk - 1) / kSplitChunk);
    const size_t b = (size_t)n * nc * 2 * kSplitChunk * sizeof(uint16_t);
    uint16_t *p = nullptr;
    double *q = nullptr;
    cudaError_t e = cudaMalloc(&p, b);
    if (e == cudaSuccess && form == FORM_FP16X3) e = cudaMalloc(&q, (size_t)n * sizeof(double));
    if (e == cudaSuccess) e = cudaMemsetAsync(p, 0, b, s);
    if (e == cudaSuccess) e = launch_split(*this, form, nc, p, q, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaFree(p);
        cudaFree(q);
        set_error(std::string("split rows: ") + cudaGetErrorString(e));
        return -1;
    }
    Xs = p;
    xinv = q;
    nchunk = nc;
    split_form = form;
    return 0;
}

DevX DeviceRows::view(int form) const
{
    DevX v;
    v.X = dense ? X : nullptr;
    v.ld = ld;
    v.rowptr = dense ? nullptr : rowptr;
    v.col = dense ? nullptr : col;
    v.val = dense ? nullptr : val;
    v.d = d;
    // the tensor forms use the float64 norms: they cost nothing and keep the
    // RBF distance as accurate as the split dot products allow
    v.xsq = xsq[is_tc_form(form) ? FORM_EXACT : form];
    const bool split = is_tc_form(form) && split_form == form;
    v.Xs = split ? Xs : nullptr;
    v.nchunk = split ? nchunk : 0;
    v.xinv = split ? xinv : nullptr;
    return v;
}

int upload_csr(const long long *rowptr, const int *col, const float *val, int n, int d, DeviceRows &out,
               int force, cudaStream_t s)
{
    out.n = n;
    out.d = d > 0 ? d : 1;
    const long long nnz = rowptr[n];
    out.ld = (out.d + 3) & ~3;
    // Dense rows only when they are not larger than the CSR arrays: a kernel
    // row streams the whole stored row of every active position, so the byte
    // count is what matters.
    const double dense_bytes = (double)n * out.ld * 4.0;
    const double csr_bytes = (double)(n + 1) * 8.0 + (double)nnz * 8.0;
    bool dense = force == 1 || (force < 0 && dense_bytes <= 1.2 * csr_bytes);
    if (dense && dense_bytes > 60e9) dense = false;
    out.dense = dense;
    // the CSR arrays always travel; dense rows are scattered on the device
    out.nnz = nnz;
    CK(cudaMalloc(&out.rowptr, (size_t)(n + 1) * sizeof(long long)));
    CK(cudaMalloc(&out.col, (size_t)std::max<long long>(nnz, 1) * sizeof(int)));
    CK(cudaMalloc(&out.val, (size_t)std::max<long long>(nnz, 1) * sizeof(float)));
    CK(xfer_async(out.rowptr, rowptr, (size_t)(n + 1) * sizeof(long long), cudaMemcpyHostToDevice, s));
    if (nnz) {
        CK(xfer_async(out.col, col, (size_t)nnz * sizeof(int), cudaMemcpyHostToDevice, s));
        CK(xfer_async(out.val, val, (size_t)nnz * sizeof(float), cudaMemcpyHostToDevice, s));
    }
    out.h2d_bytes = (size_t)(n + 1) * 8 + (size_t)nnz * 8;
    if (dense) {
        const size_t elems = std::max<size_t>((size_t)n * out.ld, 4);
        CK(cudaMalloc(&out.X, elems * sizeof(float)));
        CK(cudaMemsetAsync(out.X, 0, elems * sizeof(float), s));
        if (n) {
            CK(launch_scatter_dense(out.rowptr, out.col, out.val, n, out.ld, out.X, s));
            count_launch();
        }
        out.bytes = (size_t)n * out.ld * sizeof(float);
    } else {
        out.bytes = (size_t)(n + 1) * 8 + (size_t)nnz * 8;
    }
    for (int f = 0; f < 2; f++) {
        CK(cudaMalloc(&out.xsq[f], (size_t)std::max(n, 1) * sizeof(double)));
        if (n) {
            CK(launch_xsq(out.view(f), n, out.xsq[f], f, s));
            count_launch();
        }
    }
    CK(cudaStreamSynchronize(s));
    return 0;
}

int upload_rows(const svm_node *const *x, int n, DeviceRows &out, int force, cudaStream_t s)
{
    // CSR with 0-based columns; libsvm indices start at 1 (index 0 is kept as a
    // column when present).  Rows are converted in parallel on the host.
    std::vector<long long> cnt((size_t)n + 1, 0);
    int min_index = INT_MAX, max_index = 0;
#pragma omp parallel for schedule(static) reduction(min : min_index) reduction(max : max_index)
    for (int r = 0; r < n; r++) {
        long long c = 0;
        for (const svm_node *p = x[r]; p->index != -1; ++p) {
            min_index = std::min(min_index, p->index);
            max_index = std::max(max_index, p->index);
            c++;
        }
        cnt[r + 1] = c;
    }
    for (int r = 0; r < n; r++) cnt[r + 1] += cnt[r];
    const long long nnz = cnt[n];
    if (nnz && min_index < 0) {
        set_error("feature index < 0");
        return -1;
    }
    const int base = (nnz && min_index == 0) ? 0 : 1;
    // CSR arrays built directly in page-locked staging memory
    std::lock_guard<std::mutex> g(g_pin_mu);
    const size_t bytes = ((size_t)n + 1) * 8 + (size_t)nnz * 8 + 64;
    char *pin = (char *)pinned_staging(bytes);
    std::vector<char> fallback;
    if (!pin) {
        fallback.resize(bytes);
        pin = fallback.data();
    }
    long long *rp = (long long *)pin;
    int *col = (int *)(pin + (((size_t)n + 1) * 8));
    float *val = (float *)(pin + (((size_t)n + 1) * 8) + (size_t)nnz * 4);
    memcpy(rp, cnt.data(), sizeof(long long) * ((size_t)n + 1));
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n; r++) {
        long long k = rp[r];
        for (const svm_node *p = x[r]; p->index != -1; ++p, ++k) {
            col[k] = p->index - base;
            val[k] = (float)p->value;
        }
    }
    const int d = nnz ? max_index - base + 1 : 1;
    return upload_csr(rp, col, val, n, d, out, force, s);
}

namespace {

struct Bump {
    size_t off = 0;
    template <class T>
    size_t take(size_t count)
    {
        off = (off + 255) & ~size_t(255);
        size_t at = off;
        off += std::max<size_t>(count, 1) * sizeof(T);
        return at;
    }
};

// Byte layout of one instance's device state (all offsets 256-aligned).
struct InstanceLayout {
    size_t G, Gb, A, P, QD, Al, Y, S, PL, PR, Sc, Out, Sync, Part, Tag, Ep, St, Data, bytes;
    int sets, ways;
};

InstanceLayout instance_layout(int l, int nb, double cache_mb)
{
    (void)nb;
    InstanceLayout L;
    memset(&L, 0, sizeof(L));
    // cache geometry: rows of l floats, at least 4, at most 2l slots
    long long slots = (long long)std::floor(cache_mb * (1 << 20) / (4.0 * std::max(l, 1)));
    slots = std::max<long long>(slots, 4);
    slots = std::min<long long>(slots, std::max<long long>(4, 2LL * l));
    L.ways = (int)std::min<long long>(kMaxWays, slots);
    L.sets = (int)(slots / L.ways);
    const size_t ns = (size_t)L.sets * L.ways;
    Bump b;
    L.G = b.take<double>(l); L.Gb = b.take<double>(l); L.QD = b.take<double>(l);
    L.S = b.take<unsigned char>(l);
    L.PL = b.take<int>(l); L.Sc = b.take<int>(2 * (size_t)l);
    L.Data = b.take<float>(ns * (size_t)l);
    L.bytes = (b.off + 255) & ~size_t(255);
    return L;
}

// Grow-only device arena for solver state: one buffer reused by every launch
// (allocating and freeing gigabytes of Q-row caches per call costs more than
// a small solve).  Calls into the engine are serialised on it.
std::mutex g_arena_mu;
char *g_arena = nullptr;
size_t g_arena_bytes = 0;

char *arena_reserve(size_t bytes)
{
    if (bytes <= g_arena_bytes) return g_arena;
    if (g_arena) cudaFree(g_arena);
    g_arena = nullptr;
    g_arena_bytes = 0;
    const size_t want = bytes + bytes / 4;
    if (cudaMalloc(&g_arena, want) != cudaSuccess) {
        cudaGetLastError();
        if (cudaMalloc(&g_arena, bytes) != cudaSuccess) {
            g_arena = nullptr;
            return nullptr;
        }
        g_arena_bytes = bytes;
        return g_arena;
    }
    g_arena_bytes = want;
    return g_arena;
}

}  // namespace

void release_arena()
{
    std::lock_guard<std::mutex> g(g_arena_mu);
    if (g_arena) cudaFree(g_arena);
    g_arena = nullptr;
    g_arena_bytes = 0;
}

int solve_batch(const DeviceRows &rows, const std::vector<SubProblem> &subs, const SolveParams &prm,
                std::vector<SolveResult> &res, cudaStream_t s)
{
    const int ninst = (int)subs.size();
    res.assign(ninst, SolveResult());
    if (ninst == 0) return 0;
    // the split bf16 copy of the rows is a derived cache of the rows, built on first use
    if (const_cast<DeviceRows &>(rows).prepare_form(prm.form, s) != 0) return -1;
    std::lock_guard<std::mutex> arena_lock(g_arena_mu);
    StageClock clk;
    const int sms = device_sm_count();
    if (sms <= 0) {
        set_error("no CUDA device");
        return -1;
    }
    // Shared memory of a block: [source staging][chunk state, kChunkBytes per position].
    constexpr int kChunkBytes = 3 * 8 + 2 * 4 + 2;     // G, alpha, QD, col, row, y, status
    int smem_total = 0, dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&smem_total, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const long long budget = (long long)smem_total - smo_static_smem() - 1024;
    int stage_cap, stage_lds;
    if (rows.dense) {
        stage_lds = rows.ld;
        stage_cap = (int)std::min<long long>(kSrcBatch, (48LL << 10) / ((long long)rows.ld * 4));
    } else {
        stage_lds = rows.d;
        stage_cap = (int)std::min<long long>(kSrcBatch, (budget / 2) / ((long long)std::max(rows.d, 1) * 4));
    }
    if (stage_cap < 2) stage_cap = 0;
    int tc_n = 0;
    long long stage_bytes;
    if (is_tc_form(prm.form)) {
        // tensor form: the operand stages of the tensor-core pipeline replace the
        // source staging; as many sources per block-product pass as leave room for
        // a useful chunk of state
        stage_cap = 0;
        tc_n = kTcMaxN;
        while (tc_n > 16 && (budget - tc_area_bytes(tc_n) - kAuxBytes) / kChunkBytes < 1024) tc_n /= 2;
        stage_bytes = tc_area_bytes(tc_n);
    } else {
        stage_bytes = (((long long)stage_cap * stage_lds * 4) + 15) & ~15LL;
    }
    stage_bytes += kAuxBytes;   // transpose tiles / prefetch candidates
    const long long chunk_max = (budget - stage_bytes) / kChunkBytes;
    if (chunk_max < 64) {
        set_error("not enough shared memory for the solver state");
        return -1;
    }
    const size_t max_dyn = (size_t)(stage_bytes + chunk_max * kChunkBytes);
    int per_sm = 0;
    CK(smo_max_blocks(prm.form, max_dyn, &per_sm));
    if (per_sm < 1) {
        set_error("solver kernel does not fit on an SM");
        return -1;
    }
    const int capacity = per_sm * sms;
    clk.mark("setup");
    for (const SubProblem &sp : subs)
        if ((long long)sp.rows.size() > chunk_max * capacity) {
            set_error("problem too large: more positions than the device's blocks can hold in shared memory");
            return -1;
        }

    // process instances in waves that fit the co-resident capacity
    int first = 0;
    while (first < ninst) {
        // blocks per instance: enough to hold the state in shared memory, more
        // for large problems, shared proportionally when instances run together
        std::vector<int> nb;
        long long total_l = 0, need = 0;
        int last = first;
        while (last < ninst) {
            const long long l = (long long)subs[last].rows.size();
            const long long nmin = std::max<long long>(1, (l + chunk_max - 1) / chunk_max);
            if (need + nmin > capacity) break;
            need += nmin;
            total_l += l;
            last++;
        }
        const int count = last - first;
        nb.assign(count, 1);
        // expected work of an instance grows like l^2 (rows evaluated x row length):
        // share the device by l^2 so that the largest instances, which bound the
        // launch, get the most blocks
        double total_w = 0;
        for (int k = 0; k < count; k++) {
            const double l = (double)subs[first + k].rows.size();
            total_w += l * l;
        }
        for (int k = 0; k < count; k++) {
            const long long l = (long long)subs[first + k].rows.size();
            const int nmin = (int)std::max<long long>(1, (l + chunk_max - 1) / chunk_max);
            int want;
            if (prm.blocks_override > 0) want = prm.blocks_override;
            else want = (int)std::max<long long>(1, std::min<long long>(sms, (l + 499) / 500));
            if (count > 1) {
                const long long share = (long long)std::floor((double)capacity * (double)l * (double)l / std::max(total_w, 1.0));
                want = (int)std::min<long long>(want, std::max<long long>(1, share));
            }
            want = (int)std::min<long long>(want, std::max<long long>(1, l));
            want = std::min(want, kThreads);
            nb[k] = std::max(want, nmin);
        }
        (void)total_l;
        int used = 0;
        for (int v : nb) used += v;
        while (used > capacity) {
            // trim the instance with the most blocks above its minimum
            int big = -1;
            long long slack = 0;
            for (int k = 0; k < count; k++) {
                const long long l = (long long)subs[first + k].rows.size();
                const long long nmin = std::max<long long>(1, (l + chunk_max - 1) / chunk_max);
                if (nb[k] - nmin > slack) { slack = nb[k] - nmin; big = k; }
            }
            if (big < 0) break;
            nb[big]--;
            used--;
        }
        long long chunk_cap = 1;
        for (int k = 0; k < count; k++) {
            const long long l = (long long)subs[first + k].rows.size();
            chunk_cap = std::max<long long>(chunk_cap, (l + nb[k] - 1) / nb[k]);
        }
        const size_t dyn_smem = (size_t)(stage_bytes + chunk_cap * kChunkBytes);

        // One arena block per wave, laid out so that the host touches it with
        // one upload, three fills and two downloads:
        //   upload   [descriptors][block map][alpha][p][row ids][labels]
        //   download [outputs][alpha by local index]
        //   zero     [group syncs][exchange records][cache epochs][cache stamps]
        //   0xff     [cache tags]
        //   per instance: G, G_bar, QD, status, position->local, shrink lists, Q rows
        auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
        std::vector<size_t> loff(count + 1, 0), poff(count + 1, 0), coff(count + 1, 0);
        std::vector<InstanceLayout> lay(count);
        for (int k = 0; k < count; k++) {
            const int l = (int)subs[first + k].rows.size();
            lay[k] = instance_layout(l, nb[k], prm.cache_mb);
            loff[k + 1] = loff[k] + (size_t)l;
            poff[k + 1] = poff[k] + 2 * (size_t)nb[k];
            coff[k + 1] = coff[k] + (size_t)lay[k].sets * lay[k].ways;
        }
        const size_t L = loff[count], P = poff[count], S = coff[count];
        size_t off = 0;
        const size_t o_desc = off; off = al(off + sizeof(InstanceDesc) * count);
        const size_t o_bmap = off; off = al(off + sizeof(int) * used);
        const size_t o_alpha = off; off = al(off + 8 * L);
        const size_t o_p = off; off = al(off + 8 * L);
        const size_t o_row = off; off = al(off + 4 * L);
        const size_t o_y = off; off = al(off + L);
        const size_t up_bytes = off;
        const size_t o_out = off; off = al(off + sizeof(SolveOut) * count);
        const size_t o_alocal = off; off = al(off + 8 * L);
        const size_t down_bytes = off - o_out;
        const size_t o_zero = off;
        const size_t o_sync = off; off = al(off + sizeof(GroupSync) * count);
        const size_t o_part = off; off = al(off + sizeof(Partial) * P);
        const size_t o_ep = off; off = al(off + 4 * S);
        const size_t o_st = off; off = al(off + 8 * S);
        const size_t zero_bytes = off - o_zero;
        const size_t o_tag = off; off = al(off + 4 * S);
        std::vector<size_t> inst_off(count);
        for (int k = 0; k < count; k++) {
            inst_off[k] = off;
            off += lay[k].bytes;
        }
        clk.mark("plan");
        char *arena = arena_reserve(off);
        clk.mark("arena");
        if (!arena) {
            set_error("device allocation for solver state failed (" + std::to_string(off >> 20) + " MiB)");
            return -1;
        }
        // host side of the upload region, in page-locked memory
        char *host = nullptr;
        std::vector<char> host_fallback;
        {
            host = (char *)pinned_staging_slot(1, up_bytes + down_bytes);
            if (!host) {
                host_fallback.resize(up_bytes + down_bytes);
                host = host_fallback.data();
            }
        }
        InstanceDesc *h_desc = (InstanceDesc *)(host + o_desc);
        int *h_bmap = (int *)(host + o_bmap);
        double *h_alpha = (double *)(host + o_alpha);
        double *h_p = (double *)(host + o_p);
        int *h_row = (int *)(host + o_row);
        signed char *h_y = (signed char *)(host + o_y);
        InstanceDesc *d_desc = (InstanceDesc *)(arena + o_desc);
        int *d_block_inst = (int *)(arena + o_bmap);
        std::vector<InstanceDesc> desc(count);
        int b0 = 0;
        for (int k = 0; k < count; k++) {
            const SubProblem &sp = subs[first + k];
            const int l = (int)sp.rows.size();
            InstanceDesc &D = desc[k];
            memset(&D, 0, sizeof(D));
            D.l = l;
            D.nu = sp.nu;
            D.shrinking = prm.shrinking;
            D.form = prm.form;
            D.Cp = sp.Cp;
            D.Cn = sp.Cn;
            D.eps = prm.eps;
            D.max_iter = std::max<long long>(10000000LL, l > INT_MAX / 100 ? (long long)INT_MAX : 100LL * l);
            D.kp = prm.kp;
            D.x = rows.view(prm.form);
            D.block0 = b0;
            D.nblocks = nb[k];
            D.stage_cap = stage_cap;
            D.stage_lds = stage_lds;
            D.chunk_cap = (int)chunk_cap;
            {
                const int limit = stage_cap > 0 ? std::min(kPrefetchMax, stage_cap) : kPrefetchMax;
                D.prefetch = prm.prefetch > 0 ? std::min(prm.prefetch, limit) : limit;
                D.lazy_gbar = prm.lazy_gbar < 0 ? (is_tc_form(prm.form) ? 1 : 0) : prm.lazy_gbar;
                D.tc_n = tc_n;
            }
            for (int b = 0; b < nb[k]; b++) h_bmap[b0 + b] = k;
            b0 += nb[k];
            const InstanceLayout &Lk = lay[k];
            char *base = arena + inst_off[k];
            D.G = (double *)(base + Lk.G);
            D.G_bar = (double *)(base + Lk.Gb);
            D.QD = (double *)(base + Lk.QD);
            D.status = (unsigned char *)(base + Lk.S);
            D.pos_local = (int *)(base + Lk.PL);
            D.scratch = (int *)(base + Lk.Sc);
            D.cache.data = (float *)(base + Lk.Data);
            // initial state lives in the shared regions (positions start as local indices)
            D.alpha = (double *)(arena + o_alpha) + loff[k];
            D.p = (double *)(arena + o_p) + loff[k];
            D.pos_row = (int *)(arena + o_row) + loff[k];
            D.y = (signed char *)(arena + o_y) + loff[k];
            D.out = (SolveOut *)(arena + o_out) + k;
            D.alpha_local = (double *)(arena + o_alocal) + loff[k];
            D.sync = (GroupSync *)(arena + o_sync) + k;
            D.partials = (Partial *)(arena + o_part) + poff[k];
            D.cache.tag = (int *)(arena + o_tag) + coff[k];
            D.cache.epoch = (int *)(arena + o_ep) + coff[k];
            D.cache.stamp = (unsigned long long *)(arena + o_st) + coff[k];
            D.cache.nsets = Lk.sets;
            D.cache.nways = Lk.ways;
            D.cache.stride = l;
            memcpy(h_alpha + loff[k], sp.alpha0.data(), sizeof(double) * l);
            memcpy(h_p + loff[k], sp.p.data(), sizeof(double) * l);
            memcpy(h_row + loff[k], sp.rows.data(), sizeof(int) * l);
            memcpy(h_y + loff[k], sp.y.data(), (size_t)l);
        }
        memcpy(h_desc, desc.data(), sizeof(InstanceDesc) * count);
        clk.mark("pack");
        CK(xfer_async(arena, host, up_bytes, cudaMemcpyHostToDevice, s));
        CK(cudaMemsetAsync(arena + o_zero, 0, zero_bytes, s));
        CK(cudaMemsetAsync(arena + o_tag, 0xff, 4 * S, s));
        cudaEvent_t ev0, ev1;
        CK(cudaEventCreate(&ev0));
        CK(cudaEventCreate(&ev1));
        CK(cudaEventRecord(ev0, s));
        cudaError_t le = launch_smo(prm.form, d_desc, d_block_inst, used, dyn_smem, true, s);
        if (le == cudaSuccess) count_launch();
        cudaEventRecord(ev1, s);
        if (le == cudaSuccess) le = xfer_async(host + up_bytes, arena + o_out, down_bytes, cudaMemcpyDeviceToHost, s);
        clk.mark("launch");
        cudaError_t se = le == cudaSuccess ? cudaStreamSynchronize(s) : le;
        clk.mark("wait");
        float ms = 0;
        if (se == cudaSuccess) cudaEventElapsedTime(&ms, ev0, ev1);
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        int rc = 0;
        if (se != cudaSuccess) {
            set_error(std::string("solver launch failed: ") + cudaGetErrorString(se));
            rc = -1;
        }
        const SolveOut *h_out = (const SolveOut *)(host + up_bytes);
        const double *h_alocal = (const double *)(host + up_bytes + (o_alocal - o_out));
        for (int k = 0; k < count && rc == 0; k++) {
            SolveResult &R = res[first + k];
            const int l = desc[k].l;
            R.alpha.assign(h_alocal + loff[k], h_alocal + loff[k] + l);
            R.out = h_out[k];
            R.seconds = ms * 1e-3;
            if (R.out.status < 0) {
                set_error("solver group barrier timed out");
                rc = -1;
            }
        }
        clk.mark("unpack");
        if (rc) return rc;
        first = last;
    }
    return 0;
}

}  // namespace svmb
