// engine.cpp -- host orchestration of the device SMO solver.
//
// Replaces the reference's CudaSolver/CudaSolverNU host classes
// (reference libsvm/cuda_solver.cpp:159-555, cuda_solverNU.cpp:64-178): instead
// of launching 7-9 kernels and two blocking device->host copies per SMO
// iteration, the whole solve of every instance runs inside one persistent
// launch (smo_kernel.cu) and the host only uploads the problem and reads the
// result back.
#include "engine.hpp"
#include "svm_b200.h"

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <queue>

#include "svm.h"

namespace svmb {

// bound of the solver groups' cross-block waits (ns, 0: the kernel's default)
// and the one-shot test hook that launches a wave without its last block
static std::atomic<long long> g_wait_ns{0};
void set_wait_limit_ms(long long ms) { g_wait_ns = ms > 0 ? ms * 1000000LL : 0; }

static std::atomic<int> g_drop_block{0};

// solver blocks a launch may place on one SM (their shared memory is split)
static int g_blocks_per_sm = 1;
int set_blocks_per_sm(int b)
{
    if (b < 1 || b > 4) return -1;
    g_blocks_per_sm = b;
    return 0;
}
void arm_drop_block() { g_drop_block = 1; }


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
void count_transfer(long long h2d, long long d2h)
{
    g_h2d += h2d;
    g_d2h += d2h;
}
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
    explicit StageClock(const char *name = "solve_batch") : what(name) {}
    const char *what;
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
        if (trace_on() && !log.empty()) fprintf(stderr, "[svmb] %s%s\n", what, log.c_str());
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

// One grow-only device block reused by the row uploads of svm_train and
// svm_cross_validation (allocating and freeing 100+ MB per call costs tens of
// milliseconds); a second concurrent user gets a plain allocation.
static std::mutex g_rowpool_mu;
static char *g_rowpool = nullptr;
static size_t g_rowpool_bytes = 0;
static bool g_rowpool_busy = false;

static char *rowpool_take(size_t bytes)
{
    std::lock_guard<std::mutex> g(g_rowpool_mu);
    if (g_rowpool_busy) return nullptr;
    if (bytes > g_rowpool_bytes) {
        if (g_rowpool) cudaFree(g_rowpool);
        g_rowpool = nullptr;
        g_rowpool_bytes = 0;
        const size_t want = bytes + bytes / 4;
        if (cudaMalloc((void **)&g_rowpool, want) != cudaSuccess) {
            cudaGetLastError();
            g_rowpool = nullptr;
            return nullptr;
        }
        g_rowpool_bytes = want;
    }
    g_rowpool_busy = true;
    return g_rowpool;
}

static void rowpool_give(char *p)
{
    std::lock_guard<std::mutex> g(g_rowpool_mu);
    if (p == g_rowpool) g_rowpool_busy = false;
}

DeviceRows::~DeviceRows()
{
    if (block && block_pooled) rowpool_give(block);
    else if (block && !block_async) cudaFree(block);
    cudaFree(Xs);
    cudaFree(xinv);
}

void DeviceRows::release_async(cudaStream_t s)
{
    if (block) {
        if (block_pooled) rowpool_give(block);
        else if (block_async) cudaFreeAsync(block, s);
        else cudaFree(block);
    }
    block = nullptr;
    X = nullptr; rowptr = nullptr; col = nullptr; val = nullptr;
    xsq[0] = xsq[1] = nullptr;
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
               int force, cudaStream_t s, int alloc)
{
    const bool async_alloc = alloc == kAllocAsync;
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
    // the CSR arrays always travel; dense rows are scattered on the device.
    // One device block holds [rowptr][col][val][dense rows][norms x 2].
    out.nnz = nnz;
    auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
    const size_t b_rp = 0;
    const size_t b_col = al(b_rp + (size_t)(n + 1) * sizeof(long long));
    const size_t b_val = al(b_col + (size_t)std::max<long long>(nnz, 1) * sizeof(int));
    const size_t b_X = al(b_val + (size_t)std::max<long long>(nnz, 1) * sizeof(float));
    const size_t b_sq = al(b_X + (dense ? std::max<size_t>((size_t)n * out.ld, 4) * sizeof(float) : 0));
    const size_t b_end = b_sq + 2 * al((size_t)std::max(n, 1) * sizeof(double));
    char *blk = nullptr;
    if (alloc == kAllocPooled) blk = rowpool_take(b_end);
    out.block_pooled = blk != nullptr;
    if (!blk) {
        if (async_alloc) CK(cudaMallocAsync((void **)&blk, b_end, s));
        else CK(cudaMalloc((void **)&blk, b_end));
    }
    out.block = blk;
    out.block_async = async_alloc;
    out.block_bytes = b_end;
    out.rowptr = (long long *)(blk + b_rp);
    out.col = (int *)(blk + b_col);
    out.val = (float *)(blk + b_val);
    out.X = dense ? (float *)(blk + b_X) : nullptr;
    out.xsq[0] = (double *)(blk + b_sq);
    out.xsq[1] = (double *)(blk + b_sq + al((size_t)std::max(n, 1) * sizeof(double)));
    CK(xfer_async(out.rowptr, rowptr, (size_t)(n + 1) * sizeof(long long), cudaMemcpyHostToDevice, s));
    if (nnz) {
        CK(xfer_async(out.col, col, (size_t)nnz * sizeof(int), cudaMemcpyHostToDevice, s));
        CK(xfer_async(out.val, val, (size_t)nnz * sizeof(float), cudaMemcpyHostToDevice, s));
    }
    out.h2d_bytes = (size_t)(n + 1) * 8 + (size_t)nnz * 8;
    if (dense) {
        const size_t elems = std::max<size_t>((size_t)n * out.ld, 4);
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
        if (n) {
            CK(launch_xsq(out.view(f), n, out.xsq[f], f, s));
            count_launch();
        }
    }
    if (!async_alloc) CK(cudaStreamSynchronize(s));
    return 0;
}

// Dense rows [n][ld] built on the host, uploaded as they are: the device
// block holds [dense rows][norms x 2] and no CSR arrays.
static int upload_dense(const float *X, int n, int d, long long nnz, DeviceRows &out, cudaStream_t s, int alloc)
{
    const bool async_alloc = alloc == kAllocAsync;
    out.n = n;
    out.d = d > 0 ? d : 1;
    out.ld = (out.d + 3) & ~3;
    out.dense = true;
    out.nnz = nnz;
    auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
    const size_t xbytes = std::max<size_t>((size_t)n * out.ld, 4) * sizeof(float);
    const size_t b_sq = al(xbytes);
    const size_t b_end = b_sq + 2 * al((size_t)std::max(n, 1) * sizeof(double));
    char *blk = nullptr;
    if (alloc == kAllocPooled) blk = rowpool_take(b_end);
    out.block_pooled = blk != nullptr;
    if (!blk) {
        if (async_alloc) CK(cudaMallocAsync((void **)&blk, b_end, s));
        else CK(cudaMalloc((void **)&blk, b_end));
    }
    out.block = blk;
    out.block_async = async_alloc;
    out.block_bytes = b_end;
    out.rowptr = nullptr;
    out.col = nullptr;
    out.val = nullptr;
    out.X = (float *)blk;
    out.xsq[0] = (double *)(blk + b_sq);
    out.xsq[1] = (double *)(blk + b_sq + al((size_t)std::max(n, 1) * sizeof(double)));
    if (n) CK(xfer_async(out.X, X, (size_t)n * out.ld * sizeof(float), cudaMemcpyHostToDevice, s));
    out.h2d_bytes = (size_t)n * out.ld * sizeof(float);
    out.bytes = (size_t)n * out.ld * sizeof(float);
    for (int f = 0; f < 2; f++) {
        if (n) {
            CK(launch_xsq(out.view(f), n, out.xsq[f], f, s));
            count_launch();
        }
    }
    if (!async_alloc) CK(cudaStreamSynchronize(s));
    return 0;
}

// Row r of x written as a dense row of width d (padded to ld with zeros),
// columns index - base.  Returns its entry count, or -1 (nothing defined)
// when an index lies outside [base, base + d).
static long long dense_row(const svm_node *row_nodes, int base, int d, int ld, float *row)
{
    long long c = 0;
    int prev = -1;
    bool inorder = true;
    for (const svm_node *p = row_nodes; p->index != -1; ++p, ++c) {
        const int k = p->index - base;
        if (k < 0 || k >= d) return -1;
        if (k <= prev) inorder = false;
        prev = k;
        row[k] = (float)p->value;
    }
    if (inorder && c == d) {
        // every column written once: only the padding is cleared
        for (int k = d; k < ld; k++) row[k] = 0.0f;
    } else {
        memset(row, 0, sizeof(float) * ld);
        for (const svm_node *p = row_nodes; p->index != -1; ++p) row[p->index - base] = (float)p->value;
    }
    return c;
}

// upload_csr's layout rule: dense rows when they are not much larger than the CSR arrays
static bool dense_layout(int force, int n, int ld, long long nnz, double *dense_bytes, double *csr_bytes)
{
    *dense_bytes = (double)n * ld * 4.0;
    *csr_bytes = (double)(n + 1) * 8.0 + (double)nnz * 8.0;
    bool dense = force == 1 || (force < 0 && *dense_bytes <= 1.2 * *csr_bytes);
    if (dense && *dense_bytes > 60e9) dense = false;
    return dense;
}

int upload_rows(const svm_node *const *x, int n, DeviceRows &out, int force, cudaStream_t s, int alloc)
{
    // CSR with 0-based columns; libsvm indices start at 1 (index 0 is kept as a
    // column when present).  Rows are converted in parallel on the host.  When
    // the dense layout is chosen and is no larger than the CSR arrays, the rows
    // are built dense here and uploaded as they are (half the bytes of the CSR
    // arrays for fully dense data, and no scatter on the device).
    StageClock clk("upload_rows");
    std::lock_guard<std::mutex> g(g_pin_mu);
    auto pinned_rows = [](size_t elems, std::vector<float> &fallback) {
        float *X = (float *)pinned_staging(elems * sizeof(float));
        if (!X) {
            fallback.resize(elems);
            X = fallback.data();
        }
        return X;
    };
    if (force != 0 && n > 0) {
        // Dense data in one pass: when the first row holds every column from
        // its first index (0 or 1) on, the rows are written as dense rows of
        // that width while they are counted.  The result is the two-pass
        // path's exactly (same base, width and values); a row with an index
        // outside that range, or the layout rule choosing CSR, sends the call
        // on to the two passes.
        const svm_node *r0 = x[0];
        int c0 = 0;
        bool inc = r0[0].index == 0 || r0[0].index == 1;
        for (; r0[c0].index != -1; c0++)
            if (c0 > 0 && r0[c0].index != r0[c0 - 1].index + 1) inc = false;
        // (only while the attempt's dense rows stay modest: sparse data whose
        // first row happens to be complete would otherwise stage n x d floats)
        if (inc && c0 > 0 && (double)n * (double)((c0 + 3) & ~3) * 4.0 <= 4e9) {
            const int base = r0[0].index, d = c0, ld = (d + 3) & ~3;
            double db, cb;
            std::vector<float> fallback_x;
            float *X = pinned_rows(std::max<size_t>((size_t)n * ld, 4), fallback_x);
            long long nnz = 0;
            int bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : nnz) reduction(| : bad)
            for (int r = 0; r < n; r++) {
                const long long c = dense_row(x[r], base, d, ld, X + (size_t)r * ld);
                if (c < 0) bad = 1;
                else nnz += c;
            }
            if (!bad && dense_layout(force, n, ld, nnz, &db, &cb) && db <= cb) {
                clk.mark("convert");
                const int rc = upload_dense(X, n, d, nnz, out, s, alloc);
                clk.mark("upload");
                return rc;
            }
        }
    }
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
    {
        const int d = nnz ? max_index - base + 1 : 1;
        const int ld = (d + 3) & ~3;
        double db, cb;
        if (dense_layout(force, n, ld, nnz, &db, &cb) && db <= cb) {
            std::vector<float> fallback_x;
            float *X = pinned_rows(std::max<size_t>((size_t)n * ld, 4), fallback_x);
#pragma omp parallel for schedule(static)
            for (int r = 0; r < n; r++) dense_row(x[r], base, d, ld, X + (size_t)r * ld);
            clk.mark("convert");
            const int rc = upload_dense(X, n, d, nnz, out, s, alloc);
            clk.mark("upload");
            return rc;
        }
    }
    // CSR arrays built directly in page-locked staging memory
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
    clk.mark("convert");
    const int rc = upload_csr(rp, col, val, n, d, out, force, s, alloc);
    clk.mark("upload");
    return rc;
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
using InstanceLayout = Wave::Layout;

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

}  // namespace

size_t instance_bytes(int l, double cache_mb) { return instance_layout(l, 1, cache_mb).bytes; }

namespace {

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

// ---------------------------------------------------------------------------
// waves: the instances of one persistent launch
// ---------------------------------------------------------------------------
namespace {

constexpr int kChunkBytes = 3 * 8 + 2 * 4 + 2;     // per position: G, alpha, QD, col, row, y, status

// dynamic shared memory a solver block can use beside its static part
long long smem_budget()
{
    int smem_total = 0, smem_sm = 0, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&smem_total, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess) return -1;
    // with several solver blocks per SM each gets its share of the SM's
    // shared memory (less the 1 KB the runtime reserves per block)
    const long long per_block = std::min<long long>(smem_total, smem_sm / g_blocks_per_sm - 1024);
    return per_block - smo_static_smem() - 1024;
}

// shared-memory staging of one instance's rows: source rows staged in
// float32 (CUDA-core forms) or the tensor-core operand stages
struct StagePlan {
    int stage_cap = 0, stage_lds = 0, tc_n = 0, tile_bufs = 2, hash_slots = 0;
    long long bytes = 0;        // staging + aux area
    long long chunk_max = 0;    // positions of state one block can hold
};

StagePlan stage_plan(const DeviceRows &rows, int form, long long budget, int tile_bufs)
{
    StagePlan p;
    p.tile_bufs = tile_bufs;
    if (is_tc_form(form)) {
        p.tc_n = kTcMaxN;
        while (p.tc_n > 16 && (budget - tc_area_bytes(p.tc_n) - kAuxBytesTc) / kChunkBytes < 1024) p.tc_n /= 2;
        p.bytes = tc_area_bytes(p.tc_n);
    } else {
        if (rows.dense) {
            p.stage_lds = rows.ld;
            p.stage_cap = (int)std::min<long long>(kSrcBatch, (48LL << 10) / ((long long)std::max(rows.ld, 4) * 4));
        } else {
            p.stage_lds = rows.d;
            p.stage_cap = (int)std::min<long long>(kSrcBatch, (budget / 2) / ((long long)std::max(rows.d, 1) * 4));
        }
        if (p.stage_cap < 2) p.stage_cap = 0;
        // the exact form stages its source values as float64
        const long long elem = form == FORM_EXACT ? 8 : 4;
        p.bytes = (((long long)p.stage_cap * p.stage_lds * elem) + 15) & ~15LL;
        if (!rows.dense && p.stage_cap == 0) {
            // too wide to scatter: the sources go into a column-keyed table
            p.hash_slots = kHashSlots;
            p.bytes = hash_bytes(form);
        }
    }
    p.bytes += aux_bytes(form, tile_bufs);   // transpose tiles / prefetch candidates / block-product partial sums
    p.chunk_max = (budget - p.bytes) / kChunkBytes;
    return p;
}

const SolveParams &params_of(const SubProblem &sp, const SolveParams &prm) { return sp.own ? *sp.own : prm; }
const DeviceRows &rows_of(const SubProblem &sp, const DeviceRows &rows) { return sp.rows_dev ? *sp.rows_dev : rows; }

}  // namespace

int wave_plan(const DeviceRows &rows, const std::vector<SubProblem> &subs, const SolveParams &prm, int first,
              int capacity, Wave &w, int limit)
{
    const int ninst = limit >= 0 && limit < (int)subs.size() ? limit : (int)subs.size();
    const int tune_pf = w.tune_prefetch, tune_rpb = w.tune_rows_per_block;
    w = Wave();
    w.tune_prefetch = tune_pf;
    w.tune_rows_per_block = tune_rpb;
    w.first = first;
    w.form = prm.form;
    const long long budget = smem_budget();
    if (budget <= 0) {
        set_error("cannot query the device's shared memory");
        return -1;
    }
    const int sms = device_sm_count();
    std::vector<StagePlan> sp_all;
    std::vector<long long> nmin;
    int last = first;
    // the instances from `first` that one launch holds with `bufs` transpose
    // tiles per warp.  Returns -1 on an error that no depth avoids, -2 when the
    // first instance does not fit at this depth (reported only at depth 1).
    auto fit = [&](int bufs, std::vector<StagePlan> &sps, std::vector<long long> &nms, int &end) -> int {
        sps.clear();
        nms.clear();
        long long need = 0;
        end = first;
        while (end < ninst) {
            const SubProblem &sp = subs[end];
            const SolveParams &p = params_of(sp, prm);
            if (p.form != prm.form) {
                set_error("instances of one launch must share the arithmetic form");
                return -1;
            }
            const StagePlan st = stage_plan(rows_of(sp, rows), prm.form, budget, bufs);
            if (st.chunk_max < 64) {
                if (bufs > 1) return -2;
                set_error("not enough shared memory for the solver state");
                return -1;
            }
            const long long l = (long long)sp.rows.size();
            const long long nm = std::max<long long>(1, (l + st.chunk_max - 1) / st.chunk_max);
            if (nm > capacity) {
                if (end == first) {
                    if (bufs > 1) return -2;
                    set_error("problem too large: more positions than the device's blocks can hold in shared memory");
                    return -1;
                }
                break;
            }
            if (need + nm > capacity) break;
            need += nm;
            sps.push_back(st);
            nms.push_back(nm);
            end++;
        }
        return 0;
    };
    if (is_tc_form(prm.form)) {
        // the tensor forms have no transpose tiles
        if (fit(2, sp_all, nmin, last) != 0) return -1;
    } else {
        // the deepest ring (deeper rings keep more of a fill in flight) among
        // those that put the most instances into this launch
        int best = first;
        std::vector<StagePlan> spb;
        std::vector<long long> nmb;
        for (int bufs = fill_depth(); bufs >= 1; bufs--) {
            int end = first;
            const int rc = fit(bufs, spb, nmb, end);
            if (rc == -1) return -1;
            if (rc == 0 && end > best) {
                best = end;
                sp_all.swap(spb);
                nmin.swap(nmb);
            }
        }
        last = best;
    }
    const int count = last - first;
    w.count = count;
    w.nb.assign(count, 1);
    // Blocks per instance: every instance starts with the blocks its state
    // needs in shared memory; the remaining blocks go one at a time to the
    // instance with the most positions per block, each up to min(SMs, l/500)
    // (or its override).  The instances of a launch iterate about equally
    // often, and an iteration's row evaluations take time in proportion to
    // the positions per block, so equal chunks make the instances finish
    // together; the l/500 cap keeps the cross-block exchanges of a small
    // instance cheap.
    std::vector<int> cap(count);
    int used = 0;
    for (int k = 0; k < count; k++) {
        const SubProblem &sp = subs[first + k];
        const long long l = (long long)sp.rows.size();
        const int bo = params_of(sp, prm).blocks_override;
        const long long rpb = std::max(1, w.tune_rows_per_block);
        long long want = bo > 0 ? bo : std::max<long long>(1, std::min<long long>(sms, (l + rpb - 1) / rpb));
        want = std::min<long long>(want, std::max<long long>(1, l));
        want = std::min<long long>(want, std::min(kThreads, kMaxGroupBlocks));
        w.nb[k] = (int)nmin[k];
        cap[k] = (int)std::max<long long>(nmin[k], want);
        used += w.nb[k];
    }
    {
        auto per_block = [&](int k) { return (double)subs[first + k].rows.size() / (double)w.nb[k]; };
        auto cmp = [&](int a, int b) { return per_block(a) < per_block(b) || (per_block(a) == per_block(b) && a > b); };
        std::priority_queue<int, std::vector<int>, decltype(cmp)> q(cmp);
        for (int k = 0; k < count; k++)
            if (w.nb[k] < cap[k]) q.push(k);
        while (used < capacity && !q.empty()) {
            const int k = q.top();
            q.pop();
            w.nb[k]++;
            used++;
            if (w.nb[k] < cap[k]) q.push(k);
        }
    }
    w.used = used;
    w.stage.resize(count);
    w.fill_path.assign(count, 0);
    w.tile_bufs = count > 0 ? sp_all[0].tile_bufs : 2;
    long long dyn = 0;
    for (int k = 0; k < count; k++) {
        const long long l = (long long)subs[first + k].rows.size();
        const long long cap = (l + w.nb[k] - 1) / w.nb[k];
        w.stage[k][0] = sp_all[k].stage_cap;
        w.stage[k][1] = sp_all[k].stage_lds;
        w.stage[k][2] = sp_all[k].tc_n;
        w.stage[k][3] = (int)cap;
        w.stage[k][4] = sp_all[k].hash_slots;
        const bool dense = rows_of(subs[first + k], rows).dense;
        w.fill_path[k] = is_tc_form(prm.form)           ? SVMB_FILL_TENSOR
                         : dense                        ? SVMB_FILL_DENSE
                         : sp_all[k].stage_cap > 0      ? SVMB_FILL_SPARSE_SCATTER
                         : sp_all[k].hash_slots > 0     ? SVMB_FILL_SPARSE_TABLE
                                                        : SVMB_FILL_SPARSE_MERGE;
        dyn = std::max(dyn, sp_all[k].bytes + cap * kChunkBytes);
    }
    w.dyn_smem = (size_t)dyn;

    // One device block per wave, laid out so that the host touches it with
    // one upload, three fills and two downloads:
    //   upload   [descriptors][block map][alpha][p][row ids][labels]
    //   download [outputs][alpha by local index]
    //   zero     [group syncs][exchange records][cache epochs][cache stamps]
    //   0xff     [cache tags]
    //   per instance: G, G_bar, QD, status, position->local, shrink lists, Q rows
    auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
    w.loff.assign(count + 1, 0);
    w.poff.assign(count + 1, 0);
    w.coff.assign(count + 1, 0);
    w.lay.resize(count);
    for (int k = 0; k < count; k++) {
        const SubProblem &sp = subs[first + k];
        const int l = (int)sp.rows.size();
        w.lay[k] = instance_layout(l, w.nb[k], params_of(sp, prm).cache_mb);
        w.loff[k + 1] = w.loff[k] + (size_t)l;
        w.poff[k + 1] = w.poff[k] + 2 * (size_t)w.nb[k];
        w.coff[k + 1] = w.coff[k] + (size_t)w.lay[k].sets * w.lay[k].ways;
    }
    const size_t L = w.loff[count], P = w.poff[count], S = w.coff[count];
    size_t off = 0;
    w.o_desc = off; off = al(off + sizeof(InstanceDesc) * count);
    w.o_bmap = off; off = al(off + sizeof(int) * used);
    w.o_alpha = off; off = al(off + 8 * L);
    w.o_p = off; off = al(off + 8 * L);
    w.o_row = off; off = al(off + 4 * L);
    w.o_y = off; off = al(off + L);
    w.up_bytes = off;
    w.o_out = off; off = al(off + sizeof(SolveOut) * count);
    w.o_alocal = off; off = al(off + 8 * L);
    w.down_bytes = off - w.o_out;
    w.o_zero = off;
    w.o_sync = off; off = al(off + sizeof(GroupSync) * count);
    w.o_part = off; off = al(off + sizeof(Partial) * P);
    w.o_ep = off; off = al(off + 4 * S);
    w.o_st = off; off = al(off + 8 * S);
    w.zero_bytes = off - w.o_zero;
    w.o_tag = off; off = al(off + 4 * S);
    w.tag_bytes = 4 * S;
    w.inst_off.resize(count);
    for (int k = 0; k < count; k++) {
        w.inst_off[k] = off;
        off += w.lay[k].bytes;
    }
    w.dev_bytes = off;
    return 0;
}

// The stream work of a wave: upload, fills, the launch between two timing
// events, the result download, and the completion event.
static cudaError_t wave_issue(Wave &w, InstanceDesc *d_desc, int *d_block_inst, cudaStream_t s, bool capturing = false)
{
    const unsigned rec = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    char *dev = w.dev, *host = w.host;
    cudaError_t e = xfer_async(dev, host, w.up_bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(dev + w.o_zero, 0, w.zero_bytes, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(dev + w.o_tag, 0xff, w.tag_bytes, s);
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(w.ev0, s, rec);
    if (e == cudaSuccess)
        e = launch_smo(w.form, d_desc, d_block_inst, w.used - (w.drop_last_block ? 1 : 0), w.dyn_smem, w.cooperative, s);
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(w.ev1, s, rec);
    if (e == cudaSuccess) e = xfer_async(host + w.up_bytes, dev + w.o_out, w.down_bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(w.done, s, rec);
    return e;
}

// ---- CUDA graphs of repeated waves ----------------------------------------
// A wave whose layout, device block and host staging are the same as an
// earlier one (the arena and the staging are reused) replays a graph of its
// stream work captured the first time: one graph launch instead of seven
// stream operations.  The graph owns its timing and completion events.
namespace {
struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, done = nullptr;
    bool failed = false;
};
std::map<std::string, GraphEntry> g_graphs;     // guarded by the arena lock of solve_batch
std::atomic<long long> g_graph_captured{0}, g_graph_replayed{0};

std::string graph_key(const Wave &w)
{
    char buf[512];
    snprintf(buf, sizeof buf, "%p:%p:%zu:%zu:%zu:%zu:%zu:%zu:%zu:%d:%zu:%d:%d", (void *)w.dev, (void *)w.host, w.up_bytes,
             w.down_bytes, w.zero_bytes, w.tag_bytes, w.o_zero, w.o_tag, w.o_out, w.used, w.dyn_smem, w.form,
             (int)w.cooperative);
    return std::string(buf) + ":" + std::to_string(w.o_desc) + ":" + std::to_string(w.o_bmap);
}
}  // namespace

void graph_counts(long long *captured, long long *replayed)
{
    if (captured) *captured = g_graph_captured.load();
    if (replayed) *replayed = g_graph_replayed.load();
}

static int wave_issue_graph(Wave &w, InstanceDesc *d_desc, int *d_block_inst, cudaStream_t s)
{
    const std::string key = graph_key(w);
    if (g_graphs.size() > 64) {
        for (auto &kv : g_graphs) {
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
            if (kv.second.ev0) cudaEventDestroy(kv.second.ev0);
            if (kv.second.ev1) cudaEventDestroy(kv.second.ev1);
            if (kv.second.done) cudaEventDestroy(kv.second.done);
        }
        g_graphs.clear();
    }
    GraphEntry &ge = g_graphs[key];
    if (!ge.ev0) {
        CK(cudaEventCreate(&ge.ev0));
        CK(cudaEventCreate(&ge.ev1));
        CK(cudaEventCreateWithFlags(&ge.done, cudaEventDisableTiming));
    }
    w.ev0 = ge.ev0;
    w.ev1 = ge.ev1;
    w.done = ge.done;
    w.own_events = false;
    if (!ge.exec && !ge.failed) {
        // capture once; a stream work that cannot be captured runs directly from then on
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            const cudaError_t ie = wave_issue(w, d_desc, d_block_inst, s, true);
            e = cudaStreamEndCapture(s, &graph);
            if (ie != cudaSuccess) e = ie;
            // captured copies did not run: take back the bytes xfer_async counted
            count_transfer(-(long long)w.up_bytes, -(long long)w.down_bytes);
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&ge.exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (trace_on()) fprintf(stderr, "[svmb] graph capture: %s\n", cudaGetErrorString(e));
        if (e != cudaSuccess) {
            cudaGetLastError();
            ge.exec = nullptr;
            ge.failed = true;
        } else {
            g_graph_captured++;
        }
    }
    if (ge.exec) {
        // the captured copies do not pass through xfer_async: count their bytes here
        count_transfer((long long)w.up_bytes, (long long)w.down_bytes);
        CK(cudaGraphLaunch(ge.exec, s));
        g_graph_replayed++;
    } else {
        cudaGetLastError();
        cudaError_t le = wave_issue(w, d_desc, d_block_inst, s);
        if (le != cudaSuccess) {
            set_error(std::string("solver launch (after a graph capture that failed) failed: ") + cudaGetErrorString(le));
            return -1;
        }
    }
    count_launch();
    return 0;
}

int wave_start(const DeviceRows &rows, const std::vector<SubProblem> &subs, const SolveParams &prm, Wave &w,
               char *dev, char *host, cudaStream_t s)
{
    const int count = w.count, first = w.first;
    w.dev = dev;
    w.host = host;
    w.stream = s;
    InstanceDesc *h_desc = (InstanceDesc *)(host + w.o_desc);
    int *h_bmap = (int *)(host + w.o_bmap);
    double *h_alpha = (double *)(host + w.o_alpha);
    double *h_p = (double *)(host + w.o_p);
    int *h_row = (int *)(host + w.o_row);
    signed char *h_y = (signed char *)(host + w.o_y);
    InstanceDesc *d_desc = (InstanceDesc *)(dev + w.o_desc);
    int *d_block_inst = (int *)(dev + w.o_bmap);
    int b0 = 0;
    for (int k = 0; k < count; k++) {
        const SubProblem &sp = subs[first + k];
        const SolveParams &p = params_of(sp, prm);
        const DeviceRows &r = rows_of(sp, rows);
        const int l = (int)sp.rows.size();
        InstanceDesc &D = h_desc[k];
        memset(&D, 0, sizeof(D));
        D.l = l;
        D.nu = sp.nu;
        D.shrinking = p.shrinking;
        D.form = prm.form;
        D.Cp = sp.Cp;
        D.Cn = sp.Cn;
        D.eps = p.eps;
        D.max_iter = std::max<long long>(10000000LL, l > INT_MAX / 100 ? (long long)INT_MAX : 100LL * l);
        D.kp = p.kp;
        D.x = r.view(prm.form);
        D.block0 = b0;
        D.nblocks = w.nb[k];
        D.stage_cap = w.stage[k][0];
        D.stage_lds = w.stage[k][1];
        D.tc_n = w.stage[k][2];
        D.chunk_cap = w.stage[k][3];
        D.hash_slots = w.stage[k][4];
        D.wait_ns = g_wait_ns.load();
        D.done_flag = w.done_flags ? w.done_flags + k : nullptr;
        D.tile_bufs = w.tile_bufs;
        {
            const int limit = D.stage_cap > 0 ? std::min(kPrefetchMax, D.stage_cap) : kPrefetchMax;
            const int pf = w.tune_prefetch > 0 ? w.tune_prefetch : p.prefetch;
            D.prefetch = pf > 0 ? std::min(pf, limit) : limit;
            D.lazy_gbar = p.lazy_gbar < 0 ? (is_tc_form(prm.form) ? 1 : 0) : p.lazy_gbar;
        }
        for (int b = 0; b < w.nb[k]; b++) h_bmap[b0 + b] = k;
        b0 += w.nb[k];
        const InstanceLayout &Lk = w.lay[k];
        char *base = dev + w.inst_off[k];
        D.G = (double *)(base + Lk.G);
        D.G_bar = (double *)(base + Lk.Gb);
        D.QD = (double *)(base + Lk.QD);
        D.status = (unsigned char *)(base + Lk.S);
        D.pos_local = (int *)(base + Lk.PL);
        D.scratch = (int *)(base + Lk.Sc);
        D.cache.data = (float *)(base + Lk.Data);
        // initial state lives in the shared regions (positions start as local indices)
        D.alpha = (double *)(dev + w.o_alpha) + w.loff[k];
        D.p = (double *)(dev + w.o_p) + w.loff[k];
        D.pos_row = (int *)(dev + w.o_row) + w.loff[k];
        D.y = (signed char *)(dev + w.o_y) + w.loff[k];
        D.out = (SolveOut *)(dev + w.o_out) + k;
        D.alpha_local = (double *)(dev + w.o_alocal) + w.loff[k];
        D.sync = (GroupSync *)(dev + w.o_sync) + k;
        D.partials = (Partial *)(dev + w.o_part) + w.poff[k];
        D.cache.tag = (int *)(dev + w.o_tag) + w.coff[k];
        D.cache.epoch = (int *)(dev + w.o_ep) + w.coff[k];
        D.cache.stamp = (unsigned long long *)(dev + w.o_st) + w.coff[k];
        D.cache.nsets = Lk.sets;
        D.cache.nways = Lk.ways;
        D.cache.stride = l;
    }
    // the instances' initial state into the staging block, on all host threads
#pragma omp parallel for schedule(dynamic, 1) if (count > 1)
    for (int k = 0; k < count; k++) {
        const SubProblem &sp = subs[first + k];
        const size_t l = sp.rows.size();
        memcpy(h_alpha + w.loff[k], sp.alpha0.data(), sizeof(double) * l);
        memcpy(h_p + w.loff[k], sp.p.data(), sizeof(double) * l);
        memcpy(h_row + w.loff[k], sp.rows.data(), sizeof(int) * l);
        memcpy(h_y + w.loff[k], sp.y.data(), l);
    }
    if (g_drop_block.exchange(0)) {
        w.drop_last_block = true;
        w.use_graph = false;
    }
    if (w.use_graph) return wave_issue_graph(w, d_desc, d_block_inst, s);
    CK(cudaEventCreate(&w.ev0));
    CK(cudaEventCreate(&w.ev1));
    CK(cudaEventCreateWithFlags(&w.done, cudaEventDisableTiming));
    w.own_events = true;
    cudaError_t le = wave_issue(w, d_desc, d_block_inst, s);
    if (le != cudaSuccess) {
        set_error(std::string("solver launch failed: ") + cudaGetErrorString(le));
        return -1;
    }
    count_launch();
    return 0;
}

bool wave_ready(const Wave &w) { return w.done && cudaEventQuery(w.done) != cudaErrorNotReady; }

int wave_fetch(const Wave &w, int k, SolveResult &r, cudaStream_t s)
{
    const size_t l = w.loff[k + 1] - w.loff[k];
    r.alpha.resize(l);
    CK(xfer_async(&r.out, w.dev + w.o_out + sizeof(SolveOut) * k, sizeof(SolveOut), cudaMemcpyDeviceToHost, s));
    if (l) CK(xfer_async(r.alpha.data(), w.dev + w.o_alocal + 8 * w.loff[k], 8 * l, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    r.seconds = 0;
    r.fill_path = w.fill_path[k];
    if (r.out.status < 0) {
        set_error("solver group barrier timed out");
        return -1;
    }
    return 0;
}

int wave_finish(Wave &w, std::vector<SolveResult> &res)
{
    cudaError_t se = w.done ? cudaEventSynchronize(w.done) : cudaErrorInvalidResourceHandle;
    float ms = 0;
    if (se == cudaSuccess) se = cudaEventElapsedTime(&ms, w.ev0, w.ev1);
    if (w.own_events) {
        if (w.ev0) cudaEventDestroy(w.ev0);
        if (w.ev1) cudaEventDestroy(w.ev1);
        if (w.done) cudaEventDestroy(w.done);
    }
    w.ev0 = w.ev1 = w.done = nullptr;
    if (se != cudaSuccess) {
        set_error(std::string("solver launch failed: ") + cudaGetErrorString(se));
        return -1;
    }
    w.ms = ms;
    const SolveOut *h_out = (const SolveOut *)(w.host + w.up_bytes);
    const double *h_alocal = (const double *)(w.host + w.up_bytes + (w.o_alocal - w.o_out));
    int rc = 0;
#pragma omp parallel for schedule(dynamic, 1) if (w.count > 1)
    for (int k = 0; k < w.count; k++) {
        SolveResult &R = res[w.first + k];
        const size_t l = w.loff[k + 1] - w.loff[k];
        R.alpha.assign(h_alocal + w.loff[k], h_alocal + w.loff[k] + l);
        R.out = h_out[k];
        R.seconds = ms * 1e-3;
        R.fill_path = w.fill_path[k];
    }
    for (int k = 0; k < w.count; k++)
        if (h_out[k].status < 0) {
            set_error("solver group barrier timed out");
            rc = -1;
        }
    return rc;
}

// ---------------------------------------------------------------------------
// autotuner
// ---------------------------------------------------------------------------
namespace {

// knobs that change only speed: rows per fill pass (prefetch depth) and the
// positions per block a solve aims at (its block count)
constexpr int kTunePrefetch[] = {0, 4, 2, 1};         // 0: as deep as staging allows
constexpr int kTuneRowsPerBlock[] = {500, 250, 1000};

struct TuneState {
    int stage = 0;          // 0: trying depths, 1: trying block targets, 2: settled
    int idx = 0;            // candidate being tried in the current stage
    int best_pf = 0, best_rpb = 500;
    double best_ms = 1e300;
};

std::mutex g_tune_mu;
std::map<std::string, TuneState> g_tune;
int g_tune_on = 1;
int g_last_pf = 0, g_last_rpb = 500, g_last_explore = 0;

}  // namespace

struct TuneChoice {
    std::string key;
    int prefetch = 0, rows_per_block = 500;
    bool active = false;
};

// signature: form, layout, width, and the instances' sizes rounded to powers of two
static std::string tune_key(const DeviceRows &rows, const std::vector<SubProblem> &subs, const SolveParams &prm)
{
    std::vector<int> b;
    for (const SubProblem &sp : subs) {
        int l = (int)sp.rows.size(), k = 0;
        while ((1 << k) < l) k++;
        b.push_back(k);
    }
    std::sort(b.begin(), b.end());
    std::string key = std::to_string(prm.form) + ":" + std::to_string(rows.dense) + ":" + std::to_string(rows.d) + ":";
    for (int v : b) key += std::to_string(v) + ",";
    return key;
}

TuneChoice tune_pick(const DeviceRows &rows, const std::vector<SubProblem> &subs, const SolveParams &prm, bool user_fixed)
{
    TuneChoice c;
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_last_explore = 0;
    if (!g_tune_on || user_fixed) {
        g_last_pf = 0;
        g_last_rpb = 500;
        return c;
    }
    c.key = tune_key(rows, subs, prm);
    c.active = true;
    TuneState &t = g_tune[c.key];
    if (t.stage == 0) {
        c.prefetch = kTunePrefetch[t.idx];
        c.rows_per_block = 500;
        g_last_explore = 1;
    } else if (t.stage == 1) {
        c.prefetch = t.best_pf;
        c.rows_per_block = kTuneRowsPerBlock[t.idx];
        g_last_explore = 1;
    } else {
        c.prefetch = t.best_pf;
        c.rows_per_block = t.best_rpb;
    }
    g_last_pf = c.prefetch;
    g_last_rpb = c.rows_per_block;
    return c;
}

void tune_record(const TuneChoice &c, double ms)
{
    if (!c.active) return;
    std::lock_guard<std::mutex> g(g_tune_mu);
    TuneState &t = g_tune[c.key];
    if (t.stage == 2) return;
    if (ms < t.best_ms) {
        t.best_ms = ms;
        t.best_pf = c.prefetch;
        t.best_rpb = c.rows_per_block;
    }
    t.idx++;
    const int n0 = (int)(sizeof(kTunePrefetch) / sizeof(int)), n1 = (int)(sizeof(kTuneRowsPerBlock) / sizeof(int));
    if (t.stage == 0 && t.idx >= n0) { t.stage = 1; t.idx = 1; }      // 500 rows per block was measured in stage 0
    else if (t.stage == 1 && t.idx >= n1) t.stage = 2;
}

void set_autotune(int on)
{
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune_on = on ? 1 : 0;
}

void autotune_last(int *prefetch, int *rows_per_block, int *exploring)
{
    std::lock_guard<std::mutex> g(g_tune_mu);
    if (prefetch) *prefetch = g_last_pf;
    if (rows_per_block) *rows_per_block = g_last_rpb;
    if (exploring) *exploring = g_last_explore;
}

static int g_graphs_on = 1;
void set_graphs(int on) { g_graphs_on = on ? 1 : 0; }


static int g_fill_depth = 2;
int set_fill_depth(int bufs)
{
    if (bufs < 1 || bufs > kMaxTileBufs) return -1;
    g_fill_depth = bufs;
    return 0;
}
int fill_depth() { return g_fill_depth; }

// one non-blocking stream per device for the waves of solve_batch
static cudaStream_t solver_stream()
{
    static std::map<int, cudaStream_t> streams;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    auto it = streams.find(dev);
    if (it != streams.end()) return it->second;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    streams[dev] = st;
    return st;
}

int solve_batch(const DeviceRows &rows, const std::vector<SubProblem> &subs, const SolveParams &prm,
                std::vector<SolveResult> &res, cudaStream_t s)
{
    const int ninst = (int)subs.size();
    res.assign(ninst, SolveResult());
    if (ninst == 0) return 0;
    // the split copy of the rows is a derived cache of the rows, built on first use
    if (const_cast<DeviceRows &>(rows).prepare_form(prm.form, s) != 0) return -1;
    for (const SubProblem &sp : subs)
        if (sp.rows_dev && const_cast<DeviceRows *>(sp.rows_dev)->prepare_form(prm.form, s) != 0) return -1;
    std::lock_guard<std::mutex> arena_lock(g_arena_mu);
    StageClock clk;
    // the waves run on the engine's own non-blocking stream (a capturable one);
    // everything they read was uploaded and synchronised before this call
    cudaStream_t ws = solver_stream();
    if (!ws) ws = s;
    const int sms = device_sm_count();
    if (sms <= 0) {
        set_error("no CUDA device");
        return -1;
    }
    // co-resident capacity of the persistent kernel at the largest shared memory it may use
    const long long budget = smem_budget();
    int per_sm = 0;
    CK(smo_max_blocks(prm.form, (size_t)std::max<long long>(budget, 0), &per_sm));
    if (per_sm < 1) {
        set_error("solver kernel does not fit on an SM");
        return -1;
    }
    const int capacity = per_sm * sms;
    clk.mark("setup");
    // More instances than one launch holds: launch instances of the same
    // parameters together (kernel, C: a grid point's solves take similar
    // numbers of iterations, other points' may take ten times as many), and
    // within those the largest first, so that each launch holds instances of
    // similar length (a launch lasts as long as its longest solve, and its
    // other SMs idle meanwhile).  Results do not depend on which instances
    // share a launch.
    std::vector<SubProblem> sorted_subs;
    std::vector<int> order;
    std::vector<int> group_end;     // per planned position: the end of its parameter group
    const std::vector<SubProblem> *plan = &subs;
    if (ninst > capacity) {
        order.resize(ninst);
        for (int k = 0; k < ninst; k++) order[k] = k;
        // group of an instance: the rank of its parameters in numeric order
        // (kernel, gamma, ..., C)
        std::vector<int> group(ninst, 0);
        {
            std::vector<std::array<double, 6>> key(ninst);
            for (int k = 0; k < ninst; k++) {
                const SolveParams &p = params_of(subs[k], prm);
                key[k] = {(double)p.kp.type, (double)p.kp.degree, p.kp.gamma, p.kp.coef0, subs[k].Cp, subs[k].Cn};
            }
            std::vector<std::array<double, 6>> uniq(key);
            std::sort(uniq.begin(), uniq.end());
            uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
            for (int k = 0; k < ninst; k++)
                group[k] = (int)(std::lower_bound(uniq.begin(), uniq.end(), key[k]) - uniq.begin());
        }
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            if (group[a] != group[b]) return group[a] < group[b];
            return subs[a].rows.size() > subs[b].rows.size();
        });
        sorted_subs.reserve(ninst);
        for (int k : order) sorted_subs.push_back(subs[k]);
        plan = &sorted_subs;
        // a launch holds the instances of one group only: the first launches
        // of the next group hold its largest instances, which (other
        // parameters, other iteration counts) would set the length of a
        // launch that mixes them with the previous group's smallest
        group_end.assign(ninst, ninst);
        for (int k = ninst - 1; k > 0; k--)
            group_end[k - 1] = group[order[k - 1]] == group[order[k]] ? group_end[k] : k;
    }
    std::vector<SolveResult> sorted_res;
    std::vector<SolveResult> &out = order.empty() ? res : sorted_res;
    if (!order.empty()) sorted_res.assign(ninst, SolveResult());
    // autotuner: the configuration for this call
    bool user_fixed = false;
    for (const SubProblem &sp : subs) {
        const SolveParams &p = params_of(sp, prm);
        if (p.prefetch > 0 || p.blocks_override > 0) user_fixed = true;
    }
    TuneChoice tune = tune_pick(rows, subs, prm, user_fixed);
    double total_ms = 0;
    int first = 0, nwave = 0;
    while (first < ninst) {
        Wave w;
        w.tune_prefetch = tune.prefetch;
        w.tune_rows_per_block = tune.rows_per_block;
        if (wave_plan(rows, *plan, prm, first, capacity, w, group_end.empty() ? -1 : group_end[first]) != 0) return -1;
        clk.mark("plan");
        char *arena = arena_reserve(w.dev_bytes);
        if (!arena) {
            set_error("device allocation for solver state failed (" + std::to_string(w.dev_bytes >> 20) + " MiB)");
            return -1;
        }
        char *host = (char *)pinned_staging_slot(1, w.up_bytes + w.down_bytes);
        std::vector<char> host_fallback;
        if (!host) {
            host_fallback.resize(w.up_bytes + w.down_bytes);
            host = host_fallback.data();
        }
        clk.mark("arena");
        w.use_graph = g_graphs_on && host != host_fallback.data();
        if (wave_start(rows, *plan, prm, w, arena, host, ws) != 0) return -1;
        clk.mark("launch");
        if (wave_finish(w, out) != 0) return -1;
        clk.mark("finish");
        total_ms += w.ms;
        for (int k = 0; k < w.count; k++) out[first + k].wave = nwave;
        nwave++;
        first += w.count;
    }
    for (size_t i = 0; i < order.size(); i++) res[order[i]] = std::move(sorted_res[i]);
    tune_record(tune, total_ms);
    return 0;
}

}  // namespace svmb
