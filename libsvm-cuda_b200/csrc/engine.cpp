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
void *g_pin = nullptr;
size_t g_pin_bytes = 0;
}  // namespace
void *pinned_staging(size_t bytes)
{
    if (bytes <= g_pin_bytes) return g_pin;
    if (g_pin) cudaFreeHost(g_pin);
    g_pin = nullptr;
    g_pin_bytes = 0;
    size_t want = std::max<size_t>(bytes, 1 << 20);
    if (cudaHostAlloc(&g_pin, want, cudaHostAllocDefault) != cudaSuccess) {
        g_pin = nullptr;
        return nullptr;
    }
    g_pin_bytes = want;
    return g_pin;
}

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
    v.xsq = xsq[form];
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
    // CSR with 0-based columns; libsvm indices start at 1 (index 0 is kept as a column when present)
    int min_index = INT_MAX, max_index = 0;
    long long nnz = 0;
    for (int r = 0; r < n; r++)
        for (const svm_node *p = x[r]; p->index != -1; ++p) {
            min_index = std::min(min_index, p->index);
            max_index = std::max(max_index, p->index);
            nnz++;
        }
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
    long long k = 0;
    for (int r = 0; r < n; r++) {
        rp[r] = k;
        for (const svm_node *p = x[r]; p->index != -1; ++p) {
            col[k] = p->index - base;
            val[k] = (float)p->value;
            k++;
        }
    }
    rp[n] = k;
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

struct InstanceAlloc {
    char *base = nullptr;
    size_t bytes = 0;
};

}  // namespace

int solve_batch(const DeviceRows &rows, const std::vector<SubProblem> &subs, const SolveParams &prm,
                std::vector<SolveResult> &res, cudaStream_t s)
{
    const int ninst = (int)subs.size();
    res.assign(ninst, SolveResult());
    if (ninst == 0) return 0;
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
    const long long stage_bytes = (((long long)stage_cap * stage_lds * 4) + 15) & ~15LL;
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
        for (int k = 0; k < count; k++) {
            const long long l = (long long)subs[first + k].rows.size();
            const int nmin = (int)std::max<long long>(1, (l + chunk_max - 1) / chunk_max);
            int want;
            if (prm.blocks_override > 0) want = prm.blocks_override;
            else want = (int)std::max<long long>(1, std::min<long long>(sms, (l + 1499) / 1500));
            if (count > 1) {
                const long long share = (long long)std::floor((double)capacity * (double)l / (double)std::max<long long>(total_l, 1));
                want = (int)std::min<long long>(want, std::max<long long>(1, share));
            }
            want = (int)std::min<long long>(want, std::max<long long>(1, l));
            nb[k] = std::max(want, nmin);
        }
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

        std::vector<InstanceAlloc> allocs(count);
        std::vector<InstanceDesc> desc(count);
        std::vector<int> block_inst(used);
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
            for (int b = 0; b < nb[k]; b++) block_inst[b0 + b] = k;
            b0 += nb[k];
            // cache geometry: rows of l floats, at least 4, at most 2l slots
            long long slots = (long long)std::floor(prm.cache_mb * (1 << 20) / (4.0 * std::max(l, 1)));
            slots = std::max<long long>(slots, 4);
            slots = std::min<long long>(slots, std::max<long long>(4, 2LL * l));
            const int ways = (int)std::min<long long>(kMaxWays, slots);
            const int sets = (int)(slots / ways);
            Bump bump;
            size_t oG = bump.take<double>(l), oGb = bump.take<double>(l), oA = bump.take<double>(l);
            size_t oP = bump.take<double>(l), oQD = bump.take<double>(l), oAl = bump.take<double>(l);
            size_t oY = bump.take<signed char>(l), oS = bump.take<unsigned char>(l);
            size_t oPL = bump.take<int>(l), oPR = bump.take<int>(l), oSc = bump.take<int>(2 * (size_t)l);
            size_t oOut = bump.take<SolveOut>(1), oSync = bump.take<GroupSync>(1);
            size_t oPart = bump.take<Partial>(2 * (size_t)nb[k]);
            size_t oTag = bump.take<int>((size_t)sets * ways), oEp = bump.take<int>((size_t)sets * ways);
            size_t oSt = bump.take<unsigned long long>((size_t)sets * ways);
            size_t oData = bump.take<float>((size_t)sets * ways * (size_t)l);
            char *base = nullptr;
            cudaError_t e = cudaMalloc(&base, bump.off);
            if (e != cudaSuccess) {
                for (int q = 0; q < k; q++) cudaFree(allocs[q].base);
                set_error(std::string("device allocation for solver state failed: ") + cudaGetErrorString(e));
                return -1;
            }
            allocs[k].base = base;
            allocs[k].bytes = bump.off;
            D.G = (double *)(base + oG);
            D.G_bar = (double *)(base + oGb);
            D.alpha = (double *)(base + oA);
            D.p = (double *)(base + oP);
            D.QD = (double *)(base + oQD);
            D.alpha_local = (double *)(base + oAl);
            D.y = (signed char *)(base + oY);
            D.status = (unsigned char *)(base + oS);
            D.pos_local = (int *)(base + oPL);
            D.pos_row = (int *)(base + oPR);
            D.scratch = (int *)(base + oSc);
            D.out = (SolveOut *)(base + oOut);
            D.sync = (GroupSync *)(base + oSync);
            D.partials = (Partial *)(base + oPart);
            D.cache.tag = (int *)(base + oTag);
            D.cache.epoch = (int *)(base + oEp);
            D.cache.stamp = (unsigned long long *)(base + oSt);
            D.cache.data = (float *)(base + oData);
            D.cache.nsets = sets;
            D.cache.nways = ways;
            D.cache.stride = l;
            // initial state
            std::vector<int> iota(l);
            for (int q = 0; q < l; q++) iota[q] = q;
            CK(xfer_async(D.alpha, sp.alpha0.data(), sizeof(double) * l, cudaMemcpyHostToDevice, s));
            CK(xfer_async(D.p, sp.p.data(), sizeof(double) * l, cudaMemcpyHostToDevice, s));
            CK(xfer_async(D.y, sp.y.data(), l, cudaMemcpyHostToDevice, s));
            CK(xfer_async(D.pos_local, iota.data(), sizeof(int) * l, cudaMemcpyHostToDevice, s));
            CK(xfer_async(D.pos_row, sp.rows.data(), sizeof(int) * l, cudaMemcpyHostToDevice, s));
            CK(cudaMemsetAsync(D.sync, 0, sizeof(GroupSync), s));
            CK(cudaMemsetAsync(D.partials, 0, sizeof(Partial) * 2 * (size_t)nb[k], s));
            CK(cudaMemsetAsync(D.cache.tag, 0xff, sizeof(int) * (size_t)sets * ways, s));
            CK(cudaMemsetAsync(D.cache.epoch, 0, sizeof(int) * (size_t)sets * ways, s));
            CK(cudaMemsetAsync(D.cache.stamp, 0, sizeof(unsigned long long) * (size_t)sets * ways, s));
        }
        InstanceDesc *d_desc = nullptr;
        int *d_block_inst = nullptr;
        CK(cudaMalloc(&d_desc, sizeof(InstanceDesc) * count));
        CK(cudaMalloc(&d_block_inst, sizeof(int) * used));
        CK(xfer_async(d_desc, desc.data(), sizeof(InstanceDesc) * count, cudaMemcpyHostToDevice, s));
        CK(xfer_async(d_block_inst, block_inst.data(), sizeof(int) * used, cudaMemcpyHostToDevice, s));
        cudaEvent_t ev0, ev1;
        CK(cudaEventCreate(&ev0));
        CK(cudaEventCreate(&ev1));
        CK(cudaEventRecord(ev0, s));
        cudaError_t le = launch_smo(prm.form, d_desc, d_block_inst, used, dyn_smem, true, s);
        if (le == cudaSuccess) count_launch();
        cudaEventRecord(ev1, s);
        cudaError_t se = le == cudaSuccess ? cudaStreamSynchronize(s) : le;
        float ms = 0;
        if (se == cudaSuccess) cudaEventElapsedTime(&ms, ev0, ev1);
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        int rc = 0;
        if (se != cudaSuccess) {
            set_error(std::string("solver launch failed: ") + cudaGetErrorString(se));
            rc = -1;
        }
        for (int k = 0; k < count && rc == 0; k++) {
            SolveResult &R = res[first + k];
            const int l = desc[k].l;
            R.alpha.resize(l);
            if (xfer(R.alpha.data(), desc[k].alpha_local, sizeof(double) * l, cudaMemcpyDeviceToHost) != cudaSuccess ||
                xfer(&R.out, desc[k].out, sizeof(SolveOut), cudaMemcpyDeviceToHost) != cudaSuccess) {
                set_error("copy of solver results failed");
                rc = -1;
                break;
            }
            R.seconds = ms * 1e-3;
            if (R.out.status < 0) {
                set_error("solver group barrier timed out");
                rc = -1;
            }
        }
        for (auto &a : allocs) cudaFree(a.base);
        cudaFree(d_desc);
        cudaFree(d_block_inst);
        if (rc) return rc;
        first = last;
    }
    return 0;
}

}  // namespace svmb
