// predict_kernel.cu -- decision values of the reference's svm_predict_values
// (reference libsvm/svm.cpp:2569-2643) for a batch of rows on the device.
//
// kvalue[t][s] = K(x_t, SV_s) with the prediction-time kernel of the reference
// (Kernel::k_function, svm.cpp:327-384: RBF walks the squared difference over
// the union of nonzero features in index order, no norm trick).  Each pair's
// sum runs sequentially over the two classes' SVs in model order, exactly as
// the reference, so decision values match it bit for bit (rows and SVs are
// kept as the doubles the caller's svm_node lists hold).
// The file is compiled with -fmad=false.
//
// Kernel values are kept SV-major, kv[s][t] for the t-th test row of a chunk,
// so that the pair sums (one thread per test row and pair, each walking the
// SVs in model order) read consecutive words across a warp.  Dense rows take
// a tiled kernel: a block computes 64 test rows x 64 SVs, 16 features at a
// time staged in shared memory, 4 x 4 values per thread.  With a
// tensor-core predict form the values come from the split-product kernel
// block of the SVs' split copy (kept with the model) and the chunk's.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "engine.hpp"
#include "predict.hpp"

namespace svmb {

namespace {

struct Rows {
    // dense [n][ld] or CSR, values in float64: a model's SVs (read from a
    // model file, say) and the caller's rows are doubles, and the exact form
    // evaluates the reference's kernel on exactly those values.  Each array
    // grows on demand and is reused by later uploads (capacities in bytes)
    double *X = nullptr;
    long long *rowptr = nullptr;
    int *col = nullptr;
    double *val = nullptr;
    size_t capX = 0, capRp = 0, capCol = 0, capVal = 0;
    int n = 0, ld = 0;
    bool dense = true;
    void release()
    {
        cudaFree(X); cudaFree(rowptr); cudaFree(col); cudaFree(val);
        X = nullptr; rowptr = nullptr; col = nullptr; val = nullptr;
        capX = capRp = capCol = capVal = 0;
    }
};

// device buffer of at least `bytes`, reallocated only when it must grow
template <typename T>
cudaError_t grow(T *&p, size_t &cap, size_t bytes)
{
    if (bytes <= cap && p) return cudaSuccess;
    cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
}

__device__ __forceinline__ double powi_p(double base, int times)
{
    double tmp = base, ret = 1.0;
    for (int t = times; t > 0; t /= 2) {
        if (t % 2 == 1) ret = __dmul_rn(ret, tmp);
        tmp = __dmul_rn(tmp, tmp);
    }
    return ret;
}

struct KP {
    int type, degree;
    double gamma, coef0;
};

// kvalue for rows given as CSR in global memory (merge walks, svm.cpp:305-384)
__device__ double kval_csr(const KP &kp, const long long *rpa, const int *ca, const double *va, int a,
                           const long long *rpb, const int *cb, const double *vb, int b)
{
    long long e = rpa[a], ee = rpa[a + 1], f = rpb[b], ff = rpb[b + 1];
    double sum = 0.0;
    if (kp.type == 2) {
        while (e < ee && f < ff) {
            const int x = ca[e], y = cb[f];
            if (x == y) {
                const double d = __dsub_rn(va[e], vb[f]);
                sum = __dadd_rn(sum, __dmul_rn(d, d));
                ++e; ++f;
            } else if (x > y) {
                sum = __dadd_rn(sum, __dmul_rn(vb[f], vb[f]));
                ++f;
            } else {
                sum = __dadd_rn(sum, __dmul_rn(va[e], va[e]));
                ++e;
            }
        }
        for (; e < ee; ++e) sum = __dadd_rn(sum, __dmul_rn(va[e], va[e]));
        for (; f < ff; ++f) sum = __dadd_rn(sum, __dmul_rn(vb[f], vb[f]));
        return exp(__dmul_rn(-kp.gamma, sum));
    }
    while (e < ee && f < ff) {
        const int x = ca[e], y = cb[f];
        if (x == y) { sum = __dadd_rn(sum, __dmul_rn(va[e], vb[f])); ++e; ++f; }
        else if (x > y) ++f;
        else ++e;
    }
    if (kp.type == 0) return sum;
    if (kp.type == 1) return powi_p(__dadd_rn(__dmul_rn(kp.gamma, sum), kp.coef0), kp.degree);
    return tanh(__dadd_rn(__dmul_rn(kp.gamma, sum), kp.coef0));
}

constexpr int kPT = 64;   // test rows per tile (dense path)
constexpr int kPS = 64;   // SVs per tile
constexpr int kPK = 16;   // features per staged slice

__device__ __forceinline__ double kfinish(const KP &kp, double acc)
{
    if (kp.type == 2) return exp(__dmul_rn(-kp.gamma, acc));
    if (kp.type == 0) return acc;
    if (kp.type == 1) return powi_p(__dadd_rn(__dmul_rn(kp.gamma, acc), kp.coef0), kp.degree);
    return tanh(__dadd_rn(__dmul_rn(kp.gamma, acc), kp.coef0));
}

// dense path: a 64 x 64 tile of K(test, SV), out[s][t] (ldo = nt).  Thread
// (ty, tx) of 16 x 16 owns test rows t0 + tx + 16i and SVs s0 + 4ty + j; every
// value accumulates over the features in order, as the reference's walk does
// (RBF: the squared difference; a feature zero in both adds nothing).
__global__ void __launch_bounds__(256) kvalue_tile(KP kp, const double *__restrict__ T, int nt,
                                                  const double *__restrict__ S, int ns, int ld,
                                                  double *__restrict__ out)
{
    __shared__ double ta[kPK][kPT + 1];
    __shared__ double sb[kPK][kPS + 1];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int t0 = blockIdx.y * kPT, s0 = blockIdx.x * kPS;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
    // loader: 64 rows x 16 features = 256 pieces of 4 doubles per operand, one per thread
    const int lr = tid >> 2, lc = (tid & 3) * 4;
    for (int k0 = 0; k0 < ld; k0 += kPK) {
        const int c = k0 + lc;
        double2 a0 = make_double2(0.0, 0.0), a1 = a0, b0 = a0, b1 = a0;
        if (t0 + lr < nt && c < ld) {
            const double2 *p = reinterpret_cast<const double2 *>(T + (long long)(t0 + lr) * ld + c);
            a0 = __ldg(p);
            a1 = __ldg(p + 1);
        }
        if (s0 + lr < ns && c < ld) {
            const double2 *p = reinterpret_cast<const double2 *>(S + (long long)(s0 + lr) * ld + c);
            b0 = __ldg(p);
            b1 = __ldg(p + 1);
        }
        __syncthreads();
        ta[lc][lr] = a0.x; ta[lc + 1][lr] = a0.y; ta[lc + 2][lr] = a1.x; ta[lc + 3][lr] = a1.y;
        sb[lc][lr] = b0.x; sb[lc + 1][lr] = b0.y; sb[lc + 2][lr] = b1.x; sb[lc + 3][lr] = b1.y;
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kPK; kk++) {
            double av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; i++) av[i] = ta[kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; j++) bv[j] = sb[kk][4 * ty + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    if (kp.type == 2) {
                        const double d = __dsub_rn(av[i], bv[j]);
                        acc[i][j] = __dadd_rn(acc[i][j], __dmul_rn(d, d));
                    } else {
                        acc[i][j] = __dadd_rn(acc[i][j], __dmul_rn(av[i], bv[j]));
                    }
                }
        }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int sv = s0 + 4 * ty + j;
        if (sv >= ns) continue;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int t = t0 + tx + 16 * i;
            if (t < nt) out[(long long)sv * nt + t] = kfinish(kp, acc[i][j]);
        }
    }
}

// sparse path: out[s][t] = K(test t, SV s) by merge walks, consecutive threads on consecutive test rows
__global__ void kvalue_csr(KP kp, Rows T, Rows S, double *__restrict__ out)
{
    const long long total = (long long)T.n * S.n;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total; id += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(id / T.n), t = (int)(id % T.n);
        out[id] = kval_csr(kp, T.rowptr, T.col, T.val, t, S.rowptr, S.col, S.val, s);
    }
}

// one thread per (test row, pair): sequential sums in model order (svm.cpp:2606-2631)
__global__ void pair_sums(const double *__restrict__ kv, int nt, int ns, int nr_class, const int *__restrict__ start,
                          const int *__restrict__ nsv, const double *__restrict__ coef, const double *__restrict__ rho,
                          double *__restrict__ dec)
{
    const int npair = nr_class * (nr_class - 1) / 2;
    const long long total = (long long)nt * npair;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total; id += (long long)gridDim.x * blockDim.x) {
        // consecutive threads on consecutive test rows of one pair
        const int p = (int)(id / nt);
        const int t = (int)(id % nt);
        // pair index -> (i,j)
        int i = 0, rem = p;
        while (rem >= nr_class - 1 - i) { rem -= nr_class - 1 - i; ++i; }
        const int j = i + 1 + rem;
        const double *k = kv + t;                // kv[s][t]: SV s of test row t at s * nt
        const double *coef1 = coef + (long long)(j - 1) * ns;
        const double *coef2 = coef + (long long)i * ns;
        double sum = 0;
        for (int q = 0; q < nsv[i]; q++)
            sum = __dadd_rn(sum, __dmul_rn(coef1[start[i] + q], k[(long long)(start[i] + q) * nt]));
        for (int q = 0; q < nsv[j]; q++)
            sum = __dadd_rn(sum, __dmul_rn(coef2[start[j] + q], k[(long long)(start[j] + q) * nt]));
        dec[(long long)t * npair + p] = __dsub_rn(sum, rho[p]);
    }
}

// Tensor forms: kv[t][s] row-major; one warp per (test row, pair), the lanes
// summing every 32nd SV of each class in model order and the lane sums
// combined by a fixed shuffle tree (the order is the same on every run; the
// exact form keeps the reference's sequential sums in pair_sums)
__global__ void pair_sums_rows(const double *__restrict__ kv, int nt, int ns, int nr_class, const int *__restrict__ start,
                               const int *__restrict__ nsv, const double *__restrict__ coef, const double *__restrict__ rho,
                               double *__restrict__ dec)
{
    const int npair = nr_class * (nr_class - 1) / 2;
    const long long total = (long long)nt * npair;
    const int lane = threadIdx.x & 31;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long id = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; id < total; id += warps) {
        const int t = (int)(id / npair), p = (int)(id % npair);
        int i = 0, rem = p;
        while (rem >= nr_class - 1 - i) { rem -= nr_class - 1 - i; ++i; }
        const int j = i + 1 + rem;
        const double *k = kv + (long long)t * ns;
        const double *coef1 = coef + (long long)(j - 1) * ns;
        const double *coef2 = coef + (long long)i * ns;
        double sum = 0;
        for (int q = lane; q < nsv[i]; q += 32) sum = __dadd_rn(sum, __dmul_rn(coef1[start[i] + q], k[start[i] + q]));
        for (int q = lane; q < nsv[j]; q += 32) sum = __dadd_rn(sum, __dmul_rn(coef2[start[j] + q], k[start[j] + q]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum = __dadd_rn(sum, __shfl_xor_sync(0xffffffffu, sum, o));
        if (lane == 0) dec[(long long)t * npair + p] = __dsub_rn(sum, rho[p]);
    }
}

struct Session {
    // fingerprint
    const svm_node *const *SV = nullptr;
    const double *coef0 = nullptr;
    int l = 0, nr_class = 0;
    double rho0 = 0;
    // device copy
    Rows sv;
    Rows sv_csr;                // CSR copy of dense SVs for the merge path (made on first need)
    std::unique_ptr<DeviceRows> sv_tc;   // the SVs in a tensor predict form (split copy), made on first need
    int d = 0, base = 1;
    double *coef = nullptr, *rho = nullptr;
    int *start = nullptr, *nsv = nullptr;
    void release()
    {
        sv.release();
        sv_csr.release();
        sv_tc.reset();
        cudaFree(coef); cudaFree(rho); cudaFree(start); cudaFree(nsv);
        coef = rho = nullptr;
        start = nsv = nullptr;
    }
};

std::mutex g_mu;
std::map<const svm_model *, std::unique_ptr<Session>> g_sessions;
int g_predict_form = FORM_EXACT;

// Per-process prediction buffers, grown on demand and kept (a loop of
// single-row svm_predict calls allocates nothing after its first call).
struct Workspace {
    double *kv = nullptr, *dec = nullptr;
    int *err = nullptr;
    size_t cap_kv = 0, cap_dec = 0, cap_err = 0;
    Rows T;                     // test rows of the current chunk
} g_ws;

#define PK(call)                                                                  \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) {                                                  \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));        \
            return -1;                                                            \
        }                                                                         \
    } while (0)

int upload_nodes(const svm_node *const *x, int n, int d, int base, bool dense, Rows &out)
{
    out.n = n;
    out.dense = dense;
    out.ld = (d + 3) & ~3;
    if (out.ld == 0) out.ld = 4;
    if (dense) {
        std::vector<double> h((size_t)std::max(n, 1) * out.ld, 0.0);
#pragma omp parallel for schedule(static)
        for (int r = 0; r < n; r++)
            for (const svm_node *p = x[r]; p->index != -1; ++p) {
                const int c = p->index - base;
                if (c >= 0 && c < out.ld) h[(size_t)r * out.ld + c] = p->value;
            }
        PK(grow(out.X, out.capX, h.size() * sizeof(double)));
        PK(xfer(out.X, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    } else {
        std::vector<long long> rp((size_t)n + 1, 0);
#pragma omp parallel for schedule(static)
        for (int r = 0; r < n; r++) {
            long long c = 0;
            for (const svm_node *p = x[r]; p->index != -1; ++p) c++;
            rp[(size_t)r + 1] = c;
        }
        for (int r = 0; r < n; r++) rp[(size_t)r + 1] += rp[r];
        std::vector<int> col((size_t)std::max<long long>(rp[n], 1), 0);
        std::vector<double> val(col.size(), 0.0);
#pragma omp parallel for schedule(static)
        for (int r = 0; r < n; r++) {
            long long k = rp[r];
            for (const svm_node *p = x[r]; p->index != -1; ++p, ++k) {
                col[k] = p->index - base;
                val[k] = p->value;
            }
        }
        PK(grow(out.rowptr, out.capRp, rp.size() * sizeof(long long)));
        PK(grow(out.col, out.capCol, col.size() * sizeof(int)));
        PK(grow(out.val, out.capVal, val.size() * sizeof(double)));
        PK(xfer(out.rowptr, rp.data(), rp.size() * sizeof(long long), cudaMemcpyHostToDevice));
        PK(xfer(out.col, col.data(), col.size() * sizeof(int), cudaMemcpyHostToDevice));
        PK(xfer(out.val, val.data(), val.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    return 0;
}

Session *get_session(const svm_model *m)
{
    auto it = g_sessions.find(m);
    if (it != g_sessions.end()) {
        Session *s = it->second.get();
        if (s->SV == m->SV && s->l == m->l && s->nr_class == m->nr_class &&
            s->coef0 == (m->nr_class > 1 ? m->sv_coef[0] : nullptr) && s->rho0 == (m->nr_class > 1 ? m->rho[0] : 0.0))
            return s;
        s->release();
        g_sessions.erase(it);
    }
    std::unique_ptr<Session> s(new Session());
    s->SV = m->SV;
    s->l = m->l;
    s->nr_class = m->nr_class;
    s->coef0 = m->nr_class > 1 ? m->sv_coef[0] : nullptr;
    s->rho0 = m->nr_class > 1 ? m->rho[0] : 0.0;
    int maxi = 0;
    long long nnz = 0;
    for (int i = 0; i < m->l; i++)
        for (const svm_node *p = m->SV[i]; p->index != -1; ++p) { maxi = std::max(maxi, p->index); nnz++; }
    s->base = 0;
    s->d = maxi + 1;
    const bool dense = m->l == 0 || (double)nnz >= 0.25 * (double)m->l * s->d || (double)m->l * s->d * 4 < 32e6;
    if (upload_nodes(m->SV, m->l, s->d, s->base, dense, s->sv) != 0) return nullptr;
    const int k = m->nr_class, npair = k * (k - 1) / 2;
    std::vector<double> coef((size_t)std::max(k - 1, 1) * std::max(m->l, 1), 0.0);
    for (int j = 0; j < k - 1; j++)
        for (int i = 0; i < m->l; i++) coef[(size_t)j * m->l + i] = m->sv_coef[j][i];
    std::vector<int> start(std::max(k, 1), 0), nsv(std::max(k, 1), 0);
    // one-class and SVR models have no classes: all SVs form one group and
    // the value is the single "pair" sum over it (svm.cpp:2571-2587)
    for (int i = 0; i < k; i++) nsv[i] = m->nSV ? m->nSV[i] : (i == 0 ? m->l : 0);
    for (int i = 1; i < k; i++) start[i] = start[i - 1] + nsv[i - 1];
    std::vector<double> rho(std::max(npair, 1), 0.0);
    for (int p = 0; p < npair; p++) rho[p] = m->rho[p];
    if (cudaMalloc(&s->coef, coef.size() * 8) != cudaSuccess || cudaMalloc(&s->rho, rho.size() * 8) != cudaSuccess ||
        cudaMalloc(&s->start, start.size() * 4) != cudaSuccess || cudaMalloc(&s->nsv, nsv.size() * 4) != cudaSuccess) {
        set_error("device allocation for prediction failed");
        s->release();
        return nullptr;
    }
    xfer(s->coef, coef.data(), coef.size() * 8, cudaMemcpyHostToDevice);
    xfer(s->rho, rho.data(), rho.size() * 8, cudaMemcpyHostToDevice);
    xfer(s->start, start.data(), start.size() * 4, cudaMemcpyHostToDevice);
    xfer(s->nsv, nsv.data(), nsv.size() * 4, cudaMemcpyHostToDevice);
    Session *raw = s.get();
    g_sessions[m] = std::move(s);
    return raw;
}

// rows as host CSR (0-based columns) of width d
int rows_to_device(const svm_node *const *x, int n, int d, int form, DeviceRows &out)
{
    // CSR of the rows (columns = libsvm indices), counted and filled in
    // parallel over rows
    std::vector<long long> rp((size_t)n + 1, 0);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n; r++) {
        long long c = 0;
        for (const svm_node *p = x[r]; p->index != -1; ++p) c++;
        rp[(size_t)r + 1] = c;
    }
    for (int r = 0; r < n; r++) rp[(size_t)r + 1] += rp[r];
    std::vector<int> col((size_t)std::max<long long>(rp[n], 1), 0);
    std::vector<float> val(col.size(), 0.0f);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n; r++) {
        long long k = rp[r];
        for (const svm_node *p = x[r]; p->index != -1; ++p, ++k) {
            col[k] = p->index;
            val[k] = (float)p->value;
        }
    }
    if (upload_csr(rp.data(), col.data(), val.data(), n, d, out, -1, 0) != 0) return -1;
    return out.prepare_form(form, 0);
}

// The SVs' split (or tf32) copy for tensor-core kernel values, made once per
// model, form and width: both row sets of the block product need the same
// split width, and test rows wider than the SVs widen it (their extra
// features still count in the RBF norms).
int prepare_tensor_svs(const svm_model *m, Session *s, int width, int form)
{
    width = std::max(width, s->d);
    if (s->sv_tc && s->sv_tc->split_form == form && s->sv_tc->d >= width) return 0;
    s->sv_tc.reset(new DeviceRows());
    if (rows_to_device(m->SV, m->l, width, form, *s->sv_tc) != 0) {
        s->sv_tc.reset();
        return -1;
    }
    return 0;
}

}  // namespace

int predict_set_form(int form)
{
    if (form != FORM_EXACT && !is_tc_form(form)) return -1;
    std::lock_guard<std::mutex> g(g_mu);
    g_predict_form = form;
    return 0;
}

void predict_forget(const svm_model *model)
{
    std::lock_guard<std::mutex> g(g_mu);
    auto it = g_sessions.find(model);
    if (it != g_sessions.end()) {
        it->second->release();
        g_sessions.erase(it);
    }
}

int predict_batch(const svm_model *m, const svm_node *const *rows, int n, double *labels, double *dec_out)
{
    const int type = m->param.svm_type;
    if (type < C_SVC || type > NU_SVR) {
        set_error("unknown svm_type in the model");
        return -1;
    }
    if (m->param.kernel_type == PRECOMPUTED) {
        set_error("precomputed kernels are not supported on the GPU");
        return -1;
    }
    const bool classify = type == C_SVC || type == NU_SVC;
    std::lock_guard<std::mutex> g(g_mu);
    Session *s = get_session(m);
    if (!s) return -1;
    const int k = m->nr_class, npair = k * (k - 1) / 2;
    if (n == 0) return 0;
    KP kp{m->param.kernel_type, m->param.degree, m->param.gamma, m->param.coef0};
    std::vector<double> dec((size_t)n * std::max(npair, 1), 0.0);
    if (npair > 0 && m->l > 0) {
        // the test rows go to the device once; kernel values are made in
        // chunks of rows whose value block stays below a quarter of the free
        // device memory (at most 4 GB)
        const bool trace = getenv("SVMB_TRACE") && *getenv("SVMB_TRACE") == '1';
        const auto c0 = std::chrono::steady_clock::now();
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 1ull << 32;
        const long long per_row = (long long)m->l * 8;
        const long long budget = std::min<long long>(4LL << 30, std::max<long long>((long long)free_b / 4, 64LL << 20));
        const int chunk = (int)std::max<long long>(1, std::min<long long>(n, budget / per_row));
        PK(grow(g_ws.kv, g_ws.cap_kv, (size_t)chunk * per_row));
        PK(grow(g_ws.dec, g_ws.cap_dec, (size_t)chunk * npair * 8));
        double *kv = g_ws.kv, *d_dec = g_ws.dec;
        // test rows: features beyond the SVs' width cannot meet an SV feature in a
        // dot product but still count in the RBF distance, so widen to cover them
        int maxi = s->d - 1;
#pragma omp parallel for schedule(static) reduction(max : maxi)
        for (int r = 0; r < n; r++)
            for (const svm_node *p = rows[r]; p->index != -1; ++p) maxi = std::max(maxi, p->index);
        const bool wider = maxi + 1 > s->d;
        const bool tensor = is_tc_form(g_predict_form);
        const bool dense = !tensor && s->sv.dense && !wider;
        Rows &T = g_ws.T;
        DeviceRows Ttc;
        if (tensor) {
            if (prepare_tensor_svs(m, s, maxi + 1, g_predict_form) != 0) return -1;
            if (rows_to_device(rows, n, s->sv_tc->d, g_predict_form, Ttc) != 0) return -1;
        } else if (dense) {
            if (upload_nodes(rows, n, s->d, s->base, true, T) != 0) return -1;
        } else {
            if (s->sv.dense && !s->sv_csr.rowptr && upload_nodes(m->SV, m->l, s->d, s->base, false, s->sv_csr) != 0)
                return -1;
            if (upload_nodes(rows, n, maxi + 1, s->base, false, T) != 0) return -1;
        }
        int *d_err = nullptr;
        if (tensor) {
            PK(grow(g_ws.err, g_ws.cap_err, sizeof(int)));
            d_err = g_ws.err;
            PK(cudaMemset(d_err, 0, sizeof(int)));
        }
        const auto c1 = std::chrono::steady_clock::now();
        KernelParams kpk{m->param.kernel_type, m->param.degree, m->param.gamma, m->param.coef0};
        for (int t0 = 0; t0 < n; t0 += chunk) {
            const int tn = std::min(chunk, n - t0);
            if (tensor) {
                PK(launch_kernel_block2(Ttc, *s->sv_tc, kpk, g_predict_form, t0, tn, m->l, kv, m->l, 0, d_err, 0));
            } else if (dense) {
                dim3 grid((m->l + kPS - 1) / kPS, (tn + kPT - 1) / kPT);
                kvalue_tile<<<grid, 256>>>(kp, T.X + (long long)t0 * T.ld, tn, s->sv.X, m->l, s->sv.ld, kv);
                count_launch();
            } else {
                const Rows &Sc = s->sv.dense ? s->sv_csr : s->sv;
                Rows Tc = T;               // a view of rows t0 .. t0+tn (row pointers stay absolute)
                Tc.rowptr = T.rowptr + t0;
                Tc.n = tn;
                kvalue_csr<<<(int)std::min<long long>(((long long)tn * m->l + 255) / 256, 148 * 16), 256>>>(kp, Tc, Sc, kv);
                count_launch();
            }
            if (tensor)
                pair_sums_rows<<<(int)std::min<long long>(((long long)tn * npair * 32 + 255) / 256, 148 * 16), 256>>>(
                    kv, tn, m->l, k, s->start, s->nsv, s->coef, s->rho, d_dec);
            else
                pair_sums<<<std::min<long long>(((long long)tn * npair + 127) / 128, 148 * 8), 128>>>(kv, tn, m->l, k, s->start, s->nsv, s->coef, s->rho, d_dec);
            count_launch();
            cudaError_t e = cudaDeviceSynchronize();
            if (e != cudaSuccess) {
                set_error(std::string("prediction kernels failed: ") + cudaGetErrorString(e));
                return -1;
            }
            PK(xfer(dec.data() + (size_t)t0 * npair, d_dec, (size_t)tn * npair * 8, cudaMemcpyDeviceToHost));
        }
        if (tensor) {
            int herr = 0;
            PK(xfer(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost));
            if (herr) {
                set_error("tensor-core kernel values: a wait timed out");
                return -1;
            }
        }
        if (trace) {
            const auto c2 = std::chrono::steady_clock::now();
            auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
                return std::chrono::duration<double, std::milli>(b - a).count();
            };
            fprintf(stderr, "[svmb] predict rows=%d svs=%d chunks=%d rows_to_device=%.2fms values+sums=%.2fms\n", n,
                    m->l, (n + chunk - 1) / chunk, ms(c0, c1), ms(c1, c2));
        }
    } else if (npair > 0) {
        for (int t = 0; t < n; t++)
            for (int p = 0; p < npair; p++) dec[(size_t)t * npair + p] = -m->rho[p];
    }
    for (int t = 0; t < n; t++) {
        if (!classify) {
            // one-class: the side of the boundary; SVR: the value (svm.cpp:2585-2587)
            const double v = dec[t];
            labels[t] = type == ONE_CLASS ? (v > 0 ? 1 : -1) : v;
            if (dec_out) dec_out[t] = v;
            continue;
        }
        // votes, ties to the lowest class index (svm.cpp:2627-2637)
        std::vector<int> vote(std::max(k, 1), 0);
        int p = 0;
        for (int i = 0; i < k; i++)
            for (int j = i + 1; j < k; j++) {
                if (dec[(size_t)t * npair + p] > 0) ++vote[i];
                else ++vote[j];
                p++;
            }
        int best = 0;
        for (int i = 1; i < k; i++)
            if (vote[i] > vote[best]) best = i;
        labels[t] = m->label ? m->label[best] : 0;
        if (dec_out)
            for (int q = 0; q < npair; q++) dec_out[(size_t)t * npair + q] = dec[(size_t)t * npair + q];
    }
    return 0;
}

}  // namespace svmb
