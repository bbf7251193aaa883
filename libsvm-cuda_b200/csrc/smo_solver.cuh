// smo_solver.cuh -- device-resident SMO solver for C-SVC and nu-SVC (device code).
//
// One persistent launch runs the whole solve of one or more instances (each a
// binary subproblem).  Every instance is owned by a group of `nblocks` thread
// blocks; block `rank` of the group owns a contiguous chunk of the active
// positions [0, A) and a chunk of the inactive tail [A, l).  The state of its
// active chunk (G, alpha, QD, label, bound status, cache column, row id) lives
// in the block's shared memory between shrink events.  Per SMO iteration there
// are exactly two group exchanges:
//
//   phase A  reduce the per-block I_up maxima -> working index i (nu-SVC: the
//            two track maxima ip/in), look up or evaluate the Q row(s) on the
//            block's chunk, scan the chunk for the second-order j candidate
//            (WSS3, reference svm.cpp:833-930 / :1076-1186)
//   --- exchange ---
//   phase B  reduce the j candidates, stopping test, look up or evaluate Q_j,
//            two-variable analytic step with box clipping (svm.cpp:636-721,
//            computed redundantly and identically by every block), gradient
//            update G += dQ (svm.cpp:729-735) and G_bar update (:744-769) on the
//            block's chunk, fused with the I_up scan for the next i
//   --- exchange ---
//
// An exchange publishes a 128-byte record per block whose last field is a
// sequence number written with release semantics; every block polls all
// records with acquire loads.  The exchange is therefore also the group
// barrier.  Records alternate between two buffers.
//
// Shrinking (svm.cpp:932-1011), gradient reconstruction (:473-513) and the
// initial gradient (:545-572) run inside the same launch as group-collective
// sections on the global copies of the state.  The position permutation of
// shrinking is the reference's (each shrunk position below the new active
// size is swapped with the highest kept position above it), so the
// position-based tie-breaks are identical.  All double arithmetic keeps the
// reference's operand order; the file is compiled with -fmad=false so that no
// multiply-add is contracted.
//
// Every wait is bounded: a poll that exceeds the instance's wait bound (30 s
// unless the host sets another) sets the group's error flag and every block
// of the group returns.
//
// The kernel template smo_persistent<FORM> is instantiated once per
// arithmetic form, each in its own translation unit (smo_form_*.cu), so the
// forms compile in parallel; the launchers are in smo_kernel.cu.
#pragma once
#include "engine.h"
#include "kernel_math.cuh"
#include "tc_sm100.cuh"

#include <cuda_runtime.h>

#include <type_traits>

namespace svmb {
// internal linkage: every form's translation unit has its own copy
namespace {


#define SVMB_INF __longlong_as_double(0x7ff0000000000000ULL)
constexpr double kTau = 1e-12;                     // reference svm.cpp:42
constexpr long long kWaitTimeoutNs = 30000000000LL;  // default bound of a cross-block wait: 30 s
// positions a thread takes at a time in the chunk scans that read Q rows from
// global memory: their loads are issued together
constexpr int kScanGroup = 8;

// --------------------------------------------------------------------------
// memory-model helpers
// --------------------------------------------------------------------------
__device__ __forceinline__ int ld_acquire_i32(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_i32(int *p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_relaxed_i32(const int *p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// --------------------------------------------------------------------------
// source-row staging and the row-block product
// --------------------------------------------------------------------------
// Sources of a row-block product are staged in dynamic shared memory when the
// instance's stage_cap > 0 (dense rows copied; sparse rows scattered into
// zeroed dense vectors), otherwise read from global memory (dense) or merged
// against the target's CSR row (sparse).  `sp[k]` points at source k.
// The exact form stages its sources as float64 (`dbl`): a float -> double
// conversion per use would otherwise outnumber the float64 multiply-adds
// (conversions issue at a quarter of their rate), and the value is the same.
struct StageSlots {
    const void *sp[kSrcBatch];
    int rows[kSrcBatch];
    int ns;
    int dbl;
    // column-keyed table of wide sparse sources (hash_slots > 0): keys, the
    // values [slot][kSrcBatch], and the sources' nonzeros flattened
    // (source k owns [hoff[k], hoff[k+1])); hash = 0 when this pass's sources
    // did not fit and merge walks are used instead
    int hash;
    int hoff[kSrcBatch + 1];
    int *hkeys;
    void *hvals;
};
// staged nonzeros a thread handles at most (a pass holds up to kHashSlots / 2)
constexpr int kHashPer = (kHashSlots / 2 + kThreads - 1) / kThreads;

__device__ __forceinline__ int hash_home(int col) { return (int)(((unsigned)col * 2654435761u) >> 22) & (kHashSlots - 1); }

// the table slot holding column `col`, or -1
__device__ __forceinline__ int hash_find(const int *keys, int col)
{
    int h = hash_home(col);
    while (true) {
        const int k = keys[h];
        if (k == col) return h;
        if (k < 0) return -1;
        h = (h + 1) & (kHashSlots - 1);
    }
}

// which source owns flattened nonzero t (hoff ascending, ns <= kSrcBatch)
__device__ __forceinline__ int hash_owner(const StageSlots &ss, int t)
{
    int k = 0;
    while (k + 1 < ss.ns && t >= ss.hoff[k + 1]) ++k;
    return k;
}

// bytes of one staged value in the form
__host__ __device__ constexpr int stage_elem(int form) { return form == FORM_EXACT ? 8 : 4; }

__device__ void stage_sources(const InstanceDesc &D, float *stage, StageSlots &ss, const int *rows, int ns)
{
    const DevX &x = D.x;
    const bool dbl = D.form == FORM_EXACT && D.stage_cap > 0;
    double *stage_d = reinterpret_cast<double *>(stage);
    if (threadIdx.x < ns) ss.rows[threadIdx.x] = rows[threadIdx.x];
    if (threadIdx.x == 0) {
        ss.ns = ns;
        ss.dbl = dbl ? 1 : 0;
        ss.hash = 0;
    }
    if (x.X) {
        // all sources in one pass: thread e moves 16 bytes of source e / ld4
        const int ld4 = x.ld >> 2;
        if (D.stage_cap > 0) {
            const int total = ns * ld4;
            for (int e = threadIdx.x; e < total; e += blockDim.x) {
                const int k = e / ld4, t = e - k * ld4;
                const float4 v = __ldg(reinterpret_cast<const float4 *>(x.X + (long long)rows[k] * x.ld) + t);
                if (dbl) {
                    double2 *dst = reinterpret_cast<double2 *>(stage_d + (long long)k * D.stage_lds);
                    dst[2 * t] = make_double2((double)v.x, (double)v.y);
                    dst[2 * t + 1] = make_double2((double)v.z, (double)v.w);
                } else {
                    reinterpret_cast<float4 *>(stage + (long long)k * D.stage_lds)[t] = v;
                }
            }
        }
        if (threadIdx.x < ns) {
            const int k = threadIdx.x;
            if (dbl) ss.sp[k] = stage_d + (long long)k * D.stage_lds;
            else if (D.stage_cap > 0) ss.sp[k] = stage + (long long)k * D.stage_lds;
            else ss.sp[k] = x.X + (long long)rows[k] * x.ld;
        }
    } else if (D.hash_slots > 0) {
        // wide sparse sources: every nonzero (column c of source k) goes to the
        // slot of c in the table; a slot shared by several sources holds each
        // one's value, the others stay zero
        if (threadIdx.x == 0) {
            int tot = 0;
            ss.hoff[0] = 0;
            for (int k = 0; k < ns; k++) {
                tot += (int)(x.rowptr[rows[k] + 1] - x.rowptr[rows[k]]);
                ss.hoff[k + 1] = tot;
            }
            ss.hash = tot <= kHashSlots / 2 ? 1 : 0;
            ss.hkeys = reinterpret_cast<int *>(stage);
            ss.hvals = reinterpret_cast<char *>(stage) + kHashSlots * 4;
            ss.dbl = D.form == FORM_EXACT ? 1 : 0;
        }
        __syncthreads();
        for (int t = threadIdx.x; ss.hash && t < ss.hoff[ns]; t += blockDim.x) {
            const int k = hash_owner(ss, t);
            const long long e = x.rowptr[rows[k]] + (t - ss.hoff[k]);
            const int col = x.col[e];
            const float v = x.val[e];
            int h = hash_home(col);
            while (true) {
                const int prev = atomicCAS(&ss.hkeys[h], -1, col);
                if (prev == -1 || prev == col) break;
                h = (h + 1) & (kHashSlots - 1);
            }
            if (D.form == FORM_EXACT) reinterpret_cast<double *>(ss.hvals)[h * kSrcBatch + k] = (double)v;
            else reinterpret_cast<float *>(ss.hvals)[h * kSrcBatch + k] = v;
        }
    } else if (D.stage_cap > 0) {
        for (int k = 0; k < ns; k++) {
            const long long a = x.rowptr[rows[k]], b = x.rowptr[rows[k] + 1];
            if (dbl) {
                double *dst = stage_d + (long long)k * D.stage_lds;
                for (long long e = a + threadIdx.x; e < b; e += blockDim.x) dst[x.col[e]] = (double)x.val[e];
                if (threadIdx.x == 0) ss.sp[k] = dst;
            } else {
                float *dst = stage + (long long)k * D.stage_lds;
                for (long long e = a + threadIdx.x; e < b; e += blockDim.x) dst[x.col[e]] = x.val[e];
                if (threadIdx.x == 0) ss.sp[k] = dst;
            }
        }
    }
    __syncthreads();
}

// Undo a sparse scatter so that the dense vectors are all-zero again.
__device__ void unstage_sources(const InstanceDesc &D, float *stage, StageSlots &ss)
{
    __syncthreads();
    const DevX &x = D.x;
    if (!x.X && D.hash_slots > 0) {
        // every slot this pass filled goes back to empty with zero values: the
        // slots are found first and cleared after a barrier, so that no
        // lookup meets a chain with a hole
        int h[kHashPer], k[kHashPer];
#pragma unroll
        for (int u = 0; u < kHashPer; u++) {
            const int t = threadIdx.x + u * (int)blockDim.x;
            h[u] = -1;
            k[u] = 0;
            if (ss.hash && t < ss.hoff[ss.ns]) {
                k[u] = hash_owner(ss, t);
                h[u] = hash_find(ss.hkeys, x.col[x.rowptr[ss.rows[k[u]]] + (t - ss.hoff[k[u]])]);
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < kHashPer; u++) {
            if (h[u] < 0) continue;
            ss.hkeys[h[u]] = -1;
            if (ss.dbl) reinterpret_cast<double *>(ss.hvals)[h[u] * kSrcBatch + k[u]] = 0.0;
            else reinterpret_cast<float *>(ss.hvals)[h[u] * kSrcBatch + k[u]] = 0.0f;
        }
    } else if (!x.X && D.stage_cap > 0) {
        for (int k = 0; k < ss.ns; k++) {
            const long long a = x.rowptr[ss.rows[k]], b = x.rowptr[ss.rows[k] + 1];
            if (ss.dbl) {
                double *dst = reinterpret_cast<double *>(stage) + (long long)k * D.stage_lds;
                for (long long e = a + threadIdx.x; e < b; e += blockDim.x) dst[x.col[e]] = 0.0;
            } else {
                float *dst = stage + (long long)k * D.stage_lds;
                for (long long e = a + threadIdx.x; e < b; e += blockDim.x) dst[x.col[e]] = 0.0f;
            }
        }
    }
    __syncthreads();
}

template <int FORM>
struct Acc {
    typedef typename std::conditional<FORM == FORM_EXACT, double, float>::type type;
};

template <int FORM>
__device__ __forceinline__ typename Acc<FORM>::type mac(float a, float b, typename Acc<FORM>::type acc)
{
    if (FORM == FORM_EXACT) return fma((double)a, (double)b, (double)acc);
    return fmaf(a, b, (float)acc);
}
// a source staged as float64 (exact form): only the target value is converted
template <int FORM>
__device__ __forceinline__ typename Acc<FORM>::type mac(float a, double b, typename Acc<FORM>::type acc)
{
    return fma((double)a, b, (double)acc);
}

// four staged source values starting at feature 4*i: float4 or two double2
__device__ __forceinline__ float4 src4(const float *p, int i) { return reinterpret_cast<const float4 *>(p)[i]; }
struct D4 { double x, y, z, w; };
__device__ __forceinline__ D4 src4(const double *p, int i)
{
    const double2 a = reinterpret_cast<const double2 *>(p)[2 * i], b = reinterpret_cast<const double2 *>(p)[2 * i + 1];
    return D4{a.x, a.y, b.x, b.y};
}

// Dot products of target row `r` with NS staged sources, accumulated in
// feature order (the order of the reference's Kernel::dot, svm.cpp:305-325:
// only matching indices contribute; zero products leave the sum unchanged).
// Dense rows are streamed 8 x 16 bytes at a time per thread.
template <int FORM, int NS, typename S>
__device__ __forceinline__ void row_dots_n(const InstanceDesc &D, const StageSlots &ss, int ns, int r,
                                           double (&out)[kSrcBatch])
{
    const DevX &x = D.x;
    typedef typename Acc<FORM>::type acc_t;
    acc_t acc[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) acc[k] = acc_t(0);
    if (x.X) {
        const float4 *row = reinterpret_cast<const float4 *>(x.X + (long long)r * x.ld);
        const S *src[NS];
#pragma unroll
        for (int k = 0; k < NS; k++) src[k] = reinterpret_cast<const S *>(ss.sp[k < ns ? k : 0]);
        const int ld4 = x.ld >> 2;
        int c = 0;
        for (; c + 8 <= ld4; c += 8) {
            float4 v[8];
#pragma unroll
            for (int u = 0; u < 8; u++) v[u] = __ldg(row + c + u);
#pragma unroll
            for (int u = 0; u < 8; u++) {
#pragma unroll
                for (int k = 0; k < NS; k++) {
                    if (NS == kSrcBatch && k >= ns) continue;
                    const auto w = src4(src[k], c + u);
                    acc[k] = mac<FORM>(v[u].x, w.x, acc[k]);
                    acc[k] = mac<FORM>(v[u].y, w.y, acc[k]);
                    acc[k] = mac<FORM>(v[u].z, w.z, acc[k]);
                    acc[k] = mac<FORM>(v[u].w, w.w, acc[k]);
                }
            }
        }
        for (; c < ld4; c++) {
            const float4 v = __ldg(row + c);
#pragma unroll
            for (int k = 0; k < NS; k++) {
                if (NS == kSrcBatch && k >= ns) continue;
                const auto w = src4(src[k], c);
                acc[k] = mac<FORM>(v.x, w.x, acc[k]);
                acc[k] = mac<FORM>(v.y, w.y, acc[k]);
                acc[k] = mac<FORM>(v.z, w.z, acc[k]);
                acc[k] = mac<FORM>(v.w, w.w, acc[k]);
            }
        }
    } else if (D.stage_cap > 0) {
        const long long a = x.rowptr[r], b = x.rowptr[r + 1];
        long long e = a;
        for (; e + 4 <= b; e += 4) {
            int cc[4];
            float vv[4];
#pragma unroll
            for (int u = 0; u < 4; u++) { cc[u] = __ldg(x.col + e + u); vv[u] = __ldg(x.val + e + u); }
#pragma unroll
            for (int u = 0; u < 4; u++) {
#pragma unroll
                for (int k = 0; k < NS; k++) {
                    if (NS == kSrcBatch && k >= ns) continue;
                    acc[k] = mac<FORM>(vv[u], reinterpret_cast<const S *>(ss.sp[k])[cc[u]], acc[k]);
                }
            }
        }
        for (; e < b; e++) {
            const int cc = __ldg(x.col + e);
            const float vv = __ldg(x.val + e);
#pragma unroll
            for (int k = 0; k < NS; k++) {
                if (NS == kSrcBatch && k >= ns) continue;
                acc[k] = mac<FORM>(vv, reinterpret_cast<const S *>(ss.sp[k])[cc], acc[k]);
            }
        }
    } else if (ss.hash) {
        // the target's nonzeros in column order, each looked up in the
        // sources' table: only matching columns contribute, in the order of
        // the reference's merge (svm.cpp:305-325)
        const long long a = x.rowptr[r], b = x.rowptr[r + 1];
        const int *keys = ss.hkeys;
        const S *vals = reinterpret_cast<const S *>(ss.hvals);
        long long e = a;
        for (; e + 4 <= b; e += 4) {
            int cc[4];
            float vv[4];
#pragma unroll
            for (int u = 0; u < 4; u++) { cc[u] = __ldg(x.col + e + u); vv[u] = __ldg(x.val + e + u); }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int h = hash_find(keys, cc[u]);
                if (h < 0) continue;
#pragma unroll
                for (int k = 0; k < NS; k++) {
                    if (NS == kSrcBatch && k >= ns) continue;
                    acc[k] = mac<FORM>(vv[u], vals[h * kSrcBatch + k], acc[k]);
                }
            }
        }
        for (; e < b; e++) {
            const int h = hash_find(keys, __ldg(x.col + e));
            if (h < 0) continue;
            const float vv = __ldg(x.val + e);
#pragma unroll
            for (int k = 0; k < NS; k++) {
                if (NS == kSrcBatch && k >= ns) continue;
                acc[k] = mac<FORM>(vv, vals[h * kSrcBatch + k], acc[k]);
            }
        }
    } else {
        // merge walk of two sorted index lists in global memory
        const long long a = x.rowptr[r], b = x.rowptr[r + 1];
#pragma unroll
        for (int k = 0; k < NS; k++) {
            if (k >= ns) continue;
            const long long sa = x.rowptr[ss.rows[k]], sb = x.rowptr[ss.rows[k] + 1];
            long long e = a, f = sa;
            acc_t s = acc_t(0);
            while (e < b && f < sb) {
                const int ce = __ldg(x.col + e), cf = __ldg(x.col + f);
                if (ce == cf) {
                    s = mac<FORM>(__ldg(x.val + e), __ldg(x.val + f), s);
                    ++e;
                    ++f;
                } else if (ce > cf) {
                    ++f;
                } else {
                    ++e;
                }
            }
            acc[k] = s;
        }
    }
#pragma unroll
    for (int k = 0; k < NS; k++) out[k] = (double)acc[k];
}

template <int FORM>
__device__ __forceinline__ void row_dots(const InstanceDesc &D, const StageSlots &ss, int ns, int r,
                                         double (&out)[kSrcBatch])
{
    if (FORM == FORM_EXACT && ss.dbl) {
        if (ns == 1) row_dots_n<FORM, 1, double>(D, ss, ns, r, out);
        else if (ns == 2) row_dots_n<FORM, 2, double>(D, ss, ns, r, out);
        else row_dots_n<FORM, kSrcBatch, double>(D, ss, ns, r, out);
    } else {
        if (ns == 1) row_dots_n<FORM, 1, float>(D, ss, ns, r, out);
        else if (ns == 2) row_dots_n<FORM, 2, float>(D, ss, ns, r, out);
        else row_dots_n<FORM, kSrcBatch, float>(D, ss, ns, r, out);
    }
}

// --------------------------------------------------------------------------
// block reductions with the reference's tie rules
// --------------------------------------------------------------------------
// argmax, ties -> larger index ("if (v >= best)" scanning upward, svm.cpp:851,860)
__device__ __forceinline__ void better_max(double &v, int &i, double v2, int i2)
{
    if (v2 > v || (v2 == v && i2 > i)) { v = v2; i = i2; }
}
// argmin, ties -> larger index ("if (obj_diff <= obj_diff_min)", svm.cpp:890,914)
__device__ __forceinline__ void better_min(double &v, int &i, double v2, int i2)
{
    if (v2 < v || (v2 == v && i2 > i)) { v = v2; i = i2; }
}

__device__ __forceinline__ void warp_argmax(double &v, int &i)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
        better_max(v, i, v2, i2);
    }
}
__device__ __forceinline__ void warp_argmin(double &v, int &i)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
        better_min(v, i, v2, i2);
    }
}
__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_sum_i(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct RedScratch {
    double v[4][kWarps];
    int i[4][kWarps];
};

// Reduce up to 4 (value,index) pairs over the block; the result is in every
// thread.  kind[k]: 0 argmax, 1 argmin, 2 max (index ignored).
template <int N>
__device__ void block_reduce(RedScratch &s, double (&v)[N], int (&idx)[N], const int (&kind)[N])
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < N; k++) {
        if (kind[k] == 0) warp_argmax(v[k], idx[k]);
        else if (kind[k] == 1) warp_argmin(v[k], idx[k]);
        else v[k] = warp_max(v[k]);
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < N; k++) { s.v[k][w] = v[k]; s.i[k][w] = idx[k]; }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; k++) {
        double vv = kind[k] == 1 ? SVMB_INF : -SVMB_INF;
        int ii = -1;
        if (lane < kWarps) { vv = s.v[k][lane]; ii = s.i[k][lane]; }
        if (kind[k] == 0) warp_argmax(vv, ii);
        else if (kind[k] == 1) warp_argmin(vv, ii);
        else vv = warp_max(vv);
        v[k] = vv;
        idx[k] = ii;
    }
}

__device__ int block_sum_i(RedScratch &s, int v)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_sum_i(v);
    __syncthreads();
    if (lane == 0) s.i[0][w] = v;
    __syncthreads();
    int tot = lane < kWarps ? s.i[0][lane] : 0;
    tot = warp_sum_i(tot);
    __syncthreads();
    return tot;
}

// exclusive prefix over the block of a 0/1 flag, in thread order; the block
// total goes to *total.
__device__ int block_excl_scan(RedScratch &s, int flag, int *total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned bal = __ballot_sync(0xffffffffu, flag);
    const int in_warp = __popc(bal & ((1u << lane) - 1u));
    __syncthreads();
    if (lane == 0) s.i[0][w] = __popc(bal);
    __syncthreads();
    int before = 0, tot = 0;
    for (int k = 0; k < kWarps; k++) {
        const int c = s.i[0][k];
        if (k < w) before += c;
        tot += c;
    }
    __syncthreads();
    *total = tot;
    return before + in_warp;
}

// --------------------------------------------------------------------------
// Q-row cache (set associative, LRU within a set).  Every block makes the same
// decisions from the same metadata; only block 0 writes metadata, one phase
// after the decision, and every reader overlays the decisions whose writes may
// still be in flight (prev) or are not yet issued (cur).
// --------------------------------------------------------------------------
struct CacheRec {
    int set, way, tag, epoch;
    unsigned long long stamp;
};

struct CacheState {
    CacheRec prev[16], cur[16];
    int nprev, ncur;
};

struct Lookup {
    long long slot;     // -1: no slot could be taken (prefetch only)
    int valid_active;   // positions [0,A) already valid
    int was_prefetched; // hit on a row that a prefetch filled and nobody used yet
};

// LRU stamps: 2*iter+1 for phase A, 2*iter+2 for phase B; bit 62 marks rows
// filled by prefetch and not yet used.
constexpr unsigned long long kPrefetchMark = 1ull << 62;

__device__ void cache_rotate(CacheState &cs, const CacheView &cv, int rank)
{
    // thread 0, right after an exchange: publish the previous phase's records
    if (rank == 0) {
        for (int k = 0; k < cs.ncur; k++) {
            const CacheRec &r = cs.cur[k];
            const long long s = (long long)r.set * cv.nways + r.way;
            cv.tag[s] = r.tag;
            cv.epoch[s] = r.epoch;
            cv.stamp[s] = r.stamp;
        }
    }
    for (int k = 0; k < cs.ncur; k++) cs.prev[k] = cs.cur[k];
    cs.nprev = cs.ncur;
    cs.ncur = 0;
}

// a cache set's metadata as stored in global memory, copied into shared memory
struct SetStage {
    int set;
    int tag[kMaxWays], ep[kMaxWays];
    unsigned long long st[kMaxWays];
};

// The set's metadata with this phase's and the previous phase's decisions
// laid over it.  Ways are visited by constant index (unrolled, guarded by the
// set's way count) so that the arrays stay in registers, and the global reads
// of a set go out together.
__device__ __forceinline__ void cache_read_set(const CacheState &cs, const CacheView &cv, int set, int (&tag)[kMaxWays],
                                               int (&ep)[kMaxWays], unsigned long long (&st)[kMaxWays],
                                               const SetStage *pre = nullptr)
{
    if (pre && pre->set == set) {
#pragma unroll
        for (int w = 0; w < kMaxWays; w++)
            if (w < cv.nways) {
                tag[w] = pre->tag[w];
                ep[w] = pre->ep[w];
                st[w] = pre->st[w];
            }
    } else {
        const long long s0 = (long long)set * cv.nways;
#pragma unroll
        for (int w = 0; w < kMaxWays; w++)
            if (w < cv.nways) {
                tag[w] = __ldcg(&cv.tag[s0 + w]);
                ep[w] = __ldcg(&cv.epoch[s0 + w]);
                st[w] = __ldcg(&cv.stamp[s0 + w]);
            }
    }
    auto overlay = [&](const CacheRec &r) {
#pragma unroll
        for (int w = 0; w < kMaxWays; w++)
            if (w == r.way) {
                tag[w] = r.tag;
                ep[w] = r.epoch;
                st[w] = r.stamp;
            }
    };
    for (int k = 0; k < cs.nprev; k++)
        if (cs.prev[k].set == set) overlay(cs.prev[k]);
    for (int k = 0; k < cs.ncur; k++)
        if (cs.cur[k].set == set) overlay(cs.cur[k]);
}

// Decide where row `local` lives; records the decision.  whole: the rows
// evaluated now cover every position (A == l), so they are complete.
// Victims are taken only among ways whose stamp is below `protect` (rows
// claimed in the phases still using them are never evicted).  A prefetch
// lookup (`prefetch`) takes a slot only if its set keeps at least two
// evictable ways, so that the rows the solver must place later always find
// one; otherwise it returns slot -1.
//
// The 32 lanes of one warp decide together: lane w reads and overlays way w
// (the set's metadata, then the previous and this phase's decisions), and
// the hit, the victim and the count of evictable ways come from ballots and
// a shuffle reduction.  A hit is the highest way holding the tag; the victim
// is the highest empty way, else the evictable way with the least stamp
// (lowest way on equal stamps).  Every lane returns the same Lookup; lane 0
// records the decision.  Called by all lanes of the warp with the same
// arguments.
__device__ Lookup cache_lookup_w(CacheState &cs, const CacheView &cv, int local, int cur_epoch,
                                 unsigned long long clk, int whole, unsigned long long protect, int prefetch,
                                 const SetStage *pre = nullptr)
{
    const int lane = threadIdx.x & 31;
    const int set = local % cv.nsets;
    const bool mine = lane < cv.nways;
    int tag = kNoTag, ep = 0;
    unsigned long long st = 0;
    if (mine) {
        if (pre && pre->set == set) {
            tag = pre->tag[lane];
            ep = pre->ep[lane];
            st = pre->st[lane];
        } else {
            const long long s = (long long)set * cv.nways + lane;
            tag = __ldcg(&cv.tag[s]);
            ep = __ldcg(&cv.epoch[s]);
            st = __ldcg(&cv.stamp[s]);
        }
    }
    // the previous phase's decisions, then this phase's, in order
    const int nprev = cs.nprev, ncur = cs.ncur;
    for (int k = 0; k < nprev; k++) {
        const CacheRec &r = cs.prev[k];
        if (r.set == set && r.way == lane) {
            tag = r.tag;
            ep = r.epoch;
            st = r.stamp;
        }
    }
    for (int k = 0; k < ncur; k++) {
        const CacheRec &r = cs.cur[k];
        if (r.set == set && r.way == lane) {
            tag = r.tag;
            ep = r.epoch;
            st = r.stamp;
        }
    }
    Lookup L;
    L.was_prefetched = 0;
    CacheRec rec;
    rec.set = set;
    rec.stamp = prefetch ? (clk | kPrefetchMark) : clk;
    rec.tag = local;
    int way;
    const unsigned hit = __ballot_sync(0xffffffffu, mine && tag == local);
    if (hit) {
        way = 31 - __clz(hit);
        const int ep_hit = __shfl_sync(0xffffffffu, ep, way);
        const unsigned long long st_hit = __shfl_sync(0xffffffffu, st, way);
        const int va = ep_hit == kEpochFull || ep_hit == cur_epoch;
        L.valid_active = va;
        L.was_prefetched = va && (st_hit & kPrefetchMark) ? 1 : 0;
        if (prefetch && va) rec.stamp = st_hit;   // a prefetch hit changes nothing
        rec.way = way;
        rec.epoch = whole ? kEpochFull : (va ? ep_hit : cur_epoch);
    } else {
        const unsigned long long sw = st & ~kPrefetchMark;
        const bool evict = mine && !(tag != kNoTag && sw >= protect);
        const unsigned em = __ballot_sync(0xffffffffu, evict);
        const unsigned empty = __ballot_sync(0xffffffffu, evict && tag == kNoTag);
        unsigned long long bv = evict ? sw : ~0ull;
        int bw = evict ? lane : 32;
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int ow = __shfl_xor_sync(0xffffffffu, bw, o);
            if (ov < bv || (ov == bv && ow < bw)) {
                bv = ov;
                bw = ow;
            }
        }
        const int victim = empty ? 31 - __clz(empty) : (em ? bw : -1);
        if (victim < 0 || (prefetch && __popc(em) < 3)) {
            L.slot = -1;
            L.valid_active = 0;
            return L;
        }
        L.valid_active = 0;
        rec.way = victim;
        rec.epoch = whole ? kEpochFull : cur_epoch;
        way = victim;
    }
    L.slot = (long long)set * cv.nways + way;
    __syncwarp();                     // every lane has read cs.cur
    if (lane == 0) {
        cs.cur[ncur] = rec;
        cs.ncur = ncur + 1;
    }
    __syncwarp();
    return L;
}

// Mark an already-decided slot as complete (after its tail has been filled).
__device__ void cache_mark_full(CacheState &cs, const CacheView &cv, long long slot, int local,
                                unsigned long long clk)
{
    CacheRec rec;
    rec.set = (int)(slot / cv.nways);
    rec.way = (int)(slot % cv.nways);
    rec.tag = local;
    rec.epoch = kEpochFull;
    rec.stamp = clk;
    cs.cur[cs.ncur++] = rec;
}

// --------------------------------------------------------------------------
// per-block solver context
// --------------------------------------------------------------------------
struct Shared {
    RedScratch red;
    CacheState cs;
    StageSlots ss;
    double bd[24];
    int bi[24];
    long long bl[8];
    int srcpos[kSrcBatch];
    int srcrow[kSrcBatch];
    int nsrc;
    int stop_at;
    Partial lrec[2];
    double cand_v[kWarps];
    int cand_p[kWarps];
    // rows of the current fill pass: row id, label, slot
    int frow[kPrefetchMax], fy[kPrefetchMax];
    long long fslot[kPrefetchMax];
    // per source of the fill pass running now: norm, label, destination row
    double fsx[kPrefetchMax];
    int fsy[kPrefetchMax];
    float *fsd[kPrefetchMax];
    int nfill;
    int pick[kPrefetchMax];
    int npick;
    SetStage sset[kPrefetchMax];    // cache sets of the prefetch picks, read in one round trip
    // tensor-core block products (FORM_BF16X3, FORM_FP16X3): sources of the current pass
    // (row id, position, alpha, norm, C, inverse scale, label, status), the
    // pipeline's mbarriers (one per operand stage) and the TMEM base address
    int tsrow[kTcMaxN], tspos[kTcMaxN];
    double tsa[kTcMaxN], tsx[kTcMaxN], tsc[kTcMaxN], tsi[kTcMaxN];
    signed char tsy[kTcMaxN];
    unsigned char tss[kTcMaxN];
    uint64_t tbar[kTcStages];
    uint32_t tmem;
    // the fill pipeline's mbarriers: operand stage loaded / free, accumulator
    // written / read; fabort is set by a role whose wait ran out
    uint64_t ffull[kFillStagesMax], fempty[kFillStagesMax], faccf[kFillAcc], facce[kFillAcc];
    int fabort;
};

// The group's prefetch candidates (kPrefetchCand per block).  They live in
// the same shared memory as the transpose tiles: candidates are read, chosen
// and looked up before the fill pass reuses the space.
struct PrefetchTable {
    double v[kMaxGroupBlocks * kPrefetchCand];
    int pos[kMaxGroupBlocks * kPrefetchCand], loc[kMaxGroupBlocks * kPrefetchCand];
    int row[kMaxGroupBlocks * kPrefetchCand], y[kMaxGroupBlocks * kPrefetchCand];
};

struct Ctx {
    const InstanceDesc *D;
    float *stage;           // source staging area (dynamic smem)
    float *tile;            // per-warp 32-row transpose tiles (dense rows) ...
    PrefetchTable *pt;      // ... sharing their space with the prefetch candidates
    // my chunk of [0,A) held in shared memory
    double *sG, *sA, *sQD;
    int *sCol, *sRow;
    signed char *sY;
    unsigned char *sS;
    int rank, nb;
    int A;                  // active size
    int a0, a1;             // my chunk of [0,A)
    int t0, t1;             // my chunk of [A,l)
    int epoch;
    int phase;              // exchange counter: selects the record buffer and sequence number
    Partial *lrec;          // single-block groups keep their two records in shared memory
    uint32_t tcbase;        // FORM_BF16X3: shared address of the operand stages (1024-aligned)
    long long tc_g, tc_t;   // tensor-core steps and tiles issued so far (mbarrier phase parities)
    long long fg;           // steps of the fill pipeline so far (its mbarrier phase parities)
    int fstages;            // operand stages of the fill pipeline (3 or 4, by the stage area)
};

__device__ __forceinline__ void set_chunks(Ctx &c)
{
    const long long n = c.A;
    c.a0 = (int)(n * c.rank / c.nb);
    c.a1 = (int)(n * (c.rank + 1) / c.nb);
    const long long m = c.D->l - c.A;
    c.t0 = c.A + (int)(m * c.rank / c.nb);
    c.t1 = c.A + (int)(m * (c.rank + 1) / c.nb);
}

__device__ __forceinline__ Partial *my_partial(const Ctx &c)
{
    if (c.nb == 1) return c.lrec + (c.phase & 1);
    return c.D->partials + (long long)(c.phase & 1) * c.nb + c.rank;
}
__device__ __forceinline__ const Partial *prev_partials(const Ctx &c)
{
    if (c.nb == 1) return c.lrec + ((c.phase - 1) & 1);
    return c.D->partials + (long long)((c.phase - 1) & 1) * c.nb;
}

// Record fields read by the reductions.  Multi-block records were written by
// other SMs: read them at L2 (ld.global.cg); single-block records live in
// shared memory.
struct RecVals {
    double v[6];
    int n[8];
    float q[2];
};
__device__ __forceinline__ void rec_load(const Ctx &c, const Partial *p, RecVals &r, int with_n_hi, int with_q)
{
    if (c.nb == 1) {
        for (int k = 0; k < 6; k++) r.v[k] = p->v[k];
        for (int k = 0; k < 8; k++) r.n[k] = p->n[k];
        r.q[0] = p->q[0];
        r.q[1] = p->q[1];
        return;
    }
    const double2 a = __ldcg(reinterpret_cast<const double2 *>(&p->v[0]));
    const double2 b = __ldcg(reinterpret_cast<const double2 *>(&p->v[2]));
    const double2 d = __ldcg(reinterpret_cast<const double2 *>(&p->v[4]));
    const int4 n0 = __ldcg(reinterpret_cast<const int4 *>(&p->n[0]));
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = b.x; r.v[3] = b.y; r.v[4] = d.x; r.v[5] = d.y;
    r.n[0] = n0.x; r.n[1] = n0.y; r.n[2] = n0.z; r.n[3] = n0.w;
    if (with_n_hi) {
        const int4 n1 = __ldcg(reinterpret_cast<const int4 *>(&p->n[4]));
        r.n[4] = n1.x; r.n[5] = n1.y; r.n[6] = n1.z; r.n[7] = n1.w;
    }
    if (with_q) {
        const float2 q = __ldcg(reinterpret_cast<const float2 *>(&p->q[0]));
        r.q[0] = q.x;
        r.q[1] = q.y;
    }
}

// Publish my record of this phase and wait for everybody's (group barrier).
__device__ bool exchange(Ctx &c, Shared &sh)
{
    __syncthreads();
    const int want = c.phase + 1;
    Partial *mine = my_partial(c);
    int ok = 1;
    if (c.nb > 1) {
        // the release store orders this thread's writes and, through the
        // barrier above, the whole block's before the record is seen
        if (threadIdx.x == 0) st_release_i32(&mine->seq, want);
        const Partial *all = c.D->partials + (long long)(c.phase & 1) * c.nb;
        const long long limit = c.D->wait_ns > 0 ? c.D->wait_ns : kWaitTimeoutNs;
        for (int b = threadIdx.x; b < c.nb; b += blockDim.x) {
            const long long t0 = (long long)tc::global_ns();
            long long spins = 0;
            // spin with relaxed loads; one acquire load of the awaited value
            // then synchronizes with the record's release store
            while (ld_relaxed_i32(&all[b].seq) != want) {
                if ((++spins & 63) == 0) {
                    if (ld_relaxed_i32(&c.D->sync->error) != 0 || (long long)tc::global_ns() - t0 > limit) {
                        atomicExch(&c.D->sync->error, 1);
                        ok = 0;
                        break;
                    }
                }
            }
            if (ok) (void)ld_acquire_i32(&all[b].seq);
        }
    }
    // the pollers' acquire loads, followed by the barrier, order every later
    // read of this block after the other blocks' releases
    ok = __syncthreads_and(ok);
    if (threadIdx.x == 0) cache_rotate(sh.cs, c.D->cache, c.rank);
    c.phase++;
    __syncthreads();
    return ok != 0;
}

__device__ __forceinline__ double get_C(const InstanceDesc &D, int y) { return y > 0 ? D.Cp : D.Cn; }

__device__ __forceinline__ unsigned char status_of(double a, double C)
{
    if (a >= C) return ST_UPPER;            // reference svm.cpp:441-449
    if (a <= 0) return ST_LOWER;
    return ST_FREE;
}

// chunk state: global -> shared / shared -> global (mutable fields only)
__device__ void chunk_load(Ctx &c)
{
    const InstanceDesc &D = *c.D;
    for (int k = threadIdx.x; k < c.a1 - c.a0; k += blockDim.x) {
        const int p = c.a0 + k;
        c.sG[k] = D.G[p];
        c.sA[k] = D.alpha[p];
        c.sQD[k] = D.QD[p];
        c.sCol[k] = D.pos_local[p];
        c.sRow[k] = D.pos_row[p];
        c.sY[k] = D.y[p];
        c.sS[k] = D.status[p];
    }
    __syncthreads();
}
__device__ void chunk_store(Ctx &c)
{
    const InstanceDesc &D = *c.D;
    __syncthreads();
    for (int k = threadIdx.x; k < c.a1 - c.a0; k += blockDim.x) {
        const int p = c.a0 + k;
        D.G[p] = c.sG[k];
        D.alpha[p] = c.sA[k];
        D.status[p] = c.sS[k];
    }
}

// Sum over the group's blocks of per-block counters of the previous exchange.
__device__ void group_counts(const Ctx &c, Shared &sh, int slot, int *below, int *above, int *total)
{
    const Partial *all = prev_partials(c);
    int b_lo = 0, b_hi = 0, tot = 0;
    for (int b = threadIdx.x; b < c.nb; b += blockDim.x) {
        const int v = c.nb == 1 ? all[b].n[slot] : __ldcg(&all[b].n[slot]);
        tot += v;
        if (b < c.rank) b_lo += v;
        if (b > c.rank) b_hi += v;
    }
    *below = block_sum_i(sh.red, b_lo);
    *above = block_sum_i(sh.red, b_hi);
    *total = block_sum_i(sh.red, tot);
}

// --------------------------------------------------------------------------
// row-block accumulation on the global state: for every target position e in
// [lo,hi), in source order over the positions s < src_end selected by the
// predicate,
//   G[e] += alpha_s * Q[s][e]  and, with `with_bar`, for upper-bound s,
//   G_bar[e] += C_s * Q[s][e].
// This is the initial gradient (svm.cpp:559-570) and the gradient
// reconstruction (svm.cpp:493-512); per target the additions happen in the
// same order as in the reference.
// --------------------------------------------------------------------------
template <int FORM>
__device__ void accumulate_rows(Ctx &c, Shared &sh, int src_end, int pick_free_only, int with_bar, int lo, int hi)
{
    const InstanceDesc &D = *c.D;
    const int cap = D.stage_cap > 0 ? D.stage_cap : kSrcBatch;
    int scan = 0;
    while (true) {
        if (threadIdx.x == 0) sh.nsrc = 0;
        __syncthreads();
        while (scan < src_end) {
            const int p = scan + threadIdx.x;
            int sel = 0;
            if (p < src_end) {
                const unsigned char s = D.status[p];
                sel = pick_free_only ? (s == ST_FREE) : (s != ST_LOWER);
            }
            int tot;
            const int pre = block_excl_scan(sh.red, sel, &tot);
            const int have = sh.nsrc;
            const int room = cap - have;
            if (sel && pre < room) sh.srcpos[have + pre] = p;
            const int take = tot < room ? tot : room;
            if (take < tot && sel && pre == take) sh.stop_at = threadIdx.x;
            __syncthreads();
            const int consumed = take == tot ? (int)blockDim.x : sh.stop_at;
            __syncthreads();
            if (threadIdx.x == 0) sh.nsrc = have + take;
            scan += consumed;
            __syncthreads();
            if (sh.nsrc == cap) break;
        }
        const int ns = sh.nsrc;
        if (ns == 0) break;
        if (threadIdx.x < ns) sh.srcrow[threadIdx.x] = D.pos_row[sh.srcpos[threadIdx.x]];
        __syncthreads();
        stage_sources(D, c.stage, sh.ss, sh.srcrow, ns);
        for (int e = lo + threadIdx.x; e < hi; e += blockDim.x) {
            double dots[kSrcBatch];
            const int r = D.pos_row[e];
            row_dots<FORM>(D, sh.ss, ns, r, dots);
            double g = D.G[e];
            double gb = with_bar ? D.G_bar[e] : 0.0;
            const int ye = D.y[e];
            const double xe = D.x.xsq ? D.x.xsq[r] : 0.0;
            for (int k = 0; k < ns; k++) {
                const int sp = sh.srcpos[k];
                const int ys = D.y[sp];
                const double xs = D.x.xsq ? D.x.xsq[sh.srcrow[k]] : 0.0;
                const float q = q_value(D.kp, ys * ye, dots[k], xs, xe);
                g = __dadd_rn(g, __dmul_rn(D.alpha[sp], (double)q));
                if (with_bar && D.status[sp] == ST_UPPER) gb = __dadd_rn(gb, __dmul_rn(get_C(D, ys), (double)q));
            }
            D.G[e] = g;
            if (with_bar) D.G_bar[e] = gb;
        }
        unstage_sources(D, c.stage, sh.ss);
        if (ns < cap) break;
    }
}

// --------------------------------------------------------------------------
// tensor-core block products (FORM_BF16X3, FORM_FP16X3)
// --------------------------------------------------------------------------
// dot(x_t, x_s) for the targets t in [lo,hi) -- chunk-local indices into the
// shared-memory chunk, or with `global_targets` positions of the global state
// -- against the ns <= tc_n sources whose row ids are in sh.tsrow, with the
// split of the form (x = hi + lo in bf16, or x 2^e = hi + lo in fp16;
// hi.lo + lo.hi + hi.hi, 3 MMAs per K-step of 16).
//
// Each step is one 64-feature chunk of one 128-target tile; its 12 MMAs start
// a fresh float32 accumulator in TMEM (two, alternating), and while the next
// chunk's MMAs run, the threads add the finished chunk into float64 registers:
// the tensor core's float32 accumulation then spans 64 features only, so its
// rounding stays at the level of a float32 dot product of that length.  The
// cross terms are issued before hi.hi so that they are added while the
// accumulator is small.  When a tile's last chunk is absorbed, `epi(tile_lo,
// acc)` runs on every thread: warp w holds TMEM lanes 32(w%4).. (targets) and,
// if 16(w/4) < N, columns 16(w/4)..+15 (sources) of the tile in acc[16].
//
// Operand stages (kTcStages deep) are filled by cp.async with 16-byte pieces
// of gathered rows into 128B-swizzled K-major tiles by all warps but the
// last; lane 0 of the last warp issues the MMAs and commits each step to its
// stage's mbarrier, queueing step g before step g-1 is waited for.  Every
// commit is waited for exactly once, in order, so the phase parities follow
// from the running step counter c.tc_g.  A wait that times out sets the group's error flag and
// the product returns false.
template <class Epi>
__device__ bool tc_product(Ctx &c, Shared &sh, int ns, int lo, int hi, bool global_targets, Epi &&epi)
{
    const InstanceDesc &D = *c.D;
    const int NK = D.x.nchunk;
    const int ntiles = hi > lo ? (hi - lo + kTcM - 1) / kTcM : 0;
    const int total = ntiles * NK;
    if (total <= 0 || ns <= 0) return true;
    const int N = (ns + 15) & ~15;                      // MMA N for M = 128: multiple of 16
    const uint32_t idesc = D.form == FORM_TF32 ? tc::idesc_tf32_f32(kTcM, N) : tc::idesc_f16_f32(kTcM, N, D.form == FORM_BF16X3);
    const uint32_t sbytes = (uint32_t)tc_stage_bytes(D.tc_n);
    const uint32_t a_lo = kTcM * 128u;                  // target lo tile
    const uint32_t b_hi = 2u * kTcM * 128u;             // source hi tile
    const uint32_t b_lo = b_hi + (uint32_t)D.tc_n * 128u;
    const long long rs = (long long)NK * 2 * kSplitChunk;
    const uint16_t *Xs = D.x.Xs;
    const int warp = threadIdx.x >> 5;
    const int lg = warp & 3, cg = warp >> 2;
    const bool reader = cg * 16 < N;
    // the last warp issues the MMAs and takes no part in the loads, so that
    // the issue overlaps the other warps' absorb and loads
    const int issuer = (int)(blockDim.x >> 5) - 1;
    const int nload = (int)blockDim.x - 32;
    auto load = [&](int g) {
        if (warp == issuer) return;
        const int tile = g / NK, kc = g - tile * NK;
        const uint32_t sa = c.tcbase + (uint32_t)((c.tc_g + g) % kTcStages) * sbytes;
        const int tb = lo + tile * kTcM;
        for (int i = threadIdx.x; i < kTcM * 16; i += nload) {
            const int r = i >> 4, q = i & 15;
            const int t = tb + r;
            const bool ok = t < hi;
            const int row = ok ? (global_targets ? D.pos_row[t] : c.sRow[t]) : 0;
            tc::cp_async16(sa + (q >= 8 ? a_lo : 0u) + tc::sw128_offset(r, q & 7),
                           Xs + (long long)row * rs + kc * 128 + q * 8, ok ? 16u : 0u);
        }
        for (int i = threadIdx.x; i < N * 16; i += nload) {
            const int r = i >> 4, q = i & 15;
            const bool ok = r < ns;
            const int row = ok ? sh.tsrow[r] : 0;
            tc::cp_async16(sa + (q >= 8 ? b_lo : b_hi) + tc::sw128_offset(r, q & 7),
                           Xs + (long long)row * rs + kc * 128 + q * 8, ok ? 16u : 0u);
        }
    };
    double acc[16];
#pragma unroll
    for (int k = 0; k < 16; k++) acc[k] = 0.0;
    // add the finished chunk of global step Gs (its MMAs have completed) into acc
    auto absorb = [&](long long Gs) {
        tc::tc_fence_after();
        if (reader) {
            float v[16];
            tc::tmem_ld16(sh.tmem + ((uint32_t)(lg * 32) << 16) + (uint32_t)((Gs & 1) * kTcMaxN + cg * 16), v);
#pragma unroll
            for (int k = 0; k < 16; k++) acc[k] = __dadd_rn(acc[k], (double)v[k]);
        }
    };
    auto finish_tile = [&](int tile) {
        epi(lo + tile * kTcM, acc);
#pragma unroll
        for (int k = 0; k < 16; k++) acc[k] = 0.0;
    };
    for (int g = 0; g < kTcStages - 1; g++) {
        if (g < total) load(g);
        tc::cp_async_commit();
    }
    bool ok = true;
    for (int g = 0; g < total; g++) {
        const long long G = c.tc_g + g;
        const int tile = g / NK, kc = g - tile * NK;
        // step g has landed: the groups of steps g+1 .. g+kTcStages-2 may still be pending
        tc::cp_async_wait<kTcStages - 2>();
        tc::fence_async_smem();
        __syncthreads();
        // step g's MMAs go in before step g-1's are waited for, so the tensor
        // core always has the next step queued.  Its accumulator (G & 1) was
        // last read by the absorb of step G-2, which ended before the barrier
        // that closed the previous iteration.
        if (threadIdx.x == (unsigned)(issuer * 32)) {
            tc::tc_fence_after();
            const uint32_t sa = c.tcbase + (uint32_t)(G % kTcStages) * sbytes;
            const uint32_t dst = sh.tmem + (uint32_t)((G & 1) * kTcMaxN);
            if (D.form == FORM_TF32) {
                // the two 128-byte halves hold features 0..31 and 32..63 of the chunk
#pragma unroll
                for (int h = 0; h < 2; h++)
#pragma unroll
                    for (int kk = 0; kk < 4; kk++)
                        tc::mma_tf32(dst, tc::sw128_desc(sa + (h ? a_lo : 0u) + kk * 32),
                                     tc::sw128_desc(sa + (h ? b_lo : b_hi) + kk * 32), idesc, h > 0 || kk > 0);
            } else {
#pragma unroll
                // the small cross terms of the whole chunk first, then hi.hi (the
                // tensor core's fp32 accumulation rounds toward zero; see the
                // kernel-block kernel): dots measured 2x less biased this way
                for (int kk = 0; kk < 4; kk++) {
                    const uint64_t ah = tc::sw128_desc(sa + kk * 32), al = tc::sw128_desc(sa + a_lo + kk * 32);
                    const uint64_t bh = tc::sw128_desc(sa + b_hi + kk * 32), bl = tc::sw128_desc(sa + b_lo + kk * 32);
                    tc::mma_bf16(dst, ah, bl, idesc, kk > 0);
                    tc::mma_bf16(dst, al, bh, idesc, true);
                }
#pragma unroll
                for (int kk = 0; kk < 4; kk++)
                    tc::mma_bf16(dst, tc::sw128_desc(sa + kk * 32), tc::sw128_desc(sa + b_hi + kk * 32), idesc, true);
            }
            tc::mma_commit(&sh.tbar[G % kTcStages]);
        }
        bool w = true;
        if (g >= 1) {
            // step g-1's MMAs have read their stage and written their accumulator
            w = tc::mbar_wait(&sh.tbar[(G - 1) % kTcStages], (unsigned)(((G - 1) / kTcStages) & 1));
            if (w) {
                absorb(G - 1);
                if (kc == 0) finish_tile(tile - 1);
            }
        }
        // the stage of step g-1 is free: step g + kTcStages - 1 goes there
        if (w && g + kTcStages - 1 < total) load(g + kTcStages - 1);
        tc::cp_async_commit();
        tc::tc_fence_before();
        ok = __syncthreads_and(w) != 0;
        if (!ok) break;
    }
    if (ok) {
        const long long G = c.tc_g + total - 1;
        ok = __syncthreads_and(tc::mbar_wait(&sh.tbar[G % kTcStages], (unsigned)((G / kTcStages) & 1))) != 0;
        if (ok) {
            absorb(G);
            finish_tile(ntiles - 1);
            tc::tc_fence_before();
        }
    }
    tc::cp_async_wait<0>();
    c.tc_g += total;
    c.tc_t += ntiles;
    if (!ok && threadIdx.x == 0) atomicExch(&D.sync->error, 1);
    __syncthreads();
    return ok;
}

// tensor-core form of fill_rows: Q rows of ns (<= kPrefetchMax) sources into
// cache slots, on my chunk of [0,A) (tail = 0) or of [A,l) (tail = 1).
//
// A warp-specialised pipeline over the steps (one 64-feature chunk of one
// 128-target tile) with no block barrier per step:
//   warps kFillLoad0..  load a step's target tile and source rows into a free
//                       operand stage (cp.async), wait for their own copies,
//                       fence them into the async proxy and arrive on ffull;
//   warp 4, one lane    waits for ffull and for a free accumulator, issues the
//                       step's MMAs and commits them to fempty (stage free) and
//                       faccf (accumulator written);
//   warps 0-3           (TMEM lanes = the tile's 128 targets) wait for faccf,
//                       add the fp32 chunk into fp64 registers, arrive on facce,
//                       and write the tile's Q values after its last chunk.
// The MMAs, their order and the fp64 flush are those of tc_product, so the Q
// values are the same bit for bit.  Every wait is bounded; a role whose wait
// runs out sets fabort, which ends the other roles' waits.
__device__ bool fill_rows_tc(Ctx &c, Shared &sh, int ns, const int *src_row, const int *src_y, const long long *slot,
                             int tail)
{
    const InstanceDesc &D = *c.D;
    if (ns == 0) return true;
    if (threadIdx.x < ns) {
        // the sources' row, norm, inverse scale, label and destination row
        const int k = threadIdx.x;
        sh.tsrow[k] = src_row[k];
        sh.fsx[k] = D.x.xsq[src_row[k]];
        sh.tsi[k] = D.x.xinv ? D.x.xinv[src_row[k]] : 1.0;
        sh.fsy[k] = src_y[k];
        sh.fsd[k] = D.cache.data + slot[k] * D.cache.stride;
    }
    __syncthreads();
    const int lo = tail ? c.t0 : 0, hi = tail ? c.t1 : c.a1 - c.a0;
    const int NK = D.x.nchunk;
    const int ntiles = hi > lo ? (hi - lo + kTcM - 1) / kTcM : 0;
    const int total = ntiles * NK;
    if (total <= 0) return true;
    const int S = c.fstages;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    volatile int *abort = &sh.fabort;
    constexpr uint32_t kStage = (uint32_t)fill_stage_bytes();
    constexpr uint32_t a_lo = kTcM * 128u;                       // target lo tile
    constexpr uint32_t b_hi = 2u * kTcM * 128u;                  // source hi tile
    constexpr uint32_t b_lo = b_hi + (uint32_t)kFillN * 128u;    // source lo tile
    const long long rs = (long long)NK * 2 * kSplitChunk;
    if (warp < 4) {
        // ---- readers and epilogue: target t = tile base + warp * 32 + lane.
        // The target's row norm, scale, label and cache column are loaded when
        // its tile starts, so the epilogue waits on no global load.
        double acc[kPrefetchMax];
#pragma unroll
        for (int k = 0; k < kPrefetchMax; k++) acc[k] = 0.0;
        int a = (int)(c.fg % kFillAcc);
        unsigned ph = (unsigned)((c.fg / kFillAcc) & 1);
        int kc = 0, tile = 0;
        int yp = 0, col = 0;
        bool tok = false;
        double xe = 0.0, ie = 1.0;
        for (int g = 0; g < total; g++) {
            if (kc == 0) {
                const int t = lo + tile * kTcM + warp * 32 + lane;
                tok = t < hi;
                if (tok) {
                    int r;
                    if (tail) {
                        r = D.pos_row[t];
                        yp = D.y[t];
                        col = D.pos_local[t];
                    } else {
                        r = c.sRow[t];
                        yp = c.sY[t];
                        col = c.sCol[t];
                    }
                    xe = D.x.xsq[r];
                    ie = D.x.xinv ? D.x.xinv[r] : 1.0;
                }
            }
            if (!tc::mbar_wait_or(&sh.faccf[a], ph, abort)) {
                *abort = 1;
                break;
            }
            tc::tc_fence_after();
            float v[kPrefetchMax];
            tc::tmem_ld8(sh.tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(a * kFillN), v);
#pragma unroll
            for (int k = 0; k < kPrefetchMax; k++) acc[k] = __dadd_rn(acc[k], (double)v[k]);
            tc::tc_fence_before();
            tc::mbar_arrive(&sh.facce[a]);
            if (++a == kFillAcc) {
                a = 0;
                ph ^= 1u;
            }
            if (++kc == NK) {
                if (tok) {
#pragma unroll
                    for (int k = 0; k < kPrefetchMax; k++)
                        if (k < ns)
                            __stcg(sh.fsd[k] + col, q_value(D.kp, sh.fsy[k] * yp,
                                                            __dmul_rn(__dmul_rn(acc[k], ie), sh.tsi[k]), sh.fsx[k], xe));
                }
#pragma unroll
                for (int k = 0; k < kPrefetchMax; k++) acc[k] = 0.0;
                kc = 0;
                tile++;
            }
        }
    } else if (warp == 4) {
        // ---- MMA issue
        if (lane == 0) {
            const uint32_t idesc = D.form == FORM_TF32 ? tc::idesc_tf32_f32(kTcM, kFillN)
                                                       : tc::idesc_f16_f32(kTcM, kFillN, D.form == FORM_BF16X3);
            int s = (int)(c.fg % S), a = (int)(c.fg % kFillAcc);
            unsigned phs = (unsigned)((c.fg / S) & 1), pha = (unsigned)((c.fg / kFillAcc) & 1);
            int issued = 0;
            for (int g = 0; g < total; g++) {
                if (!tc::mbar_wait_or(&sh.ffull[s], phs, abort) || !tc::mbar_wait_or(&sh.facce[a], pha ^ 1u, abort)) {
                    *abort = 1;
                    break;
                }
                tc::tc_fence_after();
                const uint32_t sa = c.tcbase + (uint32_t)s * kStage;
                const uint32_t dst = sh.tmem + (uint32_t)(a * kFillN);
                if (D.form == FORM_TF32) {
#pragma unroll
                    for (int h = 0; h < 2; h++)
#pragma unroll
                        for (int kk = 0; kk < 4; kk++)
                            tc::mma_tf32(dst, tc::sw128_desc(sa + (h ? a_lo : 0u) + kk * 32),
                                         tc::sw128_desc(sa + (h ? b_lo : b_hi) + kk * 32), idesc, h > 0 || kk > 0);
                } else {
                    // cross terms of the chunk first, then hi.hi (as in tc_product)
#pragma unroll
                    for (int kk = 0; kk < 4; kk++) {
                        tc::mma_bf16(dst, tc::sw128_desc(sa + kk * 32), tc::sw128_desc(sa + b_lo + kk * 32), idesc,
                                     kk > 0);
                        tc::mma_bf16(dst, tc::sw128_desc(sa + a_lo + kk * 32), tc::sw128_desc(sa + b_hi + kk * 32),
                                     idesc, true);
                    }
#pragma unroll
                    for (int kk = 0; kk < 4; kk++)
                        tc::mma_bf16(dst, tc::sw128_desc(sa + kk * 32), tc::sw128_desc(sa + b_hi + kk * 32), idesc, true);
                }
                tc::mma_commit(&sh.fempty[s]);
                tc::mma_commit(&sh.faccf[a]);
                issued++;
                if (++s == S) {
                    s = 0;
                    phs ^= 1u;
                }
                if (++a == kFillAcc) {
                    a = 0;
                    pha ^= 1u;
                }
            }
            if (issued < total && issued > 0) {
                // stopped early: let the MMAs already issued finish before the
                // stages and the accumulators are given up
                const long long G = c.fg + issued - 1;
                tc::mbar_wait(&sh.fempty[G % S], (unsigned)((G / S) & 1));
            }
        }
        __syncwarp();
    } else {
        // ---- operand loads: piece i of a step is a 16-byte piece of a target
        // row (i < 16 * kTcM) or of a source row; the pieces of a thread keep
        // their rows for a whole tile, only the chunk moves
        constexpr int kLoaders = kThreads - kFillLoad0 * 32;
        constexpr int kPieces = (16 * kTcM + 16 * kPrefetchMax + kLoaders - 1) / kLoaders;
        const int lt = threadIdx.x - kFillLoad0 * 32;
        const uint16_t *Xs = D.x.Xs;
        const uint16_t *src[kPieces];
        uint32_t off[kPieces];
        int s = (int)(c.fg % S), sd = s;
        unsigned phs = (unsigned)((c.fg / S) & 1);
        int kc = 0, tile = 0;
        bool run = true;
        // up to S - 1 steps in flight; a landed step is handed to the MMA
        // before this thread waits for a free stage, so that the MMAs of
        // consecutive steps queue back to back
        for (int g = 0; g < total + S - 1; g++) {
            if (g >= S - 1 && run) {
                // step g - (S - 1) has landed (S - 2 younger groups may be pending)
                tc::cp_async_wait_n(S - 2);
                tc::fence_async_smem();
                tc::mbar_arrive(&sh.ffull[sd]);
                if (++sd == S) sd = 0;
            }
            if (g < total && run) {
                if (kc == 0) {
                    const int tb = lo + tile * kTcM;
#pragma unroll
                    for (int j = 0; j < kPieces; j++) {
                        const int i = lt + j * kLoaders;
                        src[j] = nullptr;
                        off[j] = 0;
                        if (i < 16 * kTcM) {
                            const int r = i >> 4, q = i & 15, t = tb + r;
                            if (t < hi) {
                                const int row = tail ? D.pos_row[t] : c.sRow[t];
                                src[j] = Xs + (long long)row * rs + q * 8;
                                off[j] = (q >= 8 ? a_lo : 0u) + tc::sw128_offset(r, q & 7);
                            }
                        } else if (i < 16 * kTcM + 16 * ns) {
                            const int r = (i - 16 * kTcM) >> 4, q = i & 15;
                            src[j] = Xs + (long long)sh.tsrow[r] * rs + q * 8;
                            off[j] = (q >= 8 ? b_lo : b_hi) + tc::sw128_offset(r, q & 7);
                        }
                    }
                }
                if (!tc::mbar_wait_or(&sh.fempty[s], phs ^ 1u, abort)) {
                    *abort = 1;
                    run = false;
                } else {
                    const uint32_t sa = c.tcbase + (uint32_t)s * kStage;
#pragma unroll
                    for (int j = 0; j < kPieces; j++)
                        if (src[j]) tc::cp_async16(sa + off[j], src[j] + kc * 128, 16u);
                }
                if (++s == S) {
                    s = 0;
                    phs ^= 1u;
                }
                if (++kc == NK) {
                    kc = 0;
                    tile++;
                }
            }
            tc::cp_async_commit();
        }
        tc::cp_async_wait<0>();
    }
    c.fg += total;
    tc::tc_fence_before();
    __syncthreads();
    const bool ok = *abort == 0;
    if (!ok && threadIdx.x == 0) atomicExch(&D.sync->error, 1);
    __syncthreads();
    tc::tc_fence_after();
    return ok;
}

// tensor-core form of accumulate_rows: sources are taken kTcMaxN (tc_n) at a
// time; per target the contributions of one pass are summed in source order
// in four column groups, which are then added in a fixed order
__device__ bool accumulate_rows_tc(Ctx &c, Shared &sh, int src_end, int pick_free_only, int with_bar, int lo, int hi)
{
    const InstanceDesc &D = *c.D;
    const int cap = D.tc_n;
    int scan = 0;
    double *red = reinterpret_cast<double *>(c.tile);   // [2][4][kTcM] partial sums (aux area)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int lg = warp & 3, cg = warp >> 2;
    while (true) {
        if (threadIdx.x == 0) sh.nsrc = 0;
        __syncthreads();
        while (scan < src_end) {
            const int p = scan + threadIdx.x;
            int sel = 0;
            if (p < src_end) {
                const unsigned char s = D.status[p];
                sel = pick_free_only ? (s == ST_FREE) : (s != ST_LOWER);
            }
            int tot;
            const int pre = block_excl_scan(sh.red, sel, &tot);
            const int have = sh.nsrc;
            const int room = cap - have;
            if (sel && pre < room) sh.tspos[have + pre] = p;
            const int take = tot < room ? tot : room;
            if (take < tot && sel && pre == take) sh.stop_at = threadIdx.x;
            __syncthreads();
            const int consumed = take == tot ? (int)blockDim.x : sh.stop_at;
            __syncthreads();
            if (threadIdx.x == 0) sh.nsrc = have + take;
            scan += consumed;
            __syncthreads();
            if (sh.nsrc == cap) break;
        }
        const int ns = sh.nsrc;
        if (ns == 0) break;
        if (threadIdx.x < ns) {
            const int sp = sh.tspos[threadIdx.x];
            const int r = D.pos_row[sp];
            const int y = D.y[sp];
            sh.tsrow[threadIdx.x] = r;
            sh.tsa[threadIdx.x] = D.alpha[sp];
            sh.tsx[threadIdx.x] = D.x.xsq[r];
            sh.tsi[threadIdx.x] = D.x.xinv ? D.x.xinv[r] : 1.0;
            sh.tsc[threadIdx.x] = get_C(D, y);
            sh.tsy[threadIdx.x] = (signed char)y;
            sh.tss[threadIdx.x] = D.status[sp];
        }
        __syncthreads();
        const bool ok = tc_product(c, sh, ns, lo, hi, true, [&](int tlo, const double *acc) {
            const int t = tlo + lg * 32 + lane;
            double part = 0.0, partb = 0.0;
            if (cg * 16 < ns && t < hi) {
                const int r = D.pos_row[t];
                const int ye = D.y[t];
                const double xe = D.x.xsq[r];
                const double ie = D.x.xinv ? D.x.xinv[r] : 1.0;
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    const int s = cg * 16 + k;
                    if (s < ns) {
                        const double dot = __dmul_rn(__dmul_rn(acc[k], ie), sh.tsi[s]);
                        const float q = q_value(D.kp, sh.tsy[s] * ye, dot, sh.tsx[s], xe);
                        part = __dadd_rn(part, __dmul_rn(sh.tsa[s], (double)q));
                        if (with_bar && sh.tss[s] == ST_UPPER) partb = __dadd_rn(partb, __dmul_rn(sh.tsc[s], (double)q));
                    }
                }
            }
            red[cg * kTcM + lg * 32 + lane] = part;
            red[4 * kTcM + cg * kTcM + lg * 32 + lane] = partb;
            __syncthreads();
            if (cg == 0 && t < hi) {
                double g = D.G[t];
                for (int k = 0; k < 4; k++) g = __dadd_rn(g, red[k * kTcM + lg * 32 + lane]);
                D.G[t] = g;
                if (with_bar) {
                    double gb = D.G_bar[t];
                    for (int k = 0; k < 4; k++) gb = __dadd_rn(gb, red[4 * kTcM + k * kTcM + lg * 32 + lane]);
                    D.G_bar[t] = gb;
                }
            }
            __syncthreads();
        });
        if (!ok) return false;
        if (ns < cap) break;
    }
    return true;
}

// the row-block product of the form: CUDA cores or tensor cores
template <int FORM>
__device__ bool accumulate(Ctx &c, Shared &sh, int src_end, int pick_free_only, int with_bar, int lo, int hi)
{
    if constexpr (is_tc_form(FORM)) {
        return accumulate_rows_tc(c, sh, src_end, pick_free_only, with_bar, lo, hi);
    } else {
        accumulate_rows<FORM>(c, sh, src_end, pick_free_only, with_bar, lo, hi);
        return true;
    }
}

// gradient reconstruction (reference svm.cpp:473-513); group collective on the
// global state (the caller has stored its chunk)
template <int FORM>
__device__ bool reconstruct(Ctx &c, Shared &sh)
{
    const InstanceDesc &D = *c.D;
    if (c.A == D.l) return true;
    if (D.lazy_gbar) {
        // G = p + sum over every alpha > 0 (active or not) of alpha * Q, on the inactive positions
        for (int e = c.t0 + threadIdx.x; e < c.t1; e += blockDim.x) D.G[e] = D.p[e];
        __syncthreads();
        if (!accumulate<FORM>(c, sh, D.l, 0, 0, c.t0, c.t1)) return false;
        return exchange(c, sh);
    }
    for (int e = c.t0 + threadIdx.x; e < c.t1; e += blockDim.x) D.G[e] = __dadd_rn(D.G_bar[e], D.p[e]);
    __syncthreads();
    if (!accumulate<FORM>(c, sh, c.A, 1, 0, c.t0, c.t1)) return false;
    return exchange(c, sh);
}

// --------------------------------------------------------------------------
// shrinking (reference svm.cpp:932-1011 / Solver_NU :1188-1258)
// --------------------------------------------------------------------------
__device__ __forceinline__ bool be_shrunk(int nu, unsigned char s, int y, double G, const double *g)
{
    if (!nu) {
        if (s == ST_UPPER) return y == +1 ? (-G > g[0]) : (-G > g[1]);
        if (s == ST_LOWER) return y == +1 ? (G > g[1]) : (G > g[0]);
        return false;
    }
    if (s == ST_UPPER) return y == +1 ? (-G > g[0]) : (-G > g[3]);
    if (s == ST_LOWER) return y == +1 ? (G > g[1]) : (G > g[2]);
    return false;
}

__device__ __forceinline__ void swap_pos(const InstanceDesc &D, int a, int b)
{
    double t;
    t = D.G[a]; D.G[a] = D.G[b]; D.G[b] = t;
    t = D.G_bar[a]; D.G_bar[a] = D.G_bar[b]; D.G_bar[b] = t;
    t = D.alpha[a]; D.alpha[a] = D.alpha[b]; D.alpha[b] = t;
    t = D.p[a]; D.p[a] = D.p[b]; D.p[b] = t;
    t = D.QD[a]; D.QD[a] = D.QD[b]; D.QD[b] = t;
    signed char ty = D.y[a]; D.y[a] = D.y[b]; D.y[b] = ty;
    unsigned char ts = D.status[a]; D.status[a] = D.status[b]; D.status[b] = ts;
    int ti = D.pos_local[a]; D.pos_local[a] = D.pos_local[b]; D.pos_local[b] = ti;
    ti = D.pos_row[a]; D.pos_row[a] = D.pos_row[b]; D.pos_row[b] = ti;
}

// widen the active set to l after a reconstruction (chunk reloaded)
__device__ void widen(Ctx &c)
{
    c.A = c.D->l;
    c.epoch++;
    set_chunks(c);
    chunk_load(c);
}

template <int FORM>
__device__ bool do_shrinking(Ctx &c, Shared &sh, int &unshrink)
{
    const InstanceDesc &D = *c.D;
    const int nu = D.nu;
    const int n = c.a1 - c.a0;
    // 1. maximal violations over the active set (C-SVC: Gmax1, Gmax2; nu: Gmax1..4)
    {
        double v[4] = {-SVMB_INF, -SVMB_INF, -SVMB_INF, -SVMB_INF};
        int ix[4] = {-1, -1, -1, -1};
        const int kind[4] = {2, 2, 2, 2};
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            const unsigned char s = c.sS[k];
            const double G = c.sG[k];
            const int y = c.sY[k];
            if (!nu) {
                if (y == +1) {
                    if (s != ST_UPPER) v[0] = fmax(v[0], -G);
                    if (s != ST_LOWER) v[1] = fmax(v[1], G);
                } else {
                    if (s != ST_UPPER) v[1] = fmax(v[1], -G);
                    if (s != ST_LOWER) v[0] = fmax(v[0], G);
                }
            } else {
                if (s != ST_UPPER) { if (y == +1) v[0] = fmax(v[0], -G); else v[3] = fmax(v[3], -G); }
                if (s != ST_LOWER) { if (y == +1) v[1] = fmax(v[1], G); else v[2] = fmax(v[2], G); }
            }
        }
        block_reduce<4>(sh.red, v, ix, kind);
        if (threadIdx.x == 0) {
            Partial *pp = my_partial(c);
            for (int k = 0; k < 4; k++) pp->v[k] = v[k];
        }
    }
    chunk_store(c);     // the swaps and a reconstruction work on the global state
    if (!exchange(c, sh)) return false;
    double g[4];
    {
        const Partial *all = prev_partials(c);
        double v[4] = {-SVMB_INF, -SVMB_INF, -SVMB_INF, -SVMB_INF};
        int ix[4] = {-1, -1, -1, -1};
        const int kind[4] = {2, 2, 2, 2};
        for (int b = threadIdx.x; b < c.nb; b += blockDim.x) {
            RecVals r;
            rec_load(c, &all[b], r, 0, 0);
            for (int k = 0; k < 4; k++) v[k] = fmax(v[k], r.v[k]);
        }
        block_reduce<4>(sh.red, v, ix, kind);
        for (int k = 0; k < 4; k++) g[k] = v[k];
    }
    const double gap = nu ? fmax(__dadd_rn(g[0], g[1]), __dadd_rn(g[2], g[3])) : __dadd_rn(g[0], g[1]);
    if (!unshrink && gap <= __dmul_rn(D.eps, 10.0)) {
        unshrink = 1;
        if (!reconstruct<FORM>(c, sh)) return false;
        widen(c);
    }
    // 2. shrunk positions per block -> new active size K
    {
        int cnt = 0;
        for (int k = threadIdx.x; k < c.a1 - c.a0; k += blockDim.x)
            cnt += be_shrunk(nu, c.sS[k], c.sY[k], c.sG[k], g) ? 1 : 0;
        cnt = block_sum_i(sh.red, cnt);
        if (threadIdx.x == 0) my_partial(c)->n[0] = cnt;
    }
    if (!exchange(c, sh)) return false;
    int K;
    {
        int below, above, tot;
        group_counts(c, sh, 0, &below, &above, &tot);
        K = c.A - tot;
    }
    // 3. holes = shrunk positions in [0,K) ascending, movers = kept positions in [K,A) descending
    {
        int h = 0, m = 0;
        for (int k = threadIdx.x; k < c.a1 - c.a0; k += blockDim.x) {
            const int p = c.a0 + k;
            const bool s = be_shrunk(nu, c.sS[k], c.sY[k], c.sG[k], g);
            if (p < K && s) h++;
            if (p >= K && !s) m++;
        }
        h = block_sum_i(sh.red, h);
        m = block_sum_i(sh.red, m);
        if (threadIdx.x == 0) { Partial *pp = my_partial(c); pp->n[0] = h; pp->n[1] = m; }
    }
    if (!exchange(c, sh)) return false;
    int hole_base, movers_below, movers_above, total_movers, dummy0, dummy1;
    group_counts(c, sh, 0, &hole_base, &dummy0, &dummy1);
    group_counts(c, sh, 1, &movers_below, &movers_above, &total_movers);
    int *holes = D.scratch;
    int *movers = D.scratch + D.l;
    {
        int h_run = 0, m_run = 0;
        for (int base = 0; base < c.a1 - c.a0; base += blockDim.x) {
            const int k = base + threadIdx.x;
            const int p = c.a0 + k;
            bool s = false;
            if (p < c.a1) s = be_shrunk(nu, c.sS[k], c.sY[k], c.sG[k], g);
            const int isH = (p < c.a1 && p < K && s) ? 1 : 0;
            const int isM = (p < c.a1 && p >= K && !s) ? 1 : 0;
            int totH, totM;
            const int preH = block_excl_scan(sh.red, isH, &totH);
            const int preM = block_excl_scan(sh.red, isM, &totM);
            if (isH) holes[hole_base + h_run + preH] = p;
            if (isM) {
                const int asc = movers_below + m_run + preM;        // ascending rank among movers
                movers[total_movers - 1 - asc] = p;                 // descending pairing order
            }
            h_run += totH;
            m_run += totM;
        }
    }
    if (!exchange(c, sh)) return false;
    // 4. swap pair r: holes[r] <-> movers[r] (the reference's swap_index loop)
    for (long long r = (long long)c.rank * blockDim.x + threadIdx.x; r < total_movers; r += (long long)c.nb * blockDim.x)
        swap_pos(D, __ldcg(&holes[r]), __ldcg(&movers[r]));
    if (!exchange(c, sh)) return false;
    c.A = K;
    set_chunks(c);
    chunk_load(c);
    return true;
}

// --------------------------------------------------------------------------
// I_up scan of my chunk (first half of WSS3): per track the max of -y_t G_t
// with its payload.  C-SVC uses track 0 only; nu-SVC: track 0 = y=+1, 1 = y=-1.
// --------------------------------------------------------------------------
// Prefetch priority of a position: how strongly it violates optimality on
// either side, max(-y G over I_up, y G over I_low) -- the quantities whose
// extremes WSS picks from, so high-priority rows are likely to be needed soon.
__device__ __forceinline__ double prefetch_priority(int y, unsigned char s, double G)
{
    double up = -SVMB_INF, low = -SVMB_INF;
    if (y == +1) {
        if (s != ST_UPPER) up = -G;
        if (s != ST_LOWER) low = G;
    } else {
        if (s != ST_LOWER) up = G;
        if (s != ST_UPPER) low = -G;
    }
    return fmax(up, low);
}

// Publish the block's I_up maxima (with payload) and its most violating
// positions (prefetch candidates: the best of each warp, top kPrefetchCand).
__device__ void iup_publish(const Ctx &c, Shared &sh, double (&v)[2], int (&ix)[2], double pv, int pix)
{
    const int kind[2] = {0, 0};
    // warp winners of the prefetch priority
    warp_argmax(pv, pix);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sh.cand_v[w] = pv;
        sh.cand_p[w] = pix;
    }
    block_reduce<2>(sh.red, v, ix, kind);   // its barriers also publish cand_*
    if (threadIdx.x < 32) {
        double cv = lane < kWarps ? sh.cand_v[lane] : -SVMB_INF;
        int cp = lane < kWarps ? sh.cand_p[lane] : -1;
        Partial *pp = my_partial(c);
        for (int t = 0; t < kPrefetchCand; t++) {
            double bv = cv;
            int bp = cp;
            warp_argmax(bv, bp);
            if (bp >= 0 && bv > -SVMB_INF) {
                if (cp == bp) cv = -SVMB_INF;        // remove the winner
                if (lane == 0) {
                    const int q = bp - c.a0;
                    pp->cv[t] = bv;
                    pp->cpos[t] = bp;
                    pp->cloc[t] = c.sCol[q];
                    pp->crow[t] = c.sRow[q];
                    pp->cy[t] = c.sY[q];
                }
            } else if (lane == 0) {
                pp->cv[t] = -SVMB_INF;
                pp->cpos[t] = -1;
            }
        }
    }
    if (threadIdx.x == 0) {
        Partial *pp = my_partial(c);
        for (int k = 0; k < 2; k++) {
            const int p = ix[k];
            const int q = p - c.a0;
            pp->v[3 * k + 0] = v[k];
            pp->n[4 * k + 0] = p;
            if (p >= 0) {
                pp->v[3 * k + 1] = c.sA[q];
                pp->v[3 * k + 2] = c.sQD[q];
                pp->n[4 * k + 1] = c.sCol[q];
                pp->n[4 * k + 2] = c.sRow[q];
                pp->n[4 * k + 3] = c.sY[q];
            }
        }
    }
}

__device__ void scan_iup(Ctx &c, Shared &sh)
{
    const int nu = c.D->nu;
    double v[2] = {-SVMB_INF, -SVMB_INF};
    int ix[2] = {-1, -1};
    double pv = -SVMB_INF;
    int pix = -1;
    for (int k = threadIdx.x; k < c.a1 - c.a0; k += blockDim.x) {
        const unsigned char s = c.sS[k];
        const double G = c.sG[k];
        const int y = c.sY[k];
        if (y == +1) {
            if (s != ST_UPPER) better_max(v[0], ix[0], -G, c.a0 + k);
        } else {
            if (s != ST_LOWER) better_max(v[nu], ix[nu], G, c.a0 + k);
        }
        better_max(pv, pix, prefetch_priority(y, s, G), c.a0 + k);
    }
    iup_publish(c, sh, v, ix, pv, pix);
}

// Dot products of the 32 rows of a warp (lane L owns row r) with up to 8
// staged dense sources.  The 32 rows are read in 16-column slices with
// coalesced 64-byte pieces per row (cp.async, 16 bytes per lane) into 32 x 16
// shared tiles (pieces swizzled).  The warp's tiles form a ring of
// D.tile_bufs slices: all but the one in use are in flight, so a warp moves
// tile_bufs slices per memory round trip.  Every lane accumulates ITS row in
// feature order from the tile -- the reference's summation order.
// shared-memory loads by 32-bit shared-window address (volatile: they stay
// after the cp.async wait and __syncwarp that publish the tile)
__device__ __forceinline__ float4 lds_f4(uint32_t a)
{
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
}
__device__ __forceinline__ double2 lds_d2(uint32_t a)
{
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
    return v;
}
// four staged source values at byte address a: float4, or two double2
__device__ __forceinline__ float4 src4_at(uint32_t a, float) { return lds_f4(a); }
__device__ __forceinline__ D4 src4_at(uint32_t a, double)
{
    const double2 p = lds_d2(a), q = lds_d2(a + 16);
    return D4{p.x, p.y, q.x, q.y};
}

template <int FORM, int NS, typename S>
__device__ __forceinline__ void warp_tile_dots(const InstanceDesc &D, const StageSlots &ss, int ns, int r, float *tile,
                                               double (&out)[kPrefetchMax])
{
    typedef typename Acc<FORM>::type acc_t;
    const int lane = threadIdx.x & 31;
    const int ld = D.x.ld;   // multiple of 4
    const float *X = D.x.X;
    acc_t acc[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) acc[k] = acc_t(0);
    // the staged sources lie D.stage_lds values apart from the first
    const uint32_t src0 = tc::smem_addr(ss.sp[0]);
    const uint32_t sstride = (uint32_t)(D.stage_lds * (int)sizeof(S));
    // a slice is 32 rows x 4 pieces of 16 bytes; lane L moves pieces L + 32i
    // (i < 4): row (L + 32i) / 4, piece L % 4.  Row t of a tile = the row of lane t.
    const float *prow[4];
#pragma unroll
    for (int i = 0; i < 4; i++) prow[i] = X + (long long)__shfl_sync(0xffffffffu, r, (lane + 32 * i) >> 2) * ld + 4 * (lane & 3);
    const uint32_t tile_s = tc::smem_addr(tile);
    auto issue = [&](int c0, int buf) {
        if (c0 < ld) {
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int t = (lane + 32 * i) >> 2;
                const bool ok = c0 + 4 * (lane & 3) < ld;     // ld is a multiple of 4
                // piece c of tile row t sits at piece position c ^ ((t >> 1) & 3): the
                // 16-byte reads of 8 consecutive lanes then hit distinct banks
                tc::cp_async16(tile_s + (uint32_t)((buf * 32 * kTileStride + t * kTileStride + 4 * ((lane & 3) ^ ((t >> 1) & 3))) * 4),
                               prow[i] + (ok ? c0 : 0), ok ? 16u : 0u);
            }
        }
        tc::cp_async_commit();
    };
    const int nb = D.tile_bufs;
    // prologue: slices 0 .. nb-2 in flight
    for (int p = 0; p + 1 < nb; p++) issue(16 * p, p);
    for (int c0 = 0, s = 0; c0 < ld; c0 += 16) {
        // slice s + nb - 1 goes to the buffer used by slice s - 1 (consumed
        // before the __syncwarp that ended the previous step)
        issue(c0 + 16 * (nb - 1), s == 0 ? nb - 1 : s - 1);
        tc::cp_async_wait_n(nb - 1);                     // slice s has landed (for this lane)
        __syncwarp();
        const uint32_t cur = tile_s + (uint32_t)(s * 32 * kTileStride * 4 + lane * kTileStride * 4);
        auto step = [&](int q) {    // columns c0 + q .. c0 + q + 3
            const float4 xv = lds_f4(cur + (uint32_t)(16 * ((q >> 2) ^ ((lane >> 1) & 3))));
            const uint32_t soff = (uint32_t)((c0 + q) * (int)sizeof(S));
#pragma unroll
            for (int k = 0; k < NS; k++) {
                const auto w = src4_at(src0 + (uint32_t)(k < ns ? k : 0) * sstride + soff, S());
                acc[k] = mac<FORM>(xv.x, w.x, acc[k]);
                acc[k] = mac<FORM>(xv.y, w.y, acc[k]);
                acc[k] = mac<FORM>(xv.z, w.z, acc[k]);
                acc[k] = mac<FORM>(xv.w, w.w, acc[k]);
            }
        };
        if (FORM == FORM_EXACT && ld - c0 >= 16) {
            // a whole slice, its four steps unrolled (the fp32 form keeps the
            // loop: eight float4 sources per step would not fit registers)
#pragma unroll
            for (int q = 0; q < 16; q += 4) step(q);
        } else {
            const int lim = ld - c0 < 16 ? ld - c0 : 16;    // multiple of 4
            for (int q = 0; q < lim; q += 4) step(q);
        }
        __syncwarp();
        s = s + 1 == nb ? 0 : s + 1;
    }
#pragma unroll
    for (int k = 0; k < NS; k++) out[k] = (double)acc[k];
}

// Evaluate the Q rows of `ns` (<= kPrefetchMax, <= stage_cap when staged)
// sources into cache slots on my chunk of [0,A) (tail = 0, from shared
// memory) or of [A,l) (tail = 1, global state).
template <int FORM, typename S>
__device__ __forceinline__ void tile_dots_ns(const InstanceDesc &D, const StageSlots &ss, int ns, int r, float *tile,
                                             double (&dots)[kPrefetchMax])
{
    switch (ns) {
    case 1: warp_tile_dots<FORM, 1, S>(D, ss, ns, r, tile, dots); break;
    case 2: warp_tile_dots<FORM, 2, S>(D, ss, ns, r, tile, dots); break;
    case 3: warp_tile_dots<FORM, 3, S>(D, ss, ns, r, tile, dots); break;
    case 4: warp_tile_dots<FORM, 4, S>(D, ss, ns, r, tile, dots); break;
    case 5: warp_tile_dots<FORM, 5, S>(D, ss, ns, r, tile, dots); break;
    case 6: warp_tile_dots<FORM, 6, S>(D, ss, ns, r, tile, dots); break;
    default: warp_tile_dots<FORM, 8, S>(D, ss, ns, r, tile, dots); break;
    }
}

template <int FORM>
__device__ void fill_rows(Ctx &c, Shared &sh, int ns, const int *src_row, const int *src_y, const long long *slot,
                          int tail)
{
    const InstanceDesc &D = *c.D;
    if (ns == 0) return;
    // per-source constants of this pass, read from shared memory where used
    if (threadIdx.x < ns) {
        const int k = threadIdx.x;
        sh.fsx[k] = D.x.xsq ? D.x.xsq[src_row[k]] : 0.0;
        sh.fsy[k] = src_y[k];
        sh.fsd[k] = D.cache.data + slot[k] * D.cache.stride;
    }
    stage_sources(D, c.stage, sh.ss, src_row, ns);   // ends with a barrier
    const int lo = tail ? c.t0 : 0, hi = tail ? c.t1 : c.a1 - c.a0;
    if (D.x.X && D.stage_cap > 0) {
        // dense rows, staged sources: warp-tiled, whole warps per 32 positions
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        float *tile = c.tile + warp * (D.tile_bufs * 32 * kTileStride);
        for (int base = lo + warp * 32; base < hi; base += blockDim.x) {
            const int k = base + lane;
            const bool valid = k < hi;
            const int kk = valid ? k : base;     // idle lanes repeat a valid row
            int r, yp, col;
            if (tail) {
                r = D.pos_row[kk];
                yp = D.y[kk];
                col = D.pos_local[kk];
            } else {
                r = c.sRow[kk];
                yp = c.sY[kk];
                col = c.sCol[kk];
            }
            // the target's norm is loaded before the dots so that its latency hides behind them
            const double xe = D.x.xsq ? D.x.xsq[r] : 0.0;
            double dots[kPrefetchMax];
            // staged sources are float64 in the exact form
            if (FORM == FORM_EXACT) tile_dots_ns<FORM, double>(D, sh.ss, ns, r, tile, dots);
            else tile_dots_ns<FORM, float>(D, sh.ss, ns, r, tile, dots);
            if (valid) {
#pragma unroll
                for (int s2 = 0; s2 < kPrefetchMax; s2++)
                    if (s2 < ns) sh.fsd[s2][col] = q_value(D.kp, sh.fsy[s2] * yp, dots[s2], sh.fsx[s2], xe);
            }
        }
    } else {
        for (int k = lo + threadIdx.x; k < hi; k += blockDim.x) {
            int r, yp, col;
            if (tail) {
                r = D.pos_row[k];
                yp = D.y[k];
                col = D.pos_local[k];
            } else {
                r = c.sRow[k];
                yp = c.sY[k];
                col = c.sCol[k];
            }
            double dots[kSrcBatch];
            row_dots<FORM>(D, sh.ss, ns, r, dots);
            const double xe = D.x.xsq ? D.x.xsq[r] : 0.0;
#pragma unroll
            for (int s2 = 0; s2 < kPrefetchMax; s2++)
                if (s2 < ns) sh.fsd[s2][col] = q_value(D.kp, sh.fsy[s2] * yp, dots[s2], sh.fsx[s2], xe);
        }
    }
    unstage_sources(D, c.stage, sh.ss);
}

// the fill pass of the form: CUDA cores or tensor cores
template <int FORM>
__device__ bool fill(Ctx &c, Shared &sh, int ns, const int *src_row, const int *src_y, const long long *slot, int tail)
{
    if constexpr (is_tc_form(FORM)) {
        return fill_rows_tc(c, sh, ns, src_row, src_y, slot, tail);
    } else {
        fill_rows<FORM>(c, sh, ns, src_row, src_y, slot, tail);
        return true;
    }
}

// position of the phase-A winner of track k (excluded from prefetching)
__device__ __forceinline__ int i0_prev_guard(const Shared &sh, int k) { return sh.bi[4 * k]; }

// --------------------------------------------------------------------------
// the persistent solver
// --------------------------------------------------------------------------
template <int FORM>
__device__ void solve_instance(const InstanceDesc &D, int rank, Shared &sh, unsigned char *dyn)
{
    Ctx c;
    c.D = &D;
    c.rank = rank;
    c.nb = D.nblocks;
    c.A = D.l;
    c.epoch = 0;
    c.phase = 0;
    c.lrec = sh.lrec;
    {
        // dynamic shared memory: [tensor-core stages][stage][tiles][G][alpha][QD][col][row][y][status]
        size_t off = 0;
        c.tcbase = 0;
        c.tc_g = 0;
        c.tc_t = 0;
        c.fg = 0;
        c.fstages = fill_stages(D.tc_n);
        if constexpr (is_tc_form(FORM)) {
            const uint32_t raw = tc::smem_addr(dyn);
            c.tcbase = (raw + 1023u) & ~1023u;
            off = (size_t)tc_area_bytes(D.tc_n);
        }
        c.stage = reinterpret_cast<float *>(dyn + off);
        off += (size_t)D.stage_cap * D.stage_lds * stage_elem(FORM);
        if (D.hash_slots > 0) off += (size_t)hash_bytes(FORM);
        off = (off + 15) & ~(size_t)15;
        c.tile = reinterpret_cast<float *>(dyn + off);
        c.pt = reinterpret_cast<PrefetchTable *>(dyn + off);
        off += aux_bytes(FORM, D.tile_bufs);
        const size_t cap = (size_t)D.chunk_cap;
        c.sG = reinterpret_cast<double *>(dyn + off); off += cap * 8;
        c.sA = reinterpret_cast<double *>(dyn + off); off += cap * 8;
        c.sQD = reinterpret_cast<double *>(dyn + off); off += cap * 8;
        c.sCol = reinterpret_cast<int *>(dyn + off); off += cap * 4;
        c.sRow = reinterpret_cast<int *>(dyn + off); off += cap * 4;
        c.sY = reinterpret_cast<signed char *>(dyn + off); off += cap;
        c.sS = reinterpret_cast<unsigned char *>(dyn + off);
    }
    set_chunks(c);
    const int l = D.l;
    const int nu = D.nu;
    long long iter = 0;
    int unshrink = 0;
    int status = 0;
    // block 0 / thread 0 work counters and section timers
    long long cnt_active = 0, cnt_q = 0, cnt_look = 0, cnt_hit = 0, cnt_fill = 0, cnt_pf = 0, cnt_pf_used = 0;
    long long cnt_tgt = 0;   // target positions of the fill passes (one row read each, whatever the sources)
    long long prof[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long tmark = clock64();
    const long long tstart = tmark;
#define SVMB_PROF(k)                                   \
    do {                                               \
        if (threadIdx.x == 0) {                        \
            const long long now_ = clock64();          \
            prof[k] += now_ - tmark;                   \
            tmark = now_;                              \
        }                                              \
    } while (0)
    if (threadIdx.x == 0) { sh.cs.nprev = 0; sh.cs.ncur = 0; }
    if (!D.x.X && D.stage_cap > 0)
        for (long long k = threadIdx.x; k < (long long)D.stage_lds * D.stage_cap * (stage_elem(FORM) / 4); k += blockDim.x)
            c.stage[k] = 0.0f;
    if (!D.x.X && D.hash_slots > 0) {
        // an empty table: keys -1, values zero
        int *keys = reinterpret_cast<int *>(c.stage);
        for (int k = threadIdx.x; k < kHashSlots; k += blockDim.x) keys[k] = -1;
        float *vals = reinterpret_cast<float *>(reinterpret_cast<char *>(c.stage) + kHashSlots * 4);
        for (int k = threadIdx.x; k < kHashSlots * kSrcBatch * (stage_elem(FORM) / 4); k += blockDim.x) vals[k] = 0.0f;
    }
    __syncthreads();

    // ---- initial state (svm.cpp:525-572, QD svm.cpp:1321-1327) on the global copies ----
    {
        for (int p = c.a0 + threadIdx.x; p < c.a1; p += blockDim.x) {
            D.pos_local[p] = p;      // positions start as local indices
            D.status[p] = status_of(D.alpha[p], get_C(D, D.y[p]));
            const int r = D.pos_row[p];
            const double xs = D.x.xsq ? D.x.xsq[r] : 0.0;
            // dot(x,x) in feature order is exactly what xsq holds
            D.QD[p] = kernel_from_dot(D.kp, xs, xs, xs);
            D.G[p] = D.p[p];
            D.G_bar[p] = 0.0;
        }
        if (!exchange(c, sh)) goto fail;
        int any = 0;
        for (int p = threadIdx.x; p < l; p += blockDim.x) any |= D.alpha[p] > 0 ? 1 : 0;
        any = __syncthreads_or(any);
        if (any) {
            if (!accumulate<FORM>(c, sh, l, 0, D.lazy_gbar ? 0 : 1, c.a0, c.a1)) goto fail;
            if (!exchange(c, sh)) goto fail;
        }
        chunk_load(c);
    }

    {
        const long long max_iter = D.max_iter;
        int counter = (l < 1000 ? l : 1000) + 1;
        scan_iup(c, sh);
        if (!exchange(c, sh)) goto fail;

        while (iter < max_iter) {
            if (--counter == 0) {
                counter = l < 1000 ? l : 1000;
                if (D.shrinking) {
                    SVMB_PROF(kProfBUpdate);
                    if (!do_shrinking<FORM>(c, sh, unshrink)) goto fail;
                    scan_iup(c, sh);
                    if (!exchange(c, sh)) goto fail;
                    SVMB_PROF(kProfShrink);
                }
            }
            int widened = 0;
            double Gmax0, Gmax1;
            int i0, i1;
        select_again:
            // ======================= phase A =======================
            const unsigned long long clkA = 4ull * (unsigned long long)iter + 1ull + (unsigned long long)widened;
            {
                const Partial *all = prev_partials(c);
                double v[2] = {-SVMB_INF, -SVMB_INF};
                int ix[2] = {-1, -1};
                const int kind[2] = {0, 0};
                RecVals r;
                r.n[0] = r.n[4] = -1;
                if (D.prefetch > 1) {
                    // the group's prefetch candidates into shared memory, one
                    // candidate per thread (its five fields loaded together)
                    const int ncand = c.nb * kPrefetchCand;
                    for (int e = threadIdx.x; e < ncand; e += blockDim.x) {
                        const Partial *pr = &all[e / kPrefetchCand];
                        const int t = e % kPrefetchCand;
                        double cv;
                        int cpos, cloc, crow, cy;
                        if (c.nb == 1) {
                            cv = pr->cv[t]; cpos = pr->cpos[t]; cloc = pr->cloc[t]; crow = pr->crow[t]; cy = pr->cy[t];
                        } else {
                            cv = __ldcg(&pr->cv[t]); cpos = __ldcg(&pr->cpos[t]); cloc = __ldcg(&pr->cloc[t]);
                            crow = __ldcg(&pr->crow[t]); cy = __ldcg(&pr->cy[t]);
                        }
                        c.pt->v[e] = cv; c.pt->pos[e] = cpos; c.pt->loc[e] = cloc; c.pt->row[e] = crow; c.pt->y[e] = cy;
                    }
                }
                if (threadIdx.x < c.nb) {
                    rec_load(c, &all[threadIdx.x], r, 1, 0);
                    better_max(v[0], ix[0], r.v[0], r.n[0]);
                    better_max(v[1], ix[1], r.v[3], r.n[4]);
                }
                block_reduce<2>(sh.red, v, ix, kind);
                // the thread holding a winning record publishes its payload
                if (threadIdx.x < c.nb) {
                    for (int k = 0; k < 2; k++) {
                        if (ix[k] >= 0 && r.n[4 * k] == ix[k]) {
                            sh.bd[3 * k + 1] = r.v[3 * k + 1];
                            sh.bd[3 * k + 2] = r.v[3 * k + 2];
                            sh.bi[4 * k + 1] = r.n[4 * k + 1];
                            sh.bi[4 * k + 2] = r.n[4 * k + 2];
                            sh.bi[4 * k + 3] = r.n[4 * k + 3];
                        }
                    }
                }
                if (threadIdx.x == 0) {
                    sh.bd[0] = v[0]; sh.bi[0] = ix[0];
                    sh.bd[3] = v[1]; sh.bi[4] = ix[1];
                }
                __syncthreads();
                if (threadIdx.x < 32) {
                    // cache decisions for the row(s) of phase A (warp 0 together; lane 0
                    // writes them); missing rows go to the fill list
                    const int whole = c.A == l;
                    int nf = 0;
                    for (int k = 0; k < 2; k++) {
                        long long slot = -1;
                        int va = 1;
                        if (sh.bi[4 * k] >= 0 && (k == 0 || nu)) {
                            const Lookup L = cache_lookup_w(sh.cs, D.cache, sh.bi[4 * k + 1], c.epoch, clkA, whole, clkA, 0);
                            slot = L.slot;
                            va = L.valid_active;
                            cnt_look++;
                            cnt_hit += L.valid_active;
                            cnt_pf_used += L.was_prefetched;
                            if (!va && threadIdx.x == 0) {
                                sh.frow[nf] = sh.bi[4 * k + 2];
                                sh.fy[nf] = sh.bi[4 * k + 3];
                                sh.fslot[nf] = slot;
                            }
                            if (!va) nf++;
                        }
                        if (threadIdx.x == 0) {
                            sh.bl[k] = slot;
                            sh.bi[8 + k] = va;
                        }
                    }
                    if (threadIdx.x == 0) sh.nfill = nf;
                }
                __syncthreads();
                // speculative prefetch: a missing row is evaluated together with
                // the rows of the group's most violating positions (this only
                // fills the cache; it never changes which pair is chosen)
                if (sh.nfill > 0 && D.prefetch > sh.nfill) {
                    // the `want` highest-priority candidates, chosen by warp 0: every
                    // lane keeps its own best few, then the lanes' heads are merged
                    // (the order of prefetched rows affects only what is cached)
                    const int ncand = c.nb * kPrefetchCand;
                    const int want = D.prefetch - sh.nfill;
                    if (threadIdx.x < 32) {
                        // `want` rounds of a warp argmax over the candidates
                        // (largest priority, the lowest table index on ties); lane
                        // L owns entries L + 32j and marks the ones taken in a mask
                        const int lane = threadIdx.x;
                        const int g0 = i0_prev_guard(sh, 0), g1 = i0_prev_guard(sh, 1);
                        unsigned taken = 0;
                        int got = 0;
                        for (; got < want; got++) {
                            double bv = -SVMB_INF;
                            int be = 0x7fffffff;
                            for (int e = lane, j = 0; e < ncand; e += 32, j++) {
                                if ((taken >> j) & 1u) continue;
                                const int pos = c.pt->pos[e];
                                const double v = c.pt->v[e];
                                if (pos < 0 || pos == g0 || pos == g1 || !(v > -SVMB_INF)) continue;
                                if (v > bv) { bv = v; be = e; }
                            }
                            for (int o = 16; o > 0; o >>= 1) {
                                const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
                                const int oe = __shfl_xor_sync(0xffffffffu, be, o);
                                if (ov > bv || (ov == bv && oe < be)) { bv = ov; be = oe; }
                            }
                            if (be == 0x7fffffff) break;
                            if ((be & 31) == lane) taken |= 1u << (be >> 5);
                            if (lane == 0) sh.pick[got] = be;
                        }
                        if (lane == 0) sh.npick = got;
                    }
                    __syncthreads();
                    // the picks' cache sets, read by one thread per way in a single round trip
                    if (threadIdx.x < sh.npick * kMaxWays) {
                        const int t = threadIdx.x / kMaxWays, w = threadIdx.x % kMaxWays;
                        const int set = c.pt->loc[sh.pick[t]] % D.cache.nsets;
                        if (w == 0) sh.sset[t].set = set;
                        if (w < D.cache.nways) {
                            const long long s = (long long)set * D.cache.nways + w;
                            sh.sset[t].tag[w] = __ldcg(&D.cache.tag[s]);
                            sh.sset[t].ep[w] = __ldcg(&D.cache.epoch[s]);
                            sh.sset[t].st[w] = __ldcg(&D.cache.stamp[s]);
                        }
                    }
                    __syncthreads();
                    if (threadIdx.x < 32) {
                        const int whole = c.A == l;
                        int nf = sh.nfill;
                        const int npick = sh.npick;
                        for (int t = 0; t < npick && nf < D.prefetch; t++) {
                            const int e = sh.pick[t];
                            const Lookup L = cache_lookup_w(sh.cs, D.cache, c.pt->loc[e], c.epoch, clkA, whole, clkA, 1,
                                                            &sh.sset[t]);
                            if (L.slot >= 0 && !L.valid_active) {
                                if (threadIdx.x == 0) {
                                    sh.frow[nf] = c.pt->row[e];
                                    sh.fy[nf] = c.pt->y[e];
                                    sh.fslot[nf] = L.slot;
                                }
                                nf++;
                                cnt_pf++;
                            }
                        }
                        __syncwarp();
                        if (threadIdx.x == 0) sh.nfill = nf;
                    }
                    __syncthreads();
                }
            }
            Gmax0 = sh.bd[0];
            Gmax1 = sh.bd[3];
            i0 = sh.bi[0];
            i1 = nu ? sh.bi[4] : -1;
            {
                // evaluate the missing (and prefetched) rows on my chunk
                const int ns = sh.nfill;
                SVMB_PROF(kProfAReduce);
                if (ns > 0) {
                    if (!fill<FORM>(c, sh, ns, sh.frow, sh.fy, sh.fslot, 0)) goto fail;
                    cnt_q += (long long)ns * c.A;
                    cnt_tgt += c.A;
                    cnt_fill++;
                }
                SVMB_PROF(kProfAFill);
            }
            {
                // second-order j scan on my chunk (svm.cpp:869-924 / :1120-1174)
                double v[3] = {SVMB_INF, -SVMB_INF, -SVMB_INF};   // obj_min, Gmax2 (C-SVC / nu p), Gmax2 (nu n)
                int ix[3] = {-1, -1, -1};
                const int kind[3] = {1, 2, 2};
                const float *Qi0 = i0 >= 0 ? D.cache.data + sh.bl[0] * D.cache.stride : nullptr;
                const float *Qi1 = i1 >= 0 ? D.cache.data + sh.bl[1] * D.cache.stride : nullptr;
                const double QDi0 = sh.bd[2], QDi1 = sh.bd[5];
                const double two_yi0 = __dmul_rn(2.0, (double)sh.bi[3]);
                const int n = c.a1 - c.a0;
                // kScanGroup positions per thread at a time: their Q_i values are
                // loaded together (one L2 round trip per group, not per position)
                for (int k0 = threadIdx.x; k0 < n; k0 += kScanGroup * blockDim.x) {
                    float qv[kScanGroup];
#pragma unroll
                    for (int u = 0; u < kScanGroup; u++) {
                        const int k = k0 + u * (int)blockDim.x;
                        qv[u] = 0.0f;
                        if (k < n) {
                            const float *Qr = (nu && c.sY[k] != +1) ? Qi1 : Qi0;
                            if (Qr) qv[u] = Qr[c.sCol[k]];
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kScanGroup; u++) {
                        const int k = k0 + u * (int)blockDim.x;
                        if (k >= n) continue;
                        const unsigned char s = c.sS[k];
                        const double G = c.sG[k];
                        if (c.sY[k] == +1) {
                            if (s != ST_LOWER) {
                                const double grad_diff = __dadd_rn(Gmax0, G);
                                v[1] = fmax(v[1], G);
                                if (grad_diff > 0) {
                                    double quad;
                                    if (!nu) quad = __dsub_rn(__dadd_rn(QDi0, c.sQD[k]), __dmul_rn(two_yi0, (double)qv[u]));
                                    else quad = __dsub_rn(__dadd_rn(QDi0, c.sQD[k]), (double)__fmul_rn(2.0f, qv[u]));
                                    const double num = __dmul_rn(grad_diff, grad_diff);
                                    const double od = quad > 0 ? -__ddiv_rn(num, quad) : -__ddiv_rn(num, kTau);
                                    better_min(v[0], ix[0], od, c.a0 + k);
                                }
                            }
                        } else {
                            if (s != ST_UPPER) {
                                const double grad_diff = __dsub_rn(nu ? Gmax1 : Gmax0, G);
                                if (nu) v[2] = fmax(v[2], -G); else v[1] = fmax(v[1], -G);
                                if (grad_diff > 0) {
                                    double quad;
                                    if (!nu) quad = __dadd_rn(__dadd_rn(QDi0, c.sQD[k]), __dmul_rn(two_yi0, (double)qv[u]));
                                    else quad = __dsub_rn(__dadd_rn(QDi1, c.sQD[k]), (double)__fmul_rn(2.0f, qv[u]));
                                    const double num = __dmul_rn(grad_diff, grad_diff);
                                    const double od = quad > 0 ? -__ddiv_rn(num, quad) : -__ddiv_rn(num, kTau);
                                    better_min(v[0], ix[0], od, c.a0 + k);
                                }
                            }
                        }
                    }
                }
                block_reduce<3>(sh.red, v, ix, kind);
                if (threadIdx.x == 0) {
                    Partial *pp = my_partial(c);
                    const int j = ix[0];
                    pp->v[0] = v[0]; pp->n[0] = j;
                    pp->v[1] = v[1]; pp->v[2] = v[2];
                    if (j >= 0) {
                        const int q = j - c.a0;
                        const int cj = c.sCol[q];
                        pp->v[3] = c.sG[q]; pp->v[4] = c.sA[q]; pp->v[5] = c.sQD[q];
                        pp->n[1] = cj; pp->n[2] = c.sRow[q]; pp->n[3] = c.sY[q];
                        pp->q[0] = Qi0 ? Qi0[cj] : 0.0f;
                        pp->q[1] = Qi1 ? Qi1[cj] : 0.0f;
                    }
                }
            }
            if (!exchange(c, sh)) goto fail;
            SVMB_PROF(kProfAScan);

            // ======================= phase B =======================
            {
                const Partial *all = prev_partials(c);
                double v[3] = {SVMB_INF, -SVMB_INF, -SVMB_INF};
                int ix[3] = {-1, -1, -1};
                const int kind[3] = {1, 2, 2};
                RecVals r;
                r.n[0] = -1;
                if (threadIdx.x < c.nb) {
                    rec_load(c, &all[threadIdx.x], r, 0, 1);
                    better_min(v[0], ix[0], r.v[0], r.n[0]);
                    v[1] = r.v[1];
                    v[2] = r.v[2];
                }
                block_reduce<3>(sh.red, v, ix, kind);
                if (threadIdx.x < c.nb && ix[0] >= 0 && r.n[0] == ix[0]) {
                    sh.bd[14] = r.v[3]; sh.bd[15] = r.v[4]; sh.bd[16] = r.v[5];
                    sh.bi[13] = r.n[1]; sh.bi[14] = r.n[2]; sh.bi[15] = r.n[3];
                    sh.bd[17] = (double)r.q[0]; sh.bd[18] = (double)r.q[1];
                }
                if (threadIdx.x == 0) { sh.bi[12] = ix[0]; sh.bd[12] = v[1]; sh.bd[13] = v[2]; }
                __syncthreads();
            }
            const int j = sh.bi[12];
            {
                bool stop;
                if (!nu) stop = __dadd_rn(Gmax0, sh.bd[12]) < D.eps;
                else stop = fmax(__dadd_rn(Gmax0, sh.bd[12]), __dadd_rn(Gmax1, sh.bd[13])) < D.eps;
                if (stop || j < 0) {
                    if (widened) break;
                    // reconstruct the whole gradient, widen, select again (svm.cpp:598-611)
                    if (c.A < l) {
                        chunk_store(c);
                        if (!exchange(c, sh)) goto fail;
                        if (!reconstruct<FORM>(c, sh)) goto fail;
                        widen(c);
                    }
                    widened = 1;
                    scan_iup(c, sh);
                    if (!exchange(c, sh)) goto fail;
                    goto select_again;
                }
                if (widened) counter = 1;
            }
            ++iter;
            cnt_active += c.A;
            // the working pair; nu-SVC takes i from the track of y_j (svm.cpp:1179-1182)
            const int yj = sh.bi[15];
            const int tr = (nu && yj != +1) ? 1 : 0;
            const int i = tr ? i1 : i0;
            const double Gi = tr ? Gmax1 : ((sh.bi[3] == +1) ? -Gmax0 : Gmax0);
            const double alpha_i = sh.bd[3 * tr + 1], QDi = sh.bd[3 * tr + 2];
            const int yi = tr ? -1 : sh.bi[3];
            const int loc_i = sh.bi[4 * tr + 1], row_i = sh.bi[4 * tr + 2];
            const long long slot_i = sh.bl[tr];
            const float Qij = (float)sh.bd[17 + tr];
            const double Gj = sh.bd[14], alpha_j = sh.bd[15], QDj = sh.bd[16];
            const int loc_j = sh.bi[13], row_j = sh.bi[14];
            // Q_j row
            // phase-B stamp: above every phase-A stamp of this iteration, below the next
            const unsigned long long clkB = 4ull * (unsigned long long)iter - 1ull;
            if (threadIdx.x < 32) {
                const Lookup L = cache_lookup_w(sh.cs, D.cache, loc_j, c.epoch, clkB, c.A == l, clkA, 0);
                if (threadIdx.x == 0) {
                    sh.bl[2] = L.slot;
                    sh.bi[16] = L.valid_active;
                }
                cnt_look++;
                cnt_hit += L.valid_active;
                cnt_pf_used += L.was_prefetched;
            }
            __syncthreads();
            SVMB_PROF(kProfBReduce);
            const long long slot_j = sh.bl[2];
            if (!sh.bi[16]) {
                const int srow[1] = {row_j};
                const int sy[1] = {yj};
                const long long ss[1] = {slot_j};
                if (!fill<FORM>(c, sh, 1, srow, sy, ss, 0)) goto fail;
                cnt_q += c.A;
                cnt_tgt += c.A;
                cnt_fill++;
            }
            // two-variable analytic step (svm.cpp:636-721), identical in every block
            const double C_i = get_C(D, yi), C_j = get_C(D, yj);
            double ai = alpha_i, aj = alpha_j;
            if (yi != yj) {
                double quad_coef = __dadd_rn(__dadd_rn(QDi, QDj), (double)__fmul_rn(2.0f, Qij));
                if (quad_coef <= 0) quad_coef = kTau;
                const double delta = __ddiv_rn(__dsub_rn(-Gi, Gj), quad_coef);
                const double diff = __dsub_rn(ai, aj);
                ai = __dadd_rn(ai, delta);
                aj = __dadd_rn(aj, delta);
                if (diff > 0) {
                    if (aj < 0) { aj = 0; ai = diff; }
                } else {
                    if (ai < 0) { ai = 0; aj = -diff; }
                }
                if (diff > __dsub_rn(C_i, C_j)) {
                    if (ai > C_i) { ai = C_i; aj = __dsub_rn(C_i, diff); }
                } else {
                    if (aj > C_j) { aj = C_j; ai = __dadd_rn(C_j, diff); }
                }
            } else {
                double quad_coef = __dsub_rn(__dadd_rn(QDi, QDj), (double)__fmul_rn(2.0f, Qij));
                if (quad_coef <= 0) quad_coef = kTau;
                const double delta = __ddiv_rn(__dsub_rn(Gi, Gj), quad_coef);
                const double sum = __dadd_rn(ai, aj);
                ai = __dsub_rn(ai, delta);
                aj = __dadd_rn(aj, delta);
                if (sum > C_i) {
                    if (ai > C_i) { ai = C_i; aj = __dsub_rn(sum, C_i); }
                } else {
                    if (aj < 0) { aj = 0; ai = sum; }
                }
                if (sum > C_j) {
                    if (aj > C_j) { aj = C_j; ai = __dsub_rn(sum, C_j); }
                } else {
                    if (ai < 0) { ai = 0; aj = sum; }
                }
            }
            const double dai = __dsub_rn(ai, alpha_i);
            const double daj = __dsub_rn(aj, alpha_j);
            const unsigned char old_si = status_of(alpha_i, C_i), old_sj = status_of(alpha_j, C_j);
            const unsigned char new_si = status_of(ai, C_i), new_sj = status_of(aj, C_j);
            const bool bar_i = !D.lazy_gbar && (old_si == ST_UPPER) != (new_si == ST_UPPER);
            const bool bar_j = !D.lazy_gbar && (old_sj == ST_UPPER) != (new_sj == ST_UPPER);
            // complete rows for the G_bar update: fill the tail [A,l) where missing
            if ((bar_i || bar_j) && c.A < l) {
                if (threadIdx.x == 0) {
                    const unsigned long long clk = clkB;
                    int tg[kMaxWays], ep[kMaxWays];
                    unsigned long long stp[kMaxWays];
                    sh.bi[17] = 0;
                    sh.bi[18] = 0;
                    if (bar_i) {
                        cache_read_set(sh.cs, D.cache, (int)(slot_i / D.cache.nways), tg, ep, stp);
                        sh.bi[17] = ep[slot_i % D.cache.nways] != kEpochFull;
                        cache_mark_full(sh.cs, D.cache, slot_i, loc_i, clk);
                    }
                    if (bar_j) {
                        cache_read_set(sh.cs, D.cache, (int)(slot_j / D.cache.nways), tg, ep, stp);
                        sh.bi[18] = ep[slot_j % D.cache.nways] != kEpochFull;
                        cache_mark_full(sh.cs, D.cache, slot_j, loc_j, clk);
                    }
                }
                __syncthreads();
                int ns = 0;
                int srow[2] = {0, 0}, sy[2] = {0, 0};
                long long sslot[2] = {0, 0};
                if (sh.bi[17]) { srow[ns] = row_i; sy[ns] = yi; sslot[ns] = slot_i; ns++; }
                if (sh.bi[18]) { srow[ns] = row_j; sy[ns] = yj; sslot[ns] = slot_j; ns++; }
                if (!fill<FORM>(c, sh, ns, srow, sy, sslot, 1)) goto fail;
                cnt_q += (long long)ns * (l - c.A);
                cnt_tgt += l - c.A;
            }
            SVMB_PROF(kProfBFill);
            // owners publish alpha/status of i and j
            if (threadIdx.x == 0) {
                if (i >= c.a0 && i < c.a1) { c.sA[i - c.a0] = ai; c.sS[i - c.a0] = new_si; }
                if (j >= c.a0 && j < c.a1) { c.sA[j - c.a0] = aj; c.sS[j - c.a0] = new_sj; }
            }
            __syncthreads();
            // G update on my chunk (svm.cpp:732-735) + G_bar (svm.cpp:744-769) + next I_up scan
            {
                const float *Qi = D.cache.data + slot_i * D.cache.stride;
                const float *Qj = D.cache.data + slot_j * D.cache.stride;
                double v[2] = {-SVMB_INF, -SVMB_INF};
                int ix[2] = {-1, -1};
                double pv = -SVMB_INF;
                int pix = -1;
                const int n = c.a1 - c.a0;
                const bool gbar = bar_i || bar_j;
                // kScanGroup positions per thread at a time, their Q_i, Q_j (and
                // G_bar) values loaded together before any is used
                for (int k0 = threadIdx.x; k0 < n; k0 += kScanGroup * blockDim.x) {
                    float qi[kScanGroup], qj[kScanGroup];
                    double gb[kScanGroup];
#pragma unroll
                    for (int u = 0; u < kScanGroup; u++) {
                        const int k = k0 + u * (int)blockDim.x;
                        qi[u] = 0.0f;
                        qj[u] = 0.0f;
                        gb[u] = 0.0;
                        if (k < n) {
                            const int col = c.sCol[k];
                            qi[u] = Qi[col];
                            qj[u] = Qj[col];
                            if (gbar) gb[u] = D.G_bar[c.a0 + k];
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kScanGroup; u++) {
                        const int k = k0 + u * (int)blockDim.x;
                        if (k >= n) continue;
                        const double G = __dadd_rn(c.sG[k], __dadd_rn(__dmul_rn((double)qi[u], dai), __dmul_rn((double)qj[u], daj)));
                        c.sG[k] = G;
                        if (gbar) {
                            double g = gb[u];
                            if (bar_i) g = (old_si == ST_UPPER) ? __dsub_rn(g, __dmul_rn(C_i, (double)qi[u])) : __dadd_rn(g, __dmul_rn(C_i, (double)qi[u]));
                            if (bar_j) g = (old_sj == ST_UPPER) ? __dsub_rn(g, __dmul_rn(C_j, (double)qj[u])) : __dadd_rn(g, __dmul_rn(C_j, (double)qj[u]));
                            D.G_bar[c.a0 + k] = g;
                        }
                        const unsigned char s = c.sS[k];
                        if (c.sY[k] == +1) {
                            if (s != ST_UPPER) better_max(v[0], ix[0], -G, c.a0 + k);
                        } else {
                            if (s != ST_LOWER) better_max(v[nu], ix[nu], G, c.a0 + k);
                        }
                        better_max(pv, pix, prefetch_priority(c.sY[k], s, G), c.a0 + k);
                    }
                }
                if (bar_i || bar_j) {
                    for (int p = c.t0 + threadIdx.x; p < c.t1; p += blockDim.x) {
                        const int col = D.pos_local[p];
                        double gb = D.G_bar[p];
                        if (bar_i) { const double q = (double)Qi[col]; gb = (old_si == ST_UPPER) ? __dsub_rn(gb, __dmul_rn(C_i, q)) : __dadd_rn(gb, __dmul_rn(C_i, q)); }
                        if (bar_j) { const double q = (double)Qj[col]; gb = (old_sj == ST_UPPER) ? __dsub_rn(gb, __dmul_rn(C_j, q)) : __dadd_rn(gb, __dmul_rn(C_j, q)); }
                        D.G_bar[p] = gb;
                    }
                }
                iup_publish(c, sh, v, ix, pv, pix);
            }
            if (!exchange(c, sh)) goto fail;
            SVMB_PROF(kProfBUpdate);
        }

        chunk_store(c);
        if (!exchange(c, sh)) goto fail;
        if (iter >= max_iter) {
            status = 1;
            if (c.A < l) {
                if (!reconstruct<FORM>(c, sh)) goto fail;
                c.A = l;
                set_chunks(c);
            }
        }
    }
    // ---- rho (svm.cpp:1013-1049 / 1260-1308), objective (:795-802), alpha out (:805-808) ----
    // The sums run sequentially in position order (bit-exact with the reference), on block 0.
    if (rank == 0) {
        __shared__ double chv[kThreads], chg[kThreads];
        __shared__ unsigned char chs[kThreads];
        __shared__ signed char chy[kThreads];
        double ub = SVMB_INF, lb = -SVMB_INF, sum_free = 0;
        int nr_free = 0;
        double ub1 = SVMB_INF, ub2 = SVMB_INF, lb1 = -SVMB_INF, lb2 = -SVMB_INF, sf1 = 0, sf2 = 0;
        int nf1 = 0, nf2 = 0;
        double objv = 0;
        const int A = c.A;
        for (int base = 0; base < l; base += blockDim.x) {
            const int p = base + threadIdx.x;
            if (p < l) {
                chs[threadIdx.x] = D.status[p];
                chy[threadIdx.x] = D.y[p];
                chg[threadIdx.x] = D.G[p];
                chv[threadIdx.x] = __dmul_rn(D.alpha[p], __dadd_rn(D.G[p], D.p[p]));
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                const int lim = l - base < (int)blockDim.x ? l - base : (int)blockDim.x;
                for (int k = 0; k < lim; k++) {
                    objv = __dadd_rn(objv, chv[k]);
                    if (base + k >= A) continue;
                    const unsigned char s = chs[k];
                    const int y = chy[k];
                    const double G = chg[k];
                    if (!nu) {
                        const double yG = __dmul_rn((double)y, G);
                        if (s == ST_UPPER) { if (y == -1) ub = fmin(ub, yG); else lb = fmax(lb, yG); }
                        else if (s == ST_LOWER) { if (y == +1) ub = fmin(ub, yG); else lb = fmax(lb, yG); }
                        else { ++nr_free; sum_free = __dadd_rn(sum_free, yG); }
                    } else {
                        if (y == +1) {
                            if (s == ST_UPPER) lb1 = fmax(lb1, G);
                            else if (s == ST_LOWER) ub1 = fmin(ub1, G);
                            else { ++nf1; sf1 = __dadd_rn(sf1, G); }
                        } else {
                            if (s == ST_UPPER) lb2 = fmax(lb2, G);
                            else if (s == ST_LOWER) ub2 = fmin(ub2, G);
                            else { ++nf2; sf2 = __dadd_rn(sf2, G); }
                        }
                    }
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            SolveOut o;
            o.iters = iter;
            o.status = status;
            o.active_size = c.A;
            o.unshrink = unshrink;
            o.obj = __ddiv_rn(objv, 2.0);
            o.gap = 0;
            o.sum_active = cnt_active;
            o.q_evals = cnt_q;
            o.lookups = cnt_look;
            o.hits = cnt_hit;
            o.fills = cnt_fill;
            o.prefetched = cnt_pf;
            o.prefetch_used = cnt_pf_used;
            o.fill_targets = cnt_tgt;
            for (int k = 0; k < 7; k++) o.prof[k] = prof[k];
            o.prof[kProfTotal] = clock64() - tstart;
            if (!nu) {
                o.rho = nr_free > 0 ? __ddiv_rn(sum_free, (double)nr_free) : __ddiv_rn(__dadd_rn(ub, lb), 2.0);
                o.r = 0;
                o.nr_free = nr_free;
            } else {
                const double r1 = nf1 > 0 ? __ddiv_rn(sf1, (double)nf1) : __ddiv_rn(__dadd_rn(ub1, lb1), 2.0);
                const double r2 = nf2 > 0 ? __ddiv_rn(sf2, (double)nf2) : __ddiv_rn(__dadd_rn(ub2, lb2), 2.0);
                o.r = __ddiv_rn(__dadd_rn(r1, r2), 2.0);
                o.rho = __ddiv_rn(__dsub_rn(r1, r2), 2.0);
                o.nr_free = nf1 + nf2;
            }
            *D.out = o;
        }
    }
    {
        const int lo = (int)((long long)l * rank / c.nb), hi = (int)((long long)l * (rank + 1) / c.nb);
        for (int p = lo + threadIdx.x; p < hi; p += blockDim.x) D.alpha_local[D.pos_local[p]] = D.alpha[p];
    }
    return;
fail:
    if (threadIdx.x == 0 && rank == 0) {
        SolveOut o;
        o.iters = iter; o.rho = 0; o.obj = 0; o.r = 0; o.status = -1; o.active_size = c.A;
        o.unshrink = unshrink; o.nr_free = 0; o.gap = 0;
        o.sum_active = cnt_active; o.q_evals = cnt_q; o.lookups = cnt_look; o.hits = cnt_hit;
        o.fills = cnt_fill; o.prefetched = cnt_pf; o.prefetch_used = cnt_pf_used; o.fill_targets = cnt_tgt;
        for (int k = 0; k < 8; k++) o.prof[k] = prof[k];
        *D.out = o;
    }
#undef SVMB_PROF
}

// Tell the host, through a word of mapped host memory, that every block of the
// instance has written its results (a request loop collects the instance and
// reuses its SMs while the rest of the launch runs on).
__device__ void signal_done(const InstanceDesc &D)
{
    if (!D.done_flag) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence_system();
        if (atomicAdd(&D.sync->finished, 1u) == (unsigned)D.nblocks - 1u) {
            __threadfence_system();
            *(volatile int *)D.done_flag = 1;
        }
    }
}

template <int FORM>
__global__ void __launch_bounds__(kThreads, 1)
smo_persistent(const InstanceDesc *__restrict__ insts, const int *__restrict__ block_inst)
{
    __shared__ Shared sh;
    extern __shared__ __align__(16) unsigned char dyn[];
    const int inst = block_inst[blockIdx.x];
    const InstanceDesc &D = insts[inst];
    const int rank = blockIdx.x - D.block0;
    if constexpr (is_tc_form(FORM)) {
        // mbarriers of the tensor-core pipeline and the TMEM accumulator (one block per SM)
        if (threadIdx.x == 0) {
            for (int k = 0; k < kTcStages; k++) tc::mbar_init(&sh.tbar[k], 1);
            for (int k = 0; k < kFillStagesMax; k++) {
                tc::mbar_init(&sh.ffull[k], kThreads - kFillLoad0 * 32);
                tc::mbar_init(&sh.fempty[k], 1);
            }
            for (int k = 0; k < kFillAcc; k++) {
                tc::mbar_init(&sh.faccf[k], 1);
                tc::mbar_init(&sh.facce[k], kTcM);
            }
            sh.fabort = 0;
            tc::mbar_init_fence();
        }
        if (threadIdx.x < 32) {
            tc::tmem_alloc(&sh.tmem, 2 * kTcMaxN);
            tc::tmem_relinquish();
        }
        tc::tc_fence_before();
        __syncthreads();
        tc::tc_fence_after();
    }
    solve_instance<FORM>(D, rank, sh, dyn);
    signal_done(D);
    if constexpr (is_tc_form(FORM)) {
        tc::tc_fence_before();
        __syncthreads();
        if (threadIdx.x < 32) tc::tmem_dealloc(sh.tmem, 2 * kTcMaxN);
    }
}

}  // namespace
}  // namespace svmb
