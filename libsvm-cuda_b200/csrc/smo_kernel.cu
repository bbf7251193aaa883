// smo_kernel.cu -- device-resident SMO solver for C-SVC and nu-SVC.
//
// One persistent launch runs the whole solve of one or more instances (each a
// binary subproblem).  Every instance is owned by a group of `nblocks` thread
// blocks; block `rank` of the group owns a contiguous chunk of the active
// positions [0, A) and a chunk of the inactive tail [A, l).  Per SMO iteration
// there are exactly two group barriers:
//
//   phase A  reduce the per-block I_up maxima  -> working index i (and, for
//            nu-SVC, the two track maxima ip/in), look up / evaluate the Q row(s)
//            for the block's chunk, scan the chunk for the second-order j
//            candidate (WSS3, reference svm.cpp:833-930 / :1076-1186)
//   --- barrier ---
//   phase B  reduce the j candidates, stopping test, look up / evaluate Q_j,
//            two-variable analytic step with box clipping (svm.cpp:636-721,
//            computed redundantly and identically by every block), gradient
//            update G += dQ (svm.cpp:729-735) and G_bar update (:744-769) on
//            the block's chunk, fused with the I_up scan for the next i
//   --- barrier ---
//
// Shrinking (svm.cpp:932-1011), unshrinking and gradient reconstruction
// (:473-513) and the initial gradient (:545-572) run inside the same launch as
// group-collective sections.  The position permutation of shrinking is the
// reference's (hole i paired with the last non-shrunk position), so
// position-based tie-breaks are identical.  All double arithmetic keeps the
// reference's operand order; the file is compiled with -fmad=false so that no
// multiply-add is contracted.
//
// Barriers are bounded: a wait that exceeds kBarrierTimeout cycles sets the
// group's error flag and every block of the group returns.
#include "engine.h"

#include <cuda_runtime.h>

#include <type_traits>

namespace svmb {

#define SVMB_INF __longlong_as_double(0x7ff0000000000000ULL)
constexpr double kTau = 1e-12;                       // reference svm.cpp:42
constexpr long long kBarrierTimeout = 60000000000LL; // ~30 s of SM clock

// --------------------------------------------------------------------------
// group barrier (sense by generation counter, bounded spin)
// --------------------------------------------------------------------------
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed_i32(const int *p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ bool group_barrier(GroupSync *s, int nblocks, int *okflag)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        int good = 1;
        if (nblocks > 1) {
            __threadfence();
            unsigned gen = ld_acquire_u32(&s->gen);
            unsigned arrived = atomicAdd(&s->count, 1u);
            if (arrived == (unsigned)(nblocks - 1)) {
                atomicExch(&s->count, 0u);
                __threadfence();
                atomicAdd(&s->gen, 1u);
            } else {
                long long t0 = clock64();
                while (ld_acquire_u32(&s->gen) == gen) {
                    if (ld_relaxed_i32(&s->error) != 0 || clock64() - t0 > kBarrierTimeout) {
                        atomicExch(&s->error, 1);
                        good = 0;
                        break;
                    }
                }
            }
            __threadfence();
        } else {
            __threadfence_block();
        }
        *okflag = good;
    }
    __syncthreads();
    return *okflag != 0;
}

// --------------------------------------------------------------------------
// kernel values (reference svm.cpp:30-40, 235-254), no contraction
// --------------------------------------------------------------------------
__device__ __forceinline__ double powi_d(double base, int times)
{
    double tmp = base, ret = 1.0;
    for (int t = times; t > 0; t /= 2) {
        if (t % 2 == 1) ret = __dmul_rn(ret, tmp);
        tmp = __dmul_rn(tmp, tmp);
    }
    return ret;
}

__device__ __forceinline__ double kernel_from_dot(const KernelParams &kp, double dot, double xsq_a, double xsq_b)
{
    switch (kp.type) {
    case 0: return dot;
    case 1: return powi_d(__dadd_rn(__dmul_rn(kp.gamma, dot), kp.coef0), kp.degree);
    case 2: return exp(__dmul_rn(-kp.gamma, __dsub_rn(__dadd_rn(xsq_a, xsq_b), __dmul_rn(2.0, dot))));
    case 3: return tanh(__dadd_rn(__dmul_rn(kp.gamma, dot), kp.coef0));
    default: return 0.0;
    }
}

// Q value exactly as the reference stores it: (Qfloat)(y_i*y_j*K)  (svm.cpp:1337)
__device__ __forceinline__ float q_value(const KernelParams &kp, int yy, double dot, double xsq_a, double xsq_b)
{
    return __double2float_rn(__dmul_rn((double)yy, kernel_from_dot(kp, dot, xsq_a, xsq_b)));
}

// --------------------------------------------------------------------------
// source-row staging and the row-block product
// --------------------------------------------------------------------------
// Sources of a row-block product are staged in dynamic shared memory when the
// instance's stage_cap > 0 (dense rows copied; sparse rows scattered into
// zeroed dense vectors), otherwise read from global memory (dense) or merged
// against the target's CSR row (sparse).  `sp[k]` points at source k.
struct StageSlots {
    const float *sp[kSrcBatch];
    int rows[kSrcBatch];
    int ns;
};

__device__ void stage_sources(const InstanceDesc &D, float *dyn, StageSlots &ss, const int *rows, int ns)
{
    const DevX &x = D.x;
    if (threadIdx.x < ns) ss.rows[threadIdx.x] = rows[threadIdx.x];
    if (threadIdx.x == 0) ss.ns = ns;
    if (x.X) {
        const int ld4 = x.ld >> 2;
        for (int k = 0; k < ns; k++) {
            const float4 *src = reinterpret_cast<const float4 *>(x.X + (long long)rows[k] * x.ld);
            if (D.stage_cap > 0) {
                float4 *dst = reinterpret_cast<float4 *>(dyn + (long long)k * D.stage_lds);
                for (int t = threadIdx.x; t < ld4; t += blockDim.x) dst[t] = __ldg(src + t);
                if (threadIdx.x == 0) ss.sp[k] = dyn + (long long)k * D.stage_lds;
            } else if (threadIdx.x == 0) {
                ss.sp[k] = x.X + (long long)rows[k] * x.ld;
            }
        }
    } else if (D.stage_cap > 0) {
        for (int k = 0; k < ns; k++) {
            long long a = x.rowptr[rows[k]], b = x.rowptr[rows[k] + 1];
            float *dst = dyn + (long long)k * D.stage_lds;
            for (long long e = a + threadIdx.x; e < b; e += blockDim.x) dst[x.col[e]] = x.val[e];
            if (threadIdx.x == 0) ss.sp[k] = dst;
        }
    }
    __syncthreads();
}

// Undo a sparse scatter so that the dense vectors are all-zero again.
__device__ void unstage_sources(const InstanceDesc &D, float *dyn, StageSlots &ss)
{
    __syncthreads();
    const DevX &x = D.x;
    if (!x.X && D.stage_cap > 0) {
        for (int k = 0; k < ss.ns; k++) {
            long long a = x.rowptr[ss.rows[k]], b = x.rowptr[ss.rows[k] + 1];
            float *dst = dyn + (long long)k * D.stage_lds;
            for (long long e = a + threadIdx.x; e < b; e += blockDim.x) dst[x.col[e]] = 0.0f;
        }
    }
    __syncthreads();
}

// Dot products of target row `r` with the staged sources, accumulated in
// feature order (the order of the reference's Kernel::dot, svm.cpp:305-325:
// only matching indices contribute; zero products leave the sum unchanged).
template <int FORM>
__device__ __forceinline__ void row_dots(const InstanceDesc &D, const StageSlots &ss, int ns, int r,
                                         double (&out)[kSrcBatch])
{
    const DevX &x = D.x;
    typedef typename std::conditional<FORM == FORM_EXACT, double, float>::type acc_t;
    acc_t acc[kSrcBatch];
#pragma unroll
    for (int k = 0; k < kSrcBatch; k++) acc[k] = acc_t(0);
    if (x.X) {
        const float4 *row = reinterpret_cast<const float4 *>(x.X + (long long)r * x.ld);
        const int ld4 = x.ld >> 2;
        for (int c = 0; c < ld4; c++) {
            const float4 v = __ldg(row + c);
#pragma unroll
            for (int k = 0; k < kSrcBatch; k++) {
                if (k < ns) {
                    const float4 w = reinterpret_cast<const float4 *>(ss.sp[k])[c];
                    if (FORM == FORM_EXACT) {
                        acc[k] = fma((double)v.x, (double)w.x, (double)acc[k]);
                        acc[k] = fma((double)v.y, (double)w.y, (double)acc[k]);
                        acc[k] = fma((double)v.z, (double)w.z, (double)acc[k]);
                        acc[k] = fma((double)v.w, (double)w.w, (double)acc[k]);
                    } else {
                        acc[k] = fmaf(v.x, w.x, (float)acc[k]);
                        acc[k] = fmaf(v.y, w.y, (float)acc[k]);
                        acc[k] = fmaf(v.z, w.z, (float)acc[k]);
                        acc[k] = fmaf(v.w, w.w, (float)acc[k]);
                    }
                }
            }
        }
    } else if (D.stage_cap > 0) {
        const long long a = x.rowptr[r], b = x.rowptr[r + 1];
        for (long long e = a; e < b; e++) {
            const int c = __ldg(x.col + e);
            const float v = __ldg(x.val + e);
#pragma unroll
            for (int k = 0; k < kSrcBatch; k++) {
                if (k < ns) {
                    if (FORM == FORM_EXACT) acc[k] = fma((double)v, (double)ss.sp[k][c], (double)acc[k]);
                    else acc[k] = fmaf(v, ss.sp[k][c], (float)acc[k]);
                }
            }
        }
    } else {
        // merge walk of two sorted index lists in global memory
        const long long a = x.rowptr[r], b = x.rowptr[r + 1];
        for (int k = 0; k < ns; k++) {
            const long long sa = x.rowptr[ss.rows[k]], sb = x.rowptr[ss.rows[k] + 1];
            long long e = a, f = sa;
            acc_t s = acc_t(0);
            while (e < b && f < sb) {
                const int ce = __ldg(x.col + e), cf = __ldg(x.col + f);
                if (ce == cf) {
                    if (FORM == FORM_EXACT) s = fma((double)__ldg(x.val + e), (double)__ldg(x.val + f), (double)s);
                    else s = fmaf(__ldg(x.val + e), __ldg(x.val + f), (float)s);
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
    for (int k = 0; k < kSrcBatch; k++) out[k] = (double)acc[k];
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
        double v2 = __shfl_xor_sync(0xffffffffu, v, o);
        int i2 = __shfl_xor_sync(0xffffffffu, i, o);
        better_max(v, i, v2, i2);
    }
}
__device__ __forceinline__ void warp_argmin(double &v, int &i)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double v2 = __shfl_xor_sync(0xffffffffu, v, o);
        int i2 = __shfl_xor_sync(0xffffffffu, i, o);
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

// Reduce up to 4 (value,index) pairs over the block.  kind[k]: 0 argmax, 1 argmin, 2 max (index ignored).
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
    if (w == 0) {
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
    __syncthreads();
}

__device__ int block_sum_i(RedScratch &s, int v)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_sum_i(v);
    __syncthreads();
    if (lane == 0) s.i[0][w] = v;
    __syncthreads();
    int tot = 0;
    for (int k = 0; k < kWarps; k++) tot += s.i[0][k];
    __syncthreads();
    return tot;
}

// exclusive prefix over the block of a 0/1 flag, in thread order; returns the
// prefix for this thread and the block total in *total.
__device__ int block_excl_scan(RedScratch &s, int flag, int *total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned bal = __ballot_sync(0xffffffffu, flag);
    int in_warp = __popc(bal & ((1u << lane) - 1u));
    __syncthreads();
    if (lane == 0) s.i[0][w] = __popc(bal);
    __syncthreads();
    int before = 0, tot = 0;
    for (int k = 0; k < kWarps; k++) {
        int c = s.i[0][k];
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
    CacheRec prev[6], cur[6];
    int nprev, ncur;
};

struct Lookup {
    long long slot;     // slot index
    int valid_active;   // positions [0,A) already valid
    int full;           // all positions valid
};

__device__ void cache_rotate(CacheState &cs, const CacheView &cv, int rank)
{
    // called by thread 0 right after a barrier: publish the previous phase's records
    if (rank == 0) {
        for (int k = 0; k < cs.ncur; k++) {
            const CacheRec &r = cs.cur[k];
            long long s = (long long)r.set * cv.nways + r.way;
            cv.tag[s] = r.tag;
            cv.epoch[s] = r.epoch;
            cv.stamp[s] = r.stamp;
        }
    }
    for (int k = 0; k < cs.ncur; k++) cs.prev[k] = cs.cur[k];
    cs.nprev = cs.ncur;
    cs.ncur = 0;
}

__device__ void cache_read_set(const CacheState &cs, const CacheView &cv, int set, int *tag, int *ep,
                               unsigned long long *st)
{
    for (int w = 0; w < cv.nways; w++) {
        long long s = (long long)set * cv.nways + w;
        tag[w] = *(volatile int *)&cv.tag[s];
        ep[w] = *(volatile int *)&cv.epoch[s];
        st[w] = *(volatile unsigned long long *)&cv.stamp[s];
    }
    for (int k = 0; k < cs.nprev; k++)
        if (cs.prev[k].set == set) { tag[cs.prev[k].way] = cs.prev[k].tag; ep[cs.prev[k].way] = cs.prev[k].epoch; st[cs.prev[k].way] = cs.prev[k].stamp; }
    for (int k = 0; k < cs.ncur; k++)
        if (cs.cur[k].set == set) { tag[cs.cur[k].way] = cs.cur[k].tag; ep[cs.cur[k].way] = cs.cur[k].epoch; st[cs.cur[k].way] = cs.cur[k].stamp; }
}

// Decide where row `local` lives; records the decision.  need_full: the caller
// will make the row complete (positions [0,l)).
__device__ Lookup cache_lookup(CacheState &cs, const CacheView &cv, int local, int cur_epoch,
                               unsigned long long clk, int need_full)
{
    int tag[kMaxWays], ep[kMaxWays];
    unsigned long long st[kMaxWays];
    const int set = local % cv.nsets;
    cache_read_set(cs, cv, set, tag, ep, st);
    int way = -1;
    for (int w = 0; w < cv.nways; w++)
        if (tag[w] == local) way = w;
    Lookup L;
    CacheRec rec;
    rec.set = set;
    rec.stamp = clk;
    rec.tag = local;
    if (way >= 0) {
        int full = ep[way] == kEpochFull;
        int va = full || ep[way] == cur_epoch;
        L.valid_active = va;
        L.full = full;
        rec.way = way;
        rec.epoch = need_full ? kEpochFull : (va ? ep[way] : cur_epoch);
    } else {
        int victim = -1;
        for (int w = 0; w < cv.nways; w++)
            if (tag[w] == kNoTag) { victim = w; break; }
        if (victim < 0) {
            victim = 0;
            for (int w = 1; w < cv.nways; w++)
                if (st[w] < st[victim]) victim = w;
        }
        L.valid_active = 0;
        L.full = 0;
        rec.way = victim;
        rec.epoch = need_full ? kEpochFull : cur_epoch;
        way = victim;
    }
    L.slot = (long long)set * cv.nways + way;
    cs.cur[cs.ncur++] = rec;
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
    int okflag;
    double bd[24];
    int bi[24];
    long long bl[8];
    int srcpos[kSrcBatch];
    int srcrow[kSrcBatch];
    int nsrc;
    int stop_at;
};

struct Ctx {
    const InstanceDesc *D;
    float *dyn;
    int rank, nb;
    int A;                  // active size
    int a0, a1;             // my chunk of [0,A)
    int t0, t1;             // my chunk of [A,l)
    int epoch;
    int phase;              // barrier count: selects the partial buffer
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

// records written in the current phase / read from the previous phase
__device__ __forceinline__ Partial *my_partial(const Ctx &c) { return c.D->partials + (long long)(c.phase & 1) * c.nb + c.rank; }
__device__ __forceinline__ const Partial *prev_partials(const Ctx &c) { return c.D->partials + (long long)((c.phase - 1) & 1) * c.nb; }

__device__ bool sync_group(Ctx &c, Shared &sh)
{
    bool ok = group_barrier(c.D->sync, c.nb, &sh.okflag);
    if (threadIdx.x == 0) cache_rotate(sh.cs, c.D->cache, c.rank);
    c.phase++;
    __syncthreads();
    return ok;
}

__device__ __forceinline__ double get_C(const InstanceDesc &D, int y) { return y > 0 ? D.Cp : D.Cn; }

__device__ __forceinline__ unsigned char status_of(double a, double C)
{
    if (a >= C) return ST_UPPER;            // reference svm.cpp:441-449
    if (a <= 0) return ST_LOWER;
    return ST_FREE;
}

// Sum over the group's blocks of per-block counters (block-parallel read).
__device__ void group_counts(const Ctx &c, Shared &sh, const Partial *all, int slot, int *below, int *above, int *total)
{
    int b_lo = 0, b_hi = 0, tot = 0;
    for (int b = threadIdx.x; b < c.nb; b += blockDim.x) {
        const int v = all[b].n[slot];
        tot += v;
        if (b < c.rank) b_lo += v;
        if (b > c.rank) b_hi += v;
    }
    *below = block_sum_i(sh.red, b_lo);
    *above = block_sum_i(sh.red, b_hi);
    *total = block_sum_i(sh.red, tot);
}

// --------------------------------------------------------------------------
// row-block accumulation: for every target position e in [lo,hi), in source
// order over the positions s < src_end selected by the predicate,
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
        stage_sources(D, c.dyn, sh.ss, sh.srcrow, ns);
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
        unstage_sources(D, c.dyn, sh.ss);
        if (ns < cap) break;
    }
}

// gradient reconstruction (reference svm.cpp:473-513); group collective
template <int FORM>
__device__ bool reconstruct(Ctx &c, Shared &sh)
{
    const InstanceDesc &D = *c.D;
    if (c.A == D.l) return true;
    for (int e = c.t0 + threadIdx.x; e < c.t1; e += blockDim.x) D.G[e] = __dadd_rn(D.G_bar[e], D.p[e]);
    __syncthreads();
    accumulate_rows<FORM>(c, sh, c.A, 1, 0, c.t0, c.t1);
    return sync_group(c, sh);
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

template <int FORM>
__device__ bool do_shrinking(Ctx &c, Shared &sh, int &unshrink)
{
    const InstanceDesc &D = *c.D;
    const int nu = D.nu;
    // 1. maximal violations over the active set (C-SVC: Gmax1, Gmax2; nu: Gmax1..4)
    {
        double v[4] = {-SVMB_INF, -SVMB_INF, -SVMB_INF, -SVMB_INF};
        int ix[4] = {-1, -1, -1, -1};
        const int kind[4] = {2, 2, 2, 2};
        for (int p = c.a0 + threadIdx.x; p < c.a1; p += blockDim.x) {
            const unsigned char s = D.status[p];
            const double G = D.G[p];
            const int y = D.y[p];
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
    if (!sync_group(c, sh)) return false;
    double g[4];
    {
        const Partial *all = prev_partials(c);
        double v[4] = {-SVMB_INF, -SVMB_INF, -SVMB_INF, -SVMB_INF};
        int ix[4] = {-1, -1, -1, -1};
        const int kind[4] = {2, 2, 2, 2};
        for (int b = threadIdx.x; b < c.nb; b += blockDim.x)
            for (int k = 0; k < 4; k++) v[k] = fmax(v[k], all[b].v[k]);
        block_reduce<4>(sh.red, v, ix, kind);
        if (threadIdx.x == 0) for (int k = 0; k < 4; k++) sh.bd[k] = v[k];
        __syncthreads();
        for (int k = 0; k < 4; k++) g[k] = sh.bd[k];
        __syncthreads();
    }
    const double gap = nu ? fmax(__dadd_rn(g[0], g[1]), __dadd_rn(g[2], g[3])) : __dadd_rn(g[0], g[1]);
    if (!unshrink && gap <= __dmul_rn(D.eps, 10.0)) {
        unshrink = 1;
        if (!reconstruct<FORM>(c, sh)) return false;
        c.A = D.l;
        c.epoch++;
        set_chunks(c);
    }
    // 2. number of shrunk positions -> new active size K
    {
        int cnt = 0;
        for (int p = c.a0 + threadIdx.x; p < c.a1; p += blockDim.x)
            cnt += be_shrunk(nu, D.status[p], D.y[p], D.G[p], g) ? 1 : 0;
        cnt = block_sum_i(sh.red, cnt);
        if (threadIdx.x == 0) my_partial(c)->n[0] = cnt;
    }
    if (!sync_group(c, sh)) return false;
    int K;
    {
        int below, above, tot;
        group_counts(c, sh, prev_partials(c), 0, &below, &above, &tot);
        K = c.A - tot;
    }
    // 3. holes = shrunk positions in [0,K) ascending, movers = kept positions in [K,A) descending
    {
        int h = 0, m = 0;
        for (int p = c.a0 + threadIdx.x; p < c.a1; p += blockDim.x) {
            const bool s = be_shrunk(nu, D.status[p], D.y[p], D.G[p], g);
            if (p < K && s) h++;
            if (p >= K && !s) m++;
        }
        h = block_sum_i(sh.red, h);
        m = block_sum_i(sh.red, m);
        if (threadIdx.x == 0) { Partial *pp = my_partial(c); pp->n[0] = h; pp->n[1] = m; }
    }
    if (!sync_group(c, sh)) return false;
    int hole_base, movers_below, movers_above, total_movers, dummy0, dummy1;
    group_counts(c, sh, prev_partials(c), 0, &hole_base, &dummy0, &dummy1);
    group_counts(c, sh, prev_partials(c), 1, &movers_below, &movers_above, &total_movers);
    int *holes = D.scratch;
    int *movers = D.scratch + D.l;
    {
        int h_run = 0, m_run = 0;
        for (int base = c.a0; base < c.a1; base += blockDim.x) {
            const int p = base + threadIdx.x;
            bool s = false;
            if (p < c.a1) s = be_shrunk(nu, D.status[p], D.y[p], D.G[p], g);
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
    if (!sync_group(c, sh)) return false;
    // 4. swap pair r: holes[r] <-> movers[r] (the reference's swap_index loop)
    for (long long r = (long long)c.rank * blockDim.x + threadIdx.x; r < total_movers; r += (long long)c.nb * blockDim.x)
        swap_pos(D, holes[r], movers[r]);
    if (!sync_group(c, sh)) return false;
    c.A = K;
    set_chunks(c);
    return true;
}

// --------------------------------------------------------------------------
// I_up scan of my chunk (first half of WSS3): per track the max of -y_t G_t
// with its payload.  C-SVC uses track 0 only; nu-SVC: track 0 = y=+1, 1 = y=-1.
// --------------------------------------------------------------------------
__device__ void iup_write(const Ctx &c, Shared &sh, double (&v)[2], int (&ix)[2])
{
    const InstanceDesc &D = *c.D;
    const int kind[2] = {0, 0};
    block_reduce<2>(sh.red, v, ix, kind);
    if (threadIdx.x == 0) {
        Partial *pp = my_partial(c);
        for (int k = 0; k < 2; k++) {
            const int p = ix[k];
            pp->v[3 * k + 0] = v[k];
            pp->n[4 * k + 0] = p;
            pp->v[3 * k + 1] = p >= 0 ? D.alpha[p] : 0.0;
            pp->v[3 * k + 2] = p >= 0 ? D.QD[p] : 0.0;
            pp->n[4 * k + 1] = p >= 0 ? D.pos_local[p] : 0;
            pp->n[4 * k + 2] = p >= 0 ? D.pos_row[p] : 0;
            pp->n[4 * k + 3] = p >= 0 ? D.y[p] : 0;
        }
    }
}

__device__ void scan_iup(Ctx &c, Shared &sh)
{
    const InstanceDesc &D = *c.D;
    const int nu = D.nu;
    double v[2] = {-SVMB_INF, -SVMB_INF};
    int ix[2] = {-1, -1};
    for (int p = c.a0 + threadIdx.x; p < c.a1; p += blockDim.x) {
        const unsigned char s = D.status[p];
        const double G = D.G[p];
        if (D.y[p] == +1) {
            if (s != ST_UPPER) better_max(v[0], ix[0], -G, p);
        } else {
            if (s != ST_LOWER) better_max(v[nu], ix[nu], G, p);
        }
    }
    iup_write(c, sh, v, ix);
}

// Evaluate the Q rows of sources (positions src_pos, rows src_row) into cache
// slots on positions [lo,hi) of my chunk.
template <int FORM>
__device__ void fill_rows(Ctx &c, Shared &sh, int ns, const int *src_row, const int *src_y,
                          const long long *slot, int lo, int hi)
{
    const InstanceDesc &D = *c.D;
    if (ns == 0) return;
    stage_sources(D, c.dyn, sh.ss, src_row, ns);
    double xs[kSrcBatch];
    for (int k = 0; k < ns; k++) xs[k] = D.x.xsq ? D.x.xsq[src_row[k]] : 0.0;
    for (int p = lo + threadIdx.x; p < hi; p += blockDim.x) {
        double dots[kSrcBatch];
        const int r = D.pos_row[p];
        row_dots<FORM>(D, sh.ss, ns, r, dots);
        const double xe = D.x.xsq ? D.x.xsq[r] : 0.0;
        const int yp = D.y[p];
        const long long col = D.pos_local[p];
        for (int k = 0; k < ns; k++)
            D.cache.data[slot[k] * D.cache.stride + col] = q_value(D.kp, src_y[k] * yp, dots[k], xs[k], xe);
    }
    unstage_sources(D, c.dyn, sh.ss);
}

// --------------------------------------------------------------------------
// the persistent solver
// --------------------------------------------------------------------------
template <int FORM>
__device__ void solve_instance(const InstanceDesc &D, int rank, Shared &sh, float *dyn)
{
    Ctx c;
    c.D = &D;
    c.dyn = dyn;
    c.rank = rank;
    c.nb = D.nblocks;
    c.A = D.l;
    c.epoch = 0;
    c.phase = 0;
    set_chunks(c);
    const int l = D.l;
    const int nu = D.nu;
    long long iter = 0;
    int unshrink = 0;
    int status = 0;
    if (threadIdx.x == 0) { sh.cs.nprev = 0; sh.cs.ncur = 0; }
    if (!D.x.X && D.stage_cap > 0)
        for (long long k = threadIdx.x; k < (long long)D.stage_lds * D.stage_cap; k += blockDim.x) dyn[k] = 0.0f;
    __syncthreads();

    // ---- initial state (svm.cpp:525-572, QD svm.cpp:1321-1327) ----
    {
        const int lo = (int)((long long)l * rank / c.nb), hi = (int)((long long)l * (rank + 1) / c.nb);
        for (int p = lo + threadIdx.x; p < hi; p += blockDim.x) {
            D.status[p] = status_of(D.alpha[p], get_C(D, D.y[p]));
            const int r = D.pos_row[p];
            const double xs = D.x.xsq ? D.x.xsq[r] : 0.0;
            double dot;
            if (D.x.xsq) {
                dot = xs;   // dot(x,x) is exactly what xsq holds
            } else {
                double acc = 0.0;
                float accf = 0.0f;
                if (D.x.X) {
                    const float4 *row = reinterpret_cast<const float4 *>(D.x.X + (long long)r * D.x.ld);
                    for (int k = 0; k < (D.x.ld >> 2); k++) {
                        const float4 v = __ldg(row + k);
                        acc = fma((double)v.x, (double)v.x, acc); acc = fma((double)v.y, (double)v.y, acc);
                        acc = fma((double)v.z, (double)v.z, acc); acc = fma((double)v.w, (double)v.w, acc);
                        accf = fmaf(v.x, v.x, accf); accf = fmaf(v.y, v.y, accf);
                        accf = fmaf(v.z, v.z, accf); accf = fmaf(v.w, v.w, accf);
                    }
                } else {
                    for (long long e = D.x.rowptr[r]; e < D.x.rowptr[r + 1]; e++) {
                        const float v = D.x.val[e];
                        acc = fma((double)v, (double)v, acc);
                        accf = fmaf(v, v, accf);
                    }
                }
                dot = FORM == FORM_EXACT ? acc : (double)accf;
            }
            D.QD[p] = kernel_from_dot(D.kp, dot, xs, xs);
            D.G[p] = D.p[p];
            D.G_bar[p] = 0.0;
        }
        if (!sync_group(c, sh)) goto fail;
        int any = 0;
        for (int p = threadIdx.x; p < l; p += blockDim.x) any |= D.alpha[p] > 0 ? 1 : 0;
        any = __syncthreads_or(any);
        if (any) {
            accumulate_rows<FORM>(c, sh, l, 0, 1, lo, hi);
            if (!sync_group(c, sh)) goto fail;
        }
    }

    {
        const long long max_iter = D.max_iter;
        int counter = (l < 1000 ? l : 1000) + 1;
        scan_iup(c, sh);
        if (!sync_group(c, sh)) goto fail;

        while (iter < max_iter) {
            if (--counter == 0) {
                counter = l < 1000 ? l : 1000;
                if (D.shrinking) {
                    if (!do_shrinking<FORM>(c, sh, unshrink)) goto fail;
                    scan_iup(c, sh);
                    if (!sync_group(c, sh)) goto fail;
                }
            }
            int widened = 0;
            double Gmax0, Gmax1;
            int i0, i1;
        select_again:
            // ======================= phase A =======================
            {
                const Partial *all = prev_partials(c);
                double v[2] = {-SVMB_INF, -SVMB_INF};
                int ix[2] = {-1, -1};
                const int kind[2] = {0, 0};
                for (int b = threadIdx.x; b < c.nb; b += blockDim.x) {
                    better_max(v[0], ix[0], all[b].v[0], all[b].n[0]);
                    better_max(v[1], ix[1], all[b].v[3], all[b].n[4]);
                }
                block_reduce<2>(sh.red, v, ix, kind);
                if (threadIdx.x == 0) {
                    sh.bd[0] = v[0]; sh.bi[0] = ix[0];
                    sh.bd[3] = v[1]; sh.bi[4] = ix[1];
                }
                __syncthreads();
                // winners' payload, found by the thread that read the winning partial
                for (int b = threadIdx.x; b < c.nb; b += blockDim.x) {
                    for (int k = 0; k < 2; k++) {
                        const int w = sh.bi[4 * k];
                        if (w >= 0 && all[b].n[4 * k] == w) {
                            sh.bd[3 * k + 1] = all[b].v[3 * k + 1];
                            sh.bd[3 * k + 2] = all[b].v[3 * k + 2];
                            sh.bi[4 * k + 1] = all[b].n[4 * k + 1];
                            sh.bi[4 * k + 2] = all[b].n[4 * k + 2];
                            sh.bi[4 * k + 3] = all[b].n[4 * k + 3];
                        }
                    }
                }
                __syncthreads();
                if (threadIdx.x == 0) {
                    // cache decisions for the row(s) of phase A
                    const unsigned long long clk = 2ull * (unsigned long long)iter + 1ull;
                    const int whole = c.A == l;
                    for (int k = 0; k < 2; k++) {
                        sh.bl[k] = -1;
                        sh.bi[8 + k] = 1;
                        if (sh.bi[4 * k] >= 0 && (k == 0 || nu)) {
                            Lookup L = cache_lookup(sh.cs, D.cache, sh.bi[4 * k + 1], c.epoch, clk, whole);
                            sh.bl[k] = L.slot;
                            sh.bi[8 + k] = L.valid_active;
                        }
                    }
                }
                __syncthreads();
            }
            Gmax0 = sh.bd[0];
            Gmax1 = sh.bd[3];
            i0 = sh.bi[0];
            i1 = nu ? sh.bi[4] : -1;
            {
                // evaluate the missing row(s) on my chunk
                int ns = 0;
                int srow[2], sy[2];
                long long sslot[2];
                for (int k = 0; k < 2; k++) {
                    const int ik = k == 0 ? i0 : i1;
                    if (ik >= 0 && !sh.bi[8 + k]) {
                        srow[ns] = sh.bi[4 * k + 2];
                        sy[ns] = sh.bi[4 * k + 3];
                        sslot[ns] = sh.bl[k];
                        ns++;
                    }
                }
                fill_rows<FORM>(c, sh, ns, srow, sy, sslot, c.a0, c.a1);
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
                for (int p = c.a0 + threadIdx.x; p < c.a1; p += blockDim.x) {
                    const unsigned char s = D.status[p];
                    const double G = D.G[p];
                    const int col = D.pos_local[p];
                    if (D.y[p] == +1) {
                        if (s != ST_LOWER) {
                            const double grad_diff = __dadd_rn(Gmax0, G);
                            v[1] = fmax(v[1], G);
                            if (grad_diff > 0) {
                                double quad;
                                if (!nu) quad = __dsub_rn(__dadd_rn(QDi0, D.QD[p]), __dmul_rn(two_yi0, (double)Qi0[col]));
                                else quad = __dsub_rn(__dadd_rn(QDi0, D.QD[p]), (double)__fmul_rn(2.0f, Qi0[col]));
                                const double num = __dmul_rn(grad_diff, grad_diff);
                                const double od = quad > 0 ? -__ddiv_rn(num, quad) : -__ddiv_rn(num, kTau);
                                better_min(v[0], ix[0], od, p);
                            }
                        }
                    } else {
                        if (s != ST_UPPER) {
                            const double grad_diff = __dsub_rn(nu ? Gmax1 : Gmax0, G);
                            if (nu) v[2] = fmax(v[2], -G); else v[1] = fmax(v[1], -G);
                            if (grad_diff > 0) {
                                double quad;
                                if (!nu) quad = __dadd_rn(__dadd_rn(QDi0, D.QD[p]), __dmul_rn(two_yi0, (double)Qi0[col]));
                                else quad = __dsub_rn(__dadd_rn(QDi1, D.QD[p]), (double)__fmul_rn(2.0f, Qi1[col]));
                                const double num = __dmul_rn(grad_diff, grad_diff);
                                const double od = quad > 0 ? -__ddiv_rn(num, quad) : -__ddiv_rn(num, kTau);
                                better_min(v[0], ix[0], od, p);
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
                        const int cj = D.pos_local[j];
                        pp->v[3] = D.G[j]; pp->v[4] = D.alpha[j]; pp->v[5] = D.QD[j];
                        pp->n[1] = cj; pp->n[2] = D.pos_row[j]; pp->n[3] = D.y[j];
                        pp->q[0] = Qi0 ? Qi0[cj] : 0.0f;
                        pp->q[1] = Qi1 ? Qi1[cj] : 0.0f;
                    }
                }
            }
            if (!sync_group(c, sh)) goto fail;

            // ======================= phase B =======================
            {
                const Partial *all = prev_partials(c);
                double v[3] = {SVMB_INF, -SVMB_INF, -SVMB_INF};
                int ix[3] = {-1, -1, -1};
                const int kind[3] = {1, 2, 2};
                for (int b = threadIdx.x; b < c.nb; b += blockDim.x) {
                    better_min(v[0], ix[0], all[b].v[0], all[b].n[0]);
                    v[1] = fmax(v[1], all[b].v[1]);
                    v[2] = fmax(v[2], all[b].v[2]);
                }
                block_reduce<3>(sh.red, v, ix, kind);
                if (threadIdx.x == 0) { sh.bi[12] = ix[0]; sh.bd[12] = v[1]; sh.bd[13] = v[2]; }
                __syncthreads();
                for (int b = threadIdx.x; b < c.nb; b += blockDim.x) {
                    const int w = sh.bi[12];
                    if (w >= 0 && all[b].n[0] == w) {
                        sh.bd[14] = all[b].v[3]; sh.bd[15] = all[b].v[4]; sh.bd[16] = all[b].v[5];
                        sh.bi[13] = all[b].n[1]; sh.bi[14] = all[b].n[2]; sh.bi[15] = all[b].n[3];
                        sh.bd[17] = (double)all[b].q[0]; sh.bd[18] = (double)all[b].q[1];
                    }
                }
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
                        if (!reconstruct<FORM>(c, sh)) goto fail;
                        c.A = l;
                        c.epoch++;
                        set_chunks(c);
                    }
                    widened = 1;
                    scan_iup(c, sh);
                    if (!sync_group(c, sh)) goto fail;
                    goto select_again;
                }
                if (widened) counter = 1;
            }
            ++iter;
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
            if (threadIdx.x == 0) {
                const unsigned long long clk = 2ull * (unsigned long long)iter;
                Lookup L = cache_lookup(sh.cs, D.cache, loc_j, c.epoch, clk, c.A == l);
                sh.bl[2] = L.slot;
                sh.bi[16] = L.valid_active;
            }
            __syncthreads();
            const long long slot_j = sh.bl[2];
            if (!sh.bi[16]) {
                const int srow[1] = {row_j};
                const int sy[1] = {yj};
                const long long ss[1] = {slot_j};
                fill_rows<FORM>(c, sh, 1, srow, sy, ss, c.a0, c.a1);
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
            const bool bar_i = (old_si == ST_UPPER) != (new_si == ST_UPPER);
            const bool bar_j = (old_sj == ST_UPPER) != (new_sj == ST_UPPER);
            // complete rows for the G_bar update: fill the tail [A,l) where missing
            if ((bar_i || bar_j) && c.A < l) {
                if (threadIdx.x == 0) {
                    const unsigned long long clk = 2ull * (unsigned long long)iter;
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
                int srow[2], sy[2];
                long long sslot[2];
                if (sh.bi[17]) { srow[ns] = row_i; sy[ns] = yi; sslot[ns] = slot_i; ns++; }
                if (sh.bi[18]) { srow[ns] = row_j; sy[ns] = yj; sslot[ns] = slot_j; ns++; }
                fill_rows<FORM>(c, sh, ns, srow, sy, sslot, c.t0, c.t1);
            }
            // owners publish alpha/status of i and j
            if (threadIdx.x == 0) {
                if (i >= c.a0 && i < c.a1) { D.alpha[i] = ai; D.status[i] = new_si; }
                if (j >= c.a0 && j < c.a1) { D.alpha[j] = aj; D.status[j] = new_sj; }
            }
            __syncthreads();
            // G update on my chunk (svm.cpp:732-735) + G_bar (svm.cpp:744-769) + next I_up scan
            {
                const float *Qi = D.cache.data + slot_i * D.cache.stride;
                const float *Qj = D.cache.data + slot_j * D.cache.stride;
                double v[2] = {-SVMB_INF, -SVMB_INF};
                int ix[2] = {-1, -1};
                for (int p = c.a0 + threadIdx.x; p < c.a1; p += blockDim.x) {
                    const int col = D.pos_local[p];
                    const float qi = Qi[col], qj = Qj[col];
                    const double G = __dadd_rn(D.G[p], __dadd_rn(__dmul_rn((double)qi, dai), __dmul_rn((double)qj, daj)));
                    D.G[p] = G;
                    if (bar_i || bar_j) {
                        double gb = D.G_bar[p];
                        if (bar_i) gb = (old_si == ST_UPPER) ? __dsub_rn(gb, __dmul_rn(C_i, (double)qi)) : __dadd_rn(gb, __dmul_rn(C_i, (double)qi));
                        if (bar_j) gb = (old_sj == ST_UPPER) ? __dsub_rn(gb, __dmul_rn(C_j, (double)qj)) : __dadd_rn(gb, __dmul_rn(C_j, (double)qj));
                        D.G_bar[p] = gb;
                    }
                    const unsigned char s = D.status[p];
                    if (D.y[p] == +1) {
                        if (s != ST_UPPER) better_max(v[0], ix[0], -G, p);
                    } else {
                        if (s != ST_LOWER) better_max(v[nu], ix[nu], G, p);
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
                iup_write(c, sh, v, ix);
            }
            if (!sync_group(c, sh)) goto fail;
        }

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
        double *cv = reinterpret_cast<double *>(sh.red.v);   // not used; keeps the compiler quiet
        (void)cv;
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
        *D.out = o;
    }
}

template <int FORM>
__global__ void __launch_bounds__(kThreads, 1)
smo_persistent(const InstanceDesc *__restrict__ insts, const int *__restrict__ block_inst)
{
    __shared__ Shared sh;
    extern __shared__ __align__(16) float dyn[];
    const int inst = block_inst[blockIdx.x];
    const InstanceDesc &D = insts[inst];
    const int rank = blockIdx.x - D.block0;
    solve_instance<FORM>(D, rank, sh, dyn);
}

// ---------------------------------------------------------------------------
// setup kernels
// ---------------------------------------------------------------------------
// ||x||^2 per row, in feature order (reference svm.cpp:282-296)
__global__ void xsq_kernel(DevX x, int n, double *out, int form)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        double acc = 0.0;
        float accf = 0.0f;
        if (x.X) {
            const float4 *row = reinterpret_cast<const float4 *>(x.X + (long long)r * x.ld);
            for (int k = 0; k < (x.ld >> 2); k++) {
                float4 v = __ldg(row + k);
                acc = fma((double)v.x, (double)v.x, acc); acc = fma((double)v.y, (double)v.y, acc);
                acc = fma((double)v.z, (double)v.z, acc); acc = fma((double)v.w, (double)v.w, acc);
                accf = fmaf(v.x, v.x, accf); accf = fmaf(v.y, v.y, accf);
                accf = fmaf(v.z, v.z, accf); accf = fmaf(v.w, v.w, accf);
            }
        } else {
            for (long long e = x.rowptr[r]; e < x.rowptr[r + 1]; e++) {
                float v = x.val[e];
                acc = fma((double)v, (double)v, acc);
                accf = fmaf(v, v, accf);
            }
        }
        out[r] = form == FORM_EXACT ? acc : (double)accf;
    }
}

// host-callable launchers ----------------------------------------------------
cudaError_t launch_xsq(const DevX &x, int n, double *out, int form, cudaStream_t s)
{
    int blocks = (n + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    xsq_kernel<<<blocks, 256, 0, s>>>(x, n, out, form);
    return cudaGetLastError();
}

cudaError_t launch_smo(int form, const InstanceDesc *d_insts, const int *d_block_inst, int nblocks,
                       size_t dyn_smem, bool cooperative, cudaStream_t s)
{
    void *args[] = {(void *)&d_insts, (void *)&d_block_inst};
    const void *fn = form == FORM_EXACT ? (const void *)smo_persistent<FORM_EXACT> : (const void *)smo_persistent<FORM_FP32>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem);
    if (e != cudaSuccess) return e;
    if (cooperative)
        return cudaLaunchCooperativeKernel(fn, dim3(nblocks), dim3(kThreads), args, dyn_smem, s);
    return cudaLaunchKernel(fn, dim3(nblocks), dim3(kThreads), args, dyn_smem, s);
}

cudaError_t smo_max_blocks(int form, size_t dyn_smem, int *blocks_per_sm)
{
    const void *fn = form == FORM_EXACT ? (const void *)smo_persistent<FORM_EXACT> : (const void *)smo_persistent<FORM_FP32>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, kThreads, dyn_smem);
}

}  // namespace svmb
