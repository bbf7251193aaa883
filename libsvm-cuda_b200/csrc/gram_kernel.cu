// gram_kernel.cu -- kernel-matrix blocks K(x_a, x_b) over sets of resident
// rows: the block form of the reference's Kernel::k_function / SVC_Q::get_Q
// (reference libsvm/svm.cpp:235-254, :305-325, :1316-1340).
//
// Three arithmetic forms:
//   FORM_EXACT   float64 accumulation in feature order (CUDA cores);
//   FORM_FP32    float32 accumulation (CUDA cores, the plain form);
//   FORM_BF16X3  tensor cores.  Every feature is split x = hi + lo with hi, lo
//                bf16 (hi = bf16(x), lo = bf16(x - hi); x - hi is exact in
//                float32), and dot(a, b) = hi_a.hi_b + hi_a.lo_b + lo_a.hi_b
//                accumulated in float32 in TMEM by tcgen05.mma (kind::f16).
//                The dropped lo.lo term and the residual of the split are
//                about 2^-16 of each product;
//   FORM_FP16X3  tensor cores, the same three products over an fp16 split of
//                each row scaled by a power of two (max |x| 2^e in [2^14, 2^15)):
//                x 2^e = hi + lo, about 2^-22 of each product; the dot is
//                multiplied back by 2^-e_a 2^-e_b (exact);
//   FORM_TF32    tensor cores, one product of the features rounded to tf32
//                (10 explicit mantissa bits, about 2^-11 of each product),
//                kind::tf32.  The tf32 copy has the same 256 bytes per
//                64-feature chunk as the split copy: two 128-byte halves of
//                32 features each, staged exactly like hi and lo.
// The split copy is dense (CSR rows are scattered into it), d padded to a
// multiple of 64.  RBF distances use the float64 row norms.
// The kernel value itself is always formed in float64 from the dot product.
//
// Tensor-core tiling: a persistent CTA per SM walks 128 x 64 tiles of dots;
// K runs in chunks of 64 features (the split rows store, per chunk, 64 hi then
// 64 lo 16-bit values = 256 contiguous bytes), staged by cp.async into
// 128B-swizzled K-major shared-memory tiles, four stages deep.  The warps are
// specialised and meet only at mbarriers: loader warps fill free stages (and
// run on into the next tile), one thread issues the 12 MMAs of a chunk (4
// K-steps x 3 products, M=128 N=64 K=16) into one of four TMEM accumulators,
// and eight reader warps add each finished chunk into float64 registers and
// write the tile's kernel values while the next tile's chunks are loaded.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cstdint>

#include "engine.hpp"
#include "kernel_math.cuh"
#include "tc_sm100.cuh"

namespace svmb {

namespace {

constexpr int kGM = 128;                                // rows of a tile (TMEM lanes)
constexpr int kGN = 64;                                 // columns of a tile
constexpr int kGReaders = 8;                            // warps 0-7: 4 lane quarters x 2 column halves
constexpr int kGIssuer = 8;                             // warp 8 issues the MMAs
constexpr int kGLoad0 = 9;                              // warps 9-15 load the operands
constexpr int kGThreads = 512;
constexpr int kGLoaders = kGThreads - kGLoad0 * 32;
constexpr int kGStages = 4;
constexpr int kGAcc = 4;                                // TMEM accumulators of kGN columns, used in turn
constexpr int kGTileA = kGM * 128;                      // bytes of a 128-row x 64-bf16 operand tile
constexpr int kGTileB = kGN * 128;                      // bytes of a 64-row x 64-bf16 operand tile
constexpr int kGStageBytes = 2 * kGTileA + 2 * kGTileB; // A hi, A lo, B hi, B lo
constexpr int kGSmem = kGStages * kGStageBytes + 1024;  // + alignment slack
constexpr int kGPieces = ((kGM + kGN) * 16 + kGLoaders - 1) / kGLoaders;   // 16-byte pieces per loader and step
static_assert(kGSmem <= 227 * 1024, "stages exceed the shared memory of a CTA");
// Column norms and scales of a tile, written by reader threads 0-63 when the
// tile starts and read by all readers at its end.  Reader warps stay within
// kGAcc steps of each other, so a slot is rewritten at the earliest
// 1 + ceil((kGAcc + 1) / nchunk) tiles later: 8 slots cover nchunk = 1.
constexpr int kGColRing = 8;
static_assert(kGColRing >= 2 + kGAcc, "column ring too short for one-chunk rows");

struct GramArgs {
    const uint16_t *xs;         // split rows [n][nchunk][128] of the tile rows (A)
    const double *xinv;         // per-row inverse scales (fp16 split) or nullptr
    long long rs;               // row stride in 16-bit elements (nchunk * 128)
    int nchunk;
    const int *ia;              // row ids of the tile rows (nullptr: identity)
    int ma;
    const int *ib;
    int nb;
    KernelParams kp;
    const double *xsq;          // norms by row id (A)
    const uint16_t *xs_b;       // the tile columns' rows (B): the same layout and nchunk
    const double *xinv_b;
    const double *xsq_b;
    double *out;                // [ma][ldo], or [nb][ldo] when `trans`
    long long ldo;
    int trans;
    int *err;
};

// Persistent CTA: tiles blockIdx.x, blockIdx.x + gridDim.x, ... of the
// ceil(ma/128) x ceil(nb/64) tiles, tile t = (t / ntn, t % ntn).  Each 64-feature
// chunk's 12 MMAs start a fresh float32 accumulator, so the tensor core's
// float32 accumulation spans 64 features; reader warp w adds it into float64
// registers (lanes 32(w%4).., columns 32(w/4)..+31).  Every wait is bounded; a
// role whose wait runs out sets `abort`, which ends the other roles' waits,
// and the launch reports the failure through a.err.
template <int SF>   // the split form: FORM_BF16X3, FORM_FP16X3 or FORM_TF32
__global__ void __launch_bounds__(kGThreads, 1) gram_split_kernel(GramArgs a)
{
    extern __shared__ uint8_t g_smem_raw[];
    __shared__ uint64_t full[kGStages], empty[kGStages], accf[kGAcc], acce[kGAcc];
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag;
    __shared__ double col_xsq[kGColRing][kGN], col_inv[kGColRing][kGN];
    __shared__ uint64_t colready[kGColRing];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t raw = tc::smem_addr(g_smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    volatile int *abort = &abort_flag;

    if (tid == 0) {
        for (int s = 0; s < kGStages; s++) {
            tc::mbar_init(&full[s], kGLoaders);
            tc::mbar_init(&empty[s], 1);
        }
        for (int s = 0; s < kGAcc; s++) {
            tc::mbar_init(&accf[s], 1);
            tc::mbar_init(&acce[s], kGReaders * 32);
        }
        for (int s = 0; s < kGColRing; s++) tc::mbar_init(&colready[s], kGN);
        abort_flag = 0;
        tc::mbar_init_fence();
    }
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, kGAcc * kGN);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = tmem_base;

    const int nk = a.nchunk;
    const int ntn = (a.nb + kGN - 1) / kGN;
    const int ntiles = ((a.ma + kGM - 1) / kGM) * ntn;
    const int mine = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int total = mine * nk;

    if (warp < kGReaders) {
        // ---- readers: add each chunk into float64, then the tile's kernel values.
        // A tile's row norm and scale (registers) and its 64 columns' norms and
        // scales (shared memory, one buffer per tile parity) are loaded when the
        // tile starts, so the epilogue waits on no global load.
        const int lq = warp & 3, ch = warp >> 2, rt = warp * 32 + lane;
        double acc[32];
#pragma unroll
        for (int k = 0; k < 32; k++) acc[k] = 0.0;
        int ab = 0, kc = 0, t = blockIdx.x, slot = 0;
        unsigned ph = 0, phc = 0;
        double xa = 0.0, sa_inv = 1.0;
        for (int g = 0; g < total; g++) {
            if (kc == 0) {
                const int m0 = (t / ntn) * kGM, n0 = (t % ntn) * kGN;
                const int row = m0 + lq * 32 + lane;
                if (row < a.ma) {
                    const int ra = a.ia ? a.ia[row] : row;
                    xa = a.xsq[ra];
                    sa_inv = a.xinv ? a.xinv[ra] : 1.0;
                }
                if (rt < kGN) {
                    const int col = n0 + rt;
                    double cx = 0.0, cs = 1.0;
                    if (col < a.nb) {
                        const int rb = a.ib ? a.ib[col] : col;
                        cx = a.xsq_b[rb];
                        cs = a.xinv_b ? a.xinv_b[rb] : 1.0;
                    }
                    col_xsq[slot][rt] = cx;
                    col_inv[slot][rt] = cs;
                    tc::mbar_arrive(&colready[slot]);
                }
            }
            if (!tc::mbar_wait_or(&accf[ab], ph, abort)) {
                *abort = 1;
                break;
            }
            tc::tc_fence_after();
            float v[16];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                tc::tmem_ld16(tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)(ab * kGN + ch * 32 + h * 16), v);
#pragma unroll
                for (int k = 0; k < 16; k++) acc[h * 16 + k] = __dadd_rn(acc[h * 16 + k], (double)v[k]);
            }
            tc::tc_fence_before();
            tc::mbar_arrive(&acce[ab]);
            if (++ab == kGAcc) {
                ab = 0;
                ph ^= 1u;
            }
            if (++kc < nk) continue;
            // epilogue of tile t: this thread's row and 32 columns, once the
            // tile's column data are in place
            if (!tc::mbar_wait_or(&colready[slot], phc, abort)) {
                *abort = 1;
                break;
            }
            const int m0 = (t / ntn) * kGM, n0 = (t % ntn) * kGN;
            const int row = m0 + lq * 32 + lane, c0 = n0 + ch * 32;
            if (row < a.ma) {
#pragma unroll
                for (int k = 0; k < 32; k++)
                    acc[k] = kernel_from_dot(a.kp, __dmul_rn(__dmul_rn(acc[k], sa_inv), col_inv[slot][ch * 32 + k]), xa,
                                             col_xsq[slot][ch * 32 + k]);
                if (a.trans) {
                    // the lanes of a warp (consecutive rows) write consecutive words
#pragma unroll
                    for (int k = 0; k < 32; k++)
                        if (c0 + k < a.nb) a.out[(long long)(c0 + k) * a.ldo + row] = acc[k];
                } else {
                    double *o = a.out + (long long)row * a.ldo + c0;
                    if (c0 + 32 <= a.nb && ((uintptr_t)o & 15u) == 0) {
#pragma unroll
                        for (int k = 0; k < 32; k += 2) *reinterpret_cast<double2 *>(o + k) = make_double2(acc[k], acc[k + 1]);
                    } else {
#pragma unroll
                        for (int k = 0; k < 32; k++)
                            if (c0 + k < a.nb) o[k] = acc[k];
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < 32; k++) acc[k] = 0.0;
            kc = 0;
            t += gridDim.x;
            if (++slot == kGColRing) {
                slot = 0;
                phc ^= 1u;
            }
        }
    } else if (warp == kGIssuer) {
        // ---- MMA issue
        if (lane == 0) {
            const uint32_t idesc = SF == FORM_TF32 ? tc::idesc_tf32_f32(kGM, kGN) : tc::idesc_f16_f32(kGM, kGN, SF == FORM_BF16X3);
            int s = 0, ab = 0, issued = 0;
            unsigned phs = 0, pha = 0;
            for (int g = 0; g < total; g++) {
                if (!tc::mbar_wait_or(&full[s], phs, abort) || !tc::mbar_wait_or(&acce[ab], pha ^ 1u, abort)) {
                    *abort = 1;
                    break;
                }
                tc::tc_fence_after();
                const uint32_t sa = base + s * kGStageBytes;
                const uint32_t dst = tmem + (uint32_t)(ab * kGN);
                if (SF == FORM_TF32) {
#pragma unroll
                    for (int h = 0; h < 2; h++)
#pragma unroll
                        for (int kk = 0; kk < 4; kk++)
                            tc::mma_tf32(dst, tc::sw128_desc(sa + h * kGTileA + kk * 32),
                                         tc::sw128_desc(sa + 2 * kGTileA + h * kGTileB + kk * 32), idesc, h > 0 || kk > 0);
                } else {
#pragma unroll
                    // the small cross terms of the whole chunk first, then hi.hi: the
                    // tensor core's fp32 accumulation rounds toward zero, and only the
                    // four hi.hi additions then land on a large partial sum
                    for (int kk = 0; kk < 4; kk++) {
                        const uint64_t ahi = tc::sw128_desc(sa + kk * 32), alo = tc::sw128_desc(sa + kGTileA + kk * 32);
                        const uint64_t bhi = tc::sw128_desc(sa + 2 * kGTileA + kk * 32);
                        const uint64_t blo = tc::sw128_desc(sa + 2 * kGTileA + kGTileB + kk * 32);
                        tc::mma_bf16(dst, ahi, blo, idesc, kk > 0);
                        tc::mma_bf16(dst, alo, bhi, idesc, true);
                    }
#pragma unroll
                    for (int kk = 0; kk < 4; kk++)
                        tc::mma_bf16(dst, tc::sw128_desc(sa + kk * 32), tc::sw128_desc(sa + 2 * kGTileA + kk * 32), idesc, true);
                }
                tc::mma_commit(&empty[s]);
                tc::mma_commit(&accf[ab]);
                issued++;
                if (++s == kGStages) {
                    s = 0;
                    phs ^= 1u;
                }
                if (++ab == kGAcc) {
                    ab = 0;
                    pha ^= 1u;
                }
            }
            if (issued < total && issued > 0) {
                // stopped early: let the MMAs already issued finish first
                const int G = issued - 1;
                tc::mbar_wait(&empty[G % kGStages], (unsigned)((G / kGStages) & 1));
            }
        }
        __syncwarp();
    } else {
        // ---- operand loads: piece i of a step is 16 bytes of an A row (i < 16 * kGM)
        // or of a B row; a thread's pieces keep their rows for a whole tile
        const int lt = tid - kGLoad0 * 32;
        const uint16_t *src[kGPieces];
        uint32_t off[kGPieces];
        int s = 0, sd = 0, kc = 0, t = blockIdx.x;
        unsigned phs = 0;
        bool run = true;
        // up to kGStages - 1 steps in flight; a landed step is handed to the
        // MMA before this thread waits for a free stage, so that the MMAs of
        // consecutive steps queue back to back
        for (int g = 0; g < total + kGStages - 1; g++) {
            if (g >= kGStages - 1 && run) {
                // step g - (kGStages - 1) has landed (kGStages - 2 younger groups may be pending)
                tc::cp_async_wait<kGStages - 2>();
                tc::fence_async_smem();
                tc::mbar_arrive(&full[sd]);
                if (++sd == kGStages) sd = 0;
            }
            if (g < total && run) {
                if (kc == 0) {
                    const int m0 = (t / ntn) * kGM, n0 = (t % ntn) * kGN;
#pragma unroll
                    for (int j = 0; j < kGPieces; j++) {
                        const int i = lt + j * kGLoaders;
                        src[j] = nullptr;
                        off[j] = 0;
                        const int q = i & 15;
                        if (i < 16 * kGM) {
                            const int r = i >> 4;
                            if (m0 + r < a.ma) {
                                src[j] = a.xs + (long long)(a.ia ? a.ia[m0 + r] : m0 + r) * a.rs + q * 8;
                                off[j] = (q >= 8 ? kGTileA : 0) + tc::sw128_offset(r, q & 7);
                            }
                        } else if (i < 16 * (kGM + kGN)) {
                            const int r = (i >> 4) - kGM;
                            if (n0 + r < a.nb) {
                                src[j] = a.xs_b + (long long)(a.ib ? a.ib[n0 + r] : n0 + r) * a.rs + q * 8;
                                off[j] = 2 * kGTileA + (q >= 8 ? kGTileB : 0) + tc::sw128_offset(r, q & 7);
                            }
                        }
                    }
                }
                if (!tc::mbar_wait_or(&empty[s], phs ^ 1u, abort)) {
                    *abort = 1;
                    run = false;
                } else {
                    const uint32_t sa = base + s * kGStageBytes;
#pragma unroll
                    for (int j = 0; j < kGPieces; j++)
                        if (src[j]) tc::cp_async16(sa + off[j], src[j] + kc * 128, 16u);
                }
                if (++s == kGStages) {
                    s = 0;
                    phs ^= 1u;
                }
                if (++kc == nk) {
                    kc = 0;
                    t += gridDim.x;
                }
            }
            tc::cp_async_commit();
        }
        tc::cp_async_wait<0>();
    }
    tc::tc_fence_before();
    __syncthreads();
    if (*abort && tid == 0) atomicExch(a.err, 1);
    if (warp == 0) tc::tmem_dealloc(tmem, kGAcc * kGN);
}

// CUDA-core kernel block: one thread per output, 16 x 16 threads per CTA
template <int FORM>
__global__ void kblock_cuda_kernel(DevX x, const int *ia, int ma, const int *ib, int nb, KernelParams kp, double *out,
                                   long long ldo)
{
    const int i = blockIdx.y * 16 + threadIdx.y, j = blockIdx.x * 16 + threadIdx.x;
    if (i >= ma || j >= nb) return;
    const int ra = ia ? ia[i] : i, rb = ib ? ib[j] : j;
    double dot;
    if (x.X) {
        const float *pa = x.X + (long long)ra * x.ld, *pb = x.X + (long long)rb * x.ld;
        if (FORM == FORM_EXACT) {
            double s = 0.0;
            for (int k = 0; k < x.d; k++) s = __dadd_rn(s, __dmul_rn((double)pa[k], (double)pb[k]));
            dot = s;
        } else {
            float s = 0.0f;
            for (int k = 0; k < x.d; k++) s = fmaf(pa[k], pb[k], s);
            dot = s;
        }
    } else {
        long long e = x.rowptr[ra], ee = x.rowptr[ra + 1], f = x.rowptr[rb], ff = x.rowptr[rb + 1];
        double s = 0.0;
        float sf = 0.0f;
        while (e < ee && f < ff) {
            const int ce = x.col[e], cf = x.col[f];
            if (ce == cf) {
                if (FORM == FORM_EXACT) s = __dadd_rn(s, __dmul_rn((double)x.val[e], (double)x.val[f]));
                else sf = fmaf(x.val[e], x.val[f], sf);
                ++e; ++f;
            } else if (ce > cf) {
                ++f;
            } else {
                ++e;
            }
        }
        dot = FORM == FORM_EXACT ? s : (double)sf;
    }
    out[(long long)i * ldo + j] = kernel_from_dot(kp, dot, x.xsq[ra], x.xsq[rb]);
}

// per-row scale of the fp16 split: xinv[r] = 2^-e with max_k |x_rk| 2^e in
// [2^14, 2^15) (1 for an all-zero row); one warp per row
__global__ void row_scale_kernel(DevX x, int n, double *__restrict__ xinv)
{
    const int lane = threadIdx.x & 31;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += (gridDim.x * blockDim.x) >> 5) {
        float m = 0.0f;
        if (x.X) {
            for (int k = lane; k < x.d; k += 32) m = fmaxf(m, fabsf(x.X[(long long)r * x.ld + k]));
        } else {
            for (long long e = x.rowptr[r] + lane; e < x.rowptr[r + 1]; e += 32) m = fmaxf(m, fabsf(x.val[e]));
        }
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) {
            int k = 0;
            if (m > 0.0f) frexpf(m, &k);            // m = f 2^k, f in [0.5, 1)
            xinv[r] = m > 0.0f ? ldexp(1.0, k - 15) : 1.0;
        }
    }
}

// feature k of a row in the tf32 copy: the chunk's 64 values as 32-bit words,
// rounded to tf32 (nearest, ties away: cvt.rna.tf32.f32)
__device__ __forceinline__ void tf32_store(float v, uint16_t *row, int k)
{
    uint32_t t;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"(v));
    reinterpret_cast<uint32_t *>(row)[(k / kSplitChunk) * kSplitChunk + (k % kSplitChunk)] = t;
}

__global__ void tf32_dense_kernel(const float *__restrict__ X, int n, int ld, int d, int nchunk, uint16_t *__restrict__ Xs)
{
    const long long rs = (long long)nchunk * 2 * kSplitChunk;
    const long long total = (long long)n * d;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long r = idx / d;
        const int k = (int)(idx - r * d);
        tf32_store(X[r * ld + k], Xs + r * rs, k);
    }
}

__global__ void tf32_csr_kernel(const long long *__restrict__ rowptr, const int *__restrict__ col,
                                const float *__restrict__ val, int n, int nchunk, uint16_t *__restrict__ Xs)
{
    const long long nnz = rowptr[n];
    const long long rs = (long long)nchunk * 2 * kSplitChunk;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nnz; e += (long long)gridDim.x * blockDim.x) {
        int a = 0, b = n;
        while (b - a > 1) {
            const int m = (a + b) >> 1;
            if (rowptr[m] <= e) a = m; else b = m;
        }
        tf32_store(val[e], Xs + a * rs, col[e]);
    }
}

template <bool BF16>
__device__ __forceinline__ void split_store(float v, float s, uint16_t *dst)
{
    if (BF16) {
        const __nv_bfloat16 hi = __float2bfloat16_rn(v);
        const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
        dst[0] = __bfloat16_as_ushort(hi);
        dst[kSplitChunk] = __bfloat16_as_ushort(lo);
    } else {
        const float w = v * s;                       // exact: s is a power of two
        const __half hi = __float2half_rn(w);
        const __half lo = __float2half_rn(w - __half2float(hi));
        dst[0] = __half_as_ushort(hi);
        dst[kSplitChunk] = __half_as_ushort(lo);
    }
}

// split dense rows: Xs[r][c][e] = hi(X[r][64c+e]), Xs[r][c][64+e] = lo(...); Xs zeroed beforehand
template <bool BF16>
__global__ void split_dense_kernel(const float *__restrict__ X, int n, int ld, int d, int nchunk,
                                   const double *__restrict__ xinv, uint16_t *__restrict__ Xs)
{
    const long long rs = (long long)nchunk * 2 * kSplitChunk;
    const long long total = (long long)n * d;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long r = idx / d;
        const int k = (int)(idx - r * d);
        const float s = BF16 ? 1.0f : (float)(1.0 / xinv[r]);
        split_store<BF16>(X[r * ld + k], s, Xs + r * rs + (long long)(k / kSplitChunk) * (2 * kSplitChunk) + (k % kSplitChunk));
    }
}

// split CSR rows (Xs zeroed beforehand): one thread per stored value
template <bool BF16>
__global__ void split_csr_kernel(const long long *__restrict__ rowptr, const int *__restrict__ col,
                                 const float *__restrict__ val, int n, int nchunk, const double *__restrict__ xinv,
                                 uint16_t *__restrict__ Xs)
{
    const long long nnz = rowptr[n];
    const long long rs = (long long)nchunk * 2 * kSplitChunk;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nnz; e += (long long)gridDim.x * blockDim.x) {
        int a = 0, b = n;                            // row of e: last a with rowptr[a] <= e
        while (b - a > 1) {
            const int m = (a + b) >> 1;
            if (rowptr[m] <= e) a = m; else b = m;
        }
        const int k = col[e];
        const float s = BF16 ? 1.0f : (float)(1.0 / xinv[a]);
        split_store<BF16>(val[e], s, Xs + a * rs + (long long)(k / kSplitChunk) * (2 * kSplitChunk) + (k % kSplitChunk));
    }
}

const void *gram_fn(int form)
{
    if (form == FORM_BF16X3) return (const void *)gram_split_kernel<FORM_BF16X3>;
    if (form == FORM_TF32) return (const void *)gram_split_kernel<FORM_TF32>;
    return (const void *)gram_split_kernel<FORM_FP16X3>;
}

// one persistent CTA per SM (or per tile, when there are fewer tiles)
void launch_gram(int form, const GramArgs &a, cudaStream_t s)
{
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    const long long tiles = (long long)((a.ma + kGM - 1) / kGM) * ((a.nb + kGN - 1) / kGN);
    const dim3 grid((unsigned)std::max<long long>(1, std::min<long long>(tiles, sms)));
    if (form == FORM_BF16X3) gram_split_kernel<FORM_BF16X3><<<grid, kGThreads, kGSmem, s>>>(a);
    else if (form == FORM_TF32) gram_split_kernel<FORM_TF32><<<grid, kGThreads, kGSmem, s>>>(a);
    else gram_split_kernel<FORM_FP16X3><<<grid, kGThreads, kGSmem, s>>>(a);
}

}  // namespace

cudaError_t launch_split(const DeviceRows &rows, int form, int nchunk, uint16_t *Xs, double *xinv, cudaStream_t s)
{
    const int n = rows.n;
    if (n <= 0) return cudaSuccess;
    const bool bf16 = form == FORM_BF16X3;
    const DevX x = rows.view(FORM_EXACT);
    if (form == FORM_TF32) {
        if (rows.dense) {
            const long long total = (long long)n * rows.d;
            const int blocks = (int)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 32));
            tf32_dense_kernel<<<blocks, 256, 0, s>>>(rows.X, n, rows.ld, rows.d, nchunk, Xs);
        } else {
            const int blocks = (int)std::max<long long>(1, std::min<long long>((rows.nnz + 255) / 256, 148LL * 32));
            tf32_csr_kernel<<<blocks, 256, 0, s>>>(rows.rowptr, rows.col, rows.val, n, nchunk, Xs);
        }
        count_launch();
        return cudaGetLastError();
    }
    if (!bf16) {
        row_scale_kernel<<<(int)std::min<long long>(((long long)n * 32 + 255) / 256, 148LL * 32), 256, 0, s>>>(x, n, xinv);
        count_launch();
    }
    if (rows.dense) {
        const long long total = (long long)n * rows.d;
        const int blocks = (int)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 32));
        if (bf16) split_dense_kernel<true><<<blocks, 256, 0, s>>>(rows.X, n, rows.ld, rows.d, nchunk, xinv, Xs);
        else split_dense_kernel<false><<<blocks, 256, 0, s>>>(rows.X, n, rows.ld, rows.d, nchunk, xinv, Xs);
    } else {
        const int blocks = (int)std::max<long long>(1, std::min<long long>((rows.nnz + 255) / 256, 148LL * 32));
        if (bf16) split_csr_kernel<true><<<blocks, 256, 0, s>>>(rows.rowptr, rows.col, rows.val, n, nchunk, xinv, Xs);
        else split_csr_kernel<false><<<blocks, 256, 0, s>>>(rows.rowptr, rows.col, rows.val, n, nchunk, xinv, Xs);
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_kernel_block(const DeviceRows &rows, const KernelParams &kp, int form, const int *d_ia, int ma,
                                const int *d_ib, int nb, double *d_out, long long ldo, int *d_err, cudaStream_t s)
{
    if (ma <= 0 || nb <= 0) return cudaSuccess;
    if (is_tc_form(form)) {
        const void *fn = gram_fn(form);
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem);
        if (e != cudaSuccess) return e;
        GramArgs a;
        a.xs = rows.Xs;
        a.xinv = rows.xinv;
        a.nchunk = rows.nchunk;
        a.rs = (long long)rows.nchunk * 2 * kSplitChunk;
        a.ia = d_ia; a.ma = ma; a.ib = d_ib; a.nb = nb;
        a.kp = kp;
        a.xsq = rows.xsq[FORM_EXACT];
        a.xs_b = rows.Xs;
        a.xinv_b = rows.xinv;
        a.xsq_b = rows.xsq[FORM_EXACT];
        a.out = d_out; a.ldo = ldo;
        a.trans = 0;
        a.err = d_err;
        launch_gram(form, a, s);
    } else {
        dim3 grid((nb + 15) / 16, (ma + 15) / 16), block(16, 16);
        if (form == FORM_EXACT)
            kblock_cuda_kernel<FORM_EXACT><<<grid, block, 0, s>>>(rows.view(FORM_EXACT), d_ia, ma, d_ib, nb, kp, d_out, ldo);
        else
            kblock_cuda_kernel<FORM_FP32><<<grid, block, 0, s>>>(rows.view(FORM_FP32), d_ia, ma, d_ib, nb, kp, d_out, ldo);
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_kernel_block2(const DeviceRows &A, const DeviceRows &B, const KernelParams &kp, int form, int a0,
                                 int ma, int nb, double *d_out, long long ldo, int trans, int *d_err, cudaStream_t s)
{
    if (ma <= 0 || nb <= 0) return cudaSuccess;
    if (!is_tc_form(form) || A.split_form != form || B.split_form != form || A.nchunk != B.nchunk)
        return cudaErrorInvalidValue;
    const void *fn = gram_fn(form);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem);
    if (e != cudaSuccess) return e;
    GramArgs a;
    // rows a0 .. a0+ma of A: the row pointers, scales and norms start there
    a.rs = (long long)A.nchunk * 2 * kSplitChunk;
    a.xs = A.Xs + (long long)a0 * a.rs;
    a.xinv = A.xinv ? A.xinv + a0 : nullptr;
    a.nchunk = A.nchunk;
    a.ia = nullptr; a.ma = ma; a.ib = nullptr; a.nb = nb;
    a.kp = kp;
    a.xsq = A.xsq[FORM_EXACT] + a0;
    a.xs_b = B.Xs;
    a.xinv_b = B.xinv;
    a.xsq_b = B.xsq[FORM_EXACT];
    a.out = d_out; a.ldo = ldo;
    a.trans = trans;
    a.err = d_err;
    launch_gram(form, a, s);
    count_launch();
    return cudaGetLastError();
}

}  // namespace svmb
