// engine.h -- structures shared by the device solver (smo_kernel.cu) and the
// host orchestration (engine.cpp).  Internal to libsvm_b200.so.
//
// One SMO "instance" is one binary subproblem of the reference's svm_train
// (reference libsvm/svm.cpp:1707 svm_train_one -> Solver::Solve :515 or
// Solver_NU::Solve :1060).  An instance is solved by a GROUP of thread blocks
// of one persistent launch; several instances (one-vs-one pairs, CV folds,
// grid points) can share a launch, each with its own group.
#pragma once
#include <cstdint>
#include <cstddef>

#ifdef __CUDACC__
#define SVMB_HD __host__ __device__
#else
#define SVMB_HD
#endif

namespace svmb {

#ifndef SVMB_THREADS
#define SVMB_THREADS 512
#endif
constexpr int kThreads = SVMB_THREADS;  // threads per block of the persistent solver (a multiple of 128)
constexpr int kWarps = kThreads / 32;
constexpr int kSrcBatch = 8;            // source rows staged per pass in the row-block product
constexpr int kMaxWays = 8;             // set associativity of the Q-row cache
constexpr int kEpochFull = -2;          // cache slot holds the complete row
constexpr int kPrefetchCand = 4;        // prefetch candidates published per block and phase
constexpr int kPrefetchMax = 8;         // rows evaluated per fill pass (the missing row + prefetched)
constexpr int kNoTag = -1;
constexpr int kMaxGroupBlocks = 160;     // blocks per instance (one per SM)
constexpr int kTileStride = 16;         // floats per row of a warp's 32x16 transpose tile (16-byte pieces swizzled)
// shared memory shared by the transpose tiles (two per warp: the next column
// slice loads while the current one is used) and the prefetch candidate table
constexpr int kTileBytes = kWarps * 32 * kTileStride * 4;      // one tile per warp
constexpr int kCandBytes = kMaxGroupBlocks * kPrefetchCand * (8 + 4 * 4);
constexpr int kAuxBytes = ((2 * kTileBytes > kCandBytes ? 2 * kTileBytes : kCandBytes) + 15) / 16 * 16;
constexpr int kAuxBytes1 = ((kTileBytes > kCandBytes ? kTileBytes : kCandBytes) + 15) / 16 * 16;
// tensor forms: no transpose tiles; candidates or the block-product partial sums
constexpr int kRedBytes = 8 * 128 * 8;
constexpr int kAuxBytesTc = ((kCandBytes > kRedBytes ? kCandBytes : kRedBytes) + 15) / 16 * 16;
// transpose tiles per warp in the CUDA-core fills: a ring of up to 4 column
// slices, all but the one in use in flight
constexpr int kMaxTileBufs = 4;
// Sparse rows too wide to scatter into shared memory (fewer than two dense
// source vectors fit) stage a fill pass's sources as one open-addressing
// table keyed by column: kHashSlots int keys (-1 = empty) followed by
// kHashSlots x kSrcBatch values (float64 in the exact form, float32 else).
// A pass whose sources hold more than kHashSlots/2 nonzeros in total falls
// back to merge walks in global memory.
constexpr int kHashSlots = 1024;
SVMB_HD constexpr int hash_bytes(int form) { return kHashSlots * 4 + kHashSlots * kSrcBatch * (form == 0 ? 8 : 4); }
SVMB_HD constexpr int tile_aux_bytes(int bufs) { return ((bufs * kTileBytes > kCandBytes ? bufs * kTileBytes : kCandBytes) + 15) / 16 * 16; }
SVMB_HD constexpr int aux_bytes(int form, int tile_bufs) { return (form == 2 || form == 3 || form == 4) ? kAuxBytesTc : tile_aux_bytes(tile_bufs); }

// tensor-core (FORM_BF16X3) block products inside the solver
constexpr int kTcM = 128;               // targets per tile (MMA M); rows are TMEM lanes
constexpr int kTcStages = 3;            // operand stages of the cp.async -> MMA pipeline
constexpr int kTcMaxN = 4 * (kThreads / 32) < 64 ? 4 * (kThreads / 32) : 64;   // sources per block-product pass
                                        // (MMA N; the epilogue reads 16 columns per group of 4 warps)
// bytes of one operand stage: target tile (128 rows x 64 bf16, hi and lo) + n source rows (hi and lo)
SVMB_HD constexpr int tc_stage_bytes(int n) { return 2 * kTcM * 128 + n * 256; }
SVMB_HD constexpr int tc_area_bytes(int n) { return 1024 + kTcStages * tc_stage_bytes(n); }
// the Q-row fill pipeline of the tensor forms reuses that area: stages of one
// target tile + kFillN source rows; warps 0-3 read the accumulators, warp 4
// issues the MMAs, warps kFillLoad0.. load the operands
constexpr int kFillN = 16;              // MMA N of a fill pass (>= kPrefetchMax sources)
constexpr int kFillStagesMax = 4;
constexpr int kFillAcc = 4;             // TMEM accumulators of kFillN columns, used in turn
constexpr int kFillLoad0 = 5;
SVMB_HD constexpr int fill_stage_bytes() { return 2 * kTcM * 128 + kFillN * 256; }
SVMB_HD constexpr int fill_stages(int tc_n)
{
    return (tc_area_bytes(tc_n) - 1024) / fill_stage_bytes() < kFillStagesMax
               ? (tc_area_bytes(tc_n) - 1024) / fill_stage_bytes()
               : kFillStagesMax;
}
static_assert(fill_stages(16) >= 3, "the fill pipeline needs three operand stages");
static_assert(kThreads / 32 > kFillLoad0, "the fill pipeline needs loader warps");

enum : uint8_t { ST_LOWER = 0, ST_UPPER = 1, ST_FREE = 2 };   // reference svm.cpp:425

// arithmetic form of the kernel-row evaluation
enum RowForm : int {
    FORM_EXACT = 0,   // fp32 X, fp64 accumulation in feature order (matches the reference's Kernel::dot)
    FORM_FP32 = 1,    // fp32 X, fp32 accumulation (the plain CUDA-core form)
    FORM_BF16X3 = 2,  // tensor cores: x = hi + lo in bf16, dot = hi.hi + hi.lo + lo.hi, fp32 accumulation
    FORM_FP16X3 = 3,  // tensor cores: x*2^e = hi + lo in fp16 (power-of-2 scale per row), same three products
    FORM_TF32 = 4,    // tensor cores: x rounded to tf32 (10-bit mantissa), one product, fp32 accumulation
};
constexpr int kNumForms = 5;
SVMB_HD constexpr bool is_tc_form(int f) { return f == FORM_BF16X3 || f == FORM_FP16X3 || f == FORM_TF32; }
constexpr int kSplitChunk = 64;         // features per K-chunk of the split rows: hi 64 then lo 64 (16-bit
                                        // values), or in FORM_TF32 the chunk's 64 tf32 values (the same 256 bytes)

struct KernelParams {
    int type;         // LINEAR, POLY, RBF, SIGMOID
    int degree;
    double gamma;
    double coef0;
};

// Feature rows on the device, shared by every instance built from the same problem.
struct DevX {
    const float *X;             // dense row-major [n_rows][ld] (nullptr for CSR)
    int ld;                     // floats per dense row, multiple of 4
    const long long *rowptr;    // CSR [n_rows+1]
    const int *col;             // CSR 0-based column
    const float *val;           // CSR value
    int d;                      // number of feature columns
    const double *xsq;          // [n_rows] dot(x,x) in the reference's order
    const uint16_t *Xs;         // split rows [n_rows][nchunk][hi 64 | lo 64] (tensor forms), or nullptr
    int nchunk;                 // 64-feature chunks per split row
    const double *xinv;         // FORM_FP16X3: per-row 2^-e undoing the split's scale (nullptr: 1)
};

// Q-row cache of one instance: `nsets` x `nways` slots of `stride` floats;
// columns are indexed by the instance's LOCAL variable index (not position),
// so shrinking permutations never move cached data.
struct CacheView {
    float *data;
    int *tag;                   // [nslots] local row held, or kNoTag
    int *epoch;                 // [nslots] active-set epoch the row is valid for, or kEpochFull
    unsigned long long *stamp;  // [nslots] LRU clock
    int nsets, nways;
    long long stride;
};

struct GroupSync {
    unsigned int count;
    unsigned int gen;
    int error;                  // nonzero: a wait timed out somewhere in the group
    unsigned int finished;      // blocks of the group that have written their results
    int pad[28];
};

// Cross-block reduction record (one per block per phase).  Besides the
// reduced value and position it carries the winner's per-variable data
// (alpha, QD, label, local index, row id) so that no block has to read
// another block's chunk of the state arrays.
// `seq` is written last with release semantics: a reader that observes
// seq == k (acquire) sees the record of exchange k, so the record exchange is
// also the group barrier.
struct Partial {
    double v[8];
    int n[8];
    float q[2];
    int seq;
    int pad[5];
    // the block's most violating positions (prefetch candidates): priority,
    // position, local index, row id, label
    double cv[kPrefetchCand];
    int cpos[kPrefetchCand];
    int cloc[kPrefetchCand];
    int crow[kPrefetchCand];
    int cy[kPrefetchCand];
    int pad2[8];
};
static_assert(sizeof(Partial) == 256, "Partial must stay 256 bytes");
static_assert(kPrefetchMax <= kSrcBatch, "a fill pass stages at most kSrcBatch rows");

struct SolveOut {
    long long iters;
    double rho, obj, r;
    int status;                 // 0 ok, 1 max_iter reached, <0 error
    int active_size;
    int unshrink;
    int nr_free;
    double gap;                 // m(alpha) - M(alpha) at exit
    // work counters (for the roofline): sum over iterations of the active
    // size, Q values evaluated, and cache lookups that hit
    long long sum_active;
    long long q_evals;
    long long lookups, hits;
    long long fills, prefetched, prefetch_used;   // fill passes, rows prefetched, prefetched rows later hit
    long long fill_targets;     // target positions of all fill passes (each pass reads its targets' rows once)
    // SM cycles spent by block 0 in each section of the loop (kProf* below)
    long long prof[8];
};
enum { kProfAReduce = 0, kProfAFill, kProfAScan, kProfBReduce, kProfBFill, kProfBUpdate, kProfShrink, kProfTotal };

struct InstanceDesc {
    int l;
    int nu;                     // 0: Solver (C-SVC), 1: Solver_NU
    int shrinking;
    int form;                   // RowForm
    double Cp, Cn, eps;
    long long max_iter;
    KernelParams kp;
    DevX x;
    // position-indexed state (permuted by shrinking exactly like the reference)
    double *G, *G_bar, *alpha, *p, *QD;
    signed char *y;
    unsigned char *status;
    int *pos_local;             // position -> local index (cache column)
    int *pos_row;               // position -> row id in DevX
    // outputs
    double *alpha_local;        // [l] final alpha by local index (unsigned, unscaled)
    SolveOut *out;
    // group
    int block0, nblocks;
    GroupSync *sync;
    Partial *partials;          // [2][nblocks]
    int *scratch;               // [2*l] shrink pair lists
    CacheView cache;
    // source-row staging in dynamic shared memory
    int stage_cap;              // rows staged at once (1..kSrcBatch); 0: read sources from global memory
    int stage_lds;              // floats per staged row (dense: ld; sparse: d)
    int chunk_cap;              // positions of per-block state held in shared memory (>= ceil(l/nblocks))
    int prefetch;               // rows evaluated per fill pass (1 = no prefetch), <= kPrefetchMax
    // 0: G_bar maintained on every bound change, as the reference does (svm.cpp:744-769);
    // 1: no G_bar -- reconstruction recomputes G = p + sum over alpha>0 of alpha*Q on the
    //    inactive positions as one block product (no full-length rows during the loop)
    int lazy_gbar;
    int tc_n;                   // FORM_BF16X3: sources per tensor-core pass (16, 32 or 64); 0 otherwise
    int *done_flag;             // host-mapped word set to 1 once the whole instance has written its results, or nullptr
    int tile_bufs;              // transpose tiles per warp in the CUDA-core fills (1 to kMaxTileBufs; same in every instance of a launch)
    int hash_slots;             // sparse rows, stage_cap == 0: sources staged in a kHashSlots table (0: merge walks)
    long long wait_ns;          // bound of every cross-block wait, in ns of %globaltimer (0: 30 s)
};

}  // namespace svmb
