// pk_kernels.cuh -- device-side views and launchers shared by the kernel and ABI
// translation units.  Everything here is internal to libpkcuda.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pk_math.cuh"
#include "pk_slab_plan.h"

namespace pk {

// Step flags (mirrored in include/pkcuda.h as PK_FLAG_*).
enum : unsigned {
    kFlagPrecomputeFailed = 0x1u,
    kFlagSingularDiag = 0x2u,
    kFlagInvalidRhs = 0x4u,
    kFlagBreakdown = 0x8u,
    kFlagNonFiniteDv = 0x10u,
    kFlagIntegrateAbort = 0x20u,
    kFlagPolarIdentity = 0x40u,
    kFlagPolarFp64 = 0x80u,
    kFlagBarrierTimeout = 0x100u,
    kFlagRowTooLong = 0x200u,
    kFlagSolved = 0x1000u,
    kFlagIntegrated = 0x2000u,
    kFlagConverged = 0x4000u,
    kFlagRefinedFp64 = 0x8000u,
};

struct GridSync {
    unsigned arrive;
    unsigned gen;
    int err;
    int pad;
};

struct DevStats {
    int iterations;
    int converged;
    double residual_norm;
    unsigned flags;
    int polar_fp64_count;
    int polar_identity_count;
    unsigned batch_missing;  // batched solve: success flags some body lacks
};

// Upper-stored symmetric BSR plus its transpose index: for row r, the blocks (c, r)
// with c < r are lt_block[lt_start[r] .. lt_start[r+1]) and c = lt_row[...].
template <class Real>
struct BsrView {
    int n;
    const int* row_start;
    const int* col;
    const Real* values;  // 9 per block, column-major
    const int* lt_start;
    const int* lt_row;
    const int* lt_block;
};

template <class Real>
struct TetView {
    int tet_count;
    const int4* nodes;               // world node ids
    const unsigned char* enabled;    // bit 0: active, rest volume > 0, body simulated; bit 1: linear FEM
    const Real* dm_inv;              // 9 per tet, column-major
    const Real* params;              // 4 per tet: rest volume, lambda, mu, damping
    // kTetRec per tet, read by the row kernel (one aligned record per tet): R (9), a 3x3
    // matrix M (9) and a form value (index 31), written by the tet kernel each step
    // (rec[kTetRec t] = NaN when the tet is skipped this step); DmInv (9), rest volume,
    // lambda, mu, damping (18..30), written once when the tets are set (launch_tet_pack).
    // Form 0: M = S = R * V * sigma, node a's elastic force is -S g_a.  Form 1 (the
    // implicit step with a slot table): M = T = -(dt S + dt^2 Q), where Q g_a is the tet's
    // sum_b K_ab v_b, so the tet adds T g_a - dt c v_a to row a's right-hand side.
    Real* rec;
};
constexpr int kTetRec = 32;
constexpr unsigned kSlotNone = 255u, kSlotMissing = 254u;
constexpr int kSlotMaxRow = 16;  // the row kernel's register-slot paths (MAXU 8 and 16)

template <class Real>
struct AssemblyArgs {
    TetView<Real> tets;
    BsrView<Real> a;
    int node_count;
    const int* dyn_to_node;
    const int* node_to_dyn;
    const Real* mass;                // per world node
    const Real* x;                   // 3 per world node
    Real* v;                         // 3 per world node (written only in explicit mode)
    Real* x_out;                     // explicit mode position update target
    const int* inc_start;            // per dyn row
    const int* inc_list;             // t*4 + a
    // Per incidence, the row slots of the tet's 4 nodes (8 bits each, node b in bits
    // 8b..8b+7): the block's index in the row's upper blocks, kSlotNone when the column is
    // not in the upper row (a lower or non-dynamic node), kSlotMissing when the pattern
    // lacks it.  NULL: no table (rows longer than kSlotMaxRow, or not built).
    const unsigned* inc_slot;
    int row_lanes;                   // with a slot table: four lanes per row (1) or one thread (0)
    Real* values;                    // out: A blocks
    Real* rhs;                       // out: b
    Real* minv;                      // out: block-Jacobi inverse
    Real dt;
    Real gravity[3];
    int use_jacobi;
    int linear;
    int explicit_mode;
    unsigned* flags;
    DevStats* stats;
    // Transient point connections (PointConnection::UpdateSystem); conn_inc_start is
    // NULL when there are none.
    int conn_count;
    const int4* conn_nodes;          // 4 world nodes per connection
    const Real* conn_params;         // kConnParams per connection: weights (4), target (3), stiffness, damping
    Real* conn_eval;                 // 4 per connection: its force (3) and 1 when it applies this step, else 0
    const int* conn_inc_start;       // per dyn row
    const int* conn_inc_list;        // connection*4 + corner (corners with a non-zero weight)
    // Host-emitted stiffness blocks and forces (SolverData::AddStiffnessBlock / AddNodeForce
    // from custom components); ext_rhs_start is NULL when there are none.
    const Real* ext_blocks;          // 9 per block, column-major
    const int2* ext_nodes;           // per block: its row node and column node
    const int* ext_rhs_start;        // per dyn row: blocks whose row node is that row (rhs -dt^2 B v_col)
    const int* ext_rhs_list;
    const int* ext_mat_start;        // per dyn row: blocks it holds in its upper row
    const int* ext_mat_list;         // block index, | 0x80000000 when the transpose is added
    const Real* ext_force;           // 3 per dyn row, or NULL
};
constexpr int kConnParams = 9;

template <class Real, class Acc>
struct PcgArgs {
    BsrView<Real> a;
    const Real* b;
    const Real* minv;
    Real* x;
    Real* r;
    // Search-direction records, 8 values per row {s.x, s.y, s.z, 0, d.x, d.y, d.z, 0}
    // (32-byte aligned for float), ping-ponged between iterations so a neighbour's
    // s + beta*d is one 256-bit load.
    Real* sd0;
    Real* sd1;
    Real* q;
    Acc* part_a;      // [grid]
    Acc* part_b;      // [grid * 2]
    int* part_bad;    // [grid * 4]: phase A, init/phase B, final check
    GridSync* sync;
    int max_iterations;
    Acc tolerance;
    int skip_on_flags;     // skip the solve when assembly flagged failure
    int integrate;
    Real dt;
    const int* dyn_to_node;
    Real* node_x;
    Real* node_v;
    unsigned* flags;
    DevStats* stats;
    // SpMV tiles staged into shared memory by TMA bulk copies, 8 ints per tile:
    // {first row, end row, rs0, row words, k0, blocks, e0, transpose entries}, each range
    // widened to 16-byte boundaries; ntiles == 0 selects the unstaged SpMV.
    int ntiles;
    const int* tile_desc;
};

// Shared-memory tile of the staged SpMV: at most kTileRowCap row_start / lt_start
// entries, kTileCapU upper blocks (values + columns) and kTileCapL transpose entries,
// each range widened to 16-byte boundaries for the bulk copies.
constexpr int kTileRowsMax = 64;
constexpr int kTileRowCap = kTileRowsMax + 8;
constexpr int kTileCapU = 576;
constexpr int kTileCapL = 512;
template <class Real>
constexpr size_t tile_buffer_bytes()
{
    return size_t(2 * kTileRowCap) * 4 + size_t(kTileCapU) * 9 * sizeof(Real) + size_t(kTileCapU) * 4 +
           size_t(2 * kTileCapL) * 4;
}

// ------------------------------------------------------------------ ring-staged PCG
// The ring-staged PCG kernel (pk_pcg_ring.cu) cuts the rows into tiles of at most kRows
// consecutive rows and streams each tile's part of the matrix -- row extents, upper
// blocks with their columns, and the transposed index (rows and block numbers of the
// lower entries) -- into shared memory with TMA bulk copies, through a ring of kStages
// buffers filled by one producer warp.  Consumer warps, in kRingGroups groups that take
// every kRingGroups-th ring position, compute the tile's rows of q = A (s + beta d)
// from the staged data plus gathers of the neighbours' {s, d} records and of the
// transposed lower blocks (both L2 hits, as the grid sweeps one wavefront through the
// matrix).  kStages is a multiple of kRingGroups, so a stage is always reused by the
// group that used it last and its mbarrier parity cannot be mistaken.
// Caps are in entries; every span is widened to 16-byte boundaries (row words to 4,
// blocks and lower entries to 4).
template <class Real>
struct RingTile;
template <>
struct RingTile<float> {
    static constexpr int kRows = 32, kRsCap = 40, kCapU = 320, kCapL = 288;
    static constexpr int kStages = 12, kLanesPerRow = 4;  // 32 rows per consumer group of 4 warps (4 stages each)
};
template <>
struct RingTile<double> {
    static constexpr int kRows = 16, kRsCap = 24, kCapU = 160, kCapL = 144;
    static constexpr int kStages = 12, kLanesPerRow = 8;  // 16 rows per consumer group of 4 warps
};
constexpr int kRingGroups = 3;  // 13 warps: at most 4 per SM sub-partition, so 128 registers
constexpr int kRingGroupWarps = 4;
constexpr int kRingConsumerWarps = kRingGroups * kRingGroupWarps;
constexpr int kRingThreads = 32 * (kRingConsumerWarps + 1);  // + one producer warp
constexpr int kRingDescInts = 8;  // per tile: ra, rb, rs0, nrs, k0, nk, e0, ne
constexpr int kRingMaxTilesPerBlock = 512;

constexpr size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Byte offsets of one ring stage, then of the block's descriptor table after the ring.
template <class Real>
struct RingLayout {
    using T = RingTile<Real>;
    static constexpr size_t kRs = 0;
    static constexpr size_t kLts = kRs + 4 * T::kRsCap;
    static constexpr size_t kVals = align_up(kLts + 4 * T::kRsCap, 16);
    static constexpr size_t kCol = align_up(kVals + sizeof(Real) * 9 * T::kCapU, 16);
    static constexpr size_t kLtr = align_up(kCol + 4 * T::kCapU, 16);
    static constexpr size_t kLtb = align_up(kLtr + 4 * T::kCapL, 16);
    static constexpr size_t kBytes = align_up(kLtb + 4 * T::kCapL, 128);
    static constexpr size_t kTable = kBytes * T::kStages;
    static constexpr size_t kTotal = kTable + 4 * kRingDescInts * size_t(kRingMaxTilesPerBlock);
};

// One block's published partials for a grid exchange (double buffered by generation).
struct __align__(32) ExSlot {
    double v0, v1;
    int bad;
    unsigned gen;
    int pad0, pad1;
};

template <class Real, class Acc>
struct RingPcgArgs {
    BsrView<Real> a;
    int nnz;                     // stored upper blocks
    int ntiles;
    const int* desc;             // kRingDescInts per tile
    const Real* b;
    const Real* minv;
    Real* x;
    Real* r;
    Real* sd0;                   // {s.xyz, 0, d.xyz, 0} per row, ping-ponged
    Real* sd1;
    Real* q4;                    // {q.xyz, 0} per row
    ExSlot* slots;               // [2][grid]
    GridSync* sync;              // err flag
    int max_iterations;
    Acc tolerance;
    int skip_on_flags;
    int integrate;
    Real dt;
    const int* dyn_to_node;
    Real* node_x;
    Real* node_v;
    unsigned* flags;
    DevStats* stats;
};

// ------------------------------------------------------------------ batched PCG
// Batched per-body solve (pk_pcg_batch.cu).  parts: 8 ints per block {body, first row,
// end row, index in the body's group, first block of the group, group size, 0, 0}.
constexpr int kBatchThreads = 256;

struct BatchBodyStats {
    int iterations;
    int converged;
    double residual_norm;
    unsigned flags;
    int pad;
};

template <class Real, class Acc>
struct BatchPcgArgs {
    BsrView<Real> a;
    int nnz;
    const int* parts;
    const Real* b;
    const Real* minv;
    Real* x;
    Real* r;
    Real* sd0;
    Real* sd1;
    Real* q4;
    ExSlot* slots;   // [2][grid]
    GridSync* sync;  // err flag
    int max_iterations;
    Acc tolerance;
    int skip_on_flags;
    int integrate;
    Real dt;
    const int* dyn_to_node;
    Real* node_x;
    Real* node_v;
    unsigned* flags;
    unsigned* missing;
    DevStats* stats;
    BatchBodyStats* body_stats;
};

// ------------------------------------------------------------------ part-resident PCG
// The part-resident ("slab") PCG kernel (pk_pcg_slab.cu; layout in pk_slab_plan.h): one
// block per part, FP32 storage.  Shared memory: the window's search directions
// (kSlabWinCap x 3 floats), the ring of kSlabStages tile stages, the part's tile table,
// and for the symmetric stream form the consumer groups' transposed-product rings.
constexpr int kSlabGroupWarps = 4;
constexpr int kSlabConsumerWarps = kSlabGroups * kSlabGroupWarps;
// + one producer warp (the stream) and one halo warp (the window's halo rows, while the
// consumers stream the part's interior tiles)
constexpr int kSlabThreads = 32 * (kSlabConsumerWarps + 2);
constexpr size_t kSlabWinBytes = 12 * size_t(kSlabWinCap);
constexpr size_t kSlabRingOffset = kSlabWinBytes;
constexpr size_t kSlabTableOffset = kSlabRingOffset + size_t(kSlabStages) * kSlabStageBytes;
constexpr size_t kSlabFullSmemBytes = kSlabTableOffset + 16 * size_t(kSlabMaxTiles);
constexpr size_t kSlabSymTableOffset = kSlabRingOffset + size_t(kSlabStages) * kSymStageBytes;
constexpr size_t kSlabSymTpOffset = kSlabSymTableOffset + 16 * size_t(kSlabMaxTiles);
constexpr size_t kSlabSymSmemBytes = kSlabSymTpOffset + 12 * size_t(kSlabGroups) * kSymRingSlots;
constexpr size_t kSlabSmemBytes = kSlabFullSmemBytes > kSlabSymSmemBytes ? kSlabFullSmemBytes : kSlabSymSmemBytes;
static_assert(kSlabStages % kSlabGroups == 0, "a stage must always return to the same consumer group");
static_assert(kSlabWinBytes % 128 == 0 && kSlabStageBytes % 128 == 0 && kSymStageBytes % 128 == 0,
              "stages must stay 128-byte aligned");
static_assert(kSlabSmemBytes + 2048 <= 232448, "dynamic + static shared memory must fit one block per SM");
static_assert(kSymRows == 2 * kSlabRows, "a symmetric tile is two passes of the group's rows");
static_assert(kSlabRows * kSlabLanesPerRow == 32 * kSlabGroupWarps, "one tile row per lane group");
static_assert(kSlabRowThreads == 32 * kSlabConsumerWarps, "the consumer warps own the rows");
static_assert(kSlabGroups * kSlabRowsPerThread * 16 <= 512, "row records must fit tensor memory");

// A part_info row whose group is {kSlabNoGroup, 0}: the block has no part in that round.
constexpr int kSlabNoGroup = -1;

// Round table of the per-body (batched) launch, rebuilt on the device before every solve
// from the previous solve's per-body iteration counts (pk_pcg_slab.cu,
// slab_schedule_kernel).  Bodies are placed largest estimated work (duration x parts)
// first; a body of k parts takes the k consecutive blocks that are free earliest (ties:
// the lowest first block), all in one round: the round after the latest of those blocks' earlier rounds
// (blocks that reach it sooner idle through the rounds in between, which costs them
// nothing).  Estimated duration of a body: iterations x (c0 + kSlabSchedRowUs x its
// largest part's rows), c0 = kSlabSchedMultiUs for several parts (grid exchanges),
// kSlabSchedSingleUs for one -- per-iteration costs measured on B200; iterations = the
// body's count in the previous solve, or the iteration cap before the first.
constexpr int kSlabSchedThreads = 256;
constexpr int kSlabSchedMaxGrid = 256;
constexpr int kSlabSchedMaxSort = 2048;  // bodies it places (more: the batched layout does not apply)
constexpr float kSlabSchedMultiUs = 8.0f, kSlabSchedSingleUs = 4.0f, kSlabSchedRowUs = 0.012f;

struct SlabScheduleArgs {
    int grid;                  // blocks of the launch (<= kSlabSchedMaxGrid)
    int rounds;                // rounds of the table (>= the number of bodies placed)
    int nbodies;               // bodies with rows
    const int* body_part0;     // [nbodies] first part (plan numbering); a body's parts are consecutive
    const int* body_parts;     // [nbodies] its parts
    const int* plan_info;      // [parts] x kSlabPartInts
    const int* plan_body;      // [parts]
    const BatchBodyStats* body_stats;  // the previous solve's, by body id
    int nstats;                // entries of body_stats
    int max_iterations;
    int* out_info;             // [rounds][grid] x kSlabPartInts
    int* out_body;             // [rounds][grid]
    int* out_rounds;           // [grid]: rounds each block runs
    unsigned* flags;           // kFlagBreakdown when a body finds no room (the host sizes the table)
};

template <class Acc>
struct SlabPcgArgs {
    int n;                       // dynamic rows
    int rounds;                  // parts per block, taken in order (1 for the coupled solve)
    const int* block_rounds;     // [grid]: rounds block b runs (NULL: all)
    const int* part_info;        // [rounds][grid] x kSlabPartInts
    const int4* tile_desc;       // per tile: stream offset / 16, bytes, first local row, rows
    int tile_count;
    int halo_count;
    const unsigned char* stream;
    unsigned long long stream_bytes;
    const int* halo_src;         // slab index of each halo row
    const unsigned char* exported;  // per slab row: 1 when another part's window holds it
    const int* perm;             // slab index -> dynamic row
    const float* b;              // per dynamic row
    const float* minv;
    float* x;                    // per dynamic row: delta-v out
    float* qs;                   // 4 per slab row: q of phase A
    float* ss;                   // 4 per slab row: s published for the window passes
    ExSlot* slots;               // [rounds][2][grid]
    unsigned* group_count;       // [rounds][grid]: arrival counter of the group starting at each block (zeroed)
    GridSync* sync;              // err flag
    int max_iterations;
    Acc tolerance;
    int skip_on_flags;
    int integrate;
    float dt;
    const int* dyn_to_node;
    float* node_x;
    float* node_v;
    unsigned* flags;
    DevStats* stats;
    // Per-body solves (grouped): each block's body, the per-body statistics and the success
    // flags some body lacks; 0 / NULL for the coupled solve (one group of all blocks).
    int grouped;
    const int* part_body;        // [rounds][grid]
    int nbodies;
    BatchBodyStats* body_stats;
    unsigned* missing;
    // Stream form (pk_slab_plan.h): 0 full symmetric rows, 1 the symmetric form (each
    // in-sub-part block once, transposed products through the groups' shared-memory rings).
    int sym;
};

// ------------------------------------------------------------------ FP64 refinement
// Kernels of the outer true-residual refinement (pk_refine.cu).
constexpr int kRefineThreads = 256;

template <class Real>
struct RefineArgs {
    BsrView<Real> a;
    const Real* b;           // assembled right-hand side (kept while corrections run)
    const Real* minv;
    const double* x64;       // FP64 solution so far (NULL: x = 0)
    Real* rhs_out;           // residual rounded to Real: the next correction's rhs (may be NULL)
    double* partials;        // 2 per block: r^T M^-1 r, r.r
    int* bad;                // non-finite residual / update flags (cleared by the caller)
    // update
    Real* dx;                // delta-v in the storage type (written by the update)
    int integrate;
    Real dt;
    const int* dyn_to_node;
    Real* node_x;
    Real* node_v;
};

template <class Real>
int refine_residual_blocks(int n);
template <class Real>
cudaError_t launch_refine_residual(const RefineArgs<Real>& args, cudaStream_t stream);
template <class Real>
cudaError_t launch_refine_accumulate(double* x64, const Real* dx, int count, int first, cudaStream_t stream);
// Check pass (delta-v rounded and written to args.dx, finiteness into *args.bad), then, if
// args.integrate, the update of velocities and positions when nothing failed.
template <class Real>
cudaError_t launch_refine_update(const RefineArgs<Real>& args, cudaStream_t stream);

// The FP64 true residual of an FP32-stored step, from the tet data rather than the stored
// blocks: r = b - A x with b = dt f - dt^2 K v + dt m g and A = M + dt^2 K evaluated
// element by element in FP64 (FP64 rest data, FP64 polar rotation and stress), i.e.
//   r_a = sum over a's tets of -(dt S + dt^2 Q(v + x~)) g_a - dt c v_a + dt m g - m x_a
// (Q the folded stiffness, x~ the solution on the dynamic nodes and 0 elsewhere).
template <class Real>
struct ElemResidualArgs {
    int n;                          // dynamic rows
    int node_count;
    int tet_count;
    const int4* tet_nodes;
    const unsigned char* enabled;   // bit 0 simulated, bit 1 linear
    const double* dm_inv;           // FP64 rest data: 9 per tet
    const double* params;           // 4 per tet: rest volume, lambda, mu, damping
    const double* mass;             // FP64, per world node
    const Real* x;                  // node state (storage type)
    const Real* v;
    const int* node_to_dyn;
    const int* dyn_to_node;
    const int* inc_start;
    const int* inc_list;
    const Real* minv;               // block-Jacobi inverse (storage type), for r^T M^-1 r
    const double* x64;              // the FP64 solution so far (NULL: 0)
    double* vx;                     // scratch: per world node v + x~
    double* u;                      // scratch: per tet -(dt S + dt^2 Q(v + x~)), NaN when skipped
    double dt;
    double gravity[3];
    int linear;
    Real* rhs_out;                  // residual rounded to Real (may be NULL)
    double* partials;               // 2 per block: r^T M^-1 r, r.r
    int* bad;
};
template <class Real>
int elem_residual_blocks(int n);
template <class Real>
cudaError_t launch_elem_residual(const ElemResidualArgs<Real>& args, cudaStream_t stream);

// ------------------------------------------------------------------ adjoint step
// Backward element kernel (pk_adjoint.cu): per tet, the sensitivities of
// J = dt w.f(x) - dt^2 w.K(x) z to the tet's node positions (12 doubles) and to its
// log Young's modulus.
template <class Real>
struct AdjointArgs {
    int tet_count;
    const int4* nodes;
    const unsigned char* enabled;
    const Real* dm_inv;
    const Real* params;      // V, lambda, mu, damping
    const Real* x;           // per world node
    const Real* v;
    const int* node_to_dyn;
    const double* w;         // adjoint solution, per dynamic row
    const double* du;        // the step's delta-v, per dynamic row
    double dt;
    int linear;
    unsigned* flags;
    double* tet_grad;        // out: 12 per tet
    double* tet_theta;       // out: 1 per tet
};

// Launchers (pk_kernels.cu).  All asynchronous on `stream`.
template <class Real>
cudaError_t launch_tet_kernel(const AssemblyArgs<Real>& args, bool fp64_polar_fallback, cudaStream_t stream);
// The static part of the tet records (DmInv and the material of every tet).
template <class Real>
cudaError_t launch_tet_pack(const Real* dm_inv, const Real* params, Real* rec, int tet_count, cudaStream_t stream);
template <class Real>
cudaError_t launch_visual_kernel(int kind, const int* nodes, const float* weights, const unsigned char* live, int count,
                                 const Real* x, float* verts, float* normals, cudaStream_t stream);
template <class Real>
cudaError_t launch_sphere_contacts(const int* nodes, const unsigned char* flags, const Real* x, int tet_count,
                                   const Real* center, Real radius, int max_out, int* count, int* out_tet,
                                   Real* out_point, cudaStream_t stream);
// Per point connection, before the row kernel: its weighted point and velocity, whether it
// applies this step, and its force (args.conn_eval).
template <class Real>
cudaError_t launch_conn_kernel(const AssemblyArgs<Real>& args, cudaStream_t stream);
template <class Real>
cudaError_t launch_row_kernel(const AssemblyArgs<Real>& args, int max_row_blocks, cudaStream_t stream);
// Builds AssemblyArgs::inc_slot for the pattern, the incidences and the tets' nodes.
cudaError_t launch_inc_slot_kernel(int n, const int* row_start, const int* col, const int* inc_start,
                                   const int* inc_list, const int4* tet_nodes, const int* node_to_dyn, unsigned* out,
                                   cudaStream_t stream);
template <class Real, class Acc>
cudaError_t launch_pcg_kernel(const PcgArgs<Real, Acc>& args, int grid, int threads, cudaStream_t stream);
// Largest cooperative grid (one wave) for the staged (args.ntiles > 0) or unstaged kernel.
template <class Real, class Acc>
int pcg_max_grid(int threads, bool staged);
template <class Real>
cudaError_t launch_spmv_kernel(const BsrView<Real>& a, const Real* x, Real* y, cudaStream_t stream);
template <class Real>
cudaError_t launch_adjoint_tet_kernel(const AdjointArgs<Real>& args, cudaStream_t stream);
// Batched per-body PCG (pk_pcg_batch.cu): cooperative, one block per body part.
template <class Real, class Acc>
cudaError_t launch_pcg_batch_kernel(const BatchPcgArgs<Real, Acc>& args, int grid, cudaStream_t stream);
template <class Real, class Acc>
int pcg_batch_max_grid();
// Ring-staged PCG (pk_pcg_ring.cu): one block of kRingThreads per SM.
template <class Real, class Acc>
cudaError_t launch_pcg_ring_kernel(const RingPcgArgs<Real, Acc>& args, int grid, cudaStream_t stream);
template <class Real, class Acc>
int pcg_ring_max_grid();

// Part-resident PCG (pk_pcg_slab.cu): cooperative, one block of kSlabThreads per part.
template <class Acc>
cudaError_t launch_pcg_slab_kernel(const SlabPcgArgs<Acc>& args, int grid, cudaStream_t stream);
cudaError_t launch_slab_schedule_kernel(const SlabScheduleArgs& args, cudaStream_t stream);
template <class Acc>
int pcg_slab_max_grid();
// Writes the assembled upper blocks and their transposes into the slab stream, tile by
// tile (tile_desc: 4 ints per tile; tile_entry0: ntiles + 1 offsets into fill_src).
cudaError_t launch_slab_fill_kernel(const float* values, int nnz, const int* tile_desc, const int* tile_entry0,
                                    int ntiles, const unsigned* fill_src, int nentries, float* stream,
                                    unsigned long long stream_floats, int sym, cudaStream_t stream_);

constexpr int kPcgThreads = 512;

}  // namespace pk
