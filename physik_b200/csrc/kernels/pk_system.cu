// pk_system.cu -- implementation of the C ABI in include/pkcuda.h: device buffers of
// one soft-body system, uploads of the host-built topology, and the launch sequence
// of one implicit substep (tet kernel, row kernel, cooperative PCG kernel).
#include <cuda_runtime.h>

#include <algorithm>
#include <iterator>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <memory>
#include <vector>

#include "../../../include/pkcuda.h"
#include "pk_kernels.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg)
{
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return PK_ERR_CUDA;
}

#define PK_CHECK(...)                                              \
    do {                                                           \
        cudaError_t e_ = (__VA_ARGS__);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #__VA_ARGS__); \
    } while (0)

// Owned device allocation; freed on reset / destruction.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    void reset()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    // Every allocation carries kSlack extra bytes so bulk copies widened to 16-byte
    // boundaries (at most 4 elements past an array's end) stay inside it.
    static constexpr size_t kSlack = 1024;
    cudaError_t ensure(size_t want)
    {
        if (want <= bytes && p) return cudaSuccess;
        reset();
        if (want == 0) want = 16;
        cudaError_t e = cudaMalloc(&p, want + kSlack);
        if (e == cudaSuccess) bytes = want;
        return e;
    }
    template <class T>
    T* as() const
    {
        return static_cast<T*>(p);
    }
    ~DevBuf() { reset(); }
};

template <class Real>
std::vector<Real> narrow(const double* src, size_t n)
{
    std::vector<Real> out(n);
    for (size_t i = 0; i < n; ++i) out[i] = static_cast<Real>(src[i]);
    return out;
}

int device_count_safe()
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// Builds the transpose index of an upper BSR (for row r: blocks (c, r) with c < r).
void build_transpose(int n, const int* row_start, const int* col, std::vector<int>& lt_start, std::vector<int>& lt_row,
                     std::vector<int>& lt_block)
{
    lt_start.assign(static_cast<size_t>(n) + 1, 0);
    for (int r = 0; r < n; ++r)
        for (int k = row_start[r]; k < row_start[r + 1]; ++k)
            if (col[k] != r) lt_start[col[k] + 1]++;
    for (int r = 0; r < n; ++r) lt_start[r + 1] += lt_start[r];
    lt_row.assign(static_cast<size_t>(lt_start[n]), 0);
    lt_block.assign(static_cast<size_t>(lt_start[n]), 0);
    std::vector<int> fill(lt_start.begin(), lt_start.end() - 1);
    for (int r = 0; r < n; ++r)
        for (int k = row_start[r]; k < row_start[r + 1]; ++k) {
            const int c = col[k];
            if (c == r) continue;
            const int at = fill[c]++;
            lt_row[at] = r;
            lt_block[at] = k;
        }
}

// Greedy SpMV tiles for the staged PCG: consecutive rows, at most `rows` per tile, with
// the 16-byte-widened row / upper-block / transpose spans inside the shared-memory caps.
// Each tile becomes 8 ints {ra, rb, rs0, row words, k0, blocks, e0, transpose entries}.
// Returns false when a single row does not fit (the unstaged kernel is used then).
bool build_tiles(int n, const int* row_start, const std::vector<int>& lt_start, int rows, std::vector<int>& desc)
{
    desc.clear();
    auto span = [&](int a, int b, int* out) {
        const int rs0 = a & ~3, rs1 = (b + 1 + 3) & ~3;
        const int k0 = row_start[a] & ~3, k1 = (row_start[b] + 3) & ~3;
        const int e0 = lt_start[a] & ~3, e1 = (lt_start[b] + 3) & ~3;
        if (out) {
            out[0] = a; out[1] = b; out[2] = rs0; out[3] = rs1 - rs0;
            out[4] = k0; out[5] = k1 - k0; out[6] = e0; out[7] = e1 - e0;
        }
        return rs1 - rs0 <= pk::kTileRowCap && k1 - k0 <= pk::kTileCapU && e1 - e0 <= pk::kTileCapL &&
               k1 > k0;
    };
    int a = 0;
    while (a < n) {
        int b = a;
        while (b < n && b - a < rows && span(a, b + 1, nullptr)) ++b;
        if (b == a) return false;
        int d[8];
        span(a, b, d);
        desc.insert(desc.end(), d, d + 8);
        a = b;
    }
    return true;
}

bool staging_enabled()
{
    const char* e = std::getenv("PK_PCG_STAGED");
    return !(e && e[0] == '0');
}

// Which PCG kernel a system uses: the part-resident kernel when its layout applies (FP32
// storage, windows that fit shared memory), else the ring-staged kernel when its tiling
// fits, else the TMA-staged or the unstaged one.  PK_PCG_KERNEL=slab / ring / staged /
// plain asks for one (-1: automatic, 0 ring, 1 staged, 2 plain, 3 slab).
int requested_kernel()
{
    const char* e = std::getenv("PK_PCG_KERNEL");
    if (e && std::strcmp(e, "ring") == 0) return 0;
    if (e && std::strcmp(e, "staged") == 0) return 1;
    if (e && std::strcmp(e, "plain") == 0) return 2;
    if (e && std::strcmp(e, "slab") == 0) return 3;
    return -1;
}

// Tiles of the ring-staged PCG kernel (pk::RingTile caps): consecutive rows, at most
// kRows per tile, grown while the row words (widened to 4) and the upper-block and
// transposed-entry spans (widened to multiples of 4) fit a ring stage.  Each tile is
// kRingDescInts ints {ra, rb, rs0, row words, k0, blocks, e0, transposed entries}.
// Returns false when a single row does not fit (an older kernel is used then).
template <class Real>
bool build_ring_tiles(int n, const int* row_start, const std::vector<int>& lts, std::vector<int>& desc)
{
    using T = pk::RingTile<Real>;
    desc.clear();
    auto span = [&](int a, int b, int* out) {
        const int rs0 = a & ~3, rs1 = (b + 1 + 3) & ~3;
        const int k0 = row_start[a] & ~3, k1 = (row_start[b] + 3) & ~3;
        const int e0 = lts[a] & ~3, e1 = (lts[b] + 3) & ~3;
        if (out) {
            const int d[pk::kRingDescInts] = {a, b, rs0, rs1 - rs0, k0, k1 - k0, e0, e1 - e0};
            std::copy(d, d + pk::kRingDescInts, out);
        }
        return rs1 - rs0 <= T::kRsCap && k1 - k0 <= T::kCapU && e1 - e0 <= T::kCapL && k1 > k0;
    };
    int a = 0;
    while (a < n) {
        int b = a;
        while (b < n && b - a < T::kRows && span(a, b + 1, nullptr)) ++b;
        if (b == a) return false;
        int d[pk::kRingDescInts];
        span(a, b, d);
        desc.insert(desc.end(), d, d + pk::kRingDescInts);
        a = b;
    }
    return true;
}

}  // namespace

struct pk_system {
    int device = 0;
    int precision = PK_PREC_MIXED;
    cudaStream_t stream = nullptr;
    int node_count = 0, tet_count = 0, dyn_count = 0, nnz = 0, lt_count = 0, inc_count = 0, max_row = 0;
    bool have_nodes = false, have_tets = false, have_pattern = false;
    bool diag_first = false;  // every row starts with its diagonal block (needed by the row kernel)
    int pcg_grid_override = 0;
    int pcg_max_grid = 0;         // cooperative wave of the unstaged PCG kernel
    int pcg_max_grid_staged = 0;  // cooperative wave of the staged PCG kernel
    int ntiles = 0;               // staged SpMV tiles (0: unstaged kernel)
    DevBuf tiles;
    int ring_tiles = 0;           // ring-staged PCG tiles (0: not used)
    int ring_max_grid = 0;
    DevBuf ring_desc, q4, slots;
    // transient point connections (cleared by set_pattern)
    int conn_count = 0;
    DevBuf conn_nodes, conn_params, conn_eval, conn_inc_start, conn_inc_list;
    // host-emitted blocks and forces of custom components (cleared by set_pattern)
    bool ext_on = false, ext_force_on = false;
    int ext_count = 0;
    DevBuf ext_blocks, ext_nodes, ext_rhs_start, ext_rhs_list, ext_mat_start, ext_mat_list, ext_force;
    // batched per-body solve
    bool batched = false;
    std::vector<int> seg_start;   // body row ranges: [seg_start[b], seg_start[b+1])
    int batch_parts = 0;
    int batch_max_grid = 0;
    int batch_min_rows = 64;      // smallest part a body is cut into (autotuned)
    DevBuf batch_parts_buf, body_stats;
    // part-resident PCG (FP32 storage): layout built lazily at the first solve
    bool slab_tried = false;
    bool slab_filled = false;     // the block stream holds the current values
    int slab_parts = 0;           // blocks of the slab kernel (0: layout not available)
    int slab_tile_count = 0, slab_halo_count = 0;
    bool slab_for_bodies = false;   // the layout is the per-body one (batched solve)
    bool batch_slab = true;         // batched solve: part-resident kernel where it applies
    int slab_rounds = 0;            // parts per block of the one launch (the per-body layout's rounds)
    int slab_grid = 0;              // blocks of the launch
    // per-body layout: the round table is rebuilt on the device before every solve
    int slab_sched_bodies = 0;
    DevBuf slab_plan_info, slab_plan_body, slab_body_part0, slab_body_parts, slab_block_rounds;
    // The round table is built on a side stream while the step assembles (fork at the
    // step's start, join before the solve).
    cudaStream_t sched_stream = nullptr;
    cudaEvent_t sched_fork = nullptr, sched_join = nullptr;
    bool sched_pending = false;
    DevBuf slab_part_body, slab_gcount;
    int slab_max_grid = 0;
    std::string slab_reason;      // why the layout does not apply
    unsigned long long slab_stream_bytes = 0;
    bool slab_sym = false;        // the layout is the symmetric stream form
    DevBuf slab_part_info, slab_tiles, slab_stream, slab_halo, slab_perm, slab_fill_src, slab_tile_e0;
    DevBuf slab_export;  // per slab row: held by another part's window
    int slab_fill_entries = 0;
    DevBuf slab_qs, slab_ss;
    // FP64 outer true-residual refinement (FP32 storage, unbatched): passes, buffers
    int refine_passes = 0;
    DevBuf ref_x64, ref_rhs, ref_part, ref_bad;
    // kernel selection: -1 automatic (slab, else ring, else staged, else plain), 0 ring,
    // 1 staged, 2 plain, 3 slab
    int kernel_choice = -1;
    int last_kernel = -1;         // kernel of the last solve (4: batched), blocks it ran on
    int last_blocks = 0;
    int staged_rows = 0;          // rows per staged tile (0: chosen from the grid)
    std::vector<int> h_row_start, h_lts;  // host copies for re-tiling
    // host copies for the adjoint step's assembly of node sensitivities
    std::vector<int> h_node_to_dyn, h_dyn_to_node, h_tet_nodes;
    std::vector<unsigned char> h_enabled;
    std::vector<double> h_mass, h_damping;
    DevBuf adj_w, adj_du, adj_grad, adj_theta;
    bool assembled = false;       // a step has assembled the system at least once
    // CUDA graph of one step
    bool use_graph = false;
    cudaGraphExec_t graph_exec = nullptr;
    pk_step_params graph_params{};
    int graph_kernels = 0;
    // nodes; snap_x: positions at the start of the last substep (pk_system_snapshot_positions)
    DevBuf x, v, mass, node_to_dyn, snap_x;
    DevBuf contact_count, contact_tet, contact_point;  // pk_system_sphere_contacts
    bool have_snapshot = false;
    // tets
    DevBuf tet_nodes, tet_enabled, dm_inv, tet_params, tet_rec;
    // rows
    DevBuf dyn_to_node, row_start, col, lt_start, lt_row, lt_block, inc_start, inc_list, values, rhs, minv;
    DevBuf inc_slot;        // per incidence: the row slots of the tet's nodes (built on first use)
    // FP64 rest data and masses of an FP32-stored system, for the refinement's element-
    // wise FP64 residual (FP64 systems use their own arrays), and its scratch.
    DevBuf dm_inv64, params64, mass64, elem_u, elem_vx;
    bool rest64_ok = false;  // pk_system_set_rest64 matches the current tets and nodes
    bool slots_ok = false;  // inc_slot matches the pattern, incidences, tets and node rows
    // solver
    DevBuf px, pr, psd0, psd1, pq, part_a, part_b, part_bad, sync, stats;
    pk::DevStats* host_stats = nullptr;  // pinned
    bool stats_pending = false;
    // timing
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::array<int, 3>> ev_pending;  // indices into ev_pool
    double t_assemble = 0, t_solve = 0;
    int timed_steps = 0;
    long long launches = 0;

    size_t rsize() const { return precision == PK_PREC_FP64 ? sizeof(double) : sizeof(float); }
};

namespace {

bool row_lanes_enabled();

template <class Real>
pk::AssemblyArgs<Real> assembly_args(pk_system* s, const pk_step_params& p)
{
    pk::AssemblyArgs<Real> a{};
    a.tets.tet_count = s->tet_count;
    a.tets.nodes = s->tet_nodes.as<int4>();
    a.tets.enabled = s->tet_enabled.as<unsigned char>();
    a.tets.dm_inv = s->dm_inv.as<Real>();
    a.tets.params = s->tet_params.as<Real>();
    a.tets.rec = s->tet_rec.as<Real>();
    a.a.n = s->dyn_count;
    a.a.row_start = s->row_start.as<int>();
    a.a.col = s->col.as<int>();
    a.a.values = s->values.as<Real>();
    a.a.lt_start = s->lt_start.as<int>();
    a.a.lt_row = s->lt_row.as<int>();
    a.a.lt_block = s->lt_block.as<int>();
    a.node_count = s->node_count;
    a.dyn_to_node = s->dyn_to_node.as<int>();
    a.node_to_dyn = s->node_to_dyn.as<int>();
    a.mass = s->mass.as<Real>();
    a.x = s->x.as<Real>();
    a.v = s->v.as<Real>();
    a.x_out = s->x.as<Real>();
    a.inc_start = s->inc_start.as<int>();
    a.inc_list = s->inc_list.as<int>();
    a.inc_slot = s->slots_ok ? s->inc_slot.as<unsigned>() : nullptr;
    a.row_lanes = row_lanes_enabled() ? 1 : 0;
    a.values = s->values.as<Real>();
    a.rhs = s->rhs.as<Real>();
    a.minv = s->minv.as<Real>();
    a.dt = static_cast<Real>(p.dt);
    for (int i = 0; i < 3; ++i) a.gravity[i] = static_cast<Real>(p.gravity[i]);
    a.use_jacobi = p.use_jacobi;
    a.linear = p.linear;
    a.explicit_mode = p.explicit_mode;
    pk::DevStats* st = s->stats.as<pk::DevStats>();
    a.flags = &st->flags;
    a.stats = st;
    if (s->conn_count > 0) {
        a.conn_count = s->conn_count;
        a.conn_nodes = s->conn_nodes.as<int4>();
        a.conn_params = s->conn_params.as<Real>();
        a.conn_eval = s->conn_eval.as<Real>();
        a.conn_inc_start = s->conn_inc_start.as<int>();
        a.conn_inc_list = s->conn_inc_list.as<int>();
    }
    if (s->ext_on) {
        a.ext_blocks = s->ext_blocks.as<Real>();
        a.ext_nodes = s->ext_nodes.as<int2>();
        a.ext_rhs_start = s->ext_rhs_start.as<int>();
        a.ext_rhs_list = s->ext_rhs_list.as<int>();
        a.ext_mat_start = s->ext_mat_start.as<int>();
        a.ext_mat_list = s->ext_mat_list.as<int>();
        a.ext_force = s->ext_force_on ? s->ext_force.as<Real>() : nullptr;
    }
    return a;
}

template <class Real, class Acc>
pk::PcgArgs<Real, Acc> pcg_args(pk_system* s, const pk_step_params& p, int skip_on_flags)
{
    pk::PcgArgs<Real, Acc> a{};
    a.a.n = s->dyn_count;
    a.a.row_start = s->row_start.as<int>();
    a.a.col = s->col.as<int>();
    a.a.values = s->values.as<Real>();
    a.a.lt_start = s->lt_start.as<int>();
    a.a.lt_row = s->lt_row.as<int>();
    a.a.lt_block = s->lt_block.as<int>();
    a.b = s->rhs.as<Real>();
    a.minv = s->minv.as<Real>();
    a.x = s->px.as<Real>();
    a.r = s->pr.as<Real>();
    a.sd0 = s->psd0.as<Real>();
    a.sd1 = s->psd1.as<Real>();
    a.q = s->pq.as<Real>();
    a.part_a = s->part_a.as<Acc>();
    a.part_b = s->part_b.as<Acc>();
    a.part_bad = s->part_bad.as<int>();
    a.sync = s->sync.as<pk::GridSync>();
    a.max_iterations = p.max_iterations;
    a.tolerance = static_cast<Acc>(static_cast<Real>(p.tolerance));
    a.skip_on_flags = skip_on_flags;
    a.integrate = p.integrate;
    a.dt = static_cast<Real>(p.dt);
    a.dyn_to_node = s->dyn_to_node.as<int>();
    a.node_x = s->x.as<Real>();
    a.node_v = s->v.as<Real>();
    pk::DevStats* st = s->stats.as<pk::DevStats>();
    a.flags = &st->flags;
    a.stats = st;
    a.ntiles = s->ntiles;
    a.tile_desc = s->tiles.as<int>();
    return a;
}

template <class Real, class Acc>
int max_grid_for(pk_system* s)
{
    if (!s->pcg_max_grid) s->pcg_max_grid = pk::pcg_max_grid<Real, Acc>(pk::kPcgThreads, false);
    if (!s->pcg_max_grid_staged) s->pcg_max_grid_staged = pk::pcg_max_grid<Real, Acc>(pk::kPcgThreads, true);
    return std::max(s->pcg_max_grid, s->pcg_max_grid_staged);
}

constexpr int kRowsPerBlockTarget = 32;

template <class Real, class Acc>
int pcg_grid_for(pk_system* s)
{
    max_grid_for<Real, Acc>(s);
    if (s->ntiles > 0) {
        // Staged kernel: whole tiles per block, one cooperative wave.
        const int mxs = s->pcg_max_grid_staged;
        if (mxs <= 0) return 0;
        const int g = s->pcg_grid_override > 0 ? s->pcg_grid_override : mxs;
        return std::max(1, std::min(std::min(mxs, g), s->ntiles));  // tiles are dealt round-robin
    }
    const int mx = s->pcg_max_grid;
    if (mx <= 0) return 0;
    if (s->pcg_grid_override > 0) return std::min(mx, s->pcg_grid_override);
    // Enough blocks that each phase is one pass over its rows (16 lanes per row in the
    // SpMV), capped at one cooperative wave.
    const int want = (s->dyn_count + kRowsPerBlockTarget - 1) / kRowsPerBlockTarget;
    return std::max(1, std::min(mx, want));
}

int ensure_solver_buffers(pk_system* s, int grid_cap)
{
    const size_t rs = s->rsize();
    const size_t v3 = 3 * rs * static_cast<size_t>(std::max(1, s->dyn_count));
    const size_t rec = 8 * rs * static_cast<size_t>(std::max(1, s->dyn_count));  // {s, 0, d, 0} records
    PK_CHECK(s->px.ensure(v3));
    PK_CHECK(s->pr.ensure(v3));
    PK_CHECK(s->psd0.ensure(rec));
    PK_CHECK(s->psd1.ensure(rec));
    PK_CHECK(s->pq.ensure(v3));
    const size_t g = static_cast<size_t>(std::max(1, grid_cap));
    PK_CHECK(s->part_a.ensure(g * sizeof(double)));
    PK_CHECK(s->part_b.ensure(2 * g * sizeof(double)));
    PK_CHECK(s->part_bad.ensure(4 * g * sizeof(int)));
    PK_CHECK(s->sync.ensure(sizeof(pk::GridSync)));
    return PK_OK;
}

template <class Real, class Acc>
int ring_max_grid(pk_system* s)
{
    if (!s->ring_max_grid) s->ring_max_grid = pk::pcg_ring_max_grid<Real, Acc>();
    return s->ring_max_grid;
}

template <class Real, class Acc>
int ring_grid_for(pk_system* s)
{
    const int mx = ring_max_grid<Real, Acc>(s);
    if (mx <= 0) return 0;
    const int g = s->pcg_grid_override > 0 ? std::min(s->pcg_grid_override, mx) : mx;
    return std::max(1, std::min(g, s->ring_tiles));
}

template <class Real, class Acc>
int run_pcg_ring(pk_system* s, const pk_step_params& p, int skip_on_flags)
{
    const int grid = ring_grid_for<Real, Acc>(s);
    if (grid <= 0) return fail(PK_ERR_CUDA, "ring PCG kernel cannot be resident");
    if ((s->ring_tiles + grid - 1) / grid > pk::kRingMaxTilesPerBlock)
        return fail(PK_ERR_UNSUPPORTED, "ring PCG: too many tiles per block for this grid");
    const size_t rs = s->rsize();
    const size_t n = static_cast<size_t>(std::max(1, s->dyn_count));
    PK_CHECK(s->q4.ensure(4 * rs * n));
    PK_CHECK(s->slots.ensure(2 * sizeof(pk::ExSlot) * static_cast<size_t>(grid)));
    PK_CHECK(cudaMemsetAsync(s->slots.p, 0, 2 * sizeof(pk::ExSlot) * static_cast<size_t>(grid), s->stream));
    PK_CHECK(cudaMemsetAsync(s->sync.p, 0, sizeof(pk::GridSync), s->stream));
    pk::RingPcgArgs<Real, Acc> a{};
    a.a.n = s->dyn_count;
    a.a.row_start = s->row_start.as<int>();
    a.a.col = s->col.as<int>();
    a.a.values = s->values.as<Real>();
    a.a.lt_start = s->lt_start.as<int>();
    a.a.lt_row = s->lt_row.as<int>();
    a.a.lt_block = s->lt_block.as<int>();
    a.nnz = s->nnz;
    a.ntiles = s->ring_tiles;
    a.desc = s->ring_desc.as<int>();
    a.b = s->rhs.as<Real>();
    a.minv = s->minv.as<Real>();
    a.x = s->px.as<Real>();
    a.r = s->pr.as<Real>();
    a.sd0 = s->psd0.as<Real>();
    a.sd1 = s->psd1.as<Real>();
    a.q4 = s->q4.as<Real>();
    a.slots = s->slots.as<pk::ExSlot>();
    a.sync = s->sync.as<pk::GridSync>();
    a.max_iterations = p.max_iterations;
    a.tolerance = static_cast<Acc>(static_cast<Real>(p.tolerance));
    a.skip_on_flags = skip_on_flags;
    a.integrate = p.integrate;
    a.dt = static_cast<Real>(p.dt);
    a.dyn_to_node = s->dyn_to_node.as<int>();
    a.node_x = s->x.as<Real>();
    a.node_v = s->v.as<Real>();
    pk::DevStats* st = s->stats.as<pk::DevStats>();
    a.flags = &st->flags;
    a.stats = st;
    PK_CHECK(pk::launch_pcg_ring_kernel<Real, Acc>(a, grid, s->stream));
    s->launches += 1;
    s->last_blocks = grid;
    return PK_OK;
}

template <class T>
int upload_raw(DevBuf& buf, const T* src, size_t n, cudaStream_t stream);
template <class Real>
int download_real(const DevBuf& buf, double* dst, size_t n, cudaStream_t stream);

void reset_slab(pk_system* s)
{
    s->slab_tried = false;
    s->slab_filled = false;
    s->slab_parts = 0;
    s->slab_reason.clear();
}

// Copies the assembled upper blocks (and their transposes) into the slab stream.
int slab_fill(pk_system* s)
{
    PK_CHECK(pk::launch_slab_fill_kernel(s->values.as<float>(), s->nnz, s->slab_tiles.as<int>(),
                                         s->slab_tile_e0.as<int>(), s->slab_tile_count,
                                         s->slab_fill_src.as<unsigned>(), s->slab_fill_entries,
                                         s->slab_stream.as<float>(), s->slab_stream_bytes / 4, s->slab_sym ? 1 : 0,
                                         s->stream));
    s->launches += 1;
    s->slab_filled = true;
    return PK_OK;
}

// PK_SLAB_FORM=full / sym asks for one stream form of the part-resident kernel's layout;
// by default the symmetric form where it applies, else the full rows.
// The part-resident kernel's stream form: full symmetric rows unless PK_SLAB_FORM asks for
// the symmetric form ("sym") or the symmetric form where it fits ("auto").  The full form
// is the default: on block128 it streams 1.5x the bytes but runs faster, the symmetric
// form's extra products, ring traffic and group barriers cost more than the bytes saved.
int requested_slab_form()
{
    const char* e = std::getenv("PK_SLAB_FORM");
    if (e && std::strcmp(e, "sym") == 0) return pk::kSlabSym;
    if (e && std::strcmp(e, "auto") == 0) return pk::kSlabAuto;
    return pk::kSlabFull;
}

bool slab_allowed(const pk_system* s)
{
    const int rk = requested_kernel();
    return s->precision != PK_PREC_FP64 && (rk == -1 || rk == 3) && s->dyn_count > 0 && s->have_pattern;
}

// Point connections may couple bodies: with any present the step solves one coupled
// system, as the reference always does.
bool batched_solve(const pk_system* s)
{
    return s->batched && s->seg_start.size() >= 2 && s->conn_count == 0 && s->ext_count == 0;
}

// Builds and uploads the part-resident kernel's layout if it has not been tried yet for
// this pattern and grid (synchronous: never called while a stream capture is open).
// Parts are cut by the rows' node positions at this moment.  Not applicable (too large
// a window, too long a row) leaves slab_parts at 0 and the reason in slab_reason.
template <class Acc>
int ensure_slab(pk_system* s)
{
    const bool bodies = batched_solve(s);
    if (s->slab_tried && s->slab_for_bodies != bodies) reset_slab(s);  // batched mode changed
    if (s->slab_tried || !slab_allowed(s)) return PK_OK;
    s->slab_tried = true;
    s->slab_for_bodies = bodies;
    s->slab_parts = 0;
    if (!s->slab_max_grid) s->slab_max_grid = pk::pcg_slab_max_grid<Acc>();
    int grid = s->slab_max_grid;
    if (s->pcg_grid_override > 0) grid = std::min(grid, s->pcg_grid_override);
    if (!bodies) grid = std::min(grid, std::max(1, s->dyn_count / 64));
    if (grid <= 0) {
        s->slab_reason = "kernel cannot be resident";
        return PK_OK;
    }
    const int n = s->dyn_count;
    // node positions -> per-row coordinates
    std::vector<double> nodes(3 * static_cast<size_t>(std::max(1, s->node_count)), 0.0);
    if (s->node_count > 0) {
        int rc = download_real<float>(s->x, nodes.data(), 3 * static_cast<size_t>(s->node_count), s->stream);
        if (rc) return rc;
    }
    std::vector<double> coords(3 * static_cast<size_t>(n));
    for (int r = 0; r < n; ++r)
        for (int a = 0; a < 3; ++a) coords[3 * (size_t)r + a] = nodes[3 * (size_t)s->h_dyn_to_node[r] + a];
    std::vector<int> col(static_cast<size_t>(s->nnz)), ltr(static_cast<size_t>(s->lt_count)),
        ltb(static_cast<size_t>(s->lt_count));
    PK_CHECK(cudaMemcpy(col.data(), s->col.p, col.size() * sizeof(int), cudaMemcpyDeviceToHost));
    if (s->lt_count > 0) {
        PK_CHECK(cudaMemcpy(ltr.data(), s->lt_row.p, ltr.size() * sizeof(int), cudaMemcpyDeviceToHost));
        PK_CHECK(cudaMemcpy(ltb.data(), s->lt_block.p, ltb.size() * sizeof(int), cudaMemcpyDeviceToHost));
    }
    pk::SlabPlan plan;
    const std::string why =
        bodies ? pk::build_slab_plan_batched(n, s->h_row_start.data(), col.data(), s->h_lts.data(), ltr.data(),
                                             ltb.data(), coords.data(), s->seg_start.data(),
                                             static_cast<int>(s->seg_start.size()) - 1, grid, plan, requested_slab_form())
               : pk::build_slab_plan(n, s->h_row_start.data(), col.data(), s->h_lts.data(), ltr.data(), ltb.data(),
                                     coords.data(), grid, plan, requested_slab_form());
    if (!why.empty()) {
        s->slab_reason = why;
        return PK_OK;
    }
    // Coupled solve: one round, block b takes part b.  Per-body solves: the device
    // scheduler (slab_schedule_kernel) places the bodies into the rounds of one launch
    // before every solve, from the previous solve's iteration counts; the plan's launches
    // only bound the blocks.
    int widest = 1;
    for (size_t l = 0; l + 1 < plan.launch_start.size(); ++l)
        widest = std::max(widest, plan.launch_start[l + 1] - plan.launch_start[l]);
    const int PI = pk::kSlabPartInts;
    int rounds = 1;
    std::vector<int> round_info, round_body;
    if (!bodies) {
        round_info.assign(plan.part_info.begin(), plan.part_info.end());
        round_body.assign(static_cast<size_t>(plan.parts), 0);
        widest = plan.parts;
        s->slab_sched_bodies = 0;
    } else {
        if (widest > pk::kSlabSchedMaxGrid) {
            s->slab_reason = "more blocks than the round scheduler holds";
            return PK_OK;
        }
        std::vector<int> part0, nparts;
        int kmax = 1;
        for (int p = 0; p < plan.parts;) {
            const int k = std::max(1, plan.part_info[static_cast<size_t>(PI) * p + 7]);
            part0.push_back(p);
            nparts.push_back(k);
            kmax = std::max(kmax, k);
            p += k;
        }
        const int nb = static_cast<int>(part0.size());
        if (nb > pk::kSlabSchedMaxSort) {
            s->slab_reason = "more bodies than the round scheduler places";
            return PK_OK;
        }
        // rounds: every placement raises a block's count by at most one, and the bodies
        // spread over the blocks a body of kmax parts leaves free
        const int spread = (nb + std::max(1, widest - kmax) - 1) / std::max(1, widest - kmax);
        rounds = std::max(1, std::min(nb, 4 * spread + 16));
        s->slab_sched_bodies = nb;
        int rc = upload_raw<int>(s->slab_plan_info, plan.part_info.data(), plan.part_info.size(), s->stream);
        if (!rc) rc = upload_raw<int>(s->slab_plan_body, plan.part_body.data(), plan.part_body.size(), s->stream);
        if (!rc) rc = upload_raw<int>(s->slab_body_part0, part0.data(), part0.size(), s->stream);
        if (!rc) rc = upload_raw<int>(s->slab_body_parts, nparts.data(), nparts.size(), s->stream);
        if (!rc) {
            std::vector<int> zero_rounds(static_cast<size_t>(widest), 0);
            rc = upload_raw<int>(s->slab_block_rounds, zero_rounds.data(), zero_rounds.size(), s->stream);
        }
        if (rc) return rc;
        round_info.assign(static_cast<size_t>(rounds) * widest * PI, 0);  // written by the scheduler
        round_body.assign(static_cast<size_t>(rounds) * widest, 0);
        if (!s->sched_stream) PK_CHECK(cudaStreamCreateWithFlags(&s->sched_stream, cudaStreamNonBlocking));
        if (!s->sched_fork) PK_CHECK(cudaEventCreateWithFlags(&s->sched_fork, cudaEventDisableTiming));
        if (!s->sched_join) PK_CHECK(cudaEventCreateWithFlags(&s->sched_join, cudaEventDisableTiming));
    }
    int rc = upload_raw<int>(s->slab_part_info, round_info.data(), round_info.size(), s->stream);
    if (!rc) rc = upload_raw<int>(s->slab_tiles, plan.tile_desc.data(), plan.tile_desc.size(), s->stream);
    if (!rc) rc = upload_raw<unsigned char>(s->slab_stream, plan.stream.data(), plan.stream.size(), s->stream);
    if (!rc && !plan.halo_src.empty())
        rc = upload_raw<int>(s->slab_halo, plan.halo_src.data(), plan.halo_src.size(), s->stream);
    if (!rc) rc = upload_raw<int>(s->slab_perm, plan.perm.data(), plan.perm.size(), s->stream);
    if (!rc) {
        std::vector<unsigned char> exported(static_cast<size_t>(n), 0);
        for (const int g : plan.halo_src)
            if (g >= 0 && g < n) exported[static_cast<size_t>(g)] = 1;
        rc = upload_raw<unsigned char>(s->slab_export, exported.data(), exported.size(), s->stream);
    }
    if (!rc) rc = upload_raw<unsigned>(s->slab_fill_src, plan.fill_src.data(), plan.fill_src.size(), s->stream);
    if (!rc) rc = upload_raw<int>(s->slab_tile_e0, plan.tile_entry0.data(), plan.tile_entry0.size(), s->stream);
    if (!rc) rc = upload_raw<int>(s->slab_part_body, round_body.data(), round_body.size(), s->stream);
    if (rc) return rc;
    const size_t round_blocks = static_cast<size_t>(rounds) * widest;
    PK_CHECK(s->slab_gcount.ensure(sizeof(unsigned) * round_blocks));
    PK_CHECK(s->slots.ensure(2 * sizeof(pk::ExSlot) * round_blocks));
    if (bodies) {
        // no earlier solve on this layout: the first round table assumes the iteration cap
        const size_t bytes = sizeof(pk::BatchBodyStats) * s->seg_start.size();
        PK_CHECK(s->body_stats.ensure(bytes));
        PK_CHECK(cudaMemsetAsync(s->body_stats.p, 0, bytes, s->stream));
    }
    s->slab_rounds = rounds;
    s->slab_grid = widest;
    const size_t rows = static_cast<size_t>(n);
    PK_CHECK(s->slab_qs.ensure(16 * rows));
    PK_CHECK(s->slab_ss.ensure(16 * rows));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    s->slab_stream_bytes = plan.stream.size();
    s->slab_sym = plan.sym;
    s->slab_tile_count = static_cast<int>(plan.tile_desc.size() / 4);
    s->slab_fill_entries = static_cast<int>(plan.fill_src.size());
    s->slab_halo_count = static_cast<int>(plan.halo_src.size());
    s->slab_parts = plan.parts;
    return PK_OK;
}

int ensure_slab_any(pk_system* s)
{
    if (s->precision == PK_PREC_FP32) return ensure_slab<float>(s);
    if (s->precision == PK_PREC_MIXED) return ensure_slab<double>(s);
    return PK_OK;
}

// The per-body round table for the next solve (slab_schedule_kernel) on `stream`.
int launch_slab_schedule(pk_system* s, int max_iterations, cudaStream_t stream)
{
    pk::SlabScheduleArgs sa{};
    sa.grid = s->slab_grid;
    sa.rounds = s->slab_rounds;
    sa.nbodies = s->slab_sched_bodies;
    sa.body_part0 = s->slab_body_part0.as<int>();
    sa.body_parts = s->slab_body_parts.as<int>();
    sa.plan_info = s->slab_plan_info.as<int>();
    sa.plan_body = s->slab_plan_body.as<int>();
    sa.body_stats = s->body_stats.as<pk::BatchBodyStats>();
    sa.nstats = static_cast<int>(s->seg_start.size()) - 1;
    sa.max_iterations = max_iterations;
    sa.out_info = s->slab_part_info.as<int>();
    sa.out_body = s->slab_part_body.as<int>();
    sa.out_rounds = s->slab_block_rounds.as<int>();
    sa.flags = &s->stats.as<pk::DevStats>()->flags;
    PK_CHECK(pk::launch_slab_schedule_kernel(sa, stream));
    s->launches += 1;
    return PK_OK;
}

template <class Real, class Acc>
int run_pcg_slab(pk_system* s, const pk_step_params& p, int skip_on_flags)
{
    if constexpr (!std::is_same<Real, float>::value) {
        return fail(PK_ERR_UNSUPPORTED, "part-resident PCG: FP32 storage only");
    } else {
        if (s->slab_parts <= 0 || s->slab_rounds < 1 || s->slab_grid < 1)
            return fail(PK_ERR_UNSUPPORTED, "part-resident PCG layout not available");
        const bool bodies = s->slab_for_bodies;
        const int nseg = static_cast<int>(s->seg_start.size()) - 1;
        int rc = ensure_solver_buffers(s, 1);
        if (rc) return rc;
        pk::DevStats* st = s->stats.as<pk::DevStats>();
        if (bodies) {
            // This solve's round table from the previous solve's iteration counts (built on
            // the side stream while the step assembled, or here), then the counts are
            // cleared for this solve.
            if (s->sched_pending) {
                PK_CHECK(cudaStreamWaitEvent(s->stream, s->sched_join, 0));
                s->sched_pending = false;
            } else {
                rc = launch_slab_schedule(s, p.max_iterations, s->stream);
                if (rc) return rc;
            }
            PK_CHECK(cudaMemsetAsync(s->body_stats.p, 0, sizeof(pk::BatchBodyStats) * static_cast<size_t>(nseg),
                                     s->stream));
        }
        if (!s->slab_filled) {
            rc = slab_fill(s);
            if (rc) return rc;
        }
        pk::SlabPcgArgs<Acc> a{};
        a.n = s->dyn_count;
        a.part_info = s->slab_part_info.as<int>();
        a.tile_desc = s->slab_tiles.as<int4>();
        a.tile_count = s->slab_tile_count;
        a.halo_count = s->slab_halo_count;
        a.stream = s->slab_stream.as<unsigned char>();
        a.stream_bytes = s->slab_stream_bytes;
        a.halo_src = s->slab_halo.as<int>();
        a.exported = s->slab_export.as<unsigned char>();
        a.perm = s->slab_perm.as<int>();
        a.b = s->rhs.as<float>();
        a.minv = s->minv.as<float>();
        a.x = s->px.as<float>();
        a.qs = s->slab_qs.as<float>();
        a.ss = s->slab_ss.as<float>();
        a.slots = s->slots.as<pk::ExSlot>();
        a.sync = s->sync.as<pk::GridSync>();
        a.max_iterations = p.max_iterations;
        a.tolerance = static_cast<Acc>(static_cast<float>(p.tolerance));
        a.skip_on_flags = skip_on_flags;
        a.integrate = p.integrate;
        a.dt = static_cast<float>(p.dt);
        a.dyn_to_node = s->dyn_to_node.as<int>();
        a.node_x = s->x.as<float>();
        a.node_v = s->v.as<float>();
        a.flags = &st->flags;
        a.stats = st;
        a.group_count = s->slab_gcount.as<unsigned>();
        a.grouped = bodies ? 1 : 0;
        a.nbodies = bodies ? nseg : 1;
        a.body_stats = bodies ? s->body_stats.as<pk::BatchBodyStats>() : nullptr;
        a.missing = &st->batch_missing;
        a.sym = s->slab_sym ? 1 : 0;
        // One persistent launch: every block takes its part of each round in turn (the
        // coupled solve: one round of all parts).
        const size_t round_blocks = static_cast<size_t>(s->slab_rounds) * s->slab_grid;
        PK_CHECK(cudaMemsetAsync(s->slots.p, 0, 2 * sizeof(pk::ExSlot) * round_blocks, s->stream));
        PK_CHECK(cudaMemsetAsync(s->slab_gcount.p, 0, sizeof(unsigned) * round_blocks, s->stream));
        PK_CHECK(cudaMemsetAsync(s->sync.p, 0, sizeof(pk::GridSync), s->stream));
        a.rounds = s->slab_rounds;
        a.block_rounds = bodies ? s->slab_block_rounds.as<int>() : nullptr;
        a.part_info = s->slab_part_info.as<int>();
        a.part_body = s->slab_part_body.as<int>();
        PK_CHECK(pk::launch_pcg_slab_kernel<Acc>(a, s->slab_grid, s->stream));
        s->launches += 1;
        s->last_kernel = bodies ? 5 : 3;
        s->last_blocks = s->slab_parts;
        return PK_OK;
    }
}

// Cuts every body (segment) into parts of about equal row count, one block each, so that
// all parts fit one cooperative wave.  parts: 8 ints per block (see pk::BatchPcgArgs).
int build_batch_parts(const std::vector<int>& seg, int capacity, int min_rows, std::vector<int>& parts)
{
    parts.clear();
    const int nseg = static_cast<int>(seg.size()) - 1;
    if (nseg <= 0 || capacity <= 0) return 0;
    const long long total = seg[nseg] - seg[0];
    long long rows_per_part = std::max<long long>(std::max(1, min_rows), (total + capacity - 1) / capacity);
    auto count = [&](long long R) {
        long long c = 0;
        for (int b = 0; b < nseg; ++b) {
            const long long rows = seg[b + 1] - seg[b];
            if (rows > 0) c += (rows + R - 1) / R;
        }
        return c;
    };
    while (count(rows_per_part) > capacity) rows_per_part += std::max<long long>(1, rows_per_part / 8);
    for (int b = 0; b < nseg; ++b) {
        const int rows = seg[b + 1] - seg[b];
        if (rows <= 0) continue;
        const int np = static_cast<int>((rows + rows_per_part - 1) / rows_per_part);
        const int g0 = static_cast<int>(parts.size() / 8);
        for (int i = 0; i < np; ++i) {
            const int a = seg[b] + static_cast<int>(static_cast<long long>(rows) * i / np);
            const int e = seg[b] + static_cast<int>(static_cast<long long>(rows) * (i + 1) / np);
            parts.insert(parts.end(), {b, a, e, i, g0, np, 0, 0});
        }
    }
    return static_cast<int>(parts.size() / 8);
}

// Builds and uploads the batched solve's part table if it is missing (synchronous: never
// called while a stream capture is open).
template <class Real, class Acc>
int ensure_batch_parts(pk_system* s)
{
    if (!s->batch_max_grid) s->batch_max_grid = pk::pcg_batch_max_grid<Real, Acc>();
    if (s->batch_parts <= 0) {
        std::vector<int> parts;
        const int np = build_batch_parts(s->seg_start, s->batch_max_grid, s->batch_min_rows, parts);
        if (np <= 0) return fail(PK_ERR_CUDA, "batched PCG: no resident blocks");
        int rc = upload_raw<int>(s->batch_parts_buf, parts.data(), parts.size(), s->stream);
        if (rc) return rc;
        s->batch_parts = np;
    }
    return PK_OK;
}

int ensure_batch_parts_any(pk_system* s)
{
    if (!s->batched || s->seg_start.size() < 2) return PK_OK;
    if (s->precision == PK_PREC_FP32) return ensure_batch_parts<float, float>(s);
    if (s->precision == PK_PREC_MIXED) return ensure_batch_parts<float, double>(s);
    return ensure_batch_parts<double, double>(s);
}

template <class Real, class Acc>
int run_pcg_batch(pk_system* s, const pk_step_params& p, int skip_on_flags)
{
    int rc0 = ensure_batch_parts<Real, Acc>(s);
    if (rc0) return rc0;
    const int grid = s->batch_parts;
    const int nseg = static_cast<int>(s->seg_start.size()) - 1;
    int rc = ensure_solver_buffers(s, 1);
    if (rc) return rc;
    const size_t rs = s->rsize();
    PK_CHECK(s->q4.ensure(4 * rs * static_cast<size_t>(std::max(1, s->dyn_count))));
    PK_CHECK(s->slots.ensure(2 * sizeof(pk::ExSlot) * static_cast<size_t>(grid)));
    PK_CHECK(s->body_stats.ensure(sizeof(pk::BatchBodyStats) * static_cast<size_t>(std::max(1, nseg))));
    PK_CHECK(cudaMemsetAsync(s->slots.p, 0, 2 * sizeof(pk::ExSlot) * static_cast<size_t>(grid), s->stream));
    PK_CHECK(cudaMemsetAsync(s->body_stats.p, 0, sizeof(pk::BatchBodyStats) * static_cast<size_t>(std::max(1, nseg)),
                             s->stream));
    PK_CHECK(cudaMemsetAsync(s->sync.p, 0, sizeof(pk::GridSync), s->stream));
    pk::BatchPcgArgs<Real, Acc> a{};
    a.a.n = s->dyn_count;
    a.a.row_start = s->row_start.as<int>();
    a.a.col = s->col.as<int>();
    a.a.values = s->values.as<Real>();
    a.a.lt_start = s->lt_start.as<int>();
    a.a.lt_row = s->lt_row.as<int>();
    a.a.lt_block = s->lt_block.as<int>();
    a.nnz = s->nnz;
    a.parts = s->batch_parts_buf.as<int>();
    a.b = s->rhs.as<Real>();
    a.minv = s->minv.as<Real>();
    a.x = s->px.as<Real>();
    a.r = s->pr.as<Real>();
    a.sd0 = s->psd0.as<Real>();
    a.sd1 = s->psd1.as<Real>();
    a.q4 = s->q4.as<Real>();
    a.slots = s->slots.as<pk::ExSlot>();
    a.sync = s->sync.as<pk::GridSync>();
    a.max_iterations = p.max_iterations;
    a.tolerance = static_cast<Acc>(static_cast<Real>(p.tolerance));
    a.skip_on_flags = skip_on_flags;
    a.integrate = p.integrate;
    a.dt = static_cast<Real>(p.dt);
    a.dyn_to_node = s->dyn_to_node.as<int>();
    a.node_x = s->x.as<Real>();
    a.node_v = s->v.as<Real>();
    pk::DevStats* st = s->stats.as<pk::DevStats>();
    a.flags = &st->flags;
    a.missing = &st->batch_missing;
    a.stats = st;
    a.body_stats = s->body_stats.as<pk::BatchBodyStats>();
    PK_CHECK(pk::launch_pcg_batch_kernel<Real, Acc>(a, grid, s->stream));
    s->launches += 1;
    s->last_blocks = grid;
    return PK_OK;
}

// The PCG kernel the next unbatched solve uses (0 ring, 1 staged, 2 plain, 3 slab).
int solve_kernel(const pk_system* s)
{
    if (s->kernel_choice == 3 && s->slab_parts <= 0) return s->ring_tiles > 0 ? 0 : (s->ntiles > 0 ? 1 : 2);
    if (s->kernel_choice >= 0) return s->kernel_choice;
    return s->slab_parts > 0 ? 3 : (s->ring_tiles > 0 ? 0 : (s->ntiles > 0 ? 1 : 2));
}

template <class Real, class Acc>
int run_pcg(pk_system* s, const pk_step_params& p, int skip_on_flags)
{
    if (batched_solve(s)) {
        // Per-body solves: the part-resident kernel with one group of parts per body where
        // its layout applies, else the per-body batch kernel.
        if constexpr (std::is_same<Real, float>::value) {
            if (s->batch_slab) {
                int rc = ensure_slab<Acc>(s);
                if (rc) return rc;
                if (s->slab_parts > 0 && s->slab_for_bodies) return run_pcg_slab<Real, Acc>(s, p, skip_on_flags);
            }
        }
        s->last_kernel = 4;
        return run_pcg_batch<Real, Acc>(s, p, skip_on_flags);
    }
    if constexpr (std::is_same<Real, float>::value) {
        int rc = ensure_slab<Acc>(s);
        if (rc) return rc;
    }
    const int kernel = solve_kernel(s);
    s->last_kernel = kernel;
    if (kernel == 3) return run_pcg_slab<Real, Acc>(s, p, skip_on_flags);
    if (kernel == 0 && s->ring_tiles > 0) {
        int rc = ensure_solver_buffers(s, 1);
        if (rc) return rc;
        return run_pcg_ring<Real, Acc>(s, p, skip_on_flags);
    }
    // Staged (TMA tiles) or plain (unstaged) kernel.
    const int saved_tiles = s->ntiles;
    if (kernel == 2) s->ntiles = 0;
    const int grid = pcg_grid_for<Real, Acc>(s);
    s->ntiles = saved_tiles;
    if (grid <= 0) return fail(PK_ERR_CUDA, "cooperative PCG kernel cannot be resident");
    int rc = ensure_solver_buffers(s, max_grid_for<Real, Acc>(s));
    if (rc) return rc;
    PK_CHECK(cudaMemsetAsync(s->sync.p, 0, sizeof(pk::GridSync), s->stream));
    pk::PcgArgs<Real, Acc> a = pcg_args<Real, Acc>(s, p, skip_on_flags);
    if (kernel == 2) a.ntiles = 0;
    PK_CHECK(pk::launch_pcg_kernel<Real, Acc>(a, grid, pk::kPcgThreads, s->stream));
    s->launches += 1;
    s->last_kernel = a.ntiles > 0 ? 1 : 2;
    s->last_blocks = grid;
    return PK_OK;
}

// The solve with the FP64 outer true-residual refinement (pk_refine.cu): the first solve
// as usual but without integration; then, while the true residual r = b - A x (FP64 over
// the stored blocks, x accumulated in FP64) misses the reference's target r^T M^-1 r <=
// tol^2 b^T M^-1 b and iterations remain of the step's budget, a correction solve A e = r
// to the matching relative tolerance, x += e.  Finally the all-or-nothing update from the
// FP64 delta-v.  Statistics: total iterations, convergence and norm of the true residual.
// Synchronous (the host reads each residual), so such steps are never graph-captured.
template <class Real, class Acc>
int run_pcg_refined(pk_system* s, const pk_step_params& p, int skip_on_flags)
{
    const int n = s->dyn_count;
    const size_t n3 = 3 * static_cast<size_t>(n);
    pk_step_params q = p;
    q.integrate = 0;
    int rc = run_pcg<Real, Acc>(s, q, skip_on_flags);
    if (rc) return rc;
    pk::DevStats st{};
    PK_CHECK(cudaMemcpyAsync(&st, s->stats.p, sizeof(st), cudaMemcpyDeviceToHost, s->stream));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    if (!(st.flags & pk::kFlagSolved)) return PK_OK;  // nothing to refine or integrate
    const int blocks = pk::refine_residual_blocks<Real>(n);
    PK_CHECK(s->ref_x64.ensure(sizeof(double) * n3));
    PK_CHECK(s->ref_rhs.ensure(sizeof(Real) * n3));
    PK_CHECK(s->ref_part.ensure(2 * sizeof(double) * static_cast<size_t>(blocks)));
    PK_CHECK(s->ref_bad.ensure(sizeof(int)));
    PK_CHECK(cudaMemcpyAsync(s->ref_rhs.p, s->rhs.p, sizeof(Real) * n3, cudaMemcpyDeviceToDevice, s->stream));
    PK_CHECK(pk::launch_refine_accumulate<Real>(s->ref_x64.as<double>(), s->px.as<Real>(), static_cast<int>(n3), 1,
                                                s->stream));
    pk::RefineArgs<Real> a{};
    a.a.n = n;
    a.a.row_start = s->row_start.as<int>();
    a.a.col = s->col.as<int>();
    a.a.values = s->values.as<Real>();
    a.a.lt_start = s->lt_start.as<int>();
    a.a.lt_row = s->lt_row.as<int>();
    a.a.lt_block = s->lt_block.as<int>();
    a.b = s->ref_rhs.as<Real>();
    a.minv = s->minv.as<Real>();
    a.partials = s->ref_part.as<double>();
    a.bad = s->ref_bad.as<int>();
    // The FP64 system's residual from the tet data when the world holds only soft bodies
    // (point connections and host-emitted blocks exist only as stored blocks).
    const bool elem = s->conn_count == 0 && !s->ext_on && s->tet_count > 0 && s->dyn_count > 0 &&
                      s->precision != PK_PREC_FP64 && s->rest64_ok;
    pk::ElemResidualArgs<Real> ea{};
    const int eblocks = pk::elem_residual_blocks<Real>(n);
    if (elem) {
        PK_CHECK(s->elem_u.ensure(9 * sizeof(double) * static_cast<size_t>(s->tet_count)));
        PK_CHECK(s->elem_vx.ensure(3 * sizeof(double) * static_cast<size_t>(std::max(1, s->node_count))));
        ea.n = n;
        ea.node_count = s->node_count;
        ea.tet_count = s->tet_count;
        ea.tet_nodes = s->tet_nodes.as<int4>();
        ea.enabled = s->tet_enabled.as<unsigned char>();
        ea.dm_inv = s->dm_inv64.as<double>();
        ea.params = s->params64.as<double>();
        ea.mass = s->mass64.as<double>();
        ea.x = s->x.as<Real>();
        ea.v = s->v.as<Real>();
        ea.node_to_dyn = s->node_to_dyn.as<int>();
        ea.dyn_to_node = s->dyn_to_node.as<int>();
        ea.inc_start = s->inc_start.as<int>();
        ea.inc_list = s->inc_list.as<int>();
        ea.minv = s->minv.as<Real>();
        ea.vx = s->elem_vx.as<double>();
        ea.u = s->elem_u.as<double>();
        ea.dt = static_cast<double>(static_cast<float>(p.dt));
        for (int i = 0; i < 3; ++i) ea.gravity[i] = static_cast<double>(static_cast<float>(p.gravity[i]));
        ea.linear = p.linear;
        ea.partials = s->ref_part.as<double>();
        ea.bad = s->ref_bad.as<int>();
    }
    std::vector<double> part(2 * static_cast<size_t>(elem ? eblocks : blocks));
    // r = b - A x (x == NULL: r = b); returns false on a non-finite residual.
    auto residual = [&](const double* x, Real* rhs_out, double& rho, double& rr) -> int {
        a.x64 = x;
        a.rhs_out = rhs_out;
        PK_CHECK(cudaMemsetAsync(s->ref_bad.p, 0, sizeof(int), s->stream));
        if (elem) {
            ea.x64 = x;
            ea.rhs_out = rhs_out;
            PK_CHECK(pk::launch_elem_residual<Real>(ea, s->stream));
        } else {
            PK_CHECK(pk::launch_refine_residual<Real>(a, s->stream));
        }
        int bad = 0;
        PK_CHECK(cudaMemcpyAsync(part.data(), s->ref_part.p, sizeof(double) * part.size(), cudaMemcpyDeviceToHost,
                                 s->stream));
        PK_CHECK(cudaMemcpyAsync(&bad, s->ref_bad.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        PK_CHECK(cudaStreamSynchronize(s->stream));
        rho = 0.0;
        rr = 0.0;
        for (size_t i = 0; 2 * i < part.size(); ++i) {
            rho += part[2 * i];
            rr += part[2 * i + 1];
        }
        return bad || !std::isfinite(rho) || !std::isfinite(rr) ? 1 : 0;
    };
    double rho0 = 0.0, rr0 = 0.0, rho = 0.0, rr = 0.0;
    residual(nullptr, nullptr, rho0, rr0);
    const double tol = static_cast<double>(static_cast<Real>(p.tolerance));
    const double target = tol * tol * rho0;
    int total = st.iterations;
    bool converged = false;
    for (int pass = 0;; ++pass) {
        if (residual(s->ref_x64.as<double>(), s->rhs.as<Real>(), rho, rr)) break;
        if (rho <= target) {
            converged = true;
            break;
        }
        const int remaining = p.max_iterations - total;
        if (remaining <= 0 || pass >= s->refine_passes || !(rho > 0.0)) break;
        q.max_iterations = remaining;
        q.tolerance = std::sqrt(target / rho);
        PK_CHECK(cudaMemsetAsync(s->stats.p, 0, sizeof(pk::DevStats), s->stream));
        rc = run_pcg<Real, Acc>(s, q, 0);
        if (rc) break;
        pk::DevStats cs{};
        PK_CHECK(cudaMemcpyAsync(&cs, s->stats.p, sizeof(cs), cudaMemcpyDeviceToHost, s->stream));
        PK_CHECK(cudaStreamSynchronize(s->stream));
        total += cs.iterations;
        if (!(cs.flags & pk::kFlagSolved)) break;  // a failed correction is discarded
        PK_CHECK(pk::launch_refine_accumulate<Real>(s->ref_x64.as<double>(), s->px.as<Real>(), static_cast<int>(n3),
                                                    0, s->stream));
        if (total >= p.max_iterations || pass + 1 > s->refine_passes) {
            residual(s->ref_x64.as<double>(), nullptr, rho, rr);
            converged = rho <= target;
            break;
        }
    }
    PK_CHECK(cudaMemcpyAsync(s->rhs.p, s->ref_rhs.p, sizeof(Real) * n3, cudaMemcpyDeviceToDevice, s->stream));
    if (rc) return rc;
    // The update from the FP64 delta-v (all or nothing), delta-v kept in px.
    a.x64 = s->ref_x64.as<double>();
    a.dx = s->px.as<Real>();
    a.integrate = p.integrate;
    a.dt = static_cast<Real>(p.dt);
    a.dyn_to_node = s->dyn_to_node.as<int>();
    a.node_x = s->x.as<Real>();
    a.node_v = s->v.as<Real>();
    PK_CHECK(cudaMemsetAsync(s->ref_bad.p, 0, sizeof(int), s->stream));
    PK_CHECK(pk::launch_refine_update<Real>(a, s->stream));
    int bad = 0;
    PK_CHECK(cudaMemcpyAsync(&bad, s->ref_bad.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    unsigned fl = st.flags & ~(pk::kFlagConverged | pk::kFlagIntegrated | pk::kFlagSolved);
    if (bad & 1) {
        fl |= pk::kFlagNonFiniteDv;
    } else {
        fl |= pk::kFlagSolved;
        if (p.integrate) fl |= (bad & 2) ? pk::kFlagIntegrateAbort : pk::kFlagIntegrated;
    }
    if (converged) fl |= pk::kFlagConverged;
    if (elem) fl |= pk::kFlagRefinedFp64;
    pk::DevStats out = st;
    out.iterations = total;
    out.converged = converged ? 1 : 0;
    out.residual_norm = std::sqrt(std::max(rr, 0.0));
    out.flags = fl;
    PK_CHECK(cudaMemcpyAsync(s->stats.p, &out, sizeof(out), cudaMemcpyHostToDevice, s->stream));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    return PK_OK;
}

// PK_ROW_KERNEL=thread assembles the rows one thread each (the four-lane kernel's blocks
// and right-hand side are the same bits; kept for comparisons).
bool row_lanes_enabled()
{
    const char* e = std::getenv("PK_ROW_KERNEL");
    return !(e && std::strcmp(e, "thread") == 0);
}

// PK_ASSEMBLY_FOLD=0 keeps every tet on the long assembly path (all 16 blocks per tet
// and K v in the row kernel), for comparisons; the default folds K v into the tet kernel.
bool assembly_fold_enabled()
{
    const char* e = std::getenv("PK_ASSEMBLY_FOLD");
    return !(e && e[0] == '0');
}

// The slot table of the folded assembly (rows of at most kSlotMaxRow upper blocks), built
// on the device after the pattern, the incidences, the tets or the node rows changed.
int ensure_inc_slots(pk_system* s)
{
    if (s->slots_ok || s->dyn_count <= 0 || s->inc_count <= 0 || !s->have_tets || s->max_row > pk::kSlotMaxRow ||
        !assembly_fold_enabled())
        return PK_OK;
    PK_CHECK(s->inc_slot.ensure(sizeof(unsigned) * static_cast<size_t>(s->inc_count)));
    PK_CHECK(pk::launch_inc_slot_kernel(s->dyn_count, s->row_start.as<int>(), s->col.as<int>(),
                                        s->inc_start.as<int>(), s->inc_list.as<int>(), s->tet_nodes.as<int4>(),
                                        s->node_to_dyn.as<int>(), s->inc_slot.as<unsigned>(), s->stream));
    s->launches += 1;
    s->slots_ok = true;
    return PK_OK;
}

template <class Real>
int run_step(pk_system* s, const pk_step_params& p)
{
    if (const int rc = ensure_inc_slots(s)) return rc;
    PK_CHECK(cudaMemsetAsync(s->stats.p, 0, sizeof(pk::DevStats), s->stream));
    // A per-body part-resident layout from an earlier step: its round table for this solve
    // is built on the side stream while the step assembles.
    s->sched_pending = false;
    if (std::is_same<Real, float>::value && !p.explicit_mode && batched_solve(s) && s->batch_slab &&
        s->slab_parts > 0 && s->slab_for_bodies && s->sched_stream && s->dyn_count > 0) {
        PK_CHECK(cudaEventRecord(s->sched_fork, s->stream));
        PK_CHECK(cudaStreamWaitEvent(s->sched_stream, s->sched_fork, 0));
        if (const int rc = launch_slab_schedule(s, p.max_iterations, s->sched_stream)) return rc;
        PK_CHECK(cudaEventRecord(s->sched_join, s->sched_stream));
        s->sched_pending = true;
    }
    int evi[3] = {-1, -1, -1};
    if (s->timing) {
        for (int i = 0; i < 3; ++i) {
            cudaEvent_t e;
            PK_CHECK(cudaEventCreate(&e));
            s->ev_pool.push_back(e);
            evi[i] = static_cast<int>(s->ev_pool.size()) - 1;
        }
        PK_CHECK(cudaEventRecord(s->ev_pool[evi[0]], s->stream));
    }
    pk::AssemblyArgs<Real> a = assembly_args<Real>(s, p);
    const bool fp64_polar = s->precision == PK_PREC_MIXED;
    if (s->tet_count > 0) {
        PK_CHECK(pk::launch_tet_kernel<Real>(a, fp64_polar, s->stream));
        s->launches += 1;
    }
    if (s->dyn_count > 0) {
        if (s->conn_count > 0) {
            PK_CHECK(pk::launch_conn_kernel<Real>(a, s->stream));
            s->launches += 1;
        }
        PK_CHECK(pk::launch_row_kernel<Real>(a, s->max_row, s->stream));
        s->launches += 1;
        s->slab_filled = false;
        // The part-resident kernel reads the blocks from its own stream: fill it here so
        // the solve time below is the PCG kernel's alone.
        if constexpr (std::is_same<Real, float>::value) {
            if (!p.explicit_mode && (!batched_solve(s) || s->batch_slab)) {
                int rc = s->precision == PK_PREC_MIXED ? ensure_slab<double>(s) : ensure_slab<float>(s);
                if (rc) return rc;
                const bool uses = batched_solve(s) ? (s->slab_parts > 0 && s->slab_for_bodies) : solve_kernel(s) == 3;
                if (uses) {
                    rc = slab_fill(s);
                    if (rc) return rc;
                }
            }
        }
    }
    if (s->timing) PK_CHECK(cudaEventRecord(s->ev_pool[evi[1]], s->stream));
    if (!p.explicit_mode && s->dyn_count > 0) {
        int rc;
        const bool refine = s->refine_passes > 0 && !batched_solve(s);
        if constexpr (std::is_same<Real, double>::value)
            rc = run_pcg<double, double>(s, p, 1);
        else if (s->precision == PK_PREC_FP32)
            rc = refine ? run_pcg_refined<float, float>(s, p, 1) : run_pcg<float, float>(s, p, 1);
        else
            rc = refine ? run_pcg_refined<float, double>(s, p, 1) : run_pcg<float, double>(s, p, 1);
        if (rc) return rc;
    }
    if (s->sched_pending) {  // the solve did not take the table: join the side stream anyway
        PK_CHECK(cudaStreamWaitEvent(s->stream, s->sched_join, 0));
        s->sched_pending = false;
    }
    if (s->timing) {
        PK_CHECK(cudaEventRecord(s->ev_pool[evi[2]], s->stream));
        s->ev_pending.push_back({evi[0], evi[1], evi[2]});
    }
    PK_CHECK(cudaMemcpyAsync(s->host_stats, s->stats.p, sizeof(pk::DevStats), cudaMemcpyDeviceToHost, s->stream));
    s->stats_pending = true;
    if (!p.explicit_mode) s->assembled = true;
    return PK_OK;
}

void drop_graph(pk_system* s)
{
    if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
    s->graph_exec = nullptr;
}

bool same_params(const pk_step_params& a, const pk_step_params& b)
{
    return a.dt == b.dt && a.gravity[0] == b.gravity[0] && a.gravity[1] == b.gravity[1] &&
           a.gravity[2] == b.gravity[2] && a.max_iterations == b.max_iterations && a.tolerance == b.tolerance &&
           a.use_jacobi == b.use_jacobi && a.linear == b.linear && a.explicit_mode == b.explicit_mode &&
           a.integrate == b.integrate;
}

// One step as a CUDA graph: captured (relaxed mode) on the first step with these
// parameters after a plain step has made every allocation and upload, replayed after.
template <class Real>
int run_step_graph(pk_system* s, const pk_step_params& p)
{
    // A refined step reads residuals on the host between its solves: not capturable.
    if (s->refine_passes > 0 && s->precision != PK_PREC_FP64 && !p.explicit_mode) {
        drop_graph(s);
        return run_step<Real>(s, p);
    }
    if (!s->graph_exec || !same_params(p, s->graph_params)) {
        drop_graph(s);
        // Everything built lazily (allocations, uploads) must exist before the capture.
        int prc = ensure_batch_parts_any(s);
        if (!prc) prc = ensure_slab_any(s);
        if (!prc) prc = ensure_inc_slots(s);
        if (prc) return prc;
        const bool timing = s->timing;
        const long long launches = s->launches;
        s->timing = false;
        PK_CHECK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeRelaxed));
        const int rc = run_step<Real>(s, p);
        cudaGraph_t graph = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(s->stream, &graph);
        s->timing = timing;
        s->graph_kernels = static_cast<int>(s->launches - launches);
        s->launches = launches;
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (ec != cudaSuccess) return cuda_fail(ec, "cudaStreamEndCapture");
        const cudaError_t ei = cudaGraphInstantiate(&s->graph_exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) {
            s->graph_exec = nullptr;
            return cuda_fail(ei, "cudaGraphInstantiate");
        }
        s->graph_params = p;
    }
    int evi[2] = {-1, -1};
    if (s->timing) {
        for (int i = 0; i < 2; ++i) {
            cudaEvent_t e;
            PK_CHECK(cudaEventCreate(&e));
            s->ev_pool.push_back(e);
            evi[i] = static_cast<int>(s->ev_pool.size()) - 1;
        }
        PK_CHECK(cudaEventRecord(s->ev_pool[evi[0]], s->stream));
    }
    PK_CHECK(cudaGraphLaunch(s->graph_exec, s->stream));
    if (s->timing) {
        PK_CHECK(cudaEventRecord(s->ev_pool[evi[1]], s->stream));
        s->ev_pending.push_back({evi[0], evi[0], evi[1]});  // the whole step counts as solve time
    }
    s->launches += s->graph_kernels;
    s->stats_pending = true;
    return PK_OK;
}

int use_device(int device)
{
    if (device_count_safe() <= 0) return fail(PK_ERR_NO_DEVICE, "no CUDA device");
    PK_CHECK(cudaSetDevice(device));
    return PK_OK;
}

template <class Real>
int upload_real(DevBuf& buf, const double* src, size_t n, cudaStream_t stream)
{
    PK_CHECK(buf.ensure(std::max<size_t>(n, 1) * sizeof(Real)));
    if (n == 0 || !src) return PK_OK;
    std::vector<Real> tmp = narrow<Real>(src, n);
    PK_CHECK(cudaMemcpyAsync(buf.p, tmp.data(), n * sizeof(Real), cudaMemcpyHostToDevice, stream));
    PK_CHECK(cudaStreamSynchronize(stream));
    return PK_OK;
}

template <class T>
int upload_raw(DevBuf& buf, const T* src, size_t n, cudaStream_t stream)
{
    PK_CHECK(buf.ensure(std::max<size_t>(n, 1) * sizeof(T)));
    if (n == 0 || !src) return PK_OK;
    PK_CHECK(cudaMemcpyAsync(buf.p, src, n * sizeof(T), cudaMemcpyHostToDevice, stream));
    PK_CHECK(cudaStreamSynchronize(stream));
    return PK_OK;
}

template <class Real>
int download_real(const DevBuf& buf, double* dst, size_t n, cudaStream_t stream)
{
    if (!dst || n == 0) return PK_OK;
    std::vector<Real> tmp(n);
    PK_CHECK(cudaMemcpyAsync(tmp.data(), buf.p, n * sizeof(Real), cudaMemcpyDeviceToHost, stream));
    PK_CHECK(cudaStreamSynchronize(stream));
    for (size_t i = 0; i < n; ++i) dst[i] = static_cast<double>(tmp[i]);
    return PK_OK;
}

int upload_real_any(pk_system* s, DevBuf& buf, const double* src, size_t n)
{
    return s->precision == PK_PREC_FP64 ? upload_real<double>(buf, src, n, s->stream)
                                        : upload_real<float>(buf, src, n, s->stream);
}
int download_real_any(pk_system* s, const DevBuf& buf, double* dst, size_t n)
{
    return s->precision == PK_PREC_FP64 ? download_real<double>(buf, dst, n, s->stream)
                                        : download_real<float>(buf, dst, n, s->stream);
}

}  // namespace

extern "C" {

PKCUDA_API const char* pk_last_error(void) { return g_last_error.c_str(); }

PKCUDA_API int pk_device_count(void) { return device_count_safe(); }

PKCUDA_API int pk_system_create(int device, int precision, pk_system** out)
{
    if (!out) return fail(PK_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (precision < PK_PREC_FP32 || precision > PK_PREC_FP64) return fail(PK_ERR_ARG, "bad precision");
    int rc = use_device(device);
    if (rc) return rc;
    pk_system* s = new pk_system();
    s->device = device;
    s->precision = precision;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete s;
        return cuda_fail(e, "cudaStreamCreate");
    }
    e = cudaMallocHost(&s->host_stats, sizeof(pk::DevStats));
    if (e == cudaSuccess) e = s->stats.ensure(sizeof(pk::DevStats));
    if (e != cudaSuccess) {
        cudaStreamDestroy(s->stream);
        delete s;
        return cuda_fail(e, "stats allocation");
    }
    std::memset(s->host_stats, 0, sizeof(pk::DevStats));
    *out = s;
    return PK_OK;
}

PKCUDA_API int pk_system_destroy(pk_system* s)
{
    if (!s) return PK_OK;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    drop_graph(s);
    for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
    if (s->host_stats) cudaFreeHost(s->host_stats);
    if (s->sched_stream) {
        cudaStreamSynchronize(s->sched_stream);
        cudaStreamDestroy(s->sched_stream);
    }
    if (s->sched_fork) cudaEventDestroy(s->sched_fork);
    if (s->sched_join) cudaEventDestroy(s->sched_join);
    cudaStreamDestroy(s->stream);
    delete s;
    return PK_OK;
}

PKCUDA_API void* pk_system_stream(pk_system* s) { return s ? static_cast<void*>(s->stream) : nullptr; }

PKCUDA_API int pk_system_set_nodes(pk_system* s, int node_count, const int* node_to_dyn, const double* mass)
{
    if (s) drop_graph(s);
    if (!s || node_count < 0 || (node_count > 0 && (!node_to_dyn || !mass))) return fail(PK_ERR_ARG, "set_nodes");
    PK_CHECK(cudaSetDevice(s->device));
    s->node_count = node_count;
    s->have_snapshot = false;
    s->h_node_to_dyn.assign(node_to_dyn, node_to_dyn + node_count);
    s->slots_ok = false;
    s->h_mass.assign(mass, mass + node_count);
    int rc = upload_raw<int>(s->node_to_dyn, node_to_dyn, node_count, s->stream);
    if (!rc) rc = upload_real_any(s, s->mass, mass, node_count);
    s->rest64_ok = false;
    if (rc) return rc;
    const size_t bytes = 3 * s->rsize() * static_cast<size_t>(std::max(1, node_count));
    PK_CHECK(s->x.ensure(bytes));
    PK_CHECK(s->v.ensure(bytes));
    PK_CHECK(cudaMemsetAsync(s->x.p, 0, bytes, s->stream));
    PK_CHECK(cudaMemsetAsync(s->v.p, 0, bytes, s->stream));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    s->have_nodes = true;
    return PK_OK;
}

PKCUDA_API int pk_system_set_state_f64(pk_system* s, const double* x, const double* v)
{
    if (!s || !s->have_nodes) return fail(PK_ERR_STATE, "set_state before set_nodes");
    PK_CHECK(cudaSetDevice(s->device));
    const size_t n = 3 * static_cast<size_t>(s->node_count);
    int rc = PK_OK;
    if (x) rc = upload_real_any(s, s->x, x, n);
    if (!rc && v) rc = upload_real_any(s, s->v, v, n);
    return rc;
}

PKCUDA_API int pk_system_set_state_f32(pk_system* s, const float* x, const float* v)
{
    if (!s || !s->have_nodes) return fail(PK_ERR_STATE, "set_state before set_nodes");
    PK_CHECK(cudaSetDevice(s->device));
    const size_t n = 3 * static_cast<size_t>(s->node_count);
    if (s->precision == PK_PREC_FP64) {
        std::vector<double> tx, tv;
        if (x) tx.assign(x, x + n);
        if (v) tv.assign(v, v + n);
        return pk_system_set_state_f64(s, x ? tx.data() : nullptr, v ? tv.data() : nullptr);
    }
    // float storage: copy straight from the caller's buffer (pinned buffers stay asynchronous)
    if (x) PK_CHECK(cudaMemcpyAsync(s->x.p, x, n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
    if (v) PK_CHECK(cudaMemcpyAsync(s->v.p, v, n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
    return PK_OK;
}

PKCUDA_API int pk_system_get_state_f64(pk_system* s, double* x, double* v)
{
    if (!s || !s->have_nodes) return fail(PK_ERR_STATE, "get_state before set_nodes");
    PK_CHECK(cudaSetDevice(s->device));
    const size_t n = 3 * static_cast<size_t>(s->node_count);
    int rc = download_real_any(s, s->x, x, n);
    if (!rc) rc = download_real_any(s, s->v, v, n);
    return rc;
}

PKCUDA_API int pk_system_get_state_f32(pk_system* s, float* x, float* v)
{
    if (!s || !s->have_nodes) return fail(PK_ERR_STATE, "get_state before set_nodes");
    PK_CHECK(cudaSetDevice(s->device));
    const size_t n = 3 * static_cast<size_t>(s->node_count);
    if (s->precision == PK_PREC_FP64) {
        std::vector<double> tx(x ? n : 0), tv(v ? n : 0);
        int rc = pk_system_get_state_f64(s, x ? tx.data() : nullptr, v ? tv.data() : nullptr);
        if (rc) return rc;
        for (size_t i = 0; x && i < n; ++i) x[i] = static_cast<float>(tx[i]);
        for (size_t i = 0; v && i < n; ++i) v[i] = static_cast<float>(tv[i]);
        return PK_OK;
    }
    if (x) PK_CHECK(cudaMemcpyAsync(x, s->x.p, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    if (v) PK_CHECK(cudaMemcpyAsync(v, s->v.p, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    return PK_OK;
}

PKCUDA_API int pk_system_snapshot_positions(pk_system* s)
{
    if (!s || !s->have_nodes) return fail(PK_ERR_STATE, "snapshot before set_nodes");
    PK_CHECK(cudaSetDevice(s->device));
    const size_t bytes = 3 * static_cast<size_t>(s->node_count) * s->rsize();
    PK_CHECK(s->snap_x.ensure(bytes));
    if (bytes) PK_CHECK(cudaMemcpyAsync(s->snap_x.p, s->x.p, bytes, cudaMemcpyDeviceToDevice, s->stream));
    s->have_snapshot = true;
    return PK_OK;
}

PKCUDA_API int pk_system_sphere_contacts(pk_system* s, const double* center, double radius, int max_contacts,
                                         int* tets, double* points)
{
    if (!s || !center || max_contacts < 0 || (max_contacts > 0 && (!tets || !points)))
        return fail(PK_ERR_ARG, "sphere_contacts");
    if (!s->have_nodes || !s->have_tets) return fail(PK_ERR_STATE, "sphere_contacts before nodes and tets");
    PK_CHECK(cudaSetDevice(s->device));
    const int T = s->tet_count;
    if (T == 0) return 0;
    PK_CHECK(s->contact_count.ensure(sizeof(int)));
    PK_CHECK(s->contact_tet.ensure(sizeof(int) * static_cast<size_t>(T)));
    PK_CHECK(s->contact_point.ensure(3 * s->rsize() * static_cast<size_t>(T)));
    PK_CHECK(cudaMemsetAsync(s->contact_count.p, 0, sizeof(int), s->stream));
    if (s->precision == PK_PREC_FP64) {
        PK_CHECK(pk::launch_sphere_contacts<double>(s->tet_nodes.as<int>(), s->tet_enabled.as<unsigned char>(),
                                                    s->x.as<double>(), T, center, radius, T,
                                                    s->contact_count.as<int>(), s->contact_tet.as<int>(),
                                                    s->contact_point.as<double>(), s->stream));
    } else {
        const float c[3] = {static_cast<float>(center[0]), static_cast<float>(center[1]),
                            static_cast<float>(center[2])};
        PK_CHECK(pk::launch_sphere_contacts<float>(s->tet_nodes.as<int>(), s->tet_enabled.as<unsigned char>(),
                                                   s->x.as<float>(), T, c, static_cast<float>(radius), T,
                                                   s->contact_count.as<int>(), s->contact_tet.as<int>(),
                                                   s->contact_point.as<float>(), s->stream));
    }
    int n = 0;
    PK_CHECK(cudaMemcpyAsync(&n, s->contact_count.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    n = std::min(n, T);
    if (n > max_contacts) return n;  // the caller's arrays are too small: only the count
    std::vector<int> t(static_cast<size_t>(n));
    std::vector<double> p(3 * static_cast<size_t>(n));
    if (n > 0) {
        PK_CHECK(cudaMemcpyAsync(t.data(), s->contact_tet.p, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
        if (s->precision == PK_PREC_FP64) {
            PK_CHECK(cudaMemcpyAsync(p.data(), s->contact_point.p, 3 * sizeof(double) * n, cudaMemcpyDeviceToHost,
                                     s->stream));
            PK_CHECK(cudaStreamSynchronize(s->stream));
        } else {
            std::vector<float> pf(3 * static_cast<size_t>(n));
            PK_CHECK(cudaMemcpyAsync(pf.data(), s->contact_point.p, 3 * sizeof(float) * n, cudaMemcpyDeviceToHost,
                                     s->stream));
            PK_CHECK(cudaStreamSynchronize(s->stream));
            for (size_t i = 0; i < pf.size(); ++i) p[i] = pf[i];
        }
    }
    // ascending tet order (the reference visits tets in order)
    std::vector<int> order(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return t[a] < t[b]; });
    for (int i = 0; i < n; ++i) {
        tets[i] = t[order[i]];
        for (int a = 0; a < 3; ++a) points[3 * (size_t)i + a] = p[3 * (size_t)order[i] + a];
    }
    return n;
}

// ------------------------------------------------------------------ post-step geometry
struct pk_visual {
    int device = 0;
    int kind = 0;
    int count = 0;
    int max_node = -1;  // the largest node id the visual reads; checked against the system at each update
    DevBuf nodes, weights, live, verts, normals;
};

PKCUDA_API int pk_visual_create(pk_system* s, int kind, int count, const int* nodes, const float* weights,
                                const float* initial, const unsigned char* live, pk_visual** out)
{
    if (!out) return fail(PK_ERR_ARG, "visual_create: out");
    *out = nullptr;
    if (!s || (kind != 0 && kind != 1) || count < 0 || (count > 0 && !nodes) ||
        (kind == 1 && count > 0 && (!weights || !initial || !live)))
        return fail(PK_ERR_ARG, "visual_create");
    if (!s->have_nodes) return fail(PK_ERR_STATE, "visual_create before set_nodes");
    const int per = kind == 0 ? 3 : 4;
    int max_node = -1;
    for (long long i = 0; i < static_cast<long long>(per) * count; ++i) {
        if (nodes[i] < 0 || nodes[i] >= s->node_count) return fail(PK_ERR_ARG, "visual node out of range");
        max_node = std::max(max_node, nodes[i]);
    }
    PK_CHECK(cudaSetDevice(s->device));
    auto v = std::make_unique<pk_visual>();
    v->device = s->device;
    v->kind = kind;
    v->count = count;
    v->max_node = max_node;
    const size_t n = static_cast<size_t>(count);
    int rc = upload_raw<int>(v->nodes, nodes, per * n, s->stream);
    if (!rc && kind == 1) rc = upload_raw<float>(v->weights, weights, 4 * n, s->stream);
    if (!rc && kind == 1) rc = upload_raw<unsigned char>(v->live, live, n, s->stream);
    if (!rc) PK_CHECK(v->verts.ensure(sizeof(float) * (kind == 0 ? 9 : 3) * std::max<size_t>(n, 1)));
    if (!rc && kind == 0) PK_CHECK(v->normals.ensure(sizeof(float) * 9 * std::max<size_t>(n, 1)));
    if (!rc && kind == 1) rc = upload_raw<float>(v->verts, initial, 3 * n, s->stream);
    if (rc) return rc;
    *out = v.release();
    return PK_OK;
}

PKCUDA_API int pk_visual_set_live(pk_visual* v, pk_system* s, const unsigned char* live)
{
    if (!v || !s || v->kind != 1 || (v->count > 0 && !live)) return fail(PK_ERR_ARG, "visual_set_live");
    if (v->device != s->device) return fail(PK_ERR_STATE, "visual on another device");
    PK_CHECK(cudaSetDevice(v->device));
    return upload_raw<unsigned char>(v->live, live, static_cast<size_t>(v->count), s->stream);
}

PKCUDA_API int pk_visual_update(pk_visual* v, pk_system* s, int from_snapshot)
{
    if (!v || !s) return fail(PK_ERR_ARG, "visual_update");
    if (v->device != s->device) return fail(PK_ERR_STATE, "visual on another device");
    if (from_snapshot && !s->have_snapshot) return fail(PK_ERR_STATE, "visual_update: no snapshot");
    if (v->max_node >= s->node_count) return fail(PK_ERR_STATE, "visual_update: nodes beyond the system");
    if (v->count == 0) return PK_OK;
    PK_CHECK(cudaSetDevice(v->device));
    const DevBuf& src = from_snapshot ? s->snap_x : s->x;
    if (s->precision == PK_PREC_FP64)
        PK_CHECK(pk::launch_visual_kernel<double>(v->kind, v->nodes.as<int>(), v->weights.as<float>(),
                                                  v->live.as<unsigned char>(), v->count, src.as<double>(),
                                                  v->verts.as<float>(), v->normals.as<float>(), s->stream));
    else
        PK_CHECK(pk::launch_visual_kernel<float>(v->kind, v->nodes.as<int>(), v->weights.as<float>(),
                                                 v->live.as<unsigned char>(), v->count, src.as<float>(),
                                                 v->verts.as<float>(), v->normals.as<float>(), s->stream));
    s->launches += 1;
    return PK_OK;
}

PKCUDA_API int pk_visual_read(pk_visual* v, pk_system* s, float* vertices, float* normals)
{
    if (!v || !s) return fail(PK_ERR_ARG, "visual_read");
    if (v->device != s->device) return fail(PK_ERR_STATE, "visual on another device");
    if (v->count == 0) return PK_OK;
    PK_CHECK(cudaSetDevice(v->device));
    const size_t n = static_cast<size_t>(v->count) * (v->kind == 0 ? 9 : 3);
    if (vertices) PK_CHECK(cudaMemcpyAsync(vertices, v->verts.p, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    if (normals && v->kind == 0)
        PK_CHECK(cudaMemcpyAsync(normals, v->normals.p, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    return PK_OK;
}

PKCUDA_API int pk_visual_destroy(pk_visual* v)
{
    if (!v) return PK_OK;
    cudaSetDevice(v->device);
    delete v;
    return PK_OK;
}

PKCUDA_API int pk_system_get_snapshot_f32(pk_system* s, int first_node, int count, float* x)
{
    if (!s || !s->have_snapshot) return fail(PK_ERR_STATE, "get_snapshot before a snapshot");
    if (first_node < 0 || count < 0 || first_node > s->node_count - count || (count > 0 && !x))
        return fail(PK_ERR_ARG, "get_snapshot: node range");
    if (count == 0) return PK_OK;
    PK_CHECK(cudaSetDevice(s->device));
    const size_t n = 3 * static_cast<size_t>(count), off = 3 * static_cast<size_t>(first_node);
    if (s->precision == PK_PREC_FP64) {
        std::vector<double> t(n);
        PK_CHECK(cudaMemcpyAsync(t.data(), s->snap_x.as<double>() + off, n * sizeof(double), cudaMemcpyDeviceToHost,
                                 s->stream));
        PK_CHECK(cudaStreamSynchronize(s->stream));
        for (size_t i = 0; i < n; ++i) x[i] = static_cast<float>(t[i]);
        return PK_OK;
    }
    PK_CHECK(cudaMemcpyAsync(x, s->snap_x.as<float>() + off, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    return PK_OK;
}

PKCUDA_API int pk_system_set_masses(pk_system* s, const double* mass)
{
    if (s) drop_graph(s);
    if (!s || !mass) return fail(PK_ERR_ARG, "set_masses");
    if (!s->have_nodes) return fail(PK_ERR_STATE, "masses before the nodes");
    PK_CHECK(cudaSetDevice(s->device));
    s->h_mass.assign(mass, mass + s->node_count);
    s->rest64_ok = false;
    return upload_real_any(s, s->mass, mass, s->node_count);
}

PKCUDA_API int pk_system_set_tets(pk_system* s, int tet_count, const int* tet_nodes, const unsigned char* enabled,
                                  const double* dm_inv, const double* volume, const double* lambda, const double* mu,
                                  const double* damping)
{
    if (s) drop_graph(s);
    if (!s || tet_count < 0) return fail(PK_ERR_ARG, "set_tets");
    if (tet_count > 0 && (!tet_nodes || !enabled || !dm_inv || !volume || !lambda || !mu || !damping))
        return fail(PK_ERR_ARG, "set_tets: NULL array");
    PK_CHECK(cudaSetDevice(s->device));
    for (long long i = 0; i < 4ll * tet_count; ++i)
        if (tet_nodes[i] < 0 || tet_nodes[i] >= s->node_count) return fail(PK_ERR_ARG, "tet node out of range");
    s->tet_count = tet_count;
    s->slots_ok = false;
    s->h_tet_nodes.assign(tet_nodes, tet_nodes + 4 * static_cast<size_t>(tet_count));
    s->h_enabled.assign(enabled, enabled + tet_count);
    s->h_damping.assign(damping, damping + tet_count);
    std::vector<double> params(4 * static_cast<size_t>(tet_count));
    for (int t = 0; t < tet_count; ++t) {
        params[4 * t + 0] = volume[t];
        params[4 * t + 1] = lambda[t];
        params[4 * t + 2] = mu[t];
        params[4 * t + 3] = damping[t];
    }
    int rc = upload_raw<int>(s->tet_nodes, tet_nodes, 4 * static_cast<size_t>(tet_count), s->stream);
    if (!rc) rc = upload_raw<unsigned char>(s->tet_enabled, enabled, tet_count, s->stream);
    if (!rc) rc = upload_real_any(s, s->dm_inv, dm_inv, 9 * static_cast<size_t>(tet_count));
    if (!rc) rc = upload_real_any(s, s->tet_params, params.data(), params.size());
    s->rest64_ok = false;
    if (rc) return rc;
    PK_CHECK(s->tet_rec.ensure(pk::kTetRec * s->rsize() * std::max<size_t>(1, tet_count)));
    if (s->precision == PK_PREC_FP64)
        PK_CHECK(pk::launch_tet_pack<double>(s->dm_inv.as<double>(), s->tet_params.as<double>(),
                                             s->tet_rec.as<double>(), tet_count, s->stream));
    else
        PK_CHECK(pk::launch_tet_pack<float>(s->dm_inv.as<float>(), s->tet_params.as<float>(),
                                            s->tet_rec.as<float>(), tet_count, s->stream));
    s->have_tets = true;
    return PK_OK;
}

PKCUDA_API int pk_system_set_rest64(pk_system* s, int tet_count, const double* dm_inv, const double* volume,
                                    const double* lambda, const double* mu, const double* damping, int node_count,
                                    const double* mass)
{
    if (!s || tet_count < 0 || node_count < 0) return fail(PK_ERR_ARG, "set_rest64");
    if (!s->have_tets || !s->have_nodes || tet_count != s->tet_count || node_count != s->node_count)
        return fail(PK_ERR_STATE, "set_rest64: not the system's tets and nodes");
    if ((tet_count > 0 && (!dm_inv || !volume || !lambda || !mu || !damping)) || (node_count > 0 && !mass))
        return fail(PK_ERR_ARG, "set_rest64: NULL array");
    PK_CHECK(cudaSetDevice(s->device));
    s->rest64_ok = false;
    std::vector<double> params(4 * static_cast<size_t>(tet_count));
    for (int t = 0; t < tet_count; ++t) {
        params[4 * t + 0] = volume[t];
        params[4 * t + 1] = lambda[t];
        params[4 * t + 2] = mu[t];
        params[4 * t + 3] = damping[t];
    }
    int rc = upload_raw<double>(s->dm_inv64, dm_inv, 9 * static_cast<size_t>(tet_count), s->stream);
    if (!rc) rc = upload_raw<double>(s->params64, params.data(), params.size(), s->stream);
    if (!rc) rc = upload_raw<double>(s->mass64, mass, static_cast<size_t>(node_count), s->stream);
    if (rc) return rc;
    PK_CHECK(cudaStreamSynchronize(s->stream));
    s->rest64_ok = true;
    return PK_OK;
}

PKCUDA_API int pk_system_set_extras(pk_system* s, int block_count, const double* blocks, const int* block_nodes,
                                    const int* rhs_start, const int* rhs_list, const int* mat_start,
                                    const int* mat_list, const double* row_force)
{
    if (!s || block_count < 0) return fail(PK_ERR_ARG, "set_extras");
    const void* old_bufs[7] = {s->ext_blocks.p, s->ext_nodes.p, s->ext_rhs_start.p, s->ext_rhs_list.p,
                               s->ext_mat_start.p, s->ext_mat_list.p, s->ext_force.p};
    const bool old_on = s->ext_on, old_force = s->ext_force_on;
    const int old_count = s->ext_count;
    s->ext_on = s->ext_force_on = false;
    s->ext_count = 0;
    const int rc = [&]() -> int {
        if (block_count == 0 && !row_force) return PK_OK;
        if (!s->have_pattern) return fail(PK_ERR_STATE, "extras before the pattern");
        if (block_count > (1 << 28)) return fail(PK_ERR_ARG, "too many blocks");
        const int n = s->dyn_count;
        if (block_count > 0 && (!blocks || !block_nodes || !rhs_start || !mat_start))
            return fail(PK_ERR_ARG, "set_extras: NULL array");
        PK_CHECK(cudaSetDevice(s->device));
        std::vector<int> zeros(static_cast<size_t>(n) + 1, 0);
        const int* rs = block_count > 0 ? rhs_start : zeros.data();
        const int* ms = block_count > 0 ? mat_start : zeros.data();
        if (rs[0] != 0 || ms[0] != 0) return fail(PK_ERR_ARG, "extras start[0] != 0");
        for (int r = 0; r < n; ++r)
            if (rs[r + 1] < rs[r] || ms[r + 1] < ms[r]) return fail(PK_ERR_ARG, "extras starts not monotone");
        for (long long i = 0; i < 2ll * block_count; ++i)
            if (block_nodes[i] < 0 || block_nodes[i] >= s->node_count) return fail(PK_ERR_ARG, "block node out of range");
        for (int i = 0; i < rs[n]; ++i)
            if (rhs_list[i] < 0 || rhs_list[i] >= block_count) return fail(PK_ERR_ARG, "bad rhs entry");
        for (int i = 0; i < ms[n]; ++i)
            if ((mat_list[i] & 0x7fffffff) >= block_count) return fail(PK_ERR_ARG, "bad matrix entry");
        int r = PK_OK;
        if (block_count > 0) {
            r = upload_real_any(s, s->ext_blocks, blocks, 9 * static_cast<size_t>(block_count));
            if (!r) r = upload_raw<int>(s->ext_nodes, block_nodes, 2 * static_cast<size_t>(block_count), s->stream);
            if (!r && rs[n] > 0) r = upload_raw<int>(s->ext_rhs_list, rhs_list, rs[n], s->stream);
            if (!r && ms[n] > 0) r = upload_raw<int>(s->ext_mat_list, mat_list, ms[n], s->stream);
        }
        if (!r) r = upload_raw<int>(s->ext_rhs_start, rs, static_cast<size_t>(n) + 1, s->stream);
        if (!r) r = upload_raw<int>(s->ext_mat_start, ms, static_cast<size_t>(n) + 1, s->stream);
        if (!r && row_force) r = upload_real_any(s, s->ext_force, row_force, 3 * static_cast<size_t>(n));
        if (r) return r;
        PK_CHECK(cudaStreamSynchronize(s->stream));  // the host arrays may go away
        s->ext_on = true;
        s->ext_force_on = row_force != nullptr;
        s->ext_count = block_count;
        return PK_OK;
    }();
    const void* new_bufs[7] = {s->ext_blocks.p, s->ext_nodes.p, s->ext_rhs_start.p, s->ext_rhs_list.p,
                               s->ext_mat_start.p, s->ext_mat_list.p, s->ext_force.p};
    bool same = rc == PK_OK && s->ext_on == old_on && s->ext_force_on == old_force && s->ext_count == old_count;
    for (int i = 0; i < 7 && same; ++i) same = old_bufs[i] == new_bufs[i];
    if (!same) drop_graph(s);
    return rc;
}

PKCUDA_API int pk_system_set_connections(pk_system* s, int count, const int* nodes, const double* params,
                                         const int* inc_start, const int* inc_list)
{
    if (!s || count < 0) return fail(PK_ERR_ARG, "set_connections");
    // A captured step reads the connection buffers in place: it stays valid when only
    // their contents change (same count, no buffer moved), e.g. a drag's new target.
    const int old_count = s->conn_count;
    const void* old_bufs[5] = {s->conn_nodes.p, s->conn_params.p, s->conn_eval.p, s->conn_inc_start.p,
                               s->conn_inc_list.p};
    s->conn_count = 0;
    const int rc = [&]() -> int {
        if (count == 0) return PK_OK;
        if (!s->have_pattern) return fail(PK_ERR_STATE, "connections before the pattern");
        if (!nodes || !params || !inc_start || (!inc_list && inc_start[s->dyn_count] > 0))
            return fail(PK_ERR_ARG, "set_connections: NULL array");
        if (count > (1 << 29)) return fail(PK_ERR_ARG, "too many connections");
        PK_CHECK(cudaSetDevice(s->device));
        for (long long i = 0; i < 4ll * count; ++i)
            if (nodes[i] < 0 || nodes[i] >= s->node_count) return fail(PK_ERR_ARG, "connection node out of range");
        const int n = s->dyn_count;
        if (inc_start[0] != 0) return fail(PK_ERR_ARG, "conn inc_start[0] != 0");
        for (int r = 0; r < n; ++r)
            if (inc_start[r + 1] < inc_start[r]) return fail(PK_ERR_ARG, "conn inc_start not monotone");
        const int total = inc_start[n];
        for (int i = 0; i < total; ++i)
            if (inc_list[i] < 0 || (inc_list[i] >> 2) >= count) return fail(PK_ERR_ARG, "bad connection incidence");
        int r = upload_raw<int>(s->conn_nodes, nodes, 4 * static_cast<size_t>(count), s->stream);
        if (!r) r = upload_real_any(s, s->conn_params, params, pk::kConnParams * static_cast<size_t>(count));
        if (!r) r = upload_raw<int>(s->conn_inc_start, inc_start, static_cast<size_t>(n) + 1, s->stream);
        if (!r && total > 0) r = upload_raw<int>(s->conn_inc_list, inc_list, total, s->stream);
        if (r) return r;
        PK_CHECK(s->conn_eval.ensure(4 * s->rsize() * static_cast<size_t>(count)));
        s->conn_count = count;
        return PK_OK;
    }();
    const void* new_bufs[5] = {s->conn_nodes.p, s->conn_params.p, s->conn_eval.p, s->conn_inc_start.p,
                               s->conn_inc_list.p};
    bool same = rc == PK_OK && s->conn_count == old_count;
    for (int i = 0; i < 5 && same; ++i) same = old_bufs[i] == new_bufs[i];
    if (!same) drop_graph(s);
    return rc;
}

PKCUDA_API int pk_system_set_pattern(pk_system* s, int dyn_count, const int* dyn_to_node, const int* row_start,
                                     const int* col_index, const int* inc_start, const int* inc_list)
{
    if (!s || dyn_count < 0) return fail(PK_ERR_ARG, "set_pattern");
    if (dyn_count > 0 && (!dyn_to_node || !row_start || !col_index || !inc_start)) return fail(PK_ERR_ARG, "NULL");
    PK_CHECK(cudaSetDevice(s->device));
    // Validate the pattern: monotone rows, sorted unique columns in [row, n).
    const int nnz = dyn_count > 0 ? row_start[dyn_count] : 0;
    if (dyn_count > 0 && row_start[0] != 0) return fail(PK_ERR_ARG, "row_start[0] != 0");
    int max_row = 0;
    bool diag_first = true;
    for (int r = 0; r < dyn_count; ++r) {
        const int a = row_start[r], b = row_start[r + 1];
        if (b < a) return fail(PK_ERR_ARG, "row_start not monotone");
        if (b == a || col_index[a] != r) diag_first = false;
        for (int k = a; k < b; ++k) {
            if (col_index[k] < r || col_index[k] >= dyn_count) return fail(PK_ERR_ARG, "column outside [row, n)");
            if (k > a && col_index[k] <= col_index[k - 1]) return fail(PK_ERR_ARG, "columns not sorted and unique");
        }
        max_row = std::max(max_row, b - a);
        if (dyn_to_node[r] < 0 || dyn_to_node[r] >= s->node_count) return fail(PK_ERR_ARG, "bad dyn_to_node");
    }
    const int inc = dyn_count > 0 ? inc_start[dyn_count] : 0;
    for (int i = 0; i < inc; ++i)
        if (inc_list[i] < 0 || (inc_list[i] >> 2) >= s->tet_count) return fail(PK_ERR_ARG, "bad incidence");
    std::vector<int> lts, ltr, ltb;
    build_transpose(dyn_count, row_start, col_index, lts, ltr, ltb);
    s->dyn_count = dyn_count;
    s->nnz = nnz;
    s->lt_count = static_cast<int>(ltr.size());
    s->inc_count = inc;
    s->slots_ok = false;
    s->max_row = max_row;
    s->diag_first = diag_first;
    int rc = upload_raw<int>(s->dyn_to_node, dyn_to_node, dyn_count, s->stream);
    if (!rc) rc = upload_raw<int>(s->row_start, row_start, dyn_count + 1, s->stream);
    if (!rc) rc = upload_raw<int>(s->col, col_index, nnz, s->stream);
    if (!rc) rc = upload_raw<int>(s->lt_start, lts.data(), lts.size(), s->stream);
    if (!rc) rc = upload_raw<int>(s->lt_row, ltr.data(), ltr.size(), s->stream);
    if (!rc) rc = upload_raw<int>(s->lt_block, ltb.data(), ltb.size(), s->stream);
    if (!rc) rc = upload_raw<int>(s->inc_start, inc_start, dyn_count + 1, s->stream);
    if (!rc) rc = upload_raw<int>(s->inc_list, inc_list, inc, s->stream);
    if (rc) return rc;
    const size_t rs = s->rsize();
    PK_CHECK(s->values.ensure(9 * rs * std::max<size_t>(1, nnz)));
    PK_CHECK(s->rhs.ensure(3 * rs * std::max<size_t>(1, dyn_count)));
    PK_CHECK(s->minv.ensure(9 * rs * std::max<size_t>(1, dyn_count)));
    rc = s->precision == PK_PREC_FP32 ? ensure_solver_buffers(s, max_grid_for<float, float>(s))
         : s->precision == PK_PREC_MIXED ? ensure_solver_buffers(s, max_grid_for<float, double>(s))
                                         : ensure_solver_buffers(s, max_grid_for<double, double>(s));
    if (rc) return rc;
    s->seg_start.clear();
    s->batch_parts = 0;
    s->conn_count = 0;
    s->ext_on = s->ext_force_on = false;
    s->ext_count = 0;
    s->assembled = false;
    drop_graph(s);
    s->h_row_start.assign(row_start, row_start + dyn_count + 1);
    s->h_dyn_to_node.assign(dyn_to_node, dyn_to_node + dyn_count);
    s->h_lts = lts;
    reset_slab(s);
    // Ring-staged PCG tiles (the kernel used where the part-resident one does not apply).
    s->ring_tiles = 0;
    const int rk = requested_kernel();
    if ((rk == -1 || rk == 0 || rk == 3) && dyn_count > 0 && diag_first) {
        std::vector<int> desc;
        const bool ok = s->precision == PK_PREC_FP64 ? build_ring_tiles<double>(dyn_count, row_start, lts, desc)
                                                     : build_ring_tiles<float>(dyn_count, row_start, lts, desc);
        const int mx = s->precision == PK_PREC_FP32    ? ring_max_grid<float, float>(s)
                       : s->precision == PK_PREC_MIXED ? ring_max_grid<float, double>(s)
                                                       : ring_max_grid<double, double>(s);
        const int ntiles = static_cast<int>(desc.size()) / pk::kRingDescInts;
        if (ok && mx > 0 && (ntiles + mx - 1) / mx <= pk::kRingMaxTilesPerBlock) {
            rc = upload_raw<int>(s->ring_desc, desc.data(), desc.size(), s->stream);
            if (rc) return rc;
            s->ring_tiles = ntiles;
        }
    }
    // Staged SpMV tiles: as many rows per tile as fill one cooperative wave (16..64).
    s->ntiles = 0;
    if (requested_kernel() != 2 && staging_enabled() && dyn_count > 0 && s->pcg_max_grid_staged > 0) {
        const int per_block = (dyn_count + s->pcg_max_grid_staged - 1) / s->pcg_max_grid_staged;
        const int rows = s->staged_rows > 0 ? s->staged_rows
                                            : (per_block <= 16 ? 16 : (per_block <= 32 ? 32 : pk::kTileRowsMax));
        std::vector<int> desc;
        if (build_tiles(dyn_count, row_start, lts, rows, desc)) {
            rc = upload_raw<int>(s->tiles, desc.data(), desc.size(), s->stream);
            if (rc) return rc;
            s->ntiles = static_cast<int>(desc.size() / 8);
        }
    }
    s->have_pattern = true;
    return PK_OK;
}

PKCUDA_API int pk_system_step(pk_system* s, const pk_step_params* p)
{
    if (!s || !p) return fail(PK_ERR_ARG, "step");
    if (!s->have_nodes || !s->have_tets || !s->have_pattern) return fail(PK_ERR_STATE, "step before topology");
    if (!(p->dt > 0.0)) return fail(PK_ERR_ARG, "dt must be > 0");
    if (s->dyn_count > 0 && !s->diag_first) return fail(PK_ERR_ARG, "every dynamic row needs its diagonal block first");
    PK_CHECK(cudaSetDevice(s->device));
    if (s->use_graph && s->assembled)
        return s->precision == PK_PREC_FP64 ? run_step_graph<double>(s, *p) : run_step_graph<float>(s, *p);
    return s->precision == PK_PREC_FP64 ? run_step<double>(s, *p) : run_step<float>(s, *p);
}

PKCUDA_API int pk_system_stats(pk_system* s, pk_step_stats* out)
{
    if (!s || !out) return fail(PK_ERR_ARG, "stats");
    PK_CHECK(cudaSetDevice(s->device));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    std::memset(out, 0, sizeof(*out));
    const pk::DevStats& d = *s->host_stats;
    out->iterations = d.iterations;
    out->converged = d.converged;
    out->residual_norm = d.residual_norm;
    out->flags = d.flags;
    out->polar_fp64_count = d.polar_fp64_count;
    out->polar_identity_count = d.polar_identity_count;
    if (s->batched && s->seg_start.size() >= 2 && !(d.flags & (PK_FLAG_PRECOMPUTE_FAILED | PK_FLAG_SINGULAR_DIAG))) {
        // Success flags hold only when every body has them.
        const unsigned success = PK_FLAG_SOLVED | PK_FLAG_INTEGRATED | PK_FLAG_CONVERGED;
        out->flags = (d.flags & ~success) | (success & ~d.batch_missing);
        out->converged = (d.batch_missing & PK_FLAG_CONVERGED) ? 0 : 1;
    }
    if (d.flags & PK_FLAG_BARRIER_TIMEOUT) return fail(PK_ERR_TIMEOUT, "grid barrier timed out");
    return PK_OK;
}

PKCUDA_API int pk_system_get_system_f64(pk_system* s, double* values, double* rhs, double* minv, double* dv)
{
    if (!s || !s->have_pattern) return fail(PK_ERR_STATE, "get_system before set_pattern");
    PK_CHECK(cudaSetDevice(s->device));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    int rc = download_real_any(s, s->values, values, 9 * static_cast<size_t>(s->nnz));
    if (!rc) rc = download_real_any(s, s->rhs, rhs, 3 * static_cast<size_t>(s->dyn_count));
    if (!rc) rc = download_real_any(s, s->minv, minv, 9 * static_cast<size_t>(s->dyn_count));
    if (!rc) rc = download_real_any(s, s->px, dv, 3 * static_cast<size_t>(s->dyn_count));
    return rc;
}

PKCUDA_API int pk_system_solve_given_f64(pk_system* s, const double* values, const double* rhs, const double* minv,
                                         const pk_step_params* p)
{
    if (!s || !p || !s->have_pattern) return fail(PK_ERR_STATE, "solve_given before set_pattern");
    PK_CHECK(cudaSetDevice(s->device));
    int rc = PK_OK;
    if (values) rc = upload_real_any(s, s->values, values, 9 * static_cast<size_t>(s->nnz));
    if (values) s->slab_filled = false;
    if (!rc && rhs) rc = upload_real_any(s, s->rhs, rhs, 3 * static_cast<size_t>(s->dyn_count));
    if (!rc && minv) rc = upload_real_any(s, s->minv, minv, 9 * static_cast<size_t>(s->dyn_count));
    if (rc) return rc;
    PK_CHECK(cudaMemsetAsync(s->stats.p, 0, sizeof(pk::DevStats), s->stream));
    if (s->dyn_count > 0) {
        if (s->precision == PK_PREC_FP32) rc = run_pcg<float, float>(s, *p, 0);
        else if (s->precision == PK_PREC_MIXED) rc = run_pcg<float, double>(s, *p, 0);
        else rc = run_pcg<double, double>(s, *p, 0);
        if (rc) return rc;
    }
    PK_CHECK(cudaMemcpyAsync(s->host_stats, s->stats.p, sizeof(pk::DevStats), cudaMemcpyDeviceToHost, s->stream));
    return PK_OK;
}

PKCUDA_API int pk_system_enable_timing(pk_system* s, int on)
{
    if (!s) return fail(PK_ERR_ARG, "timing");
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
    s->ev_pool.clear();
    s->ev_pending.clear();
    s->t_assemble = s->t_solve = 0;
    s->timed_steps = 0;
    s->launches = 0;
    s->timing = on != 0;
    return PK_OK;
}

PKCUDA_API int pk_system_timings(pk_system* s, double* assemble_ms, double* solve_ms, int* steps,
                                 long long* kernel_launches)
{
    if (!s) return fail(PK_ERR_ARG, "timings");
    PK_CHECK(cudaSetDevice(s->device));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    for (const auto& tr : s->ev_pending) {
        float a = 0, b = 0;
        PK_CHECK(cudaEventElapsedTime(&a, s->ev_pool[tr[0]], s->ev_pool[tr[1]]));
        PK_CHECK(cudaEventElapsedTime(&b, s->ev_pool[tr[1]], s->ev_pool[tr[2]]));
        s->t_assemble += a;
        s->t_solve += b;
        s->timed_steps += 1;
    }
    for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
    s->ev_pool.clear();
    s->ev_pending.clear();
    if (assemble_ms) *assemble_ms = s->t_assemble;
    if (solve_ms) *solve_ms = s->t_solve;
    if (steps) *steps = s->timed_steps;
    if (kernel_launches) *kernel_launches = s->launches;
    return PK_OK;
}

PKCUDA_API int pk_system_set_pcg_grid(pk_system* s, int grid)
{
    if (!s) return fail(PK_ERR_ARG, "pcg grid");
    PK_CHECK(cudaSetDevice(s->device));
    drop_graph(s);
    s->pcg_grid_override = std::max(0, grid);
    reset_slab(s);
    if (s->ring_tiles > 0) {
        if (s->precision == PK_PREC_FP32) return ring_grid_for<float, float>(s);
        if (s->precision == PK_PREC_MIXED) return ring_grid_for<float, double>(s);
        return ring_grid_for<double, double>(s);
    }
    if (s->precision == PK_PREC_FP32) return pcg_grid_for<float, float>(s);
    if (s->precision == PK_PREC_MIXED) return pcg_grid_for<float, double>(s);
    return pcg_grid_for<double, double>(s);
}

PKCUDA_API int pk_system_set_segments(pk_system* s, int segment_count, const int* segment_row_start)
{
    if (!s || segment_count < 0 || (segment_count > 0 && !segment_row_start)) return fail(PK_ERR_ARG, "segments");
    if (!s->have_pattern) return fail(PK_ERR_STATE, "set_segments before set_pattern");
    if (segment_count > 0) {
        if (segment_row_start[0] != 0 || segment_row_start[segment_count] != s->dyn_count)
            return fail(PK_ERR_ARG, "segments must cover the dynamic rows");
        for (int b = 0; b < segment_count; ++b)
            if (segment_row_start[b + 1] < segment_row_start[b]) return fail(PK_ERR_ARG, "segments not monotone");
        // A body's rows must not reference another body's rows (independent systems).
        std::vector<int> seg_of(static_cast<size_t>(s->dyn_count));
        for (int b = 0; b < segment_count; ++b)
            for (int r = segment_row_start[b]; r < segment_row_start[b + 1]; ++r) seg_of[r] = b;
        std::vector<int> rs(static_cast<size_t>(s->dyn_count) + 1), col(static_cast<size_t>(s->nnz));
        PK_CHECK(cudaSetDevice(s->device));
        PK_CHECK(cudaMemcpy(rs.data(), s->row_start.p, rs.size() * sizeof(int), cudaMemcpyDeviceToHost));
        PK_CHECK(cudaMemcpy(col.data(), s->col.p, col.size() * sizeof(int), cudaMemcpyDeviceToHost));
        for (int r = 0; r < s->dyn_count; ++r)
            for (int k = rs[r]; k < rs[r + 1]; ++k)
                if (seg_of[col[k]] != seg_of[r]) return fail(PK_ERR_ARG, "a block couples two segments");
    }
    s->seg_start.assign(segment_row_start, segment_row_start + (segment_count > 0 ? segment_count + 1 : 0));
    s->batch_parts = 0;
    reset_slab(s);
    drop_graph(s);
    return PK_OK;
}

PKCUDA_API int pk_system_set_batched(pk_system* s, int on)
{
    if (!s) return fail(PK_ERR_ARG, "batched");
    if (s->batched != (on != 0)) drop_graph(s);
    s->batched = on != 0;
    return PK_OK;
}

PKCUDA_API int pk_system_segment_stats(pk_system* s, int segment_count, int* iterations, int* converged,
                                       double* residual_norm, unsigned* flags)
{
    if (!s || segment_count < 0) return fail(PK_ERR_ARG, "segment_stats");
    const int nseg = static_cast<int>(s->seg_start.size()) - 1;
    if (!s->batched || nseg <= 0) return fail(PK_ERR_STATE, "no batched solve");
    if (segment_count != nseg) return fail(PK_ERR_ARG, "segment count mismatch");
    PK_CHECK(cudaSetDevice(s->device));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    std::vector<pk::BatchBodyStats> bs(static_cast<size_t>(nseg));
    if (s->body_stats.p)
        PK_CHECK(cudaMemcpy(bs.data(), s->body_stats.p, bs.size() * sizeof(pk::BatchBodyStats), cudaMemcpyDeviceToHost));
    for (int b = 0; b < nseg; ++b) {
        if (iterations) iterations[b] = bs[b].iterations;
        if (converged) converged[b] = bs[b].converged;
        if (residual_norm) residual_norm[b] = bs[b].residual_norm;
        if (flags) flags[b] = bs[b].flags;
    }
    return PK_OK;
}

PKCUDA_API int pk_system_set_refinement(pk_system* s, int passes)
{
    if (!s || passes < 0 || passes > 16) return fail(PK_ERR_ARG, "refinement passes must be 0..16");
    if (s->refine_passes != passes) drop_graph(s);
    s->refine_passes = passes;
    return PK_OK;
}

PKCUDA_API int pk_system_slab_form(pk_system* s)
{
    if (!s || (s->last_kernel != 3 && s->last_kernel != 5)) return -1;
    return s->slab_sym ? 1 : 0;
}

PKCUDA_API int pk_system_pcg_kernel(pk_system* s, int* blocks)
{
    if (!s) return fail(PK_ERR_ARG, "pcg_kernel");
    if (blocks) *blocks = s->last_blocks;
    return s->last_kernel;
}

PKCUDA_API int pk_system_set_graph(pk_system* s, int on)
{
    if (!s) return fail(PK_ERR_ARG, "graph");
    PK_CHECK(cudaSetDevice(s->device));
    if (!on) {
        cudaStreamSynchronize(s->stream);
        drop_graph(s);
    }
    s->use_graph = on != 0;
    return PK_OK;
}

namespace {

// Times `repeats` solves (no integration) of the assembled system with the current
// kernel settings; mean milliseconds, or a negative PK_ERR_* code.
double time_solves(pk_system* s, const pk_step_params& p, int repeats)
{
    pk_step_params q = p;
    q.integrate = 0;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return PK_ERR_CUDA;
    int rc = PK_OK;
    auto solve = [&] {
        if (s->precision == PK_PREC_FP32) return run_pcg<float, float>(s, q, 0);
        if (s->precision == PK_PREC_MIXED) return run_pcg<float, double>(s, q, 0);
        return run_pcg<double, double>(s, q, 0);
    };
    rc = solve();  // warm-up (also builds batch parts)
    if (!rc && cudaEventRecord(e0, s->stream) != cudaSuccess) rc = PK_ERR_CUDA;
    for (int i = 0; i < repeats && !rc; ++i) rc = solve();
    float ms = 0.0f;
    if (!rc && (cudaEventRecord(e1, s->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
        rc = PK_ERR_CUDA;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc ? double(rc) : double(ms) / std::max(1, repeats);
}

}  // namespace

PKCUDA_API int pk_system_autotune(pk_system* s, const pk_step_params* p, int repeats, int* chosen, double* best_ms)
{
    if (!s || !p) return fail(PK_ERR_ARG, "autotune");
    if (!s->have_pattern || !s->assembled || s->dyn_count <= 0)
        return fail(PK_ERR_STATE, "autotune needs an assembled system (step once first)");
    PK_CHECK(cudaSetDevice(s->device));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    drop_graph(s);
    repeats = std::max(1, repeats);
    int best = -1;
    double best_t = 1e300;
    if (s->batched && s->seg_start.size() >= 2) {
        // Candidates: the per-body batch kernel with the smallest part a body is cut into
        // (0-5); the part-resident kernel with one group per body (6) where it applies.
        const int cand[] = {32, 64, 128, 256, 512, 1024};
        int i = 0;
        double slab_t = -1.0;
        if (s->precision != PK_PREC_FP64) {
            s->batch_slab = true;
            int rc = ensure_slab_any(s);
            if (rc) return rc;
            if (s->slab_parts > 0 && s->slab_for_bodies) {
                slab_t = time_solves(s, *p, repeats);
                if (slab_t < 0) return static_cast<int>(slab_t);
            }
        }
        s->batch_slab = false;
        for (int rows : cand) {
            s->batch_min_rows = rows;
            s->batch_parts = 0;
            const double t = time_solves(s, *p, repeats);
            if (t < 0) return static_cast<int>(t);
            if (t < best_t) best_t = t, best = i;
            ++i;
        }
        s->batch_min_rows = cand[best];
        s->batch_parts = 0;
        int rc = ensure_batch_parts_any(s);
        if (rc) return rc;
        if (slab_t >= 0.0 && slab_t < best_t) {
            best_t = slab_t;
            best = 6;
            s->batch_slab = true;
        }
    } else {
        // Candidates: ring kernel; staged kernel with 16 / 32 / 64-row tiles; plain kernel;
        // part-resident kernel.
        struct Cand {
            int kernel, rows;
        };
        const Cand cand[] = {{0, 0}, {1, 16}, {1, 32}, {1, pk::kTileRowsMax}, {2, 0}, {3, 0}};
        int rc0 = ensure_slab_any(s);
        if (rc0) return rc0;
        auto retile = [&](int rows) -> int {
            std::vector<int> desc;
            s->ntiles = 0;
            if (!build_tiles(s->dyn_count, s->h_row_start.data(), s->h_lts, rows, desc)) return PK_OK;
            int rc = upload_raw<int>(s->tiles, desc.data(), desc.size(), s->stream);
            if (rc) return rc;
            s->ntiles = static_cast<int>(desc.size() / 8);
            return PK_OK;
        };
        int i = 0;
        for (const Cand& c : cand) {
            if (c.kernel == 0 && s->ring_tiles <= 0) { ++i; continue; }
            if (c.kernel == 3 && s->slab_parts <= 0) { ++i; continue; }
            if (c.kernel == 1) {
                int rc = retile(c.rows);
                if (rc) return rc;
                if (s->ntiles <= 0) { ++i; continue; }
            }
            s->kernel_choice = c.kernel;
            const double t = time_solves(s, *p, repeats);
            if (t < 0) return static_cast<int>(t);
            if (t < best_t) best_t = t, best = i;
            ++i;
        }
        if (best < 0) return fail(PK_ERR_UNSUPPORTED, "no PCG kernel candidate");
        s->kernel_choice = cand[best].kernel;
        s->staged_rows = cand[best].rows;
        if (cand[best].kernel == 1) {
            int rc = retile(cand[best].rows);
            if (rc) return rc;
        }
    }
    if (chosen) *chosen = best;
    if (best_ms) *best_ms = best_t;
    return PK_OK;
}

}  // extern "C"

namespace {

template <class Real>
int adjoint_step(pk_system* s, const pk_step_params& p, const double* xbar_next, const double* vbar_next, double* xbar,
                 double* vbar, double* theta_bar)
{
    const int n = s->dyn_count, nn = s->node_count, T = s->tet_count;
    // 1. The forward step at the current state, without integration: A, b, delta-v.
    pk_step_params q = p;
    q.integrate = 0;
    q.explicit_mode = 0;
    int rc = run_step<Real>(s, q);
    if (rc) return rc;
    pk_step_stats st{};
    rc = pk_system_stats(s, &st);
    if (rc) return rc;
    if (!(st.flags & PK_FLAG_SOLVED)) return fail(PK_ERR_STATE, "adjoint: the forward solve failed");
    std::vector<double> du(3 * static_cast<size_t>(n)), g(3 * static_cast<size_t>(n));
    rc = download_real<Real>(s->px, du.data(), du.size(), s->stream);
    if (rc) return rc;
    // 2. Adjoint right-hand side: adjoint of v' plus dt times the adjoint of x' (dynamic rows).
    for (int r = 0; r < n; ++r) {
        const int node = s->h_dyn_to_node[r];
        for (int c = 0; c < 3; ++c) g[3 * r + c] = vbar_next[3 * node + c] + p.dt * xbar_next[3 * node + c];
    }
    rc = upload_real<Real>(s->rhs, g.data(), g.size(), s->stream);
    if (rc) return rc;
    // 3. A w = g with the same PCG (A symmetric).
    PK_CHECK(cudaMemsetAsync(s->stats.p, 0, sizeof(pk::DevStats), s->stream));
    if (s->precision == PK_PREC_FP32) rc = run_pcg<float, float>(s, q, 0);
    else if (s->precision == PK_PREC_MIXED) rc = run_pcg<float, double>(s, q, 0);
    else rc = run_pcg<double, double>(s, q, 0);
    if (rc) return rc;
    PK_CHECK(cudaMemcpyAsync(s->host_stats, s->stats.p, sizeof(pk::DevStats), cudaMemcpyDeviceToHost, s->stream));
    PK_CHECK(cudaStreamSynchronize(s->stream));
    if (!(s->host_stats->flags & PK_FLAG_SOLVED)) return fail(PK_ERR_STATE, "adjoint: the adjoint solve failed");
    std::vector<double> w(3 * static_cast<size_t>(n)), aw(3 * static_cast<size_t>(n));
    rc = download_real<Real>(s->px, w.data(), w.size(), s->stream);
    if (rc) return rc;
    // A w (for the velocity sensitivity dt^2 K w = A w - M w)
    pk::BsrView<Real> view{};
    view.n = n;
    view.row_start = s->row_start.as<int>();
    view.col = s->col.as<int>();
    view.values = s->values.as<Real>();
    view.lt_start = s->lt_start.as<int>();
    view.lt_row = s->lt_row.as<int>();
    view.lt_block = s->lt_block.as<int>();
    PK_CHECK(pk::launch_spmv_kernel<Real>(view, s->px.as<Real>(), s->pq.as<Real>(), s->stream));
    rc = download_real<Real>(s->pq, aw.data(), aw.size(), s->stream);
    if (rc) return rc;
    // 4. Element sensitivities.
    PK_CHECK(s->adj_w.ensure(sizeof(double) * w.size()));
    PK_CHECK(s->adj_du.ensure(sizeof(double) * du.size()));
    PK_CHECK(s->adj_grad.ensure(sizeof(double) * 12 * static_cast<size_t>(std::max(1, T))));
    PK_CHECK(s->adj_theta.ensure(sizeof(double) * static_cast<size_t>(std::max(1, T))));
    PK_CHECK(cudaMemcpyAsync(s->adj_w.p, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice, s->stream));
    PK_CHECK(cudaMemcpyAsync(s->adj_du.p, du.data(), sizeof(double) * du.size(), cudaMemcpyHostToDevice, s->stream));
    pk::AdjointArgs<Real> a{};
    a.tet_count = T;
    a.nodes = s->tet_nodes.as<int4>();
    a.enabled = s->tet_enabled.as<unsigned char>();
    a.dm_inv = s->dm_inv.as<Real>();
    a.params = s->tet_params.as<Real>();
    a.x = s->x.as<Real>();
    a.v = s->v.as<Real>();
    a.node_to_dyn = s->node_to_dyn.as<int>();
    a.w = s->adj_w.as<double>();
    a.du = s->adj_du.as<double>();
    a.dt = static_cast<double>(static_cast<Real>(p.dt));
    a.linear = p.linear;
    a.flags = &s->stats.as<pk::DevStats>()->flags;
    a.tet_grad = s->adj_grad.as<double>();
    a.tet_theta = s->adj_theta.as<double>();
    PK_CHECK(pk::launch_adjoint_tet_kernel<Real>(a, s->stream));
    std::vector<double> grad(12 * static_cast<size_t>(T)), th(static_cast<size_t>(T));
    if (T > 0) {
        PK_CHECK(cudaMemcpyAsync(grad.data(), s->adj_grad.p, sizeof(double) * grad.size(), cudaMemcpyDeviceToHost,
                                 s->stream));
        PK_CHECK(cudaMemcpyAsync(th.data(), s->adj_theta.p, sizeof(double) * th.size(), cudaMemcpyDeviceToHost,
                                 s->stream));
    }
    PK_CHECK(cudaStreamSynchronize(s->stream));
    // 5. Node sensitivities before the step.  Positions: x' = x + dt v' carries the
    // adjoint of x' back unchanged, plus dJ/dx on dynamic nodes (fixed nodes never move).
    // Velocities: v' = v + du carries g back on dynamic rows, plus d(w.b)/dv = -dt^2 K w
    // - dt c w with dt^2 K w = A w - m w (c: the damping of the node's active tets);
    // fixed nodes keep their adjoint (their velocity only enters through b's coupling
    // blocks, which the dynamic-row matrix does not hold: not propagated).
    std::copy(xbar_next, xbar_next + 3 * static_cast<size_t>(nn), xbar);
    std::copy(vbar_next, vbar_next + 3 * static_cast<size_t>(nn), vbar);
    std::vector<double> csum(static_cast<size_t>(nn), 0.0);
    for (int t = 0; t < T; ++t) {
        if (!(s->h_enabled[t] & 1u)) continue;
        for (int k = 0; k < 4; ++k) {
            const int node = s->h_tet_nodes[4 * static_cast<size_t>(t) + k];
            csum[node] += s->h_damping[t];
            if (s->h_node_to_dyn[node] < 0) continue;
            for (int c = 0; c < 3; ++c) xbar[3 * node + c] += grad[12 * static_cast<size_t>(t) + 3 * k + c];
        }
        if (theta_bar) theta_bar[t] += th[t];
    }
    for (int r = 0; r < n; ++r) {
        const int node = s->h_dyn_to_node[r];
        const double m = s->h_mass[node];
        for (int c = 0; c < 3; ++c)
            vbar[3 * node + c] = g[3 * r + c] - aw[3 * r + c] + m * w[3 * r + c] - p.dt * csum[node] * w[3 * r + c];
    }
    return PK_OK;
}

}  // namespace

extern "C" {

PKCUDA_API int pk_system_adjoint_step(pk_system* s, const pk_step_params* p, const double* xbar_next,
                                      const double* vbar_next, double* xbar, double* vbar, double* theta_bar)
{
    if (!s || !p || !xbar_next || !vbar_next || !xbar || !vbar) return fail(PK_ERR_ARG, "adjoint_step");
    if (!s->have_nodes || !s->have_tets || !s->have_pattern) return fail(PK_ERR_STATE, "adjoint before topology");
    if (!(p->dt > 0.0)) return fail(PK_ERR_ARG, "dt must be > 0");
    if (s->dyn_count > 0 && !s->diag_first) return fail(PK_ERR_ARG, "every dynamic row needs its diagonal block first");
    if (s->conn_count > 0) return fail(PK_ERR_STATE, "the adjoint step does not take point connections");
    if (s->ext_on) return fail(PK_ERR_STATE, "the adjoint step does not take host-emitted contributions");
    PK_CHECK(cudaSetDevice(s->device));
    drop_graph(s);
    if (s->dyn_count == 0) {
        std::copy(xbar_next, xbar_next + 3 * static_cast<size_t>(s->node_count), xbar);
        std::copy(vbar_next, vbar_next + 3 * static_cast<size_t>(s->node_count), vbar);
        return PK_OK;
    }
    const bool batched = s->batched;
    s->batched = false;  // one coupled solve: the adjoint of the world's step
    const int rc = s->precision == PK_PREC_FP64
                       ? adjoint_step<double>(s, *p, xbar_next, vbar_next, xbar, vbar, theta_bar)
                       : adjoint_step<float>(s, *p, xbar_next, vbar_next, xbar, vbar, theta_bar);
    s->batched = batched;
    return rc;
}

PKCUDA_API int pk_bsr_transpose_index(int n, const int* row_start, const int* col_index, int* lt_start, int* lt_row,
                                      int* lt_block)
{
    if (n < 0 || (n > 0 && (!row_start || !col_index))) return fail(PK_ERR_ARG, "transpose index");
    std::vector<int> a, b, c;
    build_transpose(n, row_start, col_index, a, b, c);
    if (lt_start) std::copy(a.begin(), a.end(), lt_start);
    if (lt_row) std::copy(b.begin(), b.end(), lt_row);
    if (lt_block) std::copy(c.begin(), c.end(), lt_block);
    return static_cast<int>(b.size());
}

}  // extern "C"

namespace {

// Host replay of the ring-staged kernel's phase A addressing (see pk_pcg_ring.cu): builds
// the tiling, fills one stage buffer per tile byte for byte as the producer's bulk copies
// do (same widened spans, same offsets, from arrays with the device allocations' slack),
// then evaluates every row as the consumer lanes do: upper blocks and columns from the
// stage, transposed lower blocks and neighbour values from the full arrays through the
// staged transposed index.  Every index is checked against its capacity and span; the
// number of violations is returned (0 = consistent).
template <class Real>
int ring_selfcheck(int n, const int* row_start, const int* col, const double* values_d, const double* x_d,
                   double* y, int* out_tiles, int* out_max_span)
{
    using T = pk::RingTile<Real>;
    using LY = pk::RingLayout<Real>;
    std::vector<int> lts, ltr, ltb, desc;
    build_transpose(n, row_start, col, lts, ltr, ltb);
    if (!build_ring_tiles<Real>(n, row_start, lts, desc)) return -1;
    const int nnz = n > 0 ? row_start[n] : 0;
    const int ntiles = static_cast<int>(desc.size()) / pk::kRingDescInts;
    // "Device" arrays with the same 1 KB slack as DevBuf.
    auto padded = [](const void* src, size_t bytes) {
        std::vector<unsigned char> v(bytes + DevBuf::kSlack, 0);
        if (bytes) std::memcpy(v.data(), src, bytes);
        return v;
    };
    std::vector<Real> vr(9 * static_cast<size_t>(nnz));
    for (size_t i = 0; i < vr.size(); ++i) vr[i] = static_cast<Real>(values_d[i]);
    const auto dvals = padded(vr.data(), sizeof(Real) * vr.size());
    const auto drs = padded(row_start, 4 * size_t(n + 1));
    const auto dlts = padded(lts.data(), 4 * lts.size());
    const auto dcol = padded(col, 4 * size_t(nnz));
    const auto dltr = padded(ltr.data(), 4 * ltr.size());
    const auto dltb = padded(ltb.data(), 4 * ltb.size());
    std::vector<unsigned char> stage(LY::kBytes);
    int bad = 0, max_span = 0;
    for (int t = 0; t < ntiles; ++t) {
        const int* d = desc.data() + pk::kRingDescInts * t;
        const int ra = d[0], rb = d[1], rs0 = d[2], nrs = d[3], k0 = d[4], nk = d[5], e0 = d[6], ne = d[7];
        // The kernel's descriptor check.
        const bool ok = rb > ra && rb - ra <= T::kRows && ra >= rs0 && nrs > 0 && nrs <= T::kRsCap &&
                        rb + 1 <= rs0 + nrs && nk > 0 && nk <= T::kCapU && ne >= 0 && ne <= T::kCapL &&
                        ((rs0 | nrs | k0 | nk | e0 | ne) & 3) == 0;
        if (!ok) {
            ++bad;
            continue;
        }
        max_span = std::max(max_span, nk);
        // Bulk copies: inside the source arrays plus slack, inside their stage regions.
        bad += (4 * size_t(rs0 + nrs) > drs.size()) + (4 * size_t(rs0 + nrs) > dlts.size()) +
               (sizeof(Real) * 9 * size_t(k0 + nk) > dvals.size()) + (4 * size_t(k0 + nk) > dcol.size()) +
               (4 * size_t(e0 + ne) > dltr.size()) + (4 * size_t(e0 + ne) > dltb.size());
        bad += (LY::kRs + 4 * size_t(nrs) > LY::kLts) + (LY::kLts + 4 * size_t(nrs) > LY::kVals) +
               (LY::kVals + sizeof(Real) * 9 * size_t(nk) > LY::kCol) + (LY::kCol + 4 * size_t(nk) > LY::kLtr) +
               (LY::kLtr + 4 * size_t(ne) > LY::kLtb) + (LY::kLtb + 4 * size_t(ne) > LY::kBytes);
        if (bad) continue;
        unsigned char* st = stage.data();
        std::fill(stage.begin(), stage.end(), 0xFF);
        std::memcpy(st + LY::kRs, drs.data() + 4 * size_t(rs0), 4 * nrs);
        std::memcpy(st + LY::kLts, dlts.data() + 4 * size_t(rs0), 4 * nrs);
        std::memcpy(st + LY::kVals, dvals.data() + sizeof(Real) * 9 * size_t(k0), sizeof(Real) * 9 * nk);
        std::memcpy(st + LY::kCol, dcol.data() + 4 * size_t(k0), 4 * nk);
        if (ne > 0) {
            std::memcpy(st + LY::kLtr, dltr.data() + 4 * size_t(e0), 4 * ne);
            std::memcpy(st + LY::kLtb, dltb.data() + 4 * size_t(e0), 4 * ne);
        }
        const int* srs = reinterpret_cast<const int*>(st + LY::kRs);
        const int* slts = reinterpret_cast<const int*>(st + LY::kLts);
        const Real* svals = reinterpret_cast<const Real*>(st + LY::kVals);
        const int* scol = reinterpret_cast<const int*>(st + LY::kCol);
        const int* sltr = reinterpret_cast<const int*>(st + LY::kLtr);
        const int* sltb = reinterpret_cast<const int*>(st + LY::kLtb);
        for (int lr = 0; lr < rb - ra; ++lr) {
            const int r = ra + lr, o = r - rs0;
            const int ks = srs[o], nu = srs[o + 1] - ks, ls = slts[o], tot = nu + (slts[o + 1] - ls);
            bad += !(ks == row_start[r] && nu == row_start[r + 1] - row_start[r] && ls == lts[r]);
            double acc[3] = {0, 0, 0};
            for (int j = 0; j < tot; ++j) {
                const bool lower = j >= nu;
                int c, k;
                const Real* B;
                if (!lower) {
                    const int kk = ks + j - k0;
                    if (!(kk >= 0 && kk < nk && kk < T::kCapU)) { ++bad; continue; }
                    c = scol[kk];
                    B = svals + 9 * kk;
                } else {
                    const int ee = ls + (j - nu) - e0;
                    if (!(ee >= 0 && ee < ne && ee < T::kCapL)) { ++bad; continue; }
                    c = sltr[ee];
                    k = sltb[ee];
                    if (!(k >= 0 && k < nnz)) { ++bad; continue; }
                    B = vr.data() + 9 * size_t(k);
                }
                if (!(c >= 0 && c < n)) { ++bad; continue; }
                const double xc[3] = {double(Real(x_d[3 * c])), double(Real(x_d[3 * c + 1])),
                                      double(Real(x_d[3 * c + 2]))};
                for (int i = 0; i < 3; ++i)
                    for (int m = 0; m < 3; ++m)
                        acc[i] += lower ? double(B[3 * i + m]) * xc[m] : double(B[3 * m + i]) * xc[m];
            }
            for (int i = 0; i < 3; ++i) y[3 * r + i] = acc[i];
        }
    }
    if (out_tiles) *out_tiles = ntiles;
    if (out_max_span) *out_max_span = max_span;
    return bad;
}

}  // namespace

extern "C" {

PKCUDA_API int pk_slab_plan_batched_selfcheck(int n, const int* row_start, const int* col_index, const double* values,
                                              const double* x, const double* coords, const int* segment_row_start,
                                              int segment_count, int max_blocks, int form, double* y, int* info)
{
    if (n <= 0 || segment_count <= 0 || max_blocks <= 0 || !row_start || !col_index || !values || !x || !y ||
        !segment_row_start)
        return fail(PK_ERR_ARG, "slab batched selfcheck");
    for (int r = 0; r < n; ++r)
        for (int k = row_start[r]; k < row_start[r + 1]; ++k)
            if (col_index[k] < r || col_index[k] >= n) return fail(PK_ERR_ARG, "column outside [row, n)");
    std::vector<int> lts, ltr, ltb;
    build_transpose(n, row_start, col_index, lts, ltr, ltb);
    pk::SlabPlan plan;
    const std::string why = pk::build_slab_plan_batched(n, row_start, col_index, lts.data(), ltr.data(), ltb.data(),
                                                        coords, segment_row_start, segment_count, max_blocks, plan,
                                                        form);
    if (!why.empty()) return fail(PK_ERR_UNSUPPORTED, "slab layout: " + why);
    // Groups: consecutive parts of one body inside one launch, sizes matching.
    const int launches = static_cast<int>(plan.launch_start.size()) - 1;
    for (int l = 0; l < launches; ++l) {
        const int p0 = plan.launch_start[l], p1 = plan.launch_start[l + 1];
        if (p1 - p0 > max_blocks || p1 <= p0) return fail(PK_ERR_STATE, "slab layout: bad launch");
        for (int p = p0; p < p1; ++p) {
            const int* pi = plan.part_info.data() + static_cast<size_t>(pk::kSlabPartInts) * p;
            const int first = pi[6], size = pi[7];
            if (first < 0 || size < 1 || p0 + first + size > p1 || p - p0 < first || p - p0 >= first + size)
                return fail(PK_ERR_STATE, "slab layout: bad group");
            for (int q = p0 + first; q < p0 + first + size; ++q)
                if (plan.part_body[q] != plan.part_body[p]) return fail(PK_ERR_STATE, "slab layout: mixed group");
            const int b = plan.part_body[p];
            const int r0 = plan.perm[pi[0]];
            if (r0 < segment_row_start[b] || r0 >= segment_row_start[b + 1])
                return fail(PK_ERR_STATE, "slab layout: part outside its body");
        }
    }
    const std::string order = pk::slab_check_halo_order(plan, row_start, col_index, lts.data(), ltr.data());
    if (!order.empty()) return fail(PK_ERR_STATE, "slab layout: " + order);
    pk::slab_spmv_host(plan, row_start[n], values, x, y);
    if (info) {
        info[0] = plan.parts;
        info[1] = plan.max_window;
        info[2] = plan.max_tiles;
        info[3] = static_cast<int>(plan.stream.size() / 1024);
        info[4] = launches;
        info[5] = plan.sym ? 1 : 0;
    }
    return PK_OK;
}

PKCUDA_API int pk_slab_plan_selfcheck(int n, const int* row_start, const int* col_index, const double* values,
                                      const double* x, const double* coords, int parts, int form, double* y, int* info)
{
    if (n <= 0 || parts <= 0 || !row_start || !col_index || !values || !x || !y)
        return fail(PK_ERR_ARG, "slab selfcheck");
    if (row_start[0] != 0) return fail(PK_ERR_ARG, "row_start[0] != 0");
    for (int r = 0; r < n; ++r) {
        if (row_start[r + 1] < row_start[r]) return fail(PK_ERR_ARG, "row_start not monotone");
        for (int k = row_start[r]; k < row_start[r + 1]; ++k) {
            if (col_index[k] < r || col_index[k] >= n) return fail(PK_ERR_ARG, "column outside [row, n)");
            if (k > row_start[r] && col_index[k] <= col_index[k - 1]) return fail(PK_ERR_ARG, "columns not sorted");
        }
    }
    std::vector<int> lts, ltr, ltb;
    build_transpose(n, row_start, col_index, lts, ltr, ltb);
    pk::SlabPlan plan;
    const std::string why =
        pk::build_slab_plan(n, row_start, col_index, lts.data(), ltr.data(), ltb.data(), coords, parts, plan, form);
    if (!why.empty()) return fail(PK_ERR_UNSUPPORTED, "slab layout: " + why);
    const std::string order = pk::slab_check_halo_order(plan, row_start, col_index, lts.data(), ltr.data());
    if (!order.empty()) return fail(PK_ERR_STATE, "slab layout: " + order);
    pk::slab_spmv_host(plan, row_start[n], values, x, y);
    if (info) {
        info[0] = plan.parts;
        info[1] = plan.max_window;
        info[2] = plan.max_tiles;
        info[3] = static_cast<int>(plan.stream.size() / 1024);
        info[4] = plan.sym ? 1 : 0;
    }
    return PK_OK;
}

PKCUDA_API int pk_ring_tiling_selfcheck(int precision, int n, const int* row_start, const int* col_index,
                                        const double* values, const double* x, double* y, int* tiles, int* max_span)
{
    if (n <= 0 || !row_start || !col_index || !values || !x || !y) return fail(PK_ERR_ARG, "selfcheck");
    const int rc = precision == PK_PREC_FP64
                       ? ring_selfcheck<double>(n, row_start, col_index, values, x, y, tiles, max_span)
                       : ring_selfcheck<float>(n, row_start, col_index, values, x, y, tiles, max_span);
    if (rc < 0) return fail(PK_ERR_UNSUPPORTED, "a row does not fit a ring stage");
    return rc;
}

// Standalone SpMV on host arrays: y = A x with A stored upper-only.
PKCUDA_API int pk_bsr_multiply(int device, int precision, int n, const int* row_start, const int* col_index,
                               const double* values, const double* x, double* y)
{
    if (n < 0 || (n > 0 && (!row_start || !col_index || !values || !x || !y))) return fail(PK_ERR_ARG, "multiply");
    if (n == 0) return PK_OK;
    int rc = use_device(device);
    if (rc) return rc;
    pk_system* s = nullptr;
    rc = pk_system_create(device, precision, &s);
    if (rc) return rc;
    struct Guard {
        pk_system* s;
        ~Guard() { pk_system_destroy(s); }
    } guard{s};
    const int nnz = row_start[n];
    std::vector<int> lts, ltr, ltb;
    build_transpose(n, row_start, col_index, lts, ltr, ltb);
    DevBuf drs, dcol, dlts, dltr, dltb, dval, dx, dy;
    rc = upload_raw<int>(drs, row_start, n + 1, s->stream);
    if (!rc) rc = upload_raw<int>(dcol, col_index, nnz, s->stream);
    if (!rc) rc = upload_raw<int>(dlts, lts.data(), lts.size(), s->stream);
    if (!rc) rc = upload_raw<int>(dltr, ltr.data(), ltr.size(), s->stream);
    if (!rc) rc = upload_raw<int>(dltb, ltb.data(), ltb.size(), s->stream);
    if (!rc) rc = upload_real_any(s, dval, values, 9 * static_cast<size_t>(nnz));
    if (!rc) rc = upload_real_any(s, dx, x, 3 * static_cast<size_t>(n));
    if (rc) return rc;
    PK_CHECK(dy.ensure(3 * s->rsize() * static_cast<size_t>(n)));
    if (precision == PK_PREC_FP64) {
        pk::BsrView<double> a{n, drs.as<int>(), dcol.as<int>(), dval.as<double>(), dlts.as<int>(), dltr.as<int>(),
                              dltb.as<int>()};
        PK_CHECK(pk::launch_spmv_kernel<double>(a, dx.as<double>(), dy.as<double>(), s->stream));
    } else {
        pk::BsrView<float> a{n, drs.as<int>(), dcol.as<int>(), dval.as<float>(), dlts.as<int>(), dltr.as<int>(),
                             dltb.as<int>()};
        PK_CHECK(pk::launch_spmv_kernel<float>(a, dx.as<float>(), dy.as<float>(), s->stream));
    }
    return download_real_any(s, dy, y, 3 * static_cast<size_t>(n));
}

// Standalone PCG on host arrays, with the reference's argument checks.
PKCUDA_API int pk_pcg(int device, int precision, int n, const int* row_start, const int* col_index,
                      const double* values, const double* b, const double* minv, int minv_count, int max_iterations,
                      double tolerance, double* x, pk_cg_result* out)
{
    if (!out || n < 0) return fail(PK_ERR_ARG, "pcg");
    std::memset(out, 0, sizeof(*out));
    if (n == 0) {
        out->converged = 1;  // empty rhs: cleared output, converged (ConjugateGradientSolver.cpp:124-131)
        return PK_OK;
    }
    if (!row_start || !col_index || !values || !b || !x) return fail(PK_ERR_ARG, "pcg: NULL array");
    if (minv_count != n || !minv) {
        // ApplyPreconditioner fails on a size mismatch: x = 0, result cleared (:150-153).
        bool bad = max_iterations <= 0 || !std::isfinite(tolerance) || tolerance <= 0.0;
        for (int i = 0; i < 3 * n && !bad; ++i) bad = !std::isfinite(b[i]);
        if (!bad) {
            for (int i = 0; i < 3 * n; ++i) x[i] = 0.0;
            out->have_solution = 1;
        }
        return PK_OK;
    }
    pk_system* s = nullptr;
    int rc = pk_system_create(device, precision, &s);
    if (rc) return rc;
    struct Guard {
        pk_system* s;
        ~Guard() { pk_system_destroy(s); }
    } guard{s};
    std::vector<int> n2d(static_cast<size_t>(n));
    std::vector<double> mass(static_cast<size_t>(n), 1.0);
    std::vector<int> inc(static_cast<size_t>(n) + 1, 0);
    for (int i = 0; i < n; ++i) n2d[i] = i;
    rc = pk_system_set_nodes(s, n, n2d.data(), mass.data());
    if (!rc) rc = pk_system_set_tets(s, 0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    if (!rc) rc = pk_system_set_pattern(s, n, n2d.data(), row_start, col_index, inc.data(), nullptr);
    if (rc) return rc;
    pk_step_params p{};
    p.dt = 1.0;
    p.max_iterations = max_iterations;
    p.tolerance = tolerance;
    p.use_jacobi = 1;
    p.integrate = 0;
    rc = pk_system_solve_given_f64(s, values, b, minv, &p);
    if (rc) return rc;
    pk_step_stats st{};
    rc = pk_system_stats(s, &st);
    if (rc) return rc;
    out->iterations = st.iterations;
    out->converged = st.converged;
    out->residual_norm = st.residual_norm;
    out->have_solution = (st.flags & PK_FLAG_INVALID_RHS) ? 0 : 1;
    if (out->have_solution) return download_real_any(s, s->px, x, 3 * static_cast<size_t>(n));
    return PK_OK;
}

}  // extern "C"
