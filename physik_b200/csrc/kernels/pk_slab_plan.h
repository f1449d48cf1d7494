// pk_slab_plan.h -- host-side layout of the part-resident ("slab") PCG kernel.
//
// The rows of the solve are split into parts, one per block of the cooperative launch
// (one block per SM), by recursive coordinate bisection of the rows' node positions.  A
// part owns a set of rows, consecutive in "slab order": parts in order; inside a part
// first the interior rows (whose blocks all lie in the part), then the others, each in
// ascending dynamic-row order.  Its window is its own rows followed by its halo (the
// rows of other parts its rows couple to).  The search direction of the whole window
// lives in shared memory for the whole solve, so the SpMV gathers only from shared memory.
//
// The matrix is stored once more, per part, as a stream of tiles of at most kSlabRows
// consecutive owned rows.  A row holds every block of its full symmetric row -- the
// stored upper blocks (r, c) and the transposes of the lower ones (c, r) -- so no block is
// fetched by another row.  A tile is one contiguous run of bytes that one TMA bulk copy
// moves into a ring stage:
//     [kSlabHeaderBytes: u16 row offsets, rows + 1 used; u16 word kSlabHaloWord: 1 when a
//      block of the tile has its column in the halo]
//     [entries x 9 floats: the blocks, column-major]
//     [entries x u16: window index of each block's column]
// with the entry count padded to a multiple of 8 so both arrays start on 16-byte
// boundaries.  fill_src names, for every entry of every tile in stream order, the
// canonical upper block it copies (kSlabLowerBit: its transpose; kSlabNoPos: padding);
// after assembly a fill kernel writes each tile's blocks in stream order from it.
//
// Plain C++ (no CUDA), shared by the runtime and its CPU self-check.
#pragma once

#include <cstddef>
#include <string>
#include <vector>

namespace pk {

// Tiles are large (about 19 KB for rows of 15 blocks): on B200 a bulk copy's throughput
// per SM grows with its size (measured: ~3.1 TB/s over all SMs with 9 KB copies, ~5.3
// TB/s with 16 KB, ~5.8 TB/s with 32 KB), not with the number of copies in flight.
constexpr int kSlabRows = 32;          // rows per tile
constexpr int kSlabLanesPerRow = 4;    // consumer lanes per row (32 rows per 128-thread group)
constexpr int kSlabHeaderBytes = 80;   // u16 row offsets of a tile (rows + 1 used)
constexpr int kSlabEntryBytes = 38;    // 9 floats + u16 column
constexpr int kSlabCapE = 512;         // entries per tile
constexpr int kSlabStageBytes = 19584; // >= kSlabHeaderBytes + kSlabCapE * kSlabEntryBytes, 128-byte multiple
constexpr int kSlabStages = 6;         // multiple of the consumer groups
constexpr int kSlabWinCap = 6144;      // window rows (owned + halo) per part
constexpr int kSlabMaxTiles = 128;     // tiles per part
constexpr int kSlabRowThreads = 384;   // threads owning rows in the per-row phases
constexpr int kSlabRowsPerThread = 10; // row records per thread in tensor memory
constexpr int kSlabMaxRows = kSlabRowThreads * kSlabRowsPerThread;  // rows per part
// Per part: row0, rows, halo0, halo rows, tile0, tiles, and for per-body solves the part's
// group (its body's parts, consecutive blocks of one launch): first block (within the
// launch) and size; a single group of all parts for the coupled solve.
constexpr int kSlabPartInts = 8;
constexpr unsigned kSlabNoPos = 0xffffffffu;   // a padding entry
constexpr unsigned kSlabLowerBit = 0x80000000u; // the entry is the transpose of the block

// The symmetric ("sym") form of the stream streams each in-part block once.  Every part is
// cut into kSlabGroups sub-parts, one per consumer group, each ordered as a sweep along its
// longest extent.  Inside a sub-part a coupled pair (r, c) with r before c is stored once,
// in row r, as a "transposing" entry: its block B adds B d_c to q_r and B^T d_r to q_c.
// The B^T d_r products go to the group's ring of kSymRingSlots 3-float slots in shared
// memory, at slots fixed by the layout: row c's slots are [lbase(c), lbase(c + 1)) (mod
// the ring), one per earlier coupled row of its sub-part, in sweep order, and row c's q is
// its own entries' sum plus its slots' sum, in that fixed order.  Pairs across sub-parts or
// parts are stored in both rows, as in the full form.  A tile is
//     [kSymHeaderBytes: u16 row offsets (rows + 1), u16 ring bases (rows + 1)]
//     [entries x 9 floats] [entries x u16 window column] [entries x u16 ring slot]
// (slot kSymNoSlot: a plain entry).  A group handles only its own sub-part's tiles,
// strictly in order, so its slots need no synchronisation beyond its own barriers; the
// layout checks that the slots alive at any time (the current tile's rows and every later
// row some processed row already wrote to) fit the ring, else it does not apply.
constexpr int kSlabGroups = 3;          // consumer groups (one sub-part each)
constexpr int kSymRows = 64;            // rows per tile (two passes of 32)
constexpr int kSymHeaderBytes = 272;    // 2 x u16[kSymRows + 1], padded to 16 bytes
constexpr int kSymEntryBytes = 40;      // 9 floats + u16 column + u16 slot
constexpr int kSymStageBytes = 17408;   // 128-byte multiple
constexpr int kSymCapE = (kSymStageBytes - kSymHeaderBytes) / kSymEntryBytes / 8 * 8;
constexpr int kSymRingSlots = 1024;     // per group, a power of two
constexpr unsigned kSymNoSlot = 0xffffu;

static_assert(kSlabHeaderBytes + kSlabCapE * kSlabEntryBytes <= kSlabStageBytes, "stage too small");
static_assert(kSymHeaderBytes >= 4 * (kSymRows + 1) && kSymHeaderBytes % 16 == 0, "sym header");
static_assert(kSymHeaderBytes + kSymCapE * kSymEntryBytes <= kSymStageBytes, "sym stage too small");
static_assert((kSymRingSlots & (kSymRingSlots - 1)) == 0 && kSymRingSlots <= 65535, "ring slots");
static_assert(kSlabCapE % 8 == 0, "entry cap must keep 16-byte alignment");
static_assert(kSlabHeaderBytes % 16 == 0, "blocks must start on a 16-byte boundary");
static_assert(2 * (kSlabRows + 1) <= kSlabHeaderBytes, "header too small");
// Inside a part the rows whose blocks all lie in the part ("interior" rows) come first, so
// a part's first tiles need no halo: the kernel streams them while the halo of the window
// is still being filled, and waits for it only at the first tile whose header word
// kSlabHaloWord is set.
constexpr int kSlabHaloWord = kSlabHeaderBytes / 2 - 1;
static_assert(kSlabHaloWord >= kSlabRows + 1, "the halo word must not overlap the row offsets");

struct SlabPlan {
    int n = 0;
    int parts = 0;
    std::vector<int> perm;       // slab index -> dynamic row
    std::vector<int> part_info;  // kSlabPartInts per part
    std::vector<int> halo_src;   // slab index of every halo row, part by part
    std::vector<int> tile_desc;  // 4 per tile: stream offset / 16, bytes, first local row, rows
    std::vector<unsigned char> stream;  // headers and columns filled, blocks zero
    std::vector<unsigned> fill_src;  // per entry, tile by tile: upper block | kSlabLowerBit, or kSlabNoPos
    std::vector<int> tile_entry0;    // per tile + 1: the tile's first fill_src index
    std::vector<int> part_body;  // body (segment) of each part; 0 for the coupled solve
    std::vector<int> launch_start;  // parts [launch_start[l], launch_start[l + 1]) form launch l
    int max_window = 0, max_tiles = 0, max_rows = 0;
    bool sym = false;  // the symmetric form (tiles and headers as described above)
};

// Which stream form a layout build uses: the full symmetric rows, the symmetric form, or
// the symmetric form where it applies and the full rows otherwise.
enum SlabForm { kSlabFull = 0, kSlabSym = 1, kSlabAuto = 2 };

// Builds the layout for `parts` parts of the upper-stored pattern (row_start, col) with
// its transpose index (lt_start, lt_row, lt_block).  coords: 3 doubles per row (NULL:
// contiguous parts of the dynamic-row order).  Returns "" on success, otherwise why the
// layout does not apply (a window or a row too large); `out` is then unusable.
std::string build_slab_plan(int n, const int* row_start, const int* col, const int* lt_start, const int* lt_row,
                            const int* lt_block, const double* coords, int parts, SlabPlan& out,
                            int form = kSlabAuto);

// The layout for per-body solves: the rows split into bodies (segments
// [seg[b], seg[b + 1]), no block coupling two bodies), every body cut by coordinate
// bisection (NULL coords: contiguous ranges) into as few parts as its rows and window
// allow, and the bodies packed, largest parts first, into "launches" of at most
// max_blocks parts (launch_start), which the runtime runs as the rounds of one persistent
// launch.  Returns "" on success, otherwise why the layout does not apply.
std::string build_slab_plan_batched(int n, const int* row_start, const int* col, const int* lt_start,
                                    const int* lt_row, const int* lt_block, const double* coords, const int* seg,
                                    int nseg, int max_blocks, SlabPlan& out, int form = kSlabAuto);

// y = A x through the plan exactly as the kernel reads it (fill, then tile decoding with
// the kernel's clamps), in double: the CPU self-check of a plan.
void slab_spmv_host(const SlabPlan& plan, int nnz, const double* values, const double* x, double* y);

// The full form's halo order, checked on the host: inside every part the interior rows
// (every block's column in the part) precede the others, and a tile's header flags a halo
// column exactly when one of its blocks has its column in the halo.  "" when it holds.
std::string slab_check_halo_order(const SlabPlan& plan, const int* row_start, const int* col, const int* lt_start,
                                  const int* lt_row);

}  // namespace pk
