// pk_slab_plan.cpp -- builds the part-resident PCG kernel's layout (see pk_slab_plan.h).
#include "pk_slab_plan.h"

#include <algorithm>
#include <cstdlib>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <thread>

namespace pk {
namespace {

// The bisection weight of a row: its streamed blocks plus this per-row share.  A part's
// streaming time follows its row count (its tiles hold at most kSlabRows rows, and rows
// fill a tile before its bytes do) more than its blocks, so the per-row share dominates:
// on block128 a share of 1000 (parts of equal rows) measured 1.5 % faster per solve than 4
// (parts of equal blocks + 4 per row).  PK_SLAB_ROW_WEIGHT overrides it.
double row_weight_extra()
{
    if (const char* e = std::getenv("PK_SLAB_ROW_WEIGHT")) {
        const double v = std::atof(e);
        if (v >= 0.0 && v < 1e6) return v;
    }
    return 1000.0;
}

// Host threads for the layout build (at most 16; 1 when none can be started).
int plan_threads()
{
    const unsigned hw = std::thread::hardware_concurrency();
    return static_cast<int>(std::max(1u, std::min(16u, hw)));
}

// f(i, thread) for i in [0, count) on up to plan_threads() threads, items handed out in
// order; each item must write only its own outputs, so the result does not depend on the
// thread count.  Falls back to one thread if a thread cannot be started.
template <class F>
void parallel_items(int count, F&& f)
{
    const int nt = std::min(count, plan_threads());
    if (nt <= 1) {
        for (int i = 0; i < count; ++i) f(i, 0);
        return;
    }
    std::atomic<int> next{0};
    auto work = [&](int t) {
        for (int i; (i = next.fetch_add(1)) < count;) f(i, t);
    };
    std::vector<std::thread> pool;
    try {
        for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
    } catch (...) {
    }
    work(0);
    for (std::thread& th : pool) th.join();
}

// Recursive coordinate bisection of ids[lo, hi) into `nparts` parts numbered from part0:
// split across the widest axis of the bounding box at the weighted position that gives
// the two halves weight in proportion to their part counts.  Ties break by row id, so
// the result depends only on the inputs.
void rcb(std::vector<int>& ids, size_t lo, size_t hi, int part0, int nparts, const double* xyz,
         const std::vector<double>& w, std::vector<int>& part_of, int depth = 0)
{
    if (nparts <= 1 || hi - lo <= 1) {
        for (size_t i = lo; i < hi; ++i) part_of[ids[i]] = part0;
        return;
    }
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (size_t i = lo; i < hi; ++i)
        for (int a = 0; a < 3; ++a) {
            mn[a] = std::min(mn[a], xyz[3 * (size_t)ids[i] + a]);
            mx[a] = std::max(mx[a], xyz[3 * (size_t)ids[i] + a]);
        }
    int ax = 0;
    for (int a = 1; a < 3; ++a)
        if (mx[a] - mn[a] > mx[ax] - mn[ax]) ax = a;
    std::sort(ids.begin() + lo, ids.begin() + hi, [&](int a, int b) {
        const double ca = xyz[3 * (size_t)a + ax], cb = xyz[3 * (size_t)b + ax];
        return ca < cb || (ca == cb && a < b);
    });
    const int left = nparts / 2;
    double total = 0.0;
    for (size_t i = lo; i < hi; ++i) total += w[ids[i]];
    const double target = total * left / nparts;
    size_t cut = lo;
    double acc = 0.0;
    while (cut < hi && acc + 0.5 * w[ids[cut]] < target) acc += w[ids[cut++]];
    // keep at least one row per part on each side when possible
    const size_t rows = hi - lo;
    if (rows >= (size_t)nparts) {
        cut = std::max(cut, lo + (size_t)left);
        cut = std::min(cut, hi - (size_t)(nparts - left));
    }
    // The two halves touch disjoint ids: the first levels of large cuts run them on two
    // threads (same result).
    if (depth < 4 && hi - lo >= 65536 && plan_threads() > 1) {
        bool threaded = false;
        std::thread first;
        try {
            first = std::thread([&] { rcb(ids, lo, cut, part0, left, xyz, w, part_of, depth + 1); });
            threaded = true;
        } catch (...) {
        }
        if (!threaded) rcb(ids, lo, cut, part0, left, xyz, w, part_of, depth + 1);
        rcb(ids, cut, hi, part0 + left, nparts - left, xyz, w, part_of, depth + 1);
        if (threaded) first.join();
        return;
    }
    rcb(ids, lo, cut, part0, left, xyz, w, part_of, depth + 1);
    rcb(ids, cut, hi, part0 + left, nparts - left, xyz, w, part_of, depth + 1);
}

inline void put_u16(std::vector<unsigned char>& s, size_t off, unsigned v)
{
    const uint16_t x = static_cast<uint16_t>(v);
    std::memcpy(s.data() + off, &x, 2);
}
inline unsigned get_u16(const std::vector<unsigned char>& s, size_t off)
{
    uint16_t x;
    std::memcpy(&x, s.data() + off, 2);
    return x;
}

}  // namespace

namespace {

// The layout for a given assignment of rows to parts (part_of[r] in [0, parts), every part
// non-empty): slab order, windows, halos, tiles, stream and the fill list.  Group fields
// of part_info are left for the caller.
//
// Pass 1 (serial) cuts every part's rows into tiles from the rows' block counts alone,
// which fixes every tile's place in the stream and in the fill list; pass 2 builds the
// parts' halos, windows and tile contents in parallel, each part writing only its own
// tiles; pass 3 joins the halos in part order and checks that every block was placed
// once (and its transpose once, off the diagonal).
std::string build_layout(int n, const int* row_start, const int* col, const int* lt_start, const int* lt_row,
                         const int* lt_block, const std::vector<int>& part_of, const std::vector<int>& len, int parts,
                         SlabPlan& out)
{
    const int nnz = row_start[n];
    // slab order: parts in order; inside a part the interior rows (every block's column in
    // the part), then the others, each ascending
    std::vector<int> count(parts + 1, 0);
    for (int r = 0; r < n; ++r) ++count[part_of[r] + 1];
    for (int p = 0; p < parts; ++p) count[p + 1] += count[p];
    for (int p = 0; p < parts; ++p)
        if (count[p + 1] == count[p]) return "a part has no rows";
    out.perm.assign(n, 0);
    std::vector<int> inv(n);
    {
        std::vector<unsigned char> interior(n, 1);
        for (int r = 0; r < n; ++r) {
            for (int k = row_start[r]; k < row_start[r + 1] && interior[r]; ++k)
                if (part_of[col[k]] != part_of[r]) interior[r] = 0;
            for (int e = lt_start[r]; e < lt_start[r + 1] && interior[r]; ++e)
                if (part_of[lt_row[e]] != part_of[r]) interior[r] = 0;
        }
        std::vector<int> fill(count.begin(), count.end() - 1);
        for (int pass = 1; pass >= 0; --pass)
            for (int r = 0; r < n; ++r) {
                if (interior[r] != pass) continue;
                const int g = fill[part_of[r]]++;
                out.perm[g] = r;
                inv[r] = g;
            }
    }
    out.n = n;
    out.parts = parts;
    out.part_info.assign((size_t)kSlabPartInts * parts, 0);
    out.fill_src.clear();
    out.tile_entry0.clear();
    out.tile_desc.clear();
    out.halo_src.clear();

    // Pass 1: tiles of consecutive owned rows, at most kSlabRows rows and kSlabCapE
    // entries (padded to a multiple of 8 so the arrays stay 16-byte aligned).
    std::vector<int> part_tile0(parts + 1, 0);
    size_t stream_bytes = 0, entries = 0;
    for (int p = 0; p < parts; ++p) {
        const int g0 = count[p], m = count[p + 1] - g0;
        if (m > kSlabMaxRows) return "a part has more rows than tensor memory holds";
        part_tile0[p] = static_cast<int>(out.tile_desc.size() / 4);
        int a = 0;
        while (a < m) {
            int b = a, e = 0;
            while (b < m && b - a < kSlabRows) {
                const int e2 = e + len[out.perm[g0 + b]];
                if (((e2 + 7) & ~7) > kSlabCapE) break;
                e = e2;
                ++b;
            }
            if (b == a) return "a row has more blocks than a tile holds";
            const int ne = (e + 7) & ~7;
            const size_t bytes = (size_t)kSlabHeaderBytes + (size_t)kSlabEntryBytes * ne;
            if (stream_bytes / 16 > 0x7fffffffULL || (stream_bytes + bytes) / 4 >= 0xffffffffULL)
                return "stream too large";
            out.tile_desc.insert(out.tile_desc.end(),
                                 {static_cast<int>(stream_bytes / 16), static_cast<int>(bytes), a, b - a});
            out.tile_entry0.push_back(static_cast<int>(entries));
            stream_bytes += bytes;  // bytes is a multiple of 16 (ne is a multiple of 8)
            entries += ne;
            if (entries > 0x7fffffffu) return "stream too large";
            a = b;
        }
        if (static_cast<int>(out.tile_desc.size() / 4) - part_tile0[p] > kSlabMaxTiles)
            return "a part has more tiles than the table holds";
    }
    part_tile0[parts] = static_cast<int>(out.tile_desc.size() / 4);
    out.tile_entry0.push_back(static_cast<int>(entries));
    out.stream.assign(stream_bytes, 0);
    out.fill_src.assign(entries, kSlabNoPos);

    // Pass 2: per part, its halo (rows of other parts its rows couple to, ascending slab
    // index), window indices, and its tiles' row offsets, blocks (upper copies and lower
    // transposes, by window index) and columns.
    struct Entry {
        int win;     // window index of the column
        int block;   // canonical upper block
        bool lower;  // transpose of that block
    };
    const int nt = std::min(parts, plan_threads());
    std::vector<std::vector<int>> win_of(nt);
    std::vector<std::vector<int>> halos(parts);
    std::vector<const char*> errors(parts, nullptr);
    auto build_part = [&](int p, int t) {
        std::vector<int>& wo = win_of[t];
        if (wo.empty()) wo.assign(n, -1);
        const int g0 = count[p], g1 = count[p + 1], m = g1 - g0;
        for (int g = g0; g < g1; ++g) wo[out.perm[g]] = g - g0;
        std::vector<int>& halo = halos[p];
        for (int g = g0; g < g1; ++g) {
            const int r = out.perm[g];
            for (int k = row_start[r]; k < row_start[r + 1]; ++k)
                if (part_of[col[k]] != p) halo.push_back(inv[col[k]]);
            for (int e = lt_start[r]; e < lt_start[r + 1]; ++e)
                if (part_of[lt_row[e]] != p) halo.push_back(inv[lt_row[e]]);
        }
        std::sort(halo.begin(), halo.end());
        halo.erase(std::unique(halo.begin(), halo.end()), halo.end());
        const int h = static_cast<int>(halo.size());
        if (m + h > kSlabWinCap) {
            errors[p] = "a part's window exceeds shared memory";
            for (int g = g0; g < g1; ++g) wo[out.perm[g]] = -1;
            return;
        }
        for (int i = 0; i < h; ++i) wo[out.perm[halo[i]]] = m + i;
        std::vector<Entry> row_entries;
        for (int ti = part_tile0[p]; ti < part_tile0[p + 1]; ++ti) {
            const int* d = out.tile_desc.data() + 4 * (size_t)ti;
            const size_t off = 16 * (size_t)d[0];
            const int a = d[2], b = d[2] + d[3];
            const int ne = out.tile_entry0[ti + 1] - out.tile_entry0[ti];
            const size_t vals_off = off + kSlabHeaderBytes;
            const size_t col_off = vals_off + 36 * (size_t)ne;
            unsigned* src = out.fill_src.data() + out.tile_entry0[ti];
            int j = 0;
            for (int i = a; i < b; ++i) {
                const int r = out.perm[g0 + i];
                put_u16(out.stream, off + 2 * (size_t)(i - a), (unsigned)j);
                row_entries.clear();
                for (int k = row_start[r]; k < row_start[r + 1]; ++k) row_entries.push_back({wo[col[k]], k, false});
                for (int e = lt_start[r]; e < lt_start[r + 1]; ++e)
                    row_entries.push_back({wo[lt_row[e]], lt_block[e], true});
                std::sort(row_entries.begin(), row_entries.end(),
                          [](const Entry& x, const Entry& y) { return x.win < y.win; });
                for (const Entry& en : row_entries) {
                    src[j] = static_cast<unsigned>(en.block) | (en.lower ? kSlabLowerBit : 0u);
                    put_u16(out.stream, col_off + 2 * (size_t)j, (unsigned)en.win);
                    if (en.win >= m) put_u16(out.stream, off + 2 * (size_t)kSlabHaloWord, 1u);
                    ++j;
                }
            }
            put_u16(out.stream, off + 2 * (size_t)(b - a), (unsigned)j);
        }
        for (int g = g0; g < g1; ++g) wo[out.perm[g]] = -1;
        for (int i = 0; i < h; ++i) wo[out.perm[halo[i]]] = -1;
    };
    parallel_items(parts, [&](int p, int t) {
        try {
            build_part(p, t);
        } catch (...) {  // nothing may leave a worker thread
            errors[p] = "host memory exhausted while building the layout";
        }
    });
    for (int p = 0; p < parts; ++p)
        if (errors[p]) return errors[p];

    // Pass 3: halos in part order, part descriptors, and every block placed once.
    for (int p = 0; p < parts; ++p) {
        const int g0 = count[p], m = count[p + 1] - g0, h = static_cast<int>(halos[p].size());
        int* pi = out.part_info.data() + (size_t)kSlabPartInts * p;
        pi[0] = g0;
        pi[1] = m;
        pi[2] = static_cast<int>(out.halo_src.size());
        pi[3] = h;
        pi[4] = part_tile0[p];
        pi[5] = part_tile0[p + 1] - part_tile0[p];
        out.halo_src.insert(out.halo_src.end(), halos[p].begin(), halos[p].end());
        out.max_window = std::max(out.max_window, m + h);
        out.max_tiles = std::max(out.max_tiles, pi[5]);
        out.max_rows = std::max(out.max_rows, m);
    }
    std::vector<unsigned char> seen(nnz, 0);  // bit 0: copy placed, bit 1: transpose placed
    for (const unsigned src : out.fill_src) {
        if (src == kSlabNoPos) continue;
        const unsigned k = src & ~kSlabLowerBit;
        const unsigned char bit = (src & kSlabLowerBit) ? 2 : 1;
        if (k >= (unsigned)nnz || (seen[k] & bit)) return "internal: a block placed twice";
        seen[k] |= bit;
    }
    for (int k = 0; k < nnz; ++k)
        if (!(seen[k] & 1)) return "internal: block without a copy";
    for (int r = 0; r < n; ++r)
        for (int k = row_start[r]; k < row_start[r + 1]; ++k)
            if ((col[k] != r) != ((seen[k] & 2) != 0)) return "internal: transposed copy mismatch";
    return "";
}


// ---------------------------------------------------------------- the symmetric form
// Typical spacing of the rows along each axis: coupled rows differ along an axis either
// by about one spacing or (for pairs in one plane across that axis) only by the mesh's
// irregularity, so the spacing is the median of the differences above half the median.
// A sweep ranks rows by their coordinates in units of these spacings, rounded, so rows of
// one plane of a jittered grid share a rank.  1 along an axis with no spread.
void axis_spacing(int n, const int* row_start, const int* col, const double* coords, double* sp)
{
    for (int a = 0; a < 3; ++a) {
        std::vector<double> d;
        const int stride = std::max(1, n / 50000);  // every block of a sample of rows is enough
        for (int r = 0; r < n; r += stride)
            for (int k = row_start[r]; k < row_start[r + 1]; ++k)
                if (col[k] != r) d.push_back(std::fabs(coords[3 * (size_t)col[k] + a] - coords[3 * (size_t)r + a]));
        sp[a] = 1.0;
        if (d.empty()) continue;
        std::sort(d.begin(), d.end());
        const double half = 0.5 * d[d.size() / 2];
        auto it = std::upper_bound(d.begin(), d.end(), half);
        if (it == d.end() || !(*it > 0.0)) continue;
        sp[a] = *(it + (d.end() - it) / 2);
    }
}

// Sub-parts and sweep order of one part: its rows cut into `nsub` sub-parts by coordinate
// bisection (NULL coords: contiguous ranges of equal weight), each ordered along the
// longest extent of its bounding box, then the next, in units of the axis spacings (ties
// by row).  Returns the part's rows in local order; sub_start[k] is the first local index
// of sub-part k (sub_start[nsub] = rows).
std::vector<int> sym_local_order(const std::vector<int>& rows, const double* coords, const double* sp,
                                 const std::vector<double>& w, int nsub, std::vector<int>& sub_start)
{
    const int m = static_cast<int>(rows.size());
    std::vector<int> sub(m, 0);
    const int ns = std::min(nsub, m);
    if (ns > 1) {
        if (coords) {
            std::vector<int> ids(m);
            std::iota(ids.begin(), ids.end(), 0);
            std::vector<double> xyz(3 * (size_t)m), wl(m);
            for (int i = 0; i < m; ++i) {
                for (int a = 0; a < 3; ++a) xyz[3 * (size_t)i + a] = coords[3 * (size_t)rows[i] + a];
                wl[i] = w[rows[i]];
            }
            rcb(ids, 0, (size_t)m, 0, ns, xyz.data(), wl, sub, 8);  // depth 8: never threaded
        } else {
            double total = 0.0, acc = 0.0;
            for (int i = 0; i < m; ++i) total += w[rows[i]];
            for (int i = 0; i < m; ++i) {
                sub[i] = std::min(ns - 1, static_cast<int>(acc * ns / total));
                acc += w[rows[i]];
            }
        }
    }
    std::vector<int> order;
    order.reserve(m);
    sub_start.assign(nsub + 1, 0);
    for (int k = 0; k < nsub; ++k) {
        std::vector<int> mine;
        for (int i = 0; i < m; ++i)
            if (sub[i] == k) mine.push_back(rows[i]);
        if (coords && mine.size() > 1) {
            double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
            for (int r : mine)
                for (int a = 0; a < 3; ++a) {
                    mn[a] = std::min(mn[a], coords[3 * (size_t)r + a]);
                    mx[a] = std::max(mx[a], coords[3 * (size_t)r + a]);
                }
            int ax[3] = {0, 1, 2};
            std::sort(ax, ax + 3, [&](int a, int b) {
                const double ea = (mx[a] - mn[a]) / sp[a], eb = (mx[b] - mn[b]) / sp[b];
                return ea > eb || (ea == eb && a < b);
            });
            std::vector<std::pair<std::array<long long, 3>, int>> key(mine.size());
            for (size_t i = 0; i < mine.size(); ++i) {
                for (int j = 0; j < 3; ++j)
                    key[i].first[j] = std::llround((coords[3 * (size_t)mine[i] + ax[j]] - mn[ax[j]]) / sp[ax[j]]);
                key[i].second = mine[i];
            }
            std::sort(key.begin(), key.end());
            for (size_t i = 0; i < mine.size(); ++i) mine[i] = key[i].second;
        }
        order.insert(order.end(), mine.begin(), mine.end());
        sub_start[k + 1] = static_cast<int>(order.size());
    }
    return order;
}

// One tile of the symmetric form while it is built: its rows (local indices), their
// entries and ring bases.
struct SymTile {
    int first = 0, rows = 0, ne = 0;     // ne padded to a multiple of 8
    std::vector<unsigned short> roff;    // rows + 1
    std::vector<unsigned short> lbase;   // rows + 1 (mod the ring)
    std::vector<unsigned short> wcol, slot;
    std::vector<unsigned> src;
};

// The tiles of one part in the symmetric form, group by group.  loc_of[c]: local index of
// row c if it is in this part, else -1; win(c): window index of row c (any increasing
// stand-in while only the fit is tested: entries are sorted by it, counts do not depend
// on it).  Sub-part s belongs to group s / (subs / kSlabGroups), its rows are local indices
// [sub_start[s], sub_start[s + 1]).  Returns "" or why the form does not fit.
template <class Win>
std::string sym_part_tiles(const int* row_start, const int* col, const int* lt_start, const int* lt_row,
                           const int* lt_block, const std::vector<int>& order, const std::vector<int>& sub_start,
                           const std::vector<int>& loc_of, Win&& win, std::vector<SymTile> (&tiles)[kSlabGroups])
{
    const int subs = static_cast<int>(sub_start.size()) - 1;
    const int per_group = subs / kSlabGroups;
    std::vector<int> sub_of_local(order.size());
    for (int sb = 0; sb < subs; ++sb)
        for (int i = sub_start[sb]; i < sub_start[sb + 1]; ++i) sub_of_local[i] = sb;
    struct Ent {
        int win;
        unsigned src;
        int target;  // local index of the row a transposing entry also feeds, or -1
    };
    for (int g = 0; g < kSlabGroups; ++g) {
        tiles[g].clear();
        // the group's rows: its sub-parts one after the other
        const int a0 = sub_start[g * per_group], a1 = sub_start[(g + 1) * per_group], ms = a1 - a0;
        if (ms <= 0) continue;
        std::vector<std::vector<Ent>> ents(ms);
        std::vector<std::vector<int>> lower(ms);
        for (int i = a0; i < a1; ++i) {
            const int r = order[i];
            auto add = [&](int c, unsigned src) {
                const int lc = loc_of[c];
                const bool inside = lc >= 0 && sub_of_local[lc] == sub_of_local[i];
                if (!inside || lc == i) {
                    ents[i - a0].push_back({win(c), src, -1});
                } else if (lc > i) {
                    ents[i - a0].push_back({win(c), src, lc});
                    lower[lc - a0].push_back(i);
                }
            };
            for (int kk = row_start[r]; kk < row_start[r + 1]; ++kk) add(col[kk], static_cast<unsigned>(kk));
            for (int e = lt_start[r]; e < lt_start[r + 1]; ++e)
                add(lt_row[e], static_cast<unsigned>(lt_block[e]) | kSlabLowerBit);
            std::sort(ents[i - a0].begin(), ents[i - a0].end(), [](const Ent& x, const Ent& y) { return x.win < y.win; });
        }
        std::vector<long long> L(ms + 1, 0);  // ring bases, not yet reduced mod the ring
        for (int j = 0; j < ms; ++j) {
            std::sort(lower[j].begin(), lower[j].end());
            L[j + 1] = L[j] + static_cast<long long>(lower[j].size());
        }
        // tiles: consecutive rows, at most kSymRows rows and kSymCapE entries
        int a = 0;
        long long maxtgt = -1;  // furthest row a processed row wrote to
        while (a < ms) {
            int b = a, e = 0;
            while (b < ms && b - a < kSymRows) {
                const int e2 = e + static_cast<int>(ents[b].size());
                if (((e2 + 7) & ~7) > kSymCapE) break;
                e = e2;
                ++b;
            }
            if (b == a) return "a row has more blocks than a tile holds";
            SymTile tl;
            tl.first = a0 + a;
            tl.rows = b - a;
            tl.ne = (e + 7) & ~7;
            tl.roff.resize(tl.rows + 1);
            tl.lbase.resize(tl.rows + 1);
            tl.wcol.assign(tl.ne, 0);
            tl.slot.assign(tl.ne, static_cast<unsigned short>(kSymNoSlot));
            tl.src.assign(tl.ne, kSlabNoPos);
            int j = 0;
            for (int i = a; i < b; ++i) {
                tl.roff[i - a] = static_cast<unsigned short>(j);
                tl.lbase[i - a] = static_cast<unsigned short>(L[i] & (kSymRingSlots - 1));
                for (const Ent& en : ents[i]) {
                    tl.wcol[j] = static_cast<unsigned short>(en.win);
                    tl.src[j] = en.src;
                    if (en.target >= 0) {
                        const int tj = en.target - a0;
                        const std::vector<int>& lw = lower[tj];
                        const long long rank = std::lower_bound(lw.begin(), lw.end(), a0 + i) - lw.begin();
                        tl.slot[j] = static_cast<unsigned short>((L[tj] + rank) & (kSymRingSlots - 1));
                        maxtgt = std::max<long long>(maxtgt, tj);
                    }
                    ++j;
                }
            }
            tl.roff[b - a] = static_cast<unsigned short>(j);
            tl.lbase[b - a] = static_cast<unsigned short>(L[b] & (kSymRingSlots - 1));
            // alive while this tile runs: its own rows' slots and every later row's slots
            // that a processed row has written
            const long long last = std::max<long long>(maxtgt, b - 1);
            if (L[last + 1] - L[a] > kSymRingSlots)
                return "the transposed products in flight exceed the ring (" + std::to_string(L[last + 1] - L[a]) +
                       " slots)";
            tiles[g].push_back(std::move(tl));
            a = b;
        }
    }
    size_t most = 0;
    for (int g = 0; g < kSlabGroups; ++g) most = std::max(most, tiles[g].size());
    if (kSlabGroups * most > (size_t)kSlabMaxTiles) return "a part has more tiles than the table holds";
    return "";
}

// The symmetric-form layout for a given assignment of rows to parts: local orders
// (sub-parts, sweeps), windows, halos, tiles in ring order (group g at positions g, g + 3,
// ...; empty positions where a group has fewer tiles), stream and fill list.  Every part
// takes the fewest sub-parts per group (1 to 4) whose transposed products fit the rings.
std::string build_layout_sym(int n, const int* row_start, const int* col, const int* lt_start, const int* lt_row,
                             const int* lt_block, const double* coords, const std::vector<int>& part_of,
                             const std::vector<double>& w, int parts, SlabPlan& out)
{
    const int nnz = row_start[n];
    std::vector<int> count(parts + 1, 0);
    for (int r = 0; r < n; ++r) ++count[part_of[r] + 1];
    for (int p = 0; p < parts; ++p) count[p + 1] += count[p];
    for (int p = 0; p < parts; ++p) {
        if (count[p + 1] == count[p]) return "a part has no rows";
        if (count[p + 1] - count[p] > kSlabMaxRows) return "a part has more rows than tensor memory holds";
    }
    std::vector<std::vector<int>> part_rows(parts);
    for (int r = 0; r < n; ++r) part_rows[part_of[r]].push_back(r);
    double sp[3] = {1.0, 1.0, 1.0};
    if (coords) axis_spacing(n, row_start, col, coords, sp);
    const int nt = std::min(parts, plan_threads());
    std::vector<std::vector<int>> loc_of(nt);
    // 1. local orders: the fewest sub-parts per group that fit
    std::vector<std::vector<int>> sub_start(parts);
    out.perm.assign(n, 0);
    std::vector<std::string> errors(parts);
    parallel_items(parts, [&](int p, int t) {
        try {
            std::vector<int>& lo = loc_of[t];
            if (lo.empty()) lo.assign(n, -1);
            std::string why, first_why;
            for (int per = 1; per <= 4; ++per) {
                std::vector<int> ss;
                const std::vector<int> ord = sym_local_order(part_rows[p], coords, sp, w, kSlabGroups * per, ss);
                for (size_t i = 0; i < ord.size(); ++i) lo[ord[i]] = static_cast<int>(i);
                std::vector<SymTile> tiles[kSlabGroups];
                why = sym_part_tiles(row_start, col, lt_start, lt_row, lt_block, ord, ss, lo,
                                     [&](int c) { return lo[c] >= 0 ? lo[c] : n + c; }, tiles);
                for (int r : ord) lo[r] = -1;
                if (why.empty()) {
                    std::copy(ord.begin(), ord.end(), out.perm.begin() + count[p]);
                    sub_start[p] = ss;
                    break;
                }
                if (first_why.empty()) first_why = why;
            }
            errors[p] = why.empty() ? why : first_why;  // the one-sub-part-per-group reason
        } catch (...) {
            errors[p] = "host memory exhausted while building the layout";
        }
    });
    for (int p = 0; p < parts; ++p)
        if (!errors[p].empty()) return errors[p];
    std::vector<int> inv(n);
    for (int g = 0; g < n; ++g) inv[out.perm[g]] = g;
    out.n = n;
    out.parts = parts;
    out.sym = true;
    out.part_info.assign((size_t)kSlabPartInts * parts, 0);
    out.fill_src.clear();
    out.tile_entry0.clear();
    out.tile_desc.clear();
    out.halo_src.clear();

    // 2. per part: halo, window indices and the tiles with their real window columns
    struct PartOut {
        std::vector<int> halo;
        std::vector<SymTile> tiles[kSlabGroups];
    };
    std::vector<PartOut> po(parts);
    std::vector<std::vector<int>> win_of(nt);
    auto build_part = [&](int p, int t) {
        std::vector<int>& wo = win_of[t];
        std::vector<int>& lo = loc_of[t];
        if (wo.empty()) wo.assign(n, -1);
        if (lo.empty()) lo.assign(n, -1);
        const int g0 = count[p], g1 = count[p + 1], m = g1 - g0;
        for (int g = g0; g < g1; ++g) wo[out.perm[g]] = lo[out.perm[g]] = g - g0;
        std::vector<int>& halo = po[p].halo;
        for (int g = g0; g < g1; ++g) {
            const int r = out.perm[g];
            for (int k = row_start[r]; k < row_start[r + 1]; ++k)
                if (part_of[col[k]] != p) halo.push_back(inv[col[k]]);
            for (int e = lt_start[r]; e < lt_start[r + 1]; ++e)
                if (part_of[lt_row[e]] != p) halo.push_back(inv[lt_row[e]]);
        }
        std::sort(halo.begin(), halo.end());
        halo.erase(std::unique(halo.begin(), halo.end()), halo.end());
        const int h = static_cast<int>(halo.size());
        if (m + h <= kSlabWinCap) {
            for (int i = 0; i < h; ++i) wo[out.perm[halo[i]]] = m + i;
            const std::vector<int> ord(out.perm.begin() + g0, out.perm.begin() + g1);
            errors[p] = sym_part_tiles(row_start, col, lt_start, lt_row, lt_block, ord, sub_start[p], lo,
                                       [&](int c) { return wo[c]; }, po[p].tiles);
        } else {
            errors[p] = "a part's window exceeds shared memory";
        }
        for (int g = g0; g < g1; ++g) wo[out.perm[g]] = lo[out.perm[g]] = -1;
        for (int i = 0; i < h; ++i) wo[out.perm[halo[i]]] = -1;
    };
    parallel_items(parts, [&](int p, int t) {
        try {
            build_part(p, t);
        } catch (...) {
            errors[p] = "host memory exhausted while building the layout";
        }
    });
    for (int p = 0; p < parts; ++p)
        if (!errors[p].empty()) return errors[p];

    // 3. stream offsets in part order, positions in ring order (group = position % 3)
    size_t stream_bytes = 0, entries = 0;
    std::vector<size_t> tile_off;  // stream byte offset of every position (empty: unused)
    std::vector<const SymTile*> tile_ptr;
    for (int p = 0; p < parts; ++p) {
        const int m = count[p + 1] - count[p], h = static_cast<int>(po[p].halo.size());
        size_t most = 0;
        for (int k = 0; k < kSlabGroups; ++k) most = std::max(most, po[p].tiles[k].size());
        int* pi = out.part_info.data() + (size_t)kSlabPartInts * p;
        pi[0] = count[p];
        pi[1] = m;
        pi[2] = static_cast<int>(out.halo_src.size());
        pi[3] = h;
        pi[4] = static_cast<int>(out.tile_desc.size() / 4);
        pi[5] = static_cast<int>(kSlabGroups * most);
        out.halo_src.insert(out.halo_src.end(), po[p].halo.begin(), po[p].halo.end());
        out.max_window = std::max(out.max_window, m + h);
        out.max_tiles = std::max(out.max_tiles, pi[5]);
        out.max_rows = std::max(out.max_rows, m);
        for (size_t q = 0; q < most; ++q)
            for (int k = 0; k < kSlabGroups; ++k) {
                out.tile_entry0.push_back(static_cast<int>(entries));
                if (q < po[p].tiles[k].size()) {
                    const SymTile& tl = po[p].tiles[k][q];
                    const size_t bytes = (size_t)kSymHeaderBytes + (size_t)kSymEntryBytes * tl.ne;
                    if (stream_bytes / 16 > 0x7fffffffULL || (stream_bytes + bytes) / 4 >= 0xffffffffULL)
                        return "stream too large";
                    out.tile_desc.insert(out.tile_desc.end(),
                                         {static_cast<int>(stream_bytes / 16), static_cast<int>(bytes), tl.first, tl.rows});
                    tile_off.push_back(stream_bytes);
                    tile_ptr.push_back(&tl);
                    stream_bytes += bytes;  // a multiple of 16 (ne is a multiple of 8)
                    entries += tl.ne;
                    if (entries > 0x7fffffffu) return "stream too large";
                } else {
                    out.tile_desc.insert(out.tile_desc.end(), {0, 0, 0, 0});  // nothing for this group
                    tile_off.push_back(0);
                    tile_ptr.push_back(nullptr);
                }
            }
    }
    out.tile_entry0.push_back(static_cast<int>(entries));
    out.stream.assign(stream_bytes, 0);
    out.fill_src.assign(entries, kSlabNoPos);
    // 4. tile contents (in parallel: every tile writes only its own bytes)
    parallel_items(static_cast<int>(tile_ptr.size()), [&](int ti, int) {
        const SymTile* tl = tile_ptr[ti];
        if (!tl) return;
        const size_t off = tile_off[ti];
        for (int i = 0; i <= tl->rows; ++i) {
            put_u16(out.stream, off + 2 * (size_t)i, tl->roff[i]);
            put_u16(out.stream, off + 2 * (size_t)(kSymRows + 1) + 2 * (size_t)i, tl->lbase[i]);
        }
        const size_t col_off = off + kSymHeaderBytes + 36 * (size_t)tl->ne;
        const size_t slot_off = col_off + 2 * (size_t)tl->ne;
        for (int j = 0; j < tl->ne; ++j) {
            put_u16(out.stream, col_off + 2 * (size_t)j, tl->wcol[j]);
            put_u16(out.stream, slot_off + 2 * (size_t)j, tl->slot[j]);
        }
        std::copy(tl->src.begin(), tl->src.end(), out.fill_src.begin() + out.tile_entry0[ti]);
    });
    // 5. every block placed as its pair requires: once for the diagonal and for a pair
    // inside one sub-part (as the block or its transpose), copy and transpose otherwise
    std::vector<int> sub_of(n);
    for (int p = 0; p < parts; ++p)
        for (size_t sb = 0; sb + 1 < sub_start[p].size(); ++sb)
            for (int i = sub_start[p][sb]; i < sub_start[p][sb + 1]; ++i) sub_of[out.perm[count[p] + i]] = (int)sb;
    std::vector<unsigned char> seen(nnz, 0);
    for (const unsigned src : out.fill_src) {
        if (src == kSlabNoPos) continue;
        const unsigned k = src & ~kSlabLowerBit;
        const unsigned char bit = (src & kSlabLowerBit) ? 2 : 1;
        if (k >= (unsigned)nnz || (seen[k] & bit)) return "internal: a block placed twice";
        seen[k] |= bit;
    }
    for (int r = 0; r < n; ++r)
        for (int k = row_start[r]; k < row_start[r + 1]; ++k) {
            const int c = col[k];
            const bool together = part_of[r] == part_of[c] && sub_of[r] == sub_of[c];
            const unsigned char want = c == r ? 1 : (together ? 0 : 3);
            if (want ? seen[k] != want : (seen[k] != 1 && seen[k] != 2)) return "internal: block placement mismatch";
        }
    return "";
}

}  // namespace

// The symmetric form where the caller allows it and it applies, else the full rows.
std::string build_layout_form(int n, const int* row_start, const int* col, const int* lt_start, const int* lt_row,
                              const int* lt_block, const double* coords, const std::vector<int>& part_of,
                              const std::vector<int>& len, const std::vector<double>& w, int parts, int form,
                              SlabPlan& out)
{
    if (form != kSlabFull) {
        const std::string why =
            build_layout_sym(n, row_start, col, lt_start, lt_row, lt_block, coords, part_of, w, parts, out);
        if (why.empty() || form == kSlabSym) return why;
        out = SlabPlan{};
    }
    return build_layout(n, row_start, col, lt_start, lt_row, lt_block, part_of, len, parts, out);
}

std::string build_slab_plan(int n, const int* row_start, const int* col, const int* lt_start, const int* lt_row,
                            const int* lt_block, const double* coords, int parts, SlabPlan& out, int form)
{
    out = SlabPlan{};
    if (n <= 0 || parts <= 0) return "empty system";
    parts = std::min(parts, n);
    std::vector<int> len(n);
    for (int r = 0; r < n; ++r) len[r] = (row_start[r + 1] - row_start[r]) + (lt_start[r + 1] - lt_start[r]);
    for (int r = 0; r < n; ++r)
        if (len[r] > kSlabCapE) return "a row has more blocks than a tile holds";
    std::vector<int> part_of(n, 0);
    std::vector<double> w(n);
    const double extra = row_weight_extra();
    for (int r = 0; r < n; ++r) w[r] = len[r] + extra;  // streamed blocks + per-row work
    if (coords) {
        std::vector<int> ids(n);
        std::iota(ids.begin(), ids.end(), 0);
        rcb(ids, 0, (size_t)n, 0, parts, coords, w, part_of);
    } else {
        const double total = std::accumulate(w.begin(), w.end(), 0.0);
        double acc = 0.0;
        for (int r = 0; r < n; ++r) {
            part_of[r] = std::min(parts - 1, static_cast<int>(acc * parts / total));
            acc += w[r];
        }
    }
    const std::string why =
        build_layout_form(n, row_start, col, lt_start, lt_row, lt_block, coords, part_of, len, w, parts, form, out);
    if (!why.empty()) return why;
    for (int p = 0; p < parts; ++p) {
        out.part_info[(size_t)kSlabPartInts * p + 6] = 0;
        out.part_info[(size_t)kSlabPartInts * p + 7] = parts;
    }
    out.part_body.assign(parts, 0);
    out.launch_start = {0, parts};
    return "";
}

std::string build_slab_plan_batched(int n, const int* row_start, const int* col, const int* lt_start,
                                    const int* lt_row, const int* lt_block, const double* coords, const int* seg,
                                    int nseg, int max_blocks, SlabPlan& out, int form)
{
    out = SlabPlan{};
    if (n <= 0 || nseg <= 0 || max_blocks <= 0) return "empty system";
    if (seg[0] != 0 || seg[nseg] != n) return "segments do not cover the rows";
    std::vector<int> len(n);
    for (int r = 0; r < n; ++r) len[r] = (row_start[r + 1] - row_start[r]) + (lt_start[r + 1] - lt_start[r]);
    for (int r = 0; r < n; ++r)
        if (len[r] > kSlabCapE) return "a row has more blocks than a tile holds";
    std::vector<double> w(n);
    const double extra = row_weight_extra();
    for (int r = 0; r < n; ++r) w[r] = len[r] + extra;
    // 0. the largest part to aim for.  The runtime places the bodies on the launch's blocks
    // before every solve, largest work (duration x parts) first, a body of k parts on the k
    // consecutive blocks free earliest (slab_schedule_kernel); per iteration a body costs about c0 + c1 * its
    // largest part's rows (c1 the streaming, ~12 ns per row on B200; c0 the window pass,
    // phase B and the exchanges: ~8 us for a group of several parts, ~4 us for a body of
    // one part, which exchanges nothing).  That placement is simulated for each candidate
    // cap with every body at the same iteration count, and the cap with the earliest
    // finish wins.
    int cap = kSlabMaxRows;
    {
        double best = 1e300;
        for (int c : {kSlabMaxRows, 3400, 3000, 2800, 2600, 2400, 2200, 2000}) {
            if (c > kSlabMaxRows) continue;
            struct Bp {
                double dur;  // per iteration
                int k;       // parts
            };
            std::vector<Bp> pb;
            bool fits = true;
            for (int b = 0; b < nseg; ++b) {
                const int rows = seg[b + 1] - seg[b];
                if (rows <= 0) continue;
                const int k = (rows + c - 1) / c;
                if (k > max_blocks) fits = false;
                pb.push_back({(k > 1 ? 8.0 : 4.0) + 0.012 * std::ceil(double(rows) / k), k});
            }
            if (!fits) continue;
            std::stable_sort(pb.begin(), pb.end(),
                             [](const Bp& x, const Bp& y) { return x.dur * x.k > y.dur * y.k; });
            std::vector<double> free_at(static_cast<size_t>(max_blocks), 0.0);
            for (const Bp& q : pb) {
                int b0 = 0;
                double start = 1e300;
                for (int b = 0; b + q.k <= max_blocks; ++b) {
                    double st = 0.0;
                    for (int j = b; j < b + q.k; ++j) st = std::max(st, free_at[j]);
                    if (st < start) {
                        start = st;
                        b0 = b;
                    }
                }
                for (int j = b0; j < b0 + q.k; ++j) free_at[j] = start + q.dur;
            }
            const double finish = *std::max_element(free_at.begin(), free_at.end());
            if (finish < best) {
                best = finish;
                cap = c;
            }
        }
    }
    // 1. every body into parts: the fewest of at most `cap` rows whose windows fit
    std::vector<int> body_parts(nseg, 0);
    std::vector<std::vector<int>> body_assign(nseg);  // part (0..k-1) of each of the body's rows
    for (int b = 0; b < nseg; ++b) {
        const int s0 = seg[b], rows = seg[b + 1] - seg[b];
        if (rows <= 0) continue;
        int k = (rows + cap - 1) / cap;
        for (;; ++k) {
            if (k > rows || k > max_blocks) return "a body does not fit one launch";
            std::vector<int> a(rows, 0);
            if (k > 1) {
                if (coords) {
                    std::vector<int> ids(rows);
                    std::iota(ids.begin(), ids.end(), 0);
                    std::vector<double> xyz(3 * (size_t)rows), wb(rows);
                    for (int i = 0; i < rows; ++i) {
                        for (int c = 0; c < 3; ++c) xyz[3 * (size_t)i + c] = coords[3 * (size_t)(s0 + i) + c];
                        wb[i] = w[s0 + i];
                    }
                    rcb(ids, 0, (size_t)rows, 0, k, xyz.data(), wb, a);
                } else {
                    double total = 0.0, acc = 0.0;
                    for (int i = 0; i < rows; ++i) total += w[s0 + i];
                    for (int i = 0; i < rows; ++i) {
                        a[i] = std::min(k - 1, static_cast<int>(acc * k / total));
                        acc += w[s0 + i];
                    }
                }
            }
            // rows and windows of the k parts (rows of one body couple only within it)
            std::vector<int> cnt(k, 0);
            for (int i = 0; i < rows; ++i) ++cnt[a[i]];
            bool ok = true;
            for (int p = 0; p < k && ok; ++p) ok = cnt[p] > 0 && cnt[p] <= kSlabMaxRows;
            if (ok) {
                std::vector<std::vector<int>> halo(k);
                for (int i = 0; i < rows; ++i) {
                    const int r = s0 + i, p = a[i];
                    for (int kk = row_start[r]; kk < row_start[r + 1]; ++kk) {
                        const int c = col[kk];
                        if (c < s0 || c >= seg[b + 1]) return "a block couples two bodies";
                        if (a[c - s0] != p) halo[p].push_back(c);
                    }
                    for (int e = lt_start[r]; e < lt_start[r + 1]; ++e) {
                        const int c = lt_row[e];
                        if (c < s0 || c >= seg[b + 1]) return "a block couples two bodies";
                        if (a[c - s0] != p) halo[p].push_back(c);
                    }
                }
                for (int p = 0; p < k && ok; ++p) {
                    std::sort(halo[p].begin(), halo[p].end());
                    halo[p].erase(std::unique(halo[p].begin(), halo[p].end()), halo[p].end());
                    ok = cnt[p] + static_cast<int>(halo[p].size()) <= kSlabWinCap;
                }
            }
            if (ok) {
                body_parts[b] = k;
                body_assign[b] = std::move(a);
                break;
            }
        }
    }
    // 2. bodies into launches (the rounds of the persistent launch), largest parts first,
    // at most max_blocks parts per launch, a body never split across launches
    std::vector<int> order;
    for (int b = 0; b < nseg; ++b)
        if (body_parts[b] > 0) order.push_back(b);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const double rx = double(seg[x + 1] - seg[x]) / body_parts[x], ry = double(seg[y + 1] - seg[y]) / body_parts[y];
        return rx > ry;
    });
    std::vector<int> launch_of(nseg, -1), launch_fill;
    for (int b : order) {
        int l = 0;
        while (l < static_cast<int>(launch_fill.size()) && launch_fill[l] + body_parts[b] > max_blocks) ++l;
        if (l == static_cast<int>(launch_fill.size())) launch_fill.push_back(0);
        launch_of[b] = l;
        launch_fill[l] += body_parts[b];
    }
    // 3. global part numbers: launch by launch, bodies in that launch in size order
    std::vector<int> part_of(n, 0);
    std::vector<int> part_body, group_first, group_size;
    out.launch_start.assign(1, 0);
    for (int l = 0; l < static_cast<int>(launch_fill.size()); ++l) {
        int local = 0;
        for (int b : order) {
            if (launch_of[b] != l) continue;
            const int first = static_cast<int>(part_body.size());
            for (int i = 0; i < seg[b + 1] - seg[b]; ++i) part_of[seg[b] + i] = first + body_assign[b][i];
            for (int p = 0; p < body_parts[b]; ++p) {
                part_body.push_back(b);
                group_first.push_back(local);
                group_size.push_back(body_parts[b]);
            }
            local += body_parts[b];
        }
        out.launch_start.push_back(static_cast<int>(part_body.size()));
    }
    const int parts = static_cast<int>(part_body.size());
    std::vector<int> launch_start = out.launch_start;
    const std::string why =
        build_layout_form(n, row_start, col, lt_start, lt_row, lt_block, coords, part_of, len, w, parts, form, out);
    if (!why.empty()) return why;
    for (int p = 0; p < parts; ++p) {
        out.part_info[(size_t)kSlabPartInts * p + 6] = group_first[p];
        out.part_info[(size_t)kSlabPartInts * p + 7] = group_size[p];
    }
    out.part_body = part_body;
    out.launch_start = launch_start;
    return "";
}

namespace {

// The symmetric form decoded as the kernel's consumer groups read it: each group's tiles
// in ring order; per tile first every entry's product (transposing entries also writing
// B^T d_r to their ring slot), then every row's q = own sum + its ring slots in order.
// The ring is emulated with its wrap-around, so a slot reused too early shows up here.
void slab_spmv_host_sym(const SlabPlan& plan, const std::vector<unsigned char>& s, const double* x, double* y)
{
    for (int p = 0; p < plan.parts; ++p) {
        const int* pi = plan.part_info.data() + (size_t)kSlabPartInts * p;
        const int g0 = pi[0], m = pi[1], halo0 = pi[2], h = pi[3], tile0 = pi[4], ntiles = pi[5];
        const int wn = m + h;
        std::vector<double> win(3 * (size_t)wn);
        for (int wi = 0; wi < wn; ++wi) {
            const int g = wi < m ? g0 + wi : plan.halo_src[halo0 + wi - m];
            const int r = plan.perm[g];
            for (int a = 0; a < 3; ++a)
                win[3 * (size_t)wi + a] = static_cast<double>(static_cast<float>(x[3 * (size_t)r + a]));
        }
        for (int grp = 0; grp < kSlabGroups; ++grp) {
            std::vector<double> ring(3 * (size_t)kSymRingSlots, std::nan(""));
            for (int t = grp; t < ntiles; t += kSlabGroups) {
                const int* d = plan.tile_desc.data() + 4 * (size_t)(tile0 + t);
                if (d[1] == 0) continue;
                const size_t off = 16 * (size_t)d[0];
                const int ne = (d[1] - kSymHeaderBytes) / kSymEntryBytes;
                const size_t vals_off = off + kSymHeaderBytes, col_off = vals_off + 36 * (size_t)ne,
                             slot_off = col_off + 2 * (size_t)ne;
                const int rows = std::min(d[3], kSymRows);
                std::vector<double> own(3 * (size_t)rows, 0.0);
                for (int i = 0; i < rows; ++i) {
                    const int li = std::min(d[2] + i, std::max(wn - 1, 0));
                    const int e0 = std::min<int>(get_u16(s, off + 2 * (size_t)i), ne);
                    const int e1 = std::min<int>(get_u16(s, off + 2 * (size_t)(i + 1)), ne);
                    for (int j = e0; j < e1; ++j) {
                        const int c = std::min<int>(get_u16(s, col_off + 2 * (size_t)j), wn - 1);
                        const unsigned sl = get_u16(s, slot_off + 2 * (size_t)j);
                        float v[9];
                        std::memcpy(v, s.data() + vals_off + 36 * (size_t)j, 36);
                        for (int a = 0; a < 3; ++a)
                            for (int mm = 0; mm < 3; ++mm) own[3 * (size_t)i + a] += double(v[3 * mm + a]) * win[3 * (size_t)c + mm];
                        if (sl != kSymNoSlot) {
                            const size_t q = 3 * (size_t)(sl & (kSymRingSlots - 1));
                            for (int a = 0; a < 3; ++a) {
                                double acc = 0.0;
                                for (int mm = 0; mm < 3; ++mm) acc += double(v[3 * a + mm]) * win[3 * (size_t)li + mm];
                                ring[q + a] = acc;
                            }
                        }
                    }
                }
                const size_t lb_off = off + 2 * (size_t)(kSymRows + 1);
                for (int i = 0; i < rows; ++i) {
                    const unsigned b0 = get_u16(s, lb_off + 2 * (size_t)i), b1 = get_u16(s, lb_off + 2 * (size_t)(i + 1));
                    const unsigned cnt = (b1 - b0) & (kSymRingSlots - 1);
                    double q[3] = {own[3 * (size_t)i], own[3 * (size_t)i + 1], own[3 * (size_t)i + 2]};
                    for (unsigned k = 0; k < cnt; ++k) {
                        const size_t sl = 3 * (size_t)((b0 + k) & (kSymRingSlots - 1));
                        for (int a = 0; a < 3; ++a) q[a] += ring[sl + a];
                        for (int a = 0; a < 3; ++a) ring[sl + a] = std::nan("");  // consumed
                    }
                    const int r = plan.perm[g0 + d[2] + i];
                    for (int a = 0; a < 3; ++a) y[3 * (size_t)r + a] = q[a];
                }
            }
        }
    }
}

}  // namespace

std::string slab_check_halo_order(const SlabPlan& plan, const int* row_start, const int* col, const int* lt_start,
                                  const int* lt_row)
{
    if (plan.sym) return "";
    const int n = plan.n;
    std::vector<int> part_of_slab(n, -1), inv(n, -1);
    for (int g = 0; g < n; ++g) inv[plan.perm[g]] = g;
    for (int p = 0; p < plan.parts; ++p) {
        const int* pi = plan.part_info.data() + (size_t)kSlabPartInts * p;
        for (int g = pi[0]; g < pi[0] + pi[1]; ++g) part_of_slab[g] = p;
    }
    for (int p = 0; p < plan.parts; ++p) {
        const int* pi = plan.part_info.data() + (size_t)kSlabPartInts * p;
        const int g0 = pi[0], m = pi[1], tile0 = pi[4], ntiles = pi[5];
        bool seen_boundary = false;
        for (int g = g0; g < g0 + m; ++g) {
            const int r = plan.perm[g];
            bool interior = true;
            for (int k = row_start[r]; k < row_start[r + 1] && interior; ++k) interior = part_of_slab[inv[col[k]]] == p;
            for (int e = lt_start[r]; e < lt_start[r + 1] && interior; ++e)
                interior = part_of_slab[inv[lt_row[e]]] == p;
            if (!interior) seen_boundary = true;
            if (interior && seen_boundary) return "an interior row after a boundary row";
        }
        for (int t = 0; t < ntiles; ++t) {
            const int* d = plan.tile_desc.data() + 4 * (size_t)(tile0 + t);
            const size_t off = 16 * (size_t)d[0];
            const int ne = (d[1] - kSlabHeaderBytes) / kSlabEntryBytes;
            const size_t col_off = off + kSlabHeaderBytes + 36 * (size_t)ne;
            const int e1 = get_u16(plan.stream, off + 2 * (size_t)d[3]);
            bool halo = false;
            for (int j = 0; j < e1; ++j) halo = halo || static_cast<int>(get_u16(plan.stream, col_off + 2 * (size_t)j)) >= m;
            const bool flag = get_u16(plan.stream, off + 2 * (size_t)kSlabHaloWord) != 0;
            if (flag != halo) return "a tile's halo flag does not match its columns";
        }
    }
    return "";
}

void slab_spmv_host(const SlabPlan& plan, int nnz, const double* values, const double* x, double* y)
{
    // Fill, as the fill kernel does (float storage).
    std::vector<unsigned char> s = plan.stream;
    const size_t sfloats = s.size() / 4;
    const size_t ntiles_all = plan.tile_desc.size() / 4;
    const int header = plan.sym ? kSymHeaderBytes : kSlabHeaderBytes;
    for (size_t t = 0; t < ntiles_all; ++t) {
        // The tile's value area, float by float in stream order; element j = 3 c + i of a
        // transposed entry is element 3 i + c of its block.
        const int e0 = plan.tile_entry0[t], ne = plan.tile_entry0[t + 1] - e0;
        if (ne == 0) continue;
        const size_t v0 = 4 * (size_t)plan.tile_desc[4 * t] + header / 4;
        if (v0 + 9 * (size_t)ne > sfloats) continue;
        for (int f = 0; f < 9 * ne; ++f) {
            const int e = f / 9, j = f - 9 * e;
            const unsigned src = plan.fill_src[(size_t)e0 + e];
            float v = 0.f;
            if (src != kSlabNoPos) {
                const unsigned k = src & ~kSlabLowerBit;
                const int jj = (src & kSlabLowerBit) ? 3 * (j % 3) + j / 3 : j;
                if (k < (unsigned)nnz) v = static_cast<float>(values[9 * (size_t)k + jj]);
            }
            std::memcpy(s.data() + 4 * (v0 + f), &v, 4);
        }
    }
    if (plan.sym) {
        slab_spmv_host_sym(plan, s, x, y);
        return;
    }
    // Decode tile by tile with the kernel's clamps.
    for (int p = 0; p < plan.parts; ++p) {
        const int* pi = plan.part_info.data() + (size_t)kSlabPartInts * p;
        const int g0 = pi[0], m = pi[1], halo0 = pi[2], h = pi[3], tile0 = pi[4], ntiles = pi[5];
        const int wn = m + h;
        std::vector<double> win(3 * (size_t)wn);
        for (int w = 0; w < wn; ++w) {
            const int g = w < m ? g0 + w : plan.halo_src[halo0 + w - m];
            const int r = plan.perm[g];
            for (int a = 0; a < 3; ++a) win[3 * (size_t)w + a] = static_cast<double>(static_cast<float>(x[3 * (size_t)r + a]));
        }
        for (int t = 0; t < ntiles; ++t) {
            const int* d = plan.tile_desc.data() + 4 * (size_t)(tile0 + t);
            const size_t off = 16 * (size_t)d[0];
            const int bytes = d[1];
            const int ne = bytes >= kSlabHeaderBytes ? (bytes - kSlabHeaderBytes) / kSlabEntryBytes : 0;
            const size_t vals_off = off + kSlabHeaderBytes, col_off = vals_off + 36 * (size_t)ne;
            for (int i = 0; i < d[3]; ++i) {
                const int e0 = std::min<int>(get_u16(s, off + 2 * (size_t)i), ne);
                const int e1 = std::min<int>(get_u16(s, off + 2 * (size_t)(i + 1)), ne);
                double acc[3] = {0, 0, 0};
                for (int j = e0; j < e1; ++j) {
                    const int c = std::min<int>(get_u16(s, col_off + 2 * (size_t)j), wn - 1);
                    float v[9];
                    std::memcpy(v, s.data() + vals_off + 36 * (size_t)j, 36);
                    for (int a = 0; a < 3; ++a)
                        for (int mm = 0; mm < 3; ++mm) acc[a] += double(v[3 * mm + a]) * win[3 * (size_t)c + mm];
                }
                const int r = plan.perm[g0 + d[2] + i];
                for (int a = 0; a < 3; ++a) y[3 * (size_t)r + a] = acc[a];
            }
        }
    }
}

}  // namespace pk
