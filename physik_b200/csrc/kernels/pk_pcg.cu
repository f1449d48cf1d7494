// pk_pcg.cu -- the cooperative block-Jacobi PCG kernel of the implicit step.
//
// One launch per solve (SolvePreconditionedConjugateGradient,
// src/Core/Solvers/Linear/ConjugateGradientSolver.cpp:114-241, with the symmetric
// upper-BSR product of SparseBlockMatrix::Multiply, src/Math/SparseBlockMatrix.cpp:209-268,
// and World::IntegrateImplicitEuler, src/Core/World/World.cpp:644-695, fused at the end).
// Per iteration two grid-wide phases:
//   A: d = s + beta*d (per row), q = A d (gathered over the row's upper blocks and its
//      transposed lower blocks), partial d.q
//   B: x += alpha d, r -= alpha q, s = M^-1 r, partials r.s and r.r
// separated by bounded grid barriers; every block reduces the per-block partials in the
// same fixed order, so all blocks take identical decisions and results do not depend on
// timing.  The reference's stopping and failure rules are kept: x0 = 0, stop when
// r.s <= tol^2 * r0.s0, break on d.q <= 0 or a non-finite scalar, cleared solution on a
// non-finite rhs or invalid settings.
//
// Staged variant: each block's SpMV tiles (<= 64 rows) have their row metadata, upper
// blocks, columns and transpose entries copied into shared memory with TMA bulk copies
// (cp.async.bulk, mbarrier completion, double buffered).  Tiles are dealt round-robin
// (block b owns tiles b, b+G, b+2G, ...) so all blocks sweep one wavefront through the
// matrix and the transposed blocks a row re-reads were fetched by a neighbouring tile
// moments earlier (L2 hits).  Neighbours' s and d sit in one 32-byte record per row and
// come in with one 256-bit load.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <cstdlib>

#include "pk_device.cuh"

namespace pk {
namespace {

// ------------------------------------------------------------------ records
template <class Real>
struct SDPair {
    V3<Real> s, d;
};

// s and d of row c from its 8-value record (L1 bypassed: written by other blocks).
// The vector load fills the two padding slots too (a3, a7), which are not used.
#pragma nv_diag_suppress 550
__device__ __forceinline__ SDPair<float> ld_sd(const float* sd, int c)
{
    float a0, a1, a2, a3, a4, a5, a6, a7;
    asm volatile("ld.global.cg.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(a0), "=f"(a1), "=f"(a2), "=f"(a3), "=f"(a4), "=f"(a5), "=f"(a6), "=f"(a7)
                 : "l"(sd + 8 * (size_t)c));
    return SDPair<float>{V3<float>{a0, a1, a2}, V3<float>{a4, a5, a6}};
}
__device__ __forceinline__ SDPair<double> ld_sd(const double* sd, int c)
{
    double a0, a1, a2, a3, a4, a5, a6, a7;
    const double* p = sd + 8 * (size_t)c;
    asm volatile("ld.global.cg.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a0), "=d"(a1), "=d"(a2), "=d"(a3) : "l"(p));
    asm volatile("ld.global.cg.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a4), "=d"(a5), "=d"(a6), "=d"(a7) : "l"(p + 4));
    return SDPair<double>{V3<double>{a0, a1, a2}, V3<double>{a4, a5, a6}};
}
#pragma nv_diag_default 550
template <class Real>
__device__ __forceinline__ V3<Real> ld_d(const Real* sd, int c)
{
    const Real* p = sd + 8 * (size_t)c + 4;
    return V3<Real>{__ldcg(p), __ldcg(p + 1), __ldcg(p + 2)};
}
template <class Real>
__device__ __forceinline__ void st_s(Real* sd, int c, V3<Real> v)
{
    Real* p = sd + 8 * (size_t)c;
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
    p[3] = Real(0);
}
template <class Real>
__device__ __forceinline__ void st_d(Real* sd, int c, V3<Real> v)
{
    Real* p = sd + 8 * (size_t)c + 4;
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
    p[3] = Real(0);
}

// A 36-byte (float) block at any 4-byte offset, as three aligned 16-byte loads and a
// select; the read-only path (values do not change during the solve).
__device__ __forceinline__ M3<float> ld_block_window(const float* values, int k)
{
    const float* base = values + 9 * (size_t)k;
    const uintptr_t addr = reinterpret_cast<uintptr_t>(base);
    const float4* w = reinterpret_cast<const float4*>(addr & ~uintptr_t(15));
    const int sh = int((addr >> 2) & 3u);
    const float4 a = __ldg(w), b = __ldg(w + 1), c = __ldg(w + 2);
    const float v[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
    float o[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) o[e] = sh == 0 ? v[e] : (sh == 1 ? v[e + 1] : (sh == 2 ? v[e + 2] : v[e + 3]));
    M3<float> m;
    m.c[0] = V3<float>{o[0], o[1], o[2]};
    m.c[1] = V3<float>{o[3], o[4], o[5]};
    m.c[2] = V3<float>{o[6], o[7], o[8]};
    return m;
}
// A 72-byte (double) block at any 8-byte offset, as five aligned 16-byte loads.
__device__ __forceinline__ M3<double> ld_block_window(const double* values, int k)
{
    const double* base = values + 9 * (size_t)k;
    const uintptr_t addr = reinterpret_cast<uintptr_t>(base);
    const double2* w = reinterpret_cast<const double2*>(addr & ~uintptr_t(15));
    const bool sh = (addr & 8u) != 0;
    double v[10];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const double2 t = __ldg(w + i);
        v[2 * i] = t.x;
        v[2 * i + 1] = t.y;
    }
    double o[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) o[e] = sh ? v[e + 1] : v[e];
    M3<double> m;
    m.c[0] = V3<double>{o[0], o[1], o[2]};
    m.c[1] = V3<double>{o[3], o[4], o[5]};
    m.c[2] = V3<double>{o[6], o[7], o[8]};
    return m;
}

template <class Real>
__device__ __forceinline__ V3<Real> reduce16(V3<Real> acc)
{
#pragma unroll
    for (int off = 8; off > 0; off >>= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
        acc.z += __shfl_xor_sync(0xffffffffu, acc.z, off);
    }
    return acc;
}

// ------------------------------------------------------------------ unstaged row
// This lane's share (entries hl, hl+16, ...) of row r of q = A (s + beta d).
template <class Real>
__device__ __forceinline__ V3<Real> row_part_global(const BsrView<Real>& A, int r, int hl, const Real* sd, Real beta)
{
    V3<Real> acc{Real(0), Real(0), Real(0)};
    if (r < 0) return acc;
    const int ks = __ldg(A.row_start + r), ke = __ldg(A.row_start + r + 1);
    const int ls = __ldg(A.lt_start + r), le = __ldg(A.lt_start + r + 1);
    const int nu = ke - ks, tot = nu + (le - ls);
    for (int j = hl; j < tot; j += 16) {
        const bool tr = j >= nu;
        const int k = tr ? __ldg(A.lt_block + ls + (j - nu)) : ks + j;
        const int c = tr ? __ldg(A.lt_row + ls + (j - nu)) : __ldg(A.col + k);
        const SDPair<Real> p = ld_sd(sd, c);
        const V3<Real> xc = p.s + p.d * beta;
        const M3<Real> B = ld_block_window(A.values, k);
        acc = acc + (tr ? mul_t(B, xc) : mul(B, xc));
    }
    return acc;
}

// ------------------------------------------------------------------ staged tile
template <class Real>
struct TileBuf {
    int* rs;     // row_start[rs0 ..)
    int* lts;    // lt_start[rs0 ..)
    Real* vals;  // values of blocks [k0 ..)
    int* col;    // col of blocks [k0 ..)
    int* ltr;    // lt_row of entries [e0 ..)
    int* ltb;    // lt_block of entries [e0 ..)
};
template <class Real>
__device__ __forceinline__ TileBuf<Real> tile_buf(unsigned char* base)
{
    TileBuf<Real> b;
    b.rs = reinterpret_cast<int*>(base);
    b.lts = b.rs + kTileRowCap;
    b.vals = reinterpret_cast<Real*>(b.lts + kTileRowCap);
    b.col = reinterpret_cast<int*>(b.vals + size_t(kTileCapU) * 9);
    b.ltr = b.col + kTileCapU;
    b.ltb = b.ltr + kTileCapL;
    return b;
}
struct TileMeta {
    int ra, rb, rs0, k0, e0, ok;
};

__device__ __forceinline__ void load_desc(const int* desc, int t, int4& lo, int4& hi)
{
    const int4* p = reinterpret_cast<const int4*>(desc + 8 * (size_t)t);
    lo = __ldg(p);
    hi = __ldg(p + 1);
}

// Issued by one thread: bulk copies of a tile described by (lo, hi) into buffer b.  A
// descriptor outside the buffer's capacity (the host's tiling never makes one) is
// marked bad and completes without copying.
template <class Real>
__device__ void issue_tile(const BsrView<Real>& A, int4 lo, int4 hi, const TileBuf<Real>& b, TileMeta* meta,
                           unsigned long long* bar)
{
    const int ra = lo.x, rb = lo.y, rs0 = lo.z, nrs = lo.w, k0 = hi.x, nk = hi.y, e0 = hi.z, ne = hi.w;
    const bool fits = rb > ra && rb - ra <= kTileRowsMax && nrs > 0 && nrs <= kTileRowCap && nk > 0 &&
                      nk <= kTileCapU && ne >= 0 && ne <= kTileCapL && ((rs0 | nrs | k0 | nk | e0 | ne) & 3) == 0;
    meta->ra = ra;
    meta->rb = rb;
    meta->rs0 = rs0;
    meta->k0 = k0;
    meta->e0 = e0;
    meta->ok = fits ? 1 : 0;
    if (!fits) {
        mbar_arrive_expect_tx(bar, 0);
        return;
    }
    const unsigned rsb = 4u * unsigned(nrs), vb = unsigned(sizeof(Real)) * 9u * unsigned(nk);
    const unsigned cb = 4u * unsigned(nk), eb = 4u * unsigned(ne);
    mbar_arrive_expect_tx(bar, 2u * rsb + vb + cb + 2u * eb);
    bulk_g2s(b.rs, A.row_start + rs0, rsb, bar);
    bulk_g2s(b.lts, A.lt_start + rs0, rsb, bar);
    bulk_g2s(b.vals, A.values + size_t(9) * k0, vb, bar);
    bulk_g2s(b.col, A.col + k0, cb, bar);
    if (eb) {
        bulk_g2s(b.ltr, A.lt_row + e0, eb, bar);
        bulk_g2s(b.ltb, A.lt_block + e0, eb, bar);
    }
}

// Where entry j of tile row lr lives: an upper block in shared memory (kk) or a
// transposed lower block in global memory (k), and its column c.
struct EntryRef {
    int c;
    int k;
    bool lower;
    bool valid;
};
template <class Real>
__device__ __forceinline__ void row_extent(const TileBuf<Real>& tb, const TileMeta& m, int lr, int& ks, int& nu,
                                           int& ls, int& tot)
{
    const int r = m.ra + lr;
    ks = tb.rs[r - m.rs0];
    nu = tb.rs[r + 1 - m.rs0] - ks;
    ls = tb.lts[r - m.rs0];
    tot = nu + (tb.lts[r + 1 - m.rs0] - ls);
}
template <class Real>
__device__ __forceinline__ EntryRef entry_ref(const TileBuf<Real>& tb, const TileMeta& m, int ks, int nu, int ls,
                                              int tot, int j)
{
    EntryRef e;
    e.valid = j < tot;
    e.lower = j >= nu;
    if (!e.valid) {
        e.c = 0;
        e.k = 0;
    } else if (!e.lower) {
        e.k = ks + j - m.k0;  // shared-memory block index
        e.c = tb.col[e.k];
    } else {
        const int ee = ls + (j - nu) - m.e0;
        e.c = tb.ltr[ee];
        e.k = tb.ltb[ee];  // global block index
    }
    return e;
}
template <class Real>
__device__ __forceinline__ M3<Real> smem_block(const TileBuf<Real>& tb, int kk)
{
    const Real* q = tb.vals + size_t(9) * kk;
    M3<Real> B;
    B.c[0] = V3<Real>{q[0], q[1], q[2]};
    B.c[1] = V3<Real>{q[3], q[4], q[5]};
    B.c[2] = V3<Real>{q[6], q[7], q[8]};
    return B;
}
template <class Real>
__device__ __forceinline__ V3<Real> entry_product(const BsrView<Real>& A, const TileBuf<Real>& tb, const EntryRef& e,
                                                  const SDPair<Real>& p, Real beta)
{
    const V3<Real> xc = p.s + p.d * beta;
    if (e.lower) return mul_t(ld_block_window(A.values, e.k), xc);
    return mul(smem_block(tb, e.k), xc);
}

// This lane's shares of two tile rows la and lb (-1: none), loads of both issued first.
template <class Real>
__device__ __forceinline__ void staged_two_rows(const BsrView<Real>& A, const TileBuf<Real>& tb, const TileMeta& m,
                                                int la, int lb, int hl, const Real* sd, Real beta, V3<Real>& qa,
                                                V3<Real>& qb)
{
    qa = V3<Real>{Real(0), Real(0), Real(0)};
    qb = qa;
    int ksa = 0, nua = 0, lsa = 0, tota = 0, ksb = 0, nub = 0, lsb = 0, totb = 0;
    if (la >= 0) row_extent(tb, m, la, ksa, nua, lsa, tota);
    if (lb >= 0) row_extent(tb, m, lb, ksb, nub, lsb, totb);
    const EntryRef ea = entry_ref(tb, m, ksa, nua, lsa, tota, hl);
    const EntryRef eb = entry_ref(tb, m, ksb, nub, lsb, totb, hl);
    SDPair<Real> pa{}, pb{};
    if (ea.valid) pa = ld_sd(sd, ea.c);
    if (eb.valid) pb = ld_sd(sd, eb.c);
    if (ea.valid) qa = entry_product(A, tb, ea, pa, beta);
    if (eb.valid) qb = entry_product(A, tb, eb, pb, beta);
    for (int j = hl + 16; j < tota; j += 16) {
        const EntryRef e = entry_ref(tb, m, ksa, nua, lsa, tota, j);
        qa = qa + entry_product(A, tb, e, ld_sd(sd, e.c), beta);
    }
    for (int j = hl + 16; j < totb; j += 16) {
        const EntryRef e = entry_ref(tb, m, ksb, nub, lsb, totb, j);
        qb = qb + entry_product(A, tb, e, ld_sd(sd, e.c), beta);
    }
}

// ------------------------------------------------------------------ PCG kernel
template <class Real, class Acc, bool kStaged, int kMinBlocks>
__global__ void __launch_bounds__(kPcgThreads, kMinBlocks) pcg_kernel(PcgArgs<Real, Acc> P)
{
    __shared__ Acc sh_acc[3 * 32];
    __shared__ int sh_int[32];
    __shared__ int s_flag;
    __shared__ __align__(8) unsigned long long tile_bar[2];
    __shared__ TileMeta tile_meta[2];
    __shared__ int s_tile_fail;
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    const int tid = threadIdx.x, T = blockDim.x, blk = blockIdx.x, G = gridDim.x;
    const int n = P.a.n;
    const int lane = tid & 31, warp = tid >> 5, nwarps = T >> 5;
    const int half = lane >> 4, hl = lane & 15;

    // Unstaged: a contiguous row range per block.  Staged: tiles blk, blk + G, ...
    int r0 = 0, r1 = 0;
    const int my_tiles = kStaged ? (blk < P.ntiles ? (P.ntiles - 1 - blk) / G + 1 : 0) : 0;
    if (!kStaged) {
        const int per = (n + G - 1) / G;
        r0 = min(n, blk * per);
        r1 = min(n, r0 + per);
    }
    // Visits every row this block owns (the same mapping in every phase).
    auto for_rows = [&](auto&& f) {
        if (kStaged) {
            const int slot = tid & (kTileRowsMax - 1), tl = tid / kTileRowsMax, ntl = T / kTileRowsMax;
            for (int i = tl; i < my_tiles; i += ntl) {
                const int t = blk + i * G;
                const int r = __ldg(P.tile_desc + 8 * (size_t)t) + slot;
                if (r < __ldg(P.tile_desc + 8 * (size_t)t + 1)) f(r);
            }
        } else {
            for (int r = r0 + tid; r < r1; r += T) f(r);
        }
    };
    unsigned bar_phase = 0u;  // parity of the next completion of tile_bar[0] (bit 0) and [1] (bit 1)
    if (kStaged) {
        if (tid == 0) {
            mbar_init(&tile_bar[0], 1);
            mbar_init(&tile_bar[1], 1);
            mbar_fence_init();
            s_tile_fail = 0;
        }
        __syncthreads();
    }

    unsigned fl = 0;
    int iterations = 0;
    bool converged = false;
    Acc residual = Acc(0);
    bool have_x = true;
    bool timed_out = false;

    const unsigned in_flags = *(volatile unsigned*)P.flags;
    if (P.skip_on_flags && (in_flags & (kFlagPrecomputeFailed | kFlagSingularDiag))) {
        if (blk == 0 && tid == 0) {
            P.stats->iterations = 0;
            P.stats->converged = 0;
            P.stats->residual_norm = 0.0;
        }
        return;
    }

    // x = 0, r = b, s = M^-1 r, d = 0 (record 0); delta = r.s; |r|^2; finiteness.
    {
        Acc loc[2] = {Acc(0), Acc(0)};
        int bad = 0;
        for_rows([&](int r) {
            const V3<Real> br = ld3(P.b, r);
            if (!finite3(br)) bad |= 1;
            const V3<Real> z{Real(0), Real(0), Real(0)};
            st3(P.x, r, z);
            st3(P.r, r, br);
            const M3<Real> mi = ld9(P.minv, (size_t)r);
            const V3<Real> s = mul(mi, br);
            if (!finite9(mi) || !finite3(s)) bad |= 2;
            st_s(P.sd0, r, s);
            st_d(P.sd0, r, z);
            loc[0] += dot_acc<Acc>(br, s);
            loc[1] += dot_acc<Acc>(br, br);
        });
        block_sum<Acc, 2>(loc, sh_acc);
        bad = block_or(bad, sh_int);
        if (tid == 0) {
            P.part_b[2 * blk + 0] = loc[0];
            P.part_b[2 * blk + 1] = loc[1];
            P.part_bad[4 * blk + 1] = bad;
        }
    }
    if (!grid_barrier(P.sync, &s_flag)) { timed_out = true; goto finish; }

    {
        Acc g[2];
        grid_sum<Acc, 2>(P.part_b, 2, g, sh_acc);
        const int bad = grid_or(P.part_bad + 1, 4, sh_int);
        Acc delta = g[0];
        Acc rr = g[1];
        if (bad & 1) {  // non-finite rhs: the reference clears x (the solve fails)
            have_x = false;
            fl |= kFlagInvalidRhs;
            goto final_check;
        }
        if (P.max_iterations <= 0 || !acc_finite(P.tolerance) || P.tolerance <= Acc(0)) {
            have_x = false;
            fl |= kFlagInvalidRhs;
            goto final_check;
        }
        if (bad & 2) goto final_check;  // preconditioner output not finite: x stays 0
        if (!acc_finite(delta) || delta < Acc(0)) goto final_check;
        const Acc target = P.tolerance * P.tolerance * delta;
        if (!acc_finite(target)) goto final_check;
        if (delta <= target) {
            converged = true;
            residual = (acc_finite(rr) && rr >= Acc(0)) ? sqrt(rr) : Acc(INFINITY);
            goto final_check;
        }
        Acc beta = Acc(0);
        Real* sdcur = P.sd0;
        Real* sdnext = P.sd1;
        for (int it = 0; it < P.max_iterations; ++it) {
            if (delta <= target) {
                converged = true;
                break;
            }
            // Phase A: d_next = s + beta d_cur; q = A d_next; partial d_next . q
            {
                Acc loc[1] = {Acc(0)};
                int qbad = 0;
                auto finish_row = [&](int r, V3<Real> q) {
                    const SDPair<Real> p = ld_sd(sdcur, r);
                    const V3<Real> dn = p.s + p.d * Real(beta);
                    st_d(sdnext, r, dn);
                    st3(P.q, r, q);
                    loc[0] += dot_acc<Acc>(dn, q);
                    if (!finite3(q)) qbad = 1;
                };
                if (kStaged) {
                    const int nhw = T >> 4, hw = tid >> 4;
                    int4 dlo{}, dhi{};  // descriptor of the next tile to issue (thread 0)
                    if (tid == 0) {
                        if (my_tiles > 0) {
                            load_desc(P.tile_desc, blk, dlo, dhi);
                            issue_tile<Real>(P.a, dlo, dhi, tile_buf<Real>(dyn_smem), &tile_meta[0], &tile_bar[0]);
                        }
                        if (my_tiles > 1) {
                            load_desc(P.tile_desc, blk + G, dlo, dhi);
                            issue_tile<Real>(P.a, dlo, dhi, tile_buf<Real>(dyn_smem + tile_buffer_bytes<Real>()),
                                             &tile_meta[1], &tile_bar[1]);
                        }
                        if (my_tiles > 2) load_desc(P.tile_desc, blk + 2 * G, dlo, dhi);
                    }
                    for (int i = 0; i < my_tiles; ++i) {
                        const int bi = i & 1;
                        if (!mbar_wait(&tile_bar[bi], (bar_phase >> bi) & 1u)) s_tile_fail = 1;
                        bar_phase ^= 1u << bi;
                        const TileMeta m = tile_meta[bi];
                        const TileBuf<Real> tb = tile_buf<Real>(dyn_smem + bi * tile_buffer_bytes<Real>());
                        const int nr = (m.ok && !s_tile_fail) ? m.rb - m.ra : 0;
                        for (int lr0 = 0; lr0 < nr; lr0 += 2 * nhw) {
                            const int la = lr0 + hw, lb = lr0 + hw + nhw;
                            V3<Real> qa, qb;
                            staged_two_rows<Real>(P.a, tb, m, la < nr ? la : -1, lb < nr ? lb : -1, hl, sdcur,
                                                  Real(beta), qa, qb);
                            qa = reduce16(qa);
                            qb = reduce16(qb);
                            if (hl == 0) {
                                if (la < nr) finish_row(m.ra + la, qa);
                                if (lb < nr) finish_row(m.ra + lb, qb);
                            }
                        }
                        if (!m.ok) qbad = 1;
                        __syncthreads();  // every warp is done with buffer bi
                        if (tid == 0 && i + 2 < my_tiles) {
                            issue_tile<Real>(P.a, dlo, dhi, tb, &tile_meta[bi], &tile_bar[bi]);
                            if (i + 3 < my_tiles) load_desc(P.tile_desc, blk + (i + 3) * G, dlo, dhi);
                        }
                    }
                    if (s_tile_fail) {
                        qbad = 1;
                        if (tid == 0) atomicExch(&P.sync->err, 1);
                    }
                } else {
                    for (int base = r0 + 2 * warp; base < r1; base += 2 * nwarps) {
                        const int r = base + half;
                        const bool valid = r < r1;
                        const V3<Real> q =
                            reduce16(row_part_global<Real>(P.a, valid ? r : -1, hl, sdcur, Real(beta)));
                        if (valid && hl == 0) finish_row(r, q);
                    }
                }
                block_sum<Acc, 1>(loc, sh_acc);
                qbad = block_or(qbad, sh_int);
                if (tid == 0) {
                    P.part_a[blk] = loc[0];
                    P.part_bad[4 * blk + 0] = qbad;
                }
            }
            if (!grid_barrier(P.sync, &s_flag)) { timed_out = true; goto finish; }
            Acc dq;
            {
                Acc g1[1];
                grid_sum<Acc, 1>(P.part_a, 1, g1, sh_acc);
                dq = g1[0];
                if (grid_or(P.part_bad, 4, sh_int)) { fl |= kFlagBreakdown; break; }
            }
            if (!acc_finite(dq) || dq <= Acc(0)) { fl |= kFlagBreakdown; break; }
            const Acc alpha = delta / dq;
            if (!acc_finite(alpha)) { fl |= kFlagBreakdown; break; }
            // Phase B: x += alpha d; r -= alpha q; s = M^-1 r; partials r.s and r.r
            {
                Acc loc[2] = {Acc(0), Acc(0)};
                int sbad = 0;
                for_rows([&](int r) {
                    const V3<Real> dn = ld_d(sdnext, r);
                    const V3<Real> q = ldcg3(P.q, r);
                    const V3<Real> xv = axpy<Real, Acc>(ldplain3(P.x, r), alpha, dn);
                    const V3<Real> rv = axpy<Real, Acc>(ldplain3(P.r, r), -alpha, q);
                    st3(P.x, r, xv);
                    st3(P.r, r, rv);
                    const V3<Real> s = mul(ld9(P.minv, (size_t)r), rv);
                    if (!finite3(s)) sbad = 1;
                    st_s(sdnext, r, s);
                    loc[0] += dot_acc<Acc>(rv, s);
                    loc[1] += dot_acc<Acc>(rv, rv);
                });
                block_sum<Acc, 2>(loc, sh_acc);
                sbad = block_or(sbad, sh_int);
                if (tid == 0) {
                    P.part_b[2 * blk + 0] = loc[0];
                    P.part_b[2 * blk + 1] = loc[1];
                    P.part_bad[4 * blk + 1] = sbad;
                }
            }
            if (!grid_barrier(P.sync, &s_flag)) { timed_out = true; goto finish; }
            {
                Acc g2[2];
                grid_sum<Acc, 2>(P.part_b, 2, g2, sh_acc);
                rr = g2[1];
                if (grid_or(P.part_bad + 1, 4, sh_int)) { fl |= kFlagBreakdown; break; }
                const Acc old = delta;
                delta = g2[0];
                if (!acc_finite(delta) || !acc_finite(old) || old <= Acc(0)) { fl |= kFlagBreakdown; break; }
                beta = delta / old;
                if (!acc_finite(beta)) { fl |= kFlagBreakdown; break; }
            }
            Real* t = sdcur;
            sdcur = sdnext;
            sdnext = t;
            iterations = it + 1;
        }
        if (delta <= target) converged = true;
        residual = (acc_finite(rr) && rr >= Acc(0)) ? sqrt(rr) : Acc(INFINITY);
    }

final_check:
    // The solve succeeds when x is present and finite; integration is all-or-nothing.
    {
        int bad = 0;
        for_rows([&](int r) {
            const V3<Real> dv = have_x ? ldplain3(P.x, r) : V3<Real>{Real(0), Real(0), Real(0)};
            if (!finite3(dv)) bad |= 1;
            if (P.integrate) {
                const int node = __ldg(P.dyn_to_node + r);
                const V3<Real> xo = ldplain3(P.node_x, node), vo = ldplain3(P.node_v, node);
                const V3<Real> nv = vo + dv;
                const V3<Real> nx = xo + nv * P.dt;
                if (!finite3(xo) || !finite3(vo) || !finite3(nv) || !finite3(nx)) bad |= 2;
            }
        });
        bad = block_or(bad, sh_int);
        if (tid == 0) P.part_bad[4 * blk + 2] = bad;
    }
    if (!grid_barrier(P.sync, &s_flag)) { timed_out = true; goto finish; }
    {
        const int bad = grid_or(P.part_bad + 2, 4, sh_int);
        const bool solved = have_x && !(bad & 1);
        if (!have_x) fl |= kFlagInvalidRhs;
        if (have_x && (bad & 1)) fl |= kFlagNonFiniteDv;
        if (solved) fl |= kFlagSolved;
        if (solved && P.integrate) {
            if (bad & 2) {
                fl |= kFlagIntegrateAbort;
            } else {
                for_rows([&](int r) {
                    const int node = __ldg(P.dyn_to_node + r);
                    const V3<Real> dv = ldplain3(P.x, r);
                    const V3<Real> nv = ldplain3(P.node_v, node) + dv;
                    const V3<Real> nx = ldplain3(P.node_x, node) + nv * P.dt;
                    st3(P.node_v, node, nv);
                    st3(P.node_x, node, nx);
                });
                fl |= kFlagIntegrated;
            }
        }
        if (converged) fl |= kFlagConverged;
    }

finish:
    if (timed_out) fl |= kFlagBarrierTimeout;
    if (blk == 0 && tid == 0) {
        P.stats->iterations = iterations;
        P.stats->converged = converged ? 1 : 0;
        P.stats->residual_norm = (double)residual;
        atomicOr(P.flags, fl);
    } else if (timed_out && tid == 0) {
        atomicOr(P.flags, kFlagBarrierTimeout);
    }
}

}  // namespace

// ------------------------------------------------------------------ launchers
// Staged kernel occupancy: 2 blocks per SM (64 registers per thread) by default, or
// 1 block per SM (up to 128 registers) with PK_PCG_MINB=1.
static int staged_min_blocks()
{
    const char* e = std::getenv("PK_PCG_MINB");
    return (e && e[0] == '1') ? 1 : 2;
}

template <class Real, class Acc>
static const void* pcg_fn(bool staged)
{
    if (!staged) return (const void*)pcg_kernel<Real, Acc, false, 2>;
    return staged_min_blocks() == 1 ? (const void*)pcg_kernel<Real, Acc, true, 1>
                                    : (const void*)pcg_kernel<Real, Acc, true, 2>;
}

template <class Real, class Acc>
static size_t pcg_dyn_smem(bool staged)
{
    return staged ? 2 * tile_buffer_bytes<Real>() : 0;
}

template <class Real, class Acc>
int pcg_max_grid(int threads, bool staged)
{
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    const size_t smem = pcg_dyn_smem<Real, Acc>(staged);
    const void* fn = pcg_fn<Real, Acc>(staged);
    cudaError_t e = cudaSuccess;
    if (staged) e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
    if (e != cudaSuccess) return 0;
    return sms * per_sm;
}

template <class Real, class Acc>
cudaError_t launch_pcg_kernel(const PcgArgs<Real, Acc>& args, int grid, int threads, cudaStream_t stream)
{
    PcgArgs<Real, Acc> a = args;
    void* kargs[] = {&a};
    const bool staged = args.ntiles > 0;
    const size_t smem = pcg_dyn_smem<Real, Acc>(staged);
    const void* fn = pcg_fn<Real, Acc>(staged);
    if (staged) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
    }
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(threads), kargs, smem, stream);
}

template cudaError_t launch_pcg_kernel<float, float>(const PcgArgs<float, float>&, int, int, cudaStream_t);
template cudaError_t launch_pcg_kernel<float, double>(const PcgArgs<float, double>&, int, int, cudaStream_t);
template cudaError_t launch_pcg_kernel<double, double>(const PcgArgs<double, double>&, int, int, cudaStream_t);
template int pcg_max_grid<float, float>(int, bool);
template int pcg_max_grid<float, double>(int, bool);
template int pcg_max_grid<double, double>(int, bool);

}  // namespace pk
