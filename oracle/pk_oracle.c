/*
 * pk_oracle.c -- CPU restatement of PhysiK's implicit soft-body step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA path, never part of
 * it: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 *
 * It restates, in plain C and in the reference's own operation order, the path
 *   World::Step                         src/Core/World/World.cpp:32-73
 *   TetMeshPhysicsComponent::UpdateSystem src/Components/TetMeshPhysicsComponent.cpp:293-354
 *   FEMModel (rest data, polar, corotated forces/stiffness, lumped mass)
 *                                       src/Core/Physics/FEM/FEMModel.cpp:115-163, 174-225,
 *                                       247-271, 312-424, 504-557, 635-713
 *   SparseBlockMatrix                   src/Math/SparseBlockMatrix.cpp:83-144, 209-282
 *   SolverData                          src/Core/Solvers/SolverData.cpp:87-465
 *   SolvePreconditionedConjugateGradient src/Core/Solvers/Linear/ConjugateGradientSolver.cpp:114-241
 *   World::IntegrateImplicitEuler       src/Core/World/World.cpp:644-695
 * so that, built with REAL=float and without FMA contraction, it reproduces the FP32
 * reference bit for bit; built with REAL=double it is the FP64 oracle.  The pin is
 * checked by tests against the reference compiled from its own sources (oracle/_ref)
 * and against committed fixtures (tests/golden).
 *
 * Compile twice: -DPKO_REAL=float -DPKO_SUFFIX=f32 and -DPKO_REAL=double -DPKO_SUFFIX=f64.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef PKO_REAL
#define PKO_REAL float
#endif
#ifndef PKO_SUFFIX
#define PKO_SUFFIX f32
#endif
#define PKO_CAT2(a, b) a##b
#define PKO_CAT(a, b) PKO_CAT2(a, b)
#define PKO(name) PKO_CAT(PKO_CAT(pko_, PKO_SUFFIX), PKO_CAT(_, name))

typedef PKO_REAL real;
#define R(x) ((real)(x))

#if defined(__GNUC__)
#define PKO_EXPORT __attribute__((visibility("default")))
#else
#define PKO_EXPORT
#endif

/* ------------------------------------------------------------------ math */
/* Vec3.h:7-95, Mat3.h:11-84.  Column-major Mat3; default Mat3 is identity. */
typedef struct { real x, y, z; } v3;
typedef struct { v3 c[3]; } m3;

static inline v3 V3(real x, real y, real z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vneg(v3 a) { return V3(-a.x, -a.y, -a.z); }
static inline v3 vmul(v3 a, real s) { return V3(a.x * s, a.y * s, a.z * s); }
static inline real vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b)
{
    return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline real vlen2(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static inline int vfinite(v3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }

static inline m3 mcols(v3 a, v3 b, v3 c) { m3 m; m.c[0] = a; m.c[1] = b; m.c[2] = c; return m; }
static inline m3 mident(void) { return mcols(V3(1, 0, 0), V3(0, 1, 0), V3(0, 0, 1)); }
static inline m3 mzero(void) { return mcols(V3(0, 0, 0), V3(0, 0, 0), V3(0, 0, 0)); }
/* Mat3::operator*(Vec3): c0*x + c1*y + c2*z, evaluated left to right. */
static inline v3 mvec(m3 m, v3 v) { return vadd(vadd(vmul(m.c[0], v.x), vmul(m.c[1], v.y)), vmul(m.c[2], v.z)); }
static inline m3 mmul(m3 a, m3 b) { return mcols(mvec(a, b.c[0]), mvec(a, b.c[1]), mvec(a, b.c[2])); }
static inline m3 mtrans(m3 m)
{
    return mcols(V3(m.c[0].x, m.c[1].x, m.c[2].x), V3(m.c[0].y, m.c[1].y, m.c[2].y),
                 V3(m.c[0].z, m.c[1].z, m.c[2].z));
}
static inline m3 madd(m3 a, m3 b) { return mcols(vadd(a.c[0], b.c[0]), vadd(a.c[1], b.c[1]), vadd(a.c[2], b.c[2])); }
static inline m3 mscale(m3 a, real s) { return mcols(vmul(a.c[0], s), vmul(a.c[1], s), vmul(a.c[2], s)); }
static inline real mdet(m3 m) { return vdot(m.c[0], vcross(m.c[1], m.c[2])); }
static inline int mfinite(m3 m) { return vfinite(m.c[0]) && vfinite(m.c[1]) && vfinite(m.c[2]); }
/* Mat3.h:67-84: adjugate inverse; identity when |det| <= 1e-6. */
static inline m3 minv(m3 m)
{
    v3 r0 = vcross(m.c[1], m.c[2]);
    v3 r1 = vcross(m.c[2], m.c[0]);
    v3 r2 = vcross(m.c[0], m.c[1]);
    real det = vdot(m.c[0], r0);
    if (fabs((double)det) <= (double)R(0.000001)) return mident();
    real inv = R(1.0) / det;
    return mtrans(mcols(vmul(r0, inv), vmul(r1, inv), vmul(r2, inv)));
}
static inline real mget(m3 m, int row, int col)
{
    v3 c = m.c[col];
    return row == 0 ? c.x : (row == 1 ? c.y : c.z);
}
static inline void mset(m3* m, int row, int col, real value)
{
    v3* c = &m->c[col];
    if (row == 0) c->x = value; else if (row == 1) c->y = value; else c->z = value;
}
static inline v3 mrow(m3 m, int row) { return V3(mget(m, row, 0), mget(m, row, 1), mget(m, row, 2)); }

/* FEMModel.cpp:104-113 */
static real frob_diff2(m3 a, m3 b)
{
    real total = R(0.0);
    for (int col = 0; col < 3; ++col) total += vlen2(vsub(a.c[col], b.c[col]));
    return total;
}

/* FEMModel.cpp:115-163: Newton polar averaging, <=12 iterations, tolerance 1e-10,
 * identity fallback when |det| <= 1e-8 or non-finite, reflection fix on column 2. */
static m3 polar_rotation(m3 f, int* out_iterations)
{
    const real min_det = R(1.0e-8);
    if (out_iterations) *out_iterations = 0;
    if (!mfinite(f) || fabs((double)mdet(f)) <= (double)min_det) return mident();
    m3 rot = f;
    for (int it = 0; it < 12; ++it) {
        if (out_iterations) *out_iterations = it + 1;
        m3 ti = minv(mtrans(rot));
        if (!mfinite(ti) || fabs((double)mdet(ti)) <= (double)min_det) return mident();
        m3 next = mscale(madd(rot, ti), R(0.5));
        if (!mfinite(next)) return mident();
        if (frob_diff2(next, rot) <= R(1.0e-10)) { rot = next; break; }
        rot = next;
    }
    if (!mfinite(rot)) return mident();
    if (mdet(rot) < R(0.0)) rot.c[2] = vmul(rot.c[2], R(-1.0));
    return rot;
}

/* ------------------------------------------------------------ per-tet data */
typedef struct {
    int n[4];
    int active;
    real rest_volume;
    m3 dm_inv;
    v3 rest[4];
    v3 grad[4];
    real young, poisson, damping;
    real ke[12][12];
} tet_t;

/* FEMModel.cpp:504-548 */
static void tet_rest_data(tet_t* t, const v3* rest_positions)
{
    v3 r0 = rest_positions[t->n[0]], r1 = rest_positions[t->n[1]];
    v3 r2 = rest_positions[t->n[2]], r3 = rest_positions[t->n[3]];
    m3 dm = mcols(vsub(r1, r0), vsub(r2, r0), vsub(r3, r0));
    real det = mdet(dm);
    t->rest[0] = r0; t->rest[1] = r1; t->rest[2] = r2; t->rest[3] = r3;
    real vol = (real)fabs((double)det) / R(6.0);
    if (vol <= R(1.0e-8)) {
        t->rest_volume = R(0.0);
        t->dm_inv = mzero();
        for (int a = 0; a < 4; ++a) t->grad[a] = V3(0, 0, 0);
        return;
    }
    t->rest_volume = vol;
    t->dm_inv = minv(dm);
    t->grad[1] = mrow(t->dm_inv, 0);
    t->grad[2] = mrow(t->dm_inv, 1);
    t->grad[3] = mrow(t->dm_inv, 2);
    t->grad[0] = vneg(vadd(vadd(t->grad[1], t->grad[2]), t->grad[3]));
}

/* FEMModel.cpp:174-200 (D), 202-225 (B), 312-334 (Ke = V * B^T D B). */
static void tet_fem_cache(tet_t* t, real b[6][12], real d[6][6])
{
    memset(b, 0, sizeof(real) * 72);
    memset(d, 0, sizeof(real) * 36);
    real e = t->young > R(0.0) ? t->young : R(0.0);
    if (e > R(0.0)) {
        real nu = t->poisson;
        if (nu > R(0.49)) nu = R(0.49);
        if (nu < R(-0.99)) nu = R(-0.99);
        real lambda = e * nu / ((R(1.0) + nu) * (R(1.0) - R(2.0) * nu));
        real mu = e / (R(2.0) * (R(1.0) + nu));
        d[0][0] = lambda + R(2.0) * mu; d[0][1] = lambda; d[0][2] = lambda;
        d[1][0] = lambda; d[1][1] = lambda + R(2.0) * mu; d[1][2] = lambda;
        d[2][0] = lambda; d[2][1] = lambda; d[2][2] = lambda + R(2.0) * mu;
        d[3][3] = mu; d[4][4] = mu; d[5][5] = mu;
    }
    for (int a = 0; a < 4; ++a) {
        v3 g = t->grad[a];
        int c = a * 3;
        b[0][c + 0] = g.x; b[1][c + 1] = g.y; b[2][c + 2] = g.z;
        b[3][c + 0] = g.y; b[3][c + 1] = g.x;
        b[4][c + 1] = g.z; b[4][c + 2] = g.y;
        b[5][c + 0] = g.z; b[5][c + 2] = g.x;
    }
    for (int row = 0; row < 12; ++row)
        for (int col = 0; col < 12; ++col) {
            real value = R(0.0);
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j < 6; ++j) value += b[i][row] * d[i][j] * b[j][col];
            t->ke[row][col] = t->rest_volume * value;
        }
}

/* Per-tet result of FEMModel::ComputeElasticForcesAndStiffness (FEMModel.cpp:377-424). */
typedef struct {
    v3 f[4];
    m3 k[4][4];
} contrib_t;

static void element_contribution(const tet_t* t, real b[6][12], real d[6][6], const v3* x, const v3* v,
                                 const m3* rot, contrib_t* out)
{
    real u[12];
    if (rot) {
        /* BuildCorotatedDisplacementVector, FEMModel.cpp:247-271 */
        v3 origin = x[t->n[0]];
        m3 inv_rot = mtrans(*rot);
        for (int a = 0; a < 4; ++a) {
            v3 local = vadd(mvec(inv_rot, vsub(x[t->n[a]], origin)), t->rest[0]);
            v3 du = vsub(local, t->rest[a]);
            u[a * 3 + 0] = du.x; u[a * 3 + 1] = du.y; u[a * 3 + 2] = du.z;
        }
    } else {
        /* BuildDisplacementVector, FEMModel.cpp:227-245 */
        for (int a = 0; a < 4; ++a) {
            v3 du = vsub(x[t->n[a]], t->rest[a]);
            u[a * 3 + 0] = du.x; u[a * 3 + 1] = du.y; u[a * 3 + 2] = du.z;
        }
    }
    real strain[6] = {0}, stress[6] = {0}, fint[12] = {0};
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 12; ++c) strain[r] += b[r][c] * u[c];
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) stress[r] += d[r][c] * strain[c];
    for (int c = 0; c < 12; ++c)
        for (int r = 0; r < 6; ++r) fint[c] += b[r][c] * stress[r];
    for (int c = 0; c < 12; ++c) fint[c] *= t->rest_volume;
    for (int a = 0; a < 4; ++a) {
        v3 fe = V3(-fint[a * 3 + 0], -fint[a * 3 + 1], -fint[a * 3 + 2]);
        if (rot) fe = mvec(*rot, fe);
        v3 fd = vmul(v[t->n[a]], -t->damping);
        out->f[a] = vadd(fe, fd);
    }
    /* AssembleStiffness, FEMModel.cpp:336-375 */
    m3 rt = rot ? mtrans(*rot) : mident();
    for (int ra = 0; ra < 4; ++ra)
        for (int cb = 0; cb < 4; ++cb) {
            m3 blk = mzero();
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) mset(&blk, i, j, t->ke[ra * 3 + i][cb * 3 + j]);
            if (rot) blk = mmul(mmul(*rot, blk), rt);
            out->k[ra][cb] = blk;
        }
}

/* ------------------------------------------------------------ sparse matrix */
/* SparseBlockMatrix: canonical (row <= col) blocks, per-row sorted unique columns. */
typedef struct {
    int n;
    int* row_start; /* n+1 */
    int* col;       /* nnz */
    m3* val;        /* nnz */
    int nnz;
} bsr_t;

static void bsr_free(bsr_t* m)
{
    free(m->row_start); free(m->col); free(m->val);
    memset(m, 0, sizeof(*m));
}

static int cmp_u64(const void* a, const void* b)
{
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* SparseBlockMatrix::BuildPattern, SparseBlockMatrix.cpp:83-129 (invalid coordinates
 * dropped, canonicalised, sorted and deduplicated per row). */
static void bsr_build(bsr_t* m, int n, const int* rows, const int* cols, long count)
{
    bsr_free(m);
    if (n <= 0) return;
    m->n = n;
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(count > 0 ? count : 1));
    long k = 0;
    for (long i = 0; i < count; ++i) {
        int r = rows[i], c = cols[i];
        if (r < 0 || r >= n || c < 0 || c >= n) continue;
        if (r > c) { int t = r; r = c; c = t; }
        keys[k++] = ((uint64_t)(uint32_t)r << 32) | (uint32_t)c;
    }
    qsort(keys, (size_t)k, sizeof(uint64_t), cmp_u64);
    long u = 0;
    for (long i = 0; i < k; ++i)
        if (u == 0 || keys[i] != keys[u - 1]) keys[u++] = keys[i];
    m->row_start = (int*)calloc((size_t)n + 1, sizeof(int));
    m->col = (int*)malloc(sizeof(int) * (size_t)(u > 0 ? u : 1));
    m->val = (m3*)malloc(sizeof(m3) * (size_t)(u > 0 ? u : 1));
    m->nnz = (int)u;
    for (long i = 0; i < u; ++i) {
        int r = (int)(keys[i] >> 32);
        m->col[i] = (int)(keys[i] & 0xffffffffu);
        m->val[i] = mzero();
        m->row_start[r + 1]++;
    }
    for (int r = 0; r < n; ++r) m->row_start[r + 1] += m->row_start[r];
    free(keys);
}

/* FindBlockIndex, SparseBlockMatrix.cpp:270-282 */
static int bsr_find(const bsr_t* m, int r, int c)
{
    if (r > c) { int t = r; r = c; c = t; }
    if (r < 0 || r >= m->n) return -1;
    int lo = m->row_start[r], hi = m->row_start[r + 1];
    while (lo < hi) {
        int mid = (lo + hi) / 2;
        if (m->col[mid] < c) lo = mid + 1; else hi = mid;
    }
    return (lo < m->row_start[r + 1] && m->col[lo] == c) ? lo : -1;
}

/* AddBlock, SparseBlockMatrix.cpp:131-144 */
static int bsr_add(bsr_t* m, int r, int c, m3 b)
{
    int k = bsr_find(m, r, c);
    if (k < 0) return 0;
    m->val[k] = madd(m->val[k], r <= c ? b : mtrans(b));
    return 1;
}

/* Multiply(vector<Vec3>), SparseBlockMatrix.cpp:209-268 */
static void bsr_mul(const bsr_t* m, const v3* in, v3* out)
{
    for (int r = 0; r < m->n; ++r) out[r] = V3(0, 0, 0);
    for (int r = 0; r < m->n; ++r)
        for (int k = m->row_start[r]; k < m->row_start[r + 1]; ++k) {
            int c = m->col[k];
            m3 b = m->val[k];
            v3 xc = in[c];
            real rx = out[r].x, ry = out[r].y, rz = out[r].z;
            rx += b.c[0].x * xc.x + b.c[1].x * xc.y + b.c[2].x * xc.z;
            ry += b.c[0].y * xc.x + b.c[1].y * xc.y + b.c[2].y * xc.z;
            rz += b.c[0].z * xc.x + b.c[1].z * xc.y + b.c[2].z * xc.z;
            out[r] = V3(rx, ry, rz);
            if (r == c) continue;
            v3 xr = in[r];
            real cx = out[c].x, cy = out[c].y, cz = out[c].z;
            cx += b.c[0].x * xr.x + b.c[0].y * xr.y + b.c[0].z * xr.z;
            cy += b.c[1].x * xr.x + b.c[1].y * xr.y + b.c[1].z * xr.z;
            cz += b.c[2].x * xr.x + b.c[2].y * xr.y + b.c[2].z * xr.z;
            out[c] = V3(cx, cy, cz);
        }
}

/* ------------------------------------------------------------------- PCG */
typedef struct {
    int iterations;
    double residual_norm;
    int converged;
} pko_cg_result;

static real vec_dot(const v3* a, const v3* b, int n)
{
    real s = R(0.0);
    for (int i = 0; i < n; ++i) s += vdot(a[i], b[i]);
    return s;
}

static int apply_precond(const m3* minv_blocks, const v3* in, v3* out, int n)
{
    for (int i = 0; i < n; ++i) {
        if (!mfinite(minv_blocks[i])) return 0;
        out[i] = mvec(minv_blocks[i], in[i]);
        if (!vfinite(out[i])) return 0;
    }
    return 1;
}

static real resid_norm(const v3* r, int n)
{
    real s = vec_dot(r, r, n);
    if (!isfinite(s) || s < R(0.0)) return (real)INFINITY;
    return (real)sqrt(s);
}

/* SolvePreconditionedConjugateGradient, ConjugateGradientSolver.cpp:114-241.
 * Returns 1 when x holds n entries, 0 when the reference would leave it cleared.
 * Loop-local failures keep the last iterate, as the reference does. */
static int pcg_solve(const bsr_t* a, const v3* b, int n, int max_it, real tol, const m3* minv_blocks,
                     int minv_count, v3* x, pko_cg_result* res)
{
    res->iterations = 0; res->residual_norm = 0.0; res->converged = 0;
    if (n == 0) { res->converged = 1; return 0; }
    int bfinite = 1;
    for (int i = 0; i < n; ++i) bfinite &= vfinite(b[i]);
    if (a->n != n || max_it <= 0 || !isfinite(tol) || tol <= R(0.0) || !bfinite) return 0;
    v3* r = (v3*)malloc(sizeof(v3) * (size_t)n);
    v3* d = (v3*)malloc(sizeof(v3) * (size_t)n);
    v3* q = (v3*)malloc(sizeof(v3) * (size_t)n);
    for (int i = 0; i < n; ++i) { x[i] = V3(0, 0, 0); r[i] = b[i]; }
    if (minv_count != n || !apply_precond(minv_blocks, r, d, n)) goto done;
    real delta = vec_dot(r, d, n);
    if (!isfinite(delta) || delta < R(0.0)) goto done;
    real target = tol * tol * delta;
    if (!isfinite(target)) goto done;
    if (delta <= target) { res->converged = 1; res->residual_norm = resid_norm(r, n); goto done; }
    for (int it = 0; it < max_it; ++it) {
        if (delta <= target) { res->converged = 1; break; }
        bsr_mul(a, d, q);
        int qf = 1;
        for (int i = 0; i < n; ++i) qf &= vfinite(q[i]);
        if (!qf) break;
        real dq = vec_dot(d, q, n);
        if (!isfinite(dq) || dq <= R(0.0)) break;
        real alpha = delta / dq;
        if (!isfinite(alpha)) break;
        for (int i = 0; i < n; ++i) x[i] = vadd(x[i], vmul(d[i], alpha));
        for (int i = 0; i < n; ++i) r[i] = vadd(r[i], vmul(q[i], -alpha));
        if (!apply_precond(minv_blocks, r, q, n)) break;
        real old = delta;
        delta = vec_dot(r, q, n);
        if (!isfinite(delta) || !isfinite(old) || old <= R(0.0)) break;
        real beta = delta / old;
        if (!isfinite(beta)) break;
        for (int i = 0; i < n; ++i) d[i] = vadd(q[i], vmul(d[i], beta));
        res->iterations = it + 1;
    }
    if (delta <= target) res->converged = 1;
    res->residual_norm = resid_norm(r, n);
done:
    free(r); free(d); free(q);
    return 1;
}

/* ---------------------------------------------------------------- problem */
typedef struct {
    int node_count;
    int tet_count;
    int body_count;
    tet_t* tets;
    real (*b)[6][12];
    real (*d)[6][6];
    int* body_tet_start;  /* body_count+1 */
    int* body_node_start; /* body_count+1 */
    real* body_density;
    unsigned char* fixed;
    unsigned char* active;
    int linear;
    v3 gravity;
    int max_iterations;
    real tolerance;
    int use_jacobi;
    /* last step, for inspection */
    bsr_t a;
    int* node_to_dyn;
    int dyn_count;
    v3* rhs;
    m3* minv;
    v3* dv;
    real* mass;
    v3* force;
    pko_cg_result cg;
    int precompute_ok;
    int solved;
    int integrated;
    int mass_error;
} problem_t;

PKO_EXPORT void* PKO(create)(int node_count, const real* rest_positions, int tet_count, const int* tet_nodes,
                             int body_count, const int* body_tet_start, const int* body_node_start,
                             const real* body_density, const real* tet_young, const real* tet_poisson,
                             const real* tet_damping)
{
    problem_t* p = (problem_t*)calloc(1, sizeof(problem_t));
    p->node_count = node_count;
    p->tet_count = tet_count;
    p->body_count = body_count;
    p->tets = (tet_t*)calloc((size_t)(tet_count > 0 ? tet_count : 1), sizeof(tet_t));
    p->b = calloc((size_t)(tet_count > 0 ? tet_count : 1), sizeof(*p->b));
    p->d = calloc((size_t)(tet_count > 0 ? tet_count : 1), sizeof(*p->d));
    p->body_tet_start = (int*)malloc(sizeof(int) * (size_t)(body_count + 1));
    p->body_node_start = (int*)malloc(sizeof(int) * (size_t)(body_count + 1));
    p->body_density = (real*)malloc(sizeof(real) * (size_t)(body_count > 0 ? body_count : 1));
    memcpy(p->body_tet_start, body_tet_start, sizeof(int) * (size_t)(body_count + 1));
    memcpy(p->body_node_start, body_node_start, sizeof(int) * (size_t)(body_count + 1));
    memcpy(p->body_density, body_density, sizeof(real) * (size_t)body_count);
    p->fixed = (unsigned char*)calloc((size_t)node_count + 1, 1);
    p->active = (unsigned char*)malloc((size_t)node_count + 1);
    memset(p->active, 1, (size_t)node_count + 1);
    const v3* rest = (const v3*)rest_positions;
    for (int t = 0; t < tet_count; ++t) {
        tet_t* tt = &p->tets[t];
        for (int a = 0; a < 4; ++a) tt->n[a] = tet_nodes[t * 4 + a];
        tt->active = 1;
        tt->young = tet_young[t];
        tt->poisson = tet_poisson[t];
        tt->damping = tet_damping[t];
        for (int a = 0; a < 4; ++a) tt->rest[a] = V3(0, 0, 0);
        tt->dm_inv = mident();
        tet_rest_data(tt, rest);
        tet_fem_cache(tt, p->b[t], p->d[t]);
    }
    p->gravity = V3(0, 0, 0);
    p->max_iterations = 128;
    p->tolerance = R(1.0e-4);
    p->use_jacobi = 1;
    return p;
}

static void clear_last(problem_t* p)
{
    bsr_free(&p->a);
    free(p->node_to_dyn); free(p->rhs); free(p->minv); free(p->dv); free(p->mass); free(p->force);
    p->node_to_dyn = NULL; p->rhs = NULL; p->minv = NULL; p->dv = NULL; p->mass = NULL; p->force = NULL;
    p->dyn_count = 0;
}

PKO_EXPORT void PKO(destroy)(void* h)
{
    problem_t* p = (problem_t*)h;
    if (!p) return;
    clear_last(p);
    free(p->tets); free(p->b); free(p->d); free(p->body_tet_start); free(p->body_node_start);
    free(p->body_density); free(p->fixed); free(p->active);
    free(p);
}

PKO_EXPORT void PKO(set_settings)(void* h, const real* gravity3, int max_iterations, real tolerance,
                                  int use_jacobi, int linear)
{
    problem_t* p = (problem_t*)h;
    p->gravity = V3(gravity3[0], gravity3[1], gravity3[2]);
    p->max_iterations = max_iterations;
    p->tolerance = tolerance;
    p->use_jacobi = use_jacobi;
    p->linear = linear;
}

PKO_EXPORT void PKO(set_node_flags)(void* h, const unsigned char* fixed, const unsigned char* active)
{
    problem_t* p = (problem_t*)h;
    for (int i = 0; i < p->node_count; ++i) {
        p->fixed[i] = fixed ? fixed[i] : 0;
        p->active[i] = active ? active[i] : 1;
    }
}

PKO_EXPORT void PKO(set_tet_active)(void* h, const unsigned char* tet_active)
{
    problem_t* p = (problem_t*)h;
    for (int t = 0; t < p->tet_count; ++t) p->tets[t].active = tet_active[t];
}

/* Per-element Young's modulus, as a C++ caller sets Tet::youngModulus and calls
 * TetMeshPhysicsComponent::RebuildTetFemCache (TetMeshPhysicsComponent.cpp:211-219). */
PKO_EXPORT void PKO(set_tet_young)(void* h, const real* young)
{
    problem_t* p = (problem_t*)h;
    for (int t = 0; t < p->tet_count; ++t) {
        p->tets[t].young = young[t];
        tet_fem_cache(&p->tets[t], p->b[t], p->d[t]);
    }
}

/* Growable list helpers */
typedef struct { int node; v3 f; } force_e;
typedef struct { int node; real m; } mass_e;
typedef struct { int a, b; m3 k; } block_e;
typedef struct { void* p; long n, cap; size_t sz; } list_t;
static void* list_push(list_t* l)
{
    if (l->n == l->cap) {
        l->cap = l->cap ? l->cap * 2 : 1024;
        l->p = realloc(l->p, l->sz * (size_t)l->cap);
    }
    return (char*)l->p + l->sz * (size_t)(l->n++);
}

/* Open-addressing set of (row, col) keys for the lower-block skip of
 * SolverData::AssembleImplicitMatrixAndRhs (SolverData.cpp:318-319, 384-385, 438-444). */
typedef struct { uint64_t* k; long cap; } kset_t;
static uint64_t mix64(uint64_t x)
{
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return x;
}
static void kset_init(kset_t* s, long n)
{
    s->cap = 16;
    while (s->cap < 2 * n + 16) s->cap <<= 1;
    s->k = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)s->cap);
    memset(s->k, 0xff, sizeof(uint64_t) * (size_t)s->cap);
}
static void kset_put(kset_t* s, uint64_t key)
{
    long i = (long)(mix64(key) & (uint64_t)(s->cap - 1));
    while (s->k[i] != ~0ULL && s->k[i] != key) i = (i + 1) & (s->cap - 1);
    s->k[i] = key;
}
static int kset_has(const kset_t* s, uint64_t key)
{
    long i = (long)(mix64(key) & (uint64_t)(s->cap - 1));
    while (s->k[i] != ~0ULL) {
        if (s->k[i] == key) return 1;
        i = (i + 1) & (s->cap - 1);
    }
    return 0;
}

/* One World::Step(dt) with one substep in implicit mode, on (x, v) in place.
 * Returns 0 on success, -1 if a non-fixed active node had no mass (the reference
 * throws std::runtime_error from World::ValidateNodeMasses, World.cpp:560-580). */
PKO_EXPORT int PKO(step)(void* h, real* x_io, real* v_io, real dt)
{
    problem_t* p = (problem_t*)h;
    clear_last(p);
    p->precompute_ok = 0; p->solved = 0; p->integrated = 0; p->mass_error = 0;
    memset(&p->cg, 0, sizeof(p->cg));
    const int nn = p->node_count;
    v3* x = (v3*)x_io;
    v3* v = (v3*)v_io;
    list_t forces = {0, 0, 0, sizeof(force_e)};
    list_t masses = {0, 0, 0, sizeof(mass_e)};
    list_t blocks = {0, 0, 0, sizeof(block_e)};
    contrib_t c;

    /* Components in execution order: TetMeshPhysicsComponent::UpdateSystem per body. */
    for (int bi = 0; bi < p->body_count; ++bi) {
        int t0 = p->body_tet_start[bi], t1 = p->body_tet_start[bi + 1];
        /* ComputeLumpedMass + ApplyMassContribution (FEMModel.cpp:681-713, TMPC.cpp:127-152) */
        real density = p->body_density[bi] > R(0.0) ? p->body_density[bi] : R(0.0);
        if (isfinite(density))
            for (int t = t0; t < t1; ++t) {
                tet_t* tt = &p->tets[t];
                if (!tt->active || !isfinite(tt->rest_volume) || tt->rest_volume <= R(0.0)) continue;
                real nodal = density * tt->rest_volume * R(0.25);
                if (!isfinite(nodal) || nodal <= R(0.0)) continue;
                for (int a = 0; a < 4; ++a) {
                    int g = tt->n[a];
                    if (g < 0 || g >= nn || p->fixed[g]) continue;
                    mass_e* e = (mass_e*)list_push(&masses);
                    e->node = g; e->m = nodal;
                }
            }
        /* Component BSR over world nodes: pattern from all tets (TMPC.cpp:36-60, 221-232). */
        long pc = (long)(t1 - t0) * 16;
        int* pr = (int*)malloc(sizeof(int) * (size_t)(pc > 0 ? pc : 1));
        int* pcl = (int*)malloc(sizeof(int) * (size_t)(pc > 0 ? pc : 1));
        long q = 0;
        for (int t = t0; t < t1; ++t)
            for (int a = 0; a < 4; ++a)
                for (int b2 = 0; b2 < 4; ++b2) { pr[q] = p->tets[t].n[a]; pcl[q] = p->tets[t].n[b2]; ++q; }
        bsr_t fem = {0};
        bsr_build(&fem, nn, pr, pcl, q);
        free(pr); free(pcl);
        /* FEM forces/stiffness (FEMModel.cpp:580-612, 635-679) + ApplyElementContribution (TMPC.cpp:78-125) */
        for (int t = t0; t < t1; ++t) {
            tet_t* tt = &p->tets[t];
            if (!tt->active || tt->rest_volume <= R(0.0)) continue;
            if (p->linear) {
                element_contribution(tt, p->b[t], p->d[t], x, v, NULL, &c);
            } else {
                m3 ds = mcols(vsub(x[tt->n[1]], x[tt->n[0]]), vsub(x[tt->n[2]], x[tt->n[0]]),
                              vsub(x[tt->n[3]], x[tt->n[0]]));
                m3 fgrad = mmul(ds, tt->dm_inv);
                if (!mfinite(fgrad)) continue;
                m3 rot = polar_rotation(fgrad, NULL);
                element_contribution(tt, p->b[t], p->d[t], x, v, &rot, &c);
            }
            for (int a = 0; a < 4; ++a) {
                force_e* e = (force_e*)list_push(&forces);
                e->node = tt->n[a]; e->f = c.f[a];
            }
            for (int ra = 0; ra < 4; ++ra)
                for (int cb = 0; cb < 4; ++cb)
                    if (tt->n[ra] <= tt->n[cb]) bsr_add(&fem, tt->n[ra], tt->n[cb], c.k[ra][cb]);
        }
        /* Re-emit every stored block as (r,c,B) and (c,r,B^T) (TMPC.cpp:62-76, 341-353). */
        for (int r = 0; r < fem.n; ++r)
            for (int k = fem.row_start[r]; k < fem.row_start[r + 1]; ++k) {
                block_e* e = (block_e*)list_push(&blocks);
                e->a = r; e->b = fem.col[k]; e->k = fem.val[k];
                if (r != fem.col[k]) {
                    e = (block_e*)list_push(&blocks);
                    e->a = fem.col[k]; e->b = r; e->k = mtrans(fem.val[k]);
                }
            }
        bsr_free(&fem);
    }

    /* SolverData::AssembleMasses (SolverData.cpp:87-101) */
    p->mass = (real*)calloc((size_t)nn + 1, sizeof(real));
    for (long i = 0; i < masses.n; ++i) {
        mass_e* e = (mass_e*)masses.p + i;
        if (e->node < 0 || e->node >= nn || !isfinite(e->m) || e->m <= R(0.0)) continue;
        p->mass[e->node] += e->m;
    }
    /* World::ValidateNodeMasses (World.cpp:560-580) */
    for (int i = 0; i < nn; ++i) {
        if (!p->active[i] || p->fixed[i]) continue;
        if (isfinite(p->mass[i]) && p->mass[i] > R(0.0)) continue;
        p->mass_error = 1;
        free(forces.p); free(masses.p); free(blocks.p);
        return -1;
    }
    /* World::AddGravityForces (World.cpp:582-600) */
    for (int i = 0; i < nn; ++i) {
        if (!p->active[i] || p->fixed[i]) continue;
        if (!isfinite(p->mass[i]) || p->mass[i] <= R(0.0)) continue;
        force_e* e = (force_e*)list_push(&forces);
        e->node = i; e->f = vmul(p->gravity, p->mass[i]);
    }

    /* SolverData::PrecomputeImplicitSolve (SolverData.cpp:126-167) */
    p->force = (v3*)calloc((size_t)nn + 1, sizeof(v3));
    for (long i = 0; i < forces.n; ++i) {
        force_e* e = (force_e*)forces.p + i;
        if (e->node < 0 || e->node >= nn || !vfinite(e->f)) continue;
        p->force[e->node] = vadd(p->force[e->node], e->f);
    }
    p->node_to_dyn = (int*)malloc(sizeof(int) * (size_t)(nn + 1));
    int dyn = 0;
    if (dt > R(0.0)) {
        /* BuildDynamicNodeMapping (SolverData.cpp:239-258) */
        for (int i = 0; i < nn; ++i) {
            p->node_to_dyn[i] = -1;
            if (p->active[i] && !p->fixed[i] && isfinite(p->mass[i]) && p->mass[i] > R(0.0))
                p->node_to_dyn[i] = dyn++;
        }
    } else {
        for (int i = 0; i < nn; ++i) p->node_to_dyn[i] = -1;
    }
    p->dyn_count = dyn;
    int ok = dyn > 0 && dt > R(0.0);
    if (ok) {
        /* AssembleImplicitMatrixAndRhs (SolverData.cpp:308-465) */
        p->rhs = (v3*)calloc((size_t)dyn, sizeof(v3));
        int* cr = (int*)malloc(sizeof(int) * (size_t)(dyn + blocks.n + 1));
        int* cc = (int*)malloc(sizeof(int) * (size_t)(dyn + blocks.n + 1));
        long nc = 0;
        for (int i = 0; i < nn; ++i)
            if (p->node_to_dyn[i] >= 0) { cr[nc] = p->node_to_dyn[i]; cc[nc] = p->node_to_dyn[i]; ++nc; }
        kset_t dset;
        kset_init(&dset, blocks.n);
        real scale = dt * dt;
        for (long i = 0; i < blocks.n && ok; ++i) {
            block_e* e = (block_e*)blocks.p + i;
            if (e->a < 0 || e->a >= nn || e->b < 0 || e->b >= nn) continue;
            int rb = p->node_to_dyn[e->a];
            if (rb < 0) continue;
            if (!mfinite(e->k)) { ok = 0; break; }
            v3 cv = v[e->b];
            if (!vfinite(cv)) { ok = 0; break; }
            v3 kv = mvec(e->k, cv);
            if (!vfinite(kv)) { ok = 0; break; }
            p->rhs[rb] = vsub(p->rhs[rb], vmul(kv, scale));
            int cb = p->node_to_dyn[e->b];
            if (cb < 0) continue;
            kset_put(&dset, ((uint64_t)(uint32_t)rb << 32) | (uint32_t)cb);
            cr[nc] = rb; cc[nc] = cb; ++nc;
        }
        if (ok) {
            bsr_build(&p->a, dyn, cr, cc, nc);
            for (int i = 0; i < nn; ++i) {
                int d = p->node_to_dyn[i];
                if (d < 0) continue;
                real m = p->mass[i];
                bsr_add(&p->a, d, d, mcols(V3(m, 0, 0), V3(0, m, 0), V3(0, 0, m)));
            }
            for (long i = 0; i < blocks.n; ++i) {
                block_e* e = (block_e*)blocks.p + i;
                if (e->a < 0 || e->a >= nn || e->b < 0 || e->b >= nn || !mfinite(e->k)) continue;
                int rb = p->node_to_dyn[e->a], cb = p->node_to_dyn[e->b];
                if (rb < 0 || cb < 0) continue;
                if (rb > cb && kset_has(&dset, ((uint64_t)(uint32_t)cb << 32) | (uint32_t)rb)) continue;
                bsr_add(&p->a, rb, cb, mscale(e->k, scale));
            }
            for (int i = 0; i < nn; ++i) {
                int d = p->node_to_dyn[i];
                if (d < 0) continue;
                p->rhs[d] = vadd(p->rhs[d], vmul(p->force[i], dt));
            }
        }
        free(dset.k); free(cr); free(cc);
    }
    p->precompute_ok = ok;
    free(forces.p); free(masses.p); free(blocks.p);

    /* SolverData::SolveImplicitLinearSystem (SolverData.cpp:169-212) */
    int solved = 0;
    if (ok && dyn > 0) {
        /* BuildInversePreconditioner (SolverData.cpp:260-306) */
        p->minv = (m3*)malloc(sizeof(m3) * (size_t)dyn);
        int pre_ok = 1;
        for (int i = 0; i < dyn; ++i) p->minv[i] = mident();
        if (p->use_jacobi)
            for (int i = 0; i < dyn && pre_ok; ++i) {
                int k = bsr_find(&p->a, i, i);
                if (k < 0) { pre_ok = 0; break; }
                m3 db = p->a.val[k];
                if (!mfinite(db)) { pre_ok = 0; break; }
                real det = mdet(db);
                if (!isfinite(det) || fabs((double)det) <= (double)R(1.0e-8)) { pre_ok = 0; break; }
                m3 inv = minv(db);
                if (!mfinite(inv)) { pre_ok = 0; break; }
                p->minv[i] = inv;
            }
        if (pre_ok) {
            p->dv = (v3*)calloc((size_t)dyn, sizeof(v3));
            int have = pcg_solve(&p->a, p->rhs, dyn, p->max_iterations, p->tolerance, p->minv, dyn, p->dv, &p->cg);
            solved = have;
            if (have)
                for (int i = 0; i < dyn; ++i) if (!vfinite(p->dv[i])) { solved = 0; break; }
        }
    }
    p->solved = solved;

    /* World::IntegrateImplicitEuler (World.cpp:644-695): all or nothing. */
    if (solved) {
        int fine = 1;
        for (int i = 0; i < nn && fine; ++i) {
            int d = p->node_to_dyn[i];
            if (d < 0) continue;
            v3 nv = vadd(v[i], p->dv[d]);
            v3 nx = vadd(x[i], vmul(nv, dt));
            if (!vfinite(x[i]) || !vfinite(v[i]) || !vfinite(p->dv[d]) || !vfinite(nv) || !vfinite(nx)) fine = 0;
        }
        if (fine) {
            for (int i = 0; i < nn; ++i) {
                int d = p->node_to_dyn[i];
                if (d < 0) continue;
                v3 nv = vadd(v[i], p->dv[d]);
                x[i] = vadd(x[i], vmul(nv, dt));
                v[i] = nv;
            }
            p->integrated = 1;
        }
    }
    return 0;
}

/* ------------------------------------------------------------ inspection */
PKO_EXPORT void PKO(last_sizes)(void* h, int* dyn, int* nnz, int* cg_iterations, double* cg_residual,
                                int* cg_converged, int* flags)
{
    problem_t* p = (problem_t*)h;
    if (dyn) *dyn = p->dyn_count;
    if (nnz) *nnz = p->a.nnz;
    if (cg_iterations) *cg_iterations = p->cg.iterations;
    if (cg_residual) *cg_residual = p->cg.residual_norm;
    if (cg_converged) *cg_converged = p->cg.converged;
    if (flags) *flags = (p->precompute_ok ? 1 : 0) | (p->solved ? 2 : 0) | (p->integrated ? 4 : 0) |
                        (p->mass_error ? 8 : 0);
}

/* Copies the last assembled system.  Any pointer may be NULL. */
PKO_EXPORT void PKO(last_system)(void* h, int* row_start, int* col, real* values, real* rhs, real* minv_out,
                                 real* dv, int* node_to_dyn, real* mass, real* force)
{
    problem_t* p = (problem_t*)h;
    if (row_start && p->a.row_start) memcpy(row_start, p->a.row_start, sizeof(int) * (size_t)(p->a.n + 1));
    if (col && p->a.col) memcpy(col, p->a.col, sizeof(int) * (size_t)p->a.nnz);
    if (values && p->a.val) memcpy(values, p->a.val, sizeof(m3) * (size_t)p->a.nnz);
    if (rhs && p->rhs) memcpy(rhs, p->rhs, sizeof(v3) * (size_t)p->dyn_count);
    if (minv_out && p->minv) memcpy(minv_out, p->minv, sizeof(m3) * (size_t)p->dyn_count);
    if (dv && p->dv) memcpy(dv, p->dv, sizeof(v3) * (size_t)p->dyn_count);
    if (node_to_dyn && p->node_to_dyn) memcpy(node_to_dyn, p->node_to_dyn, sizeof(int) * (size_t)p->node_count);
    if (mass && p->mass) memcpy(mass, p->mass, sizeof(real) * (size_t)p->node_count);
    if (force && p->force) memcpy(force, p->force, sizeof(v3) * (size_t)p->node_count);
}

/* Per-tet rest data: volume, DmInv (column-major 9), shape gradients (4x3). */
PKO_EXPORT void PKO(tet_rest)(void* h, real* volume, real* dm_inv, real* grads)
{
    problem_t* p = (problem_t*)h;
    for (int t = 0; t < p->tet_count; ++t) {
        if (volume) volume[t] = p->tets[t].rest_volume;
        if (dm_inv) memcpy(dm_inv + 9 * t, &p->tets[t].dm_inv, sizeof(m3));
        if (grads) memcpy(grads + 12 * t, p->tets[t].grad, sizeof(v3) * 4);
    }
}

/* ------------------------------------------------------- standalone kernels */
/* y = A x for an upper-stored symmetric BSR (SparseBlockMatrix.cpp:209-268). */
PKO_EXPORT void PKO(bsr_multiply)(int n, const int* row_start, const int* col, const real* values, const real* x,
                                  real* y)
{
    bsr_t a;
    a.n = n; a.row_start = (int*)row_start; a.col = (int*)col; a.val = (m3*)values; a.nnz = row_start[n];
    bsr_mul(&a, (const v3*)x, (v3*)y);
}

/* SolvePreconditionedConjugateGradient on caller arrays; returns 1 if x was filled. */
PKO_EXPORT int PKO(pcg)(int n, const int* row_start, const int* col, const real* values, const real* b,
                        const real* minv_blocks, int minv_count, int max_iterations, real tolerance, real* x,
                        int* iterations, double* residual_norm, int* converged)
{
    bsr_t a;
    a.n = n; a.row_start = (int*)row_start; a.col = (int*)col; a.val = (m3*)values;
    a.nnz = n > 0 ? row_start[n] : 0;
    pko_cg_result res;
    int have = pcg_solve(&a, (const v3*)b, n, max_iterations, tolerance, (const m3*)minv_blocks, minv_count,
                         (v3*)x, &res);
    if (iterations) *iterations = res.iterations;
    if (residual_norm) *residual_norm = res.residual_norm;
    if (converged) *converged = res.converged;
    return have;
}

/* Builds the canonical upper pattern of BuildPattern from coordinate lists.
 * Returns nnz; row_start (n+1) and col (capacity cap) are filled when non-NULL. */
PKO_EXPORT int PKO(build_pattern)(int n, const int* rows, const int* cols, long count, int* row_start, int* col,
                                  int cap)
{
    bsr_t a = {0};
    bsr_build(&a, n, rows, cols, count);
    int nnz = a.nnz;
    if (row_start && a.row_start) memcpy(row_start, a.row_start, sizeof(int) * (size_t)(n + 1));
    if (col && a.col && nnz <= cap) memcpy(col, a.col, sizeof(int) * (size_t)nnz);
    bsr_free(&a);
    return nnz;
}

/* ExtractRotationPolar on one column-major 3x3. */
PKO_EXPORT void PKO(polar)(const real* f9, real* r9, int* iterations)
{
    m3 f;
    memcpy(&f, f9, sizeof(m3));
    m3 r = polar_rotation(f, iterations);
    memcpy(r9, &r, sizeof(m3));
}
