/*
 * pkcuda.h -- the thin C ABI over the sm_100a kernels of PhysiK's implicit
 * soft-body step.  Plain pointers and sizes, an int status on every call, one CUDA
 * stream per system.  The C++ host layer (World, TetMeshPhysicsComponent,
 * SolverData, SparseBlockMatrix, SolvePreconditionedConjugateGradient) calls these;
 * tests call them directly for kernel-level parity.
 *
 * Reference interfaces each entry point replaces (paths inside mauriciomedg/PhysiK):
 *   pk_system_step        one implicit substep: FEMModel::ComputeCorotationalElasticForces
 *                         (src/Core/Physics/FEM/FEMModel.cpp:635-679) + TetMeshPhysicsComponent::
 *                         UpdateSystem (src/Components/TetMeshPhysicsComponent.cpp:293-354) +
 *                         SolverData::PrecomputeImplicitSolve / SolveImplicitLinearSystem
 *                         (src/Core/Solvers/SolverData.cpp:126-212) + World::IntegrateImplicitEuler
 *                         (src/Core/World/World.cpp:644-695); explicit mode replaces
 *                         World::IntegrateExplicitEuler (World.cpp:697-725)
 *   pk_bsr_multiply       SparseBlockMatrix::Multiply (src/Math/SparseBlockMatrix.cpp:209-268)
 *   pk_pcg                SolvePreconditionedConjugateGradient
 *                         (src/Core/Solvers/Linear/ConjugateGradientSolver.cpp:114-241,
 *                          include/PhysiK/Core/Solvers/Linear/ConjugateGradientSolver.h:26-35)
 *   pk_system_get_state_* / set_state_*   World::GetNodePosition / GetNodeVelocity and the
 *                         PHYSIK_Get/SetNodePosition/Velocity accessors (src/API/PhysiKAPI.cpp:1477-1558),
 *                         in bulk
 *
 * Threading: calls on one pk_system must be serialised by the caller (as the
 * reference's World is single-threaded).  Steps are asynchronous on the system's
 * stream; pk_system_stats and the get_* calls wait for it.
 */
#ifndef PKCUDA_H
#define PKCUDA_H

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define PKCUDA_API __attribute__((visibility("default")))
#else
#define PKCUDA_API
#endif

/* Precision of a system: storage / accumulation. */
#define PK_PREC_FP32 0  /* float storage, float dot products (the reference's scalar type) */
#define PK_PREC_MIXED 1 /* float storage, double CG scalars and updates, double polar for near-inverted tets */
#define PK_PREC_FP64 2  /* double everywhere */

/* Return codes. */
#define PK_OK 0
#define PK_ERR_NO_DEVICE (-1)   /* no usable CUDA device */
#define PK_ERR_CUDA (-2)        /* a CUDA call failed: pk_last_error() */
#define PK_ERR_ARG (-3)         /* invalid argument */
#define PK_ERR_STATE (-4)       /* call out of order (e.g. a step before the topology) */
#define PK_ERR_UNSUPPORTED (-5) /* a size the kernels were not built for */
#define PK_ERR_TIMEOUT (-6)     /* a grid barrier gave up waiting; the step was not applied */

/* Step flags, reported in pk_step_stats.flags. */
#define PK_FLAG_PRECOMPUTE_FAILED 0x1u /* non-finite velocity / stiffness block / rhs: no solve (SolverData.cpp:353-373) */
#define PK_FLAG_SINGULAR_DIAG 0x2u     /* a diagonal block with |det| <= 1e-8 or non-finite (SolverData.cpp:284-303) */
#define PK_FLAG_INVALID_RHS 0x4u       /* non-finite rhs or invalid settings: solution cleared (ConjugateGradientSolver.cpp:137-149) */
#define PK_FLAG_BREAKDOWN 0x8u         /* d.q <= 0 or a non-finite CG scalar: iteration stopped early */
#define PK_FLAG_NONFINITE_DV 0x10u     /* delta-v not finite: solve reported failure (SolverData.cpp:203-209) */
#define PK_FLAG_INTEGRATE_ABORT 0x20u  /* integration would produce non-finite state: not applied (World.cpp:667-677) */
#define PK_FLAG_POLAR_IDENTITY 0x40u   /* some polar decomposition fell back to the identity */
#define PK_FLAG_POLAR_FP64 0x80u       /* some near-inverted tet used the double-precision polar (mixed mode) */
#define PK_FLAG_BARRIER_TIMEOUT 0x100u /* a grid barrier timed out */
#define PK_FLAG_ROW_TOO_LONG 0x200u    /* internal: a row exceeded the row kernel's slot count */
#define PK_FLAG_SOLVED 0x1000u         /* SolveImplicitLinearSystem would return true */
#define PK_FLAG_INTEGRATED 0x2000u     /* positions and velocities were advanced */
#define PK_FLAG_CONVERGED 0x4000u      /* CG met its relative tolerance */
#define PK_FLAG_REFINED_FP64 0x8000u   /* the refinement measured the FP64 system element by element */

typedef struct pk_step_params {
    double dt;               /* substep size (World::Step divides the frame by the substep count) */
    double gravity[3];
    int max_iterations;      /* ConjugateGradientSettings::maxIterations */
    double tolerance;        /* ConjugateGradientSettings::tolerance (relative, preconditioned) */
    int use_jacobi;          /* ConjugateGradientSettings::useJacobiPreconditioner */
    int linear;              /* 1: FemModel::Linear (R = I), 0: FemModel::Corotational */
    int explicit_mode;       /* 1: SolverMode::Explicit, 0: SolverMode::ImplicitEuler */
    int integrate;           /* 0: assemble and solve only (delta-v stays on the device) */
} pk_step_params;

typedef struct pk_step_stats {
    int iterations;          /* ConjugateGradientResult::iterations */
    int converged;           /* ConjugateGradientResult::converged */
    double residual_norm;    /* ConjugateGradientResult::residualNorm = ||r||_2 */
    unsigned flags;          /* PK_FLAG_* */
    int polar_fp64_count;
    int polar_identity_count;
} pk_step_stats;

typedef struct pk_cg_result {
    int iterations;
    int converged;
    double residual_norm;
    int have_solution;       /* 0 when the reference would have cleared the solution vector */
} pk_cg_result;

typedef struct pk_system pk_system;

PKCUDA_API const char* pk_last_error(void);
PKCUDA_API int pk_device_count(void);

PKCUDA_API int pk_system_create(int device, int precision, pk_system** out);
PKCUDA_API int pk_system_destroy(pk_system* sys);
PKCUDA_API void* pk_system_stream(pk_system* sys);

/* Nodes in world order: node_to_dyn[i] is node i's dynamic row or -1; mass[i] the
 * assembled lumped mass (SolverData::AssembleMasses order).  Resets state to zero. */
PKCUDA_API int pk_system_set_nodes(pk_system* sys, int node_count, const int* node_to_dyn, const double* mass);
/* New lumped masses for the same nodes (after tets were deactivated or a material changed,
 * with the dynamic-row map unchanged); the nodes' state is kept. */
PKCUDA_API int pk_system_set_masses(pk_system* sys, const double* mass);
/* Either pointer may be NULL.  3*node_count values each. */
PKCUDA_API int pk_system_set_state_f32(pk_system* sys, const float* x, const float* v);
PKCUDA_API int pk_system_set_state_f64(pk_system* sys, const double* x, const double* v);
PKCUDA_API int pk_system_get_state_f32(pk_system* sys, float* x, float* v);
PKCUDA_API int pk_system_get_state_f64(pk_system* sys, double* x, double* v);
/* Copies the node positions, on the device and in stream order, into a snapshot buffer
 * (the host calls it at the end of every frame: TetMeshPhysicsComponent::PostUpdate's
 * SyncCurrentPositionsFromWorld, TetMeshPhysicsComponent.cpp:234-252, 356-363, keeps the
 * positions a component's GetLocalCurrentPosition returns, TetMeshComponent.cpp:113-122).
 * pk_system_get_snapshot_f32 reads nodes [first_node, first_node + count) of the last
 * snapshot (3 floats each) and waits for the stream. */
PKCUDA_API int pk_system_snapshot_positions(pk_system* sys);
/* The tets (of those set with flag bit 2, "active") whose centroid lies strictly inside the
 * sphere (center[3], radius), at the current node positions -- CollisionSphereComponent::
 * UpdateSystem's test (CollisionSphereComponent.cpp:141-190): centroid = ((x0/4 + x1/4) +
 * x2/4) + x3/4 and |centroid - center| computed in the state's precision with every
 * operation rounded once.  Writes up to max_contacts tet indices (ascending) and their
 * centroids (3 each); returns the number of contacts (when above max_contacts nothing is
 * written), or a negative PK_ERR_*.  Waits for the stream. */
PKCUDA_API int pk_system_sphere_contacts(pk_system* sys, const double* center, double radius, int max_contacts,
                                         int* tets, double* points);
PKCUDA_API int pk_system_get_snapshot_f32(pk_system* sys, int first_node, int count, float* x);

/* FP64 rest data and lumped masses of an FP32-stored system (FP32 or mixed precision):
 * DmInv (9 per tet, column-major), rest volume, lambda, mu, damping per tet and the mass
 * per world node, computed in FP64 from the same inputs (FEMModel::InitializeTetRestData,
 * FEMModel.cpp:504-548; BuildElasticityMatrix's lambda and mu; the lumped mass rho V / 4).
 * With them the refinement (pk_system_set_refinement) measures the residual of the FP64
 * system element by element instead of over the FP32-stored blocks, when the system has
 * no point connections and no host-emitted blocks.  Must follow pk_system_set_tets and
 * pk_system_set_nodes (the counts must match); those and pk_system_set_masses drop it. */
PKCUDA_API int pk_system_set_rest64(pk_system* sys, int tet_count, const double* dm_inv, const double* volume,
                                    const double* lambda, const double* mu, const double* damping, int node_count,
                                    const double* mass);

/* Post-step geometry on the device, read back only when asked for.
 * kind 0, surface triangles (SurfaceVisualComponent::UpdateVisualSurfaceGeometry,
 *   SurfaceVisualComponent.cpp:150-213): `count` triangles of 3 world nodes each; an update
 *   writes per triangle its 3 vertices (the node positions) and its flat normal
 *   Cross(p1 - p0, p2 - p0) / length ((0, 1, 0) when the length is at most 1e-6) for
 *   each of them (9 + 9 floats).
 * kind 1, embedded vertices (VisualMeshComponent::UpdateDeformedVertices,
 *   VisualMeshComponent.cpp:257-333): `count` vertices with 4 world nodes and 4 weights
 *   each; an update writes ((x0 w0 + x1 w1) + x2 w2) + x3 w3 for the vertices marked live,
 *   the others keep their value (`initial` at creation; 3 floats per vertex).
 * Updates read the current positions or the frame-end snapshot
 * (pk_system_snapshot_positions), on the system's stream, rounded to float (the copies the
 * components hold), every operation a float operation rounded once.  An update fails with
 * PK_ERR_STATE when a node id is beyond the system's node count.  The visual keeps its own
 * device buffers; pk_visual_read copies them to the host (normals: kind 0 only, may be
 * NULL) and waits for the stream. */
typedef struct pk_visual pk_visual;
PKCUDA_API int pk_visual_create(pk_system* sys, int kind, int count, const int* nodes, const float* weights,
                                const float* initial, const unsigned char* live, pk_visual** out);
PKCUDA_API int pk_visual_set_live(pk_visual* visual, pk_system* sys, const unsigned char* live);
PKCUDA_API int pk_visual_update(pk_visual* visual, pk_system* sys, int from_snapshot);
PKCUDA_API int pk_visual_read(pk_visual* visual, pk_system* sys, float* vertices, float* normals);
PKCUDA_API int pk_visual_destroy(pk_visual* visual);

/* Tets with world node ids and rest data already computed in the system precision
 * (FEMModel::InitializeTetRestData, BuildElasticityMatrix's lambda and mu).
 * enabled[t]: bit 0 = tet active, rest volume > 0 and its body simulated; bit 1 = linear FEM
 * (FemModel::Linear, R = I) instead of corotated. */
PKCUDA_API int pk_system_set_tets(pk_system* sys, int tet_count, const int* tet_nodes, const unsigned char* enabled,
                                  const double* dm_inv, const double* volume, const double* lambda, const double* mu,
                                  const double* damping);

/* Dynamic rows: the canonical upper BSR of SolverData (row_start[dyn+1], col_index[nnz]),
 * the row -> world node map, and per row the incidence list of its node's tets
 * (entries t*4 + corner, ascending t). */
PKCUDA_API int pk_system_set_pattern(pk_system* sys, int dyn_count, const int* dyn_to_node, const int* row_start,
                                     const int* col_index, const int* inc_start, const int* inc_list);

/* Transient point connections for the next steps (PointConnection::UpdateSystem,
 * src/Core/PhysicsConnections/PointConnection.cpp:55-140), evaluated on the device during
 * assembly: nodes[4*count] world nodes; params[9*count] barycentric weights (4), target
 * position (3), stiffness, damping; per dynamic row the list of entries connection*4 +
 * corner whose corner node is that row and whose weight is non-zero, in connection order
 * (inc_start[dyn+1], inc_list).  The pattern must already hold the blocks the connections
 * couple (every pair of corners with non-zero weights whose rows are both dynamic), and
 * the caller drops connections whose nodes are inactive or whose stiffness or damping is
 * negative or not finite (World::HasValidNodeIndices and the checks of UpdateSystem).
 * count 0 removes them; set_pattern removes them too.  With connections present the
 * batched solve runs as one coupled solve and the adjoint step is refused. */
PKCUDA_API int pk_system_set_connections(pk_system* sys, int count, const int* nodes, const double* params,
                                         const int* inc_start, const int* inc_list);

/* Host-emitted contributions of custom components for the next steps (SolverData::
 * AddStiffnessBlock / AddNodeForce, SolverData.h:41-54, assembled as
 * SolverData::AssembleImplicitMatrixAndRhs does, SolverData.cpp:308-465): blocks[9*count]
 * (column-major) with block_nodes[2*count] {row node, column node}; per dynamic row the
 * blocks whose row node is that row (rhs_start[dyn+1], rhs_list: the rhs gets
 * -dt^2 B v_column) and the blocks it holds in its upper row (mat_start, mat_list: block
 * index, | 0x80000000 for the transpose of a lower block); row_force[3*dyn] the summed
 * node forces of each dynamic row (NULL: none).  Masses (AddNodeMass) enter the node
 * masses (pk_system_set_nodes / set_masses).  The pattern must hold the blocks; count 0
 * with row_force NULL removes them; set_pattern removes them too.  With blocks present the
 * batched solve runs as one coupled solve and the adjoint step is refused. */
PKCUDA_API int pk_system_set_extras(pk_system* sys, int block_count, const double* blocks, const int* block_nodes,
                                    const int* rhs_start, const int* rhs_list, const int* mat_start,
                                    const int* mat_list, const double* row_force);

/* Batched per-body solve (no counterpart in the reference, whose World solves all of its
 * bodies as one coupled system): the dynamic rows split into independent segments
 * (bodies) [segment_row_start[b], segment_row_start[b+1]), covering all rows, with no
 * block coupling two segments.  With batching on, pk_system_step runs one PCG per
 * segment -- own scalars, stopping test, iteration count and all-or-nothing integration,
 * as a reference World holding only that body -- all in one launch.  Step statistics then
 * report the largest iteration count, the largest residual, and success flags that hold
 * for every body.  Call set_segments after set_pattern (set_pattern clears them). */
PKCUDA_API int pk_system_set_segments(pk_system* sys, int segment_count, const int* segment_row_start);
PKCUDA_API int pk_system_set_batched(pk_system* sys, int on);
/* Per-segment statistics of the last batched step (waits); any pointer may be NULL. */
PKCUDA_API int pk_system_segment_stats(pk_system* sys, int segment_count, int* iterations, int* converged,
                                       double* residual_norm, unsigned* flags);

/* One substep, asynchronous on the system stream. */
PKCUDA_API int pk_system_step(pk_system* sys, const pk_step_params* params);
/* Waits for the last step and reports its statistics. */
PKCUDA_API int pk_system_stats(pk_system* sys, pk_step_stats* out);

/* The last assembled system (waits).  values: 9*nnz column-major; rhs, dv: 3*dyn;
 * minv: 9*dyn.  Any pointer may be NULL. */
PKCUDA_API int pk_system_get_system_f64(pk_system* sys, double* values, double* rhs, double* minv, double* dv);
/* Overwrites the matrix, rhs and inverse preconditioner (same layout) and runs only the
 * solve of pk_system_step (no assembly); used to drive the PCG on an exact system. */
PKCUDA_API int pk_system_solve_given_f64(pk_system* sys, const double* values, const double* rhs,
                                         const double* minv, const pk_step_params* params);

/* Device-event timing of the step's phases on the system stream. */
PKCUDA_API int pk_system_enable_timing(pk_system* sys, int on);
/* Accumulated since enable: assembly (tet + row kernels) and solve (PCG kernel) times in ms,
 * the number of timed steps, and the kernels launched. */
PKCUDA_API int pk_system_timings(pk_system* sys, double* assemble_ms, double* solve_ms, int* steps,
                                 long long* kernel_launches);
/* Grid size of the cooperative PCG launch (0 = automatic).  Returns the grid used next. */
PKCUDA_API int pk_system_set_pcg_grid(pk_system* sys, int grid);

/* Backward (adjoint) step of pk_system_step -- no counterpart in the reference.  With the
 * system at the state (x, v) a forward step starts from, and the loss sensitivities to
 * the state after that step (xbar_next, vbar_next: 3*node_count each, world order), it
 * writes the sensitivities to (x, v) (xbar, vbar) and ADDS each tet's sensitivity to its
 * log Young's modulus to theta_bar[tet] (may be NULL).  It re-runs the step's assembly and
 * solve (no integration, state unchanged), solves the adjoint system A w = g with the same
 * PCG (A is symmetric; the solve is treated as exact), and evaluates the element terms on
 * the GPU (pk_adjoint.cu).  The velocity sensitivity of fixed nodes is passed through
 * unchanged.  A batched system is differentiated as one coupled solve. */
PKCUDA_API int pk_system_adjoint_step(pk_system* sys, const pk_step_params* params, const double* xbar_next,
                                      const double* vbar_next, double* xbar, double* vbar, double* theta_bar);

/* FP64 outer true-residual refinement for FP32 storage (FP32 and mixed precision,
 * unbatched; no counterpart in the reference): after the step's PCG, while the true
 * residual b - A x computed with FP64 arithmetic over the assembled blocks misses the
 * reference's stopping target r^T M^-1 r <= tol^2 b^T M^-1 b and iterations remain of the
 * step's max_iterations, up to `passes` correction solves are run and added in FP64; the
 * update then uses the FP64 delta-v.  The step's statistics become the total iterations
 * and the true residual's convergence and norm.  0 (the default) turns it off.  Such
 * steps synchronise with the host and are not graph-captured. */
PKCUDA_API int pk_system_set_refinement(pk_system* sys, int passes);
/* The PCG kernel of the last solve: 0 ring-staged, 1 TMA-staged, 2 unstaged, 3
 * part-resident, 4 per-body batch kernel, 5 part-resident with one group of parts per body
 * (batched solve); -1 before the first solve (or a negative PK_ERR_*).
 * blocks (may be NULL) receives the blocks it ran on. */
PKCUDA_API int pk_system_pcg_kernel(pk_system* sys, int* blocks);
/* Stream form of the part-resident kernel's layout in the last solve: 0 full symmetric
 * rows, 1 the symmetric form (each in-sub-part block streamed once); -1 when the last
 * solve did not run on the part-resident kernel. */
PKCUDA_API int pk_system_slab_form(pk_system* sys);
/* Captures each step into a CUDA graph (relaxed capture mode) and replays it: the first
 * step after enabling runs normally (allocations, uploads), the next one with the same
 * parameters is captured, later ones launch the graph.  Any topology, segment, grid or
 * parameter change drops the graph.  With timing on, a graph step counts as solve time. */
PKCUDA_API int pk_system_set_graph(pk_system* sys, int on);
/* Autotuner: times `repeats` solves (without integration) of the last assembled system
 * for each candidate and keeps the fastest -- unbatched: the ring-staged kernel (0), the
 * TMA-staged kernel with 16 / 32 / 64-row tiles (1-3), the unstaged kernel (4), the
 * part-resident kernel (5, FP32 storage, where its layout applies); batched: the per-body
 * batch kernel with the smallest part (32 .. 1024 rows) a body is cut into (0-5), the
 * part-resident kernel with one group of parts per body (6, FP32 storage).  Needs one step first.  Reports the
 * candidate index and its mean solve time.  Candidates differ only in summation order. */
PKCUDA_API int pk_system_autotune(pk_system* sys, const pk_step_params* params, int repeats, int* chosen,
                                  double* best_ms);

/* Standalone kernels on host arrays (values column-major, 9 per block). */
PKCUDA_API int pk_bsr_multiply(int device, int precision, int n, const int* row_start, const int* col_index,
                               const double* values, const double* x, double* y);
PKCUDA_API int pk_pcg(int device, int precision, int n, const int* row_start, const int* col_index,
                      const double* values, const double* b, const double* minv, int minv_count, int max_iterations,
                      double tolerance, double* x, pk_cg_result* out);

/* The block-Jacobi PCG solve of pk_pcg on caller-owned DEVICE buffers, allocating nothing.
 * No counterpart in the reference: it serves callers that may not allocate device memory
 * while they solve (a game-engine plugin solving inside its frame loop under a fixed
 * memory budget, or a host that routes all device memory through its own pool).
 * Inputs: the upper BSR (row_start[n+1], col_index, values: 9 per block in the precision's
 * scalar type) with its transposed index from pk_bsr_transpose_index (lt_start[n+1],
 * lt_row, lt_block; a matrix without off-diagonal blocks passes 1-element lt_row /
 * lt_block buffers: every pointer must be non-NULL when n > 0), the rhs b (3n), the
 * block-Jacobi inverse minv (9n); output x (3n).
 * The CG working vectors live in one fixed 8 MiB array per GPU, held by every GPU that
 * loads the library until exit: at most 32,768 rows (PK_ERR_UNSUPPORTED above that).
 * All calls on a device share that array and it keeps the last call's contents (the call
 * clears what must start at zero); calls whose GPU work overlaps race on it.  The first
 * call on a device looks up the array's address, with that device current.  Every call
 * runs on `stream` of the current device and synchronises that stream to return the
 * statistics, so it must not be called while the stream is being captured into a graph. */
PKCUDA_API int pk_pcg_noalloc(int precision, int n, const int* row_start, const int* col_index, const void* values,
                              const int* lt_start, const int* lt_row, const int* lt_block, const void* b,
                              const void* minv, int max_iterations, double tolerance, void* x, pk_cg_result* out,
                              void* stream);
PKCUDA_API const char* pk_pcg_noalloc_last_error(void);

/* Device check of the bounded waits every PCG kernel's grid exchange makes: `blocks`
 * (2..64) co-resident blocks exchange two partial sums as a group of blocks + missing
 * members, each wait giving up after `limit` polls.  out (3 doubles per block) receives
 * {1 if the block's exchange succeeded else 0, sum of 1..blocks, blocks}.  Returns PK_OK
 * when every exchange completed; PK_ERR_TIMEOUT when a wait ran out (always, for
 * missing > 0) -- the launch still ends normally and the context stays usable.  No
 * counterpart in the reference (it checks this library's failure path). */
PKCUDA_API int pk_exchange_wait_selftest(int device, int blocks, int missing, unsigned long long limit, double* out);

/* Host-only consistency check of the ring-staged PCG kernel's tiling (no device needed):
 * builds its tiles for the upper BSR (values 9 per block, x 3 per row), replays the
 * kernel's shared-memory staging byte for byte and evaluates y = A x through the staged
 * data as the kernel's lanes index it.  Returns the number of index / span violations
 * (0 = consistent), or a negative PK_ERR_* code; tiles and max_span (may be NULL)
 * receive the tile count and the largest staged block span.  No counterpart in the
 * reference (it checks this library's own layout). */
PKCUDA_API int pk_ring_tiling_selfcheck(int precision, int n, const int* row_start, const int* col_index,
                                        const double* values, const double* x, double* y, int* tiles, int* max_span);

/* CPU self-check of the part-resident PCG kernel's layout: builds it for the upper BSR
 * (parts parts, cut by coords -- 3 doubles per row -- or, when coords is NULL, as
 * contiguous row ranges) in stream form `form` (0 full symmetric rows, 1 the symmetric
 * form that streams each in-part block once, 2 the symmetric form where it applies),
 * fills the block stream as the device fill does (float storage) and evaluates y = A x by
 * decoding the tiles exactly as the kernel's lanes read them (for the symmetric form
 * with its per-group rings of transposed products, wrap-around included).  info (may be
 * NULL) receives {parts, largest window, most tiles in a part, stream KiB, 1 if the
 * symmetric form was built}.  PK_ERR_UNSUPPORTED when the layout does not apply (a
 * window or a row too large, or for the symmetric form a ring too small).  No
 * counterpart in the reference (it checks this library's own layout). */
PKCUDA_API int pk_slab_plan_selfcheck(int n, const int* row_start, const int* col_index, const double* values,
                                      const double* x, const double* coords, int parts, int form, double* y,
                                      int* info);

/* The same for the per-body (batched) layout: rows in segments (bodies), every body cut
 * into parts that fit, bodies packed into launches of at most max_blocks parts; also
 * checks that every part's group is its body's consecutive parts within one launch.
 * info (may be NULL) receives {parts, largest window, most tiles in a part, stream KiB,
 * launches, 1 if the symmetric form was built}. */
PKCUDA_API int pk_slab_plan_batched_selfcheck(int n, const int* row_start, const int* col_index, const double* values,
                                              const double* x, const double* coords, const int* segment_row_start,
                                              int segment_count, int max_blocks, int form, double* y, int* info);

/* Builds the transposed index of an upper BSR: for row r the blocks (c, r), c < r.
 * lt_start[n+1]; lt_row / lt_block sized nnz - n.  Host-only, no device needed. */
PKCUDA_API int pk_bsr_transpose_index(int n, const int* row_start, const int* col_index, int* lt_start, int* lt_row,
                                      int* lt_block);

#ifdef __cplusplus
}
#endif

#endif /* PKCUDA_H */
