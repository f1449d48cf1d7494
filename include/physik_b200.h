/*
 * physik_b200.h -- the drop-in C ABI of PhysiK's soft-body step, backed by sm_100a
 * kernels.  The PHYSIK_* functions below keep the names, argument types and error
 * behaviour of the reference's Unity-facing API (include/PhysiK/API/PhysiKAPI.h) for
 * the implicit soft-body path, so a P/Invoke or ctypes binding written against the
 * reference binds unchanged.  Each declaration cites the reference function it
 * replaces (file:line in mauriciomedg/PhysiK).
 *
 * Error conventions kept from the reference: a NULL world is a silent no-op, getters
 * return 0 / -1 / an invalid handle, out-pointers are written only when non-NULL.
 * One deliberate difference: the reference lets World::ValidateNodeMasses throw
 * std::runtime_error through PHYSIK_Step (src/Core/World/World.cpp:576-578); here the
 * C ABI catches every exception at the boundary, leaves the state unchanged and
 * records the message for PHYSIK_B200_GetLastError.
 *
 * PHYSIK_B200_* functions are extensions with no counterpart in the reference.
 */
#ifndef PHYSIK_B200_H
#define PHYSIK_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define PHYSIK_B200_API __attribute__((visibility("default")))
#else
#define PHYSIK_B200_API
#endif

typedef void* PhysikWorldHandle;            /* PhysiK::WorldHandle (include/PhysiK/API/Handles.h:7) */
typedef void* PhysikGeneratedTetMeshHandle; /* PhysiK::GeneratedTetMeshHandle (Handles.h:8) */

/* PhysiK::ComponentHandle (Handles.h:10-19): index 0xFFFFFFFF or generation 0 is invalid. */
typedef struct PhysikComponentHandle {
    uint32_t index;
    uint32_t generation;
} PhysikComponentHandle;

/* PhysikMaterialDesc (include/PhysiK/API/PhysiKAPI.h:16-22) */
typedef struct PhysikMaterialDesc {
    float density;
    float youngModulus;
    float poissonRatio;
    float damping;
} PhysikMaterialDesc;

/* PhysiK::ExternalLogicCallback (Handles.h:23): a script's per-frame callback. */
typedef void (*PhysikExternalLogicCallback)(PhysikWorldHandle world, void* userData);

/* PhysiK::Vec3 (include/PhysiK/Math/Vec3.h:7-12): three packed floats. */
typedef struct PhysikVec3 {
    float x, y, z;
} PhysikVec3;

/* ---- world ------------------------------------------------------------ */
/* PHYSIK_CreateWorld / PHYSIK_DestroyWorld   PhysiKAPI.h:57-58, PhysiKAPI.cpp:312-320 */
PHYSIK_B200_API PhysikWorldHandle PHYSIK_CreateWorld(void);
PHYSIK_B200_API void PHYSIK_DestroyWorld(PhysikWorldHandle world);
/* PHYSIK_Step   PhysiKAPI.h:60, PhysiKAPI.cpp:322-328 -> World::Step (World.cpp:32-73) */
PHYSIK_B200_API void PHYSIK_Step(PhysikWorldHandle world, float dt);
/* PHYSIK_SetSubstepCount   PhysiKAPI.h:61, World.cpp:157-160 (count clamped to >= 1) */
PHYSIK_B200_API void PHYSIK_SetSubstepCount(PhysikWorldHandle world, int substepCount);
/* PHYSIK_SetSolverMode   PhysiKAPI.h:62, PhysiKAPI.cpp:338-345 (1 = implicit Euler, else explicit) */
PHYSIK_B200_API void PHYSIK_SetSolverMode(PhysikWorldHandle world, int mode);
/* CG settings   PhysiKAPI.h:63-72, World.cpp:177-205 (tolerance clamped to [1e-8, 0.1],
 * non-finite ignored; iterations clamped to [1, 1024]) */
PHYSIK_B200_API void PHYSIK_SetConjugateGradientTolerance(PhysikWorldHandle world, float tolerance);
PHYSIK_B200_API float PHYSIK_GetConjugateGradientTolerance(PhysikWorldHandle world);
PHYSIK_B200_API void PHYSIK_SetConjugateGradientMaxIterations(PhysikWorldHandle world, int maxIterations);
PHYSIK_B200_API int PHYSIK_GetConjugateGradientMaxIterations(PhysikWorldHandle world);
/* Last-solve diagnostics   PhysiKAPI.h:73-78, World.cpp:208-221 */
PHYSIK_B200_API int PHYSIK_GetLastConjugateGradientIterations(PhysikWorldHandle world);
PHYSIK_B200_API float PHYSIK_GetLastConjugateGradientResidualNorm(PhysikWorldHandle world);
PHYSIK_B200_API int PHYSIK_DidLastConjugateGradientSolveConverge(PhysikWorldHandle world);
/* PHYSIK_SetGravity   PhysiKAPI.h:79-83 (default gravity is zero) */
PHYSIK_B200_API void PHYSIK_SetGravity(PhysikWorldHandle world, float x, float y, float z);
/* PHYSIK_AddNode   PhysiKAPI.h:84-88, World.cpp:75-83 */
PHYSIK_B200_API int PHYSIK_AddNode(PhysikWorldHandle world, float x, float y, float z);
/* PHYSIK_SetNodeFixed / PHYSIK_IsNodeFixed   PhysiKAPI.h:90-97, World.cpp:403-423 (fixing zeroes the velocity) */
PHYSIK_B200_API void PHYSIK_SetNodeFixed(PhysikWorldHandle world, int nodeIndex, int fixed);
PHYSIK_B200_API int PHYSIK_IsNodeFixed(PhysikWorldHandle world, int nodeIndex);

/* ---- generated meshes ------------------------------------------------- */
/* PHYSIK_GenerateTetMesh   PhysiKAPI.h:99-103 -> TetMeshGenerator::Generate (TetMeshGenerator.cpp:153-282) */
PHYSIK_B200_API PhysikGeneratedTetMeshHandle PHYSIK_GenerateTetMesh(const PhysikVec3* positions, int nodeCount,
                                                                     const int* tetLocalNodeIndices, int tetCount);
/* PhysiKAPI.h:105-130 */
PHYSIK_B200_API int PHYSIK_IsGeneratedTetMeshHandleValid(PhysikGeneratedTetMeshHandle mesh);
PHYSIK_B200_API void PHYSIK_DestroyGeneratedTetMesh(PhysikGeneratedTetMeshHandle mesh);
PHYSIK_B200_API int PHYSIK_GetGeneratedTetMeshVertexCount(PhysikGeneratedTetMeshHandle mesh);
PHYSIK_B200_API int PHYSIK_GetGeneratedTetMeshTetCount(PhysikGeneratedTetMeshHandle mesh);
PHYSIK_B200_API int PHYSIK_GetGeneratedTetMeshTetIndexCount(PhysikGeneratedTetMeshHandle mesh);
PHYSIK_B200_API int PHYSIK_GetGeneratedTetMeshVertex(PhysikGeneratedTetMeshHandle mesh, int vertexIndex, float* outX,
                                                     float* outY, float* outZ);
PHYSIK_B200_API int PHYSIK_GetGeneratedTetMeshTetNodeIndex(PhysikGeneratedTetMeshHandle mesh, int tetIndexArrayIndex,
                                                           int* outNodeIndex);

/* ---- components ------------------------------------------------------- */
/* PHYSIK_CreateTetMeshComponent   PhysiKAPI.h:132-134, PhysiKAPI.cpp:599-616 */
PHYSIK_B200_API PhysikComponentHandle PHYSIK_CreateTetMeshComponent(PhysikWorldHandle world,
                                                                     PhysikGeneratedTetMeshHandle mesh);
/* PHYSIK_CreateTetMeshPhysicsComponent   PhysiKAPI.h:136-139, PhysiKAPI.cpp:618-640 */
PHYSIK_B200_API PhysikComponentHandle PHYSIK_CreateTetMeshPhysicsComponent(PhysikWorldHandle world,
                                                                            PhysikGeneratedTetMeshHandle mesh,
                                                                            const PhysikMaterialDesc* material);
/* PhysiKAPI.h:141-157 */
PHYSIK_B200_API int PHYSIK_GetTetMeshGlobalNodeBeginIndex(PhysikWorldHandle world, PhysikComponentHandle tetMesh);
PHYSIK_B200_API int PHYSIK_GetTetMeshGlobalNodeCount(PhysikWorldHandle world, PhysikComponentHandle tetMesh);
PHYSIK_B200_API int PHYSIK_GetTetMeshGlobalNodeIndex(PhysikWorldHandle world, PhysikComponentHandle tetMesh,
                                                     int localNodeIndex);
/* PHYSIK_SetTetMeshLocalCurrentPosition / PHYSIK_GetTetMeshLocalCurrentPosition
 * PhysiKAPI.h:236-251, PhysiKAPI.cpp:992-1053: a tet mesh's own copy of its node
 * positions (TetMeshComponent::nodePositions).  A physics mesh's copy is the world's
 * positions at the end of the last PHYSIK_Step (dt > 0) it took part in (its creation
 * positions before that); Set writes that copy only, not the world's node, and the next
 * step overwrites it.  Return 1, or 0 for an invalid world, mesh, index or NULL
 * out-pointer. */
PHYSIK_B200_API int PHYSIK_SetTetMeshLocalCurrentPosition(PhysikWorldHandle world, PhysikComponentHandle tetMesh,
                                                          int localNodeIndex, float x, float y, float z);
PHYSIK_B200_API int PHYSIK_GetTetMeshLocalCurrentPosition(PhysikWorldHandle world, PhysikComponentHandle tetMesh,
                                                          int localNodeIndex, float* outX, float* outY, float* outZ);
PHYSIK_B200_API void PHYSIK_SetTetMeshMaterial(PhysikWorldHandle world, PhysikComponentHandle component,
                                               const PhysikMaterialDesc* material);
/* Collision spheres   PhysiKAPI.h:159-164, 288-298, 346-351; PhysiKAPI.cpp:685-701,
 * 1180-1218, 1407-1429; CollisionSphereComponent.cpp, CollisionComponent.cpp.  Every substep
 * each active tet of every active soft body whose centroid lies strictly inside an active
 * sphere gets a point connection (weights 1/4) pulling its centroid to the sphere's
 * surface, with the sphere's connection stiffness and damping (defaults 1000 and 10;
 * negative or non-finite settings become 0).  The radius is clamped at 0.  A kinematic
 * target moves the sphere at the next PHYSIK_Step's start.  The contacts are found on the
 * GPU at the substep's positions (pk_system_sphere_contacts).  Invalid handles are
 * ignored; getters leave their out-pointers alone then. */
PHYSIK_B200_API PhysikComponentHandle PHYSIK_CreateCollisionSphereComponent(PhysikWorldHandle world, float x, float y,
                                                                            float z, float radius);
PHYSIK_B200_API void PHYSIK_SetCollisionSphereConnectionSettings(PhysikWorldHandle world,
                                                                 PhysikComponentHandle sphereComponent,
                                                                 float stiffness, float damping);
PHYSIK_B200_API void PHYSIK_GetCollisionSphereConnectionSettings(PhysikWorldHandle world,
                                                                 PhysikComponentHandle sphereComponent,
                                                                 float* outStiffness, float* outDamping);
PHYSIK_B200_API void PHYSIK_SetCollisionComponentKinematicTarget(PhysikWorldHandle world,
                                                                 PhysikComponentHandle component, float x, float y,
                                                                 float z);

/* Host-emitted SolverData contributions (extension; the reference offers them only to C++
 * components: SolverData::AddNodeForce / AddNodeMass / AddStiffnessBlock, SolverData.h:41-54).
 * A contribution component calls `callback(solverData, dt, userData)` from its UpdateSystem
 * every substep, in execution-priority order (`priority` as ComponentExecutionPriority:
 * 100 scripts ... 400 soft bodies ... 1000 default); the callback emits through the
 * PHYSIK_B200_SolverDataAdd* functions on the handle it received, which is valid only
 * during the call.  The device step assembles them as the reference's SolverData does:
 * masses join the lumped masses (and may make nodes dynamic), forces the rhs, blocks the
 * matrix (upper triangle) and -dt^2 B v the rhs; a non-finite block skips the substep.
 * block9: the 3x3 block column-major (9 floats). */
typedef void (*PhysikContributionCallback)(void* solverData, float dt, void* userData);
PHYSIK_B200_API PhysikComponentHandle PHYSIK_B200_CreateContributionComponent(PhysikWorldHandle world, int priority);
PHYSIK_B200_API void PHYSIK_B200_SetContributionCallback(PhysikWorldHandle world, PhysikComponentHandle component,
                                                         PhysikContributionCallback callback, void* userData);
PHYSIK_B200_API void PHYSIK_B200_SolverDataAddNodeForce(void* solverData, int node, float fx, float fy, float fz);
PHYSIK_B200_API void PHYSIK_B200_SolverDataAddNodeMass(void* solverData, int node, float mass);
PHYSIK_B200_API void PHYSIK_B200_SolverDataAddStiffnessBlock(void* solverData, int nodeA, int nodeB,
                                                             const float* block9);

/* Script components   PhysiKAPI.h:166-177, PhysiKAPI.cpp:719-765; ScriptComponent.cpp: the
 * callback runs once per PHYSIK_Step, before the substeps (Component::PreUpdate, in
 * execution-priority order), with the world handle, so a script can call PHYSIK_* (add
 * point connections, move nodes, ...) for the frame.  Invalid handles are ignored. */
PHYSIK_B200_API PhysikComponentHandle PHYSIK_CreateScriptComponent(PhysikWorldHandle world);
PHYSIK_B200_API void PHYSIK_SetScriptComponentCallback(PhysikWorldHandle world, PhysikComponentHandle scriptComponent,
                                                       PhysikExternalLogicCallback callback, void* userData);
PHYSIK_B200_API void PHYSIK_ClearScriptComponentCallback(PhysikWorldHandle world,
                                                         PhysikComponentHandle scriptComponent);
/* Post-step geometry: render buffers rebuilt after each PHYSIK_Step (Component::PostUpdate).
 * Surface extraction   PhysiKAPI.h:179-191, PhysiKAPI.cpp:767-823; SurfaceExtractionComponent.cpp:
 *   the boundary faces of the host mesh's active tets (3 local node indices each), wound
 *   away from their tet, rebuilt when the host's topology changed.
 * Surface visual       PhysiKAPI.h:193-228, PhysiKAPI.cpp:825-980; SurfaceVisualComponent.cpp:
 *   three vertices per surface triangle at the host's local current positions, index
 *   buffer 0, 1, 2, ..., flat normals ((0, 1, 0) for a degenerate triangle).
 * Visual mesh          PhysiKAPI.h:252-287, PhysiKAPI.cpp:703-717, 1055-1170; VisualMeshComponent.cpp:
 *   a render mesh embedded in the host's rest shape (PHYSIK_BuildVisualMeshEmbedding
 *   returns 1 if any vertex landed in an active tet), skinned with the world positions
 *   of its tets' nodes; triangles with a vertex outside the active tets are filtered out.
 * The per-frame vertex and normal updates run on the device for a physics host and stay
 * there until a getter reads them.  Getters return 0 on an invalid handle, index or
 * NULL out-pointer; the Copy* functions return the number of elements written. */
PHYSIK_B200_API PhysikComponentHandle PHYSIK_CreateSurfaceExtractionComponent(PhysikWorldHandle world,
                                                                              PhysikComponentHandle hostTetMesh);
PHYSIK_B200_API int PHYSIK_GetSurfaceTriangleIndexCount(PhysikWorldHandle world, PhysikComponentHandle surfaceExtraction);
PHYSIK_B200_API int PHYSIK_CopySurfaceTriangleIndices(PhysikWorldHandle world, PhysikComponentHandle surfaceExtraction,
                                                      int* outIndices, int maxIndexCount);
PHYSIK_B200_API PhysikComponentHandle PHYSIK_CreateSurfaceVisualComponent(PhysikWorldHandle world,
                                                                          PhysikComponentHandle surfaceExtraction);
PHYSIK_B200_API int PHYSIK_GetSurfaceVisualVertexCount(PhysikWorldHandle world, PhysikComponentHandle surfaceVisual);
PHYSIK_B200_API int PHYSIK_GetSurfaceVisualTriangleIndexCount(PhysikWorldHandle world,
                                                              PhysikComponentHandle surfaceVisual);
PHYSIK_B200_API int PHYSIK_GetSurfaceVisualNormalCount(PhysikWorldHandle world, PhysikComponentHandle surfaceVisual);
PHYSIK_B200_API int PHYSIK_GetSurfaceVisualVertex(PhysikWorldHandle world, PhysikComponentHandle surfaceVisual,
                                                  int visualVertexIndex, float* outX, float* outY, float* outZ);
PHYSIK_B200_API int PHYSIK_GetSurfaceVisualTriangleIndex(PhysikWorldHandle world, PhysikComponentHandle surfaceVisual,
                                                         int triangleIndexArrayIndex, int* outIndex);
PHYSIK_B200_API int PHYSIK_GetSurfaceVisualNormal(PhysikWorldHandle world, PhysikComponentHandle surfaceVisual,
                                                  int visualNormalIndex, float* outX, float* outY, float* outZ);
PHYSIK_B200_API PhysikComponentHandle PHYSIK_CreateVisualMeshComponent(PhysikWorldHandle world,
                                                                       PhysikComponentHandle hostTetMesh);
PHYSIK_B200_API void PHYSIK_SetVisualMeshData(PhysikWorldHandle world, PhysikComponentHandle visualMesh,
                                              const PhysikVec3* vertices, int vertexCount, const int* triangleIndices,
                                              int triangleIndexCount);
PHYSIK_B200_API int PHYSIK_BuildVisualMeshEmbedding(PhysikWorldHandle world, PhysikComponentHandle visualMesh);
PHYSIK_B200_API int PHYSIK_GetVisualMeshVertexCount(PhysikWorldHandle world, PhysikComponentHandle visualMesh);
PHYSIK_B200_API int PHYSIK_GetVisualMeshTriangleIndexCount(PhysikWorldHandle world, PhysikComponentHandle visualMesh);
PHYSIK_B200_API int PHYSIK_CopyVisualMeshVertices(PhysikWorldHandle world, PhysikComponentHandle visualMesh,
                                                  PhysikVec3* outVertices, int maxVertexCount);
PHYSIK_B200_API int PHYSIK_CopyVisualMeshTriangleIndices(PhysikWorldHandle world, PhysikComponentHandle visualMesh,
                                                         int* outIndices, int maxIndexCount);
/* Whether a surface visual's or visual mesh's last update ran on the device: 1 / 0, -1
 * for another handle (extension). */
PHYSIK_B200_API int PHYSIK_B200_GetVisualUpdateOnDevice(PhysikWorldHandle world, PhysikComponentHandle visual);

/* PhysiKAPI.h:300-334 */
PHYSIK_B200_API void PHYSIK_DestroyComponent(PhysikWorldHandle world, PhysikComponentHandle component);
PHYSIK_B200_API int PHYSIK_IsComponentHandleValid(PhysikWorldHandle world, PhysikComponentHandle component);
PHYSIK_B200_API int PHYSIK_GetTetMeshTetCount(PhysikWorldHandle world, PhysikComponentHandle component);
PHYSIK_B200_API int PHYSIK_GetTetMeshNodeCount(PhysikWorldHandle world, PhysikComponentHandle component);
PHYSIK_B200_API int PHYSIK_IsTetActive(PhysikWorldHandle world, PhysikComponentHandle component, int tetIndex);
/* PHYSIK_SetTetActive   PhysiKAPI.h:321-325, PhysiKAPI.cpp:1324-1346 (node activity reconciled) */
PHYSIK_B200_API void PHYSIK_SetTetActive(PhysikWorldHandle world, PhysikComponentHandle component, int tetIndex,
                                         int active);
PHYSIK_B200_API void PHYSIK_DeactivateTet(PhysikWorldHandle world, PhysikComponentHandle component, int tetIndex);
PHYSIK_B200_API int PHYSIK_GetActiveTetCount(PhysikWorldHandle world, PhysikComponentHandle component);

/* ---- node state ------------------------------------------------------- */
/* PhysiKAPI.h:371-397, PhysiKAPI.cpp:1477-1558 (SetNodePosition zeroes the velocity) */
PHYSIK_B200_API void PHYSIK_GetNodePosition(PhysikWorldHandle world, int nodeIndex, float* outX, float* outY,
                                            float* outZ);
PHYSIK_B200_API void PHYSIK_GetNodeVelocity(PhysikWorldHandle world, int nodeIndex, float* outX, float* outY,
                                            float* outZ);
PHYSIK_B200_API void PHYSIK_SetNodePosition(PhysikWorldHandle world, int nodeIndex, float x, float y, float z);
PHYSIK_B200_API void PHYSIK_SetNodeVelocity(PhysikWorldHandle world, int nodeIndex, float x, float y, float z);

/* ---- point connections ----------------------------------------------- */
/* PHYSIK_GetPointConnectionCount / PHYSIK_AddPointConnection   PhysiKAPI.h:353-369,
 * PhysiKAPI.cpp:1431-1475, World.cpp:126-131: a transient barycentric spring between the
 * point sum_i w_i x(node_i) and a target, kept until the end of the next PHYSIK_Step
 * (dropped at once unless its four nodes exist and are active); its forces and stiffness
 * blocks (PointConnection.cpp:55-140) join the device system of that step. */
PHYSIK_B200_API int PHYSIK_GetPointConnectionCount(PhysikWorldHandle world);
PHYSIK_B200_API void PHYSIK_AddPointConnection(PhysikWorldHandle world, int node0, int node1, int node2, int node3,
                                               float barycentricX, float barycentricY, float barycentricZ,
                                               float barycentricW, float targetX, float targetY, float targetZ,
                                               float stiffness, float damping);

/* ---- extensions (no counterpart in the reference) --------------------- */
#define PHYSIK_B200_PRECISION_FP32 0  /* the reference's scalar type: float storage and dot products */
#define PHYSIK_B200_PRECISION_MIXED 1 /* float storage, double CG scalars, double polar for near-inverted tets */
#define PHYSIK_B200_PRECISION_FP64 2  /* double everywhere */
PHYSIK_B200_API void PHYSIK_B200_SetPrecision(PhysikWorldHandle world, int precision);
PHYSIK_B200_API int PHYSIK_B200_GetPrecision(PhysikWorldHandle world);
PHYSIK_B200_API void PHYSIK_B200_SetDevice(PhysikWorldHandle world, int device);
PHYSIK_B200_API int PHYSIK_B200_GetNodeCount(PhysikWorldHandle world);
/* Bulk state, 3 values per node in world order; returns nodes copied or -1.  The F64
 * variants move FP64 values to and from the device system once it is uploaded (after the
 * first step, or PHYSIK_B200_PrepareScene(world, 1)); before that the world keeps its state
 * in float host copies. */
PHYSIK_B200_API int PHYSIK_B200_GetNodeStates(PhysikWorldHandle world, float* positions, float* velocities, int count);
PHYSIK_B200_API int PHYSIK_B200_SetNodeStates(PhysikWorldHandle world, const float* positions, const float* velocities,
                                              int count);
PHYSIK_B200_API int PHYSIK_B200_GetNodeStatesF64(PhysikWorldHandle world, double* positions, double* velocities,
                                                 int count);
PHYSIK_B200_API int PHYSIK_B200_SetNodeStatesF64(PhysikWorldHandle world, const double* positions,
                                                 const double* velocities, int count);
/* Per-element Young's modulus (the reference's C++ route: Tet::youngModulus + RebuildTetFemCache). */
PHYSIK_B200_API int PHYSIK_B200_SetTetMeshYoungModulus(PhysikWorldHandle world, PhysikComponentHandle component,
                                                       const float* youngModulus, int tetCount);
/* FemModel selector: 0 linear, 1 corotated (default), 2 NeoHookean (not implemented, as in the reference). */
PHYSIK_B200_API int PHYSIK_B200_SetTetMeshFemModel(PhysikWorldHandle world, PhysikComponentHandle component, int model);
/* Flags of the last device substep (PK_FLAG_* of include/pkcuda.h). */
PHYSIK_B200_API unsigned PHYSIK_B200_GetLastStepFlags(PhysikWorldHandle world);
/* Message of the last failure caught at this boundary ("" if none). */
PHYSIK_B200_API const char* PHYSIK_B200_GetLastError(void);
/* Builds the solver scene (lumped masses, dynamic-node mapping, canonical upper BSR
 * pattern) without stepping; uploads it to the GPU when `upload` is non-zero (with
 * upload = 0 no CUDA call is made).  Returns the dynamic row count or -1. */
PHYSIK_B200_API int PHYSIK_B200_PrepareScene(PhysikWorldHandle world, int upload);
/* The solver pattern (canonical upper BSR over dynamic rows) and node mapping of the
 * last prepared scene (SolverData's matrix pattern, SolverData.cpp:389-401). */
PHYSIK_B200_API int PHYSIK_B200_GetSolverSizes(PhysikWorldHandle world, int* dynamicRows, int* blocks);
PHYSIK_B200_API int PHYSIK_B200_GetSolverPattern(PhysikWorldHandle world, int* rowStart, int* colIndex,
                                                 int* nodeToDynamic);
/* Assembled lumped masses per world node (SolverData::AssembleMasses). */
PHYSIK_B200_API int PHYSIK_B200_GetSolverMasses(PhysikWorldHandle world, double* masses);
/* The last substep's assembled system: values 9*blocks (column-major), rhs 3*rows,
 * block-Jacobi inverse 9*rows, delta-v 3*rows. */
PHYSIK_B200_API int PHYSIK_B200_GetSolverSystem(PhysikWorldHandle world, double* values, double* rhs, double* minv,
                                                double* deltaVelocity);
/* Device timing of the step phases (see pk_system_timings). */
PHYSIK_B200_API int PHYSIK_B200_EnableTiming(PhysikWorldHandle world, int on);
PHYSIK_B200_API int PHYSIK_B200_GetTimings(PhysikWorldHandle world, double* assembleMs, double* solveMs, int* steps,
                                           long long* kernelLaunches);
PHYSIK_B200_API int PHYSIK_B200_SetPcgGrid(PhysikWorldHandle world, int grid);
/* Adjoint of one implicit substep of size dt (no counterpart in the reference): with the
 * world at the state the substep starts from and the loss sensitivities to the state
 * after it (3 doubles per node each, world order), writes the sensitivities to the current
 * state and adds each tet's sensitivity to its log Young's modulus to youngLogBar (may be
 * NULL; tets of the tet-mesh physics components in creation order, see
 * PHYSIK_B200_GetTetCount).  The state is left unchanged.  0 on success, -1 on failure. */
PHYSIK_B200_API int PHYSIK_B200_AdjointStep(PhysikWorldHandle world, float dt, const double* positionsBarNext,
                                            const double* velocitiesBarNext, double* positionsBar,
                                            double* velocitiesBar, double* youngLogBar);
/* Tets of the world's tet-mesh physics components (the adjoint's tet order), or -1. */
PHYSIK_B200_API int PHYSIK_B200_GetTetCount(PhysikWorldHandle world);
/* Captures the device step in a CUDA graph and replays it (see pk_system_set_graph). */
PHYSIK_B200_API void PHYSIK_B200_SetGraphCapture(PhysikWorldHandle world, int on);
/* Picks the fastest PCG kernel and tile (or, batched, part) size for the world's scene by
 * timing `repeats` solves of the last assembled system; call after a step.  Returns the
 * chosen candidate (see pk_system_autotune) or -1; bestSolveMs (may be NULL) receives its
 * mean solve time. */
PHYSIK_B200_API int PHYSIK_B200_Autotune(PhysikWorldHandle world, int repeats, double* bestSolveMs);
/* The PCG kernel of the last step's solve (see pk_system_pcg_kernel: 0 ring-staged, 1
 * TMA-staged, 2 unstaged, 3 part-resident, 4 batched) or -1; blocks (may be NULL)
 * receives the blocks it ran on. */
PHYSIK_B200_API int PHYSIK_B200_GetPcgKernel(PhysikWorldHandle world, int* blocks);
/* The part-resident kernel's stream form in the last step's solve (pk_system_slab_form:
 * 0 full rows, 1 symmetric form, -1 another kernel).  No counterpart in the reference. */
PHYSIK_B200_API int PHYSIK_B200_GetPcgStreamForm(PhysikWorldHandle world);
/* The world's device system (a pk_system* of include/pkcuda.h) once a step has uploaded it,
 * else NULL: lets a caller use the device ABI on the world's own buffers (e.g.
 * pk_system_sphere_contacts).  The world owns it.  No counterpart in the reference. */
PHYSIK_B200_API void* PHYSIK_B200_GetDeviceSystem(PhysikWorldHandle world);
/* FP64 outer true-residual refinement of the implicit solve for FP32 and mixed precision
 * (no counterpart in the reference; see pk_system_set_refinement): up to `passes`
 * correction solves (0..16, 0 = off, the default) within the step's iteration budget,
 * until the true residual meets the CG's stopping target.  0 on success, -1 on error. */
PHYSIK_B200_API int PHYSIK_B200_SetRefinement(PhysikWorldHandle world, int passes);
/* Batched solve: one PCG per tet-mesh physics component (own scalars, stopping test,
 * iteration count and all-or-nothing integration, as a world holding only that body),
 * all bodies in one launch, instead of the reference's single coupled PCG over the whole
 * world.  The world's CG getters then report the largest iteration count, the largest
 * residual and "converged" only if every body converged. */
PHYSIK_B200_API void PHYSIK_B200_SetBatchedSolve(PhysikWorldHandle world, int on);
/* One body's statistics of the last batched step; 0 on success, -1 if unavailable. */
PHYSIK_B200_API int PHYSIK_B200_GetBodyConjugateGradientStats(PhysikWorldHandle world, PhysikComponentHandle body,
                                                              int* iterations, int* converged, float* residualNorm,
                                                              unsigned* flags);
/* The CUDA stream (cudaStream_t) the world's device work runs on, or NULL before the
 * first upload; lets a caller record its own events around steps. */
PHYSIK_B200_API void* PHYSIK_B200_GetStream(PhysikWorldHandle world);
/* Waits for the device work queued by the world. */
PHYSIK_B200_API int PHYSIK_B200_Synchronize(PhysikWorldHandle world);

#ifdef __cplusplus
}
#endif

#endif /* PHYSIK_B200_H */
