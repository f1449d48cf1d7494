// physik_core.h -- the host-side mirror of PhysiK's soft-body path, backed by the
// sm_100a kernels of libpkcuda.  Class and member names follow the reference's
// component API so code written against it keeps compiling:
//
//   TetMeshGenerator        include/PhysiK/Geometry/TetMeshGenerator.h:7-46
//   SparseBlockMatrix       include/PhysiK/Math/SparseBlockMatrix.h:14-42
//   ConjugateGradient*      include/PhysiK/Core/Solvers/Linear/ConjugateGradientSolver.h:12-35
//   LinearSolver            include/PhysiK/Core/Solvers/Linear/LinearSolver.h:13-55
//   SolverData              include/PhysiK/Core/Solvers/SolverData.h:15-134
//   Component / TetMesh*    include/PhysiK/Components/Component.h:13-44,
//                           TetMeshComponent.h:11-42, TetMeshPhysicsComponent.h:13-85
//   World                   include/PhysiK/Core/World/World.h:30-137
//   PointConnection         include/PhysiK/Core/PhysicsConnections/PointConnection.h:12-26
//
// What differs by design: node state lives on the GPU (the host copies are synced on
// access), SolverData owns a device BSR, and World::Step launches one device substep
// (tet kernel, row kernel, cooperative PCG + integration) per substep.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <tuple>
#include <vector>

#include "physik_math.h"

struct pk_system;
struct pk_visual;

namespace PhysiK {

// ------------------------------------------------------------------ handles / data
struct ComponentHandle {
    std::uint32_t index = 0xFFFFFFFFu;
    std::uint32_t generation = 0u;
    bool IsValid() const { return index != 0xFFFFFFFFu && generation != 0u; }
};

struct Node {
    int stateIndex = -1;
    bool active = true;
    bool fixed = false;
    bool hasRotation = false;
};

struct Material {
    float density = 1.0f;
    float youngModulus = 25.0f;
    float poissonRatio = 0.3f;
    float damping = 0.25f;
};

struct Tet {
    int node0 = -1, node1 = -1, node2 = -1, node3 = -1;
    bool active = true;
    float restVolume = 0.0f;
    Mat3 restDmInverse;
    Vec3 restPositions[4];
    Vec3 shapeFunctionGradients[4];
    float youngModulus = 25.0f;
    float poissonRatio = 0.3f;
    float damping = 0.25f;
};

enum class FemModel : std::uint32_t { Linear = 0, Corotational = 1, NeoHookean = 2 };
enum class SolverMode { Explicit, ImplicitEuler };
enum class ComponentExecutionPriority : int {
    ScriptComponent = 100,
    CollisionSphereComponent = 200,
    TetMeshComponent = 300,
    TetMeshPhysicsComponent = 400,
    TopologyMeshComponent = 500,
    TetMeshMapperComponent = 600,
    SurfaceExtractionComponent = 700,
    SurfaceVisualComponent = 800,
    VisualMeshComponent = 900,
    Default = 1000
};

// Device precision of a World (extension: the reference is FP32 only).
enum class Precision : int { FP32 = 0, Mixed = 1, FP64 = 2 };

// ------------------------------------------------------------------ generator
struct TetMeshBuildOptions {
    bool weldCoincidentNodes = true;
    float weldTolerance = 1.0e-5f;
    bool removeDegenerateTets = true;
};
struct TetMeshTopologyDiagnostics {
    int boundaryFaceCount = 0;
    int internalFaceCount = 0;
    int nonManifoldFaceCount = 0;
};
struct GeneratedTetMesh {
    std::vector<Vec3> positions;
    std::vector<int> tetLocalNodeIndices;
    TetMeshTopologyDiagnostics topologyDiagnostics;
    int rawNodeCount = 0;
    int rawTetCount = 0;
    int weldedNodeCount = 0;
    int weldedAwayNodeCount = 0;
    int removedDegenerateTetCount = 0;
    float weldTolerance = 0.0f;
};
class TetMeshGenerator {
public:
    static GeneratedTetMesh Generate(const Vec3* positions, int nodeCount, const int* tetLocalNodeIndices, int tetCount,
                                     const TetMeshBuildOptions& options = TetMeshBuildOptions{});
};

// ------------------------------------------------------------------ sparse matrix
// Canonical upper BSR (row <= col), per-row sorted unique columns, column-major blocks.
class SparseBlockMatrix {
public:
    int blockCount = 0;
    std::vector<int> rowStart;
    std::vector<int> colIndex;
    std::vector<Mat3> values;

    void Clear();
    void ClearValues();
    void BuildPattern(int newBlockCount, const std::vector<std::pair<int, int>>& blockCoordinates);
    bool AddBlock(int rowBlock, int colBlock, const Mat3& block);
    // y = A x on the GPU (symmetric product of the upper storage).
    void Multiply(const std::vector<float>& input, std::vector<float>& output) const;
    void Multiply(const std::vector<Vec3>& input, std::vector<Vec3>& output) const;
    int FindBlockIndex(int rowBlock, int colBlock) const;

private:
    std::unordered_map<std::uint64_t, int> blockLookup;
    static std::uint64_t MakeKey(int rowBlock, int colBlock);
};

// ------------------------------------------------------------------ solver
struct ConjugateGradientSettings {
    int maxIterations = 128;
    float tolerance = 1.0e-4f;
    bool useJacobiPreconditioner = true;
};
struct ConjugateGradientResult {
    int iterations = 0;
    float residualNorm = 0.0f;
    bool converged = false;
};
// Block-Jacobi PCG on the GPU with the reference's argument checks and results.
ConjugateGradientResult SolvePreconditionedConjugateGradient(std::vector<Vec3>& x, const SparseBlockMatrix& A,
                                                             const std::vector<Vec3>& b, int maxIterations,
                                                             float tolerance, const std::vector<Mat3>& MInv,
                                                             std::vector<Vec3>& r, std::vector<Vec3>& d,
                                                             std::vector<Vec3>& qOrS);

struct LinearSolveSettings {
    int maxIterations = 128;
    float tolerance = 1.0e-5f;
    bool useJacobiPreconditioner = true;
};
struct LinearSolveResult {
    int iterations = 0;
    float residualNorm = 0.0f;
    bool converged = false;
};
class LinearSolver {
public:
    virtual ~LinearSolver() = default;
    virtual LinearSolveResult Solve(const SparseBlockMatrix& matrix, const std::vector<Vec3>& rhs,
                                    std::vector<Vec3>& solution, const LinearSolveSettings& settings) = 0;
};
// The GPU solver behind the reference's CurrentLinearSolver seam.
class CurrentLinearSolver final : public LinearSolver {
public:
    LinearSolveResult Solve(const SparseBlockMatrix& matrix, const std::vector<Vec3>& rhs, std::vector<Vec3>& solution,
                            const LinearSolveSettings& settings) override;

private:
    std::vector<Mat3> inversePreconditioner;
    std::vector<Vec3> residual, direction, temp;
};
LinearSolver& GetCurrentLinearSolver();

// Index of the process-wide CUDA device used by the solver entry points (default 0).
int GetSolverDevice();
void SetSolverDevice(int device);

class World;
class TetMeshPhysicsComponent;

// ------------------------------------------------------------------ SolverData
class SolverData {
public:
    struct NodeForce {
        int node = -1;
        Vec3 force;
    };
    struct NodeMass {
        int node = -1;
        float mass = 0.0f;
    };
    struct StiffnessBlock {
        int nodeA = -1;
        int nodeB = -1;
        Mat3 block;
    };

    void Clear();
    void ClearTransientState();
    void MarkImplicitPatternDirty() { implicitPatternDirty = true; }

    void AddNodeForce(int node, const Vec3& force) { nodeForces.push_back(NodeForce{node, force}); }
    void AddNodeMass(int node, float mass) { nodeMasses.push_back(NodeMass{node, mass}); }
    void AddStiffnessBlock(int nodeA, int nodeB, const Mat3& block)
    {
        stiffnessBlocks.push_back(StiffnessBlock{nodeA, nodeB, block});
    }
    // Device path: a soft body whose per-tet forces and stiffness the GPU computes.
    void AddFemBody(const TetMeshPhysicsComponent* body)
    {
        femBodies.push_back(body);
        femMassMark.push_back(nodeMasses.size());  // masses emitted before this body's
    }

    const std::vector<NodeForce>& GetNodeForces() const { return nodeForces; }
    const std::vector<NodeMass>& GetNodeMasses() const { return nodeMasses; }
    const std::vector<StiffnessBlock>& GetStiffnessBlocks() const { return stiffnessBlocks; }
    const std::vector<const TetMeshPhysicsComponent*>& GetFemBodies() const { return femBodies; }

    void AssembleMasses(int nodeCount);
    bool HasNodeMassContribution(int nodeIndex) const;
    float GetAssembledMassForNode(int nodeIndex) const;

    // Generic path (host-emitted forces, masses and blocks): builds SolverData's
    // mapping and pattern, assembles A and b and solves on the GPU.
    bool PrecomputeImplicitSolve(const std::vector<Node>& nodes, const std::vector<Vec3>& nodeVelocities, float dt);
    bool SolveImplicitLinearSystem(const ConjugateGradientSettings& settings);
    const LinearSolveResult& GetLastLinearSolveResult() const { return lastLinearSolveResult; }
    int GetLastCgIterationCount() const { return lastLinearSolveResult.iterations; }
    float GetLastCgResidualNorm() const { return lastLinearSolveResult.residualNorm; }

    int GetDynamicBlockForNode(int nodeIndex) const;
    int GetDynamicBlockCount() const { return dynamicBlockCount; }
    const std::vector<Vec3>& GetDeltaVelocity() const { return deltaVelocity; }
    const std::vector<float>& GetAssembledMasses() const { return assembledMasses; }
    const std::vector<Vec3>& GetAssembledForces() const { return assembledForces; }
    const SparseBlockMatrix& GetMatrix() const { return matrix; }
    const std::vector<Vec3>& GetRhs() const { return rhs; }

private:
    friend class World;
    bool BuildDynamicNodeMapping(const std::vector<Node>& nodes);

    std::vector<NodeForce> nodeForces;
    std::vector<NodeMass> nodeMasses;
    std::vector<StiffnessBlock> stiffnessBlocks;
    std::vector<const TetMeshPhysicsComponent*> femBodies;
    std::vector<std::size_t> femMassMark;  // per FEM body: nodeMasses.size() when it registered

    std::vector<float> assembledMasses;
    std::vector<Vec3> assembledForces;
    std::vector<int> nodeToDynamicBlock;
    int dynamicBlockCount = 0;
    std::vector<Vec3> rhs;
    SparseBlockMatrix matrix;
    std::vector<Vec3> deltaVelocity;
    LinearSolveResult lastLinearSolveResult;
    bool implicitPatternDirty = true;
    bool precomputeOk = false;
    float precomputeDt = 0.0f;
};

// ------------------------------------------------------------------ components
enum class PhysicsEventType { TetMeshTopologyChanged };

class Component {
public:
    bool active = true;
    virtual ComponentExecutionPriority GetExecutionPriority() const { return ComponentExecutionPriority::Default; }
    virtual void PreUpdate(World&, float) {}
    virtual void UpdateSystem(World&, SolverData&, float) {}
    virtual void PostUpdate(World&, float) {}
    // Called before the world's device system is replaced: copy any result still on the
    // device to the host and drop what was allocated on that system (extension).
    virtual void ReleaseDeviceResources() {}
    virtual ~Component() = default;
};

// ScriptComponent (ScriptComponent.cpp): calls an external callback with the world once
// per frame, in PreUpdate.
using ExternalLogicCallback = void (*)(void* world, void* userData);
class ScriptComponent : public Component {
public:
    ComponentExecutionPriority GetExecutionPriority() const override
    {
        return ComponentExecutionPriority::ScriptComponent;
    }
    void SetExternalLogicCallback(ExternalLogicCallback callback, void* userData)
    {
        externalLogicCallback = callback;
        externalLogicUserData = userData;
    }
    void ClearExternalLogicCallback() { SetExternalLogicCallback(nullptr, nullptr); }
    ExternalLogicCallback GetExternalLogicCallback() const { return externalLogicCallback; }
    void* GetExternalLogicUserData() const { return externalLogicUserData; }
    void PreUpdate(World& world, float) override
    {
        if (externalLogicCallback) externalLogicCallback(static_cast<void*>(&world), externalLogicUserData);
    }

private:
    ExternalLogicCallback externalLogicCallback = nullptr;
    void* externalLogicUserData = nullptr;
};

// A component whose UpdateSystem hands the substep's SolverData to an external callback,
// which emits contributions through the C ABI (PHYSIK_B200_SolverDataAdd*) as a C++
// component would through SolverData::AddNodeForce / AddNodeMass / AddStiffnessBlock.
using ContributionCallback = void (*)(void* solverData, float dt, void* userData);
class ContributionComponent : public Component {
public:
    explicit ContributionComponent(int priority) : priority_(priority) {}
    ComponentExecutionPriority GetExecutionPriority() const override
    {
        return static_cast<ComponentExecutionPriority>(priority_);
    }
    void SetCallback(ContributionCallback cb, void* user)
    {
        callback = cb;
        userData = user;
    }
    void UpdateSystem(World&, SolverData& solverData, float dt) override
    {
        if (callback) callback(static_cast<void*>(&solverData), dt, userData);
    }

private:
    int priority_;
    ContributionCallback callback = nullptr;
    void* userData = nullptr;
};

// Transform of a collision component (Transform.h:8-16; the sphere uses its position).
struct Transform {
    Vec3 position;
};

// CollisionComponent (CollisionComponent.h, .cpp): a kinematic target set by the C ABI is
// applied at the next frame's PreUpdate.
class CollisionComponent : public Component {
public:
    Transform transform;
    bool generateConnections = true;
    bool generateEvents = false;
    bool isSensor = false;
    float contactStiffness = 1000.0f;
    float contactDamping = 10.0f;

    void SetKinematicTarget(const Transform& target)
    {
        kinematicTarget = target;
        hasKinematicTarget = true;
    }
    bool ConsumeKinematicTarget(Transform& out)
    {
        if (!hasKinematicTarget) return false;
        out = kinematicTarget;
        hasKinematicTarget = false;
        return true;
    }
    void PreUpdate(World&, float) override
    {
        Transform target;
        if (ConsumeKinematicTarget(target)) transform = target;
    }

private:
    bool hasKinematicTarget = false;
    Transform kinematicTarget;
};

// CollisionSphereComponent (CollisionSphereComponent.cpp): every substep, each active tet
// of every active soft body whose centroid lies inside the sphere gets a point connection
// from its centroid (weights 1/4) to the sphere's surface along the centre-to-centroid
// direction.  UpdateSystem only registers the request; the world finds the contacts on
// the device once the substep's state is there (World::AddSphereContacts) and adds the
// connections in the same order as the reference.
class CollisionSphereComponent : public CollisionComponent {
public:
    static std::unique_ptr<CollisionSphereComponent> Create(const Vec3& position, float radius);
    ComponentExecutionPriority GetExecutionPriority() const override
    {
        return ComponentExecutionPriority::CollisionSphereComponent;
    }
    float radius = 0.5f;
    void SetConnectionSettings(float stiffness, float damping);
    void SetConnectionStiffness(float stiffness);
    float GetConnectionStiffness() const { return contactStiffness; }
    void SetConnectionDamping(float damping);
    float GetConnectionDamping() const { return contactDamping; }
    void UpdateSystem(World& world, SolverData& solverData, float dt) override;
};

class TetMeshComponent : public Component {
public:
    std::vector<Vec3> restNodePositions;
    std::vector<Vec3> nodePositions;
    std::vector<Tet> tets;
    bool topologyDirty = false;
    // TetMeshTopologyChanged events emitted so far (TetMeshComponent::PostUpdate,
    // TetMeshComponent.cpp:190-206, emits one when topologyDirty is set).  Listeners keep
    // the count they have seen and compare it in their own PostUpdate, which comes later in
    // the frame, so they see an event in the frame it is emitted, as the reference's
    // synchronous dispatch delivers it.
    std::uint64_t topologyEvents = 0;
    // SetLocalCurrentPosition calls so far (a copy edited after the frame is no longer the
    // frame-end snapshot the device holds).
    std::uint64_t localEdits = 0;

    ComponentExecutionPriority GetExecutionPriority() const override
    {
        return ComponentExecutionPriority::TetMeshComponent;
    }
    void SetGeometry(const GeneratedTetMesh& generatedMesh);
    int GetNodeCount() const { return static_cast<int>(restNodePositions.size()); }
    int GetTetCount() const { return static_cast<int>(tets.size()); }
    int GetTetNodeIndex(int tetIndex, int cornerIndex) const;
    const Vec3& GetLocalRestPosition(int localNodeIndex) const;
    const Vec3& GetLocalCurrentPosition(int localNodeIndex) const;
    virtual int GetGlobalNodeIndex(int localNodeIndex) const;
    virtual void SetLocalCurrentPosition(int localNodeIndex, const Vec3& position);
    bool IsTetActive(int tetIndex) const;
    virtual bool SetTetActive(int tetIndex, bool active);
    virtual bool DeactivateTet(int tetIndex) { return SetTetActive(tetIndex, false); }
    int GetActiveTetCount() const;
    void PostUpdate(World& world, float dt) override;
    // The local index of world node `globalNodeIndex` in this mesh, or -1.
    int GetLocalNodeIndexOf(int globalNodeIndex) const;
    // Whether an active tet of this mesh has local node `localNodeIndex` as a corner (the
    // node-to-tet lists are built on first use and dropped by SetGeometry or when `tets`
    // is resized or moved).
    bool HasActiveTetAtLocalNode(int localNodeIndex) const;

private:
    mutable std::vector<int> nodeTetStart, nodeTetList;
    mutable std::size_t nodeTetCount = 0;
    mutable const Tet* nodeTetData = nullptr;
};

struct TetMeshPhysicsComponentDesc {
    Material material;
    FemModel femModel = FemModel::Corotational;
};

class TetMeshPhysicsComponent : public TetMeshComponent {
public:
    static std::unique_ptr<TetMeshPhysicsComponent> CreateFromGeneratedTetMesh(World& world,
                                                                               const GeneratedTetMesh& generatedMesh,
                                                                               const Material& material);
    static std::unique_ptr<TetMeshPhysicsComponent> CreateFromGeneratedTetMesh(
        World& world, const GeneratedTetMesh& generatedMesh, const TetMeshPhysicsComponentDesc& desc);

    ComponentExecutionPriority GetExecutionPriority() const override
    {
        return ComponentExecutionPriority::TetMeshPhysicsComponent;
    }

    int globalNodeBeginIndex = -1;
    int globalNodeCount = 0;
    std::vector<Vec3> nodeVelocities;
    Material material;
    FemModel selectedFemModel = FemModel::Corotational;
    bool physicsEnabled = true;

    void SetMaterial(const Material& value);
    void SetFemModel(FemModel value) { selectedFemModel = value; ++version; }
    FemModel GetFemModel() const { return selectedFemModel; }
    void RebuildFemRestData();
    // Per-element material edits (Tet::youngModulus etc.) take effect after this call.
    void RebuildTetFemCache() { ++version; }
    void SyncCurrentPositionsFromWorld(const World& world);

    int GetGlobalNodeBeginIndex() const { return globalNodeBeginIndex; }
    int GetGlobalNodeCount() const { return globalNodeCount; }
    int GetGlobalNodeIndex(int localNodeIndex) const override;
    bool SetTetActive(int tetIndex, bool active) override;

    void UpdateSystem(World& world, SolverData& solverData, float dt) override;
    void PostUpdate(World& world, float dt) override;

    // Bumped whenever rest data, material or tet activity changes.
    std::uint64_t version = 1;
    // nodePositions is the world's positions at the end of the last frame in which this
    // component was active (SyncCurrentPositionsFromWorld in PostUpdate).  The device keeps
    // that snapshot; the host copy is refreshed on access: snapshotWanted is the world's
    // snapshot generation this component's copy should show, snapshotLoaded the one it
    // holds.
    std::uint64_t snapshotWanted = 0, snapshotLoaded = 0;
    std::uint64_t snapshotEdits = 0;  // localEdits when the copy last became the frame-end snapshot
};

// ------------------------------------------------------------------ post-step geometry
// Render buffers built after the step (SurfaceExtractionComponent.cpp,
// SurfaceVisualComponent.cpp, VisualMeshComponent.cpp).  The per-frame updates run on the
// device when the positions they read are there (World::GeometrySystem): the frame-end
// snapshot behind a physics body's local copies, or the world's current positions.  The
// results stay on the device until a getter asks for them, so a frame costs no
// device-to-host copy of the nodes.  Otherwise (a plain tet mesh, local copies edited on
// the host, host-side state) the host computes them as the reference does.

// A device visual (pk_visual) on the world's device system and whether it holds a result
// the host buffers have not received yet.
struct DeviceVisual {
    pk_visual* visual = nullptr;
    pk_system* system = nullptr;
    bool pending = false;
    DeviceVisual() = default;
    DeviceVisual(const DeviceVisual&) = delete;
    DeviceVisual& operator=(const DeviceVisual&) = delete;
    ~DeviceVisual() { Release(); }
    void Release();
    // Copies a pending result (vertices: 3 floats each; normals may be null) and clears it.
    void Fetch(float* vertices, float* normals);
};

// SurfaceExtractionComponent (SurfaceExtractionComponent.cpp:138-250): the boundary faces
// of the host mesh's active tets, each oriented away from its tet's fourth node at the
// local current positions, rebuilt in PostUpdate when the host's topology changed.
class SurfaceExtractionComponent : public Component {
public:
    SurfaceExtractionComponent(ComponentHandle hostTetMeshHandle, std::uint64_t topologyEventsSeen);
    ComponentExecutionPriority GetExecutionPriority() const override
    {
        return ComponentExecutionPriority::SurfaceExtractionComponent;
    }
    ComponentHandle hostTetMeshHandle;
    std::vector<int> surfaceTriangleIndices;
    bool surfaceDirty = true;

    void RebuildSurface(World& world);
    const std::vector<int>& GetSurfaceTriangleIndices() const { return surfaceTriangleIndices; }
    ComponentHandle GetHostTetMeshHandle() const { return hostTetMeshHandle; }
    void PostUpdate(World& world, float dt) override;

private:
    std::uint64_t topologyEventsSeen = 0;
};

// SurfaceVisualComponent (SurfaceVisualComponent.cpp): three unshared vertices per surface
// triangle at the local current positions of its nodes, each with the triangle's flat
// normal.  The topology is rebuilt when the extraction's host mesh changed; the vertices
// and normals are recomputed every PostUpdate.
class SurfaceVisualComponent : public Component {
public:
    SurfaceVisualComponent(ComponentHandle surfaceExtractionHandle, std::uint64_t topologyEventsSeen);
    ComponentExecutionPriority GetExecutionPriority() const override
    {
        return ComponentExecutionPriority::SurfaceVisualComponent;
    }
    void RebuildVisualSurfaceTopology(World& world);
    void UpdateVisualSurfaceGeometry(World& world);
    const std::vector<Vec3>& GetVisualVertices() const;
    const std::vector<int>& GetVisualTriangleIndices() const { return visualTriangleIndices; }
    const std::vector<Vec3>& GetVisualNormals() const;
    ComponentHandle GetSurfaceExtractionHandle() const { return surfaceExtractionHandle; }
    void PostUpdate(World& world, float dt) override;
    void ReleaseDeviceResources() override;
    // Whether the last update ran on the device (extension, for tests).
    bool LastUpdateOnDevice() const { return lastOnDevice; }

private:
    void FetchDevice() const;
    ComponentHandle surfaceExtractionHandle;
    mutable std::vector<Vec3> visualVertices;
    std::vector<int> visualTriangleIndices;
    mutable std::vector<Vec3> visualNormals;
    std::vector<int> visualVertexSourceNodeIndices;
    bool topologyDirty = true;
    std::uint64_t topologyEventsSeen = 0;
    bool lastOnDevice = false;
    mutable DeviceVisual device;
    int deviceNodeCount = -1;  // the host mesh's node count the device visual was built for
};

// VisualMeshComponent::EmbeddedVertex (VisualMeshComponent.h:10-15).
struct EmbeddedVertex {
    int tetIndex = -1;
    Vec4 barycentric;
    bool valid = false;
};

// ComputeTetBarycentric (VisualMeshComponent.cpp:14-42): the barycentric coordinates of p
// in tet (a, b, c, d); false (and zeros) when |det| <= 1e-8.
bool ComputeTetBarycentric(const Vec3& p, const Vec3& a, const Vec3& b, const Vec3& c, const Vec3& d,
                           Vec4& outBarycentric);

// VisualMeshComponent (VisualMeshComponent.cpp): a render mesh embedded in the host tet
// mesh's rest shape (each vertex in the first active tet, in index order, that holds it
// within -1e-4 barycentric slack), deformed every PostUpdate with the world positions of
// that tet's nodes; triangles with a vertex outside the active tets are filtered out.
class VisualMeshComponent : public Component {
public:
    VisualMeshComponent(ComponentHandle hostTetMeshHandle, std::string debugEntityName,
                        std::uint64_t topologyEventsSeen);
    ComponentExecutionPriority GetExecutionPriority() const override
    {
        return ComponentExecutionPriority::VisualMeshComponent;
    }
    ComponentHandle hostTetMeshHandle;
    std::string debugEntityName;
    bool topologyDirty = false;
    std::vector<Vec3> restVisualVertices;
    std::vector<int> triangleIndices;
    std::vector<int> filteredTriangleIndices;
    std::vector<EmbeddedVertex> embeddedVertices;
    std::vector<bool> triangleValid;

    void SetVisualMesh(const Vec3* vertices, int vertexCount, const int* triangleIndices, int triangleIndexCount);
    void BuildEmbedding(World& world);
    void UpdateTriangleValidity(World& world);
    void UpdateDeformedVertices(World& world);
    const std::vector<Vec3>& GetDeformedVertices() const;
    const std::vector<int>& GetTriangleIndices() const { return filteredTriangleIndices; }
    void PostUpdate(World& world, float dt) override;
    void ReleaseDeviceResources() override;
    bool LastUpdateOnDevice() const { return lastOnDevice; }

private:
    void FetchDevice() const;
    mutable std::vector<Vec3> deformedVisualVertices;
    std::uint64_t topologyEventsSeen = 0;
    bool lastOnDevice = false;
    mutable DeviceVisual device;
    std::uint64_t embeddingVersion = 1;  // bumped by SetVisualMesh / BuildEmbedding
    std::uint64_t deviceEmbedding = 0;   // the embedding the device visual was built from
    std::uint64_t deviceBodyVersion = 0; // the host body's version its live flags follow
    std::vector<unsigned char> LiveFlags(const TetMeshComponent& host) const;
};

// ------------------------------------------------------------------ world
struct DeviceScene;

// A transient barycentric spring (PointConnection.h:12-26): the point sum_i w_i x(node_i)
// pulled towards targetPosition with `stiffness`, its velocity damped with `damping`.
// World::AddPointConnection keeps it until the end of the frame's World::Step.  Its
// contributions (PointConnection::UpdateSystem, PointConnection.cpp:55-140: the force
// times each corner's weight, blocks stiffness * w_i * w_j * I between its corners) are
// evaluated on the device during assembly.
struct PointConnection {
    int node0 = -1;
    int node1 = -1;
    int node2 = -1;
    int node3 = -1;
    Vec4 barycentric;
    Vec3 targetPosition;
    float stiffness = 0.0f;
    float damping = 0.0f;
};

class World {
public:
    World();
    ~World();
    World(const World&) = delete;
    World& operator=(const World&) = delete;

    void Step(float frameDt);

    int AddNode(const Vec3& position);
    ComponentHandle AddComponent(std::unique_ptr<Component> component);
    Component* GetComponent(ComponentHandle handle);
    const Component* GetComponent(ComponentHandle handle) const;
    void DestroyComponent(ComponentHandle handle);
    bool IsComponentHandleValid(ComponentHandle handle) const;

    void SetSubstepCount(int count);
    int GetSubstepCount() const { return substepCount; }
    void SetSolverMode(SolverMode mode) { solverMode = mode; }
    SolverMode GetSolverMode() const { return solverMode; }
    void SetConjugateGradientTolerance(float tolerance);
    float GetConjugateGradientTolerance() const { return conjugateGradientSettings.tolerance; }
    void SetConjugateGradientMaxIterations(int maxIterations);
    int GetConjugateGradientMaxIterations() const { return conjugateGradientSettings.maxIterations; }
    int GetLastConjugateGradientIterations() const;
    float GetLastConjugateGradientResidualNorm() const;
    bool DidLastConjugateGradientSolveConverge() const;
    void SetGravity(const Vec3& value) { gravity = value; }
    const Vec3& GetGravity() const { return gravity; }

    // Batched solve (extension): one PCG per TetMeshPhysicsComponent -- own scalars,
    // stopping test, iteration count and all-or-nothing integration, as a World holding
    // only that body -- instead of the reference's single coupled PCG over all bodies.
    void SetBatchedSolve(bool on);
    bool GetBatchedSolve() const { return batchedSolve; }
    // Last step's solve statistics of one body in batched mode; false if unavailable.
    bool GetBodyConjugateGradientStats(const Component* body, int& iterations, bool& converged, float& residualNorm,
                                       unsigned& flags) const;

    // Adjoint of one implicit substep (extension, no counterpart in the reference): with
    // the world at the state a substep of size dt starts from and the loss sensitivities
    // to the state after it (3 doubles per node each), writes the sensitivities to the
    // current state and adds each tet's log-Young's-modulus sensitivity to thetaBar
    // (tets of the tet-mesh physics components in creation order).  See
    // pk_system_adjoint_step.
    void AdjointStep(float dt, const double* xbarNext, const double* vbarNext, double* xbar, double* vbar,
                     double* thetaBar);

    // CUDA-graph capture of the device step (extension).
    void SetGraphCapture(bool on) { graphCapture = on; }
    // FP64 outer true-residual refinement passes for FP32 storage (extension; see
    // pk_system_set_refinement).  0: off.
    void SetRefinement(int passes)
    {
        const int p = passes < 0 ? 0 : passes;
        if (p > 0 && refinePasses == 0 && precision != Precision::FP64) ++topologyVersion;  // FP64 rest data
        refinePasses = p;
    }
    int GetRefinement() const { return refinePasses; }
    // Autotuner (extension): picks the fastest PCG kernel / tile or part size for the
    // current scene by timing `repeats` solves of the last assembled system (call after a
    // step).  Returns the chosen candidate index (see pk_system_autotune) or -1.
    int Autotune(int repeats, double* bestMs);
    // PCG kernel of the last solve (see pk_system_pcg_kernel) and its block count.
    int GetPcgKernel(int* blocks) const;
    // Stream form of the part-resident kernel in the last solve (pk_system_slab_form).
    int GetPcgStreamForm() const;

    // Device precision (extension).  Changing it rebuilds the device scene.
    void SetPrecision(Precision p);
    Precision GetPrecision() const { return precision; }
    void SetDevice(int device);

    Node& GetNode(int index);
    const Node& GetNode(int index) const;
    const std::vector<Node>& GetNodes() const { return nodes; }
    const Vec3& GetNodePosition(int nodeIndex) const;
    const Vec3& GetNodeVelocity(int nodeIndex) const;
    void SetNodePosition(int index, const Vec3& position);  // zeroes the velocity, as the reference does
    void SetNodeVelocity(int index, const Vec3& velocity);
    void SetNodeFixed(int nodeIndex, bool fixed);
    bool IsNodeFixed(int nodeIndex) const;
    void SetNodeActive(int nodeIndex, bool active);
    const std::vector<std::unique_ptr<Component>>& GetComponents() const { return components; }

    // Transient point connections (World.cpp:126-131, 727-759): added if its four nodes
    // exist and are active; cleared when the next World::Step ends (those added during a
    // substep, after that substep).
    void AddPointConnection(const PointConnection& connection);
    // A collision sphere asks for this substep's contacts (CollisionSphereComponent::UpdateSystem).
    void RequestSphereContacts(const CollisionSphereComponent* sphere) { sphereRequests.push_back(sphere); }
    int GetTransientConnectionCount() const { return static_cast<int>(transientConnections.size()); }
    bool HasValidNodeIndices(const PointConnection& connection) const;

    // Bulk state access (extension): 3 floats (or doubles) per node, world order.
    void GetNodeStates(float* positions, float* velocities) const;
    void SetNodeStates(const float* positions, const float* velocities);
    void GetNodeStatesF64(double* positions, double* velocities) const;
    void SetNodeStatesF64(const double* positions, const double* velocities);

    // Device access for measurement and tests (extension).
    pk_system* GetDeviceSystem();
    // Whether the device holds the pattern the host scene describes (a prepare after the
    // end of a frame with point connections changes the host's before the next upload).
    bool SceneMatchesDevice() const;
    // Builds the host side of the device scene (and uploads it when `upload`): runs the
    // components' UpdateSystem pass, then mass / mapping / pattern.  Returns dynamic rows.
    int PrepareScene(bool upload);
    int GetSceneDynamicCount() const;
    int GetSceneBlockCount() const;
    int GetSceneTetCount() const;
    const std::vector<int>* GetSceneRowStart() const;
    const std::vector<int>* GetSceneColIndex() const;
    const std::vector<int>* GetSceneNodeToDyn() const;
    const std::vector<double>* GetSceneMass() const;
    unsigned GetLastStepFlags() const;
    // Brings a component's nodePositions up to the snapshot of the last substep it took part
    // in (TetMeshPhysicsComponent::SyncCurrentPositionsFromWorld, done lazily).
    void RefreshLocalPositions(TetMeshPhysicsComponent& component) const;
    std::uint64_t GetSnapshotGeneration() const { return snapshotGeneration; }
    // This substep's valid host-emitted masses (node, mass, after its body's lumped masses).
    const std::vector<std::tuple<int, float, bool>>& GetExtraMasses() const { return extras.masses; }
    // The device system when it holds the positions a post-step geometry update reads:
    // `body`'s frame-end local copies (snapshot, while the host copy has not been loaded
    // or edited) or the world's current positions; nullptr when only the host has them.
    pk_system* GeometrySystem(const TetMeshPhysicsComponent* body, bool snapshot) const;
    void MarkTopologyDirty() { ++topologyVersion; }
    std::uint64_t GetTopologyVersion() const { return topologyVersion; }

private:
    friend class TetMeshPhysicsComponent;
    void EnsureHostState() const;
    void SyncStats() const;
    void PreUpdateComponents(float dt);
    void PostUpdateComponents(float dt);
    void RunSubstep(float dt);
    void CollectContributions(float dt);
    void EnsureScene(bool upload);
    void FlushLocalPositionSnapshots();  // host copies of every stale component snapshot
    void ReleaseDeviceScene();           // state, local copies and visuals to the host, then drop the system
    void AddSphereContacts();            // the requested spheres' contacts as point connections
    void SnapshotPositions();            // the frame's end positions for the components' copies
    bool SyncConnections();
    void MarkSubstepConnectionBegin() { firstSubstepConnectionIndex = transientConnections.size(); }
    void ClearSubstepConnections();
    void ClearFrameConnections();

    std::vector<Node> nodes;
    mutable std::vector<Vec3> positions;
    mutable std::vector<Vec3> velocities;
    mutable bool hostStale = false;   // device holds newer state than the host copies
    bool deviceStale = true;          // host copies hold newer state than the device

    std::vector<std::unique_ptr<Component>> components;
    std::vector<std::uint32_t> componentGenerations;
    std::vector<std::uint32_t> freeComponentSlots;
    std::multimap<int, Component*> orderedComponents;

    int substepCount = 1;
    SolverMode solverMode = SolverMode::Explicit;
    ConjugateGradientSettings conjugateGradientSettings;
    Vec3 gravity{};
    Precision precision = Precision::FP32;
    int device = 0;
    bool batchedSolve = false;
    bool graphCapture = false;
    int refinePasses = 0;
    float lastSubstepDt = 0.0f;
    std::uint64_t topologyVersion = 1;

    std::vector<PointConnection> transientConnections;
    std::size_t firstSubstepConnectionIndex = 0;
    std::uint64_t connectionVersion = 1;  // bumped whenever transientConnections changes

    SolverData solverData;
    std::unique_ptr<DeviceScene> scene;
    mutable ConjugateGradientResult lastConjugateGradientResult;
    mutable unsigned lastFlags = 0;
    mutable bool statsPending = false;
    std::uint64_t snapshotGeneration = 0;  // frames whose end positions the device snapshot held
    bool snapshotOnDevice = false;         // the device holds snapshot `snapshotGeneration`
    std::vector<const CollisionSphereComponent*> sphereRequests;  // this substep's, in update order
    // Host-emitted SolverData contributions of this substep (custom components'
    // AddNodeMass / AddNodeForce / AddStiffnessBlock), sorted out for the device step.
    struct Extras {
        bool any = false;     // some contribution was emitted
        bool failed = false;  // a non-finite stiffness block: the step is not applied
        // valid masses in emission order: node, mass, whether it comes after the node's
        // soft body's own lumped masses
        std::vector<std::tuple<int, float, bool>> masses;
        std::vector<Vec3> force;  // per world node (empty: no force)
        std::vector<SolverData::StiffnessBlock> blocks;  // those with both nodes in range
    } extras;
    void BuildExtras();
    bool SyncExtras(std::vector<std::pair<int, int>>& pairs);  // device lists; adds the blocks' pattern pairs
};

}  // namespace PhysiK
