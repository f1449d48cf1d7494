// The PHYSIK_* C ABI (include/physik_b200.h) over the host World.  Behaviour follows
// the reference's src/API/PhysiKAPI.cpp for the soft-body path; every exception is
// caught at this boundary and recorded for PHYSIK_B200_GetLastError.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <string>
#include <unordered_set>
#include <vector>

#include "../../../include/physik_b200.h"
#include "../../../include/pkcuda.h"
#include "physik_core.h"

using namespace PhysiK;

namespace {

thread_local std::string g_error;
std::unordered_set<GeneratedTetMesh*> g_meshes;  // live generated meshes (PhysiKAPI.cpp:24)

World* AsWorld(PhysikWorldHandle h) { return static_cast<World*>(h); }

GeneratedTetMesh* AsMesh(PhysikGeneratedTetMeshHandle h)
{
    auto* m = static_cast<GeneratedTetMesh*>(h);
    return (m && g_meshes.count(m)) ? m : nullptr;
}

ComponentHandle ToHandle(PhysikComponentHandle h) { return ComponentHandle{h.index, h.generation}; }
PhysikComponentHandle FromHandle(ComponentHandle h) { return PhysikComponentHandle{h.index, h.generation}; }
PhysikComponentHandle InvalidHandle() { return PhysikComponentHandle{0xFFFFFFFFu, 0u}; }

TetMeshComponent* AsTetMesh(World* w, PhysikComponentHandle h)
{
    return w ? dynamic_cast<TetMeshComponent*>(w->GetComponent(ToHandle(h))) : nullptr;
}
TetMeshPhysicsComponent* AsTetMeshPhysics(World* w, PhysikComponentHandle h)
{
    return w ? dynamic_cast<TetMeshPhysicsComponent*>(w->GetComponent(ToHandle(h))) : nullptr;
}

bool ValidNode(const World& w, int i) { return i >= 0 && i < static_cast<int>(w.GetNodes().size()); }

Material ToMaterial(const PhysikMaterialDesc& d)
{
    Material m;
    m.density = d.density;
    m.youngModulus = d.youngModulus;
    m.poissonRatio = d.poissonRatio;
    m.damping = d.damping;
    return m;
}

// A node stays active while some active tet of an active tet mesh references it
// (ReconcileTetNodeActiveStates, PhysiKAPI.cpp:159-229).
void ReconcileNodes(World& w, const TetMeshComponent& mesh, int tetIndex)
{
    for (int corner = 0; corner < 4; ++corner) {
        const int g = mesh.GetGlobalNodeIndex(mesh.GetTetNodeIndex(tetIndex, corner));
        if (!ValidNode(w, g)) continue;
        // Any active tet of an active mesh with g as a corner (through each mesh's cached
        // node-to-tet lists instead of a scan of every tet).
        bool referenced = false;
        for (const auto& c : w.GetComponents()) {
            const auto* tm = dynamic_cast<const TetMeshComponent*>(c.get());
            if (!tm || !tm->active) continue;
            const int local = tm->GetLocalNodeIndexOf(g);
            if (local >= 0 && tm->HasActiveTetAtLocalNode(local)) {
                referenced = true;
                break;
            }
        }
        w.SetNodeActive(g, referenced);
    }
}

template <class F>
auto Guard(F&& f, decltype(f()) fallback) -> decltype(f())
{
    try {
        return f();
    } catch (const std::exception& e) {
        g_error = e.what();
    } catch (...) {
        g_error = "unknown error";
    }
    return fallback;
}

template <class F>
void GuardVoid(F&& f)
{
    try {
        f();
    } catch (const std::exception& e) {
        g_error = e.what();
    } catch (...) {
        g_error = "unknown error";
    }
}

}  // namespace

extern "C" {

PHYSIK_B200_API PhysikWorldHandle PHYSIK_CreateWorld(void)
{
    return Guard([]() -> PhysikWorldHandle { return new World(); }, nullptr);
}

PHYSIK_B200_API void PHYSIK_DestroyWorld(PhysikWorldHandle world)
{
    GuardVoid([&] { delete AsWorld(world); });
}

PHYSIK_B200_API void PHYSIK_Step(PhysikWorldHandle world, float dt)
{
    if (World* w = AsWorld(world)) GuardVoid([&] { w->Step(dt); });
}

PHYSIK_B200_API void PHYSIK_SetSubstepCount(PhysikWorldHandle world, int substepCount)
{
    if (World* w = AsWorld(world)) w->SetSubstepCount(substepCount);
}

PHYSIK_B200_API void PHYSIK_SetSolverMode(PhysikWorldHandle world, int mode)
{
    if (World* w = AsWorld(world)) w->SetSolverMode(mode == 1 ? SolverMode::ImplicitEuler : SolverMode::Explicit);
}

PHYSIK_B200_API void PHYSIK_SetConjugateGradientTolerance(PhysikWorldHandle world, float tolerance)
{
    if (World* w = AsWorld(world)) w->SetConjugateGradientTolerance(tolerance);
}

PHYSIK_B200_API float PHYSIK_GetConjugateGradientTolerance(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    return w ? w->GetConjugateGradientTolerance() : 0.0f;
}

PHYSIK_B200_API void PHYSIK_SetConjugateGradientMaxIterations(PhysikWorldHandle world, int maxIterations)
{
    if (World* w = AsWorld(world)) w->SetConjugateGradientMaxIterations(maxIterations);
}

PHYSIK_B200_API int PHYSIK_GetConjugateGradientMaxIterations(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    return w ? w->GetConjugateGradientMaxIterations() : 0;
}

PHYSIK_B200_API int PHYSIK_GetLastConjugateGradientIterations(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    return w ? Guard([&] { return w->GetLastConjugateGradientIterations(); }, 0) : 0;
}

PHYSIK_B200_API float PHYSIK_GetLastConjugateGradientResidualNorm(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    return w ? Guard([&] { return w->GetLastConjugateGradientResidualNorm(); }, 0.0f) : 0.0f;
}

PHYSIK_B200_API int PHYSIK_DidLastConjugateGradientSolveConverge(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    return w ? Guard([&] { return w->DidLastConjugateGradientSolveConverge() ? 1 : 0; }, 0) : 0;
}

PHYSIK_B200_API void PHYSIK_SetGravity(PhysikWorldHandle world, float x, float y, float z)
{
    if (World* w = AsWorld(world)) w->SetGravity(Vec3{x, y, z});
}

PHYSIK_B200_API int PHYSIK_AddNode(PhysikWorldHandle world, float x, float y, float z)
{
    World* w = AsWorld(world);
    return w ? Guard([&] { return w->AddNode(Vec3{x, y, z}); }, -1) : -1;
}

PHYSIK_B200_API void PHYSIK_SetNodeFixed(PhysikWorldHandle world, int nodeIndex, int fixed)
{
    World* w = AsWorld(world);
    if (w && ValidNode(*w, nodeIndex)) GuardVoid([&] { w->SetNodeFixed(nodeIndex, fixed != 0); });
}

PHYSIK_B200_API int PHYSIK_IsNodeFixed(PhysikWorldHandle world, int nodeIndex)
{
    World* w = AsWorld(world);
    return (w && ValidNode(*w, nodeIndex) && w->IsNodeFixed(nodeIndex)) ? 1 : 0;
}

PHYSIK_B200_API PhysikGeneratedTetMeshHandle PHYSIK_GenerateTetMesh(const PhysikVec3* positions, int nodeCount,
                                                                     const int* tetLocalNodeIndices, int tetCount)
{
    return Guard(
        [&]() -> PhysikGeneratedTetMeshHandle {
            auto* m = new GeneratedTetMesh(TetMeshGenerator::Generate(reinterpret_cast<const Vec3*>(positions),
                                                                      nodeCount, tetLocalNodeIndices, tetCount));
            g_meshes.insert(m);
            return m;
        },
        nullptr);
}

PHYSIK_B200_API int PHYSIK_IsGeneratedTetMeshHandleValid(PhysikGeneratedTetMeshHandle mesh)
{
    return AsMesh(mesh) ? 1 : 0;
}

PHYSIK_B200_API void PHYSIK_DestroyGeneratedTetMesh(PhysikGeneratedTetMeshHandle mesh)
{
    GeneratedTetMesh* m = AsMesh(mesh);
    if (!m) return;
    g_meshes.erase(m);
    delete m;
}

PHYSIK_B200_API int PHYSIK_GetGeneratedTetMeshVertexCount(PhysikGeneratedTetMeshHandle mesh)
{
    const GeneratedTetMesh* m = AsMesh(mesh);
    return m ? static_cast<int>(m->positions.size()) : 0;
}

PHYSIK_B200_API int PHYSIK_GetGeneratedTetMeshTetCount(PhysikGeneratedTetMeshHandle mesh)
{
    const GeneratedTetMesh* m = AsMesh(mesh);
    return m ? static_cast<int>(m->tetLocalNodeIndices.size() / 4u) : 0;
}

PHYSIK_B200_API int PHYSIK_GetGeneratedTetMeshTetIndexCount(PhysikGeneratedTetMeshHandle mesh)
{
    const GeneratedTetMesh* m = AsMesh(mesh);
    return m ? static_cast<int>(m->tetLocalNodeIndices.size()) : 0;
}

PHYSIK_B200_API int PHYSIK_GetGeneratedTetMeshVertex(PhysikGeneratedTetMeshHandle mesh, int vertexIndex, float* outX,
                                                     float* outY, float* outZ)
{
    const GeneratedTetMesh* m = AsMesh(mesh);
    if (!m || !outX || !outY || !outZ || vertexIndex < 0 || vertexIndex >= static_cast<int>(m->positions.size()))
        return 0;
    const Vec3& p = m->positions[static_cast<std::size_t>(vertexIndex)];
    *outX = p.x;
    *outY = p.y;
    *outZ = p.z;
    return 1;
}

PHYSIK_B200_API int PHYSIK_GetGeneratedTetMeshTetNodeIndex(PhysikGeneratedTetMeshHandle mesh, int i, int* out)
{
    const GeneratedTetMesh* m = AsMesh(mesh);
    if (!m || !out || i < 0 || i >= static_cast<int>(m->tetLocalNodeIndices.size())) return 0;
    *out = m->tetLocalNodeIndices[static_cast<std::size_t>(i)];
    return 1;
}

PHYSIK_B200_API PhysikComponentHandle PHYSIK_CreateCollisionSphereComponent(PhysikWorldHandle world, float x, float y,
                                                                            float z, float radius)
{
    World* w = AsWorld(world);
    if (!w) return InvalidHandle();
    return Guard([&] { return FromHandle(w->AddComponent(CollisionSphereComponent::Create(Vec3{x, y, z}, radius))); },
                 InvalidHandle());
}

PHYSIK_B200_API void PHYSIK_SetCollisionSphereConnectionSettings(PhysikWorldHandle world,
                                                                 PhysikComponentHandle sphereComponent,
                                                                 float stiffness, float damping)
{
    World* w = AsWorld(world);
    auto* c = w ? dynamic_cast<CollisionSphereComponent*>(w->GetComponent(ToHandle(sphereComponent))) : nullptr;
    if (c) c->SetConnectionSettings(stiffness, damping);
}

PHYSIK_B200_API void PHYSIK_GetCollisionSphereConnectionSettings(PhysikWorldHandle world,
                                                                 PhysikComponentHandle sphereComponent,
                                                                 float* outStiffness, float* outDamping)
{
    World* w = AsWorld(world);
    auto* c = w ? dynamic_cast<CollisionSphereComponent*>(w->GetComponent(ToHandle(sphereComponent))) : nullptr;
    if (!c) return;
    if (outStiffness) *outStiffness = c->GetConnectionStiffness();
    if (outDamping) *outDamping = c->GetConnectionDamping();
}

PHYSIK_B200_API void PHYSIK_SetCollisionComponentKinematicTarget(PhysikWorldHandle world,
                                                                 PhysikComponentHandle component, float x, float y,
                                                                 float z)
{
    World* w = AsWorld(world);
    auto* c = w ? dynamic_cast<CollisionComponent*>(w->GetComponent(ToHandle(component))) : nullptr;
    if (!c) return;
    Transform target = c->transform;
    target.position = Vec3{x, y, z};
    c->SetKinematicTarget(target);
}

PHYSIK_B200_API PhysikComponentHandle PHYSIK_B200_CreateContributionComponent(PhysikWorldHandle world, int priority)
{
    World* w = AsWorld(world);
    if (!w) return InvalidHandle();
    return Guard([&] { return FromHandle(w->AddComponent(std::make_unique<ContributionComponent>(priority))); },
                 InvalidHandle());
}

PHYSIK_B200_API void PHYSIK_B200_SetContributionCallback(PhysikWorldHandle world, PhysikComponentHandle component,
                                                         PhysikContributionCallback callback, void* userData)
{
    World* w = AsWorld(world);
    auto* c = w ? dynamic_cast<ContributionComponent*>(w->GetComponent(ToHandle(component))) : nullptr;
    if (c) c->SetCallback(reinterpret_cast<ContributionCallback>(callback), userData);
}

PHYSIK_B200_API void PHYSIK_B200_SolverDataAddNodeForce(void* solverData, int node, float fx, float fy, float fz)
{
    if (solverData) static_cast<SolverData*>(solverData)->AddNodeForce(node, Vec3{fx, fy, fz});
}

PHYSIK_B200_API void PHYSIK_B200_SolverDataAddNodeMass(void* solverData, int node, float mass)
{
    if (solverData) static_cast<SolverData*>(solverData)->AddNodeMass(node, mass);
}

PHYSIK_B200_API void PHYSIK_B200_SolverDataAddStiffnessBlock(void* solverData, int nodeA, int nodeB,
                                                             const float* block9)
{
    if (!solverData || !block9) return;
    const Mat3 b = Mat3::FromColumns(Vec3{block9[0], block9[1], block9[2]}, Vec3{block9[3], block9[4], block9[5]},
                                     Vec3{block9[6], block9[7], block9[8]});
    static_cast<SolverData*>(solverData)->AddStiffnessBlock(nodeA, nodeB, b);
}

PHYSIK_B200_API PhysikComponentHandle PHYSIK_CreateScriptComponent(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    if (!w) return InvalidHandle();
    return Guard([&] { return FromHandle(w->AddComponent(std::make_unique<ScriptComponent>())); }, InvalidHandle());
}

PHYSIK_B200_API void PHYSIK_SetScriptComponentCallback(PhysikWorldHandle world, PhysikComponentHandle scriptComponent,
                                                       PhysikExternalLogicCallback callback, void* userData)
{
    World* w = AsWorld(world);
    auto* c = w ? dynamic_cast<ScriptComponent*>(w->GetComponent(ToHandle(scriptComponent))) : nullptr;
    if (c) c->SetExternalLogicCallback(reinterpret_cast<ExternalLogicCallback>(callback), userData);
}

PHYSIK_B200_API void PHYSIK_ClearScriptComponentCallback(PhysikWorldHandle world, PhysikComponentHandle scriptComponent)
{
    World* w = AsWorld(world);
    auto* c = w ? dynamic_cast<ScriptComponent*>(w->GetComponent(ToHandle(scriptComponent))) : nullptr;
    if (c) c->ClearExternalLogicCallback();
}

// ---- post-step geometry (PhysiKAPI.cpp:703-717, 767-980, 1055-1170) ----
namespace {
SurfaceExtractionComponent* AsSurfaceExtraction(World* w, PhysikComponentHandle h)
{
    return w ? dynamic_cast<SurfaceExtractionComponent*>(w->GetComponent(ToHandle(h))) : nullptr;
}
SurfaceVisualComponent* AsSurfaceVisual(World* w, PhysikComponentHandle h)
{
    return w ? dynamic_cast<SurfaceVisualComponent*>(w->GetComponent(ToHandle(h))) : nullptr;
}
VisualMeshComponent* AsVisualMesh(World* w, PhysikComponentHandle h)
{
    return w ? dynamic_cast<VisualMeshComponent*>(w->GetComponent(ToHandle(h))) : nullptr;
}
// Writes element i of a vector of Vec3 (getters fetch a pending device result first).
int GetVec3(const std::vector<Vec3>& v, int i, float* x, float* y, float* z)
{
    if (i < 0 || i >= static_cast<int>(v.size())) return 0;
    *x = v[static_cast<std::size_t>(i)].x;
    *y = v[static_cast<std::size_t>(i)].y;
    *z = v[static_cast<std::size_t>(i)].z;
    return 1;
}
}  // namespace

PHYSIK_B200_API PhysikComponentHandle PHYSIK_CreateSurfaceExtractionComponent(PhysikWorldHandle world,
                                                                              PhysikComponentHandle hostTetMesh)
{
    World* w = AsWorld(world);
    TetMeshComponent* host = AsTetMesh(w, hostTetMesh);
    if (!w || !host) return InvalidHandle();
    return Guard(
        [&] {
            return FromHandle(w->AddComponent(
                std::make_unique<SurfaceExtractionComponent>(ToHandle(hostTetMesh), host->topologyEvents)));
        },
        InvalidHandle());
}

PHYSIK_B200_API int PHYSIK_GetSurfaceTriangleIndexCount(PhysikWorldHandle world, PhysikComponentHandle surfaceExtraction)
{
    const SurfaceExtractionComponent* c = AsSurfaceExtraction(AsWorld(world), surfaceExtraction);
    return c ? static_cast<int>(c->GetSurfaceTriangleIndices().size()) : 0;
}

PHYSIK_B200_API int PHYSIK_CopySurfaceTriangleIndices(PhysikWorldHandle world, PhysikComponentHandle surfaceExtraction,
                                                      int* outIndices, int maxIndexCount)
{
    if (!outIndices || maxIndexCount <= 0) return 0;
    const SurfaceExtractionComponent* c = AsSurfaceExtraction(AsWorld(world), surfaceExtraction);
    if (!c) return 0;
    const std::vector<int>& v = c->GetSurfaceTriangleIndices();
    const int n = std::min(maxIndexCount, static_cast<int>(v.size()));
    std::copy(v.begin(), v.begin() + n, outIndices);
    return n;
}

PHYSIK_B200_API PhysikComponentHandle PHYSIK_CreateSurfaceVisualComponent(PhysikWorldHandle world,
                                                                          PhysikComponentHandle surfaceExtraction)
{
    World* w = AsWorld(world);
    const SurfaceExtractionComponent* ex = AsSurfaceExtraction(w, surfaceExtraction);
    if (!w || !ex) return InvalidHandle();
    const TetMeshComponent* host = AsTetMesh(w, FromHandle(ex->GetHostTetMeshHandle()));
    const std::uint64_t seen = host ? host->topologyEvents : 0;
    return Guard(
        [&] {
            return FromHandle(
                w->AddComponent(std::make_unique<SurfaceVisualComponent>(ToHandle(surfaceExtraction), seen)));
        },
        InvalidHandle());
}

PHYSIK_B200_API int PHYSIK_GetSurfaceVisualVertexCount(PhysikWorldHandle world, PhysikComponentHandle surfaceVisual)
{
    const SurfaceVisualComponent* c = AsSurfaceVisual(AsWorld(world), surfaceVisual);
    return c ? Guard([&] { return static_cast<int>(c->GetVisualVertices().size()); }, 0) : 0;
}

PHYSIK_B200_API int PHYSIK_GetSurfaceVisualTriangleIndexCount(PhysikWorldHandle world,
                                                              PhysikComponentHandle surfaceVisual)
{
    const SurfaceVisualComponent* c = AsSurfaceVisual(AsWorld(world), surfaceVisual);
    return c ? static_cast<int>(c->GetVisualTriangleIndices().size()) : 0;
}

PHYSIK_B200_API int PHYSIK_GetSurfaceVisualNormalCount(PhysikWorldHandle world, PhysikComponentHandle surfaceVisual)
{
    const SurfaceVisualComponent* c = AsSurfaceVisual(AsWorld(world), surfaceVisual);
    return c ? Guard([&] { return static_cast<int>(c->GetVisualNormals().size()); }, 0) : 0;
}

PHYSIK_B200_API int PHYSIK_GetSurfaceVisualVertex(PhysikWorldHandle world, PhysikComponentHandle surfaceVisual,
                                                  int visualVertexIndex, float* outX, float* outY, float* outZ)
{
    if (!outX || !outY || !outZ) return 0;
    const SurfaceVisualComponent* c = AsSurfaceVisual(AsWorld(world), surfaceVisual);
    if (!c) return 0;
    return Guard([&] { return GetVec3(c->GetVisualVertices(), visualVertexIndex, outX, outY, outZ); }, 0);
}

PHYSIK_B200_API int PHYSIK_GetSurfaceVisualTriangleIndex(PhysikWorldHandle world, PhysikComponentHandle surfaceVisual,
                                                         int triangleIndexArrayIndex, int* outIndex)
{
    if (!outIndex) return 0;
    const SurfaceVisualComponent* c = AsSurfaceVisual(AsWorld(world), surfaceVisual);
    if (!c) return 0;
    const std::vector<int>& v = c->GetVisualTriangleIndices();
    if (triangleIndexArrayIndex < 0 || triangleIndexArrayIndex >= static_cast<int>(v.size())) return 0;
    *outIndex = v[static_cast<std::size_t>(triangleIndexArrayIndex)];
    return 1;
}

PHYSIK_B200_API int PHYSIK_GetSurfaceVisualNormal(PhysikWorldHandle world, PhysikComponentHandle surfaceVisual,
                                                  int visualNormalIndex, float* outX, float* outY, float* outZ)
{
    if (!outX || !outY || !outZ) return 0;
    const SurfaceVisualComponent* c = AsSurfaceVisual(AsWorld(world), surfaceVisual);
    if (!c) return 0;
    return Guard([&] { return GetVec3(c->GetVisualNormals(), visualNormalIndex, outX, outY, outZ); }, 0);
}

PHYSIK_B200_API PhysikComponentHandle PHYSIK_CreateVisualMeshComponent(PhysikWorldHandle world,
                                                                       PhysikComponentHandle hostTetMesh)
{
    World* w = AsWorld(world);
    TetMeshComponent* host = AsTetMesh(w, hostTetMesh);
    if (!w || !host) return InvalidHandle();
    return Guard(
        [&] {
            return FromHandle(w->AddComponent(
                std::make_unique<VisualMeshComponent>(ToHandle(hostTetMesh), std::string{}, host->topologyEvents)));
        },
        InvalidHandle());
}

PHYSIK_B200_API void PHYSIK_SetVisualMeshData(PhysikWorldHandle world, PhysikComponentHandle visualMesh,
                                              const PhysikVec3* vertices, int vertexCount, const int* triangleIndices,
                                              int triangleIndexCount)
{
    VisualMeshComponent* c = AsVisualMesh(AsWorld(world), visualMesh);
    if (!c) return;
    GuardVoid([&] {
        c->SetVisualMesh(reinterpret_cast<const Vec3*>(vertices), vertexCount, triangleIndices, triangleIndexCount);
    });
}

PHYSIK_B200_API int PHYSIK_BuildVisualMeshEmbedding(PhysikWorldHandle world, PhysikComponentHandle visualMesh)
{
    World* w = AsWorld(world);
    VisualMeshComponent* c = AsVisualMesh(w, visualMesh);
    if (!w || !c) return 0;
    return Guard(
        [&] {
            c->BuildEmbedding(*w);
            for (const EmbeddedVertex& e : c->embeddedVertices)
                if (e.valid) return 1;
            return 0;
        },
        0);
}

PHYSIK_B200_API int PHYSIK_GetVisualMeshVertexCount(PhysikWorldHandle world, PhysikComponentHandle visualMesh)
{
    const VisualMeshComponent* c = AsVisualMesh(AsWorld(world), visualMesh);
    return c ? Guard([&] { return static_cast<int>(c->GetDeformedVertices().size()); }, 0) : 0;
}

PHYSIK_B200_API int PHYSIK_GetVisualMeshTriangleIndexCount(PhysikWorldHandle world, PhysikComponentHandle visualMesh)
{
    const VisualMeshComponent* c = AsVisualMesh(AsWorld(world), visualMesh);
    return c ? static_cast<int>(c->GetTriangleIndices().size()) : 0;
}

PHYSIK_B200_API int PHYSIK_CopyVisualMeshVertices(PhysikWorldHandle world, PhysikComponentHandle visualMesh,
                                                  PhysikVec3* outVertices, int maxVertexCount)
{
    if (!outVertices || maxVertexCount <= 0) return 0;
    const VisualMeshComponent* c = AsVisualMesh(AsWorld(world), visualMesh);
    if (!c) return 0;
    return Guard(
        [&] {
            const std::vector<Vec3>& v = c->GetDeformedVertices();
            const int n = std::min(maxVertexCount, static_cast<int>(v.size()));
            for (int i = 0; i < n; ++i)
                outVertices[i] = PhysikVec3{v[static_cast<std::size_t>(i)].x, v[static_cast<std::size_t>(i)].y,
                                            v[static_cast<std::size_t>(i)].z};
            return n;
        },
        0);
}

PHYSIK_B200_API int PHYSIK_CopyVisualMeshTriangleIndices(PhysikWorldHandle world, PhysikComponentHandle visualMesh,
                                                         int* outIndices, int maxIndexCount)
{
    if (!outIndices || maxIndexCount <= 0) return 0;
    const VisualMeshComponent* c = AsVisualMesh(AsWorld(world), visualMesh);
    if (!c) return 0;
    const std::vector<int>& v = c->GetTriangleIndices();
    const int n = std::min(maxIndexCount, static_cast<int>(v.size()));
    std::copy(v.begin(), v.begin() + n, outIndices);
    return n;
}

// Whether a surface visual's / visual mesh's last update ran on the device (extension).
PHYSIK_B200_API int PHYSIK_B200_GetVisualUpdateOnDevice(PhysikWorldHandle world, PhysikComponentHandle visual)
{
    World* w = AsWorld(world);
    if (const SurfaceVisualComponent* s = AsSurfaceVisual(w, visual)) return s->LastUpdateOnDevice() ? 1 : 0;
    if (const VisualMeshComponent* m = AsVisualMesh(w, visual)) return m->LastUpdateOnDevice() ? 1 : 0;
    return -1;
}

PHYSIK_B200_API PhysikComponentHandle PHYSIK_CreateTetMeshComponent(PhysikWorldHandle world,
                                                                     PhysikGeneratedTetMeshHandle mesh)
{
    World* w = AsWorld(world);
    const GeneratedTetMesh* m = AsMesh(mesh);
    if (!w || !m || m->positions.empty() || m->tetLocalNodeIndices.empty()) return InvalidHandle();
    return Guard(
        [&] {
            auto c = std::make_unique<TetMeshComponent>();
            c->SetGeometry(*m);
            return FromHandle(w->AddComponent(std::move(c)));
        },
        InvalidHandle());
}

PHYSIK_B200_API PhysikComponentHandle PHYSIK_CreateTetMeshPhysicsComponent(PhysikWorldHandle world,
                                                                            PhysikGeneratedTetMeshHandle mesh,
                                                                            const PhysikMaterialDesc* material)
{
    World* w = AsWorld(world);
    const GeneratedTetMesh* m = AsMesh(mesh);
    if (!w || !m || !material || m->positions.empty() || m->tetLocalNodeIndices.empty()) return InvalidHandle();
    return Guard(
        [&] {
            auto c = TetMeshPhysicsComponent::CreateFromGeneratedTetMesh(*w, *m, ToMaterial(*material));
            return FromHandle(w->AddComponent(std::move(c)));
        },
        InvalidHandle());
}

PHYSIK_B200_API int PHYSIK_GetTetMeshGlobalNodeBeginIndex(PhysikWorldHandle world, PhysikComponentHandle tetMesh)
{
    const TetMeshPhysicsComponent* c = AsTetMeshPhysics(AsWorld(world), tetMesh);
    return c ? c->GetGlobalNodeBeginIndex() : -1;
}

PHYSIK_B200_API int PHYSIK_GetTetMeshGlobalNodeCount(PhysikWorldHandle world, PhysikComponentHandle tetMesh)
{
    const TetMeshPhysicsComponent* c = AsTetMeshPhysics(AsWorld(world), tetMesh);
    return c ? c->GetGlobalNodeCount() : -1;
}

PHYSIK_B200_API int PHYSIK_GetTetMeshGlobalNodeIndex(PhysikWorldHandle world, PhysikComponentHandle tetMesh,
                                                     int localNodeIndex)
{
    const TetMeshPhysicsComponent* c = AsTetMeshPhysics(AsWorld(world), tetMesh);
    return c ? c->GetGlobalNodeIndex(localNodeIndex) : -1;
}

PHYSIK_B200_API int PHYSIK_SetTetMeshLocalCurrentPosition(PhysikWorldHandle world, PhysikComponentHandle tetMesh,
                                                          int localNodeIndex, float x, float y, float z)
{
    World* w = AsWorld(world);
    TetMeshComponent* c = AsTetMesh(w, tetMesh);
    if (!c || localNodeIndex < 0 || localNodeIndex >= c->GetNodeCount()) return 0;
    return Guard(
        [&]() -> int {
            if (auto* p = dynamic_cast<TetMeshPhysicsComponent*>(c)) w->RefreshLocalPositions(*p);
            c->SetLocalCurrentPosition(localNodeIndex, Vec3{x, y, z});
            return 1;
        },
        0);
}

PHYSIK_B200_API int PHYSIK_GetTetMeshLocalCurrentPosition(PhysikWorldHandle world, PhysikComponentHandle tetMesh,
                                                          int localNodeIndex, float* outX, float* outY, float* outZ)
{
    World* w = AsWorld(world);
    if (!w || !outX || !outY || !outZ) return 0;
    TetMeshComponent* c = AsTetMesh(w, tetMesh);
    if (!c || localNodeIndex < 0 || localNodeIndex >= c->GetNodeCount()) return 0;
    return Guard(
        [&]() -> int {
            if (auto* p = dynamic_cast<TetMeshPhysicsComponent*>(c)) w->RefreshLocalPositions(*p);
            const Vec3& v = c->GetLocalCurrentPosition(localNodeIndex);
            *outX = v.x;
            *outY = v.y;
            *outZ = v.z;
            return 1;
        },
        0);
}

PHYSIK_B200_API void PHYSIK_SetTetMeshMaterial(PhysikWorldHandle world, PhysikComponentHandle component,
                                               const PhysikMaterialDesc* material)
{
    TetMeshPhysicsComponent* c = AsTetMeshPhysics(AsWorld(world), component);
    if (c && material) c->SetMaterial(ToMaterial(*material));
}

PHYSIK_B200_API void PHYSIK_DestroyComponent(PhysikWorldHandle world, PhysikComponentHandle component)
{
    if (World* w = AsWorld(world)) GuardVoid([&] { w->DestroyComponent(ToHandle(component)); });
}

PHYSIK_B200_API int PHYSIK_IsComponentHandleValid(PhysikWorldHandle world, PhysikComponentHandle component)
{
    World* w = AsWorld(world);
    return (w && w->IsComponentHandleValid(ToHandle(component))) ? 1 : 0;
}

PHYSIK_B200_API int PHYSIK_GetTetMeshTetCount(PhysikWorldHandle world, PhysikComponentHandle component)
{
    const TetMeshComponent* c = AsTetMesh(AsWorld(world), component);
    return c ? c->GetTetCount() : 0;
}

PHYSIK_B200_API int PHYSIK_GetTetMeshNodeCount(PhysikWorldHandle world, PhysikComponentHandle component)
{
    const TetMeshComponent* c = AsTetMesh(AsWorld(world), component);
    return c ? c->GetNodeCount() : 0;
}

PHYSIK_B200_API int PHYSIK_IsTetActive(PhysikWorldHandle world, PhysikComponentHandle component, int tetIndex)
{
    const TetMeshComponent* c = AsTetMesh(AsWorld(world), component);
    return (c && c->IsTetActive(tetIndex)) ? 1 : 0;
}

PHYSIK_B200_API void PHYSIK_SetTetActive(PhysikWorldHandle world, PhysikComponentHandle component, int tetIndex,
                                         int active)
{
    World* w = AsWorld(world);
    TetMeshComponent* c = AsTetMesh(w, component);
    if (!c) return;
    GuardVoid([&] {
        if (c->SetTetActive(tetIndex, active != 0)) ReconcileNodes(*w, *c, tetIndex);
    });
}

PHYSIK_B200_API void PHYSIK_DeactivateTet(PhysikWorldHandle world, PhysikComponentHandle component, int tetIndex)
{
    PHYSIK_SetTetActive(world, component, tetIndex, 0);
}

PHYSIK_B200_API int PHYSIK_GetActiveTetCount(PhysikWorldHandle world, PhysikComponentHandle component)
{
    const TetMeshComponent* c = AsTetMesh(AsWorld(world), component);
    return c ? c->GetActiveTetCount() : 0;
}

PHYSIK_B200_API void PHYSIK_GetNodePosition(PhysikWorldHandle world, int nodeIndex, float* outX, float* outY,
                                            float* outZ)
{
    World* w = AsWorld(world);
    if (!w || !ValidNode(*w, nodeIndex)) return;
    GuardVoid([&] {
        const Vec3& p = w->GetNodePosition(nodeIndex);
        if (outX) *outX = p.x;
        if (outY) *outY = p.y;
        if (outZ) *outZ = p.z;
    });
}

PHYSIK_B200_API void PHYSIK_GetNodeVelocity(PhysikWorldHandle world, int nodeIndex, float* outX, float* outY,
                                            float* outZ)
{
    World* w = AsWorld(world);
    if (!w || !ValidNode(*w, nodeIndex)) return;
    GuardVoid([&] {
        const Vec3& v = w->GetNodeVelocity(nodeIndex);
        if (outX) *outX = v.x;
        if (outY) *outY = v.y;
        if (outZ) *outZ = v.z;
    });
}

PHYSIK_B200_API void PHYSIK_SetNodePosition(PhysikWorldHandle world, int nodeIndex, float x, float y, float z)
{
    World* w = AsWorld(world);
    if (w && ValidNode(*w, nodeIndex)) GuardVoid([&] { w->SetNodePosition(nodeIndex, Vec3{x, y, z}); });
}

PHYSIK_B200_API void PHYSIK_SetNodeVelocity(PhysikWorldHandle world, int nodeIndex, float x, float y, float z)
{
    World* w = AsWorld(world);
    if (w && ValidNode(*w, nodeIndex)) GuardVoid([&] { w->SetNodeVelocity(nodeIndex, Vec3{x, y, z}); });
}

// ---------------------------------------------------------------- point connections
PHYSIK_B200_API int PHYSIK_GetPointConnectionCount(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    return w ? w->GetTransientConnectionCount() : 0;
}

PHYSIK_B200_API void PHYSIK_AddPointConnection(PhysikWorldHandle world, int node0, int node1, int node2, int node3,
                                               float barycentricX, float barycentricY, float barycentricZ,
                                               float barycentricW, float targetX, float targetY, float targetZ,
                                               float stiffness, float damping)
{
    World* w = AsWorld(world);
    if (!w) return;
    PointConnection c;
    c.node0 = node0;
    c.node1 = node1;
    c.node2 = node2;
    c.node3 = node3;
    c.barycentric = Vec4{barycentricX, barycentricY, barycentricZ, barycentricW};
    c.targetPosition = Vec3{targetX, targetY, targetZ};
    c.stiffness = stiffness;
    c.damping = damping;
    GuardVoid([&] { w->AddPointConnection(c); });
}

// ---------------------------------------------------------------- extensions
PHYSIK_B200_API void PHYSIK_B200_SetPrecision(PhysikWorldHandle world, int precision)
{
    World* w = AsWorld(world);
    if (!w || precision < 0 || precision > 2) return;
    GuardVoid([&] { w->SetPrecision(static_cast<Precision>(precision)); });
}

PHYSIK_B200_API int PHYSIK_B200_GetPrecision(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    return w ? static_cast<int>(w->GetPrecision()) : -1;
}

PHYSIK_B200_API void PHYSIK_B200_SetDevice(PhysikWorldHandle world, int device)
{
    if (World* w = AsWorld(world)) GuardVoid([&] { w->SetDevice(device); });
}

PHYSIK_B200_API int PHYSIK_B200_GetNodeCount(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    return w ? static_cast<int>(w->GetNodes().size()) : 0;
}

PHYSIK_B200_API int PHYSIK_B200_GetNodeStates(PhysikWorldHandle world, float* positions, float* velocities, int count)
{
    World* w = AsWorld(world);
    if (!w || count != static_cast<int>(w->GetNodes().size())) return -1;
    return Guard([&] { w->GetNodeStates(positions, velocities); return count; }, -1);
}

PHYSIK_B200_API int PHYSIK_B200_SetNodeStates(PhysikWorldHandle world, const float* positions, const float* velocities,
                                              int count)
{
    World* w = AsWorld(world);
    if (!w || count != static_cast<int>(w->GetNodes().size())) return -1;
    return Guard([&] { w->SetNodeStates(positions, velocities); return count; }, -1);
}

PHYSIK_B200_API int PHYSIK_B200_GetNodeStatesF64(PhysikWorldHandle world, double* positions, double* velocities,
                                                 int count)
{
    World* w = AsWorld(world);
    if (!w || count != static_cast<int>(w->GetNodes().size())) return -1;
    return Guard([&] { w->GetNodeStatesF64(positions, velocities); return count; }, -1);
}

PHYSIK_B200_API int PHYSIK_B200_SetNodeStatesF64(PhysikWorldHandle world, const double* positions,
                                                 const double* velocities, int count)
{
    World* w = AsWorld(world);
    if (!w || count != static_cast<int>(w->GetNodes().size())) return -1;
    return Guard([&] { w->SetNodeStatesF64(positions, velocities); return count; }, -1);
}

PHYSIK_B200_API int PHYSIK_B200_SetTetMeshYoungModulus(PhysikWorldHandle world, PhysikComponentHandle component,
                                                       const float* youngModulus, int tetCount)
{
    TetMeshPhysicsComponent* c = AsTetMeshPhysics(AsWorld(world), component);
    if (!c || !youngModulus || tetCount != c->GetTetCount()) return 0;
    for (int t = 0; t < tetCount; ++t) c->tets[static_cast<std::size_t>(t)].youngModulus = youngModulus[t];
    c->RebuildTetFemCache();
    return 1;
}

PHYSIK_B200_API int PHYSIK_B200_SetTetMeshFemModel(PhysikWorldHandle world, PhysikComponentHandle component, int model)
{
    TetMeshPhysicsComponent* c = AsTetMeshPhysics(AsWorld(world), component);
    if (!c || model < 0 || model > 2) return 0;
    c->SetFemModel(static_cast<FemModel>(model));
    return 1;
}

PHYSIK_B200_API unsigned PHYSIK_B200_GetLastStepFlags(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    return w ? Guard([&] { return w->GetLastStepFlags(); }, 0u) : 0u;
}

PHYSIK_B200_API const char* PHYSIK_B200_GetLastError(void) { return g_error.c_str(); }

PHYSIK_B200_API int PHYSIK_B200_PrepareScene(PhysikWorldHandle world, int upload)
{
    World* w = AsWorld(world);
    if (!w) return -1;
    return Guard([&] { return w->PrepareScene(upload != 0); }, -1);
}

PHYSIK_B200_API int PHYSIK_B200_GetSolverSizes(PhysikWorldHandle world, int* dynamicRows, int* blocks)
{
    World* w = AsWorld(world);
    if (!w || w->GetSceneDynamicCount() < 0) return -1;
    if (dynamicRows) *dynamicRows = w->GetSceneDynamicCount();
    if (blocks) *blocks = w->GetSceneBlockCount();
    return 0;
}

PHYSIK_B200_API int PHYSIK_B200_GetSolverPattern(PhysikWorldHandle world, int* rowStart, int* colIndex,
                                                 int* nodeToDynamic)
{
    World* w = AsWorld(world);
    if (!w || w->GetSceneDynamicCount() < 0) return -1;
    if (rowStart) std::copy(w->GetSceneRowStart()->begin(), w->GetSceneRowStart()->end(), rowStart);
    if (colIndex) std::copy(w->GetSceneColIndex()->begin(), w->GetSceneColIndex()->end(), colIndex);
    if (nodeToDynamic) std::copy(w->GetSceneNodeToDyn()->begin(), w->GetSceneNodeToDyn()->end(), nodeToDynamic);
    return 0;
}

PHYSIK_B200_API int PHYSIK_B200_GetSolverMasses(PhysikWorldHandle world, double* masses)
{
    World* w = AsWorld(world);
    if (!w || !w->GetSceneMass()) return -1;
    if (masses) std::copy(w->GetSceneMass()->begin(), w->GetSceneMass()->end(), masses);
    return 0;
}

PHYSIK_B200_API int PHYSIK_B200_GetSolverSystem(PhysikWorldHandle world, double* values, double* rhs, double* minv,
                                                double* deltaVelocity)
{
    World* w = AsWorld(world);
    if (!w || !w->GetDeviceSystem()) return -1;
    if (!w->SceneMatchesDevice()) return -1;  // the caller's arrays are sized by the host scene
    return Guard([&] { return pk_system_get_system_f64(w->GetDeviceSystem(), values, rhs, minv, deltaVelocity); }, -1);
}

PHYSIK_B200_API int PHYSIK_B200_EnableTiming(PhysikWorldHandle world, int on)
{
    World* w = AsWorld(world);
    if (!w || !w->GetDeviceSystem()) return -1;
    return pk_system_enable_timing(w->GetDeviceSystem(), on);
}

PHYSIK_B200_API int PHYSIK_B200_GetTimings(PhysikWorldHandle world, double* assembleMs, double* solveMs, int* steps,
                                           long long* kernelLaunches)
{
    World* w = AsWorld(world);
    if (!w || !w->GetDeviceSystem()) return -1;
    return pk_system_timings(w->GetDeviceSystem(), assembleMs, solveMs, steps, kernelLaunches);
}

PHYSIK_B200_API void PHYSIK_B200_SetBatchedSolve(PhysikWorldHandle world, int on)
{
    World* w = AsWorld(world);
    if (w) w->SetBatchedSolve(on != 0);
}

PHYSIK_B200_API int PHYSIK_B200_GetBodyConjugateGradientStats(PhysikWorldHandle world, PhysikComponentHandle body,
                                                              int* iterations, int* converged, float* residualNorm,
                                                              unsigned* flags)
{
    World* w = AsWorld(world);
    if (!w) return -1;
    return Guard(
        [&] {
            Component* c = w->GetComponent(ToHandle(body));
            int it = 0;
            bool conv = false;
            float res = 0.0f;
            unsigned fl = 0;
            if (!c || !w->GetBodyConjugateGradientStats(c, it, conv, res, fl)) return -1;
            if (iterations) *iterations = it;
            if (converged) *converged = conv ? 1 : 0;
            if (residualNorm) *residualNorm = res;
            if (flags) *flags = fl;
            return 0;
        },
        -1);
}

PHYSIK_B200_API int PHYSIK_B200_AdjointStep(PhysikWorldHandle world, float dt, const double* positionsBarNext,
                                            const double* velocitiesBarNext, double* positionsBar,
                                            double* velocitiesBar, double* youngLogBar)
{
    World* w = AsWorld(world);
    if (!w || !positionsBarNext || !velocitiesBarNext || !positionsBar || !velocitiesBar) return -1;
    return Guard(
        [&] {
            w->AdjointStep(dt, positionsBarNext, velocitiesBarNext, positionsBar, velocitiesBar, youngLogBar);
            return 0;
        },
        -1);
}

PHYSIK_B200_API int PHYSIK_B200_GetTetCount(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    if (!w) return -1;
    return Guard([&] { return w->PrepareScene(false) >= 0 ? w->GetSceneTetCount() : -1; }, -1);
}

PHYSIK_B200_API void PHYSIK_B200_SetGraphCapture(PhysikWorldHandle world, int on)
{
    World* w = AsWorld(world);
    if (w) w->SetGraphCapture(on != 0);
}

PHYSIK_B200_API int PHYSIK_B200_Autotune(PhysikWorldHandle world, int repeats, double* bestSolveMs)
{
    World* w = AsWorld(world);
    if (!w) return -1;
    return Guard([&] { return w->Autotune(repeats, bestSolveMs); }, -1);
}

PHYSIK_B200_API int PHYSIK_B200_GetPcgKernel(PhysikWorldHandle world, int* blocks)
{
    World* w = AsWorld(world);
    if (!w) return -1;
    return Guard([&] { return w->GetPcgKernel(blocks); }, -1);
}

PHYSIK_B200_API int PHYSIK_B200_GetPcgStreamForm(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    if (!w) return -1;
    return Guard([&] { return w->GetPcgStreamForm(); }, -1);
}

PHYSIK_B200_API void* PHYSIK_B200_GetDeviceSystem(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    return w ? static_cast<void*>(w->GetDeviceSystem()) : nullptr;
}

PHYSIK_B200_API int PHYSIK_B200_SetRefinement(PhysikWorldHandle world, int passes)
{
    World* w = AsWorld(world);
    if (!w || passes < 0 || passes > 16) return -1;
    w->SetRefinement(passes);
    return 0;
}

PHYSIK_B200_API int PHYSIK_B200_SetPcgGrid(PhysikWorldHandle world, int grid)
{
    World* w = AsWorld(world);
    if (!w || !w->GetDeviceSystem()) return -1;
    return pk_system_set_pcg_grid(w->GetDeviceSystem(), grid);
}

PHYSIK_B200_API void* PHYSIK_B200_GetStream(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    return (w && w->GetDeviceSystem()) ? pk_system_stream(w->GetDeviceSystem()) : nullptr;
}

PHYSIK_B200_API int PHYSIK_B200_Synchronize(PhysikWorldHandle world)
{
    World* w = AsWorld(world);
    if (!w) return -1;
    return Guard([&] { (void)w->GetLastStepFlags(); return 0; }, -1);
}

}  // extern "C"
