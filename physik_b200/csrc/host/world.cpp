// World, the tet-mesh components and SolverData, with the device scene behind them.
//
// Stepping follows World::Step (src/Core/World/World.cpp:32-73): pre-update, then per
// substep the components' UpdateSystem in execution-priority order, then the solve and
// integration, then post-update.  TetMeshPhysicsComponent::UpdateSystem registers its
// body with SolverData; the World then runs the whole substep on the GPU through one
// pk_system (tet kernel, row kernel, cooperative PCG with fused integration).
//
// The device scene (rest data, lumped masses, dynamic-node mapping, canonical upper
// BSR pattern, per-row tet incidence lists) is built on the host when the topology
// changes, with the reference's rules:
//   rest data       FEMModel::InitializeTetRestData (FEMModel.cpp:504-548)
//   lambda, mu      FEMModel BuildElasticityMatrix (FEMModel.cpp:174-200)
//   lumped mass     FEMModel::ComputeLumpedMass + ApplyMassContribution
//                   (FEMModel.cpp:681-713, TetMeshPhysicsComponent.cpp:127-152)
//   mass check      World::ValidateNodeMasses (World.cpp:560-580) -- throws
//   dynamic rows    SolverData::BuildDynamicNodeMapping (SolverData.cpp:239-258)
//   pattern         diagonal of every dynamic row plus every tet-edge block between two
//                   dynamic nodes, from all tets of each simulated body, active or not
//                   (TetMeshPhysicsComponent.cpp:36-60, 221-232, 341-353;
//                    SolverData.cpp:321-405; SparseBlockMatrix.cpp:83-129)
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../../include/pkcuda.h"
#include "physik_core.h"

namespace PhysiK {

namespace {

constexpr float kMinConjugateGradientTolerance = 1.0e-8f;
constexpr float kMaxConjugateGradientTolerance = 1.0e-1f;
constexpr int kMinConjugateGradientMaxIterations = 1;
constexpr int kMaxConjugateGradientMaxIterations = 1024;

const Vec3 kZero{};

// f(lo, hi) over [0, count) in contiguous chunks on up to 16 host threads (one thread
// for small counts or when no thread can be started); chunks write disjoint outputs.
template <class F>
void ParallelRanges(std::size_t count, F&& f)
{
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const std::size_t nt = count < 65536 ? 1 : std::min<std::size_t>(hw, count / 16384);
    if (nt <= 1) {
        f(std::size_t(0), count);
        return;
    }
    const std::size_t chunk = (count + nt - 1) / nt;
    std::vector<std::thread> pool;
    std::size_t started = 0;
    try {
        for (std::size_t t = 1; t < nt; ++t) {
            const std::size_t lo = t * chunk, hi = std::min(count, lo + chunk);
            if (lo >= hi) break;
            pool.emplace_back([&f, lo, hi] { f(lo, hi); });
            started = t;
        }
    } catch (...) {
    }
    f(std::size_t(0), std::min(count, chunk));
    for (std::size_t t = started + 1; t < nt; ++t) {  // chunks whose thread could not start
        const std::size_t lo = t * chunk, hi = std::min(count, lo + chunk);
        if (lo < hi) f(lo, hi);
    }
    for (std::thread& th : pool) th.join();
}

void Check(int rc, const char* what)
{
    if (rc != PK_OK) throw std::runtime_error(std::string(what) + ": " + pk_last_error());
}

// Rest data of one tet in precision T (FEMModel.cpp:504-548).
template <class T>
struct RestData {
    T volume = T(0);
    detail::M<T> dm_inv{};
};

template <class T>
RestData<T> ComputeRest(const Vec3& p0, const Vec3& p1, const Vec3& p2, const Vec3& p3)
{
    using V = detail::V<T>;
    auto cv = [](const Vec3& p) { return V{T(p.x), T(p.y), T(p.z)}; };
    const V r0 = cv(p0), r1 = cv(p1), r2 = cv(p2), r3 = cv(p3);
    const detail::M<T> dm{{detail::sub(r1, r0), detail::sub(r2, r0), detail::sub(r3, r0)}};
    const T det = detail::det(dm);
    RestData<T> out;
    const T vol = std::abs(det) / T(6);
    if (vol <= T(1.0e-8)) {
        out.volume = T(0);
        out.dm_inv = detail::M<T>{{V{0, 0, 0}, V{0, 0, 0}, V{0, 0, 0}}};
        return out;
    }
    out.volume = vol;
    out.dm_inv = detail::inverse(dm);
    return out;
}

// lambda and mu of BuildElasticityMatrix in precision T (zero when E <= 0).
template <class T>
void LameParameters(float young, float poisson, T& lambda, T& mu)
{
    const T e = std::max(T(0), T(young));
    lambda = T(0);
    mu = T(0);
    if (e <= T(0)) return;
    const T nu = std::max(T(-0.99), std::min(T(0.49), T(poisson)));
    lambda = e * nu / ((T(1) + nu) * (T(1) - T(2) * nu));
    mu = e / (T(2) * (T(1) + nu));
}

}  // namespace

// ------------------------------------------------------------------ TetMeshComponent
void TetMeshComponent::SetGeometry(const GeneratedTetMesh& mesh)
{
    nodeTetStart.clear();
    nodeTetList.clear();
    nodeTetData = nullptr;
    restNodePositions = mesh.positions;
    nodePositions = restNodePositions;
    tets.clear();
    const int count = static_cast<int>(mesh.tetLocalNodeIndices.size() / 4u);
    const int nodeCount = static_cast<int>(restNodePositions.size());
    tets.reserve(static_cast<std::size_t>(std::max(0, count)));
    for (int t = 0; t < count; ++t) {
        const int* n = &mesh.tetLocalNodeIndices[static_cast<std::size_t>(4 * t)];
        bool ok = true;
        for (int k = 0; k < 4; ++k) ok = ok && n[k] >= 0 && n[k] < nodeCount;
        if (!ok) continue;
        Tet tet;
        tet.node0 = n[0];
        tet.node1 = n[1];
        tet.node2 = n[2];
        tet.node3 = n[3];
        tets.push_back(tet);
    }
}

int TetMeshComponent::GetTetNodeIndex(int tetIndex, int corner) const
{
    if (tetIndex < 0 || tetIndex >= static_cast<int>(tets.size())) return -1;
    const Tet& t = tets[static_cast<std::size_t>(tetIndex)];
    switch (corner) {
    case 0: return t.node0;
    case 1: return t.node1;
    case 2: return t.node2;
    case 3: return t.node3;
    default: return -1;
    }
}

const Vec3& TetMeshComponent::GetLocalRestPosition(int i) const
{
    if (i < 0 || i >= static_cast<int>(restNodePositions.size())) return kZero;
    return restNodePositions[static_cast<std::size_t>(i)];
}

const Vec3& TetMeshComponent::GetLocalCurrentPosition(int i) const
{
    if (i < 0 || i >= static_cast<int>(nodePositions.size())) return kZero;
    return nodePositions[static_cast<std::size_t>(i)];
}

int TetMeshComponent::GetGlobalNodeIndex(int) const { return -1; }

void TetMeshComponent::SetLocalCurrentPosition(int i, const Vec3& p)
{
    if (i < 0 || i >= static_cast<int>(nodePositions.size())) return;
    nodePositions[static_cast<std::size_t>(i)] = p;
    ++localEdits;
}

int TetMeshComponent::GetLocalNodeIndexOf(int globalNodeIndex) const
{
    // GetGlobalNodeIndex is begin + local for the meshes that own world nodes, -1 otherwise.
    const int n = GetNodeCount();
    if (n <= 0) return -1;
    const int begin = GetGlobalNodeIndex(0);
    if (begin < 0) return -1;
    const int local = globalNodeIndex - begin;
    return (local >= 0 && local < n && GetGlobalNodeIndex(local) == globalNodeIndex) ? local : -1;
}

bool TetMeshComponent::HasActiveTetAtLocalNode(int localNodeIndex) const
{
    const int n = GetNodeCount();
    if (localNodeIndex < 0 || localNodeIndex >= n) return false;
    if (nodeTetData != tets.data() || nodeTetCount != tets.size() || nodeTetStart.size() != static_cast<std::size_t>(n) + 1) {
        nodeTetStart.assign(static_cast<std::size_t>(n) + 1, 0);
        for (const Tet& t : tets)
            for (int k : {t.node0, t.node1, t.node2, t.node3})
                if (k >= 0 && k < n) ++nodeTetStart[static_cast<std::size_t>(k) + 1];
        for (int i = 0; i < n; ++i) nodeTetStart[i + 1] += nodeTetStart[i];
        nodeTetList.assign(static_cast<std::size_t>(nodeTetStart[n]), 0);
        std::vector<int> fill(nodeTetStart.begin(), nodeTetStart.end() - 1);
        for (int ti = 0; ti < static_cast<int>(tets.size()); ++ti) {
            const Tet& t = tets[static_cast<std::size_t>(ti)];
            for (int k : {t.node0, t.node1, t.node2, t.node3})
                if (k >= 0 && k < n) nodeTetList[static_cast<std::size_t>(fill[k]++)] = ti;
        }
        nodeTetData = tets.data();
        nodeTetCount = tets.size();
    }
    for (int i = nodeTetStart[localNodeIndex]; i < nodeTetStart[localNodeIndex + 1]; ++i)
        if (tets[static_cast<std::size_t>(nodeTetList[static_cast<std::size_t>(i)])].active) return true;
    return false;
}

bool TetMeshComponent::IsTetActive(int tetIndex) const
{
    if (tetIndex < 0 || tetIndex >= static_cast<int>(tets.size())) return false;
    return tets[static_cast<std::size_t>(tetIndex)].active;
}

bool TetMeshComponent::SetTetActive(int tetIndex, bool activeValue)
{
    if (tetIndex < 0 || tetIndex >= static_cast<int>(tets.size())) return false;
    Tet& t = tets[static_cast<std::size_t>(tetIndex)];
    if (t.active == activeValue) return false;
    t.active = activeValue;
    topologyDirty = true;
    return true;
}

int TetMeshComponent::GetActiveTetCount() const
{
    int c = 0;
    for (const Tet& t : tets) c += t.active ? 1 : 0;
    return c;
}

void TetMeshComponent::PostUpdate(World&, float)
{
    if (topologyDirty) ++topologyEvents;  // TetMeshTopologyChanged (TetMeshComponent.cpp:190-206)
    topologyDirty = false;
}

// ------------------------------------------------------------------ TetMeshPhysicsComponent
std::unique_ptr<TetMeshPhysicsComponent> TetMeshPhysicsComponent::CreateFromGeneratedTetMesh(
    World& world, const GeneratedTetMesh& mesh, const Material& material)
{
    TetMeshPhysicsComponentDesc desc;
    desc.material = material;
    return CreateFromGeneratedTetMesh(world, mesh, desc);
}

std::unique_ptr<TetMeshPhysicsComponent> TetMeshPhysicsComponent::CreateFromGeneratedTetMesh(
    World& world, const GeneratedTetMesh& mesh, const TetMeshPhysicsComponentDesc& desc)
{
    auto c = std::make_unique<TetMeshPhysicsComponent>();
    c->material = desc.material;
    c->selectedFemModel = desc.femModel;
    c->SetGeometry(mesh);
    c->globalNodeBeginIndex = static_cast<int>(world.GetNodes().size());
    c->globalNodeCount = static_cast<int>(c->restNodePositions.size());
    for (const Vec3& p : c->restNodePositions) world.AddNode(p);
    c->RebuildFemRestData();
    return c;
}

void TetMeshPhysicsComponent::SetMaterial(const Material& value)
{
    material = value;
    for (Tet& t : tets) {
        t.youngModulus = value.youngModulus;
        t.poissonRatio = value.poissonRatio;
        t.damping = value.damping;
    }
    ++version;
}

void TetMeshPhysicsComponent::RebuildFemRestData()
{
    for (Tet& t : tets) {
        t.youngModulus = material.youngModulus;
        t.poissonRatio = material.poissonRatio;
        t.damping = material.damping;
        const int n[4] = {t.node0, t.node1, t.node2, t.node3};
        for (int k = 0; k < 4; ++k) t.restPositions[k] = restNodePositions[static_cast<std::size_t>(n[k])];
        const RestData<float> rd = ComputeRest<float>(t.restPositions[0], t.restPositions[1], t.restPositions[2],
                                                      t.restPositions[3]);
        t.restVolume = rd.volume;
        if (rd.volume <= 0.0f) {
            t.restDmInverse = Mat3::Zero();
            for (Vec3& g : t.shapeFunctionGradients) g = Vec3{};
            continue;
        }
        const auto& m = rd.dm_inv;
        t.restDmInverse = Mat3::FromColumns(Vec3{m.c[0].x, m.c[0].y, m.c[0].z}, Vec3{m.c[1].x, m.c[1].y, m.c[1].z},
                                            Vec3{m.c[2].x, m.c[2].y, m.c[2].z});
        t.shapeFunctionGradients[1] = Vec3{m.c[0].x, m.c[1].x, m.c[2].x};
        t.shapeFunctionGradients[2] = Vec3{m.c[0].y, m.c[1].y, m.c[2].y};
        t.shapeFunctionGradients[3] = Vec3{m.c[0].z, m.c[1].z, m.c[2].z};
        t.shapeFunctionGradients[0] =
            -(t.shapeFunctionGradients[1] + t.shapeFunctionGradients[2] + t.shapeFunctionGradients[3]);
    }
    ++version;
}

void TetMeshPhysicsComponent::SyncCurrentPositionsFromWorld(const World& world)
{
    nodePositions.resize(static_cast<std::size_t>(globalNodeCount));
    nodeVelocities.resize(static_cast<std::size_t>(globalNodeCount));
    for (int i = 0; i < globalNodeCount; ++i) {
        const int g = GetGlobalNodeIndex(i);
        if (g < 0 || g >= static_cast<int>(world.GetNodes().size())) continue;
        nodePositions[static_cast<std::size_t>(i)] = world.GetNodePosition(g);
        nodeVelocities[static_cast<std::size_t>(i)] = world.GetNodeVelocity(g);
    }
}

int TetMeshPhysicsComponent::GetGlobalNodeIndex(int local) const
{
    if (globalNodeBeginIndex < 0 || local < 0 || local >= globalNodeCount) return -1;
    return globalNodeBeginIndex + local;
}

bool TetMeshPhysicsComponent::SetTetActive(int tetIndex, bool activeValue)
{
    const bool changed = TetMeshComponent::SetTetActive(tetIndex, activeValue);
    if (changed) ++version;
    return changed;
}

// The device computes this body's forces and stiffness; the host only registers it.
// The component-local position copies are refreshed on demand (SyncCurrentPositionsFromWorld)
// rather than every substep, so a step never waits for a device-to-host copy.
void TetMeshPhysicsComponent::UpdateSystem(World&, SolverData& solverData, float)
{
    if (!physicsEnabled) return;
    solverData.AddFemBody(this);
}

void TetMeshPhysicsComponent::PostUpdate(World& world, float dt)
{
    if (dt > 0.0f) {  // SyncCurrentPositionsFromWorld, lazily
        snapshotWanted = world.GetSnapshotGeneration();
        snapshotEdits = localEdits;
    }
    TetMeshComponent::PostUpdate(world, dt);
}

// ------------------------------------------------------------------ SolverData
void SolverData::Clear()
{
    ClearTransientState();
    matrix.Clear();
    implicitPatternDirty = true;
}

void SolverData::ClearTransientState()
{
    nodeForces.clear();
    nodeMasses.clear();
    stiffnessBlocks.clear();
    femBodies.clear();
    femMassMark.clear();
    assembledMasses.clear();
    assembledForces.clear();
    nodeToDynamicBlock.clear();
    dynamicBlockCount = 0;
    rhs.clear();
    deltaVelocity.clear();
    lastLinearSolveResult = LinearSolveResult{};
    precomputeOk = false;
}

void SolverData::AssembleMasses(int nodeCount)
{
    assembledMasses.assign(static_cast<std::size_t>(std::max(0, nodeCount)), 0.0f);
    for (const NodeMass& m : nodeMasses) {
        if (m.node < 0 || m.node >= nodeCount || !std::isfinite(m.mass) || m.mass <= 0.0f) continue;
        assembledMasses[static_cast<std::size_t>(m.node)] += m.mass;
    }
}

bool SolverData::HasNodeMassContribution(int nodeIndex) const
{
    for (const NodeMass& m : nodeMasses)
        if (m.node == nodeIndex) return true;
    return false;
}

float SolverData::GetAssembledMassForNode(int nodeIndex) const
{
    if (nodeIndex < 0 || nodeIndex >= static_cast<int>(assembledMasses.size())) return 0.0f;
    return assembledMasses[static_cast<std::size_t>(nodeIndex)];
}

int SolverData::GetDynamicBlockForNode(int nodeIndex) const
{
    if (nodeIndex < 0 || nodeIndex >= static_cast<int>(nodeToDynamicBlock.size())) return -1;
    return nodeToDynamicBlock[static_cast<std::size_t>(nodeIndex)];
}

bool SolverData::BuildDynamicNodeMapping(const std::vector<Node>& nodes)
{
    nodeToDynamicBlock.assign(nodes.size(), -1);
    dynamicBlockCount = 0;
    for (std::size_t i = 0; i < nodes.size(); ++i) {
        const float m = assembledMasses[i];
        if (nodes[i].active && !nodes[i].fixed && std::isfinite(m) && m > 0.0f)
            nodeToDynamicBlock[i] = dynamicBlockCount++;
    }
    return dynamicBlockCount > 0;
}

// ------------------------------------------------------------------ device scene
// Host-built topology of the simulated bodies plus the device system it is uploaded to.
struct DeviceScene {
    pk_system* sys = nullptr;
    Precision precision = Precision::FP32;
    int device = 0;
    std::uint64_t worldVersion = 0;
    std::vector<std::pair<const TetMeshPhysicsComponent*, std::uint64_t>> bodies;
    bool built = false;
    bool uploaded = false;
    int nodeCount = 0;
    int dynCount = 0;
    int tetCount = 0;
    std::vector<int> nodeToDyn, dynToNode, rowStart, colIndex, tetNodes, incStart, incList;
    // Batched solve: the bodies' dynamic row ranges in row order (segStart), each body's
    // segment, and whether every dynamic row belongs to one body (else no batching).
    std::vector<int> segStart;
    std::vector<std::pair<const Component*, int>> bodySegment;
    bool segmentsCover = false;
    bool batchedOnDevice = false;
    bool graphOnDevice = false;
    int refineOnDevice = 0;
    std::vector<unsigned char> enabled;
    std::vector<double> mass, dmInv, volume, lam, mu, damp;
    // FP32 storage with refinement on: the same rest data and masses in FP64
    // (pk_system_set_rest64).
    bool rest64 = false;
    std::vector<double> mass64, dmInv64, volume64, lam64, mu64;
    // The FEM bodies' pattern; rowStart / colIndex above are it joined with the blocks of
    // the current point connections (connPairs, canonical row <= column).
    std::vector<int> femRowStart, femColIndex;
    std::vector<std::pair<int, int>> connPairs;
    std::uint64_t connVersion = 0;  // World::connectionVersion the connection arrays are for
    std::vector<std::pair<int, int>> connOnlyPairs;  // the connections' own pairs (sorted)
    std::vector<std::tuple<int, float, bool>> extraMasses;  // host-emitted masses this scene holds
    // host-emitted blocks and forces (World::SyncExtras)
    bool extOnDevice = false;       // the device holds host-emitted blocks / forces
    int extCount = 0;
    std::vector<double> extBlocks, extForce;
    std::vector<int> extNodes, extRhsStart, extRhsList, extMatStart, extMatList;
    int connCount = 0;
    std::vector<int> connNodes, connIncStart, connIncList;
    std::vector<double> connParams;
    bool connOnDevice = false;
    int devDyn = -1, devNnz = -1;  // the pattern the device holds

    ~DeviceScene()
    {
        if (sys) pk_system_destroy(sys);
    }
    bool Matches(const World& w, const std::vector<const TetMeshPhysicsComponent*>& fem) const
    {
        if (!built || worldVersion != w.GetTopologyVersion() || precision != w.GetPrecision()) return false;
        if (fem.size() != bodies.size()) return false;
        if (extraMasses != w.GetExtraMasses()) return false;
        for (std::size_t i = 0; i < fem.size(); ++i)
            if (fem[i] != bodies[i].first || fem[i]->version != bodies[i].second) return false;
        return true;
    }
};

namespace {

template <class T>
void BuildHostScene(DeviceScene& sc, const World& w, const std::vector<const TetMeshPhysicsComponent*>& fem)
{
    const std::vector<Node>& nodes = w.GetNodes();
    const int nn = static_cast<int>(nodes.size());
    std::size_t total = 0;
    for (const TetMeshPhysicsComponent* body : fem) total += body->tets.size();
    sc.tetNodes.assign(4 * total, 0);
    sc.enabled.assign(total, 0);
    sc.dmInv.assign(9 * total, 0.0);
    sc.volume.assign(total, 0.0);
    sc.lam.assign(total, 0.0);
    sc.mu.assign(total, 0.0);
    sc.damp.assign(total, 0.0);
    std::vector<T> nodal(total, T(0));  // each tet's lumped mass share (0: none)
    std::vector<T> massT(static_cast<std::size_t>(nn), T(0));
    // FP32 storage with refinement: the rest data and masses once more in FP64.
    sc.rest64 = !std::is_same<T, double>::value && w.GetRefinement() > 0;
    std::vector<double> nodal64;
    if (sc.rest64) {
        sc.dmInv64.assign(9 * total, 0.0);
        sc.volume64.assign(total, 0.0);
        sc.lam64.assign(total, 0.0);
        sc.mu64.assign(total, 0.0);
        nodal64.assign(total, 0.0);
    } else {
        sc.dmInv64.clear();
        sc.volume64.clear();
        sc.lam64.clear();
        sc.mu64.clear();
        sc.mass64.clear();
    }
    std::size_t first = 0;
    for (const TetMeshPhysicsComponent* body : fem) {
        const int base = body->GetGlobalNodeBeginIndex();
        const T density = std::max(T(0), T(body->material.density));
        const bool femImplemented = body->GetFemModel() != FemModel::NeoHookean;
        const unsigned char linearBit = body->GetFemModel() == FemModel::Linear ? 2 : 0;
        const std::vector<Tet>& tets = body->tets;
        // Per tet, independent of the others (on host threads for large bodies).
        ParallelRanges(tets.size(), [&](std::size_t lo, std::size_t hi) {
            for (std::size_t i = lo; i < hi; ++i) {
                const Tet& t = tets[i];
                const std::size_t g = first + i;
                const RestData<T> rd = ComputeRest<T>(body->restNodePositions[t.node0], body->restNodePositions[t.node1],
                                                      body->restNodePositions[t.node2], body->restNodePositions[t.node3]);
                sc.tetNodes[4 * g + 0] = t.node0 + base;
                sc.tetNodes[4 * g + 1] = t.node1 + base;
                sc.tetNodes[4 * g + 2] = t.node2 + base;
                sc.tetNodes[4 * g + 3] = t.node3 + base;
                sc.enabled[g] = static_cast<unsigned char>((t.active && rd.volume > T(0) && femImplemented ? 1 : 0) |
                                                           linearBit | (t.active ? 4 : 0));
                for (int c = 0; c < 3; ++c) {
                    sc.dmInv[9 * g + 3 * c + 0] = static_cast<double>(rd.dm_inv.c[c].x);
                    sc.dmInv[9 * g + 3 * c + 1] = static_cast<double>(rd.dm_inv.c[c].y);
                    sc.dmInv[9 * g + 3 * c + 2] = static_cast<double>(rd.dm_inv.c[c].z);
                }
                sc.volume[g] = static_cast<double>(rd.volume);
                T l, m;
                LameParameters<T>(t.youngModulus, t.poissonRatio, l, m);
                sc.lam[g] = static_cast<double>(l);
                sc.mu[g] = static_cast<double>(m);
                sc.damp[g] = static_cast<double>(T(t.damping));
                if (std::isfinite(static_cast<double>(density)) && t.active &&
                    std::isfinite(static_cast<double>(rd.volume)) && rd.volume > T(0)) {
                    const T share = density * rd.volume * T(0.25);
                    if (std::isfinite(static_cast<double>(share)) && share > T(0)) nodal[g] = share;
                }
                if (sc.rest64) {
                    const RestData<double> r64 =
                        ComputeRest<double>(body->restNodePositions[t.node0], body->restNodePositions[t.node1],
                                            body->restNodePositions[t.node2], body->restNodePositions[t.node3]);
                    for (int c = 0; c < 3; ++c) {
                        sc.dmInv64[9 * g + 3 * c + 0] = r64.dm_inv.c[c].x;
                        sc.dmInv64[9 * g + 3 * c + 1] = r64.dm_inv.c[c].y;
                        sc.dmInv64[9 * g + 3 * c + 2] = r64.dm_inv.c[c].z;
                    }
                    sc.volume64[g] = r64.volume;
                    double l64, m64;
                    LameParameters<double>(t.youngModulus, t.poissonRatio, l64, m64);
                    sc.lam64[g] = l64;
                    sc.mu64[g] = m64;
                    const double d64 = std::max(0.0, static_cast<double>(body->material.density));
                    if (std::isfinite(d64) && t.active && std::isfinite(r64.volume) && r64.volume > 0.0) {
                        const double share = d64 * r64.volume * 0.25;
                        if (std::isfinite(share) && share > 0.0) nodal64[g] = share;
                    }
                }
            }
        });
        first += tets.size();
    }
    // Host-emitted masses of custom components emitted before the node's soft body, then the
    // lumped mass rho V / 4 to the non-fixed nodes of active tets, summed in tet order, then
    // the host-emitted masses emitted after it (SolverData::AssembleMasses sums every mass
    // in emission order).
    const auto& extraMasses = w.GetExtraMasses();
    for (const auto& e : extraMasses)
        if (!std::get<2>(e)) massT[static_cast<std::size_t>(std::get<0>(e))] += T(std::get<1>(e));
    for (std::size_t g = 0; g < total; ++g) {
        if (!(nodal[g] > T(0))) continue;
        for (int k = 0; k < 4; ++k) {
            const int n = sc.tetNodes[4 * g + k];
            if (!nodes[static_cast<std::size_t>(n)].fixed) massT[static_cast<std::size_t>(n)] += nodal[g];
        }
    }
    for (const auto& e : extraMasses)
        if (std::get<2>(e)) massT[static_cast<std::size_t>(std::get<0>(e))] += T(std::get<1>(e));
    sc.extraMasses = extraMasses;
    if (sc.rest64) {
        // the same sums in FP64, in the same order
        sc.mass64.assign(static_cast<std::size_t>(nn), 0.0);
        for (const auto& e : extraMasses)
            if (!std::get<2>(e)) sc.mass64[static_cast<std::size_t>(std::get<0>(e))] += double(std::get<1>(e));
        for (std::size_t g = 0; g < total; ++g) {
            if (!(nodal64[g] > 0.0)) continue;
            for (int k = 0; k < 4; ++k) {
                const int n = sc.tetNodes[4 * g + k];
                if (!nodes[static_cast<std::size_t>(n)].fixed) sc.mass64[static_cast<std::size_t>(n)] += nodal64[g];
            }
        }
        for (const auto& e : extraMasses)
            if (std::get<2>(e)) sc.mass64[static_cast<std::size_t>(std::get<0>(e))] += double(std::get<1>(e));
    }
    // World::ValidateNodeMasses
    for (int i = 0; i < nn; ++i) {
        const Node& nd = nodes[static_cast<std::size_t>(i)];
        if (!nd.active || nd.fixed) continue;
        const T m = massT[static_cast<std::size_t>(i)];
        if (std::isfinite(static_cast<double>(m)) && m > T(0)) continue;
        throw std::runtime_error("Non-fixed node has no physical mass contribution. nodeIndex=" + std::to_string(i));
    }
    // Dynamic rows.
    sc.nodeToDyn.assign(static_cast<std::size_t>(nn), -1);
    sc.dynToNode.clear();
    for (int i = 0; i < nn; ++i) {
        const Node& nd = nodes[static_cast<std::size_t>(i)];
        const T m = massT[static_cast<std::size_t>(i)];
        if (nd.active && !nd.fixed && std::isfinite(static_cast<double>(m)) && m > T(0)) {
            sc.nodeToDyn[static_cast<std::size_t>(i)] = static_cast<int>(sc.dynToNode.size());
            sc.dynToNode.push_back(i);
        }
    }
    const int dyn = static_cast<int>(sc.dynToNode.size());
    const int tetCount = static_cast<int>(sc.enabled.size());
    // Per-row incidence lists (ascending tet id) and the canonical upper pattern.
    sc.incStart.assign(static_cast<std::size_t>(dyn) + 1, 0);
    for (int t = 0; t < tetCount; ++t)
        for (int k = 0; k < 4; ++k) {
            const int r = sc.nodeToDyn[static_cast<std::size_t>(sc.tetNodes[4 * t + k])];
            if (r >= 0) sc.incStart[static_cast<std::size_t>(r) + 1]++;
        }
    for (int r = 0; r < dyn; ++r) sc.incStart[r + 1] += sc.incStart[r];
    sc.incList.assign(static_cast<std::size_t>(sc.incStart[dyn]), 0);
    {
        std::vector<int> fill(sc.incStart.begin(), sc.incStart.end() - 1);
        for (int t = 0; t < tetCount; ++t)
            for (int k = 0; k < 4; ++k) {
                const int r = sc.nodeToDyn[static_cast<std::size_t>(sc.tetNodes[4 * t + k])];
                if (r >= 0) sc.incList[static_cast<std::size_t>(fill[r]++)] = t * 4 + k;
            }
    }
    sc.rowStart.assign(static_cast<std::size_t>(dyn) + 1, 0);
    sc.colIndex.clear();
    sc.colIndex.reserve(static_cast<std::size_t>(sc.incStart[dyn]) / 2 + static_cast<std::size_t>(dyn));
    std::vector<int> cols;
    std::vector<int> seen(static_cast<std::size_t>(dyn), -1);  // the last row that listed the column
    for (int r = 0; r < dyn; ++r) {
        cols.clear();
        cols.push_back(r);
        seen[static_cast<std::size_t>(r)] = r;
        for (int i = sc.incStart[r]; i < sc.incStart[r + 1]; ++i) {
            const int t = sc.incList[static_cast<std::size_t>(i)] >> 2;
            for (int k = 0; k < 4; ++k) {
                const int c = sc.nodeToDyn[static_cast<std::size_t>(sc.tetNodes[4 * t + k])];
                if (c > r && seen[static_cast<std::size_t>(c)] != r) {
                    seen[static_cast<std::size_t>(c)] = r;
                    cols.push_back(c);
                }
            }
        }
        std::sort(cols.begin(), cols.end());
        sc.colIndex.insert(sc.colIndex.end(), cols.begin(), cols.end());
        sc.rowStart[static_cast<std::size_t>(r) + 1] = static_cast<int>(sc.colIndex.size());
    }
    // Body segments: each body's nodes are one contiguous world range, so its dynamic rows
    // are one contiguous row range; bodies taken in node order.
    {
        std::vector<std::pair<int, const TetMeshPhysicsComponent*>> byBase;
        for (const TetMeshPhysicsComponent* body : fem) byBase.emplace_back(body->GetGlobalNodeBeginIndex(), body);
        std::sort(byBase.begin(), byBase.end(),
                  [](const auto& a, const auto& b) { return a.first < b.first; });
        sc.segStart.assign(1, 0);
        sc.bodySegment.clear();
        int covered = 0;
        bool ok = true;
        for (const auto& e : byBase) {
            const int b0 = e.first, b1 = b0 + e.second->GetGlobalNodeCount();
            int first = -1, last = -1;
            for (int i = b0; i < b1 && i < nn; ++i) {
                const int r = sc.nodeToDyn[static_cast<std::size_t>(i)];
                if (r < 0) continue;
                if (first < 0) first = r;
                last = r;
            }
            if (first < 0) {  // no dynamic row: an empty segment
                sc.bodySegment.emplace_back(e.second, static_cast<int>(sc.segStart.size()) - 1);
                sc.segStart.push_back(covered);
                continue;
            }
            if (first != covered || last - first + 1 != [&] {
                    int c = 0;
                    for (int i = b0; i < b1 && i < nn; ++i) c += sc.nodeToDyn[static_cast<std::size_t>(i)] >= 0;
                    return c;
                }())
                ok = false;
            sc.bodySegment.emplace_back(e.second, static_cast<int>(sc.segStart.size()) - 1);
            covered = last + 1;
            sc.segStart.push_back(covered);
        }
        sc.segmentsCover = ok && covered == dyn && !byBase.empty();
    }
    sc.mass.assign(massT.begin(), massT.end());
    sc.nodeCount = nn;
    sc.dynCount = dyn;
    sc.tetCount = tetCount;
    sc.femRowStart = sc.rowStart;
    sc.femColIndex = sc.colIndex;
    sc.connPairs.clear();
    sc.connVersion = 0;
    sc.connCount = 0;
    sc.connOnDevice = false;
}

void UploadRest64(DeviceScene& sc)
{
    if (!sc.rest64) return;
    Check(pk_system_set_rest64(sc.sys, sc.tetCount, sc.dmInv64.data(), sc.volume64.data(), sc.lam64.data(),
                               sc.mu64.data(), sc.damp.data(), sc.nodeCount, sc.mass64.data()),
          "set_rest64");
}

void UploadScene(DeviceScene& sc, const std::vector<Vec3>& positions, const std::vector<Vec3>& velocities)
{
    const int nn = sc.nodeCount;
    Check(pk_system_set_nodes(sc.sys, nn, sc.nodeToDyn.data(), sc.mass.data()), "set_nodes");
    std::vector<float> x(3 * static_cast<std::size_t>(nn)), v(3 * static_cast<std::size_t>(nn));
    for (int i = 0; i < nn; ++i) {
        x[3 * i] = positions[i].x; x[3 * i + 1] = positions[i].y; x[3 * i + 2] = positions[i].z;
        v[3 * i] = velocities[i].x; v[3 * i + 1] = velocities[i].y; v[3 * i + 2] = velocities[i].z;
    }
    Check(pk_system_set_state_f32(sc.sys, x.data(), v.data()), "set_state");
    Check(pk_system_set_tets(sc.sys, sc.tetCount, sc.tetNodes.data(), sc.enabled.data(), sc.dmInv.data(),
                             sc.volume.data(), sc.lam.data(), sc.mu.data(), sc.damp.data()),
          "set_tets");
    Check(pk_system_set_pattern(sc.sys, sc.dynCount, sc.dynToNode.data(), sc.rowStart.data(), sc.colIndex.data(),
                                sc.incStart.data(), sc.incList.data()),
          "set_pattern");
    UploadRest64(sc);
    sc.devDyn = sc.dynCount;
    sc.devNnz = static_cast<int>(sc.colIndex.size());
    sc.batchedOnDevice = false;
    sc.graphOnDevice = false;
    sc.refineOnDevice = 0;
    sc.uploaded = true;
}

}  // namespace

// ------------------------------------------------------------------ World
World::World() = default;
World::~World() = default;

void World::SetSubstepCount(int count) { substepCount = std::max(1, count); }

void World::SetConjugateGradientTolerance(float tolerance)
{
    if (!std::isfinite(tolerance)) return;
    conjugateGradientSettings.tolerance =
        std::clamp(tolerance, kMinConjugateGradientTolerance, kMaxConjugateGradientTolerance);
}

void World::SetConjugateGradientMaxIterations(int maxIterations)
{
    conjugateGradientSettings.maxIterations =
        std::clamp(maxIterations, kMinConjugateGradientMaxIterations, kMaxConjugateGradientMaxIterations);
}

// Everything that lives on the device system is brought to the host before the system
// goes: the node state, the components' local position copies, pending visual results.
void World::ReleaseDeviceScene()
{
    EnsureHostState();
    FlushLocalPositionSnapshots();
    for (auto& c : components)
        if (c) c->ReleaseDeviceResources();
    snapshotOnDevice = false;
    scene.reset();
}

void World::SetPrecision(Precision p)
{
    if (p == precision) return;
    ReleaseDeviceScene();
    precision = p;
    deviceStale = true;
    ++topologyVersion;
}

void World::SetDevice(int dev)
{
    if (dev == device) return;
    ReleaseDeviceScene();
    device = dev;
    deviceStale = true;
    ++topologyVersion;
}

int World::AddNode(const Vec3& position)
{
    EnsureHostState();
    Node n;
    n.stateIndex = static_cast<int>(positions.size());
    nodes.push_back(n);
    positions.push_back(position);
    velocities.push_back(Vec3{});
    deviceStale = true;
    ++topologyVersion;
    return static_cast<int>(nodes.size()) - 1;
}

ComponentHandle World::AddComponent(std::unique_ptr<Component> component)
{
    if (!component) return ComponentHandle{};
    Component* raw = component.get();
    std::uint32_t slot;
    if (!freeComponentSlots.empty()) {
        slot = freeComponentSlots.back();
        freeComponentSlots.pop_back();
        components[slot] = std::move(component);
    } else {
        components.push_back(std::move(component));
        componentGenerations.push_back(1u);
        slot = static_cast<std::uint32_t>(components.size() - 1);
    }
    orderedComponents.emplace(static_cast<int>(raw->GetExecutionPriority()), raw);
    // Render-buffer components add nothing to the implicit system.
    const bool geometry = dynamic_cast<SurfaceExtractionComponent*>(raw) || dynamic_cast<SurfaceVisualComponent*>(raw) ||
                          dynamic_cast<VisualMeshComponent*>(raw);
    if (!geometry) ++topologyVersion;
    return ComponentHandle{slot, componentGenerations[slot]};
}

bool World::IsComponentHandleValid(ComponentHandle h) const
{
    if (!h.IsValid() || h.index >= components.size()) return false;
    return componentGenerations[h.index] == h.generation && components[h.index] != nullptr;
}

Component* World::GetComponent(ComponentHandle h) { return IsComponentHandleValid(h) ? components[h.index].get() : nullptr; }
const Component* World::GetComponent(ComponentHandle h) const
{
    return IsComponentHandleValid(h) ? components[h.index].get() : nullptr;
}

void World::DestroyComponent(ComponentHandle h)
{
    if (!IsComponentHandleValid(h)) return;
    Component* c = components[h.index].get();
    const bool geometry = dynamic_cast<SurfaceExtractionComponent*>(c) || dynamic_cast<SurfaceVisualComponent*>(c) ||
                          dynamic_cast<VisualMeshComponent*>(c);
    for (auto it = orderedComponents.begin(); it != orderedComponents.end();)
        it = it->second == c ? orderedComponents.erase(it) : std::next(it);
    components[h.index].reset();
    if (++componentGenerations[h.index] == 0u) componentGenerations[h.index] = 1u;
    freeComponentSlots.push_back(h.index);
    if (!geometry) ++topologyVersion;
}

Node& World::GetNode(int index) { return nodes.at(static_cast<std::size_t>(index)); }
const Node& World::GetNode(int index) const { return nodes.at(static_cast<std::size_t>(index)); }

void World::EnsureHostState() const
{
    if (!hostStale || !scene || !scene->uploaded) return;
    const std::size_t n = positions.size();
    std::vector<float> x(3 * n), v(3 * n);
    Check(pk_system_get_state_f32(scene->sys, x.data(), v.data()), "get_state");
    for (std::size_t i = 0; i < n; ++i) {
        positions[i] = Vec3{x[3 * i], x[3 * i + 1], x[3 * i + 2]};
        velocities[i] = Vec3{v[3 * i], v[3 * i + 1], v[3 * i + 2]};
    }
    hostStale = false;
}

const Vec3& World::GetNodePosition(int i) const
{
    EnsureHostState();
    return positions.at(static_cast<std::size_t>(i));
}

const Vec3& World::GetNodeVelocity(int i) const
{
    EnsureHostState();
    return velocities.at(static_cast<std::size_t>(i));
}

void World::SetNodePosition(int i, const Vec3& p)
{
    EnsureHostState();
    positions.at(static_cast<std::size_t>(i)) = p;
    velocities.at(static_cast<std::size_t>(i)) = Vec3{};
    deviceStale = true;
}

void World::SetNodeVelocity(int i, const Vec3& v)
{
    EnsureHostState();
    velocities.at(static_cast<std::size_t>(i)) = v;
    deviceStale = true;
}

void World::SetNodeFixed(int i, bool fixed)
{
    EnsureHostState();
    Node& n = nodes.at(static_cast<std::size_t>(i));
    if (fixed) velocities[static_cast<std::size_t>(i)] = Vec3{};
    if (n.fixed != fixed) ++topologyVersion;
    n.fixed = fixed;
    deviceStale = true;
}

bool World::IsNodeFixed(int i) const { return nodes.at(static_cast<std::size_t>(i)).fixed; }

void World::SetNodeActive(int i, bool activeValue)
{
    // An active node that stays active changes nothing (the tet-deactivation reconcile
    // asks this of every corner): leave the state where it is, on the device.
    if (activeValue && nodes.at(static_cast<std::size_t>(i)).active) return;
    EnsureHostState();
    Node& n = nodes.at(static_cast<std::size_t>(i));
    if (n.active != activeValue) ++topologyVersion;
    n.active = activeValue;
    if (!activeValue) velocities[static_cast<std::size_t>(i)] = Vec3{};
    deviceStale = true;
}

void World::GetNodeStates(float* x, float* v) const
{
    if (hostStale && scene && scene->uploaded) {
        Check(pk_system_get_state_f32(scene->sys, x, v), "get_state");
        return;
    }
    for (std::size_t i = 0; i < positions.size(); ++i) {
        if (x) { x[3 * i] = positions[i].x; x[3 * i + 1] = positions[i].y; x[3 * i + 2] = positions[i].z; }
        if (v) { v[3 * i] = velocities[i].x; v[3 * i + 1] = velocities[i].y; v[3 * i + 2] = velocities[i].z; }
    }
}

void World::SetNodeStates(const float* x, const float* v)
{
    const bool live = scene && scene->uploaded && !deviceStale && scene->worldVersion == topologyVersion;
    if (live && x && v) {
        Check(pk_system_set_state_f32(scene->sys, x, v), "set_state");
        hostStale = true;
        return;
    }
    EnsureHostState();
    for (std::size_t i = 0; i < positions.size(); ++i) {
        if (x) positions[i] = Vec3{x[3 * i], x[3 * i + 1], x[3 * i + 2]};
        if (v) velocities[i] = Vec3{v[3 * i], v[3 * i + 1], v[3 * i + 2]};
    }
    deviceStale = true;
}

void World::GetNodeStatesF64(double* x, double* v) const
{
    if (hostStale && scene && scene->uploaded) {
        Check(pk_system_get_state_f64(scene->sys, x, v), "get_state");
        return;
    }
    for (std::size_t i = 0; i < positions.size(); ++i) {
        if (x) { x[3 * i] = positions[i].x; x[3 * i + 1] = positions[i].y; x[3 * i + 2] = positions[i].z; }
        if (v) { v[3 * i] = velocities[i].x; v[3 * i + 1] = velocities[i].y; v[3 * i + 2] = velocities[i].z; }
    }
}

void World::SetNodeStatesF64(const double* x, const double* v)
{
    const bool live = scene && scene->uploaded && !deviceStale && scene->worldVersion == topologyVersion;
    if (live && x && v) {
        Check(pk_system_set_state_f64(scene->sys, x, v), "set_state");
        hostStale = true;
        return;
    }
    EnsureHostState();
    for (std::size_t i = 0; i < positions.size(); ++i) {
        if (x) positions[i] = Vec3{static_cast<float>(x[3 * i]), static_cast<float>(x[3 * i + 1]),
                                   static_cast<float>(x[3 * i + 2])};
        if (v) velocities[i] = Vec3{static_cast<float>(v[3 * i]), static_cast<float>(v[3 * i + 1]),
                                    static_cast<float>(v[3 * i + 2])};
    }
    deviceStale = true;
}

void World::SyncStats() const
{
    if (!statsPending || !scene || !scene->uploaded) return;
    pk_step_stats st{};
    const int rc = pk_system_stats(scene->sys, &st);
    statsPending = false;
    lastFlags = st.flags;
    if (rc == PK_ERR_TIMEOUT) throw std::runtime_error("device step timed out in a grid barrier");
    Check(rc, "stats");
    lastConjugateGradientResult.iterations = st.iterations;
    lastConjugateGradientResult.residualNorm = static_cast<float>(st.residual_norm);
    lastConjugateGradientResult.converged = st.converged != 0;
}

int World::GetLastConjugateGradientIterations() const
{
    SyncStats();
    return lastConjugateGradientResult.iterations;
}
float World::GetLastConjugateGradientResidualNorm() const
{
    SyncStats();
    return lastConjugateGradientResult.residualNorm;
}
bool World::DidLastConjugateGradientSolveConverge() const
{
    SyncStats();
    return lastConjugateGradientResult.converged;
}
unsigned World::GetLastStepFlags() const
{
    SyncStats();
    return lastFlags;
}

pk_system* World::GetDeviceSystem() { return scene && scene->uploaded ? scene->sys : nullptr; }

pk_system* World::GeometrySystem(const TetMeshPhysicsComponent* body, bool snapshot) const
{
    if (!scene || !scene->sys) return nullptr;
    if (snapshot)
        return snapshotOnDevice && body && body->snapshotWanted == snapshotGeneration &&
                       body->localEdits == body->snapshotEdits
                   ? scene->sys
                   : nullptr;
    const bool live = scene->uploaded && !deviceStale && scene->worldVersion == topologyVersion;
    return live ? scene->sys : nullptr;
}

bool World::SceneMatchesDevice() const
{
    return scene && scene->uploaded && scene->devDyn == scene->dynCount &&
           scene->devNnz == static_cast<int>(scene->colIndex.size());
}

void World::PreUpdateComponents(float dt)
{
    for (auto& e : orderedComponents)
        if (e.second && e.second->active) e.second->PreUpdate(*this, dt);
}

void World::PostUpdateComponents(float dt)
{
    for (auto& e : orderedComponents)
        if (e.second && e.second->active) e.second->PostUpdate(*this, dt);
}

// ------------------------------------------------------------------ collision spheres
std::unique_ptr<CollisionSphereComponent> CollisionSphereComponent::Create(const Vec3& position, float radius)
{
    auto c = std::make_unique<CollisionSphereComponent>();
    c->transform.position = position;
    c->radius = std::max(0.0f, radius);
    return c;
}

namespace {
float SanitizeConnectionValue(float v) { return std::isfinite(v) ? std::max(0.0f, v) : 0.0f; }
}  // namespace

void CollisionSphereComponent::SetConnectionSettings(float stiffness, float damping)
{
    SetConnectionStiffness(stiffness);
    SetConnectionDamping(damping);
}
void CollisionSphereComponent::SetConnectionStiffness(float stiffness) { contactStiffness = SanitizeConnectionValue(stiffness); }
void CollisionSphereComponent::SetConnectionDamping(float damping) { contactDamping = SanitizeConnectionValue(damping); }

void CollisionSphereComponent::UpdateSystem(World& world, SolverData&, float)
{
    if (!active || radius <= 0.0f) return;
    if (isSensor || !generateConnections) return;
    world.RequestSphereContacts(this);
}

namespace {
// The contact of CollisionSphereComponent::UpdateSystem and AddPointConnectionFromContact
// (CollisionSphereComponent.cpp:46-66, 165-188) from a centroid, in the arithmetic T of the
// state (float as the reference; double for FP64 worlds, rounded to the connection's
// floats at the end).  Returns false when the penetration is not positive.
template <class T>
bool SphereContact(const double* point, const Vec3& center, float radius, float stiffness, float damping,
                   const int* nodes, PointConnection& out)
{
    const T px = T(point[0]), py = T(point[1]), pz = T(point[2]);
    const T cx = px - T(center.x), cy = py - T(center.y), cz = pz - T(center.z);
    const T dist = std::sqrt(cx * cx + cy * cy + cz * cz);
    T nx = T(0), ny = T(0), nz = T(1);  // NormalizeOrFallback
    if (dist > T(0.00001f)) {
        nx = cx / dist;
        ny = cy / dist;
        nz = cz / dist;
    }
    const T depth = T(radius) - dist;
    if (!(depth > T(0))) return false;
    out.node0 = nodes[0];
    out.node1 = nodes[1];
    out.node2 = nodes[2];
    out.node3 = nodes[3];
    out.barycentric = Vec4{0.25f, 0.25f, 0.25f, 0.25f};
    out.targetPosition = Vec3{static_cast<float>(px + nx * depth), static_cast<float>(py + ny * depth),
                              static_cast<float>(pz + nz * depth)};
    out.stiffness = stiffness;
    out.damping = damping;
    return true;
}
}  // namespace

void World::AddSphereContacts()
{
    if (sphereRequests.empty() || !scene || !scene->sys) return;
    std::vector<int> tets;
    std::vector<double> points;
    for (const CollisionSphereComponent* sphere : sphereRequests) {
        const double center[3] = {sphere->transform.position.x, sphere->transform.position.y,
                                  sphere->transform.position.z};
        const int n = pk_system_sphere_contacts(scene->sys, center, sphere->radius, 0, nullptr, nullptr);
        Check(n < 0 ? n : 0, "sphere_contacts");
        if (n == 0) continue;
        tets.resize(static_cast<std::size_t>(n));
        points.resize(3 * static_cast<std::size_t>(n));
        Check(pk_system_sphere_contacts(scene->sys, center, sphere->radius, n, tets.data(), points.data()) == n ? 0
                                                                                                              : PK_ERR_STATE,
              "sphere_contacts");
        for (int i = 0; i < n; ++i) {
            const int t = tets[static_cast<std::size_t>(i)];
            PointConnection c;
            const bool ok =
                precision == Precision::FP64
                    ? SphereContact<double>(&points[3 * static_cast<std::size_t>(i)], sphere->transform.position,
                                            sphere->radius, sphere->GetConnectionStiffness(),
                                            sphere->GetConnectionDamping(), &scene->tetNodes[4 * static_cast<std::size_t>(t)], c)
                    : SphereContact<float>(&points[3 * static_cast<std::size_t>(i)], sphere->transform.position,
                                           sphere->radius, sphere->GetConnectionStiffness(),
                                           sphere->GetConnectionDamping(), &scene->tetNodes[4 * static_cast<std::size_t>(t)], c);
            if (ok) AddPointConnection(c);
        }
    }
    sphereRequests.clear();
}

void World::CollectContributions(float dt)
{
    solverData.ClearTransientState();
    sphereRequests.clear();
    for (auto& e : orderedComponents)
        if (e.second && e.second->active) e.second->UpdateSystem(*this, solverData, dt);
    BuildExtras();
}

// The host-emitted contributions of custom components, checked as SolverData does:
// masses that are out of range, not finite or not positive are dropped (AssembleMasses,
// SolverData.cpp:87-101), so are forces out of range or not finite (PrecomputeImplicitSolve,
// :145-154) and blocks with a node out of range (:337-343); a non-finite block fails the
// step (:351-354).  A mass counts after its node's soft-body masses when it was emitted
// after that body registered (execution priority), so the sums keep the reference's order.
void World::BuildExtras()
{
    extras = Extras{};
    const int nn = static_cast<int>(nodes.size());
    const auto& masses = solverData.GetNodeMasses();
    const auto& forces = solverData.GetNodeForces();
    const auto& blocks = solverData.GetStiffnessBlocks();
    extras.any = !masses.empty() || !forces.empty() || !blocks.empty();
    if (!extras.any) return;
    // The registration mark of the soft body holding each node (-1: none).
    std::vector<long long> mark;
    if (!masses.empty()) {
        mark.assign(static_cast<std::size_t>(nn), -1);
        const auto& fem = solverData.GetFemBodies();
        for (std::size_t b = 0; b < fem.size(); ++b) {
            const int b0 = fem[b]->GetGlobalNodeBeginIndex(), cnt = fem[b]->GetGlobalNodeCount();
            for (int i = std::max(0, b0); i < std::min(nn, b0 + cnt); ++i)
                mark[static_cast<std::size_t>(i)] = static_cast<long long>(solverData.femMassMark[b]);
        }
    }
    for (std::size_t k = 0; k < masses.size(); ++k) {
        const auto& m = masses[k];
        if (m.node < 0 || m.node >= nn || !std::isfinite(m.mass) || !(m.mass > 0.0f)) continue;
        const long long mk = mark[static_cast<std::size_t>(m.node)];
        extras.masses.emplace_back(m.node, m.mass, mk >= 0 && static_cast<long long>(k) >= mk);
    }
    for (const auto& f : forces) {
        if (f.node < 0 || f.node >= nn || !std::isfinite(f.force.x) || !std::isfinite(f.force.y) ||
            !std::isfinite(f.force.z))
            continue;
        if (extras.force.empty()) extras.force.assign(static_cast<std::size_t>(nn), Vec3{});
        extras.force[static_cast<std::size_t>(f.node)] += f.force;
    }
    for (const auto& b : blocks) {
        if (b.nodeA < 0 || b.nodeA >= nn || b.nodeB < 0 || b.nodeB >= nn) continue;
        extras.blocks.push_back(b);
    }
}

void World::EnsureScene(bool upload)
{
    const std::vector<const TetMeshPhysicsComponent*>& fem = solverData.GetFemBodies();
    if (!scene || scene->precision != precision || scene->device != device) {
        if (scene) ReleaseDeviceScene();
        EnsureHostState();
        scene = std::make_unique<DeviceScene>();
        scene->precision = precision;
        scene->device = device;
    }
    if (!scene->Matches(*this, fem)) {
        EnsureHostState();
        // What the device holds: when a rebuild keeps the dynamic rows, the pattern, the
        // incidences and the tets' nodes (tets deactivated while their nodes stay dynamic,
        // a material change), only the masses and the tet data are uploaded again -- the
        // device keeps its state, its PCG layouts and its segments.
        const bool update = scene->uploaded && scene->connPairs.empty();
        std::vector<int> oldN2D, oldRowStart, oldCol, oldIncStart, oldInc, oldTets;
        if (update) {
            oldN2D.swap(scene->nodeToDyn);
            oldRowStart.swap(scene->femRowStart);
            oldCol.swap(scene->femColIndex);
            oldIncStart.swap(scene->incStart);
            oldInc.swap(scene->incList);
            oldTets.swap(scene->tetNodes);
        }
        scene->built = false;
        scene->uploaded = false;
        scene->bodies.clear();
        for (const TetMeshPhysicsComponent* b : fem) scene->bodies.emplace_back(b, b->version);
        if (precision == Precision::FP64)
            BuildHostScene<double>(*scene, *this, fem);
        else
            BuildHostScene<float>(*scene, *this, fem);
        scene->worldVersion = topologyVersion;
        scene->built = true;
        DeviceScene& sc = *scene;
        if (update && oldN2D == sc.nodeToDyn && oldRowStart == sc.femRowStart && oldCol == sc.femColIndex &&
            oldIncStart == sc.incStart && oldInc == sc.incList && oldTets == sc.tetNodes) {
            Check(pk_system_set_masses(sc.sys, sc.mass.data()), "set_masses");
            Check(pk_system_set_tets(sc.sys, sc.tetCount, sc.tetNodes.data(), sc.enabled.data(), sc.dmInv.data(),
                                     sc.volume.data(), sc.lam.data(), sc.mu.data(), sc.damp.data()),
                  "set_tets");
            UploadRest64(sc);
            sc.uploaded = true;
        }
    }
    const bool patternChanged = SyncConnections();
    if (upload && !scene->uploaded) {
        FlushLocalPositionSnapshots();  // the upload drops the device snapshot
        snapshotOnDevice = false;
        EnsureHostState();
        if (!scene->sys) Check(pk_system_create(device, static_cast<int>(precision), &scene->sys), "pk_system_create");
        UploadScene(*scene, positions, velocities);
        scene->connOnDevice = false;
        scene->extOnDevice = false;
        deviceStale = false;
        hostStale = false;
    } else if (upload && patternChanged) {
        DeviceScene& sc = *scene;
        Check(pk_system_set_pattern(sc.sys, sc.dynCount, sc.dynToNode.data(), sc.rowStart.data(), sc.colIndex.data(),
                                    sc.incStart.data(), sc.incList.data()),
              "set_pattern");
        sc.devDyn = sc.dynCount;
        sc.devNnz = static_cast<int>(sc.colIndex.size());
        sc.batchedOnDevice = false;  // set_pattern drops the segments
        sc.connOnDevice = false;
        sc.extOnDevice = false;
    }
    if (upload && scene->uploaded && !scene->connOnDevice) {
        DeviceScene& sc = *scene;
        Check(pk_system_set_connections(sc.sys, sc.connCount, sc.connNodes.data(), sc.connParams.data(),
                                        sc.connIncStart.data(), sc.connIncList.data()),
              "set_connections");
        sc.connOnDevice = true;
    }
    if (upload && scene->uploaded && (extras.any || scene->extOnDevice) && !extras.failed) {
        DeviceScene& sc = *scene;
        const bool on = extras.any;
        Check(pk_system_set_extras(sc.sys, on ? sc.extCount : 0, sc.extBlocks.data(), sc.extNodes.data(),
                                   sc.extRhsStart.data(), sc.extRhsList.data(), sc.extMatStart.data(),
                                   sc.extMatList.data(), on && !sc.extForce.empty() ? sc.extForce.data() : nullptr),
              "set_extras");
        sc.extOnDevice = on;
    }
}

// The device lists of this substep's host-emitted blocks and forces (World::BuildExtras),
// assembled as SolverData::AssembleImplicitMatrixAndRhs does (SolverData.cpp:308-465):
// every block whose row node is dynamic adds -dt^2 B v_column to that row's rhs; when its
// column node is dynamic too it is a matrix block, kept in the upper triangle -- B at
// (row, column), or B^T at (column, row) for a lower block -- except a lower block whose
// upper twin is emitted as well (by another host block, or by the soft bodies and point
// connections, which emit both orientations).  The dynamic coordinate pairs of the kept
// blocks join the pattern (`pairs`).  Returns whether host-emitted contributions exist.
bool World::SyncExtras(std::vector<std::pair<int, int>>& pairs)
{
    DeviceScene& sc = *scene;
    sc.extCount = 0;
    sc.extBlocks.clear();
    sc.extNodes.clear();
    sc.extForce.clear();
    sc.extRhsList.clear();
    sc.extMatList.clear();
    sc.extRhsStart.clear();
    sc.extMatStart.clear();
    extras.failed = false;
    if (!extras.any) return false;
    const int dyn = sc.dynCount;
    auto dynOf = [&](int node) { return sc.nodeToDyn[static_cast<std::size_t>(node)]; };
    auto key = [](int r, int c) {
        return (static_cast<std::uint64_t>(static_cast<std::uint32_t>(r)) << 32) | static_cast<std::uint32_t>(c);
    };
    std::vector<std::pair<int, int>> rhsInc, matInc;  // (row, entry)
    std::unordered_map<std::uint64_t, int> emitted;   // dynamic (row, column) coordinates emitted
    std::vector<int> kept;                            // extras.blocks index of each device block
    for (std::size_t i = 0; i < extras.blocks.size(); ++i) {
        const auto& b = extras.blocks[i];
        const int ra = dynOf(b.nodeA);
        if (ra < 0) continue;
        const Mat3& m = b.block;
        for (int c = 0; c < 3; ++c)
            if (!std::isfinite(m.columns[c].x) || !std::isfinite(m.columns[c].y) || !std::isfinite(m.columns[c].z)) {
                extras.failed = true;
                return true;
            }
        const int k = static_cast<int>(kept.size());
        kept.push_back(static_cast<int>(i));
        rhsInc.emplace_back(ra, k);
        const int cb = dynOf(b.nodeB);
        if (cb >= 0) emitted.emplace(key(ra, cb), 1);
    }
    auto femHas = [&](int r, int c) {  // the soft bodies couple dynamic rows r <= c
        const auto b0 = sc.femColIndex.begin() + sc.femRowStart[static_cast<std::size_t>(r)];
        const auto b1 = sc.femColIndex.begin() + sc.femRowStart[static_cast<std::size_t>(r) + 1];
        return std::binary_search(b0, b1, c);
    };
    for (int k = 0; k < static_cast<int>(kept.size()); ++k) {
        const auto& b = extras.blocks[static_cast<std::size_t>(kept[static_cast<std::size_t>(k)])];
        const int ra = dynOf(b.nodeA), cb = dynOf(b.nodeB);
        if (cb < 0) continue;
        if (ra > cb && (emitted.count(key(cb, ra)) || femHas(cb, ra) ||
                        std::binary_search(sc.connOnlyPairs.begin(), sc.connOnlyPairs.end(), std::make_pair(cb, ra))))
            continue;
        const bool tr = ra > cb;
        matInc.emplace_back(tr ? cb : ra, k | (tr ? static_cast<int>(0x80000000u) : 0));
        pairs.emplace_back(std::min(ra, cb), std::max(ra, cb));
    }
    sc.extCount = static_cast<int>(kept.size());
    for (int k : kept) {
        const auto& b = extras.blocks[static_cast<std::size_t>(k)];
        for (int c = 0; c < 3; ++c) {
            sc.extBlocks.push_back(b.block.columns[c].x);
            sc.extBlocks.push_back(b.block.columns[c].y);
            sc.extBlocks.push_back(b.block.columns[c].z);
        }
        sc.extNodes.push_back(b.nodeA);
        sc.extNodes.push_back(b.nodeB);
    }
    auto csr = [&](const std::vector<std::pair<int, int>>& inc, std::vector<int>& start, std::vector<int>& list) {
        start.assign(static_cast<std::size_t>(dyn) + 1, 0);
        for (const auto& e : inc) start[static_cast<std::size_t>(e.first) + 1]++;
        for (int r = 0; r < dyn; ++r) start[static_cast<std::size_t>(r) + 1] += start[static_cast<std::size_t>(r)];
        list.assign(inc.size(), 0);
        std::vector<int> fill(start.begin(), start.end() - 1);
        for (const auto& e : inc) list[static_cast<std::size_t>(fill[static_cast<std::size_t>(e.first)]++)] = e.second;
    };
    csr(rhsInc, sc.extRhsStart, sc.extRhsList);
    csr(matInc, sc.extMatStart, sc.extMatList);
    if (!extras.force.empty()) {
        sc.extForce.assign(3 * static_cast<std::size_t>(dyn), 0.0);
        for (int r = 0; r < dyn; ++r) {
            const Vec3& f = extras.force[static_cast<std::size_t>(sc.dynToNode[static_cast<std::size_t>(r)])];
            sc.extForce[3 * static_cast<std::size_t>(r)] = f.x;
            sc.extForce[3 * static_cast<std::size_t>(r) + 1] = f.y;
            sc.extForce[3 * static_cast<std::size_t>(r) + 2] = f.z;
        }
    }
    return true;
}

// The device arrays of the current point connections and the pattern they need:
// PointConnection::UpdateSystem's checks that do not depend on the state (valid, active
// nodes; finite, non-negative stiffness and damping; finite target) drop a connection;
// each kept one lists its corners with a non-zero weight under their dynamic rows
// (connection order), and with stiffness > 0 couples every pair of them
// (SolverData::AssembleImplicitMatrixAndRhs gives both orientations one canonical block,
// SolverData.cpp:337-393).  A kept connection whose point or velocity is not finite in a
// step contributes nothing then (the device checks), its blocks staying in the pattern as
// zeros.  Returns whether the joined pattern changed.
bool World::SyncConnections()
{
    DeviceScene& sc = *scene;
    const bool connChanged = sc.connVersion != connectionVersion;
    if (!connChanged && !extras.any && !sc.extOnDevice) return false;
    std::vector<std::pair<int, int>> pairs;
    const int dyn = sc.dynCount;
    if (connChanged) {
        sc.connVersion = connectionVersion;
        sc.connNodes.clear();
        sc.connParams.clear();
        std::vector<std::pair<int, int>> inc;  // (row, connection * 4 + corner)
        int count = 0;
        for (const PointConnection& pc : transientConnections) {
            if (!HasValidNodeIndices(pc) || !std::isfinite(pc.stiffness) || !std::isfinite(pc.damping) ||
                pc.stiffness < 0.0f || pc.damping < 0.0f || !std::isfinite(pc.targetPosition.x) ||
                !std::isfinite(pc.targetPosition.y) || !std::isfinite(pc.targetPosition.z))
                continue;
            const int nd[4] = {pc.node0, pc.node1, pc.node2, pc.node3};
            const float w[4] = {pc.barycentric.x, pc.barycentric.y, pc.barycentric.z, pc.barycentric.w};
            for (int a = 0; a < 4; ++a) {
                sc.connNodes.push_back(nd[a]);
                sc.connParams.push_back(w[a]);
            }
            sc.connParams.push_back(pc.targetPosition.x);
            sc.connParams.push_back(pc.targetPosition.y);
            sc.connParams.push_back(pc.targetPosition.z);
            sc.connParams.push_back(pc.stiffness);
            sc.connParams.push_back(pc.damping);
            for (int a = 0; a < 4; ++a) {
                const int ra = sc.nodeToDyn[static_cast<std::size_t>(nd[a])];
                if (w[a] == 0.0f || ra < 0) continue;
                inc.emplace_back(ra, count * 4 + a);
                if (!(pc.stiffness > 0.0f)) continue;
                for (int b = 0; b < 4; ++b) {
                    const int rb = sc.nodeToDyn[static_cast<std::size_t>(nd[b])];
                    if (w[b] == 0.0f || rb < 0) continue;
                    pairs.emplace_back(std::min(ra, rb), std::max(ra, rb));
                }
            }
            ++count;
        }
        sc.connCount = count;
        sc.connIncStart.assign(static_cast<std::size_t>(dyn) + 1, 0);
        for (const auto& e : inc) sc.connIncStart[static_cast<std::size_t>(e.first) + 1]++;
        for (int r = 0; r < dyn; ++r) sc.connIncStart[r + 1] += sc.connIncStart[r];
        sc.connIncList.assign(inc.size(), 0);
        {
            std::vector<int> fill(sc.connIncStart.begin(), sc.connIncStart.end() - 1);
            for (const auto& e : inc) sc.connIncList[static_cast<std::size_t>(fill[e.first]++)] = e.second;
        }
        sc.connOnDevice = false;
        std::sort(pairs.begin(), pairs.end());
        pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
        sc.connOnlyPairs = pairs;
    }
    pairs = sc.connOnlyPairs;
    SyncExtras(pairs);
    std::sort(pairs.begin(), pairs.end());
    pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
    if (pairs == sc.connPairs) return false;
    sc.connPairs = pairs;
    sc.rowStart.assign(static_cast<std::size_t>(dyn) + 1, 0);
    sc.colIndex.clear();
    std::vector<int> cols;
    std::size_t pi = 0;
    for (int r = 0; r < dyn; ++r) {
        cols.assign(sc.femColIndex.begin() + sc.femRowStart[r], sc.femColIndex.begin() + sc.femRowStart[r + 1]);
        for (; pi < pairs.size() && pairs[pi].first == r; ++pi) cols.push_back(pairs[pi].second);
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        sc.colIndex.insert(sc.colIndex.end(), cols.begin(), cols.end());
        sc.rowStart[static_cast<std::size_t>(r) + 1] = static_cast<int>(sc.colIndex.size());
    }
    return true;
}

void World::AddPointConnection(const PointConnection& connection)
{
    if (!HasValidNodeIndices(connection)) return;
    transientConnections.push_back(connection);
    ++connectionVersion;
}

bool World::HasValidNodeIndices(const PointConnection& c) const
{
    const int n = static_cast<int>(nodes.size());
    const int nd[4] = {c.node0, c.node1, c.node2, c.node3};
    for (int i : nd)
        if (i < 0 || i >= n || !nodes[static_cast<std::size_t>(i)].active) return false;
    return true;
}

void World::ClearSubstepConnections()
{
    if (firstSubstepConnectionIndex > transientConnections.size())
        firstSubstepConnectionIndex = transientConnections.size();
    if (transientConnections.size() != firstSubstepConnectionIndex) {
        transientConnections.resize(firstSubstepConnectionIndex);
        ++connectionVersion;
    }
}

void World::ClearFrameConnections()
{
    if (!transientConnections.empty()) {
        transientConnections.clear();
        ++connectionVersion;
    }
    firstSubstepConnectionIndex = 0;
}

void World::SetBatchedSolve(bool on) { batchedSolve = on; }

void World::AdjointStep(float dt, const double* xbarNext, const double* vbarNext, double* xbar, double* vbar,
                        double* thetaBar)
{
    if (solverMode != SolverMode::ImplicitEuler) throw std::runtime_error("the adjoint step needs the implicit solver");
    if (!transientConnections.empty()) throw std::runtime_error("the adjoint step does not take point connections");
    if (!(dt > 0.0f)) throw std::runtime_error("dt must be > 0");
    CollectContributions(dt);
    EnsureScene(true);
    if (deviceStale) {
        std::vector<float> x(3 * positions.size()), v(3 * positions.size());
        for (std::size_t i = 0; i < positions.size(); ++i) {
            x[3 * i] = positions[i].x; x[3 * i + 1] = positions[i].y; x[3 * i + 2] = positions[i].z;
            v[3 * i] = velocities[i].x; v[3 * i + 1] = velocities[i].y; v[3 * i + 2] = velocities[i].z;
        }
        Check(pk_system_set_state_f32(scene->sys, x.data(), v.data()), "set_state");
        deviceStale = false;
    }
    pk_step_params p{};
    p.dt = dt;
    p.gravity[0] = gravity.x;
    p.gravity[1] = gravity.y;
    p.gravity[2] = gravity.z;
    p.max_iterations = conjugateGradientSettings.maxIterations;
    p.tolerance = conjugateGradientSettings.tolerance;
    p.use_jacobi = conjugateGradientSettings.useJacobiPreconditioner ? 1 : 0;
    p.integrate = 0;
    Check(pk_system_adjoint_step(scene->sys, &p, xbarNext, vbarNext, xbar, vbar, thetaBar), "adjoint_step");
    statsPending = false;
}

int World::GetPcgKernel(int* blocks) const
{
    if (blocks) *blocks = 0;
    if (!scene || !scene->sys) return -1;
    return pk_system_pcg_kernel(scene->sys, blocks);
}

int World::GetPcgStreamForm() const
{
    if (!scene || !scene->sys) return -1;
    return pk_system_slab_form(scene->sys);
}

int World::Autotune(int repeats, double* bestMs)
{
    SyncStats();
    if (!scene || !scene->uploaded || solverMode != SolverMode::ImplicitEuler || scene->dynCount == 0) return -1;
    pk_step_params p{};
    p.dt = lastSubstepDt > 0.0f ? lastSubstepDt : 1.0f / 60.0f;
    p.gravity[0] = gravity.x;
    p.gravity[1] = gravity.y;
    p.gravity[2] = gravity.z;
    p.max_iterations = conjugateGradientSettings.maxIterations;
    p.tolerance = conjugateGradientSettings.tolerance;
    p.use_jacobi = conjugateGradientSettings.useJacobiPreconditioner ? 1 : 0;
    p.integrate = 0;
    int chosen = -1;
    double ms = 0.0;
    Check(pk_system_autotune(scene->sys, &p, repeats, &chosen, &ms), "autotune");
    if (bestMs) *bestMs = ms;
    return chosen;
}

bool World::GetBodyConjugateGradientStats(const Component* body, int& iterations, bool& converged,
                                          float& residualNorm, unsigned& flags) const
{
    SyncStats();
    if (!scene || !scene->uploaded || !scene->batchedOnDevice) return false;
    const int nseg = static_cast<int>(scene->segStart.size()) - 1;
    for (const auto& e : scene->bodySegment) {
        if (e.first != body) continue;
        std::vector<int> it(static_cast<std::size_t>(nseg)), conv(static_cast<std::size_t>(nseg));
        std::vector<double> res(static_cast<std::size_t>(nseg));
        std::vector<unsigned> fl(static_cast<std::size_t>(nseg));
        Check(pk_system_segment_stats(scene->sys, nseg, it.data(), conv.data(), res.data(), fl.data()),
              "segment_stats");
        iterations = it[static_cast<std::size_t>(e.second)];
        converged = conv[static_cast<std::size_t>(e.second)] != 0;
        residualNorm = static_cast<float>(res[static_cast<std::size_t>(e.second)]);
        flags = fl[static_cast<std::size_t>(e.second)];
        return true;
    }
    return false;
}

void World::FlushLocalPositionSnapshots()
{
    for (auto& e : orderedComponents) {
        auto* c = dynamic_cast<TetMeshPhysicsComponent*>(e.second);
        if (c && c->snapshotLoaded != c->snapshotWanted) RefreshLocalPositions(*c);
    }
}

void World::RefreshLocalPositions(TetMeshPhysicsComponent& c) const
{
    if (c.snapshotLoaded == c.snapshotWanted) return;
    const int count = c.globalNodeCount;
    if (!scene || !scene->sys || c.globalNodeBeginIndex < 0 || count <= 0) {
        c.snapshotLoaded = c.snapshotWanted;
        return;
    }
    std::vector<float> x(3 * static_cast<std::size_t>(count));
    Check(pk_system_get_snapshot_f32(scene->sys, c.globalNodeBeginIndex, count, x.data()), "get_snapshot");
    c.nodePositions.resize(static_cast<std::size_t>(count));
    for (int i = 0; i < count; ++i)
        c.nodePositions[static_cast<std::size_t>(i)] = Vec3{x[3 * i], x[3 * i + 1], x[3 * i + 2]};
    c.snapshotLoaded = c.snapshotWanted;
}

int World::PrepareScene(bool upload)
{
    CollectContributions(0.0f);
    EnsureScene(upload);
    return scene->dynCount;
}

int World::GetSceneDynamicCount() const { return scene && scene->built ? scene->dynCount : -1; }
int World::GetSceneBlockCount() const
{
    return scene && scene->built ? static_cast<int>(scene->colIndex.size()) : -1;
}
int World::GetSceneTetCount() const { return scene && scene->built ? scene->tetCount : -1; }
const std::vector<int>* World::GetSceneRowStart() const { return scene && scene->built ? &scene->rowStart : nullptr; }
const std::vector<int>* World::GetSceneColIndex() const { return scene && scene->built ? &scene->colIndex : nullptr; }
const std::vector<int>* World::GetSceneNodeToDyn() const { return scene && scene->built ? &scene->nodeToDyn : nullptr; }
const std::vector<double>* World::GetSceneMass() const { return scene && scene->built ? &scene->mass : nullptr; }

void World::RunSubstep(float dt)
{
    CollectContributions(dt);
    EnsureScene(true);
    if (deviceStale) {
        std::vector<float> x(3 * positions.size()), v(3 * positions.size());
        for (std::size_t i = 0; i < positions.size(); ++i) {
            x[3 * i] = positions[i].x; x[3 * i + 1] = positions[i].y; x[3 * i + 2] = positions[i].z;
            v[3 * i] = velocities[i].x; v[3 * i + 1] = velocities[i].y; v[3 * i + 2] = velocities[i].z;
        }
        Check(pk_system_set_state_f32(scene->sys, x.data(), v.data()), "set_state");
        deviceStale = false;
    }
    // Collision spheres' contacts, found on the device at this substep's positions, join
    // the point connections (after the frame's own ones, as the reference appends them).
    if (!sphereRequests.empty()) {
        AddSphereContacts();
        EnsureScene(true);
    }
    if (extras.failed) {
        // A non-finite host-emitted block: the implicit system cannot be assembled and the
        // substep is not applied (the reference would solve the part assembled so far).
        lastConjugateGradientResult = ConjugateGradientResult{};
        statsPending = false;
        lastFlags = PK_FLAG_PRECOMPUTE_FAILED;
        return;
    }
    if (scene->dynCount == 0) {
        // No dynamic node: PrecomputeImplicitSolve fails and nothing moves.
        if (solverMode == SolverMode::ImplicitEuler) lastConjugateGradientResult = ConjugateGradientResult{};
        return;
    }
    pk_step_params p{};
    p.dt = dt;
    p.gravity[0] = gravity.x;
    p.gravity[1] = gravity.y;
    p.gravity[2] = gravity.z;
    p.max_iterations = conjugateGradientSettings.maxIterations;
    p.tolerance = conjugateGradientSettings.tolerance;
    p.use_jacobi = conjugateGradientSettings.useJacobiPreconditioner ? 1 : 0;
    p.linear = 0;
    p.explicit_mode = solverMode == SolverMode::Explicit ? 1 : 0;
    p.integrate = 1;
    // Point connections may couple bodies: one coupled solve while any is present.
    const bool batch = batchedSolve && scene->segmentsCover && scene->segStart.size() > 2 && scene->connCount == 0;
    if (batch != scene->batchedOnDevice) {
        if (batch)
            Check(pk_system_set_segments(scene->sys, static_cast<int>(scene->segStart.size()) - 1,
                                         scene->segStart.data()),
                  "set_segments");
        Check(pk_system_set_batched(scene->sys, batch ? 1 : 0), "set_batched");
        scene->batchedOnDevice = batch;
    }
    if (graphCapture != scene->graphOnDevice) {
        Check(pk_system_set_graph(scene->sys, graphCapture ? 1 : 0), "set_graph");
        scene->graphOnDevice = graphCapture;
    }
    if (refinePasses != scene->refineOnDevice) {
        Check(pk_system_set_refinement(scene->sys, refinePasses), "set_refinement");
        scene->refineOnDevice = refinePasses;
    }
    lastSubstepDt = dt;
    Check(pk_system_step(scene->sys, &p), "pk_system_step");
    hostStale = true;
    if (solverMode == SolverMode::ImplicitEuler) statsPending = true;
}

void World::Step(float frameDt)
{
    if (frameDt < 0.0f) return;
    PreUpdateComponents(frameDt);
    MarkSubstepConnectionBegin();
    if (frameDt == 0.0f) {
        PostUpdateComponents(frameDt);
        ClearFrameConnections();
        return;
    }
    const int steps = std::max(1, substepCount);
    const float dt = frameDt / static_cast<float>(steps);
    for (int i = 0; i < steps; ++i) {
        RunSubstep(dt);
        ClearSubstepConnections();
    }
    SnapshotPositions();
    PostUpdateComponents(frameDt);
    ClearFrameConnections();
}

// Every active physics component copies the world's positions into its own at the end of
// a frame (TetMeshPhysicsComponent::PostUpdate, TetMeshPhysicsComponent.cpp:356-363).  The
// device copies the positions aside and a component's host copy is read from there on
// access (RefreshLocalPositions); a component that sits the frame out keeps its older copy,
// so it is fetched before the device copy is overwritten.
void World::SnapshotPositions()
{
    if (!scene || !scene->sys || !scene->uploaded) return;
    for (auto& e : orderedComponents) {
        auto* c = dynamic_cast<TetMeshPhysicsComponent*>(e.second);
        if (c && !c->active && c->snapshotLoaded != c->snapshotWanted) RefreshLocalPositions(*c);
    }
    Check(pk_system_snapshot_positions(scene->sys), "snapshot_positions");
    ++snapshotGeneration;
    snapshotOnDevice = true;
}

}  // namespace PhysiK
