// ref_harness.cpp -- drives the reference PhysiK library, compiled from its own
// sources by oracle/Makefile, for the parity tests and the CPU baseline.
//
// TEST INFRASTRUCTURE ONLY.  Scenes are built through the reference's own C++ API
// (TetMeshGenerator::Generate, TetMeshPhysicsComponent::CreateFromGeneratedTetMesh,
// World::AddComponent / SetNodeFixed / Step).  To read the assembled implicit system
// (SolverData's matrix, rhs, inverse preconditioner and delta velocity, which the
// reference keeps private) this translation unit opens the class internals; the
// library itself is compiled unmodified in its own translation units.
//
// All arrays cross this boundary as double so one Python wrapper serves the FP32
// reference and its float->double rebuild (the FP64 oracle).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#define private public
#define protected public
#include "PhysiK/Components/CollisionSphereComponent.h"
#include "PhysiK/Components/ScriptComponent.h"
#include "PhysiK/Components/TetMeshPhysicsComponent.h"
#include "PhysiK/Core/PhysicsConnections/PointConnection.h"
#include "PhysiK/Core/Solvers/SolverData.h"
#include "PhysiK/Core/World/World.h"
#include "PhysiK/Geometry/TetMeshGenerator.h"
#undef private
#undef protected

using namespace PhysiK;
using Real = decltype(Vec3{}.x);

namespace {
struct Harness {
    World world;
    std::vector<TetMeshPhysicsComponent*> bodies;
    std::vector<ComponentHandle> bodyHandles;
    std::vector<CollisionSphereComponent*> spheres;
    std::unique_ptr<SolverData> dump;
    std::string error;
};

Harness* H(void* h) { return static_cast<Harness*>(h); }
}  // namespace

extern "C" {

__attribute__((visibility("default"))) int ref_real_bytes() { return static_cast<int>(sizeof(Real)); }

__attribute__((visibility("default"))) void* ref_world_create() { return new Harness(); }

__attribute__((visibility("default"))) void ref_world_destroy(void* h) { delete H(h); }

__attribute__((visibility("default"))) void ref_world_settings(void* h, int implicit_mode, const double* gravity3,
                                                               int max_iterations, double tolerance, int substeps)
{
    World& w = H(h)->world;
    w.SetSolverMode(implicit_mode == 1 ? SolverMode::ImplicitEuler : SolverMode::Explicit);
    w.SetGravity(Vec3{static_cast<Real>(gravity3[0]), static_cast<Real>(gravity3[1]),
                      static_cast<Real>(gravity3[2])});
    w.SetConjugateGradientMaxIterations(max_iterations);
    w.SetConjugateGradientTolerance(static_cast<Real>(tolerance));
    w.SetSubstepCount(substeps);
}

// Adds one body through TetMeshGenerator + TetMeshPhysicsComponent.  Returns the
// global index of its first node, or -1.
__attribute__((visibility("default"))) int ref_add_body(void* h, const double* positions, int vertex_count,
                                                        const int* tets, int tet_count, double density,
                                                        double young, double poisson, double damping)
{
    Harness* hh = H(h);
    std::vector<Vec3> pos(static_cast<std::size_t>(vertex_count));
    for (int i = 0; i < vertex_count; ++i)
        pos[i] = Vec3{static_cast<Real>(positions[3 * i]), static_cast<Real>(positions[3 * i + 1]),
                      static_cast<Real>(positions[3 * i + 2])};
    GeneratedTetMesh mesh = TetMeshGenerator::Generate(pos.data(), vertex_count, tets, tet_count);
    if (mesh.positions.empty() || mesh.tetLocalNodeIndices.empty()) return -1;
    Material material;
    material.density = static_cast<Real>(density);
    material.youngModulus = static_cast<Real>(young);
    material.poissonRatio = static_cast<Real>(poisson);
    material.damping = static_cast<Real>(damping);
    auto component = TetMeshPhysicsComponent::CreateFromGeneratedTetMesh(hh->world, mesh, material);
    TetMeshPhysicsComponent* raw = component.get();
    ComponentHandle handle = hh->world.AddComponent(std::move(component));
    if (!handle.IsValid()) return -1;
    hh->bodies.push_back(raw);
    hh->bodyHandles.push_back(handle);
    return raw->GetGlobalNodeBeginIndex();
}

// The component handle of a body, for the reference's own C ABI (index, generation).
__attribute__((visibility("default"))) void ref_body_handle(void* h, int body, std::uint32_t* out2)
{
    const ComponentHandle c = H(h)->bodyHandles.at(static_cast<std::size_t>(body));
    out2[0] = c.index;
    out2[1] = c.generation;
}

__attribute__((visibility("default"))) int ref_body_tet_count(void* h, int body)
{
    return static_cast<int>(H(h)->bodies.at(static_cast<std::size_t>(body))->tets.size());
}

// TetMeshComponent::GetLocalCurrentPosition / SetLocalCurrentPosition of a body through the
// reference's own C ABI (PHYSIK_GetTetMeshLocalCurrentPosition, PhysiKAPI.cpp:1021-1053, needs
// the component handle, which this harness does not keep, so the component methods that
// those functions call are used directly).  Positions cross as double.
__attribute__((visibility("default"))) int ref_get_local_positions(void* h, int body, double* out)
{
    TetMeshPhysicsComponent* c = H(h)->bodies.at(static_cast<std::size_t>(body));
    const int count = c->GetNodeCount();
    for (int i = 0; i < count; ++i) {
        const Vec3& p = c->GetLocalCurrentPosition(i);
        out[3 * i] = p.x;
        out[3 * i + 1] = p.y;
        out[3 * i + 2] = p.z;
    }
    return count;
}

__attribute__((visibility("default"))) void ref_set_local_position(void* h, int body, int node, double x, double y,
                                                                   double z)
{
    H(h)->bodies.at(static_cast<std::size_t>(body))
        ->SetLocalCurrentPosition(node, Vec3{static_cast<Real>(x), static_cast<Real>(y), static_cast<Real>(z)});
}

// A component that hands SolverData to a C callback from UpdateSystem (what a custom C++
// component of the reference does), at the given execution priority; the callback emits
// through ref_solverdata_add_* (SolverData::AddNodeForce / AddNodeMass / AddStiffnessBlock).
namespace {
using RefContribution = void (*)(void* solverData, double dt, void* user);
class RefContributionComponent : public Component {
public:
    RefContributionComponent(int priority, RefContribution cb, void* user) : priority_(priority), cb_(cb), user_(user) {}
    ComponentExecutionPriority GetExecutionPriority() const override
    {
        return static_cast<ComponentExecutionPriority>(priority_);
    }
    void UpdateSystem(World&, SolverData& solverData, Real dt) override { cb_(&solverData, dt, user_); }

private:
    int priority_;
    RefContribution cb_;
    void* user_;
};
}  // namespace

__attribute__((visibility("default"))) int ref_add_contribution(void* h, int priority, RefContribution cb, void* user)
{
    return H(h)->world.AddComponent(std::make_unique<RefContributionComponent>(priority, cb, user)).IsValid() ? 1 : 0;
}
__attribute__((visibility("default"))) void ref_solverdata_add_force(void* sd, int node, double x, double y, double z)
{
    static_cast<SolverData*>(sd)->AddNodeForce(node, Vec3{static_cast<Real>(x), static_cast<Real>(y), static_cast<Real>(z)});
}
__attribute__((visibility("default"))) void ref_solverdata_add_mass(void* sd, int node, double m)
{
    static_cast<SolverData*>(sd)->AddNodeMass(node, static_cast<Real>(m));
}
__attribute__((visibility("default"))) void ref_solverdata_add_block(void* sd, int a, int b, const double* block9)
{
    Vec3 c[3];
    for (int i = 0; i < 3; ++i)
        c[i] = Vec3{static_cast<Real>(block9[3 * i]), static_cast<Real>(block9[3 * i + 1]),
                    static_cast<Real>(block9[3 * i + 2])};
    static_cast<SolverData*>(sd)->AddStiffnessBlock(a, b, Mat3::FromColumns(c[0], c[1], c[2]));
}

// A ScriptComponent with its external callback (World::AddComponent,
// ScriptComponent::SetExternalLogicCallback), as PHYSIK_CreateScriptComponent and
// PHYSIK_SetScriptComponentCallback do.  Returns 1 on success.
__attribute__((visibility("default"))) int ref_add_script(void* h, ExternalLogicCallback callback, void* user)
{
    auto component = std::make_unique<ScriptComponent>();
    component->SetExternalLogicCallback(callback, user);
    return H(h)->world.AddComponent(std::move(component)).IsValid() ? 1 : 0;
}

// A collision sphere (CollisionSphereComponent::Create + SetConnectionSettings +
// World::AddComponent, as PHYSIK_CreateCollisionSphereComponent and
// PHYSIK_SetCollisionSphereConnectionSettings do).  Returns its index, or -1.
__attribute__((visibility("default"))) int ref_add_sphere(void* h, double x, double y, double z, double radius,
                                                          double stiffness, double damping)
{
    auto sphere = CollisionSphereComponent::Create(
        Vec3{static_cast<Real>(x), static_cast<Real>(y), static_cast<Real>(z)}, static_cast<Real>(radius));
    sphere->SetConnectionSettings(static_cast<Real>(stiffness), static_cast<Real>(damping));
    CollisionSphereComponent* raw = sphere.get();
    if (!H(h)->world.AddComponent(std::move(sphere)).IsValid()) return -1;
    H(h)->spheres.push_back(raw);
    return static_cast<int>(H(h)->spheres.size()) - 1;
}

// CollisionComponent::SetKinematicTarget with the sphere's transform moved to (x, y, z),
// as PHYSIK_SetCollisionComponentKinematicTarget does (PhysiKAPI.cpp:1407-1429).
__attribute__((visibility("default"))) void ref_sphere_target(void* h, int sphere, double x, double y, double z)
{
    CollisionSphereComponent* c = H(h)->spheres.at(static_cast<std::size_t>(sphere));
    Transform target = c->transform;
    target.position = Vec3{static_cast<Real>(x), static_cast<Real>(y), static_cast<Real>(z)};
    c->SetKinematicTarget(target);
}

// The reference world's handle, as the C ABI passes it to scripts.
__attribute__((visibility("default"))) void* ref_world_handle(void* h) { return static_cast<WorldHandle>(&H(h)->world); }

// TetMeshPhysicsComponent::SetFemModel (FemModel: 0 linear, 1 corotated, 2 NeoHookean).
__attribute__((visibility("default"))) void ref_set_fem_model(void* h, int body, int model)
{
    H(h)->bodies.at(static_cast<std::size_t>(body))->SetFemModel(static_cast<FemModel>(model));
}

// Per-element Young's modulus through the C++ route (Tet::youngModulus +
// TetMeshPhysicsComponent::RebuildTetFemCache).
__attribute__((visibility("default"))) void ref_set_tet_young(void* h, int body, const double* young)
{
    TetMeshPhysicsComponent* c = H(h)->bodies.at(static_cast<std::size_t>(body));
    for (std::size_t t = 0; t < c->tets.size(); ++t) c->tets[t].youngModulus = static_cast<Real>(young[t]);
    c->RebuildTetFemCache();
}

__attribute__((visibility("default"))) void ref_set_fixed(void* h, const unsigned char* fixed, int count)
{
    World& w = H(h)->world;
    for (int i = 0; i < count; ++i)
        if (fixed[i]) w.SetNodeFixed(i, true);
}

__attribute__((visibility("default"))) int ref_node_count(void* h)
{
    return static_cast<int>(H(h)->world.GetNodes().size());
}

// Writes positions and velocities directly (World::SetNodePosition would zero the velocity).
__attribute__((visibility("default"))) void ref_set_state(void* h, const double* x, const double* v)
{
    World& w = H(h)->world;
    const int n = static_cast<int>(w.GetNodes().size());
    for (int i = 0; i < n; ++i) {
        if (x)
            w.GetNodePosition(i) = Vec3{static_cast<Real>(x[3 * i]), static_cast<Real>(x[3 * i + 1]),
                                        static_cast<Real>(x[3 * i + 2])};
        if (v)
            w.GetNodeVelocity(i) = Vec3{static_cast<Real>(v[3 * i]), static_cast<Real>(v[3 * i + 1]),
                                        static_cast<Real>(v[3 * i + 2])};
    }
}

__attribute__((visibility("default"))) void ref_get_state(void* h, double* x, double* v)
{
    World& w = H(h)->world;
    const int n = static_cast<int>(w.GetNodes().size());
    for (int i = 0; i < n; ++i) {
        const Vec3& p = w.GetNodePosition(i);
        const Vec3& q = w.GetNodeVelocity(i);
        if (x) { x[3 * i] = p.x; x[3 * i + 1] = p.y; x[3 * i + 2] = p.z; }
        if (v) { v[3 * i] = q.x; v[3 * i + 1] = q.y; v[3 * i + 2] = q.z; }
    }
}

// World::AddPointConnection (kept until the end of the next World::Step).
__attribute__((visibility("default"))) void ref_add_point_connection(void* h, const int* nodes4, const double* weights4,
                                                                     const double* target3, double stiffness,
                                                                     double damping)
{
    PointConnection c;
    c.node0 = nodes4[0];
    c.node1 = nodes4[1];
    c.node2 = nodes4[2];
    c.node3 = nodes4[3];
    c.barycentric = Vec4{static_cast<Real>(weights4[0]), static_cast<Real>(weights4[1]),
                         static_cast<Real>(weights4[2]), static_cast<Real>(weights4[3])};
    c.targetPosition = Vec3{static_cast<Real>(target3[0]), static_cast<Real>(target3[1]),
                            static_cast<Real>(target3[2])};
    c.stiffness = static_cast<Real>(stiffness);
    c.damping = static_cast<Real>(damping);
    H(h)->world.AddPointConnection(c);
}

__attribute__((visibility("default"))) int ref_point_connection_count(void* h)
{
    return H(h)->world.GetTransientConnectionCount();
}

// World::Step.  Returns 0, or -1 if the reference threw (e.g. a massless dynamic node).
__attribute__((visibility("default"))) int ref_step(void* h, double dt)
{
    try {
        H(h)->world.Step(static_cast<Real>(dt));
    } catch (const std::exception& e) {
        H(h)->error = e.what();
        return -1;
    }
    return 0;
}

__attribute__((visibility("default"))) void ref_cg_stats(void* h, int* iterations, double* residual, int* converged)
{
    World& w = H(h)->world;
    if (iterations) *iterations = w.GetLastConjugateGradientIterations();
    if (residual) *residual = w.GetLastConjugateGradientResidualNorm();
    if (converged) *converged = w.DidLastConjugateGradientSolveConverge() ? 1 : 0;
}

// Runs one substep's assembly and solve (World::PrecomputeSolve followed by
// SolverData::SolveImplicitLinearSystem) without integrating, keeping the
// SolverData for ref_dump_copy.  Returns the solve result (1/0) or -1 on throw.
__attribute__((visibility("default"))) int ref_dump_begin(void* h, double dt, int* dyn, int* nnz)
{
    Harness* hh = H(h);
    hh->dump = std::make_unique<SolverData>();
    int solved = 0;
    try {
        hh->world.PrecomputeSolve(*hh->dump, static_cast<Real>(dt));
        solved = hh->dump->SolveImplicitLinearSystem(hh->world.conjugateGradientSettings) ? 1 : 0;
    } catch (const std::exception& e) {
        hh->error = e.what();
        return -1;
    }
    if (dyn) *dyn = hh->dump->dynamicBlockCount;
    if (nnz) *nnz = static_cast<int>(hh->dump->matrix.colIndex.size());
    return solved;
}

__attribute__((visibility("default"))) void ref_dump_copy(void* h, int* row_start, int* col, double* values,
                                                          double* rhs, double* minv, double* dv,
                                                          int* node_to_dyn, double* mass, double* force)
{
    SolverData& s = *H(h)->dump;
    const SparseBlockMatrix& m = s.matrix;
    if (row_start) std::copy(m.rowStart.begin(), m.rowStart.end(), row_start);
    if (col) std::copy(m.colIndex.begin(), m.colIndex.end(), col);
    if (values)
        for (std::size_t k = 0; k < m.values.size(); ++k)
            for (int c = 0; c < 3; ++c) {
                values[9 * k + 3 * c + 0] = m.values[k].columns[c].x;
                values[9 * k + 3 * c + 1] = m.values[k].columns[c].y;
                values[9 * k + 3 * c + 2] = m.values[k].columns[c].z;
            }
    if (rhs)
        for (std::size_t i = 0; i < s.rhs.size(); ++i) {
            rhs[3 * i] = s.rhs[i].x; rhs[3 * i + 1] = s.rhs[i].y; rhs[3 * i + 2] = s.rhs[i].z;
        }
    if (minv)
        for (std::size_t k = 0; k < s.inversePreconditioner.size(); ++k)
            for (int c = 0; c < 3; ++c) {
                minv[9 * k + 3 * c + 0] = s.inversePreconditioner[k].columns[c].x;
                minv[9 * k + 3 * c + 1] = s.inversePreconditioner[k].columns[c].y;
                minv[9 * k + 3 * c + 2] = s.inversePreconditioner[k].columns[c].z;
            }
    if (dv)
        for (std::size_t i = 0; i < s.deltaVelocity.size(); ++i) {
            dv[3 * i] = s.deltaVelocity[i].x; dv[3 * i + 1] = s.deltaVelocity[i].y;
            dv[3 * i + 2] = s.deltaVelocity[i].z;
        }
    if (node_to_dyn) std::copy(s.nodeToDynamicBlock.begin(), s.nodeToDynamicBlock.end(), node_to_dyn);
    if (mass) std::copy(s.assembledMasses.begin(), s.assembledMasses.end(), mass);
    if (force)
        for (std::size_t i = 0; i < s.assembledForces.size(); ++i) {
            force[3 * i] = s.assembledForces[i].x; force[3 * i + 1] = s.assembledForces[i].y;
            force[3 * i + 2] = s.assembledForces[i].z;
        }
}

__attribute__((visibility("default"))) void ref_dump_cg(void* h, int* iterations, double* residual, int* converged)
{
    const LinearSolveResult& r = H(h)->dump->GetLastLinearSolveResult();
    if (iterations) *iterations = r.iterations;
    if (residual) *residual = r.residualNorm;
    if (converged) *converged = r.converged ? 1 : 0;
}

// SparseBlockMatrix::BuildPattern + AddBlock + Multiply on caller data (KAT parity).
__attribute__((visibility("default"))) int ref_bsr_pattern(int n, const int* rows, const int* cols, int count,
                                                           int* row_start, int* col, int cap)
{
    SparseBlockMatrix m;
    std::vector<std::pair<int, int>> coords(static_cast<std::size_t>(count));
    for (int i = 0; i < count; ++i) coords[i] = {rows[i], cols[i]};
    m.BuildPattern(n, coords);
    const int nnz = static_cast<int>(m.colIndex.size());
    if (row_start) std::copy(m.rowStart.begin(), m.rowStart.end(), row_start);
    if (col && nnz <= cap) std::copy(m.colIndex.begin(), m.colIndex.end(), col);
    return nnz;
}

// SparseBlockMatrix::Multiply(vector<Vec3>) on a caller BSR (upper storage, column-major blocks).
__attribute__((visibility("default"))) void ref_bsr_multiply(int n, const int* row_start, const int* col,
                                                             const double* values, const double* x, double* y)
{
    SparseBlockMatrix m;
    m.blockCount = n;
    m.rowStart.assign(row_start, row_start + n + 1);
    const int nnz = row_start[n];
    m.colIndex.assign(col, col + nnz);
    m.values.resize(static_cast<std::size_t>(nnz));
    for (int k = 0; k < nnz; ++k)
        for (int c = 0; c < 3; ++c)
            m.values[k].columns[c] = Vec3{static_cast<Real>(values[9 * k + 3 * c]),
                                          static_cast<Real>(values[9 * k + 3 * c + 1]),
                                          static_cast<Real>(values[9 * k + 3 * c + 2])};
    std::vector<Vec3> in(static_cast<std::size_t>(n)), out;
    for (int i = 0; i < n; ++i)
        in[i] = Vec3{static_cast<Real>(x[3 * i]), static_cast<Real>(x[3 * i + 1]), static_cast<Real>(x[3 * i + 2])};
    m.Multiply(in, out);
    for (std::size_t i = 0; i < out.size(); ++i) {
        y[3 * i] = out[i].x; y[3 * i + 1] = out[i].y; y[3 * i + 2] = out[i].z;
    }
}

// SolvePreconditionedConjugateGradient on a caller BSR (upper storage, column-major blocks).
__attribute__((visibility("default"))) int ref_pcg(int n, const int* row_start, const int* col,
                                                   const double* values, const double* b, const double* minv,
                                                   int max_iterations, double tolerance, double* x,
                                                   int* iterations, double* residual, int* converged)
{
    SparseBlockMatrix m;
    m.blockCount = n;
    m.rowStart.assign(row_start, row_start + n + 1);
    const int nnz = row_start[n];
    m.colIndex.assign(col, col + nnz);
    m.values.resize(static_cast<std::size_t>(nnz));
    for (int k = 0; k < nnz; ++k)
        for (int c = 0; c < 3; ++c)
            m.values[k].columns[c] = Vec3{static_cast<Real>(values[9 * k + 3 * c]),
                                          static_cast<Real>(values[9 * k + 3 * c + 1]),
                                          static_cast<Real>(values[9 * k + 3 * c + 2])};
    std::vector<Vec3> rhs(static_cast<std::size_t>(n)), sol, r, d, q;
    for (int i = 0; i < n; ++i)
        rhs[i] = Vec3{static_cast<Real>(b[3 * i]), static_cast<Real>(b[3 * i + 1]), static_cast<Real>(b[3 * i + 2])};
    std::vector<Mat3> pre(static_cast<std::size_t>(n));
    for (int k = 0; k < n; ++k)
        for (int c = 0; c < 3; ++c)
            pre[k].columns[c] = Vec3{static_cast<Real>(minv[9 * k + 3 * c]), static_cast<Real>(minv[9 * k + 3 * c + 1]),
                                     static_cast<Real>(minv[9 * k + 3 * c + 2])};
    ConjugateGradientResult res =
        SolvePreconditionedConjugateGradient(sol, m, rhs, max_iterations, static_cast<Real>(tolerance), pre, r, d, q);
    for (std::size_t i = 0; i < sol.size(); ++i) {
        x[3 * i] = sol[i].x; x[3 * i + 1] = sol[i].y; x[3 * i + 2] = sol[i].z;
    }
    if (iterations) *iterations = res.iterations;
    if (residual) *residual = res.residualNorm;
    if (converged) *converged = res.converged ? 1 : 0;
    return static_cast<int>(sol.size());
}
}
