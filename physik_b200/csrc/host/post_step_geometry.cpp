// Post-step geometry: surface extraction, surface visuals and embedded visual meshes.
//
//   SurfaceExtractionComponent   src/Components/SurfaceExtractionComponent.cpp:138-250
//   SurfaceVisualComponent       src/Components/SurfaceVisualComponent.cpp:26-254
//   VisualMeshComponent          src/Components/VisualMeshComponent.cpp:14-347
//
// The per-frame work of the visuals (copying node positions into render vertices, flat
// normals, barycentric skinning) runs on the device (pk_visual_update) whenever the
// positions it reads are there, and stays there until a getter asks for it.  The
// topology work (boundary faces, embedding, triangle filtering) follows topology events
// and runs on the host, in the reference's order, so the index buffers match it exactly.
#include <algorithm>
#include <cmath>
#include <functional>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../../include/pkcuda.h"
#include "physik_core.h"

namespace PhysiK {

namespace {

void CheckPk(int rc, const char* what)
{
    if (rc != PK_OK) throw std::runtime_error(std::string(what) + ": " + pk_last_error());
}

TetMeshComponent* HostMesh(World& world, ComponentHandle handle)
{
    return dynamic_cast<TetMeshComponent*>(world.GetComponent(handle));
}

// The host mesh's local current positions as of now (a physics body's copy is loaded
// from the device snapshot on first use).
void LoadLocalPositions(World& world, TetMeshComponent* mesh)
{
    if (auto* body = dynamic_cast<TetMeshPhysicsComponent*>(mesh)) world.RefreshLocalPositions(*body);
}

// Whether `mesh` emitted a topology event since `seen` (the listener's OnPhysicsEvent).
bool SeeTopologyEvents(const TetMeshComponent* mesh, std::uint64_t& seen)
{
    if (!mesh || mesh->topologyEvents == seen) return false;
    seen = mesh->topologyEvents;
    return true;
}

// A physics body whose nodes are world nodes begin..begin+count-1: its positions can be
// read on the device.
const TetMeshPhysicsComponent* DeviceBody(const TetMeshComponent* mesh)
{
    const auto* body = dynamic_cast<const TetMeshPhysicsComponent*>(mesh);
    if (!body || body->GetGlobalNodeBeginIndex() < 0 || body->GetGlobalNodeCount() != body->GetNodeCount())
        return nullptr;
    return body;
}

// ---- surface extraction (SurfaceExtractionComponent.cpp:14-134) ----
struct Face {
    int node0 = -1, node1 = -1, node2 = -1;
};

// The sorted node triple that identifies a face.
struct FaceKey {
    int node0 = -1, node1 = -1, node2 = -1;
    bool operator==(const FaceKey& o) const { return node0 == o.node0 && node1 == o.node1 && node2 == o.node2; }
};

// The reference's face hash.  The boundary faces come out in the order the hash map
// holds them, so the same hash and the same container (libstdc++'s unordered_map, fed
// the faces in the same order) give the same triangle order.
struct FaceKeyHash {
    std::size_t operator()(const FaceKey& k) const
    {
        const std::size_t h0 = std::hash<int>{}(k.node0), h1 = std::hash<int>{}(k.node1), h2 = std::hash<int>{}(k.node2);
        return h0 ^ (h1 << 1u) ^ (h2 << 2u);
    }
};

struct FaceEntry {
    Face orientedFace;
    int count = 0;
};

FaceKey SortedKey(const Face& f)
{
    int a = f.node0, b = f.node1, c = f.node2;
    if (b < a) std::swap(a, b);
    if (c < b) std::swap(b, c);
    if (b < a) std::swap(a, b);
    return FaceKey{a, b, c};
}

// Face `faceIndex` of a tet with corners n[0..3] and the corner opposite it.
void TetFace(const int n[4], int faceIndex, Face& face, int& opposite)
{
    switch (faceIndex) {
    case 0: face = Face{n[0], n[1], n[2]}; opposite = n[3]; break;
    case 1: face = Face{n[0], n[3], n[1]}; opposite = n[2]; break;
    case 2: face = Face{n[0], n[2], n[3]}; opposite = n[1]; break;
    default: face = Face{n[1], n[3], n[2]}; opposite = n[0]; break;
    }
}

// The face wound so that its normal points away from the opposite corner, at the local
// current positions; unchanged when a node is out of range or the face is degenerate
// (|normal|^2 <= 1e-12).
Face OrientOutward(const TetMeshComponent& mesh, Face face, int opposite)
{
    const int count = mesh.GetNodeCount();
    if (face.node0 < 0 || face.node0 >= count || face.node1 < 0 || face.node1 >= count || face.node2 < 0 ||
        face.node2 >= count || opposite < 0 || opposite >= count)
        return face;
    const Vec3& p0 = mesh.GetLocalCurrentPosition(face.node0);
    const Vec3& p1 = mesh.GetLocalCurrentPosition(face.node1);
    const Vec3& p2 = mesh.GetLocalCurrentPosition(face.node2);
    const Vec3& po = mesh.GetLocalCurrentPosition(opposite);
    const Vec3 normal = Cross(p1 - p0, p2 - p0);
    if (normal.LengthSquared() <= 0.000000000001f) return face;
    if (Dot(normal, po - p0) > 0.0f) std::swap(face.node1, face.node2);
    return face;
}

Vec3 NormalizeOrFallback(const Vec3& v)
{
    const float length = v.Length();
    if (length <= 0.000001f) return Vec3{0.0f, 1.0f, 0.0f};
    return v / length;
}

}  // namespace

// ------------------------------------------------------------------ DeviceVisual
void DeviceVisual::Release()
{
    if (visual) pk_visual_destroy(visual);
    visual = nullptr;
    system = nullptr;
    pending = false;
}

void DeviceVisual::Fetch(float* vertices, float* normals)
{
    if (!pending) return;
    CheckPk(pk_visual_read(visual, system, vertices, normals), "pk_visual_read");
    pending = false;
}

// ------------------------------------------------------------------ SurfaceExtractionComponent
SurfaceExtractionComponent::SurfaceExtractionComponent(ComponentHandle host, std::uint64_t seen)
    : hostTetMeshHandle(host), topologyEventsSeen(seen)
{
}

void SurfaceExtractionComponent::RebuildSurface(World& world)
{
    surfaceTriangleIndices.clear();
    TetMeshComponent* mesh = HostMesh(world, hostTetMeshHandle);
    if (!mesh) return;
    LoadLocalPositions(world, mesh);
    surfaceTriangleIndices.reserve(static_cast<std::size_t>(mesh->GetTetCount()) * 12u);
    std::unordered_map<FaceKey, FaceEntry, FaceKeyHash> faces;
    for (int t = 0; t < mesh->GetTetCount(); ++t) {
        if (!mesh->IsTetActive(t)) continue;
        const int n[4] = {mesh->GetTetNodeIndex(t, 0), mesh->GetTetNodeIndex(t, 1), mesh->GetTetNodeIndex(t, 2),
                          mesh->GetTetNodeIndex(t, 3)};
        for (int f = 0; f < 4; ++f) {
            Face face;
            int opposite = -1;
            TetFace(n, f, face, opposite);
            const Face oriented = OrientOutward(*mesh, face, opposite);
            FaceEntry& entry = faces[SortedKey(oriented)];
            if (entry.count == 0) entry.orientedFace = oriented;
            ++entry.count;
        }
    }
    for (const auto& item : faces) {
        if (item.second.count != 1) continue;
        surfaceTriangleIndices.push_back(item.second.orientedFace.node0);
        surfaceTriangleIndices.push_back(item.second.orientedFace.node1);
        surfaceTriangleIndices.push_back(item.second.orientedFace.node2);
    }
}

void SurfaceExtractionComponent::PostUpdate(World& world, float)
{
    if (SeeTopologyEvents(HostMesh(world, hostTetMeshHandle), topologyEventsSeen)) surfaceDirty = true;
    if (!surfaceDirty) return;
    RebuildSurface(world);
    surfaceDirty = false;
}

// ------------------------------------------------------------------ SurfaceVisualComponent
SurfaceVisualComponent::SurfaceVisualComponent(ComponentHandle extraction, std::uint64_t seen)
    : surfaceExtractionHandle(extraction), topologyEventsSeen(seen)
{
}

void SurfaceVisualComponent::FetchDevice() const
{
    if (!device.pending) return;
    const std::size_t n = visualVertices.size();
    std::vector<float> v(3 * n), nr(3 * n);
    device.Fetch(v.data(), nr.data());
    for (std::size_t i = 0; i < n; ++i) {
        visualVertices[i] = Vec3{v[3 * i], v[3 * i + 1], v[3 * i + 2]};
        visualNormals[i] = Vec3{nr[3 * i], nr[3 * i + 1], nr[3 * i + 2]};
    }
}

const std::vector<Vec3>& SurfaceVisualComponent::GetVisualVertices() const
{
    FetchDevice();
    return visualVertices;
}

const std::vector<Vec3>& SurfaceVisualComponent::GetVisualNormals() const
{
    FetchDevice();
    return visualNormals;
}

void SurfaceVisualComponent::ReleaseDeviceResources()
{
    FetchDevice();
    device.Release();
}

void SurfaceVisualComponent::RebuildVisualSurfaceTopology(World& world)
{
    device.Release();
    visualVertices.clear();
    visualTriangleIndices.clear();
    visualNormals.clear();
    visualVertexSourceNodeIndices.clear();
    const auto* extraction = dynamic_cast<const SurfaceExtractionComponent*>(world.GetComponent(surfaceExtractionHandle));
    if (!extraction) return;
    TetMeshComponent* mesh = HostMesh(world, extraction->GetHostTetMeshHandle());
    if (!mesh) return;
    const std::vector<int>& raw = extraction->GetSurfaceTriangleIndices();
    if (raw.size() % 3u != 0u) return;
    LoadLocalPositions(world, mesh);
    const std::size_t triangles = raw.size() / 3u;
    visualVertices.reserve(3 * triangles);
    visualTriangleIndices.reserve(3 * triangles);
    visualNormals.reserve(3 * triangles);
    visualVertexSourceNodeIndices.reserve(3 * triangles);
    const int count = mesh->GetNodeCount();
    for (std::size_t t = 0; t < triangles; ++t) {
        const int n0 = raw[3 * t], n1 = raw[3 * t + 1], n2 = raw[3 * t + 2];
        if (n0 < 0 || n0 >= count || n1 < 0 || n1 >= count || n2 < 0 || n2 >= count) continue;
        const int base = static_cast<int>(visualVertices.size());
        for (int n : {n0, n1, n2}) {
            visualVertices.push_back(mesh->GetLocalCurrentPosition(n));
            visualVertexSourceNodeIndices.push_back(n);
            visualNormals.push_back(Vec3{0.0f, 1.0f, 0.0f});
        }
        visualTriangleIndices.push_back(base);
        visualTriangleIndices.push_back(base + 1);
        visualTriangleIndices.push_back(base + 2);
    }
    UpdateVisualSurfaceGeometry(world);
}

void SurfaceVisualComponent::UpdateVisualSurfaceGeometry(World& world)
{
    const auto* extraction = dynamic_cast<const SurfaceExtractionComponent*>(world.GetComponent(surfaceExtractionHandle));
    if (!extraction) return;
    TetMeshComponent* mesh = HostMesh(world, extraction->GetHostTetMeshHandle());
    if (!mesh) return;
    if (visualVertices.size() != visualVertexSourceNodeIndices.size() || visualNormals.size() != visualVertices.size() ||
        visualTriangleIndices.size() % 3u != 0u) {
        FetchDevice();
        topologyDirty = true;
        return;
    }
    const int count = mesh->GetNodeCount();
    // Device route: the vertices are the body's frame-end snapshot at the source nodes.
    // The rebuild lays out three vertices per triangle in triangle order (index buffer
    // 0, 1, 2, ...), which is the device visual's layout.
    const TetMeshPhysicsComponent* body = DeviceBody(mesh);
    pk_system* sys = body && !visualVertices.empty() ? world.GeometrySystem(body, true) : nullptr;
    if (sys && (!device.visual || device.system != sys || deviceNodeCount != count)) {
        const bool inRange = std::all_of(visualVertexSourceNodeIndices.begin(), visualVertexSourceNodeIndices.end(),
                                         [count](int n) { return n >= 0 && n < count; });
        FetchDevice();
        device.Release();
        if (inRange) {
            std::vector<int> nodes(visualVertexSourceNodeIndices.size());
            for (std::size_t i = 0; i < nodes.size(); ++i)
                nodes[i] = body->GetGlobalNodeIndex(visualVertexSourceNodeIndices[i]);
            CheckPk(pk_visual_create(sys, 0, static_cast<int>(nodes.size() / 3), nodes.data(), nullptr, nullptr,
                                     nullptr, &device.visual),
                    "pk_visual_create");
            device.system = sys;
            deviceNodeCount = count;
        } else {
            sys = nullptr;
        }
    }
    if (sys) {
        CheckPk(pk_visual_update(device.visual, sys, 1), "pk_visual_update");
        device.pending = true;
        lastOnDevice = true;
        return;
    }
    FetchDevice();
    lastOnDevice = false;
    LoadLocalPositions(world, mesh);
    for (std::size_t i = 0; i < visualVertices.size(); ++i) {
        const int source = visualVertexSourceNodeIndices[i];
        if (source < 0 || source >= count) {
            topologyDirty = true;
            return;
        }
        visualVertices[i] = mesh->GetLocalCurrentPosition(source);
    }
    const int nv = static_cast<int>(visualVertices.size());
    for (std::size_t i = 0; i < visualTriangleIndices.size(); i += 3u) {
        const int ia = visualTriangleIndices[i], ib = visualTriangleIndices[i + 1], ic = visualTriangleIndices[i + 2];
        if (ia < 0 || ib < 0 || ic < 0 || ia >= nv || ib >= nv || ic >= nv) {
            topologyDirty = true;
            return;
        }
        const Vec3& p0 = visualVertices[static_cast<std::size_t>(ia)];
        const Vec3& p1 = visualVertices[static_cast<std::size_t>(ib)];
        const Vec3& p2 = visualVertices[static_cast<std::size_t>(ic)];
        const Vec3 normal = NormalizeOrFallback(Cross(p1 - p0, p2 - p0));
        visualNormals[static_cast<std::size_t>(ia)] = normal;
        visualNormals[static_cast<std::size_t>(ib)] = normal;
        visualNormals[static_cast<std::size_t>(ic)] = normal;
    }
}

void SurfaceVisualComponent::PostUpdate(World& world, float)
{
    const auto* extraction = dynamic_cast<const SurfaceExtractionComponent*>(world.GetComponent(surfaceExtractionHandle));
    if (extraction && SeeTopologyEvents(HostMesh(world, extraction->GetHostTetMeshHandle()), topologyEventsSeen))
        topologyDirty = true;
    if (topologyDirty) {
        RebuildVisualSurfaceTopology(world);
        topologyDirty = false;
    }
    UpdateVisualSurfaceGeometry(world);
}

// ------------------------------------------------------------------ VisualMeshComponent
bool ComputeTetBarycentric(const Vec3& p, const Vec3& a, const Vec3& b, const Vec3& c, const Vec3& d, Vec4& out)
{
    const Vec3 ab = b - a, ac = c - a, ad = d - a, ap = p - a;
    const float det = Dot(ab, Cross(ac, ad));
    if (std::abs(det) <= 0.00000001f) {
        out = Vec4{};
        return false;
    }
    const float inv = 1.0f / det;
    const float wb = Dot(ap, Cross(ac, ad)) * inv;
    const float wc = Dot(ab, Cross(ap, ad)) * inv;
    const float wd = Dot(ab, Cross(ac, ap)) * inv;
    out = Vec4{1.0f - wb - wc - wd, wb, wc, wd};
    return true;
}

VisualMeshComponent::VisualMeshComponent(ComponentHandle host, std::string name, std::uint64_t seen)
    : hostTetMeshHandle(host), debugEntityName(std::move(name)), topologyEventsSeen(seen)
{
}

void VisualMeshComponent::FetchDevice() const
{
    if (!device.pending) return;
    const std::size_t n = deformedVisualVertices.size();
    std::vector<float> v(3 * n);
    device.Fetch(v.data(), nullptr);
    for (std::size_t i = 0; i < n; ++i) deformedVisualVertices[i] = Vec3{v[3 * i], v[3 * i + 1], v[3 * i + 2]};
}

const std::vector<Vec3>& VisualMeshComponent::GetDeformedVertices() const
{
    FetchDevice();
    return deformedVisualVertices;
}

void VisualMeshComponent::ReleaseDeviceResources()
{
    FetchDevice();
    device.Release();
}

void VisualMeshComponent::SetVisualMesh(const Vec3* vertices, int vertexCount, const int* indices, int indexCount)
{
    device.Release();
    ++embeddingVersion;
    restVisualVertices.clear();
    deformedVisualVertices.clear();
    triangleIndices.clear();
    filteredTriangleIndices.clear();
    embeddedVertices.clear();
    triangleValid.clear();
    if (vertices && vertexCount > 0) {
        restVisualVertices.assign(vertices, vertices + vertexCount);
        deformedVisualVertices = restVisualVertices;
        embeddedVertices.resize(static_cast<std::size_t>(vertexCount));
    }
    if (indices && indexCount > 0) {
        triangleIndices.assign(indices, indices + indexCount);
        filteredTriangleIndices = triangleIndices;
        triangleValid.assign(static_cast<std::size_t>(indexCount / 3), true);
    }
}

// Every vertex scans the active tets in index order for the first that holds it (the
// vertices are independent, so they are split over host threads).
void VisualMeshComponent::BuildEmbedding(World& world)
{
    FetchDevice();
    device.Release();
    ++embeddingVersion;
    embeddedVertices.assign(restVisualVertices.size(), EmbeddedVertex{});
    const TetMeshComponent* mesh = HostMesh(world, hostTetMeshHandle);
    if (!mesh) return;
    constexpr float insideEpsilon = -0.0001f;
    const int nodeCount = mesh->GetNodeCount();
    auto embed = [&](std::size_t lo, std::size_t hi) {
        for (std::size_t v = lo; v < hi; ++v) {
            EmbeddedVertex& e = embeddedVertices[v];
            for (int t = 0; t < mesh->GetTetCount(); ++t) {
                if (!mesh->IsTetActive(t)) continue;
                const int n[4] = {mesh->GetTetNodeIndex(t, 0), mesh->GetTetNodeIndex(t, 1),
                                  mesh->GetTetNodeIndex(t, 2), mesh->GetTetNodeIndex(t, 3)};
                if (std::any_of(n, n + 4, [nodeCount](int k) { return k < 0 || k >= nodeCount; })) continue;
                Vec4 w;
                if (!ComputeTetBarycentric(restVisualVertices[v], mesh->GetLocalRestPosition(n[0]),
                                           mesh->GetLocalRestPosition(n[1]), mesh->GetLocalRestPosition(n[2]),
                                           mesh->GetLocalRestPosition(n[3]), w))
                    continue;
                if (w.x >= insideEpsilon && w.y >= insideEpsilon && w.z >= insideEpsilon && w.w >= insideEpsilon) {
                    e.tetIndex = t;
                    e.barycentric = w;
                    e.valid = true;
                    break;
                }
            }
        }
    };
    const std::size_t count = embeddedVertices.size();
    const std::size_t work = count * static_cast<std::size_t>(std::max(1, mesh->GetTetCount()));
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const std::size_t threads = work < (1u << 20) ? 1 : std::min<std::size_t>(hw, count);
    if (threads <= 1) {
        embed(0, count);
    } else {
        const std::size_t chunk = (count + threads - 1) / threads;
        std::vector<std::thread> pool;
        std::size_t next = chunk;  // the first chunk not handed to a thread
        try {
            for (; next < count; next += chunk) pool.emplace_back(embed, next, std::min(count, next + chunk));
        } catch (...) {
        }
        embed(0, std::min(count, chunk));
        if (next < count) embed(next, count);  // the chunks whose thread could not start
        for (std::thread& th : pool) th.join();
    }
    UpdateTriangleValidity(world);
}

void VisualMeshComponent::UpdateTriangleValidity(World& world)
{
    filteredTriangleIndices.clear();
    const std::size_t triangles = triangleIndices.size() / 3u;
    triangleValid.assign(triangles, false);
    if (triangles == 0u) return;
    const TetMeshComponent* mesh = HostMesh(world, hostTetMeshHandle);
    if (!mesh) return;
    const int nv = static_cast<int>(embeddedVertices.size());
    for (std::size_t t = 0; t < triangles; ++t) {
        const int v[3] = {triangleIndices[3 * t], triangleIndices[3 * t + 1], triangleIndices[3 * t + 2]};
        bool valid = true;
        for (int k : v) {
            if (k < 0 || k >= nv) {
                valid = false;
                break;
            }
            const EmbeddedVertex& e = embeddedVertices[static_cast<std::size_t>(k)];
            if (!e.valid || e.tetIndex < 0 || e.tetIndex >= mesh->GetTetCount() || !mesh->IsTetActive(e.tetIndex)) {
                valid = false;
                break;
            }
        }
        triangleValid[t] = valid;
        if (valid) filteredTriangleIndices.insert(filteredTriangleIndices.end(), v, v + 3);
    }
}

// A vertex is skinned when its tet exists, is active and has all its nodes in range.
std::vector<unsigned char> VisualMeshComponent::LiveFlags(const TetMeshComponent& mesh) const
{
    std::vector<unsigned char> live(embeddedVertices.size(), 0);
    const int nodeCount = mesh.GetNodeCount();
    for (std::size_t v = 0; v < embeddedVertices.size(); ++v) {
        const EmbeddedVertex& e = embeddedVertices[v];
        if (!e.valid || e.tetIndex < 0 || e.tetIndex >= mesh.GetTetCount() || !mesh.IsTetActive(e.tetIndex)) continue;
        bool ok = true;
        for (int k = 0; k < 4; ++k) {
            const int n = mesh.GetTetNodeIndex(e.tetIndex, k);
            ok = ok && n >= 0 && n < nodeCount;
        }
        live[v] = ok ? 1 : 0;
    }
    return live;
}

void VisualMeshComponent::UpdateDeformedVertices(World& world)
{
    if (deformedVisualVertices.size() != restVisualVertices.size()) {
        device.Release();
        deformedVisualVertices = restVisualVertices;
    }
    if (embeddedVertices.size() != restVisualVertices.size()) return;
    TetMeshComponent* mesh = HostMesh(world, hostTetMeshHandle);
    if (!mesh) return;
    // Device route: every vertex reads world positions of its tet's nodes (the body's
    // nodes are all world nodes), the vertices outside active tets keep their value.
    const TetMeshPhysicsComponent* body = DeviceBody(mesh);
    pk_system* sys = body && !restVisualVertices.empty() ? world.GeometrySystem(nullptr, false) : nullptr;
    if (sys) {
        if (!device.visual || device.system != sys || deviceEmbedding != embeddingVersion) {
            FetchDevice();
            device.Release();
            const std::size_t n = embeddedVertices.size();
            const int nodeCount = mesh->GetNodeCount();
            const int anyNode = body->GetGlobalNodeBeginIndex();
            std::vector<int> nodes(4 * n, anyNode);
            std::vector<float> weights(4 * n, 0.0f), initial(3 * n);
            for (std::size_t v = 0; v < n; ++v) {
                const EmbeddedVertex& e = embeddedVertices[v];
                initial[3 * v] = deformedVisualVertices[v].x;
                initial[3 * v + 1] = deformedVisualVertices[v].y;
                initial[3 * v + 2] = deformedVisualVertices[v].z;
                if (!e.valid || e.tetIndex < 0 || e.tetIndex >= mesh->GetTetCount()) continue;
                int local[4];
                bool ok = true;
                for (int k = 0; k < 4; ++k) {
                    local[k] = mesh->GetTetNodeIndex(e.tetIndex, k);
                    ok = ok && local[k] >= 0 && local[k] < nodeCount;
                }
                if (!ok) continue;
                const float w[4] = {e.barycentric.x, e.barycentric.y, e.barycentric.z, e.barycentric.w};
                for (int k = 0; k < 4; ++k) {
                    nodes[4 * v + k] = body->GetGlobalNodeIndex(local[k]);
                    weights[4 * v + k] = w[k];
                }
            }
            const std::vector<unsigned char> live = LiveFlags(*mesh);
            CheckPk(pk_visual_create(sys, 1, static_cast<int>(n), nodes.data(), weights.data(), initial.data(),
                                     live.data(), &device.visual),
                    "pk_visual_create");
            device.system = sys;
            deviceEmbedding = embeddingVersion;
            deviceBodyVersion = body->version;
        } else if (deviceBodyVersion != body->version) {
            const std::vector<unsigned char> live = LiveFlags(*mesh);
            CheckPk(pk_visual_set_live(device.visual, sys, live.data()), "pk_visual_set_live");
            deviceBodyVersion = body->version;
        }
        CheckPk(pk_visual_update(device.visual, sys, 0), "pk_visual_update");
        device.pending = true;
        lastOnDevice = true;
        return;
    }
    FetchDevice();
    device.Release();
    lastOnDevice = false;
    const int nodeCount = mesh->GetNodeCount();
    for (std::size_t v = 0; v < embeddedVertices.size(); ++v) {
        const EmbeddedVertex& e = embeddedVertices[v];
        if (!e.valid || e.tetIndex < 0 || e.tetIndex >= mesh->GetTetCount()) continue;
        if (!mesh->IsTetActive(e.tetIndex)) continue;
        int local[4];
        bool ok = true;
        for (int k = 0; k < 4; ++k) {
            local[k] = mesh->GetTetNodeIndex(e.tetIndex, k);
            ok = ok && local[k] >= 0 && local[k] < nodeCount;
        }
        if (!ok) continue;
        Vec3 p[4];
        for (int k = 0; k < 4; ++k) {
            const int g = mesh->GetGlobalNodeIndex(local[k]);
            if (g >= 0) {
                p[k] = world.GetNodePosition(g);
            } else {
                LoadLocalPositions(world, mesh);
                p[k] = mesh->GetLocalCurrentPosition(local[k]);
            }
        }
        const Vec4& w = e.barycentric;
        deformedVisualVertices[v] = p[0] * w.x + p[1] * w.y + p[2] * w.z + p[3] * w.w;
    }
}

void VisualMeshComponent::PostUpdate(World& world, float)
{
    if (SeeTopologyEvents(HostMesh(world, hostTetMeshHandle), topologyEventsSeen)) topologyDirty = true;
    if (topologyDirty) {
        UpdateTriangleValidity(world);
        topologyDirty = false;
    }
    UpdateDeformedVertices(world);
}

}  // namespace PhysiK
