// TetMeshGenerator::Generate -- the reference's mesh preparation
// (src/Geometry/TetMeshGenerator.cpp:153-282): weld nodes that lie within the weld
// tolerance (first-seen node wins, 3x3x3 neighbour cells of a uniform hash grid),
// drop tets with out-of-range, repeated or near-coplanar corners (6V)^2 <= 1e-24, and
// count boundary / internal / non-manifold faces.  The node order it produces fixes the
// world node order and therefore the BSR pattern, so it is reproduced exactly.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "physik_core.h"

namespace PhysiK {
namespace {

struct Cell {
    int x, y, z;
    bool operator==(const Cell& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct CellHash {
    std::size_t operator()(const Cell& c) const
    {
        std::size_t h = static_cast<std::size_t>(static_cast<unsigned>(c.x)) * 73856093u;
        h ^= static_cast<std::size_t>(static_cast<unsigned>(c.y)) * 19349663u;
        h ^= static_cast<std::size_t>(static_cast<unsigned>(c.z)) * 83492791u;
        return h;
    }
};

Cell CellOf(const Vec3& p, float size)
{
    return Cell{static_cast<int>(std::floor(p.x / size)), static_cast<int>(std::floor(p.y / size)),
                static_cast<int>(std::floor(p.z / size))};
}

struct Face {
    int a, b, c;
    bool operator==(const Face& o) const { return a == o.a && b == o.b && c == o.c; }
};
Face SortedFace(int a, int b, int c)
{
    if (b < a) std::swap(a, b);
    if (c < b) std::swap(b, c);
    if (b < a) std::swap(a, b);
    return Face{a, b, c};
}

}  // namespace

GeneratedTetMesh TetMeshGenerator::Generate(const Vec3* positions, int nodeCount, const int* tetLocalNodeIndices,
                                            int tetCount, const TetMeshBuildOptions& options)
{
    GeneratedTetMesh out;
    out.rawNodeCount = nodeCount > 0 ? nodeCount : 0;
    out.rawTetCount = tetCount > 0 ? tetCount : 0;
    out.weldTolerance = options.weldTolerance;
    if (positions == nullptr || nodeCount <= 0) return out;

    const float tol = options.weldTolerance > 0.0f ? options.weldTolerance : 0.0f;
    const float tol2 = tol * tol;
    const bool weld = options.weldCoincidentNodes && tol > 0.0f;
    std::vector<int> remap(static_cast<std::size_t>(nodeCount), -1);
    // Hash grid: per cell the first and last kept node, chained in insertion order
    // through `next` (no allocation per cell).
    std::unordered_map<Cell, std::pair<int, int>, CellHash> grid;
    std::vector<int> next;
    // A bit per hashed cell, set when a node is stored in the cell: a clear bit means the
    // cell is empty, so most of the 27 neighbour probes skip the map.
    constexpr std::size_t kOccBits = std::size_t(1) << 24;
    std::vector<std::uint64_t> occ(weld ? kOccBits / 64 : 0, 0);
    const CellHash hasher;
    auto occ_bit = [&](const Cell& c) { return hasher(c) & (kOccBits - 1); };
    if (weld) {
        grid.reserve(static_cast<std::size_t>(nodeCount));
        next.reserve(static_cast<std::size_t>(nodeCount));
    }
    out.positions.reserve(static_cast<std::size_t>(nodeCount));
    for (int i = 0; i < nodeCount; ++i) {
        const Vec3& p = positions[i];
        int found = -1;
        if (weld) {
            const Cell c = CellOf(p, tol);
            for (int dz = -1; dz <= 1 && found < 0; ++dz)
                for (int dy = -1; dy <= 1 && found < 0; ++dy)
                    for (int dx = -1; dx <= 1 && found < 0; ++dx) {
                        const Cell nc{c.x + dx, c.y + dy, c.z + dz};
                        const std::size_t bit = occ_bit(nc);
                        if (!(occ[bit >> 6] >> (bit & 63) & 1u)) continue;
                        auto it = grid.find(nc);
                        if (it == grid.end()) continue;
                        for (int cand = it->second.first; cand >= 0; cand = next[static_cast<std::size_t>(cand)])
                            if ((out.positions[static_cast<std::size_t>(cand)] - p).LengthSquared() <= tol2) {
                                found = cand;
                                break;
                            }
                    }
        }
        if (found >= 0) {
            remap[static_cast<std::size_t>(i)] = found;
            continue;
        }
        const int id = static_cast<int>(out.positions.size());
        out.positions.push_back(p);
        remap[static_cast<std::size_t>(i)] = id;
        if (weld) {
            next.push_back(-1);
            const Cell pc = CellOf(p, tol);
            const std::size_t bit = occ_bit(pc);
            occ[bit >> 6] |= std::uint64_t(1) << (bit & 63);
            auto ins = grid.emplace(pc, std::make_pair(id, id));
            if (!ins.second) {
                next[static_cast<std::size_t>(ins.first->second.second)] = id;
                ins.first->second.second = id;
            }
        }
    }
    out.weldedNodeCount = static_cast<int>(out.positions.size());
    out.weldedAwayNodeCount = out.rawNodeCount - out.weldedNodeCount;

    if (tetLocalNodeIndices != nullptr && tetCount > 0) {
        out.tetLocalNodeIndices.reserve(static_cast<std::size_t>(tetCount) * 4u);
        for (int t = 0; t < tetCount; ++t) {
            const int* raw = tetLocalNodeIndices + 4 * t;
            bool inRange = true;
            for (int k = 0; k < 4; ++k) inRange = inRange && raw[k] >= 0 && raw[k] < nodeCount;
            if (!inRange) {
                ++out.removedDegenerateTetCount;
                continue;
            }
            const int a = remap[raw[0]], b = remap[raw[1]], c = remap[raw[2]], d = remap[raw[3]];
            if (options.removeDegenerateTets) {
                const bool dup = a == b || a == c || a == d || b == c || b == d || c == d;
                bool flat = false;
                if (!dup) {
                    const Vec3 ab = out.positions[b] - out.positions[a];
                    const Vec3 ac = out.positions[c] - out.positions[a];
                    const Vec3 ad = out.positions[d] - out.positions[a];
                    const float six = Dot(Cross(ab, ac), ad);
                    flat = six * six <= 1.0e-24f;
                }
                if (dup || flat) {
                    ++out.removedDegenerateTetCount;
                    continue;
                }
            }
            out.tetLocalNodeIndices.push_back(a);
            out.tetLocalNodeIndices.push_back(b);
            out.tetLocalNodeIndices.push_back(c);
            out.tetLocalNodeIndices.push_back(d);
        }
    }

    // Faces by how many kept tets share them: every tet's four sorted faces, sorted, then
    // counted run by run (the same counts as a map from face to tets).
    const int kept = static_cast<int>(out.tetLocalNodeIndices.size() / 4u);
    std::vector<Face> faces;
    faces.reserve(4 * static_cast<std::size_t>(kept));
    for (int t = 0; t < kept; ++t) {
        const int* n = &out.tetLocalNodeIndices[static_cast<std::size_t>(4 * t)];
        faces.push_back(SortedFace(n[0], n[1], n[2]));
        faces.push_back(SortedFace(n[0], n[3], n[1]));
        faces.push_back(SortedFace(n[0], n[2], n[3]));
        faces.push_back(SortedFace(n[1], n[3], n[2]));
    }
    const int nn = static_cast<int>(out.positions.size());
    if (nn < (1 << 21)) {
        // 21 bits per node index: one 64-bit key per face.
        std::vector<std::uint64_t> keys(faces.size());
        for (std::size_t i = 0; i < faces.size(); ++i)
            keys[i] = (static_cast<std::uint64_t>(faces[i].a) << 42) | (static_cast<std::uint64_t>(faces[i].b) << 21) |
                      static_cast<std::uint64_t>(faces[i].c);
        std::sort(keys.begin(), keys.end());
        for (std::size_t i = 0; i < keys.size();) {
            std::size_t j = i + 1;
            while (j < keys.size() && keys[j] == keys[i]) ++j;
            const std::size_t k = j - i;
            if (k == 1) ++out.topologyDiagnostics.boundaryFaceCount;
            else if (k == 2) ++out.topologyDiagnostics.internalFaceCount;
            else ++out.topologyDiagnostics.nonManifoldFaceCount;
            i = j;
        }
    } else {
        std::sort(faces.begin(), faces.end(), [](const Face& x, const Face& y) {
            return x.a < y.a || (x.a == y.a && (x.b < y.b || (x.b == y.b && x.c < y.c)));
        });
        for (std::size_t i = 0; i < faces.size();) {
            std::size_t j = i + 1;
            while (j < faces.size() && faces[j] == faces[i]) ++j;
            const std::size_t k = j - i;
            if (k == 1) ++out.topologyDiagnostics.boundaryFaceCount;
            else if (k == 2) ++out.topologyDiagnostics.internalFaceCount;
            else ++out.topologyDiagnostics.nonManifoldFaceCount;
            i = j;
        }
    }
    return out;
}

}  // namespace PhysiK
