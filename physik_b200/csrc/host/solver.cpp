// SparseBlockMatrix, SolvePreconditionedConjugateGradient and LinearSolver on the GPU.
//
// SparseBlockMatrix keeps the reference's host-side data structure and its cold-path
// pattern operations (src/Math/SparseBlockMatrix.cpp:83-144, 270-288: canonical
// coordinates, per-row sorted unique columns, (row << 32 | col) lookup keys), while the
// product runs in the libpkcuda SpMV kernel.  The free PCG function and the
// CurrentLinearSolver seam run the cooperative PCG kernel.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/pkcuda.h"
#include "physik_core.h"

namespace PhysiK {
namespace {

int g_solver_device = 0;

void ThrowOnError(int rc, const char* what)
{
    if (rc != PK_OK) throw std::runtime_error(std::string(what) + ": " + pk_last_error());
}

void PackValues(const std::vector<Mat3>& values, std::vector<double>& out)
{
    out.resize(values.size() * 9);
    for (std::size_t k = 0; k < values.size(); ++k)
        for (int c = 0; c < 3; ++c) {
            out[9 * k + 3 * c + 0] = values[k].columns[c].x;
            out[9 * k + 3 * c + 1] = values[k].columns[c].y;
            out[9 * k + 3 * c + 2] = values[k].columns[c].z;
        }
}

bool IsFinite(const Vec3& v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }
bool IsFinite(const Mat3& m) { return IsFinite(m.columns[0]) && IsFinite(m.columns[1]) && IsFinite(m.columns[2]); }

}  // namespace

int GetSolverDevice() { return g_solver_device; }
void SetSolverDevice(int device) { g_solver_device = device; }

std::uint64_t SparseBlockMatrix::MakeKey(int rowBlock, int colBlock)
{
    return (static_cast<std::uint64_t>(static_cast<std::uint32_t>(rowBlock)) << 32u) |
           static_cast<std::uint32_t>(colBlock);
}

void SparseBlockMatrix::Clear()
{
    blockCount = 0;
    rowStart.clear();
    colIndex.clear();
    values.clear();
    blockLookup.clear();
}

void SparseBlockMatrix::ClearValues() { std::fill(values.begin(), values.end(), Mat3::Zero()); }

void SparseBlockMatrix::BuildPattern(int newBlockCount, const std::vector<std::pair<int, int>>& blockCoordinates)
{
    Clear();
    if (newBlockCount <= 0) return;
    blockCount = newBlockCount;
    std::vector<std::vector<int>> rows(static_cast<std::size_t>(blockCount));
    for (const auto& c : blockCoordinates) {
        int r = c.first, k = c.second;
        if (r < 0 || r >= blockCount || k < 0 || k >= blockCount) continue;
        if (r > k) std::swap(r, k);
        rows[static_cast<std::size_t>(r)].push_back(k);
    }
    rowStart.assign(static_cast<std::size_t>(blockCount) + 1, 0);
    for (int r = 0; r < blockCount; ++r) {
        std::vector<int>& cols = rows[static_cast<std::size_t>(r)];
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        rowStart[r + 1] = rowStart[r] + static_cast<int>(cols.size());
        for (int c : cols) {
            blockLookup[MakeKey(r, c)] = static_cast<int>(colIndex.size());
            colIndex.push_back(c);
            values.push_back(Mat3::Zero());
        }
    }
}

int SparseBlockMatrix::FindBlockIndex(int rowBlock, int colBlock) const
{
    if (rowBlock > colBlock) std::swap(rowBlock, colBlock);
    auto it = blockLookup.find(MakeKey(rowBlock, colBlock));
    return it == blockLookup.end() ? -1 : it->second;
}

bool SparseBlockMatrix::AddBlock(int rowBlock, int colBlock, const Mat3& block)
{
    const int k = FindBlockIndex(rowBlock, colBlock);
    if (k < 0) return false;
    const Mat3 add = rowBlock <= colBlock ? block : Transpose(block);
    Mat3& v = values[static_cast<std::size_t>(k)];
    v = Mat3::FromColumns(v.columns[0] + add.columns[0], v.columns[1] + add.columns[1], v.columns[2] + add.columns[2]);
    return true;
}

void SparseBlockMatrix::Multiply(const std::vector<Vec3>& input, std::vector<Vec3>& output) const
{
    const std::size_t n = static_cast<std::size_t>(std::max(0, blockCount));
    if (input.size() < n || rowStart.size() != n + 1) {
        output.assign(n, Vec3{});
        return;
    }
    output.assign(n, Vec3{});
    if (n == 0) return;
    std::vector<double> vals, x(3 * n), y(3 * n);
    PackValues(values, vals);
    for (std::size_t i = 0; i < n; ++i) {
        x[3 * i] = input[i].x;
        x[3 * i + 1] = input[i].y;
        x[3 * i + 2] = input[i].z;
    }
    ThrowOnError(pk_bsr_multiply(g_solver_device, PK_PREC_FP32, blockCount, rowStart.data(), colIndex.data(),
                                 vals.data(), x.data(), y.data()),
                 "SparseBlockMatrix::Multiply");
    for (std::size_t i = 0; i < n; ++i)
        output[i] = Vec3{static_cast<float>(y[3 * i]), static_cast<float>(y[3 * i + 1]), static_cast<float>(y[3 * i + 2])};
}

void SparseBlockMatrix::Multiply(const std::vector<float>& input, std::vector<float>& output) const
{
    const std::size_t n = static_cast<std::size_t>(std::max(0, blockCount));
    if (input.size() < 3 * n || rowStart.size() != n + 1) {
        output.assign(3 * n, 0.0f);
        return;
    }
    std::vector<Vec3> in(n), out;
    for (std::size_t i = 0; i < n; ++i) in[i] = Vec3{input[3 * i], input[3 * i + 1], input[3 * i + 2]};
    Multiply(in, out);
    output.assign(3 * n, 0.0f);
    for (std::size_t i = 0; i < n; ++i) {
        output[3 * i] = out[i].x;
        output[3 * i + 1] = out[i].y;
        output[3 * i + 2] = out[i].z;
    }
}

ConjugateGradientResult SolvePreconditionedConjugateGradient(std::vector<Vec3>& x, const SparseBlockMatrix& A,
                                                             const std::vector<Vec3>& b, int maxIterations,
                                                             float tolerance, const std::vector<Mat3>& MInv,
                                                             std::vector<Vec3>& r, std::vector<Vec3>& d,
                                                             std::vector<Vec3>& qOrS)
{
    ConjugateGradientResult result;
    auto cleared = [&]() {
        x.clear();
        r.clear();
        d.clear();
        qOrS.clear();
    };
    if (b.empty()) {
        cleared();
        result.converged = true;
        return result;
    }
    bool bFinite = true;
    for (const Vec3& v : b) bFinite = bFinite && IsFinite(v);
    if (A.blockCount != static_cast<int>(b.size()) || A.rowStart.size() != static_cast<std::size_t>(A.blockCount + 1) ||
        maxIterations <= 0 || !std::isfinite(tolerance) || tolerance <= 0.0f || !bFinite) {
        cleared();
        return result;
    }
    const int n = A.blockCount;
    std::vector<double> vals, bb(3 * static_cast<std::size_t>(n)), mi, xx(3 * static_cast<std::size_t>(n));
    PackValues(A.values, vals);
    PackValues(MInv, mi);
    for (int i = 0; i < n; ++i) {
        bb[3 * i] = b[i].x;
        bb[3 * i + 1] = b[i].y;
        bb[3 * i + 2] = b[i].z;
    }
    pk_cg_result res{};
    ThrowOnError(pk_pcg(g_solver_device, PK_PREC_FP32, n, A.rowStart.data(), A.colIndex.data(), vals.data(), bb.data(),
                        mi.data(), static_cast<int>(MInv.size()), maxIterations, tolerance, xx.data(), &res),
                 "SolvePreconditionedConjugateGradient");
    result.iterations = res.iterations;
    result.converged = res.converged != 0;
    result.residualNorm = static_cast<float>(res.residual_norm);
    if (!res.have_solution) {
        cleared();
        return result;
    }
    x.assign(static_cast<std::size_t>(n), Vec3{});
    for (int i = 0; i < n; ++i)
        x[i] = Vec3{static_cast<float>(xx[3 * i]), static_cast<float>(xx[3 * i + 1]), static_cast<float>(xx[3 * i + 2])};
    r.assign(static_cast<std::size_t>(n), Vec3{});
    d.assign(static_cast<std::size_t>(n), Vec3{});
    qOrS.assign(static_cast<std::size_t>(n), Vec3{});
    return result;
}

LinearSolveResult CurrentLinearSolver::Solve(const SparseBlockMatrix& matrix, const std::vector<Vec3>& rhs,
                                             std::vector<Vec3>& solution, const LinearSolveSettings& settings)
{
    // LinearSolver.cpp:150-187: maxIterations <= 0 means 3n; the block-Jacobi inverse
    // fails on a missing, non-finite or near-singular (|det| <= 1e-8) diagonal block.
    LinearSolveResult result;
    const int maxIterations =
        settings.maxIterations > 0 ? settings.maxIterations : static_cast<int>(rhs.size()) * 3;
    const std::size_t n = static_cast<std::size_t>(std::max(0, matrix.blockCount));
    inversePreconditioner.assign(n, Mat3::Identity());
    if (settings.useJacobiPreconditioner)
        for (int i = 0; i < matrix.blockCount; ++i) {
            const int k = matrix.FindBlockIndex(i, i);
            if (k < 0) {
                solution.clear();
                return result;
            }
            const Mat3& db = matrix.values[static_cast<std::size_t>(k)];
            const float det = Determinant(db);
            if (!IsFinite(db) || !std::isfinite(det) || std::abs(det) <= 1.0e-8f) {
                solution.clear();
                return result;
            }
            const Mat3 inv = Inverse(db);
            if (!IsFinite(inv)) {
                solution.clear();
                return result;
            }
            inversePreconditioner[static_cast<std::size_t>(i)] = inv;
        }
    const ConjugateGradientResult cg = SolvePreconditionedConjugateGradient(
        solution, matrix, rhs, maxIterations, settings.tolerance, inversePreconditioner, residual, direction, temp);
    result.iterations = cg.iterations;
    result.residualNorm = cg.residualNorm;
    result.converged = cg.converged;
    return result;
}

LinearSolver& GetCurrentLinearSolver()
{
    static CurrentLinearSolver solver;
    return solver;
}

}  // namespace PhysiK
