/*
 * CPU ORACLE -- test infrastructure, not product code.
 *
 * A plain C++17 restatement of the Equelle reference serial backend
 * (sintefmath/equelle backends/serial), exporting the same C ABI as the
 * product (include/eqg.h) so that one simulator source and one test harness
 * run against both.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.
 *
 * What it restates, and from where:
 *   - Cartesian UnstructuredGrid numbering and geometry: OPM GridManager as
 *     used by backends/serial/src/EquelleRuntimeCPU.cpp:20-49; numbering
 *     pinned by backends/cuda/test/gridTest.cpp:104-144 (2D); 3D adds the
 *     K faces last (OPM cart_grid, not vendored).
 *   - HelperOps (internal_faces, ngrad, grad, div, fullngrad, fulldiv):
 *     backends/cuda/src/deviceHelperOps.cpp:84-148.
 *   - CollOfScalar = Opm::AutoDiffBlock<double> (equelleTypes.hpp:67-84):
 *     value + one sparse Jacobian block; sum, product and quotient rules with
 *     Eigen's conservative sparse semantics (union patterns, explicit zeros
 *     kept, no pruning), restated from the rules SINTEF wrote out in
 *     backends/cuda/src/collOfScalar.cu:273-401.  OPM and Eigen are third
 *     party and absent here (versions unpinned; OPM 2018-2019 era by header
 *     paths): the restatement follows their published semantics.
 *   - Every EquelleRuntimeCPU method (EquelleRuntimeCPU.cpp,
 *     EquelleRuntimeCPU_impl.hpp) including newtonSolve.
 *   - The linear solver: BiCGStab (van der Vorst 1992) right-preconditioned
 *     with ILU(0) in natural order (Saad, Iterative Methods, Alg. 10.4),
 *     with a fixed pseudo-random shadow residual (shadow_entry); the
 *     reference delegates to Opm::LinearSolverFactory (not vendored).
 *
 * Parity status: grid topology, index sets, geometry and the On/Extend,
 * trinaryIf, Gradient and Divergence values are pinned by the reference's
 * golden vectors (tests/golden).  Jacobian patterns/values, linear solves
 * and Newton results are "parity unpinned": no runnable reference test
 * produces them (OPM is absent), so this file's documented semantics are
 * the contract.
 */
#include "eqg.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_last_error;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const std::string& msg) { throw Error(code, msg); }

template <class F>
int guarded(F&& f)
{
    try {
        f();
        return EQG_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return EQG_ERR_ARG;
    }
}

// ---------------------------------------------------------------------------
// Sparse matrices in CSR with ascending column indices.  All operations keep
// structural entries (no pruning of numerical zeros), as Eigen's sparse
// sum/difference and conservative product do.
// ---------------------------------------------------------------------------
struct Csr {
    int64_t rows = 0, cols = 0;
    std::vector<int64_t> ptr{0};
    std::vector<int32_t> col;
    std::vector<double> val;
    int64_t nnz() const { return (int64_t)col.size(); }
};

Csr csr_identity(int64_t n)
{
    Csr m;
    m.rows = m.cols = n;
    m.ptr.resize(n + 1);
    m.col.resize(n);
    m.val.assign(n, 1.0);
    for (int64_t i = 0; i <= n; ++i) m.ptr[i] = i;
    for (int64_t i = 0; i < n; ++i) m.col[i] = (int32_t)i;
    return m;
}

// diag(d) * A
Csr csr_scale_rows(const std::vector<double>& d, const Csr& a)
{
    Csr m = a;
    for (int64_t i = 0; i < a.rows; ++i)
        for (int64_t e = a.ptr[i]; e < a.ptr[i + 1]; ++e) m.val[e] = d[i] * a.val[e];
    return m;
}

Csr csr_scale(const Csr& a, double s)
{
    Csr m = a;
    for (auto& v : m.val) v = v * s;
    return m;
}

Csr csr_negate(const Csr& a)
{
    Csr m = a;
    for (auto& v : m.val) v = -v;
    return m;
}

// A + B (sign = +1) or A - B (sign = -1) over the union pattern.
Csr csr_add(const Csr& a, const Csr& b, int sign)
{
    if (a.rows != b.rows || a.cols != b.cols) fail(EQG_ERR_ARG, "Jacobian shape mismatch in sum");
    Csr m;
    m.rows = a.rows;
    m.cols = a.cols;
    m.ptr.assign(a.rows + 1, 0);
    m.col.reserve(a.nnz() + b.nnz());
    m.val.reserve(a.nnz() + b.nnz());
    for (int64_t i = 0; i < a.rows; ++i) {
        int64_t p = a.ptr[i], pe = a.ptr[i + 1], q = b.ptr[i], qe = b.ptr[i + 1];
        while (p < pe || q < qe) {
            if (q >= qe || (p < pe && a.col[p] < b.col[q])) {
                m.col.push_back(a.col[p]);
                m.val.push_back(a.val[p]);
                ++p;
            } else if (p >= pe || b.col[q] < a.col[p]) {
                m.col.push_back(b.col[q]);
                m.val.push_back(sign > 0 ? b.val[q] : -b.val[q]);
                ++q;
            } else {
                m.col.push_back(a.col[p]);
                m.val.push_back(sign > 0 ? a.val[p] + b.val[q] : a.val[p] - b.val[q]);
                ++p;
                ++q;
            }
        }
        m.ptr[i + 1] = (int64_t)m.col.size();
    }
    return m;
}

// Conservative product A*B: every structural product term creates an entry;
// entry (i,j) accumulates A(i,k)*B(k,j) over k ascending (Eigen's order).
Csr csr_multiply(const Csr& a, const Csr& b)
{
    if (a.cols != b.rows) fail(EQG_ERR_ARG, "shape mismatch in sparse product");
    Csr m;
    m.rows = a.rows;
    m.cols = b.cols;
    m.ptr.assign(a.rows + 1, 0);
    std::vector<int64_t> marker(b.cols, -1);
    std::vector<double> acc(b.cols, 0.0);
    std::vector<int32_t> cols_row;
    for (int64_t i = 0; i < a.rows; ++i) {
        cols_row.clear();
        for (int64_t e = a.ptr[i]; e < a.ptr[i + 1]; ++e) {
            const int32_t k = a.col[e];
            const double av = a.val[e];
            for (int64_t f = b.ptr[k]; f < b.ptr[k + 1]; ++f) {
                const int32_t j = b.col[f];
                if (marker[j] != i) {
                    marker[j] = i;
                    acc[j] = 0.0;
                    cols_row.push_back(j);
                }
                acc[j] += av * b.val[f];
            }
        }
        std::sort(cols_row.begin(), cols_row.end());
        for (int32_t j : cols_row) {
            m.col.push_back(j);
            m.val.push_back(acc[j]);
        }
        m.ptr[i + 1] = (int64_t)m.col.size();
    }
    return m;
}

Csr csr_transpose(const Csr& a)
{
    Csr t;
    t.rows = a.cols;
    t.cols = a.rows;
    t.ptr.assign(a.cols + 1, 0);
    for (int32_t c : a.col) t.ptr[c + 1]++;
    for (int64_t i = 0; i < a.cols; ++i) t.ptr[i + 1] += t.ptr[i];
    t.col.resize(a.nnz());
    t.val.resize(a.nnz());
    std::vector<int64_t> pos(t.ptr.begin(), t.ptr.end() - 1);
    for (int64_t i = 0; i < a.rows; ++i)
        for (int64_t e = a.ptr[i]; e < a.ptr[i + 1]; ++e) {
            const int64_t p = pos[a.col[e]]++;
            t.col[p] = (int32_t)i;
            t.val[p] = a.val[e];
        }
    return t;
}

// y = A x, accumulating each row over ascending columns from 0.0.
std::vector<double> csr_apply(const Csr& a, const std::vector<double>& x)
{
    std::vector<double> y(a.rows, 0.0);
#pragma omp parallel for schedule(static) if (a.rows > 4096)
    for (int64_t i = 0; i < a.rows; ++i) {
        double s = 0.0;
        for (int64_t e = a.ptr[i]; e < a.ptr[i + 1]; ++e) s += a.val[e] * x[a.col[e]];
        y[i] = s;
    }
    return y;
}

// Row-selection matrix S (m x n) with S(i, idx[i]) = 1: the matrix
// Opm::subset multiplies by.
Csr selection_matrix(const std::vector<int64_t>& idx, int64_t n)
{
    Csr s;
    s.rows = (int64_t)idx.size();
    s.cols = n;
    s.ptr.resize(idx.size() + 1);
    s.col.resize(idx.size());
    s.val.assign(idx.size(), 1.0);
    for (size_t i = 0; i <= idx.size(); ++i) s.ptr[i] = (int64_t)i;
    for (size_t i = 0; i < idx.size(); ++i) {
        if (idx[i] < 0 || idx[i] >= n) fail(EQG_ERR_ARG, "selection index out of range");
        s.col[i] = (int32_t)idx[i];
    }
    return s;
}

// ---------------------------------------------------------------------------
// AutoDiffBlock<double> with at most one Jacobian block.
// ---------------------------------------------------------------------------
struct Adb {
    std::vector<double> v;
    bool has_jac = false;
    Csr jac;
    int64_t size() const { return (int64_t)v.size(); }
};

Adb adb_constant(std::vector<double> v)
{
    Adb a;
    a.v = std::move(v);
    return a;
}

void check_same_size(const Adb& a, const Adb& b, const char* what)
{
    if (a.size() != b.size())
        fail(EQG_ERR_ARG, std::string("size mismatch in ") + what + ": " + std::to_string(a.size()) +
                              " vs " + std::to_string(b.size()));
    if (a.has_jac && b.has_jac && a.jac.cols != b.jac.cols)
        fail(EQG_ERR_ARG, std::string("Jacobian column mismatch in ") + what);
}

// Binary operator with AutoDiffBlock semantics.  A missing Jacobian acts as
// the Zero block of the other operand's shape (AutoDiffBlock::constant(V,
// blockPattern) in the mixed free operators).
Adb adb_binary(int op, const Adb& a, const Adb& b)
{
    check_same_size(a, b, "binary operator");
    const int64_t n = a.size();
    Adb r;
    r.v.resize(n);
    for (int64_t i = 0; i < n; ++i) {
        switch (op) {
        case EQG_ADD: r.v[i] = a.v[i] + b.v[i]; break;
        case EQG_SUB: r.v[i] = a.v[i] - b.v[i]; break;
        case EQG_MUL: r.v[i] = a.v[i] * b.v[i]; break;
        case EQG_DIV: r.v[i] = a.v[i] / b.v[i]; break;
        default: fail(EQG_ERR_ARG, "unknown binary operator");
        }
    }
    if (!a.has_jac && !b.has_jac) return r;
    r.has_jac = true;
    switch (op) {
    case EQG_ADD:
        r.jac = !a.has_jac ? b.jac : (!b.has_jac ? a.jac : csr_add(a.jac, b.jac, +1));
        break;
    case EQG_SUB:
        r.jac = !a.has_jac ? csr_negate(b.jac) : (!b.has_jac ? a.jac : csr_add(a.jac, b.jac, -1));
        break;
    case EQG_MUL:
        // D2*Ja + D1*Jb, D1 = diag(a.v), D2 = diag(b.v)
        if (!a.has_jac) r.jac = csr_scale_rows(a.v, b.jac);
        else if (!b.has_jac) r.jac = csr_scale_rows(b.v, a.jac);
        else r.jac = csr_add(csr_scale_rows(b.v, a.jac), csr_scale_rows(a.v, b.jac), +1);
        break;
    case EQG_DIV: {
        // D3*(D2*Ja - D1*Jb), D3 = diag(1/(b.v*b.v))
        std::vector<double> d3(n);
        for (int64_t i = 0; i < n; ++i) d3[i] = 1.0 / (b.v[i] * b.v[i]);
        Csr inner;
        if (!a.has_jac) inner = csr_negate(csr_scale_rows(a.v, b.jac));
        else if (!b.has_jac) inner = csr_scale_rows(b.v, a.jac);
        else inner = csr_add(csr_scale_rows(b.v, a.jac), csr_scale_rows(a.v, b.jac), -1);
        r.jac = csr_scale_rows(d3, inner);
        break;
    }
    }
    return r;
}

// Sparse operator times ADB (HelperOps matrix * ADB, Opm::subset/superset).
Adb adb_apply_operator(const Csr& m, const Adb& x)
{
    if (m.cols != x.size()) fail(EQG_ERR_ARG, "operator size mismatch");
    Adb r;
    r.v = csr_apply(m, x.v);
    if (x.has_jac) {
        r.has_jac = true;
        r.jac = csr_multiply(m, x.jac);
    }
    return r;
}

// ---------------------------------------------------------------------------
// Cartesian grid with OPM UnstructuredGrid numbering.
// ---------------------------------------------------------------------------
struct Grid {
    int dim = 2;
    int nx = 6, ny = 1, nz = 1;
    double dx = 1, dy = 1, dz = 1;
    int64_t nc = 0, nf = 0;
    std::vector<int32_t> face_cells;   // 2*nf
    std::vector<double> face_areas;    // nf
    std::vector<double> face_centroids;// dim*nf
    std::vector<double> face_normals;  // dim*nf, area scaled
    std::vector<double> cell_volumes;  // nc
    std::vector<double> cell_centroids;// dim*nc
    std::vector<int64_t> cell_facepos; // nc+1
    std::vector<int32_t> cell_faces;
};

Grid build_grid(int dim, int nx, int ny, int nz, double dx, double dy, double dz)
{
    if (nx < 1 || ny < 1 || nz < 1) fail(EQG_ERR_ARG, "grid dimensions must be positive");
    Grid g;
    g.dim = dim;
    g.nx = nx;
    g.ny = ny;
    g.nz = dim == 3 ? nz : 1;
    g.dx = dx;
    g.dy = dy;
    g.dz = dim == 3 ? dz : 1.0;
    const int NZ = g.nz;
    std::vector<double> X(nx + 1), Y(ny + 1), Z(NZ + 1);
    for (int i = 0; i <= nx; ++i) X[i] = i * dx;
    for (int j = 0; j <= ny; ++j) Y[j] = j * dy;
    for (int k = 0; k <= NZ; ++k) Z[k] = k * g.dz;
    g.nc = (int64_t)nx * ny * NZ;
    auto cell = [&](int i, int j, int k) -> int32_t { return (int32_t)(i + (int64_t)nx * (j + (int64_t)ny * k)); };
    const int64_t fx = (int64_t)(nx + 1) * ny * NZ;
    const int64_t fy = (int64_t)nx * (ny + 1) * NZ;
    const int64_t fz = dim == 3 ? (int64_t)nx * ny * (NZ + 1) : 0;
    g.nf = fx + fy + fz;
    g.face_cells.resize(2 * g.nf);
    g.face_areas.resize(g.nf);
    g.face_centroids.resize(dim * g.nf);
    g.face_normals.assign(dim * g.nf, 0.0);
    int64_t f = 0;
    for (int k = 0; k < NZ; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i <= nx; ++i, ++f) {
                g.face_cells[2 * f] = i > 0 ? cell(i - 1, j, k) : -1;
                g.face_cells[2 * f + 1] = i < nx ? cell(i, j, k) : -1;
                const double a = dim == 3 ? (Y[j + 1] - Y[j]) * (Z[k + 1] - Z[k]) : (Y[j + 1] - Y[j]);
                g.face_areas[f] = a;
                g.face_normals[dim * f + 0] = a;
                g.face_centroids[dim * f + 0] = X[i];
                g.face_centroids[dim * f + 1] = 0.5 * (Y[j] + Y[j + 1]);
                if (dim == 3) g.face_centroids[dim * f + 2] = 0.5 * (Z[k] + Z[k + 1]);
            }
    for (int k = 0; k < NZ; ++k)
        for (int j = 0; j <= ny; ++j)
            for (int i = 0; i < nx; ++i, ++f) {
                g.face_cells[2 * f] = j > 0 ? cell(i, j - 1, k) : -1;
                g.face_cells[2 * f + 1] = j < ny ? cell(i, j, k) : -1;
                const double a = dim == 3 ? (X[i + 1] - X[i]) * (Z[k + 1] - Z[k]) : (X[i + 1] - X[i]);
                g.face_areas[f] = a;
                g.face_normals[dim * f + 1] = a;
                g.face_centroids[dim * f + 0] = 0.5 * (X[i] + X[i + 1]);
                g.face_centroids[dim * f + 1] = Y[j];
                if (dim == 3) g.face_centroids[dim * f + 2] = 0.5 * (Z[k] + Z[k + 1]);
            }
    if (dim == 3)
        for (int k = 0; k <= NZ; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i, ++f) {
                    g.face_cells[2 * f] = k > 0 ? cell(i, j, k - 1) : -1;
                    g.face_cells[2 * f + 1] = k < NZ ? cell(i, j, k) : -1;
                    const double a = (X[i + 1] - X[i]) * (Y[j + 1] - Y[j]);
                    g.face_areas[f] = a;
                    g.face_normals[dim * f + 2] = a;
                    g.face_centroids[dim * f + 0] = 0.5 * (X[i] + X[i + 1]);
                    g.face_centroids[dim * f + 1] = 0.5 * (Y[j] + Y[j + 1]);
                    g.face_centroids[dim * f + 2] = Z[k];
                }
    g.cell_volumes.resize(g.nc);
    g.cell_centroids.resize(dim * g.nc);
    for (int k = 0; k < NZ; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const int32_t c = cell(i, j, k);
                double vol = (X[i + 1] - X[i]) * (Y[j + 1] - Y[j]);
                if (dim == 3) vol *= (Z[k + 1] - Z[k]);
                g.cell_volumes[c] = vol;
                g.cell_centroids[dim * c + 0] = 0.5 * (X[i] + X[i + 1]);
                g.cell_centroids[dim * c + 1] = 0.5 * (Y[j] + Y[j + 1]);
                if (dim == 3) g.cell_centroids[dim * c + 2] = 0.5 * (Z[k] + Z[k + 1]);
            }
    // cell -> faces
    g.cell_facepos.assign(g.nc + 1, 0);
    for (int64_t ff = 0; ff < g.nf; ++ff)
        for (int s = 0; s < 2; ++s)
            if (g.face_cells[2 * ff + s] >= 0) g.cell_facepos[g.face_cells[2 * ff + s] + 1]++;
    for (int64_t c = 0; c < g.nc; ++c) g.cell_facepos[c + 1] += g.cell_facepos[c];
    g.cell_faces.resize(g.cell_facepos[g.nc]);
    std::vector<int64_t> pos(g.cell_facepos.begin(), g.cell_facepos.end() - 1);
    for (int64_t ff = 0; ff < g.nf; ++ff)
        for (int s = 0; s < 2; ++s) {
            const int32_t c = g.face_cells[2 * ff + s];
            if (c >= 0) g.cell_faces[pos[c]++] = (int32_t)ff;
        }
    return g;
}

// A grid read from a file (grid_filename; the reference's
// Opm::GridManager(grid_filename), EquelleRuntimeCPU.cpp:20-24): the
// UnstructuredGrid arrays after the header "eqg-grid 1", each after its
// keyword, as whitespace-separated text (the layout equelle_b200/grids.py
// writes).  nx = ny = nz = 0 mark it as not Cartesian.
Grid read_grid_file(const std::string& path)
{
    std::ifstream in(path.c_str());
    if (!in) fail(EQG_ERR_ARG, "Failed to read grid from file " + path);
    auto expect = [&](const char* key) {
        std::string w;
        in >> w;
        if (w != key) fail(EQG_ERR_ARG, "grid file " + path + ": expected '" + key + "', found '" + w + "'");
    };
    auto number = [&](auto& v) {
        if (!(in >> v)) fail(EQG_ERR_ARG, "grid file " + path + ": expected a number");
    };
    Grid g;
    int version = 0;
    expect("eqg-grid");
    number(version);
    if (version != 1) fail(EQG_ERR_ARG, "grid file " + path + ": unknown format version");
    expect("dimensions");
    number(g.dim);
    expect("cells");
    number(g.nc);
    expect("faces");
    number(g.nf);
    if (g.dim != 2 && g.dim != 3) fail(EQG_ERR_ARG, "Cannot handle " + std::to_string(g.dim) + " dimensions.");
    if (g.nc < 1 || g.nf < 1) fail(EQG_ERR_ARG, "grid file " + path + ": cell or face count out of range");
    g.nx = g.ny = g.nz = 0;
    g.dx = g.dy = g.dz = 0.0;
    auto read_ints = [&](const char* key, int64_t n, auto& v) {
        expect(key);
        v.resize(n);
        for (auto& x : v) number(x);
    };
    auto read_reals = [&](const char* key, int64_t n, std::vector<double>& v) {
        expect(key);
        v.resize(n);
        for (auto& x : v) number(x);
    };
    read_ints("face_cells", 2 * g.nf, g.face_cells);
    read_ints("cell_facepos", g.nc + 1, g.cell_facepos);
    for (int64_t c = 0; c < g.nc; ++c)
        if (g.cell_facepos[c + 1] < g.cell_facepos[c] || g.cell_facepos[0] != 0)
            fail(EQG_ERR_ARG, "grid file " + path + ": bad cell_facepos");
    read_ints("cell_faces", g.cell_facepos[g.nc], g.cell_faces);
    read_reals("face_areas", g.nf, g.face_areas);
    read_reals("face_centroids", g.dim * g.nf, g.face_centroids);
    read_reals("face_normals", g.dim * g.nf, g.face_normals);
    read_reals("cell_volumes", g.nc, g.cell_volumes);
    read_reals("cell_centroids", g.dim * g.nc, g.cell_centroids);
    for (int64_t f = 0; f < g.nf; ++f) {
        const int32_t a = g.face_cells[2 * f], b = g.face_cells[2 * f + 1];
        if (a < -1 || a >= g.nc || b < -1 || b >= g.nc || (a < 0 && b < 0) || a == b)
            fail(EQG_ERR_ARG, "grid file " + path + ": face " + std::to_string(f) + " has invalid cells");
    }
    for (int64_t c = 0; c < g.nc; ++c)
        for (int64_t k = g.cell_facepos[c]; k < g.cell_facepos[c + 1]; ++k) {
            const int32_t f = g.cell_faces[k];
            if (f < 0 || f >= g.nf || (g.face_cells[2 * (int64_t)f] != c && g.face_cells[2 * (int64_t)f + 1] != c))
                fail(EQG_ERR_ARG, "grid file " + path + ": face list of cell " + std::to_string(c) +
                                      " does not match face_cells");
        }
    return g;
}

// HelperOps, construction as in backends/cuda/src/deviceHelperOps.cpp:84-148.
struct HelperOps {
    std::vector<int32_t> internal_faces;
    Csr ngrad, grad, div, fullngrad, fulldiv;
};

HelperOps build_ops(const Grid& g)
{
    HelperOps ops;
    for (int64_t f = 0; f < g.nf; ++f)
        if (g.face_cells[2 * f] >= 0 && g.face_cells[2 * f + 1] >= 0) ops.internal_faces.push_back((int32_t)f);
    const int64_t ni = (int64_t)ops.internal_faces.size();
    Csr& ng = ops.ngrad;
    ng.rows = ni;
    ng.cols = g.nc;
    ng.ptr.resize(ni + 1);
    for (int64_t i = 0; i < ni; ++i) {
        const int32_t f = ops.internal_faces[i];
        int32_t c0 = g.face_cells[2 * f], c1 = g.face_cells[2 * f + 1];
        double v0 = 1.0, v1 = -1.0;
        if (c1 < c0) {
            std::swap(c0, c1);
            std::swap(v0, v1);
        }
        ng.ptr[i] = 2 * i;
        ng.col.push_back(c0);
        ng.val.push_back(v0);
        ng.col.push_back(c1);
        ng.val.push_back(v1);
    }
    ng.ptr[ni] = 2 * ni;
    ops.grad = csr_negate(ops.ngrad);
    ops.div = csr_transpose(ops.ngrad);
    Csr& fg = ops.fullngrad;
    fg.rows = g.nf;
    fg.cols = g.nc;
    fg.ptr.assign(g.nf + 1, 0);
    for (int64_t f = 0; f < g.nf; ++f) {
        int32_t c[2] = {g.face_cells[2 * f], g.face_cells[2 * f + 1]};
        double v[2] = {1.0, -1.0};
        if (c[0] >= 0 && c[1] >= 0 && c[1] < c[0]) {
            std::swap(c[0], c[1]);
            std::swap(v[0], v[1]);
        }
        for (int s = 0; s < 2; ++s)
            if (c[s] >= 0) {
                fg.col.push_back(c[s]);
                fg.val.push_back(v[s]);
            }
        fg.ptr[f + 1] = (int64_t)fg.col.size();
    }
    ops.fulldiv = csr_transpose(ops.fullngrad);
    return ops;
}

// ---------------------------------------------------------------------------
// ILU(0) in natural order and BiCGStab.
// ---------------------------------------------------------------------------
struct Ilu0 {
    Csr lu;                     // L (unit, strictly lower) and U in one pattern
    std::vector<int64_t> diag;  // position of the diagonal in each row
    // Built with OpenMP only: rows grouped by wavefront level of the forward
    // (L) and backward (U) solves, so that rows of one level run in
    // parallel with the same per-row operations as the serial loops.
    std::vector<int64_t> fwd_ptr, fwd_rows, bwd_ptr, bwd_rows;
};

#ifdef _OPENMP
// Rows in wavefront levels: level(i) = 1 + max level of the rows it reads.
void wavefronts(const Ilu0& f, bool lower, std::vector<int64_t>& ptr, std::vector<int64_t>& rows)
{
    const Csr& m = f.lu;
    const int64_t n = m.rows;
    std::vector<int64_t> lev(n, 0);
    int64_t nl = 0;
    for (int64_t k = 0; k < n; ++k) {
        const int64_t i = lower ? k : n - 1 - k;
        int64_t l = 0;
        const int64_t e0 = lower ? m.ptr[i] : f.diag[i] + 1, e1 = lower ? f.diag[i] : m.ptr[i + 1];
        for (int64_t e = e0; e < e1; ++e) l = std::max(l, lev[m.col[e]] + 1);
        lev[i] = l;
        nl = std::max(nl, l + 1);
    }
    ptr.assign(nl + 1, 0);
    for (int64_t i = 0; i < n; ++i) ptr[lev[i] + 1]++;
    for (int64_t l = 0; l < nl; ++l) ptr[l + 1] += ptr[l];
    rows.resize(n);
    std::vector<int64_t> pos(ptr.begin(), ptr.end() - 1);
    for (int64_t i = 0; i < n; ++i) rows[pos[lev[i]]++] = i;
}
#endif

bool ilu0_factor(const Csr& a, Ilu0& f)
{
    f.lu = a;
    const int64_t n = a.rows;
    f.diag.assign(n, -1);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t e = a.ptr[i]; e < a.ptr[i + 1]; ++e)
            if (a.col[e] == i) f.diag[i] = e;
    for (int64_t i = 0; i < n; ++i)
        if (f.diag[i] < 0) return false;
    std::vector<int64_t> where(n, -1);
    Csr& m = f.lu;
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t e = m.ptr[i]; e < m.ptr[i + 1]; ++e) where[m.col[e]] = e;
        for (int64_t e = m.ptr[i]; e < m.ptr[i + 1] && m.col[e] < i; ++e) {
            const int32_t k = m.col[e];
            const double piv = m.val[f.diag[k]];
            if (piv == 0.0) return false;
            const double lik = m.val[e] / piv;
            m.val[e] = lik;
            for (int64_t g = f.diag[k] + 1; g < m.ptr[k + 1]; ++g) {
                const int64_t w = where[m.col[g]];
                if (w >= 0) m.val[w] -= lik * m.val[g];
            }
        }
        for (int64_t e = m.ptr[i]; e < m.ptr[i + 1]; ++e) where[m.col[e]] = -1;
        if (m.val[f.diag[i]] == 0.0) return false;
    }
#ifdef _OPENMP
    wavefronts(f, true, f.fwd_ptr, f.fwd_rows);
    wavefronts(f, false, f.bwd_ptr, f.bwd_rows);
#endif
    return true;
}

void ilu0_apply(const Ilu0& f, const std::vector<double>& b, std::vector<double>& x)
{
    const Csr& m = f.lu;
    const int64_t n = m.rows;
    x.resize(n);
#ifdef _OPENMP
#pragma omp parallel
    {
        for (size_t l = 0; l + 1 < f.fwd_ptr.size(); ++l) {
#pragma omp for schedule(static)
            for (int64_t k = f.fwd_ptr[l]; k < f.fwd_ptr[l + 1]; ++k) {
                const int64_t i = f.fwd_rows[k];
                double s = b[i];
                for (int64_t e = m.ptr[i]; e < f.diag[i]; ++e) s -= m.val[e] * x[m.col[e]];
                x[i] = s;
            }
        }
        for (size_t l = 0; l + 1 < f.bwd_ptr.size(); ++l) {
#pragma omp for schedule(static)
            for (int64_t k = f.bwd_ptr[l]; k < f.bwd_ptr[l + 1]; ++k) {
                const int64_t i = f.bwd_rows[k];
                double s = x[i];
                for (int64_t e = f.diag[i] + 1; e < m.ptr[i + 1]; ++e) s -= m.val[e] * x[m.col[e]];
                x[i] = s / m.val[f.diag[i]];
            }
        }
    }
#else
    for (int64_t i = 0; i < n; ++i) {
        double s = b[i];
        for (int64_t e = m.ptr[i]; e < f.diag[i]; ++e) s -= m.val[e] * x[m.col[e]];
        x[i] = s;
    }
    for (int64_t i = n - 1; i >= 0; --i) {
        double s = x[i];
        for (int64_t e = f.diag[i] + 1; e < m.ptr[i + 1]; ++e) s -= m.val[e] * x[m.col[e]];
        x[i] = s / m.val[f.diag[i]];
    }
#endif
}

double dot(const std::vector<double>& a, const std::vector<double>& b)
{
    double s = 0.0;
    const int64_t n = (int64_t)a.size();
#pragma omp parallel for schedule(static) reduction(+ : s) if (n > 4096)
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

// Shadow residual of BiCGStab: a fixed, dense pseudo-random vector in
// [-1, 1) from a 32-bit integer hash of the row index.  The textbook choice
// rhat = r0 breaks down when r0 is nearly a unit vector, which is the case
// at the first Newton iteration of well-driven flow (the residual is nonzero
// only in the well cells).
double shadow_entry(int64_t i)
{
    uint32_t x = (uint32_t)((uint64_t)i * 0x9E3779B1ull);
    x ^= x >> 16;
    x *= 0x85EBCA6Bu;
    x ^= x >> 13;
    return 2.0 * ((double)x / 4294967296.0) - 1.0;
}

struct SolveReport {
    bool converged = false;
    int iterations = 0;
    double rel_residual = 0.0;
    double factor_ms = 0.0, krylov_ms = 0.0;
};

double ms_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Solves A x = b from x = 0; converged when ||b - A x|| <= tol * ||b||.
SolveReport bicgstab_ilu0(const Csr& a, const std::vector<double>& b, std::vector<double>& x, double tol,
                          int max_iter)
{
    SolveReport rep;
    const int64_t n = a.rows;
    x.assign(n, 0.0);
    const double bnorm = std::sqrt(dot(b, b));
    if (bnorm == 0.0) {
        rep.converged = true;
        return rep;
    }
    Ilu0 prec;
    const auto t0 = std::chrono::steady_clock::now();
    const bool factored = ilu0_factor(a, prec);
    rep.factor_ms = ms_since(t0);
    if (!factored) return rep;
    const auto t1 = std::chrono::steady_clock::now();
    struct KrylovClock {
        SolveReport& r;
        std::chrono::steady_clock::time_point t;
        ~KrylovClock() { r.krylov_ms = ms_since(t); }
    } kclock{rep, t1};
    std::vector<double> r = b, rhat(n), p(n, 0.0), v(n, 0.0), s(n), t(n), ph(n), sh(n);
    for (int64_t i = 0; i < n; ++i) rhat[i] = shadow_entry(i);
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    for (int it = 1; it <= max_iter; ++it) {
        const double rho_new = dot(rhat, r);
        if (rho_new == 0.0) break;
        const double beta = (rho_new / rho) * (alpha / omega);
#pragma omp parallel for schedule(static) if (n > 4096)
        for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        ilu0_apply(prec, p, ph);
        v = csr_apply(a, ph);
        const double rv = dot(rhat, v);
        if (rv == 0.0) break;
        alpha = rho_new / rv;
#pragma omp parallel for schedule(static) if (n > 4096)
        for (int64_t i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
        const double snorm = std::sqrt(dot(s, s));
        rep.iterations = it;
        if (snorm <= tol * bnorm) {
            for (int64_t i = 0; i < n; ++i) x[i] += alpha * ph[i];
            rep.converged = true;
            rep.rel_residual = snorm / bnorm;
            return rep;
        }
        ilu0_apply(prec, s, sh);
        t = csr_apply(a, sh);
        const double tt = dot(t, t);
        if (tt == 0.0) break;
        omega = dot(t, s) / tt;
#pragma omp parallel for schedule(static) if (n > 4096)
        for (int64_t i = 0; i < n; ++i) {
            x[i] += alpha * ph[i] + omega * sh[i];
            r[i] = s[i] - omega * t[i];
        }
        rho = rho_new;
        const double rnorm = std::sqrt(dot(r, r));
        rep.rel_residual = rnorm / bnorm;
        if (rnorm <= tol * bnorm) {
            rep.converged = true;
            return rep;
        }
        if (omega == 0.0) break;
    }
    return rep;
}

}  // namespace

// ---------------------------------------------------------------------------
// Handles
// ---------------------------------------------------------------------------
struct eqg_runtime {
    std::map<std::string, std::string> params;
    Grid grid;
    HelperOps ops;
    int verbose = 0;
    int max_iter = 10;
    double abs_res_tol = 1e-6;
    double lin_tol = 1e-8;
    int lin_max_iter = 1000;
    eqg_set* builtin[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    std::vector<std::chrono::steady_clock::time_point> marks;
    std::vector<eqg_solve_info> solves;
    eqg_stats stats{};
    // output copies (eqg_output_*), made at once; shared with a waiting thread
    std::mutex output_mutex;
    std::map<int64_t, std::vector<double>> outputs;
    int64_t next_ticket = 1;
};

struct eqg_set {
    std::atomic<int> refs{1};
    int entity = EQG_CELLS;
    std::vector<int32_t> idx;
};

struct eqg_mask {
    std::atomic<int> refs{1};
    std::vector<uint8_t> v;
};

struct eqg_coll {
    std::atomic<int> refs{1};
    Adb a;
};

namespace {

void need(const void* p, const char* what)
{
    if (!p) fail(EQG_ERR_ARG, std::string("null handle: ") + what);
}

eqg_coll* make_coll(Adb a)
{
    auto* c = new eqg_coll;
    c->a = std::move(a);
    return c;
}

eqg_set* make_set(int entity, std::vector<int32_t> idx)
{
    auto* s = new eqg_set;
    s->entity = entity;
    s->idx = std::move(idx);
    return s;
}

double param_d(const eqg_runtime* rt, const std::string& k, double d)
{
    auto it = rt->params.find(k);
    return it == rt->params.end() ? d : std::stod(it->second);
}

int param_i(const eqg_runtime* rt, const std::string& k, int d)
{
    auto it = rt->params.find(k);
    if (it == rt->params.end()) return d;
    if (it->second == "true") return 1;
    if (it->second == "false") return 0;
    return (int)std::stol(it->second);
}

bool is_boundary_cell(const Grid& g, int64_t c)
{
    for (int64_t h = g.cell_facepos[c]; h < g.cell_facepos[c + 1]; ++h) {
        const int32_t f = g.cell_faces[h];
        if (g.face_cells[2 * f] < 0 || g.face_cells[2 * f + 1] < 0) return true;
    }
    return false;
}

// subsetIndices (EquelleRuntimeCPU_impl.hpp:28-83): for each element of
// `sub`, its position in the sorted, duplicate-free `super`.  Unmatched
// elements are an error here (the reference only asserts).
std::vector<int64_t> subset_indices(const std::vector<int32_t>& super, const std::vector<int32_t>& sub)
{
    for (size_t i = 1; i < super.size(); ++i)
        if (!(super[i - 1] < super[i])) fail(EQG_ERR_ARG, "superset is not sorted and unique");
    std::vector<int64_t> out(sub.size());
    for (size_t i = 0; i < sub.size(); ++i) {
        auto it = std::lower_bound(super.begin(), super.end(), sub[i]);
        if (it == super.end() || *it != sub[i])
            fail(EQG_ERR_ARG, "element " + std::to_string(sub[i]) + " is not in the given superset");
        out[i] = it - super.begin();
    }
    return out;
}

}  // namespace

extern "C" {

const char* eqg_last_error(void) { return g_last_error.c_str(); }
const char* eqg_backend_name(void) { return "cpu-oracle"; }

int eqg_runtime_create(int nparams, const char* const* keys, const char* const* values, eqg_runtime** out)
{
    return guarded([&] {
        need(out, "out");
        auto rt = std::make_unique<eqg_runtime>();
        for (int i = 0; i < nparams; ++i) rt->params[keys[i]] = values[i];
        if (rt->params.count("grid_filename")) {
            rt->grid = read_grid_file(rt->params["grid_filename"]);
        } else {
            const int dim = param_i(rt.get(), "grid_dim", 2);
            if (dim != 2 && dim != 3) fail(EQG_ERR_ARG, "Cannot handle " + std::to_string(dim) + " dimensions.");
            rt->grid = build_grid(dim, param_i(rt.get(), "nx", 6), param_i(rt.get(), "ny", 1),
                                  param_i(rt.get(), "nz", 1), param_d(rt.get(), "dx", 1.0),
                                  param_d(rt.get(), "dy", 1.0), param_d(rt.get(), "dz", 1.0));
        }
        rt->ops = build_ops(rt->grid);
        rt->verbose = param_i(rt.get(), "verbose", 0);
        rt->max_iter = param_i(rt.get(), "max_iter", 10);
        rt->abs_res_tol = param_d(rt.get(), "abs_res_tol", 1e-6);
        rt->lin_tol = param_d(rt.get(), "linsolver_residual_tolerance", 1e-8);
        rt->lin_max_iter = param_i(rt.get(), "linsolver_max_iterations", 1000);
        const Grid& g = rt->grid;
        std::vector<int32_t> all_c(g.nc), bc, ic, all_f(g.nf), bf;
        std::iota(all_c.begin(), all_c.end(), 0);
        std::iota(all_f.begin(), all_f.end(), 0);
        for (int64_t c = 0; c < g.nc; ++c) (is_boundary_cell(g, c) ? bc : ic).push_back((int32_t)c);
        for (int64_t f = 0; f < g.nf; ++f)
            if (g.face_cells[2 * f] < 0 || g.face_cells[2 * f + 1] < 0) bf.push_back((int32_t)f);
        rt->builtin[EQG_ALL_CELLS] = make_set(EQG_CELLS, all_c);
        rt->builtin[EQG_BOUNDARY_CELLS] = make_set(EQG_CELLS, bc);
        rt->builtin[EQG_INTERIOR_CELLS] = make_set(EQG_CELLS, ic);
        rt->builtin[EQG_ALL_FACES] = make_set(EQG_FACES, all_f);
        rt->builtin[EQG_BOUNDARY_FACES] = make_set(EQG_FACES, bf);
        rt->builtin[EQG_INTERIOR_FACES] = make_set(EQG_FACES, rt->ops.internal_faces);
        *out = rt.release();
    });
}

void eqg_runtime_destroy(eqg_runtime* rt)
{
    if (!rt) return;
    for (auto* s : rt->builtin) eqg_set_release(s);
    delete rt;
}

int eqg_runtime_grid_info(const eqg_runtime* rt, eqg_grid_info* out)
{
    return guarded([&] {
        need(rt, "runtime");
        const Grid& g = rt->grid;
        out->dimensions = g.dim;
        out->nx = g.nx;
        out->ny = g.ny;
        out->nz = g.nz;
        out->dx = g.dx;
        out->dy = g.dy;
        out->dz = g.dz;
        out->number_of_cells = g.nc;
        out->number_of_faces = g.nf;
        out->number_of_interior_faces = (int64_t)rt->ops.internal_faces.size();
    });
}

int eqg_runtime_synchronize(eqg_runtime* rt) { return guarded([&] { need(rt, "runtime"); }); }

int eqg_runtime_stats(const eqg_runtime* rt, eqg_stats* out)
{
    return guarded([&] {
        need(rt, "runtime");
        *out = rt->stats;
    });
}

int eqg_runtime_reset_stats(eqg_runtime* rt)
{
    return guarded([&] {
        need(rt, "runtime");
        rt->stats = eqg_stats{};
    });
}

int eqg_runtime_kernel_profile(const eqg_runtime* rt, char* buf, int64_t len, int64_t* needed)
{
    return guarded([&] {
        need(rt, "runtime");
        *needed = 3;  // the oracle launches no kernels: "{}"
        if (buf && len > 0) std::snprintf(buf, (size_t)len, "{}");
    });
}

int eqg_runtime_mark(eqg_runtime* rt, int* mark_id)
{
    return guarded([&] {
        need(rt, "runtime");
        rt->marks.push_back(std::chrono::steady_clock::now());
        *mark_id = (int)rt->marks.size() - 1;
    });
}

int eqg_runtime_elapsed_ms(eqg_runtime* rt, int a, int b, double* ms)
{
    return guarded([&] {
        need(rt, "runtime");
        if (a < 0 || b < 0 || a >= (int)rt->marks.size() || b >= (int)rt->marks.size())
            fail(EQG_ERR_ARG, "mark id out of range");
        *ms = std::chrono::duration<double, std::milli>(rt->marks[b] - rt->marks[a]).count();
    });
}

int eqg_runtime_solve_marks(const eqg_runtime* rt, int64_t k, int* s, int* e)
{
    return guarded([&] {
        need(rt, "runtime");
        if (k < 0 || k >= (int64_t)rt->solves.size()) fail(EQG_ERR_ARG, "solve index out of range");
        *s = rt->solves[k].start_mark;
        *e = rt->solves[k].end_mark;
    });
}

int eqg_runtime_solve_info(const eqg_runtime* rt, int64_t k, eqg_solve_info* out)
{
    return guarded([&] {
        need(rt, "runtime");
        if (k < 0 || k >= (int64_t)rt->solves.size()) fail(EQG_ERR_ARG, "solve index out of range");
        *out = rt->solves[k];
    });
}

// ---- sets -------------------------------------------------------------
int eqg_set_builtin(eqg_runtime* rt, int which, eqg_set** out)
{
    return guarded([&] {
        need(rt, "runtime");
        if (which < 0 || which > 5) fail(EQG_ERR_ARG, "unknown builtin set");
        eqg_set_retain(rt->builtin[which]);
        *out = rt->builtin[which];
    });
}

int eqg_set_from_host(eqg_runtime* rt, int entity, const int32_t* idx, int64_t n, eqg_set** out)
{
    return guarded([&] {
        need(rt, "runtime");
        if (entity != EQG_CELLS && entity != EQG_FACES) fail(EQG_ERR_ARG, "bad entity kind");
        const int64_t lim = entity == EQG_CELLS ? rt->grid.nc : rt->grid.nf;
        for (int64_t i = 0; i < n; ++i)
            if (idx[i] < -1 || idx[i] >= lim) fail(EQG_ERR_ARG, "entity index out of range");
        *out = make_set(entity, std::vector<int32_t>(idx, idx + n));
    });
}

int eqg_set_size(const eqg_set* s, int64_t* n)
{
    return guarded([&] {
        need(s, "set");
        *n = (int64_t)s->idx.size();
    });
}

int eqg_set_entity(const eqg_set* s, int* e)
{
    return guarded([&] {
        need(s, "set");
        *e = s->entity;
    });
}

int eqg_set_to_host(const eqg_set* s, int32_t* out)
{
    return guarded([&] {
        need(s, "set");
        std::copy(s->idx.begin(), s->idx.end(), out);
    });
}

void eqg_set_retain(eqg_set* s)
{
    if (s) s->refs++;
}
void eqg_set_release(eqg_set* s)
{
    if (s && --s->refs == 0) delete s;
}

static int neighbour_cell(eqg_runtime* rt, const eqg_set* faces, int side, eqg_set** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(faces, "faces");
        if (faces->entity != EQG_FACES) fail(EQG_ERR_ARG, "firstCell/secondCell need a face collection");
        std::vector<int32_t> r(faces->idx.size());
        for (size_t i = 0; i < r.size(); ++i) {
            const int32_t f = faces->idx[i];
            if (f < 0) fail(EQG_ERR_ARG, "firstCell/secondCell of an empty face");
            r[i] = rt->grid.face_cells[2 * f + side];
        }
        *out = make_set(EQG_CELLS, std::move(r));
    });
}

int eqg_first_cell(eqg_runtime* rt, const eqg_set* f, eqg_set** out) { return neighbour_cell(rt, f, 0, out); }
int eqg_second_cell(eqg_runtime* rt, const eqg_set* f, eqg_set** out) { return neighbour_cell(rt, f, 1, out); }

int eqg_set_is_empty(eqg_runtime* rt, const eqg_set* s, eqg_mask** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(s, "set");
        auto* m = new eqg_mask;
        m->v.resize(s->idx.size());
        for (size_t i = 0; i < s->idx.size(); ++i) m->v[i] = s->idx[i] < 0;
        *out = m;
    });
}

int eqg_set_on(eqg_runtime* rt, const eqg_set* data, const eqg_set* from, const eqg_set* to, eqg_set** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(data, "data");
        need(from, "from");
        need(to, "to");
        if (data->idx.size() != from->idx.size()) fail(EQG_ERR_ARG, "On: data size differs from its set");
        if (from->entity != to->entity) fail(EQG_ERR_ARG, "On: sets of different entity kinds");
        auto ind = subset_indices(from->idx, to->idx);
        std::vector<int32_t> r(ind.size());
        for (size_t i = 0; i < ind.size(); ++i) r[i] = data->idx[ind[i]];
        *out = make_set(data->entity, std::move(r));
    });
}

int eqg_set_extend(eqg_runtime* rt, const eqg_set* data, const eqg_set* from, const eqg_set* to, eqg_set** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(data, "data");
        need(from, "from");
        need(to, "to");
        if (data->idx.size() != from->idx.size()) fail(EQG_ERR_ARG, "Extend: data size differs from its set");
        if (from->entity != to->entity) fail(EQG_ERR_ARG, "Extend: sets of different entity kinds");
        auto ind = subset_indices(to->idx, from->idx);
        std::vector<int32_t> r(to->idx.size(), -1);
        for (size_t i = 0; i < ind.size(); ++i) r[ind[i]] = data->idx[i];
        *out = make_set(data->entity, std::move(r));
    });
}

int eqg_set_select(eqg_runtime* rt, const eqg_mask* pred, const eqg_set* a, const eqg_set* b, eqg_set** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(pred, "predicate");
        need(a, "iftrue");
        need(b, "iffalse");
        const size_t n = pred->v.size();
        if (a->idx.size() != n || b->idx.size() != n) fail(EQG_ERR_ARG, "trinaryIf: size mismatch");
        if (a->entity != b->entity) fail(EQG_ERR_ARG, "trinaryIf: entity kinds differ");
        std::vector<int32_t> r(n);
        for (size_t i = 0; i < n; ++i) r[i] = pred->v[i] ? a->idx[i] : b->idx[i];
        *out = make_set(a->entity, std::move(r));
    });
}

int eqg_set_check_subset(eqg_runtime* rt, const eqg_set* sub, const eqg_set* super, int* is_sorted, int* is_included)
{
    return guarded([&] {
        need(rt, "runtime");
        need(sub, "subset");
        need(super, "superset");
        *is_sorted = std::is_sorted(sub->idx.begin(), sub->idx.end()) ? 1 : 0;
        *is_included = (*is_sorted && std::is_sorted(super->idx.begin(), super->idx.end()) &&
                        std::includes(super->idx.begin(), super->idx.end(), sub->idx.begin(), sub->idx.end()))
                           ? 1
                           : 0;
    });
}

// ---- masks -------------------------------------------------------------
int eqg_mask_from_host(eqg_runtime* rt, const uint8_t* v, int64_t n, eqg_mask** out)
{
    return guarded([&] {
        need(rt, "runtime");
        auto* m = new eqg_mask;
        m->v.resize(n);
        for (int64_t i = 0; i < n; ++i) m->v[i] = v[i] ? 1 : 0;
        *out = m;
    });
}

int eqg_mask_size(const eqg_mask* m, int64_t* n)
{
    return guarded([&] {
        need(m, "mask");
        *n = (int64_t)m->v.size();
    });
}

int eqg_mask_to_host(const eqg_mask* m, uint8_t* out)
{
    return guarded([&] {
        need(m, "mask");
        std::copy(m->v.begin(), m->v.end(), out);
    });
}

void eqg_mask_retain(eqg_mask* m)
{
    if (m) m->refs++;
}
void eqg_mask_release(eqg_mask* m)
{
    if (m && --m->refs == 0) delete m;
}

int eqg_mask_logic(eqg_runtime* rt, int op, const eqg_mask* a, const eqg_mask* b, eqg_mask** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(a, "mask");
        if (op != EQG_NOT) {
            need(b, "mask");
            if (a->v.size() != b->v.size()) fail(EQG_ERR_ARG, "mask size mismatch");
        }
        auto* m = new eqg_mask;
        m->v.resize(a->v.size());
        for (size_t i = 0; i < a->v.size(); ++i) {
            switch (op) {
            case EQG_AND: m->v[i] = a->v[i] && b->v[i]; break;
            case EQG_OR: m->v[i] = a->v[i] || b->v[i]; break;
            case EQG_NOT: m->v[i] = !a->v[i]; break;
            default: delete m; fail(EQG_ERR_ARG, "unknown mask operator");
            }
        }
        *out = m;
    });
}

// ---- scalar collections -------------------------------------------------
int eqg_coll_from_host(eqg_runtime* rt, const double* v, int64_t n, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        if (n < 0) fail(EQG_ERR_ARG, "negative size");
        *out = make_coll(adb_constant(std::vector<double>(v, v + n)));
    });
}

int eqg_coll_constant(eqg_runtime* rt, double v, int64_t n, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        if (n < 0) fail(EQG_ERR_ARG, "negative size");
        *out = make_coll(adb_constant(std::vector<double>(n, v)));
    });
}

int eqg_coll_size(const eqg_coll* c, int64_t* n)
{
    return guarded([&] {
        need(c, "collection");
        *n = c->a.size();
    });
}

int eqg_coll_to_host(const eqg_coll* c, double* out)
{
    return guarded([&] {
        need(c, "collection");
        std::copy(c->a.v.begin(), c->a.v.end(), out);
    });
}

// Nothing is deferred here: every operation computes its values when called.
int eqg_coll_evaluate(eqg_runtime* rt, const eqg_coll* c)
{
    return guarded([&] {
        need(rt, "runtime");
        need(c, "collection");
    });
}

int eqg_output_begin(eqg_runtime* rt, const eqg_coll* c, int64_t* ticket)
{
    return guarded([&] {
        need(rt, "runtime");
        need(c, "collection");
        std::lock_guard<std::mutex> lock(rt->output_mutex);
        *ticket = rt->next_ticket++;
        rt->outputs[*ticket] = c->a.v;
    });
}

int eqg_output_wait(eqg_runtime* rt, int64_t ticket, const double** values, int64_t* n)
{
    return guarded([&] {
        need(rt, "runtime");
        std::lock_guard<std::mutex> lock(rt->output_mutex);
        auto it = rt->outputs.find(ticket);
        if (it == rt->outputs.end()) fail(EQG_ERR_ARG, "unknown output ticket");
        *values = it->second.data();
        *n = (int64_t)it->second.size();
    });
}

int eqg_output_release(eqg_runtime* rt, int64_t ticket)
{
    return guarded([&] {
        need(rt, "runtime");
        std::lock_guard<std::mutex> lock(rt->output_mutex);
        if (!rt->outputs.erase(ticket)) fail(EQG_ERR_ARG, "unknown output ticket");
    });
}

int eqg_coll_jacobian_info(const eqg_coll* c, int64_t* rows, int64_t* cols, int64_t* nnz)
{
    return guarded([&] {
        need(c, "collection");
        if (!c->a.has_jac) {
            *rows = c->a.size();
            *cols = 0;
            *nnz = -1;
            return;
        }
        *rows = c->a.jac.rows;
        *cols = c->a.jac.cols;
        *nnz = c->a.jac.nnz();
    });
}

int eqg_coll_jacobian_to_host(const eqg_coll* c, int64_t* rowptr, int32_t* colind, double* vals)
{
    return guarded([&] {
        need(c, "collection");
        if (!c->a.has_jac) fail(EQG_ERR_ARG, "collection has no Jacobian");
        const Csr& j = c->a.jac;
        if (rowptr) std::copy(j.ptr.begin(), j.ptr.end(), rowptr);
        if (colind) std::copy(j.col.begin(), j.col.end(), colind);
        if (vals) std::copy(j.val.begin(), j.val.end(), vals);
    });
}

void eqg_coll_retain(eqg_coll* c)
{
    if (c) c->refs++;
}
void eqg_coll_release(eqg_coll* c)
{
    if (c && --c->refs == 0) delete c;
}

int eqg_variable(eqg_runtime* rt, const eqg_coll* init, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(init, "collection");
        Adb a;
        a.v = init->a.v;
        a.has_jac = true;
        a.jac = csr_identity(a.size());
        *out = make_coll(std::move(a));
    });
}

int eqg_value_of(eqg_runtime* rt, const eqg_coll* c, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(c, "collection");
        *out = make_coll(adb_constant(c->a.v));
    });
}

int eqg_binary(eqg_runtime* rt, int op, const eqg_coll* a, const eqg_coll* b, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(a, "lhs");
        need(b, "rhs");
        *out = make_coll(adb_binary(op, a->a, b->a));
    });
}

int eqg_binary_scalar(eqg_runtime* rt, int op, const eqg_coll* a, double s, int scalar_left, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(a, "collection");
        if (op == EQG_MUL) {
            // ADB * Scalar: value v*s, Jacobian J*s.
            Adb r;
            r.v.resize(a->a.size());
            for (int64_t i = 0; i < a->a.size(); ++i) r.v[i] = a->a.v[i] * s;
            if (a->a.has_jac) {
                r.has_jac = true;
                r.jac = csr_scale(a->a.jac, s);
            }
            *out = make_coll(std::move(r));
            return;
        }
        // Other scalar operators go through V::Constant(size, s)
        // (equelleTypes.hpp:93-102).
        Adb c = adb_constant(std::vector<double>(a->a.size(), s));
        *out = make_coll(scalar_left ? adb_binary(op, c, a->a) : adb_binary(op, a->a, c));
    });
}

int eqg_unary(eqg_runtime* rt, int op, const eqg_coll* a, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(a, "collection");
        const Adb& x = a->a;
        const int64_t n = x.size();
        switch (op) {
        case EQG_NEG:
            *out = make_coll(adb_binary(EQG_SUB, adb_constant(std::vector<double>(n, 0.0)), x));
            return;
        case EQG_SQRT: {
            Adb r;
            r.v.resize(n);
            for (int64_t i = 0; i < n; ++i) r.v[i] = std::sqrt(x.v[i]);
            if (x.has_jac) {
                std::vector<double> d(n);
                for (int64_t i = 0; i < n; ++i) d[i] = 0.5 / r.v[i];
                r.has_jac = true;
                r.jac = csr_scale_rows(d, x.jac);
            }
            *out = make_coll(std::move(r));
            return;
        }
        case EQG_ABS: {
            std::vector<double> f(n);
            for (int64_t i = 0; i < n; ++i) f[i] = x.v[i] >= 0.0 ? 1.0 : -1.0;
            *out = make_coll(adb_binary(EQG_MUL, adb_constant(f), x));
            return;
        }
        default: fail(EQG_ERR_ARG, "unknown unary operator");
        }
    });
}

static uint8_t compare_values(int op, double a, double b)
{
    switch (op) {
    case EQG_LT: return a < b;
    case EQG_LE: return a <= b;
    case EQG_GT: return a > b;
    case EQG_GE: return a >= b;
    case EQG_EQ: return a == b;
    case EQG_NE: return a != b;
    }
    fail(EQG_ERR_ARG, "unknown comparison");
}

int eqg_compare(eqg_runtime* rt, int op, const eqg_coll* a, const eqg_coll* b, eqg_mask** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(a, "lhs");
        need(b, "rhs");
        if (a->a.size() != b->a.size()) fail(EQG_ERR_ARG, "comparison size mismatch");
        auto* m = new eqg_mask;
        m->v.resize(a->a.size());
        for (int64_t i = 0; i < a->a.size(); ++i) m->v[i] = compare_values(op, a->a.v[i], b->a.v[i]);
        *out = m;
    });
}

int eqg_compare_scalar(eqg_runtime* rt, int op, const eqg_coll* a, double s, int scalar_left, eqg_mask** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(a, "collection");
        auto* m = new eqg_mask;
        m->v.resize(a->a.size());
        for (int64_t i = 0; i < a->a.size(); ++i)
            m->v[i] = scalar_left ? compare_values(op, s, a->a.v[i]) : compare_values(op, a->a.v[i], s);
        *out = m;
    });
}

int eqg_gradient(eqg_runtime* rt, const eqg_coll* a, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(a, "collection");
        if (a->a.size() != rt->grid.nc) fail(EQG_ERR_ARG, "Gradient needs a collection on all cells");
        *out = make_coll(adb_apply_operator(rt->ops.grad, a->a));
    });
}

int eqg_neg_gradient(eqg_runtime* rt, const eqg_coll* a, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(a, "collection");
        if (a->a.size() != rt->grid.nc) fail(EQG_ERR_ARG, "negGradient needs a collection on all cells");
        *out = make_coll(adb_apply_operator(rt->ops.ngrad, a->a));
    });
}

int eqg_interior_divergence(eqg_runtime* rt, const eqg_coll* a, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(a, "collection");
        if (a->a.size() != (int64_t)rt->ops.internal_faces.size())
            fail(EQG_ERR_ARG, "interiorDivergence needs a collection on interior faces");
        *out = make_coll(adb_apply_operator(rt->ops.div, a->a));
    });
}

int eqg_divergence(eqg_runtime* rt, const eqg_coll* a, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(a, "collection");
        if (a->a.size() == (int64_t)rt->ops.internal_faces.size()) {
            *out = make_coll(adb_apply_operator(rt->ops.div, a->a));
            return;
        }
        if (a->a.size() != rt->grid.nf) fail(EQG_ERR_ARG, "Divergence needs a collection on all or interior faces");
        *out = make_coll(adb_apply_operator(rt->ops.fulldiv, a->a));
    });
}

int eqg_on(eqg_runtime* rt, const eqg_coll* data, const eqg_set* from, const eqg_set* to, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(data, "data");
        need(from, "from");
        need(to, "to");
        if (data->a.size() != (int64_t)from->idx.size()) fail(EQG_ERR_ARG, "On: data size differs from its set");
        if (from->entity != to->entity) fail(EQG_ERR_ARG, "On: sets of different entity kinds");
        auto ind = subset_indices(from->idx, to->idx);
        *out = make_coll(adb_apply_operator(selection_matrix(ind, data->a.size()), data->a));
    });
}

int eqg_extend(eqg_runtime* rt, const eqg_coll* data, const eqg_set* from, const eqg_set* to, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(data, "data");
        need(from, "from");
        need(to, "to");
        if (data->a.size() != (int64_t)from->idx.size()) fail(EQG_ERR_ARG, "Extend: data size differs from its set");
        if (from->entity != to->entity) fail(EQG_ERR_ARG, "Extend: sets of different entity kinds");
        auto ind = subset_indices(to->idx, from->idx);
        // superset = S^T * x with S the selection matrix of `ind`.
        Csr st = csr_transpose(selection_matrix(ind, (int64_t)to->idx.size()));
        *out = make_coll(adb_apply_operator(st, data->a));
    });
}

int eqg_select(eqg_runtime* rt, const eqg_mask* pred, const eqg_coll* a, const eqg_coll* b, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(pred, "predicate");
        need(a, "iftrue");
        need(b, "iffalse");
        const int64_t n = (int64_t)pred->v.size();
        if (a->a.size() != n || b->a.size() != n) fail(EQG_ERR_ARG, "trinaryIf: size mismatch");
        std::vector<double> t(n, 1.0), f(n, 0.0);
        for (int64_t i = 0; i < n; ++i)
            if (!pred->v[i]) {
                t[i] = 0.0;
                f[i] = 1.0;
            }
        // iftrue * trueones + iffalse * falseones
        Adb lhs = adb_binary(EQG_MUL, adb_constant(t), a->a);
        Adb rhs = adb_binary(EQG_MUL, adb_constant(f), b->a);
        *out = make_coll(adb_binary(EQG_ADD, lhs, rhs));
    });
}

int eqg_span_subset(eqg_runtime* rt, const eqg_coll* a, int64_t start, int64_t num, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(a, "collection");
        if (start < 0 || num < 0 || start + num > a->a.size()) fail(EQG_ERR_ARG, "span out of range");
        std::vector<int64_t> ind(num);
        for (int64_t i = 0; i < num; ++i) ind[i] = start + i;
        *out = make_coll(adb_apply_operator(selection_matrix(ind, a->a.size()), a->a));
    });
}

int eqg_span_superset(eqg_runtime* rt, const eqg_coll* a, int64_t start, int64_t total, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(a, "collection");
        if (start < 0 || start + a->a.size() > total) fail(EQG_ERR_ARG, "span out of range");
        std::vector<int64_t> ind(a->a.size());
        for (int64_t i = 0; i < a->a.size(); ++i) ind[i] = start + i;
        Csr st = csr_transpose(selection_matrix(ind, total));
        *out = make_coll(adb_apply_operator(st, a->a));
    });
}

int eqg_reduce(eqg_runtime* rt, int op, const eqg_coll* a, double* out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(a, "collection");
        const auto& v = a->a.v;
        switch (op) {
        case EQG_MIN:
            if (v.empty()) fail(EQG_ERR_ARG, "minReduce of an empty collection");
            *out = *std::min_element(v.begin(), v.end());
            break;
        case EQG_MAX:
            if (v.empty()) fail(EQG_ERR_ARG, "maxReduce of an empty collection");
            *out = *std::max_element(v.begin(), v.end());
            break;
        case EQG_SUM: {
            double s = 0.0;
            for (double x : v) s += x;
            *out = s;
            break;
        }
        case EQG_PROD: {
            double p = 1.0;
            for (double x : v) p *= x;
            *out = p;
            break;
        }
        default: fail(EQG_ERR_ARG, "unknown reduction");
        }
    });
}

int eqg_two_norm(eqg_runtime* rt, const eqg_coll* a, double* out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(a, "collection");
        *out = std::sqrt(dot(a->a.v, a->a.v));
    });
}

int eqg_measure(eqg_runtime* rt, const eqg_set* s, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(s, "set");
        const auto& src = s->entity == EQG_CELLS ? rt->grid.cell_volumes : rt->grid.face_areas;
        std::vector<double> v(s->idx.size());
        for (size_t i = 0; i < v.size(); ++i) {
            if (s->idx[i] < 0) fail(EQG_ERR_ARG, "norm of an empty entity");
            v[i] = src[s->idx[i]];
        }
        *out = make_coll(adb_constant(std::move(v)));
    });
}

int eqg_centroid(eqg_runtime* rt, const eqg_set* s, int comp, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(s, "set");
        const int dim = rt->grid.dim;
        if (comp < 0 || comp >= dim) fail(EQG_ERR_ARG, "centroid component out of range");
        const auto& src = s->entity == EQG_CELLS ? rt->grid.cell_centroids : rt->grid.face_centroids;
        std::vector<double> v(s->idx.size());
        for (size_t i = 0; i < v.size(); ++i) {
            if (s->idx[i] < 0) fail(EQG_ERR_ARG, "centroid of an empty entity");
            v[i] = src[(size_t)dim * s->idx[i] + comp];
        }
        *out = make_coll(adb_constant(std::move(v)));
    });
}

int eqg_normal(eqg_runtime* rt, const eqg_set* s, int comp, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(s, "set");
        if (s->entity != EQG_FACES) fail(EQG_ERR_ARG, "normal needs a face collection");
        const int dim = rt->grid.dim;
        if (comp < 0 || comp >= dim) fail(EQG_ERR_ARG, "normal component out of range");
        std::vector<double> v(s->idx.size());
        for (size_t i = 0; i < v.size(); ++i) {
            if (s->idx[i] < 0) fail(EQG_ERR_ARG, "normal of an empty face");
            const double* n = &rt->grid.face_normals[(size_t)dim * s->idx[i]];
            double nn = 0.0;
            for (int d = 0; d < dim; ++d) nn += n[d] * n[d];
            v[i] = n[comp] / std::sqrt(nn);
        }
        *out = make_coll(adb_constant(std::move(v)));
    });
}

int eqg_solve_for_update(eqg_runtime* rt, const eqg_coll* residual, eqg_coll** du)
{
    return guarded([&] {
        need(rt, "runtime");
        need(residual, "residual");
        const Adb& r = residual->a;
        if (!r.has_jac) fail(EQG_ERR_ARG, "solveForUpdate: residual has no Jacobian");
        if (r.jac.rows != r.jac.cols) fail(EQG_ERR_ARG, "solveForUpdate: Jacobian is not square");
        std::vector<double> x;
        SolveReport rep = bicgstab_ilu0(r.jac, r.v, x, rt->lin_tol, rt->lin_max_iter);
        rt->stats.linear_solves++;
        rt->stats.krylov_iterations += rep.iterations;
        rt->stats.last_linear_residual = rep.rel_residual;
        rt->stats.factor_ms += rep.factor_ms;
        rt->stats.krylov_ms += rep.krylov_ms;
        rt->stats.last_matrix_rows = r.jac.rows;
        rt->stats.last_matrix_nnz = r.jac.nnz();
        rt->stats.last_block_size = 1;
        rt->stats.last_matrix_blocks = r.jac.nnz();
        if (rt->verbose > 2)
            std::printf("        solveForUpdate: BiCGStab+ILU0 %d iterations, rel. residual %g\n", rep.iterations,
                        rep.rel_residual);
        if (!rep.converged) fail(EQG_ERR_SOLVER, "Linear solver convergence failure.");
        *du = make_coll(adb_constant(std::move(x)));
    });
}

int eqg_newton_solve(eqg_runtime* rt, eqg_residual_fn fn, void* user, const eqg_coll* u0, eqg_coll** out)
{
    return guarded([&] {
        need(rt, "runtime");
        need(u0, "initial guess");
        if (!fn) fail(EQG_ERR_ARG, "null residual function");
        int m0 = 0;
        eqg_runtime_mark(rt, &m0);
        rt->stats.newton_solves++;
        const int64_t krylov0 = rt->stats.krylov_iterations;
        const double res_ms0 = rt->stats.residual_ms, fac_ms0 = rt->stats.factor_ms, kry_ms0 = rt->stats.krylov_ms;
        eqg_coll* u = nullptr;
        if (eqg_variable(rt, u0, &u) != EQG_OK) fail(EQG_ERR_ARG, g_last_error);
        auto cleanup = [&](eqg_coll* a) { eqg_coll_release(a); };
        eqg_coll* res = nullptr;
        auto evaluate = [&](eqg_coll* uu, eqg_coll** out) {
            const auto t0 = std::chrono::steady_clock::now();
            const int st = fn(user, uu, out);
            rt->stats.residual_ms += ms_since(t0);
            rt->stats.residual_evaluations++;
            return st;
        };
        if (evaluate(u, &res) != 0 || !res) {
            cleanup(u);
            fail(EQG_ERR_CALLBACK, "residual callback failed");
        }
        auto norm = [&](const eqg_coll* c) { return std::sqrt(dot(c->a.v, c->a.v)); };
        int iter = 0;
        if (rt->verbose > 1)
            std::printf("    newtonSolve: iter = %d (max = %d), norm(residual) = %g (tol = %g)\n", iter, rt->max_iter,
                        norm(res), rt->abs_res_tol);
        while (norm(res) > rt->abs_res_tol && iter < rt->max_iter) {
            eqg_coll* du = nullptr;
            int st = eqg_solve_for_update(rt, res, &du);
            if (st != EQG_OK) {
                cleanup(u);
                cleanup(res);
                fail(st, g_last_error);
            }
            eqg_coll* un = make_coll(adb_binary(EQG_SUB, u->a, du->a));
            cleanup(du);
            cleanup(u);
            u = un;
            cleanup(res);
            res = nullptr;
            if (evaluate(u, &res) != 0 || !res) {
                cleanup(u);
                fail(EQG_ERR_CALLBACK, "residual callback failed");
            }
            ++iter;
            rt->stats.newton_iterations++;
            if (rt->verbose > 1)
                std::printf("    newtonSolve: iter = %d (max = %d), norm(residual) = %g (tol = %g)\n", iter,
                            rt->max_iter, norm(res), rt->abs_res_tol);
        }
        if (rt->verbose > 0) {
            if (norm(res) > rt->abs_res_tol)
                std::printf("Newton solver failed to converge in %d iterations\n", rt->max_iter);
            else
                std::printf("Newton solver converged in %d iterations\n", iter);
        }
        eqg_solve_info info{};
        info.start_mark = m0;
        info.newton_iterations = iter;
        info.converged = norm(res) <= rt->abs_res_tol ? 1 : 0;
        info.krylov_iterations = rt->stats.krylov_iterations - krylov0;
        info.residual_ms = rt->stats.residual_ms - res_ms0;
        info.factor_ms = rt->stats.factor_ms - fac_ms0;
        info.krylov_ms = rt->stats.krylov_ms - kry_ms0;
        *out = make_coll(adb_constant(u->a.v));
        cleanup(u);
        cleanup(res);
        eqg_runtime_mark(rt, &info.end_mark);
        rt->solves.push_back(info);
    });
}

}  // extern "C"
