"""Grid files for the runtime's `grid_filename` parameter.

The reference builds Opm::GridManager(grid_filename) (backends/serial/src/
EquelleRuntimeCPU.cpp:20-24) and then uses only the arrays of the
resulting UnstructuredGrid.  The runtime (libeqg.so) and the CPU oracle read
those arrays from a text file of this layout:

    eqg-grid 1
    dimensions <2|3>
    cells <nc>
    faces <nf>
    face_cells      2 nf integers: first and second cell of each face (-1: outside)
    cell_facepos    nc + 1 integers
    cell_faces      cell_facepos[nc] integers (cell c: cell_faces[facepos[c]:facepos[c+1]])
    face_areas      nf reals
    face_centroids  dim nf reals, face by face
    face_normals    dim nf reals, face by face, scaled by the area, first cell -> second
    cell_volumes    nc reals
    cell_centroids  dim nc reals, cell by cell

Reals are written with 17 significant digits, so they read back exactly.

Builders here:
- `cartesian`: the Cartesian grid in the numbering and with the geometry the
  runtime builds itself from grid_dim, nx, ... (OPM's Cartesian
  UnstructuredGrid), so a run from the file can be compared bit for bit
  with a run on the built-in grid;
- `mixed_2d`: quadrilaterals on a seeded, jittered node lattice, a seeded
  fraction of them split into two triangles (cells with 3 and 4 faces);
- `extruded`: a 2D grid extruded into layers (prisms and hexahedra).
"""
import numpy as np


class Grid:
    """UnstructuredGrid arrays (face_centroids, face_normals and
    cell_centroids as (n, dim) arrays)."""

    def __init__(self, dim, face_cells, cell_facepos, cell_faces, face_areas, face_centroids, face_normals,
                 cell_volumes, cell_centroids):
        self.dim = int(dim)
        self.face_cells = np.asarray(face_cells, dtype=np.int64).reshape(-1, 2)
        self.cell_facepos = np.asarray(cell_facepos, dtype=np.int64)
        self.cell_faces = np.asarray(cell_faces, dtype=np.int64)
        self.face_areas = np.asarray(face_areas, dtype=np.float64)
        self.face_centroids = np.asarray(face_centroids, dtype=np.float64).reshape(-1, self.dim)
        self.face_normals = np.asarray(face_normals, dtype=np.float64).reshape(-1, self.dim)
        self.cell_volumes = np.asarray(cell_volumes, dtype=np.float64)
        self.cell_centroids = np.asarray(cell_centroids, dtype=np.float64).reshape(-1, self.dim)

    @property
    def nc(self):
        return len(self.cell_volumes)

    @property
    def nf(self):
        return len(self.face_areas)

    def boundary_faces(self):
        return np.nonzero((self.face_cells < 0).any(axis=1))[0]

    def write(self, path):
        def ints(a):
            return " ".join(str(int(x)) for x in np.asarray(a).reshape(-1))

        def reals(a):
            return " ".join("%.17g" % x for x in np.asarray(a, dtype=np.float64).reshape(-1))

        with open(path, "w") as f:
            f.write("eqg-grid 1\ndimensions %d\ncells %d\nfaces %d\n" % (self.dim, self.nc, self.nf))
            f.write("face_cells %s\n" % ints(self.face_cells))
            f.write("cell_facepos %s\n" % ints(self.cell_facepos))
            f.write("cell_faces %s\n" % ints(self.cell_faces))
            f.write("face_areas %s\n" % reals(self.face_areas))
            f.write("face_centroids %s\n" % reals(self.face_centroids))
            f.write("face_normals %s\n" % reals(self.face_normals))
            f.write("cell_volumes %s\n" % reals(self.cell_volumes))
            f.write("cell_centroids %s\n" % reals(self.cell_centroids))
        return path


def _cell_faces_from(face_cells, nc):
    """cell_facepos / cell_faces: each cell's faces in ascending order."""
    fc = np.asarray(face_cells).reshape(-1, 2)
    pairs = [(c, f) for f in range(len(fc)) for c in fc[f] if c >= 0]
    pairs.sort()
    counts = np.zeros(nc + 1, dtype=np.int64)
    for c, _ in pairs:
        counts[c + 1] += 1
    return np.cumsum(counts), np.array([f for _, f in pairs], dtype=np.int64)


def cartesian(nx, ny, nz=None, dx=1.0, dy=1.0, dz=1.0):
    """The grid the runtime builds from grid_dim = 2 (nz None) or 3, nx, ny,
    nz, dx, dy, dz: x faces (i fastest, then j, then k), then y faces, then
    z faces; face_cells (lower/left neighbour or -1, upper/right or -1);
    node coordinates i * dx, widths and midpoints as their differences and
    half sums."""
    dim = 2 if nz is None else 3
    NZ = 1 if nz is None else nz
    hz = 1.0 if nz is None else dz
    X = np.arange(nx + 1, dtype=np.float64) * dx
    Y = np.arange(ny + 1, dtype=np.float64) * dy
    Z = np.arange(NZ + 1, dtype=np.float64) * hz

    def cell(i, j, k):
        return i + nx * (j + ny * k)

    fc, fa, fcen, fnor = [], [], [], []
    for k in range(NZ):
        for j in range(ny):
            for i in range(nx + 1):
                fc.append((cell(i - 1, j, k) if i > 0 else -1, cell(i, j, k) if i < nx else -1))
                a = (Y[j + 1] - Y[j]) * (Z[k + 1] - Z[k]) if dim == 3 else (Y[j + 1] - Y[j])
                fa.append(a)
                cen = [X[i], 0.5 * (Y[j] + Y[j + 1])] + ([0.5 * (Z[k] + Z[k + 1])] if dim == 3 else [])
                fcen.append(cen)
                fnor.append([a, 0.0] + ([0.0] if dim == 3 else []))
    for k in range(NZ):
        for j in range(ny + 1):
            for i in range(nx):
                fc.append((cell(i, j - 1, k) if j > 0 else -1, cell(i, j, k) if j < ny else -1))
                a = (X[i + 1] - X[i]) * (Z[k + 1] - Z[k]) if dim == 3 else (X[i + 1] - X[i])
                fa.append(a)
                cen = [0.5 * (X[i] + X[i + 1]), Y[j]] + ([0.5 * (Z[k] + Z[k + 1])] if dim == 3 else [])
                fcen.append(cen)
                fnor.append([0.0, a] + ([0.0] if dim == 3 else []))
    if dim == 3:
        for k in range(NZ + 1):
            for j in range(ny):
                for i in range(nx):
                    fc.append((cell(i, j, k - 1) if k > 0 else -1, cell(i, j, k) if k < NZ else -1))
                    a = (X[i + 1] - X[i]) * (Y[j + 1] - Y[j])
                    fa.append(a)
                    fcen.append([0.5 * (X[i] + X[i + 1]), 0.5 * (Y[j] + Y[j + 1]), Z[k]])
                    fnor.append([0.0, 0.0, a])
    nc = nx * ny * NZ
    vol = np.zeros(nc)
    ccen = np.zeros((nc, dim))
    for k in range(NZ):
        for j in range(ny):
            for i in range(nx):
                c = cell(i, j, k)
                v = (X[i + 1] - X[i]) * (Y[j + 1] - Y[j])
                if dim == 3:
                    v = v * (Z[k + 1] - Z[k])
                vol[c] = v
                ccen[c, 0] = 0.5 * (X[i] + X[i + 1])
                ccen[c, 1] = 0.5 * (Y[j] + Y[j + 1])
                if dim == 3:
                    ccen[c, 2] = 0.5 * (Z[k] + Z[k + 1])
    facepos, faces = _cell_faces_from(fc, nc)
    return Grid(dim, fc, facepos, faces, fa, fcen, fnor, vol, ccen)


def _polygon(xy):
    """Area and centroid of a counter-clockwise polygon (shoelace)."""
    x, y = xy[:, 0], xy[:, 1]
    xn, yn = np.roll(x, -1), np.roll(y, -1)
    cross = x * yn - xn * y
    a = 0.5 * cross.sum()
    cx = ((x + xn) * cross).sum() / (6.0 * a)
    cy = ((y + yn) * cross).sum() / (6.0 * a)
    return a, cx, cy


def mixed_2d(nx, ny, seed=0, jitter=0.25, split=0.5, dx=1.0, dy=1.0):
    """A 2D grid of nx x ny quadrilaterals on a lattice whose interior nodes
    are moved by up to `jitter` cell widths (seeded), a seeded fraction
    `split` of them cut into two triangles along a diagonal.  Faces are the
    edges, numbered by (lower node, higher node); a face's first cell is the
    one that runs along it from its lower to its higher node counter-
    clockwise, so boundary faces come as (cell, -1) and (-1, cell)."""
    rng = np.random.default_rng(seed)
    nodes = np.zeros(((nx + 1) * (ny + 1), 2))
    for j in range(ny + 1):
        for i in range(nx + 1):
            px, py = i * dx, j * dy
            if 0 < i < nx:
                px += rng.uniform(-jitter, jitter) * dx
            if 0 < j < ny:
                py += rng.uniform(-jitter, jitter) * dy
            nodes[i + (nx + 1) * j] = (px, py)
    cells = []
    for j in range(ny):
        for i in range(nx):
            a, b = i + (nx + 1) * j, i + 1 + (nx + 1) * j
            c, d = i + 1 + (nx + 1) * (j + 1), i + (nx + 1) * (j + 1)
            if rng.uniform() < split:
                if rng.uniform() < 0.5:
                    cells += [[a, b, c], [a, c, d]]
                else:
                    cells += [[a, b, d], [b, c, d]]
            else:
                cells.append([a, b, c, d])
    return _from_polygons(nodes, cells)


def _from_polygons(nodes, cells):
    edges = {}
    for ci, poly in enumerate(cells):
        for t in range(len(poly)):
            p, q = poly[t], poly[(t + 1) % len(poly)]
            key = (min(p, q), max(p, q))
            side = 0 if p < q else 1  # runs low -> high: first cell
            edges.setdefault(key, [-1, -1])[side] = ci
    keys = sorted(edges)
    fc = np.array([edges[k] for k in keys], dtype=np.int64)
    fa, fcen, fnor = [], [], []
    for p, q in keys:
        ex, ey = nodes[q] - nodes[p]
        fa.append(np.sqrt(ex * ex + ey * ey))
        fcen.append(0.5 * (nodes[p] + nodes[q]))
        fnor.append([ey, -ex])  # right of low -> high: out of the first cell
    vol, ccen = [], []
    for poly in cells:
        a, cx, cy = _polygon(nodes[poly])
        vol.append(a)
        ccen.append([cx, cy])
    facepos, faces = _cell_faces_from(fc, len(cells))
    return Grid(2, fc, facepos, faces, fa, fcen, fnor, vol, ccen)


def extruded(g2, nz, dz=1.0):
    """A 2D grid extruded into nz layers of thickness dz: layer k of 2D cell
    c is cell k n2 + c; lateral faces layer by layer, then the horizontal
    faces from the bottom up, each from the cell below to the cell above."""
    n2c, n2f = g2.nc, g2.nf
    fc, fa, fcen, fnor = [], [], [], []
    for k in range(nz):
        zc = (k + 0.5) * dz
        for f in range(n2f):
            a, b = g2.face_cells[f]
            fc.append((a + k * n2c if a >= 0 else -1, b + k * n2c if b >= 0 else -1))
            fa.append(g2.face_areas[f] * dz)
            fcen.append([g2.face_centroids[f, 0], g2.face_centroids[f, 1], zc])
            fnor.append([g2.face_normals[f, 0] * dz, g2.face_normals[f, 1] * dz, 0.0])
    for k in range(nz + 1):
        for c in range(n2c):
            fc.append((c + (k - 1) * n2c if k > 0 else -1, c + k * n2c if k < nz else -1))
            fa.append(g2.cell_volumes[c])
            fcen.append([g2.cell_centroids[c, 0], g2.cell_centroids[c, 1], k * dz])
            fnor.append([0.0, 0.0, g2.cell_volumes[c]])
    vol, ccen = [], []
    for k in range(nz):
        for c in range(n2c):
            vol.append(g2.cell_volumes[c] * dz)
            ccen.append([g2.cell_centroids[c, 0], g2.cell_centroids[c, 1], (k + 0.5) * dz])
    facepos, faces = _cell_faces_from(fc, n2c * nz)
    return Grid(3, fc, facepos, faces, fa, fcen, fnor, vol, ccen)
