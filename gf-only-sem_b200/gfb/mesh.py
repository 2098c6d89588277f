"""Synthetic partition inputs for the CG-SEM elastic time loop.

Builds, for a structured (optionally deformed) hexahedral mesh, every array
the reference forward solver reads from ``partition_{r}.h5`` / ``config.h5``
after ``read_partition_all`` merges the partitions (RankData, forward/share/
include/gf/types.hpp:27-140).  The formulas follow the reference
preprocessor:

* corner order and trilinear geometry: preprocess/gll_geometry.py:14-26,
  53-67, 132-186 (``dxi_dx = inv(J).ravel()`` with ``J = dS.T @ corners``,
  ``mass = detJ * w_i w_j w_k``, later multiplied by density, cli.py:448);
* GLL points/weights: preprocess/gll_geometry.py:29-50 (values equal the
  forward solver's gll.hpp tables to rounding);
* element numbering x fastest, then y, then z, z positive downward with the
  free surface at z = zmin (preprocess/model_writer.py:68-72,
  recording_map.py:53);
* PML flags for structured meshes: preprocess/cli.py:247-264;
  legacy ramp damping: preprocess/pml.py:23-124;
* C-PML coefficients: preprocess/pml_cpml.py:42-147 (profiles), 174-253
  (regions), 261-345 (convolution coefficients), 353-515 (A1..A5);
* global node numbering (ibool): quantised-coordinate lexsort,
  preprocess/partition.py:192-254;
* point-force location and Lagrange weights, normalised over all
  containing cells: preprocess/source_locator.py:74-213, 244-375;
* recording map: preprocess/recording_map.py:18-170;
* Lame parameters mu = rho vs^2, lambda = rho (vp^2 - 2 vs^2): cli.py:374-376;
* CFL step ``cfl * h_min / vp_max``: preprocess/cfl_validator.py:21-74.

Everything is float64 / int32 / int64 exactly as the reference stores it.
The arrays are inputs to the solver; they are produced here, never by the
solver itself.
"""

from __future__ import annotations

import dataclasses
import math
from typing import Callable, Optional

import numpy as np

# GMSH hex corner order in reference coordinates (gll_geometry.py:14-26)
HEX_CORNERS = np.array(
    [
        [-1, -1, -1],
        [1, -1, -1],
        [1, 1, -1],
        [-1, 1, -1],
        [-1, -1, 1],
        [1, -1, 1],
        [1, 1, 1],
        [-1, 1, 1],
    ],
    dtype=np.float64,
)

# C-PML constants (pml_cpml.py:20-34)
THETA = 1.0 / 8.0
K_MIN_PML = 1.0
K_MAX_PML = 1.0
NPOWER = 2
R_COEF = 1e-5
MIN_DISTANCE = 1e-6
CPML_X_ONLY, CPML_Y_ONLY, CPML_Z_ONLY = 1, 2, 3
CPML_XY_ONLY, CPML_XZ_ONLY, CPML_YZ_ONLY, CPML_XYZ = 4, 5, 6, 7


# ---------------------------------------------------------------------------
# GLL tables
# ---------------------------------------------------------------------------


def for_chunks(fn, starts, threads: int = 1):
    """fn(start) for every start; on ``threads`` host threads when > 1 (numpy
    releases the interpreter lock in its array loops and matrix products)."""
    starts = list(starts)
    if threads <= 1 or len(starts) <= 1:
        for c0 in starts:
            fn(c0)
        return
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(max_workers=threads) as ex:
        for _ in ex.map(fn, starts):
            pass


def _legendre(n: int, x):
    x = np.asarray(x, dtype=np.float64)
    if n == 0:
        return np.ones_like(x)
    p0, p1 = np.ones_like(x), x.copy()
    for k in range(1, n):
        p0, p1 = p1, ((2.0 * k + 1.0) * x * p1 - k * p0) / (k + 1.0)
    return p1


def gll_points(N: int) -> np.ndarray:
    """GLL points on [-1, 1] (roots of P_N' plus endpoints), by Newton."""
    if N < 1:
        raise ValueError("polynomial order must be >= 1")
    x = np.empty(N + 1)
    x[0], x[N] = -1.0, 1.0
    for i in range(1, N):
        xi = -math.cos(math.pi * i / N)
        for _ in range(100):
            pn = float(_legendre(N, xi))
            pnm1 = float(_legendre(N - 1, xi))
            f = N * (xi * pn - pnm1) / (xi * xi - 1.0)
            df = (2.0 * xi * f - N * (N + 1.0) * pn) / (1.0 - xi * xi)
            dx = -f / df
            xi += dx
            if abs(dx) < 1e-15 * (1.0 + abs(xi)):
                break
        x[i] = xi
    return x


def gll_weights(x: np.ndarray) -> np.ndarray:
    N = len(x) - 1
    pn = _legendre(N, x)
    return 2.0 / (N * (N + 1.0) * pn * pn)


def gll_derivative(x: np.ndarray) -> np.ndarray:
    """D[i, j] = l_j'(x_i) (forward/share/include/gf/gll.hpp:109-131)."""
    N = len(x) - 1
    pn = _legendre(N, x)
    D = np.zeros((N + 1, N + 1))
    for i in range(N + 1):
        for j in range(N + 1):
            if i != j:
                D[i, j] = pn[i] / (pn[j] * (x[i] - x[j]))
    D[0, 0] = -0.25 * N * (N + 1.0)
    D[N, N] = 0.25 * N * (N + 1.0)
    return D


def lagrange_1d(xe: float, nodes: np.ndarray) -> np.ndarray:
    """l_i(xe) (source_locator.py:145-161)."""
    n = len(nodes)
    w = np.ones(n)
    for i in range(n):
        for j in range(n):
            if i != j:
                w[i] *= (xe - nodes[j]) / (nodes[i] - nodes[j])
    return w


# ---------------------------------------------------------------------------
# Mesh description
# ---------------------------------------------------------------------------


@dataclasses.dataclass
class MeshSpec:
    """Structured hex mesh, x fastest / y / z slowest, z positive down."""

    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    order: int = 4
    # interior-vertex jitter as a fraction of the edge length (uniform +-)
    jitter: float = 0.0
    # top-surface relief: number of random-phase sinusoids and max amplitude
    topo_terms: int = 0
    topo_amp: float = 0.0
    seed: int = 0
    # PML thickness in elements (zmin is the free surface: always 0)
    pml: dict = dataclasses.field(default_factory=dict)

    @property
    def n_cell(self) -> int:
        return self.nx * self.ny * self.nz


def vertex_grid(spec: MeshSpec) -> np.ndarray:
    """Vertex coordinates [nx+1, ny+1, nz+1, 3].

    Deformation (seeded): interior vertices are jittered by a uniform
    +-jitter fraction of the edge length; the top surface is lowered/raised
    by a sum of random-phase sinusoids whose displacement fades linearly to
    zero at the bottom so every hex stays valid.
    """
    rng = np.random.default_rng(spec.seed)
    ix = np.arange(spec.nx + 1) * spec.dx
    iy = np.arange(spec.ny + 1) * spec.dy
    iz = np.arange(spec.nz + 1) * spec.dz
    X, Y, Z = np.meshgrid(ix, iy, iz, indexing="ij")
    V = np.stack([X, Y, Z], axis=-1).astype(np.float64)
    lz = spec.nz * spec.dz
    if spec.topo_terms > 0 and spec.topo_amp > 0.0:
        lx, ly = spec.nx * spec.dx, spec.ny * spec.dy
        h = np.zeros((spec.nx + 1, spec.ny + 1))
        amp = spec.topo_amp / spec.topo_terms
        for _ in range(spec.topo_terms):
            kx = rng.integers(1, 4) * 2.0 * math.pi / lx
            ky = rng.integers(1, 4) * 2.0 * math.pi / ly
            ph = rng.uniform(0.0, 2.0 * math.pi)
            h += amp * np.sin(kx * X[:, :, 0] + ky * Y[:, :, 0] + ph)
        # keep the top surface the domain's zmin so the free surface is flat
        # in z-min terms only at its lowest point; shift rows proportionally
        fade = 1.0 - Z / lz
        V[..., 2] = Z + h[:, :, None] * fade
        V[..., 2] -= V[..., 2].min()
    if spec.jitter > 0.0:
        J = rng.uniform(-spec.jitter, spec.jitter, size=V.shape)
        J[..., 0] *= spec.dx
        J[..., 1] *= spec.dy
        J[..., 2] *= spec.dz
        interior = np.zeros(V.shape[:3], dtype=bool)
        interior[1:-1, 1:-1, 1:-1] = True
        V[interior] += J[interior]
    return V


def cell_corners(spec: MeshSpec, V: np.ndarray) -> np.ndarray:
    """[n_cell, 8, 3] corners in GMSH order, cells numbered x fastest."""
    nx, ny, nz = spec.nx, spec.ny, spec.nz
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    out = np.empty((nx * ny * nz, 8, 3))
    for a, (ca, cb, cc) in enumerate(HEX_CORNERS.astype(int)):
        out[:, a] = V[i + (ca > 0), j + (cb > 0), k + (cc > 0)]
    return out


def gll_geometry(corners: np.ndarray, order: int, chunk: int = 65536, threads: int = 1):
    """coords, jacobian (det J), dxi_dx (inv(J) raveled), geometric mass.

    Same trilinear map as gll_geometry.py:160-184, vectorised over cells;
    ``threads`` > 1 processes chunks of cells on that many host threads (the
    per-cell arithmetic, hence every value, is the same)."""
    pts = gll_points(order)
    w = gll_weights(pts)
    ng = order + 1
    n_cell = corners.shape[0]
    xi, eta, zeta = np.meshgrid(pts, pts, pts, indexing="ij")  # [ng,ng,ng]
    xi, eta, zeta = xi.ravel(), eta.ravel(), zeta.ravel()
    ca, cb, cc = HEX_CORNERS[:, 0], HEX_CORNERS[:, 1], HEX_CORNERS[:, 2]
    # S [nn, 8], dS [nn, 8, 3]
    fa = 1 + np.outer(xi, ca)
    fb = 1 + np.outer(eta, cb)
    fc = 1 + np.outer(zeta, cc)
    S = 0.125 * fa * fb * fc
    dS = np.stack([0.125 * ca * fb * fc, 0.125 * fa * cb * fc, 0.125 * fa * fb * cc], axis=-1)
    nn = ng**3
    coords = np.empty((n_cell, nn, 3))
    jac = np.empty((n_cell, nn))
    dxi = np.empty((n_cell, nn, 9))
    # shape-function products as matrix products over all cells of a chunk
    dSm = np.ascontiguousarray(dS.transpose(0, 2, 1).reshape(nn * 3, 8))  # [(n, m), a]

    def one(c0):
        cv = corners[c0 : c0 + chunk]
        ne = cv.shape[0]
        xa = np.ascontiguousarray(cv.transpose(1, 0, 2).reshape(8, ne * 3))  # [a, (e, c)]
        coords[c0 : c0 + chunk] = (S @ xa).reshape(nn, ne, 3).transpose(1, 0, 2)
        # J[m, c] = sum_a dS[a, m] x_a[c]  (J = dS.T @ corners, gll_geometry.py:173)
        J = (dSm @ xa).reshape(nn, 3, ne, 3).transpose(2, 0, 1, 3)  # [e, n, m, c]
        a, b, c = J[..., 0, 0], J[..., 0, 1], J[..., 0, 2]
        d, e, f = J[..., 1, 0], J[..., 1, 1], J[..., 1, 2]
        g, h, i = J[..., 2, 0], J[..., 2, 1], J[..., 2, 2]
        # determinant and inverse by cofactors (equal to LU-based det/inv to
        # rounding; the reference's np.linalg calls differ from these only in
        # the last bits)
        A, B, C = e * i - f * h, f * g - d * i, d * h - e * g
        det = a * A + b * B + c * C
        jac[c0 : c0 + chunk] = det
        ok = det > 0
        rdet = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
        inv = np.empty((ne, nn, 9))
        inv[..., 0], inv[..., 1], inv[..., 2] = A * rdet, (c * h - b * i) * rdet, (b * f - c * e) * rdet
        inv[..., 3], inv[..., 4], inv[..., 5] = B * rdet, (a * i - c * g) * rdet, (c * d - a * f) * rdet
        inv[..., 6], inv[..., 7], inv[..., 8] = C * rdet, (b * g - a * h) * rdet, (a * e - b * d) * rdet
        dxi[c0 : c0 + chunk] = inv

    for_chunks(one, range(0, n_cell, chunk), threads)
    wijk = (w[:, None, None] * w[None, :, None] * w[None, None, :]).ravel()
    mass = jac * wijk[None, :]
    return (
        coords.reshape(n_cell, ng, ng, ng, 3),
        jac.reshape(n_cell, ng, ng, ng),
        dxi.reshape(n_cell, ng, ng, ng, 9),
        mass.reshape(n_cell, ng, ng, ng),
    )


def global_numbering(coords: np.ndarray):
    """ibool by quantised-coordinate lexsort (partition.py:192-254)."""
    n_cell, ng = coords.shape[0], coords.shape[1]
    nn = ng**3
    if n_cell == 0:
        return np.zeros((0, ng, ng, ng), dtype=np.int32), 0
    extent = float(
        max(
            coords[..., 0].max() - coords[..., 0].min(),
            coords[..., 1].max() - coords[..., 1].min(),
            coords[..., 2].max() - coords[..., 2].min(),
            np.finfo(np.float64).eps,
        )
    )
    tol = np.float64(1e-12 * extent)
    flat = coords.reshape(-1, 3)
    scale = np.float64(1.0) / tol
    q = np.rint(flat * scale).astype(np.int64)
    order = np.lexsort((q[:, 2], q[:, 1], q[:, 0]))
    sq = q[order]
    is_new = np.any(np.diff(sq, axis=0, prepend=sq[:1] - 1) != 0, axis=1)
    ids = np.cumsum(is_new, dtype=np.int32) - 1
    ibool = np.empty(n_cell * nn, dtype=np.int32)
    ibool[order] = ids
    return ibool.reshape(n_cell, ng, ng, ng), int(ids[-1]) + 1


def pml_flags(spec: MeshSpec) -> np.ndarray:
    """Structured PML expansion (cli.py:247-264); zmin is the free surface."""
    c = {k: int(spec.pml.get(k, 0)) for k in ("xmin", "xmax", "ymin", "ymax", "zmax")}
    e = np.arange(spec.n_cell)
    i, j, k = e % spec.nx, (e // spec.nx) % spec.ny, e // (spec.nx * spec.ny)
    return (
        (i < c["xmin"])
        | (i >= spec.nx - c["xmax"])
        | (j < c["ymin"])
        | (j >= spec.ny - c["ymax"])
        | (k >= spec.nz - c["zmax"])
    )


def legacy_damping(spec: MeshSpec, coords: np.ndarray, bounds: dict, is_pml: np.ndarray):
    """Linear-ramp damping profile (pml.py:23-124)."""
    n_cell = coords.shape[0]
    damping = np.zeros(coords.shape[:4])
    pairs = [("xmin", 0), ("xmax", 0), ("ymin", 1), ("ymax", 1), ("zmin", 2), ("zmax", 2)]
    lo = {0: "xmin", 1: "ymin", 2: "zmin"}
    hi = {0: "xmax", 1: "ymax", 2: "zmax"}
    for face, axis in pairs:
        th = int(spec.pml.get(face, 0))
        if th <= 0:
            continue
        extent = bounds[hi[axis]] - bounds[lo[axis]]
        ncell_approx = max(1, int(np.ceil(n_cell ** (1.0 / 3.0))))
        width = th * (extent / ncell_approx)
        if width <= 0:
            continue
        ca = coords[..., axis]
        bv = bounds[face]
        for e in np.nonzero(is_pml)[0]:
            if face.endswith("min"):
                start = bv + width
                emax = ca[e].max()
                if emax > start + 1e-12 and emax > bv + width + 1e-12:
                    continue
                ramp = np.clip((start - ca[e]) / width, 0.0, 1.0)
            else:
                start = bv - width
                if ca[e].min() < start - 1e-12:
                    continue
                ramp = np.clip((ca[e] - start) / width, 0.0, 1.0)
            damping[e] = np.maximum(damping[e], ramp)
    return damping


def _axis_active(region: np.ndarray, axis: int) -> np.ndarray:
    sets = {
        0: (CPML_X_ONLY, CPML_XY_ONLY, CPML_XZ_ONLY, CPML_XYZ),
        1: (CPML_Y_ONLY, CPML_XY_ONLY, CPML_YZ_ONLY, CPML_XYZ),
        2: (CPML_Z_ONLY, CPML_XZ_ONLY, CPML_YZ_ONLY, CPML_XYZ),
    }[axis]
    return np.isin(region, sets)


def cpml_regions(coords, is_pml, bounds, widths, tol=1e-6):
    """Region code per cell from its GLL-centroid (pml_cpml.py:174-253)."""
    n_cell = coords.shape[0]
    regions = np.zeros(n_cell, dtype=np.int32)
    idx = np.nonzero(is_pml)[0]
    if idx.size == 0:
        return regions
    ctr = coords[idx].mean(axis=(1, 2, 3))
    act = []
    for axis, (kmin, kmax) in enumerate((("xmin", "xmax"), ("ymin", "ymax"), ("zmin", "zmax"))):
        a = np.zeros(idx.size, dtype=bool)
        if widths.get(kmin, 0) > 0:
            a |= ctr[:, axis] < bounds[kmin] + widths[kmin] + tol * widths[kmin]
        if widths.get(kmax, 0) > 0:
            a |= ctr[:, axis] > bounds[kmax] - widths[kmax] - tol * widths[kmax]
        act.append(a)
    ax, ay, az = act
    r = np.full(idx.size, CPML_XYZ, dtype=np.int32)
    r[ax & ay & az] = CPML_XYZ
    r[ax & ay & ~az] = CPML_XY_ONLY
    r[ax & ~ay & az] = CPML_XZ_ONLY
    r[~ax & ay & az] = CPML_YZ_ONLY
    r[ax & ~ay & ~az] = CPML_X_ONLY
    r[~ax & ay & ~az] = CPML_Y_ONLY
    r[~ax & ~ay & az] = CPML_Z_ONLY
    regions[idx] = r
    return regions


def cpml_profiles(coords, is_pml, regions, bounds, widths, vp, f0):
    """K, d, alpha per node and axis (pml_cpml.py:42-147)."""
    n_cell, ng = coords.shape[0], coords.shape[1]
    nn = ng**3
    K = np.ones((n_cell, nn, 3))
    d = np.zeros((n_cell, nn, 3))
    al = np.zeros((n_cell, nn, 3))
    amax = [np.pi * f0 * 0.9, np.pi * f0 * 1.0, np.pi * f0 * 1.1]
    faces = [(0, "xmin"), (0, "xmax"), (1, "ymin"), (1, "ymax"), (2, "zmin"), (2, "zmax")]
    idx = np.nonzero(is_pml)[0]
    if idx.size == 0:
        return K, d, al
    cf = coords[idx].reshape(idx.size, nn, 3)
    vpf = vp[idx].reshape(idx.size, nn)
    reg = regions[idx]
    for axis, face in faces:
        width = widths.get(face, 0.0)
        if width <= 0:
            continue
        act = _axis_active(reg, axis)
        if not act.any():
            continue
        dist = np.clip(np.abs(cf[:, :, axis] - bounds[face]) / width, 0.0, 1.0)
        Kv = K_MIN_PML + (K_MAX_PML - 1.0) * dist
        dv = -((NPOWER + 1.0) * vpf * np.log(R_COEF) / (2.0 * width)) * np.power(dist, 1.2 * NPOWER)
        av = amax[axis] * (1.0 - dist)
        mask = (Kv < 1.0) | (dv < 0.0)
        Kv[mask] = 1.0
        dv[mask] = 0.0
        av = np.maximum(av, 0.0)
        # faces are applied in order; later faces of the same axis overwrite
        sel = idx[act]
        K[sel, :, axis] = Kv[act]
        d[sel, :, axis] = dv[act]
        al[sel, :, axis] = av[act]
    return K, d, al


def convolution_coef(b: np.ndarray, dt: float):
    """coef0, coef1, coef2 of the second-order recursive convolution
    (pml_cpml.py:261-305)."""
    b = np.atleast_1d(np.asarray(b, dtype=np.float64))
    temp = np.exp(-0.5 * b * dt)
    c0 = temp * temp
    large = np.abs(b) >= MIN_DISTANCE
    safe = np.where(large, b, 1.0)
    c1 = np.where(large, (1.0 - temp) / safe, 0.0)
    c2 = c1 * temp
    small = ~large
    if np.any(small):
        dt2, dt3, dt4 = dt * dt, dt * dt * dt, dt * dt * dt * dt
        bs = b[small]
        b2, b3 = bs * bs, bs * bs * bs
        c1[small] = dt * 0.5 + (-0.125 * dt2 * bs + (1.0 / 48.0) * dt3 * b2 - (1.0 / 384.0) * dt4 * b3)
        c2[small] = dt * 0.5 + (-0.375 * dt2 * bs + (7.0 / 48.0) * dt3 * b2 - (5.0 / 128.0) * dt4 * b3)
    return c0, c1, c2


def _safe(x):
    return np.where(np.abs(x) < MIN_DISTANCE, MIN_DISTANCE, x)


def abar_coefficients(K, d, al, regions):
    """A1..A5 per node (pml_cpml.py:353-515)."""
    n_cell, nn, _ = K.shape
    out = np.zeros((n_cell, nn, 5))
    for reg in range(1, 8):
        cells = np.nonzero(regions == reg)[0]
        if cells.size == 0:
            continue
        kx, ky, kz = K[cells, :, 0], K[cells, :, 1], K[cells, :, 2]
        dx, dy, dz = d[cells, :, 0], d[cells, :, 1], d[cells, :, 2]
        ax, ay, az = al[cells, :, 0], al[cells, :, 1], al[cells, :, 2]
        bx = ax + dx / np.maximum(kx, 1.0)
        by = ay + dy / np.maximum(ky, 1.0)
        bz = az + dz / np.maximum(kz, 1.0)
        zero = np.zeros_like(kx)
        if reg == CPML_XYZ:
            A0 = kx * ky * kz
            A1 = A0 * (bx + by + bz - ax - ay - az)
            A2 = A0 * (bx - ax) * (by - ay - ax) + A0 * (by - ay) * (bz - az - ay) + A0 * (bz - az) * (bx - ax - az)
            A3 = A0 * ax**2 * (bx - ax) * (by - ax) * (bz - ax) / (_safe(ay - ax) * _safe(az - ax))
            A4 = A0 * ay**2 * (bx - ay) * (by - ay) * (bz - ay) / (_safe(ax - ay) * _safe(az - ay))
            A5 = A0 * az**2 * (bx - az) * (by - az) * (bz - az) / (_safe(ay - az) * _safe(az - ax))
        elif reg == CPML_XY_ONLY:
            A0 = kx * ky
            A1 = A0 * (bx + by - ax - ay)
            A2 = A0 * (bx - ax) * (by - ay - ax) - A0 * (by - ay) * ay
            A3 = A0 * ax**2 * (bx - ax) * (by - ax) / _safe(ay - ax)
            A4 = A0 * ay**2 * (bx - ay) * (by - ay) / _safe(ax - ay)
            A5 = zero
        elif reg == CPML_XZ_ONLY:
            A0 = kx * kz
            A1 = A0 * (bx + bz - ax - az)
            A2 = A0 * (bx - ax) * (-ax) + A0 * (bz - az) * (bx - ax - az)
            A3 = A0 * ax**2 * (bx - ax) * (bz - ax) / _safe(az - ax)
            A4 = zero
            A5 = A0 * az**2 * (bx - az) * (bz - az) / _safe(ax - az)
        elif reg == CPML_YZ_ONLY:
            A0 = ky * kz
            A1 = A0 * (by + bz - ay - az)
            A2 = A0 * (by - ay) * (bz - az - ay) - A0 * (bz - az) * az
            A3 = zero
            A4 = A0 * ay**2 * (by - ay) * (bz - ay) / _safe(az - ay)
            A5 = A0 * az**2 * (by - az) * (bz - az) / _safe(ay - az)
        elif reg == CPML_X_ONLY:
            A0 = kx
            diff = bx - ax
            A1, A2, A3, A4, A5 = A0 * diff, -A0 * ax * diff, A0 * ax**2 * diff, zero, zero
        elif reg == CPML_Y_ONLY:
            A0 = ky
            diff = by - ay
            A1, A2, A3, A4, A5 = A0 * diff, -A0 * ay * diff, zero, A0 * ay**2 * diff, zero
        else:  # CPML_Z_ONLY
            A0 = kz
            diff = bz - az
            A1, A2, A3, A4, A5 = A0 * diff, -A0 * az * diff, zero, zero, A0 * az**2 * diff
        for c, A in enumerate((A1, A2, A3, A4, A5)):
            out[cells, :, c] = A
    return out


def cpml_parameters(coords, is_pml, bounds, widths, vp, f0, dt, threads: int = 1, chunk: int = 65536):
    """Region, coef_alpha [n_cell, nn, 9] and A1..A5 [n_cell, nn, 5]; every
    value depends on its own cell only, so ``threads`` > 1 computes chunks of
    cells on that many host threads with the same arithmetic."""
    n_cell = coords.shape[0]
    if threads <= 1 or n_cell <= chunk:
        return _cpml_parameters(coords, is_pml, bounds, widths, vp, f0, dt)
    nn = int(np.prod(coords.shape[1:-1]))
    region = np.empty(n_cell, dtype=np.int32)
    calpha = np.empty((n_cell, nn, 9))
    abar = np.empty((n_cell, nn, 5))

    def one(c0):
        sl = slice(c0, c0 + chunk)
        r, ca, ab = _cpml_parameters(coords[sl], is_pml[sl], bounds, widths, vp[sl], f0, dt)
        region[sl], calpha[sl], abar[sl] = r, ca, ab

    for_chunks(one, range(0, n_cell, chunk), threads)
    return region, calpha, abar


def _cpml_parameters(coords, is_pml, bounds, widths, vp, f0, dt):
    regions = cpml_regions(coords, is_pml, bounds, widths)
    K, d, al = cpml_profiles(coords, is_pml, regions, bounds, widths, vp, f0)
    n_cell, nn = K.shape[0], K.shape[1]
    # outside C-PML cells alpha = 0, whose coefficients are (1, dt/2, dt/2)
    # exactly (the |b| < MIN_DISTANCE series at b = 0)
    c0z, c1z, c2z = convolution_coef(np.zeros(1), dt)
    coef_alpha = np.empty((n_cell, nn, 9))
    for axis in range(3):
        coef_alpha[:, :, axis * 3 + 0] = c0z[0]
        coef_alpha[:, :, axis * 3 + 1] = c1z[0]
        coef_alpha[:, :, axis * 3 + 2] = c2z[0]
    idx = np.nonzero(is_pml)[0]
    for axis in range(3):
        if idx.size == 0:
            break
        c0, c1, c2 = convolution_coef(al[idx, :, axis], dt)
        coef_alpha[idx, :, axis * 3 + 0] = c0.reshape(idx.size, nn)
        coef_alpha[idx, :, axis * 3 + 1] = c1.reshape(idx.size, nn)
        coef_alpha[idx, :, axis * 3 + 2] = c2.reshape(idx.size, nn)
    abar = abar_coefficients(K, d, al, regions)
    return regions, coef_alpha, abar


def hex_newton(x_target, corners, max_iter=50, tol=1e-12):
    """Natural coordinates of a point in a trilinear hex (source_locator.py:74-123)."""
    xi = np.zeros(3)
    for _ in range(max_iter):
        fa = 1 + HEX_CORNERS[:, 0] * xi[0]
        fb = 1 + HEX_CORNERS[:, 1] * xi[1]
        fc = 1 + HEX_CORNERS[:, 2] * xi[2]
        Nv = 0.125 * fa * fb * fc
        dN = np.stack(
            [0.125 * HEX_CORNERS[:, 0] * fb * fc, 0.125 * fa * HEX_CORNERS[:, 1] * fc, 0.125 * fa * fb * HEX_CORNERS[:, 2]],
            axis=1,
        )
        res = x_target - Nv @ corners
        J = dN.T @ corners
        try:
            dxi = np.linalg.solve(J, res)
        except np.linalg.LinAlgError:
            return None
        xi = xi + dxi
        if np.linalg.norm(dxi) < tol:
            break
    else:
        return None
    if np.any(xi < -(1.0 + 1e-8)) or np.any(xi > 1.0 + 1e-8):
        return None
    return xi


def locate_point_source(coords, corners, source_xyz, is_pml, order):
    """Buried-mode source location: AABB candidates among non-PML cells,
    Newton, Lagrange weights normalised over all containing cells
    (source_locator.py:186-213, 295-375)."""
    ng = order + 1
    pts = gll_points(order)
    lo = coords.reshape(coords.shape[0], -1, 3).min(axis=1)
    hi = coords.reshape(coords.shape[0], -1, 3).max(axis=1)
    m = 1e-10
    cand = np.nonzero(np.all((lo - m <= source_xyz) & (source_xyz <= hi + m), axis=1) & ~is_pml)[0]
    ids, ws = [], []
    for e in cand:
        xi = hex_newton(np.asarray(source_xyz, dtype=np.float64), corners[e])
        if xi is None:
            continue
        lx, ly, lz = (lagrange_1d(xi[a], pts) for a in range(3))
        w = lx[:, None, None] * ly[None, :, None] * lz[None, None, :]
        if np.sum(w) < 1e-12:
            continue
        ids.append(int(e))
        ws.append(w)
    if not ids:
        raise ValueError(f"source {source_xyz} not inside any non-PML cell")
    total = float(sum(np.sum(w) for w in ws))
    return np.array(ids, dtype=np.int64), np.array([w / total for w in ws]).reshape(len(ids), ng, ng, ng)


def recording_map(coords, ibool, is_pml, bounds, record_depth_max_m, tile=None, nxy=None):
    """Recording cells and GLL node map (recording_map.py:18-170), single rank.

    ``tile`` = (i0, j0, n) records instead the top cell of each column
    i0..i0+n-1, j0..j0+n-1 (``nxy`` = (nx, ny) cells per row): a tile of n x n
    surface elements for strain Green's function extraction, which follows
    the free surface where it is not flat."""
    n_cell, ng = coords.shape[0], coords.shape[1]
    nn = ng**3
    zmin, zmax = bounds["zmin"], bounds["zmax"]
    target = zmin + record_depth_max_m
    cz = coords[..., 2].reshape(n_cell, nn)
    levels = np.concatenate([cz.min(axis=1), cz.max(axis=1)])
    levels = np.unique(levels[(levels >= zmin) & (levels <= zmax)])
    above = levels[levels >= target]
    actual = float(above[0] - zmin) if above.size else float(zmax - zmin)
    cen = coords.reshape(n_cell, nn, 3).mean(axis=1)
    sel = (~is_pml) & (cen[:, 2] <= zmin + actual + 1e-12)
    if tile is not None:
        i0, j0, n = tile
        e = np.arange(n_cell)
        ci, cj, ck = e % nxy[0], (e // nxy[0]) % nxy[1], e // (nxy[0] * nxy[1])
        sel = (~is_pml) & (ck == 0) & (ci >= i0) & (ci < i0 + n) & (cj >= j0) & (cj < j0 + n)
        actual = float((cz.max(axis=1) - cz.min(axis=1))[sel].max()) if sel.any() else 0.0
    rec_cell = np.nonzero(sel)[0].astype(np.int32)
    nodes = ibool.reshape(n_cell, nn)[rec_cell]
    gll_ids, first, inv = np.unique(nodes.ravel(), return_index=True, return_inverse=True)
    cell_index = inv.reshape(rec_cell.size, nn).astype(np.int32)
    flatc = coords.reshape(n_cell, nn, 3)[rec_cell].reshape(-1, 3)
    return {
        "record_depth_actual_m": actual,
        "rec_cell_local": rec_cell,
        "rec_cell_global": rec_cell.astype(np.int64),
        "gll_node_ids": gll_ids.astype(np.int64),
        "gll_node_coords": flatc[first],
        "cell_gll_node_index": cell_index,
    }


def ricker(t, f0=2.0, t0=1.0, amp=1.0e20):
    a = np.pi * f0 * (np.asarray(t) - t0)
    return amp * (1.0 - 2.0 * a**2) * np.exp(-(a**2))


def h_min(coords: np.ndarray, threads: int = 1, chunk: int = 65536) -> float:
    """Smallest distance between adjacent GLL nodes of any cell (cfl_validator.py:38-62)."""
    out = {}

    def one(c0):
        c = coords[c0 : c0 + chunk]
        best = np.inf
        for ax in (1, 2, 3):
            a = np.take(c, np.arange(1, c.shape[ax]), axis=ax)
            b = np.take(c, np.arange(0, c.shape[ax] - 1), axis=ax)
            best = min(best, float(np.sqrt(((a - b) ** 2).sum(-1)).min()))
        out[c0] = best

    for_chunks(one, range(0, coords.shape[0], chunk), threads)
    return min(out.values()) if out else np.inf


# ---------------------------------------------------------------------------
# Complete problem
# ---------------------------------------------------------------------------

MaterialFn = Callable[[np.ndarray], tuple]


def homogeneous(vp=6000.0, vs=3464.0, rho=2700.0) -> MaterialFn:
    def f(c):
        s = c.shape[:-1]
        return np.full(s, vp), np.full(s, vs), np.full(s, rho)

    return f


def layered(depths, vps, vss, rhos) -> MaterialFn:
    """Flat layers: layer i spans depths[i-1] <= z < depths[i] (z down)."""
    depths = np.asarray(depths, dtype=np.float64)

    def f(c):
        z = c[..., 2]
        li = np.searchsorted(depths, z, side="right")
        return np.asarray(vps)[li], np.asarray(vss)[li], np.asarray(rhos)[li]

    return f


def gaussian_field(lo, hi, corr_len: float, seed: int, spacing: Optional[float] = None):
    """Seeded random field with Gaussian correlation exp(-r^2/corr_len^2),
    unit variance, clipped to +-1, on a regular grid over the box [lo, hi];
    returns f(coords) -> values by trilinear interpolation.

    White noise filtered by a Gaussian kernel of standard deviation
    corr_len/2 has exactly that correlation function."""
    from scipy import ndimage

    lo, hi = np.asarray(lo, dtype=np.float64), np.asarray(hi, dtype=np.float64)
    h = spacing if spacing is not None else corr_len / 3.0
    shape = tuple(int(np.ceil((hi[a] - lo[a]) / h)) + 2 for a in range(3))
    rng = np.random.default_rng(seed)
    g = ndimage.gaussian_filter(rng.standard_normal(shape), sigma=0.5 * corr_len / h, mode="wrap")
    g = np.clip(g / g.std(), -1.0, 1.0)

    def f(c):
        flat = np.asarray(c, dtype=np.float64).reshape(-1, 3)
        out = np.empty(flat.shape[0])
        for a0 in range(0, flat.shape[0], 1 << 22):
            x = ((flat[a0 : a0 + (1 << 22)] - lo) / h).T
            out[a0 : a0 + (1 << 22)] = ndimage.map_coordinates(g, x, order=1, mode="nearest")
        return out.reshape(np.shape(c)[:-1])

    return f


def perturbed(base: "MaterialFn", field, amp: float = 0.1) -> "MaterialFn":
    """Background model with its velocities scaled by (1 + amp * field)."""

    def f(c):
        vp, vs, rho = base(c)
        s = 1.0 + amp * field(c)
        return vp * s, vs * s, rho

    return f


def seeded_layers(seed: int, lz: float, n_layers: int = 3):
    """Three flat layers with seeded interfaces and (vp, vp/vs, rho) in
    vp 3000-7000 m/s, vp/vs 1.6-1.9, rho 2200-3000 kg/m^3; vp grows with depth."""
    rng = np.random.default_rng(seed)
    depths = np.sort(rng.uniform(0.15, 0.85, size=n_layers - 1)) * lz
    vps = np.sort(rng.uniform(3000.0, 7000.0, size=n_layers))
    ratio = rng.uniform(1.6, 1.9, size=n_layers)
    rhos = np.sort(rng.uniform(2200.0, 3000.0, size=n_layers))
    return layered(depths, vps, vps / ratio, rhos)


def build_problem(
    spec: MeshSpec,
    material: MaterialFn,
    source_xyz,
    *,
    dt: Optional[float] = None,
    cfl: float = 0.5,
    nsteps: int = 100,
    snapshot_stride: int = 10,
    record_depth_max_m: float = 0.0,
    f0: float = 2.0,
    t0: float = 1.0,
    amp: float = 1.0e20,
    with_cpml: bool = True,
    record_tile=None,
    device: Optional[int] = None,
    numbering_device: Optional[int] = None,
    threads: int = 1,
    cell_window=None,
    require_source: bool = True,
) -> dict:
    """Every solver input for one synthetic model, reference layouts.

    ``device`` = a GPU index computes the GLL geometry, the node numbering
    and the C-PML coefficients there (``gfb.prep``) instead of on the host.
    ``numbering_device`` = a GPU index numbers the host-computed points there
    (the same ids as the host's lexsort of the same points, partition.py's
    rule, in a fraction of the time).  ``threads`` = host threads for the
    per-cell host stages (same values for any count).  ``cell_window`` =
    (i0, i1, j0, j1, k0, k1) keeps only the cells with i0 <= i < i1,
    j0 <= j < j1, k0 <= k < k1 of the full mesh (x fastest), a piece of the
    model with the full model's vertices, bounds and C-PML layers.  With
    ``require_source`` False a source outside every non-C-PML cell leaves the
    model without a source instead of raising."""
    if device is not None or numbering_device is not None:
        from . import prep
    V = vertex_grid(spec)
    corners = cell_corners(spec, V)
    is_pml = pml_flags(spec)
    n_cell = spec.n_cell
    if cell_window is not None:
        i0, i1, j0, j1, k0, k1 = cell_window
        if record_tile is not None:
            raise ValueError("a recording tile is defined on the full mesh")
        k, j, i = np.meshgrid(np.arange(k0, k1), np.arange(j0, j1), np.arange(i0, i1), indexing="ij")
        sel = (i.ravel() + spec.nx * (j.ravel() + spec.ny * k.ravel())).astype(np.int64)
        corners, is_pml, n_cell = corners[sel], is_pml[sel], int(sel.size)
    if device is None:
        coords, jac, dxi, mgeo = gll_geometry(corners, spec.order, threads=threads)
    else:
        coords, jac, dxi, mgeo = prep.gll_geometry(corners, spec.order, device=device)
    bounds = {
        "xmin": float(V[..., 0].min()),
        "xmax": float(V[..., 0].max()),
        "ymin": float(V[..., 1].min()),
        "ymax": float(V[..., 1].max()),
        "zmin": float(V[..., 2].min()),
        "zmax": float(V[..., 2].max()),
    }
    if threads > 1:
        vp, vs, rho = (np.empty(coords.shape[:-1]) for _ in range(3))

        def mat(c0, n=65536):
            vp[c0 : c0 + n], vs[c0 : c0 + n], rho[c0 : c0 + n] = material(coords[c0 : c0 + n])

        for_chunks(mat, range(0, coords.shape[0], 65536), threads)
    else:
        vp, vs, rho = material(coords)
    mu = rho * vs**2
    lam = rho * (vp**2 - 2.0 * vs**2)
    mass = mgeo * rho
    if dt is None:
        dt = cfl * h_min(coords, threads=threads) / float(vp.max())
    ndev = device if device is not None else numbering_device
    ibool, n_node = global_numbering(coords) if ndev is None else prep.global_numbering(coords, device=ndev)
    widths = {
        "xmin": spec.pml.get("xmin", 0) * (bounds["xmax"] - bounds["xmin"]) / spec.nx,
        "xmax": spec.pml.get("xmax", 0) * (bounds["xmax"] - bounds["xmin"]) / spec.nx,
        "ymin": spec.pml.get("ymin", 0) * (bounds["ymax"] - bounds["ymin"]) / spec.ny,
        "ymax": spec.pml.get("ymax", 0) * (bounds["ymax"] - bounds["ymin"]) / spec.ny,
        "zmin": spec.pml.get("zmin", 0) * (bounds["zmax"] - bounds["zmin"]) / spec.nz,
        "zmax": spec.pml.get("zmax", 0) * (bounds["zmax"] - bounds["zmin"]) / spec.nz,
    }
    out = {
        "spec": spec,
        "ngll": spec.order + 1,
        "n_cell": n_cell,
        "n_node": n_node,
        "bounds": bounds,
        "coords": coords,
        "jacobian": jac,
        "dxi_dx": dxi,
        "mass": mass,
        "vp": vp,
        "vs": vs,
        "density": rho,
        "lambda": lam,
        "mu": mu,
        "ibool": ibool,
        "cell_ids": np.arange(n_cell, dtype=np.int64),
        "is_pml": is_pml,
        "dt": float(dt),
        "nsteps": int(nsteps),
        "snapshot_stride": int(snapshot_stride),
    }
    if with_cpml:
        if device is None:
            region, calpha, abar = cpml_parameters(coords, is_pml, bounds, widths, vp, f0, dt, threads=threads)
        else:
            region, calpha, abar = prep.cpml_parameters(coords, is_pml, bounds, widths, vp, f0, dt, device=device)
        out["pml_region"] = region
        out["pml_coef_alpha"] = calpha.reshape(coords.shape[:4] + (9,))
        out["pml_coef_abar"] = abar.reshape(coords.shape[:4] + (5,))
        out["damping"] = np.zeros(coords.shape[:4])
    else:
        out["damping"] = legacy_damping(spec, coords, bounds, is_pml)
    try:
        src_ids, src_w = locate_point_source(coords, corners, source_xyz, is_pml, spec.order)
    except ValueError:
        if require_source:
            raise
        ng = spec.order + 1
        src_ids, src_w = np.zeros(0, dtype=np.int64), np.zeros((0, ng, ng, ng))
    out["src_cell_ids"] = src_ids
    out["src_weights"] = src_w
    t = np.arange(nsteps) * dt
    out["stf_t"] = t
    out["stf"] = ricker(t, f0=f0, t0=t0, amp=amp)
    if record_depth_max_m > 0.0:
        out["recording"] = recording_map(coords, ibool, is_pml, bounds, record_depth_max_m, tile=record_tile,
                                         nxy=(spec.nx, spec.ny))
    return out
