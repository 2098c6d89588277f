"""Mesh inputs computed on the GPU (gfb.prep) against the host generator
(gfb.mesh), which follows the reference preprocessor.

* node numbering: bit-exact (integer map) on the same points, including
  point clouds with many coincident points and a single cell;
* GLL geometry: the trilinear map's sums are rounded in a fixed order on the
  device and by BLAS on the host, so coordinates, det J, inv(J) and mass agree
  to 1e-13 relative (max |diff| / max |value| per array); the device's
  coordinates of a shared point are bit-identical in every cell holding it;
* C-PML: region codes bit-exact; coef_alpha and A1..A5 to 1e-12 relative
  (exp, log and pow of the two math libraries differ in the last bits);
* a whole problem built on the GPU numbers its nodes as the host build does
  (on a mesh where the host build has no split node), and the solver's FP64
  traces from the two builds agree to 1e-12."""

import numpy as np
import pytest

import gfb
from gfb import mesh, prep

pytestmark = pytest.mark.gpu

GEOM_TOL = 1e-13
CPML_TOL = 1e-12


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def spec_of(nx, ny, nz, seed, jitter=0.1, topo=0, pml=None):
    return mesh.MeshSpec(nx=nx, ny=ny, nz=nz, dx=500.0, dy=400.0, dz=300.0, order=4, jitter=jitter,
                         topo_terms=topo, topo_amp=150.0 if topo else 0.0, seed=seed,
                         pml=pml if pml is not None else {"xmin": 2, "xmax": 2, "ymin": 2, "ymax": 2, "zmax": 2})


@pytest.mark.parametrize("order", [2, 4, 5])
def test_geometry_matches_host(order):
    spec = spec_of(9, 7, 6, seed=5, topo=3)
    spec.order = order
    corners = mesh.cell_corners(spec, mesh.vertex_grid(spec))
    ref = mesh.gll_geometry(corners, order)
    got = prep.gll_geometry(corners, order)
    for name, a, b in zip(("coords", "jacobian", "dxi_dx", "mass"), got, ref):
        assert a.shape == b.shape
        assert rel(a, b) <= GEOM_TOL, name


@pytest.mark.parametrize("seed", [0, 1])
def test_numbering_bit_exact_on_mesh_points(seed):
    spec = spec_of(8, 6, 5, seed=seed, topo=2)
    corners = mesh.cell_corners(spec, mesh.vertex_grid(spec))
    coords = mesh.gll_geometry(corners, 4)[0]
    ref, n_ref = mesh.global_numbering(coords)
    got, n_got = prep.global_numbering(coords)
    assert n_got == n_ref
    np.testing.assert_array_equal(got, ref)


def test_gpu_coordinates_number_every_shared_point_once():
    """The device evaluates the trilinear map one axis at a time, so the
    copies of a shared point are bit-identical and the quantised sort gives
    exactly (order n + 1) nodes per axis.  The host generator adds the four
    face corners in a cell-dependent order, as the reference's one-sum form
    does; on this mesh one shared point's copies round to two grid values."""
    spec = spec_of(20, 18, 9, seed=3, jitter=0.1, topo=8)
    corners = mesh.cell_corners(spec, mesh.vertex_grid(spec))
    exact = (4 * 20 + 1) * (4 * 18 + 1) * (4 * 9 + 1)
    _, n_dev = prep.global_numbering(prep.gll_geometry(corners, 4)[0])
    _, n_host = mesh.global_numbering(mesh.gll_geometry(corners, 4)[0])
    assert n_dev == exact
    assert n_host >= exact


def test_numbering_bit_exact_on_point_clouds():
    rng = np.random.default_rng(7)
    # coincident points (a coarse integer lattice) in random order, negative
    # coordinates included, as cells of 2x2x2 points
    base = rng.integers(-40, 40, size=(4096 * 8, 3)) * 0.37
    cloud = base.reshape(-1, 2, 2, 2, 3)
    ref, n_ref = mesh.global_numbering(cloud)
    got, n_got = prep.global_numbering(cloud)
    assert n_got == n_ref and n_ref < cloud.size // 3
    np.testing.assert_array_equal(got, ref)
    one = cloud[:1]
    r1, m1 = mesh.global_numbering(one)
    g1, k1 = prep.global_numbering(one)
    assert k1 == m1
    np.testing.assert_array_equal(g1, r1)


@pytest.mark.parametrize("pml", [{"xmin": 2, "xmax": 2, "ymin": 2, "ymax": 2, "zmax": 2},
                                 {"xmin": 1, "xmax": 3, "ymin": 2, "ymax": 1, "zmin": 1, "zmax": 2},
                                 {"xmax": 2}])
def test_cpml_matches_host(pml):
    spec = spec_of(10, 9, 8, seed=3, jitter=0.05, pml=pml)
    V = mesh.vertex_grid(spec)
    corners = mesh.cell_corners(spec, V)
    coords = mesh.gll_geometry(corners, 4)[0]
    bounds = {"xmin": float(V[..., 0].min()), "xmax": float(V[..., 0].max()),
              "ymin": float(V[..., 1].min()), "ymax": float(V[..., 1].max()),
              "zmin": float(V[..., 2].min()), "zmax": float(V[..., 2].max())}
    ext = {"x": spec.nx, "y": spec.ny, "z": spec.nz}
    widths = {f: pml.get(f, 0) * (bounds[f[0] + "max"] - bounds[f[0] + "min"]) / ext[f[0]]
              for f in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")}
    vp, _, _ = mesh.seeded_layers(3, spec.nz * spec.dz)(coords)
    is_pml = mesh.pml_flags(spec)
    if "zmin" in pml:  # the generator's flags leave zmin out (free surface); mark it here
        k = np.arange(spec.n_cell) // (spec.nx * spec.ny)
        is_pml = is_pml | (k < pml["zmin"])
    dt = 0.004
    r0, a0, b0 = mesh.cpml_parameters(coords, is_pml, bounds, widths, vp, 2.0, dt)
    r1, a1, b1 = prep.cpml_parameters(coords, is_pml, bounds, widths, vp, 2.0, dt)
    np.testing.assert_array_equal(r1, r0)
    assert rel(a1, a0) <= CPML_TOL
    assert rel(b1, b0) <= CPML_TOL
    if len(pml) == 6:
        assert set(np.unique(r0[r0 > 0])) == set(range(1, 8))  # every region type covered


def test_problem_built_on_gpu_runs_like_host_build():
    spec = spec_of(7, 6, 5, seed=9, topo=2, pml={"xmin": 1, "xmax": 1, "ymin": 1, "ymax": 1, "zmax": 1})
    mat = mesh.seeded_layers(9, spec.nz * spec.dz)
    src = np.array([1700.0, 1200.0, 800.0])
    host = mesh.build_problem(spec, mat, src, nsteps=60, snapshot_stride=10, record_depth_max_m=300.0)
    dev = mesh.build_problem(spec, mat, src, nsteps=60, snapshot_stride=10, record_depth_max_m=300.0, device=0)
    assert dev["n_node"] == host["n_node"]
    np.testing.assert_array_equal(dev["ibool"], host["ibool"])
    np.testing.assert_array_equal(dev["pml_region"], host["pml_region"])
    for name in ("dxi_dx", "jacobian", "mass"):
        assert rel(dev[name], host[name]) <= GEOM_TOL, name
    # here the C-PML inputs come from each build's own coordinates, which
    # differ in the last bits; A3..A5 divide by differences of alpha
    # profiles that vanish together at the outer boundary, which amplifies
    # those bits (up to ~3e-10 seen on a 32x32x16 deformed mesh)
    assert rel(dev["pml_coef_alpha"], host["pml_coef_alpha"]) <= CPML_TOL
    assert rel(dev["pml_coef_abar"], host["pml_coef_abar"]) <= 1e-9
    out = []
    for p in (host, dev):
        s = gfb.Solver(p, dirs=[0, 2], precision=gfb.FP64)
        s.advance(60)
        out.append((s.drain(), s.state(1)))
        s.close()
    (ra, sa), (rb, sb) = out
    for f in (0, 1):
        for name in ("strain", "u"):
            assert rel(rb[f][name], ra[f][name]) <= 1e-12, name
    for x, y in zip(sb, sa):
        assert rel(x, y) <= 1e-12
