"""Input generator pins (no GPU).

The synthetic partition arrays produced by gfb.mesh are compared with the
arrays the reference preprocessor's own functions produced for the golden
cases (tests/golden/make_golden.py): integer maps bit-exact, floating-point
fields to a few ulp.  Property checks follow tests/preprocess/
test_partition.py:419-510 (ibool), test_recording_map.py (PML exclusion) and
test_source_locator.py (weights sum to one).
"""

import numpy as np
import pytest
from conftest import golden_cases, load_golden

from gfb import mesh


def regenerate(g):
    spec = mesh.MeshSpec(nx=int(g["nx"]), ny=int(g["ny"]), nz=int(g["nz"]), dx=float(g["d"]), dy=float(g["d"]),
                         dz=float(g["d"]), order=4, jitter=float(g["jitter"]), seed=int(g["seed"]),
                         pml={"xmin": 1, "xmax": 1, "ymin": 1, "ymax": 1, "zmax": 1})
    if bool(g["layered"]):
        mat = mesh.layered([400.0, 1000.0], [4000.0, 5500.0, 6500.0], [2300.0, 3100.0, 3600.0],
                           [2400.0, 2600.0, 2800.0])
    else:
        mat = mesh.homogeneous()
    return mesh.build_problem(spec, mat, g["src_xyz"], dt=float(g["dt"]), nsteps=int(g["nsteps"]),
                              snapshot_stride=int(g["stride"]), record_depth_max_m=float(g["depth"]),
                              with_cpml=bool(g["cpml"]))


def close(a, b, rtol=1e-14):
    a, b = np.asarray(a), np.asarray(b).reshape(np.shape(a))
    scale = max(np.abs(b).max(), 1e-300)
    assert np.abs(a - b).max() <= rtol * scale


@pytest.mark.parametrize("name", golden_cases())
def test_generator_matches_reference_preprocessor(name):
    g = load_golden(name)
    p = regenerate(g)
    np.testing.assert_array_equal(p["ibool"], g["ibool"])
    assert p["n_node"] == int(g["n_node"])
    for key, gk in (("coords", "coords"), ("jacobian", "jacobian"), ("dxi_dx", "dxi_dx"), ("mass", "mass"),
                    ("lambda", "lam"), ("mu", "mu"), ("damping", "damping")):
        close(p[key], g[gk], 1e-13)
    if bool(g["cpml"]):
        np.testing.assert_array_equal(p["pml_region"], g["pml_region"])
        close(p["pml_coef_alpha"], g["pml_coef_alpha"], 1e-13)
        close(p["pml_coef_abar"], g["pml_coef_abar"], 1e-13)
    np.testing.assert_array_equal(p["src_cell_ids"], g["src_cell_ids"])
    close(p["src_weights"], g["src_weights"], 1e-14)
    r = p["recording"]
    np.testing.assert_array_equal(r["rec_cell_local"], g["rec_cell_local"])
    np.testing.assert_array_equal(r["gll_node_ids"], g["gll_node_ids"])
    np.testing.assert_array_equal(r["cell_gll_node_index"], g["cell_gll_node_index"])
    close(r["gll_node_coords"], g["gll_node_coords"], 1e-14)
    assert r["record_depth_actual_m"] == pytest.approx(float(g["record_depth_actual_m"]), rel=1e-14)


def test_ibool_properties():
    spec = mesh.MeshSpec(nx=3, ny=2, nz=2, dx=1.0, dy=1.0, dz=1.0, order=4)
    V = mesh.vertex_grid(spec)
    coords, *_ = mesh.gll_geometry(mesh.cell_corners(spec, V), 4)
    ib, n = mesh.global_numbering(coords)
    # n equals the number of distinct GLL positions: (3*4+1)(2*4+1)(2*4+1)
    assert n == 13 * 9 * 9 == len(np.unique(ib))
    # a shared face gets the same ids: cell 0 (+x face) and cell 1 (-x face)
    np.testing.assert_array_equal(ib[0][4], ib[1][0])
    # zero cells
    z, nz = mesh.global_numbering(np.zeros((0, 5, 5, 5, 3)))
    assert nz == 0 and z.shape[0] == 0


def test_recording_excludes_pml_and_source_weights_sum_to_one():
    spec = mesh.MeshSpec(nx=5, ny=5, nz=3, dx=500.0, dy=500.0, dz=500.0, order=4,
                         pml={"xmin": 1, "xmax": 1, "ymin": 1, "ymax": 1, "zmax": 1})
    p = mesh.build_problem(spec, mesh.homogeneous(), np.array([1250.0, 1250.0, 250.0]), nsteps=5,
                           record_depth_max_m=300.0)
    rec = p["recording"]["rec_cell_local"]
    assert rec.size == 9 and not p["is_pml"][rec].any()
    assert abs(p["src_weights"].sum() - 1.0) < 1e-12
