"""CPU oracle pins (no GPU).

* The plain-C restatement (oracle/lib) is bit-identical to the reference's
  own compiled functions (oracle/_ref) on the golden fixtures.
* It reproduces the golden traces that the reference build produced.
* Known-answer tests of the reference suite, re-expressed:
  GLL tables (tests/test_gll.cpp:11-103) and the element kernel
  (tests/test_element.cpp:78-156).
"""

import os

import numpy as np
import pytest
from conftest import golden_cases, golden_problem, load_golden

import oracle
from gfb import mesh

HAVE_REF = os.path.exists(oracle.LIB_REF)


@pytest.mark.parametrize("name", golden_cases())
def test_oracle_reproduces_golden_traces_bit_exact(name):
    g = load_golden(name)
    prob = golden_problem(g)
    for d in g["dirs"]:
        run = oracle.Run(prob, int(d), "oracle")
        snaps = run.advance(int(g["nsteps"]))
        u, v, a = run.state()
        np.testing.assert_array_equal(snaps["steps"], g[f"trace_steps_{d}"])
        for key in ("strain", "u", "v", "a"):
            np.testing.assert_array_equal(snaps[key], g[f"trace_{key}_{d}"])
        np.testing.assert_array_equal(u, g[f"final_u_{d}"])
        np.testing.assert_array_equal(v, g[f"final_v_{d}"])
        np.testing.assert_array_equal(a, g[f"final_a_{d}"])


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built (needs the reference tree)")
def test_restatement_matches_reference_build_on_random_mesh():
    spec = mesh.MeshSpec(nx=4, ny=3, nz=3, dx=400.0, dy=450.0, dz=500.0, order=3, jitter=0.1, seed=3,
                         pml={"xmin": 1, "xmax": 1, "ymax": 1, "zmax": 1})
    prob = mesh.build_problem(spec, mesh.layered([700.0], [4000.0, 6000.0], [2300.0, 3400.0], [2300.0, 2700.0]),
                              np.array([820.0, 640.0, 530.0]), nsteps=40, snapshot_stride=7,
                              record_depth_max_m=600.0)
    for d in (0, 1, 2):
        a = oracle.Run(prob, d, "oracle", threads=3)
        b = oracle.Run(prob, d, "ref", threads=2)
        sa, sb = a.advance(40), b.advance(40)
        for k in ("strain", "u", "v", "a"):
            np.testing.assert_array_equal(sa[k], sb[k])
        for x, y in zip(a.state(), b.state()):
            np.testing.assert_array_equal(x, y)


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built (needs the reference tree)")
@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6])
def test_gll_tables_match_reference_build(N):
    for x, y in zip(oracle.gll(N, "oracle"), oracle.gll(N, "ref")):
        np.testing.assert_array_equal(x, y)


def test_gll_known_answers():
    x, w, D = oracle.gll(1)
    assert abs(x[0] + 1) < 1e-15 and abs(x[1] - 1) < 1e-15
    x, w, D = oracle.gll(2)
    np.testing.assert_allclose(x, [-1, 0, 1], atol=1e-15)
    np.testing.assert_allclose(w, [1 / 3, 4 / 3, 1 / 3], atol=1e-15)
    for N in (3, 4, 5):
        x, w, D = oracle.gll(N)
        assert np.all(np.diff(x) > 0)
        np.testing.assert_allclose(x + x[::-1], 0.0, atol=1e-14)
    for N in (1, 2, 3, 4, 5):
        assert abs(oracle.gll(N)[1].sum() - 2.0) < 1e-14
    for N in (2, 3, 4):
        assert np.abs(oracle.gll(N)[2].sum(axis=1)).max() < 1e-14
    # D differentiates polynomials of degree <= N exactly
    for N in (3, 4, 5):
        x, w, D = oracle.gll(N)
        for deg in range(N + 1):
            np.testing.assert_allclose(D @ x**deg, deg * x ** max(deg - 1, 0) if deg else 0 * x, atol=1e-12)


def unit_cube(N):
    """One element mapping [-1,1]^3 to [0,1]^3 (tests/test_element.cpp:15-75)."""
    x, w, D = oracle.gll(N)
    ng = N + 1
    nn = ng**3
    coords = np.zeros((nn, 3))
    for i in range(ng):
        for j in range(ng):
            for k in range(ng):
                coords[(i * ng + j) * ng + k] = 0.5 * (np.array([x[i], x[j], x[k]]) + 1.0)
    dxi = np.zeros((nn, 9))
    dxi[:, 0] = dxi[:, 4] = dxi[:, 8] = 2.0
    jac = np.full(nn, 0.125)
    vp, vs, rho = 3000.0, 1500.0, 2500.0
    mu = np.full(nn, rho * vs * vs)
    lam = np.full(nn, rho * (vp * vp - 2 * vs * vs))
    return coords, dxi, jac, lam, mu


def test_element_known_answers():
    N = 3
    coords, dxi, jac, lam, mu = unit_cube(N)
    nn = coords.shape[0]
    # rigid translation -> zero residual (test_element.cpp:78-100)
    u = np.tile([1.0, 2.0, 3.0], (nn, 1))
    r = oracle.element_residual(dxi, jac, lam, mu, u, N + 1)
    assert np.abs(r).max() < 1e-5
    # small rotation -> near-zero residual (102-125)
    th = 1e-6
    u = np.stack([-th * coords[:, 1], th * coords[:, 0], 0 * coords[:, 0]], axis=1)
    r = oracle.element_residual(dxi, jac, lam, mu, u, N + 1)
    assert np.abs(r).max() < 1e-6
    # uniaxial strain: internal forces self-equilibrate (127-156)
    u = np.stack([1e-3 * coords[:, 0], 0 * coords[:, 0], 0 * coords[:, 0]], axis=1)
    r = oracle.element_residual(dxi, jac, lam, mu, u, N + 1).reshape(-1, 3)
    assert abs(r[:, 0].sum()) < 1e-8
