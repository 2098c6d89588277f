"""GPU parity tests: the CUDA path through the C ABI against the CPU oracle.

Tolerances (stated by the spec of this path):
  * FP64 path: relative L2 <= 1e-10 on recorded traces and final state;
    element kernel max relative difference <= 1e-12
    (the reference's own CUDA-vs-CPU bound, tests/test_element_cuda.cu:99-136);
  * FP32 batched path: relative L2 <= 1e-4 against the FP64 oracle.
Integer/map outputs (snapshot step indices) are compared exactly.
"""

import numpy as np
import pytest
from conftest import golden_cases, golden_problem, load_golden, rel_l2

import gfb
import oracle
from gfb import mesh

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_TOL = 1e-4


def random_elements(ngll, n_elem, seed):
    """Random elements by the rules of tests/test_element_cuda.cu:35-95."""
    rng = np.random.default_rng(seed)
    nn = ngll**3
    P = n_elem * nn
    dxi = rng.uniform(-1, 1, (P, 9))
    dxi[:, 0] += 3.0
    dxi[:, 4] += 3.0
    dxi[:, 8] += 3.0
    jac = np.abs(rng.uniform(-1, 1, P)) + 0.01
    vp = np.abs(rng.uniform(-1, 1, P)) + 1000.0
    vs = np.abs(rng.uniform(-1, 1, P)) + 500.0
    rho = np.abs(rng.uniform(-1, 1, P)) + 1000.0
    mu = rho * vs * vs
    lam = rho * (vp * vp - 2.0 * vs * vs)
    u = rng.uniform(-1, 1, (P, 3))
    return dxi, jac, lam, mu, u


@pytest.mark.parametrize("ngll", [3, 4, 5, 6])
def test_element_kernel_fp64_matches_oracle(ngll):
    dxi, jac, lam, mu, u = random_elements(ngll, 7, 123 + ngll)
    ref = oracle.element_residual(dxi, jac, lam, mu, u, ngll)
    got = gfb.element_residual(dxi, jac, lam, mu, u, ngll, gfb.FP64)
    rel = np.abs(got - ref).max() / np.abs(ref).max()
    assert rel < 1e-12, rel


@pytest.mark.parametrize("n_elem,prec", [(262, gfb.FP64), (300, gfb.FP64), (600, gfb.FP32), (2000, gfb.FP32)])
def test_element_kernel_sizes_around_the_host_copy_staging(n_elem, prec):
    """Inputs of about 1 MB, where a pageable-memory copy used to return
    before reaching the device and the kernel read a stale tail."""
    dxi, jac, lam, mu, u = random_elements(5, n_elem, 11)
    ref = oracle.element_residual(dxi, jac, lam, mu, u, 5)
    got = gfb.element_residual(dxi, jac, lam, mu, u, 5, prec)
    tol = 1e-12 if prec == gfb.FP64 else 1e-5
    assert np.abs(got - ref).max() / np.abs(ref).max() < tol


@pytest.mark.parametrize("ngll", [4, 5])
def test_element_kernel_fp32_and_rigid_translation(ngll):
    dxi, jac, lam, mu, u = random_elements(ngll, 5, 7)
    ref = oracle.element_residual(dxi, jac, lam, mu, u, ngll)
    got = gfb.element_residual(dxi, jac, lam, mu, u, ngll, gfb.FP32)
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-5
    # rigid translation gives a zero residual (tests/test_element_cuda.cu:168-187)
    ut = np.tile([1.0, -2.0, 0.5], (u.shape[0], 1))
    r = gfb.element_residual(dxi, jac, lam, mu, ut, ngll, gfb.FP64)
    scale = np.abs(gfb.element_residual(dxi, jac, lam, mu, u, ngll, gfb.FP64)).max()
    assert np.abs(r).max() < 1e-10 * scale


def compare_runs(gpu_snaps, orc_snaps, tol, what=""):
    np.testing.assert_array_equal(np.asarray(gpu_snaps["steps"]), orc_snaps["steps"])
    for k in ("strain", "u", "v", "a"):
        e = rel_l2(gpu_snaps[k], orc_snaps[k])
        assert e <= tol, f"{what} {k}: rel L2 {e:.3e} > {tol}"


@pytest.mark.parametrize("name", golden_cases())
def test_time_loop_fp64_matches_golden_traces(name):
    g = load_golden(name)
    prob = golden_problem(g)
    for d in g["dirs"]:
        s = gfb.Solver(prob, dirs=[int(d)], precision=gfb.FP64)
        s.advance(int(g["nsteps"]))
        snaps = s.drain()[0]
        gold = {k: g[f"trace_{k}_{d}"] for k in ("strain", "u", "v", "a")}
        gold["steps"] = g[f"trace_steps_{d}"]
        compare_runs(snaps, gold, FP64_TOL, f"{name} dir {d}")
        u, v, a = s.state(0)
        assert rel_l2(u, g[f"final_u_{d}"]) <= FP64_TOL
        assert rel_l2(v, g[f"final_v_{d}"]) <= FP64_TOL
        assert rel_l2(a, g[f"final_a_{d}"]) <= FP64_TOL
        s.close()


def layered_problem(nsteps=120, jitter=0.08, order=4, cpml=True, seed=5):
    spec = mesh.MeshSpec(nx=6, ny=5, nz=4, dx=500.0, dy=500.0, dz=500.0, order=order, jitter=jitter, seed=seed,
                         pml={"xmin": 1, "xmax": 1, "ymin": 1, "ymax": 1, "zmax": 1})
    mat = mesh.layered([600.0, 1300.0], [3500.0, 5000.0, 6500.0], [2000.0, 2900.0, 3700.0], [2300.0, 2550.0, 2800.0])
    return mesh.build_problem(spec, mat, np.array([1430.0, 1270.0, 620.0]), nsteps=nsteps, snapshot_stride=10,
                              record_depth_max_m=500.0, with_cpml=cpml)


def oracle_snaps(prob, d, nsteps):
    run = oracle.Run(prob, d, "oracle", threads=4)
    snaps = run.advance(nsteps)
    return snaps, run.state()


def test_three_wavefields_fp64_match_three_oracle_runs():
    prob = layered_problem()
    n = prob["nsteps"]
    s = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP64)
    s.advance(n)
    snaps = s.drain()
    for d in range(3):
        ref, (u, v, a) = oracle_snaps(prob, d, n)
        compare_runs(snaps[d], ref, FP64_TOL, f"field {d}")
        gu, gv, ga = s.state(d)
        assert rel_l2(gu, u) <= FP64_TOL and rel_l2(gv, v) <= FP64_TOL and rel_l2(ga, a) <= FP64_TOL


def test_fp32_batched_within_1e4_of_fp64_oracle():
    prob = layered_problem(nsteps=300)
    n = prob["nsteps"]
    s = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32)
    s.advance(n)
    snaps = s.drain()
    for d in range(3):
        ref, _ = oracle_snaps(prob, d, n)
        compare_runs(snaps[d], ref, FP32_TOL, f"fp32 field {d}")


def deformed_problem(nsteps):
    """Jittered interior vertices, sinusoid topography, a Gaussian-correlated
    velocity perturbation and a recording tile that follows the surface (the
    construction of the 128 x 128 x 64 deformed workload at 7 x 6 x 5 cells)."""
    spec = mesh.MeshSpec(nx=7, ny=6, nz=5, dx=200.0, dy=200.0, dz=200.0, order=4, jitter=0.1, topo_terms=8,
                         topo_amp=150.0, seed=9, pml={"xmin": 1, "xmax": 1, "ymin": 1, "ymax": 1, "zmax": 1})
    field = mesh.gaussian_field((-200.0, -200.0, -200.0), (1600.0, 1400.0, 1500.0), 150.0, 10)
    mat = mesh.perturbed(mesh.seeded_layers(9, 1000.0), field, 0.1)
    return mesh.build_problem(spec, mat, np.array([700.0, 600.0, 450.0]), nsteps=nsteps, snapshot_stride=10,
                              record_depth_max_m=200.0, record_tile=(1, 1, 4))


def test_fp32_deformed_perturbed_mesh_within_1e4_of_fp64_oracle():
    prob = deformed_problem(250)
    assert prob["recording"]["rec_cell_local"].size == 16
    n = prob["nsteps"]
    s = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32)
    s.advance(n)
    snaps = s.drain()
    for d in range(3):
        ref, _ = oracle_snaps(prob, d, n)
        compare_runs(snaps[d], ref, FP32_TOL, f"deformed fp32 field {d}")


def test_fp32_node_and_cell_cpml_forms_agree():
    """The FP32 path keeps C-PML memory per global node when the cells agree
    on each axis's coefficients at shared nodes; the per-cell form
    (GFB_FLAG_CELL_PML, the reference's pml.cpp:112-216 layout) must give the
    same traces to FP32 rounding, and both stay within 1e-4 of the oracle."""
    prob = layered_problem(nsteps=200)
    n = prob["nsteps"]
    node = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32)
    cell = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32, flags=gfb.FLAG_CELL_PML)
    assert node.info()["n_pml_node"] > 0 and cell.info()["n_pml_node"] == 0
    node.advance(n)
    cell.advance(n)
    a, b = node.drain(), cell.drain()
    for d in range(3):
        ref, _ = oracle_snaps(prob, d, n)
        compare_runs(a[d], ref, FP32_TOL, f"node-cpml field {d}")
        for k in ("u", "strain"):
            assert rel_l2(a[d][k], b[d][k]) < 1e-5


def test_float32_snapshots_and_a_concurrent_reader():
    """Snapshots stored as float (snapshot_precision = "float32") match the
    double ones to float rounding; a reader thread draining snapshots while
    gfb_advance runs receives every one, in step order."""
    import threading

    prob = layered_problem(nsteps=150)
    a = gfb.Solver(prob, dirs=[0, 2], precision=gfb.FP32, record_slots=2)
    b = gfb.Solver(prob, dirs=[0, 2], precision=gfb.FP32, record_slots=2, flags=gfb.FLAG_RECORD_F32)
    got, stop = [], threading.Event()

    def reader():
        while not stop.is_set() or b.pending() > 0:
            if b.pending() > 0:
                got.append((b.read_record(0), b.read_record(1)))

    th = threading.Thread(target=reader)
    th.start()
    b.advance(150)
    b.synchronize()
    stop.set()
    th.join()
    a.advance(150)
    ref = a.drain()
    assert [r0["step"] for r0, _ in got] == list(ref[0]["steps"])
    for n, (r0, r1) in enumerate(got):
        for f, r in ((0, r0), (1, r1)):
            for k in ("u", "strain"):
                x, y = r[k], ref[f][k][n]
                assert np.abs(x - y).max() <= 1e-6 * np.abs(y).max() + 1e-30


def test_node_cpml_falls_back_when_cell_coefficients_disagree():
    prob = layered_problem(nsteps=40)
    nc = prob["n_cell"]
    alpha = prob["pml_coef_alpha"].copy().reshape(nc, -1, 9)
    A3 = prob["pml_coef_abar"].reshape(nc, -1, 5)[:, :, 2]
    ib = prob["ibool"].reshape(nc, -1)
    # a cell whose x-axis memory term (A3) is live at a node it shares with
    # another cell where it is live too; perturb that cell's x coefficients
    live = np.zeros(prob["n_node"], dtype=int)
    np.add.at(live, ib[A3 != 0], 1)
    e = next(c for c in range(nc) if np.any(live[ib[c][A3[c] != 0]] > 1))
    alpha[e, :, 1] *= 1.01
    prob["pml_coef_alpha"] = alpha
    s = gfb.Solver(prob, dirs=[0], precision=gfb.FP32)
    assert s.info()["n_pml_node"] == 0
    s.advance(40)
    ref, _ = oracle_snaps(prob, 0, 40)
    compare_runs(s.drain()[0], ref, FP32_TOL, "fallback")


@pytest.mark.parametrize("prec", [gfb.FP64, gfb.FP32])
def test_fused_node_update_equals_separate_pass(prec):
    """Finalising each node in the element kernel of the highest colour that
    touches it computes the same expressions as the separate node pass."""
    prob = layered_problem(nsteps=70)
    runs = []
    # the fused update lives in the thread-per-point kernel; compare with the
    # same kernel and a separate node pass, both evaluating the element force
    # in full every step (the fused update always does)
    for flags in (gfb.FLAG_POINT_KERNEL | gfb.FLAG_DIRECT_FORCE, gfb.FLAG_FUSED_NODE):
        s = gfb.Solver(prob, dirs=[0, 1, 2], precision=prec, flags=flags)
        s.advance(70)
        runs.append((s.drain(), [s.state(f) for f in range(3)]))
        s.close()
    (a, sa), (b, sb) = runs
    for f in range(3):
        for k in ("strain", "u", "v", "a"):
            np.testing.assert_array_equal(a[f][k], b[f][k])
        for x, y in zip(sa[f], sb[f]):
            np.testing.assert_array_equal(x, y)


def test_fp32_line_and_point_kernels_agree():
    """The FP32 path's thread-per-xi-line element kernel and the thread-per-
    point kernel compute the same sums in a different order: traces agree to
    FP32 rounding and both stay within 1e-4 of the oracle."""
    prob = layered_problem(nsteps=200)
    n = prob["nsteps"]
    runs = []
    for flags in (0, gfb.FLAG_POINT_KERNEL):
        s = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32, flags=flags)
        s.advance(n)
        runs.append(s.drain())
        s.close()
    line, point = runs
    for d in range(3):
        ref, _ = oracle_snaps(prob, d, n)
        compare_runs(line[d], ref, FP32_TOL, f"line kernel field {d}")
        compare_runs(point[d], ref, FP32_TOL, f"point kernel field {d}")
        for k in ("u", "strain"):
            assert rel_l2(line[d][k], point[d][k]) < 1e-5


@pytest.mark.parametrize("dirs", [[2], [0, 1], [0, 1, 2]])
def test_fp32_line_kernel_variants_agree(dirs):
    """Every variant of the line kernel at order 4: the default (line-owner
    exchange) and, with the exchange done by every thread, cells per group
    fewer, more and default (the same sums in the same order per xi-line:
    bit-identical to each other; the line owners add the eta and zeta sums
    in another order: within 1e-5); all within 1e-4 of the oracle; and
    kernels switched between steps."""
    n = 120
    prob = layered_problem(nsteps=n)
    runs = {}
    s = gfb.Solver(prob, dirs=dirs, precision=gfb.FP32)
    n_var = s.info()["n_elem_variants"]
    s.close()
    assert n_var == 4
    for v in range(n_var):
        s = gfb.Solver(prob, dirs=dirs, precision=gfb.FP32)
        s.select_element_kernel(v)
        assert s.info()["elem_variant"] == v
        s.advance(n)
        runs[v] = s.drain()
        s.close()
    for f, d in enumerate(dirs):
        ref, _ = oracle_snaps(prob, d, n)
        compare_runs(runs[0][f], ref, FP32_TOL, f"line-owner exchange field {d}")
        compare_runs(runs[3][f], ref, FP32_TOL, f"exchange by every thread field {d}")
        for v in (1, 2):
            for k in ("strain", "u", "v", "a"):
                np.testing.assert_array_equal(runs[v][f][k], runs[3][f][k], err_msg=f"variant {v} {k}")
        for k in ("u", "strain"):
            assert rel_l2(runs[0][f][k], runs[3][f][k]) < 1e-5
    # switching kernels between steps (the next step evaluates in full, off
    # the refresh schedule): still within 1e-4 of the oracle
    s = gfb.Solver(prob, dirs=dirs, precision=gfb.FP32)
    s.advance(n // 3)
    s.select_element_kernel(3)
    s.advance(n // 3)
    s.select_element_kernel(-1)
    assert s.info()["elem_variant"] == -1
    s.advance(n - 2 * (n // 3))
    mixed = s.drain()
    s.close()
    for f, d in enumerate(dirs):
        ref, _ = oracle_snaps(prob, d, n)
        compare_runs(mixed[f], ref, FP32_TOL, f"switched kernels field {d}")


def test_element_kernel_selection_is_checked():
    prob = layered_problem(nsteps=10)
    s = gfb.Solver(prob, dirs=[0], precision=gfb.FP32)
    for bad in (-2, s.info()["n_elem_variants"]):
        with pytest.raises(gfb.GfbError, match="out of range"):
            s.select_element_kernel(bad)
    s.close()
    s = gfb.Solver(prob, dirs=[0], precision=gfb.FP64)
    assert s.info()["n_elem_variants"] == 0 and s.info()["elem_variant"] == -1
    with pytest.raises(gfb.GfbError, match="one element kernel"):
        s.select_element_kernel(0)
    s.close()


@pytest.mark.parametrize("order,dirs", [(2, [1]), (3, [0, 2]), (5, [0, 1, 2]), (4, [2])])
def test_fp32_line_kernel_orders_and_field_counts(order, dirs):
    """Every (order, wavefield count) shape of the line kernel: its cells per
    group and thread count change with both."""
    n = 80
    prob = layered_problem(nsteps=n, order=order)
    s = gfb.Solver(prob, dirs=dirs, precision=gfb.FP32)
    s.advance(n)
    snaps = s.drain()
    for f, d in enumerate(dirs):
        ref, _ = oracle_snaps(prob, d, n)
        compare_runs(snaps[f], ref, FP32_TOL, f"order {order} field {d}")


@pytest.mark.parametrize("prec", [gfb.FP64, gfb.FP32])
def test_assembly_is_bit_reproducible(prec):
    prob = layered_problem(nsteps=60)
    out = []
    for _ in range(2):
        s = gfb.Solver(prob, dirs=[0, 2], precision=prec)
        s.advance(60)
        out.append((s.drain(), s.state(1)))
        s.close()
    (a, sa), (b, sb) = out
    for f in (0, 1):
        for k in ("strain", "u", "v", "a"):
            np.testing.assert_array_equal(a[f][k], b[f][k])
    for x, y in zip(sa, sb):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("order", [2, 3, 5])
def test_other_polynomial_orders_fp64(order):
    prob = layered_problem(nsteps=50, order=order)
    s = gfb.Solver(prob, dirs=[1], precision=gfb.FP64)
    s.advance(50)
    ref, (u, v, a) = oracle_snaps(prob, 1, 50)
    compare_runs(s.drain()[0], ref, FP64_TOL, f"order {order}")


def test_edge_cases_fp64():
    """Legacy ramp damping (no C-PML), mu <= 0 nodes skipped
    (element_cpu.cpp:42-43), a zero-mass node held at a = 0
    (solver.cpp:58-61), an STF shorter than the run (solver.cpp:579-582) and a
    source cell absent from the mesh (solver.cpp:584-587)."""
    prob = layered_problem(nsteps=80, cpml=False)
    assert prob["damping"].max() > 0
    mu = prob["mu"].copy()
    mu.reshape(prob["n_cell"], -1)[7, :11] = 0.0
    prob["mu"] = mu
    mass = prob["mass"].copy().reshape(prob["n_cell"], -1)
    ib = prob["ibool"].reshape(prob["n_cell"], -1)
    g0 = ib[3, 62]
    mass[ib == g0] = 0.0
    prob["mass"] = mass
    prob["stf"] = prob["stf"][:55]
    prob["src_cell_ids"] = np.concatenate([prob["src_cell_ids"], [10**9]])
    prob["src_weights"] = np.concatenate([prob["src_weights"], prob["src_weights"][:1]])
    s = gfb.Solver(prob, dirs=[2], precision=gfb.FP64)
    s.advance(80)
    ref, (u, v, a) = oracle_snaps(prob, 2, 80)
    compare_runs(s.drain()[0], ref, FP64_TOL, "edge")
    gu, gv, ga = s.state(0)
    assert rel_l2(gu, u) <= FP64_TOL and rel_l2(gv, v) <= FP64_TOL
    assert np.all(ga[g0] == 0.0)


def test_resume_from_state_matches_uninterrupted_run():
    prob = layered_problem(nsteps=90, cpml=False)
    full = gfb.Solver(prob, dirs=[0], precision=gfb.FP64, record=False)
    full.advance(90)
    first = gfb.Solver(prob, dirs=[0], precision=gfb.FP64, record=False)
    first.advance(40)
    u, v, a = first.state(0)
    second = gfb.Solver(prob, dirs=[0], precision=gfb.FP64, record=False)
    second.set_state(0, 40, u, v, a)
    assert second.step == 40
    second.advance(50)
    for x, y in zip(second.state(0), full.state(0)):
        np.testing.assert_allclose(x, y, rtol=1e-12, atol=1e-12 * np.abs(y).max())


def two_positions():
    """The layered 6 x 5 x 4 problem with a second point force at another
    position (its own cells, weights and a Ricker of another frequency)."""
    prob = layered_problem(nsteps=120)
    other = layered_problem(nsteps=120)
    spec = other["spec"]
    src2 = mesh.locate_point_source(other["coords"], mesh.cell_corners(spec, mesh.vertex_grid(spec)),
                                    np.array([2150.0, 1020.0, 880.0]), other["is_pml"], spec.order)
    s2 = {"src_cell_ids": src2[0], "src_weights": src2[1],
          "stf": mesh.ricker(np.arange(120) * prob["dt"], f0=2.7, t0=0.8)}
    s1 = {k: prob[k] for k in ("src_cell_ids", "src_weights", "stf")}
    return prob, [s1, s2]


@pytest.mark.parametrize("prec,tol", [(gfb.FP64, FP64_TOL), (gfb.FP32, FP32_TOL)])
def test_two_source_positions_times_three_directions_in_one_solver(prec, tol):
    """2 positions x 3 directions = 6 wavefields in one launch per colour
    (gfb_create_sources); each wavefield equals the oracle run of its own
    source and direction."""
    prob, sources = two_positions()
    dirs, fsrc = [0, 1, 2, 0, 1, 2], [0, 0, 0, 1, 1, 1]
    s = gfb.Solver(prob, dirs=dirs, precision=prec, sources=sources, field_source=fsrc)
    assert s.info()["n_field"] == 6
    s.advance(120)
    snaps = s.drain()
    for f, (d, k) in enumerate(zip(dirs, fsrc)):
        p = dict(prob, **sources[k])
        ref, (u, v, a) = oracle_snaps(p, d, 120)
        for q in ("strain", "u", "v"):
            e = rel_l2(snaps[f][q], ref[q])
            assert e <= tol, (f, q, e)
        if prec == gfb.FP64:
            compare_runs(snaps[f], ref, tol, f"field {f}")
            gu, gv, ga = s.state(f)
            assert rel_l2(gu, u) <= tol and rel_l2(gv, v) <= tol


def test_source_sets_are_checked():
    prob, sources = two_positions()
    with pytest.raises(gfb.GfbError):
        gfb.Solver(prob, dirs=[0, 1, 2, 0], precision=gfb.FP32, sources=sources, field_source=[0, 0, 0, 1])
    with pytest.raises(gfb.GfbError):
        gfb.Solver(prob, dirs=[0, 1], precision=gfb.FP32, sources=sources, field_source=[0, 2])


def test_fp32_force_by_increments_against_full_evaluation():
    """FP32 path: the element force of most steps is the stored force plus
    the force of the predicted displacement's increment (full evaluation
    every 800 steps, and after a state overwrite); evaluating it in full
    every step (GFB_FLAG_DIRECT_FORCE) gives the same traces to FP32 rounding,
    both within 1e-4 of the FP64 oracle, and a resume through set_state
    continues correctly."""
    prob = layered_problem(nsteps=260)
    n = prob["nsteps"]
    inc = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32)
    full = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32, flags=gfb.FLAG_DIRECT_FORCE)
    inc.advance(n)
    full.advance(n)
    a, b = inc.drain(), full.drain()
    for d in range(3):
        ref, _ = oracle_snaps(prob, d, n)
        compare_runs(a[d], ref, FP32_TOL, f"increments field {d}")
        compare_runs(b[d], ref, FP32_TOL, f"full field {d}")
    # state overwrite mid-run: the next step is a full evaluation
    half = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32, record=False)
    half.advance(130)
    st = [half.state(f) for f in range(3)]
    res = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32, record=False)
    for f in range(3):
        res.set_state(f, 130, *st[f])
    res.advance(130)
    inc2 = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32, record=False)
    inc2.advance(260)
    for f in range(3):
        assert rel_l2(res.state(f)[0], inc2.state(f)[0]) < FP32_TOL


def test_force_refresh_period_is_settable_and_checked():
    """gfb_set_force_refresh: every period gives traces within 1e-4 of the
    FP64 oracle (1: in full every step, as GFB_FLAG_DIRECT_FORCE, which also
    keeps (v, a) at every node: the same traces to rounding); a period of 1
    after increments, and a change mid-run, evaluate the next step in full;
    a solver that evaluates in full every step rejects a longer period."""
    prob = layered_problem(nsteps=240)
    n = prob["nsteps"]
    runs = {}
    for period in (1, 7, 50, 1000):
        s = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32)
        s.set_force_refresh(period)
        assert s.info()["force_refresh"] == period
        s.advance(n)
        runs[period] = s.drain()
        s.close()
    full = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32, flags=gfb.FLAG_DIRECT_FORCE)
    full.advance(n)
    direct = full.drain()
    full.close()
    for d in range(3):
        ref, _ = oracle_snaps(prob, d, n)
        for period, snaps in runs.items():
            compare_runs(snaps[d], ref, FP32_TOL, f"refresh {period} field {d}")
        for k in ("strain", "u"):
            assert rel_l2(runs[1][d][k], direct[d][k]) < 1e-5
    s = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32)
    s.advance(n // 3)
    s.set_force_refresh(3)
    s.advance(n // 3)
    s.set_force_refresh(1)
    s.advance(n // 6)
    s.set_force_refresh(40)  # back to increments
    assert s.info()["force_refresh"] == 40
    s.advance(n - 2 * (n // 3) - n // 6)
    mixed = s.drain()
    s.close()
    for d in range(3):
        ref, _ = oracle_snaps(prob, d, n)
        compare_runs(mixed[d], ref, FP32_TOL, f"changed refresh field {d}")
    with pytest.raises(gfb.GfbError, match=">= 1"):
        gfb.Solver(prob, dirs=[0], precision=gfb.FP32).set_force_refresh(0)
    s64 = gfb.Solver(prob, dirs=[0], precision=gfb.FP64)
    s64.set_force_refresh(1)  # what it does anyway
    with pytest.raises(gfb.GfbError, match="in full every step"):
        s64.set_force_refresh(100)
    s64.close()
