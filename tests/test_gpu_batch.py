"""Several independent models in one solver (gfb_create_batch), and the
CUDA-graph step.

A batch runs one element launch per colour over the cells of every model.
Colours are assigned per model exactly as for the model alone, and assembly
is colour-ordered, so every node sums its cell contributions in the same
order as in a run of its model alone: per-model traces and states must be
bit-identical to separate runs, including models that stop earlier than
the others."""

import numpy as np
import pytest

import gfb
from gfb import mesh

pytestmark = pytest.mark.gpu


def model(nx, ny, nz, seed, src, order=4):
    spec = mesh.MeshSpec(nx=nx, ny=ny, nz=nz, dx=500.0, dy=500.0, dz=500.0, order=order, jitter=0.06, seed=seed,
                         pml={"xmin": 1, "xmax": 1, "ymin": 1, "ymax": 1, "zmax": 1})
    mat = mesh.seeded_layers(seed, nz * 500.0)
    return mesh.build_problem(spec, mat, np.asarray(src, dtype=float), nsteps=60, snapshot_stride=10,
                              record_depth_max_m=500.0)


@pytest.fixture(scope="module")
def models():
    return [model(5, 4, 4, 11, [1200.0, 900.0, 700.0]),
            model(4, 4, 3, 12, [900.0, 1100.0, 400.0]),
            model(6, 5, 4, 13, [1700.0, 1300.0, 900.0])]


@pytest.mark.parametrize("prec", [gfb.FP32, gfb.FP64])
def test_batch_models_equal_separate_runs(models, prec):
    n_steps = [60, 35, 47]
    assert len({m["dt"] for m in models}) == 3  # each model keeps its own dt
    dirs = [0, 2]
    b = gfb.BatchSolver(models, dirs=dirs, precision=prec, n_steps=n_steps)
    b.advance(max(n_steps))
    got = b.drain_models()
    for k, p in enumerate(models):
        s = gfb.Solver(p, dirs=dirs, precision=prec)
        s.advance(n_steps[k])
        ref = s.drain()
        for f in range(len(dirs)):
            np.testing.assert_array_equal(got[k][f]["steps"], ref[f]["steps"])
            for name in ("strain", "u", "v", "a"):
                np.testing.assert_array_equal(got[k][f][name], ref[f][name], err_msg=f"model {k} {name}")
            for x, y in zip(b.model_state(k, f), s.state(f)):
                np.testing.assert_array_equal(x, y)
        s.close()
    b.close()


def test_batch_of_one_model_equals_plain_solver(models):
    p = models[0]
    b = gfb.BatchSolver([p], dirs=[1], precision=gfb.FP32, n_steps=[40])
    s = gfb.Solver(p, dirs=[1], precision=gfb.FP32)
    b.advance(40)
    s.advance(40)
    for x, y in zip(b.model_state(0, 0), s.state(0)):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("prec", [gfb.FP32, gfb.FP64])
def test_graph_replay_equals_eager_launches(models, prec):
    p = models[2]
    runs = []
    for flags in (0, gfb.FLAG_NO_GRAPH):
        s = gfb.Solver(p, dirs=[0, 1, 2], precision=prec, flags=flags)
        s.advance(23)
        s.advance(30)  # a second call replays the captured step again
        runs.append((s.drain(), [s.state(f) for f in range(3)], s.info()["kernel_launches"]))
        s.close()
    (a, sa, la), (b, sb, lb) = runs
    assert la == lb  # the graph's kernels are counted as launches
    for f in range(3):
        for name in ("strain", "u", "v", "a"):
            np.testing.assert_array_equal(a[f][name], b[f][name])
        for x, y in zip(sa[f], sb[f]):
            np.testing.assert_array_equal(x, y)


def test_resume_after_set_state_with_graph(models):
    """gfb_set_state moves the device step counter too: the source time
    function continues from the resumed step."""
    spec = mesh.MeshSpec(nx=4, ny=4, nz=3, dx=500.0, dy=500.0, dz=500.0, order=4, jitter=0.06, seed=3)
    p = mesh.build_problem(spec, mesh.seeded_layers(3, 1500.0), np.array([900.0, 1100.0, 400.0]), nsteps=60,
                           snapshot_stride=10, record_depth_max_m=500.0, with_cpml=False)
    full = gfb.Solver(p, dirs=[2], precision=gfb.FP32)
    full.advance(50)
    part = gfb.Solver(p, dirs=[2], precision=gfb.FP32)
    part.advance(20)
    u, v, a = part.state(0)
    res = gfb.Solver(p, dirs=[2], precision=gfb.FP32)
    res.set_state(0, 20, u, v, a)
    res.advance(30)
    for x, y in zip(res.state(0), full.state(0)):
        np.testing.assert_allclose(x, y, rtol=0, atol=1e-6 * np.abs(y).max())


@pytest.mark.parametrize("prec,flags", [(gfb.FP32, 0), (gfb.FP32, gfb.FLAG_CELL_PML), (gfb.FP64, 0)])
def test_checkpoint_resume_is_exact_with_cpml(models, prec, flags):
    """gfb_checkpoint_save/load carry the C-PML memory, so a resumed run
    continues bit for bit (the reference's restart keeps u, v, a only)."""
    p = models[0]
    a = gfb.Solver(p, dirs=[0, 2], precision=prec, flags=flags)
    a.advance(30)
    ck = a.checkpoint()
    a.drain()
    a.advance(45)
    ref = a.drain()
    sa = [a.state(f) for f in range(2)]
    b = gfb.Solver(p, dirs=[0, 2], precision=prec, flags=flags)
    b.restore(ck)
    assert b.step == 30
    b.advance(45)
    got = b.drain()
    for f in range(2):
        np.testing.assert_array_equal(got[f]["steps"], ref[f]["steps"])
        for name in ("strain", "u", "v", "a"):
            np.testing.assert_array_equal(got[f][name], ref[f][name])
        for x, y in zip(b.state(f), sa[f]):
            np.testing.assert_array_equal(x, y)
    # a checkpoint of another configuration is refused
    c = gfb.Solver(p, dirs=[0], precision=prec, flags=flags)
    with pytest.raises(gfb.GfbError):
        c.restore(ck)
