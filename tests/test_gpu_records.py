"""Snapshot read-out through the public API, and the mesh checks of
gfb_create.

``Solver.run`` reads every snapshot on a second thread while the steps run;
with two ring slots the stepping thread also moves unread snapshots to
pageable memory and waits on readers.  Its arrays must equal those of
``advance`` followed by ``drain`` bit for bit.  The mesh check of gfb_create
reports the first offending ibool entry in mesh order, as the serial check of
one entry after another would."""

import numpy as np
import pytest

import gfb
from gfb import mesh

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def prob():
    spec = mesh.MeshSpec(nx=6, ny=5, nz=4, dx=500.0, dy=500.0, dz=500.0, order=4, jitter=0.05, seed=21,
                         pml={"xmin": 1, "xmax": 1, "ymin": 1, "ymax": 1, "zmax": 1})
    mat = mesh.seeded_layers(21, 4 * 500.0)
    return mesh.build_problem(spec, mat, np.asarray([1400.0, 1100.0, 800.0]), nsteps=80, snapshot_stride=4,
                              record_depth_max_m=500.0)


@pytest.mark.parametrize("flags", [0, gfb.FLAG_RECORD_F32])
def test_run_equals_advance_then_drain(prob, flags):
    dirs = [0, 1, 2]
    a = gfb.Solver(prob, dirs=dirs, precision=gfb.FP32, record_slots=2, flags=flags)
    a.advance(3)
    a.drain()
    a.advance(77)
    ref = a.drain()
    b = gfb.Solver(prob, dirs=dirs, precision=gfb.FP32, record_slots=2, flags=flags)
    b.advance(3)
    b.read_record(0)  # the step-0 snapshot half read: run() reads it again, whole
    first = b.run(0)
    got = b.run(77)
    assert list(first[0]["steps"]) == [0]
    assert b.pending() == 0
    for f in range(len(dirs)):
        np.testing.assert_array_equal(got[f]["steps"], ref[f]["steps"])
        assert list(got[f]["steps"]) == list(range(4, 80, 4))
        for name in ("strain", "u", "v", "a"):
            np.testing.assert_array_equal(got[f][name], ref[f][name], err_msg=name)
    a.close()
    b.close()


def test_read_record_into_caller_arrays(prob):
    s = gfb.Solver(prob, dirs=[2], precision=gfb.FP32, record_slots=3)
    s.advance(9)
    ref = s.drain()
    s2 = gfb.Solver(prob, dirs=[2], precision=gfb.FP32, record_slots=3)
    s2.advance(9)
    u = np.full((s2.n_rec, s2.nn, 3), np.nan)
    r = s2.read_record(0, out={"u": u})
    assert r["u"] is u and r["strain"] is None
    np.testing.assert_array_equal(u, ref[0]["u"][0])
    with pytest.raises(ValueError):
        s2.read_record(0, out={"v": np.zeros((s2.n_rec, s2.nn, 3), dtype=np.int32)})
    # float32 read-out (gfb_read_record_f32) of this double record: rounded
    # to float32 as numpy rounds
    r = s2.read_record(0, dtype=np.float32)
    assert r["u"].dtype == np.float32
    for k in ("strain", "u", "v", "a"):
        np.testing.assert_array_equal(r[k], ref[0][k][1].astype(np.float32))
    s.close()
    s2.close()


def test_run_float32_equals_float64_read(prob):
    """Solver.run with float32 arrays reads the same float records as the
    float64 read-out, and a double record rounded to float32."""
    for flags in (gfb.FLAG_RECORD_F32, 0):
        a = gfb.Solver(prob, dirs=[0, 2], precision=gfb.FP32, record_slots=3, flags=flags)
        ref = a.run(40)
        b = gfb.Solver(prob, dirs=[0, 2], precision=gfb.FP32, record_slots=3, flags=flags)
        got = b.run(40, dtype=np.float32)
        for f in range(2):
            np.testing.assert_array_equal(got[f]["steps"], ref[f]["steps"])
            for k in ("strain", "u", "v", "a"):
                assert got[f][k].dtype == np.float32
                np.testing.assert_array_equal(got[f][k], ref[f][k].astype(np.float32))
        a.close()
        b.close()


def test_mesh_check_reports_first_offending_entry(prob):
    nn = prob["ngll"] ** 3
    bad = dict(prob)
    ib = np.array(prob["ibool"], dtype=np.int32).reshape(-1, nn).copy()
    # cell 7 repeats its point 3 at point 40; cell 9 has an entry out of range
    ib[7, 40] = ib[7, 3]
    ib[9, 2] = prob["n_node"]
    bad["ibool"] = ib
    with pytest.raises(gfb.GfbError, match=r"cell 7 lists node %d twice" % ib[7, 3]):
        gfb.Solver(bad, dirs=[0], precision=gfb.FP32)
    ib2 = np.array(prob["ibool"], dtype=np.int32).reshape(-1, nn).copy()
    # in one cell: an out-of-range entry before the repeat is the one reported
    ib2[5, 10] = -1
    ib2[5, 60] = ib2[5, 0]
    bad["ibool"] = ib2
    with pytest.raises(gfb.GfbError, match=r"ibool\[%d\]=-1 outside" % (5 * nn + 10)):
        gfb.Solver(bad, dirs=[0], precision=gfb.FP32)
