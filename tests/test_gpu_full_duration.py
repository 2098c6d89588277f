"""Parity over a whole run of the CPU-runnable workload: the homogeneous
halfspace of 20 x 20 x 10 cells (order 4, 3-cell C-PML, 2000 steps, every
surface cell recorded every 10 steps: 200 snapshots), as the reference's
example configures it.

* FP64 path, direction x, against the reference's own compiled CPU functions
  (oracle/_ref; the C restatement, bit-identical to it, when it is not
  built): relative L2 <= 1e-10 over every snapshot (strain, u, v, a) and on
  the final state.
* FP32 batched x/y/z path: <= 1e-4 against the same CPU run for x, and
  against the FP64 GPU path (validated above) for x, y and z.

And the layered 64 x 64 x 32 workload over its 4000 steps: FP32 batched
x/y/z against the FP64 path, <= 1e-4.

The errors are accumulated snapshot by snapshot (gfb.accuracy.TraceError):
||gpu - ref|| / ||ref|| over all snapshots, cells, points and components.
"""

import os

import numpy as np
import pytest
from conftest import rel_l2

import gfb
import oracle
from gfb.accuracy import QUANTITIES, TraceError
from gfb.workloads import build_workload

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_TOL = 1e-4


def test_halfspace_2000_steps_fp64_and_fp32_against_the_cpu_reference():
    prob = build_workload("halfspace_20x20x10", prep="reference", device=None)
    n = prob["nsteps"]
    assert n == 2000 and prob["n_cell"] == 4000
    which = "ref" if os.path.exists(oracle.LIB_REF) else "oracle"
    run = oracle.Run(prob, 0, which, threads=os.cpu_count() or 1)
    s64 = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP64, record_slots=8)
    s32 = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32, record_slots=8)
    e64, e32, e32_64 = TraceError(), TraceError(), TraceError()
    step, snaps = 0, 0
    while step < n:
        k = min(100, n - step)
        ref = run.advance(k, step0=step)
        s64.advance(k)
        s32.advance(k)
        for i, ref_step in enumerate(ref["steps"]):
            for f in range(3):
                a = s64.read_record(f, release=f == 2)
                b = s32.read_record(f, release=f == 2)
                assert a["step"] == b["step"] == ref_step
                for q in QUANTITIES:
                    if f == 0:
                        e64.add(q, a[q], ref[q][i])
                        e32.add(q, b[q], ref[q][i])
                    e32_64.add(f"{q}/{f}", b[q], a[q])
            snaps += 1
        step += k
    assert snaps == 200
    u, v, a = run.state()
    gu, gv, ga = s64.state(0)
    final = {"u": rel_l2(gu, u), "v": rel_l2(gv, v), "a": rel_l2(ga, a)}
    run.close()
    s64.close()
    s32.close()
    print(f"fp64 vs {which}: {e64.summary()} final {final}")
    print(f"fp32 vs {which}: {e32.summary()}")
    print(f"fp32 vs fp64 gpu: worst {e32_64.worst():.3e}")
    for q in QUANTITIES:
        assert e64.rel(q) <= FP64_TOL, (q, e64.rel(q))
        assert e32.rel(q) <= FP32_TOL, (q, e32.rel(q))
    for k, v in final.items():
        assert v <= FP64_TOL, (k, v)
    assert e32_64.worst() <= FP32_TOL, e32_64.summary()


def test_layered_64x64x32_4000_steps_fp32_within_1e4_of_fp64():
    """The layered 64 x 64 x 32 workload (131,072 cells, 4-cell C-PML, 4000
    steps, 400 snapshots of the surface cells) with the
    host generator's inputs: the FP32 batched x/y/z path against the FP64
    path (validated against the reference's CPU functions above) over the
    whole run, every snapshot, every quantity <= 1e-4."""
    from gfb.accuracy import compare_solvers

    prob = build_workload("layered_64x64x32", prep="reference", device=0)
    n = prob["nsteps"]
    assert n == 4000
    s32 = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP32, record_slots=8)
    s64 = gfb.Solver(prob, dirs=[0, 1, 2], precision=gfb.FP64, record_slots=8)
    assert s32.info()["force_refresh"] > 1 and s32.info()["half_v"] == 1
    err = compare_solvers(s32, s64, n, chunk=8 * int(prob["snapshot_stride"]))
    s32.close()
    s64.close()
    print(f"fp32 vs fp64, layered 64x64x32, {n} steps: {err.summary()}")
    assert err.snapshots == 400
    assert err.worst() <= FP32_TOL, err.summary()
