"""Host-side logic of the snapshot read-out and of the batch placement (no
GPU): ``Solver.run`` reading every snapshot on a second thread while the
steps run, ``drain`` into arrays allocated once, the float32 path, error
propagation from the reader thread, and ``BatchSolver`` placing models in
decreasing order of their step counts while answering in the caller's
order.

The library's snapshot calls are replaced by a fake with the same contract
as gfb_records_pending / gfb_read_record(_f32) / gfb_advance /
gfb_current_step: snapshots are taken at steps that are multiples of the
stride, a snapshot is released once each wavefield has been read (or at
once with release), and reading with none pending is an error."""

import ctypes as C
import threading
import time

import numpy as np
import pytest

import gfb
from test_batch_host import small_model  # noqa: F401  (tiny problems on the host)


class FakeLib:
    """Snapshot queue of a solver; every value of snapshot `step`, wavefield
    `field` is step * 10 + field.  advance() takes one step at a time with a
    short sleep, so a reader thread interleaves with it."""

    def __init__(self, n_field, n_rec, nn, stride, fail_at=None):
        self.lock = threading.Lock()
        self.pending = []  # [step, set of wavefields read]
        self.step = 0
        self.n_field, self.n_rec, self.nn, self.stride = n_field, n_rec, nn, stride
        self.fail_at = fail_at
        self.calls = {"f64": 0, "f32": 0}

    def gfb_current_step(self, h, ref):
        ref._obj.value = self.step
        return 0

    def gfb_records_pending(self, h, ref):
        with self.lock:
            ref._obj.value = len(self.pending)
        return 0

    def gfb_advance(self, h, n):
        for _ in range(int(n)):
            with self.lock:
                if self.stride > 0 and self.step % self.stride == 0:
                    self.pending.append([self.step, set()])
                self.step += 1
            time.sleep(0.0005)
        return 0

    def _read(self, field, ref, ptrs, release, kind):
        with self.lock:
            if not self.pending:
                return 3
            snap = self.pending[0]
            if self.fail_at is not None and snap[0] == self.fail_at:
                return 4
            npt = self.n_rec * self.nn
            for p, width in zip(ptrs, (6, 3, 3, 3)):
                if p:
                    np.ctypeslib.as_array(p, shape=(npt * width,))[:] = snap[0] * 10 + field
            snap[1].add(int(field))
            ref._obj.value = snap[0]
            if release or len(snap[1]) == self.n_field:
                self.pending.pop(0)
            self.calls[kind] += 1
        return 0

    def gfb_read_record(self, h, field, ref, s, u, v, a, release):
        return self._read(field, ref, (s, u, v, a), release, "f64")

    def gfb_read_record_f32(self, h, field, ref, s, u, v, a, release):
        return self._read(field, ref, (s, u, v, a), release, "f32")

    def gfb_last_error(self):
        return b"fake failure"


def fake_solver(n_field=2, n_rec=3, nn=8, stride=4, fail_at=None):
    s = object.__new__(gfb.Solver)
    s.lib = FakeLib(n_field, n_rec, nn, stride, fail_at)
    s.h = None  # close() then has nothing to destroy
    s.n_field, s.n_rec, s.nn, s.stride = n_field, n_rec, nn, stride
    return s


def check(rec, steps, n_field, dtype):
    for f in range(n_field):
        np.testing.assert_array_equal(rec[f]["steps"], steps)
        for k in ("strain", "u", "v", "a"):
            x = rec[f][k]
            assert x.dtype == dtype and x.shape[0] == len(steps)
            for i, t in enumerate(steps):
                assert np.all(x[i] == t * 10 + f)


def test_run_reads_every_snapshot_while_stepping():
    s = fake_solver()
    rec = s.run(30)
    check(rec, list(range(0, 30, 4)), 2, np.float64)
    assert s.pending() == 0
    # a second call continues from the current step
    rec = s.run(10)
    check(rec, [32, 36], 2, np.float64)


def test_run_includes_a_half_read_snapshot_and_float32():
    s = fake_solver(n_field=3)
    s.advance(1)
    s.read_record(0)  # step 0 half read: still pending, read whole by run()
    rec = s.run(9, dtype=np.float32)
    check(rec, [0, 4, 8], 3, np.float32)
    assert s.lib.calls["f32"] == 9 and s.lib.calls["f64"] == 1


def test_drain_allocates_once_and_reads_in_order():
    s = fake_solver(n_field=1, stride=2)
    s.advance(7)
    rec = s.drain()
    check(rec, [0, 2, 4, 6], 1, np.float64)
    assert rec[0]["strain"].shape == (4, 3, 8, 6)
    assert s.drain()[0]["u"].shape == (0, 3, 8, 3)


def test_reader_error_reaches_the_caller():
    s = fake_solver(fail_at=8)
    # the status becomes a GfbError carrying the library's last message (the
    # built library is loaded for it)
    with pytest.raises(gfb.GfbError):
        s.run(20)


def test_batch_places_models_by_decreasing_steps(monkeypatch):
    probs = [small_model(3, 3, 2, 10 + k, [700.0, 800.0, 300.0]) for k in range(3)]
    n_steps = [5, 20, 10]
    seen = {}

    def fake_init(self, prob, dirs=(0,), precision=0, device=0, record_slots=4, record=True, flags=0, models=None):
        seen["models"] = models
        self.lib, self.h = None, None
        self.n_field, self.n_rec, self.nn, self.n_node = len(dirs), prob["recording"]["rec_cell_local"].size, \
            prob["ngll"] ** 3, prob["n_node"]

    monkeypatch.setattr(gfb.Solver, "__init__", fake_init)
    b = gfb.BatchSolver(probs, dirs=[0], n_steps=n_steps)
    assert b.placement == [1, 2, 0] and b.position == [2, 0, 1]
    assert [m["n_steps"] for m in seen["models"]] == [20, 10, 5]
    # model_state answers in the caller's order: node ranges of the placed models
    node_off = b.layout["node_off"]

    def fake_state(field=0):
        u = np.arange(node_off[-1], dtype=float)[:, None].repeat(3, axis=1)
        return u, u, u

    monkeypatch.setattr(b, "state", fake_state)
    for k in range(3):
        u, _, _ = b.model_state(k)
        pos = b.position[k]
        assert u.shape[0] == probs[k]["n_node"]
        assert u[0, 0] == node_off[pos]
