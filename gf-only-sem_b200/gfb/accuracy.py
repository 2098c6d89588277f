"""Relative L2 error of recorded traces between two runs, accumulated
snapshot by snapshot so full-length runs need no more host memory than one
snapshot of each.

The error of a quantity over a run is ||x - y|| / ||y|| with the norms over
every snapshot, recording cell, GLL point and component (y the reference
run), the measure the time-loop parity tolerances are stated in.
"""

from __future__ import annotations

from typing import Dict, Optional

import numpy as np

QUANTITIES = ("strain", "u", "v", "a")


class TraceError:
    """Running sums of squared differences and squared reference values."""

    def __init__(self):
        self.num: Dict[str, float] = {}
        self.den: Dict[str, float] = {}
        self.snapshots = 0

    def add(self, key: str, x, y):
        x = np.asarray(x, dtype=np.float64)
        y = np.asarray(y, dtype=np.float64)
        self.num[key] = self.num.get(key, 0.0) + float(np.sum(np.square(x - y)))
        self.den[key] = self.den.get(key, 0.0) + float(np.sum(np.square(y)))

    def rel(self, key: str) -> float:
        d = self.den.get(key, 0.0)
        return float(np.sqrt(self.num.get(key, 0.0) / d)) if d > 0 else float(np.sqrt(self.num.get(key, 0.0)))

    def summary(self) -> Dict[str, float]:
        return {k: self.rel(k) for k in sorted(self.num)}

    def worst(self, prefix: str = "") -> float:
        vals = [self.rel(k) for k in self.num if k.startswith(prefix)]
        return max(vals) if vals else 0.0


def compare_solvers(test, ref, n_steps: int, chunk: int = 200, fields=None, green: bool = False,
                    ref_fields=None, err: Optional[TraceError] = None, on_chunk=None) -> TraceError:
    """Advance two solvers built on the same inputs n_steps in chunks and
    accumulate the error of every snapshot of test against ref: keys
    "<quantity>/<field>" for the recording cells' traces and, with green,
    "green_<quantity>" for the values merged per recording node (the strain
    Green's functions).  ``fields`` / ``ref_fields``: wavefield indices of
    test and the matching ones of ref (default: all of test, same indices)."""
    err = err or TraceError()
    fields = list(range(test.n_field)) if fields is None else list(fields)
    ref_fields = fields if ref_fields is None else list(ref_fields)
    done = 0
    while done < n_steps:
        k = min(chunk, n_steps - done)
        test.advance(k)
        ref.advance(k)
        done += k
        while test.pending() > 0:
            if green:
                gt = test.read_green(release=False)
                gr = ref.read_green(release=False)
                if gt["step"] != gr["step"]:
                    raise AssertionError(f"snapshot steps differ: {gt['step']} vs {gr['step']}")
                for q in QUANTITIES:
                    err.add(f"green_{q}", gt[q][:, fields], gr[q][:, ref_fields])
            for i, (f, g) in enumerate(zip(fields, ref_fields)):
                last = i == len(fields) - 1  # the last read releases the snapshot of every field
                a = test.read_record(f, release=last)
                b = ref.read_record(g, release=last)
                if a["step"] != b["step"]:
                    raise AssertionError(f"snapshot steps differ: {a['step']} vs {b['step']}")
                for q in QUANTITIES:
                    err.add(f"{q}/{f}", a[q], b[q])
            err.snapshots += 1
        if on_chunk:
            on_chunk(done)
    return err
