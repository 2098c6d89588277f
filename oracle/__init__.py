"""CPU FP64 oracle of the CG-SEM elastic time loop (TEST INFRASTRUCTURE).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this package, and only as the checker.  It wraps two libraries with one C
interface (sem_oracle.h):

* ``lib/liboracle.so`` -- the plain-C restatement in sem_oracle.c of the
  reference CPU loop (forward/share/src/solver.cpp:510-688 and the functions
  it calls);
* ``_ref/libgf_ref.so`` -- the reference's own element_cpu.cpp, assembly.cpp
  and pml.cpp compiled from the reference tree, driven by ref_driver.cpp.

Both are built by ``oracle/Makefile`` (``make -C oracle``).
"""

from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "lib", "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libgf_ref.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


class Problem(C.Structure):
    _fields_ = [
        ("n_cell", C.c_int32),
        ("ngll", C.c_int32),
        ("n_node", C.c_int32),
        ("ibool", _ip),
        ("cell_ids", _lp),
        ("dxi_dx", _dp),
        ("jacobian", _dp),
        ("lambda_", _dp),
        ("mu", _dp),
        ("density", _dp),
        ("mass", _dp),
        ("damping", _dp),
        ("pml_region", _ip),
        ("pml_coef_alpha", _dp),
        ("pml_coef_abar", _dp),
        ("dt", C.c_double),
        ("snapshot_stride", C.c_int32),
        ("direction", C.c_int32),
        ("n_src", C.c_int32),
        ("src_cell_ids", _lp),
        ("src_weights", _dp),
        ("n_stf", C.c_int32),
        ("stf", _dp),
        ("n_rec", C.c_int32),
        ("rec_cell_local", _ip),
    ]


def _ptr(a: Optional[np.ndarray], ctype):
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    return a.ctypes.data_as(C.POINTER(ctype))


_libs: dict = {}


def load(which: str = "oracle") -> C.CDLL:
    """Load ``oracle`` (restatement) or ``ref`` (reference-compiled) library."""
    if which in _libs:
        return _libs[which]
    path = LIB_ORACLE if which == "oracle" else LIB_REF
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built; run `make -C oracle`")
    lib = C.CDLL(path)
    pre = "orc_" if which == "oracle" else "ref_"
    f = getattr(lib, pre + "create")
    f.restype = C.c_void_p
    f.argtypes = [C.POINTER(Problem)]
    getattr(lib, pre + "destroy").argtypes = [C.c_void_p]
    adv = getattr(lib, pre + "advance")
    adv.restype = C.c_int32
    adv.argtypes = [C.c_void_p, C.c_int32, C.c_int32, _ip, _dp, _dp, _dp, _dp]
    getattr(lib, pre + "get_state").argtypes = [C.c_void_p, _dp, _dp, _dp]
    getattr(lib, pre + "set_threads").argtypes = [C.c_int32]
    g = getattr(lib, pre + "gll")
    g.restype = C.c_int
    g.argtypes = [C.c_int32, _dp, _dp, _dp]
    er = getattr(lib, pre + "element_residual")
    er.argtypes = [C.c_int32, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int32, _dp, _dp]
    _libs[which] = lib
    return lib


def gll(N: int, which: str = "oracle"):
    lib = load(which)
    ng = N + 1
    x, w, D = np.zeros(ng), np.zeros(ng), np.zeros(ng * ng)
    rc = getattr(lib, ("orc_" if which == "oracle" else "ref_") + "gll")(
        N, _ptr(x, C.c_double), _ptr(w, C.c_double), _ptr(D, C.c_double)
    )
    if rc != 0:
        raise ValueError("GLL construction failed")
    return x, w, D.reshape(ng, ng)


def element_residual(dxi_dx, jacobian, lam, mu, u, ngll, which: str = "oracle"):
    """r = K_e u for a batch of elements (element_cpu.cpp:19-162)."""
    lib = load(which)
    nn = ngll**3
    n_elem = int(np.asarray(jacobian).size // nn)
    arrs = [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (dxi_dx, jacobian, lam, mu, u)]
    _, w, D = gll(ngll - 1, which)
    D = np.ascontiguousarray(D.ravel())
    r = np.zeros(n_elem * nn * 3)
    getattr(lib, ("orc_" if which == "oracle" else "ref_") + "element_residual")(
        n_elem, *[_ptr(a, C.c_double) for a in arrs[:4]], _ptr(D, C.c_double), _ptr(w, C.c_double),
        ngll, _ptr(arrs[4], C.c_double), _ptr(r, C.c_double)
    )
    return r


class Run:
    """One direction of the CPU time loop over a problem dict (gfb.mesh)."""

    def __init__(self, prob: dict, direction: int, which: str = "oracle", threads: int = 1):
        self.lib = load(which)
        self.pre = "orc_" if which == "oracle" else "ref_"
        getattr(self.lib, self.pre + "set_threads")(threads)
        keep = {}

        def arr(name, dtype):
            if name not in prob or prob[name] is None:
                return None
            a = np.ascontiguousarray(prob[name], dtype=dtype).ravel()
            keep[name] = a
            return a

        rec = prob.get("recording")
        rec_cells = None
        if rec is not None:
            rec_cells = np.ascontiguousarray(rec["rec_cell_local"], dtype=np.int32)
            keep["rec"] = rec_cells
        p = Problem()
        p.n_cell = int(prob["n_cell"])
        p.ngll = int(prob["ngll"])
        p.n_node = int(prob["n_node"])
        p.ibool = _ptr(arr("ibool", np.int32), C.c_int32)
        p.cell_ids = _ptr(arr("cell_ids", np.int64), C.c_int64)
        p.dxi_dx = _ptr(arr("dxi_dx", np.float64), C.c_double)
        p.jacobian = _ptr(arr("jacobian", np.float64), C.c_double)
        p.lambda_ = _ptr(arr("lambda", np.float64), C.c_double)
        p.mu = _ptr(arr("mu", np.float64), C.c_double)
        p.density = _ptr(arr("density", np.float64), C.c_double)
        p.mass = _ptr(arr("mass", np.float64), C.c_double)
        p.damping = _ptr(arr("damping", np.float64), C.c_double)
        p.pml_region = _ptr(arr("pml_region", np.int32), C.c_int32)
        p.pml_coef_alpha = _ptr(arr("pml_coef_alpha", np.float64), C.c_double)
        p.pml_coef_abar = _ptr(arr("pml_coef_abar", np.float64), C.c_double)
        p.dt = float(prob["dt"])
        p.snapshot_stride = int(prob.get("snapshot_stride", 0))
        p.direction = int(direction)
        src_ids = arr("src_cell_ids", np.int64)
        p.n_src = 0 if src_ids is None else int(src_ids.size)
        p.src_cell_ids = _ptr(src_ids, C.c_int64)
        p.src_weights = _ptr(arr("src_weights", np.float64), C.c_double)
        stf = arr("stf", np.float64)
        p.n_stf = 0 if stf is None else int(stf.size)
        p.stf = _ptr(stf, C.c_double)
        p.n_rec = 0 if rec_cells is None else int(rec_cells.size)
        p.rec_cell_local = _ptr(rec_cells, C.c_int32)
        self._keep = keep
        self._p = p
        self.h = getattr(self.lib, self.pre + "create")(C.byref(p))
        if not self.h:
            raise RuntimeError("oracle create failed")
        self.n_node = p.n_node
        self.n_rec = p.n_rec
        self.nn = p.ngll**3
        self.stride = p.snapshot_stride

    def advance(self, n_steps: int, step0: int = 0):
        """Run n_steps; returns dict of snapshots (steps, strain, u, v, a)."""
        nsnap = 0
        if self.stride > 0 and self.n_rec > 0:
            nsnap = len([s for s in range(step0, step0 + n_steps) if s % self.stride == 0])
        shape = (max(nsnap, 1), self.n_rec, self.nn)
        steps = np.zeros(max(nsnap, 1), dtype=np.int32)
        strain = np.zeros(shape + (6,))
        u, v, a = (np.zeros(shape + (3,)) for _ in range(3))
        n = getattr(self.lib, self.pre + "advance")(
            self.h, n_steps, max(nsnap, 1), _ptr(steps, C.c_int32), _ptr(strain, C.c_double),
            _ptr(u, C.c_double), _ptr(v, C.c_double), _ptr(a, C.c_double)
        )
        if n < 0:
            raise RuntimeError("snapshot buffer overflow")
        return {"steps": steps[:n], "strain": strain[:n], "u": u[:n], "v": v[:n], "a": a[:n]}

    def state(self):
        u, v, a = (np.zeros(self.n_node * 3) for _ in range(3))
        getattr(self.lib, self.pre + "get_state")(
            self.h, _ptr(u, C.c_double), _ptr(v, C.c_double), _ptr(a, C.c_double)
        )
        return u.reshape(-1, 3), v.reshape(-1, 3), a.reshape(-1, 3)

    def close(self):
        if getattr(self, "h", None):
            getattr(self.lib, self.pre + "destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
