"""gfb -- Python binding of the B200 CG-SEM elastic time loop.

Thin ctypes layer over the C ABI declared in include/gfb.h and implemented
in lib/libgfb.so (CUDA, sm_100a).  There is no CPU fallback: constructing a
``Solver`` without the library or without a GPU raises.

Reference interface mirrored: the single-GPU device API of the reference
forward solver (forward/share/include/gf/cuda_step.hpp:70-129) driven the way
``run_forward`` drives it (forward/share/src/solver.cpp:389-508).
"""

from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libgfb.so")
HEADER_PATH = os.path.join(os.path.dirname(PKG_ROOT), "include", "gfb.h")

FP64, FP32 = 0, 1
FLAG_CELL_PML = 1
FLAG_RECORD_F32 = 2
FLAG_FUSED_NODE = 4
FLAG_POINT_KERNEL = 8
FLAG_NO_GRAPH = 16
FLAG_AUTOTUNE = 32
FLAG_DIRECT_FORCE = 64

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


class GfbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"gfb status {status}: {message}")
        self.status = status


class Mesh(C.Structure):
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
        ("n_rec_cell", C.c_int32),
        ("rec_cell_local", _ip),
    ]


class Config(C.Structure):
    _fields_ = [
        ("dt", C.c_double),
        ("snapshot_stride", C.c_int32),
        ("precision", C.c_int32),
        ("n_field", C.c_int32),
        ("field_dir", C.c_int32 * 3),
        ("device", C.c_int32),
        ("record_slots", C.c_int32),
        ("flags", C.c_int32),
    ]


class Info(C.Structure):
    _fields_ = [
        ("n_colour", C.c_int32),
        ("n_pml_cell", C.c_int32),
        ("n_rec_cell", C.c_int32),
        ("n_field", C.c_int32),
        ("precision", C.c_int32),
        ("n_cell", C.c_int32),
        ("n_node", C.c_int32),
        ("ngll", C.c_int32),
        ("device_bytes", C.c_int64),
        ("upload_bytes", C.c_int64),
        ("kernel_launches", C.c_int64),
        ("n_pml_node", C.c_int32),
        ("elem_blocks", C.c_int32),
        ("elem_kernel", C.c_int32),
        ("cells_per_group", C.c_int32),
        ("force_refresh", C.c_int32),
        ("half_v", C.c_int32),
        ("elem_variant", C.c_int32),
        ("n_elem_variants", C.c_int32),
    ]


class Source(C.Structure):
    _fields_ = [
        ("n_src_cell", C.c_int32),
        ("cell_ids", _lp),
        ("weights", _dp),
        ("n_stf", C.c_int32),
        ("stf", _dp),
    ]


class Model(C.Structure):
    _fields_ = [
        ("cell_begin", C.c_int32),
        ("cell_end", C.c_int32),
        ("node_begin", C.c_int32),
        ("node_end", C.c_int32),
        ("dt", C.c_double),
        ("n_steps", C.c_int32),
        ("n_stf", C.c_int32),
        ("stf", C.POINTER(C.c_double)),
    ]


_lib: Optional[C.CDLL] = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load lib/libgfb.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: build it with `make -C gf-only-sem_b200`")
    lib = C.CDLL(path)
    lib.gfb_abi_version.restype = C.c_int32
    lib.gfb_last_error.restype = C.c_char_p
    lib.gfb_create.argtypes = [C.POINTER(Mesh), C.POINTER(Config), C.POINTER(Source), C.POINTER(C.c_void_p)]
    lib.gfb_destroy.argtypes = [C.c_void_p]
    lib.gfb_advance.argtypes = [C.c_void_p, C.c_int32]
    lib.gfb_synchronize.argtypes = [C.c_void_p]
    lib.gfb_advance_profiled.argtypes = [C.c_void_p, C.c_int32, _dp, _dp, _dp]
    lib.gfb_advance_timed.argtypes = [C.c_void_p, C.c_int32, _dp]
    lib.gfb_rec_nodes.argtypes = [C.c_void_p, _ip, _lp]
    lib.gfb_read_green.argtypes = [C.c_void_p, _ip, _dp, _dp, _dp, _dp, C.c_int32]
    lib.gfb_checkpoint_size.argtypes = [C.c_void_p, _lp]
    lib.gfb_checkpoint_save.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
    lib.gfb_checkpoint_load.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
    lib.gfb_create_batch.argtypes = [C.POINTER(Mesh), C.POINTER(Config), C.POINTER(Source), C.c_int32,
                                     C.POINTER(Model), C.POINTER(C.c_void_p)]
    lib.gfb_create_sources.argtypes = [C.POINTER(Mesh), C.POINTER(Config), C.c_int32, C.POINTER(Source), C.c_int32,
                                       _ip, _ip, C.POINTER(C.c_void_p)]
    lib.gfb_get_info.argtypes = [C.c_void_p, C.POINTER(Info)]
    lib.gfb_select_element_kernel.argtypes = [C.c_void_p, C.c_int32]
    lib.gfb_set_force_refresh.argtypes = [C.c_void_p, C.c_int32]
    lib.gfb_current_step.argtypes = [C.c_void_p, _ip]
    lib.gfb_get_state.argtypes = [C.c_void_p, C.c_int32, _dp, _dp, _dp]
    lib.gfb_set_state.argtypes = [C.c_void_p, C.c_int32, C.c_int32, _dp, _dp, _dp]
    lib.gfb_records_pending.argtypes = [C.c_void_p, _ip]
    lib.gfb_read_record.argtypes = [C.c_void_p, C.c_int32, _ip, _dp, _dp, _dp, _dp, C.c_int32]
    _fp = C.POINTER(C.c_float)
    lib.gfb_read_record_f32.argtypes = [C.c_void_p, C.c_int32, _ip, _fp, _fp, _fp, _fp, C.c_int32]
    lib.gfb_element_residual.argtypes = [C.c_int32, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int32, _dp, _dp, C.c_int32, C.c_int32]
    lib.gfb_run_forward.argtypes = [C.c_char_p, C.c_int32, C.c_int32]
    lib.gfb_run_forward.restype = C.c_int32
    for name in (
        "gfb_create", "gfb_destroy", "gfb_advance", "gfb_synchronize", "gfb_current_step",
        "gfb_get_state", "gfb_set_state", "gfb_records_pending", "gfb_read_record",
        "gfb_element_residual", "gfb_advance_profiled", "gfb_get_info", "gfb_advance_timed",
        "gfb_create_batch", "gfb_checkpoint_size", "gfb_checkpoint_save", "gfb_checkpoint_load",
        "gfb_rec_nodes", "gfb_read_green", "gfb_read_record_f32", "gfb_create_sources",
        "gfb_select_element_kernel", "gfb_set_force_refresh",
    ):
        getattr(lib, name).restype = C.c_int
    _lib = lib
    return lib


def _check(st: int):
    if st != 0:
        raise GfbError(st, load_library().gfb_last_error().decode())


def _ptr(a, ctype):
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    return a.ctypes.data_as(C.POINTER(ctype))


def element_residual(dxi_dx, jacobian, lam, mu, u, ngll: int, precision: int = FP64, device: int = 0):
    """K_e u for independent elements on the GPU (compute_element_residual<BackendCUDA>)."""
    lib = load_library()
    nn = ngll**3
    arrs = [np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (dxi_dx, jacobian, lam, mu, u)]
    n_elem = arrs[1].size // nn
    r = np.zeros(n_elem * nn * 3)
    _check(
        lib.gfb_element_residual(
            n_elem, *[_ptr(a, C.c_double) for a in arrs[:4]], None, None, ngll,
            _ptr(arrs[4], C.c_double), _ptr(r, C.c_double), precision, device
        )
    )
    return r


class Solver:
    """All wavefields of one model advanced together on one GPU.

    ``prob`` is a dict of reference-layout arrays (see gfb.mesh.build_problem);
    ``dirs`` lists the force direction (0=x, 1=y, 2=z) of each wavefield.
    """

    def __init__(self, prob: dict, dirs: Sequence[int] = (0,), precision: int = FP64,
                 device: int = 0, record_slots: int = 4, record: bool = True, flags: int = 0,
                 models: Optional[Sequence[dict]] = None, sources: Optional[Sequence[dict]] = None,
                 field_source: Optional[Sequence[int]] = None):
        """``sources`` (several source positions, gfb_create_sources): dicts
        with src_cell_ids, src_weights and stf; wavefield f is driven by
        sources[field_source[f]] in direction dirs[f]."""
        self.lib = load_library()
        keep = {}

        def arr(name, dtype):
            if name not in prob or prob[name] is None:
                return None
            a = np.ascontiguousarray(prob[name], dtype=dtype).ravel()
            keep[name] = a
            return a

        m = Mesh()
        m.n_cell = int(prob["n_cell"])
        m.ngll = int(prob["ngll"])
        m.n_node = int(prob["n_node"])
        m.ibool = _ptr(arr("ibool", np.int32), C.c_int32)
        m.cell_ids = _ptr(arr("cell_ids", np.int64), C.c_int64)
        m.dxi_dx = _ptr(arr("dxi_dx", np.float64), C.c_double)
        m.jacobian = _ptr(arr("jacobian", np.float64), C.c_double)
        m.lambda_ = _ptr(arr("lambda", np.float64), C.c_double)
        m.mu = _ptr(arr("mu", np.float64), C.c_double)
        m.density = _ptr(arr("density", np.float64), C.c_double)
        m.mass = _ptr(arr("mass", np.float64), C.c_double)
        m.damping = _ptr(arr("damping", np.float64), C.c_double)
        m.pml_region = _ptr(arr("pml_region", np.int32), C.c_int32)
        m.pml_coef_alpha = _ptr(arr("pml_coef_alpha", np.float64), C.c_double)
        m.pml_coef_abar = _ptr(arr("pml_coef_abar", np.float64), C.c_double)
        rec = prob.get("recording") if record else None
        if rec is not None:
            rc = np.ascontiguousarray(rec["rec_cell_local"], dtype=np.int32)
            keep["rec"] = rc
            m.n_rec_cell = int(rc.size)
            m.rec_cell_local = _ptr(rc, C.c_int32)
        else:
            m.n_rec_cell = 0
            m.rec_cell_local = _ptr(None, C.c_int32)
        c = Config()
        c.dt = float(prob["dt"])
        c.snapshot_stride = int(prob.get("snapshot_stride", 0))
        self.stride = c.snapshot_stride
        c.precision = int(precision)
        c.n_field = len(dirs)
        for i, d in enumerate(dirs[:3]):
            c.field_dir[i] = int(d)
        c.device = int(device)
        c.record_slots = int(record_slots)
        c.flags = int(flags)
        s = Source()
        ids = arr("src_cell_ids", np.int64)
        s.n_src_cell = 0 if ids is None else int(ids.size)
        s.cell_ids = _ptr(ids, C.c_int64)
        s.weights = _ptr(arr("src_weights", np.float64), C.c_double)
        stf = arr("stf", np.float64)
        s.n_stf = 0 if stf is None else int(stf.size)
        s.stf = _ptr(stf, C.c_double)
        h = C.c_void_p()
        if sources is not None:
            if field_source is None or len(field_source) != len(dirs):
                raise ValueError("field_source must give the source of every wavefield")
            c.n_field = 1
            c.field_dir[0] = 0
            ss = (Source * len(sources))()
            for k, d in enumerate(sources):
                ids = np.ascontiguousarray(d["src_cell_ids"], dtype=np.int64).ravel()
                w = np.ascontiguousarray(d["src_weights"], dtype=np.float64).ravel()
                st = np.ascontiguousarray(d["stf"], dtype=np.float64).ravel()
                keep[f"sids{k}"], keep[f"sw{k}"], keep[f"sstf{k}"] = ids, w, st
                ss[k].n_src_cell = int(ids.size)
                ss[k].cell_ids = _ptr(ids, C.c_int64)
                ss[k].weights = _ptr(w, C.c_double)
                ss[k].n_stf = int(st.size)
                ss[k].stf = _ptr(st, C.c_double)
            fd = np.ascontiguousarray(dirs, dtype=np.int32)
            fsrc = np.ascontiguousarray(field_source, dtype=np.int32)
            keep["fd"], keep["fsrc"] = fd, fsrc
            _check(self.lib.gfb_create_sources(C.byref(m), C.byref(c), len(sources), ss, len(dirs),
                                               _ptr(fd, C.c_int32), _ptr(fsrc, C.c_int32), C.byref(h)))
        elif models is None:
            _check(self.lib.gfb_create(C.byref(m), C.byref(c), C.byref(s), C.byref(h)))
        else:
            md = (Model * len(models))()
            for k, d in enumerate(models):
                st = np.ascontiguousarray(d["stf"], dtype=np.float64).ravel()
                keep[f"stf{k}"] = st
                md[k].cell_begin, md[k].cell_end = int(d["cell_begin"]), int(d["cell_end"])
                md[k].node_begin, md[k].node_end = int(d["node_begin"]), int(d["node_end"])
                md[k].dt = float(d["dt"])
                md[k].n_steps = int(d["n_steps"])
                md[k].n_stf = int(st.size)
                md[k].stf = _ptr(st, C.c_double)
            _check(self.lib.gfb_create_batch(C.byref(m), C.byref(c), C.byref(s), len(models), md, C.byref(h)))
        self.h = h
        self.n_node = m.n_node
        self.n_field = len(dirs)
        self.n_rec = m.n_rec_cell
        self.nn = m.ngll**3
        del keep

    def advance(self, n_steps: int):
        _check(self.lib.gfb_advance(self.h, int(n_steps)))

    def checkpoint(self) -> bytes:
        """Exact checkpoint of the time-loop state (gfb_checkpoint_save)."""
        n = C.c_int64()
        _check(self.lib.gfb_checkpoint_size(self.h, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        _check(self.lib.gfb_checkpoint_save(self.h, buf, n.value))
        return buf.raw

    def restore(self, data: bytes):
        """Continue from a checkpoint of a solver built from the same inputs."""
        buf = C.create_string_buffer(data, len(data))
        _check(self.lib.gfb_checkpoint_load(self.h, buf, len(data)))

    def advance_timed(self, n_steps: int) -> float:
        """Advance and return the device milliseconds of the n_steps steps."""
        t = C.c_double(0.0)
        _check(self.lib.gfb_advance_timed(self.h, int(n_steps), C.byref(t)))
        return t.value

    def advance_profiled(self, n_steps: int):
        """Advance and return device milliseconds per phase (element, node, record)."""
        t = [C.c_double(0.0) for _ in range(3)]
        _check(self.lib.gfb_advance_profiled(self.h, int(n_steps), *[C.byref(x) for x in t]))
        return tuple(x.value for x in t)

    def info(self) -> dict:
        i = Info()
        _check(self.lib.gfb_get_info(self.h, C.byref(i)))
        return {name: getattr(i, name) for name, _ in Info._fields_}

    def select_element_kernel(self, variant: int):
        """Use element-kernel variant `variant` from the next step on (-1: the
        thread-per-point kernel; 0..n_elem_variants-1: the line kernel's)."""
        _check(self.lib.gfb_select_element_kernel(self.h, int(variant)))

    def set_force_refresh(self, steps: int):
        """FP32 path: steps between full evaluations of the element force."""
        _check(self.lib.gfb_set_force_refresh(self.h, int(steps)))

    def synchronize(self):
        _check(self.lib.gfb_synchronize(self.h))

    @property
    def step(self) -> int:
        s = C.c_int32()
        _check(self.lib.gfb_current_step(self.h, C.byref(s)))
        return s.value

    def state(self, field: int = 0):
        u, v, a = (np.zeros(self.n_node * 3) for _ in range(3))
        _check(self.lib.gfb_get_state(self.h, field, _ptr(u, C.c_double), _ptr(v, C.c_double), _ptr(a, C.c_double)))
        return u.reshape(-1, 3), v.reshape(-1, 3), a.reshape(-1, 3)

    def set_state(self, field: int, step: int, u=None, v=None, a=None):
        cv = [None if x is None else np.ascontiguousarray(x, dtype=np.float64).ravel() for x in (u, v, a)]
        _check(self.lib.gfb_set_state(self.h, field, step, *[_ptr(x, C.c_double) for x in cv]))

    def pending(self) -> int:
        n = C.c_int32()
        _check(self.lib.gfb_records_pending(self.h, C.byref(n)))
        return n.value

    def _record_arrays(self, n: Optional[int] = None, dtype=np.float64):
        lead = () if n is None else (n,)
        out = {"strain": np.empty(lead + (self.n_rec, self.nn, 6), dtype=dtype)}
        for k in ("u", "v", "a"):
            out[k] = np.empty(lead + (self.n_rec, self.nn, 3), dtype=dtype)
        return out

    def read_record(self, field: int = 0, release: bool = False, out: Optional[dict] = None, dtype=np.float64):
        """Oldest unread snapshot of one field: strain [cell][point][6],
        u, v, a [cell][point][3] over the recording cells, float64 or
        float32 (``dtype``; float32 is what the reference writes with
        snapshot_precision "float32").  ``out`` gives C-contiguous arrays of
        those shapes and one of the two types to fill instead of new ones (a
        missing key is not read)."""
        step = C.c_int32()
        if out is None:
            out = self._record_arrays(dtype=dtype)
        arrs, types = {}, set()
        for k, last in (("strain", 6), ("u", 3), ("v", 3), ("a", 3)):
            x = out.get(k)
            if x is not None:
                if (x.dtype not in (np.float64, np.float32) or not x.flags.c_contiguous
                        or x.shape != (self.n_rec, self.nn, last)):
                    raise ValueError(f"out[{k!r}] must be C-contiguous float64 or float32 of shape "
                                     f"{(self.n_rec, self.nn, last)}")
                types.add(x.dtype)
            arrs[k] = x
        if len(types) > 1:
            raise ValueError("out arrays must share one dtype")
        f32 = types == {np.dtype(np.float32)}
        fn, ct = (self.lib.gfb_read_record_f32, C.c_float) if f32 else (self.lib.gfb_read_record, C.c_double)
        _check(fn(self.h, field, C.byref(step), *[_ptr(arrs[k], ct) for k in ("strain", "u", "v", "a")],
                  1 if release else 0))
        return {"step": step.value, **arrs}

    def rec_nodes(self) -> np.ndarray:
        """Node ids of the recording nodes (ascending)."""
        n = C.c_int32()
        _check(self.lib.gfb_rec_nodes(self.h, C.byref(n), _ptr(None, C.c_int64)))
        ids = np.zeros(n.value, dtype=np.int64)
        _check(self.lib.gfb_rec_nodes(self.h, C.byref(n), ids.ctypes.data_as(C.POINTER(C.c_int64))))
        return ids

    def read_green(self, release: bool = True):
        """Oldest pending snapshot merged per recording node: strain
        [node][field][6] (the Green's tensor with fields x, y, z), u, v, a
        [node][field][3]."""
        n = len(self.rec_nodes())
        step = C.c_int32()
        strain = np.zeros((n, self.n_field, 6))
        u, v, a = (np.zeros((n, self.n_field, 3)) for _ in range(3))
        _check(self.lib.gfb_read_green(self.h, C.byref(step), _ptr(strain, C.c_double), _ptr(u, C.c_double),
                                       _ptr(v, C.c_double), _ptr(a, C.c_double), 1 if release else 0))
        return {"step": step.value, "strain": strain, "u": u, "v": v, "a": a}

    def _read_snapshots(self, n: int, wait=None, dtype=np.float64):
        """n snapshots, every field, read into arrays allocated once:
        {field: {"steps": [n], "strain": [n][cell][point][6], "u"/"v"/"a":
        [n][cell][point][3]}}.  ``wait()`` is called while none is pending
        (returns False to give up)."""
        out = {}
        for f in range(self.n_field):
            out[f] = {"steps": np.zeros(n, dtype=np.int64), **self._record_arrays(n, dtype)}
        for i in range(n):
            while wait is not None and self.pending() == 0:
                if not wait():
                    raise GfbError(3, "snapshot reader stopped before all snapshots arrived")
            for f in range(self.n_field):
                r = self.read_record(f, out={k: out[f][k][i] for k in ("strain", "u", "v", "a")})
                out[f]["steps"][i] = r["step"]
        return out

    def drain(self, dtype=np.float64):
        """All pending snapshots as {field: dict of stacked arrays}."""
        return self._read_snapshots(self.pending(), dtype=dtype)

    def run(self, n_steps: int, dtype=np.float64):
        """Advance n_steps and return every snapshot pending before them or
        recorded by them (as ``drain``), read out by a second thread while the
        steps run, as the reference's time loop writes each snapshot when it
        is taken."""
        import threading

        first = self.step
        n = self.pending()
        if self.stride > 0 and self.n_rec > 0:
            n += sum(1 for t in range(first, first + int(n_steps)) if t % self.stride == 0)
        done = threading.Event()
        box = {}

        def wait():
            if done.is_set() and self.pending() == 0:
                return False
            done.wait(0.0002)
            return True

        def reader():
            try:
                box["out"] = self._read_snapshots(n, wait, dtype)
            except BaseException as e:  # re-raised in the caller's thread
                box["err"] = e

        th = threading.Thread(target=reader, daemon=True)
        th.start()
        try:
            self.advance(n_steps)
        finally:
            done.set()
            th.join()
        if "err" in box:
            raise box["err"]
        return box["out"]

    def close(self):
        if getattr(self, "h", None):
            self.lib.gfb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# several independent models in one solver (gfb_create_batch)
# ---------------------------------------------------------------------------

def merge_problems(probs: Sequence[dict], n_steps: Optional[Sequence[int]] = None):
    """One batch mesh from independent models, and the model table.

    Cells, nodes, recording cells and source cells of model k follow those of
    models 0..k-1; node ids are offset so no two models share a node.  Every
    model keeps its own dt and source time function.  Returns (merged problem
    dict, list of model dicts for Solver(models=...), layout dict with the
    cell/node/recording-cell ranges of each model).
    """
    if not probs:
        raise ValueError("no models")
    ngll = int(probs[0]["ngll"])
    strides = {int(p.get("snapshot_stride", 0)) for p in probs}
    if any(int(p["ngll"]) != ngll for p in probs) or len(strides) != 1:
        raise ValueError("models must share ngll and snapshot_stride")
    cpml = [p.get("pml_coef_abar") is not None for p in probs]
    if any(cpml) and not all(cpml):
        raise ValueError("either every model has C-PML or none")
    nn = ngll ** 3
    cell_off = np.cumsum([0] + [int(p["n_cell"]) for p in probs])
    node_off = np.cumsum([0] + [int(p["n_node"]) for p in probs])
    rec_n = [0 if p.get("recording") is None else int(np.asarray(p["recording"]["rec_cell_local"]).size)
             for p in probs]
    rec_off = np.cumsum([0] + rec_n)

    def cat(name, dtype):
        if probs[0].get(name) is None:
            return None
        return np.concatenate([np.asarray(p[name], dtype=dtype).ravel() for p in probs])

    merged = {"n_cell": int(cell_off[-1]), "n_node": int(node_off[-1]), "ngll": ngll,
              "dt": float(probs[0]["dt"]), "snapshot_stride": strides.pop()}
    merged["ibool"] = np.concatenate([np.asarray(p["ibool"], dtype=np.int64).ravel() + node_off[k]
                                      for k, p in enumerate(probs)]).astype(np.int32)
    merged["cell_ids"] = np.arange(merged["n_cell"], dtype=np.int64)
    for name in ("dxi_dx", "jacobian", "lambda", "mu", "density", "mass", "pml_coef_alpha", "pml_coef_abar"):
        merged[name] = cat(name, np.float64)
    if all(p.get("damping") is not None for p in probs):
        merged["damping"] = cat("damping", np.float64)
    if all(cpml):
        merged["pml_region"] = cat("pml_region", np.int32)
    if sum(rec_n) > 0:
        merged["recording"] = {"rec_cell_local": np.concatenate(
            [np.asarray(p["recording"]["rec_cell_local"], dtype=np.int64) + cell_off[k]
             for k, p in enumerate(probs) if p.get("recording") is not None]).astype(np.int32)}
    ids, wts = [], []
    for k, p in enumerate(probs):
        if p.get("src_cell_ids") is None:
            continue
        cid = np.asarray(p.get("cell_ids", np.arange(int(p["n_cell"]))), dtype=np.int64)
        pos = {int(c): i for i, c in enumerate(cid)}
        for c, w in zip(np.asarray(p["src_cell_ids"], dtype=np.int64),
                        np.asarray(p["src_weights"], dtype=np.float64).reshape(-1, nn)):
            if int(c) in pos:  # a source cell outside the mesh is skipped, as in one model
                ids.append(cell_off[k] + pos[int(c)])
                wts.append(w)
    if ids:
        merged["src_cell_ids"] = np.asarray(ids, dtype=np.int64)
        merged["src_weights"] = np.concatenate(wts)
    models = []
    for k, p in enumerate(probs):
        ns = int(n_steps[k]) if n_steps is not None else int(p.get("nsteps", 2**31 - 1))
        models.append({"cell_begin": int(cell_off[k]), "cell_end": int(cell_off[k + 1]),
                       "node_begin": int(node_off[k]), "node_end": int(node_off[k + 1]),
                       "dt": float(p["dt"]), "n_steps": ns,
                       "stf": np.asarray(p.get("stf", np.zeros(0)), dtype=np.float64)})
    layout = {"cell_off": cell_off, "node_off": node_off, "rec_off": rec_off}
    return merged, models, layout


class BatchSolver(Solver):
    """Several independent models advanced together by one solver.

    ``probs`` are per-model problem dicts (gfb.mesh.build_problem layout);
    ``n_steps`` the steps each model takes (default: its "nsteps").  The
    models share ngll, snapshot stride, precision and wavefield directions.

    The models are placed in the solver in decreasing order of their step
    counts, so the ones that have finished are always the last cells of
    each colour and the last nodes: each step's launches stop before them.
    Model indices in this class's methods are the caller's.
    """

    def __init__(self, probs: Sequence[dict], dirs: Sequence[int] = (0,), precision: int = FP64,
                 device: int = 0, record_slots: int = 4, flags: int = 0, n_steps: Optional[Sequence[int]] = None):
        steps = [int(n) for n in (n_steps if n_steps is not None else [p["nsteps"] for p in probs])]
        self.placement = sorted(range(len(probs)), key=lambda k: -steps[k])  # position -> caller index
        self.position = [0] * len(probs)  # caller index -> position
        for pos, k in enumerate(self.placement):
            self.position[k] = pos
        merged, models, layout = merge_problems([probs[k] for k in self.placement],
                                                [steps[k] for k in self.placement])
        super().__init__(merged, dirs=dirs, precision=precision, device=device, record_slots=record_slots,
                         flags=flags, models=models)
        self.models = models  # in placement order
        self.layout = layout  # in placement order
        self.n_model = len(models)

    def model_state(self, k: int, field: int = 0):
        u, v, a = self.state(field)
        pos = self.position[k]
        a0, a1 = self.layout["node_off"][pos], self.layout["node_off"][pos + 1]
        return u[a0:a1], v[a0:a1], a[a0:a1]

    def drain_models(self):
        """Pending snapshots split by model: list over models of
        {field: {"steps", "strain", "u", "v", "a"}}, keeping the snapshots of
        steps each model has taken."""
        snaps = self.drain()
        out = []
        for k in range(self.n_model):
            pos = self.position[k]
            r0, r1 = self.layout["rec_off"][pos], self.layout["rec_off"][pos + 1]
            per = {}
            for f, d in snaps.items():
                steps = np.asarray(d["steps"])
                keep = steps < self.models[pos]["n_steps"]
                per[f] = {"steps": steps[keep]}
                for name in ("strain", "u", "v", "a"):
                    x = np.asarray(d[name])
                    per[f][name] = x[keep][:, r0:r1] if x.size else x
            out.append(per)
        return out

