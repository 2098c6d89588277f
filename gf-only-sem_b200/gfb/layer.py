"""Learned absorbing layer: thin domain + small networks, trained from replays
of a thick-C-PML run (C ABI in include/gfb.h, kernels in csrc/gfb_layer.cu).

A model is built twice from the same interior: *thick* with a ``n_thick``-
element C-PML on the five absorbing faces (x-, x+, y-, y+ and the bottom;
the top is the free surface) and *thin* with a one-element C-PML.  The thin
domain's layer nodes get a force correction from one network per node class
(side or bottom face x depth plane inside the layer cell); the networks are
trained so that the thin run follows the thick run, which is also the reference
of the reflection error.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import (FP32, FLAG_RECORD_F32, Solver, _check, _ptr, load_library)
from . import mesh

N_PARAMS = 6592      # GFB_LAYER_PARAMS
N_WEIGHTS = 8768     # GFB_LAYER_WEIGHTS
N_IN, N_HID, N_OUT = 36, 64, 3


class LayerDesc(C.Structure):
    _fields_ = [
        ("n_node", C.c_int32),
        ("node", C.POINTER(C.c_int32)),
        ("frame", C.POINTER(C.c_int8)),
        ("net", C.POINTER(C.c_uint8)),
        ("n_net", C.c_int32),
    ]


def _bind(lib):
    if getattr(lib, "_layer_bound", False):
        return lib
    vp, i32, i64, u64, f32p, dp = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64, C.POINTER(C.c_float), C.POINTER(C.c_double)
    lib.gfb_layer_pack.argtypes = [i32, f32p, C.POINTER(C.c_uint16)]
    lib.gfb_layer_attach.argtypes = [vp, C.POINTER(LayerDesc), C.POINTER(C.c_uint16), f32p, C.c_double]
    lib.gfb_layer_status.argtypes = [vp, C.POINTER(C.c_int32), dp]
    lib.gfb_layer_set_gains.argtypes = [vp, i32, f32p]
    lib.gfb_trainer_create.argtypes = [i32, i64, i32, u64, C.POINTER(vp)]
    lib.gfb_trainer_destroy.argtypes = [vp]
    lib.gfb_trainer_collect.argtypes = [vp, vp, vp, C.POINTER(C.c_int32), C.POINTER(LayerDesc), i32, i32, i32]
    lib.gfb_trainer_samples.argtypes = [vp, C.POINTER(C.c_int64)]
    lib.gfb_trainer_set_scales.argtypes = [vp, f32p]
    lib.gfb_trainer_fit.argtypes = [vp, i32, i32, C.c_float, u64, dp]
    lib.gfb_trainer_gradient.argtypes = [vp, i32, i32, f32p, f32p, f32p, dp]
    lib.gfb_trainer_get_params.argtypes = [vp, f32p, f32p]
    lib.gfb_trainer_set_params.argtypes = [vp, f32p]
    lib.gfb_trainer_evaluate.argtypes = [vp, dp]
    for n in ("gfb_layer_pack", "gfb_layer_attach", "gfb_layer_status", "gfb_layer_set_gains",
              "gfb_trainer_create", "gfb_trainer_destroy",
              "gfb_trainer_collect", "gfb_trainer_samples", "gfb_trainer_set_scales", "gfb_trainer_fit",
              "gfb_trainer_gradient", "gfb_trainer_get_params", "gfb_trainer_set_params", "gfb_trainer_evaluate"):
        getattr(lib, n).restype = C.c_int
    lib._layer_bound = True
    return lib


# ---------------------------------------------------------------------------
# models
# ---------------------------------------------------------------------------

@dataclass
class PairSpec:
    """Interior of ni x nj x nk cells of size d; layered material; a point
    source in the interior (interior coordinates); Ricker f0."""
    ni: int
    nj: int
    nk: int
    d: float
    seed: int
    src: tuple
    f0: float = 2.0
    nsteps: int = 1000
    stride: int = 10
    n_thick: int = 10
    n_thin: int = 1
    dt: Optional[float] = None


def build_domain(p: PairSpec, n_layer: int, dt: Optional[float] = None, with_cpml: bool = True) -> dict:
    """The model with an n_layer-element C-PML (or the legacy damping layer)
    on the absorbing faces; interior cell (0, 0, 0) starts at
    (n_layer d, n_layer d, 0)."""
    faces = {"xmin": n_layer, "xmax": n_layer, "ymin": n_layer, "ymax": n_layer, "zmax": n_layer}
    spec = mesh.MeshSpec(nx=p.ni + 2 * n_layer, ny=p.nj + 2 * n_layer, nz=p.nk + n_layer, dx=p.d, dy=p.d, dz=p.d,
                         order=4, pml=faces)
    mat = mesh.seeded_layers(p.seed, p.nk * p.d)
    src = np.array([p.src[0] + n_layer * p.d, p.src[1] + n_layer * p.d, p.src[2]])
    prob = mesh.build_problem(spec, mat, src, dt=dt, nsteps=p.nsteps, snapshot_stride=p.stride,
                              record_depth_max_m=p.d, f0=p.f0, with_cpml=with_cpml)
    prob["n_layer"] = n_layer
    return prob


def build_pair(p: PairSpec):
    """(thin, thick) problems with one time step (the smaller of the two
    CFL steps) and the thin->thick node map."""
    thick = build_domain(p, p.n_thick, p.dt)
    thin = build_domain(p, p.n_thin, thick["dt"])
    return thin, thick, node_map(thin, thick, (p.n_thick - p.n_thin) * p.d)


def _node_coords(prob):
    nn = prob["ngll"] ** 3
    c = np.asarray(prob["coords"]).reshape(-1, 3)
    ib = np.asarray(prob["ibool"]).ravel()
    out = np.empty((prob["n_node"], 3))
    out[ib] = c
    return out


def node_map(thin: dict, thick: dict, shift: float) -> np.ndarray:
    """thick node id of every thin node (positions equal after shifting the
    thin mesh by `shift` in x and y)."""
    a = _node_coords(thin) + np.array([shift, shift, 0.0])
    b = _node_coords(thick)
    scale = 1e-6 * max(np.ptp(b[:, 0]), 1.0)
    qa = np.rint(a / scale).astype(np.int64)
    qb = np.rint(b / scale).astype(np.int64)
    ka = (qa[:, 0] * 1_000_003 + qa[:, 1]) * 1_000_033 + qa[:, 2]
    kb = (qb[:, 0] * 1_000_003 + qb[:, 1]) * 1_000_033 + qb[:, 2]
    order = np.argsort(kb)
    pos = np.searchsorted(kb[order], ka)
    pos = np.clip(pos, 0, kb.size - 1)
    hit = order[pos]
    if not np.all(np.all(qb[hit] == qa, axis=1)):
        raise ValueError("thin mesh nodes not found in the thick mesh")
    return hit.astype(np.int32)


# ---------------------------------------------------------------------------
# layer nodes: class (network), face frame
# ---------------------------------------------------------------------------

FACES = ("xmin", "xmax", "ymin", "ymax", "zmax")
# local axes (1-based global axis, signed; local 0 = outward normal)
FRAMES = {"xmin": (-1, 2, 3), "xmax": (1, 2, 3), "ymin": (-2, 1, 3), "ymax": (2, 1, 3), "zmax": (3, 1, 2)}


def layer_nodes(prob: dict, planes=None):
    """Nodes of the one-element layer cells of a thin domain: node ids, face
    frames and network index = (0 side face, 1 bottom) * 5 + depth plane
    (0 at the interior interface, 4 at the truncation surface).  A node in
    the layer of several faces takes the face it is deepest in.  ``planes``
    keeps only those depth planes (default: the truncation surface, where
    the missing outer domain acts on the thin one)."""
    d = prob["spec"].dx
    L = prob["n_layer"]
    ng = prob["ngll"]
    gll = mesh.gll_points(ng - 1)
    pos = (gll + 1.0) / 2.0  # fraction across an element
    X = _node_coords(prob)
    b = prob["bounds"]
    # distance into each face's layer, in elements (0 at the interface)
    inward = {
        "xmin": (b["xmin"] + L * d - X[:, 0]) / d,
        "xmax": (X[:, 0] - (b["xmax"] - L * d)) / d,
        "ymin": (b["ymin"] + L * d - X[:, 1]) / d,
        "ymax": (X[:, 1] - (b["ymax"] - L * d)) / d,
        "zmax": (X[:, 2] - (b["zmax"] - L * d)) / d,
    }
    best = np.full(X.shape[0], -1.0)
    face = np.full(X.shape[0], -1)
    for k, f in enumerate(FACES):
        dist = inward[f]
        take = (dist > -1e-9) & (dist > best + 1e-9)
        best[take] = dist[take]
        face[take] = k
    sel = np.nonzero(face >= 0)[0]
    plane = np.abs(best[sel][:, None] - pos[None, :]).argmin(axis=1)
    keep = np.isin(plane, list(planes if planes is not None else (ng - 1,)))
    sel, plane = sel[keep], plane[keep]
    fr = np.array([FRAMES[FACES[k]] for k in face[sel]], dtype=np.int8)
    net = np.where(face[sel] == 4, 1, 0) * ng + plane
    return sel.astype(np.int32), fr, net.astype(np.uint8), 2 * ng


class Layer:
    """Layer description passed through the C ABI."""

    def __init__(self, prob: dict, planes=None):
        self.node, self.frame, self.net, self.n_net = layer_nodes(prob, planes)
        self.desc = LayerDesc()
        self.desc.n_node = int(self.node.size)
        self.desc.node = _ptr(self.node, C.c_int32)
        self.desc.frame = self.frame.ctypes.data_as(C.POINTER(C.c_int8))
        self.desc.net = self.net.ctypes.data_as(C.POINTER(C.c_uint8))
        self.desc.n_net = int(self.n_net)


# ---------------------------------------------------------------------------
# training
# ---------------------------------------------------------------------------

class Trainer:
    def __init__(self, n_net: int, capacity: int, device: int = 0, seed: int = 0):
        self.lib = _bind(load_library())
        self.n_net = n_net
        h = C.c_void_p()
        _check(self.lib.gfb_trainer_create(n_net, int(capacity), device, int(seed), C.byref(h)))
        self.h = h

    def collect(self, thin: Solver, thick: Solver, thin_to_thick: np.ndarray, layer: Layer, n_steps: int,
                sample_stride: int = 1, node_stride: int = 1):
        m = np.ascontiguousarray(thin_to_thick, dtype=np.int32)
        _check(self.lib.gfb_trainer_collect(self.h, thin.h, thick.h, _ptr(m, C.c_int32), C.byref(layer.desc),
                                            int(n_steps), int(sample_stride), int(node_stride)))

    def samples(self) -> np.ndarray:
        c = np.zeros(self.n_net, dtype=np.int64)
        _check(self.lib.gfb_trainer_samples(self.h, c.ctypes.data_as(C.POINTER(C.c_int64))))
        return c

    def set_scales(self, scales):
        s = np.ascontiguousarray(scales, dtype=np.float32)
        _check(self.lib.gfb_trainer_set_scales(self.h, _ptr(s, C.c_float)))

    def evaluate(self) -> float:
        """Mean loss over every collected sample at the current parameters."""
        l = C.c_double()
        _check(self.lib.gfb_trainer_evaluate(self.h, C.byref(l)))
        return l.value

    def baseline_loss(self) -> float:
        """Mean loss of predicting zero on the collected samples (with the
        scales the fit uses): the yardstick of the fitted loss."""
        p, _ = self.params()
        self.set_params(np.zeros_like(p))
        l = self.evaluate()
        self.set_params(p)
        return l

    def fit(self, epochs: int, batch: int = 2048, lr: float = 1e-3, seed: int = 0):
        loss = np.zeros(max(epochs, 1))
        _check(self.lib.gfb_trainer_fit(self.h, int(epochs), int(batch), C.c_float(lr), int(seed),
                                        _ptr(loss, C.c_double)))
        return loss[:epochs]

    def gradient(self, net: int, x: np.ndarray, y: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        g = np.zeros(N_PARAMS, dtype=np.float32)
        loss = C.c_double()
        _check(self.lib.gfb_trainer_gradient(self.h, int(net), int(x.shape[0]), _ptr(x, C.c_float),
                                             _ptr(y, C.c_float), _ptr(g, C.c_float), C.byref(loss)))
        return g, loss.value

    def params(self):
        p = np.zeros((self.n_net, N_PARAMS), dtype=np.float32)
        s = np.zeros(4, dtype=np.float32)
        _check(self.lib.gfb_trainer_get_params(self.h, _ptr(p, C.c_float), _ptr(s, C.c_float)))
        return p, s

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(self.lib.gfb_trainer_set_params(self.h, _ptr(p, C.c_float)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.gfb_trainer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pack(params: np.ndarray) -> np.ndarray:
    lib = _bind(load_library())
    p = np.ascontiguousarray(params, dtype=np.float32)
    n_net = p.shape[0]
    w = np.zeros(n_net * N_WEIGHTS, dtype=np.uint16)
    _check(lib.gfb_layer_pack(n_net, _ptr(p, C.c_float), w.ctypes.data_as(C.POINTER(C.c_uint16))))
    return w


def attach(solver: Solver, layer: Layer, params: np.ndarray, scales: np.ndarray, threshold: float = 0.05):
    lib = _bind(load_library())
    w = pack(params)
    s = np.ascontiguousarray(scales, dtype=np.float32)
    _check(lib.gfb_layer_attach(solver.h, C.byref(layer.desc), w.ctypes.data_as(C.POINTER(C.c_uint16)),
                                _ptr(s, C.c_float), float(threshold)))
    solver._layer_keep = (layer, w, s)


def set_gains(solver: Solver, gains: np.ndarray):
    """Damping gains [n_net][3] of the attached layer (network, face axis)."""
    lib = _bind(load_library())
    g = np.ascontiguousarray(gains, dtype=np.float32)
    _check(lib.gfb_layer_set_gains(solver.h, int(g.shape[0]), _ptr(g, C.c_float)))


def status(solver: Solver):
    lib = _bind(load_library())
    a = C.c_int32()
    r = C.c_double()
    _check(lib.gfb_layer_status(solver.h, C.byref(a), C.byref(r)))
    return bool(a.value), r.value


def collect_pair(trainer: Trainer, p: PairSpec, dirs=(0, 1, 2), n_steps: Optional[int] = None,
                 sample_stride: int = 2, node_stride: int = 1, device: int = 0):
    """Replay one thin/thick pair into the trainer's data set."""
    thin, thick, m = build_pair(p)
    layer = Layer(thin)
    st = Solver(thin, dirs=dirs, precision=FP32, device=device, record=False)
    sk = Solver(thick, dirs=dirs, precision=FP32, device=device, record=False)
    trainer.collect(st, sk, m, layer, n_steps or p.nsteps, sample_stride, node_stride)
    st.close()
    sk.close()


# ---------------------------------------------------------------------------
# evaluation against the thick-C-PML reference run
# ---------------------------------------------------------------------------

def surface_records(prob: dict, snaps: dict, shift: float):
    """Recorded displacement of the interior surface cells, keyed by cell
    centre (so thin and thick runs can be matched)."""
    nn = prob["ngll"] ** 3
    rec = np.asarray(prob["recording"]["rec_cell_local"])
    c = np.asarray(prob["coords"]).reshape(prob["n_cell"], nn, 3)[rec].mean(axis=1) + np.array([shift, shift, 0.0])
    key = np.rint(c / 1e-3).astype(np.int64)
    return key, np.asarray(snaps["u"])  # [n_snap][n_rec][nn][3]


def surface_keys(prob: dict, shift: float = 0.0) -> np.ndarray:
    """Cell-centre keys of the recorded cells (see surface_records)."""
    return surface_records(prob, {"u": np.zeros(0)}, shift)[0]


def reflection_error(thin: dict, thin_snaps: dict, thick, thick_snaps: dict, shift: float) -> float:
    """||u_thin - u_thick|| / ||u_thick|| over every snapshot of the thin
    domain's recorded interior surface cells; `thick` is the thick problem
    or its surface_keys."""
    ka, ua = surface_records(thin, thin_snaps, shift)
    if isinstance(thick, dict):
        kb, ub = surface_records(thick, thick_snaps, 0.0)
    else:
        kb, ub = thick, np.asarray(thick_snaps["u"])
    idx = {tuple(k): i for i, k in enumerate(kb)}
    sel = [i for i, k in enumerate(ka) if tuple(k) in idx]
    if not sel:
        raise ValueError("no common recording cells")
    pick = [idx[tuple(ka[i])] for i in sel]
    a = ua[:, sel]
    b = ub[:, pick]
    n = min(a.shape[0], b.shape[0])
    return float(np.linalg.norm(a[:n] - b[:n]) / max(np.linalg.norm(b[:n]), 1e-300))


# ---------------------------------------------------------------------------
# closed loop: whole runs of the thin domain against the thick reference
# ---------------------------------------------------------------------------

def run_domain(prob: dict, params: Optional[np.ndarray] = None, scales: Optional[np.ndarray] = None,
               gains: Optional[np.ndarray] = None, scale_mult: float = 1.0, dirs=(0, 1, 2), device: int = 0,
               n_steps: Optional[int] = None, threshold: float = 0.05, chunk: int = 200, planes=None):
    """Step prob (FP32, wavefields ``dirs``; with the learned layer when
    ``params`` are given: output scale times ``scale_mult``, damping gains
    ``gains``, layer nodes on the depth ``planes``) and return
    ({field: {"u": float32 [n_snap][n_rec][nn][3]}}, device ms per step,
    layer status or None)."""
    n_steps = int(n_steps or prob["nsteps"])
    s = Solver(prob, dirs=list(dirs), precision=FP32, device=device, record_slots=16, flags=FLAG_RECORD_F32)
    try:
        if params is not None:
            sc = np.array(scales, dtype=np.float32)
            sc[3] *= scale_mult
            layer = Layer(prob, planes)
            attach(s, layer, params, sc, threshold=threshold)
            if gains is not None:
                set_gains(s, gains)
        us = {f: [] for f in range(len(dirs))}
        ms, done = 0.0, 0
        while done < n_steps:
            k = min(chunk, n_steps - done)
            ms += s.advance_timed(k)
            while s.pending() > 0:
                for f in range(len(dirs)):
                    u = np.empty((s.n_rec, s.nn, 3), dtype=np.float32)
                    s.read_record(f, release=f == len(dirs) - 1, out={"u": u})
                    us[f].append(u)
            done += k
        st = status(s) if params is not None else None
    finally:
        s.close()
    return {f: {"u": np.stack(us[f])} for f in us}, ms / max(n_steps, 1), st


class LoopCase:
    """A thin domain, the recorded surface displacement of its thick-C-PML
    reference run (the target of the closed-loop stage), and a solver of the
    thin domain kept for repeated runs: restored to its step-0 checkpoint
    and given a freshly attached layer before each."""

    def __init__(self, thin: dict, keys: np.ndarray, ref: dict, shift: float, dirs=(0, 1, 2), device: int = 0):
        self.thin, self.shift, self.dirs, self.device = thin, shift, tuple(dirs), device
        ka = surface_keys(thin, shift)
        idx = {tuple(k): i for i, k in enumerate(keys)}
        self.sel = np.array([i for i, k in enumerate(ka) if tuple(k) in idx], dtype=np.int64)
        if self.sel.size == 0:
            raise ValueError("no common recording cells")
        pick = np.array([idx[tuple(ka[i])] for i in self.sel], dtype=np.int64)
        self.ref = {f: np.asarray(ref[f]["u"])[:, pick] for f in ref}
        self._solver, self._blob, self._layers, self._plain = None, None, {}, None

    def _layer(self, planes):
        key = None if planes is None else tuple(planes)
        if key not in self._layers:
            self._layers[key] = Layer(self.thin, planes)
        return self._layers[key]

    def _errors(self, snaps) -> list:
        out = []
        for f, ref in self.ref.items():
            a = np.asarray(snaps[f]["u"])[:, self.sel]
            n = min(a.shape[0], ref.shape[0])
            out.append(float(np.linalg.norm(a[:n] - ref[:n]) / max(np.linalg.norm(ref[:n]), 1e-300)))
        return out

    def errors(self, params=None, scales=None, gains=None, scale_mult: float = 1.0, planes=None) -> list:
        """Reflection error of each wavefield with the given layer (none when
        params is None)."""
        if params is None:
            if self._plain is None:
                rec, _, _ = run_domain(self.thin, dirs=self.dirs, device=self.device)
                self._plain = self._errors(rec)
            return list(self._plain)
        if self._solver is None:
            s = Solver(self.thin, dirs=list(self.dirs), precision=FP32, device=self.device, record_slots=16,
                       flags=FLAG_RECORD_F32)
            attach(s, self._layer(None), np.zeros_like(params), np.ones(4, dtype=np.float32))
            self._solver, self._blob = s, s.checkpoint()
        s = self._solver
        s.restore(self._blob)
        sc = np.array(scales, dtype=np.float32)
        sc[3] *= scale_mult
        attach(s, self._layer(planes), params, sc)
        if gains is not None:
            set_gains(s, gains)
        n_steps, nf = int(self.thin["nsteps"]), len(self.dirs)
        us = {f: [] for f in range(nf)}
        done = 0
        while done < n_steps:
            k = min(200, n_steps - done)
            s.advance(k)
            s.synchronize()
            while s.pending() > 0:
                for f in range(nf):
                    u = np.empty((s.n_rec, s.nn, 3), dtype=np.float32)
                    s.read_record(f, release=f == nf - 1, out={"u": u})
                    us[f].append(u)
            done += k
        return self._errors({f: {"u": np.stack(us[f])} for f in us})

    def close(self):
        if self._solver is not None:
            self._solver.close()
            self._solver = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def loop_case(p: PairSpec, dirs=(0, 1, 2), device: int = 0) -> LoopCase:
    thick = build_domain(p, p.n_thick, p.dt)
    ref, _, _ = run_domain(thick, dirs=dirs, device=device)
    keys, dt = surface_keys(thick), thick["dt"]
    del thick
    return LoopCase(build_domain(p, p.n_thin, dt), keys, ref, (p.n_thick - p.n_thin) * p.d, dirs, device)


def case_errors(case: LoopCase, params=None, scales=None, gains=None, scale_mult: float = 1.0,
                device: int = 0, planes=None) -> list:
    """Reflection error of each wavefield of one case with the given layer
    (none when params is None)."""
    return case.errors(params, scales, gains, scale_mult, planes)


def loop_error(cases, params=None, scales=None, gains=None, scale_mult: float = 1.0, device: int = 0,
               planes=None) -> float:
    """RMS reflection error over the cases and their wavefields."""
    e = [x for c in cases for x in c.errors(params, scales, gains, scale_mult, planes)]
    return float(np.sqrt(np.mean(np.square(e))))


LOG_GAIN_BOUND = 6.0  # gains within e^-6 .. e^6 (the kernel caps the damping at m/dt anyway)


def fit_gains(cases, params: np.ndarray, scales: np.ndarray, nets=None, step: float = 1.0,
              min_step: float = 0.125, max_evals: int = 120, device: int = 0, planes=None,
              init: Optional[np.ndarray] = None):
    """Closed-loop stage of training: the damping gains [n_net][3] (one per
    network and face axis) that minimise the reflection error of whole runs
    of the training cases with the given networks, by coordinate search on
    log-gains (steps +-step, halved when a sweep brings no improvement,
    down to min_step).  ``nets``: the networks whose gains are fitted
    (default: those with nodes in the first case's layer; ``planes`` as in
    layer_nodes); ``init``: starting gains [n_net][3] (default 1).  Returns
    (gains, error, history of (evaluations, error))."""
    n_net = params.shape[0]
    if nets is None:
        nets = sorted(set(int(k) for k in Layer(cases[0].thin, planes).net))
    lg = np.zeros((n_net, 3)) if init is None else np.clip(np.log(np.maximum(np.asarray(init, dtype=np.float64),
                                                                            1e-30)), -LOG_GAIN_BOUND, LOG_GAIN_BOUND)
    best = loop_error(cases, params, scales, np.exp(lg), 1.0, device, planes)
    evals, hist = 1, [(1, best)]
    while step >= min_step and evals < max_evals:
        improved = False
        for k in nets:
            for j in range(3):
                for sgn in (1.0, -1.0):
                    if evals >= max_evals:
                        break
                    trial = lg.copy()
                    trial[k, j] = np.clip(trial[k, j] + sgn * step, -LOG_GAIN_BOUND, LOG_GAIN_BOUND)
                    if trial[k, j] == lg[k, j]:
                        continue
                    e = loop_error(cases, params, scales, np.exp(trial), 1.0, device, planes)
                    evals += 1
                    if e < best:
                        best, lg, improved = e, trial, True
                        hist.append((evals, best))
                        break
        if not improved:
            step *= 0.5
    return np.exp(lg).astype(np.float32), best, hist


W3_OFFSET = N_IN * N_HID + N_HID * N_HID  # W3 [3][64] in the FP32 parameters of a network


def scale_output_rows(params: np.ndarray, alpha: np.ndarray) -> np.ndarray:
    """Parameters with row j of network k's output layer W3 times
    alpha[k][j] (alpha 0: the constant damping softplus(0) on that axis;
    1: the network as given)."""
    p = np.array(params, dtype=np.float32, copy=True)
    w3 = p[:, W3_OFFSET:W3_OFFSET + N_OUT * N_HID].reshape(p.shape[0], N_OUT, N_HID)
    w3 *= np.asarray(alpha, dtype=np.float32)[:, :, None]
    return p


def fit_output_layer(cases, params: np.ndarray, scales: np.ndarray, gains: Optional[np.ndarray] = None,
                     nets=None, step: float = 0.5, min_step: float = 0.0625, max_alpha: float = 4.0,
                     max_evals: int = 60, device: int = 0, planes=None):
    """Closed-loop stage for the networks' output layer: a factor alpha per
    network and face axis on the rows of W3 (how much of the damping
    follows the network's reading of the node's history rather than the
    constant softplus(0)), fitted to the reflection error of whole runs of
    the training cases by coordinate search (steps +-step on alpha in
    [0, max_alpha], halved when a sweep brings no improvement, down to
    min_step), starting from the network as given (alpha = 1) with the
    given damping gains.  Returns (params with the fitted rows, alpha,
    error, history of (evaluations, error))."""
    n_net = params.shape[0]
    if nets is None:
        nets = sorted(set(int(k) for k in Layer(cases[0].thin, planes).net))
    alpha = np.ones((n_net, N_OUT))
    best = loop_error(cases, scale_output_rows(params, alpha), scales, gains, 1.0, device, planes)
    evals, hist = 1, [(1, best)]
    while step >= min_step and evals < max_evals:
        improved = False
        for k in nets:
            for j in range(N_OUT):
                for sgn in (1.0, -1.0):
                    if evals >= max_evals:
                        break
                    trial = alpha.copy()
                    trial[k, j] = np.clip(trial[k, j] + sgn * step, 0.0, max_alpha)
                    if trial[k, j] == alpha[k, j]:
                        continue
                    e = loop_error(cases, scale_output_rows(params, trial), scales, gains, 1.0, device, planes)
                    evals += 1
                    if e < best:
                        best, alpha, improved = e, trial, True
                        hist.append((evals, best))
                        break
        if not improved:
            step *= 0.5
    return scale_output_rows(params, alpha), alpha.astype(np.float32), best, hist
