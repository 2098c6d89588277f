"""Benchmark of the B200 CG-SEM elastic time loop.

Workload (N=1, default): the deformed heterogeneous mesh of 128 x 128 x 64
hexahedra of 200 m, polynomial order 4 (5 GLL points per axis, 131 M
element-local GLL points): jittered interior vertices, 8-sinusoid
topography, layered background with a Gaussian-correlated +-10 % velocity
perturbation, 5-element C-PML, 2 Hz Ricker point force, a 16 x 16-cell
recording tile; the x/y/z force directions advanced together in FP32 with
FP64 displacement/velocity accumulation.  Inputs come from the host
generator, whose arithmetic is the reference preprocessor's (its numbering
splits the nodes the reference's would), unless --gpu-prep.  One bench
"step" is one solver time step of all three wavefields over the whole mesh
(snapshots of the recording cells every 10 steps included).

Metric: GLL-point updates per second = n_cell * 125 * n_field * steps / time
(element-local points, as the reference's "~135M GLL points" count).

Arms:
  default          this repo's CUDA path through its C ABI (gfb)
  --impl reference the reference's own CPU functions (oracle/_ref, compiled
                   from the reference sources; the C restatement if absent)
                   on the host cores, on a sample of the same workload
  --accuracy       trace error of the FP32 batched path over the full run

Multi-GPU (torchrun): independent replicas, one per GPU ("replicas only":
the directions/models are independent; there is no data-path exchange).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "gf-only-sem_b200")
for _p in (REPO, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

from gfb.workloads import WORKLOADS, build_workload, split_nodes  # noqa: E402

# 32 independent models of uneven size stepped together
BATCH = dict(n_model=32, seed=4, d=250.0, pml=4, nmin=(16, 16, 8), nmax=(48, 48, 24), f0=(1.0, 3.0),
             steps=(1000, 3000), stride=50)

# learned one-element absorbing layer on a 96 x 96 x 48 layered
# model (interior 94 x 94 x 47), scored against the same interior with a
# 10-element C-PML; networks trained on replays of small seeded models
LAYER = {
    "layer96": dict(ni=94, nk=47, d=250.0, seed=2, steps=2000, stride=50,
                    train_pairs=24, train_ni=10, train_nk=6, train_steps=700, epochs=30,
                    loop_cases=3, loop_ni=16, loop_nk=8, loop_steps=800, loop_evals=100,
                    val_ni=22, val_nk=11, val_steps=900),
    "layer24": dict(ni=22, nk=11, d=250.0, seed=2, steps=900, stride=10,
                    train_pairs=6, train_ni=8, train_nk=5, train_steps=500, epochs=15,
                    loop_cases=3, loop_ni=12, loop_nk=6, loop_steps=600, loop_evals=80,
                    val_ni=16, val_nk=8, val_steps=600),
}

METRIC = "GLL-point updates/s (FP32 batched x/y/z, 1 B200)"
UNIT = "GLL-pt/s"


def batch_specs(seed: int = BATCH["seed"], n_model: int = BATCH["n_model"]):
    """Seeded descriptions of the uneven models: cells per axis, halfspace or
    layered material, source position, Ricker frequency and step count."""
    rng = np.random.default_rng(seed)
    d, pml = BATCH["d"], BATCH["pml"]
    out = []
    for k in range(n_model):
        nx, ny, nz = (int(rng.integers(lo, hi + 1)) for lo, hi in zip(BATCH["nmin"], BATCH["nmax"]))
        out.append(dict(
            nx=nx, ny=ny, nz=nz, layered=bool(rng.random() < 0.5), mseed=int(rng.integers(1 << 30)),
            vp=float(rng.uniform(4000.0, 7000.0)), vpvs=float(rng.uniform(1.6, 1.9)), rho=float(rng.uniform(2200.0, 3000.0)),
            src=(float(rng.uniform(pml + 1, nx - pml - 1) * d), float(rng.uniform(pml + 1, ny - pml - 1) * d),
                 float(rng.uniform(1.0, nz - pml - 1) * d)),
            f0=float(rng.uniform(*BATCH["f0"])), steps=int(rng.integers(BATCH["steps"][0], BATCH["steps"][1] + 1))))
    return out


def build_batch_model(sp):
    from gfb import mesh

    d, pml = BATCH["d"], BATCH["pml"]
    faces = {"xmin": pml, "xmax": pml, "ymin": pml, "ymax": pml, "zmax": pml}
    spec = mesh.MeshSpec(nx=sp["nx"], ny=sp["ny"], nz=sp["nz"], dx=d, dy=d, dz=d, order=4, pml=faces)
    mat = (mesh.seeded_layers(sp["mseed"], sp["nz"] * d) if sp["layered"]
           else mesh.homogeneous(sp["vp"], sp["vp"] / sp["vpvs"], sp["rho"]))
    p = mesh.build_problem(spec, mat, np.array(sp["src"]), nsteps=sp["steps"], snapshot_stride=BATCH["stride"],
                           record_depth_max_m=d, f0=sp["f0"])
    for k in ("coords", "vp", "vs"):  # not solver inputs
        p.pop(k, None)
    return p


def build_batch(threads: int = 8):
    from concurrent.futures import ThreadPoolExecutor

    specs = batch_specs()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        probs = list(ex.map(build_batch_model, specs))
    return specs, probs


def run_batch(args):
    """32 models of uneven size in one solver: one element launch per colour
    over all of them, the step replayed as a CUDA graph, kernel variant picked
    by the autotuner.  Reported: aggregate GLL-point updates/s over the whole
    run (every model to its last step) and each model's completion time."""
    import gfb

    t0 = time.perf_counter()
    specs, probs = build_batch()
    t_gen = time.perf_counter() - t0
    dirs = [0, 1, 2][: args.fields]
    n_steps = [sp["steps"] for sp in specs]
    flags = gfb.FLAG_RECORD_F32 | gfb.FLAG_AUTOTUNE
    t0 = time.perf_counter()
    b = gfb.BatchSolver(probs, dirs=dirs, precision=gfb.FP32, device=args.device, record_slots=8, flags=flags,
                        n_steps=n_steps)
    t_create = time.perf_counter() - t0
    info = b.info()
    consumer = RecordConsumer(b)
    order = sorted(set(n_steps))
    finish, done, dev_ms = {}, 0, 0.0
    with ClockSampler(args.device) as clk:
        consumer.start()
        for target in order:
            dev_ms += b.advance_timed(target - done)
            done = target
            finish[target] = dev_ms
        consumer.stop()
    launches = b.info()["kernel_launches"]
    b.drain()
    b.close()
    units = sum(p["n_cell"] * 125 * len(dirs) * n for p, n in zip(probs, n_steps))
    value = units / (dev_ms / 1e3)
    per_model = [{"cells": p["n_cell"], "steps": n, "finish_ms": finish[n],
                  "gll_pt_updates": p["n_cell"] * 125 * len(dirs) * n} for p, n in zip(probs, n_steps)]
    line = {
        "metric": "aggregate GLL-point updates/s, 32 uneven models batched (FP32 x/y/z, 1 B200)",
        "value": value, "unit": UNIT, "n_gpus": 1, "steps": max(n_steps), "warmup": 0,
        "ms_per_step": dev_ms / max(n_steps), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batch32", "n_model": len(probs), "cells_total": int(sum(p["n_cell"] for p in probs)),
                   "fields": len(dirs), "seed": BATCH["seed"], "generation_s": t_gen, "create_s": t_create,
                   "elem_kernel": "line" if info["elem_kernel"] else "point",
                   "cells_per_group": info["cells_per_group"], "elem_blocks": info["elem_blocks"],
                   "graph": True, "l2": "inputs larger than L2"},
        "per_model": per_model,
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


def run_layer(args):
    """Learned absorbing layer: train on replays, then the reflection error of
    the thin domain with and without the learned layer against the thick
    C-PML run, at the recorded interior surface cells."""
    import gfb
    from gfb import layer as gl

    w = LAYER[args.workload]
    rng = np.random.default_rng(w["seed"])
    d = w["d"]

    def pair(seed, ni, nk, steps, stride=10):
        r = np.random.default_rng(seed)
        return gl.PairSpec(ni=ni, nj=ni, nk=nk, d=d, seed=seed, f0=float(r.uniform(1.5, 2.5)),
                           src=(float(r.uniform(1.5, ni - 1.5) * d), float(r.uniform(1.5, ni - 1.5) * d),
                                float(r.uniform(1.0, nk - 1.5) * d)), nsteps=steps, stride=stride)

    t0 = time.perf_counter()
    p0 = pair(1, w["train_ni"], w["train_nk"], 10)
    n_net = gl.Layer(gl.build_domain(p0, 1)).n_net
    tr = gl.Trainer(n_net=n_net, capacity=8_000_000, device=args.device, seed=1)
    for k in range(w["train_pairs"]):
        gl.collect_pair(tr, pair(1000 + k, w["train_ni"], w["train_nk"], w["train_steps"]), sample_stride=3,
                        node_stride=2, device=args.device)
    t_collect = time.perf_counter() - t0
    base = tr.baseline_loss()
    t0 = time.perf_counter()
    loss = tr.fit(w["epochs"], batch=2048, lr=1e-3, seed=3)
    t_fit = time.perf_counter() - t0
    params, scales = tr.params()
    samples = int(tr.samples().sum())
    tr.close()

    def run(prob, weights=None, scale_mult=1.0, gains=None, planes=None):
        """Step prob with the layer when weights are given (its output
        scale times scale_mult, damping gains `gains`, nodes on the depth
        `planes`) and keep the recorded displacement (float32)."""
        return gl.run_domain(prob, weights, scales, gains, scale_mult, device=args.device, planes=planes)

    def rms(x):
        return float(np.sqrt(np.mean(np.square(x))))

    zero = params * 0.0  # untrained: constant damping softplus(0) on every axis
    # closed-loop stage of training: damping gains per network and face axis
    # fitted to the reflection error of whole runs of further training
    # models (their thick-C-PML runs are the targets), for the untrained and
    # for the replay-trained networks
    t0 = time.perf_counter()
    cases = [gl.loop_case(pair(3000 + k, w["loop_ni"], w["loop_nk"], w["loop_steps"]), device=args.device)
             for k in range(w["loop_cases"])]
    fits = {}
    all_planes = tuple(range(5))
    for name, wts, planes in (("untrained", zero, None), ("trained", params, None),
                              ("untrained, 5 planes", zero, all_planes)):
        init = None
        if planes:
            # start from the truncation surface's fit with the inner planes
            # undamped (unit damping on every plane reflects strongly)
            surface = sorted(set(int(k) for k in gl.Layer(cases[0].thin).net))
            init = np.full_like(fits["untrained"]["gains"], np.exp(-gl.LOG_GAIN_BOUND))
            init[surface] = fits["untrained"]["gains"][surface]
        g, e, hist = gl.fit_gains(cases, wts, scales, max_evals=w["loop_evals"] * (3 if planes else 1),
                                  device=args.device, planes=planes, init=init)
        fits[name] = dict(gains=g, train_error=e, start_error=hist[0][1], evals=hist[-1][0], planes=planes,
                          weights=wts)
    # then the replay-trained networks' output rows, with their gains: how
    # much of each axis's damping follows the network's reading of the history
    ft = fits["trained"]
    wts, alpha, e, hist = gl.fit_output_layer(cases, params, scales, ft["gains"], max_evals=w["loop_evals"],
                                              device=args.device)
    fits["trained, output rows"] = dict(gains=ft["gains"], train_error=e, start_error=hist[0][1],
                                        evals=hist[-1][0], planes=None, weights=wts, alpha=alpha)
    for c in cases:
        c.close()
    del cases
    t_loop = time.perf_counter() - t0

    # selection on held-out models: the candidates (replay-trained or
    # untrained networks at output scale x 0.25 .. 4 with unit gains, and
    # each network with its closed-loop gains) are compared by the
    # reflection error they give when stepping two validation models (seeds
    # of none of the training models nor the test model), and the best is
    # the layer that goes to the test model
    t0 = time.perf_counter()
    val = []
    for vseed in (5000, 5001):
        pv = pair(vseed, w["val_ni"], w["val_nk"], w["val_steps"], 10)
        thv = gl.build_domain(pv, pv.n_thick)
        thv_rec, _, _ = run(thv)
        keys, dtv = gl.surface_keys(thv), thv["dt"]
        del thv
        val.append((pv, gl.build_domain(pv, pv.n_thin, dtv), keys, thv_rec))
    cands = [(wname, wts, k, None, None) for wname, wts in (("trained", params), ("untrained", zero))
             for k in (0.25, 0.5, 1.0, 2.0, 4.0)]
    cands += [(f"{name} + closed-loop gains", f["weights"], 1.0, f["gains"], f["planes"]) for name, f in fits.items()]
    scores = []
    for wname, wts, k, g, planes in cands:
        errs = []
        for pv, tn, keys, thv_rec in val:
            rec, _, _ = run(tn, wts, k, g, planes)
            errs += [gl.reflection_error(tn, rec[f], keys, thv_rec[f], (pv.n_thick - pv.n_thin) * d)
                     for f in range(3)]
        scores.append(rms(errs))
    best = int(np.argmin(scores))
    sel_name, sel_w, sel_k, sel_g, sel_planes = cands[best]
    t_select = time.perf_counter() - t0
    del val

    # the test model: the thick-C-PML reference first, then (with the thick
    # problem freed) the thin domain at the same time step
    p = pair(w["seed"], w["ni"], w["nk"], w["steps"], w["stride"])
    thick = gl.build_domain(p, p.n_thick)
    shift = (p.n_thick - p.n_thin) * d
    thick_rec, ms_thick, _ = run(thick)
    thick_keys, thick_cells, dt = gl.surface_keys(thick), thick["n_cell"], thick["dt"]
    del thick
    thin = gl.build_domain(p, p.n_thin, dt)
    plain, ms_plain, _ = run(thin)
    selected, ms_learned, st = run(thin, sel_w, sel_k, sel_g, sel_planes)
    trained_k1, _, _ = run(thin, params, 1.0)
    untrained, _, _ = run(thin, zero, 1.0)
    loops = {name: run(thin, f["weights"], 1.0, f["gains"], f["planes"])[0] for name, f in fits.items()}

    def errs_of(snaps):
        return [gl.reflection_error(thin, snaps[f], thick_keys, thick_rec[f], shift) for f in range(3)]

    err_plain, err_sel, err_trained, err_untrained = (errs_of(x) for x in (plain, selected, trained_k1, untrained))
    err_loops = {name: errs_of(x) for name, x in loops.items()}
    value = rms(err_sel)
    line = {
        "metric": "reflection error of a learned 1-element absorbing layer vs a 10-element C-PML "
                  "(rel L2 of recorded surface displacement, x/y/z)",
        "value": value, "unit": "rel L2", "n_gpus": 1, "steps": w["steps"], "warmup": 0,
        "ms_per_step": ms_learned, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 solver, bf16 network weights", "data": "synthetic",
        "config": {"workload": args.workload, "thin_cells": thin["n_cell"], "thick_cells": thick_cells,
                   "fewer_elements": 1.0 - thin["n_cell"] / thick_cells,
                   "train_pairs": w["train_pairs"], "train_samples": samples, "epochs": w["epochs"],
                   "loss_zero_prediction": base, "loss_first_epoch": float(loss[0]) if len(loss) else None,
                   "loss_last_epoch": float(loss[-1]) if len(loss) else None,
                   "collect_s": t_collect, "fit_s": t_fit, "closed_loop_s": t_loop, "select_s": t_select},
        "closed_loop": {"on": f"{w['loop_cases']} training models {w['loop_ni']}x{w['loop_ni']}x{w['loop_nk']} "
                              f"cells, {w['loop_steps']} steps",
                        **{name: {"gains": {f"net {k}": [float(x) for x in f["gains"][k]]
                                            for k in sorted(set(int(q) for q in gl.Layer(thin, f["planes"]).net))},
                                  **({"output_row_factors": {f"net {k}": [float(x) for x in f["alpha"][k]]
                                                             for k in sorted(set(int(q) for q in gl.Layer(thin).net))}}
                                     if "alpha" in f else {}),
                                  "train_error_start": f["start_error"], "train_error_fitted": f["train_error"],
                                  "evaluations": f["evals"]} for name, f in fits.items()}},
        "selection": {"on": f"2 held-out models {w['val_ni']}x{w['val_ni']}x{w['val_nk']} cells, "
                            f"{w['val_steps']} steps",
                      "chosen": {"weights": sel_name, "output_scale_x": sel_k,
                                 "depth_planes": list(sel_planes) if sel_planes else [4]},
                      "validation_error": {f"{c[0]} x{c[2]}": sc for c, sc in zip(cands, scores)}},
        "reflection_error": {"learned_selected": err_sel, "thin_cpml_only": err_plain,
                             "trained_network_scale_x1": err_trained,
                             "untrained_network_constant_damping": err_untrained,
                             **{f"{name} + closed-loop gains": e for name, e in err_loops.items()}},
        "ms_per_step": {"thick_cpml": ms_thick, "thin_cpml_only": ms_plain, "thin_learned": ms_learned},
        "layer_active_at_end": bool(st[0]) if st else None, "monitored_residual": st[1] if st else None,
    }
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(seconds: float, dist, device: str) -> float:
    """Slowest rank's timed region (replicas run independently; the job
    finishes with the slowest)."""
    import torch

    t = torch.tensor([seconds], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_units(n_cell: int, n_field: int, steps: int, world: int) -> int:
    """GLL-point updates done by all replicas in the timed region."""
    return n_cell * 125 * n_field * steps * world


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").strip()
        ids = [x.strip() for x in vis.split(",") if x.strip()] if vis else []
        self.device = ids[device] if device < len(ids) else str(device)
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def node_pml_live_axes(prob):
    """Per global node: number of C-PML memory axes with a nonzero assembled
    coefficient (the node form keeps and updates only those)."""
    from gfb import mesh as gmesh

    nc, nn = prob["n_cell"], 125
    cells = np.nonzero(prob["pml_region"])[0]
    A = prob["pml_coef_abar"].reshape(nc, nn, 5)[cells]
    w = gmesh.gll_weights(gmesh.gll_points(4))
    wg = (w[:, None, None] * w[None, :, None] * w[None, None, :]).ravel()
    rho = prob["density"].reshape(nc, nn)[cells]
    jac = prob["jacobian"].reshape(nc, nn)[cells]
    scale = wg[None, :] * np.where(rho > 0, 1.0 / rho, 0.0) * jac
    ib = prob["ibool"].reshape(nc, nn)[cells]
    B = np.zeros((prob["n_node"], 5))
    for k in range(5):
        np.add.at(B[:, k], ib.ravel(), (scale * A[:, :, k]).ravel())
    has = np.zeros(prob["n_node"], dtype=bool)
    has[ib.ravel()[np.any(A != 0, axis=2).ravel()]] = True
    return int(has.sum()), int((B[:, 2:] != 0).sum())


def elem_bytes_per_step(prob, info, n_field, prec):
    """Algorithmic DRAM bytes of one step's element/assembly launches
    (unpadded component bytes; the [node][field][4] layout moves 4/3 of the
    gather/force bytes, visible in the ncu traffic).  With the force updated
    by increments (all but one step in the refresh period) every touch of a
    node reads and writes its force."""
    nn = 125
    P = prob["n_cell"] * nn
    G = prob["n_node"]
    sr = 4 if prec == 1 else 8
    F = 3 * n_field
    geom = P * 12 * sr + P * 4                      # geometry + ibool
    gather = P * F * sr                              # predicted displacement (or its increment)
    if info.get("force_refresh", 1) > 1:             # force by increments: every touch reads and writes
        force = P * F * sr * 2
    else:                                            # in full: first touch writes, others read+write
        force = G * F * sr + (P - G) * F * sr * 2
    pml = 0
    if info["n_pml_node"] == 0:                      # per-cell C-PML in this kernel
        Ppml = info["n_pml_cell"] * nn
        pml = Ppml * (15 * sr + F * 3 * sr * 2 + F * sr * 2 + F * 16 + F * sr)
    return geom + gather + force + pml


def node_bytes_per_step(prob, info, n_field, prec):
    """Algorithmic DRAM bytes of one step's node passes: per node and value
    u and v read and written (FP64; at plain nodes in the half-step velocity
    form the velocity is the half-step one in FP32 and there is no
    acceleration), the acceleration read and written (Real), the assembled
    force read and the next predicted displacement (or its increment)
    written (Real, unpadded), the mass (1/m in FP32); plus the node-form
    C-PML coefficients, previous field and memory of the live axes."""
    sr = 4 if prec == 1 else 8
    F = 3 * n_field
    n_pml = info["n_pml_node"]
    n_plain = prob["n_node"] - n_pml
    state = 16 + 8 if info.get("half_v") else 16 + 16 + 2 * sr   # u (+ w | v, a) read and written
    mass = 4 if prec == 1 else 8
    base = n_plain * (F * (state + 2 * sr) + mass) + n_pml * (F * (32 + 4 * sr) + mass)
    if n_pml > 0:                                    # node-form C-PML in this kernel
        n_live, live = node_pml_live_axes(prob)
        base += n_live * (14 * sr + F * sr * 2) + live * F * sr * 2
    return base


def committed_traffic():
    path = os.path.join(REPO, "profiles", "elem_col_traffic_deformed_64x64x32.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


def fp64_plain_sample(prob, device, args, fp32_value_per_gpu, peak):
    """The plain FP64 single-direction GPU path on the same workload (the
    denominator of the FP32-batched speed-up): one wavefield, FP64 state and
    arithmetic, per-cell C-PML as the reference lays it out.  Reported with
    its element kernel's fraction of the HBM roofline, so the speed-up can be
    read against how close that denominator is to its own bound."""
    import gfb

    s = gfb.Solver(prob, dirs=[0], precision=gfb.FP64, device=device, record_slots=8,
                   flags=gfb.FLAG_RECORD_F32 if args.record_f32 else 0)
    info = s.info()
    s.advance(args.warmup)
    s.drain()
    s.synchronize()
    n = max(20, args.steps // 4)
    consumer = RecordConsumer(s)
    consumer.start()
    ms = s.advance_timed(n) / n
    k = min(n, 50)
    ms_e, ms_n, ms_r = s.advance_profiled(k)
    consumer.stop()
    s.close()
    val = prob["n_cell"] * 125 * 1 / (ms / 1e3)
    eb = elem_bytes_per_step(prob, info, 1, 0)
    nb = node_bytes_per_step(prob, info, 1, 0)
    return {"value": val, "unit": UNIT, "steps": n, "ms_per_step": ms,
            "phases_ms_per_step": {"element": ms_e / k, "node": ms_n / k, "record": ms_r / k},
            "roofline_element": {"achieved": eb / (ms_e / k / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                                 "frac": eb / (ms_e / k / 1e3) / 1e9 / peak, "algorithmic_bytes_per_step": eb,
                                 "kernel": "elem_pipe_kernel<double,5,1> (all colour launches of a step)"},
            "roofline_node": {"achieved": nb / (ms_n / k / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                              "algorithmic_bytes_per_step": nb},
            "fp32_batched_over_fp64_plain": fp32_value_per_gpu / val}


def committed_accuracy(workload: str):
    """The trace error of the FP32 batched path on this workload as measured
    by `bench.py --accuracy` over the workload's full run and committed in
    profiles/accuracy_<workload>.json (None if not measured)."""
    path = os.path.join(REPO, "profiles", f"accuracy_{workload}.json")
    try:
        with open(path) as f:
            d = json.load(f)
    except Exception:
        return None
    return {"trace_rel_l2": d.get("value"), "gf_rel_l2": d.get("gf_rel_l2_worst"), "steps": d.get("steps"),
            "against": d.get("against"), "source": f"profiles/accuracy_{workload}.json (bench.py --accuracy)"}


def _cpu_piece(name, window, which, seconds, barrier, out):
    """One process of the aggregate CPU measurement (spawned): build its
    piece of the sample on the host, step it once, wait for the others, then
    time as many single-threaded steps as fit in about ``seconds``."""
    import time as _t

    from gfb.workloads import build_window

    import oracle

    try:
        prob = build_window(name, window, threads=1)
        run = oracle.Run(prob, 0, which, threads=1)
        t0 = _t.perf_counter()
        run.advance(1)
        n = max(1, int(seconds / max(_t.perf_counter() - t0, 1e-6)))
        barrier.wait(timeout=600)
        t0 = _t.perf_counter()
        run.advance(n)
        dt = _t.perf_counter() - t0
        out.put((prob["n_cell"] * 125 * n, dt, None))
        run.close()
    except BaseException as e:  # reported by the parent
        try:
            barrier.abort()
        except Exception:
            pass
        out.put((0, 0.0, repr(e)))


def cpu_measure(name: str, seconds: float = 12.0, max_procs: int = 64):
    """The reference's CPU functions (oracle/_ref when built, else the C
    restatement) on a sample of the workload -- the slab of cells through
    the source that gfb.workloads.sample_window picks -- in the two ways the
    reference can run on one host (its forward has no threads):
      single:    one process, one thread, the whole sample;
      aggregate: k processes of one thread each (k = the host cores this
                 process may use), each stepping its own 1/k of the sample
                 with no halo exchange, started together: an upper bound
                 for the reference's MPI build on these cores.
    Rates in GLL-point updates/s (one direction; every step includes the
    C-PML, source and snapshot work of the sample's cells)."""
    import multiprocessing as mp

    from gfb.workloads import WORKLOADS, build_window, host_threads, sample_window

    import oracle

    which = "ref" if os.path.exists(oracle.LIB_REF) else "oracle"
    win = sample_window(name)
    w = WORKLOADS[name]
    t0 = time.perf_counter()
    prob = build_window(name, win, threads=host_threads())
    t_gen = time.perf_counter() - t0
    cells = prob["n_cell"]
    pml_share = float(np.mean(prob["pml_region"] != 0)) if "pml_region" in prob else 0.0
    run = oracle.Run(prob, 0, which, threads=1)
    t0 = time.perf_counter()
    run.advance(1)
    n = max(1, int(seconds / max(time.perf_counter() - t0, 1e-6)))
    t0 = time.perf_counter()
    run.advance(n)
    dt1 = time.perf_counter() - t0
    run.close()
    del prob, run
    single = cells * 125 * n / dt1
    # aggregate: k processes over x-slices of the sample
    k = max(1, min(max_procs, host_threads(), win[1] - win[0]))
    xs = [win[0] + (win[1] - win[0]) * q // k for q in range(k + 1)]
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(k)
    out = ctx.Queue()
    procs = [ctx.Process(target=_cpu_piece, args=(name, (xs[q], xs[q + 1]) + tuple(win[2:]), which, seconds,
                                                  barrier, out), daemon=True) for q in range(k)]
    for pr in procs:
        pr.start()
    res = [out.get(timeout=1800) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
    errs = [r[2] for r in res if r[2]]
    if errs:
        raise RuntimeError(f"CPU measurement process failed: {errs[0]}")
    agg = sum(r[0] for r in res) / max(r[1] for r in res)
    full_cells = w["nx"] * w["ny"] * w["nz"]
    return {
        "kind": "reference" if which == "ref" else "port",
        "single": single, "single_steps": n, "aggregate": agg, "procs": k,
        "sample": f"cells i {win[0]}-{win[1] - 1}, j {win[2]}-{win[3] - 1}, k {win[4]}-{win[5] - 1} of the "
                  f"{w['nx']}x{w['ny']}x{w['nz']} mesh ({cells} of {full_cells} cells, C-PML share {pml_share:.3f}), "
                  f"full FP64 solver steps of direction x; single: one process, one thread, {n} steps; "
                  f"aggregate: {k} single-threaded processes on x-slices of the sample, about {seconds:.0f} s each, "
                  f"started together, no exchange",
        "generation_s": t_gen,
    }


class RecordConsumer(threading.Thread):
    """Releases each snapshot once it has reached pinned host memory, while
    the solver steps (the device-side throughput then includes the snapshot
    kernel and its device-to-host copy; converting into user arrays is part
    of the end-to-end number, where every snapshot is read out)."""

    def __init__(self, solver):
        super().__init__(daemon=True)
        self.s = solver
        self.halt = threading.Event()
        self.count = 0

    def _read_all(self):
        import ctypes as C

        import gfb

        step = C.c_int32()
        null = C.cast(None, C.POINTER(C.c_double))
        while self.s.pending() > 0:
            gfb._check(self.s.lib.gfb_read_record(self.s.h, 0, C.byref(step), null, null, null, null, 1))
            self.count += 1

    def run(self):
        while not self.halt.is_set():
            self._read_all()
            time.sleep(0.0005)
        self._read_all()

    def stop(self):
        self.halt.set()
        self.join()


def run_reference(args):
    """The reference's CPU implementation of the time loop on this host's
    cores (oracle/_ref: its own element_cpu.cpp, assembly.cpp and pml.cpp
    with the loop of solver.cpp:510-688 around them), timed on a sample of
    the workload: value = the aggregate rate of one single-threaded process
    per core, each stepping its own part of the sample (cpu_measure)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    m = cpu_measure(args.workload, seconds=args.cpu_seconds)
    val = m["aggregate"]
    w = WORKLOADS[args.workload]
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup,
        # one full-mesh step of one direction at the measured rate
        "ms_per_step": w["nx"] * w["ny"] * w["nz"] * 125 / val * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "ngll": 5, "directions": "x (y, z cost the same)"},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": m["procs"], "kind": m["kind"],
                         "sample": m["sample"], "single_thread": m["single"]},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the rate does not depend on the step count; each process times the steps that fit in "
                f"about {args.cpu_seconds:.0f} s after one warm-up step",
    }
    print(json.dumps(line), flush=True)
    return 0


def run_gfb(args):
    import gfb

    rank, world, local = dist_env()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(local)
        # every rank does the same work between collectives (input generation,
        # create, the timed steps), so a rank that is minutes late has failed:
        # a short timeout ends the others with an error instead of a hang
        tdist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=180))
        dist = tdist
    device = local if world > 1 else args.device
    prec = gfb.FP32 if args.precision == "fp32" else gfb.FP64
    dirs = [0, 1, 2][: args.fields]
    t_gen = time.perf_counter()
    # the ranks of one node generate their inputs at the same time: each
    # takes its share of the host cores
    from gfb.workloads import host_threads
    threads = max(1, host_threads() // max(1, int(os.environ.get("LOCAL_WORLD_SIZE", "1"))))
    prob = build_workload(args.workload, prep="gpu" if args.gpu_prep else "reference", device=device,
                          threads=threads)
    t_gen = time.perf_counter() - t_gen
    flags = (gfb.FLAG_RECORD_F32 if args.record_f32 else 0) | (gfb.FLAG_POINT_KERNEL if args.point_kernel else 0)
    s = gfb.Solver(prob, dirs=dirs, precision=prec, device=device, record_slots=8, flags=flags)
    info = s.info()
    if prec == gfb.FP32 and not args.point_kernel:
        kname = f"elem_col_kernel<5,{len(dirs)}>"
    else:
        kname = f"elem_pipe_kernel<{'float' if prec == gfb.FP32 else 'double'},5,{len(dirs)}>"
    s.advance(args.warmup)
    s.drain()
    s.synchronize()

    def barrier():
        if dist:
            import torch

            t = torch.zeros(1, device=f"cuda:{local}")
            dist.all_reduce(t)
            torch.cuda.synchronize(local)

    # timed region: K steps replayed as the captured step graph, one pair of
    # CUDA events on the solver's stream around them; snapshots are copied
    # out by a reader thread meanwhile
    barrier()
    s.synchronize()
    launches0 = s.info()["kernel_launches"]
    consumer = RecordConsumer(s)
    with ClockSampler(device) as clk:
        consumer.start()
        t0 = time.perf_counter()
        dev_ms = s.advance_timed(args.steps)
        t1 = time.perf_counter()
        consumer.stop()
    barrier()
    launches = s.info()["kernel_launches"] - launches0
    wall = t1 - t0
    elapsed = dev_ms / 1e3
    # per-phase device time: a further run of eagerly launched steps with
    # CUDA events between the phases
    n_prof = min(args.steps, 100)
    consumer = RecordConsumer(s)
    consumer.start()
    ms_elem, ms_node, ms_rec = (x * args.steps / n_prof for x in s.advance_profiled(n_prof))
    consumer.stop()
    if dist:
        elapsed = max_over_ranks(elapsed, dist, f"cuda:{local}")
    units = replica_units(prob["n_cell"], len(dirs), args.steps, world)
    value = units / elapsed
    s.drain()
    s.close()

    # end to end through the public API from host arrays: create (upload and
    # set-up), K steps with every snapshot read into host arrays by a second
    # thread as it arrives (Solver.run), destroy
    t0 = time.perf_counter()
    s2 = gfb.Solver(prob, dirs=dirs, precision=prec, device=device, record_slots=8, flags=flags)
    t_create = time.perf_counter() - t0
    up = s2.info()["upload_bytes"]
    rec = s2.run(args.steps, dtype=np.float32 if args.record_f32 else np.float64)
    s2.synchronize()
    s2.close()
    e2e_t = time.perf_counter() - t0
    rec_bytes = sum(np.asarray(rec[f][k]).size * (4 if args.record_f32 else 8) for f in rec
                    for k in ("strain", "u", "v", "a"))
    del rec
    e2e_val = prob["n_cell"] * 125 * len(dirs) * args.steps / e2e_t
    # the same over the workload's whole run (what a user of the solver sees:
    # set-up amortised over every step and every snapshot read out)
    e2e_full = None
    if not args.no_e2e_full:
        n_full = int(prob["nsteps"])
        t0 = time.perf_counter()
        s3 = gfb.Solver(prob, dirs=dirs, precision=prec, device=device, record_slots=8, flags=flags)
        t_create3 = time.perf_counter() - t0
        rec = s3.run(n_full, dtype=np.float32 if args.record_f32 else np.float64)
        s3.synchronize()
        s3.close()
        t_full = time.perf_counter() - t0
        rb = sum(np.asarray(rec[f][k]).size * (4 if args.record_f32 else 8) for f in rec
                 for k in ("strain", "u", "v", "a"))
        del rec
        e2e_full = {"value": prob["n_cell"] * 125 * len(dirs) * n_full / t_full, "unit": UNIT, "steps": n_full,
                    "create_s": t_create3, "total_s": t_full, "h2d_bytes_per_step": up / n_full,
                    "d2h_bytes_per_step": rb / n_full,
                    "note": "as e2e, over the workload's full step count"}

    peak, peak_kind = measured_peak_hbm()
    eb = elem_bytes_per_step(prob, info, len(dirs), prec)
    achieved = eb / (ms_elem / args.steps / 1e3) / 1e9
    nb = node_bytes_per_step(prob, info, len(dirs), prec)
    traffic = committed_traffic()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if prec == gfb.FP32 else "f64",
        "data": "synthetic",
        "config": {"workload": args.workload, "n_cell": prob["n_cell"], "ngll": 5, "n_node": prob["n_node"],
                   "fields": len(dirs), "precision": args.precision,
                   "state": ("f64 u, f32 half-step velocity at the plain nodes, f64 u,v + f32 a at the C-PML nodes"
                             if info["half_v"] else "f64 u,v"),
                   "l2": (f"inputs larger than L2 (geometry alone {prob['n_cell'] * 6000 / 1e6:.0f} MB)"
                          if prob["n_cell"] * 6000 > 126e6 else
                          f"inputs partly L2-resident (geometry {prob['n_cell'] * 6000 / 1e6:.0f} MB, L2 126 MB)"),
                   "parallelism": f"replicas{world}",
                   "n_colour": info["n_colour"], "n_pml_cell": info["n_pml_cell"],
                   "elem_blocks": info["elem_blocks"], "elem_variant": info["elem_variant"],
                   "force_refresh": info["force_refresh"],
                   "inputs": (f"GPU generator (gfb.prep, crack-free coordinates), {t_gen:.1f} s" if args.gpu_prep
                              else f"host generator (the reference preprocessor's arithmetic; numbering of its "
                                   f"points on the GPU, the same ids as the host lexsort), {t_gen:.1f} s"),
                   "split_nodes": split_nodes(prob),
                   "snapshots": f"every {prob['snapshot_stride']} steps, {info['n_rec_cell']} surface cells, "
                                f"{'float32' if args.record_f32 else 'float64'}, copied to pinned host memory during the step "
                                f"loop and released by a reader thread"},
        "phases_ms_per_step": {"element": ms_elem / args.steps, "node": ms_node / args.steps,
                               "record": ms_rec / args.steps, "wall": wall / args.steps * 1e3,
                               "note": f"phases from {n_prof} eagerly launched steps; value from the graph-replayed K"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "kernel": f"{kname} (all colour launches of a step)",
                     "algorithmic_bytes_per_step": eb,
                     "traffic": (traffic["bytes_per_cell"] * prob["n_cell"]
                                 if traffic and prec == gfb.FP32 and not args.point_kernel else None),
                     "traffic_source": (traffic or {}).get("source") if traffic else None},
        "roofline_node": {"achieved": nb / (ms_node / args.steps / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                          "algorithmic_bytes_per_step": nb},
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": up / args.steps,
                "d2h_bytes_per_step": rec_bytes / args.steps,
                "create_s": t_create, "total_s": e2e_t,
                "note": "gfb_create from host arrays + K steps with every snapshot read into host arrays "
                        "(Solver.run, in the recorded precision) + destroy"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if e2e_full:
        line["e2e_full_run"] = e2e_full
    acc = committed_accuracy(args.workload)
    if acc:
        line["accuracy"] = acc
    if rank == 0 and not args.no_plain:
        line["fp64_plain"] = fp64_plain_sample(prob, device, args, value / world, peak)
    del prob
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        m = cpu_measure(args.workload, seconds=args.cpu_seconds)
        line["cpu_baseline"] = {"value": m["aggregate"], "unit": UNIT, "cores": m["procs"], "kind": m["kind"],
                                "sample": m["sample"], "single_thread": m["single"]}
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_accuracy(args):
    """Relative L2 error of the FP32 batched x/y/z path over the workload's
    whole run (every snapshot of every recording cell: strain, u, v, a) and,
    on workloads with a recording tile, of the strain Green's functions
    merged per recording node.

    Against: on the CPU-runnable halfspace_20x20x10, the reference's own CPU
    functions (oracle/_ref) for direction x, with the FP64 GPU path checked
    against the same run; elsewhere the FP64 GPU path (x/y/z in one solver),
    which that comparison validates at <= 1e-10 (the CPU oracle cannot hold
    the larger meshes: per-cell C-PML arrays of 83 doubles per GLL point)."""
    import gfb
    from gfb.accuracy import QUANTITIES, TraceError, compare_solvers

    t_all = time.perf_counter()
    device = args.device
    n = args.accuracy_steps or WORKLOADS[args.workload]["nsteps"]
    prob = build_workload(args.workload, prep="gpu" if args.gpu_prep else "reference", device=device)
    dirs = [0, 1, 2]
    rs = 8
    flags = 0
    s32 = gfb.Solver(prob, dirs=dirs, precision=gfb.FP32, device=device, record_slots=rs, flags=flags)
    if args.force_refresh:
        s32.set_force_refresh(args.force_refresh)
    s64 = gfb.Solver(prob, dirs=dirs, precision=gfb.FP64, device=device, record_slots=rs, flags=flags)
    green = "recording" in prob and WORKLOADS[args.workload].get("tile") is not None
    out = {"workload": args.workload, "steps": n, "split_nodes": split_nodes(prob),
           "inputs": "GPU generator" if args.gpu_prep else "host generator, numbering on the GPU",
           "fp32_force_refresh": s32.info()["force_refresh"], "fp32_half_v": s32.info()["half_v"]}
    if args.workload == "halfspace_20x20x10":
        import oracle

        which = "ref" if os.path.exists(oracle.LIB_REF) else "oracle"
        from gfb.workloads import host_threads

        run = oracle.Run(prob, 0, which, threads=host_threads())
        e64, e32, e32_64 = TraceError(), TraceError(), TraceError()
        step = 0
        while step < n:
            k = min(100, n - step)
            ref = run.advance(k, step0=step)
            s64.advance(k)
            s32.advance(k)
            for i in range(len(ref["steps"])):
                for f in range(3):
                    a = s64.read_record(f, release=f == 2)
                    b = s32.read_record(f, release=f == 2)
                    for q in QUANTITIES:
                        if f == 0:
                            e64.add(q, a[q], ref[q][i])
                            e32.add(q, b[q], ref[q][i])
                        e32_64.add(f"{q}/{f}", b[q], a[q])
                e64.snapshots += 1
            step += k
        u, v, a = run.state()
        gu, gv, ga = s64.state(0)
        from numpy.linalg import norm

        final = {k: float(norm(x - y) / norm(y)) for k, x, y in (("u", gu, u), ("v", gv, v), ("a", ga, a))}
        run.close()
        out.update({
            "metric": "relative L2 trace error after the full run (FP32 batched x/y/z; FP64 GPU path)",
            "value": max(e32.worst(), e32_64.worst()), "unit": "rel L2",
            "against": f"reference CPU functions ({'oracle/_ref' if which == 'ref' else 'C restatement'}), "
                       "direction x; FP32 y/z against the FP64 GPU path",
            "trace_rel_l2": {"fp32_vs_cpu_x": e32.summary(), "fp32_vs_fp64_gpu": e32_64.summary(),
                             "fp64_gpu_vs_cpu_x": e64.summary(), "fp64_gpu_vs_cpu_final_state_x": final},
            "fp64_worst": max(e64.worst(), max(final.values())), "snapshots": e64.snapshots,
        })
    else:
        err = compare_solvers(s32, s64, n, chunk=rs * int(prob["snapshot_stride"]), green=green)
        out.update({
            "metric": "relative L2 trace error after the full run (FP32 batched x/y/z vs FP64 x/y/z)",
            "value": max(err.rel(k) for k in err.num if not k.startswith("green")), "unit": "rel L2",
            "against": "FP64 GPU path (x/y/z in one solver), validated against the reference's CPU functions "
                       "at <= 1e-10 on halfspace_20x20x10",
            "trace_rel_l2": {k: v for k, v in err.summary().items() if not k.startswith("green")},
            "snapshots": err.snapshots,
        })
        if green:
            g = {k: v for k, v in err.summary().items() if k.startswith("green")}
            out["gf_rel_l2"] = g
            out["gf_rel_l2_worst"] = max(g.values())
            out["gf_nodes"] = int(len(s32.rec_nodes()))
    s32.close()
    s64.close()
    out["wall_s"] = time.perf_counter() - t_all
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gfb", choices=["gfb", "reference"])
    ap.add_argument("--workload", default="deformed_128x128x64",
                    choices=sorted(WORKLOADS) + ["batch32"] + sorted(LAYER))
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--fields", type=int, default=3)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="seconds of stepping per process in the CPU measurements")
    ap.add_argument("--no-plain", action="store_true", help="skip the FP64 single-direction comparison")
    ap.add_argument("--no-e2e-full", action="store_true",
                    help="skip the end-to-end run over the workload's full step count")
    ap.add_argument("--point-kernel", action="store_true",
                    help="FP32 path with the thread-per-point element kernel instead of the line kernel")
    ap.add_argument("--gpu-prep", action="store_true",
                    help="compute every mesh input on the GPU (gfb.prep; crack-free coordinates) instead of "
                         "the host generator, whose arithmetic is the reference preprocessor's")
    ap.add_argument("--accuracy", action="store_true",
                    help="measure the FP32 batched path's trace error over the workload's full run instead")
    ap.add_argument("--accuracy-steps", type=int, default=0, help="steps of --accuracy (default: the full run)")
    ap.add_argument("--force-refresh", type=int, default=0,
                    help="FP32 steps between full element-force evaluations (default: the solver's, 800)")
    ap.add_argument("--record-f64", dest="record_f32", action="store_false",
                    help="snapshots in double (default: float, the reference example's snapshot_precision)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.accuracy:
        return run_accuracy(args)
    if args.workload == "batch32":
        return run_batch(args)
    if args.workload in LAYER:
        return run_layer(args)
    return run_gfb(args)


if __name__ == "__main__":
    sys.exit(main())
