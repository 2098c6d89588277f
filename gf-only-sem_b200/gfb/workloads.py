"""Named synthetic workloads: the model sizes, materials and run lengths the
solver is measured and checked on, built with gfb.mesh.

* ``halfspace_20x20x10`` -- homogeneous elastic halfspace, 20 x 20 x 10
  cells of 500 m, order 4, vp/vs/rho 6000/3464/2700, 3-cell C-PML on x/y and
  the bottom, free top, point force at (5 km, 5 km, 1 km), 2 Hz Ricker,
  2000 steps, every surface cell (500 m deep) recorded every 10 steps.  Small
  enough for the CPU oracle to run in full.
* ``layered_64x64x32`` -- three seeded flat layers (vp 3000-7000 m/s,
  vp/vs 1.6-1.9, rho 2200-3000), 64 x 64 x 32 cells of 250 m, 4-cell C-PML,
  4000 steps.
* ``deformed_128x128x64`` -- 128 x 128 x 64 cells of 200 m (135 M GLL
  points): interior vertices jittered by a seeded +-10 % of the edge, a top
  surface of 8 random-phase sinusoids of at most 300 m, the layered
  background scaled by (1 + 0.1 g) with g a seeded Gaussian-correlated field
  (150 m correlation length), 5-cell C-PML, 6000 steps, recording on a
  16 x 16-cell surface tile (strain Green's functions).
* ``layered_40x40x20`` / ``deformed_32x32x16`` -- the same constructions at
  sizes for profiling and quick checks.

Inputs (``prep``):
  ``"reference"`` -- geometry, materials and C-PML coefficients by the host
      generator (the reference preprocessor's arithmetic, so on deformed
      meshes its numbering splits the nodes that partition.py would split);
      the numbering of those points runs on the GPU when ``device`` is given
      (the same ids as the host lexsort of the same points), else on the host.
  ``"gpu"`` -- every input computed on the GPU (gfb.prep): crack-free
      coordinates, so no split nodes.
"""

from __future__ import annotations

import os
from typing import Optional

import numpy as np

WORKLOADS = {
    "halfspace_20x20x10": dict(nx=20, ny=20, nz=10, d=500.0, pml=3, seed=0, src=(5000.0, 5000.0, 1000.0),
                               nsteps=2000, stride=10, depth=500.0),
    "layered_64x64x32": dict(nx=64, ny=64, nz=32, d=250.0, pml=4, seed=2, src=(8000.0, 8000.0, 2000.0),
                             nsteps=4000, stride=10, depth=250.0),
    "layered_40x40x20": dict(nx=40, ny=40, nz=20, d=400.0, pml=4, seed=2, src=(8000.0, 8000.0, 2000.0),
                             nsteps=2500, stride=10, depth=400.0),
    "deformed_128x128x64": dict(nx=128, ny=128, nz=64, d=200.0, pml=5, seed=3, src=(12800.0, 12800.0, 2000.0),
                                nsteps=6000, stride=10, depth=200.0, jitter=0.1, topo=(8, 300.0), corr=150.0,
                                pert=0.1, tile=16),
    "deformed_64x64x32": dict(nx=64, ny=64, nz=32, d=200.0, pml=5, seed=3, src=(6400.0, 6400.0, 2000.0),
                              nsteps=3000, stride=10, depth=200.0, jitter=0.1, topo=(8, 300.0), corr=150.0,
                              pert=0.1, tile=16),
    "deformed_32x32x16": dict(nx=32, ny=32, nz=16, d=200.0, pml=5, seed=3, src=(3200.0, 3200.0, 1400.0),
                              nsteps=1500, stride=10, depth=200.0, jitter=0.1, topo=(8, 300.0), corr=150.0,
                              pert=0.1, tile=8),
}


def _model(name: str):
    """(parameters, MeshSpec, material function, recording tile) of a workload."""
    from . import mesh

    w = WORKLOADS[name]
    pml = {"xmin": w["pml"], "xmax": w["pml"], "ymin": w["pml"], "ymax": w["pml"], "zmax": w["pml"]}
    topo = w.get("topo", (0, 0.0))
    spec = mesh.MeshSpec(nx=w["nx"], ny=w["ny"], nz=w["nz"], dx=w["d"], dy=w["d"], dz=w["d"], order=4, pml=pml,
                         jitter=w.get("jitter", 0.0), topo_terms=topo[0], topo_amp=topo[1], seed=w["seed"])
    tile = None
    if name.startswith("layered"):
        mat = mesh.seeded_layers(w["seed"], w["nz"] * w["d"])
    elif name.startswith("deformed"):
        d = w["d"]
        lo = (-d, -d, -d)
        hi = (w["nx"] * d + d, w["ny"] * d + d, w["nz"] * d + 2.0 * topo[1] + d)
        field = mesh.gaussian_field(lo, hi, w["corr"], w["seed"] + 1)
        mat = mesh.perturbed(mesh.seeded_layers(w["seed"], w["nz"] * d), field, w["pert"])
        n = w["tile"]
        tile = ((w["nx"] - n) // 2, (w["ny"] - n) // 2, n)
    else:
        mat = mesh.homogeneous()
    return w, spec, mat, tile


def build_workload(name: str, prep: str = "reference", device: Optional[int] = None,
                   threads: Optional[int] = None) -> dict:
    """Solver inputs of a named workload (reference layouts, gfb.mesh).

    prep = "reference" (host generator; numbering on GPU ``device`` if
    given) or "gpu" (every input on GPU ``device``)."""
    from . import mesh

    if prep not in ("reference", "gpu"):
        raise ValueError(f"prep must be 'reference' or 'gpu', not {prep!r}")
    if prep == "gpu" and device is None:
        raise ValueError("prep='gpu' needs a device")
    w, spec, mat, tile = _model(name)
    if threads is None:
        threads = host_threads()
    return mesh.build_problem(spec, mat, np.array(w["src"]), nsteps=w["nsteps"], snapshot_stride=w["stride"],
                              record_depth_max_m=w["depth"], record_tile=tile,
                              device=device if prep == "gpu" else None,
                              numbering_device=device if prep == "reference" else None, threads=threads)


def host_threads() -> int:
    """Host cores this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def split_nodes(prob: dict) -> int:
    """Nodes the numbering gives beyond the (4n+1) per axis of a structured
    order-4 mesh: copies of a shared point whose coordinates differ in the
    last bits (0 for crack-free inputs)."""
    sp = prob["spec"]
    o = sp.order
    return int(prob["n_node"]) - (o * sp.nx + 1) * (o * sp.ny + 1) * (o * sp.nz + 1)


def sample_window(name: str, max_cells: int = 65536):
    """The cells the CPU measurements step: a slab of whole x rows and z
    columns through the source (y rows j0 .. j1-1), at most max_cells cells
    (the whole mesh when it is that small).  Returns (i0, i1, j0, j1, k0, k1)."""
    w = WORKLOADS[name]
    nx, ny, nz = w["nx"], w["ny"], w["nz"]
    rows = max(1, min(ny, max_cells // (nx * nz)))
    js = int(w["src"][1] // w["d"])
    j0 = max(0, min(ny - rows, js - rows // 2))
    return (0, nx, j0, j0 + rows, 0, nz)


def build_window(name: str, window, threads: int = 1, with_source: bool = True) -> dict:
    """Inputs of the cells of ``window`` of a named workload, computed by the
    host generator alone (no GPU): the same model, vertices and C-PML layers
    as the full mesh.  Without ``with_source``, or when the source lies
    outside the window, the piece has no source."""
    from . import mesh

    w, spec, mat, _ = _model(name)
    src = np.array(w["src"]) if with_source else np.array([-1e30, -1e30, -1e30])
    return mesh.build_problem(spec, mat, src, nsteps=w["nsteps"], snapshot_stride=w["stride"],
                              record_depth_max_m=w["depth"], threads=threads, cell_window=tuple(window),
                              require_source=False)
