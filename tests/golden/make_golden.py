"""Generate the golden fixtures in this directory from the reference itself.

Run in a container that has the reference tree (its path as the first
argument, or GF_REFERENCE_ROOT, else /root/reference) and
the oracle built (``make -C oracle``):

    python tests/golden/make_golden.py [REFERENCE_ROOT]

For each small case it
  1. builds a structured topology and calls the reference preprocessor's own
     numpy functions (imported with ``h5py`` stubbed, since they only need it
     for file I/O):
       gll_geometry.compute_gll_geometry, partition.compute_global_cell2global_node,
       pml_cpml.compute_cpml_parameters, source_locator.locate_source (buried
       mode), recording_map.build_recording_map, pml.compute_pml_damping;
  2. runs the reference's own compiled CPU functions (oracle/_ref, driven by
     oracle/ref_driver.cpp) for the time loop, recording traces at every
     snapshot;
  3. saves inputs and traces to ``<case>.npz``.

The tests never import the reference: they load these files.
"""

from __future__ import annotations

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "gf-only-sem_b200"))


def import_reference(ref_root: str):
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    sys.path.insert(0, ref_root)
    from preprocess import gll_geometry, partition, pml, pml_cpml, recording_map, source_locator
    from preprocess.topology_reader import TopologyData

    return types.SimpleNamespace(
        gll_geometry=gll_geometry,
        partition=partition,
        pml=pml,
        pml_cpml=pml_cpml,
        recording_map=recording_map,
        source_locator=source_locator,
        TopologyData=TopologyData,
    )


def structured_topology(R, V: np.ndarray, nx: int, ny: int, nz: int):
    """TopologyData for a structured hex mesh with per-cell faces/edges.

    Faces per cell in the order -z, +z, -y, +y, -x, +x; each face lists its
    four boundary edges; vertex ids are 1-based into the flattened grid.
    """
    vid = lambda i, j, k: (i * (ny + 1) + j) * (nz + 1) + k + 1  # noqa: E731
    verts = V.reshape(-1, 3)
    e2v, s2e, c2s = [], [], []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                corner = {}
                for a in (0, 1):
                    for b in (0, 1):
                        for c in (0, 1):
                            corner[(a, b, c)] = vid(i + a, j + b, k + c)
                faces = [
                    [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0)],  # -z
                    [(0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)],  # +z
                    [(0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1)],  # -y
                    [(0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1)],  # +y
                    [(0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1)],  # -x
                    [(1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1)],  # +x
                ]
                sids = []
                for f in faces:
                    eids = []
                    for q in range(4):
                        e2v.append([corner[f[q]], corner[f[(q + 1) % 4]]])
                        eids.append(len(e2v))
                    s2e.append(eids)
                    sids.append(len(s2e))
                c2s.append(sids)
    return R.TopologyData(
        vertex_to_coord=verts,
        edge_to_vertex=np.array(e2v, dtype=np.int64),
        surface_to_edge=np.array(s2e, dtype=np.int64),
        cell_to_surface=np.array(c2s, dtype=np.int64),
        n_vertex=len(verts),
        n_edge=len(e2v),
        n_surface=len(s2e),
        n_cell=len(c2s),
    )


CASES = {
    # homogeneous halfspace, 1-element C-PML on x/y/zmax, vertex source in
    # two non-PML cells (weights normalised across both)
    "halfspace_cpml_3x3x3": dict(
        nx=3, ny=3, nz=3, d=500.0, jitter=0.0, cpml=True, src=(1000.0, 1000.0, 500.0),
        nsteps=200, stride=10, depth=400.0, dirs=(0, 2), layered=False,
    ),
    # jittered vertices (non-diagonal Jacobian), layered material, legacy
    # ramp damping (no C-PML), source inside a cell
    "jitter_damping_3x3x3": dict(
        nx=3, ny=3, nz=3, d=500.0, jitter=0.12, cpml=False, src=(780.0, 820.0, 260.0),
        nsteps=160, stride=8, depth=400.0, dirs=(1,), layered=True,
    ),
}


def make_case(R, name: str, c: dict):
    from gfb import mesh

    import oracle

    spec = mesh.MeshSpec(
        nx=c["nx"], ny=c["ny"], nz=c["nz"], dx=c["d"], dy=c["d"], dz=c["d"], order=4,
        jitter=c["jitter"], seed=7, pml={"xmin": 1, "xmax": 1, "ymin": 1, "ymax": 1, "zmax": 1},
    )
    V = mesh.vertex_grid(spec)
    topo = structured_topology(R, V, spec.nx, spec.ny, spec.nz)
    N = spec.order
    coords, jac, dxi, mgeo = R.gll_geometry.compute_gll_geometry(topo, N)
    if c["layered"]:
        mat = mesh.layered([400.0, 1000.0], [4000.0, 5500.0, 6500.0], [2300.0, 3100.0, 3600.0],
                           [2400.0, 2600.0, 2800.0])
    else:
        mat = mesh.homogeneous()
    vp, vs, rho = mat(coords)
    mu = rho * vs**2
    lam = rho * (vp**2 - 2.0 * vs**2)
    mass = mgeo * rho
    bounds = {k: float(f(V[..., a])) for a, (k, f) in enumerate([("xmin", np.min), ("ymin", np.min), ("zmin", np.min)])}
    bounds.update({k: float(f(V[..., a])) for a, (k, f) in enumerate([("xmax", np.max), ("ymax", np.max), ("zmax", np.max)])})
    is_pml = mesh.pml_flags(spec)
    ibool, n_node = R.partition.compute_global_cell2global_node(coords)
    dt = 0.5 * mesh.h_min(coords) / float(vp.max())
    out = dict(
        coords=coords, jacobian=jac, dxi_dx=dxi, mass=mass, lam=lam, mu=mu, density=rho,
        ibool=ibool.astype(np.int32), n_node=np.int64(n_node), dt=np.float64(dt),
        is_pml=is_pml, vertices=V, nx=spec.nx, ny=spec.ny, nz=spec.nz, d=c["d"],
        jitter=c["jitter"], seed=7, layered=c["layered"], cpml=c["cpml"],
        src_xyz=np.array(c["src"]), nsteps=c["nsteps"], stride=c["stride"],
        depth=c["depth"], dirs=np.array(c["dirs"], dtype=np.int32),
    )
    widths = {k: (1 if k != "zmin" else 0) * c["d"] for k in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")}
    if c["cpml"]:
        cp = R.pml_cpml.compute_cpml_parameters(coords, is_pml, bounds, widths, vp, 2.0, dt)
        out["pml_region"] = cp["pml_region"].astype(np.int32)
        out["pml_coef_alpha"] = cp["pml_coef_alpha"]
        out["pml_coef_abar"] = cp["pml_coef_abar"]
        damping = np.zeros(jac.shape)
    else:
        damping = R.pml.compute_pml_damping(
            topo, coords, {"xmin": 1, "xmax": 1, "ymin": 1, "ymax": 1, "zmax": 1}, bounds, is_pml
        )
    out["damping"] = damping
    src = R.source_locator.locate_source(topo, np.array(c["src"]), coords, np.zeros(topo.n_surface, dtype=np.int64), N, is_pml=is_pml)
    out["src_cell_ids"] = src["cell_ids"].astype(np.int64)
    out["src_weights"] = src["weights"]
    rec = R.recording_map.build_recording_map(topo, bounds, is_pml, c["depth"], ibool, coords)
    r0 = rec["per_rank_recording"][0]
    out["record_depth_actual_m"] = rec["record_depth_actual_m"]
    out["rec_cell_local"] = np.array(r0["rec_cell_local_index"], dtype=np.int32)
    out["gll_node_ids"] = np.array(r0["gll_node_ids"], dtype=np.int64)
    out["gll_node_coords"] = np.array(r0["gll_node_coords"], dtype=np.float64)
    out["cell_gll_node_index"] = np.array(r0["cell_gll_node_index"], dtype=np.int32)
    t = np.arange(c["nsteps"]) * dt
    out["stf"] = mesh.ricker(t)
    prob = {
        "n_cell": spec.n_cell, "ngll": N + 1, "n_node": n_node, "ibool": ibool,
        "cell_ids": np.arange(spec.n_cell, dtype=np.int64), "dxi_dx": dxi, "jacobian": jac,
        "lambda": lam, "mu": mu, "density": rho, "mass": mass, "damping": damping,
        "dt": dt, "snapshot_stride": c["stride"], "src_cell_ids": out["src_cell_ids"],
        "src_weights": out["src_weights"], "stf": out["stf"],
        "recording": {"rec_cell_local": out["rec_cell_local"]},
    }
    if c["cpml"]:
        prob.update(pml_region=out["pml_region"], pml_coef_alpha=out["pml_coef_alpha"], pml_coef_abar=out["pml_coef_abar"])
    for d in c["dirs"]:
        run = oracle.Run(prob, d, "ref")
        snaps = run.advance(c["nsteps"])
        u, v, a = run.state()
        out[f"trace_steps_{d}"] = snaps["steps"]
        for key in ("strain", "u", "v", "a"):
            out[f"trace_{key}_{d}"] = snaps[key]
        out[f"final_u_{d}"] = u
        out[f"final_v_{d}"] = v
        out[f"final_a_{d}"] = a
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, {k: np.asarray(v).shape for k, v in out.items() if np.asarray(v).size > 1})


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GF_REFERENCE_ROOT", "/root/reference")
    R = import_reference(ref_root)
    for name, c in CASES.items():
        make_case(R, name, c)


if __name__ == "__main__":
    main()
