"""Input and output files of the file-level driver (gf_solver_elastic_cuda,
gfb_run_forward) in the raw ``.gfr`` container.

The container holds the same dataset and attribute names as the
reference's HDF5 files; its layout (csrc/gfb_files.h) is: "GFBRAW01", u32
entry count, then per entry u16 name length, name (a dataset path, or
"<object>@<attribute>"), u8 type, u8 ndim, u64 dims, u64 offset, u64 bytes;
data blocks on 64-byte boundaries.

``write_case`` lays out a working directory the way the reference's
preprocessor does (config + partitions/partition_{r}, model_writer.py:245-470,
config_writer.py) from a problem dict of gfb.mesh, split into R partitions;
``merge_partitions`` restates read_partition_all (io.cpp:319-450) in numpy,
the check of the driver's own merge.
"""

from __future__ import annotations

import os
import struct
from typing import Dict, Optional, Sequence

import numpy as np

MAGIC = b"GFBRAW01"
_TYPES = {1: np.float64, 2: np.float32, 3: np.int64, 4: np.int32, 5: np.uint8}
_CODES = {np.dtype(np.float64): 1, np.dtype(np.float32): 2, np.dtype(np.int64): 3, np.dtype(np.int32): 4,
          np.dtype(np.uint8): 5, np.dtype(np.bool_): 5}


def write(path: str, entries: Dict[str, object]):
    """Write a container: name -> ndarray / number / str / bool.  Names with
    '@' are attributes ("/simulation@solver_dt"); scalars become 0-d
    entries of their type (int -> int32, float -> float64)."""
    items = []
    for name, v in entries.items():
        if isinstance(v, str):
            data = v.encode()
            items.append((name, 6, (len(data),), data))
            continue
        if isinstance(v, (bool, np.bool_)):
            a = np.asarray(v, dtype=np.uint8)
        elif isinstance(v, (int, np.integer)) and not isinstance(v, np.ndarray):
            a = np.asarray(v, dtype=np.int32)
        elif isinstance(v, float):
            a = np.asarray(v, dtype=np.float64)
        else:
            a = np.asarray(v)
        if a.dtype not in _CODES:
            raise TypeError(f"{name}: unsupported dtype {a.dtype}")
        a = np.array(a.astype(np.uint8) if a.dtype == np.bool_ else a, order="C", copy=True)
        items.append((name, _CODES[a.dtype], a.shape, a.tobytes()))
    header = 8 + 4 + sum(2 + len(n.encode()) + 2 + 8 * len(sh) + 16 for n, _, sh, _ in items)
    off = (header + 63) // 64 * 64
    offs = []
    for _, _, _, data in items:
        offs.append(off)
        off = (off + len(data) + 63) // 64 * 64
    with open(path, "wb") as f:
        f.write(MAGIC + struct.pack("<I", len(items)))
        for (name, code, shape, data), o in zip(items, offs):
            nb = name.encode()
            f.write(struct.pack("<H", len(nb)) + nb + struct.pack("<BB", code, len(shape)))
            f.write(b"".join(struct.pack("<Q", int(d)) for d in shape))
            f.write(struct.pack("<QQ", o, len(data)))
        pos = header
        for (_, _, _, data), o in zip(items, offs):
            f.write(b"\0" * (o - pos))
            f.write(data)
            pos = o + len(data)


def read(path: str) -> Dict[str, object]:
    """Read a container into name -> ndarray (0-d for scalars) or str."""
    out = {}
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != MAGIC:
        raise ValueError(f"{path} is not a GFBRAW01 container")
    (n,) = struct.unpack_from("<I", buf, 8)
    p = 12
    for _ in range(n):
        (ln,) = struct.unpack_from("<H", buf, p)
        p += 2
        name = buf[p:p + ln].decode()
        p += ln
        code, nd = struct.unpack_from("<BB", buf, p)
        p += 2
        shape = struct.unpack_from("<" + "Q" * nd, buf, p)
        p += 8 * nd
        off, nbytes = struct.unpack_from("<QQ", buf, p)
        p += 16
        raw = buf[off:off + nbytes]
        if code == 6:
            out[name] = raw.decode()
        else:
            out[name] = np.frombuffer(raw, dtype=_TYPES[code]).reshape(shape).copy()
    return out


def partition_cells(n_cell: int, n_part: int, spec=None) -> np.ndarray:
    """Rank of every cell: slabs along x of a structured mesh (cells are
    numbered x fastest), so every partition holds cells of every row and the
    merged order differs from the model's."""
    if spec is None:
        return (np.arange(n_cell) * n_part // max(n_cell, 1)).astype(np.int32)
    i = np.arange(n_cell) % spec.nx
    return (i * n_part // spec.nx).astype(np.int32)


def write_case(root: str, prob: dict, n_part: int = 1, snapshot_precision: str = "float64",
               log_stride: int = 100, restart_stride: int = 0, nsteps: Optional[int] = None,
               element_to_rank: Optional[np.ndarray] = None):
    """config.gfr and partitions/partition_{r}.gfr for a problem dict of
    gfb.mesh, the cells split over n_part partitions.  Global node ids are
    the problem's ibool (the reference's local_cell2global_node); each
    partition's own compact numbering (local_cell2rank_node) numbers its
    nodes in order of first use.  Returns the rank of every cell."""
    os.makedirs(os.path.join(root, "partitions"), exist_ok=True)
    nc, ng = int(prob["n_cell"]), int(prob["ngll"])
    nn = ng**3
    rank = (partition_cells(nc, n_part, prob.get("spec")) if element_to_rank is None
            else np.asarray(element_to_rank, dtype=np.int32))
    ibool = np.asarray(prob["ibool"]).reshape(nc, nn).astype(np.int32)
    rec = prob.get("recording")
    rec_cells = np.asarray(rec["rec_cell_local"], dtype=np.int64) if rec is not None else np.zeros(0, np.int64)
    nsteps = int(prob["nsteps"]) if nsteps is None else int(nsteps)
    cfg = {
        "/simulation@title": "gfb case",
        "/simulation@polynomial_order": ng - 1,
        "/simulation@solver_dt": float(prob["dt"]),
        "/simulation@output_dt_s": float(prob["dt"]) * int(prob["snapshot_stride"]),
        "/simulation@snapshot_stride": int(prob["snapshot_stride"]),
        "/simulation@nsteps": nsteps,
        "/simulation@cfl_safety": 0.5,
        "/simulation@snapshot_precision": snapshot_precision,
        "/simulation@record_depth_max_m": float(rec.get("record_depth_actual_m", 0.0)) if rec is not None else 0.0,
        "/simulation@record_depth_actual_m": float(rec.get("record_depth_actual_m", 0.0)) if rec is not None else 0.0,
        "/simulation@log_stride": int(log_stride),
        "/simulation@restart_stride": int(restart_stride),
        "/source/stf_t": np.asarray(prob["stf_t"], dtype=np.float64) if "stf_t" in prob else
        np.arange(len(prob["stf"])) * float(prob["dt"]),
        "/source/stf_values": np.asarray(prob["stf"], dtype=np.float64),
        "/source@x": 0.0, "/source@y": 0.0, "/source@z": 0.0,
        "/source/cells/cell_ids": np.asarray(prob["src_cell_ids"], dtype=np.int64),
        "/source/cells/weights": np.asarray(prob["src_weights"], dtype=np.float64).reshape(-1, ng, ng, ng),
    }
    b = prob.get("bounds") or {}
    for k in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax"):
        cfg[f"/domain@{k}"] = float(b.get(k, 0.0))
    write(os.path.join(root, "config.gfr"), cfg)
    coords = prob.get("coords")
    for r in range(n_part):
        cells = np.nonzero(rank == r)[0]
        e = {}

        def cell_field(key, name=None, shape=(ng, ng, ng)):
            a = prob.get(key)
            if a is None:
                return
            a = np.asarray(a)
            per = a.size // nc
            tail = shape + ((per // nn,) if per != nn else ())
            e[f"/field/cell/{name or key}"] = np.ascontiguousarray(a.reshape((nc,) + tail)[cells])

        for key in ("jacobian", "mass", "vp", "vs", "density", "lambda", "mu", "damping"):
            cell_field(key)
        cell_field("dxi_dx")
        if coords is not None:
            cell_field("coords")
        else:
            e["/field/cell/coords"] = np.zeros((cells.size, ng, ng, ng, 3))
        if "pml_coef_abar" in prob:
            cell_field("pml_coef_alpha")
            cell_field("pml_coef_abar")
            e["/field/cell/pml_region"] = np.asarray(prob["pml_region"], dtype=np.int32)[cells]
        gl = ibool[cells]
        _, compact = np.unique(gl.ravel(), return_inverse=True)
        e["/field/cell/local_cell2global_node"] = gl.ravel()
        e["/field/cell/local_cell2rank_node"] = compact.astype(np.int32)
        e["/field/cell@n_rank_node"] = int(compact.max()) + 1 if compact.size else 0
        e["/partition@n_ranks"] = int(n_part)
        e["/partition/element_to_rank"] = rank
        e["/partition/local_cell_ids"] = np.asarray(prob["cell_ids"], dtype=np.int64)[cells]
        mine = np.nonzero(rank[rec_cells] == r)[0] if rec_cells.size else np.zeros(0, np.int64)
        if mine.size:
            rc = rec_cells[mine]
            local = np.searchsorted(cells, rc).astype(np.int32)
            nodes = ibool[rc]
            ids, inv = np.unique(nodes.ravel(), return_inverse=True)
            cflat = coords.reshape(nc * nn, 3) if coords is not None else None
            first = np.zeros(ids.size, dtype=np.int64)
            first[inv[::-1]] = (rc[:, None] * nn + np.arange(nn)[None, :]).ravel()[::-1]
            e["/recording@basis"] = "gll"
            e["/recording@excludes_pml"] = True
            e["/recording/gll_node_ids"] = ids.astype(np.int64)
            e["/recording/gll_node_coords"] = (cflat[first] if cflat is not None else np.zeros((ids.size, 3)))
            e["/recording/rec_cell_local"] = local
            e["/recording/rec_cell_global_ids"] = rc.astype(np.int64)
            e["/recording/cell_gll_node_index"] = inv.astype(np.int32)
            e["/recording@n_unique_gll"] = int(ids.size)
            e["/recording@n_rec_cell"] = int(rc.size)
        write(os.path.join(root, "partitions", f"partition_{r}.gfr"), e)
    return rank


def merge_partitions(parts: Sequence[dict]) -> dict:
    """read_partition_all (io.cpp:319-450) over containers read with
    ``read``: concatenation in partition order, merged ibool from
    local_cell2global_node, recording nodes deduplicated by global id in
    first-seen order, rec_cell_local offset by the cells before the
    partition, cell_gll_node_index remapped, n_rank_node = max id + 1."""
    R = "recording/"
    out = {"local_cell_ids": [], "local_cell2rank_node": [], R + "gll_node_ids": [], R + "gll_node_coords": [],
           R + "rec_cell_local": [], R + "rec_cell_global_ids": [], R + "cell_gll_node_index": []}
    fields = ("jacobian", "dxi_dx", "mass", "density", "lambda", "mu", "damping", "pml_coef_alpha", "pml_coef_abar")
    for k in fields:
        out[k] = []
    out["pml_region"] = []
    index = {}
    cum = 0
    for p in parts:
        n = int(p["/partition/local_cell_ids"].size)
        out["local_cell_ids"].append(p["/partition/local_cell_ids"])
        out["local_cell2rank_node"].append(p["/field/cell/local_cell2global_node"].ravel())
        for k in fields:
            if f"/field/cell/{k}" in p:
                out[k].append(p[f"/field/cell/{k}"].ravel())
        if "/field/cell/pml_region" in p:
            out["pml_region"].append(p["/field/cell/pml_region"].ravel())
        if "/recording/gll_node_ids" in p:
            ids = p["/recording/gll_node_ids"]
            xyz = p["/recording/gll_node_coords"].reshape(-1, 3)
            to = np.empty(ids.size, dtype=np.int32)
            for i, g in enumerate(ids.tolist()):
                if g not in index:
                    index[g] = len(out[R + "gll_node_ids"])
                    out[R + "gll_node_ids"].append(g)
                    out[R + "gll_node_coords"].append(xyz[i])
                to[i] = index[g]
            out[R + "rec_cell_local"].append(p["/recording/rec_cell_local"] + cum)
            out[R + "rec_cell_global_ids"].append(p["/recording/rec_cell_global_ids"])
            out[R + "cell_gll_node_index"].append(to[p["/recording/cell_gll_node_index"].ravel()])
        cum += n
    m = {"n_cell": cum}
    for k, v in out.items():
        if k == R + "gll_node_coords":
            m[k] = np.array(v, dtype=np.float64).reshape(-1, 3)
        elif k == R + "gll_node_ids":
            m[k] = np.array(v, dtype=np.int64)
        else:
            m[k] = np.concatenate(v) if v else np.zeros(0)
    m["n_rank_node"] = int(m["local_cell2rank_node"].max()) + 1
    return m


def merged_problem(prob: dict, rank: np.ndarray) -> dict:
    """The problem dict in the merged cell order of a case written by
    ``write_case`` (the cells of partition 0, then 1, ...), the input the
    driver's solve sees; for checking its traces with the oracle."""
    nc, ng = int(prob["n_cell"]), int(prob["ngll"])
    order = np.concatenate([np.nonzero(rank == r)[0] for r in range(int(rank.max()) + 1)])
    pos = np.empty(nc, dtype=np.int64)
    pos[order] = np.arange(nc)
    out = dict(prob)
    for k in ("coords", "jacobian", "dxi_dx", "mass", "vp", "vs", "density", "lambda", "mu", "ibool", "is_pml",
              "pml_region", "pml_coef_alpha", "pml_coef_abar", "damping", "cell_ids"):
        if prob.get(k) is not None:
            out[k] = np.asarray(prob[k]).reshape((nc,) + np.shape(prob[k])[1:])[order]
    rec = prob.get("recording")
    if rec is not None:
        rc = np.asarray(rec["rec_cell_local"])
        # merged recording order: partition by partition, each in cell order
        new = np.sort(pos[rc])
        out["recording"] = dict(rec, rec_cell_local=new.astype(np.int32))
    return out
