"""Host-side checks of the multi-model batch (no GPU): how independent
models are laid out as one batch mesh, and the layout errors gfb_create_batch
reports before touching a device."""

import numpy as np
import pytest

import gfb
from gfb import mesh


def small_model(nx, ny, nz, seed, src):
    spec = mesh.MeshSpec(nx=nx, ny=ny, nz=nz, dx=500.0, dy=500.0, dz=500.0, order=2, jitter=0.05, seed=seed,
                         pml={"xmin": 1, "xmax": 1, "zmax": 1})
    mat = mesh.seeded_layers(seed, nz * 500.0)
    return mesh.build_problem(spec, mat, np.asarray(src, dtype=float), nsteps=20, snapshot_stride=5,
                              record_depth_max_m=500.0)


@pytest.fixture(scope="module")
def two_models():
    return [small_model(3, 3, 2, 1, [700.0, 800.0, 300.0]), small_model(4, 2, 3, 2, [1100.0, 400.0, 600.0])]


def test_merged_layout_offsets_nodes_cells_sources_and_records(two_models):
    a, b = two_models
    merged, models, lay = gfb.merge_problems(two_models, n_steps=[20, 11])
    nn = a["ngll"] ** 3
    assert merged["n_cell"] == a["n_cell"] + b["n_cell"] and merged["n_node"] == a["n_node"] + b["n_node"]
    ib = merged["ibool"].reshape(-1, nn)
    np.testing.assert_array_equal(ib[: a["n_cell"]], a["ibool"].reshape(-1, nn))
    np.testing.assert_array_equal(ib[a["n_cell"]:], b["ibool"].reshape(-1, nn) + a["n_node"])
    # model k's cells use only model k's nodes
    for k, m in enumerate(models):
        blk = ib[m["cell_begin"]:m["cell_end"]]
        assert blk.min() >= m["node_begin"] and blk.max() < m["node_end"]
    assert [m["n_steps"] for m in models] == [20, 11]
    assert models[0]["dt"] == a["dt"] and models[1]["dt"] == b["dt"]
    # sources: model b's cells follow model a's
    na = np.asarray(a["src_cell_ids"]).size
    np.testing.assert_array_equal(merged["src_cell_ids"][:na], a["src_cell_ids"])
    np.testing.assert_array_equal(merged["src_cell_ids"][na:], np.asarray(b["src_cell_ids"]) + a["n_cell"])
    # recording cells
    ra = np.asarray(a["recording"]["rec_cell_local"])
    rb = np.asarray(b["recording"]["rec_cell_local"])
    np.testing.assert_array_equal(merged["recording"]["rec_cell_local"], np.concatenate([ra, rb + a["n_cell"]]))
    assert list(lay["rec_off"]) == [0, ra.size, ra.size + rb.size]
    # per-point arrays concatenated in cell order
    np.testing.assert_array_equal(merged["jacobian"], np.concatenate([a["jacobian"].ravel(), b["jacobian"].ravel()]))


def test_models_must_share_order_and_stride(two_models):
    a, b = two_models
    c = dict(b)
    c["snapshot_stride"] = 7
    with pytest.raises(ValueError):
        gfb.merge_problems([a, c])


def _raw_batch(merged, models):
    """Call gfb_create_batch directly and return (status, message)."""
    import ctypes as C

    lib = gfb.load_library()
    keep = {}

    def ptr(name, dtype, ctype):
        x = merged.get(name)
        if x is None:
            return C.cast(None, C.POINTER(ctype))
        x = np.ascontiguousarray(x, dtype=dtype).ravel()
        keep[name] = x
        return x.ctypes.data_as(C.POINTER(ctype))

    m = gfb.Mesh()
    m.n_cell, m.ngll, m.n_node = merged["n_cell"], merged["ngll"], merged["n_node"]
    m.ibool = ptr("ibool", np.int32, C.c_int32)
    m.dxi_dx = ptr("dxi_dx", np.float64, C.c_double)
    m.jacobian = ptr("jacobian", np.float64, C.c_double)
    m.lambda_ = ptr("lambda", np.float64, C.c_double)
    m.mu = ptr("mu", np.float64, C.c_double)
    m.mass = ptr("mass", np.float64, C.c_double)
    c = gfb.Config()
    c.dt, c.n_field, c.precision = 1.0, 1, gfb.FP32
    md = (gfb.Model * len(models))()
    for k, d in enumerate(models):
        md[k].cell_begin, md[k].cell_end = d["cell_begin"], d["cell_end"]
        md[k].node_begin, md[k].node_end = d["node_begin"], d["node_end"]
        md[k].dt, md[k].n_steps = d["dt"], d["n_steps"]
    h = C.c_void_p()
    st = lib.gfb_create_batch(C.byref(m), C.byref(c), None, len(models), md, C.byref(h))
    return st, lib.gfb_last_error().decode()


def test_batch_layout_errors_are_reported(two_models):
    merged, models, _ = gfb.merge_problems(two_models)
    # ranges that do not follow each other
    bad = [dict(m) for m in models]
    bad[1]["cell_begin"] += 1
    st, msg = _raw_batch(merged, bad)
    assert st == 1 and "follow" in msg
    # a cell of model 1 using a node of model 0
    nn = merged["ngll"] ** 3
    m2 = dict(merged)
    ib = merged["ibool"].copy()
    ib[models[1]["cell_begin"] * nn] = 0
    m2["ibool"] = ib
    st, msg = _raw_batch(m2, models)
    assert st == 1 and "another model" in msg
    # coverage
    short = [dict(m) for m in models]
    short[1]["node_end"] -= 1
    st, msg = _raw_batch(merged, short)
    assert st == 1 and "cover" in msg
