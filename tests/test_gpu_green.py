"""Strain Green's functions at the recording nodes: the snapshot's values
merged per node on the device (postprocess/cpp/main.cpp:300-425 mass-weighted
strain, averaged displacement) against the same merge of the per-cell
records in numpy, and against the merge of the FP64 oracle's records."""

import numpy as np
import pytest

import gfb
import oracle
from gfb import mesh

pytestmark = pytest.mark.gpu


def problem():
    spec = mesh.MeshSpec(nx=6, ny=5, nz=4, dx=500.0, dy=500.0, dz=500.0, order=4, jitter=0.06, seed=8,
                         pml={"xmin": 1, "xmax": 1, "ymin": 1, "ymax": 1, "zmax": 1})
    return mesh.build_problem(spec, mesh.seeded_layers(8, 2000.0), np.array([1400.0, 1200.0, 800.0]), nsteps=60,
                              snapshot_stride=20, record_depth_max_m=500.0)


def merge(prob, strain, u):
    """numpy restatement of the post-processing merge: [node][6], [node][3]."""
    nn = prob["ngll"] ** 3
    rec = np.asarray(prob["recording"]["rec_cell_local"])
    ib = np.asarray(prob["ibool"]).reshape(-1, nn)[rec].ravel()
    w = np.asarray(prob["mass"]).reshape(-1, nn)[rec].ravel()
    ids = np.unique(ib)
    pos = np.searchsorted(ids, ib)
    ws = np.zeros(ids.size)
    np.add.at(ws, pos, w)
    cnt = np.zeros(ids.size)
    np.add.at(cnt, pos, 1.0)
    es = np.zeros((ids.size, 6))
    np.add.at(es, pos, strain.reshape(-1, 6) * w[:, None])
    us = np.zeros((ids.size, 3))
    np.add.at(us, pos, u.reshape(-1, 3))
    return ids, es / ws[:, None], us / cnt[:, None]


@pytest.mark.parametrize("prec", [gfb.FP64, gfb.FP32])
def test_green_functions_merge_matches_numpy_and_oracle(prec):
    prob = problem()
    dirs = [0, 1, 2]
    s = gfb.Solver(prob, dirs=dirs, precision=prec, record_slots=8)
    ids = s.rec_nodes()
    np.testing.assert_array_equal(ids, np.asarray(prob["recording"]["gll_node_ids"]))
    s.advance(prob["nsteps"])
    greens, records = [], []
    while s.pending() > 0:
        g = s.read_green(release=False)
        r = [s.read_record(f) for f in range(3)]
        assert all(x["step"] == g["step"] for x in r)
        greens.append(g)
        records.append(r)
    assert [g["step"] for g in greens] == [0, 20, 40]
    tol_self = 1e-12 if prec == gfb.FP64 else 1e-6
    for g, r in zip(greens, records):
        for f in range(3):
            nid, e, u = merge(prob, r[f]["strain"], r[f]["u"])
            np.testing.assert_array_equal(nid, ids)
            scale = max(np.abs(e).max(), 1e-300)
            assert np.abs(g["strain"][:, f] - e).max() <= tol_self * scale
            assert np.abs(g["u"][:, f] - u).max() <= tol_self * max(np.abs(u).max(), 1e-300)
    # against the oracle's records merged the same way (FP64 path: 1e-10)
    if prec == gfb.FP64:
        for d in dirs:
            run = oracle.Run(prob, d, "oracle", threads=4)
            snaps = run.advance(prob["nsteps"])
            for k, g in enumerate(greens):
                _, e, _ = merge(prob, np.asarray(snaps["strain"][k]), np.asarray(snaps["u"][k]))
                num = np.linalg.norm(g["strain"][:, d] - e)
                den = np.linalg.norm(e)
                assert num <= 1e-10 * max(den, 1e-300) or den == 0.0
            run.close()
