"""The process entry gf_solver_elastic_cuda on a B200, run as the reference
is run: in a working directory holding config + partitions/partition_{r}
(here three partitions of the raw .gfr container), writing
wavefields/{dir}/record_0_{step}, wavefields/{dir}/restart_0 and
log/forward_{dir}_0.log.

The records are checked against the CPU oracle run on the merged problem
(FP64, relative L2 <= 1e-10), their datasets and attributes against
RecordWriter::write_step (record.cpp:175-257), and --resume against an
uninterrupted run."""

import glob
import os
import subprocess

import numpy as np
import pytest
from conftest import rel_l2

import oracle
from gfb import files, mesh

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(REPO, "gf-only-sem_b200", "bin", "gf_solver_elastic_cuda")


def problem(cpml=True, nsteps=120):
    spec = mesh.MeshSpec(nx=6, ny=5, nz=4, dx=500.0, dy=500.0, dz=500.0, order=4, jitter=0.08, seed=5,
                         pml={"xmin": 1, "xmax": 1, "ymin": 1, "ymax": 1, "zmax": 1})
    mat = mesh.layered([600.0, 1300.0], [3500.0, 5000.0, 6500.0], [2000.0, 2900.0, 3700.0],
                       [2300.0, 2550.0, 2800.0])
    return mesh.build_problem(spec, mat, np.array([1430.0, 1270.0, 620.0]), nsteps=nsteps, snapshot_stride=10,
                              record_depth_max_m=500.0, with_cpml=cpml)


def run(cwd, *args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([BIN, *args], cwd=cwd, capture_output=True, text=True, timeout=600, env=e)


def records(cwd, d):
    out = {}
    for p in glob.glob(os.path.join(cwd, "wavefields", d, "record_0_*.gfr")):
        step = int(os.path.basename(p)[len("record_0_"):-4])
        out[step] = files.read(p)
    return dict(sorted(out.items()))


def test_bad_direction_prints_usage_and_exits_1(tmp_path):
    out = run(tmp_path, "--direction", "w")
    assert out.returncode == 1
    assert "--direction must be x, y, or z, got 'w'" in out.stderr and "Usage:" in out.stderr
    assert not (tmp_path / "log").exists()


@pytest.mark.parametrize("direction", ["y"])
def test_three_partitions_fp64_records_match_the_oracle(tmp_path, direction):
    prob = problem()
    rank = files.write_case(str(tmp_path), prob, n_part=3, log_stride=25, restart_stride=50)
    out = run(tmp_path, "--direction", direction)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    assert f"gf_solver: direction={direction}" in out.stdout
    log = (tmp_path / "log" / f"forward_{direction}_0.log").read_text()
    assert "simulation complete, 120 steps" in log and "[PROG] 100/120" in log
    recs = records(str(tmp_path), direction)
    assert list(recs) == list(range(0, 120, 10))
    m = files.merged_problem(prob, rank)
    d = "xyz".index(direction)
    ref = oracle.Run(m, d, "oracle", threads=4).advance(120)
    np.testing.assert_array_equal(ref["steps"], list(recs))
    merged = files.merge_partitions([files.read(str(tmp_path / "partitions" / f"partition_{r}.gfr"))
                                     for r in range(3)])
    nrec = m["recording"]["rec_cell_local"].size
    for i, (step, r) in enumerate(recs.items()):
        assert r["/@source_direction"] == direction and int(r["/@rank"]) == 0 and int(r["/@ngll"]) == 5
        assert r["/@basis"] == "gll" and int(r["/@n_rec_cell"]) == nrec and int(r["/@excludes_pml"]) == 1
        assert int(r["/@n_unique_gll"]) == merged["recording/gll_node_ids"].size
        np.testing.assert_array_equal(r["gll_node_ids"], merged["recording/gll_node_ids"])
        np.testing.assert_array_equal(r["cell_gll_node_index"].ravel(), merged["recording/cell_gll_node_index"])
        np.testing.assert_array_equal(r["recording_cell_model_index"], merged["recording/rec_cell_global_ids"])
        assert r["strain"].shape == (1, nrec, 125, 6) and r["strain"].dtype == np.float64
        for k, q in (("strain", "strain"), ("displacement", "u"), ("velocity", "v"), ("acceleration", "a")):
            assert rel_l2(r[k][0], ref[q][i]) <= 1e-10, (step, k)
    rs = files.read(str(tmp_path / "wavefields" / direction / "restart_0.gfr"))
    assert int(rs["/@step"]) == 100 and rs["displacement"].size == prob["n_node"] * 3


def test_float32_records_and_resume(tmp_path):
    """snapshot_precision "float32" writes float datasets (record.cpp:91-98);
    --resume continues from the restart file: without C-PML (whose memory
    the restart does not hold, restart.cpp:120-139) the resumed records
    equal the uninterrupted run's."""
    prob = problem(cpml=False, nsteps=100)
    files.write_case(str(tmp_path), prob, n_part=2, snapshot_precision="float32", restart_stride=40)
    out = run(tmp_path, "--direction", "x")
    assert out.returncode == 0, out.stderr[-2000:]
    first = records(str(tmp_path), "x")
    assert first[0]["displacement"].dtype == np.float32
    out = run(tmp_path, "--direction", "x", "--resume")
    assert out.returncode == 0, out.stderr[-2000:]
    assert "resumed at step 81" in out.stdout
    again = records(str(tmp_path), "x")
    for step in (90,):
        for k in ("displacement", "velocity", "strain"):
            assert rel_l2(again[step][k], first[step][k]) <= 1e-6, (step, k)


def test_fp32_path_from_the_environment(tmp_path):
    prob = problem(nsteps=60)
    rank = files.write_case(str(tmp_path), prob, n_part=1)
    out = run(tmp_path, "--direction", "z", env={"GFB_PRECISION": "fp32"})
    assert out.returncode == 0, out.stderr[-2000:]
    recs = records(str(tmp_path), "z")
    m = files.merged_problem(prob, rank)
    ref = oracle.Run(m, 2, "oracle", threads=4).advance(60)
    got = np.stack([r["displacement"][0] for r in recs.values()])
    assert rel_l2(got, ref["u"]) <= 1e-4
