"""File-level driver pieces that need no GPU: the raw dataset container
(read by the library, written by gfb.files and back), the partition merge
of gfb_run_forward against the numpy restatement of read_partition_all
(io.cpp:319-450), and the process entry's and driver's failure paths (exit
code 1, the log file log/forward_{dir}_0.log, logger.hpp:23-30)."""

import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

import gfb
from gfb import files, mesh

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(REPO, "gf-only-sem_b200", "bin", "gf_solver_elastic_cuda")


def small_problem(cpml=True, nsteps=40):
    spec = mesh.MeshSpec(nx=6, ny=5, nz=4, dx=500.0, dy=500.0, dz=500.0, order=4, jitter=0.08, seed=5,
                         pml={"xmin": 1, "xmax": 1, "ymin": 1, "ymax": 1, "zmax": 1})
    mat = mesh.layered([600.0, 1300.0], [3500.0, 5000.0, 6500.0], [2000.0, 2900.0, 3700.0],
                       [2300.0, 2550.0, 2800.0])
    return mesh.build_problem(spec, mat, np.array([1430.0, 1270.0, 620.0]), nsteps=nsteps, snapshot_stride=10,
                              record_depth_max_m=500.0, with_cpml=cpml)


def merge_with_library(part_dir, out):
    lib = gfb.load_library()
    lib.gfb_merge_partitions.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p]
    st = lib.gfb_merge_partitions(part_dir.encode(), b"gfr", out.encode())
    assert st == 0, lib.gfb_last_error()
    return files.read(out)


def test_container_round_trip_of_every_type(tmp_path):
    entries = {"/a@f": 1.5, "/a@i": 7, "/a@s": "float32", "/a@b": True, "/a/x": np.arange(12.0).reshape(3, 4),
               "/a/y": np.arange(5, dtype=np.int64), "/a/z": np.arange(6, dtype=np.int32).reshape(2, 3),
               "/a/w": np.linspace(0, 1, 7, dtype=np.float32), "/empty": np.zeros(0)}
    p = str(tmp_path / "t.gfr")
    files.write(p, entries)
    got = files.read(p)
    assert got["/a@s"] == "float32"
    assert float(got["/a@f"]) == 1.5 and int(got["/a@i"]) == 7 and int(got["/a@b"]) == 1
    for k in ("/a/x", "/a/y", "/a/z", "/a/w", "/empty"):
        np.testing.assert_array_equal(got[k], entries[k])
        assert got[k].dtype == np.asarray(entries[k]).dtype


@pytest.mark.parametrize("n_part", [1, 3])
def test_partition_merge_matches_the_numpy_restatement(tmp_path, n_part):
    prob = small_problem()
    rank = files.write_case(str(tmp_path), prob, n_part=n_part)
    parts = [files.read(str(tmp_path / "partitions" / f"partition_{r}.gfr")) for r in range(n_part)]
    ref = files.merge_partitions(parts)
    got = merge_with_library(str(tmp_path / "partitions"), str(tmp_path / "merged.gfr"))
    assert int(got["/@n_partitions"]) == n_part and int(got["/@n_cell"]) == prob["n_cell"]
    assert int(got["/@n_rank_node"]) == ref["n_rank_node"] == prob["n_node"]
    for k in ("local_cell_ids", "local_cell2rank_node", "jacobian", "dxi_dx", "mass", "lambda", "mu",
              "pml_coef_alpha", "pml_coef_abar", "pml_region", "recording/gll_node_ids",
              "recording/gll_node_coords", "recording/rec_cell_local", "recording/rec_cell_global_ids",
              "recording/cell_gll_node_index"):
        np.testing.assert_array_equal(got[k].ravel(), np.asarray(ref[k]).ravel(), err_msg=k)
    # the merged set is the problem in partition order, recording cells
    # offset by the cells of the partitions before theirs (io.cpp:425-427)
    m = files.merged_problem(prob, rank)
    np.testing.assert_array_equal(got["local_cell2rank_node"].ravel(), np.asarray(m["ibool"]).ravel())
    np.testing.assert_array_equal(got["recording/rec_cell_local"], m["recording"]["rec_cell_local"])
    ids = got["recording/gll_node_ids"]
    idx = got["recording/cell_gll_node_index"].reshape(-1, 125)
    ib = np.asarray(m["ibool"]).reshape(prob["n_cell"], 125)
    np.testing.assert_array_equal(ids[idx], ib[got["recording/rec_cell_local"]])
    if n_part > 1:
        assert not np.array_equal(got["local_cell_ids"], np.arange(prob["n_cell"]))


def test_merge_reports_missing_partitions_and_bad_files(tmp_path):
    lib = gfb.load_library()
    lib.gfb_merge_partitions.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p]
    st = lib.gfb_merge_partitions(str(tmp_path).encode(), b"gfr", str(tmp_path / "m.gfr").encode())
    assert st == 7 and b"no partition files" in lib.gfb_last_error()
    (tmp_path / "partition_0.gfr").write_bytes(b"not a container")
    st = lib.gfb_merge_partitions(str(tmp_path).encode(), b"gfr", str(tmp_path / "m.gfr").encode())
    assert st == 7 and b"GFBRAW01" in lib.gfb_last_error()


def cuda_visible():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(cuda_visible(), reason="checks the no-GPU exit path")
def test_process_entry_without_gpu_exits_1(tmp_path):
    out = subprocess.run([BIN, "--direction", "x"], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert out.returncode == 1
    assert "no CUDA-capable GPU found" in out.stderr


def test_driver_without_config_fails_with_a_log_file(tmp_path):
    code = ("import sys, ctypes; sys.path[:0] = [%r, %r]; import gfb; lib = gfb.load_library(); "
            "sys.exit(lib.gfb_run_forward(b'z', 0, 0))" % (REPO, os.path.join(REPO, "gf-only-sem_b200")))
    out = subprocess.run([sys.executable, "-c", code], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert out.returncode == 1
    log = (tmp_path / "log" / "forward_z_0.log").read_text()
    assert "[ INFO] single process, direction=z" in log
    assert "[ERROR] Error: cannot open config.gfr" in log
    assert "[Rank 0] Error: cannot open config.gfr" in out.stderr
