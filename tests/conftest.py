"""Shared test setup: import paths, the `gpu` marker, oracle build."""

import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "gf-only-sem_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and lib/libgfb.so")


def _ensure_oracle():
    lib = os.path.join(REPO, "oracle", "lib", "liboracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "oracle"], check=True,
                       stdout=subprocess.DEVNULL)


_ensure_oracle()


def golden_cases():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load_golden(name):
    import numpy as np

    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def golden_problem(g):
    """Reference-layout problem dict from a golden fixture."""
    import numpy as np

    n_cell = int(g["nx"]) * int(g["ny"]) * int(g["nz"])
    prob = {
        "n_cell": n_cell, "ngll": int(g["ibool"].shape[1]), "n_node": int(g["n_node"]),
        "ibool": g["ibool"], "cell_ids": np.arange(n_cell, dtype=np.int64),
        "dxi_dx": g["dxi_dx"], "jacobian": g["jacobian"], "lambda": g["lam"], "mu": g["mu"],
        "density": g["density"], "mass": g["mass"], "damping": g["damping"], "dt": float(g["dt"]),
        "snapshot_stride": int(g["stride"]), "src_cell_ids": g["src_cell_ids"],
        "src_weights": g["src_weights"], "stf": g["stf"],
        "recording": {"rec_cell_local": g["rec_cell_local"]},
    }
    if "pml_region" in g:
        prob.update(pml_region=g["pml_region"], pml_coef_alpha=g["pml_coef_alpha"],
                    pml_coef_abar=g["pml_coef_abar"])
    return prob


def rel_l2(a, b):
    import numpy as np

    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
