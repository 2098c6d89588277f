"""C-ABI library checks that need no GPU: it loads, exports every function
include/gfb.h declares, and reports errors through status codes instead of
aborting (the reference aborts in GF_CUDA_CHECK, cuda_check.h:16-24)."""

import ctypes as C
import os
import re

import numpy as np
import pytest

import gfb


def declared_functions():
    text = open(gfb.HEADER_PATH).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gfb_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = gfb.load_library()
    names = declared_functions()
    assert "gfb_create" in names and "gfb_advance" in names
    for n in names:
        assert hasattr(lib, n), n
    assert lib.gfb_abi_version() == 1


@pytest.mark.gpu
def test_library_kernels_run_as_sm100():
    """The runtime's own report on a kernel of the loaded library: built for
    compute capability 10.0 (sm_100a)."""
    lib = gfb.load_library()
    b, p = C.c_int32(), C.c_int32()
    st = lib.gfb_kernel_arch(0, C.byref(b), C.byref(p))
    assert st == 0, lib.gfb_last_error()
    assert b.value == 100, b.value


def cuda_visible():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(cuda_visible(), reason="checks the no-GPU error path")
def test_create_without_gpu_returns_status_not_abort():
    from gfb import mesh

    spec = mesh.MeshSpec(nx=2, ny=2, nz=2, dx=100.0, dy=100.0, dz=100.0, order=4)
    p = mesh.build_problem(spec, mesh.homogeneous(), np.array([100.0, 100.0, 100.0]), nsteps=2,
                           with_cpml=False)
    with pytest.raises(gfb.GfbError) as ei:
        gfb.Solver(p)
    assert ei.value.status == 6  # GFB_ERR_NO_DEVICE
    assert "GPU" in str(ei.value)


def test_invalid_arguments_are_rejected_before_device_use():
    lib = gfb.load_library()
    m = gfb.Mesh()
    m.n_cell = 1
    m.ngll = 9  # unsupported order
    c = gfb.Config()
    c.dt = 1.0
    c.n_field = 1
    h = C.c_void_p()
    st = lib.gfb_create(C.byref(m), C.byref(c), None, C.byref(h))
    assert st == 5 and b"ngll" in lib.gfb_last_error()
    m.ngll = 5
    m.n_node = 10
    st = lib.gfb_create(C.byref(m), C.byref(c), None, C.byref(h))
    assert st == 1  # missing arrays
    assert lib.gfb_run_forward(b"w", 0, 0) == 1
