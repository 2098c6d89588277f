"""The allocation-free element-residual entry point.

gfb_element_residual_noalloc serves callers that cannot call cudaMalloc
(their device memory is owned by a pool or a host framework, or they cannot
afford cudaMalloc's implicit synchronisation inside their loop).  They pass
device buffers for inputs and output; the kernel's scratch lives in a fixed
array inside the library.  This test passes device buffers through the C
ABI, as such a caller would, and checks two calls in a row against the
allocating entry point gfb_element_residual, within the element-kernel
tolerance used by the other tests (max relative difference <= 1e-12).  It
also checks that a call larger than the fixed scratch is rejected with a
message.  The file is named to be collected last.
"""

import ctypes as C

import numpy as np
import pytest

import gfb

pytestmark = pytest.mark.gpu


def random_elements(ngll, n_elem, seed):
    rng = np.random.default_rng(seed)
    P = n_elem * ngll**3
    dxi = rng.uniform(-1, 1, (P, 9))
    dxi[:, 0] += 3.0
    dxi[:, 4] += 3.0
    dxi[:, 8] += 3.0
    jac = np.abs(rng.uniform(-1, 1, P)) + 0.01
    vp = np.abs(rng.uniform(-1, 1, P)) + 1000.0
    vs = np.abs(rng.uniform(-1, 1, P)) + 500.0
    rho = np.abs(rng.uniform(-1, 1, P)) + 1000.0
    mu = rho * vs * vs
    lam = rho * (vp * vp - 2.0 * vs * vs)
    u = rng.uniform(-1, 1, (P, 3))
    return dxi, jac, lam, mu, u


def bind():
    lib = gfb.load_library()
    f = lib.gfb_element_residual_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                  C.c_void_p]
    return lib, f


def test_no_alloc_matches_allocating_entry_on_two_calls_in_a_row():
    import torch

    lib, f = bind()
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    # two calls in a row with different sizes; the second is smaller so a
    # stale scratch from the first call would show up
    for ngll, n_elem, seed in ((5, 300, 11), (5, 37, 12)):
        dxi, jac, lam, mu, u = random_elements(ngll, n_elem, seed)
        ref = gfb.element_residual(dxi, jac, lam, mu, u, ngll, gfb.FP64)
        dev = {k: torch.tensor(v.ravel(), dtype=torch.float64, device="cuda")
               for k, v in (("dxi", dxi), ("jac", jac), ("lam", lam), ("mu", mu), ("u", u))}
        r = torch.full((u.size,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        st = f(n_elem, dev["dxi"].data_ptr(), dev["jac"].data_ptr(), dev["lam"].data_ptr(), dev["mu"].data_ptr(),
               ngll, dev["u"].data_ptr(), r.data_ptr(), C.c_void_p(stream.cuda_stream))
        assert st == 0, lib.gfb_last_error()
        stream.synchronize()
        got = r.cpu().numpy()
        assert np.all(np.isfinite(got))
        rel = np.abs(got - ref).max() / np.abs(ref).max()
        assert rel <= 1e-12, rel


def test_no_alloc_rejects_calls_beyond_the_scratch():
    import torch

    lib, f = bind()
    torch.cuda.set_device(0)
    x = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = x.data_ptr()
    st = f(672, p, p, p, p, 5, p, p, None)  # 671 cells fit at ngll=5
    assert st == 1
    msg = lib.gfb_last_error().decode()
    assert "maximum of 671 cells" in msg
