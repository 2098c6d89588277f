"""The allocation-free element-residual entry point.

gfb_element_residual_noalloc serves callers that cannot call cudaMalloc
(their device memory is owned by a pool or a host framework, or they cannot
afford cudaMalloc's implicit synchronisation inside their loop).  They pass
device buffers for inputs and output; the kernel's scratch lives in a fixed
array inside the library.  These tests pass device buffers through the C
ABI, as such a caller would, and check the results against the allocating
entry point gfb_element_residual and against the CPU oracle
(compute_element_residual, element_cpu.cpp:19-162), within the
element-kernel tolerance used by the other tests (max relative difference
<= 1e-12): two calls in a row, and one call at the largest cell count the
scratch holds for every supported ngll, whose next size up must be rejected
with a message.  The file is named to be collected last.
"""

import ctypes as C

import numpy as np
import pytest

import gfb
import oracle

pytestmark = pytest.mark.gpu

TOL = 1e-12
# largest call the fixed 8 MiB scratch holds, per ngll (include/gfb.h)
MAX_CELLS = {3: 3106, 4: 1310, 5: 671, 6: 388}


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


def call_no_alloc(f, lib, stream, ngll, n_elem, arrays):
    """One call on device copies of the inputs; returns r on the host."""
    import torch

    dxi, jac, lam, mu, u = arrays
    dev = [torch.tensor(np.ascontiguousarray(a).ravel(), dtype=torch.float64, device="cuda")
           for a in (dxi, jac, lam, mu, u)]
    r = torch.full((u.size,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = f(n_elem, dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(), dev[3].data_ptr(), ngll,
           dev[4].data_ptr(), r.data_ptr(), C.c_void_p(stream.cuda_stream))
    assert st == 0, lib.gfb_last_error()
    stream.synchronize()
    return r.cpu().numpy()


def check_against_references(got, arrays, ngll):
    dxi, jac, lam, mu, u = arrays
    assert np.all(np.isfinite(got))
    for ref in (gfb.element_residual(dxi, jac, lam, mu, u, ngll, gfb.FP64),
                oracle.element_residual(dxi, jac, lam, mu, u, ngll)):
        rel = np.abs(got - ref).max() / np.abs(ref).max()
        assert rel <= TOL, rel


def test_no_alloc_matches_allocating_entry_and_oracle_on_two_calls_in_a_row():
    import torch

    lib, f = bind()
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    # two calls in a row with different sizes; the second is smaller, so a
    # stale scratch from the first call would show up
    for ngll, n_elem, seed in ((5, 300, 11), (5, 37, 12)):
        arrays = random_elements(ngll, n_elem, seed)
        check_against_references(call_no_alloc(f, lib, stream, ngll, n_elem, arrays), arrays, ngll)


@pytest.mark.parametrize("ngll", [3, 4, 5, 6])
def test_no_alloc_at_the_largest_call_of_each_ngll(ngll):
    """Every ngll has its own kernel shape (cells per block 8 / 2 / 2 / 1)
    and its own limit; the largest call must run and the next be refused."""
    import torch

    lib, f = bind()
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    n = MAX_CELLS[ngll]
    arrays = random_elements(ngll, n, 100 + ngll)
    check_against_references(call_no_alloc(f, lib, stream, ngll, n, arrays), arrays, ngll)
    x = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = x.data_ptr()
    st = f(n + 1, p, p, p, p, ngll, p, p, None)
    assert st == 1
    assert f"maximum of {n} cells" in lib.gfb_last_error().decode()
