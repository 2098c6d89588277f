"""Mesh inputs computed on the GPU (gfb_prep_* in include/gfb.h).

Device counterparts of the host generator's ``gll_geometry``,
``global_numbering`` and ``cpml_parameters`` in ``gfb.mesh`` (which follow
preprocess/gll_geometry.py:132-186, preprocess/partition.py:192-254 and
preprocess/pml_cpml.py:42-515): same arguments, same outputs, one GPU thread
per GLL point and CUB radix sorts for the numbering.  Requires the CUDA
library and a GPU; there is no host fallback here (the host versions live in
``gfb.mesh``).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _check, load_library

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_bp = C.POINTER(C.c_uint8)


def _lib():
    lib = load_library()
    if not getattr(lib, "_prep_bound", False):
        lib.gfb_prep_geometry.argtypes = [C.c_int32, C.c_int64, C.c_int32, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.gfb_prep_numbering.argtypes = [C.c_int32, C.c_int64, _dp, _ip, _ip]
        lib.gfb_prep_cpml.argtypes = [C.c_int32, C.c_int64, C.c_int32, _dp, _bp, _dp, _dp, _dp, C.c_double,
                                      C.c_double, C.c_double, _ip, _dp, _dp]
        for name in ("gfb_prep_geometry", "gfb_prep_numbering", "gfb_prep_cpml"):
            getattr(lib, name).restype = C.c_int
        lib._prep_bound = True
    return lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def gll_geometry(corners: np.ndarray, order: int, device: int = 0):
    """coords, jacobian, dxi_dx, geometric mass as ``gfb.mesh.gll_geometry``."""
    from .mesh import gll_points, gll_weights

    pts = np.ascontiguousarray(gll_points(order), dtype=np.float64)
    w = np.ascontiguousarray(gll_weights(pts), dtype=np.float64)
    ng = order + 1
    cv = np.ascontiguousarray(corners, dtype=np.float64)
    n_cell = cv.shape[0]
    coords = np.empty((n_cell, ng, ng, ng, 3))
    jac = np.empty((n_cell, ng, ng, ng))
    dxi = np.empty((n_cell, ng, ng, ng, 9))
    mass = np.empty((n_cell, ng, ng, ng))
    _check(_lib().gfb_prep_geometry(int(device), n_cell, ng, _p(pts, C.c_double), _p(w, C.c_double),
                                     _p(cv, C.c_double), _p(coords, C.c_double), _p(jac, C.c_double),
                                     _p(dxi, C.c_double), _p(mass, C.c_double)))
    return coords, jac, dxi, mass


def global_numbering(coords: np.ndarray, device: int = 0):
    """(ibool, n_node) as ``gfb.mesh.global_numbering``."""
    n_cell, ng = coords.shape[0], coords.shape[1]
    xyz = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
    ibool = np.empty(xyz.shape[0], dtype=np.int32)
    n = C.c_int32()
    _check(_lib().gfb_prep_numbering(int(device), xyz.shape[0], _p(xyz, C.c_double), _p(ibool, C.c_int32),
                                      C.byref(n)))
    return ibool.reshape(n_cell, ng, ng, ng), int(n.value)


def cpml_parameters(coords, is_pml, bounds, widths, vp, f0, dt, device: int = 0):
    """(regions, coef_alpha [n_cell, nn, 9], abar [n_cell, nn, 5]) as
    ``gfb.mesh.cpml_parameters``."""
    from .mesh import R_COEF

    n_cell, ng = coords.shape[0], coords.shape[1]
    nn = ng**3
    xyz = np.ascontiguousarray(coords, dtype=np.float64)
    flags = np.ascontiguousarray(is_pml, dtype=np.uint8)
    v = np.ascontiguousarray(vp, dtype=np.float64)
    faces = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")
    b = np.array([bounds[f] for f in faces], dtype=np.float64)
    wd = np.array([max(0.0, float(widths.get(f, 0.0))) for f in faces], dtype=np.float64)
    region = np.empty(n_cell, dtype=np.int32)
    calpha = np.empty((n_cell, nn, 9))
    abar = np.empty((n_cell, nn, 5))
    _check(_lib().gfb_prep_cpml(int(device), n_cell, ng, _p(xyz, C.c_double), _p(flags, C.c_uint8),
                                 _p(v, C.c_double), _p(b, C.c_double), _p(wd, C.c_double), float(f0), float(dt),
                                 float(np.log(R_COEF)), _p(region, C.c_int32), _p(calpha, C.c_double),
                                 _p(abar, C.c_double)))
    return region, calpha, abar
