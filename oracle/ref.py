"""ctypes access to oracle/_ref/libhyteg_ref.so: the reference's own generated P1 kernels and
FEniCS P1 diffusion form, compiled from the reference sources by oracle/Makefile.

TEST INFRASTRUCTURE ONLY (pins the oracle; CPU baseline of bench.py).
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "_ref", "libhyteg_ref.so")
_lib = None


def available():
    return os.path.exists(PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(PATH)
        dp = C.POINTER(C.c_double)
        L.ref_cell_apply.argtypes = [dp, dp, C.c_int, dp]
        L.ref_cell_apply_many.argtypes = [C.c_int, C.POINTER(dp), C.POINTER(dp), C.c_int, dp, C.c_int]
        L.ref_restrict.argtypes = [dp, dp, C.c_int, dp]
        L.ref_prolongate.argtypes = [dp, dp, C.c_int, dp]
        L.ref_p1_diffusion_element.argtypes = [dp, dp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def cell_apply(src_cell, level, stencil15):
    dst = np.zeros_like(src_cell)
    lib().ref_cell_apply(_p(dst), _p(np.ascontiguousarray(src_cell)), level, _p(np.ascontiguousarray(stencil15, dtype=np.float64)))
    return dst


def restrict(fine_cell, coarse_level, nc14):
    n = 1 << coarse_level
    coarse = np.zeros(((n + 3) * (n + 2) * (n + 1)) // 6)
    lib().ref_restrict(_p(coarse), _p(np.ascontiguousarray(fine_cell)), coarse_level, _p(np.asarray(nc14, dtype=np.float64)))
    return coarse


def prolongate(coarse_cell, coarse_level, nc14, fine_init=None):
    n = 2 << coarse_level
    fine = np.zeros(((n + 3) * (n + 2) * (n + 1)) // 6) if fine_init is None else np.array(fine_init, dtype=np.float64)
    lib().ref_prolongate(_p(np.ascontiguousarray(coarse_cell)), _p(fine), coarse_level, _p(np.asarray(nc14, dtype=np.float64)))
    return fine


def p1_diffusion_element(X):
    """X: (4, 3) vertex coordinates -> 4x4 element matrix from the FEniCS form."""
    A = np.zeros(16)
    lib().ref_p1_diffusion_element(_p(np.ascontiguousarray(X, dtype=np.float64).ravel()), _p(A))
    return A.reshape(4, 4)


def p1_divkgrad_blending_element(X, map_kind=0, map_a=0.0, k_amp=0.5, k_phase=(0.0, 0.0, 0.0)):
    """Element matrix from the reference's p1_div_k_grad_blending_q3 form with a test blending map
    (0 identity, 1 F(x) = x (1 + a x0 x1)) and k = exp(amp sin cos sin)."""
    L = lib()
    f = L.ref_p1_divkgrad_blending_element
    dp = C.POINTER(C.c_double)
    f.argtypes = [dp, C.c_int, C.c_double, C.c_double, dp, dp]
    A = np.zeros(16)
    ph = np.asarray(k_phase, dtype=np.float64)
    f(_p(np.ascontiguousarray(X, dtype=np.float64).ravel()), map_kind, map_a, k_amp, _p(ph), _p(A))
    return A.reshape(4, 4)


def p2_divkgrad_blending_element(X, map_kind=0, map_a=0.0, k_amp=0.5, k_phase=(0.0, 0.0, 0.0)):
    """10x10 element matrix from the reference's p2_div_k_grad_blending_q4 form (same test maps and
    coefficient as p1_divkgrad_blending_element); DoFs: vertices, then edges (2,3),(1,3),(1,2),(0,3),(0,2),(0,1)."""
    L = lib()
    f = L.ref_p2_divkgrad_blending_element
    dp = C.POINTER(C.c_double)
    f.argtypes = [dp, C.c_int, C.c_double, C.c_double, dp, dp]
    A = np.zeros(100)
    ph = np.asarray(k_phase, dtype=np.float64)
    f(_p(np.ascontiguousarray(X, dtype=np.float64).ravel()), map_kind, map_a, k_amp, _p(ph), _p(A))
    return A.reshape(10, 10)


SHELL_PATH = os.path.join(HERE, "_ref", "libhyteg_ref_shell.so")
_shell = None


def shell_available():
    return os.path.exists(SHELL_PATH)


def shell_map_eval(coords, tets, cell, pts):
    """The reference's IcosahedralShellMap of macro-cell `cell` (classified by the reference's own
    code from the whole mesh): F (n, 3), DF (n, 3, 3) and the determinant evalDF returns, at the
    points pts (n, 3)."""
    global _shell
    if _shell is None:
        _shell = C.CDLL(SHELL_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        _shell.ref_shell_map_eval.argtypes = [C.c_int, dp, C.c_int, ip, C.c_int, C.c_int, dp, dp, dp, dp]
        _shell.ref_shell_map_eval.restype = C.c_int
    xyz = np.ascontiguousarray(coords, dtype=np.float64)
    tt = np.ascontiguousarray(tets, dtype=np.int32)
    x = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    F = np.zeros_like(x)
    DF = np.zeros((x.shape[0], 3, 3))
    det = np.zeros(x.shape[0])
    rc = _shell.ref_shell_map_eval(len(xyz), _p(xyz), len(tt), tt.ctypes.data_as(C.POINTER(C.c_int)), int(cell), x.shape[0], _p(x),
                                   _p(F), _p(DF), _p(det))
    if rc:
        raise ValueError("cell out of range")
    return F, DF, det
