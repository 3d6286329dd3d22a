"""hyteg_b200: B200-native matrix-free multigrid for HyTeG-style hybrid tetrahedral grids.

Python mirror of the reference's C++ interface for this path (class and method names follow
HyTeG: ``P1Function``, ``P1ConstantLaplaceOperator.apply(src, dst, level, flag, updateType)``,
``smooth_jac``, ``P1toP1LinearRestriction``, ``P1toP1LinearProlongation``,
``GeometricMultigridSolver``, ``CGSolver``, ``ChebyshevSmoother``).  Every call goes through the
C ABI declared in ``include/hyteg_b200.h`` and runs CUDA kernels built for sm_100a; there is no
CPU fallback: without the compiled library or a GPU the calls raise.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libhyteg_b200.so")

# DoFType (types/types.hpp:29-43) and UpdateType
Inner = 1
DirichletBoundary = 2
NeumannBoundary = 4
FreeslipBoundary = 8
All = 15
Replace = 0
Add = 1

F64, F32, F16 = 0, 1, 2
_DTYPES = {"float64": F64, "double": F64, "f64": F64, "float32": F32, "float": F32, "f32": F32,
           "float16": F16, "half": F16, "f16": F16}

P1_CONST_LAPLACE = 1
P1_CONST_MASS = 2
P2_CONST_LAPLACE = 8
SMOOTHER_JACOBI = 0
SMOOTHER_CHEBYSHEV = 1
SMOOTHER_GAUSS_SEIDEL = 2
SMOOTHER_SOR = 3
VCYCLE = 0
WCYCLE = 1

_lib = None


class HybError(RuntimeError):
    pass


class _GmgParams(C.Structure):
    _fields_ = [
        ("min_level", C.c_int), ("max_level", C.c_int),
        ("pre_smooth", C.c_int), ("post_smooth", C.c_int), ("smooth_increment", C.c_int),
        ("cycle", C.c_int), ("smoother", C.c_int), ("jacobi_relax", C.c_double),
        ("cheb_order", C.c_int), ("cheb_upper_factor", C.c_double), ("cheb_lower_factor", C.c_double),
        ("cheb_power_iterations", C.c_int), ("coarse_max_iter", C.c_int),
        ("coarse_rtol", C.c_double), ("coarse_atol", C.c_double), ("use_graph", C.c_int),
        ("coarse_fp64", C.c_int),
    ]


_SIGS = {
    "hyb_version": (C.c_char_p, []),
    "hyb_last_error": (C.c_char_p, []),
    "hyb_ctx_create": (C.c_int, [C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "hyb_ctx_destroy": (C.c_int, [C.c_void_p]),
    "hyb_ctx_synchronize": (C.c_int, [C.c_void_p]),
    "hyb_ctx_launch_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "hyb_ctx_scratch_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "hyb_ctx_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "hyb_mesh_create": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "hyb_mesh_create_cuboid": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                         C.POINTER(C.c_void_p)]),
    "hyb_mesh_create_gmsh": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    "hyb_mesh_create_spherical_shell": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double,
                                                  C.POINTER(C.c_void_p)]),
    "hyb_mesh_destroy": (C.c_int, [C.c_void_p]),
    "hyb_mesh_set_boundary_flags_on_boundary": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "hyb_mesh_set_bc_type": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32]),
    "hyb_mesh_counts": (C.c_int, [C.c_void_p, C.c_void_p]),
    "hyb_mesh_primitive_vertices": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "hyb_mesh_vertex_coords": (C.c_int, [C.c_void_p, C.c_void_p]),
    "hyb_mesh_primitive_flag": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "hyb_layout_packed_size": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int64)]),
    "hyb_layout_primitive_offsets": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "hyb_layout_cell_index": (C.c_int64, [C.c_int, C.c_int, C.c_int, C.c_int]),
    "hyb_layout_face_index": (C.c_int64, [C.c_int, C.c_int, C.c_int]),
    "hyb_fn_create": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "hyb_fn_destroy": (C.c_int, [C.c_void_p]),
    "hyb_fn_upload": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "hyb_fn_download": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "hyb_fn_interpolate_const": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_uint32]),
    "hyb_fn_interpolate_callback": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_uint32]),
    "hyb_fn_assign": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_uint32]),
    "hyb_fn_add": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_uint32]),
    "hyb_fn_mult_elementwise": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_uint32]),
    "hyb_fn_invert_elementwise": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32]),
    "hyb_fn_dot": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_uint32, C.POINTER(C.c_double)]),
    "hyb_fn_copy_from": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "hyb_fn_swap": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "hyb_fn_device_ptr": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]),
    "hyb_op_create": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "hyb_op_destroy": (C.c_int, [C.c_void_p]),
    "hyb_op_create_divkgrad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                         C.POINTER(C.c_void_p)]),
    "hyb_op_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_uint32, C.c_int]),
    "hyb_op_smooth_jac": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_uint32]),
    "hyb_op_inverse_diagonal": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_uint32]),
    "hyb_op_stencil": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "hyb_restrict": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32]),
    "hyb_prolongate": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32, C.c_int]),
    "hyb_gmg_params_default": (C.c_int, [C.POINTER(_GmgParams)]),
    "hyb_gmg_create": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(_GmgParams), C.POINTER(C.c_void_p)]),
    "hyb_gmg_destroy": (C.c_int, [C.c_void_p]),
    "hyb_gmg_set_radii": (C.c_int, [C.c_void_p, C.c_void_p]),
    "hyb_gmg_get_radii": (C.c_int, [C.c_void_p, C.c_void_p]),
    "hyb_gmg_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "hyb_gmg_smooth": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "hyb_gmg_solve_cycles": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_void_p,
                                       C.POINTER(C.c_int)]),
    "hyb_estimate_radius": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "hyb_chebyshev_coefficients": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_void_p]),
    "hyb_cg_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double,
                               C.POINTER(C.c_int)]),
    "hyb_mixed_solve": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                  C.c_double, C.c_void_p, C.POINTER(C.c_int)]),
    "hyb_residual_norm": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_uint32,
                                    C.POINTER(C.c_double)]),
    "hyb_fn_fill_random": (C.c_int, [C.c_void_p, C.c_int, C.c_uint64]),
    "hyb_op_store_element_matrices": (C.c_int, [C.c_void_p]),
    "hyb_fn_create_p2": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "hyb_p2_layout_sizes": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "hyb_fn_upload_async": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "hyb_fn_download_async": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "hyb_op_create_p2p1_div": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "hyb_p2p1_div_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_uint32, C.c_int]),
    "hyb_p1p2_divt_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_uint32, C.c_int]),
    "hyb_op_create_p1_pspg": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "hyb_op_smooth_sor": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_uint32, C.c_int]),
    "hyb_op_create_p2_full_viscous": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                                C.POINTER(C.c_void_p)]),
    "hyb_p2_full_viscous_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_uint32, C.c_int]),
    "hyb_p2_full_viscous_inverse_diagonal": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "hyb_stokes_params_default": (C.c_int, [C.c_void_p]),
    "hyb_stokes_create": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "hyb_stokes_destroy": (C.c_int, [C.c_void_p]),
    "hyb_stokes_set_velocity_radii": (C.c_int, [C.c_void_p, C.c_void_p]),
    "hyb_stokes_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "hyb_stokes_uzawa_smooth": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "hyb_stokes_residual_norm": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                           C.POINTER(C.c_double)]),
    "hyb_stokes_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                   C.c_double, C.c_void_p, C.POINTER(C.c_int)]),
    "hyb_stokes_mixed_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_int, C.c_int, C.c_double, C.c_void_p, C.POINTER(C.c_int)]),
    "hyb_p2_fn_download_reference": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "hyb_p2_fn_upload_reference": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "hyb_op_create_p2_divkgrad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                            C.POINTER(C.c_void_p)]),
    "hyb_op_create_p2_divkgrad_nodal": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                                  C.POINTER(C.c_void_p)]),
    "hyb_op_create_p2_divkgrad_fn": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                               C.POINTER(C.c_void_p)]),
    "hyb_fn_dot_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_uint32, C.POINTER(C.c_double)]),
    "hyb_stokes_set_omega": (C.c_int, [C.c_void_p, C.c_double]),
    "hyb_stokes_estimate_relaxation": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "hyb_serve_params_default": (C.c_int, [C.c_void_p]),
    "hyb_serve_create": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "hyb_serve_destroy": (C.c_int, [C.c_void_p]),
    "hyb_serve_now": (C.c_double, [C.c_void_p]),
    "hyb_serve_submit": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]),
    "hyb_serve_step": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "hyb_serve_status": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                   C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int),
                                   C.POINTER(C.c_double)]),
    "hyb_serve_last_error": (C.c_char_p, []),
    "hyb_fn_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "hyb_vtk_create": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]),
    "hyb_vtk_destroy": (C.c_int, [C.c_void_p]),
    "hyb_vtk_set_blending": (C.c_int, [C.c_void_p, C.c_int]),
    "hyb_vtk_set_parameter": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p]),
    "hyb_vtk_add": (C.c_int, [C.c_void_p, C.c_void_p, C.c_char_p]),
    "hyb_vtk_remove": (C.c_int, [C.c_void_p, C.c_void_p]),
    "hyb_vtk_write": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "hyb_vtk_write_packed": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.POINTER(C.c_char_p), C.POINTER(C.c_int), C.POINTER(C.c_void_p)]),
    "hyb_checkpoint_store": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_char_p),
                                       C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "hyb_checkpoint_function_count": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.c_int)]),
    "hyb_checkpoint_function_info": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_char_p, C.c_int, C.c_char_p, C.c_int,
                                               C.c_char_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "hyb_checkpoint_restore": (C.c_int, [C.c_char_p, C.c_char_p, C.c_void_p, C.c_char_p, C.c_int, C.c_int]),
}


def lib():
    """Load the compiled C-ABI library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY_PATH):
            raise HybError(f"{LIBRARY_PATH} is missing: build it with `python -m hyteg_b200.build`")
        L = C.CDLL(LIBRARY_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise HybError(f"hyteg_b200 error {rc}: {lib().hyb_last_error().decode()}")


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class Context:
    """Device + stream.  ``stream``: an integer cudaStream_t handle (e.g. torch's) or None."""

    def __init__(self, device=0, stream=None):
        h = C.c_void_p()
        _check(lib().hyb_ctx_create(device, C.c_void_p(stream) if stream else None, C.byref(h)))
        self.h = h

    def synchronize(self):
        _check(lib().hyb_ctx_synchronize(self.h))

    @property
    def launches(self):
        v = C.c_int64()
        _check(lib().hyb_ctx_launch_count(self.h, C.byref(v)))
        return v.value

    @property
    def scratch_bytes(self):
        """Bytes of device scratch this context holds (partials, smoother scratch, staging)."""
        v = C.c_int64()
        _check(lib().hyb_ctx_scratch_bytes(self.h, C.byref(v)))
        return v.value

    @property
    def stream(self):
        v = C.c_void_p()
        _check(lib().hyb_ctx_stream(self.h, C.byref(v)))
        return v.value or 0

    def close(self):
        if getattr(self, "h", None):
            lib().hyb_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PrimitiveStorage:
    """Macro mesh with HyTeG's primitive ids, orientations and boundary flags."""

    def __init__(self, handle, ctx=None):
        self.h = handle
        self.ctx = ctx

    @classmethod
    def from_tets(cls, coords, tets, ctx=None):
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        tets = np.ascontiguousarray(tets, dtype=np.int32)
        h = C.c_void_p()
        _check(lib().hyb_mesh_create(ctx.h if ctx else None, coords.shape[0], _ptr(coords), tets.shape[0], _ptr(tets),
                                     C.byref(h)))
        return cls(h, ctx)

    @classmethod
    def cuboid(cls, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), nx=1, ny=1, nz=1, ctx=None):
        """MeshInfo::meshCuboid; nx=ny=nz=1 gives the six-tetrahedra unit cube."""
        lo = np.asarray(lo, dtype=np.float64)
        hi = np.asarray(hi, dtype=np.float64)
        h = C.c_void_p()
        _check(lib().hyb_mesh_create_cuboid(ctx.h if ctx else None, _ptr(lo), _ptr(hi), nx, ny, nz, C.byref(h)))
        return cls(h, ctx)

    @classmethod
    def spherical_shell(cls, ntan, nrad, rmin, rmax, ctx=None):
        """MeshInfo::meshSphericalShell (SHELLMESH_CLASSIC)."""
        h = C.c_void_p()
        _check(lib().hyb_mesh_create_spherical_shell(ctx.h if ctx else None, ntan, nrad, rmin, rmax, C.byref(h)))
        return cls(h, ctx)

    @classmethod
    def from_gmsh(cls, path, ctx=None):
        h = C.c_void_p()
        _check(lib().hyb_mesh_create_gmsh(ctx.h if ctx else None, str(path).encode(), C.byref(h)))
        return cls(h, ctx)

    def set_boundary_flags_on_boundary(self, on_boundary=1, inner=0):
        _check(lib().hyb_mesh_set_boundary_flags_on_boundary(self.h, on_boundary, inner))

    def set_bc_type(self, flag, dof_type):
        _check(lib().hyb_mesh_set_bc_type(self.h, flag, dof_type))

    def counts(self):
        a = np.zeros(4, dtype=np.int32)
        _check(lib().hyb_mesh_counts(self.h, _ptr(a)))
        return tuple(int(v) for v in a)

    def primitive_vertices(self, kind, idx):
        a = np.zeros(4, dtype=np.int32)
        _check(lib().hyb_mesh_primitive_vertices(self.h, kind, idx, _ptr(a)))
        return [int(v) for v in a if v >= 0]

    def vertex_coords(self):
        a = np.zeros((self.counts()[0], 3))
        _check(lib().hyb_mesh_vertex_coords(self.h, _ptr(a)))
        return a

    def primitive_flag(self, kind, idx):
        v = C.c_int()
        _check(lib().hyb_mesh_primitive_flag(self.h, kind, idx, C.byref(v)))
        return v.value

    def packed_size(self, level):
        v = C.c_int64()
        _check(lib().hyb_layout_packed_size(self.h, level, C.byref(v)))
        return v.value

    def primitive_offsets(self, level):
        n = sum(self.counts())
        off = np.zeros(n, dtype=np.int64)
        sz = np.zeros(n, dtype=np.int64)
        _check(lib().hyb_layout_primitive_offsets(self.h, level, _ptr(off), _ptr(sz)))
        return off, sz

    def close(self):
        if getattr(self, "h", None):
            lib().hyb_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_CALLBACK = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_void_p)


class P1Function:
    """P1Function<ValueType> on levels min_level..max_level (device storage, HyTeG layout)."""

    _lshift = 0
    _create = "hyb_fn_create"

    def __init__(self, name, storage, min_level, max_level, ctx, dtype="float64"):
        self.name = name
        self.storage = storage
        self.ctx = ctx
        self.min_level, self.max_level = min_level, max_level
        self.dtype = _DTYPES[dtype] if isinstance(dtype, str) else int(dtype)
        h = C.c_void_p()
        _check(getattr(lib(), self._create)(ctx.h, storage.h, self.dtype, min_level, max_level, C.byref(h)))
        self.h = h

    def packed_size(self, level):
        """Values of the packed level vector (upload/download)."""
        return self.storage.packed_size(level + self._lshift)

    # data movement -----------------------------------------------------------------------
    def upload(self, level, packed):
        a = np.ascontiguousarray(packed, dtype=np.float64)
        if a.size != self.packed_size(level):
            raise ValueError("packed vector has the wrong size for this level")
        _check(lib().hyb_fn_upload(self.h, level, _ptr(a)))

    def upload_async(self, level, packed):
        """Queue the upload on the context's stream; `packed` (pinned for full bandwidth) must stay
        valid until the context is synchronised."""
        if packed.dtype != np.float64 or packed.size != self.packed_size(level) or not packed.flags["C_CONTIGUOUS"]:
            raise ValueError("packed must be a contiguous float64 array of the packed size")
        _check(lib().hyb_fn_upload_async(self.h, level, _ptr(packed)))

    def download_async(self, level, out):
        """Queue the download into `out` (contiguous float64, packed size) on the context's stream."""
        if out.dtype != np.float64 or out.size != self.packed_size(level) or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a contiguous float64 array of the packed size")
        _check(lib().hyb_fn_download_async(self.h, level, _ptr(out)))

    def fill_random(self, level, seed):
        """Seeded uniform values in [-1, 1] on every DoF of `level` (generated on the device)."""
        _check(lib().hyb_fn_fill_random(self.h, level, seed))

    def download(self, level, out=None):
        """Packed level vector; `out` (a contiguous float64 array of packed_size, e.g. in pinned
        memory) is filled and returned instead of a new array."""
        n = self.packed_size(level)
        if out is None:
            out = np.zeros(n, dtype=np.float64)
        elif out.dtype != np.float64 or out.size != n or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a contiguous float64 array of the packed size")
        _check(lib().hyb_fn_download(self.h, level, _ptr(out)))
        return out

    # HyTeG function API ---------------------------------------------------------------------
    def interpolate(self, value, level, flag=All):
        if callable(value):
            def cb(xyz, _user):
                return float(value(xyz[0], xyz[1], xyz[2]))
            fn = _CALLBACK(cb)
            _check(lib().hyb_fn_interpolate_callback(self.h, fn, None, level, flag))
        else:
            _check(lib().hyb_fn_interpolate_const(self.h, float(value), level, flag))

    def setToZero(self, level):
        self.interpolate(0.0, level, All)

    def assign(self, scalars, functions, level, flag=All):
        s = np.ascontiguousarray(scalars, dtype=np.float64)
        arr = (C.c_void_p * len(functions))(*[f.h.value for f in functions])
        _check(lib().hyb_fn_assign(self.h, len(functions), _ptr(s), arr, level, flag))

    def add(self, scalars, functions, level, flag=All):
        s = np.ascontiguousarray(scalars, dtype=np.float64)
        arr = (C.c_void_p * len(functions))(*[f.h.value for f in functions])
        _check(lib().hyb_fn_add(self.h, len(functions), _ptr(s), arr, level, flag))

    def multElementwise(self, functions, level, flag=All):
        a, b = functions
        _check(lib().hyb_fn_mult_elementwise(self.h, a.h, b.h, level, flag))

    def invertElementwise(self, level, flag=All):
        _check(lib().hyb_fn_invert_elementwise(self.h, level, flag))

    def dotGlobal(self, other, level, flag=All):
        v = C.c_double()
        _check(lib().hyb_fn_dot(self.h, other.h, level, flag, C.byref(v)))
        return v.value

    def dotGlobalNoAlloc(self, other, level, flag=All):
        """dotGlobal without any device allocation (fixed static scratch; see hyb_fn_dot_noalloc)."""
        v = C.c_double()
        _check(lib().hyb_fn_dot_noalloc(self.h, other.h, level, flag, C.byref(v)))
        return v.value

    def copyFrom(self, other, level):
        _check(lib().hyb_fn_copy_from(self.h, other.h, level))

    def swap(self, other, level):
        _check(lib().hyb_fn_swap(self.h, other.h, level))

    def device_ptr(self, level):
        p, n = C.c_void_p(), C.c_int64()
        _check(lib().hyb_fn_device_ptr(self.h, level, C.byref(p), C.byref(n)))
        return p.value, n.value

    def close(self):
        if getattr(self, "h", None):
            lib().hyb_fn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _ConstantOperator:
    kind = None

    def __init__(self, storage, min_level, max_level, ctx):
        self.storage, self.ctx = storage, ctx
        self.min_level, self.max_level = min_level, max_level
        h = C.c_void_p()
        _check(lib().hyb_op_create(ctx.h, storage.h, self.kind, min_level, max_level, C.byref(h)))
        self.h = h

    def apply(self, src, dst, level, flag, updateType=Replace):
        _check(lib().hyb_op_apply(self.h, src.h, dst.h, level, flag, updateType))

    def smooth_jac(self, dst, rhs, src, relax, level, flag):
        _check(lib().hyb_op_smooth_jac(self.h, dst.h, rhs.h, src.h, float(relax), level, flag))

    def getInverseDiagonalValues(self, out, level, flag=All):
        _check(lib().hyb_op_inverse_diagonal(self.h, out.h, level, flag))
        return out

    def smooth_sor(self, dst, rhs, relax, level, flag, backwards=False):
        """P1Operator::smooth_sor (constant-stencil operators): in place in dst."""
        _check(lib().hyb_op_smooth_sor(self.h, dst.h, rhs.h, float(relax), level, flag, 1 if backwards else 0))

    def smooth_gs(self, dst, rhs, level, flag):
        self.smooth_sor(dst, rhs, 1.0, level, flag)

    def smooth_sor_backwards(self, dst, rhs, relax, level, flag):
        self.smooth_sor(dst, rhs, relax, level, flag, backwards=True)

    def smooth_gs_backwards(self, dst, rhs, level, flag):
        self.smooth_sor(dst, rhs, 1.0, level, flag, backwards=True)

    def stencil(self, level, cell, cls=0):
        a = np.zeros(15)
        _check(lib().hyb_op_stencil(self.h, level, cell, cls, _ptr(a)))
        return a

    def close(self):
        if getattr(self, "h", None):
            lib().hyb_op_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class P1ConstantLaplaceOperator(_ConstantOperator):
    kind = P1_CONST_LAPLACE


class P1ConstantMassOperator(_ConstantOperator):
    kind = P1_CONST_MASS


class _Coeff(C.Structure):
    _fields_ = [("kind", C.c_int), ("value", C.c_double), ("amp", C.c_double), ("freq", C.c_double),
                ("phase", C.c_double * 3)]


def _coeff(k):
    """hyb_coeff from None (k = 1), a constant, ("expsin", amp, (p0, p1, p2)[, freq]) or
    ("radial", amp, r0, scale) for exp(amp (r0 - |x|) / scale)."""
    c = _Coeff()
    c.kind, c.value, c.amp, c.freq = 0, 1.0, 0.5, 1.0
    if isinstance(k, (int, float)):
        c.value = float(k)
    elif k is not None and k[0] == "radial":
        c.kind, c.amp, c.value, c.freq = 2, float(k[1]), float(k[2]), float(k[3])
    elif k is not None:
        c.kind = 1
        c.amp = float(k[1])
        for d in range(3):
            c.phase[d] = float(k[2][d])
        if len(k) > 3:
            c.freq = float(k[3])
    return c


class P1ElementwiseBlendingDivKGradOperator(_ConstantOperator):
    """-div(k grad u), elementwise P1 with the form p1_div_k_grad_blending_q3.

    k: None (k = 1), a constant, or ("expsin", amp, (p0, p1, p2)[, freq]) for
    k = exp(amp sin(2 pi f (x+p0)) cos(2 pi f (y+p1)) sin(2 pi f (z+p2))).  blending: None or "shell".
    """

    def __init__(self, storage, min_level, max_level, ctx, k=None, blending=None):
        self.storage, self.ctx = storage, ctx
        self.min_level, self.max_level = min_level, max_level
        c = _coeff(k)
        h = C.c_void_p()
        _check(lib().hyb_op_create_divkgrad(ctx.h, storage.h, min_level, max_level, C.byref(c),
                                            1 if blending == "shell" else 0, C.byref(h)))
        self.h = h

    def computeAndStoreLocalElementMatrices(self):
        """Element matrices are computed once per level and read back by every later apply."""
        _check(lib().hyb_op_store_element_matrices(self.h))


class P2Function(P1Function):
    """P2Function<ValueType>: quadratic Lagrange DoFs of level l (micro-vertices and micro-edge
    midpoints), stored on the node set of level l+1; packed vectors use the level-(l+1) vertex layout."""

    _lshift = 1
    _create = "hyb_fn_create_p2"

    def reference_layout_sizes(self, level):
        """(vertex-DoF values, edge-DoF values) of the reference's P2Function memory of `level`."""
        v, e = C.c_int64(), C.c_int64()
        _check(lib().hyb_p2_layout_sizes(self.storage.h, level, C.byref(v), C.byref(e)))
        return v.value, e.value

    def download_reference(self, level):
        """The vertex-DoF part followed by the edge-DoF part, in the reference's memory layout."""
        a = np.zeros(sum(self.reference_layout_sizes(level)), dtype=np.float64)
        _check(lib().hyb_p2_fn_download_reference(self.h, level, _ptr(a)))
        return a

    def upload_reference(self, level, values):
        a = np.ascontiguousarray(values, dtype=np.float64)
        if a.size != sum(self.reference_layout_sizes(level)):
            raise ValueError("vector has the wrong size for the reference P2 layout of this level")
        _check(lib().hyb_p2_fn_upload_reference(self.h, level, _ptr(a)))


class P2ElementwiseBlendingDivKGradOperator(_ConstantOperator):
    """-div(k grad u), elementwise P2 with the form p2_div_k_grad_blending_q4 (same k and blending
    conventions as the P1 class)."""

    def __init__(self, storage, min_level, max_level, ctx, k=None, blending=None):
        self.storage, self.ctx = storage, ctx
        self.min_level, self.max_level = min_level, max_level
        c = _coeff(k)
        h = C.c_void_p()
        _check(lib().hyb_op_create_p2_divkgrad(ctx.h, storage.h, min_level, max_level, C.byref(c),
                                               1 if blending == "shell" else 0, C.byref(h)))
        self.h = h

    def computeAndStoreLocalElementMatrices(self):
        _check(lib().hyb_op_store_element_matrices(self.h))


class P2ElementwiseDivKGradOperator(_ConstantOperator):
    """operatorgeneration::P2ElementwiseDivKGrad / P2ElementwiseDivKGradIcosahedralShellMap (hyteg-operators):
    -div(k grad u) with k stored as a P2 function and evaluated at the quadrature points through the P2
    basis.  k is a P2Function (FP64, levels min_level..max_level, copied at creation) or a coefficient spec
    as for P2ElementwiseBlendingDivKGradOperator, interpolated at the (blended) nodes of every level."""

    def __init__(self, storage, min_level, max_level, ctx, k=None, blending=None):
        self.storage, self.ctx = storage, ctx
        self.min_level, self.max_level = min_level, max_level
        h = C.c_void_p()
        bl = 1 if blending == "shell" else 0
        if isinstance(k, P2Function):
            _check(lib().hyb_op_create_p2_divkgrad_fn(ctx.h, storage.h, min_level, max_level, k.h, bl, C.byref(h)))
        else:
            c = _coeff(k)
            _check(lib().hyb_op_create_p2_divkgrad_nodal(ctx.h, storage.h, min_level, max_level, C.byref(c), bl,
                                                         C.byref(h)))
        self.h = h

    def computeAndStoreLocalElementMatrices(self):
        _check(lib().hyb_op_store_element_matrices(self.h))


class P2ConstantLaplaceOperator(_ConstantOperator):
    """P2ConstantLaplaceOperator (P2ConstantOperator.cpp:100-114): one constant stencil per parity class of
    the P2 node grid and macro-cell, applied as a memory-bound stencil sweep.  Levels are P2 levels."""

    kind = P2_CONST_LAPLACE


class P1toP1LinearRestriction:
    def restrict(self, function, sourceLevel, flag):
        _check(lib().hyb_restrict(function.h, sourceLevel, flag))


class P1toP1LinearProlongation:
    def prolongate(self, function, sourceLevel, flag):
        _check(lib().hyb_prolongate(function.h, sourceLevel, flag, Replace))

    def prolongateAndAdd(self, function, sourceLevel, flag):
        _check(lib().hyb_prolongate(function.h, sourceLevel, flag, Add))


class P2ToP1ElementwiseBlendingDivOperator:
    """The coupling blocks of P2P1ElementwiseBlendingStokesOperator: div (P2ToP1ElementwiseBlending
    Div{x,y,z}) maps three P2 velocity components of level l to a P1 pressure of level l; divT
    (P1ToP2ElementwiseBlendingDivT{x,y,z}) is the transpose."""

    def __init__(self, storage, min_level, max_level, ctx, blending=None):
        self.storage, self.ctx = storage, ctx
        h = C.c_void_p()
        _check(lib().hyb_op_create_p2p1_div(ctx.h, storage.h, min_level, max_level, 1 if blending == "shell" else 0,
                                            C.byref(h)))
        self.h = h

    def apply(self, u, p, level, flag=All, updateType=Replace):
        arr = (C.c_void_p * 3)(*[f.h.value for f in u])
        _check(lib().hyb_p2p1_div_apply(self.h, arr, p.h, level, flag, updateType))

    def applyTranspose(self, p, u, level, flag=Inner, updateType=Replace):
        arr = (C.c_void_p * 3)(*[f.h.value for f in u])
        _check(lib().hyb_p1p2_divt_apply(self.h, p.h, arr, level, flag, updateType))

    def close(self):
        if getattr(self, "h", None):
            lib().hyb_op_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class P2ElementwiseBlendingFullViscousOperator:
    """The full viscous velocity block 2 mu eps(u) : eps(v) - (2/3) mu div u div v on three P2
    components (P2ElementwiseBlendingFullViscousOperator, a VectorToVectorOperator of the nine forms
    p2_full_stokesvar_{i}_{j}_blending_q3); mu as the k argument of the other elementwise operators."""

    def __init__(self, storage, min_level, max_level, ctx, viscosity=None, blending=None):
        self.storage, self.ctx = storage, ctx
        self.min_level, self.max_level = min_level, max_level
        c = _coeff(viscosity)
        h = C.c_void_p()
        _check(lib().hyb_op_create_p2_full_viscous(ctx.h, storage.h, min_level, max_level, C.byref(c),
                                                   1 if blending == "shell" else 0, C.byref(h)))
        self.h = h

    @staticmethod
    def _arr(u):
        return (C.c_void_p * 3)(*[f.h.value for f in u])

    def apply(self, src, dst, level, flag=Inner, updateType=Replace):
        _check(lib().hyb_p2_full_viscous_apply(self.h, self._arr(src), self._arr(dst), level, flag, updateType))

    def getInverseDiagonalValues(self, out, level):
        _check(lib().hyb_p2_full_viscous_inverse_diagonal(self.h, self._arr(out), level))

    def close(self):
        if getattr(self, "h", None):
            lib().hyb_op_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class P1PSPGOperator(_ConstantOperator):
    """P1PSPGOperator on the affine macro geometry; getInverseDiagonalValues gives the values of
    P1PSPGInvDiagOperator (the Uzawa pressure scaling)."""

    def __init__(self, storage, min_level, max_level, ctx):
        self.storage, self.ctx = storage, ctx
        self.min_level, self.max_level = min_level, max_level
        h = C.c_void_p()
        _check(lib().hyb_op_create_p1_pspg(ctx.h, storage.h, min_level, max_level, C.byref(h)))
        self.h = h


class _StokesParams(C.Structure):
    _fields_ = [("min_level", C.c_int), ("max_level", C.c_int), ("pre_smooth", C.c_int), ("post_smooth", C.c_int),
                ("velocity_sweeps", C.c_int), ("cheb_order", C.c_int), ("power_iterations", C.c_int),
                ("omega", C.c_double), ("coarse_sweeps", C.c_int), ("velocity_block", C.c_int),
                ("pressure_scaling", C.c_int)]


class StokesUzawaMultigrid:
    """GeometricMultigridSolver< P2P1ElementwiseBlendingStokesOperator > with UzawaSmoother (block-Laplace
    variant): the velocity block -div(eta grad) per component (eta: see _coeff, e.g.
    ("radial", 2.99, 1.0, 0.45)), Chebyshev velocity smoothing, pressure update with the inverted PSPG
    diagonal, quadratic/linear transfers, coarse_sweeps Uzawa steps on the coarsest level.
    velocity_block="full_viscous" uses P2ElementwiseBlendingFullViscousOperator (2 eta eps(u) : eps(v) -
    (2/3) eta div u div v, the three components coupled) with Chebyshev on the coupled block."""

    def __init__(self, ctx, storage, min_level, max_level, viscosity=None, blending=None, pre=3, post=3,
                 velocity_sweeps=3, cheb_order=3, power_iterations=20, omega=0.7, coarse_sweeps=30,
                 velocity_block="laplace", pressure_scaling="pspg"):
        if velocity_block not in ("laplace", "full_viscous"):
            raise ValueError("velocity_block must be 'laplace' or 'full_viscous'")
        if pressure_scaling not in ("pspg", "lumped_mass"):
            raise ValueError("pressure_scaling must be 'pspg' or 'lumped_mass'")
        p = _StokesParams()
        _check(lib().hyb_stokes_params_default(C.byref(p)))
        p.min_level, p.max_level, p.pre_smooth, p.post_smooth = min_level, max_level, pre, post
        p.velocity_sweeps, p.cheb_order, p.power_iterations = velocity_sweeps, cheb_order, power_iterations
        p.omega, p.coarse_sweeps = float(omega), coarse_sweeps
        p.velocity_block = 1 if velocity_block == "full_viscous" else 0
        p.pressure_scaling = 1 if pressure_scaling == "lumped_mass" else 0
        self.params, self.ctx, self.storage = p, ctx, storage
        c = _coeff(viscosity)
        h = C.c_void_p()
        _check(lib().hyb_stokes_create(ctx.h, storage.h, C.byref(c), 1 if blending == "shell" else 0, C.byref(p), C.byref(h)))
        self.h = h

    @staticmethod
    def _arr(u):
        return (C.c_void_p * 3)(*[f.h.value for f in u])

    def set_velocity_radii(self, radii):
        r = np.ascontiguousarray(radii, dtype=np.float64)
        _check(lib().hyb_stokes_set_velocity_radii(self.h, _ptr(r)))

    def set_omega(self, omega):
        """UzawaSmoother::setRelaxationParameter"""
        _check(lib().hyb_stokes_set_omega(self.h, float(omega)))
        self.params.omega = float(omega)

    def estimate_relaxation(self, level, iterations=20, velocity_sweeps=2):
        """estimateUzawaRelaxationParameter: spectral radius of |S|^-1 B A~^-1 B^T by power iteration
        (use omega = 1 / the radius with this solver's pressure scaling)"""
        r = C.c_double()
        _check(lib().hyb_stokes_estimate_relaxation(self.h, level, iterations, velocity_sweeps, C.byref(r)))
        return r.value

    def apply(self, u, p, du, dp, level):
        _check(lib().hyb_stokes_apply(self.h, self._arr(u), p.h, self._arr(du), dp.h, level))

    def uzawa_smooth(self, u, p, bu, bp, level):
        _check(lib().hyb_stokes_uzawa_smooth(self.h, self._arr(u), p.h, self._arr(bu), bp.h, level))

    def residual_norm(self, u, p, bu, bp, level):
        r = C.c_double()
        _check(lib().hyb_stokes_residual_norm(self.h, self._arr(u), p.h, self._arr(bu), bp.h, level, C.byref(r)))
        return r.value

    def solve(self, u, p, bu, bp, level, max_cycles, rtol=0.0):
        hist = np.zeros(max_cycles + 1)
        done = C.c_int()
        _check(lib().hyb_stokes_solve(self.h, self._arr(u), p.h, self._arr(bu), bp.h, level, max_cycles, float(rtol),
                                      _ptr(hist), C.byref(done)))
        return hist[: done.value + 1]

    def mixed_solve(self, inner, u, p, bu, bp, level, max_outer=50, rtol=1e-8, inner_dtype="float32"):
        """Defect correction: FP64 residual of this solver, one V-cycle of `inner` (a second
        StokesUzawaMultigrid on the same mesh and levels) in inner_dtype per iteration."""
        dt = _DTYPES[inner_dtype] if isinstance(inner_dtype, str) else int(inner_dtype)
        hist = np.zeros(max_outer + 1)
        done = C.c_int()
        _check(lib().hyb_stokes_mixed_solve(self.h, inner.h, dt, self._arr(u), p.h, self._arr(bu), bp.h, level, max_outer,
                                            float(rtol), _ptr(hist), C.byref(done)))
        return hist[: done.value + 1]

    def close(self):
        if getattr(self, "h", None):
            lib().hyb_stokes_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


P2toP2QuadraticRestriction = P1toP1LinearRestriction  # hyb_restrict dispatches on the function's space
P2toP2QuadraticProlongation = P1toP1LinearProlongation


def chebyshev_coefficients(order, lower, upper):
    out = np.zeros(order)
    _check(lib().hyb_chebyshev_coefficients(order, lower, upper, _ptr(out)))
    return out


def estimate_radius(op, x, tmp, level, iterations):
    """chebyshev::estimateRadius: power iteration on D^-1 A (x is the start vector, overwritten)."""
    v = C.c_double()
    _check(lib().hyb_estimate_radius(op.h, x.h, tmp.h, level, iterations, C.byref(v)))
    return v.value


class CGSolver:
    def __init__(self, storage, minLevel, maxLevel, maxIter=10**6, relativeTolerance=1e-16, absoluteTolerance=1e-16):
        self.maxIter, self.rtol, self.atol = maxIter, relativeTolerance, absoluteTolerance
        self.iterations = 0

    def solve(self, A, x, b, level):
        it = C.c_int()
        _check(lib().hyb_cg_solve(A.h, x.h, b.h, level, self.maxIter, self.rtol, self.atol, C.byref(it)))
        self.iterations = it.value


def residual_norm(A, x, b, tmp, level, flag=Inner | NeumannBoundary | FreeslipBoundary):
    v = C.c_double()
    _check(lib().hyb_residual_norm(A.h, x.h, b.h, tmp.h, level, flag, C.byref(v)))
    return v.value


class GeometricMultigridSolver:
    """GeometricMultigridSolver with weighted-Jacobi or Chebyshev smoothing and a device CG coarse solver."""

    def __init__(self, ctx, A, minLevel, maxLevel, preSmoothSteps=3, postSmoothSteps=3, smoothIncrementOnCoarserGrids=0,
                 cycleType=VCYCLE, smoother="jacobi", relax=2.0 / 3.0, chebyshev_order=3, chebyshev_upper=1.2,
                 chebyshev_lower=0.3, power_iterations=50, coarse_max_iter=1000, coarse_rtol=1e-14, coarse_atol=1e-16,
                 use_graph=True):
        p = _GmgParams()
        _check(lib().hyb_gmg_params_default(C.byref(p)))
        p.min_level, p.max_level = minLevel, maxLevel
        p.pre_smooth, p.post_smooth, p.smooth_increment = preSmoothSteps, postSmoothSteps, smoothIncrementOnCoarserGrids
        p.cycle = cycleType
        kinds = {"jacobi": SMOOTHER_JACOBI, "chebyshev": SMOOTHER_CHEBYSHEV, "gauss_seidel": SMOOTHER_GAUSS_SEIDEL,
                 "sor": SMOOTHER_SOR}
        if smoother not in kinds:
            raise ValueError("smoother must be one of " + ", ".join(kinds))
        p.smoother = kinds[smoother]
        p.jacobi_relax = relax
        p.cheb_order, p.cheb_upper_factor, p.cheb_lower_factor = chebyshev_order, chebyshev_upper, chebyshev_lower
        p.cheb_power_iterations = power_iterations
        p.coarse_max_iter, p.coarse_rtol, p.coarse_atol = coarse_max_iter, coarse_rtol, coarse_atol
        p.use_graph = 1 if use_graph else 0
        self.params = p
        self.A, self.ctx = A, ctx
        h = C.c_void_p()
        _check(lib().hyb_gmg_create(ctx.h, A.h, C.byref(p), C.byref(h)))
        self.h = h

    def set_radii(self, radii):
        r = np.ascontiguousarray(radii, dtype=np.float64)
        _check(lib().hyb_gmg_set_radii(self.h, _ptr(r)))

    def radii(self):
        r = np.zeros(self.params.max_level - self.params.min_level + 1)
        _check(lib().hyb_gmg_get_radii(self.h, _ptr(r)))
        return r

    def solve(self, A, x, b, level):
        _check(lib().hyb_gmg_solve(self.h, x.h, b.h, level))

    def smooth(self, x, b, level, iterations=1):
        """The smoother alone on one level (ChebyshevSmoother::solve / WeightedJacobiSmoother::solve)."""
        _check(lib().hyb_gmg_smooth(self.h, x.h, b.h, level, iterations))

    def solve_cycles(self, x, b, level, max_cycles, rtol=0.0):
        hist = np.zeros(max_cycles + 1)
        done = C.c_int()
        _check(lib().hyb_gmg_solve_cycles(self.h, x.h, b.h, level, max_cycles, rtol, _ptr(hist), C.byref(done)))
        return hist[: done.value + 1]

    def mixed_solve(self, A, x, b, level, inner_dtype="float32", inner_cycles=1, max_outer=50, rtol=1e-8):
        """Mixed-precision defect correction: FP64 x, b; inner cycles of this solver in `inner_dtype`."""
        dt = _DTYPES[inner_dtype] if isinstance(inner_dtype, str) else int(inner_dtype)
        hist = np.zeros(max_outer + 1)
        done = C.c_int()
        _check(lib().hyb_mixed_solve(self.h, dt, A.h, x.h, b.h, level, inner_cycles, max_outer, rtol, _ptr(hist),
                                     C.byref(done)))
        return hist[: done.value + 1]

    def close(self):
        if getattr(self, "h", None):
            lib().hyb_gmg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------------------------------- serving
class _ServeParams(C.Structure):
    _fields_ = [("max_slots", C.c_int), ("hbm_budget_bytes", C.c_double), ("inner_dtype", C.c_int),
                ("pre_smooth", C.c_int), ("post_smooth", C.c_int), ("power_iterations", C.c_int),
                ("batch_width", C.c_int)]


class _Request(C.Structure):
    _fields_ = [("mesh", C.c_void_p), ("op_kind", C.c_int), ("coeff", _Coeff), ("blending", C.c_int),
                ("level", C.c_int), ("rhs", C.c_void_p), ("seed", C.c_uint64), ("rtol", C.c_double),
                ("max_cycles", C.c_int), ("mixed", C.c_int), ("arrival_time", C.c_double),
                ("x_out", C.c_void_p)]


QUEUED, RUNNING, CONVERGED, STOPPED = 0, 1, 2, 3


class SolveServer:
    """Continuous-batching solve server over resident multigrid hierarchies (no reference counterpart).

    ``submit`` queues a Poisson / div-k-grad solve; ``step`` runs one scheduler pass (retire finished
    solves, launch the next V-cycle of every running solve, admit queued requests into free slots);
    ``status`` reports (state, t_arrival, t_admit, t_done, cycles, relative residual).
    """

    def __init__(self, ctx, max_slots=32, hbm_budget_bytes=0.0, inner_dtype="float32", pre_smooth=3, post_smooth=3,
                 power_iterations=20, batch_width=1):
        p = _ServeParams()
        _check(lib().hyb_serve_params_default(C.byref(p)))
        p.max_slots, p.hbm_budget_bytes = max_slots, float(hbm_budget_bytes)
        p.batch_width = int(batch_width)
        p.inner_dtype = _DTYPES[inner_dtype] if isinstance(inner_dtype, str) else int(inner_dtype)
        p.pre_smooth, p.post_smooth, p.power_iterations = pre_smooth, post_smooth, power_iterations
        self.ctx = ctx
        self._keep = {}
        h = C.c_void_p()
        rc = lib().hyb_serve_create(ctx.h, C.byref(p), C.byref(h))
        if rc != 0:
            raise HybError(f"hyb_serve_create: {lib().hyb_serve_last_error().decode()}")
        self.h = h

    def now(self):
        return lib().hyb_serve_now(self.h)

    def submit(self, storage, level, kind="laplace", k=None, blending=None, rhs=None, seed=0, rtol=1e-8,
               max_cycles=50, mixed=False, arrival_time=-1.0, want_solution=False):
        kinds = {"laplace": P1_CONST_LAPLACE, "divkgrad": 3, "p2_divkgrad": 4, "p2_laplace": P2_CONST_LAPLACE}
        if kind not in kinds:
            raise ValueError("kind must be one of " + ", ".join(kinds))
        r = _Request()
        r.mesh = storage.h
        r.op_kind = kinds[kind]
        r.coeff.kind, r.coeff.value, r.coeff.amp, r.coeff.freq = 0, 1.0, 0.5, 1.0
        if isinstance(k, (int, float)):
            r.coeff.value = float(k)
        elif k is not None:
            r.coeff.kind, r.coeff.amp = 1, float(k[1])
            for d in range(3):
                r.coeff.phase[d] = float(k[2][d])
            if len(k) > 3:
                r.coeff.freq = float(k[3])
        r.blending = 1 if blending == "shell" else 0
        r.level, r.seed, r.rtol, r.max_cycles = level, seed, rtol, max_cycles
        r.mixed, r.arrival_time = 1 if mixed else 0, float(arrival_time)
        keep = []
        if rhs is not None:
            a = np.ascontiguousarray(rhs, dtype=np.float64)
            keep.append(a)
            r.rhs = a.ctypes.data
        out = None
        if want_solution:
            out = np.zeros(storage.packed_size(level + (1 if kind.startswith("p2") else 0)))
            keep.append(out)
            r.x_out = out.ctypes.data
        rid = C.c_int64()
        rc = lib().hyb_serve_submit(self.h, C.byref(r), C.byref(rid))
        if rc != 0:
            raise HybError(f"hyb_serve_submit failed with status {rc}")
        self._keep[rid.value] = (keep, out)
        return rid.value

    def step(self):
        run, q = C.c_int(), C.c_int()
        rc = lib().hyb_serve_step(self.h, C.byref(run), C.byref(q))
        if rc != 0:
            raise HybError(f"hyb_serve_step: {lib().hyb_serve_last_error().decode()}")
        return run.value, q.value

    def status(self, rid):
        st, ta, tb, tc, cy, rr = C.c_int(), C.c_double(), C.c_double(), C.c_double(), C.c_int(), C.c_double()
        _check(lib().hyb_serve_status(self.h, rid, C.byref(st), C.byref(ta), C.byref(tb), C.byref(tc), C.byref(cy),
                                      C.byref(rr)))
        return {"state": st.value, "t_arrival": ta.value, "t_admit": tb.value, "t_done": tc.value, "cycles": cy.value,
                "rel_res": rr.value}

    def solution(self, rid):
        return self._keep[rid][1]

    def drain(self, poll=None):
        """Run scheduler passes until no request is queued or running."""
        while True:
            run, q = self.step()
            if run == 0 and q == 0:
                return
            if poll:
                poll()

    def close(self):
        if getattr(self, "h", None):
            lib().hyb_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------------------------ data export
class VTKOutput:
    """VTKOutput( dir, filename, storage, writeFrequency ) (dataexport/VTKOutput/VTKOutput.hpp:44-139):
    ``add`` functions, ``write(level, timestep)`` writes <dir>/<filename>_VertexDoF_level<L>_ts<T>.vtu for
    the P1 functions and ..._P2_level<L>_ts<T>.vtu for the P2 functions when timestep % writeFrequency
    == 0; ``setParameter("vtkDataFormat", "ASCII" | "BINARY")``.  ``blending="shell"`` writes the points
    under the icosahedral shell map (the storage's geometry map in the reference)."""

    def __init__(self, dir, filename, storage, writeFrequency=1, blending=None):
        h = C.c_void_p()
        _check(lib().hyb_vtk_create(storage.h, dir.encode(), filename.encode(), int(writeFrequency), C.byref(h)))
        self.h = h
        self.storage = storage
        self._fns = []
        if blending is not None:
            _check(lib().hyb_vtk_set_blending(h, 1 if blending == "shell" else 0))

    def add(self, function, name=None):
        _check(lib().hyb_vtk_add(self.h, function.h, (name or function.name).encode()))
        self._fns.append(function)

    def remove(self, function):
        _check(lib().hyb_vtk_remove(self.h, function.h))
        self._fns = [f for f in self._fns if f is not function]

    def setParameter(self, key, value):
        _check(lib().hyb_vtk_set_parameter(self.h, key.encode(), value.encode()))

    def write(self, level, timestep=0):
        _check(lib().hyb_vtk_write(self.h, level, timestep))

    def close(self):
        if self.h:
            lib().hyb_vtk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_vtu_packed(storage, path, level, fields, order=1, blending=None, binary=False):
    """Write one VTK file from host data: ``fields`` maps names to packed level vectors (the
    ``download`` layout; P2 vectors of the level+1 node set when order=2), or to (vector, dtype)."""
    names, dts, ptrs, keep = [], [], [], []
    for name, v in fields.items():
        dt = F64
        if isinstance(v, tuple):
            v, dt = v[0], (_DTYPES[v[1]] if isinstance(v[1], str) else int(v[1]))
        a = np.ascontiguousarray(v, dtype=np.float64)
        keep.append(a)
        names.append(name.encode())
        dts.append(dt)
        ptrs.append(a.ctypes.data)
    n = len(names)
    _check(lib().hyb_vtk_write_packed(storage.h, path.encode(), level, order, 1 if blending == "shell" else 0, 1 if binary else 0, n,
                                      (C.c_char_p * max(n, 1))(*names), (C.c_int * max(n, 1))(*dts),
                                      (C.c_void_p * max(n, 1))(*ptrs)))


class CheckpointExporter:
    """registerFunction( function, minLevel, maxLevel ) / storeCheckpoint( filePath, fileName )
    (checkpointrestore/CheckpointExporter.hpp:26-60); the file is <filePath>/<fileName>.hybckpt."""

    def __init__(self):
        self._reg = []

    def registerFunction(self, function, minLevel=None, maxLevel=None):
        lo = function.min_level if minLevel is None else minLevel
        hi = function.max_level if maxLevel is None else maxLevel
        self._reg = [r for r in self._reg if r[0] is not function] + [(function, lo, hi)]

    def deregisterFunction(self, function):
        self._reg = [r for r in self._reg if r[0] is not function]

    def storeCheckpoint(self, filePath, fileName):
        n = len(self._reg)
        _check(lib().hyb_checkpoint_store(filePath.encode(), fileName.encode(), n,
                                          (C.c_void_p * max(n, 1))(*[r[0].h.value for r in self._reg]),
                                          (C.c_char_p * max(n, 1))(*[r[0].name.encode() for r in self._reg]),
                                          (C.c_int * max(n, 1))(*[r[1] for r in self._reg]),
                                          (C.c_int * max(n, 1))(*[r[2] for r in self._reg])))


class CheckpointImporter:
    """The importer side (ADIOS2/AdiosCheckpointImporter.hpp:97-170): ``getFunctionDetails()`` lists
    (name, kind, valueType, minLevel, maxLevel); ``restoreFunction(function, minLevel, maxLevel)``
    fills the function's levels from the checkpoint entry of the same name."""

    def __init__(self, filePath, fileName):
        self.dir, self.name = filePath.encode(), fileName.encode()

    def getFunctionDetails(self):
        n = C.c_int()
        _check(lib().hyb_checkpoint_function_count(self.dir, self.name, C.byref(n)))
        out = []
        for i in range(n.value):
            nb, kb, vb = C.create_string_buffer(1024), C.create_string_buffer(64), C.create_string_buffer(64)
            lo, hi = C.c_int(), C.c_int()
            _check(lib().hyb_checkpoint_function_info(self.dir, self.name, i, nb, 1024, kb, 64, vb, 64, C.byref(lo), C.byref(hi)))
            out.append({"name": nb.value.decode(), "kind": kb.value.decode(), "valueType": vb.value.decode(),
                        "minLevel": lo.value, "maxLevel": hi.value})
        return out

    def restoreFunction(self, function, minLevel=None, maxLevel=None):
        lo = function.min_level if minLevel is None else minLevel
        hi = function.max_level if maxLevel is None else maxLevel
        _check(lib().hyb_checkpoint_restore(self.dir, self.name, function.h, function.name.encode(), lo, hi))
