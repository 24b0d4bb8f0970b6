"""anitowave_adaptive_b200 — B200 (sm_100a) FLIP step on a multiresolution sparse block grid.

Python binding of the C ABI declared in include/anitowave.h (libanitowave.so, built in-tree by
anitowave_adaptive_b200/csrc/build.py).  The classes mirror the reference's managers:

    MSBG      ~ MSBGManager          (MSBG.cuh:502-677)
    Solver    ~ VCycleSolver + AdaptiveSmoother + MultigridTransfer (VCycle.cuh:140-305,
                Smoother.cuh:227-292, MultigridTransfer.cuh:104-150)
    p2g/g2p/advect ~ P2GTransfer::run / G2PManager (P2G.cuh:173-195, G2P.cuh:175-228)
    Flip      — the whole FLIP step (no counterpart in the reference)

Device buffers are passed as torch CUDA tensors (or raw device pointers).  There is no CPU
fallback: every compute call goes to the CUDA library, and importing a call without the
library raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libanitowave.so")

AW_OK = 0
STATUS = {0: "AW_OK", 1: "AW_ERR_INVALID_ARGUMENT", 2: "AW_ERR_CUDA", 3: "AW_ERR_OUT_OF_MEMORY",
          4: "AW_ERR_NOT_CONVERGED", 5: "AW_ERR_NAN", 6: "AW_ERR_STATE", 7: "AW_ERR_UNSUPPORTED",
          8: "AW_ERR_IO"}

# channels (MSBG.cuh:12-50)
VELOCITY_X, VELOCITY_Y, VELOCITY_Z, PRESSURE = 0, 1, 2, 3
PHASE_FIELD_X, PHASE_FIELD_Y, PHASE_FIELD_Z = 4, 5, 6
BETA_COEFF_X, BETA_COEFF_Y, BETA_COEFF_Z = 7, 8, 9
MASS_DENSITY_X, MASS_DENSITY_Y, MASS_DENSITY_Z = 10, 11, 12
MOMENTUM_X, MOMENTUM_Y, MOMENTUM_Z = 13, 14, 15
DIVERGENCE, CELL_TYPE = 16, 19
VELOCITY_OLD_X, VELOCITY_OLD_Y, VELOCITY_OLD_Z = 20, 21, 22

OPERATOR_FV, OPERATOR_REFERENCE = 0, 1
PRECISION_FP32, PRECISION_MIXED, PRECISION_FP32_PCG = 0, 1, 2


class AWError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class GridDesc(C.Structure):
    _fields_ = [("dims", C.c_int32 * 3), ("block_size", C.c_float), ("domain_min", C.c_float * 3),
                ("base_res", C.c_int32), ("num_levels", C.c_int32)]


class SolverDesc(C.Structure):
    _fields_ = [("operator_mode", C.c_int32), ("precision", C.c_int32), ("mg_levels", C.c_int32),
                ("pre_smooth", C.c_int32), ("post_smooth", C.c_int32), ("coarsest_iterations", C.c_int32),
                ("block_iterations", C.c_int32), ("dense_sweeps", C.c_int32), ("omega", C.c_float),
                ("target_reduction", C.c_float), ("theta", C.c_float), ("max_cycles", C.c_int32),
                ("tolerance", C.c_double)]


class FlipDesc(C.Structure):
    _fields_ = [("dt", C.c_float), ("alpha", C.c_float), ("gravity", C.c_float * 3), ("precision", C.c_int32),
                ("tolerance", C.c_double), ("max_cycles", C.c_int32)]


class FlipStats(C.Structure):
    _fields_ = [("cycles", C.c_int32), ("residual", C.c_double), ("div_before", C.c_double),
                ("div_after", C.c_double), ("ms_sort", C.c_float), ("ms_p2g", C.c_float), ("ms_solve", C.c_float),
                ("ms_g2p", C.c_float), ("ms_advect", C.c_float), ("ms_other", C.c_float)]


# name -> (restype, argtypes); every symbol declared in include/anitowave.h
_VP, _I32, _I64, _U32, _F, _D = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32, C.c_float, C.c_double
_PP = C.POINTER(C.c_void_p)
SIGNATURES = {
    "aw_last_error": (C.c_char_p, []),
    "aw_version": (C.c_char_p, []),
    "aw_launch_count": (C.c_uint64, []),
    "aw_morton3d": (_U32, [_U32, _U32, _U32]),
    "aw_block_layout": (None, [_I32, _I32, C.POINTER(_U32)]),
    "aw_msbg_create": (C.c_int, [C.POINTER(GridDesc), _PP]),
    "aw_msbg_destroy": (C.c_int, [_VP]),
    "aw_msbg_desc": (C.c_int, [_VP, C.POINTER(GridDesc)]),
    "aw_msbg_init_refinement_map": (C.c_int, [_VP, _U32, _VP]),
    "aw_msbg_refinement_map": (C.c_int, [_VP, _PP]),
    "aw_msbg_block_info": (C.c_int, [_VP, _VP, _VP]),
    "aw_msbg_levels_from_particles": (C.c_int, [_VP, _VP, _I64, C.POINTER(_I32), _VP]),
    "aw_msbg_enforce_grading": (C.c_int, [_VP, C.POINTER(_I32), _VP]),
    "aw_msbg_allocate": (C.c_int, [_VP, _VP]),
    "aw_msbg_totals": (C.c_int, [_VP, C.POINTER(_U32)]),
    "aw_msbg_offsets": (C.c_int, [_VP, _I32, _PP]),
    "aw_msbg_coarse_offsets": (C.c_int, [_VP, _I32, _I32, _VP, C.POINTER(_U32), _VP]),
    "aw_msbg_channel": (C.c_int, [_VP, _I32, _PP, C.POINTER(_U32)]),
    "aw_msbg_run_galerkin": (C.c_int, [_VP, _PP, _PP, _I32, _VP]),
    "aw_p2g": (C.c_int, [_VP, _VP, _VP, _I64, _VP]),
    "aw_p2g_phase": (C.c_int, [_VP, _VP, _VP, _VP, _I64, _F, _F, _VP]),
    "aw_backup_grid_velocity": (C.c_int, [_VP, _VP]),
    "aw_g2p": (C.c_int, [_VP, _VP, _VP, _I64, _F, _VP]),
    "aw_g2p_noalloc": (C.c_int, [_VP, _VP, _VP, _I64, _F, _VP]),
    "aw_test_arm_copy_timeout": (C.c_int, [_VP]),
    "aw_advect": (C.c_int, [_VP, _VP, _I64, _F, _VP]),
    "aw_sample_velocity": (C.c_int, [_VP, _VP, _I64, _I32, _VP, _VP]),
    "aw_resample_lattice": (C.c_int, [_VP, C.POINTER(_I32), C.POINTER(_F), C.POINTER(_F)]),
    "aw_resample_cells": (C.c_int, [_VP, _I32, C.POINTER(_I32), _VP, _VP]),
    "aw_resample_velocity": (C.c_int, [_VP, _I32, C.POINTER(_I32), _VP, _VP]),
    "aw_vtk_write_structured_points": (C.c_int, [C.c_char_p, C.POINTER(_I32), C.POINTER(_F), C.POINTER(_F),
                                                 C.c_char_p, _I32, _VP]),
    "aw_vtk_write_blocks": (C.c_int, [_VP, C.c_char_p]),
    "aw_vtk_write_particles": (C.c_int, [C.c_char_p, _VP, _I64, C.c_char_p, _VP]),
    "aw_sort_particles": (C.c_int, [_VP, _VP, _I64, _VP, _VP, _VP]),
    "aw_face_positions": (C.c_int, [_VP, _I32, _VP, _VP]),
    "aw_face_sync": (C.c_int, [_VP, _I32, _VP]),
    "aw_wall_bc": (C.c_int, [_VP, _I32, _VP]),
    "aw_add_gravity": (C.c_int, [_VP, C.POINTER(_F), _F, _VP]),
    "aw_velocity_divergence": (C.c_int, [_VP, _VP, _F, _VP, _VP, _VP]),
    "aw_velocity_divergence_max64": (C.c_int, [_VP, _VP, _VP, _VP]),
    "aw_pressure_gradient": (C.c_int, [_VP, _VP, _VP, _I32, _VP, _F, _VP]),
    "aw_solver_default_desc": (C.c_int, [_I32, C.POINTER(SolverDesc)]),
    "aw_solver_create": (C.c_int, [_VP, C.POINTER(SolverDesc), _PP]),
    "aw_solver_destroy": (C.c_int, [_VP]),
    "aw_solver_setup": (C.c_int, [_VP, _VP, _VP]),
    "aw_solver_update_coefficients": (C.c_int, [_VP, _VP]),
    "aw_solver_num_levels": (C.c_int, [_VP, C.POINTER(_I32)]),
    "aw_solver_level_array": (C.c_int, [_VP, _I32, _I32, _PP, C.POINTER(_U32)]),
    "aw_smoother_solve_level": (C.c_int, [_VP, _I32, _I32, _VP]),
    "aw_mg_residual": (C.c_int, [_VP, _I32, _VP]),
    "aw_mg_restrict": (C.c_int, [_VP, _I32, _VP]),
    "aw_mg_prolongate": (C.c_int, [_VP, _I32, _VP]),
    "aw_solver_coarsest_solve": (C.c_int, [_VP, _VP]),
    "aw_vcycle_run": (C.c_int, [_VP, _VP]),
    "aw_solve": (C.c_int, [_VP, _VP, _VP, C.POINTER(_I32), C.POINTER(_D), _VP]),
    "aw_flip_create": (C.c_int, [_VP, C.POINTER(FlipDesc), _VP, _VP, _I64, _PP]),
    "aw_flip_destroy": (C.c_int, [_VP]),
    "aw_flip_step": (C.c_int, [_VP, _VP]),
    "aw_flip_stats_get": (C.c_int, [_VP, C.POINTER(FlipStats)]),
    "aw_flip_particles": (C.c_int, [_VP, _VP, _VP]),
    "aw_flip_solver": (C.c_int, [_VP, _PP]),
    "aw_flip_rebuild_levels": (C.c_int, [_VP, C.POINTER(_I32), C.POINTER(_I32), _VP]),
    "aw_flip_set_phase": (C.c_int, [_VP, _VP, _F, _F]),
    "aw_solver_precision": (C.c_int, [_VP, C.POINTER(_I32)]),
    "aw_project": (C.c_int, [_VP, _VP, _VP, _F, _VP]),
    "aw_vjp_project": (C.c_int, [_VP, _VP, _VP, _F, _PP, _VP]),
    "aw_vjp_p2g": (C.c_int, [_VP, _VP, _VP, _I64, _PP, _VP, _VP, _VP]),
    "aw_vjp_g2p": (C.c_int, [_VP, _VP, _I64, _F, _VP, _VP, _PP, _PP, _VP]),
    "aw_vjp_advect": (C.c_int, [_VP, _VP, _I64, _F, _VP, _PP, _VP]),
    "aw_vjp_sample": (C.c_int, [_VP, _VP, _I64, _I32, _VP, _PP, _VP, _VP]),
    "aw_rollout_create": (C.c_int, [_VP, C.POINTER(FlipDesc), _VP, _I64, _I32, _I32, _PP]),
    "aw_rollout_destroy": (C.c_int, [_VP]),
    "aw_rollout_forward": (C.c_int, [_VP, _VP, _VP, _I32, C.POINTER(_D), _VP]),
    "aw_rollout_final_positions": (C.c_int, [_VP, _VP, _VP]),
    "aw_vjp_rollout": (C.c_int, [_VP, _VP, _VP]),
}

_lib = None


def lib():
    """Load libanitowave.so.  Raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with anitowave_adaptive_b200.csrc.build "
                              "(or __graft_entry__.build()); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != AW_OK:
        raise AWError(status, lib().aw_last_error().decode())


def _ptr(x):
    """Device pointer of a torch CUDA tensor (or an int pointer)."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return x.data_ptr()


def _stream(s=None):
    if s is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return s


def version():
    return lib().aw_version().decode()


def launch_count():
    return lib().aw_launch_count()


def morton3d(x, y, z):
    return lib().aw_morton3d(x, y, z)


def block_layout(base_res, level):
    out = (C.c_uint32 * 6)()
    lib().aw_block_layout(base_res, level, out)
    return list(out)


class MSBG:
    """MSBGManager (MSBG.cuh:502-677) over the C ABI."""

    def __init__(self, dims, block_size, domain_min=(0.0, 0.0, 0.0), base_res=16, num_levels=3):
        d = GridDesc()
        d.dims[:] = [int(v) for v in dims]
        d.block_size = float(block_size)
        d.domain_min[:] = [float(v) for v in domain_min]
        d.base_res = int(base_res)
        d.num_levels = int(num_levels)
        self.desc = d
        self.dims = tuple(int(v) for v in dims)
        self.nb = int(np.prod(self.dims))
        self.base_res, self.num_levels = int(base_res), int(num_levels)
        self.block_size = float(block_size)
        self.domain_min = tuple(float(v) for v in domain_min)
        h = C.c_void_p()
        check(lib().aw_msbg_create(C.byref(d), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().aw_msbg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # topology ------------------------------------------------------------------------------
    def init_refinement_map(self, value, stream=None):
        check(lib().aw_msbg_init_refinement_map(self.h, int(value), _stream(stream)))

    def refinement_map_ptr(self):
        p = C.c_void_p()
        check(lib().aw_msbg_refinement_map(self.h, C.byref(p)))
        return p.value

    def set_refinement_map(self, levels):
        import torch
        t = torch.as_tensor(np.ascontiguousarray(levels, np.uint32).view(np.int32), device="cuda")
        torch.cuda.synchronize()
        _cudart_copy(self.refinement_map_ptr(), t.data_ptr(), 4 * self.nb)
        self.allocated = False

    def refinement_map(self):
        import torch
        t = torch.empty(self.nb, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        _cudart_copy(t.data_ptr(), self.refinement_map_ptr(), 4 * self.nb)
        return t.cpu().numpy().view(np.uint32)

    def block_info(self):
        import torch
        t = torch.empty(4 * self.nb, dtype=torch.int32, device="cuda")
        check(lib().aw_msbg_block_info(self.h, t.data_ptr(), _stream()))
        return t.cpu().numpy().view(np.uint32).reshape(-1, 4)

    def levels_from_particles(self, pos, thresholds, stream=None):
        th = (C.c_int32 * max(1, len(thresholds)))(*[int(t) for t in thresholds])
        check(lib().aw_msbg_levels_from_particles(self.h, _ptr(pos), int(pos.shape[0]) if pos is not None else 0, th,
                                                  _stream(stream)))

    def enforce_grading(self, stream=None):
        n = C.c_int32()
        check(lib().aw_msbg_enforce_grading(self.h, C.byref(n), _stream(stream)))
        return n.value

    def allocate(self, stream=None):
        check(lib().aw_msbg_allocate(self.h, _stream(stream)))

    def totals(self):
        t = (C.c_uint32 * 4)()
        check(lib().aw_msbg_totals(self.h, t))
        return list(t)

    def offsets_ptr(self, kind):
        p = C.c_void_p()
        check(lib().aw_msbg_offsets(self.h, kind, C.byref(p)))
        return p.value

    def offsets(self, kind):
        import torch
        t = torch.empty(self.nb, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        _cudart_copy(t.data_ptr(), self.offsets_ptr(kind), 4 * self.nb)
        return t.cpu().numpy().view(np.uint32)

    def coarse_offsets(self, mg_level, kind):
        import torch
        t = torch.empty(self.nb, dtype=torch.int32, device="cuda")
        tot = C.c_uint32()
        check(lib().aw_msbg_coarse_offsets(self.h, mg_level, kind, t.data_ptr(), C.byref(tot), _stream()))
        return t.cpu().numpy().view(np.uint32), tot.value

    def channel(self, ch):
        """torch float32 view of a channel (shares device memory with the grid)."""
        import torch
        p = C.c_void_p()
        n = C.c_uint32()
        check(lib().aw_msbg_channel(self.h, ch, C.byref(p), C.byref(n)))
        return _tensor_from_ptr(p.value, n.value, torch.float32)

    def run_galerkin(self, fine, coarse, dest, stream=None):
        f = (C.c_void_p * 3)(*[_ptr(x) for x in fine])
        c = (C.c_void_p * 3)(*[_ptr(x) for x in coarse])
        check(lib().aw_msbg_run_galerkin(self.h, f, c, int(dest), _stream(stream)))

    # transfers ----------------------------------------------------------------------------
    def p2g(self, pos, vel, stream=None):
        check(lib().aw_p2g(self.h, _ptr(pos), _ptr(vel), int(pos.shape[0]), _stream(stream)))

    def p2g_phase(self, pos, vel, phase, rho0, rho1, stream=None):
        """p2g plus PHASE_FIELD_* and BETA_COEFF_* = 1/rho from per-particle phases in [0,1]."""
        check(lib().aw_p2g_phase(self.h, _ptr(pos), _ptr(vel), _ptr(phase), int(pos.shape[0]), float(rho0),
                                 float(rho1), _stream(stream)))

    def backup_grid_velocity(self, stream=None):
        check(lib().aw_backup_grid_velocity(self.h, _stream(stream)))

    def g2p(self, vel, pos, alpha, stream=None):
        check(lib().aw_g2p(self.h, _ptr(vel), _ptr(pos), int(pos.shape[0]), float(alpha), _stream(stream)))

    def advect(self, pos, dt, stream=None):
        check(lib().aw_advect(self.h, _ptr(pos), int(pos.shape[0]), float(dt), _stream(stream)))

    def sample_velocity(self, pts, old=False, stream=None):
        import torch
        out = torch.empty_like(pts)
        check(lib().aw_sample_velocity(self.h, _ptr(pts), int(pts.shape[0]), int(bool(old)), out.data_ptr(),
                                       _stream(stream)))
        return out

    # inspection ---------------------------------------------------------------------------
    def resample_lattice(self, dims):
        """(origin, spacing) of the dense lattice of `dims` points over the domain."""
        d = (_I32 * 3)(*[int(x) for x in dims])
        o, s = (_F * 3)(), (_F * 3)()
        check(lib().aw_resample_lattice(self.h, d, o, s))
        return tuple(o), tuple(s)

    def resample_cells(self, channel, dims, stream=None):
        """A cell channel at the dense lattice points: torch tensor (dims[2], dims[1], dims[0])."""
        import torch
        d = (_I32 * 3)(*[int(x) for x in dims])
        out = torch.empty((int(dims[2]), int(dims[1]), int(dims[0])), dtype=torch.float32, device="cuda")
        check(lib().aw_resample_cells(self.h, int(channel), d, out.data_ptr(), _stream(stream)))
        return out

    def resample_velocity(self, dims, old=False, stream=None):
        """The MAC velocity at the dense lattice points: torch tensor (dims[2], dims[1], dims[0], 3)."""
        import torch
        d = (_I32 * 3)(*[int(x) for x in dims])
        out = torch.empty((int(dims[2]), int(dims[1]), int(dims[0]), 3), dtype=torch.float32, device="cuda")
        check(lib().aw_resample_velocity(self.h, 1 if old else 0, d, out.data_ptr(), _stream(stream)))
        return out

    def vtk_write_blocks(self, path):
        check(lib().aw_vtk_write_blocks(self.h, str(path).encode()))

    def face_positions(self, axis, stream=None):
        import torch
        n = self.totals()[0 if axis == 3 else 1 + axis]
        out = torch.empty((n, 3), dtype=torch.float32, device="cuda")
        check(lib().aw_face_positions(self.h, axis, out.data_ptr(), _stream(stream)))
        return out

    def face_sync(self, channel=VELOCITY_X, stream=None):
        check(lib().aw_face_sync(self.h, channel, _stream(stream)))

    def wall_bc(self, channel=VELOCITY_X, stream=None):
        check(lib().aw_wall_bc(self.h, channel, _stream(stream)))

    def add_gravity(self, gravity, dt, stream=None):
        g = (C.c_float * 3)(*[float(v) for v in gravity])
        check(lib().aw_add_gravity(self.h, g, float(dt), _stream(stream)))

    def divergence(self, fluid, dt, stream=None):
        """(rhs = flux/dt per cell, max |div u| per unit volume)"""
        import torch
        out = torch.empty(self.totals()[0], dtype=torch.float32, device="cuda")
        mx = torch.zeros(1, dtype=torch.float32, device="cuda")
        check(lib().aw_velocity_divergence(self.h, _ptr(fluid), 1.0 / float(dt), out.data_ptr(), mx.data_ptr(),
                                           _stream(stream)))
        return out, mx

    def divergence_max64(self, fluid=None, stream=None):
        """max |div u| per unit volume of VELOCITY_* over fluid cells, face sums in FP64"""
        import torch
        out = torch.zeros(1, dtype=torch.float64, device="cuda")
        check(lib().aw_velocity_divergence_max64(self.h, _ptr(fluid), out.data_ptr(), _stream(stream)))
        return float(out.item())

    def pressure_gradient(self, solver, p, fluid, dt, stream=None):
        import torch
        check(lib().aw_pressure_gradient(self.h, solver.h, _ptr(p), int(p.dtype == torch.float64), _ptr(fluid),
                                         float(dt), _stream(stream)))

    # projection and adjoints -----------------------------------------------------------------
    def face_arrays(self, dtype=None):
        """three zeroed torch arrays shaped like the VELOCITY_* channels"""
        import torch
        t = self.totals()
        return [torch.zeros(int(t[1 + a]), dtype=dtype or torch.float32, device="cuda") for a in range(3)]

    def project(self, solver, fluid, dt, stream=None):
        check(lib().aw_project(self.h, solver.h, _ptr(fluid), float(dt), _stream(stream)))

    def vjp_project(self, solver, fluid, dt, u_bar, stream=None):
        ub = (C.c_void_p * 3)(*[_ptr(x) for x in u_bar])
        check(lib().aw_vjp_project(self.h, solver.h, _ptr(fluid), float(dt), ub, _stream(stream)))

    def vjp_p2g(self, pos, vel, u_bar, pos_bar, vel_bar, stream=None):
        ub = (C.c_void_p * 3)(*[_ptr(x) for x in u_bar])
        check(lib().aw_vjp_p2g(self.h, _ptr(pos), _ptr(vel), int(pos.shape[0]), ub, _ptr(pos_bar), _ptr(vel_bar),
                               _stream(stream)))

    def vjp_g2p(self, pos, alpha, vel_bar, pos_bar, un_bar, uo_bar, stream=None):
        a = (C.c_void_p * 3)(*[_ptr(x) for x in un_bar])
        b = (C.c_void_p * 3)(*[_ptr(x) for x in uo_bar])
        check(lib().aw_vjp_g2p(self.h, _ptr(pos), int(pos.shape[0]), float(alpha), _ptr(vel_bar), _ptr(pos_bar), a, b,
                               _stream(stream)))

    def vjp_advect(self, pos, dt, pos_bar, u_bar, stream=None):
        ub = (C.c_void_p * 3)(*[_ptr(x) for x in u_bar])
        check(lib().aw_vjp_advect(self.h, _ptr(pos), int(pos.shape[0]), float(dt), _ptr(pos_bar), ub,
                                  _stream(stream)))

    def vjp_sample(self, pts, out_bar, u_bar, pts_bar=None, old=False, stream=None):
        ub = (C.c_void_p * 3)(*[_ptr(x) for x in u_bar])
        check(lib().aw_vjp_sample(self.h, _ptr(pts), int(pts.shape[0]), int(bool(old)), _ptr(out_bar), ub,
                                  _ptr(pts_bar), _stream(stream)))

    def sort_particles(self, pos, stream=None):
        import torch
        n = int(pos.shape[0])
        keys = torch.empty(n, dtype=torch.int32, device="cuda")
        perm = torch.empty(n, dtype=torch.int32, device="cuda")
        check(lib().aw_sort_particles(self.h, _ptr(pos), n, keys.data_ptr(), perm.data_ptr(), _stream(stream)))
        return keys, perm


def vtk_write_structured_points(path, data, origin, spacing, name="field"):
    """Binary legacy VTK STRUCTURED_POINTS from a host array (nz, ny, nx) or (nz, ny, nx, 3)."""
    a = np.ascontiguousarray(data, np.float32)
    ncomp = 3 if a.ndim == 4 else 1
    dims = (_I32 * 3)(a.shape[2], a.shape[1], a.shape[0])
    check(lib().aw_vtk_write_structured_points(str(path).encode(), dims, (_F * 3)(*origin), (_F * 3)(*spacing),
                                               name.encode(), ncomp, a.ctypes.data))


def vtk_write_particles(path, pos, scalar=None, name="scalar"):
    """Binary legacy VTK POLYDATA of host positions (n, 3) with an optional float per particle."""
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    s = None if scalar is None else np.ascontiguousarray(scalar, np.float32).reshape(-1)
    if s is not None and s.shape[0] != p.shape[0]:
        raise ValueError("one scalar per particle")
    check(lib().aw_vtk_write_particles(str(path).encode(), p.ctypes.data, p.shape[0], name.encode(),
                                       None if s is None else s.ctypes.data))


def solver_default_desc(mode=OPERATOR_FV):
    d = SolverDesc()
    check(lib().aw_solver_default_desc(mode, C.byref(d)))
    return d


class Solver:
    """VCycleSolver / AdaptiveSmoother / MultigridTransfer over the C ABI."""

    def __init__(self, grid: MSBG, desc: SolverDesc | None = None, **kw):
        if desc is None:
            desc = solver_default_desc(kw.pop("operator_mode", OPERATOR_FV))
        for k, v in kw.items():
            setattr(desc, k, v)
        self.grid = grid
        self.desc = desc
        h = C.c_void_p()
        check(lib().aw_solver_create(grid.h, C.byref(desc), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().aw_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setup(self, fluid=None, stream=None):
        check(lib().aw_solver_setup(self.h, _ptr(fluid), _stream(stream)))

    def update_coefficients(self, stream=None):
        """Rebuild every level's coefficients from the grid's current BETA_COEFF_*."""
        check(lib().aw_solver_update_coefficients(self.h, _stream(stream)))

    def num_levels(self):
        n = C.c_int32()
        check(lib().aw_solver_num_levels(self.h, C.byref(n)))
        return n.value

    def level_array(self, level, which):
        """torch view of a level array: 0 x, 1 b, 2 r, 3-5 coefficients, 6 fluid (u8),
        7-10 offsets (u32 as int32), 11 res (int32)."""
        import torch
        p = C.c_void_p()
        n = C.c_uint32()
        check(lib().aw_solver_level_array(self.h, level, which, C.byref(p), C.byref(n)))
        dt = {6: torch.uint8}.get(which, torch.int32 if which >= 7 else torch.float32)
        return _tensor_from_ptr(p.value, n.value, dt)

    def smooth(self, level, iterations, stream=None):
        check(lib().aw_smoother_solve_level(self.h, level, iterations, _stream(stream)))

    def residual(self, level, stream=None):
        check(lib().aw_mg_residual(self.h, level, _stream(stream)))

    def restrict(self, level, stream=None):
        check(lib().aw_mg_restrict(self.h, level, _stream(stream)))

    def prolongate(self, level, stream=None):
        check(lib().aw_mg_prolongate(self.h, level, _stream(stream)))

    def coarsest_solve(self, stream=None):
        check(lib().aw_solver_coarsest_solve(self.h, _stream(stream)))

    def vcycle(self, stream=None):
        check(lib().aw_vcycle_run(self.h, _stream(stream)))

    def solve(self, b, p, stream=None, raise_on_error=True):
        cyc = C.c_int32()
        rel = C.c_double()
        st = lib().aw_solve(self.h, _ptr(b), _ptr(p), C.byref(cyc), C.byref(rel), _stream(stream))
        if raise_on_error:
            check(st)
        return cyc.value, rel.value, st


class Flip:
    """FLIP simulation on library-owned particle state."""

    def __init__(self, grid: MSBG, pos, vel, dt, alpha=0.95, gravity=(0.0, -9.81, 0.0), precision=PRECISION_FP32,
                 tolerance=1e-6, max_cycles=100):
        d = FlipDesc()
        d.dt, d.alpha = float(dt), float(alpha)
        d.gravity[:] = [float(g) for g in gravity]
        d.precision, d.tolerance, d.max_cycles = int(precision), float(tolerance), int(max_cycles)
        pos = np.ascontiguousarray(pos, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        self.n = pos.shape[0]
        self.grid = grid
        h = C.c_void_p()
        check(lib().aw_flip_create(grid.h, C.byref(d), pos.ctypes.data, vel.ctypes.data, self.n, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().aw_flip_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, stream=None):
        check(lib().aw_flip_step(self.h, _stream(stream)))

    def stats(self):
        s = FlipStats()
        check(lib().aw_flip_stats_get(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in FlipStats._fields_}

    def rebuild_levels(self, thresholds, stream=None):
        """Re-derive the level map from the current particles; True when the layout changed."""
        th = (C.c_int32 * max(1, len(thresholds)))(*[int(t) for t in thresholds])
        ch = C.c_int32()
        check(lib().aw_flip_rebuild_levels(self.h, th, C.byref(ch), _stream(stream)))
        return bool(ch.value)

    def set_phase(self, phase=None, rho0=1.0, rho1=1.0):
        """Two-phase simulation: phase[i] in [0,1] per particle (original order); None = one phase."""
        if phase is None:
            check(lib().aw_flip_set_phase(self.h, None, 1.0, 1.0))
            return
        ph = np.ascontiguousarray(phase, np.float32).reshape(-1)
        if ph.shape[0] != self.n:
            raise ValueError("one phase per particle")
        check(lib().aw_flip_set_phase(self.h, ph.ctypes.data, float(rho0), float(rho1)))

    def particles(self):
        pos = np.zeros((self.n, 3), np.float32)
        vel = np.zeros((self.n, 3), np.float32)
        check(lib().aw_flip_particles(self.h, pos.ctypes.data, vel.ctypes.data))
        return pos, vel


class Rollout:
    """Differentiable FLIP rollout with checkpointing (aw_rollout_* / aw_vjp_rollout).

    Particles start at `pos0` with velocities sampled from a MAC face field u0; loss = mean over
    particles of |x_final - target|^2.  u0 and its gradient are flat float32 CUDA tensors holding
    the three face arrays of the grid one after the other."""

    def __init__(self, grid: MSBG, pos0, steps, dt, alpha=0.95, gravity=(0.0, -9.81, 0.0),
                 precision=PRECISION_MIXED, tolerance=1e-6, max_cycles=100, checkpoint_every=10):
        import torch
        d = FlipDesc()
        d.dt, d.alpha = float(dt), float(alpha)
        d.gravity[:] = [float(g) for g in gravity]
        d.precision, d.tolerance, d.max_cycles = int(precision), float(tolerance), int(max_cycles)
        p = torch.as_tensor(np.ascontiguousarray(pos0, np.float32), device="cuda")
        self.n = int(p.shape[0])
        self.grid = grid
        h = C.c_void_p()
        check(lib().aw_rollout_create(grid.h, C.byref(d), p.data_ptr(), self.n, int(steps), int(checkpoint_every),
                                      C.byref(h)))
        self.h = h
        self.nfaces = sum(grid.totals()[1:])

    def close(self):
        if getattr(self, "h", None):
            lib().aw_rollout_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, u0, target, freeze_fluid=False, stream=None):
        loss = C.c_double()
        check(lib().aw_rollout_forward(self.h, _ptr(u0), _ptr(target), int(bool(freeze_fluid)), C.byref(loss),
                                       _stream(stream)))
        return loss.value

    def final_positions(self, stream=None):
        import torch
        out = torch.empty((self.n, 3), dtype=torch.float32, device="cuda")
        check(lib().aw_rollout_final_positions(self.h, out.data_ptr(), _stream(stream)))
        return out

    def vjp(self, stream=None):
        import torch
        g = torch.empty(self.nfaces, dtype=torch.float32, device="cuda")
        check(lib().aw_vjp_rollout(self.h, g.data_ptr(), _stream(stream)))
        return g


# ------------------------------------------------------------------------------------------------
def _cudart_copy(dst, src, nbytes):
    import torch
    a = _tensor_from_ptr(src, nbytes, torch.uint8)
    b = _tensor_from_ptr(dst, nbytes, torch.uint8)
    b.copy_(a)
    torch.cuda.synchronize()


def _tensor_from_ptr(ptr, count, dtype):
    """Non-owning torch CUDA tensor over library memory (lifetime tied to the owning handle)."""
    import torch
    itemsize = torch.empty((), dtype=dtype).element_size()
    if not ptr or count == 0:
        return torch.empty(0, dtype=dtype, device="cuda")

    class _CAI:
        __cuda_array_interface__ = {
            "shape": (int(count),),
            "typestr": {torch.float32: "<f4", torch.int32: "<i4", torch.uint8: "|u1", torch.float64: "<f8",
                        torch.float16: "<f2"}[dtype],
            "data": (int(ptr), False),
            "version": 3,
            "strides": None,
        }

    del itemsize
    return torch.as_tensor(_CAI(), device="cuda")


def build_grid(scene, levels=None, stream=None):
    """MSBG for a scene: level map from particles + grading + allocation (all on the GPU)."""
    import torch
    g = MSBG(scene.dims, scene.block_size, scene.domain_min, scene.base_res, scene.num_levels)
    if levels is None:
        pos = torch.as_tensor(scene.pos, device="cuda")
        g.levels_from_particles(pos, scene.thresholds, stream)
        passes = g.enforce_grading(stream)
    else:
        g.set_refinement_map(levels)
        passes = g.enforce_grading(stream)
    g.allocate(stream)
    g.grading_passes = passes
    return g
