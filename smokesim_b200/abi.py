"""ctypes mirror of include/smokesim.h and the loader of libsmokesim.so.

The structures here are byte-for-byte the POD types of the C ABI; the same
definitions are used to drive the CPU oracle in the tests.  Loading the
library fails loudly: there is no CPU fallback for the smoke step.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)
LIB_PATH = os.path.join(PKG_DIR, "libsmokesim.so")

SS_OK = 0
SS_E_INVALID = -1
SS_E_CUDA = -2
SS_E_OOM = -3
SS_E_NOT_CONVERGED = -4
SS_E_NONFINITE = -5
SS_E_UNSUPPORTED = -6

SS_MAX_LEVELS = 16
SS_MAX_EMITTERS = 256
SS_MAX_OBSTACLES = 4096
SS_MAX_BOXES = 256

# stage bits (reference physics_step_settings, common/physics/physics.h:10-18)
STAGE_HANDLE_EMITTERS = 1 << 0
STAGE_ADVECT_VELOCITIES = 1 << 1
STAGE_APPLY_BUOYANCY = 1 << 2
STAGE_APPLY_VORTICITY = 1 << 3
STAGE_RESOLVE_PRESSURE = 1 << 4
STAGE_UPDATE_VELOCITIES = 1 << 5
STAGE_ADVECT_SMOKE = 1 << 6
STAGE_OBSTACLES = 1 << 7
STAGE_ALL = 0xFF

PREC_FP32 = 0
PREC_MIXED = 1
PREC_MIXED_BF16 = 2

FIELD_VX = 0
FIELD_VY = 1
FIELD_VZ = 2
FIELD_DENSITY = 3
FIELD_TEMPERATURE = 4
FIELD_PRESSURE = 5
FIELD_SOLID = 6
FIELD_DIVERGENCE = 7

LEVEL_PRESSURE = 0
LEVEL_RESIDUAL = 1
LEVEL_FLUID_WEIGHT = 2


class Desc(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("n", C.c_int * 3),
        ("cell_size", C.c_float),
        ("density_channels", C.c_int),
        ("enclosed", C.c_int),
        ("min_coarse", C.c_int),
        ("t_ambient", C.c_float),
    ]


class Emitter(C.Structure):
    _fields_ = [
        ("pos", C.c_float * 3),
        ("radius", C.c_float),
        ("density", C.c_float * 3),
        ("temperature", C.c_float),
        ("delay", C.c_int),
        ("last_emit", C.c_int),
        ("emit", C.c_int),
        ("falloff", C.c_int),
        ("set_velocity", C.c_int),
        ("velocity", C.c_float * 3),
    ]


class Obstacle(C.Structure):
    _fields_ = [
        ("pos", C.c_float * 3),
        ("radius", C.c_float),
        ("velocity", C.c_float * 3),
        ("anchored", C.c_float),
    ]


class Box(C.Structure):
    _fields_ = [
        ("lo", C.c_float * 3),
        ("hi", C.c_float * 3),
        ("velocity", C.c_float * 3),
        ("anchored", C.c_float),
    ]


class MGSchedule(C.Structure):
    _fields_ = [
        ("n_pre", C.c_int),
        ("n_post", C.c_int),
        ("n_coarse", C.c_int),
        ("n_vcycles", C.c_int),
        ("tol", C.c_double),
        ("ref_quirks", C.c_int),
        ("precision", C.c_int),
        ("warm_start", C.c_int),
    ]


class Params(C.Structure):
    _fields_ = [
        ("time_step", C.c_float),
        ("density", C.c_float),
        ("t_ambient", C.c_float),
        ("t_weight_coeff", C.c_float),
        ("t_temp_coeff", C.c_float),
        ("vorticity_confinement", C.c_float),
        ("wind", C.c_float * 3),
        ("current_time", C.c_float),
        ("stage_mask", C.c_int),
        ("collect_stats", C.c_int),
        ("mg", MGSchedule),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("vcycles", C.c_int),
        ("converged", C.c_int),
        ("div_before", C.c_double),
        ("residual", C.c_double),
        ("div_after", C.c_double),
        ("rel_div", C.c_double),
        ("steps", C.c_int),
        ("fluid_cells", C.c_int),
        ("kernel_launches", C.c_longlong),
    ]


class RenderDesc(C.Structure):
    _fields_ = [
        ("width", C.c_int),
        ("height", C.c_int),
        ("camera_pos", C.c_float * 3),
        ("camera_target", C.c_float * 3),
        ("camera_up", C.c_float * 3),
        ("fov_y", C.c_float),
        ("light_direction", C.c_float * 3),
        ("light_color", C.c_float * 3),
        ("ambient_color", C.c_float * 3),
        ("smoke_density_factor", C.c_float),
        ("shadow_density_factor", C.c_float),
        ("step_size", C.c_float),
        ("shadow_step_factor", C.c_float),
        ("shadow_steps", C.c_int),
        ("phase_g", C.c_float),
    ]


def make_desc(dim, n, cell_size=1.0, density_channels=1, enclosed=1, min_coarse=4, t_ambient=0.0):
    d = Desc()
    d.dim = dim
    n = list(n) + [1] * (3 - len(n))
    if dim == 2:
        n[2] = 1
    d.n[0], d.n[1], d.n[2] = n[0], n[1], n[2]
    d.cell_size = cell_size
    d.density_channels = density_channels
    d.enclosed = enclosed
    d.min_coarse = min_coarse
    d.t_ambient = t_ambient
    return d


def reference_params():
    """Reference defaults: physics.c:7-33 and the solver schedule of grid.c:259-295."""
    p = Params()
    p.time_step = 1.0 / 120.0
    p.density = 1.0
    p.t_ambient = 293.0
    p.t_weight_coeff = 0.07
    p.t_temp_coeff = 1.0
    p.vorticity_confinement = 1.0
    p.current_time = 0.0
    p.stage_mask = STAGE_ALL
    p.collect_stats = 0
    p.mg.n_pre = 16
    p.mg.n_post = 16
    p.mg.n_coarse = 80
    p.mg.n_vcycles = 1
    p.mg.tol = 0.0
    p.mg.ref_quirks = 1
    p.mg.precision = PREC_FP32
    return p


def make_params(dt=0.1, rho=1.0, t_ambient=0.0, alpha=0.05, beta=0.3, eps=0.2, wind=(0, 0, 0),
                n_pre=2, n_post=2, n_coarse=80, n_vcycles=4, tol=0.0, ref_quirks=1,
                precision=PREC_FP32, stage_mask=STAGE_ALL, current_time=0.0, collect_stats=1, warm_start=0):
    p = Params()
    p.time_step = dt
    p.density = rho
    p.t_ambient = t_ambient
    p.t_weight_coeff = alpha
    p.t_temp_coeff = beta
    p.vorticity_confinement = eps
    p.wind[0], p.wind[1], p.wind[2] = wind
    p.current_time = current_time
    p.stage_mask = stage_mask
    p.collect_stats = collect_stats
    p.mg.n_pre = n_pre
    p.mg.n_post = n_post
    p.mg.n_coarse = n_coarse
    p.mg.n_vcycles = n_vcycles
    p.mg.tol = tol
    p.mg.ref_quirks = ref_quirks
    p.mg.precision = precision
    p.mg.warm_start = warm_start
    return p


def field_count(dim, n, field, density_channels=1):
    nx, ny = n[0], n[1]
    nz = 1 if dim == 2 else n[2]
    cells = nx * ny * nz
    if field == FIELD_VX:
        return (nx + 1) * ny * nz
    if field == FIELD_VY:
        return nx * (ny + 1) * nz
    if field == FIELD_VZ:
        return nx * ny * (nz + 1) if dim == 3 else 0
    if field == FIELD_DENSITY:
        return cells * density_channels
    return cells


def field_shape(dim, n, field, density_channels=1):
    """numpy shape (z, y, x) of a field (density: (channels, z, y, x))."""
    nx, ny = n[0], n[1]
    nz = 1 if dim == 2 else n[2]
    if field == FIELD_VX:
        return (nz, ny, nx + 1)
    if field == FIELD_VY:
        return (nz, ny + 1, nx)
    if field == FIELD_VZ:
        return (nz + 1, ny, nx)
    if field == FIELD_DENSITY:
        return (density_channels, nz, ny, nx)
    return (nz, ny, nx)


_lock = threading.Lock()
_lib = None


def build_library(force=False):
    """Compile libsmokesim.so in-tree with nvcc for sm_100a."""
    from . import build as _build
    return _build.build(force=force)


def lib():
    """The loaded product library.  Raises if it is missing or unloadable."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            build_library()
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libsmokesim.so is missing ({LIB_PATH}); build it with __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        _declare(L)
        if L.ss_abi_version() != 1:
            raise RuntimeError("libsmokesim.so ABI version mismatch")
        _lib = L
        return L


EXPORTED = [
    "ss_create", "ss_destroy", "ss_get_desc", "ss_strerror", "ss_last_error_message", "ss_abi_version",
    "ss_default_params", "ss_set_scene", "ss_get_scene", "ss_set_field", "ss_get_field",
    "ss_field_device_ptr", "ss_clear_grid", "ss_run_physics_step", "ss_get_stats",
    "ss_update_emitters_status", "ss_handle_emitters", "ss_advect_velocities", "ss_apply_buoyancy",
    "ss_apply_vorticity", "ss_multigrid_pressure_solve", "ss_v_cycle", "ss_smooth",
    "ss_compute_residual", "ss_compute_restrict", "ss_prolong_and_add", "ss_update_velocities",
    "ss_advect_smoke", "ss_obstacle_update_step", "ss_update_solid_map", "ss_init_solid_map",
    "ss_get_level", "ss_set_level", "ss_divergence_norm_noalloc",
    "ss_set_emitter_force", "ss_set_force_field", "ss_adjoint_force_field_grad", "ss_adjoint_create", "ss_adjoint_destroy", "ss_adjoint_forward",
    "ss_adjoint_backward", "ss_adjoint_field_device_ptr", "ss_adjoint_get_field", "ss_adjoint_info",
    "ss_adjoint_set_deterministic", "ss_adjoint_set_pressure_store",
    "ss_set_field_device", "ss_get_field_device", "ss_render_default", "ss_render",
    "ss_save_state", "ss_load_state",
]


def _declare(L):
    vp, i, sz = C.c_void_p, C.c_int, C.c_size_t
    fp = C.POINTER(C.c_float)
    L.ss_create.argtypes = [C.POINTER(Desc), vp, C.POINTER(vp)]
    L.ss_destroy.argtypes = [vp]
    L.ss_get_desc.argtypes = [vp, C.POINTER(Desc), C.POINTER(i), C.POINTER(C.c_int * 3)]
    L.ss_strerror.argtypes = [i]
    L.ss_strerror.restype = C.c_char_p
    L.ss_last_error_message.argtypes = []
    L.ss_last_error_message.restype = C.c_char_p
    L.ss_abi_version.argtypes = []
    L.ss_default_params.argtypes = [C.POINTER(Params)]
    L.ss_default_params.restype = None
    L.ss_set_scene.argtypes = [vp, C.POINTER(Emitter), i, C.POINTER(Obstacle), i, C.POINTER(Box), i, vp]
    L.ss_get_scene.argtypes = [vp, C.POINTER(Emitter), i, C.POINTER(Obstacle), i]
    L.ss_set_field.argtypes = [vp, i, fp, sz, vp]
    L.ss_get_field.argtypes = [vp, i, fp, sz, vp]
    L.ss_field_device_ptr.argtypes = [vp, i, C.POINTER(vp), C.POINTER(sz)]
    L.ss_clear_grid.argtypes = [vp, C.c_float, vp]
    L.ss_run_physics_step.argtypes = [vp, C.POINTER(Params), i, vp]
    L.ss_get_stats.argtypes = [vp, C.POINTER(Stats)]
    for name in ["ss_update_emitters_status", "ss_handle_emitters", "ss_advect_velocities", "ss_apply_buoyancy",
                 "ss_apply_vorticity", "ss_multigrid_pressure_solve", "ss_update_velocities", "ss_advect_smoke",
                 "ss_obstacle_update_step"]:
        getattr(L, name).argtypes = [vp, C.POINTER(Params), vp]
    L.ss_v_cycle.argtypes = [vp, C.POINTER(Params), i, vp]
    L.ss_smooth.argtypes = [vp, C.POINTER(Params), i, i, vp]
    L.ss_compute_residual.argtypes = [vp, C.POINTER(Params), i, vp]
    L.ss_compute_restrict.argtypes = [vp, C.POINTER(Params), i, vp]
    L.ss_prolong_and_add.argtypes = [vp, C.POINTER(Params), i, vp]
    L.ss_update_solid_map.argtypes = [vp, vp]
    L.ss_init_solid_map.argtypes = [vp, vp]
    L.ss_get_level.argtypes = [vp, i, i, fp, sz, vp]
    L.ss_divergence_norm_noalloc.argtypes = [i, C.POINTER(C.c_int * 3), vp, vp, vp, vp, vp, vp]
    L.ss_set_level.argtypes = [vp, i, i, fp, sz, vp]
    L.ss_set_emitter_force.argtypes = [vp, C.POINTER(C.c_float * 3)]
    L.ss_set_force_field.argtypes = [vp, C.c_int, C.POINTER(C.c_float), vp]
    L.ss_adjoint_force_field_grad.argtypes = [vp, C.POINTER(C.c_float), C.c_size_t]
    L.ss_adjoint_create.argtypes = [vp, i, i, C.POINTER(vp)]
    L.ss_adjoint_destroy.argtypes = [vp]
    L.ss_adjoint_forward.argtypes = [vp, C.POINTER(Params), fp, vp]
    L.ss_adjoint_backward.argtypes = [vp, C.POINTER(Params), vp, vp, C.POINTER(vp * 3), fp, vp]
    L.ss_adjoint_field_device_ptr.argtypes = [vp, i, C.POINTER(vp), C.POINTER(sz)]
    L.ss_adjoint_info.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    L.ss_adjoint_set_deterministic.argtypes = [vp, i]
    L.ss_adjoint_set_pressure_store.argtypes = [vp, i]
    L.ss_adjoint_get_field.argtypes = [vp, i, vp, sz, i, vp]
    L.ss_set_field_device.argtypes = [vp, i, vp, sz, vp]
    L.ss_render_default.argtypes = [vp, i, i, C.POINTER(RenderDesc)]
    L.ss_render.argtypes = [vp, C.POINTER(RenderDesc), vp, i, vp]
    L.ss_save_state.argtypes = [vp, C.c_char_p, vp]
    L.ss_load_state.argtypes = [vp, C.c_char_p, vp]
    L.ss_get_field_device.argtypes = [vp, i, vp, sz, vp]
