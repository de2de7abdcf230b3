"""Host-side mirror of the reference's grid / physics_info interface.

`Sim` owns one ss_sim handle of libsmokesim.so.  Method names follow the
reference's stage functions (common/physics/grid.h:31-68 and
common/physics/physics.h:59): run_physics_step, advect_velocities,
apply_buoyancy, apply_vorticity, multigrid_pressure_solve, v_cycle, smooth,
compute_residual, compute_restrict, prolong_and_add, update_velocities,
advect_smoke, handle_emitters, update_solid_map, clear_grid.  Every call goes
through the C ABI; a non-zero status raises SmokeSimError.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi


class SmokeSimError(RuntimeError):
    def __init__(self, code, where):
        L = abi.lib()
        msg = L.ss_last_error_message().decode(errors="replace")
        super().__init__(f"{where}: {L.ss_strerror(code).decode()} ({code}): {msg}")
        self.code = code


def _check(rc, where):
    if rc != abi.SS_OK:
        raise SmokeSimError(rc, where)
    return rc


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Sim:
    def __init__(self, desc: abi.Desc, stream=None):
        self.L = abi.lib()
        self.desc = desc
        self.dim = desc.dim
        self.n = (desc.n[0], desc.n[1], 1 if desc.dim == 2 else desc.n[2])
        self.nch = desc.density_channels
        self.stream = C.c_void_p(stream) if stream is not None else C.c_void_p(None)
        h = C.c_void_p()
        _check(self.L.ss_create(C.byref(desc), self.stream, C.byref(h)), "ss_create")
        self.h = h
        lv = C.c_int()
        sizes = (C.c_int * 3 * abi.SS_MAX_LEVELS)()
        _check(self.L.ss_get_desc(self.h, None, C.byref(lv), sizes), "ss_get_desc")
        self.levels = lv.value
        self.level_sizes = [tuple(sizes[l]) for l in range(self.levels)]

    def close(self):
        if getattr(self, "h", None):
            self.L.ss_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- scene / state
    def shape(self, field):
        return abi.field_shape(self.dim, self.n, field, self.nch)

    def set_scene(self, emitters=(), obstacles=(), boxes=()):
        em = (abi.Emitter * max(1, len(emitters)))(*emitters)
        ob = (abi.Obstacle * max(1, len(obstacles)))(*obstacles)
        bx = (abi.Box * max(1, len(boxes)))(*boxes)
        _check(self.L.ss_set_scene(self.h, em, len(emitters), ob, len(obstacles), bx, len(boxes), self.stream),
               "ss_set_scene")

    def get_scene(self, n_emitters, n_obstacles):
        em = (abi.Emitter * max(1, n_emitters))()
        ob = (abi.Obstacle * max(1, n_obstacles))()
        _check(self.L.ss_get_scene(self.h, em, n_emitters, ob, n_obstacles), "ss_get_scene")
        return list(em)[:n_emitters], list(ob)[:n_obstacles]

    def set_field(self, field, arr):
        a = np.ascontiguousarray(arr, dtype=np.float32).reshape(-1)
        _check(self.L.ss_set_field(self.h, field, _fptr(a), a.size, self.stream), "ss_set_field")

    def get_field(self, field):
        shp = self.shape(field)
        a = np.empty(int(np.prod(shp)), np.float32)
        _check(self.L.ss_get_field(self.h, field, _fptr(a), a.size, self.stream), "ss_get_field")
        return a.reshape(shp)

    def device_ptr(self, field):
        p = C.c_void_p()
        n = C.c_size_t()
        _check(self.L.ss_field_device_ptr(self.h, field, C.byref(p), C.byref(n)), "ss_field_device_ptr")
        return p.value, n.value

    def get_level(self, level, what):
        nx, ny, nz = self.level_sizes[level]
        a = np.empty(nx * ny * nz, np.float32)
        _check(self.L.ss_get_level(self.h, level, what, _fptr(a), a.size, self.stream), "ss_get_level")
        return a.reshape(nz, ny, nx)

    def set_level(self, level, what, arr):
        a = np.ascontiguousarray(arr, dtype=np.float32).reshape(-1)
        _check(self.L.ss_set_level(self.h, level, what, _fptr(a), a.size, self.stream), "ss_set_level")

    def render_desc(self, width=256, height=256):
        """The reference's default render settings for this grid (ss_render_default)."""
        d = abi.RenderDesc()
        _check(self.L.ss_render_default(self.h, width, height, C.byref(d)), "ss_render_default")
        return d

    def render(self, desc=None, width=256, height=256):
        """Headless image of the current smoke, (height, width, 4) uint8, top row first."""
        d = desc if desc is not None else self.render_desc(width, height)
        out = np.empty((d.height, d.width, 4), np.uint8)
        _check(self.L.ss_render(self.h, C.byref(d), out.ctypes.data, 0, self.stream), "ss_render")
        return out

    def save_state(self, path):
        _check(self.L.ss_save_state(self.h, str(path).encode(), self.stream), "ss_save_state")

    def load_state(self, path):
        _check(self.L.ss_load_state(self.h, str(path).encode(), self.stream), "ss_load_state")

    def set_emitter_force(self, force):
        f = (C.c_float * 3)(*[float(x) for x in force])
        _check(self.L.ss_set_emitter_force(self.h, C.byref(f)), "ss_set_emitter_force")

    def set_force_field(self, field):
        """Coarse control force field, shape (3, n, n, n) (None removes it)."""
        if field is None:
            _check(self.L.ss_set_force_field(self.h, 0, None, self.stream), "ss_set_force_field")
            return
        a = np.ascontiguousarray(field, dtype=np.float32)
        n = a.shape[-1]
        if a.shape != (3, n, n, n):
            raise ValueError(f"force field must have shape (3, n, n, n), got {a.shape}")
        _check(self.L.ss_set_force_field(self.h, n, a.ctypes.data_as(C.POINTER(C.c_float)), self.stream),
               "ss_set_force_field")

    def clear_grid(self, t_ambient):
        _check(self.L.ss_clear_grid(self.h, C.c_float(t_ambient), self.stream), "ss_clear_grid")

    # ---- the step and its stages
    def run_physics_step(self, params, nsteps=1, stream=None):
        st = C.c_void_p(stream) if stream is not None else self.stream
        return _check(self.L.ss_run_physics_step(self.h, C.byref(params), nsteps, st), "ss_run_physics_step")

    step = run_physics_step

    def stats(self):
        s = abi.Stats()
        _check(self.L.ss_get_stats(self.h, C.byref(s)), "ss_get_stats")
        return s

    def _stage(self, name, params):
        _check(getattr(self.L, name)(self.h, C.byref(params), self.stream), name)

    def update_emitters_status(self, params):
        self._stage("ss_update_emitters_status", params)

    def handle_emitters(self, params):
        self._stage("ss_handle_emitters", params)

    def advect_velocities(self, params):
        self._stage("ss_advect_velocities", params)

    def apply_buoyancy(self, params):
        self._stage("ss_apply_buoyancy", params)

    def apply_vorticity(self, params):
        self._stage("ss_apply_vorticity", params)

    def multigrid_pressure_solve(self, params):
        self._stage("ss_multigrid_pressure_solve", params)

    def update_velocities(self, params):
        self._stage("ss_update_velocities", params)

    def advect_smoke(self, params):
        self._stage("ss_advect_smoke", params)

    def obstacle_update_step(self, params):
        self._stage("ss_obstacle_update_step", params)

    def v_cycle(self, params, level=0):
        _check(self.L.ss_v_cycle(self.h, C.byref(params), level, self.stream), "ss_v_cycle")

    def smooth(self, params, level, iterations):
        _check(self.L.ss_smooth(self.h, C.byref(params), level, iterations, self.stream), "ss_smooth")

    def compute_residual(self, params, level):
        _check(self.L.ss_compute_residual(self.h, C.byref(params), level, self.stream), "ss_compute_residual")

    def compute_restrict(self, params, level):
        _check(self.L.ss_compute_restrict(self.h, C.byref(params), level, self.stream), "ss_compute_restrict")

    def prolong_and_add(self, params, level):
        _check(self.L.ss_prolong_and_add(self.h, C.byref(params), level, self.stream), "ss_prolong_and_add")

    def update_solid_map(self):
        _check(self.L.ss_update_solid_map(self.h, self.stream), "ss_update_solid_map")


def write_ppm(path, rgba, background=(0, 0, 0)):
    """Binary PPM (P6) of an RGBA8 image, composited over `background`
    (premultiplied colour + (1 - alpha) * background)."""
    img = np.asarray(rgba, dtype=np.float32)
    a = img[..., 3:4] / 255.0
    rgb = img[..., :3] + (1.0 - a) * np.asarray(background, np.float32)
    rgb = np.clip(rgb + 0.5, 0, 255).astype(np.uint8)
    h, w = rgb.shape[:2]
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (w, h))
        f.write(rgb.tobytes())


def read_state(path):
    """A snapshot written by ss_save_state as (header dict, {section: array});
    FP32 sections are numpy arrays in their stated shape, record sections
    raw bytes."""
    import json
    with open(path, "rb") as f:
        header = json.loads(f.readline().decode())
        out = {}
        for sec in header["sections"]:
            f.seek(sec["offset"])
            raw = f.read(sec["bytes"])
            out[sec["name"]] = (np.frombuffer(raw, "<f4").reshape(sec["shape"]) if sec["dtype"] == "<f4" else raw)
    return header, out
