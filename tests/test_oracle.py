"""CPU tests of the oracle (the checker): known answers the reference's
algorithm must satisfy, FP32 vs FP64 agreement, and the reference quirks it
restates.  The reference ships no tests or golden vectors and its GLSL
cannot run here (no OpenGL stack), so the oracle's parity is unpinned: these
known-answer tests are what pins it."""
import numpy as np
import pytest

from conftest import rel_l2
from smokesim_b200 import abi, scene


def _open_grid(dim, n, **kw):
    return abi.make_desc(dim, n, enclosed=0, min_coarse=kw.pop("min_coarse", 4), **kw)


def test_fixed_point_zero_state(oracle_mod):
    """No emitters, zero velocity, ambient smoke: one full step changes nothing."""
    for dim, n in [(2, (20, 17, 1)), (3, (12, 11, 9))]:
        o = oracle_mod.OracleSim(abi.make_desc(dim, n, enclosed=1, t_ambient=0.0))
        p = abi.make_params(t_ambient=0.0)
        o.step(p, 2)
        for f in [abi.FIELD_VX, abi.FIELD_VY, abi.FIELD_DENSITY, abi.FIELD_TEMPERATURE, abi.FIELD_PRESSURE]:
            assert not np.any(o.get_field(f)), f


def test_uniform_translation_integer_cfl(oracle_mod):
    """Semi-Lagrangian advection with u = 1, dt = h = 1 shifts the smoke by
    exactly one cell (the back-traced point is a texel centre)."""
    n = (16, 8, 1)
    o = oracle_mod.OracleSim(_open_grid(2, n))
    o.set_field(abi.FIELD_VX, np.ones((1, 8, 17), np.float32))
    rng = np.random.default_rng(1)
    d = rng.random((1, 1, 8, 16)).astype(np.float32)
    o.set_field(abi.FIELD_DENSITY, d)
    p = abi.make_params(dt=1.0, t_ambient=0.0, stage_mask=abi.STAGE_ADVECT_SMOKE)
    o.step(p)
    out = o.get_field(abi.FIELD_DENSITY)
    assert np.array_equal(out[..., 1:], d[..., :-1])
    assert np.all(out[..., 0] == 0.0)  # border colour 0 flows in


def test_emitter_injection_exact(oracle_mod):
    """handle_emitters adds density*dt (no falloff) inside the radius, nothing outside."""
    n = (24, 24, 1)
    o = oracle_mod.OracleSim(abi.make_desc(2, n, enclosed=1))
    e = scene.emitter((10.0, 9.0, 0.0), 4.0, density=3.0, temperature=2.0, velocity=(0.0, 1.5, 0.0))
    o.set_scene([e])
    p = abi.make_params(dt=0.5, stage_mask=abi.STAGE_HANDLE_EMITTERS)
    o.step(p)
    d = o.get_field(abi.FIELD_DENSITY)[0, 0]
    T = o.get_field(abi.FIELD_TEMPERATURE)[0]
    yy, xx = np.mgrid[0:24, 0:24]
    inside = np.sqrt((xx - 10.0) ** 2 + (yy - 9.0) ** 2) < 4.0
    assert np.all(d[inside] == np.float32(1.5)) and np.all(d[~inside] == 0)
    assert np.all(T[inside] == np.float32(1.0)) and np.all(T[~inside] == 0)
    vy = o.get_field(abi.FIELD_VY)[0]
    yv, xv = np.mgrid[0:25, 0:24]
    inv = np.sqrt((xv - 10.0) ** 2 + (yv - 9.0) ** 2) < 4.0
    assert np.all(vy[inv] == np.float32(1.5)) and np.all(vy[~inv] == 0)


def test_emitter_smoothstep_falloff(oracle_mod):
    """falloff = smoothstep(r, 0, dist): 1 at the centre, 0 at the rim."""
    o = oracle_mod.OracleSim(abi.make_desc(2, (16, 16, 1), enclosed=0))
    e = scene.emitter((8.0, 8.0, 0.0), 5.0, density=1.0, temperature=0.0, falloff=1)
    e.set_velocity = 0
    o.set_scene([e])
    o.step(abi.make_params(dt=1.0, stage_mask=abi.STAGE_HANDLE_EMITTERS))
    d = o.get_field(abi.FIELD_DENSITY)[0, 0]
    assert d[8, 8] == 1.0
    t = (5.0 - 3.0) / 5.0
    assert abs(d[8, 11] - t * t * (3 - 2 * t)) < 1e-6
    assert d[8, 13] == 0.0


def test_emitter_status_delay_toggles(oracle_mod):
    """update_emitters_status: with a delay the emitter fires one frame, then waits."""
    o = oracle_mod.OracleSim(abi.make_desc(2, (8, 8, 1), enclosed=0))
    e = scene.emitter((4.0, 4.0, 0.0), 2.0)
    e.delay = 2
    e.last_emit = 0
    o.set_scene([e])
    p = abi.make_params(stage_mask=abi.STAGE_HANDLE_EMITTERS)
    seq = []
    for t in [0.0, 1.0, 2.0, 3.0, 4.0, 5.0]:
        p.current_time = t
        o.step(p)
        em, _ = o.get_scene(1, 0)
        seq.append(em[0].emit)
    assert seq == [0, 0, 1, 0, 0, 1]  # fire at t=2, reset last_emit=3, fire again at t=5


def test_solid_pyramid_alpha_values(oracle_mod):
    """restrict_solid: coarse alpha is the FP16 mean of the children, zeroed below 0.5."""
    sc = scene.plume3d(seed=3, n=32)
    o = oracle_mod.OracleSim(sc["desc"])
    o.set_scene(sc["emitters"], sc["obstacles"], sc["boxes"])
    o.restrict_solid_all()
    for L in range(1, o.levels):
        a = 1.0 - o.get_level(L, abi.LEVEL_FLUID_WEIGHT)
        assert np.all((a == 0) | ((a >= 0.5) & (a <= 1.0)))
    # an empty enclosed box: the wall survives level 1 (half of the children are
    # wall) and dissolves below it (a quarter), except along edges and corners
    o = oracle_mod.OracleSim(abi.make_desc(3, (32, 32, 32), enclosed=1))
    o.set_scene()
    o.restrict_solid_all()
    a1 = 1.0 - o.get_level(1, abi.LEVEL_FLUID_WEIGHT)
    a2 = 1.0 - o.get_level(2, abi.LEVEL_FLUID_WEIGHT)
    assert np.all(a1[0] >= 0.5) and np.all(a1[1:-1, 1:-1, 1:-1] == 0)
    assert np.all(a2[0, 1:-1, 1:-1] == 0) and a2[0, 0, 0] > 0.5


def test_wall_shell_and_valid_range(oracle_mod):
    """init_solid_map marks the shell; update_solid_map writes only 2..n-2."""
    o = oracle_mod.OracleSim(abi.make_desc(3, (10, 10, 10), enclosed=1))
    o.set_scene([], [scene.obstacle((1.0, 5.0, 5.0), 3.0)])
    s = o.get_field(abi.FIELD_SOLID)
    assert np.all(s[0] == 1) and np.all(s[-1] == 1) and np.all(s[:, :, 0] == 1)
    assert np.all(s[2:-2, 2:-2, 1] == 0)  # index 1 is never written by update_solid_map
    assert s[5, 5, 2] == 1 and s[5, 5, 3] == 1 and s[5, 5, 4] == 0


def test_buoyancy_stale_buffer_quirk(oracle_mod):
    """apply_buoyancy does not write faces touching solid: after advection the
    reference's write buffer there holds the pre-advection velocity."""
    n = (10, 10, 1)
    o = oracle_mod.OracleSim(abi.make_desc(2, n, enclosed=1))
    vy = np.full((1, 11, 10), 0.25, np.float32)
    o.set_field(abi.FIELD_VY, vy)
    o.set_field(abi.FIELD_TEMPERATURE, np.ones((1, 10, 10), np.float32))
    p = abi.make_params(stage_mask=abi.STAGE_ADVECT_VELOCITIES | abi.STAGE_APPLY_BUOYANCY)
    o.step(p)
    out = o.get_field(abi.FIELD_VY)[0]
    assert out[0, 5] == np.float32(0.25) and out[1, 5] == np.float32(0.25)  # faces touching the wall
    # interior faces: advected uniform field + beta*(T - T_amb)*dt
    assert out[5, 5] == np.float32(np.float32(0.25) + np.float32(0.3) * np.float32(1.0) * np.float32(0.1))


def test_vorticity_2d_sign(oracle_mod):
    """2D confinement uses f_x = -n_y*w (the 3D cross product gives +n_y*w)."""
    n = (12, 12, 1)
    o = oracle_mod.OracleSim(abi.make_desc(2, n, enclosed=0))
    # a solid-body rotation patch: u = -(y - c), v = (x - c) near the centre
    yy, xx = np.mgrid[0:12, 0:13].astype(np.float32)
    u = -(yy + 0.5 - 6.0) * 0.1
    yv, xv = np.mgrid[0:13, 0:12].astype(np.float32)
    v = (xv + 0.5 - 6.0) * 0.1
    o.set_field(abi.FIELD_VX, u[None])
    o.set_field(abi.FIELD_VY, v[None])
    p = abi.make_params(eps=1.0, stage_mask=abi.STAGE_APPLY_VORTICITY)
    o.step(p)
    du = o.get_field(abi.FIELD_VX)[0] - u
    assert np.any(du != 0)


def test_poisson_vcycles_converge_corrected(oracle_mod):
    """With the RHS fix (ref_quirks = 0) repeated V-cycles drive the projected
    divergence down geometrically on an obstacle domain."""
    sc = scene.plume3d(seed=1, n=32)
    o = oracle_mod.OracleSim(sc["desc"], "f64")
    o.set_scene(sc["emitters"], sc["obstacles"], sc["boxes"])
    rng = scene.Rng(7)
    f = scene.random_state(rng, 3, (32, 32, 32))
    for k in (abi.FIELD_VX, abi.FIELD_VY, abi.FIELD_VZ):
        o.set_field(k, f[k])
    p = scene.workload_params(ref_quirks=0, n_vcycles=1, stage_mask=abi.STAGE_RESOLVE_PRESSURE)
    res = []
    for _ in range(8):
        o.step(p)
        res.append(o.stats().residual / o.stats().div_before)
    assert all(b < a for a, b in zip(res, res[1:]))
    assert res[-1] < 1e-3


def test_tolerance_solve_reaches_tol_fp64(oracle_mod):
    sc = scene.plume3d(seed=2, n=32)
    o = oracle_mod.OracleSim(sc["desc"], "f64")
    o.set_scene(sc["emitters"], sc["obstacles"], sc["boxes"])
    f = scene.random_state(scene.Rng(9), 3, (32, 32, 32))
    for k in (abi.FIELD_VX, abi.FIELD_VY, abi.FIELD_VZ):
        o.set_field(k, f[k])
    p = scene.workload_params(ref_quirks=0, n_vcycles=60, tol=1e-8,
                              stage_mask=abi.STAGE_RESOLVE_PRESSURE | abi.STAGE_UPDATE_VELOCITIES)
    o.step(p)
    st = o.stats()
    assert st.converged == 1 and st.residual <= 1e-8 * st.div_before
    # the projected residual predicts the divergence actually left in the velocities
    assert st.rel_div < 1e-7


def test_fp32_vs_fp64_one_step(oracle_mod):
    """The FP32 oracle stays within 1e-4 relative L2 of the FP64 oracle after one step."""
    sc = scene.plume2d(seed=5, n=64)
    outs = []
    for prec in ("f32", "f64"):
        o = oracle_mod.OracleSim(sc["desc"], prec)
        scene.apply(o, sc)
        f = scene.random_state(scene.Rng(11), 2, (64, 64, 1))
        for k in (abi.FIELD_VX, abi.FIELD_VY, abi.FIELD_DENSITY):
            o.set_field(k, f[k])
        o.step(sc["params"])
        outs.append([o.get_field(k, f64=True) for k in (abi.FIELD_VX, abi.FIELD_VY, abi.FIELD_DENSITY, abi.FIELD_PRESSURE)])
    for a, b in zip(*outs):
        assert rel_l2(a, b) < 1e-4


def test_obstacle_falls_under_gravity(oracle_mod):
    o = oracle_mod.OracleSim(abi.make_desc(3, (16, 16, 16), enclosed=1))
    ob = scene.obstacle((8.0, 8.0, 8.0), 2.0, anchored=0.0)
    o.set_scene([], [ob])
    p = abi.make_params(dt=0.1, stage_mask=abi.STAGE_OBSTACLES)
    o.step(p)
    _, obs = o.get_scene(0, 1)
    vy = np.float32(0) + np.float32(-9.81) * np.float32(0.1) * np.float32(1.0)
    assert obs[0].velocity[1] == np.float32(vy * np.float32(0.999))
    assert obs[0].pos[1] == np.float32(np.float32(8.0) + vy * np.float32(0.1) * np.float32(1.0))


def test_mixed_precision_refinement_reaches_tolerance(oracle_mod):
    """GRF scene at 32^3: FP32 V-cycles floor above a 1e-6 relative projected
    residual; refinement on the FP64 residual with FP16 / BF16 coarse
    corrections reaches it within a few V-cycles and agrees with the FP64
    oracle's pressure to the tolerance."""
    out = {}
    for prec in (abi.PREC_FP32, abi.PREC_MIXED, abi.PREC_MIXED_BF16):
        sc = scene.grf256(seed=0, n=32)
        o = oracle_mod.OracleSim(sc["desc"], "f32")
        scene.apply(o, sc)
        o.step(scene.workload_params(ref_quirks=0, tol=1e-6, n_vcycles=40, precision=prec))
        st = o.stats()
        out[prec] = (st.converged, st.vcycles, st.residual / st.div_before, o.get_field(abi.FIELD_PRESSURE, f64=True))
    assert out[abi.PREC_FP32][0] == 0 and out[abi.PREC_FP32][2] > 1e-6
    for prec in (abi.PREC_MIXED, abi.PREC_MIXED_BF16):
        assert out[prec][0] == 1 and out[prec][1] <= 15 and out[prec][2] <= 1e-6
    sc = scene.grf256(seed=0, n=32)
    ref = oracle_mod.OracleSim(sc["desc"], "f64")
    scene.apply(ref, sc)
    ref.step(scene.workload_params(ref_quirks=0, tol=1e-10, n_vcycles=80))
    p64 = ref.get_field(abi.FIELD_PRESSURE, f64=True)
    fluid = ref.get_field(abi.FIELD_SOLID) == 0
    err = rel_l2(out[abi.PREC_MIXED][3][fluid] - out[abi.PREC_MIXED][3][fluid].mean(), p64[fluid] - p64[fluid].mean())
    assert err < 1e-4, err


@pytest.mark.parametrize("prec", [abi.PREC_MIXED, abi.PREC_MIXED_BF16])
def test_mixed_coarse_matrix_matches_sweeps(oracle_mod, prec):
    """The mixed solve's coarsest level as one product with the response
    matrix of its sweeps (default) against the sweeps themselves (GRF scene at
    32^3, coarsest 4^3, 80 iterations): the same linear map up to rounding,
    so the two solves take the same refinement steps (within one) to 1e-6 and
    their pressures agree to what that tolerance fixes (a 1e-6 relative
    residual leaves ~1e-4 in the pressure on this grid)."""
    res = {}
    for on in (True, False):
        sc = scene.grf256(seed=0, n=32)
        o = oracle_mod.OracleSim(sc["desc"], "f32")
        scene.apply(o, sc)
        o.set_coarse_matrix(on)
        for _ in range(2):
            o.step(scene.workload_params(ref_quirks=0, tol=1e-6, n_vcycles=40, precision=prec))
        st = o.stats()
        res[on] = (st.converged, st.vcycles, o.get_field(abi.FIELD_PRESSURE, f64=True))
        fluid = o.get_field(abi.FIELD_SOLID) == 0
    assert res[True][0] == res[False][0] == 1
    assert abs(res[True][1] - res[False][1]) <= 1
    a, b = res[True][2][fluid], res[False][2][fluid]
    assert rel_l2(a - a.mean(), b - b.mean()) < 1e-3


def test_render_known_answers(oracle_mod):
    """The render restatement: an empty 3D grid leaves every pixel transparent
    (the ray marches through zero density); an empty 2D grid shows the ambient
    colour; a dense block in front of the camera is opaque in the middle."""
    d = abi.RenderDesc()
    d.width, d.height = 48, 32
    o = oracle_mod.OracleSim(abi.make_desc(3, (16, 16, 16), enclosed=1))
    d.camera_pos[:] = [0.5, 0.5, 2.3]
    d.camera_target[:] = [0.5, 0.5, 0.5]
    d.camera_up[:] = [0.0, 1.0, 0.0]
    d.fov_y = 0.785398
    d.light_direction[:] = [1.0, 1.0, 1.0]
    d.light_color[:] = [1.5, 1.35, 1.2]
    d.ambient_color[:] = [0.678, 0.847, 0.902]
    d.smoke_density_factor, d.shadow_density_factor = 50.0, 50.0
    d.step_size, d.shadow_step_factor, d.shadow_steps, d.phase_g = 0.01, 3.0, 6, 0.5
    img = o.render(d)
    assert img.shape == (32, 48, 4) and not img.any()
    rho = np.zeros((16, 16, 16), np.float32)
    rho[4:12, 4:12, 4:12] = 5.0
    o.set_field(abi.FIELD_DENSITY, rho)
    img = o.render(d)
    assert img[16, 24, 3] == 255 and img[0, 0, 3] == 0
    o2 = oracle_mod.OracleSim(abi.make_desc(2, (20, 20, 1), enclosed=1))
    d.width, d.height = 10, 10
    img2 = o2.render(d)
    amb = np.round(np.array([0.678, 0.847, 0.902]) * 255).astype(np.uint8)
    assert (img2[..., :3] == amb).all() and (img2[..., 3] == 255).all()


def test_extrapolated_warm_start_saves_refinement_steps(oracle_mod):
    """The mixed solve to 1e-6 on the GRF plume at 32^3: once the start-up
    transient is over, starting from 2 p(n-1) - p(n-2) (warm_start = 1) needs
    fewer refinement steps than starting from p(n-1); the first two solves,
    without a history, are the same."""
    counts = {}
    for ws in (0, 1):
        sc = scene.grf256(seed=0, n=32)
        sc.pop("rng", None)
        o = oracle_mod.OracleSim(sc["desc"])
        scene.apply(o, sc)
        p = scene.workload_params(ref_quirks=0, precision=abi.PREC_MIXED, tol=1e-6, n_vcycles=40, collect_stats=1,
                                  warm_start=ws)
        vc = []
        for _ in range(16):
            o.step(p)
            vc.append(o.stats().vcycles)
            assert o.stats().converged == 1
        counts[ws] = vc
        o.close()
    assert counts[0][:2] == counts[1][:2]
    assert sum(counts[1][10:]) < sum(counts[0][10:]), counts
