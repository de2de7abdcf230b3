"""Parity of the CUDA path (through the C ABI) with the FP32 oracle.

The kernels are compiled without multiply-add contraction and with IEEE
division / square root, and keep the oracle's per-cell operation order, so
single stages are expected to match BIT FOR BIT (np.array_equal, which counts
-0.0 == 0.0).  Whole steps are checked bit for bit and additionally against
the 1e-5 relative L2 bound of the specification."""
import numpy as np
import pytest

from conftest import max_abs, rel_l2
from smokesim_b200 import abi, scene

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-5  # per-field relative L2 after one step from an identical state

GRIDS = [
    ("2d_odd", 2, (37, 29, 1), 1, 1),
    ("2d_rgb_open", 2, (33, 40, 1), 3, 0),
    ("3d_odd", 3, (19, 17, 13), 1, 1),
    ("3d_rgb_open", 3, (16, 21, 18), 3, 0),
    # nx % 8 == 0: the level-0 kernels take four cells per thread
    ("2d_quad", 2, (64, 40, 1), 1, 1),
    ("2d_quad_open_rgb", 2, (48, 34, 1), 3, 0),
    ("3d_quad_odd_y", 3, (24, 19, 18), 1, 1),
    # taller than two z chunks and wider than one x tile of the fused
    # vorticity kernel (32 x 8 cells, 32 planes per block)
    ("3d_tall_open", 3, (35, 10, 70), 1, 0),
    # colour rows of 256 cells and a row block (8 rows) that straddles the
    # grid edge
    ("3d_long_rows", 3, (512, 12, 10), 1, 1),
]


def _scene_for(dim, n, rng):
    nx, ny = n[0], n[1]
    nz = n[2]
    em = [scene.emitter((rng.uniform(None, 3, nx - 3), rng.uniform(None, 3, ny / 2), rng.uniform(None, 3, max(4, nz - 3))),
                        3.5, density=1.0, temperature=1.5, velocity=(0.2, 2.0, -0.1), falloff=1)]
    em.append(scene.emitter((nx / 2, 4.0, nz / 2), 2.5, density=0.5, temperature=1.0, velocity=(0.0, 1.0, 0.0)))
    em[1].density[1] = 0.25
    em[1].density[2] = 0.75
    ob = [scene.obstacle((nx / 2 + 0.3, ny / 2, nz / 2), min(nx, ny) / 6.0)]
    bx = [scene.box((3.0, ny - 9.0, 2.0), (9.0, ny - 5.0, max(3.0, nz - 4.0)))]
    return em, ob, bx


def make_pair(dim, n, nch, enclosed, seed=0, min_coarse=4, state=True, t_amb=0.0, stream=None):
    """stream: a CUDA stream handle for the library's simulation (the solve
    records and replays CUDA graphs only on a stream of the caller's)."""
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    desc = abi.make_desc(dim, n, cell_size=1.0, density_channels=nch, enclosed=enclosed, min_coarse=min_coarse,
                         t_ambient=t_amb)
    g = Sim(desc, stream=stream)
    o = OracleSim(desc)
    rng = scene.Rng(seed)
    em, ob, bx = _scene_for(dim, n, rng)
    for s in (g, o):
        s.set_scene(em, ob, bx)
    if state:
        f = scene.random_state(rng, dim, n, nch)
        for k, a in f.items():
            if k == abi.FIELD_DENSITY:
                a = a[: int(np.prod(g.shape(k)))]
            g.set_field(k, a)
            o.set_field(k, a)
    return g, o


def fields(dim):
    f = [abi.FIELD_VX, abi.FIELD_VY, abi.FIELD_DENSITY, abi.FIELD_TEMPERATURE, abi.FIELD_PRESSURE]
    if dim == 3:
        f.insert(2, abi.FIELD_VZ)
    return f


def assert_same(g, o, dim, what, exact=True):
    for f in fields(dim):
        a, b = g.get_field(f), o.get_field(f)
        if exact:
            assert np.array_equal(a, b), f"{what}: field {f} differs, max |d| = {max_abs(a, b):.3e}, rel L2 {rel_l2(a, b):.3e}"
        else:
            assert rel_l2(a, b) <= TOL_STEP, f"{what}: field {f} rel L2 {rel_l2(a, b):.3e}"


@pytest.mark.parametrize("name,dim,n,nch,enc", GRIDS)
def test_solid_map_and_pyramid(name, dim, n, nch, enc):
    g, o = make_pair(dim, n, nch, enc, min_coarse=3)
    assert np.array_equal(g.get_field(abi.FIELD_SOLID), o.get_field(abi.FIELD_SOLID))
    o.restrict_solid_all()
    for L in range(g.levels):
        assert np.array_equal(g.get_level(L, abi.LEVEL_FLUID_WEIGHT), o.get_level(L, abi.LEVEL_FLUID_WEIGHT)), L


STAGES = [
    ("handle_emitters", abi.STAGE_HANDLE_EMITTERS),
    ("advect_velocities", abi.STAGE_ADVECT_VELOCITIES),
    ("apply_buoyancy", abi.STAGE_APPLY_BUOYANCY),
    ("advect_velocities+buoyancy", abi.STAGE_ADVECT_VELOCITIES | abi.STAGE_APPLY_BUOYANCY),
    ("apply_vorticity", abi.STAGE_APPLY_VORTICITY),
    ("update_velocities", abi.STAGE_UPDATE_VELOCITIES),
    ("advect_smoke", abi.STAGE_ADVECT_SMOKE),
]


@pytest.mark.parametrize("name,dim,n,nch,enc", GRIDS)
@pytest.mark.parametrize("stage,mask", STAGES)
def test_single_stage_bitwise(name, dim, n, nch, enc, stage, mask):
    g, o = make_pair(dim, n, nch, enc, seed=hash(stage) & 0xFFFF)
    p = scene.workload_params(stage_mask=mask, wind=(0.3, 0.0, 0.0) if not enc else (0, 0, 0), t_ambient=0.5)
    # run twice so the ping-pong "other" buffers are exercised too
    for k in range(2):
        g.step(p)
        o.step(p)
        assert_same(g, o, dim, f"{stage} step {k}")


# 3D advection reads its taps from shared-memory tiles with a two-cell rim;
# velocities of up to ~40 cells a second (displacements of several cells at
# dt = 0.1) send many back-traces outside the tile, onto the array path.
LONG_TRACE_GRIDS = [g for g in GRIDS if g[1] == 3]


@pytest.mark.parametrize("name,dim,n,nch,enc", LONG_TRACE_GRIDS)
@pytest.mark.parametrize("stage,mask", [("advect_velocities+buoyancy", abi.STAGE_ADVECT_VELOCITIES | abi.STAGE_APPLY_BUOYANCY),
                                        ("advect_velocities", abi.STAGE_ADVECT_VELOCITIES),
                                        ("advect_smoke", abi.STAGE_ADVECT_SMOKE),
                                        ("apply_vorticity", abi.STAGE_APPLY_VORTICITY)])
@pytest.mark.parametrize("vel_scale", [4.0, 15.0])
def test_long_backtrace_bitwise(name, dim, n, nch, enc, stage, mask, vel_scale):
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    desc = abi.make_desc(dim, n, cell_size=1.0, density_channels=nch, enclosed=enc, min_coarse=3, t_ambient=0.3)
    g, o = Sim(desc), OracleSim(desc)
    rng = scene.Rng(101)
    em, ob, bx = _scene_for(dim, n, rng)
    for s in (g, o):
        s.set_scene(em, ob, bx)
    for k, a in scene.random_state(rng, dim, n, nch, vel_scale=vel_scale).items():
        if k == abi.FIELD_DENSITY:
            a = a[: int(np.prod(g.shape(k)))]
        g.set_field(k, a)
        o.set_field(k, a)
    p = scene.workload_params(stage_mask=mask, t_ambient=0.3, wind=(0.7, 0.0, 0.0) if not enc else (0, 0, 0))
    for k in range(2):
        g.step(p)
        o.step(p)
        assert_same(g, o, dim, f"{stage} x{vel_scale} step {k}")


@pytest.mark.parametrize("name,dim,n,nch,enc", GRIDS)
@pytest.mark.parametrize("quirks", [1, 0])
def test_multigrid_levels_bitwise(name, dim, n, nch, enc, quirks):
    g, o = make_pair(dim, n, nch, enc, seed=5, min_coarse=3)
    p = scene.workload_params(ref_quirks=quirks)
    o.restrict_solid_all()
    # seed the coarse right-hand sides identically
    rng = scene.Rng(77)
    for L in range(1, g.levels):
        nx, ny, nz = g.level_sizes[L]
        r = rng.normal(nx * ny * nz).astype(np.float32)
        g.set_level(L, abi.LEVEL_RESIDUAL, r)
        o.set_level(L, abi.LEVEL_RESIDUAL, r)
    for L in range(g.levels):
        g.smooth(p, L, 3)
        o.smooth(L, 3, p)
        assert np.array_equal(g.get_level(L, abi.LEVEL_PRESSURE), o.get_level(L, abi.LEVEL_PRESSURE)), f"smooth L{L}"
        g.compute_residual(p, L)
        o.compute_residual(L, p)
        assert np.array_equal(g.get_level(L, abi.LEVEL_RESIDUAL), o.get_level(L, abi.LEVEL_RESIDUAL)), f"residual L{L}"
        if L + 1 < g.levels:
            g.compute_restrict(p, L)
            o.compute_restrict(L)
            assert np.array_equal(g.get_level(L + 1, abi.LEVEL_RESIDUAL), o.get_level(L + 1, abi.LEVEL_RESIDUAL)), f"restrict L{L}"
    for L in reversed(range(g.levels - 1)):
        g.prolong_and_add(p, L)
        o.prolong_and_add(L)
        assert np.array_equal(g.get_level(L, abi.LEVEL_PRESSURE), o.get_level(L, abi.LEVEL_PRESSURE)), f"prolong L{L}"


@pytest.mark.parametrize("name,dim,n,nch,enc", GRIDS)
@pytest.mark.parametrize("quirks", [1, 0])
def test_v_cycle_bitwise(name, dim, n, nch, enc, quirks):
    g, o = make_pair(dim, n, nch, enc, seed=9, min_coarse=3)
    p = scene.workload_params(ref_quirks=quirks, n_pre=2, n_post=3, n_coarse=7)
    for _ in range(2):
        g.v_cycle(p, 0)
        o.v_cycle(0, p)
    for L in range(g.levels):
        assert np.array_equal(g.get_level(L, abi.LEVEL_PRESSURE), o.get_level(L, abi.LEVEL_PRESSURE)), f"p L{L}"


@pytest.mark.parametrize("name,dim,n,nch,enc", GRIDS)
def test_full_step_bitwise(name, dim, n, nch, enc):
    g, o = make_pair(dim, n, nch, enc, seed=21, min_coarse=3, t_amb=0.25)
    p = scene.workload_params(t_ambient=0.25, n_coarse=10)
    for k in range(3):
        g.step(p)
        o.step(p)
        assert_same(g, o, dim, f"full step {k}")
        assert_same(g, o, dim, f"full step {k}", exact=False)
    sg, so = g.stats(), o.stats()
    assert sg.vcycles == so.vcycles
    for a, b in [(sg.div_before, so.div_before), (sg.div_after, so.div_after), (sg.residual, so.residual)]:
        assert abs(a - b) <= 1e-9 * max(1.0, abs(b))


def test_reference_schedule_step_bitwise():
    """Reference defaults: dt 1/120, T_amb 293, 16+16 sweeps, 80 coarse, 1 V-cycle, h = 0.1."""
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    desc = abi.make_desc(3, (24, 24, 24), cell_size=0.1, density_channels=3, enclosed=1, min_coarse=4, t_ambient=293.0)
    g, o = Sim(desc), OracleSim(desc)
    em = [scene.emitter((12.0, 2.0, 12.0), 1.0, density=30.0, temperature=200.0, falloff=1)]
    em[0].set_velocity = 0
    ob = [scene.obstacle((12.0, 12.0, 12.0), 3.0)]
    for s in (g, o):
        s.set_scene(em, ob)
    p = abi.reference_params()
    p.collect_stats = 1
    for k in range(4):
        g.step(p)
        o.step(p)
        assert_same(g, o, 3, f"reference step {k}")


def test_tolerance_solve_matches_oracle():
    g, o = make_pair(3, (24, 20, 22), 1, 1, seed=3, min_coarse=3)
    p = scene.workload_params(ref_quirks=0, n_vcycles=40, tol=1e-5,
                              stage_mask=abi.STAGE_RESOLVE_PRESSURE | abi.STAGE_UPDATE_VELOCITIES)
    g.step(p)
    o.step(p)
    sg, so = g.stats(), o.stats()
    assert sg.converged == 1 and so.converged == 1
    assert sg.vcycles == so.vcycles
    assert sg.residual <= 1e-5 * sg.div_before
    assert_same(g, o, 3, "tolerance solve")


def test_not_converged_status():
    """A tolerance the cap cannot reach returns SS_E_NOT_CONVERGED (no hang)."""
    from smokesim_b200 import SmokeSimError
    g, _ = make_pair(3, (16, 16, 16), 1, 1, seed=4)
    p = scene.workload_params(ref_quirks=0, n_vcycles=1, tol=1e-12,
                              stage_mask=abi.STAGE_RESOLVE_PRESSURE | abi.STAGE_UPDATE_VELOCITIES)
    with pytest.raises(SmokeSimError) as e:
        g.step(p)
    assert e.value.code == abi.SS_E_NOT_CONVERGED
    assert g.stats().vcycles == 1 and g.stats().converged == 0


def test_moving_obstacle_step_bitwise():
    """A falling sphere: host dynamics + per-step rasterisation with FP16 solid velocities."""
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    desc = abi.make_desc(3, (20, 24, 20), enclosed=1, min_coarse=3)
    g, o = Sim(desc), OracleSim(desc)
    ob = [scene.obstacle((10.0, 14.0, 10.0), 3.5, velocity=(0.3, -1.0, 0.1), anchored=0.0),
          scene.obstacle((6.0, 6.0, 6.0), 2.5)]
    for s in (g, o):
        s.set_scene([scene.emitter((10.0, 4.0, 10.0), 3.0)], ob)
    p = scene.workload_params(n_coarse=10)
    for k in range(3):
        g.step(p)
        o.step(p)
        assert_same(g, o, 3, f"moving obstacle step {k}")
    _, og_ = o.get_scene(0, 2)
    _, gg = g.get_scene(0, 2)
    assert [tuple(x.pos) for x in gg] == [tuple(x.pos) for x in og_]


@pytest.mark.parametrize("workload", ["plume2d", "plume3d"])
def test_workload_scene_steps(workload):
    """The benchmark scenes (scaled down) step identically to the oracle."""
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    sc = scene.plume2d(seed=1, n=64) if workload == "plume2d" else scene.plume3d(seed=1, n=32)
    sc.pop("rng", None)
    g, o = Sim(sc["desc"]), OracleSim(sc["desc"])
    for s in (g, o):
        scene.apply(s, sc)
    dim = sc["desc"].dim
    for k in range(5):
        g.step(sc["params"])
        o.step(sc["params"])
    assert_same(g, o, dim, workload)


# Grids whose level-0 (and, for the last one, level-1) row pitch is a multiple
# of 16 bytes of flags: the red-black sweeps fetch their tiles with TMA there.
TMA_GRIDS = [
    ("3d_tma", 3, (32, 24, 20), 1, 1, 4),
    ("3d_tma_open_rgb", 3, (48, 32, 36), 3, 0, 4),
    ("3d_tma_l1", 3, (64, 48, 48), 1, 1, 8),
]


@pytest.mark.parametrize("name,dim,n,nch,enc,mc", TMA_GRIDS)
@pytest.mark.parametrize("quirks", [1, 0])
def test_v_cycle_bitwise_tma(name, dim, n, nch, enc, mc, quirks):
    g, o = make_pair(dim, n, nch, enc, seed=13, min_coarse=mc)
    p = scene.workload_params(ref_quirks=quirks, n_pre=2, n_post=2, n_coarse=12)
    for _ in range(2):
        g.v_cycle(p, 0)
        o.v_cycle(0, p)
    for L in range(g.levels):
        assert np.array_equal(g.get_level(L, abi.LEVEL_PRESSURE), o.get_level(L, abi.LEVEL_PRESSURE)), f"p L{L}"
        assert np.array_equal(g.get_level(L, abi.LEVEL_RESIDUAL), o.get_level(L, abi.LEVEL_RESIDUAL)) or L == 0, f"r L{L}"


@pytest.mark.parametrize("name,dim,n,nch,enc,mc", TMA_GRIDS)
def test_full_step_bitwise_tma(name, dim, n, nch, enc, mc):
    g, o = make_pair(dim, n, nch, enc, seed=17, min_coarse=mc, t_amb=0.1)
    p = scene.workload_params(t_ambient=0.1, n_coarse=20, n_pre=3, n_post=1)
    for k in range(2):
        g.step(p)
        o.step(p)
        assert_same(g, o, dim, f"tma full step {k}")


# Full steps with the coarse-level sweeps on TMA tiles (default) and on
# per-thread loads (SMOKESIM_TMA=0), FP32 and mixed precision.
L0_TMA_GRIDS = [
    ("3d_tma", 3, (32, 24, 20), 1, 1, 4),
    ("3d_tma_l1", 3, (64, 48, 48), 1, 1, 8),
    ("3d_long_rows", 3, (512, 12, 10), 1, 1, 4),
    ("3d_long_rows_open", 3, (512, 20, 9), 1, 0, 4),
]


@pytest.mark.parametrize("name,dim,n,nch,enc,mc", L0_TMA_GRIDS)
@pytest.mark.parametrize("tma", ["0", "1"])
@pytest.mark.parametrize("prec", [abi.PREC_FP32, abi.PREC_MIXED])
def test_full_step_bitwise_level0_paths(monkeypatch, name, dim, n, nch, enc, mc, tma, prec):
    monkeypatch.setenv("SMOKESIM_TMA", tma)
    g, o = make_pair(dim, n, nch, enc, seed=23, min_coarse=mc, t_amb=0.1)
    p = scene.workload_params(t_ambient=0.1, n_coarse=12, ref_quirks=0, precision=prec, n_vcycles=2)
    for k in range(2):
        g.step(p)
        o.step(p)
        assert_same(g, o, dim, f"level-0 path {tma} step {k}")


@pytest.mark.parametrize("h,rho", [(1.0, 2.0), (0.5, 0.75), (0.3, 0.5)])
def test_vorticity_divisor_paths(h, rho):
    """Fused vorticity confinement with 2h and rho powers of two (divisions
    taken as multiplications by the exact reciprocals) and not."""
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    n = (35, 10, 40)
    desc = abi.make_desc(3, n, cell_size=h, density_channels=1, enclosed=0, min_coarse=3)
    g, o = Sim(desc), OracleSim(desc)
    rng = scene.Rng(29)
    em, ob, bx = _scene_for(3, n, rng)
    for s in (g, o):
        s.set_scene(em, ob, bx)
    for k, a in scene.random_state(rng, 3, n, 1).items():
        g.set_field(k, a)
        o.set_field(k, a)
    p = scene.workload_params(stage_mask=abi.STAGE_APPLY_VORTICITY, rho=rho, eps=0.7)
    for _ in range(2):
        g.step(p)
        o.step(p)
    assert_same(g, o, 3, f"vorticity h={h} rho={rho}")


@pytest.mark.parametrize("n,enc,nf", [((19, 17, 13), 1, 4), ((24, 20, 18), 0, 16)])
def test_force_field_step_bitwise(n, enc, nf):
    """Coarse control force field (trilinear, clamp to edge, added after the
    emitters every step): full steps match the oracle bit for bit."""
    g, o = make_pair(3, n, 1, enc, seed=43, min_coarse=3)
    field = np.random.default_rng(3).standard_normal((3, nf, nf, nf)).astype(np.float32) * 0.5
    g.set_force_field(field)
    o.set_force_field(field)
    p = scene.workload_params(ref_quirks=0, n_coarse=10)
    for k in range(3):
        g.step(p)
        o.step(p)
        assert_same(g, o, 3, f"force field step {k}")
    g.set_force_field(None)
    o.set_force_field(None)
    g.step(p)
    o.step(p)
    assert_same(g, o, 3, "force field removed")
