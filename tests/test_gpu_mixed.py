"""Mixed-precision projection: FP64 fine-level residual and iterative
refinement, FP32 level-0 smoothing, FP16 / BF16 coarse corrections.

The oracle restates the same iteration (oracle/smokesim_oracle.c,
og_mixed_pressure_solve), rounding every coarse-level store the way the CUDA
path stores it, so a fixed number of refinement steps must agree bit for bit.
"""
import numpy as np
import pytest

from smokesim_b200 import abi, scene
from test_gpu_parity import assert_same, make_pair

# grids with an even nx (the mixed solve runs on the colour-split level 0)
MIXED_GRIDS = [
    ("3d_rgb_open", 3, (16, 21, 18), 3, 0, 4),
    ("2d_quad", 2, (64, 40, 1), 1, 1, 4),
    ("2d_quad_open_rgb", 2, (48, 34, 1), 3, 0, 4),
    ("3d_quad_odd_y", 3, (24, 19, 18), 1, 1, 4),
    ("3d_tma", 3, (32, 24, 20), 1, 1, 4),
    ("3d_l1", 3, (64, 48, 48), 1, 1, 8),
    ("3d_even_not_quad", 3, (20, 18, 14), 1, 0, 4),   # nx % 8 != 0: one cell per thread
    ("3d_long_rows", 3, (512, 12, 10), 1, 1, 4),       # colour rows of 256 cells
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,dim,n,nch,enc,mc", MIXED_GRIDS)
@pytest.mark.parametrize("prec", [abi.PREC_MIXED, abi.PREC_MIXED_BF16])
def test_mixed_solve_bitwise(name, dim, n, nch, enc, mc, prec):
    g, o = make_pair(dim, n, nch, enc, seed=31, min_coarse=mc)
    p = scene.workload_params(ref_quirks=0, precision=prec, n_vcycles=3, n_coarse=12)
    for k in range(2):
        g.step(p)
        o.step(p)
        assert_same(g, o, dim, f"mixed step {k}")
    sg, so = g.stats(), o.stats()
    assert sg.vcycles == so.vcycles == 3
    assert abs(sg.residual - so.residual) <= 1e-9 * max(1e-30, so.residual)


# Grids where the correction solve's level 0 takes the select-free
# four-cells-a-thread operators (even sizes with a whole number of quads per
# colour row): several z slabs of blocks, open and enclosed, three density
# channels, 256-cell rows, h^2 != 1 (the residual's own right-hand side).
ZERO_FORM_GRIDS = [
    ("3d_cube", 3, (32, 32, 32), 1, 1, 4, 1.0),
    ("3d_open_rgb", 3, (64, 40, 34), 3, 0, 4, 1.0),
    ("3d_tall_rows", 3, (32, 120, 12), 1, 1, 4, 1.0),
    ("3d_wide", 3, (256, 52, 10), 1, 1, 4, 1.0),
    ("3d_wide_open", 3, (128, 30, 22), 1, 0, 4, 1.0),
    ("3d_h_half", 3, (64, 32, 24), 1, 1, 4, 0.5),
    ("3d_h_03", 3, (64, 32, 24), 1, 1, 4, 0.3),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,dim,n,nch,enc,mc,h", ZERO_FORM_GRIDS)
@pytest.mark.parametrize("prec", [abi.PREC_MIXED, abi.PREC_MIXED_BF16])
def test_mixed_select_free_level0_bitwise(name, dim, n, nch, enc, mc, h, prec):
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    desc = abi.make_desc(dim, n, cell_size=h, density_channels=nch, enclosed=enc, min_coarse=mc)
    g, o = Sim(desc), OracleSim(desc)
    rng = scene.Rng(47)
    from test_gpu_parity import _scene_for
    em, ob, bx = _scene_for(dim, n, rng)
    for s_ in (g, o):
        s_.set_scene(em, ob, bx)
    for k, a in scene.random_state(rng, dim, n, nch).items():
        if k == abi.FIELD_DENSITY:
            a = a[: int(np.prod(g.shape(k)))]
        g.set_field(k, a)
        o.set_field(k, a)
    p = scene.workload_params(ref_quirks=0, precision=prec, n_vcycles=3, n_coarse=12)
    for k in range(2):
        g.step(p)
        o.step(p)
        assert_same(g, o, dim, f"select-free level 0 step {k}")
    sg, so = g.stats(), o.stats()
    assert sg.vcycles == so.vcycles == 3


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [abi.PREC_MIXED, abi.PREC_MIXED_BF16])
def test_mixed_tolerance_matches_oracle(prec):
    g, o = make_pair(3, (32, 24, 20), 1, 1, seed=3, min_coarse=4)
    p = scene.workload_params(ref_quirks=0, precision=prec, n_vcycles=40, tol=1e-6)
    for k in range(2):
        g.step(p)
        o.step(p)
        sg, so = g.stats(), o.stats()
        assert sg.converged == 1 and so.converged == 1
        assert sg.vcycles == so.vcycles
        assert sg.residual <= 1e-6 * sg.div_before
        assert_same(g, o, 3, f"mixed tolerance step {k}")


@pytest.mark.gpu
def test_mixed_reaches_tolerance_where_fp32_stalls():
    """GRF scene at 64^3: the FP32 V-cycle's FP32 residual floors above 1e-6
    relative, while refinement on the FP64 residual reaches it."""
    from smokesim_b200 import Sim, SmokeSimError
    res = {}
    for prec in (abi.PREC_FP32, abi.PREC_MIXED):
        sc = scene.grf256(seed=0, n=64)
        g = Sim(sc["desc"])
        scene.apply(g, sc)
        p = scene.workload_params(ref_quirks=0, precision=prec, n_vcycles=40, tol=1e-6)
        try:
            g.step(p)
        except SmokeSimError as e:
            assert e.code == abi.SS_E_NOT_CONVERGED
        st = g.stats()
        res[prec] = (st.converged, st.vcycles, st.residual / st.div_before)
        g.close()
    assert res[abi.PREC_MIXED][0] == 1 and res[abi.PREC_MIXED][1] <= 15, res
    assert res[abi.PREC_FP32][0] == 0 or res[abi.PREC_FP32][1] > res[abi.PREC_MIXED][1], res


@pytest.mark.gpu
def test_mixed_unsupported_and_invalid():
    from smokesim_b200 import SmokeSimError
    g, _ = make_pair(3, (19, 17, 13), 1, 1, seed=2, min_coarse=3)
    with pytest.raises(SmokeSimError) as e:
        g.step(scene.workload_params(ref_quirks=0, precision=abi.PREC_MIXED))
    assert e.value.code == abi.SS_E_UNSUPPORTED
    g2, _ = make_pair(3, (16, 16, 16), 1, 1, seed=2)
    with pytest.raises(SmokeSimError) as e:
        g2.step(scene.workload_params(ref_quirks=1, precision=abi.PREC_MIXED))
    assert e.value.code == abi.SS_E_INVALID


@pytest.mark.gpu
def test_mixed_then_fp32_warm_start():
    """Switching precision mid-run: the FP32 solve continues from the rounded
    FP64 pressure, the mixed solve from the FP32 pressure after a set_level."""
    g, o = make_pair(3, (32, 24, 20), 1, 1, seed=8, min_coarse=4)
    pm = scene.workload_params(ref_quirks=0, precision=abi.PREC_MIXED, n_vcycles=2)
    pf = scene.workload_params(ref_quirks=0, precision=abi.PREC_FP32, n_vcycles=2)
    for p in (pm, pf, pm):
        g.step(p)
        o.step(p)
        assert_same(g, o, 3, "precision switch")
    pr = np.linspace(-1, 1, 32 * 24 * 20).astype(np.float32)
    g.set_level(0, abi.LEVEL_PRESSURE, pr)
    o.set_level(0, abi.LEVEL_PRESSURE, pr)
    g.step(pm)
    o.step(pm)
    assert_same(g, o, 3, "mixed after set_level")


@pytest.mark.gpu
@pytest.mark.parametrize("stages", ["solve_only", "solve_update", "solve_update_smoke"])
def test_mixed_stage_subsets(stages):
    """The FP32 pressure copy comes from the velocity update when it follows
    the mixed solve, else from the solve itself; the post-projection
    divergence norm comes from the smoke advection when that stage runs, else
    from its own kernel.  Every subset matches the oracle."""
    masks = {
        "solve_only": abi.STAGE_RESOLVE_PRESSURE,
        "solve_update": abi.STAGE_RESOLVE_PRESSURE | abi.STAGE_UPDATE_VELOCITIES,
        "solve_update_smoke": abi.STAGE_RESOLVE_PRESSURE | abi.STAGE_UPDATE_VELOCITIES | abi.STAGE_ADVECT_SMOKE,
    }
    g, o = make_pair(3, (32, 24, 20), 1, 1, seed=41, min_coarse=4)
    p = scene.workload_params(ref_quirks=0, precision=abi.PREC_MIXED, n_vcycles=3, n_coarse=12,
                              stage_mask=masks[stages], collect_stats=1)
    for k in range(2):
        g.step(p)
        o.step(p)
        assert_same(g, o, 3, f"{stages} step {k}")
    sg, so = g.stats(), o.stats()
    pairs = [(sg.div_before, so.div_before), (sg.residual, so.residual)]
    if stages != "solve_only":
        pairs.append((sg.div_after, so.div_after))
    for a, b in pairs:
        assert abs(a - b) <= 1e-9 * max(1.0, abs(b))


@pytest.mark.gpu
@pytest.mark.parametrize("name,dim,n,nch,enc,mc", [MIXED_GRIDS[0], MIXED_GRIDS[1], MIXED_GRIDS[5]])
def test_mixed_coarse_sweeps_bitwise(monkeypatch, name, dim, n, nch, enc, mc):
    """SMOKESIM_COARSE_SWEEPS=1 sweeps the coarsest level instead of applying
    its response matrix; the oracle's sweeping form matches it bit for bit."""
    monkeypatch.setenv("SMOKESIM_COARSE_SWEEPS", "1")
    g, o = make_pair(dim, n, nch, enc, seed=41, min_coarse=mc)
    o.set_coarse_matrix(False)
    p = scene.workload_params(ref_quirks=0, precision=abi.PREC_MIXED, n_vcycles=3, n_coarse=12)
    for k in range(2):
        g.step(p)
        o.step(p)
        assert_same(g, o, dim, f"coarse sweeps step {k}")


@pytest.mark.gpu
@pytest.mark.parametrize("name,dim,n,nch,enc,mc", [MIXED_GRIDS[0], MIXED_GRIDS[1], MIXED_GRIDS[4], MIXED_GRIDS[5]])
@pytest.mark.parametrize("prec", [abi.PREC_MIXED, abi.PREC_MIXED_BF16])
def test_extrapolated_warm_start_bitwise(name, dim, n, nch, enc, mc, prec):
    """warm_start = 1: from the third consecutive mixed solve on, the solve
    starts from 2 p(n-1) - p(n-2).  Six steps of 4 refinement steps, then the
    history is broken and rebuilt twice - a step with warm_start = 0, a new
    pressure field - and each time the GPU follows the oracle bit for bit.
    (The random test state is not smooth in time, so a tolerance solve from an
    extrapolated start can take many refinement steps here; the tolerance form
    runs on the benchmark scene in test_gpu_configs.py.)"""
    g, o = make_pair(dim, n, nch, enc, seed=37, min_coarse=mc)
    p = scene.workload_params(ref_quirks=0, precision=prec, n_vcycles=4, n_coarse=12, collect_stats=1, warm_start=1)
    p0 = scene.workload_params(ref_quirks=0, precision=prec, n_vcycles=4, n_coarse=12, collect_stats=1)
    rng = np.random.default_rng(5)

    def both(params, label):
        g.step(params)
        o.step(params)
        assert_same(g, o, dim, label)
        assert g.stats().vcycles == o.stats().vcycles, (label, g.stats().vcycles, o.stats().vcycles)

    for k in range(6):
        both(p, f"extrapolated step {k}")
    both(p0, "plain warm start")
    for k in range(3):
        both(p, f"after plain step {k}")
    pr = (0.01 * rng.standard_normal(int(np.prod(g.shape(abi.FIELD_PRESSURE))))).astype(np.float32)
    g.set_field(abi.FIELD_PRESSURE, pr)
    o.set_field(abi.FIELD_PRESSURE, pr)
    for k in range(3):
        both(p, f"after a new pressure step {k}")


@pytest.mark.gpu
def test_adjoint_rejects_extrapolated_warm_start():
    from smokesim_b200 import Sim, SmokeSimError
    from smokesim_b200.adjoint import Rollout
    sc = scene.rollout64(seed=1, n=16)
    g = Sim(sc["desc"])
    scene.apply(g, sc)
    ro = Rollout(g, 2, 1)
    p = scene.workload_params(ref_quirks=0, precision=abi.PREC_MIXED, n_vcycles=2, warm_start=1)
    with pytest.raises(SmokeSimError) as e:
        ro.forward(p, np.zeros((2, 3), np.float32))
    assert e.value.code == abi.SS_E_UNSUPPORTED
    ro.close()
    g.close()
