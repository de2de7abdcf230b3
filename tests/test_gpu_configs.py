"""Parity of the CUDA path with the FP32 oracle on the benchmark workloads at
their full sizes, and of the host-side scene logic that drives them.

The small odd grids of test_gpu_parity.py cover every boundary branch; these
run the seeded workload scenes themselves - the 2D 256^2 plume, the 3D 128^3
plume (FP32, 4 fixed V-cycles and the reference boundary rules) and the
mixed-precision projection on the Gaussian-random-field scene at 128^3 - from
the same initial state, step by step, through the C ABI.  Every field must
match bit for bit (np.array_equal) and, as the specification states it,
within 1e-5 relative L2; the divergence statistics must agree to 1e-9.
Reference: run_physics_step (common/physics/physics.c:72-101)."""
import numpy as np
import pytest

from conftest import rel_l2
from smokesim_b200 import abi, scene
from test_gpu_parity import TOL_STEP, assert_same, fields

pytestmark = pytest.mark.gpu


def _pair(sc):
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    sc.pop("rng", None)
    g, o = Sim(sc["desc"]), OracleSim(sc["desc"])
    for s in (g, o):
        scene.apply(s, sc)
    return g, o


def _step_and_compare(g, o, p, steps, what):
    dim = g.dim
    for k in range(steps):
        g.step(p)
        o.step(p)
        assert_same(g, o, dim, f"{what} step {k}")
        for f in fields(dim):
            assert rel_l2(g.get_field(f), o.get_field(f)) <= TOL_STEP
        sg, so = g.stats(), o.stats()
        assert sg.vcycles == so.vcycles, (sg.vcycles, so.vcycles)
        for a, b in [(sg.div_before, so.div_before), (sg.div_after, so.div_after), (sg.residual, so.residual)]:
            assert abs(a - b) <= 1e-9 * max(1e-30, abs(b)), (what, k, a, b)


def test_plume2d_256_steps_bitwise():
    """2D 256^2 plume: one r=12 disc emitter, a 40x20 box, solid walls, 4
    V-cycles of 2+2 sweeps down to 8^2, the reference's boundary rules."""
    sc = scene.plume2d(seed=0, n=256)
    g, o = _pair(sc)
    _step_and_compare(g, o, sc["params"], 4, "plume2d 256")


def test_plume3d_128_steps_bitwise():
    """3D 128^3 plume: two r=8 emitters, an r=16 sphere and three cubes."""
    sc = scene.plume3d(seed=0, n=128)
    g, o = _pair(sc)
    _step_and_compare(g, o, sc["params"], 2, "plume3d 128")


@pytest.mark.parametrize("prec,warm_start,steps", [(abi.PREC_MIXED, 0, 2), (abi.PREC_MIXED_BF16, 0, 2),
                                                   (abi.PREC_MIXED, 1, 4)])
def test_grf128_mixed_tolerance_steps_bitwise(prec, warm_start, steps):
    """The benchmark's headline variant (mixed-precision projection to a
    projected divergence of 1e-6, cap 40) on its Gaussian-random-field scene
    at 128^3: the same refinement steps and the same bits as the oracle.  With
    warm_start = 1 the third and fourth solves start from the extrapolated
    pressure 2 p(n-1) - p(n-2)."""
    sc = scene.grf256(seed=0, n=128, with_grf=True)
    g, o = _pair(sc)
    p = scene.workload_params(ref_quirks=0, precision=prec, tol=1e-6, n_vcycles=40, collect_stats=1,
                              warm_start=warm_start)
    _step_and_compare(g, o, p, steps, f"grf128 mixed {prec} warm start {warm_start}")
    assert g.stats().converged == 1


def test_emitter_delay_clock_bitwise():
    """update_emitters_status (shaders3d/compute/update_emitters_status.comp:
    49-59): emitters with delays switch on and off as current_time advances
    through the steps; the records, and every field, follow the oracle."""
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    desc = abi.make_desc(3, (32, 24, 20), enclosed=1, min_coarse=4)
    g, o = Sim(desc), OracleSim(desc)
    em = [scene.emitter((8.0, 4.0, 10.0), 3.0), scene.emitter((22.0, 5.0, 9.0), 2.5, density=0.5),
          scene.emitter((16.0, 12.0, 10.0), 2.0, temperature=2.0)]
    em[0].delay = 2
    em[1].delay = 3
    em[1].last_emit = 1
    em[2].delay = 0
    for s in (g, o):
        s.set_scene(em, [scene.obstacle((16.0, 16.0, 10.0), 3.0)])
    p = scene.workload_params(n_coarse=10)
    history = []
    for k in range(14):
        p.current_time = 0.7 * k
        g.step(p)
        o.step(p)
        ge, _ = g.get_scene(3, 1)
        oe, _ = o.get_scene(3, 1)
        for a, b in zip(ge, oe):
            assert (a.emit, a.last_emit) == (b.emit, b.last_emit), (k, a.emit, a.last_emit, b.emit, b.last_emit)
        history.append(tuple(e.emit for e in ge))
        assert_same(g, o, 3, f"emitter clock step {k}")
    # the delayed emitters really toggled (on, then off for a delay, then on)
    for i in (0, 1):
        seq = [h[i] for h in history]
        assert 0 in seq and 1 in seq, seq
    assert all(h[2] == 1 for h in history)
    # the stage on its own, as the reference dispatches it
    p.current_time = 20.0
    g.update_emitters_status(p)
    o.update_emitters_status(p)
    ge, _ = g.get_scene(3, 1)
    oe, _ = o.get_scene(3, 1)
    assert [(e.emit, e.last_emit) for e in ge] == [(e.emit, e.last_emit) for e in oe]


@pytest.mark.parametrize("prec", [abi.PREC_MIXED, abi.PREC_MIXED_BF16])
def test_moving_obstacle_mixed_rebuilds_coarse_matrix(prec):
    """The mixed solve applies the coarsest level through a cached response
    matrix that must be rebuilt whenever the solid pyramid or the coarse
    iteration count changes: a falling sphere (new solid map every step), a
    change of n_coarse, and a new scene between mixed steps all follow the
    oracle, whose coarse matrix is rebuilt the same way, bit for bit."""
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    desc = abi.make_desc(3, (24, 24, 20), enclosed=1, min_coarse=3)
    g, o = Sim(desc), OracleSim(desc)
    ob = [scene.obstacle((12.0, 15.0, 10.0), 3.5, velocity=(0.3, -1.0, 0.1), anchored=0.0),
          scene.obstacle((6.0, 6.0, 6.0), 2.5)]
    for s in (g, o):
        s.set_scene([scene.emitter((12.0, 4.0, 10.0), 3.0)], ob)
    p = scene.workload_params(ref_quirks=0, precision=prec, n_vcycles=3, n_coarse=10)
    for k in range(3):
        g.step(p)
        o.step(p)
        assert_same(g, o, 3, f"moving obstacle mixed step {k}")
    p.mg.n_coarse = 17
    for k in range(2):
        g.step(p)
        o.step(p)
        assert_same(g, o, 3, f"n_coarse 17 step {k}")
    bx = [scene.box((4.0, 10.0, 4.0), (10.0, 16.0, 12.0))]
    for s in (g, o):
        s.set_scene([scene.emitter((12.0, 4.0, 10.0), 3.0)], [scene.obstacle((16.0, 12.0, 10.0), 4.0)], bx)
    for k in range(2):
        g.step(p)
        o.step(p)
        assert_same(g, o, 3, f"new scene step {k}")
