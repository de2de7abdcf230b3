"""GPU test of ss_divergence_norm_noalloc, the allocation-free divergence norm.

That entry point serves callers that cannot call cudaMalloc (a host that
hands out all device memory from its own fixed budget, or a per-frame
callback where an allocation would stall the frame): it reads the caller's
velocity and solid arrays and keeps its scratch in a static device array.
Here it must agree with the divergence norm the solver reports through the
existing entry points (ss_multigrid_pressure_solve + ss_get_stats, whose
reduction uses scratch the ss_sim handle allocated), on two calls in a row,
and a repeated call must not change the device's free memory.  This file is
collected last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

from smokesim_b200 import Sim, abi, scene

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # both are FP64 sums of the same FP32 cell divergences, summed in different orders


def _grid(dim, n, seed):
    desc = abi.make_desc(dim, n, enclosed=1, min_coarse=4)
    sim = Sim(desc)
    rng = scene.Rng(seed)
    nz = n[2] if dim == 3 else 1
    em = [scene.emitter((n[0] / 2, 3.0, nz / 2), 2.5)]
    ob = [scene.obstacle((n[0] / 2, n[1] / 2, nz / 2), min(n[0], n[1]) / 5.0)]
    bx = [scene.box((2.0, n[1] - 8.0, 0.0), (7.0, n[1] - 4.0, max(1.0, nz - 3.0)))]
    sim.set_scene(em, ob, bx)
    for k, a in scene.random_state(rng, dim, n).items():
        sim.set_field(k, a)
    return sim


def _existing_norm(sim):
    p = scene.workload_params(n_vcycles=1, collect_stats=1)
    sim.multigrid_pressure_solve(p)
    return sim.stats().div_before


def _noalloc_norm(sim, out):
    import torch
    L = abi.lib()
    n = (C.c_int * 3)(*sim.n)
    u, _ = sim.device_ptr(abi.FIELD_VX)
    v, _ = sim.device_ptr(abi.FIELD_VY)
    w = sim.device_ptr(abi.FIELD_VZ)[0] if sim.dim == 3 else None
    solid, _ = sim.device_ptr(abi.FIELD_SOLID)
    rc = L.ss_divergence_norm_noalloc(sim.dim, C.byref(n), u, v, w, solid, out.data_ptr(), None)
    assert rc == abi.SS_OK, L.ss_last_error_message()
    torch.cuda.synchronize()
    return float(out.item())


@pytest.mark.parametrize("dim,n", [(3, (40, 36, 30)), (2, (70, 52, 1))])
def test_noalloc_norm_matches_solver_norm(dim, n):
    import torch
    sim = _grid(dim, n, seed=dim)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    for call in range(2):
        ref = _existing_norm(sim)
        got = [_noalloc_norm(sim, out), _noalloc_norm(sim, out)]  # two calls in a row
        assert ref > 0
        for g in got:
            assert abs(g - ref) <= RTOL * ref, (call, g, ref)
        assert got[0] == got[1]
        # advance the state so the second round sees different velocities
        sim.step(scene.workload_params(n_vcycles=1))
    sim.close()


def test_noalloc_allocates_nothing():
    import torch
    sim = _grid(3, (48, 48, 48), seed=5)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    _noalloc_norm(sim, out)  # first call on this device: one-time set-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    vals = [_noalloc_norm(sim, out) for _ in range(3)]
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free0 == free1
    assert vals[0] == vals[1] == vals[2]
    sim.close()


def test_noalloc_rejects_oversized_grid():
    import torch
    sim = _grid(3, (16, 16, 16), seed=6)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    L = abi.lib()
    n = (C.c_int * 3)(512, 512, 512)  # 134M cells > 67,108,864
    ptr = lambda f: sim.device_ptr(f)[0]
    rc = L.ss_divergence_norm_noalloc(3, C.byref(n), ptr(abi.FIELD_VX), ptr(abi.FIELD_VY), ptr(abi.FIELD_VZ),
                                      ptr(abi.FIELD_SOLID), out.data_ptr(), None)
    assert rc == abi.SS_E_INVALID
    assert b"67108864" in L.ss_last_error_message()
    assert out.item() == 0.0
    sim.close()
