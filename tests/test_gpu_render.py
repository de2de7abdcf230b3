"""Headless renderer (k_render.cu through ss_render) against the oracle's
restatement of the reference's fragment shaders.

The kernels and the oracle evaluate the same FP32 operations; sinf (the
per-pixel jitter hash) and expf are the CUDA and the C library versions, which
may differ in the last bit, so images are compared within one or two levels
of the 8-bit output instead of bit for bit.
"""
import numpy as np
import pytest

from smokesim_b200 import abi, scene

pytestmark = pytest.mark.gpu


def _pair(sc, steps):
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    g, o = Sim(sc["desc"]), OracleSim(sc["desc"])
    for s in (g, o):
        scene.apply(s, sc)
    for _ in range(steps):
        g.step(sc["params"])
        o.step(sc["params"])
    return g, o


def _close(a, b):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    assert d.max() <= 12, d.max()
    assert (d > 2).mean() < 2e-3, (d > 2).mean()
    assert d.mean() < 0.05, d.mean()


@pytest.mark.parametrize("nch", [1, 3])
def test_raymarch_matches_oracle(nch):
    sc = scene.plume3d(seed=3, n=32)
    sc.pop("rng", None)
    sc["desc"].density_channels = nch
    if nch == 3:
        for e in sc["emitters"]:
            e.density[1], e.density[2] = 0.5, 0.25
    g, o = _pair(sc, 8)
    d = g.render_desc(160, 120)
    img_g, img_o = g.render(d), o.render(d)
    assert img_g[..., 3].max() > 0        # some smoke is visible
    _close(img_g, img_o)


def test_draw2d_matches_oracle():
    sc = scene.plume2d(seed=2, n=64)
    sc.pop("rng", None)
    g, o = _pair(sc, 10)
    d = g.render_desc(128, 128)
    _close(g.render(d), o.render(d))


def test_render_to_device_and_ppm(tmp_path):
    import ctypes as C
    import torch
    from smokesim_b200.sim import write_ppm
    sc = scene.plume3d(seed=1, n=32)
    sc.pop("rng", None)
    g, _ = _pair(sc, 4)
    d = g.render_desc(64, 48)
    host = g.render(d)
    dev = torch.empty(64 * 48 * 4, dtype=torch.uint8, device="cuda")
    rc = g.L.ss_render(g.h, C.byref(d), C.c_void_p(dev.data_ptr()), 1, None)
    assert rc == abi.SS_OK
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy().reshape(48, 64, 4), host)
    path = tmp_path / "frame.ppm"
    write_ppm(path, host, background=(173, 216, 230))
    raw = path.read_bytes()
    assert raw.startswith(b"P6\n64 48\n255\n") and len(raw) == len(b"P6\n64 48\n255\n") + 64 * 48 * 3


@pytest.mark.parametrize("dim,nch", [(3, 1), (3, 3), (2, 1)])
def test_state_snapshot_round_trip(tmp_path, dim, nch):
    """ss_save_state / ss_load_state: the JSON header describes every section,
    the raw sections hold the fields, and a fresh simulation loaded from the
    file continues bit for bit like the original."""
    from smokesim_b200 import Sim
    from smokesim_b200.sim import read_state
    from test_gpu_parity import fields, make_pair
    n = (20, 16, 12) if dim == 3 else (24, 20, 1)
    g, _ = make_pair(dim, n, nch, 1, seed=4)
    p = scene.workload_params(ref_quirks=0, n_vcycles=2)
    g.step(p, 3)
    path = tmp_path / "state.bin"
    g.save_state(path)
    header, sec = read_state(path)
    assert header["format"] == "smokesim-state" and header["n"] == [n[0], n[1], n[2]]
    assert np.array_equal(sec["density"].ravel(), g.get_field(abi.FIELD_DENSITY).ravel())
    assert np.array_equal(sec["vx"].ravel(), g.get_field(abi.FIELD_VX).ravel())
    h = Sim(g.desc)
    h.load_state(path)
    for f in fields(dim):
        assert np.array_equal(h.get_field(f), g.get_field(f)), f
    g.step(p, 2)
    h.step(p, 2)
    for f in fields(dim):
        assert np.array_equal(h.get_field(f), g.get_field(f)), f
    other = Sim(abi.make_desc(dim, (n[0] + 2, n[1], n[2]), density_channels=nch))
    from smokesim_b200 import SmokeSimError
    with pytest.raises(SmokeSimError):
        other.load_state(path)
