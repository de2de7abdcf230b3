"""Adjoint of the step (k_adjoint.cu through ss_adjoint_*), checked against
central finite differences of the FP64 oracle.

For a random adjoint seed ybar on the output fields and a random direction d
on the inputs, <xbar, d> from the CUDA adjoint must match
(L(x + eps d) - L(x - eps d)) / (2 eps), L(x) = <ybar, F(x)>, F the FP64
oracle's step from the same (FP32) state.  Single stages first (stage_mask),
then full steps, rollouts with checkpointing and the control force.
"""
import numpy as np
import pytest

from smokesim_b200 import abi, scene

pytestmark = pytest.mark.gpu

VEL = [abi.FIELD_VX, abi.FIELD_VY, abi.FIELD_VZ]
ADJ_PARAMS = dict(ref_quirks=0, n_vcycles=2, n_pre=2, n_post=2, n_coarse=6)


def _setup(dim, n, nch, enc, seed, mask, force=(0.0, 0.0, 0.0), state_scale=1.0):
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    desc = abi.make_desc(dim, n, cell_size=1.0, density_channels=nch, enclosed=enc, min_coarse=4, t_ambient=0.0)
    rng = scene.Rng(seed)
    nx, ny = n[0], n[1]
    nz = n[2] if dim == 3 else 1
    em = [scene.emitter((nx / 2 + 0.3, 3.5, nz / 2 + 0.2), 3.0, density=1.0, temperature=1.0, velocity=(0.0, 1.5, 0.0))]
    ob = [scene.obstacle((nx / 2, ny / 2 + 1.0, nz / 2), min(nx, ny) / 6.0)]
    f = scene.random_state(rng, dim, n, nch, vel_scale=state_scale)
    p = scene.workload_params(stage_mask=mask, **ADJ_PARAMS)
    g = Sim(desc)
    g.set_scene(em, ob, [])
    for k, a in f.items():
        g.set_field(k, a[: abi.field_count(dim, n, k, nch)] if k == abi.FIELD_DENSITY else a)
    return desc, em, ob, f, p, g


def _fields(dim):
    return VEL[:dim] + [abi.FIELD_DENSITY, abi.FIELD_TEMPERATURE, abi.FIELD_PRESSURE]


def _oracle_loss(desc, em, ob, f, p, ybar, x_dir, eps, force, dim, nch, n):
    """<ybar, F(x + eps * x_dir)> in the FP64 oracle."""
    from oracle.oracle import OracleSim
    o = OracleSim(desc, "f64")
    o.set_scene(em, ob, [])
    for k, a in f.items():
        base = (a[: abi.field_count(dim, n, k, nch)] if k == abi.FIELD_DENSITY else a).astype(np.float64)
        if k in x_dir:
            base = base + eps * x_dir[k]
        o.set_field_f64(k, base)
    o.set_emitter_force(force)
    o.step(p)
    tot = 0.0
    for k, yb in ybar.items():
        tot += float(np.dot(yb.astype(np.float64), o.get_field(k, f64=True).ravel()))
    o.close()
    return tot


def _directional(dim, n, nch, enc, mask, seed=1, force=(0.0, 0.0, 0.0), eps=1e-4, tol=2e-3, deterministic=False):
    from smokesim_b200.adjoint import Rollout
    import torch
    desc, em, ob, f, p, g = _setup(dim, n, nch, enc, seed, mask)
    rng = np.random.default_rng(seed + 100)
    outs = VEL[:dim] + [abi.FIELD_DENSITY, abi.FIELD_TEMPERATURE]
    ybar = {k: rng.standard_normal(abi.field_count(dim, n, k, nch)).astype(np.float32) for k in outs}
    ins = _fields(dim)
    x_dir = {k: rng.standard_normal(abi.field_count(dim, n, k, nch)) for k in ins}
    ro = Rollout(g, 1, deterministic=deterministic)
    fr = np.array([force], np.float32)
    ro.forward(p, fr)
    dev = {k: torch.from_numpy(v).cuda() for k, v in ybar.items()}
    torch.cuda.synchronize()
    gf = ro.backward(p, grad_density=dev[abi.FIELD_DENSITY].data_ptr(),
                     grad_temperature=dev[abi.FIELD_TEMPERATURE].data_ptr(),
                     grad_velocity=[dev[k].data_ptr() for k in VEL[:dim]])
    adj = sum(float(np.dot(ro.grad(k).astype(np.float64), x_dir[k])) for k in ins)
    lp = _oracle_loss(desc, em, ob, f, p, ybar, x_dir, eps, force, dim, nch, n)
    lm = _oracle_loss(desc, em, ob, f, p, ybar, x_dir, -eps, force, dim, nch, n)
    fd = (lp - lm) / (2 * eps)
    assert abs(adj - fd) <= tol * max(abs(fd), 1e-6), (adj, fd)
    # force gradient (emitter stage): FD on each component
    if mask & abi.STAGE_HANDLE_EMITTERS:
        for d in range(dim):
            fp_, fm_ = list(force), list(force)
            fp_[d] += eps
            fm_[d] -= eps
            zero = {k: np.zeros_like(v) for k, v in x_dir.items()}
            fdf = (_oracle_loss(desc, em, ob, f, p, ybar, zero, 0.0, fp_, dim, nch, n) -
                   _oracle_loss(desc, em, ob, f, p, ybar, zero, 0.0, fm_, dim, nch, n)) / (2 * eps)
            assert abs(gf[0, d] - fdf) <= tol * max(abs(fdf), 1e-6), (d, gf[0, d], fdf)
    ro.close()
    g.close()


STAGES = [
    ("emitters", abi.STAGE_HANDLE_EMITTERS),
    ("advect", abi.STAGE_ADVECT_VELOCITIES),
    ("advect_buoyancy", abi.STAGE_ADVECT_VELOCITIES | abi.STAGE_APPLY_BUOYANCY),
    ("buoyancy", abi.STAGE_APPLY_BUOYANCY),
    ("vorticity", abi.STAGE_APPLY_VORTICITY),
    ("update", abi.STAGE_UPDATE_VELOCITIES),
    ("projection", abi.STAGE_RESOLVE_PRESSURE | abi.STAGE_UPDATE_VELOCITIES),
    ("smoke", abi.STAGE_ADVECT_SMOKE),
    ("full", abi.STAGE_ALL),
]
GRIDS = [
    ("3d", 3, (16, 14, 12), 1, 1),
    ("3d_open_rgb", 3, (12, 16, 10), 3, 0),
    ("2d", 2, (24, 20, 1), 1, 1),
]


@pytest.mark.parametrize("gname,dim,n,nch,enc", GRIDS)
@pytest.mark.parametrize("stage,mask", STAGES)
def test_stage_adjoint_matches_fd(gname, dim, n, nch, enc, stage, mask):
    _directional(dim, n, nch, enc, mask, seed=3, force=(0.3, -0.2, 0.1)[:dim] + (0.0,) * (3 - dim))


def test_rollout_checkpointing_consistent():
    """The same rollout's gradients with checkpoints every 1, 3 and 8 steps
    (recomputation in between) agree up to the atomics' summation order."""
    from smokesim_b200 import Sim
    from smokesim_b200.adjoint import Rollout
    import torch
    sc = scene.rollout64(seed=2, n=24)
    p = scene.workload_params(ref_quirks=0, n_vcycles=4)
    nsteps = 8
    forces = np.random.default_rng(0).standard_normal((nsteps, 3)).astype(np.float32) * 0.2
    res = []
    for every in (1, 3, 8):
        g = Sim(sc["desc"])
        scene.apply(g, sc)
        ro = Rollout(g, nsteps, every)
        ro.forward(p, forces)
        target = torch.ones(abi.field_count(3, g.n, abi.FIELD_DENSITY), device="cuda") * 0.1
        gd = 2 * (torch.from_numpy(g.get_field(abi.FIELD_DENSITY).ravel()).cuda() - target)
        torch.cuda.synchronize()
        gf = ro.backward(p, grad_density=gd.data_ptr())
        res.append((gf, [ro.grad(k) for k in VEL], ro.info()))
        ro.close()
        g.close()
    for gf, gv, _ in res[1:]:
        assert np.allclose(gf, res[0][0], rtol=1e-4, atol=1e-6 * np.abs(res[0][0]).max())
        for a, b in zip(gv, res[0][1]):
            assert np.allclose(a, b, rtol=1e-3, atol=1e-5 * np.abs(b).max())
    # every step: 8 checkpoints + 1 step record; every 3: 3 checkpoints + 3 records
    assert res[1][2]["checkpoint_bytes"] < res[0][2]["checkpoint_bytes"]


# Coordinates whose derivative is at least this fraction of the largest one
# are held to the relative bound one by one; smaller ones (where the FP32
# gradient's absolute rounding dominates) to the same absolute error as a
# coordinate at the floor.
FD_FLOOR = 1e-2
FD_REL = 1e-3


@pytest.mark.parametrize("prec", [abi.PREC_FP32, abi.PREC_MIXED])
def test_rollout_gradient_vs_fp64_fd(prec):
    """The differentiable-rollout configuration at 32^3: 64 steps, checkpoint
    every 8, 4 V-cycles (refinement steps) a step, L2 loss between the final
    density and a target run whose emitter is shifted 6 cells in x.
    dL/d(initial velocity) and dL/d(per-step force) on 32 random control
    coordinates against FP64 central differences with h = 1e-3, coordinate by
    coordinate: relative error <= 1e-3 wherever |dL/dx| >= 1e-2 max |dL/dx|,
    absolute error <= 1e-5 max |dL/dx| below that floor.  Semi-Lagrangian
    advection is piecewise smooth: where h = 1e-3 straddles a kink (the 1e-3
    and 1e-4 differences disagree by more than the bound) the h = 1e-4
    difference is the reference for that coordinate.  The GPU forward runs the
    FP32 or the mixed-precision projection; the FP64 differences use the FP32
    scheme, the same map in exact arithmetic."""
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    from smokesim_b200.adjoint import Rollout
    import torch
    n, nsteps, every = 32, 64, 8
    sc = scene.rollout64(seed=5, n=n)
    p = scene.workload_params(ref_quirks=0, n_vcycles=4)
    rng = np.random.default_rng(7)
    forces = (rng.standard_normal((nsteps, 3)) * 0.2).astype(np.float32)
    target = scene.rollout64(seed=6, n=n)
    # target density: a rollout with the emitter shifted by 6 cells (x 32/64) in x
    tsim = OracleSim(target["desc"], "f64")
    target["emitters"][0].pos[0] += 6.0 * n / 64
    scene.apply(tsim, target)
    for _ in range(nsteps):
        tsim.step(p)
    rho_t = tsim.get_field(abi.FIELD_DENSITY, f64=True).ravel()

    def loss_fp64(dvel, dforce, h):
        o = OracleSim(sc["desc"], "f64")
        scene.apply(o, sc)
        for k in VEL:
            base = sc["fields"][k].astype(np.float64).ravel()
            if k in dvel:
                base = base.copy()
                base[dvel[k]] += h
            o.set_field_f64(k, base)
        for s in range(nsteps):
            fo = forces[s].astype(np.float64).copy()
            if dforce is not None and dforce[0] == s:
                fo[dforce[1]] += h
            o.set_emitter_force(fo)
            o.step(p)
        r = o.get_field(abi.FIELD_DENSITY, f64=True).ravel()
        o.close()
        return float(np.sum((r - rho_t) ** 2))

    g = Sim(sc["desc"])
    scene.apply(g, sc)
    pg = scene.workload_params(ref_quirks=0, n_vcycles=4, precision=prec)
    ro = Rollout(g, nsteps, every)
    ro.forward(pg, forces)
    rho = torch.from_numpy(g.get_field(abi.FIELD_DENSITY).ravel()).cuda().double()
    gd = (2 * (rho - torch.from_numpy(rho_t).cuda())).float().contiguous()
    torch.cuda.synchronize()
    gf = ro.backward(pg, grad_density=gd.data_ptr())
    gvel = {k: ro.grad(k) for k in VEL}
    # 32 coordinates: 24 initial face velocities in the plume's region (the
    # column of cells within 8 of the emitter in x and z, below mid-height:
    # elsewhere the final density does not depend on them), 8 force components
    picks = []
    ex, ez = int(sc["emitters"][0].pos[0]), int(sc["emitters"][0].pos[2])
    for _ in range(24):
        c = int(rng.integers(0, 3))
        k = VEL[c]
        x = int(rng.integers(ex - 8, ex + 8)) + (c == 0)
        y = int(rng.integers(1, n // 2))
        z = int(rng.integers(ez - 8, ez + 8)) + (c == 2)
        ax, ay = n + (c == 0), n + (c == 1)
        picks.append(("v", k, (z * ay + y) * ax + x))
    for _ in range(8):
        picks.append(("f", int(rng.integers(0, nsteps)), int(rng.integers(0, 3))))

    def central(kind, a, b, hh):
        if kind == "v":
            return (loss_fp64({a: b}, None, hh) - loss_fp64({a: b}, None, -hh)) / (2 * hh)
        return (loss_fp64({}, (a, b), hh) - loss_fp64({}, (a, b), -hh)) / (2 * hh)

    adj = np.array([gvel[a][b] if kind == "v" else gf[a, b] for kind, a, b in picks], np.float64)
    fd = np.array([central(kind, a, b, 1e-3) for kind, a, b in picks])
    scale = np.abs(fd).max()
    assert scale > 0

    def bad(x, ref):
        return abs(x - ref) > (FD_REL * abs(ref) if abs(ref) >= FD_FLOOR * scale else FD_REL * FD_FLOOR * scale)

    kinks = 0
    for i, (kind, a, b) in enumerate(picks):
        if bad(adj[i], fd[i]):
            fd4 = central(kind, a, b, 1e-4)
            if bad(fd[i], fd4):   # h = 1e-3 crosses a kink
                fd[i] = fd4
                kinks += 1
    above = np.abs(fd) >= FD_FLOOR * scale
    rel = np.abs(adj - fd) / np.maximum(np.abs(fd), 1e-300)
    absn = np.abs(adj - fd) / scale
    report = [(kind, float(x), float(y)) for (kind, _, _), x, y in zip(picks, adj, fd)]
    assert above.sum() >= 12, (int(above.sum()), report)
    assert rel[above].max() <= FD_REL, (float(rel[above].max()), report)
    assert (~above).sum() == 0 or absn[~above].max() <= FD_REL * FD_FLOOR, (float(absn[~above].max()), report)
    assert kinks <= 6, (kinks, report)
    ro.close()
    g.close()


def test_inverse_problem_reduces_loss():
    """Fit per-step emitter forces to a target density with Adam through the
    autograd binding: the loss must fall."""
    import torch
    from smokesim_b200 import Sim
    from smokesim_b200.adjoint import Rollout, rollout_fn
    n, nsteps = 24, 6
    sc = scene.rollout64(seed=1, n=n)
    p = scene.workload_params(ref_quirks=0, n_vcycles=2)
    tgt = scene.rollout64(seed=1, n=n)
    tgt["emitters"][0].pos[0] += 3.0
    t = Sim(tgt["desc"])
    scene.apply(t, tgt)
    t.step(p, nsteps)
    rho_t = torch.from_numpy(t.get_field(abi.FIELD_DENSITY).ravel()).cuda()
    g = Sim(sc["desc"])
    scene.apply(g, sc)
    ro = Rollout(g, nsteps, 2)
    fn = rollout_fn(ro, p)
    vel0 = [torch.from_numpy(sc["fields"][k].ravel()).cuda() for k in VEL]
    forces = torch.zeros(nsteps, 3, requires_grad=True)
    opt = torch.optim.Adam([forces], lr=0.5)
    losses = []
    for _ in range(6):
        opt.zero_grad()
        rho = fn(forces.cuda(), *vel0)
        loss = ((rho - rho_t) ** 2).sum()
        loss.backward()
        opt.step()
        losses.append(float(loss))
    assert losses[-1] < losses[0], losses
    ro.close()
    g.close()


def test_force_field_gradient_vs_fp64_fd():
    """dL/d(coarse force field) of a 4-step rollout at 24^3 (a 4^3 field) on 8
    random field coordinates against FP64 central differences (h = 1e-3,
    h = 1e-4 where h = 1e-3 crosses an advection kink)."""
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    from smokesim_b200.adjoint import Rollout
    import torch
    n, nsteps, nf = 24, 4, 4
    sc = scene.rollout64(seed=8, n=n)
    p = scene.workload_params(ref_quirks=0, n_vcycles=4)
    rng = np.random.default_rng(9)
    field = (rng.standard_normal((3, nf, nf, nf)) * 0.3).astype(np.float32)
    rho_t = np.full(abi.field_count(3, (n, n, n), abi.FIELD_DENSITY), 0.05)

    def loss_fp64(coord, h):
        o = OracleSim(sc["desc"], "f64")
        scene.apply(o, sc)
        f = field.astype(np.float64).copy()
        if coord is not None:
            f[coord] += h
        o.set_force_field(f)
        for _ in range(nsteps):
            o.step(p)
        r = o.get_field(abi.FIELD_DENSITY, f64=True).ravel()
        o.close()
        return float(np.sum((r - rho_t) ** 2))

    g = Sim(sc["desc"])
    scene.apply(g, sc)
    g.set_force_field(field)
    ro = Rollout(g, nsteps, 2)
    ro.forward(p, np.zeros((nsteps, 3), np.float32))
    rho = torch.from_numpy(g.get_field(abi.FIELD_DENSITY).ravel()).cuda().double()
    gd = (2 * (rho - torch.from_numpy(rho_t).cuda())).float().contiguous()
    torch.cuda.synchronize()
    ro.backward(p, grad_density=gd.data_ptr())
    grad = ro.force_field_grad(nf)
    picks = [tuple(int(v) for v in (rng.integers(0, 3), rng.integers(0, nf), rng.integers(0, nf), rng.integers(0, nf)))
             for _ in range(8)]

    def central(c, hh):
        return (loss_fp64(c, hh) - loss_fp64(c, -hh)) / (2 * hh)

    adj = np.array([grad[c] for c in picks], np.float64)
    fd = np.array([central(c, 1e-3) for c in picks])
    scale = np.abs(fd).max()
    assert scale > 0
    for i, c in enumerate(picks):
        if abs(adj[i] - fd[i]) > 1e-3 * scale:
            fd4 = central(c, 1e-4)
            if abs(fd4 - fd[i]) > 1e-3 * scale:
                fd[i] = fd4
    err = np.abs(adj - fd) / scale
    assert err.max() <= 1e-3, (err.max(), list(zip(adj, fd)))
    ro.close()
    g.close()


def test_inverse_control_gradient_vs_fp64_fd():
    """The inverse-control configuration at its full size: plume scene at
    128^3, controls = per-step emitter forces + a 16^3 coarse force field,
    mixed-precision projection in the forward, checkpoints every 14 steps,
    loss = L2 to the density of a run whose two emitters sit 10 cells further
    apart in x.  The gradient on control coordinates against FP64 central
    differences of the oracle, coordinate by coordinate to 1e-3 relative.  The
    FP64 differences over 200 steps at 128^3 take hours on the host, so the
    horizon here is 28 steps (two checkpoint segments, the recomputation
    included) at a fixed 6 refinement steps a step (the tolerance solve's
    typical count), the FP64 run using the FP32 scheme's 6 V-cycles - the same
    map in exact arithmetic.

    Vorticity confinement is off in both runs.  Its force direction N =
    g / (|g| + 1e-20), g the gradient of |curl u|, turns with g, so near every
    extremum of |curl u| (every vortex core, once the plume has rolled up) its
    exact derivative grows like |curl u| / |g|: at 28 steps the adjoint's
    largest field coefficient is ~1e6 where h = 1e-3 differences see ~1e-2.
    The derivative is exact but holds only for perturbations far below any
    finite difference, so this check leaves that stage to the stage-level
    checks.  Every other stage runs.

    First iteration (all controls zero, as Adam starts): the emitter sets the
    faces inside it to its velocity (0, 2, 0) plus dt times the force, so at a
    zero force their x and z velocities are exactly zero and the velocity
    advection that follows traces them back exactly onto grid nodes, where
    the trilinear interpolant's slope jumps.  The loss has a kink there in the
    force's x and z components (and partly in the x and z field
    coefficients): central differences average the two one-sided slopes, the
    adjoint returns the slope of the cell its floor selects.  So the first
    iteration is checked on a y force, a y field coefficient and the field
    coefficient of largest gradient, and all five picks (x and y of each
    kind, and that coefficient) at controls of the size of Adam's first step
    (lr 1e-2), seeded Gaussian with standard deviation 1e-2.  (Adam's first
    step itself, every control at exactly -1e-2 sign(gradient), lands on the
    kinks again: emitter force and interpolated field cancel exactly on some
    emitter faces.)"""
    from oracle.oracle import OracleSim
    from smokesim_b200 import Sim
    from smokesim_b200.adjoint import Rollout
    import torch
    n, nsteps, every, nf, ncyc = 128, 28, 14, 16, 6
    mask = abi.STAGE_ALL & ~abi.STAGE_APPLY_VORTICITY
    sc = scene.plume3d(seed=0, n=n)
    sc.pop("rng", None)
    tgt = scene.plume3d(seed=0, n=n)
    tgt.pop("rng", None)
    tgt["emitters"][0].pos[0] -= 5.0
    tgt["emitters"][1].pos[0] += 5.0
    p64 = scene.workload_params(ref_quirks=0, n_vcycles=ncyc, stage_mask=mask)
    pg = scene.workload_params(ref_quirks=0, n_vcycles=ncyc, precision=abi.PREC_MIXED, stage_mask=mask)
    to = OracleSim(tgt["desc"], "f64")
    scene.apply(to, tgt)
    for _ in range(nsteps):
        to.step(p64)
    rho_t = to.get_field(abi.FIELD_DENSITY, f64=True).ravel()
    to.close()

    def loss_fp64(forces, field, dforce, dfield, h):
        o = OracleSim(sc["desc"], "f64")
        scene.apply(o, sc)
        f = field.astype(np.float64).copy()
        if dfield is not None:
            f[dfield] += h
        o.set_force_field(f)
        for s_ in range(nsteps):
            fo = forces[s_].astype(np.float64).copy()
            if dforce is not None and dforce[0] == s_:
                fo[dforce[1]] += h
            o.set_emitter_force(fo)
            o.step(p64)
        r = o.get_field(abi.FIELD_DENSITY, f64=True).ravel()
        o.close()
        return float(np.sum((r - rho_t) ** 2))

    def adjoint(forces, field):
        g = Sim(sc["desc"])
        scene.apply(g, sc)
        g.set_force_field(field)
        ro = Rollout(g, nsteps, every)
        ro.forward(pg, forces)
        rho = torch.from_numpy(g.get_field(abi.FIELD_DENSITY).ravel()).cuda().double()
        gd = (2 * (rho - torch.from_numpy(rho_t).cuda())).float().contiguous()
        torch.cuda.synchronize()
        gf = ro.backward(pg, grad_density=gd.data_ptr())
        gfield = ro.force_field_grad(nf)
        ro.close()
        g.close()
        return gf, gfield

    def check(forces, field, gf, gfield, picks):
        def central(pk, hh):
            if pk[0] == "f":
                return (loss_fp64(forces, field, (pk[1], pk[2]), None, hh)
                        - loss_fp64(forces, field, (pk[1], pk[2]), None, -hh)) / (2 * hh)
            return (loss_fp64(forces, field, None, pk[1], hh) - loss_fp64(forces, field, None, pk[1], -hh)) / (2 * hh)

        adj = np.array([gf[pk[1], pk[2]] if pk[0] == "f" else gfield[pk[1]] for pk in picks], np.float64)
        fd = np.array([central(pk, 1e-3) for pk in picks])
        for i, pk in enumerate(picks):
            if abs(adj[i] - fd[i]) > FD_REL * abs(fd[i]):
                fd4 = central(pk, 1e-4)
                if abs(fd4 - fd[i]) > FD_REL * abs(fd4):   # h = 1e-3 crosses an advection kink
                    fd[i] = fd4
        assert np.all(np.abs(fd) > 0)
        rel = np.abs(adj - fd) / np.abs(fd)
        assert rel.max() <= FD_REL, (rel.tolist(), list(zip(adj.tolist(), fd.tolist())))

    # the coarse cells holding the two emitters (cell-centred samples of n/nf cells)
    ex = [int(e.pos[0] * nf / n) for e in sc["emitters"]]
    ez = [int(e.pos[2] * nf / n) for e in sc["emitters"]]
    ey = int(sc["emitters"][0].pos[1] * nf / n)
    fy, fx = ("f", 5, 1), ("f", 17, 0)
    ffy, ffx = ("ff", (1, ez[0], ey + 1, ex[0])), ("ff", (0, ez[1], ey + 1, ex[1]))
    forces = np.zeros((nsteps, 3), np.float32)
    field = np.zeros((3, nf, nf, nf), np.float32)
    gf, gfield = adjoint(forces, field)
    ffmax = ("ff", tuple(int(i) for i in np.unravel_index(np.argmax(np.abs(gfield)), gfield.shape)))
    check(forces, field, gf, gfield, [fy, ffy, ffmax])
    rng = np.random.default_rng(11)
    forces2 = (1e-2 * rng.standard_normal(forces.shape)).astype(np.float32)
    field2 = (1e-2 * rng.standard_normal(field.shape)).astype(np.float32)
    gf2, gfield2 = adjoint(forces2, field2)
    check(forces2, field2, gf2, gfield2, [fy, fx, ffy, ffx, ffmax])


# ------------------------------------------------ owner-computes scatter-adds
def _stage_grads(dim, n, nch, enc, mask, deterministic, seed=3, state_scale=1.0):
    """Adjoint of one step of the given stages for a random output seed: the
    gradients of every input field and of the control force."""
    from smokesim_b200.adjoint import Rollout
    import torch
    desc, em, ob, f, p, g = _setup(dim, n, nch, enc, seed, mask, state_scale=state_scale)
    rng = np.random.default_rng(seed + 100)
    outs = VEL[:dim] + [abi.FIELD_DENSITY, abi.FIELD_TEMPERATURE]
    ybar = {k: rng.standard_normal(abi.field_count(dim, n, k, nch)).astype(np.float32) for k in outs}
    ro = Rollout(g, 1, deterministic=deterministic)
    force = np.array([(0.3, -0.2, 0.1)[:dim] + (0.0,) * (3 - dim)], np.float32)
    ro.forward(p, force)
    dev = {k: torch.from_numpy(v).cuda() for k, v in ybar.items()}
    torch.cuda.synchronize()
    gf = ro.backward(p, grad_density=dev[abi.FIELD_DENSITY].data_ptr(),
                     grad_temperature=dev[abi.FIELD_TEMPERATURE].data_ptr(),
                     grad_velocity=[dev[k].data_ptr() for k in VEL[:dim]])
    out = {k: ro.grad(k).copy() for k in _fields(dim)}
    out["force"] = np.asarray(gf, np.float32).copy()
    ro.close()
    g.close()
    return out


OWNER_STAGES = [
    ("advect", abi.STAGE_ADVECT_VELOCITIES),
    ("advect_buoyancy", abi.STAGE_ADVECT_VELOCITIES | abi.STAGE_APPLY_BUOYANCY),
    ("buoyancy", abi.STAGE_APPLY_BUOYANCY),
    ("smoke", abi.STAGE_ADVECT_SMOKE),
    ("full", abi.STAGE_ALL),
]


@pytest.mark.parametrize("gname,dim,n,nch,enc", GRIDS)
@pytest.mark.parametrize("stage,mask", OWNER_STAGES)
@pytest.mark.parametrize("scale", [1.0, 4.0])
def test_owner_computes_matches_atomic(gname, dim, n, nch, enc, stage, mask, scale):
    """The owner-computes scatter-adds give the atomic variant's gradients up
    to summation order, and bitwise the same gradients run to run.  scale 4
    multiplies the random velocities (back-traces several cells long, so the
    inverse-footprint boxes are wide)."""
    a = _stage_grads(dim, n, nch, enc, mask, False, state_scale=scale)
    b = _stage_grads(dim, n, nch, enc, mask, True, state_scale=scale)
    c = _stage_grads(dim, n, nch, enc, mask, True, state_scale=scale)
    for k in a:
        assert b[k].tobytes() == c[k].tobytes(), k
        tol = 1e-5 * max(float(np.abs(a[k]).max()), 1e-30)
        assert np.allclose(b[k], a[k], rtol=1e-5, atol=tol), (k, float(np.abs(b[k] - a[k]).max()), tol)


def test_owner_computes_stage_matches_fd():
    """Full step, owner-computes scatters, against FP64 central differences."""
    _directional(3, (16, 14, 12), 1, 1, abi.STAGE_ALL, seed=3, force=(0.3, -0.2, 0.1), deterministic=True)


def test_rollout_deterministic_bitwise():
    """A 32^3 rollout of 8 steps (checkpoint every 3) with per-step forces and
    a 4^3 control force field: two reverse passes with the owner-computes
    scatters give bitwise-identical gradients of the initial velocity, smoke,
    forces and force field; the atomic variant agrees with them to rounding."""
    from smokesim_b200 import Sim
    from smokesim_b200.adjoint import Rollout
    import torch
    n, nsteps, nf = 32, 8, 4
    sc = scene.rollout64(seed=4, n=n)
    p = scene.workload_params(ref_quirks=0, n_vcycles=4)
    rng = np.random.default_rng(5)
    forces = (rng.standard_normal((nsteps, 3)) * 0.2).astype(np.float32)
    field = (rng.standard_normal((3, nf, nf, nf)) * 0.3).astype(np.float32)

    def run(det):
        g = Sim(sc["desc"])
        scene.apply(g, sc)
        g.set_force_field(field)
        ro = Rollout(g, nsteps, 3, deterministic=det)
        ro.forward(p, forces)
        rho = torch.from_numpy(g.get_field(abi.FIELD_DENSITY).ravel()).cuda()
        gd = (2 * (rho - 0.05)).contiguous()
        torch.cuda.synchronize()
        gf = ro.backward(p, grad_density=gd.data_ptr())
        out = {k: ro.grad(k).copy() for k in VEL + [abi.FIELD_DENSITY, abi.FIELD_TEMPERATURE]}
        out["force"] = np.asarray(gf, np.float32).copy()
        out["field"] = ro.force_field_grad(nf).copy()
        ro.close()
        g.close()
        return out

    d1, d2, at = run(True), run(True), run(False)
    for k in d1:
        assert d1[k].tobytes() == d2[k].tobytes(), k
        scale = max(float(np.abs(at[k]).max()), 1e-30)
        assert np.allclose(d1[k], at[k], rtol=1e-3, atol=1e-5 * scale), (k, float(np.abs(d1[k] - at[k]).max()), scale)


@pytest.mark.parametrize("prec", [abi.PREC_FP32, abi.PREC_MIXED])
def test_pressure_store_same_gradients(prec):
    """ss_adjoint_set_pressure_store: the reverse pass recomputes each
    segment with the pressures the forward pass stored instead of solving
    again.  With owner-computes scatters the gradients are bitwise those of
    the plain recomputation (32^3, 9 steps, checkpoint every 3, FP32 or mixed
    projection - whose checkpoints keep the FP64 warm-start pressure)."""
    from smokesim_b200 import Sim
    from smokesim_b200.adjoint import Rollout
    import torch
    n, nsteps = 32, 9
    sc = scene.rollout64(seed=6, n=n)
    p = scene.workload_params(ref_quirks=0, n_vcycles=4, precision=prec)
    forces = (np.random.default_rng(7).standard_normal((nsteps, 3)) * 0.2).astype(np.float32)

    def run(store):
        g = Sim(sc["desc"])
        scene.apply(g, sc)
        ro = Rollout(g, nsteps, 3, deterministic=True, store_pressure=store)
        ro.forward(p, forces)
        rho = torch.from_numpy(g.get_field(abi.FIELD_DENSITY).ravel()).cuda()
        gd = (2 * (rho - 0.05)).contiguous()
        torch.cuda.synchronize()
        gf = ro.backward(p, grad_density=gd.data_ptr())
        out = {k: ro.grad(k).copy() for k in VEL + [abi.FIELD_DENSITY, abi.FIELD_TEMPERATURE]}
        out["force"] = np.asarray(gf, np.float32).copy()
        info = ro.info()
        ro.close()
        g.close()
        return out, info

    (a, ia), (b, ib) = run(False), run(True)
    for k in a:
        assert a[k].tobytes() == b[k].tobytes(), k
    assert ib["kernel_launches"] < ia["kernel_launches"]


def test_coarse_response_matches_sweeps(monkeypatch):
    """The bottom solve's adjoint applies the coarsest level's sweeps as one
    product with their response matrix (default); transposing them sweep by
    sweep (SMOKESIM_ADJ_COARSE_SWEEPS=1) gives the same gradients to
    rounding (8-step 32^3 rollout, 4 V-cycles a step, forces)."""
    from smokesim_b200 import Sim
    from smokesim_b200.adjoint import Rollout
    import torch
    n, nsteps = 32, 8
    sc = scene.rollout64(seed=6, n=n)
    p = scene.workload_params(ref_quirks=0, n_vcycles=4)
    forces = (np.random.default_rng(7).standard_normal((nsteps, 3)) * 0.2).astype(np.float32)

    def run(sweeps):
        if sweeps:
            monkeypatch.setenv("SMOKESIM_ADJ_COARSE_SWEEPS", "1")
        else:
            monkeypatch.delenv("SMOKESIM_ADJ_COARSE_SWEEPS", raising=False)
        g = Sim(sc["desc"])
        scene.apply(g, sc)
        ro = Rollout(g, nsteps, 4)
        ro.forward(p, forces)
        rho = torch.from_numpy(g.get_field(abi.FIELD_DENSITY).ravel()).cuda()
        gd = (2 * (rho - 0.05)).contiguous()
        torch.cuda.synchronize()
        gf = ro.backward(p, grad_density=gd.data_ptr())
        out = {k: ro.grad(k).copy() for k in VEL + [abi.FIELD_DENSITY, abi.FIELD_TEMPERATURE, abi.FIELD_PRESSURE]}
        out["force"] = np.asarray(gf, np.float32).copy()
        info = ro.info()
        ro.close()
        g.close()
        return out, info

    (a, ia), (b, ib) = run(False), run(True)
    assert ia["workspace_bytes"] > ib["workspace_bytes"]   # the matrix was allocated
    # the warm-start pressure's gradient is tiny (the V-cycles damp the initial
    # guess), so rounding is measured against the largest state gradient
    scale = max(float(np.abs(b[k]).max()) for k in b if k != "force")
    for k in a:
        s_k = max(float(np.abs(b[k]).max()), 1e-30) if k == "force" else scale
        assert np.allclose(a[k], b[k], rtol=1e-4, atol=1e-5 * s_k), (k, float(np.abs(a[k] - b[k]).max()), s_k)
