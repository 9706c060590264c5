"""GPU checks of the derivative entry points (FP64): the gravity Jacobian against central
differences of the gravity kernel and of the CPU oracle, the forward variational STM against
central finite differences of the propagation (h = 1e-3 m, 1e-6 m/s; 1e-5 relative), the adjoint
(vector-Jacobian product, checkpointed every 64 steps) against the STM, and the adjoint gradient of
the closest-approach miss distance against finite differences, through torch.autograd wrappers."""
import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu

START = (2024, 1, 1, 0, 0, 0.0)
# Central-difference steps (m, m/s). At the differentiation configuration's steps (1e-3 m,
# 1e-6 m/s) the difference quotient of an FP64 propagation is limited by its rounding noise: about
# 1e-4 relative after 24 h of LEO (the two perturbed runs round differently; measured 1.8e-4).
# The resolved steps (1 m, 1e-3 m/s) keep the truncation error below 1e-7 and the noise below
# 1e-8, so the 1e-5 bound is asserted against them; the configuration's steps are checked at
# their noise level.
H_R, H_V = 1.0, 1e-3
H_R_CFG, H_V_CFG = 1e-3, 1e-6


@pytest.fixture(scope="module")
def ctx():
    import opengpop_b200 as G
    c = G.Context(precision=G.FP64)
    yield c
    c.close()


def _point_mass_jac(r, gm):
    rn = np.linalg.norm(r, axis=1)
    rh = r / rn[:, None]
    return -gm / rn[:, None, None] ** 3 * (np.eye(3)[None] - 3 * rh[:, :, None] * rh[:, None, :])


def _jac(ctx, r, frame=None):
    from gpu_util import dev, host, zeros
    J = zeros(r.shape[0], 3, 3)
    a = zeros(r.shape[0], 3)
    ctx.gravity_jacobian(dev(r), J, None if frame is None else dev(frame), acc=a)
    return host(J), host(a)


def _grav(ctx, r, frame=None):
    from gpu_util import dev, host, zeros
    a = zeros(r.shape[0], 3)
    ctx.gravity(dev(r), a, None if frame is None else dev(frame), precision=0)
    return host(a)


def _fd_jac(fn, r, h):
    cols = []
    for j in range(3):
        d = np.zeros(3)
        d[j] = h
        cols.append((fn(r + d) - fn(r - d)) / (2 * h))
    return np.stack(cols, axis=2)  # [n, i, j] = d a_i / d r_j


@pytest.mark.parametrize("framed", [False, True])
def test_jacobian_matches_fd_of_gravity(ctx, oracle_data, framed):
    from opengpop_b200 import orbits
    r, _ = orbits.mixed_population(512, seed=21)
    frame = None
    if framed:
        m, _ = O.frame_matrices(oracle_data, START, 30.0, 1, before=0)
        frame = m[0]
    J, a = _jac(ctx, r, frame)
    assert np.abs(a - _grav(ctx, r, frame)).max() <= 1e-12 * np.abs(a).max()
    sym = np.abs(J - np.transpose(J, (0, 2, 1))).max(axis=(1, 2)) / np.abs(J).max(axis=(1, 2))
    assert sym.max() < 1e-11
    fd = _fd_jac(lambda x: _grav(ctx, x, frame), r, 10.0)
    pm = _point_mass_jac(r, oracle_data.gm)
    # whole Jacobian, and the harmonic part alone (point mass removed) at a looser bound
    err = np.abs(J - fd).max(axis=(1, 2)) / np.abs(J).max(axis=(1, 2))
    assert err.max() < 1e-7
    res = np.abs((J - pm) - (fd - pm)).max(axis=(1, 2)) / np.abs(J - pm).max(axis=(1, 2))
    assert res.max() < 1e-4


def test_jacobian_matches_fd_of_oracle(ctx, oracle_data):
    # independent gravity (the reference's P-bar triangle restated on the CPU)
    from opengpop_b200 import orbits
    r, _ = orbits.mixed_population(64, seed=22)
    J, _ = _jac(ctx, r)
    fd = _fd_jac(lambda x: O.gravity(oracle_data, x), r, 10.0)
    pm = _point_mass_jac(r, oracle_data.gm)
    res = np.abs((J - pm) - (fd - pm)).max(axis=(1, 2)) / np.abs(J - pm).max(axis=(1, 2))
    assert res.max() < 1e-4


def _fd_stm(ctx, steps, r, v, h=30.0, hr=H_R, hv=H_V):
    n = r.shape[0]
    out = np.zeros((n, 6, 6))
    for j in range(6):
        step = hr if j < 3 else hv
        dr = np.zeros((n, 3))
        dv = np.zeros((n, 3))
        (dr if j < 3 else dv)[:, j % 3] = step
        rp, vp = ctx.propagate(START, h, steps, r + dr, v + dv)
        rm, vm = ctx.propagate(START, h, steps, r - dr, v - dv)
        out[:, :3, j] = (rp - rm) / (2 * step)
        out[:, 3:, j] = (vp - vm) / (2 * step)
    return out


@pytest.mark.parametrize("steps", [1, 4, 5, 64, 65, 200])
def test_stm_matches_finite_differences(ctx, steps):
    from opengpop_b200 import orbits
    r, v = orbits.mixed_population(6, seed=23)
    ro, vo, phi = ctx.stm(START, 30.0, steps, r, v)
    r_ref, v_ref = ctx.propagate(START, 30.0, steps, r, v)
    assert np.abs(ro - r_ref).max() < 1e-6 and np.abs(vo - v_ref).max() < 1e-9
    fd = _fd_stm(ctx, steps, r, v)
    err = np.linalg.norm(phi - fd, axis=1) / np.linalg.norm(fd, axis=1)  # per column
    assert err.max() < 1e-5, err.max()


def test_stm_one_day_leo(ctx):
    # the differentiation configuration's duration (24 h at 30 s)
    from opengpop_b200 import orbits
    r, v = orbits.leo(4, seed=30)
    steps = 2880
    _, _, phi = ctx.stm(START, 30.0, steps, r, v)
    fd = _fd_stm(ctx, steps, r, v)
    err = np.linalg.norm(phi - fd, axis=1) / np.linalg.norm(fd, axis=1)
    assert err.max() < 1e-5, err.max()
    fd = _fd_stm(ctx, steps, r, v, hr=H_R_CFG, hv=H_V_CFG)
    err = np.linalg.norm(phi - fd, axis=1) / np.linalg.norm(fd, axis=1)
    assert err.max() < 1e-3, err.max()  # rounding-limited difference quotient


def test_stm_zero_steps_is_identity(ctx):
    from opengpop_b200 import orbits
    r, v = orbits.leo(3, seed=24)
    ro, vo, phi = ctx.stm(START, 30.0, 0, r, v)
    assert np.array_equal(ro, r) and np.array_equal(phi, np.broadcast_to(np.eye(6), (3, 6, 6)))


@pytest.mark.parametrize("steps", [3, 64, 130, 200])
def test_adjoint_matches_stm(ctx, steps):
    # the reverse sweep (checkpoints every 64 steps) and the forward tangents differentiate the
    # same discrete map: phi^T (r_bar, v_bar) == vjp(r_bar, v_bar)
    from opengpop_b200 import orbits
    r, v = orbits.mixed_population(5, seed=25)
    rng = np.random.default_rng(26)
    rb = rng.normal(size=(5, 3))
    vb = rng.normal(size=(5, 3)) * 1e3
    _, _, phi = ctx.stm(START, 30.0, steps, r, v)
    gr, gv = ctx.propagate_vjp(START, 30.0, steps, r, v, rb, vb)
    ref = np.einsum("nij,ni->nj", phi, np.concatenate([rb, vb], axis=1))
    got = np.concatenate([gr, gv], axis=1)
    err = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert err.max() < 1e-9


def test_autograd_propagate(ctx):
    torch = pytest.importorskip("torch")
    from autograd_fns import Propagate
    from opengpop_b200 import orbits
    r, v = orbits.leo(3, seed=27)
    steps = 90
    r0 = torch.tensor(r, requires_grad=True)
    v0 = torch.tensor(v, requires_grad=True)
    w = torch.tensor(np.random.default_rng(28).normal(size=(3, 3)))
    rN, vN = Propagate.apply(r0, v0, ctx, START, 30.0, steps)
    loss = (rN * w).sum() + 100.0 * (vN * w).sum()
    loss.backward()
    # central differences of the same scalar
    def f(rr, vv):
        a, b = ctx.propagate(START, 30.0, steps, rr, vv)
        return float((a * w.numpy()).sum() + 100.0 * (b * w.numpy()).sum())
    for k, (x, g, step) in enumerate([(r, r0.grad.numpy(), H_R), (v, v0.grad.numpy(), H_V)]):
        fd = np.zeros_like(x)
        for i in range(x.shape[0]):
            for j in range(3):
                d = np.zeros_like(x)
                d[i, j] = step
                fd[i, j] = ((f(r + d, v) - f(r - d, v)) if k == 0 else (f(r, v + d) - f(r, v - d))) / (2 * step)
        assert np.linalg.norm(g - fd) / np.linalg.norm(fd) < 1e-5


def _pairs_scenario():
    from opengpop_b200 import orbits
    r, v = orbits.leo(8, seed=29)
    # object 8 starts 180 m from object 0 and moves away along the offset: over a few minutes its
    # distance grows monotonically, so its minimum is the first sample
    off = np.array([150.0, -80.0, 60.0])
    r = np.vstack([r, r[0] + off])
    v = np.vstack([v, v[0] + 0.5 * off / np.linalg.norm(off)])
    pairs = np.array([[0, 1], [2, 3], [4, 5], [6, 7], [1, 6]], dtype=np.int32)
    return r, v, pairs


def _check_fd(ctx, r, v, pairs, steps, grad):
    for p, (a, b) in enumerate(pairs):
        for side, o in enumerate((a, b)):
            for blk, step in ((0, H_R), (1, H_V)):
                fd = np.zeros(3)
                for j in range(3):
                    dr = np.zeros_like(r)
                    dv = np.zeros_like(v)
                    (dr if blk == 0 else dv)[o, j] = step
                    mp = ctx.miss_gradient(START, 30.0, steps, r + dr, v + dv, pairs[p:p + 1])[1][0]
                    mm = ctx.miss_gradient(START, 30.0, steps, r - dr, v - dv, pairs[p:p + 1])[1][0]
                    fd[j] = (mp - mm) / (2 * step)
                g = grad[p, 6 * side + 3 * blk:6 * side + 3 * blk + 3]
                assert np.linalg.norm(g - fd) <= 1e-5 * np.linalg.norm(fd) + 1e-9, (p, side, blk, g, fd)


def test_miss_gradient_matches_finite_differences(ctx):
    r, v, pairs = _pairs_scenario()
    steps = 120
    tca, miss, grad = ctx.miss_gradient(START, 30.0, steps, r, v, pairs)
    assert np.all(np.isfinite(miss)) and np.all(miss > 0)
    assert np.all((tca >= 0) & (tca <= steps * 30.0))
    _check_fd(ctx, r, v, pairs, steps, grad)


def test_miss_gradient_first_sample_minimum(ctx):
    # a minimum on the first sample is not refined (device.cu:100-110): TCA 0, the sampled distance
    r, v, _ = _pairs_scenario()
    pairs = np.array([[0, 8]], np.int32)
    steps = 10
    tca, miss, grad = ctx.miss_gradient(START, 30.0, steps, r, v, pairs)
    rt, _ = ctx.propagate(START, 30.0, 1, r, v)
    assert tca[0] == 0.0 and abs(miss[0] - np.linalg.norm(rt[0] - rt[8])) < 1e-9
    _check_fd(ctx, r, v, pairs, steps, grad)


def test_miss_matches_pairwise_closest_approach(ctx):
    # the pair-list kernel reproduces the set-partitioned closest approach of the same objects
    r, v, pairs = _pairs_scenario()
    steps = 120
    tca, miss, _ = ctx.miss_gradient(START, 30.0, steps, r, v, pairs[:2])
    sel = np.array([0, 1, 2, 3])
    ca = ctx.closest_approach(START, 30.0, r[sel], v[sel], np.array([0, 1, 2, 3], np.uint32))
    ca.propagate(steps)
    rec = {(int(x.object_index1), int(x.object_index2)): x for x in ca.find()}
    ca.close()
    for p, (a, b) in enumerate(pairs[:2]):
        x = rec[(a, b)]
        assert abs(x.distance - miss[p]) < 1e-6 and abs(x.time - tca[p]) < 1e-6


def test_autograd_miss_distance(ctx):
    torch = pytest.importorskip("torch")
    from autograd_fns import MissDistance
    r, v, pairs = _pairs_scenario()
    steps = 120
    r0 = torch.tensor(r, requires_grad=True)
    v0 = torch.tensor(v, requires_grad=True)
    miss = MissDistance.apply(r0, v0, ctx, START, 30.0, steps, pairs)
    w = torch.linspace(0.5, 1.5, len(pairs), dtype=torch.float64)
    (miss * w).sum().backward()
    _, _, grad = ctx.miss_gradient(START, 30.0, steps, r, v, pairs)
    exp_r = np.zeros_like(r)
    for p, (a, b) in enumerate(pairs):
        exp_r[a] += w[p].item() * grad[p, 0:3]
        exp_r[b] += w[p].item() * grad[p, 6:9]
    assert np.allclose(r0.grad.numpy(), exp_r, rtol=1e-12, atol=0)


def test_invalid_pairs_rejected(ctx):
    import opengpop_b200 as G
    r, v, _ = _pairs_scenario()
    for bad in ([[0, 0]], [[0, 99]], [[-1, 2]]):
        with pytest.raises(G.GpopError):
            ctx.miss_gradient(START, 30.0, 10, r, v, np.array(bad, np.int32))


def test_miss_gradient_at_configuration_steps_long_double_fd(ctx, oracle_data):
    """The differentiation configuration (24 h, 30 s steps, 70x70, FP64) on three of its seeded
    pairs: the adjoint gradient of each miss distance against central differences at the
    configuration's steps (1e-3 m, 1e-6 m/s), taken in long double by the oracle so that the
    difference quotient is not limited by double rounding noise. Bound 1e-5 relative per
    (object, position | velocity) block."""
    from opengpop_b200 import orbits
    r, v, pairs = orbits.conjunction_pairs(10000, 20240101)
    pairs = pairs[:3]
    objs = np.unique(pairs)
    remap = {int(o): i for i, o in enumerate(objs)}
    sub = np.array([[remap[int(a)], remap[int(b)]] for a, b in pairs], np.int32)
    steps = 2880
    tca, miss, grad = ctx.miss_gradient(START, 30.0, steps, r[objs], v[objs], sub)
    a, b = pairs[:, 0], pairs[:, 1]
    m_ld, t_ld, fd = O.miss_fd_ld(oracle_data, START, 30.0, steps, r[a], v[a], r[b], v[b],
                                  H_R_CFG, H_V_CFG)
    assert np.allclose(miss, m_ld, rtol=1e-9, atol=1e-4) and np.allclose(tca, t_ld, rtol=0, atol=1e-4)
    worst = 0.0
    for p in range(len(pairs)):
        for blk in range(4):
            g = grad[p, 3 * blk:3 * blk + 3]
            f = fd[p, 3 * blk:3 * blk + 3]
            err = np.linalg.norm(g - f) / np.linalg.norm(f)
            worst = max(worst, err)
            assert err <= 1e-5, (p, blk, g, f)
    print("\nadjoint vs long double central differences (1e-3 m, 1e-6 m/s), 24 h: max relative "
          "error %.2e" % worst)
