"""Known-answer tests of the CPU oracle (the restatement of the reference's
time step).  The reference ships no tests or fixtures; these follow from its
formulas: interpolateF (2M:649-660) is exact on quadratics, the ISLBM weights
on an integer-spaced grid reduce streaming to plain pull streaming bit for bit,
and the rest state without buoyancy is a fixed point."""
import numpy as np
import pytest


def test_interpolateF_exact_on_quadratics(ora):
    rng = np.random.default_rng(1)
    for _ in range(200):
        x = np.sort(rng.uniform(0, 10, 3))
        if np.min(np.diff(x)) < 1e-3:
            continue
        a, b, c = rng.normal(size=3)
        q = lambda t: a * t * t + b * t + c  # noqa: E731
        t = rng.uniform(x[0], x[2])
        got = ora.interpolateF(x[0], x[1], x[2], t, q(x[0]), q(x[1]), q(x[2]))
        assert got == pytest.approx(q(t), rel=1e-11, abs=1e-11)


def test_interpolateF_zero_shift_is_identity(ora):
    # an axis with no lattice shift: weights (0, 1, 0) exactly
    rng = np.random.default_rng(2)
    for _ in range(50):
        x = np.sort(rng.uniform(0, 10, 3))
        f = rng.normal(size=3)
        for order in ((0, 1, 2), (1, 0, 2), (1, 2, 0)):
            xs = x[list(order)]
            assert ora.interpolateF(xs[0], xs[1], xs[2], xs[1], f[0], f[1], f[2]) == f[1]


def _uniform_coords(n):
    # nodes at i - 1/2 (the reference's half-cell shift), dt = 1
    return np.arange(n + 2, dtype=np.float64) - 0.5


@pytest.mark.parametrize("dim", [2, 3])
def test_uniform_grid_streaming_is_pull_streaming(ora, dim):
    n = 9
    c = _uniform_coords(n)
    c[0], c[-1] = 0.0, float(n)
    o = ora.Oracle(dim, n, n, n if dim == 3 else 1, x=c, y=c, z=c if dim == 3 else None, dt=1.0,
                   length_LB=float(n + 1), Ra=1e4)
    o.step(3)
    fpost = o.pops("f_post")
    f = o.pops("f")
    Q = o.Q
    ex = [0, 1, 0, -1, 0, 1, -1, -1, 1] if dim == 2 else [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0]
    ey = [0, 0, 1, 0, -1, 1, 1, -1, -1] if dim == 2 else [0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1]
    ez = [0] * 9 if dim == 2 else [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1]
    # interior nodes: f_a(x) = f_post_a(x - e_a), bit for bit
    sl = (slice(1, -1),) * dim
    for a in range(1, Q):
        if dim == 2:
            shifted = np.roll(np.roll(fpost[..., a], ey[a], axis=0), ex[a], axis=1)
        else:
            shifted = np.roll(np.roll(np.roll(fpost[..., a], ez[a], axis=0), ey[a], axis=1), ex[a], axis=2)
        assert np.array_equal(f[sl + (a,)], shifted[sl]), f"direction {a}"


@pytest.mark.parametrize("dim", [2, 3])
def test_rest_state_without_buoyancy_is_fixed_point(ora, dim):
    n = 10
    o = ora.Oracle(dim, n, n, n if dim == 3 else 1, grid="tanh", stretch=1.5, Ra=1e4, Thot=1.0, Tcold=0.0)
    shape = o.shape
    one, zero = np.ones(shape), np.zeros(shape)
    # T = 0 everywhere gives no buoyancy; only the hot wall feeds heat in,
    # which does not move the flow within one step's ordering, so test the
    # flow populations only on the first step
    o.set_macro(one, zero, zero, zero if dim == 3 else None, zero)
    o.step(1)
    u, v = o.field("u"), o.field("v")
    assert np.abs(u).max() < 1e-15 and np.abs(v).max() < 1e-15
    assert np.abs(o.field("rho") - 1.0).max() < 1e-14


def test_parameters_reference_values(ora):
    # derived values quoted for the reference's own 2D case (513^2, Ra = 1e5):
    # L_LB = 3560.08, tau_f = 2.1426, sigma_k = 0.279 (rounded)
    x, y, z, dx0, L, dt = ora.mesh("erf", 3.2, 513, 513)
    o = ora.Oracle(2, 513, 513, x=x, y=y, dt=dt, length_LB=L, Ra=float(np.float32(1e5)))
    p = o.params()
    assert L == pytest.approx(3560.08, abs=0.01)
    assert p["tauf"] == pytest.approx(2.1426, abs=1e-4)
    assert p["sig_k"] == pytest.approx(0.279, abs=1e-3)
    # node 1 sits half a lattice unit from the wall at 0; the wall at the far end is at L - 1
    assert x[1] == pytest.approx(0.5, abs=1e-9)
    assert x[513] + 0.5 == pytest.approx(L - 1.0, abs=1e-8)


def test_nusselt_of_linear_conduction_profile(ora):
    # T linear in position between the walls (w_lo = x1 - dt/2 at Thot,
    # w_hi = xn + dt/2 at Tcold): the one-sided quadratic is exact, so
    # Nu = (L_LB - 1) / (w_hi - w_lo) at both walls
    for dim, n in ((2, 33), (3, 12)):
        o = ora.Oracle(dim, n, n, n if dim == 3 else 1, grid="erf", stretch=3.2, Ra=1e4)
        ax = o.coords("x" if dim == 2 else "y")
        lo, hi = ax[1] - 0.5 * o.dt, ax[n] + 0.5 * o.dt
        prof = (hi - ax[1:n + 1]) / (hi - lo)
        shape = o.shape
        T = np.broadcast_to(prof if dim == 2 else prof[:, None], shape).copy()
        one, zero = np.ones(shape), np.zeros(shape)
        o.set_macro(one, zero, zero, zero if dim == 3 else None, T)
        nh, nc = o.nusselt()
        expect = (o.length_LB - 1.0) / (hi - lo)
        assert nh == pytest.approx(expect, rel=1e-12)
        assert nc == pytest.approx(expect, rel=1e-12)
        mass, energy = o.sums()
        vol = (hi - lo) ** dim
        assert mass == pytest.approx(vol, rel=1e-12)
        assert energy == pytest.approx(0.5 * vol, rel=1e-9)


def test_slope3_exact_on_quadratics(ora):
    rng = np.random.default_rng(5)
    for _ in range(200):
        x = rng.uniform(0, 10, 3)
        if min(abs(x[0] - x[1]), abs(x[0] - x[2]), abs(x[1] - x[2])) < 1e-2:
            continue
        a, b, c = rng.normal(size=3)
        q = lambda t: a * t * t + b * t + c  # noqa: E731
        got = ora.slope3(x[0], q(x[0]), x[1], q(x[1]), x[2], q(x[2]))
        assert got == pytest.approx(2 * a * x[1] + b, rel=1e-9, abs=1e-9)


@pytest.mark.parametrize("dim", [2, 3])
def test_warm_start_non_equilibrium_moments(ora, dim):
    # Linear fields have exact stencil gradients.  The added part must carry
    # no mass and no momentum, its second moment must be the Chapman-Enskog
    # stress -tau_f dt rho / 3 (du_a/dx_b + du_b/dx_a), and its thermal first
    # moment the diffusive flux -(dt / sig_k) cs_T^2 grad T.
    n = 9
    o = ora.Oracle(dim, n, n + 2, n + 1 if dim == 3 else 1, grid="tanh", stretch=1.5, Ra=1e4)
    shape = o.shape
    ax = [o.coords(a) for a in ("x", "y", "z")[:dim]]
    grids = np.meshgrid(*[c[1:-1] for c in ax[::-1]], indexing="ij")[::-1]  # x, y(, z) arrays of `shape`
    rng = np.random.default_rng(3)
    G = rng.normal(scale=1e-4, size=(dim, dim))  # G[a, b] = d u_b / d x_a
    gT = rng.normal(scale=1e-3, size=dim)
    vel = [sum(G[a, b] * grids[a] for a in range(dim)) for b in range(dim)]
    T = 0.5 + sum(gT[a] * grids[a] for a in range(dim))
    rho = np.full(shape, 1.02)
    w = vel[2] if dim == 3 else None
    o.set_macro(rho, vel[0], vel[1], w, T)
    f0, g0 = o.pops("f"), o.pops("g")
    o.set_macro_neq(rho, vel[0], vel[1], w, T)
    df, dg = o.pops("f") - f0, o.pops("g") - g0
    p = o.params()
    ex = np.array([[0, 1, 0, -1, 0, 1, -1, -1, 1], [0, 0, 1, 0, -1, 1, 1, -1, -1]]) if dim == 2 else np.array([
        [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0],
        [0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1],
        [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1]])
    QT = 5 if dim == 2 else 7
    assert np.abs(df.sum(-1)).max() < 1e-15
    for a in range(dim):
        assert np.abs((df * ex[a]).sum(-1)).max() < 1e-15
        for b in range(dim):
            pi = (df * ex[a] * ex[b]).sum(-1)
            expect = -p["tauf"] * o.dt * 1.02 / 3.0 * (G[a, b] + G[b, a])
            assert np.abs(pi - expect).max() <= 1e-10 * max(abs(expect), 1e-9), (a, b)
    cs2T = 0.25 if dim == 2 else 1.0 / 6.0
    assert np.abs(dg.sum(-1)).max() < 1e-15
    for a in range(dim):
        flux = (dg * ex[a][:QT]).sum(-1)
        expect = -(o.dt / p["sig_k"]) * cs2T * gT[a]
        assert np.abs(flux - expect).max() <= 1e-10 * abs(expect), a  # cancellation in g - g_eq
