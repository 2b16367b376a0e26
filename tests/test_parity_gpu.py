"""GPU parity: the sm_100a kernels, called through the C ABI, against the CPU
oracle on the same grids and parameters.

exact mode   FP64, the reference's operation order, no contraction: populations
             and macroscopic fields bit-identical to the oracle;
fast mode    FP64 with multiply-add contraction: <= 1e-12 relative in the
             populations after 1000 steps, <= 1e-10 in the average Nusselt
             number (the drop-in tolerance);
f32          reduced storage: errors against the FP64 oracle stay within the
             bounds written in each test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def pair(pkg, ora, dim, nx, ny, nz=1, grid="erf", stretch=3.2, Ra=1e5, Pr=0.71, mode="fast", storage="f64",
         kernel="auto", nblocks=0):
    cav = pkg.Cavity(dim, nx, ny, nz, Ra=Ra, Pr=Pr, grid=grid, stretch=stretch, mode=mode, storage=storage,
                     kernel=kernel, nblocks=nblocks)
    o = ora.Oracle(dim, nx, ny, nz, x=cav.mesh.x, y=cav.mesh.y, z=cav.mesh.z, dt=cav.mesh.dt,
                   length_LB=cav.mesh.length_LB, Ra=Ra, Pr=Pr)
    cav.initial()
    return cav, o


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


FIELDS2 = ("rho", "u", "v", "T")
FIELDS3 = ("rho", "u", "v", "w", "T")


@pytest.mark.parametrize("kernel", ["direct", "march"])
@pytest.mark.parametrize("case", [
    dict(dim=2, nx=32, ny=32, grid="erf", stretch=3.2, steps=150),
    dict(dim=2, nx=40, ny=24, grid="tanh", stretch=1.5, steps=120),
    dict(dim=2, nx=150, ny=20, grid="tanh", stretch=1.5, steps=40),
    dict(dim=3, nx=14, ny=12, nz=10, grid="erf", stretch=3.2, steps=40),
    dict(dim=3, nx=16, ny=16, nz=16, grid="tanh", stretch=1.5, steps=30),
    dict(dim=3, nx=40, ny=18, nz=7, grid="tanh", stretch=1.5, steps=25),
])
def test_exact_mode_bit_identical(pkg, ora, case, kernel):
    c = dict(case)
    steps = c.pop("steps")
    cav, o = pair(pkg, ora, mode="exact", kernel=kernel, **c)
    assert cav.kernel == kernel
    cav.step(steps)
    o.step(steps)
    m = cav.macro()
    for k in (FIELDS2 if c["dim"] == 2 else FIELDS3):
        assert np.array_equal(m[k], o.field(k)), f"{k}: max diff {np.abs(m[k] - o.field(k)).max():.3e}"
    f, g = cav.populations()
    assert np.array_equal(f, o.pops("f"))
    assert np.array_equal(g, o.pops("g"))
    cav.close()


@pytest.mark.parametrize("kernel", ["direct", "march"])
@pytest.mark.parametrize("case", [
    dict(dim=2, nx=48, ny=48, grid="tanh", stretch=1.5, Ra=1e4),
    dict(dim=2, nx=33, ny=33, grid="erf", stretch=3.2, Ra=1e5),
    dict(dim=3, nx=20, ny=20, nz=20, grid="tanh", stretch=1.5, Ra=1e5),
])
def test_fast_fp64_within_1e12_after_1000_steps(pkg, ora, case, kernel):
    cav, o = pair(pkg, ora, mode="fast", kernel=kernel, **case)
    cav.step(1000)
    o.step(1000)
    f, g = cav.populations()
    assert rel_err(f, o.pops("f")) <= 1e-12
    assert rel_err(g, o.pops("g")) <= 1e-12
    nh, nc = cav.nusselt()
    onh, onc = o.nusselt()
    assert abs(nh - onh) <= 1e-10 * abs(onh)
    assert abs(nc - onc) <= 1e-10 * abs(onc)
    cav.close()


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_check_nusselt_sums_match_oracle(pkg, ora, mode):
    cav, o = pair(pkg, ora, 2, 36, 36, grid="erf", Ra=1e5, mode=mode)
    tol = 1e-13 if mode == "exact" else 1e-10
    for _ in range(3):
        cav.step(40)
        o.step(40)
        eu, et = cav.check()
        ou, ot = o.check()
        assert eu == pytest.approx(ou, rel=tol) and et == pytest.approx(ot, rel=tol)
    for a, b in zip(cav.nusselt(), o.nusselt()):
        assert a == pytest.approx(b, rel=tol)
    for a, b in zip(cav.sums(), o.sums()):
        assert a == pytest.approx(b, rel=tol)
    assert cav.itc == 120
    cav.close()


def test_check_nusselt_sums_3d(pkg, ora):
    cav, o = pair(pkg, ora, 3, 14, 14, 14, grid="tanh", stretch=1.5, Ra=1e5, mode="exact")
    cav.step(25)
    o.step(25)
    for a, b in zip(cav.check(), o.check()):
        assert a == pytest.approx(b, rel=1e-13)
    for a, b in zip(cav.nusselt(), o.nusselt()):
        assert a == pytest.approx(b, rel=1e-13)
    for a, b in zip(cav.sums(), o.sums()):
        assert a == pytest.approx(b, rel=1e-13)
    cav.close()


@pytest.mark.parametrize("dim", [2, 3])
def test_checkpoint_restart_is_exact(pkg, ora, dim):
    n = (30, 30, 1) if dim == 2 else (12, 12, 12)
    a, _ = pair(pkg, ora, dim, *n, mode="exact")
    b, _ = pair(pkg, ora, dim, *n, mode="exact")
    a.step(37)
    f, g = a.populations()
    mac = a.macro()
    a.step(23)
    b.step(5)  # some other state, then restore the checkpoint
    b.set_populations(f, g)
    b.set_macro(**mac)
    b.step(23)
    ma, mb = a.macro(), b.macro()
    for k in ma:
        assert np.array_equal(ma[k], mb[k]), k
    a.close()
    b.close()


@pytest.mark.parametrize("storage,tol_u,tol_T", [("f32", 5e-4, 3e-5)])
@pytest.mark.parametrize("dim", [2, 3])
def test_reduced_precision_storage(pkg, ora, storage, tol_u, tol_T, dim):
    n = (48, 48, 1) if dim == 2 else (16, 16, 16)
    cav, o = pair(pkg, ora, dim, *n, grid="tanh", stretch=1.5, Ra=1e5, storage=storage)
    cav.step(500)
    o.step(500)
    m = cav.macro()
    umax = max(np.abs(o.field(k)).max() for k in ("u", "v"))
    du = max(np.abs(m[k] - o.field(k)).max() for k in ("u", "v"))
    dT = np.abs(m["T"] - o.field("T")).max()
    print(f"{storage} {dim}D: |du|/umax = {du / umax:.3e}, |dT| = {dT:.3e}")
    assert du / umax <= tol_u
    assert dT <= tol_T
    cav.close()


@pytest.mark.parametrize("dim,shape", [(3, (40, 18, 12)), (2, (300, 30, 1))])
def test_march_grid_sizes_bit_identical(pkg, ora, dim, shape):
    # persistent grids of 1, 3, 7 blocks make every CTA march across several
    # tiles and restart its ring at tile boundaries
    o = None
    for nb in (1, 3, 7, 0):
        cav, o2 = pair(pkg, ora, dim, *shape, grid="tanh", stretch=1.5, mode="exact", kernel="march", nblocks=nb)
        cav.step(12)
        if o is None:
            o = o2
            o.step(12)
        m = cav.macro()
        for k in (FIELDS2 if dim == 2 else FIELDS3):
            assert np.array_equal(m[k], o.field(k)), (nb, k)
        cav.close()


def test_kernel_option_reports_choice(pkg):
    big = pkg.Cavity(3, 64, 64, 64)
    assert big.kernel == "march" and big.get_option(pkg.lbm.OPT_NBLOCKS) > 0
    small = pkg.Cavity(2, 20, 20)
    assert small.kernel == "direct"
    odd = pkg.Cavity(3, 32, 17, 8)  # a last tile row of one y-row: direct-load only
    assert odd.kernel == "direct"
    with pytest.raises(pkg.LBMError) as e:
        odd.set_option(pkg.lbm.OPT_KERNEL, 2)
    assert e.value.status == -8
    for c in (big, small, odd):
        c.close()


def test_step_before_init_is_a_state_error(pkg):
    cav = pkg.Cavity(2, 16, 16)
    with pytest.raises(pkg.LBMError) as e:
        cav.step(1)
    assert e.value.status == -6
    cav.initial()
    cav.step(1)
    cav.close()


def test_init_equilibrium_rest_state(pkg, ora):
    # the rest initial state (rho = 1, u = 0, T = 0) through the
    # equilibrium entry point, against the oracle's set_macro
    cav = pkg.Cavity(2, 40, 40, grid="tanh", stretch=1.5, Ra=1e4, mode="exact")
    o = ora.Oracle(2, 40, 40, x=cav.mesh.x, y=cav.mesh.y, dt=cav.mesh.dt, length_LB=cav.mesh.length_LB, Ra=1e4)
    one, zero = np.ones(cav.shape), np.zeros(cav.shape)
    rng = np.random.default_rng(7)
    T = rng.uniform(-1e-4, 1e-4, cav.shape)
    cav.init_equilibrium(one, zero, zero, None, T)
    o.set_macro(one, zero, zero, None, T)
    cav.step(60)
    o.step(60)
    m = cav.macro()
    for k in FIELDS2:
        assert np.array_equal(m[k], o.field(k)), k
    cav.close()


@pytest.mark.parametrize("dim,n,steps", [(3, 128, 3), (2, 2048, 2)])
def test_full_size_against_oracle(pkg, ora, dim, n, steps):
    # the benchmark sizes (128^3 D3Q19+D3Q7, 2048^2 D2Q9+D2Q5) for a few steps
    ns = (n, n, n) if dim == 3 else (n, n, 1)
    cav, o = pair(pkg, ora, dim, *ns, grid="tanh", stretch=1.5, Ra=1e5, mode="fast")
    cav.step(steps)
    o.step(steps)
    m = cav.macro()
    f, g = cav.populations()
    assert rel_err(f, o.pops("f")) <= 1e-12
    assert rel_err(g, o.pops("g")) <= 1e-12
    # fields against the population scale (velocities are differences of populations)
    fscale = np.abs(o.pops("f")).max()
    for k in (FIELDS2 if dim == 2 else FIELDS3):
        assert np.abs(m[k] - o.field(k)).max() <= 1e-12 * fscale, k
    cav.close()


def test_runs_are_deterministic(pkg):
    out = []
    for _ in range(2):
        cav = pkg.Cavity(3, 64, 64, 64, grid="tanh", stretch=1.5, Ra=1e5)
        cav.initial()
        cav.step(50)
        out.append((cav.macro(), cav.check(), cav.nusselt()))
        cav.close()
    for k in out[0][0]:
        assert np.array_equal(out[0][0][k], out[1][0][k])
    assert out[0][1] == out[1][1] and out[0][2] == out[1][2]


# ---------------------------------------------------------------------------
# against the golden fixtures produced by the reference programs themselves
# ---------------------------------------------------------------------------
import glob as _glob  # noqa: E402
import os as _os  # noqa: E402

_GOLDEN = sorted(_glob.glob(_os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "golden", "ref_*.npz")))


@pytest.mark.parametrize("kernel", ["direct", "march"])
@pytest.mark.parametrize("path", _GOLDEN, ids=[_os.path.basename(p) for p in _GOLDEN])
def test_gpu_matches_reference_fixture(pkg, path, kernel):
    d = dict(np.load(path))
    dim = d["f"].ndim - 1
    shape = d["f"].shape[:-1]
    nz, ny, nx = (shape if dim == 3 else (1,) + shape)
    m = pkg.Mesh(d["x"], d["y"], d.get("z"), 0.0, float(d["length_LB"]), float(d["dt"]))
    for mode in ("exact", "fast"):
        cav = pkg.Cavity(dim, nx, ny, nz, Ra=float(d["Ra"]), Pr=float(d["Pr"]), Ma=float(d["Ma"]), coords=m,
                         mode=mode, kernel=kernel)
        cav.initial()
        cav.step(int(d["itc"]))
        f, g = cav.populations()
        mac = cav.macro()
        if mode == "exact":
            assert np.array_equal(f, d["f"]) and np.array_equal(g, d["g"])
            for k in mac:
                assert np.array_equal(mac[k], d[k]), k
        else:
            assert rel_err(f, d["f"]) <= 1e-12 and rel_err(g, d["g"]) <= 1e-12
        cav.close()


@pytest.mark.parametrize("dim,shape,kernel", [(2, (64, 48, 1), "direct"), (2, (300, 40, 1), "march"),
                                              (3, (40, 18, 12), "march"), (3, (14, 12, 10), "direct")])
def test_graph_replay_is_bit_identical(pkg, dim, shape, kernel):
    out = []
    for graphs in (1, 0):
        c = pkg.Cavity(dim, *shape, grid="tanh", stretch=1.5, mode="exact", kernel=kernel)
        c.set_option(pkg.lbm.OPT_GRAPHS, graphs)
        c.initial()
        for n in (7, 1, 10, 3):
            c.step(n)
        out.append((c.macro(), c.populations()))
        c.close()
    for k in out[0][0]:
        assert np.array_equal(out[0][0][k], out[1][0][k]), k
    assert np.array_equal(out[0][1][0], out[1][1][0]) and np.array_equal(out[0][1][1], out[1][1][1])


@pytest.mark.parametrize("dim,shape", [(2, (300, 40, 1)), (3, (40, 18, 12))])
def test_programmatic_dependent_launch_is_bit_identical(pkg, dim, shape):
    # march steps launched as programmatic dependents (the default) against
    # plain stream order: single steps, graph replays and a run to a criterion
    out = []
    for pdl in (1, 0):
        c = pkg.Cavity(dim, *shape, grid="tanh", stretch=1.5, Ra=1e4, mode="exact", kernel="march")
        assert c.get_option(pkg.lbm.OPT_PDL) == 1
        c.set_option(pkg.lbm.OPT_PDL, pdl)
        assert c.get_option(pkg.lbm.OPT_PDL) == pdl
        c.initial()
        for n in (7, 1, 10, 3):
            c.step(n)
        run = c.run(max_steps=3000, check_every=300, eps=1e-3)
        out.append((c.macro(), c.populations(), run))
        c.close()
    assert out[0][2] == out[1][2]
    for k in out[0][0]:
        assert np.array_equal(out[0][0][k], out[1][0][k]), k
    assert np.array_equal(out[0][1][0], out[1][1][0]) and np.array_equal(out[0][1][1], out[1][1][1])


def test_run_matches_manual_loop(pkg):
    eps = 2e-2
    a = pkg.Cavity(2, 40, 40, Ra=1e4, grid="tanh", stretch=1.5, mode="exact")
    a.initial()
    steps, eu, et = a.run(max_steps=20000, check_every=200, eps=eps)
    b = pkg.Cavity(2, 40, 40, Ra=1e4, grid="tanh", stretch=1.5, mode="exact")
    b.initial()
    n, ref = 0, (100.0, 100.0)
    while (ref[0] > eps or ref[1] > eps) and n < 20000:
        b.step(200)
        n += 200
        ref = b.check()
    assert steps == n and (eu, et) == ref
    assert steps % 200 == 0 and steps < 20000 and eu <= eps and et <= eps
    ma, mb = a.macro(), b.macro()
    for k in ma:
        assert np.array_equal(ma[k], mb[k])
    a.close()
    b.close()


@pytest.mark.parametrize("dim,shape,ce,eps,max_steps,pre", [
    (2, (40, 40, 1), 200, 2e-2, 20000, 0),
    (2, (40, 40, 1), 137, 2e-2, 20000, 55),    # odd period; the first period is partial
    (2, (48, 40, 1), 200, 1e-12, 1500, 0),     # never met: max_steps is not a multiple of the period
    (2, (96, 80, 1), 300, 3e-2, 30000, 0),     # the TMA march kernel
    (3, (20, 16, 12), 100, 5e-2, 6000, 10),
], ids=["2d", "2d-odd-offset", "2d-cap", "2d-march", "3d"])
def test_device_stop_test_matches_host_loop(pkg, dim, shape, ce, eps, max_steps, pre):
    # lbm_run tests the criterion on the device and reads its state once every
    # few checks; iterations, residuals, counter and state equal the
    # reference's loop driven from the host (2M:307-330: step, check every
    # check_every iterations, stop when errorU and errorT are at most eps)
    kern = "march" if shape[0] >= 96 else "auto"
    a = pkg.Cavity(dim, *shape, Ra=1e4, grid="tanh", stretch=1.5, mode="exact", kernel=kern)
    b = pkg.Cavity(dim, *shape, Ra=1e4, grid="tanh", stretch=1.5, mode="exact", kernel=kern)
    for c in (a, b):
        c.initial()
        if pre:
            c.step(pre)
            c.check()
    steps, eu, et = a.run(max_steps=max_steps, check_every=ce, eps=eps)
    done, ref = 0, (100.0, 100.0)
    while (ref[0] > eps or ref[1] > eps) and done < max_steps:
        k = min(ce - b.itc % ce, max_steps - done)
        b.step(k)
        done += k
        if b.itc % ce == 0:
            ref = b.check()
    assert steps == done and (eu, et) == ref
    assert a.itc == b.itc == pre + done
    ma, mb = a.macro(), b.macro()
    for k in ma:
        assert np.array_equal(ma[k], mb[k]), k
    fa, ga = a.populations()
    fb, gb = b.populations()
    assert np.array_equal(fa, fb) and np.array_equal(ga, gb)
    # stepping after the run continues from the same state
    a.step(3)
    b.step(3)
    assert np.array_equal(a.macro()["u"], b.macro()["u"])
    a.close()
    b.close()


def _smooth_fields(shape, dim, seed):
    # smooth random fields: products of low-order sines in the node index
    rng = np.random.default_rng(seed)
    idx = np.meshgrid(*[np.linspace(0, np.pi, s) for s in shape], indexing="ij")
    def one(scale):
        a = rng.uniform(0.5, 2.0, len(shape))
        return scale * np.prod([np.sin(a[k] * idx[k] + rng.uniform()) for k in range(len(shape))], axis=0)
    return 1.0 + one(1e-3), one(2e-2), one(2e-2), (one(2e-2) if dim == 3 else None), 0.5 + one(0.3)


@pytest.mark.parametrize("mode", ["exact", "fast"])
@pytest.mark.parametrize("dim,shape", [(2, (36, 28, 1)), (3, (14, 12, 10))])
def test_init_warm_matches_oracle(pkg, ora, dim, shape, mode):
    # equilibrium + first-order non-equilibrium part, then steps: bit-identical
    # in exact mode, 1e-12 in fast mode
    cav = pkg.Cavity(dim, *shape, grid="tanh", stretch=1.5, Ra=1e5, mode=mode)
    o = ora.Oracle(dim, *shape, x=cav.mesh.x, y=cav.mesh.y, z=cav.mesh.z, dt=cav.mesh.dt,
                   length_LB=cav.mesh.length_LB, Ra=1e5)
    rho, u, v, w, T = _smooth_fields(cav.shape, dim, 11)
    cav.init_warm(rho, u, v, w, T)
    o.set_macro_neq(rho, u, v, w, T)
    f, g = cav.populations()
    if mode == "exact":
        assert np.array_equal(f, o.pops("f")) and np.array_equal(g, o.pops("g"))
    else:
        assert rel_err(f, o.pops("f")) <= 1e-14 and rel_err(g, o.pops("g")) <= 1e-14
    cav.step(20)
    o.step(20)
    f, g = cav.populations()
    if mode == "exact":
        assert np.array_equal(f, o.pops("f")) and np.array_equal(g, o.pops("g"))
    else:
        assert rel_err(f, o.pops("f")) <= 1e-12 and rel_err(g, o.pops("g")) <= 1e-12
    cav.close()


def test_init_warm_rejects_non_finite(pkg):
    cav = pkg.Cavity(2, 16, 16, grid="tanh", stretch=1.5, Ra=1e4)
    one, zero = np.ones(cav.shape), np.zeros(cav.shape)
    bad = zero.copy()
    bad[3, 4] = np.nan
    with pytest.raises(pkg.LBMError):
        cav.init_warm(one, bad, zero, None, zero)
    cav.close()


@pytest.mark.parametrize("dim,shape,Ra", [(2, (48, 48, 1), 1e3), (2, (40, 56, 1), 1e4)])
def test_fp32_storage_reaches_the_reference_criterion(pkg, dim, shape, Ra):
    # FP32 storage keeps the flow populations as deviations from the rest
    # state, so its check() residual falls below the reference's 1e-6 like
    # FP64's, in about as many iterations, to a Nusselt number within 1e-4
    eps = float(np.float32(1e-6))
    out = {}
    for st in ("f64", "f32"):
        c = pkg.Cavity(dim, *shape, Ra=Ra, grid="tanh", stretch=1.5, storage=st,
                       coords=pkg.mesh_box(shape[0], shape[1], 0, 1.0, shape[1] / shape[0], 1.0, "tanh", 1.5))
        c.initial()
        steps, eu, et = c.run(400000, 2000, eps)
        out[st] = (steps, eu, et, c.nusselt()[0])
        c.close()
    s64, s32 = out["f64"][0], out["f32"][0]
    assert s64 < 400000 and s32 < 400000
    assert out["f32"][1] <= eps and out["f32"][2] <= eps
    assert s32 <= 1.5 * s64 + 4000
    assert abs(out["f32"][3] - out["f64"][3]) <= 1e-4 * abs(out["f64"][3])


@pytest.mark.parametrize("mode", ["exact", "fast"])
@pytest.mark.parametrize("shape", [(40, 24), (128, 128), (100, 37)])
def test_resident_multistep_launch_is_bit_identical(pkg, shape, mode):
    # small 2D domains run an lbm_step call's iterations in one cooperative
    # launch; the result is the per-iteration path's, bit for bit
    out = []
    for resident in (1, 0):
        c = pkg.Cavity(2, *shape, Ra=1e4, grid="tanh", stretch=1.5, mode=mode,
                       coords=pkg.mesh_box(shape[0], shape[1], 0, 1.0, shape[1] / shape[0], 1.0, "tanh", 1.5))
        c.set_option(pkg.lbm.OPT_RESIDENT, resident)
        assert c.get_option(pkg.lbm.OPT_RESIDENT) == resident
        c.initial()
        c.step(37)
        c.step(101)
        f, g = c.populations()
        out.append((f, g, c.macro()))
        c.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    for k in FIELDS2:
        assert np.array_equal(out[0][2][k], out[1][2][k]), k


def test_resident_path_matches_oracle_in_exact_mode(pkg, ora):
    cav, o = pair(pkg, ora, 2, 48, 48, grid="tanh", stretch=1.5, Ra=1e4, mode="exact")
    assert cav.get_option(pkg.lbm.OPT_RESIDENT) == 0  # opt-in
    cav.set_option(pkg.lbm.OPT_RESIDENT, 1)
    assert cav.get_option(pkg.lbm.OPT_RESIDENT) == 1
    cav.step(200)
    o.step(200)
    f, g = cav.populations()
    assert np.array_equal(f, o.pops("f")) and np.array_equal(g, o.pops("g"))
    cav.close()



# ---------------------------------------------------------------------------
# the drop-in tolerance at the benchmark configurations, through the kernels
# and grids the benchmark times
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("case", [
    # 2D differentially heated square cavity, 128^2, tanh 1.5, Ra 1e4 (both step kernels)
    dict(dim=2, n=(128, 128, 1), Ra=1e4, kernel="direct", steps=1000),
    dict(dim=2, n=(128, 128, 1), Ra=1e4, kernel="march", steps=1000),
    # 3D cubic cavity, 128^3, tanh 1.5, Ra 1e5: the TMA march kernel on its default
    # persistent grid and work plan, as the benchmark runs it
    dict(dim=3, n=(128, 128, 128), Ra=1e5, kernel="auto", steps=1000),
], ids=["C1-direct", "C1-march", "C2-march"])
def test_benchmark_config_within_drop_in_tolerance(pkg, ora, case):
    # populations <= 1e-12 relative after 1000 steps, Nu_avg <= 1e-10 (the
    # reference's loop body natural-convection_3dim_mono.f90:373-396 repeated)
    cav, o = pair(pkg, ora, case["dim"], *case["n"], grid="tanh", stretch=1.5, Ra=case["Ra"], mode="fast",
                  kernel=case["kernel"])
    if case["dim"] == 3:
        assert cav.kernel == "march"
        assert cav.get_option(pkg.lbm.OPT_PLAN) == 0
    cav.step(case["steps"])
    o.step(case["steps"])
    f, g = cav.populations()
    assert rel_err(f, o.pops("f")) <= 1e-12
    assert rel_err(g, o.pops("g")) <= 1e-12
    for a, b in zip(cav.nusselt(), o.nusselt()):
        assert abs(a - b) <= 1e-10 * abs(b)
    fscale = np.abs(o.pops("f")).max()
    m = cav.macro()
    for k in (FIELDS2 if case["dim"] == 2 else FIELDS3):
        assert np.abs(m[k] - o.field(k)).max() <= 1e-12 * fscale, k
    cav.close()


@pytest.mark.parametrize("ty,plan,nblocks", [(8, 0, 0), (4, 0, 0), (8, 1, 0), (4, 1, 0), (8, 0, 37), (4, 0, 300)])
def test_march3d_tiles_and_plans_bit_identical(pkg, ora, ty, plan, nblocks):
    # every tile shape and work plan of the 3D march kernel gives the oracle's
    # populations bit for bit (exact mode), on a domain with partial tiles
    cav, o = pair(pkg, ora, 3, 72, 30, 24, grid="tanh", stretch=1.5, Ra=1e5, mode="exact", kernel="march")
    cav.set_option(pkg.lbm.OPT_TILEY, ty)
    cav.set_option(pkg.lbm.OPT_PLAN, plan)
    if nblocks:
        cav.set_option(pkg.lbm.OPT_NBLOCKS, nblocks)
    assert cav.get_option(pkg.lbm.OPT_TILEY) == ty and cav.kernel == "march"
    cav.step(9)
    o.step(9)
    f, g = cav.populations()
    assert np.array_equal(f, o.pops("f")) and np.array_equal(g, o.pops("g"))
    m = cav.macro()
    for k in FIELDS3:
        assert np.array_equal(m[k], o.field(k)), k
    cav.close()


@pytest.mark.parametrize("dim,shape", [(3, (64, 24, 16)), (2, (256, 48, 1))])
def test_wait_timeout_is_reported_and_recoverable(pkg, dim, shape):
    # the march kernels bound every wait for their TMA copies; a limit that
    # runs out makes the step report LBM_ERR_TIMEOUT (the kernel stops issuing,
    # drains its copies and returns), and the context stays usable: with the
    # limit restored a re-initialised run is bit-identical to an untouched one
    def run(c, n):
        c.initial()
        c.step(n)
        return c.populations()

    ref = pkg.Cavity(dim, *shape, grid="tanh", stretch=1.5, mode="exact", kernel="march")
    f0, g0 = run(ref, 6)
    ref.close()
    cav = pkg.Cavity(dim, *shape, grid="tanh", stretch=1.5, mode="exact", kernel="march")
    cav.initial()
    cav.set_option(pkg.lbm.OPT_WAIT_LIMIT, 1)
    try:
        assert cav.get_option(pkg.lbm.OPT_WAIT_LIMIT) == 1
        with pytest.raises(pkg.LBMError) as e:
            cav.step(4)
            cav.synchronize()
        assert e.value.status == -5
        assert "bounded wait" in str(e.value)
    finally:
        cav.set_option(pkg.lbm.OPT_WAIT_LIMIT, 0)
    cav.synchronize()  # the flag was cleared when it was reported
    f, g = run(cav, 6)
    assert np.array_equal(f, f0) and np.array_equal(g, g0)
    cav.close()


@pytest.mark.parametrize("name", ["2dim_mono", "3dim_mono"])
def test_output_ascii_matches_reference_writer(pkg, name, tmp_path):
    # the GPU's fields (exact mode) written by output_ascii are byte for byte
    # the Tecplot file the reference program's own output_ASCII wrote
    import gzip
    gold = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "golden")
    d = dict(np.load(_os.path.join(gold, f"ref_{name}.npz")))
    dim = d["f"].ndim - 1
    shape = d["f"].shape[:-1]
    nz, ny, nx = (shape if dim == 3 else (1,) + shape)
    m = pkg.Mesh(d["x"], d["y"], d.get("z"), 0.0, float(d["length_LB"]), float(d["dt"]))
    cav = pkg.Cavity(dim, nx, ny, nz, Ra=float(d["Ra"]), Pr=float(d["Pr"]), Ma=float(d["Ma"]), coords=m,
                     mode="exact")
    cav.initial()
    cav.step(int(d["itc"]))
    path = str(tmp_path / "out.dat")
    pkg.output_ascii(cav, path)
    cav.close()
    with gzip.open(_os.path.join(gold, f"ref_{name}_tecplot.dat.gz"), "rt") as fh:
        assert open(path).read() == fh.read()


@pytest.mark.parametrize("dim,shape", [(2, (64, 48, 1)), (3, (40, 24, 18))])
def test_storage_conversion_in_place(pkg, dim, shape):
    # FP32 -> FP64 -> FP32 returns every stored FP32 deviation except the
    # lowest bits of values below ~2^-31 (their sum with the O(1) shift in FP64
    # rounds), so a run converted there and back stays within FP32 rounding of
    # the unconverted one (measured 7.5e-9 after 30 steps); FP64
    # -> FP32 rounds each stored deviation once (<= 2^-24 relative); the check
    # history is kept
    kw = dict(Ra=1e5, grid="tanh", stretch=1.5, kernel="march" if dim == 3 else "auto")
    a = pkg.Cavity(dim, *shape, storage="f32", **kw)
    b = pkg.Cavity(dim, *shape, storage="f32", **kw)
    for c in (a, b):
        c.initial()
        c.step(20)
    b.set_storage("f64")
    assert b.storage == "f64"
    b.set_storage("f32")
    for x, y in zip(a.populations(), b.populations()):
        assert np.abs(x - y).max() <= 1e-15
    a.step(30)
    b.step(30)
    for x, y in zip(a.populations(), b.populations()):
        assert np.abs(x - y).max() <= 1e-6
    c = pkg.Cavity(dim, *shape, storage="f64", **kw)
    c.initial()
    c.step(25)
    c.check()
    f64 = c.populations()
    c.set_storage("f32")
    f32 = c.populations()
    for x, y in zip(f32, f64):
        assert np.abs(x - y).max() <= 1e-7
    c.step(5)  # steps on in FP32 storage
    eu, et = c.check()
    assert np.isfinite(eu) and np.isfinite(et) and eu < 1.0
    for cav in (a, b, c):
        cav.close()