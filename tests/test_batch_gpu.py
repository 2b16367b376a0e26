"""Batches of cavities through the C ABI (lbm_batch_*): every member of a
batch must evolve exactly as the same cavity run alone (exact mode: bit for
bit), whatever the tile width, persistent grid, graph replay or launch mode;
the per-member stop test retires converged members."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

def _specs():
    from __graft_entry__ import load_package
    pkg = load_package()
    raw = [dict(nx=64, ny=80, Ra=1e4, Pr=0.71, grid="tanh", stretch=1.2),
           dict(nx=96, ny=96, Ra=1e5, Pr=2.0, grid="tanh", stretch=1.7),
           dict(nx=40, ny=150, Ra=3e3, Pr=7.0, grid="erf", stretch=3.2),
           dict(nx=130, ny=33, Ra=1e6, Pr=0.71, grid="tanh", stretch=1.0),
           dict(nx=33, ny=33, Ra=1e5, Pr=0.71, grid="erf", stretch=3.2)]
    for sp in raw:  # physical size 1 x ny/nx: cells of similar shape on both axes
        sp["coords"] = pkg.mesh_box(sp["nx"], sp["ny"], 0, 1.0, sp["ny"] / sp["nx"], 1.0, sp["grid"], sp["stretch"])
    return raw


SPECS = _specs()


def standalone(pkg, sp, steps, mode="exact"):
    c = pkg.Cavity(2, sp["nx"], sp["ny"], Ra=sp["Ra"], Pr=sp["Pr"], grid=sp["grid"], stretch=sp["stretch"],
                   mode=mode, kernel="direct", coords=sp["coords"])
    c.initial()
    c.step(steps)
    m = c.macro()
    c.close()
    return m


@pytest.fixture(scope="module")
def reference(pkg):
    return [standalone(pkg, sp, 37) for sp in SPECS]


@pytest.mark.parametrize("tile,nblocks,graphs", [(64, 0, 1), (32, 0, 1), (128, 0, 0), (64, 1, 1), (32, 5, 0),
                                                 (128, 7, 1)])
def test_batch_members_match_standalone_bitwise(pkg, reference, tile, nblocks, graphs):
    b = pkg.Batch(2, SPECS, mode="exact")
    b.set_option("tile", tile)
    b.set_option("nblocks", nblocks)
    b.set_option("graphs", graphs)
    b.initial()
    b.step(20)
    b.step(17)
    for m, ref in zip(b.members, reference):
        got = m.macro()
        assert m.itc == 37
        assert np.isfinite(got["rho"]).all()
        for k in ref:
            assert np.array_equal(got[k], ref[k]), k
    b.close()


@pytest.mark.parametrize("dim", [2, 3])
def test_batch_programmatic_dependent_launch_is_bit_identical(pkg, dim):
    # the batch's step kernels as programmatic dependents (the default) against
    # plain stream order: steps, graph replays and the device-side run loop
    if dim == 2:
        specs = SPECS
    else:
        specs = [dict(nx=16, ny=16, nz=12, Ra=1e4, Pr=0.71, grid="tanh", stretch=1.5),
                 dict(nx=20, ny=12, nz=10, Ra=1e3, Pr=2.0, grid="tanh", stretch=1.2)]
    out = []
    for pdl in (1, 0):
        b = pkg.Batch(dim, specs, mode="exact")
        assert b.get_option("pdl") == 1
        b.set_option("pdl", pdl)
        b.initial()
        b.step(20)
        b.step(17)
        status, steps = b.run_masked(None, 1200, 150, 3e-2)
        out.append(([m.macro() for m in b.members], status.tolist(), steps.tolist()))
        b.close()
    assert out[0][1:] == out[1][1:]
    for a, c in zip(out[0][0], out[1][0]):
        for k in a:
            assert np.array_equal(a[k], c[k]), k


def test_batch_one_launch_per_cavity_matches(pkg, reference):
    b = pkg.Batch(2, SPECS, mode="exact")
    b.set_option("persistent", 0)
    b.initial()
    b.step(37)
    for m, ref in zip(b.members, reference):
        got = m.macro()
        for k in ref:
            assert np.array_equal(got[k], ref[k]), k
    b.close()


def test_batch_fast_mode_close_to_standalone(pkg):
    b = pkg.Batch(2, SPECS, mode="fast")
    b.initial()
    b.step(200)
    for m, sp in zip(b.members, SPECS):
        ref = standalone(pkg, sp, 200, mode="fast")
        got = m.macro()
        for k in ref:
            assert np.isfinite(got[k]).all() and np.abs(got[k] - ref[k]).max() <= 1e-12, k
    b.close()


def test_batch_check_and_nusselt_per_member(pkg):
    b = pkg.Batch(2, SPECS, mode="exact")
    b.initial()
    b.step(30)
    eu, et = b.check()
    nh, nc = b.nusselt()
    for i, sp in enumerate(SPECS):
        c = pkg.Cavity(2, sp["nx"], sp["ny"], Ra=sp["Ra"], Pr=sp["Pr"], grid=sp["grid"], stretch=sp["stretch"],
                       mode="exact", coords=sp["coords"])
        c.initial()
        c.step(30)
        assert (eu[i], et[i]) == c.check()
        assert (nh[i], nc[i]) == c.nusselt()
        c.close()
    b.close()


def test_batch_run_retires_converged_members(pkg):
    specs = [dict(nx=32, ny=32, Ra=1e3, Pr=0.71, grid="tanh", stretch=1.5),
             dict(nx=48, ny=96, Ra=1e5, Pr=0.71, grid="tanh", stretch=1.5)]
    b = pkg.Batch(2, specs, mode="fast")
    b.initial()
    conv, steps = b.run(max_steps=3000, check_every=100, eps=2e-2)
    assert conv.dtype == bool and steps.shape == (2,)
    assert conv[0] and steps[0] < 3000
    frozen = b.members[0].macro()
    # the retired member no longer moves while the others continue
    if not conv[1]:
        assert steps[1] == 3000
    b.step(50)
    # after run() every member is active again
    moved = b.members[0].macro()
    assert not np.array_equal(frozen["u"], moved["u"])
    b.close()


def test_batch_tune_picks_a_tile(pkg):
    b = pkg.Batch(2, pkg.sweep_specs(24, seed=3, sides=(64, 96, 128), aspect=(1.0, 2.0)))
    b.initial()
    r = b.tune(steps=6)
    assert r["tile"] in (32, 64, 128) and r["nblocks"] > 0 and r["mlups"] > 0
    assert b.get_option("tile") == r["tile"]
    b.step(4)
    b.synchronize()
    b.close()


def test_batch_3d_members_match_standalone(pkg):
    specs = [dict(nx=16, ny=16, nz=12, Ra=1e5, Pr=0.71, grid="tanh", stretch=1.5),
             dict(nx=20, ny=12, nz=10, Ra=1e4, Pr=2.0, grid="erf", stretch=3.2)]
    b = pkg.Batch(3, specs, mode="exact")
    b.initial()
    b.step(15)
    for m, sp in zip(b.members, specs):
        c = pkg.Cavity(3, sp["nx"], sp["ny"], sp["nz"], Ra=sp["Ra"], Pr=sp["Pr"], grid=sp["grid"],
                       stretch=sp["stretch"], mode="exact", coords=m.mesh)
        c.initial()
        c.step(15)
        ref = c.macro()
        got = m.macro()
        for k in ref:
            assert np.array_equal(got[k], ref[k]), k
        c.close()
    b.close()



def test_sweep_members_against_oracle(pkg, ora):
    # members of the benchmark's seeded 256-cavity sweep (smallest to largest,
    # aspect up to 4) advanced together by the persistent batch kernel in fast
    # mode, each against the oracle: populations <= 1e-12 relative, Nu <= 1e-10
    specs = pkg.sweep_specs(256, seed=0)
    order = sorted(range(len(specs)), key=lambda i: specs[i]["nx"] * specs[i]["ny"])
    pick = sorted({order[0], order[1], order[len(order) // 4], order[len(order) // 2], order[3 * len(order) // 4],
                   max(range(len(specs)), key=lambda i: specs[i]["aspect"]), order[-2], order[-1]})
    sel = [specs[i] for i in pick]
    assert max(sp["aspect"] for sp in sel) > 3.5 and max(sp["nx"] for sp in sel) == 512
    steps = 300
    b = pkg.Batch(2, sel, mode="fast")
    assert b.get_option("persistent") == 1
    b.initial()
    b.step(steps)
    for m, sp in zip(b.members, sel):
        c = sp["coords"]
        o = ora.Oracle(2, sp["nx"], sp["ny"], 1, x=c.x, y=c.y, dt=c.dt, length_LB=c.length_LB, Ra=sp["Ra"],
                       Pr=sp["Pr"])
        o.step(steps)
        f, g = m.populations()
        for got, ref in ((f, o.pops("f")), (g, o.pops("g"))):
            assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
        for a, r in zip(m.nusselt(), o.nusselt()):
            assert abs(a - r) <= 1e-10 * abs(r)
    b.close()


@pytest.mark.parametrize("dim,growth", [(2, 0), (2, 100), (3, 0)])
def test_batch_run_matches_host_loop(pkg, dim, growth):
    # the device-side stop test of lbm_batch_run against each member run alone
    # with the reference's loop on the host: the same iterations, the same
    # stop, the same fields (exact mode, bit for bit)
    if dim == 2:
        specs = [dict(nx=32, ny=32, Ra=1e3, Pr=0.71, grid="tanh", stretch=1.5),
                 dict(nx=48, ny=40, Ra=1e4, Pr=2.0, grid="tanh", stretch=1.2),
                 dict(nx=40, ny=64, Ra=3e4, Pr=0.71, grid="tanh", stretch=1.7),
                 dict(nx=64, ny=64, Ra=1e5, Pr=7.0, grid="tanh", stretch=1.0)]
        for sp in specs:
            sp["coords"] = pkg.mesh_box(sp["nx"], sp["ny"], 0, 1.0, sp["ny"] / sp["nx"], 1.0, sp["grid"],
                                        sp["stretch"])
    else:
        specs = [dict(nx=16, ny=16, nz=12, Ra=1e4, Pr=0.71, grid="tanh", stretch=1.5),
                 dict(nx=20, ny=12, nz=10, Ra=1e3, Pr=2.0, grid="tanh", stretch=1.2)]
    ce, eps, max_steps = 150, 3e-2, 4500
    b = pkg.Batch(dim, specs, mode="exact")
    b.set_option("growth", growth)
    b.initial()
    status, steps = b.run_masked(None, max_steps, ce, eps)
    assert (status == 1).any()
    for m, sp, st, n in zip(b.members, specs, status, steps):
        c = pkg.Cavity(dim, sp["nx"], sp["ny"], sp.get("nz", 1), Ra=sp["Ra"], Pr=sp["Pr"], grid=sp["grid"],
                       stretch=sp["stretch"], mode="exact", coords=m.mesh)
        c.initial()
        done, ref = 0, (100.0, 100.0)
        while done < max_steps:
            c.step(ce)
            done += ce
            ref = c.check()
            if not (ref[0] > eps or ref[1] > eps):
                break
        conv = not (ref[0] > eps or ref[1] > eps)
        assert n == done and st == (1 if conv else 0)
        assert m.itc == done
        got, want = m.macro(), c.macro()
        for k in want:
            assert np.array_equal(got[k], want[k]), k
        c.close()
    b.close()


@pytest.mark.parametrize("persistent", [1, 0])
def test_batch_3d_persistent_matches_standalone(pkg, persistent):
    # 3D members of different sizes in one persistent kernel (or one launch
    # each) evolve bit for bit as each cavity alone
    specs = [dict(nx=40, ny=24, nz=18, Ra=1e5, Pr=0.71, grid="tanh", stretch=1.5),
             dict(nx=33, ny=16, nz=12, Ra=1e4, Pr=2.0, grid="erf", stretch=3.2),
             dict(nx=64, ny=32, nz=20, Ra=3e5, Pr=0.71, grid="tanh", stretch=1.2)]
    b = pkg.Batch(3, specs, mode="exact")
    b.set_option("persistent", persistent)
    b.initial()
    b.step(9)
    b.step(4)
    for m, sp in zip(b.members, specs):
        c = pkg.Cavity(3, sp["nx"], sp["ny"], sp["nz"], Ra=sp["Ra"], Pr=sp["Pr"], grid=sp["grid"],
                       stretch=sp["stretch"], mode="exact", coords=m.mesh, kernel="direct")
        c.initial()
        c.step(13)
        ref, got = c.macro(), m.macro()
        for k in ref:
            assert np.array_equal(got[k], ref[k]), k
        c.close()
    if persistent:
        r = b.tune(steps=4)
        assert r["tile"] == 32 and r["nblocks"] > 0
    b.close()


def test_batch_tuner_chooses_storage(pkg):
    # the autotuner's storage axis: with FP32 and FP64 allowed (the rule for a
    # run's transient) it keeps the faster one, converting the batch in place;
    # the members then step on, and FP64 alone converts back
    b = pkg.Batch(2, pkg.sweep_specs(12, seed=5, sides=(64, 96, 128), aspect=(1.0, 2.0)), storage="f64")
    b.initial()
    b.step(10)
    r = b.tune(steps=6, storages=("f32", "f64"))
    assert r["storage"] in ("f32", "f64") and r["mlups"] > 0
    assert all(m.storage == r["storage"] for m in b.members)
    b.step(20)
    b.set_storage("f64")
    b.step(10)
    eu, et = b.check()
    assert np.isfinite(eu).all() and np.isfinite(et).all()
    b.close()


def test_batch_run_mixed_member_by_member(pkg):
    # lbm_batch_run_mixed: each member runs FP32 to switch_eps, is converted
    # alone to FP64 and runs on to eps; the result is the FP64 fixed point
    # (continued to a tight criterion it meets the all-FP64 run's to 1e-8)
    specs = [dict(nx=32, ny=32, Ra=1e3, Pr=0.71, grid="tanh", stretch=1.5),
             dict(nx=40, ny=40, Ra=1e4, Pr=2.0, grid="tanh", stretch=1.2),
             dict(nx=48, ny=32, Ra=3e4, Pr=0.71, grid="tanh", stretch=1.7),
             dict(nx=36, ny=36, Ra=1e5, Pr=7.0, grid="tanh", stretch=1.3)]
    for sp in specs:
        sp["coords"] = pkg.mesh_box(sp["nx"], sp["ny"], 0, 1.0, sp["ny"] / sp["nx"], 1.0, sp["grid"], sp["stretch"])
    mix = pkg.Batch(2, specs, storage="f32")
    ref = pkg.Batch(2, specs, storage="f64")
    for b in (mix, ref):
        b.initial()
    st, n, low = mix.run_mixed(None, 400000, 500, switch_eps=1e-4, eps=1e-6)
    assert (st == 1).all()
    assert ((low > 0) & (low < n)).all()
    assert len(set(low.tolist())) > 1          # members switched at different times
    assert mix.get_option("storage") == 0      # every member ended in FP64
    assert all(m.itc == k for m, k in zip(mix.members, n))
    st2, _ = ref.run_masked(None, 400000, 500, 1e-6)
    assert (st2 == 1).all()
    for b in (mix, ref):
        s, _ = b.run_masked(None, 2000000, 500, 1e-11)
        assert (s == 1).all()
    a, r = mix.nusselt()[0], ref.nusselt()[0]
    assert np.abs(a - r).max() <= 1e-8 * np.abs(r).max()
    mix.close()
    ref.close()
