"""Host logic of the warm-start driver on CPU: warmstart.solve's cold-start
fallback and its mixed-precision hand-over, driven through a stand-in for the
batch API (no GPU), and the evaluation summary."""
import numpy as np
import pytest


class _FakeMember:
    def __init__(self, log, i):
        self.log, self.i, self.nnode = log, i, 100 + i
        self.state = None
        self.itc = 0

    def initial(self):
        self.log.append(("initial", self.i))
        self.state = "cold"

    def init_warm(self, rho, u, v, w, T):
        self.log.append(("warm", self.i))
        self.state = "warm"

    def populations(self):
        return ("f", self.i), ("g", self.i)

    def set_populations(self, f, g):
        self.log.append(("set", self.i, f[1], g[1]))
        self.state = "loaded"


class _FakeBatch:
    """Scripted lbm_batch_run_masked outcomes: statuses[k] for the k-th run."""
    instances = []

    def __init__(self, dim, specs, storage="f64", device=0):
        self.storage, self.n = storage, len(specs)
        self.log = []
        self.members = [_FakeMember(self.log, i) for i in range(self.n)]
        self.runs = []
        self.closed = False
        _FakeBatch.instances.append(self)

    def initial(self):
        for m in self.members:
            m.initial()

    def set_option(self, name, value):
        self.log.append(("option", name, value))

    def set_storage(self, storage):
        self.log.append(("storage", storage))
        self.storage = storage

    def synchronize(self):
        pass

    def run_masked(self, mask, max_steps, check_every, eps):
        k = len(self.runs)
        self.runs.append((None if mask is None else [bool(x) for x in mask], eps))
        script = self.script[k]
        status = np.array(script["status"], dtype=np.int32)
        steps = np.array(script["steps"], dtype=np.int64)
        if mask is not None:
            status = np.where(mask, status, 0)
            steps = np.where(mask, steps, 0)
        return status, steps

    def run_mixed(self, mask, max_steps, check_every, switch_eps, eps):
        k = len(self.runs)
        self.runs.append((None if mask is None else [bool(x) for x in mask], (switch_eps, eps), max_steps))
        script = self.script[k]
        out = [np.array(script[key], dtype=t) for key, t in (("status", np.int32), ("steps", np.int64),
                                                               ("low", np.int64))]
        if mask is not None:
            out = [np.where(mask, a, 0) for a in out]
        return tuple(out)

    def tune(self, steps=20, storages=None):
        self.log.append(("tune", tuple(storages)))
        for m in self.members:
            m.itc += 36
        self.storage = storages[0]
        return {"tile": 64, "nblocks": 1184, "mlups": self.rates[storages[0]], "storage": storages[0]}

    def nusselt(self):
        return np.arange(self.n, dtype=float) + 1.0, np.zeros(self.n)

    def close(self):
        self.closed = True


@pytest.fixture
def fake(pkg, monkeypatch):
    _FakeBatch.instances.clear()
    monkeypatch.setattr(pkg.warmstart.L, "Batch", _FakeBatch)
    return _FakeBatch


def _cases(n):
    return [{"nx": 8, "ny": 8, "Ra": 1e4, "Pr": 0.71} for _ in range(n)]


def _preds(n):
    z = np.zeros((8, 8))
    return [{"rho": z + 1, "u": z, "v": z, "T": z} for _ in range(n)]


def test_diverged_members_restart_cold_and_their_steps_add_up(pkg, fake):
    W = pkg.warmstart
    _FakeBatch.script = [{"status": [1, -1, 1], "steps": [4000, 6000, 8000]},
                         {"status": [0, 1, 0], "steps": [0, 10000, 0]}]
    r = W.solve(_cases(3), init="warm", predictions=_preds(3), storage="f64", eps=1e-6, growth=50)
    b = _FakeBatch.instances[0]
    assert ("option", "growth", 50) in b.log
    # only the diverged member was re-initialised and re-run
    assert [e for e in b.log if e[0] == "initial"] == [("initial", 1)]
    assert b.runs[1][0] == [False, True, False]
    assert r["status"].tolist() == [1, 1, 1]
    assert r["steps"].tolist() == [4000, 16000, 8000]
    assert r["fallback"].tolist() == [False, True, False]
    assert b.closed


def test_mixed_precision_member_by_member(pkg, fake):
    # one batch in FP32; the library hands each member to FP64 on its own
    # (lbm_batch_run_mixed); a member stopped for divergence restarts cold and
    # runs mixed again on what is left of its budget
    W = pkg.warmstart
    _FakeBatch.script = [{"status": [1, -1], "steps": [26000, 9000], "low": [20000, 9000]},
                         {"status": [0, 1], "steps": [0, 30000], "low": [0, 21000]}]
    r = W.solve(_cases(2), init="warm", predictions=_preds(2), storage="mixed", eps=1e-6, switch_eps=1e-5,
                max_steps=40000)
    assert len(_FakeBatch.instances) == 1
    b = _FakeBatch.instances[0]
    assert b.storage == "f32"
    assert b.runs[0] == (None, (1e-5, 1e-6), 40000)
    assert b.runs[1] == ([False, True], (1e-5, 1e-6), 31000)
    assert [e for e in b.log if e[0] == "initial"] == [("initial", 1)]
    assert b.closed
    assert r["steps"].tolist() == [26000, 39000]
    assert r["steps_low_precision"].tolist() == [20000, 30000]
    assert r["status"].tolist() == [1, 1] and r["fallback"].tolist() == [False, True]


def test_summary_counts_and_ratios(pkg):
    W = pkg.warmstart
    ref = np.array([1.0, 2.0, 4.0])
    rows = {
        "f64_ref": {"nu": ref},
        "f64_cold": {"status": np.array([1, 1, 0]), "steps": np.array([10, 20, 30]), "seconds": 6.0,
                     "nu": ref * (1 + np.array([1e-5, 2e-5, 1e-3])), "sequential_seconds": 12.0},
        "mixed_warm": {"status": np.array([1, 1, 1]), "steps": np.array([5, 10, 15]), "seconds": 3.0,
                       "predict_seconds": 1.0, "nu": ref * (1 + np.array([5e-5, 2e-4, 0.0])),
                       "fallback": np.array([False, True, False])},
    }
    s = W.summarize(rows)
    m = s["mixed_warm"]
    assert m["converged"] == 3 and m["nu_within_1e-4"] == 2 and m["fallbacks"] == 1
    assert m["step_ratio_vs_f64_cold"] == pytest.approx(2.0)
    assert m["speedup_vs_f64_cold_sequential"] == pytest.approx(4.0)
    assert m["speedup_vs_f64_cold_batched"] == pytest.approx(2.0)
    assert s["f64_cold"]["nu_within_1e-4"] == 2


@pytest.mark.parametrize("rates,mixed", [({"f64": 20000.0, "f32": 25000.0}, False),
                                         ({"f64": 20000.0, "f32": 38000.0}, True)])
def test_auto_storage_weighs_the_fp32_handover(pkg, fake, rates, mixed):
    # "auto": the tuner times FP64 and FP32 stepping on the batch; mixed
    # precision is chosen only if FP32 is faster than FP32_HANDOVER_COST x FP64
    W = pkg.warmstart
    _FakeBatch.rates = rates
    _FakeBatch.script = [{"status": [1, 1], "steps": [5000, 7000], "low": [3000, 4000]}]
    r = W.solve(_cases(2), init="warm", predictions=_preds(2), storage="auto", max_steps=100000)
    b = _FakeBatch.instances[0]
    assert [e for e in b.log if e[0] == "tune"] == [("tune", ("f64",)), ("tune", ("f32",))]
    assert r["tuned"]["chosen"] == ("mixed" if mixed else "f64")
    assert (b.runs[0][1] == (1e-5, W.F32_EPS)) == mixed
    if not mixed:
        assert ("storage", "f64") in b.log and ("option", "tile", 64) in b.log
    # the tuner's steps count toward each member's iterations and budget
    assert r["steps"].tolist() == [5072, 7072]


# ---------------------------------------------------------------------------
# extrapolation of the slowest mode (warmstart.lyusternik_factor,
# warmstart._run_extrapolated)
# ---------------------------------------------------------------------------
def test_lyusternik_factor_recovers_a_geometric_limit(pkg):
    W = pkg.warmstart
    rng = np.random.default_rng(3)
    s_star, v = rng.normal(size=50), rng.normal(size=50)
    for r in (0.3, 0.9, 0.97):
        s = [s_star + 0.2 * r ** k * v for k in range(3)]
        fac, rr = W.lyusternik_factor(*s)
        assert rr == pytest.approx(r, rel=1e-12)
        assert np.allclose(s[2] + fac * (s[2] - s[1]), s_star, rtol=0, atol=1e-12)
    # an oscillating or growing sequence, or no change at all: no extrapolation
    for r in (-0.5, 1.2):
        s = [s_star + 0.2 * r ** k * v for k in range(3)]
        assert W.lyusternik_factor(*s)[0] == 0.0
    assert W.lyusternik_factor(s_star, s_star, s_star) == (0.0, 0.0)
    # the factor is capped
    s = [s_star + 0.2 * 0.999 ** k * v for k in range(3)]
    assert W.lyusternik_factor(*s, fmax=50.0)[0] == 50.0


class _GeoMember:
    """A member whose state relaxes geometrically to a fixed point: every
    iteration multiplies its deviation by rho_it.  Loading a state (as
    set_populations does) flips its buffer parity, like a first collision."""

    def __init__(self, rho_it, seed):
        rng = np.random.default_rng(seed)
        self.rho_it = rho_it
        self.star = {"f": rng.normal(size=(4, 3, 9)), "g": rng.normal(size=(4, 3, 5)),
                     "u": rng.normal(size=(4, 3)) + 2.0, "rho": np.ones((4, 3)), "v": rng.normal(size=(4, 3)),
                     "T": rng.normal(size=(4, 3))}
        self.v = {k: 1e-2 * rng.normal(size=a.shape) for k, a in self.star.items()}
        self.t = 0.0            # "time" of the state: deviation = v * rho_it ** t
        self.parity = 0
        self.u_prev = np.zeros((4, 3))
        self.loads = 0

    def _get(self, k):
        return self.star[k] + self.v[k] * self.rho_it ** self.t

    def populations(self):
        return self._get("f"), self._get("g")

    def macro(self):
        return {k: self._get(k) for k in ("rho", "u", "v", "T")}

    def set_populations(self, f, g):
        # the loaded deviation along v fixes the new time of the state
        dev = (f - self.star["f"]).ravel() @ self.v["f"].ravel() / (self.v["f"].ravel() @ self.v["f"].ravel())
        self.loaded_dev = dev
        self.t = np.inf if dev <= 1e-300 else np.log(dev) / np.log(self.rho_it)
        self.parity ^= 1
        self.loads += 1

    def set_macro(self, rho, u, v, w, T):
        assert w is None

    def initial(self):
        raise AssertionError("no member diverges here")


class _GeoBatch:
    def __init__(self, members):
        self.members = members
        self.n = len(members)

    def run_masked(self, mask, max_steps, check_every, eps):
        on = np.ones(self.n, bool) if mask is None else np.asarray(mask, bool)
        par = {self.members[i].parity for i in np.nonzero(on)[0]}
        assert len(par) <= 1, "members on the mask out of step"
        status = np.zeros(self.n, np.int32)
        done = np.zeros(self.n, np.int64)
        for i in np.nonzero(on)[0]:
            m = self.members[i]
            while done[i] < max_steps:
                k = min(check_every, max_steps - done[i])
                m.t += k
                done[i] += k
                if k == check_every:  # a check: the reference's relative change of u
                    u = m._get("u")
                    res = np.linalg.norm(u - m.u_prev) / np.linalg.norm(u)
                    m.u_prev = u
                    if res <= eps:
                        status[i] = 1
                        break
        return status, done


def test_extrapolated_run_jumps_to_the_fixed_point(pkg):
    W = pkg.warmstart
    # per-iteration contraction: slow (1e-4 per 2000-iteration check ~ 0.82)
    # and slower; the last member has no budget left for the snapshots
    members = [_GeoMember(1 - 1e-4, 0), _GeoMember(1 - 2e-5, 1), _GeoMember(1 - 5e-4, 2)]
    limit = np.array([3_000_000, 3_000_000, 30_000])
    plain = _GeoBatch([_GeoMember(m.rho_it, s) for m, s in zip(members, range(3))])
    st0, n0, fb0, _ = W._run(plain, W.F32_EPS, limit, 2000)
    b = _GeoBatch(members)
    status, steps, fallback, low, facs = W._run_extrapolated(b, W.F32_EPS, limit, 2000, 3e-5, 10_000)
    assert (status == 1).all() and not fallback.any() and low is None
    assert facs[0] > 0 and facs[1] > 0 and facs[2] == 0.0
    # a one-mode deviation is removed by the jump (to rounding; it started at 1)
    assert abs(members[0].loaded_dev) < 1e-9 and abs(members[1].loaded_dev) < 1e-9
    # every member that went on after the jump was loaded
    assert [m.loads for m in members] == [1, 1, 0]
    assert steps[1] < 0.5 * n0[1]
    assert (steps <= limit).all()


def test_extrapolated_run_reports_tau_as_not_converged(pkg):
    W = pkg.warmstart
    # the step count at which this member reaches tau, from a copy of it
    probe = _GeoBatch([_GeoMember(1 - 5e-4, 7)])
    st, n, _, _ = W._run(probe, 3e-5, 1_000_000, 2000)
    assert st[0] == 1
    # a budget that ends exactly there: the member met tau, not the criterion
    b = _GeoBatch([_GeoMember(1 - 5e-4, 7)])
    status, steps, fallback, _, facs = W._run_extrapolated(b, W.F32_EPS, n, 2000, 3e-5, 10_000)
    assert status[0] == 0 and steps[0] == n[0] and facs[0] == 0.0 and b.members[0].loads == 0
