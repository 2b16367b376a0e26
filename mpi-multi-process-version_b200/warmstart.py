"""Learned warm start for the differentially heated cavity.

The reference starts every run from the conduction state of initial()
(natural-convection_2dim_mono.f90:199-240) and iterates until the check()
residuals fall below 1e-6 (2M:307).  Here a U-Net (surrogate.Net, trained on
the GPU by this library's own kernels) predicts the steady (u, v, T) field of
a cavity from (Ra, Pr, grid-coordinate maps); lbm_init_warm turns the
prediction into populations (equilibrium plus the first-order
non-equilibrium part), and the solver then runs to the same residual
criterion as a cold start, so it alone judges the result.  A member whose
residual diverges is restarted from the conduction state (the cold-start
fallback).

Representation.  Fields live on the cavity's nodes; the network sees an
R x R image in index space (node i of n sits at (i + 1/2)/n, pixel r of R at
(r + 1/2)/R; linear interpolation between the two).  Inputs: the wall-
normalised physical node coordinates X, Y (which carry the grid stretching),
(log10 Ra - 4.5)/1.5, (Pr - 3.855)/3.145 and (stretch - 1.5)/0.5.  Outputs:
u/U0, v/U0 with U0 = Ma/sqrt(3) (the free-fall velocity of the reference's
parameter choice, 2M:152-162) and (T - Tcold)/(Thot - Tcold), each
standardised with the training set's mean and deviation.
"""
from __future__ import annotations

import functools
import json
import time

import numpy as np

from . import lbm as L
from . import surrogate as S

F32_EPS = float(np.float32(1e-6))   # the reference's epsU/epsT (single-precision literals, 2M:35)
# how much faster FP32 stepping must be for the mixed run to pay off: its
# hand-over to FP64 costs 9-25 % more iterations, and while members of both
# storages run every step launches two kernels side by side.  Measured on B200
# (first 64 held-out cavities, warm start): FP32 batch stepping 1.40x FP64's,
# yet the mixed run took 68.3 s against FP64's 62.0 s
FP32_HANDOVER_COST = 1.6


# ---------------------------------------------------------------------------
# index-space resampling
# ---------------------------------------------------------------------------
@functools.lru_cache(maxsize=64)
def _interp_matrix(n_src: int, n_dst: int) -> np.ndarray:
    xs = (np.arange(n_src) + 0.5) / n_src
    xd = (np.arange(n_dst) + 0.5) / n_dst
    W = np.zeros((n_dst, n_src))
    for k, x in enumerate(xd):
        j = np.searchsorted(xs, x) - 1
        if j < 0:
            W[k, 0] = 1.0
        elif j >= n_src - 1:
            W[k, n_src - 1] = 1.0
        else:
            t = (x - xs[j]) / (xs[j + 1] - xs[j])
            W[k, j], W[k, j + 1] = 1.0 - t, t
    return W


def resample(a: np.ndarray, shape) -> np.ndarray:
    """Bilinear resampling of a (ny, nx) field to `shape` in index space."""
    a = np.asarray(a, dtype=np.float64)
    Wy = _interp_matrix(a.shape[0], int(shape[0]))
    Wx = _interp_matrix(a.shape[1], int(shape[1]))
    return Wy @ a @ Wx.T


def unit_coords(c, n, dt):
    """Node coordinates 1..n of one axis scaled to [0, 1] between the two
    halfway bounce-back walls (dt/2 outside the end nodes)."""
    c = np.asarray(c, dtype=np.float64)
    lo, hi = c[1] - 0.5 * dt, c[n] + 0.5 * dt
    return (c[1:n + 1] - lo) / (hi - lo)


# ---------------------------------------------------------------------------
# cases
# ---------------------------------------------------------------------------
def sample_cases(n, seed, sizes=(128, 160, 192, 224, 256), log10_ra=(3.0, 6.0), pr=(0.71, 7.0),
                 stretch=(1.0, 2.0)):
    """Seeded square cavities: side from `sizes`, Ra log-uniform, Pr and the
    tanh stretch uniform."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        side = int(rng.choice(sizes))
        b = float(rng.uniform(*stretch))
        out.append({"nx": side, "ny": side, "Ra": float(10 ** rng.uniform(*log10_ra)),
                    "Pr": float(rng.uniform(*pr)), "grid": "tanh", "stretch": b,
                    "coords": L.mesh_box(side, side, 0, 1.0, 1.0, 1.0, "tanh", b)})
    return out


NF = 8   # feature channels built on the host (the network's input has IN_CH, zero beyond NF)


def features(case, R):
    """(R, R, NF) float32 input image of one case."""
    m = case["coords"]
    nx, ny = case["nx"], case["ny"]
    pix = (np.arange(R) + 0.5) / R
    X = np.interp(pix, (np.arange(nx) + 0.5) / nx, unit_coords(m.x, nx, m.dt))
    Y = np.interp(pix, (np.arange(ny) + 0.5) / ny, unit_coords(m.y, ny, m.dt))
    f = np.zeros((R, R, NF), dtype=np.float32)
    f[..., 0] = X[None, :]
    f[..., 1] = Y[:, None]
    f[..., 2] = (np.log10(case["Ra"]) - 4.5) / 1.5
    f[..., 3] = (case["Pr"] - 3.855) / 3.145
    f[..., 4] = (case.get("stretch", 1.5) - 1.5) / 0.5
    return f


def velocity_scale(case):
    return float(case.get("Ma", 0.1)) / np.sqrt(3.0)


def targets(case, fields, R):
    """(R, R, 3) float32 target image (u/U0, v/U0, theta) of one steady field."""
    U0 = velocity_scale(case)
    Th, Tc = float(case.get("Thot", 1.0)), float(case.get("Tcold", 0.0))
    chans = (fields["u"] / U0, fields["v"] / U0, (fields["T"] - Tc) / (Th - Tc))
    return np.stack([resample(c, (R, R)) for c in chans], axis=-1).astype(np.float32)


def centro_symmetrize(u, v, T, Th, Tc):
    """Project fields onto the cavity's centro-symmetry.  The mesh is mirror
    symmetric about the centre (node i of n mirrors node n+1-i), the walls are
    the same under a half turn with hot and cold exchanged, and the steady
    state satisfies u -> -u, v -> -v, T -> Th + Tc - T under that half turn.
    The conduction start is exactly symmetric; a prediction with small
    asymmetric errors would excite the slowly decaying antisymmetric modes, so
    the warm start keeps only the symmetric part."""
    rot = lambda a: a[::-1, ::-1]  # noqa: E731
    return 0.5 * (u - rot(u)), 0.5 * (v - rot(v)), 0.5 * (T + (Th + Tc) - rot(T))


def fields_from_image(case, img, symmetrize=True):
    """Invert `targets`: (R, R, 3) physical-scale image -> node fields,
    projected onto the centro-symmetry of a cavity (centro_symmetrize)."""
    U0 = velocity_scale(case)
    Th, Tc = float(case.get("Thot", 1.0)), float(case.get("Tcold", 0.0))
    shape = (case["ny"], case["nx"])
    u = resample(img[..., 0], shape) * U0
    v = resample(img[..., 1], shape) * U0
    T = Tc + resample(img[..., 2], shape) * (Th - Tc)
    if symmetrize:
        u, v, T = centro_symmetrize(u, v, T, Th, Tc)
    return {"rho": np.ones(shape), "u": u, "v": v, "T": T}


# ---------------------------------------------------------------------------
# the model
# ---------------------------------------------------------------------------
class WarmStart:
    """The surrogate network plus its target normalisation."""

    def __init__(self, R=128, device=0, seed=0):
        self.net = S.Net(R=R, device=device, seed=seed)
        self.R = R
        self.mean = np.zeros(3, dtype=np.float32)
        self.std = np.ones(3, dtype=np.float32)
        self.history = []

    # -- training ---------------------------------------------------------
    def fit(self, X, Y, steps=3000, batch=16, lr=2e-3, warmup=100, seed=0, log_every=100, log=None):
        """Train on inputs X (N, R, R, IN_CH) and targets Y (N, R, R, 3).
        Adam with linear warm-up and cosine decay; samples drawn with a seeded
        generator.  Returns the loss history [(step, loss)]."""
        torch = self.net.torch
        dev = self.net.dev
        self.mean = Y.reshape(-1, 3).mean(0).astype(np.float32)
        self.std = (Y.reshape(-1, 3).std(0) + 1e-6).astype(np.float32)
        Xd = self._device_inputs(X)
        Yd = torch.from_numpy(np.ascontiguousarray((Y - self.mean) / self.std, dtype=np.float32)).to(dev)
        N = X.shape[0]
        rng = np.random.default_rng(seed)
        buf = self.net.buffers(batch)
        tgt = torch.empty(batch * self.R * self.R, 3, dtype=torch.float32, device=dev)
        hist = []
        t0 = time.perf_counter()
        for it in range(steps):
            idx = torch.from_numpy(rng.integers(0, N, size=batch)).to(dev)
            buf["x"].copy_(Xd.index_select(0, idx))
            tgt.copy_(Yd.index_select(0, idx).reshape(-1, 3))
            self.net.forward(B=batch)
            loss = self.net.loss(tgt, batch)
            self.net.backward(batch)
            frac = it / max(1, steps - 1)
            lr_t = lr * min(1.0, (it + 1) / warmup) * 0.5 * (1.0 + np.cos(np.pi * frac))
            self.net.adam(lr_t)
            if (it + 1) % log_every == 0 or it == steps - 1:
                val = float(loss.item())
                hist.append((it + 1, val))
                if log:
                    log(f"step {it + 1:6d}  loss {val:.5f}  lr {lr_t:.2e}  {time.perf_counter() - t0:.1f}s")
        torch.cuda.synchronize(dev)
        self.history += hist
        self.train_seconds = time.perf_counter() - t0
        return hist

    def _device_inputs(self, X):
        """(N, R, R, IN_CH) bf16 device tensor from host features (N, R, R, <= IN_CH)."""
        torch = self.net.torch
        Xd = torch.zeros(X.shape[0], self.R, self.R, S.IN_CH, dtype=torch.bfloat16, device=self.net.dev)
        for k in range(0, X.shape[0], 256):
            chunk = torch.from_numpy(np.ascontiguousarray(X[k:k + 256], dtype=np.float32))
            Xd[k:k + chunk.shape[0], ..., :X.shape[-1]] = chunk.to(self.net.dev).to(torch.bfloat16)
        return Xd

    # -- inference --------------------------------------------------------
    def predict_images(self, X, batch=16):
        """Physical-scale (N, R, R, 3) predictions for inputs X."""
        out = np.empty((X.shape[0], self.R, self.R, 3), dtype=np.float32)
        for k in range(0, X.shape[0], batch):
            xb = self._device_inputs(X[k:k + batch])
            y = self.net.forward(xb).reshape(xb.shape[0], self.R, self.R, 3)
            out[k:k + xb.shape[0]] = y.cpu().numpy()
        return out * self.std + self.mean

    def predict_fields(self, cases):
        X = np.stack([features(c, self.R) for c in cases])
        return [fields_from_image(c, img) for c, img in zip(cases, self.predict_images(X))]

    # -- persistence ------------------------------------------------------
    def save(self, path, meta=None):
        """Weights as bf16 bit patterns (what the kernels use) plus the
        normalisation and metadata."""
        torch = self.net.torch
        bits = self.net.master.to(torch.bfloat16).view(torch.int16).cpu().numpy()
        np.savez_compressed(path, weights_bf16=bits, mean=self.mean, std=self.std, R=np.int32(self.R),
                            meta=np.array(json.dumps(meta or {})))

    @classmethod
    def load(cls, path, device=0):
        d = np.load(path, allow_pickle=False)
        ws = cls(R=int(d["R"]), device=device)
        torch = ws.net.torch
        bits = torch.from_numpy(d["weights_bf16"].astype(np.int16))
        master = bits.view(torch.bfloat16).to(torch.float32).numpy()
        ws.net.load_state(master)
        ws.mean, ws.std = d["mean"].astype(np.float32), d["std"].astype(np.float32)
        ws.meta = json.loads(str(d["meta"]))
        return ws


# ---------------------------------------------------------------------------
# solving to a steady state
# ---------------------------------------------------------------------------
def _prepare(cases, storage, device, growth):
    specs = [{k: v for k, v in c.items()} for c in cases]
    b = L.Batch(2, specs, storage=storage, device=device)
    b.set_option("growth", int(growth))
    return b


def _init(b, cases, init, model, predictions):
    """Initial state of every member: the conduction state (cold) or the
    model's prediction through lbm_init_warm.  Returns the prediction time."""
    if init == "cold":
        b.initial()
        return 0.0
    t0 = time.perf_counter()
    preds = predictions if predictions is not None else model.predict_fields(cases)
    t_pred = time.perf_counter() - t0
    for mem, f in zip(b.members, preds):
        mem.init_warm(f["rho"], f["u"], f["v"], None, f["T"])
    return t_pred


def _run(b, eps, max_steps, check_every, mask=None, switch_eps=None):
    """The batch run to the stop criterion, with the cold-start fallback for
    members stopped for a diverging residual; max_steps is per member (an
    array or a number).  switch_eps: mixed precision member by member
    (lbm_batch_run_mixed: FP32 to switch_eps, then FP64 to eps).  Returns
    (status, steps, fallback, FP32 steps or None)."""
    limit = np.broadcast_to(np.asarray(max_steps, dtype=np.int64), (b.n,)).copy()
    on = np.ones(b.n, bool) if mask is None else np.asarray(mask, bool).copy()
    status = np.zeros(b.n, np.int32)
    steps = np.zeros(b.n, np.int64)
    low = np.zeros(b.n, np.int64)
    # all members run together up to the smallest remaining budget; those still
    # running with budget left go on together, so no member exceeds its own
    sel = on & (limit > 0)
    while sel.any():
        cap = int((limit - steps)[sel].min())
        m = None if sel.all() else sel
        if switch_eps is None:
            st, n = b.run_masked(m, cap, check_every, eps)
            lo = np.zeros(b.n, np.int64)
        else:
            st, n, lo = b.run_mixed(m, cap, check_every, switch_eps, eps)
        status = np.where(sel, st, status)
        steps = np.where(sel, steps + n, steps)
        low = np.where(sel, low + lo, low)
        sel = sel & (st == 0) & (steps < limit)
    fallback = on & (status == -1)
    if fallback.any():
        for i in np.nonzero(fallback)[0]:
            b.members[i].initial()
        left = np.where(fallback, limit - steps, 0)
        st2, n2, _, lo2 = _run(b, eps, left, check_every, mask=fallback & (left > 0), switch_eps=switch_eps)
        status = np.where(fallback, st2, status)
        steps = np.where(fallback, steps + n2, steps)
        if lo2 is not None:
            low = np.where(fallback, low + lo2, low)
    return status, steps, fallback, (low if switch_eps is not None else None)


# ---------------------------------------------------------------------------
# extrapolation of the slowest mode (no reference counterpart)
# ---------------------------------------------------------------------------
# Near the steady state a run converges geometrically, s_k = s* + c r^k v,
# and in slowly converging cavities one real mode dominates (successive
# changes d1 = s1 - s0, d2 = s2 - s1 a fixed number of iterations apart are
# nearly parallel).  Lyusternik's (Aitken's) extrapolation then removes that
# mode: s* = s2 + r / (1 - r) d2 with r = <d2, d1> / <d1, d1>.  The solver
# still judges the result by the reference's criterion afterwards.
EXTRAP_MAX_FACTOR = 50.0


def lyusternik_factor(s0, s1, s2, fmax=EXTRAP_MAX_FACTOR):
    """(factor, r) of the extrapolation s2 + factor * (s2 - s1) from three
    states an equal number of iterations apart; factor 0 unless 0 < r < 1,
    and at most fmax."""
    d1 = np.asarray(s1, np.float64) - np.asarray(s0, np.float64)
    d2 = np.asarray(s2, np.float64) - np.asarray(s1, np.float64)
    den = float(d1.ravel() @ d1.ravel())
    if not den > 0.0:
        return 0.0, 0.0
    r = float(d2.ravel() @ d1.ravel()) / den
    if not 0.0 < r < 1.0:
        return 0.0, r
    return min(r / (1.0 - r), float(fmax)), r


def _state(m):
    """A member's populations and macroscopic fields (host copies)."""
    f, g = m.populations()
    mac = {k: v for k, v in m.macro().items() if k in ("rho", "u", "v", "w", "T")}
    return f, g, mac


def _load_extrapolated(m, a, b, fac):
    """Load b + fac * (b - a) (populations and fields) into member m: an exact
    restart of b when fac is 0 (set_populations + set_macro)."""
    f = b[0] + fac * (b[0] - a[0])
    g = b[1] + fac * (b[1] - a[1])
    mac = {k: b[2][k] + fac * (b[2][k] - a[2][k]) for k in b[2]}
    m.set_populations(f, g)
    m.set_macro(mac["rho"], mac["u"], mac["v"], mac.get("w"), mac["T"])


def _run_extrapolated(b, eps, max_steps, check_every, tau, delta):
    """_run with one extrapolation of the slowest mode per member: every
    member runs to the residual tau, then `delta` and again `delta` more
    iterations (three states); each member that has the budget is loaded with
    its extrapolated state and all of them run on to eps.  Every member that
    continues is loaded (unchanged ones with their own state, an exact
    restart), so they stay in step.  Returns _run's tuple and the factors."""
    limit = np.broadcast_to(np.asarray(max_steps, dtype=np.int64), (b.n,)).copy()
    status, steps, fallback, _ = _run(b, tau, limit, check_every)
    reached = status == 1
    status = np.where(reached, 0, status)  # tau is not the criterion: a member out of budget here is capped
    cont = reached & (steps < limit)
    go = cont & (limit - steps > 2 * delta)
    facs = np.zeros(b.n)
    if go.any():
        idx = np.nonzero(go)[0]
        snaps = [[_state(b.members[i]) for i in idx]]
        ok = np.ones(len(idx), bool)
        for _ in range(2):
            st, n = b.run_masked(go, int(delta), check_every, 0.0)  # eps 0: exactly delta iterations
            steps = np.where(go, steps + n, steps)
            snaps.append([_state(b.members[i]) for i in idx])
            ok &= st[idx] == 0  # stopped by the iteration count, not by a bad residual
        for j, i in enumerate(idx):
            s0, s1, s2 = (snaps[k][j] for k in range(3))
            fac = 0.0
            if ok[j]:
                fac, _ = lyusternik_factor(np.concatenate([s0[0].ravel(), s0[1].ravel()]),
                                           np.concatenate([s1[0].ravel(), s1[1].ravel()]),
                                           np.concatenate([s2[0].ravel(), s2[1].ravel()]))
            facs[i] = fac
            _load_extrapolated(b.members[i], s1, s2, fac)
    for part in (go, cont & ~go):  # the loaded members together, then any others
        if part.any():
            st, n, fb, _ = _run(b, eps, np.where(part, limit - steps, 0), check_every, mask=part)
            status = np.where(part, st, status)
            steps = np.where(part, steps + n, steps)
            fallback = fallback | (part & fb)
    return status, steps, fallback, None, facs


def solve(cases, init="cold", model=None, storage="f64", eps=F32_EPS, check_every=2000, max_steps=1_000_000,
          growth=100, want_fields=False, device=0, predictions=None, field_fn=None, switch_eps=1e-5,
          extrapolate=None):
    """Run every case to the reference's stop criterion (errorU, errorT <= eps
    at a check every `check_every` iterations) in one batch, with the stop
    test on the device.

    init "cold": the conduction state of initial(); "warm": the model's
    prediction (or `predictions`, a list of node-field dicts) through
    lbm_init_warm.  Members whose residual diverges (not finite, or growth x
    above its smallest value) restart cold and their steps add up.
    storage "f64" / "f32"; "mixed": member by member, FP32 storage until the
    residuals reach `switch_eps`, then that member alone converts in place to
    FP64 and runs to `eps` (lbm_batch_run_mixed), so the result is the FP64
    fixed point while the other members go on in FP32; "auto": the autotuner
    (lbm_batch_tune) times FP32 and FP64 stepping on the batch and the run is
    "mixed" if FP32 is more than FP32_HANDOVER_COST times faster, else FP64.
    max_steps bounds each member's iterations over all phases.
    extrapolate (tau, delta): one extrapolation of each member's slowest mode
    (_run_extrapolated) at residual tau from states delta iterations apart;
    ignored when the run is mixed.
    Returns a dict of per-case arrays and the wall time: `seconds` from the
    first initialisation to the result (prediction and lbm_init_warm included),
    of which `predict_seconds` was the network."""
    first = "f32" if storage in ("mixed", "auto") else storage
    b = _prepare(cases, first, device, growth)
    b.synchronize()
    t0 = time.perf_counter()
    t_pred = _init(b, cases, init, model, predictions)
    tuned = None
    tune_steps = 0
    mixed = storage == "mixed"
    if storage == "auto":
        # the autotuner times the transient's storages on this batch; FP32 pays
        # for its hand-over to FP64 with more iterations (measured 9-25 % on
        # the held-out cavities), so it is chosen only when it is that much faster
        it0 = b.members[0].itc
        t64 = b.tune(steps=4, storages=("f64",))
        t32 = b.tune(steps=4, storages=("f32",))
        mixed = t32["mlups"] > FP32_HANDOVER_COST * t64["mlups"]
        if not mixed:
            b.set_storage("f64")
            b.set_option("tile", t64["tile"])
            b.set_option("nblocks", t64["nblocks"])
        tune_steps = b.members[0].itc - it0
        tuned = {"f64": t64, "f32": t32, "chosen": "mixed" if mixed else "f64"}
    b.synchronize()
    facs = None
    if extrapolate is not None and not mixed:
        tau, delta = extrapolate
        status, steps, fallback, steps_low, facs = _run_extrapolated(b, eps, max_steps - tune_steps, check_every,
                                                                     float(tau), int(delta))
    else:
        status, steps, fallback, steps_low = _run(b, eps, max_steps - tune_steps, check_every,
                                                   switch_eps=switch_eps if mixed else None)
    steps = steps + tune_steps
    b.synchronize()
    seconds = time.perf_counter() - t0
    nu_hot, nu_cold = b.nusselt()
    out = {"status": status, "steps": steps, "fallback": fallback, "nu_hot": nu_hot, "nu_cold": nu_cold,
           "seconds": seconds, "predict_seconds": t_pred, "nodes": np.array([m.nnode for m in b.members]),
           "storage": storage, "init": init, "steps_low_precision": steps_low, "tuned": tuned,
           "extrapolation_factors": facs}
    if want_fields:
        out["fields"] = [{k: v for k, v in m.macro().items() if k in ("rho", "u", "v", "T")} for m in b.members]
    if field_fn is not None:
        out["field_out"] = [field_fn(i, m.macro()) for i, m in enumerate(b.members)]
    b.close()
    return out


# ---------------------------------------------------------------------------
# 3D cavities from the 2D model
# ---------------------------------------------------------------------------
def fields_3d_from_2d(case3d, model):
    """Warm-start fields of a 3D cube from the 2D model: the cube is heated
    along y and gravity points along -z (3M:563, 953-956), so the 2D image's
    (x, y, u, v) map to the cube's (y, z, v, w); the prediction is extruded
    along x with u = 0."""
    m = case3d["coords"]
    nx, ny, nz = case3d["nx"], case3d["ny"], case3d["nz"]
    c2 = {"nx": ny, "ny": nz, "Ra": case3d["Ra"], "Pr": case3d["Pr"], "stretch": case3d.get("stretch", 1.5),
          "coords": L.Mesh(m.y, m.z, None, m.dx0, m.length_LB, m.dt)}
    f2 = model.predict_fields([c2])[0]                # arrays (nz, ny)
    shape = (nz, ny, nx)
    ext = lambda a: np.broadcast_to(a[:, :, None], shape).copy()  # noqa: E731
    return {"rho": np.ones(shape), "u": np.zeros(shape), "v": ext(f2["u"]), "w": ext(f2["v"]), "T": ext(f2["T"])}


# ---------------------------------------------------------------------------
# the pipeline: solver-generated data -> training -> held-out evaluation
# ---------------------------------------------------------------------------
def build_dataset(cases, R, storage="f32", eps=1e-5, max_steps=400_000, log=print):
    """Steady fields of `cases` from the solver (cold start, one batch) and
    their (features, targets) images."""
    t0 = time.perf_counter()
    res = solve(cases, init="cold", storage=storage, eps=eps, max_steps=max_steps,
                field_fn=lambda i, f: targets(cases[i], f, R))
    X = np.stack([features(c, R) for c in cases])
    Y = np.stack(res.pop("field_out"))
    if log:
        log(f"dataset: {len(cases)} cases, {int((res['status'] == 1).sum())} converged to {eps:g}, "
            f"{int(np.sum(res['steps'] * res['nodes'])) / 1e9:.1f} G lattice updates in "
            f"{time.perf_counter() - t0:.0f} s")
    return X, Y, res


def step_seconds(sizes, storage="f64", steps=4000):
    """Measured seconds per iteration of one square cavity of each side
    (one cavity per launch: the drop-in's time)."""
    out = {}
    for n in sizes:
        c = L.Cavity(2, n, n, Ra=1e5, grid="tanh", stretch=1.5, storage=storage)
        c.initial()
        c.step(200)
        c.synchronize()
        t0 = time.perf_counter()
        c.step(steps)
        c.synchronize()
        out[int(n)] = (time.perf_counter() - t0) / steps
        c.close()
    return out


def evaluate(model, cases, max_steps=1_500_000, log=print):
    """Steps and time to the reference's criterion for FP64 cold (the drop-in)
    and the mixed-precision warm start (FP32 to residual 1e-5, then FP64; one
    batch; the model's prediction), Nu error against the FP64 fixed point
    (FP64 continued to residual 1e-8), plus single-change variants (FP64 warm,
    mixed cold) and FP32 alone."""
    rows = {}
    b = L.Batch(2, [dict(c) for c in cases], storage="f64")
    b.initial()
    b.synchronize()
    t0 = time.perf_counter()
    st, steps = b.run_masked(None, max_steps, 2000, F32_EPS)
    b.synchronize()
    rows["f64_cold"] = {"status": st, "steps": steps, "seconds": time.perf_counter() - t0,
                        "nu": b.nusselt()[0]}
    st2, steps2 = b.run_masked(None, max_steps, 2000, 1e-8)
    rows["f64_ref"] = {"status": st2, "steps": steps + steps2, "nu": b.nusselt()[0]}
    b.close()
    if log:
        log(f"f64 cold: {rows['f64_cold']['seconds']:.1f} s, converged {int((st == 1).sum())}/{len(cases)}")
    for name, init, storage in (("mixed_warm", "warm", "mixed"), ("f64_warm", "warm", "f64"),
                                ("mixed_cold", "cold", "mixed"), ("f32_warm", "warm", "f32")):
        r = solve(cases, init=init, model=model, storage=storage, max_steps=max_steps)
        rows[name] = {"status": r["status"], "steps": r["steps"], "seconds": r["seconds"], "nu": r["nu_hot"],
                      "fallback": r["fallback"], "predict_seconds": r["predict_seconds"],
                      "steps_low_precision": r["steps_low_precision"]}
        if log:
            log(f"{name}: {r['seconds']:.1f} s (of which {r['predict_seconds']:.2f} s prediction), converged "
                f"{int((r['status'] == 1).sum())}/{len(cases)}, fallbacks {int(r['fallback'].sum())}")
    return rows


def summarize(rows):
    """Headline numbers of an evaluation: time and steps of each variant
    against FP64 cold, and the Nusselt error against the FP64 fixed point."""
    ref = np.asarray(rows["f64_ref"]["nu"])
    base = rows["f64_cold"]
    out = {"cases": int(len(ref)), "f64_cold_converged": int((np.asarray(base["status"]) == 1).sum()),
           "f64_cold_batched_seconds": base["seconds"], "f64_cold_sequential_seconds": base.get("sequential_seconds"),
           "f64_cold_steps": int(np.sum(base["steps"]))}
    for name in [k for k in ("mixed_warm", "f64_warm", "mixed_cold", "f32_warm", "f32_cold", "f64_cold") if k in rows]:
        r = rows[name]
        ok = np.asarray(r["status"]) == 1
        err = np.abs(np.asarray(r["nu"]) - ref) / np.abs(ref)
        secs = r["seconds"]  # from the first initialisation to the result, prediction included
        out[name] = {"seconds": secs, "steps": int(np.sum(r["steps"])), "converged": int(ok.sum()),
                     "nu_within_1e-4": int((ok & (err <= 1e-4)).sum()),
                     "max_nu_rel_err_converged": float(err[ok].max()) if ok.any() else None,
                     "step_ratio_vs_f64_cold": float(np.sum(base["steps"]) / max(1, np.sum(r["steps"]))),
                     "speedup_vs_f64_cold_sequential": (base.get("sequential_seconds") or 0.0) / secs,
                     "speedup_vs_f64_cold_batched": base["seconds"] / secs,
                     "fallbacks": int(np.sum(r.get("fallback", 0)))}
    return out


def _jsonable(x):
    if isinstance(x, dict):
        return {k: _jsonable(v) for k, v in x.items()}
    if isinstance(x, np.ndarray):
        return x.tolist()
    if isinstance(x, (np.floating, np.integer)):
        return x.item()
    return x


def main(argv=None):
    """pipeline [--train N] [--test N] [--sizes a,b,..] [--R R] [--steps S]
    [--data-steps M] [--eval-steps M] [--out DIR]"""
    import argparse
    import os
    import sys
    ap = argparse.ArgumentParser(prog="warmstart")
    ap.add_argument("what", choices=["pipeline"])
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--test", type=int, default=200)
    ap.add_argument("--sizes", default="128,160,192,224,256")
    ap.add_argument("--R", type=int, default=128)
    ap.add_argument("--steps", type=int, default=8000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--data-eps", type=float, default=1e-5)
    ap.add_argument("--data-steps", type=int, default=400_000)
    ap.add_argument("--eval-steps", type=int, default=1_500_000)
    ap.add_argument("--with3d", type=int, default=0, help="side of a 3D cube to evaluate (0: none)")
    ap.add_argument("--out", default="warmstart_out")
    ap.add_argument("--phase", default="all", choices=["all", "train", "eval"],
                    help="train: data + training + held-out image error; eval: time to steady state with --model")
    ap.add_argument("--model", default=None, help="eval phase: a saved model (.npz)")
    a = ap.parse_args(sys.argv[1:] if argv is None else argv)
    os.makedirs(a.out, exist_ok=True)
    sizes = tuple(int(s) for s in a.sizes.split(","))
    logf = open(os.path.join(a.out, "log.txt"), "a")

    def log(msg):
        print(msg, flush=True)
        logf.write(msg + "\n")
        logf.flush()

    train_cases = sample_cases(a.train, seed=1000, sizes=sizes)
    test_cases = sample_cases(a.test, seed=2000, sizes=sizes)
    if a.phase in ("all", "train"):
        X, Y, _ = build_dataset(train_cases, a.R, eps=a.data_eps, max_steps=a.data_steps, log=log)
        Xt, Yt, _ = build_dataset(test_cases, a.R, eps=a.data_eps, max_steps=a.data_steps, log=log)
        model = WarmStart(R=a.R, seed=0)
        model.fit(X, Y, steps=a.steps, batch=a.batch, lr=a.lr, log_every=250, log=log)
        log(f"training: {a.steps} steps of {a.batch} in {model.train_seconds:.1f} s")
        pred = model.predict_images(Xt)
        rel = [float(np.linalg.norm(pred[..., k] - Yt[..., k]) / np.linalg.norm(Yt[..., k])) for k in range(3)]
        log(f"held-out relative L2 error (u, v, theta): {rel}")
        meta = {"train": a.train, "test": a.test, "sizes": sizes, "R": a.R, "steps": a.steps, "batch": a.batch,
                "lr": a.lr, "data_eps": a.data_eps, "data_steps": a.data_steps, "train_seed": 1000,
                "test_seed": 2000, "heldout_rel_l2": rel, "train_seconds": model.train_seconds,
                "history": model.history}
        model.save(os.path.join(a.out, "warmstart_unet.npz"), meta)
        del X, Y
        if a.phase == "train":
            log("done")
            return
    else:
        model = WarmStart.load(a.model)
        meta = model.meta
    rows = evaluate(model, test_cases, max_steps=a.eval_steps, log=log)
    tstep = step_seconds(sorted(set(sizes)))
    side = np.array([c["nx"] for c in test_cases])
    rows["f64_cold"]["sequential_seconds"] = float(sum(rows["f64_cold"]["steps"][i] * tstep[int(side[i])]
                                                       for i in range(len(side))))
    out = {"meta": meta, "cases": [{k: v for k, v in c.items() if k != "coords"} for c in test_cases],
           "step_seconds_f64_single": tstep, "rows": rows}
    if a.with3d:
        n = a.with3d
        m3 = L.mesh_box(n, n, n, 1.0, 1.0, 1.0, "tanh", 1.5)
        c3 = {"nx": n, "ny": n, "nz": n, "Ra": 1e5, "Pr": 0.71, "stretch": 1.5, "coords": m3}
        res3 = {}
        for init in ("cold", "warm"):
            cav = L.Cavity(3, n, n, n, Ra=1e5, Pr=0.71, coords=m3)
            if init == "cold":
                cav.initial()
            else:
                f = fields_3d_from_2d(c3, model)
                cav.init_warm(f["rho"], f["u"], f["v"], f["w"], f["T"])
            cav.synchronize()
            t0 = time.perf_counter()
            steps, eu, et = cav.run(a.eval_steps, 2000, F32_EPS)
            cav.synchronize()
            res3[init] = {"steps": int(steps), "seconds": time.perf_counter() - t0, "nu": cav.nusselt()[0],
                          "errU": eu, "errT": et}
            log(f"3D {n}^3 {init}: {res3[init]}")
            cav.close()
        out["cube"] = res3
    out["summary"] = summarize(rows)
    log(f"summary: {json.dumps(_jsonable(out['summary']))}")
    with open(os.path.join(a.out, "eval.json"), "w") as f:
        json.dump(_jsonable(out), f)
    log("done")


if __name__ == "__main__":
    main()
