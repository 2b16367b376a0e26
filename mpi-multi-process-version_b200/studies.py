"""Measurement studies on the GPU: storage-precision errors and time to a
steady Nusselt number.

Run as `python -m` style through the package loader, e.g.

    python -c "from __graft_entry__ import load_package as L; L().studies.main()" precision3d

Every study prints one JSON line per result.  The FP64 results they compare
against come from the library's FP64 path, which the test suite holds to
the CPU restatement of the reference (bit-identical in exact mode, 1e-12 in
the fast mode used here).
"""
from __future__ import annotations

import json
import sys
import time

import numpy as np

from . import lbm as L


def _max_abs(m, keys):
    return {k: float(np.abs(m[k]).max()) for k in keys}


def precision_errors(dim, shape, Ra, Pr=0.71, steps=20000, grid="tanh", stretch=1.5, noise=0.0, seed=0,
                     storages=("f64", "f32")):
    """Run the same cavity in each storage precision from the same initial
    state for `steps` iterations; report Nu_avg, max |u|, max |v| (max |w|)
    and their errors against FP64, plus the throughput of each variant."""
    nx, ny, nz = shape
    res = {}
    rng = np.random.default_rng(seed)
    for st in storages:
        c = L.Cavity(dim, nx, ny, nz, Ra=Ra, Pr=Pr, grid=grid, stretch=stretch, storage=st)
        sh = c.shape
        T0 = rng.uniform(-noise, noise, sh) if noise else np.zeros(sh)
        rng = np.random.default_rng(seed)  # same noise for every precision
        one, zero = np.ones(sh), np.zeros(sh)
        c.init_equilibrium(one, zero, zero, zero if dim == 3 else None, T0)
        c.step(10)
        c.synchronize()
        t0 = time.perf_counter()
        c.step(steps - 10)
        c.synchronize()
        dt = time.perf_counter() - t0
        m = c.macro()
        nu = c.nusselt()
        keys = ("u", "v", "w") if dim == 3 else ("u", "v")
        res[st] = {"nu_hot": nu[0], "nu_cold": nu[1], **{f"max_{k}": v for k, v in _max_abs(m, keys).items()},
                   "mlups": c.nnode * (steps - 10) / dt / 1e6, "kernel": c.kernel}
        c.close()
    base = res["f64"]
    out = []
    for st, r in res.items():
        row = {"storage": st, "dim": dim, "shape": list(shape), "Ra": Ra, "Pr": Pr, "steps": steps, "noise": noise, **r}
        if st != "f64":
            row["err_nu_hot"] = abs(r["nu_hot"] - base["nu_hot"])
            row["rel_err_nu_hot"] = abs(r["nu_hot"] - base["nu_hot"]) / abs(base["nu_hot"])
            for k in [k for k in r if k.startswith("max_")]:
                row["rel_err_" + k] = abs(r[k] - base[k]) / max(base[k], 1e-300)
        out.append(row)
    return out


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    what = argv[0] if argv else "precision3d"
    if what == "precision3d":
        # 3D differentially heated cube, 128^3, tanh 1.5, Ra 1e5: FP64 vs FP32 storage
        rows = precision_errors(3, (128, 128, 128), 1e5, steps=int(argv[1]) if len(argv) > 1 else 20000)
    elif what == "precision2d":
        # 2D 2048^2, tanh 1.5, Ra in {1e6, 1e7, 1e8}, seeded temperature noise 1e-4
        steps = int(argv[1]) if len(argv) > 1 else 20000
        rows = []
        for Ra in (1e6, 1e7, 1e8):
            rows += precision_errors(2, (2048, 2048, 1), Ra, steps=steps, noise=1e-4, seed=0)
    else:
        raise SystemExit(f"unknown study {what}")
    for r in rows:
        print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
