"""Generate the golden fixtures from the reference programs themselves.

Each of the four programs of zzhao0930/MPI-Multi-Process-Version is read from
its source, translated mechanically to Python (f90py.py) and executed with an
emulated MPI on the smallest rank count at which it applies every wall (2
ranks for the slab programs, a 2 x 2 (x 1) Cartesian grid for the block
programs).  Only compile-time parameters are patched: the grid size nx (ny, nz
follow as in the source), itc_max, and the check interval MOD(itc,2000).  The
fields the program holds at STOP (populations f, g of every rank, the
macroscopic fields gathered on rank 0, the grid coordinates and the check()
history) are written to ref_<program>.npz next to this script; the slab
programs also run their Tecplot writer output_ASCII, whose file is kept as
ref_<program>_tecplot.dat.gz.

Run here, where the reference is mounted:

    python tests/golden/make_golden.py [--reference /root/reference]

The fixtures are small (< 1 MB together) and committed; nothing else reads the
reference at run time.
"""
from __future__ import annotations

import argparse
import gzip
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import f90py  # noqa: E402

CONFIGS = [
    # name, file, ranks, parameter overrides, check interval
    ("2dim_mono", "natural-convection_2dim_mono.f90", 2, {"nx": 24, "itc_max": 40}, 20),
    ("2dim_block", "natural-convection_2dim_block.f90", 4, {"nx": 24, "itc_max": 40}, 20),
    ("3dim_mono", "natural-convection_3dim_mono.f90", 2, {"nx": 12, "itc_max": 12}, 6),
    ("3dim_block", "natural-convection_3dim_block.f90", 4, {"nx": 12, "itc_max": 12}, 6),
]


def arr(fa):
    """FArray -> numpy array in Fortran order with the declared extents."""
    return np.array(fa.data, dtype=np.float64).reshape(fa.ext, order="F")


def assemble(name, states):
    S0 = states[0]
    dim = 3 if name.startswith("3") else 2
    nx, ny = S0.nx, S0.ny
    nz = S0.nz if dim == 3 else 1
    Q, QT = (9, 5) if dim == 2 else (19, 7)
    f = np.full((nz, ny, nx, Q) if dim == 3 else (ny, nx, Q), np.nan)
    g = np.full((nz, ny, nx, QT) if dim == 3 else (ny, nx, QT), np.nan)
    for S in states:
        r = S.myid
        lf, lg = arr(S.f), arr(S.g)          # (Q, nxL, nyL[, nzL]) Fortran order
        if name == "2dim_mono":
            j0, i0 = S.start1d[r] - 1, 0
        elif name == "2dim_block":
            i0, j0 = S.i_start[r] - 1, S.j_start[r] - 1
        elif name == "3dim_mono":
            i0, j0, k0 = 0, 0, S.start1d[r] - 1
        else:
            i0, j0, k0 = S.i_start[r] - 1, S.j_start[r] - 1, S.k_start[r] - 1
        if dim == 2:
            nxl, nyl = lf.shape[1], lf.shape[2]
            f[j0:j0 + nyl, i0:i0 + nxl, :] = lf.transpose(2, 1, 0)
            g[j0:j0 + nyl, i0:i0 + nxl, :] = lg.transpose(2, 1, 0)
        else:
            nxl, nyl, nzl = lf.shape[1], lf.shape[2], lf.shape[3]
            f[k0:k0 + nzl, j0:j0 + nyl, i0:i0 + nxl, :] = lf.transpose(3, 2, 1, 0)
            g[k0:k0 + nzl, j0:j0 + nyl, i0:i0 + nxl, :] = lg.transpose(3, 2, 1, 0)
    assert not np.isnan(f).any() and not np.isnan(g).any()
    out = {"f": f, "g": g, "itc": S0.itc, "dt": S0.dt, "length_LB": S0.length_lb,
           "Ra": S0.ra, "Pr": S0.pr, "Ma": S0.ma, "Thot": S0.thot, "Tcold": S0.tcold,
           "checks": np.array(S0._checks, dtype=np.float64).reshape(-1, 3), "ranks": len(states)}
    fields = {"u": "u_all", "v": "v_all", "rho": "rho_all", "T": "t_all"}
    if dim == 3:
        fields["w"] = "w_all"
    for k, attr in fields.items():
        a = arr(getattr(S0, attr))      # (nx, ny[, nz]) Fortran order
        out[k] = a.transpose(2, 1, 0) if dim == 3 else a.transpose(1, 0)
    if name == "2dim_mono":
        out["x"], out["y"] = arr(S0.xgrid), arr(S0.y)
    elif name == "2dim_block":
        out["x"], out["y"] = arr(S0.x), arr(S0.y)
    elif name == "3dim_mono":
        out["x"], out["y"], out["z"] = arr(S0.xgrid), arr(S0.ygrid), arr(S0.z)
    else:
        out["x"], out["y"], out["z"] = arr(S0.x), arr(S0.y), arr(S0.z)
    return out


# where the reference programs are mounted (read-only) in the build container
REFERENCE_DIR = os.environ.get("LBM_REFERENCE_DIR", "/root/reference")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=REFERENCE_DIR)
    ap.add_argument("--only", default=None)
    ap.add_argument("--dump-python", default=None, help="write the translated programs here")
    args = ap.parse_args()
    for name, fname, ranks, over, every in CONFIGS:
        if args.only and args.only != name:
            continue
        src = open(os.path.join(args.reference, fname)).read()
        t0 = time.time()
        # the slab programs also run their Tecplot writer, output_ASCII
        # (2dim_mono.f90:818-843, 3dim_mono.f90:1097-1121); rank 0 writes unit 2
        mono = name.endswith("_mono")
        states, code = f90py.run(src, ranks, over, every, with_output=mono)
        if mono:
            tec = os.path.join(HERE, f"ref_{name}_tecplot.dat.gz")
            with open(tec, "wb") as fh, gzip.GzipFile(fileobj=fh, mode="wb", mtime=0, filename="") as gz:
                gz.write("".join(states[0]._io[2]).encode())
        if args.dump_python:
            os.makedirs(args.dump_python, exist_ok=True)
            open(os.path.join(args.dump_python, name + ".py"), "w").write(code)
        out = assemble(name, states)
        path = os.path.join(HERE, f"ref_{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{name}: {ranks} ranks, itc={out['itc']}, checks={out['checks'].tolist()}, "
              f"{time.time() - t0:.1f} s -> {os.path.basename(path)}")


if __name__ == "__main__":
    main()
