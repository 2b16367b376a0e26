"""The oracle against golden fixtures produced by the reference programs
themselves (tests/golden/make_golden.py: the four Fortran programs translated
mechanically and run on emulated MPI ranks).  Populations and macroscopic
fields must match to the bit; the check() residuals, whose sums the reference
splits across ranks, to 1e-13 relative."""
import glob
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# the reference programs (read-only, present only where the fixtures are made)
REFERENCE_DIR = os.environ.get("LBM_REFERENCE_DIR", "/root/reference")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz")))


def load(path):
    d = dict(np.load(path))
    dim = d["f"].ndim - 1
    shape = d["f"].shape[:-1]
    nz, ny, nx = (shape if dim == 3 else (1,) + shape)
    return d, dim, nx, ny, nz


def run_oracle(ora, d, dim, nx, ny, nz):
    o = ora.Oracle(dim, nx, ny, nz, x=d["x"], y=d["y"], z=d.get("z"), dt=float(d["dt"]),
                   length_LB=float(d["length_LB"]), Ra=float(d["Ra"]), Pr=float(d["Pr"]), Ma=float(d["Ma"]),
                   Thot=float(d["Thot"]), Tcold=float(d["Tcold"]))
    every = int(d["checks"][0][0])
    checks = []
    for it in range(1, int(d["itc"]) + 1):
        o.step(1)
        if it % every == 0:
            checks.append((it,) + o.check())
    return o, checks


def test_fixtures_present():
    names = {os.path.basename(p) for p in FIXTURES}
    assert names == {"ref_2dim_mono.npz", "ref_2dim_block.npz", "ref_3dim_mono.npz", "ref_3dim_block.npz"}


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_oracle_matches_reference_bitwise(ora, path):
    d, dim, nx, ny, nz = load(path)
    # the reference's mesh() as restated by the oracle gives the same grid
    x, y, z, _, L, dt = ora.mesh("erf", 3.2, nx, ny, nz if dim == 3 else 0)
    assert np.array_equal(x, d["x"]) and np.array_equal(y, d["y"]) and L == d["length_LB"] and dt == d["dt"]
    if dim == 3:
        assert np.array_equal(z, d["z"])
    o, checks = run_oracle(ora, d, dim, nx, ny, nz)
    assert np.array_equal(o.pops("f"), d["f"])
    assert np.array_equal(o.pops("g"), d["g"])
    for k in ("u", "v", "T", "rho") + (("w",) if dim == 3 else ()):
        assert np.array_equal(o.field(k), d[k]), k
    assert len(checks) == len(d["checks"])
    for (it, eu, et), ref in zip(checks, d["checks"]):
        assert it == ref[0]
        assert eu == pytest.approx(ref[1], rel=1e-13) and et == pytest.approx(ref[2], rel=1e-13)


def test_mono_and_block_decompositions_agree():
    # the slab and the Cartesian programs compute the same fields
    for dim in ("2dim", "3dim"):
        a = dict(np.load(os.path.join(GOLDEN, f"ref_{dim}_mono.npz")))
        b = dict(np.load(os.path.join(GOLDEN, f"ref_{dim}_block.npz")))
        for k in ("f", "g", "u", "v", "T", "rho"):
            assert np.array_equal(a[k], b[k]), (dim, k)


@pytest.mark.skipif(not os.path.isdir(REFERENCE_DIR), reason="reference sources not mounted")
def test_fixture_regenerates_from_reference(tmp_path):
    # regenerate the smallest fixture from the reference source and compare
    import subprocess
    import sys
    src = os.path.join(GOLDEN, "make_golden.py")
    code = ("import sys, numpy as np; sys.path.insert(0, %r); import f90py, make_golden as m; "
            "src = open(%r).read(); "
            "states, _ = f90py.run(src, 2, {'nx': 24, 'itc_max': 40}, 20); "
            "out = m.assemble('2dim_mono', states); "
            "ref = np.load(%r); "
            "assert all(np.array_equal(out[k], ref[k]) for k in ('f', 'g', 'u', 'v', 'T', 'rho'))"
            % (GOLDEN, os.path.join(REFERENCE_DIR, "natural-convection_2dim_mono.f90"),
               os.path.join(GOLDEN, "ref_2dim_mono.npz")))
    subprocess.check_call([sys.executable, "-c", code])
    assert os.path.exists(src)


# ---------------------------------------------------------------------------
# the Tecplot writer against the file the reference's own output_ASCII wrote
# ---------------------------------------------------------------------------
def _tecplot_fixture(name):
    import gzip
    with gzip.open(os.path.join(GOLDEN, f"ref_{name}_tecplot.dat.gz"), "rt") as fh:
        return fh.read()


@pytest.mark.parametrize("name", ["2dim_mono", "3dim_mono"])
def test_tecplot_writer_reproduces_reference_file(pkg, name, tmp_path):
    # output_ASCII (2dim_mono.f90:818-843, 3dim_mono.f90:1097-1121), run by the
    # interpreted reference program on its gathered fields, wrote the fixture;
    # the library's writer given the same fields writes the same bytes
    d = dict(np.load(os.path.join(GOLDEN, f"ref_{name}.npz")))
    dim = 3 if name.startswith("3") else 2
    fields = {k: d[k] for k in ("rho", "u", "v", "T")}
    if dim == 3:
        fields["w"] = d["w"]
    path = str(tmp_path / "out.dat")
    pkg.write_tecplot(path, d["x"], d["y"], d["z"] if dim == 3 else None, fields)
    got = open(path).read()
    ref = _tecplot_fixture(name)
    assert got.splitlines()[:3] == ref.splitlines()[:3]  # title, variables, zone
    assert got == ref


def test_fortran_format_engine_pinned():
    # the fixture's renderer, against values whose Ew.d forms are known
    import sys
    sys.path.insert(0, GOLDEN)
    import f90fmt
    assert f90fmt.edit_e(1.23456789, 11, 4) == " 0.1235E+01"
    assert f90fmt.edit_e(-0.000123456, 13, 6) == "-0.123456E-03"
    assert f90fmt.edit_e(0.0, 11, 4) == " 0.0000E+00"
    assert f90fmt.edit_e(999.99996, 11, 4) == " 0.1000E+04"
    assert f90fmt.edit_e(1e-120, 11, 4) == " 0.1000-119"
    assert f90fmt.render("('ZONE',1x,'I=',1x,i5,2x,'J=',1x,i5,1x,'F=POINT')", [24, 7]) == \
        "ZONE I=    24  J=     7 F=POINT\n"
    assert f90fmt.render("(1x,2(e11.4,' '),10(e13.6,' '))", [1.0, 2.0, 3.0]) == \
        "  0.1000E+01  0.2000E+01  0.300000E+01 \n"
