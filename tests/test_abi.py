"""The C-ABI library loads on a machine without a GPU, exports every symbol
include/lbm_b200.h declares, reproduces the reference's host arithmetic
(mesh(), the parameter block of initial()) bit for bit against the oracle, and
rejects bad input before touching a device."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols(header="lbm_b200.h"):
    hdr = open(os.path.join(ROOT, "include", header)).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(lbm_[a-z0-9_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol(pkg):
    L = pkg.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), f"{s} declared in lbm_b200.h but not exported"
    assert sorted(pkg.EXPORTS) == syms


def test_library_exports_every_surrogate_symbol(pkg):
    L = pkg.lib()
    syms = declared_symbols("lbm_surrogate.h")
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), f"{s} declared in lbm_surrogate.h but not exported"
    assert sorted(pkg.surrogate.NN_EXPORTS) == syms
    pkg.surrogate.nn()  # every signature binds


def test_include_headers_are_covered():
    # every header of the C ABI is checked by one of the export tests above
    assert sorted(os.listdir(os.path.join(ROOT, "include"))) == ["lbm_b200.h", "lbm_surrogate.h"]


def test_abi_version(pkg):
    assert pkg.lib().lbm_abi_version() == 1


@pytest.mark.parametrize("grid,stretch", [("erf", 3.2), ("tanh", 1.5), ("uniform", 0.0)])
@pytest.mark.parametrize("dims", [(33, 33, 0), (16, 20, 12)])
def test_mesh_matches_oracle_bitwise(pkg, ora, grid, stretch, dims):
    nx, ny, nz = dims
    m = pkg.mesh(nx, ny, nz, grid, stretch)
    x, y, z, dx0, L, dt = ora.mesh(grid, stretch, nx, ny, nz)
    assert np.array_equal(m.x, x) and np.array_equal(m.y, y)
    if nz:
        assert np.array_equal(m.z, z)
    assert (m.dx0, m.length_LB, m.dt) == (dx0, L, dt)


@pytest.mark.parametrize("dim,Ra,Pr", [(2, 1e5, 0.71), (2, 1e4, 7.0), (3, 1e6, 0.71), (3, 1e5, 2.0)])
def test_derived_parameters_match_oracle_bitwise(pkg, ora, dim, Ra, Pr):
    n = 40
    m = pkg.mesh(n, n, n if dim == 3 else 0, "erf", 3.2)
    p = pkg.lbm_params(dim, n, n, n if dim == 3 else 1, Ra, Pr, 0.1, 1.0, 0.0, m.dt, m.length_LB, 0, 0, 0, 0)
    out = np.zeros(9)
    assert pkg.lib().lbm_derived_params(ctypes.byref(p), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
    o = ora.Oracle(dim, n, n, n if dim == 3 else 1, x=m.x, y=m.y, z=m.z, dt=m.dt, length_LB=m.length_LB,
                   Ra=Ra, Pr=Pr)
    ref = o.params()
    keys = ["viscosity_LB", "kappa", "gbeta", "tauf", "Snu", "Sq", "sig_k", "dt", "length_LB"]
    for k, v in zip(keys, out):
        assert v == ref[k], k


def _params(pkg, **kw):
    base = dict(dim=2, nx=16, ny=16, nz=1, Ra=1e5, Pr=0.71, Ma=0.1, Thot=1.0, Tcold=0.0, dt=1.0,
                length_LB=40.0, storage=0, mode=0, device=0, reserved=0)
    base.update(kw)
    return pkg.lbm_params(**base)


@pytest.mark.parametrize("bad", [dict(dim=4), dict(nx=2), dict(Ra=-1.0), dict(Pr=0.0), dict(dt=float("nan")),
                                 dict(length_LB=0.5), dict(storage=7), dict(mode=3), dict(mode=1, storage=1),
                                 dict(Thot=0.0), dict(reserved=1)])
def test_bad_parameters_rejected_without_device(pkg, bad):
    p = _params(pkg, **bad)
    out = np.zeros(9)
    st = pkg.lib().lbm_derived_params(ctypes.byref(p), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert st in (-1, -8)
    assert pkg.lib().lbm_last_error()


def test_retired_binary16_storage_is_rejected(pkg):
    # LBM_STORE_F16S (2) is retired: its errors against FP64 were of order one
    p = _params(pkg, storage=2)
    out = np.zeros(9)
    st = pkg.lib().lbm_derived_params(ctypes.byref(p), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert st == -8
    assert b"retired" in pkg.lib().lbm_last_error()


def test_create_without_gpu_reports_no_device(pkg, has_gpu):
    if has_gpu:
        pytest.skip("a GPU is present")
    m = pkg.mesh(16, 16, 0)
    with pytest.raises(pkg.LBMError) as e:
        pkg.Cavity(2, 16, 16, coords=m)
    assert e.value.status == -9


def test_create_rejects_non_increasing_coordinates(pkg):
    m = pkg.mesh(16, 16, 0)
    m.x[5] = m.x[4]
    with pytest.raises(pkg.LBMError) as e:
        pkg.Cavity(2, 16, 16, coords=m)
    assert e.value.status == -1


def test_fortran_e_format(pkg):
    # Fortran (1x,2(e11.4,' '),10(e13.6,' ')) as in output_ASCII (2M:838)
    assert pkg.fortran_e(1.23456789, 11, 4) == " 0.1235E+01"
    assert pkg.fortran_e(-0.000123456, 13, 6) == "-0.123456E-03"
    assert pkg.fortran_e(0.0, 13, 6) == " 0.000000E+00"
    assert pkg.fortran_e(999.99996, 11, 4) == " 0.1000E+04"


def test_mesh_box_reduces_to_mesh_for_unit_square(pkg):
    for grid, b in (("erf", 3.2), ("tanh", 1.5)):
        a = pkg.mesh(33, 33, 0, grid, b)
        m = pkg.mesh_box(33, 33, 0, 1.0, 1.0, 1.0, grid, b)
        assert np.array_equal(a.x, m.x) and np.array_equal(a.y, m.y) and a.dt == m.dt and a.length_LB == m.length_LB


def test_mesh_box_tall_cavity_spacings(pkg):
    # 1 x 3 cavity with 40 x 120 nodes: every node spacing is at least one
    # lattice unit and the walls lie half a unit outside the end nodes
    m = pkg.mesh_box(40, 120, 0, 1.0, 3.0, 1.0, "tanh", 1.5)
    for c, n in ((m.x, 40), (m.y, 120)):
        d = np.diff(c[1:n + 1])
        assert d.min() >= 1.0 - 1e-12
    assert m.x[1] == pytest.approx(0.5) or m.y[1] == pytest.approx(0.5)
