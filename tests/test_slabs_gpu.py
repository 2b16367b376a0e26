"""A cavity split into slabs (lbm_create_slab + the per-step ghost exchange;
rows in 2D, z-slices in 3D) must evolve exactly as the whole cavity: in exact
mode the fields are bit-identical, through both step kernels; the combined
check and Nusselt sums agree to rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def whole_and_slabs(pkg, nslabs, kernel, storage="f64", steps=60, shape=(300, 120), mode="exact"):
    nx, ny = shape
    m = pkg.lbm.mesh_box(nx, ny, 0, 1.0, ny / nx, 1.0, "tanh", 1.5)
    c = pkg.Cavity(2, nx, ny, Ra=1e5, Pr=0.71, coords=m, mode=mode, storage=storage, kernel=kernel)
    c.initial()
    c.step(steps)
    dom = pkg.slabs.Domain(nx, ny, Ra=1e5, Pr=0.71, coords=m, mode=mode, storage=storage)
    s = pkg.slabs.Slabs(dom, nslabs, kernel=kernel)
    s.initial()
    s.step(steps)
    return c, s


@pytest.mark.parametrize("kernel", ["direct", "march"])
@pytest.mark.parametrize("nslabs", [2, 3])
def test_slabs_match_the_whole_cavity_bitwise(pkg, nslabs, kernel):
    c, s = whole_and_slabs(pkg, nslabs, kernel)
    assert all(sl.kernel == kernel for sl in s.slabs)
    want, got = c.macro(), s.macro()
    for k in want:
        assert np.array_equal(got[k], want[k]), k
    eu, et = c.check()
    su, st = s.check()
    assert abs(su - eu) <= 1e-12 * eu and abs(st - et) <= 1e-12 * et
    nh, nc = c.nusselt()
    sh, sc = s.nusselt()
    assert abs(sh - nh) <= 1e-12 * abs(nh) and abs(sc - nc) <= 1e-12 * abs(nc)
    s.close()
    c.close()


def test_fp32_slabs_match_the_whole_cavity(pkg):
    # FP32 storage runs the fast build only; its node arithmetic is the same in
    # a slab as in the whole cavity, so the fields are still identical
    c, s = whole_and_slabs(pkg, 2, "march", storage="f32", steps=40, mode="fast")
    want, got = c.macro(), s.macro()
    for k in want:
        assert np.array_equal(got[k], want[k]), k
    s.close()
    c.close()


def test_halo_calls_reject_walls(pkg):
    dom = pkg.slabs.Domain(64, 40, mode="exact")
    s = pkg.slabs.Slabs(dom, 2)
    s.initial()
    lo, hi = s.slabs
    buf = lo.halo_buffer()
    with pytest.raises(pkg.LBMError):
        lo.pack(0, buf)         # the bottom wall: no neighbour below
    with pytest.raises(pkg.LBMError):
        hi.unpack(1, buf)       # the top wall
    lo.pack(1, buf)
    s.close()


def whole_and_slabs3d(pkg, nslabs, kernel, storage="f64", steps=30, shape=(40, 36, 30), mode="exact"):
    nx, ny, nz = shape
    m = pkg.lbm.mesh_box(nx, ny, nz, 1.0, ny / nx, nz / nx, "tanh", 1.5)
    c = pkg.Cavity(3, nx, ny, nz, Ra=1e5, Pr=0.71, coords=m, mode=mode, storage=storage, kernel=kernel)
    c.initial()
    c.step(steps)
    dom = pkg.slabs.Domain(nx, ny, nz, Ra=1e5, Pr=0.71, coords=m, mode=mode, storage=storage)
    s = pkg.slabs.Slabs(dom, nslabs, kernel=kernel)
    s.initial()
    s.step(steps)
    return c, s


@pytest.mark.parametrize("kernel", ["direct", "march"])
@pytest.mark.parametrize("nslabs", [2, 3])
def test_3d_slabs_match_the_whole_cavity_bitwise(pkg, nslabs, kernel):
    c, s = whole_and_slabs3d(pkg, nslabs, kernel)
    assert all(sl.kernel == kernel for sl in s.slabs)
    assert [sl.nz for sl in s.slabs][0] == s.rows[0][1] + 1  # own z-slices plus one ghost slice
    want, got = c.macro(), s.macro()
    assert set(got) == {"rho", "u", "v", "w", "T"}
    for k in want:
        assert np.array_equal(got[k], want[k]), k
    eu, et = c.check()
    su, st = s.check()
    assert abs(su - eu) <= 1e-12 * eu and abs(st - et) <= 1e-12 * et
    nh, nc = c.nusselt()
    sh, sc = s.nusselt()
    assert abs(sh - nh) <= 1e-12 * abs(nh) and abs(sc - nc) <= 1e-12 * abs(nc)
    mass, energy = c.sums()
    sm = sum(sl.sums()[0] for sl in s.slabs)
    assert abs(sm - mass) <= 1e-12 * abs(mass)
    s.close()
    c.close()


def test_3d_fp32_slabs_match_the_whole_cavity(pkg):
    c, s = whole_and_slabs3d(pkg, 2, "march", storage="f32", steps=20, mode="fast")
    want, got = c.macro(), s.macro()
    for k in want:
        assert np.array_equal(got[k], want[k]), k
    s.close()
    c.close()
