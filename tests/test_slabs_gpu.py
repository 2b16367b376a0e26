"""A 2D cavity split into row slabs (lbm_create_slab + the per-step ghost-row
exchange) must evolve exactly as the whole cavity: in exact mode the fields
are bit-identical, through both step kernels; the combined check and Nusselt
sums agree to rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def whole_and_slabs(pkg, nslabs, kernel, storage="f64", steps=60, shape=(300, 120)):
    nx, ny = shape
    m = pkg.lbm.mesh_box(nx, ny, 0, 1.0, ny / nx, 1.0, "tanh", 1.5)
    c = pkg.Cavity(2, nx, ny, Ra=1e5, Pr=0.71, coords=m, mode="exact", storage=storage, kernel=kernel)
    c.initial()
    c.step(steps)
    dom = pkg.slabs.Domain(nx, ny, Ra=1e5, Pr=0.71, coords=m, mode="exact", storage=storage)
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
    c, s = whole_and_slabs(pkg, 2, "march", storage="f32", steps=40)
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
