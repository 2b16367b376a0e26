"""lbm_check_noalloc, the check() residual for callers that cannot allocate
device memory (a host that keeps every field in device arrays of its own pool
and must not let a library allocate).  Called through the C ABI on device
arrays the test owns, it must agree with lbm_check on the same fields, on two
checks in a row (the second one against the fields the first one stored as
the previous state)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64).ravel()).to("cuda:0")


@pytest.mark.parametrize("dim", [3, 2])
def test_check_noalloc_agrees_with_lbm_check(pkg, dim):
    import torch
    shape = (20, 18, 14) if dim == 3 else (40, 36, 1)
    cav = pkg.Cavity(dim, *shape, Ra=1e5, grid="tanh", stretch=1.5)
    cav.initial()
    n = cav.nnode
    # the previous-check fields start at zero, as lbm_check's do after initial()
    prev = {k: torch.zeros(n, dtype=torch.float64, device="cuda:0") for k in ("u", "v", "w", "T")}
    for it in range(2):
        cav.step(25)
        m = cav.macro()
        cur = {k: _dev(m[k], torch) for k in m}
        torch.cuda.synchronize()
        w = cur["w"].data_ptr() if dim == 3 else None
        wp = prev["w"].data_ptr() if dim == 3 else None
        free0 = torch.cuda.mem_get_info(0)[0]
        eu, et = pkg.check_noalloc(cur["u"].data_ptr(), cur["v"].data_ptr(), w, cur["T"].data_ptr(),
                                   prev["u"].data_ptr(), prev["v"].data_ptr(), wp, prev["T"].data_ptr(), n)
        torch.cuda.synchronize()
        if it > 0:
            # after the first call on the device, whose set-up only looks up the
            # static scratch array's address, a call leaves the device's free
            # memory exactly as it found it
            assert torch.cuda.mem_get_info(0)[0] == free0
        ru, rt = cav.check()
        # same sums, different block partition: equal to rounding
        assert eu == pytest.approx(ru, rel=1e-12, abs=0.0)
        assert et == pytest.approx(rt, rel=1e-12, abs=0.0)
        for k in ("u", "v", "T") + (("w",) if dim == 3 else ()):
            assert torch.equal(prev[k], cur[k]), k
    cav.close()


def test_check_noalloc_rejects_too_many_nodes(pkg):
    with pytest.raises(pkg.LBMError) as e:
        pkg.check_noalloc(1, 1, None, 1, 1, 1, None, 1, pkg.NOALLOC_MAX_NODES + 1)
    assert e.value.status == -1
    assert "scratch limit" in str(e.value)
