"""qq_vecdot_noalloc: vecdot from device-resident reference-layout half-vectors with
no device allocation.  Compared with qq_vecdot on the same inputs (tolerance 1e-13
relative: both sum in FP64, in different orders) and with a numpy sum over the
interior sites.  Collected last so it also runs after every other GPU test."""
import numpy as np
import pytest

from qqtest import random_half

pytestmark = pytest.mark.gpu

TOL = 1e-13


@pytest.fixture(scope="module", params=[(4, 4, 4, 8), (8, 8, 8, 16)], ids=["4x4x4x8", "8x8x8x16"])
def lat(request):
    import baylorlqcd_b200 as qq

    lat = qq.Lattice(*request.param, bc=(1, 1, 1, -1))
    yield lat
    lat.close()


def numpy_vecdot(a, b, nvhalf):
    ca = a[:, :, :, :nvhalf, 0::2] + 1j * a[:, :, :, :nvhalf, 1::2]
    cb = b[:, :, :, :nvhalf, 0::2] + 1j * b[:, :, :, :nvhalf, 1::2]
    return np.vdot(ca.ravel(), cb.ravel())


def test_matches_vecdot_twice(lat):
    import torch

    a = random_half(lat.ntotal, lat.nvhalf, 81)
    b = random_half(lat.ntotal, lat.nvhalf, 82)
    a[:, :, :, lat.nvhalf:, :] = 1e6  # halo slots are scratch and must not count
    b[:, :, :, lat.nvhalf:, :] = -3e5
    ref = lat.vecdot(a, b)
    ad, bd = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    first = lat.vecdot_noalloc(ad, bd)
    second = lat.vecdot_noalloc(ad, bd)
    for out in (first, second):
        assert abs(out - ref) / abs(ref) < TOL
    assert first == second  # fixed reduction order
    assert abs(first - numpy_vecdot(a, b, lat.nvhalf)) / abs(ref) < TOL
    # <a, a> is real and positive
    aa = lat.vecdot_noalloc(ad, ad)
    assert abs(aa.imag) < 1e-12 * aa.real and aa.real > 0


def test_no_device_memory_taken(lat):
    import torch

    a = torch.from_numpy(random_half(lat.ntotal, lat.nvhalf, 83)).cuda()
    b = torch.from_numpy(random_half(lat.ntotal, lat.nvhalf, 84)).cuda()
    lat.vecdot_noalloc(a, b)  # first call on the device does the one-time setup
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        lat.vecdot_noalloc(a, b)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_rejects_host_arrays(lat):
    import baylorlqcd_b200 as qq

    a = random_half(lat.ntotal, lat.nvhalf, 85)
    with pytest.raises(qq.QQError) as e:
        lat.vecdot_noalloc(a, a)
    assert e.value.status == qq.QQ_BAD_ARG


def test_rejects_oversized_lattice():
    """32^3 x 160 = 5,242,880 sites exceeds the 4,194,304-site scratch bound; the
    check comes before any pointer is read, so small tensors suffice."""
    import torch

    import baylorlqcd_b200 as qq

    big = qq.Lattice(32, 32, 32, 160)
    try:
        t = torch.zeros(16, dtype=torch.float64, device="cuda")
        with pytest.raises(qq.QQError) as e:
            big.vecdot_noalloc(t, t)
        assert e.value.status == qq.QQ_BAD_ARG
        assert "4194304" in str(e.value)
    finally:
        big.close()
