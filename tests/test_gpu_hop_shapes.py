"""GPU parity of every hopping-kernel shape against the oracle's FP64 Hsingle
(Q/diracops.f90:554-599), through qq_hsingle_block: nrhs half vectors converted to one
RHS-interleaved block field in FP32, FP16 or BF16, multiplied by the forced kernel shape
with FP32 recon-12 links, and returned in FP64.

Tolerances (max-abs error over max-abs value, interior sites): 5e-6 for FP32 (inputs,
links and accumulation rounded to 24-bit mantissas, eight terms per site), 2e-3 for
FP16 (11 significant bits against a per-site FP32 norm) and 1.5e-2 for BF16 (8
significant bits against the same norm; its rounding 2^-9 of the largest component,
summed over the eight hops, with FP32 arithmetic).

The lattice 8x4x8x12 has V/2 = 1536 sites, so 5 right-hand sides (25 sites per block)
leave the last block partly empty, and 12 or 24 fill blocks of 8 or 16 sites exactly."""
import numpy as np
import pytest

import oracle
from qqtest import random_gauge, random_half

pytestmark = pytest.mark.gpu

DIMS = (8, 4, 8, 12)
BC = (1, 1, 1, -1)

FP32_12 = [0, 1, 2, 4, 64, 128, 202, 203, 204, 301, 302, 303, 304, 305, 306, 307, 308, 309, 310, 311]
FP32_24 = [0, 306, 307, 308, 309, 310, 311]
FP32_1 = [1, 2, 4, 32, 128, 301, 304, 306, 307, 308, 309, 310, 311]
FP32_5 = [1, 301, 304, 306, 307, 308, 309, 310, 311]
FP16_12 = [1, 2, 64, 202, 203, 204]
BF16_12 = [1, 2, 64, 202, 203, 204]


@pytest.fixture(scope="module")
def pair():
    import baylorlqcd_b200 as qq

    ol = oracle.OracleLattice(*DIMS, bc=BC)
    _, u = random_gauge(DIMS, ol.ntotal, seed=5)
    ol.set_gauge(u)
    lat = qq.Lattice(*DIMS, bc=BC)
    lat.gauge_upload(u, recon=12)
    yield ol, lat
    lat.close()


def check(ol, lat, precision, nrhs, shape, idag, gblclr, tol):
    nv = ol.nvhalf
    gin = np.stack([random_half(ol.ntotal, nv, seed=100 + 7 * k) for k in range(nrhs)])
    out = lat.hsingle_block(gin, idag, gblclr, precision=precision, shape=shape)
    for k in range(nrhs):
        ref = ol.hsingle(gin[k], idag, gblclr)
        err = np.abs(out[k][:, :, :, :nv] - ref[:, :, :, :nv]).max() / np.abs(ref[:, :, :, :nv]).max()
        assert err < tol, (k, err)


@pytest.mark.parametrize("idag,gblclr", [(0, 1), (1, 2)])
@pytest.mark.parametrize("shape", FP32_12)
def test_fp32_block12(pair, shape, idag, gblclr):
    check(*pair, 32, 12, shape, idag, gblclr, 5e-6)


@pytest.mark.parametrize("shape", FP32_24)
def test_fp32_block24(pair, shape):
    check(*pair, 32, 24, shape, 1, 2, 5e-6)


@pytest.mark.parametrize("shape", FP32_1)
def test_fp32_single(pair, shape):
    check(*pair, 32, 1, shape, 0, 2, 5e-6)


@pytest.mark.parametrize("shape", FP32_5)
def test_fp32_block5_ragged(pair, shape):
    check(*pair, 32, 5, shape, 1, 1, 5e-6)


@pytest.mark.parametrize("shape", FP16_12)
def test_fp16_block12(pair, shape):
    check(*pair, 16, 12, shape, 0, 1, 2e-3)


@pytest.mark.parametrize("shape", BF16_12)
def test_bf16_block12(pair, shape):
    check(*pair, -16, 12, shape, 1, 2, 1.5e-2)


def test_bf16_single(pair):
    check(*pair, -16, 1, 1, 0, 1, 1.5e-2)


def test_unsupported_shape_is_an_error(pair):
    import baylorlqcd_b200 as qq

    ol, lat = pair
    gin = np.stack([random_half(ol.ntotal, ol.nvhalf, seed=3) for _ in range(5)])
    with pytest.raises(qq.QQError, match="BAD_ARG"):
        lat.hsingle_block(gin, 0, 1, precision=32, shape=305)  # staged links need >= 8 RHS
    with pytest.raises(qq.QQError, match="BAD_ARG"):
        lat.hsingle_block(gin, 0, 1, precision=16, shape=301)  # packed FP32 kernel
    with pytest.raises(qq.QQError, match="BAD_ARG"):
        lat.hsingle_block(gin, 0, 1, precision=32, shape=312)  # no such shape
