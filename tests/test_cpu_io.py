"""Gauge and propagator files in the reference's Fortran unformatted formats
(G/gaugetools.f90 GFwrite/GFread :1260-1334, fixsu3 :1338-1432; Q/quark.f90
FPwrite/FPread :3379-3481), through the C ABI on the host.  The byte layout is
checked against an independent numpy reading of the records."""
import numpy as np
import pytest

import baylorlqcd_b200 as qq
import oracle
from qqtest import golden_gauge, random_half

DIMS = (4, 4, 4, 8)
VECBLINV = [[1, 2, 2, 1, 2, 1, 1, 2, 2, 1, 1, 2, 1, 2, 2, 1], [1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8]]


@pytest.fixture(scope="module")
def geom():
    ol = oracle.OracleLattice(*DIMS)
    return ol.nvhalf, ol.ntotal


def records(path):
    raw = open(path, "rb").read()
    out, i = [], 0
    while i < len(raw):
        n = int(np.frombuffer(raw, np.int32, 1, i)[0])
        out.append(raw[i + 4:i + 4 + n])
        assert int(np.frombuffer(raw, np.int32, 1, i + 4 + n)[0]) == n
        i += 8 + n
    return out


def test_gauge_roundtrip_and_layout(tmp_path, geom):
    nvhalf, ntotal = geom
    _, u = golden_gauge(DIMS, ntotal, seed=3, eps=0.7)  # exact SU(3): fixsu3 changes it only by rounding
    u0 = u.copy()
    path = tmp_path / "cfg.dat"
    qq.gfwrite(path, u, nvhalf, gaction=(1, 1, 1, 2), beta=5.9, alat=(1, 1, 1, 2.5), tad=(0.9, 0.9, 0.9, 0.8),
               icfgsave=17, myid=0)
    assert np.abs(u - u0).max() < 1e-14
    rec = records(path)
    assert len(rec) == 12 * nvhalf * 16 + 1 and all(len(r) == 64 for r in rec[:-1]) and len(rec[-1]) == 96
    # record (icri, isite, ibl) holds (u(icri,isite,mu,1,ibl), u(icri,isite,mu,2,ibl), mu=1..4)
    for icri, isite, ibl in [(1, 1, 1), (5, 3, 9), (12, nvhalf, 16)]:
        k = ((icri - 1) * nvhalf + (isite - 1)) * 16 + (ibl - 1)
        want = [u[ibl - 1, ieo, mu, isite - 1, icri - 1] for mu in range(4) for ieo in range(2)]
        assert np.array_equal(np.frombuffer(rec[k], np.float64), want)
    assert tuple(np.frombuffer(rec[-1][:16], np.int32)) == (1, 1, 1, 2)
    u2, hdr = qq.gfread(path, nvhalf, ntotal)
    assert hdr == dict(gaction=(1, 1, 1, 2), beta=5.9, alat=(1, 1, 1, 2.5), tad=(0.9, 0.9, 0.9, 0.8), icfgsave=17,
                       myid=0)
    assert np.abs(u2[:, :, :, :nvhalf] - u[:, :, :, :nvhalf]).max() < 1e-14  # row 3 rebuilt by fixsu3


def test_fixsu3_repairs_rows(tmp_path, geom):
    """A perturbed field comes back special unitary: row 1 and 2 orthonormalised, row 3 =
    conj(row1 x row2)."""
    nvhalf, ntotal = geom
    _, u = golden_gauge(DIMS, ntotal, seed=4, eps=0.7)
    u[:, :, :, :nvhalf, :12] += 1e-3 * np.random.default_rng(1).standard_normal(u[:, :, :, :nvhalf, :12].shape)
    path = tmp_path / "cfg.dat"
    qq.gfwrite(path, u, nvhalf)
    v, _ = qq.gfread(path, nvhalf, ntotal)
    m = v[:, :, :, :nvhalf].reshape(-1, 9, 2)
    m = (m[..., 0] + 1j * m[..., 1]).reshape(-1, 3, 3)
    assert np.abs(np.einsum("nij,nkj->nik", m, m.conj()) - np.eye(3)).max() < 1e-14
    assert np.abs(np.linalg.det(m) - 1).max() < 1e-14


def test_gfwrite_refuses_existing_file(tmp_path, geom):
    nvhalf, ntotal = geom
    _, u = golden_gauge(DIMS, ntotal, seed=3)
    path = tmp_path / "cfg.dat"
    path.write_bytes(b"x")
    with pytest.raises(qq.QQError) as e:
        qq.gfwrite(path, u, nvhalf)
    assert e.value.status == qq.QQ_BAD_ARG


def test_propagator_roundtrip_and_layout(tmp_path, geom):
    nvhalf, ntotal = geom
    xe, xo = random_half(ntotal, nvhalf, 1), random_half(ntotal, nvhalf, 2)
    path = tmp_path / "prop.dat"
    qq.fpwrite(path, xe, xo, nvhalf, kappa=0.1565, tmqcd=0.005, cSW=0.0, icsrc=2, idsrc=3, icfg=9, myid=0)
    rec = records(path)
    assert len(rec) == nvhalf * 16 * 6 + 1 and len(rec[-1]) == 40
    for isite, ibl, icri in [(1, 1, 1), (2, 6, 4), (nvhalf, 15, 6)]:
        k = ((isite - 1) * 16 + (ibl - 1)) * 6 + (icri - 1)
        x = xe if VECBLINV[0][ibl - 1] == 1 else xo
        ibleo = VECBLINV[1][ibl - 1]
        want = [x[ibleo - 1, ieo, idd, isite - 1, icri - 1] for idd in range(4) for ieo in range(2)]
        assert np.array_equal(np.frombuffer(rec[k], np.float64), want)
    ye, yo, hdr = qq.fpread(path, nvhalf, ntotal)
    assert np.array_equal(ye[:, :, :, :nvhalf], xe[:, :, :, :nvhalf])
    assert np.array_equal(yo[:, :, :, :nvhalf], xo[:, :, :, :nvhalf])
    assert hdr == dict(kappa=0.1565, tmqcd=0.005, cSW=0.0, icsrc=2, idsrc=3, icfg=9, myid=0)


def test_reading_a_file_of_another_size_fails(tmp_path, geom):
    nvhalf, ntotal = geom
    xe, xo = random_half(ntotal, nvhalf, 1), random_half(ntotal, nvhalf, 2)
    path = tmp_path / "prop.dat"
    qq.fpwrite(path, xe, xo, nvhalf)
    with pytest.raises(qq.QQError):
        qq.fpread(path, 2 * nvhalf, 2 * ntotal)
