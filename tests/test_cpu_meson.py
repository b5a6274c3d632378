"""The oracle's pionrho (a loop-by-loop restatement of Q/quark.f90:1033-1212 on the
blocked layout) against an independent lexicographic computation: per time slice, the
sum over sites and colours of |x|^2 (pion), of (|x_1|^2 - |x_2|^2 - |x_3|^2 + |x_4|^2)
times rsgn(idsrc) (rho) and of (|x_1|^2 + |x_2|^2 - |x_3|^2 - |x_4|^2) (decay)."""
import numpy as np
import pytest

import oracle
from qqtest import half_to_lex, random_half


@pytest.mark.parametrize("dims", [(4, 4, 4, 8), (8, 4, 4, 12)])
@pytest.mark.parametrize("idsrc", [1, 2, 3, 4])
def test_pionrho_matches_lexicographic(dims, idsrc):
    ol = oracle.OracleLattice(*dims)
    xe = random_half(ol.ntotal, ol.nvhalf, seed=idsrc)
    xo = random_half(ol.ntotal, ol.nvhalf, seed=10 + idsrc)
    pion, rho, decay = ol.pionrho(xe, xo, idsrc)
    full = half_to_lex(xe, dims, 1) + half_to_lex(xo, dims, 2)  # (t, z, y, x, spin, colour)
    sq = np.sum(np.abs(full) ** 2, axis=(1, 2, 3, 5))             # (t, spin)
    rsgn = [1.0, -1.0, -1.0, 1.0][idsrc - 1]
    np.testing.assert_allclose(pion, sq.sum(axis=1), rtol=1e-13)
    np.testing.assert_allclose(rho, rsgn * (sq[:, 0] - sq[:, 1] - sq[:, 2] + sq[:, 3]), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(decay, sq[:, 0] + sq[:, 1] - sq[:, 2] - sq[:, 3], rtol=1e-12, atol=1e-12)


# ---- sink smearing and mesoncorr (oracle/meson.cpp) ----
from qqtest import random_gauge  # noqa: E402

JD2 = [[3, 4, 1, 2], [1, 2, 3, 4], [2, 1, 4, 3], [2, 1, 4, 3], [1, 2, 3, 4], [3, 4, 1, 2], [4, 3, 2, 1],
       [4, 3, 2, 1], [3, 4, 1, 2], [1, 2, 3, 4], [3, 4, 1, 2], [4, 3, 2, 1], [4, 3, 2, 1], [2, 1, 4, 3],
       [2, 1, 4, 3], [1, 2, 3, 4]]
ROOTM1 = [-1, 1, -1, 1, -1, -1, 1, -1, 1, 1, 1, -1, 1, -1, 1, -1]
SGNI = [[-1, -1, 1, 1], [1, 1, 1, 1], [-1, -1, 1, 1], [1, -1, -1, 1], [-1, 1, 1, -1], [1, 1, 1, 1],
        [-1, -1, -1, -1], [1, -1, 1, -1], [-1, 1, -1, 1], [-1, -1, 1, 1], [1, -1, -1, 1], [-1, 1, 1, -1],
        [1, 1, -1, -1], [1, 1, 1, 1], [-1, 1, -1, 1], [1, -1, 1, -1]]
SGNJ = [[1, 1, -1, -1], [1, 1, 1, 1], [1, 1, -1, -1], [-1, 1, 1, -1], [1, -1, -1, 1], [1, 1, 1, 1],
        [1, 1, 1, 1], [-1, 1, -1, 1], [1, -1, 1, -1], [-1, -1, 1, 1], [-1, 1, 1, -1], [1, -1, -1, 1],
        [-1, -1, 1, 1], [1, 1, 1, 1], [-1, 1, -1, 1], [1, -1, 1, -1]]
JOP = [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 6, 2, 3, 4, 5, 7, 8, 9]
IOP = [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 2, 6, 7, 8, 9, 10, 3, 4, 5, 6, 2, 1, 14, 15, 16, 14, 15, 16]


def test_smear_matches_lexicographic():
    """h <- (1 - 6a) h + a sum_{mu<3} [U_mu(x) h(x+mu) + U_mu(x-mu)^+ h(x-mu)], bc across the
    edge, in numpy on the full lattice, two sweeps."""
    dims, bc = (4, 8, 4, 4), (1, -1, 1, -1)
    ol = oracle.OracleLattice(*dims, bc=bc)
    links, u = random_gauge(dims, ol.ntotal, seed=4)
    ol.set_gauge(u)
    ge, go = random_half(ol.ntotal, ol.nvhalf, 5), random_half(ol.ntotal, ol.nvhalf, 6)
    a, n = 0.15, 2
    he, ho = ol.smear(ge, go, a, n)
    h = half_to_lex(ge, dims, 1) + half_to_lex(go, dims, 2)
    axes = {0: 3, 1: 2, 2: 1}
    for _ in range(n):
        acc = np.zeros_like(h)
        for mu in range(3):
            ax, U, L = axes[mu], links[mu], dims[mu]
            fwd = np.roll(h, -1, axis=ax)
            sl = [slice(None)] * 4
            sl[ax] = L - 1
            fwd[tuple(sl)] *= bc[mu]
            acc += np.einsum("...ab,...sb->...sa", U, fwd)
            bwd = np.roll(h, 1, axis=ax)
            Ub = np.roll(U, 1, axis=ax)
            sl[ax] = 0
            bwd[tuple(sl)] *= bc[mu]
            acc += np.einsum("...ba,...sb->...sa", np.conj(Ub), bwd)
        h = (1 - 6 * a) * h + a * acc
    got = half_to_lex(he, dims, 1) + half_to_lex(ho, dims, 2)
    assert np.abs(got - h).max() <= 1e-13 * np.abs(h).max()


def lex_props(cols, dims):
    """S[t,z,y,x, ic, id, jc, jd] from 12 columns (jc-1)*4 + jd-1 of (even, odd) halves."""
    S = np.zeros(tuple(reversed(dims)) + (3, 4, 3, 4), complex)
    for jc in range(3):
        for jd in range(4):
            c = cols[jc * 4 + jd]
            f = half_to_lex(c[0], dims, 1) + half_to_lex(c[1], dims, 2)  # (..., spin, colour)
            S[..., :, :, jc, jd] = np.transpose(f, (0, 1, 2, 3, 5, 4))
    return S


@pytest.mark.parametrize("channels", [0, 1])
def test_mesoncorr_matches_numpy(channels):
    """The contraction, signs and rootm1 rule per operator pair and the momentum sum
    e^{2 pi i p.(x - src)/L}, p in [-4, 4]^3, in vectorised numpy; the P->P channel at
    zero momentum is also the pion correlator sum |S|^2 of pionrho."""
    dims, src = (4, 4, 4, 8), (2, 3, 1, 4)
    ol = oracle.OracleLattice(*dims)
    rng = np.random.default_rng(7)
    q = np.zeros((12, 2) + ol.half_shape)
    qb = np.zeros_like(q)
    q[..., :ol.nvhalf, :] = rng.standard_normal(q[..., :ol.nvhalf, :].shape)
    qb[..., :ol.nvhalf, :] = rng.standard_normal(qb[..., :ol.nvhalf, :].shape)
    re, im = ol.mesoncorr(q, src, qbar=qb, channels=channels)
    S, Sb = lex_props(q, dims), lex_props(qb, dims)
    nt, nz, ny, nx = S.shape[:4]
    ph = []
    for a, n in enumerate((nx, ny, nz)):
        k = np.arange(1, n + 1)
        ph.append(np.exp(2j * np.pi * np.outer(np.arange(-4, 5), k - src[a]) / n))  # (9, n)
    for ii in range(28):
        jop, iop = JOP[ii], IOP[ii]
        want = np.zeros((9, 9, 9, nt), complex)
        if channels == 1 or (jop <= 2 and iop <= 2 and not (jop == 1 and iop == 1)):
            bit = np.zeros((nt, nz, ny, nx), complex)
            for idd in range(4):
                for jd in range(4):
                    a = S[..., :, JD2[iop - 1][idd] - 1, :, jd]           # (..., ic, jc)
                    b = Sb[..., :, idd, :, JD2[jop - 1][jd] - 1]
                    bit += SGNJ[jop - 1][jd] * SGNI[iop - 1][idd] * np.sum(a * np.conj(b), axis=(-2, -1))
            r1, r2 = ROOTM1[jop - 1], ROOTM1[iop - 1]
            if r1 == -1 and r2 == -1:
                bit = -bit
            elif r1 != r2:
                bit = 1j * np.conj(bit)
            # corr[pz, py, px, t]
            want = np.einsum("tzyx,ax,by,cz->cbat", bit, ph[0], ph[1], ph[2])
        got = re[ii] + 1j * im[ii]  # (pz, py, px, t)
        assert np.abs(got - want).max() <= 1e-11 * max(1.0, np.abs(want).max()), ii
    # P->P (ii = 2) of q with itself at p = 0: the pion correlator, sum |S|^2 per slice
    pion = np.sum(np.abs(S) ** 2, axis=(1, 2, 3, 4, 5, 6, 7))
    re2, _ = ol.mesoncorr(q, src, channels=0)
    np.testing.assert_allclose(re2[1, 4, 4, 4], pion, rtol=1e-12)
