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
