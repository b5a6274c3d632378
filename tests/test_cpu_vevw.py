"""CPU checks of the oracle's restatement of the Wilson loop driver's vacuum values
(oracle/vevw.cpp: vev, Q/disconloops.f90:4653-5339).

1. The average plaquette it returns equals aveplaq (G/gaugetools.f90:1436-1474, the
   oracle's oq_aveplaq) to 1e-14 on a heatbath configuration; the restated site
   enumeration agrees with the pointsource site map (the routine checks it).
2. Unit links: every plaquette is the unit matrix, Re Tr P = 3 and Im Tr P = 0, so the
   scalar loop is -(8 + 4 (+ 4)) 8 kappa^4 (3 * 3 V3) per slice in closed form and every
   current vanishes.
3. An independent numpy statement on random SU(3) links (lexicographic arrays, np.roll
   neighbours, the trig weights at the plaquette's four corners): Jvev to 1e-12 of its
   largest entry for two momentum origins and two lattice shapes, plaq and psi to 1e-13."""
import numpy as np
import pytest

import oracle
from qqtest import random_gauge

TWO_PI = float(np.float32(6.283185307179586))  # the reference's default-kind literal
AX = (3, 2, 1, 0)  # array axis of direction mu in (nt, nz, ny, nx)


def dag(a):
    return np.conj(np.swapaxes(a, -1, -2))


def vev_numpy(links, dims, kappa, io):
    """Jvev (5 op, 5 mom, nt, 2), plaq, psi from lexicographic links (4, nt, nz, ny, nx, 3, 3)."""
    nx, ny, nz, nt = dims
    n = (nx, ny, nz)
    coords = [np.arange(nx)[None, None, None, :], np.arange(ny)[None, None, :, None],
              np.arange(nz)[None, :, None, None]]

    def trig(a, shift):
        arg = (coords[a] + 1 + shift - io[a]).astype(float)
        return {"c": np.cos(TWO_PI * arg / n[a]), "s": np.sin(TWO_PI * arg / n[a]),
                "c2": np.cos(TWO_PI * (2 * arg) / n[a]), "s2": np.sin(TWO_PI * (2 * arg) / n[a])}

    def slices(a):
        return np.broadcast_to(a, (nt, nz, ny, nx)).sum(axis=(1, 2, 3))

    S = {k: np.zeros(nt) for k in ("t", "s", "j1t", "j2t", "j3t")}
    for k in ("mt", "ms", "j4", "j12s", "j13s", "j21s", "j23s", "j31s", "j32s",
              "j12t", "j13t", "j21t", "j23t", "j31t", "j32t"):
        S[k] = np.zeros((4, nt))
    for mu in range(3):
        for nu in range(mu + 1, 4):
            U = links
            P = U[mu] @ np.roll(U[nu], -1, axis=AX[mu]) @ dag(np.roll(U[mu], -1, axis=AX[nu])) @ dag(U[nu])
            tr = np.trace(P, axis1=-2, axis2=-1)
            re, im = tr.real, tr.imag
            corner = []
            for v in range(4):
                corner.append([trig(a, int(((v & 1) and a == mu) or ((v & 2) and a == nu))) for a in range(3)])

            def cosw(q):
                c = [q[a]["c"] for a in range(3)]
                return ((c[0] + c[1] + c[2]) / 3.0, (c[0] * c[1] + c[0] * c[2] + c[1] * c[2]) / 3.0,
                        c[0] * c[1] * c[2], (q[0]["c2"] + q[1]["c2"] + q[2]["c2"]) / 3.0)

            def sinw(q, a):
                b, c = [x for x in range(3) if x != a]
                return (q[a]["s"], q[a]["s"] * (q[b]["c"] + q[c]["c"]) / 2.0, q[a]["s"] * q[b]["c"] * q[c]["c"],
                        q[a]["s2"])

            def acc(key, ws, w):
                for i in range(4):
                    S[key][i] += slices(ws[i] * w)

            S["t" if nu == 3 else "s"] += slices(re)
            cw = [cosw(q) for q in corner]
            acc("mt" if nu == 3 else "ms", [sum(cw[v][i] for v in range(4)) for i in range(4)], re)
            if nu == 3:
                acc("j4", [cw[0][i] - cw[1][i] for i in range(4)], -im)
            c0 = corner[0]
            X, Y, Z = 0, 1, 2
            if nu == 3:
                S[("j1t", "j2t", "j3t")[mu]] += slices(im)
                pair = {0: (("j13t", Z), ("j12t", Y)), 1: (("j21t", X), ("j23t", Z)),
                        2: (("j32t", Y), ("j31t", X))}[mu]
                for key, a in pair:
                    acc(key, sinw(c0, a), im)
            diff = lambda v, a: [x - y for x, y in zip(sinw(c0, a), sinw(corner[v], a))]  # noqa: E731
            if mu == 0 and nu != 3:
                acc("j13s", diff(2, Z), im)
                acc("j12s", diff(2, Y), im)
            if mu == 1 and nu == 2:
                acc("j21s", diff(2, X), im)
                acc("j23s", diff(2, Z), im)
            elif mu == 0 and nu == 1:
                acc("j21s", diff(1, X), -im)
                acc("j23s", diff(1, Z), -im)
            if nu == 2:
                acc("j32s", diff(1, Y), -im)
                acc("j31s", diff(1, X), -im)
    V = nx * ny * nz * nt
    plaq = (S["t"].sum() + S["s"].sum()) / (18 * V)
    f = 8.0 * kappa ** 4
    t, s = S["t"] * 4 * f, S["s"] * 8 * f
    sc = {k: S[k] * 2 * f for k in S if k not in ("t", "s", "mt", "ms")}
    mt, ms = S["mt"] * f, S["ms"] * 2 * f
    psi = (s.sum() + t.sum() + t[:-1].sum()) / V
    J = np.zeros((5, 5, nt, 2))  # [op, mom, t, ri]

    def prev(a):  # a(t - 1), zero before the first slice
        out = np.zeros_like(a)
        out[..., 1:] = a[..., :-1]
        return out

    J[4, 0, :, 0] = s + t + prev(t)
    J[4, 1:, :, 0] = ms + mt + prev(mt)
    J[3, 1:, :, 1] = sc["j4"]
    for op, key in enumerate(("j1t", "j2t", "j3t")):
        J[op, 0, :, 1] = sc[key] - prev(sc[key])
    for op, ri, ks, kt in ((0, 0, "j13s", "j13t"), (0, 1, "j21s", "j21t"), (1, 0, "j32s", "j32t"),
                           (1, 1, "j12s", "j12t"), (2, 0, "j23s", "j23t"), (2, 1, "j31s", "j31t")):
        J[op, 1:, :, ri] = sc[ks] + sc[kt] - prev(sc[kt])
    return -J, plaq, psi


def test_plaquette_matches_aveplaq():
    dims = (4, 4, 4, 8)
    ol = oracle.OracleLattice(*dims, bc=(1, 1, 1, -1))
    u = ol.coldstart()
    oracle.initlagfib(0, 7)
    ol.heatbath(u, 5.8, 10)
    ol.set_gauge(u)
    _, plaq, _ = ol.vev(0.15)
    assert abs(plaq - ol.aveplaq(u)) < 1e-14


def test_unit_links_closed_form():
    dims = (4, 4, 8, 4)
    ol = oracle.OracleLattice(*dims, bc=(1, 1, 1, -1))
    ol.set_gauge(ol.coldstart())
    kappa = 0.15
    J, plaq, psi = ol.vev(kappa, io=(2, 1, 3))
    v3 = dims[0] * dims[1] * dims[2]
    f = 8 * kappa ** 4
    tsum, ssum = 9 * v3 * 4 * f, 9 * v3 * 8 * f
    assert plaq == pytest.approx(1.0, abs=1e-15)
    np.testing.assert_allclose(J[4, 0, 0, 0], -(tsum + ssum), rtol=1e-14)
    np.testing.assert_allclose(J[4, 0, 1:, 0], -(2 * tsum + ssum), rtol=1e-14)
    assert np.abs(J[:, :, :, 1]).max() < 1e-12  # every current: Im Tr P = 0
    assert np.abs(J[:3, :, :, 0]).max() < 1e-12
    assert psi == pytest.approx((dims[3] * (tsum + ssum) + (dims[3] - 1) * tsum) / (v3 * dims[3]), rel=1e-14)


@pytest.mark.parametrize("dims,io,seed", [((4, 4, 4, 8), (1, 1, 1), 3), ((8, 4, 4, 4), (2, 4, 3), 4)])
def test_against_numpy(dims, io, seed):
    ol = oracle.OracleLattice(*dims, bc=(1, 1, 1, -1))
    links, u = random_gauge(dims, ol.ntotal, seed=seed)
    ol.set_gauge(u)
    kappa = 0.1565
    J, plaq, psi = ol.vev(kappa, io=io)
    Jn, plaq_n, psi_n = vev_numpy(links, dims, kappa, io)
    assert np.abs(J - Jn).max() <= 1e-12 * np.abs(Jn).max()
    assert abs(plaq - plaq_n) <= 1e-13 and abs(psi - psi_n) <= 1e-13 * abs(psi_n)
    assert np.abs(J[:3, 1:]).max() > 1e-6 * np.abs(J).max()  # the momentum currents are exercised
