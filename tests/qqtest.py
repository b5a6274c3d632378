"""Shared test helpers: the reference's blocked site map in numpy, random SU(3) gauge
fields and conversions between the reference layout and a lexicographic
(t, z, y, x, spin, colour) complex array.

Site map (G/lattice.f90 siteindex/setblk/gblchker, Q/quark.f90:70-105): for 0-based
global coordinates x_mu = 2*xb_mu + b_mu,
  isite = 1 + xb/2 + yb*nx/4 + zb*nx*ny/8 + tb*nx*ny*nz/16
  ieo   = 1 + (xb+yb+zb+tb) mod 2
  ibl   = 1 + bx + 2 by + 4 bz + 8 bt,  gblclr = 1 + (bx+by+bz+bt) mod 2,
  ibleo = 1 + (ibl-1)//2.
"""
from __future__ import annotations

import numpy as np


def site_map(dims):
    nx, ny, nz, nt = dims
    t, z, y, x = np.meshgrid(np.arange(nt), np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    xb, yb, zb, tb = x >> 1, y >> 1, z >> 1, t >> 1
    bx, by, bz, bt = x & 1, y & 1, z & 1, t & 1
    isite = 1 + (xb >> 1) + yb * (nx // 4) + zb * (nx * ny // 8) + tb * (nx * ny * nz // 16)
    ieo = 1 + ((xb + yb + zb + tb) & 1)
    ibl = 1 + bx + 2 * by + 4 * bz + 8 * bt
    gblclr = 1 + ((bx + by + bz + bt) & 1)
    ibleo = 1 + (ibl - 1) // 2
    return dict(isite=isite, ieo=ieo, ibl=ibl, gblclr=gblclr, ibleo=ibleo)


def random_su3(n, rng, eps=None):
    """n random SU(3) matrices (Haar if eps is None, else exp(i eps H) near 1)."""
    if eps is None:
        z = (rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))) / np.sqrt(2)
        q, r = np.linalg.qr(z)
        d = np.diagonal(r, axis1=1, axis2=2)
        q = q * (d / np.abs(d))[:, None, :]
    else:
        a = rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))
        h = 0.5 * (a + np.conj(np.transpose(a, (0, 2, 1))))
        w, v = np.linalg.eigh(h)
        q = np.einsum("nij,nj,nkj->nik", v, np.exp(1j * eps * w), np.conj(v))
    det = np.linalg.det(q)
    q = q / (det ** (1.0 / 3.0))[:, None, None]
    # re-orthonormalise in FP64 so that row3 = conj(row1 x row2) to ~1e-16
    r1 = q[:, 0] / np.linalg.norm(q[:, 0], axis=1)[:, None]
    r2 = q[:, 1] - np.sum(np.conj(r1) * q[:, 1], axis=1)[:, None] * r1
    r2 = r2 / np.linalg.norm(r2, axis=1)[:, None]
    r3 = np.conj(np.cross(r1, r2))
    return np.stack([r1, r2, r3], axis=1)


def gauge_to_ref(links, dims, ntotal):
    """links: complex (4, nt, nz, ny, nx, 3, 3) -> reference u(18,ntotal,4,2,16)
    as numpy (16, 2, 4, ntotal, 18)."""
    sm = site_map(dims)
    u = np.zeros((16, 2, 4, ntotal, 18))
    ibl = sm["ibl"].ravel() - 1
    ieo = sm["ieo"].ravel() - 1
    isite = sm["isite"].ravel() - 1
    for mu in range(4):
        m = links[mu].reshape(-1, 9)
        u[ibl, ieo, mu, isite, 0::2] = m.real
        u[ibl, ieo, mu, isite, 1::2] = m.imag
    return u


def random_gauge(dims, ntotal, seed=1, eps=None):
    rng = np.random.default_rng(seed)
    nx, ny, nz, nt = dims
    V = nx * ny * nz * nt
    links = random_su3(4 * V, rng, eps).reshape(4, nt, nz, ny, nx, 3, 3)
    return links, gauge_to_ref(links, dims, ntotal)


def half_to_lex(g, dims, gblclr):
    """Reference half-vector -> complex (nt,nz,ny,nx,4,3), zero on the other parity."""
    sm = site_map(dims)
    out = np.zeros(tuple(reversed(dims)) + (4, 3), complex)
    mask = sm["gblclr"] == gblclr
    ibleo = sm["ibleo"][mask] - 1
    ieo = sm["ieo"][mask] - 1
    isite = sm["isite"][mask] - 1
    vals = g[ibleo, ieo, :, isite, :]  # (n, 4, 6)
    out[mask] = vals[..., 0::2] + 1j * vals[..., 1::2]
    return out


def lex_to_half(psi, dims, ntotal, gblclr):
    sm = site_map(dims)
    g = np.zeros((8, 2, 4, ntotal, 6))
    mask = sm["gblclr"] == gblclr
    ibleo = sm["ibleo"][mask] - 1
    ieo = sm["ieo"][mask] - 1
    isite = sm["isite"][mask] - 1
    v = psi[mask]  # (n, 4, 3)
    tmp = np.zeros(v.shape[:2] + (6,))
    tmp[..., 0::2] = v.real
    tmp[..., 1::2] = v.imag
    g[ibleo, ieo, :, isite, :] = tmp
    return g


def random_half(ntotal, nvhalf, seed):
    rng = np.random.default_rng(seed)
    g = np.zeros((8, 2, 4, ntotal, 6))
    g[:, :, :, :nvhalf, :] = rng.standard_normal((8, 2, 4, nvhalf, 6))
    return g


# Dirac matrices of Q/diracops.f90:61-71
I = 1j
GAMMA = [
    np.array([[0, 0, 0, 1], [0, 0, 1, 0], [0, 1, 0, 0], [1, 0, 0, 0]], complex),
    np.array([[0, 0, 0, -I], [0, 0, I, 0], [0, -I, 0, 0], [I, 0, 0, 0]], complex),
    np.array([[0, 0, 1, 0], [0, 0, 0, -1], [1, 0, 0, 0], [0, -1, 0, 0]], complex),
    np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, -1, 0], [0, 0, 0, -1]], complex),
]
GAMMA5 = GAMMA[0] @ GAMMA[1] @ GAMMA[2] @ GAMMA[3]


def hop_lex(links, psi, bc, c1=(1, 1, 1, 1), c2=(1, 1, 1, 1), idag=0):
    """Full-lattice hopping term H psi in numpy (independent of the oracle):
    (H psi)(x) = sum_mu (c1 - s c2 g_mu) U_mu(x) psi(x+mu) + (c1 + s c2 g_mu) U_mu(x-mu)^+ psi(x-mu),
    s = +1 (idag = 0) or -1 (idag = 1); bc(mu) multiplies hops across the boundary."""
    out = np.zeros_like(psi)
    s = 1 if idag == 0 else -1
    axes = {0: 3, 1: 2, 2: 1, 3: 0}  # mu -> array axis of (t,z,y,x)
    for mu in range(4):
        ax = axes[mu]
        n = psi.shape[ax]
        U = links[mu]
        fwd = np.roll(psi, -1, axis=ax)
        sl = [slice(None)] * 4
        sl[ax] = n - 1
        fwd[tuple(sl)] *= bc[mu]
        Up = np.einsum("...ab,...sb->...sa", U, fwd)
        P = c1[mu] * np.eye(4) - s * c2[mu] * GAMMA[mu]
        out += np.einsum("st,...ta->...sa", P, Up)
        bwd = np.roll(psi, 1, axis=ax)
        Ub = np.roll(U, 1, axis=ax)
        sl[ax] = 0
        bwd[tuple(sl)] *= bc[mu]
        Um = np.einsum("...ba,...sb->...sa", np.conj(Ub), bwd)
        P = c1[mu] * np.eye(4) + s * c2[mu] * GAMMA[mu]
        out += np.einsum("st,...ta->...sa", P, Um)
    return out


def su3_gram_schmidt(n, rng, eps=None):
    """n SU(3) matrices from Gram-Schmidt on Gaussian complex matrices (near 1 when eps
    is given).  Elementwise arithmetic only -- no LAPACK -- so the fields are
    bit-reproducible on any machine, as the golden fixtures need."""
    a = rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))
    if eps is not None:
        a = np.eye(3)[None] + eps * a
    r1 = a[:, 0] / np.sqrt(np.sum((a[:, 0] * np.conj(a[:, 0])).real, axis=1))[:, None]
    r2 = a[:, 1] - np.sum(np.conj(r1) * a[:, 1], axis=1)[:, None] * r1
    r2 = r2 / np.sqrt(np.sum((r2 * np.conj(r2)).real, axis=1))[:, None]
    r3 = np.conj(np.cross(r1, r2))
    return np.stack([r1, r2, r3], axis=1)


def golden_gauge(dims, ntotal, seed, eps=0.5):
    """Seeded, machine-independent gauge field: (links (4,nt,nz,ny,nx,3,3), u_ref)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz, nt = dims
    links = su3_gram_schmidt(4 * nx * ny * nz * nt, rng, eps).reshape(4, nt, nz, ny, nx, 3, 3)
    return links, gauge_to_ref(links, dims, ntotal)


def interior_basis(nvhalf):
    """Index tuples (ibleo, ieo, id, isite, icri) of the real slot of every complex
    interior component of a half-vector, in C order."""
    ib, ie, idd, isite, ic = np.meshgrid(np.arange(8), np.arange(2), np.arange(4), np.arange(nvhalf),
                                         np.arange(3), indexing="ij")
    return ib.ravel(), ie.ravel(), idd.ravel(), isite.ravel(), 2 * ic.ravel()


def half_to_vec(g, nvhalf):
    """Interior entries of a half-vector as one complex vector (interior_basis order)."""
    v = g[:, :, :, :nvhalf, :]
    return (v[..., 0::2] + 1j * v[..., 1::2]).ravel()


def vec_to_half(v, ntotal, nvhalf):
    g = np.zeros((8, 2, 4, ntotal, 6))
    c = v.reshape(8, 2, 4, nvhalf, 3)
    g[:, :, :, :nvhalf, 0::2] = c.real
    g[:, :, :, :nvhalf, 1::2] = c.imag
    return g
