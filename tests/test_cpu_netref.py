"""CPU checks of the learned preconditioner's numpy restatement (netref.py), the
reference the GPU network is tested against: a layer's adjoint is its adjoint, every
layer commutes with gauge transformations, and the Wirtinger gradient of the loss
matches central finite differences."""
import numpy as np

import netref
from qqtest import random_su3

DIMS = (4, 4, 4, 4)
BC = (1, 1, 1, -1)


def setup(seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz, nt = DIMS
    V = nx * ny * nz * nt
    links = random_su3(4 * V, rng).reshape(4, nt, nz, ny, nx, 3, 3)

    def rc(*s):
        return rng.standard_normal(s) + 1j * rng.standard_normal(s)

    return rng, links, rc


def test_adjoint():
    rng, links, rc = setup(0)
    nx, ny, nz, nt = DIMS
    W, f, g = rc(9, 3, 2), rc(nt, nz, ny, nx, 2, 3), rc(nt, nz, ny, nx, 3, 3)
    lhs = np.vdot(g, netref.layer(W, links, f, BC))
    rhs = np.vdot(netref.layer_adjoint(W, links, g, BC), f)
    assert abs(lhs - rhs) / abs(lhs) < 1e-13


def test_gauge_covariance():
    rng, links, rc = setup(1)
    nx, ny, nz, nt = DIMS
    V = nx * ny * nz * nt
    W, f = rc(9, 3, 2), rc(nt, nz, ny, nx, 2, 3)
    G = random_su3(V, rng).reshape(nt, nz, ny, nx, 3, 3)
    lt = np.empty_like(links)
    for mu in range(4):
        lt[mu] = np.einsum("...ab,...bc,...dc->...ad", G, links[mu], np.conj(netref._shift(G, mu, 1)))
    ft = np.einsum("...ab,...cb->...ca", G, f)
    o1 = np.einsum("...ab,...cb->...ca", G, netref.layer(W, links, f, BC))
    assert np.abs(o1 - netref.layer(W, lt, ft, BC)).max() < 1e-12


def test_gradient_finite_differences():
    rng, links, rc = setup(2)
    nx, ny, nz, nt = DIMS
    Ws = [0.3 * rc(9, 4, 4), 0.3 * rc(9, 4, 4)]
    bs = [rc(nt, nz, ny, nx, 4, 3) for _ in range(2)]
    xs = [rc(nt, nz, ny, nx, 4, 3) for _ in range(2)]
    _, grads = netref.loss_grad(Ws, links, bs, xs, BC)
    for l in range(2):
        E, eps = rc(9, 4, 4), 1e-6

        def loss(W1):
            W = list(Ws)
            W[l] = W1
            return netref.loss_grad(W, links, bs, xs, BC)[0]

        fd = (loss(Ws[l] + eps * E) - loss(Ws[l] - eps * E)) / (2 * eps)
        an = 2 * np.real(np.vdot(grads[l], E))
        assert abs(fd - an) / abs(an) < 1e-7
