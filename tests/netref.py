"""numpy restatement of the learned preconditioner's network, for the GPU tests.

A layer is a gauge-covariant parallel-transport convolution on the full lattice.
Fields are complex arrays (nt, nz, ny, nx, C, 3): C channels, each a colour vector.
Nine paths p transport a field to the site x:
    p = 0           f(x)
    p = 1 + 2 mu    bc * U_mu(x) f(x + mu)             (forward hop)
    p = 2 + 2 mu    bc * U_mu(x - mu)^+ f(x - mu)      (backward hop)
with bc the boundary factor of direction mu on hops that wrap around the lattice.  A
layer with weights W (9, Cout, Cin) maps f to  out_co = sum_p sum_ci W[p, co, ci] T_p f_ci.
Weights act on channels only, never on colour, so every layer commutes with gauge
transformations.  The adjoint of T_{mu+} is T_{mu-}.

The network maps an even-site vector (spin = channel, colour) to an even-site vector:
embed with zeros on odd sites, apply the layers, keep the even sites.

Loss of pairs (b_i, x_i):  l = (1/S) sum_i |N(b_i) - x_i|^2 / |x_i|^2 over even sites;
grad[l][p, co, ci] = dl / d conj(W[l][p, co, ci]) (Wirtinger), so a real step along
-grad lowers l.
"""
from __future__ import annotations

import numpy as np


def _shift(f, mu, d):
    """f(x + d * mu) for fields laid out (t, z, y, x, ...)."""
    return np.roll(f, -d, axis=3 - mu)


def _wrap_mask(dims, mu, d):
    """Sites whose hop by d along mu wraps around the lattice: shape (nt, nz, ny, nx)."""
    nx, ny, nz, nt = dims
    coords = np.meshgrid(np.arange(nt), np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    xm = coords[3 - mu]
    n = dims[mu]
    return (xm == n - 1) if d > 0 else (xm == 0)


def transport(links, f, p, bc):
    """T_p f; links (4, nt, nz, ny, nx, 3, 3), f (nt, nz, ny, nx, C, 3)."""
    if p == 0:
        return f.copy()
    mu, back = (p - 1) // 2, (p - 1) % 2
    dims = (f.shape[3], f.shape[2], f.shape[1], f.shape[0])
    fac = np.where(_wrap_mask(dims, mu, -1 if back else 1), float(bc[mu]), 1.0)
    if not back:
        g = _shift(f, mu, 1)
        out = np.einsum("...ab,...cb->...ca", links[mu], g)
    else:
        g = _shift(f, mu, -1)
        ub = _shift(links[mu], mu, -1)
        out = np.einsum("...ba,...cb->...ca", np.conj(ub), g)
    return out * fac[..., None, None]


def layer(W, links, f, bc):
    out = 0
    for p in range(9):
        out = out + np.einsum("oc,...ca->...oa", W[p], transport(links, f, p, bc))
    return out


def adjoint_weights(W):
    """Weights of the adjoint layer: W'[0] = W[0]^H, W'[mu+] = W[mu-]^H, W'[mu-] = W[mu+]^H."""
    Wa = np.empty((9, W.shape[2], W.shape[1]), complex)
    Wa[0] = np.conj(W[0].T)
    for mu in range(4):
        Wa[1 + 2 * mu] = np.conj(W[2 + 2 * mu].T)
        Wa[2 + 2 * mu] = np.conj(W[1 + 2 * mu].T)
    return Wa


def layer_adjoint(W, links, f, bc):
    return layer(adjoint_weights(W), links, f, bc)


def weight_grad(delta, fin, links, bc):
    """G[p, co, ci] = sum_x sum_a delta[x, co, a] conj((T_p fin)[x, ci, a])."""
    G = np.empty((9, delta.shape[-2], fin.shape[-2]), complex)
    for p in range(9):
        t = transport(links, fin, p, bc)
        G[p] = np.einsum("noa,nca->oc", delta.reshape(-1, *delta.shape[-2:]), np.conj(t.reshape(-1, *t.shape[-2:])))
    return G


def even_mask(dims):
    nx, ny, nz, nt = dims
    t, z, y, x = np.meshgrid(np.arange(nt), np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return ((x + y + z + t) & 1) == 0


def apply(Ws, links, psi_even, bc):
    """Network on a lexicographic even-site spinor (nt, nz, ny, nx, 4, 3), odd sites zero."""
    dims = (psi_even.shape[3], psi_even.shape[2], psi_even.shape[1], psi_even.shape[0])
    f = psi_even * even_mask(dims)[..., None, None]
    for W in Ws:
        f = layer(W, links, f, bc)
    return f * even_mask(dims)[..., None, None]


def loss_grad(Ws, links, bs, xs, bc):
    """Loss and Wirtinger gradients over pairs (lexicographic even-site spinors)."""
    dims = (bs[0].shape[3], bs[0].shape[2], bs[0].shape[1], bs[0].shape[0])
    mask = even_mask(dims)[..., None, None]
    S = len(bs)
    loss = 0.0
    grads = [np.zeros_like(W) for W in Ws]
    for b, x in zip(bs, xs):
        acts = [b * mask]
        for W in Ws:
            acts.append(layer(W, links, acts[-1], bc))
        r = (acts[-1] - x) * mask
        nx2 = np.sum(np.abs(x * mask) ** 2)
        loss += np.sum(np.abs(r) ** 2) / nx2 / S
        delta = r / nx2 / S
        for l in range(len(Ws) - 1, -1, -1):
            grads[l] += weight_grad(delta, acts[l], links, bc)
            if l > 0:
                delta = layer_adjoint(Ws[l], links, delta, bc)
    return loss, grads
