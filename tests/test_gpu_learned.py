"""GPU tests of the learned preconditioner (qq_net_*, qq_fgmres).

The network's forward pass and its loss gradient are checked against the numpy
restatement in netref.py (whose gradient is itself checked against finite differences
in test_cpu_netref.py).  Tolerances: 2e-5 relative for the FP32 forward pass, 1e-4 for
the gradient (FP32 fields, FP64 reductions).  Then: training lowers the loss, and the
trained network cuts the operator applications of flexible GMRES against the same
method without it, with the FP64 true residual judging both; a network that cannot
span the solution stalls and plain GMRES-DR takes over."""
import numpy as np
import pytest

import netref
import oracle
from qqtest import half_to_lex, random_gauge, random_half

pytestmark = pytest.mark.gpu

BC = (1, 1, 1, -1)
SMALL = (4, 4, 4, 8)


def split(net, w):
    ch, Ws, o = net.channels, [], 0
    for l in range(len(ch) - 1):
        n = 9 * ch[l + 1] * ch[l]
        Ws.append(w[o:o + n].reshape(9, ch[l + 1], ch[l]))
        o += n
    return Ws


@pytest.fixture(scope="module")
def small():
    import baylorlqcd_b200 as qq

    ol = oracle.OracleLattice(*SMALL, bc=BC)
    links, u = random_gauge(SMALL, ol.ntotal, seed=3)
    lat = qq.Lattice(*SMALL, bc=BC)
    lat.gauge_upload(u, recon=12)
    yield lat, ol, links
    lat.close()


def random_weights(net, seed):
    rng = np.random.default_rng(seed)
    n = net.nweights
    return 0.3 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))


@pytest.mark.parametrize("channels", [(4, 4), (4, 8, 4), (4, 16, 8, 4)])
def test_forward_matches_numpy(small, channels):
    import baylorlqcd_b200 as qq

    lat, ol, links = small
    net = qq.Net(channels, seed=1)
    w = random_weights(net, 11)
    net.set_weights(w)
    g = random_half(ol.ntotal, ol.nvhalf, seed=5)
    out = net.apply(lat, g)
    ref = netref.apply(split(net, w), links, half_to_lex(g, SMALL, 1), BC)
    got = half_to_lex(out, SMALL, 1)
    assert np.abs(got - ref).max() / np.abs(ref).max() < 2e-5
    net.close()


def test_gradient_matches_numpy(small):
    import baylorlqcd_b200 as qq

    lat, ol, links = small
    net = qq.Net((4, 8, 4), seed=2)
    w = random_weights(net, 12)
    net.set_weights(w)
    b = np.stack([random_half(ol.ntotal, ol.nvhalf, seed=20 + i) for i in range(2)])
    x = np.stack([random_half(ol.ntotal, ol.nvhalf, seed=30 + i) for i in range(2)])
    loss, grad = net.loss_grad(lat, b, x)
    lref, gref = netref.loss_grad(split(net, w), links, [half_to_lex(v, SMALL, 1) for v in b],
                                  [half_to_lex(v, SMALL, 1) for v in x], BC)
    assert abs(loss - lref) / lref < 1e-5
    gref = np.concatenate([gl.ravel() for gl in gref])
    assert np.abs(grad - gref).max() / np.abs(gref).max() < 1e-4
    net.close()


@pytest.fixture(scope="module")
def config():
    import baylorlqcd_b200 as qq

    lat = qq.Lattice(8, 8, 8, 8, bc=BC)
    u, _ = lat.heatbath(6.0, 100, seed=7)
    yield lat, u
    lat.close()


KAPPA = (0.150, 0.0)


def test_training_lowers_loss(config):
    import baylorlqcd_b200 as qq

    lat, _ = config
    net = qq.Net((4, 8, 4), seed=3, scale=KAPPA[0] ** 2)
    losses = net.train(lat, KAPPA, nsamples=4, nsteps=60, lr=2e-3, seed=5)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.6 * losses[0]
    net.close()


def test_trained_preconditioner_gains(config):
    """Same source, same FGMRES(16), same 1e-10 true residual: the trained network
    needs fewer applications of Hdbletm than no preconditioner, and both solutions
    agree with GMRES-DR's."""
    import baylorlqcd_b200 as qq

    lat, _ = config
    net = qq.Net((4, 8, 8, 4), seed=4, scale=KAPPA[0] ** 2)
    net.train(lat, KAPPA, nsamples=6, nsteps=150, lr=2e-3, seed=6)
    phi = random_half(lat.ntotal, lat.nvhalf, seed=9)
    x_net, inet = lat.fgmres(phi, KAPPA, m=16, resmax=1e-10, net=net)
    x_pl, ipl = lat.fgmres(phi, KAPPA, m=16, resmax=1e-10, net=None)
    x_dr, _ = lat.gmresdr(phi, np.zeros_like(phi), (16, 5), 1e-11, kappa=KAPPA)
    assert inet.status == 0 and ipl.status == 0
    assert inet.true_rel < 1e-10 and ipl.true_rel < 1e-10
    assert inet.fallback == 0
    nv = lat.nvhalf
    for x in (x_net, x_pl):
        assert np.linalg.norm((x - x_dr)[:, :, :, :nv]) / np.linalg.norm(x_dr[:, :, :, :nv]) < 1e-8
    assert inet.mvp < 0.8 * ipl.mvp, (inet.mvp, ipl.mvp)
    net.close()


def test_stalled_preconditioner_falls_back(config):
    """A network that drops spins 2 and 3 cannot span the solution: flexible GMRES
    stalls, plain GMRES-DR takes over and converges."""
    import baylorlqcd_b200 as qq

    lat, _ = config
    net = qq.Net((4, 4), seed=5)
    w = np.zeros(net.nweights, complex)
    w[0 * 4 + 0] = w[1 * 4 + 1] = KAPPA[0] ** 2      # path 0, channels 0 and 1 only
    net.set_weights(w)
    phi = random_half(lat.ntotal, lat.nvhalf, seed=10)
    x, info = lat.fgmres(phi, KAPPA, m=16, resmax=1e-10, net=net)
    assert info.fallback == 1
    assert info.status == 0 and info.true_rel < 1e-10
    net.close()


def test_flexible_gmresdr_gains(config):
    """Flexible GMRES-DR(32, 10) with the trained network against the same method
    without it (which is GMRES-DR(32, 10) in flexible form): same 1e-10 true residual,
    fewer applications of Hdbletm, no fallback; the unpreconditioned flexible form
    needs the applications of the reference's GMRES-DR."""
    import baylorlqcd_b200 as qq

    lat, _ = config
    net = qq.Net((4, 8, 8, 4), seed=4, scale=KAPPA[0] ** 2)
    net.train(lat, KAPPA, nsamples=6, nsteps=150, lr=2e-3, seed=6)
    phi = random_half(lat.ntotal, lat.nvhalf, seed=9)
    x_net, inet = lat.fgmres(phi, KAPPA, m=32, k=10, resmax=1e-10, net=net)
    x_pl, ipl = lat.fgmres(phi, KAPPA, m=32, k=10, resmax=1e-10, net=None)
    x_dr, idr = lat.gmresdr(phi, np.zeros_like(phi), (32, 10), 1e-10, kappa=KAPPA)
    assert inet.status == 0 and ipl.status == 0 and inet.fallback == 0 and ipl.fallback == 0
    assert inet.true_rel < 1e-10 and ipl.true_rel < 1e-10
    assert ipl.mvp == idr.mvp
    nv = lat.nvhalf
    assert np.linalg.norm((x_net - x_dr)[:, :, :, :nv]) / np.linalg.norm(x_dr[:, :, :, :nv]) < 1e-8
    assert inet.mvp < 0.8 * ipl.mvp, (inet.mvp, ipl.mvp)
    net.close()


def test_deflation_vectors_are_the_gmresdr_space(config):
    """qq_defl_vector returns the k + 1 orthonormal vectors the GMRES-DR restart keeps,
    and A maps the first k into their span (A V_k = V_{k+1} H_k): the projection of each
    A v_j onto the k + 1 vectors leaves a residual at rounding level."""
    lat, _ = config
    phi = random_half(lat.ntotal, lat.nvhalf, seed=12)
    d = lat.deflation(24, 8)
    lat.gmresdr(phi, np.zeros_like(phi), (24, 8), 1e-10, kappa=KAPPA, defl=d)
    k = d.k
    assert k == 8
    nv = lat.nvhalf
    V = [d.vector(j) for j in range(k + 1)]
    cv = np.stack([(v[:, :, :, :nv, 0::2] + 1j * v[:, :, :, :nv, 1::2]).ravel() for v in V])
    np.testing.assert_allclose(cv.conj() @ cv.T, np.eye(k + 1), atol=1e-10)
    for j in range(k):
        av = lat.hdbletm(V[j], 0, KAPPA)
        ca = (av[:, :, :, :nv, 0::2] + 1j * av[:, :, :, :nv, 1::2]).ravel()
        res = ca - cv.T @ (cv.conj() @ ca)
        assert np.linalg.norm(res) < 1e-9 * np.linalg.norm(ca), j
    with pytest.raises(Exception):
        d.vector(k + 1)
    d.close()


def test_training_on_solver_pairs_gains(config):
    """The network trained on the deflated inverter's own output -- (source, FP64
    solution) pairs of GMRES-DR solves of Z(2) noises and (A v, v) of its deflation
    vectors -- lowers its loss and cuts the operator applications of flexible GMRES-DR
    on a held-out source, with the FP64 true residual judging the answer."""
    import baylorlqcd_b200 as qq

    lat, _ = config
    qq.initlagfib(0, 3)
    d = lat.deflation(32, 10)
    B, X = [], []
    for i in range(4):
        b, _ = lat.z2source()
        x, info = lat.gmresdr(b, lat.new_half(), (32, 10), 1e-10, kappa=KAPPA, defl=d if i == 0 else None)
        assert info.status == 0
        B.append(b)
        X.append(x)
    for j in range(d.k):
        v = d.vector(j)
        X.append(v)
        B.append(lat.hdbletm(v, 0, KAPPA))
    d.close()
    net = qq.Net((4, 8, 8, 4), seed=4, scale=KAPPA[0] ** 2)
    losses = net.train_pairs(lat, np.stack(B), np.stack(X), nsteps=150, lr=2e-3)
    # the solutions are dominated by low modes the network cannot represent (the flexible
    # method's deflation keeps those): the loss falls by about a quarter, not to zero
    assert np.all(np.isfinite(losses)) and losses[-1] < 0.85 * losses[0]
    phi = random_half(lat.ntotal, lat.nvhalf, seed=21)
    _, inet = lat.fgmres(phi, KAPPA, m=32, k=10, resmax=1e-10, net=net)
    _, ipl = lat.fgmres(phi, KAPPA, m=32, k=10, resmax=1e-10, net=None)
    assert inet.status == 0 and inet.true_rel < 1e-10 and inet.fallback == 0
    assert inet.mvp < 0.8 * ipl.mvp, (inet.mvp, ipl.mvp)
    net.close()
