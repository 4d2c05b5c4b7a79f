"""The learned VR warm start: its network kernels against the CPU oracle of the
network (oracle/mlp_oracle.py), its training, and the gated warm start inside
the tolerance-driven Jacobi iteration.

Tolerances: the GPU kernels round features, weights, activations and the
back-propagated dz to BF16 and accumulate in FP32; the oracle with bf16=True
rounds at the same points in FP64, so GPU and oracle agree to accumulation
order (and the rare BF16 tie that order flips): 1e-3 relative, in norm.  Against
the all-FP64 oracle the BF16 network is held to 2e-2 relative.
"""
import numpy as np
import pytest

import mlp_oracle as mo

from dnds_b200 import _lib


# ---------------------------------------------------------------------- CPU: the oracle itself
def test_oracle_layout_matches_library():
    assert (mo.N_IN, mo.N_OUT, mo.N_PARAM) == (_lib.MLP_IN, _lib.MLP_OUT, _lib.MLP_NPARAM)


def test_oracle_backward_matches_finite_differences():
    p = mo.random_params(1).astype(np.float64)
    rng = np.random.default_rng(0)
    X = rng.normal(size=(9, mo.N_IN))
    T = rng.normal(size=(9, mo.N_OUT))
    _, g = mo.loss_and_grad(p, X, T)
    idx = rng.choice(np.nonzero(g)[0], 40, replace=False)
    h = 1e-6
    for i in idx:
        a, b = p.copy(), p.copy()
        a[i] += h
        b[i] -= h
        fd = (mo.loss_and_grad(a, X, T)[0] - mo.loss_and_grad(b, X, T)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(abs(g[i]), 1e-3), (i, fd, g[i])


def test_oracle_padding_has_no_gradient():
    p = mo.random_params(2)
    rng = np.random.default_rng(1)
    _, g = mo.loss_and_grad(p, rng.normal(size=(5, mo.N_IN)), rng.normal(size=(5, mo.N_OUT)))
    W4 = g[mo.OFF_W4:mo.OFF_B4].reshape(mo.N_OUTP, mo.N_HID)
    assert not W4[mo.N_OUT:].any() and not g[mo.OFF_B4 + mo.N_OUT:].any()


def test_bf16_rounding_known_answers():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.0e38, 1e-40])
    r = mo.bf16(x)
    # ties go to even: 1 + 2^-8 -> 1, 1 + 3*2^-8 -> 1 + 2^-6; 2^-9 rounds down
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == 1.0
    assert r[4] == -2.5 and np.isfinite(r[5]) and abs(r[6] - 1e-40) < 1e-41


# ---------------------------------------------------------------------- GPU: kernels vs oracle
def _torch():
    import torch

    return torch, torch.device("cuda:0")


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def test_bounded_pairs_drops_only_unbounded_targets():
    import torch

    from dnds_b200.learned import bounded_pairs

    X = torch.arange(12, dtype=torch.float32).reshape(4, 3)
    T = torch.tensor([[0.5, -2.0], [11.0, 0.0], [-10.0, 10.0], [0.0, -10.5]])
    Xk, Tk, kept = bounded_pairs(X, T, bound=10.0)
    assert kept == 0.5
    assert torch.equal(Xk, X[[0, 2]]) and torch.equal(Tk, T[[0, 2]])


@pytest.mark.gpu
def test_forward_matches_oracle():
    torch, dev = _torch()
    from dnds_b200.learned import WarmStartNet

    p = mo.random_params(3)
    net = WarmStartNet(0, params=p)
    rng = np.random.default_rng(4)
    X = rng.normal(size=(1001, mo.N_IN)).astype(np.float32)  # not a multiple of the 16-row tile
    Y = net.forward(torch.from_numpy(X).to(dev)).cpu().numpy()
    assert _rel(Y, mo.forward(p, X, bf=True)) < 1e-3
    assert _rel(Y, mo.forward(p, X, bf=False)) < 2e-2
    assert np.array_equal(net.params, p)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 127, 128, 129, 4097])
def test_forward_tile_edges_and_row_independence(n):
    """The tensor-core forward works on 128-row tiles: partial tiles agree with the oracle, and each
    row's output depends on that row only (permuting the rows permutes the outputs bit for bit)."""
    torch, dev = _torch()
    from dnds_b200.learned import WarmStartNet

    p = mo.random_params(5)
    net = WarmStartNet(0, params=p)
    X = np.random.default_rng(n).normal(size=(n, mo.N_IN)).astype(np.float32)
    Y = net.forward(torch.from_numpy(X).to(dev)).cpu().numpy()
    assert _rel(Y, mo.forward(p, X, bf=True)) < 1e-3
    perm = np.random.default_rng(1).permutation(n)
    Yp = net.forward(torch.from_numpy(X[perm]).to(dev)).cpu().numpy()
    assert np.array_equal(Yp, Y[perm])


@pytest.mark.gpu
def test_gradient_matches_oracle():
    torch, dev = _torch()
    from dnds_b200.learned import WarmStartNet

    p = mo.random_params(5)
    net = WarmStartNet(0, params=p)
    rng = np.random.default_rng(6)
    n = 3000  # several 64-row tiles per CTA and a ragged last tile
    X = rng.normal(size=(n, mo.N_IN)).astype(np.float32)
    T = (0.3 * rng.normal(size=(n, mo.N_OUT))).astype(np.float32)
    loss, g = net.gradient(torch.from_numpy(X).to(dev), torch.from_numpy(T).to(dev))
    lb, gb = mo.loss_and_grad(p, X.astype(np.float64), T.astype(np.float64), bf=True)
    l6, g6 = mo.loss_and_grad(p, X.astype(np.float64), T.astype(np.float64), bf=False)
    assert abs(loss - lb) < 1e-5 * lb and abs(loss - l6) < 1e-3 * l6
    assert _rel(g, gb) < 1e-3
    assert _rel(g, g6) < 2e-2
    for a, b in ((mo.OFF_W1, mo.OFF_B1), (mo.OFF_B1, mo.OFF_W2), (mo.OFF_W2, mo.OFF_B2), (mo.OFF_W3, mo.OFF_B3),
                 (mo.OFF_W4, mo.OFF_B4), (mo.OFF_B4, mo.N_PARAM)):
        assert _rel(g[a:b], gb[a:b]) < 2e-3, (a, b)


@pytest.mark.gpu
def test_adam_step():
    torch, dev = _torch()
    from dnds_b200.learned import WarmStartNet

    p = mo.random_params(7)
    net = WarmStartNet(0, params=p)
    rng = np.random.default_rng(8)
    X = torch.from_numpy(rng.normal(size=(500, mo.N_IN)).astype(np.float32)).to(dev)
    T = torch.from_numpy(rng.normal(size=(500, mo.N_OUT)).astype(np.float32)).to(dev)
    _, g = net.gradient(X, T)
    lr = 1e-3
    net.train_step(X, T, lr)
    # first Adam step: m_hat = g, v_hat = g^2
    expect = p - lr * g / (np.sqrt(g.astype(np.float64) ** 2) + 1e-8)
    got = net.params
    assert np.abs(got - expect).max() < 1e-6
    pad = np.zeros(mo.N_PARAM, bool)
    pad[mo.OFF_W1:mo.OFF_B1].reshape(mo.N_HID, mo.N_INP)[:, mo.N_IN:] = True
    pad[mo.OFF_W4:mo.OFF_B4].reshape(mo.N_OUTP, mo.N_HID)[mo.N_OUT:] = True
    pad[mo.OFF_B4 + mo.N_OUT:] = True
    assert not got[pad].any()


@pytest.mark.gpu
def test_training_fits_a_teacher_network():
    torch, dev = _torch()
    from dnds_b200.learned import WarmStartNet, train

    teacher = mo.random_params(9, scale=0.7)
    rng = np.random.default_rng(10)
    X = rng.normal(size=(40000, mo.N_IN))
    T = mo.forward(teacher, X)
    Xd = torch.from_numpy(X.astype(np.float32)).to(dev)
    Td = torch.from_numpy(T.astype(np.float32)).to(dev)
    net = WarmStartNet(0, seed=11)
    l0, _ = net.gradient(Xd, Td)
    hist, val = train(net, Xd, Td, epochs=40, batch=4096, lr=3e-3, lr_end=1e-4)
    assert val < 0.1 * l0, (l0, val)


# ---------------------------------------------------------------------- GPU: warm start in the solver
def _vortex(n, seed, precision=1):
    from dnds_b200 import geometry as G
    from dnds_b200 import mesh as M
    from dnds_b200 import settings as S
    from dnds_b200.solver import Solver

    m = M.vortex_mesh(n, True, jitter=0.2, seed=seed)
    s = Solver(m, S.preset("vortex"), precision=precision)
    s.set_u(G.isentropic_vortex(m, 0.0))
    return s


@pytest.mark.gpu
def test_features_and_harvest():
    torch, dev = _torch()
    from dnds_b200.learned import harvest

    s = _vortex(32, 21)
    s.vr_to_tolerance(1e-7, 300)
    X, T, sweeps = harvest(s, 2, 0.5, 1e-7, 300)
    N = s.N
    assert X.shape == (3 * 2 * N, mo.N_IN) and T.shape == (3 * 2 * N, mo.N_OUT)
    X, T = X.cpu().numpy(), T.cpu().numpy()
    assert np.isfinite(X).all() and np.isfinite(T).all()
    assert all(2 <= k <= 3 * 300 for k in sweeps)
    # the first increment block is scaled per variable by its own largest entry
    d1 = X[:, 16:36].reshape(-1, 5, 4)
    m = np.abs(d1).max(axis=1)
    live = m > 0
    assert np.allclose(m[live], 1.0, atol=1e-6)
    # geometry is the same at every stage and step
    assert np.array_equal(X[:N, 56:64], X[-N:, 56:64])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [1, 0])
def test_gate_keeps_the_jacobi_tolerance(precision):
    """With any network -- trained, random or absurd -- the iteration still stops only at the
    plain Jacobi tolerance, and the reconstruction matches the plain one to that tolerance
    (FP32-bulk and FP64 contexts: the tensor-core warm start reads either coefficient type)."""
    torch, dev = _torch()
    from dnds_b200.learned import WarmStartNet

    tol = 1e-7
    ref = _vortex(48, 22, precision)
    ref.ssprk3_step(0.5)
    n0, _ = ref.vr_to_tolerance(tol, 2000)
    x_ref = ref.get_urec()
    u_ref = ref.get_u()
    for scale in (1.0, 1e3):
        net = WarmStartNet(0, params=mo.random_params(23, scale=scale))
        s = _vortex(48, 22, precision)
        s.ssprk3_step(0.5)
        n1, acc = s.vr_to_tolerance(tol, 2000, net)
        assert n1 < 2000 and 0 <= acc <= s.N
        assert np.array_equal(s.get_u(), u_ref)
        x = s.get_urec()
        # two iterates that both stopped at increment tol differ by O(tol / (1 - rho))
        assert np.sqrt(np.mean(np.sum((x - x_ref) ** 2, axis=(1, 2)))) < 200 * tol
    flags, _ = s.status()
    assert flags == 0


@pytest.mark.gpu
def test_learned_start_sweeps_report(capsys):
    """Harvests on two meshes, trains, and reports Jacobi sweeps per SSP-RK3 step with and
    without the network on a fresh seed; the plain and learned runs must both converge."""
    torch, dev = _torch()
    from dnds_b200.learned import WarmStartNet, harvest, sweep_counts, train

    tol = 1e-7
    Xs, Ts = [], []
    for seed in (31, 32):
        s = _vortex(96, seed)
        s.vr_to_tolerance(tol, 1000)
        X, T, _ = harvest(s, 6, 0.5, tol, 1000)
        Xs.append(X)
        Ts.append(T)
    X, T = torch.cat(Xs), torch.cat(Ts)
    net = WarmStartNet(0, seed=33)
    _, val = train(net, X, T, epochs=15, batch=32768)
    assert val < float((T ** 2).mean())
    res = {}
    for name, use in (("plain", None), ("learned", net)):
        s = _vortex(96, 9999)
        s.vr_to_tolerance(tol, 1000)
        res[name] = sweep_counts(s, 4, 0.5, tol, use, 1000)
        assert max(res[name]) < 3 * 1000
    with capsys.disabled():
        print(f"\nJacobi sweeps per step to rms increment {tol:g} (vortex 96x96x2, fresh seed): "
              f"plain {res['plain']}, learned start {res['learned']}")


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [1, 0])
def test_previous_coefficient_design_keeps_the_tolerance(precision):
    """Input design 1 (neighbour mean differences and the previous-step coefficients, before any
    sweep): harvested targets are (converged - x0) / s with finite features, a network of the other
    design is refused, and with a random or absurd network the iteration still stops only at the
    plain Jacobi tolerance."""
    torch, dev = _torch()
    from dnds_b200.learned import WarmStartNet, harvest
    from dnds_b200.solver import DndsgError

    tol = 1e-7
    s = _vortex(48, 22, precision)
    s.set_warm_start_features(1)
    s.vr_to_tolerance(tol, 2000)
    X, T, sweeps = harvest(s, 1, 0.5, tol, 2000)
    X, T = X.cpu().numpy(), T.cpu().numpy()
    assert np.isfinite(X).all() and np.isfinite(T).all()
    assert np.all(X[:, 36:56] == 0)
    # the mean-difference block is scaled per variable by its own largest entry, floored at 1e-12 of the
    # cell's own mean (near-uniform cells, far from the vortex, stay below 1)
    du = X[:, :16].reshape(-1, 4, 4)
    m = np.abs(du).max(axis=1)
    assert (m <= 1.0 + 1e-6).all()
    assert np.mean(np.isclose(m, 1.0, atol=1e-6)) > 0.5
    ref = _vortex(48, 22, precision)
    ref.ssprk3_step(0.5)
    ref.vr_to_tolerance(tol, 2000)
    x_ref = ref.get_urec()
    with pytest.raises(DndsgError, match="feature design"):
        t = _vortex(48, 22, precision)
        t.set_warm_start_features(1)
        t.vr_to_tolerance(tol, 2000, WarmStartNet(0, params=mo.random_params(5), features=0))
    for scale in (1.0, 1e3):
        net = WarmStartNet(0, params=mo.random_params(23, scale=scale), features=1)
        t = _vortex(48, 22, precision)
        t.set_warm_start_features(1)
        t.ssprk3_step(0.5)
        n1, acc = t.vr_to_tolerance(tol, 2000, net)
        assert n1 < 2000 and 0 <= acc <= t.N
        x = t.get_urec()
        assert np.sqrt(np.mean(np.sum((x - x_ref) ** 2, axis=(1, 2)))) < 200 * tol
        flags, _ = t.status()
        assert flags == 0
