"""Learned warm start on the device: the tensor-core network's forward pass,
gradient and Adam step against the CPU oracle, the Grad-13 seed and the 13
moments against their CPU restatements, and a short training run."""
import numpy as np
import pytest

from oracle import warm_oracle as W

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _inputs(n, seed=0):
    rng = np.random.default_rng(seed)
    return np.column_stack([rng.uniform(0, 1, n), rng.uniform(0, 1, n),
                            rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)]).astype(np.float32)


def _params(seed=0):
    from alebgk4paper_b200.warmstart import init_params
    p = init_params(seed)
    p[W.B_OFF[0]:] = np.random.default_rng(seed + 1).normal(0, 0.1, W.N_PARAMS - W.B_OFF[0])
    p[W.B_OFF[4] + W.N_USED:] = 0
    return p


@pytest.mark.parametrize("n", [128, 1000, 40000])
def test_forward_matches_oracle(n):
    _torch()
    from alebgk4paper_b200.warmstart import WarmStartNet
    q = _inputs(n)
    p = _params()
    net = WarmStartNet(p)
    out = net.forward(q).cpu().numpy()
    ref, _ = W.forward(p, W.features(q))
    scale = np.abs(ref[:, :W.N_USED]).max()
    err = np.abs(out[:, :W.N_USED] - ref[:, :W.N_USED])
    assert err.max() <= 2e-2 * scale, err.max() / scale
    # most rows agree to FP32 summation order (BF16 rounding flips are rare)
    assert np.median(err) / scale < 1e-4
    assert np.all(out[:, W.N_USED:] == 0)
    net.close()


def test_forward_gathers_rows_by_index():
    _torch()
    from alebgk4paper_b200.warmstart import WarmStartNet
    q = _inputs(5000, seed=2)
    net = WarmStartNet(_params(3))
    idx = np.random.default_rng(0).permutation(5000)[:777].astype(np.int32)
    a = net.forward(q, idx=idx).cpu().numpy()
    b = net.forward(q[idx]).cpu().numpy()
    assert np.array_equal(a, b)
    net.close()


@pytest.mark.parametrize("n", [256, 3000])
def test_gradient_matches_oracle(n):
    _torch()
    from alebgk4paper_b200.warmstart import WarmStartNet
    q = _inputs(n, seed=5)
    rng = np.random.default_rng(6)
    T = rng.normal(size=(n, W.N_OUT)).astype(np.float32)
    T[:, W.N_USED:] = 0
    w = np.linspace(0.5, 2.0, W.N_USED).astype(np.float32)
    p = _params(1)
    net = WarmStartNet(p)
    loss, g = net.grad(q, T, chan_w=w)
    rl, rg = W.loss_grad(p, W.features(q), T, w)
    assert abs(loss - rl) <= 1e-3 * rl
    for l, (i, o) in enumerate(W.LAYERS):
        a = g[W.W_OFF[l]:W.W_OFF[l] + i * o].astype(np.float64)
        b = rg[W.W_OFF[l]:W.W_OFF[l] + i * o].astype(np.float64)
        assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b), l
        assert a @ b >= 0.999 * np.linalg.norm(a) * np.linalg.norm(b), l
        ab = g[W.B_OFF[l]:W.B_OFF[l] + o].astype(np.float64)
        bb = rg[W.B_OFF[l]:W.B_OFF[l] + o].astype(np.float64)
        assert np.linalg.norm(ab - bb) <= 2e-2 * np.linalg.norm(bb) + 1e-12, l
    # padded outputs carry no gradient
    assert np.all(g[W.W_OFF[4] + W.N_USED * W.N_HID:W.W_OFF[4] + W.N_OUT * W.N_HID] == 0)
    # and the exact FP64 gradient agrees to BF16 accuracy
    ge = W.grad_exact(p.astype(np.float64), W.bf16(W.features(q)), T, w)
    assert np.linalg.norm(g - ge) <= 5e-2 * np.linalg.norm(ge)
    net.close()


def test_adam_step_matches_oracle():
    _torch()
    from alebgk4paper_b200.warmstart import WarmStartNet
    q = _inputs(2048, seed=8)
    T = np.random.default_rng(9).normal(size=(2048, W.N_OUT)).astype(np.float32)
    p = _params(2)
    net = WarmStartNet(p)
    _, g = net.grad(q, T)
    net.fit(q, T, steps=1, batch=2048, lr=1e-3, lr_final=1e-3, log_every=0)
    # the step's batch is a permutation of all rows: the same gradient up to order
    ref, _, _ = W.adam(p, np.zeros_like(p), np.zeros_like(p), g, 1, 1e-3)
    new = net.params()
    assert np.allclose(new, ref, rtol=0, atol=2e-6)
    assert np.abs(new - p).max() > 5e-4
    net.close()


def test_training_reduces_the_loss():
    _torch()
    from alebgk4paper_b200.warmstart import WarmStartNet
    q = _inputs(20000, seed=11)
    x, y, a, b = q.T
    T = np.zeros((20000, W.N_USED), np.float32)
    for c in range(W.N_USED):
        T[:, c] = np.sin(np.pi * (c + 1) * x / 3) * np.cos(np.pi * y) * (1 + 0.3 * a) + 0.2 * b
    net = WarmStartNet(seed=4)
    log = net.fit(q, T, steps=400, batch=4096, lr=3e-3, lr_final=3e-4, log_every=100)
    assert log[-1][1] < 0.05 * log[0][1], log
    net.close()


def _cavity(precision, Nx=12, Nv=16):
    from alebgk4paper_b200 import Case, Solver
    c = Case("cavity2d", Nx=Nx, Nv=Nv, lid_speed=5.0, rho0=2.0, tau=3.7142e-10 / 2)
    return c, Solver(c, precision=precision)


@pytest.mark.parametrize("precision", [64, 32])
def test_grad13_seed_matches_oracle(precision):
    torch = _torch()
    from alebgk4paper_b200 import _abi
    case, s = _cavity(precision)
    N = case.N
    x = case.xyz[:, 0] / case.xyz[:, 0].max()
    mom = np.column_stack([2.0 * (1 + 0.01 * np.sin(3 * x)), 3.0 * x, -2.0 * x ** 2,
                           270 + 2 * x, 50 * x, -20 * x, 10 * x, 2e3 * x, -1e3 * x])
    mom = mom.astype(np.float32).astype(np.float64)
    net = torch.zeros((N, 16), dtype=torch.float32, device="cuda")
    net[:, :9] = torch.as_tensor(mom, dtype=torch.float32, device="cuda")
    one, zero = np.ones(9), np.zeros(9)
    rc = _abi.load().alebgk_seed_grad13(s.ctx, net.data_ptr(), 16,
                                        one.ctypes.data_as(_abi.c_double_p),
                                        zero.ctypes.data_as(_abi.c_double_p))
    assert rc == 0
    g, m = s.cudaDownloadFull()
    V = case.Nv ** 2
    p = case.params
    g1, g2 = W.grad13_rows(mom, case.Nv, p["vmin"], p["dv"], p["R"])
    tol = 1e-13 if precision == 64 else 1e-7
    assert np.allclose(g[:, :V], g1, rtol=tol, atol=tol * g1.max())
    assert np.allclose(g[:, V:2 * V], g2, rtol=tol, atol=tol * g2.max())
    # the macros are the discrete moments of the seeded rows
    mm = W.moments13(g[:, :V], g[:, V:2 * V], case.Nv, p["vmin"], p["dv"], p["R"])
    assert np.allclose(m[:, 0], mm[:, 0], rtol=1e-6)
    assert np.allclose(m[:, 4], mm[:, 3], rtol=1e-6)
    # and the seeded state steps
    s.step(3)
    s.sync()
    s.cudaFreeCloud()


@pytest.mark.parametrize("precision", [64, 32])
def test_moments13_matches_oracle(precision):
    _torch()
    from alebgk4paper_b200 import warmstart as ws
    case, s = _cavity(precision)
    s.step(20)
    dev = ws.moments13(s)
    g, _ = s.cudaDownloadFull()
    V = case.Nv ** 2
    p = case.params
    ref = W.moments13(g[:, :V], g[:, V:2 * V], case.Nv, p["vmin"], p["dv"], p["R"])
    rtol = 1e-10 if precision == 64 else 1e-6
    scale = np.abs(ref).max(0)
    assert np.all(np.abs(dev - ref) <= rtol * scale), np.abs(dev - ref).max(0) / scale
    s.cudaFreeCloud()


def test_trained_warm_start_beats_the_plain_start():
    """What the committed network gains: held-out cavities (Nx = 48, Nv = 20,
    seeds not used in training) reach the steady residual (5e-7 per step,
    momentum against the lid momentum, as a mean over 200-step intervals) in
    at least twice fewer steps when seeded by the network than from the
    Maxwellian at rest, and the seeded run's steady fields lie within 1e-3
    of the plain run's (relative to each field's range)."""
    _torch()
    from alebgk4paper_b200 import warmstart as ws
    from alebgk4paper_b200 import warm_train as wt
    net = ws.WarmStartNet.load(wt.DEFAULT_MODEL)
    assert net.meta["cases"] == 2000
    r = wt.evaluate(net, wt.heldout_specs(4), reference_steps=4000)
    print({k: r[k] for k in ("steps_ratio", "wall_ratio", "field_rel_err_max",
                             "vs_converged_max")})
    assert r["all_steady"] and r["residual"] == "lid"
    assert r["steps_ratio"] >= 2.0, r["cold_steps"] + r["warm_steps"]
    assert r["wall_ratio"] >= 1.5
    for k in ("rho", "ux", "uy", "T"):
        assert r["field_rel_err_max"][k] < 1e-3, k
    net.close()
