"""The learned precision router: its GPU forward/backward kernels against the
numpy restatement (oracle/mlp.py), and what the trained network gains over
the rigorous Schwarz x density routing while the routed build stays within
the error budget (max|dG| <= 1e-8 against the FP64 build)."""

import numpy as np
import pytest

from felizjueves_b200 import configs

pytestmark = pytest.mark.gpu


def test_mlp_kernels_match_numpy(cuda, lib_built):
    from felizjueves_b200 import router
    from oracle import mlp as omlp
    rng = np.random.default_rng(3)
    X = rng.normal(size=(3000, 12)).astype(np.float32) * 3 + 1
    T = rng.normal(size=3000).astype(np.float32)
    p = router.init_params(X, seed=5)
    p[24:] += rng.normal(scale=0.05, size=p.size - 24).astype(np.float32)  # nonzero biases too
    m = router.MLP(p)
    y = m.predict(X, exact=True).cpu().numpy()
    yo, _ = omlp.forward(p, X)
    assert np.abs(y - yo).max() <= 1e-5 * max(1.0, np.abs(yo).max())
    # the routing arithmetic (FP16 tensor-core products, tanh.approx) on a
    # network whose hidden layers carry the output (w3 of order 1): each
    # hidden unit within 4e-3 of its FP32 value (FP16 operands and tanh.approx
    # are 2^-11 relative), so |dy| <= 4e-3 sum|w3|; 4,099 samples = a ragged
    # last warp
    p2 = p.copy()
    p2[-65:-1] = rng.normal(scale=0.3, size=64).astype(np.float32)
    X2 = np.concatenate([X, X[:1099]])
    y2 = router.MLP(p2).predict(X2).cpu().numpy()
    yo2, _ = omlp.forward(p2, X2)
    d = float(np.abs(y2 - yo2).max())
    print(f"tensor-core forward vs FP32: max|dy| {d:.2e} (sum|w3| {np.abs(p2[-65:-1]).sum():.1f})")
    assert d <= 4e-3 * np.abs(p2[-65:-1]).sum()
    g, mse = m.gradient(X, T)
    go = omlp.gradient(p, X, T)
    g = g.cpu().numpy()
    assert np.abs(g - go).max() <= 1e-4 * np.abs(go).max()
    assert abs(mse - float(np.mean((yo - T) ** 2))) <= 1e-4 * max(1.0, mse)


def test_trained_router_gains_within_budget(cuda, lib_built):
    import torch
    from felizjueves_b200 import _lib, router
    from felizjueves_b200.fock import FockEngine
    train = [configs.cluster(n, 100 + n) for n in (4, 5, 6, 7, 8, 10)]
    X, y = router.training_set(train, n_per=12000, seed=1)
    perm = np.random.default_rng(2).permutation(len(X))
    cut = int(0.8 * len(X))
    tr, va = perm[:cut], perm[cut:]
    mlp = router.MLP(router.init_params(X[tr], y[tr], seed=0))
    losses = mlp.train(X[tr], y[tr], epochs=60, batch=2048, lr=3e-3)
    margin = router.calibrate(mlp, X[va], y[va], 0.999)
    rmse = float(np.sqrt(np.mean((mlp.predict(X[va]).cpu().numpy() - y[va]) ** 2)))
    d_tc = float((mlp.predict(X[va]) - mlp.predict(X[va], exact=True)).abs().max())
    print(f"trained network: tensor-core vs FP32 forward max|dy| {d_tc:.2e} decades")
    assert d_tc <= 0.05
    gap = y[tr] - router.bound_log10(X[tr])
    rmse_bound = float(np.sqrt(np.mean((router.bound_log10(X[va]) + gap.mean() - y[va]) ** 2)))

    w = configs.cluster(12, 77)  # held out
    eng = FockEngine(w.basis)
    eng.plan(w.D, w.tau, w.n_mag)
    D = torch.tensor(w.D, device=cuda)
    G64 = eng.build(D)[2].clone()
    Gb = eng.build(D, precision=_lib.FJB_ROUTED, threshold=1e-9)[2].clone()
    n32_bound, n64_bound = router.route_stats(eng)
    router.install(eng, mlp, threshold=1e-9, margin=margin)
    Gm = eng.build(D, precision=_lib.FJB_ROUTED, threshold=1e-9)[2].clone()
    n32_mlp, n64_mlp = router.route_stats(eng)
    torch.cuda.synchronize()
    d_bound = float((Gb - G64).abs().max())
    d_mlp = float((Gm - G64).abs().max())
    print(f"router: {len(X)} samples, val rmse {rmse:.3f} log10, margin {margin:.3f}; FP32 units "
          f"bound {n32_bound}/{n32_bound + n64_bound}, learned {n32_mlp}/{n32_mlp + n64_mlp}; "
          f"max|dG| bound {d_bound:.2e}, learned {d_mlp:.2e}; rmse of bound x mean gap {rmse_bound:.3f}, "
          f"loss {losses[0]:.4f} -> {losses[-1]:.4f}")
    assert losses[-1] < losses[0]
    assert rmse < 0.5 * rmse_bound  # the network knows more than the bound
    assert n32_mlp > n32_bound      # and that moves work to FP32
    assert d_mlp <= 1e-8
    v = router.validate(eng, D)
    assert v["within_budget"]


def test_shipped_network_within_budget(cuda, lib_built):
    """The network trained for config c3 (router.load_default), installed
    with its margin, reach and class gate on a 6-atom cluster: the routed
    build within the 1e-8 budget of the FP64 build, and at least the bound's
    FP32 units."""
    import torch
    from felizjueves_b200 import _lib, router
    from felizjueves_b200.fock import FockEngine
    w = configs.cluster(6, 11)
    eng = FockEngine(w.basis)
    eng.plan(w.D, w.tau, w.n_mag)
    D = torch.tensor(w.D, device=cuda)
    G64 = eng.build(D)[2].clone()
    eng.build(D, precision=_lib.FJB_ROUTED, threshold=1e-9)
    n32_bound, _ = router.route_stats(eng)
    mlp, margin, reach, min_l = router.load_default()
    router.install(eng, mlp, threshold=1e-9, margin=margin, reach=reach, min_total_l=min_l)
    G = eng.build(D, precision=_lib.FJB_ROUTED, threshold=1e-9)[2]
    n32, _ = router.route_stats(eng)
    d = float((G - G64).abs().max())
    print(f"shipped network: {n32} FP32 units vs {n32_bound} by the bound, max|dG| {d:.2e}")
    assert d <= 1e-8 and n32 >= n32_bound
