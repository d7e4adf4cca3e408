"""GPU: the learned MDF warm start — the network's fused training and inference
kernels against the CPU oracle (oracle/mlp_oracle.py), and what the trained
network gains over plain MDF on an oscillating cylinder."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _rand_net(torch, seed):
    from iblbm_b200.learned import MdfNet
    net = MdfNet(seed=seed)
    rng = np.random.default_rng(seed)
    P = net.params.cpu().numpy()
    P[0:64] = rng.standard_normal(64) * 0.1
    P[64:128] = 1.0 + 0.1 * rng.random(64)
    P[128:130] = [2.0, 0.5]
    net.params.copy_(torch.as_tensor(P))
    return net, rng


def test_gradient_matches_oracle(torch):
    from oracle import mlp_oracle as M
    net, rng = _rand_net(torch, 3)
    n = 200  # three full CTAs and a partial one
    X = rng.standard_normal((n, 64)).astype(np.float32)
    T = rng.standard_normal((n, 2)).astype(np.float32)
    net.loss.zero_()
    net.train_step(torch.as_tensor(X, device="cuda"), torch.as_tensor(T, device="cuda"), apply=False)
    g = net.summed_gradient().cpu().numpy().astype(np.float64)
    L = float(net.loss.item())
    P = net.params.cpu().numpy()
    # against the oracle with the tensor cores' TF32 operand rounding: only the
    # FP32 accumulation order differs
    Lo, go = M.loss_and_grad(P, X, T, tc=True)
    assert abs(L - Lo) <= 1e-4 * Lo
    scale = np.abs(go).max()
    np.testing.assert_allclose(g[:go.size], go, rtol=2e-3, atol=2e-5 * scale)
    assert np.all(g[go.size:] == 0.0)  # padding of the parameter block
    # and within TF32's operand precision of the exact gradient
    _, ge = M.loss_and_grad(P, X, T)
    assert np.abs(g[:ge.size] - ge).max() <= 2e-2 * np.abs(ge).max()


def test_adam_step_matches_oracle(torch):
    from oracle import mlp_oracle as M
    net, rng = _rand_net(torch, 4)
    n = 256
    X = rng.standard_normal((n, 64)).astype(np.float32)
    T = rng.standard_normal((n, 2)).astype(np.float32)
    P0 = net.params.cpu().numpy().astype(np.float64)
    _, go = M.loss_and_grad(P0, X, T, tc=True)
    go = np.concatenate([go, np.zeros(P0.size - go.size)])
    net.train_step(torch.as_tensor(X, device="cuda"), torch.as_tensor(T, device="cuda"), lr=1e-3)
    torch.cuda.synchronize()
    P1 = net.params.cpu().numpy().astype(np.float64)
    Po, _, _ = M.adam_step(P0, go, np.zeros_like(P0), np.zeros_like(P0), 1, 1e-3)
    big = np.abs(go) > 1e-3 * np.abs(go).max()  # sign steps of well-resolved gradients
    np.testing.assert_allclose(P1[big], Po[big], rtol=0, atol=2e-6)


def test_training_is_deterministic(torch):
    """Two networks from the same state take the same training steps to the
    same parameters bit for bit: every block of 64 samples writes its own
    gradient slot and the slots are summed in block order (no atomics)."""
    nets = [_rand_net(torch, 6)[0] for _ in range(2)]
    rng = np.random.default_rng(6)
    X = torch.as_tensor(rng.standard_normal((1000, 64)).astype(np.float32), device="cuda")
    T = torch.as_tensor(rng.standard_normal((1000, 2)).astype(np.float32), device="cuda")
    for net in nets:
        net.loss.zero_()
        for k in range(5):
            net.train_step(X[200 * k:200 * k + 200].contiguous(), T[200 * k:200 * k + 200].contiguous(), lr=1e-3)
    torch.cuda.synchronize()
    assert torch.equal(nets[0].params, nets[1].params)
    assert torch.equal(nets[0].m, nets[1].m) and torch.equal(nets[0].v, nets[1].v)
    assert float(nets[0].loss.item()) == float(nets[1].loss.item())


def test_inference_matches_oracle(torch):
    from oracle import mlp_oracle as M
    net, rng = _rand_net(torch, 5)
    X = rng.standard_normal((300, 64)).astype(np.float32)
    Y = net.predict(torch.as_tensor(X, device="cuda")).cpu().numpy()
    # against the oracle with TF32 operands: an activation that lands on the other
    # side of a TF32 rounding boundary (the kernel's FP32 sums differ from the
    # oracle's in the last bits) moves a few outputs by ~1e-4 of the scale
    Yo = M.predict(net.params.cpu().numpy(), X, tc=True)
    np.testing.assert_allclose(Y, Yo, rtol=1e-4, atol=1e-4 * np.abs(Yo).max())
    Ye = M.predict(net.params.cpu().numpy(), X)
    assert np.abs(Y - Ye).max() <= 1e-2 * np.abs(Ye).max()


def _osc_cfg(steps):
    from iblbm_b200.config import SimConfig
    return SimConfig(Re=20, NN=161, xmax=1, ymax=1, cylinder_center=(0.5, 0.5), cylinder_D_ratio=0.125,
                     lattice_u=0.02, inflow_u=0.0, bc_type="open_boundary", delta_type="peskin4pt", ibm_method="MDF",
                     collision_model="BGK", motion_type="oscillating", KC=5.0, nx_formula="simple",
                     marker_spacing_factor=1.0, mdf_iterations=20, mdf_min_iterations=20,
                     mdf_tolerance=1e-12, max_steps=steps + 10, use_convergence=False, check_interval=50)


PLAIN_ITERS = 20


def test_warm_start_saves_iterations(torch):
    """Plain MDF (20 iterations per step) generates (features, accumulated
    force) pairs for 240 steps of an oscillating cylinder.  For the next 60
    steps a second engine, warm-started by the network trained on them, iterates
    each step only until its slip residual is down to what plain MDF reached
    after 20 iterations at that step (20 at most, the plain loop being the
    fallback); the saving is the iterations it does not need."""
    from iblbm_b200.engine import Engine
    from iblbm_b200.learned import MdfNet, collect
    # the motion of this reference scenario sets the desired velocity to the
    # displacement, so the flow keeps gaining speed; 300 steps stay well inside
    # the stable range of both forms
    n_train, n_eval = 240, 60
    cfg = _osc_cfg(n_train + n_eval)
    plain = Engine(cfg, precision="f32")
    for _ in range(n_train):
        plain.advance(1, outputs_last=False, use_graph=False)
    warm = Engine(cfg, precision="f32")
    X, T, its = collect(warm, n_train)
    assert its == [PLAIN_ITERS] * n_train
    net = MdfNet(seed=0)
    hist = net.fit(X, T, epochs=40, batch=512, lr=2e-3)
    assert hist[-1] < 0.2 * hist[0]
    warm.set_mlp(mode=2, net=net)
    for a in warm.ibm_args:
        a.mdf_min_iterations = 1
    warm_its, conv = [], []
    for k in range(n_eval):
        last = k == n_eval - 1
        plain.advance(1, outputs_last=last, use_graph=False)
        r_plain = float(plain.d_dstats[0].item())
        for a in warm.ibm_args:
            a.mdf_tol = r_plain * (1.0 + 1e-6)
        warm.advance(1, outputs_last=last, use_graph=False)
        warm_its.append(int(warm.d_stats[0].item()))
        conv.append(int(warm.d_stats[2].item()))
    w_mean = float(np.mean(warm_its))
    print(f"MDF iterations to the plain residual: plain {PLAIN_ITERS}, warm-started {w_mean:.2f}, "
          f"saved {PLAIN_ITERS - w_mean:.2f}; reached in {sum(conv)}/{n_eval} steps")
    assert sum(conv) >= 0.9 * n_eval
    assert np.isfinite(warm.read_state().U).all()
    assert w_mean <= 0.5 * PLAIN_ITERS
    cd_p, _ = plain.cd_cl()
    cd_w, _ = warm.cd_cl()
    assert abs(cd_w - cd_p) <= 1e-3 * abs(cd_p)
