"""The learned warm start: its network's kernels against an FP64 CPU
restatement, its training, and what the trained network gains over the
feasible start it replaces.

* Gradient check: the GPU's forward output and parameter gradient of the mean
  squared error (BF16 weights, FP32 arithmetic) against a numpy FP64 forward /
  backward pass with the same BF16-rounded weights; tolerance 2e-3 of the
  largest gradient entry (FP32 sums over 300 rows).
* Training on converged solutions of seeded synthetic active spaces (n = 6),
  then solves of held-out seeds from the projected proposal: same energy as
  the feasible start (1e-6 Eh), and the iteration counts of both are
  reported (the ablation).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F, O = 16, 3


def _bf16(a):
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _unpack(params, hidden):
    dims = [F, hidden, hidden, hidden, O]
    out, o = [], 0
    for l in range(4):
        W = params[o:o + dims[l + 1] * dims[l]].reshape(dims[l + 1], dims[l])
        o += W.size
        b = params[o:o + dims[l + 1]]
        o += b.size
        out.append((W, b))
    return out


def _cpu_forward_backward(params, hidden, X, T):
    """FP64 restatement of the network (BF16 weights, FP32 biases) and of the
    gradient of mean((Y - T)^2) with respect to every parameter."""
    layers = _unpack(params.astype(np.float64), hidden)
    acts = [X.astype(np.float64)]
    for l, (W, b) in enumerate(layers):
        z = acts[-1] @ _bf16(W).T + b
        acts.append(np.maximum(z, 0.0) if l < 3 else z)
    Y = acts[-1]
    loss = np.mean((Y - T) ** 2)
    dy = 2.0 * (Y - T) / Y.size
    grads = [None] * 4
    for l in range(3, -1, -1):
        W, _ = layers[l]
        grads[l] = (dy.T @ acts[l], dy.sum(axis=0))
        if l == 0:
            break
        dy = (dy @ _bf16(W)) * (acts[l] > 0)
    flat = np.concatenate([np.concatenate([gw.reshape(-1), gb]) for gw, gb in grads])
    return Y, loss, flat


def test_ws_gradient_matches_cpu_fp64(v2g):
    hidden = 48
    ws = v2g.WarmStart(hidden=hidden, seed=3)
    rng = np.random.default_rng(0)
    X = rng.standard_normal((300, F)).astype(np.float32)
    T = rng.standard_normal((300, O)).astype(np.float32)
    p = ws.params
    Y_cpu, loss_cpu, g_cpu = _cpu_forward_backward(p, hidden, X, T)
    Y_gpu = ws.forward(X)
    assert np.abs(Y_gpu - Y_cpu).max() <= 1e-4 * max(1.0, np.abs(Y_cpu).max())
    loss, g = ws.gradient(X, T)
    assert abs(loss - loss_cpu) <= 1e-5 * loss_cpu
    assert g.shape == g_cpu.shape
    assert np.abs(g - g_cpu).max() <= 2e-3 * np.abs(g_cpu).max()


def test_ws_training_reduces_the_loss(v2g):
    ws = v2g.WarmStart(hidden=64, seed=1)
    rng = np.random.default_rng(1)
    X = rng.standard_normal((2048, F)).astype(np.float32)
    T = np.stack([np.tanh(X[:, 0] - X[:, 3]), X[:, 1] * X[:, 2], 0.5 * X[:, 4]], axis=1).astype(np.float32)
    l0, _ = ws.gradient(X, T)
    l1 = ws.train(X, T, epochs=200, batch_rows=256, lr=2e-3)
    assert l1 < 0.2 * l0


@pytest.mark.late
def test_learned_start_reaches_the_same_energy(v2g):
    from v2rdm_casscf_b200.hamiltonian import synthetic

    opts = dict(R_CONVERGENCE=1e-6, E_CONVERGENCE=1e-7)
    # training data: converged solutions of seeds 100.. (n = 6)
    train = [v2g.V2RDMSolver.from_active_space(synthetic(6, 100 + s), options=opts, start="feasible",
                                               projection="adaptive") for s in range(24)]
    res = v2g.solve_batch(train)
    assert all(r["status"] == 0 for r in res)
    X = np.concatenate([v2g.WarmStart.features(s) for s in train])
    T = np.concatenate([v2g.WarmStart.targets(s) for s in train])
    ws = v2g.WarmStart(hidden=224, seed=0)
    assert 90_000 <= ws.nparams <= 120_000
    l0, _ = ws.gradient(X, T)
    loss = ws.train(X, T, epochs=400, batch_rows=128, lr=1e-3)
    print("warm-start training: loss", l0, "->", loss)
    assert loss < 0.25 * l0
    # held-out seeds: the learned start (with the network's mu, and with mu = 1
    # as the feasible start has it) against the feasible start
    held = [synthetic(6, s) for s in range(6)]
    feas = [v2g.V2RDMSolver.from_active_space(a, options=opts, start="feasible", projection="adaptive") for a in held]
    lrn = [v2g.V2RDMSolver.from_active_space(a, options=opts, start="learned", projection="adaptive") for a in held]
    lr1 = [v2g.V2RDMSolver.from_active_space(a, options=opts, start="learned", projection="adaptive") for a in held]
    for s in lrn:
        ws.propose(s)
    for s in lr1:
        ws.propose(s, use_mu=False)
    rf, rl, r1 = v2g.solve_batch(feas), v2g.solve_batch(lrn), v2g.solve_batch(lr1)
    for a, b, c in zip(rf, rl, r1):
        assert a["status"] == 0 and b["status"] == 0 and c["status"] == 0
        assert abs(a["e_total"] - b["e_total"]) <= 1e-6
        assert abs(a["e_total"] - c["e_total"]) <= 1e-6
    print("ablation (outer iterations per held-out seed: feasible, learned, learned with mu = 1):",
          [(a["oiter"], b["oiter"], c["oiter"]) for a, b, c in zip(rf, rl, r1)])
