"""The learned cost model and the configuration tuner on the GPU.

The MLP's forward pass, gradients, loss gradient and Adam update (the engine's own kernels,
csrc/mlp.cu) are checked against the float64 oracle (oracle/mlp_oracle.py); training on a known
function must converge; and the tuner, trained on timings the engine measures on a sweep of
problems, must pick on held-out problems only configurations whose measured error meets the
tolerance, faster than the reference heuristic (where that one meets it) and than the rule
"heuristic width + 1, default method and tile" by stated margins, after measuring fewer
candidates than exhaustive autotuning.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_mlp_kernels_match_oracle(cuda, engine):
    import torch
    from neonufft_b200.costmodel import MLP
    from oracle import mlp_oracle as MO
    rng = np.random.default_rng(9)
    widths = [7, 16, 12, 1]
    net = MLP(widths, seed=4)
    x = torch.from_numpy(rng.standard_normal((33, 7)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal(33).astype(np.float32)).cuda()
    p = net.params.cpu().numpy().astype(np.float64)
    xs = x.cpu().numpy().astype(np.float64)
    acts, out = net.forward(x)
    ref_acts = MO.forward(widths, p, xs)
    assert np.allclose(out.cpu().numpy().reshape(-1), ref_acts[-1].reshape(-1), rtol=1e-5, atol=1e-5)
    loss, dy = net.mse(out, t)
    ref_loss, ref_dy = MO.mse(ref_acts[-1], t.cpu().numpy())
    assert abs(float(loss.item()) - ref_loss) <= 1e-5 * max(1.0, ref_loss)
    net.backward(x, acts, dy.view(out.shape))
    ref_g = MO.backward(widths, p, xs, ref_acts, ref_dy.reshape(-1, 1))
    g = net.grads.cpu().numpy()
    assert np.max(np.abs(g - ref_g)) <= 1e-4 * max(1.0, np.max(np.abs(ref_g)))
    net.adam(lr=1e-2)
    ref_p, _, _ = MO.adam(p, ref_g, np.zeros_like(p), np.zeros_like(p), 1e-2, 0.9, 0.999, 1e-8, 1)
    assert np.max(np.abs(net.params.cpu().numpy() - ref_p)) <= 1e-5


def test_mlp_training_converges(cuda, engine):
    import torch
    from neonufft_b200.costmodel import MLP
    rng = np.random.default_rng(2)
    xs = rng.uniform(-1, 1, (512, 3))
    ys = np.sin(2 * xs[:, 0]) + xs[:, 1] ** 2 - 0.5 * xs[:, 2]
    net = MLP([3, 32, 32, 1], seed=1)
    x = torch.from_numpy(xs.astype(np.float32)).cuda()
    y = torch.from_numpy(ys.astype(np.float32)).cuda().view(-1, 1)
    first = float(net.mse(net.forward(x)[1], y)[0].item())
    final = net.fit(x, y, epochs=1500, lr=1e-2)
    assert final < 2e-3 and final < first / 50


# Margins the learned picks must keep on the held-out problems (geometric means of the other
# configuration's time over the pick's time, where that configuration meets tol).
MARGIN_VS_HEURISTIC = 1.10
MARGIN_VS_RULE_PLUS_ONE = 1.05


def _problems(T, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        dim = 2 if i % 2 == 0 else 3
        N = int(rng.choice([48, 64, 96]) if dim == 3 else rng.choice([128, 256, 512]))
        M = int(10 ** rng.uniform(5.0, 6.3))
        tol = float(rng.choice([1e-3, 1e-6]))
        out.append(T.Problem(dim=dim, type=int(1 + i % 3 // 2), M=M, N=N, tol=tol,
                             blob=bool(i % 4 == 3), seed=i))
    return out


def test_tuner_picks_meet_tol_and_beat_the_rules(cuda, engine):
    """On held-out problems the learned picks meet tol, run faster than the reference heuristic
    (where it meets tol) and than the width-plus-one rule by the stated margins, and measure
    far fewer candidates than exhaustive autotuning."""
    from neonufft_b200 import tuner as T
    problems = _problems(T, 52, 11)
    train, held = problems[:40], problems[40:]
    tuner = T.Tuner()
    tuner.sweep(train)
    loss = tuner.train(epochs=3000)
    assert math.isfinite(loss)
    ev = T.evaluate(tuner, held)
    print("\ntuner on held-out problems:", ev)
    assert ev["picks_missing_tol"] == 0
    assert ev["speedup_vs_rule_plus_one_geomean"] >= MARGIN_VS_RULE_PLUS_ONE, ev
    if ev["speedup_vs_heuristic_geomean"] is not None:
        assert ev["speedup_vs_heuristic_geomean"] >= MARGIN_VS_HEURISTIC, ev
    assert ev["measurements_per_pick"] <= 0.6 * ev["measurements_exhaustive"], ev


def test_trained_tuner_round_trips_through_a_file(tmp_path, cuda, engine):
    """A trained cost model and its rows saved and loaded again rank candidates identically
    (the network's parameters and feature standardisation are restored exactly)."""
    from neonufft_b200 import tuner as T
    rng = np.random.default_rng(3)
    t = T.Tuner()
    for i in range(12):
        p = T.Problem(dim=2 + i % 2, type=1 + i % 3 // 2, M=int(10 ** rng.uniform(4, 6)),
                      N=int(rng.choice([32, 64, 128])), tol=float(rng.choice([1e-3, 1e-6])),
                      seed=i)
        for c in T.candidates(p):
            f = T.features(p, c)
            t.rows.append((f, float(0.1 * f[2] + 0.05 * f[9] + rng.normal(0, 0.01)), 1e-7, p, c))
    t.train(epochs=300)
    path = tmp_path / "tuner.json"
    t.save(path)
    u = T.Tuner.load(path)
    feats = np.stack([r[0] for r in t.rows])
    assert np.array_equal(t.model.predict(feats), u.model.predict(feats))
