"""The autotuner's learned cost model: the CPU oracle of the network is
checked by finite differences, the CUDA forward/backward/Adam kernels
against the oracle, and the trained network against the method without it
on held-out bins of a measured B200 tuning sweep."""
from __future__ import annotations

import json
import math
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import mlp_oracle as O  # noqa: E402

from saruman_b200 import costmodel as CM  # noqa: E402

SWEEP = CM.SWEEP
DIMS = [CM.N_FEATURES, 32, 32, 1]


def random_case(n=257, seed=0):
    rng = np.random.default_rng(seed)
    count = sum(a * b + b for a, b in zip(DIMS[:-1], DIMS[1:]))
    p = rng.normal(0, 0.4, count)
    X = rng.uniform(0, 1, (n, DIMS[0]))
    y = rng.normal(0, 1, n)
    return p, X, y


def test_oracle_gradient_matches_finite_differences():
    p, X, y = random_case(n=31, seed=1)
    _, g = O.loss_grad(p, DIMS, X, y)
    rng = np.random.default_rng(2)
    for i in rng.choice(p.size, 40, replace=False):
        e = np.zeros_like(p)
        e[i] = 1e-6
        fd = (O.loss_grad(p + e, DIMS, X, y)[0] - O.loss_grad(p - e, DIMS, X, y)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i])


def test_features_are_bounded():
    f = CM.features(250, 15, 1.0, 4_000_000, (4, 3, 64))
    assert f.shape == (CM.N_FEATURES,) and np.all(f >= 0) and np.all(f <= 1.5)


@pytest.mark.gpu
def test_kernels_match_the_oracle(saru_lib):
    """fp32 kernels vs the float64 oracle: forward, loss, every gradient
    entry, and one Adam step (tolerance 1e-4 relative + 1e-5 absolute)."""
    import torch
    p, X, y = random_case()
    net = CM.CostModel(seed=0)
    net.params = torch.from_numpy(p.astype(np.float32)).cuda()
    pf = p.astype(np.float32).astype(np.float64)
    Xf = X.astype(np.float32).astype(np.float64)
    yf = y.astype(np.float32).astype(np.float64)
    out = net.forward_raw(X)
    np.testing.assert_allclose(out, O.forward(pf, DIMS, Xf)[-1][:, 0], rtol=1e-4, atol=1e-5)
    loss, g = net.loss_grad(X, y)
    loss_o, g_o = O.loss_grad(pf, DIMS, Xf, yf)
    assert abs(loss - loss_o) <= 1e-4 * abs(loss_o) + 1e-5
    np.testing.assert_allclose(g, g_o, rtol=1e-4, atol=1e-5)
    # one Adam step on the device against the oracle's
    lib = net.lib
    m = torch.zeros_like(net.params)
    v = torch.zeros_like(net.params)
    gd = torch.from_numpy(g.astype(np.float32)).cuda()
    assert lib.saru_mlp_adam_step(net.params.data_ptr(), gd.data_ptr(), m.data_ptr(),
                                  v.data_ptr(), net.params.numel(), 1e-2, 0.9, 0.999, 1e-8, 1,
                                  None) == 0
    torch.cuda.synchronize()
    p1, _, _ = O.adam(pf, g.astype(np.float64), 0 * pf, 0 * pf, 1e-2, 0.9, 0.999, 1e-8, 1)
    np.testing.assert_allclose(net.params.cpu().numpy(), p1, rtol=1e-5, atol=1e-6)


def load_sweep():
    data = json.loads(SWEEP.read_text())
    bins = {}
    for r in data["rows"]:
        bins.setdefault((r["m"], r["k"], r["n"]), []).append(r)
    return data, bins


def default_equivalent(k):
    """The library's default shape as it runs: 4 warps per CTA, as many
    CTAs per SM as fit, 32-bit band words for k <= 7."""
    return [4, 0, 32 if k <= 7 else 64]


@pytest.mark.gpu
def test_trained_model_beats_the_method_without_it(saru_lib):
    """Trained on the bins of six read lengths, the network ranks the launch
    shapes of the two held-out read lengths.  Without it the tuner either
    keeps the default shape (no trials) or times the whole search space
    (12-24 trials per bin).  With it, its top-ranked shape alone is at
    least as fast as the default on average, and timing its top 3 comes
    within 3% of the exhaustive search's best."""
    data, bins = load_sweep()
    held = {75, 200}
    train = [r for key, rs in bins.items() if key[0] not in held for r in rs]
    X, y = CM.dataset(train)
    net = CM.CostModel(seed=0)
    hist = net.fit(X, y, steps=3000)
    assert hist[-1] < 0.25 * hist[0]
    r_top1, r_top3, r_default, trials = [], [], [], []
    for (m, k, n), rs in bins.items():
        if m not in held:
            continue
        ms = {tuple(r["shape"]): r["ms"] for r in rs}
        best = min(ms.values())
        ranked = net.rank(m, k, rs[0]["so_frac"], n, list(ms))
        r_top1.append(ms[ranked[0]] / best)
        r_top3.append(min(ms[s] for s in ranked[:3]) / best)
        r_default.append(ms[tuple(default_equivalent(k))] / best)
        trials.append(len(ms))
    top1, top3, dflt = (float(np.mean(v)) for v in (r_top1, r_top3, r_default))
    print(f"held-out bins {len(r_top1)}: default/best {dflt:.3f}, model top-1/best {top1:.3f}, "
          f"model top-3/best {top3:.3f} (3 trials instead of {np.mean(trials):.1f})")
    assert top1 <= dflt + 1e-9
    assert top3 <= 1.03
