"""The learned insertion scheduler: its CPU oracle, the device training
kernels (gradients against the oracle), the fused BF16 inference (against a
BF16-emulating restatement), the training log, and the scheduler itself --
same tet set as the plain method, and the gain it brings."""
import os

import numpy as np
import pytest

import fixtures as fx
from oracle import mlp as OM


def _random_params(seed, scale=1.0):
    r = np.random.default_rng(seed)
    d = {}
    for name, shape in OM.SIZES:
        fan = shape[-1] if len(shape) == 2 else OM.H
        d[name] = r.normal(0, scale / np.sqrt(fan), shape) if name.startswith("W") else r.normal(0, 0.1, shape)
    return OM.pack(d)


def _samples(n, seed):
    r = np.random.default_rng(seed)
    X = r.normal(0, 1, (n, OM.IN)).astype(np.float32)
    y = (r.random(n) < 0.3).astype(np.float32)
    return X, y


# ---------------------------------------------------------------- CPU ----

def test_oracle_gradient_matches_finite_differences():
    X, y = _samples(64, 1)
    p = _random_params(2)
    loss, g = OM.loss_grad(X, y, p)
    r = np.random.default_rng(3)
    for j in r.choice(OM.NUM_PARAMS, 60, replace=False):
        e = np.zeros(OM.NUM_PARAMS)
        e[j] = 1e-6
        num = (OM.loss_grad(X, y, p + e)[0] - OM.loss_grad(X, y, p - e)[0]) / 2e-6
        assert abs(num - g[j]) <= 1e-6 + 1e-4 * abs(num), (j, num, g[j])
    assert np.isclose(loss, np.mean(np.logaddexp(0, OM.forward(X, p)) - y * OM.forward(X, p)))


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-8, 1.0 + 2**-9, -2.5, 3.0e38], np.float32)
    want = np.array([1.0, 1.0, 1.0 + 2**-6, 1.0, -2.5, 2.9908e38], np.float32)
    got = OM.bf16(vals)
    assert np.array_equal(got[:5], want[:5])
    assert abs(got[5] / vals[5] - 1) < 2**-8


def test_parameter_layout_matches_header(wt):
    from wtet_b200 import learned

    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "wtet.h")).read()
    assert f"#define WTET_MLP_PARAMS {learned.NUM_PARAMS}" in hdr
    assert f"#define WTET_MLP_FEATURES {learned.NUM_FEATURES}" in hdr
    assert learned.NUM_PARAMS == OM.NUM_PARAMS
    assert len(learned.FEATURES) == learned.NUM_FEATURES == OM.IN
    p = _random_params(4).astype(np.float32)
    assert np.array_equal(learned.pack(learned.unpack(p)), p)


def test_standardisation_folds_into_first_layer(wt):
    from wtet_b200 import learned

    X, _ = _samples(200, 5)
    X = X * np.float32(3) + np.float32(1.5)
    mean, std = X.mean(0).astype(np.float64), X.std(0).astype(np.float64)
    p = _random_params(6)
    folded = learned.fold_standardization(p, mean, std)
    a = OM.forward((X - mean) / std, p)
    b = OM.forward(X, folded.astype(np.float64))
    assert np.allclose(a, b, rtol=1e-4, atol=1e-4)


def test_packaged_weights_are_valid(wt):
    from wtet_b200 import learned

    with np.load(learned.DEFAULT_WEIGHTS) as z:
        p = z["params"]
        assert p.shape == (learned.NUM_PARAMS,) and p.dtype == np.float32
        assert np.isfinite(p).all()
        assert float(z["val_accuracy"]) > float(z["majority"])


# ---------------------------------------------------------------- GPU ----

@pytest.mark.gpu
def test_device_gradients_match_oracle(gpu):
    from wtet_b200 import learned

    for n, seed in ((1, 7), (37, 8), (3000, 9)):
        X, y = _samples(n, seed)
        p = _random_params(seed).astype(np.float32)
        loss, g = learned.loss_grad(X, y, p)
        want_loss, want = OM.loss_grad(X, y, p.astype(np.float64))
        assert abs(loss - want_loss) <= 1e-5 * max(1.0, abs(want_loss))
        # FP32 kernels against a float64 restatement
        assert np.abs(g - want).max() <= 1e-5 * np.abs(want).max() + 1e-7, n


@pytest.mark.gpu
def test_fused_inference_matches_bf16_restatement(gpu):
    from wtet_b200 import learned

    X, _ = _samples(5000, 10)
    p = _random_params(11).astype(np.float32)
    learned.set_weights(p)
    got = learned.score(X)
    want = OM.score_bf16(X, p)
    exact = OM.forward(X, p)
    # BF16 operands with FP32 sums: only the summation order differs from the restatement
    assert np.abs(got - want).max() <= 2e-3 * max(1.0, np.abs(want).max())
    # and BF16 stays close to the FP32 network
    assert np.corrcoef(got, exact)[0, 1] > 0.999


@pytest.mark.gpu
def test_training_is_deterministic_and_learns(gpu):
    from wtet_b200 import learned

    r = np.random.default_rng(12)
    X = r.normal(0, 1, (20000, 12)).astype(np.float32)
    y = ((X[:, 0] - 0.5 * X[:, 3] + 0.25 * X[:, 8] ** 2) > 0.3).astype(np.float32)
    p1, l1 = learned.train(X, y, epochs=5, batch=1024, lr=3e-3, seed=1)
    p2, l2 = learned.train(X, y, epochs=5, batch=1024, lr=3e-3, seed=1)
    assert np.array_equal(p1, p2) and np.array_equal(l1, l2)
    assert l1[-1] < 0.5 * l1[0]
    learned.set_weights(p1)
    acc = ((learned.score(X) > 0) == (y > 0.5)).mean()
    assert acc > 0.95


@pytest.mark.gpu
def test_collect_records(gpu):
    from wtet_b200 import learned

    pts = fx.mixture(50_000, 21)
    X, y, st = learned.collect([pts], sample_shift=0)
    assert 0 < X.shape[0] == y.shape[0] <= st["vote_winners"]
    assert np.isfinite(X).all()
    assert set(np.unique(y)) == {0, 1}                     # inserted in its round, or not
    assert (X[:, 0] >= 0).all() and (X[:, 0] <= 1).all()   # circumcenter distance
    assert (X[:, 4] >= 0).all() and (X[:, 4] <= 1).all()   # rival neighbours / 4
    assert (X[:, 5] >= 0).all() and (X[:, 5] <= X[:, 4]).all()  # better-scored rivals among the rivals
    assert (X[:, 8] >= 0).all() and (X[:, 8] <= 1).all()   # stratum progress
    assert set(np.unique(X[:, 11])) <= {0.0, 1.0}          # super-vertex flag
    # a winner that shares its neighbourhood with other winners inserts less often
    crowded = X[:, 4] > np.median(X[:, 4])
    assert y[crowded].mean() < y[~crowded].mean()
    # the gate: with a small one only the small rounds are recorded
    Xs, _, _ = learned.collect([pts], gpu.Config(learned_gate=1), sample_shift=0)
    assert Xs.shape[0] < X.shape[0]
    assert (Xs[:, 9] <= np.log2(1 + 1024) / 24 + 1e-6).all()


LEARNED_CASES = ["cube", "icosahedron", "grid12", "lattice24", "shell5k", "unit_sphere20k", "uniform100k",
                 "clusters", "mixture50k", "duplicates", "coplanar_offset"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", LEARNED_CASES)
def test_learned_scheduler_parity(gpu, oracle_mod, name):
    from test_gpu_parity import CASES, assert_parity

    assert_parity(gpu, oracle_mod, CASES[name](), gpu.Config(vote="learned"))


@pytest.mark.gpu
def test_trained_network_predicts_insertions(gpu):
    """What the trained network knows: on records logged from clouds it was
    not trained on, its prediction of which gated winners insert beats the
    base rate (lower cross-entropy, AUC well above chance)."""
    from wtet_b200 import learned

    learned.load_default()
    for pts in (fx.mixture(300_000, 202), fx.lattice(40)):
        X, y, _ = learned.collect([pts], sample_shift=0)
        logit = learned.score(X).astype(np.float64)
        y = y.astype(np.float64)
        bce = np.mean(np.logaddexp(0, logit) - y * logit)
        q = y.mean()
        base = -(q * np.log(q) + (1 - q) * np.log(1 - q))
        auc = learned.roc_auc(logit, y)
        print(f"records {len(y)} inserted {q:.3f} bce {bce:.4f} base-rate entropy {base:.4f} auc {auc:.3f}")
        assert bce < base - 0.01
        assert auc > 0.65


@pytest.mark.gpu
def test_learned_scheduler_gain(gpu):
    """What the learned scheduler gains over the plain one on its
    configuration, an 8M-point mixture cloud from a seed no training run saw:
    the same tet set in fewer insertion rounds and less device time (median
    of five runs each, interleaved)."""
    import torch

    pts = fx.mixture(8_000_000, 106)
    d_pts = torch.from_numpy(pts).cuda()
    cfg_plain, cfg_learned = gpu.Config(), gpu.Config(vote="learned")
    runs = {"plain": [], "learned": []}
    digests = {}
    for k in range(6):
        for name, cfg in (("plain", cfg_plain), ("learned", cfg_learned)):
            t, a, st = gpu.delaunay_device(d_pts, cfg, with_stats=True)
            if k:
                runs[name].append(st)
            else:
                digests[name] = gpu.canonical_digest(*gpu.canonical_device(t, a, len(pts)))
            del t, a
    assert digests["plain"] == digests["learned"]
    med = {name: float(np.median([s["device_ms"] for s in r])) for name, r in runs.items()}
    rounds = {name: float(np.median([s["rounds"] for s in r])) for name, r in runs.items()}
    print(f"device ms {med}, rounds {rounds}")
    assert rounds["learned"] < 0.95 * rounds["plain"]
    assert med["learned"] < med["plain"]
