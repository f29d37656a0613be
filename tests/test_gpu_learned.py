"""GPU: the learned k-th-score model.

The training kernels' gradients and the inference kernel are checked against the
FP64 CPU oracle (oracle/mlp_oracle.py); a fitted model is then used as the
starting threshold of pruned queries, whose results must equal the exact top-k,
and it must scan fewer partitions than the method without it.
"""
import numpy as np
import pytest

import topk_b200 as T
from oracle import mlp_oracle as M
from oracle import oracle as O
from tests import helpers as H
from topk_b200 import learned as L

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("F,B", [(25, 128), (33, 100), (5, 1)])
def test_mlp_gradient_matches_fp64_oracle(F, B):
    rng = np.random.default_rng(F * 1000 + B)
    p = L.init_params(F, seed=F, bias=0.3)
    p[F * 64:F * 64 + 64] = rng.normal(0, 0.1, 64)  # non-zero hidden biases
    X = rng.uniform(0, 1, (B, F)).astype(np.float32)
    y = rng.uniform(0, 1, B).astype(np.float32)
    loss, g = L.grad(p, X, y)
    want_loss, want = M.loss_grad(p.astype(np.float64), X.astype(np.float64), y.astype(np.float64))
    assert abs(loss - want_loss) <= 1e-5 * max(1.0, want_loss)
    # FP32 sums of at most 128 terms against FP64: relative to the gradient's scale
    scale = np.abs(want).max()
    err = np.abs(g.astype(np.float64) - want).max()
    print(f"F={F} B={B}: max |grad - grad_fp64| = {err:.3e} (scale {scale:.3e})")
    assert err <= 1e-4 * scale


def test_mlp_predict_matches_fp64_oracle():
    rng = np.random.default_rng(1)
    F = 25
    p = L.init_params(F, seed=3, bias=0.1)
    X = rng.uniform(0, 1, (1000, F)).astype(np.float32)
    got = L.predict(p, X)
    want, _, _ = M.forward(p.astype(np.float64), X.astype(np.float64))
    assert np.abs(got - want).max() <= 1e-4 * max(1.0, np.abs(want).max())


def test_mlp_training_fits_a_smooth_target():
    rng = np.random.default_rng(2)
    F, N = 10, 20000
    X = rng.uniform(0, 1, (N, F)).astype(np.float32)
    y = (np.sin(3 * X[:, 0]) + X[:, 1] * X[:, 2] + 0.5 * X[:, 3]).astype(np.float32)
    p0 = L.init_params(F, seed=4, bias=float(y.mean()))
    p, losses = L.train(p0, X, y, epochs=8, lr=2e-3, seed=5)
    assert losses[-1] < 0.1 * losses[0]
    pred = L.predict(p, X[:2000])
    assert np.sqrt(np.mean((pred - y[:2000]) ** 2)) < 0.1
    assert np.all(np.isfinite(p))


def random_queries(rng, nq, d, kmin=16, kmax=1024):
    ks = np.exp(rng.uniform(np.log(kmin), np.log(kmax + 1), nq)).astype(np.uint64).clip(kmin, kmax)
    W = ((rng.integers(0, 1 << 24, size=(nq, d)) + 1) * 2.0 ** -24).astype(np.float32)
    A = np.zeros((nq, d), np.uint8)
    qqs = np.zeros(nq, np.uint32)
    for j in range(nq):
        q = int(rng.integers(2, d + 1))
        A[j, :q] = np.sort(rng.choice(d, size=q, replace=False))
        qqs[j] = q
    return ks, W, A, qqs


def test_features_match_host_restatement():
    n, d = 200000, 8
    rng = np.random.default_rng(6)
    with T.Table(n, d) as t:
        t.generate(2, 1)
        t.normalize()
        t.build_partitions(4096)
        R, mins, maxs, means = t.partition_info()
        ks, W, A, qqs = random_queries(rng, 20, d)
        X, S = t.query_features(ks, W, A, qqs)
        for j in range(20):
            a = A[j, :qqs[j]]
            w = W[j][a]
            s = np.abs(w).sum()
            assert np.isclose(S[j], s, rtol=1e-6)
            bnd = np.sort((maxs[:, a] * w).sum(axis=1))[::-1]
            mu = np.sort((means[:, a] * w).sum(axis=1))[::-1]
            ranks = [min(1 << r, len(bnd)) - 1 for r in range(8)]
            wf = np.zeros(d)
            np.add.at(wf, a, w / s)
            lw = np.where(wf != 0, np.log(np.abs(np.where(wf != 0, wf, 1))), 0)
            want = np.concatenate([wf, lw, [np.log2(float(ks[j])) / 10, qqs[j] / 16], bnd[ranks] / s, mu[ranks] / s])
            assert np.allclose(X[j], want, rtol=1e-5, atol=1e-5)


def test_learned_fit_and_exact_queries_gain_over_plain_pruning():
    n, d = (1 << 21) + 5, 8
    rng = np.random.default_rng(7)
    with T.Table(n, d) as t:
        t.generate(2, 11)  # anticorrelated
        t.normalize()
        t.build_partitions(8192)
        tn = t.download()
        rep = t.learned_fit(n_train=16384, n_val=2048, kmin=16, kmax=1024, qmin=2, qmax=d, epochs=12,
                            miss_rate=0.02, seed=1)
        print("fit:", rep)
        # target u = qq * ln(gap / S): an error e in u scales the objects above the cut by about e^e
        assert np.isfinite(rep["val_rmse"]) and np.isfinite(rep["margin"])
        ks, W, A, qqs = random_queries(rng, 60, d)
        plain, learned, accepted, scans_l, scans_p = [], [], 0, [], []
        for j in range(60):
            a = A[j, :qqs[j]]
            want = O.topk_numpy(tn, int(ks[j]), W[j], a)
            ids, sc, th, st, cut = t.query_learned(int(ks[j]), W[j], a)
            H.assert_same_result((ids, sc, th), want)
            ids2, sc2, th2, st2 = t.query_pruned(int(ks[j]), W[j], a)
            H.assert_same_result((ids2, sc2, th2), want)
            accepted += st[2]
            learned.append(st[0])
            plain.append(st2[0])
            scans_l.append(st[3])
            scans_p.append(st2[3])
        print(f"accepted {accepted}/60, partitions scanned: learned {np.mean(learned):.1f}, "
              f"plain {np.mean(plain):.1f} of {st[1]}; scans per query: learned {np.mean(scans_l):.2f}, "
              f"plain {np.mean(scans_p):.2f}")
        assert accepted >= 50
        # the gain: plain pruning first scans the best partitions to learn a threshold
        # (two scans per query); the model's cut lets one scan start from a threshold
        assert np.mean(scans_l) < 0.6 * np.mean(scans_p)


def test_batched_learned_start_is_exact_and_cuts_candidates():
    n, d = (1 << 21) + 77, 16
    rng = np.random.default_rng(8)
    with T.Table(n, d) as t:
        t.generate(1, 5)
        t.normalize()
        t.build_partitions(8192)
        rep = t.learned_fit(n_train=8192, n_val=1024, kmin=1, kmax=1024, qmin=2, qmax=16, epochs=10,
                            miss_rate=0.01, seed=2)
        print("fit:", rep)
        ks, W, A, qqs = random_queries(rng, 300, d, kmin=1, kmax=1024)
        t.set_batch_method(T.BATCH_FP32)
        want = t.query_batch(ks, W, A, qqs)
        t.set_batch_method(T.BATCH_BF16)
        t.query_batch(ks, W, A, qqs)
        plain = t.last_batch_stats()
        t.set_batch_method(T.BATCH_LEARNED)
        got = t.query_batch(ks, W, A, qqs)
        st = t.last_batch_stats()
        print("bf16:", plain, "learned:", st)
        assert st["method"] == T.BATCH_LEARNED
        for x, y in zip(got, want):
            assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))
        assert st["candidates"] < 0.5 * plain["candidates"]
        assert st["learned_misses"] <= 15
        # a model that predicts far too high: every query misses and is answered again
        p, m = t.get_learned_model()
        p2 = p.copy()
        p2[-1] -= 100.0  # u far below: the cut sits at the largest bound
        t.set_learned_model(p2, m)
        got = t.query_batch(ks, W, A, qqs)
        assert t.last_batch_stats()["learned_misses"] == len(ks)
        for x, y in zip(got, want):
            assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))
