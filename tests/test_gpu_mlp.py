"""The surrogate MLP on tensor cores (tcgen05 BF16 GEMM), checked against the
numpy oracle of oracle/mlp_oracle.py: the GEMM, one batch's gradients, and
that training fits a log-likelihood surface."""
import numpy as np
import pytest

from oracle import mlp_oracle as MO

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 128, 192), (384, 64, 128),
                                   (128, 256, 512), (256, 64, 4096)])
def test_tcgen05_gemm_matches_numpy(gpu, M, N, K):
    rng = np.random.default_rng(M + N + K)
    A = rng.standard_normal((M, K)).astype(np.float32)
    B = rng.standard_normal((N, K)).astype(np.float32)
    C = gpu.gemm_check(A, B)
    ref = MO.bf16(A) @ MO.bf16(B).T
    assert np.max(np.abs(C - ref)) <= 1e-4 * np.sqrt(K) * np.max(np.abs(ref)) + 1e-5


def _quadratic_pairs(d, n, seed):
    rng = np.random.default_rng(seed)
    mu = rng.normal(0, 1, d)
    A = rng.normal(0, 1, (d, d))
    P = A @ A.T / d + np.eye(d)
    theta = mu + rng.normal(0, 1, (n, d))
    dev = theta - mu
    ll = -0.5 * np.einsum("ni,ij,nj->n", dev, P, dev) * 100.0 - 2.5e4
    return theta, ll


@pytest.mark.parametrize("d,H", [(5, 256), (65, 512)])
def test_gradients_match_cpu_oracle(gpu, d, H):
    theta, ll = _quadratic_pairs(d, 300, 1)
    s = gpu.Surrogate(d, hidden=H, batch=384, seed=3)
    xm, xs = theta.mean(0), theta.std(0)
    ym, ys = ll.mean(), ll.std()
    s.set_normalizer(xm, xs, ym, ys)
    g, loss = s.gradients(theta, ll)
    # the GPU standardises in f32 with f32 copies of the mean and 1/sd
    X = MO.f32((theta.astype(np.float32) - xm.astype(np.float32)) * (1.0 / xs).astype(np.float32))
    t = MO.f32((ll - MO.f32(ym)) * MO.f32(1.0 / ys))
    ref_loss, ref = MO.forward_backward(s.params(), d, H, X, t)
    assert abs(loss - ref_loss) <= 1e-4 * abs(ref_loss)
    names = ["dW1", "db1", "dW2", "db2", "dw3", "db3"]
    off = 0
    for name, r in zip(names, ref):
        got = g[off:off + r.size].reshape(r.shape)
        off += r.size
        rel = np.linalg.norm(got - r) / max(np.linalg.norm(r), 1e-30)
        assert rel < 5e-3, (name, rel)


def test_training_fits_a_loglik_surface(gpu):
    d = 5
    theta, ll = _quadratic_pairs(d, 1 << 16, 2)
    s = gpu.Surrogate(d, hidden=256, batch=4096, seed=1)
    s.fit_normalizer(theta, ll)
    losses = s.train(theta, ll, steps=1500, lr=2e-3)
    assert losses[-50:].mean() < 0.02 * losses[:10].mean()
    test_theta, test_ll = _quadratic_pairs(d, 2000, 2)
    pred = s.predict(test_theta)
    resid = pred - test_ll
    r2 = 1 - resid.var() / test_ll.var()
    assert r2 > 0.99, r2
    s2 = gpu.Surrogate(d, hidden=256, batch=4096, seed=1)
    s2.fit_normalizer(theta, ll)
    losses2 = s2.train(theta, ll, steps=20, lr=2e-3)
    assert np.array_equal(losses[:20], losses2)   # fixed-order reductions: repeatable


@pytest.mark.parametrize("d,H,whiten", [(5, 128, False), (17, 256, True), (17, 256, False),
                                        (65, 512, False)])
def test_inference_matches_cpu_oracle(gpu, d, H, whiten):
    # d <= 64 with H in {128, 256} runs the fused tcgen05 inference kernel,
    # the others the layer-by-layer path; both against the numpy forward
    theta, ll = _quadratic_pairs(d, 1000, 4)
    s = gpu.Surrogate(d, hidden=H, batch=512, seed=5)
    s.fit_normalizer(theta, ll, whiten=whiten)
    s.train(theta, ll, steps=40, lr=2e-3)
    got = s.predict(theta[:300])
    th = theta[:300].astype(np.float32)
    mu = theta.mean(axis=0).astype(np.float32)
    if whiten:
        cov = np.cov(theta, rowvar=False)
        cov = cov + np.eye(d) * 1e-10 * max(float(np.mean(np.diag(cov))), 1e-300)
        W = np.linalg.inv(np.linalg.cholesky(cov)).astype(np.float32)
        X = MO.f32((th - mu) @ W.T)
    else:
        X = MO.f32((th - mu) * (1.0 / theta.std(axis=0)).astype(np.float32))
    ym, ys = float(np.mean(ll)), float(np.std(ll))
    ref = MO.predict(s.params(), d, H, X) * MO.f32(ys) + MO.f32(ym)
    scale = np.std(ref)
    assert np.max(np.abs(got - ref)) < 2e-2 * scale, np.max(np.abs(got - ref)) / scale
    assert np.corrcoef(got, ref)[0, 1] > 0.9999
