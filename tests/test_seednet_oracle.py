"""CPU checks of the seed-network oracle (oracle/seednet_np.py): bfloat16
rounding, the analytic loss gradient and the back-propagated parameter
gradient against central finite differences in FP64, and the loss's
invariance to the basis chosen for the reference eigenvectors."""
import numpy as np

from oracle import seednet_np as sn


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 3.0e-3, 0.0])
    got = sn.bf16(x)
    assert got[0] == 1.0
    assert got[1] == 1.0                       # tie -> even mantissa
    assert got[2] == 1.0 + 2.0 ** -6           # tie -> even mantissa
    assert got[3] == -2.5
    assert abs(got[4] - 3.0e-3) <= 3.0e-3 * 2.0 ** -8
    assert got[5] == 0.0


def _problem(seed, B=2, H=6, W=8):
    rng = np.random.default_rng(seed)
    V = -50.0 * rng.random((B, H, W))
    U = np.stack([np.linalg.qr(rng.standard_normal((H * W, sn.NOUT)))[0] for _ in range(B)])
    return V, U


def test_loss_gradient_finite_differences():
    rng = np.random.default_rng(3)
    Y = rng.standard_normal((2, 40, sn.NOUT))
    U = np.stack([np.linalg.qr(rng.standard_normal((40, sn.NOUT)))[0] for _ in range(2)])
    L, dY = sn.loss_terms(Y, U, lam=0.7)
    for _ in range(5):
        d = rng.standard_normal(Y.shape)
        h = 1e-6
        fd = (sn.loss_terms(Y + h * d, U, 0.7)[0].sum() - sn.loss_terms(Y - h * d, U, 0.7)[0].sum()) / (2 * h)
        assert abs(fd - np.sum(dY * d)) <= 1e-6 * max(1.0, abs(fd))


def test_parameter_gradient_finite_differences():
    V, U = _problem(5)
    p = sn.init_params(11)
    L, g = sn.loss_and_grad(p, V, U, lam=0.5, emulate=False)
    rng = np.random.default_rng(7)
    mask = np.concatenate([np.concatenate([
        np.pad(np.ones((sn.TAPS, sn.CIN[l], sn.COUT[l])), ((0, 0), (0, sn.NC - sn.CIN[l]), (0, sn.NC - sn.COUT[l]))).reshape(-1),
        np.pad(np.ones(sn.COUT[l]), (0, sn.NC - sn.COUT[l]))]) for l in range(5)])
    # Gradient entries outside the real channels are zero.
    assert np.all(g[mask == 0] == 0.0)
    for _ in range(4):
        d = rng.standard_normal(p.size) * mask
        # Small steps: larger ones cross ReLU kinks.
        h = 1e-7
        lp = sn.loss_and_grad(p + h * d, V, U, 0.5, emulate=False)[0].mean()
        lm = sn.loss_and_grad(p - h * d, V, U, 0.5, emulate=False)[0].mean()
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g @ d) <= 1e-6 * max(1.0, abs(fd)), (fd, g @ d)


def test_per_layer_finite_differences():
    V, U = _problem(9)
    p = sn.init_params(13)
    _, g = sn.loss_and_grad(p, V, U, lam=1.0, emulate=False)
    rng = np.random.default_rng(1)
    for l in range(5):
        d = np.zeros(p.size)
        base = l * sn.LAYER_LEN
        W = rng.standard_normal((sn.TAPS, sn.NC, sn.NC))
        W[:, sn.CIN[l]:, :] = 0.0
        W[:, :, sn.COUT[l]:] = 0.0
        d[base:base + sn.TAPS * sn.NC * sn.NC] = W.reshape(-1)
        d[base + sn.TAPS * sn.NC * sn.NC:base + sn.LAYER_LEN][:sn.COUT[l]] = rng.standard_normal(sn.COUT[l])
        h = 1e-7
        fd = (sn.loss_and_grad(p + h * d, V, U, 1.0, emulate=False)[0].mean()
              - sn.loss_and_grad(p - h * d, V, U, 1.0, emulate=False)[0].mean()) / (2 * h)
        assert abs(fd - g @ d) <= 1e-6 * max(1.0, abs(fd)), (l, fd, g @ d)


def test_loss_invariant_to_reference_basis():
    V, U = _problem(21)
    p = sn.init_params(2)
    Q = np.linalg.qr(np.random.default_rng(0).standard_normal((sn.NOUT, sn.NOUT)))[0]
    L1, g1 = sn.loss_and_grad(p, V, U, 1.0, emulate=False)
    L2, g2 = sn.loss_and_grad(p, V, U @ Q, 1.0, emulate=False)
    np.testing.assert_allclose(L1, L2, rtol=1e-12)
    np.testing.assert_allclose(g1, g2, rtol=1e-9, atol=1e-12)


def test_emulated_path_is_close_to_fp64():
    V, U = _problem(4)
    p = sn.init_params(6)
    L1, g1 = sn.loss_and_grad(p, V, U, 1.0, emulate=False)
    L2, g2 = sn.loss_and_grad(p, V, U, 1.0, emulate=True)
    np.testing.assert_allclose(L1, L2, rtol=2e-2)
    assert np.linalg.norm(g1 - g2) <= 0.1 * np.linalg.norm(g1)
