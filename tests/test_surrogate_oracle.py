"""The surrogate's CPU oracle (oracle/surrogate.py), pinned on the CPU:
its backward pass against central finite differences of its own forward
pass (float64), its bfloat16 rounding against known values, and its
convolution against a direct loop."""
import numpy as np

from oracle import surrogate as S


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-8, 65504.0])
    r = S.bf16(x)
    # 1 + 2^-8 is a tie -> even (1.0); 1 + 3*2^-8 is a tie -> even (1 + 2^-6)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -7
    assert r[3] == 1.0 + 2 ** -6 and r[4] == -2.5
    assert abs(r[5] - 3.0e-8) / 3.0e-8 < 2 ** -8 and r[6] == 65536.0


def test_conv_matches_direct_loop():
    rng = np.random.default_rng(0)
    x = rng.normal(size=(2, 4, 5, 3))
    w = rng.normal(size=(2, 9, 3))
    out = S.conv(x, w)
    B, H, W, _ = x.shape
    ref = np.zeros((B, H, W, 2))
    for b in range(B):
        for y in range(H):
            for xx in range(W):
                for ky in range(3):
                    for kx in range(3):
                        ref[b, y, xx] += w[:, 3 * ky + kx, :] @ x[b, (y + ky - 1) % H, (xx + kx - 1) % W]
    assert np.allclose(out, ref, atol=1e-12)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = S.init_params(seed=2, out_scale=1.0)
    for k in p:
        if k.endswith(".b"):
            p[k] = rng.normal(0, 0.1, p[k].shape)
    x = rng.normal(size=(1, 3, 4, S.NF))
    target = x + rng.normal(0, 0.5, x.shape)
    loss, _, g = S.loss_and_grads(p, x, target)
    assert np.isfinite(loss)
    eps = 1e-6
    for name in ("in.w", "in.b", "b0c1.w", "b2c2.w", "b5c1.b", "b5c2.w", "out.w", "out.b"):
        flat = p[name].reshape(-1)
        for j in rng.choice(flat.size, 3, replace=False):
            old = flat[j]
            flat[j] = old + eps
            lp = S.loss_and_grads(p, x, target)[0]
            flat[j] = old - eps
            lm = S.loss_and_grads(p, x, target)[0]
            flat[j] = old
            fd = (lp - lm) / (2 * eps)
            an = g[name].reshape(-1)[j]
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (name, j, fd, an)


def test_parameter_count():
    p = S.init_params()
    assert sum(v.size for v in p.values()) == 448965


def test_adamw_first_step_is_sign_step():
    p = {"a.w": np.ones((1, 9, 1)), "a.b": np.zeros(1)}
    g = {"a.w": np.full((1, 9, 1), 3.0), "a.b": np.array([-2.0])}
    m = {k: np.zeros_like(v) for k, v in p.items()}
    v = {k: np.zeros_like(vv) for k, vv in p.items()}
    S.adamw(p, m, v, g, step=1, lr=0.1, wd=0.0)
    assert np.allclose(p["a.w"], 0.9, atol=1e-7) and np.allclose(p["a.b"], 0.1, atol=1e-7)
