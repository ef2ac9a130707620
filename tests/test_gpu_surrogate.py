"""Surrogate kernels on the GPU against the CPU oracle (oracle/surrogate.py).

Tolerances (relative L2): bf16-stored outputs of one convolution <= 3e-3
(half a bf16 ulp is 2^-9 relative); fp32 outputs <= 1e-5; the weight
gradient (fp32 sum of bf16 products) <= 1e-5; whole-network prediction
<= 1e-2 and gradients <= 3e-2 per tensor against the bf16-emulating oracle
(a bf16 rounding that lands differently in one layer propagates through
the 13 layers after it).

Buffers passed to the kernels are held in variables for the duration of
each call: a temporary tensor's memory returns to torch's caching allocator
as soon as its pointer is taken and the next allocation reuses it.
"""
import numpy as np
import pytest
import torch

from oracle import surrogate as S

pytestmark = pytest.mark.gpu

import mass_hd_b200.surrogate as G  # noqa: E402
from tests.helpers import rel_l2  # noqa: E402


def to_padded(x):
    """[B, H, W, C] -> padded NHWC64 numpy with the periodic ring."""
    B, H, W, C = x.shape
    out = np.zeros((B, H + 2, W + 2, 64))
    core = np.zeros((B, H, W, 64))
    core[..., :C] = x
    out[:, 1:-1, 1:-1] = core
    out[:, 0, 1:-1] = core[:, -1]
    out[:, -1, 1:-1] = core[:, 0]
    out[:, :, 0] = out[:, :, -2]
    out[:, :, -1] = out[:, :, 1]
    return out


def dev_bf16(a):
    return torch.tensor(np.asarray(a, dtype=np.float32)).to(torch.bfloat16).cuda().contiguous()


def host(t):
    return t.float().cpu().numpy().astype(np.float64)


def core(p):
    return p[:, 1:-1, 1:-1]


def check_ring(p):
    c = core(p)
    assert np.array_equal(p[:, 0, 1:-1], c[:, -1]) and np.array_equal(p[:, -1, 1:-1], c[:, 0])
    assert np.array_equal(p[:, :, 0], p[:, :, -2]) and np.array_equal(p[:, :, -1], p[:, :, 1])


def fwd_weights(w, nout):
    """[cout, 9, cin] -> bf16 [9][nout][64]"""
    cout, _, cin = w.shape
    out = np.zeros((9, nout, 64))
    out[:, :cout, :cin] = w.transpose(1, 0, 2)
    return out


def dgrad_weights(w):
    cout, _, cin = w.shape
    out = np.zeros((9, 64, 64))
    for t in range(9):
        out[8 - t, :cin, :cout] = w[:, t, :].T
    return out


SIZES = [(2, 3, 128), (1, 1, 256), (1, 5, 384)]


def run_conv(x, wt, nout, mode, bias=None, resid=None, aux=None, resid_f=None):
    B, Hp, Wp, _ = x.shape
    H, W = Hp - 2, Wp - 2
    out = torch.zeros_like(x)
    out2 = torch.zeros_like(x)
    out_f = torch.zeros((B, H, W, 5), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    b = torch.tensor(np.zeros(nout) if bias is None else bias, dtype=torch.float32).cuda()
    G._call("mass_sg_conv3x3", G._p(x), G._p(wt), nout, mode, B, H, W, G._p(b), G._p(resid),
            G._p(aux), G._p(out), G._p(out2), G._p(resid_f), G._p(out_f), G._p(err), G._stream())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return out, out2, out_f


@pytest.mark.parametrize("B,H,W", SIZES)
def test_forward_modes(B, H, W):
    rng = np.random.default_rng(B * 100 + H)
    x = S.bf16(rng.normal(size=(B, H, W, 64)))
    w = S.bf16(rng.normal(0, 0.05, (64, 9, 64)))
    bias = rng.normal(0, 0.1, 64)
    r = S.bf16(rng.normal(size=(B, H, W, 64)))
    X, Wt, R = dev_bf16(to_padded(x)), dev_bf16(fwd_weights(w, 64)), dev_bf16(to_padded(r))
    ref = S.conv(x, w) + bias
    out, _, _ = run_conv(X, Wt, 64, G.FWD_BIAS, bias)
    o = host(out)
    check_ring(o)
    assert rel_l2(core(o), ref) < 3e-3
    out, out2, _ = run_conv(X, Wt, 64, G.FWD_GELU, bias)
    o, t = host(out), host(out2)
    check_ring(o)
    assert rel_l2(core(t), ref) < 3e-3
    assert rel_l2(core(o), S.gelu(ref)) < 3e-3
    out, _, _ = run_conv(X, Wt, 64, G.FWD_RESID, bias, resid=R)
    o = host(out)
    check_ring(o)
    assert rel_l2(core(o), ref + r) < 3e-3


@pytest.mark.parametrize("B,H,W", SIZES[:2])
def test_output_layer(B, H, W):
    rng = np.random.default_rng(7)
    x = S.bf16(rng.normal(size=(B, H, W, 64)))
    w = S.bf16(rng.normal(0, 0.05, (5, 9, 64)))
    bias = np.zeros(16)
    bias[:5] = rng.normal(0, 0.1, 5)
    xf = rng.normal(size=(B, H, W, 5)).astype(np.float32)
    X, Wt, XF = dev_bf16(to_padded(x)), dev_bf16(fwd_weights(w, 16)), torch.tensor(xf).cuda()
    _, _, of = run_conv(X, Wt, 16, G.FWD_OUT, bias, resid_f=XF)
    ref = S.conv(x, w) + bias[:5] + xf
    assert rel_l2(of.cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("B,H,W", SIZES[:2])
def test_backward_modes(B, H, W):
    rng = np.random.default_rng(11)
    dy = S.bf16(rng.normal(size=(B, H, W, 64)))
    w = S.bf16(rng.normal(0, 0.05, (64, 9, 64)))
    t = S.bf16(rng.normal(size=(B, H, W, 64)))
    r = S.bf16(rng.normal(size=(B, H, W, 64)))
    D, Wd = dev_bf16(to_padded(dy)), dev_bf16(dgrad_weights(w))
    T, R = dev_bf16(to_padded(t)), dev_bf16(to_padded(r))
    ref = S.conv_input_grad(dy, w)
    out, _, _ = run_conv(D, Wd, 64, G.BWD_PLAIN)
    o = host(out)
    check_ring(o)
    assert rel_l2(core(o), ref) < 3e-3
    out, _, _ = run_conv(D, Wd, 64, G.BWD_GELU, aux=T)
    assert rel_l2(core(host(out)), ref * S.gelu_grad(t)) < 3e-3
    out, _, _ = run_conv(D, Wd, 64, G.BWD_RESID, resid=R)
    assert rel_l2(core(host(out)), ref + r) < 3e-3


@pytest.mark.parametrize("rows", [1, 2, 3, 8, 24])
def test_strip_heights(rows, monkeypatch):
    """Each CTA marches down strips of `rows` output rows and reuses every
    input slab's A operand for the up to three output rows it feeds. Every
    strip height gives the same convolution: 8 x 24 x 256 has 384 half-row
    tiles, so strips of 1 or 2 rows put several strips on one CTA (the four
    accumulators wrap) and 3, 8 and 24 rows cover the strip edges."""
    monkeypatch.setenv("MASS_SG_CONV_ROWS", str(rows))
    B, H, W = 8, 24, 256
    rng = np.random.default_rng(rows)
    x = S.bf16(rng.normal(size=(B, H, W, 64)))
    w = S.bf16(rng.normal(0, 0.05, (64, 9, 64)))
    bias = rng.normal(0, 0.1, 64)
    r = S.bf16(rng.normal(size=(B, H, W, 64)))
    X, Wt, R = dev_bf16(to_padded(x)), dev_bf16(fwd_weights(w, 64)), dev_bf16(to_padded(r))
    out, _, _ = run_conv(X, Wt, 64, G.FWD_RESID, bias, resid=R)
    o = host(out)
    check_ring(o)
    assert rel_l2(core(o), S.conv(x, w) + bias + r) < 3e-3
    Wd = dev_bf16(dgrad_weights(w))
    out, _, _ = run_conv(X, Wd, 64, G.BWD_GELU, aux=R)
    assert rel_l2(core(host(out)), S.conv_input_grad(x, w) * S.gelu_grad(r)) < 3e-3
    w5 = S.bf16(rng.normal(0, 0.05, (5, 9, 64)))
    b16 = np.zeros(16)
    b16[:5] = bias[:5]
    _, _, of = run_conv(X, dev_bf16(fwd_weights(w5, 16)), 16, G.FWD_OUT, b16)
    assert rel_l2(of.cpu().numpy(), S.conv(x, w5) + bias[:5]) < 1e-5


def test_profile_entry_point_matches_and_counts():
    """mass_sg_conv3x3_profile gives mass_sg_conv3x3's output bit for bit and
    fills 4 cycle counters per CTA (total >= span to the last issue >= each
    wait)."""
    import ctypes
    B, H, W = 4, 32, 256
    rng = np.random.default_rng(5)
    x = S.bf16(rng.normal(size=(B, H, W, 64)))
    w = S.bf16(rng.normal(0, 0.05, (64, 9, 64)))
    bias = rng.normal(0, 0.1, 64)
    X, Wt = dev_bf16(to_padded(x)), dev_bf16(fwd_weights(w, 64))
    ref, ref2, _ = run_conv(X, Wt, 64, G.FWD_GELU, bias)
    out, out2 = torch.zeros_like(X), torch.zeros_like(X)
    b = torch.tensor(bias, dtype=torch.float32).cuda()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    cyc = torch.zeros(4 * 1024, dtype=torch.int64, device="cuda")
    ncta = ctypes.c_int(0)
    G._call("mass_sg_conv3x3_profile", G._p(X), G._p(Wt), 64, G.FWD_GELU, B, H, W, G._p(b), None,
            None, G._p(out), G._p(out2), None, None, G._p(err), G._p(cyc), ctypes.addressof(ncta),
            G._stream())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(out, ref) and torch.equal(out2, ref2)
    c = cyc[:4 * ncta.value].view(-1, 4).cpu().numpy()
    assert ncta.value >= 1
    assert (c[:, 0] >= c[:, 1]).all() and (c[:, 1] > 0).all()
    assert (c[:, 1] >= c[:, 2]).all() and (c[:, 1] >= c[:, 3]).all()


@pytest.mark.parametrize("B,H,W", SIZES)
def test_weight_gradient(B, H, W):
    rng = np.random.default_rng(13)
    x = S.bf16(rng.normal(size=(B, H, W, 64)))
    dy = S.bf16(rng.normal(size=(B, H, W, 64)))
    dW = torch.zeros((9, 64, 64), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    X, D = dev_bf16(to_padded(x)), dev_bf16(to_padded(dy))
    G._call("mass_sg_conv3x3_wgrad", G._p(X), G._p(D), G._p(dW), B, H, W, G._p(err), G._stream())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = S.conv_weight_grad(x, dy)                     # [co, tap, ci]
    got = dW.cpu().numpy().astype(np.float64).transpose(2, 0, 1)
    assert rel_l2(got, ref) < 1e-5


def test_bias_grad_pack_mse():
    rng = np.random.default_rng(17)
    B, H, W = 2, 3, 128
    dy = S.bf16(rng.normal(size=(B, H, W, 64)))
    db = torch.zeros(64, dtype=torch.float32, device="cuda")
    D = dev_bf16(to_padded(dy))
    G._call("mass_sg_bias_grad", G._p(D), G._p(db), B, H, W, G._stream())
    assert rel_l2(db.cpu().numpy(), dy.sum(axis=(0, 1, 2))) < 1e-6

    fields = rng.normal(size=(4, H, W, 5)).astype(np.float32)
    F = torch.tensor(fields).cuda()
    P = G.Params(seed=0)
    net = G.Net(P, B, H, W, train=True)
    net.pack(F, [2, 0], [3, 1])
    torch.cuda.synchronize()
    xin = host(net.x_in)
    check_ring(xin)
    assert np.array_equal(core(xin)[..., :5], S.bf16(fields[[2, 0]]))
    assert not core(xin)[..., 5:].any()
    assert np.array_equal(net.xf.cpu().numpy(), fields[[2, 0]])
    assert np.array_equal(net.target.cpu().numpy(), fields[[3, 1]])

    net.pred.copy_(torch.tensor(fields[[1, 3]]).cuda())
    net.sse.zero_()
    G._call("mass_sg_mse", G._p(net.pred), G._p(net.target), B, H, W, G._p(net.sse),
            G._p(net.dout), G._stream())
    e = fields[[1, 3]].astype(np.float64) - fields[[3, 1]]
    assert abs(net.sse.item() - (e * e).sum()) < 1e-6 * (e * e).sum()
    d = host(net.dout)
    check_ring(d)
    assert rel_l2(core(d)[..., :5], 2 * e / e.size) < 3e-3
    assert not core(d)[..., 5:].any()


def test_adamw_matches_oracle():
    rng = np.random.default_rng(19)
    P = G.Params(seed=3)
    p0 = P.state_dict()
    g = {k: rng.normal(size=v.shape) for k, v in p0.items()}
    for L in P.layers:
        dW = np.zeros((9, 64, 64))
        dW[:, :L.cin, :L.cout] = g[L.name + ".w"].transpose(1, 2, 0)
        L.dW.copy_(torch.tensor(dW, dtype=torch.float32))
        db = np.zeros(64)
        db[:L.cout] = g[L.name + ".b"]
        L.db.copy_(torch.tensor(db, dtype=torch.float32))
    ref = {k: v.copy() for k, v in p0.items()}
    m = {k: np.zeros_like(v) for k, v in ref.items()}
    v = {k: np.zeros_like(vv) for k, vv in ref.items()}
    for step in (1, 2):
        for L in P.layers:
            L.adamw(1e-3, 0.9, 0.999, 1e-8, 0.01, step)
        S.adamw(ref, m, v, g, step, 1e-3)
    got = P.state_dict()
    for k in ref:
        assert rel_l2(got[k] - p0[k], ref[k] - p0[k]) < 1e-4, k
    L = P.by_name["b3c1"]
    wt = L.wt.float().cpu().numpy()
    assert np.array_equal(wt, fwd_weights(S.bf16(got["b3c1.w"]), 64))
    assert np.array_equal(L.wd.float().cpu().numpy(), dgrad_weights(S.bf16(got["b3c1.w"])))


@pytest.mark.parametrize("B,H,W", [(2, 4, 128), (1, 3, 256)])
def test_network_gradients_match_oracle(B, H, W):
    rng = np.random.default_rng(23)
    p = S.init_params(seed=5, out_scale=0.3)
    for k in p:
        if k.endswith(".b"):
            p[k] = rng.normal(0, 0.05, p[k].shape)
    P = G.Params(seed=0)
    P.load(p)
    fields = rng.normal(size=(2 * B, H, W, 5)).astype(np.float32)
    F = torch.tensor(fields).cuda()
    net = G.Net(P, B, H, W, train=True)
    src, dst = np.arange(B), np.arange(B, 2 * B)
    net.pack(F, src, dst)
    pred = net.forward().cpu().numpy().astype(np.float64)
    sse = net.backward().item()
    torch.cuda.synchronize()
    net.check_error_flag()
    x, target = fields[src].astype(np.float64), fields[dst].astype(np.float64)
    loss, pred_ref, g_ref = S.loss_and_grads(p, x, target, bf=True)
    assert rel_l2(pred, pred_ref) < 1e-2
    assert abs(sse / target.size - loss) < 2e-3 * loss
    g = P.grads()
    for k in g_ref:
        assert rel_l2(g[k], g_ref[k]) < 3e-2, (k, rel_l2(g[k], g_ref[k]))


def test_state_field_round_trip():
    from mass_hd_b200 import lb
    from mass_hd_b200.run_case import PARAMS
    rng = np.random.default_rng(29)
    L = 128
    lat = lb.Lattice(lb.LYOTROPIC, PARAMS["lyotropic"], L, L, 0, lb.FP32)
    lat.upload_state(G.initial_state(L, rng))
    lat.step(20)
    lat.synchronize()
    mean = np.array([0.1, -0.2, 0.5, 0.0, 0.0], np.float32)
    scale = np.array([0.5, 0.5, 0.4, 1e-3, 1e-3], np.float32)
    f = torch.zeros((L, L, 5), dtype=torch.float32, device="cuda")
    G.fields_from_lattice(lat, f, mean, scale)
    torch.cuda.synchronize()
    st = {n: lat.get(n) for n in ("ff", "QQxx", "QQyx", "phi")}
    ff = st["ff"]
    rho = ff.sum(axis=1)
    ux = (ff[:, 1] - ff[:, 2] + ff[:, 5] - ff[:, 6] - ff[:, 7] + ff[:, 8]) / rho
    uy = (ff[:, 3] - ff[:, 4] + ff[:, 5] - ff[:, 6] + ff[:, 7] - ff[:, 8]) / rho
    ref = (np.stack([st["QQxx"], st["QQyx"], st["phi"], ux, uy], axis=1) - mean) / scale
    assert rel_l2(f.cpu().numpy().reshape(-1, 5), ref) < 1e-4
    # fields -> equilibrium state -> fields keeps Q, phi, u
    G.lattice_from_fields(lat, f, mean, scale)
    g2 = torch.zeros_like(f)
    G.fields_from_lattice(lat, g2, mean, scale)
    torch.cuda.synchronize()
    assert rel_l2(g2.cpu().numpy(), f.cpu().numpy()) < 1e-4
    ff2 = lat.get("ff")
    assert abs(ff2.sum(axis=1).mean() - 40.0) < 1e-4
    lat.close()


def test_short_training_lowers_the_loss():
    rng = np.random.default_rng(31)
    B, H, W = 4, 16, 128
    # a learnable map: target = input shifted by one pixel and scaled
    base = rng.normal(size=(8, H, W, 5)).astype(np.float32)
    fields = np.concatenate([base, 0.8 * np.roll(base, 1, axis=2)], axis=0)
    F = torch.tensor(fields).cuda()
    pairs = np.array([(i, 8 + i) for i in range(8)], dtype=np.int32)
    P = G.Params(seed=1)
    losses = G.train(P, F, pairs, epochs=30, batch=B, lr=2e-3)
    assert losses[-1] < 0.3 * losses[0], losses


def test_tiled_prediction_equals_the_whole_torus():
    """TiledSurrogate: windows of tile + 2*halo with circular halos give,
    on their interiors, what the network gives applied to the whole
    periodic lattice at once (the halo covers the 14-site receptive
    field)."""
    torch.manual_seed(3)
    P = G.Params(seed=4)
    P.mean = np.zeros(G.NF, dtype=np.float32)
    P.scale = np.ones(G.NF, dtype=np.float32)
    L = 512
    cur = torch.randn((L, L, G.NF), device="cuda") * 0.5
    whole = G.Net(P, 1, L, L, train=False)
    whole.pack(cur[None].contiguous(), np.array([0]))
    want = whole.forward()[0].clone()
    tiler = G.TiledSurrogate(P, L, L, tile=256, halo=64, batch=2)
    got = tiler.predict(cur, torch.empty_like(cur))
    err = (got - want).abs().max().item()
    assert err <= 1e-6 * want.abs().max().item(), err
    with pytest.raises(ValueError):
        G.TiledSurrogate(P, L, L, tile=256, halo=8)


def test_tiled_hybrid_at_threshold_zero_is_plain_lb():
    """hybrid_tiled with threshold 0 never accepts a surrogate jump: the
    lattice ends bit-identical to the plain method stepped as long, and
    every check error is an honest ratio (a read of the state before its
    steps had finished would give ratios near 1e12)."""
    from oracle import oracle as O
    from mass_hd_b200 import lb
    from mass_hd_b200.run_case import PARAMS
    L = 512
    P = G.Params(seed=2)
    st = O.synthetic_state(O.LYOTROPIC, L, L, seed=5, flow=0.02)
    a = lb.Lattice(lb.LYOTROPIC, PARAMS["lyotropic"], L, L, 0, lb.FP32)
    b = lb.Lattice(lb.LYOTROPIC, PARAMS["lyotropic"], L, L, 0, lb.FP32)
    for x in (a, b):
        x.set_tile(32, 64)
        x.upload_state(st)
        x.step(20)
    P.mean = np.zeros(G.NF, dtype=np.float32)
    P.scale = np.ones(G.NF, dtype=np.float32)
    tiler = G.TiledSurrogate(P, L, L, tile=256, halo=64, batch=4)
    res = G.hybrid_tiled(P, a, 200, jump=20, M=5, threshold=0.0, tiler=tiler)
    b.step(200)
    assert res["surrogate_jumps"] == 0 and res["checks"] == 2
    assert all(0 < e < 1e6 for e in res["check_errors"]), res["check_errors"]
    for n in ("ff", "QQxx", "QQyx", "phi"):
        assert np.array_equal(a.get(n), b.get(n)), n
    a.close()
    b.close()
