"""Learned surrogate of the lyotropic step: training driver and hybrid loop.

A residual CNN maps the lattice fields (Qxx, Qyx, phi, ux, uy), normalised
per channel, forward by `jump` LB steps: a linear 3x3 convolution 5 -> 64,
6 residual blocks h <- h + conv(gelu(conv(h))) with 64 channels, and a 3x3
convolution 64 -> 5 added to the input (448,965 parameters). All
convolutions are circular (periodic lattice). Forward, backward, loss and
AdamW run in the library's own kernels (include/mass_surrogate.h): BF16
tensor-core convolutions with FP32 accumulation and fused bias / GELU /
residual epilogues, FP32 master weights and moments. torch only allocates
device buffers and provides the stream.

Training data come from the GPU simulator itself (`generate_dataset`): an
ensemble of 256^2 runs with zeta ~ U[0.005, 0.03], from each run (t, t+jump)
snapshot pairs at times spread evenly over the window the hybrid loop is
run in.

`hybrid()` advances lattices alternately with the plain method and the
surrogate: every M jumps the plain method runs one jump from the current
state and the surrogate predicts the same jump; if their difference is
below the threshold the surrogate takes the next M-1 jumps (the lattice is
re-initialised from the predicted fields with equilibrium populations),
otherwise - or if the surrogate's rollout left the finite range - the
plain method does.

Buffers passed to the kernels must stay referenced for the duration of
each call: a temporary tensor's memory goes back to torch's caching
allocator as soon as its pointer is taken, and the next allocation reuses it.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np
import torch

from . import lb

NBLOCKS = 6
CH = 64
NF = 5
FIELD_NAMES = ("Qxx", "Qyx", "phi", "ux", "uy")

FWD_BIAS, FWD_GELU, FWD_RESID, FWD_OUT, BWD_GELU, BWD_RESID, BWD_PLAIN = range(7)

_sg = None


def library():
    global _sg
    if _sg is not None:
        return _sg
    lib = lb.load_library()
    vp, i, f = C.c_void_p, C.c_int, C.c_float
    fl = C.POINTER(C.c_float)
    sig = {
        "mass_sg_conv3x3": [vp, vp, i, i, i, i, i, vp, vp, vp, vp, vp, vp, vp, vp, vp],
        "mass_sg_conv3x3_profile": [vp, vp, i, i, i, i, i, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                    vp],
        "mass_sg_conv3x3_wgrad": [vp, vp, vp, i, i, i, vp, vp],
        "mass_sg_bias_grad": [vp, vp, i, i, i, vp],
        "mass_sg_pack": [vp, vp, vp, i, i, i, vp, vp, vp, vp],
        "mass_sg_mse": [vp, vp, i, i, i, vp, vp, vp],
        "mass_sg_adamw": [vp] * 8 + [i, i, i, f, f, f, f, f, f, f, vp, vp, vp],
        "mass_sg_fields_from_state": [vp, C.c_longlong, i, i, C.c_double, fl, fl, vp, vp],
        "mass_sg_state_from_fields": [vp, i, i, C.c_double, fl, fl, vp, C.c_longlong, vp],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.restype = C.c_int
        fn.argtypes = args
    _sg = lib
    return lib


def _call(name, *args):
    code = getattr(library(), name)(*args)
    if code != 0:
        raise lb.MassLBError(code, library().mass_lb_last_error().decode())


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def padded(B, H, W, device="cuda"):
    return torch.zeros((B, H + 2, W + 2, CH), dtype=torch.bfloat16, device=device)


def layer_shapes():
    """[(name, cout, cin)] in network order."""
    out = [("in", CH, NF)]
    for i in range(NBLOCKS):
        out += [(f"b{i}c1", CH, CH), (f"b{i}c2", CH, CH)]
    out.append(("out", NF, CH))
    return out


class Layer:
    def __init__(self, name, cout, cin, device):
        self.name, self.cout, self.cin = name, cout, cin
        self.nout = 16 if cout <= 16 else 64
        z = lambda *s: torch.zeros(s, dtype=torch.float32, device=device)
        self.w, self.b = z(cout, 9, cin), z(self.nout)     # bias padded to the kernel's width
        self.mw, self.vw, self.mb, self.vb = z(cout, 9, cin), z(cout, 9, cin), z(cout), z(cout)
        self.wt = torch.zeros((9, self.nout, CH), dtype=torch.bfloat16, device=device)
        self.wd = torch.zeros((9, CH, CH), dtype=torch.bfloat16, device=device)
        self.dW, self.db = z(9, CH, CH), z(CH)

    def adamw(self, lr, beta1, beta2, eps, wd, step):
        bc1 = 1.0 - beta1 ** step if step > 0 else 1.0
        bc2 = 1.0 - beta2 ** step if step > 0 else 1.0
        _call("mass_sg_adamw", _p(self.w), _p(self.b), _p(self.mw), _p(self.vw), _p(self.mb),
              _p(self.vb), _p(self.dW), _p(self.db), self.cout, self.cin, self.nout, lr, beta1,
              beta2, eps, wd, bc1, bc2, _p(self.wt), _p(self.wd), _stream())

    def sync_bf16(self):
        """Write the bf16 forward / input-gradient weights from the master
        (an AdamW call with zero gradients and zero learning rate; the
        moments are restored afterwards)."""
        self.dW.zero_()
        self.db.zero_()
        saved = [x.clone() for x in (self.mw, self.vw, self.mb, self.vb)]
        self.adamw(0.0, 0.9, 0.999, 1e-8, 0.0, 0)
        for x, s in zip((self.mw, self.vw, self.mb, self.vb), saved):
            x.copy_(s)


class Params:
    """Master weights, AdamW moments and bf16 copies of every layer."""

    def __init__(self, seed=0, device="cuda", out_scale=0.1):
        self.layers = [Layer(n, co, ci, device) for n, co, ci in layer_shapes()]
        self.by_name = {L.name: L for L in self.layers}
        g = torch.Generator(device="cpu").manual_seed(seed)
        for L in self.layers:
            std = math.sqrt(2.0 / (9 * L.cin))
            if L.name == "out" or L.name.endswith("c2"):
                std *= out_scale
            L.w.copy_(torch.randn((L.cout, 9, L.cin), generator=g, dtype=torch.float64) * std)
            L.sync_bf16()
        self.step = 0
        self.mean = np.zeros(NF, dtype=np.float32)
        self.scale = np.ones(NF, dtype=np.float32)

    def count(self) -> int:
        return sum(L.w.numel() + L.cout for L in self.layers)

    def load(self, p: dict):
        """Set master weights from {name.w: [cout, 9, cin], name.b: [cout]}."""
        for L in self.layers:
            L.w.copy_(torch.as_tensor(np.asarray(p[L.name + ".w"]), dtype=torch.float32))
            L.b[:L.cout].copy_(torch.as_tensor(np.asarray(p[L.name + ".b"]), dtype=torch.float32))
            L.sync_bf16()

    def state_dict(self) -> dict:
        out = {}
        for L in self.layers:
            out[L.name + ".w"] = L.w.detach().cpu().numpy().astype(np.float64)
            out[L.name + ".b"] = L.b[:L.cout].detach().cpu().numpy().astype(np.float64)
        return out

    def grads(self) -> dict:
        """Last gradients as {name.w: [cout, 9, cin], name.b: [cout]}."""
        out = {}
        for L in self.layers:
            dW = L.dW.detach().cpu().numpy().astype(np.float64)      # [tap][ci][co]
            out[L.name + ".w"] = dW[:, :L.cin, :L.cout].transpose(2, 0, 1).copy()
            out[L.name + ".b"] = L.db.detach().cpu().numpy()[:L.cout].astype(np.float64)
        return out


class Net:
    """Activation buffers for batches of B images of H x W, and the
    forward / backward passes over a Params."""

    def __init__(self, params: Params, B: int, H: int, W: int, train: bool = True,
                 device="cuda"):
        if W % 128:
            raise ValueError("W must be a multiple of 128")
        self.P, self.B, self.H, self.W = params, B, H, W
        self.x_in = padded(B, H, W, device)
        self.h = [padded(B, H, W, device) for _ in range(NBLOCKS + 1)]
        self.t = [padded(B, H, W, device) for _ in range(NBLOCKS)]
        self.u = [padded(B, H, W, device) for _ in range(NBLOCKS)]
        f = lambda: torch.zeros((B, H, W, NF), dtype=torch.float32, device=device)
        self.xf, self.target, self.pred = f(), f(), f()
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        self.sse = torch.zeros(1, dtype=torch.float64, device=device)
        if train:
            self.dout = padded(B, H, W, device)
            self.dh = [padded(B, H, W, device), padded(B, H, W, device)]
            self.dt = padded(B, H, W, device)
        self.src = torch.zeros(B, dtype=torch.int32, device=device)
        self.dst = torch.zeros(B, dtype=torch.int32, device=device)

    # -- kernels ---------------------------------------------------------------
    def _conv(self, x, L, mode, out=None, out2=None, resid=None, aux=None, resid_f=None,
              out_f=None, weights=None):
        w = L.wt if weights is None else weights
        nout = L.nout if weights is None else CH
        _call("mass_sg_conv3x3", _p(x), _p(w), nout, mode, self.B, self.H, self.W,
              _p(L.b), _p(resid), _p(aux), _p(out), _p(out2), _p(resid_f), _p(out_f),
              _p(self.err), _stream())

    def pack(self, fields, src, dst=None):
        """Batch from stored fields [S, H, W, 5] (device fp32)."""
        self.src.copy_(torch.as_tensor(np.asarray(src), dtype=torch.int32))
        if dst is not None:
            self.dst.copy_(torch.as_tensor(np.asarray(dst), dtype=torch.int32))
        _call("mass_sg_pack", _p(fields), _p(self.src), _p(self.dst), self.B, self.H, self.W,
              _p(self.x_in), _p(self.xf), _p(self.target) if dst is not None else None, _stream())

    def forward(self):
        """x_in, xf -> pred."""
        Ls = self.P.by_name
        self._conv(self.x_in, Ls["in"], FWD_BIAS, out=self.h[0])
        for i in range(NBLOCKS):
            self._conv(self.h[i], Ls[f"b{i}c1"], FWD_GELU, out=self.u[i], out2=self.t[i])
            self._conv(self.u[i], Ls[f"b{i}c2"], FWD_RESID, out=self.h[i + 1], resid=self.h[i])
        self._conv(self.h[NBLOCKS], Ls["out"], FWD_OUT, resid_f=self.xf, out_f=self.pred)
        return self.pred

    def _wgrad(self, x, dy, L):
        _call("mass_sg_conv3x3_wgrad", _p(x), _p(dy), _p(L.dW), self.B, self.H, self.W,
              _p(self.err), _stream())
        _call("mass_sg_bias_grad", _p(dy), _p(L.db), self.B, self.H, self.W, _stream())

    def backward(self):
        """Gradients of the mean squared error of pred against target, into
        every layer's dW / db. Returns the sum of squared errors as a device
        tensor (divide by B*H*W*5 for the loss)."""
        Ls = self.P.by_name
        self.sse.zero_()
        _call("mass_sg_mse", _p(self.pred), _p(self.target), self.B, self.H, self.W,
              _p(self.sse), _p(self.dout), _stream())
        out = Ls["out"]
        self._wgrad(self.h[NBLOCKS], self.dout, out)
        dh, spare = self.dh
        self._conv(self.dout, out, BWD_PLAIN, out=dh, weights=out.wd)
        for i in reversed(range(NBLOCKS)):
            c1, c2 = Ls[f"b{i}c1"], Ls[f"b{i}c2"]
            self._wgrad(self.u[i], dh, c2)
            self._conv(dh, c2, BWD_GELU, out=self.dt, aux=self.t[i], weights=c2.wd)
            self._wgrad(self.h[i], self.dt, c1)
            self._conv(self.dt, c1, BWD_RESID, out=spare, resid=dh, weights=c1.wd)
            dh, spare = spare, dh
        self._wgrad(self.x_in, dh, Ls["in"])
        return self.sse

    def optimizer_step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, wd=0.01):
        self.P.step += 1
        for L in self.P.layers:
            L.adamw(lr, beta1, beta2, eps, wd, self.P.step)

    def check_error_flag(self):
        if int(self.err.item()) != 0:
            raise lb.MassLBError(-2, "surrogate kernel: a bounded wait timed out")


# -- data ---------------------------------------------------------------------

def _norm_args(mean, scale):
    m = (C.c_float * NF)(*[float(v) for v in mean])
    s = (C.c_float * NF)(*[float(v) for v in scale])
    return m, s


def fields_from_lattice(lat: lb.Lattice, out: torch.Tensor, mean, scale, rho=40.0):
    """Normalised fields of a fused FP32 lattice into out [LX, LY, 5]."""
    ptr, stride, _ = lat.device_state()
    m, s = _norm_args(mean, scale)
    _call("mass_sg_fields_from_state", C.c_void_p(ptr), stride, lat.LX, lat.LY, rho, m, s,
          _p(out), _stream())


def lattice_from_fields(lat: lb.Lattice, fields: torch.Tensor, mean, scale, rho=40.0):
    """Lattice state from normalised fields [LX, LY, 5] (equilibrium
    populations at density rho)."""
    ptr, stride, _ = lat.device_state()
    m, s = _norm_args(mean, scale)
    _call("mass_sg_state_from_fields", _p(fields), lat.LX, lat.LY, rho, m, s, C.c_void_p(ptr),
          stride, _stream())


def training_params(zeta: float) -> dict:
    from .run_case import PARAMS
    p = dict(PARAMS["lyotropic"])
    p["zeta"] = float(zeta)
    return p


def initial_state(L: int, rng: np.random.Generator, phi: str = "disk") -> dict:
    """Random director (S = 1) and either a tanh phi disk of radius L/4
    (phi="disk") or phi ~ N(0.5, 0.05) i.i.d. (phi="random")."""
    from .run_case import REST
    theta = rng.uniform(0.0, np.pi, L * L)
    st = {"QQxx": np.cos(2 * theta), "QQyx": np.sin(2 * theta),
          "ff": np.tile(REST * 40.0, (L * L, 1))}
    if phi == "random":
        st["phi"] = rng.normal(0.5, 0.05, L * L)
    else:
        x = np.arange(L)[:, None] - L / 2
        y = np.arange(L)[None, :] - L / 2
        r = np.sqrt(x * x + y * y).reshape(-1)
        st["phi"] = 0.5 * (1 - np.tanh((r - L / 4) / 2))
    return st


def generate_dataset(ntraj=40, L=256, pairs=50, jump=50, t_min=2000, t_max=22000, seed=0,
                     zeta_range=(0.005, 0.03), phi="disk"):
    """Simulate ntraj lattices together (one ensemble) and record the raw
    fields of `pairs` (t, t+jump) pairs per trajectory, t evenly spaced over
    [t_min, t_max). Returns (fields [ntraj*2*pairs, L, L, 5] device fp32,
    zetas); snapshots 2k and 2k+1 of a trajectory form pair k."""
    rng = np.random.default_rng(seed)
    zetas = rng.uniform(*zeta_range, ntraj)
    ens = lb.Ensemble(lb.LYOTROPIC, [training_params(z) for z in zetas], [(L, L)] * ntraj)
    for run in ens.runs:
        run.upload_state(initial_state(L, rng, phi))
    per = 2 * pairs
    fields = torch.empty((ntraj * per, L, L, NF), dtype=torch.float32, device="cuda")
    zero, one = np.zeros(NF), np.ones(NF)
    gap = (t_max - t_min) // pairs
    t = 0
    for k in range(pairs):
        t0 = t_min + k * gap
        ens.step(t0 - t)
        for half in (0, 1):
            if half:
                ens.step(jump)
            for r, run in enumerate(ens.runs):
                fields_from_lattice(run, fields[r * per + 2 * k + half], zero, one)
            torch.cuda.current_stream().synchronize()
        t = t0 + jump
    ens.close()
    return fields, zetas


def normalise(fields: torch.Tensor):
    """In place; returns (mean, scale) per channel."""
    mean = fields.double().mean(dim=(0, 1, 2))
    scale = fields.double().std(dim=(0, 1, 2)).clamp_min(1e-12)
    fields.sub_(mean.float()).div_(scale.float())
    return mean.cpu().numpy().astype(np.float32), scale.cpu().numpy().astype(np.float32)


def pair_indices(ntraj, pairs):
    """(input, target) snapshot indices of generate_dataset's layout."""
    return np.array([(t * 2 * pairs + 2 * k, t * 2 * pairs + 2 * k + 1)
                     for t in range(ntraj) for k in range(pairs)], dtype=np.int32)


def train(params: Params, fields: torch.Tensor, pairs: np.ndarray, epochs=20, batch=32,
          lr=1e-3, seed=0, log=None):
    """AdamW with a cosine learning rate. Returns the per-epoch mean loss."""
    _, H, W, _ = fields.shape
    net = Net(params, batch, H, W, train=True)
    rng = np.random.default_rng(seed)
    nb = len(pairs) // batch
    total = epochs * nb
    losses = []
    k = 0
    for ep in range(epochs):
        order = rng.permutation(len(pairs))
        acc = torch.zeros(1, dtype=torch.float64, device="cuda")
        for b in range(nb):
            idx = pairs[order[b * batch:(b + 1) * batch]]
            net.pack(fields, idx[:, 0], idx[:, 1])
            net.forward()
            acc += net.backward()
            lr_k = lr * 0.5 * (1 + math.cos(math.pi * k / total))
            net.optimizer_step(lr_k)
            k += 1
        loss = float(acc.item()) / (nb * batch * H * W * NF)
        losses.append(loss)
        net.check_error_flag()
        if log:
            log(f"epoch {ep}: loss {loss:.5g}")
    return losses


def evaluate(params: Params, fields: torch.Tensor, pairs: np.ndarray, batch=32) -> dict:
    """Mean squared error of the surrogate and of persistence (prediction =
    input) over the pairs, per channel, in normalised units."""
    _, H, W, _ = fields.shape
    batch = min(batch, len(pairs))
    net = Net(params, batch, H, W, train=False)
    se = torch.zeros(NF, dtype=torch.float64, device="cuda")
    sp = torch.zeros(NF, dtype=torch.float64, device="cuda")
    n = 0
    for b in range(0, len(pairs) - batch + 1, batch):
        idx = pairs[b:b + batch]
        net.pack(fields, idx[:, 0], idx[:, 1])
        pred = net.forward()
        se += ((pred - net.target).double() ** 2).sum(dim=(0, 1, 2))
        sp += ((net.xf - net.target).double() ** 2).sum(dim=(0, 1, 2))
        n += batch * H * W
    net.check_error_flag()
    return {"surrogate_mse": (se / n).cpu().numpy().tolist(),
            "persistence_mse": (sp / n).cpu().numpy().tolist()}


# -- hybrid loop --------------------------------------------------------------

def hybrid(params: Params, ens: lb.Ensemble, steps: int, jump=50, M=10, threshold=0.5,
           stats_every=None):
    """Advance every run of `ens` by `steps` LB steps (a multiple of jump*M)
    alternating plain and surrogate jumps (module docstring). threshold: the
    surrogate's error on the check jump, relative to the change the plain
    method made over that jump (L2 over all runs and channels, normalised
    units). Returns wall time, jumps taken by each method and statistics
    samples (every stats_every steps)."""
    runs = ens.runs
    B = len(runs)
    LX, LY = runs[0].LX, runs[0].LY
    net = Net(params, B, LX, LY, train=False)
    cur = torch.zeros((B, LX, LY, NF), dtype=torch.float32, device="cuda")
    after = torch.zeros_like(cur)
    x = torch.zeros_like(cur)
    idx = np.arange(B)
    t = 0
    taken = rejected = checks = nonfinite = 0
    errors = []
    samples = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    while t < steps:
        for r, run in enumerate(runs):
            fields_from_lattice(run, cur[r], params.mean, params.scale)
        net.pack(cur, idx)
        pred = net.forward()
        torch.cuda.current_stream().synchronize()
        ens.step(jump)
        for r, run in enumerate(runs):
            fields_from_lattice(run, after[r], params.mean, params.scale)
        err = float((torch.linalg.vector_norm(pred - after) /
                     torch.linalg.vector_norm(after - cur).clamp_min(1e-12)).item())
        errors.append(err)
        checks += 1
        accepted = False
        if err < threshold:
            x.copy_(after)
            for _ in range(M - 1):
                net.pack(x, idx)
                x.copy_(net.forward())
            # a rollout that left the finite range never reaches the lattice
            if bool(torch.isfinite(x).all().item()):
                for r, run in enumerate(runs):
                    lattice_from_fields(run, x[r], params.mean, params.scale)
                torch.cuda.current_stream().synchronize()
                taken += M - 1
                accepted = True
            else:
                nonfinite += 1
        if not accepted:
            ens.step(jump * (M - 1))
            rejected += M - 1
        t += jump * M
        if stats_every and t % stats_every == 0:
            samples.append([run.statistics() for run in runs])
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    net.check_error_flag()
    return {"steps": t, "wall_s": wall, "surrogate_jumps": taken, "plain_jumps_rejected": rejected,
            "checks": checks, "nonfinite_rollouts": nonfinite, "check_errors": errors,
            "samples": samples}


# -- one large lattice, tile by tile --------------------------------------------

RECEPTIVE = 2 * NBLOCKS + 2   # sites one forward pass reaches: 14 3x3 convolutions


class TiledSurrogate:
    """The surrogate applied to one large periodic lattice tile by tile.

    Each tile x tile interior is predicted from a (tile + 2 halo)^2 window
    cut from the lattice's fields with circular indices. The network pads
    every image circularly, so the window's own wrap reaches RECEPTIVE
    sites into it; with halo >= RECEPTIVE the interior sees only true
    neighbours, and the interiors together equal the network applied to the
    whole torus. `batch` windows go through the network at once."""

    def __init__(self, params: Params, LX: int, LY: int, tile: int = 1024, halo: int = 64,
                 batch: int = 8):
        if halo < RECEPTIVE:
            raise ValueError(f"halo must be at least {RECEPTIVE}")
        if LX % tile or LY % tile:
            raise ValueError("the lattice must be a whole number of tiles")
        self.P, self.LX, self.LY, self.T, self.h = params, LX, LY, tile, halo
        W = tile + 2 * halo
        self.W = W
        self.batch = batch
        self.net = Net(params, batch, W, W, train=False)
        self.cur = torch.empty((LX, LY, NF), dtype=torch.float32, device="cuda")
        self.pred = torch.empty_like(self.cur)
        self.win = torch.empty((batch, W, W, NF), dtype=torch.float32, device="cuda")
        self.tiles = [(tx, ty) for tx in range(LX // tile) for ty in range(LY // tile)]
        self.idx = np.arange(batch)

    def _rows(self, t0, n):
        return (torch.arange(-self.h, self.T + self.h, device="cuda") + t0) % n

    def predict(self, cur: torch.Tensor, out: torch.Tensor):
        """out <- the network's prediction for the normalised fields cur
        [LX, LY, 5], window by window."""
        T, h = self.T, self.h
        for b0 in range(0, len(self.tiles), self.batch):
            chunk = self.tiles[b0:b0 + self.batch]
            for k, (tx, ty) in enumerate(chunk):
                rows = self._rows(tx * T, self.LX)
                cols = self._rows(ty * T, self.LY)
                self.win[k].copy_(cur.index_select(0, rows).index_select(1, cols))
            self.net.pack(self.win, self.idx)
            p = self.net.forward()
            for k, (tx, ty) in enumerate(chunk):
                out[tx * T:(tx + 1) * T, ty * T:(ty + 1) * T].copy_(p[k, h:h + T, h:h + T])
        return out


def hybrid_tiled(params: Params, lat: lb.Lattice, steps: int, jump=50, M=10, threshold=0.5,
                 stats_every=None, tiler: TiledSurrogate = None):
    """hybrid() for one large lattice: every M jumps the plain method runs
    one jump while the tiled surrogate predicts it; if the surrogate's error
    relative to the plain change is below `threshold` it takes the next M-1
    jumps (the lattice rebuilt from its fields with equilibrium
    populations), else the plain method does. Returns wall time, jumps per
    method, the check errors and statistics samples every stats_every steps."""
    tiler = tiler or TiledSurrogate(params, lat.LX, lat.LY)
    cur, pred = tiler.cur, tiler.pred
    after = torch.empty_like(cur)
    t = 0
    taken = rejected = checks = nonfinite = 0
    errors, samples = [], []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    # The lattice steps on its own stream and the field conversions run on
    # torch's: each hand-over waits for the other side (a read of the state
    # before its steps have finished would see the old state).
    while t < steps:
        lat.synchronize()
        fields_from_lattice(lat, cur, params.mean, params.scale)
        tiler.predict(cur, pred)
        torch.cuda.current_stream().synchronize()
        lat.step(jump)
        lat.synchronize()
        fields_from_lattice(lat, after, params.mean, params.scale)
        err = float((torch.linalg.vector_norm(pred - after) /
                     torch.linalg.vector_norm(after - cur).clamp_min(1e-12)).item())
        errors.append(err)
        checks += 1
        accepted = False
        if err < threshold:
            # roll the surrogate M - 1 jumps on from the plain state,
            # ping-ponging two scratch buffers
            a, b = after, pred
            for _ in range(M - 1):
                tiler.predict(a, b)
                a, b = b, a
            if bool(torch.isfinite(a).all().item()):
                lattice_from_fields(lat, a, params.mean, params.scale)
                torch.cuda.current_stream().synchronize()
                taken += M - 1
                accepted = True
            else:
                nonfinite += 1
            after, pred = a, b
        if not accepted:
            torch.cuda.current_stream().synchronize()
            lat.step(jump * (M - 1))
            rejected += M - 1
        t += jump * M
        if stats_every and t % stats_every == 0:
            samples.append((t, lat.statistics()))
    lat.synchronize()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    tiler.net.check_error_flag()
    return {"steps": t, "wall_s": wall, "surrogate_jumps": taken, "plain_jumps_rejected": rejected,
            "checks": checks, "nonfinite_rollouts": nonfinite, "check_errors": errors,
            "samples": samples}
