"""Asynchronous transfers (mass_lb_upload_async / mass_lb_download_async):
the same state, totals and results as the synchronous calls, ordered with
the steps on the handle's stream, and pinned host buffers required."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import LYO_C1, NEM_C2, bits_equal

pytestmark = pytest.mark.gpu

import torch  # noqa: E402

import mass_hd_b200 as M  # noqa: E402


def pinned(a):
    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
    out = t.numpy()
    out[:] = a.reshape(-1)
    return out, t


@pytest.mark.parametrize("model,params,LX,LY,prec", [
    (M.LYOTROPIC, LYO_C1, 64, 128, M.FP32),     # fused warp-strip kernel
    (M.LYOTROPIC, LYO_C1, 48, 40, M.FP64),      # sub-step kernels
    (M.NEMATIC, NEM_C2, 30, 66, M.FP32),        # unfused FP32
])
def test_async_transfers_equal_sync(model, params, LX, LY, prec):
    st = O.synthetic_state(model, LX, LY, seed=5, flow=0.01)
    names = ("ff", "QQxx", "QQyx", "phi") if model == M.LYOTROPIC else ("ff", "QQxx", "QQyx")
    keep = []
    host = {}
    for k in names:
        host[k], t = pinned(np.asarray(st[k], dtype=np.float64))
        keep.append(t)
    outs = {}
    for k in names:
        outs[k], t = pinned(np.zeros_like(host[k]))
        keep.append(t)
    a = M.Lattice(model, params, LX, LY, 0, prec)
    b = M.Lattice(model, params, LX, LY, 0, prec)
    a.upload(host["ff"], host["QQxx"], host["QQyx"], host.get("phi"))
    a.step(3)
    # two jobs back to back on b's stream, no wait in between
    for _ in range(2):
        b.upload_async(host["ff"], host["QQxx"], host["QQyx"], host.get("phi"))
        b.step(3)
        for k in names:
            b.get_into_async(k, outs[k])
    b.synchronize()
    for k in names:
        assert bits_equal(outs[k].reshape(a.get(k).shape), a.get(k)), k
    assert a.initial_totals() == b.initial_totals()
    # pageable buffers are refused
    with pytest.raises(M.MassLBError):
        b.get_into_async("QQxx", np.zeros(LX * LY))
    with pytest.raises(M.MassLBError):
        b.upload_async(np.asarray(st["ff"], dtype=np.float64).reshape(-1), host["QQxx"],
                       host["QQyx"], host.get("phi"))
    with pytest.raises(M.MassLBError):
        b.get_into_async("sigmaXX", outs["QQxx"])
    a.close()
    b.close()


@pytest.mark.parametrize("prec", [M.FP64, M.FP32])
def test_async_go_or_grow_with_relaxation(prec):
    """Go-or-grow: uploading phi through mass_lb_upload_async also refreshes
    chi on the device. An asynchronous upload followed by a step and a dry
    relaxation must leave the relaxed phi total as the reference total (the
    upload's own sums, still in flight when the relaxation starts, must not
    overwrite it later), and every field equal to the synchronous path."""
    from tests.test_gpu_go_or_grow import GOG

    LX, LY = 40, 36
    ref = O.RefOracle(O.GO_OR_GROW, GOG, LX, LY, 0)
    ref.configure(9)
    names = ("ff", "QQxx", "QQyx", "phi")
    keep, host = [], {}
    for k in names:
        host[k], t = pinned(np.asarray(ref.get(k), dtype=np.float64))
        keep.append(t)
    m = np.asarray(ref.get("m"), dtype=np.float64)
    a = M.Lattice(M.GO_OR_GROW, GOG, LX, LY, 0, prec)
    b = M.Lattice(M.GO_OR_GROW, GOG, LX, LY, 0, prec)
    a.upload(host["ff"], host["QQxx"], host["QQyx"], host["phi"])
    a.upload_field("m", m)
    a.step(2)
    ta = a.relax_free_energy(5, 0.8, True, True)
    b.upload_async(host["ff"], host["QQxx"], host["QQyx"], host["phi"])
    b.upload_field("m", m)
    b.step(2)
    tb = b.relax_free_energy(5, 0.8, True, True)
    b.synchronize()
    assert ta == tb
    assert a.initial_totals() == b.initial_totals()
    assert b.initial_totals()[1] == tb
    for k in names + ("m", "chi"):
        assert bits_equal(a.get(k), b.get(k)), k
    a.close()
    b.close()


@pytest.mark.parametrize("prec,LX,LY", [(M.FP32, 256, 192), (M.FP64, 40, 48)])
def test_pipeline_over_handles_equals_jobs_run_alone(prec, LX, LY):
    """Jobs with different inputs rotated over three handles, the runs of
    steps ordered with mass_lb_stream_wait and the transfers asynchronous
    (the bench's end-to-end pipeline): every job's result equals the job run
    alone with synchronous calls, bit for bit."""
    model, params, names = M.LYOTROPIC, LYO_C1, ("ff", "QQxx", "QQyx", "phi")
    njobs, nbuf, steps = 7, 3, 4
    keep, ins, outs = [], [], []
    for j in range(njobs):
        st = O.synthetic_state(model, LX, LY, seed=40 + j, flow=0.02)
        d, o = {}, {}
        for k in names:
            d[k], t = pinned(np.asarray(st[k], dtype=np.float64))
            keep.append(t)
            o[k], t = pinned(np.zeros_like(d[k]))
            keep.append(t)
        ins.append(d)
        outs.append(o)
    lats = [M.Lattice(model, params, LX, LY, 0, prec) for _ in range(nbuf)]
    for j in range(njobs):
        x = lats[j % nbuf]
        if j >= nbuf:
            x.synchronize()
        x.upload_async(*(ins[j][k] for k in names))
        if j > 0:
            x.wait_for(lats[(j - 1) % nbuf])
        x.step(steps)
        if j > 0:
            for k in names:
                lats[(j - 1) % nbuf].get_into_async(k, outs[j - 1][k])
    for k in names:
        lats[(njobs - 1) % nbuf].get_into_async(k, outs[njobs - 1][k])
    for x in lats:
        x.synchronize()
    ref = M.Lattice(model, params, LX, LY, 0, prec)
    for j in range(njobs):
        ref.upload(*(ins[j][k] for k in names))
        ref.step(steps)
        for k in names:
            want = ref.get(k)
            assert bits_equal(outs[j][k].reshape(want.shape), want), (j, k)
    # ordering calls: the same handle is a no-op, a null handle an error
    lats[0].wait_for(lats[0])
    from mass_hd_b200 import lb
    assert lb.load_library().mass_lb_stream_wait(lats[0].h, None) != 0
