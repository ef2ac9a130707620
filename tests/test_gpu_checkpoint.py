"""Binary checkpoints (mass_lb_save / mass_lb_load).

A run that is saved, continued, and compared with a second lattice that
loads the checkpoint and takes the same steps must match bit for bit (FP64,
FP32 fused, walls, nematic), carry the step count and conservation totals
over, and reject files of another model, size, or with a damaged payload.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import LYO_ALL, NEM_C2

pytestmark = pytest.mark.gpu

import mass_hd_b200 as M  # noqa: E402


def fields(model):
    return ("ff", "QQxx", "QQyx", "phi") if model == M.LYOTROPIC else ("ff", "QQxx", "QQyx")


CASES = [(M.LYOTROPIC, LYO_ALL, 40, 36, 0, M.FP64), (M.LYOTROPIC, LYO_ALL, 64, 64, 0, M.FP32),
         (M.LYOTROPIC, LYO_ALL, 36, 40, 3, M.FP64), (M.NEMATIC, NEM_C2, 64, 64, 0, M.FP32),
         (M.NEMATIC, NEM_C2, 40, 36, 1, M.FP64)]


@pytest.mark.parametrize("model,params,LX,LY,bc,prec", CASES)
def test_resume_is_bit_identical(tmp_path, model, params, LX, LY, bc, prec):
    st = O.synthetic_state(model, LX, LY, seed=3)
    a = M.Lattice(model, params, LX, LY, bc, prec)
    a.upload_state(st)
    a.step(5)
    path = str(tmp_path / "run.ckpt")
    a.save(path)
    totals = a.initial_totals()
    a.step(7)
    b = M.Lattice(model, params, LX, LY, bc, prec)
    b.load(path)
    assert b.initial_totals() == totals
    b.step(7)
    for n in fields(model):
        assert np.array_equal(a.get(n), b.get(n)), n
    assert os.path.getsize(path) > 9 * 8 * LX * LY
    a.close()
    b.close()


def test_checkpoint_moves_between_precisions(tmp_path):
    st = O.synthetic_state(M.LYOTROPIC, 64, 64, seed=4)
    a = M.Lattice(M.LYOTROPIC, LYO_ALL, 64, 64, 0, M.FP64)
    a.upload_state(st)
    a.step(3)
    path = str(tmp_path / "f64.ckpt")
    a.save(path)
    b = M.Lattice(M.LYOTROPIC, LYO_ALL, 64, 64, 0, M.FP32)
    b.load(path)
    c = M.Lattice(M.LYOTROPIC, LYO_ALL, 64, 64, 0, M.FP32)
    c.upload_state({n: a.get(n) for n in fields(M.LYOTROPIC)})
    b.step(4)
    c.step(4)
    for n in fields(M.LYOTROPIC):
        assert np.array_equal(b.get(n), c.get(n)), n
    for x in (a, b, c):
        x.close()


def test_bad_checkpoints_are_rejected(tmp_path):
    st = O.synthetic_state(M.LYOTROPIC, 40, 36, seed=5)
    a = M.Lattice(M.LYOTROPIC, LYO_ALL, 40, 36, 0, M.FP64)
    a.upload_state(st)
    path = str(tmp_path / "ok.ckpt")
    a.save(path)
    raw = open(path, "rb").read()
    # damaged payload
    bad = bytearray(raw)
    bad[-100] ^= 0x40
    open(tmp_path / "bad.ckpt", "wb").write(bytes(bad))
    # truncated file, wrong magic
    open(tmp_path / "short.ckpt", "wb").write(raw[:len(raw) // 2])
    open(tmp_path / "magic.ckpt", "wb").write(b"NOTACKPT" + raw[8:])
    for name in ("bad.ckpt", "short.ckpt", "magic.ckpt", "missing.ckpt"):
        with pytest.raises(M.MassLBError):
            a.load(str(tmp_path / name))
    other_size = M.Lattice(M.LYOTROPIC, LYO_ALL, 36, 40, 0, M.FP64)
    with pytest.raises(M.MassLBError):
        other_size.load(path)
    nem = M.Lattice(M.NEMATIC, NEM_C2, 40, 36, 0, M.FP64)
    with pytest.raises(M.MassLBError):
        nem.load(path)
    # the lattice is untouched by a failed load
    a.load(path)
    for n in fields(M.LYOTROPIC):
        assert np.array_equal(a.get(n), np.asarray(st[n]).reshape(a.get(n).shape)), n
    for x in (a, other_size, nem):
        x.close()
