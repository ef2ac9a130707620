"""The wall-band decomposition of a fused lattice with walls, pinned in FP64
on the CPU with the oracle (the C restatement of Step(), bit-identical to
the reference's build).

A walled lattice steps as (1) the periodic step of the whole lattice and
(2) a band lattice made of the 8 rows next to each wall of an axis, side by
side, stepped with the lattice's own walls; the band's outer 4 rows per side
replace the periodic result there (for boxes, a second band across x does
the same for the left and right walls). mass_hd_b200/csrc/api.cu
(k_band_gather, band_compute, band_emit) does this on the device around the fused
kernel. Here the same splice, restated with the oracle, must equal the
oracle's own walled step bit for bit, step after step, for every wall kind;
with 7-row halves it must not (one Step() reaches 4 sites, so the kept rows
need 4 more behind them). With npc correctors a step reaches 2 + 2*npc
sites; npc = 2 keeps 6 rows of 12-row halves.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import LYO_ALL, NEM_ALL


def _names(model):
    return ("ff", "QQxx", "QQyx") + (("phi",) if model == O.LYOTROPIC else ())


def _oracle(model, params, LX, LY, bc, fields):
    o = O.PortOracle(model, params, LX, LY, bc)
    for k, v in fields.items():
        o.set(k, v.reshape(-1, 9) if k == "ff" else v.reshape(-1))
    return o


def spliced_step(model, params, cur, LX, LY, bc, half, keep):
    """One walled step as the periodic step plus the wall bands."""
    names = _names(model)
    per = _oracle(model, params, LX, LY, 0, cur)
    per.step(1)
    nxt = {k: per.get(k).reshape(LX, LY, -1).copy() for k in names}
    ys = np.r_[0:half, LY - half:LY]
    yb = _oracle(model, params, LX, 2 * half, bc, {k: cur[k][:, ys] for k in names})
    yb.step(1)
    for k in names:
        r = yb.get(k).reshape(LX, 2 * half, -1)
        nxt[k][:, :keep] = r[:, :keep]
        nxt[k][:, LY - keep:] = r[:, 2 * half - keep:]
    if model == O.LYOTROPIC and bc in (3, 4):
        xs = np.r_[0:half, LX - half:LX]
        xb = _oracle(model, params, 2 * half, LY, bc, {k: cur[k][xs] for k in names})
        xb.step(1)
        for k in names:
            r = xb.get(k).reshape(2 * half, LY, -1)
            nxt[k][:keep] = r[:keep]
            nxt[k][LX - keep:] = r[2 * half - keep:]
    return nxt


def _run(model, params, LX, LY, bc, steps, half, keep=4):
    names = _names(model)
    st = O.synthetic_state(model, LX, LY, seed=31, flow=0.03)
    full = O.PortOracle(model, params, LX, LY, bc)
    for k, v in st.items():
        full.set(k, v)
    full.step(steps)
    cur = {k: np.asarray(st[k], dtype=np.float64).reshape(LX, LY, -1).copy() for k in names}
    for _ in range(steps):
        cur = spliced_step(model, params, cur, LX, LY, bc, half, keep)
    return {k: (full.get(k).reshape(LX, LY, -1), cur[k]) for k in names}


@pytest.mark.parametrize("model,params,bc", [(O.LYOTROPIC, LYO_ALL, 1), (O.LYOTROPIC, LYO_ALL, 2),
                                             (O.LYOTROPIC, LYO_ALL, 3), (O.LYOTROPIC, LYO_ALL, 4),
                                             (O.NEMATIC, NEM_ALL, 1)])
def test_bands_splice_into_the_walled_step(model, params, bc):
    for k, (want, got) in _run(model, params, 22, 26, bc, 3, 8).items():
        assert np.array_equal(want.view(np.uint64), got.view(np.uint64)), (bc, k)


def test_narrower_bands_do_not():
    out = _run(O.LYOTROPIC, LYO_ALL, 22, 26, 4, 1, 7)
    assert any(not np.array_equal(w, g) for w, g in out.values())


@pytest.mark.parametrize("bc", [1, 4])
def test_bands_with_two_correctors(bc):
    p = dict(LYO_ALL, npc=2)
    for k, (want, got) in _run(O.LYOTROPIC, p, 30, 32, bc, 2, 12, 6).items():
        assert np.array_equal(want.view(np.uint64), got.view(np.uint64)), (bc, k)
    out = _run(O.LYOTROPIC, p, 30, 32, bc, 1, 11, 6)
    assert any(not np.array_equal(w, g) for w, g in out.values())
