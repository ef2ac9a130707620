"""The FP32 fused kernel's restated arithmetic, checked on the CPU.

The warp-strip kernel (mass_hd_b200/csrc/fused_warp.cu) does not follow the
reference's expression order: it keeps central differences as raw
differences with their factors folded into constants, forms the molecular
field as (CC*term - 4 LL)*Q + LL*(neighbour sum), moves Gamma*H - u.grad(Q)
into UpdateQuantities, folds the forcing term into the equilibrium through
j' = j + tau*F and uses the closed form of the rest population. Those are
identities of real arithmetic. This test restates the kernel's formulas in
numpy FP64, steps a periodic lattice with them and compares with the C
restatement of the reference (the oracle, pinned bit for bit to the
reference's own build): they must agree to FP64 rounding, so any algebra
slip shows up here, before FP32 rounding hides it in the GPU tolerances.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import LYO_ALL, NEM_ALL

CX = np.array([0, 1, -1, 0, 0, 1, -1, -1, 1])
CY = np.array([0, 0, 0, 1, -1, 1, -1, 1, -1])
T = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


def sh(a, dx, dy):
    """a at (x + dx, y + dy) on the torus."""
    return np.roll(np.roll(a, -dx, axis=0), -dy, axis=1)


def stencil(a):
    xp, xm, yp, ym = sh(a, 1, 0), sh(a, -1, 0), sh(a, 0, 1), sh(a, 0, -1)
    return dict(c=a, s=(xp + xm) + (yp + ym), X=xp - xm, Y=yp - ym)


def uq2(P, lyo, g, A, B, Ph):
    """UpdateQuantities as uq2() in the kernel (g: deviations)."""
    dn = g.sum(axis=0)
    inv = 1.0 / (P["rho"] + dn)
    d56, d87 = g[5] - g[6], g[8] - g[7]
    jx = (g[1] - g[2]) + (d56 + d87)
    jy = (g[3] - g[4]) + (d56 - d87)
    vx, vy = jx * inv, jy * inv
    Qxx, Qyx = A["c"], B["c"]
    S2 = Qxx * Qxx + Qyx * Qyx
    c4k = -4 * P["LL"] if lyo else P["CC"] - 4 * P["LL"]
    c4 = -P["CC"] * S2 + c4k
    LsA, LsB = P["LL"] * A["s"], P["LL"] * B["s"]
    Hxx, Hyx = c4 * Qxx + LsA, c4 * Qyx + LsB
    aQ = Qxx * LsB - Qyx * LsA
    elr = (A["Y"] ** 2 + B["Y"] ** 2) - (A["X"] ** 2 + B["X"] ** 2)
    elSr = A["X"] * A["Y"] + B["X"] * B["Y"]
    QQ = Qxx * Qyx
    fF = (Qxx * Qxx - 1) * Hxx + QQ * Hyx
    fS = QQ * Hxx + (Qyx * Qyx - 1) * Hyx
    o = dict(dn=dn, ux=vx, uy=vy)
    if lyo:
        p = Ph["c"]
        nact = P["zeta"] * p - P["zeta"]
        pf = P["KK"] / 8 * ((Ph["Y"] - Ph["X"]) * (Ph["Y"] + Ph["X"]))
        pfS = -P["KK"] / 4 * (Ph["X"] * Ph["Y"])
        sigmaF = 2 * P["xi"] * fF + (nact * Qxx + (P["LL"] / 4 * elr + pf))
        sigmaS = 2 * P["xi"] * fS + (nact * Qyx + (-P["LL"] / 2 * elSr + pfS))
        pq = p * (1 - p)
        lp = Ph["s"] - 4 * p
        mu = P["AA"] * pq * (1 - 2 * p) - P["KK"] * lp
        y = 0.5 * P["CC"] * S2 * S2 + 0.5 * P["AA"] * pq * pq
        bi = P["zetaI"] * (P["conc"] - p) + (y - mu * p)
        o.update(MU=mu, uxp=vx * p, uyp=vy * p)
    else:
        nact = -P["zeta"]
        sigmaF = 2 * P["xi"] * fF + (nact * Qxx + P["LL"] / 4 * elr)
        sigmaS = 2 * P["xi"] * fS + (nact * Qyx - P["LL"] / 2 * elSr)
        bi = 0.5 * P["CC"] * (1 - S2) ** 2
        z = np.zeros_like(dn)
        o.update(MU=z, uxp=z, uyp=z)
    o.update(sXX=bi + sigmaF, sYY=bi - sigmaF, sXY=2 * aQ + sigmaS, sYX=-2 * aQ + sigmaS,
             BEx=P["GammaQ"] * Hxx - 0.5 * (vx * A["X"] + vy * A["Y"]),
             BEy=P["GammaQ"] * Hyx - 0.5 * (vx * B["X"] + vy * B["Y"]))
    return o


def uf2(P, lyo, c, Qxx, Qyx, tau):
    """UpdateFields up to the node update, as uf2() in the kernel: the
    rates and the equilibrium with the force folded in."""
    X = lambda k: sh(c[k], 1, 0) - sh(c[k], -1, 0)
    Y = lambda k: sh(c[k], 0, 1) - sh(c[k], 0, -1)
    Dxux, Dxuy, Dyux, Dyuy = X("ux"), X("uy"), Y("ux"), Y("uy")
    E2, S4, V4 = Dxux + Dyuy, Dxuy + Dyux, Dxuy - Dyux
    QS = Qyx * S4
    T2 = Qxx * (Dxux - Dyuy) + QS
    bx2 = (Qxx + 1) * (2 * Dxux - T2) + (QS - E2)
    by2 = Qyx * (E2 - T2) + S4
    Dxx = 0.5 * P["xi"] * bx2 + (-0.5 * V4 * Qyx + c["BEx"])
    Dyx = 0.5 * P["xi"] * by2 + (0.5 * V4 * Qxx + c["BEy"])
    Fx2 = -2 * P["friction"] * c["ux"] + (X("sXX") + Y("sXY"))
    Fy2 = -2 * P["friction"] * c["uy"] + (X("sYX") + Y("sYY"))
    if lyo:
        sMU = (sh(c["MU"], 1, 0) + sh(c["MU"], -1, 0)) + (sh(c["MU"], 0, 1) + sh(c["MU"], 0, -1))
        Dp = P["GammaP"] * (sMU - 4 * c["MU"]) - 0.5 * (X("uxp") + Y("uyp"))
    else:
        Dp = np.zeros_like(Dxx)
    dn = c["dn"]
    nn = P["rho"] + dn
    jx, jy = nn * c["ux"], nn * c["uy"]
    kxx, kyy, kxy = jx * c["ux"], jy * c["uy"], jx * c["uy"]
    k2 = kxx + kyy
    jxF, jyF = jx + 0.5 * tau * Fx2, jy + 0.5 * tau * Fy2
    A = k2 / 3 + dn / 9
    E1, E3 = A - 0.5 * kyy, A - 0.5 * kxx
    B = k2 / 12 + dn / 36
    Bp, Bm = B + 0.25 * kxy, B - 0.25 * kxy
    s, d = jxF + jyF, jxF - jyF
    fe = np.stack([4 / 9 * dn - 2 / 3 * k2, E1 + jxF / 3, E1 - jxF / 3, E3 + jyF / 3,
                   E3 - jyF / 3, Bp + s / 12, Bp - s / 12, Bm - d / 12, Bm + d / 12])
    return fe, Dxx, Dyx, Dp


def params_of(model, p):
    if model == O.LYOTROPIC:
        return dict(p)
    q = dict(p)
    q.update(GammaQ=p["Gamma"], tauNem=p["tau"], tauIso=p["tau"], GammaP=0.0, AA=0.0,
             KK=0.0, zetaI=0.0, conc=0.0)
    return q


def step(P, lyo, g, Qxx, Qyx, phi):
    """One Step() with npc = 1 on deviations g (9, LX, LY)."""
    st = lambda a: stencil(a)
    zero = np.zeros_like(Qxx)
    ph = phi if lyo else zero
    tau_of = lambda p: P["tauIso"] + (P["tauNem"] - P["tauIso"]) * p if lyo else \
        np.full_like(p, P["tauNem"])
    # predictor
    c = uq2(P, lyo, g, st(Qxx), st(Qyx), st(ph))
    tau = tau_of(ph)
    fe, Dxx, Dyx, Dp = uf2(P, lyo, c, Qxx, Qyx, tau)
    it = 1.0 / tau
    fn = g + 0.5 * it * (fe - g)
    ff = g + it * (fe - g)
    QNxx, QNyx, phn = Qxx + 0.5 * Dxx, Qyx + 0.5 * Dyx, ph + 0.5 * Dp
    Qxx, Qyx, ph = Qxx + Dxx, Qyx + Dyx, ph + Dp
    # Move (push: f_v(x + cx, y + cy) <- f_v(x, y))
    ff = np.stack([sh(ff[v], -CX[v], -CY[v]) for v in range(9)])
    fn = np.stack([sh(fn[v], -CX[v], -CY[v]) for v in range(9)])
    # corrector
    c = uq2(P, lyo, ff, st(Qxx), st(Qyx), st(ph))
    tau = tau_of(ph)
    fe, Dxx, Dyx, Dp = uf2(P, lyo, c, Qxx, Qyx, tau)
    h = fn - 0.5 / tau * ff
    g = h + 0.5 / tau * fe
    return g, QNxx + 0.5 * Dxx, QNyx + 0.5 * Dyx, (phn + 0.5 * Dp) if lyo else zero


@pytest.mark.parametrize("model,params", [(O.LYOTROPIC, LYO_ALL), (O.NEMATIC, NEM_ALL)])
def test_restated_algebra_equals_the_reference_in_fp64(model, params):
    LX, LY, steps = 12, 10, 3
    lyo = model == O.LYOTROPIC
    st = O.synthetic_state(model, LX, LY, seed=4, flow=0.03)
    ref = O.PortOracle(model, params, LX, LY, 0)
    for k, v in st.items():
        ref.set(k, v)
    ref.step(steps)
    P = params_of(model, params)
    g = (np.asarray(st["ff"]).reshape(LX, LY, 9) - T * P["rho"]).transpose(2, 0, 1)
    Qxx = np.asarray(st["QQxx"]).reshape(LX, LY)
    Qyx = np.asarray(st["QQyx"]).reshape(LX, LY)
    phi = np.asarray(st["phi"]).reshape(LX, LY) if lyo else np.zeros((LX, LY))
    for _ in range(steps):
        g, Qxx, Qyx, phi = step(P, lyo, g, Qxx, Qyx, phi)
    ff = g.transpose(1, 2, 0).reshape(-1, 9) + T * P["rho"]
    want_ff = ref.get("ff")
    dev = lambda a: a - T * P["rho"]
    assert np.abs(dev(ff) - dev(want_ff)).max() <= 1e-12 * np.abs(dev(want_ff)).max()
    for name, mine in (("QQxx", Qxx), ("QQyx", Qyx)) + ((("phi", phi),) if lyo else ()):
        w = ref.get(name)
        assert np.abs(mine.reshape(-1) - w).max() <= 1e-12 * max(np.abs(w).max(), 1.0), name
