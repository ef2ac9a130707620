"""Golden fixtures for the on-GPU flow/defect statistics, from the
reference's OWN post-processing code.

The states are lattices evolved by the CPU oracle (oracle/mass_oracle.c,
pinned to the reference) from seeded random directors, so they hold
defects and flow. The statistics are computed with the reference's Python:
  * defects: POST/massPy/nematic/nematicPy.py get_defects (threshold 0.4)
    on top of POST/massPy/base_modules/defects.py get_charge;
  * velocity, vorticity, perimeter_4, enstrophy density:
    plot/python/passive_q1_alpha_regime_analysis.py velocity_fields,
    vorticity, perimeter_4 and the 0.5*mean(omega^2) of its statistics.
massPy's package __init__ files import its plotting modules (matplotlib is
absent here), so the three modules used are loaded file by file. The analysis
script's
functions are taken from its source with `ast` and executed alone, so the
script's own imports and plotting set-up do not run.

    python tests/golden/gen_stats_golden.py
"""
from __future__ import annotations

import ast
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

REF = O.REF_DIR


def load_massPy():
    """nematicPy and base_modules.defects/numdiff of the reference's massPy,
    loaded file by file under empty package shells, so the package
    __init__ files (which import the plotting modules) do not run."""
    import importlib.util
    base = os.path.join(REF, "POST", "massPy")
    for pkg, path in (("mp", base), ("mp.base_modules", os.path.join(base, "base_modules")),
                      ("mp.nematic", os.path.join(base, "nematic"))):
        m = types.ModuleType(pkg)
        m.__path__ = [path]
        sys.modules[pkg] = m

    def load(name, path):
        spec = importlib.util.spec_from_file_location(name, path)
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
        return mod

    load("mp.base_modules.numdiff", os.path.join(base, "base_modules", "numdiff.py"))
    load("mp.base_modules.defects", os.path.join(base, "base_modules", "defects.py"))
    return load("mp.nematic.nematicPy", os.path.join(base, "nematic", "nematicPy.py"))


def load_analysis_functions():
    path = os.path.join(REF, "plot", "python", "passive_q1_alpha_regime_analysis.py")
    tree = ast.parse(open(path).read())
    want = {"velocity_fields", "vorticity", "perimeter_4"}
    mod = ast.Module(body=[n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in want],
                     type_ignores=[])
    ns = {"np": np}
    exec(compile(mod, path, "exec"), ns)
    return ns


class Frame:
    pass


def stats_for(state, LX, LY, nematicPy, fns):
    fr = Frame()
    fr.parameters = {"LX": LX, "LY": LY}
    fr.ff = state["ff"]
    vx, vy = fns["velocity_fields"](fr)
    omega = fns["vorticity"](vx, vy)
    out = {
        "mean_u2": float(np.mean(vx * vx + vy * vy)),
        "enstrophy_density": float(0.5 * np.mean(omega * omega)),
    }
    d = nematicPy.get_defects(state["QQxx"], state["QQyx"], LX, LY)
    out["defects_plus"] = sum(1 for x in d if x["charge"] > 0)
    out["defects_minus"] = sum(1 for x in d if x["charge"] < 0)
    if "phi" in state:
        mask = state["phi"].reshape(LX, LY) > 0.5
        out["perimeter"] = fns["perimeter_4"](mask)
        om = omega[mask]
        out["enstrophy_density_phi"] = float(0.5 * np.mean(om * om)) if om.size else 0.0
    return out


def main():
    nematicPy = load_massPy()
    fns = load_analysis_functions()
    cases = [
        ("stats_nem_64x48", O.NEMATIC, dict(Gamma=0.3, xi=0.7, tau=1.5, rho=40.0, CC=0.1,
                                            LL=0.05, zeta=0.02, npc=1), 64, 48, 30),
        ("stats_lyo_64x64", O.LYOTROPIC, dict(GammaQ=0.3, GammaP=0.1, xi=0.7, tauNem=1.5,
                                              tauIso=1.5, rho=40.0, AA=0.1, CC=0.1, LL=0.05,
                                              KK=0.05, zeta=0.03, conc=1.0, npc=1), 64, 64, 30),
    ]
    for name, model, params, LX, LY, steps in cases:
        st = O.synthetic_state(model, LX, LY, seed=5, flow=0.01, radius=LX / 4)
        P = O.PortOracle(model, params, LX, LY, 0)
        for k, v in st.items():
            P.set(k, v)
        P.step(steps)
        state = {k: P.get(k) for k in (["ff", "QQxx", "QQyx"] + (["phi"] if model == O.LYOTROPIC else []))}
        s = stats_for(state, LX, LY, nematicPy, fns)
        meta = dict(model=model, LX=LX, LY=LY, params=params, steps=steps, stats=s)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), meta=json.dumps(meta), **state)
        print(name, s)


if __name__ == "__main__":
    main()
