"""Generate the golden fixtures in this directory from the REFERENCE itself.

Runs the reference's own model sources (compiled by ``make -C oracle ref``
into ``oracle/_ref/libmass_ref.so`` from the read-only reference checkout)
and stores, per case, the seeded input state and the in-memory FP64 fields
after a number of Step() calls. Also stores the reference's Configure()
output for a given seed and the reference's JSON writer output for a tiny
lattice. The fixtures let the CPU test suite pin the oracle restatement (and
the GPU suite pin the CUDA path) without the reference being present.

    python tests/golden/gen_golden.py
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

LYO = dict(GammaQ=0.3, GammaP=0.1, xi=0.7, tauNem=1.5, tauIso=1.5, rho=40.0,
           friction=0.0, AA=0.1, CC=0.1, LL=0.05, KK=0.05, zeta=0.01,
           zetaI=0.0, conc=1.0, npc=1)
NEM = dict(Gamma=0.3, xi=0.7, tau=1.5, rho=40.0, friction=0.0, CC=0.1,
           LL=0.05, zeta=0.02, npc=1)

# (name, model, params, LX, LY, bc, steps, seed, flow)
CASES = [
    ("lyo_bc0_24x20", O.LYOTROPIC, dict(LYO), 24, 20, 0, 10, 1, 0.0),
    ("lyo_bc0_flow_17x13", O.LYOTROPIC,
     dict(LYO, zetaI=0.02, friction=0.01, tauIso=1.2, npc=2), 17, 13, 0, 6, 2, 0.01),
    ("lyo_bc1_12x10", O.LYOTROPIC, dict(LYO, zeta=0.05), 12, 10, 1, 5, 3, 0.01),
    ("lyo_bc2_12x10", O.LYOTROPIC, dict(LYO, zeta=0.05), 12, 10, 2, 5, 4, 0.01),
    ("lyo_bc3_12x10", O.LYOTROPIC, dict(LYO, zeta=0.05), 12, 10, 3, 5, 5, 0.01),
    ("lyo_bc4_12x10", O.LYOTROPIC, dict(LYO, zeta=0.05), 12, 10, 4, 5, 6, 0.01),
    ("lyo_bc5_12x10", O.LYOTROPIC, dict(LYO, zeta=0.05), 12, 10, 5, 5, 7, 0.01),
    ("nem_bc0_24x20", O.NEMATIC, dict(NEM), 24, 20, 0, 10, 8, 0.0),
    ("nem_bc0_flow_9x31", O.NEMATIC, dict(NEM, friction=0.02, npc=3), 9, 31, 0, 4, 9, 0.01),
    ("nem_bc1_12x10", O.NEMATIC, dict(NEM), 12, 10, 1, 5, 10, 0.01),
]

OUT_FIELDS_LYO = ("ff", "fn", "QQxx", "QQyx", "phi", "QNxx", "phn", "ux", "uy",
                  "n", "MU", "sigmaXX", "sigmaYY", "sigmaXY", "sigmaYX",
                  "sigma_bulk", "sigma_elastic_xx", "sigma_elastic_yx",
                  "sigma_phase_field_xx", "sigma_phase_field_yx",
                  "sigma_active_xx", "sigma_active_yx")
OUT_FIELDS_NEM = ("ff", "fn", "QQxx", "QQyx", "QNxx", "ux", "uy", "n",
                  "sigmaXX", "sigmaYY", "sigmaXY", "sigmaYX")


def gen_cases():
    for (name, model, params, LX, LY, bc, steps, seed, flow) in CASES:
        st = O.synthetic_state(model, LX, LY, seed=seed, flow=flow)
        r = O.RefOracle(model, params, LX, LY, bc)
        for k, v in st.items():
            r.set(k, v)
        r.step(steps)
        out = {"in_" + k: v for k, v in st.items()}
        fields = OUT_FIELDS_LYO if model == O.LYOTROPIC else OUT_FIELDS_NEM
        for f in fields:
            out["out_" + f] = r.get(f)
        meta = dict(model=model, params=params, LX=LX, LY=LY, bc=bc,
                    steps=steps, seed=seed, flow=flow)
        np.savez_compressed(os.path.join(HERE, name + ".npz"),
                            meta=json.dumps(meta), **out)
        print("wrote", name)


def gen_configure():
    """Reference Configure() for a few init configs and seeds (x-major k
    order, one random_real() per site)."""
    out = {}
    cfgs = [
        ("lyo_circle", O.LYOTROPIC, dict(LYO, config="circle", radius=5.0,
                                         conc=1.0, angle=30.0, noise=0.4), 20, 16, 0),
        ("lyo_stripe", O.LYOTROPIC, dict(LYO, config="stripe", level=6.0,
                                         conc=0.8, angle=0.0, noise=1.0), 16, 12, 0),
        ("lyo_square", O.LYOTROPIC, dict(LYO, config="square", level=7.0,
                                         conc=1.0, angle=10.0, noise=0.2), 16, 12, 0),
        ("lyo_half", O.LYOTROPIC, dict(LYO, config="half", level=5.0,
                                       conc=1.0, angle=45.0, noise=1.0), 12, 12, 0),
        ("lyo_boxatwall_bc4", O.LYOTROPIC, dict(LYO, config="boxatwall", level=4.0,
                                                conc=1.0, angle=0.0, noise=1.0), 12, 10, 4),
        ("lyo_wettedwall_bc1", O.LYOTROPIC, dict(LYO, config="wettedwall", level=3.0,
                                                 conc=1.0, angle=0.0, noise=1.0), 12, 10, 1),
        ("nem_random", O.NEMATIC, dict(NEM, angle=0.0, noise=1.0), 16, 12, 0),
    ]
    meta = {}
    for (name, model, params, LX, LY, bc) in cfgs:
        r = O.RefOracle(model, params, LX, LY, bc)
        r.configure(1234)
        keys = ["ff", "QQxx", "QQyx"] + (["phi"] if model == O.LYOTROPIC else [])
        for k in keys:
            out[name + "__" + k] = r.get(k)
        meta[name] = dict(model=model, params=params, LX=LX, LY=LY, bc=bc, seed=1234)
    out["random_reals_seed42"] = O.ref_random_reals(42, 64)
    np.savez_compressed(os.path.join(HERE, "configure.npz"),
                        meta=json.dumps(meta), **out)
    print("wrote configure")


def gen_json():
    """Reference oarchive output (parameters.json, frame<t>.json) for a tiny
    lattice after 3 steps."""
    for tag, model, params, LX, LY in (("lyo", O.LYOTROPIC, dict(LYO, config="circle", radius=2.0, level=0.0, conc=1.0, angle=0.0, noise=1.0), 4, 3),
                                       ("nem", O.NEMATIC, dict(NEM, angle=0.0, noise=1.0), 4, 3)):
        r = O.RefOracle(model, params, LX, LY, 0)
        r.configure(7)
        r.step(3)
        with tempfile.TemporaryDirectory() as d:
            pth = os.path.join(d, "p.json")
            fr = os.path.join(d, "f.json")
            r.write_params(pth, 3, 1, 0, "lyotropic" if model == O.LYOTROPIC else "nematic")
            r.write_frame(fr)
            for src, dst in ((pth, f"{tag}_parameters.json"), (fr, f"{tag}_frame3.json")):
                with open(src) as fi, open(os.path.join(HERE, dst), "w") as fo:
                    fo.write(fi.read())
        names = ["ff", "QQxx", "QQyx"]
        if model == O.LYOTROPIC:
            names += ["phi", "sigmaXX", "sigmaXY", "sigmaYX", "sigmaYY", "sigma_bulk",
                      "sigma_elastic_xx", "sigma_elastic_yx", "sigma_phase_field_xx",
                      "sigma_phase_field_yx", "sigma_active_xx", "sigma_active_yx"]
        st = {k: r.get(k) for k in names}
        np.savez_compressed(os.path.join(HERE, f"{tag}_frame3_state.npz"), **st)
        print("wrote json", tag)


DIV_JSON = {"alpha": 0.05, "beta": 0.03, "division-rate": 0.6, "division-time": 1,
            "division-radius": 1.5, "death-rate": 0.3, "death-time": 2, "death-radius": 1.0,
            "phi-critical": 1.5}


def gen_json_division():
    """Reference output of LyotropicWithDivision (masks included in the
    frame) for an 8x6 lattice after 5 steps with division and death on."""
    params = dict(LYO, config="circle", radius=2.5, level=0.0, conc=1.0, angle=0.0, noise=1.0)
    params.update(DIV_JSON)
    r = O.RefOracle(O.LYOTROPIC, params, 8, 6, 0, division=True)
    r.configure(7)
    r.step(5)
    with tempfile.TemporaryDirectory() as d:
        pth = os.path.join(d, "p.json")
        fr = os.path.join(d, "f.json")
        r.write_params(pth, 5, 5, 0, "lyotropic-with-division")
        r.write_frame(fr)
        for src, dst in ((pth, "div_parameters.json"), (fr, "div_frame5.json")):
            with open(src) as fi, open(os.path.join(HERE, dst), "w") as fo:
                fo.write(fi.read())
    print("wrote json div")


# go-or-grow: every phenotype term on, crowding active (phi-critical below
# the circle's plateau), relaxation, division and death
GOG_JSON = {"B": 0.1, "Snem": 1.0, "Dchi": 0.01, "Achi": 0.1, "Ochi": 0.05, "phiswitch": 0.5,
            "growTogether": 1, "chi0": 0.6, "chi-noise": 0.05, "chi-length": 1.5,
            "relax-steps": 10, "relax-dt": 1.0, "relax-phi": 1, "relax-Q": 1,
            "alpha": 0.01, "beta": 0.005, "division-rate": 0.6, "division-time": 1,
            "division-radius": 1.5, "death-rate": 0.3, "death-time": 2, "death-radius": 1.0,
            "phi-critical": 0.9}
# (fixture prefix, bc, chi-config, LX, LY)
GOG_CASES = (("gog", 0, "noise", 16, 12), ("gog_box", 3, "front", 12, 10))


def gen_json_gog(outdir: str = HERE):
    """Reference output of GoOrGrow (masks, m and chi included in the frame)
    after 5 steps: a periodic lattice with smoothed phenotype noise, and a
    box with the phenotype front. Written to `outdir`."""
    for prefix, bc, cfg, LX, LY in GOG_CASES:
        params = dict(LYO, config="circle", radius=3.5, level=0.0, conc=1.0, angle=0.0,
                      noise=1.0, zeta=0.02)
        params.update(GOG_JSON)
        params["chi-config"] = cfg
        r = O.RefOracle(O.GO_OR_GROW, params, LX, LY, bc)
        r.configure(7)
        r.step(5)
        with tempfile.TemporaryDirectory() as d:
            pth = os.path.join(d, "p.json")
            fr = os.path.join(d, "f.json")
            r.write_params(pth, 5, 5, 0, "go-or-grow")
            r.write_frame(fr)
            for src, dst in ((pth, f"{prefix}_parameters.json"), (fr, f"{prefix}_frame5.json")):
                with open(src) as fi, open(os.path.join(outdir, dst), "w") as fo:
                    fo.write(fi.read())
    print("wrote json go-or-grow")


if __name__ == "__main__":
    if not O.ref_available():
        O.build(ref=True)
    which = sys.argv[1:] or ["cases", "configure", "json", "division", "go-or-grow"]
    if "cases" in which:
        gen_cases()
    if "configure" in which:
        gen_configure()
    if "json" in which:
        gen_json()
    if "division" in which:
        gen_json_division()
    if "go-or-grow" in which:
        gen_json_gog()
