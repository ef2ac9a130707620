"""Python front-end of libmass_lb.so (include/mass_lb.h) through ctypes.

This mirrors the reference's model interface for one lattice: construct with
the runcard parameters and (LX, LY, BC) as declare_model's factory does
(src/models.hpp:197-205), upload the configured state, `step()` as
Model::Step(), read fields by their reference member names, and
`runtime_checks()` with the semantics of Model::RuntimeChecks()
(src/models/lyotropic.cpp:527-549): an error when |sum f - ftot| > 1.

There is no CPU fallback: if the CUDA library is missing or no sm_100 device
is present, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libmass_lb.so")

LYOTROPIC, NEMATIC, GO_OR_GROW = 0, 1, 2
FP64, FP32 = 0, 1

FIELDS = ("ff", "QQxx", "QQyx", "phi", "n", "ux", "uy", "ux_phi", "uy_phi",
          "HHxx", "HHyx", "MU", "dxQQxx", "dyQQxx", "dxQQyx", "dyQQyx",
          "sigmaXX", "sigmaYY", "sigmaYX", "sigmaXY", "sigma_bulk",
          "sigma_elastic_xx", "sigma_elastic_yx", "sigma_phase_field_xx",
          "sigma_phase_field_yx", "sigma_active_xx", "sigma_active_yx", "fn",
          "QNxx", "QNyx", "phn", "m", "chi", "mN")
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}

STATUS = {0: "OK", -1: "EINVAL", -2: "ECUDA", -3: "ENOMEM", -4: "EUNSUPPORTED",
          -5: "ENOTFINITE", -6: "ENODEV"}


class MassLBError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [("model", C.c_int)] + [
        (n, C.c_double) for n in ("GammaQ", "GammaP", "xi", "tauNem", "tauIso",
                                  "rho", "friction", "AA", "CC", "LL", "KK",
                                  "zeta", "zetaI", "conc")
    ] + [("npc", C.c_uint)]


class GogParams(C.Structure):
    """mass_lb_go_or_grow_params (include/mass_lb_ext.h)."""
    _fields_ = [(n, C.c_double) for n in ("B", "Snem", "Dchi", "Achi", "Ochi", "phiswitch",
                                          "phi_critical")] + [("growTogether", C.c_int)]


# GoOrGrow runcard names -> mass_lb_go_or_grow_params fields, with the
# reference's initialisers (src/models/go-or-grow.hpp:9-13) as defaults
GOG_PARAMS = (("B", "B", 0.0), ("Snem", "Snem", 1.0), ("Dchi", "Dchi", 0.0),
              ("Achi", "Achi", 0.0), ("Ochi", "Ochi", 0.0), ("phiswitch", "phiswitch", 0.0),
              ("phi-critical", "phi_critical", 1.0))


def make_gog_params(params: dict) -> GogParams:
    g = GogParams()
    for key, field, default in GOG_PARAMS:
        setattr(g, field, float(params.get(key, default)))
    g.growTogether = int(params.get("growTogether", 0))
    return g


class Stats(C.Structure):
    """mass_lb_stats (include/mass_lb_ext.h)."""
    _fields_ = [("mean_u2", C.c_double), ("enstrophy_density", C.c_double),
                ("enstrophy_density_phi", C.c_double), ("phi_area", C.c_double),
                ("perimeter", C.c_double), ("defects_plus", C.c_longlong),
                ("defects_minus", C.c_longlong), ("charged_sites", C.c_longlong)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


_lib = None


def library_path() -> str:
    return LIB_PATH


def load_library(build_if_missing: bool = False):
    """Load libmass_lb.so (raises if it is absent and not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if build_if_missing:
            from . import build as _b
            _b.build()
        else:
            raise MassLBError(-6, f"{LIB_PATH} is missing; run python -m mass_hd_b200.build")
    lib = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    sig = {
        "mass_lb_abi_version": (C.c_int, []),
        "mass_lb_last_error": (C.c_char_p, []),
        "mass_lb_field_name": (C.c_char_p, [C.c_int]),
        "mass_lb_create": (C.c_int, [C.POINTER(Params), C.c_uint, C.c_uint, C.c_uint,
                                     C.c_int, C.POINTER(vp)]),
        "mass_lb_destroy": (None, [vp]),
        "mass_lb_upload": (C.c_int, [vp, dp, dp, dp, dp]),
        "mass_lb_upload_field": (C.c_int, [vp, C.c_int, dp]),
        "mass_lb_step": (C.c_int, [vp, C.c_uint]),
        "mass_lb_download": (C.c_int, [vp, C.c_int, dp]),
        "mass_lb_checks": (C.c_int, [vp, dp, dp, ip]),
        "mass_lb_initial_totals": (C.c_int, [vp, dp, dp]),
        "mass_lb_synchronize": (C.c_int, [vp]),
        "mass_lb_stream": (vp, [vp]),
        "mass_lb_launches_per_step": (C.c_int, [vp]),
        "mass_lb_get_tile": (C.c_int, [vp, ip, ip]),
        "mass_lb_set_tile": (C.c_int, [vp, C.c_int, C.c_int]),
        "mass_lb_autotune": (C.c_int, [vp]),
        "mass_lb_uses_fused": (C.c_int, [vp]),
        "mass_lb_device_state": (C.c_int, [vp, C.POINTER(vp), C.POINTER(C.c_longlong), ip]),
        "mass_lb_rows_layout": (C.c_int, [vp, ip, ip]),
        "mass_lb_get_rows": (C.c_int, [vp, C.c_uint, C.c_uint, vp]),
        "mass_lb_put_rows": (C.c_int, [vp, C.c_uint, C.c_uint, vp]),
        "mass_lb_checks_rows": (C.c_int, [vp, C.c_uint, C.c_uint, dp, dp, ip]),
        "mass_lb_statistics": (C.c_int, [vp, C.POINTER(Stats)]),
        "mass_lb_save": (C.c_int, [vp, C.c_char_p]),
        "mass_lb_load": (C.c_int, [vp, C.c_char_p]),
        "mass_lb_set_phi_source": (C.c_int, [vp, dp]),
        "mass_lb_set_phi_conservation": (C.c_int, [vp, C.c_int, C.c_double]),
        "mass_lb_set_go_or_grow_params": (C.c_int, [vp, C.POINTER(GogParams)]),
        "mass_lb_mask_candidates": (C.c_int, [vp, C.POINTER(C.c_longlong)]),
        "mass_lb_draw_mask": (C.c_int, [vp, C.c_int, dp, C.c_longlong, C.c_double, C.c_double,
                                        C.c_double, C.c_double, C.c_double]),
        "mass_lb_get_mask": (C.c_int, [vp, C.c_int, C.POINTER(C.c_ubyte)]),
        "mass_lb_mask_supply": (C.c_int, [vp, dp, C.c_longlong]),
        "mass_lb_mask_staging": (C.c_int, [vp, C.c_longlong, C.POINTER(dp)]),
        "mass_lb_upload_async": (C.c_int, [vp, dp, dp, dp, dp]),
        "mass_lb_download_async": (C.c_int, [vp, C.c_int, dp]),
        "mass_lb_stream_wait": (C.c_int, [vp, vp]),
        "mass_lb_set_step_rows": (C.c_int, [vp, C.c_uint, C.c_uint]),
        "mass_lb_draw_masks_queued": (C.c_int, [vp, C.c_int] + [C.c_double] * 7),
        "mass_lb_mask_consumed": (C.c_int, [vp, C.POINTER(C.c_longlong)]),
        "mass_lb_mask_progress": (C.c_int, [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_int)]),
        "mass_lb_relax_free_energy": (C.c_int, [vp, C.c_uint, C.c_double, C.c_int, C.c_int, dp]),
        "mass_lb_ensemble_create": (C.c_int, [C.c_int, C.POINTER(Params), C.POINTER(C.c_uint),
                                              C.POINTER(C.c_uint), C.POINTER(vp)]),
        "mass_lb_ensemble_destroy": (None, [vp]),
        "mass_lb_ensemble_size": (C.c_int, [vp]),
        "mass_lb_ensemble_run": (vp, [vp, C.c_int]),
        "mass_lb_ensemble_step": (C.c_int, [vp, C.c_uint]),
        "mass_lb_ensemble_get_rows": (C.c_int, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _check(code: int):
    if code != 0:
        raise MassLBError(code, load_library().mass_lb_last_error().decode())


def make_params(model: int, params: dict) -> Params:
    """Runcard names -> mass_lb_params. Lyotropic and go-or-grow: GammaQ,
    GammaP, xi, tauNem, tauIso, rho, friction, AA, CC, LL, KK, zeta, zetaI,
    conc, npc. Nematic: Gamma, xi, tau, rho, friction, CC, LL, zeta, npc
    (Q_kBT and u_kBT must be 0)."""
    p = Params()
    p.model = model
    g = lambda k, d=0.0: float(params.get(k, d))
    if model in (LYOTROPIC, GO_OR_GROW):
        for k in ("GammaQ", "GammaP", "xi", "tauNem", "tauIso", "friction",
                  "AA", "CC", "LL", "KK", "zeta", "zetaI", "conc"):
            setattr(p, k, g(k))
        p.rho = g("rho", 40.0)
    else:
        if g("Q_kBT") != 0.0 or g("u_kBT") != 0.0:
            raise MassLBError(-4, "thermal fluctuations (Q_kBT, u_kBT) are not supported")
        p.GammaQ = g("Gamma")
        p.xi = g("xi")
        p.tauNem = p.tauIso = g("tau")
        p.rho = g("rho", 40.0)
        p.friction = g("friction")
        p.CC = g("CC")
        p.LL = g("LL")
        p.zeta = g("zeta")
    p.npc = int(params.get("npc", 1))
    return p


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Lattice:
    """One lattice on the current CUDA device (see module docstring)."""

    def __init__(self, model: int, params: dict, LX: int, LY: int, bc: int = 0,
                 precision: int = FP64):
        lib = load_library()
        self.model, self.LX, self.LY, self.bc, self.precision = model, LX, LY, bc, precision
        self._params = make_params(model, params)
        h = C.c_void_p()
        _check(lib.mass_lb_create(C.byref(self._params), LX, LY, bc, precision, C.byref(h)))
        self.h = h
        if model == GO_OR_GROW:
            self.set_go_or_grow_params(params)

    @classmethod
    def _borrowed(cls, h, model: int, LX: int, LY: int, params: Params) -> "Lattice":
        """A view of a handle owned elsewhere (an ensemble run)."""
        self = cls.__new__(cls)
        self.model, self.LX, self.LY, self.bc, self.precision = model, LX, LY, 0, FP32
        self._params = params
        self.h = C.c_void_p(h)
        self._owned = False
        return self

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "_owned", True):
                load_library().mass_lb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state -------------------------------------------------------------
    def upload(self, ff, QQxx, QQyx, phi=None):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (ff, QQxx, QQyx)]
        ph = None if phi is None else np.ascontiguousarray(phi, dtype=np.float64)
        N = self.LX * self.LY
        assert arrs[0].size == 9 * N and arrs[1].size == N and arrs[2].size == N
        _check(load_library().mass_lb_upload(self.h, _dp(arrs[0]), _dp(arrs[1]), _dp(arrs[2]),
                                             _dp(ph) if ph is not None else None))

    def upload_state(self, state: dict):
        """ff, QQxx, QQyx, phi and (go-or-grow) m from a dict of arrays."""
        if self.model == GO_OR_GROW and "m" in state:
            self.upload_field("m", state["m"])
        self.upload(state["ff"], state["QQxx"], state["QQyx"], state.get("phi"))

    def upload_field(self, name: str, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        _check(load_library().mass_lb_upload_field(self.h, FIELD_ID[name], _dp(a)))

    def get(self, name: str) -> np.ndarray:
        n = self.LX * self.LY * (9 if name in ("ff", "fn") else 1)
        out = np.empty(n, dtype=np.float64)
        _check(load_library().mass_lb_download(self.h, FIELD_ID[name], _dp(out)))
        return out.reshape(-1, 9) if name in ("ff", "fn") else out

    def upload_async(self, ff, QQxx, QQyx, phi=None):
        """mass_lb_upload_async: the arrays must be pinned, contiguous float64
        and left untouched until synchronize()."""
        arrs = [ff, QQxx, QQyx] + ([phi] if phi is not None else [])
        for a in arrs:
            assert a.dtype == np.float64 and a.flags.c_contiguous
        _check(load_library().mass_lb_upload_async(self.h, _dp(ff), _dp(QQxx), _dp(QQyx),
                                                   _dp(phi) if phi is not None else None))

    def get_into_async(self, name: str, out: np.ndarray) -> np.ndarray:
        """mass_lb_download_async into a pinned, contiguous float64 array;
        valid after synchronize()."""
        assert out.dtype == np.float64 and out.flags.c_contiguous
        _check(load_library().mass_lb_download_async(self.h, FIELD_ID[name], _dp(out)))
        return out

    def get_into(self, name: str, out: np.ndarray) -> np.ndarray:
        assert out.dtype == np.float64 and out.flags.c_contiguous
        _check(load_library().mass_lb_download(self.h, FIELD_ID[name], _dp(out)))
        return out

    def step(self, n: int = 1):
        _check(load_library().mass_lb_step(self.h, n))

    def save(self, path: str):
        """Full-precision binary checkpoint of the state (mass_lb_save)."""
        _check(load_library().mass_lb_save(self.h, os.fsencode(path)))

    def load(self, path: str):
        """Restore a checkpoint written by save() (same model and size)."""
        _check(load_library().mass_lb_load(self.h, os.fsencode(path)))

    def set_phi_source(self, rate):
        """Per-site phi source rate r (LX*LY values, site order; None
        removes it): phi_tmp += phi*r after every UpdateFields, as the
        division models do with r = alpha*division_mask - beta*death_mask."""
        if rate is None:
            _check(load_library().mass_lb_set_phi_source(self.h, None))
            return
        r = np.ascontiguousarray(rate, dtype=np.float64)
        assert r.size == self.LX * self.LY
        _check(load_library().mass_lb_set_phi_source(self.h, _dp(r)))

    def set_phi_conservation(self, on: bool, totalphi: float = 0.0):
        """The division models' conserve_phi correction
        Dp -= (sum phi - totalphi)/(LX*LY) (FP64 / walls only)."""
        _check(load_library().mass_lb_set_phi_conservation(self.h, int(bool(on)), float(totalphi)))

    def mask_candidates(self) -> int:
        """Number of sites with phi >= 0.5 (one random draw each)."""
        n = C.c_longlong()
        _check(load_library().mass_lb_mask_candidates(self.h, C.byref(n)))
        return n.value

    def draw_mask(self, kind: int, draws, coef: float, phi_critical: float, radius: float,
                  alpha: float, beta: float):
        """Division (kind 0) or death (kind 1) mask from one uniform draw per
        candidate site (site order), then the phi source
        alpha*division_mask - beta*death_mask."""
        d = np.ascontiguousarray(draws, dtype=np.float64)
        _check(load_library().mass_lb_draw_mask(self.h, int(kind), _dp(d), d.size, float(coef),
                                                float(phi_critical), float(radius),
                                                float(alpha), float(beta)))

    def mask_supply(self, draws, staged: bool = False):
        """Queue uniforms (stream order) for draw_masks_queued. staged: write
        them into the library's pinned staging buffer first
        (mass_lb_mask_staging), which the supply then sends up as it is."""
        d = np.ascontiguousarray(draws, dtype=np.float64)
        lib = load_library()
        if staged:
            buf = C.POINTER(C.c_double)()
            _check(lib.mass_lb_mask_staging(self.h, d.size, C.byref(buf)))
            C.memmove(buf, d.ctypes.data, d.nbytes)
            _check(lib.mass_lb_mask_supply(self.h, buf, d.size))
        else:
            _check(lib.mass_lb_mask_supply(self.h, _dp(d), d.size))

    def draw_masks_queued(self, kinds: int, division_coef: float, division_radius: float,
                          death_coef: float, death_radius: float, phi_critical: float,
                          alpha: float, beta: float):
        """Division (bit 0) and/or death (bit 1) masks from queued draws."""
        _check(load_library().mass_lb_draw_masks_queued(
            self.h, int(kinds), float(division_coef), float(division_radius), float(death_coef),
            float(death_radius), float(phi_critical), float(alpha), float(beta)))

    def mask_consumed(self) -> int:
        n = C.c_longlong()
        _check(load_library().mass_lb_mask_consumed(self.h, C.byref(n)))
        return n.value

    def mask_progress(self):
        """(consumed, pending) without waiting: draws consumed up to the last
        finished queued draw, and the queued draws issued after it."""
        n = C.c_longlong()
        k = C.c_int()
        _check(load_library().mass_lb_mask_progress(self.h, C.byref(n), C.byref(k)))
        return n.value, k.value

    def get_mask(self, kind: int) -> np.ndarray:
        out = np.empty(self.LX * self.LY, dtype=np.uint8)
        _check(load_library().mass_lb_get_mask(self.h, int(kind),
                                               out.ctypes.data_as(C.POINTER(C.c_ubyte))))
        return out.astype(bool)

    def set_go_or_grow_params(self, params: dict):
        """Go-or-grow runcard values (B, Snem, Dchi, Achi, Ochi, phiswitch,
        phi-critical, growTogether); missing keys take the reference's
        defaults. Called by the constructor for GO_OR_GROW lattices."""
        self._gog = make_gog_params(params)
        _check(load_library().mass_lb_set_go_or_grow_params(self.h, C.byref(self._gog)))

    def relax_free_energy(self, steps: int, dt: float = 1.0, relax_phi: bool = True,
                          relax_Q: bool = True) -> float:
        """GoOrGrow::RelaxFreeEnergy on the device; returns the relaxed
        total of phi (the reference's totalphi)."""
        out = C.c_double()
        _check(load_library().mass_lb_relax_free_energy(self.h, int(steps), float(dt),
                                                        int(bool(relax_phi)), int(bool(relax_Q)),
                                                        C.byref(out)))
        return out.value

    def synchronize(self):
        _check(load_library().mass_lb_synchronize(self.h))

    def set_step_rows(self, x0: int, nrows: int):
        """mass_lb_set_step_rows: steps write rows [x0, x0 + nrows) only
        (nrows = 0: the whole lattice again)."""
        _check(load_library().mass_lb_set_step_rows(self.h, x0, nrows))

    def wait_for(self, before: "Lattice"):
        """mass_lb_stream_wait: work queued on this lattice from now on starts
        after the work queued on `before` so far (no wait on the host)."""
        _check(load_library().mass_lb_stream_wait(self.h, before.h))

    def checks(self):
        f, p, bad = C.c_double(), C.c_double(), C.c_int()
        _check(load_library().mass_lb_checks(self.h, C.byref(f), C.byref(p), C.byref(bad)))
        return f.value, p.value, bool(bad.value)

    def initial_totals(self):
        f, p = C.c_double(), C.c_double()
        _check(load_library().mass_lb_initial_totals(self.h, C.byref(f), C.byref(p)))
        return f.value, p.value

    def runtime_checks(self):
        """Model::RuntimeChecks(): raise when the population sum drifted by
        more than 1 from its value at upload (src/models/lyotropic.cpp:529-536)
        or the state holds NaN/Inf."""
        f, p, bad = self.checks()
        ftot, _ = self.initial_totals()
        if bad:
            raise MassLBError(-5, "nan found in the lattice state")
        if abs(ftot - f) > 1:
            raise MassLBError(-5, f"f is not conserved ({ftot}/{f})")
        return f, p

    # -- introspection -------------------------------------------------------
    @property
    def stream(self) -> int:
        return load_library().mass_lb_stream(self.h) or 0

    @property
    def launches_per_step(self) -> int:
        return load_library().mass_lb_launches_per_step(self.h)

    @property
    def uses_fused(self) -> bool:
        return bool(load_library().mass_lb_uses_fused(self.h))

    def tile(self):
        a, b = C.c_int(), C.c_int()
        _check(load_library().mass_lb_get_tile(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_tile(self, threads: int, rows: int):
        _check(load_library().mass_lb_set_tile(self.h, threads, rows))

    def autotune(self):
        _check(load_library().mass_lb_autotune(self.h))

    def statistics(self) -> dict:
        """Flow and defect statistics of the current state (see
        mass_lb_statistics): mean_u2, enstrophy_density, enstrophy_density_phi,
        phi_area, perimeter, defects_plus, defects_minus, charged_sites."""
        st = Stats()
        _check(load_library().mass_lb_statistics(self.h, C.byref(st)))
        return st.as_dict()

    def device_state(self):
        p, stride, n = C.c_void_p(), C.c_longlong(), C.c_int()
        _check(load_library().mass_lb_device_state(self.h, C.byref(p), C.byref(stride), C.byref(n)))
        return p.value, stride.value, n.value

    # -- rows of the primary state (domain decomposition) ---------------------
    def rows_layout(self):
        """(planes per site, bytes per value) of get_rows / put_rows."""
        n, b = C.c_int(), C.c_int()
        _check(load_library().mass_lb_rows_layout(self.h, C.byref(n), C.byref(b)))
        return n.value, b.value

    def get_rows(self, x0: int, nrows: int, dst_ptr: int):
        """Rows [x0, x0+nrows) of every primary plane into the device buffer
        at dst_ptr ([plane][row][y], storage format), on the lattice's
        stream."""
        _check(load_library().mass_lb_get_rows(self.h, x0, nrows, C.c_void_p(dst_ptr)))

    def put_rows(self, x0: int, nrows: int, src_ptr: int):
        _check(load_library().mass_lb_put_rows(self.h, x0, nrows, C.c_void_p(src_ptr)))

    def checks_rows(self, x0: int, nrows: int):
        f, p, bad = C.c_double(), C.c_double(), C.c_int()
        _check(load_library().mass_lb_checks_rows(self.h, x0, nrows, C.byref(f), C.byref(p),
                                                  C.byref(bad)))
        return f.value, p.value, bool(bad.value)


class Ensemble:
    """Independent FP32 periodic lattices of uneven sizes and parameters,
    stepped together by one persistent kernel launch per step
    (mass_lb_ensemble_*, include/mass_lb_ext.h). `runs[i]` is a Lattice
    view of run i for upload, get, checks and statistics."""

    def __init__(self, model: int, params: list, sizes: list):
        lib = load_library()
        n = len(params)
        assert n == len(sizes) and n > 0
        self.model = model
        arr = (Params * n)(*[make_params(model, p) for p in params])
        lx = (C.c_uint * n)(*[int(s[0]) for s in sizes])
        ly = (C.c_uint * n)(*[int(s[1]) for s in sizes])
        h = C.c_void_p()
        _check(lib.mass_lb_ensemble_create(n, arr, lx, ly, C.byref(h)))
        self.h = h
        self.runs = [Lattice._borrowed(lib.mass_lb_ensemble_run(h, i), model, int(sizes[i][0]),
                                       int(sizes[i][1]), arr[i]) for i in range(n)]

    def __len__(self):
        return len(self.runs)

    def step(self, n: int = 1):
        _check(load_library().mass_lb_ensemble_step(self.h, n))

    @property
    def rows(self) -> int:
        return load_library().mass_lb_ensemble_get_rows(self.h)

    def close(self):
        if getattr(self, "h", None):
            for r in self.runs:
                r.h = None
            load_library().mass_lb_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
