"""ctypes front-ends for the two CPU oracles (test infrastructure only).

* ``PortOracle`` - the plain-C FP64 restatement in ``oracle/mass_oracle.c``
  (built to ``oracle/_build/libmass_oracle.so``).
* ``RefOracle``  - the reference's own model sources compiled with the
  harness ``oracle/ref_harness.cpp`` (built to ``oracle/_ref/libmass_ref.so``).

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference legs import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "libmass_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmass_ref.so")
# The reference checkout read by the oracle recipes and the fixture scripts:
# MASS_REFERENCE_DIR when set, else the same default oracle/Makefile uses.
REF_DIR = os.environ.get("MASS_REFERENCE_DIR") or "/root/reference"

LYOTROPIC, NEMATIC, GO_OR_GROW = 0, 1, 2

# Runcard option names per model (src/models/lyotropic.cpp:556-599,
# src/models/nematic.cpp:414-442).
LYO_OPTIONS = ("GammaQ", "GammaP", "xi", "tauNem", "tauIso", "rho", "friction",
               "AA", "CC", "LL", "KK", "zeta", "zetaI", "npc", "config",
               "level", "conc", "radius", "angle", "noise")
NEM_OPTIONS = ("Gamma", "xi", "tau", "rho", "Q_kBT", "u_kBT", "friction", "CC",
               "LL", "zeta", "npc", "angle", "noise")
# LyotropicWithDivision::GetOptions (src/models/lyotropic-with-division.cpp:126-142)
DIV_OPTIONS = ("alpha", "beta", "division-rate", "division-time", "division-radius",
               "death-rate", "death-time", "death-radius", "phi-critical")
# GoOrGrow::GetOptions (src/models/go-or-grow.cpp:420-470)
GOG_OPTIONS = ("B", "Snem", "Dchi", "Achi", "Ochi", "phiswitch", "growTogether",
               "chi-config", "chi0", "chi-noise", "chi-length", "relax-steps",
               "relax-dt", "relax-phi", "relax-Q")

SCALAR_FIELDS_LYO = ("QQxx", "QQyx", "QNxx", "QNyx", "phi", "phn", "n", "ux",
                     "uy", "ux_phi", "uy_phi", "HHxx", "HHyx", "MU", "dxQQxx",
                     "dyQQxx", "dxQQyx", "dyQQyx", "sigmaXX", "sigmaYY",
                     "sigmaYX", "sigmaXY", "sigma_bulk", "sigma_elastic_xx",
                     "sigma_elastic_yx", "sigma_phase_field_xx",
                     "sigma_phase_field_yx", "sigma_active_xx",
                     "sigma_active_yx")
SCALAR_FIELDS_NEM = ("QQxx", "QQyx", "QNxx", "QNyx", "n", "ux", "uy", "HHxx",
                     "HHyx", "dxQQxx", "dyQQxx", "dxQQyx", "dyQQyx", "sigmaXX",
                     "sigmaYY", "sigmaYX", "sigmaXY")


def build(ref: bool = True) -> None:
    """Build the port (always) and the reference library (when its sources
    are present) with oracle/Makefile."""
    targets = ["port"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


class _MoParams(C.Structure):
    _fields_ = [("model", C.c_int)] + [
        (n, C.c_double) for n in ("GammaQ", "GammaP", "xi", "tauNem", "tauIso",
                                  "rho", "friction", "AA", "CC", "LL", "KK",
                                  "zeta", "zetaI", "conc")
    ] + [("npc", C.c_uint)]


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


_port_lib = None


def _port():
    global _port_lib
    if _port_lib is None:
        if not os.path.exists(PORT_SO):
            build(ref=False)
        lib = C.CDLL(PORT_SO)
        lib.mo_new.restype = C.c_void_p
        lib.mo_new.argtypes = [C.POINTER(_MoParams), C.c_uint, C.c_uint, C.c_uint]
        lib.mo_free.argtypes = [C.c_void_p]
        lib.mo_set_field.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double)]
        lib.mo_get_field.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double)]
        lib.mo_step.argtypes = [C.c_void_p, C.c_uint]
        lib.mo_totals.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _port_lib = lib
    return _port_lib


def params_struct(model: int, params: dict) -> _MoParams:
    """Map runcard names of either model onto the restatement's struct."""
    p = _MoParams()
    p.model = model
    g = lambda k, d=0.0: float(params.get(k, d))
    if model == LYOTROPIC:
        for k in ("GammaQ", "GammaP", "xi", "tauNem", "tauIso", "friction",
                  "AA", "CC", "LL", "KK", "zeta", "zetaI", "conc"):
            setattr(p, k, g(k))
        p.rho = g("rho", 40.0)
    else:
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


class PortOracle:
    """FP64 C restatement of Step(); state set/read by field name."""

    def __init__(self, model: int, params: dict, LX: int, LY: int, bc: int = 0):
        self.model, self.LX, self.LY, self.bc = model, LX, LY, bc
        self._p = params_struct(model, params)
        self.h = _port().mo_new(C.byref(self._p), LX, LY, bc)
        if not self.h:
            raise RuntimeError("mo_new failed")

    def __del__(self):
        if getattr(self, "h", None):
            _port().mo_free(self.h)
            self.h = None

    def set(self, name: str, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if _port().mo_set_field(self.h, name.encode(), _dp(a)) != 0:
            raise KeyError(name)

    def get(self, name: str) -> np.ndarray:
        n = self.LX * self.LY * (9 if name in ("ff", "fn") else 1)
        out = np.empty(n, dtype=np.float64)
        if _port().mo_get_field(self.h, name.encode(), _dp(out)) != 0:
            raise KeyError(name)
        return out.reshape(-1, 9) if name in ("ff", "fn") else out

    def step(self, n: int = 1) -> None:
        _port().mo_step(self.h, n)

    def totals(self):
        f, p = C.c_double(), C.c_double()
        _port().mo_totals(self.h, C.byref(f), C.byref(p))
        return f.value, p.value


_ref_lib = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _ref():
    global _ref_lib
    if _ref_lib is None:
        lib = C.CDLL(REF_SO)
        lib.ref_new.restype = C.c_void_p
        lib.ref_new.argtypes = [C.c_char_p, C.c_uint, C.c_uint, C.c_uint]
        lib.ref_free.argtypes = [C.c_void_p]
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_set_option.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p]
        lib.ref_initialize.argtypes = [C.c_void_p]
        lib.ref_configure.argtypes = [C.c_void_p, C.c_uint]
        lib.ref_set_field.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double)]
        lib.ref_get_field.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double)]
        lib.ref_get_mask.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_ubyte)]
        lib.ref_get_value.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double)]
        lib.ref_reset_totals.argtypes = [C.c_void_p]
        lib.ref_step.argtypes = [C.c_void_p, C.c_uint, C.c_uint]
        lib.ref_time_steps.argtypes = [C.c_void_p, C.c_uint, C.c_uint]
        lib.ref_time_steps.restype = C.c_double
        lib.ref_runtime_checks.argtypes = [C.c_void_p]
        lib.ref_write_params.argtypes = [C.c_void_p, C.c_char_p, C.c_uint,
                                         C.c_uint, C.c_uint, C.c_char_p]
        lib.ref_write_frame.argtypes = [C.c_void_p, C.c_char_p]
        lib.ref_random_reals.argtypes = [C.c_uint, C.c_int, C.c_uint,
                                         C.POINTER(C.c_double)]
        _ref_lib = lib
    return _ref_lib


class RefOracle:
    """The reference's own Lyotropic / LyotropicWithDivision / GoOrGrow /
    Nematic model objects (`division=True` selects "lyotropic-with-division";
    model GO_OR_GROW selects "go-or-grow", which carries the division
    options too)."""

    def __init__(self, model: int, params: dict, LX: int, LY: int, bc: int = 0,
                 division: bool = False):
        self.model, self.LX, self.LY, self.bc = model, LX, LY, bc
        if model == GO_OR_GROW:
            name = b"go-or-grow"
        elif model == LYOTROPIC:
            name = b"lyotropic-with-division" if division else b"lyotropic"
        else:
            name = b"nematic"
        self.h = _ref().ref_new(name, LX, LY, bc)
        if not self.h:
            raise RuntimeError(_ref().ref_last_error().decode())
        names = NEM_OPTIONS if model == NEMATIC else LYO_OPTIONS
        if division or model == GO_OR_GROW:
            names = names + DIV_OPTIONS
        if model == GO_OR_GROW:
            names = names + GOG_OPTIONS
        # every option gets a value: the reference leaves them uninitialised
        defaults = {"config": "circle", "level": 0.0, "conc": 1.0,
                    "radius": 0.0, "angle": 0.0, "noise": 0.0,
                    "Q_kBT": 0.0, "u_kBT": 0.0, "npc": 1, "rho": 40.0,
                    "Snem": 1.0, "relax-dt": 1.0, "chi-config": "noise",
                    "phi-critical": 1.0}
        for k in names:
            v = params.get(k, defaults.get(k, 0.0))
            r = _ref().ref_set_option(self.h, k.encode(), str(v).encode())
            if r != 0:
                raise KeyError(f"option {k}={v}: {r}")
        if _ref().ref_initialize(self.h) != 0:
            raise RuntimeError(_ref().ref_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            _ref().ref_free(self.h)
            self.h = None

    def configure(self, seed: int) -> None:
        if _ref().ref_configure(self.h, seed) != 0:
            raise RuntimeError(_ref().ref_last_error().decode())

    def set(self, name: str, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if _ref().ref_set_field(self.h, name.encode(), _dp(a)) != 0:
            raise KeyError(name)

    def reset_totals(self) -> None:
        _ref().ref_reset_totals(self.h)

    def get(self, name: str) -> np.ndarray:
        n = self.LX * self.LY * (9 if name in ("ff", "fn") else 1)
        out = np.empty(n, dtype=np.float64)
        if _ref().ref_get_field(self.h, name.encode(), _dp(out)) != 0:
            raise KeyError(name)
        return out.reshape(-1, 9) if name in ("ff", "fn") else out

    def mask(self, name: str) -> np.ndarray:
        """division_mask / death_mask of the division model (bool array)."""
        out = np.empty(self.LX * self.LY, dtype=np.uint8)
        if _ref().ref_get_mask(self.h, name.encode(), out.ctypes.data_as(C.POINTER(C.c_ubyte))) != 0:
            raise KeyError(name)
        return out.astype(bool)

    def value(self, name: str) -> float:
        """totalphi, countphi or conserve_phi of the lyotropic models."""
        out = C.c_double()
        if _ref().ref_get_value(self.h, name.encode(), C.byref(out)) != 0:
            raise KeyError(name)
        return out.value

    def step(self, n: int = 1, threads: int = 0) -> None:
        _ref().ref_step(self.h, n, threads)

    def time_steps(self, n: int, threads: int) -> float:
        return _ref().ref_time_steps(self.h, n, threads)

    def runtime_checks(self) -> str | None:
        r = _ref().ref_runtime_checks(self.h)
        return None if r == 0 else _ref().ref_last_error().decode()

    def write_params(self, path: str, nsteps: int, ninfo: int, nstart: int,
                     model_name: str) -> None:
        if _ref().ref_write_params(self.h, path.encode(), nsteps, ninfo, nstart,
                                   model_name.encode()) != 0:
            raise RuntimeError(_ref().ref_last_error().decode())

    def write_frame(self, path: str) -> None:
        if _ref().ref_write_frame(self.h, path.encode()) != 0:
            raise RuntimeError(_ref().ref_last_error().decode())


def ref_random_reals(seed: int, n: int) -> np.ndarray:
    """n draws of the reference's random_real() after set_seed(seed)."""
    out = np.empty(n, dtype=np.float64)
    _ref().ref_random_reals(seed, 1, n, _dp(out))
    return out


# ---------------------------------------------------------------------------
# Seeded synthetic states used by the tests (same arrays go to every side).

W_EQ = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


def equilibrium_np(vx, vy, nn):
    """src/lb.hpp:24-41 vectorised (same operation order per element)."""
    v2 = vx * vx + vy * vy
    fe = np.empty(np.shape(nn) + (9,))
    fe[..., 1] = nn * (1. / 9. + 1. / 3. * vx + 1. / 3. * v2 - 1. / 2. * vy * vy)
    fe[..., 2] = nn * (1. / 9. - 1. / 3. * vx + 1. / 3. * v2 - 1. / 2. * vy * vy)
    fe[..., 3] = nn * (1. / 9. + 1. / 3. * vy - 1. / 2. * vx * vx + 1. / 3. * v2)
    fe[..., 4] = nn * (1. / 9. - 1. / 3. * vy - 1. / 2. * vx * vx + 1. / 3. * v2)
    fe[..., 5] = nn * (1. / 36. + 1. / 12. * vx + 1. / 12. * vy + 1. / 12. * v2 + 1. / 4. * vx * vy)
    fe[..., 6] = nn * (1. / 36. - 1. / 12. * vx - 1. / 12. * vy + 1. / 12. * v2 + 1. / 4. * vx * vy)
    fe[..., 7] = nn * (1. / 36. - 1. / 12. * vx + 1. / 12. * vy + 1. / 12. * v2 - 1. / 4. * vx * vy)
    fe[..., 8] = nn * (1. / 36. + 1. / 12. * vx - 1. / 12. * vy + 1. / 12. * v2 - 1. / 4. * vx * vy)
    fe[..., 0] = nn - fe[..., 1] - fe[..., 2] - fe[..., 3] - fe[..., 4] - fe[..., 5] \
        - fe[..., 6] - fe[..., 7] - fe[..., 8]
    return fe


def synthetic_state(model: int, LX: int, LY: int, seed: int, rho: float = 40.0,
                    flow: float = 0.0, phi_kind: str = "disk",
                    radius: float | None = None):
    """Random director (S=1, angle U[0, pi)) on every site; for lyotropic a
    tanh disk phi = 0.5(1 - tanh((r-R)/2)) centred at (LX/2, LY/2), or
    phi ~ N(0.5, 0.05) i.i.d. (phi_kind="noise"). `flow` > 0 adds a random
    velocity of that amplitude to the equilibrium populations so that the
    first steps already exercise every term."""
    rng = np.random.default_rng(seed)
    N = LX * LY
    theta = rng.uniform(0.0, np.pi, N)
    state = {"QQxx": np.cos(2 * theta), "QQyx": np.sin(2 * theta)}
    if flow > 0:
        vx = flow * rng.uniform(-1, 1, N)
        vy = flow * rng.uniform(-1, 1, N)
    else:
        vx = np.zeros(N)
        vy = np.zeros(N)
    state["ff"] = equilibrium_np(vx, vy, np.full(N, rho))
    if model == LYOTROPIC:
        if phi_kind == "noise":
            state["phi"] = rng.normal(0.5, 0.05, N)
        else:
            R = radius if radius is not None else LX / 4
            x = np.arange(LX)[:, None] - LX / 2
            y = np.arange(LY)[None, :] - LY / 2
            r = np.sqrt(x * x + y * y).reshape(-1)
            state["phi"] = 0.5 * (1 - np.tanh((r - R) / 2))
    return state
