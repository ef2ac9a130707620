"""Benchmark of the FP32 lyotropic Model::Step() on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--size L] [--model lyotropic|nematic|go-or-grow]
                    [--precision fp32|fp64]

Workload (default): the lyotropic model on a periodic 4096 x 4096 lattice in
FP32 - the throughput target named for this path - with the physics of the
256^2 CPU configuration (rho=40, tau=1.5, CC=0.1, AA=0.1, KK=0.05, LL=0.05,
GammaQ=0.3, GammaP=0.1, xi=0.7, zeta=0.01, npc=1), director angle i.i.d.
U[0, pi) with S=1, phi a tanh disk of radius L/4. Seeded synthetic input.

A step is one Model::Step() over the whole lattice (one fused kernel
launch). `value` is site-updates/s with the state resident in HBM, timed
with CUDA events on the library's stream; the 805 MB state per buffer is
larger than the 126 MB L2, so no flush is needed. `e2e` goes through the C
ABI with host buffers: each e2e step uploads the state from pinned host
memory, runs 100 steps (the output interval of the configuration) and
downloads the primary frame fields (ff, QQxx, QQyx, phi). Jobs alternate
between two handles, so that one job's transfers overlap the other's steps;
the serial rate (one handle, one job after another) is reported beside it.

With --gpus N (torchrun), every rank advances its own lattice of the same
size (independent runs, weak scaling, no collective on the data path); time
is the max over ranks. --decomp slab instead splits ONE lattice into
x-slabs over the ranks, with a halo-row exchange over NCCL before every
step (strong scaling).

The line also carries `fp64`: the FP64 mode (bit-identical to the
reference's double-precision build) timed on the same seeded lattice, the
like-for-like counterpart of the reference's FP64 CPU build; and
`ensemble`: the 96-run batched sweep against the same runs one after
another (a bounded sample of 200 steps per run); and `surrogate`: the
learned surrogate's tcgen05 convolutions at the training shape, each with
its fraction of the measured BF16 peak, and its training step.

--impl reference times the reference's own OpenMP build of the same step
(oracle/_ref, compiled from the reference sources) on the host cores, on a
bounded sample of the same workload.

--model go-or-grow measures the model every shipped runcard uses, with the
physics and division settings of the reference's cases/test/test.dat on an
L x L periodic lattice (default 500, the runcards' size). `value` times
the device step alone (a fixed growth-rate plane, CUDA events); `e2e` runs
the mass-gpu driver on the runcard (Configure with the device relaxation,
then the time loop with the division masks drawn on the host every step
they are due, as Model::Step() does) and divides by the driver's own
time-loop clock. The CPU baseline and the reference arm time the
reference's GoOrGrow::Step(), masks included, on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "site-updates/s"
BC_NAMES = {1: "free-slip channel walls", 2: "no-slip channel walls",
            3: "free-slip box walls", 4: "no-slip box walls"}
UNIT = "site-updates/s"
NINFO = 100

LYO_C1 = dict(GammaQ=0.3, GammaP=0.1, xi=0.7, tauNem=1.5, tauIso=1.5, rho=40.0,
              friction=0.0, AA=0.1, CC=0.1, LL=0.05, KK=0.05, zeta=0.01,
              zetaI=0.0, conc=1.0, npc=1)
NEM_C2 = dict(Gamma=0.3, xi=0.7, tau=1.5, rho=40.0, friction=0.0, CC=0.1,
              LL=0.05, zeta=0.02, npc=1)


# go-or-grow: the physics and division settings of the reference's
# cases/test/test.dat (its lattice is 100^2; the study runcards use 500^2)
GOG_RUNCARD = dict(GammaQ=0.3, GammaP=5e-2, zeta=0.0, zetaI=0.0, friction=0.0, tauNem=1.0,
                   tauIso=1.0, AA=0.03, CC=0.1, LL=0.002, KK=0.06, rho=40.0, xi=0.3, B=0.1,
                   Snem=1.0, config="circle", level=50, conc=1.0, noise=1.0, angle=0,
                   npc=1, **{"relax-steps": 2000, "relax-dt": 1.0, "relax-phi": 1,
                             "relax-Q": 1, "chi-config": "noise", "chi0": 1.0,
                             "chi-noise": 0.0, "chi-length": 0.0, "Dchi": 0.0,
                             "Achi": 0.0, "Ochi": 0.0, "phiswitch": 0.0,
                             "growTogether": 0, "beta": 0.0, "death-rate": 0.0,
                             "death-time": 1, "death-radius": 0.0,
                             "division-rate": 0.1, "division-time": 2, "alpha": 0.001,
                             "phi-critical": 1.2, "division-radius": 3})


def gog_runcard(L: int) -> dict:
    """The runcard at lattice L: the circle's radius scales with L (20 at
    the runcard's 100^2)."""
    p = dict(GOG_RUNCARD)
    p["radius"] = 0.2 * L
    return p


def algorithmic_bytes(model: str, precision: str) -> int:
    """Primary state read once and written once per site-update:
    (9 populations + Qxx + Qyx [+ phi [+ m]]) x 2 x element size."""
    planes = {"lyotropic": 12, "nematic": 11, "go-or-grow": 13}[model]
    return planes * 2 * (4 if precision == "fp32" else 8)


def measured_hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_site(model: str, precision: str):
    """DRAM bytes per site-update of the fused kernel from the committed ncu
    summary (profiles/fused_step_traffic.json), or None."""
    path = os.path.join(ROOT, "profiles", "fused_step_traffic.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d[f"{model}_{precision}"]["dram_bytes_per_site"])
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def synthetic_state(model: str, L: int, seed: int):
    from oracle.oracle import LYOTROPIC, NEMATIC, synthetic_state as st
    return st(LYOTROPIC if model == "lyotropic" else NEMATIC, L, L, seed=seed,
              radius=L / 4)


def pinned_copy(a: np.ndarray):
    import torch
    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
    out = t.numpy()
    out[:] = a.reshape(-1)
    return out, t


def dist_setup(n: int, backend: str | None = None, timeout_s: float = 300.0):
    """Join the process group of a torchrun launch (RANK, WORLD_SIZE,
    LOCAL_RANK, MASTER_ADDR/PORT from the environment). NCCL on GPUs, gloo
    where there are none (the CPU tests of the rank logic)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local


def max_over_ranks(x: float, world: int) -> float:
    """The largest x over all ranks (every rank gets it)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def whole_job_rate(sites_per_rank: int, world: int, steps: int, ms_max: float) -> float:
    """Site-updates per second of the whole job: every rank advances its own
    lattice of sites_per_rank sites by `steps` steps; the job takes the
    slowest rank's time ms_max."""
    return sites_per_rank * world * steps / (ms_max / 1e3)


def cpu_reference_run(model: str, L: int, steps: int, warmup: int, budget_s: float):
    """Time the reference's own build (oracle/_ref) or, if that library is
    absent, the C restatement, on all host cores. Returns (site-updates/s,
    kind, cores, sample description)."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    mcode = O.LYOTROPIC if model == "lyotropic" else O.NEMATIC
    params = LYO_C1 if model == "lyotropic" else NEM_C2
    # the reference keeps ~550 bytes per site; shrink the lattice if the
    # host cannot hold it
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 64 << 30
    Ls = L
    while Ls > 256 and Ls * Ls * 600 > 0.5 * avail:
        Ls //= 2
    st = synthetic_state(model, Ls, seed=1)
    if O.ref_available():
        m = O.RefOracle(mcode, params, Ls, Ls, 0)
        for k, v in st.items():
            m.set(k, v)
        kind, threads = "reference", cores
        run = lambda n: m.time_steps(n, threads)
    else:
        m = O.PortOracle(mcode, params, Ls, Ls, 0)
        for k, v in st.items():
            m.set(k, v)
        kind, threads = "port", 1

        def run(n):
            t0 = time.perf_counter()
            m.step(n)
            return time.perf_counter() - t0
    for _ in range(warmup):
        run(1)
    times = []
    t_start = time.perf_counter()
    for _ in range(steps):
        times.append(run(1))
        if time.perf_counter() - t_start > budget_s:
            break
    per_step = statistics.median(times)
    rate = Ls * Ls / per_step
    sample = (f"{model} {Ls}x{Ls} periodic FP64, {len(times)} timed Step() calls "
              f"after {warmup} warm-up, median step {per_step:.3f} s")
    return rate, kind, threads, sample


def cpu_reference_gog(L: int, steps: int, warmup: int, budget_s: float):
    """The reference's GoOrGrow::Step() (division masks included) on all host
    cores, on the runcard at lattice L. Configure() runs without the dry
    relaxation (it is not part of Step()). Returns (site-updates/s, kind,
    cores, sample description)."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    p = gog_runcard(L)
    p["relax-steps"] = 0
    m = O.RefOracle(O.GO_OR_GROW, p, L, L, 0)
    m.configure(1001)
    # blocks of 6 steps hold the masks' schedule (division every 3rd step,
    # death every 2nd) in its true proportion
    for _ in range(warmup):
        m.time_steps(6, cores)
    times = []
    t_start = time.perf_counter()
    for _ in range(max(1, steps)):
        times.append(m.time_steps(6, cores) / 6)
        if time.perf_counter() - t_start > budget_s:
            break
    per_step = statistics.median(times)
    sample = (f"go-or-grow {L}x{L} periodic FP64 (cases/test/test.dat physics, division masks "
              f"every 3rd step, death masks every 2nd), {len(times)} timed blocks of 6 Step() "
              f"calls after {warmup} warm-up block(s), median {per_step:.4f} s per step")
    return L * L / per_step, "reference", cores, sample


def run_reference(args):
    rank, world, _ = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), 0
    if rank != 0:
        return 0
    if args.model == "go-or-grow":
        rate, kind, cores, sample = cpu_reference_gog(args.size, args.steps,
                                                      max(1, min(args.warmup, 2)), 120.0)
    else:
        rate, kind, cores, sample = cpu_reference_run(args.model, args.size, args.steps,
                                                      max(1, min(args.warmup, 2)), 240.0)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": (f"go-or-grow {args.size}x{args.size} periodic, cases/test/test.dat "
                                f"physics and division settings" if args.model == "go-or-grow"
                                else f"{args.model} {args.size}x{args.size} periodic"),
                   "model": args.model,
                   "LX": args.size, "LY": args.size, "precision": "fp64 (reference build)"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def driver_path() -> str:
    host = os.path.join(ROOT, "mass_hd_b200", "host")
    exe = os.path.join(host, "_build", "mass-gpu")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", host], check=True)
    return exe


def run_driver_gog(L: int, nsteps: int, precision: str, workdir: str) -> float:
    """mass-gpu on the go-or-grow runcard at lattice L; returns the driver's
    own clock around its time loop (seconds)."""
    card = os.path.join(workdir, f"gog_{L}.dat")
    opts = gog_runcard(L)
    opts.update(LX=L, LY=L, nsteps=nsteps, ninfo=max(nsteps, 1), seed=1001, precision=precision)
    with open(card, "w") as fh:
        fh.write("model = go-or-grow\n")
        for k, v in opts.items():
            fh.write(f"{k} = {v}\n")
    r = subprocess.run([driver_path(), card, "--no-write", "-o", workdir], capture_output=True,
                       text=True, timeout=900)
    if r.returncode != 0:
        raise RuntimeError(f"mass-gpu failed: {r.stderr.strip()[-400:]}")
    for line in r.stdout.splitlines():
        if line.startswith("Total run time"):
            return float(line.split(":")[1].split()[0])
    raise RuntimeError("mass-gpu printed no run time")


def gog_state(L: int, seed: int):
    """Runcard-like go-or-grow state: random director (S=1), tanh phi disk of
    radius L/5, m = phi (chi0 = 1, no phenotype noise), rest populations."""
    st = synthetic_state("lyotropic", L, seed)
    x = np.arange(L)[:, None] - L / 2
    y = np.arange(L)[None, :] - L / 2
    r = np.sqrt(x * x + y * y).reshape(-1)
    st["phi"] = 0.5 * (1 - np.tanh((r - 0.2 * L) / 2))
    st["m"] = np.maximum(st["phi"], 0.0)
    return st


def run_ours_gog(args):
    """--model go-or-grow (see the module docstring)."""
    import tempfile

    import torch

    import mass_hd_b200 as M

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    prec = M.FP32 if args.precision == "fp32" else M.FP64
    L = args.size
    sites = L * L
    p = gog_runcard(L)
    st = gog_state(L, seed=1 + rank)
    lat = M.Lattice(M.GO_OR_GROW, p, L, L, 0, prec)
    lat.upload_state(st)
    # the dry relaxation of Configure(), timed on its own
    t0 = time.perf_counter()
    lat.relax_free_energy(int(p["relax-steps"]), p["relax-dt"], True, True)
    relax_s = time.perf_counter() - t0
    # a fixed growth-rate plane: alpha on every 7th site with phi >= 0.5
    phi = lat.get("phi")
    rate = np.where((phi >= 0.5) & (np.arange(sites) % 7 == 0), p["alpha"], 0.0)
    lat.set_phi_source(rate)
    stream = torch.cuda.ExternalStream(lat.stream)
    for _ in range(max(args.warmup, 3)):
        lat.step(1)
    lat.synchronize()
    sampler = ClockSampler(local) if rank == 0 else None
    barrier(world)
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
        time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    # L2: the FP32 state of a 500^2 lattice (~60 MB with all sweep fields)
    # stays in the 126 MB L2 between steps, as it does in a real run
    e0.record(stream)
    for _ in range(args.steps):
        lat.step(1)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    clocks = sampler.stop() if sampler else None
    ms_per_step = ms / args.steps
    value = whole_job_rate(sites, world, args.steps, ms)
    launches = args.steps * lat.launches_per_step
    bps = algorithmic_bytes("go-or-grow", args.precision)
    peak, peak_kind = measured_hbm_peak()
    achieved = sites * bps / (ms_per_step / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "bytes_per_site": bps,
                "traffic": (traffic_per_site("go-or-grow", args.precision) * sites
                            if lat.uses_fused and traffic_per_site("go-or-grow", args.precision)
                            else None),
                "note": ("whole step in one fused launch" if lat.uses_fused else
                         "whole step (one sub-step kernel per predictor and corrector)") +
                        " against the primary state's bytes (13 planes); lattices whose state "
                        "fits in L2 are latency-bound"}
    lat.close()

    # end to end: the driver on the runcard (host masks, Configure excluded),
    # long enough that the start (first supply, first checks) is amortised
    # as in a production run
    n_e2e = max(args.steps, 1000)
    with tempfile.TemporaryDirectory() as d:
        run_driver_gog(L, 3, args.precision, d)          # warm-up (build, first launch)
        t_loop = run_driver_gog(L, n_e2e, args.precision, d)
    t_loop = max_over_ranks(t_loop, world)
    # per step: one uniform (8 B) per phi >= 0.5 site up for every mask
    # drawn (division every 3rd step, death every 2nd), and the 16-byte
    # queue state (draws consumed, error flag) down on the steps that draw
    masks = sum((t % 3 == 0) + (t % 2 == 0) for t in range(n_e2e)) / n_e2e
    redraw = sum(1 for t in range(n_e2e) if t % 3 == 0 or t % 2 == 0) / n_e2e
    cand = int((st["phi"] >= 0.5).sum())
    e2e = {"value": whole_job_rate(sites, world, n_e2e, t_loop * 1e3), "unit": UNIT,
           "h2d_bytes_per_step": int(8 * cand * masks),
           "d2h_bytes_per_step": int(16 * redraw),
           "e2e_steps": n_e2e,
           "note": "mass-gpu driver on the runcard: Step() = host draws of the reference's "
                   "random stream for the masks when due, written into pinned staging and "
                   "queued up to three draws ahead; masks (one cooperative kernel per draw) "
                   "and step on the device; driver clock around the time loop, device "
                   "synchronised at its end"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate_c, kind, cores, sample = cpu_reference_gog(L, 5, 1, 30.0)
        cpu = {"value": rate_c, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f64",
            "data": "synthetic (seeded random director S=1, tanh phi disk R=L/5, m = phi)",
            "config": {"workload": f"go-or-grow {args.precision.upper()} {L}x{L} periodic, "
                                   f"cases/test/test.dat physics and division settings",
                       "model": "go-or-grow", "LX": L, "LY": L, "precision": args.precision,
                       "lattices": world, "relax_2000_steps_s": relax_s,
                       "l2": "state fits in L2 (as in a real run), no flush"},
            "gpu_launches": launches,
            "roofline": roofline,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def fp64_record(model: str, st: dict, L: int, steps: int, warmup: int, world: int) -> dict:
    """The FP64 mode (the reference's double-precision arithmetic, bit for
    bit) on the same seeded workload: device time per step with CUDA events
    on the library's stream, max over ranks, and its roofline against the
    FP64 state's algorithmic bytes. It is the like-for-like counterpart of
    the reference's FP64 OpenMP build."""
    import torch

    import mass_hd_b200 as M
    mcode = M.LYOTROPIC if model == "lyotropic" else M.NEMATIC
    params = LYO_C1 if model == "lyotropic" else NEM_C2
    lat = M.Lattice(mcode, params, L, L, 0, M.FP64)
    lat.upload_state(st)
    stream = torch.cuda.ExternalStream(lat.stream)
    for _ in range(max(warmup, 3)):
        lat.step(1)
    lat.synchronize()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        lat.step(1)
    e1.record(stream)
    e1.synchronize()
    lat.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    launches = steps * lat.launches_per_step
    lat.close()
    ms_per_step = ms / steps
    bps = algorithmic_bytes(model, "fp64")
    peak, peak_kind = measured_hbm_peak()
    achieved = L * L * bps / (ms_per_step / 1e3) / 1e9
    return {"value": whole_job_rate(L * L, world, steps, ms), "unit": UNIT,
            "ms_per_step": ms_per_step, "steps": steps, "dtype": "f64", "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "bytes_per_site": bps},
            "note": "FP64 mode (bit-identical to the reference's double-precision build) on "
                    "the same seeded lattice: one sub-step kernel per predictor and corrector"}


def ensemble_record(steps: int = 200, nruns: int = 96) -> dict:
    """The batched ensemble (configuration 3: 96 lyotropic runs, L from
    {128, 192, 256, 384, 512}, zeta, LL and xi swept, FP32) against the same
    runs stepped one after another through mass_lb_step, on a bounded
    sample of `steps` steps per run (the configuration runs 10k). Both from
    the same seeded states, device-synchronised wall clock; the states must
    come out bit-identical."""
    from mass_hd_b200 import ensemble_case as E
    r = E.compare(nruns, steps)
    return {"runs": nruns, "steps_per_run": steps, "sites": r["sites"],
            "batched_site_updates_per_s": r["batched_site_updates_per_s"],
            "sequential_site_updates_per_s": r["sequential_site_updates_per_s"],
            "speedup": r["speedup"], "bit_identical": r["bit_identical"],
            "chunk_rows": r["ensemble_rows"],
            "note": "one persistent warp-strip launch per step for all runs, replayed from a "
                    "CUDA graph, against mass_lb_step per run with its own autotuned tile; "
                    f"{steps} steps per run as a bounded sample of the 10k-step sweep"}


def surrogate_record() -> dict:
    """The learned surrogate's tensor-core convolutions at the training shape
    (batch 32, 256^2, 64 channels in and out, BF16 operands, FP32
    accumulation): CUDA-event time of each convolution kind with its
    fraction of the measured BF16 peak, and of one training step and one
    forward pass (mass_hd_b200.surrogate_run bench). An auxiliary record:
    if it fails, the line carries the error instead."""
    try:
        from mass_hd_b200 import surrogate_run as R
        r = R.bench()
        rec = {"batch": r["batch"], "size": r["size"], "gflop_per_conv": r["gflop_per_conv"],
               "peak_tflops": r["peak_tflops"], "peak_kind": r["peak_kind"]}
        for k in ("fwd_gelu", "fwd_resid", "dgrad_gelu", "wgrad"):
            rec[k] = {"ms": r[k]["ms"], "tflops": r[k]["tflops"], "frac": r[k]["frac_of_peak"]}
        rec["fwd_gelu"]["mma_thread"] = r["fwd_gelu"].get("mma_thread")
        rec["train_step_ms"] = r["train_step"]["ms"]
        rec["forward_images_per_s"] = r["forward"]["images_per_s"]
        return rec
    except Exception as e:
        return {"error": f"{type(e).__name__}: {e}"}


def run_ours_slab(args):
    """--decomp slab: ONE lattice of size^2 split into x-slabs over the ranks
    (strong scaling), halo rows exchanged before every step over NCCL
    (mass_hd_b200/slab.py). A step is the exchange plus the step of every
    slab; time is the slowest rank's, with CUDA events on its lattice
    stream."""
    import torch

    import mass_hd_b200 as M
    from mass_hd_b200 import slab as S

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    model = args.model
    mcode = M.LYOTROPIC if model == "lyotropic" else M.NEMATIC
    params = LYO_C1 if model == "lyotropic" else NEM_C2
    prec = M.FP32 if args.precision == "fp32" else M.FP64
    L = args.size
    x0, n = S.partition(L, world)[rank]
    sl = S.LatticeSlab(mcode, params, L, L, prec, x0, n)
    sl.upload_global(synthetic_state(model, L, seed=1))
    run = S.SlabRun(sl, S.DistExchange())
    run.step(max(args.warmup, 3))
    sl.synchronize()
    barrier(world)
    stream = torch.cuda.ExternalStream(sl.lat.stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    sl.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    f, p, bad = run.checks()
    if rank == 0:
        line = {
            "metric": METRIC, "value": L * L * args.steps / (ms / 1e3), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else "f64",
            "data": "synthetic (seeded random director S=1, tanh phi disk R=L/4)",
            "config": {"workload": f"{model} {args.precision.upper()} {L}x{L} periodic, one "
                                   f"lattice in x-slabs", "model": model, "LX": L, "LY": L,
                       "precision": args.precision, "parallelism": f"x-slabs over {world} ranks",
                       "halo_bytes_per_step_per_rank": sl.bufs.bytes_per_exchange},
            "gpu_launches": args.steps * sl.lat.launches_per_step,
            "checks": {"fsum": f, "phisum": p, "nonfinite": bad},
        }
        print(json.dumps(line), flush=True)
    sl.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def run_ours(args):
    import torch

    import mass_hd_b200 as M

    if args.model == "go-or-grow":
        return run_ours_gog(args)
    if args.decomp == "slab":
        return run_ours_slab(args)
    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    model = args.model
    mcode = M.LYOTROPIC if model == "lyotropic" else M.NEMATIC
    params = LYO_C1 if model == "lyotropic" else NEM_C2
    prec = M.FP32 if args.precision == "fp32" else M.FP64
    L = args.size
    sites = L * L

    st = synthetic_state(model, L, seed=1 + rank)
    bc = args.bc
    lat = M.Lattice(mcode, params, L, L, bc, prec)
    lat.upload_state(st)
    stream = torch.cuda.ExternalStream(lat.stream)

    # warm-up (also runs the tile autotuner before the first step)
    for _ in range(max(args.warmup, 3)):
        lat.step(1)
    lat.synchronize()

    sampler = ClockSampler(local) if rank == 0 else None
    barrier(world)
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
        time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        lat.step(1)
    e1.record(stream)
    e1.synchronize()
    lat.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    ms = e0.elapsed_time(e1)
    clocks = sampler.stop() if sampler else None
    ms = max_over_ranks(ms, world)
    ms_per_step = ms / args.steps
    value = whole_job_rate(sites, world, args.steps, ms)
    launches = args.steps * lat.launches_per_step

    # roofline of the dominant kernel (one fused launch per step)
    bps = algorithmic_bytes(model, args.precision)
    peak, peak_kind = measured_hbm_peak()
    achieved = sites * bps / (ms_per_step / 1e3) / 1e9
    tps = traffic_per_site(model, args.precision)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "bytes_per_site": bps,
                "traffic": (tps * sites if tps is not None else None)}

    # end-to-end through the C ABI with pinned host buffers
    e2e = None
    host = {}
    keep = []
    for k in (("ff", "QQxx", "QQyx", "phi") if model == "lyotropic" else ("ff", "QQxx", "QQyx")):
        arr, t = pinned_copy(st[k])
        host[k] = arr
        keep.append(t)
    outs = {}
    for k, a in host.items():
        o, t = pinned_copy(np.zeros_like(a))
        outs[k] = o
        keep.append(t)
    h2d = sum(a.nbytes for a in host.values())
    d2h = sum(a.nbytes for a in outs.values())

    def e2e_step():
        lat.upload(host["ff"], host["QQxx"], host["QQyx"], host.get("phi"))
        lat.step(NINFO)
        for k, o in outs.items():
            lat.get_into(k, o)

    e2e_step()     # warm-up
    n_e2e = 3
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        e2e_step()
    dt = time.perf_counter() - t0
    dt_serial = max_over_ranks(dt, world)

    # The same jobs pipelined over NBUF handles: each job's upload and the
    # previous job's download run on their handles' transfer streams while
    # another handle steps, and mass_lb_stream_wait keeps the runs of steps
    # one after another on the device, so each has the whole GPU. Every job
    # still uploads its input from pinned host memory and downloads its
    # result into pinned host memory; the host reuses a handle (and its
    # output buffers) only after synchronizing on it.
    NBUF = 3
    lats = [lat] + [M.Lattice(mcode, params, L, L, bc, prec) for _ in range(NBUF - 1)]
    outsets = [outs]
    for x in lats[1:]:
        if lat.uses_fused:
            x.set_tile(*lat.tile())
        o2 = {}
        for k, a in host.items():
            o, t = pinned_copy(np.zeros_like(a))
            o2[k] = o
            keep.append(t)
        outsets.append(o2)

    def upload_async(x):
        x.upload_async(host["ff"], host["QQxx"], host["QQyx"], host.get("phi"))

    def download_async(i):
        for k, o in outsets[i].items():
            lats[i].get_into_async(k, o)

    def pipeline(njobs):
        for j in range(njobs):
            i = j % NBUF
            x = lats[i]
            if j >= NBUF:
                x.synchronize()                    # job j - NBUF has landed
            upload_async(x)                        # beside the previous job's steps
            if j < NBUF - 1:
                # filling the pipeline: one upload at a time, so that the
                # first job's input is not slowed by the next ones' sharing
                # the host link (the GPU steps the previous job meanwhile)
                x.synchronize()
            if j > 0:
                x.wait_for(lats[(j - 1) % NBUF])   # steps after the previous job's
            x.step(NINFO)
            if j > 0:
                download_async((j - 1) % NBUF)     # beside this job's steps
        download_async((njobs - 1) % NBUF)
        for x in lats:
            x.synchronize()

    pipeline(NBUF)                   # warm-up of every handle
    n_pipe = 16
    barrier(world)
    t0 = time.perf_counter()
    pipeline(n_pipe)
    dt = time.perf_counter() - t0
    dt_pipe = max_over_ranks(dt, world)
    for x in lats[1:]:
        x.close()
    e2e = {"value": whole_job_rate(sites, world, NINFO * n_pipe, dt_pipe * 1e3), "unit": UNIT,
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "steps_per_e2e_step": NINFO, "e2e_steps": n_pipe, "handles": NBUF,
           "serial_value": whole_job_rate(sites, world, NINFO * n_e2e, dt_serial * 1e3),
           "note": "per e2e step (a job): upload the state from pinned host memory, 100 Step() "
                   "calls, download ff/QQxx/QQyx/phi into pinned host memory, through the C "
                   "ABI; jobs rotate over 3 handles with asynchronous transfers and "
                   "mass_lb_stream_wait ordering the runs of steps, the first upload and the "
                   "last download inside the timed region; serial_value: the same jobs one "
                   "after another on one handle with synchronous calls; host wall clock"}
    launches_e2e = n_pipe * NINFO * lat.launches_per_step

    fp64 = None
    if args.precision == "fp32" and not args.no_fp64:
        fp64 = fp64_record(model, st, L, min(args.steps, 20), 3, world)
    ens = None
    if model == "lyotropic" and world == 1 and not args.no_ensemble:
        ens = ensemble_record()
    sg = None
    if model == "lyotropic" and world == 1 and not args.no_surrogate:
        sg = surrogate_record()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, kind, cores, sample = cpu_reference_run(model, L, 5, 1, 20.0)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}

    tile = list(lat.tile()) if lat.uses_fused else None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f64",
            "data": "synthetic (seeded random director S=1, tanh phi disk R=L/4)",
            "config": {"workload": f"{model} {args.precision.upper()} {L}x{L} "
                                   f"{BC_NAMES.get(bc, 'periodic') if bc else 'periodic'}, "
                                   f"256^2-config physics, npc=1",
                       "model": model, "LX": L, "LY": L, "bc": bc,
                       "precision": args.precision,
                       "lattices": world,
                       "parallelism": "independent lattice per GPU" if world > 1 else "single GPU",
                       "l2": f"state {sites * bps // 2 / 1e6:.0f} MB per buffer > 126 MB L2, no flush",
                       "tile": tile},
            "gpu_launches": launches,
            "gpu_launches_e2e": launches_e2e,
            "roofline": roofline,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "fp64": fp64,
            "ensemble": ens,
            "surrogate": sg,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    lat.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=None,
                    help="lattice side (default 4096; 500 for go-or-grow)")
    ap.add_argument("--model", default="lyotropic", choices=["lyotropic", "nematic", "go-or-grow"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--bc", type=int, default=0,
                    help="walls (lyotropic 1/2: free-slip/no-slip channel, 3/4: box; "
                         "nematic 1: channel); the FP64, ensemble and CPU records "
                         "stay periodic and are skipped")
    ap.add_argument("--decomp", default="independent", choices=["independent", "slab"],
                    help="independent: a lattice per rank (weak scaling, default); slab: one "
                         "lattice split into x-slabs over the ranks (strong scaling)")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the batched-ensemble record beside the lyotropic line")
    ap.add_argument("--no-fp64", action="store_true",
                    help="skip the FP64-mode record beside the FP32 line")
    ap.add_argument("--no-surrogate", action="store_true",
                    help="skip the surrogate-convolution record beside the lyotropic line")
    args = ap.parse_args()
    if args.size is None:
        args.size = 500 if args.model == "go-or-grow" else 4096
    if args.impl == "reference":
        return run_reference(args)
    if args.bc:
        args.no_fp64 = args.no_ensemble = args.no_cpu_baseline = args.no_surrogate = True
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
