"""Benchmark: lattice updates per second of the fused D3Q19 fluid+thermal step.

Workload (one "step" = one iteration of the reference driver loop, src/main.c:67-161):
3-D Rayleigh-Benard convection, 256x256x128 lattice (y vertical, no-slip bounce-back
and fixed-temperature walls at y=0 and y=256, periodic in x and z), D3Q19 fluid +
D3Q19 temperature populations, Boussinesq buoyancy, Ra = 1e8, Pr = 1, initial linear
T profile + seeded uniform +-1e-3 noise.  Synthetic data (the reference ships no
dataset); FP32 arithmetic with FP32 population storage by default.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--storage f32|f16|f64]
  python bench.py --impl reference ...   (the reference solver's own CPU build)

With N > 1 the lattice is NX x NY x (N*NZ), one z-slab of NX x NY x NZ per GPU (one
process per GPU; launched under torchrun, or by this script itself when --gpus N > 1 is
given without it), the slab faces exchanged over NCCL after every step (weak scaling),
timed as the max over ranks.  Prints ONE JSON line on rank 0.

At N = 1 the line also carries the reduced-precision error against the FP64 path on the
same input (`error_vs_fp64`: u and T after the timed steps, Nusselt number and kinetic
energy over the configuration's 20,000-step run) and the FP64 path's own throughput
(`fp64`), the end-to-end run's phases (`e2e.breakdown`), and the forced-HIT
configuration (256^3, FP32, 10^6 two-way coupled particles) as its own record
(`hit_particles`: MLUPS, particle updates/s, ms per step; `--no-hit` skips it), the batched
ensemble (`ensemble`: solves/hour against the FP64 path one case at a time) and the served
request stream (`serve`: p50/p99 latency and aggregate MLUPS against the FP64 path serving the
same requests one at a time, step counts scaled by --serve-step-scale).
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "ch4-project_b200"))

NX, NY, NZ = 256, 256, 128
RA, PR = 1e8, 1.0
BYTES_PER_CELL = {  # algorithmic bytes per cell update: read+write of 2 x 19 populations + T_prev r/w
    "f64": 2 * 2 * 19 * 8 + 2 * 8,
    "f32": 2 * 2 * 19 * 4 + 2 * 4,
    "f16": 2 * 2 * 19 * 2 + 2 * 4,
}
WORKLOAD = "rayleigh_benard_256x256x128_d3q19_fluid+thermal"


def rb_params():
    """tau, beta*g from Ra, Pr with a free-fall velocity of 0.05 lattice units."""
    H = float(NY)
    dT = 1.0
    bg = (0.05 ** 2) / (H * dT)            # beta_t * g_y
    nu = (bg * dT * H ** 3 * PR / RA) ** 0.5
    kappa = nu / PR
    return dict(tau_u=0.5 + 3 * nu, tau_t=0.5 + 3 * kappa, beta_t=1.0, gravity_y=bg,
                T_bot=1.0, T_top=0.0, T_ref=0.5)


def make_cfg(storage):
    import ch4b200
    from ch4b200 import abi
    c = ch4b200.default_config()
    c.NX, c.NY, c.NZ = NX, NY, NZ
    c.SX, c.SY, c.SZ = float(NX), float(NY), float(NZ)
    c.flags = abi.flags_of(["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_TEMPERATURE",
                            "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_BC_Y"])
    c.storage = {"f64": abi.STORE_F64, "f32": abi.STORE_F32, "f16": abi.STORE_F16}[storage]
    for k, v in rb_params().items():
        setattr(c, k, v)
    c.nu = (c.tau_u - 0.5 * c.time_dt) / 3.0
    c.kappa = (c.tau_t - 0.5 * c.time_dt) / 3.0
    c.deltaT = c.T_bot - c.T_top
    return c


def initial_state(seed=1234):
    """rho=1, u=0 (p = w) and linear T with uniform +-1e-3 noise (g = w*T), AoS FP64."""
    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
    rng = np.random.default_rng(seed)
    y = (np.arange(NY) + 0.5) / NY
    T = (1.0 - y)[None, :, None] + 1e-3 * (2 * rng.random((NZ, NY, NX)) - 1)
    p = np.broadcast_to(w, (NZ, NY, NX, 19))
    g = T[..., None] * w
    return np.ascontiguousarray(p), np.ascontiguousarray(g)


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([s.strip() for s in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for n, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def measured_peak():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(storage):
    """dram bytes per launch of the step kernel from the committed ncu summary (or None)."""
    path = os.path.join(REPO, "profiles", "lb_step_rb256_%s.json" % storage)
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_launch_full_lattice")
    except Exception:
        return None


def cpu_reference_run(steps, procs=None):
    """Time the reference solver's own CPU build (oracle/_ref/rb) on the host cores.

    The build links the single-rank MPI stand-in, so the reference's domain
    decomposition is reproduced by running one single-rank process per core on its own
    box of the lattice (x and z split, y walls kept whole), all at once: the MPI run
    without its halo exchange, i.e. an upper bound on the MPI build's throughput.
    Returns (MLUPS of the whole lattice, cores, sample description)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    exe = O.ref_binary("rb")
    if not os.path.exists(exe):
        return None, 0, "oracle/_ref/rb/ch4ref not built"
    cores = procs or len(os.sched_getaffinity(0))
    px = pz = 1
    while px * pz * 2 <= cores and (NX // (px * 2) >= 8 or NZ // (pz * 2) >= 8):
        if NX // (px * 2) >= 8 and (px <= pz or NZ // (pz * 2) < 8):
            px *= 2
        else:
            pz *= 2
    nx, nz = NX // px, NZ // pz
    cfg = O.make_config(nx, NY, nz, O.FLAGSETS["rb"], **rb_params())
    runs = []
    for r in range(px * pz):
        tmp = tempfile.mkdtemp(prefix="ch4cpu_")
        O.write_param_in(os.path.join(tmp, "param.in"), cfg, steps)
        runs.append((tmp, subprocess.Popen([exe, str(steps), str(1 + r)], cwd=tmp, stdout=subprocess.DEVNULL,
                                           stderr=subprocess.PIPE, text=True)))
    secs = []
    for tmp, pr in runs:
        _, err = pr.communicate()
        if pr.returncode != 0:
            return None, 0, "reference run failed: " + err[-300:]
        with open(os.path.join(tmp, "timing.json")) as f:
            secs.append(json.load(f)["seconds"])
        shutil.rmtree(tmp, ignore_errors=True)  # the harness also dumps the final state there
    mlups = NX * NY * NZ * steps / max(secs) / 1e6
    return mlups, px * pz, ("%d step(s) of the 256x256x128 lattice as %d concurrent single-rank reference processes "
                            "on %dx%dx%d boxes (x and z split, one per core): the MPI decomposition without its "
                            "halo exchange" % (steps, px * pz, nx, NY, nz))


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_sample_steps():
    """Steps for ~15 s of reference CPU work on all usable cores (2.4 MLUPS per core measured)."""
    cores = len(os.sched_getaffinity(0))
    return int(min(100, max(2, round(15.0 * 2.4e6 * cores / (NX * NY * NZ)))))


def run_reference_arm(args):
    """The reference's own CPU build on all host cores: W untimed warm-up steps in one
    run, then exactly K timed steps of the whole lattice in another (the harness times
    its step loop)."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    if args.warmup > 0:
        cpu_reference_run(args.warmup)
    mlups, cores, sample = cpu_reference_run(args.steps)
    if mlups is None:
        print(json.dumps({"impl": "reference", "unavailable": sample}))
        return 0
    line = {
        "impl": "reference", "metric": "MLUPS", "value": mlups, "unit": "MLUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": NX * NY * NZ / mlups / 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "lattice": [NX, NY, NZ], "Ra": RA, "Pr": PR},
        "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def error_vs_fp64(W, K, window=20000, every=1000):
    """FP32 and FP16-deviation storage against the FP64 path, all three from the same
    initial state: relative L2 of u and T after the bench's W + K steps, and the Nusselt
    number (nuy, src/output.c:332-349,577-579) and kinetic energy (ene) every `every`
    steps up to `window` steps (the configuration's 20,000-step run).  Also the FP64
    path's own throughput (K steps after W, CUDA events on its stream).  The FP64 path is
    bit-identical to the reference's CPU build, so these are errors against the reference."""
    import torch
    import ch4b200
    p0, g0 = initial_state(1234)
    marks = list(range(every, window + 1, every))
    runs = {}
    fp64 = None
    cells = NX * NY * NZ
    for st in ("f64", "f32", "f16"):
        with ch4b200.Simulation(make_cfg(st)) as sim:
            sim.set_pop("p", p0)
            sim.set_pop("g", g0)
            sim.initialize()
            sim.step(W)
            sec = _event_time(sim.stream_handle, lambda: sim.step(K))
            f = sim.fields()
            done = W + K
            nu, ke = [], []
            for m in marks:
                if m > done:
                    sim.step(m - done)
                    done = m
                a = sim.averages()
                nu.append(a["nuy"])
                ke.append(a["ene"])
            runs[st] = {"u": f["u"], "t": f["t"], "nu": np.array(nu), "ke": np.array(ke)}
            del f
            if st == "f64":
                peak, kind = measured_peak()
                ms = sec / K * 1e3
                fp64 = {"value": cells / (ms * 1e-3) / 1e6, "unit": "MLUPS", "ms_per_step": ms, "steps": K,
                        "warmup": W, "bytes_per_cell": BYTES_PER_CELL["f64"],
                        "roofline_frac": BYTES_PER_CELL["f64"] * cells / (ms * 1e-3) / 1e9 / peak,
                        "peak_kind": kind}
    ref = runs["f64"]
    rel = lambda a, b: float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))
    out = {"against": "FP64 path (bit-identical to the reference CPU build)", "lattice": [NX, NY, NZ],
           "fields_after_steps": W + K, "window_steps": [every, window], "every": every,
           "nu_fp64": [float(ref["nu"][0]), float(ref["nu"][-1])],
           "ke_fp64": [float(ref["ke"][0]), float(ref["ke"][-1])]}
    for st in ("f32", "f16"):
        r = runs[st]
        enu = np.abs(r["nu"] - ref["nu"]) / np.abs(ref["nu"])
        eke = np.abs(r["ke"] - ref["ke"]) / np.abs(ref["ke"])
        out[st] = {"u_rel_l2": rel(r["u"], ref["u"]), "t_rel_l2": rel(r["t"], ref["t"]),
                   "nu_rel_err_max": float(enu.max()), "nu_rel_err_final": float(enu[-1]),
                   "nu_window_mean_rel_err": float(abs(r["nu"].mean() - ref["nu"].mean()) / abs(ref["nu"].mean())),
                   "ke_rel_err_max": float(eke.max()), "ke_rel_err_final": float(eke[-1])}
    return out, fp64


def spawn_ranks(args):
    """--gpus N > 1 without a launcher: run this script as N local ranks (one per GPU)
    under torch.distributed.run; rank 0 prints the line."""
    import signal
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    pr = subprocess.Popen(cmd, start_new_session=True)
    try:
        return pr.wait(timeout=1800)
    except subprocess.TimeoutExpired:
        os.killpg(pr.pid, signal.SIGTERM)
        pr.wait(timeout=60)
        return 1


# ---------------------------------------------------------------------------
# other workloads (not the driver's default line)

def _event_time(stream_handle, fn):
    import torch
    st = torch.cuda.ExternalStream(stream_handle)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    fn()
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) * 1e-3


def bench_ensemble(args):
    """512 independent quasi-2D Rayleigh-Benard cells (NZ = 1) of log-uniform sizes
    64x64 .. 512x256 and Ra in [1e5, 1e8], Pr = 1, advanced together.  Throughput as
    solves/hour for S steps per solve, against the plain FP64 path run one case at a
    time (per-case step time fitted as a + b*cells on a sample).  Accuracy on the same
    sample: Nusselt number averaged over steps [S/2, S] (every 500 steps), ensemble
    against FP64, relative error."""
    import math
    import torch
    import ch4b200
    from ch4b200 import abi
    torch.cuda.set_device(0)
    rng = np.random.default_rng(4)
    S = args.steps_per_solve
    every = 500
    storage = {"f32": abi.STORE_F32, "f16": abi.STORE_F16}.get(args.storage, abi.STORE_F32)
    cases = []
    for i in range(args.cases):
        nx = int(round(math.exp(rng.uniform(math.log(64), math.log(512)))))
        ny = int(round(math.exp(rng.uniform(math.log(64), math.log(256)))))
        ra = math.exp(rng.uniform(math.log(1e5), math.log(1e8)))
        cases.append((nx, ny, ra))
    sample = sorted(int(i) for i in rng.choice(len(cases), size=min(args.sample, len(cases)), replace=False))

    def cfg_of(nx, ny, ra, st):
        c = ch4b200.default_config()
        c.NX, c.NY, c.NZ = nx, ny, 1
        c.SX, c.SY, c.SZ = float(nx), float(ny), 1.0
        c.flags = abi.flags_of(["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_TEMPERATURE",
                                "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_BC_Y"])
        c.storage = st
        bg = 0.05 ** 2 / ny
        nu = (bg * ny ** 3 / ra) ** 0.5
        c.tau_u = c.tau_t = 0.5 + 3 * nu
        c.beta_t, c.gravity_y, c.T_bot, c.T_top, c.T_ref = 1.0, bg, 1.0, 0.0, 0.5
        c.nu = (c.tau_u - 0.5) / 3.0
        c.kappa = (c.tau_t - 0.5) / 3.0
        c.deltaT = 1.0
        return c

    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)

    def state_of(i, nx, ny):
        r = np.random.default_rng(100 + i)
        y = (np.arange(ny) + 0.5) / ny
        T = (1.0 - y)[None, :, None] + 1e-3 * (2 * r.random((1, ny, nx)) - 1)
        return np.ascontiguousarray(np.broadcast_to(w, (1, ny, nx, 19))), np.ascontiguousarray(T[..., None] * w)

    ens = ch4b200.Ensemble(storage)
    slots = []
    cells = 0
    for i, (nx, ny, ra) in enumerate(cases):
        s = ens.add(cfg_of(nx, ny, ra, storage))
        p0, g0 = state_of(i, nx, ny)
        ens.set_pop(s, "p", p0)
        ens.set_pop(s, "g", g0)
        ens.initialize(s)
        slots.append(s)
        cells += nx * ny
    block, rows = ens.tune()
    ens.step(100)
    ens.synchronize()
    K = args.steps
    t_step = _event_time(ens.stream_handle, lambda: ens.step(K)) / K
    solves_h = len(cases) * 3600.0 / (S * t_step)
    if args.throughput_only:  # tuning runs: the timed ensemble step alone
        ens.close()
        print(json.dumps({"metric": "ensemble solves/hour", "value": solves_h, "unit": "solves/h",
                          "ensemble_mlups": cells / t_step / 1e6, "tile_block": block, "tile_rows": rows,
                          "throughput_only": True}))
        return 0
    if getattr(args, "record_only", False):
        # throughput against the FP64 path's per-case step time (a + b cells, fitted on the
        # sample); the accuracy study is the standalone line's
        ens.close()
        xs, ts = [], []
        for i in sample:
            nx, ny, ra = cases[i]
            p0, g0 = state_of(i, nx, ny)
            with ch4b200.Simulation(cfg_of(nx, ny, ra, abi.STORE_F64)) as sim:
                sim.set_pop("p", p0)
                sim.set_pop("g", g0)
                sim.initialize()
                sim.step(20)
                sim.synchronize()
                ts.append(_event_time(sim.stream_handle, lambda: sim.step(100)) / 100)
            xs.append(nx * ny)
        a, b = np.polyfit(np.array(xs, float), np.array(ts), 1)[::-1]
        t64 = sum(max(a + b * nx * ny, min(ts)) for nx, ny, _ in cases)
        solves_h64 = 3600.0 * len(cases) / (S * t64)
        peak, kind = measured_peak()
        bpc = BYTES_PER_CELL.get(args.storage, BYTES_PER_CELL["f32"])
        return {"metric": "ensemble solves/hour", "value": solves_h, "unit": "solves/h",
                "config": {"workload": "ensemble_%d_quasi2d_rayleigh_benard" % len(cases), "cells_total": cells,
                           "steps_per_solve": S, "storage": args.storage, "tile_block": block, "tile_rows": rows},
                "ensemble_ms_per_step": t_step * 1e3, "ensemble_mlups": cells / t_step / 1e6,
                "roofline_frac": bpc * cells / t_step / 1e9 / peak, "peak_kind": kind,
                "fp64_one_at_a_time": {"solves_per_hour": solves_h64, "fit_seconds_per_step": [a, b],
                                       "sample_cases": len(sample)},
                "speedup_vs_fp64_one_at_a_time": solves_h / solves_h64,
                "accuracy": "bench.py --workload ensemble (Nusselt and kinetic energy against FP64)"}
    # the rest of the solve: T fields of the sampled cases at the short horizon, then Nu over [S/2, S]
    done = 100 + K
    nu_ens = {i: [] for i in sample}
    t_ens = {}
    marks = sorted({min(S, args.short_horizon)} | set(range(every, S + 1, every)))
    for target in marks:
        if target <= done:
            continue
        ens.step(target - done)
        done = target
        if done == args.short_horizon:
            for i in sample:
                t_ens[i] = (ens.fields(slots[i])["t"], ens.averages(slots[i]))
        if done >= S // 2 and done % every == 0:
            for i in sample:
                nu_ens[i].append(ens.averages(slots[i])["nuy"])
    ens.close()
    # plain FP64, one case at a time, on the sample
    xs, ts, errs, nus, terrs, per_case, short_nu, short_ke = [], [], [], [], [], [], [], []
    for i in sample:
        nx, ny, ra = cases[i]
        p0, g0 = state_of(i, nx, ny)
        with ch4b200.Simulation(cfg_of(nx, ny, ra, abi.STORE_F64)) as sim:
            sim.set_pop("p", p0)
            sim.set_pop("g", g0)
            sim.initialize()
            sim.step(20)
            sim.synchronize()
            t = _event_time(sim.stream_handle, lambda: sim.step(100))
            d, nu64 = 120, []
            for target in marks:
                if target <= d:
                    continue
                sim.step(target - d)
                d = target
                if d == args.short_horizon and i in t_ens:
                    t64, a64 = sim.fields()["t"], sim.averages()
                    te, ae = t_ens[i]
                    terrs.append(float(np.linalg.norm(te - t64) / np.linalg.norm(t64)))
                    short_nu.append(abs(ae["nuy"] - a64["nuy"]) / abs(a64["nuy"]))
                    short_ke.append(abs(ae["ene"] - a64["ene"]) / abs(a64["ene"]))
                if d >= S // 2 and d % every == 0:
                    nu64.append(sim.averages()["nuy"])
        xs.append(nx * ny)
        ts.append(t / 100)
        m64, m32 = float(np.mean(nu64)), float(np.mean(nu_ens[i]))
        nus.append(m64)
        errs.append(abs(m32 - m64) / abs(m64))
        per_case.append({"NX": nx, "NY": ny, "Ra": float("%.4g" % ra), "nu_fp64": round(m64, 5), "nu": round(m32, 5),
                         "t_rel_l2_at_short_horizon": float("%.3g" % terrs[-1]) if terrs else None})
    # steady laminar cells, where FP32 and FP64 can be compared at the end of the run:
    # 32x16 cells at Ra 3e3 - 1e4, many thermal diffusion times (H^2 / kappa = 17 k - 32 k steps)
    lam = [(32, 16, float(ra)) for ra in np.geomspace(3e3, 1e4, args.laminar_cases)]
    lam_ens = ch4b200.Ensemble(storage)
    lam_slots = []
    for i, (nx, ny, ra) in enumerate(lam):
        sl = lam_ens.add(cfg_of(nx, ny, ra, storage))
        p0, g0 = state_of(1000 + i, nx, ny)
        lam_ens.set_pop(sl, "p", p0)
        lam_ens.set_pop(sl, "g", g0)
        lam_ens.initialize(sl)
        lam_slots.append(sl)
    lam_ens.step(args.laminar_steps)
    lam_ens.synchronize()
    lam_err_nu, lam_err_ke, lam_nu = [], [], []
    for i, ((nx, ny, ra), sl) in enumerate(zip(lam, lam_slots)):
        a32 = lam_ens.averages(sl)
        p0, g0 = state_of(1000 + i, nx, ny)
        with ch4b200.Simulation(cfg_of(nx, ny, ra, abi.STORE_F64)) as sim:
            sim.set_pop("p", p0)
            sim.set_pop("g", g0)
            sim.initialize()
            sim.step(args.laminar_steps)
            a64 = sim.averages()
        lam_nu.append(round(a64["nuy"], 6))
        lam_err_nu.append(abs(a32["nuy"] - a64["nuy"]) / abs(a64["nuy"]))
        lam_err_ke.append(abs(a32["ene"] - a64["ene"]) / abs(a64["ene"]))
    lam_ens.close()
    a, b = np.polyfit(np.array(xs, float), np.array(ts), 1)[::-1]
    t64 = sum(max(a + b * nx * ny, min(ts)) for nx, ny, _ in cases)
    solves_h64 = 3600.0 * len(cases) / (S * t64)
    st_name = "f16" if storage == abi.STORE_F16 else "f32"
    print(json.dumps({
        "metric": "ensemble solves/hour", "value": solves_h, "unit": "solves/h", "n_gpus": 1, "steps": K,
        "higher_is_better": True, "dtype": "f32 (%s storage)" % st_name, "data": "synthetic",
        "config": {"workload": "ensemble_%d_quasi2d_rayleigh_benard" % len(cases), "cells_total": cells,
                   "steps_per_solve": S, "tile_block": block, "tile_rows": rows, "graph_block_steps": 100,
                   "storage": st_name},
        "ensemble_ms_per_step": t_step * 1e3, "ensemble_mlups": cells / t_step / 1e6,
        "fp64_one_at_a_time": {"solves_per_hour": solves_h64, "fit_seconds_per_step": [a, b],
                               "sample_cases": len(sample)},
        "speedup_vs_fp64_one_at_a_time": solves_h / solves_h64,
        "nusselt_vs_fp64": {"window": [S // 2, S], "every": every, "cases": len(errs),
                            "rel_error_median": float(np.median(errs)), "rel_error_max": float(np.max(errs)),
                            "nu_fp64_range": [float(min(nus)), float(max(nus))]},
        "t_field_vs_fp64": {"after_steps": args.short_horizon, "rel_l2_median": float(np.median(terrs)),
                            "rel_l2_max": float(np.max(terrs))},
        "nusselt_and_kinetic_energy_vs_fp64": {"after_steps": args.short_horizon,
                                               "nu_rel_error_max": float(np.max(short_nu)),
                                               "ke_rel_error_max": float(np.max(short_ke)),
                                               "nu_rel_error_median": float(np.median(short_nu)),
                                               "ke_rel_error_median": float(np.median(short_ke))},
        "steady_laminar_vs_fp64": {"cases": len(lam), "lattice": [32, 16], "Ra": [3e3, 1e4],
                                   "steps": args.laminar_steps, "nu_fp64": lam_nu,
                                   "nu_rel_error_max": float(max(lam_err_nu)),
                                   "ke_rel_error_max": float(max(lam_err_ke))},
        "sample": per_case,
    }))
    return 0


def bench_serve(args, record_only=False):
    """Poisson request stream (20/s) of Kolmogorov and Rayleigh-Benard cubes, half with
    LES (C_s 0.17) and 1e4-1e5 tracers; step counts log-uniform in [500, 20000] times
    --step-scale.  p50/p99 latency and aggregate MLUPS against the FP64 path serving the
    same requests one at a time."""
    import copy
    import torch
    from ch4b200 import abi, serve
    torch.cuda.set_device(0)
    reqs = serve.make_requests(args.requests, rate=20.0, step_scale=args.step_scale)
    work = sum(r.cells * r.steps for r in reqs)
    for r in reqs:  # requests arrive with their initial state: build them outside both timed runs
        serve.request_state(r)
        serve.request_particles(r)
    runs = {}
    policies = (("all_in_flight", None), ("cells_in_flight_%d" % args.cells_in_flight, args.cells_in_flight))
    if record_only:  # the default bench line's record: the capped policy alone
        policies = policies[1:]
    for name, cap in policies:
        srv = serve.Server(abi.STORE_F32, block=100, cells_in_flight=cap)
        t0 = time.perf_counter()
        done = srv.run(copy.deepcopy(reqs))
        span = time.perf_counter() - t0
        lat = np.array([r.latency for r in done])
        runs[name] = {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                      "makespan_s": span, "mlups": work / span / 1e6}
    best = min(runs, key=lambda k: runs[k]["p50_s"])
    base = serve.serve_fp64_one_at_a_time(copy.deepcopy(reqs))
    lat64 = np.array([r.latency for r in base])
    span64 = max(r.finished for r in base) - min(r.arrival for r in base)
    rec = {
        "metric": "served p50/p99 latency and aggregate MLUPS", "value": runs[best]["mlups"], "unit": "MLUPS",
        "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic", "policy": best,
        "config": {"workload": "served_stream", "requests": len(reqs), "rate_per_s": 20.0,
                   "sizes": [32, 64, 96, 128, 192], "steps": "log-uniform [500,20000] x %g" % args.step_scale,
                   "les_fraction": 0.5, "block_steps": 100},
        "p50_s": runs[best]["p50_s"], "p99_s": runs[best]["p99_s"], "makespan_s": runs[best]["makespan_s"],
        "policies": runs,
        "fp64_one_at_a_time": {"p50_s": float(np.percentile(lat64, 50)), "p99_s": float(np.percentile(lat64, 99)),
                               "mlups": work / span64 / 1e6},
        "throughput_vs_fp64_one_at_a_time": runs[best]["mlups"] / (work / span64 / 1e6),
    }
    if record_only:
        return rec
    print(json.dumps(rec))
    return 0


TAU_ETA = 10.0  # Kolmogorov time in steps that sets tau_p = St * tau_eta


def hit_particles_run(n, npart, steps, warmup, storage="f32"):
    """Forced HIT n^3 with npart two-way coupled particles: tracers and Stokes particles with
    added mass, beta in {0, 1, 3} x St in {0.1, 1, 5} with tau_p = St * 10 steps, except that
    the bubbles (beta = 3) stop at St = 2: at St = 5 their radius sqrt(3 nu beta tau_p) is
    1.22 cells and the explicit two-way deposit diverges within ~20 steps (the FP64 oracle
    shows the same).  Trilinear interpolation with gradients, two-way momentum deposit.
    Device-resident timing of `steps` steps (CUDA events on the handle's stream)."""
    import torch
    import ch4b200
    from ch4b200 import abi
    torch.cuda.set_device(0)
    c = ch4b200.default_config()
    c.NX = c.NY = c.NZ = n
    c.SX = c.SY = c.SZ = float(n)
    c.flags = abi.flags_of(["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LAGRANGE", "LAGRANGE_WRAP",
                            "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_TWOWAY",
                            "LAGRANGE_TWOWAY_MOMENTUM"])
    c.storage = {"f64": abi.STORE_F64, "f16": abi.STORE_F16}.get(storage, abi.STORE_F32)
    c.tau_u = 0.51
    c.nu = (c.tau_u - 0.5) / 3.0
    c.Amp_x = c.Amp_y = c.Amp_z = 5e-6
    c.time_dt_lagr_factor = 1.0
    c.seed = 11
    rng = np.random.default_rng(5)
    # one record of 43 doubles per particle (name, tau_drag, beta_coeff, x, y, z, ...), at rest;
    # kinds cycle over tracers and the 9 (St, beta) Stokes classes
    rec = np.zeros((npart, len(abi.Particle._fields_)))
    rec[:, 0] = np.arange(npart)
    rec[:, 3:6] = rng.random((npart, 3)) * n
    kind = np.arange(npart) % 10
    stokes = kind > 0
    beta = np.array([0.0, 1.0, 3.0])[(kind[stokes] - 1) % 3]
    st = np.array([0.1, 1.0, 5.0])[(kind[stokes] - 1) // 3]
    st = np.where(beta == 3.0, np.minimum(st, 2.0), st)
    rec[stokes, 2] = beta
    rec[stokes, 1] = st * TAU_ETA
    parts = (abi.Particle * npart).from_buffer(rec)
    with ch4b200.Simulation(c) as sim:
        sim.set_particles(parts)
        sim.initialize()
        sim.step(max(3, warmup))
        sim.synchronize()
        sec = _event_time(sim.stream_handle, lambda: sim.step(steps))
        f = sim.fields()
    cells = n ** 3
    ms_step = sec / steps * 1e3
    peak, peak_kind = measured_peak()
    # lb_step's own bytes per cell: populations read + written, the two-way force read
    # (the hydro pass for the interpolation and the particle kernels come on top)
    bpc = 2 * 19 * {"f64": 8, "f16": 2}.get(storage, 4) + 12 + 24
    achieved = bpc * cells / (ms_step * 1e-3) / 1e9
    return {
        "metric": "MLUPS and particle updates/s", "value": cells * steps / sec / 1e6, "unit": "MLUPS",
        "particles_per_s": npart * steps / sec, "n_gpus": 1, "steps": steps, "warmup": max(3, warmup),
        "ms_per_step": ms_step, "higher_is_better": True, "dtype": storage, "data": "synthetic",
        "config": {"workload": "hit_%d3_particles_%d_twoway" % (n, npart), "tau_eta_steps": TAU_ETA,
                   "classes": "tracers + beta{0,1,3} x St{0.1,1,5}, bubbles St<=2"},
        "roofline": {"bound": "hbm", "bytes_per_cell": bpc, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "basis": "whole step time against the lattice step's own bytes per cell"},
        "finite": bool(np.isfinite(f["u"]).all()),
    }


def bench_hit_particles(args):
    """The HIT + particles configuration on its own line (MLUPS and particle updates/s)."""
    print(json.dumps(hit_particles_run(args.hit_size, args.particles, args.steps, args.warmup, args.storage)))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "f64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--zslab", action="store_true", help="run the z-slab path (face exchange every step) at N = 1 too")
    ap.add_argument("--lattice", default=None, help="NX,NY,NZ override (profiling runs on a smaller case)")
    ap.add_argument("--workload", default="rb", choices=["rb", "ensemble", "serve", "hit_particles"])
    ap.add_argument("--cases", type=int, default=512)
    ap.add_argument("--steps-per-solve", type=int, default=20000)
    ap.add_argument("--sample", type=int, default=16)
    ap.add_argument("--short-horizon", type=int, default=2000)
    ap.add_argument("--laminar-cases", type=int, default=8)
    ap.add_argument("--throughput-only", action="store_true")
    ap.add_argument("--laminar-steps", type=int, default=200000)
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--cells-in-flight", type=int, default=8 << 20)
    ap.add_argument("--step-scale", type=float, default=1.0)
    ap.add_argument("--hit-size", type=int, default=256)
    ap.add_argument("--particles", type=int, default=1000000)
    ap.add_argument("--no-error", action="store_true", help="skip the FP32/FP16 error study against FP64")
    ap.add_argument("--error-window", type=int, default=20000)
    ap.add_argument("--error-every", type=int, default=1000)
    ap.add_argument("--no-hit", action="store_true", help="skip the HIT + particles sub-record")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the ensemble sub-record")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-stream sub-record")
    ap.add_argument("--serve-step-scale", type=float, default=1.0,
                    help="step counts of the served-stream sub-record, times the configuration's")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and args.impl == "ours":
        return spawn_ranks(args)
    if args.workload == "ensemble":
        return bench_ensemble(args)
    if args.workload == "serve":
        return bench_serve(args)
    if args.workload == "hit_particles":
        return bench_hit_particles(args)
    if args.lattice:
        global NX, NY, NZ
        NX, NY, NZ = (int(v) for v in args.lattice.split(","))
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import ch4b200
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    W = max(3, args.warmup)
    K = args.steps
    cfg = make_cfg(args.storage)
    p0, g0 = initial_state(1234 + rank)
    cells = NX * NY * NZ
    # N > 1: one lattice NX x NY x (N*NZ), a z-slab of NX x NY x NZ per GPU, the slab
    # faces exchanged over NCCL after every step (weak scaling)
    slab_mode = world > 1 or args.zslab
    if slab_mode:
        from ch4b200 import slab as slabmod
        gcfg = make_cfg(args.storage)
        gcfg.NZ = NZ * world
        gcfg.SZ = float(NZ * world)

    def new_sim():
        if slab_mode:
            s = slabmod.Slab(gcfg, rank * NZ, NZ)
            # the faces move inside ch4_step, overlapped with the slab's interior planes
            # (one rank: the slab's own faces, a device copy on the handle's second stream)
            s.use_process_group(rank, world)
            return s.sim, (lambda n: s.step(n, rank, world))
        s = ch4b200.Simulation(cfg)
        return s, s.step

    # ---- device-resident timing --------------------------------------------
    sim, run = new_sim()
    sim.set_pop("p", p0)
    sim.set_pop("g", g0)
    sim.initialize()
    stream = torch.cuda.ExternalStream(sim.stream_handle)
    run(W)
    sim.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        run(K)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
        torch.distributed.barrier()
    ms_step = ms / K
    value = world * cells * K / (ms * 1e-3) / 1e6
    peak, peak_kind = measured_peak()
    achieved = BYTES_PER_CELL[args.storage] * cells / (ms_step * 1e-3) / 1e9
    fields = sim.fields()
    finite = bool(np.isfinite(fields["u"]).all() and np.isfinite(fields["t"]).all())
    sim.close()

    # ---- end to end through the C ABI with host buffers ---------------------
    e2e = None
    if not args.no_e2e:
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ph = {}
        t0 = time.perf_counter()
        s2, run2 = new_sim()
        with s2:
            t1 = time.perf_counter()
            s2.set_pop("p", p0)
            s2.set_pop("g", g0)
            t2 = time.perf_counter()
            s2.initialize()
            t3 = time.perf_counter()
            run2(K)
            s2.synchronize()
            t4 = time.perf_counter()
            f2 = s2.fields()
            t5 = time.perf_counter()
        t6 = time.perf_counter()
        sec = t6 - t0
        if world > 1:
            t = torch.tensor([sec], device="cuda")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            sec = float(t.item())
        # bytes over the bus: the library rounds the caller's FP64 populations to the
        # arithmetic type on the host before the copy (FP32 forms: 4 bytes per value)
        wire = 8 if args.storage == "f64" else 4
        h2d = 2 * p0.size * wire
        d2h = 5 * cells * 8  # dens, u(3), t of ch4_get_fields (no scalar set: s is zero-filled on the host)
        ph = {"create_s": t1 - t0, "upload_s": t2 - t1, "upload_gbps": h2d / (t2 - t1) / 1e9,
              "initialize_s": t3 - t2, "steps_s": t4 - t3, "download_s": t5 - t4,
              "download_gbps": d2h / (t5 - t4) / 1e9, "close_s": t6 - t5,
              "caller_bytes_uploaded": 2 * p0.nbytes}
        e2e = {"value": world * cells * K / sec / 1e6, "unit": "MLUPS",
               "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
               "includes": "create + AoS FP64 upload of p,g (rounded to the storage's arithmetic type on the host) "
                           "+ initialize + K steps + hydro-field download",
               "breakdown": ph}
        del f2

    err = fp64 = None
    if world == 1 and not args.no_error:
        err, fp64 = error_vs_fp64(W, K, args.error_window, args.error_every)

    # the third configuration (forced HIT 256^3 + 10^6 two-way particles) beside the headline
    hit = None
    if world == 1 and not args.no_hit:
        hit = hit_particles_run(args.hit_size, args.particles, max(K, 20), W)
    # the batched ensemble (fourth configuration) and the served stream (fifth, step counts
    # scaled by --serve-step-scale) against the FP64 path one case at a time
    ens_rec = srv_rec = None
    if world == 1 and not args.no_ensemble:
        import copy as _copy
        ea = _copy.copy(args)
        ea.record_only, ea.storage, ea.steps = True, "f32", 100
        ens_rec = bench_ensemble(ea)
    if world == 1 and not args.no_serve:
        import copy as _copy
        sa = _copy.copy(args)
        sa.step_scale = args.serve_step_scale
        srv_rec = bench_serve(sa, record_only=True)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        mlups, cores, sample = cpu_reference_run(cpu_sample_steps())
        cpu = {"value": mlups, "unit": "MLUPS", "cores": cores, "kind": "reference", "sample": sample}

    if rank == 0:
        line = {
            "metric": "MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"f32": "f32", "f16": "f32 (f16 storage)", "f64": "f64"}[args.storage], "data": "synthetic",
            "config": {"workload": WORKLOAD, "lattice": [NX, NY, NZ * world], "lattice_per_gpu": [NX, NY, NZ],
                       "Ra": RA, "Pr": PR,
                       "storage": args.storage, "l2": "inputs larger than L2 (%.2f GB of populations)" %
                       (2 * 19 * cells * {"f64": 8, "f32": 4, "f16": 2}[args.storage] / 1e9),
                       "parallelism": "zslab%d" % world if slab_mode else "single"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": ncu_traffic(args.storage),
                         "bytes_per_cell": BYTES_PER_CELL[args.storage], "kernel": "lb_step_kernel"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            # lb_step (slabs: face planes + interior, halo pack and unpack per step)
            "gpu_launches": K * (4 if slab_mode else 1),
            "clocks": clk.summary(),
            "finite": finite,
            "error_vs_fp64": err,
            "fp64": fp64,
            "hit_particles": hit,
            "ensemble": ens_rec,
            "serve": srv_rec,
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
