"""Continuous-batching server for simulation requests (parameter sweeps).

Requests (Kolmogorov flow or Rayleigh-Benard convection, a cubic lattice, a step
count, optionally Smagorinsky LES and tracer particles) arrive over time.  The server
keeps every admitted simulation resident on the device and advances all of them
together in blocks of steps:

* plain requests become slots of a shared ensemble (one work-queue launch per step
  for all of them, ch4_ensemble_*), one ensemble per population-set layout;
* LES and particle requests run on their own handle and CUDA stream
  (ch4_create/ch4_step), overlapping with the ensembles on the device;
* while a block runs, waiting requests are admitted (built and uploaded) in arrival order
  while the device-memory budget allows and,
  with `cells_in_flight`, while the admitted lattices stay under that many cells (a
  request is always admitted when nothing runs): small requests then batch together
  while large ones do not share the device with a long queue, which shortens the
  median latency without leaving the device idle; after a block finished requests are
  retired (their memory freed).

A request's result is the same alone and in the mix: ensemble slots advance
bit-for-bit as they would alone, and dedicated handles are independent.
"""
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi
from . import Ensemble, Simulation, default_config, device_bytes, ensemble_slot_bytes, CH4Error

W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


@dataclass
class Request:
    rid: int
    kind: str          # "kolmogorov" or "rb"
    size: int          # cube edge
    steps: int
    les: bool = False
    tracers: int = 0
    arrival: float = 0.0
    # filled by the server
    admitted: float = None
    finished: float = None
    result: dict = field(default_factory=dict)

    @property
    def cells(self):
        return self.size ** 3

    @property
    def latency(self):
        return None if self.finished is None else self.finished - self.arrival


def request_config(req, storage):
    """Configuration of a request: Kolmogorov (periodic, F_x = 1e-5 sin(2 pi y / L)) at
    tau 0.6, or Rayleigh-Benard (y walls, Ra 1e6, Pr 1); LES with C_s = 0.17."""
    n = req.size
    flags = ["LB_FLUID", "LB_FLUID_FORCING"]
    c = default_config()
    c.NX = c.NY = c.NZ = n
    c.SX = c.SY = c.SZ = float(n)
    c.time_dt = 1.0
    c.storage = storage
    c.C_smag = 0.17
    c.time_dt_lagr_factor = 1.0
    c.seed = 1 + req.rid
    if req.kind == "kolmogorov":
        flags += ["LB_FLUID_FORCING_KOLMOGOROV"]
        c.tau_u = 0.6
        nu = (c.tau_u - 0.5) / 3.0
        c.Amp_x = 1e-5 / (nu * (2 * 3.14159265359 / n) ** 2)
    else:
        flags += ["LB_FLUID_BC_Y", "LB_TEMPERATURE", "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_BC_Y"]
        bg = 0.05 ** 2 / n
        nu = (bg * n ** 3 / 1e6) ** 0.5
        c.tau_u = c.tau_t = 0.5 + 3 * nu
        c.beta_t, c.gravity_y = 1.0, bg
        c.T_bot, c.T_top, c.T_ref = 1.0, 0.0, 0.5
    if req.les:
        flags += ["LB_FLUID_LES"]
    if req.tracers and req.kind == "kolmogorov":
        flags += ["LAGRANGE", "LAGRANGE_WRAP"]
    c.flags = abi.flags_of(flags)
    c.nu = (c.tau_u - 0.5 * c.time_dt) / 3.0
    c.kappa = (c.tau_t - 0.5 * c.time_dt) / 3.0
    c.deltaT = c.T_bot - c.T_top
    return c


_STATES = {}


def request_state(req):
    """Seeded initial populations: rest + uniform velocity noise 1e-4 (Kolmogorov), or
    the linear conductive temperature profile + noise 1e-3 (Rayleigh-Benard).  One
    state per (kind, size), built once and kept: a request arrives with its initial
    state, so building it is not part of serving it."""
    key = (req.kind, req.size)
    if key not in _STATES:
        _STATES[key] = _make_state(req.kind, req.size)
    return _STATES[key]


def _make_state(kind, n):
    rng = np.random.default_rng(1000 + 7 * n + (kind == "rb"))
    u = 1e-4 * (2 * rng.random((n, n, n, 3)) - 1)
    cx = np.array([0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, -1, 1, -1, 0, 0, 0, 0])
    cy = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1])
    cz = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, -1, 1, -1])
    cu = u[..., 0:1] * cx + u[..., 1:2] * cy + u[..., 2:3] * cz
    u2 = (u ** 2).sum(-1, keepdims=True)
    p = W * (1 + 3 * cu + 4.5 * cu ** 2 - 1.5 * u2)
    state = {"p": np.ascontiguousarray(p)}
    if kind == "rb":
        y = (np.arange(n) + 0.5) / n
        T = (1.0 - y)[None, :, None] + 1e-3 * (2 * rng.random((n, n, n)) - 1)
        state["g"] = np.ascontiguousarray(T[..., None] * W)
    return state


_PARTICLES = {}


def request_particles(req):
    """Seeded tracer records of a request (built once and kept, like the state)."""
    if not (req.tracers and req.kind == "kolmogorov"):
        return None
    key = (req.rid, req.size, req.tracers)
    if key not in _PARTICLES:
        _PARTICLES[key] = _make_particles(req)
    return _PARTICLES[key]


def _make_particles(req):
    rng = np.random.default_rng(2000 + req.rid)
    rec = np.zeros((req.tracers, len(abi.Particle._fields_)))  # name, tau_drag = 0 (tracer), beta, x, y, z, ...
    rec[:, 0] = np.arange(req.tracers)
    rec[:, 3:6] = rng.random((req.tracers, 3)) * req.size
    return (abi.Particle * req.tracers).from_buffer(rec)


def make_requests(n, rate=20.0, sizes=(32, 64, 96, 128, 192), steps=(500, 20000), step_scale=1.0, seed=7):
    """Poisson arrivals; kinds and LES alternate at random; steps log-uniform."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        les = bool(rng.random() < 0.5)
        kind = "kolmogorov" if rng.random() < 0.5 else "rb"
        st = int(round(math.exp(rng.uniform(math.log(steps[0]), math.log(steps[1]))) * step_scale))
        tracers = int(math.exp(rng.uniform(math.log(1e4), math.log(1e5)))) if les else 0
        out.append(Request(i, kind, int(rng.choice(sizes)), max(1, st), les, tracers, t))
    return out


class Server:
    """Admits, advances and retires requests; every simulation stays resident on the device."""

    def __init__(self, storage=abi.STORE_F32, budget_bytes=None, block=100, cells_in_flight=None):
        import torch  # noqa: F401  (CUDA context shared with the library)
        self.storage = storage
        self.block = block
        if budget_bytes is None:
            import torch
            free, _ = torch.cuda.mem_get_info()
            budget_bytes = int(0.8 * free)
        self.budget = budget_bytes
        self.cells_in_flight = cells_in_flight
        self.used = 0
        self.ensembles = {}
        self.active = []  # (req, kind, handle, slot, bytes, remaining)

    def _bytes(self, req, cfg):
        if self._dedicated(req):
            return device_bytes(cfg) + (req.tracers * 45 * 8 if req.tracers else 0)
        return ensemble_slot_bytes(cfg, self.storage)

    @staticmethod
    def _dedicated(req):
        return req.les or (req.tracers > 0 and req.kind == "kolmogorov")

    def try_admit(self, req, now):
        if self.cells_in_flight is not None and self.active:
            if sum(a[0].cells for a in self.active) + req.cells > self.cells_in_flight:
                return False
        cfg = request_config(req, self.storage)
        need = self._bytes(req, cfg)
        if self.used + need > self.budget:
            return False
        state = request_state(req)
        if self._dedicated(req):
            sim = Simulation(cfg)
            for k, v in state.items():
                sim.set_pop(k, v)
            parts = request_particles(req)
            if parts is not None:
                sim.set_particles(parts)
            sim.initialize()
            self.active.append([req, "sim", sim, None, need, req.steps])
        else:
            layout = "thermal" if req.kind == "rb" else "fluid"
            ens = self.ensembles.get(layout)
            if ens is None:
                ens = self.ensembles[layout] = Ensemble(self.storage, budget_bytes=self.budget)
            try:
                slot = ens.add(cfg)
            except CH4Error as e:
                if e.status == abi.ERR_NOMEM:
                    return False
                raise
            for k, v in state.items():
                ens.set_pop(slot, k, v)
            ens.initialize(slot)
            self.active.append([req, "ens", ens, slot, need, req.steps])
        self.used += need
        req.admitted = now
        return True

    def launch(self):
        """Enqueue one block: every active simulation advances by the same number of steps
        (asynchronously, each on its stream).  Returns the block and the entries in it."""
        n = min(self.block, min(a[5] for a in self.active))
        for ens in self.ensembles.values():
            ens.step(n)
        for a in self.active:
            if a[1] == "sim":
                a[2].step(n)
        return n, list(self.active)

    def finish(self, n, launched):
        """Wait for a launched block and count its steps."""
        for ens in self.ensembles.values():
            ens.synchronize()
        for a in launched:
            if a[1] == "sim":
                a[2].synchronize()
            a[5] -= n

    def advance(self):
        """One block, launched and waited for."""
        n, launched = self.launch()
        self.finish(n, launched)
        return n

    def retire(self, now):
        keep = []
        for a in self.active:
            req, kind, h, slot, need, remaining = a
            if remaining > 0:
                keep.append(a)
                continue
            req.result = h.averages(slot) if kind == "ens" else h.averages()
            if kind == "ens":
                h.remove(slot)
            else:
                h.close()
            self.used -= need
            req.finished = now
        self.active = keep

    def run(self, requests, clock=time.perf_counter):
        """Serve `requests` (arrival times in seconds from the start).  The next block is on
        the device while the host admits the requests that arrived meanwhile: a new
        simulation (its handle, state upload and initialisation) is built while the others
        step, and joins from the next block on."""
        pending = sorted(requests, key=lambda r: r.arrival)
        waiting = []
        t0 = clock()
        while pending or waiting or self.active:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.pop(0))
            block = self.launch() if self.active else None
            while waiting and self.try_admit(waiting[0], clock() - t0):
                waiting.pop(0)
            if block is None:
                if self.active:
                    continue
                if pending:
                    time.sleep(max(0.0, pending[0].arrival - (clock() - t0)))
                    continue
                if waiting:
                    raise RuntimeError("request %d does not fit the device-memory budget" % waiting[0].rid)
                break
            self.finish(*block)
            self.retire(clock() - t0)
        for ens in self.ensembles.values():
            ens.close()
        self.ensembles = {}
        return requests


def serve_fp64_one_at_a_time(requests, clock=time.perf_counter):
    """The plain FP64 path serving the same requests one at a time (FIFO): measured
    service time per request; latency = queueing behind earlier requests + service."""
    t_free = 0.0
    for req in sorted(requests, key=lambda r: r.arrival):
        cfg = request_config(req, abi.STORE_F64)
        state = request_state(req)
        t0 = clock()
        with Simulation(cfg) as sim:
            for k, v in state.items():
                sim.set_pop(k, v)
            parts = request_particles(req)
            if parts is not None:
                sim.set_particles(parts)
            sim.initialize()
            sim.step(req.steps)
            req.result = sim.averages()
        service = clock() - t0
        start = max(req.arrival, t_free)
        t_free = start + service
        req.admitted = start
        req.finished = t_free
    return requests
