"""Python mirror of the B200 lattice-Boltzmann C ABI (include/ch4.h).

`Simulation` follows the reference driver (src/main.c): configure (define.h flags +
param.in keys), set the initial populations, `initialize()` (src/main.c:24-48),
`step(n)` (src/main.c:67-196), read back populations / hydro fields.  Every call goes
through libch4b200.so; there is no CPU fallback -- if the library or a GPU is
missing, construction raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi
from .abi import NPOP, Config, Particle, Averages, FLAGS, flags_of  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("CH4B200_LIB") or os.path.join(HERE, "libch4b200.so")  # override: another build of the library

_lib = None


class CH4Error(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (abi.STATUS_NAMES.get(status, status), msg))
        self.status = status


def lib():
    """Load libch4b200.so (built in-tree by ch4-project_b200/build.py)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libch4b200.so is not built (run ch4-project_b200/build.py)")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        D = C.POINTER(C.c_double)
        L.ch4_config_default.argtypes = [C.POINTER(Config)]
        L.ch4_config_read_define.argtypes = [C.POINTER(Config), C.c_char_p, C.c_char_p, C.c_size_t]
        L.ch4_config_read_param.argtypes = [C.POINTER(Config), C.c_char_p, C.c_char_p, C.c_size_t]
        L.ch4_read_parameter.argtypes = [C.c_char_p, C.c_char_p, D]
        L.ch4_create.argtypes = [C.POINTER(Config), C.POINTER(P)]
        L.ch4_destroy.argtypes = [P]
        L.ch4_last_error.argtypes = [P]
        L.ch4_last_error.restype = C.c_char_p
        L.ch4_device_bytes.argtypes = [C.POINTER(Config), C.POINTER(C.c_size_t)]
        L.ch4_set_pop.argtypes = [P, C.c_char, D, C.c_int]
        L.ch4_get_pop.argtypes = [P, C.c_char, D, C.c_int]
        L.ch4_set_hit_phases.argtypes = [P, D]
        L.ch4_get_hit_phases.argtypes = [P, D]
        L.ch4_set_particles.argtypes = [P, C.POINTER(Particle), C.c_int]
        L.ch4_get_particles.argtypes = [P, C.POINTER(Particle), C.c_int]
        L.ch4_initialize.argtypes = [P]
        L.ch4_step.argtypes = [P, C.c_int]
        L.ch4_synchronize.argtypes = [P]
        L.ch4_get_fields.argtypes = [P, D, D, D, D, C.c_int]
        L.ch4_get_force.argtypes = [P, D, C.c_int]
        L.ch4_averages_get.argtypes = [P, C.POINTER(Averages)]
        L.ch4_get_itime.argtypes = [P, C.POINTER(C.c_int)]
        L.ch4_get_stream.argtypes = [P, C.POINTER(C.c_void_p)]
        I = C.POINTER(C.c_int)
        L.ch4_ensemble_create.argtypes = [C.c_int, C.c_size_t, C.POINTER(P)]
        L.ch4_ensemble_destroy.argtypes = [P]
        L.ch4_ensemble_last_error.argtypes = [P]
        L.ch4_ensemble_last_error.restype = C.c_char_p
        L.ch4_ensemble_add.argtypes = [P, C.POINTER(Config), I]
        L.ch4_ensemble_remove.argtypes = [P, C.c_int]
        L.ch4_ensemble_set_pop.argtypes = [P, C.c_int, C.c_char, D, C.c_int]
        L.ch4_ensemble_get_pop.argtypes = [P, C.c_int, C.c_char, D, C.c_int]
        L.ch4_ensemble_initialize.argtypes = [P, C.c_int]
        L.ch4_ensemble_step.argtypes = [P, C.c_int]
        L.ch4_ensemble_synchronize.argtypes = [P]
        L.ch4_ensemble_get_fields.argtypes = [P, C.c_int, D, D, D, D, C.c_int]
        L.ch4_ensemble_averages.argtypes = [P, C.c_int, C.POINTER(Averages)]
        L.ch4_ensemble_itime.argtypes = [P, C.c_int, I]
        L.ch4_ensemble_slot_bytes.argtypes = [C.POINTER(Config), C.c_int, C.POINTER(C.c_size_t)]
        L.ch4_ensemble_bytes_in_use.argtypes = [P, C.POINTER(C.c_size_t)]
        L.ch4_ensemble_tune.argtypes = [P, I, I]
        L.ch4_ensemble_set_shape.argtypes = [P, C.c_int, C.c_int]
        L.ch4_ensemble_get_stream.argtypes = [P, C.POINTER(C.c_void_p)]
        L.ch4_initial_populations.argtypes = [C.POINTER(Config), D, D, D, D]
        L.ch4_initial_conditions.argtypes = [P]
        L.ch4_diagnostics.argtypes = [P, D, D, D, D]
        L.ch4_dump_averages.argtypes = [P, C.c_char_p, C.c_double, C.c_int]
        L.ch4_dump_fields_ascii.argtypes = [P, C.c_char_p, C.c_int]
        L.ch4_output_h5.argtypes = [P, C.c_char_p, C.c_int, C.c_double, C.c_int]
        L.ch4_write_pop_h5.argtypes = [P, C.c_char_p]
        L.ch4_read_pop_h5.argtypes = [P, C.c_char_p, C.c_int, C.c_int, C.c_int]
        L.ch4_output_particles_h5.argtypes = [P, C.c_char_p, C.c_int, C.c_double, C.c_int]
        L.ch4_write_particles_h5.argtypes = [P, C.c_char_p]
        L.ch4_read_particles_h5.argtypes = [P, C.c_char_p]
        L.ch4_particle_averages.argtypes = [P, D]
        L.ch4_halo_bytes.argtypes = [P, C.POINTER(C.c_size_t)]
        L.ch4_halo_pack.argtypes = [P, C.c_void_p, C.c_void_p]
        L.ch4_halo_unpack.argtypes = [P, C.c_void_p, C.c_void_p]
        L.ch4_set_gather.argtypes = [P, C.c_void_p, C.c_int, C.c_void_p]
        L.ch4_set_exchange.argtypes = [P, C.c_void_p, C.c_void_p]
        L.ch4_dump_particle_averages.argtypes = [P, C.c_char_p, C.c_double]
        V = C.c_void_p
        L.ch4_averages_noalloc.argtypes = [V, V, V, V, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                           C.c_double, V, V]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def default_config():
    c = Config()
    lib().ch4_config_default(C.byref(c))
    return c


def read_define(cfg, path):
    """Set cfg.flags from a reference define.h (CH4Error on a flag outside the hot path)."""
    bad = C.create_string_buffer(256)
    rc = lib().ch4_config_read_define(C.byref(cfg), path.encode(), bad, 256)
    if rc:
        raise CH4Error(rc, "define.h flag %s" % bad.value.decode())
    return cfg


def read_param(cfg, path):
    """Fill cfg from param.in with the reference's read_parameter semantics."""
    bad = C.create_string_buffer(256)
    rc = lib().ch4_config_read_param(C.byref(cfg), path.encode(), bad, 256)
    if rc:
        raise CH4Error(rc, "param.in key %s" % bad.value.decode())
    return cfg


def read_parameter(path, key):
    v = C.c_double()
    rc = lib().ch4_read_parameter(path.encode(), key.encode(), C.byref(v))
    if rc:
        raise CH4Error(rc, "%s not found in %s" % (key, path))
    return v.value


def initial_populations(cfg):
    """ch4_initial_populations: the reference's initial fields for the *_INITIAL_*
    flags of cfg (host only).  Returns {"p", "g", "h": AoS (NZ, NY, NX, 19) float64,
    "phi": (6, 3) HIT phases drawn after them}."""
    shape = (cfg.NZ, cfg.NY, cfg.NX, abi.NPOP)
    out = {"p": np.zeros(shape)}
    if cfg.flags & abi.FLAGS["LB_TEMPERATURE"]:
        out["g"] = np.zeros(shape)
    if cfg.flags & abi.FLAGS["LB_SCALAR"]:
        out["h"] = np.zeros(shape)
    phi = np.zeros((abi.NK, 3))
    rc = lib().ch4_initial_populations(C.byref(cfg), _dp(out["p"]), _dp(out.get("g")), _dp(out.get("h")), _dp(phi))
    if rc:
        raise CH4Error(rc, "ch4_initial_populations")
    out["phi"] = phi
    return out


def device_bytes(cfg):
    n = C.c_size_t()
    rc = lib().ch4_device_bytes(C.byref(cfg), C.byref(n))
    if rc:
        raise CH4Error(rc, "device_bytes")
    return n.value


class Simulation:
    """One lattice on the current CUDA device (handle of include/ch4.h)."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.h = C.c_void_p()
        rc = lib().ch4_create(C.byref(cfg), C.byref(self.h))
        if rc:
            raise CH4Error(rc, "ch4_create")

    def close(self):
        if self.h:
            lib().ch4_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what):
        if rc:
            raise CH4Error(rc, "%s: %s" % (what, lib().ch4_last_error(self.h).decode()))

    def set_pop(self, which, aos, brd=0):
        a = np.ascontiguousarray(aos, dtype=np.float64)
        self._check(lib().ch4_set_pop(self.h, which.encode(), _dp(a), brd), "set_pop")

    def get_pop(self, which, brd=0, out=None):
        c = self.cfg
        a = out if out is not None else np.empty((c.NZ + 2 * brd, c.NY + 2 * brd, c.NX + 2 * brd, NPOP))
        self._check(lib().ch4_get_pop(self.h, which.encode(), _dp(a), brd), "get_pop")
        return a

    def set_hit_phases(self, phi):
        a = np.ascontiguousarray(phi, dtype=np.float64)
        self._check(lib().ch4_set_hit_phases(self.h, _dp(a)), "set_hit_phases")

    def get_hit_phases(self):
        a = np.empty((abi.NK, 3))
        self._check(lib().ch4_get_hit_phases(self.h, _dp(a)), "get_hit_phases")
        return a

    def set_particles(self, parts):
        self._check(lib().ch4_set_particles(self.h, parts, len(parts)), "set_particles")

    def get_particles(self, n):
        arr = (Particle * n)()
        self._check(lib().ch4_get_particles(self.h, arr, n), "get_particles")
        return arr

    def initial_conditions(self):
        """ch4_initial_conditions: the reference's initial fields and HIT phases."""
        self._check(lib().ch4_initial_conditions(self.h), "initial_conditions")

    def initialize(self):
        self._check(lib().ch4_initialize(self.h), "initialize")

    def step(self, n=1):
        self._check(lib().ch4_step(self.h, n), "step")

    def synchronize(self):
        self._check(lib().ch4_synchronize(self.h), "synchronize")

    def fields(self):
        c = self.cfg
        dens = np.empty((c.NZ, c.NY, c.NX))
        u = np.empty((c.NZ, c.NY, c.NX, 3))
        t = np.empty((c.NZ, c.NY, c.NX))
        s = np.empty((c.NZ, c.NY, c.NX))
        self._check(lib().ch4_get_fields(self.h, _dp(dens), _dp(u), _dp(t), _dp(s), 0), "get_fields")
        return {"dens": dens, "u": u, "t": t, "s": s}

    def force(self):
        c = self.cfg
        f = np.empty((c.NZ, c.NY, c.NX, 3))
        self._check(lib().ch4_get_force(self.h, _dp(f), 0), "get_force")
        return f

    def averages(self):
        a = Averages()
        self._check(lib().ch4_averages_get(self.h, C.byref(a)), "averages")
        return {n: getattr(a, n) for n in abi.AVERAGE_FIELDS}

    def diagnostics(self, rulers=True):
        """ch4_diagnostics: dump_averages' volume averages ({field: value}) and, with
        rulers, the per-plane averages along x, y, z as {field: array over the planes}."""
        c = self.cfg
        nf = len(abi.DIAG_FIELDS)
        g = np.zeros(nf)
        rs = [np.zeros((n, nf)) for n in (c.NX, c.NY, c.NZ)] if rulers else [None] * 3
        self._check(lib().ch4_diagnostics(self.h, _dp(g), *[_dp(r) for r in rs]), "diagnostics")
        out = {"global": dict(zip(abi.DIAG_FIELDS, g))}
        if rulers:
            for axis, r in zip("xyz", rs):
                out[axis] = {f: r[:, q].copy() for q, f in enumerate(abi.DIAG_FIELDS)}
        return out

    def dump_averages(self, directory, time_now, irun):
        """ch4_dump_averages: the reference's dump_averages ASCII files in `directory`."""
        self._check(lib().ch4_dump_averages(self.h, str(directory).encode(), float(time_now), int(irun)),
                    "dump_averages")

    def particle_averages(self):
        """ch4_particle_averages: dump_particle_averages' means per particle type, as
        {field: array over the cfg.particle_types types} (field "count" included)."""
        nt = max(1, self.cfg.particle_types)
        a = np.zeros((nt, len(abi.PART_AVG_FIELDS)))
        self._check(lib().ch4_particle_averages(self.h, _dp(a)), "particle_averages")
        return {f: a[:, q].copy() for q, f in enumerate(abi.PART_AVG_FIELDS)}

    def dump_particle_averages(self, directory, time_now):
        """ch4_dump_particle_averages: appends the types' lines to directory/particle_averages.dat."""
        self._check(lib().ch4_dump_particle_averages(self.h, str(directory).encode(), float(time_now)),
                    "dump_particle_averages")

    def dump_fields_ascii(self, directory, itime):
        """ch4_dump_fields_ascii: the OUTPUT_ASCII vel/temp/scal.<itime> files in `directory`."""
        self._check(lib().ch4_dump_fields_ascii(self.h, str(directory).encode(), int(itime)), "dump_fields_ascii")

    def output_h5(self, directory, itime, time_now=0.0, grid=True, timestamp_real=False):
        """ch4_output_h5: field_<n>.h5 (group /euler) and field_<n>.xmf in `directory`
        (OUTPUT_H5_GRID adds the cell-centre coordinates; OUTPUT_H5_TIMESTAMP_REAL names the
        files by (int)time_now instead of itime)."""
        opts = (abi.H5_GRID if grid else 0) | (abi.H5_TIMESTAMP_REAL if timestamp_real else 0)
        self._check(lib().ch4_output_h5(self.h, str(directory).encode(), int(itime), float(time_now), opts),
                    "output_h5")

    def write_pop_h5(self, path="pop.h5"):
        """ch4_write_pop_h5: the populations (and HIT phases) as the reference's pop.h5."""
        self._check(lib().ch4_write_pop_h5(self.h, str(path).encode()), "write_pop_h5")

    def output_particles_h5(self, directory, itime, time_now=0.0, output_fluid=False, timestamp_real=False):
        """ch4_output_particles_h5: particle_<n>.h5 (group /lagrange) and particle_<n>.xmf."""
        opts = (abi.H5_LAGRANGE_OUTPUT_FLUID if output_fluid else 0) | (abi.H5_TIMESTAMP_REAL if timestamp_real else 0)
        self._check(lib().ch4_output_particles_h5(self.h, str(directory).encode(), int(itime), float(time_now), opts),
                    "output_particles_h5")

    def write_particles_h5(self, path="part.h5"):
        """ch4_write_particles_h5: the particles as the reference's part.h5."""
        self._check(lib().ch4_write_particles_h5(self.h, str(path).encode()), "write_particles_h5")

    def read_particles_h5(self, path="part.h5"):
        """ch4_read_particles_h5: load part.h5 into the handle (before initialize)."""
        self._check(lib().ch4_read_particles_h5(self.h, str(path).encode()), "read_particles_h5")

    def read_pop_h5(self, path="pop.h5", resume_u=True, resume_t=True, resume_s=True):
        """ch4_read_pop_h5: load pop.h5 (before initialize), as the reference's resume does."""
        self._check(lib().ch4_read_pop_h5(self.h, str(path).encode(), int(resume_u), int(resume_t), int(resume_s)),
                    "read_pop_h5")

    @property
    def stream_handle(self):
        """cudaStream_t of this handle as an integer (for torch.cuda.ExternalStream)."""
        v = C.c_void_p()
        self._check(lib().ch4_get_stream(self.h, C.byref(v)), "get_stream")
        return v.value or 0

    @property
    def itime(self):
        v = C.c_int()
        self._check(lib().ch4_get_itime(self.h, C.byref(v)), "get_itime")
        return v.value


class Ensemble:
    """Many independent lattices advanced together (ch4_ensemble_* of include/ch4.h)."""

    def __init__(self, storage=abi.STORE_F32, budget_bytes=0):
        self.h = C.c_void_p()
        rc = lib().ch4_ensemble_create(storage, budget_bytes, C.byref(self.h))
        if rc:
            raise CH4Error(rc, "ch4_ensemble_create")
        self.cfgs = {}

    def close(self):
        if self.h:
            lib().ch4_ensemble_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what):
        if rc:
            raise CH4Error(rc, "%s: %s" % (what, lib().ch4_ensemble_last_error(self.h).decode()))

    def add(self, cfg):
        slot = C.c_int()
        self._check(lib().ch4_ensemble_add(self.h, C.byref(cfg), C.byref(slot)), "add")
        self.cfgs[slot.value] = cfg
        return slot.value

    def remove(self, slot):
        self._check(lib().ch4_ensemble_remove(self.h, slot), "remove")
        self.cfgs.pop(slot, None)

    def set_pop(self, slot, which, aos, brd=0):
        a = np.ascontiguousarray(aos, dtype=np.float64)
        self._check(lib().ch4_ensemble_set_pop(self.h, slot, which.encode(), _dp(a), brd), "set_pop")

    def get_pop(self, slot, which, brd=0):
        c = self.cfgs[slot]
        a = np.empty((c.NZ + 2 * brd, c.NY + 2 * brd, c.NX + 2 * brd, NPOP))
        self._check(lib().ch4_ensemble_get_pop(self.h, slot, which.encode(), _dp(a), brd), "get_pop")
        return a

    def initialize(self, slot):
        self._check(lib().ch4_ensemble_initialize(self.h, slot), "initialize")

    def step(self, n=1):
        self._check(lib().ch4_ensemble_step(self.h, n), "step")

    def synchronize(self):
        self._check(lib().ch4_ensemble_synchronize(self.h), "synchronize")

    def fields(self, slot):
        c = self.cfgs[slot]
        dens = np.empty((c.NZ, c.NY, c.NX))
        u = np.empty((c.NZ, c.NY, c.NX, 3))
        t = np.empty((c.NZ, c.NY, c.NX))
        s = np.empty((c.NZ, c.NY, c.NX))
        self._check(lib().ch4_ensemble_get_fields(self.h, slot, _dp(dens), _dp(u), _dp(t), _dp(s), 0), "fields")
        return {"dens": dens, "u": u, "t": t, "s": s}

    def averages(self, slot):
        a = Averages()
        self._check(lib().ch4_ensemble_averages(self.h, slot, C.byref(a)), "averages")
        return {n: getattr(a, n) for n in abi.AVERAGE_FIELDS}

    def itime(self, slot):
        v = C.c_int()
        self._check(lib().ch4_ensemble_itime(self.h, slot, C.byref(v)), "itime")
        return v.value

    def bytes_in_use(self):
        v = C.c_size_t()
        self._check(lib().ch4_ensemble_bytes_in_use(self.h, C.byref(v)), "bytes_in_use")
        return v.value

    def tune(self):
        b, r = C.c_int(), C.c_int()
        self._check(lib().ch4_ensemble_tune(self.h, C.byref(b), C.byref(r)), "tune")
        return b.value, r.value

    @property
    def stream_handle(self):
        """cudaStream_t of the ensemble as an integer (for torch.cuda.ExternalStream)."""
        v = C.c_void_p()
        self._check(lib().ch4_ensemble_get_stream(self.h, C.byref(v)), "get_stream")
        return v.value or 0

    def set_shape(self, block, rows):
        self._check(lib().ch4_ensemble_set_shape(self.h, block, rows), "set_shape")


def ensemble_slot_bytes(cfg, storage):
    v = C.c_size_t()
    rc = lib().ch4_ensemble_slot_bytes(C.byref(cfg), storage, C.byref(v))
    if rc:
        raise CH4Error(rc, "slot_bytes")
    return v.value


NOALLOC_MAX_CELLS = 2048 * 65536  # CH4_NOALLOC_MAX_BLOCKS * CH4_NOALLOC_CELLS_PER_BLOCK


def averages_noalloc(dens, u, t, s, NX, NY, NZ, fluid_walls, scalar_walls, nu, kappa, sums, stream=0):
    """ch4_averages_noalloc: raw dump_averages sums of FP64 device fields (device
    addresses as integers) into `sums` (23 device doubles); allocates nothing.
    For callers that cannot call cudaMalloc (a diagnostic inside a stream-ordered
    time loop, or a fully reserved device-memory budget)."""
    rc = lib().ch4_averages_noalloc(dens, u, t, s, NX, NY, NZ, int(fluid_walls), int(scalar_walls), nu, kappa,
                                    sums, stream)
    if rc:
        raise CH4Error(rc, "ch4_averages_noalloc")
