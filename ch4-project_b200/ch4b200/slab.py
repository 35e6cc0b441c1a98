"""One lattice as z-slabs, one handle per GPU (ch4_halo_pack / ch4_halo_unpack).

Each slab holds NZ_local planes of a lattice NZ planes deep (ch4_config.nz_global,
z_offset).  Its step streams the populations leaving through the z faces periodically
onto its own opposite face; after every step the slabs swap those values: every slab
sends the 5 c_z = -1 directions of its top plane to the slab below and the 5 c_z = +1
directions of its bottom plane to the slab above (SZ * NX*NY values per set and
face), and writes what it receives into the same places.  The x and y directions,
y walls and forcing are plane-local, so the decomposition reproduces the single
lattice bit for bit (HIT tables run over the whole lattice's z).

The transfer is the caller's plumbing: `exchange` pairs the four point-to-point
transfers of one step over a torch.distributed process group (NCCL between GPUs, or
through host copies over gloo); `step_local` runs several slabs of one process, each
unpacking straight from its neighbours' send buffers.  Registered as the handle's face
exchange (ch4_set_face_exchange: `Slab.use_process_group`, `use_local_faces`), the
transfer runs inside ch4_step on a second stream while the slab's interior planes are
stepped.

With LB_FLUID_FORCING_NOZEROMODE / _CONSTANT_POWER every step also needs the force summed
over the whole lattice: each slab's handle calls back (ch4_set_gather) with its block
partial sums, and the callback gathers every slab's in z order -- an all-gather over the
process group (`Slab.use_process_group`), or, for the slabs of one process stepped in
threads, through host memory (`LocalGather`).

With LB_FLUID_LES the eddy viscosity differentiates u across the z faces: in the middle
of every step each slab's handle calls back (ch4_set_exchange) with the u of its bottom
and top planes, and the callback swaps them with the neighbours -- point to point over
the process group, or between the threads of one process (`LocalExchange`).

Lagrangian particles (periodic lattices, one-way coupling) use the same callback: after
the hydrodynamic pass every slab swaps the two planes of u next to each face (the
interpolation stencil reaches two planes beyond the slab), and after every sub-step the
particles that left the slab move to the neighbour below or above
(sendrecv_particles, src/lagrange.c:4028-4221).  Every slab takes the whole particle
array (`Slab.set_particles`) and keeps the particles in its planes; `gather_particles`
puts the slabs' particles back into one array in the caller's order.
"""
import ctypes as C
import threading

import numpy as np

from . import Simulation, lib
from . import abi


GATHER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p)
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                          C.c_void_p)


class _DeviceBytes:
    """A device byte range as a __cuda_array_interface__ object (zero-copy torch view)."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3, "strides": None}


def _view(ptr, nbytes):
    import torch
    return torch.as_tensor(_DeviceBytes(ptr, nbytes), device="cuda")


class LocalGather:
    """The force-sum gather of n slabs of one process, each stepped in its own thread:
    every slab copies its partials to host memory, waits for the others, and copies
    the whole z-ordered set back to its device buffer on its stream."""

    def __init__(self, n):
        self.n = n
        self.slots = [None] * n
        self.barrier = threading.Barrier(n)

    def callback(self, index):
        import torch

        def cb(local, all_, nbytes, stream, user):
            try:
                st = torch.cuda.ExternalStream(stream)
                with torch.cuda.stream(st):
                    self.slots[index] = _view(local, nbytes).cpu()
                self.barrier.wait()
                whole = torch.cat(self.slots)
                with torch.cuda.stream(st):
                    _view(all_, nbytes * self.n).copy_(whole)
                    st.synchronize()
                self.barrier.wait()  # nobody refills a slot before every slab has read them all
                return 0
            except Exception:  # noqa: BLE001 - reported to the library as a failed gather
                self.barrier.abort()
                return 1
        return GATHER_FN(cb)


class LocalExchange:
    """The u-face exchange of n slabs of one process (one device), each stepped in its
    own thread: every slab publishes its send buffers once its stream has written them,
    then copies its neighbours' into its own receive buffers."""

    def __init__(self, n):
        self.n = n
        self.sends = [None] * n
        self.barrier = threading.Barrier(n)

    def callback(self, index):
        import torch

        def cb(send_down, send_up, from_up, from_down, nbytes, stream, user):
            try:
                st = torch.cuda.ExternalStream(stream)
                st.synchronize()
                self.sends[index] = (send_down, send_up)
                self.barrier.wait()
                above, below = self.sends[(index + 1) % self.n], self.sends[(index - 1) % self.n]
                with torch.cuda.stream(st):
                    _view(from_up, nbytes).copy_(_view(above[0], nbytes))
                    _view(from_down, nbytes).copy_(_view(below[1], nbytes))
                    st.synchronize()
                self.barrier.wait()  # no slab rewrites its send buffers before all have read them
                return 0
            except Exception:  # noqa: BLE001 - reported to the library as a failed exchange
                self.barrier.abort()
                return 1
        return EXCHANGE_FN(cb)


def bounds(nz, nslabs):
    """(z_offset, planes) of each slab: an even split, the first nz % nslabs one plane deeper."""
    if not 1 <= nslabs <= nz:
        raise ValueError("need 1 <= slabs <= NZ")
    q, r = divmod(nz, nslabs)
    out, z = [], 0
    for i in range(nslabs):
        n = q + (1 if i < r else 0)
        out.append((z, n))
        z += n
    return out


def slab_config(cfg, z0, nz):
    """The configuration of planes z0 .. z0+nz-1 of the whole-lattice configuration cfg."""
    c = abi.Config()
    C.pointer(c)[0] = cfg
    c.nz_global = cfg.NZ
    c.z_offset = z0
    c.NZ = nz
    return c


def neighbours(rank, world):
    """(below, above): the ranks holding the slabs under and over this one (periodic in z)."""
    return (rank - 1) % world, (rank + 1) % world


def exchange(send_down, send_up, recv_up, recv_down, rank, world, group=None):
    """One step's face exchange over torch.distributed: send_down -> the slab below (its
    recv_up), send_up -> the slab above (its recv_down).  With one rank the slab is its
    own neighbour (the periodic lattice).  The four transfers are issued as one batch in
    the same order on every rank, so a pair of ranks that are each other's neighbour on
    both sides (two slabs) still matches them one to one."""
    import torch.distributed as dist
    if world == 1:
        recv_up.copy_(send_down)
        recv_down.copy_(send_up)
        return
    below, above = neighbours(rank, world)
    staged = send_down.is_cuda and dist.get_backend(group) == "gloo"
    if staged:  # gloo moves host memory: device faces through host copies (blocking)
        import torch
        torch.cuda.current_stream().synchronize()
        bufs = [send_down.cpu(), torch.empty(recv_up.shape, dtype=recv_up.dtype), send_up.cpu(),
                torch.empty(recv_down.shape, dtype=recv_down.dtype)]
    else:
        bufs = [send_down, recv_up, send_up, recv_down]
    ops = [dist.P2POp(dist.isend, bufs[0], below, group), dist.P2POp(dist.irecv, bufs[1], above, group),
           dist.P2POp(dist.isend, bufs[2], above, group), dist.P2POp(dist.irecv, bufs[3], below, group)]
    for w in dist.batch_isend_irecv(ops):
        w.wait()
    if staged:
        recv_up.copy_(bufs[1])
        recv_down.copy_(bufs[3])


def all_gather(whole, local, world, group=None):
    """whole <- the `local` of every rank in rank order (NCCL on the current stream, or
    through host memory over gloo)."""
    import torch
    import torch.distributed as dist
    if world == 1:
        whole.copy_(local)
    elif local.is_cuda and dist.get_backend(group) == "gloo":
        torch.cuda.current_stream().synchronize()
        parts = [torch.empty(local.shape, dtype=local.dtype) for _ in range(world)]
        dist.all_gather(parts, local.cpu(), group=group)
        whole.copy_(torch.cat(parts))
    else:
        dist.all_gather_into_tensor(whole, local, group=group)


class Slab:
    """A Simulation holding planes z0 .. z0+nz-1 of the lattice `cfg`, with its four
    face buffers as device tensors."""

    def __init__(self, cfg, z0, nz, device=None):
        import torch
        self.z0, self.nz = z0, nz
        self.sim = Simulation(slab_config(cfg, z0, nz))
        n = C.c_size_t()
        self.sim._check(lib().ch4_halo_bytes(self.sim.h, C.byref(n)), "halo_bytes")
        dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.send_down, self.send_up, self.recv_up, self.recv_down = (
            torch.empty(n.value, dtype=torch.uint8, device=dev) for _ in range(4))

    def set_gather(self, fn, nslabs):
        """Register the force-sum gather (a GATHER_FN); kept alive with the slab."""
        self._gather = fn
        self.sim._check(lib().ch4_set_gather(self.sim.h, C.cast(fn, C.c_void_p), nslabs, None), "set_gather")

    def set_exchange(self, fn):
        """Register the u-face exchange (an EXCHANGE_FN) for LES; kept alive with the slab."""
        self._exchange = fn
        self.sim._check(lib().ch4_set_exchange(self.sim.h, C.cast(fn, C.c_void_p), None), "set_exchange")

    def set_face_exchange(self, fn):
        """Register the population-face transfer (an EXCHANGE_FN) that ch4_step runs itself,
        overlapped with the interior planes; kept alive with the slab."""
        self._faces = fn
        self.sim._check(lib().ch4_set_face_exchange(self.sim.h, C.cast(fn, C.c_void_p) if fn else None, None),
                        "set_face_exchange")
        self.self_exchanging = fn is not None

    def use_process_group(self, rank, world, group=None, overlap=True):
        """Over the process group: the force sums all-gathered (z order = rank order), the
        LES u faces and the population faces swapped point to point with the neighbouring
        ranks -- NCCL on the handle's streams, or host-staged over gloo.  With `overlap` the
        population faces move inside ch4_step while the interior planes are stepped."""
        import torch

        def xcb(send_down, send_up, from_up, from_down, nbytes, stream, user):
            try:
                with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                    exchange(_view(send_down, nbytes), _view(send_up, nbytes), _view(from_up, nbytes),
                             _view(from_down, nbytes), rank, world, group)
                return 0
            except Exception:  # noqa: BLE001 - reported to the library as a failed exchange
                return 1
        self.set_exchange(EXCHANGE_FN(xcb))
        if overlap:
            self.set_face_exchange(EXCHANGE_FN(xcb))

        def cb(local, all_, nbytes, stream, user):
            try:
                with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                    all_gather(_view(all_, nbytes * world), _view(local, nbytes), world, group)
                return 0
            except Exception:  # noqa: BLE001 - reported to the library as a failed gather
                return 1
        self.set_gather(GATHER_FN(cb), world)

    def set_particles(self, parts):
        """Every particle of the lattice (a ch4b200.Particle array): the slab keeps those in
        its planes."""
        self.sim.set_particles(parts)
        self.nparts = len(parts)

    def get_particles_into(self, parts):
        """Write this slab's particles into their entries of `parts` (all particles)."""
        self.sim._check(lib().ch4_get_particles(self.sim.h, parts, len(parts)), "get_particles")

    def set_pop(self, which, aos_whole):
        """Populations of the whole lattice, AoS [NZ][NY][NX][19]: this slab's planes."""
        self.sim.set_pop(which, np.ascontiguousarray(aos_whole[self.z0:self.z0 + self.nz]))

    def pack(self):
        self.sim._check(lib().ch4_halo_pack(self.sim.h, C.c_void_p(self.send_down.data_ptr()),
                                            C.c_void_p(self.send_up.data_ptr())), "halo_pack")

    def unpack(self, from_up=None, from_down=None):
        fu = self.recv_up if from_up is None else from_up
        fd = self.recv_down if from_down is None else from_down
        self.sim._check(lib().ch4_halo_unpack(self.sim.h, C.c_void_p(fu.data_ptr()), C.c_void_p(fd.data_ptr())),
                        "halo_unpack")

    def step(self, n, rank, world, group=None):
        """n steps of a slab of a multi-rank lattice: with the face exchange registered,
        ch4_step moves the faces itself; else step, pack, exchange on the handle's stream,
        unpack."""
        import torch
        if getattr(self, "self_exchanging", False):
            self.sim.step(n)
            return
        stream = torch.cuda.ExternalStream(self.sim.stream_handle)
        for _ in range(n):
            self.sim.step(1)
            self.pack()
            with torch.cuda.stream(stream):
                exchange(self.send_down, self.send_up, self.recv_up, self.recv_down, rank, world, group)
            self.unpack()

    def close(self):
        self.sim.close()


def gather_particles(slabs, n):
    """The particles of the slabs of one process as one array of n, in the caller's order."""
    from . import Particle
    out = (Particle * n)()
    for s in slabs:
        s.get_particles_into(out)
    return out


def _in_threads(slabs, fn):
    """fn(slab) for every slab at once, one thread each (the force-sum gather of slabs of
    one process meets in the middle of their steps)."""
    errs = []

    def run(s):
        try:
            fn(s)
        except Exception as e:  # noqa: BLE001 - re-raised below
            errs.append(e)
    ts = [threading.Thread(target=run, args=(s,)) for s in slabs]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errs:
        raise errs[0]


def use_local_gather(slabs):
    """Slabs of one process: gather the force sums through host memory (step_local and
    initialize_local then run the slabs in threads)."""
    g = LocalGather(len(slabs))
    for i, s in enumerate(slabs):
        s.set_gather(g.callback(i), len(slabs))
        s.local_gather = True


def use_local_exchange(slabs):
    """Slabs of one process with LES: swap the u faces between their threads
    (step_local then runs the slabs in threads)."""
    x = LocalExchange(len(slabs))
    for i, s in enumerate(slabs):
        s.set_exchange(x.callback(i))
        s.local_gather = True


def use_local_faces(slabs):
    """Slabs of one process: the population faces move inside every ch4_step, overlapped
    with the slab's interior planes, swapped between the slabs' threads (step_local then
    runs the slabs in threads)."""
    x = LocalExchange(len(slabs))
    for i, s in enumerate(slabs):
        s.set_face_exchange(x.callback(i))
        s.local_gather = True


def initialize_local(slabs):
    if any(getattr(s, "local_gather", False) for s in slabs):
        _in_threads(slabs, lambda s: s.sim.initialize())
    else:
        for s in slabs:
            s.sim.initialize()


def step_local(slabs, n):
    """n steps of the slabs of one process (in z order): every slab unpacks straight
    from its neighbours' send buffers once all have packed."""
    m = len(slabs)
    if all(getattr(s, "self_exchanging", False) for s in slabs):
        _in_threads(slabs, lambda s: s.sim.step(n))
        return
    threaded = any(getattr(s, "local_gather", False) for s in slabs)
    for _ in range(n):
        if threaded:
            _in_threads(slabs, lambda s: s.sim.step(1))
        else:
            for s in slabs:
                s.sim.step(1)
        for s in slabs:
            s.pack()
        for s in slabs:
            s.sim.synchronize()
        for i, s in enumerate(slabs):
            s.unpack(from_up=slabs[(i + 1) % m].send_down, from_down=slabs[(i - 1) % m].send_up)
        for s in slabs:
            s.sim.synchronize()
