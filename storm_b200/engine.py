"""ctypes binding of libstorm_cuda.so (include/storm_cuda.h).

The engine has no CPU fallback: loading fails loudly when the shared library is
missing, and creating a handle fails with STORM_ERR_NO_DEVICE without a GPU.
"""
import ctypes as C
import os
import numpy as np

from . import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libstorm_cuda.so")
_lib = None


class StormError(RuntimeError):
    """Raised for a nonzero status; mirrors STORM::StormError (StormError.hpp:13-48)."""

    def __init__(self, status, msg, derr=0, cell=0, particle=0):
        self.status, self.derr, self.cell, self.particle = status, derr, cell, particle
        super().__init__(f"{A.STATUS_NAMES.get(status, status)}: {msg} "
                         f"(device error {A.DERR_NAMES.get(derr, derr)}, cell {cell}, particle {particle})")


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"CUDA engine library not built: {LIB_PATH} (run python -m storm_b200.build)")
        L = C.CDLL(LIB_PATH)
        vp, dp = C.c_void_p, C.POINTER(C.c_double)
        u64p, u32p, i32p = C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.POINTER(C.c_int32)
        L.storm_cuda_create.argtypes = [C.POINTER(A.StormProblemDesc), C.POINTER(vp)]
        L.storm_mesh_voronoi.argtypes = [dp, C.c_uint32, dp, C.POINTER(C.POINTER(A.StormPolyMesh))]
        L.storm_mesh_free.argtypes = [C.POINTER(A.StormPolyMesh)]
        L.storm_cuda_checkpoint_size.argtypes = [vp, u64p]
        L.storm_cuda_checkpoint_save.argtypes = [vp, C.c_void_p, C.c_uint64]
        L.storm_cuda_checkpoint_load.argtypes = [vp, C.c_void_p, C.c_uint64]
        L.storm_cuda_destroy.argtypes = [vp]
        L.storm_cuda_step.argtypes = [vp, C.c_double, C.POINTER(A.StormStepStats)]
        for f in ("begin", "prestep", "emit", "poststep"):
            getattr(L, "storm_cuda_phase_" + f).argtypes = [vp, C.c_double]
        for f in ("transport", "comb"):
            getattr(L, "storm_cuda_phase_" + f).argtypes = [vp]
        L.storm_cuda_phase_stats.argtypes = [vp, C.POINTER(A.StormStepStats)]
        L.storm_cuda_set_census.argtypes = [vp, C.POINTER(A.StormParticlesSoA)]
        L.storm_cuda_get_census.argtypes = [vp, C.POINTER(A.StormParticlesSoA), C.c_uint64, u64p]
        L.storm_cuda_step_host.argtypes = [vp, C.c_double, C.POINTER(A.StormParticlesSoA),
                                           C.POINTER(A.StormParticlesSoA), C.c_uint64, u64p,
                                           C.POINTER(A.StormStepStats)]
        L.storm_cuda_census_count.argtypes = [vp, u64p]
        L.storm_cuda_get_bank.argtypes = [vp, C.POINTER(A.StormParticlesSoA), C.c_uint64, u64p]
        L.storm_cuda_population_control.argtypes = [vp, C.POINTER(A.StormParticlesSoA)]
        L.storm_cuda_get_cell_arrays.argtypes = [vp, dp, dp, dp, dp, dp, dp, u64p]
        L.storm_cuda_set_cell_state.argtypes = [vp, dp, dp, dp]
        L.storm_cuda_set_cell_physics.argtypes = [vp, dp, dp, dp]
        L.storm_cuda_set_opacity_tables.argtypes = [vp, dp, dp]
        L.storm_cuda_set_cell_motion.argtypes = [vp, dp, dp]
        L.storm_cuda_get_cell_motion.argtypes = [vp, dp, dp]
        L.storm_cuda_get_group_tallies.argtypes = [vp, dp]
        L.storm_cuda_set_sharding.argtypes = [vp, C.c_uint32, C.c_uint32, C.c_uint32, A.ExchangeFn, vp]
        L.storm_cuda_get_beginning_counts.argtypes = [vp, u64p]
        L.storm_cuda_set_face_temperature.argtypes = [vp, C.c_int, C.c_double]
        L.storm_cuda_get_emission.argtypes = [vp, u64p, dp]
        L.storm_cuda_replay_segments.argtypes = [vp, C.POINTER(A.StormReplayBatch)]
        L.storm_cuda_get_random_walk_tables.argtypes = [vp, dp, dp, dp]
        L.storm_cuda_random_walk_sample.argtypes = [vp, C.c_uint64, dp, dp, dp, dp, dp]
        L.storm_cuda_last_error.argtypes = [vp, i32p, u64p, u64p, C.c_char_p, C.c_size_t]
        L.storm_cuda_memory_bytes.argtypes = [vp, u64p]
        L.storm_cuda_launch_count.argtypes = [vp, u64p]
        L.storm_cuda_set_segments_per_visit.argtypes = [vp, C.c_uint32]
        L.storm_cuda_set_profiling.argtypes = [vp, C.c_int]
        L.storm_cuda_set_transport_variant.argtypes = [vp, C.c_int, C.c_int]
        L.storm_cuda_set_transport_mode.argtypes = [vp, C.c_int, C.c_uint32]
        L.storm_cuda_autotune_transport.argtypes = [vp, C.c_uint32]
        L.storm_cuda_transport_burst.argtypes = [vp, u32p, C.POINTER(C.c_int)]
        L.storm_cuda_transport_timing.argtypes = [vp, dp, u64p, u64p, C.c_int]
        L.storm_cuda_release_cached.argtypes = [C.c_int, u64p]
        L.storm_cuda_pool_counters.argtypes = [u64p, u64p, u64p, u64p]
        L.storm_server_create.argtypes = [C.POINTER(A.StormServerConfig), C.POINTER(vp)]
        L.storm_server_submit.argtypes = [vp, C.POINTER(A.StormProblemDesc), C.c_uint32, C.c_double, dp, u64p]
        L.storm_server_poll.argtypes = [vp, C.POINTER(A.StormRequestResult), C.c_uint32, C.POINTER(C.c_uint32)]
        L.storm_server_drain.argtypes = [vp]
        L.storm_server_stats.argtypes = [vp, C.POINTER(A.StormServerStats)]
        L.storm_server_destroy.argtypes = [vp]
        L.storm_cuda_status_string.restype = C.c_char_p
        L.storm_cuda_status_string.argtypes = [C.c_int]
        L.storm_cuda_abi_version.restype = C.c_int
        _lib = L
    return _lib


def pool_counters():
    """The device memory cache's counters: cudaMalloc and cudaFree calls since
    the library loaded, bytes cached and bytes handed out."""
    v = [C.c_uint64() for _ in range(4)]
    lib().storm_cuda_pool_counters(*[C.byref(x) for x in v])
    return dict(zip(("mallocs", "frees", "cached_bytes", "live_bytes"), (x.value for x in v)))


def release_cached(device=0):
    """Return the device memory cache's blocks on `device` to the driver; the bytes released."""
    b = C.c_uint64()
    rc = lib().storm_cuda_release_cached(device, C.byref(b))
    if rc != A.STORM_OK:
        raise StormError(rc, lib().storm_cuda_status_string(rc).decode())
    return b.value


class Particles:
    """Host struct-of-arrays census (the fields of Particle<T,Grid> the gray path uses)."""
    FIELDS = ("x", "y", "z", "vx", "vy", "vz", "time_left", "weight", "initial_weight")

    def __init__(self, n=0):
        for f in self.FIELDS:
            setattr(self, f, np.zeros(n))
        self.cell = np.zeros(n, np.uint32)
        self.id = np.zeros(n, np.uint64)
        self.n = n
        self.frequency = np.zeros(n)   # photon energy (multigroup)

    @classmethod
    def pinned(cls, capacity):
        """A buffer in page-locked host memory (full-rate host<->device copies);
        id is left out (None)."""
        import torch
        p = cls(0)
        for f in cls.FIELDS:
            setattr(p, f, torch.empty(capacity, dtype=torch.float64, pin_memory=True).numpy())
        p.cell = torch.empty(capacity, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
        p.id = None
        p.frequency = None
        p.n = capacity
        return p

    def view(self, n):
        """The first n particles, sharing this buffer's memory."""
        if n > self.n:
            raise ValueError(f"buffer holds {self.n} particles, {n} requested")
        v = Particles(0)
        for f in self.FIELDS:
            a = getattr(self, f)
            setattr(v, f, None if a is None else a[:n])
        v.cell = self.cell[:n]
        v.id = None if self.id is None else self.id[:n]
        v.frequency = None if getattr(self, "frequency", None) is None else self.frequency[:n]
        v.n = n
        return v

    def soa(self):
        """Struct of pointers; every field is made contiguous first (the C side
        reads plain arrays).  id may be None (not read or written); so may
        time_left and initial_weight for storm_cuda_set_census, which a step
        sets itself."""
        for f in self.FIELDS:
            if getattr(self, f) is not None:
                setattr(self, f, np.ascontiguousarray(getattr(self, f), dtype=np.float64))
        self.cell = np.ascontiguousarray(self.cell, dtype=np.uint32)
        s = A.StormParticlesSoA()
        for f in self.FIELDS:
            if getattr(self, f) is not None:
                setattr(s, f, A.ptr(getattr(self, f)))
        s.cell = A.ptr(self.cell, C.c_uint32)
        if self.id is not None:
            self.id = np.ascontiguousarray(self.id, dtype=np.uint64)
            s.id = A.ptr(self.id, C.c_uint64)
        if getattr(self, "frequency", None) is not None:
            self.frequency = np.ascontiguousarray(self.frequency, dtype=np.float64)
            s.frequency = A.ptr(self.frequency)
        s.count = self.n
        return s

    def __len__(self):
        return self.n


class Engine:
    """One IMC problem on the GPU (a StormHandle)."""

    def __init__(self, problem):
        self.problem = problem
        self.desc = problem.to_desc()
        h = C.c_void_p()
        self._check(lib().storm_cuda_create(C.byref(self.desc), C.byref(h)), handle=None)
        self.h = h
        self.n = problem.ncells

    def close(self):
        if getattr(self, "h", None):
            lib().storm_cuda_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc, handle="self"):
        if rc == A.STORM_OK:
            return
        derr, cell, part = C.c_int32(), C.c_uint64(), C.c_uint64()
        msg = C.create_string_buffer(512)
        hh = self.h if handle == "self" else None
        if hh:
            lib().storm_cuda_last_error(hh, C.byref(derr), C.byref(cell), C.byref(part), msg, 512)
        raise StormError(rc, msg.value.decode() or lib().storm_cuda_status_string(rc).decode(), derr.value,
                         cell.value, part.value)

    # ---------------------------------------------------------------- shards
    def set_sharding(self, shards, lo, hi, exchange=None):
        """Hold particle shards [lo, hi) of `shards` (storm_cuda_set_sharding).
        `exchange(ptr, count, stream)` sums `count` float64 values at device
        address `ptr` in place over every rank, ordered on the CUDA stream
        `stream`; None when this handle holds every shard.  See
        `torch_exchange` for the NCCL one."""
        if exchange is None:
            cb = A.ExchangeFn()
        else:
            def call(user, values, count, stream):
                try:
                    exchange(C.cast(values, C.c_void_p).value, int(count), stream or 0)
                    return 0
                except Exception:   # the engine fails the step with STORM_ERR_INVALID_ARG
                    import traceback
                    traceback.print_exc()
                    return 1
            cb = A.ExchangeFn(call)
        self._exchange = cb   # the callback must outlive the handle's steps
        self._check(lib().storm_cuda_set_sharding(self.h, shards, lo, hi, cb, None))

    # ---------------------------------------------------------------- step
    def step(self, dt=None):
        st = A.StormStepStats()
        self._check(lib().storm_cuda_step(self.h, self.problem.dt if dt is None else dt, C.byref(st)))
        return st.as_dict()

    def phase(self, name, dt=None):
        dt = self.problem.dt if dt is None else dt
        L = lib()
        if name in ("begin", "prestep", "emit", "poststep"):
            self._check(getattr(L, "storm_cuda_phase_" + name)(self.h, dt))
        else:
            self._check(getattr(L, "storm_cuda_phase_" + name)(self.h))

    def stats(self):
        st = A.StormStepStats()
        self._check(lib().storm_cuda_phase_stats(self.h, C.byref(st)))
        return st.as_dict()

    # ---------------------------------------------------------------- state
    def census_count(self):
        n = C.c_uint64()
        self._check(lib().storm_cuda_census_count(self.h, C.byref(n)))
        return n.value

    def census(self, out=None):
        """The census as host particles; with `out` (e.g. Particles.pinned) the
        census is written into its first n slots and a view of them returned."""
        n = self.census_count()
        p = Particles(n) if out is None else out.view(n)
        s = p.soa()
        cnt = C.c_uint64()
        self._check(lib().storm_cuda_get_census(self.h, C.byref(s), n, C.byref(cnt)))
        return p

    def bank(self):
        """The transport bank after phase('emit'): census then source packets."""
        cnt = C.c_uint64()
        self._check(lib().storm_cuda_get_bank(self.h, None, 0, C.byref(cnt)))
        p = Particles(cnt.value)
        s = p.soa()
        self._check(lib().storm_cuda_get_bank(self.h, C.byref(s), cnt.value, C.byref(cnt)))
        return p

    def step_host(self, census, out, dt=None, step_fields=False):
        """One step with the census on the host (storm_cuda_step_host): `census`
        goes in, the new census comes back into `out` (e.g. Particles.pinned),
        the upload overlapping the step's work that does not need it.  Without
        step_fields, time_left and initial_weight are neither sent nor read
        back (every step sets them).  Returns (stats, view of out)."""
        if not step_fields:
            v = census.view(census.n)
            v.time_left = v.initial_weight = None
            census = v
            o = out.view(out.n)
            o.time_left = o.initial_weight = None
            out = o
        sin, sout = census.soa(), out.soa()
        st = A.StormStepStats()
        cnt = C.c_uint64()
        self._check(lib().storm_cuda_step_host(self.h, self.problem.dt if dt is None else dt, C.byref(sin),
                                                C.byref(sout), out.n, C.byref(cnt), C.byref(st)))
        if cnt.value > out.n:
            raise ValueError(f"census of {cnt.value} particles does not fit the {out.n} of out")
        return st.as_dict(), out.view(cnt.value)

    def set_census(self, p, step_fields=True):
        """Replace the census.  step_fields=False leaves out time_left and
        initial_weight, which the next step sets itself."""
        if not step_fields:
            v = p.view(p.n)
            v.time_left = v.initial_weight = None
            p = v
        s = p.soa()
        self._check(lib().storm_cuda_set_census(self.h, C.byref(s)))

    def population_control(self, p):
        """CombPopulationControl::activate on host particles; returns the new census."""
        s = p.soa()
        self._check(lib().storm_cuda_population_control(self.h, C.byref(s)))
        return self.census()

    def temperature(self, out=None):
        """Material temperatures into `out` (or a new array)."""
        out = np.zeros(self.n) if out is None else out
        null = C.POINTER(C.c_double)()
        self._check(lib().storm_cuda_get_cell_arrays(self.h, A.ptr(out), null, null, null, null, null,
                                                      C.POINTER(C.c_uint64)()))
        return out

    def cells(self):
        keys = ("temperature", "internal_energy", "erad_time_avg", "erad_census", "sigma_a", "fleck")
        out = {k: np.zeros(self.n) for k in keys}
        segs = np.zeros(self.n, np.uint64)
        self._check(lib().storm_cuda_get_cell_arrays(self.h, *[A.ptr(out[k]) for k in keys], A.ptr(segs, C.c_uint64)))
        out["segments"] = segs
        return out

    def set_cell_state(self, temperature=None, internal_energy=None, cell_internal_energy=None):
        arr = [None if a is None else np.ascontiguousarray(a, float)
               for a in (temperature, internal_energy, cell_internal_energy)]
        self._check(lib().storm_cuda_set_cell_state(self.h, *[A.ptr(a) for a in arr]))

    def set_cell_physics(self, sigma_a=None, sigma_s=None, fleck=None):
        arr = [None if a is None else np.ascontiguousarray(a, float) for a in (sigma_a, sigma_s, fleck)]
        self._check(lib().storm_cuda_set_cell_physics(self.h, *[A.ptr(a) for a in arr]))

    def set_opacity_tables(self, sigma_a=None, sigma_s=None):
        """Per-cell opacity plug-in values for the next prestep (table opacity kinds)."""
        arr = [None if a is None else np.ascontiguousarray(a, float) for a in (sigma_a, sigma_s)]
        self._check(lib().storm_cuda_set_opacity_tables(self.h, *[A.ptr(a) for a in arr]))

    def set_cell_motion(self, velocity=None, momentum=None):
        """Cell velocities / momenta, (ncells, 3) each (handles with moving material)."""
        arr = [None if a is None else np.ascontiguousarray(a, float).reshape(-1) for a in (velocity, momentum)]
        self._check(lib().storm_cuda_set_cell_motion(self.h, *[A.ptr(a) for a in arr]))

    def cell_motion(self):
        """(velocity, momentum), (ncells, 3) each."""
        v = np.zeros(3 * self.n)
        m = np.zeros(3 * self.n)
        self._check(lib().storm_cuda_get_cell_motion(self.h, A.ptr(v), A.ptr(m)))
        return v.reshape(-1, 3), m.reshape(-1, 3)

    def group_tallies(self):
        """Group time averages of the last step (problems with
        with_eg_time_avg): (ncells, groups)."""
        G = self.problem.groups
        out = np.zeros(self.n * G)
        self._check(lib().storm_cuda_get_group_tallies(self.h, A.ptr(out)))
        return out.reshape(self.n, G)

    def beginning_counts(self):
        """Particles per cell when the last step's transport began (handles with
        per-cell counters)."""
        out = np.zeros(self.n, np.uint64)
        self._check(lib().storm_cuda_get_beginning_counts(self.h, A.ptr(out, C.c_uint64)))
        return out

    def checkpoint(self):
        """The handle's step-to-step state (census bank, cell state, face
        temperatures, step counter) as bytes."""
        n = C.c_uint64()
        self._check(lib().storm_cuda_checkpoint_size(self.h, C.byref(n)))
        buf = np.empty(n.value, np.uint8)
        self._check(lib().storm_cuda_checkpoint_save(self.h, buf.ctypes.data, n.value))
        return buf.tobytes()

    def restore(self, blob):
        """Load a checkpoint taken from a handle of the same problem."""
        buf = np.frombuffer(blob, np.uint8)
        self._check(lib().storm_cuda_checkpoint_load(self.h, buf.ctypes.data, len(buf)))

    def set_face_temperature(self, face, T):
        self._check(lib().storm_cuda_set_face_temperature(self.h, face, T))

    def emission(self):
        c = np.zeros(self.n, np.uint64)
        e = np.zeros(self.n)
        self._check(lib().storm_cuda_get_emission(self.h, A.ptr(c, C.c_uint64), A.ptr(e)))
        return c, e

    # ---------------------------------------------------------------- parity
    def replay(self, batch):
        """batch: object with .struct (StormReplayBatch) and host arrays."""
        self._check(lib().storm_cuda_replay_segments(self.h, C.byref(batch.struct)))
        return batch

    def rw_tables(self):
        tau, s, r = np.zeros(1024), np.zeros(1024), np.zeros(1024 * 256)
        self._check(lib().storm_cuda_get_random_walk_tables(self.h, A.ptr(tau), A.ptr(s), A.ptr(r)))
        return tau, s, r.reshape(1024, 256)

    def rw_sample(self, xi_leak, tau, xi_rad):
        n = len(xi_leak)
        leak, rad = np.zeros(n), np.zeros(n)
        a = [np.ascontiguousarray(v, float) for v in (xi_leak, tau, xi_rad)]
        self._check(lib().storm_cuda_random_walk_sample(self.h, n, A.ptr(a[0]), A.ptr(a[1]), A.ptr(a[2]),
                                                        A.ptr(leak), A.ptr(rad)))
        return leak, rad

    # ---------------------------------------------------------------- diagnostics
    def memory_bytes(self):
        b = C.c_uint64()
        self._check(lib().storm_cuda_memory_bytes(self.h, C.byref(b)))
        return b.value

    def launches(self):
        b = C.c_uint64()
        self._check(lib().storm_cuda_launch_count(self.h, C.byref(b)))
        return b.value

    def set_profiling(self, on=True):
        self._check(lib().storm_cuda_set_profiling(self.h, int(on)))

    def transport_timing(self, reset=False):
        ms, n, s = C.c_double(), C.c_uint64(), C.c_uint64()
        self._check(lib().storm_cuda_transport_timing(self.h, C.byref(ms), C.byref(n), C.byref(s), int(reset)))
        return {"kernel_ms": ms.value, "launches": n.value, "segments": s.value}

    def set_transport_variant(self, min_blocks_per_sm, waves=4):
        self._check(lib().storm_cuda_set_transport_variant(self.h, min_blocks_per_sm, waves))

    def set_transport_mode(self, refill=True, burst=4):
        self._check(lib().storm_cuda_set_transport_mode(self.h, int(refill), burst))

    def autotune_transport(self, steps_per_candidate=1):
        """Tune the refill burst over the next 10 * steps_per_candidate steps
        (storm_cuda_autotune_transport); 0 stops a tuning in progress."""
        self._check(lib().storm_cuda_autotune_transport(self.h, steps_per_candidate))

    def transport_burst(self):
        """(burst in use, tuning in progress)."""
        b, t = C.c_uint32(), C.c_int()
        self._check(lib().storm_cuda_transport_burst(self.h, C.byref(b), C.byref(t)))
        return b.value, bool(t.value)

    def set_segments_per_visit(self, k):
        self._check(lib().storm_cuda_set_segments_per_visit(self.h, k))


def device_array(ptr, count, device=None):
    """A torch float64 tensor over `count` doubles of device memory at `ptr`
    (no copy), through the CUDA array interface."""
    import torch

    class _Buf:
        pass
    b = _Buf()
    b.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                  "strides": None, "stream": None}
    return torch.as_tensor(b, device=device if device is not None else torch.device("cuda",
                                                                                      torch.cuda.current_device()))


def torch_exchange(group=None):
    """The exchange of a sharded engine over torch.distributed: an in-place
    sum all-reduce (NCCL across GPUs) of the engine's buffer, ordered on the
    engine's stream."""
    import torch
    import torch.distributed as dist

    def exchange(ptr, count, stream):
        t = device_array(ptr, count)
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return exchange


class Server:
    """Many independent problems on one GPU (storm_server_*): requests queue,
    are admitted by slots and an HBM budget, and advance concurrently."""

    def __init__(self, max_active=6, workers=3, hbm_budget_bytes=0, device=0):
        cfg = A.StormServerConfig(device, max_active, workers, 0, hbm_budget_bytes)
        h = C.c_void_p()
        rc = lib().storm_server_create(C.byref(cfg), C.byref(h))
        if rc != A.STORM_OK:
            raise StormError(rc, lib().storm_cuda_status_string(rc).decode())
        self.h = h
        self._keep = {}   # ticket -> (descriptor, problem, temperature buffer)

    def submit(self, problem, steps, dt=None, want_temperature=True):
        desc = problem.to_desc()
        T = np.zeros(problem.ncells) if want_temperature else None
        t = C.c_uint64()
        rc = lib().storm_server_submit(self.h, C.byref(desc), steps, problem.dt if dt is None else dt,
                                       A.ptr(T) if T is not None else None, C.byref(t))
        if rc != A.STORM_OK:
            raise StormError(rc, lib().storm_cuda_status_string(rc).decode())
        self._keep[t.value] = (desc, problem, T)
        return t.value

    def poll(self, capacity=1024):
        buf = (A.StormRequestResult * capacity)()
        n = C.c_uint32()
        lib().storm_server_poll(self.h, buf, capacity, C.byref(n))
        out = []
        for k in range(n.value):
            r = buf[k].as_dict()
            keep = self._keep.pop(r["ticket"], None)
            r["temperature"] = keep[2] if keep else None
            out.append(r)
        return out

    def drain(self):
        lib().storm_server_drain(self.h)

    def stats(self):
        st = A.StormServerStats()
        lib().storm_server_stats(self.h, C.byref(st))
        return st.as_dict()

    def close(self):
        if getattr(self, "h", None):
            lib().storm_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
