"""Test infrastructure only: ctypes wrapper of oracle/_ref/liboracle.so, the C
restatement of the reference's gray IMC path (oracle/imc_oracle.c).  Used by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker;
never by the product."""
import ctypes as C
import os
import numpy as np

from storm_b200 import _abi as A
from .ref import Particles

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "liboracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        vp, dp = C.c_void_p, C.POINTER(C.c_double)
        u64p, u32p = C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.POINTER(A.StormProblemDesc)]
        L.orc_destroy.argtypes = [vp]
        for f in ("orc_phase_begin", "orc_phase_prestep", "orc_phase_emit", "orc_phase_poststep"):
            getattr(L, f).argtypes = [vp, C.c_double]
        for f in ("orc_phase_transport", "orc_phase_comb"):
            getattr(L, f).argtypes = [vp]
        L.orc_step.argtypes = [vp, C.c_double, C.POINTER(A.StormStepStats)]
        L.orc_phase_stats.argtypes = [vp, C.POINTER(A.StormStepStats)]
        L.orc_set_census.argtypes = [vp, C.POINTER(A.StormParticlesSoA)]
        L.orc_census_count.restype = C.c_uint64
        L.orc_census_count.argtypes = [vp]
        L.orc_get_census.argtypes = [vp, C.POINTER(A.StormParticlesSoA)]
        L.orc_bank_count.restype = C.c_uint64
        L.orc_bank_count.argtypes = [vp]
        L.orc_get_bank.argtypes = [vp, C.POINTER(A.StormParticlesSoA)]
        L.orc_get_cell_arrays.argtypes = [vp, dp, dp, dp, dp, dp, dp, u64p]
        L.orc_set_cell_physics.argtypes = [vp, dp, dp, dp]
        L.orc_get_emission.argtypes = [vp, u64p, dp]
        L.orc_set_face_temperature.argtypes = [vp, C.c_int, C.c_double]
        L.orc_last_error.argtypes = [vp, C.POINTER(C.c_int32), u64p, u64p]
        L.orc_replay_segments.argtypes = [vp, C.POINTER(A.StormReplayBatch)]
        L.orc_rw_tables.argtypes = [dp, dp, dp]
        L.orc_rw_sample_leak.restype = C.c_double
        L.orc_rw_sample_leak.argtypes = [C.c_double]
        L.orc_rw_sample_radius.restype = C.c_double
        L.orc_rw_sample_radius.argtypes = [C.c_double, C.c_double]
        L.orc_rw_survival.restype = C.c_double
        L.orc_rw_survival.argtypes = [C.c_double]
        L.orc_rw_radial_cdf.restype = C.c_double
        L.orc_rw_radial_cdf.argtypes = [C.c_double, C.c_double]
        L.orc_sample_in_cell.argtypes = [vp, C.c_uint32, dp, dp]
        L.orc_point_on_face.argtypes = [vp, C.c_uint64, dp, dp]
        L.orc_isotropic.argtypes = [dp, C.c_double, dp]
        L.orc_philox4x32_10.argtypes = [u32p, u32p, u32p]
        L.orc_uniform.restype = C.c_double
        L.orc_uniform.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_set_sharding.argtypes = [vp, C.c_uint32, C.c_uint32, C.c_uint32, A.ExchangeFn, vp]
        L.orc_comb_key.restype = C.c_uint32
        L.orc_comb_key.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_int]
        _lib = L
    return _lib


class Oracle:
    def __init__(self, problem):
        self.problem = problem
        self.desc = problem.to_desc()
        self.h = lib().orc_create(C.byref(self.desc))
        self.n = problem.ncells

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _rc(self, rc, what):
        if rc != 0:
            d, c, p = C.c_int32(), C.c_uint64(), C.c_uint64()
            lib().orc_last_error(self.h, C.byref(d), C.byref(c), C.byref(p))
            raise RuntimeError(f"oracle {what} failed: {A.DERR_NAMES.get(d.value, d.value)} cell={c.value} "
                               f"particle={p.value}")

    def set_sharding(self, shards, lo, hi, exchange=None):
        """Hold particle shards [lo, hi) of `shards`; `exchange(values)` sums a
        float64 numpy array in place over every rank (None: this instance holds
        every shard)."""
        if exchange is None:
            cb = A.ExchangeFn()
        else:
            def call(user, values, count, stream):
                try:
                    exchange(np.ctypeslib.as_array(values, shape=(count,)))
                    return 0
                except Exception:   # reported to the oracle as a failed exchange
                    return 1
            cb = A.ExchangeFn(call)
        self._exchange = cb
        self._rc(lib().orc_set_sharding(self.h, shards, lo, hi, cb, None), "set_sharding")

    def step(self, dt=None):
        st = A.StormStepStats()
        self._rc(lib().orc_step(self.h, self.problem.dt if dt is None else dt, C.byref(st)), "step")
        return st.as_dict()

    def phase(self, name, dt=None):
        L = lib()
        dt = self.problem.dt if dt is None else dt
        if name in ("begin", "prestep", "emit", "poststep"):
            self._rc(getattr(L, "orc_phase_" + name)(self.h, dt), name)
        else:
            self._rc(getattr(L, "orc_phase_" + name)(self.h), name)

    def stats(self):
        st = A.StormStepStats()
        lib().orc_phase_stats(self.h, C.byref(st))
        return st.as_dict()

    def set_census(self, p):
        s = p.soa()
        lib().orc_set_census(self.h, C.byref(s))

    def census(self):
        n = lib().orc_census_count(self.h)
        p = Particles(n)
        s = p.soa()
        lib().orc_get_census(self.h, C.byref(s))
        return p

    def bank(self):
        n = lib().orc_bank_count(self.h)
        p = Particles(n)
        s = p.soa()
        lib().orc_get_bank(self.h, C.byref(s))
        return p

    def cells(self):
        n = self.n
        keys = ("temperature", "internal_energy", "erad_time_avg", "erad_census", "sigma_a", "fleck")
        out = {k: np.zeros(n) for k in keys}
        segs = np.zeros(n, dtype=np.uint64)
        lib().orc_get_cell_arrays(self.h, *[A.ptr(out[k]) for k in keys], A.ptr(segs, C.c_uint64))
        out["segments"] = segs
        return out

    def set_cell_physics(self, sigma_a, sigma_s, fleck):
        lib().orc_set_cell_physics(self.h, A.ptr(np.ascontiguousarray(sigma_a, float)),
                                   A.ptr(np.ascontiguousarray(sigma_s, float)),
                                   A.ptr(np.ascontiguousarray(fleck, float)))

    def emission(self):
        c = np.zeros(self.n, np.uint64)
        e = np.zeros(self.n)
        lib().orc_get_emission(self.h, A.ptr(c, C.c_uint64), A.ptr(e))
        return c, e

    def set_face_temperature(self, face, T):
        lib().orc_set_face_temperature(self.h, face, T)

    def replay(self, batch):
        lib().orc_replay_segments(self.h, C.byref(batch.struct))
        return batch

    def sample_in_cell(self, cell, tape4):
        out = np.zeros(3)
        lib().orc_sample_in_cell(self.h, cell, A.ptr(np.ascontiguousarray(tape4, float)), A.ptr(out))
        return out

    def point_on_face(self, face, tape3):
        out = np.zeros(3)
        lib().orc_point_on_face(self.h, face, A.ptr(np.ascontiguousarray(tape3, float)), A.ptr(out))
        return out


def rw_tables():
    tau = np.zeros(1024)
    s = np.zeros(1024)
    r = np.zeros(1024 * 256)
    lib().orc_rw_tables(A.ptr(tau), A.ptr(s), A.ptr(r))
    return tau, s, r.reshape(1024, 256)


def isotropic(tape2, clight):
    out = np.zeros(3)
    lib().orc_isotropic(A.ptr(np.ascontiguousarray(tape2, float)), clight, A.ptr(out))
    return out


def philox(ctr, key):
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    o = np.zeros(4, np.uint32)
    lib().orc_philox4x32_10(A.ptr(c, C.c_uint32), A.ptr(k, C.c_uint32), A.ptr(o, C.c_uint32))
    return o


def uniform(seed, tag, step, pid, draw):
    return lib().orc_uniform(seed, tag, step, pid, draw)


class ReplayBatch:
    """Host buffers of a StormReplayBatch built from reference records."""
    IN = ("x", "y", "z", "vx", "vy", "vz", "time_left", "weight", "initial_weight")
    OUT_D = ("phys_x", "phys_y", "phys_z", "phys_vx", "phys_vy", "phys_vz", "phys_time_left", "phys_weight",
             "dep_material", "dep_erad", "mgr_x", "mgr_y", "mgr_z", "mgr_vx", "mgr_vy", "mgr_vz")

    def __init__(self, before, cell, tape_offset, tape_length, tape, frequency=None, momentum=False):
        n = len(cell)
        self.n = n
        self.arrays = {}
        for k, name in enumerate(self.IN):
            self.arrays[name] = np.ascontiguousarray(before[:, k])
        if frequency is not None:   # multigroup: frequency in and out
            self.arrays["frequency"] = np.ascontiguousarray(frequency, float)
            self.arrays["phys_frequency"] = np.zeros(n)
        if momentum:   # moving material: each segment's momentum deposit, 3 per item
            self.arrays["phys_momentum"] = np.zeros(3 * n)
        self.arrays["cell"] = np.ascontiguousarray(cell, np.uint32)
        self.arrays["tape_offset"] = np.ascontiguousarray(tape_offset, np.uint64)
        self.arrays["tape_length"] = np.ascontiguousarray(tape_length, np.uint32)
        self.arrays["tape"] = np.ascontiguousarray(tape, float)
        for name in self.OUT_D:
            self.arrays[name] = np.zeros(n)
        for name in ("phys_status", "mgr_status", "used_random_walk"):
            self.arrays[name] = np.zeros(n, np.int32)
        for name in ("phys_next_cell", "mgr_cell", "draws_used"):
            self.arrays[name] = np.zeros(n, np.uint32)
        s = A.StormReplayBatch()
        s.n = n
        for name, arr in self.arrays.items():
            ct = {np.dtype(np.float64): C.c_double, np.dtype(np.uint32): C.c_uint32,
                  np.dtype(np.int32): C.c_int32, np.dtype(np.uint64): C.c_uint64}[arr.dtype]
            setattr(s, name, A.ptr(arr, ct))
        self.struct = s

    def __getitem__(self, k):
        return self.arrays[k]
