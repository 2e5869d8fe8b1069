"""Test infrastructure only: ctypes wrapper of oracle/_ref/libstormref.so, the
reference's own serial IMC path (MonteCarloManagerSerial + RadiationIMC +
CombPopulationControl + boundaries) compiled here from the reference sources
against the stand-ins in oracle/shims (see oracle/ref_harness.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's reference / cpu_baseline
legs use this module, and only as the checker or the timed CPU baseline.
"""
import ctypes as C
import os
import numpy as np

from storm_b200 import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libstormref.so")

BOUNDARY_DESCRIPTOR = 0
BOUNDARY_RIGID = 1
BOUNDARY_VACUUM = 2
BOUNDARY_SIDE_TEMPERATURE = 3
BOUNDARY_TWO_SIDES_TEMPERATURE = 4


class RefStepOut(C.Structure):
    _fields_ = [("initial", C.c_uint64), ("prestep", C.c_uint64), ("start", C.c_uint64), ("end", C.c_uint64),
                ("segments", C.c_uint64), ("rw_steps", C.c_uint64), ("wall_seconds", C.c_double),
                ("escaped_energy", C.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        u64p = C.POINTER(C.c_uint64)
        u32p = C.POINTER(C.c_uint32)
        i32p = C.POINTER(C.c_int32)
        L.ref_create.restype = vp
        L.ref_create.argtypes = [C.POINTER(A.StormProblemDesc), C.c_int, C.c_char_p, C.c_size_t]
        L.ref_destroy.argtypes = [vp]
        L.ref_set_face_temperature.argtypes = [vp, C.c_int, C.c_double]
        L.ref_last_error.restype = C.c_char_p
        L.ref_last_error.argtypes = [vp]
        L.ref_step.argtypes = [vp, C.c_double, C.POINTER(RefStepOut)]
        L.ref_prestep_only.argtypes = [vp, C.c_double, u64p]
        L.ref_census_count.restype = C.c_uint64
        L.ref_census_count.argtypes = [vp]
        L.ref_get_census.argtypes = [vp, C.POINTER(A.StormParticlesSoA)]
        L.ref_set_census.argtypes = [vp, C.POINTER(A.StormParticlesSoA)]
        L.ref_get_cells.argtypes = [vp, dp, dp, dp, dp, dp, dp, u64p]
        L.ref_get_emission.argtypes = [vp, u64p]
        L.ref_record_begin.argtypes = [vp, C.c_uint64]
        L.ref_record_end.argtypes = [vp]
        L.ref_record_count.restype = C.c_uint64
        L.ref_record_count.argtypes = [vp]
        L.ref_record_tape_size.restype = C.c_uint64
        L.ref_record_tape_size.argtypes = [vp]
        L.ref_record_get.argtypes = [vp, u64p, u32p, dp, dp, i32p, u64p, dp, u64p, u32p, i32p, dp]
        L.ref_record_get_frequency.argtypes = [vp, dp, dp]
        L.ref_mg_thermal_energy.argtypes = [vp, C.c_uint64, u32p, dp, dp]
        L.ref_rw_sample.argtypes = [C.c_uint64, dp, dp, dp, dp, dp]
        L.ref_rw_functions.argtypes = [C.c_uint64, dp, dp, dp, dp]
        L.ref_sample_in_cell.argtypes = [vp, C.c_uint64, u32p, C.c_uint64, dp, dp, u32p]
        L.ref_isotropic.argtypes = [C.c_uint64, C.c_uint64, dp, dp]
        L.ref_point_on_face.argtypes = [vp, C.c_uint64, u64p, dp, dp]
        L.ref_comb.argtypes = [vp, C.POINTER(A.StormParticlesSoA), C.POINTER(A.StormParticlesSoA), u64p]
        L.ref_advance_face_stream.argtypes = [vp, C.c_uint64]
        L.ref_record_get_momentum.argtypes = [vp, dp]
        L.ref_get_motion.argtypes = [vp, dp, dp]
        L.ref_get_group_tallies.argtypes = [vp, dp]
        L.ref_units.argtypes = [dp]
        L.ref_planck_integral.restype = C.c_double
        L.ref_planck_integral.argtypes = [C.c_double, C.c_double]
        _lib = L
    return _lib


class Particles:
    """Host struct-of-arrays particle buffer."""
    FIELDS = ("x", "y", "z", "vx", "vy", "vz", "time_left", "weight", "initial_weight")

    def __init__(self, n):
        for f in self.FIELDS:
            setattr(self, f, np.zeros(n))
        self.cell = np.zeros(n, dtype=np.uint32)
        self.id = np.zeros(n, dtype=np.uint64)
        self.n = n
        self.frequency = np.zeros(n)   # photon energy (multigroup)

    def soa(self):
        """Struct of pointers; every field is made contiguous first (the C side
        reads plain arrays)."""
        for f in self.FIELDS:
            setattr(self, f, np.ascontiguousarray(getattr(self, f), dtype=np.float64))
        self.cell = np.ascontiguousarray(self.cell, dtype=np.uint32)
        self.id = np.ascontiguousarray(self.id, dtype=np.uint64)
        s = A.StormParticlesSoA()
        for f in self.FIELDS:
            setattr(s, f, A.ptr(getattr(self, f)))
        s.cell = A.ptr(self.cell, C.c_uint32)
        s.id = A.ptr(self.id, C.c_uint64)
        if getattr(self, "frequency", None) is not None:
            self.frequency = np.ascontiguousarray(self.frequency, dtype=np.float64)
            s.frequency = A.ptr(self.frequency)
        s.count = self.n
        return s

    def take(self, idx):
        p = Particles(len(idx))
        for f in self.FIELDS + ("cell", "id", "frequency"):
            setattr(p, f, np.ascontiguousarray(getattr(self, f)[idx]))
        return p


class Reference:
    """One reference problem instance (grid, cells, plug-ins, serial manager)."""

    def __init__(self, problem, boundary_kind=BOUNDARY_DESCRIPTOR):
        self.problem = problem
        self.desc = problem.to_desc()
        err = C.create_string_buffer(512)
        self.h = lib().ref_create(C.byref(self.desc), boundary_kind, err, 512)
        if not self.h:
            raise RuntimeError("ref_create failed: " + err.value.decode())
        self.n = problem.ncells

    def close(self):
        if self.h:
            lib().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError("reference error: " + lib().ref_last_error(self.h).decode())

    def set_face_temperature(self, face, T):
        self._check(lib().ref_set_face_temperature(self.h, face, T))

    def step(self, dt=None):
        out = RefStepOut()
        self._check(lib().ref_step(self.h, self.problem.dt if dt is None else dt, C.byref(out)))
        return out.as_dict()

    def advance_face_stream(self, calls):
        """Move the process-wide RandomPointOnFace stream forward by `calls`
        points (independent face-source positions for batch runs)."""
        self._check(lib().ref_advance_face_stream(self.h, calls))

    def prestep_only(self, dt=None):
        n = C.c_uint64()
        self._check(lib().ref_prestep_only(self.h, self.problem.dt if dt is None else dt, C.byref(n)))
        return n.value

    def census(self):
        n = lib().ref_census_count(self.h)
        p = Particles(n)
        s = p.soa()
        lib().ref_get_census(self.h, C.byref(s))
        return p

    def set_census(self, p):
        s = p.soa()
        lib().ref_set_census(self.h, C.byref(s))

    def cells(self):
        n = self.n
        out = {k: np.zeros(n) for k in ("temperature", "internal_energy", "erad_time_avg", "erad_census",
                                         "sigma_a", "fleck")}
        segs = np.zeros(n, dtype=np.uint64)
        lib().ref_get_cells(self.h, *[A.ptr(out[k]) for k in ("temperature", "internal_energy", "erad_time_avg",
                                                                 "erad_census", "sigma_a", "fleck")],
                            A.ptr(segs, C.c_uint64))
        out["segments"] = segs
        return out

    def emission_counts(self):
        c = np.zeros(self.n, dtype=np.uint64)
        lib().ref_get_emission(self.h, A.ptr(c, C.c_uint64))
        return c

    def record_begin(self, max_records):
        lib().ref_record_begin(self.h, max_records)

    def record_end(self):
        lib().ref_record_end(self.h)

    def records(self):
        L = lib()
        n = L.ref_record_count(self.h)
        t = L.ref_record_tape_size(self.h)
        r = {
            "id": np.zeros(n, np.uint64), "cell": np.zeros(n, np.uint32), "before": np.zeros((n, 9)),
            "after": np.zeros((n, 8)), "status": np.zeros(n, np.int32), "next": np.zeros(n, np.uint64),
            "tallies": np.zeros((n, 4)), "tape_offset": np.zeros(n, np.uint64), "tape_length": np.zeros(n, np.uint32),
            "used_rw": np.zeros(n, np.int32), "tape": np.zeros(max(t, 1)),
        }
        L.ref_record_get(self.h, A.ptr(r["id"], C.c_uint64), A.ptr(r["cell"], C.c_uint32), A.ptr(r["before"]),
                         A.ptr(r["after"]), A.ptr(r["status"], C.c_int32), A.ptr(r["next"], C.c_uint64),
                         A.ptr(r["tallies"]), A.ptr(r["tape_offset"], C.c_uint64),
                         A.ptr(r["tape_length"], C.c_uint32), A.ptr(r["used_rw"], C.c_int32), A.ptr(r["tape"]))
        r["freq_before"] = np.zeros(n)
        r["freq_after"] = np.zeros(n)
        L.ref_record_get_frequency(self.h, A.ptr(r["freq_before"]), A.ptr(r["freq_after"]))
        r["momentum"] = np.zeros((n, 3))
        L.ref_record_get_momentum(self.h, A.ptr(r["momentum"]))
        return r

    def motion(self):
        """Cell velocities and momenta, (ncells, 3) each."""
        v = np.zeros((self.n, 3))
        m = np.zeros((self.n, 3))
        lib().ref_get_motion(self.h, A.ptr(v), A.ptr(m))
        return v, m

    def group_tallies(self):
        """getEgTimeAvg after the last step (withEgTimeAvg), (ncells, groups)."""
        G = self.problem.groups
        out = np.zeros(self.n * G)
        if lib().ref_get_group_tallies(self.h, A.ptr(out)) != 0:
            raise RuntimeError("group time averages not kept")
        return out.reshape(self.n, G)

    def thermal_energy(self, cells, xi):
        """The opacity plug-in's GetThermalEnergy at given uniforms (multigroup)."""
        cells = np.ascontiguousarray(cells, np.uint32)
        xi = np.ascontiguousarray(xi, float)
        out = np.zeros(len(xi))
        self._check(lib().ref_mg_thermal_energy(self.h, len(xi), A.ptr(cells, C.c_uint32), A.ptr(xi), A.ptr(out)))
        return out

    def sample_in_cell(self, cells, seed):
        cells = np.ascontiguousarray(cells, np.uint32)
        n = len(cells)
        pos = np.zeros((n, 3))
        tape = np.zeros(8 * n)
        nd = np.zeros(n, np.uint32)
        lib().ref_sample_in_cell(self.h, n, A.ptr(cells, C.c_uint32), seed, A.ptr(pos), A.ptr(tape),
                                 A.ptr(nd, C.c_uint32))
        return pos, tape[: int(nd.sum())], nd

    def point_on_face(self, faces):
        faces = np.ascontiguousarray(faces, np.uint64)
        n = len(faces)
        pos = np.zeros((n, 3))
        tape = np.zeros(3 * n)
        lib().ref_point_on_face(self.h, n, A.ptr(faces, C.c_uint64), A.ptr(pos), A.ptr(tape))
        return pos, tape

    def comb(self, p):
        s_in = p.soa()
        cap = max(4 * p.n, 1024) + 10 * self.problem.comb_nmin * self.n * 20
        out = Particles(cap)
        s_out = out.soa()
        cnt = C.c_uint64()
        self._check(lib().ref_comb(self.h, C.byref(s_in), C.byref(s_out), C.byref(cnt)))
        return out.take(np.arange(cnt.value))


def rw_sample(xi_leak, tau, xi_rad):
    n = len(xi_leak)
    leak = np.zeros(n)
    rad = np.zeros(n)
    lib().ref_rw_sample(n, A.ptr(np.ascontiguousarray(xi_leak, float)), A.ptr(np.ascontiguousarray(tau, float)),
                        A.ptr(np.ascontiguousarray(xi_rad, float)), A.ptr(leak), A.ptr(rad))
    return leak, rad


def rw_functions(tau, x):
    n = len(tau)
    s = np.zeros(n)
    c = np.zeros(n)
    lib().ref_rw_functions(n, A.ptr(np.ascontiguousarray(tau, float)), A.ptr(np.ascontiguousarray(x, float)),
                           A.ptr(s), A.ptr(c))
    return s, c


def isotropic(n, seed):
    v = np.zeros((n, 3))
    tape = np.zeros(2 * n)
    lib().ref_isotropic(n, seed, A.ptr(v), A.ptr(tape))
    return v, tape


def units():
    out = np.zeros(6)
    lib().ref_units(A.ptr(out))
    return dict(zip(("clight", "arad", "sigma_sb", "kev_kelvin", "k_boltz", "kev"), out))


def planck_integral(a, b):
    return lib().ref_planck_integral(a, b)
