"""ctypes mirror of include/storm_cuda.h (the engine's C ABI).

Field order and types follow the header exactly; tests/test_abi.py checks the
sizes against the compiled library.
"""
import ctypes as C

ABI_VERSION = 8

STORM_OK = 0
STATUS_NAMES = {
    0: "STORM_OK", 1: "STORM_ERR_INVALID_ARG", 2: "STORM_ERR_CUDA", 3: "STORM_ERR_OOM",
    4: "STORM_ERR_DEVICE", 5: "STORM_ERR_CAPACITY", 6: "STORM_ERR_UNSUPPORTED", 7: "STORM_ERR_NO_DEVICE",
}
DERR_NAMES = {
    0: "NONE", 1: "NO_FACE", 2: "NOT_ON_BOUNDARY", 3: "FLECK", 4: "NEGATIVE_ENERGY", 5: "COMB_OUTSIDE",
    6: "COMB_WEIGHT", 7: "RW_SHRINK", 8: "HISTORY_CAP", 9: "BANK_OVERFLOW", 10: "TAPE_EXHAUSTED",
    11: "COMB_TOTAL",
}

PRECISION_FP64 = 0
PRECISION_FP32_TRACK = 1
FACE_REFLECT = 0
FACE_ESCAPE = 1
OPACITY_CELL_TABLE = 0
OPACITY_POWER_LAW = 1
OPACITY_MG_POWER = 2
COMB_PLAIN = 0
COMB_STRATIFIED = 1
STRAT_MAX_BINS = 64
EOS_LINEAR = 0
EOS_POWER_LAW = 1

_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_i32p = C.POINTER(C.c_int32)


class StormBoxFace(C.Structure):
    _fields_ = [
        ("action", C.c_int32),
        ("pad_", C.c_int32),
        ("source_temperature", C.c_double),
        ("packets_per_face", C.c_uint64),
    ]


class StormPolyMesh(C.Structure):
    _fields_ = [
        ("ncells", C.c_uint32), ("nfaces", C.c_uint32), ("nvertices", C.c_uint32), ("pad_", C.c_uint32),
        ("box", C.c_double * 6), ("points", _dp), ("volume", _dp),
        ("cell_face_offset", _u32p), ("cell_faces", _u32p), ("face_cells", _u32p),
        ("face_normal", _dp), ("face_cm", _dp), ("face_area", _dp),
        ("face_vertex_offset", _u32p), ("face_vertices", _u32p), ("vertices", _dp),
    ]


class StormProblemDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("precision", C.c_int32),
        ("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32),
        ("x_edges", _dp), ("y_edges", _dp), ("z_edges", _dp),
        ("temperature", _dp), ("mass", _dp), ("internal_energy", _dp), ("cell_internal_energy", _dp),
        ("opacity_kind", C.c_int32), ("eos_kind", C.c_int32),
        ("sigma_a", _dp), ("sigma_s", _dp),
        ("kP0", C.c_double), ("kR0", C.c_double), ("alpha", C.c_double), ("beta", C.c_double),
        ("t_floor", C.c_double), ("cap", C.c_double),
        ("density_factor", _dp),
        ("cv_per_mass", C.c_double),
        ("eos_f", C.c_double), ("eos_beta", C.c_double), ("eos_mu", C.c_double),
        ("faces", StormBoxFace * 6),
        ("escape_without_check", C.c_int32), ("pad0_", C.c_int32),
        ("new_photons_per_cell", C.c_uint64),
        ("with_random_walk", C.c_int32), ("no_hydro_feedback", C.c_int32),
        ("rw_min_cell_optical_depth", C.c_double), ("rw_min_particle_optical_depth", C.c_double),
        ("comb_enabled", C.c_int32), ("pad1_", C.c_int32),
        ("comb_nmin", C.c_uint64), ("comb_factor", C.c_double),
        ("clight", C.c_double), ("arad", C.c_double), ("sigma_sb", C.c_double), ("kev_kelvin", C.c_double),
        ("seed", C.c_uint64), ("capacity", C.c_uint64),
        ("segments_per_visit", C.c_uint32), ("max_rounds", C.c_uint32),
        ("per_cell_segment_counters", C.c_int32), ("device", C.c_int32),
        ("groups", C.c_uint32), ("mg_group_constant", C.c_int32), ("group_bounds", _dp),
        ("mg_p", C.c_double), ("mg_q", C.c_double), ("mg_s", C.c_double), ("k_boltz", C.c_double),
        ("with_ddmc", C.c_int32), ("ddmc_use_multigroup_pgrw", C.c_int32),
        ("ddmc_min_cell_optical_depth", C.c_double), ("ddmc_min_particle_optical_depth", C.c_double),
        ("comb_kind", C.c_int32), ("strat_bins", C.c_uint32), ("strat_bounds", _dp),
        ("strat_min_per_bin", C.c_uint64),
        ("mesh", C.POINTER(StormPolyMesh)),
        ("with_hydro", C.c_int32),
        ("pad2_", C.c_int32),
        ("cell_velocity", C.POINTER(C.c_double)),
        ("with_eg_time_avg", C.c_int32),
        ("reproducible_tallies", C.c_int32),
    ]


class StormParticlesSoA(C.Structure):
    _fields_ = [
        ("x", _dp), ("y", _dp), ("z", _dp),
        ("vx", _dp), ("vy", _dp), ("vz", _dp),
        ("time_left", _dp), ("weight", _dp), ("initial_weight", _dp),
        ("cell", _u32p), ("id", _u64p), ("count", C.c_uint64), ("frequency", _dp),
    ]


class StormStepStats(C.Structure):
    _fields_ = [
        ("census_in", C.c_uint64), ("emitted_cells", C.c_uint64), ("emitted_faces", C.c_uint64),
        ("census_out_pre_comb", C.c_uint64), ("census_out", C.c_uint64), ("segments", C.c_uint64),
        ("rw_steps", C.c_uint64), ("escaped", C.c_uint64), ("cutoff", C.c_uint64), ("rounds", C.c_uint64),
        ("energy_census_in", C.c_double), ("energy_emitted", C.c_double), ("energy_deposited", C.c_double),
        ("energy_escaped", C.c_double), ("energy_census_pre_comb", C.c_double), ("energy_census_out", C.c_double),
        ("energy_emission_debit", C.c_double), ("transport_ms", C.c_double), ("step_ms", C.c_double),
        ("emit_ms", C.c_double), ("comb_ms", C.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class StormReplayBatch(C.Structure):
    _fields_ = [
        ("n", C.c_uint64),
        ("x", _dp), ("y", _dp), ("z", _dp), ("vx", _dp), ("vy", _dp), ("vz", _dp),
        ("time_left", _dp), ("weight", _dp), ("initial_weight", _dp),
        ("cell", _u32p), ("tape_offset", _u64p), ("tape_length", _u32p), ("tape", _dp),
        ("phys_x", _dp), ("phys_y", _dp), ("phys_z", _dp), ("phys_vx", _dp), ("phys_vy", _dp), ("phys_vz", _dp),
        ("phys_time_left", _dp), ("phys_weight", _dp),
        ("phys_status", _i32p), ("phys_next_cell", _u32p),
        ("dep_material", _dp), ("dep_erad", _dp),
        ("mgr_x", _dp), ("mgr_y", _dp), ("mgr_z", _dp), ("mgr_vx", _dp), ("mgr_vy", _dp), ("mgr_vz", _dp),
        ("mgr_cell", _u32p), ("mgr_status", _i32p), ("draws_used", _u32p), ("used_random_walk", _i32p),
        ("frequency", _dp), ("phys_frequency", _dp), ("phys_momentum", _dp),
    ]


# StormExchangeFn: int (*)(void *user, double *values, uint64_t count, void *stream)
ExchangeFn = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double), C.c_uint64, C.c_void_p)


def ptr(arr, ctype=C.c_double):
    """ctypes pointer to a contiguous numpy array (or None)."""
    if arr is None:
        return None
    return arr.ctypes.data_as(C.POINTER(ctype))


class StormServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_active", C.c_uint32), ("workers", C.c_uint32), ("pad_", C.c_uint32),
                ("hbm_budget_bytes", C.c_uint64)]


class StormRequestResult(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("status", C.c_int32), ("steps", C.c_uint32), ("segments", C.c_uint64),
                ("device_bytes", C.c_uint64), ("queued_ms", C.c_double), ("active_ms", C.c_double),
                ("step_ms_p50", C.c_double), ("step_ms_p99", C.c_double), ("step_ms_max", C.c_double),
                ("device_ms", C.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class StormServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64), ("active", C.c_uint64),
                ("queued", C.c_uint64), ("segments", C.c_uint64), ("busy_ms", C.c_double),
                ("step_ms_p50", C.c_double), ("step_ms_p99", C.c_double), ("peak_device_bytes", C.c_uint64),
                ("budget_bytes", C.c_uint64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}
