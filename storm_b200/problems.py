"""Problem descriptors: the mesh, material, opacity/EOS plug-ins, boundary faces,
IMC parameters and comb settings of one IMC problem, packed into the C ABI's
StormProblemDesc.

The builders at the bottom produce the synthetic workloads the engine is
measured on (seeded, no external data):

* ``gray_slab``  -- 100x1x1 slab on [0,1]x[0,0.01]^2, x=0 face at 1 keV,
  vacuum at x=1, reflecting y/z, kappa_a = min(10 T_keV^-3, 1e6), constant cv.
* ``step_cube``  -- 64^3 unit cube, kappa_a = 1 (x<0.5) / 1000 (x>=0.5) 1/cm,
  hot face x=0 at 1 keV, vacuum elsewhere, Random Walk where kappa*dx > 10.
"""
import ctypes as C
from dataclasses import dataclass, field
import numpy as np

from . import _abi as A
from .units import UNITS


@dataclass
class BoxFace:
    action: int = A.FACE_REFLECT
    source_temperature: float = 0.0     # K
    packets_per_face: int = 0


@dataclass
class Problem:
    x_edges: np.ndarray
    y_edges: np.ndarray
    z_edges: np.ndarray
    temperature: np.ndarray             # K, per cell
    mass: np.ndarray                    # g
    internal_energy: np.ndarray         # erg (extensive)
    cell_internal_energy: np.ndarray = None
    opacity_kind: int = A.OPACITY_CELL_TABLE
    sigma_a: np.ndarray = None
    sigma_s: np.ndarray = None
    kP0: float = 0.0
    kR0: float = 0.0
    alpha: float = 0.0
    beta: float = 0.0
    t_floor: float = 1.0
    cap: float = 0.0
    density_factor: np.ndarray = None
    eos_kind: int = A.EOS_LINEAR
    cv_per_mass: float = 1.0
    eos_f: float = 1.0
    eos_beta: float = 1.0
    eos_mu: float = 0.0
    faces: list = field(default_factory=lambda: [BoxFace() for _ in range(6)])
    escape_without_check: bool = False
    new_photons_per_cell: int = 1
    with_random_walk: bool = False
    no_hydro_feedback: bool = False
    rw_min_cell_optical_depth: float = 25.0      # RadiationIMCParameters defaults
    rw_min_particle_optical_depth: float = 5.0
    comb_enabled: bool = True
    comb_nmin: int = 20
    comb_factor: float = 2.0
    seed: int = 42
    precision: int = A.PRECISION_FP64
    capacity: int = 0
    segments_per_visit: int = 0
    max_rounds: int = 0
    per_cell_segment_counters: bool = True
    device: int = 0
    dt: float = 1e-11
    name: str = "problem"
    # multigroup (groups >= 2): STORM_OPACITY_MG_POWER with sigma_a = sigma0 per cell
    groups: int = 0
    group_bounds: np.ndarray = None
    mg_group_constant: bool = False
    mg_p: float = 3.0
    mg_q: float = 0.0
    mg_s: float = 0.0
    # DDMC-style leakage (RadiationIMCParameters defaults)
    with_ddmc: bool = False
    ddmc_use_multigroup_pgrw: bool = False
    ddmc_min_cell_optical_depth: float = 15.0
    ddmc_min_particle_optical_depth: float = 5.0
    # population control: CombPopulationControl, or StratifiedCombPopulationControl with frequency bins
    comb_kind: int = A.COMB_PLAIN
    strat_bins: int = 1
    strat_bounds: np.ndarray = None
    strat_min_per_bin: int = 2

    # convex-polyhedral mesh (storm_b200.mesh.PolyMesh); None for the Cartesian grid
    mesh: object = None
    # moving material (withHydro): per-cell velocity [cm/s], shape (ncells, 3); None = at rest
    with_hydro: bool = False
    cell_velocity: np.ndarray = None
    # group time averages (withEgTimeAvg, multigroup problems): per cell and group
    with_eg_time_avg: bool = False
    # tallies summed in fixed point, so that runs repeat bit for bit
    reproducible_tallies: bool = False

    @property
    def shape(self):
        return (len(self.x_edges) - 1, len(self.y_edges) - 1, len(self.z_edges) - 1)

    @property
    def ncells(self):
        if self.mesh is not None:
            return self.mesh.ncells
        nx, ny, nz = self.shape
        return nx * ny * nz

    def cell_centers(self):
        """Cell centres with the grid's own arithmetic: 0.5*(e_i + e_{i+1});
        on a polyhedral mesh its mesh points."""
        if self.mesh is not None:
            return self.mesh.points[:, 0].copy(), self.mesh.points[:, 1].copy(), self.mesh.points[:, 2].copy()
        xc = 0.5 * (self.x_edges[:-1] + self.x_edges[1:])
        yc = 0.5 * (self.y_edges[:-1] + self.y_edges[1:])
        zc = 0.5 * (self.z_edges[:-1] + self.z_edges[1:])
        Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
        return X.ravel(), Y.ravel(), Z.ravel()

    def volumes(self):
        if self.mesh is not None:
            return self.mesh.volume.copy()
        dx = np.diff(self.x_edges)
        dy = np.diff(self.y_edges)
        dz = np.diff(self.z_edges)
        Z, Y, X = np.meshgrid(dz, dy, dx, indexing="ij")
        return ((X * Y) * Z).ravel()

    def to_desc(self):
        """Pack into a ctypes StormProblemDesc.  The returned object keeps the
        numpy arrays it points to alive (attribute ``_keep``)."""
        keep = []

        def arr(a, dtype=np.float64):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dtype)
            keep.append(a)
            return A.ptr(a)

        d = A.StormProblemDesc()
        d.abi_version = A.ABI_VERSION
        d.precision = self.precision
        nx, ny, nz = self.shape
        d.nx, d.ny, d.nz = nx, ny, nz
        d.x_edges = arr(self.x_edges)
        d.y_edges = arr(self.y_edges)
        d.z_edges = arr(self.z_edges)
        d.temperature = arr(self.temperature)
        d.mass = arr(self.mass)
        d.internal_energy = arr(self.internal_energy)
        d.cell_internal_energy = arr(self.cell_internal_energy)
        d.opacity_kind = self.opacity_kind
        d.eos_kind = self.eos_kind
        d.sigma_a = arr(self.sigma_a)
        d.sigma_s = arr(self.sigma_s)
        d.kP0, d.kR0, d.alpha, d.beta, d.t_floor, d.cap = self.kP0, self.kR0, self.alpha, self.beta, self.t_floor, self.cap
        d.density_factor = arr(self.density_factor)
        d.cv_per_mass = self.cv_per_mass
        d.eos_f, d.eos_beta, d.eos_mu = self.eos_f, self.eos_beta, self.eos_mu
        for k, f in enumerate(self.faces):
            d.faces[k].action = f.action
            d.faces[k].source_temperature = f.source_temperature
            d.faces[k].packets_per_face = f.packets_per_face
        d.escape_without_check = int(self.escape_without_check)
        d.new_photons_per_cell = self.new_photons_per_cell
        d.with_random_walk = int(self.with_random_walk)
        d.no_hydro_feedback = int(self.no_hydro_feedback)
        d.rw_min_cell_optical_depth = self.rw_min_cell_optical_depth
        d.rw_min_particle_optical_depth = self.rw_min_particle_optical_depth
        d.comb_enabled = int(self.comb_enabled)
        d.comb_nmin = self.comb_nmin
        d.comb_factor = self.comb_factor
        d.clight, d.arad, d.sigma_sb, d.kev_kelvin = (UNITS["clight"], UNITS["arad"], UNITS["sigma_sb"],
                                                      UNITS["kev_kelvin"])
        d.seed = self.seed
        d.capacity = self.capacity
        d.segments_per_visit = self.segments_per_visit
        d.max_rounds = self.max_rounds
        d.per_cell_segment_counters = int(self.per_cell_segment_counters)
        d.device = self.device
        d.groups = self.groups
        d.mg_group_constant = int(self.mg_group_constant)
        d.group_bounds = arr(self.group_bounds)
        d.mg_p, d.mg_q, d.mg_s = self.mg_p, self.mg_q, self.mg_s
        d.k_boltz = UNITS["k_boltz"]
        d.with_ddmc = int(self.with_ddmc)
        d.ddmc_use_multigroup_pgrw = int(self.ddmc_use_multigroup_pgrw)
        d.ddmc_min_cell_optical_depth = self.ddmc_min_cell_optical_depth
        d.ddmc_min_particle_optical_depth = self.ddmc_min_particle_optical_depth
        d.comb_kind = self.comb_kind
        d.strat_bins = self.strat_bins
        d.strat_bounds = arr(self.strat_bounds)
        d.strat_min_per_bin = self.strat_min_per_bin
        if self.mesh is not None:
            md = self.mesh.desc()
            keep.append(md)
            d.mesh = C.pointer(md)
        d.with_hydro = int(self.with_hydro)
        d.cell_velocity = arr(None if self.cell_velocity is None else np.asarray(self.cell_velocity).reshape(-1))
        d.with_eg_time_avg = int(self.with_eg_time_avg)
        d.reproducible_tallies = int(self.reproducible_tallies)
        d._keep = keep
        return d


def uniform_edges(a, b, n):
    """a + (b - a) * i / n with the last edge exactly b (the grid's own rule)."""
    e = np.array([a + (b - a) * i / n for i in range(n + 1)], dtype=np.float64)
    e[n] = b
    return e


def _material(p, T0, cv_per_volume, density=1.0):
    vol = p.volumes()
    n = p.ncells
    p.temperature = np.full(n, T0)
    p.mass = density * vol
    p.internal_energy = cv_per_volume * T0 * vol
    p.cell_internal_energy = p.internal_energy.copy()
    p.cv_per_mass = cv_per_volume / density
    p.eos_kind = A.EOS_LINEAR


# Densmore's volumetric heat capacity, 1e15 erg/cm^3/keV
# (examples/densmore2012/main.cpp:142).
CV_PER_VOLUME = 1e15 / UNITS["kev_kelvin"]


def gray_slab(nx=100, new_photons_per_cell=50, face_packets=50000, comb_nmin=500, comb_factor=2.0,
              seed=42, dt=1e-11, precision=A.PRECISION_FP64):
    """Plain gray FP64 IMC slab (the reference's CPU-runnable case)."""
    keV = UNITS["kev_kelvin"]
    empty = np.zeros(1)
    p = Problem(uniform_edges(0.0, 1.0, nx), uniform_edges(0.0, 0.01, 1), uniform_edges(0.0, 0.01, 1),
                empty, empty, empty)
    _material(p, 1e-3 * keV, CV_PER_VOLUME)
    p.opacity_kind = A.OPACITY_POWER_LAW
    p.kP0, p.alpha, p.cap, p.t_floor, p.kR0 = 10.0, 3.0, 1e6, 1.0, 0.0
    p.faces = [BoxFace(A.FACE_ESCAPE, 1.0 * keV, face_packets), BoxFace(A.FACE_ESCAPE)] + \
              [BoxFace(A.FACE_REFLECT) for _ in range(4)]
    p.new_photons_per_cell = new_photons_per_cell
    p.with_random_walk = False
    p.comb_enabled = True
    p.comb_nmin, p.comb_factor = comb_nmin, comb_factor
    p.seed, p.dt, p.precision, p.name = seed, dt, precision, "gray_slab"
    return p


def step_cube(n=64, new_photons_per_cell=3, face_packets=450, comb_nmin=20, comb_factor=2.0, seed=42,
              dt=1e-11, precision=A.PRECISION_FP64, with_random_walk=True):
    """Two-material step-opacity cube with Random Walk."""
    keV = UNITS["kev_kelvin"]
    empty = np.zeros(1)
    e = uniform_edges(0.0, 1.0, n)
    p = Problem(e, e.copy(), e.copy(), empty, empty, empty)
    _material(p, 0.01 * keV, CV_PER_VOLUME)
    xc, _, _ = p.cell_centers()
    p.opacity_kind = A.OPACITY_CELL_TABLE
    p.sigma_a = np.where(xc < 0.5, 1.0, 1000.0)
    p.sigma_s = np.zeros(p.ncells)
    p.faces = [BoxFace(A.FACE_ESCAPE, 1.0 * keV, face_packets)] + [BoxFace(A.FACE_ESCAPE) for _ in range(5)]
    p.new_photons_per_cell = new_photons_per_cell
    p.with_random_walk = with_random_walk
    # mean chord 4V/S = 2 dx / 3 for a cube cell: kappa*dx > 10 <=> kappa*chord > 20/3
    p.rw_min_cell_optical_depth = 20.0 / 3.0
    p.rw_min_particle_optical_depth = 5.0
    p.comb_enabled = True
    p.comb_nmin, p.comb_factor = comb_nmin, comb_factor
    p.seed, p.dt, p.precision, p.name = seed, dt, precision, "step_cube"
    return p


def uniform_cube(n=32, kappa=10.0, packets_per_step=100000, seed=42, dt=1e-11, precision=A.PRECISION_FP32_TRACK):
    """Gray cube of one material (kappa_a uniform), hot face at x=0 (1 keV),
    vacuum elsewhere, Random Walk where kappa*dx > 10.  Half of the packets per
    step come from the cells, half from the hot face; the comb keeps about
    packets_per_step in census."""
    keV = UNITS["kev_kelvin"]
    empty = np.zeros(1)
    e = uniform_edges(0.0, 1.0, n)
    p = Problem(e, e.copy(), e.copy(), empty, empty, empty)
    _material(p, 0.01 * keV, CV_PER_VOLUME)
    p.opacity_kind = A.OPACITY_CELL_TABLE
    p.sigma_a = np.full(p.ncells, float(kappa))
    p.sigma_s = np.zeros(p.ncells)
    face = max(1, int(round(0.5 * packets_per_step / (n * n))))
    p.faces = [BoxFace(A.FACE_ESCAPE, 1.0 * keV, face)] + [BoxFace(A.FACE_ESCAPE) for _ in range(5)]
    p.new_photons_per_cell = max(1, int(round(0.5 * packets_per_step / p.ncells)))
    p.with_random_walk = True
    p.rw_min_cell_optical_depth = 20.0 / 3.0
    p.rw_min_particle_optical_depth = 5.0
    p.comb_enabled = True
    p.comb_nmin, p.comb_factor = max(1, int(packets_per_step / (2 * p.ncells))), 2.0
    p.seed, p.dt, p.precision, p.name = seed, dt, precision, "uniform_cube"
    return p


def serving_mix(count, n_range=(16, 48), packets_range=(1e4, 1e6), kappa_range=(0.1, 1000.0), steps_range=(5, 20),
                seed=7, precision=A.PRECISION_FP32_TRACK):
    """A seeded stream of independent requests: N log-uniform in n_range,
    packets per step log-uniform in packets_range, kappa uniform in
    kappa_range, steps uniform in steps_range.  Returns [(problem, steps)]."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))))
        packets = float(np.exp(rng.uniform(np.log(packets_range[0]), np.log(packets_range[1]))))
        kappa = float(rng.uniform(*kappa_range))
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        out.append((uniform_cube(n=n, kappa=kappa, packets_per_step=packets, seed=1000 + k, precision=precision),
                    steps))
    return out


def mg_cube(n=16, groups=64, kappa0=100.0, new_photons_per_cell=4, comb_nmin=4, seed=42, dt=1e-11,
            precision=A.PRECISION_FP64, T_range_kev=(0.01, 0.1), with_random_walk=True, face_source=False,
            group_constant=True):
    """Multigroup gray-material cube: `groups` log-spaced groups over
    [0.01, 100] keV, kappa_g = kappa0 nu_g^-3 (1 - exp(-nu_g/T)) (nu_g the group
    centre in keV), initial T uniform in T_range_kev per cell (seeded), cell
    emission sampled from the Planck-weighted opacity spectrum; vacuum faces
    (optionally a 1 keV source on x=0)."""
    keV = UNITS["kev_kelvin"]
    kev_erg = UNITS["kev"]
    empty = np.zeros(1)
    e = uniform_edges(0.0, 1.0, n)
    p = Problem(e, e.copy(), e.copy(), empty, empty, empty)
    rng = np.random.default_rng(seed + 17)
    T0 = rng.uniform(T_range_kev[0], T_range_kev[1], p.ncells) * keV
    _material(p, 1.0, CV_PER_VOLUME)
    p.temperature = T0
    p.internal_energy = CV_PER_VOLUME * T0 * p.volumes()
    p.cell_internal_energy = p.internal_energy.copy()
    p.opacity_kind = A.OPACITY_MG_POWER
    p.sigma_a = np.full(p.ncells, kappa0 * kev_erg ** 3)     # kappa0 (E/keV)^-3
    p.sigma_s = np.zeros(p.ncells)
    p.groups = groups
    p.group_bounds = np.exp(np.linspace(np.log(0.01), np.log(100.0), groups + 1)) * kev_erg
    p.mg_group_constant = group_constant
    p.mg_p, p.mg_q, p.mg_s = 3.0, 0.0, 1.0
    p.faces = [BoxFace(A.FACE_ESCAPE, 1.0 * keV if face_source else 0.0, 50 if face_source else 0)] + \
              [BoxFace(A.FACE_ESCAPE) for _ in range(5)]
    p.new_photons_per_cell = new_photons_per_cell
    p.with_random_walk = with_random_walk
    p.rw_min_cell_optical_depth = 20.0 / 3.0
    p.rw_min_particle_optical_depth = 5.0
    p.comb_enabled = True
    p.comb_nmin, p.comb_factor = comb_nmin, 2.0
    p.seed, p.dt, p.precision, p.name = seed, dt, precision, "mg_cube"
    return p


# ---------------------------------------------------------------- the reference's benchmark problems

# Krief & McClarren (2024) Marshak waves 1-4 as the reference states them
# (examples/marshak_wave/MarshakCommon.hpp:48-113): power-law opacity
# kappa = kappa0 (keV / T)^alpha rho^betaRho (Planck kappaP0, total kappaR0),
# EOS e_vol = f T^beta rho^(1 - mu), bath T(t) = coeff (t / ns)^exponent keV.
MARSHAK_PARAMS = {
    1: dict(length=0.2, x_offset=0.0, kP0=0.1, kR0=100.0, alpha=3.0, beta_rho=0.0, f_keV=6.860085e14, eos_beta=4.0,
            eos_mu=0.0, bath_coeff=1.008038, bath_exp=1.0 / 3.0, initial_dt=1e-15),
    2: dict(length=0.2, x_offset=0.0, kP0=100.0, kR0=100.0, alpha=3.0, beta_rho=0.0, f_keV=6.860085e14, eos_beta=4.0,
            eos_mu=0.0, bath_coeff=1.014565, bath_exp=1.0 / 3.0, initial_dt=1e-15),
    3: dict(length=1.0, x_offset=0.0, kP0=0.1, kR0=40.0, alpha=1.5, beta_rho=1.2, f_keV=1e14, eos_beta=3.4,
            eos_mu=0.14, bath_coeff=1.0470478, bath_exp=86.0 / 57.0, initial_dt=1e-15),
    4: dict(length=1.0, x_offset=1e-5, kP0=0.001, kR0=2.0, alpha=4.5, beta_rho=1.9, f_keV=1e14, eos_beta=6.0,
            eos_mu=0.3, bath_coeff=1.01008116, bath_exp=14.0 / 139.0, initial_dt=1e-17),
}
MARSHAK_FINAL_TIME = 1e-9


def marshak_density(problem, x):
    """ComputeDensity (MarshakCommon.hpp:115-124)."""
    x = np.asarray(x, dtype=np.float64)
    if problem == 3:
        return np.power(np.maximum(x, 1e-30), 20.0 / 19.0)
    if problem == 4:
        return np.power(np.maximum(x, 1e-30), -40.0 / 139.0)
    return np.ones_like(x)


def marshak_bath_temperature(problem, t):
    """BathTemperature (MarshakCommon.hpp:141-145), in K."""
    q = MARSHAK_PARAMS[problem]
    t_ns = max(t, 1e-20) * 1e9
    return q["bath_coeff"] * t_ns ** q["bath_exp"] * UNITS["kev_kelvin"]


def marshak4_edges(x_offset, x_max):
    """BuildMarshak4MeshEdges (MarshakCommon.hpp:249-263): 512 cells, the first
    7e-5 cm wide, each 1.0096903847403653 times the last, the last edge x_max."""
    edges = np.empty(513)
    edges[0] = x_offset
    width = 7.0e-5
    for i in range(512):
        edges[i + 1] = x_max if i + 1 == 512 else edges[i] + width
        width *= 1.0096903847403653
    return edges


def marshak_wave(problem=1, nx=256, new_photons_per_cell=15, boundary_per_face=100, seed=42,
                 precision=A.PRECISION_FP64):
    """Marshak wave `problem` (1-4) as RunMarshakWave sets it up
    (MarshakCommon.hpp:265-320): an nx x 1 x 1 slab (problem 4: the fixed
    512-cell graded mesh), T0 = 1 eV, the bath on x=0 (packets that reach it
    escape), the other faces reflecting, Random Walk on with its default
    thresholds, comb (15, 6).  The time loop and the bath updates are
    `benchmarks.run_marshak_wave`."""
    q = MARSHAK_PARAMS[problem]
    keV = UNITS["kev_kelvin"]
    x_max = q["x_offset"] + q["length"]
    if problem == 4:
        xe = marshak4_edges(q["x_offset"], x_max)
        dy = x_max / (len(xe) - 1)
    else:
        dy = x_max / nx
        xe = uniform_edges(0.0, x_max, nx)
    empty = np.zeros(1)
    p = Problem(xe, uniform_edges(0.0, dy, 1), uniform_edges(0.0, dy, 1), empty, empty, empty)
    xc, _, _ = p.cell_centers()
    rho = marshak_density(problem, xc)
    vol = p.volumes()
    f = q["f_keV"] / keV ** q["eos_beta"]
    T0 = 1e-3 * keV
    p.temperature = np.full(p.ncells, T0)
    p.internal_energy = f * T0 ** q["eos_beta"] * np.power(rho, 1.0 - q["eos_mu"]) * vol
    p.cell_internal_energy = p.internal_energy.copy()
    p.mass = rho * vol
    p.eos_kind = A.EOS_POWER_LAW
    p.eos_f, p.eos_beta, p.eos_mu = f, q["eos_beta"], q["eos_mu"]
    p.opacity_kind = A.OPACITY_POWER_LAW
    p.kP0, p.kR0, p.alpha, p.t_floor, p.cap = q["kP0"], q["kR0"], q["alpha"], 1.0, 0.0
    p.density_factor = np.power(rho, q["beta_rho"]) if q["beta_rho"] != 0.0 else None
    p.faces = [BoxFace(A.FACE_ESCAPE, marshak_bath_temperature(problem, q["initial_dt"]), boundary_per_face)] + \
              [BoxFace(A.FACE_REFLECT) for _ in range(5)]
    p.new_photons_per_cell = new_photons_per_cell
    p.with_random_walk = True
    p.comb_enabled = True
    p.comb_nmin, p.comb_factor = 15, 6.0
    p.seed, p.dt, p.precision, p.name = seed, q["initial_dt"], precision, f"marshak_wave_{problem}"
    return p


def densmore_group_bounds(groups=30):
    """Group bounds of the Densmore benchmark (examples/densmore2012/main.cpp:151-158):
    1e-4 keV times ratio^g, ratio = (100 keV / 1e-4 keV)^(1/groups), built by
    repeated multiplication as there."""
    kev = UNITS["kev"]
    e_min, e_max = kev * 1e-4, kev * 1e2
    ratio = (e_max / e_min) ** (1.0 / groups)
    b = np.empty(groups + 1)
    b[0] = e_min
    for g in range(groups):
        b[g + 1] = b[g] * ratio
    return b


def densmore2012(nx=512, new_photons_per_cell=16, boundary_per_face=100, seed=42, precision=A.PRECISION_FP64,
                 comb_nmin=200):
    """Densmore et al. (2012) Fig. 4, as examples/densmore2012/main.cpp:128-208
    sets it up: x in [0, 3] cm (nx x 1 x 1), sigma(E) = sigma0 / (sqrt(kT) E^3)
    with sigma0 = 10 keV^3.5/cm below x = 2 and 1000 keV^3.5/cm above, 30
    groups, cv = 1e15 erg/cm^3/keV, T0 = 1 eV, a 1 keV Planck source on x=0
    (packets that reach it escape), reflecting elsewhere, Random Walk with its
    default thresholds, comb (200, 5), dt = 5e-12 s (200 steps to 1 ns)."""
    keV = UNITS["kev_kelvin"]
    kev = UNITS["kev"]
    length = 3.0
    dy = length / nx
    empty = np.zeros(1)
    p = Problem(uniform_edges(0.0, length, nx), uniform_edges(0.0, dy, 1), uniform_edges(0.0, dy, 1),
                empty, empty, empty)
    _material(p, keV / 1000.0, CV_PER_VOLUME)
    xc, _, _ = p.cell_centers()
    p.opacity_kind = A.OPACITY_MG_POWER
    p.sigma_a = np.where(xc < 2.0, 10.0 * kev ** 3.5, 1000.0 * kev ** 3.5)
    p.sigma_s = np.zeros(p.ncells)
    p.groups = 30
    p.group_bounds = densmore_group_bounds(30)
    p.mg_group_constant = False
    p.mg_p, p.mg_q, p.mg_s = 3.0, 0.5, 0.0
    p.faces = [BoxFace(A.FACE_ESCAPE, keV, boundary_per_face)] + [BoxFace(A.FACE_REFLECT) for _ in range(5)]
    p.new_photons_per_cell = new_photons_per_cell
    p.with_random_walk = True
    p.comb_enabled = True
    p.comb_nmin, p.comb_factor = comb_nmin, 5.0
    p.seed, p.dt, p.precision, p.name = seed, 5e-12, precision, "densmore2012"
    return p


def ddmc_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=20, seed=42, dt=1e-10,
              precision=A.PRECISION_FP64, with_random_walk=False, rw_min_particle_optical_depth=5.0,
              sigma_a_thick=1.0, sigma_s_thick=1000.0):
    """A step cube with DDMC-style leakage on (withDDMC, the reference's
    default depths 15 and 5): sigma_a = 1, no scattering for x < 0.5; a
    scattering-dominated half (sigma_a_thick, sigma_s_thick) for x >= 0.5 that
    is DDMC eligible, so that particles there diffuse between cells by face
    leaks rather than being absorbed in place.  1 keV source on x=0, vacuum
    elsewhere, T0 = 0.01 keV.  With Random Walk also on, a particle deep enough
    for a Random Walk jump takes it first and DDMC covers the depths between
    the two particle thresholds."""
    p = step_cube(n=n, new_photons_per_cell=new_photons_per_cell, face_packets=face_packets, comb_nmin=comb_nmin,
                  seed=seed, dt=dt, precision=precision, with_random_walk=with_random_walk)
    xc, _, _ = p.cell_centers()
    thick = xc >= 0.5
    p.sigma_a = np.where(thick, sigma_a_thick, 1.0)
    p.sigma_s = np.where(thick, sigma_s_thick, 0.0)
    p.with_ddmc = True
    p.rw_min_particle_optical_depth = rw_min_particle_optical_depth
    p.name = "ddmc_cube"
    return p


def voronoi_ddmc(ncells=300, packets_per_step=3e4, seed=23, dt=2e-10, precision=A.PRECISION_FP64, mesh=None,
                 sigma_s_thick=500.0, with_random_walk=False):
    """DDMC-style leakage (withDDMC, depths 15 and 5) on a Voronoi mesh: the
    cells of voronoi_cube with sigma_a = 1 everywhere and an elastic opacity
    sigma_s_thick in the cells whose generators lie at x >= 0.5, which makes
    them DDMC eligible; cell emission only, vacuum on the box."""
    p = voronoi_cube(ncells=ncells, packets_per_step=packets_per_step, seed=seed, dt=dt, precision=precision,
                     with_random_walk=with_random_walk, mesh=mesh)
    thick = p.mesh.points[:, 0] >= 0.5
    p.sigma_a = np.ones(p.ncells)
    p.sigma_s = np.where(thick, sigma_s_thick, 0.0)
    p.with_ddmc = True
    p.name = "voronoi_ddmc"
    return p


def strat_cube(n=4, groups=30, bins=6, comb_nmin=4, comb_factor=2.0, min_per_bin=2, new_photons_per_cell=6, seed=42,
               precision=A.PRECISION_FP64):
    """A small multigroup cube whose population control is
    StratifiedCombPopulationControl with `bins` frequency bins, every
    (groups / bins)-th group bound an edge."""
    p = mg_cube(n=n, groups=groups, kappa0=1.0, new_photons_per_cell=new_photons_per_cell, comb_nmin=comb_nmin,
                seed=seed, precision=precision, group_constant=False)
    p.comb_factor = comb_factor
    p.comb_kind = A.COMB_STRATIFIED
    p.strat_bins = bins
    p.strat_bounds = p.group_bounds[::groups // bins].copy()
    p.strat_min_per_bin = min_per_bin
    p.name = "strat_cube"
    return p


def voronoi_cube(ncells=200000, packets_per_step=2e7, seed=42, dt=1e-11, precision=A.PRECISION_FP64,
                 kappa_median=10.0, kappa_sigma_ln=1.0, T_median_kev=0.05, T_sigma_ln=1.0, with_random_walk=True,
                 mesh=None, comb_factor=2.0):
    """Gray IMC on a Voronoi mesh of `ncells` seeded uniform generators in the
    unit cube (about 15 faces per cell): per-cell lognormal absorption opacity
    (median kappa_median 1/cm, sigma_ln), lognormal initial temperature
    (median T_median_kev), constant volumetric heat capacity, vacuum on every
    box face, cell emission only (about packets_per_step per step), Random Walk
    where sigma 4V/S >= 20/3, comb to about packets_per_step."""
    from .mesh import build_voronoi
    keV = UNITS["kev_kelvin"]
    rng = np.random.default_rng(seed)
    if mesh is None:
        pts = rng.random((ncells, 3)) * (1 - 2e-9) + 1e-9
        mesh = build_voronoi(pts)
    else:
        rng.random((ncells, 3))
    n = mesh.ncells
    empty = np.zeros(1)
    p = Problem(uniform_edges(0.0, 1.0, 1), uniform_edges(0.0, 1.0, 1), uniform_edges(0.0, 1.0, 1), empty, empty,
                empty)
    p.mesh = mesh
    T0 = T_median_kev * np.exp(T_sigma_ln * rng.standard_normal(n)) * keV
    _material(p, 1.0, CV_PER_VOLUME)
    p.temperature = T0
    p.internal_energy = CV_PER_VOLUME * T0 * p.volumes()
    p.cell_internal_energy = p.internal_energy.copy()
    p.opacity_kind = A.OPACITY_CELL_TABLE
    p.sigma_a = kappa_median * np.exp(kappa_sigma_ln * rng.standard_normal(n))
    p.sigma_s = np.zeros(n)
    p.faces = [BoxFace(A.FACE_ESCAPE) for _ in range(6)]
    # the allocation floors each cell at newPhotonsPerCell and gives hot cells up
    # to 20 times it; with these lognormal temperatures the total is about 3.1
    # times the floor, so the floor is a third of the per-cell mean
    p.new_photons_per_cell = max(1, int(round(packets_per_step / (3.1 * n))))
    p.with_random_walk = with_random_walk
    p.rw_min_cell_optical_depth = 20.0 / 3.0
    p.rw_min_particle_optical_depth = 5.0
    p.comb_enabled = True
    p.comb_nmin, p.comb_factor = max(1, int(packets_per_step / (comb_factor * n))), comb_factor
    p.seed, p.dt, p.precision, p.name = seed, dt, precision, "voronoi_cube"
    return p
