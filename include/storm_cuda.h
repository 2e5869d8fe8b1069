/*
 * storm_cuda.h -- C ABI of the B200 Implicit Monte Carlo (IMC) transport engine.
 *
 * This is the host->device crossing of the drop-in replacement for STORM's
 * serial manager.  In STORM the whole time step is
 *
 *     std::vector<Particle> MonteCarloManagerSerial<T,Grid>::step(std::vector<Particle>&&, dt_t)
 *     (manager/MonteCarloManagerSerial.hpp:44, 386-469)
 *
 * which calls RadiationIMC::preStep (radiation/RadiationIMC.hpp:1618-1694), the
 * per-particle RadiationIMC::step (radiation/RadiationIMC.hpp:1700-1881) until
 * census/escape/absorption, CombPopulationControl::activate
 * (population/CombPopulationControl.hpp:79-253) and RadiationIMC::postStep
 * (radiation/RadiationIMC.hpp:1887-2029).  Here the same step runs on one GPU
 * behind an opaque handle.  Everything is plain C: pointers, sizes, int status.
 *
 * Error convention: every entry point returns an int status (0 = STORM_OK).  No
 * exception crosses the ABI.  A nonzero status carries the class below; the
 * device error word (STORM_DERR_*) that a kernel raised is read with
 * storm_cuda_last_error().  The C++ host template (storm/MonteCarloManagerCUDA.hpp)
 * converts a nonzero status into STORM::StormError, matching the reference's
 * "report and rethrow" behaviour (manager/MonteCarloManagerSerial.hpp:458-462).
 *
 * Threading: one CUDA stream per handle; calls on one handle must be serialised
 * by the caller (the reference manager is single-threaded and not reentrant,
 * manager/MonteCarloManagerSerial.hpp:269-270).  Different handles are
 * independent.
 */
#ifndef STORM_CUDA_H
#define STORM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STORM_CUDA_ABI_VERSION 8

/* ---------------------------------------------------------------- status */
enum StormStatus {
    STORM_OK = 0,
    STORM_ERR_INVALID_ARG = 1,   /* bad descriptor / argument (host-side check) */
    STORM_ERR_CUDA = 2,          /* a CUDA runtime call failed */
    STORM_ERR_OOM = 3,           /* device allocation failed */
    STORM_ERR_DEVICE = 4,        /* a kernel raised a STORM_DERR_* error word */
    STORM_ERR_CAPACITY = 5,      /* particle bank capacity exceeded */
    STORM_ERR_UNSUPPORTED = 6,   /* option not supported by this engine */
    STORM_ERR_NO_DEVICE = 7      /* no CUDA device visible */
};

/* Device error words (first error wins, recorded with cell / particle index).
 * Each corresponds to a StormError the reference throws. */
enum StormDeviceError {
    STORM_DERR_NONE = 0,
    STORM_DERR_NO_FACE = 1,          /* particle/Particle.hpp:257-278 "no face intersection found" */
    STORM_DERR_NOT_ON_BOUNDARY = 2,  /* boundary/RigidBoundary.hpp:66-68, SideTemperature.hpp:110-111 */
    STORM_DERR_FLECK = 3,            /* radiation/RadiationIMC.hpp:1650-1661 invalid Fleck factor */
    STORM_DERR_NEGATIVE_ENERGY = 4,  /* radiation/RadiationIMC.hpp:771-817 */
    STORM_DERR_COMB_OUTSIDE = 5,     /* population/CombPopulationControl.hpp:110-121 */
    STORM_DERR_COMB_WEIGHT = 6,      /* population/CombPopulationControl.hpp:122-135 (non-finite or negative) */
    STORM_DERR_RW_SHRINK = 7,        /* RW shrink-to-inside loop exceeded its iteration limit */
    STORM_DERR_HISTORY_CAP = 8,      /* a history exceeded max_rounds * segments_per_visit segments */
    STORM_DERR_BANK_OVERFLOW = 9,    /* more particles than bank capacity */
    STORM_DERR_TAPE_EXHAUSTED = 10,  /* replay: uniform tape too short */
    STORM_DERR_COMB_TOTAL = 11,      /* population/CombPopulationControl.hpp:147-153 total weight not finite */
    STORM_DERR_MG_SAMPLE = 12        /* utils/LinearInterpolation.hpp:22-28 "X too large" in a thermal energy draw */
};

/* ---------------------------------------------------------------- enums */
enum StormPrecision {
    STORM_PRECISION_FP64 = 0,        /* all-FP64 tracking (reference arithmetic) */
    STORM_PRECISION_FP32_TRACK = 1   /* cell index + FP32 cell-local offset, FP32 direction/distance;
                                        weights, time, tallies and material update in FP64 */
};

enum StormFaceAction {
    STORM_FACE_REFLECT = 0,          /* BoundaryCondition::reflectParticleOnBoxFace (boundary/BoundaryCondition.hpp:87-108) */
    STORM_FACE_ESCAPE = 1            /* particle removed, its weight tallied as escaped */
};

enum StormOpacityKind {
    /* sigma_a[cell], sigma_s[cell] given per cell (temperature independent) */
    STORM_OPACITY_CELL_TABLE = 0,
    /* sigma_a = min(kP0 * (kev_kelvin / max(T, t_floor))^alpha * rho^beta, cap)
       sigma_s = max(kR0 * f - kP0 * f, 0) with the same factors f.
       Marshak form: examples/marshak_wave/MarshakOpacity.hpp:30-46 (cap = +inf there). */
    STORM_OPACITY_POWER_LAW = 1,
    /* Multigroup (groups >= 2): sigma_a(E, T) = sigma_a[cell] / ((kT)^q E^p) * (1 - exp(-E/kT))^s
       with kT = k_B max(T, 1 K), E = max(frequency, group_bounds[0]), or the centre of the
       particle's group when mg_group_constant; sigma_s[cell] elastic.  Planck mean, emission
       spectrum and group CDF from the group centres with planck_integral weights, as
       examples/densmore2012/DensmoreOpacity.hpp:36-56, 71-82, 146-165. */
    STORM_OPACITY_MG_POWER = 2
};

enum StormEosKind {
    /* dT2cv = cv_per_mass ; de2T = e / cv_per_mass   (examples/densmore2012/main.cpp:56-77) */
    STORM_EOS_LINEAR = 0,
    /* e_vol = f * T^beta * rho^(1-mu)   (examples/marshak_wave/MarshakCommon.hpp:138-155, 162-183) */
    STORM_EOS_POWER_LAW = 1
};

/* ---------------------------------------------------------------- descriptor */

/* A convex-polyhedral mesh in a box (the engine's stand-in for the reference's
 * Voronoi grids, MadVoro): cells, each with its faces in GetCellFaces order, and
 * per face the two cells it separates (the second >= ncells for a face on the
 * box: the ghost ncells + face index), its unit normal from the first cell to
 * the second, centroid, area and polygon.  Cell-move nudges aim at the mesh
 * points (the Voronoi generators), as the reference's manager does with
 * GetMeshPoint (manager/MonteCarloManagerSerial.hpp:323-327). */
typedef struct StormPolyMesh {
    uint32_t ncells, nfaces, nvertices, pad_;
    double box[6];                       /* lo x, y, z, hi x, y, z */
    const double *points;                /* 3 ncells: mesh points */
    const double *volume;                /* ncells */
    const uint32_t *cell_face_offset;    /* ncells + 1 */
    const uint32_t *cell_faces;          /* global face indices */
    const uint32_t *face_cells;          /* 2 nfaces */
    const double *face_normal;           /* 3 nfaces */
    const double *face_cm;               /* 3 nfaces */
    const double *face_area;             /* nfaces */
    const uint32_t *face_vertex_offset;  /* nfaces + 1 */
    const uint32_t *face_vertices;       /* ordered around each face */
    const double *vertices;              /* 3 nvertices */
} StormPolyMesh;

/* One of the six faces of the bounding box, in GetBoxFaces() order:
 * 0 x-low, 1 x-high, 2 y-low, 3 y-high, 4 z-low, 5 z-high. */
typedef struct StormBoxFace {
    int32_t action;              /* StormFaceAction */
    int32_t pad_;
    double source_temperature;   /* K; > 0 makes this face a Planck surface source */
    uint64_t packets_per_face;   /* packets per boundary cell-face per step (SideTemperature::Npercell) */
} StormBoxFace;

typedef struct StormProblemDesc {
    uint32_t abi_version;        /* must be STORM_CUDA_ABI_VERSION */
    int32_t precision;           /* StormPrecision */

    /* ---- rectilinear mesh (the Cartesian Grid of the reference examples).
     * Cell index = i + nx*(j + ny*k).  Edges strictly increasing. */
    uint32_t nx, ny, nz;
    const double *x_edges;       /* nx+1 */
    const double *y_edges;       /* ny+1 */
    const double *z_edges;       /* nz+1 */

    /* ---- per-cell material state (host arrays, Ncells each).  Units as in
     * radiation/RadiationCell.hpp:6-19: temperature [K], mass [g],
     * internal_energy = extensive material energy [erg]. */
    const double *temperature;
    const double *mass;
    const double *internal_energy;
    const double *cell_internal_energy;  /* RadiationCell::internalEnergy (positivity floor); NULL = internal_energy */

    /* ---- opacity plug-in lowered to a device descriptor */
    int32_t opacity_kind;        /* StormOpacityKind */
    int32_t eos_kind;            /* StormEosKind */
    const double *sigma_a;       /* CELL_TABLE: absorption (Planck) opacity [1/cm], Ncells */
    const double *sigma_s;       /* CELL_TABLE: scattering opacity [1/cm], Ncells (NULL = 0) */
    double kP0, kR0, alpha, beta, t_floor, cap;   /* POWER_LAW parameters */
    const double *density_factor;               /* POWER_LAW: rho^beta per cell (NULL = 1) */

    /* ---- EOS */
    double cv_per_mass;          /* LINEAR */
    double eos_f, eos_beta, eos_mu;  /* POWER_LAW */

    /* ---- boundary plug-in lowered to per-box-face actions */
    StormBoxFace faces[6];
    int32_t escape_without_check;    /* VacuumBoundary::apply removes without a closeness test (boundary/Vacuum.hpp:18-22) */
    int32_t pad0_;

    /* ---- RadiationIMCParameters<1> (radiation/RadiationIMCParameters.hpp:13-56) */
    uint64_t new_photons_per_cell;
    int32_t with_random_walk;
    int32_t no_hydro_feedback;
    double rw_min_cell_optical_depth;
    double rw_min_particle_optical_depth;

    /* ---- CombPopulationControl(grid, Nmin, factor) (population/CombPopulationControl.hpp:21-31) */
    int32_t comb_enabled;
    int32_t pad1_;
    uint64_t comb_nmin;
    double comb_factor;

    /* ---- physical constants, taken from the caller's `units` so that host and
     * device agree with whatever constants the caller's physics uses. */
    double clight, arad, sigma_sb, kev_kelvin;

    /* ---- engine settings (MonteCarloConfig-like) */
    uint64_t seed;
    uint64_t capacity;               /* max particles in flight (0 = automatic) */
    uint32_t segments_per_visit;     /* segments a thread runs per bank visit (0 = automatic) */
    uint32_t max_rounds;             /* bank visits per step before STORM_DERR_HISTORY_CAP (0 = automatic) */
    int32_t per_cell_segment_counters;   /* fill GetCellsStepsCounters() (costs one atomic per segment) */
    int32_t device;                  /* CUDA device ordinal */

    /* ---- multigroup (RadiationIMC<..., NumGroups> with withMultigroupOpacity;
     * the Random Walk becomes the PGRW of radiation/RadiationIMC.hpp:1008-1061) */
    uint32_t groups;                 /* 0 or 1: gray; G >= 2: G groups */
    int32_t mg_group_constant;       /* opacity at the centre of the particle's group */
    const double *group_bounds;      /* G+1 increasing energies [erg] (energyBoundaries) */
    double mg_p, mg_q, mg_s;         /* STORM_OPACITY_MG_POWER exponents */
    double k_boltz;                  /* erg/K, for kT */

    /* ---- DDMC-style leakage in optically thick cells (RadiationIMCParameters
     * withDDMC, ddmcMinCellOpticalDepth, ddmcMinParticleOpticalDepth,
     * ddmcUseMultigroupPGRW; radiation/RadiationIMC.hpp:1282-1612) */
    int32_t with_ddmc;
    int32_t ddmc_use_multigroup_pgrw;
    double ddmc_min_cell_optical_depth;      /* reference default 15 */
    double ddmc_min_particle_optical_depth;  /* reference default 5 */

    /* ---- population control: CombPopulationControl (0) or
     * StratifiedCombPopulationControl (1, population/CombPopulationControl.hpp:35-511)
     * with the particle classifier lowered to frequency bins: bin g holds
     * frequencies below strat_bounds[g + 1] (the last bin everything above),
     * RadiationOpacityModel::findGroup's rule.  comb_nmin and comb_factor are
     * its Nmin and totalParticlesFactor. */
    int32_t comb_kind;               /* StormCombKind */
    uint32_t strat_bins;             /* groupCount, 1..STORM_STRAT_MAX_BINS */
    const double *strat_bounds;      /* strat_bins + 1 increasing frequencies [erg]; NULL: one bin (gray), or the
                                        problem's group_bounds when strat_bins equals groups */
    uint64_t strat_min_per_bin;      /* minParticlesPerGroup (reference default 2) */

    /* ---- convex-polyhedral mesh (NULL: the Cartesian grid of nx, ny, nz and the
     * edges).  With a mesh, the per-cell arrays follow its cell order and the box
     * faces are the mesh's box; either form, with DDMC and face sources, but a
     * gray opacity only (no groups) and no moving material. */
    const struct StormPolyMesh *mesh;

    /* ---- moving material (RadiationIMCParameters::withHydro with cells that
     * carry a velocity and extensives that carry a momentum): Doppler-shifted
     * opacities, comoving scatters and emission transformed to the lab frame,
     * momentum deposition (radiation/RadiationIMC.hpp:228-314, 1700-1881,
     * 2035-2510, 830-866).  FP64 form on the Cartesian grid only. */
    int32_t with_hydro;
    int32_t pad2_;
    const double *cell_velocity;     /* 3 per cell [cm/s]: the cells' velocity (NULL = at rest) */

    /* ---- group time averages (RadiationIMCParameters::withEgTimeAvg): per cell
     * and group the time-integrated radiation energy of the particles whose lab
     * frequency is in the group, tallied with Erad_time_avg in every segment,
     * Random Walk jump and DDMC step and divided by dt V after the step
     * (radiation/RadiationIMC.hpp:1166-1172, 1485-1491, 1802-1808, 1896-1902).
     * Multigroup problems only, as in the reference; not with particle shards. */
    int32_t with_eg_time_avg;

    /* ---- reproducible tallies: the material deposits and the time-integrated
     * radiation energy of the transport are summed per cell in 120-bit fixed
     * point with integer atomics, at a per-step scale from the step's energy
     * budget, and folded into FP64 after transport, so that a run repeats bit
     * for bit (FP64 atomics add in an order that varies from run to run).  Not
     * with moving material, group time averages, particle shards or without
     * population control (STORM_ERR_UNSUPPORTED). */
    int32_t reproducible_tallies;
} StormProblemDesc;

#define STORM_STRAT_MAX_BINS 64

enum StormCombKind {
    STORM_COMB_PLAIN = 0,            /* CombPopulationControl (population/CombPopulationControl.hpp:79-253) */
    STORM_COMB_STRATIFIED = 1        /* StratifiedCombPopulationControl (population/CombPopulationControl.hpp:255-511) */
};

/* Particle arrays, struct-of-arrays.  Mirrors the fields of
 * Particle<T,Grid> (particle/Particle.hpp:67-85) that the gray path uses.
 * Host or device pointers depending on the call. */
typedef struct StormParticlesSoA {
    double *x, *y, *z;           /* location [cm] */
    double *vx, *vy, *vz;        /* velocity = c * direction [cm/s] */
    double *time_left;           /* [s] */
    double *weight;              /* [erg] */
    double *initial_weight;      /* [erg] */
    uint32_t *cell;              /* cellIndex */
    uint64_t *id;                /* particle id within the step (may be NULL on input) */
    uint64_t count;
    double *frequency;           /* photon energy [erg], multigroup problems (NULL otherwise) */
} StormParticlesSoA;

typedef struct StormStepStats {
    uint64_t census_in;          /* particles handed to the step (GetInitialParticleCount) */
    uint64_t emitted_cells;      /* cell-source packets (RadiationIMC::generateParticles) */
    uint64_t emitted_faces;      /* boundary-source packets */
    uint64_t census_out_pre_comb;/* DONE particles before population control */
    uint64_t census_out;         /* particles after population control (GetEndParticleCount) */
    uint64_t segments;           /* sum of GetCellsStepsCounters() */
    uint64_t rw_steps;           /* getRandomWalkStepCount() */
    uint64_t escaped;            /* particles removed at the boundary */
    uint64_t cutoff;             /* particles removed by the weight cutoff */
    uint64_t rounds;             /* bank visits used by transport */
    double energy_census_in;     /* sum of census weights at step start */
    double energy_emitted;       /* cell + face source energy */
    double energy_deposited;     /* sum of material deposits during transport (incl. cutoff) */
    double energy_escaped;       /* weight that left through ESCAPE faces */
    double energy_census_pre_comb;
    double energy_census_out;
    double energy_emission_debit;/* material energy removed by cell emission */
    double transport_ms;         /* device time of transport (CUDA events) */
    double step_ms;              /* device time of the whole step */
    double emit_ms;              /* device time from step start through emission (begin, prestep, emit) */
    double comb_ms;              /* device time of population control */
} StormStepStats;

/* Replay of single segments against a recorded uniform tape: the parity
 * entry point.  Each item is one call of RadiationIMC::step plus the manager's
 * face/boundary handling (manager/MonteCarloManagerSerial.hpp:318-369). */
typedef struct StormReplayBatch {
    uint64_t n;
    /* inputs, n each (host) */
    const double *x, *y, *z, *vx, *vy, *vz, *time_left, *weight, *initial_weight;
    const uint32_t *cell;
    const uint64_t *tape_offset;     /* into tape */
    const uint32_t *tape_length;
    const double *tape;              /* raw std::uniform_real_distribution draws */
    /* outputs, n each (host) */
    double *phys_x, *phys_y, *phys_z, *phys_vx, *phys_vy, *phys_vz, *phys_time_left, *phys_weight;
    int32_t *phys_status;            /* ParticleStatus of RadiationIMC::step (particle/ParticleStatus.hpp:8-15) */
    uint32_t *phys_next_cell;        /* StepResult::nextCellIndex (face crossings), else UINT32_MAX */
    double *dep_material;            /* sum added to extensives[cell].internal_energy */
    double *dep_erad;                /* sum added to Erad_time_avg_[cell] */
    double *mgr_x, *mgr_y, *mgr_z, *mgr_vx, *mgr_vy, *mgr_vz; /* after the manager's nudge / boundary */
    uint32_t *mgr_cell;
    int32_t *mgr_status;             /* 0 continue, 1 census, 2 removed (cutoff), 3 escaped */
    uint32_t *draws_used;
    int32_t *used_random_walk;
    /* multigroup: the particle's frequency before and after (NULL for gray) */
    const double *frequency;
    double *phys_frequency;
    /* moving material: the momentum the segment left in its cell, 3 per item
     * (extensives[cell].momentum; NULL = not returned) */
    double *phys_momentum;
} StormReplayBatch;

typedef struct StormHandle StormHandle;

/* ---------------------------------------------------------------- lifecycle */

/* Replaces constructing MonteCarloManagerSerial(grid, physics, populationControl,
 * boundaryCondition) (manager/MonteCarloManagerSerial.hpp:38-40, 120-129) and the
 * RadiationIMC constructor (radiation/RadiationIMC.hpp:562-640). */
int storm_cuda_create(const StormProblemDesc *desc, StormHandle **out);
/* Replaces ~MonteCarloManagerSerial (manager/MonteCarloManagerSerial.hpp:186-195). */
int storm_cuda_destroy(StormHandle *h);

/* ---------------------------------------------------------------- particle shards */

/* One problem split over several ranks (one GPU each) by particle-id ranges.
 * The mesh and every per-cell table are replicated; the census and each
 * step's emission are cut into `shards` particle shards, and a rank holds the
 * contiguous shards [shard_lo, shard_hi).  Three times per step the engine
 * hands the exchange callback a device buffer of doubles to be summed in
 * place over all ranks (an all-reduce, ordered on `stream`):
 *   1. after transport: the per-cell material deposits and the time-averaged
 *      radiation tallies (2 N values);
 *   2. in the comb: the census weight and particle count of every
 *      (shard, cell) run (2 S N values, each rank filling its own shards'
 *      entries and zeros elsewhere);
 *   3. after the comb: the census particles per shard and the census radiation
 *      energy per cell (S + N values).
 * This mirrors the reference's MPI reductions of the step totals
 * (radiation/RadiationIMC.hpp:2070-2071; population/CombPopulationControl.hpp:102,
 * 145), with the per-cell sums the shared mesh needs.  The comb keeps the
 * census of each shard on its rank and places every shard's teeth after the
 * weight of the lower shards in the same cell, so for a given `shards` the
 * step's results do not depend on how the shards are spread over ranks, up
 * to the summation order of the floating-point tallies.  A callback returning
 * nonzero fails the step with STORM_ERR_INVALID_ARG.  The exchange may be NULL
 * when one rank holds every shard. */
typedef int (*StormExchangeFn)(void *user, double *values, uint64_t count, void *stream);

/* Configure particle shards on a handle whose census is empty (before its first
 * step).  shards = 1 turns sharding off.  Requires CombPopulationControl (the
 * plain comb); other population controls return STORM_ERR_INVALID_ARG. */
int storm_cuda_set_sharding(StormHandle *h, uint32_t shards, uint32_t shard_lo, uint32_t shard_hi,
                            StormExchangeFn exchange, void *user);

/* ---------------------------------------------------------------- the step */

/* One full time step on the device-resident census: MonteCarloManagerSerial::step
 * (manager/MonteCarloManagerSerial.hpp:386-469).  stats may be NULL. */
int storm_cuda_step(StormHandle *h, double dt, StormStepStats *stats);

/* The phases of storm_cuda_step, callable one at a time (parity tests):
 *   prestep   -> RadiationIMC::preStep minus emission (RadiationIMC.hpp:1618-1672)
 *   emit      -> generateParticles + boundary->generateNewBoundaryParticles (RadiationIMC.hpp:1674-1692, 2035-2510)
 *   transport -> the HandleAll loop (MonteCarloManagerSerial.hpp:267-383, 436-456)
 *   comb      -> populationControl->activate (MonteCarloManagerSerial.hpp:464)
 *   poststep  -> physics->postStep (MonteCarloManagerSerial.hpp:466) */
int storm_cuda_phase_prestep(StormHandle *h, double dt);
int storm_cuda_phase_emit(StormHandle *h, double dt);
int storm_cuda_phase_transport(StormHandle *h);
int storm_cuda_phase_comb(StormHandle *h);
int storm_cuda_phase_poststep(StormHandle *h, double dt);
/* statistics gathered by the phases since the last storm_cuda_phase_begin / storm_cuda_step */
int storm_cuda_phase_begin(StormHandle *h, double dt);
int storm_cuda_phase_stats(StormHandle *h, StormStepStats *stats);

/* ---------------------------------------------------------------- state in/out */

/* Replace the census with host particles (the std::vector<Particle>&& argument
 * of step()).  Copies host -> device.  time_left and initial_weight may be
 * NULL: the step sets them for every census particle (timeLeft = dt,
 * initialWeight = |weight|, manager/MonteCarloManagerSerial.hpp:391-405), so a
 * caller that only steps need not copy them; they read 0 until then. */
int storm_cuda_set_census(StormHandle *h, const StormParticlesSoA *host_in);
/* Copy the census (the vector step() returns) device -> host.  host_out arrays
 * must hold `capacity` entries; *count receives the census size.  A NULL field
 * is not copied: a caller that hands the census back to the next step can leave
 * out time_left and initial_weight, which that step sets again. */
int storm_cuda_get_census(StormHandle *h, StormParticlesSoA *host_out, uint64_t capacity, uint64_t *count);
int storm_cuda_census_count(StormHandle *h, uint64_t *count);
/* set_census(census_in), step(dt) and get_census(census_out) in one call, as
 * a caller that keeps its census on the host runs a step (the vector in, the
 * vector out of MonteCarloManagerSerial::step, manager/MonteCarloManagerSerial.hpp).
 * The upload runs on a stream of its own while the step's prestep, emission
 * and the transport of its new packets proceed; the census joins once it is in
 * place.  The result is the three calls' result: each particle draws from its
 * own stream and the comb orders the census by key (FP64 tally sums can differ
 * in their last bits, by their order).  The census's cells are checked before
 * the step changes any cell state: a cell outside the mesh returns
 * STORM_ERR_INVALID_ARG with the cell state unchanged and an empty census.
 * Page-locked host arrays let the upload overlap; census_out's NULL fields are
 * not written (as get_census).  Particle shards, moving material,
 * reproducible tallies, the burst tuner, profiling and the bank-visit
 * transport mode run the three calls in turn. */
int storm_cuda_step_host(StormHandle *h, double dt, const StormParticlesSoA *census_in, StormParticlesSoA *census_out,
                         uint64_t out_capacity, uint64_t *out_count, StormStepStats *stats);
/* The transport bank after storm_cuda_phase_emit: the census followed by the
 * step's cell and face source packets (RadiationIMC::generateParticles and the
 * boundary's generateNewBoundaryParticles, in that order), id = the particle's
 * stream index.  For inspecting the emission phase.  host_out = NULL returns
 * the count alone. */
int storm_cuda_get_bank(StormHandle *h, StormParticlesSoA *host_out, uint64_t capacity, uint64_t *count);
/* populationControl->activate(particles) on host particles: the result becomes
 * the handle's census (CombPopulationControl::activate,
 * population/CombPopulationControl.hpp:79-253; with comb disabled the
 * particles pass unchanged, NoPopulationControl.hpp:25-28). */
int storm_cuda_population_control(StormHandle *h, const StormParticlesSoA *host_in);

/* Per-cell arrays (host, Ncells each; any pointer may be NULL):
 * temperature [K], internal_energy [erg], erad_time_avg (getEradTimeAvg(),
 * RadiationIMC.hpp:431), erad_census (SimpleExtensives::Erad), sigma_a
 * (getPlanckOpacities), fleck (getFactorFleck), segment counters
 * (GetCellsStepsCounters, MonteCarloManagerSerial.hpp:74). */
int storm_cuda_get_cell_arrays(StormHandle *h, double *temperature, double *internal_energy,
                               double *erad_time_avg, double *erad_census,
                               double *sigma_a, double *fleck, uint64_t *segment_counters);
/* Overwrite the material state (e.g. after the caller's hydro step). */
int storm_cuda_set_cell_state(StormHandle *h, const double *temperature, const double *internal_energy,
                              const double *cell_internal_energy);
/* Overwrite the per-cell physics tables prestep would compute (sigma_a,
 * sigma_s, Fleck factor).  Replay parity uses the reference's own tables. */
int storm_cuda_set_cell_physics(StormHandle *h, const double *sigma_a, const double *sigma_s,
                                const double *fleck);
/* Replace the per-cell opacity plug-in values the next prestep reads
 * (STORM_OPACITY_CELL_TABLE: sigma_a and sigma_s per cell; STORM_OPACITY_MG_POWER:
 * sigma0 and the elastic opacity per cell); either pointer may be NULL.  The
 * reference evaluates opacity_->CalcPlanckOpacity(cell) and
 * CalcScatteringOpacity(cell) for every cell in every RadiationIMC::preStep
 * (radiation/RadiationIMC.hpp:1645); a caller whose opacity depends on the
 * cell state refreshes the tables before each step.  Other opacity kinds
 * return STORM_ERR_INVALID_ARG. */
int storm_cuda_set_opacity_tables(StormHandle *h, const double *sigma_a, const double *sigma_s);
/* Particles per cell when the last step's transport began (the census plus
 * the step's emission): MonteCarloManagerSerial::GetBeginningParticleCount
 * (manager/MonteCarloManagerSerial.hpp:81-82, filled at :419-424).  Kept only
 * for handles created with per_cell_segment_counters; others return
 * STORM_ERR_INVALID_ARG. */
int storm_cuda_get_beginning_counts(StormHandle *h, uint64_t *counts);
/* Moving material (with_hydro): the cells' velocity and the extensives'
 * momentum, 3 per cell each ([cm/s], [g cm/s]); either pointer may be NULL.
 * RadiationIMC reads cell.velocity and updates extensives[cell].momentum
 * (radiation/RadiationIMC.hpp:1793-1798, 1853-1871, 2200-2206) and sets
 * velocity = momentum / mass in synchronizeMaterialCell (:853-866).  Set
 * before a step when a hydro solver moved the cells; read after it. */
int storm_cuda_set_cell_motion(StormHandle *h, const double *velocity, const double *momentum);
int storm_cuda_get_cell_motion(StormHandle *h, double *velocity, double *momentum);
/* Group time averages of the last step (with_eg_time_avg): ncells x groups
 * doubles, cell-major (cell c, group g at c * groups + g), RadiationIMC::
 * getEgTimeAvg (radiation/RadiationIMC.hpp:433) after postStep.  Handles
 * created without them return STORM_ERR_INVALID_ARG. */
int storm_cuda_get_group_tallies(StormHandle *h, double *eg_time_avg);
/* MarshakBoundary::SetTemperature / SideTemperature::SetTemperature. */
int storm_cuda_set_face_temperature(StormHandle *h, int face, double temperature);

/* Source counts per cell of the last emission (getLastSourcePhotonsPerCell,
 * RadiationIMC.hpp:437) and the emission energy per cell. */
int storm_cuda_get_emission(StormHandle *h, uint64_t *photons_per_cell, double *energy_per_cell);

/* ---------------------------------------------------------------- parity */

/* Run each replay item as one segment fed by its uniform tape. Uses the
 * handle's mesh, per-cell tables and Random Walk tables. */
int storm_cuda_replay_segments(StormHandle *h, StormReplayBatch *batch);

/* The Random Walk tables (radiation/RandomWalk.hpp:23-79), 1024 tau values,
 * 1024 survival values, 1024*256 radius values; host buffers. */
int storm_cuda_get_random_walk_tables(StormHandle *h, double *tau, double *survival, double *radius);
/* Evaluate RandomWalk::sampleLeakTime / sampleRadius on the device for n inputs. */
int storm_cuda_random_walk_sample(StormHandle *h, uint64_t n, const double *xi_leak, const double *tau,
                                  const double *xi_radius, double *leak_out, double *radius_out);

/* ---------------------------------------------------------------- allocation-free variant */

/* Largest cell count storm_cuda_emission_allocation_noalloc accepts. */
#define STORM_NOALLOC_MAX_CELLS (1u << 24)

/* Photon counts per cell for an emission step (the per-cell counts
 * storm_cuda_phase_emit computes and storm_cuda_get_emission returns), for
 * callers that cannot allocate device memory while they run: a host
 * framework whose allocator owns the device memory, a loop with a
 * no-allocation rule.  This entry point has no counterpart in
 * the reference; it calls no cudaMalloc / cudaFree and no allocating library
 * routine.
 *   d_energy   per-cell emission energy (device, ncells)
 *   d_photons  out: photons per cell (device, ncells)
 *   d_offsets  out: exclusive prefix sum of d_photons, d_offsets[ncells] = total (device, ncells + 1)
 *   stream     cudaStream_t to run on (NULL = the legacy default stream)
 * Its scratch is one fixed array inside the library (about 128 KiB per GPU
 * that loads the library, held until exit).  The first call on a device looks
 * up that array's device address once; do not use the entry point across a
 * cudaDeviceReset of that device.  Calls whose work overlaps on the GPU share the array and race.
 * The whole computation stays on the device (no host readback), including
 * the exact left-to-right total that ambiguous floors fall back to.
 * ncells above STORM_NOALLOC_MAX_CELLS returns STORM_ERR_INVALID_ARG; a CUDA
 * error already pending on the calling thread is left pending and the call
 * returns STORM_ERR_CUDA without launching. */
int storm_cuda_emission_allocation_noalloc(int device, const double *d_energy, uint32_t ncells,
                                           uint64_t new_photons_per_cell, uint64_t *d_photons,
                                           uint64_t *d_offsets, void *stream);

/* ---------------------------------------------------------------- checkpoints */

/* The state one step hands the next -- the census bank in the handle's own
 * layout, every cell's temperature and internal energies, the face source
 * temperatures and the step counter that keys the random streams -- copied
 * to a host buffer of storm_cuda_checkpoint_size bytes, and back into a handle
 * created from the same problem (same cells, precision and groups), after
 * which the following steps repeat those of the original run.  No reference
 * counterpart: the reference's managers keep no restartable state. */
int storm_cuda_checkpoint_size(StormHandle *h, uint64_t *bytes);
int storm_cuda_checkpoint_save(StormHandle *h, void *buffer, uint64_t bytes);
int storm_cuda_checkpoint_load(StormHandle *h, const void *buffer, uint64_t bytes);

/* ---------------------------------------------------------------- meshes */

/* A bounded Voronoi tessellation of `n` generator points (3 n doubles, strictly
 * inside the box lo x, y, z, hi x, y, z), built on the host.  No reference
 * counterpart in this repository's path: the reference takes Voronoi grids from
 * the MadVoro library.  The mesh is owned by the library until storm_mesh_free. */
int storm_mesh_voronoi(const double *points, uint32_t n, const double box[6], StormPolyMesh **out);
int storm_mesh_free(StormPolyMesh *mesh);

/* ---------------------------------------------------------------- serving */

/* Many independent problems on one GPU.  A request (descriptor, steps, dt) is
 * admitted when a slot is free and its estimated device memory fits the HBM
 * budget; its census and material state then stay on the device until its
 * last step.  Worker threads advance the active problems round-robin, one time
 * step at a time, each problem on its own stream, so the work of different
 * problems overlaps on the GPU.  No reference counterpart (the reference runs
 * one problem per process). */
typedef struct StormServer StormServer;

typedef struct StormServerConfig {
    int32_t device;
    uint32_t max_active;             /* problems on the device at once */
    uint32_t workers;                /* host threads issuing steps (1-256) */
    uint32_t pad_;
    uint64_t hbm_budget_bytes;       /* admission budget (0 = 90% of free device memory) */
} StormServerConfig;

typedef struct StormRequestResult {
    uint64_t ticket;
    int32_t status;                  /* StormStatus of the request */
    uint32_t steps;                  /* time steps run */
    uint64_t segments;
    uint64_t device_bytes;           /* device memory the problem held */
    double queued_ms;                /* submission to admission (wall clock) */
    double active_ms;                /* admission to completion (wall clock) */
    double step_ms_p50, step_ms_p99, step_ms_max;   /* wall time of each step, issue to completion */
    double device_ms;                /* summed device time of its steps */
} StormRequestResult;

typedef struct StormServerStats {
    uint64_t submitted, completed, failed, active, queued;
    uint64_t segments;               /* of completed requests */
    double busy_ms;                  /* first admission to last completion (wall clock) */
    double step_ms_p50, step_ms_p99; /* over every step of every completed request */
    uint64_t peak_device_bytes;
    uint64_t budget_bytes;
} StormServerStats;

int storm_server_create(const StormServerConfig *config, StormServer **out);
/* Queue a problem.  The descriptor and its arrays are copied; temperature_out
 * (Ncells doubles, may be NULL) receives the final material temperatures and
 * must stay valid until the request's result has been polled. */
int storm_server_submit(StormServer *s, const StormProblemDesc *desc, uint32_t steps, double dt,
                        double *temperature_out, uint64_t *ticket);
/* Results of requests finished since the last poll (up to capacity). */
int storm_server_poll(StormServer *s, StormRequestResult *results, uint32_t capacity, uint32_t *count);
/* Block until every submitted request has finished. */
int storm_server_drain(StormServer *s);
int storm_server_stats(StormServer *s, StormServerStats *out);
/* Finishes the queued work, then stops the workers. */
int storm_server_destroy(StormServer *s);

/* ---------------------------------------------------------------- diagnostics */

/* First device error word, the cell and particle it was raised for, and a message. */
int storm_cuda_last_error(StormHandle *h, int32_t *derr, uint64_t *cell, uint64_t *particle,
                          char *msg, size_t msg_len);
/* Device memory freed by destroyed handles is cached for reuse by later
 * handles on the same device (cudaFree would wait for every stream on the
 * device).  This returns the cached blocks of `device` to the driver. */
int storm_cuda_release_cached(int device, uint64_t *bytes);
/* The cache's cudaMalloc and cudaFree calls since the library loaded, and the
 * bytes it holds cached and handed out, over all devices. */
int storm_cuda_pool_counters(uint64_t *mallocs, uint64_t *frees, uint64_t *cached_bytes, uint64_t *live_bytes);
/* Bytes of device memory the handle holds (GetHandlerMemoryBytes). */
int storm_cuda_memory_bytes(StormHandle *h, uint64_t *bytes);
/* Kernel launches issued by the handle since creation (for launch accounting). */
int storm_cuda_launch_count(StormHandle *h, uint64_t *launches);
/* Per-launch CUDA-event timing of the transport kernel (off by default). When
 * on, each transport launch is bracketed by events on the handle's stream and
 * storm_cuda_transport_timing() returns the summed kernel time, the number of
 * launches and the segments they ran since the last reset. */
int storm_cuda_set_profiling(StormHandle *h, int on);
int storm_cuda_transport_timing(StormHandle *h, double *kernel_ms, uint64_t *launches, uint64_t *segments, int reset);
/* Transport scheduling (autotuner hook).  refill = 1 (default): one
 * persistent launch in which each lane takes the next unstarted particle as
 * soon as its history ends, running `burst` segments between refills (default
 * 1 for multigroup problems, 4 on polyhedral meshes, 8 otherwise).
 * refill = 0: bank visits of segments_per_visit segments with survivors
 * compacted between launches. */
int storm_cuda_set_transport_mode(StormHandle *h, int refill, uint32_t burst);
/* Online tuning of the refill burst: the next 10 * steps_per_candidate calls
 * of storm_cuda_step run the bursts 1, 2, 4, 8, 16 and back (16, 8, 4, 2, 1),
 * steps_per_candidate steps each, and the burst with the most segments per
 * millisecond of transport is kept.  The burst changes no result (each
 * history's random stream is keyed by its particle), only the order of the
 * FP64 tally sums.  steps_per_candidate = 0 stops a tuning in progress and
 * keeps the current burst. */
int storm_cuda_autotune_transport(StormHandle *h, uint32_t steps_per_candidate);
/* The burst in use, and whether a tuning is in progress (1) or not (0). */
int storm_cuda_transport_burst(StormHandle *h, uint32_t *burst, int *tuning);
/* Transport kernel variant (autotuner hook): the occupancy target of the
 * kernel (__launch_bounds__ minimum blocks per SM, 1-4) and the grid size in
 * waves of resident blocks. */
int storm_cuda_set_transport_variant(StormHandle *h, int min_blocks_per_sm, int waves);
/* Segment-per-visit override (autotuner hook). */
int storm_cuda_set_segments_per_visit(StormHandle *h, uint32_t k);
const char *storm_cuda_status_string(int status);
int storm_cuda_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* STORM_CUDA_H */
