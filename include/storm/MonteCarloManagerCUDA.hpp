// MonteCarloManagerCUDA -- drop-in replacement for STORM's MonteCarloManagerSerial
// (manager/MonteCarloManagerSerial.hpp:26-117) that runs the IMC time step on a
// B200 through the C ABI in storm_cuda.h.
//
// Same constructor shape and the same step() contract:
//     std::vector<Particle<T,Grid>> step(std::vector<Particle<T,Grid>> &&census, dt_t dt)
// consumes the census and returns the post-comb census; the caller's cells and
// extensives are updated in place exactly where RadiationIMC::postStep updates
// them (radiation/RadiationIMC.hpp:1887-2029).  Getters mirror the serial
// manager's (manager/MonteCarloManagerSerial.hpp:72-83).  Errors arrive as
// STORM::StormError, after reportError, like the serial manager
// (manager/MonteCarloManagerSerial.hpp:458-462).
//
// What the plug-ins keep private -- the opacity and EOS models, the comb's
// Nmin / factor, the RNG seed, and the cell vectors RadiationIMC holds by
// reference -- is handed over in a CudaIMCBinding.  bind_parameters() copies
// the public RadiationIMCParameters, the group energy boundaries of a
// multigroup RadiationIMC included; census frequencies travel with the
// particles.  A table opacity (CELL_TABLE, MG_POWER's sigma0) is evaluated
// through the binding's callbacks for every cell before every step, as
// RadiationIMC::preStep evaluates the opacity plug-in
// (radiation/RadiationIMC.hpp:1645).
//
// The four stock boundaries are recognised by type and lowered to per-box-face
// actions without the binding: VacuumBoundary (every face escapes),
// RigidBoundary (every face reflects), SideTemperature (x-low escapes and
// emits, the rest reflect) and TwoSidesTemperature (both x faces escape and
// emit, the rest reflect).  The source temperatures and packets per face of the
// last two are private, so they are read off one batch of the boundary's own
// packets (generateNewBoundaryParticles) at construction.  Any other boundary
// takes its faces from the binding.  An unsupported plug-in or option is
// rejected with StormError; there is no CPU fallback.
//
// Include after the reference headers (Particle, MonteCarloPhysics,
// PopulationControl, BoundaryCondition, MonteCarloConfig, RadiationCell, and
// the stock boundaries boundary/Vacuum.hpp, RigidBoundary.hpp,
// SideTemperature.hpp, TwoSidesTemperature.hpp).
#ifndef STORM_MONTE_CARLO_MANAGER_CUDA_HPP
#define STORM_MONTE_CARLO_MANAGER_CUDA_HPP

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <iostream>
#include <limits>
#include <memory>
#include <set>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../storm_cuda.h"

namespace STORM {

namespace cuda_detail {
// cells that move (a `velocity`) and extensives that carry a `momentum` and
// a total `energy`: RadiationIMC's moving-material terms need the first two
template <class T, class = void> struct has_velocity : std::false_type {};
template <class T> struct has_velocity<T, std::void_t<decltype(std::declval<T &>().velocity)>> : std::true_type {};
template <class T, class = void> struct has_momentum : std::false_type {};
template <class T> struct has_momentum<T, std::void_t<decltype(std::declval<T &>().momentum)>> : std::true_type {};
template <class T, class = void> struct has_total_energy : std::false_type {};
template <class T> struct has_total_energy<T, std::void_t<decltype(std::declval<T &>().energy)>> : std::true_type {};
}  // namespace cuda_detail

template <typename CellT, typename ExtensivesT>
struct CudaIMCBinding {
    // the vectors RadiationIMC was constructed with (it mutates them in place)
    std::vector<CellT> *cells = nullptr;
    std::vector<ExtensivesT> *extensives = nullptr;
    // opacity plug-in lowered to a device descriptor
    int opacityKind = STORM_OPACITY_CELL_TABLE;
    std::function<double(std::size_t)> planckOpacity;       // CELL_TABLE: sigma_a of cell i
    std::function<double(std::size_t)> scatteringOpacity;   // CELL_TABLE: sigma_s of cell i (empty = 0)
    double kP0 = 0, kR0 = 0, alpha = 0, beta = 0, tFloor = 1.0, cap = 0;
    std::vector<double> densityFactor;                        // POWER_LAW: rho^beta per cell
    // MG_POWER (RadiationIMC<..., NumGroups> with withMultigroupOpacity):
    // sigma(E, T) = sigma0 / ((kT)^q E^p) (1 - e^{-E/kT})^s, kT = kBoltz max(T, 1 K)
    std::function<double(std::size_t)> sigma0;              // sigma0 of cell i
    std::vector<double> groupBounds;                          // NumGroups + 1 energies (bind_parameters copies them)
    double mgP = 3.0, mgQ = 0.0, mgS = 0.0, kBoltz = 0.0;
    bool mgGroupConstant = false;                             // opacity at the centre of the particle's group
    // EOS plug-in
    int eosKind = STORM_EOS_LINEAR;
    double cvPerMass = 1.0, eosF = 1.0, eosBeta = 1.0, eosMu = 0.0;
    // boundary plug-in as per-box-face actions, GetBoxFaces() order
    std::array<StormBoxFace, 6> faces{};
    bool escapeWithoutCheck = false;
    // RadiationIMCParameters<NumGroups> (copy with bind_parameters)
    std::size_t newPhotonsPerCell = 1;
    bool withRandomWalk = false, noHydroFeedback = false;
    bool withHydro = false;   // moving material: CellT::velocity and ExtensivesT::momentum (FP64 form)
    bool withEgTimeAvg = false;   // group time averages (multigroup problems): getEgTimeAvg()
    bool reproducibleTallies = false;   // fixed-point tally sums: runs repeat bit for bit
    double rwMinCellOpticalDepth = 25.0, rwMinParticleOpticalDepth = 5.0;
    bool withDDMC = false, ddmcUseMultigroupPGRW = false;
    double ddmcMinCellOpticalDepth = 15.0, ddmcMinParticleOpticalDepth = 5.0;
    // CombPopulationControl(grid, Nmin, factor), or StratifiedCombPopulationControl(grid,
    // groupCount, classifier, Nmin, factor, minParticlesPerGroup) with the classifier
    // given as frequency bin edges (groupCount + 1; empty with groupCount equal to the
    // number of energy groups: one bin per group)
    bool combEnabled = true;
    std::size_t combNmin = 20;
    double combFactor = 2.0;
    int combKind = STORM_COMB_PLAIN;
    std::uint32_t stratBins = 1;
    std::vector<double> stratBounds;
    std::size_t stratMinPerBin = 2;
    // constants the caller's physics uses (units::*)
    double clight = 0, arad = 0, sigmaSB = 0, kevKelvin = 0;
    // engine
    std::uint64_t seed = 42;
    int precision = STORM_PRECISION_FP64;
    int device = 0;
    std::uint32_t segmentsPerVisit = 0;

    template <typename ParametersT>
    void bind_parameters(const ParametersT &p) {
        newPhotonsPerCell = p.newPhotonsPerCell;
        withRandomWalk = p.withRandomWalk;
        noHydroFeedback = p.noHydroFeedback;
        rwMinCellOpticalDepth = p.rwMinCellOpticalDepth;
        rwMinParticleOpticalDepth = p.rwMinParticleOpticalDepth;
        withDDMC = p.withDDMC;
        ddmcUseMultigroupPGRW = p.ddmcUseMultigroupPGRW;
        ddmcMinCellOpticalDepth = p.ddmcMinCellOpticalDepth;
        ddmcMinParticleOpticalDepth = p.ddmcMinParticleOpticalDepth;
        constexpr bool moving = cuda_detail::has_velocity<CellT>::value && cuda_detail::has_momentum<ExtensivesT>::value;
        withHydro = p.withHydro;
        withEgTimeAvg = p.withEgTimeAvg;
        if ((p.withHydro && !moving) || p.MMC || p.withCompton || p.diffusionPressureGradient || p.postProcess.enabled) {
            StormError eo("MonteCarloManagerCUDA: RadiationIMC option not supported on the device path");
            eo.addEntry("withHydro", p.withHydro);
            eo.addEntry("MMC", p.MMC);
            eo.addEntry("withCompton", p.withCompton);
            eo.addEntry("diffusionPressureGradient", p.diffusionPressureGradient);
            eo.addEntry("postProcess.enabled", p.postProcess.enabled);
            throw eo;
        }
        groupBounds.clear();
        if (p.withMultigroupOpacity) {
            if (!p.energyBoundariesProvided || p.energyBoundaries.size() < 3)
                throw StormError("MonteCarloManagerCUDA: multigroup opacity needs the group energy boundaries");
            groupBounds.assign(p.energyBoundaries.begin(), p.energyBoundaries.end());
            opacityKind = STORM_OPACITY_MG_POWER;
        }
    }
};

namespace cuda_detail {

inline void check(int rc, StormHandle *h, const char *what) {
    if (rc == STORM_OK) return;
    StormError eo(std::string("MonteCarloManagerCUDA: ") + what + " failed");
    eo.addEntry("Status", storm_cuda_status_string(rc));
    if (h) {
        std::int32_t derr = 0;
        std::uint64_t cell = 0, particle = 0;
        char msg[256] = {0};
        storm_cuda_last_error(h, &derr, &cell, &particle, msg, sizeof(msg));
        eo.addEntry("Device error", derr);
        eo.addEntry("Cell index", cell);
        eo.addEntry("Particle", particle);
        eo.addEntry("Message", msg);
    }
    throw eo;
}

// Rectilinear edges of a Cartesian Grid through the reference Grid API: every
// face centroid lies on a plane x = const, y = const or z = const.
template <typename Grid>
std::array<std::vector<double>, 3> rectilinear_edges(const Grid &grid) {
    std::array<std::set<double>, 3> planes;
    const std::size_t N = grid.GetPointNo();
    for (std::size_t c = 0; c < N; ++c) {
        for (const std::size_t &f : grid.GetCellFaces(c)) {
            auto n = grid.Normal(f);
            auto cm = grid.FaceCM(f);
            double a[3] = {std::fabs(n.x), std::fabs(n.y), std::fabs(n.z)};
            int axis = (a[0] >= a[1] && a[0] >= a[2]) ? 0 : (a[1] >= a[2] ? 1 : 2);
            planes[axis].insert(axis == 0 ? cm.x : (axis == 1 ? cm.y : cm.z));
        }
    }
    std::array<std::vector<double>, 3> e;
    for (int a = 0; a < 3; ++a) e[a].assign(planes[a].begin(), planes[a].end());
    const std::size_t nx = e[0].size() - 1, ny = e[1].size() - 1, nz = e[2].size() - 1;
    if (e[0].size() < 2 || e[1].size() < 2 || e[2].size() < 2 || nx * ny * nz != N) {
        StormError eo("MonteCarloManagerCUDA: the grid is not a rectilinear Cartesian grid");
        eo.addEntry("Cells", N);
        throw eo;
    }
    for (std::size_t c = 0; c < N; ++c) {   // cell index = i + nx (j + ny k)
        std::size_t i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
        auto p = grid.GetMeshPoint(c);
        if (!(p.x > e[0][i] && p.x < e[0][i + 1] && p.y > e[1][j] && p.y < e[1][j + 1] && p.z > e[2][k] &&
              p.z < e[2][k + 1])) {
            StormError eo("MonteCarloManagerCUDA: cell ordering is not i + nx*(j + ny*k)");
            eo.addEntry("Cell", c);
            throw eo;
        }
    }
    return e;
}

// A grid that is not rectilinear (a Voronoi grid) lowered through the reference
// Grid API into the engine's convex-polyhedral mesh: per cell its faces in
// GetCellFaces order; per face the real cell first, its neighbour (ghost
// indices >= N kept as they are), Normal, FaceCM, GetArea and the polygon of
// GetPointsInFace over GetFacePoints; mesh points GetMeshPoint; volumes GetVolume.
struct PolyMeshArrays {
    StormPolyMesh mesh{};
    std::vector<double> points, volume, normal, cm, area, vertices;
    std::vector<std::uint32_t> cellFaceOffset, cellFaces, faceCells, faceVertexOffset, faceVertices;
};

template <typename Grid>
void lower_polyhedral(const Grid &grid, PolyMeshArrays &m) {
    const std::size_t N = grid.GetPointNo();
    const std::size_t F = grid.GetTotalFacesNumber();
    const auto box = grid.GetBoxCoordinates();
    m.points.resize(3 * N);
    m.volume.resize(N);
    m.cellFaceOffset.assign(1, 0);
    for (std::size_t c = 0; c < N; ++c) {
        const auto p = grid.GetMeshPoint(c);
        m.points[3 * c] = p.x; m.points[3 * c + 1] = p.y; m.points[3 * c + 2] = p.z;
        m.volume[c] = grid.GetVolume(c);
        for (const std::size_t &f : grid.GetCellFaces(c)) m.cellFaces.push_back(static_cast<std::uint32_t>(f));
        m.cellFaceOffset.push_back(static_cast<std::uint32_t>(m.cellFaces.size()));
    }
    const auto &nodes = grid.GetFacePoints();
    m.vertices.resize(3 * nodes.size());
    for (std::size_t v = 0; v < nodes.size(); ++v) {
        m.vertices[3 * v] = nodes[v].x; m.vertices[3 * v + 1] = nodes[v].y; m.vertices[3 * v + 2] = nodes[v].z;
    }
    m.faceVertexOffset.assign(1, 0);
    for (std::size_t f = 0; f < F; ++f) {
        auto nb = grid.GetFaceNeighbors(f);
        if (nb.first >= N) std::swap(nb.first, nb.second);
        m.faceCells.push_back(static_cast<std::uint32_t>(nb.first));
        m.faceCells.push_back(static_cast<std::uint32_t>(nb.second < N ? nb.second : N + f));
        const auto n = grid.Normal(f);
        const auto q = grid.FaceCM(f);
        m.normal.insert(m.normal.end(), {n.x, n.y, n.z});
        m.cm.insert(m.cm.end(), {q.x, q.y, q.z});
        m.area.push_back(grid.GetArea(f));
        for (const std::size_t &v : grid.GetPointsInFace(f)) m.faceVertices.push_back(static_cast<std::uint32_t>(v));
        m.faceVertexOffset.push_back(static_cast<std::uint32_t>(m.faceVertices.size()));
    }
    StormPolyMesh &d = m.mesh;
    d.ncells = static_cast<std::uint32_t>(N);
    d.nfaces = static_cast<std::uint32_t>(F);
    d.nvertices = static_cast<std::uint32_t>(nodes.size());
    d.box[0] = box.first.x; d.box[1] = box.first.y; d.box[2] = box.first.z;
    d.box[3] = box.second.x; d.box[4] = box.second.y; d.box[5] = box.second.z;
    d.points = m.points.data(); d.volume = m.volume.data();
    d.cell_face_offset = m.cellFaceOffset.data(); d.cell_faces = m.cellFaces.data(); d.face_cells = m.faceCells.data();
    d.face_normal = m.normal.data(); d.face_cm = m.cm.data(); d.face_area = m.area.data();
    d.face_vertex_offset = m.faceVertexOffset.data(); d.face_vertices = m.faceVertices.data();
    d.vertices = m.vertices.data();
}

}  // namespace cuda_detail

template <typename T, typename Grid, typename CellT = RadiationCell, typename ExtensivesT = SimpleExtensives>
class MonteCarloManagerCUDA {
    using MCParticle = Particle<T, Grid>;

public:
    // MonteCarloManagerSerial::Tracker (manager/MonteCarloManagerSerial.hpp:46-70).
    // The device path records no per-segment routes: a census particle with
    // on_track set makes step() throw StormError, so the tracker stays empty.
    class Tracker {
    public:
        void Reset(void) { track_.clear(); }
        std::vector<MCParticle> GetTrackParticleRoute(std::size_t) const { return std::vector<MCParticle>(); }

    private:
        std::vector<MCParticle> track_;
    };

    MonteCarloManagerCUDA(const Grid &grid, const std::shared_ptr<MonteCarloPhysics<T, Grid>> &physics,
                          const std::shared_ptr<PopulationControl<T, Grid>> &populationControl,
                          const std::shared_ptr<BoundaryCondition<T, Grid>> &boundaryCondition,
                          const CudaIMCBinding<CellT, ExtensivesT> &binding,
                          const MonteCarloConfig &config = MonteCarloConfig())
        : grid_(grid), physics_(physics), populationControl_(populationControl), boundary_(boundaryCondition),
          binding_(binding), config_(config) {
        if (!physics_ || !populationControl_ || !boundary_)
            throw StormError("MonteCarloManagerCUDA: physics, population control and boundary are required");
        if (!binding_.cells || !binding_.extensives)
            throw StormError("MonteCarloManagerCUDA: the binding needs the cells and extensives vectors");
        create();
    }
    ~MonteCarloManagerCUDA() {
        if (h_) storm_cuda_destroy(h_);
    }
    MonteCarloManagerCUDA(const MonteCarloManagerCUDA &) = delete;
    MonteCarloManagerCUDA &operator=(const MonteCarloManagerCUDA &) = delete;

    // MonteCarloManagerSerial::step (manager/MonteCarloManagerSerial.hpp:386-469)
    std::vector<MCParticle> step(std::vector<MCParticle> &&particleList, dt_t fullDt) {
        try {
            auto t0 = std::chrono::steady_clock::now();
            upload_cells();
            // the census goes in with the step itself (storm_cuda_step_host: its
            // upload overlaps the step's emission and new-packet transport); the
            // new census comes back below with every field
            CensusArrays in = pack_census(particleList);
            std::vector<MCParticle>().swap(particleList);
            StormStepStats st{};
            StormParticlesSoA none{};
            std::uint64_t nOut = 0;
            cuda_detail::check(storm_cuda_step_host(h_, fullDt, &in.soa, &none, 0, &nOut, &st), h_,
                               "storm_cuda_step_host");
            download_cells();
            {
                std::vector<std::uint64_t> begin(N_);
                cuda_detail::check(storm_cuda_get_beginning_counts(h_, begin.data()), h_, "get_beginning_counts");
                beginningParticleCount_.assign(begin.begin(), begin.end());
            }
            std::vector<MCParticle> out = download_census();
            initialParticleCount_ = st.census_in;
            preStepParticleCount_ = st.emitted_cells + st.emitted_faces;
            startParticleCount_ = initialParticleCount_ + preStepParticleCount_;
            endParticleCount_ = st.census_out;
            pureComputeTime_ = st.step_ms * 1e-3;
            wallTime_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            return out;
        } catch (const StormError &eo) {
            reportError(eo);
            throw;
        }
    }

    inline const std::vector<std::size_t> &GetCellsStepsCounters(void) const { return cellsStepsCounters_; }
    inline std::vector<std::size_t> &GetCellsStepsCounters(void) { return cellsStepsCounters_; }
    inline std::size_t GetStartParticleCount(void) const { return startParticleCount_; }
    inline std::size_t GetInitialParticleCount(void) const { return initialParticleCount_; }
    inline std::size_t GetPreStepParticleCount(void) const { return preStepParticleCount_; }
    inline std::size_t GetEndParticleCount(void) const { return endParticleCount_; }
    inline double GetPureComputeTime(void) const { return pureComputeTime_; }
    // particles per cell when the last step's transport began (census + emission)
    inline const std::vector<std::size_t> &GetBeginningParticleCount(void) const { return beginningParticleCount_; }
    inline std::vector<std::size_t> &GetBeginningParticleCount(void) { return beginningParticleCount_; }
    inline const Tracker &getTracker(void) { return tracker_; }
    inline void resetTracker(void) { tracker_.Reset(); }
    inline double GetWallTime(void) const { return wallTime_; }
    inline std::size_t GetHandlerMemoryBytes(void) const {
        std::uint64_t b = 0;
        storm_cuda_memory_bytes(h_, &b);
        return b;
    }
    // Erad_time_avg_ of the last step (RadiationIMC::getEradTimeAvg, radiation/RadiationIMC.hpp:431)
    inline const std::vector<double> &getEradTimeAvg(void) const { return eradAvg_; }
    inline const std::vector<double> &getPlanckOpacities(void) const { return sigmaA_; }
    // Eg_time_avg_ of the last step (RadiationIMC::getEgTimeAvg, radiation/RadiationIMC.hpp:433) for
    // multigroup problems bound with withEgTimeAvg: cell-major, the groups of cell i at
    // [i * groups, (i + 1) * groups); empty otherwise
    inline const std::vector<double> &getEgTimeAvg(void) const { return egAvg_; }
    inline const std::vector<double> &getFactorFleck(void) const { return fleck_; }
    // the boundary's drive temperature (MarshakBoundary::SetTemperature, SideTemperature::SetTemperature)
    void SetFaceTemperature(int face, double temperature) {
        cuda_detail::check(storm_cuda_set_face_temperature(h_, face, temperature), h_, "set_face_temperature");
    }

private:
    void create() {
        // a rectilinear Cartesian grid runs on the engine's Cartesian path; any
        // other grid (Voronoi) is lowered to its convex-polyhedral mesh
        std::array<std::vector<double>, 3> edges;
        bool rectilinear = true;
        try {
            edges = cuda_detail::rectilinear_edges(grid_);
        } catch (const StormError &) {
            rectilinear = false;
            cuda_detail::lower_polyhedral(grid_, poly_);
            for (auto &e : edges) e = {0.0, 1.0};
        }
        const std::size_t N = grid_.GetPointNo();
        auto &cells = *binding_.cells;
        auto &ext = *binding_.extensives;
        if (cells.size() < N || ext.size() < N) throw StormError("MonteCarloManagerCUDA: cells/extensives too small");
        std::vector<double> temp(N), mass(N), eint(N), ceint(N), sa, ss;
        for (std::size_t i = 0; i < N; ++i) {
            temp[i] = cells[i].temperature;
            mass[i] = ext[i].mass;
            eint[i] = ext[i].internal_energy;
            ceint[i] = cells[i].internalEnergy;
        }
        StormProblemDesc d;
        std::memset(&d, 0, sizeof(d));
        d.abi_version = STORM_CUDA_ABI_VERSION;
        d.precision = binding_.precision;
        d.nx = static_cast<std::uint32_t>(edges[0].size() - 1);
        d.ny = static_cast<std::uint32_t>(edges[1].size() - 1);
        d.nz = static_cast<std::uint32_t>(edges[2].size() - 1);
        d.x_edges = edges[0].data();
        d.y_edges = edges[1].data();
        d.z_edges = edges[2].data();
        d.temperature = temp.data();
        d.mass = mass.data();
        d.internal_energy = eint.data();
        d.cell_internal_energy = ceint.data();
        d.opacity_kind = binding_.opacityKind;
        if (binding_.opacityKind == STORM_OPACITY_CELL_TABLE) {
            if (!binding_.planckOpacity) throw StormError("MonteCarloManagerCUDA: CELL_TABLE opacity needs planckOpacity");
            sa.resize(N);
            ss.assign(N, 0.0);
            for (std::size_t i = 0; i < N; ++i) {
                sa[i] = binding_.planckOpacity(i);
                if (binding_.scatteringOpacity) ss[i] = binding_.scatteringOpacity(i);
            }
            d.sigma_a = sa.data();
            d.sigma_s = ss.data();
        } else if (binding_.opacityKind == STORM_OPACITY_MG_POWER) {
            if (!binding_.sigma0 || binding_.groupBounds.size() < 3 || !(binding_.kBoltz > 0.0))
                throw StormError("MonteCarloManagerCUDA: MG_POWER opacity needs sigma0, the group bounds and kBoltz");
            sa.resize(N);
            ss.assign(N, 0.0);
            for (std::size_t i = 0; i < N; ++i) {
                sa[i] = binding_.sigma0(i);
                if (binding_.scatteringOpacity) ss[i] = binding_.scatteringOpacity(i);
            }
            d.sigma_a = sa.data();
            d.sigma_s = ss.data();
            d.groups = static_cast<std::uint32_t>(binding_.groupBounds.size() - 1);
            d.group_bounds = binding_.groupBounds.data();
            d.mg_p = binding_.mgP; d.mg_q = binding_.mgQ; d.mg_s = binding_.mgS;
            d.mg_group_constant = binding_.mgGroupConstant;
            d.k_boltz = binding_.kBoltz;
            multigroup_ = true;
        }
        d.kP0 = binding_.kP0; d.kR0 = binding_.kR0; d.alpha = binding_.alpha; d.beta = binding_.beta;
        d.t_floor = binding_.tFloor;
        d.cap = binding_.cap;
        d.density_factor = binding_.densityFactor.empty() ? nullptr : binding_.densityFactor.data();
        d.eos_kind = binding_.eosKind;
        d.cv_per_mass = binding_.cvPerMass;
        d.eos_f = binding_.eosF; d.eos_beta = binding_.eosBeta; d.eos_mu = binding_.eosMu;
        std::array<StormBoxFace, 6> faces = binding_.faces;
        bool escapeNoCheck = binding_.escapeWithoutCheck;
        lower_stock_boundary(faces, escapeNoCheck);
        for (int f = 0; f < 6; ++f) d.faces[f] = faces[f];
        d.escape_without_check = escapeNoCheck;
        d.new_photons_per_cell = binding_.newPhotonsPerCell;
        d.with_random_walk = binding_.withRandomWalk;
        d.no_hydro_feedback = binding_.noHydroFeedback;
        std::vector<double> vel;
        if constexpr (cuda_detail::has_velocity<CellT>::value && cuda_detail::has_momentum<ExtensivesT>::value) {
            if (binding_.withHydro) {   // the cells' velocity (RadiationIMC reads cell.velocity)
                vel.resize(3 * N);
                for (std::size_t i = 0; i < N; ++i) {
                    vel[3 * i] = cells[i].velocity.x;
                    vel[3 * i + 1] = cells[i].velocity.y;
                    vel[3 * i + 2] = cells[i].velocity.z;
                }
                d.with_hydro = 1;
                d.cell_velocity = vel.data();
            }
        }
        d.rw_min_cell_optical_depth = binding_.rwMinCellOpticalDepth;
        d.rw_min_particle_optical_depth = binding_.rwMinParticleOpticalDepth;
        d.with_eg_time_avg = binding_.withEgTimeAvg ? 1 : 0;   // kept for multigroup problems, as in the reference
        d.reproducible_tallies = binding_.reproducibleTallies ? 1 : 0;
        d.with_ddmc = binding_.withDDMC;
        d.ddmc_use_multigroup_pgrw = binding_.ddmcUseMultigroupPGRW;
        d.ddmc_min_cell_optical_depth = binding_.ddmcMinCellOpticalDepth;
        d.ddmc_min_particle_optical_depth = binding_.ddmcMinParticleOpticalDepth;
        d.comb_enabled = binding_.combEnabled;
        d.comb_nmin = binding_.combNmin;
        d.comb_factor = binding_.combFactor;
        d.comb_kind = binding_.combKind;
        d.strat_bins = binding_.stratBins;
        d.strat_bounds = binding_.stratBounds.empty() ? nullptr : binding_.stratBounds.data();
        d.strat_min_per_bin = binding_.stratMinPerBin;
        d.clight = binding_.clight; d.arad = binding_.arad; d.sigma_sb = binding_.sigmaSB; d.kev_kelvin = binding_.kevKelvin;
        d.seed = binding_.seed;
        // MonteCarloConfig sizes the serial manager's buffer; here it seeds the bank capacity
        d.capacity = config_.initialBufferSize > 5000 ? config_.initialBufferSize : 0;
        d.segments_per_visit = binding_.segmentsPerVisit;
        d.per_cell_segment_counters = 1;
        d.device = binding_.device;
        if (!rectilinear) d.mesh = &poly_.mesh;
        cuda_detail::check(storm_cuda_create(&d, &h_), nullptr, "storm_cuda_create");
        N_ = N;
        cellsStepsCounters_.assign(N, 0);
    }

    // The stock boundaries, recognised by type (see the file comment).
    void lower_stock_boundary(std::array<StormBoxFace, 6> &faces, bool &escapeNoCheck) {
        BoundaryCondition<T, Grid> *b = boundary_.get();
        const StormBoxFace escape{STORM_FACE_ESCAPE, 0, 0.0, 0}, reflect{STORM_FACE_REFLECT, 0, 0.0, 0};
        if (dynamic_cast<VacuumBoundary<T, Grid> *>(b)) {
            faces.fill(escape);
            escapeNoCheck = true;   // VacuumBoundary::apply removes without a face test (boundary/Vacuum.hpp:18-22)
            return;
        }
        if (dynamic_cast<RigidBoundary<T, Grid> *>(b)) {
            faces.fill(reflect);
            escapeNoCheck = false;
            return;
        }
        const bool side = dynamic_cast<SideTemperature<T, Grid> *>(b) != nullptr;
        const bool two = dynamic_cast<TwoSidesTemperature<T, Grid> *>(b) != nullptr;
        if (!side && !two) return;
        // SideTemperature::apply removes at x-low and reflects at x-high
        // (boundary/SideTemperature.hpp:84-112); TwoSidesTemperature::apply
        // removes at both x faces (boundary/TwoSidesTemperature.hpp:97-123);
        // every other box face reflects.
        faces.fill(reflect);
        faces[0] = escape;
        if (two) faces[1] = escape;
        escapeNoCheck = false;
        if (!(binding_.sigmaSB > 0.0))
            throw StormError("MonteCarloManagerCUDA: the binding needs sigmaSB to lower a temperature boundary");
        // Each x-low (x-high) boundary face gets Npercell packets of weight
        // sigma_SB T^4 A dt / Npercell (:114-163, :126-199); one batch at dt = 1
        // gives both.  Packets leave the x-low face with vx > 0.
        const std::size_t N = grid_.GetPointNo();
        std::size_t xFaces[2] = {0, 0};
        std::vector<double> xArea(2 * N, 0.0);
        for (std::size_t i = 0; i < N; ++i) {
            const auto point = grid_.GetMeshPoint(i);
            for (const std::size_t &f : grid_.GetCellFaces(i)) {
                const auto nb = grid_.GetFaceNeighbors(f);
                const std::size_t o = (nb.first == i) ? nb.second : nb.first;
                if (!(o >= N && grid_.IsPointOutsideBox(o))) continue;
                const auto d = grid_.GetMeshPoint(o) - point;
                const double nx = d.x / std::sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
                if (std::fabs(nx) <= 0.99) continue;
                const int sideIdx = nx < 0 ? 0 : 1;
                ++xFaces[sideIdx];
                xArea[2 * i + sideIdx] = grid_.GetArea(f);
            }
        }
        const std::vector<MCParticle> probe = b->generateNewBoundaryParticles(1.0);
        std::size_t count[2] = {0, 0};
        double weight[2] = {-1.0, -1.0}, area[2] = {0.0, 0.0};
        for (const MCParticle &q : probe) {
            const int sideIdx = q.velocity.x > 0 ? 0 : 1;
            ++count[sideIdx];
            if (weight[sideIdx] < 0.0 && q.cellIndex < N) {
                weight[sideIdx] = q.weight;
                area[sideIdx] = xArea[2 * q.cellIndex + sideIdx];
            }
        }
        for (int sideIdx = 0; sideIdx < (two ? 2 : 1); ++sideIdx) {
            if (!xFaces[sideIdx] || !count[sideIdx]) continue;
            const std::size_t perFace = count[sideIdx] / xFaces[sideIdx];
            if (perFace * xFaces[sideIdx] != count[sideIdx] || !(area[sideIdx] > 0.0)) {
                StormError eo("MonteCarloManagerCUDA: could not read the boundary's packets per face");
                eo.addEntry("Packets", count[sideIdx]);
                eo.addEntry("Boundary faces", xFaces[sideIdx]);
                throw eo;
            }
            const double t4 = weight[sideIdx] * static_cast<double>(perFace) / (binding_.sigmaSB * area[sideIdx]);
            faces[sideIdx].source_temperature = t4 > 0.0 ? std::sqrt(std::sqrt(t4)) : 0.0;
            faces[sideIdx].packets_per_face = faces[sideIdx].source_temperature > 0.0 ? perFace : 0;
        }
    }

    void upload_cells() {
        auto &cells = *binding_.cells;
        auto &ext = *binding_.extensives;
        hostT_.resize(N_); hostE_.resize(N_); hostCE_.resize(N_);
        for (std::size_t i = 0; i < N_; ++i) {
            hostT_[i] = cells[i].temperature;
            hostE_[i] = ext[i].internal_energy;
            hostCE_[i] = cells[i].internalEnergy;
        }
        cuda_detail::check(storm_cuda_set_cell_state(h_, hostT_.data(), hostE_.data(), hostCE_.data()), h_,
                           "set_cell_state");
        if constexpr (cuda_detail::has_velocity<CellT>::value && cuda_detail::has_momentum<ExtensivesT>::value) {
            if (binding_.withHydro) {   // the velocities and momenta a hydro step may have moved
                hostV_.resize(3 * N_);
                hostM_.resize(3 * N_);
                for (std::size_t i = 0; i < N_; ++i) {
                    hostV_[3 * i] = cells[i].velocity.x; hostV_[3 * i + 1] = cells[i].velocity.y;
                    hostV_[3 * i + 2] = cells[i].velocity.z;
                    hostM_[3 * i] = ext[i].momentum.x; hostM_[3 * i + 1] = ext[i].momentum.y;
                    hostM_[3 * i + 2] = ext[i].momentum.z;
                }
                cuda_detail::check(storm_cuda_set_cell_motion(h_, hostV_.data(), hostM_.data()), h_,
                                   "set_cell_motion");
            }
        }
        // the opacity plug-in at this step's cell state (RadiationIMC::preStep, :1645)
        if (binding_.opacityKind == STORM_OPACITY_CELL_TABLE || binding_.opacityKind == STORM_OPACITY_MG_POWER) {
            hostSA_.resize(N_);
            hostSS_.assign(N_, 0.0);
            const auto &absorption = binding_.opacityKind == STORM_OPACITY_CELL_TABLE ? binding_.planckOpacity
                                                                                      : binding_.sigma0;
            for (std::size_t i = 0; i < N_; ++i) {
                hostSA_[i] = absorption(i);
                if (binding_.scatteringOpacity) hostSS_[i] = binding_.scatteringOpacity(i);
            }
            cuda_detail::check(storm_cuda_set_opacity_tables(h_, hostSA_.data(), hostSS_.data()), h_,
                               "set_opacity_tables");
        }
    }

    // a census as the C ABI's arrays (the vectors own what soa points at)
    struct CensusArrays {
        std::vector<double> x, y, z, vx, vy, vz, w, nu;
        std::vector<std::uint32_t> cell;
        StormParticlesSoA soa{};
    };
    CensusArrays pack_census(const std::vector<MCParticle> &ps) const {
        const std::size_t n = ps.size();
        for (const MCParticle &p : ps)
            if (p.on_track) {
                StormError eo("MonteCarloManagerCUDA: particle tracking (Particle::on_track) is not available on the device path");
                eo.addEntry("Particle id", p.id);
                throw eo;
            }
        // timeLeft and initialWeight are not copied: step() sets them for every
        // census particle (manager/MonteCarloManagerSerial.hpp:391-405)
        CensusArrays a;
        for (auto *v : {&a.x, &a.y, &a.z, &a.vx, &a.vy, &a.vz, &a.w}) v->resize(n);
        a.nu.resize(multigroup_ ? n : 0);
        a.cell.resize(n);
        for (std::size_t q = 0; q < n; ++q) {
            const MCParticle &p = ps[q];
            a.x[q] = p.location.x; a.y[q] = p.location.y; a.z[q] = p.location.z;
            a.vx[q] = p.velocity.x; a.vy[q] = p.velocity.y; a.vz[q] = p.velocity.z;
            a.w[q] = p.weight;
            a.cell[q] = static_cast<std::uint32_t>(p.cellIndex);
            if (multigroup_) a.nu[q] = p.frequency;
        }
        a.soa = StormParticlesSoA{a.x.data(), a.y.data(), a.z.data(), a.vx.data(), a.vy.data(), a.vz.data(), nullptr,
                                  a.w.data(), nullptr, a.cell.data(), nullptr, n, multigroup_ ? a.nu.data() : nullptr};
        return a;
    }

    std::vector<MCParticle> download_census() {
        std::uint64_t n = 0;
        cuda_detail::check(storm_cuda_census_count(h_, &n), h_, "census_count");
        std::vector<double> x(n), y(n), z(n), vx(n), vy(n), vz(n), t(n), w(n), w0(n), nu(multigroup_ ? n : 0);
        std::vector<std::uint32_t> cell(n);
        std::vector<std::uint64_t> id(n);
        StormParticlesSoA s{x.data(), y.data(), z.data(), vx.data(), vy.data(), vz.data(), t.data(), w.data(),
                            w0.data(), cell.data(), id.data(), n, multigroup_ ? nu.data() : nullptr};
        std::uint64_t got = 0;
        cuda_detail::check(storm_cuda_get_census(h_, &s, n, &got), h_, "get_census");
        std::vector<MCParticle> out(n);
        for (std::size_t q = 0; q < n; ++q) {
            MCParticle &p = out[q];
            p.location = T(x[q], y[q], z[q]);
            p.velocity = T(vx[q], vy[q], vz[q]);
            p.timeLeft = t[q]; p.weight = w[q]; p.initialWeight = w0[q];
            p.cellIndex = cell[q];
            p.frequency = multigroup_ ? nu[q] : 0.0;
            p.id = std::numeric_limits<std::size_t>::max();   // ids are reassigned at the next step, as comb copies are
        }
        return out;
    }

    // RadiationIMC::postStep's writes into the caller's state (:1887-2029)
    void download_cells() {
        std::vector<double> temp(N_), eint(N_), eradCensus(N_);
        std::vector<std::uint64_t> segs(N_);
        eradAvg_.resize(N_); sigmaA_.resize(N_); fleck_.resize(N_);
        cuda_detail::check(storm_cuda_get_cell_arrays(h_, temp.data(), eint.data(), eradAvg_.data(), eradCensus.data(),
                                                      sigmaA_.data(), fleck_.data(), segs.data()),
                           h_, "get_cell_arrays");
        auto &cells = *binding_.cells;
        auto &ext = *binding_.extensives;
        for (std::size_t i = 0; i < N_; ++i) {
            cellsStepsCounters_[i] = segs[i];
            ext[i].internal_energy = eint[i];
            cells[i].temperature = temp[i];
            if (!binding_.noHydroFeedback) cells[i].internalEnergy = eint[i];   // synchronizeMaterialCell, radiation/RadiationIMC.hpp:831-848
            ext[i].Erad = eradCensus[i];
            cells[i].Erad = ext[i].mass > 0.0 ? eradCensus[i] / ext[i].mass : 0.0;
        }
        if (binding_.withEgTimeAvg && multigroup_) {   // postStep's group time averages (:1896-1902)
            egAvg_.resize(N_ * (binding_.groupBounds.size() - 1));
            cuda_detail::check(storm_cuda_get_group_tallies(h_, egAvg_.data()), h_, "get_group_tallies");
        }
        if constexpr (cuda_detail::has_velocity<CellT>::value && cuda_detail::has_momentum<ExtensivesT>::value) {
            if (binding_.withHydro) {   // momentum deposits and velocity = momentum / mass (:853-866)
                hostV_.resize(3 * N_);
                hostM_.resize(3 * N_);
                cuda_detail::check(storm_cuda_get_cell_motion(h_, hostV_.data(), hostM_.data()), h_, "get_cell_motion");
                for (std::size_t i = 0; i < N_; ++i) {
                    ext[i].momentum.x = hostM_[3 * i]; ext[i].momentum.y = hostM_[3 * i + 1];
                    ext[i].momentum.z = hostM_[3 * i + 2];
                    cells[i].velocity.x = hostV_[3 * i]; cells[i].velocity.y = hostV_[3 * i + 1];
                    cells[i].velocity.z = hostV_[3 * i + 2];
                    if constexpr (cuda_detail::has_total_energy<ExtensivesT>::value) {
                        const double p2 = hostM_[3 * i] * hostM_[3 * i] + hostM_[3 * i + 1] * hostM_[3 * i + 1] +
                                          hostM_[3 * i + 2] * hostM_[3 * i + 2];
                        ext[i].energy = ext[i].internal_energy + 0.5 * p2 / ext[i].mass;
                    }
                }
            }
        }
    }

    const Grid &grid_;
    std::shared_ptr<MonteCarloPhysics<T, Grid>> physics_;
    std::shared_ptr<PopulationControl<T, Grid>> populationControl_;
    std::shared_ptr<BoundaryCondition<T, Grid>> boundary_;
    CudaIMCBinding<CellT, ExtensivesT> binding_;
    MonteCarloConfig config_;
    StormHandle *h_ = nullptr;
    std::size_t N_ = 0;
    bool multigroup_ = false;
    cuda_detail::PolyMeshArrays poly_;
    std::vector<std::size_t> cellsStepsCounters_;
    std::vector<double> hostT_, hostE_, hostCE_, hostSA_, hostSS_, hostV_, hostM_, eradAvg_, sigmaA_, fleck_, egAvg_;
    std::vector<std::size_t> beginningParticleCount_;
    Tracker tracker_;
    std::size_t startParticleCount_ = 0, initialParticleCount_ = 0, preStepParticleCount_ = 0, endParticleCount_ = 0;
    double pureComputeTime_ = 0.0, wallTime_ = 0.0;
};

}  // namespace STORM

#endif
