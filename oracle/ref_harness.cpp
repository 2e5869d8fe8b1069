// Test infrastructure only (the oracle's reference build).  Nothing in the
// product links, loads or runs this file.
//
// Builds STORM's own serial path -- MonteCarloManagerSerial + RadiationIMC +
// CombPopulationControl + boundary plug-ins, compiled unmodified from the
// reference sources -- against the project-written stand-ins in oracle/shims
// for the dependencies the reference does not vendor (Boost pieces, `units`,
// `planck_integral`, a MadCart-compatible Cartesian grid).  It exposes a C API
// so the tests can:
//   * run full reference time steps on the same problem descriptor the CUDA
//     engine takes (CPU baseline and statistical parity),
//   * record, for every RadiationIMC::step call, the particle before/after,
//     the tallies before/after and the exact uniforms the call drew from the
//     reference's private std::mt19937_64 (replay parity),
//   * probe single components (RandomWalk samplers, the in-cell and on-face
//     position samplers, isotropic directions, comb) with recorded draws.
//
// The engine is reached through the opacity plug-in: RadiationIMC passes its
// private engine by reference to getRandomVelocity (radiation/RadiationIMC.hpp:2543),
// so the harness opacity model keeps the address on first use.  Engine states
// compare with ==, so the draws of one step are counted by advancing a copy
// taken before the call, and replayed through a second copy to log the doubles.
#include <algorithm>
#include <array>
#include <cassert>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "examples/Vector3D.hpp"
#include "MadCart/CartesianMesh3D.hpp"
#include <units/units.hpp>
#include "radiation/RadiationIMC.hpp"
#include "radiation/RadiationCell.hpp"
#include "radiation/RandomWalk.hpp"
#include "population/CombPopulationControl.hpp"
#include "population/NoPopulationControl.hpp"
#include "boundary/RigidBoundary.hpp"
#include "boundary/Vacuum.hpp"
#include "boundary/SideTemperature.hpp"
#include "boundary/TwoSidesTemperature.hpp"
#include "manager/MonteCarloManagerSerial.hpp"
#include "utils/RandomInCell.hpp"
#include "utils/RandomOnFace.hpp"
#include "utils/LinearInterpolation.hpp"
#include <planck_integral/planck_integral.hpp>

#include "storm_cuda.h"

using Grid = MadCart::CartesianMesh3D<Vector3D>;
// Cells with a velocity and extensives with a momentum: RadiationIMC's coupling
// to moving material (withHydro) compiles in only for such types.  Without
// withHydro its hydro branches stay inactive, and the results are those of the
// plain RadiationCell / SimpleExtensives.
struct Cell : STORM::RadiationCell {
    Vector3D velocity;
};
struct Ext : STORM::SimpleExtensives {
    Vector3D momentum;
};
using MCParticle = STORM::Particle<Vector3D, Grid>;

namespace {

// ------------------------------------------------------------------ EOS
// Linear EOS as examples/densmore2012/main.cpp:56-77; power law as
// examples/marshak_wave/MarshakCommon.hpp:138-155, 162-183.
struct HarnessEOS {
    int kind = STORM_EOS_LINEAR;
    double cvPerMass = 1.0, f = 1.0, beta = 1.0, mu = 0.0;
    double dT2cv(double density, double temperature, const std::vector<double> &, const std::vector<std::string> &) const {
        if (kind == STORM_EOS_LINEAR) return cvPerMass;
        double cvVol = f * beta * std::pow(std::max(temperature, 1.0), beta - 1.0) * std::pow(density, 1.0 - mu);
        return cvVol / density;
    }
    double de2T(double density, double specificEnergy, const std::vector<double> &, const std::vector<std::string> &) const {
        if (kind == STORM_EOS_LINEAR) return (cvPerMass > 0.0) ? specificEnergy / cvPerMass : 0.0;
        double energyPerVolume = specificEnergy * density;
        double rhoFactor = std::pow(density, 1.0 - mu);
        double ratio = std::max(energyPerVolume, 0.0) / (f * rhoFactor);
        return std::pow(std::max(ratio, 0.0), 1.0 / beta);
    }
};

// ------------------------------------------------------------------ opacity
// Gray (NumGroups = 1): per-cell table or the Marshak power law.  Multigroup
// (STORM_OPACITY_MG_POWER): sigma(E, T) = sigma0[cell] / ((kT)^q E^p) (1 - e^{-E/kT})^s
// with the group machinery of examples/densmore2012/DensmoreOpacity.hpp:36-165
// (Planck mean and emission spectrum from group centres weighted by
// planck_integral, inverse-CDF sampling by LinearInterpolation).
template <std::size_t G>
class HarnessOpacityT : public STORM::RadiationOpacityModel<Vector3D, Grid, Cell, G> {
public:
    using Base = STORM::RadiationOpacityModel<Vector3D, Grid, Cell, G>;
    using GroupArray = typename Base::GroupArray;
    using GroupBoundaries = typename Base::GroupBoundaries;
    using GroupCdf = std::array<double, G + 1>;
    int kind = STORM_OPACITY_CELL_TABLE;
    std::vector<double> sigA, sigS, rhoFactor;
    double kP0 = 0, kR0 = 0, alpha = 0, tFloor = 1.0, cap = 0, kevKelvin = units::kev_kelvin;
    GroupBoundaries bounds{};
    bool groupConstant = false;
    double mgP = 3.0, mgQ = 0.0, mgS = 0.0, kBoltz = units::k_boltz;
    const std::vector<Cell> *cells = nullptr;
    std::mt19937_64 *captured = nullptr;

    double CalcPlanckOpacity(const Cell &cell) override {
        std::size_t i = index(cell);
        if (kind == STORM_OPACITY_MG_POWER) {
            double kT = kBoltz * std::max(cell.temperature, 1.0);
            double weightedSum = 0, totalWeight = 0;
            for (std::size_t g = 0; g < G; ++g) {
                double Ec = 0.5 * (bounds[g] + bounds[g + 1]);
                double a = bounds[g] / kT, b = bounds[g + 1] / kT;
                double Bg = (a > 0.0 && b > a) ? planck_integral::planck_integral(a, b) : 0.0;
                weightedSum += sigmaAt(i, Ec, kT) * Bg;
                totalWeight += Bg;
            }
            return (totalWeight > 0) ? weightedSum / totalWeight : 1e-20;
        }
        if (kind == STORM_OPACITY_CELL_TABLE) return sigA[i];
        double tf = std::pow(kevKelvin / std::max(cell.temperature, tFloor), alpha);
        double k = kP0 * tf * rf(i);
        return (cap > 0.0) ? std::min(k, cap) : k;
    }
    double CalcAbsorptionOpacity(const Cell &cell, double frequency) override {
        if (kind != STORM_OPACITY_MG_POWER) return CalcPlanckOpacity(cell);
        std::size_t i = index(cell);
        double kT = kBoltz * std::max(cell.temperature, 1.0);
        double E;
        if (groupConstant) {
            std::size_t g = this->findGroup(frequency, bounds);
            E = 0.5 * (bounds[g] + bounds[g + 1]);
        } else {
            E = std::max(frequency, bounds[0]);
        }
        return sigmaAt(i, E, kT);
    }
    double CalcScatteringOpacity(const Cell &cell) override {
        std::size_t i = index(cell);
        if (kind == STORM_OPACITY_CELL_TABLE || kind == STORM_OPACITY_MG_POWER) return sigS.empty() ? 0.0 : sigS[i];
        if (!(kR0 > 0.0)) return 0.0;
        double tf = std::pow(kevKelvin / std::max(cell.temperature, tFloor), alpha);
        double kR = kR0 * tf * rf(i);
        double kP = kP0 * tf * rf(i);
        return std::max(kR - kP, 0.0);
    }
    double GetThermalEnergy(const Cell &cell, double random, const GroupBoundaries &boundaries) const override {
        if (kind != STORM_OPACITY_MG_POWER) return Base::GetThermalEnergy(cell, random, boundaries);
        GroupCdf cumulative = cumulativePlanck(cell, boundaries);
        double total = cumulative[G];
        if (!(total > 0.0) || !std::isfinite(total)) return Base::GetThermalEnergy(cell, random, boundaries);
        double r = std::isfinite(random) ? std::clamp(random, 0.0, std::nextafter(1.0, 0.0)) : 0.5;
        return STORM::LinearInterpolation(cumulative, boundaries, r * total);
    }
    GroupArray GetCumulativeOpacity(const Cell &cell, const GroupBoundaries &boundaries) const override {
        if (kind != STORM_OPACITY_MG_POWER) return Base::GetCumulativeOpacity(cell, boundaries);
        GroupArray upper{};
        GroupCdf cumulative = cumulativePlanck(cell, boundaries);
        for (std::size_t g = 0; g < G; ++g) upper[g] = cumulative[g + 1];
        return upper;
    }
    Vector3D getRandomVelocity(const Cell &cell, std::mt19937_64 &rng, std::uniform_real_distribution<double> &dist) override {
        captured = &rng;
        return Base::getRandomVelocity(cell, rng, dist);
    }
    static Vector3D isotropic(std::mt19937_64 &rng, std::uniform_real_distribution<double> &dist) {
        return Base::isotropicVelocity(rng, dist);
    }
    double sigmaAt(std::size_t i, double E, double kT) const {
        double v = sigA[i] / (std::pow(kT, mgQ) * std::pow(E, mgP));
        if (mgS != 0.0) v *= std::pow(-std::expm1(-E / kT), mgS);
        return v;
    }

private:
    std::size_t index(const Cell &cell) const { return static_cast<std::size_t>(&cell - cells->data()); }
    double rf(std::size_t i) const { return rhoFactor.empty() ? 1.0 : rhoFactor[i]; }
    GroupCdf cumulativePlanck(const Cell &cell, const GroupBoundaries &boundaries) const {
        GroupCdf cdf{};
        cdf[0] = 0.0;
        std::size_t i = index(cell);
        double kT = kBoltz * std::max(cell.temperature, 1.0);
        for (std::size_t g = 0; g < G; ++g) {
            double a = boundaries[g] / kT, b = boundaries[g + 1] / kT;
            double bg = (a > 0.0 && b > a) ? planck_integral::planck_integral(a, b) : 0.0;
            double Ec = 0.5 * (boundaries[g] + boundaries[g + 1]);
            double sg = sigmaAt(i, Ec, kT);
            double weight = (sg > 0.0 && std::isfinite(sg) && std::isfinite(bg)) ? sg * bg : 0.0;
            cdf[g + 1] = cdf[g] + weight;
        }
        return cdf;
    }
};
using HarnessOpacity = HarnessOpacityT<1>;

// ------------------------------------------------------------------ boundary
// A per-box-face boundary plug-in written against STORM's BoundaryCondition
// API (the same shape as examples/marshak_wave/MarshakBoundary.hpp): faces
// either escape or reflect with the reference's own reflectParticleOnBoxFace;
// faces with a source temperature emit Planck surface packets like
// SideTemperature::generateNewBoundaryParticles (boundary/SideTemperature.hpp:114-163),
// including TwoSidesTemperature's outside-box repair (boundary/TwoSidesTemperature.hpp:178-189).
// With group bounds set (multigroup problems) each packet's frequency follows
// DensmoreBoundary::generateNewBoundaryParticles
// (examples/densmore2012/DensmoreBoundary.hpp:99-109, 128-139): a group from the
// face's cumulative Planck integrals, then a uniform energy inside it.
class HarnessBoundary : public STORM::BoundaryCondition<Vector3D, Grid> {
public:
    StormBoxFace faces[6];
    bool escapeNoCheck = false;
    double sigmaSB = units::sigma_sb, clight = units::clight;
    double escaped = 0.0;
    std::vector<double> bounds;   // groups + 1 energies [erg]; empty for gray problems
    double kBoltz = units::k_boltz;
    std::mt19937_64 re{0};

    explicit HarnessBoundary(const Grid &g) : STORM::BoundaryCondition<Vector3D, Grid>(g) { std::memset(faces, 0, sizeof(faces)); }

    STORM::ParticleStatus apply(MCParticle &particle) override {
        if (escapeNoCheck) {
            escaped += particle.weight;
            return STORM::ParticleStatus::REMOVE;
        }
        STORM::ParticleStatus status = STORM::ParticleStatus::DONE;
        const auto &bfs = this->grid.GetBoxFaces();
        for (std::size_t f = 0; f < bfs.size(); ++f) {
            Vector3D normal;
            double faceScale = 0.0;
            if (this->getInwardBoxFaceNormalIfClose(bfs[f], particle.location, normal, faceScale)) {
                if (faces[f].action == STORM_FACE_ESCAPE) {
                    escaped += particle.weight;
                    return STORM::ParticleStatus::REMOVE;
                }
                if (this->reflectParticleOnBoxFace(particle, bfs[f])) status = STORM::ParticleStatus::REFLECT;
            }
        }
        if (status == STORM::ParticleStatus::REFLECT) return status;
        STORM::StormError eo("Particle is not on any boundary");
        eo.addEntry("Particle", particle);
        throw eo;
    }

    std::vector<MCParticle> generateNewBoundaryParticles(double fullDt) override {
        std::uniform_real_distribution<double> unif(0, 1);
        std::vector<MCParticle> out;
        std::size_t N = this->grid.GetPointNo();
        for (std::size_t i = 0; i < N; ++i) {
            const Vector3D &point = this->grid.GetMeshPoint(i);
            for (const std::size_t &faceIdx : this->grid.GetCellFaces(i)) {
                const auto &nb = this->grid.GetFaceNeighbors(faceIdx);
                std::size_t nbIdx = (nb.first == i) ? nb.second : nb.first;
                if (!(nbIdx >= N && this->grid.IsPointOutsideBox(nbIdx))) continue;
                Vector3D out_n = STORM::fallback::normalize(this->grid.GetMeshPoint(nbIdx) - point);
                int bf = -1, axis = 0;
                double sgn = 1.0;
                if (out_n.x < -0.99) { bf = 0; axis = 0; sgn = 1.0; }
                else if (out_n.x > 0.99) { bf = 1; axis = 0; sgn = -1.0; }
                else if (out_n.y < -0.99) { bf = 2; axis = 1; sgn = 1.0; }
                else if (out_n.y > 0.99) { bf = 3; axis = 1; sgn = -1.0; }
                else if (out_n.z < -0.99) { bf = 4; axis = 2; sgn = 1.0; }
                else if (out_n.z > 0.99) { bf = 5; axis = 2; sgn = -1.0; }
                if (bf < 0 || !(faces[bf].source_temperature > 0.0) || faces[bf].packets_per_face == 0) continue;
                const std::size_t Np = faces[bf].packets_per_face;
                const double T4 = boost::math::pow<4>(faces[bf].source_temperature);
                double energyToProduce = sigmaSB * T4 * this->grid.GetArea(faceIdx) * fullDt / Np;
                const std::size_t G = bounds.empty() ? 0 : bounds.size() - 1;
                std::vector<double> cdf(G + 1, 0.0);
                if (G) {
                    const double kT = kBoltz * faces[bf].source_temperature;
                    for (std::size_t g = 0; g < G; ++g) {
                        double a = bounds[g] / kT, b = bounds[g + 1] / kT;
                        double bg = (a > 0.0 && b > a) ? planck_integral::planck_integral(a, b) : 0.0;
                        cdf[g + 1] = cdf[g] + bg;
                    }
                }
                for (std::size_t j = 0; j < Np; ++j) {
                    out.emplace_back();
                    MCParticle &p = out.back();
                    p.location = STORM::RandomPointOnFace<Vector3D, Grid>(this->grid, faceIdx);
                    double mu = std::sqrt(unif(re));
                    double v[3];
                    v[axis] = sgn * mu;
                    double _1mmu = std::sqrt(1 - mu * mu);
                    double theta = 2 * M_PI * unif(re);
                    v[(axis + 1) % 3] = _1mmu * std::cos(theta);
                    v[(axis + 2) % 3] = _1mmu * std::sin(theta);
                    p.velocity = Vector3D(v[0], v[1], v[2]);
                    p.velocity *= clight;
                    p.frequency = 0;
                    if (G) {
                        const double total = cdf[G];
                        if (total > 0.0) {
                            double r = unif(re) * total;
                            std::size_t g = 0;
                            while (g + 1 < G && cdf[g + 1] < r) ++g;
                            p.frequency = bounds[g] + unif(re) * (bounds[g + 1] - bounds[g]);
                        } else {
                            p.frequency = 0.5 * (bounds[0] + bounds[G]);
                        }
                    }
                    p.weight = energyToProduce;
                    p.initialWeight = p.weight;
                    p.timeLeft = fullDt * unif(re);
                    p.cellIndex = i;
                    if (this->grid.IsPointOutsideBox(p.location)) {
                        Vector3D original = p.location;
                        Vector3D direction = point - original;
                        double t = 1e-8;
                        while (this->grid.IsPointOutsideBox(p.location) && t < 1.0) {
                            p.location = original + t * direction;
                            t *= 2;
                        }
                        p.location = p.location + 1e-8 * (point - p.location);
                    }
                }
            }
        }
        return out;
    }
};

// ------------------------------------------------------------------ recording IMC
struct Record {
    uint64_t id;
    uint32_t cell;
    double before[9];   // x y z vx vy vz timeLeft weight initialWeight
    double after[8];    // x y z vx vy vz timeLeft weight
    int32_t status;
    uint64_t nextCell;
    double ematBefore, ematAfter, eradBefore, eradAfter;
    uint64_t tapeOffset;
    uint32_t tapeLength;
    int32_t usedRW;
    double freqBefore, freqAfter;
    double momBefore[3], momAfter[3];   // the cell's momentum (hydro)
};

struct RecordState {
    bool recording = false;
    std::size_t maxRecords = 0;
    std::vector<Record> records;
    std::vector<double> tape;
};

template <std::size_t G>
using IMCBaseT = STORM::RadiationIMC<Vector3D, Grid, Cell, Ext, HarnessEOS, G>;

template <std::size_t G>
class RecordingIMC : public IMCBaseT<G> {
public:
    using Base = IMCBaseT<G>;
    using Functionality = typename Base::Functionality;
    using Base::Base;
    HarnessOpacityT<G> *opac = nullptr;
    std::vector<Ext> *ext = nullptr;
    RecordState rs;

    Functionality step(MCParticle &p, std::vector<MCParticle> &add) override {
        if (!rs.recording || opac == nullptr || opac->captured == nullptr || rs.records.size() >= rs.maxRecords)
            return Base::step(p, add);
        Record r{};
        r.id = p.id;
        r.cell = static_cast<uint32_t>(p.cellIndex);
        const std::size_t c = p.cellIndex;
        double b[9] = {p.location.x, p.location.y, p.location.z, p.velocity.x, p.velocity.y, p.velocity.z,
                       p.timeLeft, p.weight, p.initialWeight};
        std::memcpy(r.before, b, sizeof(b));
        r.freqBefore = p.frequency;
        r.eradBefore = this->getEradTimeAvg()[c];
        r.ematBefore = (*ext)[c].internal_energy;
        {
            const Vector3D &m = (*ext)[c].momentum;
            r.momBefore[0] = m.x; r.momBefore[1] = m.y; r.momBefore[2] = m.z;
        }
        std::mt19937_64 snap = *opac->captured;
        std::size_t rwBefore = this->getRandomWalkStepCount();
        std::size_t ddmcBefore = this->getDDMCStepCount();
        Functionality res = Base::step(p, add);
        std::mt19937_64 counter = snap;
        uint32_t n = 0;
        while (!(counter == *opac->captured)) {
            counter.discard(1);
            if (++n > 4096) throw STORM::StormError("recording: could not match the engine state");
        }
        std::uniform_real_distribution<double> dist(0.0, 1.0);
        r.tapeOffset = rs.tape.size();
        r.tapeLength = n;
        for (uint32_t k = 0; k < n; ++k) rs.tape.push_back(dist(snap));
        double a[8] = {p.location.x, p.location.y, p.location.z, p.velocity.x, p.velocity.y, p.velocity.z,
                       p.timeLeft, p.weight};
        std::memcpy(r.after, a, sizeof(a));
        r.freqAfter = p.frequency;
        r.status = static_cast<int32_t>(res.change);
        r.nextCell = res.nextCellIndex;
        r.eradAfter = this->getEradTimeAvg()[c];
        r.ematAfter = (*ext)[c].internal_energy;
        {
            const Vector3D &m = (*ext)[c].momentum;
            r.momAfter[0] = m.x; r.momAfter[1] = m.y; r.momAfter[2] = m.z;
        }
        // 1: a Random Walk jump, 2: a DDMC step (tryDDMCStep took the segment)
        r.usedRW = (this->getRandomWalkStepCount() != rwBefore) ? 1 : (this->getDDMCStepCount() != ddmcBefore ? 2 : 0);
        rs.records.push_back(r);
        return res;
    }
};

// The RadiationIMC calls the C API needs, independent of the group count.
struct PhysicsView {
    virtual ~PhysicsView() = default;
    virtual void updateGridData() = 0;
    virtual std::vector<MCParticle> preStep(double dt) = 0;
    virtual const std::vector<double> &eradTimeAvg() const = 0;
    virtual const std::vector<double> &planckOpacities() const = 0;
    virtual const std::vector<double> &factorFleck() const = 0;
    virtual std::vector<std::size_t> lastSourcePhotonsPerCell() const = 0;
    virtual std::size_t randomWalkStepCount() const = 0;
    virtual RecordState &records() = 0;
    virtual int thermalEnergy(uint64_t n, const uint32_t *cells, const double *xi, double *energy) = 0;
    virtual int groupTallies(double *out) const = 0;   // getEgTimeAvg, cell-major
};
template <std::size_t G>
struct PhysicsViewT : PhysicsView {
    std::shared_ptr<RecordingIMC<G>> p;
    explicit PhysicsViewT(std::shared_ptr<RecordingIMC<G>> q) : p(std::move(q)) {}
    void updateGridData() override { p->updateGridData(); }
    std::vector<MCParticle> preStep(double dt) override { return p->preStep(dt); }
    const std::vector<double> &eradTimeAvg() const override { return p->getEradTimeAvg(); }
    const std::vector<double> &planckOpacities() const override { return p->getPlanckOpacities(); }
    const std::vector<double> &factorFleck() const override { return p->getFactorFleck(); }
    std::vector<std::size_t> lastSourcePhotonsPerCell() const override {
        const auto &v = p->getLastSourcePhotonsPerCell();
        return std::vector<std::size_t>(v.begin(), v.end());
    }
    std::size_t randomWalkStepCount() const override { return p->getRandomWalkStepCount(); }
    RecordState &records() override { return p->rs; }
    int thermalEnergy(uint64_t n, const uint32_t *cells, const double *xi, double *energy) override {
        typename HarnessOpacityT<G>::GroupBoundaries b = p->opac->bounds;
        for (uint64_t k = 0; k < n; ++k) energy[k] = p->opac->GetThermalEnergy((*p->opac->cells)[cells[k]], xi[k], b);
        return 0;
    }
    int groupTallies(double *out) const override {
        const auto &eg = p->getEgTimeAvg();
        if (G < 2 || eg.empty()) return 1;
        for (std::size_t i = 0; i < eg.size(); ++i)
            for (std::size_t g = 0; g < G; ++g) out[i * G + g] = eg[i][g];
        return 0;
    }
};

class NullBuf : public std::streambuf {
protected:
    int overflow(int c) override { return c; }
};

} // namespace

// ------------------------------------------------------------------ handle
struct RefHandle {
    std::vector<double> xe, ye, ze;
    std::unique_ptr<Grid> grid;
    std::vector<Cell> cells;
    std::vector<Ext> ext;
    std::shared_ptr<HarnessEOS> eos;
    std::shared_ptr<STORM::BoundaryCondition<Vector3D, Grid>> boundary;
    HarnessBoundary *harnessBoundary = nullptr;
    std::shared_ptr<STORM::MonteCarloPhysics<Vector3D, Grid>> physics;   // RecordingIMC<G>
    std::unique_ptr<PhysicsView> view;
    std::shared_ptr<STORM::PopulationControl<Vector3D, Grid>> pop;
    std::unique_ptr<STORM::MonteCarloManagerSerial<Vector3D, Grid>> manager;
    std::vector<MCParticle> census;
    std::string lastError;
};

// Multigroup instantiations of RadiationIMC held by this build: 30 groups (the
// Densmore 2012 benchmark) and 64 groups (the 128^3 multigroup cube).
constexpr std::size_t kMGGroupsA = 30, kMGGroupsB = 64;

// RadiationIMC<..., G> with the harness opacity plug-in built from the descriptor.
template <std::size_t G>
void build_physics(RefHandle &h, const StormProblemDesc *d) {
    const std::size_t N = h.grid->GetPointNo();
    auto opacity = std::make_shared<HarnessOpacityT<G>>();
    auto &op = *opacity;
    op.kind = d->opacity_kind;
    op.cells = &h.cells;
    if (d->opacity_kind == STORM_OPACITY_CELL_TABLE || d->opacity_kind == STORM_OPACITY_MG_POWER) {
        op.sigA.assign(d->sigma_a, d->sigma_a + N);
        if (d->sigma_s) op.sigS.assign(d->sigma_s, d->sigma_s + N);
    } else {
        op.kP0 = d->kP0; op.kR0 = d->kR0; op.alpha = d->alpha; op.tFloor = d->t_floor; op.cap = d->cap;
        op.kevKelvin = d->kev_kelvin;
        if (d->density_factor) op.rhoFactor.assign(d->density_factor, d->density_factor + N);
    }
    STORM::RadiationIMCParameters<G> p;
    if constexpr (G > 1) {
        for (std::size_t g = 0; g <= G; ++g) op.bounds[g] = d->group_bounds[g];
        op.groupConstant = d->mg_group_constant != 0;
        op.mgP = d->mg_p; op.mgQ = d->mg_q; op.mgS = d->mg_s;
        op.kBoltz = d->k_boltz;
        p.withMultigroupOpacity = true;
        p.energyBoundaries = op.bounds;
        p.energyBoundariesProvided = true;
    }
    p.newPhotonsPerCell = d->new_photons_per_cell;
    p.withRandomWalk = d->with_random_walk != 0;
    p.rwMinCellOpticalDepth = d->rw_min_cell_optical_depth;
    p.rwMinParticleOpticalDepth = d->rw_min_particle_optical_depth;
    p.noHydroFeedback = d->no_hydro_feedback != 0;
    p.withDDMC = d->with_ddmc != 0;
    p.ddmcUseMultigroupPGRW = d->ddmc_use_multigroup_pgrw != 0;
    p.ddmcMinCellOpticalDepth = d->ddmc_min_cell_optical_depth;
    p.ddmcMinParticleOpticalDepth = d->ddmc_min_particle_optical_depth;
    p.withHydro = d->with_hydro != 0;
    p.withEgTimeAvg = d->with_eg_time_avg != 0;
    auto physics = std::make_shared<RecordingIMC<G>>(*h.grid, h.boundary, h.cells, h.ext, h.eos, opacity, p,
                                                     STORM::DirectRadiationIMCTraits<Vector3D, Cell, Ext, G>(),
                                                     RandomInCellPositionSampler<Vector3D, Grid>(), d->seed);
    physics->opac = opacity.get();
    physics->ext = &h.ext;
    h.physics = physics;
    h.view = std::make_unique<PhysicsViewT<G>>(physics);
}

extern "C" {

typedef struct RefStepOut {
    uint64_t initial, prestep, start, end, segments, rw_steps;
    double wall_seconds;
    double escaped_energy;
} RefStepOut;

// boundary_kind: 0 per-face descriptor (HarnessBoundary), 1 RigidBoundary,
// 2 VacuumBoundary, 3 SideTemperature(faces[0]), 4 TwoSidesTemperature(faces[0], faces[1]).
RefHandle *ref_create(const StormProblemDesc *d, int boundary_kind, char *err, size_t errlen) {
    try {
        auto h = std::make_unique<RefHandle>();
        if (d->mesh) {   // a convex-polyhedral mesh, in the grid stand-in's polyhedral mode
            const StormPolyMesh *m = d->mesh;
            const std::size_t n = m->ncells, F = m->nfaces;
            std::vector<Vector3D> pts(n), nrm(F), cm(F), nodes(m->nvertices);
            for (std::size_t c = 0; c < n; ++c) pts[c] = Vector3D(m->points[3 * c], m->points[3 * c + 1], m->points[3 * c + 2]);
            std::vector<std::vector<std::size_t>> cf(n), fv(F);
            for (std::size_t c = 0; c < n; ++c)
                for (uint32_t q = m->cell_face_offset[c]; q < m->cell_face_offset[c + 1]; ++q) cf[c].push_back(m->cell_faces[q]);
            std::vector<std::pair<std::size_t, std::size_t>> fn(F);
            std::vector<double> area(m->face_area, m->face_area + F), vol(m->volume, m->volume + n);
            for (std::size_t f = 0; f < F; ++f) {
                fn[f] = {m->face_cells[2 * f], m->face_cells[2 * f + 1]};
                nrm[f] = Vector3D(m->face_normal[3 * f], m->face_normal[3 * f + 1], m->face_normal[3 * f + 2]);
                cm[f] = Vector3D(m->face_cm[3 * f], m->face_cm[3 * f + 1], m->face_cm[3 * f + 2]);
                for (uint32_t q = m->face_vertex_offset[f]; q < m->face_vertex_offset[f + 1]; ++q) fv[f].push_back(m->face_vertices[q]);
            }
            for (std::size_t v = 0; v < m->nvertices; ++v)
                nodes[v] = Vector3D(m->vertices[3 * v], m->vertices[3 * v + 1], m->vertices[3 * v + 2]);
            h->grid = std::make_unique<Grid>(Vector3D(m->box[0], m->box[1], m->box[2]), Vector3D(m->box[3], m->box[4], m->box[5]),
                                             pts, cf, fn, nrm, cm, area, vol, fv, nodes);
        } else {
            std::vector<double> xe(d->x_edges, d->x_edges + d->nx + 1), ye(d->y_edges, d->y_edges + d->ny + 1),
                ze(d->z_edges, d->z_edges + d->nz + 1);
            h->xe = xe; h->ye = ye; h->ze = ze;
            h->grid = std::make_unique<Grid>(xe, ye, ze);
        }
        const std::size_t N = h->grid->GetPointNo();
        h->cells.resize(N);
        h->ext.resize(N);
        for (std::size_t i = 0; i < N; ++i) {
            h->cells[i].temperature = d->temperature[i];
            h->cells[i].internalEnergy = d->cell_internal_energy ? d->cell_internal_energy[i] : d->internal_energy[i];
            h->ext[i].mass = d->mass[i];
            h->ext[i].internal_energy = d->internal_energy[i];
            if (d->cell_velocity) {
                h->cells[i].velocity = Vector3D(d->cell_velocity[3 * i], d->cell_velocity[3 * i + 1], d->cell_velocity[3 * i + 2]);
                h->ext[i].momentum = h->cells[i].velocity * h->ext[i].mass;
            }
        }
        h->eos = std::make_shared<HarnessEOS>();
        h->eos->kind = d->eos_kind;
        h->eos->cvPerMass = d->cv_per_mass;
        h->eos->f = d->eos_f;
        h->eos->beta = d->eos_beta;
        h->eos->mu = d->eos_mu;
        switch (boundary_kind) {
        case 0: {
            auto b = std::make_shared<HarnessBoundary>(*h->grid);
            std::memcpy(b->faces, d->faces, sizeof(b->faces));
            b->escapeNoCheck = d->escape_without_check != 0;
            b->sigmaSB = d->sigma_sb;
            b->clight = d->clight;
            // the packets' directions, times and frequencies follow the problem
            // seed, so runs of different seeds are independent realisations
            // (SideTemperature keeps a function-static engine seeded with 0)
            b->re.seed(d->seed);
            if (d->groups >= 2) {
                b->bounds.assign(d->group_bounds, d->group_bounds + d->groups + 1);
                b->kBoltz = d->k_boltz;
            }
            h->harnessBoundary = b.get();
            h->boundary = b;
            break;
        }
        case 1: h->boundary = std::make_shared<STORM::RigidBoundary<Vector3D, Grid>>(*h->grid); break;
        case 2: h->boundary = std::make_shared<STORM::VacuumBoundary<Vector3D, Grid>>(*h->grid); break;
        case 3:
            h->boundary = std::make_shared<STORM::SideTemperature<Vector3D, Grid>>(*h->grid, d->faces[0].source_temperature,
                                                                                   d->faces[0].packets_per_face);
            break;
        case 4:
            h->boundary = std::make_shared<STORM::TwoSidesTemperature<Vector3D, Grid>>(
                *h->grid, d->faces[0].source_temperature, d->faces[1].source_temperature, d->faces[0].packets_per_face);
            break;
        default: throw STORM::StormError("unknown boundary kind");
        }
        if (d->groups >= 2) {
            if (d->groups == kMGGroupsA) build_physics<kMGGroupsA>(*h, d);
            else if (d->groups == kMGGroupsB) build_physics<kMGGroupsB>(*h, d);
            else throw STORM::StormError("reference build holds multigroup for 30 and 64 groups only");
        } else {
            build_physics<1>(*h, d);
        }
        if (d->comb_enabled && d->comb_kind == STORM_COMB_STRATIFIED) {
            // the classifier as the engine lowers it: frequency bins by findGroup's rule
            std::vector<double> edges;
            const std::size_t B = d->strat_bins;
            if (B > 1) {
                const double *sb = d->strat_bounds ? d->strat_bounds : d->group_bounds;
                edges.assign(sb, sb + B + 1);
            }
            auto classifier = [edges, B](const MCParticle &p) -> std::size_t {
                for (std::size_t g = 0; g + 1 < B; ++g)
                    if (p.frequency < edges[g + 1]) return g;
                return B - 1;
            };
            h->pop = std::make_shared<STORM::StratifiedCombPopulationControl<Vector3D, Grid>>(
                *h->grid, B, classifier, d->comb_nmin, d->comb_factor, d->strat_min_per_bin);
        } else if (d->comb_enabled)
            h->pop = std::make_shared<STORM::CombPopulationControl<Vector3D, Grid>>(*h->grid, d->comb_nmin, d->comb_factor);
        else
            h->pop = std::make_shared<STORM::NoPopulationControl<Vector3D, Grid>>(*h->grid);
        h->manager = std::make_unique<STORM::MonteCarloManagerSerial<Vector3D, Grid>>(*h->grid, h->physics, h->pop, h->boundary);
        return h.release();
    } catch (const std::exception &e) {
        if (err && errlen) std::snprintf(err, errlen, "%s", e.what());
        return nullptr;
    }
}

void ref_destroy(RefHandle *h) { delete h; }

// The per-face descriptor boundary's SetTemperature (MarshakBoundary.hpp:33,
// DensmoreBoundary.hpp:42): a new source temperature for box face `face`.
int ref_set_face_temperature(RefHandle *h, int face, double T) {
    if (!h->harnessBoundary || face < 0 || face > 5) return -1;
    h->harnessBoundary->faces[face].source_temperature = T;
    return 0;
}

const char *ref_last_error(RefHandle *h) { return h->lastError.c_str(); }

int ref_step(RefHandle *h, double dt, RefStepOut *out) {
    NullBuf nb;
    std::streambuf *old = std::cout.rdbuf(&nb);
    try {
        if (h->harnessBoundary) h->harnessBoundary->escaped = 0.0;
        auto t0 = std::chrono::steady_clock::now();
        h->census = h->manager->step(std::move(h->census), dt);
        auto t1 = std::chrono::steady_clock::now();
        std::cout.rdbuf(old);
        if (out) {
            out->initial = h->manager->GetInitialParticleCount();
            out->prestep = h->manager->GetPreStepParticleCount();
            out->start = h->manager->GetStartParticleCount();
            out->end = h->manager->GetEndParticleCount();
            uint64_t s = 0;
            for (auto c : h->manager->GetCellsStepsCounters()) s += c;
            out->segments = s;
            out->rw_steps = h->view->randomWalkStepCount();
            out->wall_seconds = std::chrono::duration<double>(t1 - t0).count();
            out->escaped_energy = h->harnessBoundary ? h->harnessBoundary->escaped : 0.0;
        }
        return 0;
    } catch (const std::exception &e) {
        std::cout.rdbuf(old);
        h->lastError = e.what();
        return 1;
    }
}

// Calls physics->preStep(dt) alone (emission included); the emitted particles
// replace the census buffer so the tests can inspect them.
int ref_prestep_only(RefHandle *h, double dt, uint64_t *emitted) {
    try {
        h->view->updateGridData();
        h->census = h->view->preStep(dt);
        if (emitted) *emitted = h->census.size();
        return 0;
    } catch (const std::exception &e) {
        h->lastError = e.what();
        return 1;
    }
}

uint64_t ref_census_count(RefHandle *h) { return h->census.size(); }

int ref_get_census(RefHandle *h, StormParticlesSoA *o) {
    for (std::size_t k = 0; k < h->census.size() && k < o->count; ++k) {
        const MCParticle &p = h->census[k];
        o->x[k] = p.location.x; o->y[k] = p.location.y; o->z[k] = p.location.z;
        o->vx[k] = p.velocity.x; o->vy[k] = p.velocity.y; o->vz[k] = p.velocity.z;
        o->time_left[k] = p.timeLeft; o->weight[k] = p.weight; o->initial_weight[k] = p.initialWeight;
        o->cell[k] = static_cast<uint32_t>(p.cellIndex);
        if (o->id) o->id[k] = p.id;
        if (o->frequency) o->frequency[k] = p.frequency;
    }
    return 0;
}

int ref_set_census(RefHandle *h, const StormParticlesSoA *in) {
    h->census.clear();
    for (uint64_t k = 0; k < in->count; ++k) {
        MCParticle p;
        p.location = Vector3D(in->x[k], in->y[k], in->z[k]);
        p.velocity = Vector3D(in->vx[k], in->vy[k], in->vz[k]);
        p.timeLeft = in->time_left[k];
        p.weight = in->weight[k];
        p.initialWeight = in->initial_weight[k];
        p.cellIndex = in->cell[k];
        p.frequency = in->frequency ? in->frequency[k] : 0.0;
        p.id = in->id ? in->id[k] : std::numeric_limits<std::size_t>::max();
        h->census.push_back(p);
    }
    return 0;
}

int ref_get_cells(RefHandle *h, double *T, double *eint, double *eradAvg, double *eradCensus, double *sigA, double *fleck,
                  uint64_t *segs) {
    const std::size_t N = h->grid->GetPointNo();
    const auto &ea = h->view->eradTimeAvg();
    const auto &sa = h->view->planckOpacities();
    const auto &ff = h->view->factorFleck();
    const auto &sc = h->manager->GetCellsStepsCounters();
    for (std::size_t i = 0; i < N; ++i) {
        if (T) T[i] = h->cells[i].temperature;
        if (eint) eint[i] = h->ext[i].internal_energy;
        if (eradAvg) eradAvg[i] = i < ea.size() ? ea[i] : 0.0;
        if (eradCensus) eradCensus[i] = h->ext[i].Erad;
        if (sigA) sigA[i] = i < sa.size() ? sa[i] : 0.0;
        if (fleck) fleck[i] = i < ff.size() ? ff[i] : 0.0;
        if (segs) segs[i] = i < sc.size() ? sc[i] : 0;
    }
    return 0;
}

int ref_get_emission(RefHandle *h, uint64_t *photons) {
    const auto v = h->view->lastSourcePhotonsPerCell();
    for (std::size_t i = 0; i < v.size(); ++i) photons[i] = v[i];
    return 0;
}

// ---------------- recording
int ref_record_begin(RefHandle *h, uint64_t maxRecords) {
    RecordState &rs = h->view->records();
    rs.records.clear();
    rs.tape.clear();
    rs.maxRecords = maxRecords;
    rs.recording = true;
    return 0;
}
int ref_record_end(RefHandle *h) {
    h->view->records().recording = false;
    return 0;
}
uint64_t ref_record_count(RefHandle *h) { return h->view->records().records.size(); }
uint64_t ref_record_tape_size(RefHandle *h) { return h->view->records().tape.size(); }

// Copies the records out as parallel arrays.  before: 9n, after: 8n,
// tallies: 4n (emat before/after, erad before/after), tape: tape_size.
int ref_record_get(RefHandle *h, uint64_t *id, uint32_t *cell, double *before, double *after, int32_t *status,
                   uint64_t *nextCell, double *tallies, uint64_t *tapeOffset, uint32_t *tapeLength, int32_t *usedRW,
                   double *tape) {
    const auto &R = h->view->records().records;
    for (std::size_t k = 0; k < R.size(); ++k) {
        id[k] = R[k].id;
        cell[k] = R[k].cell;
        std::memcpy(before + 9 * k, R[k].before, sizeof(R[k].before));
        std::memcpy(after + 8 * k, R[k].after, sizeof(R[k].after));
        status[k] = R[k].status;
        nextCell[k] = R[k].nextCell;
        tallies[4 * k + 0] = R[k].ematBefore;
        tallies[4 * k + 1] = R[k].ematAfter;
        tallies[4 * k + 2] = R[k].eradBefore;
        tallies[4 * k + 3] = R[k].eradAfter;
        tapeOffset[k] = R[k].tapeOffset;
        tapeLength[k] = R[k].tapeLength;
        usedRW[k] = R[k].usedRW;
    }
    std::memcpy(tape, h->view->records().tape.data(), h->view->records().tape.size() * sizeof(double));
    return 0;
}

// Frequencies of the records (multigroup): before and after, n each.
int ref_record_get_frequency(RefHandle *h, double *before, double *after) {
    const auto &R = h->view->records().records;
    for (std::size_t k = 0; k < R.size(); ++k) {
        before[k] = R[k].freqBefore;
        after[k] = R[k].freqAfter;
    }
    return 0;
}

// Momentum the segment deposited into its cell (3 per record; hydro problems).
int ref_record_get_momentum(RefHandle *h, double *dmom) {
    const auto &R = h->view->records().records;
    for (std::size_t k = 0; k < R.size(); ++k)
        for (int d = 0; d < 3; ++d) dmom[3 * k + d] = R[k].momAfter[d] - R[k].momBefore[d];
    return 0;
}

// Multigroup tables the reference computes per cell: the Planck mean opacity
// of its opacity plug-in and the thermal energy it samples at given uniforms.
int ref_mg_thermal_energy(RefHandle *h, uint64_t n, const uint32_t *cells, const double *xi, double *energy) {
    try {
        return h->view->thermalEnergy(n, cells, xi, energy);
    } catch (const std::exception &e) {
        h->lastError = e.what();
        return 1;
    }
}

// ---------------- component probes
int ref_rw_sample(uint64_t n, const double *xiLeak, const double *tau, const double *xiRad, double *leak, double *rad) {
    static STORM::RandomWalk rw;
    for (uint64_t k = 0; k < n; ++k) {
        if (xiLeak) leak[k] = rw.sampleLeakTime(xiLeak[k]);
        if (tau && xiRad) rad[k] = rw.sampleRadius(tau[k], xiRad[k]);
    }
    return 0;
}
int ref_rw_functions(uint64_t n, const double *tau, const double *x, double *survival, double *cdf) {
    static STORM::RandomWalk rw;
    for (uint64_t k = 0; k < n; ++k) {
        if (survival) survival[k] = rw.computeSurvival(tau[k]);
        if (cdf) cdf[k] = rw.computeRadialCDF(x[k], tau[k]);
    }
    return 0;
}

// RandomInCellPositionSampler (utils/RandomInCell.hpp:11-67) driven by a
// seeded std::mt19937_64; the draws each call consumed are logged (tape, 4 per call).
int ref_sample_in_cell(RefHandle *h, uint64_t n, const uint32_t *cells, uint64_t seed, double *pos, double *tape,
                       uint32_t *ndraws) {
    std::mt19937_64 eng(seed);
    std::uniform_real_distribution<double> dist(0.0, 1.0);
    RandomInCellPositionSampler<Vector3D, Grid> sampler;
    uint64_t t = 0;
    for (uint64_t k = 0; k < n; ++k) {
        std::mt19937_64 snap = eng;
        Vector3D p = sampler(*h->grid, cells[k], eng, dist);
        pos[3 * k] = p.x; pos[3 * k + 1] = p.y; pos[3 * k + 2] = p.z;
        std::mt19937_64 cnt = snap;
        uint32_t m = 0;
        while (!(cnt == eng)) { cnt.discard(1); ++m; }
        ndraws[k] = m;
        for (uint32_t q = 0; q < m; ++q) tape[t++] = dist(snap);
    }
    return 0;
}

// RadiationOpacityModel::isotropicVelocity (radiation/RadiationOpacityModel.hpp:139-150), 2 draws per call.
int ref_isotropic(uint64_t n, uint64_t seed, double *vel, double *tape) {
    std::mt19937_64 eng(seed);
    std::uniform_real_distribution<double> dist(0.0, 1.0);
    for (uint64_t k = 0; k < n; ++k) {
        std::mt19937_64 snap = eng;
        Vector3D v = HarnessOpacity::isotropic(eng, dist);
        vel[3 * k] = v.x; vel[3 * k + 1] = v.y; vel[3 * k + 2] = v.z;
        tape[2 * k] = dist(snap);
        tape[2 * k + 1] = dist(snap);
    }
    return 0;
}

// RandomPointOnFace (utils/RandomOnFace.hpp:15-66) keeps a function-static
// std::mt19937(0).  A distinct grid type gives this probe its own template
// instance, hence its own fresh engine, which a mirror engine here tracks
// draw for draw (3 doubles per call).
namespace {
struct ProbeGrid : public Grid {
    using Grid::Grid;
};
} // namespace
int ref_point_on_face(RefHandle *h, uint64_t n, const uint64_t *faces, double *pos, double *tape) {
    static std::unique_ptr<ProbeGrid> pg;
    static std::mt19937 mirror(0);
    static std::uniform_real_distribution<double> mdist(0.0, 1.0);
    pg = std::make_unique<ProbeGrid>(h->xe, h->ye, h->ze);
    for (uint64_t k = 0; k < n; ++k) {
        Vector3D p = STORM::RandomPointOnFace<Vector3D, ProbeGrid>(*pg, faces[k]);
        pos[3 * k] = p.x; pos[3 * k + 1] = p.y; pos[3 * k + 2] = p.z;
        tape[3 * k] = mdist(mirror);
        tape[3 * k + 1] = mdist(mirror);
        tape[3 * k + 2] = mdist(mirror);
    }
    return 0;
}

// The cells' velocity and the extensives' momentum (3 per cell each).
int ref_get_motion(RefHandle *h, double *velocity, double *momentum) {
    for (std::size_t i = 0; i < h->cells.size(); ++i) {
        const Vector3D &v = h->cells[i].velocity, &m = h->ext[i].momentum;
        if (velocity) { velocity[3 * i] = v.x; velocity[3 * i + 1] = v.y; velocity[3 * i + 2] = v.z; }
        if (momentum) { momentum[3 * i] = m.x; momentum[3 * i + 1] = m.y; momentum[3 * i + 2] = m.z; }
    }
    return 0;
}

// RadiationIMC::getEgTimeAvg after the last step (withEgTimeAvg), cells x groups.
int ref_get_group_tallies(RefHandle *h, double *out) { return h->view ? h->view->groupTallies(out) : 1; }

// The serial manager's GetBeginningParticleCount after its last ref_step.
int ref_beginning_counts(RefHandle *h, uint64_t *counts) {
    if (!h->manager) return 1;
    const auto &v = h->manager->GetBeginningParticleCount();
    for (std::size_t i = 0; i < v.size(); ++i) counts[i] = v[i];
    return 0;
}

// RandomPointOnFace (utils/RandomOnFace.hpp:15-66) draws from a function-static
// std::mt19937(0) shared by every handle of the process.  Batch runs of
// different seeds each start a fresh process and move that stream forward by
// `calls` points first, so that their face-source positions do not repeat.
int ref_advance_face_stream(RefHandle *h, uint64_t calls) {
    try {
        const std::size_t face = h->grid->GetCellFaces(0)[0];
        for (uint64_t k = 0; k < calls; ++k) (void)STORM::RandomPointOnFace<Vector3D, Grid>(*h->grid, face);
    } catch (const std::exception &e) {
        h->lastError = e.what();
        return 1;
    }
    return 0;
}

// The population control's activate (CombPopulationControl or
// StratifiedCombPopulationControl) on a given particle list (invariant tests).
int ref_comb(RefHandle *h, const StormParticlesSoA *in, StormParticlesSoA *out, uint64_t *outCount) {
    try {
        std::vector<MCParticle> v;
        for (uint64_t k = 0; k < in->count; ++k) {
            MCParticle p;
            p.location = Vector3D(in->x[k], in->y[k], in->z[k]);
            p.velocity = Vector3D(in->vx[k], in->vy[k], in->vz[k]);
            p.timeLeft = in->time_left[k];
            p.weight = in->weight[k];
            p.initialWeight = in->initial_weight[k];
            p.cellIndex = in->cell[k];
            p.frequency = in->frequency ? in->frequency[k] : 0.0;
            p.id = in->id ? in->id[k] : k;
            v.push_back(p);
        }
        std::vector<MCParticle> r = h->pop->activate(v);
        *outCount = r.size();
        for (std::size_t k = 0; k < r.size() && k < out->count; ++k) {
            out->x[k] = r[k].location.x; out->y[k] = r[k].location.y; out->z[k] = r[k].location.z;
            out->vx[k] = r[k].velocity.x; out->vy[k] = r[k].velocity.y; out->vz[k] = r[k].velocity.z;
            out->time_left[k] = r[k].timeLeft; out->weight[k] = r[k].weight; out->initial_weight[k] = r[k].initialWeight;
            out->cell[k] = static_cast<uint32_t>(r[k].cellIndex);
            if (out->id) out->id[k] = r[k].id;
            if (out->frequency) out->frequency[k] = r[k].frequency;
        }
        return 0;
    } catch (const std::exception &e) {
        h->lastError = e.what();
        return 1;
    }
}

// The unit constants this build of the reference was compiled with.
int ref_units(double *out) {
    out[0] = units::clight; out[1] = units::arad; out[2] = units::sigma_sb; out[3] = units::kev_kelvin;
    out[4] = units::k_boltz; out[5] = units::kev;
    return 0;
}

double ref_planck_integral(double a, double b) { return planck_integral::planck_integral(a, b); }

} // extern "C"
