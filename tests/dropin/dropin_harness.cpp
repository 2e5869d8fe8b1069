// Test infrastructure only: MonteCarloManagerCUDA (include/storm/) compiled
// against the reference's own types and plug-ins.  The reference problem set-up
// of oracle/ref_harness.cpp (grid, cells, extensives, RadiationIMC, comb,
// boundary) is reused unchanged; dropin_create swaps the serial manager for the
// CUDA one, bound to the same vectors, so ref_get_cells / ref_get_census read
// what the drop-in wrote back.  Built by oracle/Makefile (target dropin) into
// oracle/_ref/libstormdropin.so, linked against storm_b200/libstorm_cuda.so.
#include "ref_harness.cpp"

#include "storm/MonteCarloManagerCUDA.hpp"

struct DropinHandle {
    RefHandle *ref = nullptr;
    std::vector<double> sigA, sigS;
    std::unique_ptr<STORM::MonteCarloManagerCUDA<Vector3D, Grid, Cell, Ext>> manager;
    std::string lastError;
};

// RadiationIMCParameters<G> as ref_create builds them, through bind_parameters
template <std::size_t G>
void bind_imc(STORM::CudaIMCBinding<Cell, Ext> &b, const StormProblemDesc *d) {
    STORM::RadiationIMCParameters<G> p;
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
    if constexpr (G > 1) {
        p.withMultigroupOpacity = true;
        for (std::size_t g = 0; g <= G; ++g) p.energyBoundaries[g] = d->group_bounds[g];
        p.energyBoundariesProvided = true;
    }
    b.bind_parameters(p);
}

extern "C" {

// boundary_kind as ref_create takes it (0 the per-face descriptor plug-in,
// 1 RigidBoundary, 2 VacuumBoundary, 3 SideTemperature, 4 TwoSidesTemperature:
// the template lowers kinds 1-4 by their type).  opacity_from_plugin: the
// binding's planckOpacity / scatteringOpacity call the reference-side opacity
// plug-in on the caller's cells (CalcPlanckOpacity, CalcScatteringOpacity),
// so a temperature-dependent opacity is re-evaluated before every step.
DropinHandle *dropin_create_plugins(const StormProblemDesc *d, int precision, int boundary_kind,
                                    int opacity_from_plugin, char *err, size_t errlen) {
    RefHandle *ref = ref_create(d, boundary_kind, err, errlen);
    if (!ref) return nullptr;
    auto h = std::make_unique<DropinHandle>();
    h->ref = ref;
    try {
        const std::size_t N = ref->grid->GetPointNo();
        STORM::CudaIMCBinding<Cell, Ext> b;
        b.cells = &ref->cells;
        b.extensives = &ref->ext;
        b.opacityKind = d->opacity_kind;
        if (d->opacity_kind == STORM_OPACITY_CELL_TABLE || d->opacity_kind == STORM_OPACITY_MG_POWER) {
            h->sigA.assign(d->sigma_a, d->sigma_a + N);
            h->sigS = d->sigma_s ? std::vector<double>(d->sigma_s, d->sigma_s + N) : std::vector<double>(N, 0.0);
            const std::vector<double> *sa = &h->sigA, *ss = &h->sigS;
            if (d->opacity_kind == STORM_OPACITY_MG_POWER) {
                b.sigma0 = [sa](std::size_t i) { return (*sa)[i]; };
                b.mgP = d->mg_p; b.mgQ = d->mg_q; b.mgS = d->mg_s;
                b.mgGroupConstant = d->mg_group_constant != 0;
                b.kBoltz = d->k_boltz;
            } else {
                b.planckOpacity = [sa](std::size_t i) { return (*sa)[i]; };
            }
            b.scatteringOpacity = [ss](std::size_t i) { return (*ss)[i]; };
        } else {
            b.kP0 = d->kP0; b.kR0 = d->kR0; b.alpha = d->alpha; b.beta = d->beta; b.tFloor = d->t_floor;
            b.cap = d->cap;
            if (d->density_factor) b.densityFactor.assign(d->density_factor, d->density_factor + N);
        }
        if (opacity_from_plugin) {
            if (d->groups >= 2) throw STORM::StormError("dropin_create_plugins: gray problems only");
            auto *opac = static_cast<RecordingIMC<1> *>(ref->physics.get())->opac;
            const std::vector<Cell> *cells = &ref->cells;
            b.opacityKind = STORM_OPACITY_CELL_TABLE;
            b.planckOpacity = [opac, cells](std::size_t i) { return opac->CalcPlanckOpacity((*cells)[i]); };
            b.scatteringOpacity = [opac, cells](std::size_t i) { return opac->CalcScatteringOpacity((*cells)[i]); };
        }
        b.eosKind = d->eos_kind;
        b.cvPerMass = d->cv_per_mass;
        b.eosF = d->eos_f; b.eosBeta = d->eos_beta; b.eosMu = d->eos_mu;
        for (int f = 0; f < 6; ++f) b.faces[f] = d->faces[f];
        b.escapeWithoutCheck = d->escape_without_check != 0;
        if (d->groups == kMGGroupsA) bind_imc<kMGGroupsA>(b, d);
        else if (d->groups == kMGGroupsB) bind_imc<kMGGroupsB>(b, d);
        else bind_imc<1>(b, d);
        b.combEnabled = d->comb_enabled != 0;
        b.combNmin = d->comb_nmin;
        b.combFactor = d->comb_factor;
        b.combKind = d->comb_kind;
        b.stratBins = d->strat_bins;
        if (d->strat_bounds) b.stratBounds.assign(d->strat_bounds, d->strat_bounds + d->strat_bins + 1);
        b.stratMinPerBin = d->strat_min_per_bin;
        b.clight = d->clight; b.arad = d->arad; b.sigmaSB = d->sigma_sb; b.kevKelvin = d->kev_kelvin;
        b.seed = d->seed;
        b.precision = precision;
        b.device = d->device;
        b.segmentsPerVisit = d->segments_per_visit;
        h->manager = std::make_unique<STORM::MonteCarloManagerCUDA<Vector3D, Grid, Cell, Ext>>(
            *ref->grid, ref->physics, ref->pop, ref->boundary, b);
        return h.release();
    } catch (const std::exception &e) {
        if (err && errlen) std::snprintf(err, errlen, "%s", e.what());
        ref_destroy(ref);
        return nullptr;
    }
}

DropinHandle *dropin_create(const StormProblemDesc *d, int precision, char *err, size_t errlen) {
    return dropin_create_plugins(d, precision, 0, 0, err, errlen);
}

// MonteCarloManagerCUDA::GetBeginningParticleCount after the last step.
int dropin_beginning_counts(DropinHandle *h, uint64_t *counts) {
    const auto &v = h->manager->GetBeginningParticleCount();
    for (std::size_t i = 0; i < v.size(); ++i) counts[i] = v[i];
    return static_cast<int>(v.size() == h->ref->grid->GetPointNo() ? 0 : 1);
}

void dropin_destroy(DropinHandle *h) {
    if (!h) return;
    h->manager.reset();
    ref_destroy(h->ref);
    delete h;
}

RefHandle *dropin_ref(DropinHandle *h) { return h->ref; }

const char *dropin_last_error(DropinHandle *h) { return h->lastError.c_str(); }

// One MonteCarloManagerCUDA::step on the handle's census; fills the same
// counters ref_step reports from the serial manager.
int dropin_step(DropinHandle *h, double dt, RefStepOut *out) {
    NullBuf nb;
    std::streambuf *old = std::cout.rdbuf(&nb);
    try {
        auto &m = *h->manager;
        h->ref->census = m.step(std::move(h->ref->census), dt);
        std::cout.rdbuf(old);
        if (out) {
            out->initial = m.GetInitialParticleCount();
            out->prestep = m.GetPreStepParticleCount();
            out->start = m.GetStartParticleCount();
            out->end = m.GetEndParticleCount();
            uint64_t s = 0;
            for (auto c : m.GetCellsStepsCounters()) s += c;
            out->segments = s;
            out->rw_steps = 0;
            out->wall_seconds = m.GetWallTime();
            out->escaped_energy = 0.0;
        }
        return 0;
    } catch (const std::exception &e) {
        std::cout.rdbuf(old);
        h->lastError = e.what();
        return 1;
    }
}

int dropin_get_cells(DropinHandle *h, double *eradAvg, double *sigA, double *fleck, uint64_t *segs) {
    const auto &m = *h->manager;
    const std::size_t N = h->ref->grid->GetPointNo();
    for (std::size_t i = 0; i < N; ++i) {
        if (eradAvg) eradAvg[i] = m.getEradTimeAvg().empty() ? 0.0 : m.getEradTimeAvg()[i];
        if (sigA) sigA[i] = m.getPlanckOpacities().empty() ? 0.0 : m.getPlanckOpacities()[i];
        if (fleck) fleck[i] = m.getFactorFleck().empty() ? 0.0 : m.getFactorFleck()[i];
        if (segs) segs[i] = m.GetCellsStepsCounters()[i];
    }
    return 0;
}

}  // extern "C"
