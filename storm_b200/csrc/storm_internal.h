// Internal interface between the host runtime (storm_runtime.cu) and the kernels
// (storm_kernels.cu).  Not part of the C ABI.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "storm_device.cuh"

namespace storm {

// Particle bank, struct of arrays.  pid keys the particle's random stream for the
// step; draw counts the uniforms it has consumed.
struct Bank {
    double *x, *y, *z, *vx, *vy, *vz, *t, *w, *w0;
    uint32_t *cell, *pid, *draw;
    double *nu;          // photon energy, multigroup problems only (NULL otherwise)
};

// Census bank: one record of 16-byte vectors per particle (96 B in the FP64
// form, 64 B in the FP32-tracking form), so the comb's random-order gather reads
// one record instead of twelve scattered array elements.
struct CensusBank {
    uint4 *rec;
};

struct CellArrays {
    double *T, *mass, *vol, *eint, *ceint;
    double *sigA, *sigS, *fleck, *rwSigT, *eradAvg, *eradCensus, *emitE;
    uint8_t *rwElig;
    uint64_t *photons;
    double4 *phys;      // per-cell segment constants (cell_phys)
    float4 *phys32;     // FP32-tracking form: 1/sigma_e, sigma_a f
    // multigroup
    double *mgCdf;      // per cell, groups + 1
    double4 *pgrw;      // per cell: sigmaT_bar, sigmaA_bar, D, gamma
    uint32_t *pgrwCut;  // per cell group cutoff
};

struct OpacityEos {
    int32_t opacityKind, eosKind;
    // multigroup: tabA holds sigma0 per cell, tabS the elastic opacity
    const double *tabA, *tabS, *rhoF;
    double kP0, kR0, alpha, tFloor, cap;
    double cvPerMass, eosF, eosBeta, eosMu;
};

// Boundary cell-faces that emit, in (cell, GetCellFaces side) order, with the
// packet prefix offset[0..count].
struct FaceSources {
    const uint32_t *cell;
    const int32_t *side;
    const uint64_t *offset;
    uint32_t count;
    // polyhedral meshes: the boundary face's index and its area (NULL on the Cartesian grid)
    const uint32_t *face;
    const double *area;
};

struct CombParams {
    uint64_t ntotal, nmin;
};

// StratifiedCombPopulationControl: frequency bins of the particle classifier
struct StratParams {
    uint32_t bins;
    const double *bounds;    // bins + 1 edges (device), NULL when bins == 1
    uint64_t minPerBin;
};

struct DevStats {
    unsigned long long segments, rwSteps, escaped, cutoff, census;
    double eCensusIn, eEmitted, eDeposited, eEscaped, eCensusPre, eCensusOut, eDebit;
};

struct ReplayDev {
    const double *in[9];
    const double *freq;     // multigroup: frequency before (NULL = 0)
    double *freqOut;        // multigroup: frequency after (NULL = not returned)
    const uint32_t *cell;
    const uint64_t *tapeOffset;
    const uint32_t *tapeLength;
    const double *tape;
    double *phys[8];
    int32_t *physStatus;
    uint32_t *physNext;
    double *dep[2];
    double *mgr[6];
    uint32_t *mgrCell;
    int32_t *mgrStatus;
    uint32_t *draws;
    int32_t *usedRW;
    double *momOut;         // moving material: 3 per record (NULL = not returned)
};

// particles [lo, n) (pids pidOffset + q)
void launch_begin(cudaStream_t s, const Bank &b, uint32_t n, uint32_t pidOffset, double dt, DevStats *st,
                  uint32_t lo = 0);
void launch_prestep(cudaStream_t s, const Ctx &C, const CellArrays &A, const OpacityEos &M, double dt);
void launch_rw_eligibility(cudaStream_t s, const Ctx &C, const CellArrays &A);
void launch_emission_energy(cudaStream_t s, const Ctx &C, const CellArrays &A, double dt);
void launch_sequential_sum(cudaStream_t s, const double *v, uint32_t n, double *out);
void launch_allocate(cudaStream_t s, const Ctx &C, const CellArrays &A, const double *total, uint64_t newPerCell);
// the same two kernels, run only where *onlyIf is nonzero (decided on the device)
void launch_sequential_sum_if(cudaStream_t s, const double *v, uint32_t n, double *out, const int32_t *onlyIf);
void launch_allocate_if(cudaStream_t s, const Ctx &C, const CellArrays &A, const double *total, uint64_t newPerCell,
                        const int32_t *onlyIf);
void launch_emission_debit(cudaStream_t s, const Ctx &C, const CellArrays &A, DevStats *st);
void launch_scan_u64(cudaStream_t s, const uint64_t *in, uint32_t n, uint64_t *out, uint64_t *tileSums, uint64_t *total);
void launch_emit_cells(cudaStream_t s, const Ctx &C, const CellArrays &A, const uint64_t *offsets, uint64_t eBegin,
                       uint64_t count, const Bank &b, uint32_t bankBase, uint32_t pidBase, double dt, DevStats *st);
void launch_ddmc_rates(cudaStream_t s, const Ctx &C, const CellArrays &A);
void launch_strat_keys(cudaStream_t s, const Ctx &C, const CensusBank &cen, uint32_t n, uint64_t *keys, uint32_t *vals,
                       uint32_t combKey, int pidBits, const StratParams &S, double *wc = nullptr);
void launch_strat_sums(cudaStream_t s, const double *wS, const uint32_t *start, uint32_t ncells, uint32_t bins,
                       double *binW, double *cellW);
void launch_strat_plan(cudaStream_t s, const Ctx &C, const CombParams &P, const StratParams &S, const double *wS,
                       const uint32_t *start, const double *binW, const double *cellW, const double *Wtot,
                       uint32_t *pCount, double *pWeight, uint64_t *cellCount, double *eradCensus, DevStats *st);
void launch_face_spectra(cudaStream_t s, const Ctx &C, double *cdf);
void launch_set_u32(cudaStream_t s, uint32_t *p, uint32_t v);
void launch_poly_tets(cudaStream_t s, const Ctx &C, const uint32_t *tetOff, double *tetCum, uint2 *tetAT);
void launch_emit_faces(cudaStream_t s, const Ctx &C, const FaceSources &F, uint64_t fBegin, uint64_t count,
                       const Bank &b, uint32_t bankBase, uint32_t pidBase, double dt, DevStats *st);
void launch_transport(cudaStream_t s, uint32_t grid, const Ctx &C, const Bank &in, const uint32_t *nIn, const Bank &out,
                      uint32_t *nOut, const CensusBank &cen, uint32_t *nCen, uint32_t K, DevStats *st, int minBlocks);
int transport_blocks_per_sm(int minBlocks, bool fp32);
void launch_transport_refill(cudaStream_t s, uint32_t grid, int minBlocks, const Ctx &C, const Bank &in, uint32_t n,
                             uint32_t *nextIdx, const CensusBank &cen, uint32_t *nCen, uint32_t burst, uint32_t maxSegs,
                             DevStats *st);
int refill_blocks_per_sm(int minBlocks, bool fp32);
void launch_bank_to_local(cudaStream_t s, const Ctx &C, const Bank &src, const Bank &dst, uint32_t n,
                          uint32_t lo = 0);   // particles [lo, n)
void launch_bank_to_global(cudaStream_t s, const Ctx &C, const Bank &src, const Bank &dst, uint32_t n);
void launch_comb_keys(cudaStream_t s, const Ctx &C, const CensusBank &cen, uint32_t n, uint64_t *keys, uint32_t *vals,
                      uint32_t combKey, int pidBits, double *wc = nullptr);
int launch_radix_sort(cudaStream_t s, uint64_t *keys, uint32_t *vals, uint64_t *keysAlt, uint32_t *valsAlt, uint32_t n,
                      int bits, uint32_t *tileHist);
uint32_t radix_tile_count(uint32_t n);
void launch_comb_ranges(cudaStream_t s, const uint64_t *keys, uint32_t n, uint32_t ncells, uint32_t *start, int pidBits);
void launch_bucket_sort(cudaStream_t s, const Ctx &C, const CensusBank &cen, const uint64_t *keys, uint32_t n,
                        int pidBits, uint32_t nRuns, uint32_t *start, uint32_t *cursor, uint64_t *scanSums,
                        uint64_t *outKeys, uint32_t *outVals, double *wS, uint32_t *longRuns, uint32_t longCap,
                        uint32_t *flags, const double *wc = nullptr);
void launch_mask_count_upto(cudaStream_t s, const uint32_t *pCount, uint32_t n, const uint32_t *nValid, uint64_t *out);
size_t bucket_scan_words(uint32_t len);
uint32_t bucket_long_capacity(uint32_t n);
void launch_sorted_weights(cudaStream_t s, const Ctx &C, const CensusBank &cen, const uint32_t *idx, uint32_t n,
                           double *wS);
void launch_comb_cell_sums(cudaStream_t s, const double *wS, const uint32_t *start, uint32_t ncells, double *W);
void launch_blocked_sum(cudaStream_t s, const double *v, uint32_t n, double *out);
void launch_comb_plan(cudaStream_t s, const Ctx &C, const CombParams &P, const double *wS, const uint32_t *start,
                      const double *W, const double *Wtot, uint32_t *pCount, double *pWeight, uint64_t *cellCount,
                      double *eradCensus, DevStats *st);
void launch_comb_emit(cudaStream_t s, const Ctx &C, const CensusBank &cen, const uint32_t *idx, const uint64_t *sortedKeys,
                      int pidBits, uint32_t bins, uint32_t nValid, const uint32_t *pCount, const double *pWeight,
                      const uint64_t *pOffset, const Bank &out);
void launch_comb_emit_out(cudaStream_t s, const Ctx &C, const CensusBank &cen, const uint32_t *idx,
                          const uint64_t *sortedKeys, int pidBits, uint32_t bins, uint32_t nValid, uint32_t total,
                          const uint32_t *pCount, const double *pWeight, const uint64_t *pOffset, uint32_t *src,
                          uint32_t *tileMax, const Bank &out);
void launch_allocate_checked(cudaStream_t s, const Ctx &C, const CellArrays &A, const double *total,
                             uint64_t newPerCell, double rel, int32_t *ambiguous);
size_t radix_scratch_words(uint32_t n);
void launch_census_keys_pid(cudaStream_t s, const Ctx &C, const CensusBank &cen, uint32_t n, uint64_t *keys,
                            uint32_t *vals);
void launch_gather(cudaStream_t s, const Ctx &C, const CensusBank &src, const uint32_t *idx, uint32_t n, const Bank &dst,
                   double *eradCensus, DevStats *st);
void launch_bank_to_census(cudaStream_t s, const Ctx &C, const Bank &src, const CensusBank &dst, uint32_t n);
void launch_count_bad_cells(cudaStream_t s, const uint32_t *cell, uint32_t n, uint32_t N, int32_t *bad);
void launch_cell_histogram(cudaStream_t s, const uint32_t *cell, uint32_t n, uint32_t N, uint32_t *count);
// particle shards (storm_cuda_set_sharding)
void launch_shard_pack_runs(cudaStream_t s, const double *runW, const uint32_t *start, uint32_t nRuns, double *x);
void launch_shard_cell_weights(cudaStream_t s, const double *x, uint32_t ncells, uint32_t shards, double *Wc);
void launch_comb_plan_sharded(cudaStream_t s, const Ctx &C, const CombParams &P, const double *wS,
                              const uint32_t *start, const double *x, const double *Wc, const double *Wtot,
                              uint32_t lo, uint32_t hi, uint32_t *pCount, double *pWeight, double *eradCensus,
                              DevStats *st);
void launch_shard_pack_census(cudaStream_t s, const uint64_t *pOff, const uint64_t *total, const uint32_t *start,
                              uint32_t n, uint32_t ncells, uint32_t shards, uint32_t lo, uint32_t hi,
                              const double *eradCensus, double *x);
void launch_add_into(cudaStream_t s, double *y, const double *x, uint32_t n);
void launch_to_float(cudaStream_t s, const double *src, float *dst, uint32_t n);
void launch_poststep(cudaStream_t s, const Ctx &C, const CellArrays &A, const OpacityEos &M, double dt);
void launch_replay(cudaStream_t s, const Ctx &C, const ReplayDev &R, uint32_t n);
void launch_rw_radius(cudaStream_t s, const double *tau, const double *surv, double *radius);
void launch_rw_sample(cudaStream_t s, const RwTables &T, uint32_t n, const double *xiLeak, const double *tau,
                      const double *xiRad, double *leak, double *rad);

}  // namespace storm
