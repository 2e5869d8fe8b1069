/*
 * Test infrastructure only: the oracle.  A plain-C restatement of STORM's gray
 * IMC hot path (RadiationIMC::preStep / step / postStep, the serial manager's
 * face and boundary handling, RandomWalk, the source samplers and
 * CombPopulationControl), used by the tests as the checker of the CUDA engine.
 * The product never links or calls it.
 *
 * Two random-number sources drive the same code:
 *   - a recorded tape of the reference's own draws (replay parity against the
 *     reference build in oracle/_ref), and
 *   - the counter-based Philox4x32-10 streams the CUDA engine uses, so that a
 *     whole time step can be compared particle by particle with the GPU.
 */
#ifndef STORM_IMC_ORACLE_H
#define STORM_IMC_ORACLE_H

#include <stdint.h>
#include "storm_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct Oracle Oracle;

Oracle *orc_create(const StormProblemDesc *d);
void orc_destroy(Oracle *o);

int orc_step(Oracle *o, double dt, StormStepStats *stats);
int orc_phase_begin(Oracle *o, double dt);
int orc_phase_prestep(Oracle *o, double dt);
int orc_phase_emit(Oracle *o, double dt);
int orc_phase_transport(Oracle *o);
int orc_phase_comb(Oracle *o);
int orc_phase_poststep(Oracle *o, double dt);
int orc_phase_stats(Oracle *o, StormStepStats *stats);

int orc_set_census(Oracle *o, const StormParticlesSoA *in);
uint64_t orc_census_count(Oracle *o);
int orc_get_census(Oracle *o, StormParticlesSoA *out);
/* particles currently in the transport bank (after emit, before transport) */
uint64_t orc_bank_count(Oracle *o);
int orc_get_bank(Oracle *o, StormParticlesSoA *out);
int orc_get_cell_arrays(Oracle *o, double *T, double *eint, double *eradAvg, double *eradCensus, double *sigA,
                        double *fleck, uint64_t *segs);
int orc_set_cell_physics(Oracle *o, const double *sigA, const double *sigS, const double *fleck);
int orc_get_emission(Oracle *o, uint64_t *photons, double *energy);
int orc_set_face_temperature(Oracle *o, int face, double T);
int orc_last_error(Oracle *o, int32_t *derr, uint64_t *cell, uint64_t *particle);

/* particle shards: the same contract as storm_cuda_set_sharding (host buffers,
 * stream NULL) */
int orc_set_sharding(Oracle *o, uint32_t shards, uint32_t lo, uint32_t hi, StormExchangeFn exchange, void *user);

/* one segment per item, driven by the item's tape */
int orc_replay_segments(Oracle *o, StormReplayBatch *b);

/* Random Walk tables and samplers (radiation/RandomWalk.hpp) */
void orc_rw_tables(double *tau, double *survival, double *radius);
double orc_rw_sample_leak(double xi);
double orc_rw_sample_radius(double tau, double xi);
double orc_rw_survival(double tau);
double orc_rw_radial_cdf(double x, double tau);

/* source samplers fed by tapes */
int orc_sample_in_cell(Oracle *o, uint32_t cell, const double *tape4, double *out3);
int orc_point_on_face(Oracle *o, uint64_t face, const double *tape3, double *out3);
void orc_isotropic(const double *tape2, double clight, double *out3);

/* Philox4x32-10 and the engine's uniform mapping */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double orc_uniform(uint64_t seed, uint32_t tag, uint32_t step, uint32_t pid, uint32_t draw);
uint32_t orc_comb_key(uint64_t seed, uint32_t step, uint32_t pid, int b);
uint32_t orc_step_index(Oracle *o);

#ifdef __cplusplus
}
#endif
#endif
