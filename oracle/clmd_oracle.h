/*
 * clmd_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A serial FP64 C restatement of the reference's hot path (the Fortran 77
 * files named in clmd_oracle.c), used as the checker of the CUDA engine and
 * as the timed CPU baseline.  Nothing in the product links or calls this:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU legs load it.
 *
 * Parity pins: no Fortran compiler exists on either machine, so the
 * reference cannot be run here and ships no golden vectors; the oracle is
 * pinned by analytic known-answer tests, by hand-derived fixtures committed
 * under tests/golden/ and by the all-pairs / cell-list cross-check.
 */
#ifndef CLMD_ORACLE_H
#define CLMD_ORACLE_H

#include "../include/clmd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sys orc_sys;

orc_sys* orc_create(const clmd_config* cfg);
void orc_destroy(orc_sys* S);

/* 0 = all pairs O(N^2) exactly as neighbor-pbc-mav.f (default),
 * 1 = cell list that must yield the same list (used for large N). */
void orc_set_neighbor_mode(orc_sys* S, int mode);

/* 0 = the reference's labelling sweeps, O(N^2) per analysis (default),
 * 1 = union-find giving the same labels, sizes and histograms (cluster
 * energies summed in atom order), for systems too large for the sweeps. */
void orc_set_label_mode(orc_sys* S, int mode);
/* 1 for the atoms the last ten Wolde-Frenkel analysis found liquid. */
int orc_get_liquid(orc_sys* S, int32_t* out);

void orc_scalars_init(const clmd_config* cfg, clmd_scalars* sc);

void orc_set_state(orc_sys* S, const double* x, const double* y, const double* z,
                   const double* vx, const double* vy, const double* vz,
                   const double* ax, const double* ay, const double* az,
                   const int32_t* api, const clmd_scalars* sc);
void orc_get_state(orc_sys* S, double* x, double* y, double* z, double* vx, double* vy,
                   double* vz, double* ax, double* ay, double* az, clmd_scalars* sc);

int orc_neighbor(orc_sys* S, int32_t* step);
int orc_accatom(orc_sys* S);
int orc_zero_acc(orc_sys* S);
int orc_integrator(orc_sys* S, int32_t step);
int orc_thermostat(orc_sys* S, int32_t step);
int orc_stopdead(orc_sys* S, int32_t step);
/* scalev-clu.f:41-83 (the cluster/gas velocity scaling variant) */
int orc_thermostat_clu(orc_sys* S, int32_t step, char eclth, int32_t ecltim);
int orc_stoddard(orc_sys* S, int32_t step);
int orc_chk_nucleation(orc_sys* S, int32_t* step);
/* rates.f:44-100 (appends to out, the reference's unit 67; the write(*,1)
 * lines go to log, NULL = stdout). */
int orc_rates(orc_sys* S, int32_t step, int32_t ctrat, const char* out, const char* log);
int orc_run(orc_sys* S, int32_t first, int32_t nsteps, int32_t* next_step);

int orc_get_halflist(orc_sys* S, int32_t* atnlist, int64_t cap, int32_t* atnidx,
                     int64_t* nentries);
int orc_get_clusters(orc_sys* S, const clmd_cluster_view* v);

/* Timing helper for the CPU baseline: the pair-test loop of
 * neighbor-pbc-mav.f:73-99 over rows i0..i1-1 (0-based) only, on the
 * current positions, without touching the list.  Returns pairs tested. */
int64_t orc_neighbor_rows_sample(orc_sys* S, int32_t i0, int32_t i1);
/* Timing helper: the labelling loop of stoddard-pbc-n-m.f:129-150 is
 * O(N^2) for monomers; this runs the whole routine (same as orc_stoddard). */

/* Reads a .3d deck like read-3d.f:11-302 into cfg (+ the file interval
 * ftcsi, ntim, sctim).  Returns 0 on success. */
int orc_readdata(const char* path, clmd_config* cfg, int32_t* ntim, int32_t* sctim);

/* The engine's seeded start (uniform positions no pair nearer than rmin,
 * Maxwell-Boltzmann velocities), restated so a CPU-only process can build
 * the same inputs without the engine library.  Byte-identical to
 * clmd_init_random(). */
int orc_init_random(int32_t n, double bx, double by, double bz, double rmin, double kT_over_m,
                    uint64_t seed, double* x, double* y, double* z, double* vx, double* vy,
                    double* vz);

/* helpers/passage-time.f:47-90 on one run's (step, largest cluster size)
 * analysis record: pt[0..endsize] first step each size >= startsize was
 * reached (-1 never), probab[0..endsize] the probab.largest counts; returns
 * the first size not reached. */
int orc_passage_time(const int32_t* ts, const int32_t* cs, int32_t nlines, int32_t startsize,
                     int32_t endsize, int32_t warmup, int32_t* pt, int32_t* probab);
/* helpers/mpt.f:52-110 over pooled passage-time lines (size cs[k] first
 * reached at step ts[k]): per size startsize..endsize the mean of
 * ts/500000, its standard error and the count. */
int orc_mpt(const int32_t* ts, const int32_t* cs, int32_t nlines, int32_t startsize,
            int32_t endsize, double* mpt, double* stda, int32_t* count);

#ifdef __cplusplus
}
#endif
#endif
