/*
 * clmd.h -- C ABI of the B200 engine for the Lennard-Jones MD step and the
 * cluster (nucleation) analysis of the Fortran 77 code "cluster"
 * (janw76/fortran-cluster-md).
 *
 * Two surfaces are exported by libclmd.so:
 *
 *  1. The reference's own subroutine surface with gfortran name mangling
 *     (lower case + trailing underscore), state passed through the common
 *     blocks, so that the unchanged Fortran host (main.f, read-3d.f and the
 *     writers) links against this library instead of the Fortran physics
 *     files.  Declared in clmd_f77.h.
 *
 *  2. A handle based C API (clmd_*) with runtime sizes (no mxa limit) that
 *     the F77 surface is built on, and that C/C++/Python hosts call directly.
 *
 * Conventions of the C API:
 *  - per-atom arrays are 0-based in memory (atom i, 1-based as in the
 *    reference, lives at element i-1); values that ARE atom indices (list
 *    entries, cluster labels) keep the reference's 1-based numbering, so a
 *    downloaded half list is byte-identical to the reference's atnlist();
 *  - histograms indexed by cluster size (csi, csif, ceks, ...) have N+1
 *    elements and are indexed by the size itself, as the reference's
 *    csi(0:mxa);
 *  - every function returns a CLMD_* status code; the first error seen on
 *    the device is also latched in clmd_scalars.status and every later device
 *    kernel of that system is a no-op until clmd_clear_status().
 *
 * Units are the reference's internal ones (length, mass, energy, time and
 * Boltzmann's constant CLMD_CIKB as in const.inc); a reduced-unit run sets
 * sigma = eps = m = 1 and att = T* / CLMD_CIKB.
 */
#ifndef CLMD_H
#define CLMD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* const.inc:10-18 */
#define CLMD_MXA 6000
#define CLMD_MXNLIST (CLMD_MXA * CLMD_MXA / 4)
#define CLMD_MXSORTS 10
#define CLMD_CIKB 1.38066e-6  /* Boltzmann constant, internal units */
#define CLMD_CIMU 1.66056     /* atomic mass unit, internal units */

/* status codes (the reference STOPs on 1-4) */
#define CLMD_OK 0
#define CLMD_ERR_SKIN 1           /* neighbor-pbc-mav.f:48-51 "Skin radius exceeded" */
#define CLMD_ERR_LIST_OVERFLOW 2  /* neighbor-pbc-mav.f:94-98 "Neighborlist is nearly full" */
#define CLMD_ERR_NH_NOCONVERGE 3  /* int-verlet-nh-mav.f:150-166 */
#define CLMD_ERR_BAD_SPECIES 4    /* for-a-lj-n-pbc-m.f:129-130 "Nanu???" */
#define CLMD_ERR_ARG 5            /* bad argument / size beyond a limit */
#define CLMD_ERR_CUDA 6           /* a CUDA runtime call failed */
#define CLMD_ERR_NOMEM 7          /* device allocation failed */
#define CLMD_ERR_NO_DEVICE 8      /* no CUDA device: the engine has no CPU path */
#define CLMD_ERR_TIMEOUT 9        /* a bounded device wait gave up */

/* integrator variants (Makefile:45-88 pick these at link time) */
#define CLMD_INT_VERLET 0 /* int-verlet-mav.f      (targets NUC/SILENT/FRENKEL) */
#define CLMD_INT_NOSE 1   /* int-verlet-nh-mav.f   (target NOSE) */
/* cluster analysis variants */
#define CLMD_CLU_STILLINGER 0 /* stoddard-pbc-n-m.f     (targets NUC/SILENT/NOSE) */
#define CLMD_CLU_FRENKEL 1    /* stoddard-pbc-n-m-fre.f (target FRENKEL) */
/* arithmetic of the pair forces */
#define CLMD_PREC_FP64 0  /* all FP64: bit-identical per-atom forces */
#define CLMD_PREC_MIXED 1 /* FP32 pair terms, Kahan-compensated FP32 sums */

/* Run parameters: the deck (.3d) fields of the hot path, after read-3d.f's
 * unit conversion (read-3d.f:152-161, 246-261). */
typedef struct clmd_config {
  double apmas[CLMD_MXSORTS]; /* mass of species s */
  double apsig[CLMD_MXSORTS]; /* LJ sigma of species s */
  double apeps[CLMD_MXSORTS]; /* LJ epsilon of species s */
  double att;                 /* system temperature */
  double atskin;              /* cluster criterion radius (absolute) */
  double atrcut;              /* potential cut-off radius (absolute) */
  double atrskin;             /* initial neighbour-list radius (absolute) */
  double Q;                   /* Nose-Hoover mass (already * m sigma^2) */
  double boxx, boxy, boxz;    /* periodic box */
  double dt;                  /* time step */
  int64_t nlist_cap;          /* atnlist capacity (mxnlist: headers + half pairs); the
                                 reference's "nearly full" rule applies; 0 = automatic */
  int32_t natom;              /* total atoms */
  int32_t atsorts;            /* species count (1..CLMD_MXSORTS) */
  int32_t apnum[CLMD_MXSORTS];/* atoms per species, contiguous, in order */
  int32_t atnenum;            /* ten Wolde-Frenkel neighbour threshold */
  int32_t nbtim;              /* target steps between list rebuilds */
  int32_t btim;               /* first step number */
  int32_t csover;             /* nucleation size threshold ("a cluster >= csover") */
  int32_t clwait;             /* steps the cluster must persist */
  int32_t ftcsi;              /* steps between cluster analyses (0 = never) */
  int32_t integrator;         /* CLMD_INT_* */
  int32_t clustering;         /* CLMD_CLU_* */
  int32_t precision;          /* CLMD_PREC_* */
  char apth[CLMD_MXSORTS];    /* 'X' = species thermostatted by velocity scaling */
  char ethst;                 /* 'X' velocity scaling every step, 'N' Nose-Hoover, '-' none */
  char clnuctrl;              /* 'X' = abort the run on nucleation */
  char forcevar;              /* 'r': pairs with species 2 are the r^-12 wall of
                                 for-a-lj-n-pbc-mr.f; else LJ (for-a-lj-n-pbc-m.f) */
  char pad[3];
} clmd_config;

/* Dynamic scalars: the hot path's scalar members of /ENERG/, /ATOMP/,
 * /DMMPP/ and /CVTPP/, plus engine bookkeeping. */
typedef struct clmd_scalars {
  double ekin, sumv2, epot, H;   /* energ.inc */
  double psi, s, atrskin;        /* atomp.inc (atrskin adapts at rebuilds) */
  double dmms, dmmsu, dmmax, dmmav;
  double dmmh[256];              /* dmmpp.inc ring of max displacements */
  double virial;                 /* sum over pairs of f_ij r_ij^2 (not in the reference) */
  int64_t npairs_half;           /* half-list entries after the last rebuild */
  int32_t dmmst, dmmi;
  int32_t clbrkt, cnum, cnumf, cstep;
  int32_t cbiggest, cbiggestf, clookfor, clookforf;
  int32_t status;                /* first error, CLMD_OK if none */
  int32_t fail_step;             /* step at which status was set */
  int32_t nh_iters;              /* sweeps of the last Nose-Hoover velocity solve */
  int32_t nrebuild;              /* neighbour-list rebuilds so far */
  int32_t last_rebuild_step;
  int32_t aborted;               /* chk_nucleation negated the step */
  int32_t maxcs;                 /* largest Stillinger cluster of the last analysis */
  int32_t pad;
} clmd_scalars;

/* Cluster-analysis outputs (cvtpp.inc).  Any pointer may be NULL.
 * Sizes: cl, clf: N.  cs, cek, cgs, cgsa, cfpt, cfptf: N, element k-1 holds
 * the reference's index k.  csi, csif, ceks, ceksf, csf, cekf, cgsf, cgsfa:
 * N+1, indexed like the reference's (0:mxa) arrays. */
typedef struct clmd_cluster_view {
  int32_t *cl, *cs, *csi;
  double *cek, *ceks;
  int32_t *clf, *csf, *csif;
  double *cekf, *ceksf;
  int32_t *cgs, *cgsa, *cgsf, *cgsfa;
  int32_t *cfpt, *cfptf;
} clmd_cluster_view;

/* Fills the scalars a fresh run starts from: read-3d.f:263-276 (dmm ring,
 * first-passage cursors) and main.f:156-166 (Nose-Hoover start values need
 * ekin, so psi is left at 0 here). */
void clmd_scalars_init(const clmd_config* cfg, clmd_scalars* sc);

typedef struct clmd_system clmd_system;

/* Allocates the device state of one system on the current CUDA device.
 * Returns CLMD_ERR_NO_DEVICE when no GPU is visible (there is no CPU path). */
int clmd_create(const clmd_config* cfg, clmd_system** out);
int clmd_destroy(clmd_system* sys);

/* Host <-> device state.  Any array pointer may be NULL (not copied).
 * api is the 1-based species of each atom (atomp.inc api()). */
int clmd_set_state(clmd_system* sys, const double* x, const double* y, const double* z,
                   const double* vx, const double* vy, const double* vz,
                   const double* ax, const double* ay, const double* az,
                   const int32_t* api, const clmd_scalars* sc);
int clmd_get_state(clmd_system* sys, double* x, double* y, double* z,
                   double* vx, double* vy, double* vz,
                   double* ax, double* ay, double* az, clmd_scalars* sc);
int clmd_get_scalars(clmd_system* sys, clmd_scalars* sc);
/* The configuration the system was created with. */
int clmd_get_config(clmd_system* sys, clmd_config* cfg);
int clmd_set_scalars(clmd_system* sys, const clmd_scalars* sc);
int clmd_clear_status(clmd_system* sys);

/* The reference's subroutines, one call each (all enqueue on the system's
 * stream; the *_sync variants of the F77 shim wait).  step follows the
 * reference: neighbor() flips a negative step to positive. */
int clmd_neighbor(clmd_system* sys, int32_t* step);        /* neighbor-pbc-mav.f:13-109 */
int clmd_accatom(clmd_system* sys);                        /* for-a-lj-n-pbc-m.f:18-154 */
int clmd_accwall(clmd_system* sys);                        /* for-w-dummy.f:9-14 */
int clmd_zero_acc(clmd_system* sys);                       /* int-verlet-mav.f:76-81 */
int clmd_integrator(clmd_system* sys, int32_t step);       /* int-verlet-mav.f / int-verlet-nh-mav.f */
int clmd_thermostat(clmd_system* sys, int32_t step);       /* scalev-nh-m.f:19-81 */
int clmd_stopdead(clmd_system* sys, int32_t step);         /* stopdead-m.f:10-78 */
int clmd_stoddard(clmd_system* sys, int32_t step);         /* stoddard-pbc-n-m[-fre].f */
int clmd_chk_nucleation(clmd_system* sys, int32_t* step);  /* chk-nucleation.f:15-58 */

/* main.f:177-228 loop body for steps first..first+nsteps-1, device-resident:
 * [stoddard every ftcsi] -> [thermostat if ethst=='X'] ->
 * [chk_nucleation every ftcsi if clnuctrl=='X'] -> integrator.  Replays
 * captured CUDA graphs.  *next_step gets the loop counter after the run
 * (negative if chk_nucleation aborted, as main.f:219-220). */
int clmd_run(clmd_system* sys, int32_t first, int32_t nsteps, int32_t* next_step);

/* The half neighbour list in the reference's layout (atomp.inc atnlist():
 * header -i, then the j>i neighbours ascending) and atnidx().  cap is the
 * capacity of atnlist in entries; *nentries gets the used length. */
int clmd_get_halflist(clmd_system* sys, int32_t* atnlist, int64_t cap,
                      int32_t* atnidx, int64_t* nentries);
int clmd_get_clusters(clmd_system* sys, const clmd_cluster_view* view);

/* nsteps consecutive integrator() calls (steps first..first+nsteps-1) in
 * one launch of the step kernel, without the main loop's analysis. */
int clmd_steps(clmd_system* sys, int32_t first, int32_t nsteps);

/* Selects the CUDA device later clmd_create calls of this thread use
 * (a host that links another CUDA runtime cannot select it for us). */
int clmd_set_device(int device);

/* Waits for the system's stream. */
int clmd_synchronize(clmd_system* sys);
/* Enqueue-only timing helpers: the CUDA stream the system launches on. */
void* clmd_stream(clmd_system* sys);
/* Number of kernels this system has launched (graph replays count each
 * kernel node). */
int64_t clmd_kernel_launches(clmd_system* sys);

/* Seeded synthetic start configuration (not part of the reference's hot
 * path): positions uniform in the box with every pair at least rmin apart
 * (random sequential addition on a cell grid), Maxwell-Boltzmann velocities
 * at temperature kT for mass m (unit-free: v = sqrt(kT/m) * N(0,1)).
 * Returns CLMD_ERR_ARG if the packing is too dense to finish. */
int clmd_init_random(int32_t n, double boxx, double boxy, double boxz, double rmin,
                     double kT_over_m, uint64_t seed, double* x, double* y, double* z,
                     double* vx, double* vy, double* vz);

/* ---------------------------------------------------------------------------
 * Ensembles: many independent replicas (batched nucleation runs, served
 * requests) in one persistent launch.  Reduced LJ units (sigma = eps = m = 1, one
 * species), the same per-replica algorithm as the drop-in (adaptive-skin
 * Verlet list, velocity Verlet or Nose-Hoover, Stillinger analysis every
 * ftcsi steps, chk_nucleation), with FP32 pair terms accumulated per atom in
 * FP32 with Kahan compensation (CLMD_PREC_MIXED) or all FP64.  Replicas are
 * admitted while the atom pool has room and run window by window (one
 * analysis + ftcsi steps), finished ones are retired: continuous batching.
 * ------------------------------------------------------------------------- */
typedef struct clmd_ens_config {
  double rc, rskin, atskin, dt;  /* sigma units: cut-off, initial list radius, cluster radius */
  int64_t max_atoms;             /* atom pool (the admission budget) */
  int32_t max_replicas;
  int32_t list_stride;           /* neighbour slots per atom (full rows); 0 = 192 */
  int32_t precision;             /* CLMD_PREC_MIXED or CLMD_PREC_FP64 */
  int32_t integrator;            /* CLMD_INT_VERLET or CLMD_INT_NOSE */
  int32_t ftcsi;                 /* steps per window (between cluster analyses) */
  int32_t nbtim;                 /* target steps between list rebuilds */
  int32_t threads;               /* threads per replica (CTA size, | CLMD_ENS_LEAN); 0 = autotune */
  int32_t pad;
} clmd_ens_config;

typedef struct clmd_replica_spec {
  double box;        /* cubic box edge */
  double temp;       /* T* */
  double Q;          /* Nose-Hoover mass (reduced), <= 0: N T* 0.25 */
  int32_t natom;
  int32_t csover;    /* nucleated once a cluster >= csover persists (chk-nucleation.f) */
  int32_t clwait;
  int32_t budget;    /* step budget */
  char ethst;        /* 'N' Nose-Hoover thermostat on, '-' off */
  char pad[7];
} clmd_replica_spec;

typedef struct clmd_replica_result {
  double ekin, epot, psi, s;
  int32_t slot, natom, step, status;
  int32_t done;        /* 1 nucleated, 2 budget spent, 0 running */
  int32_t clbrkt;      /* first step the >= csover cluster was seen (time to nucleation) */
  int32_t maxcs;       /* largest cluster at the last analysis */
  int32_t nrebuild;
} clmd_replica_result;

typedef struct clmd_ensemble clmd_ensemble;

int clmd_ens_create(const clmd_ens_config* cfg, clmd_ensemble** out);
int clmd_ens_destroy(clmd_ensemble* e);
/* Admits a replica from host positions/velocities (x..vz, natom each): the
 * reference's start (stopdead(-1), neighbor(0), AccAtom, and main.f:156-160
 * for PSI) runs on the device at the next step call.  *slot gets its id.
 * CLMD_ERR_NOMEM when the pool or the replica table has no room now. */
int clmd_ens_add(clmd_ensemble* e, const clmd_replica_spec* spec, const double* x,
                 const double* y, const double* z, const double* vx, const double* vy,
                 const double* vz, int32_t* slot);
/* Advances every running replica by up to nwin windows of ftcsi steps (one
 * persistent launch per size class, the classes concurrently); replicas stop
 * when done.  A replica runs on one CTA, or -- when its positions do not fit
 * in one SM's shared memory (about 9,000 atoms and more) -- on a
 * thread-block cluster of 2, 4, 8 or 16 CTAs (about 6,144 atoms per CTA or
 * more) that splits its atoms and meets at cluster barriers
 * (CLMD_ENS_CLUSTERS=0 in the environment at creation: one CTA each).  The
 * launch sequence is captured once into a CUDA graph and replayed while the
 * set of running replicas and the launch shapes stay the same
 * (CLMD_ENS_GRAPHS=0 in the environment at creation: direct launches). */
int clmd_ens_step(clmd_ensemble* e, int32_t nwin);
/* Balanced step for mixed sizes: every running replica advances for about
 * ms of device time (at least one MD step), from the time per step the
 * kernel measured for it in earlier launches (a replica not yet timed runs
 * a few steps); when the replicas' CTAs cannot all be resident at once, a
 * replica on a cluster of c CTAs runs for about ms / c instead (the same SM
 * time as a single-CTA replica).  Small replicas then do not idle while the largest finish,
 * and a launch lasts about ms whatever the sizes.  Launch boundaries may
 * fall inside a window: the analysis still runs at every multiple of ftcsi,
 * and trajectories are those of clmd_ens_step. */
int clmd_ens_step_timed(clmd_ensemble* e, float ms);
/* Block shape flag: the register-lean variant of a 128-, 256- or 512-thread
 * CTA (64 registers per thread, so 8, 4 or 2 CTAs fit per SM where shared
 * memory allows; the plain shapes allow up to 128 registers below 1024
 * threads). */
#define CLMD_ENS_LEAN 0x10000
/* Block shape field: lanes per atom in the mixed-precision force pass,
 * 1 << ((shape >> CLMD_ENS_LANES_SHIFT) & 3), i.e. 1, 2 or 4 (consecutive
 * lanes share an atom's row and merge their Kahan sums in a fixed tree). */
#define CLMD_ENS_LANES_SHIFT 20
/* Autotuner: picks the block shape of each of the 4 replica-size classes
 * (atoms <= 2048, <= 4096, <= 6144, larger) from 128, 256, 512, 1024 and
 * the CLMD_ENS_LEAN 128, 256 and 512 by timing one window per candidate and
 * class, each class alone on the GPU, on the running replicas; then, in
 * mixed precision, the lanes per atom of the force pass (1, 2 or 4) with
 * that shape.  Every replica advances by those 7 (+ 2) windows.  threads_out (4 entries, may be NULL) gets the choice (threads
 * in the low 16 bits).  Without it the classes use lean 512, 1024, 1024 and
 * 1024 threads (the tuner's picks on the batched workload), or
 * clmd_ens_config.threads for all if that is set (the flag allowed). */
int clmd_ens_autotune(clmd_ensemble* e, int32_t* threads_out);
/* Per-slot results of all occupied slots (n gets the count). */
int clmd_ens_results(clmd_ensemble* e, clmd_replica_result* out, int32_t cap, int32_t* n);
/* Per-window status without the full table copy: for every occupied slot
 * slot, natom, step, status, done and maxcs from the summary the last step
 * call read back; the rest of the record (energies, clbrkt, nrebuild) only
 * for replicas that finished (done != 0 or status != 0), zero otherwise. */
int clmd_ens_poll(clmd_ensemble* e, clmd_replica_result* out, int32_t cap, int32_t* n);
/* Frees a finished (or unwanted) replica's pool range and slot. */
int clmd_ens_remove(clmd_ensemble* e, int32_t slot);
/* Copies one replica's state (x..vz, ax..az, cluster labels cl, 1-based) out;
 * any pointer may be NULL. */
int clmd_ens_get_state(clmd_ensemble* e, int32_t slot, double* x, double* y, double* z,
                       double* vx, double* vy, double* vz, double* ax, double* ay,
                       double* az, int32_t* cl);
/* Bulk host<->device copies of every occupied slot's x..vz, concatenated in
 * slot order (natom of each slot, as admitted).  NULL arrays are skipped. */
int clmd_ens_upload(clmd_ensemble* e, const double* x, const double* y, const double* z,
                    const double* vx, const double* vy, const double* vz);
int clmd_ens_download(clmd_ensemble* e, double* x, double* y, double* z, double* vx,
                      double* vy, double* vz);
/* clmd_ens_upload + clmd_ens_step(nwin) + clmd_ens_download in one call, with
 * the copies done by the window kernel itself: each running replica's x..vz
 * are read from these host arrays when a CTA takes the replica and written
 * back when it leaves it, so the transfers of one replica overlap the
 * compute of the others.  The arrays use the upload/download layout and must
 * be pinned host memory (cudaMallocHost / cudaHostAlloc / cudaHostRegister:
 * anything else returns CLMD_ERR_ARG); finished replicas' parts are neither
 * read nor written.  Returns when the windows are done. */
int clmd_ens_step_io(clmd_ensemble* e, int32_t nwin, double* x, double* y, double* z,
                     double* vx, double* vy, double* vz);
/* First step at which the largest cluster reached each size 1..cap (-1 if
 * not yet). */
int clmd_ens_fpt(clmd_ensemble* e, int32_t slot, int32_t* fpt, int32_t cap);
/* ---- restart files and analysis writers ---------------------------------
 * wrt-rst.f:30-45: the reference's restart file, a gfortran unformatted
 * sequential file (each record framed by its 4-byte length): mxa;
 * (ekin, epot, ekin, epot, ekin); (ewall, ewallsum, fwall, fwallsum), zero
 * here (no wall); x0,y0,z0; x1,y1,z1; x2,y2,z2; and the Gear derivatives
 * x3..z5, zero here; every array padded to mxa entries (mxa <= 0: natom).
 * One more record follows the reference's ones: the engine state that the
 * reference would rebuild from the deck (PSI, s, the adaptive list radius,
 * the displacement ring, the cluster cursors), tagged "CLMDSC01" + the
 * clmd_scalars struct.  A Fortran readRST never reads past its own records. */
int clmd_write_rst(clmd_system* sys, const char* path, int32_t mxa);
/* read-rst.f:37-65: loads x, v, a and (ekin, epot) from such a file (its mxa
 * must hold natom atoms, else CLMD_ERR_ARG), the engine record when present,
 * then rebuilds the list as the reference does: step = btim,
 * neighbor(step).  *step (may be NULL) gets btim. */
int clmd_read_rst(clmd_system* sys, const char* path, int32_t* step);
/* wrt-csi.f (Stillinger) / wrt-csi-fre.f:32-57 (ten Wolde-Frenkel): appends
 * this step's cluster-size distribution from the last stoddard() to
 * csi_path and, for ten Wolde-Frenkel, the liquid-cluster one to fsi_path
 * (NULL: skipped), in the reference's fixed formats. */
int clmd_write_csi(clmd_system* sys, int32_t step, const char* csi_path, const char* fsi_path);
/* wrt-fpt.f:30-37: the first-passage table (size, Stillinger time, tWF time
 * in the reference's dt*1e6 units), appended to path. */
int clmd_write_fpt(clmd_system* sys, const char* path);
/* One replica's restart file (reference records; its engine record, tagged
 * "CLMDRP01", is the replica's clmd_replica_result) and its first-passage table in the
 * wrt-fpt.f layout (Stillinger column; the tWF column is -1 / the
 * reference's placeholder). */
int clmd_ens_write_rst(clmd_ensemble* e, int32_t slot, const char* path, int32_t mxa);
int clmd_ens_write_fpt(clmd_ensemble* e, int32_t slot, double dt, const char* path);
/* rates.f:44-100: condensation / evaporation of the largest cluster.  Keeps
 * the previous analysis's labels, sizes and kinetic energies, runs
 * stoddard(step) unless this step was analysed already (then the
 * reference's warning), finds the largest cluster before and after (first
 * label of the largest size), counts atoms that joined (cn) and left (en)
 * it, and appends the reference's unit-67 line to out every ctrat steps
 * (ctrat = 1: every call with cn + en != 0); the write(*,1) line for a
 * change of size goes to log (NULL: stdout).  acc holds the /CVTPP/
 * counters the reference keeps across calls (zero them at the start, as
 * read-3d.f:109-111 does). */
typedef struct clmd_rates_acc {
  double mcts, omcts;  /* cvtpp.inc mcts, omcts */
  int32_t ccn, cen;    /* cvtpp.inc ccn, cen */
} clmd_rates_acc;
int clmd_rates(clmd_system* sys, int32_t step, int32_t ctrat, clmd_rates_acc* acc,
               const char* out, const char* log);
/* scalev-clu.f:41-83, the cluster/gas velocity scaling variant of
 * thermostat(step): when eclth == 'X' and step is a multiple of ecltim
 * (read-3d.f:176-180), stoddard(step) if not done, then the biggest cluster
 * (first label of the largest size) is scaled to 1.5 kT per atom and the
 * rest of the system separately; otherwise every velocity is scaled by
 * sqrt(ekinT / ekin) with the current ekin.  ekin = ekinT afterwards. */
int clmd_thermostat_clu(clmd_system* sys, int32_t step, char eclth, int32_t ecltim);
/* Mean first-passage statistics over the occupied slots, on the device
 * (helpers/passage-time.f + helpers/mpt.f:80-92 in one pass): for each size
 * j = 1..cap, count[j-1] replicas whose largest cluster reached j, the mean
 * of their first-passage steps (-1 when none) and its standard error
 * sqrt((<t^2> - <t>^2) / count).  Steps, not time: multiply by dt. */
int clmd_ens_mfpt(clmd_ensemble* e, int32_t cap, double* mean, double* sem, int32_t* count);
/* Device time (ms, CUDA events) of the last window's launch of each of the 4
 * size classes (-1 if the class was empty) and the atoms it advanced; the
 * fourth entry also covers the replicas run on thread-block clusters (the
 * longest of those launches, the sum of their atoms). */
int clmd_ens_last_ms(clmd_ensemble* e, float* ms, int64_t* atoms);
/* Pair terms (full neighbour-list entries, each an FP64 minimum image and
 * cut-off test and, within rc, an LJ term) the force passes of all current
 * replicas have evaluated since admission: the work measure of the force
 * kernel. */
int clmd_ens_pair_terms(clmd_ensemble* e, int64_t* total);
/* Atoms currently free in the pool. */
int64_t clmd_ens_free_atoms(clmd_ensemble* e);
/* Kernel launches issued so far. */
int64_t clmd_ens_launches(clmd_ensemble* e);

/* ---- served mode: continuous batching over a request trace ---------------
 * Requests arrive at given times (seconds after the call starts).  At every
 * window boundary the loop admits, in arrival order, each arrived request
 * whose start state is ready and whose atoms fit the free pool (the pool is
 * the admission budget, sized from free device memory by the caller), runs
 * one window for everything resident, and retires replicas whose largest
 * cluster crossed csover (chk_nucleation) or whose budget is spent.  Start
 * states (uniform positions, pairs >= 0.9 apart, Maxwell-Boltzmann) are
 * generated ahead of admission by a pool of host threads. */
typedef struct clmd_request {
  double arrival;    /* seconds after the start of clmd_serve */
  double rho, temp;  /* reduced density and temperature */
  uint64_t seed;
  int32_t natom, budget, csover, pad;
} clmd_request;

typedef struct clmd_request_result {
  double arrival, admitted, finished; /* seconds; admitted/finished < 0: never */
  int32_t natom, steps;               /* steps run */
  int32_t done;                       /* 1 nucleated, 2 budget spent, 0 not finished
                                         or failed (status) */
  int32_t clbrkt;                     /* step the >= csover cluster was first seen */
  int32_t status;                     /* CLMD_OK, or the error that ended the replica */
  int32_t pad;
} clmd_request_result;

typedef struct clmd_serve_stats {
  double wall;        /* seconds */
  double atom_steps;  /* every replica's steps x atoms */
  int32_t windows, admitted, completed, peak_resident;
  int64_t peak_atoms;
} clmd_serve_stats;

/* Runs the trace until every request finished or max_seconds passed.
 * out[nreq] gets per-request timings. */
int clmd_serve(clmd_ensemble* e, const clmd_request* reqs, int32_t nreq, double max_seconds,
               clmd_request_result* out, clmd_serve_stats* stats);

/* No counterpart in the reference: the Stillinger analysis (what stoddard()
 * of stoddard-pbc-n-m.f computes: labels cl, sizes cs, histogram csi) for
 * callers that cannot let the library allocate device memory -- hosts that
 * pass only buffers from their own pool or fixed budget.  It allocates
 * nothing: its one scratch array (the union-find parents) is a file-scope
 * device array of CLMD_NOALLOC_MAX_ATOMS ints (4 MiB) that every GPU which
 * loads the library holds until exit.  All pointers are device pointers:
 * x, y, z, api (1-based species), the reference's half list atnlist (nlist
 * entries) and atnidx, and the outputs cl[natom], cs[natom],
 * csi[natom+1] (csi[0] accumulates across calls like the reference's).
 * Enqueued on `stream`; natom > CLMD_NOALLOC_MAX_ATOMS returns CLMD_ERR_ARG.
 * Every call looks up the array's address on the current device; the first
 * call on a device loads the module (make it before any stream capture).  A
 * CUDA error left pending by the caller's earlier work is reported as
 * CLMD_ERR_CUDA, without launching and without clearing it.  Every call
 * shares the array, so calls that overlap on the GPU race: serialise them. */
#define CLMD_NOALLOC_MAX_ATOMS (1 << 20)
int clmd_stoddard_noalloc(int32_t natom, const double* x, const double* y, const double* z,
                          const int32_t* api, const int32_t* atnlist, int64_t nlist,
                          const int32_t* atnidx, double boxx, double boxy, double boxz,
                          double atrskin, double sigma1, double atskin, int32_t* cl,
                          int32_t* cs, int32_t* csi, void* stream);

/* Failure-path testing of the grid barrier of the persistent kernels: from
 * now on every barrier of this system waits for `extra_arrivals` blocks
 * beyond the grid (none come) and gives up after `spin_limit` polls (0: the
 * default, ~2 s); the launch then ends with CLMD_ERR_TIMEOUT, latched in the
 * status like any other error.  (0, 0) restores normal barriers.  Only for
 * tests: a timed-out system must be cleared (clmd_clear_status) or dropped. */
int clmd_debug_barrier(clmd_system* S, int32_t extra_arrivals, int64_t spin_limit);

const char* clmd_status_string(int status);
/* sizeof of the ABI structs (0 config, 1 scalars, 2 cluster view, 3 ensemble
 * config, 4 replica spec, 5 replica result, 6 request, 7 request result,
 * 8 serve stats), so that bindings in other languages can check their
 * layout. */
int64_t clmd_struct_size(int which);
/* Last status returned by any clmd_* or F77 entry point of this process. */
int32_t clmd_last_status(void);

#ifdef __cplusplus
}
#endif

#endif /* CLMD_H */
