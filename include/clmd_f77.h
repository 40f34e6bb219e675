/*
 * clmd_f77.h -- the reference's own subroutine surface, exported by
 * libclmd.so with gfortran's external-name mangling (lower case + '_'),
 * and the common blocks it reads and writes, laid out member for member as
 * the `common` statements of the reference's .inc files (mxa = 6000,
 * const.inc:10-12).  A Fortran host that links main.f, read-3d.f and the
 * writers against libclmd.so instead of the physics .f files gets the same
 * call sequence; each entry point below replaces the subroutine cited.
 *
 * Which variant a call runs is chosen at run time by the environment
 * variable CLMD_TARGET, named after the Makefile targets that choose it at
 * link time: SILENT / NUC (int-verlet-mav + stoddard-pbc-n-m, default),
 * FRENKEL (int-verlet-mav + stoddard-pbc-n-m-fre), NOSE (int-verlet-nh-mav +
 * stoddard-pbc-n-m + scalev-nh-m) -- Makefile:36-88.
 *
 * Host/device ownership (CLMD_SYNC):
 *   resident (default): the device holds x,v,a between calls.  The shim
 *     uploads the common blocks at the first call and at every host-called
 *     neighbor_/stopdead_/accatom_ when the host has seen the latest state
 *     (these are the reference's init/restart/N-change boundaries), and
 *     downloads x0..z2 after integrator_(i) when step i+1 runs a host
 *     reader (ftxyz/ftvel/ftacc/ftrst/ftave, chgNtim, boxt).  Scalars
 *     (ekin, epot, sumv2, psi, s, atrskin, dmm*, cluster scalars) are
 *     published after every call; cluster arrays after every stoddard_.
 *   mirror: every call uploads the common blocks and downloads them again.
 * Errors: the reference STOPs; so does the shim (same message, exit 1).
 */
#ifndef CLMD_F77_H
#define CLMD_F77_H

#include <stdint.h>

#include "clmd.h"

#ifdef __cplusplus
extern "C" {
#endif

/* atomc.inc:19-20 */
typedef struct clmd_atomc_t {
  double x0[CLMD_MXA], y0[CLMD_MXA], z0[CLMD_MXA];
  double x1[CLMD_MXA], y1[CLMD_MXA], z1[CLMD_MXA];
  double x2[CLMD_MXA], y2[CLMD_MXA], z2[CLMD_MXA];
  double x3[CLMD_MXA], y3[CLMD_MXA], z3[CLMD_MXA];
  double x4[CLMD_MXA], y4[CLMD_MXA], z4[CLMD_MXA];
  double x5[CLMD_MXA], y5[CLMD_MXA], z5[CLMD_MXA];
} clmd_atomc_t;

/* atomp.inc:27-31 */
typedef struct clmd_atomp_t {
  int32_t natom, atsorts, apnum[CLMD_MXSORTS];
  double apmas[CLMD_MXSORTS], apsig[CLMD_MXSORTS], apeps[CLMD_MXSORTS];
  double appr[CLMD_MXSORTS], appa[CLMD_MXSORTS];
  double atskin, atrskin, atrcut, att, psi, Q, s;
  int32_t atnlist[CLMD_MXNLIST], atnidx[CLMD_MXA], api[CLMD_MXA];
  int32_t apnnum[CLMD_MXSORTS], atnenum;
  char apsym[CLMD_MXSORTS][2], apsymi[CLMD_MXA][2], apth[CLMD_MXSORTS];
  char apNch[CLMD_MXSORTS], rndctrl;
} clmd_atomp_t;

/* boxpp.inc:13-15 */
typedef struct clmd_boxpp_t {
  double boxx, boxy, boxz, boxxn, boxyn, boxzn, boxxs, boxys, boxzs, bpot, beng;
  int32_t boxt;
  char bcor, bshr, bperx, bpery, bperz;
} clmd_boxpp_t;

/* energ.inc:12-15 */
typedef struct clmd_energ_t {
  double ekin, sumv2, epot, ekinA[CLMD_MXSORTS], H, ewall, ewallsum, fwall, fwallsum;
  int32_t ecltim;
  char ethst, eclth;
} clmd_energ_t;

/* timep.inc:9 */
typedef struct clmd_timep_t {
  double dt;
  int32_t ntim, btim, sctim, nbtim, chgNtim;
} clmd_timep_t;

/* dmmpp.inc:12-13 */
typedef struct clmd_dmmpp_t {
  double dmmh[256], dmmx, dmmy, dmmz, dmms, dmmsu, dmmax, dmmav;
  int32_t dmmst, dmmi;
} clmd_dmmpp_t;

/* cvtpp.inc:17-20 */
typedef struct clmd_cvtpp_t {
  double cek[CLMD_MXA], cekf[CLMD_MXA + 1], ceks[CLMD_MXA + 1], ceksf[CLMD_MXA + 1];
  double mcts, omcts;
  int32_t cl[CLMD_MXA], clf[CLMD_MXA], cs[CLMD_MXA], csf[CLMD_MXA + 1], cc[CLMD_MXA];
  int32_t ccf[CLMD_MXA], csi[CLMD_MXA + 1], csif[CLMD_MXA + 1], cgs[CLMD_MXA];
  int32_t cgsf[CLMD_MXA + 1], cgsa[CLMD_MXA], cgsfa[CLMD_MXA + 1], cnum, cnumf;
  int32_t cfpt[CLMD_MXA], cfptf[CLMD_MXA], ccn, cen, ctrat, cstep, csover, cbiggest;
  int32_t cbiggestf, clookfor, clookforf, clwait, clbrkt;
  char clnuctrl;
} clmd_cvtpp_t;

/* filep.inc:13-17 */
typedef struct clmd_filep_t {
  char fpath[40], fxyz[40], fvel[40], facc[40], frst[40], fcsi[40], fcsif[40], fave[40];
  char finp[40], frat[40];
  int32_t ftxyz, ftvel, ftacc, ftrst, ftcsi;
  char fxcsif[80];
  int32_t ftave;
  char fxinp[80], fxxyz[80], fxvel[80], fxacc[80], fxrst[80], fxcsi[80], fxave[80];
  int32_t ftrat;
  char fxrat[80], frctrl, ffpt[40], fxfpt[80];
} clmd_filep_t;

extern clmd_atomc_t atomc_;
extern clmd_atomp_t atomp_;
extern clmd_boxpp_t boxpp_;
extern clmd_energ_t energ_;
extern clmd_timep_t timep_;
extern clmd_dmmpp_t dmmpp_;
extern clmd_cvtpp_t cvtpp_;
extern clmd_filep_t filep_;

void neighbor_(int32_t* step);       /* neighbor-pbc-mav.f:13 / neighbor-pbc-mav-silent.f:13 */
void accatom_(void);                 /* for-a-lj-n-pbc-m.f:18 */
void accwall_(void);                 /* for-w-dummy.f:9 */
void integrator_(int32_t* step);     /* int-verlet-mav.f:18 / int-verlet-nh-mav.f:13 */
void thermostat_(int32_t* step);     /* scalev-m.f:15 / scalev-nh-m.f:19 */
void stopdead_(int32_t* step);       /* stopdead-m.f:10 */
void stoddard_(int32_t* step);       /* stoddard-pbc-n-m.f:11 / stoddard-pbc-n-m-fre.f:11 */
void chk_nucleation_(int32_t* step); /* chk-nucleation.f:15 */
void chk_nucleation__(int32_t* step);/* same, g77 / -fsecond-underscore mangling */
/* rates.f:12-100 (rates(step), main.f:119 when ftrat != 0): appends to the
 * file fxrat names; /CVTPP/ ccn, cen, mcts, omcts, ctrat as in the
 * reference. */
void rates_(int32_t* step);

/* read-3d.f:11-302 for C/C++ hosts without a Fortran readdata(): parses the
 * .3d deck at path into the common blocks (returns 0 on success). */
int clmd_f77_readdata(const char* path);
/* Drops the device copy (the next call re-uploads the common blocks). */
void clmd_f77_reset(void);
/* Copies the device state into the common blocks now. */
void clmd_f77_sync_to_host(void);

#ifdef __cplusplus
}
#endif
#endif
