// clmd_f77.cpp -- the drop-in F77 surface: gfortran-mangled entry points over
// the common blocks, built on the handle API.  See include/clmd_f77.h for the
// ownership rules.
#include "../../include/clmd_f77.h"

#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

extern "C" {
clmd_atomc_t atomc_;
clmd_atomp_t atomp_;
clmd_boxpp_t boxpp_;
clmd_energ_t energ_;
clmd_timep_t timep_;
clmd_dmmpp_t dmmpp_;
clmd_cvtpp_t cvtpp_;
clmd_filep_t filep_;
}

// offsets the Fortran compiler gives these commons (no padding is needed
// in any of them: every REAL*8 member sits at a multiple of 8)
static_assert(offsetof(clmd_atomp_t, apmas) == 48, "ATOMP layout");
static_assert(offsetof(clmd_atomp_t, atnlist) == 504, "ATOMP layout");
static_assert(offsetof(clmd_atomp_t, apsym) ==
                  504 + 4 * ((size_t)CLMD_MXNLIST + 2 * CLMD_MXA + CLMD_MXSORTS + 1),
              "ATOMP layout");
static_assert(offsetof(clmd_boxpp_t, boxt) == 88, "BOXPP layout");
static_assert(offsetof(clmd_energ_t, ecltim) == 144, "ENERG layout");
static_assert(offsetof(clmd_timep_t, ntim) == 8, "TIMEP layout");
static_assert(offsetof(clmd_dmmpp_t, dmmst) == 2104, "DMMPP layout");
static_assert(offsetof(clmd_cvtpp_t, cl) == 8 * (4 * CLMD_MXA + 3 + 2), "CVTPP layout");
static_assert(offsetof(clmd_filep_t, ftxyz) == 400, "FILEP layout");
static_assert(offsetof(clmd_filep_t, ftave) == 500, "FILEP layout");
static_assert(offsetof(clmd_filep_t, ftrat) == 1064, "FILEP layout");

namespace {

clmd_system* g_sys = nullptr;
int g_natom = 0;
bool g_dev_newer = false;  // device state newer than the common blocks
bool g_mirror = false;
int g_integrator = CLMD_INT_VERLET, g_clustering = CLMD_CLU_STILLINGER;

void fatal(int st, int step) {
  // the reference's messages, then STOP
  fprintf(stdout, " %s\n", clmd_status_string(st));
  if (st == CLMD_ERR_NH_NOCONVERGE) fprintf(stdout, " ---> stopping simulation!\n");
  fprintf(stdout, " (step %d)\n", step);
  fflush(stdout);
  exit(1);
}

void read_target() {
  const char* t = getenv("CLMD_TARGET");
  std::string s = t ? t : "SILENT";
  for (auto& ch : s) ch = (char)toupper(ch);
  g_integrator = (s == "NOSE") ? CLMD_INT_NOSE : CLMD_INT_VERLET;
  g_clustering = (s == "FRENKEL") ? CLMD_CLU_FRENKEL : CLMD_CLU_STILLINGER;
  const char* m = getenv("CLMD_SYNC");
  g_mirror = m && std::string(m) == "mirror";
}

void cfg_from_commons(clmd_config* c) {
  memset(c, 0, sizeof(*c));
  c->natom = atomp_.natom;
  c->atsorts = atomp_.atsorts;
  for (int s = 0; s < CLMD_MXSORTS; s++) {
    c->apnum[s] = atomp_.apnum[s];
    c->apmas[s] = atomp_.apmas[s];
    c->apsig[s] = atomp_.apsig[s];
    c->apeps[s] = atomp_.apeps[s];
    c->apth[s] = atomp_.apth[s];
  }
  c->att = atomp_.att;
  c->atskin = atomp_.atskin;
  c->atrcut = atomp_.atrcut;
  c->atrskin = atomp_.atrskin;
  c->Q = atomp_.Q;
  c->atnenum = atomp_.atnenum;
  c->boxx = boxpp_.boxx;
  c->boxy = boxpp_.boxy;
  c->boxz = boxpp_.boxz;
  c->dt = timep_.dt;
  c->nbtim = timep_.nbtim;
  c->btim = timep_.btim;
  c->csover = cvtpp_.csover;
  c->clwait = cvtpp_.clwait;
  c->ftcsi = filep_.ftcsi;
  c->ethst = energ_.ethst;
  c->clnuctrl = cvtpp_.clnuctrl;
  c->integrator = g_integrator;
  c->clustering = g_clustering;
  c->precision = CLMD_PREC_FP64;
  // for-a-lj-n-pbc-mr.f linked instead of for-a-lj-n-pbc-m.f
  const char* fv = getenv("CLMD_FORCE");
  c->forcevar = (fv && strcmp(fv, "mr") == 0) ? 'r' : '-';
}

void scalars_from_commons(clmd_scalars* q) {
  clmd_get_scalars(g_sys, q);  // keeps engine bookkeeping fields
  q->ekin = energ_.ekin;
  q->sumv2 = energ_.sumv2;
  q->epot = energ_.epot;
  q->H = energ_.H;
  q->psi = atomp_.psi;
  q->s = atomp_.s;
  q->atrskin = atomp_.atrskin;
  q->dmms = dmmpp_.dmms;
  q->dmmsu = dmmpp_.dmmsu;
  q->dmmax = dmmpp_.dmmax;
  q->dmmav = dmmpp_.dmmav;
  memcpy(q->dmmh, dmmpp_.dmmh, sizeof(q->dmmh));
  q->dmmst = dmmpp_.dmmst;
  q->dmmi = dmmpp_.dmmi;
  q->clbrkt = cvtpp_.clbrkt;
  q->cnum = cvtpp_.cnum;
  q->cnumf = cvtpp_.cnumf;
  q->cstep = cvtpp_.cstep;
  q->cbiggest = cvtpp_.cbiggest;
  q->cbiggestf = cvtpp_.cbiggestf;
  q->clookfor = cvtpp_.clookfor;
  q->clookforf = cvtpp_.clookforf;
}

void scalars_to_commons(const clmd_scalars& q) {
  energ_.ekin = q.ekin;
  energ_.sumv2 = q.sumv2;
  energ_.epot = q.epot;
  atomp_.psi = q.psi;
  atomp_.s = q.s;
  atomp_.atrskin = q.atrskin;
  dmmpp_.dmms = q.dmms;
  dmmpp_.dmmsu = q.dmmsu;
  dmmpp_.dmmax = q.dmmax;
  dmmpp_.dmmav = q.dmmav;
  memcpy(dmmpp_.dmmh, q.dmmh, sizeof(q.dmmh));
  dmmpp_.dmmst = q.dmmst;
  dmmpp_.dmmi = q.dmmi;
  cvtpp_.clbrkt = q.clbrkt;
  cvtpp_.cnum = q.cnum;
  cvtpp_.cnumf = q.cnumf;
  cvtpp_.cstep = q.cstep;
  cvtpp_.cbiggest = q.cbiggest;
  cvtpp_.cbiggestf = q.cbiggestf;
  cvtpp_.clookfor = q.clookfor;
  cvtpp_.clookforf = q.clookforf;
}

void upload() {
  int N = atomp_.natom;
  clmd_scalars q;
  scalars_from_commons(&q);
  int st = clmd_set_state(g_sys, atomc_.x0, atomc_.y0, atomc_.z0, atomc_.x1, atomc_.y1,
                          atomc_.z1, atomc_.x2, atomc_.y2, atomc_.z2, atomp_.api, &q);
  (void)N;
  if (st) fatal(st, 0);
  g_dev_newer = false;
}

void download_arrays() {
  clmd_scalars q;
  clmd_get_state(g_sys, atomc_.x0, atomc_.y0, atomc_.z0, atomc_.x1, atomc_.y1, atomc_.z1,
                 atomc_.x2, atomc_.y2, atomc_.z2, &q);
  g_dev_newer = false;
}

void publish(int step) {
  clmd_scalars q;
  clmd_get_scalars(g_sys, &q);
  scalars_to_commons(q);
  if (q.status) fatal(q.status, q.fail_step ? q.fail_step : step);
}

void ensure() {
  if (g_sys && g_natom == atomp_.natom) return;
  if (atomp_.natom < 1 || atomp_.natom > CLMD_MXA) {
    fprintf(stdout, " ERROR --- natom %d outside 1..mxa (%d)\n", atomp_.natom, CLMD_MXA);
    exit(1);
  }
  if (g_sys) clmd_destroy(g_sys);
  g_sys = nullptr;
  read_target();
  clmd_config c;
  cfg_from_commons(&c);
  int st = clmd_create(&c, &g_sys);
  if (st) {
    fprintf(stdout, " clmd: cannot create the device system: %s\n", clmd_status_string(st));
    exit(1);
  }
  g_natom = atomp_.natom;
  g_dev_newer = false;
  upload();
}

// the host has seen the latest state -> it may have changed the arrays
void boundary_upload() {
  ensure();
  if (g_mirror || !g_dev_newer) upload();
}

void after_call(int step) {
  publish(step);
  if (g_mirror) download_arrays();
}

bool host_reads_at(int i) {
  auto hit = [&](int every) { return every > 0 && i % every == 0; };
  return hit(filep_.ftxyz) || hit(filep_.ftvel) || hit(filep_.ftacc) || hit(filep_.ftrst) ||
         hit(filep_.ftave) || (atomp_.apNch[0] == 'X' && hit(timep_.chgNtim)) ||
         (boxpp_.bshr == 'X' && hit(boxpp_.boxt)) || hit(filep_.ftrat);
}

void download_clusters() {
  int N = atomp_.natom;
  std::vector<int> csf(N + 1), cgsf(N + 1), cgsfa(N + 1), csi(N + 1), csif(N + 1);
  std::vector<double> cekf(N + 1), ceks(N + 1), ceksf(N + 1);
  clmd_cluster_view v = {};
  v.cl = cvtpp_.cl;
  v.cs = cvtpp_.cs;
  v.cek = cvtpp_.cek;
  v.csi = csi.data();
  v.ceks = ceks.data();
  v.clf = cvtpp_.clf;
  v.csf = csf.data();
  v.csif = csif.data();
  v.cekf = cekf.data();
  v.ceksf = ceksf.data();
  v.cgs = cvtpp_.cgs;
  v.cgsa = cvtpp_.cgsa;
  v.cgsf = cgsf.data();
  v.cgsfa = cgsfa.data();
  v.cfpt = cvtpp_.cfpt;
  v.cfptf = cvtpp_.cfptf;
  clmd_get_clusters(g_sys, &v);
  // (0:mxa) arrays: element 0 first
  memcpy(cvtpp_.csi, csi.data(), sizeof(int) * (N + 1));
  memcpy(cvtpp_.csif, csif.data(), sizeof(int) * (N + 1));
  memcpy(cvtpp_.csf, csf.data(), sizeof(int) * (N + 1));
  memcpy(cvtpp_.cgsf, cgsf.data(), sizeof(int) * (N + 1));
  memcpy(cvtpp_.cgsfa, cgsfa.data(), sizeof(int) * (N + 1));
  memcpy(cvtpp_.cekf, cekf.data(), sizeof(double) * (N + 1));
  memcpy(cvtpp_.ceks, ceks.data(), sizeof(double) * (N + 1));
  memcpy(cvtpp_.ceksf, ceksf.data(), sizeof(double) * (N + 1));
}

}  // namespace

extern "C" {

void neighbor_(int32_t* step) {
  boundary_upload();
  int st = clmd_neighbor(g_sys, step);
  if (st) fatal(st, *step);
  after_call(*step);
  // readRST / initconf / resize / chgNatom read x after the wrap
  download_arrays();
}

void accatom_(void) {
  boundary_upload();
  int st = clmd_accatom(g_sys);
  if (st) fatal(st, 0);
  after_call(0);
  download_arrays();
}

void accwall_(void) {}

void integrator_(int32_t* step) {
  ensure();
  if (g_mirror) upload();
  int st = clmd_integrator(g_sys, *step);
  if (st) fatal(st, *step);
  publish(*step);
  g_dev_newer = true;
  if (g_mirror || host_reads_at(*step + 1)) download_arrays();
}

void thermostat_(int32_t* step) {
  ensure();
  if (g_mirror) upload();
  // CLMD_THERMOSTAT=clu: scalev-clu.f linked instead of scalev-m.f
  const char* tv = getenv("CLMD_THERMOSTAT");
  int st = (tv && strcmp(tv, "clu") == 0)
               ? clmd_thermostat_clu(g_sys, *step, energ_.eclth, energ_.ecltim)
               : clmd_thermostat(g_sys, *step);
  if (st) fatal(st, *step);
  publish(*step);
  g_dev_newer = true;
  if (g_mirror) download_arrays();
}

void stopdead_(int32_t* step) {
  boundary_upload();
  int st = clmd_stopdead(g_sys, *step);
  if (st) fatal(st, *step);
  after_call(*step);
  download_arrays();
}

void stoddard_(int32_t* step) {
  ensure();
  if (g_mirror) upload();
  int st = clmd_stoddard(g_sys, *step);
  if (st) fatal(st, *step);
  publish(*step);
  download_clusters();
}

void chk_nucleation_(int32_t* step) {
  ensure();
  if (g_mirror) upload();
  int st = clmd_chk_nucleation(g_sys, step);
  if (st) fatal(st, *step);
  publish(*step);
  if (*step < 0) {
    printf("\n Found a cluster larger than: %d!\n", cvtpp_.csover);
    printf(" ---> ABORTING simulation at timestep: %d!\n\n", -*step);
  }
}

void chk_nucleation__(int32_t* step) { chk_nucleation_(step); }

// rates.f on the device; unit 67 is the file fxrat names (main.f:49), the
// counters are the /CVTPP/ ones
void rates_(int32_t* step) {
  ensure();
  if (g_mirror) upload();
  char path[81];
  memcpy(path, filep_.fxrat, 80);
  path[80] = 0;
  for (int k = 79; k >= 0 && (path[k] == ' ' || path[k] == 0); k--) path[k] = 0;
  clmd_rates_acc acc = {cvtpp_.mcts, cvtpp_.omcts, cvtpp_.ccn, cvtpp_.cen};
  int st = clmd_rates(g_sys, *step, cvtpp_.ctrat, &acc, path[0] ? path : nullptr, nullptr);
  if (st) fatal(st, *step);
  cvtpp_.mcts = acc.mcts;
  cvtpp_.omcts = acc.omcts;
  cvtpp_.ccn = acc.ccn;
  cvtpp_.cen = acc.cen;
  publish(*step);
  download_clusters();
}

void clmd_f77_reset(void) {
  if (g_sys) clmd_destroy(g_sys);
  g_sys = nullptr;
  g_natom = 0;
  g_dev_newer = false;
}

void clmd_f77_sync_to_host(void) {
  if (!g_sys) return;
  download_arrays();
  publish(0);
}

}  // extern "C"
