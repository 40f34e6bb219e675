/*
 * clmd_oracle.c -- TEST INFRASTRUCTURE ONLY (see clmd_oracle.h).
 *
 * Serial FP64 restatement of the reference's hot path with gfortran -O2
 * semantics: left-to-right evaluation, no FMA contraction (built with
 * -ffp-contract=off), Fortran int() = truncation toward zero, dmod = fmod,
 * REAL(4) literals (0.5, 2.0) and real(dmmst) promoted exactly.  Arrays are
 * kept 1-based internally so that every loop reads like the Fortran it
 * follows; file:line citations refer to janw76/fortran-cluster-md/cluster/.
 *
 * Pinned by: analytic LJ known answers, hand-derived fixtures
 * (tests/golden/), the all-pairs / cell-list cross-check.  The reference
 * ships no golden vectors and cannot be compiled here (no Fortran compiler).
 */
#include "clmd_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

struct orc_sys {
  clmd_config c;
  clmd_scalars sc;
  int N;
  int nbmode;
  int lbmode; /* 0: the reference's O(N^2) labelling loops, 1: union-find */
  /* atomc.inc / atomp.inc, 1-based */
  double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az;
  int *api;
  int *atnlist; /* 1-based, capacity nl_cap */
  int64_t nl_cap, nl_used;
  int *atnidx;
  /* cvtpp.inc, 1-based (0:N where the reference has 0:mxa) */
  int *cl, *clf, *cs, *csf, *cc, *ccf, *csi, *csif, *cgs, *cgsf, *cgsa, *cgsfa, *cfpt, *cfptf;
  double *cek, *cekf, *ceks, *ceksf;
  /* NH scratch (int-verlet-nh-mav.f:28-30) */
  double *vxn, *vyn, *vzn, *vxo, *vyo, *vzo, *bx, *by, *bz;
  double *fsx, *fsy, *fsz; /* for-a-lj-n-pbc-m.f:37 */
  /* rates.f: its local ocs/ocl/ocek and the /CVTPP/ counters */
  int *ocs, *ocl;
  double* ocek;
  int ccn, cen;
  double mcts, omcts;
};

static void* xc(size_t n, size_t sz) {
  void* p = calloc(n ? n : 1, sz);
  if (!p) {
    fprintf(stderr, "oracle: out of memory\n");
    abort();
  }
  return p;
}

static int latch(orc_sys* S, int st, int step) {
  if (S->sc.status == CLMD_OK && st != CLMD_OK) {
    S->sc.status = st;
    S->sc.fail_step = step;
  }
  return S->sc.status;
}

/* read-3d.f:263-276 */
void orc_scalars_init(const clmd_config* c, clmd_scalars* sc) {
  memset(sc, 0, sizeof(*sc));
  sc->atrskin = c->atrskin;
  for (int i = 0; i < 256; i++) sc->dmmh[i] = (c->atrskin - c->atrcut) / (double)(float)c->nbtim;
  sc->dmmst = 0;
  sc->dmmi = 0;
  sc->dmmsu = 256.0 * (c->atrskin - c->atrcut) / (double)(float)c->nbtim;
  sc->dmms = 0.0;
  sc->clookfor = 1;
  sc->clookforf = 1;
  sc->cbiggest = 0;
  sc->cbiggestf = 0;
  sc->cstep = -1;
  sc->last_rebuild_step = -1;
}

orc_sys* orc_create(const clmd_config* cfg) {
  orc_sys* S = (orc_sys*)xc(1, sizeof(orc_sys));
  S->c = *cfg;
  int N = cfg->natom;
  S->N = N;
  size_t n1 = (size_t)N + 2;
  S->x = xc(n1, 8); S->y = xc(n1, 8); S->z = xc(n1, 8);
  S->vx = xc(n1, 8); S->vy = xc(n1, 8); S->vz = xc(n1, 8);
  S->ax = xc(n1, 8); S->ay = xc(n1, 8); S->az = xc(n1, 8);
  S->api = xc(n1, 4);
  S->nl_cap = cfg->nlist_cap > 0 ? cfg->nlist_cap : (int64_t)N * 64 + 1024;
  S->atnlist = xc((size_t)S->nl_cap + 2, 4);
  S->atnidx = xc(n1, 4);
  S->cl = xc(n1, 4); S->clf = xc(n1, 4); S->cs = xc(n1, 4); S->csf = xc(n1, 4);
  S->cc = xc(n1, 4); S->ccf = xc(n1, 4); S->csi = xc(n1, 4); S->csif = xc(n1, 4);
  S->cgs = xc(n1, 4); S->cgsf = xc(n1, 4); S->cgsa = xc(n1, 4); S->cgsfa = xc(n1, 4);
  S->cfpt = xc(n1, 4); S->cfptf = xc(n1, 4);
  S->cek = xc(n1, 8); S->cekf = xc(n1, 8); S->ceks = xc(n1, 8); S->ceksf = xc(n1, 8);
  S->vxn = xc(n1, 8); S->vyn = xc(n1, 8); S->vzn = xc(n1, 8);
  S->vxo = xc(n1, 8); S->vyo = xc(n1, 8); S->vzo = xc(n1, 8);
  S->bx = xc(n1, 8); S->by = xc(n1, 8); S->bz = xc(n1, 8);
  S->fsx = xc(n1, 8); S->fsy = xc(n1, 8); S->fsz = xc(n1, 8);
  /* read-3d.f:228-253: api() by contiguous species blocks */
  int n = 1;
  for (int s = 1; s <= cfg->atsorts; s++)
    for (int j = 0; j < cfg->apnum[s - 1] && n <= N; j++) S->api[n++] = s;
  /* read-3d.f:297-298 */
  for (int i = 1; i <= N; i++) { S->cfpt[i] = -1; S->cfptf[i] = -1; }
  orc_scalars_init(cfg, &S->sc);
  return S;
}

void orc_destroy(orc_sys* S) {
  if (S && S->ocs) {
    free(S->ocs);
    free(S->ocl);
    free(S->ocek);
  }
  if (!S) return;
  void* ps[] = {S->x, S->y, S->z, S->vx, S->vy, S->vz, S->ax, S->ay, S->az, S->api,
                S->atnlist, S->atnidx, S->cl, S->clf, S->cs, S->csf, S->cc, S->ccf,
                S->csi, S->csif, S->cgs, S->cgsf, S->cgsa, S->cgsfa, S->cfpt, S->cfptf,
                S->cek, S->cekf, S->ceks, S->ceksf, S->vxn, S->vyn, S->vzn, S->vxo,
                S->vyo, S->vzo, S->bx, S->by, S->bz, S->fsx, S->fsy, S->fsz};
  for (size_t i = 0; i < sizeof(ps) / sizeof(ps[0]); i++) free(ps[i]);
  free(S);
}

void orc_set_neighbor_mode(orc_sys* S, int mode) { S->nbmode = mode; }
void orc_set_label_mode(orc_sys* S, int mode) { S->lbmode = mode; }

/* ccf() of the last ten Wolde-Frenkel analysis: 1 for the liquid atoms
 * (stoddard-pbc-n-m-fre.f:148-168 puts exactly those in liqmon, and the
 * component sweep :198-225 visits every one of them), 0 otherwise. */
int orc_get_liquid(orc_sys* S, int32_t* out) {
  if (!out) return CLMD_ERR_ARG;
  for (int i = 1; i <= S->N; i++) out[i - 1] = S->ccf[i];
  return CLMD_OK;
}

static void cp_in(double* dst1, const double* src0, int N) {
  if (src0) memcpy(dst1 + 1, src0, sizeof(double) * (size_t)N);
}
static void cp_out(double* dst0, const double* src1, int N) {
  if (dst0) memcpy(dst0, src1 + 1, sizeof(double) * (size_t)N);
}

void orc_set_state(orc_sys* S, const double* x, const double* y, const double* z,
                   const double* vx, const double* vy, const double* vz,
                   const double* ax, const double* ay, const double* az,
                   const int32_t* api, const clmd_scalars* sc) {
  int N = S->N;
  cp_in(S->x, x, N); cp_in(S->y, y, N); cp_in(S->z, z, N);
  cp_in(S->vx, vx, N); cp_in(S->vy, vy, N); cp_in(S->vz, vz, N);
  cp_in(S->ax, ax, N); cp_in(S->ay, ay, N); cp_in(S->az, az, N);
  if (api) memcpy(S->api + 1, api, sizeof(int) * (size_t)N);
  if (sc) S->sc = *sc;
}

void orc_get_state(orc_sys* S, double* x, double* y, double* z, double* vx, double* vy,
                   double* vz, double* ax, double* ay, double* az, clmd_scalars* sc) {
  int N = S->N;
  cp_out(x, S->x, N); cp_out(y, S->y, N); cp_out(z, S->z, N);
  cp_out(vx, S->vx, N); cp_out(vy, S->vy, N); cp_out(vz, S->vz, N);
  cp_out(ax, S->ax, N); cp_out(ay, S->ay, N); cp_out(az, S->az, N);
  if (sc) *sc = S->sc;
}

/* ------------------------------------------------------------------------ */
/* neighbor-pbc-mav.f:13-109                                                 */
/* ------------------------------------------------------------------------ */

/* the pair test of neighbor-pbc-mav.f:81-89 (wrapped positions) */
static inline int nb_pair(double tx, double ty, double tz, double xj, double yj, double zj,
                          double bx, double by, double bz, double ibx, double iby,
                          double ibz, double rs2) {
  double dx = tx - xj, dy = ty - yj, dz = tz - zj;
  dx = dx + bx - bx * (double)(int)(1.5 + dx * ibx);
  dy = dy + by - by * (double)(int)(1.5 + dy * iby);
  dz = dz + bz - bz * (double)(int)(1.5 + dz * ibz);
  double r2 = dx * dx + dy * dy + dz * dz;
  return r2 <= rs2;
}

static int cmp_int(const void* a, const void* b) {
  int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

/* Distinct neighbour-cell offsets along one axis with n cells. */
static int cell_offsets(int n, int* off) {
  if (n >= 3) { off[0] = -1; off[1] = 0; off[2] = 1; return 3; }
  if (n == 2) { off[0] = 0; off[1] = 1; return 2; }
  off[0] = 0;
  return 1;
}

/* Cells of side >= rs (with a relative margin far above rounding); a pair
 * that passes the reference's test is always in adjacent cells, and every
 * candidate is decided by the reference's own test, so the list equals the
 * all-pairs list once each row is sorted ascending. */
static int build_cells(orc_sys* S, double rs, int* ncv, int** start_o, int** atoms_o) {
  int N = S->N;
  double side = rs * (1.0 + 1e-9);
  int nx = (int)floor(S->c.boxx / side), ny = (int)floor(S->c.boxy / side),
      nz = (int)floor(S->c.boxz / side);
  if (nx < 1) nx = 1;
  if (ny < 1) ny = 1;
  if (nz < 1) nz = 1;
  ncv[0] = nx; ncv[1] = ny; ncv[2] = nz;
  int64_t nc = (int64_t)nx * ny * nz;
  int* cnt = xc((size_t)nc + 1, 4);
  int* cid = xc((size_t)N + 1, 4);
  for (int i = 1; i <= N; i++) {
    int cx = (int)(S->x[i] * ((double)nx / S->c.boxx));
    int cy = (int)(S->y[i] * ((double)ny / S->c.boxy));
    int cz = (int)(S->z[i] * ((double)nz / S->c.boxz));
    if (cx >= nx) cx = nx - 1;
    if (cy >= ny) cy = ny - 1;
    if (cz >= nz) cz = nz - 1;
    if (cx < 0) cx = 0;
    if (cy < 0) cy = 0;
    if (cz < 0) cz = 0;
    cid[i] = (cz * ny + cy) * nx + cx;
    cnt[cid[i] + 1]++;
  }
  for (int64_t c = 0; c < nc; c++) cnt[c + 1] += cnt[c];
  int* fill = xc((size_t)nc + 1, 4);
  memcpy(fill, cnt, sizeof(int) * (size_t)(nc + 1));
  int* atoms = xc((size_t)N + 1, 4);
  for (int i = 1; i <= N; i++) atoms[fill[cid[i]]++] = i;
  free(fill);
  free(cid);
  *start_o = cnt;
  *atoms_o = atoms;
  return 0;
}

int orc_neighbor(orc_sys* S, int32_t* step) {
  clmd_scalars* q = &S->sc;
  const clmd_config* c = &S->c;
  int N = S->N;
  if (q->status) return q->status;
  double ibx = 1.0 / c->boxx, iby = 1.0 / c->boxy, ibz = 1.0 / c->boxz;
  /* :48-51 */
  if (q->dmms > (q->atrskin - c->atrcut)) return latch(S, CLMD_ERR_SKIN, *step);
  /* :53 */
  q->dmmav = (double)(float)q->dmmst * q->dmmsu / 256.0;
  /* :55-60 */
  if (*step != c->btim && *step > 0) {
    q->atrskin = c->atrcut + (q->atrskin - c->atrcut) * (double)c->nbtim / (double)q->dmmst;
    q->atrskin = fmin(c->boxx / 2.0, q->atrskin);
    q->atrskin = fmin(c->boxy / 2.0, q->atrskin);
    q->atrskin = fmin(c->boxz / 2.0, q->atrskin);
  }
  /* :63 */
  if (*step < 0) *step = -*step;
  double rs2 = q->atrskin * q->atrskin;
  /* :67-71 */
  for (int i = 1; i <= N; i++) {
    S->x[i] = fmod(fmod(S->x[i], c->boxx) + c->boxx, c->boxx);
    S->y[i] = fmod(fmod(S->y[i], c->boxy) + c->boxy, c->boxy);
    S->z[i] = fmod(fmod(S->z[i], c->boxz) + c->boxz, c->boxz);
  }
  int64_t ind = 1;
  int overflow = 0;
  if (S->nbmode == 0) {
    /* :73-99 */
    for (int i = 1; i <= N; i++) {
      S->atnlist[ind] = -i;
      S->atnidx[i] = (int)ind;
      ind++;
      double tx = S->x[i], ty = S->y[i], tz = S->z[i];
      for (int j = i + 1; j <= N; j++) {
        if (nb_pair(tx, ty, tz, S->x[j], S->y[j], S->z[j], c->boxx, c->boxy, c->boxz, ibx,
                    iby, ibz, rs2)) {
          if (ind <= S->nl_cap) S->atnlist[ind] = j;
          ind++;
        }
      }
      if (ind + N > S->nl_cap) { overflow = 1; break; }
    }
  } else {
    int ncv[3], *start, *atoms;
    build_cells(S, q->atrskin, ncv, &start, &atoms);
    int ox[3], oy[3], oz[3];
    int nox = cell_offsets(ncv[0], ox), noy = cell_offsets(ncv[1], oy),
        noz = cell_offsets(ncv[2], oz);
    int* row = xc(1024, 4);
    int rowcap = 1024;
    for (int i = 1; i <= N && !overflow; i++) {
      S->atnlist[ind] = -i;
      S->atnidx[i] = (int)ind;
      ind++;
      double tx = S->x[i], ty = S->y[i], tz = S->z[i];
      int cx = (int)(tx * ((double)ncv[0] / c->boxx));
      int cy = (int)(ty * ((double)ncv[1] / c->boxy));
      int cz = (int)(tz * ((double)ncv[2] / c->boxz));
      if (cx >= ncv[0]) cx = ncv[0] - 1;
      if (cy >= ncv[1]) cy = ncv[1] - 1;
      if (cz >= ncv[2]) cz = ncv[2] - 1;
      int nrow = 0;
      for (int a = 0; a < noz; a++)
        for (int b = 0; b < noy; b++)
          for (int d = 0; d < nox; d++) {
            int zz = (cz + oz[a] + ncv[2]) % ncv[2];
            int yy = (cy + oy[b] + ncv[1]) % ncv[1];
            int xx = (cx + ox[d] + ncv[0]) % ncv[0];
            int cell = (zz * ncv[1] + yy) * ncv[0] + xx;
            for (int p = start[cell]; p < start[cell + 1]; p++) {
              int j = atoms[p];
              if (j <= i) continue;
              if (nb_pair(tx, ty, tz, S->x[j], S->y[j], S->z[j], c->boxx, c->boxy, c->boxz,
                          ibx, iby, ibz, rs2)) {
                if (nrow == rowcap) {
                  rowcap *= 2;
                  row = realloc(row, sizeof(int) * (size_t)rowcap);
                }
                row[nrow++] = j;
              }
            }
          }
      qsort(row, (size_t)nrow, sizeof(int), cmp_int);
      for (int k = 0; k < nrow; k++) {
        if (ind <= S->nl_cap) S->atnlist[ind] = row[k];
        ind++;
      }
      if (ind + N > S->nl_cap) overflow = 1;
    }
    free(row);
    free(start);
    free(atoms);
  }
  if (overflow) return latch(S, CLMD_ERR_LIST_OVERFLOW, *step);
  S->nl_used = ind - 1;
  q->npairs_half = ind - 1 - N;
  /* :101-105 */
  q->dmmax = fmax(q->dmms, q->dmmax);
  q->dmms = 0.0;
  q->dmmst = 0;
  q->nrebuild++;
  q->last_rebuild_step = *step;
  return CLMD_OK;
}

int64_t orc_neighbor_rows_sample(orc_sys* S, int32_t i0, int32_t i1) {
  const clmd_config* c = &S->c;
  int N = S->N;
  double ibx = 1.0 / c->boxx, iby = 1.0 / c->boxy, ibz = 1.0 / c->boxz;
  double rs2 = S->sc.atrskin * S->sc.atrskin;
  int64_t tested = 0, hits = 0;
  for (int i = i0 + 1; i <= i1 && i <= N; i++) {
    double tx = S->x[i], ty = S->y[i], tz = S->z[i];
    for (int j = i + 1; j <= N; j++) {
      hits += nb_pair(tx, ty, tz, S->x[j], S->y[j], S->z[j], c->boxx, c->boxy, c->boxz, ibx,
                      iby, ibz, rs2);
    }
    tested += N - i;
  }
  /* keep the loop from being optimised away */
  if (hits < 0) fprintf(stderr, "impossible\n");
  return tested;
}

int orc_get_halflist(orc_sys* S, int32_t* atnlist, int64_t cap, int32_t* atnidx,
                     int64_t* nentries) {
  if (nentries) *nentries = S->nl_used;
  if (atnlist) {
    int64_t n = S->nl_used < cap ? S->nl_used : cap;
    memcpy(atnlist, S->atnlist + 1, sizeof(int) * (size_t)n);
  }
  if (atnidx) memcpy(atnidx, S->atnidx + 1, sizeof(int) * (size_t)S->N);
  return CLMD_OK;
}

/* ------------------------------------------------------------------------ */
/* for-a-lj-n-pbc-m.f:18-154 (AccAtom); for-w-dummy.f:9-14 (AccWall)        */
/* ------------------------------------------------------------------------ */
int orc_accatom(orc_sys* S) {
  clmd_scalars* q = &S->sc;
  const clmd_config* c = &S->c;
  int N = S->N;
  if (q->status) return q->status;
  /* :61-79 */
  double atr2 = c->atrcut * c->atrcut;
  double s1 = c->apsig[0], s2 = c->apsig[1];
  double c111 = s1 * s1 * s1 * s1 * s1 * s1;
  double c112 = c111 * c111;
  double c113 = 0.5 * c111;
  double eps11 = c->apeps[0];
  double c221 = s2 * s2 * s2 * s2 * s2 * s2;
  double c222 = c221 * c221;
  double c223 = 0.5 * c221;
  double eps22 = c->apeps[1];
  double c121 = 0.5 * (s1 + s2);
  c121 = c121 * c121 * c121 * c121 * c121 * c121;
  double c122 = c121 * c121;
  double c123 = 0.5 * c121;
  double eps12 = sqrt(c->apeps[0] * c->apeps[1]);
  double bf1 = 2.0 + (double)(int)(q->atrskin / c->apsig[0]);
  double bf2 = bf1 + 0.5;
  double esum = 0.0, vir = 0.0;
  double ibx = 1.0 / c->boxx, iby = 1.0 / c->boxy, ibz = 1.0 / c->boxz;
  /* :86-90 */
  for (int i = 1; i <= N; i++) { S->fsx[i] = 0.0; S->fsy[i] = 0.0; S->fsz[i] = 0.0; }
  double fij = 0.0;
  /* :92-144 */
  int64_t k = 1;
  for (;;) {
    int i = -S->atnlist[k];
    if (i == N) break;
    k++;
    double tx = S->x[i], ty = S->y[i], tz = S->z[i];
    for (;;) {
      int j = S->atnlist[k];
      if (j <= 0) break;
      k++;
      double dx = tx - S->x[j], dy = ty - S->y[j], dz = tz - S->z[j];
      dx = dx + c->boxx * (bf1 - (double)(int)(bf2 + dx * ibx));
      dy = dy + c->boxy * (bf1 - (double)(int)(bf2 + dy * iby));
      dz = dz + c->boxz * (bf1 - (double)(int)(bf2 + dz * ibz));
      double rij2 = dx * dx + dy * dy + dz * dz;
      if (rij2 <= atr2) {
        double r2 = rij2;
        rij2 = 1.0 / rij2;
        double rij6 = rij2 * rij2 * rij2;
        int ij = S->api[i] + S->api[j];
        if (ij == 2) {
          fij = eps11 * 48.0 * rij2 * rij6 * (c112 * rij6 - c113);
          esum = esum + eps11 * 4.0 * rij6 * (c112 * rij6 - c111);
        } else if (ij == 4 && c->forcevar == 'r') { /* for-a-lj-n-pbc-mr.f:121-123 */
          fij = eps22 * 12.0 * c222 * rij2 * rij6 * rij6;
          esum = esum + eps22 * c222 * rij6 * rij6;
        } else if (ij == 3 && c->forcevar == 'r') { /* for-a-lj-n-pbc-mr.f:125-127 */
          fij = eps12 * 12.0 * c122 * rij2 * rij6 * rij6;
          esum = esum + eps12 * c122 * rij6 * rij6;
        } else if (ij == 4) {
          fij = eps22 * 48.0 * rij2 * rij6 * (c222 * rij6 - c223);
          esum = esum + eps22 * 4.0 * rij6 * (c222 * rij6 - c221);
        } else if (ij == 3) {
          fij = eps12 * 48.0 * rij2 * rij6 * (c122 * rij6 - c123);
          esum = esum + eps12 * 4.0 * rij6 * (c122 * rij6 - c121);
        } else {
          /* :129-130 prints and reuses the previous fij; the engine
           * reports the species error instead */
          latch(S, CLMD_ERR_BAD_SPECIES, q->cstep);
        }
        vir = vir + fij * r2;
        S->fsx[i] = S->fsx[i] + fij * dx;
        S->fsx[j] = S->fsx[j] - fij * dx;
        S->fsy[i] = S->fsy[i] + fij * dy;
        S->fsy[j] = S->fsy[j] - fij * dy;
        S->fsz[i] = S->fsz[i] + fij * dz;
        S->fsz[j] = S->fsz[j] - fij * dz;
      }
    }
  }
  /* :146-152 */
  q->epot = esum;
  q->virial = vir;
  for (int i = 1; i <= N; i++) {
    double iatm = 1.0 / c->apmas[S->api[i] - 1];
    S->ax[i] = S->ax[i] + S->fsx[i] * iatm;
    S->ay[i] = S->ay[i] + S->fsy[i] * iatm;
    S->az[i] = S->az[i] + S->fsz[i] * iatm;
  }
  return q->status;
}

int orc_zero_acc(orc_sys* S) {
  for (int i = 1; i <= S->N; i++) { S->ax[i] = 0.0; S->ay[i] = 0.0; S->az[i] = 0.0; }
  return CLMD_OK;
}

/* the skin bookkeeping shared by int-verlet-mav.f:64-74 and
 * int-verlet-nh-mav.f:70-78; returns 1 if the list must be rebuilt */
static int skin_update(orc_sys* S, double dmmr) {
  clmd_scalars* q = &S->sc;
  dmmr = 2.2 * sqrt(dmmr);
  q->dmms = q->dmms + dmmr;
  q->dmmsu = q->dmmsu + dmmr - q->dmmh[q->dmmi];
  q->dmmh[q->dmmi] = dmmr;
  q->dmmi = (q->dmmi + 1) & 255;
  q->dmmst = q->dmmst + 1;
  return q->dmms > (q->atrskin - S->c.atrcut - 2.0 * q->dmms / (double)(float)q->dmmst);
}

/* ------------------------------------------------------------------------ */
/* int-verlet-mav.f:18-95                                                     */
/* ------------------------------------------------------------------------ */
static int integrator_vv(orc_sys* S, int32_t step) {
  const clmd_config* c = &S->c;
  clmd_scalars* q = &S->sc;
  int N = S->N;
  double dt = c->dt;
  double dmmr = 0.0;
  /* :44-56 */
  for (int i = 1; i <= N; i++) {
    double dx = (S->vx[i] + 0.5 * S->ax[i] * dt) * dt;
    double dy = (S->vy[i] + 0.5 * S->ay[i] * dt) * dt;
    double dz = (S->vz[i] + 0.5 * S->az[i] * dt) * dt;
    S->x[i] = S->x[i] + dx;
    S->y[i] = S->y[i] + dy;
    S->z[i] = S->z[i] + dz;
    S->vx[i] = S->vx[i] + 0.5 * S->ax[i] * dt;
    S->vy[i] = S->vy[i] + 0.5 * S->ay[i] * dt;
    S->vz[i] = S->vz[i] + 0.5 * S->az[i] * dt;
    dmmr = fmax(dmmr, dx * dx + dy * dy + dz * dz);
  }
  /* :64-74 */
  if (skin_update(S, dmmr)) {
    int32_t st = step;
    if (orc_neighbor(S, &st)) return q->status;
  }
  /* :76-84 */
  q->epot = 0.0;
  orc_zero_acc(S);
  if (orc_accatom(S)) return q->status;
  /* :86-92 */
  q->ekin = 0.0;
  for (int i = 1; i <= N; i++) {
    S->vx[i] = S->vx[i] + 0.5 * S->ax[i] * dt;
    S->vy[i] = S->vy[i] + 0.5 * S->ay[i] * dt;
    S->vz[i] = S->vz[i] + 0.5 * S->az[i] * dt;
    q->ekin = q->ekin + 0.5 * c->apmas[S->api[i] - 1] *
                            (S->vx[i] * S->vx[i] + S->vy[i] * S->vy[i] + S->vz[i] * S->vz[i]);
  }
  return CLMD_OK;
}

/* ------------------------------------------------------------------------ */
/* int-verlet-nh-mav.f:13-204                                                 */
/* ------------------------------------------------------------------------ */
static int integrator_nh(orc_sys* S, int32_t step) {
  const clmd_config* c = &S->c;
  clmd_scalars* q = &S->sc;
  int N = S->N;
  double dt = c->dt, Q = c->Q, m = c->apmas[0], att = c->att;
  double dt2 = dt * dt / 2;
  double dth = dt / 2;
  double dmmr = 0.0;
  q->sumv2 = 0;
  /* :49-61 */
  for (int i = 1; i <= N; i++) {
    double dx = dt * S->vx[i] + dt2 * (S->ax[i] - q->psi * S->vx[i]);
    double dy = dt * S->vy[i] + dt2 * (S->ay[i] - q->psi * S->vy[i]);
    double dz = dt * S->vz[i] + dt2 * (S->az[i] - q->psi * S->vz[i]);
    S->x[i] = S->x[i] + dx;
    S->y[i] = S->y[i] + dy;
    S->z[i] = S->z[i] + dz;
    q->sumv2 = q->sumv2 + S->vx[i] * S->vx[i] + S->vy[i] * S->vy[i] + S->vz[i] * S->vz[i];
    S->vx[i] = S->vx[i] + dth * (S->ax[i] - q->psi * S->vx[i]);
    S->vy[i] = S->vy[i] + dth * (S->ay[i] - q->psi * S->vy[i]);
    S->vz[i] = S->vz[i] + dth * (S->az[i] - q->psi * S->vz[i]);
    dmmr = fmax(dmmr, dx * dx + dy * dy + dz * dz);
  }
  /* :64-67 */
  if (c->ethst == 'N') {
    q->s = q->s + q->psi * dt + (m * q->sumv2 - 3.0 * N * CLMD_CIKB * att) * dt2 / Q;
    q->psi = q->psi + (m * q->sumv2 - 3.0 * N * CLMD_CIKB * att) * dth / Q;
  }
  /* :70-78 */
  if (skin_update(S, dmmr)) {
    int32_t st = step;
    if (orc_neighbor(S, &st)) return q->status;
  }
  /* :81-88 */
  q->epot = 0.0;
  orc_zero_acc(S);
  if (orc_accatom(S)) return q->status;
  /* :91-103 */
  q->ekin = 0.0;
  double err = 1.0e-10;
  q->sumv2 = 0;
  for (int i = 1; i <= N; i++) {
    S->vxn[i] = S->vx[i];
    S->vyn[i] = S->vy[i];
    S->vzn[i] = S->vz[i];
    q->sumv2 = q->sumv2 + S->vxn[i] * S->vxn[i] + S->vyn[i] * S->vyn[i] + S->vzn[i] * S->vzn[i];
  }
  double psn = q->psi, pso = 0.0, delps, di;
  int ready = 0, iter;
  const double nkt3 = (double)(3 * N) * CLMD_CIKB * att; /* 3*natom*cikb*att, integer 3*natom */
  /* :106-147 */
  for (iter = 1; iter <= 1000; iter++) {
    pso = psn;
    delps = 0;
    for (int i = 1; i <= N; i++) {
      S->vxo[i] = S->vxn[i];
      S->vyo[i] = S->vyn[i];
      S->vzo[i] = S->vzn[i];
      S->bx[i] = -dth * (S->ax[i] - pso * S->vxo[i]) - (S->vx[i] - S->vxo[i]);
      delps = delps + S->bx[i] * m * S->vxo[i] * dt / Q;
      S->by[i] = -dth * (S->ay[i] - pso * S->vyo[i]) - (S->vy[i] - S->vyo[i]);
      delps = delps + S->by[i] * m * S->vyo[i] * dt / Q;
      S->bz[i] = -dth * (S->az[i] - pso * S->vzo[i]) - (S->vz[i] - S->vzo[i]);
      delps = delps + S->bz[i] * m * S->vzo[i] * dt / Q;
    }
    di = -(pso * dth + 1);
    delps = delps - di * ((-m * q->sumv2 + nkt3) * dth / Q - (q->psi - pso));
    delps = delps / (-dt2 * m * q->sumv2 / Q + di);
    q->sumv2 = 0;
    for (int i = 1; i <= N; i++) {
      S->vxn[i] = S->vxn[i] + (S->bx[i] + dth * S->vxo[i] * delps) / di;
      S->vyn[i] = S->vyn[i] + (S->by[i] + dth * S->vyo[i] * delps) / di;
      S->vzn[i] = S->vzn[i] + (S->bz[i] + dth * S->vzo[i] * delps) / di;
      q->sumv2 =
          q->sumv2 + S->vxn[i] * S->vxn[i] + S->vyn[i] * S->vyn[i] + S->vzn[i] * S->vzn[i];
    }
    psn = pso + delps;
    ready = 1;
    for (int i = 1; i <= N; i++) {
      /* ABS(x).GT.err is false for NaN, as in Fortran */
      if (fabs((S->vxn[i] - S->vxo[i]) / S->vxn[i]) > err) ready = 0;
      if (fabs((S->vyn[i] - S->vyo[i]) / S->vyn[i]) > err) ready = 0;
      if (fabs((S->vzn[i] - S->vzo[i]) / S->vzn[i]) > err) ready = 0;
    }
    if (ready) break;
  }
  q->nh_iters = ready ? iter : 1000;
  /* :150-166 */
  if (!ready) return latch(S, CLMD_ERR_NH_NOCONVERGE, step);
  /* :171-180 */
  q->sumv2 = 0;
  for (int i = 1; i <= N; i++) {
    S->vx[i] = S->vxn[i];
    S->vy[i] = S->vyn[i];
    S->vz[i] = S->vzn[i];
    q->sumv2 = q->sumv2 + S->vx[i] * S->vx[i] + S->vy[i] * S->vy[i] + S->vz[i] * S->vz[i];
  }
  q->psi = psn;
  q->ekin = 0.5 * m * q->sumv2;
  return CLMD_OK;
}

int orc_integrator(orc_sys* S, int32_t step) {
  if (S->sc.status) return S->sc.status;
  if (S->c.integrator == CLMD_INT_NOSE) return integrator_nh(S, step);
  return integrator_vv(S, step);
}

/* ------------------------------------------------------------------------ */
/* scalev-nh-m.f:19-81 (same arithmetic as scalev-m.f:15-70)                  */
/* ------------------------------------------------------------------------ */
int orc_thermostat(orc_sys* S, int32_t step) {
  const clmd_config* c = &S->c;
  clmd_scalars* q = &S->sc;
  if (q->status) return q->status;
  int n = 1;
  q->ekin = 0.0;
  for (int i = 1; i <= c->atsorts; i++) {
    double ekinT = 1.5 * CLMD_CIKB * c->att * c->apnum[i - 1];
    double ek = 0.0;
    for (int j = n; j <= n + c->apnum[i - 1] - 1; j++)
      ek = ek + 0.5 * c->apmas[i - 1] *
                    (S->vx[j] * S->vx[j] + S->vy[j] * S->vy[j] + S->vz[j] * S->vz[j]);
    q->ekin = q->ekin + ek;
    double kf = sqrt(ekinT / ek);
    if (c->apth[i - 1] == 'X' || step == -1) {
      for (int j = n; j <= n + c->apnum[i - 1] - 1; j++) {
        S->vx[j] = S->vx[j] * kf;
        S->vy[j] = S->vy[j] * kf;
        S->vz[j] = S->vz[j] * kf;
      }
      q->ekin = q->ekin - ek + ekinT;
    }
    n = n + c->apnum[i - 1];
  }
  return CLMD_OK;
}

/* scalev-clu.f:41-83: the biggest cluster and the rest scaled separately
 * every ecltim steps when eclth == 'X', else one factor from the current
 * ekin; ekin = ekinT afterwards */
int orc_thermostat_clu(orc_sys* S, int32_t step, char eclth, int32_t ecltim) {
  const clmd_config* c = &S->c;
  clmd_scalars* q = &S->sc;
  if (q->status) return q->status;
  const int N = S->N;
  const double cikb = CLMD_CIKB;
  double ekinT = 1.5 * cikb * c->att * N;
  if (eclth == 'X' && ecltim > 0 && step % ecltim == 0) {
    if (q->cstep != step) orc_stoddard(S, step);
    int cb = 0, ci = 0;
    for (int i = 1; i <= N; i++)
      if (cb < S->cs[i]) {
        cb = S->cs[i];
        ci = i;
      }
    double ekinG = 0.0;
    for (int i = 1; i <= N; i++)
      if (i != ci) ekinG = ekinG + S->cek[i];
    double kfG = sqrt(1.5 * cikb * c->att * (N - S->cs[ci]) / ekinG);
    double kfC = sqrt(1.5 * cikb * c->att * S->cs[ci] / S->cek[ci]);
    for (int i = 1; i <= N; i++) {
      double k = S->cl[i] == ci ? kfC : kfG;
      S->vx[i] = S->vx[i] * k;
      S->vy[i] = S->vy[i] * k;
      S->vz[i] = S->vz[i] * k;
    }
  } else if (eclth == 'X' && ecltim <= 0) {
    return CLMD_ERR_ARG;
  } else {
    double kfG = sqrt(ekinT / q->ekin);
    for (int i = 1; i <= N; i++) {
      S->vx[i] = S->vx[i] * kfG;
      S->vy[i] = S->vy[i] * kfG;
      S->vz[i] = S->vz[i] * kfG;
    }
  }
  q->ekin = ekinT;
  return CLMD_OK;
}

/* stopdead-m.f:10-78 */
int orc_stopdead(orc_sys* S, int32_t step) {
  const clmd_config* c = &S->c;
  clmd_scalars* q = &S->sc;
  int N = S->N;
  if (q->status) return q->status;
  for (int loop = 1; loop <= 10; loop++) {
    double vxs = 0.0, vys = 0.0, vzs = 0.0;
    for (int i = 1; i <= N; i++) {
      double mas = c->apmas[S->api[i] - 1];
      vxs = vxs + S->vx[i] * mas;
      vys = vys + S->vy[i] * mas;
      vzs = vzs + S->vz[i] * mas;
    }
    vxs = vxs / (double)N;
    vys = vys / (double)N;
    vzs = vzs / (double)N;
    q->ekin = 0.0;
    for (int i = 1; i <= N; i++) {
      double mas = c->apmas[S->api[i] - 1];
      double imas = 1.0 / mas;
      S->vx[i] = S->vx[i] - vxs * imas;
      S->vy[i] = S->vy[i] - vys * imas;
      S->vz[i] = S->vz[i] - vzs * imas;
      q->ekin = q->ekin + mas * (S->vx[i] * S->vx[i] + S->vy[i] * S->vy[i] + S->vz[i] * S->vz[i]);
    }
    q->ekin = 0.5 * q->ekin;
    orc_thermostat(S, step);
  }
  return CLMD_OK;
}

/* ------------------------------------------------------------------------ */
/* stoddard-pbc-n-m.f:11-158 (Stillinger) and stoddard-pbc-n-m-fre.f:11-261  */
/* ------------------------------------------------------------------------ */

/* Bond lists shared by both variants: stoddard-pbc-n-m.f:70-127. */
typedef struct {
  int *cvtnt, *cvtn, *cvti, *cvtii, *cvtl;
} bondlists;

static void bonds_build(orc_sys* S, int species_filter, bondlists* B) {
  const clmd_config* c = &S->c;
  int N = S->N;
  double rijc2 = c->atskin * c->atskin;
  double bf1 = (double)(int)(S->sc.atrskin / c->apsig[0]) + 2.0;
  double bf2 = bf1 + 0.5;
  double ibx = 1.0 / c->boxx, iby = 1.0 / c->boxy, ibz = 1.0 / c->boxz;
  size_t cap = (size_t)S->nl_used + (size_t)N + 4;
  B->cvtnt = xc(cap, 4);
  B->cvtn = xc(2 * cap, 4);
  B->cvti = xc((size_t)N + 2, 4);
  B->cvtii = xc((size_t)N + 2, 4);
  B->cvtl = xc((size_t)N + 2, 4);
  int ind = 1;
  for (int i = 1; i <= N; i++) {
    B->cvtnt[ind] = -i;
    ind++;
    if (i == N) continue;
    if (species_filter && S->api[i] != 1) continue;
    double tx = S->x[i], ty = S->y[i], tz = S->z[i];
    int k = S->atnidx[i];
    for (;;) {
      k = k + 1;
      int j = S->atnlist[k];
      /* stoddard-pbc-n-m.f:85-86: a species-2 neighbour ends the row,
       * as does the next header (j < 0) */
      if (j < 0) break;
      if (species_filter && S->api[j] != 1) break;
      double dx = tx - S->x[j], dy = ty - S->y[j], dz = tz - S->z[j];
      dx = dx + c->boxx * (bf1 - (double)(int)(bf2 + dx * ibx));
      dy = dy + c->boxy * (bf1 - (double)(int)(bf2 + dy * iby));
      dz = dz + c->boxz * (bf1 - (double)(int)(bf2 + dz * ibz));
      double rij2 = dx * dx + dy * dy + dz * dz;
      if (rij2 <= rijc2) {
        B->cvtnt[ind] = j;
        B->cvtl[i]++;
        B->cvtl[j]++;
        ind++;
      }
    }
  }
  B->cvtnt[ind] = -(N + 1);
  /* :106-113 */
  ind = 1;
  for (int i = 1; i <= N; i++) {
    B->cvti[i] = ind;
    B->cvtn[ind] = -i;
    ind = ind + B->cvtl[i] + 1;
    B->cvtii[i] = B->cvti[i];
  }
  B->cvtn[ind] = -(N + 1);
  /* :115-127 */
  ind = 1;
  for (;;) {
    int i = -B->cvtnt[ind];
    ind++;
    if (i == N) break;
    for (;;) {
      int j = B->cvtnt[ind];
      if (j < 0) break;
      ind++;
      B->cvtii[i]++;
      B->cvtii[j]++;
      B->cvtn[B->cvtii[j]] = i;
      B->cvtn[B->cvtii[i]] = j;
    }
  }
}

static void bonds_free(bondlists* B) {
  free(B->cvtnt); free(B->cvtn); free(B->cvti); free(B->cvtii); free(B->cvtl);
}

/* Union-find over the bond lists, restricted to atoms with keep[i] != 0
 * (NULL: all): lab[i] = the smallest atom number of i's component.  The
 * reference's sweeps (stoddard-pbc-n-m.f:129-150, -fre.f:171-225) give every
 * member of a component the counter value of the sweep that found its
 * smallest member first; label_mode 1 derives the same labels in O(bonds)
 * so the oracle can check systems too large for the O(N^2) rescans. */
static int uf_find(int* par, int x) {
  while (par[x] != x) {
    par[x] = par[par[x]];
    x = par[x];
  }
  return x;
}
static void components(orc_sys* S, const bondlists* B, const int* keep, int* lab) {
  int N = S->N;
  int* par = xc((size_t)N + 2, 4);
  for (int i = 1; i <= N; i++) par[i] = i;
  for (int i = 1; i <= N; i++) {
    if (keep && !keep[i]) continue;
    int ind = B->cvti[i] + 1;
    for (int k = ind; k <= ind + B->cvtl[i] - 1; k++) {
      int j = B->cvtn[k];
      if (keep && !keep[j]) continue;
      int a = uf_find(par, i), b = uf_find(par, j);
      if (a == b) continue;
      if (a < b) par[b] = a; else par[a] = b; /* the root stays the smallest */
    }
  }
  for (int i = 1; i <= N; i++) lab[i] = uf_find(par, i);
  free(par);
}

static inline double kin(orc_sys* S, int j) {
  return 0.5 * S->c.apmas[S->api[j] - 1] *
         (S->vx[j] * S->vx[j] + S->vy[j] * S->vy[j] + S->vz[j] * S->vz[j]);
}

static int stoddard_stillinger(orc_sys* S, int32_t step) {
  clmd_scalars* q = &S->sc;
  int N = S->N;
  q->cstep = step;
  /* :60-68 (csi(0), ceks(0) are never reset) */
  for (int i = 1; i <= N; i++) {
    S->cl[i] = 0; S->cc[i] = 0; S->cs[i] = 0; S->csi[i] = 0;
    S->cek[i] = 0; S->ceks[i] = 0;
  }
  bondlists B;
  bonds_build(S, 1, &B);
  /* :129-150 */
  int cnum = 0;
  if (S->lbmode == 1) {
    /* the same labels and sizes; cek() summed in atom order, not in the
     * sweep's visiting order (rounding only) */
    components(S, &B, NULL, S->cl);
    for (int i = 1; i <= N; i++) {
      S->cc[i] = 1;
      S->cs[S->cl[i]]++;
      S->cek[S->cl[i]] = S->cek[S->cl[i]] + kin(S, i);
    }
    cnum = N;
  } else {
    for (int k = 1; k <= N; k++) {
      cnum = cnum + 1;
      int j = k;
      if (S->cc[j] == 0) {
      visit:
        S->cl[j] = cnum;
        S->cc[j] = 1;
        S->cs[cnum] = S->cs[cnum] + 1;
        S->cek[cnum] = S->cek[cnum] + kin(S, j);
        {
          int ind = B.cvti[j] + 1;
          for (int i = ind; i <= ind + B.cvtl[j] - 1; i++) S->cl[B.cvtn[i]] = cnum;
        }
        for (j = k + 1; j <= N; j++)
          if (S->cc[j] == 0 && S->cl[j] == cnum) goto visit;
      }
    }
  }
  q->cnum = cnum;
  /* :152-155 */
  int maxcs = 0;
  for (int i = 1; i <= cnum; i++) {
    S->csi[S->cs[i]] = S->csi[S->cs[i]] + 1;
    S->ceks[S->cs[i]] = S->ceks[S->cs[i]] + S->cek[i];
    if (S->cs[i] > maxcs) maxcs = S->cs[i];
  }
  q->maxcs = maxcs;
  bonds_free(&B);
  return CLMD_OK;
}

static int stoddard_frenkel(orc_sys* S, int32_t step) {
  const clmd_config* c = &S->c;
  clmd_scalars* q = &S->sc;
  int N = S->N;
  q->cstep = step;
  /* :60-82 */
  for (int i = 1; i <= N; i++) {
    S->cl[i] = 0; S->cc[i] = 0; S->cs[i] = 0; S->csi[i] = 0; S->cek[i] = 0; S->ceks[i] = 0;
    S->clf[i] = 0; S->ccf[i] = 0; S->csf[i] = 0; S->csif[i] = 0; S->cekf[i] = 0;
    S->ceksf[i] = 0; S->cgs[i] = 0; S->cgsf[i] = 0; S->cgsa[i] = 0; S->cgsfa[i] = 0;
  }
  S->csif[0] = 0; S->cgsf[0] = 0; S->cgsfa[0] = 0; S->cekf[0] = 0.0; S->ceksf[0] = 0.0;
  bondlists B;
  bonds_build(S, 0, &B);
  /* :143-168 */
  int* liqmon = xc((size_t)N + 2, 4);
  int lind = 1, nliqmon = 0, cnum = 0;
  for (int k = 1; k <= N; k++) {
    if (S->api[k] == 1 && B.cvtl[k] >= c->atnenum) {
      int filter = 0;
      int ind = B.cvti[k] + 1;
      for (int i = ind; i <= ind + B.cvtl[k] - 1; i++)
        if (S->api[B.cvtn[i]] == 1) filter++;
      if (filter >= c->atnenum) {
        liqmon[lind] = k;
        nliqmon++;
        lind++;
      } else {
        S->cekf[0] = S->cekf[0] + kin(S, k);
      }
    }
  }
  if (S->lbmode == 1) {
    /* :171-195 and :198-225 by union-find.  Liquid components link liquid
     * atoms only (the sweep never visits a non-liquid atom, so it never
     * follows that atom's bonds); a liquid component's label is the rank
     * in liqmon of its smallest member; a non-liquid atom keeps the label
     * its last liquid neighbour wrote, i.e. the largest of their labels. */
    components(S, &B, NULL, S->cl);
    for (int i = 1; i <= N; i++) {
      S->cc[i] = 1;
      int r = S->cl[i];
      if (S->api[i] != 1) {
        S->cgs[r]++;
      } else {
        S->cs[r]++;
        S->cek[r] = S->cek[r] + kin(S, i);
      }
    }
    cnum = N;
    int* liq = xc((size_t)N + 2, 4);
    int* rank = xc((size_t)N + 2, 4);
    for (int k = 1; k <= nliqmon; k++) {
      liq[liqmon[k]] = 1;
      rank[liqmon[k]] = k;
    }
    int* lab = xc((size_t)N + 2, 4);
    components(S, &B, liq, lab);
    for (int k = 1; k <= nliqmon; k++) {
      int m = liqmon[k];
      int f = rank[lab[m]];
      S->clf[m] = f;
      S->ccf[m] = 1;
      S->csf[f]++;
      S->cekf[f] = S->cekf[f] + kin(S, m);
    }
    for (int i = 1; i <= N; i++) {
      if (liq[i]) continue;
      int ind = B.cvti[i] + 1, f = 0;
      for (int k = ind; k <= ind + B.cvtl[i] - 1; k++)
        if (liq[B.cvtn[k]] && S->clf[B.cvtn[k]] > f) f = S->clf[B.cvtn[k]];
      S->clf[i] = f;
    }
    free(lab);
    free(rank);
    free(liq);
    q->cnum = cnum;
    q->cnumf = nliqmon;
    goto tally;
  }
  /* :171-195 */
  for (int k = 1; k <= N; k++) {
    cnum = cnum + 1;
    int j = k;
    if (S->cc[j] == 0) {
    visit:
      S->cl[j] = cnum;
      S->cc[j] = 1;
      if (S->api[j] != 1) {
        S->cgs[cnum]++;
      } else {
        S->cs[cnum]++;
        S->cek[cnum] = S->cek[cnum] + kin(S, j);
      }
      {
        int ind = B.cvti[j] + 1;
        for (int i = ind; i <= ind + B.cvtl[j] - 1; i++) S->cl[B.cvtn[i]] = cnum;
      }
      for (j = k + 1; j <= N; j++)
        if (S->cc[j] == 0 && S->cl[j] == cnum) goto visit;
    }
  }
  /* :198-225 */
  int cnumf = 0;
  for (int k = 1; k <= nliqmon; k++) {
    cnumf = cnumf + 1;
    int j = k;
    int m = liqmon[j];
    if (S->ccf[m] == 0) {
    visitf:
      S->clf[m] = cnumf;
      S->ccf[m] = 1;
      if (S->api[m] == 1) {
        S->csf[cnumf]++;
        S->cekf[cnumf] = S->cekf[cnumf] + kin(S, m);
      } else {
        S->cgsf[cnumf]++;
      }
      {
        int ind = B.cvti[m] + 1;
        for (int i = ind; i <= ind + B.cvtl[m] - 1; i++) S->clf[B.cvtn[i]] = cnumf;
      }
      for (j = k + 1; j <= nliqmon; j++) {
        m = liqmon[j];
        if (S->ccf[m] == 0 && S->clf[m] == cnumf) goto visitf;
      }
    }
  }
  q->cnum = cnum;
  q->cnumf = cnumf;
tally:;
  /* :229-241 */
  cnumf = q->cnumf;
  int maxcs = 0;
  for (int i = 1; i <= cnum; i++) {
    if (S->cs[i] > q->cbiggest) q->cbiggest = S->cs[i];
    if (S->cs[i] > maxcs) maxcs = S->cs[i];
    S->csi[S->cs[i]]++;
    S->ceks[S->cs[i]] = S->ceks[S->cs[i]] + S->cek[i];
  }
  q->maxcs = maxcs;
  if (q->cbiggest >= q->clookfor) {
    for (int i = q->clookfor; i <= q->cbiggest; i++) S->cfpt[i] = step;
    q->clookfor++;
  }
  /* :243-258 */
  int catoms = 0;
  for (int i = 1; i <= cnumf; i++) {
    if (S->csf[i] > q->cbiggestf) q->cbiggestf = S->csf[i];
    S->csif[S->csf[i]]++;
    S->ceksf[S->csf[i]] = S->ceksf[S->csf[i]] + S->cekf[i];
    S->cgsfa[S->csf[i]] = S->cgsfa[S->csf[i]] + S->cgsf[i];
    catoms = catoms + S->csf[i];
  }
  S->csif[0] = c->apnum[0] - catoms;
  if (q->cbiggestf >= q->clookforf) {
    for (int i = q->clookforf; i <= q->cbiggestf; i++) S->cfptf[i] = step;
    q->clookforf++;
  }
  free(liqmon);
  bonds_free(&B);
  return CLMD_OK;
}

int orc_stoddard(orc_sys* S, int32_t step) {
  if (S->sc.status) return S->sc.status;
  if (S->c.clustering == CLMD_CLU_FRENKEL) return stoddard_frenkel(S, step);
  return stoddard_stillinger(S, step);
}

/* Fortran's Iw / Fw.d edit descriptors: right-justified, asterisks when
 * the value does not fit */
static void fput_i(FILE* f, long long v, int w) {
  char b[32];
  int n = snprintf(b, sizeof(b), "%lld", v);
  if (n > w) {
    for (int k = 0; k < w; k++) fputc('*', f);
  } else {
    fprintf(f, "%*s", w, b);
  }
}
static void fput_f(FILE* f, double v, int w, int d) {
  char b[64];
  int n = snprintf(b, sizeof(b), "%.*f", d, v);
  if (n > w || v != v) {
    for (int k = 0; k < w; k++) fputc('*', f);
  } else {
    fprintf(f, "%*s", w, b);
  }
}

/* rates.f:44-100: evaporation / condensation of the largest cluster between
 * the previous analysis and this step's.  out = unit 67, log = the
 * write(*,1) lines (NULL: stdout). */
int orc_rates(orc_sys* S, int32_t step, int32_t ctrat, const char* out, const char* log) {
  const int N = S->N;
  if (ctrat < 1) return CLMD_ERR_ARG;
  if (!S->ocs) {
    S->ocs = (int*)xc((size_t)N + 1, sizeof(int));
    S->ocl = (int*)xc((size_t)N + 1, sizeof(int));
    S->ocek = (double*)xc((size_t)N + 1, sizeof(double));
  }
  FILE* lg = log ? fopen(log, "a") : stdout;
  if (!lg) return CLMD_ERR_ARG;
  for (int i = 1; i <= N; i++) { /* :44-48 */
    S->ocs[i] = S->cs[i];
    S->ocl[i] = S->cl[i];
    S->ocek[i] = S->cek[i];
  }
  if (S->sc.cstep != step) { /* :50-54 */
    orc_stoddard(S, step);
  } else {
    fprintf(lg, " *** WARNING *** No old Stoddard-list !!\n");
  }
  int mcs = 0, omcs = 0, mcln = 0, omcln = 0;
  for (int i = 1; i <= N; i++) { /* :56-67 */
    if (S->ocs[i] > omcs) {
      omcs = S->ocs[i];
      omcln = i;
    }
    if (S->cs[i] > mcs) {
      mcs = S->cs[i];
      mcln = i;
    }
  }
  int cn = 0, en = 0;
  for (int i = 1; i <= N; i++) { /* :69-73 */
    if (S->cl[i] == mcln && S->ocl[i] != omcln) cn = cn + 1;
    if (S->cl[i] != mcln && S->ocl[i] == omcln) en = en + 1;
  }
  if (mcs != omcs) { /* :75-76 */
    fput_i(lg, step, 12);
    int v4[4] = {omcs, mcs, omcln, mcln};
    for (int k = 0; k < 4; k++) {
      fputs("  ", lg);
      fput_i(lg, v4[k], 5);
    }
    fputs("  ", lg);
    fput_i(lg, cn, 2);
    fputs("  ", lg);
    fput_i(lg, en, 2);
    fputc('\n', lg);
  }
  if (log) fclose(lg);
  const double cikb = CLMD_CIKB;
  double mct = S->cek[mcln] / ((double)mcs * 1.5 * cikb); /* :78-81 */
  S->mcts = S->mcts + mct;
  double omct = S->ocek[omcln] / ((double)omcs * 1.5 * cikb);
  S->omcts = S->omcts + omct;
  S->cen = S->cen + en; /* :83-84 */
  S->ccn = S->ccn + cn;
  int write = 0;
  double c4 = mct, c5 = omct;
  int c6 = cn, c7 = en;
  if (ctrat != 1) { /* :85-98 */
    if (step % ctrat == 0) {
      write = 1;
      c4 = S->mcts / (double)(float)ctrat;
      c5 = S->omcts / (double)(float)ctrat;
      c6 = S->ccn;
      c7 = S->cen;
      S->ccn = 0;
      S->cen = 0;
      S->mcts = 0.0;
    }
  } else if ((en + cn) != 0) {
    write = 1;
  }
  if (write && out) { /* format 10 */
    FILE* f = fopen(out, "a");
    if (!f) return CLMD_ERR_ARG;
    fput_i(f, step, 12);
    fputc(' ', f); fput_i(f, omcs, 6);
    fputc(' ', f); fput_i(f, mcs, 6);
    fputc(' ', f); fput_f(f, c4, 10, 4);
    fputc(' ', f); fput_f(f, c5, 10, 4);
    fputc(' ', f); fput_i(f, c6, 3);
    fputc(' ', f); fput_i(f, c7, 3);
    fputc(' ', f); fput_i(f, mcln, 6);
    fputc(' ', f); fput_i(f, omcln, 6);
    fputc('\n', f);
    fclose(f);
  }
  return S->sc.status;
}

/* chk-nucleation.f:15-58 */
int orc_chk_nucleation(orc_sys* S, int32_t* step) {
  clmd_scalars* q = &S->sc;
  int N = S->N;
  int tim = 0;
  for (int i = S->c.csover; i <= N; i++) {
    if (i >= 0 && S->csi[i] > 0) {
      tim = *step;
      break;
    }
  }
  if (tim > 0) {
    if (q->clbrkt == 0) {
      q->clbrkt = tim;
    } else if ((tim - q->clbrkt) >= S->c.clwait) {
      *step = -*step;
      q->aborted = 1;
    }
  } else {
    q->clbrkt = 0;
  }
  return CLMD_OK;
}

/* main.f:177-228 with the writers off: wrtCSI's stoddard call every ftcsi
 * steps (wrt-csi.f:27), thermostat if ethst=='X', chk_nucleation every ftcsi
 * steps if clnuctrl=='X', then integrator. */
int orc_run(orc_sys* S, int32_t first, int32_t nsteps, int32_t* next_step) {
  const clmd_config* c = &S->c;
  int32_t i = first;
  for (int32_t n = 0; n < nsteps; n++) {
    if (c->ftcsi != 0 && i % c->ftcsi == 0 && S->sc.cstep != i) orc_stoddard(S, i);
    if (c->ethst == 'X') orc_thermostat(S, i);
    if (c->clnuctrl == 'X' && c->ftcsi != 0 && i % c->ftcsi == 0) {
      orc_chk_nucleation(S, &i);
      if (i < 0) break;
    }
    orc_integrator(S, i);
    if (S->sc.status) break;
    i = i + 1;
  }
  if (next_step) *next_step = i;
  return S->sc.status;
}

int orc_get_clusters(orc_sys* S, const clmd_cluster_view* v) {
  int N = S->N;
#define OUT1(f, T) \
  if (v->f) memcpy(v->f, S->f + 1, sizeof(T) * (size_t)N)
#define OUT0(f, T) \
  if (v->f) memcpy(v->f, S->f, sizeof(T) * (size_t)(N + 1))
  OUT1(cl, int); OUT1(cs, int); OUT0(csi, int); OUT1(cek, double); OUT0(ceks, double);
  OUT1(clf, int); OUT0(csf, int); OUT0(csif, int); OUT0(cekf, double); OUT0(ceksf, double);
  OUT1(cgs, int); OUT1(cgsa, int); OUT0(cgsf, int); OUT0(cgsfa, int);
  OUT1(cfpt, int); OUT1(cfptf, int);
#undef OUT1
#undef OUT0
  return CLMD_OK;
}

/* ------------------------------------------------------------------------ */
/* read-3d.f:11-302: the .3d deck                                             */
/* ------------------------------------------------------------------------ */
typedef struct {
  FILE* f;
  char line[512];
  int ok;
} deck;

static int dk_next(deck* d) {
  if (!d->ok) return 0;
  if (!fgets(d->line, sizeof d->line, d->f)) {
    d->ok = 0;
    d->line[0] = 0;
    return 0;
  }
  size_t n = strlen(d->line);
  while (n && (d->line[n - 1] == '\n' || d->line[n - 1] == '\r')) d->line[--n] = 0;
  return 1;
}
/* the field of width w starting after skip columns, blanks removed (BN) */
static void dk_field(deck* d, int skip, int w, char* out) {
  int n = (int)strlen(d->line), k = 0;
  for (int i = skip; i < skip + w && i < n; i++)
    if (d->line[i] != ' ' && d->line[i] != '\t') out[k++] = d->line[i];
  out[k] = 0;
}
/* What gfortran's formatted input accepts (blanks already dropped, BN):
 * Iw an optional sign and digits; Fw.d an optional sign, digits with at
 * most one point, and an exponent (a letter E/D/Q with an optional sign, or
 * a bare sign) followed by digits.  Anything else stops the reference's
 * read with a runtime error ("Bad value during ... read"). */
static int dk_int_ok(const char* b) {
  if (*b == '+' || *b == '-') b++;
  for (; *b; b++)
    if (*b < '0' || *b > '9') return 0;
  return 1;
}
/* Fw.d of a blank-free field b: 1 and *v on success, 0 where gfortran
 * stops the read.  Without a decimal point the rightmost d digits of the
 * mantissa are the fraction (an exponent, if any, scales the result); the
 * digits are handed to strtod as one decimal string, as gfortran does, so
 * the value is the correctly rounded one. */
static int dk_real(const char* b, int d, double* v) {
  char m[160];
  int k = 0, nd = 0, point = -1;
  if (*b == '+' || *b == '-') m[k++] = *b++;
  const int m0 = k;
  for (; (*b >= '0' && *b <= '9') || *b == '.'; b++) {
    if (*b == '.') {
      if (point >= 0) return 0;
      point = nd;
      continue;
    }
    if (k > 120) return 0;
    m[k++] = *b;
    nd++;
  }
  if (!nd) return 0;
  long e = 0;
  if (*b) {
    if (strchr("eEdDqQ", *b)) b++;
    else if (*b != '+' && *b != '-') return 0;
    int neg = *b == '-';
    if (*b == '+' || *b == '-') b++;
    if (!*b) return 0;
    for (; *b; b++) {
      if (*b < '0' || *b > '9') return 0;
      if (e < 100000) e = 10 * e + (*b - '0');
    }
    if (neg) e = -e;
  }
  if (point < 0) point = nd - d;  /* the implied point */
  /* digits d1..dn with the point after `point` digits: 0.d1..dn x 10^point */
  char out[200];
  int o = 0;
  if (m0) out[o++] = m[0];
  out[o++] = '0';
  out[o++] = '.';
  for (int i = m0; i < k; i++) out[o++] = m[i];
  o += snprintf(out + o, sizeof out - o, "e%ld", e + point);
  *v = strtod(out, NULL);
  return 1;
}

/* Fw.d input (see dk_real) */
static double dk_f(deck* d, int skip, int w, int dd) {
  char b[128];
  dk_next(d);
  dk_field(d, skip, w, b);
  if (!b[0]) return 0.0;
  double v = 0.0;
  if (!dk_real(b, dd, &v)) d->ok = 0;
  return v;
}
static int dk_i(deck* d, int skip) {
  char b[128];
  dk_next(d);
  dk_field(d, skip, 10, b);
  if (!dk_int_ok(b)) {
    d->ok = 0;
    return 0;
  }
  return b[0] ? (int)strtol(b, NULL, 10) : 0;
}
static char dk_a1(deck* d) {
  dk_next(d);
  return (int)strlen(d->line) > 41 ? d->line[41] : ' ';
}
static void dk_skip(deck* d) { dk_next(d); }

int orc_readdata(const char* path, clmd_config* cfg, int32_t* ntim, int32_t* sctim) {
  deck d = {fopen(path, "r"), {0}, 1};
  if (!d.f) return 1;
  memset(cfg, 0, sizeof(*cfg));
  int atsorts = 0, ftcsi;
  dk_skip(&d);
  float fver = (float)dk_f(&d, 41, 8, 6);
  if (fver < 1.02f) { fclose(d.f); return 2; }
  dk_skip(&d);
  dk_skip(&d);                  /* fpath */
  dk_skip(&d); dk_skip(&d);     /* fxyz, ftxyz */
  dk_skip(&d); dk_skip(&d);     /* fvel */
  dk_skip(&d); dk_skip(&d);     /* facc */
  dk_skip(&d); dk_skip(&d);     /* frst */
  dk_skip(&d);                  /* fcsi */
  ftcsi = dk_i(&d, 41);
  dk_skip(&d); dk_skip(&d);     /* fave */
  if (fver >= 1.06f) { dk_skip(&d); dk_skip(&d); }
  dk_skip(&d);
  cfg->dt = dk_f(&d, 41, 14, 5);
  int nt = dk_i(&d, 40);
  cfg->btim = dk_i(&d, 41);
  int sc = dk_i(&d, 41);
  dk_skip(&d);
  cfg->boxx = dk_f(&d, 41, 14, 5);
  cfg->boxy = dk_f(&d, 41, 14, 5);
  cfg->boxz = dk_f(&d, 41, 14, 5);
  if (fver >= 1.08f) { dk_skip(&d); dk_skip(&d); dk_skip(&d); }
  dk_skip(&d); dk_skip(&d); dk_skip(&d); /* bpot, beng, bcor */
  if (fver >= 1.05f) for (int i = 0; i < 8; i++) dk_skip(&d);
  cfg->boxx *= 10; cfg->boxy *= 10; cfg->boxz *= 10;
  dk_skip(&d);
  if (fver < 1.10f) atsorts = dk_i(&d, 41);
  dk_skip(&d); dk_skip(&d);      /* frctrl, finp */
  cfg->ethst = dk_a1(&d);
  double Qin = 0.0;
  if (fver >= 1.2f) Qin = dk_f(&d, 41, 14, 5);
  dk_skip(&d);                   /* rndctrl */
  if (fver >= 1.07f) { dk_skip(&d); dk_skip(&d); }
  double atr_rel = 0, atrcut_rel = 0, atrskin_rel = 0, atskin_rel = 0;
  if (fver >= 1.10f) {
    dk_skip(&d);
    cfg->att = dk_f(&d, 41, 14, 5);
    atskin_rel = dk_f(&d, 41, 14, 5);
    if (fver >= 1.30f) cfg->atnenum = dk_i(&d, 41);
    atrcut_rel = dk_f(&d, 41, 14, 5);
    atrskin_rel = dk_f(&d, 41, 14, 5);
    cfg->nbtim = dk_i(&d, 41);
    if (fver >= 1.11f) dk_skip(&d);
    if (fver >= 1.12f) {
      dk_skip(&d);
      cfg->clnuctrl = dk_a1(&d);
      cfg->csover = dk_i(&d, 41);
      cfg->clwait = dk_i(&d, 41);
    }
    dk_skip(&d);
    atsorts = dk_i(&d, 41);
  }
  dk_skip(&d);
  if (fver < 1.10f) {
    dk_skip(&d);
    cfg->apnum[0] = dk_i(&d, 41);
    cfg->apmas[0] = dk_f(&d, 41, 14, 5) * CLMD_CIMU;
    cfg->apsig[0] = dk_f(&d, 41, 14, 5) * 10.0;
    cfg->apeps[0] = dk_f(&d, 41, 14, 5) * CLMD_CIKB;
    dk_skip(&d); dk_skip(&d);
    cfg->att = dk_f(&d, 41, 14, 5);
    atskin_rel = dk_f(&d, 41, 14, 5);
    atrcut_rel = dk_f(&d, 41, 14, 5);
    atrskin_rel = dk_f(&d, 41, 14, 5);
    cfg->nbtim = dk_i(&d, 41);
    cfg->natom = cfg->apnum[0];
    atsorts = atsorts ? atsorts : 1;
  } else {
    int natom = 1;
    for (int i = 0; i < atsorts && i < CLMD_MXSORTS; i++) {
      dk_skip(&d); /* apsym */
      cfg->apnum[i] = dk_i(&d, 41);
      cfg->apmas[i] = dk_f(&d, 41, 14, 5);
      cfg->apsig[i] = dk_f(&d, 41, 14, 5);
      cfg->apeps[i] = dk_f(&d, 41, 14, 5);
      dk_skip(&d); dk_skip(&d); /* appr, appa */
      cfg->apth[i] = dk_a1(&d);
      if (fver >= 1.11f) { dk_skip(&d); dk_skip(&d); }
      dk_skip(&d);
      cfg->apmas[i] = cfg->apmas[i] * CLMD_CIMU;
      cfg->apsig[i] = cfg->apsig[i] * 10.0;
      cfg->apeps[i] = cfg->apeps[i] * CLMD_CIKB;
      natom += cfg->apnum[i];
    }
    Qin = Qin * cfg->apmas[0] * cfg->apsig[0] * cfg->apsig[0];
    cfg->natom = natom - 1;
  }
  atr_rel = cfg->apsig[0];
  cfg->Q = Qin;
  cfg->atsorts = atsorts;
  cfg->atskin = atskin_rel * atr_rel;
  cfg->atrcut = atrcut_rel * atr_rel;
  cfg->atrskin = atrskin_rel * atr_rel;
  cfg->ftcsi = ftcsi;
  if (ntim) *ntim = nt;
  if (sctim) *sctim = sc;
  fclose(d.f);
  return d.ok ? 0 : 3;
}

/* ------------------------------------------------------------------------ */
/* The engine's seeded start configuration, restated so that the CPU        */
/* baseline can build its inputs without loading the engine library: the    */
/* same xoshiro256** stream (seeded by splitmix64), the same rejection of    */
/* pairs nearer than rmin on a cell grid, the same Box-Muller velocities.    */
/* It must give the engine's clmd_init_random() bytes exactly (tested).      */
/* ------------------------------------------------------------------------ */
typedef struct {
  uint64_t s[4];
} orc_rng;

static uint64_t orc_splitmix(uint64_t* x) {
  uint64_t z = (*x += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
static uint64_t orc_rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t orc_next(orc_rng* r) {
  uint64_t* s = r->s;
  uint64_t res = orc_rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = orc_rotl(s[3], 45);
  return res;
}
static double orc_uniform(orc_rng* r) {
  return (double)(orc_next(r) >> 11) * (1.0 / 9007199254740992.0);
}
static double orc_gauss(orc_rng* r) {
  double u1 = orc_uniform(r), u2 = orc_uniform(r);
  if (u1 < 1e-300) u1 = 1e-300;
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

int orc_init_random(int32_t n, double bx, double by, double bz, double rmin, double kT_over_m,
                    uint64_t seed, double* x, double* y, double* z, double* vx, double* vy,
                    double* vz) {
  if (n < 1 || !(bx > 0 && by > 0 && bz > 0) || rmin < 0 || !x || !y || !z)
    return CLMD_ERR_ARG;
  orc_rng rng;
  for (int i = 0; i < 4; i++) rng.s[i] = orc_splitmix(&seed);
  double vol = bx * by * bz;
  double side = cbrt(vol / n);
  if (side < rmin) side = rmin;
  int nx = (int)(bx / side), ny = (int)(by / side), nz = (int)(bz / side);
  if (nx < 1) nx = 1;
  if (ny < 1) ny = 1;
  if (nz < 1) nz = 1;
  int* head = xc((size_t)nx * ny * nz, 4);
  int* next = xc((size_t)n, 4);
  for (size_t k = 0; k < (size_t)nx * ny * nz; k++) head[k] = -1;
  for (int i = 0; i < n; i++) next[i] = -1;
  double r2 = rmin * rmin;
  int rc = CLMD_OK;
  for (int i = 0; i < n && rc == CLMD_OK; i++) {
    int tries = 0;
    for (;;) {
      if (++tries > 100000) {
        rc = CLMD_ERR_ARG;
        break;
      }
      double px = orc_uniform(&rng) * bx, py = orc_uniform(&rng) * by,
             pz = orc_uniform(&rng) * bz;
      int c0 = (int)(px / bx * nx), c1 = (int)(py / by * ny), c2 = (int)(pz / bz * nz);
      if (c0 > nx - 1) c0 = nx - 1;
      if (c1 > ny - 1) c1 = ny - 1;
      if (c2 > nz - 1) c2 = nz - 1;
      int ok = 1;
      for (int a = -1; a <= 1 && ok; a++)
        for (int b = -1; b <= 1 && ok; b++)
          for (int d = -1; d <= 1 && ok; d++) {
            int xx = (c0 + d + nx) % nx, yy = (c1 + b + ny) % ny, zz = (c2 + a + nz) % nz;
            for (int j = head[((size_t)zz * ny + yy) * nx + xx]; j >= 0; j = next[j]) {
              double dx = px - x[j], dy = py - y[j], dz = pz - z[j];
              dx -= bx * nearbyint(dx / bx);
              dy -= by * nearbyint(dy / by);
              dz -= bz * nearbyint(dz / bz);
              if (dx * dx + dy * dy + dz * dz < r2) {
                ok = 0;
                break;
              }
            }
          }
      if (!ok) continue;
      x[i] = px;
      y[i] = py;
      z[i] = pz;
      size_t k = ((size_t)c2 * ny + c1) * nx + c0;
      next[i] = head[k];
      head[k] = i;
      break;
    }
  }
  free(head);
  free(next);
  if (rc) return rc;
  double sd = sqrt(kT_over_m > 0 ? kT_over_m : 0.0);
  for (int i = 0; i < n; i++) {
    double a = orc_gauss(&rng), b = orc_gauss(&rng), c = orc_gauss(&rng);
    if (vx) vx[i] = sd * a;
    if (vy) vy[i] = sd * b;
    if (vz) vz[i] = sd * c;
  }
  return CLMD_OK;
}

/* ------------------------------------------------------------------------ */
/* helpers/passage-time.f:47-90 on one run's analysis record: ts[k] the     */
/* step and cs[k] the largest cluster size of analysis k (the columns the   */
/* reference reads from its sizer file).  pt[j] (j = 0..endsize) receives   */
/* the first step at which the largest cluster reached size j for j >=     */
/* startsize (-1 where it never did; the lines the reference writes to its  */
/* dump), probab[j] the reference's probab.largest counts: analyses at or   */
/* after `warmup` with largest size j, up to and including the one that     */
/* first reached endsize.  Returns the next size not reached (the           */
/* reference's i at :77).                                                   */
/* ------------------------------------------------------------------------ */
int orc_passage_time(const int32_t* ts, const int32_t* cs, int32_t nlines, int32_t startsize,
                     int32_t endsize, int32_t warmup, int32_t* pt, int32_t* probab) {
  for (int j = 0; j <= endsize; j++) {
    if (pt) pt[j] = -1;
    if (probab) probab[j] = 0;
  }
  int i = startsize, flag = -1;
  for (int k = 0; k < nlines; k++) {
    const int t = ts[k], c = cs[k];
    /* :62-65 */
    if (flag != 1) {
      if (c >= endsize) flag = 1;
      if (t >= warmup && probab && c >= 0 && c <= endsize) probab[c] = probab[c] + 1;
    }
    /* :67-72 */
    if (c >= i) {
      for (int j = i; j <= c; j++)
        if (pt && j <= endsize) pt[j] = t;
      i = c + 1;
    }
  }
  return i;
}

/* helpers/mpt.f:52-110 over the pooled dump lines of many runs (size cs[k]
 * first reached at step ts[k]): for every size i in startsize..endsize,
 * mpt[i - startsize] = mean of ts/500000 (the reference's nanoseconds at a
 * 2 fs step, :80), stda = sqrt((mean of squares - mean^2) / count) (:95-97)
 * and count.  A size no run reached gives 0/0 as in the reference (NaN). */
int orc_mpt(const int32_t* ts, const int32_t* cs, int32_t nlines, int32_t startsize,
            int32_t endsize, double* mpt, double* stda, int32_t* count) {
  if (startsize < 1 || endsize > 4096 || endsize < startsize) return CLMD_ERR_ARG;
  double pt[4097], ptsq[4097];
  int cnt[4097];
  for (int i = 0; i <= 4096; i++) {
    pt[i] = 0.0;
    ptsq[i] = 0.0;
    cnt[i] = 0;
  }
  for (int k = 0; k < nlines; k++) {
    const int c = cs[k];
    if (c < 1 || c > 4096) continue;
    pt[c] = pt[c] + (double)ts[k] / 500000;
    ptsq[c] = ptsq[c] + ((double)ts[k] / 500000) * ((double)ts[k] / 500000);
    cnt[c] = cnt[c] + 1;
  }
  for (int i = startsize; i <= endsize; i++) {
    const double m = pt[i] / cnt[i];
    double sd = ptsq[i] / cnt[i] - m * m;
    sd = sqrt(sd / cnt[i]);
    mpt[i - startsize] = m;
    stda[i - startsize] = sd;
    count[i - startsize] = cnt[i];
  }
  return CLMD_OK;
}
