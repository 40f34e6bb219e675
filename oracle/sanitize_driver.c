/*
 * sanitize_driver.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Runs every oracle routine once or more on a small seeded system so that
 * tests/test_oracle_sanitizers.py can build the oracle with AddressSanitizer
 * and UndefinedBehaviorSanitizer (-fno-sanitize-recover) and check that no
 * routine reads or writes out of bounds or hits undefined behaviour: the
 * deck reader (read-3d.f), both neighbour modes, forces, both integrators,
 * the thermostats, stopdead, both cluster criteria, chk_nucleation, rates,
 * the main loop and the list / cluster exports.
 *
 * usage: sanitize_driver <deck.3d>
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "clmd_oracle.h"

static unsigned long long rng = 88172645463325252ull;
static double urand(void) {
  rng ^= rng << 13;
  rng ^= rng >> 7;
  rng ^= rng << 17;
  return (double)(rng >> 11) * (1.0 / 9007199254740992.0);
}

/* jittered cubic lattice: no pair closer than half a lattice spacing */
static void lattice(int n, double L, double* x, double* y, double* z) {
  int m = (int)ceil(cbrt((double)n));
  double a = L / m;
  for (int i = 0; i < n; i++) {
    int ix = i % m, iy = (i / m) % m, iz = i / (m * m);
    x[i] = (ix + 0.5 + 0.25 * (urand() - 0.5)) * a;
    y[i] = (iy + 0.5 + 0.25 * (urand() - 0.5)) * a;
    z[i] = (iz + 0.5 + 0.25 * (urand() - 0.5)) * a;
  }
}

static int run(clmd_config c, int mode, int integrator, int clustering, char forcevar) {
  const int n = c.natom;
  c.integrator = integrator;
  c.clustering = clustering;
  c.forcevar = forcevar;
  c.ethst = integrator == CLMD_INT_NOSE ? 'N' : '-';
  c.ftcsi = 20;
  c.csover = 8;
  c.clwait = 40;
  c.clnuctrl = 'X';
  c.atnenum = 3;
  double* b = calloc((size_t)9 * n, sizeof(double));
  double *x = b, *y = b + n, *z = b + 2 * n, *vx = b + 3 * n, *vy = b + 4 * n, *vz = b + 5 * n;
  lattice(n, c.boxx, x, y, z);
  double kt = CLMD_CIKB * c.att / c.apmas[0];
  for (int i = 0; i < n; i++) {
    vx[i] = sqrt(kt) * (urand() - 0.5) * 3.4;
    vy[i] = sqrt(kt) * (urand() - 0.5) * 3.4;
    vz[i] = sqrt(kt) * (urand() - 0.5) * 3.4;
  }
  orc_sys* S = orc_create(&c);
  orc_set_neighbor_mode(S, mode);
  clmd_scalars sc;
  orc_scalars_init(&c, &sc);
  orc_set_state(S, x, y, z, vx, vy, vz, b + 6 * n, b + 7 * n, b + 8 * n, NULL, &sc);
  int st = orc_stopdead(S, -1);
  int32_t step = 0;
  st |= orc_neighbor(S, &step);
  st |= orc_zero_acc(S);
  st |= orc_accatom(S);
  st |= orc_stoddard(S, -1);
  for (int k = 1; k <= 30; k++) {
    st |= orc_rates(S, k, 10, "/dev/null", "/dev/null");
    st |= orc_thermostat(S, k);
    st |= orc_integrator(S, k);
  }
  st |= orc_thermostat_clu(S, 40, 'X', 20);
  st |= orc_thermostat_clu(S, 41, 'X', 20);
  int32_t next = 0;
  st |= orc_run(S, 31, 60, &next);
  int32_t s2 = next;
  orc_chk_nucleation(S, &s2);
  int64_t used = 0;
  int64_t cap = (int64_t)n * 200 + 2 * n + 1;
  int32_t* list = malloc(sizeof(int32_t) * (size_t)cap);
  int32_t* idx = malloc(sizeof(int32_t) * (size_t)n);
  st |= orc_get_halflist(S, list, cap, idx, &used);
  clmd_cluster_view v;
  memset(&v, 0, sizeof(v));
  int32_t* ib = calloc((size_t)16 * (n + 1), sizeof(int32_t));
  double* db = calloc((size_t)6 * (n + 1), sizeof(double));
  v.cl = ib; v.cs = ib + (n + 1); v.csi = ib + 2 * (n + 1); v.clf = ib + 3 * (n + 1);
  v.csf = ib + 4 * (n + 1); v.csif = ib + 5 * (n + 1); v.cgs = ib + 6 * (n + 1);
  v.cgsa = ib + 7 * (n + 1); v.cgsf = ib + 8 * (n + 1); v.cgsfa = ib + 9 * (n + 1);
  v.cfpt = ib + 10 * (n + 1); v.cfptf = ib + 11 * (n + 1);
  v.cek = db; v.ceks = db + (n + 1); v.cekf = db + 2 * (n + 1); v.ceksf = db + 3 * (n + 1);
  st |= orc_get_clusters(S, &v);
  orc_get_state(S, x, y, z, vx, vy, vz, b + 6 * n, b + 7 * n, b + 8 * n, &sc);
  printf("mode %d int %d clu %d var %c: status %d, step %d, pairs %lld\n", mode, integrator,
         clustering, forcevar ? forcevar : '-', st, next, (long long)used);
  orc_destroy(S);
  free(b);
  free(list);
  free(idx);
  free(ib);
  free(db);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  clmd_config c;
  int32_t ntim = 0, sctim = 0;
  if (orc_readdata(argv[1], &c, &ntim, &sctim)) {
    fprintf(stderr, "cannot read %s\n", argv[1]);
    return 2;
  }
  /* a denser, smaller box than the deck's, keeping its species and units */
  const int n = c.natom;
  const double L = cbrt((double)n / 0.1) * c.apsig[0];
  c.boxx = c.boxy = c.boxz = L;
  c.nlist_cap = (int64_t)n * 200 + 2 * n + 1;
  for (int mode = 0; mode < 2; mode++)
    for (int integ = 0; integ < 2; integ++)
      for (int clu = 0; clu < 2; clu++) run(c, mode, integ, clu, integ ? 'r' : '-');
  return 0;
}
