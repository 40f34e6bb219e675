// clmd_host.cpp -- host-side helpers of the engine: status strings and the
// seeded synthetic start configuration.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/clmd.h"

extern "C" const char* clmd_status_string(int s) {
  switch (s) {
    case CLMD_OK: return "ok";
    case CLMD_ERR_SKIN: return "*** FATAL ERROR! ***  Skin radius exceeded!!";
    case CLMD_ERR_LIST_OVERFLOW: return "*** FATAL ERROR *** Neighborlist is nearly full!";
    case CLMD_ERR_NH_NOCONVERGE: return "Numerical integration did not converge!";
    case CLMD_ERR_BAD_SPECIES: return "Nanu??? (species pair without LJ parameters)";
    case CLMD_ERR_ARG: return "invalid argument";
    case CLMD_ERR_CUDA: return "CUDA runtime error";
    case CLMD_ERR_NOMEM: return "device out of memory";
    case CLMD_ERR_NO_DEVICE: return "no CUDA device (the engine has no CPU path)";
    case CLMD_ERR_TIMEOUT: return "bounded device wait timed out";
    default: return "unknown status";
  }
}

namespace {
// xoshiro256** seeded by splitmix64
struct Rng {
  uint64_t s[4];
  static uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  }
  explicit Rng(uint64_t seed) {
    for (int i = 0; i < 4; i++) s[i] = splitmix(seed);
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  double gauss() {  // Box-Muller
    double u1 = uniform(), u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
  }
};
}  // namespace

extern "C" int clmd_init_random(int32_t n, double bx, double by, double bz, double rmin,
                                double kT_over_m, uint64_t seed, double* x, double* y,
                                double* z, double* vx, double* vy, double* vz) {
  if (n < 1 || !(bx > 0 && by > 0 && bz > 0) || rmin < 0 || !x || !y || !z)
    return CLMD_ERR_ARG;
  Rng rng(seed);
  double vol = bx * by * bz;
  double side = std::max(rmin, cbrt(vol / n));
  int nx = std::max(1, (int)(bx / side)), ny = std::max(1, (int)(by / side)),
      nz = std::max(1, (int)(bz / side));
  std::vector<int> head((size_t)nx * ny * nz, -1), next(n, -1);
  double r2 = rmin * rmin;
  auto cell = [&](double px, double py, double pz, int* c3) {
    c3[0] = std::min(nx - 1, (int)(px / bx * nx));
    c3[1] = std::min(ny - 1, (int)(py / by * ny));
    c3[2] = std::min(nz - 1, (int)(pz / bz * nz));
  };
  for (int i = 0; i < n; i++) {
    int tries = 0;
    for (;;) {
      if (++tries > 100000) return CLMD_ERR_ARG;
      double px = rng.uniform() * bx, py = rng.uniform() * by, pz = rng.uniform() * bz;
      int c[3];
      cell(px, py, pz, c);
      bool ok = true;
      for (int a = -1; a <= 1 && ok; a++)
        for (int b = -1; b <= 1 && ok; b++)
          for (int d = -1; d <= 1 && ok; d++) {
            int xx = (c[0] + d + nx) % nx, yy = (c[1] + b + ny) % ny, zz = (c[2] + a + nz) % nz;
            for (int j = head[((size_t)zz * ny + yy) * nx + xx]; j >= 0; j = next[j]) {
              double dx = px - x[j], dy = py - y[j], dz = pz - z[j];
              dx -= bx * nearbyint(dx / bx);
              dy -= by * nearbyint(dy / by);
              dz -= bz * nearbyint(dz / bz);
              if (dx * dx + dy * dy + dz * dz < r2) {
                ok = false;
                break;
              }
            }
          }
      if (!ok) continue;
      x[i] = px;
      y[i] = py;
      z[i] = pz;
      size_t k = ((size_t)c[2] * ny + c[1]) * nx + c[0];
      next[i] = head[k];
      head[k] = i;
      break;
    }
  }
  double sd = sqrt(kT_over_m > 0 ? kT_over_m : 0.0);
  for (int i = 0; i < n; i++) {
    double a = rng.gauss(), b = rng.gauss(), c = rng.gauss();
    if (vx) vx[i] = sd * a;
    if (vy) vy[i] = sd * b;
    if (vz) vz[i] = sd * c;
  }
  return CLMD_OK;
}

extern "C" int64_t clmd_struct_size(int which) {
  switch (which) {
    case 0: return (int64_t)sizeof(clmd_config);
    case 1: return (int64_t)sizeof(clmd_scalars);
    case 2: return (int64_t)sizeof(clmd_cluster_view);
    case 3: return (int64_t)sizeof(clmd_ens_config);
    case 4: return (int64_t)sizeof(clmd_replica_spec);
    case 5: return (int64_t)sizeof(clmd_replica_result);
    case 6: return (int64_t)sizeof(clmd_request);
    case 7: return (int64_t)sizeof(clmd_request_result);
    case 8: return (int64_t)sizeof(clmd_serve_stats);
    default: return -1;
  }
}
