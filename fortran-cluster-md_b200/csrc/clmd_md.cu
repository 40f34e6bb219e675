// clmd_md.cu -- the MD step on the device, FP64 and bit-faithful to the
// reference: cell-list binning (counting sort), the Verlet-list rebuild with
// the adaptive skin (neighbor-pbc-mav.f), the LJ pair forces
// (for-a-lj-n-pbc-m.f), velocity Verlet (int-verlet-mav.f), Nose-Hoover
// (int-verlet-nh-mav.f), velocity scaling (scalev-nh-m.f) and momentum
// removal (stopdead-m.f).
//
// Built with -fmad=false: every FP64 expression is evaluated in the
// reference's order without contraction, so per-atom results (positions,
// velocities, accelerations, list membership) are bit-identical to a
// serial FP64 evaluation; only the order of global sums (ekin, epot,
// sumv2) differs.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdio.h>

#include "clmd_system.hpp"

namespace clmd {

// ---------------------------------------------------------------------------
// step counter (main.f's loop variable i lives on the device)
// ---------------------------------------------------------------------------
__global__ void k_set_step(DevState* st, int step) { st->cur_step = step; }

__global__ void k_step_advance(DevState* st) {
  if (gated(st)) return;
  st->cur_step = st->cur_step + 1;
}

// ---------------------------------------------------------------------------
// neighbor-pbc-mav.f:42-65 + 101-105: scalar prologue of a rebuild.
// Single thread.  Sets st->rebuild = 0 on the fatal skin error.
// ---------------------------------------------------------------------------
__device__ void nb_prologue(const Params& P, DevState* st) {
  clmd_scalars& q = st->s;
  int step = st->cur_step;
  // :48-51
  if (q.dmms > (q.atrskin - P.atrcut)) {
    if (q.status == 0) {
      q.status = CLMD_ERR_SKIN;
      q.fail_step = step;
    }
    st->rebuild = 0;
    return;
  }
  // :53
  q.dmmav = (double)(float)q.dmmst * q.dmmsu / 256.0;
  // :55-60
  if (step != P.btim && step > 0) {
    q.atrskin = P.atrcut + (q.atrskin - P.atrcut) * (double)P.nbtim / (double)q.dmmst;
    q.atrskin = fmin(P.boxx / 2.0, q.atrskin);
    q.atrskin = fmin(P.boxy / 2.0, q.atrskin);
    q.atrskin = fmin(P.boxz / 2.0, q.atrskin);
  }
  st->rs2 = q.atrskin * q.atrskin;
  // cell grid: side >= rs (relative margin far above rounding), capped by
  // the allocation (larger cells stay correct)
  double side = q.atrskin * (1.0 + 1e-9);
  int nx = (int)floor(P.boxx / side), ny = (int)floor(P.boxy / side),
      nz = (int)floor(P.boxz / side);
  nx = max(1, min(nx, P.ncx_max));
  ny = max(1, min(ny, P.ncy_max));
  nz = max(1, min(nz, P.ncz_max));
  st->ncx = nx;
  st->ncy = ny;
  st->ncz = nz;
  st->ncell = nx * ny * nz;
  st->cfx = (double)nx / P.boxx;
  st->cfy = (double)ny / P.boxy;
  st->cfz = (double)nz / P.boxz;
  int n3[3] = {nx, ny, nz};
  int* offs[3] = {st->offx, st->offy, st->offz};
  int* nos[3] = {&st->nox, &st->noy, &st->noz};
  for (int d = 0; d < 3; d++) {
    if (n3[d] >= 3) {
      offs[d][0] = -1; offs[d][1] = 0; offs[d][2] = 1; *nos[d] = 3;
    } else if (n3[d] == 2) {
      offs[d][0] = 0; offs[d][1] = 1; *nos[d] = 2;
    } else {
      offs[d][0] = 0; *nos[d] = 1;
    }
  }
  st->list_used = 0ull;
  // :101-105
  q.dmmax = fmax(q.dmms, q.dmmax);
  q.dmms = 0.0;
  q.dmmst = 0;
  q.nrebuild = q.nrebuild + 1;
  q.last_rebuild_step = step;
}

__global__ void k_nb_prologue(Params P, DevState* st) {
  if (gated(st)) {
    st->rebuild = 0;
    return;
  }
  st->rebuild = 1;
  nb_prologue(P, st);
}

__global__ void k_nb_clear(DevState* st, int* cell_count, int n) {
  if (!st->rebuild || gated(st)) return;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    cell_count[c] = 0;
}

__device__ __forceinline__ int cell_of(const DevState* st, double x, double y, double z) {
  int cx = min((int)(x * st->cfx), st->ncx - 1);
  int cy = min((int)(y * st->cfy), st->ncy - 1);
  int cz = min((int)(z * st->cfz), st->ncz - 1);
  return (cz * st->ncy + cy) * st->ncx + cx;
}

// neighbor-pbc-mav.f:67-71 wrap, then the counting sort's histogram
__global__ void k_nb_bin(Params P, DevState* st, double4* pos, int* atom_cell,
                         int* cell_count) {
  if (!st->rebuild || gated(st)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.N) return;
  double4 p = pos[i];
  p.x = fmod(fmod(p.x, P.boxx) + P.boxx, P.boxx);
  p.y = fmod(fmod(p.y, P.boxy) + P.boxy, P.boxy);
  p.z = fmod(fmod(p.z, P.boxz) + P.boxz, P.boxz);
  pos[i] = p;
  int c = cell_of(st, p.x, p.y, p.z);
  atom_cell[i] = c;
  atomicAdd(&cell_count[c], 1);
}

// exclusive scan of cell counts: tile sums -> scan of tile sums -> tiles
__device__ __forceinline__ int block_scan_excl(int v, int* sh, int* total) {
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  __syncthreads();
  if (lane == 31) sh[w] = incl;
  __syncthreads();
  if (w == 0) {
    int s = lane < nw ? sh[lane] : 0;
    int si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si += t;
    }
    if (lane < nw) sh[lane] = si - s;
    if (lane == nw - 1) sh[32] = si;
  }
  __syncthreads();
  *total = sh[32];
  return sh[w] + incl - v;
}

constexpr int kScanPer = kScanTile / kBlock;

__global__ void k_scan_tiles(DevState* st, const int* cnt, int* aux) {
  if (!st->rebuild || gated(st)) return;
  int n = st->ncell;
  int base = blockIdx.x * kScanTile;
  if (base >= n) return;
  __shared__ double sh[kBlock / 32];
  int s = 0;
  for (int k = 0; k < kScanPer; k++) {
    int c = base + threadIdx.x * kScanPer + k;
    if (c < n) s += cnt[c];
  }
  double t = block_sum((double)s, sh);
  if (threadIdx.x == 0) aux[blockIdx.x] = (int)t;
}

__global__ void k_scan_top(Params P, DevState* st, int* aux, int* cell_start) {
  if (!st->rebuild || gated(st)) return;
  int ntiles = (st->ncell + kScanTile - 1) / kScanTile;
  __shared__ int sh[33];
  int carry = 0;
  for (int b0 = 0; b0 < ntiles; b0 += blockDim.x) {
    int b = b0 + threadIdx.x;
    int v = b < ntiles ? aux[b] : 0;
    int tot;
    int ex = block_scan_excl(v, sh, &tot);
    if (b < ntiles) aux[b] = carry + ex;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) cell_start[st->ncell] = P.N;
}

__global__ void k_scan_final(DevState* st, const int* cnt, const int* aux, int* cell_start,
                             int* cell_fill) {
  if (!st->rebuild || gated(st)) return;
  int n = st->ncell;
  int base = blockIdx.x * kScanTile;
  if (base >= n) return;
  __shared__ int sh[33];
  int loc[kScanPer];
  int s = 0;
  for (int k = 0; k < kScanPer; k++) {
    int c = base + threadIdx.x * kScanPer + k;
    loc[k] = c < n ? cnt[c] : 0;
    s += loc[k];
  }
  int tot;
  int ex = block_scan_excl(s, sh, &tot) + aux[blockIdx.x];
  for (int k = 0; k < kScanPer; k++) {
    int c = base + threadIdx.x * kScanPer + k;
    if (c < n) {
      cell_start[c] = ex;
      cell_fill[c] = ex;
    }
    ex += loc[k];
  }
}

__global__ void k_nb_scatter(Params P, DevState* st, const double4* pos, const int* atom_cell,
                             int* cell_fill, int* cell_atoms, double4* spos) {
  if (!st->rebuild || gated(st)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.N) return;
  int slot = atomicAdd(&cell_fill[atom_cell[i]], 1);
  cell_atoms[slot] = i;
  spos[slot] = pos[i];
}

// neighbor-pbc-mav.f:73-99 on the cell list.  One thread per cell-sorted
// slot; every candidate is decided by the reference's own test, evaluated in
// the reference's orientation (row of the smaller index), so the pair set
// equals the all-pairs one.  Rows are counted, allocated warp-wise from a
// global cursor, filled, and sorted ascending.
__device__ __forceinline__ bool nb_test(const Params& P, double rs2, const double4& a,
                                        const double4& b) {
  double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
  dx = mimage_nb(dx, P.boxx, P.ibx);
  dy = mimage_nb(dy, P.boxy, P.iby);
  dz = mimage_nb(dz, P.boxz, P.ibz);
  double r2 = dx * dx + dy * dy + dz * dz;
  return r2 <= rs2;
}

template <bool FILL>
__device__ __forceinline__ int nb_scan_cells(const Params& P, const DevState* st, int i,
                                             const double4& pi, const double4* spos,
                                             const int* cell_atoms, const int* cell_start,
                                             int* row) {
  int cx = min((int)(pi.x * st->cfx), st->ncx - 1);
  int cy = min((int)(pi.y * st->cfy), st->ncy - 1);
  int cz = min((int)(pi.z * st->cfz), st->ncz - 1);
  const double rs2 = st->rs2;
  int n = 0;
  for (int a = 0; a < st->noz; a++) {
    int zz = cz + st->offz[a];
    zz += (zz < 0) ? st->ncz : 0;
    zz -= (zz >= st->ncz) ? st->ncz : 0;
    for (int b = 0; b < st->noy; b++) {
      int yy = cy + st->offy[b];
      yy += (yy < 0) ? st->ncy : 0;
      yy -= (yy >= st->ncy) ? st->ncy : 0;
      for (int d = 0; d < st->nox; d++) {
        int xx = cx + st->offx[d];
        xx += (xx < 0) ? st->ncx : 0;
        xx -= (xx >= st->ncx) ? st->ncx : 0;
        int cell = (zz * st->ncy + yy) * st->ncx + xx;
        int q1 = cell_start[cell + 1];
        for (int q = cell_start[cell]; q < q1; q++) {
          int j = cell_atoms[q];
          if (j == i) continue;
          double4 pj = spos[q];
          bool hit = (i < j) ? nb_test(P, rs2, pi, pj) : nb_test(P, rs2, pj, pi);
          if (hit) {
            if (FILL) row[n] = j;
            n++;
          }
        }
      }
    }
  }
  return n;
}

__global__ void k_nb_search(Params P, DevState* st, const double4* spos, const int* cell_atoms,
                            const int* cell_start, int* list, int* row_start, int* row_len,
                            int* row_lo) {
  if (!st->rebuild || gated(st)) return;
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  int lane = threadIdx.x & 31;
  bool active = p < P.N;
  int i = 0, cnt = 0;
  double4 pi = make_double4(0, 0, 0, 0);
  if (active) {
    i = cell_atoms[p];
    pi = spos[p];
    cnt = nb_scan_cells<false>(P, st, i, pi, spos, cell_atoms, cell_start, nullptr);
  }
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  unsigned long long base = 0;
  if (lane == 31) base = atomicAdd(&st->list_used, (unsigned long long)incl);
  base = __shfl_sync(0xffffffffu, base, 31);
  if (!active) return;
  unsigned long long start = base + (unsigned long long)(incl - cnt);
  if (start + (unsigned long long)cnt > (unsigned long long)P.list_cap) {
    raise_err(st, CLMD_ERR_LIST_OVERFLOW);
    row_start[i] = 0;
    row_len[i] = 0;
    row_lo[i] = 0;
    return;
  }
  int* row = list + start;
  nb_scan_cells<true>(P, st, i, pi, spos, cell_atoms, cell_start, row);
  // ascending order = the reference's summation order
  for (int a = 1; a < cnt; a++) {
    int key = row[a];
    int b = a - 1;
    while (b >= 0 && row[b] > key) {
      row[b + 1] = row[b];
      b--;
    }
    row[b + 1] = key;
  }
  int lo = 0;
  while (lo < cnt && row[lo] < i) lo++;
  row_start[i] = (int)start;
  row_len[i] = cnt;
  row_lo[i] = lo;
}

// ---------------------------------------------------------------------------
// skin bookkeeping, int-verlet-mav.f:64-74 (= int-verlet-nh-mav.f:70-78)
// ---------------------------------------------------------------------------
__device__ void skin_update(const Params& P, DevState* st, double dmmr) {
  clmd_scalars& q = st->s;
  dmmr = 2.2 * sqrt(dmmr);
  q.dmms = q.dmms + dmmr;
  q.dmmsu = q.dmmsu + dmmr - q.dmmh[q.dmmi];
  q.dmmh[q.dmmi] = dmmr;
  q.dmmi = (q.dmmi + 1) & 255;
  q.dmmst = q.dmmst + 1;
  int rb = q.dmms > (q.atrskin - P.atrcut - 2.0 * q.dmms / (double)(float)q.dmmst);
  st->rebuild = rb;
  if (rb) nb_prologue(P, st);
}

// int-verlet-mav.f:44-74: drift + first half kick + max displacement
__global__ void k_vv_drift(Params P, DevState* st, double4* pos, double* vx, double* vy,
                           double* vz, const double* ax, const double* ay, const double* az,
                           unsigned long long cond, int use_cond) {
  if (gated(st)) return;
  __shared__ double sh[kBlock / 32];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double d2 = 0.0;
  if (i < P.N) {
    const double dt = P.dt;
    double4 p = pos[i];
    double hx = 0.5 * ax[i] * dt, hy = 0.5 * ay[i] * dt, hz = 0.5 * az[i] * dt;
    double vxi = vx[i], vyi = vy[i], vzi = vz[i];
    double dx = (vxi + hx) * dt, dy = (vyi + hy) * dt, dz = (vzi + hz) * dt;
    p.x = p.x + dx;
    p.y = p.y + dy;
    p.z = p.z + dz;
    pos[i] = p;
    vx[i] = vxi + hx;
    vy[i] = vyi + hy;
    vz[i] = vzi + hz;
    d2 = dx * dx + dy * dy + dz * dz;
  }
  double m = block_max(d2, sh);
  if (threadIdx.x == 0) atomicMax(&st->dmax2, (unsigned long long)__double_as_longlong(m));
  if (last_block(&st->ctr[CTR_DRIFT])) {
    if (threadIdx.x == 0) {
      double dmmr = __longlong_as_double((long long)atomicExch(&st->dmax2, 0ull));
      skin_update(P, st, dmmr);
      if (use_cond) cudaGraphSetConditional(cond, st->rebuild ? 1u : 0u);
    }
  }
}

// int-verlet-nh-mav.f:43-78: drift with friction, sumv2 of the old
// velocities, explicit s/PSI half step, skin bookkeeping
__global__ void k_nh_drift(Params P, DevState* st, double4* pos, double* vx, double* vy,
                           double* vz, const double* ax, const double* ay, const double* az,
                           double* partials, unsigned long long cond, int use_cond) {
  if (gated(st)) return;
  __shared__ double sh[kBlock / 32];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double dt = P.dt, dt2 = dt * dt / 2, dth = dt / 2;
  const double psi = st->s.psi;
  double d2 = 0.0, sv = 0.0;
  if (i < P.N) {
    double4 p = pos[i];
    double vxi = vx[i], vyi = vy[i], vzi = vz[i];
    double axi = ax[i], ayi = ay[i], azi = az[i];
    double dx = dt * vxi + dt2 * (axi - psi * vxi);
    double dy = dt * vyi + dt2 * (ayi - psi * vyi);
    double dz = dt * vzi + dt2 * (azi - psi * vzi);
    p.x = p.x + dx;
    p.y = p.y + dy;
    p.z = p.z + dz;
    pos[i] = p;
    sv = vxi * vxi + vyi * vyi + vzi * vzi;
    vx[i] = vxi + dth * (axi - psi * vxi);
    vy[i] = vyi + dth * (ayi - psi * vyi);
    vz[i] = vzi + dth * (azi - psi * vzi);
    d2 = dx * dx + dy * dy + dz * dz;
  }
  double m = block_max(d2, sh);
  if (threadIdx.x == 0) atomicMax(&st->dmax2, (unsigned long long)__double_as_longlong(m));
  double s = block_sum(sv, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
  if (last_block(&st->ctr[CTR_DRIFT])) {
    double tot = reduce_partials(partials, gridDim.x, sh);
    if (threadIdx.x == 0) {
      clmd_scalars& q = st->s;
      q.sumv2 = tot;
      // :64-67
      if (P.ethst == 'N') {
        q.s = q.s + q.psi * dt + (P.apmas[0] * q.sumv2 - P.nkt3_d) * dt2 / P.Q;
        q.psi = q.psi + (P.apmas[0] * q.sumv2 - P.nkt3_d) * dth / P.Q;
      }
      double dmmr = __longlong_as_double((long long)atomicExch(&st->dmax2, 0ull));
      skin_update(P, st, dmmr);
      if (use_cond) cudaGraphSetConditional(cond, st->rebuild ? 1u : 0u);
    }
  }
}

// ---------------------------------------------------------------------------
// for-a-lj-n-pbc-m.f:61-152: pair forces over the full list.  Each atom sums
// its pair terms in ascending neighbour order, each term computed in the
// reference's orientation (dx = x(min) - x(max), +f for the smaller index,
// -f for the larger), which is exactly the order in which the reference's
// serial scatter accumulates fsum(i); so fsum, and a, are bit-identical.
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_force(Params P, DevState* st, const double4* pos,
                                                  const int* list, const int* row_start,
                                                  const int* row_len, double* ax, double* ay,
                                                  double* az, double* vx, double* vy, double* vz,
                                                  double* partials) {
  if (gated(st)) return;
  __shared__ double sh[kBlock / 32];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double esum = 0.0, vir = 0.0, ek = 0.0;
  const double bf1 = 2.0 + (double)(int)(st->s.atrskin / P.sig1);
  const double bf2 = bf1 + 0.5;
  if (i < P.N) {
    double4 pa = pos[i];
    int sa = (int)pa.w;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    int k0 = row_start[i], k1 = k0 + row_len[i];
    for (int k = k0; k < k1; k++) {
      int j = list[k];
      double4 pb = pos[j];
      bool own = i < j;  // this atom is the reference's row atom
      double dx, dy, dz;
      if (own) {
        dx = pa.x - pb.x; dy = pa.y - pb.y; dz = pa.z - pb.z;
      } else {
        dx = pb.x - pa.x; dy = pb.y - pa.y; dz = pb.z - pa.z;
      }
      dx = mimage_bf(dx, P.boxx, P.ibx, bf1, bf2);
      dy = mimage_bf(dy, P.boxy, P.iby, bf1, bf2);
      dz = mimage_bf(dz, P.boxz, P.ibz, bf1, bf2);
      double rij2 = dx * dx + dy * dy + dz * dz;
      if (rij2 <= P.atr2) {
        double r2 = rij2;
        rij2 = 1.0 / rij2;
        double rij6 = rij2 * rij2 * rij2;
        int ij = sa + (int)pb.w;
        if (ij < 2 || ij > 4) {
          raise_err(st, CLMD_ERR_BAD_SPECIES);
          continue;
        }
        double fij = P.eps[ij] * 48.0 * rij2 * rij6 * (P.c2[ij] * rij6 - P.c3[ij]);
        if (own) {
          esum = esum + P.eps[ij] * 4.0 * rij6 * (P.c2[ij] * rij6 - P.c1[ij]);
          vir = vir + fij * r2;
          fx = fx + fij * dx;
          fy = fy + fij * dy;
          fz = fz + fij * dz;
        } else {
          fx = fx - fij * dx;
          fy = fy - fij * dy;
          fz = fz - fij * dz;
        }
      }
    }
    double iatm = 1.0 / P.apmas[sa - 1];
    double a0x = 0.0, a0y = 0.0, a0z = 0.0;
    if (MODE == FORCE_ACCUMULATE) {
      a0x = ax[i]; a0y = ay[i]; a0z = az[i];
    }
    double axi = a0x + fx * iatm, ayi = a0y + fy * iatm, azi = a0z + fz * iatm;
    ax[i] = axi;
    ay[i] = ayi;
    az[i] = azi;
    if (MODE == FORCE_VV_KICK) {
      // int-verlet-mav.f:86-92
      const double dt = P.dt;
      double vxi = vx[i] + 0.5 * axi * dt;
      double vyi = vy[i] + 0.5 * ayi * dt;
      double vzi = vz[i] + 0.5 * azi * dt;
      vx[i] = vxi;
      vy[i] = vyi;
      vz[i] = vzi;
      ek = 0.5 * P.apmas[sa - 1] * (vxi * vxi + vyi * vyi + vzi * vzi);
    }
  }
  int nb = gridDim.x;
  double t0 = block_sum(esum, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t0;
  double t1 = block_sum(vir, sh);
  if (threadIdx.x == 0) partials[nb + blockIdx.x] = t1;
  if (MODE == FORCE_VV_KICK) {
    double t2 = block_sum(ek, sh);
    if (threadIdx.x == 0) partials[2 * nb + blockIdx.x] = t2;
  }
  if (last_block(&st->ctr[CTR_FORCE])) {
    double e = reduce_partials(partials, nb, sh);
    double w = reduce_partials(partials + nb, nb, sh);
    double k = 0.0;
    if (MODE == FORCE_VV_KICK) k = reduce_partials(partials + 2 * nb, nb, sh);
    if (threadIdx.x == 0) {
      clmd_scalars& q = st->s;
      q.epot = e;
      q.virial = w;
      if (MODE == FORCE_VV_KICK) q.ekin = k;
      q.npairs_half = (long long)(st->list_used / 2ull);
      int err = atomicExch(&st->err_new, 0);
      if (err && q.status == 0) {
        q.status = err;
        q.fail_step = st->cur_step;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// int-verlet-nh-mav.f:91-180: implicit solve for v(t+dt) and PSI.  One
// cooperative launch; each sweep has two grid-wide sums (delps; sumv2 with
// the all-converged test).  Every block reduces the partials itself in the
// same order, so all blocks hold identical scalars and agree on when to stop.
// ---------------------------------------------------------------------------
__device__ bool grid_sync(DevState* st) {
  __shared__ int fail;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* gen = &st->bar_gen;
    unsigned int g = *gen;
    __threadfence();
    unsigned int arrived = atomicAdd(&st->bar_count, 1u);
    fail = 0;
    if (arrived == gridDim.x - 1) {
      atomicExch(&st->bar_count, 0u);
      __threadfence();
      atomicAdd(&st->bar_gen, 1u);
    } else {
      long long spins = 0;
      while (*gen == g) {
        __nanosleep(64);
        if (++spins > (1ll << 25)) {
          fail = 1;
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
  return fail == 0;
}

__device__ __forceinline__ double all_sum(const double* p, int n, double* sh) {
  __shared__ double res;
  double v = reduce_partials(p, n, sh);
  if (threadIdx.x == 0) res = v;
  __syncthreads();
  double r = res;
  __syncthreads();
  return r;
}

__global__ void k_nh_solve(Params P, DevState* st, const double* ax, const double* ay,
                           const double* az, double* vx, double* vy, double* vz, double* vxn,
                           double* vyn, double* vzn, double* pA, double* pB, double* pC) {
  if (gated(st)) return;
  __shared__ double sh[32];
  const int N = P.N;
  const int G = gridDim.x * blockDim.x;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int nb = gridDim.x;
  const double dt = P.dt, dt2 = dt * dt / 2, dth = dt / 2, Q = P.Q, m = P.apmas[0];
  const double err = 1.0e-10;
  const double psi = st->s.psi;
  // :94-100
  double sv = 0.0;
  for (int i = t0; i < N; i += G) {
    double a = vx[i], b = vy[i], c = vz[i];
    vxn[i] = a;
    vyn[i] = b;
    vzn[i] = c;
    sv = sv + a * a + b * b + c * c;
  }
  double bs = block_sum(sv, sh);
  if (threadIdx.x == 0) pB[blockIdx.x] = bs;
  if (!grid_sync(st)) goto timeout;
  {
    double sumv2 = all_sum(pB, nb, sh);
    double psn = psi, pso = psi;
    int ready = 0, iter;
    for (iter = 1; iter <= 1000; iter++) {
      pso = psn;
      // :110-120
      double dp = 0.0;
      for (int i = t0; i < N; i += G) {
        double vo = vxn[i];
        double b = -dth * (ax[i] - pso * vo) - (vx[i] - vo);
        dp = dp + b * m * vo * dt / Q;
        vo = vyn[i];
        b = -dth * (ay[i] - pso * vo) - (vy[i] - vo);
        dp = dp + b * m * vo * dt / Q;
        vo = vzn[i];
        b = -dth * (az[i] - pso * vo) - (vz[i] - vo);
        dp = dp + b * m * vo * dt / Q;
      }
      bs = block_sum(dp, sh);
      if (threadIdx.x == 0) pA[blockIdx.x] = bs;
      if (!grid_sync(st)) goto timeout;
      double delps = all_sum(pA, nb, sh);
      // :122-125
      double di = -(pso * dth + 1);
      delps = delps - di * ((-m * sumv2 + P.nkt3_i) * dth / Q - (psi - pso));
      delps = delps / (-dt2 * m * sumv2 / Q + di);
      // :127-143
      double s2 = 0.0;
      int notready = 0;
      for (int i = t0; i < N; i += G) {
        double vo = vxn[i];
        double b = -dth * (ax[i] - pso * vo) - (vx[i] - vo);
        double nx = vo + (b + dth * vo * delps) / di;
        vo = vyn[i];
        b = -dth * (ay[i] - pso * vo) - (vy[i] - vo);
        double ny = vo + (b + dth * vo * delps) / di;
        vo = vzn[i];
        b = -dth * (az[i] - pso * vo) - (vz[i] - vo);
        double nz = vo + (b + dth * vo * delps) / di;
        if (fabs((nx - vxn[i]) / nx) > err) notready = 1;
        if (fabs((ny - vyn[i]) / ny) > err) notready = 1;
        if (fabs((nz - vzn[i]) / nz) > err) notready = 1;
        vxn[i] = nx;
        vyn[i] = ny;
        vzn[i] = nz;
        s2 = s2 + nx * nx + ny * ny + nz * nz;
      }
      bs = block_sum(s2, sh);
      int anynr = __syncthreads_or(notready);
      if (threadIdx.x == 0) {
        pB[blockIdx.x] = bs;
        pC[blockIdx.x] = (double)anynr;
      }
      if (!grid_sync(st)) goto timeout;
      sumv2 = all_sum(pB, nb, sh);
      double nr = all_sum(pC, nb, sh);
      psn = pso + delps;
      ready = (nr == 0.0);
      if (ready) break;
    }
    // :150-180
    if (!ready) {
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->s.nh_iters = 1000;
        if (st->s.status == 0) {
          st->s.status = CLMD_ERR_NH_NOCONVERGE;
          st->s.fail_step = st->cur_step;
        }
      }
      return;
    }
    for (int i = t0; i < N; i += G) {
      vx[i] = vxn[i];
      vy[i] = vyn[i];
      vz[i] = vzn[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->s.sumv2 = sumv2;
      st->s.psi = psn;
      st->s.ekin = 0.5 * m * sumv2;
      st->s.nh_iters = iter;
    }
    return;
  }
timeout:
  if (threadIdx.x == 0) atomicCAS(&st->s.status, 0, CLMD_ERR_TIMEOUT);
}

// ---------------------------------------------------------------------------
// scalev-nh-m.f:39-76 velocity scaling per species block
// ---------------------------------------------------------------------------
__device__ __forceinline__ int species_block(const Params& P, int i) {
  for (int s = 0; s < P.atsorts; s++)
    if (i >= P.sp_start[s] && i < P.sp_start[s + 1]) return s;
  return -1;
}

__global__ void k_thermo_sum(Params P, DevState* st, const double* vx, const double* vy,
                             const double* vz, double* partials, int step) {
  if (gated(st)) return;
  __shared__ double sh[kBlock / 32];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int sp = -1;
  double e = 0.0;
  if (i < P.N) {
    sp = species_block(P, i);
    if (sp >= 0)
      e = 0.5 * P.apmas[sp] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
  }
  int nb = gridDim.x;
  for (int s = 0; s < P.atsorts; s++) {
    double t = block_sum(sp == s ? e : 0.0, sh);
    if (threadIdx.x == 0) partials[s * nb + blockIdx.x] = t;
  }
  if (last_block(&st->ctr[CTR_THERMO])) {
    __shared__ double eks[CLMD_MXSORTS];
    for (int s = 0; s < P.atsorts; s++) {
      double t = reduce_partials(partials + s * nb, nb, sh);
      if (threadIdx.x == 0) eks[s] = t;
    }
    if (threadIdx.x == 0) {
      double ekin = 0.0;
      for (int s = 0; s < P.atsorts; s++) {
        double ek = eks[s];
        ekin = ekin + ek;
        double kf = sqrt(P.ekinT[s] / ek);
        st->kf[s] = kf;
        int sc = (P.apth[s] == 'X' || step == -1);
        st->scale[s] = sc;
        if (sc) ekin = ekin - ek + P.ekinT[s];
      }
      st->s.ekin = ekin;
    }
  }
}

__global__ void k_thermo_scale(Params P, DevState* st, double* vx, double* vy, double* vz) {
  if (gated(st)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.N) return;
  int sp = species_block(P, i);
  if (sp < 0 || !st->scale[sp]) return;
  double kf = st->kf[sp];
  vx[i] = vx[i] * kf;
  vy[i] = vy[i] * kf;
  vz[i] = vz[i] * kf;
}

// stopdead-m.f:30-55
__global__ void k_mom_sum(Params P, DevState* st, const int* api, const double* vx,
                          const double* vy, const double* vz, double* partials) {
  if (gated(st)) return;
  __shared__ double sh[kBlock / 32];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double px = 0.0, py = 0.0, pz = 0.0;
  if (i < P.N) {
    double mas = P.apmas[api[i] - 1];
    px = vx[i] * mas;
    py = vy[i] * mas;
    pz = vz[i] * mas;
  }
  int nb = gridDim.x;
  double t = block_sum(px, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
  t = block_sum(py, sh);
  if (threadIdx.x == 0) partials[nb + blockIdx.x] = t;
  t = block_sum(pz, sh);
  if (threadIdx.x == 0) partials[2 * nb + blockIdx.x] = t;
  if (last_block(&st->ctr[CTR_MOM])) {
    double a = reduce_partials(partials, nb, sh);
    double b = reduce_partials(partials + nb, nb, sh);
    double c = reduce_partials(partials + 2 * nb, nb, sh);
    if (threadIdx.x == 0) {
      st->vcom[0] = a / (double)P.N;
      st->vcom[1] = b / (double)P.N;
      st->vcom[2] = c / (double)P.N;
    }
  }
}

__global__ void k_mom_sub(Params P, DevState* st, const int* api, double* vx, double* vy,
                          double* vz, double* partials) {
  if (gated(st)) return;
  __shared__ double sh[kBlock / 32];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  if (i < P.N) {
    double mas = P.apmas[api[i] - 1];
    double imas = 1.0 / mas;
    double a = vx[i] - st->vcom[0] * imas;
    double b = vy[i] - st->vcom[1] * imas;
    double c = vz[i] - st->vcom[2] * imas;
    vx[i] = a;
    vy[i] = b;
    vz[i] = c;
    e = mas * (a * a + b * b + c * c);
  }
  double t = block_sum(e, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
  if (last_block(&st->ctr[CTR_MOM2])) {
    double s = reduce_partials(partials, gridDim.x, sh);
    if (threadIdx.x == 0) st->s.ekin = 0.5 * s;
  }
}

__global__ void k_zero_acc(int N, double* ax, double* ay, double* az) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  ax[i] = 0.0;
  ay[i] = 0.0;
  az[i] = 0.0;
}

__global__ void k_pack_pos(int N, const double* sx, const double* sy, const double* sz,
                           const int* api, double4* pos, int hx, int hy, int hz) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double4 p = pos[i];
  if (hx) p.x = sx[i];
  if (hy) p.y = sy[i];
  if (hz) p.z = sz[i];
  p.w = (double)api[i];
  pos[i] = p;
}

__global__ void k_unpack_pos(int N, const double4* pos, double* sx, double* sy, double* sz) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double4 p = pos[i];
  sx[i] = p.x;
  sy[i] = p.y;
  sz[i] = p.z;
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
void k_set_step_launch(clmd_system* S, int step) {
  k_set_step<<<1, 1, 0, S->stream>>>(S->st, step);
  S->launches++;
}
void k_step_advance_launch(clmd_system* S) {
  k_step_advance<<<1, 1, 0, S->stream>>>(S->st);
  S->launches++;
}
void nb_prologue_launch(clmd_system* S) {
  k_nb_prologue<<<1, 1, 0, S->stream>>>(S->P, S->st);
  S->launches++;
}

void rebuild_launch(clmd_system* S, cudaStream_t s) {
  const Params& P = S->P;
  int nb = S->nblk;
  int nclr = (S->ncell_alloc + kBlock - 1) / kBlock;
  nclr = nclr > 4 * S->num_sms ? 4 * S->num_sms : (nclr < 1 ? 1 : nclr);
  int ntiles = (S->ncell_alloc + kScanTile - 1) / kScanTile;
  k_nb_clear<<<nclr, kBlock, 0, s>>>(S->st, S->cell_count, S->ncell_alloc);
  k_nb_bin<<<nb, kBlock, 0, s>>>(P, S->st, S->pos, S->atom_cell, S->cell_count);
  k_scan_tiles<<<ntiles, kBlock, 0, s>>>(S->st, S->cell_count, S->scan_aux);
  k_scan_top<<<1, 1024, 0, s>>>(P, S->st, S->scan_aux, S->cell_start);
  k_scan_final<<<ntiles, kBlock, 0, s>>>(S->st, S->cell_count, S->scan_aux, S->cell_start,
                                          S->cell_fill);
  k_nb_scatter<<<nb, kBlock, 0, s>>>(P, S->st, S->pos, S->atom_cell, S->cell_fill,
                                      S->cell_atoms, S->spos);
  k_nb_search<<<nb, kBlock, 0, s>>>(P, S->st, S->spos, S->cell_atoms, S->cell_start, S->list,
                                     S->row_start, S->row_len, S->row_lo);
  S->launches += 7;
}

void drift_launch(clmd_system* S, unsigned long long cond, int use_cond) {
  if (S->P.integrator == CLMD_INT_NOSE)
    k_nh_drift<<<S->nblk, kBlock, 0, S->stream>>>(S->P, S->st, S->pos, S->vx, S->vy, S->vz,
                                                   S->ax, S->ay, S->az, S->partials, cond,
                                                   use_cond);
  else
    k_vv_drift<<<S->nblk, kBlock, 0, S->stream>>>(S->P, S->st, S->pos, S->vx, S->vy, S->vz,
                                                   S->ax, S->ay, S->az, cond, use_cond);
  S->launches++;
}

void force_launch(clmd_system* S, int mode) {
  auto args = [&](auto kern) {
    kern<<<S->nblk, kBlock, 0, S->stream>>>(S->P, S->st, S->pos, S->list, S->row_start,
                                             S->row_len, S->ax, S->ay, S->az, S->vx, S->vy,
                                             S->vz, S->partials);
  };
  if (mode == FORCE_VV_KICK)
    args(k_force<FORCE_VV_KICK>);
  else if (mode == FORCE_ZERO_FIRST)
    args(k_force<FORCE_ZERO_FIRST>);
  else
    args(k_force<FORCE_ACCUMULATE>);
  S->launches++;
}

int coop_blocks_for(clmd_system* S) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_nh_solve, 512, 0);
  if (per_sm < 1) per_sm = 1;
  if (per_sm > 2) per_sm = 2;
  int nb = S->num_sms * per_sm;
  int need = (S->P.N + 511) / 512;
  if (need < nb) nb = need < 1 ? 1 : need;
  return nb;
}

void nh_solve_launch(clmd_system* S) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(S->coop_blocks);
  cfg.blockDim = dim3(512);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = S->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int nb = S->coop_blocks;
  double* pA = S->partials;
  double* pB = S->partials + kMaxRedBlocks;
  double* pC = S->partials + 2 * kMaxRedBlocks;
  (void)nb;
  cudaLaunchKernelEx(&cfg, k_nh_solve, S->P, S->st, (const double*)S->ax,
                     (const double*)S->ay, (const double*)S->az, S->vx, S->vy, S->vz, S->vxn,
                     S->vyn, S->vzn, pA, pB, pC);
  S->launches++;
}

void thermostat_launch(clmd_system* S, int step) {
  k_thermo_sum<<<S->nblk, kBlock, 0, S->stream>>>(S->P, S->st, S->vx, S->vy, S->vz,
                                                   S->partials, step);
  k_thermo_scale<<<S->nblk, kBlock, 0, S->stream>>>(S->P, S->st, S->vx, S->vy, S->vz);
  S->launches += 2;
}

void stopdead_launch(clmd_system* S, int step) {
  for (int loop = 0; loop < 10; loop++) {
    k_mom_sum<<<S->nblk, kBlock, 0, S->stream>>>(S->P, S->st, S->api, S->vx, S->vy, S->vz,
                                                  S->partials);
    k_mom_sub<<<S->nblk, kBlock, 0, S->stream>>>(S->P, S->st, S->api, S->vx, S->vy, S->vz,
                                                  S->partials);
    S->launches += 2;
    thermostat_launch(S, step);
  }
}

void zero_acc_launch(clmd_system* S) {
  k_zero_acc<<<S->nblk, kBlock, 0, S->stream>>>(S->P.N, S->ax, S->ay, S->az);
  S->launches++;
}

void pack_pos_launch(clmd_system* S, int hx, int hy, int hz) {
  k_pack_pos<<<S->nblk, kBlock, 0, S->stream>>>(S->P.N, S->sx, S->sy, S->sz, S->api, S->pos,
                                                 hx, hy, hz);
  S->launches++;
}

void unpack_pos_launch(clmd_system* S) {
  k_unpack_pos<<<S->nblk, kBlock, 0, S->stream>>>(S->P.N, S->pos, S->sx, S->sy, S->sz);
  S->launches++;
}

}  // namespace clmd
