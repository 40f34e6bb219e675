// clmd_cycle.cu -- the MD step as ONE persistent cooperative kernel.
//
// A launch runs `nsteps` consecutive integrator(i) calls (int-verlet-mav.f
// or int-verlet-nh-mav.f, with scalev velocity scaling before each step when
// ethst == 'X', main.f:207) for one system, or one neighbor() call.  Phases
// are separated by a grid barrier instead of kernel boundaries:
//
//   velocity Verlet, per step:  [force_n + kick_n + drift_n+1] -> barrier
//                               -> skin decision -> (rebuild: 7 barriers)
//   Nose-Hoover, per step:      drift -> barrier -> (rebuild) -> force +
//                               first sweep -> barrier -> one barrier per
//                               further sweep of the implicit solve
//
// Forces of step n read the positions of step n while the fused drift writes
// step n+1's, so positions are double-buffered (pos0/pos1); v and a are only
// ever touched by their own atom.  Every block keeps a replica of the scalar
// state (clmd_scalars, grid geometry) in shared memory and updates it from
// the same reduced values in the same order, so all blocks take the same
// branches; block 0 writes the replica back at the end.  Grid-wide sums are
// per-block partials reduced by every block in a fixed order: deterministic.
//
// Per-atom arithmetic is the same code as the standalone kernels (built with
// -fmad=false): positions, velocities, accelerations and lists stay
// bit-identical to the serial FP64 reference.
#include <cuda_runtime.h>
#include <stdio.h>

#include "clmd_mixed.cuh"
#include "clmd_system.hpp"

namespace clmd {

constexpr int kPB = 256;          // threads per block
#ifndef CLMD_CYCLE_MINB
#define CLMD_CYCLE_MINB 4         // resident blocks per SM the registers must allow
#endif
constexpr int kRowBufC = 32;      // candidate buffer of the list search
constexpr int kRedSlots = 16;     // partial-sum slots per buffer

struct Geo {
  double rs2, cfx, cfy, cfz;
  int ncx, ncy, ncz, ncell;
  int nox, noy, noz, pad;
  int offx[3], offy[3], offz[3];
};

struct Blk {
  clmd_scalars q;
  Geo g;
  double kf[CLMD_MXSORTS];
  double bcast[4];
  int scale[CLMD_MXSORTS];
  int rebuild;
  int stop;
};

// ---------------------------------------------------------------------------
// grid barrier (co-residency guaranteed by the cooperative launch); every
// wait is bounded and reports CLMD_ERR_TIMEOUT instead of hanging
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool gbar(DevState* st) {
  __shared__ int fail;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* gen = &st->bar_gen;
    unsigned int g = *gen;
    __threadfence();
    unsigned int arrived = atomicAdd(&st->bar_count, 1u);
    fail = 0;
    if (arrived == gridDim.x - 1 + st->bar_extra) {
      atomicExch(&st->bar_count, 0u);
      __threadfence();
      atomicAdd(&st->bar_gen, 1u);
    } else {
      const long long limit = st->bar_limit > 0 ? st->bar_limit : (1ll << 25);
      long long spins = 0;
      while (*gen == g) {
        __nanosleep(32);
        if (++spins > limit) {
          fail = 1;
          // recorded here as well: a rebuild cut short by a timeout leaves
          // the launch through its normal end, which latches err_new
          atomicCAS(&st->err_new, 0, CLMD_ERR_TIMEOUT);
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
  return fail == 0;
}

// partials: buf[slot * nb + block]
__device__ __forceinline__ void put_sum(double* buf, int slot, double v, double* sh) {
  double t = block_sum(v, sh);
  if (threadIdx.x == 0) buf[slot * gridDim.x + blockIdx.x] = t;
}
__device__ __forceinline__ void put_max(double* buf, int slot, double v, double* sh) {
  double t = block_max(v, sh);
  if (threadIdx.x == 0) buf[slot * gridDim.x + blockIdx.x] = t;
}
// every thread of every block gets the same total
__device__ __forceinline__ double get_sum(const double* buf, int slot, double* sh,
                                          double* bc) {
  double v = 0.0;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x)
    v += __ldcg(buf + slot * gridDim.x + k);
  double t = block_sum(v, sh);
  if (threadIdx.x == 0) *bc = t;
  __syncthreads();
  double r = *bc;
  __syncthreads();
  return r;
}
__device__ __forceinline__ double get_max(const double* buf, int slot, double* sh,
                                          double* bc) {
  double v = 0.0;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x)
    v = fmax(v, __ldcg(buf + slot * gridDim.x + k));
  double t = block_max(v, sh);
  if (threadIdx.x == 0) *bc = t;
  __syncthreads();
  double r = *bc;
  __syncthreads();
  return r;
}

// ---------------------------------------------------------------------------
// scalar logic (thread 0 of each block on its replica)
// ---------------------------------------------------------------------------

// neighbor-pbc-mav.f:48-60, 101-105 and the cell grid
static __device__ void prologue(const Params& P, Blk& B, int step) {
  clmd_scalars& q = B.q;
  if (q.dmms > (q.atrskin - P.atrcut)) {  // :48-51
    if (q.status == 0) {
      q.status = CLMD_ERR_SKIN;
      q.fail_step = step;
    }
    B.stop = 1;
    B.rebuild = 0;
    return;
  }
  q.dmmav = (double)(float)q.dmmst * q.dmmsu / 256.0;  // :53
  if (step != P.btim && step > 0) {                      // :55-60
    q.atrskin = P.atrcut + (q.atrskin - P.atrcut) * (double)P.nbtim / (double)q.dmmst;
    q.atrskin = fmin(P.boxx / 2.0, q.atrskin);
    q.atrskin = fmin(P.boxy / 2.0, q.atrskin);
    q.atrskin = fmin(P.boxz / 2.0, q.atrskin);
  }
  Geo& g = B.g;
  g.rs2 = q.atrskin * q.atrskin;
  double side = q.atrskin * (1.0 + 1e-9);
  int n3[3] = {(int)floor(P.boxx / side), (int)floor(P.boxy / side), (int)floor(P.boxz / side)};
  int mx[3] = {P.ncx_max, P.ncy_max, P.ncz_max};
  int* offs[3] = {g.offx, g.offy, g.offz};
  int* nos[3] = {&g.nox, &g.noy, &g.noz};
  for (int d = 0; d < 3; d++) {
    n3[d] = max(1, min(n3[d], mx[d]));
    if (n3[d] >= 3) {
      offs[d][0] = -1; offs[d][1] = 0; offs[d][2] = 1; *nos[d] = 3;
    } else if (n3[d] == 2) {
      offs[d][0] = 0; offs[d][1] = 1; *nos[d] = 2;
    } else {
      offs[d][0] = 0; *nos[d] = 1;
    }
  }
  g.ncx = n3[0];
  g.ncy = n3[1];
  g.ncz = n3[2];
  g.ncell = n3[0] * n3[1] * n3[2];
  g.cfx = (double)g.ncx / P.boxx;
  g.cfy = (double)g.ncy / P.boxy;
  g.cfz = (double)g.ncz / P.boxz;
  q.dmmax = fmax(q.dmms, q.dmmax);  // :101-105
  q.dmms = 0.0;
  q.dmmst = 0;
  q.nrebuild = q.nrebuild + 1;
  q.last_rebuild_step = step;
}

// int-verlet-mav.f:64-74 / int-verlet-nh-mav.f:70-78
static __device__ void skin(const Params& P, Blk& B, double dmmr, int step) {
  clmd_scalars& q = B.q;
  dmmr = 2.2 * sqrt(dmmr);
  q.dmms = q.dmms + dmmr;
  q.dmmsu = q.dmmsu + dmmr - q.dmmh[q.dmmi];
  q.dmmh[q.dmmi] = dmmr;
  q.dmmi = (q.dmmi + 1) & 255;
  q.dmmst = q.dmmst + 1;
  B.rebuild = q.dmms > (q.atrskin - P.atrcut - 2.0 * q.dmms / (double)(float)q.dmmst);
  if (B.rebuild) prologue(P, B, step);
}

// ---------------------------------------------------------------------------
// the list rebuild (neighbor-pbc-mav.f:67-99) as barrier-separated phases
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool nbt(const Params& P, double rs2, const double4& a,
                                    const double4& b) {
  double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
  dx = mimage_nb(dx, P.boxx, P.ibx);
  dy = mimage_nb(dy, P.boxy, P.iby);
  dz = mimage_nb(dz, P.boxz, P.ibz);
  double r2 = dx * dx + dy * dy + dz * dz;
  return r2 <= rs2;
}

// the candidate slots of a cell row: [a0, b0) and, where the x-neighbours
// wrap, [a1, b1) (scalars, not arrays indexed by the range: those would live
// in local memory)
__device__ __forceinline__ int xr(const Geo& g, const int* cs, int row, int cx, int& a0,
                                  int& b0, int& a1, int& b1) {
  int n = g.ncx;
  if (n >= 3) {
    if (cx >= 1 && cx <= n - 2) {
      a0 = cs[row + cx - 1]; b0 = cs[row + cx + 2];
      return 1;
    }
    if (cx == 0) {
      a0 = cs[row]; b0 = cs[row + 2];
      a1 = cs[row + n - 1]; b1 = cs[row + n];
      return 2;
    }
    a0 = cs[row + n - 2]; b0 = cs[row + n];
    a1 = cs[row]; b1 = cs[row + 1];
    return 2;
  }
  a0 = cs[row];
  b0 = cs[row + n];
  return 1;
}

template <bool FILL>
__device__ __forceinline__ int scan_cells(const Params& P, const Geo& g, int p, int refi,
                                          const double4& pi, const double4* pos,
                                          const int* perm, const int* cs, int* bq, int* bref,
                                          int* out) {
  int cx = min((int)(pi.x * g.cfx), g.ncx - 1);
  int cy = min((int)(pi.y * g.cfy), g.ncy - 1);
  int cz = min((int)(pi.z * g.cfz), g.ncz - 1);
  int n = 0;
  for (int a = 0; a < g.noz; a++) {
    int zz = cz + g.offz[a];
    zz += (zz < 0) ? g.ncz : 0;
    zz -= (zz >= g.ncz) ? g.ncz : 0;
    for (int b = 0; b < g.noy; b++) {
      int yy = cy + g.offy[b];
      yy += (yy < 0) ? g.ncy : 0;
      yy -= (yy >= g.ncy) ? g.ncy : 0;
      int row = (zz * g.ncy + yy) * g.ncx;
      int a0, b0, a1 = 0, b1 = 0;
      const int nr = xr(g, cs, row, cx, a0, b0, a1, b1);
      for (int r = 0; r < nr; r++) {
        const int qb = r ? b1 : b0;
        for (int q = r ? a1 : a0; q < qb; q++) {
          if (q == p) continue;
          double4 pq = pos[q];
          int refq = perm[q];
          bool hit = (refi < refq) ? nbt(P, g.rs2, pi, pq) : nbt(P, g.rs2, pq, pi);
          if (hit) {
            if (FILL) {
              out[n] = q;
            } else if (n < kRowBufC) {
              bq[n] = q;
              bref[n] = refq;
            }
            n++;
          }
        }
      }
    }
  }
  return n;
}

struct CycleArgs {
  double4* pos0;
  double4* pos1;
  double *vx, *vy, *vz, *ax, *ay, *az;
  double *vxn, *vyn, *vzn;
  // mixed Nose-Hoover: the accelerations between a step's force pass and its
  // velocity pass, FP32 (the storage of the FP64 sweeps' iterate vxn..vzn,
  // which that path does not use)
  float *afx, *afy, *afz;
  int *perm, *iperm;
  double4* pos_s;
  double *vx_s, *vy_s, *vz_s, *ax_s, *ay_s, *az_s;
  int* perm_s;
  int *cell_count, *cell_start, *cell_fill, *cell_atoms, *atom_cell, *scan_aux;
  int *list, *row_start, *row_len, *row_lo;
  double* red;  // 2 x kRedSlots x gridDim partials
};

// neighbor-pbc-mav.f:67-71
__device__ __forceinline__ double4 wrap_box(const Params& P, double4 v) {
  v.x = fmod(fmod(v.x, P.boxx) + P.boxx, P.boxx);
  v.y = fmod(fmod(v.y, P.boxy) + P.boxy, P.boxy);
  v.z = fmod(fmod(v.z, P.boxz) + P.boxz, P.boxz);
  return v;
}

// The list rebuild, in place: positions wrapped and, with the velocities and
// perm, put in cell order (gathered into pos_s, vx_s.., perm_s; the search
// reads the new order there and copies each slot back as it takes it).
// Returns false if the grid must stop (error).  acc: carry the accelerations
// into the new order too; a rebuild inside the step loop runs between the
// drift (the last reader of a step's accelerations) and the force pass that
// overwrites them, so there they are not moved
static __device__ bool rebuild(const Params& P, DevState* st, Blk& B, const CycleArgs& A,
                               double4* pos, double* sh, bool acc) {
  const int N = P.N;
  const int G = gridDim.x * blockDim.x;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
  const Geo& g = B.g;
  // R1: histogram of the wrapped positions (neighbor-pbc-mav.f:67-71; the
  // gather below stores them wrapped)
  if (t0 == 0) st->list_used = 0ull;
  for (int p = t0; p < N; p += G) {
    const double4 v = wrap_box(P, pos[p]);
    int cx = min((int)(v.x * g.cfx), g.ncx - 1);
    int cy = min((int)(v.y * g.cfy), g.ncy - 1);
    int cz = min((int)(v.z * g.cfz), g.ncz - 1);
    int c = (cz * g.ncy + cy) * g.ncx + cx;
    A.atom_cell[p] = c;
    atomicAdd(&A.cell_count[c], 1);
  }
  if (!gbar(st)) return false;
  // R2: tile sums
  const int ncell = g.ncell;
  const int ntiles = (ncell + kScanTile - 1) / kScanTile;
  constexpr int per = kScanTile / kPB;
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    int base = b * kScanTile, s = 0;
    for (int k = 0; k < per; k++) {
      int c = base + threadIdx.x * per + k;
      if (c < ncell) s += A.cell_count[c];
    }
    double t = block_sum((double)s, sh);
    if (threadIdx.x == 0) A.scan_aux[b] = (int)t;
  }
  if (!gbar(st)) return false;
  // R3: offsets of each tile, exclusive scan inside it, counts cleared
  __shared__ int ssh[33];
  for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    double pre = 0.0;
    for (int k = threadIdx.x; k < b; k += blockDim.x) pre += (double)__ldcg(A.scan_aux + k);
    double pt = block_sum(pre, sh);
    __shared__ int tile_off;
    if (threadIdx.x == 0) tile_off = (int)pt;
    __syncthreads();
    int base = b * kScanTile;
    int loc[per];
    int s = 0;
    for (int k = 0; k < per; k++) {
      int c = base + threadIdx.x * per + k;
      loc[k] = c < ncell ? A.cell_count[c] : 0;
      s += loc[k];
    }
    // block exclusive scan of s
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) ssh[w] = incl;
    __syncthreads();
    if (w == 0) {
      int v = lane < nw ? ssh[lane] : 0;
      int vi = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, vi, o);
        if (lane >= o) vi += t;
      }
      if (lane < nw) ssh[lane] = vi - v;
    }
    __syncthreads();
    int ex = tile_off + ssh[w] + incl - s;
    for (int k = 0; k < per; k++) {
      int c = base + threadIdx.x * per + k;
      if (c < ncell) {
        A.cell_start[c] = ex;
        A.cell_fill[c] = ex;
        A.cell_count[c] = 0;
      }
      ex += loc[k];
    }
    __syncthreads();
  }
  if (t0 == 0) A.cell_start[ncell] = N;
  if (!gbar(st)) return false;
  // R4: counting-sort scatter
  for (int p = t0; p < N; p += G) {
    int slot = atomicAdd(&A.cell_fill[A.atom_cell[p]], 1);
    A.cell_atoms[slot] = p;
  }
  if (!gbar(st)) return false;
  // R5: per cell: order by reference index, gather into scratch
  for (int c = t0; c < ncell; c += G) {
    int c0 = A.cell_start[c], c1 = A.cell_start[c + 1];
    for (int a = c0 + 1; a < c1; a++) {
      int key = A.cell_atoms[a], kr = A.perm[key];
      int b = a - 1;
      while (b >= c0 && A.perm[A.cell_atoms[b]] > kr) {
        A.cell_atoms[b + 1] = A.cell_atoms[b];
        b--;
      }
      A.cell_atoms[b + 1] = key;
    }
    for (int q = c0; q < c1; q++) {
      int o = A.cell_atoms[q];
      A.pos_s[q] = wrap_box(P, pos[o]);
      A.vx_s[q] = A.vx[o];
      A.vy_s[q] = A.vy[o];
      A.vz_s[q] = A.vz[o];
      if (acc) {
        A.ax_s[q] = A.ax[o];
        A.ay_s[q] = A.ay[o];
        A.az_s[q] = A.az[o];
      }
      A.perm_s[q] = A.perm[o];
    }
  }
  if (!gbar(st)) return false;
  // R6: rows (neighbor-pbc-mav.f:73-99), warp-aligned grid-stride, over the
  // new order in the scratch arrays; each slot is committed (copied back)
  // by the thread that takes it
  const double4* npos = A.pos_s;
  const int* perm = A.perm_s;
  const int lane = threadIdx.x & 31;
  for (int base0 = t0 - lane; base0 < N; base0 += G) {
    int p = base0 + lane;
    bool active = p < N;
    int cnt = 0, refi = 0;
    double4 pi = make_double4(0, 0, 0, 0);
    int bq[kRowBufC], bref[kRowBufC];
    if (active) {
      pi = npos[p];
      refi = perm[p];
      pos[p] = pi;
      A.vx[p] = A.vx_s[p];
      A.vy[p] = A.vy_s[p];
      A.vz[p] = A.vz_s[p];
      if (acc) {
        A.ax[p] = A.ax_s[p];
        A.ay[p] = A.ay_s[p];
        A.az[p] = A.az_s[p];
      }
      A.perm[p] = refi;
      A.iperm[refi] = p;
      cnt = scan_cells<false>(P, g, p, refi, pi, npos, perm, A.cell_start, bq, bref, nullptr);
    }
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    unsigned long long wbase = 0;
    if (lane == 31) wbase = atomicAdd(&st->list_used, (unsigned long long)incl);
    wbase = __shfl_sync(0xffffffffu, wbase, 31);
    if (!active) continue;
    unsigned long long start = wbase + (unsigned long long)(incl - cnt);
    if (start + (unsigned long long)cnt > (unsigned long long)P.list_cap) {
      raise_err(st, CLMD_ERR_LIST_OVERFLOW);
      A.row_start[p] = 0;
      A.row_len[p] = 0;
      A.row_lo[p] = 0;
      continue;
    }
    int* row = A.list + start;
    int lo = 0;
    if (cnt <= kRowBufC) {
      for (int a = 1; a < cnt; a++) {
        int kr = bref[a], kq = bq[a];
        int b = a - 1;
        while (b >= 0 && bref[b] > kr) {
          bref[b + 1] = bref[b];
          bq[b + 1] = bq[b];
          b--;
        }
        bref[b + 1] = kr;
        bq[b + 1] = kq;
      }
      for (int a = 0; a < cnt; a++) {
        row[a] = bq[a];
        lo += bref[a] < refi;
      }
    } else {
      scan_cells<true>(P, g, p, refi, pi, npos, perm, A.cell_start, nullptr, nullptr, row);
      for (int a = 1; a < cnt; a++) {
        int kq = row[a], kr = perm[kq];
        int b = a - 1;
        while (b >= 0 && perm[row[b]] > kr) {
          row[b + 1] = row[b];
          b--;
        }
        row[b + 1] = kq;
      }
      for (int a = 0; a < cnt; a++) lo += perm[row[a]] < refi;
    }
    A.row_start[p] = (int)start;
    A.row_len[p] = cnt;
    A.row_lo[p] = lo;
  }
  if (!gbar(st)) return false;
  // neighbor-pbc-mav.f:95-97: the half list's write cursor after the last
  // row (1 + natom headers + half pairs) plus natom must stay within mxnlist
  const bool full = P.half_cap > 0 &&
                    (long long)(__ldcg(&st->list_used) / 2ull) + 2LL * P.N + 1 > P.half_cap;
  if (__ldcg(&st->err_new) != 0 || full) {
    if (threadIdx.x == 0 && B.q.status == 0) {
      B.q.status = CLMD_ERR_LIST_OVERFLOW;
      B.q.fail_step = st->cur_step;
    }
    return false;
  }
  return true;
}

// for-a-lj-n-pbc-m.f:92-142 for one atom: fsum in the reference's order
// (accumulated by warp_forces below)
struct Pair {
  double fx, fy, fz, esum, vir;
};

// Pair forces, warp-cooperative, for the 32 consecutive slots of a warp, whose
// rows are contiguous in the list (the search allocates them with one
// warp-wide cursor step).  Lanes evaluate the pair terms of 32 consecutive
// list entries at a time (balanced work whatever the row lengths), stage them
// in shared memory, and each owner lane then adds its own terms in list
// order, i.e. in the reference's order, with the same +/- as the serial code.
// FP64: the terms of kGroup chunks are staged before the owner lanes add
// theirs, so that more owners work at once (a row's terms still go in
// list order)
#ifndef CLMD_FORCE_GROUP
#define CLMD_FORCE_GROUP 4
#endif
constexpr int kGroup = CLMD_FORCE_GROUP;
struct WarpStage {
  double tx[32 * kGroup], ty[32 * kGroup], tz[32 * kGroup];
  int flag[32 * kGroup];  // 0 nothing, 1 add, 2 subtract
};

template <bool MIXED>
__device__ __forceinline__ void warp_forces(const Params& P, DevState* st, const double4* pos,
                                            const int* list, int st0, int len, int lo,
                                            const double4& pa, double bf1, double bf2,
                                            double& fx, double& fy, double& fz, double& esum,
                                            double& vir, WarpStage& W) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int e = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(FULL, e, o);
    if (lane >= o) e += t;
  }
  const int tot = __shfl_sync(FULL, e, 31);
  e -= len;  // exclusive prefix: this lane's row starts at wbase + e
  const int wbase = __shfl_sync(FULL, st0, 0);
  const int sa = (int)pa.w;
  constexpr bool mixed = MIXED;
  float sx = 0.f, sy = 0.f, sz = 0.f, kx = 0.f, ky = 0.f, kz = 0.f;  // mixed: Kahan sums
  fx = 0.0;
  fy = 0.0;
  fz = 0.0;
  // this chunk's entry and neighbour position are fetched first, and the
  // next chunk's entry with them, so that the loads overlap the owner search
  int jnext = lane < tot ? list[wbase + lane] : 0;
  for (int c = 0; c < tot; c += 32) {
    const int k = c + lane;
    const int kk = k < tot ? k : tot - 1;
    const int jc = jnext;
    double4 pb = make_double4(0.0, 0.0, 0.0, 0.0);
    if (k < tot) pb = pos[jc];
    if (k + 32 < tot) jnext = list[wbase + k + 32];
    int ow = 0;
#pragma unroll
    for (int sft = 16; sft >= 1; sft >>= 1) {
      int cand = ow + sft;
      int ec = __shfl_sync(FULL, e, cand & 31);
      if (cand <= 31 && ec <= kk) ow = cand;
    }
    const double ox = __shfl_sync(FULL, pa.x, ow);
    const double oy = __shfl_sync(FULL, pa.y, ow);
    const double oz = __shfl_sync(FULL, pa.z, ow);
    const int osp = __shfl_sync(FULL, sa, ow);
    const int oe = __shfl_sync(FULL, e, ow);
    const int olo = __shfl_sync(FULL, lo, ow);
    int flag = 0;
    double tx = 0.0, ty = 0.0, tz = 0.0;
    if (k < tot) {
      bool own = (k - oe) >= olo;  // neighbour has the larger reference index
      double dx, dy, dz;
      if (own) {
        dx = ox - pb.x; dy = oy - pb.y; dz = oz - pb.z;
      } else {
        dx = pb.x - ox; dy = pb.y - oy; dz = pb.z - oz;
      }
      dx = mimage_bf(dx, P.boxx, P.ibx, bf1, bf2);
      dy = mimage_bf(dy, P.boxy, P.iby, bf1, bf2);
      dz = mimage_bf(dz, P.boxz, P.ibz, bf1, bf2);
      double rij2 = dx * dx + dy * dy + dz * dz;
      if (rij2 <= P.atr2) {
        double r2 = rij2;
        double rij6 = 0.0;
        if (!mixed) {
          rij2 = 1.0 / rij2;
          rij6 = rij2 * rij2 * rij2;
        }
        int ij = osp + (int)pb.w;
        if (ij < 2 || ij > 4) {
          raise_err(st, CLMD_ERR_BAD_SPECIES);
        } else if (mixed) {
          double e, w;
          pair_term_f32(P, ij, r2, dx, dy, dz, tx, ty, tz, e, w);
          if (own) {
            esum = esum + e;
            vir = vir + w;
            flag = 1;
          } else {
            flag = 2;
          }
        } else {
          double fij = pair_fij(P, ij, rij2, rij6);
          tx = fij * dx;
          ty = fij * dy;
          tz = fij * dz;
          if (own) {
            esum = esum + pair_e(P, ij, rij6);
            vir = vir + fij * r2;
            flag = 1;
          } else {
            flag = 2;
          }
        }
      }
    }
    const int a0 = e > c ? e : c;
    const int a1 = (e + len) < (c + 32) ? (e + len) : (c + 32);
    if (mixed) {
      // each row's terms in this chunk summed by a segmented scan across the
      // lanes (a fixed tree: deterministic), then added to the owner's
      // Kahan sums chunk by chunk: every lane works, where the ordered
      // FP64 sum below has only the owners working
      const float sg = flag == 1 ? 1.0f : (flag == 2 ? -1.0f : 0.0f);
      float v0 = sg * (float)tx, v1 = sg * (float)ty, v2 = sg * (float)tz;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int ou = __shfl_up_sync(FULL, ow, off);
        const float u0 = __shfl_up_sync(FULL, v0, off);
        const float u1 = __shfl_up_sync(FULL, v1, off);
        const float u2 = __shfl_up_sync(FULL, v2, off);
        if (lane >= off && ou == ow) {
          v0 = __fadd_rn(v0, u0);
          v1 = __fadd_rn(v1, u1);
          v2 = __fadd_rn(v2, u2);
        }
      }
      const int last = a1 > a0 ? a1 - 1 - c : 0;  // my row's last entry in the chunk
      const float p0 = __shfl_sync(FULL, v0, last);
      const float p1 = __shfl_sync(FULL, v1, last);
      const float p2 = __shfl_sync(FULL, v2, last);
      if (a1 > a0) {
        kahan_add(sx, kx, p0);
        kahan_add(sy, ky, p1);
        kahan_add(sz, kz, p2);
      }
      continue;
    }
    const int g = (c >> 5) % kGroup;
    W.tx[32 * g + lane] = tx;
    W.ty[32 * g + lane] = ty;
    W.tz[32 * g + lane] = tz;
    W.flag[32 * g + lane] = flag;
    if (g != kGroup - 1 && c + 32 < tot) continue;  // the group is not full yet
    __syncwarp();
    const int cg = c - 32 * g;  // the group's first entry
    const int b0 = e > cg ? e : cg;
    const int b1 = (e + len) < (c + 32) ? (e + len) : (c + 32);
    for (int a = b0; a < b1; a++) {
      int q = a - cg;
      int f = W.flag[q];
      if (f == 1) {
        fx = fx + W.tx[q];
        fy = fy + W.ty[q];
        fz = fz + W.tz[q];
      } else if (f == 2) {
        fx = fx - W.tx[q];
        fy = fy - W.ty[q];
        fz = fz - W.tz[q];
      }
    }
    __syncwarp();
  }
  if (mixed) {
    fx = (double)sx;
    fy = (double)sy;
    fz = (double)sz;
  }
}

__device__ __forceinline__ int sp_block(const Params& P, int ref) {
  for (int s = 0; s < P.atsorts; s++)
    if (ref >= P.sp_start[s] && ref < P.sp_start[s + 1]) return s;
  return -1;
}

enum { SLOT_MAX = 0, SLOT_SUMV2 = 1, SLOT_EPOT = 2, SLOT_VIR = 3, SLOT_EKIN = 4,
       SLOT_DELPS = 5, SLOT_NR = 6, SLOT_EK0 = 6 /* ek per species: 6..15 */ };

template <bool NH, bool THERMO, bool MIXED>
__global__ void __launch_bounds__(kPB, CLMD_CYCLE_MINB) k_cycle(Params P, DevState* st,
                                                                CycleArgs A, int nsteps,
                                                                int mode) {
  if (gated(st)) return;
  __shared__ Blk B;
  __shared__ double sh[kPB / 32];
  const int N = P.N;
  const int G = gridDim.x * blockDim.x;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
  constexpr bool nh = NH;
  constexpr bool thermo = THERMO;
  const double dt = P.dt;
  if (threadIdx.x == 0) {
    B.q = st->s;
    B.g.rs2 = st->rs2;
    B.g.cfx = st->cfx; B.g.cfy = st->cfy; B.g.cfz = st->cfz;
    B.g.ncx = st->ncx; B.g.ncy = st->ncy; B.g.ncz = st->ncz; B.g.ncell = st->ncell;
    B.g.nox = st->nox; B.g.noy = st->noy; B.g.noz = st->noz;
    for (int d = 0; d < 3; d++) {
      B.g.offx[d] = st->offx[d]; B.g.offy[d] = st->offy[d]; B.g.offz[d] = st->offz[d];
    }
    B.stop = 0;
    B.rebuild = 0;
  }
  __syncthreads();
  int step = st->cur_step;
  int cur = 0;  // positions of the current step live in pos0 / pos1
  auto posb = [&](int k) { return k ? A.pos1 : A.pos0; };
  int rb = 0;  // partial-buffer toggle
  auto red = [&]() { return A.red + (size_t)rb * kRedSlots * gridDim.x; };

  if (mode == 1) {
    // neighbor(step) called directly: a forced rebuild
    if (threadIdx.x == 0) {
      B.rebuild = 1;
      prologue(P, B, step);
    }
    __syncthreads();
    if (!B.stop) rebuild(P, st, B, A, posb(0), sh, true);
    goto done;
  }

  {
    bool drift_done = false;  // the current step's drift already ran (fused)
    const double psi0 = B.q.psi;
    (void)psi0;
    for (int s = 0; s < nsteps; s++, step++) {
      const bool last = (s == nsteps - 1);
      if (!drift_done) {
        // ---- velocity scaling (scalev-nh-m.f), main.f:207, before the step
        if (thermo) {
          for (int sp = 0; sp < P.atsorts; sp++) {
            double e = 0.0;
            for (int p = t0; p < N; p += G) {
              int b = sp_block(P, A.perm[p]);
              if (b == sp)
                e = e + 0.5 * P.apmas[sp] * (A.vx[p] * A.vx[p] + A.vy[p] * A.vy[p] +
                                             A.vz[p] * A.vz[p]);
            }
            put_sum(red(), SLOT_EK0 + sp, e, sh);
          }
          if (!gbar(st)) goto timeout;
          for (int sp = 0; sp < P.atsorts; sp++) {
            double ek = get_sum(red(), SLOT_EK0 + sp, sh, B.bcast);
            if (threadIdx.x == 0) {
              B.kf[sp] = sqrt(P.ekinT[sp] / ek);
              B.scale[sp] = (P.apth[sp] == 'X');
            }
          }
          __syncthreads();
          rb ^= 1;
        }
        // ---- drift (int-verlet-mav.f:44-56 / int-verlet-nh-mav.f:49-61)
        double d2 = 0.0, sv = 0.0;
        const double psi = B.q.psi;
        const double dt2 = dt * dt / 2, dth = dt / 2;
        double4* pos = posb(cur);
        for (int p = t0; p < N; p += G) {
          double vxi = A.vx[p], vyi = A.vy[p], vzi = A.vz[p];
          if (thermo) {
            int b = sp_block(P, A.perm[p]);
            if (b >= 0 && B.scale[b]) {
              double kf = B.kf[b];
              vxi = vxi * kf;
              vyi = vyi * kf;
              vzi = vzi * kf;
            }
          }
          double4 q = pos[p];
          double axi = A.ax[p], ayi = A.ay[p], azi = A.az[p];
          double dx, dy, dz;
          if (!nh) {
            double hx = 0.5 * axi * dt, hy = 0.5 * ayi * dt, hz = 0.5 * azi * dt;
            dx = (vxi + hx) * dt;
            dy = (vyi + hy) * dt;
            dz = (vzi + hz) * dt;
            vxi = vxi + hx;
            vyi = vyi + hy;
            vzi = vzi + hz;
          } else {
            dx = dt * vxi + dt2 * (axi - psi * vxi);
            dy = dt * vyi + dt2 * (ayi - psi * vyi);
            dz = dt * vzi + dt2 * (azi - psi * vzi);
            sv = sv + vxi * vxi + vyi * vyi + vzi * vzi;
            vxi = vxi + dth * (axi - psi * vxi);
            vyi = vyi + dth * (ayi - psi * vyi);
            vzi = vzi + dth * (azi - psi * vzi);
          }
          q.x = q.x + dx;
          q.y = q.y + dy;
          q.z = q.z + dz;
          pos[p] = q;
          A.vx[p] = vxi;
          A.vy[p] = vyi;
          A.vz[p] = vzi;
          d2 = fmax(d2, dx * dx + dy * dy + dz * dz);
        }
        put_max(red(), SLOT_MAX, d2, sh);
        if (nh) put_sum(red(), SLOT_SUMV2, sv, sh);
        if (!gbar(st)) goto timeout;
      }
      // ---- scalars after the drift: NH s/PSI half step, skin decision
      {
        double dmmr = get_max(red(), SLOT_MAX, sh, B.bcast);
        double sumv2 = nh ? get_sum(red(), SLOT_SUMV2, sh, B.bcast) : 0.0;
        if (threadIdx.x == 0) {
          if (nh) {
            clmd_scalars& q = B.q;
            const double dt2 = dt * dt / 2, dth = dt / 2;
            q.sumv2 = sumv2;
            if (P.ethst == 'N') {  // int-verlet-nh-mav.f:64-67
              q.s = q.s + q.psi * dt + (P.apmas[0] * q.sumv2 - P.nkt3_d) * dt2 / P.Q;
              q.psi = q.psi + (P.apmas[0] * q.sumv2 - P.nkt3_d) * dth / P.Q;
            }
          }
          skin(P, B, dmmr, step);
        }
        __syncthreads();
        rb ^= 1;
        if (B.stop) goto done;
        if (B.rebuild) {
          if (!rebuild(P, st, B, A, posb(cur), sh, false)) goto stop_or_timeout;
        }
      }
      // ---- forces (+ kick, + next drift)
      {
        double4* pos = posb(cur);
        double4* nxt = posb(cur ^ 1);
        const double bf1 = 2.0 + (double)(int)(B.q.atrskin / P.sig1);
        const double bf2 = bf1 + 0.5;
        const bool fuse = !nh && !thermo && !last;
        // mixed Nose-Hoover: the velocity pass fuses the next drift unless
        // this is the launch's last step or velocities are rescaled first
        const bool keep64 = last || thermo;
        (void)keep64;
        double esum = 0.0, vir = 0.0, ek = 0.0, d2 = 0.0, dp = 0.0, sv = 0.0;
        const double psi = B.q.psi;
        const double dth = dt / 2, m = P.apmas[0], Q = P.Q;
        __shared__ WarpStage stage[kPB / 32];
        WarpStage& W = stage[threadIdx.x >> 5];
        const int lane = threadIdx.x & 31;
        for (int base0 = t0 - lane; base0 < N; base0 += G) {
          const int p = base0 + lane;
          const bool act = p < N;
          double4 pa = act ? pos[p] : make_double4(0.0, 0.0, 0.0, 1.0);
          Pair f;
          f.esum = 0.0;
          f.vir = 0.0;
          // lane 0 is active whenever the warp is; only its row start is used
          warp_forces<MIXED>(P, st, pos, A.list, lane == 0 ? A.row_start[p] : 0,
                      act ? A.row_len[p] : 0,
                      act ? A.row_lo[p] : 0, pa, bf1, bf2, f.fx, f.fy, f.fz, f.esum, f.vir, W);
          // lanes past N still evaluated pair terms of their warp's atoms
          esum = esum + f.esum;
          vir = vir + f.vir;
          if (!act) continue;
          int sa = (int)pa.w;
          double iatm = 1.0 / P.apmas[sa - 1];
          // int-verlet-mav.f:76-84: a = 0, AccAtom adds fsum/m
          double axi = 0.0 + f.fx * iatm, ayi = 0.0 + f.fy * iatm, azi = 0.0 + f.fz * iatm;
          if (MIXED && nh) {
            // FP32 accelerations (the pair terms' precision); FP64 in the
            // state only where the next reader is an unfused drift
            const float fx32 = (float)axi, fy32 = (float)ayi, fz32 = (float)azi;
            axi = fx32;
            ayi = fy32;
            azi = fz32;
            if (keep64) {
              A.ax[p] = axi;
              A.ay[p] = ayi;
              A.az[p] = azi;
            } else {
              A.afx[p] = fx32;
              A.afy[p] = fy32;
              A.afz[p] = fz32;
            }
          } else {
            A.ax[p] = axi;
            A.ay[p] = ayi;
            A.az[p] = azi;
          }
          if (!nh) {
            // :86-92
            double vxi = A.vx[p] + 0.5 * axi * dt;
            double vyi = A.vy[p] + 0.5 * ayi * dt;
            double vzi = A.vz[p] + 0.5 * azi * dt;
            if (last || thermo)
              ek = ek + 0.5 * P.apmas[sa - 1] * (vxi * vxi + vyi * vyi + vzi * vzi);
            if (fuse) {
              // next step's drift (:44-56)
              double hx = 0.5 * axi * dt, hy = 0.5 * ayi * dt, hz = 0.5 * azi * dt;
              double dx = (vxi + hx) * dt, dy = (vyi + hy) * dt, dz = (vzi + hz) * dt;
              double4 q = pa;
              q.x = q.x + dx;
              q.y = q.y + dy;
              q.z = q.z + dz;
              nxt[p] = q;
              vxi = vxi + hx;
              vyi = vyi + hy;
              vzi = vzi + hz;
              d2 = fmax(d2, dx * dx + dy * dy + dz * dz);
            }
            A.vx[p] = vxi;
            A.vy[p] = vyi;
            A.vz[p] = vzi;
          } else if (MIXED) {
            // closed-form solve (clmd_nh_root): sv = sum W^2, W = V + dth a
            // (the velocity pass forms W again from V and a)
            double wx = A.vx[p] + dth * axi, wy = A.vy[p] + dth * ayi, wz = A.vz[p] + dth * azi;
            sv = sv + wx * wx + wy * wy + wz * wz;
          } else {
            // int-verlet-nh-mav.f:94-120: vn = V, sumv2, first sweep's delps
            double vxi = A.vx[p], vyi = A.vy[p], vzi = A.vz[p];
            A.vxn[p] = vxi;
            A.vyn[p] = vyi;
            A.vzn[p] = vzi;
            sv = sv + vxi * vxi + vyi * vyi + vzi * vzi;
            double b = -dth * (axi - psi * vxi) - (vxi - vxi);
            dp = dp + b * m * vxi * dt / Q;
            b = -dth * (ayi - psi * vyi) - (vyi - vyi);
            dp = dp + b * m * vyi * dt / Q;
            b = -dth * (azi - psi * vzi) - (vzi - vzi);
            dp = dp + b * m * vzi * dt / Q;
          }
        }
        if (last) {
          put_sum(red(), SLOT_EPOT, esum, sh);
          put_sum(red(), SLOT_VIR, vir, sh);
          if (!nh) put_sum(red(), SLOT_EKIN, ek, sh);
        }
        if (fuse) put_max(red(), SLOT_MAX, d2, sh);
        if (nh) {
          put_sum(red(), SLOT_SUMV2, sv, sh);
          put_sum(red(), SLOT_DELPS, dp, sh);
        }
        if (!gbar(st)) goto timeout;
        if (__ldcg(&st->err_new) != 0) {
          if (threadIdx.x == 0 && B.q.status == 0) {
            B.q.status = __ldcg(&st->err_new);
            B.q.fail_step = step;
          }
          goto done;
        }
        if (last) {
          double e = get_sum(red(), SLOT_EPOT, sh, B.bcast);
          double w = get_sum(red(), SLOT_VIR, sh, B.bcast);
          double k = nh ? 0.0 : get_sum(red(), SLOT_EKIN, sh, B.bcast);
          if (threadIdx.x == 0) {
            B.q.epot = e;
            B.q.virial = w;
            if (!nh) B.q.ekin = k;
          }
        }
        if (fuse) {
          cur ^= 1;
          drift_done = true;
        } else {
          drift_done = false;
        }
        if (!nh) {
          // the fused drift's reduction stays in this buffer for the
          // decision of the next step
          if (!fuse) rb ^= 1;
          continue;
        }
      }
      // ---- Nose-Hoover implicit solve (int-verlet-nh-mav.f:105-180)
      {
        const double dt2 = dt * dt / 2, dth = dt / 2, m = P.apmas[0], Q = P.Q;
        const double err = 1.0e-10;
        const double psi = B.q.psi;
        double sumv2 = get_sum(red(), SLOT_SUMV2, sh, B.bcast);
        double draw = get_sum(red(), SLOT_DELPS, sh, B.bcast);
        rb ^= 1;
        if (MIXED) {
          // every block solves the same scalar equation from the same sums
          double pn;
          if (!clmd_nh_root(m * sumv2, psi, P.nkt3_i, dth, Q, pn)) {
            if (threadIdx.x == 0 && B.q.status == 0) {
              B.q.status = CLMD_ERR_NH_NOCONVERGE;
              B.q.fail_step = step;
            }
            __syncthreads();
            goto done;
          }
          // v = W c, fused with the next step's drift (the same expressions
          // as the drift at the top of the step, PSI = pn) unless this is the
          // launch's last step or velocities are rescaled before each step
          const double c = 1.0 / (1.0 + dth * pn);
          const bool fuse = !thermo && !last;
          double d2 = 0.0, sv = 0.0;
          double4* pos = posb(cur);
          for (int p = t0; p < N; p += G) {
            double axi, ayi, azi;
            if (fuse) {
              axi = A.afx[p];
              ayi = A.afy[p];
              azi = A.afz[p];
            } else {
              axi = A.ax[p];
              ayi = A.ay[p];
              azi = A.az[p];
            }
            double vxi = (A.vx[p] + dth * axi) * c, vyi = (A.vy[p] + dth * ayi) * c,
                   vzi = (A.vz[p] + dth * azi) * c;
            if (fuse) {
              double dx = dt * vxi + dt2 * (axi - pn * vxi);
              double dy = dt * vyi + dt2 * (ayi - pn * vyi);
              double dz = dt * vzi + dt2 * (azi - pn * vzi);
              sv = sv + vxi * vxi + vyi * vyi + vzi * vzi;
              vxi = vxi + dth * (axi - pn * vxi);
              vyi = vyi + dth * (ayi - pn * vyi);
              vzi = vzi + dth * (azi - pn * vzi);
              double4 q = pos[p];
              q.x = q.x + dx;
              q.y = q.y + dy;
              q.z = q.z + dz;
              pos[p] = q;
              d2 = fmax(d2, dx * dx + dy * dy + dz * dz);
            }
            A.vx[p] = vxi;
            A.vy[p] = vyi;
            A.vz[p] = vzi;
          }
          if (threadIdx.x == 0) {
            B.q.nh_iters = 1;
            B.q.sumv2 = sumv2 * c * c;
            B.q.psi = pn;
            B.q.ekin = 0.5 * m * B.q.sumv2;
          }
          if (fuse) {
            // the forces' reads of pos ended at the barrier before the root
            put_max(red(), SLOT_MAX, d2, sh);
            put_sum(red(), SLOT_SUMV2, sv, sh);
            if (!gbar(st)) goto timeout;
            drift_done = true;
          } else {
            __syncthreads();
            drift_done = false;
          }
          continue;
        }
        double psn = psi;
        int ready = 0, iter;
        for (iter = 1; iter <= 1000; iter++) {
          double pso = psn;
          double di = -(pso * dth + 1);
          double delps = draw - di * ((-m * sumv2 + P.nkt3_i) * dth / Q - (psi - pso));
          delps = delps / (-dt2 * m * sumv2 / Q + di);
          double pnext = pso + delps;
          double s2 = 0.0, dp = 0.0;
          int notready = 0;
          for (int p = t0; p < N; p += G) {
            double V[3] = {A.vx[p], A.vy[p], A.vz[p]};
            double a[3] = {A.ax[p], A.ay[p], A.az[p]};
            double* vn[3] = {A.vxn, A.vyn, A.vzn};
            double nv[3];
#pragma unroll
            for (int d = 0; d < 3; d++) {
              double vo = vn[d][p];
              double b = -dth * (a[d] - pso * vo) - (V[d] - vo);
              double nx = vo + (b + dth * vo * delps) / di;
              if (fabs((nx - vo) / nx) > err) notready = 1;
              nv[d] = nx;
            }
#pragma unroll
            for (int d = 0; d < 3; d++) {
              vn[d][p] = nv[d];
              s2 = s2 + nv[d] * nv[d];
            }
            // the next sweep's delps terms (:110-120 with vo = this vn)
#pragma unroll
            for (int d = 0; d < 3; d++) {
              double b = -dth * (a[d] - pnext * nv[d]) - (V[d] - nv[d]);
              dp = dp + b * m * nv[d] * dt / Q;
            }
          }
          put_sum(red(), SLOT_SUMV2, s2, sh);
          put_sum(red(), SLOT_DELPS, dp, sh);
          put_max(red(), SLOT_NR, (double)notready, sh);
          if (!gbar(st)) goto timeout;
          sumv2 = get_sum(red(), SLOT_SUMV2, sh, B.bcast);
          draw = get_sum(red(), SLOT_DELPS, sh, B.bcast);
          double nr = get_max(red(), SLOT_NR, sh, B.bcast);
          rb ^= 1;
          psn = pnext;
          if (nr == 0.0) {
            ready = 1;
            break;
          }
        }
        if (threadIdx.x == 0) B.q.nh_iters = ready ? iter : 1000;
        if (!ready) {
          if (threadIdx.x == 0 && B.q.status == 0) {
            B.q.status = CLMD_ERR_NH_NOCONVERGE;
            B.q.fail_step = step;
          }
          __syncthreads();
          goto done;
        }
        // :171-180 write back (sumv2 of V = vn: same sum)
        for (int p = t0; p < N; p += G) {
          A.vx[p] = A.vxn[p];
          A.vy[p] = A.vyn[p];
          A.vz[p] = A.vzn[p];
        }
        if (threadIdx.x == 0) {
          B.q.sumv2 = sumv2;
          B.q.psi = psn;
          B.q.ekin = 0.5 * m * sumv2;
        }
        __syncthreads();
        drift_done = false;
        // the next drift reads only this atom's v: no barrier needed
      }
    }
  }
  goto done;
stop_or_timeout:
  goto done;
timeout:
  if (threadIdx.x == 0) atomicCAS(&st->s.status, 0, CLMD_ERR_TIMEOUT);
  return;
done:
  // positions back in pos0, then block 0 publishes its replica
  if (cur == 1)
    for (int p = t0; p < N; p += G) A.pos0[p] = A.pos1[p];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    clmd_scalars q = B.q;
    q.npairs_half = (long long)(st->list_used / 2ull);
    // err_new stays set (other blocks may still read it); the status latches it
    int err = __ldcg(&st->err_new);
    if (err && q.status == 0) {
      q.status = err;
      q.fail_step = step;
    }
    st->s = q;
    st->cur_step = (mode == 1) ? st->cur_step : step;
    st->rs2 = B.g.rs2;
    st->cfx = B.g.cfx; st->cfy = B.g.cfy; st->cfz = B.g.cfz;
    st->ncx = B.g.ncx; st->ncy = B.g.ncy; st->ncz = B.g.ncz; st->ncell = B.g.ncell;
    st->nox = B.g.nox; st->noy = B.g.noy; st->noz = B.g.noz;
    for (int d = 0; d < 3; d++) {
      st->offx[d] = B.g.offx[d]; st->offy[d] = B.g.offy[d]; st->offz[d] = B.g.offz[d];
    }
  }
}

// This file is compiled twice: as is (the FP64 kernels and the host side)
// and with CLMD_CYCLE_MIXED (the mixed-precision kernels only).  In one
// translation unit the two sets got larger local frames and ran ~4% slower.
typedef void (*CycleKernel)(Params, DevState*, CycleArgs, int, int);

#ifdef CLMD_CYCLE_MIXED
CycleKernel cycle_kernel_mixed(bool nh, bool th) {
  if (nh) return th ? k_cycle<true, true, true> : k_cycle<true, false, true>;
  return th ? k_cycle<false, true, true> : k_cycle<false, false, true>;
}
#else
CycleKernel cycle_kernel_mixed(bool nh, bool th);

static CycleArgs cycle_args(clmd_system* S) {
  CycleArgs A;
  A.pos0 = S->pos;
  A.pos1 = S->pos_alt;
  A.vx = S->vx; A.vy = S->vy; A.vz = S->vz;
  A.ax = S->ax; A.ay = S->ay; A.az = S->az;
  A.vxn = S->vxn; A.vyn = S->vyn; A.vzn = S->vzn;
  A.afx = reinterpret_cast<float*>(S->vxn);
  A.afy = reinterpret_cast<float*>(S->vyn);
  A.afz = reinterpret_cast<float*>(S->vzn);
  A.perm = S->perm; A.iperm = S->iperm;
  A.pos_s = S->pos_s;
  A.vx_s = S->vx_s; A.vy_s = S->vy_s; A.vz_s = S->vz_s;
  A.ax_s = S->ax_s; A.ay_s = S->ay_s; A.az_s = S->az_s;
  A.perm_s = S->perm_s;
  A.cell_count = S->cell_count; A.cell_start = S->cell_start; A.cell_fill = S->cell_fill;
  A.cell_atoms = S->cell_atoms; A.atom_cell = S->atom_cell; A.scan_aux = S->scan_aux;
  A.list = S->list; A.row_start = S->row_start; A.row_len = S->row_len; A.row_lo = S->row_lo;
  A.red = S->red;
  return A;
}

static CycleKernel cycle_kernel(const clmd_system* S) {
  bool nh = S->P.integrator == CLMD_INT_NOSE, th = S->P.ethst == 'X';
  if (S->P.precision == CLMD_PREC_MIXED) return cycle_kernel_mixed(nh, th);
  if (nh) return th ? k_cycle<true, true, false> : k_cycle<true, false, false>;
  return th ? k_cycle<false, true, false> : k_cycle<false, false, false>;
}

int cycle_blocks_for(clmd_system* S) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cycle_kernel(S), kPB, 0);
  if (per_sm < 1) per_sm = 1;
  int nb = S->num_sms * per_sm;
  int need = (S->P.N + kPB - 1) / kPB;
  need = need < 1 ? 1 : need;
  return nb < need ? nb : need;
}

void cycle_launch(clmd_system* S, int nsteps, int mode) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(S->cyc_blocks);
  cfg.blockDim = dim3(kPB);
  cfg.stream = S->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, cycle_kernel(S), S->P, S->st, cycle_args(S), nsteps, mode);
  S->launches++;
}
#endif  // CLMD_CYCLE_MIXED

}  // namespace clmd
