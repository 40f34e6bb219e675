// clmd_ensemble.cu -- batched / served ensembles of independent replicas.
//
// One persistent launch per window: each CTA repeatedly claims a replica
// (largest first) from a device counter and runs it through one window --
// the Stillinger analysis + chk_nucleation at the window's first step, then
// ftcsi integrator steps -- with every phase separated by __syncthreads
// instead of a grid barrier.  The replica's positions (FP64) stay in shared
// memory for the whole window when they fit (<= ~8k atoms per CTA), so the
// neighbour gathers of the list search, the forces and the cluster test never
// leave the SM.  Per replica the algorithm is the drop-in's: adaptive-skin
// Verlet list (neighbor-pbc-mav.f) on a counting-sorted cell grid, velocity
// Verlet (int-verlet-mav.f) or Nose-Hoover (int-verlet-nh-mav.f), the
// Stillinger criterion (stoddard-pbc-n-m.f) and chk_nucleation
// (chk-nucleation.f); the start sequence (stopdead-m.f, neighbor(0),
// AccAtom, main.f:156-166) runs on the device when a replica is admitted.
//
// Mixed precision: minimum image, cut-off test, list and cluster tests in
// FP64 on FP64 positions; each pair term (1/r^2, r^-6, f_ij and its
// components) in FP32, summed per atom in FP32 with Kahan compensation in a
// fixed order (rows ordered by the cell sweep over index-sorted cells), so a
// replica's result does not depend on which other replicas share the launch.
// Positions, velocities, PSI, energies and the virial stay FP64.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/clmd.h"
#include "clmd_mixed.cuh"

namespace clmd_ens {

namespace cg = cooperative_groups;

constexpr int kFptCap = 128;  // first-passage sizes tracked per replica
#ifndef CLMD_SEARCH_PRUNE
#define CLMD_SEARCH_PRUNE 0
#endif
#ifndef CLMD_SEARCH_CHUNK
#define CLMD_SEARCH_CHUNK 2
#endif
// list search: candidate indices loaded ahead of their tests (2: measured
// best of 1, 2, 4 and 8 on the batched workload, all bit-identical)
constexpr int kSearchChunk = CLMD_SEARCH_CHUNK;
constexpr int kNcMax = 28;    // cells per dimension at most (cells never narrower than the list radius)

struct Rep {
  // parameters (reduced units: sigma = eps = m = 1)
  double box, ibox, att, Q, nkt3_i, nkt3_d, ekinT;
  int natom, off, csover, clwait, budget;
  int ethst;
  // state
  double psi, s, sumv2, ekin, epot, virial;
  double atrskin, dmms, dmmsu, dmmax, dmmav;
  double dmmh[256];
  int dmmst, dmmi, step, status, done, clbrkt, maxcs, fpt_top, nrebuild, cstep, started;
  int ncmax;  // cell-grid cap, fixed at admission from this replica's size only
  // the atoms' order inside the engine, fixed at admission (orig[] maps each
  // slot to its atom): 1 (positions too large for shared memory) cell order,
  // 2 (the others) by the rows' lengths; both renewed at every k-th rebuild
  int reorder;
  int nfull;                // full-list entries (pair terms per force pass) of the last rebuild
  long long pterms;         // pair terms evaluated by this replica's force passes
};

struct Args {
  double *x, *y, *z, *vx, *vy, *vz;
  double *vxn, *vyn, *vzn;
  void* a;  // float[3][pool] (mixed) or double[3][pool] (FP64)
  long long pool;
  int *list, *rlen, *sorted, *cellid, *parent, *cs, *cl, *fpt;
  int* orig;  // per slot: the pool index (offset + atom number) of the atom it holds
  Rep* reps;
  const int* items;
  const int* iwin;  // MD steps per item (nullptr: nwin windows for every item)
  int nitems;
  int* ctr;
  double rc, atskin, dt;
  int nbtim, ftcsi, lstride, integrator, nwin;
  int lg;  // mixed force pass: 1 << lg lanes per atom (0: one thread per atom)
  int reorder_every;  // the atoms' order renewed at every k-th rebuild
  int ncmax;  // cells per dimension this launch's shared memory holds
  int4* summary;  // per slot: done, status, step, maxcs
  float* wtime;   // per slot: device ms per MD step in its last launch (one CTA)
  // replicas run by a thread-block cluster: each cluster's cell counts and
  // scatter cursors (kNcMax^3 + 2 ints per cluster, indexed by cluster)
  int* cscr;
  long long cscr_stride;
  // clmd_ens_step_io: the window kernel itself reads each running replica's
  // x..vz from pinned host memory when it takes the replica and writes them
  // back when it leaves it (atom order, replica of slot r at hoff[r] of the
  // concatenation); nullptr: no host I/O
  const double *hx, *hy, *hz, *hvx, *hvy, *hvz;
  double *ox, *oy, *oz, *ovx, *ovy, *ovz;
  const long long* hoff;
};

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double wmax(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// block-wide sum returned to every thread, fixed shape: deterministic
template <int NT>
__device__ __forceinline__ double cta_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = wsum(v);
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    double t = lane < NT / 32 ? sh[lane] : 0.0;
    t = wsum(t);
    if (lane == 0) sh[32] = t;
  }
  __syncthreads();
  double r = sh[32];
  __syncthreads();
  return r;
}
template <int NT>
__device__ __forceinline__ double cta_max(double v, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = wmax(v);
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    double t = lane < NT / 32 ? sh[lane] : 0.0;
    t = wmax(t);
    if (lane == 0) sh[32] = t;
  }
  __syncthreads();
  double r = sh[32];
  __syncthreads();
  return r;
}

// two block-wide sums and an "any" flag in one round: every warp reduces the
// per-warp partials itself, so one barrier publishes them and one guards the
// buffer's reuse (fixed shape: deterministic)
template <int NT>
__device__ __forceinline__ void cta_sum2(double& a, double& b, int& f, double* sh) {
  constexpr int W = NT / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  a = wsum(a);
  b = wsum(b);
  f = __any_sync(0xffffffffu, f);
  if (lane == 0) {
    sh[w] = a;
    sh[W + w] = b;
    sh[2 * W + w] = f ? 1.0 : 0.0;
  }
  __syncthreads();
  double ta = lane < W ? sh[lane] : 0.0, tb = lane < W ? sh[W + lane] : 0.0;
  const int tf = lane < W ? (sh[2 * W + lane] != 0.0) : 0;
  a = wsum(ta);
  b = wsum(tb);
  f = __any_sync(0xffffffffu, tf);
  __syncthreads();
}

// the block sum of S (the tree of cta_sum2) and the closed-form Nose-Hoover
// root (clmd_nh_root) on warp 0 alone, published by the second barrier:
// the other warps skip the scalar Newton steps and their divisions
template <int NT>
__device__ __forceinline__ bool cta_nh_root(double S, double psi1, double nkt3, double dth,
                                            double Q, double* sh, double& Stot, double& p) {
  constexpr int W = NT / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  S = wsum(S);
  if (lane == 0) sh[w] = S;
  __syncthreads();
  if (w == 0) {
    const double t = wsum(lane < W ? sh[lane] : 0.0);
    double pr;
    const bool ok = clmd_nh_root(t, psi1, nkt3, dth, Q, pr);
    if (lane == 0) {
      sh[32] = t;
      sh[33] = pr;
      sh[34] = ok ? 1.0 : 0.0;
    }
  }
  __syncthreads();
  Stot = sh[32];
  p = sh[33];
  return sh[34] != 0.0;
}

// cta_nh_root with the step's end folded in (one CTA per replica): lane 0
// of warp 0 also records the replica's new PSI, sum v^2, ekin, step and pair
// terms (or the solve's failure) before the barrier that publishes the root,
// so the step needs no barrier of its own to publish them
template <int NT>
__device__ __forceinline__ bool cta_nh_root_commit(double S, double psi1, double nkt3,
                                                   double dth, double Q, double* sh, Rep& R,
                                                   int step, double& p) {
  constexpr int W = NT / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  S = wsum(S);
  if (lane == 0) sh[w] = S;
  __syncthreads();
  if (w == 0) {
    const double t = wsum(lane < W ? sh[lane] : 0.0);
    double pr;
    const bool ok = clmd_nh_root(t, psi1, nkt3, dth, Q, pr);
    if (lane == 0) {
      // slots 100, 101: past every slot a reduction of the next step writes
      // (up to 3 * 32), since no barrier separates these reads from them
      sh[100] = pr;
      sh[101] = ok ? 1.0 : 0.0;
      if (ok) {
        const double vsc = 1.0 / (1.0 + dth * pr);
        R.sumv2 = t * vsc * vsc;
        R.psi = pr;
        R.ekin = 0.5 * R.sumv2;
        R.step = step + 1;
        R.pterms += R.nfull;
      } else if (R.status == 0) {
        R.status = CLMD_ERR_NH_NOCONVERGE;
      }
    }
  }
  __syncthreads();
  p = sh[100];
  return sh[101] != 0.0;
}

// block max of a and sum of b in one round (as cta_sum2)
template <int NT>
__device__ __forceinline__ void cta_maxsum(double& a, double& b, double* sh) {
  constexpr int W = NT / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  a = wmax(a);
  b = wsum(b);
  if (lane == 0) {
    sh[w] = a;
    sh[W + w] = b;
  }
  __syncthreads();
  double ta = lane < W ? sh[lane] : 0.0, tb = lane < W ? sh[W + lane] : 0.0;
  a = wmax(ta);
  b = wsum(tb);
  __syncthreads();
}

// minimum image of a pair difference d in (-L - skin, L + skin): the image
// the reference's formulas pick for every pair nearer than L/2 (they differ
// only within rounding of |d| = L/2, beyond every cut-off since the list
// radius never exceeds L/2), with the same single rounding of d -/+ L
__device__ __forceinline__ double mi_sel(double d, double L, double hL) {
  if (fabs(d) > hL) d = d > 0.0 ? __dsub_rn(d, L) : __dadd_rn(d, L);
  return d;
}

// into [0, L] (neighbor-pbc-mav.f:67-71 up to rounding): between rebuilds an
// atom moves less than the skin, so one shift suffices; dmod for the rest
__device__ __forceinline__ double wrap_box(double x, double L) {
  if (x < 0.0)
    x = __dadd_rn(x, L);
  else if (x >= L)
    x = __dsub_rn(x, L);
  if (!(x >= 0.0 && x <= L)) x = fmod(fmod(x, L) + L, L);
  return x;
}

__device__ __forceinline__ void kahan(float& s, float& c, float t) {
  float y = __fsub_rn(t, c);
  float u = __fadd_rn(s, y);
  c = __fsub_rn(__fsub_rn(u, s), y);
  s = u;
}

// the reference's minimum images (neighbor-pbc-mav.f:84, for-a-lj-n-pbc-m.f:109)
__device__ __forceinline__ double mi_nb(double d, double L, double iL) {
  return __dsub_rn(__dadd_rn(d, L), __dmul_rn(L, (double)(int)__dadd_rn(1.5, __dmul_rn(d, iL))));
}
__device__ __forceinline__ double mi_bf(double d, double L, double iL, double bf1, double bf2) {
  return __dadd_rn(d, __dmul_rn(L, __dsub_rn(bf1, (double)(int)__dadd_rn(bf2, __dmul_rn(d, iL)))));
}

struct Cta {
  double xred[3 * 16];  // cluster reductions: the CTAs' partials (rank 0's copy is read)
  double xloc[4];       // cluster reductions: the totals, for this CTA's threads
  double* sx;  // positions in shared memory (nullptr: global)
  double* sy;
  double* sz;
  int* cstart;  // [ncell + 1]: cell c holds sorted[cstart[c] .. cstart[c + 1])
  double red[3 * 32 + 8];
  int ncx, ncell, nox, offx[3];
  double cf, rs2;
  int flag;
  int ident;  // sorted[] is the identity (the slots are in cell order)
  int rep;  // slot of the replica being run
  int nsteps;  // MD steps this replica runs in this launch
};

// ---------------------------------------------------------------------------
// A replica runs on one CTA (CS = 1) or on a thread-block cluster of CS CTAs
// (replicas whose positions do not fit in one SM's shared memory).  Every
// per-atom loop starts at gtid<NT, CS>() with stride NT * CS; gsync<CS>() is
// the barrier over the replica's threads (__syncthreads, or the cluster
// barrier whose release/acquire orders global and shared memory across the
// cluster); the grp_* reductions add a second level for CS > 1: each CTA's
// total goes to rank 0's shared memory (distributed shared memory), every
// CTA sums the CS partials in one fixed tree, so all CTAs hold bit-identical
// totals and keep identical copies of the replica record.  With CS = 1 the
// code is exactly the single-CTA code.
template <int CS>
__device__ __forceinline__ unsigned grank() {
  if constexpr (CS == 1)
    return 0u;
  else
    return cg::this_cluster().block_rank();
}
template <int NT, int CS>
__device__ __forceinline__ int gtid() {
  return (int)grank<CS>() * NT + (int)threadIdx.x;
}
template <int CS>
__device__ __forceinline__ void gsync() {
  if constexpr (CS == 1)
    __syncthreads();
  else
    cg::this_cluster().sync();
}

// the cluster level of a reduction of nv values (v[k]: this CTA's totals,
// the same in every thread): returns the cluster totals in v.  op 0 sums,
// op 1 takes maxima.  Two cluster barriers: the partials are published, then
// read by every CTA before any CTA may write the next reduction's.
template <int CS>
__device__ __forceinline__ void cl_reduce(double* v, int nv, const int* op, Cta& C) {
  auto cl = cg::this_cluster();
  const unsigned r = cl.block_rank();
  double* b0 = cl.map_shared_rank(C.xred, 0);
  if (threadIdx.x == 0)
    for (int k = 0; k < nv; k++) b0[k * 16 + r] = v[k];
  cl.sync();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    for (int k = 0; k < nv; k++) {
      double t = lane < CS ? b0[k * 16 + lane] : (op[k] ? -1.0e300 : 0.0);
      t = op[k] ? wmax(t) : wsum(t);
      if (lane == 0) C.xloc[k] = t;
    }
  }
  cl.sync();
  for (int k = 0; k < nv; k++) v[k] = C.xloc[k];
}

template <int NT, int CS>
__device__ __forceinline__ double grp_sum(double v, Cta& C) {
  double t = cta_sum<NT>(v, C.red);
  if constexpr (CS > 1) {
    const int op[1] = {0};
    cl_reduce<CS>(&t, 1, op, C);
  }
  return t;
}
template <int NT, int CS>
__device__ __forceinline__ double grp_max(double v, Cta& C) {
  double t = cta_max<NT>(v, C.red);
  if constexpr (CS > 1) {
    const int op[1] = {1};
    cl_reduce<CS>(&t, 1, op, C);
  }
  return t;
}
template <int NT, int CS>
__device__ __forceinline__ void grp_maxsum(double& a, double& b, Cta& C) {
  cta_maxsum<NT>(a, b, C.red);
  if constexpr (CS > 1) {
    double v[2] = {a, b};
    const int op[2] = {1, 0};
    cl_reduce<CS>(v, 2, op, C);
    a = v[0];
    b = v[1];
  }
}
template <int NT, int CS>
__device__ __forceinline__ void grp_sum2(double& a, double& b, int& f, Cta& C) {
  cta_sum2<NT>(a, b, f, C.red);
  if constexpr (CS > 1) {
    double v[3] = {a, b, f ? 1.0 : 0.0};
    const int op[3] = {0, 0, 1};
    cl_reduce<CS>(v, 3, op, C);
    a = v[0];
    b = v[1];
    f = v[2] != 0.0;
  }
}
template <int NT, int CS>
__device__ __forceinline__ int grp_or(int f, Cta& C) {
  if constexpr (CS == 1) {
    return __syncthreads_or(f);
  } else {
    double v[1] = {(double)__syncthreads_or(f)};
    const int op[1] = {1};
    cl_reduce<CS>(v, 1, op, C);
    return v[0] != 0.0;
  }
}
// the closed-form Nose-Hoover root of the group total of S (cta_nh_root for
// one CTA; for a cluster the total first, then warp 0 of every CTA takes the
// same root from the same total)
template <int NT, int CS>
__device__ __forceinline__ bool grp_nh_root(double S, double psi1, double nkt3, double dth,
                                            double Q, Cta& C, double& Stot, double& p) {
  if constexpr (CS == 1) {
    return cta_nh_root<NT>(S, psi1, nkt3, dth, Q, C.red, Stot, p);
  } else {
    double t = grp_sum<NT, CS>(S, C);
    if (threadIdx.x < 32) {
      double pr;
      const bool ok = clmd_nh_root(t, psi1, nkt3, dth, Q, pr);
      if (threadIdx.x == 0) {
        C.red[33] = pr;
        C.red[34] = ok ? 1.0 : 0.0;
      }
    }
    __syncthreads();
    Stot = t;
    p = C.red[33];
    const bool ok = C.red[34] != 0.0;
    __syncthreads();
    return ok;
  }
}

template <bool SM>
struct Pos {
  const Args& A;
  const Cta& C;
  int off;
  __device__ __forceinline__ double x(int i) const { return SM ? C.sx[i] : A.x[off + i]; }
  __device__ __forceinline__ double y(int i) const { return SM ? C.sy[i] : A.y[off + i]; }
  __device__ __forceinline__ double z(int i) const { return SM ? C.sz[i] : A.z[off + i]; }
  __device__ __forceinline__ void set(int i, double a, double b, double c) const {
    if (SM) {
      C.sx[i] = a; C.sy[i] = b; C.sz[i] = c;
    } else {
      A.x[off + i] = a; A.y[off + i] = b; A.z[off + i] = c;
    }
  }
};

// neighbor-pbc-mav.f:48-60, 101-105 on the replica record (thread 0)
__device__ bool prologue(Rep& R, Cta& C, const Args& A, int step) {
  const int kNcMax = R.ncmax;
  if (R.dmms > (R.atrskin - A.rc)) {
    if (R.status == 0) R.status = CLMD_ERR_SKIN;
    return false;
  }
  R.dmmav = (double)(float)R.dmmst * R.dmmsu / 256.0;
  if (step != 0 && step > 0) {
    R.atrskin = A.rc + (R.atrskin - A.rc) * (double)A.nbtim / (double)R.dmmst;
    R.atrskin = fmin(R.box / 2.0, R.atrskin);
  }
  C.rs2 = R.atrskin * R.atrskin;
  int n = (int)floor(R.box / (R.atrskin * (1.0 + 1e-9)));
  n = max(1, min(n, kNcMax));
  C.ncx = n;
  C.ncell = n * n * n;
  C.cf = (double)n / R.box;
  if (n >= 3) {
    C.nox = 3; C.offx[0] = -1; C.offx[1] = 0; C.offx[2] = 1;
  } else if (n == 2) {
    C.nox = 2; C.offx[0] = 0; C.offx[1] = 1;
  } else {
    C.nox = 1; C.offx[0] = 0;
  }
  R.dmmax = fmax(R.dmms, R.dmmax);
  R.dmms = 0.0;
  R.dmmst = 0;
  R.nrebuild++;
  return true;
}

// reorder 2: new slot p <- old atom cs[p] (new slot of old atom i in
// cellid[i]), a stable order (by index) of the atoms bucketed by their rows'
// lengths at the last rebuild.  Per tile of NT atoms, warp ballots rank the
// atoms of each bucket and the warps' counts (shared memory) place them.
constexpr int kLenBuckets = 16;  // lengths 0..11 each, 12-14, 15-19, 20-31, 32+
__device__ __forceinline__ int len_bucket(int len) {
  return len <= 11 ? len : len <= 14 ? 12 : len <= 19 ? 13 : len <= 31 ? 14 : 15;
}
template <int NT>
__device__ void length_order(const Rep& R, Cta& C, const Args& A) {
  constexpr int W = NT / 32;
  __shared__ int lsort[W * kLenBuckets + kLenBuckets];
  const int N = R.natom, off = R.off, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const unsigned lt = (1u << lane) - 1u;
  int* cnt = lsort;                   // [W][kLenBuckets]
  int* base = cnt + W * kLenBuckets;  // [kLenBuckets]
  // bucket sizes -> bucket starts
  // bucket sizes per warp by ballots (lane b keeps bucket b's count; no
  // per-thread array, which would live in local memory)
  int mine = 0;
  for (int i0 = 0; i0 < N; i0 += NT) {  // uniform: every thread takes every tile
    const int i = i0 + tid;
    const int key = i < N ? len_bucket(A.rlen[off + i]) : -1;
#pragma unroll
    for (int b = 0; b < kLenBuckets; b++) {
      const int c = __popc(__ballot_sync(0xffffffffu, key == b));
      if (lane == b) mine += c;
    }
  }
  if (lane < kLenBuckets) cnt[w * kLenBuckets + lane] = mine;
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int b = 0; b < kLenBuckets; b++) {
      int t = 0;
      for (int k = 0; k < W; k++) t += cnt[k * kLenBuckets + b];
      base[b] = acc;
      acc += t;
    }
  }
  __syncthreads();
  for (int i0 = 0; i0 < N; i0 += NT) {  // uniform: every thread takes every tile
    const int i = i0 + tid;
    const int key = i < N ? len_bucket(A.rlen[off + i]) : -1;
    int rank = 0;
#pragma unroll
    for (int b = 0; b < kLenBuckets; b++) {
      const unsigned m = __ballot_sync(0xffffffffu, key == b);
      if (key == b) rank = __popc(m & lt);
      if (lane == 0) cnt[w * kLenBuckets + b] = __popc(m);
    }
    __syncthreads();
    if (key >= 0) {
      int pre = base[key];
      for (int k = 0; k < w; k++) pre += cnt[k * kLenBuckets + key];
      const int slot = pre + rank;
      A.cellid[off + i] = slot;
      A.cs[off + slot] = i;
    }
    __syncthreads();
    if (tid < kLenBuckets) {
      int t = 0;
      for (int k = 0; k < W; k++) t += cnt[k * kLenBuckets + tid];
      base[tid] += t;
    }
    __syncthreads();
  }
}

// exclusive scan in place of cnt[0..n) by one CTA (thread 0 walks the warp
// sums): cnt[c] becomes the sum of the counts before c
template <int NT>
__device__ void cta_scan(int* cnt, int n) {
  __shared__ int wsums[NT / 32 + 1];
  const int tid = threadIdx.x;
  const int per = (n + NT - 1) / NT;
  int b0 = tid * per, s = 0;
  for (int k = 0; k < per; k++)
    if (b0 + k < n) s += cnt[b0 + k];
  int lane = tid & 31, w = tid >> 5, incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsums[w] = incl;
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int k = 0; k < NT / 32; k++) {
      int t = wsums[k];
      wsums[k] = acc;
      acc += t;
    }
  }
  __syncthreads();
  int ex = wsums[w] + incl - s;
  for (int k = 0; k < per; k++)
    if (b0 + k < n) {
      int v = cnt[b0 + k];
      cnt[b0 + k] = ex;
      ex += v;
    }
  __syncthreads();
}

// cell list + rows (ELL, transposed per replica: entry k of atom i at
// list[off*stride + k*N + i]); cells are index-sorted so row order is fixed
template <int NT, bool SM, int CS>
__device__ bool rebuild(Rep& R, Cta& C, const Args& A, const Pos<SM>& P) {
  const int N = R.natom, off = R.off, tid = threadIdx.x;
  const int gt = gtid<NT, CS>();
  constexpr int GT = NT * CS;
  const double L = R.box;
  // one array does the counting sort: counts at cnt[c + 1], an in-place
  // exclusive scan turns them into starts, and the scatter's atomics advance
  // each to its cell's end = the next cell's start.  One CTA keeps it in
  // shared memory; a cluster keeps it in global memory (its scratch) and
  // then copies the result into every CTA's shared memory for the search.
  int* cnt = C.cstart;
  if constexpr (CS > 1) cnt = A.cscr + (long long)(blockIdx.x / CS) * A.cscr_stride;
  for (int c = gt; c <= C.ncell; c += GT) cnt[c] = 0;
  if (tid == 0) C.ident = 0;  // until a reorder into cell order below
  gsync<CS>();
  for (int i = gt; i < N; i += GT) {
    const double x = wrap_box(P.x(i), L), y = wrap_box(P.y(i), L), z = wrap_box(P.z(i), L);
    P.set(i, x, y, z);
    int cx = min((int)(x * C.cf), C.ncx - 1), cy = min((int)(y * C.cf), C.ncx - 1),
        cz = min((int)(z * C.cf), C.ncx - 1);
    int c = (cz * C.ncx + cy) * C.ncx + cx;
    A.cellid[off + i] = c;
    atomicAdd(&cnt[c + 1], 1);
  }
  gsync<CS>();
  if (grank<CS>() == 0) cta_scan<NT>(cnt + 1, C.ncell);
  gsync<CS>();
  // scatter in arrival order (parent[] is free outside the analysis), then
  // each atom takes the place of its rank by index inside its cell: the
  // cell order is fixed whatever the order of the atomics
  int* tmp = A.parent + off;
  for (int i = gt; i < N; i += GT) {
    int slot = atomicAdd(&cnt[A.cellid[off + i] + 1], 1);
    tmp[slot] = i;
  }
  gsync<CS>();
  if constexpr (CS > 1) {
    for (int c = tid; c <= C.ncell; c += NT) C.cstart[c] = __ldcg(cnt + c);
    __syncthreads();
  }
  for (int i = gt; i < N; i += GT) {
    const int c = A.cellid[off + i], c0 = C.cstart[c], c1 = C.cstart[c + 1];
    int r = 0;
    for (int q = c0; q < c1; q++) r += tmp[q] < i;
    A.sorted[off + c0 + r] = i;
  }
  gsync<CS>();
  // either order may be kept for a few rebuilds (atoms move little between
  // rebuilds: measured +1.8% for cell-ordered cluster replicas renewed every
  // third rebuild instead of every one); the search and the forces use
  // whatever order the slots have, so skipping it changes nothing but the
  // order
  if (R.nrebuild % A.reorder_every == 0) {
    // reorder 1 (positions in global memory): the atoms move into cell
    // order, so that a warp's neighbour gathers fall within a few cells'
    // worth of memory.  reorder 2: a stable order by the previous rows'
    // lengths (bucketed), so that a warp's rows are of similar length and
    // its lanes finish together (rows change little between rebuilds).
    // vn and parent[] are dead here (the force pass and the analysis
    // rewrite them), so they hold the gathered copies.  Accelerations are
    // dead too: the force pass after a rebuild writes them before any read.
    const int* srt = A.sorted + off;
    if constexpr (CS == 1) {
      if (R.reorder == 2) {
        length_order<NT>(R, C, A);
        srt = A.cs + off;
      }
    }
    double *gx = A.vxn + off, *gy = A.vyn + off, *gz = A.vzn + off;
    int* go = A.parent + off;
    for (int p = gt; p < N; p += GT) {
      const int q = srt[p];
      gx[p] = P.x(q);
      gy[p] = P.y(q);
      gz[p] = P.z(q);
      go[p] = A.orig[off + q];
    }
    gsync<CS>();
    for (int p = gt; p < N; p += GT) {
      P.set(p, gx[p], gy[p], gz[p]);
      A.orig[off + p] = go[p];
    }
    gsync<CS>();
    for (int p = gt; p < N; p += GT) {
      const int q = srt[p];
      gx[p] = A.vx[off + q];
      gy[p] = A.vy[off + q];
      gz[p] = A.vz[off + q];
    }
    gsync<CS>();
    for (int p = gt; p < N; p += GT) {
      A.vx[off + p] = gx[p];
      A.vy[off + p] = gy[p];
      A.vz[off + p] = gz[p];
      if (R.reorder == 2)
        A.sorted[off + p] = A.cellid[off + A.sorted[off + p]];  // old index -> new slot
      else
        A.sorted[off + p] = p;  // the cells now hold consecutive slots
    }
    if (tid == 0) C.ident = R.reorder == 1;
    gsync<CS>();
  }
  const double hL = 0.5 * L, rs2 = C.rs2;
  const long long lbase = (long long)off * A.lstride;
  int over = 0, nsum = 0;
  // the atoms in cell order (sorted[]), whatever order their slots have: the
  // lanes of a warp then search overlapping stencils (similar candidate
  // counts, the same candidates read by several lanes at once)
  const bool ident = C.ident;
  for (int q0 = gt; q0 < N; q0 += GT) {
    const int i = ident ? q0 : A.sorted[off + q0];
    const double xi = P.x(i), yi = P.y(i), zi = P.z(i);
    int cx = min((int)(xi * C.cf), C.ncx - 1), cy = min((int)(yi * C.cf), C.ncx - 1),
        cz = min((int)(zi * C.cf), C.ncx - 1);
    int n = 0;
    // with three or more cells per dimension the stencil's cells hold each
    // neighbour once, at the periodic image nearest to atom i for every pair
    // within the list radius (cells are at least that wide): the image
    // shift is the cell range's, added to xi - xj with the same single
    // rounding the minimum image (mi_sel) gives, so the pair set and r^2
    // are those of mi_sel without its per-candidate tests; r^2 does not
    // depend on the pair's orientation (IEEE subtraction is sign-symmetric)
    const bool sel = C.nox < 3;
#if CLMD_SEARCH_PRUNE
    // the atom's distances to its cell's faces: a neighbour row (and an end
    // cell of a row) whose nearest point is farther than the list radius
    // holds no neighbour and is skipped (a margin of 1e-9 L covers the
    // rounding of the cell assignment).  Off by default: bit-identical, but
    // 3% slower on the batched workload (the per-row tests cost more than
    // the ~20% of candidates they save)
    const double cw = 1.0 / C.cf, mg = 1e-9 * L;
    const double fxl = fmax(xi - cx * cw - mg, 0.0), fxr = fmax((cx + 1) * cw - xi - mg, 0.0);
    const double fyl = fmax(yi - cy * cw - mg, 0.0), fyr = fmax((cy + 1) * cw - yi - mg, 0.0);
    const double fzl = fmax(zi - cz * cw - mg, 0.0), fzr = fmax((cz + 1) * cw - zi - mg, 0.0);
#endif
    for (int a = 0; a < C.nox; a++) {
      int zz = cz + C.offx[a];
      const double szL = sel ? 0.0 : (zz < 0 ? L : (zz >= C.ncx ? -L : 0.0));
      zz += zz < 0 ? C.ncx : 0;
      zz -= zz >= C.ncx ? C.ncx : 0;
      for (int b = 0; b < C.nox; b++) {
        int yy = cy + C.offx[b];
        const double syL = sel ? 0.0 : (yy < 0 ? L : (yy >= C.ncx ? -L : 0.0));
        yy += yy < 0 ? C.ncx : 0;
        yy -= yy >= C.ncx ? C.ncx : 0;
        const int rowc = (zz * C.ncx + yy) * C.ncx;
#if CLMD_SEARCH_PRUNE
        bool lft = true, rgt = true;
        if (!sel) {
          const int oz = C.offx[a], oy = C.offx[b];
          const double dz = oz < 0 ? fzl : (oz > 0 ? fzr : 0.0);
          const double dy = oy < 0 ? fyl : (oy > 0 ? fyr : 0.0);
          const double bx = rs2 - (dy * dy + dz * dz);
          if (bx < 0.0) continue;
          lft = fxl * fxl <= bx;
          rgt = fxr * fxr <= bx;
        }
#else
        const bool lft = true, rgt = true;
#endif
        // the x-neighbours of a cell row are contiguous in cell order: one
        // candidate range [ca0, cb0), a second [ca1, cb1) with image shift
        // sx1 where the row wraps (all of the row when ncx <= 2).  Scalars
        // picked per range, not arrays indexed by it: those would live in
        // local memory.
        int ca0, cb0, ca1 = 0, cb1 = 0, nr = 1;
        double sx1 = 0.0;
        if (sel) {
          ca0 = rowc; cb0 = rowc + C.ncx;
        } else if (cx == 0) {
          ca0 = rowc; cb0 = rowc + (rgt ? 2 : 1);
          ca1 = rowc + C.ncx - 1; cb1 = rowc + C.ncx; nr = lft ? 2 : 1;
          sx1 = L;
        } else if (cx == C.ncx - 1) {
          ca0 = rowc + cx - (lft ? 1 : 0); cb0 = rowc + C.ncx;
          ca1 = rowc; cb1 = rowc + 1; nr = rgt ? 2 : 1;
          sx1 = -L;
        } else {
          ca0 = rowc + cx - (lft ? 1 : 0); cb0 = rowc + cx + (rgt ? 2 : 1);
        }
        for (int d = 0; d < nr; d++) {
          const int q1 = C.cstart[d ? cb1 : cb0];
          const double sxL = d ? sx1 : 0.0;
          // kSearchChunk candidates' indices loaded ahead of their tests
          for (int q = C.cstart[d ? ca1 : ca0]; q < q1; q += kSearchChunk) {
            int js[kSearchChunk];
#pragma unroll
            for (int u = 0; u < kSearchChunk; u++)
              js[u] = q + u < q1 ? (ident ? q + u : A.sorted[off + q + u]) : i;
#pragma unroll
            for (int u = 0; u < kSearchChunk; u++) {
              const int j = js[u];
              if (j == i) continue;
              double dx = __dsub_rn(xi, P.x(j)), dy = __dsub_rn(yi, P.y(j)),
                     dz = __dsub_rn(zi, P.z(j));
              if (sel) {
                dx = mi_sel(dx, L, hL);
                dy = mi_sel(dy, L, hL);
                dz = mi_sel(dz, L, hL);
              } else {
                dx = __dadd_rn(dx, sxL);
                dy = __dadd_rn(dy, syL);
                dz = __dadd_rn(dz, szL);
              }
              double r2 =
                  __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
              if (r2 <= rs2) {
                if (n < A.lstride) A.list[lbase + (long long)n * N + i] = j;
                n++;
              }
            }
          }
        }
      }
    }
    if (n > A.lstride) {
      over = 1;
      n = A.lstride;
    }
    A.rlen[off + i] = n;
    nsum += n;
  }
  {
    // the rows' total (pair terms of each force pass until the next
    // rebuild) and "any row overflowed" in one reduction
    double tn = (double)nsum, unused = 0.0;
    grp_sum2<NT, CS>(tn, unused, over, C);
    if (tid == 0) R.nfull = (int)tn;
  }
  if (over) {
    if (tid == 0 && R.status == 0) R.status = CLMD_ERR_LIST_OVERFLOW;
    gsync<CS>();
    return false;
  }
  return true;
}

// int-verlet-mav.f:64-74 skin bookkeeping (thread 0)
__device__ int skin(Rep& R, const Args& A, double dmmr) {
  dmmr = 2.2 * sqrt(dmmr);
  R.dmms = R.dmms + dmmr;
  R.dmmsu = R.dmmsu + dmmr - R.dmmh[R.dmmi];
  R.dmmh[R.dmmi] = dmmr;
  R.dmmi = (R.dmmi + 1) & 255;
  R.dmmst = R.dmmst + 1;
  return R.dmms > (R.atrskin - A.rc - 2.0 * R.dmms / (double)(float)R.dmmst);
}

// pair forces (for-a-lj-n-pbc-m.f, sigma = eps = m = 1) -> a; optional
// velocity-Verlet second half kick; FP64 energy/virial sums when asked
// NHF: also the Nose-Hoover solve's first pass on the fresh accelerations
// (vo = v: vxn = v, s0 += v.v, dp += b vo dt/Q with b = -dth (a - psi1 vo))
template <int NT, bool SM, bool MIXED, int CS, bool NHF = false>
__device__ void forces(Rep& R, Cta& C, const Args& A, const Pos<SM>& P, bool kick,
                       bool energies, double psi1 = 0.0, double dtQ = 0.0, double* s0 = nullptr,
                       double* dp = nullptr) {
  const int N = R.natom, off = R.off, tid = threadIdx.x;
  const int gt = gtid<NT, CS>();
  constexpr int GT = NT * CS;
  const double L = R.box, hL = 0.5 * R.box, rc2 = A.rc * A.rc, dt = A.dt;
  const long long lbase = (long long)off * A.lstride;
  double esum = 0.0, vir = 0.0, ek = 0.0;
  if (MIXED && A.lg > 0) {
    // 1 << lg consecutive lanes per atom (rows of a liquid droplet run to
    // ~130 entries): lane `sub` of the group takes entries sub, sub + G, ...
    // with its own Kahan sums; the group then merges them in a fixed tree
    // (xor shuffles), so the result is deterministic for a given G.  The
    // loop is warp-uniform (32 / G atoms per warp and pass) so that every
    // lane takes part in the shuffles.
    const int lg = A.lg, G = 1 << lg, lane = tid & 31, sub = tid & (G - 1);
    for (int w0 = (gt - lane) >> lg; w0 < N; w0 += GT >> lg) {
      const int i = w0 + (lane >> lg);
      const bool own = i < N;
      const int ii = own ? i : w0;
      const double xi = P.x(ii), yi = P.y(ii), zi = P.z(ii);
      const int len = own ? A.rlen[off + i] : 0;
      float fx = 0.f, fy = 0.f, fz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
      const int* lp = A.list + lbase + (long long)sub * N + ii;
      const long long step = (long long)G * N;
      for (int k = sub; k < len; k += G, lp += step) {
        const int j = *lp;
        double dx = mi_sel(xi - P.x(j), L, hL);
        double dy = mi_sel(yi - P.y(j), L, hL);
        double dz = mi_sel(zi - P.z(j), L, hL);
        double r2d = dx * dx + dy * dy + dz * dz;
        if (r2d <= rc2) {
          float r2 = (float)r2d;
          float ri2 = clmd_rcp_f32(r2);
          float r6 = ri2 * ri2 * ri2;
          float fij = 48.0f * ri2 * r6 * (r6 - 0.5f);
          kahan(fx, cx, fij * (float)dx);
          kahan(fy, cy, fij * (float)dy);
          kahan(fz, cz, fij * (float)dz);
          if (energies && i < j) {
            esum += (double)(4.0f * r6 * (r6 - 1.0f));
            vir += (double)(fij * r2);
          }
        }
      }
      for (int o = 1; o < G; o <<= 1) {  // each partner's compensated sum
        const float px = __shfl_xor_sync(0xffffffffu, __fsub_rn(fx, cx), o);
        const float py = __shfl_xor_sync(0xffffffffu, __fsub_rn(fy, cy), o);
        const float pz = __shfl_xor_sync(0xffffffffu, __fsub_rn(fz, cz), o);
        kahan(fx, cx, px);
        kahan(fy, cy, py);
        kahan(fz, cz, pz);
      }
      if (!own || sub != 0) continue;
      float* a = (float*)A.a;
      a[off + i] = fx;
      a[A.pool + off + i] = fy;
      a[2 * A.pool + off + i] = fz;
      const double ax = (double)fx, ay = (double)fy, az = (double)fz;
      if (NHF) {
        const double dth = 0.5 * dt;
        const double wx = A.vx[off + i] + dth * ax;
        const double wy = A.vy[off + i] + dth * ay;
        const double wz = A.vz[off + i] + dth * az;
        A.vxn[off + i] = wx;
        A.vyn[off + i] = wy;
        A.vzn[off + i] = wz;
        *s0 += wx * wx + wy * wy + wz * wz;
      }
      if (kick) {
        double vxi = A.vx[off + i] + 0.5 * ax * dt;
        double vyi = A.vy[off + i] + 0.5 * ay * dt;
        double vzi = A.vz[off + i] + 0.5 * az * dt;
        A.vx[off + i] = vxi;
        A.vy[off + i] = vyi;
        A.vz[off + i] = vzi;
        if (energies) ek += 0.5 * (vxi * vxi + vyi * vyi + vzi * vzi);
      }
    }
  } else
  for (int i0 = 0; i0 < N; i0 += GT) {
    const int i = i0 + gt;
    if (i >= N) continue;
    const double xi = P.x(i), yi = P.y(i), zi = P.z(i);
    const int len = A.rlen[off + i];
    double ax, ay, az;
    if (MIXED) {
      float fx = 0.f, fy = 0.f, fz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
      // the next row entry is loaded while this pair is evaluated
      const int* lp = A.list + lbase + i;
      int jn = len > 0 ? lp[0] : 0;
#pragma unroll 2
      for (int k = 0; k < len; k++) {
        const int j = jn;
        lp += N;
        if (k + 1 < len) jn = *lp;
        double dx = mi_sel(xi - P.x(j), L, hL);
        double dy = mi_sel(yi - P.y(j), L, hL);
        double dz = mi_sel(zi - P.z(j), L, hL);
        double r2d = dx * dx + dy * dy + dz * dz;
        if (r2d <= rc2) {
          float r2 = (float)r2d;
          float ri2 = clmd_rcp_f32(r2);
          float r6 = ri2 * ri2 * ri2;
          float fij = 48.0f * ri2 * r6 * (r6 - 0.5f);
          kahan(fx, cx, fij * (float)dx);
          kahan(fy, cy, fij * (float)dy);
          kahan(fz, cz, fij * (float)dz);
          if (energies && i < j) {
            esum += (double)(4.0f * r6 * (r6 - 1.0f));
            vir += (double)(fij * r2);
          }
        }
      }
      float* a = (float*)A.a;
      a[off + i] = fx;
      a[A.pool + off + i] = fy;
      a[2 * A.pool + off + i] = fz;
      ax = (double)fx;
      ay = (double)fy;
      az = (double)fz;
    } else {
      double fx = 0.0, fy = 0.0, fz = 0.0;
      // the next row entry is loaded while this pair is evaluated
      const int* lp = A.list + lbase + i;
      int jn = len > 0 ? lp[0] : 0;
      for (int k = 0; k < len; k++) {
        const int j = jn;
        lp += N;
        if (k + 1 < len) jn = *lp;
        double dx = mi_sel(xi - P.x(j), L, hL);
        double dy = mi_sel(yi - P.y(j), L, hL);
        double dz = mi_sel(zi - P.z(j), L, hL);
        double r2d = dx * dx + dy * dy + dz * dz;
        if (r2d <= rc2) {
          double ri2 = 1.0 / r2d;
          double r6 = ri2 * ri2 * ri2;
          double fij = 48.0 * ri2 * r6 * (r6 - 0.5);
          fx += fij * dx;
          fy += fij * dy;
          fz += fij * dz;
          if (energies && i < j) {
            esum += 4.0 * r6 * (r6 - 1.0);
            vir += fij * r2d;
          }
        }
      }
      double* a = (double*)A.a;
      a[off + i] = fx;
      a[A.pool + off + i] = fy;
      a[2 * A.pool + off + i] = fz;
      ax = fx;
      ay = fy;
      az = fz;
    }
    if (NHF && MIXED) {
      // closed-form solve (clmd_nh_root): W = V + dth a into vn, s0 += W.W
      const double dth = 0.5 * dt;
      const double wx = A.vx[off + i] + dth * ax;
      const double wy = A.vy[off + i] + dth * ay;
      const double wz = A.vz[off + i] + dth * az;
      A.vxn[off + i] = wx;
      A.vyn[off + i] = wy;
      A.vzn[off + i] = wz;
      *s0 += wx * wx + wy * wy + wz * wz;
    } else if (NHF) {
      const double dth = 0.5 * dt;
      const double V[3] = {A.vx[off + i], A.vy[off + i], A.vz[off + i]};
      const double a3[3] = {ax, ay, az};
      A.vxn[off + i] = V[0];
      A.vyn[off + i] = V[1];
      A.vzn[off + i] = V[2];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        *s0 += V[d] * V[d];
        *dp += (-dth * (a3[d] - psi1 * V[d])) * V[d] * dtQ;
      }
    }
    if (kick) {
      double vxi = A.vx[off + i] + 0.5 * ax * dt;
      double vyi = A.vy[off + i] + 0.5 * ay * dt;
      double vzi = A.vz[off + i] + 0.5 * az * dt;
      A.vx[off + i] = vxi;
      A.vy[off + i] = vyi;
      A.vz[off + i] = vzi;
      if (energies) ek += 0.5 * (vxi * vxi + vyi * vyi + vzi * vzi);
    }
  }
  if (energies) {
    double e = grp_sum<NT, CS>(esum, C);
    double w = grp_sum<NT, CS>(vir, C);
    double k = kick ? grp_sum<NT, CS>(ek, C) : 0.0;
    if (tid == 0) {
      R.epot = e;
      R.virial = w;
      if (kick) R.ekin = k;
    }
  }
  // one CTA, mixed Nose-Hoover: the closed-form root that follows opens with
  // barriers of its own (cta_nh_root_commit), which order this pass's
  // per-atom writes before anyone reads them
  if constexpr (!(NHF && MIXED && CS == 1)) gsync<CS>();
}

template <bool MIXED>
__device__ __forceinline__ void get_a(const Args& A, int k, double& ax, double& ay, double& az) {
  if (MIXED) {
    const float* a = (const float*)A.a;
    ax = a[k];
    ay = a[A.pool + k];
    az = a[2 * A.pool + k];
  } else {
    const double* a = (const double*)A.a;
    ax = a[k];
    ay = a[A.pool + k];
    az = a[2 * A.pool + k];
  }
}

// stopdead-m.f:28-69 (one species, m = 1): COM removal and rescale to T
template <int NT, int CS>
__device__ void stopdead(Rep& R, Cta& C, const Args& A) {
  const int N = R.natom, off = R.off, tid = threadIdx.x;
  const int gt = gtid<NT, CS>();
  constexpr int GT = NT * CS;
  for (int loop = 0; loop < 10; loop++) {
    double px = 0, py = 0, pz = 0;
    for (int i = gt; i < N; i += GT) {
      px += A.vx[off + i];
      py += A.vy[off + i];
      pz += A.vz[off + i];
    }
    double vxs = grp_sum<NT, CS>(px, C) / (double)N;
    double vys = grp_sum<NT, CS>(py, C) / (double)N;
    double vzs = grp_sum<NT, CS>(pz, C) / (double)N;
    double ek = 0.0;
    for (int i = gt; i < N; i += GT) {
      double a = A.vx[off + i] - vxs, b = A.vy[off + i] - vys, c = A.vz[off + i] - vzs;
      A.vx[off + i] = a;
      A.vy[off + i] = b;
      A.vz[off + i] = c;
      ek += 0.5 * (a * a + b * b + c * c);
    }
    ek = grp_sum<NT, CS>(ek, C);
    double kf = sqrt(R.ekinT / ek);  // scalev-nh-m.f with step = -1
    for (int i = gt; i < N; i += GT) {
      A.vx[off + i] *= kf;
      A.vy[off + i] *= kf;
      A.vz[off + i] *= kf;
    }
    if (tid == 0) R.ekin = R.ekinT;
    gsync<CS>();
  }
}

__device__ __forceinline__ int ufind(int* par, int x) {
  for (;;) {
    int p = __ldcg(par + x);
    if (p == x) return x;
    int gp = __ldcg(par + p);
    if (gp != p) par[x] = gp;
    x = gp;
  }
}
__device__ __forceinline__ void uunion(int* par, int a, int b) {
  for (;;) {
    a = ufind(par, a);
    b = ufind(par, b);
    if (a == b) return;
    if (a < b) {
      int t = a;
      a = b;
      b = t;
    }
    if (atomicCAS(par + a, a, b) == a) return;
  }
}

// stoddard-pbc-n-m.f (one species) + chk-nucleation.f at step `step`
template <int NT, bool SM, int CS>
__device__ void analysis(Rep& R, Cta& C, const Args& A, const Pos<SM>& P, int step) {
  const int N = R.natom, off = R.off, tid = threadIdx.x;
  const int gt = gtid<NT, CS>();
  constexpr int GT = NT * CS;
  int* par = A.parent + off;
  int* cs = A.cs + off;
  for (int i = gt; i < N; i += GT) {
    par[i] = i;
    cs[i] = 0;
  }
  gsync<CS>();
  const double L = R.box, iL = R.ibox, rc2 = A.atskin * A.atskin;
  const double bf1 = (double)(int)(R.atrskin) + 2.0, bf2 = bf1 + 0.5;
  const long long lbase = (long long)off * A.lstride;
  for (int i = gt; i < N - 1; i += GT) {
    const double xi = P.x(i), yi = P.y(i), zi = P.z(i);
    const int len = A.rlen[off + i];
    for (int k = 0; k < len; k++) {
      int j = A.list[lbase + (long long)k * N + i];
      if (j <= i) continue;
      double dx = mi_bf(__dsub_rn(xi, P.x(j)), L, iL, bf1, bf2);
      double dy = mi_bf(__dsub_rn(yi, P.y(j)), L, iL, bf1, bf2);
      double dz = mi_bf(__dsub_rn(zi, P.z(j)), L, iL, bf1, bf2);
      double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
      if (r2 <= rc2) uunion(par, i, j);
    }
  }
  gsync<CS>();
  if (R.reorder) {
    // slots are in cell order: a cluster's label is the smallest atom number
    // (orig) among its slots, as for atoms kept in their own order.  sorted[]
    // is free outside the rebuild.
    int* mo = A.sorted + off;
    for (int i = gt; i < N; i += GT) mo[i] = 0x7fffffff;
    gsync<CS>();
    for (int i = gt; i < N; i += GT) atomicMin(mo + ufind(par, i), A.orig[off + i] - off);
    gsync<CS>();
    for (int i = gt; i < N; i += GT) {
      int r = ufind(par, i);
      A.cl[A.orig[off + i]] = mo[r] + 1;  // by atom number: slots move at rebuilds
      atomicAdd(cs + r, 1);
    }
  } else {
    for (int i = gt; i < N; i += GT) {
      int r = ufind(par, i);
      A.cl[off + i] = r + 1;
      atomicAdd(cs + r, 1);
    }
  }
  gsync<CS>();
  double m = 0.0;
  for (int i = gt; i < N; i += GT) m = fmax(m, (double)cs[i]);
  int maxcs = (int)grp_max<NT, CS>(m, C);
  if (tid == 0) {
    R.maxcs = maxcs;
    R.cstep = step;
    // first step at which the largest cluster reached each size
    int* fpt = A.fpt + (size_t)C.rep * kFptCap;
    if (grank<CS>() == 0)
      for (int s = R.fpt_top + 1; s <= maxcs && s <= kFptCap; s++) fpt[s - 1] = step;
    if (maxcs > R.fpt_top) R.fpt_top = maxcs;
    // chk-nucleation.f:33-56
    int tim = (maxcs >= R.csover && R.csover <= N) ? step : 0;
    if (tim > 0) {
      if (R.clbrkt == 0)
        R.clbrkt = tim;
      else if ((tim - R.clbrkt) >= R.clwait)
        R.done = 1;
    } else {
      R.clbrkt = 0;
    }
  }
  gsync<CS>();
}

// ---------------------------------------------------------------------------
// one replica, one window
// ---------------------------------------------------------------------------
// clmd_ens_step_io: this replica's state between pinned host memory (atom
// order) and its pool slots (engine order).  parent[] is free at a window's
// ends and holds the inverse of orig[] (atom -> slot), so that host memory
// is read and written in coalesced atom order.
template <int NT, int CS>
__device__ void host_io(const Rep& R, const Cta& C, const Args& A, bool in) {
  const int N = R.natom, off = R.off;
  const int gt = gtid<NT, CS>();
  constexpr int GT = NT * CS;
  int* inv = A.parent + off;
  for (int i = gt; i < N; i += GT) inv[A.orig[off + i] - off] = i;
  gsync<CS>();
  const long long h = A.hoff[C.rep];
  for (int a = gt; a < N; a += GT) {
    const long long s = off + inv[a];
    if (in) {
      A.x[s] = A.hx[h + a];
      A.y[s] = A.hy[h + a];
      A.z[s] = A.hz[h + a];
      A.vx[s] = A.hvx[h + a];
      A.vy[s] = A.hvy[h + a];
      A.vz[s] = A.hvz[h + a];
    } else {
      A.ox[h + a] = A.x[s];
      A.oy[h + a] = A.y[s];
      A.oz[h + a] = A.z[s];
      A.ovx[h + a] = A.vx[s];
      A.ovy[h + a] = A.vy[s];
      A.ovz[h + a] = A.vz[s];
    }
  }
  gsync<CS>();
}

template <int NT, bool SM, bool MIXED, int CS>
__device__ void run_window(Rep& R, Cta& C, const Args& A) {
  const int tid = threadIdx.x;
  const int gt = gtid<NT, CS>();
  constexpr int GT = NT * CS;
  const int N = R.natom, off = R.off;
  const bool nh = A.integrator == CLMD_INT_NOSE;
  const double dt = A.dt;
  Pos<SM> P{A, C, off};
  bool vin_n = false;  // uniform: the current velocities are in vxn, not vx
  double vsc = 1.0;    // mixed: the velocities are vn * vsc (clmd_nh_root)
  if (A.hx) host_io<NT, CS>(R, C, A, true);
  if (SM) {
    for (int i = gt; i < N; i += GT) {
      C.sx[i] = A.x[off + i];
      C.sy[i] = A.y[off + i];
      C.sz[i] = A.z[off + i];
    }
    gsync<CS>();
  }
  // the grid of the current list
  if (tid == 0) {
    int n = (int)floor(R.box / (R.atrskin * (1.0 + 1e-9)));
    n = max(1, min(n, R.ncmax));
    C.ncx = n;
    C.ncell = n * n * n;
    C.cf = (double)n / R.box;
    C.rs2 = R.atrskin * R.atrskin;
    C.nox = n >= 3 ? 3 : n;
    C.offx[0] = n >= 3 ? -1 : 0;
    C.offx[1] = n >= 3 ? 0 : 1;
    C.offx[2] = 1;
  }
  gsync<CS>();
  if (!R.started) {
    // stopdead(-1), neighbor(0), a = 0 + AccAtom, main.f:156-166
    stopdead<NT, CS>(R, C, A);
    if (tid == 0) C.flag = prologue(R, C, A, 0);
    gsync<CS>();
    if (!C.flag || !rebuild<NT, SM, CS>(R, C, A, P)) goto out;
    forces<NT, SM, MIXED, CS>(R, C, A, P, false, true);
    if (tid == 0) {
      R.sumv2 = 2.0 * R.ekin;
      R.psi = (R.ethst == 'N') ? (R.sumv2 - R.nkt3_d) / R.Q : 0.0;
      R.s = 0.0;
      R.started = 1;
      R.cstep = -1;
    }
    gsync<CS>();
  }
  // C.nsteps MD steps in this launch; the analysis and chk_nucleation run
  // whenever the step counter reaches a multiple of ftcsi (wrt-csi.f:27,
  // main.f:157-161), wherever the launch boundaries fall
  for (int todo = C.nsteps; todo > 0; todo--) {
    if (R.done || R.status) break;
    if (A.ftcsi > 0 && R.step % A.ftcsi == 0 && R.cstep != R.step) {
      if (vin_n) {  // velocities back in vx for the analysis
        for (int i = gt; i < N; i += GT) {
          A.vx[off + i] = MIXED ? A.vxn[off + i] * vsc : A.vxn[off + i];
          A.vy[off + i] = MIXED ? A.vyn[off + i] * vsc : A.vyn[off + i];
          A.vz[off + i] = MIXED ? A.vzn[off + i] * vsc : A.vzn[off + i];
        }
        vin_n = false;
        gsync<CS>();
      }
      analysis<NT, SM, CS>(R, C, A, P, R.step);
      if (R.done) break;
    }
    if (R.step >= R.budget) {
      gsync<CS>();
      if (tid == 0) R.done = 2;
      gsync<CS>();
      break;
    }
    {
      // energies at the end of every window and of the launch
      const bool last = todo == 1 || (R.step + 1) % (A.ftcsi > 0 ? A.ftcsi : 1) == 0;
      bool committed = false;  // the step's end already recorded (uniform)
      const int step = R.step;
      // drift
      double d2 = 0.0, sv = 0.0;
      const double psi = R.psi, dt2 = dt * dt / 2, dth = dt / 2;
      const double* svx = vin_n ? A.vxn : A.vx;
      const double* svy = vin_n ? A.vyn : A.vy;
      const double* svz = vin_n ? A.vzn : A.vz;
      const double sc = vin_n ? vsc : 1.0;
      vin_n = false;
      for (int i = gt; i < N; i += GT) {
        double vxi = svx[off + i], vyi = svy[off + i], vzi = svz[off + i];
        if (MIXED) {
          vxi = vxi * sc;
          vyi = vyi * sc;
          vzi = vzi * sc;
        }
        double axi, ayi, azi;
        get_a<MIXED>(A, off + i, axi, ayi, azi);
        double dx, dy, dz;
        if (!nh) {
          double hx = 0.5 * axi * dt, hy = 0.5 * ayi * dt, hz = 0.5 * azi * dt;
          dx = (vxi + hx) * dt;
          dy = (vyi + hy) * dt;
          dz = (vzi + hz) * dt;
          vxi += hx;
          vyi += hy;
          vzi += hz;
        } else {
          dx = dt * vxi + dt2 * (axi - psi * vxi);
          dy = dt * vyi + dt2 * (ayi - psi * vyi);
          dz = dt * vzi + dt2 * (azi - psi * vzi);
          sv += vxi * vxi + vyi * vyi + vzi * vzi;
          vxi = vxi + dth * (axi - psi * vxi);
          vyi = vyi + dth * (ayi - psi * vyi);
          vzi = vzi + dth * (azi - psi * vzi);
        }
        P.set(i, P.x(i) + dx, P.y(i) + dy, P.z(i) + dz);
        A.vx[off + i] = vxi;
        A.vy[off + i] = vyi;
        A.vz[off + i] = vzi;
        d2 = fmax(d2, dx * dx + dy * dy + dz * dz);
      }
      // the step's scalar logic on thread 0 (the reference's NH half step of
      // PSI and s, int-verlet-mav.f:64-74 skin bookkeeping, the rebuild
      // decision); one CTA: warp 0 takes the block totals between the two
      // barriers (the same tree as cta_maxsum), so one barrier fewer
      double dmmr = 0.0, sumv2 = 0.0;
      if constexpr (CS == 1) {
        constexpr int W = NT / 32;
        const int lane = tid & 31, w = tid >> 5;
        d2 = wmax(d2);
        sv = wsum(sv);
        if (lane == 0) {
          C.red[w] = d2;
          C.red[W + w] = sv;
        }
        __syncthreads();
        if (w == 0) {
          dmmr = wmax(lane < W ? C.red[lane] : 0.0);
          sumv2 = wsum(lane < W ? C.red[W + lane] : 0.0);
        }
      } else {
        grp_maxsum<NT, CS>(d2, sv, C);
        dmmr = d2;
        sumv2 = sv;
      }
      if (tid == 0) {
        if (nh) {
          R.sumv2 = sumv2;
          if (R.ethst == 'N') {
            R.s = R.s + R.psi * dt + (R.sumv2 - R.nkt3_d) * dt2 / R.Q;
            R.psi = R.psi + (R.sumv2 - R.nkt3_d) * dth / R.Q;
          }
        }
        C.flag = 1;
        if (skin(R, A, dmmr)) C.flag = prologue(R, C, A, step) ? 2 : 0;
      }
      gsync<CS>();
      if (C.flag == 0) goto out;
      if (C.flag == 2 && !rebuild<NT, SM, CS>(R, C, A, P)) goto out;
      if (!nh) {
        forces<NT, SM, MIXED, CS>(R, C, A, P, true, last);
      } else {
        // int-verlet-nh-mav.f:91-180 with block reductions.  Each sweep is one
        // pass: it updates vn from this sweep's delps and accumulates the
        // next sweep's sums (sum vn^2, sum b vo dt/Q at pso + delps) in the
        // same loop; the first pass rides on the force pass.
        const double Q = R.Q, err = 1.0e-10, psi1 = R.psi, dtQ = dt / Q;
        if (MIXED) {
          double S = 0.0, unused = 0.0, p;
          forces<NT, SM, MIXED, CS, true>(R, C, A, P, false, last, psi1, dtQ, &S, &unused);
          if constexpr (CS == 1) {
            if (!cta_nh_root_commit<NT>(S, psi1, R.nkt3_i, dth, Q, C.red, R, step, p)) goto out;
            committed = true;
          } else {
            if (!grp_nh_root<NT, CS>(S, psi1, R.nkt3_i, dth, Q, C, S, p)) {
              if (tid == 0 && R.status == 0) R.status = CLMD_ERR_NH_NOCONVERGE;
              gsync<CS>();
              goto out;
            }
            if (tid == 0) {
              const double c = 1.0 / (1.0 + dth * p);
              R.sumv2 = S * c * c;
              R.psi = p;
              R.ekin = 0.5 * R.sumv2;
            }
          }
          vsc = 1.0 / (1.0 + dth * p);
          vin_n = true;
        } else {
          double sumv2n = 0.0, dpsum = 0.0;
          forces<NT, SM, MIXED, CS, true>(R, C, A, P, false, last, psi1, dtQ, &sumv2n, &dpsum);
          int nr0 = 0;
          grp_sum2<NT, CS>(sumv2n, dpsum, nr0, C);
          double psn = psi1;
          int ready = 0;
          for (int iter = 1; iter <= 1000; iter++) {
            const double pso = psn;
            const double di = -(pso * dth + 1);
            double delps = dpsum - di * ((-sumv2n + R.nkt3_i) * dth / Q - (psi1 - pso));
            delps = delps / (-dt2 * sumv2n / Q + di);
            psn = pso + delps;
            const double rdi = 1.0 / di;
            double s2 = 0.0, dpn = 0.0;
            int nr = 0;
            for (int i = gt; i < N; i += GT) {
              double ax, ay, az;
              get_a<MIXED>(A, off + i, ax, ay, az);
              const double V[3] = {A.vx[off + i], A.vy[off + i], A.vz[off + i]};
              const double a3[3] = {ax, ay, az};
              double* vn[3] = {A.vxn, A.vyn, A.vzn};
              // the update rounded term by term: with fused multiply-adds the
              // residual b never reaches exactly zero, the sweep keeps moving a
              // near-zero component by ~1e-18 and the relative test then fails
              // where the reference's sweep (int-verlet-nh-mav.f:117-147)
              // settles on an exact fixed point
  #pragma unroll
              for (int d = 0; d < 3; d++) {
                const double vo = vn[d][off + i];
                const double b = __dsub_rn(__dmul_rn(-dth, __dsub_rn(a3[d], __dmul_rn(pso, vo))),
                                           __dsub_rn(V[d], vo));
                const double nx =
                    __dadd_rn(vo, __dmul_rn(__dadd_rn(b, __dmul_rn(__dmul_rn(dth, vo), delps)), rdi));
                if (fabs(__dsub_rn(nx, vo)) > err * fabs(nx)) nr = 1;
                vn[d][off + i] = nx;
                s2 += nx * nx;
                dpn += (-dth * (a3[d] - psn * nx) - (V[d] - nx)) * nx * dtQ;
              }
            }
            sumv2n = s2;
            dpsum = dpn;
            grp_sum2<NT, CS>(sumv2n, dpsum, nr, C);
            if (!nr) {
              ready = 1;
              break;
            }
          }
          if (!ready) {
            if (tid == 0 && R.status == 0) R.status = CLMD_ERR_NH_NOCONVERGE;
            gsync<CS>();
            goto out;
          }
          vin_n = true;  // the step's velocities are in vxn until the next drift
          if (tid == 0) {
            R.sumv2 = sumv2n;
            R.psi = psn;
            R.ekin = 0.5 * sumv2n;
          }
        }
      }
      if (!committed) {
        if (tid == 0) {
          R.step = step + 1;
          R.pterms += R.nfull;
        }
        gsync<CS>();
      }
    }
    // a spent budget ends the replica at once, after the analysis due at its
    // last step, rather than at the start of the next launch
    if (R.step >= R.budget) {
      if (vin_n) {
        for (int i = gt; i < N; i += GT) {
          A.vx[off + i] = MIXED ? A.vxn[off + i] * vsc : A.vxn[off + i];
          A.vy[off + i] = MIXED ? A.vyn[off + i] * vsc : A.vyn[off + i];
          A.vz[off + i] = MIXED ? A.vzn[off + i] * vsc : A.vzn[off + i];
        }
        vin_n = false;
        gsync<CS>();
      }
      if (A.ftcsi > 0 && R.step % A.ftcsi == 0 && R.cstep != R.step)
        analysis<NT, SM, CS>(R, C, A, P, R.step);
      gsync<CS>();
      if (tid == 0 && !R.done) R.done = 2;
      gsync<CS>();
      break;
    }
  }
out:
  gsync<CS>();
  if (vin_n) {
    for (int i = gt; i < N; i += GT) {
      A.vx[off + i] = MIXED ? A.vxn[off + i] * vsc : A.vxn[off + i];
      A.vy[off + i] = MIXED ? A.vyn[off + i] * vsc : A.vyn[off + i];
      A.vz[off + i] = MIXED ? A.vzn[off + i] * vsc : A.vzn[off + i];
    }
  }
  if (SM) {
    for (int i = gt; i < N; i += GT) {
      A.x[off + i] = C.sx[i];
      A.y[off + i] = C.sy[i];
      A.z[off + i] = C.sz[i];
    }
  }
  gsync<CS>();
  if (A.hx) host_io<NT, CS>(R, C, A, false);
}

// MINB: CTAs per SM the register budget must allow -- 512 / NT (<= 128
// registers per thread) or, for the register-lean shapes, 1024 / NT (64)
template <int NT, bool SM, bool MIXED, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_ens(Args A) {
  extern __shared__ double dsm[];
  __shared__ Rep R;
  __shared__ Cta C;
  __shared__ int item;
  for (;;) {
    if (threadIdx.x == 0) item = atomicAdd(A.ctr, 1);
    __syncthreads();
    const int it = item;
    if (it >= A.nitems) break;
    const int r = A.items[it];
    // replica record -> shared memory
    {
      const int* src = (const int*)(A.reps + r);
      int* dst = (int*)&R;
      for (int k = threadIdx.x; k < (int)(sizeof(Rep) / 4); k += NT) dst[k] = src[k];
    }
    __syncthreads();  // every word of R is written before thread 0 lays out smem from it
    if (threadIdx.x == 0) {
      int nmax = R.natom;
      const int ncell = R.ncmax * R.ncmax * R.ncmax;
      C.rep = r;
      C.cstart = (int*)dsm;
      double* p = (double*)(C.cstart + ((ncell + 2) & ~1));
      C.sx = SM ? p : nullptr;
      C.sy = SM ? p + nmax : nullptr;
      C.sz = SM ? p + 2 * nmax : nullptr;
    }
    __syncthreads();
    unsigned long long t0 = 0;
    const int step0 = R.step;
    if (threadIdx.x == 0) {
      C.nsteps = A.iwin ? A.iwin[it] : A.nwin * (A.ftcsi > 0 ? A.ftcsi : 1);
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    }
    __syncthreads();
    if (!R.done && !R.status) run_window<NT, SM, MIXED, 1>(R, C, A);
    if (threadIdx.x == 0 && R.step > step0) {
      unsigned long long t1;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
      A.wtime[r] = (float)((double)(t1 - t0) * 1e-6 / (double)(R.step - step0));
    }
    {
      const int* src = (const int*)&R;
      int* dst = (int*)(A.reps + r);
      for (int k = threadIdx.x; k < (int)(sizeof(Rep) / 4); k += NT) dst[k] = src[k];
    }
    if (threadIdx.x == 0) A.summary[r] = make_int4(R.done, R.status, R.step, R.maxcs);
    __syncthreads();
  }
}

// A replica too large for one SM's shared memory on a thread-block cluster
// of CS CTAs (one per SM): positions in global memory, the per-atom loops
// split over the cluster's CS * NT threads, the replica-wide barriers and
// reductions cluster-wide (see grp_*).  Every CTA keeps its own copy of the
// replica record and cell starts and applies the same scalar logic to the
// same totals; rank 0 alone writes the shared results back.  Each cluster
// takes replicas from the device counter like the single-CTA kernel.
template <int NT, bool MIXED, int CS>
__global__ void __launch_bounds__(NT, 1) k_ens_cl(Args A) {
  extern __shared__ double dsm[];
  __shared__ Rep R;
  __shared__ Cta C;
  __shared__ int item;
  auto cl = cg::this_cluster();
  const unsigned rank = cl.block_rank();
  for (;;) {
    if (rank == 0 && threadIdx.x == 0) item = atomicAdd(A.ctr, 1);
    cl.sync();
    const int it = *cl.map_shared_rank(&item, 0);
    cl.sync();  // rank 0's item is read by all before any CTA claims again or exits
    if (it >= A.nitems) break;
    const int r = A.items[it];
    {
      const int* src = (const int*)(A.reps + r);
      int* dst = (int*)&R;
      for (int k = threadIdx.x; k < (int)(sizeof(Rep) / 4); k += NT) dst[k] = src[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      C.rep = r;
      C.cstart = (int*)dsm;
      C.sx = C.sy = C.sz = nullptr;
    }
    unsigned long long t0 = 0;
    const int step0 = R.step;
    if (threadIdx.x == 0) {
      C.nsteps = A.iwin ? A.iwin[it] : A.nwin * (A.ftcsi > 0 ? A.ftcsi : 1);
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    }
    cl.sync();
    if (!R.done && !R.status) run_window<NT, false, MIXED, CS>(R, C, A);
    if (rank == 0) {
      if (threadIdx.x == 0 && R.step > step0) {
        unsigned long long t1;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
        A.wtime[r] = (float)((double)(t1 - t0) * 1e-6 / (double)(R.step - step0));
      }
      const int* src = (const int*)&R;
      int* dst = (int*)(A.reps + r);
      for (int k = threadIdx.x; k < (int)(sizeof(Rep) / 4); k += NT) dst[k] = src[k];
      if (threadIdx.x == 0) A.summary[r] = make_int4(R.done, R.status, R.step, R.maxcs);
    }
    cl.sync();
  }
}

}  // namespace clmd_ens

// ===========================================================================
// host side
// ===========================================================================
using namespace clmd_ens;

struct Range {
  long long off, len;
};

struct clmd_ensemble {
  clmd_ens_config cfg;
  int dev = 0, nsm = 148;
  cudaStream_t stream = nullptr;
  Args A;
  Rep* h_reps = nullptr;  // pinned mirror
  std::vector<int> used;  // slot in use
  std::vector<long long> slot_off;
  std::vector<Range> free_list;
  int* d_items = nullptr;
  int* d_ctr = nullptr;
  int* h_items = nullptr;  // pinned
  int* d_iwin = nullptr;   // windows per item (balanced launches)
  int* h_iwin = nullptr;   // pinned
  float* h_wtime = nullptr;  // pinned copy of A.wtime
  double* d_stage = nullptr;  // bulk copies in atom order (pool doubles, on first use)
  long long* d_hoff = nullptr;  // clmd_ens_step_io: each slot's offset in the host arrays
  int4* h_summary = nullptr;  // pinned copy of A.summary
  bool reps_stale = false;    // h_reps older than the device records
  // size classes: each has its own block size, shared-memory budget, stream.
  // 0-3: one CTA per replica, split by atom count (cls_max); 4-7: replicas
  // whose positions do not fit in shared memory, one thread-block cluster
  // of 2, 4, 8 or 16 CTAs per replica (kClusterAtoms atoms per CTA or more)
  static constexpr int kClasses = 8;
  static constexpr int kCtaClasses = 4;
  int cls_max[kCtaClasses] = {2048, 4096, 6144, 1 << 30};  // measured best of a few splits
  // the shapes the autotuner picks on the batched workload (used until it runs)
  int cls_threads[kClasses] = {512 | CLMD_ENS_LEAN, 1024, 1024, 1024, 1024, 1024, 1024, 1024};
  int cls_cs[kClasses] = {1, 1, 1, 1, 2, 4, 8, 16};
  int cls_lg[kClasses] = {};  // mixed force pass: 1 << lg lanes per atom
  int cl_max_clusters[kClasses] = {};  // co-resident clusters per launch (0: size unusable)
  int cl_region0[kClasses] = {};       // first cell-count region of each cluster class
  bool use_clusters = true;
  bool cell_order = false;  // every replica in cell order (CLMD_ENS_ORDER=cell)
  cudaStream_t cstream[kClasses] = {};
  cudaEvent_t ev0[kClasses] = {}, ev1[kClasses] = {}, evj = nullptr;
  cudaEvent_t evdone[kClasses] = {};  // join of each class stream
  // the window launch sequence replayed from a CUDA graph while the
  // replicas, their classes and the launch shapes stay the same
  bool use_graphs = true;
  std::map<void*, size_t> attr_smem;  // dynamic shared memory limit set per kernel
  cudaGraphExec_t gexec = nullptr;
  std::vector<long long> gkey;
  float last_ms[kClasses] = {};
  long long last_atoms[kClasses] = {};
  bool tuned = false;
  long long launches = 0;
  size_t smem_cap = 0;
  int threads = 256;
  std::mutex mu;
};

static int ck(cudaError_t e, const char* w) {
  if (e == cudaSuccess) return CLMD_OK;
  fprintf(stderr, "clmd_ens: %s: %s\n", w, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? CLMD_ERR_NOMEM : CLMD_ERR_CUDA;
}
#define ECK(call)                        \
  do {                                   \
    int _r = ck((call), #call);          \
    if (_r) return _r;                   \
  } while (0)

static size_t smem_bytes(int nmax, int ncmax, bool sm) {
  size_t nc = (size_t)ncmax * ncmax * ncmax;
  return sizeof(int) * ((nc + 2) & ~(size_t)1) + (sm ? 3 * sizeof(double) * (size_t)nmax : 0);
}

// the largest cell grid that fits beside the resident positions (at least
// 6^3 cells; positions go to global memory when even that does not fit)
static int cells_for(size_t cap, int nmax, bool* sm) {
  const size_t reserve = 8192;  // static shared memory of the kernel
  for (int nc = kNcMax; nc >= 6; nc--)
    if (smem_bytes(nmax, nc, true) + reserve <= cap) {
      *sm = true;
      return nc;
    }
  *sm = false;
  return kNcMax;
}

// the block shapes k_ens is compiled for (0: autotune)
static bool shape_ok(int shape) {
  const int lanes = (shape >> CLMD_ENS_LANES_SHIFT) & 0xff;
  if (lanes > 2) return false;
  shape &= ~(0xff << CLMD_ENS_LANES_SHIFT);
  switch (shape) {
    case 0: case 128: case 256: case 512: case 1024:
    case 128 | CLMD_ENS_LEAN: case 256 | CLMD_ENS_LEAN: case 512 | CLMD_ENS_LEAN:
      return true;
    default:
      return false;
  }
}

typedef void (*EnsKernel)(Args);

// the cluster kernel of cs CTAs per replica (1024 threads each)
static EnsKernel cluster_kernel(int cs, bool mixed) {
  switch (cs) {
    case 2: return mixed ? k_ens_cl<1024, true, 2> : k_ens_cl<1024, false, 2>;
    case 4: return mixed ? k_ens_cl<1024, true, 4> : k_ens_cl<1024, false, 4>;
    case 8: return mixed ? k_ens_cl<1024, true, 8> : k_ens_cl<1024, false, 8>;
    default: return mixed ? k_ens_cl<1024, true, 16> : k_ens_cl<1024, false, 16>;
  }
}
static size_t cluster_smem(int ncmax) {
  return sizeof(int) * (((size_t)ncmax * ncmax * ncmax + 2 + 1) & ~(size_t)1);
}

// how many clusters of each size can be resident at once (0: that size
// cannot be launched here, e.g. 16 without non-portable cluster support),
// and each class's share of the cell-count regions
static int setup_clusters(clmd_ensemble* E) {
  const bool mixed = E->cfg.precision == CLMD_PREC_MIXED;
  const size_t smem = cluster_smem(kNcMax);
  int region = 0;
  for (int c = clmd_ensemble::kCtaClasses; c < clmd_ensemble::kClasses; c++) {
    const int cs = E->cls_cs[c];
    EnsKernel k = cluster_kernel(cs, mixed);
    E->cl_max_clusters[c] = 0;
    if (cs > 8 && cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                      cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    E->attr_smem[(void*)k] = smem;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(cs);
    lc.blockDim = dim3(1024);
    lc.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, (void*)k, &lc) != cudaSuccess) {
      cudaGetLastError();
      n = 0;
    }
    n = std::min(n, E->nsm / cs);  // regions: the classes' shares sum to < nsm
    E->cl_max_clusters[c] = n;
    E->cl_region0[c] = region;
    region += E->nsm / cs;
  }
  return CLMD_OK;
}

extern "C" int clmd_ens_create(const clmd_ens_config* cfg, clmd_ensemble** out) {
  if (!cfg || !out || cfg->max_atoms < 2 || cfg->max_replicas < 1 || cfg->dt <= 0 ||
      cfg->rc <= 0 || cfg->rskin < cfg->rc || cfg->nbtim < 1 || !shape_ok(cfg->threads))
    return CLMD_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    return CLMD_ERR_NO_DEVICE;
  }
  clmd_ensemble* E = new clmd_ensemble();
  E->cfg = *cfg;
  // a full list row holds every neighbour within the list radius: ~5 in the
  // vapour, ~130 inside a liquid droplet (rho* 0.85, radius 3.3); the stride
  // only sizes the allocation, rebuilds write the rows' real lengths
  if (E->cfg.list_stride <= 0) E->cfg.list_stride = 192;
  if (E->cfg.threads <= 0) E->cfg.threads = 256;
  E->threads = E->cfg.threads;
  ECK(cudaGetDevice(&E->dev));
  ECK(cudaDeviceGetAttribute(&E->nsm, cudaDevAttrMultiProcessorCount, E->dev));
  int optin = 0;
  ECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, E->dev));
  E->smem_cap = (size_t)optin;
  ECK(cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking));
  for (int c = 0; c < clmd_ensemble::kClasses; c++) {
    ECK(cudaStreamCreateWithFlags(&E->cstream[c], cudaStreamNonBlocking));
    ECK(cudaEventCreate(&E->ev0[c]));
    ECK(cudaEventCreate(&E->ev1[c]));
    ECK(cudaEventCreateWithFlags(&E->evdone[c], cudaEventDisableTiming));
    if (cfg->threads > 0 && c < clmd_ensemble::kCtaClasses) E->cls_threads[c] = cfg->threads;
  }
  ECK(cudaEventCreateWithFlags(&E->evj, cudaEventDisableTiming));
  {
    const char* g = getenv("CLMD_ENS_GRAPHS");
    E->use_graphs = !(g && g[0] == '0');
    // CLMD_ENS_CLUSTERS=0: replicas too large for shared memory run on one
    // CTA each (class 3) instead of on a thread-block cluster
    const char* k = getenv("CLMD_ENS_CLUSTERS");
    E->use_clusters = !(k && k[0] == '0');
    const char* o = getenv("CLMD_ENS_ORDER");
    E->cell_order = o && strcmp(o, "cell") == 0;
    // CLMD_ENS_CLASSES="a,b,c": upper atom counts of the first three size
    // classes (ascending), for tuning the split
    const char* cs = getenv("CLMD_ENS_CLASSES");
    int b[3];
    if (cs && sscanf(cs, "%d,%d,%d", &b[0], &b[1], &b[2]) == 3 && 0 < b[0] && b[0] < b[1] &&
        b[1] < b[2])
      for (int c = 0; c < 3; c++) E->cls_max[c] = b[c];
  }
  E->tuned = cfg->threads > 0;
  const long long P = cfg->max_atoms;
  Args& A = E->A;
  memset(&A, 0, sizeof(A));
  A.pool = P;
  ECK(cudaMalloc(&A.x, 8 * P)); ECK(cudaMalloc(&A.y, 8 * P)); ECK(cudaMalloc(&A.z, 8 * P));
  ECK(cudaMalloc(&A.vx, 8 * P)); ECK(cudaMalloc(&A.vy, 8 * P)); ECK(cudaMalloc(&A.vz, 8 * P));
  ECK(cudaMalloc(&A.vxn, 8 * P)); ECK(cudaMalloc(&A.vyn, 8 * P)); ECK(cudaMalloc(&A.vzn, 8 * P));
  ECK(cudaMalloc(&A.a, 3 * 8 * P));
  ECK(cudaMalloc(&A.list, 4 * P * (long long)E->cfg.list_stride));
  ECK(cudaMalloc(&A.rlen, 4 * P)); ECK(cudaMalloc(&A.sorted, 4 * P));
  ECK(cudaMalloc(&A.cellid, 4 * P)); ECK(cudaMalloc(&A.parent, 4 * P));
  ECK(cudaMalloc(&A.cs, 4 * P)); ECK(cudaMalloc(&A.cl, 4 * P));
  ECK(cudaMalloc(&A.orig, 4 * P));
  ECK(cudaMemset(A.a, 0, 3 * 8 * P));
  ECK(cudaMemset(A.rlen, 0, 4 * P));
  ECK(cudaMemset(A.cl, 0, 4 * P));
  const int R = cfg->max_replicas;
  ECK(cudaMalloc(&A.reps, sizeof(Rep) * R));
  ECK(cudaMemset(A.reps, 0, sizeof(Rep) * R));
  ECK(cudaMalloc(&A.fpt, sizeof(int) * kFptCap * R));
  ECK(cudaMalloc(&A.summary, sizeof(int4) * R));
  ECK(cudaMemset(A.summary, 0, sizeof(int4) * R));
  ECK(cudaMallocHost(&E->h_summary, sizeof(int4) * R));
  memset(E->h_summary, 0, sizeof(int4) * R);
  ECK(cudaMallocHost(&E->h_reps, sizeof(Rep) * R));
  memset(E->h_reps, 0, sizeof(Rep) * R);
  ECK(cudaMalloc(&E->d_items, sizeof(int) * R));
  ECK(cudaMalloc(&E->d_iwin, sizeof(int) * R));
  ECK(cudaMallocHost(&E->h_iwin, sizeof(int) * R));
  ECK(cudaMalloc(&A.wtime, sizeof(float) * R));
  // cell counts of the cluster classes: one region per co-resident cluster
  A.cscr_stride = (long long)kNcMax * kNcMax * kNcMax + 2;
  ECK(cudaMalloc(&A.cscr, sizeof(int) * A.cscr_stride * (long long)E->nsm));
  {
    int st = setup_clusters(E);
    if (st) return st;
  }
  ECK(cudaMemset(A.wtime, 0, sizeof(float) * R));
  ECK(cudaMallocHost(&E->h_wtime, sizeof(float) * R));
  memset(E->h_wtime, 0, sizeof(float) * R);
  ECK(cudaMalloc(&E->d_ctr, sizeof(int) * 16));
  ECK(cudaMallocHost(&E->h_items, sizeof(int) * R));
  A.items = E->d_items;
  A.ctr = E->d_ctr;
  A.rc = cfg->rc;
  A.atskin = cfg->atskin;
  A.dt = cfg->dt;
  A.nbtim = cfg->nbtim;
  A.ftcsi = cfg->ftcsi;
  A.lstride = E->cfg.list_stride;
  A.integrator = cfg->integrator;
  {
    // CLMD_ENS_REORDER_EVERY=k: renew the length order at every k-th rebuild
    // (default 3: measured best of 1, 2 and 3 on the batched workload)
    const char* r = getenv("CLMD_ENS_REORDER_EVERY");
    A.reorder_every = (r && atoi(r) > 0) ? atoi(r) : 3;
  }
  E->used.assign(R, 0);
  E->slot_off.assign(R, -1);
  E->free_list.push_back({0, P});
  *out = E;
  return CLMD_OK;
}

extern "C" int clmd_ens_destroy(clmd_ensemble* E) {
  if (!E) return CLMD_OK;
  cudaStreamSynchronize(E->stream);
  Args& A = E->A;
  void* ps[] = {A.x, A.y, A.z, A.vx, A.vy, A.vz, A.vxn, A.vyn, A.vzn, A.a, A.list, A.rlen,
                A.sorted, A.cellid, A.parent, A.cs, A.cl, A.orig, A.reps, A.fpt, A.summary,
                E->d_items, E->d_ctr, E->d_iwin, A.wtime, E->d_stage, A.cscr,
                E->d_hoff};
  for (void* p : ps)
    if (p) cudaFree(p);
  if (E->h_reps) cudaFreeHost(E->h_reps);
  if (E->h_items) cudaFreeHost(E->h_items);
  if (E->h_iwin) cudaFreeHost(E->h_iwin);
  if (E->h_wtime) cudaFreeHost(E->h_wtime);
  if (E->h_summary) cudaFreeHost(E->h_summary);
  if (E->stream) cudaStreamDestroy(E->stream);
  for (int c = 0; c < clmd_ensemble::kClasses; c++) {
    if (E->cstream[c]) cudaStreamDestroy(E->cstream[c]);
    if (E->ev0[c]) cudaEventDestroy(E->ev0[c]);
    if (E->ev1[c]) cudaEventDestroy(E->ev1[c]);
    if (E->evdone[c]) cudaEventDestroy(E->evdone[c]);
  }
  if (E->evj) cudaEventDestroy(E->evj);
  if (E->gexec) cudaGraphExecDestroy(E->gexec);
  delete E;
  return CLMD_OK;
}

static long long pool_alloc(clmd_ensemble* E, long long n) {
  for (size_t k = 0; k < E->free_list.size(); k++) {
    Range& r = E->free_list[k];
    if (r.len >= n) {
      long long off = r.off;
      r.off += n;
      r.len -= n;
      if (r.len == 0) E->free_list.erase(E->free_list.begin() + k);
      return off;
    }
  }
  return -1;
}

static void pool_free(clmd_ensemble* E, long long off, long long n) {
  E->free_list.push_back({off, n});
  std::sort(E->free_list.begin(), E->free_list.end(),
            [](const Range& a, const Range& b) { return a.off < b.off; });
  std::vector<Range> m;
  for (auto& r : E->free_list) {
    if (!m.empty() && m.back().off + m.back().len == r.off)
      m.back().len += r.len;
    else
      m.push_back(r);
  }
  E->free_list.swap(m);
}

static int refresh_reps(clmd_ensemble* E) {
  if (!E->reps_stale) return CLMD_OK;
  ECK(cudaMemcpyAsync(E->h_reps, E->A.reps, sizeof(Rep) * E->cfg.max_replicas,
                      cudaMemcpyDeviceToHost, E->stream));
  ECK(cudaStreamSynchronize(E->stream));
  E->reps_stale = false;
  return CLMD_OK;
}

extern "C" int64_t clmd_ens_free_atoms(clmd_ensemble* E) {
  if (!E) return 0;
  long long s = 0;
  for (auto& r : E->free_list) s += r.len;
  return s;
}

extern "C" int64_t clmd_ens_launches(clmd_ensemble* E) { return E ? E->launches : 0; }

extern "C" int clmd_ens_pair_terms(clmd_ensemble* E, int64_t* total) {
  if (!E || !total) return CLMD_ERR_ARG;
  std::lock_guard<std::mutex> lock(E->mu);
  int rs = refresh_reps(E);
  if (rs) return rs;
  long long t = 0;
  for (int s = 0; s < E->cfg.max_replicas; s++)
    if (E->used[s]) t += E->h_reps[s].pterms;
  *total = t;
  return CLMD_OK;
}

extern "C" int clmd_ens_add(clmd_ensemble* E, const clmd_replica_spec* sp, const double* x,
                            const double* y, const double* z, const double* vx,
                            const double* vy, const double* vz, int32_t* slot) {
  if (!E || !sp || !x || !y || !z || !vx || !vy || !vz || !slot) return CLMD_ERR_ARG;
  const int N = sp->natom;
  if (N < 2 || !(sp->box > 2 * E->cfg.rc) || !(sp->temp > 0)) return CLMD_ERR_ARG;
  std::lock_guard<std::mutex> lock(E->mu);
  int s = -1;
  for (int k = 0; k < E->cfg.max_replicas; k++)
    if (!E->used[k]) {
      s = k;
      break;
    }
  if (s < 0) return CLMD_ERR_NOMEM;
  long long off = pool_alloc(E, N);
  if (off < 0) return CLMD_ERR_NOMEM;
  Args& A = E->A;
  cudaStream_t st = E->stream;
  ECK(cudaMemcpyAsync(A.x + off, x, 8 * N, cudaMemcpyHostToDevice, st));
  ECK(cudaMemcpyAsync(A.y + off, y, 8 * N, cudaMemcpyHostToDevice, st));
  ECK(cudaMemcpyAsync(A.z + off, z, 8 * N, cudaMemcpyHostToDevice, st));
  ECK(cudaMemcpyAsync(A.vx + off, vx, 8 * N, cudaMemcpyHostToDevice, st));
  ECK(cudaMemcpyAsync(A.vy + off, vy, 8 * N, cudaMemcpyHostToDevice, st));
  ECK(cudaMemcpyAsync(A.vz + off, vz, 8 * N, cudaMemcpyHostToDevice, st));
  Rep& R = E->h_reps[s];
  memset(&R, 0, sizeof(Rep));
  R.box = sp->box;
  R.ibox = 1.0 / sp->box;
  R.att = sp->temp / CLMD_CIKB;
  R.Q = sp->Q > 0 ? sp->Q : N * sp->temp * 0.25;
  R.nkt3_i = (double)(3 * N) * CLMD_CIKB * R.att;
  R.nkt3_d = 3.0 * N * CLMD_CIKB * R.att;
  R.ekinT = 1.5 * CLMD_CIKB * R.att * N;
  R.natom = N;
  R.off = (int)off;
  R.csover = sp->csover > 0 ? sp->csover : N + 1;
  R.clwait = sp->clwait;
  R.budget = sp->budget > 0 ? sp->budget : 0x7fffffff;
  R.ethst = sp->ethst;
  // read-3d.f:263-276
  R.atrskin = E->cfg.rskin;
  for (int i = 0; i < 256; i++)
    R.dmmh[i] = (E->cfg.rskin - E->cfg.rc) / (double)(float)E->cfg.nbtim;
  R.dmmsu = 256.0 * (E->cfg.rskin - E->cfg.rc) / (double)(float)E->cfg.nbtim;
  R.cstep = -1;
  bool fits = false;
  // the cell grid never needs more than box / rc cells per dimension (the
  // list radius stays above rc): small boxes keep their shared memory small
  R.ncmax = std::max(1, std::min(cells_for(E->smem_cap, N, &fits), (int)(sp->box / E->cfg.rc)));
  // (rows of similar length per warp; large: gathers near).
  // CLMD_ENS_ORDER=cell: cell order for every replica
  R.reorder = (fits && !E->cell_order) ? 2 : 1;
  std::vector<int> iota(N);
  for (int i = 0; i < N; i++) iota[i] = (int)off + i;
  ECK(cudaMemcpyAsync(A.orig + off, iota.data(), 4 * (size_t)N, cudaMemcpyHostToDevice, st));
  ECK(cudaMemsetAsync(A.rlen + off, 0, 4 * (size_t)N, st));  // the first order: pool history-free
  ECK(cudaMemcpyAsync(A.reps + s, &R, sizeof(Rep), cudaMemcpyHostToDevice, st));
  E->h_summary[s] = make_int4(0, 0, 0, 0);
  ECK(cudaMemcpyAsync(A.summary + s, &E->h_summary[s], sizeof(int4), cudaMemcpyHostToDevice,
                      st));
  std::vector<int> neg(kFptCap, -1);
  ECK(cudaMemcpyAsync(A.fpt + (size_t)s * kFptCap, neg.data(), sizeof(int) * kFptCap,
                      cudaMemcpyHostToDevice, st));
  ECK(cudaStreamSynchronize(st));
  E->used[s] = 1;
  E->slot_off[s] = off;
  *slot = s;
  return CLMD_OK;
}

extern "C" int clmd_ens_remove(clmd_ensemble* E, int32_t slot) {
  if (!E || slot < 0 || slot >= E->cfg.max_replicas || !E->used[slot]) return CLMD_ERR_ARG;
  std::lock_guard<std::mutex> lock(E->mu);
  ECK(cudaStreamSynchronize(E->stream));
  // natom is the admission value on the host whether or not h_reps is stale
  pool_free(E, E->slot_off[slot], E->h_reps[slot].natom);
  E->used[slot] = 0;
  E->slot_off[slot] = -1;
  memset(&E->h_reps[slot], 0, sizeof(Rep));
  E->h_reps[slot].done = 3;  // free
  E->h_summary[slot] = make_int4(3, 0, 0, 0);
  ECK(cudaMemcpyAsync(E->A.reps + slot, &E->h_reps[slot], sizeof(Rep), cudaMemcpyHostToDevice,
                      E->stream));
  ECK(cudaStreamSynchronize(E->stream));
  return CLMD_OK;
}

template <int NT, int MINB>
static EnsKernel pick(bool sm, bool mixed) {
  if (sm) return mixed ? k_ens<NT, true, true, MINB> : k_ens<NT, true, false, MINB>;
  return mixed ? k_ens<NT, false, true, MINB> : k_ens<NT, false, false, MINB>;
}

// a block shape: threads per CTA, with CLMD_ENS_LEAN for the 64-register
// variant (128, 256 and 512 threads)
static int shape_threads(int shape) { return shape & 0xffff; }
static int shape_lanes_log2(int shape) { return (shape >> CLMD_ENS_LANES_SHIFT) & 3; }

static EnsKernel kernel_for(int shape, bool sm, bool mixed) {
  const bool lean = (shape & CLMD_ENS_LEAN) != 0;
  switch (shape_threads(shape)) {
    case 128: return lean ? pick<128, 8>(sm, mixed) : pick<128, 4>(sm, mixed);
    case 512: return lean ? pick<512, 2>(sm, mixed) : pick<512, 1>(sm, mixed);
    case 1024: return pick<1024, 1>(sm, mixed);
    default: return lean ? pick<256, 4>(sm, mixed) : pick<256, 2>(sm, mixed);
  }
}

// the launch shape of one size class: kernel, dynamic shared memory, grid
struct ClassLaunch {
  EnsKernel k = nullptr;
  size_t smem = 0;
  int grid = 0, nt = 0, ncmax = 1, item0 = 0, nitems = 0;
  int cs = 1;       // CTAs per replica (thread-block cluster size)
  int lg = 0;       // lanes per atom in the mixed force pass: 1 << lg
  int region0 = 0;  // first cell-count region (cluster classes)
};

static int prepare_class(clmd_ensemble* E, int c, int item0, int nitems, const int* slots,
                         int shape, ClassLaunch& L) {
  L = ClassLaunch();
  L.item0 = item0;
  L.nitems = nitems;
  const int nt = shape_threads(shape);
  L.nt = nt;
  if (nitems == 0) return CLMD_OK;
  const bool mixed = E->cfg.precision == CLMD_PREC_MIXED;
  L.lg = mixed ? shape_lanes_log2(shape) : 0;
  if (c >= clmd_ensemble::kCtaClasses) {
    // one thread-block cluster per replica: 1024 threads per CTA, the cell
    // starts (kNcMax^3 at most) in each CTA's shared memory
    L.cs = E->cls_cs[c];
    L.nt = 1024;
    L.k = cluster_kernel(L.cs, mixed);
    for (int k = 0; k < nitems; k++) L.ncmax = std::max(L.ncmax, E->h_reps[slots[k]].ncmax);
    L.smem = cluster_smem(L.ncmax);
    L.region0 = E->cl_region0[c];
    const int nclu = std::min(E->cl_max_clusters[c], nitems);
    if (nclu < 1) return CLMD_ERR_ARG;
    L.grid = nclu * L.cs;
    return CLMD_OK;
  }
  // positions stay in shared memory if every replica of the class fits
  bool sm = true;
  for (int k = 0; k < nitems; k++) {
    const Rep& R = E->h_reps[slots[k]];
    if (smem_bytes(R.natom, R.ncmax, true) + 8192 > E->smem_cap) sm = false;
  }
  for (int k = 0; k < nitems; k++) {
    const Rep& R = E->h_reps[slots[k]];
    L.smem = std::max(L.smem, smem_bytes(R.natom, R.ncmax, sm));
    L.ncmax = std::max(L.ncmax, R.ncmax);
  }
  L.k = kernel_for(shape, sm, mixed);
  // the attribute only grows: classes that share a kernel may launch it
  // with different amounts in one sequence (occupancy follows each launch)
  size_t& lim = E->attr_smem[(void*)L.k];
  if (L.smem > lim) {
    ECK(cudaFuncSetAttribute(L.k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem));
    lim = L.smem;
  }
  int per_sm = 0;
  ECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, L.k, nt, L.smem));
  if (per_sm < 1) return CLMD_ERR_ARG;
  L.grid = (int)std::min<long long>((long long)per_sm * E->nsm, (long long)nitems);
  return CLMD_OK;
}

// one launch of one size class on its stream: every listed replica advances
// by nwin windows (or its balanced step count)
static int enqueue_class(clmd_ensemble* E, int c, const ClassLaunch& L, int nwin, bool balanced,
                         bool capturing) {
  cudaStream_t st = E->cstream[c];
  ECK(cudaMemsetAsync(E->d_ctr + c, 0, sizeof(int), st));
  Args A = E->A;
  A.items = E->d_items + L.item0;
  A.iwin = balanced ? E->d_iwin + L.item0 : nullptr;
  A.ctr = E->d_ctr + c;
  A.nitems = L.nitems;
  A.nwin = nwin;
  A.ncmax = L.ncmax;
  A.lg = L.lg;
  const unsigned fl = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
  ECK(cudaEventRecordWithFlags(E->ev0[c], st, fl));
  if (L.cs > 1) {
    A.cscr = E->A.cscr + (long long)L.region0 * E->A.cscr_stride;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(L.grid);
    lc.blockDim = dim3(L.nt);
    lc.dynamicSmemBytes = L.smem;
    lc.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = L.cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    ECK(cudaLaunchKernelEx(&lc, L.k, A));
  } else {
    L.k<<<L.grid, L.nt, L.smem, st>>>(A);
  }
  ECK(cudaGetLastError());
  ECK(cudaEventRecordWithFlags(E->ev1[c], st, fl));
  ECK(cudaEventRecord(E->evdone[c], st));
  return CLMD_OK;
}

// all running replicas, split by size class, each class largest first; the
// classes run concurrently on their own streams
// min_ms > 0: balanced launch -- replica i runs max(1, floor(min_ms / t_i))
// steps, t_i its device time per step measured in its earlier launches, so
// that every CTA stays busy about min_ms whatever its replica's size (a
// replica not yet timed runs a few steps)
// only >= 0: that size class alone (the autotuner's trials)
// the cluster class of a replica whose positions do not fit in shared
// memory: about kClusterAtoms atoms or more per CTA, the cluster size a power
// of two in [2, 16], the largest usable one not above it (-1: none usable).
// 6144 rather than 3072: on 300 replicas of 9,000-50,000 atoms 6.92e9 vs
// 6.66e9 atom-steps/s, served 9.49e9 vs 8.69e9 (1536: 5.50e9); the largest
// served size (50,000) gets 16 CTAs either way
constexpr int kClusterAtoms = 6144;
static int cluster_class(const clmd_ensemble* E, int n) {
  int want = 2;
  while (want < 16 && want * kClusterAtoms < n) want *= 2;
  for (int c = clmd_ensemble::kClasses - 1; c >= clmd_ensemble::kCtaClasses; c--)
    if (E->cls_cs[c] <= want && E->cl_max_clusters[c] > 0) return c;
  return -1;
}

static int launch_all(clmd_ensemble* E, int nwin, const int* threads, float min_ms = 0.0f,
                      int only = -1) {
  std::vector<int> cls[clmd_ensemble::kClasses];
  int nmax[clmd_ensemble::kClasses] = {};
  for (int s = 0; s < E->cfg.max_replicas; s++)
    if (E->used[s] && !E->h_summary[s].x && !E->h_summary[s].y) {
      const int n = E->h_reps[s].natom;
      int c = -1;
      if (E->use_clusters && E->h_reps[s].reorder == 1) c = cluster_class(E, n);
      if (c < 0) {
        c = 0;
        while (c < clmd_ensemble::kCtaClasses - 1 && n > E->cls_max[c]) c++;
      }
      if (only >= 0 && c != only) continue;
      cls[c].push_back(s);
      nmax[c] = std::max(nmax[c], n);
    }
  int total = 0;
  for (int c = 0; c < clmd_ensemble::kClasses; c++) {
    std::sort(cls[c].begin(), cls[c].end(), [&](int a, int b) {
      return E->h_reps[a].natom != E->h_reps[b].natom
                 ? E->h_reps[a].natom > E->h_reps[b].natom
                 : a < b;
    });
    memcpy(E->h_items + total, cls[c].data(), sizeof(int) * cls[c].size());
    total += (int)cls[c].size();
  }
  const bool balanced = min_ms > 0.0f;
  if (balanced && total > 0) {
    const int win = E->cfg.ftcsi > 0 ? E->cfg.ftcsi : 1;
    // while every replica's CTAs fit on the GPU at once, each runs for about
    // min_ms; when they do not (they then take turns on the SMs), each gets
    // about min_ms of SM time: a replica on a cluster of cs CTAs runs 1 / cs
    // of the steps that would fill min_ms, so that large replicas do not
    // take the SMs from the small ones in proportion to their cluster size
    long long demand = 0;
    int k0 = 0;
    std::vector<int> item_cs(total, 1);
    for (int c = 0; c < clmd_ensemble::kClasses; c++) {
      for (size_t q = 0; q < cls[c].size(); q++) item_cs[k0 + q] = E->cls_cs[c];
      demand += (long long)cls[c].size() * E->cls_cs[c];
      k0 += (int)cls[c].size();
    }
    const bool shared = demand > E->nsm;
    for (int k = 0; k < total; k++) {  // a replica not timed yet runs a few steps
      const float t = E->h_wtime[E->h_items[k]];  // ms per step, 0 = not timed yet
      const float ms = shared ? min_ms / (float)item_cs[k] : min_ms;
      long long n = t > 0.0f ? (long long)(ms / t) : (long long)std::min(win, 10);
      E->h_iwin[k] = (int)std::max(1LL, std::min(n, (long long)1 << 24));
    }
    ECK(cudaMemcpyAsync(E->d_iwin, E->h_iwin, sizeof(int) * total, cudaMemcpyHostToDevice,
                        E->stream));
  }
  for (int c = 0; c < clmd_ensemble::kClasses; c++) {
    E->last_ms[c] = -1.0f;
    E->last_atoms[c] = 0;
  }
  if (total == 0) return CLMD_OK;
  ClassLaunch L[clmd_ensemble::kClasses];
  std::vector<long long> key;
  key.reserve(total + 64);
  key.push_back(total);
  key.push_back(nwin);
  key.push_back(balanced);
  for (int k = 0; k < total; k++) key.push_back(E->h_items[k]);
  {
    int off = 0;
    for (int c = 0; c < clmd_ensemble::kClasses; c++) {
      for (int s : cls[c]) E->last_atoms[c] += E->h_reps[s].natom;
      int st = prepare_class(E, c, off, (int)cls[c].size(), cls[c].data(), threads[c], L[c]);
      if (st) return st;
      key.push_back(L[c].nt);
      key.push_back(L[c].lg);
      key.push_back(L[c].grid);
      key.push_back((long long)L[c].smem);
      key.push_back((long long)(size_t)L[c].k);
      off += (int)cls[c].size();
    }
  }
  // the sequence: item list (+ balanced step counts) in, the classes on their
  // streams, per-slot timings and summaries out
  auto enqueue = [&](bool capturing) -> int {
    if (balanced)
      ECK(cudaMemcpyAsync(E->d_iwin, E->h_iwin, sizeof(int) * total, cudaMemcpyHostToDevice,
                          E->stream));
    ECK(cudaMemcpyAsync(E->d_items, E->h_items, sizeof(int) * total, cudaMemcpyHostToDevice,
                        E->stream));
    ECK(cudaEventRecord(E->evj, E->stream));
    // the classes of the largest replicas first: their CTAs take SMs first
    for (int c = clmd_ensemble::kClasses - 1; c >= 0; c--) {
      if (L[c].nitems == 0) continue;
      ECK(cudaStreamWaitEvent(E->cstream[c], E->evj, 0));
      int st = enqueue_class(E, c, L[c], nwin, balanced, capturing);
      if (st) return st;
    }
    for (int c = 0; c < clmd_ensemble::kClasses; c++)
      if (L[c].nitems) ECK(cudaStreamWaitEvent(E->stream, E->evdone[c], 0));
    ECK(cudaMemcpyAsync(E->h_wtime, E->A.wtime, sizeof(float) * E->cfg.max_replicas,
                        cudaMemcpyDeviceToHost, E->stream));
    ECK(cudaMemcpyAsync(E->h_summary, E->A.summary, sizeof(int4) * E->cfg.max_replicas,
                        cudaMemcpyDeviceToHost, E->stream));
    return CLMD_OK;
  };
  if (E->use_graphs) {
    if (!E->gexec || key != E->gkey) {
      if (E->gexec) cudaGraphExecDestroy(E->gexec);
      E->gexec = nullptr;
      E->gkey.clear();
      ECK(cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeThreadLocal));
      int st = enqueue(true);
      cudaGraph_t g = nullptr;
      cudaError_t ce = cudaStreamEndCapture(E->stream, &g);
      if (st) {
        if (g) cudaGraphDestroy(g);
        return st;
      }
      ECK(ce);
      ce = cudaGraphInstantiate(&E->gexec, g, 0);
      cudaGraphDestroy(g);
      ECK(ce);
      E->gkey = key;
    }
    ECK(cudaGraphLaunch(E->gexec, E->stream));
  } else {
    int st = enqueue(false);
    if (st) return st;
  }
  for (int c = 0; c < clmd_ensemble::kClasses; c++)
    if (L[c].nitems) E->launches++;
  ECK(cudaStreamSynchronize(E->stream));
  for (int c = 0; c < clmd_ensemble::kClasses; c++) {
    if (L[c].nitems)
      ECK(cudaEventElapsedTime(&E->last_ms[c], E->ev0[c], E->ev1[c]));
    else
      E->last_ms[c] = -1.0f;
  }
  E->reps_stale = true;
  return CLMD_OK;
}

// Picks the block shape of each size class from 128, 256, 512 and 1024
// threads (<= 128 registers per thread below 1024) and the register-lean
// 128, 256 and 512 (64 registers: 8, 4 and 2 CTAs per SM where shared
// memory allows) by timing one window per candidate and class on the
// running replicas, each class alone (the classes share the GPU when they
// run together, and the window then takes about the sum of their times
// alone; the trial windows advance the simulation like any other window).
static int autotune(clmd_ensemble* E) {
  constexpr int kCand = 7;
  const int cand[kCand] = {128, 256, 512, 1024, 128 | CLMD_ENS_LEAN, 256 | CLMD_ENS_LEAN,
                           512 | CLMD_ENS_LEAN};
  float best[clmd_ensemble::kClasses];
  int pick[clmd_ensemble::kClasses];
  for (int c = 0; c < clmd_ensemble::kClasses; c++) {
    best[c] = 1e30f;
    pick[c] = E->cls_threads[c];
  }
  for (int k = 0; k < kCand; k++) {
    int th[clmd_ensemble::kClasses];
    for (int c = 0; c < clmd_ensemble::kClasses; c++)
      th[c] = c < clmd_ensemble::kCtaClasses ? cand[k] : E->cls_threads[c];
    for (int c = 0; c < clmd_ensemble::kCtaClasses; c++) {
      int st = launch_all(E, 1, th, 0.0f, c);
      if (st) return st;
      if (E->last_ms[c] < 0 || E->last_atoms[c] == 0) continue;
      float per_atom = E->last_ms[c] / (float)E->last_atoms[c];
      if (per_atom < best[c]) {
        best[c] = per_atom;
        pick[c] = cand[k];
      }
    }
  }
  // second axis (mixed precision): lanes per atom in the force pass, with
  // each class's shape from the first stage
  if (E->cfg.precision == CLMD_PREC_MIXED) {
    for (int lg = 1; lg <= 2; lg++) {
      int th[clmd_ensemble::kClasses];
      for (int c = 0; c < clmd_ensemble::kClasses; c++)
        th[c] = c < clmd_ensemble::kCtaClasses ? (pick[c] & ~(0xff << CLMD_ENS_LANES_SHIFT)) |
                                                     (lg << CLMD_ENS_LANES_SHIFT)
                                               : E->cls_threads[c];
      for (int c = 0; c < clmd_ensemble::kCtaClasses; c++) {
        int st = launch_all(E, 1, th, 0.0f, c);
        if (st) return st;
        if (E->last_ms[c] < 0 || E->last_atoms[c] == 0) continue;
        float per_atom = E->last_ms[c] / (float)E->last_atoms[c];
        if (per_atom < best[c]) {
          best[c] = per_atom;
          pick[c] = th[c];
        }
      }
    }
  }
  for (int c = 0; c < clmd_ensemble::kCtaClasses; c++) E->cls_threads[c] = pick[c];
  E->tuned = true;
  return CLMD_OK;
}

extern "C" int clmd_ens_step(clmd_ensemble* E, int32_t nwin) {
  if (!E || nwin < 1) return CLMD_ERR_ARG;
  std::lock_guard<std::mutex> lock(E->mu);
  return launch_all(E, nwin, E->cls_threads);
}

extern "C" int clmd_ens_step_timed(clmd_ensemble* E, float min_ms) {
  if (!E || !(min_ms > 0.0f)) return CLMD_ERR_ARG;
  std::lock_guard<std::mutex> lock(E->mu);
  return launch_all(E, 1, E->cls_threads, min_ms);
}

extern "C" int clmd_ens_autotune(clmd_ensemble* E, int32_t* threads_out) {
  if (!E) return CLMD_ERR_ARG;
  std::lock_guard<std::mutex> lock(E->mu);
  int st = autotune(E);
  if (threads_out)
    for (int c = 0; c < clmd_ensemble::kCtaClasses; c++) threads_out[c] = E->cls_threads[c];
  return st;
}

static void fill_result(const Rep& R, int s, clmd_replica_result& o) {
  o.ekin = R.ekin;
  o.epot = R.epot;
  o.psi = R.psi;
  o.s = R.s;
  o.slot = s;
  o.natom = R.natom;
  o.step = R.step;
  o.status = R.status;
  o.done = R.done;
  o.clbrkt = R.clbrkt;
  o.maxcs = R.maxcs;
  o.nrebuild = R.nrebuild;
}

extern "C" int clmd_ens_results(clmd_ensemble* E, clmd_replica_result* out, int32_t cap,
                                int32_t* n) {
  if (!E || !n) return CLMD_ERR_ARG;
  std::lock_guard<std::mutex> lock(E->mu);
  int rs = refresh_reps(E);
  if (rs) return rs;
  int k = 0;
  for (int s = 0; s < E->cfg.max_replicas; s++) {
    if (!E->used[s]) continue;
    if (out && k < cap) {
      fill_result(E->h_reps[s], s, out[k]);
    }
    k++;
  }
  *n = k;
  return CLMD_OK;
}

extern "C" int clmd_ens_poll(clmd_ensemble* E, clmd_replica_result* out, int32_t cap,
                             int32_t* n) {
  if (!E || !n) return CLMD_ERR_ARG;
  std::lock_guard<std::mutex> lock(E->mu);
  int k = 0;
  for (int s = 0; s < E->cfg.max_replicas; s++) {
    if (!E->used[s]) continue;
    if (out && k < cap) {
      const int4 q = E->h_summary[s];
      clmd_replica_result& o = out[k];
      if (q.x || q.y) {  // finished: its full record, one slot's copy
        if (E->reps_stale) {
          Rep R;
          ECK(cudaMemcpyAsync(&R, E->A.reps + s, sizeof(Rep), cudaMemcpyDeviceToHost,
                              E->stream));
          ECK(cudaStreamSynchronize(E->stream));
          fill_result(R, s, o);
        } else {
          fill_result(E->h_reps[s], s, o);
        }
      } else {
        memset(&o, 0, sizeof(o));
        o.slot = s;
        o.natom = E->h_reps[s].natom;
        o.step = q.z;
        o.maxcs = q.w;
      }
    }
    k++;
  }
  *n = k;
  return CLMD_OK;
}

// the atom number each slot of a reordered replica holds (orig[])
static int slot_orig(clmd_ensemble* E, int slot, std::vector<int>& o) {
  const int N = E->h_reps[slot].natom;
  o.resize(N);
  ECK(cudaMemcpyAsync(o.data(), E->A.orig + E->slot_off[slot], 4 * (size_t)N,
                      cudaMemcpyDeviceToHost, E->stream));
  ECK(cudaStreamSynchronize(E->stream));
  for (int& v : o) v -= (int)E->slot_off[slot];  // pool index -> atom number
  return CLMD_OK;
}

// a[p] (slot order) -> a[o[p]] (atom order)
template <typename T>
static void unpermute(T* a, const std::vector<int>& o) {
  std::vector<T> t(a, a + o.size());
  for (size_t p = 0; p < o.size(); p++) a[o[p]] = t[p];
}

extern "C" int clmd_ens_get_state(clmd_ensemble* E, int32_t slot, double* x, double* y,
                                  double* z, double* vx, double* vy, double* vz, double* ax,
                                  double* ay, double* az, int32_t* cl) {
  if (!E || slot < 0 || slot >= E->cfg.max_replicas || !E->used[slot]) return CLMD_ERR_ARG;
  std::lock_guard<std::mutex> lock(E->mu);
  const Args& A = E->A;
  const long long off = E->slot_off[slot];
  const int N = E->h_reps[slot].natom;
  cudaStream_t st = E->stream;
  double* dst[6] = {x, y, z, vx, vy, vz};
  double* src[6] = {A.x, A.y, A.z, A.vx, A.vy, A.vz};
  for (int k = 0; k < 6; k++)
    if (dst[k]) ECK(cudaMemcpyAsync(dst[k], src[k] + off, 8 * N, cudaMemcpyDeviceToHost, st));
  double* ad[3] = {ax, ay, az};
  if (E->cfg.precision == CLMD_PREC_MIXED) {
    std::vector<float> tmp(N);
    for (int k = 0; k < 3; k++)
      if (ad[k]) {
        ECK(cudaMemcpyAsync(tmp.data(), (float*)A.a + k * A.pool + off, 4 * N,
                            cudaMemcpyDeviceToHost, st));
        ECK(cudaStreamSynchronize(st));
        for (int i = 0; i < N; i++) ad[k][i] = tmp[i];
      }
  } else {
    for (int k = 0; k < 3; k++)
      if (ad[k])
        ECK(cudaMemcpyAsync(ad[k], (double*)A.a + k * A.pool + off, 8 * N,
                            cudaMemcpyDeviceToHost, st));
  }
  if (cl) ECK(cudaMemcpyAsync(cl, A.cl + off, 4 * N, cudaMemcpyDeviceToHost, st));
  ECK(cudaStreamSynchronize(st));
  if (E->h_reps[slot].reorder) {  // slots in cell order: back to atom order
    std::vector<int> o;
    int rc = slot_orig(E, slot, o);
    if (rc) return rc;
    double* arr[9] = {x, y, z, vx, vy, vz, ax, ay, az};
    for (double* a : arr)
      if (a) unpermute(a, o);  // (labels are stored by atom number already)
  }
  return CLMD_OK;
}

extern "C" int clmd_ens_fpt(clmd_ensemble* E, int32_t slot, int32_t* fpt, int32_t cap) {
  if (!E || !fpt || slot < 0 || slot >= E->cfg.max_replicas || !E->used[slot])
    return CLMD_ERR_ARG;
  int n = std::min(cap, kFptCap);
  ECK(cudaMemcpy(fpt, E->A.fpt + (size_t)slot * kFptCap, sizeof(int) * n,
                 cudaMemcpyDeviceToHost));
  for (int k = n; k < cap; k++) fpt[k] = -1;
  return CLMD_OK;
}

// helpers/mpt.f:80-92 over the replicas instead of over sizer files: per
// size, the mean first-passage step of the replicas whose largest cluster
// reached it, and its standard error sqrt((<t^2> - <t>^2) / count); sums in
// slot order (deterministic)
__global__ void k_mfpt(const int* fpt, const int* use, int nslot, int cap, double* mean,
                       double* sem, int* count) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cap) return;
  double t = 0.0, tt = 0.0;
  int n = 0;
  for (int s = 0; s < nslot; s++) {
    if (!use[s]) continue;
    const int v = fpt[(size_t)s * kFptCap + j];
    if (v < 0) continue;
    const double d = (double)v;
    t += d;
    tt += d * d;
    n++;
  }
  count[j] = n;
  if (n == 0) {
    mean[j] = -1.0;
    sem[j] = 0.0;
    return;
  }
  const double m = t / (double)n;
  mean[j] = m;
  sem[j] = sqrt(fmax(tt / (double)n - m * m, 0.0) / (double)n);
}

extern "C" int clmd_ens_mfpt(clmd_ensemble* E, int32_t cap, double* mean, double* sem,
                             int32_t* count) {
  if (!E || !mean || !sem || !count || cap < 1) return CLMD_ERR_ARG;
  std::lock_guard<std::mutex> lock(E->mu);
  const int n = std::min(cap, kFptCap), R = E->cfg.max_replicas;
  int* d_use = nullptr;
  double* d_out = nullptr;
  int* d_cnt = nullptr;
  ECK(cudaMalloc(&d_use, sizeof(int) * R));
  ECK(cudaMalloc(&d_out, sizeof(double) * 2 * n));
  ECK(cudaMalloc(&d_cnt, sizeof(int) * n));
  std::vector<int> use(E->used.begin(), E->used.end());
  cudaStream_t st = E->stream;
  ECK(cudaMemcpyAsync(d_use, use.data(), sizeof(int) * R, cudaMemcpyHostToDevice, st));
  k_mfpt<<<(n + 127) / 128, 128, 0, st>>>(E->A.fpt, d_use, R, n, d_out, d_out + n, d_cnt);
  E->launches++;
  ECK(cudaGetLastError());
  ECK(cudaMemcpyAsync(mean, d_out, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  ECK(cudaMemcpyAsync(sem, d_out + n, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  ECK(cudaMemcpyAsync(count, d_cnt, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  ECK(cudaStreamSynchronize(st));
  cudaFree(d_use);
  cudaFree(d_out);
  cudaFree(d_cnt);
  for (int k = n; k < cap; k++) {
    mean[k] = -1.0;
    sem[k] = 0.0;
    count[k] = 0;
  }
  return CLMD_OK;
}

// pool ranges of the occupied slots in slot order (the host layout), with
// consecutive slots whose pool ranges abut merged into one copy
static void host_ranges(clmd_ensemble* E, std::vector<std::pair<long long, long long>>& r) {
  r.clear();
  for (int s = 0; s < E->cfg.max_replicas; s++) {
    if (!E->used[s]) continue;
    const long long off = E->slot_off[s], n = E->h_reps[s].natom;
    if (!r.empty() && r.back().first + r.back().second == off)
      r.back().second += n;
    else
      r.push_back({off, n});
  }
}

// bulk copies in atom order: slot g holds pool index orig[g] (the replicas
// that keep their atoms reordered move them, the others hold orig[g] = g)
__global__ void k_from_atom_order(double* dst, const double* stage, const int* orig,
                                  long long first, long long n) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) dst[first + k] = stage[orig[first + k]];
}
__global__ void k_to_atom_order(double* stage, const double* src, const int* orig,
                                long long first, long long n) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) stage[orig[first + k]] = src[first + k];
}

static int ensure_stage(clmd_ensemble* E) {
  if (!E->d_stage) ECK(cudaMalloc(&E->d_stage, 8 * (size_t)E->A.pool));
  return CLMD_OK;
}

extern "C" int clmd_ens_upload(clmd_ensemble* E, const double* x, const double* y,
                               const double* z, const double* vx, const double* vy,
                               const double* vz) {
  if (!E) return CLMD_ERR_ARG;
  std::lock_guard<std::mutex> lock(E->mu);
  int rc = ensure_stage(E);
  if (rc) return rc;
  std::vector<std::pair<long long, long long>> r;
  host_ranges(E, r);
  const double* src[6] = {x, y, z, vx, vy, vz};
  double* dst[6] = {E->A.x, E->A.y, E->A.z, E->A.vx, E->A.vy, E->A.vz};
  for (int k = 0; k < 6; k++) {
    if (!src[k]) continue;
    long long h = 0;
    for (auto& q : r) {
      ECK(cudaMemcpyAsync(E->d_stage + q.first, src[k] + h, 8 * (size_t)q.second,
                          cudaMemcpyHostToDevice, E->stream));
      const unsigned nb = (unsigned)((q.second + 255) / 256);
      k_from_atom_order<<<nb, 256, 0, E->stream>>>(dst[k], E->d_stage, E->A.orig, q.first,
                                                    q.second);
      ECK(cudaGetLastError());
      E->launches++;
      h += q.second;
    }
  }
  ECK(cudaStreamSynchronize(E->stream));
  return CLMD_OK;
}

extern "C" int clmd_ens_download(clmd_ensemble* E, double* x, double* y, double* z,
                                 double* vx, double* vy, double* vz) {
  if (!E) return CLMD_ERR_ARG;
  std::lock_guard<std::mutex> lock(E->mu);
  int rc = ensure_stage(E);
  if (rc) return rc;
  std::vector<std::pair<long long, long long>> r;
  host_ranges(E, r);
  double* dst[6] = {x, y, z, vx, vy, vz};
  const double* src[6] = {E->A.x, E->A.y, E->A.z, E->A.vx, E->A.vy, E->A.vz};
  for (int k = 0; k < 6; k++) {
    if (!dst[k]) continue;
    long long h = 0;
    for (auto& q : r) {
      const unsigned nb = (unsigned)((q.second + 255) / 256);
      k_to_atom_order<<<nb, 256, 0, E->stream>>>(E->d_stage, src[k], E->A.orig, q.first,
                                                  q.second);
      ECK(cudaGetLastError());
      E->launches++;
      ECK(cudaMemcpyAsync(dst[k] + h, E->d_stage + q.first, 8 * (size_t)q.second,
                          cudaMemcpyDeviceToHost, E->stream));
      h += q.second;
    }
  }
  ECK(cudaStreamSynchronize(E->stream));
  return CLMD_OK;
}

// the device address of pinned host memory (CLMD_ERR_ARG for anything else)
static int mapped_host(const void* p, void** d) {
  cudaPointerAttributes at;
  if (!p || cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return CLMD_ERR_ARG;
  }
  if (at.type != cudaMemoryTypeHost || !at.devicePointer) return CLMD_ERR_ARG;
  *d = at.devicePointer;
  return CLMD_OK;
}

extern "C" int clmd_ens_step_io(clmd_ensemble* E, int32_t nwin, double* x, double* y, double* z,
                                double* vx, double* vy, double* vz) {
  if (!E || nwin < 1) return CLMD_ERR_ARG;
  std::lock_guard<std::mutex> lock(E->mu);
  double* h[6] = {x, y, z, vx, vy, vz};
  void* d[6];
  for (int k = 0; k < 6; k++)
    if (mapped_host(h[k], &d[k])) return CLMD_ERR_ARG;
  const int R = E->cfg.max_replicas;
  if (!E->d_hoff) ECK(cudaMalloc(&E->d_hoff, sizeof(long long) * R));
  // the layout of clmd_ens_upload: occupied slots concatenated in slot order
  std::vector<long long> hoff(R, 0);
  long long pos = 0;
  for (int s = 0; s < R; s++)
    if (E->used[s]) {
      hoff[s] = pos;
      pos += E->h_reps[s].natom;
    }
  ECK(cudaMemcpyAsync(E->d_hoff, hoff.data(), sizeof(long long) * R, cudaMemcpyHostToDevice,
                      E->stream));
  Args& A = E->A;
  A.hx = A.ox = (double*)d[0];
  A.hy = A.oy = (double*)d[1];
  A.hz = A.oz = (double*)d[2];
  A.hvx = A.ovx = (double*)d[3];
  A.hvy = A.ovy = (double*)d[4];
  A.hvz = A.ovz = (double*)d[5];
  A.hoff = E->d_hoff;
  // direct launches: a graph would keep these host addresses
  const bool graphs = E->use_graphs;
  E->use_graphs = false;
  int st = launch_all(E, nwin, E->cls_threads);
  E->use_graphs = graphs;
  A.hx = A.hy = A.hz = A.hvx = A.hvy = A.hvz = nullptr;
  A.ox = A.oy = A.oz = A.ovx = A.ovy = A.ovz = nullptr;
  A.hoff = nullptr;
  if (st) return st;
  ECK(cudaStreamSynchronize(E->stream));
  return CLMD_OK;
}

extern "C" int clmd_ens_last_ms(clmd_ensemble* E, float* ms, int64_t* atoms) {
  if (!E) return CLMD_ERR_ARG;
  // four entries: the single-CTA classes 0-2, then class 3 together with the
  // cluster classes (the longest of their times, the sum of their atoms)
  for (int c = 0; c < clmd_ensemble::kCtaClasses; c++) {
    float m = E->last_ms[c];
    long long a = E->last_atoms[c];
    if (c == clmd_ensemble::kCtaClasses - 1)
      for (int k = clmd_ensemble::kCtaClasses; k < clmd_ensemble::kClasses; k++) {
        m = std::max(m, E->last_ms[k]);
        a += E->last_atoms[k];
      }
    if (ms) ms[c] = m;
    if (atoms) atoms[c] = a;
  }
  return CLMD_OK;
}
