// clmd_internal.cuh -- device state layout, launch parameters and reduction
// helpers shared by the engine's CUDA translation units.
//
// Data layout in HBM (one system):
//   pos    double4[N]  x, y, z, w = species (as double); packed so that a
//                      neighbour gather is one 32-byte sector
//   vx..vz double[N]   SoA, like /ATOMC/ x1,y1,z1
//   ax..az double[N]   SoA, like /ATOMC/ x2,y2,z2
//   list   int32[cap]  full Verlet list in CSR rows (0-based atom indices,
//                      each row ascending); rows are placed by a warp-
//                      aggregated cursor, row_start/row_len/row_lo index them
//   cells  counting-sort bins: cell_count/start/fill, cell_atoms, spos
//   DevState           scalars (clmd_scalars first, so the host copies it
//                      with one memcpy), reduction counters, grid geometry
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/clmd.h"

#include "clmd_mixed.cuh"

namespace clmd {

constexpr int kBlock = 256;        // threads per block of the per-atom kernels
constexpr int kMaxRedBlocks = 4096; // partial-sum slots per reduction
constexpr int kScanTile = 2048;    // counts per block of the cell scan

// LJ coefficients by ij = api(i)+api(j) (for-a-lj-n-pbc-m.f:61-76,119-131):
// index 2 = species 1-1, 3 = 1-2, 4 = 2-2.
struct Params {
  double apmas[CLMD_MXSORTS];
  double boxx, boxy, boxz, ibx, iby, ibz;
  double dt, atrcut, atr2, atskin2, sig1;
  double c1[5], c2[5], c3[5], eps[5];
  double Q, att;
  double nkt3_i;  // 3*natom*cikb*att with 3*natom an INTEGER product
  double nkt3_d;  // 3.0d0*natom*cikb*att
  double ekinT[CLMD_MXSORTS];  // 1.5d0*cikb*att*apnum(s)
  int N, atsorts;
  int apnum[CLMD_MXSORTS];
  int sp_start[CLMD_MXSORTS + 1];  // first atom (0-based) of each species block
  int nbtim, btim, atnenum, csover, clwait, ftcsi;
  int ncx_max, ncy_max, ncz_max;
  int list_cap;         // full-list entries allocated
  long long half_cap;   // the caller's atnlist capacity (0: none): the reference's overflow rule
  int integrator, clustering;
  int precision;  // CLMD_PREC_FP64 or CLMD_PREC_MIXED (pair terms)
  int r12;        // pairs with species 2 purely repulsive (for-a-lj-n-pbc-mr.f)
  char apth[CLMD_MXSORTS];
  char ethst, clnuctrl;
};

struct DevState {
  clmd_scalars s;               // must stay first: copied to the host as is
  unsigned long long dmax2;     // max displacement^2 bits (atomicMax)
  unsigned long long list_used; // CSR cursor
  int rebuild;                  // this step rebuilds the list
  int cur_step;                 // the reference's loop counter i
  int err_new;                  // error raised inside a kernel, merged later
  int ncx, ncy, ncz, ncell;
  int nox, noy, noz;
  int offx[3], offy[3], offz[3];
  double cfx, cfy, cfz;         // cells per unit length
  double rs2;
  // thermostat
  double kf[CLMD_MXSORTS];
  int scale[CLMD_MXSORTS];
  double vcom[3];
  // clustering
  int nroots, nliq, nroots_f;
  int clu_force;                // next analysis runs even if cstep == step
  unsigned int ctr[16];         // last-block counters (one per reduction site)
  unsigned int bar_count, bar_gen;  // grid barrier of cooperative kernels
  // failure-path tests only (clmd_debug_barrier): arrivals a barrier waits
  // for beyond the grid (0 in use), and its spin limit (0: the default)
  unsigned int bar_extra, bar_pad;
  long long bar_limit;
};

enum CtrSlot {
  CTR_DRIFT = 0,
  CTR_FORCE,
  CTR_THERMO,
  CTR_MOM,
  CTR_MOM2,
  CTR_CLU,
  CTR_CLU2,
  CTR_NHSOLVE,
  CTR_SCAN,
};

__device__ __forceinline__ bool gated(const DevState* st) {
  return st->s.status != 0 || st->s.aborted != 0;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Fixed-shape block sum (deterministic for a given block size); result valid
// in thread 0.  sh must hold blockDim.x/32 doubles.
__device__ __forceinline__ double block_sum(double v, double* sh) {
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = lane < nw ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  return r;
}

__device__ __forceinline__ double block_max(double v, double* sh) {
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = lane < nw ? sh[lane] : 0.0;
    r = warp_max(r);
  }
  return r;
}

// Returns true in every thread of the block that arrives last; that block
// may then read all partials (written before the fence) with __ldcg.
__device__ __forceinline__ bool last_block(unsigned int* ctr) {
  __shared__ int am_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int t = atomicAdd(ctr, 1u);
    am_last = (t == gridDim.x - 1);
    if (am_last) *ctr = 0u;
  }
  __syncthreads();
  if (am_last) __threadfence();
  return am_last != 0;
}

// Sum of n partials in a fixed order by one block (deterministic).
__device__ __forceinline__ double reduce_partials(const double* p, int n, double* sh) {
  double v = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) v += __ldcg(p + k);
  return block_sum(v, sh);
}

// The reference's minimum image for force and cluster distances
// (for-a-lj-n-pbc-m.f:109-111): d + L*(bf1 - int(bf2 + d/L)).
__device__ __forceinline__ double mimage_bf(double d, double L, double iL, double bf1,
                                            double bf2) {
  return d + L * (bf1 - (double)(int)(bf2 + d * iL));
}

// LJ pair factor f_ij and energy term (for-a-lj-n-pbc-m.f:113-131); with
// P.r12 the pairs involving species 2 (ij = 3, 4) are the r^-12 wall of
// for-a-lj-n-pbc-mr.f:121-127.  Left to right, as the reference's
// expressions.
__device__ __forceinline__ double pair_fij(const Params& P, int ij, double rij2, double rij6) {
  if (P.r12 && ij >= 3) return P.eps[ij] * 12.0 * P.c2[ij] * rij2 * rij6 * rij6;
  return P.eps[ij] * 48.0 * rij2 * rij6 * (P.c2[ij] * rij6 - P.c3[ij]);
}
__device__ __forceinline__ double pair_e(const Params& P, int ij, double rij6) {
  if (P.r12 && ij >= 3) return P.eps[ij] * P.c2[ij] * rij6 * rij6;
  return P.eps[ij] * 4.0 * rij6 * (P.c2[ij] * rij6 - P.c1[ij]);
}

// Mixed-precision pair term (CLMD_PREC_MIXED): the caller has the FP64
// minimum-image difference and r^2 (the cut-off test stays FP64); the LJ
// factors, f_ij and the energy and virial terms are FP32.  t* get the FP32
// force components (exact in double), e and w the FP32 energy/virial terms.
__device__ __forceinline__ void pair_term_f32(const Params& P, int ij, double r2d, double dx,
                                              double dy, double dz, double& tx, double& ty,
                                              double& tz, double& e, double& w) {
  const float r2 = (float)r2d;
  const float ri2 = clmd_rcp_f32(r2);
  const float r6 = ri2 * ri2 * ri2;
  const float eps = (float)P.eps[ij], c1 = (float)P.c1[ij], c2 = (float)P.c2[ij],
              c3 = (float)P.c3[ij];
  const bool r12 = P.r12 && ij >= 3;
  const float fij = r12 ? eps * 12.0f * c2 * ri2 * r6 * r6 : eps * 48.0f * ri2 * r6 * (c2 * r6 - c3);
  tx = (double)(fij * (float)dx);
  ty = (double)(fij * (float)dy);
  tz = (double)(fij * (float)dz);
  e = (double)(r12 ? eps * c2 * r6 * r6 : eps * 4.0f * r6 * (c2 * r6 - c1));
  w = (double)(fij * r2);
}

// Kahan-compensated FP32 running sum (s += t), rounded step by step
__device__ __forceinline__ void kahan_add(float& s, float& c, float t) {
  const float y = __fsub_rn(t, c);
  const float u = __fadd_rn(s, y);
  c = __fsub_rn(__fsub_rn(u, s), y);
  s = u;
}

// The neighbour-list minimum image (neighbor-pbc-mav.f:84-86).
__device__ __forceinline__ double mimage_nb(double d, double L, double iL) {
  return d + L - L * (double)(int)(1.5 + d * iL);
}

__device__ __forceinline__ void raise_err(DevState* st, int code) {
  atomicCAS(&st->err_new, 0, code);
}

}  // namespace clmd
