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
                                                  const int* row_len, const int* row_lo,
                                                  double* ax, double* ay, double* az,
                                                  double* vx, double* vy, double* vz,
                                                  double* partials, int advance) {
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
    const bool mixed = P.precision == CLMD_PREC_MIXED;
    float sx = 0.f, sy = 0.f, sz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;  // mixed: Kahan sums
    int k0 = row_start[i], k1 = k0 + row_len[i], kown = k0 + row_lo[i];
    for (int k = k0; k < k1; k++) {
      int j = list[k];
      double4 pb = pos[j];
      bool own = k >= kown;  // neighbour has the larger reference index
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
        double rij6 = 0.0;
        if (!mixed) {
          rij2 = 1.0 / rij2;
          rij6 = rij2 * rij2 * rij2;
        }
        int ij = sa + (int)pb.w;
        if (ij < 2 || ij > 4) {
          raise_err(st, CLMD_ERR_BAD_SPECIES);
          continue;
        }
        if (mixed) {
          double tx, ty, tz, e, w;
          pair_term_f32(P, ij, r2, dx, dy, dz, tx, ty, tz, e, w);
          const float sg = own ? 1.0f : -1.0f;
          if (own) {
            esum = esum + e;
            vir = vir + w;
          }
          kahan_add(sx, cx, sg * (float)tx);
          kahan_add(sy, cy, sg * (float)ty);
          kahan_add(sz, cz, sg * (float)tz);
          continue;
        }
        double fij = pair_fij(P, ij, rij2, rij6);
        if (own) {
          esum = esum + pair_e(P, ij, rij6);
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
    if (mixed) {
      fx = (double)sx;
      fy = (double)sy;
      fz = (double)sz;
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
      // main.f:226 i = i + 1 (velocity Verlet: the force kernel ends the step)
      if (advance && q.status == 0) st->cur_step = st->cur_step + 1;
    }
  }
}

// ---------------------------------------------------------------------------
// scalev-nh-m.f:39-76 velocity scaling per species block
// ---------------------------------------------------------------------------
__device__ __forceinline__ int species_block(const Params& P, int i) {
  for (int s = 0; s < P.atsorts; s++)
    if (i >= P.sp_start[s] && i < P.sp_start[s + 1]) return s;
  return -1;
}

__global__ void k_thermo_sum(Params P, DevState* st, const int* perm, const double* vx,
                             const double* vy, const double* vz, double* partials, int step) {
  if (gated(st)) return;
  __shared__ double sh[kBlock / 32];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int sp = -1;
  double e = 0.0;
  if (i < P.N) {
    sp = species_block(P, perm[i]);
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

__global__ void k_thermo_scale(Params P, DevState* st, const int* perm, double* vx, double* vy,
                               double* vz) {
  if (gated(st)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.N) return;
  int sp = species_block(P, perm[i]);
  if (sp < 0 || !st->scale[sp]) return;
  double kf = st->kf[sp];
  vx[i] = vx[i] * kf;
  vy[i] = vy[i] * kf;
  vz[i] = vz[i] * kf;
}

// stopdead-m.f:30-55
__global__ void k_mom_sum(Params P, DevState* st, const double4* pos, const double* vx,
                          const double* vy, const double* vz, double* partials) {
  if (gated(st)) return;
  __shared__ double sh[kBlock / 32];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double px = 0.0, py = 0.0, pz = 0.0;
  if (i < P.N) {
    double mas = P.apmas[(int)pos[i].w - 1];
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

__global__ void k_mom_sub(Params P, DevState* st, const double4* pos, double* vx, double* vy,
                          double* vz, double* partials) {
  if (gated(st)) return;
  __shared__ double sh[kBlock / 32];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  if (i < P.N) {
    double mas = P.apmas[(int)pos[i].w - 1];
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

// host input (reference order, staging arrays) -> state (slot order)
__global__ void k_scatter_in(int N, const int* iperm, const double* sx, const double* sy,
                             const double* sz, const double* svx, const double* svy,
                             const double* svz, const double* sax, const double* say,
                             const double* saz, const int* api, double4* pos, double* vx,
                             double* vy, double* vz, double* ax, double* ay, double* az,
                             unsigned int mask) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int p = iperm[i];
  double4 q = pos[p];
  if (mask & 1u) q.x = sx[i];
  if (mask & 2u) q.y = sy[i];
  if (mask & 4u) q.z = sz[i];
  q.w = (double)api[i];
  pos[p] = q;
  if (mask & 8u) vx[p] = svx[i];
  if (mask & 16u) vy[p] = svy[i];
  if (mask & 32u) vz[p] = svz[i];
  if (mask & 64u) ax[p] = sax[i];
  if (mask & 128u) ay[p] = say[i];
  if (mask & 256u) az[p] = saz[i];
}

// state (slot order) -> staging arrays (reference order)
__global__ void k_gather_out(int N, const int* iperm, const double4* pos, const double* vx,
                             const double* vy, const double* vz, const double* ax,
                             const double* ay, const double* az, double* sx, double* sy,
                             double* sz, double* svx, double* svy, double* svz, double* sax,
                             double* say, double* saz) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int p = iperm[i];
  double4 q = pos[p];
  sx[i] = q.x;
  sy[i] = q.y;
  sz[i] = q.z;
  svx[i] = vx[p];
  svy[i] = vy[p];
  svz[i] = vz[p];
  sax[i] = ax[p];
  say[i] = ay[p];
  saz[i] = az[p];
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
void k_set_step_launch(clmd_system* S, int step) {
  k_set_step<<<1, 1, 0, S->stream>>>(S->st, step);
  S->launches++;
}
void clear_cells(clmd_system* S) {
  cudaMemsetAsync(S->cell_count, 0, sizeof(int) * (S->ncell_alloc + 1), S->stream);
}

void force_launch(clmd_system* S, int mode, int advance) {
  auto args = [&](auto kern) {
    kern<<<S->nblk, kBlock, 0, S->stream>>>(S->P, S->st, S->pos, S->list, S->row_start,
                                             S->row_len, S->row_lo, S->ax, S->ay, S->az, S->vx,
                                             S->vy, S->vz, S->partials, advance);
  };
  if (mode == FORCE_VV_KICK)
    args(k_force<FORCE_VV_KICK>);
  else if (mode == FORCE_ZERO_FIRST)
    args(k_force<FORCE_ZERO_FIRST>);
  else
    args(k_force<FORCE_ACCUMULATE>);
  S->launches++;
}

void thermostat_launch(clmd_system* S, int step) {
  k_thermo_sum<<<S->nblk, kBlock, 0, S->stream>>>(S->P, S->st, S->perm, S->vx, S->vy, S->vz,
                                                   S->partials, step);
  k_thermo_scale<<<S->nblk, kBlock, 0, S->stream>>>(S->P, S->st, S->perm, S->vx, S->vy,
                                                     S->vz);
  S->launches += 2;
}

void stopdead_launch(clmd_system* S, int step) {
  for (int loop = 0; loop < 10; loop++) {
    k_mom_sum<<<S->nblk, kBlock, 0, S->stream>>>(S->P, S->st, S->pos, S->vx, S->vy, S->vz,
                                                  S->partials);
    k_mom_sub<<<S->nblk, kBlock, 0, S->stream>>>(S->P, S->st, S->pos, S->vx, S->vy, S->vz,
                                                  S->partials);
    S->launches += 2;
    thermostat_launch(S, step);
  }
}

void zero_acc_launch(clmd_system* S) {
  k_zero_acc<<<S->nblk, kBlock, 0, S->stream>>>(S->P.N, S->ax, S->ay, S->az);
  S->launches++;
}

void scatter_in_launch(clmd_system* S, int hx, int hy, int hz, int hvx, int hvy, int hvz,
                       int hax, int hay, int haz) {
  unsigned int m = (hx ? 1u : 0u) | (hy ? 2u : 0u) | (hz ? 4u : 0u) | (hvx ? 8u : 0u) |
                   (hvy ? 16u : 0u) | (hvz ? 32u : 0u) | (hax ? 64u : 0u) | (hay ? 128u : 0u) |
                   (haz ? 256u : 0u);
  k_scatter_in<<<S->nblk, kBlock, 0, S->stream>>>(S->P.N, S->iperm, S->sx, S->sy, S->sz,
                                                   S->vx_s, S->vy_s, S->vz_s, S->ax_s,
                                                   S->ay_s, S->az_s, S->api, S->pos, S->vx,
                                                   S->vy, S->vz, S->ax, S->ay, S->az, m);
  S->launches++;
}

void gather_out_launch(clmd_system* S) {
  k_gather_out<<<S->nblk, kBlock, 0, S->stream>>>(S->P.N, S->iperm, S->pos, S->vx, S->vy,
                                                   S->vz, S->ax, S->ay, S->az, S->sx, S->sy,
                                                   S->sz, S->vx_s, S->vy_s, S->vz_s, S->ax_s,
                                                   S->ay_s, S->az_s);
  S->launches++;
}

}  // namespace clmd
