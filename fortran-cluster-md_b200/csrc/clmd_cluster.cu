// clmd_cluster.cu -- cluster analysis on the device: the Stillinger
// criterion (stoddard-pbc-n-m.f) and the ten Wolde-Frenkel liquid-atom
// criterion (stoddard-pbc-n-m-fre.f) as connected components of the bond
// graph by lock-free union-find (link the larger root under the smaller,
// path halving), the size histograms, first-passage bookkeeping, and
// chk_nucleation (chk-nucleation.f).
//
// The reference labels components by flood fill with a counter that steps
// once per atom, so a component's label is its smallest atom index
// (stoddard-pbc-n-m.f:129-150); linking roots larger-under-smaller makes the
// union-find root that same atom, so labels are identical, not just
// equivalent.  Built with -fmad=false like the MD kernels: bond tests use
// the reference's minimum-image expression bit for bit.
#include <cuda_runtime.h>

#include "clmd_system.hpp"

namespace clmd {

// Union-find over storage slots keyed by the reference index key[] (slot ->
// atom number): a root is linked under the root with the smaller key, so a
// component's root is its atom with the smallest reference index.
__device__ __forceinline__ int uf_find(int* par, int x) {
  for (;;) {
    int p = __ldcg(par + x);
    if (p == x) return x;
    int gp = __ldcg(par + p);
    if (gp != p) par[x] = gp;  // halving; keys only ever decrease along a path
    x = gp;
  }
}

__device__ __forceinline__ void uf_union(int* par, const int* key, int a, int b) {
  for (;;) {
    a = uf_find(par, a);
    b = uf_find(par, b);
    if (a == b) return;
    if (key[a] < key[b]) {
      int t = a;
      a = b;
      b = t;
    }
    int old = atomicCAS(par + a, a, b);  // a has the larger key
    if (old == a) return;
  }
}

// the main loop analyses a step once (wrt-csi.f:27 "if(cstep.ne.step)");
// a direct stoddard() call always recomputes (clu_force)
__device__ __forceinline__ bool clu_gate(const DevState* st) {
  return gated(st) || (!st->clu_force && st->s.cstep == st->cur_step);
}

__device__ __forceinline__ double kin_energy(const Params& P, int sp, double vx, double vy,
                                             double vz) {
  return 0.5 * P.apmas[sp - 1] * (vx * vx + vy * vy + vz * vz);
}

// stoddard-pbc-n-m.f:60-68 / -fre.f:60-82 resets (csi(0), ceks(0) persist)
__global__ void k_clu_init(Params P, DevState* st, int* parent, int* cs, double* cek,
                           int* csi, double* ceks, int* deg, int* deg1, int* cgs, int* clf,
                           int* csf, int* csif, double* cekf, double* ceksf, int* cgsf,
                           int* cgsa, int* cgsfa, unsigned long long* nbonds) {
  if (clu_gate(st)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool fre = P.clustering == CLMD_CLU_FRENKEL;
  if (i < P.N) {
    parent[i] = i;
    cs[i] = 0;
    cek[i] = 0.0;
    csi[i + 1] = 0;
    ceks[i + 1] = 0.0;
    if (fre) {
      deg[i] = 0;
      deg1[i] = 0;
      cgs[i] = 0;
      cgsa[i] = 0;
      clf[i] = 0;
      csf[i + 1] = 0;
      csif[i + 1] = 0;
      cekf[i + 1] = 0.0;
      ceksf[i + 1] = 0.0;
      cgsf[i + 1] = 0;
      cgsfa[i + 1] = 0;
    }
  }
  if (i == 0) {
    *nbonds = 0ull;
    st->nroots = 0;
    if (fre) {
      csif[0] = 0;
      cgsf[0] = 0;
      cgsfa[0] = 0;
      cekf[0] = 0.0;
      ceksf[0] = 0.0;
      csf[0] = 0;
    }
  }
}

// stoddard-pbc-n-m.f:70-104 / -fre.f:84-117 over the half rows (j > i,
// ascending).  Stillinger: species-1 atoms only, and a species-2 neighbour
// ends the row (:85).  tWF: every pair, with degree counts for the liquid
// test and the bond kept for the second (liquid-only) union-find.
__global__ void k_clu_bonds(Params P, DevState* st, const double4* pos, const int* perm,
                            const int* list, const int* row_start, const int* row_len,
                            const int* row_lo, int* parent, int* deg, int* deg1, int2* bonds,
                            unsigned long long* nbonds, int bond_cap) {
  if (clu_gate(st)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.N) return;
  if (perm[i] == P.N - 1) return;  // the last atom has no row (:74)
  bool fre = P.clustering == CLMD_CLU_FRENKEL;
  double4 pi = pos[i];
  int si = (int)pi.w;
  if (!fre && si != 1) return;
  const double bf1 = (double)(int)(st->s.atrskin / P.sig1) + 2.0;
  const double bf2 = bf1 + 0.5;
  int k0 = row_start[i] + row_lo[i], k1 = row_start[i] + row_len[i];
  for (int k = k0; k < k1; k++) {
    int j = list[k];
    double4 pj = pos[j];
    int sj = (int)pj.w;
    if (!fre && sj != 1) break;
    double dx = mimage_bf(pi.x - pj.x, P.boxx, P.ibx, bf1, bf2);
    double dy = mimage_bf(pi.y - pj.y, P.boxy, P.iby, bf1, bf2);
    double dz = mimage_bf(pi.z - pj.z, P.boxz, P.ibz, bf1, bf2);
    double rij2 = dx * dx + dy * dy + dz * dz;
    if (rij2 <= P.atskin2) {
      uf_union(parent, perm, i, j);
      if (fre) {
        atomicAdd(deg + i, 1);
        atomicAdd(deg + j, 1);
        if (sj == 1) atomicAdd(deg1 + i, 1);
        if (si == 1) atomicAdd(deg1 + j, 1);
        unsigned long long b = atomicAdd(nbonds, 1ull);
        if (b < (unsigned long long)bond_cap) bonds[b] = make_int2(i, j);
        else raise_err(st, CLMD_ERR_LIST_OVERFLOW);
      }
    }
  }
}

// labels (1-based, = smallest atom index of the component), sizes and
// kinetic energy per label
__global__ void k_clu_label(Params P, DevState* st, const double4* pos, const int* perm,
                            const double* vx, const double* vy, const double* vz, int* parent,
                            int* cl, int* cs, double* cek, int* cgs) {
  if (clu_gate(st)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.N) return;
  int r = perm[uf_find(parent, i)];
  cl[perm[i]] = r + 1;
  int sp = (int)pos[i].w;
  bool fre = P.clustering == CLMD_CLU_FRENKEL;
  if (fre && sp != 1) {
    atomicAdd(cgs + r, 1);  // stoddard-pbc-n-m-fre.f:177-178
  } else {
    atomicAdd(cs + r, 1);
    atomicAdd(cek + r, kin_energy(P, sp, vx[i], vy[i], vz[i]));
  }
}

// stoddard-pbc-n-m.f:152-155 / -fre.f:229-234: one histogram entry per label
// value 1..natom (labels that are not a root have cs = 0 and land in csi(0),
// which the reference never resets)
constexpr int kSmallBins = 64;

__global__ void k_clu_hist(Params P, DevState* st, const int* cs, const double* cek, int* csi,
                           double* ceks) {
  if (clu_gate(st)) return;
  __shared__ int hc[kSmallBins];
  __shared__ double he[kSmallBins];
  __shared__ int bmax;
  for (int b = threadIdx.x; b < kSmallBins; b += blockDim.x) {
    hc[b] = 0;
    he[b] = 0.0;
  }
  if (threadIdx.x == 0) bmax = 0;
  __syncthreads();
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < P.N) {
    int s = cs[k];
    double e = cek[k];
    if (s < kSmallBins) {
      atomicAdd(&hc[s], 1);
      if (e != 0.0) atomicAdd(&he[s], e);
    } else {
      atomicAdd(csi + s, 1);
      atomicAdd(ceks + s, e);
    }
    if (s > 0) atomicMax(&bmax, s);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < kSmallBins; b += blockDim.x) {
    if (hc[b]) atomicAdd(csi + b, hc[b]);
    if (he[b] != 0.0) atomicAdd(ceks + b, he[b]);
  }
  if (threadIdx.x == 0 && bmax > 0) atomicMax(&st->s.maxcs, bmax);
}

__global__ void k_clu_prep(DevState* st) {
  if (clu_gate(st)) return;
  st->s.maxcs = 0;
}

// first-passage cursor (stoddard-pbc-n-m-fre.f:229-241) and bookkeeping
__global__ void k_clu_finish(Params P, DevState* st, int* cfpt) {
  if (clu_gate(st)) return;
  clmd_scalars& q = st->s;
  int step = st->cur_step;
  q.cnum = P.N;
  if (P.clustering == CLMD_CLU_FRENKEL) {
    if (q.maxcs > q.cbiggest) q.cbiggest = q.maxcs;
    if (q.cbiggest >= q.clookfor) {
      for (int i = q.clookfor; i <= q.cbiggest; i++) cfpt[i - 1] = step;
      q.clookfor = q.clookfor + 1;
    }
  }
}

// ---- ten Wolde-Frenkel part (stoddard-pbc-n-m-fre.f:143-168, 198-258) -----

// liquid atoms and cekf(0) (species-1 atoms with >= atnenum bonds of which
// fewer than atnenum go to species 1)
__global__ void k_liq_flag(Params P, DevState* st, const double4* pos, const int* perm,
                           const double* vx, const double* vy, const double* vz,
                           const int* deg, const int* deg1, int* liq, int* liqref,
                           int* parent2, double* cekf) {
  if (clu_gate(st)) return;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= P.N) return;
  int sp = (int)pos[k].w;
  int l = 0;
  if (sp == 1 && deg[k] >= P.atnenum) {
    if (deg1[k] >= P.atnenum)
      l = 1;
    else
      atomicAdd(cekf, kin_energy(P, sp, vx[k], vy[k], vz[k]));
  }
  liq[k] = l;
  liqref[perm[k]] = l;
  parent2[k] = k;
}

// exclusive scan of liq -> rank among liquid atoms (liqmon index - 1)
__device__ __forceinline__ int bscan_excl(int v, int* sh, int* total) {
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

__global__ void k_liq_tiles(Params P, DevState* st, const int* liq, int* aux) {
  if (clu_gate(st)) return;
  __shared__ int sh[33];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int v = i < P.N ? liq[i] : 0;
  int tot;
  bscan_excl(v, sh, &tot);
  if (threadIdx.x == 0) aux[blockIdx.x] = tot;
}

__global__ void k_liq_top(DevState* st, int* aux, int ntiles) {
  if (clu_gate(st)) return;
  __shared__ int sh[33];
  int carry = 0;
  for (int b0 = 0; b0 < ntiles; b0 += blockDim.x) {
    int b = b0 + threadIdx.x;
    int v = b < ntiles ? aux[b] : 0;
    int tot;
    int ex = bscan_excl(v, sh, &tot);
    if (b < ntiles) aux[b] = carry + ex;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) st->nliq = carry;
}

__global__ void k_liq_rank(Params P, DevState* st, const int* liq, const int* aux, int* rank) {
  if (clu_gate(st)) return;
  __shared__ int sh[33];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int v = i < P.N ? liq[i] : 0;
  int tot;
  int ex = bscan_excl(v, sh, &tot);
  if (i < P.N) rank[i] = aux[blockIdx.x] + ex;
}

__global__ void k_liq_union(DevState* st, const int2* bonds, const unsigned long long* nbonds,
                            int bond_cap, const int* liq, const int* perm, int* parent2) {
  if (clu_gate(st)) return;
  unsigned long long nb = *nbonds;
  if (nb > (unsigned long long)bond_cap) nb = bond_cap;
  for (unsigned long long b = blockIdx.x * blockDim.x + threadIdx.x; b < nb;
       b += (unsigned long long)gridDim.x * blockDim.x) {
    int2 e = bonds[b];
    if (liq[e.x] && liq[e.y]) uf_union(parent2, perm, e.x, e.y);
  }
}

// tWF labels are the rank (1-based) of the component's smallest liquid atom
// in liqmon(); the reference leaves clf() of non-liquid atoms as whatever
// the flood fill wrote (:215-218), the engine writes 0 there.
__global__ void k_liq_label(Params P, DevState* st, const double4* pos, const int* perm,
                            const double* vx, const double* vy, const double* vz,
                            const int* liq, const int* rank, int* parent2, int* clf, int* csf,
                            double* cekf) {
  if (clu_gate(st)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.N) return;
  if (!liq[i]) {
    clf[perm[i]] = 0;
    return;
  }
  int r = perm[uf_find(parent2, i)];
  int lab = rank[r] + 1;
  clf[perm[i]] = lab;
  atomicAdd(csf + lab, 1);
  int sp = (int)pos[i].w;
  atomicAdd(cekf + lab, kin_energy(P, sp, vx[i], vy[i], vz[i]));
}

__global__ void k_liq_hist(Params P, DevState* st, const int* csf, const double* cekf,
                           const int* cgsf, int* csif, double* ceksf, int* cgsfa) {
  if (clu_gate(st)) return;
  __shared__ int bmax;
  if (threadIdx.x == 0) bmax = 0;
  __syncthreads();
  int r = blockIdx.x * blockDim.x + threadIdx.x + 1;  // rank label 1..nliq
  if (r <= st->nliq) {
    int s = csf[r];
    if (s > 0) {
      atomicAdd(csif + s, 1);
      atomicAdd(ceksf + s, cekf[r]);
      atomicAdd(cgsfa + s, cgsf[r]);
      atomicMax(&bmax, s);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) atomicMax(&st->nroots_f, bmax);
}

__global__ void k_liq_finish(Params P, DevState* st, int* csif, int* cfptf) {
  if (clu_gate(st)) return;
  clmd_scalars& q = st->s;
  int step = st->cur_step;
  q.cnumf = st->nliq;
  csif[0] = P.apnum[0] - st->nliq;  // :251 (sum of csf = number of liquid atoms)
  int bf = st->nroots_f;
  if (bf > q.cbiggestf) q.cbiggestf = bf;
  if (q.cbiggestf >= q.clookforf) {
    for (int i = q.clookforf; i <= q.cbiggestf; i++) cfptf[i - 1] = step;
    q.clookforf = q.clookforf + 1;
  }
  st->nroots_f = 0;
}

// cstep = step marks the analysis done for this step (wrt-csi.f:27)
__global__ void k_clu_done(DevState* st) {
  if (clu_gate(st)) return;
  st->s.cstep = st->cur_step;
  st->clu_force = 0;
  int err = atomicExch(&st->err_new, 0);
  if (err && st->s.status == 0) {
    st->s.status = err;
    st->s.fail_step = st->cur_step;
  }
}

// chk-nucleation.f:33-56 on the histogram just computed
__global__ void k_chk_nucleation(Params P, DevState* st, const int* csi) {
  if (gated(st)) return;
  clmd_scalars& q = st->s;
  int step = st->cur_step;
  bool hit;
  if (P.csover >= 1)
    hit = q.maxcs >= P.csover && P.csover <= P.N;
  else
    hit = csi[0] > 0 || q.maxcs >= 1;
  int tim = hit ? step : 0;
  if (tim > 0) {
    if (q.clbrkt == 0) {
      q.clbrkt = tim;
    } else if ((tim - q.clbrkt) >= P.clwait) {
      q.aborted = 1;  // step = -step (main.f:219-220 leaves the loop)
    }
  } else {
    q.clbrkt = 0;
  }
}

__global__ void k_clu_force(DevState* st, int f) { st->clu_force = f; }

void stoddard_launch(clmd_system* S, int force) {
  const Params& P = S->P;
  cudaStream_t s = S->stream;
  int nb = S->nblk;
  if (force) {
    k_clu_force<<<1, 1, 0, s>>>(S->st, 1);
    S->launches++;
  }
  k_clu_prep<<<1, 1, 0, s>>>(S->st);
  k_clu_init<<<nb, kBlock, 0, s>>>(P, S->st, S->parent, S->cs, S->cek, S->csi, S->ceks,
                                    S->deg, S->deg1, S->cgs, S->clf, S->csf, S->csif, S->cekf,
                                    S->ceksf, S->cgsf, S->cgsa, S->cgsfa, S->nbonds);
  k_clu_bonds<<<nb, kBlock, 0, s>>>(P, S->st, S->pos, S->perm, S->list, S->row_start,
                                     S->row_len, S->row_lo, S->parent, S->deg, S->deg1,
                                     S->bonds, S->nbonds, S->bond_cap);
  k_clu_label<<<nb, kBlock, 0, s>>>(P, S->st, S->pos, S->perm, S->vx, S->vy, S->vz, S->parent,
                                     S->cl, S->cs, S->cek, S->cgs);
  k_clu_hist<<<nb, kBlock, 0, s>>>(P, S->st, S->cs, S->cek, S->csi, S->ceks);
  k_clu_finish<<<1, 1, 0, s>>>(P, S->st, S->cfpt);
  S->launches += 6;
  if (P.clustering == CLMD_CLU_FRENKEL) {
    k_liq_flag<<<nb, kBlock, 0, s>>>(P, S->st, S->pos, S->perm, S->vx, S->vy, S->vz, S->deg,
                                      S->deg1, S->liq, S->liqref, S->parent2, S->cekf);
    k_liq_tiles<<<nb, kBlock, 0, s>>>(P, S->st, S->liqref, S->scan_aux);
    k_liq_top<<<1, 1024, 0, s>>>(S->st, S->scan_aux, nb);
    k_liq_rank<<<nb, kBlock, 0, s>>>(P, S->st, S->liqref, S->scan_aux, S->liqrank);
    int ub = 4 * S->num_sms;
    k_liq_union<<<ub, kBlock, 0, s>>>(S->st, S->bonds, S->nbonds, S->bond_cap, S->liq,
                                       S->perm, S->parent2);
    k_liq_label<<<nb, kBlock, 0, s>>>(P, S->st, S->pos, S->perm, S->vx, S->vy, S->vz, S->liq,
                                       S->liqrank, S->parent2, S->clf, S->csf, S->cekf);
    k_liq_hist<<<nb, kBlock, 0, s>>>(P, S->st, S->csf, S->cekf, S->cgsf, S->csif, S->ceksf,
                                      S->cgsfa);
    k_liq_finish<<<1, 1, 0, s>>>(P, S->st, S->csif, S->cfptf);
    S->launches += 8;
  }
  k_clu_done<<<1, 1, 0, s>>>(S->st);
  S->launches += 1;
}

void chk_nucleation_launch(clmd_system* S) {
  k_chk_nucleation<<<1, 1, 0, S->stream>>>(S->P, S->st, S->csi);
  S->launches++;
}

}  // namespace clmd
