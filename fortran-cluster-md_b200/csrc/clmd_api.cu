// clmd_api.cu -- the handle-based C API: system creation, host<->device
// state, one call per reference subroutine, and the device-resident main
// loop (main.f:177-228) replayed from captured CUDA graphs.  In the graphs
// each step's list rebuild sits in a conditional (IF) node whose flag the
// drift kernel sets on the device, so no step waits for the host.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "clmd_system.hpp"

using namespace clmd;

static thread_local int g_last_status = CLMD_OK;
static int set_last(int s) {
  g_last_status = s;
  return s;
}

extern "C" int32_t clmd_last_status(void) { return g_last_status; }

namespace clmd {
int check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return CLMD_OK;
  fprintf(stderr, "clmd: %s: %s\n", what, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? CLMD_ERR_NOMEM : CLMD_ERR_CUDA;
}
}  // namespace clmd

#define CK(call)                              \
  do {                                        \
    int _r = clmd::check((call), #call);      \
    if (_r != CLMD_OK) return set_last(_r);   \
  } while (0)

template <class T>
static cudaError_t dalloc(T** p, size_t n) {
  return cudaMalloc((void**)p, sizeof(T) * (n ? n : 1));
}

static void fill_params(const clmd_config* c, Params* P) {
  memset(P, 0, sizeof(*P));
  for (int s = 0; s < CLMD_MXSORTS; s++) {
    P->apmas[s] = c->apmas[s];
    P->apnum[s] = c->apnum[s];
    P->apth[s] = c->apth[s];
  }
  P->N = c->natom;
  P->atsorts = c->atsorts;
  P->boxx = c->boxx;
  P->boxy = c->boxy;
  P->boxz = c->boxz;
  P->ibx = 1.0 / c->boxx;
  P->iby = 1.0 / c->boxy;
  P->ibz = 1.0 / c->boxz;
  P->dt = c->dt;
  P->atrcut = c->atrcut;
  P->atr2 = c->atrcut * c->atrcut;
  P->atskin2 = c->atskin * c->atskin;
  P->sig1 = c->apsig[0];
  // for-a-lj-n-pbc-m.f:61-76
  double s1 = c->apsig[0], s2 = c->apsig[1];
  double c111 = s1 * s1 * s1 * s1 * s1 * s1;
  double c112 = c111 * c111;
  double c113 = 0.5 * c111;
  double c221 = s2 * s2 * s2 * s2 * s2 * s2;
  double c222 = c221 * c221;
  double c223 = 0.5 * c221;
  double c121 = 0.5 * (s1 + s2);
  c121 = c121 * c121 * c121 * c121 * c121 * c121;
  double c122 = c121 * c121;
  double c123 = 0.5 * c121;
  P->c1[2] = c111; P->c2[2] = c112; P->c3[2] = c113; P->eps[2] = c->apeps[0];
  P->c1[3] = c121; P->c2[3] = c122; P->c3[3] = c123; P->eps[3] = sqrt(c->apeps[0] * c->apeps[1]);
  P->c1[4] = c221; P->c2[4] = c222; P->c3[4] = c223; P->eps[4] = c->apeps[1];
  P->Q = c->Q;
  P->att = c->att;
  P->nkt3_i = (double)(3 * c->natom) * CLMD_CIKB * c->att;
  P->nkt3_d = 3.0 * c->natom * CLMD_CIKB * c->att;
  int n = 0;
  for (int s = 0; s < c->atsorts; s++) {
    P->ekinT[s] = 1.5 * CLMD_CIKB * c->att * c->apnum[s];
    P->sp_start[s] = n;
    n += c->apnum[s];
  }
  P->sp_start[c->atsorts] = n;
  P->nbtim = c->nbtim;
  P->btim = c->btim;
  P->atnenum = c->atnenum;
  P->csover = c->csover;
  P->clwait = c->clwait;
  P->ftcsi = c->ftcsi;
  P->integrator = c->integrator;
  P->precision = c->precision == CLMD_PREC_MIXED ? CLMD_PREC_MIXED : CLMD_PREC_FP64;
  P->r12 = c->forcevar == 'r';
  P->clustering = c->clustering;
  P->ethst = c->ethst;
  P->clnuctrl = c->clnuctrl;
}

extern "C" void clmd_scalars_init(const clmd_config* c, clmd_scalars* sc) {
  // read-3d.f:263-276
  memset(sc, 0, sizeof(*sc));
  sc->atrskin = c->atrskin;
  for (int i = 0; i < 256; i++) sc->dmmh[i] = (c->atrskin - c->atrcut) / (double)(float)c->nbtim;
  sc->dmmsu = 256.0 * (c->atrskin - c->atrcut) / (double)(float)c->nbtim;
  sc->clookfor = 1;
  sc->clookforf = 1;
  sc->cstep = -1;
  sc->last_rebuild_step = -1;
}

static int validate(const clmd_config* c) {
  if (!c || c->natom < 2 || c->atsorts < 1 || c->atsorts > CLMD_MXSORTS) return CLMD_ERR_ARG;
  long long sum = 0;
  for (int s = 0; s < c->atsorts; s++) {
    if (c->apnum[s] < 0 || c->apmas[s] <= 0.0) return CLMD_ERR_ARG;
    sum += c->apnum[s];
  }
  if (sum != c->natom) return CLMD_ERR_ARG;
  if (!(c->boxx > 0 && c->boxy > 0 && c->boxz > 0 && c->dt > 0 && c->atrcut > 0 &&
        c->atrskin >= c->atrcut && c->apsig[0] > 0 && c->nbtim > 0))
    return CLMD_ERR_ARG;
  if (c->integrator == CLMD_INT_NOSE && c->ethst == 'N' && !(c->Q > 0)) return CLMD_ERR_ARG;
  if (c->natom > (1 << 28)) return CLMD_ERR_ARG;
  return CLMD_OK;
}

extern "C" int clmd_create(const clmd_config* cfg, clmd_system** out) {
  if (!out) return set_last(CLMD_ERR_ARG);
  *out = nullptr;
  int v = validate(cfg);
  if (v) return set_last(v);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    return set_last(CLMD_ERR_NO_DEVICE);
  }
  clmd_system* S = new clmd_system();
  S->cfg = *cfg;
  fill_params(cfg, &S->P);
  Params& P = S->P;
  const int N = cfg->natom;
  CK(cudaGetDevice(&S->dev));
  CK(cudaDeviceGetAttribute(&S->num_sms, cudaDevAttrMultiProcessorCount, S->dev));
  CK(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&S->side, cudaStreamNonBlocking));
  // cell grid allocation: side >= min(atrcut, atrskin), total cells bounded
  double rmin = std::min(cfg->atrcut, cfg->atrskin) * (1.0 + 1e-9);
  int nx = std::max(1, (int)floor(cfg->boxx / rmin));
  int ny = std::max(1, (int)floor(cfg->boxy / rmin));
  int nz = std::max(1, (int)floor(cfg->boxz / rmin));
  long long cap_cells = std::max<long long>(8LL * N, 4096);
  while ((long long)nx * ny * nz > cap_cells) {
    nx = std::max(1, nx * 7 / 8);
    ny = std::max(1, ny * 7 / 8);
    nz = std::max(1, nz * 7 / 8);
  }
  P.ncx_max = nx;
  P.ncy_max = ny;
  P.ncz_max = nz;
  S->ncell_alloc = nx * ny * nz;
  // the full list holds every pair twice; a caller-given atnlist capacity
  // (headers + half pairs) is enforced with the reference's rule instead
  long long cap = cfg->nlist_cap > 0 ? 2 * cfg->nlist_cap : (long long)N * 64 + (1 << 20);
  if (cap > 0x7fffffffLL - 1024) cap = 0x7fffffffLL - 1024;
  P.list_cap = (int)cap;
  P.half_cap = cfg->nlist_cap > 0 ? cfg->nlist_cap : 0;
  S->bond_cap = (int)std::max<long long>(cap / 2, 1024);
  S->nblk = (N + kBlock - 1) / kBlock;
  size_t npart = std::max<size_t>((size_t)S->nblk * 12, (size_t)kMaxRedBlocks * 3) + 64;
  int ntiles = (S->ncell_alloc + kScanTile - 1) / kScanTile;
  size_t naux = std::max<size_t>((size_t)ntiles, (size_t)S->nblk) + 64;

  CK(dalloc(&S->pos, N));
  CK(dalloc(&S->pos_alt, N));
  CK(dalloc(&S->vx, N)); CK(dalloc(&S->vy, N)); CK(dalloc(&S->vz, N));
  CK(dalloc(&S->ax, N)); CK(dalloc(&S->ay, N)); CK(dalloc(&S->az, N));
  CK(dalloc(&S->api, N));
  CK(dalloc(&S->perm, N)); CK(dalloc(&S->iperm, N)); CK(dalloc(&S->perm_s, N));
  CK(dalloc(&S->pos_s, N));
  CK(dalloc(&S->vx_s, N)); CK(dalloc(&S->vy_s, N)); CK(dalloc(&S->vz_s, N));
  CK(dalloc(&S->ax_s, N)); CK(dalloc(&S->ay_s, N)); CK(dalloc(&S->az_s, N));
  CK(dalloc(&S->sx, N)); CK(dalloc(&S->sy, N)); CK(dalloc(&S->sz, N));
  CK(dalloc(&S->vxn, N)); CK(dalloc(&S->vyn, N)); CK(dalloc(&S->vzn, N));
  CK(dalloc(&S->list, (size_t)cap));
  CK(dalloc(&S->row_start, N)); CK(dalloc(&S->row_len, N)); CK(dalloc(&S->row_lo, N));
  CK(dalloc(&S->cell_count, S->ncell_alloc + 1));
  CK(dalloc(&S->cell_start, S->ncell_alloc + 1));
  CK(dalloc(&S->cell_fill, S->ncell_alloc + 1));
  CK(dalloc(&S->cell_atoms, N));
  CK(dalloc(&S->atom_cell, N));
  CK(dalloc(&S->scan_aux, naux));
  CK(dalloc(&S->partials, npart));
  S->cyc_blocks = cycle_blocks_for(S);
  CK(dalloc(&S->red, (size_t)2 * 16 * S->cyc_blocks + 64));
  CK(dalloc(&S->st, 1));
  CK(cudaMallocHost((void**)&S->h_sc, sizeof(clmd_scalars)));
  CK(dalloc(&S->parent, N)); CK(dalloc(&S->parent2, N));
  CK(dalloc(&S->cl, N)); CK(dalloc(&S->clf, N));
  CK(dalloc(&S->cs, N)); CK(dalloc(&S->csf, N + 1));
  CK(dalloc(&S->csi, N + 1)); CK(dalloc(&S->csif, N + 1));
  CK(dalloc(&S->cgs, N)); CK(dalloc(&S->cgsf, N + 1));
  CK(dalloc(&S->cgsa, N)); CK(dalloc(&S->cgsfa, N + 1));
  CK(dalloc(&S->cfpt, N)); CK(dalloc(&S->cfptf, N));
  CK(dalloc(&S->cek, N)); CK(dalloc(&S->cekf, N + 1));
  CK(dalloc(&S->ceks, N + 1)); CK(dalloc(&S->ceksf, N + 1));
  CK(dalloc(&S->deg, N)); CK(dalloc(&S->deg1, N));
  CK(dalloc(&S->liq, N)); CK(dalloc(&S->liqrank, N)); CK(dalloc(&S->liqref, N));
  CK(dalloc(&S->bonds, (size_t)S->bond_cap));
  CK(dalloc(&S->nbonds, 1));

  // zeroed state: list rows empty, histograms clear, cfpt = -1 (read-3d.f:297)
  CK(cudaMemsetAsync(S->st, 0, sizeof(DevState), S->stream));
  CK(cudaMemsetAsync(S->pos, 0, sizeof(double4) * N, S->stream));
  double* dz[] = {S->vx, S->vy, S->vz, S->ax, S->ay, S->az};
  for (double* p : dz) CK(cudaMemsetAsync(p, 0, sizeof(double) * N, S->stream));
  int* iz[] = {S->row_start, S->row_len, S->row_lo, S->cl, S->clf, S->cs, S->cgs, S->cgsa};
  for (int* p : iz) CK(cudaMemsetAsync(p, 0, sizeof(int) * N, S->stream));
  int* iz1[] = {S->csf, S->csi, S->csif, S->cgsf, S->cgsfa};
  for (int* p : iz1) CK(cudaMemsetAsync(p, 0, sizeof(int) * (N + 1), S->stream));
  CK(cudaMemsetAsync(S->cek, 0, sizeof(double) * N, S->stream));
  double* dz1[] = {S->cekf, S->ceks, S->ceksf};
  for (double* p : dz1) CK(cudaMemsetAsync(p, 0, sizeof(double) * (N + 1), S->stream));
  CK(cudaMemsetAsync(S->cell_count, 0, sizeof(int) * (S->ncell_alloc + 1), S->stream));
  CK(cudaMemsetAsync(S->cfpt, 0xff, sizeof(int) * N, S->stream));
  CK(cudaMemsetAsync(S->cfptf, 0xff, sizeof(int) * N, S->stream));
  // species from the contiguous blocks (read-3d.f:249-252)
  std::vector<int> api(N);
  int n = 0;
  for (int s = 0; s < cfg->atsorts; s++)
    for (int j = 0; j < cfg->apnum[s]; j++) api[n++] = s + 1;
  CK(cudaMemcpyAsync(S->api, api.data(), sizeof(int) * N, cudaMemcpyHostToDevice, S->stream));
  // storage starts in reference order
  std::vector<int> ident(N);
  for (int i = 0; i < N; i++) ident[i] = i;
  CK(cudaMemcpy(S->perm, ident.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(S->iperm, ident.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
  clmd_scalars_init(cfg, S->h_sc);
  CK(cudaMemcpyAsync(&S->st->s, S->h_sc, sizeof(clmd_scalars), cudaMemcpyHostToDevice,
                     S->stream));
  scatter_in_launch(S, 0, 0, 0, 0, 0, 0, 0, 0, 0);
  CK(cudaStreamSynchronize(S->stream));
  CK(cudaGetLastError());
  *out = S;
  return set_last(CLMD_OK);
}

static void free_graphs(clmd_system* S) {
  if (S->cyc_exec) cudaGraphExecDestroy(S->cyc_exec);
  S->cyc_exec = nullptr;
  S->graphs_ok = false;
}

extern "C" int clmd_destroy(clmd_system* S) {
  if (!S) return CLMD_OK;
  cudaStreamSynchronize(S->stream);
  free_graphs(S);
  void* ps[] = {S->pos, S->pos_alt, S->red, S->vx, S->vy, S->vz, S->ax, S->ay, S->az, S->api, S->perm, S->iperm,
                S->perm_s, S->pos_s, S->vx_s, S->vy_s, S->vz_s, S->ax_s, S->ay_s, S->az_s,
                S->liqref, S->sx, S->sy,
                S->sz, S->vxn, S->vyn, S->vzn, S->list, S->row_start, S->row_len, S->row_lo,
                S->cell_count, S->cell_start, S->cell_fill, S->cell_atoms, S->atom_cell,
                S->scan_aux, S->partials, S->st, S->parent, S->parent2, S->cl,
                S->clf, S->cs, S->csf, S->csi, S->csif, S->cgs, S->cgsf, S->cgsa, S->cgsfa,
                S->cfpt, S->cfptf, S->cek, S->cekf, S->ceks, S->ceksf, S->deg, S->deg1,
                S->liq, S->liqrank, S->bonds, S->nbonds, S->r_ocl, S->r_ocs, S->r_ocek,
                S->r_dev};
  for (void* p : ps)
    if (p) cudaFree(p);
  if (S->h_sc) cudaFreeHost(S->h_sc);
  if (S->r_host) cudaFreeHost(S->r_host);
  if (S->stream) cudaStreamDestroy(S->stream);
  if (S->side) cudaStreamDestroy(S->side);
  delete S;
  return CLMD_OK;
}

// fetch scalars (waits), return the device status
static int fetch(clmd_system* S) {
  CK(cudaMemcpyAsync(S->h_sc, &S->st->s, sizeof(clmd_scalars), cudaMemcpyDeviceToHost,
                     S->stream));
  CK(cudaStreamSynchronize(S->stream));
  CK(cudaGetLastError());
  return set_last(S->h_sc->status);
}

extern "C" int clmd_set_state(clmd_system* S, const double* x, const double* y,
                              const double* z, const double* vx, const double* vy,
                              const double* vz, const double* ax, const double* ay,
                              const double* az, const int32_t* api, const clmd_scalars* sc) {
  if (!S) return set_last(CLMD_ERR_ARG);
  const size_t nb = sizeof(double) * S->P.N;
  cudaStream_t s = S->stream;
  CK(cudaStreamSynchronize(s));
  if (api) {
    for (int i = 0; i < S->P.N; i++)
      if (api[i] < 1 || api[i] > S->P.atsorts) return set_last(CLMD_ERR_ARG);
    CK(cudaMemcpyAsync(S->api, api, sizeof(int) * S->P.N, cudaMemcpyHostToDevice, s));
  }
  const double* src[9] = {x, y, z, vx, vy, vz, ax, ay, az};
  double* stg[9] = {S->sx, S->sy, S->sz, S->vx_s, S->vy_s, S->vz_s, S->ax_s, S->ay_s, S->az_s};
  bool any = api != nullptr;
  for (int k = 0; k < 9; k++)
    if (src[k]) {
      CK(cudaMemcpyAsync(stg[k], src[k], nb, cudaMemcpyHostToDevice, s));
      any = true;
    }
  if (any)
    scatter_in_launch(S, x != nullptr, y != nullptr, z != nullptr, vx != nullptr,
                      vy != nullptr, vz != nullptr, ax != nullptr, ay != nullptr,
                      az != nullptr);
  if (sc) {
    *S->h_sc = *sc;
    CK(cudaMemcpyAsync(&S->st->s, S->h_sc, sizeof(clmd_scalars), cudaMemcpyHostToDevice, s));
  }
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return set_last(CLMD_OK);
}

extern "C" int clmd_get_state(clmd_system* S, double* x, double* y, double* z, double* vx,
                              double* vy, double* vz, double* ax, double* ay, double* az,
                              clmd_scalars* sc) {
  if (!S) return set_last(CLMD_ERR_ARG);
  const size_t nb = sizeof(double) * S->P.N;
  cudaStream_t s = S->stream;
  double* dst[9] = {x, y, z, vx, vy, vz, ax, ay, az};
  double* stg[9] = {S->sx, S->sy, S->sz, S->vx_s, S->vy_s, S->vz_s, S->ax_s, S->ay_s, S->az_s};
  bool any = false;
  for (int k = 0; k < 9; k++) any = any || dst[k];
  if (any) gather_out_launch(S);
  for (int k = 0; k < 9; k++)
    if (dst[k]) CK(cudaMemcpyAsync(dst[k], stg[k], nb, cudaMemcpyDeviceToHost, s));
  int st = fetch(S);
  if (sc) *sc = *S->h_sc;
  return st == CLMD_OK || st > 0 ? set_last(CLMD_OK) : st;
}

extern "C" int clmd_get_scalars(clmd_system* S, clmd_scalars* sc) {
  if (!S || !sc) return set_last(CLMD_ERR_ARG);
  fetch(S);
  *sc = *S->h_sc;
  return set_last(CLMD_OK);
}

extern "C" int clmd_get_config(clmd_system* S, clmd_config* cfg) {
  if (!S || !cfg) return set_last(CLMD_ERR_ARG);
  *cfg = S->cfg;
  return set_last(CLMD_OK);
}

extern "C" int clmd_set_scalars(clmd_system* S, const clmd_scalars* sc) {
  return clmd_set_state(S, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                        nullptr, nullptr, nullptr, sc);
}

__global__ void k_clear_status(DevState* st) {
  st->s.status = 0;
  st->s.fail_step = 0;
  st->s.aborted = 0;
  st->err_new = 0;
  st->bar_count = 0;  // a barrier that timed out leaves its arrivals counted
}

__global__ void k_merge_err(DevState* st) {
  int err = atomicExch(&st->err_new, 0);
  if (err && st->s.status == 0) {
    st->s.status = err;
    st->s.fail_step = st->cur_step;
  }
}

__global__ void k_debug_barrier(DevState* st, unsigned int extra, long long limit) {
  st->bar_extra = extra;
  st->bar_limit = limit;
  st->bar_count = 0;
}

extern "C" int clmd_debug_barrier(clmd_system* S, int32_t extra_arrivals, int64_t spin_limit) {
  if (!S || extra_arrivals < 0 || spin_limit < 0) return set_last(CLMD_ERR_ARG);
  CK(cudaStreamSynchronize(S->stream));
  k_debug_barrier<<<1, 1, 0, S->stream>>>(S->st, (unsigned)extra_arrivals, (long long)spin_limit);
  S->launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(S->stream));
  return set_last(CLMD_OK);
}

extern "C" int clmd_clear_status(clmd_system* S) {
  if (!S) return set_last(CLMD_ERR_ARG);
  clear_cells(S);  // a rebuild cut short by an error may have left counts
  k_clear_status<<<1, 1, 0, S->stream>>>(S->st);
  S->launches++;
  return fetch(S);
}

extern "C" int clmd_neighbor(clmd_system* S, int32_t* step) {
  if (!S || !step) return set_last(CLMD_ERR_ARG);
  k_set_step_launch(S, *step);
  cycle_launch(S, 0, 1);
  if (*step < 0) *step = -*step;  // neighbor-pbc-mav.f:63
  return fetch(S);
}

extern "C" int clmd_accatom(clmd_system* S) {
  if (!S) return set_last(CLMD_ERR_ARG);
  force_launch(S, FORCE_ACCUMULATE);
  return fetch(S);
}

extern "C" int clmd_accwall(clmd_system* S) {
  // for-w-dummy.f: no walls on the periodic nucleation path
  return set_last(S ? CLMD_OK : CLMD_ERR_ARG);
}

extern "C" int clmd_zero_acc(clmd_system* S) {
  if (!S) return set_last(CLMD_ERR_ARG);
  zero_acc_launch(S);
  return fetch(S);
}

extern "C" int clmd_integrator(clmd_system* S, int32_t step) {
  if (!S) return set_last(CLMD_ERR_ARG);
  k_set_step_launch(S, step);
  cycle_launch(S, 1, 0);
  return fetch(S);
}

extern "C" int clmd_steps(clmd_system* S, int32_t first, int32_t nsteps) {
  if (!S || nsteps < 0) return set_last(CLMD_ERR_ARG);
  k_set_step_launch(S, first);
  if (nsteps > 0) cycle_launch(S, nsteps, 0);
  return fetch(S);
}

extern "C" int clmd_set_device(int device) {
  CK(cudaSetDevice(device));
  return set_last(CLMD_OK);
}

extern "C" int clmd_thermostat(clmd_system* S, int32_t step) {
  if (!S) return set_last(CLMD_ERR_ARG);
  thermostat_launch(S, step);
  return fetch(S);
}

extern "C" int clmd_stopdead(clmd_system* S, int32_t step) {
  if (!S) return set_last(CLMD_ERR_ARG);
  stopdead_launch(S, step);
  return fetch(S);
}

extern "C" int clmd_stoddard(clmd_system* S, int32_t step) {
  if (!S) return set_last(CLMD_ERR_ARG);
  k_set_step_launch(S, step);
  stoddard_launch(S, 1);
  return fetch(S);
}

extern "C" int clmd_chk_nucleation(clmd_system* S, int32_t* step) {
  if (!S || !step) return set_last(CLMD_ERR_ARG);
  k_set_step_launch(S, *step);
  chk_nucleation_launch(S);
  int st = fetch(S);
  if (S->h_sc->aborted) *step = -*step;
  return st;
}

// main.f:179-226 with the writers off, for the steps first..first+n-1 of
// one analysis cycle: wrtCSI's stoddard at an analysis step (wrt-csi.f:27),
// chk_nucleation, then the steps (velocity scaling inside the step kernel
// when ethst == 'X', main.f:207).
static void enqueue_cycle(clmd_system* S, bool analysis, int nsteps) {
  const clmd_config& c = S->cfg;
  if (analysis && c.ftcsi != 0) stoddard_launch(S, 0);
  if (analysis && c.clnuctrl == 'X' && c.ftcsi != 0) chk_nucleation_launch(S);
  if (nsteps > 0) cycle_launch(S, nsteps, 0);
}

static int ensure_graphs(clmd_system* S) {
  if (S->graphs_ok || S->cfg.ftcsi <= 0) return CLMD_OK;
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeRelaxed));
  long long before = S->launches;
  enqueue_cycle(S, true, S->cfg.ftcsi);
  S->cyc_kernels = S->launches - before;
  S->launches = before;
  CK(cudaStreamEndCapture(S->stream, &g));
  cudaError_t e = cudaGraphInstantiate(&S->cyc_exec, g, 0);
  cudaGraphDestroy(g);
  CK(e);
  S->graphs_ok = true;
  return CLMD_OK;
}

extern "C" int clmd_run(clmd_system* S, int32_t first, int32_t nsteps, int32_t* next_step) {
  if (!S || nsteps < 0) return set_last(CLMD_ERR_ARG);
  int r = ensure_graphs(S);
  if (r) return set_last(r);
  k_set_step_launch(S, first);
  const int f = S->cfg.ftcsi;
  long long i = first, left = nsteps;
  while (left > 0) {
    if (f > 0 && i % f == 0 && left >= f) {
      CK(cudaGraphLaunch(S->cyc_exec, S->stream));  // a whole analysis cycle
      S->launches += S->cyc_kernels;
      i += f;
      left -= f;
      continue;
    }
    // a partial cycle: up to the next analysis step
    bool analysis = f > 0 && i % f == 0;
    long long n = f > 0 ? (f - (i % f + f) % f) : left;
    if (n > left) n = left;
    enqueue_cycle(S, analysis, (int)n);
    i += n;
    left -= n;
  }
  int st = fetch(S);
  if (next_step) {
    int cur = 0;
    CK(cudaMemcpy(&cur, &S->st->cur_step, sizeof(int), cudaMemcpyDeviceToHost));
    *next_step = S->h_sc->aborted ? -cur : cur;
  }
  return st;
}

// row of reference atom i: header -(i+1), then the j>i neighbours ascending
__global__ void k_halflist(int N, const int* iperm, const int* perm, const int* list,
                           const int* row_start, const int* row_len, const int* row_lo,
                           const long long* hstart, int* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int p = iperm[i];
  long long o = hstart[i];
  out[o] = -(i + 1);
  int k0 = row_start[p] + row_lo[p], k1 = row_start[p] + row_len[p];
  for (int k = k0; k < k1; k++) out[++o] = perm[list[k]] + 1;
}

__global__ void k_rowlens(int N, const int* iperm, const int* row_len, const int* row_lo,
                          int* half) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int p = iperm[i];
  half[i] = row_len[p] - row_lo[p];
}

extern "C" int clmd_get_halflist(clmd_system* S, int32_t* atnlist, int64_t cap,
                                 int32_t* atnidx, int64_t* nentries) {
  if (!S) return set_last(CLMD_ERR_ARG);
  const int N = S->P.N;
  std::vector<int> half(N);
  k_rowlens<<<S->nblk, kBlock, 0, S->stream>>>(N, S->iperm, S->row_len, S->row_lo, S->liq);
  S->launches++;
  CK(cudaMemcpyAsync(half.data(), S->liq, sizeof(int) * N, cudaMemcpyDeviceToHost,
                     S->stream));
  CK(cudaStreamSynchronize(S->stream));
  std::vector<long long> hs(N);
  long long tot = 0;
  for (int i = 0; i < N; i++) {
    hs[i] = tot;
    tot += 1 + half[i];
  }
  if (nentries) *nentries = tot;
  if (atnidx)
    for (int i = 0; i < N; i++) atnidx[i] = (int)(hs[i] + 1);
  if (atnlist) {
    if (cap < tot) return set_last(CLMD_ERR_ARG);
    long long* dhs;
    int* dout;
    CK(cudaMalloc(&dhs, sizeof(long long) * N));
    CK(cudaMalloc(&dout, sizeof(int) * (tot + 1)));
    CK(cudaMemcpyAsync(dhs, hs.data(), sizeof(long long) * N, cudaMemcpyHostToDevice,
                       S->stream));
    k_halflist<<<S->nblk, kBlock, 0, S->stream>>>(N, S->iperm, S->perm, S->list, S->row_start,
                                                   S->row_len, S->row_lo, dhs, dout);
    S->launches++;
    CK(cudaMemcpyAsync(atnlist, dout, sizeof(int) * tot, cudaMemcpyDeviceToHost, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    cudaFree(dhs);
    cudaFree(dout);
  }
  return set_last(CLMD_OK);
}

extern "C" int clmd_get_clusters(clmd_system* S, const clmd_cluster_view* v) {
  if (!S || !v) return set_last(CLMD_ERR_ARG);
  const size_t N = S->P.N;
  cudaStream_t s = S->stream;
  auto cp = [&](void* dst, const void* src, size_t bytes) -> int {
    if (!dst) return CLMD_OK;
    return clmd::check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), "D2H");
  };
  int r = 0;
  r |= cp(v->cl, S->cl, 4 * N);
  r |= cp(v->cs, S->cs, 4 * N);
  r |= cp(v->csi, S->csi, 4 * (N + 1));
  r |= cp(v->cek, S->cek, 8 * N);
  r |= cp(v->ceks, S->ceks, 8 * (N + 1));
  r |= cp(v->clf, S->clf, 4 * N);
  r |= cp(v->csf, S->csf, 4 * (N + 1));
  r |= cp(v->csif, S->csif, 4 * (N + 1));
  r |= cp(v->cekf, S->cekf, 8 * (N + 1));
  r |= cp(v->ceksf, S->ceksf, 8 * (N + 1));
  r |= cp(v->cgs, S->cgs, 4 * N);
  r |= cp(v->cgsa, S->cgsa, 4 * N);
  r |= cp(v->cgsf, S->cgsf, 4 * (N + 1));
  r |= cp(v->cgsfa, S->cgsfa, 4 * (N + 1));
  r |= cp(v->cfpt, S->cfpt, 4 * N);
  r |= cp(v->cfptf, S->cfptf, 4 * N);
  CK(cudaStreamSynchronize(s));
  return set_last(r ? CLMD_ERR_CUDA : CLMD_OK);
}

extern "C" int clmd_synchronize(clmd_system* S) {
  if (!S) return set_last(CLMD_ERR_ARG);
  CK(cudaStreamSynchronize(S->stream));
  return set_last(CLMD_OK);
}

extern "C" void* clmd_stream(clmd_system* S) { return S ? (void*)S->stream : nullptr; }

extern "C" int64_t clmd_kernel_launches(clmd_system* S) { return S ? S->launches : 0; }
