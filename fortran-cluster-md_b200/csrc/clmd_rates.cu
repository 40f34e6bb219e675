// clmd_rates.cu -- the routines that act on the largest cluster.
//
// rates(step) (rates.f:44-100): atoms that condensed on or
// evaporated from the largest cluster between two cluster analyses, on the
// device: the previous labels are kept, the largest cluster before and after
// is an atomic max over (size, -label) keys, and the two counts are block
// reductions; the host keeps the reference's running sums and writes its
// fixed-format lines.
//
// thermostat(step) of scalev-clu.f:41-83: every ecltim steps the biggest
// cluster and the gas are scaled to the temperature separately, otherwise
// all atoms with one factor from the current ekin.
#include <cuda_runtime.h>
#include <stdio.h>

#include "clmd_system.hpp"

namespace clmd {

namespace {

constexpr int kRB = 256;

// key = size << 32 | (0xffffffff - label index): the max is the largest
// size, and among equal sizes the first label, as rates.f:56-67's strict >
__global__ void k_rates_max(int n, const int* ocs, const int* cs, unsigned long long* keys) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long ko = 0, kn = 0;
  if (i < n) {
    const unsigned long long tag = 0xffffffffull - (unsigned long long)i;
    if (ocs[i] > 0) ko = ((unsigned long long)ocs[i] << 32) | tag;
    if (cs[i] > 0) kn = ((unsigned long long)cs[i] << 32) | tag;
  }
  for (int o = 16; o > 0; o >>= 1) {
    ko = max(ko, __shfl_xor_sync(0xffffffffu, ko, o));
    kn = max(kn, __shfl_xor_sync(0xffffffffu, kn, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&keys[0], ko);
    atomicMax(&keys[1], kn);
  }
}

__device__ __forceinline__ int key_label(unsigned long long k) {
  return (int)(0xffffffffull - (k & 0xffffffffull)) + 1;  // 1-based label
}

// rates.f:69-73
__global__ void k_rates_count(int n, const int* cl, const int* ocl, unsigned long long* r) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int omcln = key_label(r[0]), mcln = key_label(r[1]);
  int cn = 0, en = 0;
  if (i < n) {
    cn = (cl[i] == mcln && ocl[i] != omcln);
    en = (cl[i] != mcln && ocl[i] == omcln);
  }
  cn = __reduce_add_sync(0xffffffffu, cn);
  en = __reduce_add_sync(0xffffffffu, en);
  if ((threadIdx.x & 31) == 0) {
    if (cn) atomicAdd(&r[2], (unsigned long long)cn);
    if (en) atomicAdd(&r[3], (unsigned long long)en);
  }
}

// the two clusters' kinetic energies (cek(mcln), ocek(omcln))
__global__ void k_rates_pick(const double* cek, const double* ocek, unsigned long long* r) {
  double* d = (double*)(r + 4);
  d[0] = r[1] ? cek[key_label(r[1]) - 1] : 0.0;
  d[1] = r[0] ? ocek[key_label(r[0]) - 1] : 0.0;
}

void put_i(FILE* f, long long v, int w) {
  char b[32];
  int n = snprintf(b, sizeof(b), "%lld", v);
  if (n > w)
    for (int k = 0; k < w; k++) fputc('*', f);
  else
    fprintf(f, "%*s", w, b);
}

void put_f(FILE* f, double v, int w, int d) {
  char b[64];
  int n = snprintf(b, sizeof(b), "%.*f", d, v);
  if (n > w || v != v)
    for (int k = 0; k < w; k++) fputc('*', f);
  else
    fprintf(f, "%*s", w, b);
}

// ---- scalev-clu.f: the biggest cluster and the gas scaled separately ------
__global__ void k_big_key(int n, const int* cs, unsigned long long* key) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long k = 0;
  if (i < n && cs[i] > 0) k = ((unsigned long long)cs[i] << 32) | (0xffffffffull - i);
  for (int o = 16; o > 0; o >>= 1) k = max(k, __shfl_xor_sync(0xffffffffu, k, o));
  if ((threadIdx.x & 31) == 0) atomicMax(key, k);
}

// per block: sum of cek over the labels other than the biggest one, in a
// fixed tree (deterministic)
__global__ void k_gas_ekin(int n, const double* cek, const unsigned long long* key,
                           double* partials) {
  __shared__ double sh[kRB / 32];
  const int ci = key_label(*key) - 1;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v = (i < n && i != ci) ? cek[i] : 0.0;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kRB / 32; w++) t += sh[w];
    partials[blockIdx.x] = t;
  }
}

// scalev-clu.f:58-59: kfG and kfC from the block sums, added in order
__global__ void k_clu_factors(Params P, int nb, const double* partials, const int* cs,
                              const double* cek, const unsigned long long* key, double* kf) {
  if (*key == 0) {  // no cluster record (no analysis has run): leave v alone
    kf[0] = 1.0;
    kf[1] = 1.0;
    return;
  }
  double ekinG = 0.0;
  for (int b = 0; b < nb; b++) ekinG += partials[b];
  const int ci = key_label(*key) - 1;
  const double cikb = CLMD_CIKB;
  kf[0] = sqrt(1.5 * cikb * P.att * (double)(P.N - cs[ci]) / ekinG);  // gas
  kf[1] = sqrt(1.5 * cikb * P.att * (double)cs[ci] / cek[ci]);        // cluster
}

// scalev-clu.f:60-70 (mode 1) or :75-80 (mode 0, one factor for all)
__global__ void k_clu_scale(Params P, DevState* st, const int* perm, const int* cl, double* vx,
                            double* vy, double* vz, const double* kf,
                            const unsigned long long* key, int mode, double ekinT) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0) st->s.ekin = ekinT;  // :82
  if (p >= P.N) return;
  double k = kf[0];
  if (mode == 1 && cl[perm[p]] == key_label(*key)) k = kf[1];
  vx[p] = vx[p] * k;
  vy[p] = vy[p] * k;
  vz[p] = vz[p] * k;
}

}  // namespace
}  // namespace clmd

using namespace clmd;

extern "C" int clmd_thermostat_clu(clmd_system* S, int32_t step, char eclth, int32_t ecltim) {
  if (!S) return CLMD_ERR_ARG;
  const bool clu = eclth == 'X';
  if (clu && ecltim <= 0) return CLMD_ERR_ARG;
  const int n = S->P.N;
  cudaStream_t st = S->stream;
  if (!S->r_dev) {
    if (cudaMalloc(&S->r_dev, 8 * 6) != cudaSuccess ||
        cudaMallocHost(&S->r_host, 8 * 6) != cudaSuccess) {
      cudaGetLastError();
      return CLMD_ERR_NOMEM;
    }
  }
  clmd_scalars q;
  int rc = clmd_get_scalars(S, &q);
  if (rc) return rc;
  const double ekinT = 1.5 * CLMD_CIKB * S->P.att * (double)n;
  const int nb = (n + kRB - 1) / kRB;
  unsigned long long* key = S->r_dev;
  double* kf = (double*)(S->r_dev + 4);
  int mode = 0;
  if (clu && step % ecltim == 0) {
    if (q.cstep != step) {
      rc = clmd_stoddard(S, step);
      if (rc) return rc;
    }
    mode = 1;
    cudaMemsetAsync(key, 0, 8, st);
    k_big_key<<<nb, kRB, 0, st>>>(n, S->cs, key);
    k_gas_ekin<<<nb, kRB, 0, st>>>(n, S->cek, key, S->partials);
    k_clu_factors<<<1, 1, 0, st>>>(S->P, nb, S->partials, S->cs, S->cek, key, kf);
    S->launches += 3;
  } else {
    const double k = sqrt(ekinT / q.ekin);  // :75 uses the current ekin
    cudaMemcpyAsync(kf, &k, 8, cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);
  }
  k_clu_scale<<<nb, kRB, 0, st>>>(S->P, S->st, S->perm, S->cl, S->vx, S->vy, S->vz, kf, key,
                                   mode, ekinT);
  S->launches++;
  return clmd_get_scalars(S, &q);
}

extern "C" int clmd_rates(clmd_system* S, int32_t step, int32_t ctrat, clmd_rates_acc* acc,
                          const char* out, const char* log) {
  if (!S || !acc || ctrat < 1) return CLMD_ERR_ARG;
  const int n = S->P.N;
  cudaStream_t st = S->stream;
  if (!S->r_ocl) {
    if (cudaMalloc(&S->r_ocl, sizeof(int) * n) != cudaSuccess ||
        cudaMalloc(&S->r_ocs, sizeof(int) * n) != cudaSuccess ||
        cudaMalloc(&S->r_ocek, sizeof(double) * n) != cudaSuccess ||
        cudaMalloc(&S->r_dev, 8 * 6) != cudaSuccess ||
        cudaMallocHost(&S->r_host, 8 * 6) != cudaSuccess) {
      cudaGetLastError();
      return CLMD_ERR_NOMEM;
    }
  }
  // rates.f:44-48
  cudaMemcpyAsync(S->r_ocl, S->cl, sizeof(int) * n, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(S->r_ocs, S->cs, sizeof(int) * n, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(S->r_ocek, S->cek, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
  clmd_scalars q;
  int rc = clmd_get_scalars(S, &q);
  if (rc) return rc;
  FILE* lg = log ? fopen(log, "a") : stdout;
  if (!lg) return CLMD_ERR_ARG;
  if (q.cstep != step) {  // :50-54
    rc = clmd_stoddard(S, step);
    if (rc) {
      if (log) fclose(lg);
      return rc;
    }
  } else {
    fprintf(lg, " *** WARNING *** No old Stoddard-list !!\n");
  }
  cudaMemsetAsync(S->r_dev, 0, 8 * 6, st);
  const int nb = (n + kRB - 1) / kRB;
  k_rates_max<<<nb, kRB, 0, st>>>(n, S->r_ocs, S->cs, S->r_dev);
  k_rates_count<<<nb, kRB, 0, st>>>(n, S->cl, S->r_ocl, S->r_dev);
  k_rates_pick<<<1, 1, 0, st>>>(S->cek, S->r_ocek, S->r_dev);
  S->launches += 3;
  cudaMemcpyAsync(S->r_host, S->r_dev, 8 * 6, cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    if (log) fclose(lg);
    return CLMD_ERR_CUDA;
  }
  const unsigned long long* r = S->r_host;
  const int omcs = (int)(r[0] >> 32), mcs = (int)(r[1] >> 32);
  const int omcln = r[0] ? (int)(0xffffffffull - (r[0] & 0xffffffffull)) + 1 : 0;
  const int mcln = r[1] ? (int)(0xffffffffull - (r[1] & 0xffffffffull)) + 1 : 0;
  const int cn = (int)r[2], en = (int)r[3];
  const double* d = (const double*)(r + 4);
  if (mcs != omcs) {  // :75-76, format (I12,4(2X,I5),2(2X,I2))
    put_i(lg, step, 12);
    const int v4[4] = {omcs, mcs, omcln, mcln};
    for (int k = 0; k < 4; k++) {
      fputs("  ", lg);
      put_i(lg, v4[k], 5);
    }
    fputs("  ", lg);
    put_i(lg, cn, 2);
    fputs("  ", lg);
    put_i(lg, en, 2);
    fputc('\n', lg);
  }
  if (log) fclose(lg);
  // :78-98
  const double cikb = CLMD_CIKB;
  const double mct = d[0] / ((double)mcs * 1.5 * cikb);
  acc->mcts = acc->mcts + mct;
  const double omct = d[1] / ((double)omcs * 1.5 * cikb);
  acc->omcts = acc->omcts + omct;
  acc->cen = acc->cen + en;
  acc->ccn = acc->ccn + cn;
  bool write = false;
  double c4 = mct, c5 = omct;
  int c6 = cn, c7 = en;
  if (ctrat != 1) {
    if (step % ctrat == 0) {
      write = true;
      c4 = acc->mcts / (double)(float)ctrat;
      c5 = acc->omcts / (double)(float)ctrat;
      c6 = acc->ccn;
      c7 = acc->cen;
      acc->ccn = 0;
      acc->cen = 0;
      acc->mcts = 0.0;  // omcts keeps accumulating, as in the reference
    }
  } else if (en + cn != 0) {
    write = true;
  }
  if (write && out) {  // format (I12,2(1X,I6),2(1X,F10.4),2(1X,I3),2(1X,I6))
    FILE* f = fopen(out, "a");
    if (!f) return CLMD_ERR_ARG;
    put_i(f, step, 12);
    fputc(' ', f); put_i(f, omcs, 6);
    fputc(' ', f); put_i(f, mcs, 6);
    fputc(' ', f); put_f(f, c4, 10, 4);
    fputc(' ', f); put_f(f, c5, 10, 4);
    fputc(' ', f); put_i(f, c6, 3);
    fputc(' ', f); put_i(f, c7, 3);
    fputc(' ', f); put_i(f, mcln, 6);
    fputc(' ', f); put_i(f, omcln, 6);
    fputc('\n', f);
    fclose(f);
  }
  return CLMD_OK;
}
