// clmd_noalloc.cu -- the Stillinger cluster analysis for callers that cannot
// allocate device memory.
//
// Some hosts hand this library only device buffers they already own -- from
// their own memory pool or under a fixed device-memory budget reserved up
// front -- and cannot let the library call cudaMalloc (it would fail, or break
// the host's accounting).  For them, clmd_stoddard_noalloc runs the same
// analysis as stoddard() (stoddard-pbc-n-m.f: bonds, connected components
// labelled by their smallest atom number, sizes, size histogram) on caller
// buffers only.  Its one scratch array, the union-find parents, is the
// file-scope device array below: CLMD_NOALLOC_MAX_ATOMS ints (4 MiB) that
// every GPU which loads the library holds until the process exits.
//
// The array is shared by every call: calls that overlap on the GPU (two
// streams, or two host threads) race on it and must be serialised by the
// caller.  Each call re-initialises the parents it uses, so nothing needs to
// start at zero; it keeps the last call's contents.
#include <cuda_runtime.h>

#include "../../include/clmd.h"

static __device__ __align__(256) int g_noalloc_parent[CLMD_NOALLOC_MAX_ATOMS];

namespace {

// Host code cannot use g_noalloc_parent as a device address (it names a
// host-side stand-in): ask the runtime for the address on the current device
// at every call.  The lookup is cheap once the module is loaded, and a
// cached value could outlive the context it came from (after
// cudaDeviceReset the module may load at another address).  The first call
// on a device loads the module; make it before any stream capture.
int parent_address(int** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_parent);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();  // the lookup's own error, raised just now
    return CLMD_ERR_CUDA;
  }
  *out = (int*)p;
  return CLMD_OK;
}

constexpr int kThreads = 256;
constexpr int kSmallBins = 64;

__device__ __forceinline__ int na_find(int* par, int x) {
  for (;;) {
    int p = __ldcg(par + x);
    if (p == x) return x;
    int gp = __ldcg(par + p);
    if (gp != p) par[x] = gp;
    x = gp;
  }
}

// link the larger root under the smaller: the root is the smallest atom
// number of the component, the reference's label
__device__ __forceinline__ void na_union(int* par, int a, int b) {
  for (;;) {
    a = na_find(par, a);
    b = na_find(par, b);
    if (a == b) return;
    if (a < b) {
      int t = a;
      a = b;
      b = t;
    }
    if (atomicCAS(par + a, a, b) == a) return;
  }
}

// stoddard-pbc-n-m.f:60-68 (csi(0) is never reset, as in the reference)
__global__ void k_na_init(int n, int* par, int* cs, int* csi) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  par[i] = i;
  cs[i] = 0;
  csi[i + 1] = 0;
}

// stoddard-pbc-n-m.f:70-104 on the reference's atnlist()/atnidx(): atom i's
// row starts after its header at 1-based position atnidx(i); a species-2
// neighbour or the next header ends the row
__global__ void k_na_bonds(int n, const double* x, const double* y, const double* z,
                           const int* api, const int* atnlist, long long nlist,
                           const int* atnidx, double bx, double by, double bz, double bf1,
                           double bf2, double rc2, int* par) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1 || api[i] != 1) return;
  const double ibx = 1.0 / bx, iby = 1.0 / by, ibz = 1.0 / bz;
  const double tx = x[i], ty = y[i], tz = z[i];
  for (long long k = atnidx[i]; k < nlist; k++) {
    int j1 = atnlist[k];
    if (j1 < 0) break;
    int j = j1 - 1;
    if (j >= n || api[j] != 1) break;
    double dx = tx - x[j], dy = ty - y[j], dz = tz - z[j];
    dx = dx + bx * (bf1 - (double)(int)(bf2 + dx * ibx));
    dy = dy + by * (bf1 - (double)(int)(bf2 + dy * iby));
    dz = dz + bz * (bf1 - (double)(int)(bf2 + dz * ibz));
    double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 <= rc2) na_union(par, i, j);
  }
}

__global__ void k_na_label(int n, int* par, int* cl, int* cs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int r = na_find(par, i);
  cl[i] = r + 1;
  atomicAdd(cs + r, 1);
}

// stoddard-pbc-n-m.f:152-155 over the label values 1..natom
__global__ void k_na_hist(int n, const int* cs, int* csi) {
  __shared__ int h[kSmallBins];
  for (int b = threadIdx.x; b < kSmallBins; b += blockDim.x) h[b] = 0;
  __syncthreads();
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) {
    int s = cs[k];
    if (s < kSmallBins)
      atomicAdd(&h[s], 1);
    else
      atomicAdd(csi + s, 1);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < kSmallBins; b += blockDim.x)
    if (h[b]) atomicAdd(csi + b, h[b]);
}

}  // namespace

extern "C" int clmd_stoddard_noalloc(int32_t natom, const double* x, const double* y,
                                     const double* z, const int32_t* api,
                                     const int32_t* atnlist, int64_t nlist,
                                     const int32_t* atnidx, double boxx, double boxy,
                                     double boxz, double atrskin, double sigma1, double atskin,
                                     int32_t* cl, int32_t* cs, int32_t* csi, void* stream) {
  if (natom < 1 || natom > CLMD_NOALLOC_MAX_ATOMS) return CLMD_ERR_ARG;
  if (!x || !y || !z || !api || !atnlist || !atnidx || !cl || !cs || !csi || nlist < natom)
    return CLMD_ERR_ARG;
  if (!(boxx > 0 && boxy > 0 && boxz > 0 && sigma1 > 0)) return CLMD_ERR_ARG;
  // an error left by the caller's earlier work stays the caller's: report
  // it without launching and without clearing it
  if (cudaPeekAtLastError() != cudaSuccess) return CLMD_ERR_CUDA;
  int* par = nullptr;
  int st = parent_address(&par);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  // stoddard-pbc-n-m.f:53-55
  const double rc2 = atskin * atskin;
  const double bf1 = (double)(int)(atrskin / sigma1) + 2.0;
  const double bf2 = bf1 + 0.5;
  const int nb = (natom + kThreads - 1) / kThreads;
  k_na_init<<<nb, kThreads, 0, s>>>(natom, par, cs, csi);
  k_na_bonds<<<nb, kThreads, 0, s>>>(natom, x, y, z, api, atnlist, nlist, atnidx, boxx, boxy,
                                      boxz, bf1, bf2, rc2, par);
  k_na_label<<<nb, kThreads, 0, s>>>(natom, par, cl, cs);
  k_na_hist<<<nb, kThreads, 0, s>>>(natom, cs, csi);
  // the error state was clean on entry: anything pending now is these launches'
  return cudaGetLastError() == cudaSuccess ? CLMD_OK : CLMD_ERR_CUDA;
}
