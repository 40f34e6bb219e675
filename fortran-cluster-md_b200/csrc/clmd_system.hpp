// clmd_system.hpp -- host-side handle of one simulated system and the
// launchers each translation unit provides.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "clmd_internal.cuh"

struct clmd_system {
  clmd_config cfg;
  clmd::Params P;
  int dev = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;  // body capture of conditional nodes
  // per-atom state
  double4* pos = nullptr;
  double4* pos_alt = nullptr;  // second position buffer of the fused steps
  double *vx = nullptr, *vy = nullptr, *vz = nullptr;
  double *ax = nullptr, *ay = nullptr, *az = nullptr;
  int* api = nullptr;                 // species by reference index (staging)
  int *perm = nullptr, *iperm = nullptr;  // slot -> reference index, inverse
  // reorder scratch (a rebuild gathers the state into cell order here)
  double4* pos_s = nullptr;
  double *vx_s = nullptr, *vy_s = nullptr, *vz_s = nullptr;
  double *ax_s = nullptr, *ay_s = nullptr, *az_s = nullptr;
  int* perm_s = nullptr;
  double *sx = nullptr, *sy = nullptr, *sz = nullptr;     // staging / scratch
  double *vxn = nullptr, *vyn = nullptr, *vzn = nullptr;  // Nose-Hoover iterate
  // neighbour list
  int* list = nullptr;
  int *row_start = nullptr, *row_len = nullptr, *row_lo = nullptr;
  int *cell_count = nullptr, *cell_start = nullptr, *cell_fill = nullptr;
  int *cell_atoms = nullptr, *atom_cell = nullptr;
  int* scan_aux = nullptr;
  int ncell_alloc = 0;
  // reductions / scalars
  double* partials = nullptr;
  double* red = nullptr;     // partial sums of the persistent kernel
  clmd::DevState* st = nullptr;
  clmd_scalars* h_sc = nullptr;  // pinned
  // cluster analysis
  int *parent = nullptr, *parent2 = nullptr;
  int *cl = nullptr, *clf = nullptr, *cs = nullptr, *csf = nullptr, *csi = nullptr,
      *csif = nullptr;
  int *cgs = nullptr, *cgsf = nullptr, *cgsa = nullptr, *cgsfa = nullptr, *cfpt = nullptr,
      *cfptf = nullptr;
  double *cek = nullptr, *cekf = nullptr, *ceks = nullptr, *ceksf = nullptr;
  int *deg = nullptr, *deg1 = nullptr, *liq = nullptr, *liqrank = nullptr, *liqref = nullptr;
  int2* bonds = nullptr;
  unsigned long long* nbonds = nullptr;
  int bond_cap = 0;
  // rates(): the previous analysis (rates.f's ocs/ocl/ocek) and the picks
  int *r_ocl = nullptr, *r_ocs = nullptr;
  double* r_ocek = nullptr;
  unsigned long long* r_dev = nullptr;  // 2 keys, 2 counts, 2 doubles
  unsigned long long* r_host = nullptr; // pinned copy
  // launch geometry
  int nblk = 1;          // ceil(N / kBlock)
  int cyc_blocks = 1;    // co-resident blocks of the persistent kernel
  long long launches = 0;
  // captured main-loop graph: analysis + ftcsi steps
  cudaGraphExec_t cyc_exec = nullptr;
  long long cyc_kernels = 0;
  bool graphs_ok = false;
};

namespace clmd {

int check(cudaError_t e, const char* what);

// clmd_md.cu
void k_set_step_launch(clmd_system* S, int step);
void clear_cells(clmd_system* S);
void force_launch(clmd_system* S, int mode, int advance = 0);
void thermostat_launch(clmd_system* S, int step);
void stopdead_launch(clmd_system* S, int step);
void zero_acc_launch(clmd_system* S);
// host I/O through the slot permutation: staging arrays (reference order)
// <-> state (slot order)
void scatter_in_launch(clmd_system* S, int hx, int hy, int hz, int hvx, int hvy, int hvz,
                       int hax, int hay, int haz);
void gather_out_launch(clmd_system* S);

// clmd_cycle.cu: the persistent step kernel (mode 0: nsteps integrator
// steps; mode 1: one neighbor() rebuild)
int cycle_blocks_for(clmd_system* S);
void cycle_launch(clmd_system* S, int nsteps, int mode);

// clmd_cluster.cu
void stoddard_launch(clmd_system* S, int force);
void chk_nucleation_launch(clmd_system* S);

enum ForceMode { FORCE_ACCUMULATE = 0, FORCE_VV_KICK = 1, FORCE_ZERO_FIRST = 2 };

}  // namespace clmd
