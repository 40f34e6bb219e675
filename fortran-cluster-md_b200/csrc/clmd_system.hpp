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
  double *vx = nullptr, *vy = nullptr, *vz = nullptr;
  double *ax = nullptr, *ay = nullptr, *az = nullptr;
  int* api = nullptr;
  double *sx = nullptr, *sy = nullptr, *sz = nullptr;     // staging / scratch
  double *vxn = nullptr, *vyn = nullptr, *vzn = nullptr;  // Nose-Hoover iterate
  // neighbour list
  int* list = nullptr;
  int *row_start = nullptr, *row_len = nullptr, *row_lo = nullptr;
  int *cell_count = nullptr, *cell_start = nullptr, *cell_fill = nullptr;
  int *cell_atoms = nullptr, *atom_cell = nullptr;
  double4* spos = nullptr;
  int* scan_aux = nullptr;
  int ncell_alloc = 0;
  // reductions / scalars
  double* partials = nullptr;
  clmd::DevState* st = nullptr;
  clmd_scalars* h_sc = nullptr;  // pinned
  // cluster analysis
  int *parent = nullptr, *parent2 = nullptr;
  int *cl = nullptr, *clf = nullptr, *cs = nullptr, *csf = nullptr, *csi = nullptr,
      *csif = nullptr;
  int *cgs = nullptr, *cgsf = nullptr, *cgsa = nullptr, *cgsfa = nullptr, *cfpt = nullptr,
      *cfptf = nullptr;
  double *cek = nullptr, *cekf = nullptr, *ceks = nullptr, *ceksf = nullptr;
  int *deg = nullptr, *deg1 = nullptr, *liq = nullptr, *liqrank = nullptr;
  int2* bonds = nullptr;
  unsigned long long* nbonds = nullptr;
  int bond_cap = 0;
  // launch geometry
  int nblk = 1;          // ceil(N / kBlock)
  int coop_blocks = 1;   // co-resident blocks of the cooperative solve
  long long launches = 0;
  // captured main-loop graphs
  cudaGraphExec_t cyc_exec = nullptr;   // ftcsi steps, analysis first
  cudaGraphExec_t step_exec = nullptr;  // one plain step
  long long cyc_kernels = 0, step_kernels = 0;
  bool graphs_ok = false;
};

namespace clmd {

int check(cudaError_t e, const char* what);

// clmd_md.cu
void k_set_step_launch(clmd_system* S, int step);
void k_step_advance_launch(clmd_system* S);
void nb_prologue_launch(clmd_system* S);
void rebuild_launch(clmd_system* S, cudaStream_t s);
void drift_launch(clmd_system* S, unsigned long long cond, int use_cond);
void force_launch(clmd_system* S, int mode);
void nh_solve_launch(clmd_system* S);
void thermostat_launch(clmd_system* S, int step);
void stopdead_launch(clmd_system* S, int step);
void zero_acc_launch(clmd_system* S);
void pack_pos_launch(clmd_system* S, int have_x, int have_y, int have_z);
void unpack_pos_launch(clmd_system* S);
int coop_blocks_for(clmd_system* S);

// clmd_cluster.cu
void stoddard_launch(clmd_system* S, int force);
void chk_nucleation_launch(clmd_system* S);

enum ForceMode { FORCE_ACCUMULATE = 0, FORCE_VV_KICK = 1, FORCE_ZERO_FIRST = 2 };

}  // namespace clmd
