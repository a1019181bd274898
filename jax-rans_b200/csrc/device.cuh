// Device-side views of a case plan and the per-case solver scalars, and the launch
// wrappers every translation unit shares.  A "canvas" is one case's grid with its
// ghost ring: NI x NJ cells, j contiguous; fields are variable-major (nvar, NI*NJ) FP64.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "physics.cuh"

namespace jr {

constexpr int MAX_KRYLOV = 64;   // largest GMRES subspace
constexpr int TILE_I = 7;        // residual tile: 7 x 16 cells, 128 threads (8 x 16 i-faces)
constexpr int TILE_J = 16;
constexpr int TILE_THREADS = 128;
constexpr int TILE_MIN_BLOCKS = 3;   // three CTAs per SM at <= 168 registers
constexpr int GHOST_THREADS = 128;

// Ghost-record kinds (the order the host plan uses)
enum GhostKind { G_COPY = 0, G_SLIP = 1, G_NOSLIP = 2, G_SYMMETRY = 3, G_FARFIELD = 4, G_INFLOW = 5, G_OUTFLOW = 6 };

// Status bits of a case (device-side status word)
enum Status : int {
  ST_OK = 0,
  ST_NONFINITE = 1,       // a non-finite value met in a reduction
  ST_REJECTED = 2,        // the last Newton step was rejected
  ST_GMRES_BREAKDOWN = 4, // an Arnoldi vector of zero norm
  ST_STAGE_FAILED = 8,    // the line solve's staged copy of a factor failed (sticky: kept across steps)
};

struct Canvas {
  int NI, NJ, nvar;
  int n_cells;                 // interior cells
  const uint8_t* interior;     // NI*NJ
  const double* volume;        // NI*NJ
  const double* fi;            // i-faces: sx plane then sy plane, each (NI+1)*NJ
  const double* fj;            // j-faces: sx plane then sy plane, each NI*(NJ+1)
  const double* centres;       // x plane then y plane, each (NI+2)*(NJ+2): one ring beyond the canvas
  const double* distance;      // NI*NJ (SA) or null
  const int* neighbours;       // NI*NJ: the partner across a block face, or the cell itself
  int n_ghost[2];
  const int* g_ghost[2];
  const int* g_source[2];
  const int* g_kind[2];
  const double* g_geom[2];     // 4 per record: nx, ny, mx, my
  const int* g_src_rec;        // stage 2: the stage-1 record that fills its source, or -1
  const int* ghost_rec;        // NI*NJ: the record (stage-1 index, or n_ghost[0] + stage-2 index)
                               // that fills a canvas cell, or -1
  int n_walls;
  const int* w_cell;
  const int* w_family;
  const int* w_face;
  const double* w_into;        // +1 where the canvas face vector points into the fluid
  const double* w_mid;         // 2 per wall face
  double volume_sum;           // over interior cells
  // line chains, one thread per chain: cells [n_chains * L] chain-major-by-row
  int n_chains, L;
  const int* ch_cells;         // [k * n_chains + c], -1 past a chain's end
  const int* ch_len;           // [c]
  const int* ch_up_face;       // flat face index (i-faces first, then j-faces)
  const int* ch_up_sign;
  const int* ch_down_face;
  const int* ch_down_sign;
  const int* ch_fbase;         // [c]: sum over earlier chains of (length + 16), the factor's row offset
  int n_offchain;              // canvas cells on no chain
  const int* offchain;

  __device__ __forceinline__ int nfi() const { return (NI + 1) * NJ; }
  __device__ __forceinline__ int nfj() const { return NI * (NJ + 1); }
  __device__ __forceinline__ int ncanvas() const { return NI * NJ; }
};

// The exit test of one case, run on the device after every block of Newton steps
// (src/jaxrans/solvers/driver.py:161-190 with the force settling of
// src/jaxrans/simulation.py:259-272): the running peak of |R|, the forces after every
// block, and why the case stopped.
constexpr int MONITOR_BLOCKS = 1024;   // blocks (force samples) a monitor holds
enum MonitorReason { MON_RUNNING = 0, MON_CONVERGED = 1, MON_SETTLED = 2, MON_MAX_ITERS = 3, MON_NON_FINITE = 4,
                     MON_STALLED = 5 };
struct Monitor {
  double tol;          // converged: the block's last |R| <= tol x the running peak
  double forces_tol;   // settled: CL, CD, CM each vary by less over the last quarter (< 0: no test)
  double peak;         // the largest finite |R| so far
  int max_blocks;      // 0: the case is not monitored
  int blocks;          // blocks seen
  int reason;          // MonitorReason
  int release;         // 1: the case leaves the launches when it stops
  double coef[MONITOR_BLOCKS][3];   // CL, CD, CM after each block
};

// Per-case solver scalars, resident on the device across a whole block of steps.
struct Scalars {
  double cfl, res_prev, norm, bnorm, rnorm, beta;
  double omega, lin_red, rnorm_sq_partial;
  double nrm, inv_nrm, worst;
  double H[(MAX_KRYLOV + 1) * MAX_KRYLOV];   // column-major: H[i + (m+1) j]
  double h1[MAX_KRYLOV + 1], h2[MAX_KRYLOV + 1];
  double y[MAX_KRYLOV], hy[MAX_KRYLOV + 1];
  int active, cycle, accept, status;
  int steps, rejected, hpos;
};

struct Config {
  double cfl_max, cfl_growth, cfl_cutback, cfl_min;
  double krylov_tol, krylov_success, max_relative_update;  // < 0: none
  int restart, maxiter, preconditioner;                    // preconditioner: 0 none, 1 line_j
};

// Reduction scratch: partial sums per block, a ticket for the last-block reduction.
struct Reduce {
  double* partial;     // [blocks * width]
  unsigned int* ticket;
  int blocks;
};

// One case of a batch on the device: its canvas, physics, solver settings, buffers and
// scalars.  Kernels take a table of these and read their case from a grid dimension, so
// one launch advances every case of a batch; a single case is a batch of one.
struct CaseDev {
  Canvas c;
  Physics P;
  Config cfg;
  double *U, *qg, *dqg, *R, *b, *x, *action, *r, *w, *z, *tmp, *vdt, *dflow, *dsa, *lam, *mflux, *dflux;
  double *tile_partial, *history, *force_out;
  void* jac;                // the linearisation: per face coefficient planes of jstride values
                            // (double, or float in the mixed form)
  double* jcell;            // ... and per cell (SA: 7 planes of NI*NJ)
  double* gmap;             // ... and per ghost record: its nvar x nvar tangent map
  double* wall_out;         // per wall face: gauge pressure, area vector into the fluid (2), viscous force (2)
  void *V, *fflow, *fsa, *scratch;
  Scalars* sc;
  Monitor* mon;             // the case's exit test on the device
  double* partial;          // reduction partials of this case
  unsigned int* ticket;     // its last-block ticket
  double force_length, moment_centre[2];   // force coefficients' reference length and moment centre
  int n_vec, m, visc, mixed, n_tiles, tiles_x, tiles_y;
  int enabled;              // 0: a free slot, every kernel returns at once
  int slot;                 // the case's index in its plan (its history column)
  int jstride, jpad;        // the coefficient planes' stride (faces rounded up to 32)
};

// Buffers a kernel may be told to read or write (resolved per case)
enum Buf { B_U = 0, B_QG, B_DQG, B_R, B_B, B_X, B_ACTION, B_RR, B_W, B_Z, B_TMP, B_VDT, B_ZERO, B_NONE };

__device__ __forceinline__ double* buf(const CaseDev& cd, int id) {
  switch (id) {
    case B_U: return cd.U;
    case B_QG: return cd.qg;
    case B_DQG: return cd.dqg;
    case B_R: return cd.R;
    case B_B: return cd.b;
    case B_X: return cd.x;
    case B_ACTION: return cd.action;
    case B_RR: return cd.r;
    case B_W: return cd.w;
    case B_Z: return cd.z;
    case B_TMP: return cd.tmp;
    case B_VDT: return cd.vdt;
    default: return nullptr;
  }
}

// Copy a case's descriptor into shared memory (every thread of the block calls it).
__device__ __forceinline__ const CaseDev& stage_case(const CaseDev* cases, int ci, CaseDev* smem) {
  static_assert(sizeof(CaseDev) % 8 == 0, "CaseDev is copied in 8-byte words");
  const unsigned long long* src = reinterpret_cast<const unsigned long long*>(cases + ci);
  unsigned long long* dst = reinterpret_cast<unsigned long long*>(smem);
  for (int k = threadIdx.x; k < (int)(sizeof(CaseDev) / 8); k += blockDim.x) dst[k] = src[k];
  __syncthreads();
  return *smem;
}

// True when a block has nothing to do for its case: a free slot, a block beyond the
// case's extent (`beyond`), or a Krylov cycle that has stopped.  Read from the table in
// global memory before the descriptor is staged, so the idle blocks of a batch whose
// cases differ in size return at once.
__device__ __forceinline__ bool idle_block(const CaseDev& g, bool beyond, int check_active) {
  return !g.enabled || beyond || (check_active && g.sc->active == 0);
}

// Grid extents of a batch's launches: the largest of each per-case count.
struct BatchDims {
  int n_cases;              // cases in the launch's table
  int n_slots;              // cases of the plan (the history's row length)
  int tiles_x, tiles_y;     // residual tiles
  int ghost_records;        // both stages
  int faces, cells;         // canvas faces, canvas cells
  int n_vec;                // nvar * cells
  int chain_blocks;         // chains + off-chain blocks of the line solve
  int max_L;                // longest chain
  int cgs_blocks;           // blocks of the basis passes
  int ls_factor_threads;    // threads per chain of the line factor and of the line solve:
  int ls_apply_threads;     // the schedule the plan's autotuner picked (results do not depend on it)
  int ls_apply_stage;       // s >= 1: the line solve stages its factor from level s-1 of the longest chain
};

constexpr int LS_MAX_THREADS = 256;   // the largest line-solve block
constexpr int APPLY_STAGES = 4;       // staged line-solve forms 1..4 (0: the factor read from global memory)

// The basis passes: a block owns a chunk of cgs_chunk(n) elements of a case of n, set by
// the case's size alone (so its sums are the same in any batch): small cases (a 385 x 97
// SA case: 194k unknowns, 380 blocks) take short chunks to keep more blocks per SM,
// large ones longer chunks.
constexpr int CGS_MAX_CHUNK = 2048;
__host__ __device__ __forceinline__ int cgs_chunk(int n) {
  return n >= 2 * 148 * 2048 ? 2048 : (n >= 2 * 148 * 1024 ? 1024 : 512);
}
__host__ __device__ __forceinline__ int cgs_blocks(int n) { return (n + cgs_chunk(n) - 1) / cgs_chunk(n); }

// the number of blocks a per-case reduction over n elements uses (<= the grid's x)
__host__ __device__ __forceinline__ int chunk_blocks(int n) {
  int b = (n + 1023) / 1024;
  return b < 1 ? 1 : (b > 2 * 148 ? 2 * 148 : b);
}

}  // namespace jr
