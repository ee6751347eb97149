// common.cuh — device-side tables and helpers shared by every kernel of the engine.
//
// Data layout in HBM (one engine, any number of jobs, each job has <= 4 species):
//   * particles: one "slot" per (job, species), FP32 SoA with cell-relative positions
//       cell (u32: j<<16 | i of the cell's lower-left node, or CELL_OUT),
//       fx, fy (f32 in [0,1): offset inside the cell), vx, vy, vz (f32, m/s or ref units),
//       pid (u32, stable id).  A second set of arrays is the counting-sort target.
//     Cell-relative positions keep ~1e-7-cell resolution everywhere in FP32, so slow ions
//     move every step even on 4097^2 grids (absolute FP32 grid coordinates round their
//     per-step displacement to 0 or 1 ulp).
//   * grids: node-centred, row-major j*nx+i like the reference (kernels.cu:65).
//       rho (f32 or int64 fixed point), phi64 x2 (FP64 ping-pong of the defect
//       correction), efield (float2 E per node, what the mover gathers from), multigrid
//       levels (f32).
#pragma once
#include <cstdint>
#include <cuda.h>            // CUtensorMap (the type only; nothing of the driver API is linked)
#include <cuda_runtime.h>
#include "pic_b200.h"

#define PIC_CELL_OUT 0xFFFFFFFFu
// A counting sort that falls due skips a slot whose particles are nearly in cell order: fewer
// than 1/32 of them follow a particle of a later cell (ions, which seldom leave their cell).
constexpr int kSortDisorderShift = 5;
#define PIC_MAX_LEVELS 14
#ifndef PIC_COARSE_MAX
#define PIC_COARSE_MAX 129          // largest level side the one-CTA coarse solver takes (smem)
#endif
#ifndef PIC_CHUNK
#define PIC_CHUNK 512               // particles per mover work item (256 threads x 2)
#endif
#define PIC_MOVER_THREADS 256
#define PIC_FIX_SHIFT 40            // int64 deposit: 2^40 per unit deposit charge

// Sticky device status bits (host maps them to PIC_ERR_*).
#define PIC_ST_CAPACITY 1u
#define PIC_ST_EVENTS 2u
#define PIC_ST_TIMEOUT 4u
#define PIC_ST_BADCELL 8u

struct ProcDev {
  int type, species;
  float threshold;        // eV
  int n;                  // table points
  const float* e;         // energies (eV), increasing
  const float* s;         // sigma (m^2)
  float log_e0, inv_dlog; // log-spaced lookup hint (0 if not log-spaced)
};

struct SlotDev {
  // primary arrays (swapped with the alt set by the counting sort)
  uint32_t* cell; float* fx; float* fy; float* vx; float* vy; float* vz; uint32_t* pid;
  uint32_t* cell_b; float* fx_b; float* fy_b; float* vx_b; float* vy_b; float* vz_b; uint32_t* pid_b;
  int32_t* hits;          // hit list of the last WALLS phase (capacity entries)
  int32_t* scratch;       // compaction / sort scratch (capacity entries)
  int32_t* scratch2;
  int32_t* cell_count;    // counting sort histogram / offsets (ncells + 1)
  int32_t* scan_part;     // counting sort tile sums
  int64_t capacity;
  int job, species;
  float qdep;             // deposit charge in deposit units (q W / Q_ref)
  float kx, ky;           // (q/m) dt / dx, (q/m) dt / dy : dv per unit phi difference
  float dtdx, dtdy;       // dt/dx, dt/dy : cells moved per unit velocity
  float half_m_over_e;    // 0.5 m / e : kinetic energy in eV = this * v^2
  float pnull;            // nu_max dt (candidate probability of the null-collision method)
  float numax;            // nu_max (1/s)
  float mass;             // kg (or ref units)
  int first_proc, n_proc; // this species' MCC processes in the job's process list
  ProcDev total;          // sum of this species' cross sections on the union of their energy
                          // grids (the null-collision test: real iff u nu_max < n sigma_T v)
  long long qfix;         // llrint(qdep * 2^40)
  double ke_factor;       // 0.5 m W (diagnostics)
};

struct JobDev {
  int nx, ny, ncx, ncy;   // nodes and cells
  int levels, lc;         // multigrid levels; first level solved by the coarse kernel
  int nl[PIC_MAX_LEVELS]; // level sizes (square)
  int pl[PIC_MAX_LEVELS]; // row pitch (floats) of level l's FP32 arrays e, f, eu (and f0b):
                          // nl rounded up to a multiple of 4, so every row starts 16-byte
                          // aligned (the tensor-map tile loads of the multigrid kernels)
  const CUtensorMap* tmaps;  // per level l: mgt::kTmapsPerLevel tensor maps (mg_tiles.h)
  float* e[PIC_MAX_LEVELS];   // down leg: pre-smoothed correction (coarse solver output at lc)
  float* f[PIC_MAX_LEVELS];
  // Up-leg outputs go to separate arrays: an up kernel reads its level's e and f with halos
  // that other CTAs of the same launch own, so it must not overwrite them in place.
  float* eu[PIC_MAX_LEVELS];  // up leg: post-smoothed correction of levels 1 .. lc-1
  float* f0b;                 // second level-0 right-hand side (new defect), see JobState::fsel
  float* rho_f;           // deposit_mode F32
  long long* rho_i;       // deposit_mode I64
  const double* rho_d;    // deposit_mode 2: caller-owned FP64 charge (stateless solver)
  // E at every node in units of the potential difference across one cell (-dphi: central
  // inside, one-sided on the edges), FP32 rounded from the FP64 potential: what the kick gathers
  float2* efield;
  double* phi64[3];       // FP64 iterates: DC ping-pong pair, + previous solution (warm_start 1)
  double* partials;       // per-CTA FP64 partial sums (norms)
  double h;               // grid spacing (dx == dy)
  float dt;
  double rhs_scale;       // F = rhs_scale * rho_dep (includes Q_ref and units)
  double qref;            // charge of one deposit unit
  float omega;
  int nu_pre, nu_post, nu_coarse;
  double tol;
  int max_cycles;
  int deposit_mode, wall_mode, n_walls, mcc_mode;
  const double* walls;    // n_walls x 4, grid units (x / dx)
  int n_proc;
  const ProcDev* procs;
  float gas_density, vth_neutral, gas_mass;
  int ion_e_species, ion_i_species;
  uint64_t seed;
  int slot0, nslots;
  int sort_every;
  // ionisation events
  struct Event* events;
  int event_capacity;
  int up_tiles0;          // number of CTAs of the level-0 update kernel (partials)
  int warm_start;         // 1: extrapolate the initial guess from the last two solutions
};

struct Event {            // one ionisation: parent state at collision time + products
  uint32_t parent_pid, cell;
  float fx, fy;
  float ve[3], vi[3];
};

// Mutable per-job state on the device.
struct JobState {
  long long step;          // MCC step index (the reference step whose kick precedes it)
  int kick_pending;        // kick (+MCC) of the last step not applied yet
  int converged;           // field solve reached tol (per solve)
  int cycles;              // V-cycles run in the current / last solve
  int phi_cur;             // which phi64 buffer is current
  double fnorm2, rnorm2, relres;
  uint32_t next_pid;
  uint32_t status;
  int event_count;
  int ticket;              // last-CTA-done counter for deterministic reductions
  int ionizations;
  int phi_nxt;             // phi64 buffer the next defect-correction update writes
  int phi_prev1;           // 1 + buffer holding the previous step's solution (0: none)
  int fsel;                // level-0 right-hand side in use: 0 = JobDev::f[0], 1 = JobDev::f0b
  unsigned long long collisions[PIC_MAX_SPECIES][8];
  double ke[PIC_MAX_SPECIES];
  double total_charge;     // filled on request (diagnostics)
};

// ---------------------------------------------------------------- Philox-4x32-10
__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
    const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
  }
}
// (2*(x>>9)+1) * 2^-24, exactly representable, in (0, 1).
__device__ __forceinline__ float u01(uint32_t x) {
  return (float)(2u * (x >> 9) + 1u) * 5.9604644775390625e-8f;
}
__device__ __forceinline__ void draw4(uint64_t seed, uint32_t pid, uint32_t step, uint32_t lane, float u[4]) {
  uint32_t c[4] = {pid, step, lane, 0u};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  u[0] = u01(c[0]); u[1] = u01(c[1]); u[2] = u01(c[2]); u[3] = u01(c[3]);
}

__device__ __forceinline__ uint32_t pack_cell(int i, int j) { return ((uint32_t)j << 16) | (uint32_t)i; }
__device__ __forceinline__ int cell_i(uint32_t c) { return (int)(c & 0xFFFFu); }
__device__ __forceinline__ int cell_j(uint32_t c) { return (int)(c >> 16); }

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// Warp-aggregated append: every lane with pred reserves one slot of *counter; returns the
// reserved index (or -1 for lanes without pred).
__device__ __forceinline__ int warp_append(bool pred, int* counter) {
  const unsigned m = __ballot_sync(0xffffffffu, pred);
  if (!m) return -1;
  const int leader = __ffs(m) - 1;
  int base = 0;
  if (lane_id() == leader) base = atomicAdd(counter, __popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  return pred ? base + __popc(m & ((1u << lane_id()) - 1u)) : -1;
}
