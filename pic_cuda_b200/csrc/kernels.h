// kernels.h — internal launch interface between the host engine and the kernel files.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"

// Phase bits (same values as the public PIC_PHASE_*), plus internal ones.
#define PIC_PHASE_KICK_I 1
#define PIC_PHASE_MCC_I 2
#define PIC_PHASE_DRIFT_I 4
#define PIC_PHASE_WALLS_I 8
#define PIC_PHASE_DEPOSIT_I 16
#define PIC_PHASE_GATED_I 256   // kick/MCC only where the job's kick_pending flag is set

// One multigrid tile of one job.
struct TileRef {
  int job;
  int ti, tj;     // tile origin in owned-node units (multiply by the tile size)
  int local;      // index of this tile inside the job's tiles of the same launch
  int nlocal;     // tiles of this job in the launch
  int pbase;      // first partial-sum slot of the job
};

struct EngineLaunch {
  const JobDev* jobs;
  JobState* st;
  const SlotDev* slots;   // device slot table (pointers may be swapped by the sort)
  SlotDev* slots_mut;
  int* counts;            // live particles per slot
  int* hit_counts;        // hits of the last WALLS phase per slot
  int* aux;               // 4 ints per slot: compaction counters, lost newborns, sort descents
  int* chunk_prefix;      // nslots + 1
  const uint8_t* active;  // per slot
  int nslots;
  int njobs;
  int mover_grid;
  int num_sms;
  int* running;           // jobs whose field solve is still iterating
  unsigned* gbar;         // arrival counter of the grid barriers in mg_levels_kernel
  int* absorbed;          // particles absorbed in the last step, per slot
  cudaEvent_t ev_mover_begin, ev_mover_end;  // optional timing of the particle pass
};

int mover_blocks_per_sm();
int launch_mover(const EngineLaunch& L, int flags, uint32_t explicit_step, cudaStream_t s);
int launch_compact(const EngineLaunch& L, cudaStream_t s);
int launch_ionize(const EngineLaunch& L, bool drift_and_deposit, cudaStream_t s);
// Counting sort of the slots in sort_mask; by_disorder: the histogram pass also counts the
// particles that follow a particle of a later cell (aux[4 s + 3]), and slots where they are
// fewer than 1/32 of the particles are left as they are.
int launch_sort(const EngineLaunch& L, uint8_t* sort_mask, int max_cells, int max_particles, bool by_disorder,
                cudaStream_t s);
int launch_step_begin(JobState* st, const JobDev* jobs, int njobs, const uint8_t* job_mask, cudaStream_t s);
int launch_ke_reset_pending(JobState* st, int njobs, cudaStream_t s);
int launch_step_end(JobState* st, int njobs, const uint8_t* job_mask, int set_pending, int advance, cudaStream_t s);
void launch_pid_max(const SlotDev* slot_dev, int64_t n, JobState* st, cudaStream_t s);
int launch_zero_rho_all(const EngineLaunch& L, int max_nodes, cudaStream_t s);
int launch_sort_mask(const EngineLaunch& L, uint8_t* mask, int offset, cudaStream_t s);
int launch_vcycle_condition(cudaGraphConditionalHandle h, const int* running, int* iterations, int max_iterations,
                            unsigned long long* total, cudaStream_t s);
void launch_rho_sum(const JobDev* jd, JobState* st, double* scratch, int nparts, cudaStream_t s);

// Multigrid (all jobs of a launch at once).
struct MgLaunch {
  const TileRef* init_tiles; int n_init;                 // level-0 residual, 32x32 owned
  const int* init_jobs; int n_init_jobs;                 // every job of the solve (mg_init_finish_kernel)
  const TileRef* down_tiles[PIC_MAX_LEVELS]; int n_down[PIC_MAX_LEVELS];   // coarse 16x16 owned
  const TileRef* up_tiles[PIC_MAX_LEVELS]; int n_up[PIC_MAX_LEVELS];       // fine 32x32 owned
  const TileRef* upd_tiles; int n_upd;                   // level-0 update for jobs with lc == 0
  const int* coarse_jobs; int n_coarse;                  // single-CTA coarse solve
  const int* cluster_jobs; int n_cluster;                // thread-block-cluster coarse solve
  const int* finish_jobs; int n_finish;                  // jobs with level-0 up tiles (lc >= 1)
  int cluster_C;
  size_t cluster_smem;
  int max_depth;                                         // max lc over jobs
  size_t coarse_smem;
  int nu_pre_max, nu_post_max;                           // shared-memory sizing of the tile kernels
  int fast_nu_pre, fast_nu_post;                         // smoothing counts shared by every job, else -1
  int pdl;                                               // programmatic dependent launches in the V-cycle
  int wide_factor;                                       // 1024-thread tile CTAs on levels with <= this x SMs tiles
  int levels_grid;                                       // >0: levels 1..lc in one cooperative launch
  size_t levels_smem, levels_quarter_floats;
};
// Arguments of the cooperative launch that runs levels 1..lc of the V-cycle.
struct MgLevelsArgs {
  const TileRef* down_tiles[PIC_MAX_LEVELS]; int n_down[PIC_MAX_LEVELS];
  const TileRef* up_tiles[PIC_MAX_LEVELS]; int n_up[PIC_MAX_LEVELS];
  const int* coarse_jobs; int n_coarse;
  int max_depth;
  size_t quarter_floats;
  const JobDev* jobs;
  JobState* st;
  unsigned* gbar;
};
// Grid size (0: not available) and shared memory of the cooperative levels kernel.
int mg_levels_configure(int num_sms, int nu_pre_max, int nu_post_max, size_t coarse_smem, size_t* smem,
                        size_t* quarter_floats);
int launch_mg_init(const EngineLaunch& L, const MgLaunch& M, cudaStream_t s);
int launch_mg_vcycle(const EngineLaunch& L, const MgLaunch& M, cudaStream_t s);
void mg_configure_coarse(size_t smem_bytes);
// Shared memory of the one-CTA coarse solver for levels lc .. levels-1.
size_t mg_coarse_smem(const int* nl, int lc, int levels);
size_t mg_cluster_smem(const int* nl, int lc, int levels, int C);
int mg_cluster_supported(int C, size_t smem);
int launch_mg_cluster(const int* job_list, int njobs, int C, size_t smem, const JobDev* jobs, const JobState* st,
                      cudaStream_t s);

// Conversions between the public FP64 domain-unit layout and the engine layout.
void launch_load_species(const SlotDev* slot_dev, const JobDev* job_dev, int64_t n, const double* x,
                         const double* y, const double* vx, const double* vy, const double* vz,
                         const uint32_t* pid, uint32_t pid_base, double inv_dx, double inv_dy, int ncx,
                         int ncy, cudaStream_t s);
void launch_export_species(const SlotDev* slot_dev, int64_t n, double* x, double* y, double* vx, double* vy,
                           double* vz, uint32_t* pid, double dx, double dy, cudaStream_t s);
void launch_snapshot(const SlotDev* slot_dev, int64_t n, float* xy, double dx, double dy, cudaStream_t s);
void launch_export_raw(const SlotDev* slot_dev, int64_t n, uint32_t* cell, float* fx, float* fy, float* vx,
                       float* vy, float* vz, uint32_t* pid, cudaStream_t s);
void launch_grid_export(const JobDev* job_dev, const JobState* st_dev, int which, double* out, int nx, int ny,
                        double dx, double dy, cudaStream_t s);
void launch_grid_import(const JobDev* job_dev, const JobState* st_dev, int which, const double* in, int nx,
                        int ny, cudaStream_t s);
void launch_zero_rho(const JobDev* job_dev, int64_t nodes, int deposit_mode, void* rho, cudaStream_t s);
void launch_efield_f64(const double* phi, double* exy, int nx, int ny, double dx, double dy, cudaStream_t s);

// ---- embedded-boundary multigrid (mg_embedded.cu)
// Level arrays of one embedded solve.  phi[l] is where level l's result ends up; alt[l] is the
// second buffer the tile kernels write into (levels above the one-CTA ones); bc[l] may be
// null (DIRICHLET nodes then keep their phi).
struct EmbLevels {
  int L = 0, lc = 0;
  int nx[PIC_MAX_LEVELS] = {}, ny[PIC_MAX_LEVELS] = {};
  double* phi[PIC_MAX_LEVELS] = {};
  double* alt[PIC_MAX_LEVELS] = {};
  double* rhs[PIC_MAX_LEVELS] = {};
  uint8_t* mask[PIC_MAX_LEVELS] = {};
  const double* bc[PIC_MAX_LEVELS] = {};
  double h = 0.0;
};
// Level sizes and the first level the one-CTA kernel solves.
void emb_layout(EmbLevels& P, int nx, int ny, int levels);
// One V-cycle of Multigrid::vcycle(l0) (Multigrid_embedded.cu:159-188) on P's arrays.
int emb_vcycle(const EmbLevels& P, int l0, int nu1, int nu2, int options, cudaStream_t s);
