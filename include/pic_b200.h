/*
 * pic_b200.h — C ABI of the B200-native 2D electrostatic PIC step.
 *
 * One engine owns a device memory pool and steps every job it holds together
 * (a plain simulation is an engine with one job).  All signatures use plain C
 * types: device streams are passed as `void*` (a cudaStream_t), host or device
 * arrays as plain pointers plus sizes.  Every function returns a PIC_* status;
 * pic_last_error() gives a message for the last failure on the calling thread.
 *
 * Reference interface each entry point replaces (file:line in dimad285/PIC_CUDA):
 *   pic_job_create            Grid2D::Grid2D (grid.cu:10), Particles2D::Particles2D
 *                             (particles.cu:112), add_species (particles.cu:174),
 *                             Boundaries2D::add_wall/compile_walls (boundaries.cu:3,11)
 *   pic_job_load_species      the host->device copies of r, r_old, v in main.cu:232-238
 *   pic_step                  updateSimulationCUDA (main.cu:37-140)
 *   pic_job_run_phases        the individual kernels of the step: update_coordinates
 *                             (kernels.cu:8), detect_intersections (collisions.cu:7),
 *                             updateDensity (kernels.cu:26), updateParticleVelocities
 *                             (kernels.cu:71), collision_kernel (mcc.cu:56)
 *   pic_job_compact           Particles2D::removeCollidedParticles (particles.cu:217)
 *   pic_job_solve_field       solve_multigrid applied to the job's own rho/phi
 *                             (Multigrid.cu:573), plus computeElectricField (kernels.cu:134)
 *   pic_solve_multigrid_f64   solve_multigrid (Multigrid.hpp:3-11, Multigrid.cu:573-642)
 *                             on caller-owned FP64 device arrays
 *   pic_efield_f64            computeElectricField (kernels.cu:134-191) on FP64 arrays
 *   pic_solve_embedded_f64    Multigrid::vcycle of Multigrid_embedded.cu:110-188 (masked
 *                             nodes, interior electrodes) driven to a tolerance
 *   pic_job_export_species    Particles2D::debugParticles read-back (particles.cu:200)
 *   pic_job_snapshot_positions  convertPositionsToFloat into the viewer's vertex buffer
 *                             (kernels.cu:268-274, render.h:384-405), headless
 *   pic_job_get_grid          Grid2D::debugGrid read-back (grid.cu:30)
 */
#ifndef PIC_B200_H
#define PIC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define PIC_OK                 0
#define PIC_ERR_ARG            1  /* invalid argument or configuration            */
#define PIC_ERR_OOM            2  /* device pool or cudaMalloc exhausted           */
#define PIC_ERR_CUDA           3  /* a CUDA runtime call failed                    */
#define PIC_ERR_NOT_CONVERGED  4  /* Poisson solve hit max_cycles above tol        */
#define PIC_ERR_TIMEOUT        5  /* a bounded device-side wait gave up            */
#define PIC_ERR_CAPACITY       6  /* particle / event / hit buffer would overflow  */
#define PIC_ERR_STATE          7  /* call not valid in the object's current state  */
#define PIC_ERR_NO_DEVICE      8  /* no CUDA device / extension not usable         */

#define PIC_MAX_SPECIES    4
#define PIC_MAX_WALLS      64
#define PIC_MAX_PROCESSES  8

/* Units of the field equation.
 *  PIC_UNITS_REF: the reference's formulation (Multigrid.cu:223,296):
 *      rho_node = sum_p q_s * w_CIC,  lap(phi) = rho_node,  v += q_s/m_s * E * dt.
 *  PIC_UNITS_SI:  rho_node = sum_p q_s * W_s * w_CIC (coulomb per node per metre of depth),
 *      lap(phi) = -rho_node / (eps0 * dx * dy),  v += q_s/m_s * E * dt  (SI). */
enum { PIC_UNITS_REF = 0, PIC_UNITS_SI = 1 };

/* Particle absorption.  BOX: a particle is absorbed when its new position leaves the
 * half-open grid rectangle [0, Lx) x [0, Ly) (the region updateDensity deposits from,
 * kernels.cu:53).  SEGMENTS: the segment old->new position is tested against each wall
 * segment (collisions.cu:7-54, without the absolute 1e-10 parallel cut-off).
 * BOX_AND_SEGMENTS: both. */
enum { PIC_WALLS_NONE = 0, PIC_WALLS_BOX = 1, PIC_WALLS_SEGMENTS = 2, PIC_WALLS_BOX_AND_SEGMENTS = 3 };

/* Charge deposition.  F32: FP32 accumulation (fast, order-dependent rounding).
 * I64: fixed-point int64 accumulation, bit-reproducible, conserves the deposited charge
 * exactly (every particle's four node weights sum to its quantised charge). */
enum { PIC_DEPOSIT_F32 = 0, PIC_DEPOSIT_I64 = 1 };

/* Monte Carlo collisions.  NULL_COLLISION: null-collision MCC (Vahedi & Surendra 1995)
 * over the configured processes.  REF_ELASTIC2D: the reference's elasticCollisions form
 * (mcc.cu:56-85): P = 1-exp(-n sigma(E)|v|dt), 2D isotropic redirect keeping |v|. */
enum { PIC_MCC_NONE = 0, PIC_MCC_NULL_COLLISION = 1, PIC_MCC_REF_ELASTIC2D = 2 };

enum {
  PIC_PROC_ELASTIC = 1,          /* electron-neutral elastic, isotropic, recoil loss 2m/M */
  PIC_PROC_EXCITATION = 2,       /* loses threshold energy, isotropic                     */
  PIC_PROC_IONIZATION = 3,       /* loses threshold, appends one electron and one ion     */
  PIC_PROC_CHARGE_EXCHANGE = 4   /* ion takes a neutral's Maxwellian velocity             */
};

/* Phase flags for pic_job_run_phases (one fused particle pass). */
enum {
  PIC_PHASE_KICK    = 1,   /* gather E from phi at the current position, v += q/m E dt  */
  PIC_PHASE_MCC     = 2,   /* collisions on the kicked velocity                          */
  PIC_PHASE_DRIFT   = 4,   /* x += v dt                                                  */
  PIC_PHASE_WALLS   = 8,   /* absorption test on the drifted segment; fills the hit list */
  PIC_PHASE_DEPOSIT = 16   /* CIC deposit at the (new) position into rho (accumulates)   */
};

enum { PIC_GRID_RHO = 0, PIC_GRID_PHI = 1, PIC_GRID_EX = 2, PIC_GRID_EY = 3 };
enum { PIC_MEM_HOST = 0, PIC_MEM_DEVICE = 1 };

typedef struct pic_species_config {
  double charge;      /* q per real particle (C in SI units; the reference's q[type] in REF) */
  double mass;        /* m per real particle (kg in SI; the reference's m[type] in REF)     */
  double weight;      /* real particles per macro-particle (use 1 in REF units)             */
  int64_t capacity;   /* maximum macro-particles held on the device for this species        */
} pic_species_config;

typedef struct pic_process_config {
  int type;                  /* PIC_PROC_*                                           */
  int species;               /* projectile species index                             */
  double threshold_ev;       /* excitation / ionisation threshold                     */
  int n_points;              /* table length (>= 2), energies strictly increasing     */
  const double* energy_ev;   /* host array, copied at job creation                     */
  const double* sigma_m2;    /* host array, copied at job creation                     */
} pic_process_config;

typedef struct pic_job_config {
  /* grid: node-centred, nx*ny nodes, row-major j*nx+i (grid.cu:10-20, kernels.cu:65) */
  int nx, ny;                /* 2^k+1 nodes each way (the multigrid coarsens by 2)     */
  double Lx, Ly;             /* domain extent; dx = Lx/(nx-1), dy = Ly/(ny-1), dx==dy    */
  double dt;
  int units;                 /* PIC_UNITS_*                                           */
  int n_species;
  pic_species_config species[PIC_MAX_SPECIES];
  /* Poisson multigrid: red-black SOR V-cycles (Multigrid.cu:539-569) run in FP32 inside
   * an FP64 defect-correction loop until ||f - A phi|| / ||f|| < tol (FP64).            */
  int mg_levels;             /* 0 = coarsen to 3x3                                     */
  int nu_pre, nu_post, nu_coarse;
  double omega;
  double tol;
  int max_cycles;
  /* walls */
  int wall_mode;             /* PIC_WALLS_*                                           */
  int n_walls;
  double walls[PIC_MAX_WALLS][4];   /* x1, y1, x2, y2 in domain units                 */
  /* deposition and particle ordering */
  int deposit_mode;          /* PIC_DEPOSIT_*                                         */
  int sort_every;            /* counting sort by cell every N steps (0 = never)         */
  /* Monte Carlo collisions */
  int mcc_mode;              /* PIC_MCC_*                                             */
  double gas_density;        /* m^-3                                                  */
  double gas_temperature;    /* K                                                     */
  double gas_mass;           /* kg                                                    */
  int n_processes;
  pic_process_config processes[PIC_MAX_PROCESSES];
  int ionization_electron_species;  /* species that receives ejected electrons          */
  int ionization_ion_species;       /* species that receives new ions                   */
  uint64_t seed;             /* Philox-4x32-10 key; streams are keyed (seed, pid, step) */
  /* warm start of each field solve: 0 = the previous step's phi (the reference keeps phi
   * between steps), 1 = linear extrapolation 2 phi_{k-1} - phi_{k-2} from the last two
   * solutions (one more FP64 grid; fewer V-cycles to the same tolerance) */
  int mg_warm_start;
} pic_job_config;

typedef struct pic_diagnostics {
  int64_t step;                          /* steps completed by this job                */
  int64_t count[PIC_MAX_SPECIES];        /* live macro-particles per species            */
  int64_t absorbed[PIC_MAX_SPECIES];     /* absorbed during the last step               */
  int64_t collisions[PIC_MAX_SPECIES][PIC_MAX_PROCESSES]; /* real collisions last step,
                                            [species][index of the process in pic_job_config] */
  int64_t ionizations;                   /* electron-ion pairs appended last step       */
  int32_t vcycles;                       /* V-cycles of the last field solve            */
  int32_t converged;                     /* last solve reached tol                      */
  double relres;                         /* last solve's FP64 relative residual         */
  double total_charge;                   /* sum of rho over nodes (FP64)                */
  /* sum 1/2 m W v^2 (FP64 sum; J in SI units) over the velocities the last particle pass
   * produced: after a step, those that drifted in it; after a read-back (which first applies
   * the pending kick and collisions), those it returned (pairs created by that read-back's
   * ionisations excepted).  Without MCC vz never changes and only vx, vy are counted. */
  double kinetic_energy[PIC_MAX_SPECIES];
  uint32_t status;                       /* sticky device status bits (PIC_ERR_* << k)  */
  uint32_t next_pid;                     /* id the next created particle receives        */
} pic_diagnostics;

typedef struct pic_engine_stats {
  int64_t kernel_launches;   /* kernels this engine launched since the last reset          */
  int64_t steps;             /* full steps taken since the last reset                      */
  int64_t vcycles;           /* V-cycle launches since the last reset                      */
  int64_t mover_launches;    /* fused particle passes timed (profiling on)                 */
  double mover_ms;           /* their summed CUDA-event time on the launching stream       */
  double phase_ms[4];        /* summed event time per phase: sort, particle pass,          */
                             /* compaction + ionisation, field solve (profiling on)        */
} pic_engine_stats;

typedef struct pic_engine pic_engine;

/* ---- engine and jobs ---- */
int pic_engine_create(int device, int64_t pool_bytes, pic_engine** out);
int pic_engine_destroy(pic_engine* e);
int pic_engine_bytes_needed(const pic_job_config* cfg, int64_t* bytes);  /* job footprint */
/* Maps `bytes` of device memory into the engine's job memory pool now (one allocation, freed
 * back to the pool at once), so that jobs created later take their arrays from memory that is
 * already mapped instead of growing the pool while they are admitted.  The pool keeps the
 * memory until the engine is destroyed.  The reservation does not count against pool_bytes
 * (only job memory does). */
int pic_engine_reserve(pic_engine* e, int64_t bytes);
int pic_job_create(pic_engine* e, const pic_job_config* cfg, int* job_id);
int pic_job_destroy(pic_engine* e, int job_id);
int pic_engine_num_jobs(pic_engine* e, int* n);

/* Load n particles of one species (replaces what was there).  Positions in domain
 * units (FP64), velocities (FP64); pid may be NULL (ids assigned from the job's counter).
 * memory = PIC_MEM_HOST (pageable or pinned) or PIC_MEM_DEVICE; device arrays may be
 * written by work still running on any stream: the call first waits for the device. */
int pic_job_load_species(pic_engine* e, int job, int species, int64_t n,
                         const double* x, const double* y,
                         const double* vx, const double* vy, const double* vz,
                         const uint32_t* pid, int memory);
int pic_job_export_species(pic_engine* e, int job, int species, int64_t capacity,
                           double* x, double* y, double* vx, double* vy, double* vz,
                           uint32_t* pid, int64_t* n_out, int memory);
/* Headless snapshot for a viewer: interleaved FP32 (x, y) of every particle of a species, 8 bytes
 * per particle, into a device buffer (memory = PIC_MEM_DEVICE, e.g. a mapped vertex buffer) or
 * host memory; what convertPositionsToFloat (kernels.cu:268-274) writes into the reference's
 * OpenGL vertex buffer.  Each value is the FP64 export's position rounded once to FP32. */
int pic_job_snapshot_positions(pic_engine* e, int job, int species, int64_t capacity, float* xy,
                               int64_t* n_out, int memory);
/* Same, in the engine's FP32 cell-relative layout (device pointers, no conversion). */
int pic_job_export_species_raw(pic_engine* e, int job, int species, int64_t capacity,
                               uint32_t* cell, float* fx, float* fy, float* vx, float* vy,
                               float* vz, uint32_t* pid, int64_t* n_out);

/* ---- stepping ---- */
/* Advance every job of the engine by nsteps full PIC steps on `stream`
 * (NULL = the engine's own stream).  No host synchronisation inside. */
int pic_step(pic_engine* e, int nsteps, void* stream);
/* Same, recorded once into a CUDA graph per engine configuration and replayed. */
int pic_step_graph(pic_engine* e, int nsteps, void* stream);
int pic_sync(pic_engine* e);
/* Record CUDA events around every fused particle pass (on the stream it runs on). */
int pic_engine_profile(pic_engine* e, int enable);
int pic_engine_get_stats(pic_engine* e, pic_engine_stats* out, int reset);
int pic_job_diagnostics(pic_engine* e, int job, pic_diagnostics* out);

/* ---- tuning (no counterpart in the reference: the knobs the autotuner sets) ---- */
/* PIC_OPT_MG_LEVELS_KERNEL: 1 = multigrid levels 1..lc as phases of one cooperative launch,
 *   0 = one launch per level (default).  Takes effect at the next field solve.
 * PIC_OPT_MG_CLUSTER_TOP: largest level side solved by a thread-block cluster (65 = none,
 *   default); applies to jobs created after the call.
 * PIC_OPT_MG_COARSE_TOP: largest level side (3..129) solved inside one CTA's shared memory
 *   (65 = default); applies to jobs created after the call.
 * PIC_OPT_MOVER_CTAS_PER_SM: CTAs per SM of the persistent particle pass (0 = as many as
 *   fit, the default; larger values are capped there).  Takes effect at the next step.
 * PIC_OPT_MG_WIDE_TILES: on multigrid tile levels with at most this many tiles per SM each
 *   tile runs on a 1024-thread CTA (a shorter latency chain when the level cannot fill the
 *   GPU), on the others on a 256-thread CTA (default 2; 0 = never).  Takes effect at the next
 *   field solve. */
enum { PIC_OPT_MG_LEVELS_KERNEL = 1, PIC_OPT_MG_CLUSTER_TOP = 2, PIC_OPT_MG_COARSE_TOP = 3,
       PIC_OPT_MOVER_CTAS_PER_SM = 4, PIC_OPT_MG_WIDE_TILES = 5 };
int pic_engine_set_option(pic_engine* e, int option, int64_t value);
int pic_engine_get_option(pic_engine* e, int option, int64_t* value);
/* Counting-sort cadence of one job (0 = never), from its next step on. */
int pic_job_set_sort_every(pic_engine* e, int job, int sort_every);

/* ---- individual phases (parity checks, the compatibility layer) ---- */
int pic_job_run_phases(pic_engine* e, int job, int phase_flags, int64_t step_index, void* stream);
int pic_job_compact(pic_engine* e, int job, void* stream);
int pic_job_zero_rho(pic_engine* e, int job, void* stream);
int pic_job_solve_field(pic_engine* e, int job, void* stream);
int pic_job_sort(pic_engine* e, int job, void* stream);
int pic_job_get_grid(pic_engine* e, int job, int which, double* out, int memory);
int pic_job_set_grid(pic_engine* e, int job, int which, const double* in, int memory);
/* Indices (into the exported order) of the particles the last WALLS phase absorbed. */
int pic_job_get_hits(pic_engine* e, int job, int species, int64_t capacity,
                     int64_t* idx, int64_t* n_out);

/* ---- stateless entry points on caller-owned FP64 device arrays ---- */
/* solve_multigrid (Multigrid.cu:573): lap(phi) = rho on an nx*ny grid, Dirichlet values
 * taken from phi's boundary, warm start from phi.  FP32 V-cycles (nu_pre/nu_post
 * red-black SOR sweeps with omega, nu_coarse on the coarsest level) inside FP64 defect
 * correction.  Scratch comes from a per-device cache keyed by (nx, ny, levels).  stream
 * NULL: the solve first waits for all work issued on the device (the caller's writes of
 * phi and rho), then runs on the solver's own stream; the call returns when it is done. */
int pic_solve_multigrid_f64(double* phi, const double* rho, int nx, int ny, int levels,
                            double h, double omega, int nu_pre, int nu_post, int nu_coarse,
                            double tol, int max_cycles, void* stream,
                            int* cycles_out, double* relres_out);
/* computeElectricField (kernels.cu:134): E = -grad(phi), central inside, one-sided on
 * edges; E is interleaved (Ex, Ey) per node like the reference's double2 array. */
int pic_efield_f64(const double* phi, double* E_xy, int nx, int ny, double dx, double dy,
                   void* stream);

/* Embedded-boundary multigrid, Multigrid_embedded.cu:1-190 (the reference's Multigrid class
 * and its vcycle, :110-188, driven to a tolerance).  Solves lap(phi) = rhs (FP64) on the FLUID
 * nodes of `mask` (nx*ny bytes, row-major like phi): PIC_NODE_DIRICHLET nodes are interior
 * electrodes held at phi_bc (phi_bc NULL: they keep the value phi holds), PIC_NODE_SOLID
 * nodes and the grid boundary keep theirs.  V-cycle of Multigrid::vcycle over `levels` levels
 * (nx_{l+1} = (nx_l - 1)/2 + 1): nu_pre red-black Gauss-Seidel sweeps ((i+j) even first;
 * the reference's colour test at :22 updates every node on its second colour, a precedence
 * slip, and this follows the intended test), residual, full weighting, coarse phi = 0,
 * recursion (the coarsest level runs the pre-sweeps only), prolongation, nu_post sweeps.
 * options 0 = the reference's transfer operators (coarse node kind injected from fine node
 * (2i, 2j), piecewise-constant prolongation from coarse (i/2, j/2)); they do not converge for
 * every geometry (an electrode edge on an odd node index makes the coarse electrode smaller
 * than the fine one).  PIC_EMB_COARSEN_ANY takes the coarse kind from the 3x3 fine nodes as
 * the reference's comment at :73 states; PIC_EMB_PROLONG_BILINEAR prolongates bilinearly.
 * Stops when ||r|| / ||rhs|| over the FLUID nodes (||r|| / ||r_0|| if rhs is 0 there) is below
 * tol or after max_cycles V-cycles (PIC_ERR_NOT_CONVERGED); reading the norm synchronises
 * `stream` once per cycle.  tol == 0 runs exactly max_cycles V-cycles without reading it in
 * between (once at the end with relres_out) and, like pic_solve_multigrid_f64, returns
 * PIC_ERR_NOT_CONVERGED.  Working arrays come from a
 * per-device cache keyed by (nx, ny, levels); calls on one device share it, so issue them on
 * one stream or one after another. */
enum { PIC_NODE_FLUID = 0, PIC_NODE_DIRICHLET = 1, PIC_NODE_SOLID = 2 };
enum { PIC_EMB_COARSEN_ANY = 1, PIC_EMB_PROLONG_BILINEAR = 2 };
int pic_solve_embedded_f64(double* phi, const double* rhs, const uint8_t* mask, const double* phi_bc,
                           int nx, int ny, int levels, double h, int nu_pre, int nu_post, int options,
                           double tol, int max_cycles, void* stream, int* cycles_out, double* relres_out);

/* No counterpart in the reference.  pic_solve_multigrid_f64 with the same arguments,
 * arithmetic and return codes, for callers that must not allocate device memory: all
 * working memory is a fixed array compiled into the library (704 KiB per device), so
 * grids are limited to PIC_STATIC_MG_MAX_SIDE nodes per side; larger grids return
 * PIC_ERR_ARG.  Callers that cannot allocate: code whose device memory is all reserved by
 * its own pool allocator (a cudaMalloc outside the pool may fail or fragment it), and
 * code in a time-critical loop that must not stall other streams (cudaMalloc/cudaFree may
 * synchronise the whole device; the other entry point's first call per shape also builds
 * an internal engine).
 * - Argument limits (both solvers): levels in [0, levels of a full hierarchy], nu_pre and
 *   nu_post in [0, 16], nu_coarse in [0, 1000], omega in (0, 2), max_cycles >= 1, tol >= 0;
 *   anything else returns PIC_ERR_ARG.
 * - The first call on each device looks up the array's address for that device
 *   (cudaGetSymbolAddress, with that device current); make that first call before any
 *   stream capture.  The address is kept for the life of the process: do not call this
 *   across a cudaDeviceReset (or a destroyed and re-created primary context) on that
 *   device, which would leave the kept address pointing at freed memory.
 * - Nothing needs to be zero beforehand: each call clears the correction on every level
 *   and recomputes every scratch value before reading it.
 * - The array is shared by all calls on a device: calls that overlap in time (on
 *   different streams, or from several threads without ordering) race on it and corrupt
 *   each other's result.  Issue them on one stream or otherwise one after another.
 * - The call waits for its stream to finish (it reads the cycle count and residual back). */
#define PIC_STATIC_MG_MAX_SIDE 257
int pic_solve_multigrid_f64_static(double* phi, const double* rho, int nx, int ny, int levels,
                                   double h, double omega, int nu_pre, int nu_post, int nu_coarse,
                                   double tol, int max_cycles, void* stream,
                                   int* cycles_out, double* relres_out);

/* ---- misc ---- */
const char* pic_last_error(void);
int pic_version(void);
/* sizeof(pic_job_config), sizeof(pic_diagnostics), sizeof(pic_species_config),
 * sizeof(pic_process_config): lets foreign-language bindings check their struct layout. */
int pic_abi_sizes(int64_t out[4]);
/* Philox-4x32-10 (Salmon et al., SC'11) as used by the MCC streams. */
void pic_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

#ifdef __cplusplus
}
#endif
#endif /* PIC_B200_H */
