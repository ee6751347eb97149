// engine.cu — host runtime behind the C ABI (include/pic_b200.h).
//
// An engine owns device tables for up to kMaxJobs jobs (slot = 4*job + species) and steps
// every live job with the same kernel launches; a plain simulation is an engine with one
// job.  One step (the sequence of updateSimulationCUDA, main.cu:60-135) is:
//   [counting sort every N steps] -> zero rho -> mover (kick+MCC of the previous step,
//   drift, walls, deposit) -> compaction -> ionisation appends -> multigrid solve
//   (FP64 defect correction over FP32 V-cycles) -> step bookkeeping.
// The only host synchronisation inside a step is the convergence read-back of the field
// solve (one 4-byte copy per V-cycle); pic_step_graph removes it with a CUDA graph whose
// V-cycle loop is a conditional WHILE node.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pic_b200.h"
#include "common.cuh"
#include "kernels.h"
#include "mg_tiles.h"

namespace {

thread_local std::string g_err;
int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
}  // namespace

// Records a failure for pic_last_error() from the other translation units of the library.
int pic_fail(int code, const char* msg) { return fail(code, msg); }

namespace {
#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return fail(PIC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr int kMaxJobs = 4096;
constexpr int kSlotsPerJob = 4;
constexpr double kEps0 = 8.8541878128e-12;
constexpr double kQe = 1.602176634e-19;
constexpr double kKb = 1.380649e-23;

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

struct MgBuild {
  TileRef* d_tiles = nullptr;
  int* d_coarse = nullptr;
  MgLaunch L{};
  int max_cycles = 1;
  bool valid = false;
  void release() {
    if (d_tiles) cudaFree(d_tiles);
    if (d_coarse) cudaFree(d_coarse);
    d_tiles = nullptr; d_coarse = nullptr; valid = false;
  }
};

struct JobHost {
  bool alive = false;
  pic_job_config cfg{};
  JobDev dev{};
  SlotDev slot[kSlotsPerJob]{};
  std::vector<void*> allocs;
  int64_t bytes = 0;
  int64_t steps = 0;
  bool pending = false;
  // JobState::total_charge holds the sum of the present rho: the level-0 residual kernel
  // of every field solve computes it; entry points that change rho otherwise clear this
  bool charge_fresh = false;
  MgBuild mg;
};

int auto_levels(int n) {
  int L = 1;
  while (n > 3 && (n & 1)) { n = (n + 1) / 2; ++L; }
  return L;
}
bool is_pow2p1(int n) { return n >= 3 && ((n - 1) & (n - 2)) == 0; }

// nu_max (Vahedi & Surendra 1995): n_g * max over table intervals of sigma_T * v, with
// sigma_T taken at the larger end point and v at the upper energy (an upper bound of the
// piecewise-linear sigma_T(E) * v(E)).
double table_eval(const pic_process_config& p, double E) {
  const int n = p.n_points;
  if (E <= p.energy_ev[0]) return p.sigma_m2[0];
  if (E >= p.energy_ev[n - 1]) return p.sigma_m2[n - 1];
  int k = (int)(std::upper_bound(p.energy_ev, p.energy_ev + n, E) - p.energy_ev) - 1;
  k = std::max(0, std::min(k, n - 2));
  const double t = (E - p.energy_ev[k]) / (p.energy_ev[k + 1] - p.energy_ev[k]);
  return p.sigma_m2[k] + t * (p.sigma_m2[k + 1] - p.sigma_m2[k]);
}
double compute_numax(const pic_job_config& c, int species) {
  std::vector<double> grid;
  for (int i = 0; i < c.n_processes; ++i)
    if (c.processes[i].species == species)
      grid.insert(grid.end(), c.processes[i].energy_ev, c.processes[i].energy_ev + c.processes[i].n_points);
  if (grid.empty()) return 0.0;
  std::sort(grid.begin(), grid.end());
  const double m = c.species[species].mass;
  double best = 0.0;
  for (size_t g = 0; g < grid.size(); ++g) {
    const double elo = grid[g > 0 ? g - 1 : 0], ehi = grid[g];
    double st = 0.0;
    for (int i = 0; i < c.n_processes; ++i)
      if (c.processes[i].species == species)
        st += std::max(table_eval(c.processes[i], elo), table_eval(c.processes[i], ehi));
    best = std::max(best, st * std::sqrt(2.0 * ehi * kQe / m));
  }
  return c.gas_density * best;
}

int validate(const pic_job_config* c, std::string& why) {
  if (!c) { why = "null config"; return PIC_ERR_ARG; }
  if (!is_pow2p1(c->nx) || c->nx != c->ny) { why = "grid must be square with 2^k+1 nodes per side"; return PIC_ERR_ARG; }
  if (c->nx > 16385) { why = "grid too large (cell index packs 16 bits per axis)"; return PIC_ERR_ARG; }
  if (!(c->Lx > 0) || !(c->Ly > 0)) { why = "domain extents must be positive"; return PIC_ERR_ARG; }
  const double dx = c->Lx / (c->nx - 1), dy = c->Ly / (c->ny - 1);
  if (std::fabs(dx - dy) > 1e-12 * dx) { why = "cells must be square (dx == dy)"; return PIC_ERR_ARG; }
  if (!(c->dt > 0)) { why = "dt must be positive"; return PIC_ERR_ARG; }
  if (c->n_species < 0 || c->n_species > PIC_MAX_SPECIES) { why = "n_species out of range"; return PIC_ERR_ARG; }
  for (int s = 0; s < c->n_species; ++s) {
    if (!(c->species[s].mass > 0) || c->species[s].capacity < 0 || c->species[s].capacity > (1ll << 31) - 4096) {
      why = "species mass must be > 0 and capacity in [0, 2^31)"; return PIC_ERR_ARG;
    }
  }
  const int maxL = auto_levels(c->nx);
  if (c->mg_levels < 0 || c->mg_levels > maxL || maxL > PIC_MAX_LEVELS) { why = "mg_levels out of range"; return PIC_ERR_ARG; }
  if (c->nu_pre < 0 || c->nu_pre > 16 || c->nu_post < 0 || c->nu_post > 16 || c->nu_coarse < 0 || c->nu_coarse > 1000) {
    why = "sweep counts out of range"; return PIC_ERR_ARG;
  }
  if (!(c->omega > 0 && c->omega < 2)) { why = "omega must be in (0, 2)"; return PIC_ERR_ARG; }
  if (c->max_cycles < 1 || !(c->tol >= 0)) { why = "max_cycles >= 1 and tol >= 0 required"; return PIC_ERR_ARG; }
  if (c->mg_warm_start != 0 && c->mg_warm_start != 1) { why = "mg_warm_start must be 0 or 1"; return PIC_ERR_ARG; }
  if (c->n_walls < 0 || c->n_walls > PIC_MAX_WALLS) { why = "too many walls"; return PIC_ERR_ARG; }
  if (c->deposit_mode != PIC_DEPOSIT_F32 && c->deposit_mode != PIC_DEPOSIT_I64) { why = "bad deposit_mode"; return PIC_ERR_ARG; }
  if (c->mcc_mode < 0 || c->mcc_mode > 2) { why = "bad mcc_mode"; return PIC_ERR_ARG; }
  if (c->mcc_mode) {
    if (c->n_processes < 1 || c->n_processes > PIC_MAX_PROCESSES) { why = "n_processes out of range"; return PIC_ERR_ARG; }
    for (int i = 0; i < c->n_processes; ++i) {
      const pic_process_config& p = c->processes[i];
      if (p.species < 0 || p.species >= c->n_species || p.n_points < 2 || !p.energy_ev || !p.sigma_m2) {
        why = "bad process table"; return PIC_ERR_ARG;
      }
      for (int k = 1; k < p.n_points; ++k)
        if (!(p.energy_ev[k] > p.energy_ev[k - 1])) { why = "process energies must increase"; return PIC_ERR_ARG; }
      if (p.type < 1 || p.type > 4) { why = "bad process type"; return PIC_ERR_ARG; }
      if (p.type == PIC_PROC_IONIZATION &&
          (c->ionization_electron_species < 0 || c->ionization_electron_species >= c->n_species ||
           c->ionization_ion_species < 0 || c->ionization_ion_species >= c->n_species)) {
        why = "ionisation product species out of range"; return PIC_ERR_ARG;
      }
    }
    if (c->mcc_mode == PIC_MCC_NULL_COLLISION && (!(c->gas_density >= 0) || !(c->gas_mass > 0))) {
      why = "gas density >= 0 and gas mass > 0 required"; return PIC_ERR_ARG;
    }
  }
  return PIC_OK;
}

bool has_ionization(const pic_job_config& c) {
  if (c.mcc_mode != PIC_MCC_NULL_COLLISION) return false;
  for (int i = 0; i < c.n_processes; ++i)
    if (c.processes[i].type == PIC_PROC_IONIZATION) return true;
  return false;
}
int event_capacity(const pic_job_config& c) {
  if (!has_ionization(c)) return 0;
  const int64_t ce = c.species[c.ionization_electron_species].capacity;
  return (int)std::max<int64_t>(16384, std::min<int64_t>(ce / 128, 1 << 24));
}

struct Layout {  // byte sizes of one job's device state
  int levels, lc;
  int nl[PIC_MAX_LEVELS];
  int ntiles0;
  int64_t total;
};
// First level handled by the coarse solver (levels above it run as tile kernels): grids up
// to coarse_top (<= PIC_COARSE_MAX) entirely in one CTA (lc = 0, the FP64 update then runs
// as its own tile launch); otherwise the first level that fits one CTA, or a C-CTA cluster
// when cluster_top asks for one above coarse_top.
Layout job_layout(const pic_job_config& c, int cluster_C = 0, int cluster_top = 0, int coarse_top = PIC_COARSE_MAX) {
  Layout L{};
  L.levels = c.mg_levels > 0 ? c.mg_levels : auto_levels(c.nx);
  const int one_cta = std::min(std::max(coarse_top, 3), PIC_COARSE_MAX);
  int cluster_max = cluster_C >= 16 ? 513 : cluster_C >= 8 ? 257 : 0;
  cluster_max = std::min(cluster_max, cluster_top);
  const int top = std::max(one_cta, cluster_max);
  int n = c.nx;
  L.lc = -1;
  for (int l = 0; l < L.levels; ++l) {
    L.nl[l] = n;
    if (L.lc < 0) {
      if (l == 0 && n <= one_cta) L.lc = 0;
      else if (l > 0 && n <= top) L.lc = l;
    }
    n = (n + 1) / 2;
  }
  if (L.lc < 0) L.lc = L.levels - 1;
  L.ntiles0 = ((c.nx + 31) / 32) * ((c.ny + 31) / 32);
  const int64_t N = (int64_t)c.nx * c.ny;
  int64_t b = N * ((c.deposit_mode == PIC_DEPOSIT_I64 ? 8 : 4) + 8 + 16 + (c.mg_warm_start ? 8 : 0));
  // level arrays at a row pitch rounded up to 4 floats; the tile tensor maps
  for (int l = 0; l < L.levels; ++l) b += 8ll * mgt::round4(L.nl[l]) * L.nl[l];
  for (int l = 1; l < L.levels; ++l) b += 4ll * mgt::round4(L.nl[l]) * L.nl[l];   // up-leg corrections
  b += 4ll * mgt::round4(c.nx) * c.ny;                                           // second level-0 rhs
  b += (int64_t)sizeof(CUtensorMap) * mgt::kTmapsPerLevel * L.levels;
  b += 24ll * L.ntiles0;
  const int64_t ncells = (int64_t)(c.nx - 1) * (c.ny - 1) + 1;
  for (int s = 0; s < c.n_species; ++s) {
    const int64_t cap = round_up(std::max<int64_t>(c.species[s].capacity, 1), PIC_CHUNK);
    b += cap * 4 * 17 + ncells * 4 + ((ncells + 2047) / 2048 + 1) * 4;
  }
  const int ev = event_capacity(c);
  if (ev) {
    int p2 = 1;
    while (p2 < ev) p2 <<= 1;
    b += (int64_t)ev * sizeof(Event) + (int64_t)p2 * 8;
  }
  L.total = b;
  return L;
}

}  // namespace

struct pic_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  // Job memory comes from a stream-ordered pool that keeps what jobs free for the next ones
  // (admitting and retiring jobs while others run should not cost a device-wide cudaFree).
  cudaMemPool_t pool = nullptr;
  int num_sms = 148;
  int mover_bps = 4;        // mover CTAs per SM: the occupancy limit
  int mover_cps = 0;        // PIC_OPT_MOVER_CTAS_PER_SM (0: mover_bps)
  int wide_factor = 2;      // PIC_OPT_MG_WIDE_TILES
  int cluster_C = 0;          // thread-block cluster size of the coarse solver (0: none)
  // Largest level side given to the cluster coarse solver.  Measured on B200 (1025^2 job):
  // tile kernels over all SMs for every level above 65^2 and one CTA below beat the
  // 16-CTA cluster from 513^2 down (V-cycle 0.20 -> 0.18 ms), so by default the cluster is
  // not used; PIC_MG_CLUSTER_TOP=<side> selects it for levels up to that side.
  int cluster_top = 65;
  // Largest level side solved by the one-CTA coarse solver (jobs created after a change).
  // Measured on B200 (1025^2 job, ncu): levels 129^2 .. 3^2 in one CTA take 49 us per
  // V-cycle, bound by that one SM's shared-memory bandwidth (7 accesses per node and
  // half-sweep), against about 16 us for 129^2 as two tile launches plus 65^2 .. 3^2 in one CTA.
  int coarse_top = 65;
  // Programmatic dependent launches between the V-cycle's kernels (PIC_PDL=0 turns them off;
  // they are also dropped if a step graph with them cannot be built).
  bool pdl = true;
  int last_solve_cycles = 1;  // V-cycles the last stream-ordered solve ran (speculation depth)
  int levels_kernel = 0;      // multigrid levels 1..lc as one cooperative launch
  size_t cluster_smem_max = 0;
  int64_t pool_bytes = 0, used_bytes = 0;
  std::vector<JobHost> jobs;
  int njobs_hw = 0;
  JobDev* d_jobs = nullptr;
  JobState* d_st = nullptr;
  SlotDev* d_slots = nullptr;
  int *d_counts = nullptr, *d_hits = nullptr, *d_aux = nullptr, *d_chunk = nullptr, *d_running = nullptr;
  uint8_t *d_active = nullptr, *d_mask = nullptr;
  int* h_pinned = nullptr;
  double* d_diag = nullptr;  // per-CTA partial sums of the diagnostics reductions
  MgBuild mg_all;
  bool mg_dirty = true;
  void* d_stage = nullptr;
  size_t stage_bytes = 0;
  std::vector<uint8_t> h_active;
  int max_nu_pre = 0, max_nu_post = 0;
  // CUDA graphs of one step (pic_step_graph): without and with the counting sort
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraphExec_t graph_exec_sort = nullptr;
  bool graph_dirty = true;
  cudaStream_t cap_stream = nullptr, body_stream = nullptr;
  // The counting sort due before a job's next step runs on side_stream, concurrently with the
  // field solve of this step (the solve touches only grids, the sort only particle arrays).
  cudaStream_t side_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int* d_loop = nullptr;                    // [0] iterations of the current solve
  unsigned long long* d_loop_total = nullptr;  // V-cycle iterations run by graph launches
  int64_t graph_fixed_launches[2] = {0, 0};
  int64_t graph_body_launches = 0;
  int64_t graph_steps = 0;
  std::mutex mu;
  // statistics and optional timing of the particle pass
  int64_t launches = 0, steps_taken = 0, vcycles = 0;
  bool profile = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> mover_events;
  size_t mover_events_used = 0;
  // per-phase timing (profile mode): sort, mover, compaction+ionisation, field solve
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> phase_events[4];
  size_t phase_used[4] = {0, 0, 0, 0};
};

namespace {

EngineLaunch make_launch(pic_engine* E, const uint8_t* active) {
  EngineLaunch L{};
  L.jobs = E->d_jobs;
  L.st = E->d_st;
  L.slots = E->d_slots;
  L.slots_mut = E->d_slots;
  L.counts = E->d_counts;
  L.hit_counts = E->d_hits;
  L.aux = E->d_aux;
  L.chunk_prefix = E->d_chunk;
  L.active = active ? active : E->d_active;
  L.nslots = E->njobs_hw * kSlotsPerJob;
  L.njobs = E->njobs_hw;
  L.num_sms = E->num_sms;
  L.mover_grid = E->num_sms * (E->mover_cps > 0 ? std::min(E->mover_cps, E->mover_bps) : E->mover_bps);
  L.running = E->d_running;
  L.gbar = reinterpret_cast<unsigned*>(E->d_running + 2);  // the grid barrier's arrival counter
  L.absorbed = E->d_aux + 4 * kMaxJobs * kSlotsPerJob;
  return L;
}

// cuTensorMapEncodeTiled, reached through the runtime's driver entry point (the library
// links only the CUDA runtime).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

// A 2-D FP32 tensor map of an n x n level array with row pitch `pitch` floats, box bw x bh;
// elements outside the n x n nodes (the pitch padding included) read as zero.
int encode_level_map(CUtensorMap* m, const float* base, int n, int pitch, int bw, int bh) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return fail(PIC_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  const cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)n};
  const cuuint64_t strides[1] = {(cuuint64_t)pitch * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
  const cuuint32_t es[2] = {1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(PIC_ERR_CUDA, "cuTensorMapEncodeTiled rejected a multigrid tile map");
  return PIC_OK;
}

// The tile tensor maps of every level the tile kernels process (levels above the coarse
// solver's; mg_tiles.h lists them), copied to `dst` on the device.  Sweep counts above the
// compile-time shapes run on the generic kernels, which read global memory directly.
int make_tile_maps(const JobDev& D, int nu_pre, int nu_post, CUtensorMap* dst) {
  std::vector<CUtensorMap> maps((size_t)mgt::kTmapsPerLevel * D.levels);
  std::memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
  int rc = PIC_OK;
  for (int l = 0; l < D.lc && !rc; ++l) {
    CUtensorMap* m = maps.data() + (size_t)mgt::kTmapsPerLevel * l;
    const int n = D.nl[l], p = D.pl[l];
    if (nu_pre <= 4) {
      const int bw = mgt::down_bw(nu_pre), bh = mgt::down_w(nu_pre);
      rc = encode_level_map(m + mgt::kMapDownF, D.f[l], n, p, bw, bh);
      if (!rc && l == 0) rc = encode_level_map(m + mgt::kMapDownF0b, D.f0b, n, p, bw, bh);
    }
    if (!rc && nu_post <= 4) {
      const int x = l == 0 ? 1 : 0;
      const int bw = mgt::up_bw(nu_post, x), bh = mgt::up_w(nu_post, x);
      rc = encode_level_map(m + mgt::kMapUpE, D.e[l], n, p, bw, bh);
      if (!rc) rc = encode_level_map(m + mgt::kMapUpF, D.f[l], n, p, bw, bh);
      if (!rc && l == 0) rc = encode_level_map(m + mgt::kMapUpF0b, D.f0b, n, p, bw, bh);
      if (!rc) {
        const float* ec = l + 1 == D.lc ? D.e[l + 1] : D.eu[l + 1];
        rc = encode_level_map(m + mgt::kMapUpC, ec, D.nl[l + 1], D.pl[l + 1], mgt::up_cbw(nu_post, x),
                              mgt::up_cw(nu_post, x));
      }
    }
  }
  if (rc) return rc;
  CK(cudaMemcpy(dst, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
  return PIC_OK;
}

int dev_alloc(pic_engine* E, JobHost& J, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (E->pool_bytes > 0 && E->used_bytes + (int64_t)bytes > E->pool_bytes)
    return fail(PIC_ERR_OOM, "engine memory budget exceeded");
  // stream-ordered on E->stream: the caller synchronises that stream once before the first
  // synchronous copy or memset touches the new blocks (then they are usable from any stream)
  cudaError_t e = cudaMallocFromPoolAsync(p, bytes, E->pool, E->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(PIC_ERR_OOM, std::string("cudaMallocFromPoolAsync: ") + cudaGetErrorString(e));
  }
  J.allocs.push_back(*p);
  J.bytes += (int64_t)bytes;
  E->used_bytes += (int64_t)bytes;
  return PIC_OK;
}

// Every stream may still use the job's memory: one device-wide wait, then the blocks go back
// to the pool in stream order.
void free_job(pic_engine* E, JobHost& J) {
  cudaDeviceSynchronize();
  for (void* p : J.allocs) cudaFreeAsync(p, E->stream);
  cudaStreamSynchronize(E->stream);
  J.allocs.clear();
  E->used_bytes -= J.bytes;
  J.bytes = 0;
  J.mg.release();
  J.alive = false;
}

// Tile lists for the multigrid kernels over the given jobs.
int build_mg(pic_engine* E, const std::vector<int>& ids, MgBuild& out) {
  out.release();
  std::vector<TileRef> init, upd, down[PIC_MAX_LEVELS], up[PIC_MAX_LEVELS];
  std::vector<int> coarse, cluster, finish;
  size_t cluster_smem = 0;
  int max_depth = 0, max_cycles = 1, nu_pre_max = 1, nu_post_max = 1;
  int nu_pre_min = 1 << 30, nu_post_min = 1 << 30;
  size_t coarse_smem = 0;
  for (int id : ids) {
    const JobHost& J = E->jobs[id];
    const JobDev& D = J.dev;
    max_depth = std::max(max_depth, D.lc);
    max_cycles = std::max(max_cycles, D.max_cycles);
    nu_pre_max = std::max(nu_pre_max, D.nu_pre);
    nu_post_max = std::max(nu_post_max, D.nu_post);
    nu_pre_min = std::min(nu_pre_min, D.nu_pre);
    nu_post_min = std::min(nu_post_min, D.nu_post);
    const int t0 = (D.nx + 31) / 32;
    for (int tj = 0; tj < t0; ++tj)
      for (int ti = 0; ti < t0; ++ti) init.push_back({id, ti, tj, tj * t0 + ti, t0 * t0, 0});
    if (D.lc == 0)
      for (int tj = 0; tj < t0; ++tj)
        for (int ti = 0; ti < t0; ++ti) upd.push_back({id, ti, tj, tj * t0 + ti, t0 * t0, 0});
    if (D.lc >= 1) finish.push_back(id);
    for (int l = 0; l < D.lc; ++l) {
      const int tc = (D.nl[l + 1] + 15) / 16;
      for (int tj = 0; tj < tc; ++tj)
        for (int ti = 0; ti < tc; ++ti) down[l].push_back({id, ti, tj, 0, 1, 0});
      const int tu = (D.nl[l] + 31) / 32;
      for (int tj = 0; tj < tu; ++tj)
        for (int ti = 0; ti < tu; ++ti) up[l].push_back({id, ti, tj, tj * tu + ti, tu * tu, 0});
    }
    if (E->cluster_C > 0 && D.nl[D.lc] > PIC_COARSE_MAX) {   // above one CTA's shared memory
      cluster.push_back(id);
      cluster_smem = std::max(cluster_smem, mg_cluster_smem(D.nl, D.lc, D.levels, E->cluster_C));
    } else {
      coarse.push_back(id);
      coarse_smem = std::max(coarse_smem, mg_coarse_smem(D.nl, D.lc, D.levels));
    }
  }
  std::vector<TileRef> all;
  size_t off_init = all.size(); all.insert(all.end(), init.begin(), init.end());
  size_t off_upd = all.size(); all.insert(all.end(), upd.begin(), upd.end());
  size_t off_down[PIC_MAX_LEVELS], off_up[PIC_MAX_LEVELS];
  for (int l = 0; l < PIC_MAX_LEVELS; ++l) { off_down[l] = all.size(); all.insert(all.end(), down[l].begin(), down[l].end()); }
  for (int l = 0; l < PIC_MAX_LEVELS; ++l) { off_up[l] = all.size(); all.insert(all.end(), up[l].begin(), up[l].end()); }
  if (!all.empty()) {
    CK(cudaMalloc(&out.d_tiles, all.size() * sizeof(TileRef)));
    CK(cudaMemcpy(out.d_tiles, all.data(), all.size() * sizeof(TileRef), cudaMemcpyHostToDevice));
  }
  std::vector<int> lists(coarse);
  lists.insert(lists.end(), cluster.begin(), cluster.end());
  lists.insert(lists.end(), finish.begin(), finish.end());
  lists.insert(lists.end(), ids.begin(), ids.end());
  if (!lists.empty()) {
    CK(cudaMalloc(&out.d_coarse, lists.size() * sizeof(int)));
    CK(cudaMemcpy(out.d_coarse, lists.data(), lists.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  MgLaunch& M = out.L;
  M = MgLaunch{};
  M.init_tiles = out.d_tiles + off_init; M.n_init = (int)init.size();
  M.upd_tiles = out.d_tiles + off_upd; M.n_upd = (int)upd.size();
  for (int l = 0; l < PIC_MAX_LEVELS; ++l) {
    M.down_tiles[l] = out.d_tiles + off_down[l]; M.n_down[l] = (int)down[l].size();
    M.up_tiles[l] = out.d_tiles + off_up[l]; M.n_up[l] = (int)up[l].size();
  }
  M.coarse_jobs = out.d_coarse; M.n_coarse = (int)coarse.size();
  M.cluster_jobs = out.d_coarse + coarse.size(); M.n_cluster = (int)cluster.size();
  M.finish_jobs = out.d_coarse + coarse.size() + cluster.size(); M.n_finish = (int)finish.size();
  M.init_jobs = M.finish_jobs + finish.size(); M.n_init_jobs = (int)ids.size();
  M.cluster_C = E->cluster_C;
  M.cluster_smem = cluster_smem;
  M.max_depth = max_depth;
  M.coarse_smem = coarse_smem;
  M.nu_pre_max = nu_pre_max;
  M.nu_post_max = nu_post_max;
  M.pdl = E->pdl ? 1 : 0;
  M.wide_factor = E->wide_factor;
  M.fast_nu_pre = (!ids.empty() && nu_pre_min == nu_pre_max) ? nu_pre_max : -1;
  M.fast_nu_post = (!ids.empty() && nu_post_min == nu_post_max) ? nu_post_max : -1;
  // Levels 1..lc as phases of one cooperative launch (PIC_OPT_MG_LEVELS_KERNEL).  Measured on
  // B200 (1025^2 job, CUDA-graph step): 1.600 ms per step against 1.555 ms with one launch per
  // level, because at these sizes each phase waits on its slowest tile either way and the grid
  // barriers add to that; so it is off by default.
  if (cluster.empty() && max_depth >= 2 && E->levels_kernel)
    M.levels_grid = mg_levels_configure(E->num_sms, nu_pre_max, nu_post_max, coarse_smem, &M.levels_smem,
                                        &M.levels_quarter_floats);
  out.max_cycles = max_cycles;
  out.valid = true;
  if (coarse_smem > 227 * 1024 || cluster_smem > 227 * 1024)
    return fail(PIC_ERR_ARG, "coarse multigrid levels exceed shared memory");
  if (!cluster.empty() && mg_cluster_supported(E->cluster_C, cluster_smem) <= 0)
    return fail(PIC_ERR_CUDA, "thread-block cluster of the coarse solver cannot be scheduled");
  mg_configure_coarse(std::max<size_t>(coarse_smem, 48 * 1024));
  return PIC_OK;
}

std::vector<int> alive_ids(pic_engine* E) {
  std::vector<int> v;
  for (int j = 0; j < E->njobs_hw; ++j)
    if (E->jobs[j].alive) v.push_back(j);
  return v;
}

int ensure_mg_all(pic_engine* E) {
  if (!E->mg_dirty && E->mg_all.valid) return PIC_OK;
  const int rc = build_mg(E, alive_ids(E), E->mg_all);
  if (rc) return rc;
  E->mg_dirty = false;
  return PIC_OK;
}

// Field solve: init residual, then V-cycles until every job stopped.  The first cycles go
// out without a host check (one fewer than the last solve needed: a converged job's kernels
// return at once, so a spare cycle costs launches only); after them the host reads the
// running-job count back after every cycle.
int solve(pic_engine* E, const MgBuild& B, const uint8_t* active, cudaStream_t s) {
  if (!B.valid) return PIC_OK;
  EngineLaunch L = make_launch(E, active);
  E->launches += launch_mg_init(L, B.L, s);
  const int unchecked = std::max(1, std::min(E->last_solve_cycles - 1, B.max_cycles));
  int c = 0;
  for (; c < B.max_cycles; ++c) {
    E->launches += launch_mg_vcycle(L, B.L, s);
    E->vcycles++;
    if (c + 1 < unchecked) continue;
    CK(cudaMemcpyAsync(E->h_pinned, E->d_running, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (*E->h_pinned <= 0) break;
  }
  E->last_solve_cycles = std::min(c + 1, B.max_cycles);
  CK(cudaGetLastError());
  return PIC_OK;
}

int upload_active(pic_engine* E) {
  CK(cudaMemcpy(E->d_active, E->h_active.data(), E->h_active.size(), cudaMemcpyHostToDevice));
  return PIC_OK;
}

int job_mask(pic_engine* E, int job, cudaStream_t s) {
  std::vector<uint8_t> m(E->njobs_hw * kSlotsPerJob, 0);
  for (int k = 0; k < kSlotsPerJob; ++k) m[job * kSlotsPerJob + k] = E->h_active[job * kSlotsPerJob + k];
  CK(cudaMemcpyAsync(E->d_mask, m.data(), m.size(), cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  return PIC_OK;
}

cudaStream_t pick(pic_engine* E, void* s) { return s ? (cudaStream_t)s : E->stream; }

// Begin/end of a timed phase (profile mode only).
int phase_mark(pic_engine* E, int ph, bool begin, cudaStream_t s) {
  if (!E->profile) return PIC_OK;
  auto& v = E->phase_events[ph];
  if (begin) {
    if (E->phase_used[ph] == v.size()) {
      std::pair<cudaEvent_t, cudaEvent_t> ev;
      CK(cudaEventCreate(&ev.first));
      CK(cudaEventCreate(&ev.second));
      v.push_back(ev);
    }
    CK(cudaEventRecord(v[E->phase_used[ph]].first, s));
  } else {
    CK(cudaEventRecord(v[E->phase_used[ph]].second, s));
    E->phase_used[ph]++;
  }
  return PIC_OK;
}

// Applies the deferred kick and collisions of the given job (of every job with job < 0) now,
// before its particles are read back or replaced; the other jobs keep theirs for their next step.
int flush(pic_engine* E, cudaStream_t s, int job = -1) {
  bool any = false;
  for (int j = 0; j < E->njobs_hw; ++j) any |= (job < 0 || j == job) && E->jobs[j].alive && E->jobs[j].pending;
  if (!any) return PIC_OK;
  const uint8_t* active = nullptr;
  JobState* st = E->d_st;
  int nst = E->njobs_hw;
  if (job >= 0) {
    const int rc = job_mask(E, job, s);
    if (rc) return rc;
    active = E->d_mask;
    st = E->d_st + job;
    nst = 1;
  }
  EngineLaunch L = make_launch(E, active);
  E->launches += launch_ke_reset_pending(st, nst, s);
  E->launches += launch_mover(L, PIC_PHASE_KICK_I | PIC_PHASE_MCC_I | PIC_PHASE_GATED_I, 0, s);
  E->launches += launch_ionize(L, false, s);
  E->launches += launch_step_end(st, nst, nullptr, 0, 0, s);
  for (int j = 0; j < E->njobs_hw; ++j)
    if (job < 0 || j == job) E->jobs[j].pending = false;
  CK(cudaGetLastError());
  return PIC_OK;
}

int ensure_stage(pic_engine* E, size_t bytes) {
  if (E->stage_bytes >= bytes) return PIC_OK;
  if (E->d_stage) cudaFree(E->d_stage);
  E->d_stage = nullptr;
  E->stage_bytes = 0;
  CK(cudaMalloc(&E->d_stage, bytes));
  E->stage_bytes = bytes;
  return PIC_OK;
}

int check_job(pic_engine* E, int job) {
  if (!E) return fail(PIC_ERR_ARG, "null engine");
  if (job < 0 || job >= E->njobs_hw || !E->jobs[job].alive) return fail(PIC_ERR_ARG, "no such job");
  return PIC_OK;
}

// One full step of every live job.
// Counting sort (stream-ordered on s) of the jobs for which `due` holds.
template <typename Due>
int sort_jobs(pic_engine* E, const EngineLaunch& L, Due due, cudaStream_t s, bool* launched) {
  std::vector<uint8_t> mask(L.nslots, 0);
  bool any = false;
  int max_cells = 0;
  int64_t max_p = 0;
  for (int j = 0; j < E->njobs_hw; ++j) {
    JobHost& J = E->jobs[j];
    if (!J.alive || J.cfg.sort_every <= 0 || !due(J)) continue;
    for (int k = 0; k < J.cfg.n_species; ++k) {
      mask[j * kSlotsPerJob + k] = 1;
      max_p = std::max<int64_t>(max_p, J.cfg.species[k].capacity);
    }
    max_cells = std::max(max_cells, J.dev.ncx * J.dev.ncy);
    any = true;
  }
  *launched = any;
  if (!any) return PIC_OK;
  CK(cudaMemcpyAsync(E->d_mask, mask.data(), mask.size(), cudaMemcpyHostToDevice, s));
  phase_mark(E, 0, true, s);
  E->launches += launch_sort(L, E->d_mask, max_cells, (int)std::min<int64_t>(max_p, 1 << 30), true, s);
  phase_mark(E, 0, false, s);
  return PIC_OK;
}
// A job's first step sorts its (freshly loaded) particles before the particle pass; later
// sorts run at the end of the step before the one that is due (step + 1 a multiple of
// sort_every), concurrently with that step's field solve.
bool sort_before_first(const JobHost& J) { return J.steps == 0; }
bool sort_after(const JobHost& J) { return (J.steps + 1) % J.cfg.sort_every == 0; }

int step_once(pic_engine* E, cudaStream_t s) {
  EngineLaunch L = make_launch(E, nullptr);
  bool sorted = false;
  int rc = sort_jobs(E, L, sort_before_first, s, &sorted);
  if (rc) return rc;
  E->launches += launch_step_begin(E->d_st, E->d_jobs, E->njobs_hw, nullptr, s);
  int max_nodes = 0;
  for (int j = 0; j < E->njobs_hw; ++j)
    if (E->jobs[j].alive) max_nodes = std::max(max_nodes, E->jobs[j].dev.nx * E->jobs[j].dev.ny);
  E->launches += launch_zero_rho_all(L, max_nodes, s);
  if (E->profile) {
    if (E->mover_events_used == E->mover_events.size()) {
      std::pair<cudaEvent_t, cudaEvent_t> ev;
      CK(cudaEventCreate(&ev.first));
      CK(cudaEventCreate(&ev.second));
      E->mover_events.push_back(ev);
    }
    L.ev_mover_begin = E->mover_events[E->mover_events_used].first;
    L.ev_mover_end = E->mover_events[E->mover_events_used].second;
    E->mover_events_used++;
  }
  E->launches += launch_mover(L, PIC_PHASE_KICK_I | PIC_PHASE_MCC_I | PIC_PHASE_DRIFT_I | PIC_PHASE_WALLS_I |
                                     PIC_PHASE_DEPOSIT_I | PIC_PHASE_GATED_I, 0, s);
  L.ev_mover_begin = L.ev_mover_end = nullptr;
  // the pairs of this step's ionisations (appended after the live particles, drifted and
  // deposited) before the field solve, which needs their charge
  E->launches += launch_ionize(L, true, s);
  // removal of the absorbed particles, then the sort due before the next step, on the side
  // stream while the field is solved (they touch only particle arrays, the solve only grids)
  CK(cudaEventRecord(E->ev_fork, s));
  CK(cudaStreamWaitEvent(E->side_stream, E->ev_fork, 0));
  phase_mark(E, 2, true, E->side_stream);
  E->launches += launch_compact(L, E->side_stream);
  phase_mark(E, 2, false, E->side_stream);
  bool side = false;
  rc = sort_jobs(E, L, sort_after, E->side_stream, &side);
  if (rc) return rc;
  CK(cudaEventRecord(E->ev_join, E->side_stream));
  phase_mark(E, 3, true, s);
  rc = solve(E, E->mg_all, nullptr, s);
  if (rc) return rc;
  phase_mark(E, 3, false, s);
  CK(cudaStreamWaitEvent(s, E->ev_join, 0));
  E->launches += launch_step_end(E->d_st, E->njobs_hw, nullptr, 1, 1, s);
  E->steps_taken++;
  for (int j = 0; j < E->njobs_hw; ++j)
    if (E->jobs[j].alive) { E->jobs[j].steps++; E->jobs[j].pending = true; }
  CK(cudaGetLastError());
  return PIC_OK;
}

// Records one full step of every live job into a CUDA graph.  The V-cycle loop of the field
// solve is a conditional WHILE node: its body is the V-cycle plus a one-thread kernel that
// keeps the loop going while any job is still iterating (bounded by max_cycles), so a step
// runs without any host synchronisation.
int build_step_graph(pic_engine* E, bool with_sort, cudaGraphExec_t* out, int64_t* fixed_launches) {
  cudaStream_t s = E->cap_stream;
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  EngineLaunch L = make_launch(E, nullptr);
  int64_t n = 0;
  int max_nodes = 0;
  for (int j = 0; j < E->njobs_hw; ++j)
    if (E->jobs[j].alive) max_nodes = std::max(max_nodes, E->jobs[j].dev.nx * E->jobs[j].dev.ny);
  cudaError_t err = cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (err != cudaSuccess) { cudaGraphDestroy(g); return fail(PIC_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(err)); }
  n += launch_step_begin(E->d_st, E->d_jobs, E->njobs_hw, nullptr, s);
  n += launch_zero_rho_all(L, max_nodes, s);
  n += launch_mover(L, PIC_PHASE_KICK_I | PIC_PHASE_MCC_I | PIC_PHASE_DRIFT_I | PIC_PHASE_WALLS_I | PIC_PHASE_DEPOSIT_I |
                           PIC_PHASE_GATED_I, 0, s);
  n += launch_ionize(L, true, s);
  // removal of the absorbed particles and the sort due before the next step, on a parallel
  // branch of the graph beside the solve
  if (err == cudaSuccess) err = cudaEventRecord(E->ev_fork, s);
  if (err == cudaSuccess) err = cudaStreamWaitEvent(E->side_stream, E->ev_fork, 0);
  n += launch_compact(L, E->side_stream);
  if (with_sort) {
    int max_cells = 0;
    int64_t max_p = 0;
    for (int j = 0; j < E->njobs_hw; ++j) {
      JobHost& J = E->jobs[j];
      if (!J.alive || J.cfg.sort_every <= 0) continue;
      for (int k = 0; k < J.cfg.n_species; ++k) max_p = std::max<int64_t>(max_p, J.cfg.species[k].capacity);
      max_cells = std::max(max_cells, J.dev.ncx * J.dev.ncy);
    }
    n += launch_sort_mask(L, E->d_mask, 1, E->side_stream);
    n += launch_sort(L, E->d_mask, max_cells, (int)std::min<int64_t>(max_p, 1 << 30), true, E->side_stream);
  }
  if (err == cudaSuccess) err = cudaEventRecord(E->ev_join, E->side_stream);
  n += launch_mg_init(L, E->mg_all.L, s);
  cudaMemsetAsync(E->d_loop, 0, sizeof(int), s);
  // conditional WHILE node for the V-cycles
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  err = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &ndeps);
  cudaGraphConditionalHandle h;
  if (err == cudaSuccess) err = cudaGraphConditionalHandleCreate(&h, cg, 1, cudaGraphCondAssignDefault);
  cudaGraphNode_t cnode = nullptr;
  alignas(cudaGraphNodeParams) unsigned char pbuf[sizeof(cudaGraphNodeParams)];
  std::memset(pbuf, 0, sizeof(pbuf));
  cudaGraphNodeParams& p = *reinterpret_cast<cudaGraphNodeParams*>(pbuf);
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  if (err == cudaSuccess) err = cudaGraphAddNode(&cnode, cg, deps, ndeps, &p);
  int64_t body = 0;
  if (err == cudaSuccess) {
    cudaGraph_t bg = p.conditional.phGraph_out[0];
    err = cudaStreamBeginCaptureToGraph(E->body_stream, bg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (err == cudaSuccess) {
      EngineLaunch LB = L;
      body += launch_mg_vcycle(LB, E->mg_all.L, E->body_stream);
      body += launch_vcycle_condition(h, E->d_running, E->d_loop, E->mg_all.max_cycles, E->d_loop_total,
                                      E->body_stream);
      cudaGraph_t tmp = nullptr;
      err = cudaStreamEndCapture(E->body_stream, &tmp);
    }
  }
  if (err == cudaSuccess) err = cudaStreamUpdateCaptureDependencies(s, &cnode, 1, cudaStreamSetCaptureDependencies);
  if (err == cudaSuccess) err = cudaStreamWaitEvent(s, E->ev_join, 0);
  if (err == cudaSuccess) n += launch_step_end(E->d_st, E->njobs_hw, nullptr, 1, 1, s);
  cudaGraph_t done = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(s, &done);
  if (err == cudaSuccess) err = e2;
  if (err == cudaSuccess) err = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (err != cudaSuccess) {
    cudaGetLastError();
    return fail(PIC_ERR_CUDA, std::string("step graph: ") + cudaGetErrorString(err));
  }
  *fixed_launches = n;
  E->graph_body_launches = body;
  return PIC_OK;
}

int ensure_graphs(pic_engine* E) {
  if (!E->graph_dirty && E->graph_exec && E->graph_exec_sort) return PIC_OK;
  if (E->graph_exec) { cudaGraphExecDestroy(E->graph_exec); E->graph_exec = nullptr; }
  if (E->graph_exec_sort) { cudaGraphExecDestroy(E->graph_exec_sort); E->graph_exec_sort = nullptr; }
  int rc = build_step_graph(E, false, &E->graph_exec, &E->graph_fixed_launches[0]);
  if (rc == PIC_OK) rc = build_step_graph(E, true, &E->graph_exec_sort, &E->graph_fixed_launches[1]);
  if (rc && E->pdl) {
    // a graph with programmatic dependencies inside the V-cycle body could not be built:
    // rebuild the multigrid plan and the graphs with ordinary launches
    if (E->graph_exec) { cudaGraphExecDestroy(E->graph_exec); E->graph_exec = nullptr; }
    E->pdl = false;
    E->mg_dirty = true;
    for (auto& J : E->jobs) J.mg.valid = false;
    rc = ensure_mg_all(E);
    if (rc == PIC_OK) rc = build_step_graph(E, false, &E->graph_exec, &E->graph_fixed_launches[0]);
    if (rc == PIC_OK) rc = build_step_graph(E, true, &E->graph_exec_sort, &E->graph_fixed_launches[1]);
  }
  if (rc) return rc;
  E->graph_dirty = false;
  return PIC_OK;
}

}  // namespace

// =====================================================================================
extern "C" {

const char* pic_last_error(void) { return g_err.c_str(); }
int pic_version(void) { return 100; }
int pic_abi_sizes(int64_t out[4]) {
  out[0] = sizeof(pic_job_config);
  out[1] = sizeof(pic_diagnostics);
  out[2] = sizeof(pic_species_config);
  out[3] = sizeof(pic_process_config);
  return PIC_OK;
}

void pic_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]}, k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
    c[0] = n0; c[1] = (uint32_t)p1; c[2] = n2; c[3] = (uint32_t)p0;
  }
  for (int i = 0; i < 4; ++i) out[i] = c[i];
}

int pic_engine_create(int device, int64_t pool_bytes, pic_engine** out) {
  if (!out) return fail(PIC_ERR_ARG, "null out");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(PIC_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= ndev) return fail(PIC_ERR_ARG, "bad device index");
  CK(cudaSetDevice(device));
  pic_engine* E = new pic_engine();
  E->device = device;
  E->pool_bytes = pool_bytes;
  cudaDeviceGetAttribute(&E->num_sms, cudaDevAttrMultiProcessorCount, device);
  E->mover_bps = mover_blocks_per_sm();
  {
    // largest cluster the device co-schedules with the shared memory its top level needs
    const int n16[] = {513, 257, 129, 65, 33, 17, 9, 5, 3};
    const size_t s16 = mg_cluster_smem(n16, 0, 9, 16);
    const int n8[] = {257, 129, 65, 33, 17, 9, 5, 3};
    const size_t s8 = mg_cluster_smem(n8, 0, 8, 8);
    if (mg_cluster_supported(16, s16) > 0) { E->cluster_C = 16; E->cluster_smem_max = s16; }
    else if (mg_cluster_supported(8, s8) > 0) { E->cluster_C = 8; E->cluster_smem_max = s8; }
    if (const char* v = std::getenv("PIC_MG_CLUSTER_TOP")) E->cluster_top = std::atoi(v);
    if (const char* v = std::getenv("PIC_MG_COARSE_TOP")) E->coarse_top = std::atoi(v);
    if (const char* v = std::getenv("PIC_PDL")) E->pdl = std::atoi(v) != 0;
    if (const char* v = std::getenv("PIC_MG_LEVELS_KERNEL")) E->levels_kernel = std::atoi(v) == 1;
    if (const char* v = std::getenv("PIC_MG_WIDE_TILES")) E->wide_factor = std::min(std::max(std::atoi(v), 0), 64);
  }
  const int nslots = kMaxJobs * kSlotsPerJob;
  cudaError_t e = cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    e = cudaMemPoolCreate(&E->pool, &props);
    if (e == cudaSuccess) {
      uint64_t keep = ~0ull;  // never trim: freed job memory stays for the next jobs
      e = cudaMemPoolSetAttribute(E->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  if (e == cudaSuccess) e = cudaMalloc(&E->d_jobs, sizeof(JobDev) * kMaxJobs);
  if (e == cudaSuccess) e = cudaMalloc(&E->d_st, sizeof(JobState) * kMaxJobs);
  if (e == cudaSuccess) e = cudaMalloc(&E->d_slots, sizeof(SlotDev) * nslots);
  if (e == cudaSuccess) e = cudaMalloc(&E->d_counts, sizeof(int) * nslots);
  if (e == cudaSuccess) e = cudaMalloc(&E->d_hits, sizeof(int) * nslots);
  if (e == cudaSuccess) e = cudaMalloc(&E->d_aux, sizeof(int) * 5 * nslots);
  if (e == cudaSuccess) e = cudaMalloc(&E->d_chunk, sizeof(int) * (nslots + 1));
  if (e == cudaSuccess) e = cudaMalloc(&E->d_running, sizeof(int) * 4);
  if (e == cudaSuccess) e = cudaMalloc(&E->d_active, nslots);
  if (e == cudaSuccess) e = cudaMalloc(&E->d_mask, nslots);
  if (e == cudaSuccess) e = cudaHostAlloc(&E->h_pinned, 64, cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaMalloc(&E->d_diag, sizeof(double) * 1024);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&E->cap_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&E->body_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&E->side_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&E->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&E->ev_join, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&E->d_loop, sizeof(int) * 4);
  if (e == cudaSuccess) e = cudaMalloc(&E->d_loop_total, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(E->d_loop_total, 0, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(E->d_counts, 0, sizeof(int) * nslots);
  if (e == cudaSuccess) e = cudaMemset(E->d_hits, 0, sizeof(int) * nslots);
  if (e == cudaSuccess) e = cudaMemset(E->d_aux, 0, sizeof(int) * 5 * nslots);
  if (e == cudaSuccess) e = cudaMemset(E->d_active, 0, nslots);
  if (e == cudaSuccess) e = cudaMemset(E->d_st, 0, sizeof(JobState) * kMaxJobs);
  if (e == cudaSuccess) e = cudaMemset(E->d_jobs, 0, sizeof(JobDev) * kMaxJobs);
  if (e == cudaSuccess) e = cudaMemset(E->d_slots, 0, sizeof(SlotDev) * nslots);
  if (e != cudaSuccess) {
    pic_engine_destroy(E);
    cudaGetLastError();
    return fail(PIC_ERR_OOM, std::string("engine tables: ") + cudaGetErrorString(e));
  }
  E->jobs.resize(kMaxJobs);
  E->h_active.assign(nslots, 0);
  *out = E;
  return PIC_OK;
}

int pic_engine_destroy(pic_engine* E) {
  if (!E) return PIC_OK;
  cudaSetDevice(E->device);
  if (E->stream) cudaStreamSynchronize(E->stream);
  for (auto& J : E->jobs)
    if (J.alive) free_job(E, J);
  E->mg_all.release();
  if (E->graph_exec) cudaGraphExecDestroy(E->graph_exec);
  if (E->graph_exec_sort) cudaGraphExecDestroy(E->graph_exec_sort);
  if (E->cap_stream) cudaStreamDestroy(E->cap_stream);
  if (E->body_stream) cudaStreamDestroy(E->body_stream);
  if (E->side_stream) cudaStreamDestroy(E->side_stream);
  if (E->ev_fork) cudaEventDestroy(E->ev_fork);
  if (E->ev_join) cudaEventDestroy(E->ev_join);
  if (E->d_loop) cudaFree(E->d_loop);
  if (E->d_loop_total) cudaFree(E->d_loop_total);
  cudaFree(E->d_jobs); cudaFree(E->d_st); cudaFree(E->d_slots); cudaFree(E->d_counts); cudaFree(E->d_hits);
  cudaFree(E->d_aux); cudaFree(E->d_chunk); cudaFree(E->d_running); cudaFree(E->d_active); cudaFree(E->d_mask);
  cudaFree(E->d_diag);
  if (E->d_stage) cudaFree(E->d_stage);
  for (auto& ev : E->mover_events) { cudaEventDestroy(ev.first); cudaEventDestroy(ev.second); }
  for (int ph = 0; ph < 4; ++ph)
    for (auto& ev : E->phase_events[ph]) { cudaEventDestroy(ev.first); cudaEventDestroy(ev.second); }
  if (E->h_pinned) cudaFreeHost(E->h_pinned);
  if (E->stream) cudaStreamDestroy(E->stream);
  if (E->pool) cudaMemPoolDestroy(E->pool);
  delete E;
  return PIC_OK;
}

int pic_engine_reserve(pic_engine* E, int64_t bytes) {
  if (!E) return fail(PIC_ERR_ARG, "null engine");
  if (bytes < 0) return fail(PIC_ERR_ARG, "negative reservation");
  if (bytes == 0) return PIC_OK;
  CK(cudaSetDevice(E->device));
  void* p = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&p, (size_t)bytes, E->pool, E->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(PIC_ERR_OOM, std::string("cudaMallocFromPoolAsync: ") + cudaGetErrorString(e));
  }
  CK(cudaFreeAsync(p, E->stream));
  CK(cudaStreamSynchronize(E->stream));
  return PIC_OK;
}

int pic_engine_bytes_needed(const pic_job_config* cfg, int64_t* bytes) {
  std::string why;
  const int rc = validate(cfg, why);
  if (rc) return fail(rc, why);
  if (bytes) *bytes = job_layout(*cfg).total;
  return PIC_OK;
}

int pic_engine_num_jobs(pic_engine* E, int* n) {
  if (!E || !n) return fail(PIC_ERR_ARG, "null argument");
  int c = 0;
  for (int j = 0; j < E->njobs_hw; ++j) c += E->jobs[j].alive;
  *n = c;
  return PIC_OK;
}

int pic_job_create(pic_engine* E, const pic_job_config* cfg, int* job_id) {
  if (!E || !job_id) return fail(PIC_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(E->mu);
  std::string why;
  int rc = validate(cfg, why);
  if (rc) return fail(rc, why);
  CK(cudaSetDevice(E->device));
  int id = -1;
  for (int j = 0; j < kMaxJobs; ++j)
    if (!E->jobs[j].alive) { id = j; break; }
  if (id < 0) return fail(PIC_ERR_CAPACITY, "engine job table full");
  const Layout lay = job_layout(*cfg, E->cluster_C, E->cluster_top, E->coarse_top);
  if (E->pool_bytes > 0 && E->used_bytes + lay.total > E->pool_bytes) return fail(PIC_ERR_OOM, "engine memory budget exceeded");
  JobHost& J = E->jobs[id];
  J = JobHost();
  J.cfg = *cfg;
  for (int i = 0; i < cfg->n_processes; ++i) { J.cfg.processes[i].energy_ev = nullptr; J.cfg.processes[i].sigma_m2 = nullptr; }
  J.alive = true;
  JobDev& D = J.dev;
  const pic_job_config& c = *cfg;
  D.nx = c.nx; D.ny = c.ny; D.ncx = c.nx - 1; D.ncy = c.ny - 1;
  D.levels = lay.levels; D.lc = lay.lc;
  for (int l = 0; l < lay.levels; ++l) { D.nl[l] = lay.nl[l]; D.pl[l] = mgt::round4(lay.nl[l]); }
  const double dx = c.Lx / (c.nx - 1), dy = c.Ly / (c.ny - 1);
  D.h = dx;
  D.dt = (float)c.dt;
  double qref = 0.0;
  for (int s = 0; s < c.n_species; ++s) qref = std::max(qref, std::fabs(c.species[s].charge * c.species[s].weight));
  if (qref == 0.0) qref = 1.0;
  D.qref = qref;
  D.rhs_scale = qref * (c.units == PIC_UNITS_SI ? -1.0 / (kEps0 * dx * dy) : 1.0);
  D.omega = (float)c.omega;
  D.nu_pre = c.nu_pre; D.nu_post = c.nu_post; D.nu_coarse = c.nu_coarse;
  D.tol = c.tol; D.max_cycles = c.max_cycles;
  D.deposit_mode = c.deposit_mode; D.wall_mode = c.wall_mode; D.n_walls = c.n_walls; D.mcc_mode = c.mcc_mode;
  D.gas_density = (float)c.gas_density;
  D.gas_mass = (float)c.gas_mass;
  D.vth_neutral = (c.gas_mass > 0) ? (float)std::sqrt(kKb * c.gas_temperature / c.gas_mass) : 0.f;
  D.ion_e_species = c.ionization_electron_species;
  D.ion_i_species = c.ionization_ion_species;
  D.seed = c.seed;
  D.slot0 = id * kSlotsPerJob;
  D.nslots = c.n_species;
  D.sort_every = c.sort_every;
  const int64_t N = (int64_t)c.nx * c.ny;
  auto A = [&](void** p, size_t b) { return dev_alloc(E, J, p, b); };
#define ALLOC(ptr, bytes)                                  \
  do {                                                     \
    int r_ = A((void**)&(ptr), (size_t)(bytes));           \
    if (r_) { free_job(E, J); return r_; }                 \
  } while (0)
  if (c.deposit_mode == PIC_DEPOSIT_F32) ALLOC(D.rho_f, N * 4); else ALLOC(D.rho_i, N * 8);
  ALLOC(D.efield, N * 8);
  ALLOC(D.phi64[0], N * 8);
  ALLOC(D.phi64[1], N * 8);
  if (c.mg_warm_start) ALLOC(D.phi64[2], N * 8);
  D.warm_start = c.mg_warm_start;
  for (int l = 0; l < lay.levels; ++l) {
    ALLOC(D.e[l], 4ll * D.pl[l] * lay.nl[l]);
    ALLOC(D.f[l], 4ll * D.pl[l] * lay.nl[l]);
    if (l > 0) ALLOC(D.eu[l], 4ll * D.pl[l] * lay.nl[l]);
  }
  ALLOC(D.f0b, 4ll * D.pl[0] * c.ny);
  {
    CUtensorMap* tm = nullptr;
    ALLOC(tm, sizeof(CUtensorMap) * mgt::kTmapsPerLevel * lay.levels);
    CK(cudaStreamSynchronize(E->stream));   // the pool allocations above have completed
    const int rc = make_tile_maps(D, c.nu_pre, c.nu_post, tm);
    if (rc) { free_job(E, J); return rc; }
    D.tmaps = tm;
  }
  ALLOC(D.partials, 24ll * lay.ntiles0);   // per level-0 tile: r^2, F^2 (pairs), then charge
  if (c.n_walls > 0) {
    std::vector<double> w(4 * c.n_walls);
    for (int k = 0; k < c.n_walls; ++k) {
      w[4 * k] = c.walls[k][0] / dx; w[4 * k + 1] = c.walls[k][1] / dy;
      w[4 * k + 2] = c.walls[k][2] / dx; w[4 * k + 3] = c.walls[k][3] / dy;
    }
    double* dw = nullptr;
    ALLOC(dw, w.size() * 8);
    CK(cudaStreamSynchronize(E->stream));
    CK(cudaMemcpy(dw, w.data(), w.size() * 8, cudaMemcpyHostToDevice));
    D.walls = dw;
  }
  // MCC tables
  std::vector<ProcDev> procs;
  std::vector<std::vector<float>> proc_tabs;   // host copies of the FP32 tables, as on the device
  if (c.mcc_mode) {
    // order processes by species so each species' processes are contiguous
    std::vector<int> order(c.n_processes);
    for (int i = 0; i < c.n_processes; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return c.processes[a].species < c.processes[b].species; });
    for (int oi : order) {
      const pic_process_config& p = c.processes[oi];
      std::vector<float> tab(2 * p.n_points);
      for (int k = 0; k < p.n_points; ++k) { tab[k] = (float)p.energy_ev[k]; tab[p.n_points + k] = (float)p.sigma_m2[k]; }
      float* dt_ = nullptr;
      ALLOC(dt_, tab.size() * 4);
      CK(cudaStreamSynchronize(E->stream));
      CK(cudaMemcpy(dt_, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice));
      ProcDev pd{};
      pd.type = p.type; pd.species = p.species; pd.threshold = (float)p.threshold_ev; pd.n = p.n_points;
      pd.e = dt_; pd.s = dt_ + p.n_points;
      // log-spaced lookup hint if the energies are log-spaced to 1e-4
      bool logsp = p.energy_ev[0] > 0;
      const double r0 = logsp ? std::log(p.energy_ev[1] / p.energy_ev[0]) : 0.0;
      for (int k = 1; logsp && k < p.n_points; ++k)
        if (!(p.energy_ev[k] > 0) || std::fabs(std::log(p.energy_ev[k] / p.energy_ev[k - 1]) - r0) > 1e-4 * std::fabs(r0)) logsp = false;
      pd.log_e0 = logsp ? (float)std::log(p.energy_ev[0]) : 0.f;
      pd.inv_dlog = logsp ? (float)(1.0 / r0) : 0.f;
      procs.push_back(pd);
      proc_tabs.push_back(tab);
    }
    ProcDev* dp = nullptr;
    ALLOC(dp, procs.size() * sizeof(ProcDev));
    CK(cudaStreamSynchronize(E->stream));
    CK(cudaMemcpy(dp, procs.data(), procs.size() * sizeof(ProcDev), cudaMemcpyHostToDevice));
    D.procs = dp;
    D.n_proc = (int)procs.size();
  }
  const int evcap = event_capacity(c);
  if (evcap) {
    int p2 = 1;
    while (p2 < evcap) p2 <<= 1;
    ALLOC(D.events, (size_t)evcap * sizeof(Event) + (size_t)p2 * 8);
    D.event_capacity = evcap;
  }
  D.up_tiles0 = lay.ntiles0;
  // particle slots
  const int64_t ncells = (int64_t)D.ncx * D.ncy + 1;
  for (int s = 0; s < kSlotsPerJob; ++s) {
    SlotDev& S = J.slot[s];
    S = SlotDev{};
    S.job = id;
    S.species = s;
    if (s >= c.n_species) continue;
    const pic_species_config& sp = c.species[s];
    const int64_t cap = round_up(std::max<int64_t>(sp.capacity, 1), PIC_CHUNK);
    S.capacity = sp.capacity;
    ALLOC(S.cell, cap * 4); ALLOC(S.fx, cap * 4); ALLOC(S.fy, cap * 4); ALLOC(S.vx, cap * 4);
    ALLOC(S.vy, cap * 4); ALLOC(S.vz, cap * 4); ALLOC(S.pid, cap * 4);
    ALLOC(S.cell_b, cap * 4); ALLOC(S.fx_b, cap * 4); ALLOC(S.fy_b, cap * 4); ALLOC(S.vx_b, cap * 4);
    ALLOC(S.vy_b, cap * 4); ALLOC(S.vz_b, cap * 4); ALLOC(S.pid_b, cap * 4);
    ALLOC(S.hits, cap * 4); ALLOC(S.scratch, cap * 4); ALLOC(S.scratch2, cap * 4);
    ALLOC(S.cell_count, ncells * 4);
    ALLOC(S.scan_part, ((ncells + 2047) / 2048 + 1) * 4);
    CK(cudaStreamSynchronize(E->stream));
    CK(cudaMemset(S.scratch, 0, cap * 4));
    // zero the vector tails so the mover's whole-chunk loads read defined values
    CK(cudaMemset(S.cell, 0, cap * 4)); CK(cudaMemset(S.fx, 0, cap * 4)); CK(cudaMemset(S.fy, 0, cap * 4));
    CK(cudaMemset(S.vx, 0, cap * 4)); CK(cudaMemset(S.vy, 0, cap * 4)); CK(cudaMemset(S.vz, 0, cap * 4));
    CK(cudaMemset(S.pid, 0, cap * 4));
    S.qdep = (float)(sp.charge * sp.weight / qref);
    S.qfix = std::llrint(sp.charge * sp.weight / qref * 1099511627776.0);
    S.kx = (float)(sp.charge / sp.mass * c.dt / dx);
    S.ky = (float)(sp.charge / sp.mass * c.dt / dy);
    S.dtdx = (float)(c.dt / dx);
    S.dtdy = (float)(c.dt / dy);
    S.half_m_over_e = (float)(0.5 * sp.mass / kQe);
    S.mass = (float)sp.mass;
    S.ke_factor = 0.5 * sp.mass * sp.weight;
    int first = 0, cnt = 0;
    for (size_t k = 0; k < procs.size(); ++k) {
      if (procs[k].species == s) { if (!cnt) first = (int)k; ++cnt; }
    }
    S.first_proc = first;
    S.n_proc = cnt;
    if (c.mcc_mode == PIC_MCC_NULL_COLLISION && cnt) {
      // the species' total cross section: every table is piecewise linear, so their sum is
      // piecewise linear on the union of their energy points (evaluated as the device does:
      // clamped outside each table, linear inside)
      std::vector<float> ug;
      for (int k = first; k < first + cnt; ++k)
        ug.insert(ug.end(), proc_tabs[k].begin(), proc_tabs[k].begin() + procs[k].n);
      std::sort(ug.begin(), ug.end());
      ug.erase(std::unique(ug.begin(), ug.end()), ug.end());
      const int nu = (int)ug.size();
      std::vector<float> tt(2 * (size_t)nu);
      for (int u = 0; u < nu; ++u) {
        double sum = 0.0;
        for (int k = first; k < first + cnt; ++k) {
          const int np = procs[k].n;
          const float* e = proc_tabs[k].data();
          const float* sg = e + np;
          const float E = ug[u];
          if (E <= e[0]) { sum += sg[0]; continue; }
          if (E >= e[np - 1]) { sum += sg[np - 1]; continue; }
          const int q = (int)(std::upper_bound(e, e + np, E) - e) - 1;
          const double t = ((double)E - e[q]) / ((double)e[q + 1] - e[q]);
          sum += sg[q] + t * ((double)sg[q + 1] - sg[q]);
        }
        tt[u] = ug[u];
        tt[nu + u] = (float)sum;
      }
      float* dtt = nullptr;
      ALLOC(dtt, tt.size() * 4);
      CK(cudaStreamSynchronize(E->stream));
      CK(cudaMemcpy(dtt, tt.data(), tt.size() * 4, cudaMemcpyHostToDevice));
      ProcDev& T = S.total;
      T = ProcDev{};
      T.type = 0; T.species = s; T.n = nu; T.e = dtt; T.s = dtt + nu;
      bool logsp = nu >= 2 && ug[0] > 0.f;
      const double r0 = logsp ? std::log((double)ug[1] / ug[0]) : 0.0;
      for (int k = 1; logsp && k < nu; ++k)
        if (std::fabs(std::log((double)ug[k] / ug[k - 1]) - r0) > 1e-4 * std::fabs(r0)) logsp = false;
      T.log_e0 = logsp ? (float)std::log((double)ug[0]) : 0.f;
      T.inv_dlog = logsp ? (float)(1.0 / r0) : 0.f;
    }
    if (c.mcc_mode == PIC_MCC_NULL_COLLISION && cnt) {
      const double numax = compute_numax(c, s);
      if (numax * c.dt > 1.0) { free_job(E, J); return fail(PIC_ERR_ARG, "nu_max * dt > 1: time step too large for MCC"); }
      S.numax = (float)numax;
      S.pnull = (float)(numax * c.dt);  // first order: real collision j with probability n sigma_j v dt
    }
  }
#undef ALLOC
  CK(cudaStreamSynchronize(E->stream));   // every allocation of the job has completed
  CK(cudaMemset(D.phi64[0], 0, N * 8));
  CK(cudaMemset(D.phi64[1], 0, N * 8));
  if (D.phi64[2]) CK(cudaMemset(D.phi64[2], 0, N * 8));
  CK(cudaMemset(D.efield, 0, N * 8));
  if (D.rho_f) CK(cudaMemset(D.rho_f, 0, N * 4));
  if (D.rho_i) CK(cudaMemset(D.rho_i, 0, N * 8));
  for (int l = 0; l < lay.levels; ++l) {
    CK(cudaMemset(D.e[l], 0, 4ll * D.pl[l] * lay.nl[l]));
    CK(cudaMemset(D.f[l], 0, 4ll * D.pl[l] * lay.nl[l]));
    if (D.eu[l]) CK(cudaMemset(D.eu[l], 0, 4ll * D.pl[l] * lay.nl[l]));
  }
  CK(cudaMemset(D.f0b, 0, 4ll * D.pl[0] * c.ny));
  CK(cudaMemcpy(E->d_jobs + id, &D, sizeof(JobDev), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(E->d_slots + id * kSlotsPerJob, J.slot, sizeof(SlotDev) * kSlotsPerJob, cudaMemcpyHostToDevice));
  CK(cudaMemset(E->d_st + id, 0, sizeof(JobState)));
  CK(cudaMemset(E->d_counts + id * kSlotsPerJob, 0, sizeof(int) * kSlotsPerJob));
  CK(cudaMemset(E->d_hits + id * kSlotsPerJob, 0, sizeof(int) * kSlotsPerJob));
  CK(cudaMemset(E->d_aux + 4 * id * kSlotsPerJob, 0, sizeof(int) * 4 * kSlotsPerJob));
  for (int s = 0; s < kSlotsPerJob; ++s) E->h_active[id * kSlotsPerJob + s] = s < c.n_species ? 1 : 0;
  E->njobs_hw = std::max(E->njobs_hw, id + 1);
  rc = upload_active(E);
  if (rc) return rc;
  E->max_nu_pre = std::max(E->max_nu_pre, c.nu_pre);
  E->max_nu_post = std::max(E->max_nu_post, c.nu_post);
  E->mg_dirty = true;
  E->graph_dirty = true;
  *job_id = id;
  return PIC_OK;
}

int pic_job_destroy(pic_engine* E, int job) {
  int rc = check_job(E, job);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(E->mu);
  CK(cudaSetDevice(E->device));
  CK(cudaStreamSynchronize(E->stream));
  free_job(E, E->jobs[job]);
  for (int s = 0; s < kSlotsPerJob; ++s) E->h_active[job * kSlotsPerJob + s] = 0;
  JobDev z{};
  CK(cudaMemcpy(E->d_jobs + job, &z, sizeof(JobDev), cudaMemcpyHostToDevice));
  CK(cudaMemset(E->d_counts + job * kSlotsPerJob, 0, sizeof(int) * kSlotsPerJob));
  CK(cudaMemset(E->d_slots + job * kSlotsPerJob, 0, sizeof(SlotDev) * kSlotsPerJob));
  rc = upload_active(E);
  if (rc) return rc;
  while (E->njobs_hw > 0 && !E->jobs[E->njobs_hw - 1].alive) E->njobs_hw--;
  E->mg_dirty = true;
  E->graph_dirty = true;
  return PIC_OK;
}

int pic_job_load_species(pic_engine* E, int job, int species, int64_t n, const double* x, const double* y,
                         const double* vx, const double* vy, const double* vz, const uint32_t* pid, int memory) {
  int rc = check_job(E, job);
  if (rc) return rc;
  JobHost& J = E->jobs[job];
  if (species < 0 || species >= J.cfg.n_species) return fail(PIC_ERR_ARG, "bad species");
  if (n < 0 || n > J.cfg.species[species].capacity) return fail(PIC_ERR_CAPACITY, "more particles than capacity");
  if (n > 0 && (!x || !y || !vx || !vy)) return fail(PIC_ERR_ARG, "null particle arrays");
  CK(cudaSetDevice(E->device));
  cudaStream_t s = E->stream;
  rc = flush(E, s, job);
  if (rc) return rc;
  const double *dx_ = x, *dy_ = y, *dvx = vx, *dvy = vy, *dvz = vz;
  const uint32_t* dpid = pid;
  // device arrays may still be in the making on another stream (the engine's streams do not
  // wait for the legacy default stream): wait for all work issued so far on the device
  if (memory == PIC_MEM_DEVICE && n > 0) CK(cudaDeviceSynchronize());
  if (memory == PIC_MEM_HOST && n > 0) {
    const size_t nb = (size_t)n * 8;
    rc = ensure_stage(E, nb * 5 + (size_t)n * 4);
    if (rc) return rc;
    char* st = (char*)E->d_stage;
    double* b[5];
    const double* src[5] = {x, y, vx, vy, vz};
    for (int k = 0; k < 5; ++k) {
      b[k] = (double*)(st + k * nb);
      if (src[k]) CK(cudaMemcpyAsync(b[k], src[k], nb, cudaMemcpyHostToDevice, s));
    }
    dx_ = b[0]; dy_ = b[1]; dvx = b[2]; dvy = b[3]; dvz = vz ? b[4] : nullptr;
    if (pid) {
      uint32_t* pb = (uint32_t*)(st + 5 * nb);
      CK(cudaMemcpyAsync(pb, pid, (size_t)n * 4, cudaMemcpyHostToDevice, s));
      dpid = pb;
    }
  }
  // pid base for implicit ids: the job's current next_pid
  JobState hs;
  CK(cudaMemcpyAsync(&hs, E->d_st + job, sizeof(JobState), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  const double dxv = J.cfg.Lx / (J.cfg.nx - 1), dyv = J.cfg.Ly / (J.cfg.ny - 1);
  const SlotDev* sd = E->d_slots + job * kSlotsPerJob + species;
  launch_load_species(sd, nullptr, n, dx_, dy_, dvx, dvy, dvz, dpid, hs.next_pid, 1.0 / dxv, 1.0 / dyv, J.dev.ncx,
                      J.dev.ncy, s);
  const int ni = (int)n;
  CK(cudaMemcpyAsync(E->d_counts + job * kSlotsPerJob + species, &ni, sizeof(int), cudaMemcpyHostToDevice, s));
  if (dpid) {
    launch_pid_max(sd, n, E->d_st + job, s);
  } else {
    const uint32_t np = hs.next_pid + (uint32_t)n;
    CK(cudaMemcpyAsync(&E->d_st[job].next_pid, &np, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  }
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return PIC_OK;
}

static int read_count(pic_engine* E, int job, int species, int* n) {
  CK(cudaMemcpyAsync(E->h_pinned, E->d_counts + job * kSlotsPerJob + species, sizeof(int), cudaMemcpyDeviceToHost,
                     E->stream));
  CK(cudaStreamSynchronize(E->stream));
  *n = *E->h_pinned;
  return PIC_OK;
}

int pic_job_export_species(pic_engine* E, int job, int species, int64_t capacity, double* x, double* y, double* vx,
                           double* vy, double* vz, uint32_t* pid, int64_t* n_out, int memory) {
  int rc = check_job(E, job);
  if (rc) return rc;
  JobHost& J = E->jobs[job];
  if (species < 0 || species >= J.cfg.n_species) return fail(PIC_ERR_ARG, "bad species");
  CK(cudaSetDevice(E->device));
  cudaStream_t s = E->stream;
  rc = flush(E, s, job);
  if (rc) return rc;
  int n = 0;
  rc = read_count(E, job, species, &n);
  if (rc) return rc;
  if (n_out) *n_out = n;
  if (n > capacity) return fail(PIC_ERR_CAPACITY, "output arrays too small");
  const double dxv = J.cfg.Lx / (J.cfg.nx - 1), dyv = J.cfg.Ly / (J.cfg.ny - 1);
  const SlotDev* sd = E->d_slots + job * kSlotsPerJob + species;
  if (memory == PIC_MEM_DEVICE) {
    launch_export_species(sd, n, x, y, vx, vy, vz, pid, dxv, dyv, s);
  } else if (n > 0) {
    const size_t nb = (size_t)n * 8;
    rc = ensure_stage(E, nb * 5 + (size_t)n * 4);
    if (rc) return rc;
    char* st = (char*)E->d_stage;
    double* b[5];
    for (int k = 0; k < 5; ++k) b[k] = (double*)(st + k * nb);
    uint32_t* pb = (uint32_t*)(st + 5 * nb);
    launch_export_species(sd, n, x ? b[0] : nullptr, y ? b[1] : nullptr, vx ? b[2] : nullptr, vy ? b[3] : nullptr,
                          vz ? b[4] : nullptr, pid ? pb : nullptr, dxv, dyv, s);
    double* dst[5] = {x, y, vx, vy, vz};
    for (int k = 0; k < 5; ++k)
      if (dst[k]) CK(cudaMemcpyAsync(dst[k], b[k], nb, cudaMemcpyDeviceToHost, s));
    if (pid) CK(cudaMemcpyAsync(pid, pb, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return PIC_OK;
}

int pic_job_snapshot_positions(pic_engine* E, int job, int species, int64_t capacity, float* xy, int64_t* n_out,
                               int memory) {
  int rc = check_job(E, job);
  if (rc) return rc;
  JobHost& J = E->jobs[job];
  if (species < 0 || species >= J.cfg.n_species) return fail(PIC_ERR_ARG, "bad species");
  if (!xy && capacity > 0) return fail(PIC_ERR_ARG, "null output buffer");
  CK(cudaSetDevice(E->device));
  cudaStream_t s = E->stream;
  int n = 0;
  rc = read_count(E, job, species, &n);   // positions do not depend on a pending kick: no flush
  if (rc) return rc;
  if (n_out) *n_out = n;
  if (n > capacity) return fail(PIC_ERR_CAPACITY, "output buffer too small");
  const double dxv = J.cfg.Lx / (J.cfg.nx - 1), dyv = J.cfg.Ly / (J.cfg.ny - 1);
  const SlotDev* sd = E->d_slots + job * kSlotsPerJob + species;
  if (memory == PIC_MEM_DEVICE) {
    launch_snapshot(sd, n, xy, dxv, dyv, s);
  } else if (n > 0) {
    rc = ensure_stage(E, (size_t)n * 8);
    if (rc) return rc;
    launch_snapshot(sd, n, (float*)E->d_stage, dxv, dyv, s);
    CK(cudaMemcpyAsync(xy, E->d_stage, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return PIC_OK;
}

int pic_job_export_species_raw(pic_engine* E, int job, int species, int64_t capacity, uint32_t* cell, float* fx,
                               float* fy, float* vx, float* vy, float* vz, uint32_t* pid, int64_t* n_out) {
  int rc = check_job(E, job);
  if (rc) return rc;
  if (species < 0 || species >= E->jobs[job].cfg.n_species) return fail(PIC_ERR_ARG, "bad species");
  CK(cudaSetDevice(E->device));
  rc = flush(E, E->stream, job);
  if (rc) return rc;
  int n = 0;
  rc = read_count(E, job, species, &n);
  if (rc) return rc;
  if (n_out) *n_out = n;
  if (n > capacity) return fail(PIC_ERR_CAPACITY, "output arrays too small");
  launch_export_raw(E->d_slots + job * kSlotsPerJob + species, n, cell, fx, fy, vx, vy, vz, pid, E->stream);
  CK(cudaStreamSynchronize(E->stream));
  CK(cudaGetLastError());
  return PIC_OK;
}

int pic_step(pic_engine* E, int nsteps, void* stream) {
  if (!E) return fail(PIC_ERR_ARG, "null engine");
  if (nsteps < 0) return fail(PIC_ERR_ARG, "negative nsteps");
  std::lock_guard<std::mutex> lk(E->mu);
  CK(cudaSetDevice(E->device));
  int rc = ensure_mg_all(E);
  if (rc) return rc;
  cudaStream_t s = pick(E, stream);
  for (int k = 0; k < nsteps; ++k) {
    rc = step_once(E, s);
    if (rc) return rc;
  }
  if (nsteps > 0)
    for (int j = 0; j < E->njobs_hw; ++j)
      if (E->jobs[j].alive) E->jobs[j].charge_fresh = true;
  return PIC_OK;
}

int pic_step_graph(pic_engine* E, int nsteps, void* stream) {
  if (!E) return fail(PIC_ERR_ARG, "null engine");
  if (nsteps < 0) return fail(PIC_ERR_ARG, "negative nsteps");
  std::lock_guard<std::mutex> lk(E->mu);
  CK(cudaSetDevice(E->device));
  int rc = ensure_mg_all(E);
  if (rc) return rc;
  rc = ensure_graphs(E);
  if (rc) return rc;
  cudaStream_t s = pick(E, stream);
  for (int k = 0; k < nsteps; ++k) {
    bool sorted = false;
    rc = sort_jobs(E, make_launch(E, nullptr), sort_before_first, s, &sorted);
    if (rc) return rc;
    bool sort_due = false;
    for (int j = 0; j < E->njobs_hw; ++j) {
      const JobHost& J = E->jobs[j];
      if (J.alive && J.cfg.sort_every > 0 && sort_after(J)) sort_due = true;
    }
    CK(cudaGraphLaunch(sort_due ? E->graph_exec_sort : E->graph_exec, s));
    E->launches += E->graph_fixed_launches[sort_due ? 1 : 0];
    E->graph_steps++;
    E->steps_taken++;
    for (int j = 0; j < E->njobs_hw; ++j)
      if (E->jobs[j].alive) { E->jobs[j].steps++; E->jobs[j].pending = true; E->jobs[j].charge_fresh = true; }
  }
  return PIC_OK;
}

int pic_engine_profile(pic_engine* E, int enable) {
  if (!E) return fail(PIC_ERR_ARG, "null engine");
  E->profile = enable != 0;
  return PIC_OK;
}

int pic_engine_get_stats(pic_engine* E, pic_engine_stats* out, int reset) {
  if (!E || !out) return fail(PIC_ERR_ARG, "null argument");
  CK(cudaSetDevice(E->device));
  std::memset(out, 0, sizeof(*out));
  unsigned long long loops = 0;
  CK(cudaMemcpy(&loops, E->d_loop_total, sizeof(loops), cudaMemcpyDeviceToHost));
  out->kernel_launches = E->launches + (int64_t)loops * E->graph_body_launches;
  out->steps = E->steps_taken;
  out->vcycles = E->vcycles + (int64_t)loops;
  double ms = 0.0;
  for (size_t k = 0; k < E->mover_events_used; ++k) {
    CK(cudaEventSynchronize(E->mover_events[k].second));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, E->mover_events[k].first, E->mover_events[k].second));
    ms += t;
  }
  out->mover_launches = (int64_t)E->mover_events_used;
  out->mover_ms = ms;
  for (int ph = 0; ph < 4; ++ph) {
    double t = 0.0;
    for (size_t k = 0; k < E->phase_used[ph]; ++k) {
      CK(cudaEventSynchronize(E->phase_events[ph][k].second));
      float x = 0.f;
      CK(cudaEventElapsedTime(&x, E->phase_events[ph][k].first, E->phase_events[ph][k].second));
      t += x;
    }
    out->phase_ms[ph] = t;
  }
  out->phase_ms[1] = ms;
  if (reset) {
    E->launches = E->steps_taken = E->vcycles = 0;
    CK(cudaMemset(E->d_loop_total, 0, sizeof(unsigned long long)));
    E->mover_events_used = 0;
    for (int ph = 0; ph < 4; ++ph) E->phase_used[ph] = 0;
  }
  return PIC_OK;
}

int pic_sync(pic_engine* E) {
  if (!E) return fail(PIC_ERR_ARG, "null engine");
  CK(cudaSetDevice(E->device));
  CK(cudaStreamSynchronize(E->stream));
  CK(cudaDeviceSynchronize());
  return PIC_OK;
}

int pic_job_diagnostics(pic_engine* E, int job, pic_diagnostics* out) {
  int rc = check_job(E, job);
  if (rc) return rc;
  if (!out) return fail(PIC_ERR_ARG, "null out");
  CK(cudaSetDevice(E->device));
  cudaStream_t s = E->stream;
  CK(cudaDeviceSynchronize());
  // the last field solve summed rho already unless rho changed since
  if (!E->jobs[job].charge_fresh)
    launch_rho_sum(E->d_jobs + job, E->d_st + job, E->d_diag, std::min(1024, 2 * E->num_sms), s);
  JobState T;
  int cnt[kSlotsPerJob], ab[kSlotsPerJob];
  CK(cudaMemcpyAsync(&T, E->d_st + job, sizeof(JobState), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(cnt, E->d_counts + job * kSlotsPerJob, sizeof(cnt), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(ab, E->d_aux + 4 * kMaxJobs * kSlotsPerJob + job * kSlotsPerJob, sizeof(ab),
                     cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  std::memset(out, 0, sizeof(*out));
  JobHost& J = E->jobs[job];
  out->step = T.step;
  for (int k = 0; k < J.cfg.n_species; ++k) {
    out->count[k] = cnt[k];
    out->absorbed[k] = ab[k];
    out->kinetic_energy[k] = T.ke[k];
    // the device counts per process of the species, in configuration order; the diagnostics
    // report them at the process's index in the job configuration
    int q = 0;
    for (int p = 0; p < J.cfg.n_processes && p < PIC_MAX_PROCESSES; ++p)
      if (J.cfg.processes[p].species == k) out->collisions[k][p] = q < 8 ? (int64_t)T.collisions[k][q++] : 0;
  }
  out->ionizations = T.ionizations;
  out->vcycles = T.cycles;
  out->converged = T.converged == 1;
  out->relres = T.relres;
  out->total_charge = T.total_charge;
  out->status = T.status;
  out->next_pid = T.next_pid;
  return PIC_OK;
}

int pic_job_run_phases(pic_engine* E, int job, int flags, int64_t step_index, void* stream) {
  int rc = check_job(E, job);
  if (rc) return rc;
  E->jobs[job].charge_fresh = false;
  CK(cudaSetDevice(E->device));
  cudaStream_t s = pick(E, stream);
  rc = flush(E, s, job);
  if (rc) return rc;
  rc = job_mask(E, job, s);
  if (rc) return rc;
  if (flags & PIC_PHASE_WALLS) CK(cudaMemsetAsync(E->d_hits + job * kSlotsPerJob, 0, sizeof(int) * kSlotsPerJob, s));
  EngineLaunch L = make_launch(E, E->d_mask);
  launch_mover(L, flags & 31, (uint32_t)step_index, s);
  if (flags & PIC_PHASE_MCC) launch_ionize(L, (flags & PIC_PHASE_DRIFT) != 0, s);
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return PIC_OK;
}

int pic_job_compact(pic_engine* E, int job, void* stream) {
  int rc = check_job(E, job);
  if (rc) return rc;
  CK(cudaSetDevice(E->device));
  cudaStream_t s = pick(E, stream);
  rc = job_mask(E, job, s);
  if (rc) return rc;
  EngineLaunch L = make_launch(E, E->d_mask);
  launch_compact(L, s);
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return PIC_OK;
}

int pic_job_zero_rho(pic_engine* E, int job, void* stream) {
  int rc = check_job(E, job);
  if (rc) return rc;
  E->jobs[job].charge_fresh = false;
  CK(cudaSetDevice(E->device));
  JobDev& D = E->jobs[job].dev;
  launch_zero_rho(nullptr, (int64_t)D.nx * D.ny, D.deposit_mode, D.deposit_mode == 0 ? (void*)D.rho_f : (void*)D.rho_i,
                  pick(E, stream));
  CK(cudaGetLastError());
  return PIC_OK;
}

int pic_job_sort(pic_engine* E, int job, void* stream) {
  int rc = check_job(E, job);
  if (rc) return rc;
  CK(cudaSetDevice(E->device));
  cudaStream_t s = pick(E, stream);
  rc = job_mask(E, job, s);
  if (rc) return rc;
  JobHost& J = E->jobs[job];
  int64_t maxp = 0;
  for (int k = 0; k < J.cfg.n_species; ++k) maxp = std::max<int64_t>(maxp, J.cfg.species[k].capacity);
  EngineLaunch L = make_launch(E, nullptr);
  launch_sort(L, E->d_mask, J.dev.ncx * J.dev.ncy, (int)std::min<int64_t>(maxp, 1 << 30), false, s);
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return PIC_OK;
}

int pic_job_solve_field(pic_engine* E, int job, void* stream) {
  int rc = check_job(E, job);
  if (rc) return rc;
  CK(cudaSetDevice(E->device));
  JobHost& J = E->jobs[job];
  J.charge_fresh = true;
  if (!J.mg.valid) {
    rc = build_mg(E, std::vector<int>{job}, J.mg);
    if (rc) return rc;
  }
  cudaStream_t s = pick(E, stream);
  rc = solve(E, J.mg, nullptr, s);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s));
  return PIC_OK;
}

int pic_job_get_grid(pic_engine* E, int job, int which, double* out, int memory) {
  int rc = check_job(E, job);
  if (rc) return rc;
  if (which < 0 || which > 3 || !out) return fail(PIC_ERR_ARG, "bad grid selector");
  CK(cudaSetDevice(E->device));
  JobHost& J = E->jobs[job];
  const int64_t N = (int64_t)J.dev.nx * J.dev.ny;
  const double dxv = J.cfg.Lx / (J.cfg.nx - 1), dyv = J.cfg.Ly / (J.cfg.ny - 1);
  cudaStream_t s = E->stream;
  double* dst = out;
  if (memory == PIC_MEM_HOST) {
    rc = ensure_stage(E, N * 8);
    if (rc) return rc;
    dst = (double*)E->d_stage;
  }
  launch_grid_export(E->d_jobs + job, E->d_st + job, which, dst, J.dev.nx, J.dev.ny, dxv, dyv, s);
  if (memory == PIC_MEM_HOST) CK(cudaMemcpyAsync(out, dst, N * 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return PIC_OK;
}

int pic_job_set_grid(pic_engine* E, int job, int which, const double* in, int memory) {
  int rc = check_job(E, job);
  if (rc) return rc;
  if (which == PIC_GRID_RHO) E->jobs[job].charge_fresh = false;
  if ((which != PIC_GRID_RHO && which != PIC_GRID_PHI) || !in) return fail(PIC_ERR_ARG, "only RHO and PHI can be set");
  CK(cudaSetDevice(E->device));
  JobHost& J = E->jobs[job];
  const int64_t N = (int64_t)J.dev.nx * J.dev.ny;
  cudaStream_t s = E->stream;
  const double* src = in;
  if (memory == PIC_MEM_DEVICE) CK(cudaDeviceSynchronize());   // the caller's writes of `in`
  if (memory == PIC_MEM_HOST) {
    rc = ensure_stage(E, N * 8);
    if (rc) return rc;
    CK(cudaMemcpyAsync(E->d_stage, in, N * 8, cudaMemcpyHostToDevice, s));
    src = (const double*)E->d_stage;
  }
  launch_grid_import(E->d_jobs + job, E->d_st + job, which, src, J.dev.nx, J.dev.ny, s);
  // a phi written from outside has no history: the next warm start is phi itself
  if (which == PIC_GRID_PHI) CK(cudaMemsetAsync(&E->d_st[job].phi_prev1, 0, sizeof(int), s));
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return PIC_OK;
}

int pic_job_get_hits(pic_engine* E, int job, int species, int64_t capacity, int64_t* idx, int64_t* n_out) {
  int rc = check_job(E, job);
  if (rc) return rc;
  JobHost& J = E->jobs[job];
  if (species < 0 || species >= J.cfg.n_species) return fail(PIC_ERR_ARG, "bad species");
  CK(cudaSetDevice(E->device));
  CK(cudaStreamSynchronize(E->stream));
  int k = 0;
  CK(cudaMemcpy(&k, E->d_hits + job * kSlotsPerJob + species, sizeof(int), cudaMemcpyDeviceToHost));
  if (n_out) *n_out = k;
  if (k > capacity) return fail(PIC_ERR_CAPACITY, "output array too small");
  std::vector<int32_t> h(k);
  if (k) CK(cudaMemcpy(h.data(), J.slot[species].hits, sizeof(int32_t) * k, cudaMemcpyDeviceToHost));
  for (int i = 0; i < k; ++i) idx[i] = h[i];
  return PIC_OK;
}

// ---------------------------------------------------------------- tuning
int pic_engine_set_option(pic_engine* E, int option, int64_t value) {
  if (!E) return fail(PIC_ERR_ARG, "null engine");
  std::lock_guard<std::mutex> lk(E->mu);
  if (option == PIC_OPT_MG_LEVELS_KERNEL) {
    if (value != 0 && value != 1) return fail(PIC_ERR_ARG, "PIC_OPT_MG_LEVELS_KERNEL takes 0 or 1");
    E->levels_kernel = (int)value;
  } else if (option == PIC_OPT_MG_CLUSTER_TOP) {
    if (value < 0 || value > 16385) return fail(PIC_ERR_ARG, "PIC_OPT_MG_CLUSTER_TOP out of range");
    E->cluster_top = (int)value;
  } else if (option == PIC_OPT_MG_COARSE_TOP) {
    if (value < 3 || value > PIC_COARSE_MAX) return fail(PIC_ERR_ARG, "PIC_OPT_MG_COARSE_TOP out of range (3..129)");
    E->coarse_top = (int)value;
  } else if (option == PIC_OPT_MOVER_CTAS_PER_SM) {
    if (value < 0 || value > 32) return fail(PIC_ERR_ARG, "PIC_OPT_MOVER_CTAS_PER_SM out of range (0..32)");
    E->mover_cps = (int)value;
  } else if (option == PIC_OPT_MG_WIDE_TILES) {
    if (value < 0 || value > 64) return fail(PIC_ERR_ARG, "PIC_OPT_MG_WIDE_TILES out of range (0..64)");
    E->wide_factor = (int)value;
  } else {
    return fail(PIC_ERR_ARG, "unknown option");
  }
  // every multigrid plan (and the step graphs that replay them) is rebuilt on next use
  E->mg_dirty = true;
  E->graph_dirty = true;
  for (auto& J : E->jobs) J.mg.valid = false;
  return PIC_OK;
}

int pic_engine_get_option(pic_engine* E, int option, int64_t* value) {
  if (!E || !value) return fail(PIC_ERR_ARG, "null argument");
  if (option == PIC_OPT_MG_LEVELS_KERNEL) *value = E->levels_kernel;
  else if (option == PIC_OPT_MG_CLUSTER_TOP) *value = E->cluster_top;
  else if (option == PIC_OPT_MG_COARSE_TOP) *value = E->coarse_top;
  else if (option == PIC_OPT_MOVER_CTAS_PER_SM) *value = E->mover_cps;
  else if (option == PIC_OPT_MG_WIDE_TILES) *value = E->wide_factor;
  else return fail(PIC_ERR_ARG, "unknown option");
  return PIC_OK;
}

int pic_job_set_sort_every(pic_engine* E, int job, int sort_every) {
  int rc = check_job(E, job);
  if (rc) return rc;
  if (sort_every < 0) return fail(PIC_ERR_ARG, "sort_every must be >= 0");
  std::lock_guard<std::mutex> lk(E->mu);
  CK(cudaSetDevice(E->device));
  JobHost& J = E->jobs[job];
  J.cfg.sort_every = sort_every;
  J.dev.sort_every = sort_every;
  CK(cudaMemcpyAsync(&E->d_jobs[job].sort_every, &J.dev.sort_every, sizeof(int), cudaMemcpyHostToDevice, E->stream));
  CK(cudaStreamSynchronize(E->stream));
  E->graph_dirty = true;
  return PIC_OK;
}

// ---------------------------------------------------------------- stateless solver
namespace {
struct SolverCtx {
  int device, nx, ny, levels, nu_pre, nu_post, nu_coarse;
  pic_engine* E = nullptr;
  int job = -1;
};
std::mutex g_solver_mu;
std::vector<SolverCtx> g_solvers;
}  // namespace

int pic_solve_multigrid_f64(double* phi, const double* rho, int nx, int ny, int levels, double h, double omega,
                            int nu_pre, int nu_post, int nu_coarse, double tol, int max_cycles, void* stream,
                            int* cycles_out, double* relres_out) {
  if (!phi || !rho) return fail(PIC_ERR_ARG, "null grid pointers");
  if (!is_pow2p1(nx) || nx != ny) return fail(PIC_ERR_ARG, "grid must be square with 2^k+1 nodes per side");
  if (!(h > 0)) return fail(PIC_ERR_ARG, "h must be positive");
  // the limits of a job's solver configuration, checked on every call (a cached solver would
  // otherwise take an omega or cycle budget that a fresh one rejects)
  if (levels < 0 || levels > auto_levels(nx)) return fail(PIC_ERR_ARG, "levels out of range");
  if (nu_pre < 0 || nu_pre > 16 || nu_post < 0 || nu_post > 16 || nu_coarse < 0 || nu_coarse > 1000)
    return fail(PIC_ERR_ARG, "sweep counts out of range");
  if (!(omega > 0 && omega < 2)) return fail(PIC_ERR_ARG, "omega must be in (0, 2)");
  if (max_cycles < 1 || !(tol >= 0)) return fail(PIC_ERR_ARG, "max_cycles >= 1 and tol >= 0 required");
  int device = 0;
  CK(cudaGetDevice(&device));
  std::lock_guard<std::mutex> lk(g_solver_mu);
  SolverCtx* ctx = nullptr;
  for (auto& c : g_solvers)
    if (c.device == device && c.nx == nx && c.ny == ny && c.levels == levels && c.nu_pre == nu_pre &&
        c.nu_post == nu_post && c.nu_coarse == nu_coarse)
      ctx = &c;
  if (!ctx) {
    SolverCtx c{device, nx, ny, levels, nu_pre, nu_post, nu_coarse};
    int rc = pic_engine_create(device, 0, &c.E);
    if (rc) return rc;
    pic_job_config cfg{};
    cfg.nx = nx; cfg.ny = ny; cfg.Lx = h * (nx - 1); cfg.Ly = h * (ny - 1); cfg.dt = 1.0;
    cfg.units = PIC_UNITS_REF; cfg.n_species = 0;
    cfg.mg_levels = levels > 0 ? levels : 0;
    cfg.nu_pre = nu_pre; cfg.nu_post = nu_post; cfg.nu_coarse = nu_coarse;
    cfg.omega = omega; cfg.tol = tol; cfg.max_cycles = max_cycles;
    rc = pic_job_create(c.E, &cfg, &c.job);
    if (rc) { pic_engine_destroy(c.E); return rc; }
    g_solvers.push_back(c);
    ctx = &g_solvers.back();
  }
  pic_engine* E = ctx->E;
  JobHost& J = E->jobs[ctx->job];
  J.dev.deposit_mode = 2;
  J.dev.rho_d = rho;
  J.dev.rhs_scale = 1.0;
  J.dev.qref = 1.0;
  J.dev.h = h;
  J.dev.omega = (float)omega;
  J.dev.tol = tol;
  J.dev.max_cycles = max_cycles;
  // without a stream the solve runs on the solver's own stream, after all work issued so far
  // on the device (the caller's writes of phi and rho)
  if (!stream) CK(cudaDeviceSynchronize());
  cudaStream_t s = stream ? (cudaStream_t)stream : E->stream;
  CK(cudaMemcpyAsync(E->d_jobs + ctx->job, &J.dev, sizeof(JobDev), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(&E->d_st[ctx->job].phi_cur, 0, sizeof(int), s));
  const size_t bytes = (size_t)nx * ny * 8;
  CK(cudaMemcpyAsync(J.dev.phi64[0], phi, bytes, cudaMemcpyDeviceToDevice, s));
  if (J.mg.valid) J.mg.max_cycles = max_cycles;
  if (!J.mg.valid) {
    int rc = build_mg(E, std::vector<int>{ctx->job}, J.mg);
    if (rc) return rc;
  }
  int rc = solve(E, J.mg, nullptr, s);
  if (rc) return rc;
  JobState T;
  CK(cudaMemcpyAsync(&T, E->d_st + ctx->job, sizeof(JobState), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaMemcpyAsync(phi, J.dev.phi64[T.phi_cur], bytes, cudaMemcpyDeviceToDevice, s));
  CK(cudaStreamSynchronize(s));
  if (cycles_out) *cycles_out = T.cycles;
  if (relres_out) *relres_out = T.relres;
  if (T.converged != 1) return fail(PIC_ERR_NOT_CONVERGED, "multigrid stopped at max_cycles above tol");
  return PIC_OK;
}

int pic_efield_f64(const double* phi, double* E_xy, int nx, int ny, double dx, double dy, void* stream) {
  if (!phi || !E_xy || nx < 2 || ny < 2) return fail(PIC_ERR_ARG, "bad arguments");
  launch_efield_f64(phi, E_xy, nx, ny, dx, dy, (cudaStream_t)stream);
  CK(cudaGetLastError());
  return PIC_OK;
}

}  // extern "C"
