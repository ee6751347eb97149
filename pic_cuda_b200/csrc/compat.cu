// compat.cu — the reference's host surface (Grid2D, Particles2D, Boundaries2D,
// solve_multigrid, read_cross_section, elasticCollisions, updateSimulationCUDA) over the
// engine's C ABI, so that a program written against the reference's headers builds against
// include/compat/ and runs on the engine.
//
// updateSimulationCUDA keeps one engine job per Particles2D (rebuilt when the grid, dt,
// species table or walls change).  Every call imports the caller's AoS arrays (split by
// `type` into the engine's per-species SoA layout, particle id = index in the caller's
// arrays), runs the steps, and writes the survivors back in their original order
// (a stable partition), the removed indices into collided_indices, and rho/phi/E into the
// grid.  Units are the reference's (lap(phi) = sum of q over CIC weights, v += q/m E dt).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "common.cuh"
#include "compat/Multigrid.hpp"
#include "compat/boundaries.h"
#include "compat/diagnostics.h"
#include "compat/grid.cuh"
#include "compat/mcc.hpp"
#include "compat/particles.cuh"
#include "compat/pic_step.h"
#include "pic_b200.h"

namespace pic_compat {

[[noreturn]] static void raise(const std::string& what) { throw std::runtime_error("pic compat: " + what); }

static void cuda_ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) raise(std::string(what) + ": " + cudaGetErrorString(e));
}

static void pic_ok(int rc, const char* what) {
  if (rc != PIC_OK) raise(std::string(what) + ": " + pic_last_error());
}

template <class T>
static T* dalloc(size_t n) {
  void* p = nullptr;
  if (n == 0) n = 1;
  cuda_ok(cudaMalloc(&p, n * sizeof(T)), "cudaMalloc");
  cuda_ok(cudaMemset(p, 0, n * sizeof(T)), "cudaMemset");
  return static_cast<T*>(p);
}

// ------------------------------------------------------------------ stable partition
// Elements 0..n-1 fall into classes 0..C-1; the partition writes every element to
// dest = (elements of lower classes) + (elements of its class before it), i.e. a stable
// class-major order.  Three launches: per-block class counts, one-block scan, scatter.
constexpr int kPartBlock = 1024;
constexpr int kMaxClass = 8;

template <class F>
__global__ void __launch_bounds__(kPartBlock) class_count_kernel(F cls, int n, int C, int* counts) {
  __shared__ int cs[kMaxClass];
  if (threadIdx.x < C) cs[threadIdx.x] = 0;
  __syncthreads();
  const int i = blockIdx.x * kPartBlock + threadIdx.x;
  const int c = i < n ? cls(i) : -1;
  for (int k = 0; k < C; ++k) {
    const unsigned m = __ballot_sync(0xffffffffu, c == k);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(&cs[k], __popc(m));
  }
  __syncthreads();
  if (threadIdx.x < C) counts[blockIdx.x * C + threadIdx.x] = cs[threadIdx.x];
}

// counts[b*C + c] -> exclusive class-major offsets; totals[c] = elements of class c.
__global__ void __launch_bounds__(1024) class_scan_kernel(int* counts, int nb, int C, int* totals) {
  __shared__ int wsum[32];
  __shared__ int carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int c = 0; c < C; ++c) {
    const int before = carry;
    for (int base = 0; base < nb; base += 1024) {
      const int b = base + threadIdx.x;
      const int v = b < nb ? counts[b * C + c] : 0;
      int x = v;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) wsum[warp] = x;
      __syncthreads();
      if (warp == 0) {
        int w = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, w, o);
          if (lane >= o) w += y;
        }
        wsum[lane] = w;
      }
      __syncthreads();
      if (b < nb) counts[b * C + c] = carry + (warp ? wsum[warp - 1] : 0) + x - v;
      __syncthreads();
      if (threadIdx.x == 0) carry += wsum[31];
      __syncthreads();
    }
    if (threadIdx.x == 0) totals[c] = carry - before;
    __syncthreads();
  }
}

template <class F, class W>
__global__ void __launch_bounds__(kPartBlock) class_scatter_kernel(F cls, W write, int n, int C,
                                                                    const int* offsets) {
  __shared__ int wcnt[32][kMaxClass];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int i = blockIdx.x * kPartBlock + threadIdx.x;
  const int c = i < n ? cls(i) : -1;
  int prefix = 0;
  for (int k = 0; k < C; ++k) {
    const unsigned m = __ballot_sync(0xffffffffu, c == k);
    if (lane == 0) wcnt[warp][k] = __popc(m);
    if (c == k) prefix = __popc(m & ((1u << lane) - 1u));
  }
  __syncthreads();
  if (c < 0) return;
  int before = 0;
  for (int w = 0; w < warp; ++w) before += wcnt[w][c];
  write(i, c, offsets[blockIdx.x * C + c] + before + prefix);
}

// Scratch for one partition of up to `cap` elements.
struct Partition {
  int* counts = nullptr;  // [blocks * kMaxClass]
  int* totals = nullptr;  // [kMaxClass]
  int cap = 0;
  void reserve(int n) {
    if (n <= cap && counts) return;
    release();
    const int nb = (n + kPartBlock - 1) / kPartBlock;
    counts = dalloc<int>((size_t)nb * kMaxClass);
    totals = dalloc<int>(kMaxClass);
    cap = n;
  }
  void release() {
    if (counts) cudaFree(counts);
    if (totals) cudaFree(totals);
    counts = totals = nullptr;
    cap = 0;
  }
  // Runs the partition and returns the class totals on the host.
  template <class F, class W>
  std::vector<int> run(F cls, W write, int n, int C, cudaStream_t s) {
    if (C > kMaxClass) raise("too many classes");
    std::vector<int> tot(C, 0);
    if (n <= 0) return tot;
    reserve(n);
    const int nb = (n + kPartBlock - 1) / kPartBlock;
    class_count_kernel<<<nb, kPartBlock, 0, s>>>(cls, n, C, counts);
    class_scan_kernel<<<1, 1024, 0, s>>>(counts, nb, C, totals);
    class_scatter_kernel<<<nb, kPartBlock, 0, s>>>(cls, write, n, C, counts);
    cuda_ok(cudaGetLastError(), "partition launch");
    cuda_ok(cudaMemcpyAsync(tot.data(), totals, sizeof(int) * C, cudaMemcpyDeviceToHost, s), "partition totals");
    cuda_ok(cudaStreamSynchronize(s), "partition");
    return tot;
  }
};

// ------------------------------------------------------------------ import / export functors
struct TypeClass {  // species index, or S for a type outside [0, S)
  const int* type;
  int S;
  __device__ int operator()(int i) const {
    const int t = type[i];
    return (t >= 0 && t < S) ? t : S;
  }
};

struct ImportWrite {  // AoS (r, v) -> per-species SoA, particle id = caller index
  const double2* r;
  const double2* v;
  double *x, *y, *vx, *vy;
  uint32_t* pid;
  int S;
  __device__ void operator()(int i, int c, int d) const {
    if (c == S) return;
    const double2 p = r[i], u = v[i];
    x[d] = p.x;
    y[d] = p.y;
    vx[d] = u.x;
    vy[d] = u.y;
    pid[d] = (uint32_t)i;
  }
};

struct AliveClass {  // 0 = kept, 1 = removed
  const uint8_t* alive;
  __device__ int operator()(int i) const { return alive[i] ? 0 : 1; }
};

// Survivors back to the caller's arrays.  r_old = r - v_drift dt, with v_drift the velocity
// before the last kick: v - q/m E(r) dt, E gathered as updateParticleVelocities does
// (kernels.cu:71-131; no kick outside the grid).
struct ExportWrite {
  const double2 *tr, *tv;
  const int* tt;
  double2 *r, *r_old, *v;
  int* type;
  int* removed;
  int n_alive;
  const double2* E;
  const double *q, *m;
  double dx, dy, dt;
  int gm, gn;
  __device__ void operator()(int i, int c, int d) const {
    if (c == 1) {
      removed[d - n_alive] = i;
      return;
    }
    const double2 p = tr[i], u = tv[i];
    const int t = tt[i];
    r[d] = p;
    v[d] = u;
    type[d] = t;
    const double X = p.x / dx, Y = p.y / dy;
    const int x0 = (int)floor(X), y0 = (int)floor(Y);
    double2 ud = u;
    if (x0 >= 0 && x0 < gm - 1 && y0 >= 0 && y0 < gn - 1) {
      const double wx = X - x0, wy = Y - y0;
      const double w0 = (1.0 - wx) * (1.0 - wy), w1 = wx * (1.0 - wy), w2 = (1.0 - wx) * wy, w3 = wx * wy;
      const double2 e0 = E[y0 * gm + x0], e1 = E[y0 * gm + x0 + 1], e2 = E[(y0 + 1) * gm + x0],
                    e3 = E[(y0 + 1) * gm + x0 + 1];
      const double ex = w0 * e0.x + w1 * e1.x + w2 * e2.x + w3 * e3.x;
      const double ey = w0 * e0.y + w1 * e1.y + w2 * e2.y + w3 * e3.y;
      const double k = q[t] / m[t] * dt;
      ud.x -= k * ex;
      ud.y -= k * ey;
    }
    r_old[d] = make_double2(p.x - ud.x * dt, p.y - ud.y * dt);
  }
};

struct KeepWrite {  // removeCollidedParticles: survivors to the staging copies
  const double2 *r, *r_old, *v;
  const int* type;
  double2 *sr, *sr_old, *sv;
  int* stype;
  __device__ void operator()(int i, int c, int d) const {
    if (c != 0) return;
    sr[d] = r[i];
    sr_old[d] = r_old[i];
    sv[d] = v[i];
    stype[d] = type[i];
  }
};

__global__ void place_kernel(const double* x, const double* y, const double* vx, const double* vy,
                             const uint32_t* pid, int n, int s, int n0, double2* tr, double2* tv, int* tt,
                             uint8_t* alive, int* err) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t p = pid[k];
  if (p >= (uint32_t)n0) {
    atomicOr(err, 1);
    return;
  }
  tr[p] = make_double2(x[k], y[k]);
  tv[p] = make_double2(vx[k], vy[k]);
  tt[p] = s;
  alive[p] = 1;
}

__global__ void interleave_kernel(const double* a, const double* b, double2* out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_double2(a[i], b[i]);
}

__global__ void fill_u8_kernel(uint8_t* f, int n, uint8_t v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) f[i] = v;
}

__global__ void unmark_kernel(const int* idx, int k, int n, uint8_t* alive) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= k) return;
  const int i = idx[t];
  if (i >= 0 && i < n) alive[i] = 0;
}

// elasticCollisions (mcc.cu:114-150 with kernels.cu:196-262): speed and energy
// (E = 1/2 m |v|^2 * 6.25e18 eV), sigma(E) by linear interpolation clipped at the table
// ends, P = 1 - exp(-n sigma |v| dt), isotropic 2D redirection keeping |v|.  The two
// uniforms per particle come from Philox-4x32-10 with counter (index, call, 0, 0).
__device__ __forceinline__ double u01_53(uint32_t a, uint32_t b) {
  const uint64_t k = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);  // 53 random bits
  return ((double)k + 0.5) * 0x1.0p-53;
}

__global__ void elastic_kernel(double2* v, double* v_abs, double* energy, double* crs, const int* type,
                               const double* mass, int nspec, const double* xs_e, const double* xs_s, int xs_len,
                               double density, double dt, int n, uint64_t seed, uint32_t call, int* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int t = type[i];
  if (t < 0 || t >= nspec) {  // not a species of the table: left untouched and reported
    atomicOr(err, 1);
    return;
  }
  const double2 u = v[i];
  const double s2 = u.x * u.x + u.y * u.y;
  const double sp = sqrt(s2);
  const double E = 0.5 * mass[t] * s2 * 6.25e18;
  double sig;
  if (E <= xs_e[0]) {
    sig = xs_s[0];
  } else if (E >= xs_e[xs_len - 1]) {
    sig = xs_s[xs_len - 1];
  } else {
    int lo = 0, hi = xs_len - 1;  // xs_e[lo] < E < xs_e[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (E < xs_e[mid]) hi = mid;
      else lo = mid;
    }
    const double t = (E - xs_e[lo]) / (xs_e[lo + 1] - xs_e[lo]);
    sig = xs_s[lo] + t * (xs_s[lo + 1] - xs_s[lo]);
  }
  v_abs[i] = sp;
  energy[i] = E;
  crs[i] = sig;
  uint32_t c[4] = {(uint32_t)i, call, 0u, 0u};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double P = 1.0 - exp(-density * sig * sp * dt);
  if (u01_53(c[0], c[1]) < P) {
    double sn, cs;
    sincospi(2.0 * u01_53(c[2], c[3]), &sn, &cs);
    v[i] = make_double2(sp * cs, sp * sn);
  }
}

inline int blocks_for(int n, int t) { return (n + t - 1) / t; }

// ------------------------------------------------------------------ per-Particles2D state
struct State {
  int device = -1;
  cudaStream_t stream = nullptr;
  // engine job and what it was built for
  pic_engine* engine = nullptr;
  int job = -1;
  int gm = 0, gn = 0, nspec = 0;
  double gx = 0, gy = 0, dt = 0;
  std::vector<double> qm;     // q0, m0, q1, m1, ...
  std::vector<double> walls;  // x1, y1, x2, y2, ...
  // scratch sized for max_particles
  int cap = 0;
  double *x = nullptr, *y = nullptr, *vx = nullptr, *vy = nullptr;
  uint32_t* pid = nullptr;
  double2 *tr = nullptr, *tv = nullptr, *tr_old = nullptr;
  int* tt = nullptr;
  uint8_t* alive = nullptr;
  int* err = nullptr;
  int grid_cap = 0;
  double *ex = nullptr, *ey = nullptr;
  Partition part;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  uint32_t mcc_calls = 0;
  uint64_t seed = 0x243F6A8885A308D3ull;

  void drop_engine() {
    if (engine) pic_engine_destroy(engine);
    engine = nullptr;
    job = -1;
  }
  void reserve(int n) {
    if (n <= cap && x) return;
    free_particles();
    const size_t k = (size_t)(n > 0 ? n : 1);
    x = dalloc<double>(k);
    y = dalloc<double>(k);
    vx = dalloc<double>(k);
    vy = dalloc<double>(k);
    pid = dalloc<uint32_t>(k);
    tr = dalloc<double2>(k);
    tv = dalloc<double2>(k);
    tr_old = dalloc<double2>(k);
    tt = dalloc<int>(k);
    alive = dalloc<uint8_t>(k);
    cap = n;
  }
  void reserve_grid(int nodes) {
    if (nodes <= grid_cap && ex) return;
    if (ex) cudaFree(ex);
    if (ey) cudaFree(ey);
    ex = dalloc<double>(nodes);
    ey = dalloc<double>(nodes);
    grid_cap = nodes;
  }
  void free_particles() {
    for (void* p : {(void*)x, (void*)y, (void*)vx, (void*)vy, (void*)pid, (void*)tr, (void*)tv, (void*)tr_old,
                    (void*)tt, (void*)alive})
      if (p) cudaFree(p);
    x = y = vx = vy = nullptr;
    pid = nullptr;
    tr = tv = tr_old = nullptr;
    tt = nullptr;
    alive = nullptr;
    cap = 0;
  }
  ~State() {
    drop_engine();
    free_particles();
    if (ex) cudaFree(ex);
    if (ey) cudaFree(ey);
    if (err) cudaFree(err);
    part.release();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  }
};

static State& state_of(Particles2D& p, pic_compat::State*& slot) {
  if (!slot) {
    auto* s = new State();
    cuda_ok(cudaGetDevice(&s->device), "cudaGetDevice");
    // a blocking stream: it follows the legacy default stream, on which the reference's
    // host code and kernels (and so the caller's writes of its arrays) run
    cuda_ok(cudaStreamCreate(&s->stream), "cudaStreamCreate");
    cuda_ok(cudaEventCreate(&s->ev0), "cudaEventCreate");
    cuda_ok(cudaEventCreate(&s->ev1), "cudaEventCreate");
    s->err = dalloc<int>(1);
    slot = s;
  }
  (void)p;
  return *slot;
}

// The reference's field-solve settings (Multigrid.cu:573-642 with main.cu:113): 5 levels,
// omega 1.25, 3 pre / 3 post sweeps, 20 coarse sweeps, 1e-5 relative residual, 50 cycles.
constexpr int kRefLevels = 5, kRefNuPre = 3, kRefNuPost = 3, kRefNuCoarse = 20, kRefMaxCycles = 50;
constexpr double kRefOmega = 1.25, kRefTol = 1e-5;

static void ensure_job(State& S, int max_particles, const Grid2D& g, const Boundaries2D& b, double dt,
                       const std::vector<double>& qm, int nspec) {
  const bool same = S.engine && S.gm == g.m && S.gn == g.n && S.gx == g.x && S.gy == g.y && S.dt == dt &&
                    S.nspec == nspec && S.qm == qm && S.walls == b.walls && S.cap >= max_particles;
  if (same) return;
  S.drop_engine();
  if (nspec > PIC_MAX_SPECIES) raise("at most 4 species");
  if (b.wall_count > PIC_MAX_WALLS) raise("at most 64 walls");
  pic_job_config c{};
  c.nx = g.m;
  c.ny = g.n;
  c.Lx = g.x;
  c.Ly = g.y;
  c.dt = dt;
  c.units = PIC_UNITS_REF;
  c.n_species = nspec;
  for (int s = 0; s < nspec; ++s) {
    c.species[s].charge = qm[2 * s];
    c.species[s].mass = qm[2 * s + 1];
    c.species[s].weight = 1.0;
    c.species[s].capacity = max_particles;
  }
  c.mg_levels = kRefLevels;
  c.nu_pre = kRefNuPre;
  c.nu_post = kRefNuPost;
  c.nu_coarse = kRefNuCoarse;
  c.omega = kRefOmega;
  c.tol = kRefTol;
  c.max_cycles = kRefMaxCycles;
  c.wall_mode = b.wall_count > 0 ? PIC_WALLS_SEGMENTS : PIC_WALLS_NONE;
  c.n_walls = b.wall_count;
  for (int w = 0; w < b.wall_count; ++w)
    for (int k = 0; k < 4; ++k) c.walls[w][k] = b.walls[4 * w + k];
  c.deposit_mode = PIC_DEPOSIT_I64;
  c.sort_every = 8;
  c.mcc_mode = PIC_MCC_NONE;
  c.seed = S.seed;
  pic_ok(pic_engine_create(S.device, 0, &S.engine), "pic_engine_create");
  int rc = pic_job_create(S.engine, &c, &S.job);
  if (rc != PIC_OK) {
    const std::string msg = pic_last_error();
    S.drop_engine();
    raise("pic_job_create: " + msg);
  }
  S.gm = g.m;
  S.gn = g.n;
  S.gx = g.x;
  S.gy = g.y;
  S.dt = dt;
  S.nspec = nspec;
  S.qm = qm;
  S.walls = b.walls;
  S.reserve(max_particles);
}

}  // namespace pic_compat

using namespace pic_compat;

// ------------------------------------------------------------------ Grid2D
Grid2D::Grid2D(int M, int N, double X, double Y) : m(M), n(N), dx(X / (M - 1)), dy(Y / (N - 1)), x(X), y(Y) {
  if (M < 2 || N < 2) raise("grid needs at least 2 nodes per side");
  rho = dalloc<double>((size_t)m * n);
  phi = dalloc<double>((size_t)m * n);
  E = dalloc<double2>((size_t)m * n);
}

Grid2D::~Grid2D() {
  cudaFree(rho);
  cudaFree(phi);
  cudaFree(E);
}

void Grid2D::debugGrid() {
  std::vector<double> h((size_t)m * n);
  const char* names[2] = {"Grid density (rho):", "Grid potential (phi):"};
  const double* src[2] = {rho, phi};
  for (int k = 0; k < 2; ++k) {
    cuda_ok(cudaMemcpy(h.data(), src[k], h.size() * sizeof(double), cudaMemcpyDeviceToHost), "debugGrid");
    if (k) std::cout << "\n";
    std::cout << names[k] << "\n";
    for (int j = 0; j < n; ++j) {
      for (int i = 0; i < m; ++i) std::cout << h[(size_t)j * m + i] << " ";
      std::cout << "\n";
    }
  }
}

// ------------------------------------------------------------------ Boundaries2D
Boundaries2D::~Boundaries2D() {
  if (d_walls) cudaFree(d_walls);
  if (d_walls_int) cudaFree(d_walls_int);
}

void Boundaries2D::add_wall(double x1, double y1, double x2, double y2) {
  walls.insert(walls.end(), {x1, y1, x2, y2});
  wall_count += 1;
}

void Boundaries2D::compile_walls() {
  if (d_walls) cudaFree(d_walls);
  if (d_walls_int) cudaFree(d_walls_int);
  d_walls = dalloc<double4>(wall_count);
  d_walls_int = dalloc<int4>(wall_count);
  std::vector<int4> wi(wall_count);
  for (int i = 0; i < wall_count; ++i)
    wi[i] = make_int4((int)walls[4 * i], (int)walls[4 * i + 1], (int)walls[4 * i + 2], (int)walls[4 * i + 3]);
  if (wall_count) {
    cuda_ok(cudaMemcpy(d_walls, walls.data(), wall_count * sizeof(double4), cudaMemcpyHostToDevice), "walls");
    cuda_ok(cudaMemcpy(d_walls_int, wi.data(), wall_count * sizeof(int4), cudaMemcpyHostToDevice), "walls");
  }
}

// ------------------------------------------------------------------ Particles2D
Particles2D::Particles2D(const int num_particles) {
  if (num_particles < 0) raise("negative particle count");
  max_particles = num_particles;
  const size_t n = (size_t)num_particles;
  r = dalloc<double2>(n);
  r_old = dalloc<double2>(n);
  v = dalloc<double2>(n);
  v_abs = dalloc<double>(n);
  energy = dalloc<double>(n);
  crs = dalloc<double>(n);
  type = dalloc<int>(n);
  q = dalloc<double>(PIC_MAX_SPECIES);
  m = dalloc<double>(PIC_MAX_SPECIES);
  collided_indices = dalloc<int>(n);
  collision_counter = dalloc<int>(1);
  const double q0 = 0.1, m0 = 1.0;
  cuda_ok(cudaMemcpy(q, &q0, sizeof(double), cudaMemcpyHostToDevice), "species");
  cuda_ok(cudaMemcpy(m, &m0, sizeof(double), cudaMemcpyHostToDevice), "species");
}

Particles2D::~Particles2D() {
  delete state_;
  for (void* p : {(void*)r, (void*)r_old, (void*)v, (void*)v_abs, (void*)energy, (void*)crs, (void*)type,
                  (void*)q, (void*)m, (void*)collided_indices, (void*)collision_counter})
    cudaFree(p);
}

void Particles2D::add_species(double new_m, double new_q) {
  if (species_num >= PIC_MAX_SPECIES) raise("at most 4 species");
  cuda_ok(cudaMemcpy(q + species_num, &new_q, sizeof(double), cudaMemcpyHostToDevice), "add_species");
  cuda_ok(cudaMemcpy(m + species_num, &new_m, sizeof(double), cudaMemcpyHostToDevice), "add_species");
  species_num++;
}

void Particles2D::change_species(int species, double new_m, double new_q) {
  if (species < 0 || species >= species_num) raise("change_species: no such species");
  cuda_ok(cudaMemcpy(q + species, &new_q, sizeof(double), cudaMemcpyHostToDevice), "change_species");
  cuda_ok(cudaMemcpy(m + species, &new_m, sizeof(double), cudaMemcpyHostToDevice), "change_species");
}

void Particles2D::debugParticles(int num_to_print) {
  const int k = std::max(0, std::min(last_alive, num_to_print));
  std::vector<double2> hp(k), hv(k);
  if (k) {
    cuda_ok(cudaMemcpy(hp.data(), r, k * sizeof(double2), cudaMemcpyDeviceToHost), "debugParticles");
    cuda_ok(cudaMemcpy(hv.data(), v, k * sizeof(double2), cudaMemcpyDeviceToHost), "debugParticles");
  }
  std::cout << "Particle debug - first " << k << " particles:\n";
  for (int i = 0; i < k; ++i)
    std::cout << "P" << i << ": pos=(" << hp[i].x << "," << hp[i].y << ") vel=(" << hv[i].x << "," << hv[i].y
              << ")\n";
}

void Particles2D::removeCollidedParticles() {
  State& S = state_of(*this, state_);
  int k = 0;
  cuda_ok(cudaMemcpy(&k, collision_counter, sizeof(int), cudaMemcpyDeviceToHost), "collision_counter");
  const int n = last_alive;
  if (n > max_particles) raise("last_alive exceeds max_particles");
  if (k <= 0 || n <= 0) return;
  if (k > max_particles) raise("collision_counter exceeds max_particles");
  S.reserve(max_particles);
  cudaStream_t s = S.stream;
  fill_u8_kernel<<<blocks_for(n, 256), 256, 0, s>>>(S.alive, n, 1);
  unmark_kernel<<<blocks_for(k, 256), 256, 0, s>>>(collided_indices, k, n, S.alive);
  KeepWrite w{r, r_old, v, type, S.tr, S.tr_old, S.tv, S.tt};
  const std::vector<int> tot = S.part.run(AliveClass{S.alive}, w, n, 2, s);
  const int kept = tot[0];
  if (kept) {
    cuda_ok(cudaMemcpyAsync(r, S.tr, kept * sizeof(double2), cudaMemcpyDeviceToDevice, s), "remove");
    cuda_ok(cudaMemcpyAsync(r_old, S.tr_old, kept * sizeof(double2), cudaMemcpyDeviceToDevice, s), "remove");
    cuda_ok(cudaMemcpyAsync(v, S.tv, kept * sizeof(double2), cudaMemcpyDeviceToDevice, s), "remove");
    cuda_ok(cudaMemcpyAsync(type, S.tt, kept * sizeof(int), cudaMemcpyDeviceToDevice, s), "remove");
  }
  cuda_ok(cudaStreamSynchronize(s), "removeCollidedParticles");
  last_alive = kept;
}

// ------------------------------------------------------------------ solve_multigrid
void solve_multigrid(double* phi_d, double* rho_d, int nx, int ny, int levels, double h, double omega) {
  int cycles = 0;
  double relres = 0.0;
  const int rc = pic_solve_multigrid_f64(phi_d, rho_d, nx, ny, levels, h, omega, kRefNuPre, kRefNuPost,
                                         kRefNuCoarse, kRefTol, kRefMaxCycles, nullptr, &cycles, &relres);
  // like the reference, stopping at the cycle limit is not an error
  if (rc != PIC_OK && rc != PIC_ERR_NOT_CONVERGED) pic_ok(rc, "solve_multigrid");
}

// ------------------------------------------------------------------ MCC
std::pair<std::vector<double>, std::vector<double>> read_cross_section(const std::string& filename) {
  std::vector<double> energies, sigmas;
  std::ifstream in(filename);
  if (!in.is_open()) {
    std::cerr << "Error: cannot open cross-section file: " << filename << std::endl;
    return {energies, sigmas};
  }
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ls(line);
    double e, s;
    if (ls >> e >> s) {
      energies.push_back(e);
      sigmas.push_back(s);
    }
  }
  return {energies, sigmas};
}

void elasticCollisions(Particles2D& particles, double density, double dt, cross_sections& xs) {
  State& S = state_of(particles, particles.state_);
  const int n = particles.last_alive;
  if (n <= 0) return;
  if (!xs.energies || !xs.sigmas || xs.size < 1) raise("elasticCollisions: empty cross-section table");
  if (n > particles.max_particles) raise("last_alive exceeds max_particles");
  cuda_ok(cudaMemsetAsync(S.err, 0, sizeof(int), S.stream), "err");
  elastic_kernel<<<blocks_for(n, 256), 256, 0, S.stream>>>(particles.v, particles.v_abs, particles.energy,
                                                           particles.crs, particles.type, particles.m,
                                                           particles.species_count(), xs.energies, xs.sigmas,
                                                           xs.size, density, dt, n, S.seed, S.mcc_calls++, S.err);
  cuda_ok(cudaGetLastError(), "elasticCollisions launch");
  int herr = 0;
  cuda_ok(cudaMemcpyAsync(&herr, S.err, sizeof(int), cudaMemcpyDeviceToHost, S.stream), "err");
  cuda_ok(cudaStreamSynchronize(S.stream), "elasticCollisions");
  if (herr) raise("elasticCollisions: particle type outside the species table");
}

// ------------------------------------------------------------------ updateSimulationCUDA
void updateSimulationCUDA(Particles2D& particles, Grid2D& grid, Boundaries2D& boundaries, int& step, double dt,
                          int steps, SimulationTiming& timing) {
  (void)step;  // the reference takes the step counter by reference but does not advance it
  timing = SimulationTiming{};
  if (steps <= 0) return;
  State& S = state_of(particles, particles.state_);
  const int n0 = particles.last_alive;
  if (n0 < 0 || n0 > particles.max_particles) raise("last_alive outside [0, max_particles]");
  const int nspec = particles.species_count();
  std::vector<double> hq(nspec), hm(nspec), qm(2 * nspec);
  cuda_ok(cudaMemcpy(hq.data(), particles.q, nspec * sizeof(double), cudaMemcpyDeviceToHost), "species q");
  cuda_ok(cudaMemcpy(hm.data(), particles.m, nspec * sizeof(double), cudaMemcpyDeviceToHost), "species m");
  for (int s = 0; s < nspec; ++s) {
    qm[2 * s] = hq[s];
    qm[2 * s + 1] = hm[s];
  }
  ensure_job(S, particles.max_particles, grid, boundaries, dt, qm, nspec);
  cudaStream_t st = S.stream;
  const int nodes = grid.m * grid.n;
  S.reserve_grid(nodes);

  // caller arrays -> engine, grouped by species in caller order
  ImportWrite iw{particles.r, particles.v, S.x, S.y, S.vx, S.vy, S.pid, nspec};
  const std::vector<int> per = S.part.run(TypeClass{particles.type, nspec}, iw, n0, nspec + 1, st);
  if (n0 > 0 && per[nspec] != 0) raise("particle type outside the species table");
  int64_t off = 0;
  for (int s = 0; s < nspec; ++s) {
    const int ns = n0 > 0 ? per[s] : 0;
    pic_ok(pic_job_load_species(S.engine, S.job, s, ns, S.x + off, S.y + off, S.vx + off, S.vy + off, nullptr,
                                S.pid + off, PIC_MEM_DEVICE),
           "pic_job_load_species");
    off += ns;
  }
  // phi carries the Dirichlet boundary values and the warm start, as in the reference
  pic_ok(pic_job_set_grid(S.engine, S.job, PIC_GRID_PHI, grid.phi, PIC_MEM_DEVICE), "pic_job_set_grid");

  pic_ok(pic_engine_profile(S.engine, 1), "pic_engine_profile");
  pic_engine_stats junk{};
  pic_ok(pic_engine_get_stats(S.engine, &junk, 1), "pic_engine_get_stats");
  cuda_ok(cudaEventRecord(S.ev0, st), "cudaEventRecord");
  pic_ok(pic_step(S.engine, steps, st), "pic_step");
  cuda_ok(cudaEventRecord(S.ev1, st), "cudaEventRecord");
  cuda_ok(cudaStreamSynchronize(st), "updateSimulationCUDA");
  float total_ms = 0.f;
  cuda_ok(cudaEventElapsedTime(&total_ms, S.ev0, S.ev1), "cudaEventElapsedTime");
  pic_engine_stats es{};
  pic_ok(pic_engine_get_stats(S.engine, &es, 1), "pic_engine_get_stats");
  pic_ok(pic_engine_profile(S.engine, 0), "pic_engine_profile");
  // the fused particle pass does drift, wall test, deposit and kick in one kernel
  timing.coordinate_update_us = es.phase_ms[1] * 1e3;
  timing.particle_removal = es.phase_ms[2] * 1e3;
  timing.solver_us = es.phase_ms[3] * 1e3;
  timing.total_us = total_ms * 1e3;

  // engine -> grid
  pic_ok(pic_job_get_grid(S.engine, S.job, PIC_GRID_RHO, grid.rho, PIC_MEM_DEVICE), "rho");
  pic_ok(pic_job_get_grid(S.engine, S.job, PIC_GRID_PHI, grid.phi, PIC_MEM_DEVICE), "phi");
  pic_ok(pic_job_get_grid(S.engine, S.job, PIC_GRID_EX, S.ex, PIC_MEM_DEVICE), "Ex");
  pic_ok(pic_job_get_grid(S.engine, S.job, PIC_GRID_EY, S.ey, PIC_MEM_DEVICE), "Ey");
  interleave_kernel<<<blocks_for(nodes, 256), 256, 0, st>>>(S.ex, S.ey, grid.E, nodes);
  cuda_ok(cudaGetLastError(), "interleave launch");

  // engine -> caller arrays: survivors in caller order, removed indices ascending
  cuda_ok(cudaMemsetAsync(S.alive, 0, (size_t)(n0 > 0 ? n0 : 1), st), "alive");
  cuda_ok(cudaMemsetAsync(S.err, 0, sizeof(int), st), "err");
  cuda_ok(cudaStreamSynchronize(st), "updateSimulationCUDA");
  off = 0;
  for (int s = 0; s < nspec; ++s) {
    int64_t ns = 0;
    pic_ok(pic_job_export_species(S.engine, S.job, s, (int64_t)n0 - off, S.x + off, S.y + off, S.vx + off,
                                  S.vy + off, nullptr, S.pid + off, &ns, PIC_MEM_DEVICE),
           "pic_job_export_species");
    if (ns) place_kernel<<<blocks_for((int)ns, 256), 256, 0, st>>>(S.x + off, S.y + off, S.vx + off, S.vy + off,
                                                                   S.pid + off, (int)ns, s, n0, S.tr, S.tv, S.tt,
                                                                   S.alive, S.err);
    off += ns;
  }
  int herr = 0;
  cuda_ok(cudaMemcpyAsync(&herr, S.err, sizeof(int), cudaMemcpyDeviceToHost, st), "err");
  cuda_ok(cudaStreamSynchronize(st), "updateSimulationCUDA");
  if (herr) raise("engine returned a particle id outside the imported range");
  const int n_alive = (int)off;
  ExportWrite ew{S.tr,   S.tv,    S.tt,    particles.r, particles.r_old, particles.v, particles.type,
                 particles.collided_indices, n_alive, grid.E, particles.q, particles.m, grid.dx, grid.dy, dt,
                 grid.m, grid.n};
  S.part.run(AliveClass{S.alive}, ew, n0, 2, st);
  const int removed = n0 - n_alive;
  cuda_ok(cudaMemcpy(particles.collision_counter, &removed, sizeof(int), cudaMemcpyHostToDevice),
          "collision_counter");
  particles.last_alive = n_alive;
}
