// multigrid.cu — Poisson solve lap(phi) = F for every job of the engine at once.
//
// Algorithm = solve_multigrid / v_cycle of the reference (Multigrid.cu:539-642): red-black
// SOR smoothing (colour (i+j) odd first, phi = fma(w, (N+S+E+W - h^2 f)/4, (1-w) phi),
// Multigrid.cu:246-265), residual f - lap(phi) (:269-297), full weighting (:299-349),
// bilinear prolongation added to the finer level (:351-407), coarse guess zeroed every
// cycle (:556), relative residual ||r|| / ||F|| checked after every cycle (:614-631).
// Precision: the V-cycle runs in FP32 on the correction equation A e = r; the residual r,
// the update phi += e and the norms are FP64 (defect correction), so the FP64 relative
// residual can be driven to 1e-9 and below.
// Kernels (one launch covers all jobs through tile lists):
//   mg_init    level 0: r = F - A phi (FP64), ||r||^2, ||F||^2; r -> f0 (FP32); per-tile
//              partials, summed in a fixed order by mg_init_finish (one CTA per job)
//   mg_down    per level above the coarse one: nu_pre sweeps from e = 0 on a 16x16 tile of
//              coarse nodes (fine tile + halo 2*nu+2 in shared memory, every sweep done
//              locally: a node at distance d from the tile edge is exact for d half-sweeps),
//              then residual + full weighting straight from shared memory
//   mg_coarse  one CTA per job runs the whole V-cycle from <= 65x65 down in shared memory
//   (opt-in: levels up to 257^2 or 513^2 in one thread-block cluster, mg_cluster.cu)
//   mg_up      prolongation + nu_post sweeps on 32x32 tiles; on level 0 also the FP64
//              update phi += e, the new FP64 residual and the tile's partial norm;
//              mg_finish (one CTA per job) sums the partials in a fixed order
//              (deterministic), counts the cycle and decides convergence.  The generic
//              kernels (mixed smoothing counts) still let the last tile CTA of a job do it.
#include <algorithm>
#include "common.cuh"
#include "kernels.h"
#include "mg_tiles.h"
#include "tma.cuh"

namespace {

constexpr int kTI = 32;   // level-0 residual / update tile
constexpr int kTC = mgt::kTC;   // down-leg coarse tile
constexpr int kTU = mgt::kTU;   // up-leg fine tile

// The charge grid of a job, copied to registers (see mg_up_kernel).
struct RhoSrc {
  int mode;
  const float* f;
  const long long* i;
  const double* d;
  __device__ __forceinline__ double operator[](size_t idx) const {
    return mode == 0 ? (double)f[idx] : mode == 1 ? (double)i[idx] * 0x1p-40 : d[idx];
  }
};

__device__ double block_sum(double v) {
  __shared__ double ws[32];
  for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) ws[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += ws[k];
  return t;  // valid in thread 0
}

// Sum of n partials (stride `stride`, offset `off`) by the whole CTA in a fixed order:
// thread t adds entries t, t+B, t+2B, ... then a fixed tree combines the threads, so the
// result does not depend on scheduling.  Valid in thread 0.  The loads of a thread's entries
// are independent of its running sum, so eight of them are issued ahead of the adds (a 4097^2
// grid has 16.4k tile partials: 64 per thread, a chain of L2 round trips otherwise).
__device__ double ordered_sum(const double* p, int n, int stride, int off) {
  double s = 0.0;
#pragma unroll 8
  for (int k = threadIdx.x; k < n; k += blockDim.x) s += p[(size_t)k * stride + off];
  __shared__ double sh[1024];   // blockDim.x <= 1024, a power of two
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  return sh[0];
}

// Last CTA of a job's tiles in this launch?  (threadfence + ticket)
__device__ bool last_of_job(JobState& T, int nlocal) {
  __shared__ int last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const int t = atomicAdd(&T.ticket, 1);
    last = (t == nlocal - 1);
    if (last) T.ticket = 0;
  }
  __syncthreads();
  return last;
}

// ---------------------------------------------------------------- mg_init
// Level-0 defect of the initial guess on a 32 x 32 tile: the potential (and with the
// extrapolated warm start the previous solution) with a one-node halo and rho arrive in one
// batch of asynchronous copies; the guess is formed once per node in shared memory.  The
// same pass sums the deposited charge (deterministic per-tile partials, like the norms).
__global__ void __launch_bounds__(256) mg_init_kernel(const TileRef* __restrict__ tiles, const JobDev* __restrict__ jobs,
                                                      const JobState* __restrict__ st) {
  constexpr int PW = kTI + 2, NT = 256;
  constexpr int NP = (PW * PW + NT - 1) / NT;
  constexpr int NO = kTI * kTI / NT;
  __shared__ __align__(16) double G[PW * PW];    // guess with halo (the current potential first)
  __shared__ __align__(16) double Q[PW * PW];    // previous solution with halo (warm start 1)
  __shared__ __align__(16) double RH[kTI * kTI]; // rho of the owned nodes, raw
  const TileRef tr = tiles[blockIdx.x];
  const JobDev& J = jobs[tr.job];
  const JobState& T = st[tr.job];
  const int nx = J.nx, ny = J.ny;
  const int cur = T.phi_cur;
  const double* __restrict__ phi = J.phi64[cur];
  // warm_start 1: the initial guess 2 phi_{k-1} - phi_{k-2} goes to a third buffer (phi_{k-1}
  // is kept as the next step's history), the defect correction then alternates between that
  // buffer and the one phi_{k-2} held
  const bool xs = J.warm_start != 0;
  const int prev = T.phi_prev1 - 1;
  const bool hist = xs && prev >= 0;
  const int tgt = hist ? 3 - cur - prev : (cur + 1) % 3;
  const double* __restrict__ pp = hist ? J.phi64[prev] : phi;
  double* guess = xs ? J.phi64[tgt] : nullptr;
  float* const f0 = T.fsel ? J.f0b : J.f[0];
  const int pl0 = J.pl[0];
  const double a = hist ? 2.0 : 1.0, b = hist ? 1.0 : 0.0;
  const double inv_h2 = 1.0 / (J.h * J.h);
  const double rhs_scale = J.rhs_scale;
  const RhoSrc rho{J.deposit_mode, J.rho_f, J.rho_i, J.rho_d};
  double* const partials = J.partials;
  const double qref = J.qref;
  const int i0 = tr.ti * kTI, j0 = tr.tj * kTI;
  const int t = threadIdx.x;
#pragma unroll
  for (int u = 0; u < NP; ++u) {
    const int k = t + u * NT;
    if (k < PW * PW) {
      const int py = k / PW, px = k - py * PW;
      const int gx = i0 - 1 + px, gy = j0 - 1 + py;
      const bool in = (unsigned)gx < (unsigned)nx && (unsigned)gy < (unsigned)ny;
      const int g = in ? gy * nx + gx : 0;
      tma::cp_async8(G + k, phi + g, in);
      if (hist) tma::cp_async8(Q + k, pp + g, in);
    }
  }
#pragma unroll
  for (int u = 0; u < NO; ++u) {
    const int k = t + u * NT;
    const int gx = i0 + (k & 31), gy = j0 + (k >> 5);
    const bool in = gx < nx && gy < ny;
    const int g = in ? gy * nx + gx : 0;
    if (rho.mode == 0) tma::cp_async4(reinterpret_cast<float*>(RH) + k, rho.f + g, in);
    else if (rho.mode == 1) tma::cp_async8(RH + k, rho.i + g, in);
    else tma::cp_async8(RH + k, rho.d + g, in);
  }
  tma::cp_async_wait_all();
  __syncthreads();
  if (hist) {
#pragma unroll
    for (int u = 0; u < NP; ++u) {
      const int k = t + u * NT;
      if (k < PW * PW) G[k] = a * G[k] - b * Q[k];
    }
    __syncthreads();
  }
  double ar = 0.0, af = 0.0, aq = 0.0;
#pragma unroll
  for (int u = 0; u < NO; ++u) {
    const int k = t + u * NT;
    const int ox = k & 31, oy = k >> 5;
    const int i = i0 + ox, j = j0 + oy;
    if (i >= nx || j >= ny) continue;
    const int c = j * nx + i;
    const int q = (oy + 1) * PW + (ox + 1);
    const double rv = rho.mode == 0 ? (double)reinterpret_cast<const float*>(RH)[k]
                      : rho.mode == 1 ? (double)reinterpret_cast<const long long*>(RH)[k] * 0x1p-40 : RH[k];
    const double F = rhs_scale * rv;
    double r = 0.0;
    const double g0 = G[q];
    if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1) {
      const double gs = G[q - PW] + G[q + PW] + G[q - 1] + G[q + 1];
      const double lap = (gs - 4.0 * g0) * inv_h2;
      r = F - lap;
    }
    if (xs) guess[c] = g0;
    f0[j * pl0 + i] = (float)r;
    ar += r * r;
    af += F * F;
    aq += rv;
  }
  const double sr = block_sum(ar);
  const double sf = block_sum(af);
  const double sq = block_sum(aq);
  if (t == 0) {
    partials[2 * (tr.pbase + tr.local)] = sr;
    partials[2 * (tr.pbase + tr.local) + 1] = sf;
    partials[2 * tr.nlocal + tr.pbase + tr.local] = sq;   // deposited charge (third block)
  }
  // the job's norms and state follow in mg_init_finish_kernel
}

// After mg_init_kernel, one 1024-thread CTA per job: the tiles' partial norms and charge summed in a fixed
// order, the relative residual of the initial guess, the potential buffers the defect
// correction uses (with the warm start, the guess's buffer), and the job joins the running
// count.
__global__ void __launch_bounds__(1024) mg_init_finish_kernel(const int* __restrict__ job_list,
                                                             const JobDev* __restrict__ jobs,
                                                             JobState* __restrict__ st, int* running) {
  const int job = job_list[blockIdx.x];
  const JobDev& J = jobs[job];
  JobState& T = st[job];
  const int t0 = (J.nx + kTI - 1) / kTI;   // the tile list's t0 x t0 tiles (square grids)
  const int n = t0 * t0;
  const double r2 = ordered_sum(J.partials, n, 2, 0);
  const double f2 = ordered_sum(J.partials, n, 2, 1);
  const double q = ordered_sum(J.partials + 2 * n, n, 1, 0);
  if (threadIdx.x != 0) return;
  const int cur = T.phi_cur;
  const bool xs = J.warm_start != 0;
  const int prev = T.phi_prev1 - 1;
  const bool hist = xs && prev >= 0;
  T.rnorm2 = r2;
  T.fnorm2 = f2;
  T.total_charge = q * J.qref;
  T.relres = f2 > 0.0 ? sqrt(r2 / f2) : sqrt(r2);
  T.cycles = 0;
  T.converged = 0;
  if (xs) {
    T.phi_prev1 = cur + 1;
    T.phi_cur = hist ? 3 - cur - prev : (cur + 1) % 3;
    T.phi_nxt = hist ? prev : (cur + 2) % 3;
  } else {
    T.phi_nxt = cur ^ 1;
  }
  atomicAdd(running, 1);
}

// Thread groups a tile is processed by: a whole 256-thread CTA, or one 256-thread quarter of a
// 1024-thread CTA synchronised by its own hardware barrier (ids 1-4; 0 is __syncthreads).
struct BlockGroup {
  static constexpr int kSize = 256;
  __device__ __forceinline__ int rank() const { return threadIdx.x; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
};
struct QuarterGroup {
  static constexpr int kSize = 256;
  int q;
  __device__ __forceinline__ int rank() const { return threadIdx.x & 255; }
  __device__ __forceinline__ void sync() const { asm volatile("bar.sync %0, 256;" ::"r"(q + 1) : "memory"); }
};

// Red-black SOR half-sweeps on a W x W shared tile whose node (0,0) is grid node (gx0,gy0).
// Only grid-interior nodes that are not on the tile's outer ring are updated.  Rows are
// spread over warps and the nodes of one colour in a row over lanes, so no thread divides
// or skips nodes of the other colour.
template <class G>
__device__ __forceinline__ void tile_sweeps(const G& g, float* e, const float* f, int W, int gx0, int gy0, int n,
                                            float h2, float omega, int nu) {
  const float om1 = 1.f - omega;
  const int lane = g.rank() & 31, warp = g.rank() >> 5, nwarp = G::kSize >> 5;
  const int ly_lo = max(1, 1 - gy0), ly_hi = min(W - 2, n - 2 - gy0);   // rows to update
  const int lx_lo = max(1, 1 - gx0), lx_hi = min(W - 2, n - 2 - gx0);   // columns to update
  for (int it = 0; it < nu; ++it) {
    for (int colour = 1; colour >= 0; --colour) {
      for (int ly = ly_lo + warp; ly <= ly_hi; ly += nwarp) {
        // first lx >= lx_lo with (gx0 + lx + gy0 + ly) % 2 == colour
        const int lx0 = lx_lo + ((colour - gx0 - lx_lo - gy0 - ly) & 1);
        float* row = e + ly * W;
        const float* frow = f + ly * W;
        for (int lx = lx0 + 2 * lane; lx <= lx_hi; lx += 64) {
          const float s = row[lx + W] + row[lx - W] + row[lx + 1] + row[lx - 1];
          const float nv = 0.25f * (s - h2 * frow[lx]);
          row[lx] = fmaf(omega, nv, om1 * row[lx]);
        }
      }
      g.sync();
    }
  }
}

// ---------------------------------------------------------------- mg_down
// Pre-smoothing of one tile of level l (from a zero correction), its residual and the full
// weighting of it to level l + 1.
template <class G>
__device__ void down_tile(const G& g, const TileRef tr, const JobDev* __restrict__ jobs,
                          const JobState* __restrict__ st, int l, float* sm) {
  const JobDev& J = jobs[tr.job];
  if (st[tr.job].converged) return;
  const int nf = J.nl[l], nc = J.nl[l + 1], pf = J.pl[l], pc = J.pl[l + 1];
  const double hl = J.h * (double)(1 << l);
  const float h2 = (float)(hl * hl), inv_h2 = (float)(1.0 / (hl * hl));
  const int nu = J.nu_pre, H = 2 * nu;
  const int ic0 = tr.ti * kTC, jc0 = tr.tj * kTC;
  const int gx0 = 2 * ic0 - 2 - H, gy0 = 2 * jc0 - 2 - H;
  const int W = 2 * kTC + 3 + 2 * H;
  float* e = sm;
  float* f = sm + W * W;
  const float* fg = (l == 0 && st[tr.job].fsel) ? J.f0b : J.f[l];
  // parameters read before the first barrier (after it, reads through J would be reloaded)
  float* const eg = J.e[l];
  float* const fc = J.f[l + 1];
  const float omega = J.omega;
  const int lane = g.rank() & 31, warp = g.rank() >> 5;
#pragma unroll 4
  for (int ly = warp; ly < W; ly += 8) {
    const int gy = gy0 + ly;
    const bool rowin = gy >= 0 && gy < nf;
    for (int lx = lane; lx < W; lx += 32) {
      const int gx = gx0 + lx;
      f[ly * W + lx] = (rowin && gx >= 0 && gx < nf) ? __ldg(fg + (size_t)gy * pf + gx) : 0.f;
      e[ly * W + lx] = 0.f;
    }
  }
  g.sync();
  tile_sweeps(g, e, f, W, gx0, gy0, nf, h2, omega, nu);
  // owned fine nodes [2 ic0, 2 ic0 + 2 kTC)
  for (int oy = warp; oy < 2 * kTC; oy += 8) {
    const int gy = 2 * jc0 + oy;
    if (gy >= nf) break;
    const int gx = 2 * ic0 + lane;
    if (gx < nf) eg[(size_t)gy * pf + gx] = e[(gy - gy0) * W + (gx - gx0)];
  }
  // residual + full weighting to the owned coarse nodes
  for (int k = g.rank(); k < kTC * kTC; k += G::kSize) {
    const int ic = ic0 + k % kTC, jc = jc0 + k / kTC;
    if (ic >= nc || jc >= nc) continue;
    float v = 0.f;
    if (ic > 0 && ic < nc - 1 && jc > 0 && jc < nc - 1) {
      const int cx = 2 * ic - gx0, cy = 2 * jc - gy0;
      float r[3][3];
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          const int q = (cy + dy) * W + (cx + dx);
          const float lap = (e[q - W] + e[q + W] + e[q - 1] + e[q + 1] - 4.f * e[q]) * inv_h2;
          r[dy + 1][dx + 1] = f[q] - lap;
        }
      const float s = 4.f * r[1][1] + 2.f * r[1][0] + 2.f * r[1][2] + 2.f * r[0][1] + 2.f * r[2][1] +
                      r[0][0] + r[0][2] + r[2][0] + r[2][2];
      v = s * 0.0625f;
    }
    fc[(size_t)jc * pc + ic] = v;
  }
  g.sync();  // the tile's shared memory is free for the group's next tile
}

__global__ void __launch_bounds__(256) mg_down_kernel(const TileRef* __restrict__ tiles, const JobDev* __restrict__ jobs,
                                                      const JobState* __restrict__ st, int l) {
  extern __shared__ __align__(16) float sm[];
  down_tile(BlockGroup{}, tiles[blockIdx.x], jobs, st, l, sm);
}

// Bilinear prolongation weights (Multigrid.cu:378-404) without a branch per parity: the
// absent neighbours enter as +0 and the scale is 1, 1/2 or 1/4, which reproduces
// c00, (c00 + c10)/2, (c00 + c01)/2 and (c00 + c10 + c01 + c11)/4 exactly.
__device__ __forceinline__ float prolong_value(const float* cp, int pitch, bool io, bool jo) {
  const float c00 = cp[0];
  const float c10 = io ? cp[1] : 0.f;
  const float c01 = jo ? cp[pitch] : 0.f;
  const float c11 = (io && jo) ? cp[pitch + 1] : 0.f;
  const float sc = io ? (jo ? 0.25f : 0.5f) : (jo ? 0.5f : 1.f);
  return sc * (c00 + c10 + c01 + c11);
}

// ---------------------------------------------------------------- mg_coarse
// Levels lc .. L-1 of one job in the shared memory of one 1024-thread CTA.  Level l occupies
// E then F, n_l rows of pitch n_l + 1 (even).  Every red-black half-sweep, restriction and
// prolongation maps thread t to a column and a row group (col_map: groups of the power of two
// at or above the n-2 interior columns) and walks the group's rows k G apart, so the lanes of
// a warp touch consecutive columns: with an even pitch the two colours of a column pair fall
// into distinct banks, and no lane idles on the other colour.  Every level uses the whole CTA
// (levels up to 17^2 the first 128 threads): the small levels are a chain of
// barrier-separated phases whose length is one node's latency when each thread has at most
// one node (measured on B200: one warp walking 17^2 .. 3^2 alone took 12 of the solve's 29 us).
constexpr int kCoarseThreads = 1024;

// Per-level constants of the coarse solve, computed once per launch (the FP64 divisions stay
// off the barrier chain).
struct CoarseLevel {
  int off;       // first float of E in the shared layout (F follows at off + n (n + 1))
  int n;         // side
  float h2;      // h_l^2
  float ih2;     // 1 / h_l^2
};

// Thread t of T on m interior columns: row groups of 2^s >= m threads (the smallest such
// power of two), column 1 + t % 2^s, group t / 2^s of G = T / 2^s; lanes past the m columns
// idle (group G).  With a power-of-two group width a warp holds whole groups or a part of one,
// so the lanes of a half-sweep fall in distinct banks; groups of exactly m threads put lanes of
// neighbouring groups, two rows apart, in the same banks (65^2: 940 shared-memory wavefronts
// per half-sweep set against 640; 33^2: 310 against 160).
struct ColMap {
  int col, g, G;
};
__device__ __forceinline__ ColMap col_map(int t, int T, int m) {
  ColMap c;
  if (m <= 0) { c.col = 1; c.g = 1; c.G = 0; return c; }
  const int sh = m > 1 ? 32 - __clz(m - 1) : 0;
  c.G = T >> sh;
  c.g = t >> sh;
  c.col = 1 + (t & ((1 << sh) - 1));
  if (c.col > m) c.g = c.G;
  return c;
}

// Barrier of the threads working on a level: the whole CTA, or (SMALL) the first
// kCoarseSmallThreads threads on hardware barrier 1 while the rest wait further on.
constexpr int kCoarseSmallThreads = 128;
constexpr int kCoarseSmallSide = 17;   // levels this small run on kCoarseSmallThreads threads
template <bool SMALL>
__device__ __forceinline__ void level_sync() {
  if (SMALL) asm volatile("bar.sync 1, %0;" ::"n"(kCoarseSmallThreads) : "memory");
  else __syncthreads();
}

// nu red-black SOR sweeps (colour (i+j) odd first, Multigrid.cu:246-265) on the interior of
// level L (row pitch n + 1) by T threads.  ZERO: e enters as +0 everywhere (pre-smoothing),
// so the first half-sweep reads no neighbours.
template <bool SMALL, bool ZERO = false>
__device__ void level_sweeps(float* sm, const CoarseLevel& L, float omega, int nu, int t, int T) {
  const int n = L.n, P = n + 1;
  float* const e = sm + L.off;
  const float* const f = e + n * P;
  const float h2 = L.h2;
  const ColMap cm = col_map(t, T, n - 2);
  const int i = cm.col, g = cm.g, G = cm.G;
  const bool on = g < G;
  const float om1 = 1.f - omega;
  for (int it = 0; it < nu; ++it)
    for (int colour = 1; colour >= 0; --colour) {
      if (on) {
        if (ZERO && it == 0 && colour == 1) {
          for (int j = 1 + ((colour - i - 1) & 1) + 2 * g; j <= n - 2; j += 2 * G) {
            const float s = 0.f;
            const float nv = 0.25f * (s - h2 * f[j * P + i]);
            e[j * P + i] = fmaf(omega, nv, om1 * 0.f);
          }
        } else {
          for (int j = 1 + ((colour - i - 1) & 1) + 2 * g; j <= n - 2; j += 2 * G) {
            float* p = e + j * P + i;
            const float s = p[P] + p[-P] + p[1] + p[-1];
            const float nv = 0.25f * (s - h2 * f[j * P + i]);
            *p = fmaf(omega, nv, om1 * *p);
          }
        }
      }
      level_sync<SMALL>();
    }
}

// Residual of level A and its full weighting (Multigrid.cu:299-349) to the interior of the
// next level's right-hand side (its boundary stays 0).
template <bool SMALL>
__device__ void level_restrict(float* sm, const CoarseLevel& A, const CoarseLevel& B, int t, int T) {
  const int n = A.n, P = n + 1, nc = B.n, Pc = nc + 1;
  const float* const e = sm + A.off;
  const float* const f = e + n * P;
  float* const fn = sm + B.off + nc * Pc;
  const float inv_h2 = A.ih2;
  const ColMap cm = col_map(t, T, nc - 2);
  const int ic = cm.col, g = cm.g, G = cm.G;
  if (g < G)
    for (int jc = 1 + g; jc <= nc - 2; jc += G) {
      float r[3][3];
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          const int q = (2 * jc + dy) * P + (2 * ic + dx);
          const float lap = (e[q - P] + e[q + P] + e[q - 1] + e[q + 1] - 4.f * e[q]) * inv_h2;
          r[dy + 1][dx + 1] = f[q] - lap;
        }
      fn[jc * Pc + ic] = (4.f * r[1][1] + 2.f * r[1][0] + 2.f * r[1][2] + 2.f * r[0][1] + 2.f * r[2][1] + r[0][0] +
                          r[0][2] + r[2][0] + r[2][2]) * 0.0625f;
    }
  level_sync<SMALL>();
}

// Bilinear prolongation (Multigrid.cu:351-407) of level B's correction added to the interior
// of level A's.
template <bool SMALL>
__device__ void level_prolong(float* sm, const CoarseLevel& A, const CoarseLevel& B, int t, int T) {
  const int n = A.n, P = n + 1, Pc = B.n + 1;
  float* const e = sm + A.off;
  const float* const c = sm + B.off;
  const ColMap cm = col_map(t, T, n - 2);
  const int i = cm.col, g = cm.g, G = cm.G;
  if (g < G)
    for (int j = 1 + g; j <= n - 2; j += G)
      e[j * P + i] += prolong_value(c + (j >> 1) * Pc + (i >> 1), Pc, i & 1, j & 1);
  level_sync<SMALL>();
}

// Shared-memory bytes of levels lc .. levels-1 in the coarse solver's layout.
__host__ __device__ inline size_t coarse_layout_bytes(const int* nl, int lc, int levels) {
  size_t b = 0;
  for (int l = lc; l < levels; ++l) b += 2ull * nl[l] * (nl[l] + 1) * sizeof(float);
  return b;
}

// n*n values from global memory (pitch n) to a shared level (pitch n + 1), all threads, the
// loads of a batch issued before any store.  Row = floor((k + 0.5) / n) in FP32 is exact
// while n^2 < 2^21: k + 0.5 is representable, and the product's rounding error
// (< n 2^-22) stays below the fraction's distance from an integer (>= 0.5 / n).
constexpr int kCoarseBatch = 5;
__device__ __forceinline__ void coarse_load(float* dst, const float* __restrict__ src, int n, int pitch) {
  const int N = n * n, T = blockDim.x;
  const float inv_n = 1.f / (float)n;
  for (int k0 = 0; k0 < N; k0 += kCoarseBatch * T) {
    float v[kCoarseBatch];
#pragma unroll
    for (int u = 0; u < kCoarseBatch; ++u) {
      const int k = k0 + (int)threadIdx.x + u * T;
      const int j = (int)(((float)k + 0.5f) * inv_n);
      v[u] = k < N ? __ldg(src + j * pitch + (k - j * n)) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < kCoarseBatch; ++u) {
      const int k = k0 + (int)threadIdx.x + u * T;
      if (k < N) {
        const int j = (int)(((float)k + 0.5f) * inv_n);
        dst[j * (n + 1) + (k - j * n)] = v[u];
      }
    }
  }
}
__device__ __forceinline__ void coarse_store(float* __restrict__ dst, const float* src, int n, int pitch) {
  const int N = n * n;
  const float inv_n = 1.f / (float)n;
  for (int k = threadIdx.x; k < N; k += blockDim.x) {
    const int j = (int)(((float)k + 0.5f) * inv_n);
    dst[j * pitch + (k - j * n)] = src[j * (n + 1) + (k - j * n)];
  }
}

__device__ void coarse_solve(const int job, const JobDev* __restrict__ jobs, const JobState* __restrict__ st,
                             float* sm) {
  const JobDev& J = jobs[job];
  if (st[job].converged) return;
  // The job's parameters are read once, before the first barrier: a barrier also orders the
  // compiler's view of global memory, so fields read through J afterwards would be reloaded.
  const int lc = J.lc, L = J.levels;
  const double h = J.h;
  const float omega = J.omega;
  const int nu_pre = J.nu_pre, nu_post = J.nu_post, nu_coarse = J.nu_coarse;
  float* const e_top = J.e[lc];
  const int p_top = J.pl[lc];
  const float* const f_top = (lc == 0 && st[job].fsel) ? J.f0b : J.f[lc];
  __shared__ CoarseLevel lv[PIC_MAX_LEVELS];
  __shared__ int total;
  const int t = threadIdx.x, T = blockDim.x;
  if (t < PIC_MAX_LEVELS) {
    const int l = t;
    const int n = (l >= lc && l < L) ? J.nl[l] : 0;
    const double hl = h * (double)(1 << l);
    lv[l].n = n;
    lv[l].h2 = (float)(hl * hl);
    lv[l].ih2 = (float)(1.0 / (hl * hl));
  }
  __syncthreads();
  if (t == 0) {
    int o = 0;
    for (int l = lc; l < L; ++l) { lv[l].off = o; o += 2 * lv[l].n * (lv[l].n + 1); }
    total = o;
  }
  __syncthreads();
  // zero every level (corrections start at 0; coarse right-hand sides keep a zero boundary);
  // the layout is a multiple of 4 floats, 16-byte aligned
  for (int k = t; k < total / 4; k += T) reinterpret_cast<float4*>(sm)[k] = make_float4(0.f, 0.f, 0.f, 0.f);
  __syncthreads();
  tma::pdl_wait();
  coarse_load(sm + lv[lc].off + lv[lc].n * (lv[lc].n + 1), f_top, lv[lc].n, p_top);
  __syncthreads();
  int l = lc;
  for (; l < L - 1 && lv[l].n > kCoarseSmallSide; ++l) {
    level_sweeps<false, true>(sm, lv[l], omega, nu_pre, t, T);
    level_restrict<false>(sm, lv[l], lv[l + 1], t, T);
  }
  if (lv[l].n > kCoarseSmallSide) {  // a large coarsest level (l == L - 1)
    level_sweeps<false>(sm, lv[l], omega, nu_coarse, t, T);
  } else {
    // the small levels: a few nodes per phase, so few threads and a cheap barrier
    constexpr int TS = kCoarseSmallThreads;
    if (t < TS) {
      for (int k = l; k < L - 1; ++k) {
        level_sweeps<true, true>(sm, lv[k], omega, nu_pre, t, TS);
        level_restrict<true>(sm, lv[k], lv[k + 1], t, TS);
      }
      level_sweeps<true>(sm, lv[L - 1], omega, nu_coarse, t, TS);
      for (int k = L - 2; k >= l; --k) {
        level_prolong<true>(sm, lv[k], lv[k + 1], t, TS);
        level_sweeps<true>(sm, lv[k], omega, nu_post, t, TS);
      }
    }
    __syncthreads();
  }
  for (int k = l - 1; k >= lc; --k) {
    level_prolong<false>(sm, lv[k], lv[k + 1], t, T);
    level_sweeps<false>(sm, lv[k], omega, nu_post, t, T);
  }
  coarse_store(e_top, sm + lv[lc].off, lv[lc].n, p_top);
  __syncthreads();  // shared memory is free for the CTA's next job
}

__global__ void __launch_bounds__(kCoarseThreads) mg_coarse_kernel(const int* __restrict__ job_list,
                                                                   const JobDev* __restrict__ jobs,
                                                                   const JobState* __restrict__ st) {
  extern __shared__ __align__(16) float sm[];
  tma::pdl_trigger();
  coarse_solve(job_list[blockIdx.x], jobs, st, sm);
}

// ---------------------------------------------------------------- mg_up
// Up leg of one tile of level l >= 1: the bilinear prolongation of the coarser correction
// added to the pre-smoothed one, nu_post sweeps, the result to eu[l].
template <class G>
__device__ void up_tile(const G& g, const TileRef tr, const JobDev* __restrict__ jobs, const JobState* __restrict__ st,
                        int l, float* sm) {
  const JobDev& J = jobs[tr.job];
  if (st[tr.job].converged) return;
  const int nf = J.nl[l], pf = J.pl[l];
  const double hl = J.h * (double)(1 << l);
  const float h2 = (float)(hl * hl);
  const int nu = J.nu_post, H = 2 * nu;
  const int i0 = tr.ti * kTU, j0 = tr.tj * kTU;
  const int gx0 = i0 - H, gy0 = j0 - H;
  const int W = kTU + 2 * H;
  float* e = sm;
  float* f = sm + W * W;
  const float* eg = J.e[l];
  const float* fg = J.f[l];
  const int pc = J.pl[l + 1];
  const float* ec = l + 1 == J.lc ? J.e[l + 1] : J.eu[l + 1];
  const float omega = J.omega;
  float* const eo = J.eu[l];
  const int lane = g.rank() & 31, warp = g.rank() >> 5;
#pragma unroll 2
  for (int ly = warp; ly < W; ly += 8)
    for (int lx = lane; lx < W; lx += 32) {
      const int k = ly * W + lx;
      const int gx = gx0 + lx, gy = gy0 + ly;
      float ev = 0.f, fv = 0.f;
      if (gx >= 0 && gx < nf && gy >= 0 && gy < nf) {
        const size_t gi = (size_t)gy * pf + gx;
        ev = __ldg(eg + gi);
        fv = __ldg(fg + gi);
        const float* cp = ec + (size_t)(gy >> 1) * pc + (gx >> 1);
        const bool io = gx & 1, jo = gy & 1;
        const float c00 = __ldg(cp);
        const float c10 = io ? __ldg(cp + 1) : 0.f;
        const float c01 = jo ? __ldg(cp + pc) : 0.f;
        const float c11 = (io && jo) ? __ldg(cp + pc + 1) : 0.f;
        float v;
        if (!io && !jo) v = c00;
        else if (io && !jo) v = 0.5f * (c00 + c10);
        else if (!io && jo) v = 0.5f * (c00 + c01);
        else v = 0.25f * (c00 + c10 + c01 + c11);
        ev += v;
      }
      e[k] = ev;
      f[k] = fv;
    }
  g.sync();
  if (nu > 0) tile_sweeps(g, e, f, W, gx0, gy0, nf, h2, omega, nu);
  for (int oy = warp; oy < kTU; oy += 8) {
    const int gy = j0 + oy, gx = i0 + lane;
    if (gy < nf && gx < nf) eo[(size_t)gy * pf + gx] = e[(gy - gy0) * W + (gx - gx0)];
  }
  g.sync();  // the tile's shared memory is free for the group's next tile
}

// mode 0: prolong + smooth, write e_l.  mode 1: level 0, prolong + smooth + FP64 update.
// mode 2: level 0 update only (e_0 produced by the coarse kernel).
__global__ void __launch_bounds__(256) mg_up_kernel(const TileRef* __restrict__ tiles, const JobDev* __restrict__ jobs,
                                                    JobState* __restrict__ st, int l, int mode, int* running) {
  extern __shared__ __align__(16) float sm[];
  const TileRef tr = tiles[blockIdx.x];
  const JobDev& J = jobs[tr.job];
  JobState& T = st[tr.job];
  if (T.converged) return;
  const int nf = J.nl[l], pf = J.pl[l];
  const double hl = J.h * (double)(1 << l);
  const float h2 = (float)(hl * hl);
  const int nu = mode == 2 ? 0 : J.nu_post, H = 2 * nu, X = (l == 0) ? 1 : 0;
  const int i0 = tr.ti * kTU, j0 = tr.tj * kTU;
  const int gx0 = i0 - H - X, gy0 = j0 - H - X;
  const int W = kTU + 2 * H + 2 * X;
  float* e = sm;
  float* f = sm + W * W;
  const int fsel = T.fsel;
  const float* eg = J.e[l];
  const float* fg = (l == 0 && fsel) ? J.f0b : J.f[l];
  const bool prolong = mode != 2;
  const int pcs = prolong ? J.pl[l + 1] : 0;
  // the coarser correction: the coarse solver's output at lc, else the up kernel's of l + 1
  const float* ec = prolong ? (l + 1 == J.lc ? J.e[l + 1] : J.eu[l + 1]) : nullptr;
  // everything else the kernel needs from the job, read before the first barrier (after it,
  // reads through J and T would be reloaded from global memory)
  const float omega = J.omega;
  float* const eo = J.eu[l];
  const int cur = T.phi_cur, nxt = T.phi_nxt;
  const double* const pc = J.phi64[cur];
  double* const pn = J.phi64[nxt];
  const double inv_h2 = 1.0 / (J.h * J.h);
  const double rhs_scale = J.rhs_scale;
  const RhoSrc rho{J.deposit_mode, J.rho_f, J.rho_i, J.rho_d};
  float* const f0 = fsel ? J.f[0] : J.f0b;   // the new defect goes to the other buffer
  double* const partials = J.partials;
  const double tol = J.tol;
  const int max_cycles = J.max_cycles;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll 2
  for (int ly = warp; ly < W; ly += 8)
  for (int lx = lane; lx < W; lx += 32) {
    const int k = ly * W + lx;
    const int gx = gx0 + lx, gy = gy0 + ly;
    float ev = 0.f, fv = 0.f;
    if (gx >= 0 && gx < nf && gy >= 0 && gy < nf) {
      const size_t g = (size_t)gy * pf + gx;
      ev = __ldg(eg + g);
      fv = __ldg(fg + g);
      if (prolong) {
        // bilinear prolongation (Multigrid.cu:378-404) as weights on the 2x2 coarse block
        const float* cp = ec + (size_t)(gy >> 1) * pcs + (gx >> 1);
        const bool io = gx & 1, jo = gy & 1;
        const float c00 = __ldg(cp);
        const float c10 = io ? __ldg(cp + 1) : 0.f;
        const float c01 = jo ? __ldg(cp + pcs) : 0.f;
        const float c11 = (io && jo) ? __ldg(cp + pcs + 1) : 0.f;
        float v;
        if (!io && !jo) v = c00;
        else if (io && !jo) v = 0.5f * (c00 + c10);
        else if (!io && jo) v = 0.5f * (c00 + c01);
        else v = 0.25f * (c00 + c10 + c01 + c11);
        ev += v;
      }
    }
    e[k] = ev;
    f[k] = fv;
  }
  __syncthreads();
  if (nu > 0) tile_sweeps(BlockGroup{}, e, f, W, gx0, gy0, nf, h2, omega, nu);
  if (mode == 0) {
    for (int oy = warp; oy < kTU; oy += 8) {
      const int gy = j0 + oy, gx = i0 + lane;
      if (gy < nf && gx < nf) eo[(size_t)gy * pf + gx] = e[(gy - gy0) * W + (gx - gx0)];
    }
    return;
  }
  // ---- level-0 FP64 update and new residual
  __shared__ double P[(kTU + 2) * (kTU + 2)];
  constexpr int PW = kTU + 2;
  for (int py = warp; py < PW; py += 8)
    for (int px = lane; px < PW; px += 32) {
      const int gx = i0 - 1 + px, gy = j0 - 1 + py;
      double v = 0.0;
      if (gx >= 0 && gx < nf && gy >= 0 && gy < nf) v = __ldg(pc + (size_t)gy * nf + gx) + (double)e[(gy - gy0) * W + (gx - gx0)];
      P[py * PW + px] = v;
    }
  __syncthreads();
  double ar = 0.0;
  for (int oy = warp; oy < kTU; oy += 8) {
    const int ox = lane;
    const int gx = i0 + ox, gy = j0 + oy;
    if (gx >= nf || gy >= nf) continue;
    const size_t g = (size_t)gy * nf + gx;
    const int q = (oy + 1) * PW + (ox + 1);
    const double F = rhs_scale * rho[g];
    double r = 0.0;
    if (gx > 0 && gx < nf - 1 && gy > 0 && gy < nf - 1) {
      const double lap = (P[q - PW] + P[q + PW] + P[q - 1] + P[q + 1] - 4.0 * P[q]) * inv_h2;
      r = F - lap;
    }
    pn[g] = P[q];
    f0[(size_t)gy * pf + gx] = (float)r;
    ar += r * r;
  }
  const double sr = block_sum(ar);
  if (threadIdx.x == 0) partials[2 * (tr.pbase + tr.local)] = sr;
  if (last_of_job(T, tr.nlocal)) {
    __threadfence();
    const double r2 = ordered_sum(partials + 2 * tr.pbase, tr.nlocal, 2, 0);
    if (threadIdx.x != 0) return;
    T.rnorm2 = r2;
    T.relres = T.fnorm2 > 0.0 ? sqrt(r2 / T.fnorm2) : sqrt(r2);
    T.cycles += 1;
    T.phi_cur = nxt;
    T.phi_nxt = cur;
    T.fsel = fsel ^ 1;
    if (T.relres < tol) { T.converged = 1; atomicSub(running, 1); }
    else if (T.cycles >= max_cycles) { T.converged = 2; atomicSub(running, 1); }
  }
}

// ---------------------------------------------------------------- tile kernels, compile-time shapes
// The per-level launches of the V-cycle for a uniform smoothing count NU (0..4): the tile
// width W is a compile-time constant, so every global input of a tile is requested in one
// unrolled batch of asynchronous copies (one memory latency per tile instead of one per row),
// and the sweeps use the column-per-thread red-black mapping of the coarse solver on an even
// row pitch P (conflict-free, every lane on a node of the current colour).  NT threads per
// CTA: 256 where a level has enough tiles to fill the GPU, 1024 on small levels, where a
// tile's latency chain (not the SM's issue rate) sets the time.  Results equal those of
// mg_down_kernel / mg_up_kernel: the same expressions in the same order at every node.
constexpr int kMaxFastNu = 4;

// NU red-black SOR sweeps on a W x W tile.  ZERO: the correction enters as 0 (pre-smoothing
// from a zero guess), so the first half-sweep reads no neighbours (they are all +0).
// MG threads make one row group (MG >= W - 2, the interior columns of a tile; the extra
// threads of a group idle): with the tile pitch P chosen for it (mg_tiles.h), the lanes of a
// warp that straddles two groups then fall into distinct banks.  Boundary tiles, with fewer
// interior columns, leave more threads of each group idle.
template <int W, int P, int NU, int NT, bool ZERO, int MG = W - 2>
__device__ __forceinline__ void tile_sweeps_cols(float* e, const float* f, int gx0, int gy0, int n, float h2,
                                                 float omega) {
  static_assert(MG >= W - 2 && MG <= NT, "row group width");
  constexpr int G = NT / MG;                                    // row groups
  constexpr int kRows = ((W - 1) / 2 + G - 1) / G;              // rows of one colour per thread, at most
  const int t = threadIdx.x;
  const int lx_lo = max(1, 1 - gx0), lx_hi = min(W - 2, n - 2 - gx0);
  const int ly_lo = max(1, 1 - gy0), ly_hi = min(W - 2, n - 2 - gy0);
  const int m = lx_hi - lx_lo + 1;
  const int c = t % MG, g = t / MG;
  const int lx = lx_lo + c;
  const bool on = g < G && c < m && ly_hi >= ly_lo;
  const int par = gx0 + gy0 + lx;  // node (lx, ly) has colour (par + ly) & 1
  const float om1 = 1.f - omega;
#pragma unroll
  for (int it = 0; it < NU; ++it)
#pragma unroll
    for (int colour = 1; colour >= 0; --colour) {
      if (on) {
        const int ly0 = ly_lo + ((colour - par - ly_lo) & 1) + 2 * g;
#pragma unroll
        for (int r = 0; r < kRows; ++r) {
          const int ly = ly0 + 2 * G * r;
          if (ly <= ly_hi) {
            float* p = e + ly * P + lx;
            if (ZERO && it == 0 && colour == 1) {
              const float s = 0.f;
              const float nv = 0.25f * (s - h2 * f[ly * P + lx]);
              *p = fmaf(omega, nv, om1 * 0.f);
            } else {
              const float s = p[P] + p[-P] + p[1] + p[-1];
              const float nv = 0.25f * (s - h2 * f[ly * P + lx]);
              *p = fmaf(omega, nv, om1 * *p);
            }
          }
        }
      }
      __syncthreads();
    }
}

// The tile loads of a fast kernel: thread 0 arms the CTA's mbarrier with the bytes of every
// box and issues the tensor-map loads; every thread then waits for the phase (bounded).  A
// wait that runs out flags PIC_ST_TIMEOUT on the job, waits once more for the copies in
// flight and reports false, and the CTA leaves.
__device__ __forceinline__ bool tiles_arrived(uint64_t* mbar, JobState* T) {
  const bool ok = __syncthreads_and(tma::mbar_wait(mbar, 0) ? 1 : 0) != 0;
  if (!ok) {
    if (threadIdx.x == 0) atomicOr(&T->status, PIC_ST_TIMEOUT);
    tma::mbar_wait(mbar, 0);
  }
  return ok;
}

// Down leg of level l (as mg_down_kernel): NU pre-sweeps from a zero correction on the tile
// of 16 x 16 coarse nodes, the smoothed fine nodes it owns to e_l, the full-weighted
// residual to f_{l+1}.  The right-hand side tile arrives by one tensor-map load.
template <int NU, int NT>
__global__ void __launch_bounds__(NT) mg_down_fast_kernel(const TileRef* __restrict__ tiles,
                                                          const JobDev* __restrict__ jobs,
                                                          const JobState* __restrict__ st, int l) {
  constexpr int H = 2 * NU, W = mgt::down_w(NU), OFF = mgt::down_off(NU), P = mgt::down_bw(NU);
  static_assert(W == 2 * kTC + 3 + 2 * H, "tile shape");
  __shared__ __align__(128) float es[W * P];
  __shared__ __align__(128) float fs[W * P];
  __shared__ __align__(8) uint64_t mbar;
  float* const e = es + OFF;
  float* const f = fs + OFF;
  tma::pdl_trigger();
  // tile, job and job-state fields: none of them is written by the previous level's launch
  const TileRef tr = tiles[blockIdx.x];
  const JobDev& J = jobs[tr.job];
  const JobState& T = st[tr.job];
  if (T.converged) return;
  const int nf = J.nl[l], nc = J.nl[l + 1], pf = J.pl[l], pc = J.pl[l + 1];
  const double hl = J.h * (double)(1 << l);
  const float h2 = (float)(hl * hl), inv_h2 = (float)(1.0 / (hl * hl));
  const int ic0 = tr.ti * kTC, jc0 = tr.tj * kTC;
  const int gx0 = 2 * ic0 - 2 - H, gy0 = 2 * jc0 - 2 - H;
  const void* map = J.tmaps + mgt::kTmapsPerLevel * l + ((l == 0 && T.fsel) ? mgt::kMapDownF0b : mgt::kMapDownF);
  float* const eg = J.e[l];
  float* const fc = J.f[l + 1];
  const float omega = J.omega;
  const int t = threadIdx.x;
  if (t == 0) {
    tma::mbar_init(&mbar, 1);
    tma::fence_mbar_init();
  }
  for (int q = t; q < W * P; q += NT) es[q] = 0.f;
  __syncthreads();
  tma::pdl_wait();
  if (t == 0) {
    tma::mbar_arrive_expect_tx(&mbar, W * P * 4);
    tma::tensor_load_2d(fs, map, gx0 - OFF, gy0, &mbar);
  }
  if (!tiles_arrived(&mbar, const_cast<JobState*>(&T))) return;
  tile_sweeps_cols<W, P, NU, NT, true, mgt::down_group(NU)>(e, f, gx0, gy0, nf, h2, omega);
  // owned fine nodes [2 ic0, 2 ic0 + 2 kTC)
#pragma unroll
  for (int u = 0; u < (4 * kTC * kTC) / NT; ++u) {
    const int k = t + u * NT;
    const int gy = 2 * jc0 + (k >> 5), gx = 2 * ic0 + (k & 31);
    if (gy < nf && gx < nf) eg[gy * pf + gx] = e[(gy - gy0) * P + (gx - gx0)];
  }
  // residual + full weighting to the owned coarse nodes
  if (t < kTC * kTC) {
    const int ic = ic0 + (t & (kTC - 1)), jc = jc0 + t / kTC;
    if (ic < nc && jc < nc) {
      float vv = 0.f;
      if (ic > 0 && ic < nc - 1 && jc > 0 && jc < nc - 1) {
        const int cx = 2 * ic - gx0, cy = 2 * jc - gy0;
        float r[3][3];
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
          for (int dx = -1; dx <= 1; ++dx) {
            const int q = (cy + dy) * P + (cx + dx);
            const float lap = (e[q - P] + e[q + P] + e[q - 1] + e[q + 1] - 4.f * e[q]) * inv_h2;
            r[dy + 1][dx + 1] = f[q] - lap;
          }
        const float sum = 4.f * r[1][1] + 2.f * r[1][0] + 2.f * r[1][2] + 2.f * r[0][1] + 2.f * r[2][1] + r[0][0] +
                          r[0][2] + r[2][0] + r[2][2];
        vv = sum * 0.0625f;
      }
      fc[jc * pc + ic] = vv;
    }
  }
}

// Up leg (as mg_up_kernel modes 0 and 1).  MODE 0, level l >= 1: the bilinear prolongation
// of the coarser correction added to the pre-smoothed one, NU post-sweeps, the owned nodes
// to eu_l.  MODE 1, level 0 (NT = 256): the same with a one-node halo, then phi <- phi + e in
// FP64, the new FP64 defect and the deterministic norm.  The e, f and coarse tiles arrive by
// tensor-map loads; on level 0 phi64 (with a one-node halo) and rho of the owned nodes come
// in one batch of asynchronous copies beside them.
template <int NU, int MODE, int NT>
__global__ void __launch_bounds__(NT, MODE ? 5 : 1) mg_up_fast_kernel(const TileRef* __restrict__ tiles,
                                                                      const JobDev* __restrict__ jobs,
                                                                      JobState* __restrict__ st, int l) {
  constexpr int H = 2 * NU, X = MODE, W = mgt::up_w(NU, X), OFF = mgt::up_off(NU, X), P = mgt::up_bw(NU, X);
  constexpr int CW = mgt::up_cw(NU, X), COFF = mgt::up_coff(NU, X), CP = mgt::up_cbw(NU, X);
  static_assert(W == kTU + 2 * H + 2 * X, "tile shape");
  constexpr int PW = kTU + 2;
  constexpr int KC = (W + X + 1) / 2;              // coarse cells per tile row
  static_assert(KC + 1 <= CW, "coarse tile holds every cell's right and upper neighbour");
  constexpr int NP = MODE ? (PW * PW + NT - 1) / NT : 0;
  constexpr int NO = kTU * kTU / NT;
  __shared__ __align__(128) float es[W * P];
  __shared__ __align__(128) float fs[W * P];
  __shared__ __align__(128) float css[CW * CP];
  __shared__ __align__(16) double P64[MODE ? PW * PW : 1];
  __shared__ __align__(16) double RH[MODE ? kTU * kTU : 1];   // rho of the owned nodes, raw
  __shared__ __align__(8) uint64_t mbar;
  float* const e = es + OFF;
  float* const f = fs + OFF;
  const float* const cs = css + COFF;
  tma::pdl_trigger();
  // tile, job and job-state fields: the state changes only in mg_finish_kernel, at the end of
  // a V-cycle (the next V-cycle's first launch waits for it), so they are read before waiting
  // for the previous launch
  const TileRef tr = tiles[blockIdx.x];
  const JobDev& J = jobs[tr.job];
  JobState& T = st[tr.job];
  if (T.converged) return;
  const int nf = J.nl[l], pf = J.pl[l];
  const double hl = J.h * (double)(1 << l);
  const float h2 = (float)(hl * hl);
  const int i0 = tr.ti * kTU, j0 = tr.tj * kTU;
  const int gx0 = i0 - H - X, gy0 = j0 - H - X;
  const int cx0 = gx0 >> 1, cy0 = gy0 >> 1;   // floor, also for negative origins
  const int fsel = T.fsel;
  const CUtensorMap* maps = J.tmaps + mgt::kTmapsPerLevel * l;
  const void* map_e = maps + mgt::kMapUpE;
  const void* map_f = maps + ((l == 0 && fsel) ? mgt::kMapUpF0b : mgt::kMapUpF);
  const void* map_c = maps + mgt::kMapUpC;
  const float omega = J.omega;
  float* const eo = J.eu[l];
  const int cur = T.phi_cur, nxt = T.phi_nxt;
  const double* __restrict__ pc = J.phi64[cur];
  double* const pn = J.phi64[nxt];
  const double inv_h2 = 1.0 / (J.h * J.h);
  const double rhs_scale = J.rhs_scale;
  const RhoSrc rho{J.deposit_mode, J.rho_f, J.rho_i, J.rho_d};
  float* const f0 = fsel ? J.f[0] : J.f0b;   // the new defect goes to the other buffer
  double* const partials = J.partials;
  const int t = threadIdx.x;
  if (t == 0) {
    tma::mbar_init(&mbar, 1);
    tma::fence_mbar_init();
  }
  __syncthreads();
  tma::pdl_wait();
  // ---- the tiles: three tensor-map loads, and on level 0 one batch of asynchronous copies
  if (t == 0) {
    tma::mbar_arrive_expect_tx(&mbar, (2 * W * P + CW * CP) * 4);
    tma::tensor_load_2d(es, map_e, gx0 - OFF, gy0, &mbar);
    tma::tensor_load_2d(fs, map_f, gx0 - OFF, gy0, &mbar);
    tma::tensor_load_2d(css, map_c, cx0 - COFF, cy0, &mbar);
  }
  if constexpr (MODE == 1) {
#pragma unroll
    for (int u = 0; u < NP; ++u) {
      const int k = t + u * NT;
      if (k < PW * PW) {
        const int py = k / PW, px = k - py * PW;
        const int gx = i0 - 1 + px, gy = j0 - 1 + py;
        const bool in = (unsigned)gx < (unsigned)nf && (unsigned)gy < (unsigned)nf;
        tma::cp_async8(P64 + k, pc + (in ? gy * nf + gx : 0), in);
      }
    }
#pragma unroll
    for (int u = 0; u < NO; ++u) {
      const int k = t + u * NT;
      const int gx = i0 + (k & 31), gy = j0 + (k >> 5);
      const bool in = gx < nf && gy < nf;
      const int g = in ? gy * nf + gx : 0;
      if (rho.mode == 0) tma::cp_async4(reinterpret_cast<float*>(RH) + k, rho.f + g, in);
      else if (rho.mode == 1) tma::cp_async8(RH + k, rho.i + g, in);
      else tma::cp_async8(RH + k, rho.d + g, in);
    }
    tma::cp_async_wait_all();
  }
  if (!tiles_arrived(&mbar, &T)) return;
  // ---- bilinear prolongation added to the pre-smoothed correction: per thread and pass one
  // tile column lx and one row ky of coarse cells, i.e. the column's two fine nodes in tile rows
  // 2 ky - X and 2 ky + 1 - X (gx0 and gy0 have the parity X), with prolong_value's expressions;
  // the lanes of a warp sit on consecutive columns, so their updates of e meet no bank conflict
  // (a 2 x 2 block of fine nodes per thread put the lanes two columns apart).
  constexpr int NPR = (W * KC + NT - 1) / NT;
#pragma unroll
  for (int u = 0; u < NPR; ++u) {
    const int q = t + u * NT;
    if (q < W * KC) {
      const int ky = q / W, lx = q - ky * W;
      const int gx = gx0 + lx, kx = (lx + X) >> 1;
      const bool io = ((lx + X) & 1) != 0;
      const int ly = 2 * ky - X, gy = gy0 + ly;
      const float* cp = cs + ky * CP + kx;
      if ((unsigned)gx < (unsigned)nf) {
        if (ly >= 0 && (unsigned)gy < (unsigned)nf) e[ly * P + lx] += prolong_value(cp, CP, io, false);
        if (ly + 1 < W && (unsigned)(gy + 1) < (unsigned)nf) e[(ly + 1) * P + lx] += prolong_value(cp, CP, io, true);
      }
    }
  }
  __syncthreads();
  tile_sweeps_cols<W, P, NU, NT, false, mgt::up_group(NU, X)>(e, f, gx0, gy0, nf, h2, omega);
  if constexpr (MODE == 0) {
#pragma unroll
    for (int u = 0; u < NO; ++u) {
      const int k = t + u * NT;
      const int gx = i0 + (k & 31), gy = j0 + (k >> 5);
      if (gy < nf && gx < nf) eo[gy * pf + gx] = e[(gy - gy0) * P + (gx - gx0)];
    }
    return;
  } else {
    // ---- level-0 FP64 update and new residual
#pragma unroll
    for (int u = 0; u < NP; ++u) {
      const int k = t + u * NT;
      if (k < PW * PW) {
        const int py = k / PW, px = k - py * PW;
        const int gx = i0 - 1 + px, gy = j0 - 1 + py;
        if ((unsigned)gx < (unsigned)nf && (unsigned)gy < (unsigned)nf)
          P64[k] += (double)e[(gy - gy0) * P + (gx - gx0)];
      }
    }
    __syncthreads();
    double ar = 0.0;
#pragma unroll
    for (int u = 0; u < NO; ++u) {
      const int k = t + u * NT;
      const int ox = k & 31, oy = k >> 5;
      const int gx = i0 + ox, gy = j0 + oy;
      if (gx >= nf || gy >= nf) continue;
      const int g = gy * nf + gx;
      const int q = (oy + 1) * PW + (ox + 1);
      const double rv = rho.mode == 0 ? (double)reinterpret_cast<const float*>(RH)[k]
                        : rho.mode == 1 ? (double)reinterpret_cast<const long long*>(RH)[k] * 0x1p-40 : RH[k];
      const double F = rhs_scale * rv;
      double r = 0.0;
      if (gx > 0 && gx < nf - 1 && gy > 0 && gy < nf - 1) {
        const double lap = (P64[q - PW] + P64[q + PW] + P64[q - 1] + P64[q + 1] - 4.0 * P64[q]) * inv_h2;
        r = F - lap;
      }
      pn[g] = P64[q];
      f0[gy * pf + gx] = (float)r;
      ar += r * r;
    }
    // the tile's partial only: the job's norm, convergence test and buffer swap follow in
    // mg_finish_kernel, so no CTA waits for its stores or a shared ticket before it leaves
    const double sr = block_sum(ar);
    if (t == 0) partials[2 * (tr.pbase + tr.local)] = sr;
  }
}

// End of a V-cycle for the jobs whose level 0 ran in mg_up_fast_kernel<., 1, .>: one
// 1024-thread CTA per job sums the tiles' partial norms in a fixed order, counts the cycle,
// swaps the potential and defect buffers and takes a converged job out of the running count.  Launched after the
// level-0 up kernel (waits for it in tma::pdl_wait); the next V-cycle's first launch waits for
// this one.
__global__ void __launch_bounds__(1024) mg_finish_kernel(const int* __restrict__ job_list,
                                                        const JobDev* __restrict__ jobs,
                                                        JobState* __restrict__ st, int* running) {
  tma::pdl_trigger();
  tma::pdl_wait();
  const int job = job_list[blockIdx.x];
  const JobDev& J = jobs[job];
  JobState& T = st[job];
  if (T.converged) return;
  const int tu = (J.nl[0] + kTU - 1) / kTU;
  const double r2 = ordered_sum(J.partials, tu * tu, 2, 0);
  if (threadIdx.x != 0) return;
  T.rnorm2 = r2;
  T.relres = T.fnorm2 > 0.0 ? sqrt(r2 / T.fnorm2) : sqrt(r2);
  T.cycles += 1;
  const int cur = T.phi_cur;
  T.phi_cur = T.phi_nxt;
  T.phi_nxt = cur;
  T.fsel ^= 1;
  if (T.relres < J.tol) { T.converged = 1; atomicSub(running, 1); }
  else if (T.cycles >= J.max_cycles) { T.converged = 2; atomicSub(running, 1); }
}

// Launch with optional programmatic stream serialisation (the kernel may start while the
// previous launch in the stream finishes; it waits in tma::pdl_wait before reading its output).
template <typename... KArgs, typename... Args>
void launch_k(void (*k)(KArgs...), int grid, int block, size_t smem, bool pdl, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k, args...);
}
template <int NU>
void launch_down_fast(int grid, bool wide, bool pdl, const TileRef* tiles, const JobDev* jobs, const JobState* st,
                      int l, cudaStream_t s) {
  if (wide) launch_k(mg_down_fast_kernel<NU, 1024>, grid, 1024, 0, pdl, s, tiles, jobs, st, l);
  else launch_k(mg_down_fast_kernel<NU, 256>, grid, 256, 0, pdl, s, tiles, jobs, st, l);
}
template <int NU>
void launch_up_fast(int grid, bool wide, bool pdl, const TileRef* tiles, const JobDev* jobs, JobState* st, int l,
                    int mode, cudaStream_t s) {
  if (mode == 1) launch_k(mg_up_fast_kernel<NU, 1, 256>, grid, 256, 0, pdl, s, tiles, jobs, st, l);
  else if (wide) launch_k(mg_up_fast_kernel<NU, 0, 1024>, grid, 1024, 0, pdl, s, tiles, jobs, st, l);
  else launch_k(mg_up_fast_kernel<NU, 0, 256>, grid, 256, 0, pdl, s, tiles, jobs, st, l);
}
void down_fast(int nu, int grid, bool wide, bool pdl, const TileRef* tiles, const JobDev* jobs, const JobState* st,
               int l, cudaStream_t s) {
  switch (nu) {
    case 0: launch_down_fast<0>(grid, wide, pdl, tiles, jobs, st, l, s); break;
    case 1: launch_down_fast<1>(grid, wide, pdl, tiles, jobs, st, l, s); break;
    case 2: launch_down_fast<2>(grid, wide, pdl, tiles, jobs, st, l, s); break;
    case 3: launch_down_fast<3>(grid, wide, pdl, tiles, jobs, st, l, s); break;
    default: launch_down_fast<4>(grid, wide, pdl, tiles, jobs, st, l, s); break;
  }
}
void up_fast(int nu, int grid, bool wide, bool pdl, const TileRef* tiles, const JobDev* jobs, JobState* st, int l,
             int mode, cudaStream_t s) {
  switch (nu) {
    case 0: launch_up_fast<0>(grid, wide, pdl, tiles, jobs, st, l, mode, s); break;
    case 1: launch_up_fast<1>(grid, wide, pdl, tiles, jobs, st, l, mode, s); break;
    case 2: launch_up_fast<2>(grid, wide, pdl, tiles, jobs, st, l, mode, s); break;
    case 3: launch_up_fast<3>(grid, wide, pdl, tiles, jobs, st, l, mode, s); break;
    default: launch_up_fast<4>(grid, wide, pdl, tiles, jobs, st, l, mode, s); break;
  }
}

// ---------------------------------------------------------------- levels 1 .. lc in one launch
// Every level below the top, and the coarse solve, as phases of one cooperative launch of
// 1024-thread CTAs (one per SM): each 256-thread quarter of a CTA processes tiles like one
// CTA of mg_down_kernel / mg_up_kernel, a whole CTA does a job's coarse solve, and grid-wide
// barriers separate the levels.  Replaces 2 (lc - 1) + 1 launches whose cost at these small
// sizes is latency, not work.
constexpr unsigned kGridPolls = 1u << 22;

// Barrier k of a cooperative launch waits for the arrival counter (zeroed before the launch)
// to reach (k + 1) * gridDim.x.  Bounded: after kGridPolls polls the CTA gives up.
__device__ bool grid_barrier(unsigned* count, unsigned target) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(count, 1u);
    int ok = 1;
    for (unsigned polls = 0; *(volatile unsigned*)count < target; ++polls) {
      if (polls >= kGridPolls) {
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

__global__ void __launch_bounds__(1024, 1) mg_levels_kernel(const __grid_constant__ MgLevelsArgs a) {
  extern __shared__ __align__(16) float sm[];
  const QuarterGroup g{(int)(threadIdx.x >> 8)};
  float* qsm = sm + g.q * a.quarter_floats;
  const int slots = gridDim.x * 4, slot = blockIdx.x * 4 + g.q;
  unsigned target = 0;
  bool ok = true;
  for (int l = 1; ok && l < a.max_depth; ++l) {
    for (int t = slot; t < a.n_down[l]; t += slots) down_tile(g, a.down_tiles[l][t], a.jobs, a.st, l, qsm);
    target += gridDim.x;
    ok = grid_barrier(a.gbar, target);
  }
  if (ok)
    for (int k = blockIdx.x; k < a.n_coarse; k += gridDim.x) coarse_solve(a.coarse_jobs[k], a.jobs, a.st, sm);
  for (int l = a.max_depth - 1; ok && l >= 1; --l) {
    target += gridDim.x;
    ok = grid_barrier(a.gbar, target);
    if (ok)
      for (int t = slot; t < a.n_up[l]; t += slots) up_tile(g, a.up_tiles[l][t], a.jobs, a.st, l, qsm);
  }
  if (!ok && threadIdx.x == 0)
    for (int k = 0; k < a.n_coarse; ++k) atomicOr(&a.st[a.coarse_jobs[k]].status, PIC_ST_TIMEOUT);
}

size_t down_smem(int nu) { const int W = 2 * kTC + 3 + 4 * nu; return (size_t)2 * W * W * sizeof(float); }
size_t up_smem(int nu) { const int W = kTU + 4 * nu + 2; return (size_t)2 * W * W * sizeof(float); }

}  // namespace

size_t mg_coarse_smem(const int* nl, int lc, int levels) { return coarse_layout_bytes(nl, lc, levels); }

void mg_configure_coarse(size_t smem_bytes) {
  // the attribute only grows, so every launch list built so far stays launchable
  static size_t configured = 0;
  if (smem_bytes > configured) {
    cudaFuncSetAttribute(mg_coarse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
    configured = smem_bytes;
  }
  cudaFuncSetAttribute(mg_down_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)down_smem(16));
  cudaFuncSetAttribute(mg_up_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)up_smem(16));
}

int launch_mg_init(const EngineLaunch& L, const MgLaunch& M, cudaStream_t s) {
  cudaMemsetAsync(L.running, 0, sizeof(int), s);
  if (!M.n_init) return 0;
  mg_init_kernel<<<M.n_init, 256, 0, s>>>(M.init_tiles, L.jobs, L.st);
  mg_init_finish_kernel<<<M.n_init_jobs, 1024, 0, s>>>(M.init_jobs, L.jobs, L.st, L.running);
  return 2;
}


int mg_levels_configure(int num_sms, int nu_pre_max, int nu_post_max, size_t coarse_smem, size_t* smem,
                        size_t* quarter_floats) {
  const size_t q = std::max(down_smem(nu_pre_max), up_smem(nu_post_max));
  *quarter_floats = q / sizeof(float);
  *smem = std::max(4 * q, coarse_smem);
  int coop = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  if (!coop || *smem > 227 * 1024) return 0;
  if (cudaFuncSetAttribute(mg_levels_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, mg_levels_kernel, 1024, *smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return b >= 1 ? num_sms : 0;  // one CTA per SM
}

// Tile launches of one level: the compile-time-shape kernels when every job of the launch
// has the same smoothing count (<= kMaxFastNu), else the generic ones.
// 1024-thread CTAs where a level has at most wide_factor (default 2) tiles per SM.  pdl: the
// launch follows a
// kernel of the V-cycle that this one's prologue may overlap (programmatic serialisation).
static bool launch_down(const MgLaunch& M, int l, const EngineLaunch& L, bool pdl, cudaStream_t s) {
  if (M.fast_nu_pre >= 0 && M.fast_nu_pre <= kMaxFastNu) {
    down_fast(M.fast_nu_pre, M.n_down[l], M.n_down[l] <= M.wide_factor * L.num_sms, pdl && M.pdl, M.down_tiles[l],
              L.jobs, L.st,
              l, s);
    return true;
  }
  mg_down_kernel<<<M.n_down[l], 256, down_smem(M.nu_pre_max), s>>>(M.down_tiles[l], L.jobs, L.st, l);
  return false;
}
static bool launch_up(const MgLaunch& M, int l, const EngineLaunch& L, bool pdl, cudaStream_t s) {
  if (M.fast_nu_post >= 0 && M.fast_nu_post <= kMaxFastNu) {
    up_fast(M.fast_nu_post, M.n_up[l], M.n_up[l] <= M.wide_factor * L.num_sms, pdl && M.pdl, M.up_tiles[l], L.jobs,
            L.st, l, l == 0 ? 1 : 0, s);
    if (l == 0)
      launch_k(mg_finish_kernel, M.n_finish, 1024, 0, M.pdl != 0, s, M.finish_jobs, L.jobs, L.st, L.running);
    return true;
  }
  mg_up_kernel<<<M.n_up[l], 256, up_smem(M.nu_post_max), s>>>(M.up_tiles[l], L.jobs, L.st, l, l == 0 ? 1 : 0,
                                                              L.running);
  return false;
}

int launch_mg_vcycle(const EngineLaunch& L, const MgLaunch& M, cudaStream_t s) {
  int k = 0;
  if (M.levels_grid > 0 && M.max_depth >= 2 && !M.n_cluster) {
    if (M.n_down[0]) { launch_down(M, 0, L, false, s); ++k; }
    MgLevelsArgs a{};
    for (int l = 0; l < PIC_MAX_LEVELS; ++l) {
      a.down_tiles[l] = M.down_tiles[l]; a.n_down[l] = M.n_down[l];
      a.up_tiles[l] = M.up_tiles[l]; a.n_up[l] = M.n_up[l];
    }
    a.coarse_jobs = M.coarse_jobs; a.n_coarse = M.n_coarse;
    a.max_depth = M.max_depth;
    a.quarter_floats = M.levels_quarter_floats;
    a.jobs = L.jobs; a.st = L.st; a.gbar = L.gbar;
    cudaMemsetAsync(L.gbar, 0, sizeof(unsigned), s);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(M.levels_grid);
    cfg.blockDim = dim3(1024);
    cfg.dynamicSmemBytes = M.levels_smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, mg_levels_kernel, a);
    ++k;
    if (M.n_up[0]) k += launch_up(M, 0, L, false, s) ? 2 : 1;   // + mg_finish_kernel
    if (M.n_upd) { mg_up_kernel<<<M.n_upd, 256, up_smem(0), s>>>(M.upd_tiles, L.jobs, L.st, 0, 2, L.running); ++k; }
    return k;
  }
  // every launch after the first may overlap its predecessor when both are compile-time-shape
  // kernels (they wait for the predecessor's output in tma::pdl_wait)
  bool prev_fast = false;
  for (int l = 0; l < M.max_depth; ++l)
    if (M.n_down[l]) { prev_fast = launch_down(M, l, L, prev_fast, s); ++k; }
  if (M.n_coarse) {
    launch_k(mg_coarse_kernel, M.n_coarse, kCoarseThreads, M.coarse_smem, prev_fast && M.pdl, s, M.coarse_jobs,
             L.jobs, L.st);
    prev_fast = true;
    ++k;
  }
  if (M.n_cluster) { k += launch_mg_cluster(M.cluster_jobs, M.n_cluster, M.cluster_C, M.cluster_smem, L.jobs, L.st, s); prev_fast = false; }
  for (int l = M.max_depth - 1; l >= 0; --l)
    if (M.n_up[l]) { prev_fast = launch_up(M, l, L, prev_fast, s); k += (prev_fast && l == 0) ? 2 : 1; }
  if (M.n_upd) { mg_up_kernel<<<M.n_upd, 256, up_smem(0), s>>>(M.upd_tiles, L.jobs, L.st, 0, 2, L.running); ++k; }
  return k;
}

namespace {
// Body-end kernel of the V-cycle WHILE node: loop again while any job is still iterating,
// never more than max_iterations times per solve.
__global__ void vcycle_condition_kernel(cudaGraphConditionalHandle h, const int* running, int* iterations,
                                        int max_iterations, unsigned long long* total) {
  const int it = ++(*iterations);
  *total += 1ull;
  cudaGraphSetConditional(h, (*running > 0 && it < max_iterations) ? 1u : 0u);
}
}  // namespace

int launch_vcycle_condition(cudaGraphConditionalHandle h, const int* running, int* iterations, int max_iterations,
                            unsigned long long* total, cudaStream_t s) {
  vcycle_condition_kernel<<<1, 1, 0, s>>>(h, running, iterations, max_iterations, total);
  return 1;
}
