// mg_embedded.cu — embedded-boundary multigrid: lap(phi) = rhs on the FLUID nodes of a node
// mask, with interior electrodes (DIRICHLET nodes held at phi_bc) and excluded regions (SOLID
// nodes left as they are).  Algorithm of the reference's Multigrid_embedded.cu:1-190
// (Multigrid::vcycle, :159-188), FP64 like the reference:
//   pre-smoothing   nu_pre red-black Gauss-Seidel sweeps, colour (i+j) even first
//                   (smooth_redblack :15-33, with the intended colour test: the reference's
//                   `(i + j) & 1 != redblack` parses as (i + j) & (1 != redblack))
//   restriction     r = rhs - lap(phi)/h^2 on FLUID nodes (residual_kernel :35-55), full
//                   weighting onto FLUID coarse nodes (restrict_kernel :57-86); coarse mask =
//                   the fine node (2i, 2j)'s, or with PIC_EMB_COARSEN_ANY the rule the
//                   reference's comment at :73 states (any DIRICHLET fine node of the 3x3
//                   stencil makes the coarse node DIRICHLET; else any other non-FLUID one
//                   makes it SOLID)
//   coarse level    phi = 0 (:151), recursion; the coarsest level runs the pre-sweeps only
//   prolongation    FLUID fine nodes add coarse (i/2, j/2) (prolongate_add_kernel :88-104),
//                   or with PIC_EMB_PROLONG_BILINEAR the bilinear interpolant
//   post-smoothing  nu_post sweeps
// Level l has spacing h 2^l.  DIRICHLET nodes take phi_bc of their level; without a phi_bc
// array they keep the value phi holds (coarse levels start from phi = 0, so that is 0, what
// the reference's zeroed coarse phi_bc arrays give).
//
// Kernels of one V-cycle:
//   emb_down_kernel<NU>  pre-smoothing fused with the restriction: a 32 x 32 output tile with
//       a halo of 2 NU + 2 nodes (phi, node kinds and the right-hand side, DIRICHLET nodes'
//       phi_bc in the same slot, staged in shared memory with every load of a thread issued
//       at once); the NU sweeps run there (after k half-sweeps every node at least k nodes
//       inside the tile edge is exact); the smoothed output region is written back, and the
//       16 x 16 coarse nodes of the tile get the full-weighted residual of their nine fine
//       nodes (from shared memory), their kind, and phi = 0.  No residual array.
//   emb_smooth_kernel<NU, PRO>  the same tile scheme with a halo of 2 NU for the
//       post-smoothing: the coarse correction is prolongated while staging (PRO).  Tiles read
//       halos that neighbouring CTAs own, so results go to the level's other phi buffer.
//   emb_coarse_kernel  every level from the first one with at most 65 x 65 nodes down, in one
//       CTA's shared memory (one launch for the whole lower V-cycle).
//   emb_norm_kernel / emb_norm_final_kernel  ||r||^2 and ||rhs||^2 over the FLUID nodes in a
//       fixed order (per-CTA partials, then one CTA), for the convergence test.
// The shared tiles store each colour's nodes contiguously (struct Tile), so a red-black
// half-sweep reads its FP64 neighbours at unit stride.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <vector>
#include "common.cuh"
#include "kernels.h"

int pic_fail(int code, const char* msg);

namespace {

constexpr uint8_t kFluid = PIC_NODE_FLUID, kDir = PIC_NODE_DIRICHLET, kSolid = PIC_NODE_SOLID;
constexpr uint8_t kFixed = 255;            // grid boundary / outside the grid: never updated
constexpr int kTile = 32;
constexpr int kSmoothThreads = 256;
constexpr int kCoarseThreads = 512;
constexpr int kCoarseMaxNodes = 65 * 65;   // first level at or below this size: one-CTA solve
constexpr int kNormBlocks = 592;

// Coarse correction at fine node (gx, gy) (an interior node, so every coarse index used
// lies inside the coarse grid: gx <= nx - 2 gives (gx + 1) / 2 <= nxc - 1).
__device__ __forceinline__ double prolong_at(const double* __restrict__ c, int nxc, int gx, int gy, bool bilinear) {
  const int ic = gx >> 1, jc = gy >> 1;
  const size_t a = (size_t)jc * nxc + ic;
  if (!bilinear) return c[a];
  const bool io = gx & 1, jo = gy & 1;
  if (!io && !jo) return c[a];
  if (io && !jo) return 0.5 * (c[a] + c[a + 1]);
  if (!io && jo) return 0.5 * (c[a] + c[a + nxc]);
  return 0.25 * (c[a] + c[a + 1] + c[a + nxc] + c[a + nxc + 1]);
}

// Node kind as the smoother treats it: FLUID, DIRICHLET (value in the rhs slot) or SOLID.
__device__ __forceinline__ uint8_t smoother_kind(uint8_t m, bool has_bc) {
  if (m == kFluid) return kFluid;
  if (m == kDir && has_bc) return kDir;
  return kSolid;
}

// Shared-memory tile of W x W nodes (W even) whose node (0, 0) is grid node (x0, y0), with
// x0 + y0 even, so a node's colour is (tx + ty) & 1.  Each colour is stored on its own: node
// (tx, ty) sits at [colour][ty * W/2 + tx/2].  A red-black half-sweep then reads the other
// colour's neighbours at consecutive FP64 words across a warp (the interleaved layout reads
// them at a stride of two words, two-way bank conflicts), and the rows of one colour share
// the parity of tx, so W/E neighbours are at q - 1 + (tx & 1) and q + (tx & 1).
template <int W>
struct Tile {
  static constexpr int HW = W / 2;
  double p[2][HW * W];    // phi
  double rb[2][HW * W];   // rhs (FLUID), phi_bc (DIRICHLET with phi_bc), 0 otherwise
  uint8_t m[2][HW * W];   // the caller's node kinds; kFixed on the grid boundary and outside
  __device__ __forceinline__ static int at(int tx, int ty) { return ty * HW + (tx >> 1); }
  __device__ __forceinline__ static int colour(int tx, int ty) { return (tx + ty) & 1; }
  __device__ __forceinline__ double phi(int tx, int ty) const { return p[colour(tx, ty)][at(tx, ty)]; }
  __device__ __forceinline__ uint8_t kind(int tx, int ty) const { return m[colour(tx, ty)][at(tx, ty)]; }
  // residual_kernel's expression at an interior tile node: rhs - (S + N + W + E - 4 phi) / h^2
  __device__ __forceinline__ double residual(int tx, int ty, double h2i) const {
    const int c = colour(tx, ty), o = c ^ 1, i = at(tx, ty);
    if (m[c][i] != kFluid) return 0.0;
    const int w = i - 1 + (tx & 1);
    const double lap = p[o][i - HW] + p[o][i + HW] + p[o][w] + p[o][w + 1] - 4.0 * p[c][i];
    return rb[c][i] - h2i * lap;
  }
};

// One colour of smooth_redblack on the interior tile nodes: thread k takes row 1 + k / H and
// the k-th node of that colour in it (H = (W-2)/2 per row), so no thread skips nodes.  FLUID
// nodes relax, DIRICHLET nodes take their phi_bc when the caller gave one, others stay.
template <int W>
__device__ __forceinline__ void tile_half_sweep(Tile<W>& T, int colour, double h2, bool has_bc) {
  constexpr int HW = W / 2, HALF = (W - 2) / 2, CNT = (W - 2) * HALF;
  double* __restrict__ own = T.p[colour];
  const double* __restrict__ oth = T.p[colour ^ 1];
  const double* __restrict__ rb = T.rb[colour];
  const uint8_t* __restrict__ mk = T.m[colour];
  for (int k = threadIdx.x; k < CNT; k += kSmoothThreads) {
    const int r = k / HALF;
    const int ty = 1 + r;
    const int odd = (colour - ty) & 1;              // tx parity of this colour in row ty
    const int i = ty * HW + (k - r * HALF) + (odd ? 0 : 1);
    const uint8_t m = mk[i];
    if (m == kFluid) {
      const int w = i - 1 + odd;
      const double sum = oth[i - HW] + oth[i + HW] + oth[w] + oth[w + 1];
      own[i] = 0.25 * (sum - h2 * rb[i]);
    } else if (m == kDir && has_bc) {
      own[i] = rb[i];
    }
  }
}

// Stages the tile: phi, the node kind and the rhs slot of every node.  Every load of a thread
// is issued before any is used, so a tile waits for one memory latency; the DIRICHLET values
// (rare) and, with PRO, the coarse correction of the FLUID nodes follow in a second round.
template <int W, bool PRO>
__device__ __forceinline__ void stage_tile(Tile<W>& T, const double* __restrict__ phi, const double* __restrict__ rhs,
                                           const uint8_t* __restrict__ mask, const double* __restrict__ bc,
                                           const double* __restrict__ coarse, int nx, int ny, int nxc, int x0, int y0,
                                           bool bilinear) {
  constexpr int IT = (W * W + kSmoothThreads - 1) / kSmoothThreads;
  double p[IT], r[IT];
  uint8_t m[IT];
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int k = threadIdx.x + it * kSmoothThreads;
    p[it] = 0.0; r[it] = 0.0; m[it] = kFixed;
    if (k < W * W) {
      const int ty = k / W, tx = k - ty * W;
      const int gx = x0 + tx, gy = y0 + ty;
      if (gx >= 0 && gy >= 0 && gx < nx && gy < ny) {
        const size_t id = (size_t)gy * nx + gx;
        p[it] = phi[id];
        if (gx > 0 && gy > 0 && gx < nx - 1 && gy < ny - 1) {
          m[it] = mask[id];
          r[it] = rhs[id];
        }
      }
    }
  }
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int k = threadIdx.x + it * kSmoothThreads;
    if (k < W * W) {
      const int ty = k / W, tx = k - ty * W;
      const int gx = x0 + tx, gy = y0 + ty;
      double pv = p[it], rv = r[it];
      if (m[it] == kFluid) {
        if (PRO) pv += prolong_at(coarse, nxc, gx, gy, bilinear);
      } else {
        rv = (m[it] == kDir && bc) ? bc[(size_t)gy * nx + gx] : 0.0;
      }
      const int c = Tile<W>::colour(tx, ty), i = Tile<W>::at(tx, ty);
      T.p[c][i] = pv; T.rb[c][i] = rv; T.m[c][i] = m[it];
    }
  }
}

// The 32 x 32 output region of a staged tile (halo H) back to global memory.
template <int W, int H>
__device__ __forceinline__ void store_tile(const Tile<W>& T, double* __restrict__ out, int nx, int ny, int x0,
                                           int y0) {
  for (int k = threadIdx.x; k < kTile * kTile; k += kSmoothThreads) {
    const int ty = k / kTile, tx = k - ty * kTile;
    const int gx = x0 + H + tx, gy = y0 + H + ty;
    if (gx < nx && gy < ny) out[(size_t)gy * nx + gx] = T.phi(tx + H, ty + H);
  }
}

// NU sweeps (post-smoothing with PRO: after adding the coarse correction) of one tile.
template <int NU, bool PRO>
__global__ void __launch_bounds__(kSmoothThreads) emb_smooth_kernel(
    const double* __restrict__ phi_in, double* __restrict__ phi_out, const double* __restrict__ rhs,
    const uint8_t* __restrict__ mask, const double* __restrict__ bc, const double* __restrict__ coarse, int nx, int ny,
    int nxc, double h2, int bilinear) {
  constexpr int H = 2 * NU, W = kTile + 2 * H;
  __shared__ Tile<W> T;
  const int x0 = blockIdx.x * kTile - H, y0 = blockIdx.y * kTile - H;
  stage_tile<W, PRO>(T, phi_in, rhs, mask, bc, coarse, nx, ny, nxc, x0, y0, bilinear != 0);
  __syncthreads();
#pragma unroll 1
  for (int s = 0; s < 2 * NU; ++s) {
    tile_half_sweep<W>(T, s & 1, h2, bc != nullptr);
    __syncthreads();
  }
  store_tile<W, H>(T, phi_out, nx, ny, x0, y0);
}

// Coarse node kind from the fine kinds around fine node (tx, ty): the kind of that node, or
// (any) DIRICHLET if any of the 3x3 is, else SOLID if any is not FLUID, else FLUID.
template <class M>
__device__ __forceinline__ uint8_t coarse_kind_of(M kind, bool any) {
  if (!any) return kind(0, 0);
  bool dir = false, other = false;
#pragma unroll
  for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
    for (int di = -1; di <= 1; ++di) {
      const uint8_t m = kind(di, dj);
      dir |= m == kDir;
      other |= m != kFluid && m != kDir;
    }
  return dir ? kDir : other ? kSolid : kFluid;
}

// Full weighting of the fine residual (restrict_kernel's sum order) around a fine node;
// res(di, dj) is the residual at offset (di, dj).
template <class R>
__device__ __forceinline__ double full_weight(R res) {
  double sum = 0.0;
  sum += res(0, 0);
  sum += 0.5 * (res(-1, 0) + res(1, 0) + res(0, -1) + res(0, 1));
  sum += 0.25 * (res(-1, -1) + res(1, -1) + res(-1, 1) + res(1, 1));
  return sum / 4.0;
}

// Pre-smoothing of one tile fused with the restriction: NU sweeps on a tile with a halo of
// 2 NU + 2 (so the smoothed phi is exact two nodes beyond the output region), the 32 x 32
// output region written back, then for the 16 x 16 coarse nodes whose fine node (2i, 2j)
// lies in the output region: the residual of the nine fine nodes from shared memory
// (residual_kernel's expression), full weighting, the coarse kind, and coarse phi = 0.
template <int NU>
__global__ void __launch_bounds__(kSmoothThreads) emb_down_kernel(
    const double* __restrict__ phi_in, double* __restrict__ phi_out, const double* __restrict__ rhs,
    const uint8_t* __restrict__ mask, const double* __restrict__ bc, int nx, int ny, double h2,
    double* __restrict__ rhs_c, uint8_t* __restrict__ mask_c, double* __restrict__ phi_c, int nxc, int nyc, int any) {
  constexpr int H = 2 * NU + 2, W = kTile + 2 * H;
  __shared__ Tile<W> T;
  const int x0 = blockIdx.x * kTile - H, y0 = blockIdx.y * kTile - H;
  stage_tile<W, false>(T, phi_in, rhs, mask, bc, nullptr, nx, ny, 0, x0, y0, false);
  __syncthreads();
#pragma unroll 1
  for (int s = 0; s < 2 * NU; ++s) {
    tile_half_sweep<W>(T, s & 1, h2, bc != nullptr);
    __syncthreads();
  }
  store_tile<W, H>(T, phi_out, nx, ny, x0, y0);
  const double h2i = 1.0 / h2;
  const int k = threadIdx.x;            // 256 threads, one coarse node each
  const int ic = blockIdx.x * (kTile / 2) + (k & 15), jc = blockIdx.y * (kTile / 2) + (k >> 4);
  if (ic >= nxc || jc >= nyc) return;
  const size_t idc = (size_t)jc * nxc + ic;
  phi_c[idc] = 0.0;
  if (ic == 0 || jc == 0 || ic == nxc - 1 || jc == nyc - 1) {
    rhs_c[idc] = 0.0;
    mask_c[idc] = kFluid;
    return;
  }
  const int tx = 2 * ic - x0, ty = 2 * jc - y0;
  const uint8_t kc = coarse_kind_of([&](int di, int dj) { return T.kind(tx + di, ty + dj); }, any != 0);
  mask_c[idc] = kc;
  rhs_c[idc] = kc == kFluid ? full_weight([&](int di, int dj) { return T.residual(tx + di, ty + dj, h2i); }) : 0.0;
}

// Residual of fine node id (interior): restatement of residual_kernel's expression.
__device__ __forceinline__ double fine_residual(const double* phi, const double* rhs, const uint8_t* mask, size_t id,
                                                int nx, double h2i) {
  if (mask[id] != kFluid) return 0.0;
  const double lap = phi[id - nx] + phi[id + nx] + phi[id - 1] + phi[id + 1] - 4.0 * phi[id];
  return rhs[id] - h2i * lap;
}

// ---------------------------------------------------------------- one-CTA lower V-cycle
struct CoarseLevelArgs {
  int n;                     // levels lc .. lc + n - 1
  int nx[PIC_MAX_LEVELS], ny[PIC_MAX_LEVELS];
  double* phi[PIC_MAX_LEVELS];
  double* rhs[PIC_MAX_LEVELS];
  uint8_t* mask[PIC_MAX_LEVELS];
  const double* bc[PIC_MAX_LEVELS];
  double h2[PIC_MAX_LEVELS];
  int soff[PIC_MAX_LEVELS];  // byte offsets in shared memory: phi, rb (doubles), then kinds
  int nu1, nu2, coarsen_any, bilinear;
};

__device__ void cta_half_sweep(double* p, const double* rb, const uint8_t* m, int nx, int ny, int colour, double h2) {
  const int half = (nx - 1) / 2;            // >= nodes of one colour per interior row
  const int cnt = (ny - 2) * half;
  for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
    const int r = k / half;
    const int j = 1 + r;
    const int i = 1 + ((1 + j + colour) & 1) + 2 * (k - r * half);
    if (i >= nx - 1) continue;
    const int t = j * nx + i;
    const uint8_t kk = m[t];
    if (kk == kFluid) {
      const double sum = p[t - nx] + p[t + nx] + p[t - 1] + p[t + 1];
      p[t] = 0.25 * (sum - h2 * rb[t]);
    } else if (kk == kDir) {
      p[t] = rb[t];
    }
  }
}

__global__ void __launch_bounds__(kCoarseThreads) emb_coarse_kernel(CoarseLevelArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int T = blockDim.x;
  auto P = [&](int l) { return reinterpret_cast<double*>(smem + A.soff[l]); };
  auto RB = [&](int l) { return reinterpret_cast<double*>(smem + A.soff[l]) + A.nx[l] * A.ny[l]; };
  auto M = [&](int l) { return reinterpret_cast<uint8_t*>(smem + A.soff[l] + 16 * A.nx[l] * A.ny[l]); };
  // stage the first level: phi, kinds, rhs (DIRICHLET: phi_bc)
  {
    const int nx = A.nx[0], ny = A.ny[0];
    double* p = P(0); double* rb = RB(0); uint8_t* m = M(0);
    for (int k = threadIdx.x; k < nx * ny; k += T) {
      const int j = k / nx, i = k - j * nx;
      p[k] = A.phi[0][k];
      uint8_t kk = kFixed;
      double v = 0.0;
      if (i > 0 && j > 0 && i < nx - 1 && j < ny - 1) {
        kk = smoother_kind(A.mask[0][k], A.bc[0] != nullptr);
        v = kk == kFluid ? A.rhs[0][k] : kk == kDir ? A.bc[0][k] : 0.0;
      }
      m[k] = kk; rb[k] = v;
    }
  }
  __syncthreads();
  // down leg
  int l = 0;
  for (;; ++l) {
    const int nx = A.nx[l], ny = A.ny[l];
    for (int s = 0; s < 2 * A.nu1; ++s) {
      cta_half_sweep(P(l), RB(l), M(l), nx, ny, s & 1, A.h2[l]);
      __syncthreads();
    }
    if (l == A.n - 1) break;
    // restriction from the staged fine level; the kinds in shared memory are the smoother's,
    // so the reference kinds come from global memory (level 0 of this CTA: the caller's;
    // below it: what this CTA wrote, visible to the whole CTA after the barrier)
    const int nxc = A.nx[l + 1], nyc = A.ny[l + 1];
    const double* pf = P(l);
    const double* rbf = RB(l);
    const uint8_t* mk = A.mask[l];   // reference kinds of level l (written above for l > 0)
    const double h2i = 1.0 / A.h2[l];
    double* pc = P(l + 1); double* rbc = RB(l + 1); uint8_t* mc = M(l + 1);
    for (int k = threadIdx.x; k < nxc * nyc; k += T) {
      const int jc = k / nxc, ic = k - jc * nxc;
      pc[k] = 0.0;
      uint8_t kc = kFluid;
      double fc = 0.0;
      if (ic > 0 && jc > 0 && ic < nxc - 1 && jc < nyc - 1) {
        const ptrdiff_t idf = (ptrdiff_t)(2 * jc) * nx + 2 * ic;
        kc = coarse_kind_of([&](int di, int dj) { return mk[idf + (ptrdiff_t)dj * nx + di]; }, A.coarsen_any != 0);
        if (kc == kFluid)
          fc = full_weight([&](int di, int dj) {
                 const ptrdiff_t id = idf + (ptrdiff_t)dj * nx + di;
                 if (mk[id] != kFluid) return 0.0;
                 const double lap = pf[id - nx] + pf[id + nx] + pf[id - 1] + pf[id + 1] - 4.0 * pf[id];
                 return rbf[id] - h2i * lap;
               });
      }
      A.mask[l + 1][k] = kc;       // the reference writes the coarse kinds and rhs of every level
      A.rhs[l + 1][k] = fc;
      const bool interior = ic > 0 && jc > 0 && ic < nxc - 1 && jc < nyc - 1;
      const uint8_t sk = interior ? smoother_kind(kc, A.bc[l + 1] != nullptr) : kFixed;
      mc[k] = sk;
      rbc[k] = sk == kFluid ? fc : sk == kDir ? A.bc[l + 1][k] : 0.0;
    }
    __syncthreads();
  }
  // up leg
  for (l = A.n - 2; l >= 0; --l) {
    const int nx = A.nx[l], ny = A.ny[l], nxc = A.nx[l + 1];
    double* p = P(l);
    const double* pc = P(l + 1);
    const uint8_t* m = M(l);
    for (int k = threadIdx.x; k < nx * ny; k += T) {
      const int j = k / nx, i = k - j * nx;
      const bool interior = i > 0 && j > 0 && i < nx - 1 && j < ny - 1;
      if (interior && m[k] == kFluid) p[k] += prolong_at(pc, nxc, i, j, A.bilinear != 0);
    }
    __syncthreads();
    for (int s = 0; s < 2 * A.nu2; ++s) {
      cta_half_sweep(p, RB(l), m, nx, ny, s & 1, A.h2[l]);
      __syncthreads();
    }
  }
  // every level's phi back to global memory (the reference keeps them in its level arrays)
  for (l = 0; l < A.n; ++l) {
    const int N = A.nx[l] * A.ny[l];
    const double* p = P(l);
    for (int k = threadIdx.x; k < N; k += T) A.phi[l][k] = p[k];
  }
}

// ---------------------------------------------------------------- norms
__device__ double cta_sum(double v, double* red) {
  for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
  return s;
}

// CTA b sums the interior rows 1 + b, 1 + b + gridDim.x, ... (threads along the row), so every
// partial is formed in a fixed order.
__global__ void __launch_bounds__(256) emb_norm_kernel(const double* __restrict__ phi, const double* __restrict__ rhs,
                                                       const uint8_t* __restrict__ mask, int nx, int ny, double h2i,
                                                       double* __restrict__ partials) {
  __shared__ double red[8];
  double r2 = 0.0, f2 = 0.0;
  for (int j = 1 + blockIdx.x; j < ny - 1; j += gridDim.x) {
    const size_t row = (size_t)j * nx;
    for (int i = 1 + threadIdx.x; i < nx - 1; i += 256) {
      const size_t k = row + i;
      if (mask[k] != kFluid) continue;
      const double r = fine_residual(phi, rhs, mask, k, nx, h2i);
      r2 += r * r;
      f2 += rhs[k] * rhs[k];
    }
  }
  const double a = cta_sum(r2, red);
  const double b = cta_sum(f2, red);
  if (threadIdx.x == 0) { partials[2 * blockIdx.x] = a; partials[2 * blockIdx.x + 1] = b; }
}

__global__ void __launch_bounds__(256) emb_norm_final_kernel(const double* __restrict__ partials, int n,
                                                             double* __restrict__ out) {
  __shared__ double red[8];
  double a = 0.0, b = 0.0;
  for (int k = threadIdx.x; k < n; k += 256) { a += partials[2 * k]; b += partials[2 * k + 1]; }
  a = cta_sum(a, red);
  b = cta_sum(b, red);
  if (threadIdx.x == 0) { out[0] = a; out[1] = b; }
}

}  // namespace

// ---------------------------------------------------------------- host side
// Level sizes (nx_{l+1} = (nx_l - 1) / 2 + 1, Multigrid_embedded.cu:140-141) and the first
// level solved by the one-CTA kernel.
void emb_layout(EmbLevels& P, int nx, int ny, int levels) {
  P.L = levels;
  int a = nx, b = ny;
  P.lc = -1;
  for (int l = 0; l < levels; ++l) {
    P.nx[l] = a; P.ny[l] = b;
    if (P.lc < 0 && (int64_t)a * b <= kCoarseMaxNodes) P.lc = l;
    a = (a - 1) / 2 + 1; b = (b - 1) / 2 + 1;
  }
  if (P.lc < 0) P.lc = levels;   // never: the sizes halve down to 2
}

namespace {

int coarse_smem_bytes(const EmbLevels& P, int l0, int offs[PIC_MAX_LEVELS]) {
  int off = 0;
  for (int l = l0; l < P.L; ++l) {
    offs[l - l0] = off;
    const int N = P.nx[l] * P.ny[l];
    off += 16 * N + ((N + 15) / 16) * 16;
  }
  return off;
}

template <int NU, bool PRO>
void launch_smooth(const EmbLevels& P, int l, const double* in, double* out, const double* coarse, bool bilinear,
                   cudaStream_t s) {
  const dim3 grid((P.nx[l] + kTile - 1) / kTile, (P.ny[l] + kTile - 1) / kTile);
  const double h2 = P.h * P.h * std::ldexp(1.0, 2 * l);
  emb_smooth_kernel<NU, PRO><<<grid, kSmoothThreads, 0, s>>>(in, out, P.rhs[l], P.mask[l], P.bc[l], coarse, P.nx[l],
                                                            P.ny[l], PRO ? P.nx[l + 1] : 0, h2, bilinear ? 1 : 0);
}

void smooth_chunk(const EmbLevels& P, int l, int nu, bool pro, const double* in, double* out, bool bilinear,
                  cudaStream_t s) {
  const double* c = pro ? P.phi[l + 1] : nullptr;
  switch (nu * 2 + (pro ? 1 : 0)) {
    case 1: launch_smooth<0, true>(P, l, in, out, c, bilinear, s); break;
    case 2: launch_smooth<1, false>(P, l, in, out, c, bilinear, s); break;
    case 3: launch_smooth<1, true>(P, l, in, out, c, bilinear, s); break;
    case 4: launch_smooth<2, false>(P, l, in, out, c, bilinear, s); break;
    case 5: launch_smooth<2, true>(P, l, in, out, c, bilinear, s); break;
    case 6: launch_smooth<3, false>(P, l, in, out, c, bilinear, s); break;
    case 7: launch_smooth<3, true>(P, l, in, out, c, bilinear, s); break;
    case 8: launch_smooth<4, false>(P, l, in, out, c, bilinear, s); break;
    case 9: launch_smooth<4, true>(P, l, in, out, c, bilinear, s); break;
    default: break;
  }
}

template <int NU>
void launch_down(const EmbLevels& P, int l, const double* in, double* out, int any, cudaStream_t s) {
  const dim3 grid((P.nx[l] + kTile - 1) / kTile, (P.ny[l] + kTile - 1) / kTile);
  const double h2 = P.h * P.h * std::ldexp(1.0, 2 * l);
  emb_down_kernel<NU><<<grid, kSmoothThreads, 0, s>>>(in, out, P.rhs[l], P.mask[l], P.bc[l], P.nx[l], P.ny[l], h2,
                                                     P.rhs[l + 1], P.mask[l + 1], P.phi[l + 1], P.nx[l + 1],
                                                     P.ny[l + 1], any);
}

// nu sweeps of level l (chunks of at most 4 per launch; the first applies the prolongation
// when pro is set); `cur` tracks which of phi[l] / alt[l] holds the level's current values.
void smooth_level(const EmbLevels& P, int l, int nu, bool pro, double*& cur, bool bilinear, cudaStream_t s) {
  while (nu > 0 || pro) {
    const int c = std::min(nu, 4);
    double* out = cur == P.phi[l] ? P.alt[l] : P.phi[l];
    smooth_chunk(P, l, c, pro, cur, out, bilinear, s);
    cur = out;
    nu -= c;
    pro = false;
  }
}

}  // namespace

// One V-cycle of Multigrid::vcycle(l0) on the level arrays of P (results in P.phi[l]).
int emb_vcycle(const EmbLevels& P, int l0, int nu1, int nu2, int options, cudaStream_t s) {
  // the one-CTA kernel's shared memory above the 48 KB default, once per device
  static std::atomic<int> smem_set[64];
  int dev = 0;
  cudaError_t e0 = cudaGetDevice(&dev);
  if (e0 != cudaSuccess) return pic_fail(PIC_ERR_CUDA, cudaGetErrorString(e0));
  if (dev >= 64) return pic_fail(PIC_ERR_ARG, "device index beyond the solver's table");
  if (!smem_set[dev].load()) {
    e0 = cudaFuncSetAttribute(emb_coarse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e0 != cudaSuccess) return pic_fail(PIC_ERR_CUDA, cudaGetErrorString(e0));
    smem_set[dev].store(1);
  }
  const bool bilinear = options & PIC_EMB_PROLONG_BILINEAR;
  const int any = (options & PIC_EMB_COARSEN_ANY) ? 1 : 0;
  const int lc = std::max(P.lc, l0);
  double* cur[PIC_MAX_LEVELS];
  for (int l = l0; l < lc; ++l) {
    cur[l] = P.phi[l];
    if (l < P.L - 1) {
      // all but the last (up to 4) pre-sweeps, then those fused with the restriction
      const int last = nu1 == 0 ? 0 : (nu1 - 1) % 4 + 1;
      smooth_level(P, l, nu1 - last, false, cur[l], bilinear, s);
      double* out = cur[l] == P.phi[l] ? P.alt[l] : P.phi[l];
      switch (last) {
        case 0: launch_down<0>(P, l, cur[l], out, any, s); break;
        case 1: launch_down<1>(P, l, cur[l], out, any, s); break;
        case 2: launch_down<2>(P, l, cur[l], out, any, s); break;
        case 3: launch_down<3>(P, l, cur[l], out, any, s); break;
        default: launch_down<4>(P, l, cur[l], out, any, s); break;
      }
      cur[l] = out;
      continue;
    }
    smooth_level(P, l, nu1, false, cur[l], bilinear, s);
    {   // coarsest level on the tile path: pre-sweeps only
      if (cur[l] != P.phi[l]) {
        const cudaError_t e = cudaMemcpyAsync(P.phi[l], cur[l], sizeof(double) * P.nx[l] * P.ny[l],
                                              cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return pic_fail(PIC_ERR_CUDA, cudaGetErrorString(e));
      }
    }
  }
  if (lc < P.L) {
    CoarseLevelArgs A{};
    A.n = P.L - lc;
    for (int k = 0; k < A.n; ++k) {
      const int l = lc + k;
      A.nx[k] = P.nx[l]; A.ny[k] = P.ny[l];
      A.phi[k] = P.phi[l]; A.rhs[k] = P.rhs[l]; A.mask[k] = P.mask[l]; A.bc[k] = P.bc[l];
      A.h2[k] = P.h * P.h * std::ldexp(1.0, 2 * l);
    }
    const int bytes = coarse_smem_bytes(P, lc, A.soff);
    A.nu1 = nu1; A.nu2 = nu2; A.coarsen_any = any; A.bilinear = bilinear ? 1 : 0;
    emb_coarse_kernel<<<1, kCoarseThreads, bytes, s>>>(A);
  }
  for (int l = std::min(lc, P.L - 1) - 1; l >= l0; --l) {
    smooth_level(P, l, nu2, true, cur[l], bilinear, s);
    if (cur[l] != P.phi[l]) {
      cudaError_t e = cudaMemcpyAsync(P.phi[l], cur[l], sizeof(double) * P.nx[l] * P.ny[l], cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return pic_fail(PIC_ERR_CUDA, cudaGetErrorString(e));
    }
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return pic_fail(PIC_ERR_CUDA, cudaGetErrorString(e));
  return PIC_OK;
}

// ||r||^2 and ||rhs||^2 over level 0's FLUID nodes into out (device, 2 doubles).
int emb_norms(const EmbLevels& P, double* partials, double* out, cudaStream_t s) {
  const double h2i = 1.0 / (P.h * P.h);
  const int nb = std::max(1, std::min(kNormBlocks, P.ny[0] - 2));
  emb_norm_kernel<<<nb, 256, 0, s>>>(P.phi[0], P.rhs[0], P.mask[0], P.nx[0], P.ny[0], h2i, partials);
  emb_norm_final_kernel<<<1, 256, 0, s>>>(partials, nb, out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return pic_fail(PIC_ERR_CUDA, cudaGetErrorString(e));
  return PIC_OK;
}

namespace {

// Working arrays of pic_solve_embedded_f64, one set per (device, nx, ny, levels), kept until
// the process exits.
struct EmbScratch {
  int device, nx, ny, levels;
  EmbLevels P;           // coarse-level pointers (level 0 is filled per call)
  double* alt0;
  double* partials;
  double* norms;         // device, 2 doubles
  double* host_norms;    // pinned, 2 doubles
};
std::mutex g_emb_mu;
std::vector<EmbScratch> g_emb;

int emb_scratch(int device, int nx, int ny, int levels, EmbScratch** out) {
  for (auto& c : g_emb)
    if (c.device == device && c.nx == nx && c.ny == ny && c.levels == levels) { *out = &c; return PIC_OK; }
  EmbScratch c{};
  c.device = device; c.nx = nx; c.ny = ny; c.levels = levels;
  emb_layout(c.P, nx, ny, levels);
  std::vector<void*> got;
  auto A = [&](void** p, size_t b) {
    const cudaError_t e = cudaMalloc(p, b);
    if (e == cudaSuccess) got.push_back(*p);
    return e;
  };
  cudaError_t e = A((void**)&c.alt0, sizeof(double) * nx * ny);
  for (int l = 1; l < levels && e == cudaSuccess; ++l) {
    const size_t N = (size_t)c.P.nx[l] * c.P.ny[l];
    e = A((void**)&c.P.phi[l], 8 * N);
    if (e == cudaSuccess && l < c.P.lc) e = A((void**)&c.P.alt[l], 8 * N);
    if (e == cudaSuccess) e = A((void**)&c.P.rhs[l], 8 * N);
    if (e == cudaSuccess) e = A((void**)&c.P.mask[l], N);
  }
  if (e == cudaSuccess) e = A((void**)&c.partials, sizeof(double) * 2 * kNormBlocks);
  if (e == cudaSuccess) e = A((void**)&c.norms, sizeof(double) * 2);
  if (e == cudaSuccess) {
    e = cudaMallocHost((void**)&c.host_norms, sizeof(double) * 2);
  }
  if (e != cudaSuccess) {
    for (void* p : got) cudaFree(p);
    cudaGetLastError();
    return pic_fail(e == cudaErrorMemoryAllocation ? PIC_ERR_OOM : PIC_ERR_CUDA, cudaGetErrorString(e));
  }
  g_emb.push_back(c);
  *out = &g_emb.back();
  return PIC_OK;
}

double emb_relative(const double n[2], double r0) {
  if (n[1] > 0.0) return std::sqrt(n[0] / n[1]);
  if (r0 > 0.0) return std::sqrt(n[0] / r0);
  return std::sqrt(n[0]);
}

}  // namespace

extern "C" int pic_solve_embedded_f64(double* phi, const double* rhs, const uint8_t* mask, const double* phi_bc, int nx,
                                      int ny, int levels, double h, int nu_pre, int nu_post, int options, double tol,
                                      int max_cycles, void* stream, int* cycles_out, double* relres_out) {
  if (!phi || !rhs || !mask) return pic_fail(PIC_ERR_ARG, "null grid pointers");
  if (nx < 3 || ny < 3) return pic_fail(PIC_ERR_ARG, "grid needs at least 3 x 3 nodes");
  if ((int64_t)nx * ny > (int64_t)1 << 31) return pic_fail(PIC_ERR_ARG, "grid too large");
  if (levels < 1 || levels > PIC_MAX_LEVELS) return pic_fail(PIC_ERR_ARG, "levels must be in 1..14");
  if (!(h > 0)) return pic_fail(PIC_ERR_ARG, "h must be positive");
  if (nu_pre < 0 || nu_post < 0 || nu_pre > 64 || nu_post > 64) return pic_fail(PIC_ERR_ARG, "sweep counts out of range");
  if (options & ~(PIC_EMB_COARSEN_ANY | PIC_EMB_PROLONG_BILINEAR)) return pic_fail(PIC_ERR_ARG, "unknown option bits");
  if (max_cycles < 1 || !(tol >= 0)) return pic_fail(PIC_ERR_ARG, "max_cycles >= 1 and tol >= 0 required");
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) { cudaGetLastError(); return pic_fail(PIC_ERR_NO_DEVICE, cudaGetErrorString(e)); }
  std::lock_guard<std::mutex> lk(g_emb_mu);
  EmbScratch* S = nullptr;
  int rc = emb_scratch(device, nx, ny, levels, &S);
  if (rc) return rc;
  EmbLevels P = S->P;
  P.phi[0] = phi; P.alt[0] = S->alt0; P.rhs[0] = const_cast<double*>(rhs);
  P.mask[0] = const_cast<uint8_t*>(mask); P.bc[0] = phi_bc; P.h = h;
  cudaStream_t s = (cudaStream_t)stream;
  const bool check = tol > 0;
  double r0 = 0.0, n[2] = {0.0, 0.0};
  auto read_norms = [&]() -> int {
    int r = emb_norms(P, S->partials, S->norms, s);
    if (r) return r;
    cudaError_t e2 = cudaMemcpyAsync(S->host_norms, S->norms, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(s);
    if (e2 != cudaSuccess) return pic_fail(PIC_ERR_CUDA, cudaGetErrorString(e2));
    n[0] = S->host_norms[0]; n[1] = S->host_norms[1];
    return PIC_OK;
  };
  if (check || relres_out) {
    if ((rc = read_norms())) return rc;
    r0 = n[0];
  }
  int cyc = 0;
  double rel = emb_relative(n, r0);
  while (cyc < max_cycles) {
    if ((rc = emb_vcycle(P, 0, nu_pre, nu_post, options, s))) return rc;
    ++cyc;
    if (check) {
      if ((rc = read_norms())) return rc;
      rel = emb_relative(n, r0);
      if (rel < tol) break;
    }
  }
  if (!check && relres_out) {
    if ((rc = read_norms())) return rc;
    rel = emb_relative(n, r0);
  }
  if (cycles_out) *cycles_out = cyc;
  if (relres_out) *relres_out = rel;
  // tol == 0 never converges (as in pic_solve_multigrid_f64): exactly max_cycles V-cycles
  if (!(rel < tol)) return pic_fail(PIC_ERR_NOT_CONVERGED, "embedded multigrid stopped at max_cycles above tol");
  return PIC_OK;
}
