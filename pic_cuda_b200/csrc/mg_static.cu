// mg_static.cu — pic_solve_multigrid_f64_static: the stateless multigrid solve on
// caller-owned FP64 arrays, for callers that must not allocate device memory.
//
// The whole solve runs in one CTA of 1024 threads.  Its working set (the FP32 correction and
// right-hand side of every level, plus a small result record) lives in g_mg_scratch, a
// file-scope __device__ array of fixed size, so the call allocates nothing: no cudaMalloc,
// no cudaFree, no library that allocates.  The arithmetic is that of
// pic_solve_multigrid_f64: FP32 red-black SOR V-cycles (odd colour first, full-weighting
// restriction, bilinear prolongation) on the correction equation, inside an FP64
// defect-correction loop; phi is updated in place, its boundary values are the Dirichlet
// data; at least one V-cycle runs; stop at ||rho - lap phi|| / ||rho|| < tol or max_cycles.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "common.cuh"
#include "pic_b200.h"

int pic_fail(int code, const char* msg);

namespace {

constexpr int kMaxSide = PIC_STATIC_MG_MAX_SIDE;  // largest grid side the scratch holds
constexpr int kThreads = 1024;
constexpr int kMaxDevices = 64;

// 2 * sum over levels of n_l^2 floats for a 257^2 grid coarsened to 3^2 is 176,816; the
// result record takes the last 64 floats.
constexpr size_t kScratchFloats = 180224;  // 704 KiB
constexpr size_t kResultOffset = kScratchFloats - 64;

struct Result {
  double relres;
  double rnorm2;
  double fnorm2;
  int cycles;
  int converged;  // 1 reached tol, 2 stopped at max_cycles
};
static_assert(sizeof(Result) <= 64 * sizeof(float), "result record does not fit");

static __device__ __align__(256) float g_mg_scratch[kScratchFloats];

int levels_for(int n) {
  int L = 1;
  while (n > 3 && (n & 1)) {
    n = (n + 1) / 2;
    ++L;
  }
  return L;
}

// Deterministic block sum: fixed per-thread assignment, fixed tree order.
__device__ double block_sum_fixed(double v, double* red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

__device__ void zero(float* a, int n) {
  for (int k = threadIdx.x; k < n; k += kThreads) a[k] = 0.f;
}

// nu red-black SOR sweeps on an n x n level, interior nodes only.
__device__ void sweeps(float* e, const float* f, int n, float h2, float omega, int nu) {
  const float om1 = 1.f - omega;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = kThreads >> 5;
  for (int it = 0; it < nu; ++it) {
    for (int colour = 1; colour >= 0; --colour) {
      for (int j = 1 + warp; j < n - 1; j += nwarp) {
        const int i0 = 1 + ((colour - 1 - j) & 1);
        for (int i = i0 + 2 * lane; i < n - 1; i += 64) {
          const int c = j * n + i;
          const float s = e[c + n] + e[c - n] + e[c + 1] + e[c - 1];
          const float nv = 0.25f * (s - h2 * f[c]);
          e[c] = fmaf(omega, nv, om1 * e[c]);
        }
      }
      __syncthreads();
    }
  }
}

// f_c = full weighting of (f - lap e) on the coarse interior, 0 on its boundary; e_c = 0.
__device__ void restrict_residual(const float* e, const float* f, int n, float inv_h2, float* ec, float* fc, int nc) {
  for (int k = threadIdx.x; k < nc * nc; k += kThreads) {
    const int ic = k % nc, jc = k / nc;
    float v = 0.f;
    if (ic > 0 && ic < nc - 1 && jc > 0 && jc < nc - 1) {
      float r[3][3];
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          const int q = (2 * jc + dy) * n + (2 * ic + dx);
          const float lap = (e[q - n] + e[q + n] + e[q - 1] + e[q + 1] - 4.f * e[q]) * inv_h2;
          r[dy + 1][dx + 1] = f[q] - lap;
        }
      v = (4.f * r[1][1] + 2.f * r[1][0] + 2.f * r[1][2] + 2.f * r[0][1] + 2.f * r[2][1] + r[0][0] + r[0][2] +
           r[2][0] + r[2][2]) * 0.0625f;
    }
    fc[k] = v;
    ec[k] = 0.f;
  }
}

// e += bilinear prolongation of the coarse correction, interior nodes (the coarse boundary is 0).
__device__ void prolong_add(float* e, int n, const float* c, int nc) {
  for (int k = threadIdx.x; k < (n - 2) * (n - 2); k += kThreads) {
    const int i = 1 + k % (n - 2), j = 1 + k / (n - 2);
    const float* cp = c + (j >> 1) * nc + (i >> 1);
    float v;
    if (!(i & 1) && !(j & 1)) v = cp[0];
    else if ((i & 1) && !(j & 1)) v = 0.5f * (cp[0] + cp[1]);
    else if (!(i & 1) && (j & 1)) v = 0.5f * (cp[0] + cp[nc]);
    else v = 0.25f * (cp[0] + cp[1] + cp[nc] + cp[nc + 1]);
    e[j * n + i] += v;
  }
}

// r = rho - lap(phi) on the interior (0 on the boundary) into f0 (FP32); returns sum r^2.
__device__ double residual_f64(const double* phi, const double* rho, int n, double inv_h2, float* f0, double* red) {
  double a = 0.0;
  for (int c = threadIdx.x; c < n * n; c += kThreads) {
    const int i = c % n, j = c / n;
    double r = 0.0;
    if (i > 0 && i < n - 1 && j > 0 && j < n - 1) {
      const double lap = (phi[c - n] + phi[c + n] + phi[c - 1] + phi[c + 1] - 4.0 * phi[c]) * inv_h2;
      r = rho[c] - lap;
    }
    f0[c] = (float)r;
    a += r * r;
  }
  return block_sum_fixed(a, red);
}

__global__ void __launch_bounds__(kThreads) mg_static_kernel(double* __restrict__ phi, const double* __restrict__ rho,
                                                             int n0, int L, double h, float omega, int nu_pre,
                                                             int nu_post, int nu_coarse, double tol, int max_cycles,
                                                             float* __restrict__ scratch) {
  __shared__ double red[kThreads];
  __shared__ int nl[PIC_MAX_LEVELS];
  __shared__ int64_t off[PIC_MAX_LEVELS];
  if (threadIdx.x == 0) {
    int n = n0;
    int64_t o = 0;
    for (int l = 0; l < L; ++l) {
      nl[l] = n;
      off[l] = o;
      o += 2ll * n * n;
      n = (n + 1) / 2;
    }
  }
  __syncthreads();
#define EL(l) (scratch + off[l])
#define FL(l) (scratch + off[l] + (int64_t)nl[l] * nl[l])
  Result* res = reinterpret_cast<Result*>(scratch + kResultOffset);
  const double inv_h2 = 1.0 / (h * h);
  // initial defect and ||rho||^2 over all nodes
  double af = 0.0;
  for (int c = threadIdx.x; c < n0 * n0; c += kThreads) af += rho[c] * rho[c];
  const double f2 = block_sum_fixed(af, red);
  double r2 = residual_f64(phi, rho, n0, inv_h2, FL(0), red);
  double relres = f2 > 0.0 ? sqrt(r2 / f2) : sqrt(r2);
  int cycles = 0, converged = 0;
  while (!converged) {
    zero(EL(0), n0 * n0);
    __syncthreads();
    for (int l = 0; l < L - 1; ++l) {
      const double hl = h * (double)(1 << l);
      sweeps(EL(l), FL(l), nl[l], (float)(hl * hl), omega, nu_pre);
      restrict_residual(EL(l), FL(l), nl[l], (float)(1.0 / (hl * hl)), EL(l + 1), FL(l + 1), nl[l + 1]);
      __syncthreads();
    }
    {
      const double hl = h * (double)(1 << (L - 1));
      sweeps(EL(L - 1), FL(L - 1), nl[L - 1], (float)(hl * hl), omega, nu_coarse);
    }
    for (int l = L - 2; l >= 0; --l) {
      prolong_add(EL(l), nl[l], EL(l + 1), nl[l + 1]);
      __syncthreads();
      const double hl = h * (double)(1 << l);
      sweeps(EL(l), FL(l), nl[l], (float)(hl * hl), omega, nu_post);
    }
    // FP64 correction update (the correction is 0 on the boundary), then the new defect
    for (int c = threadIdx.x; c < n0 * n0; c += kThreads) phi[c] = phi[c] + (double)EL(0)[c];
    __syncthreads();
    r2 = residual_f64(phi, rho, n0, inv_h2, FL(0), red);
    relres = f2 > 0.0 ? sqrt(r2 / f2) : sqrt(r2);
    ++cycles;
    if (relres < tol) converged = 1;
    else if (cycles >= max_cycles) converged = 2;
  }
  if (threadIdx.x == 0) {
    res->relres = relres;
    res->rnorm2 = r2;
    res->fnorm2 = f2;
    res->cycles = cycles;
    res->converged = converged;
  }
#undef EL
#undef FL
}

std::mutex g_mu;
float* g_scratch_ptr[kMaxDevices] = {};

}  // namespace

extern "C" int pic_solve_multigrid_f64_static(double* phi, const double* rho, int nx, int ny, int levels, double h,
                                              double omega, int nu_pre, int nu_post, int nu_coarse, double tol,
                                              int max_cycles, void* stream, int* cycles_out, double* relres_out) {
  if (!phi || !rho) return pic_fail(PIC_ERR_ARG, "null grid pointers");
  if (nx != ny || nx < 3 || ((nx - 1) & (nx - 2)) != 0)
    return pic_fail(PIC_ERR_ARG, "grid must be square with 2^k+1 nodes per side");
  if (nx > kMaxSide) return pic_fail(PIC_ERR_ARG, "grid larger than the static scratch holds (max 257 x 257 nodes)");
  if (!(h > 0)) return pic_fail(PIC_ERR_ARG, "h must be positive");
  const int maxL = levels_for(nx);
  if (levels < 0 || levels > maxL) return pic_fail(PIC_ERR_ARG, "levels out of range");
  if (nu_pre < 0 || nu_pre > 16 || nu_post < 0 || nu_post > 16 || nu_coarse < 0 || nu_coarse > 1000)
    return pic_fail(PIC_ERR_ARG, "sweep counts out of range");
  if (!(omega > 0 && omega < 2)) return pic_fail(PIC_ERR_ARG, "omega must be in (0, 2)");
  if (max_cycles < 1 || !(tol >= 0)) return pic_fail(PIC_ERR_ARG, "max_cycles >= 1 and tol >= 0 required");
  const int L = levels > 0 ? levels : maxL;
  int device = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err != cudaSuccess) {
    cudaGetLastError();
    return pic_fail(PIC_ERR_NO_DEVICE, cudaGetErrorString(err));
  }
  if (device < 0 || device >= kMaxDevices) return pic_fail(PIC_ERR_ARG, "device index beyond the scratch table");
  float* scratch = nullptr;
  {
    // once per device, with that device current: the address of this device's copy
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[device]) {
      void* p = nullptr;
      err = cudaGetSymbolAddress(&p, g_mg_scratch);
      if (err != cudaSuccess || !p) {
        cudaGetLastError();
        return pic_fail(PIC_ERR_CUDA, err != cudaSuccess ? cudaGetErrorString(err) : "null symbol address");
      }
      g_scratch_ptr[device] = static_cast<float*>(p);
    }
    scratch = g_scratch_ptr[device];
  }
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  mg_static_kernel<<<1, kThreads, 0, s>>>(phi, rho, nx, L, h, (float)omega, nu_pre, nu_post, nu_coarse, tol,
                                          max_cycles, scratch);
  err = cudaGetLastError();
  if (err != cudaSuccess) return pic_fail(PIC_ERR_CUDA, cudaGetErrorString(err));
  Result r{};
  err = cudaMemcpyAsync(&r, scratch + kResultOffset, sizeof(Result), cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return pic_fail(PIC_ERR_CUDA, cudaGetErrorString(err));
  if (cycles_out) *cycles_out = r.cycles;
  if (relres_out) *relres_out = r.relres;
  if (r.converged != 1) return pic_fail(PIC_ERR_NOT_CONVERGED, "multigrid stopped at max_cycles above tol");
  return PIC_OK;
}
