// mg_cluster.cu — the coarse part of the V-cycle (levels 513^2 .. 3^2) in one thread-block
// cluster, with the whole level hierarchy resident in distributed shared memory.
//
// Same algorithm as mg_coarse_kernel / v_cycle of the reference (Multigrid.cu:539-569):
// nu_pre red-black SOR sweeps from a zero guess, residual + full weighting, recursion,
// bilinear prolongation added, nu_post sweeps; nu_coarse sweeps on the coarsest level.
// Layout: a cluster of C CTAs per job.  For every "cluster level" (n_l - 1 divisible by C and
// n_l >= 65) CTA r owns rows [r*B, (r+1)*B) with B = (n_l - 1)/C (the last CTA also owns row
// n_l - 1); rows a CTA reads from a neighbour (stencil halos, restriction, prolongation) come
// over DSMEM.  Levels below are "local levels": rank 0 runs them alone.  Every phase that
// reads what another CTA wrote is separated by a hardware cluster barrier.
#include <cooperative_groups.h>
#include "common.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace {

constexpr int kMaxC = 16;
constexpr int kClusterThreads = 512;

struct Lv {
  int n, B, rows;       // nodes per side, rows per CTA (cluster levels), rows allocated per CTA
  int offE, offF;       // float offsets of this level's e and f blocks in every CTA's smem
  bool cluster;         // distributed level (else local to rank 0)
};

struct ClusterCtx {
  float* sm;            // this CTA's shared memory
  int rank, C;
};

// Row j of level v's e (or f) block: own rows through the CTA's own shared memory, other
// rows through the owner's shared memory mapped into the cluster window (DSMEM).
__device__ __forceinline__ float* row_ptr(cg::cluster_group& cl, const ClusterCtx& X, const Lv v, int j, bool f) {
  const int off = f ? v.offF : v.offE;
  if (!v.cluster) {
    float* b = X.rank == 0 ? X.sm : cl.map_shared_rank(X.sm, 0);
    return b + off + j * v.n;
  }
  const int r = min(j / v.B, X.C - 1);
  float* b = (r == X.rank) ? X.sm : cl.map_shared_rank(X.sm, r);
  return b + off + (j - r * v.B) * v.n;
}
// rows [j0, j1) this CTA updates on level v (cluster levels: own strip; local: all on rank 0)
__device__ __forceinline__ void own_rows(const ClusterCtx& X, const Lv v, int& j0, int& j1) {
  if (v.cluster) {
    j0 = X.rank * v.B;
    j1 = (X.rank == X.C - 1) ? v.n : j0 + v.B;
  } else {
    j0 = 0;
    j1 = (X.rank == 0) ? v.n : 0;
  }
}

__device__ __forceinline__ void phase_sync(cg::cluster_group& cl, const Lv v) {
  if (v.cluster) cl.sync(); else __syncthreads();
}

// Red-black SOR half-sweeps on the owned rows of one level; a cluster barrier between
// colours for distributed levels (the strip's edge rows read the neighbours' rows).
__device__ void sweeps(cg::cluster_group& cl, const ClusterCtx& X, const Lv v, float h2, float omega, int nu) {
  const float om1 = 1.f - omega;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  int j0, j1;
  own_rows(X, v, j0, j1);
  j0 = max(j0, 1);
  j1 = min(j1, v.n - 1);
  for (int it = 0; it < nu; ++it) {
    for (int colour = 1; colour >= 0; --colour) {
      for (int j = j0 + warp; j < j1; j += nwarp) {
        float* e = row_ptr(cl, X, v, j, false);
        const float* f = row_ptr(cl, X, v, j, true);
        const float* up = row_ptr(cl, X, v, j + 1, false);
        const float* dn = row_ptr(cl, X, v, j - 1, false);
        const int i0 = 1 + ((colour - 1 - j) & 1);
        for (int i = i0 + 2 * lane; i < v.n - 1; i += 64) {
          const float s = up[i] + dn[i] + e[i + 1] + e[i - 1];
          const float nv = 0.25f * (s - h2 * f[i]);
          e[i] = fmaf(omega, nv, om1 * e[i]);
        }
      }
      phase_sync(cl, v);
    }
  }
}

// Residual of fine level a, full weighting into f of coarse level b; e of b zeroed.
__device__ void restrict_to(cg::cluster_group& cl, const ClusterCtx& X, const Lv a, const Lv b, float inv_h2) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  int j0, j1;
  own_rows(X, b, j0, j1);
  for (int jc = j0 + warp; jc < j1; jc += nwarp) {
    float* fc = row_ptr(cl, X, b, jc, true);
    float* ec = row_ptr(cl, X, b, jc, false);
    const bool interior_row = jc > 0 && jc < b.n - 1;
    const float* E[5];
    const float* F[3];
    if (interior_row) {
#pragma unroll
      for (int d = 0; d < 5; ++d) E[d] = row_ptr(cl, X, a, 2 * jc - 2 + d, false);
#pragma unroll
      for (int d = 0; d < 3; ++d) F[d] = row_ptr(cl, X, a, 2 * jc - 1 + d, true);
    }
    for (int ic = lane; ic < b.n; ic += 32) {
      float v = 0.f;
      if (interior_row && ic > 0 && ic < b.n - 1) {
        float r[3][3];
#pragma unroll
        for (int dy = 0; dy < 3; ++dy)
#pragma unroll
          for (int dx = -1; dx <= 1; ++dx) {
            const int i = 2 * ic + dx;
            const float* e = E[dy + 1];
            const float lap = (E[dy][i] + E[dy + 2][i] + e[i - 1] + e[i + 1] - 4.f * e[i]) * inv_h2;
            r[dy][dx + 1] = F[dy][i] - lap;
          }
        v = (4.f * r[1][1] + 2.f * r[1][0] + 2.f * r[1][2] + 2.f * r[0][1] + 2.f * r[2][1] + r[0][0] + r[0][2] +
             r[2][0] + r[2][2]) * 0.0625f;
      }
      fc[ic] = v;
      ec[ic] = 0.f;
    }
  }
}

// e of fine level a += bilinear prolongation of e of coarse level b (interior rows/cols).
__device__ void prolong_from(cg::cluster_group& cl, const ClusterCtx& X, const Lv a, const Lv b) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  int j0, j1;
  own_rows(X, a, j0, j1);
  j0 = max(j0, 1);
  j1 = min(j1, a.n - 1);
  for (int j = j0 + warp; j < j1; j += nwarp) {
    float* e = row_ptr(cl, X, a, j, false);
    const float* c0 = row_ptr(cl, X, b, j >> 1, false);
    const float* c1 = (j & 1) ? row_ptr(cl, X, b, (j >> 1) + 1, false) : c0;
    for (int i = 1 + lane; i < a.n - 1; i += 32) {
      const int ic = i >> 1;
      float v;
      if (!(i & 1) && !(j & 1)) v = c0[ic];
      else if ((i & 1) && !(j & 1)) v = 0.5f * (c0[ic] + c0[ic + 1]);
      else if (!(i & 1) && (j & 1)) v = 0.5f * (c0[ic] + c1[ic]);
      else v = 0.25f * (c0[ic] + c0[ic + 1] + c1[ic] + c1[ic + 1]);
      e[i] += v;
    }
  }
}

}  // namespace

// One cluster per job of the list; level lc of the job is the first cluster level.
__global__ void __launch_bounds__(kClusterThreads, 1) mg_cluster_kernel(const int* __restrict__ job_list, const JobDev* __restrict__ jobs,
                                                            const JobState* __restrict__ st) {
  extern __shared__ float sm[];
  cg::cluster_group cl = cg::this_cluster();
  const int job = job_list[blockIdx.x / cl.num_blocks()];
  const JobDev& J = jobs[job];
  if (st[job].converged) return;  // uniform over the cluster: no barrier is skipped by part of it
  ClusterCtx X;
  X.sm = sm;
  X.C = (int)cl.num_blocks();
  X.rank = (int)cl.block_rank();
  const int lc = J.lc, L = J.levels;
  Lv lv[PIC_MAX_LEVELS];
  {
    int off = 0;
    for (int l = lc; l < L; ++l) {
      Lv& v = lv[l];
      v.n = J.nl[l];
      v.cluster = ((v.n - 1) % X.C == 0) && v.n >= 65;
      v.B = v.cluster ? (v.n - 1) / X.C : v.n;
      v.rows = v.cluster ? v.B + 1 : v.n;
      v.offE = off;
      off += v.rows * v.n;
      v.offF = off;
      off += v.rows * v.n;
    }
  }
  // load f of the top level (own rows), e = 0
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  {
    const Lv v = lv[lc];
    int j0, j1;
    own_rows(X, v, j0, j1);
    const float* fg = J.f[lc];
    for (int j = j0 + warp; j < j1; j += nwarp) {
      float* fr = row_ptr(cl, X, v, j, true);
      float* er = row_ptr(cl, X, v, j, false);
      for (int i = lane; i < v.n; i += 32) { fr[i] = __ldg(fg + (size_t)j * J.pl[lc] + i); er[i] = 0.f; }
    }
  }
  cl.sync();
  // down
  for (int l = lc; l < L - 1; ++l) {
    const double hl = J.h * (double)(1 << l);
    sweeps(cl, X, lv[l], (float)(hl * hl), J.omega, J.nu_pre);
    restrict_to(cl, X, lv[l], lv[l + 1], (float)(1.0 / (hl * hl)));
    phase_sync(cl, lv[l]);
  }
  {
    const double hl = J.h * (double)(1 << (L - 1));
    sweeps(cl, X, lv[L - 1], (float)(hl * hl), J.omega, J.nu_coarse);
  }
  // up
  for (int l = L - 2; l >= lc; --l) {
    // a local coarse level was finished by rank 0 alone: wait for it before reading it
    if (lv[l].cluster && !lv[l + 1].cluster) cl.sync();
    prolong_from(cl, X, lv[l], lv[l + 1]);
    phase_sync(cl, lv[l]);
    const double hl = J.h * (double)(1 << l);
    sweeps(cl, X, lv[l], (float)(hl * hl), J.omega, J.nu_post);
  }
  // store e of the top level (own rows)
  {
    const Lv v = lv[lc];
    int j0, j1;
    own_rows(X, v, j0, j1);
    float* eg = J.e[lc];
    for (int j = j0 + warp; j < j1; j += nwarp) {
      const float* er = row_ptr(cl, X, v, j, false);
      for (int i = lane; i < v.n; i += 32) eg[(size_t)j * J.pl[lc] + i] = er[i];
    }
  }
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

// Shared memory per CTA for a job whose first cluster level is lc.
size_t mg_cluster_smem(const int* nl, int lc, int levels, int C) {
  size_t off = 0;
  for (int l = lc; l < levels; ++l) {
    const int n = nl[l];
    const bool cl = ((n - 1) % C == 0) && n >= 65;
    const int rows = cl ? (n - 1) / C + 1 : n;
    off += 2ull * rows * n;
  }
  return off * sizeof(float);
}

int mg_cluster_supported(int C, size_t smem) {
  if (cudaFuncSetAttribute(mg_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess ||
      cudaFuncSetAttribute(mg_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(kClusterThreads);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute a[1];
  a[0].id = cudaLaunchAttributeClusterDimension;
  a[0].val.clusterDim.x = C;
  a[0].val.clusterDim.y = 1;
  a[0].val.clusterDim.z = 1;
  cfg.attrs = a;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, mg_cluster_kernel, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int launch_mg_cluster(const int* job_list, int njobs, int C, size_t smem, const JobDev* jobs, const JobState* st,
                      cudaStream_t s) {
  if (njobs == 0) return 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C * njobs);
  cfg.blockDim = dim3(kClusterThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute a[1];
  a[0].id = cudaLaunchAttributeClusterDimension;
  a[0].val.clusterDim.x = C;
  a[0].val.clusterDim.y = 1;
  a[0].val.clusterDim.z = 1;
  cfg.attrs = a;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, mg_cluster_kernel, job_list, jobs, st);
  return 1;
}
