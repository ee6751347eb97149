// convert.cu — layout conversions and small bookkeeping kernels.
//   load:   FP64 domain-unit positions/velocities (the reference's double2 r, v arrays,
//           main.cu:232-238) -> cell index + FP32 in-cell offsets + FP32 velocities
//   export: the reverse (Particles2D::debugParticles-style read-back, particles.cu:200)
//   grids:  rho in charge units, phi (FP64), E = -grad(phi) with the stencils of
//           computeElectricField (kernels.cu:134-191)
#include <algorithm>
#include <cstdint>
#include "common.cuh"
#include "kernels.h"

namespace {

__global__ void load_kernel(const SlotDev* __restrict__ sd, int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ vx, const double* __restrict__ vy, const double* __restrict__ vz,
                            const uint32_t* __restrict__ pid, uint32_t pid_base, double inv_dx, double inv_dy, int ncx,
                            int ncy) {
  const SlotDev S = *sd;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const double xi = x[p] * inv_dx, eta = y[p] * inv_dy;
    const double fi = floor(xi), fj = floor(eta);
    if (fi >= 0.0 && fi < (double)ncx && fj >= 0.0 && fj < (double)ncy) {
      const int i = (int)fi, j = (int)fj;
      S.cell[p] = pack_cell(i, j);
      S.fx[p] = fminf((float)(xi - fi), 0.99999994f);
      S.fy[p] = fminf((float)(eta - fj), 0.99999994f);
    } else {
      S.cell[p] = PIC_CELL_OUT;
      S.fx[p] = (float)xi;
      S.fy[p] = (float)eta;
    }
    S.vx[p] = (float)vx[p];
    S.vy[p] = (float)vy[p];
    S.vz[p] = vz ? (float)vz[p] : 0.f;
    S.pid[p] = pid ? pid[p] : pid_base + (uint32_t)p;
  }
}

__global__ void export_kernel(const SlotDev* __restrict__ sd, int64_t n, double* x, double* y, double* vx, double* vy,
                              double* vz, uint32_t* pid, double dx, double dy) {
  const SlotDev S = *sd;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t c = S.cell[p];
    double gx, gy;
    if (c != PIC_CELL_OUT) { gx = (double)cell_i(c) + (double)S.fx[p]; gy = (double)cell_j(c) + (double)S.fy[p]; }
    else { gx = (double)S.fx[p]; gy = (double)S.fy[p]; }
    if (x) x[p] = gx * dx;
    if (y) y[p] = gy * dy;
    if (vx) vx[p] = (double)S.vx[p];
    if (vy) vy[p] = (double)S.vy[p];
    if (vz) vz[p] = (double)S.vz[p];
    if (pid) pid[p] = S.pid[p];
  }
}

// Interleaved FP32 (x, y) of every particle: what convertPositionsToFloat (kernels.cu:268-274)
// writes into the reference's OpenGL vertex buffer, here into a plain buffer.  Rounded once from
// the FP64 position the FP64 export returns.
__global__ void snapshot_kernel(const SlotDev* __restrict__ sd, int64_t n, float2* __restrict__ xy, double dx,
                                double dy) {
  const SlotDev S = *sd;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t c = S.cell[p];
    double gx, gy;
    if (c != PIC_CELL_OUT) { gx = (double)cell_i(c) + (double)S.fx[p]; gy = (double)cell_j(c) + (double)S.fy[p]; }
    else { gx = (double)S.fx[p]; gy = (double)S.fy[p]; }
    xy[p] = make_float2((float)(gx * dx), (float)(gy * dy));
  }
}

__global__ void export_raw_kernel(const SlotDev* __restrict__ sd, int64_t n, uint32_t* cell, float* fx, float* fy,
                                  float* vx, float* vy, float* vz, uint32_t* pid) {
  const SlotDev S = *sd;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    if (cell) cell[p] = S.cell[p];
    if (fx) fx[p] = S.fx[p];
    if (fy) fy[p] = S.fy[p];
    if (vx) vx[p] = S.vx[p];
    if (vy) vy[p] = S.vy[p];
    if (vz) vz[p] = S.vz[p];
    if (pid) pid[p] = S.pid[p];
  }
}

__global__ void pid_max_kernel(const SlotDev* __restrict__ sd, int64_t n, JobState* st) {
  uint32_t m = 0;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
    m = max(m, sd->pid[p] + 1u);
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(&st->next_pid, m);
}

__device__ __forceinline__ double rho_at(const JobDev& J, size_t idx) {
  return J.deposit_mode == 0 ? (double)J.rho_f[idx] : J.deposit_mode == 1 ? (double)J.rho_i[idx] * 0x1p-40 : J.rho_d[idx];
}

__global__ void grid_export_kernel(const JobDev* __restrict__ jd, const JobState* __restrict__ st, int which, double* out,
                                   int nx, int ny, double dx, double dy) {
  const JobDev& J = *jd;
  const double* phi = J.phi64[st->phi_cur];
  const int64_t N = (int64_t)nx * ny;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N; k += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(k % nx), j = (int)(k / nx);
    double v;
    if (which == 0) v = rho_at(J, k) * J.qref;
    else if (which == 1) v = phi[k];
    else if (which == 2) {
      if (i == 0) v = -(phi[k + 1] - phi[k]) / dx;
      else if (i == nx - 1) v = -(phi[k] - phi[k - 1]) / dx;
      else v = -(phi[k + 1] - phi[k - 1]) / (2 * dx);
    } else {
      if (j == 0) v = -(phi[k + nx] - phi[k]) / dy;
      else if (j == ny - 1) v = -(phi[k] - phi[k - nx]) / dy;
      else v = -(phi[k + nx] - phi[k - nx]) / (2 * dy);
    }
    out[k] = v;
  }
}

__global__ void grid_import_kernel(const JobDev* __restrict__ jd, const JobState* __restrict__ st, int which,
                                   const double* in, int64_t N) {
  const JobDev& J = *jd;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N; k += (int64_t)gridDim.x * blockDim.x) {
    if (which == 0) {
      const double v = in[k] / J.qref;
      if (J.deposit_mode == 0) J.rho_f[k] = (float)v;
      else J.rho_i[k] = __double2ll_rn(v * 0x1p40);
    } else {
      J.phi64[st->phi_cur][k] = in[k];
    }
  }
}

__global__ void efield_f64_kernel(const double* __restrict__ phi, double* __restrict__ exy, int m, int n, double dx,
                                  double dy) {
  const int64_t N = (int64_t)m * n;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < N; c += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(c % m), y = (int)(c / m);
    double ex, ey;
    if (x == 0) ex = -(phi[c + 1] - phi[c]) / dx;
    else if (x == m - 1) ex = -(phi[c] - phi[c - 1]) / dx;
    else ex = -(phi[c + 1] - phi[c - 1]) / (2 * dx);
    if (y == 0) ey = -(phi[c + m] - phi[c]) / dy;
    else if (y == n - 1) ey = -(phi[c] - phi[c - m]) / dy;
    else ey = -(phi[c + m] - phi[c - m]) / (2 * dy);
    exy[2 * c] = ex;
    exy[2 * c + 1] = ey;
  }
}

__global__ void step_begin_kernel(JobState* st, const JobDev* jobs, int njobs, const uint8_t* job_mask) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs || (job_mask && !job_mask[j])) return;
  JobState& T = st[j];
  for (int s = 0; s < PIC_MAX_SPECIES; ++s) {
    T.ke[s] = 0.0;
    for (int q = 0; q < 8; ++q) T.collisions[s][q] = 0ull;
  }
}

// Before a flush pass (the pending kick and collisions of the last step, applied ahead of a
// read-back): the kinetic energy of the jobs it applies to restarts, so that afterwards it is
// the energy of the velocities the read-back returns.
__global__ void ke_reset_pending_kernel(JobState* st, int njobs) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs || !st[j].kick_pending) return;
  for (int s = 0; s < PIC_MAX_SPECIES; ++s) st[j].ke[s] = 0.0;
}
__global__ void step_end_kernel(JobState* st, int njobs, const uint8_t* job_mask, int set_pending, int advance) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs || (job_mask && !job_mask[j])) return;
  if (advance) st[j].step += 1;
  st[j].kick_pending = set_pending;
}

// Sum of rho (charge units) in FP64 with a fixed reduction order: per-CTA partial sums,
// then one CTA adds them in index order.
__global__ void __launch_bounds__(256) rho_sum_partial_kernel(const JobDev* __restrict__ jd, double* part) {
  const JobDev& J = *jd;
  const int64_t N = (int64_t)J.nx * J.ny;
  double s = 0.0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N; k += (int64_t)gridDim.x * blockDim.x)
    s += rho_at(J, k);
  __shared__ double sh[256];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void rho_sum_final_kernel(const JobDev* __restrict__ jd, const double* part, int nparts, JobState* st) {
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < nparts; ++k) s += part[k];
    st->total_charge = s * jd->qref;
  }
}

__global__ void zero_rho_all_kernel(const JobDev* __restrict__ jobs, int njobs) {
  const JobDev& J = jobs[blockIdx.y];
  if (J.nslots == 0 && J.nx == 0) return;
  const int64_t N = (int64_t)J.nx * J.ny;
  if (J.deposit_mode == 0 && J.rho_f) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N; k += (int64_t)gridDim.x * blockDim.x) J.rho_f[k] = 0.f;
  } else if (J.deposit_mode == 1 && J.rho_i) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N; k += (int64_t)gridDim.x * blockDim.x) J.rho_i[k] = 0;
  }
}

}  // namespace

static int grid_for(int64_t n, int cap = 4096) {
  int64_t g = (n + 255) / 256;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

void launch_load_species(const SlotDev* slot_dev, const JobDev*, int64_t n, const double* x, const double* y,
                         const double* vx, const double* vy, const double* vz, const uint32_t* pid, uint32_t pid_base,
                         double inv_dx, double inv_dy, int ncx, int ncy, cudaStream_t s) {
  if (n <= 0) return;
  load_kernel<<<grid_for(n), 256, 0, s>>>(slot_dev, n, x, y, vx, vy, vz, pid, pid_base, inv_dx, inv_dy, ncx, ncy);
}
void launch_pid_max(const SlotDev* slot_dev, int64_t n, JobState* st, cudaStream_t s) {
  if (n <= 0) return;
  pid_max_kernel<<<grid_for(n, 1024), 256, 0, s>>>(slot_dev, n, st);
}
void launch_export_species(const SlotDev* slot_dev, int64_t n, double* x, double* y, double* vx, double* vy, double* vz,
                           uint32_t* pid, double dx, double dy, cudaStream_t s) {
  if (n <= 0) return;
  export_kernel<<<grid_for(n), 256, 0, s>>>(slot_dev, n, x, y, vx, vy, vz, pid, dx, dy);
}
void launch_snapshot(const SlotDev* slot_dev, int64_t n, float* xy, double dx, double dy, cudaStream_t s) {
  if (n <= 0) return;
  snapshot_kernel<<<grid_for(n), 256, 0, s>>>(slot_dev, n, reinterpret_cast<float2*>(xy), dx, dy);
}
void launch_export_raw(const SlotDev* slot_dev, int64_t n, uint32_t* cell, float* fx, float* fy, float* vx, float* vy,
                       float* vz, uint32_t* pid, cudaStream_t s) {
  if (n <= 0) return;
  export_raw_kernel<<<grid_for(n), 256, 0, s>>>(slot_dev, n, cell, fx, fy, vx, vy, vz, pid);
}
void launch_grid_export(const JobDev* jd, const JobState* st, int which, double* out, int nx, int ny, double dx,
                        double dy, cudaStream_t s) {
  grid_export_kernel<<<grid_for((int64_t)nx * ny), 256, 0, s>>>(jd, st, which, out, nx, ny, dx, dy);
}
void launch_grid_import(const JobDev* jd, const JobState* st, int which, const double* in, int nx, int ny,
                        cudaStream_t s) {
  grid_import_kernel<<<grid_for((int64_t)nx * ny), 256, 0, s>>>(jd, st, which, in, (int64_t)nx * ny);
}
void launch_zero_rho(const JobDev*, int64_t nodes, int deposit_mode, void* rho, cudaStream_t s) {
  cudaMemsetAsync(rho, 0, (size_t)nodes * (deposit_mode == 0 ? 4 : 8), s);
}
void launch_efield_f64(const double* phi, double* exy, int nx, int ny, double dx, double dy, cudaStream_t s) {
  efield_f64_kernel<<<grid_for((int64_t)nx * ny), 256, 0, s>>>(phi, exy, nx, ny, dx, dy);
}
int launch_ke_reset_pending(JobState* st, int njobs, cudaStream_t s) {
  if (njobs <= 0) return 0;
  ke_reset_pending_kernel<<<(njobs + 127) / 128, 128, 0, s>>>(st, njobs);
  return 1;
}
int launch_step_begin(JobState* st, const JobDev* jobs, int njobs, const uint8_t* job_mask, cudaStream_t s) {
  if (!njobs) return 0;
  step_begin_kernel<<<(njobs + 127) / 128, 128, 0, s>>>(st, jobs, njobs, job_mask);
  return 1;
}
int launch_step_end(JobState* st, int njobs, const uint8_t* job_mask, int set_pending, int advance, cudaStream_t s) {
  if (!njobs) return 0;
  step_end_kernel<<<(njobs + 127) / 128, 128, 0, s>>>(st, njobs, job_mask, set_pending, advance);
  return 1;
}
int launch_zero_rho_all(const EngineLaunch& L, int max_nodes, cudaStream_t s) {
  if (!L.njobs) return 0;
  const int gx = (int)std::min<int64_t>(std::max<int64_t>(((int64_t)max_nodes + 1023) / 1024, 1), 1024);
  zero_rho_all_kernel<<<dim3(gx, L.njobs), 256, 0, s>>>(L.jobs, L.njobs);
  return 1;
}
void launch_rho_sum(const JobDev* jd, JobState* st, double* scratch, int nparts, cudaStream_t s) {
  rho_sum_partial_kernel<<<nparts, 256, 0, s>>>(jd, scratch);
  rho_sum_final_kernel<<<1, 32, 0, s>>>(jd, scratch, nparts, st);
}
