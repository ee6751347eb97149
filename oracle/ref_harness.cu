// ref_harness.cu — headless driver for the reference's own CUDA kernels.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile together with the reference's
// sources where they lie (kernels.cu, collisions.cu, particles.cu, Multigrid.cu, grid.cu,
// boundaries.cu, mcc.cu, Multigrid_embedded.cu of dimad285/PIC_CUDA) into
// oracle/_ref/libpicref.so.  main.cu
// cannot be compiled (it needs GL/glew.h, render.h:4), so the step sequence of
// updateSimulationCUDA (main.cu:60-135) is re-sequenced here without the viewer.
// Every entry point takes and returns host arrays; it is used only to pin the FP64
// oracle (tests/golden/make_golden.py) and to time the reference's CUDA step.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <vector>
#include <cuda_runtime.h>

#include <boundaries.h>
#include <collisions.cuh>
#include <grid.cuh>
#include <kernels.cuh>
#include <mcc.hpp>
#include <Multigrid.hpp>
#include <particles.cuh>

#define RH_API extern "C" __attribute__((visibility("default")))

static int ck(cudaError_t e) {
  if (e != cudaSuccess) {
    fprintf(stderr, "ref_harness: %s\n", cudaGetErrorString(e));
    return 1;
  }
  return 0;
}

RH_API int refh_device_ok(void) {
  int n = 0;
  return cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
}

// updateDensity (kernels.cu:26) on host inputs.
RH_API int refh_deposit(int n, const double* x, const double* y, const int* type, const double* qtab,
                        int nspec, int m, int nn, double dx, double dy, double* rho_out) {
  std::vector<double2> r(n);
  for (int i = 0; i < n; ++i) r[i] = make_double2(x[i], y[i]);
  double2* dr = nullptr; int* dt = nullptr; double *dq = nullptr, *drho = nullptr;
  int bad = ck(cudaMalloc(&dr, sizeof(double2) * (n > 0 ? n : 1))) | ck(cudaMalloc(&dt, sizeof(int) * (n > 0 ? n : 1))) |
            ck(cudaMalloc(&dq, sizeof(double) * nspec)) | ck(cudaMalloc(&drho, sizeof(double) * m * nn));
  if (bad) return 1;
  cudaMemcpy(dr, r.data(), sizeof(double2) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(dt, type, sizeof(int) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(dq, qtab, sizeof(double) * nspec, cudaMemcpyHostToDevice);
  cudaMemset(drho, 0, sizeof(double) * m * nn);
  if (n > 0) updateDensity<<<(n + 255) / 256, 256>>>(drho, dr, dq, dt, m, nn, dx, dy, n);
  bad = ck(cudaDeviceSynchronize());
  cudaMemcpy(rho_out, drho, sizeof(double) * m * nn, cudaMemcpyDeviceToHost);
  cudaFree(dr); cudaFree(dt); cudaFree(dq); cudaFree(drho);
  return bad;
}

// solve_multigrid (Multigrid.cu:573) on host arrays; phi is the warm start and carries the
// Dirichlet values on its boundary.
RH_API int refh_solve(double* phi, const double* rho, int nx, int ny, int levels, double h, double omega) {
  double *dphi = nullptr, *drho = nullptr;
  if (ck(cudaMalloc(&dphi, sizeof(double) * nx * ny)) | ck(cudaMalloc(&drho, sizeof(double) * nx * ny))) return 1;
  cudaMemcpy(dphi, phi, sizeof(double) * nx * ny, cudaMemcpyHostToDevice);
  cudaMemcpy(drho, rho, sizeof(double) * nx * ny, cudaMemcpyHostToDevice);
  solve_multigrid(dphi, drho, nx, ny, levels, h, omega);
  int bad = ck(cudaDeviceSynchronize());
  cudaMemcpy(phi, dphi, sizeof(double) * nx * ny, cudaMemcpyDeviceToHost);
  cudaFree(dphi); cudaFree(drho);
  return bad;
}

// computeElectricField (kernels.cu:134); E out interleaved (Ex, Ey) per node.
RH_API int refh_efield(const double* phi, int m, int n, double dx, double dy, double* exy) {
  double* dphi = nullptr; double2* dE = nullptr;
  if (ck(cudaMalloc(&dphi, sizeof(double) * m * n)) | ck(cudaMalloc(&dE, sizeof(double2) * m * n))) return 1;
  cudaMemcpy(dphi, phi, sizeof(double) * m * n, cudaMemcpyHostToDevice);
  dim3 b(16, 16), g((m + 15) / 16, (n + 15) / 16);
  computeElectricField<<<g, b>>>(dE, dphi, m, n, dx, dy);
  int bad = ck(cudaDeviceSynchronize());
  cudaMemcpy(exy, dE, sizeof(double2) * m * n, cudaMemcpyDeviceToHost);
  cudaFree(dphi); cudaFree(dE);
  return bad;
}

// The kernels of Multigrid_embedded.cu (compiled from the reference's file with -rdc; it has
// no header), launched with the reference's 8x8 blocks (Multigrid_embedded.cu:162-163).
__global__ void smooth_redblack(double* phi, const double* rhs, const unsigned char* mask, const double* phi_bc,
                                int nx, int ny, double h2, int redblack);
__global__ void residual_kernel(const double* phi, const double* rhs, const unsigned char* mask,
                                const double* phi_bc, double* res, int nx, int ny, double h2i);
__global__ void restrict_kernel(const double* fine, double* coarse, const unsigned char* mask_fine,
                                unsigned char* mask_coarse, int nxf, int nyf, int nxc, int nyc);
__global__ void prolongate_add_kernel(const double* coarse, double* fine, const unsigned char* mask_fine, int nxf,
                                      int nyf, int nxc, int nyc);

// On host arrays of an nx*ny level and its (nx-1)/2+1 x (ny-1)/2+1 coarse level:
//   phi_sweep0    phi after smooth_redblack with redblack = 0 (the colour whose test the
//                 reference evaluates as intended; redblack = 1 updates every node at once)
//   res           residual_kernel of phi into a zeroed array
//   rhs_c, mask_c restrict_kernel of res into zeroed arrays
//   phi_prol      phi after prolongate_add_kernel of phi_c
RH_API int refh_emb_kernels(int nx, int ny, const double* phi, const double* rhs, const unsigned char* mask,
                            const double* bc, double h2, const double* phi_c, double* phi_sweep0, double* res,
                            double* rhs_c, unsigned char* mask_c, double* phi_prol) {
  const int nxc = (nx - 1) / 2 + 1, nyc = (ny - 1) / 2 + 1;
  const size_t N = (size_t)nx * ny, Nc = (size_t)nxc * nyc;
  double *dphi = nullptr, *drhs = nullptr, *dbc = nullptr, *dres = nullptr, *drc = nullptr, *dpc = nullptr;
  unsigned char *dm = nullptr, *dmc = nullptr;
  int bad = ck(cudaMalloc(&dphi, 8 * N)) | ck(cudaMalloc(&drhs, 8 * N)) | ck(cudaMalloc(&dbc, 8 * N)) |
            ck(cudaMalloc(&dres, 8 * N)) | ck(cudaMalloc(&drc, 8 * Nc)) | ck(cudaMalloc(&dpc, 8 * Nc)) |
            ck(cudaMalloc(&dm, N)) | ck(cudaMalloc(&dmc, Nc));
  if (bad) return 1;
  cudaMemcpy(drhs, rhs, 8 * N, cudaMemcpyHostToDevice);
  cudaMemcpy(dbc, bc, 8 * N, cudaMemcpyHostToDevice);
  cudaMemcpy(dm, mask, N, cudaMemcpyHostToDevice);
  cudaMemcpy(dpc, phi_c, 8 * Nc, cudaMemcpyHostToDevice);
  cudaMemset(dres, 0, 8 * N);
  cudaMemset(drc, 0, 8 * Nc);
  cudaMemset(dmc, 0, Nc);
  const dim3 t(8, 8), b((nx + 7) / 8, (ny + 7) / 8), bc2((nxc + 7) / 8, (nyc + 7) / 8);
  cudaMemcpy(dphi, phi, 8 * N, cudaMemcpyHostToDevice);
  smooth_redblack<<<b, t>>>(dphi, drhs, dm, dbc, nx, ny, h2, 0);
  bad |= ck(cudaDeviceSynchronize());
  cudaMemcpy(phi_sweep0, dphi, 8 * N, cudaMemcpyDeviceToHost);
  cudaMemcpy(dphi, phi, 8 * N, cudaMemcpyHostToDevice);
  residual_kernel<<<b, t>>>(dphi, drhs, dm, dbc, dres, nx, ny, 1.0 / h2);
  restrict_kernel<<<bc2, t>>>(dres, drc, dm, dmc, nx, ny, nxc, nyc);
  prolongate_add_kernel<<<b, t>>>(dpc, dphi, dm, nx, ny, nxc, nyc);
  bad |= ck(cudaDeviceSynchronize());
  cudaMemcpy(res, dres, 8 * N, cudaMemcpyDeviceToHost);
  cudaMemcpy(rhs_c, drc, 8 * Nc, cudaMemcpyDeviceToHost);
  cudaMemcpy(mask_c, dmc, Nc, cudaMemcpyDeviceToHost);
  cudaMemcpy(phi_prol, dphi, 8 * N, cudaMemcpyDeviceToHost);
  cudaFree(dphi); cudaFree(drhs); cudaFree(dbc); cudaFree(dres); cudaFree(drc); cudaFree(dpc);
  cudaFree(dm); cudaFree(dmc);
  return bad;
}

// Multigrid::vcycle (Multigrid_embedded.cu:159-188) re-sequenced on the reference's kernels:
// the class itself cannot be linked (its members are defined inside the class body of a .cu
// file with no header).  Level arrays as its constructor makes them (:119-146).  Runs `cycles`
// V-cycles from level 0 after `warmup` untimed ones and returns phi and the mean time per
// V-cycle (CUDA events on the legacy stream, as the class launches).  The second colour of
// its smoother updates every node at once (:22), so phi is what the reference computes, races
// included; only the time is meant to be compared.
namespace {
struct RefEmbLevel { int nx, ny; double *phi, *rhs, *res, *bc; unsigned char* mask; };
void ref_emb_vcycle(std::vector<RefEmbLevel>& Ls, int l, double h) {
  RefEmbLevel& L = Ls[l];
  const dim3 t(8, 8), b((L.nx + 7) / 8, (L.ny + 7) / 8);
  const double h2 = h * h * std::pow(2.0, l) * std::pow(2.0, l), h2i = 1.0 / h2;
  for (int k = 0; k < 2; ++k) {
    smooth_redblack<<<b, t>>>(L.phi, L.rhs, L.mask, L.bc, L.nx, L.ny, h2, 0);
    smooth_redblack<<<b, t>>>(L.phi, L.rhs, L.mask, L.bc, L.nx, L.ny, h2, 1);
  }
  if (l == (int)Ls.size() - 1) return;
  residual_kernel<<<b, t>>>(L.phi, L.rhs, L.mask, L.bc, L.res, L.nx, L.ny, h2i);
  RefEmbLevel& C = Ls[l + 1];
  const dim3 bc((C.nx + 7) / 8, (C.ny + 7) / 8);
  restrict_kernel<<<bc, t>>>(L.res, C.rhs, L.mask, C.mask, L.nx, L.ny, C.nx, C.ny);
  cudaMemset(C.phi, 0, sizeof(double) * C.nx * C.ny);
  ref_emb_vcycle(Ls, l + 1, h);
  prolongate_add_kernel<<<b, t>>>(C.phi, L.phi, L.mask, L.nx, L.ny, C.nx, C.ny);
  for (int k = 0; k < 2; ++k) {
    smooth_redblack<<<b, t>>>(L.phi, L.rhs, L.mask, L.bc, L.nx, L.ny, h2, 0);
    smooth_redblack<<<b, t>>>(L.phi, L.rhs, L.mask, L.bc, L.nx, L.ny, h2, 1);
  }
}
}  // namespace

RH_API int refh_emb_vcycles(int nx, int ny, int levels, double h, int warmup, int cycles, double* phi,
                            const double* rhs, const unsigned char* mask, const double* bc, float* ms_per_cycle) {
  std::vector<RefEmbLevel> Ls;
  int bad = 0;
  for (int l = 0, a = nx, b = ny; l < levels; ++l, a = (a - 1) / 2 + 1, b = (b - 1) / 2 + 1) {
    RefEmbLevel L{a, b, nullptr, nullptr, nullptr, nullptr, nullptr};
    const size_t N = (size_t)a * b;
    bad |= ck(cudaMalloc(&L.phi, 8 * N)) | ck(cudaMalloc(&L.rhs, 8 * N)) | ck(cudaMalloc(&L.res, 8 * N)) |
           ck(cudaMalloc(&L.bc, 8 * N)) | ck(cudaMalloc(&L.mask, N));
    if (bad) return 1;
    cudaMemset(L.phi, 0, 8 * N); cudaMemset(L.rhs, 0, 8 * N); cudaMemset(L.res, 0, 8 * N);
    cudaMemset(L.bc, 0, 8 * N); cudaMemset(L.mask, 0, N);
    Ls.push_back(L);
  }
  const size_t N = (size_t)nx * ny;
  cudaMemcpy(Ls[0].phi, phi, 8 * N, cudaMemcpyHostToDevice);
  cudaMemcpy(Ls[0].rhs, rhs, 8 * N, cudaMemcpyHostToDevice);
  cudaMemcpy(Ls[0].mask, mask, N, cudaMemcpyHostToDevice);
  cudaMemcpy(Ls[0].bc, bc, 8 * N, cudaMemcpyHostToDevice);
  for (int c = 0; c < warmup; ++c) ref_emb_vcycle(Ls, 0, h);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0); cudaEventCreate(&e1);
  cudaEventRecord(e0);
  for (int c = 0; c < cycles; ++c) ref_emb_vcycle(Ls, 0, h);
  cudaEventRecord(e1);
  bad |= ck(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  if (ms_per_cycle) *ms_per_cycle = cycles > 0 ? ms / cycles : 0.f;
  cudaMemcpy(phi, Ls[0].phi, 8 * N, cudaMemcpyDeviceToHost);
  bad |= ck(cudaGetLastError());
  cudaEventDestroy(e0); cudaEventDestroy(e1);
  for (auto& L : Ls) { cudaFree(L.phi); cudaFree(L.rhs); cudaFree(L.res); cudaFree(L.bc); cudaFree(L.mask); }
  return bad;
}

// One re-sequenced step of updateSimulationCUDA (main.cu:60-135) on host state.
// Species table: q[k], m[k] for k < nspec (species 0 is overwritten through change_species).
// Walls: nwalls segments (x1,y1,x2,y2).  On return: x, y, vx, vy hold the first *n_alive
// particles after the reference's own removal; hits/n_hits the pre-removal hit set of the
// last step (unordered, as produced by the atomic append); rho/phi/exy the grids.
RH_API int refh_steps(int nsteps, int n, double* x, double* y, double* vx, double* vy, int* type,
                      const double* q, const double* mass, int nspec, int m, int nn, double X,
                      double Y, const double* walls, int nwalls, double dt, double* phi_inout,
                      double* rho_out, double* exy_out, int* hits, int* n_hits, int* n_alive,
                      float* ms_per_step) {
  Particles2D particles(n > 0 ? n : 1);
  particles.change_species(0, mass[0], q[0]);
  for (int k = 1; k < nspec; ++k) particles.add_species(mass[k], q[k]);
  Grid2D grid(m, nn, X, Y);
  Boundaries2D boundaries((int)X, (int)Y, m, nn);
  for (int w = 0; w < nwalls; ++w) boundaries.add_wall(walls[4 * w], walls[4 * w + 1], walls[4 * w + 2], walls[4 * w + 3]);
  if (nwalls > 0) boundaries.compile_walls();
  {
    std::vector<double2> r(n), v(n);
    for (int i = 0; i < n; ++i) { r[i] = make_double2(x[i], y[i]); v[i] = make_double2(vx[i], vy[i]); }
    cudaMemcpy(particles.r, r.data(), sizeof(double2) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(particles.r_old, r.data(), sizeof(double2) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(particles.v, v.data(), sizeof(double2) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(particles.type, type, sizeof(int) * n, cudaMemcpyHostToDevice);
  }
  particles.last_alive = n;
  cudaMemcpy(grid.phi, phi_inout, sizeof(double) * m * nn, cudaMemcpyHostToDevice);

  const int tpb = 256;
  dim3 bd(16, 16), gd((grid.m + 15) / 16, (grid.n + 15) / 16);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0); cudaEventCreate(&e1);
  cudaDeviceSynchronize();
  cudaEventRecord(e0);
  for (int s = 0; s < nsteps; ++s) {
    const int pb = (particles.last_alive + tpb - 1) / tpb;
    if (particles.last_alive > 0)
      update_coordinates<<<pb, tpb>>>(particles.r, particles.r_old, particles.v, particles.last_alive, dt);
    cudaMemset(particles.collision_counter, 0, sizeof(int));
    cudaMemset(particles.collided_indices, -1, particles.last_alive * sizeof(int));
    if (particles.last_alive > 0 && boundaries.wall_count > 0)
      detect_intersections<<<pb, tpb>>>(particles.r_old, particles.r, boundaries.d_walls,
                                        particles.collided_indices, particles.collision_counter,
                                        particles.last_alive, boundaries.wall_count);
    if (s == nsteps - 1 && hits) {
      int h = 0;
      cudaMemcpy(&h, particles.collision_counter, sizeof(int), cudaMemcpyDeviceToHost);
      *n_hits = h;
      if (h > 0) cudaMemcpy(hits, particles.collided_indices, sizeof(int) * h, cudaMemcpyDeviceToHost);
    }
    particles.removeCollidedParticles();
    cudaMemset(grid.rho, 0, grid.m * grid.n * sizeof(double));
    const int pb2 = (particles.last_alive + tpb - 1) / tpb;
    if (particles.last_alive > 0)
      updateDensity<<<pb2, tpb>>>(grid.rho, particles.r, particles.q, particles.type, grid.m, grid.n,
                                  grid.dx, grid.dy, particles.last_alive);
    solve_multigrid(grid.phi, grid.rho, grid.m, grid.n, 5, grid.dx);
    computeElectricField<<<gd, bd>>>(grid.E, grid.phi, grid.m, grid.n, grid.dx, grid.dy);
    if (particles.last_alive > 0)
      updateParticleVelocities<<<pb2, tpb>>>(particles.v, grid.E, particles.r, particles.type, particles.q,
                                             particles.m, particles.last_alive, grid.dx, grid.dy, grid.m,
                                             grid.n, dt);
  }
  cudaEventRecord(e1);
  int bad = ck(cudaDeviceSynchronize());
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  if (ms_per_step) *ms_per_step = nsteps > 0 ? ms / nsteps : 0.f;
  const int na = particles.last_alive;
  *n_alive = na;
  std::vector<double2> r(na), v(na);
  cudaMemcpy(r.data(), particles.r, sizeof(double2) * na, cudaMemcpyDeviceToHost);
  cudaMemcpy(v.data(), particles.v, sizeof(double2) * na, cudaMemcpyDeviceToHost);
  cudaMemcpy(type, particles.type, sizeof(int) * na, cudaMemcpyDeviceToHost);
  for (int i = 0; i < na; ++i) { x[i] = r[i].x; y[i] = r[i].y; vx[i] = v[i].x; vy[i] = v[i].y; }
  cudaMemcpy(phi_inout, grid.phi, sizeof(double) * m * nn, cudaMemcpyDeviceToHost);
  if (rho_out) cudaMemcpy(rho_out, grid.rho, sizeof(double) * m * nn, cudaMemcpyDeviceToHost);
  if (exy_out) cudaMemcpy(exy_out, grid.E, sizeof(double2) * m * nn, cudaMemcpyDeviceToHost);
  cudaEventDestroy(e0); cudaEventDestroy(e1);
  if (boundaries.d_walls) cudaFree(boundaries.d_walls);
  if (boundaries.d_walls_int) cudaFree(boundaries.d_walls_int);
  return bad;
}

// elasticCollisions (mcc.cu:114-150) on host state: one call on n particles of species 0.
// cuRAND is seeded from time(NULL) inside the reference, so only statistics are comparable.
RH_API int refh_elastic(int n, double* vx, double* vy, double mass, double density, double dt,
                        const double* xs_e, const double* xs_s, int nxs) {
  Particles2D particles(n);
  particles.change_species(0, mass, 0.0);
  std::vector<double2> v(n);
  for (int i = 0; i < n; ++i) v[i] = make_double2(vx[i], vy[i]);
  cudaMemcpy(particles.v, v.data(), sizeof(double2) * n, cudaMemcpyHostToDevice);
  cudaMemset(particles.type, 0, sizeof(int) * n);
  particles.last_alive = n;
  cross_sections xs;
  std::memset(&xs, 0, sizeof(xs));
  cudaMalloc(&xs.energies, sizeof(double) * nxs);
  cudaMalloc(&xs.sigmas, sizeof(double) * nxs);
  cudaMemcpy(xs.energies, xs_e, sizeof(double) * nxs, cudaMemcpyHostToDevice);
  cudaMemcpy(xs.sigmas, xs_s, sizeof(double) * nxs, cudaMemcpyHostToDevice);
  xs.size = nxs;
  elasticCollisions(particles, density, dt, xs);
  int bad = ck(cudaDeviceSynchronize());
  cudaMemcpy(v.data(), particles.v, sizeof(double2) * n, cudaMemcpyDeviceToHost);
  for (int i = 0; i < n; ++i) { vx[i] = v[i].x; vy[i] = v[i].y; }
  cudaFree(xs.energies); cudaFree(xs.sigmas);
  return bad;
}

// Timing of the reference's four particle kernels of a step on n particles of the reference's
// FP64 AoS state (Particles2D), on an m x nn grid over X x Y with the four domain walls
// (main.cu:190-193), in the order and launch shape of updateSimulationCUDA (main.cu:60-127):
//   ms_out[0] update_coordinates (kernels.cu:8)
//   ms_out[1] the hit-list memsets (main.cu:72-73) + detect_intersections (collisions.cu:7)
//   ms_out[2] the rho memset (main.cu:93) + updateDensity (kernels.cu:26)
//   ms_out[3] updateParticleVelocities (kernels.cu:71)
// each averaged over `iters` launches after one untimed round (CUDA events, legacy stream).
// The state is filled on the device: positions uniform in the domain, velocities uniform in
// [-vmax_s, vmax_s] for species s = type (half the particles each, interleaved at random), as
// the reference holds particles unsorted.  Removal and the field solve are not timed.
namespace {
__device__ __forceinline__ unsigned long long rh_mix(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double rh_u01(unsigned long long z) { return (double)(z >> 11) * (1.0 / 9007199254740992.0); }
__global__ void rh_fill_state(double2* r, double2* r_old, double2* v, int* type, int n, double X, double Y,
                              double vmax0, double vmax1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long b = 4ull * (unsigned long long)i;
  const int t = (int)(rh_mix(b) & 1ull);
  const double vm = t ? vmax1 : vmax0;
  const double2 p = make_double2(X * rh_u01(rh_mix(b + 1)), Y * rh_u01(rh_mix(b + 2)));
  const unsigned long long zv = rh_mix(b + 3);
  r[i] = p;
  r_old[i] = p;
  v[i] = make_double2(vm * (2.0 * rh_u01(zv) - 1.0), vm * (2.0 * rh_u01(rh_mix(zv)) - 1.0));
  type[i] = t;
}
}  // namespace

RH_API int refh_particle_kernels_timed(int n, int m, int nn, double X, double Y, double dt, const double* q,
                                       const double* mass, double vmax0, double vmax1, int iters, float* ms_out) {
  if (n <= 0 || iters <= 0) return 1;
  Particles2D particles(n);
  particles.change_species(0, mass[0], q[0]);
  particles.add_species(mass[1], q[1]);
  Grid2D grid(m, nn, X, Y);
  Boundaries2D boundaries((int)X, (int)Y, m, nn);
  boundaries.add_wall(0, 0, X, 0);
  boundaries.add_wall(X, 0, X, Y);
  boundaries.add_wall(X, Y, 0, Y);
  boundaries.add_wall(0, Y, 0, 0);
  boundaries.compile_walls();
  const int tpb = 256, pb = (n + tpb - 1) / tpb;
  rh_fill_state<<<pb, tpb>>>(particles.r, particles.r_old, particles.v, particles.type, n, X, Y, vmax0, vmax1);
  cudaMemset(grid.phi, 0, sizeof(double) * m * nn);
  cudaMemset(grid.E, 0, sizeof(double2) * m * nn);
  particles.last_alive = n;
  int bad = ck(cudaDeviceSynchronize());
  if (bad) return bad;
  cudaEvent_t ev[5];
  for (auto& e : ev) cudaEventCreate(&e);
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int it = 0; it <= iters; ++it) {
    cudaEventRecord(ev[0]);
    update_coordinates<<<pb, tpb>>>(particles.r, particles.r_old, particles.v, n, dt);
    cudaEventRecord(ev[1]);
    cudaMemset(particles.collision_counter, 0, sizeof(int));
    cudaMemset(particles.collided_indices, -1, n * sizeof(int));
    detect_intersections<<<pb, tpb>>>(particles.r_old, particles.r, boundaries.d_walls, particles.collided_indices,
                                      particles.collision_counter, n, boundaries.wall_count);
    cudaEventRecord(ev[2]);
    cudaMemset(grid.rho, 0, grid.m * grid.n * sizeof(double));
    updateDensity<<<pb, tpb>>>(grid.rho, particles.r, particles.q, particles.type, grid.m, grid.n, grid.dx, grid.dy,
                               n);
    cudaEventRecord(ev[3]);
    updateParticleVelocities<<<pb, tpb>>>(particles.v, grid.E, particles.r, particles.type, particles.q, particles.m,
                                          n, grid.dx, grid.dy, grid.m, grid.n, dt);
    cudaEventRecord(ev[4]);
    bad |= ck(cudaEventSynchronize(ev[4]));
    if (it == 0) continue;
    for (int k = 0; k < 4; ++k) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
      acc[k] += ms;
    }
  }
  for (int k = 0; k < 4; ++k) ms_out[k] = acc[k] / iters;
  bad |= ck(cudaGetLastError());
  for (auto& e : ev) cudaEventDestroy(e);
  if (boundaries.d_walls) cudaFree(boundaries.d_walls);
  if (boundaries.d_walls_int) cudaFree(boundaries.d_walls_int);
  return bad;
}
