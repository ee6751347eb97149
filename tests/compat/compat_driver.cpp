// compat_driver.cpp — a headless program written against the reference's own headers
// (grid.cuh, particles.cuh, boundaries.h, Multigrid.hpp, mcc.hpp, diagnostics.h and
// updateSimulationCUDA from main.cu) and linked to libpic_b200.so, used by
// tests/test_gpu_compat.py.  It follows main.cu:186-238's set-up sequence (construct,
// add species, add/compile walls, cudaMemcpy the particle arrays, set last_alive) and
// then calls the entry point under test.
//
// I/O: the input file is a sequence of records (int64 byte count, raw bytes) in the order
// each mode reads them; the output file is written the same way.
//   step    in: i32[m, nspec, nwalls, steps, max_particles, calls], f64[X, Y, dt], f64 q[S],
//               f64 m[S], f64 walls[4W], f64 x, y, vx, vy [N], i32 type[N], f64 phi0[m*m]
//           out: i32[last_alive, collision_counter], f64 r[2A], r_old[2A], v[2A], i32 type[A],
//               i32 collided[K], f64 rho[m*m], phi[m*m], E[2*m*m], f64 timing[4]
//   remove  in: i32[max_particles], f64 r[2N], r_old[2N], v[2N], i32 type[N], i32 idx[K]
//           out: i32[last_alive], f64 r, r_old, v, i32 type
//   elastic in: i32[calls], f64[density, dt], f64 m[S], f64 q[S], f64 v[2N], i32 type[N]
//           (argv[4] = cross-section text file)
//           out: f64 v[2N], v_abs[N], energy[N], crs[N], f64 table energies, sigmas
//   solve   in: i32[n, levels], f64[h, omega], f64 phi0[n*n], rho[n*n]
//           out: f64 phi[n*n]
//   embedded in: i32[nx, ny, levels, cycles], f64[h], f64 phi0, rhs, phi_bc [nx*ny], u8 mask
//           out: f64 phi[nx*ny] after `cycles` vcycle(0) calls, level 1's f64 rhs and u8 mask
//   kernels in: i32[m], f64[dx, dt], f64 q[S], m[S], walls[4W], r[2N], v[2N], i32 type[N],
//               f64 phi[m*m], f64 table energies, sigmas
//           (the reference's kernel sequence main.cu:64-127 plus kernels.cu:196-274, one
//           host wrapper per kernel)
//           out: f64 r[2N], r_old[2N], i32 hits[K], f64 rho[m*m], E[2*m*m], v[2N],
//               v_abs[N], energy[N], crs[N], f32 pos[2N]
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include "compat/Multigrid.hpp"
#include "compat/Multigrid_embedded.hpp"
#include "compat/boundaries.h"
#include "compat/collisions.cuh"
#include "compat/diagnostics.h"
#include "compat/grid.cuh"
#include "compat/kernels.cuh"
#include "compat/mcc.hpp"
#include "compat/particles.cuh"
#include "compat/pic_step.h"

namespace {

struct In {
  FILE* f;
  template <class T>
  std::vector<T> rec() {
    int64_t nb = 0;
    if (fread(&nb, 8, 1, f) != 1 || nb % (int64_t)sizeof(T)) throw std::runtime_error("bad record");
    std::vector<T> v(nb / sizeof(T));
    if (nb && fread(v.data(), 1, nb, f) != (size_t)nb) throw std::runtime_error("short record");
    return v;
  }
};

struct Out {
  FILE* f;
  template <class T>
  void rec(const T* p, size_t n) {
    const int64_t nb = (int64_t)(n * sizeof(T));
    fwrite(&nb, 8, 1, f);
    if (n) fwrite(p, 1, nb, f);
  }
  template <class T>
  void rec(const std::vector<T>& v) { rec(v.data(), v.size()); }
};

void ck(cudaError_t e) {
  if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
}

template <class T>
std::vector<T> d2h(const T* d, size_t n) {
  std::vector<T> h(n);
  if (n) ck(cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost));
  return h;
}

template <class T>
void h2d(T* d, const std::vector<T>& h) {
  if (!h.empty()) ck(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
}

std::vector<double> interleave(const std::vector<double>& a, const std::vector<double>& b) {
  std::vector<double> o(2 * a.size());
  for (size_t i = 0; i < a.size(); ++i) {
    o[2 * i] = a[i];
    o[2 * i + 1] = b[i];
  }
  return o;
}

void set_species(Particles2D& p, const std::vector<double>& q, const std::vector<double>& m) {
  p.change_species(0, m[0], q[0]);
  for (size_t s = 1; s < q.size(); ++s) p.add_species(m[s], q[s]);
}

void run_step(In& in, Out& out) {
  const auto hi = in.rec<int32_t>();
  const int gm = hi[0], nspec = hi[1], nwalls = hi[2], steps = hi[3], maxp = hi[4], calls = hi[5];
  const auto hd = in.rec<double>();
  const auto q = in.rec<double>(), m = in.rec<double>(), walls = in.rec<double>();
  const auto x = in.rec<double>(), y = in.rec<double>(), vx = in.rec<double>(), vy = in.rec<double>();
  const auto type = in.rec<int32_t>();
  const auto phi0 = in.rec<double>();
  const int n = (int)x.size();
  if ((int)q.size() != nspec || (int)walls.size() != 4 * nwalls) throw std::runtime_error("bad header");

  Particles2D particles(maxp);
  set_species(particles, q, m);
  Grid2D grid(gm, gm, hd[0], hd[1]);
  Boundaries2D boundaries((int)hd[0], (int)hd[1], gm, gm);
  for (int w = 0; w < nwalls; ++w) boundaries.add_wall(walls[4 * w], walls[4 * w + 1], walls[4 * w + 2], walls[4 * w + 3]);
  boundaries.compile_walls();
  const auto pos = interleave(x, y);
  h2d((double*)particles.r, pos);
  h2d((double*)particles.r_old, pos);
  h2d((double*)particles.v, interleave(vx, vy));
  h2d(particles.type, type);
  h2d(grid.phi, phi0);
  particles.last_alive = n;

  SimulationTiming timing;
  int step = 1;
  for (int c = 0; c < calls; ++c) updateSimulationCUDA(particles, grid, boundaries, step, hd[2], steps, timing);

  const int a = particles.last_alive;
  int k = 0;
  ck(cudaMemcpy(&k, particles.collision_counter, sizeof(int), cudaMemcpyDeviceToHost));
  const int32_t head[2] = {a, k};
  out.rec(head, 2);
  out.rec(d2h((const double*)particles.r, 2 * (size_t)a));
  out.rec(d2h((const double*)particles.r_old, 2 * (size_t)a));
  out.rec(d2h((const double*)particles.v, 2 * (size_t)a));
  out.rec(d2h(particles.type, a));
  out.rec(d2h(particles.collided_indices, k));
  const size_t nodes = (size_t)gm * gm;
  out.rec(d2h(grid.rho, nodes));
  out.rec(d2h(grid.phi, nodes));
  out.rec(d2h((const double*)grid.E, 2 * nodes));
  const double t[4] = {timing.coordinate_update_us, timing.particle_removal, timing.solver_us, timing.total_us};
  out.rec(t, 4);
}

void run_remove(In& in, Out& out) {
  const int maxp = in.rec<int32_t>()[0];
  const auto r = in.rec<double>(), r_old = in.rec<double>(), v = in.rec<double>();
  const auto type = in.rec<int32_t>(), idx = in.rec<int32_t>();
  Particles2D p(maxp);
  h2d((double*)p.r, r);
  h2d((double*)p.r_old, r_old);
  h2d((double*)p.v, v);
  h2d(p.type, type);
  h2d(p.collided_indices, idx);
  const int k = (int)idx.size();
  ck(cudaMemcpy(p.collision_counter, &k, sizeof(int), cudaMemcpyHostToDevice));
  p.last_alive = (int)type.size();
  p.removeCollidedParticles();
  const int32_t a = p.last_alive;
  out.rec(&a, 1);
  out.rec(d2h((const double*)p.r, 2 * (size_t)a));
  out.rec(d2h((const double*)p.r_old, 2 * (size_t)a));
  out.rec(d2h((const double*)p.v, 2 * (size_t)a));
  out.rec(d2h(p.type, a));
}

void run_elastic(In& in, Out& out, const std::string& table) {
  const int calls = in.rec<int32_t>()[0];
  const auto hd = in.rec<double>();
  const auto m = in.rec<double>(), q = in.rec<double>(), v = in.rec<double>();
  const auto type = in.rec<int32_t>();
  const int n = (int)type.size();
  Particles2D p(n);
  set_species(p, q, m);
  h2d((double*)p.v, v);
  h2d(p.type, type);
  p.last_alive = n;
  auto css = read_cross_section(table);
  cross_sections xs{};
  ck(cudaMalloc(&xs.energies, css.first.size() * sizeof(double)));
  ck(cudaMalloc(&xs.sigmas, css.second.size() * sizeof(double)));
  h2d(xs.energies, css.first);
  h2d(xs.sigmas, css.second);
  xs.size = (int)css.first.size();
  for (int c = 0; c < calls; ++c) elasticCollisions(p, hd[0], hd[1], xs);
  out.rec(d2h((const double*)p.v, 2 * (size_t)n));
  out.rec(d2h(p.v_abs, n));
  out.rec(d2h(p.energy, n));
  out.rec(d2h(p.crs, n));
  out.rec(css.first);
  out.rec(css.second);
  cudaFree(xs.energies);
  cudaFree(xs.sigmas);
}

void run_solve(In& in, Out& out) {
  const auto hi = in.rec<int32_t>();
  const auto hd = in.rec<double>();
  const auto phi0 = in.rec<double>(), rho = in.rec<double>();
  const int n = hi[0];
  double *phi_d = nullptr, *rho_d = nullptr;
  ck(cudaMalloc(&phi_d, phi0.size() * 8));
  ck(cudaMalloc(&rho_d, rho.size() * 8));
  h2d(phi_d, phi0);
  h2d(rho_d, rho);
  solve_multigrid(phi_d, rho_d, n, n, hi[1], hd[0], hd[1]);
  out.rec(d2h(phi_d, (size_t)n * n));
  cudaFree(phi_d);
  cudaFree(rho_d);
}

// The reference's embedded-boundary class (Multigrid_embedded.cu:106-190) used as its
// vcycle is written to be used: fill level 0, call vcycle(0) repeatedly.
void run_embedded(In& in, Out& out) {
  const auto hi = in.rec<int32_t>();
  const double h = in.rec<double>()[0];
  const auto phi0 = in.rec<double>(), rhs = in.rec<double>(), bc = in.rec<double>();
  const auto mask = in.rec<uint8_t>();
  const int nx = hi[0], ny = hi[1], levels = hi[2], cycles = hi[3];
  Multigrid mg(nx, ny, levels, h);
  h2d(mg.levels[0].phi, phi0);
  h2d(mg.levels[0].rhs, rhs);
  h2d(mg.levels[0].phi_bc, bc);
  h2d(mg.levels[0].mask, mask);
  for (int c = 0; c < cycles; ++c) mg.vcycle(0);
  ck(cudaDeviceSynchronize());
  const MGLevel& L1 = mg.levels[levels > 1 ? 1 : 0];
  out.rec(d2h(mg.levels[0].phi, (size_t)nx * ny));
  out.rec(d2h(L1.rhs, (size_t)L1.nx * L1.ny));
  out.rec(d2h(L1.mask, (size_t)L1.nx * L1.ny));
}

void run_kernels(In& in, Out& out) {
  const int gm = in.rec<int32_t>()[0];
  const auto hd = in.rec<double>();
  const auto q = in.rec<double>(), m = in.rec<double>(), walls = in.rec<double>();
  const auto r = in.rec<double>(), v = in.rec<double>();
  const auto type = in.rec<int32_t>();
  const auto phi = in.rec<double>(), xe = in.rec<double>(), xv = in.rec<double>();
  const int n = (int)type.size(), nw = (int)walls.size() / 4, S = (int)q.size();
  const double dx = hd[0], dt = hd[1];
  Particles2D p(n);
  set_species(p, q, m);
  Grid2D grid(gm, gm, dx * (gm - 1), dx * (gm - 1));
  Boundaries2D b(1, 1, gm, gm);
  for (int w = 0; w < nw; ++w) b.add_wall(walls[4 * w], walls[4 * w + 1], walls[4 * w + 2], walls[4 * w + 3]);
  b.compile_walls();
  h2d((double*)p.r, r);
  h2d((double*)p.v, v);
  h2d(p.type, type);
  h2d(grid.phi, phi);
  double *dxe = nullptr, *dxv = nullptr;
  float2* fpos = nullptr;
  ck(cudaMalloc(&dxe, xe.size() * 8));
  ck(cudaMalloc(&dxv, xv.size() * 8));
  ck(cudaMalloc(&fpos, (size_t)n * sizeof(float2) + 8));
  h2d(dxe, xe);
  h2d(dxv, xv);
  (void)S;
  update_coordinates(p.r, p.r_old, p.v, n, dt);
  ck(cudaMemset(p.collision_counter, 0, sizeof(int)));
  detect_intersections(p.r_old, p.r, b.d_walls, p.collided_indices, p.collision_counter, n, b.wall_count);
  ck(cudaMemset(grid.rho, 0, (size_t)gm * gm * 8));
  updateDensity(grid.rho, p.r, p.q, p.type, gm, gm, grid.dx, grid.dy, n);
  computeElectricField(grid.E, grid.phi, gm, gm, grid.dx, grid.dy);
  updateParticleVelocities(p.v, grid.E, p.r, p.type, p.q, p.m, n, grid.dx, grid.dy, gm, gm, dt);
  compute_speeds_and_energies(p.v, p.v_abs, p.energy, p.type, p.m, n);
  interpolate_cross_sections(p.energy, dxe, dxv, p.crs, (int)xe.size(), n);
  convertPositionsToFloat(p.r, fpos, n);
  ck(cudaDeviceSynchronize());
  int k = 0;
  ck(cudaMemcpy(&k, p.collision_counter, sizeof(int), cudaMemcpyDeviceToHost));
  out.rec(d2h((const double*)p.r, 2 * (size_t)n));
  out.rec(d2h((const double*)p.r_old, 2 * (size_t)n));
  out.rec(d2h(p.collided_indices, k));
  out.rec(d2h(grid.rho, (size_t)gm * gm));
  out.rec(d2h((const double*)grid.E, 2 * (size_t)gm * gm));
  out.rec(d2h((const double*)p.v, 2 * (size_t)n));
  out.rec(d2h(p.v_abs, n));
  out.rec(d2h(p.energy, n));
  out.rec(d2h(p.crs, n));
  out.rec(d2h((const float*)fpos, 2 * (size_t)n));
  cudaFree(dxe);
  cudaFree(dxv);
  cudaFree(fpos);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s step|remove|elastic|solve|kernels <in> <out> [table]\n", argv[0]);
    return 2;
  }
  const std::string mode = argv[1];
  FILE* fi = fopen(argv[2], "rb");
  FILE* fo = fopen(argv[3], "wb");
  if (!fi || !fo) {
    fprintf(stderr, "cannot open files\n");
    return 2;
  }
  In in{fi};
  Out out{fo};
  try {
    if (mode == "step") run_step(in, out);
    else if (mode == "remove") run_remove(in, out);
    else if (mode == "elastic") run_elastic(in, out, argc > 4 ? argv[4] : "");
    else if (mode == "solve") run_solve(in, out);
    else if (mode == "kernels") run_kernels(in, out);
    else if (mode == "embedded") run_embedded(in, out);
    else throw std::runtime_error("unknown mode");
  } catch (const std::exception& e) {
    fprintf(stderr, "compat_driver: %s\n", e.what());
    return 1;
  }
  fclose(fi);
  fclose(fo);
  return 0;
}
