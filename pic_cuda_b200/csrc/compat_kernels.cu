// compat_kernels.cu — the reference's individual step kernels (kernels.cuh, collisions.cuh)
// as host functions over FP64 AoS device arrays, for callers that drive the step kernel by
// kernel.  The fused engine does not use them; they share its conventions: node-centred
// row-major grid j*m + i, CIC weights, skip outside [0, m-2] x [0, n-2].
#include <cstdint>

#include "compat/collisions.cuh"
#include "compat/kernels.cuh"

namespace {

constexpr int kThreads = 256;

inline int blocks(int64_t n) { return (int)((n + kThreads - 1) / kThreads); }

struct Cic {
  int i0, j0;
  double w00, w10, w01, w11;
  bool inside;
};

__device__ __forceinline__ Cic cic(double2 p, double dx, double dy, int m, int n) {
  Cic c;
  const double X = p.x / dx, Y = p.y / dy;
  c.i0 = (int)floor(X);
  c.j0 = (int)floor(Y);
  c.inside = c.i0 >= 0 && c.i0 < m - 1 && c.j0 >= 0 && c.j0 < n - 1;
  const double wx = X - c.i0, wy = Y - c.j0;
  c.w00 = (1.0 - wx) * (1.0 - wy);
  c.w10 = wx * (1.0 - wy);
  c.w01 = (1.0 - wx) * wy;
  c.w11 = wx * wy;
  return c;
}

__global__ void drift_kernel(double2* r, double2* r_old, const double2* v, int n, double dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double2 p = r[i], u = v[i];
  r_old[i] = p;
  // product and sum rounded separately (no fused multiply-add): the position, and with it
  // every wall decision taken on it, is the one an FP64 CPU evaluation gives
  r[i] = make_double2(__dadd_rn(p.x, __dmul_rn(u.x, dt)), __dadd_rn(p.y, __dmul_rn(u.y, dt)));
}

__global__ void deposit_kernel(double* rho, const double2* r, const double* q, const int* type, int m, int n,
                               double dx, double dy, int np) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const Cic c = cic(r[i], dx, dy, m, n);
  if (!c.inside) return;
  const double qq = q[type[i]];
  double* base = rho + (int64_t)c.j0 * m + c.i0;
  atomicAdd(base, qq * c.w00);
  atomicAdd(base + 1, qq * c.w10);
  atomicAdd(base + m, qq * c.w01);
  atomicAdd(base + m + 1, qq * c.w11);
}

__global__ void kick_kernel(double2* v, const double2* E, const double2* r, const int* type, const double* q,
                            const double* mass, int np, double dx, double dy, int m, int n, double dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const Cic c = cic(r[i], dx, dy, m, n);
  if (!c.inside) return;
  const int t = type[i];
  const double k = q[t] * (1.0 / mass[t]) * dt;
  const double2* e = E + (int64_t)c.j0 * m + c.i0;
  const double2 a = e[0], b = e[1], d = e[m], f = e[m + 1];
  const double ex = c.w00 * a.x + c.w10 * b.x + c.w01 * d.x + c.w11 * f.x;
  const double ey = c.w00 * a.y + c.w10 * b.y + c.w01 * d.y + c.w11 * f.y;
  double2 u = v[i];
  u.x += k * ex;
  u.y += k * ey;
  v[i] = u;
}

__global__ void efield_kernel(double2* E, const double* phi, int m, int n, double dx, double dy) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= (int64_t)m * n) return;
  const int i = (int)(c % m), j = (int)(c / m);
  double ex, ey;
  if (i == 0) ex = -(phi[c + 1] - phi[c]) / dx;
  else if (i == m - 1) ex = -(phi[c] - phi[c - 1]) / dx;
  else ex = -(phi[c + 1] - phi[c - 1]) / (2.0 * dx);
  if (j == 0) ey = -(phi[c + m] - phi[c]) / dy;
  else if (j == n - 1) ey = -(phi[c] - phi[c - m]) / dy;
  else ey = -(phi[c + m] - phi[c - m]) / (2.0 * dy);
  E[c] = make_double2(ex, ey);
}

__global__ void energy_kernel(const double2* v, double* vabs, double* energy, const int* type, const double* mass,
                              int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double2 u = v[i];
  const double s2 = u.x * u.x + u.y * u.y;
  vabs[i] = sqrt(s2);
  energy[i] = 0.5 * mass[type[i]] * s2 * 6.25e18;
}

__global__ void xs_kernel(const double* energy, const double* xe, const double* xv, double* out, int len, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double E = energy[i];
  if (E <= xe[0]) {
    out[i] = xv[0];
    return;
  }
  if (E >= xe[len - 1]) {
    out[i] = xv[len - 1];
    return;
  }
  int lo = 0, hi = len - 1;  // xe[lo] < E < xe[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (E < xe[mid]) hi = mid;
    else lo = mid;
  }
  const double t = (E - xe[lo]) / (xe[lo + 1] - xe[lo]);
  out[i] = xv[lo] + t * (xv[lo + 1] - xv[lo]);
}

__global__ void to_float_kernel(const double2* p, float2* f, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) f[i] = make_float2((float)p[i].x, (float)p[i].y);
}

// Parametric segment test, every product and difference rounded on its own (no fused
// multiply-add), so the decision is the one an FP64 CPU evaluation of the same formula makes.
__device__ __forceinline__ bool crosses(double X1, double Y1, double X2, double Y2, double4 w) {
  const double ax = __dsub_rn(w.z, w.x), ay = __dsub_rn(w.w, w.y);
  const double px = __dsub_rn(X2, X1), py = __dsub_rn(Y2, Y1);
  const double sx = __dsub_rn(X1, w.x), sy = __dsub_rn(Y1, w.y);
  const double den = __dsub_rn(__dmul_rn(ay, px), __dmul_rn(ax, py));
  if (den == 0.0) return false;
  const double ua = __dsub_rn(__dmul_rn(ax, sy), __dmul_rn(ay, sx)) / den;
  const double ub = __dsub_rn(__dmul_rn(px, sy), __dmul_rn(py, sx)) / den;
  return ua >= 0.0 && ua <= 1.0 && ub >= 0.0 && ub <= 1.0;
}

__global__ void walls_kernel(const double2* p0, const double2* p1, const double4* walls, int* idx, int* count, int n,
                             int nw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool hit = false;
  if (i < n) {
    const double2 a = p0[i], b = p1[i];
    for (int k = 0; k < nw && !hit; ++k) hit = crosses(a.x, a.y, b.x, b.y, walls[k]);
  }
  // one atomic per warp
  const unsigned m = __ballot_sync(0xffffffffu, hit);
  if (!m) return;
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == __ffs(m) - 1) base = atomicAdd(count, __popc(m));
  base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
  if (hit) idx[base + __popc(m & ((1u << lane) - 1u))] = i;
}

}  // namespace

void update_coordinates(double2* positions_new, double2* positions_old, const double2* velocities,
                        const int num_particles, const double dt, cudaStream_t stream) {
  if (num_particles <= 0) return;
  drift_kernel<<<blocks(num_particles), kThreads, 0, stream>>>(positions_new, positions_old, velocities,
                                                               num_particles, dt);
}

void updateDensity(double* d_rho, const double2* d_positions, const double* d_q_type, const int* d_part_type, int m,
                   int n, double dx, double dy, int last_alive, cudaStream_t stream) {
  if (last_alive <= 0) return;
  deposit_kernel<<<blocks(last_alive), kThreads, 0, stream>>>(d_rho, d_positions, d_q_type, d_part_type, m, n, dx,
                                                              dy, last_alive);
}

void updateParticleVelocities(double2* velocities, const double2* E_grid, const double2* positions,
                              const int* part_types, const double* charge, const double* mass, int num_particles,
                              double dx, double dy, int m, int n, double dt, cudaStream_t stream) {
  if (num_particles <= 0) return;
  kick_kernel<<<blocks(num_particles), kThreads, 0, stream>>>(velocities, E_grid, positions, part_types, charge,
                                                              mass, num_particles, dx, dy, m, n, dt);
}

void computeElectricField(double2* E_grid, const double* phi, int m, int n, double dx, double dy,
                          cudaStream_t stream) {
  if (m < 2 || n < 2) return;
  efield_kernel<<<blocks((int64_t)m * n), kThreads, 0, stream>>>(E_grid, phi, m, n, dx, dy);
}

void compute_speeds_and_energies(const double2* V, double* V_abs, double* energies, const int* type_arr,
                                 const double* m_type, const int N, cudaStream_t stream) {
  if (N <= 0) return;
  energy_kernel<<<blocks(N), kThreads, 0, stream>>>(V, V_abs, energies, type_arr, m_type, N);
}

void interpolate_cross_sections(const double* energies, const double* xs_energy, const double* xs_values,
                                double* output, const int xs_len, const int N, cudaStream_t stream) {
  if (N <= 0 || xs_len < 1) return;
  xs_kernel<<<blocks(N), kThreads, 0, stream>>>(energies, xs_energy, xs_values, output, xs_len, N);
}

void convertPositionsToFloat(const double2* d_positions, float2* f_positions, int count, cudaStream_t stream) {
  if (count <= 0) return;
  to_float_kernel<<<blocks(count), kThreads, 0, stream>>>(d_positions, f_positions, count);
}

void detect_intersections(const double2* p0, const double2* p1, const double4* walls, int* collided_indices,
                          int* collision_counter, const int num_particles, const int num_walls,
                          cudaStream_t stream) {
  if (num_particles <= 0 || num_walls <= 0) return;
  walls_kernel<<<blocks(num_particles), kThreads, 0, stream>>>(p0, p1, walls, collided_indices, collision_counter,
                                                               num_particles, num_walls);
}
