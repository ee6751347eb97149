// pic_oracle.cpp — FP64 CPU oracle of the 2D electrostatic PIC step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker, not the product: only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm may load the
// library built from it.  The product (pic_cuda_b200) never links or calls it.
//
// It restates, in plain FP64 C++ (OpenMP over particles and grid rows), the reference's
// step as driven by updateSimulationCUDA (main.cu:60-135) of dimad285/PIC_CUDA:
//   drift                 kernels.cu:8-23
//   wall segment test     collisions.cu:7-54  (ref-faithful, absolute EPSILON 1e-10)
//   box absorption        the region updateDensity deposits from (kernels.cu:53)
//   particle removal      particles.cu:217-262, intended semantics (remove exactly the hit
//                         set; the reference's copy can move hit tail particles into holes
//                         and fills at most 256 holes per step, particles.cu:63-66, 255)
//   CIC deposit           kernels.cu:26-69 (charge per node, skip rule)
//   multigrid solve       Multigrid.cu:192-642 (red-black SOR, red = (i+j) odd first,
//                         residual, full weighting, bilinear prolongation, warm start,
//                         coarse zeroing, ||r||/||rho|| convergence)
//   embedded-boundary MG  Multigrid_embedded.cu:15-188 (masked red-black Gauss-Seidel,
//                         residual, restriction with coarse node kinds, prolongation)
//   E field               kernels.cu:134-191
//   gather + kick         kernels.cu:71-131
//   reference MCC form    kernels.cu:196-263 + mcc.cu:56-85 (with Philox instead of cuRAND)
// and the null-collision MCC that the reference does not have, written from the method of
// Vahedi & Surendra, Comput. Phys. Commun. 87 (1995) 179, with the ejected-electron energy
// sharing of Opal et al. (B = 10 eV for argon) and Philox-4x32-10 (Salmon et al., SC'11).
//
// Parity pins: analytic known-answer tests (tests/test_oracle_kat.py) and fixtures produced
// by the reference's own CUDA kernels (oracle/ref_harness.cu -> tests/golden/).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "../include/pic_b200.h"

#define ORC_API extern "C" __attribute__((visibility("default")))

static const double kEps0 = 8.8541878128e-12;
static const double kQe = 1.602176634e-19;
static const double kKb = 1.380649e-23;
static const double kPi = 3.14159265358979323846;

// ------------------------------------------------------------------ Philox-4x32-10
static inline void philox_round(uint32_t c[4], const uint32_t k[2]) {
  const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
  const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
  const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
  const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
  const uint32_t n0 = hi1 ^ c[1] ^ k[0], n2 = hi0 ^ c[3] ^ k[1];
  c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
}
ORC_API void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]}, k[2] = {key[0], key[1]};
  for (int r = 0; r < 10; ++r) {
    if (r) { k[0] += 0x9E3779B9u; k[1] += 0xBB67AE85u; }
    philox_round(c, k);
  }
  out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = c[3];
}
// (2*(x>>9)+1) * 2^-24: in (0,1), exactly representable in FP32 and FP64.
static inline double u01(uint32_t x) { return (double)(2u * (x >> 9) + 1u) * (1.0 / 16777216.0); }
ORC_API double orc_u01(uint32_t x) { return u01(x); }
static inline void draw4(uint64_t seed, uint32_t pid, uint32_t step, uint32_t lane, double u[4]) {
  const uint32_t ctr[4] = {pid, step, lane, 0u};
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  orc_philox4x32_10(ctr, key, o);
  for (int i = 0; i < 4; ++i) u[i] = u01(o[i]);
}

// ------------------------------------------------------------------ particle kernels
// update_coordinates (kernels.cu:8-23)
ORC_API void orc_drift(int64_t n, double* x, double* y, const double* vx, const double* vy,
                       double* xold, double* yold, double dt) {
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < n; ++p) {
    if (xold) xold[p] = x[p];
    if (yold) yold[p] = y[p];
    x[p] = x[p] + vx[p] * dt;
    y[p] = y[p] + vy[p] * dt;
  }
}

// detect_intersections (collisions.cu:7-54), reference-faithful: absolute EPSILON,
// inclusive parameter ranges, first hit ends the wall loop.
ORC_API void orc_walls_segments_ref(int64_t n, const double* x0, const double* y0,
                                    const double* x1, const double* y1, const double* walls,
                                    int nwalls, uint8_t* hit) {
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < n; ++p) {
    const double X1 = x0[p], Y1 = y0[p], X2 = x1[p], Y2 = y1[p];
    bool inter = false;
    const double EPSILON = 1e-10;
    for (int j = 0; j < nwalls && !inter; ++j) {
      const double x3 = walls[4 * j], y3 = walls[4 * j + 1], x4 = walls[4 * j + 2], y4 = walls[4 * j + 3];
      const double denom = (y4 - y3) * (X2 - X1) - (x4 - x3) * (Y2 - Y1);
      if (std::fabs(denom) < EPSILON) continue;
      const double ua = ((x4 - x3) * (Y1 - y3) - (y4 - y3) * (X1 - x3)) / denom;
      const double ub = ((X2 - X1) * (Y1 - y3) - (Y2 - Y1) * (X1 - x3)) / denom;
      if (ua >= 0.0 && ua <= 1.0 && ub >= 0.0 && ub <= 1.0) inter = true;
    }
    hit[p] = inter ? 1 : 0;
  }
}

// The product's segment test: same parametric test with an exact parallel check
// (denom == 0) instead of the absolute cut-off that drops slow particles in SI units.
static inline bool seg_hit(double X1, double Y1, double X2, double Y2, const double* w) {
  const double x3 = w[0], y3 = w[1], x4 = w[2], y4 = w[3];
  const double denom = (y4 - y3) * (X2 - X1) - (x4 - x3) * (Y2 - Y1);
  if (denom == 0.0) return false;
  const double ua = ((x4 - x3) * (Y1 - y3) - (y4 - y3) * (X1 - x3)) / denom;
  const double ub = ((X2 - X1) * (Y1 - y3) - (Y2 - Y1) * (X1 - x3)) / denom;
  return ua >= 0.0 && ua <= 1.0 && ub >= 0.0 && ub <= 1.0;
}
ORC_API void orc_walls_segments(int64_t n, const double* x0, const double* y0, const double* x1,
                                const double* y1, const double* walls, int nwalls, uint8_t* hit) {
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < n; ++p) {
    bool h = false;
    for (int j = 0; j < nwalls && !h; ++j) h = seg_hit(x0[p], y0[p], x1[p], y1[p], walls + 4 * j);
    hit[p] = h ? 1 : 0;
  }
}

// Box absorption: outside the half-open rectangle [0, (m-1)dx) x [0, (n-1)dy) that
// updateDensity deposits from (kernels.cu:47-53).
static inline bool outside_grid(double x, double y, int m, int nn, double dx, double dy) {
  const double xr = x / dx, yr = y / dy;
  const double fx = std::floor(xr), fy = std::floor(yr);
  return !(fx >= 0.0 && fx < (double)(m - 1) && fy >= 0.0 && fy < (double)(nn - 1));
}
ORC_API void orc_walls_box(int64_t n, const double* x, const double* y, int m, int nn, double dx,
                           double dy, uint8_t* hit) {
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < n; ++p) hit[p] = outside_grid(x[p], y[p], m, nn, dx, dy) ? 1 : 0;
}

// updateDensity (kernels.cu:26-69): rho[j*m+i] += q * bilinear weight; skip outside.
ORC_API void orc_deposit(int64_t n, const double* x, const double* y, const double* qp, int m,
                         int nn, double dx, double dy, double* rho) {
  const int64_t nodes = (int64_t)m * nn;
  int nth = 1;
#ifdef _OPENMP
  nth = omp_get_max_threads();
#endif
  std::vector<std::vector<double>> priv(nth);
#pragma omp parallel
  {
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
    std::vector<double>& r = priv[t];
    r.assign(nodes, 0.0);
#pragma omp for schedule(static)
    for (int64_t p = 0; p < n; ++p) {
      const double xr = x[p] / dx, yr = y[p] / dy;
      const double fxf = std::floor(xr), fyf = std::floor(yr);
      if (!(fxf >= 0.0 && fxf < (double)(m - 1) && fyf >= 0.0 && fyf < (double)(nn - 1))) continue;
      const int x0 = (int)fxf, y0 = (int)fyf;
      const double wx = xr - x0, wy = yr - y0, wx1 = 1.0 - wx, wy1 = 1.0 - wy;
      const double q = qp[p];
      r[(int64_t)y0 * m + x0] += q * wx1 * wy1;
      r[(int64_t)y0 * m + x0 + 1] += q * wx * wy1;
      r[(int64_t)(y0 + 1) * m + x0] += q * wx1 * wy;
      r[(int64_t)(y0 + 1) * m + x0 + 1] += q * wx * wy;
    }
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nodes; ++i) {
    double s = 0.0;
    for (int t = 0; t < nth; ++t) s += priv[t][i];
    rho[i] += s;
  }
}

// computeElectricField (kernels.cu:134-191): E = -grad(phi); central inside, one-sided
// first order on edges and corners.
ORC_API void orc_efield(const double* phi, int m, int n, double dx, double dy, double* Ex,
                        double* Ey) {
#pragma omp parallel for schedule(static)
  for (int y = 0; y < n; ++y) {
    for (int x = 0; x < m; ++x) {
      double ex, ey;
      const int64_t c = (int64_t)y * m + x;
      if (x == 0) ex = -(phi[c + 1] - phi[c]) / dx;
      else if (x == m - 1) ex = -(phi[c] - phi[c - 1]) / dx;
      else ex = -(phi[c + 1] - phi[c - 1]) / (2 * dx);
      if (y == 0) ey = -(phi[c + m] - phi[c]) / dy;
      else if (y == n - 1) ey = -(phi[c] - phi[c - m]) / dy;
      else ey = -(phi[c + m] - phi[c - m]) / (2 * dy);
      Ex[c] = ex;
      Ey[c] = ey;
    }
  }
}

// updateParticleVelocities (kernels.cu:71-131): v += q*E*(1/m)*dt with E bilinearly
// interpolated; particles outside the grid are skipped.
ORC_API void orc_kick(int64_t n, const double* x, const double* y, double* vx, double* vy,
                      const double* qp, const double* mp, const double* Ex, const double* Ey,
                      int m, int nn, double dx, double dy, double dt) {
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < n; ++p) {
    const double xr = x[p] / dx, yr = y[p] / dy;
    const double fxf = std::floor(xr), fyf = std::floor(yr);
    if (!(fxf >= 0.0 && fxf < (double)(m - 1) && fyf >= 0.0 && fyf < (double)(nn - 1))) continue;
    const int x0 = (int)fxf, y0 = (int)fyf;
    const double wx = xr - x0, wy = yr - y0, wx1 = 1.0 - wx, wy1 = 1.0 - wy;
    const double w0 = wx1 * wy1, w1 = wx * wy1, w2 = wx1 * wy, w3 = wx * wy;
    const int64_t a = (int64_t)y0 * m + x0, b = a + 1, c = a + m, d = a + m + 1;
    const double ex = w0 * Ex[a] + w1 * Ex[b] + w2 * Ex[c] + w3 * Ex[d];
    const double ey = w0 * Ey[a] + w1 * Ey[b] + w2 * Ey[c] + w3 * Ey[d];
    const double m_inv = 1.0 / mp[p];
    vx[p] += qp[p] * ex * m_inv * dt;
    vy[p] += qp[p] * ey * m_inv * dt;
  }
}

// ------------------------------------------------------------------ multigrid (FP64)
// gauss_seidel_rb_2d_coop (Multigrid.cu:229-267): per iteration the (i+j) odd colour
// first, then the even colour; phi = fma(omega, 0.25*(N+S+E+W - h^2 f), (1-omega)*phi).
static void smooth(double* phi, const double* f, int nx, int ny, double h, double omega, int iters) {
  const double h2 = h * h;
  for (int it = 0; it < iters; ++it) {
    for (int colour = 1; colour >= 0; --colour) {
#pragma omp parallel for schedule(static)
      for (int j = 1; j < ny - 1; ++j) {
        int i0 = 1 + (((1 + j) & 1) != colour ? 1 : 0);
        for (int i = i0; i < nx - 1; i += 2) {
          const int64_t c = (int64_t)j * nx + i;
          const double st = phi[c + nx] + phi[c - nx] + phi[c + 1] + phi[c - 1];
          const double nv = 0.25 * (st - h2 * f[c]);
          phi[c] = std::fma(omega, nv, (1.0 - omega) * phi[c]);
        }
      }
    }
  }
}
// residual_2d (Multigrid.cu:269-297): r = f - lap(phi) inside, 0 on the boundary.
static void residual(double* r, const double* phi, const double* f, int nx, int ny, double h) {
  const double inv_h2 = 1.0 / (h * h);
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const int64_t c = (int64_t)j * nx + i;
      if (i == 0 || i == nx - 1 || j == 0 || j == ny - 1) { r[c] = 0.0; continue; }
      const double lap = (phi[c - nx] + phi[c + nx] + phi[c - 1] + phi[c + 1] - 4.0 * phi[c]) * inv_h2;
      r[c] = f[c] - lap;
    }
}
// restrict_2d (Multigrid.cu:299-349): full weighting, truncated at the boundary.
static void restrict_fw(const double* fine, double* coarse, int nxf, int nyf, int nxc, int nyc) {
#pragma omp parallel for schedule(static)
  for (int jc = 0; jc < nyc; ++jc)
    for (int ic = 0; ic < nxc; ++ic) {
      const int i = 2 * ic, j = 2 * jc;
      if (i >= nxf || j >= nyf) { coarse[(int64_t)jc * nxc + ic] = 0.0; continue; }
      const int64_t c = (int64_t)j * nxf + i;
      double s = 4.0 * fine[c];
      if (i > 0) s += 2.0 * fine[c - 1];
      if (i < nxf - 1) s += 2.0 * fine[c + 1];
      if (j > 0) s += 2.0 * fine[c - nxf];
      if (j < nyf - 1) s += 2.0 * fine[c + nxf];
      if (i > 0 && j > 0) s += fine[c - nxf - 1];
      if (i < nxf - 1 && j > 0) s += fine[c - nxf + 1];
      if (i > 0 && j < nyf - 1) s += fine[c + nxf - 1];
      if (i < nxf - 1 && j < nyf - 1) s += fine[c + nxf + 1];
      coarse[(int64_t)jc * nxc + ic] = s * 0.0625;
    }
}
// prolong_2d (Multigrid.cu:351-407): bilinear, added to the fine array.
static void prolong_add(double* fine, const double* coarse, int nxc, int nyc, int nxf, int nyf) {
#pragma omp parallel for schedule(static)
  for (int jf = 0; jf < nyf; ++jf)
    for (int i = 0; i < nxf; ++i) {
      const int ic = i / 2, jc = jf / 2;
      if (ic >= nxc || jc >= nyc) continue;
      const int64_t c = (int64_t)jc * nxc + ic;
      const bool io = i & 1, jo = jf & 1;
      double v;
      if (!io && !jo) v = coarse[c];
      else if (io && !jo) v = (ic + 1 < nxc) ? 0.5 * (coarse[c] + coarse[c + 1]) : coarse[c];
      else if (!io && jo) v = (jc + 1 < nyc) ? 0.5 * (coarse[c] + coarse[c + nxc]) : coarse[c];
      else v = (ic + 1 < nxc && jc + 1 < nyc)
                   ? 0.25 * (coarse[c] + coarse[c + 1] + coarse[c + nxc] + coarse[c + nxc + 1])
                   : coarse[c];
      fine[(int64_t)jf * nxf + i] += v;
    }
}
static double norm2sq(const double* v, int64_t n) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t i = 0; i < n; ++i) s += v[i] * v[i];
  return s;
}

struct MgWork {
  int nx = 0, ny = 0, levels = 0;
  std::vector<std::vector<double>> phi, rhs, res;
  std::vector<int> nxl, nyl;
  void ensure(int nx_, int ny_, int levels_) {
    if (nx_ == nx && ny_ == ny && levels_ == levels) return;
    nx = nx_; ny = ny_; levels = levels_;
    phi.assign(levels, {}); rhs.assign(levels, {}); res.assign(levels, {});
    nxl.assign(levels, 0); nyl.assign(levels, 0);
    int a = nx, b = ny;
    for (int l = 0; l < levels; ++l) {
      nxl[l] = a; nyl[l] = b;
      phi[l].assign((size_t)a * b, 0.0); rhs[l].assign((size_t)a * b, 0.0); res[l].assign((size_t)a * b, 0.0);
      a = (a + 1) / 2; b = (b + 1) / 2;
    }
  }
};

// v_cycle (Multigrid.cu:539-569) with the sweep counts as parameters (reference: 3, 3, 20).
static void v_cycle(MgWork& w, double* phi0, const double* f0, double h, double omega, int nu1,
                    int nu2, int nuc) {
  const int L = w.levels;
  std::vector<double*> phi(L);
  std::vector<const double*> rhs(L);
  for (int l = 0; l < L; ++l) { phi[l] = w.phi[l].data(); rhs[l] = w.rhs[l].data(); }
  phi[0] = phi0; rhs[0] = f0;
  double hh = h;
  for (int l = 0; l < L - 1; ++l) {
    smooth(phi[l], rhs[l], w.nxl[l], w.nyl[l], hh, omega, nu1);
    residual(w.res[l].data(), phi[l], rhs[l], w.nxl[l], w.nyl[l], hh);
    restrict_fw(w.res[l].data(), w.rhs[l + 1].data(), w.nxl[l], w.nyl[l], w.nxl[l + 1], w.nyl[l + 1]);
    std::fill(w.phi[l + 1].begin(), w.phi[l + 1].end(), 0.0);
    hh *= 2;
  }
  smooth(phi[L - 1], rhs[L - 1], w.nxl[L - 1], w.nyl[L - 1], hh, omega, nuc);
  for (int l = L - 2; l >= 0; --l) {
    hh /= 2;
    prolong_add(phi[l], phi[l + 1], w.nxl[l + 1], w.nyl[l + 1], w.nxl[l], w.nyl[l]);
    smooth(phi[l], rhs[l], w.nxl[l], w.nyl[l], hh, omega, nu2);
  }
}

static int auto_levels(int nx, int ny) {
  int L = 1, a = nx, b = ny;
  while (a > 3 && b > 3 && (a & 1) && (b & 1)) { a = (a + 1) / 2; b = (b + 1) / 2; ++L; }
  return L;
}
ORC_API int orc_auto_levels(int nx, int ny) { return auto_levels(nx, ny); }

static MgWork g_mg;
static int g_ref_convergence = 0;
// conv_mode 1 reproduces the reference's own stopping test: check_convergence_kernel divides
// ||r|| by the value l2_norm_device left in rhs_norm, which is the SQUARED norm ||rho||^2
// (Multigrid.cu:413-453, 466-467, 602), so the reference stops at ||r|| < tol ||rho||^2.
ORC_API void orc_set_reference_convergence(int on) { g_ref_convergence = on; }
// solve_multigrid (Multigrid.cu:573-642): V-cycles until ||f - A phi|| / ||f|| < tol or
// max_cycles; the check follows every cycle, so at least one cycle runs.  Returns the
// number of cycles; relres_out gets the final relative residual.
ORC_API int orc_mg_solve(double* phi, const double* f, int nx, int ny, int levels, double h,
                         double omega, int nu1, int nu2, int nuc, double tol, int max_cycles,
                         double* relres_out) {
  if (levels <= 0) levels = auto_levels(nx, ny);
  g_mg.ensure(nx, ny, levels);
  const int64_t N = (int64_t)nx * ny;
  const double fn2 = norm2sq(f, N);
  const double fn = g_ref_convergence ? fn2 : std::sqrt(fn2);
  std::vector<double> r(N);
  int cyc = 0;
  double rel = 0.0;
  for (; cyc < max_cycles;) {
    v_cycle(g_mg, phi, f, h, omega, nu1, nu2, nuc);
    ++cyc;
    residual(r.data(), phi, f, nx, ny, h);
    rel = std::sqrt(norm2sq(r.data(), N)) / fn;
    if (rel < tol) break;
  }
  if (relres_out) *relres_out = rel;
  return cyc;
}
ORC_API void orc_mg_vcycles(double* phi, const double* f, int nx, int ny, int levels, double h,
                            double omega, int nu1, int nu2, int nuc, int cycles) {
  if (levels <= 0) levels = auto_levels(nx, ny);
  g_mg.ensure(nx, ny, levels);
  for (int c = 0; c < cycles; ++c) v_cycle(g_mg, phi, f, h, omega, nu1, nu2, nuc);
}
ORC_API double orc_relres(const double* phi, const double* f, int nx, int ny, double h) {
  const int64_t N = (int64_t)nx * ny;
  std::vector<double> r(N);
  residual(r.data(), phi, f, nx, ny, h);
  return std::sqrt(norm2sq(r.data(), N)) / std::sqrt(norm2sq(f, N));
}
ORC_API void orc_residual(double* r, const double* phi, const double* f, int nx, int ny, double h) {
  residual(r, phi, f, nx, ny, h);
}

// ------------------------------------------------------------------ embedded-boundary multigrid (FP64)
// Multigrid_embedded.cu:1-190: a per-node mask marks FLUID (0) nodes, where lap(phi) = rhs
// is solved, DIRICHLET (1) nodes (interior electrodes: phi = phi_bc) and SOLID (2) nodes
// (left as they are).  V-cycle of Multigrid::vcycle (:159-188): nu1 red-black Gauss-Seidel
// sweeps (colour 0 = (i+j) even first), residual, full weighting with the coarse mask
// injected from the fine node (2i, 2j), coarse phi zeroed, recursion, piecewise-constant
// prolongation (fine FLUID node += coarse (i/2, j/2)), nu2 sweeps; the coarsest level only
// runs the nu1 pre-sweeps.  Level l has spacing h 2^l.  DIRICHLET nodes take phi_bc; without a
// phi_bc array they keep the value phi holds, which below level 0 is the zeroed coarse phi:
// what the reference's coarse phi_bc arrays, left at their cudaMemset zero (:124-137), give.
// The reference's colour test `(i + j) & 1 != redblack` (:22) parses as
// (i + j) & (1 != redblack): colour 0 updates the even nodes as intended, colour 1 updates
// every interior node concurrently (a data race).  This restatement applies the intended
// test, (i + j) & 1 == colour, to both colours.
static const uint8_t kFluid = 0, kDirichlet = 1;

// smooth_redblack (Multigrid_embedded.cu:15-33), one colour.
static void emb_half_sweep(double* phi, const double* rhs, const uint8_t* mask, const double* bc, int nx, int ny,
                           double h2, int colour) {
#pragma omp parallel for schedule(static)
  for (int j = 1; j < ny - 1; ++j)
    for (int i = 1 + ((1 + j + colour) & 1); i < nx - 1; i += 2) {
      const int64_t id = (int64_t)j * nx + i;
      if (mask[id] == kFluid) {
        const double sum = phi[id - nx] + phi[id + nx] + phi[id - 1] + phi[id + 1];
        phi[id] = 0.25 * (sum - h2 * rhs[id]);
      } else if (mask[id] == kDirichlet && bc) {
        phi[id] = bc[id];   // without phi_bc the node keeps the value phi holds
      }
    }
}
// residual_kernel (Multigrid_embedded.cu:35-55): r = rhs - lap(phi) / h^2 on interior FLUID
// nodes, 0 on other interior nodes; boundary entries are left as they are (the reference's
// res arrays are zeroed once and their boundary is never written).
static void emb_residual(double* res, const double* phi, const double* rhs, const uint8_t* mask, int nx, int ny,
                         double h2i) {
#pragma omp parallel for schedule(static)
  for (int j = 1; j < ny - 1; ++j)
    for (int i = 1; i < nx - 1; ++i) {
      const int64_t id = (int64_t)j * nx + i;
      if (mask[id] == kFluid) {
        const double lap = phi[id - nx] + phi[id + nx] + phi[id - 1] + phi[id + 1] - 4.0 * phi[id];
        res[id] = rhs[id] - h2i * lap;
      } else {
        res[id] = 0.0;
      }
    }
}
// restrict_kernel (Multigrid_embedded.cu:57-86) on interior coarse nodes: the coarse mask is
// the fine node (2ic, 2jc)'s; FLUID coarse nodes get the full-weighted fine residual.
// any: the coarse kind from the 3x3 fine nodes instead, the rule the reference's comment at
// :73 states: DIRICHLET if any of them is, else SOLID if any is not FLUID, else FLUID.
static uint8_t emb_coarse_kind(const uint8_t* mf, int64_t idf, int nxf, bool any) {
  if (!any) return mf[idf];
  bool dir = false, other = false;
  for (int dj = -1; dj <= 1; ++dj)
    for (int di = -1; di <= 1; ++di) {
      const uint8_t m = mf[idf + (int64_t)dj * nxf + di];
      dir |= m == kDirichlet;
      other |= m != kFluid && m != kDirichlet;
    }
  return dir ? kDirichlet : other ? 2 : kFluid;
}
static void emb_restrict(const double* fine, double* coarse, const uint8_t* mf, uint8_t* mc, int nxf, int nxc,
                         int nyc, bool any) {
#pragma omp parallel for schedule(static)
  for (int jc = 1; jc < nyc - 1; ++jc)
    for (int ic = 1; ic < nxc - 1; ++ic) {
      const int64_t idc = (int64_t)jc * nxc + ic, idf = (int64_t)(2 * jc) * nxf + 2 * ic;
      const uint8_t m = emb_coarse_kind(mf, idf, nxf, any);
      mc[idc] = m;
      if (m == kFluid) {
        double sum = 0.0;
        sum += fine[idf];
        sum += 0.5 * (fine[idf - 1] + fine[idf + 1] + fine[idf - nxf] + fine[idf + nxf]);
        sum += 0.25 * (fine[idf - nxf - 1] + fine[idf - nxf + 1] + fine[idf + nxf - 1] + fine[idf + nxf + 1]);
        coarse[idc] = sum / 4.0;
      } else {
        coarse[idc] = 0.0;
      }
    }
}
// prolongate_add_kernel (Multigrid_embedded.cu:88-104): interior FLUID fine nodes add the
// coarse value at (i/2, j/2); bilinear: the bilinear interpolant of the coarse values instead.
static void emb_prolong(const double* coarse, double* fine, const uint8_t* mf, int nxf, int nyf, int nxc,
                        bool bilinear) {
#pragma omp parallel for schedule(static)
  for (int j = 1; j < nyf - 1; ++j)
    for (int i = 1; i < nxf - 1; ++i) {
      const int64_t idf = (int64_t)j * nxf + i;
      if (mf[idf] != kFluid) continue;
      const int64_t a = (int64_t)(j / 2) * nxc + i / 2;
      const bool io = i & 1, jo = j & 1;
      double v;
      if (!bilinear || (!io && !jo)) v = coarse[a];
      else if (io && !jo) v = 0.5 * (coarse[a] + coarse[a + 1]);
      else if (!io && jo) v = 0.5 * (coarse[a] + coarse[a + nxc]);
      else v = 0.25 * (coarse[a] + coarse[a + 1] + coarse[a + nxc] + coarse[a + nxc + 1]);
      fine[idf] += v;
    }
}

struct EmbWork {
  int nx = 0, ny = 0, levels = 0;
  std::vector<std::vector<double>> phi, rhs, res;
  std::vector<std::vector<uint8_t>> mask;
  std::vector<int> nxl, nyl;
  void ensure(int nx_, int ny_, int levels_) {
    if (nx_ == nx && ny_ == ny && levels_ == levels) return;
    nx = nx_; ny = ny_; levels = levels_;
    phi.assign(levels, {}); rhs.assign(levels, {}); res.assign(levels, {}); mask.assign(levels, {});
    nxl.assign(levels, 0); nyl.assign(levels, 0);
    int a = nx, b = ny;
    for (int l = 0; l < levels; ++l) {
      nxl[l] = a; nyl[l] = b;
      phi[l].assign((size_t)a * b, 0.0); rhs[l].assign((size_t)a * b, 0.0);
      res[l].assign((size_t)a * b, 0.0); mask[l].assign((size_t)a * b, 0);
      a = (a - 1) / 2 + 1; b = (b - 1) / 2 + 1;   // Multigrid_embedded.cu:140-141
    }
  }
};
static EmbWork g_emb;

// Multigrid::vcycle(l) (Multigrid_embedded.cu:159-188); level 0 works on the caller's arrays.
static void emb_vcycle(EmbWork& w, int l, double* phi0, const double* rhs0, const uint8_t* mask0,
                       const double* bc0, double h, int nu1, int nu2, int options) {
  double* phi = l ? w.phi[l].data() : phi0;
  const double* rhs = l ? w.rhs[l].data() : rhs0;
  const uint8_t* mask = l ? w.mask[l].data() : mask0;
  const double* bc = l ? nullptr : bc0;
  const int nx = w.nxl[l], ny = w.nyl[l];
  const double h2 = h * h * std::ldexp(1.0, 2 * l), h2i = 1.0 / h2;
  for (int k = 0; k < nu1; ++k) {
    emb_half_sweep(phi, rhs, mask, bc, nx, ny, h2, 0);
    emb_half_sweep(phi, rhs, mask, bc, nx, ny, h2, 1);
  }
  if (l == w.levels - 1) return;
  emb_residual(w.res[l].data(), phi, rhs, mask, nx, ny, h2i);
  emb_restrict(w.res[l].data(), w.rhs[l + 1].data(), mask, w.mask[l + 1].data(), nx, w.nxl[l + 1], w.nyl[l + 1],
               options & PIC_EMB_COARSEN_ANY);
  std::fill(w.phi[l + 1].begin(), w.phi[l + 1].end(), 0.0);
  emb_vcycle(w, l + 1, phi0, rhs0, mask0, bc0, h, nu1, nu2, options);
  emb_prolong(w.phi[l + 1].data(), phi, mask, nx, ny, w.nxl[l + 1], options & PIC_EMB_PROLONG_BILINEAR);
  for (int k = 0; k < nu2; ++k) {
    emb_half_sweep(phi, rhs, mask, bc, nx, ny, h2, 0);
    emb_half_sweep(phi, rhs, mask, bc, nx, ny, h2, 1);
  }
}
// Squared norms over the interior FLUID nodes of level 0: [0] residual, [1] rhs.
static void emb_norms(const double* phi, const double* rhs, const uint8_t* mask, int nx, int ny, double h,
                      double out[2]) {
  const double h2i = 1.0 / (h * h);
  double r2 = 0.0, f2 = 0.0;
#pragma omp parallel for reduction(+ : r2, f2) schedule(static)
  for (int j = 1; j < ny - 1; ++j)
    for (int i = 1; i < nx - 1; ++i) {
      const int64_t id = (int64_t)j * nx + i;
      if (mask[id] != kFluid) continue;
      const double lap = phi[id - nx] + phi[id + nx] + phi[id - 1] + phi[id + 1] - 4.0 * phi[id];
      const double r = rhs[id] - h2i * lap;
      r2 += r * r;
      f2 += rhs[id] * rhs[id];
    }
  out[0] = r2; out[1] = f2;
}

ORC_API void orc_emb_half_sweep(double* phi, const double* rhs, const uint8_t* mask, const double* bc, int nx, int ny,
                                double h2, int colour) {
  emb_half_sweep(phi, rhs, mask, bc, nx, ny, h2, colour);
}
ORC_API void orc_emb_residual(double* res, const double* phi, const double* rhs, const uint8_t* mask, int nx, int ny,
                              double h2i) {
  emb_residual(res, phi, rhs, mask, nx, ny, h2i);
}
ORC_API void orc_emb_restrict(const double* fine, double* coarse, const uint8_t* mf, uint8_t* mc, int nxf, int nyf,
                              int nxc, int nyc, int options) {
  (void)nyf;
  emb_restrict(fine, coarse, mf, mc, nxf, nxc, nyc, options & PIC_EMB_COARSEN_ANY);
}
ORC_API void orc_emb_prolong(const double* coarse, double* fine, const uint8_t* mf, int nxf, int nyf, int nxc,
                             int nyc, int options) {
  (void)nyc;
  emb_prolong(coarse, fine, mf, nxf, nyf, nxc, options & PIC_EMB_PROLONG_BILINEAR);
}
ORC_API void orc_emb_vcycles(double* phi, const double* rhs, const uint8_t* mask, const double* bc, int nx, int ny,
                             int levels, double h, int nu1, int nu2, int options, int cycles) {
  g_emb.ensure(nx, ny, levels);
  for (int c = 0; c < cycles; ++c) emb_vcycle(g_emb, 0, phi, rhs, mask, bc, h, nu1, nu2, options);
}
// Relative residual of the embedded problem: ||r|| / ||rhs|| over the interior FLUID nodes,
// or ||r|| / ||r_0|| (the residual of the initial guess) when rhs is zero there (a Laplace
// problem driven by the electrodes alone); 0 when both are zero.
static double emb_rel(const double n[2], double r0) {
  if (n[1] > 0.0) return std::sqrt(n[0] / n[1]);
  if (r0 > 0.0) return std::sqrt(n[0] / r0);
  return std::sqrt(n[0]);
}
// V-cycles until the relative residual drops below tol or max_cycles ran (checked after every
// cycle).  Returns the number of cycles; relres_out gets the final relative residual.
ORC_API int orc_emb_solve(double* phi, const double* rhs, const uint8_t* mask, const double* bc, int nx, int ny,
                          int levels, double h, int nu1, int nu2, int options, double tol, int max_cycles,
                          double* relres_out) {
  g_emb.ensure(nx, ny, levels);
  double n[2];
  emb_norms(phi, rhs, mask, nx, ny, h, n);
  const double r0 = n[0];
  int cyc = 0;
  double rel = emb_rel(n, r0);
  while (cyc < max_cycles) {
    emb_vcycle(g_emb, 0, phi, rhs, mask, bc, h, nu1, nu2, options);
    ++cyc;
    emb_norms(phi, rhs, mask, nx, ny, h, n);
    rel = emb_rel(n, r0);
    if (rel < tol) break;
  }
  if (relres_out) *relres_out = rel;
  return cyc;
}
ORC_API void orc_emb_norms(const double* phi, const double* rhs, const uint8_t* mask, int nx, int ny, double h,
                           double out[2]) {
  emb_norms(phi, rhs, mask, nx, ny, h, out);
}

// ------------------------------------------------------------------ cross sections
struct Table {
  std::vector<double> e, s;
  // interpolate_cross_sections (kernels.cu:219-263): clamp outside, linear inside.
  double eval(double E) const {
    const int n = (int)e.size();
    if (E <= e[0]) return s[0];
    if (E >= e[n - 1]) return s[n - 1];
    int k = (int)(std::upper_bound(e.begin(), e.end(), E) - e.begin()) - 1;
    k = std::max(0, std::min(k, n - 2));
    const double t = (E - e[k]) / (e[k + 1] - e[k]);
    return s[k] + t * (s[k + 1] - s[k]);
  }
};

// ------------------------------------------------------------------ full-step simulation
struct Species {
  double q = 0, m = 1, w = 1;
  std::vector<double> x, y, vx, vy, vz;
  std::vector<uint32_t> pid;
};
struct Proc { int type, species; double thr; Table t; };

struct OracleSim {
  pic_job_config cfg;
  int nx, ny;
  double dx, dy, dt, qref, rhs_scale;
  std::vector<Species> sp;
  std::vector<double> rho, phi, f, Ex, Ey;
  std::vector<double> phi_prev;   // previous solution (mg_warm_start 1)
  bool have_prev = false;
  std::vector<Proc> procs;
  std::vector<double> numax;  // per species
  uint32_t next_pid = 0;
  int64_t step = 0;
  int last_cycles = 0;
  double last_relres = 0;
  std::vector<int64_t> absorbed;
  std::vector<std::vector<int64_t>> ncoll;
  int64_t nioniz = 0;
};

static double speed_of_energy(double Eev, double m) { return std::sqrt(2.0 * Eev * kQe / m); }

ORC_API void* orc_sim_create(const pic_job_config* c) {
  OracleSim* s = new OracleSim();
  s->cfg = *c;
  for (int i = 0; i < c->n_processes; ++i) s->cfg.processes[i].energy_ev = nullptr, s->cfg.processes[i].sigma_m2 = nullptr;
  s->nx = c->nx; s->ny = c->ny;
  s->dx = c->Lx / (c->nx - 1); s->dy = c->Ly / (c->ny - 1); s->dt = c->dt;
  s->sp.resize(c->n_species);
  s->qref = 0.0;
  for (int k = 0; k < c->n_species; ++k) {
    s->sp[k].q = c->species[k].charge; s->sp[k].m = c->species[k].mass; s->sp[k].w = c->species[k].weight;
    s->qref = std::max(s->qref, std::fabs(c->species[k].charge * c->species[k].weight));
  }
  s->rhs_scale = (c->units == PIC_UNITS_SI) ? -1.0 / (kEps0 * s->dx * s->dy) : 1.0;
  const size_t N = (size_t)s->nx * s->ny;
  s->rho.assign(N, 0); s->phi.assign(N, 0); s->f.assign(N, 0); s->Ex.assign(N, 0); s->Ey.assign(N, 0);
  for (int i = 0; i < c->n_processes; ++i) {
    Proc p;
    p.type = c->processes[i].type; p.species = c->processes[i].species; p.thr = c->processes[i].threshold_ev;
    p.t.e.assign(c->processes[i].energy_ev, c->processes[i].energy_ev + c->processes[i].n_points);
    p.t.s.assign(c->processes[i].sigma_m2, c->processes[i].sigma_m2 + c->processes[i].n_points);
    s->procs.push_back(p);
  }
  // nu_max per species: n_g * max over table intervals of max(sigma_T) * v(upper energy).
  s->numax.assign(c->n_species, 0.0);
  for (int k = 0; k < c->n_species; ++k) {
    std::vector<double> grid;
    for (auto& p : s->procs) if (p.species == k) grid.insert(grid.end(), p.t.e.begin(), p.t.e.end());
    if (grid.empty()) continue;
    std::sort(grid.begin(), grid.end());
    double best = 0.0;
    for (size_t g = 0; g < grid.size(); ++g) {
      const double elo = grid[g > 0 ? g - 1 : 0], ehi = grid[g];
      double st = 0.0;
      for (auto& p : s->procs) if (p.species == k) st += std::max(p.t.eval(elo), p.t.eval(ehi));
      best = std::max(best, st * speed_of_energy(ehi, s->sp[k].m));
    }
    s->numax[k] = c->gas_density * best;
  }
  s->absorbed.assign(c->n_species, 0);
  s->ncoll.assign(c->n_species, std::vector<int64_t>(PIC_MAX_PROCESSES, 0));
  return s;
}
ORC_API void orc_sim_destroy(void* h) { delete (OracleSim*)h; }
ORC_API double orc_sim_numax(void* h, int k) { return ((OracleSim*)h)->numax[k]; }

ORC_API void orc_sim_load(void* h, int k, int64_t n, const double* x, const double* y,
                          const double* vx, const double* vy, const double* vz, const uint32_t* pid) {
  OracleSim* s = (OracleSim*)h;
  Species& S = s->sp[k];
  S.x.assign(x, x + n); S.y.assign(y, y + n); S.vx.assign(vx, vx + n); S.vy.assign(vy, vy + n);
  if (vz) S.vz.assign(vz, vz + n); else S.vz.assign(n, 0.0);
  S.pid.resize(n);
  for (int64_t i = 0; i < n; ++i) S.pid[i] = pid ? pid[i] : s->next_pid + (uint32_t)i;
  uint32_t mx = 0;
  for (int64_t i = 0; i < n; ++i) mx = std::max(mx, S.pid[i] + 1);
  s->next_pid = std::max(s->next_pid, mx);
}
ORC_API int64_t orc_sim_count(void* h, int k) { return (int64_t)((OracleSim*)h)->sp[k].x.size(); }
ORC_API void orc_sim_export(void* h, int k, double* x, double* y, double* vx, double* vy, double* vz,
                            uint32_t* pid) {
  Species& S = ((OracleSim*)h)->sp[k];
  const size_t n = S.x.size();
  std::copy(S.x.begin(), S.x.end(), x); std::copy(S.y.begin(), S.y.end(), y);
  std::copy(S.vx.begin(), S.vx.end(), vx); std::copy(S.vy.begin(), S.vy.end(), vy);
  if (vz) std::copy(S.vz.begin(), S.vz.end(), vz);
  if (pid) std::copy(S.pid.begin(), S.pid.begin() + n, pid);
}
ORC_API void orc_sim_get_grid(void* h, int which, double* out) {
  OracleSim* s = (OracleSim*)h;
  const std::vector<double>& g = which == PIC_GRID_RHO ? s->rho : which == PIC_GRID_PHI ? s->phi
                                 : which == PIC_GRID_EX ? s->Ex : s->Ey;
  std::copy(g.begin(), g.end(), out);
}
ORC_API void orc_sim_set_grid(void* h, int which, const double* in) {
  OracleSim* s = (OracleSim*)h;
  std::vector<double>& g = which == PIC_GRID_RHO ? s->rho : which == PIC_GRID_PHI ? s->phi
                           : which == PIC_GRID_EX ? s->Ex : s->Ey;
  std::copy(in, in + g.size(), g.begin());
  if (which == PIC_GRID_PHI) s->have_prev = false;
}
// Step index (the Philox key of the next collision phase) and the id the next created
// particle receives: set from a running engine job so that the oracle continues it.
ORC_API void orc_sim_set_counters(void* h, int64_t step, uint32_t next_pid) {
  OracleSim* s = (OracleSim*)h;
  s->step = step;
  s->next_pid = next_pid;
}
ORC_API void orc_sim_stats(void* h, int64_t* step, int* cycles, double* relres, int64_t* absorbed,
                           int64_t* ncoll, int64_t* nioniz) {
  OracleSim* s = (OracleSim*)h;
  *step = s->step; *cycles = s->last_cycles; *relres = s->last_relres;
  for (int k = 0; k < s->cfg.n_species; ++k) {
    absorbed[k] = s->absorbed[k];
    for (int p = 0; p < PIC_MAX_PROCESSES; ++p) ncoll[k * PIC_MAX_PROCESSES + p] = s->ncoll[k][p];
  }
  *nioniz = s->nioniz;
}

static void remove_hits(Species& S, const std::vector<uint8_t>& hit) {
  size_t w = 0;
  for (size_t r = 0; r < S.x.size(); ++r) {
    if (hit[r]) continue;
    S.x[w] = S.x[r]; S.y[w] = S.y[r]; S.vx[w] = S.vx[r]; S.vy[w] = S.vy[r]; S.vz[w] = S.vz[r]; S.pid[w] = S.pid[r];
    ++w;
  }
  S.x.resize(w); S.y.resize(w); S.vx.resize(w); S.vy.resize(w); S.vz.resize(w); S.pid.resize(w);
}

// Phase: drift + absorption + removal for every species (main.cu:64-87, particles.cu:217).
ORC_API void orc_sim_drift_walls(void* h) {
  OracleSim* s = (OracleSim*)h;
  const pic_job_config& c = s->cfg;
  for (int k = 0; k < c.n_species; ++k) {
    Species& S = s->sp[k];
    const int64_t n = (int64_t)S.x.size();
    std::vector<double> xo(n), yo(n);
    orc_drift(n, S.x.data(), S.y.data(), S.vx.data(), S.vy.data(), xo.data(), yo.data(), s->dt);
    std::vector<uint8_t> hit(n, 0), h2(n, 0);
    if (c.wall_mode == PIC_WALLS_BOX || c.wall_mode == PIC_WALLS_BOX_AND_SEGMENTS)
      orc_walls_box(n, S.x.data(), S.y.data(), s->nx, s->ny, s->dx, s->dy, hit.data());
    if ((c.wall_mode == PIC_WALLS_SEGMENTS || c.wall_mode == PIC_WALLS_BOX_AND_SEGMENTS) && c.n_walls > 0) {
      orc_walls_segments(n, xo.data(), yo.data(), S.x.data(), S.y.data(), &c.walls[0][0], c.n_walls, h2.data());
      for (int64_t p = 0; p < n; ++p) hit[p] |= h2[p];
    }
    int64_t nh = 0;
    for (int64_t p = 0; p < n; ++p) nh += hit[p];
    s->absorbed[k] = nh;
    remove_hits(S, hit);
  }
}
// Phase: rho = sum_s deposit(q_s * W_s) (main.cu:93-98).
ORC_API void orc_sim_deposit(void* h) {
  OracleSim* s = (OracleSim*)h;
  std::fill(s->rho.begin(), s->rho.end(), 0.0);
  for (auto& S : s->sp) {
    const int64_t n = (int64_t)S.x.size();
    std::vector<double> q(n, S.q * S.w);
    orc_deposit(n, S.x.data(), S.y.data(), q.data(), s->nx, s->ny, s->dx, s->dy, s->rho.data());
  }
}
// Phase: Poisson solve + E (main.cu:111-120).
ORC_API void orc_sim_solve(void* h) {
  OracleSim* s = (OracleSim*)h;
  const pic_job_config& c = s->cfg;
  for (size_t i = 0; i < s->rho.size(); ++i) s->f[i] = s->rhs_scale * s->rho[i];
  if (c.mg_warm_start) {
    // initial guess 2 phi_{k-1} - phi_{k-2} once two solutions exist, else phi_{k-1}
    if (s->have_prev) {
      for (size_t i = 0; i < s->phi.size(); ++i) {
        const double g = 2.0 * s->phi[i] - s->phi_prev[i];
        s->phi_prev[i] = s->phi[i];
        s->phi[i] = g;
      }
    } else {
      s->phi_prev = s->phi;
      s->have_prev = true;
    }
  }
  s->last_cycles = orc_mg_solve(s->phi.data(), s->f.data(), s->nx, s->ny, c.mg_levels, s->dx, c.omega,
                                c.nu_pre, c.nu_post, c.nu_coarse, c.tol, c.max_cycles, &s->last_relres);
  orc_efield(s->phi.data(), s->nx, s->ny, s->dx, s->dy, s->Ex.data(), s->Ey.data());
}
// Phase: gather + kick (main.cu:124-127).
ORC_API void orc_sim_kick(void* h) {
  OracleSim* s = (OracleSim*)h;
  for (auto& S : s->sp) {
    const int64_t n = (int64_t)S.x.size();
    std::vector<double> q(n, S.q), m(n, S.m);
    orc_kick(n, S.x.data(), S.y.data(), S.vx.data(), S.vy.data(), q.data(), m.data(), s->Ex.data(),
             s->Ey.data(), s->nx, s->ny, s->dx, s->dy, s->dt);
  }
}

// Isotropic unit vector from two uniforms: cos(chi) = 1 - 2 u_a, azimuth 2 pi u_b.
static inline void iso_dir(double ua, double ub, double d[3]) {
  const double c = 1.0 - 2.0 * ua, sn = std::sqrt(std::max(0.0, 1.0 - c * c)), ph = 2.0 * kPi * ub;
  d[0] = sn * std::cos(ph); d[1] = sn * std::sin(ph); d[2] = c;
}
// Three Maxwellian components of a neutral at temperature T (Box-Muller on draw lane 2).
static inline void neutral_velocity(uint64_t seed, uint32_t pid, uint32_t step, double sig, double v[3]) {
  double u[4];
  draw4(seed, pid, step, 2u, u);
  const double r0 = std::sqrt(-2.0 * std::log(u[0])), r1 = std::sqrt(-2.0 * std::log(u[2]));
  v[0] = sig * r0 * std::cos(2.0 * kPi * u[1]);
  v[1] = sig * r0 * std::sin(2.0 * kPi * u[1]);
  v[2] = sig * r1 * std::cos(2.0 * kPi * u[3]);
}

struct NewPair { uint32_t parent; double x, y, ve[3], vi[3]; };

// Phase: Monte Carlo collisions on the kicked velocities (after the kick, as the
// commented-out elasticCollisions call in main.cu:131-134).
ORC_API void orc_sim_mcc(void* h) {
  OracleSim* s = (OracleSim*)h;
  const pic_job_config& c = s->cfg;
  for (auto& v : s->ncoll) std::fill(v.begin(), v.end(), 0);
  s->nioniz = 0;
  if (c.mcc_mode == PIC_MCC_NONE) return;
  const uint32_t step = (uint32_t)s->step;
  std::vector<NewPair> pairs;
  const double ng = c.gas_density;
  const double vth_n = std::sqrt(kKb * c.gas_temperature / c.gas_mass);
  for (int k = 0; k < c.n_species; ++k) {
    Species& S = s->sp[k];
    std::vector<int> mine;
    for (int p = 0; p < (int)s->procs.size(); ++p) if (s->procs[p].species == k) mine.push_back(p);
    if (mine.empty()) continue;
    const int64_t n = (int64_t)S.x.size();
    if (c.mcc_mode == PIC_MCC_REF_ELASTIC2D) {
      // collision_kernel (mcc.cu:56-85): P = 1 - exp(-n sigma |v| dt); v <- |v| (cos, sin).
      const Table& t = s->procs[mine[0]].t;
      for (int64_t p = 0; p < n; ++p) {
        double u[4];
        draw4(c.seed, S.pid[p], step, 0u, u);
        const double v2 = S.vx[p] * S.vx[p] + S.vy[p] * S.vy[p], sp = std::sqrt(v2);
        const double E = 0.5 * S.m * v2 / kQe;
        const double P = 1.0 - std::exp(-ng * t.eval(E) * sp * s->dt);
        if (u[0] < P) {
          const double th = u[1] * 2.0 * kPi;
          S.vx[p] = sp * std::cos(th); S.vy[p] = sp * std::sin(th);
          s->ncoll[k][mine[0]]++;
        }
      }
      continue;
    }
    // First-order null-collision probability: a particle is a candidate with probability
    // nu_max dt and collides for real in process j with probability nu_j dt = n sigma_j v dt
    // (the configuration guarantees nu_max dt <= 1).
    const double numax = s->numax[k];
    const double pnull = numax * s->dt;
    // particles are independent: OpenMP over them, per-thread counters and pair lists (the
    // pairs are ordered by parent pid afterwards, so the result does not depend on threads)
    std::vector<int64_t> cnt(PIC_MAX_PROCESSES, 0);
#pragma omp parallel
    {
      std::vector<int64_t> my_cnt(PIC_MAX_PROCESSES, 0);
      std::vector<NewPair> my_pairs;
#pragma omp for schedule(static)
      for (int64_t p = 0; p < n; ++p) {
        double u[4];
        draw4(c.seed, S.pid[p], step, 0u, u);
        if (!(u[0] < pnull)) continue;
        const double v2 = S.vx[p] * S.vx[p] + S.vy[p] * S.vy[p] + S.vz[p] * S.vz[p];
        const double sp = std::sqrt(v2);
        const double E = 0.5 * S.m * v2 / kQe;
        const double target = u[1] * numax;
        double acc = 0.0;
        int chosen = -1;
        for (int q : mine) {
          acc += ng * s->procs[q].t.eval(E) * sp;
          if (target < acc) { chosen = q; break; }
        }
        if (chosen < 0) continue;
        const Proc& P = s->procs[chosen];
        double d[3];
        if (P.type == PIC_PROC_ELASTIC) {
          iso_dir(u[2], u[3], d);
          const double cosx = sp > 0 ? (S.vx[p] * d[0] + S.vy[p] * d[1] + S.vz[p] * d[2]) / sp : 1.0;
          const double Ep = E * (1.0 - 2.0 * S.m / c.gas_mass * (1.0 - cosx));
          const double vn = speed_of_energy(std::max(0.0, Ep), S.m);
          S.vx[p] = vn * d[0]; S.vy[p] = vn * d[1]; S.vz[p] = vn * d[2];
        } else if (P.type == PIC_PROC_EXCITATION) {
          if (E < P.thr) continue;
          iso_dir(u[2], u[3], d);
          const double vn = speed_of_energy(E - P.thr, S.m);
          S.vx[p] = vn * d[0]; S.vy[p] = vn * d[1]; S.vz[p] = vn * d[2];
        } else if (P.type == PIC_PROC_IONIZATION) {
          if (E < P.thr) continue;
          double u2[4];
          draw4(c.seed, S.pid[p], step, 1u, u2);
          const double Er = E - P.thr, B = 10.0;
          const double Eej = B * std::tan(u2[0] * std::atan(Er / (2.0 * B)));
          const double Esc = std::max(0.0, Er - Eej);
          iso_dir(u[2], u[3], d);
          const double vs = speed_of_energy(Esc, S.m);
          NewPair np;
          np.parent = S.pid[p]; np.x = S.x[p]; np.y = S.y[p];
          double d2[3];
          iso_dir(u2[1], u2[2], d2);
          const double ve = speed_of_energy(Eej, s->sp[c.ionization_electron_species].m);
          for (int a = 0; a < 3; ++a) np.ve[a] = ve * d2[a];
          neutral_velocity(c.seed, S.pid[p], step, vth_n, np.vi);
          my_pairs.push_back(np);
          S.vx[p] = vs * d[0]; S.vy[p] = vs * d[1]; S.vz[p] = vs * d[2];
        } else if (P.type == PIC_PROC_CHARGE_EXCHANGE) {
          double vn[3];
          neutral_velocity(c.seed, S.pid[p], step, vth_n, vn);
          S.vx[p] = vn[0]; S.vy[p] = vn[1]; S.vz[p] = vn[2];
        }
        my_cnt[chosen]++;
      }
#pragma omp critical
      {
        for (int q = 0; q < PIC_MAX_PROCESSES; ++q) cnt[q] += my_cnt[q];
        pairs.insert(pairs.end(), my_pairs.begin(), my_pairs.end());
      }
    }
    for (int q = 0; q < PIC_MAX_PROCESSES; ++q) s->ncoll[k][q] += cnt[q];
  }
  // New pairs in ascending parent-pid order: electron pid = next + 2r, ion pid = next + 2r + 1.
  std::sort(pairs.begin(), pairs.end(), [](const NewPair& a, const NewPair& b) { return a.parent < b.parent; });
  Species& E = s->sp[c.ionization_electron_species];
  Species& I = s->sp[c.ionization_ion_species];
  for (size_t r = 0; r < pairs.size(); ++r) {
    const NewPair& np = pairs[r];
    E.x.push_back(np.x); E.y.push_back(np.y); E.vx.push_back(np.ve[0]); E.vy.push_back(np.ve[1]);
    E.vz.push_back(np.ve[2]); E.pid.push_back(s->next_pid + 2 * (uint32_t)r);
    I.x.push_back(np.x); I.y.push_back(np.y); I.vx.push_back(np.vi[0]); I.vy.push_back(np.vi[1]);
    I.vz.push_back(np.vi[2]); I.pid.push_back(s->next_pid + 2 * (uint32_t)r + 1);
  }
  s->next_pid += 2 * (uint32_t)pairs.size();
  s->nioniz = (int64_t)pairs.size();
}

// One full step in the reference's order: drift, walls, removal, deposit, solve, E, kick,
// then collisions.
ORC_API void orc_sim_step(void* h, int nsteps) {
  OracleSim* s = (OracleSim*)h;
  for (int i = 0; i < nsteps; ++i) {
    orc_sim_drift_walls(h);
    orc_sim_deposit(h);
    orc_sim_solve(h);
    orc_sim_kick(h);
    orc_sim_mcc(h);
    s->step++;
  }
}
ORC_API double orc_sim_total_charge(void* h) {
  OracleSim* s = (OracleSim*)h;
  double t = 0;
  for (double v : s->rho) t += v;
  return t;
}
ORC_API int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
