// particle_ops.cuh — per-particle drift / absorption / deposit shared by the mover and the
// ionisation kernel (new particles take the same path as old ones).
#pragma once
#include "common.cuh"

// detect_intersections (collisions.cu:7-54) without the absolute 1e-10 cut-off: the segment
// old->new (relative to the base cell corner bi,bj, in cell units) against every wall.
// Walls are stored in grid units (FP64) and shifted to the base cell before the FP32 test,
// so the test keeps sub-cell precision anywhere on the grid.
__device__ __forceinline__ bool segment_hits(const JobDev& J, int bi, int bj, float x1, float y1,
                                             float x2, float y2) {
  for (int w = 0; w < J.n_walls; ++w) {
    const double* W = J.walls + 4 * w;
    const float x3 = (float)(W[0] - bi), y3 = (float)(W[1] - bj);
    const float x4 = (float)(W[2] - bi), y4 = (float)(W[3] - bj);
    const float denom = (y4 - y3) * (x2 - x1) - (x4 - x3) * (y2 - y1);
    if (denom == 0.f) continue;
    const float ua = ((x4 - x3) * (y1 - y3) - (y4 - y3) * (x1 - x3)) / denom;
    const float ub = ((x2 - x1) * (y1 - y3) - (y2 - y1) * (x1 - x3)) / denom;
    if (ua >= 0.f && ua <= 1.f && ub >= 0.f && ub <= 1.f) return true;
  }
  return false;
}

struct Drifted {
  uint32_t cell;
  float fx, fy;
  bool absorbed;
};

// update_coordinates (kernels.cu:8-23) on a cell-relative position, followed by the
// absorption test.  BOX absorbs whatever leaves [0,ncx) x [0,ncy) cells; SEGMENTS tests the
// path against the walls.  Particles outside the grid (segment-only walls) keep absolute
// grid coordinates in fx, fy with cell = PIC_CELL_OUT.
__device__ __forceinline__ Drifted drift_particle(const JobDev& J, const SlotDev& S, uint32_t c, float fx, float fy,
                                                  float vx, float vy, bool walls) {
  Drifted d;
  d.absorbed = false;
  const bool box = walls && (J.wall_mode & 1);
  const bool segs = walls && (J.wall_mode & 2) && J.n_walls > 0;
  if (c != PIC_CELL_OUT) {
    const int i = cell_i(c), j = cell_j(c);
    const float ax = fx + vx * S.dtdx, ay = fy + vy * S.dtdy;
    const float fi = fminf(fmaxf(floorf(ax), -1.0e9f), 1.0e9f);
    const float fj = fminf(fmaxf(floorf(ay), -1.0e9f), 1.0e9f);
    int ni = i + (int)fi, nj = j + (int)fj;
    float nfx = ax - fi, nfy = ay - fj;
    if (nfx >= 1.f) { nfx -= 1.f; ++ni; }
    if (nfy >= 1.f) { nfy -= 1.f; ++nj; }
    const bool inside = ni >= 0 && ni < J.ncx && nj >= 0 && nj < J.ncy;
    if (segs) d.absorbed = segment_hits(J, i, j, fx, fy, ax, ay);
    if (box && !inside) d.absorbed = true;
    if (inside) { d.cell = pack_cell(ni, nj); d.fx = nfx; d.fy = nfy; }
    else { d.cell = PIC_CELL_OUT; d.fx = (float)i + ax; d.fy = (float)j + ay; }
  } else {
    const float ax = fx + vx * S.dtdx, ay = fy + vy * S.dtdy;
    if (segs) d.absorbed = segment_hits(J, 0, 0, fx, fy, ax, ay);
    const float fi = floorf(ax), fj = floorf(ay);
    if (fi >= 0.f && fi < (float)J.ncx && fj >= 0.f && fj < (float)J.ncy) {
      d.cell = pack_cell((int)fi, (int)fj);
      d.fx = fminf(ax - fi, 0.99999994f);
      d.fy = fminf(ay - fj, 0.99999994f);
    } else {
      d.cell = PIC_CELL_OUT; d.fx = ax; d.fy = ay;
      if (box) d.absorbed = true;
    }
  }
  return d;
}

// CIC deposit of one particle with plain atomics (updateDensity, kernels.cu:56-68).
__device__ __forceinline__ void deposit_one(const JobDev& J, const SlotDev& S, uint32_t c, float fx, float fy) {
  if (c == PIC_CELL_OUT) return;
  const int i = cell_i(c), j = cell_j(c);
  const size_t a = (size_t)j * J.nx + i;
  const float w00 = (1.f - fx) * (1.f - fy), w10 = fx * (1.f - fy), w01 = (1.f - fx) * fy, w11 = fx * fy;
  if (J.deposit_mode == 0) {
    atomicAdd(J.rho_f + a, S.qdep * w00);
    atomicAdd(J.rho_f + a + 1, S.qdep * w10);
    atomicAdd(J.rho_f + a + J.nx, S.qdep * w01);
    atomicAdd(J.rho_f + a + J.nx + 1, S.qdep * w11);
  } else {
    const double Q = (double)S.qfix;
    const long long v0 = __double2ll_rn((double)w00 * Q), v1 = __double2ll_rn((double)w10 * Q);
    const long long v2 = __double2ll_rn((double)w01 * Q), v3 = S.qfix - v0 - v1 - v2;
    unsigned long long* rho = (unsigned long long*)J.rho_i;
    atomicAdd(rho + a, (unsigned long long)v0);
    atomicAdd(rho + a + 1, (unsigned long long)v1);
    atomicAdd(rho + a + J.nx, (unsigned long long)v2);
    atomicAdd(rho + a + J.nx + 1, (unsigned long long)v3);
  }
}
