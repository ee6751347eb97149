// mover.cu — the fused particle pass of one PIC step.
//
// One pass over each particle slot does, in the reference's order (main.cu:64-134):
//   kick     updateParticleVelocities (kernels.cu:71-131) with E = -grad(phi) taken on the
//            fly from phi32 through the computeElectricField stencils (kernels.cu:134-191)
//   MCC      null-collision Monte Carlo (or the reference's elastic form, mcc.cu:56-85)
//   drift    update_coordinates (kernels.cu:8-23) on cell-relative FP32 positions
//   walls    detect_intersections (collisions.cu:7-54) / box absorption; hits are appended
//            with warp-aggregated atomics (compaction happens in compact.cu)
//   deposit  updateDensity (kernels.cu:26-69) at the new position: per warp a segmented
//            reduction over lanes that share a cell (particles are counting-sorted by cell),
//            then one atomic per node per segment; FP32 or int64 fixed point.
// The kick + MCC of step k are fused into the pass of step k+1 (the job's kick_pending
// flag); an explicit flush applies them before any read-back.
#include "common.cuh"
#include "kernels.h"
#include "particle_ops.cuh"

namespace {

struct PhiGather {
  const float* phi;
  int nx, ny;
};

// E at the four nodes of cell (i,j), interpolated at (fx,fy), returned as the phi
// difference per unit cell (so dv = k * this).  Edge nodes use one-sided differences,
// interior nodes central ones, like computeElectricField.
__device__ __forceinline__ void gather_dphi(const PhiGather& g, int i, int j, float fx, float fy,
                                            float& gx, float& gy) {
  const int nx = g.nx;
  const float* r0 = g.phi + (size_t)j * nx;
  const float* r1 = r0 + nx;
  const int xl = i > 0 ? i - 1 : 0, xr = (i + 2 < nx) ? i + 2 : nx - 1;
  const float sx0 = i > 0 ? 0.5f : 1.0f, sx1 = (i + 2 < nx) ? 0.5f : 1.0f;
  const float a_l = __ldg(r0 + xl), a_0 = __ldg(r0 + i), a_1 = __ldg(r0 + i + 1), a_r = __ldg(r0 + xr);
  const float b_l = __ldg(r1 + xl), b_0 = __ldg(r1 + i), b_1 = __ldg(r1 + i + 1), b_r = __ldg(r1 + xr);
  const int yl = j > 0 ? j - 1 : 0, yr = (j + 2 < g.ny) ? j + 2 : g.ny - 1;
  const float sy0 = j > 0 ? 0.5f : 1.0f, sy1 = (j + 2 < g.ny) ? 0.5f : 1.0f;
  const float c_0 = __ldg(g.phi + (size_t)yl * nx + i), c_1 = __ldg(g.phi + (size_t)yl * nx + i + 1);
  const float d_0 = __ldg(g.phi + (size_t)yr * nx + i), d_1 = __ldg(g.phi + (size_t)yr * nx + i + 1);
  // -dphi/dx at the four nodes (in units of 1/dx)
  const float ex00 = (a_l - a_1) * sx0, ex10 = (a_0 - a_r) * sx1;
  const float ex01 = (b_l - b_1) * sx0, ex11 = (b_0 - b_r) * sx1;
  const float ey00 = (c_0 - b_0) * sy0, ey10 = (c_1 - b_1) * sy0;
  const float ey01 = (a_0 - d_0) * sy1, ey11 = (a_1 - d_1) * sy1;
  const float w00 = (1.f - fx) * (1.f - fy), w10 = fx * (1.f - fy), w01 = (1.f - fx) * fy, w11 = fx * fy;
  gx = w00 * ex00 + w10 * ex10 + w01 * ex01 + w11 * ex11;
  gy = w00 * ey00 + w10 * ey10 + w01 * ey01 + w11 * ey11;
}

__device__ __forceinline__ float xs_lookup(const ProcDev& p, float E) {
  const float* e = p.e;
  const int n = p.n;
  if (E <= e[0]) return p.s[0];
  if (E >= e[n - 1]) return p.s[n - 1];
  int k;
  if (p.inv_dlog > 0.f) {
    k = (int)((__logf(E) - p.log_e0) * p.inv_dlog);
    k = max(0, min(k, n - 2));
    while (k > 0 && E < e[k]) --k;
    while (k < n - 2 && E >= e[k + 1]) ++k;
  } else {
    int lo = 0, hi = n - 2;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (e[mid] <= E) lo = mid; else hi = mid - 1;
    }
    k = lo;
  }
  const float t = (E - e[k]) / (e[k + 1] - e[k]);
  return p.s[k] + t * (p.s[k + 1] - p.s[k]);
}

__device__ __forceinline__ void iso_dir(float ua, float ub, float d[3]) {
  const float c = 1.f - 2.f * ua;
  const float sn = sqrtf(fmaxf(0.f, 1.f - c * c));
  float s, co;
  sincospif(2.f * ub, &s, &co);
  d[0] = sn * co; d[1] = sn * s; d[2] = c;
}

__device__ __forceinline__ void neutral_velocity(uint64_t seed, uint32_t pid, uint32_t step, float sig, float v[3]) {
  float u[4];
  draw4(seed, pid, step, 2u, u);
  const float r0 = sqrtf(-2.f * logf(u[0])), r1 = sqrtf(-2.f * logf(u[2]));
  float s, c, s2, c2;
  sincospif(2.f * u[1], &s, &c);
  sincospif(2.f * u[3], &s2, &c2);
  v[0] = sig * r0 * c; v[1] = sig * r0 * s; v[2] = sig * r1 * c2;
}

template <typename T>
__device__ __forceinline__ void seg_reduce4(T& a, T& b, T& c, T& d, int seg) {
  const int lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T ta = __shfl_down_sync(0xffffffffu, a, o);
    const T tb = __shfl_down_sync(0xffffffffu, b, o);
    const T tc = __shfl_down_sync(0xffffffffu, c, o);
    const T td = __shfl_down_sync(0xffffffffu, d, o);
    const int ts = __shfl_down_sync(0xffffffffu, seg, o);
    if (lane + o < 32 && ts == seg) { a += ta; b += tb; c += tc; d += td; }
  }
}

}  // namespace

// Deposit one particle per lane (key = packed cell or CELL_OUT) with a warp-segmented
// reduction; must be called by all 32 lanes.
__device__ __forceinline__ void warp_deposit(const JobDev& J, const SlotDev& S, uint32_t key, float fx, float fy) {
  const int lane = lane_id();
  const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
  const bool head = (lane == 0) || (key != prev);
  const unsigned heads = __ballot_sync(0xffffffffu, head);
  const int seg = __popc(heads & (0xffffffffu >> (31 - lane)));
  const float w00 = (1.f - fx) * (1.f - fy), w10 = fx * (1.f - fy), w01 = (1.f - fx) * fy, w11 = fx * fy;
  const bool valid = key != PIC_CELL_OUT;
  const int i = cell_i(key), j = cell_j(key);
  const size_t a = (size_t)j * J.nx + i;
  if (J.deposit_mode == 0) {
    const float q = S.qdep;
    float v0 = valid ? q * w00 : 0.f, v1 = valid ? q * w10 : 0.f, v2 = valid ? q * w01 : 0.f, v3 = valid ? q * w11 : 0.f;
    seg_reduce4(v0, v1, v2, v3, seg);
    if (head && valid) {
      float* rho = J.rho_f;
      atomicAdd(rho + a, v0);
      atomicAdd(rho + a + 1, v1);
      atomicAdd(rho + a + J.nx, v2);
      atomicAdd(rho + a + J.nx + 1, v3);
    }
  } else {
    const double Q = (double)S.qfix;
    long long v0 = 0, v1 = 0, v2 = 0, v3 = 0;
    if (valid) {
      v0 = __double2ll_rn((double)w00 * Q);
      v1 = __double2ll_rn((double)w10 * Q);
      v2 = __double2ll_rn((double)w01 * Q);
      v3 = S.qfix - v0 - v1 - v2;
    }
    seg_reduce4(v0, v1, v2, v3, seg);
    if (head && valid) {
      unsigned long long* rho = (unsigned long long*)J.rho_i;
      atomicAdd(rho + a, (unsigned long long)v0);
      atomicAdd(rho + a + 1, (unsigned long long)v1);
      atomicAdd(rho + a + J.nx, (unsigned long long)v2);
      atomicAdd(rho + a + J.nx + 1, (unsigned long long)v3);
    }
  }
}

__global__ void __launch_bounds__(PIC_MOVER_THREADS)
mover_kernel(const JobDev* __restrict__ jobs, JobState* __restrict__ st, const SlotDev* __restrict__ slots,
             const int* __restrict__ counts, int* __restrict__ hit_counts, const int* __restrict__ chunk_prefix,
             int nslots, int flags, uint32_t explicit_step) {
  const int total = chunk_prefix[nslots];
  for (int g = blockIdx.x; g < total; g += gridDim.x) {
    // chunk -> slot (binary search on the exclusive prefix)
    int lo = 0, hi = nslots - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (chunk_prefix[mid] <= g) lo = mid; else hi = mid - 1;
    }
    const int s = lo;
    const SlotDev& S = slots[s];
    const JobDev& J = jobs[S.job];
    JobState& T = st[S.job];
    const int n = counts[s];
    const int base = (g - chunk_prefix[s]) * PIC_CHUNK + 4 * threadIdx.x;

    const bool gated = flags & PIC_PHASE_GATED_I;
    const bool pending = T.kick_pending != 0;
    const bool do_kick = (flags & PIC_PHASE_KICK_I) && (!gated || pending);
    const bool do_mcc = (flags & PIC_PHASE_MCC_I) && (!gated || pending) && J.mcc_mode != 0 &&
                        (J.mcc_mode == 2 ? S.n_proc > 0 : S.n_proc > 0);
    const bool do_drift = flags & PIC_PHASE_DRIFT_I;
    const bool do_walls = (flags & PIC_PHASE_WALLS_I) && J.wall_mode != 0;
    const bool do_dep = flags & PIC_PHASE_DEPOSIT_I;
    const uint32_t mcc_step = gated ? (uint32_t)(T.step - 1) : explicit_step;

    // vector loads (arrays are allocated in whole chunks, so the tail is in bounds)
    const uint4 c4 = *reinterpret_cast<const uint4*>(S.cell + base);
    const float4 fx4 = *reinterpret_cast<const float4*>(S.fx + base);
    const float4 fy4 = *reinterpret_cast<const float4*>(S.fy + base);
    float4 vx4 = *reinterpret_cast<const float4*>(S.vx + base);
    float4 vy4 = *reinterpret_cast<const float4*>(S.vy + base);
    float4 vz4 = make_float4(0.f, 0.f, 0.f, 0.f);
    uint4 pid4 = make_uint4(0, 0, 0, 0);
    if (do_mcc) {
      vz4 = *reinterpret_cast<const float4*>(S.vz + base);
      pid4 = *reinterpret_cast<const uint4*>(S.pid + base);
    }
    uint32_t cl[4] = {c4.x, c4.y, c4.z, c4.w};
    float px[4] = {fx4.x, fx4.y, fx4.z, fx4.w}, py[4] = {fy4.x, fy4.y, fy4.z, fy4.w};
    float vx[4] = {vx4.x, vx4.y, vx4.z, vx4.w}, vy[4] = {vy4.x, vy4.y, vy4.z, vy4.w};
    float vz[4] = {vz4.x, vz4.y, vz4.z, vz4.w};
    const uint32_t pd[4] = {pid4.x, pid4.y, pid4.z, pid4.w};
    double ke = 0.0;
    unsigned ncoll[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    PhiGather pg{J.phi32, J.nx, J.ny};

#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int p = base + r;
      const bool valid = p < n;
      uint32_t c = cl[r];
      const bool in_grid = valid && c != PIC_CELL_OUT;
      const int i = in_grid ? cell_i(c) : 0, j = in_grid ? cell_j(c) : 0;
      // ---- kick
      if (do_kick && in_grid) {
        float gx, gy;
        gather_dphi(pg, i, j, px[r], py[r], gx, gy);
        vx[r] += S.kx * gx;
        vy[r] += S.ky * gy;
      }
      // ---- collisions
      if (do_mcc && valid) {
        float u[4];
        draw4(J.seed, pd[r], mcc_step, 0u, u);
        if (J.mcc_mode == 2) {
          const ProcDev& P = J.procs[S.first_proc];
          const float v2 = vx[r] * vx[r] + vy[r] * vy[r];
          const float sp = sqrtf(v2);
          const float E = S.half_m_over_e * v2;
          const float Pc = 1.f - expf(-J.gas_density * xs_lookup(P, E) * sp * J.dt);
          if (u[0] < Pc) {
            float sn, cs;
            sincospif(2.f * u[1], &sn, &cs);
            vx[r] = sp * cs; vy[r] = sp * sn;
            ncoll[0]++;
          }
        } else if (u[0] < S.pnull) {
          const float v2 = vx[r] * vx[r] + vy[r] * vy[r] + vz[r] * vz[r];
          const float sp = sqrtf(v2);
          const float E = S.half_m_over_e * v2;
          const float target = u[1] * S.numax;
          float acc = 0.f;
          int chosen = -1;
          for (int q = 0; q < S.n_proc; ++q) {
            acc += J.gas_density * xs_lookup(J.procs[S.first_proc + q], E) * sp;
            if (target < acc) { chosen = q; break; }
          }
          if (chosen >= 0) {
            const ProcDev& P = J.procs[S.first_proc + chosen];
            float d[3];
            bool real = true;
            if (P.type == 1) {  // elastic
              iso_dir(u[2], u[3], d);
              const float cosx = sp > 0.f ? (vx[r] * d[0] + vy[r] * d[1] + vz[r] * d[2]) / sp : 1.f;
              const float Ep = E * (1.f - 2.f * S.mass / J.gas_mass * (1.f - cosx));
              const float vn = sqrtf(fmaxf(0.f, Ep) / S.half_m_over_e);
              vx[r] = vn * d[0]; vy[r] = vn * d[1]; vz[r] = vn * d[2];
            } else if (P.type == 2) {  // excitation
              if (E < P.threshold) real = false;
              else {
                iso_dir(u[2], u[3], d);
                const float vn = sqrtf((E - P.threshold) / S.half_m_over_e);
                vx[r] = vn * d[0]; vy[r] = vn * d[1]; vz[r] = vn * d[2];
              }
            } else if (P.type == 3) {  // ionisation
              if (E < P.threshold) real = false;
              else {
                float u2[4];
                draw4(J.seed, pd[r], mcc_step, 1u, u2);
                const float Er = E - P.threshold, B = 10.f;
                const float Eej = B * tanf(u2[0] * atanf(Er / (2.f * B)));
                const float Esc = fmaxf(0.f, Er - Eej);
                iso_dir(u[2], u[3], d);
                const float vs = sqrtf(Esc / S.half_m_over_e);
                Event ev;
                ev.parent_pid = pd[r]; ev.cell = c; ev.fx = px[r]; ev.fy = py[r];
                float d2[3];
                iso_dir(u2[1], u2[2], d2);
                const SlotDev& SE = slots[J.slot0 + J.ion_e_species];
                const float ve = sqrtf(Eej / SE.half_m_over_e);
                ev.ve[0] = ve * d2[0]; ev.ve[1] = ve * d2[1]; ev.ve[2] = ve * d2[2];
                neutral_velocity(J.seed, pd[r], mcc_step, J.vth_neutral, ev.vi);
                const int k = atomicAdd(&T.event_count, 1);
                if (k < J.event_capacity) J.events[k] = ev;
                else atomicOr(&T.status, PIC_ST_EVENTS);
                vx[r] = vs * d[0]; vy[r] = vs * d[1]; vz[r] = vs * d[2];
              }
            } else if (P.type == 4) {  // charge exchange
              float vn[3];
              neutral_velocity(J.seed, pd[r], mcc_step, J.vth_neutral, vn);
              vx[r] = vn[0]; vy[r] = vn[1]; vz[r] = vn[2];
            }
            if (real) ncoll[chosen & 7]++;
          }
        }
      }
      if (valid && (do_kick || do_mcc)) ke += (double)(vx[r] * vx[r] + vy[r] * vy[r] + vz[r] * vz[r]);
      // ---- drift + walls
      bool absorbed = false;
      float nfx = px[r], nfy = py[r];
      uint32_t nc = c;
      if (do_drift && valid) {
        const Drifted d = drift_particle(J, S, c, px[r], py[r], vx[r], vy[r], do_walls);
        absorbed = d.absorbed; nc = d.cell; nfx = d.fx; nfy = d.fy;
      }
      const int hslot = warp_append(valid && absorbed, hit_counts + s);
      if (hslot >= 0) S.hits[hslot] = p;
      // ---- deposit at the new position
      if (do_dep) warp_deposit(J, S, (valid && !absorbed) ? nc : PIC_CELL_OUT, nfx, nfy);
      cl[r] = nc; px[r] = nfx; py[r] = nfy;
    }
    // ---- write back
    if (do_drift) {
      if (base + 3 < n) {
        *reinterpret_cast<uint4*>(S.cell + base) = make_uint4(cl[0], cl[1], cl[2], cl[3]);
        *reinterpret_cast<float4*>(S.fx + base) = make_float4(px[0], px[1], px[2], px[3]);
        *reinterpret_cast<float4*>(S.fy + base) = make_float4(py[0], py[1], py[2], py[3]);
      } else {
        for (int r = 0; r < 4; ++r)
          if (base + r < n) { S.cell[base + r] = cl[r]; S.fx[base + r] = px[r]; S.fy[base + r] = py[r]; }
      }
    }
    if (do_kick || do_mcc) {
      if (base + 3 < n) {
        *reinterpret_cast<float4*>(S.vx + base) = make_float4(vx[0], vx[1], vx[2], vx[3]);
        *reinterpret_cast<float4*>(S.vy + base) = make_float4(vy[0], vy[1], vy[2], vy[3]);
        if (do_mcc) *reinterpret_cast<float4*>(S.vz + base) = make_float4(vz[0], vz[1], vz[2], vz[3]);
      } else {
        for (int r = 0; r < 4; ++r)
          if (base + r < n) {
            S.vx[base + r] = vx[r]; S.vy[base + r] = vy[r];
            if (do_mcc) S.vz[base + r] = vz[r];
          }
      }
    }
    // ---- diagnostics: kinetic energy and collision counts (one atomic per warp)
    if (do_kick || do_mcc) {
      for (int o = 16; o; o >>= 1) ke += __shfl_down_sync(0xffffffffu, ke, o);
      if (lane_id() == 0 && ke != 0.0) atomicAdd(&T.ke[S.species], ke * S.ke_factor);
    }
    if (do_mcc) {
      for (int q = 0; q < S.n_proc && q < 8; ++q) {
        const unsigned tot = __reduce_add_sync(0xffffffffu, ncoll[q]);
        if (lane_id() == 0 && tot) atomicAdd(&T.collisions[S.species][q], (unsigned long long)tot);
      }
    }
  }
}

// Exclusive prefix of mover chunks per slot (one CTA; slots are few).
__global__ void chunk_table_kernel(const int* __restrict__ counts, const uint8_t* __restrict__ active,
                                   int* __restrict__ chunk_prefix, int nslots) {
  __shared__ int acc;
  if (threadIdx.x == 0) {
    int a = 0;
    for (int s = 0; s < nslots; ++s) {
      chunk_prefix[s] = a;
      if (!active || active[s]) a += (counts[s] + PIC_CHUNK - 1) / PIC_CHUNK;
    }
    chunk_prefix[nslots] = a;
    acc = a;
  }
}

int launch_mover(const EngineLaunch& L, int flags, uint32_t explicit_step, cudaStream_t stream) {
  chunk_table_kernel<<<1, 32, 0, stream>>>(L.counts, L.active, L.chunk_prefix, L.nslots);
  if (L.ev_mover_begin) cudaEventRecord(L.ev_mover_begin, stream);
  mover_kernel<<<L.mover_grid, PIC_MOVER_THREADS, 0, stream>>>(L.jobs, L.st, L.slots, L.counts, L.hit_counts,
                                                              L.chunk_prefix, L.nslots, flags, explicit_step);
  if (L.ev_mover_end) cudaEventRecord(L.ev_mover_end, stream);
  return 2;
}
