// mover.cu — the fused particle pass of one PIC step.
//
// One pass over each particle slot does, in the reference's order (main.cu:64-134):
//   kick     updateParticleVelocities (kernels.cu:71-131): E bilinearly gathered from the
//            node field that efield32_kernel computes once per step from the FP64 potential
//            with the computeElectricField stencils (kernels.cu:134-191)
//   MCC      null-collision Monte Carlo (or the reference's elastic form, mcc.cu:56-85)
//   drift    update_coordinates (kernels.cu:8-23) on cell-relative FP32 positions
//   walls    detect_intersections (collisions.cu:7-54) / box absorption; hits are appended
//            with warp-aggregated atomics (compaction happens in compact.cu)
//   deposit  updateDensity (kernels.cu:26-69) at the new position: per warp a segmented
//            reduction over lanes that share a cell (particles are counting-sorted by cell),
//            then one atomic per node per segment; FP32 or int64 fixed point.
// The kick + MCC of step k are fused into the pass of step k+1 (the job's kick_pending
// flag); an explicit flush applies them before any read-back.
#include <algorithm>
#include "common.cuh"
#include "kernels.h"
#include "particle_ops.cuh"
#include "tma.cuh"

namespace {

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

// 512-particle chunks and 5 CTAs (40 warps) per SM (47 registers, no spills).  Measured on
// B200 (1025^2, 2e7 particles): 1024-particle chunks at 2 CTAs per SM take 15% longer than
// 512 at 4, and 5 CTAs per SM take 3% less than 4 (0.574 against 0.593 ms per pass).
#ifndef PIC_MOVER_MIN_BLOCKS
#define PIC_MOVER_MIN_BLOCKS 5
#endif
constexpr int kRounds = PIC_CHUNK / PIC_MOVER_THREADS;
constexpr int kWarps = PIC_MOVER_THREADS / 32;

// One real-or-null collision of a null-collision candidate (Vahedi & Surendra 1995): the
// candidate's process is chosen with u1 * nu_max against the cumulative n sigma_j(E) v.
__device__ void collide(const JobDev& J, const SlotDev& S, const SlotDev* slots, JobState& T, uint32_t pid,
                        uint32_t cell, float fx, float fy, float& vx, float& vy, float& vz, const float u[4],
                        uint32_t step, unsigned* proc_count) {
  const float v2 = vx * vx + vy * vy + vz * vz;
  const float sp = sqrtf(v2);
  const float E = S.half_m_over_e * v2;
  const float target = u[1] * S.numax;
  float acc = 0.f;
  int chosen = -1;
  for (int q = 0; q < S.n_proc; ++q) {
    acc += J.gas_density * xs_lookup(J.procs[S.first_proc + q], E) * sp;
    if (target < acc) { chosen = q; break; }
  }
  if (chosen < 0) return;
  const ProcDev& P = J.procs[S.first_proc + chosen];
  float d[3];
  if (P.type == PIC_PROC_ELASTIC) {
    iso_dir(u[2], u[3], d);
    const float cosx = sp > 0.f ? (vx * d[0] + vy * d[1] + vz * d[2]) / sp : 1.f;
    const float Ep = E * (1.f - 2.f * S.mass / J.gas_mass * (1.f - cosx));
    const float vn = sqrtf(fmaxf(0.f, Ep) / S.half_m_over_e);
    vx = vn * d[0]; vy = vn * d[1]; vz = vn * d[2];
  } else if (P.type == PIC_PROC_EXCITATION) {
    if (E < P.threshold) return;
    iso_dir(u[2], u[3], d);
    const float vn = sqrtf((E - P.threshold) / S.half_m_over_e);
    vx = vn * d[0]; vy = vn * d[1]; vz = vn * d[2];
  } else if (P.type == PIC_PROC_IONIZATION) {
    if (E < P.threshold) return;
    float u2[4];
    draw4(J.seed, pid, step, 1u, u2);
    const float Er = E - P.threshold, B = 10.f;
    const float Eej = B * tanf(u2[0] * atanf(Er / (2.f * B)));
    const float Esc = fmaxf(0.f, Er - Eej);
    iso_dir(u[2], u[3], d);
    const float vs = sqrtf(Esc / S.half_m_over_e);
    Event ev;
    ev.parent_pid = pid; ev.cell = cell; ev.fx = fx; ev.fy = fy;
    float d2[3];
    iso_dir(u2[1], u2[2], d2);
    const SlotDev& SE = slots[J.slot0 + J.ion_e_species];
    const float ve = sqrtf(Eej / SE.half_m_over_e);
    ev.ve[0] = ve * d2[0]; ev.ve[1] = ve * d2[1]; ev.ve[2] = ve * d2[2];
    neutral_velocity(J.seed, pid, step, J.vth_neutral, ev.vi);
    const int k = atomicAdd(&T.event_count, 1);
    if (k < J.event_capacity) J.events[k] = ev;
    else atomicOr(&T.status, PIC_ST_EVENTS);
    vx = vs * d[0]; vy = vs * d[1]; vz = vs * d[2];
  } else if (P.type == PIC_PROC_CHARGE_EXCHANGE) {
    float vn[3];
    neutral_velocity(J.seed, pid, step, J.vth_neutral, vn);
    vx = vn[0]; vy = vn[1]; vz = vn[2];
  }
  atomicAdd(&proc_count[chosen & 7], 1u);
}

// E per unit cell (-dphi across one cell) at every node of every job, from the job's
// current FP64 potential with the computeElectricField stencils (kernels.cu:134-191):
// (phi[i-1] - phi[i+1]) / 2 inside, phi[i] - phi[i+1] on the first and phi[i-1] - phi[i]
// on the last node of a row, the same along columns; rounded to FP32 once.  Job j uses
// blockIdx.y == j and a grid-stride loop over its nodes.
__global__ void __launch_bounds__(256) efield32_kernel(const JobDev* __restrict__ jobs, const JobState* __restrict__ st) {
  const JobDev& J = jobs[blockIdx.y];
  float2* const out = J.efield;
  if (!out) return;
  const double* __restrict__ phi = J.phi64[st[blockIdx.y].phi_cur];
  const int nx = J.nx, ny = J.ny, N = nx * ny;
  for (int k = blockIdx.x * 256 + threadIdx.x; k < N; k += gridDim.x * 256) {
    const int j = k / nx, i = k - j * nx;
    const int il = i > 0 ? i - 1 : 0, ir = i < nx - 1 ? i + 1 : nx - 1;
    const int jl = j > 0 ? j - 1 : 0, jr = j < ny - 1 ? j + 1 : ny - 1;
    const double sx = (i > 0 && i < nx - 1) ? 0.5 : 1.0, sy = (j > 0 && j < ny - 1) ? 0.5 : 1.0;
    const double ex = (phi[j * nx + il] - phi[j * nx + ir]) * sx;
    const double ey = (phi[jl * nx + i] - phi[jr * nx + i]) * sy;
    out[k] = make_float2((float)ex, (float)ey);
  }
}

// Particle arrays of one chunk staged in shared memory.
enum { A_CELL = 0, A_FX, A_FY, A_VX, A_VY, A_VZ, A_PID, kNArr };
constexpr int kChunkBytes = PIC_CHUNK * 4;
constexpr size_t kMoverDynSmem = 2ull * kNArr * kChunkBytes;

__device__ __forceinline__ int chunk_slot(const int* __restrict__ chunk_prefix, int nslots, int g) {
  int lo = 0, hi = nslots - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (chunk_prefix[mid] <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Issue the bulk copies of chunk g into buffer b (one thread).  vz and pid are staged only
// for jobs with collisions.
__device__ __forceinline__ void issue_chunk(const JobDev* __restrict__ jobs, const SlotDev* __restrict__ slots,
                                            const int* __restrict__ chunk_prefix, int nslots, int g, uint32_t* buf,
                                            uint64_t* mbar) {
  const int s = chunk_slot(chunk_prefix, nslots, g);
  const SlotDev& S = slots[s];
  const size_t base = (size_t)(g - chunk_prefix[s]) * PIC_CHUNK;
  const bool mcc = jobs[S.job].mcc_mode != 0 && S.n_proc > 0;
  tma::mbar_arrive_expect_tx(mbar, (uint32_t)(kChunkBytes * (mcc ? 7 : 5)));
  tma::bulk_g2s(buf + A_CELL * PIC_CHUNK, S.cell + base, kChunkBytes, mbar);
  tma::bulk_g2s(buf + A_FX * PIC_CHUNK, S.fx + base, kChunkBytes, mbar);
  tma::bulk_g2s(buf + A_FY * PIC_CHUNK, S.fy + base, kChunkBytes, mbar);
  tma::bulk_g2s(buf + A_VX * PIC_CHUNK, S.vx + base, kChunkBytes, mbar);
  tma::bulk_g2s(buf + A_VY * PIC_CHUNK, S.vy + base, kChunkBytes, mbar);
  if (mcc) {
    tma::bulk_g2s(buf + A_VZ * PIC_CHUNK, S.vz + base, kChunkBytes, mbar);
    tma::bulk_g2s(buf + A_PID * PIC_CHUNK, S.pid + base, kChunkBytes, mbar);
  }
}

// One chunk = PIC_CHUNK particles of one slot; warp w owns the contiguous entries
// [w * kPerWarp, (w + 1) * kPerWarp), lane l handles w * kPerWarp + r * 32 + l.
// Chunks reach shared memory through bulk asynchronous copies, double buffered: while the
// CTA works on chunk k, chunk k+1 is in flight, so HBM latency is covered by the copy engine
// rather than by resident warps; results return with bulk stores.
//  pass A  kick and the null-collision candidate test.  E comes from the per-step node field
//          (float2 loads; particles are cell-sorted, so a warp's loads hit a few cache lines);
//          candidates (~nu_max dt of the particles) are listed per warp and collided by that
//          warp's lanes afterwards
//  pass B  drift, absorption, hit list and CIC deposit
// Two block barriers per chunk (chunk data ready; results complete before the bulk stores),
// a third only when the chunk starts a new slot and the slot and job tables are copied to
// shared memory (every parameter read in the per-particle code is a shared-memory load).
__global__ void __launch_bounds__(PIC_MOVER_THREADS, PIC_MOVER_MIN_BLOCKS)
mover_kernel(const JobDev* __restrict__ jobs, JobState* __restrict__ st, const SlotDev* __restrict__ slots,
             const int* __restrict__ counts, int* __restrict__ hit_counts, const int* __restrict__ chunk_prefix,
             int nslots, int flags, uint32_t explicit_step) {
  extern __shared__ __align__(128) uint32_t dsm[];
  constexpr int kPerWarp = PIC_CHUNK / kWarps;
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ int wlist[kWarps][kPerWarp];
  __shared__ int wcount[kWarps];
  __shared__ unsigned proc_count[8];
  __shared__ double ke_sh[kWarps];
  __shared__ SlotDev sS;
  __shared__ JobDev sJ;
  __shared__ int cur_slot;
  __shared__ int abort_flag;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int wbase = warp * kPerWarp;
  const int total = chunk_prefix[nslots];
  if (t == 0) {
    cur_slot = -1;
    abort_flag = 0;
    tma::mbar_init(&mbar[0], 1);
    tma::mbar_init(&mbar[1], 1);
    tma::fence_mbar_init();
  }
  if (t < 8) proc_count[t] = 0u;
  __syncthreads();
  uint32_t parity[2] = {0u, 0u};
  if (t == 0 && (int)blockIdx.x < total) issue_chunk(jobs, slots, chunk_prefix, nslots, blockIdx.x, dsm, &mbar[0]);
  int k = 0;
  for (int g = blockIdx.x; g < total; g += gridDim.x, ++k) {
    const int b = k & 1;
    uint32_t* buf = dsm + b * kNArr * PIC_CHUNK;
    // prefetch the next chunk into the other buffer, once the bulk stores of the chunk that
    // used it have read their source (every thread finished with that buffer before the
    // previous iteration's second barrier)
    if (t == 0 && g + (int)gridDim.x < total) {
      tma::bulk_wait_read_all();
      issue_chunk(jobs, slots, chunk_prefix, nslots, g + gridDim.x, dsm + (b ^ 1) * kNArr * PIC_CHUNK, &mbar[b ^ 1]);
    }
    const int s = chunk_slot(chunk_prefix, nslots, g);
    if (cur_slot != s) {  // uniform: cur_slot changed before the previous iteration's last barrier
      __syncthreads();    // thread 0 may still read the old tables for the previous chunk's stores
      const int* srcS = reinterpret_cast<const int*>(slots + s);
      const int* srcJ = reinterpret_cast<const int*>(jobs + slots[s].job);
      int* dS = reinterpret_cast<int*>(&sS);
      int* dJ = reinterpret_cast<int*>(&sJ);
      for (int q = t; q < (int)(sizeof(SlotDev) / 4); q += PIC_MOVER_THREADS) dS[q] = srcS[q];
      for (int q = t; q < (int)(sizeof(JobDev) / 4); q += PIC_MOVER_THREADS) dJ[q] = srcJ[q];
    }
    // wait for this chunk's data (bounded)
    if (!tma::mbar_wait(&mbar[b], parity[b])) atomicOr(&abort_flag, 1);
    parity[b] ^= 1u;
    __syncthreads();
    if (abort_flag) {
      if (t == 0) atomicOr(&st[slots[s].job].status, PIC_ST_TIMEOUT);
      break;
    }
    if (t == 0) cur_slot = s;
    const SlotDev& S = sS;
    const JobDev& J = sJ;
    JobState& T = st[S.job];
    const int n = counts[s];
    const int base = (g - chunk_prefix[s]) * PIC_CHUNK;
    const bool gated = flags & PIC_PHASE_GATED_I;
    const bool pending = T.kick_pending != 0;
    const bool do_kick = (flags & PIC_PHASE_KICK_I) && (!gated || pending);
    const bool do_mcc = (flags & PIC_PHASE_MCC_I) && (!gated || pending) && J.mcc_mode != 0 && S.n_proc > 0;
    const bool do_drift = flags & PIC_PHASE_DRIFT_I;
    const bool do_walls = (flags & PIC_PHASE_WALLS_I) && J.wall_mode != 0;
    const bool do_dep = flags & PIC_PHASE_DEPOSIT_I;
    const uint32_t mcc_step = gated ? (uint32_t)(T.step - 1) : explicit_step;
    uint32_t* s_cell = buf + A_CELL * PIC_CHUNK;
    float* s_fx = reinterpret_cast<float*>(buf + A_FX * PIC_CHUNK);
    float* s_fy = reinterpret_cast<float*>(buf + A_FY * PIC_CHUNK);
    float* s_vx = reinterpret_cast<float*>(buf + A_VX * PIC_CHUNK);
    float* s_vy = reinterpret_cast<float*>(buf + A_VY * PIC_CHUNK);
    float* s_vz = reinterpret_cast<float*>(buf + A_VZ * PIC_CHUNK);
    const uint32_t* s_pid = buf + A_PID * PIC_CHUNK;

    // ---- pass A: kick and collisions
    if (do_kick || do_mcc) {
      const float2* __restrict__ ef = J.efield;
      const int enx = J.nx;
      if (lane == 0) wcount[warp] = 0;
      __syncwarp();
#pragma unroll
      for (int r = 0; r < kRounds; ++r) {
        const int q = wbase + r * 32 + lane;
        const bool valid = base + q < n;
        bool cand = false;
        if (valid) {
          const uint32_t c = s_cell[q];
          float vx = s_vx[q], vy = s_vy[q];
          if (do_kick && c != PIC_CELL_OUT) {
            float gx, gy;
            const float fx = s_fx[q], fy = s_fy[q];
            const float2* e0 = ef + cell_j(c) * enx + cell_i(c);
            const float2 e00 = __ldg(e0), e10 = __ldg(e0 + 1), e01 = __ldg(e0 + enx), e11 = __ldg(e0 + enx + 1);
            const float w00 = (1.f - fx) * (1.f - fy), w10 = fx * (1.f - fy), w01 = (1.f - fx) * fy, w11 = fx * fy;
            gx = w00 * e00.x + w10 * e10.x + w01 * e01.x + w11 * e11.x;
            gy = w00 * e00.y + w10 * e10.y + w01 * e01.y + w11 * e11.y;
            vx += S.kx * gx;
            vy += S.ky * gy;
          }
          if (do_mcc) {
            if (J.mcc_mode == 2) {
              float u[4];
              draw4(J.seed, s_pid[q], mcc_step, 0u, u);
              const ProcDev& P = J.procs[S.first_proc];
              const float v2 = vx * vx + vy * vy;
              const float sp = sqrtf(v2);
              const float Pc = 1.f - expf(-J.gas_density * xs_lookup(P, S.half_m_over_e * v2) * sp * J.dt);
              if (u[0] < Pc) {
                float sn, cs;
                sincospif(2.f * u[1], &sn, &cs);
                vx = sp * cs; vy = sp * sn;
                atomicAdd(&proc_count[0], 1u);
              }
            } else {
              cand = draw_first(J.seed, s_pid[q], mcc_step, 0u) < S.pnull;
            }
          }
          s_vx[q] = vx;
          s_vy[q] = vy;
        }
        const unsigned m = __ballot_sync(0xffffffffu, cand);
        if (cand) wlist[warp][wcount[warp] + __popc(m & ((1u << lane) - 1u))] = q;
        __syncwarp();
        if (lane == 0) wcount[warp] += __popc(m);
        __syncwarp();
      }
      const int ncand = wcount[warp];
      for (int c = lane; c < ncand; c += 32) {
        const int q = wlist[warp][c];
        float u[4];
        const uint32_t pid = s_pid[q];
        draw4(J.seed, pid, mcc_step, 0u, u);
        float vx = s_vx[q], vy = s_vy[q], vz = s_vz[q];
        collide(J, S, slots, T, pid, s_cell[q], s_fx[q], s_fy[q], vx, vy, vz, u, mcc_step, proc_count);
        s_vx[q] = vx; s_vy[q] = vy; s_vz[q] = vz;
      }
      __syncwarp();
    }

    // ---- pass B: drift, walls, deposit
    double ke = 0.0;
    const bool want_ke = do_kick || do_mcc;
    if (do_drift || do_dep || want_ke) {
#pragma unroll
      for (int r = 0; r < kRounds; ++r) {
        const int q = wbase + r * 32 + lane;
        const bool valid = base + q < n;
        uint32_t c = PIC_CELL_OUT;
        float fx = 0.f, fy = 0.f, vx = 0.f, vy = 0.f;
        if (valid) { c = s_cell[q]; fx = s_fx[q]; fy = s_fy[q]; vx = s_vx[q]; vy = s_vy[q]; }
        if (valid && want_ke) {
          const float vz = do_mcc ? s_vz[q] : 0.f;
          ke += (double)(vx * vx + vy * vy + vz * vz);
        }
        bool absorbed = false;
        uint32_t nc = c;
        float nfx = fx, nfy = fy;
        if (do_drift && valid) {
          const Drifted d = drift_particle(J, S, c, fx, fy, vx, vy, do_walls);
          absorbed = d.absorbed; nc = d.cell; nfx = d.fx; nfy = d.fy;
        }
        if (do_walls) {
          const int hslot = warp_append(valid && absorbed, hit_counts + s);
          if (hslot >= 0) S.hits[hslot] = base + q;
        }
        if (do_dep) warp_deposit(J, S, (valid && !absorbed) ? nc : PIC_CELL_OUT, nfx, nfy);
        if (valid && do_drift) { s_cell[q] = nc; s_fx[q] = nfx; s_fy[q] = nfy; }
      }
    }
    // ---- results back to global memory with bulk stores
    tma::fence_proxy_async();
    if (want_ke) {
      for (int o = 16; o; o >>= 1) ke += __shfl_down_sync(0xffffffffu, ke, o);
      if (lane == 0) ke_sh[warp] = ke;
    }
    __syncthreads();
    if (t == 0) {
      if (do_drift) {
        tma::bulk_s2g(S.cell + base, s_cell, kChunkBytes);
        tma::bulk_s2g(S.fx + base, s_fx, kChunkBytes);
        tma::bulk_s2g(S.fy + base, s_fy, kChunkBytes);
      }
      if (do_kick || do_mcc) {
        tma::bulk_s2g(S.vx + base, s_vx, kChunkBytes);
        tma::bulk_s2g(S.vy + base, s_vy, kChunkBytes);
      }
      if (do_mcc) tma::bulk_s2g(S.vz + base, s_vz, kChunkBytes);
      tma::bulk_commit();
      if (want_ke) {
        double tk = 0.0;
        for (int w = 0; w < kWarps; ++w) tk += ke_sh[w];
        if (tk != 0.0) atomicAdd(&T.ke[S.species], tk * S.ke_factor);
      }
      // read and clear the collision counters; the next chunk's collisions start after its
      // first barrier, which thread 0 reaches only after this
      for (int p = 0; p < 8; ++p) {
        const unsigned c = proc_count[p];
        if (c) {
          atomicAdd(&T.collisions[S.species][p], (unsigned long long)c);
          proc_count[p] = 0u;
        }
      }
    }
  }
  if (t == 0) tma::bulk_wait_all();
}

// Exclusive prefix of mover chunks per slot (one CTA; slots are few).
__global__ void chunk_table_kernel(const int* __restrict__ counts, const uint8_t* __restrict__ active,
                                   int* __restrict__ chunk_prefix, int nslots) {
  if (threadIdx.x == 0) {
    int a = 0;
    for (int s = 0; s < nslots; ++s) {
      chunk_prefix[s] = a;
      if (!active || active[s]) a += (counts[s] + PIC_CHUNK - 1) / PIC_CHUNK;
    }
    chunk_prefix[nslots] = a;
  }
}

int mover_blocks_per_sm() {
  cudaFuncSetAttribute(mover_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMoverDynSmem);
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, mover_kernel, PIC_MOVER_THREADS, kMoverDynSmem) != cudaSuccess ||
      b < 1) {
    cudaGetLastError();
    b = 1;
  }
  return b;
}

int launch_mover(const EngineLaunch& L, int flags, uint32_t explicit_step, cudaStream_t stream) {
  int k = 2;
  if ((flags & PIC_PHASE_KICK_I) && L.njobs > 0) {
    // the node field of every job's current potential, for the kick
    const int gx = std::max(1, std::min(4096, 8 * L.num_sms / L.njobs));
    efield32_kernel<<<dim3(gx, L.njobs), 256, 0, stream>>>(L.jobs, L.st);
    ++k;
  }
  chunk_table_kernel<<<1, 32, 0, stream>>>(L.counts, L.active, L.chunk_prefix, L.nslots);
  if (L.ev_mover_begin) cudaEventRecord(L.ev_mover_begin, stream);
  mover_kernel<<<L.mover_grid, PIC_MOVER_THREADS, kMoverDynSmem, stream>>>(L.jobs, L.st, L.slots, L.counts,
                                                                          L.hit_counts, L.chunk_prefix, L.nslots, flags,
                                                                          explicit_step);
  if (L.ev_mover_end) cudaEventRecord(L.ev_mover_end, stream);
  return k;
}
