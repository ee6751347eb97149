// mover.cu — the fused particle pass of one PIC step.
//
// One pass over each particle slot does, in the reference's order (main.cu:64-134):
//   kick     updateParticleVelocities (kernels.cu:71-131): E bilinearly gathered from the
//            node field that efield32_kernel computes once per step from the FP64 potential
//            with the computeElectricField stencils (kernels.cu:134-191)
//   MCC      null-collision Monte Carlo (or the reference's elastic form, mcc.cu:56-85)
//   drift    update_coordinates (kernels.cu:8-23) on cell-relative FP32 positions
//   walls    detect_intersections (collisions.cu:7-54) / box absorption; hits are appended
//            with one atomic per warp item (compaction happens in compact.cu)
//   deposit  updateDensity (kernels.cu:26-69) at the new position: runs of equal cells are
//            summed in registers (particles are counting-sorted by cell), then a warp-segmented
//            reduction and one atomic per node per segment; FP32 or int64 fixed point.
// The kick + MCC of step k are fused into the pass of step k+1 (the job's kick_pending
// flag); an explicit flush applies them before any read-back.
#include <algorithm>
#include "common.cuh"
#include "kernels.h"
#include "particle_ops.cuh"

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

// Segmented sums towards each segment's first lane; maxlen (warp-uniform) bounds the segment
// lengths, so only ceil(log2(maxlen)) shuffle levels run.
template <typename T>
__device__ __forceinline__ void seg_reduce4(T& a, T& b, T& c, T& d, int seg, int maxlen) {
  const int lane = lane_id();
  for (int o = 1; o < maxlen; o <<= 1) {
    const T ta = __shfl_down_sync(0xffffffffu, a, o);
    const T tb = __shfl_down_sync(0xffffffffu, b, o);
    const T tc = __shfl_down_sync(0xffffffffu, c, o);
    const T td = __shfl_down_sync(0xffffffffu, d, o);
    const int ts = __shfl_down_sync(0xffffffffu, seg, o);
    if (lane + o < 32 && ts == seg) { a += ta; b += tb; c += tc; d += td; }
  }
}

}  // namespace

// Particles per lane and per warp work item: lane l of a warp holds particles kPPL l ..
// kPPL l + kPPL - 1 of a (32 kPPL)-particle item in registers, loaded with one vector load per
// array (contiguous per warp and array).  Capacities are multiples of PIC_CHUNK, so every item
// lies inside the arrays.  With the CTAs per SM below, measured on B200 (1025^2, 2e7
// particles, ms per pass): 2 per lane at 4 CTAs per SM 0.441; 2 at 3 CTAs 0.466, at 5 CTAs
// 0.476; 4 per lane at 3 CTAs 0.467, at 4 CTAs 0.510 (register spills).
#ifndef PIC_MOVER_PPL
#define PIC_MOVER_PPL 2
#endif
constexpr int kPPL = PIC_MOVER_PPL;
constexpr int kItem = 32 * kPPL;

// kPPL consecutive 4-byte values of one lane as one evict-first vector load / store.
__device__ __forceinline__ void ld_lane(const float* p, float (&a)[4]) {
  const float4 v = __ldcs(reinterpret_cast<const float4*>(p)); a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w;
}
__device__ __forceinline__ void ld_lane(const float* p, float (&a)[2]) {
  const float2 v = __ldcs(reinterpret_cast<const float2*>(p)); a[0] = v.x; a[1] = v.y;
}
__device__ __forceinline__ void ld_lane(const uint32_t* p, uint32_t (&a)[4]) {
  const uint4 v = __ldcs(reinterpret_cast<const uint4*>(p)); a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w;
}
__device__ __forceinline__ void ld_lane(const uint32_t* p, uint32_t (&a)[2]) {
  const uint2 v = __ldcs(reinterpret_cast<const uint2*>(p)); a[0] = v.x; a[1] = v.y;
}
__device__ __forceinline__ void st_lane(float* p, const float (&a)[4]) {
  __stcs(reinterpret_cast<float4*>(p), make_float4(a[0], a[1], a[2], a[3]));
}
__device__ __forceinline__ void st_lane(float* p, const float (&a)[2]) {
  __stcs(reinterpret_cast<float2*>(p), make_float2(a[0], a[1]));
}
__device__ __forceinline__ void st_lane(uint32_t* p, const uint32_t (&a)[4]) {
  __stcs(reinterpret_cast<uint4*>(p), make_uint4(a[0], a[1], a[2], a[3]));
}
__device__ __forceinline__ void st_lane(uint32_t* p, const uint32_t (&a)[2]) {
  __stcs(reinterpret_cast<uint2*>(p), make_uint2(a[0], a[1]));
}
constexpr int kWarps = PIC_MOVER_THREADS / 32;
#ifndef PIC_MOVER_MIN_BLOCKS
#define PIC_MOVER_MIN_BLOCKS 4
#endif

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

// The slot and job tables of the slot a warp works on, copied to shared memory when the
// warp moves to another slot (every parameter read in the per-particle code is then a
// shared-memory load, and the functions shared with the ionisation kernel take them as is).
struct WarpTables {
  SlotDev S;
  JobDev J;
};

__device__ __forceinline__ void copy_words(void* dst, const void* src, int bytes, int lane) {
  int* d = reinterpret_cast<int*>(dst);
  const int* s = reinterpret_cast<const int*>(src);
  for (int q = lane; q < bytes / 4; q += 32) d[q] = s[q];
}

// Segmented sum of the four corner weights of one run per lane over the warp (runs of equal
// keys in lane order); the head lane of each segment adds the totals to rho.
template <typename V>
__device__ __forceinline__ void warp_runs_deposit(V* rho, int nx, uint32_t key, V v0, V v1, V v2, V v3) {
  const int lane = lane_id();
  const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
  const bool head = (lane == 0) || (key != prev);
  const unsigned heads = __ballot_sync(0xffffffffu, head);
  const int seg = __popc(heads & (0xffffffffu >> (31 - lane)));
  // longest segment: each lane measures its own from its head to the next head
  const unsigned after = lane == 31 ? 0u : heads & (0xfffffffeu << lane);
  const int first = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
  const int next = after ? __ffs(after) - 1 : 32;
  const int maxlen = (int)__reduce_max_sync(0xffffffffu, (unsigned)(next - first));
  seg_reduce4(v0, v1, v2, v3, seg, maxlen);
  if (head && key != PIC_CELL_OUT) {
    V* r = rho + (size_t)cell_j(key) * nx + cell_i(key);
    atomicAdd(r, v0);
    atomicAdd(r + 1, v1);
    atomicAdd(r + nx, v2);
    atomicAdd(r + nx + 1, v3);
  }
}

// CIC weights of one particle (updateDensity, kernels.cu:56-68) in deposit units: FP32, or
// int64 fixed point whose four parts sum to the particle's quantised charge exactly.
__device__ __forceinline__ void cic_f32(float q, float fx, float fy, float& a, float& b, float& c, float& d) {
  a = q * ((1.f - fx) * (1.f - fy)); b = q * (fx * (1.f - fy)); c = q * ((1.f - fx) * fy); d = q * (fx * fy);
}
__device__ __forceinline__ void cic_i64(long long qf, float fx, float fy, long long& a, long long& b, long long& c,
                                        long long& d) {
  const double Q = (double)qf;
  a = __double2ll_rn((double)((1.f - fx) * (1.f - fy)) * Q);
  b = __double2ll_rn((double)(fx * (1.f - fy)) * Q);
  c = __double2ll_rn((double)((1.f - fx) * fy) * Q);
  d = qf - a - b - c;
}

// Deposit of a lane's kPPL particles (keys in lane order): runs of equal keys inside the lane
// are summed in registers; every finished run but the lane's last goes to rho directly, and
// the last runs of all lanes go through one warp-segmented reduction.  Called by all lanes.
template <typename V, typename W>
__device__ __forceinline__ void lane_deposit(V* rho, int nx, const uint32_t key[kPPL], const float fx[kPPL],
                                             const float fy[kPPL], W weights) {
  V a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  uint32_t rk = key[0];
  if (rk != PIC_CELL_OUT) weights(fx[0], fy[0], a0, a1, a2, a3);
#pragma unroll
  for (int k = 1; k < kPPL; ++k) {
    V b0 = 0, b1 = 0, b2 = 0, b3 = 0;
    if (key[k] != PIC_CELL_OUT) weights(fx[k], fy[k], b0, b1, b2, b3);
    if (key[k] == rk) {
      a0 += b0; a1 += b1; a2 += b2; a3 += b3;
    } else {
      if (rk != PIC_CELL_OUT) {
        V* r = rho + (size_t)cell_j(rk) * nx + cell_i(rk);
        atomicAdd(r, a0); atomicAdd(r + 1, a1); atomicAdd(r + nx, a2); atomicAdd(r + nx + 1, a3);
      }
      rk = key[k]; a0 = b0; a1 = b1; a2 = b2; a3 = b3;
    }
  }
  warp_runs_deposit(rho, nx, rk, a0, a1, a2, a3);
}

// Deferred collision candidates of a warp: cell fx fy vx vy vz pid index, up to one round of
// 32 left over plus one item's worth.
constexpr int kQueue = 32 + kItem;
constexpr int kQFields = 8;
constexpr size_t kMoverSmem = (size_t)kWarps * kQFields * kQueue * sizeof(uint32_t);

// The fused particle pass.  Warp w of the grid takes items w, w + W, w + 2W, ... (W warps in
// the grid) over the concatenated items of all active slots; the slot of an item comes from
// the item prefix, and a warp's items only move forward through the slots.  Per item:
//   loads    cell, fx, fy, vx, vy (+ vz, pid with collisions): one evict-first vector load
//            per array and lane
//   pass A   kick (E gathered from the per-step node field; particles are cell-sorted, so a
//            warp's gathers hit a few cache lines) and the null-collision test: candidates
//            (~nu_max dt of the particles) whose collision is real (u1 nu_max below the
//            species' total n sigma_T v, one table lookup) leave the item for the warp's queue
//            in shared memory.  Whenever 32 are queued (and when the warp leaves a slot), one
//            round chooses the process and collides, drifts, deposits and stores them, one
//            per lane, after their owners have stored the rest of their items.
//   pass B   drift, absorption (hits appended with one atomic per item), CIC deposit
//   stores   evict-first vector stores of what changed (vz only in the queue rounds; the
//            cell word only when some particle of the warp crossed a cell edge)
// The particle stream bypasses L2 retention (evict-first loads and stores) so the grids the
// gathers and deposits touch stay resident.  No block-level synchronisation.
__global__ void __launch_bounds__(PIC_MOVER_THREADS, PIC_MOVER_MIN_BLOCKS)
mover_kernel(const JobDev* __restrict__ jobs, JobState* __restrict__ st, const SlotDev* __restrict__ slots,
             const int* __restrict__ counts, int* __restrict__ hit_counts, const int* __restrict__ item_prefix,
             int nslots, int flags, uint32_t explicit_step) {
  extern __shared__ __align__(16) uint32_t qbuf[];
  __shared__ WarpTables tab[kWarps];
  __shared__ unsigned pcount[kWarps][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int total = item_prefix[nslots];
  const SlotDev& S = tab[warp].S;
  const JobDev& J = tab[warp].J;
  unsigned* const pc = pcount[warp];
  uint32_t* const cq = qbuf + (size_t)warp * kQFields * kQueue;   // field f of entry e: cq[f * kQueue + e]
  int qn = 0;                                                      // queued candidates (warp-uniform)
  if (lane < 8) pc[lane] = 0u;
  __syncwarp();
  int cur = -1;
  double ke = 0.0;
  bool do_kick = false, do_mcc = false, do_drift = false, do_walls = false, do_dep = false, want_ke = false;
  uint32_t mcc_step = 0;
  int n = 0;
  // One round over the first cnt queued candidates (one per lane): collide (Philox stream
  // (seed, pid, step) as for the candidate test), drift, absorb, deposit, store at the
  // particle's index; then the queue moves down by cnt.  The owners' stores of these
  // particles were issued before (the barrier orders them first).
  auto round = [&](int cnt) {
    __syncwarp();
    const int s = cur;
    bool absorbed = false;
    int idx = 0;
    if (lane < cnt) {
      uint32_t qc = cq[0 * kQueue + lane];
      float qfx = __uint_as_float(cq[1 * kQueue + lane]), qfy = __uint_as_float(cq[2 * kQueue + lane]);
      float qvx = __uint_as_float(cq[3 * kQueue + lane]), qvy = __uint_as_float(cq[4 * kQueue + lane]);
      float qvz = __uint_as_float(cq[5 * kQueue + lane]);
      const uint32_t qpid = cq[6 * kQueue + lane];
      idx = (int)cq[7 * kQueue + lane];
      float u[4];
      draw4(J.seed, qpid, mcc_step, 0u, u);
      collide(J, S, slots, st[S.job], qpid, qc, qfx, qfy, qvx, qvy, qvz, u, mcc_step, pc);
      if (want_ke) ke += (double)(qvx * qvx + qvy * qvy + qvz * qvz);
      if (do_drift) {
        const Drifted d = drift_particle(J, S, qc, qfx, qfy, qvx, qvy, do_walls);
        absorbed = d.absorbed; qc = d.cell; qfx = d.fx; qfy = d.fy;
        S.cell[idx] = qc; S.fx[idx] = qfx; S.fy[idx] = qfy;
      }
      if (do_dep && !absorbed) deposit_one(J, S, qc, qfx, qfy);
      S.vx[idx] = qvx; S.vy[idx] = qvy; S.vz[idx] = qvz;
    }
    if (do_walls) {
      const int h = warp_append(lane < cnt && absorbed, hit_counts + s);
      if (h >= 0) S.hits[h] = idx;
    }
    __syncwarp();
    for (int q = lane; q < qn - cnt; q += 32)
#pragma unroll
      for (int f = 0; f < kQFields; ++f) cq[f * kQueue + q] = cq[f * kQueue + q + cnt];
    __syncwarp();
    qn -= cnt;
  };
  // kinetic energy and collision counts of the slot a warp leaves go to its job's state
  auto flush = [&]() {
    if (cur < 0) return;
    if (qn > 0) round(qn);
    if (want_ke) {
      double v = ke;
#pragma unroll
      for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0 && v != 0.0) atomicAdd(&st[S.job].ke[S.species], v * S.ke_factor);
    }
    ke = 0.0;
    if (lane < 8) {
      const unsigned c = pc[lane];
      if (c) { atomicAdd(&st[S.job].collisions[S.species][lane], (unsigned long long)c); pc[lane] = 0u; }
    }
    __syncwarp();
  };
  const int nwarps = gridDim.x * kWarps;
  for (int item = blockIdx.x * kWarps + warp; item < total; item += nwarps) {
    int s = cur < 0 ? 0 : cur;
    while (s < nslots - 1 && item_prefix[s + 1] <= item) ++s;
    if (s != cur) {
      flush();
      copy_words(&tab[warp].S, slots + s, sizeof(SlotDev), lane);
      __syncwarp();
      copy_words(&tab[warp].J, jobs + S.job, sizeof(JobDev), lane);
      __syncwarp();
      cur = s;
      const JobState& T0 = st[S.job];
      const bool gated = flags & PIC_PHASE_GATED_I;
      const bool pending = T0.kick_pending != 0;
      do_kick = (flags & PIC_PHASE_KICK_I) && (!gated || pending);
      do_mcc = (flags & PIC_PHASE_MCC_I) && (!gated || pending) && J.mcc_mode != 0 && S.n_proc > 0;
      do_drift = flags & PIC_PHASE_DRIFT_I;
      do_walls = (flags & PIC_PHASE_WALLS_I) && J.wall_mode != 0;
      do_dep = flags & PIC_PHASE_DEPOSIT_I;
      want_ke = do_kick || do_mcc;
      mcc_step = gated ? (uint32_t)(T0.step - 1) : explicit_step;
      n = counts[s];
    }
    const int i0 = (item - item_prefix[s]) * kItem + kPPL * lane;
    // ---- loads
    uint32_t c[kPPL], pid[kPPL];
    float fx[kPPL], fy[kPPL], vx[kPPL], vy[kPPL], vz[kPPL];
    {
      ld_lane(S.cell + i0, c);
      ld_lane(S.fx + i0, fx);
      ld_lane(S.fy + i0, fy);
      ld_lane(S.vx + i0, vx);
      ld_lane(S.vy + i0, vy);
      if (do_mcc) {
        ld_lane(S.vz + i0, vz);
        ld_lane(S.pid + i0, pid);
      } else {
#pragma unroll
        for (int k = 0; k < kPPL; ++k) { vz[k] = 0.f; pid[k] = 0u; }
      }
    }
    bool valid[kPPL];
#pragma unroll
    for (int k = 0; k < kPPL; ++k) valid[k] = i0 + k < n;
    // ---- pass A: kick and collisions
    if (do_kick) {
      const float2* __restrict__ ef = J.efield;
      const int enx = J.nx;
      const float kx = S.kx, ky = S.ky;
#pragma unroll
      for (int k = 0; k < kPPL; ++k)
        if (valid[k] && c[k] != PIC_CELL_OUT) {
          const float2* e0 = ef + cell_j(c[k]) * enx + cell_i(c[k]);
          const float2 e00 = __ldg(e0), e10 = __ldg(e0 + 1), e01 = __ldg(e0 + enx), e11 = __ldg(e0 + enx + 1);
          const float x = fx[k], y = fy[k];
          const float w00 = (1.f - x) * (1.f - y), w10 = x * (1.f - y), w01 = (1.f - x) * y, w11 = x * y;
          const float gx = w00 * e00.x + w10 * e10.x + w01 * e01.x + w11 * e11.x;
          const float gy = w00 * e00.y + w10 * e10.y + w01 * e01.y + w11 * e11.y;
          vx[k] += kx * gx;
          vy[k] += ky * gy;
        }
    }
    if (do_mcc) {
      if (J.mcc_mode == 2) {
        const ProcDev& P = J.procs[S.first_proc];
#pragma unroll
        for (int k = 0; k < kPPL; ++k)
          if (valid[k]) {
            float u[4];
            draw4(J.seed, pid[k], mcc_step, 0u, u);
            const float v2 = vx[k] * vx[k] + vy[k] * vy[k];
            const float sp = sqrtf(v2);
            const float Pc = 1.f - expf(-J.gas_density * xs_lookup(P, S.half_m_over_e * v2) * sp * J.dt);
            if (u[0] < Pc) {
              float sn, cs;
              sincospif(2.f * u[1], &sn, &cs);
              vx[k] = sp * cs; vy[k] = sp * sn;
              atomicAdd(&pc[0], 1u);
            }
          }
      } else {
        bool cand[kPPL];
        unsigned m[kPPL];
        int before[kPPL];
        int ncand = 0;
#pragma unroll
        for (int k = 0; k < kPPL; ++k) {
          // candidate with probability nu_max dt; a candidate's collision is real when
          // u1 nu_max < n sigma_T(E) v (the process is chosen in the queue round, with the
          // same draw).  Null candidates stay in the item like every other particle.
          cand[k] = false;
          if (valid[k]) {
            float u[4];
            draw4(J.seed, pid[k], mcc_step, 0u, u);
            if (u[0] < S.pnull) {
              const float v2 = vx[k] * vx[k] + vy[k] * vy[k] + vz[k] * vz[k];
              cand[k] = u[1] * S.numax < J.gas_density * xs_lookup(S.total, S.half_m_over_e * v2) * sqrtf(v2);
            }
          }
          m[k] = __ballot_sync(0xffffffffu, cand[k]);
          before[k] = ncand;
          ncand += __popc(m[k]);
        }
        // rank of candidate (lane, k): item order k-major, then lane
        int rank[kPPL];
#pragma unroll
        for (int k = 0; k < kPPL; ++k) rank[k] = before[k] + __popc(m[k] & ((1u << lane) - 1u));
        // candidates leave the item for the warp's queue
#pragma unroll
        for (int k = 0; k < kPPL; ++k)
          if (cand[k]) {
            const int q = qn + rank[k];
            cq[0 * kQueue + q] = c[k];
            cq[1 * kQueue + q] = __float_as_uint(fx[k]); cq[2 * kQueue + q] = __float_as_uint(fy[k]);
            cq[3 * kQueue + q] = __float_as_uint(vx[k]); cq[4 * kQueue + q] = __float_as_uint(vy[k]);
            cq[5 * kQueue + q] = __float_as_uint(vz[k]); cq[6 * kQueue + q] = pid[k];
            cq[7 * kQueue + q] = (uint32_t)(i0 + k);
            valid[k] = false;   // the queue round finishes this particle
          }
        qn += ncand;
      }
    }
    if (want_ke) {
#pragma unroll
      for (int k = 0; k < kPPL; ++k)
        if (valid[k]) ke += (double)(vx[k] * vx[k] + vy[k] * vy[k] + vz[k] * vz[k]);
    }
    // ---- pass B: drift, walls, deposit
    uint32_t c_in[kPPL];
#pragma unroll
    for (int k = 0; k < kPPL; ++k) c_in[k] = c[k];
    uint32_t key[kPPL];
    bool absorbed[kPPL];
#pragma unroll
    for (int k = 0; k < kPPL; ++k) {
      absorbed[k] = false;
      key[k] = valid[k] ? c[k] : PIC_CELL_OUT;
      if (do_drift && valid[k]) {
        const Drifted d = drift_particle(J, S, c[k], fx[k], fy[k], vx[k], vy[k], do_walls);
        absorbed[k] = d.absorbed; c[k] = d.cell; fx[k] = d.fx; fy[k] = d.fy;
        key[k] = d.absorbed ? PIC_CELL_OUT : d.cell;
      }
    }
    if (do_walls) {
      unsigned hm[kPPL];
      int nh = 0, hb[kPPL];
#pragma unroll
      for (int k = 0; k < kPPL; ++k) {
        hm[k] = __ballot_sync(0xffffffffu, valid[k] && absorbed[k]);
        hb[k] = nh;
        nh += __popc(hm[k]);
      }
      if (nh) {
        int base = 0;
        if (lane == 0) base = atomicAdd(hit_counts + s, nh);
        base = __shfl_sync(0xffffffffu, base, 0);
#pragma unroll
        for (int k = 0; k < kPPL; ++k)
          if (valid[k] && absorbed[k]) S.hits[base + hb[k] + __popc(hm[k] & ((1u << lane) - 1u))] = i0 + k;
      }
    }
    if (do_dep) {
      if (J.deposit_mode == 0) {
        const float q = S.qdep;
        lane_deposit<float>(J.rho_f, J.nx, key, fx, fy,
                            [q](float x, float y, float& a, float& b, float& cc, float& d) { cic_f32(q, x, y, a, b, cc, d); });
      } else {
        const long long qf = S.qfix;
        lane_deposit<unsigned long long>(
            reinterpret_cast<unsigned long long*>(J.rho_i), J.nx, key, fx, fy,
            [qf](float x, float y, unsigned long long& a, unsigned long long& b, unsigned long long& cc,
                 unsigned long long& d) {
              long long a_, b_, c_, d_;
              cic_i64(qf, x, y, a_, b_, c_, d_);
              a = (unsigned long long)a_; b = (unsigned long long)b_; cc = (unsigned long long)c_;
              d = (unsigned long long)d_;
            });
      }
    }
    // ---- stores
    if (do_drift) {
      // the cell word changes only when a particle crosses a cell edge (rare for ions): a warp
      // whose cells all stayed leaves them in place
      bool moved = false;
#pragma unroll
      for (int k = 0; k < kPPL; ++k) moved |= c[k] != c_in[k];
      if (__any_sync(0xffffffffu, moved)) st_lane(S.cell + i0, c);
      st_lane(S.fx + i0, fx);
      st_lane(S.fy + i0, fy);
    }
    if (do_kick || do_mcc) {
      st_lane(S.vx + i0, vx);
      st_lane(S.vy + i0, vy);
    }
    // vz changes only in a collision, and the queue round stores the collided particles
    // full rounds of queued candidates, after this item's stores
    while (qn >= 32) round(32);
  }
  flush();
}

// Exclusive prefix of mover work items (kItem particles) per active slot.
__global__ void chunk_table_kernel(const int* __restrict__ counts, const uint8_t* __restrict__ active,
                                   int* __restrict__ chunk_prefix, int nslots) {
  if (threadIdx.x == 0) {
    int a = 0;
    for (int s = 0; s < nslots; ++s) {
      chunk_prefix[s] = a;
      if (!active || active[s]) a += (counts[s] + kItem - 1) / kItem;
    }
    chunk_prefix[nslots] = a;
  }
}

int mover_blocks_per_sm() {
  cudaFuncSetAttribute(mover_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMoverSmem);
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, mover_kernel, PIC_MOVER_THREADS, kMoverSmem) != cudaSuccess ||
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
  mover_kernel<<<L.mover_grid, PIC_MOVER_THREADS, kMoverSmem, stream>>>(L.jobs, L.st, L.slots, L.counts,
                                                                          L.hit_counts, L.chunk_prefix, L.nslots, flags,
                                                                          explicit_step);
  if (L.ev_mover_end) cudaEventRecord(L.ev_mover_end, stream);
  return k;
}
