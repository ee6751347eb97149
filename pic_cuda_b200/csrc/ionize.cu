// ionize.cu — appends the electron-ion pairs of this step's ionising collisions.
//
// The reference has no ionisation with particle creation (ionization_kernel, mcc.cu:88-112,
// only zeroes v and is never launched).  The mover appends one event per ionisation with a
// warp-aggregated atomic (arbitrary order); this kernel, one CTA per job, sorts the events
// by parent pid so that the new pids (next_pid + 2r for the electron, +1 for the ion), the
// array positions and therefore the whole run are independent of that order.  The pair is
// born at the parent's position at collision time; in the fused step it then takes the same
// drift / absorption / deposit path as every other particle of this step.
#include "common.cuh"
#include "kernels.h"
#include "particle_ops.cuh"

namespace {

constexpr int kSmemKeys = 2048;

__device__ void bitonic_sort(unsigned long long* keys, int n_pow2) {
  for (int k = 2; k <= n_pow2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < n_pow2; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const bool asc = (i & k) == 0;
          const unsigned long long a = keys[i], b = keys[ixj];
          if ((a > b) == asc) { keys[i] = b; keys[ixj] = a; }
        }
      }
      __syncthreads();
    }
  }
}

// Exclusive block scan of a 0/1 flag (256 threads); returns the prefix, *total the sum.
__device__ int block_scan01(int v, int* total) {
  __shared__ int warp_sums[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned m = __ballot_sync(0xffffffffu, v);
  const int in_warp = __popc(m & ((1u << lane) - 1u));
  if (lane == 0) warp_sums[w] = __popc(m);
  __syncthreads();
  int off = 0, tot = 0;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
    if (k < w) off += warp_sums[k];
    tot += warp_sums[k];
  }
  __syncthreads();
  *total = tot;
  return off + in_warp;
}

__global__ void __launch_bounds__(256)
ionize_kernel(const JobDev* __restrict__ jobs, JobState* __restrict__ st, const SlotDev* __restrict__ slots,
              int* __restrict__ counts, int* __restrict__ aux, int drift_dep) {
  const int job = blockIdx.x;
  const JobDev& J = jobs[job];
  JobState& T = st[job];
  if (J.mcc_mode != 1 || J.nslots == 0) return;
  __shared__ unsigned long long skeys[kSmemKeys];
  const int ne = min(T.event_count, J.event_capacity);
  __syncthreads();
  if (ne == 0) {
    if (threadIdx.x == 0) { T.ionizations = 0; T.event_count = 0; }
    return;
  }
  int np2 = 1;
  while (np2 < ne) np2 <<= 1;
  unsigned long long* keys = np2 <= kSmemKeys ? skeys : reinterpret_cast<unsigned long long*>(J.events + J.event_capacity);
  for (int i = threadIdx.x; i < np2; i += blockDim.x)
    keys[i] = i < ne ? (((unsigned long long)J.events[i].parent_pid << 32) | (unsigned)i) : ~0ull;
  __syncthreads();
  bitonic_sort(keys, np2);

  const int se = J.slot0 + J.ion_e_species, si = J.slot0 + J.ion_i_species;
  const SlotDev& SE = slots[se];
  const SlotDev& SI = slots[si];
  int ce = counts[se], ci = counts[si];
  const uint32_t pid0 = T.next_pid;
  int lost_e = 0, lost_i = 0;
  for (int r0 = 0; r0 < ne; r0 += blockDim.x) {
    const int r = r0 + threadIdx.x;
    const bool valid = r < ne;
    Event ev;
    if (valid) ev = J.events[(int)(keys[r] & 0xffffffffu)];
    uint32_t c_e = 0, c_i = 0;
    float x_e = 0, y_e = 0, x_i = 0, y_i = 0;
    bool keep_e = valid, keep_i = valid;
    if (valid) {
      c_e = c_i = ev.cell;
      x_e = x_i = ev.fx;
      y_e = y_i = ev.fy;
      if (drift_dep) {
        const Drifted de = drift_particle(J, SE, ev.cell, ev.fx, ev.fy, ev.ve[0], ev.ve[1], true);
        const Drifted di = drift_particle(J, SI, ev.cell, ev.fx, ev.fy, ev.vi[0], ev.vi[1], true);
        keep_e = !de.absorbed; keep_i = !di.absorbed;
        c_e = de.cell; x_e = de.fx; y_e = de.fy;
        c_i = di.cell; x_i = di.fx; y_i = di.fy;
      }
    }
    int tot_e, tot_i;
    const int oe = block_scan01(keep_e ? 1 : 0, &tot_e);
    const int oi = block_scan01(keep_i ? 1 : 0, &tot_i);
    if (valid && keep_e) {
      const int at = ce + oe;
      if (at < SE.capacity) {
        SE.cell[at] = c_e; SE.fx[at] = x_e; SE.fy[at] = y_e;
        SE.vx[at] = ev.ve[0]; SE.vy[at] = ev.ve[1]; SE.vz[at] = ev.ve[2]; SE.pid[at] = pid0 + 2u * (uint32_t)r;
        if (drift_dep) deposit_one(J, SE, c_e, x_e, y_e);
      } else {
        atomicOr(&T.status, PIC_ST_CAPACITY);
      }
    }
    if (valid && keep_i) {
      const int at = ci + oi;
      if (at < SI.capacity) {
        SI.cell[at] = c_i; SI.fx[at] = x_i; SI.fy[at] = y_i;
        SI.vx[at] = ev.vi[0]; SI.vy[at] = ev.vi[1]; SI.vz[at] = ev.vi[2]; SI.pid[at] = pid0 + 2u * (uint32_t)r + 1u;
        if (drift_dep) deposit_one(J, SI, c_i, x_i, y_i);
      } else {
        atomicOr(&T.status, PIC_ST_CAPACITY);
      }
    }
    int lost;
    block_scan01(valid && !keep_e ? 1 : 0, &lost);
    lost_e += lost;
    block_scan01(valid && !keep_i ? 1 : 0, &lost);
    lost_i += lost;
    ce += tot_e; ci += tot_i;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    counts[se] = min(ce, (int)SE.capacity);
    counts[si] = min(ci, (int)SI.capacity);
    // newborns absorbed in their first drift: added to the slots' absorbed counts by the
    // next compaction (aux[4 s + 2])
    if (aux) { aux[4 * se + 2] += lost_e; aux[4 * si + 2] += lost_i; }
    T.next_pid = pid0 + 2u * (uint32_t)ne;
    T.ionizations = ne;
    T.event_count = 0;
  }
}

}  // namespace

int launch_ionize(const EngineLaunch& L, bool drift_and_deposit, cudaStream_t s) {
  if (L.njobs == 0) return 0;
  ionize_kernel<<<L.njobs, 256, 0, s>>>(L.jobs, L.st, L.slots, L.counts, L.aux, drift_and_deposit ? 1 : 0);
  return 1;
}
