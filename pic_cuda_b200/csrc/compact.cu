// compact.cu — removal of absorbed particles without a host round trip.
//
// Replaces Particles2D::removeCollidedParticles (particles.cu:217-262).  The reference
// reads the hit count back to the host every step and then fills holes in the head
// [0, n-k) with survivors from the tail [n-k, n).  Here the same hole-filling runs
// entirely on the device from the hit list the mover appended, for every slot of every
// job in one launch sequence (blockIdx.y = slot), and copies every field (the reference
// copies only r, v, type, particles.cu:107-109).  Unlike the reference it pairs each hole
// with a tail particle that survived (the reference can copy dead tail particles into
// holes and copies at most 256 per step, particles.cu:63-66, 255), so the survivor set is
// exactly "all minus hits".  Pairing order is unspecified; the survivor set is not.
#include "common.cuh"
#include "kernels.h"

namespace {

// aux[4*s + 0] = holes found, aux[4*s + 1] = tail survivors found, aux[4*s + 2] = ionisation
// newborns absorbed since the last compaction.
__global__ void compact_mark(const SlotDev* __restrict__ slots, const int* __restrict__ counts,
                             const int* __restrict__ hit_counts, int* __restrict__ aux, const uint8_t* active) {
  const int s = blockIdx.y;
  if (active && !active[s]) return;
  const int k = hit_counts[s];
  if (k == 0) return;
  const int head = counts[s] - k;
  const SlotDev& S = slots[s];
  if (blockIdx.x == 0 && threadIdx.x == 0) { aux[4 * s] = 0; aux[4 * s + 1] = 0; }
  // scratch[0, k) is all zero between compactions; mark tail slots that were hit.
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < k; t += gridDim.x * blockDim.x) {
    const int h = S.hits[t];
    if (h >= head) S.scratch[h - head] = 1;
  }
}

__global__ void compact_lists(const SlotDev* __restrict__ slots, const int* __restrict__ counts,
                              const int* __restrict__ hit_counts, int* __restrict__ aux, const uint8_t* active) {
  const int s = blockIdx.y;
  if (active && !active[s]) return;
  const int k = hit_counts[s];
  if (k == 0) return;
  const int head = counts[s] - k;
  const SlotDev& S = slots[s];
  // warp-uniform loop: every lane of a warp runs the same iterations (warp_append votes)
  for (int wb = blockIdx.x * blockDim.x + (threadIdx.x & ~31); wb < k; wb += gridDim.x * blockDim.x) {
    const int t = wb + lane_id();
    const bool in = t < k;
    const int h = in ? S.hits[t] : 0;
    const int hole = warp_append(in && h < head, aux + 4 * s);
    if (hole >= 0) S.scratch2[hole] = h;
    const bool surv = in && S.scratch[t] == 0;
    if (in) S.scratch[t] = 0;
    const int sv = warp_append(surv, aux + 4 * s + 1);
    if (sv >= 0) S.scratch2[head + sv] = head + t;
  }
}

__global__ void compact_move(const SlotDev* __restrict__ slots, int* __restrict__ counts,
                             int* __restrict__ hit_counts, const int* __restrict__ aux, const uint8_t* active) {
  const int s = blockIdx.y;
  if (active && !active[s]) return;
  const int k = hit_counts[s];
  if (k == 0) return;
  const int head = counts[s] - k;
  const SlotDev& S = slots[s];
  const int nh = aux[4 * s];
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nh; r += gridDim.x * blockDim.x) {
    const int dst = S.scratch2[r], src = S.scratch2[head + r];
    S.cell[dst] = S.cell[src]; S.fx[dst] = S.fx[src]; S.fy[dst] = S.fy[src];
    S.vx[dst] = S.vx[src]; S.vy[dst] = S.vy[src]; S.vz[dst] = S.vz[src]; S.pid[dst] = S.pid[src];
  }
}

// absorbed_out[s] = this pass's hits plus the ionisation newborns lost since the last
// compaction (aux[4 s + 2], which the ionisation kernel accumulates).
__global__ void compact_finish(int* __restrict__ counts, int* __restrict__ hit_counts, int nslots,
                               const uint8_t* active, int* aux, int* absorbed_out) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nslots; s += gridDim.x * blockDim.x) {
    if (active && !active[s]) continue;
    const int k = hit_counts[s];
    const int lost = aux[4 * s + 2];
    aux[4 * s + 2] = 0;
    if (absorbed_out) absorbed_out[s] = k + lost;
    if (k == 0) continue;
    counts[s] -= k;
    hit_counts[s] = 0;
  }
}

}  // namespace

int launch_compact(const EngineLaunch& L, cudaStream_t st) {
  if (L.nslots == 0) return 0;
  dim3 grid(8, L.nslots);
  compact_mark<<<grid, 256, 0, st>>>(L.slots, L.counts, L.hit_counts, L.aux, L.active);
  compact_lists<<<grid, 256, 0, st>>>(L.slots, L.counts, L.hit_counts, L.aux, L.active);
  compact_move<<<grid, 256, 0, st>>>(L.slots, L.counts, L.hit_counts, L.aux, L.active);
  compact_finish<<<(L.nslots + 255) / 256, 256, 0, st>>>(L.counts, L.hit_counts, L.nslots, L.active, L.aux,
                                                         L.absorbed);
  return 4;
}
