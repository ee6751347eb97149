// sort.cu — counting sort of every particle slot by cell (row-major cell index).
//
// The reference never orders particles (Thrust is included but unused, particles.cu:7-10),
// so its scatter/gather kernels hit random nodes.  Sorting by cell every N steps makes the
// warps of the mover touch a handful of neighbouring nodes, which turns the deposit's
// atomics into one per cell segment and the gather into L1 hits.
//   histogram (runs of equal keys counted in registers and over warp segments) -> exclusive
//   scan over cells
//   (tile sums, per-slot scan of tile sums, tile rescan) -> scatter of all seven fields into
//   the slot's second set of arrays -> pointer swap in the device slot table.
// All slots of all jobs are processed by the same launches (blockIdx.y = slot).
#include <algorithm>
#include "common.cuh"
#include "kernels.h"

namespace {

constexpr int kTile = 2048;     // cells per scan tile (256 threads x 8)

__device__ __forceinline__ uint32_t dense_key(uint32_t c, int ncx, uint32_t ncells) {
  return c == PIC_CELL_OUT ? ncells : (uint32_t)cell_j(c) * (uint32_t)ncx + (uint32_t)cell_i(c);
}

__global__ void sort_zero(const JobDev* jobs, const SlotDev* slots, const uint8_t* mask) {
  const int s = blockIdx.y;
  if (!mask[s]) return;
  const SlotDev& S = slots[s];
  const JobDev& J = jobs[S.job];
  const int ncells = J.ncx * J.ncy + 1;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < ncells; k += gridDim.x * blockDim.x) S.cell_count[k] = 0;
}

constexpr uint32_t kNoKey = 0xFFFFFFFFu;   // a lane past the slot's count

// Segments of equal keys over the warp, in lane order: the first and last lane of this
// lane's segment.  Particles are sorted by cell between sorts and drift slowly, so equal keys
// mostly sit in neighbouring lanes; where they do not, a key forms several segments, each
// counted on its own (still correct, one more atomic).
__device__ __forceinline__ void run_segment(uint32_t key, int& first, int& last) {
  const int lane = lane_id();
  const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
  const bool head = lane == 0 || key != prev;
  const unsigned heads = __ballot_sync(0xffffffffu, head);
  first = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
  const unsigned after = lane == 31 ? 0u : heads & (0xfffffffeu << lane);
  last = (after ? __ffs(after) - 1 : 32) - 1;
}

// Histogram of cell keys, one atomic per warp segment of equal keys.
__global__ void sort_hist(const JobDev* jobs, const SlotDev* slots, const int* counts, const uint8_t* mask) {
  const int s = blockIdx.y;
  if (!mask[s]) return;
  const SlotDev& S = slots[s];
  const JobDev& J = jobs[S.job];
  const int n = counts[s];
  const uint32_t ncells = (uint32_t)(J.ncx * J.ncy);
  const int lane = lane_id();
  for (int wb = blockIdx.x * blockDim.x + (threadIdx.x & ~31); wb < n; wb += gridDim.x * blockDim.x) {
    const int p = wb + lane;
    const uint32_t key = p < n ? dense_key(S.cell[p], J.ncx, ncells) : kNoKey;
    int first, last;
    run_segment(key, first, last);
    if (lane == last && key != kNoKey) atomicAdd(S.cell_count + key, last - first + 1);
  }
}

// Exclusive scan of 8 values per thread over a 2048-entry tile; returns the tile total.
__device__ int tile_exclusive_scan(int v[8]) {
  __shared__ int warp_tot[8];
  int t = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) { const int x = v[k]; v[k] = t; t += x; }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int incl = t;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[w] = incl;
  __syncthreads();
  int woff = 0, total = 0;
  for (int k = 0; k < 8; ++k) { if (k < w) woff += warp_tot[k]; total += warp_tot[k]; }
  __syncthreads();
  const int off = woff + incl - t;
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] += off;
  return total;
}

__global__ void __launch_bounds__(256) sort_tile_sums(const JobDev* jobs, const SlotDev* slots, const uint8_t* mask) {
  const int s = blockIdx.y;
  if (!mask[s]) return;
  const SlotDev& S = slots[s];
  const JobDev& J = jobs[S.job];
  const int ncells = J.ncx * J.ncy + 1;
  const int ntiles = (ncells + kTile - 1) / kTile;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int sum = 0;
    for (int k = 0; k < 8; ++k) {
      const int c = tile * kTile + threadIdx.x * 8 + k;
      if (c < ncells) sum += S.cell_count[c];
    }
    for (int o = 16; o; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
    __shared__ int ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
      int t = 0;
      for (int k = 0; k < 8; ++k) t += ws[k];
      S.scan_part[tile] = t;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) sort_scan_parts(const JobDev* jobs, const SlotDev* slots, const uint8_t* mask) {
  const int s = blockIdx.x;
  if (!mask[s]) return;
  const SlotDev& S = slots[s];
  const JobDev& J = jobs[S.job];
  const int ntiles = (J.ncx * J.ncy + 1 + kTile - 1) / kTile;
  int carry = 0;
  for (int b = 0; b < ntiles; b += kTile) {
    int v[8];
    for (int k = 0; k < 8; ++k) {
      const int c = b + threadIdx.x * 8 + k;
      v[k] = c < ntiles ? S.scan_part[c] : 0;
    }
    const int tot = tile_exclusive_scan(v);
    for (int k = 0; k < 8; ++k) {
      const int c = b + threadIdx.x * 8 + k;
      if (c < ntiles) S.scan_part[c] = v[k] + carry;
    }
    carry += tot;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) sort_apply(const JobDev* jobs, const SlotDev* slots, const uint8_t* mask) {
  const int s = blockIdx.y;
  if (!mask[s]) return;
  const SlotDev& S = slots[s];
  const JobDev& J = jobs[S.job];
  const int ncells = J.ncx * J.ncy + 1;
  const int ntiles = (ncells + kTile - 1) / kTile;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int v[8];
    for (int k = 0; k < 8; ++k) {
      const int c = tile * kTile + threadIdx.x * 8 + k;
      v[k] = c < ncells ? S.cell_count[c] : 0;
    }
    tile_exclusive_scan(v);
    const int base = S.scan_part[tile];
    for (int k = 0; k < 8; ++k) {
      const int c = tile * kTile + threadIdx.x * 8 + k;
      if (c < ncells) S.cell_count[c] = v[k] + base;
    }
    __syncthreads();
  }
}

// Scatter of all seven fields to the positions the scanned counts give: one atomic per warp
// segment of equal keys returns the segment's first position.  Every field is loaded before
// the atomic, so the loads and the atomic's round trip overlap.
__global__ void sort_scatter(const JobDev* jobs, const SlotDev* slots, const int* counts, const uint8_t* mask) {
  const int s = blockIdx.y;
  if (!mask[s]) return;
  const SlotDev& S = slots[s];
  const JobDev& J = jobs[S.job];
  const int n = counts[s];
  const uint32_t ncells = (uint32_t)(J.ncx * J.ncy);
  const int lane = lane_id();
  for (int wb = blockIdx.x * blockDim.x + (threadIdx.x & ~31); wb < n; wb += gridDim.x * blockDim.x) {
    const int p = wb + lane;
    const bool in = p < n;
    const int q = in ? p : 0;
    const uint32_t c = S.cell[q];
    const float fx = S.fx[q], fy = S.fy[q], vx = S.vx[q], vy = S.vy[q], vz = S.vz[q];
    const uint32_t pid = S.pid[q];
    const uint32_t key = in ? dense_key(c, J.ncx, ncells) : kNoKey;
    int first, last;
    run_segment(key, first, last);
    int base = 0;
    if (lane == last && in) base = atomicAdd(S.cell_count + key, last - first + 1);
    base = __shfl_sync(0xffffffffu, base, last);
    if (in) {
      const int at = base + lane - first;
      S.cell_b[at] = c; S.fx_b[at] = fx; S.fy_b[at] = fy;
      S.vx_b[at] = vx; S.vy_b[at] = vy; S.vz_b[at] = vz; S.pid_b[at] = pid;
    }
  }
}

template <typename T>
__device__ __forceinline__ void swp(T*& a, T*& b) { T* t = a; a = b; b = t; }

__global__ void sort_swap(SlotDev* slots, const uint8_t* mask, int nslots) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots || !mask[s]) return;
  SlotDev& S = slots[s];
  swp(S.cell, S.cell_b); swp(S.fx, S.fx_b); swp(S.fy, S.fy_b);
  swp(S.vx, S.vx_b); swp(S.vy, S.vy_b); swp(S.vz, S.vz_b); swp(S.pid, S.pid_b);
}

// Slots whose job is due for a counting sort: sort_every > 0 and (step + offset) % sort_every
// == 0 (offset 1: the sort at the end of a step, before the step counter advances).
__global__ void sort_mask_kernel(const JobDev* jobs, const JobState* st, const uint8_t* active, uint8_t* mask, int nslots,
                                 int offset) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  const int j = s / PIC_MAX_SPECIES;
  const JobDev& J = jobs[j];
  const bool due = active[s] && J.sort_every > 0 && ((st[j].step + offset) % J.sort_every) == 0;
  mask[s] = due ? 1 : 0;
}

}  // namespace

int launch_sort_mask(const EngineLaunch& L, uint8_t* mask, int offset, cudaStream_t st) {
  if (L.nslots == 0) return 0;
  sort_mask_kernel<<<(L.nslots + 255) / 256, 256, 0, st>>>(L.jobs, L.st, L.active, mask, L.nslots, offset);
  return 1;
}

int launch_sort(const EngineLaunch& L, const uint8_t* mask, int max_cells, int max_particles, cudaStream_t st) {
  if (L.nslots == 0) return 0;
  const int ncells = max_cells + 1;
  const int ntiles = (ncells + kTile - 1) / kTile;
  const int gz = std::min(std::max((ncells + 255) / 256, 1), 4 * L.num_sms);
  const int gp = std::min(std::max((max_particles + 255) / 256, 1), 8 * L.num_sms);
  sort_zero<<<dim3(gz, L.nslots), 256, 0, st>>>(L.jobs, L.slots, mask);
  sort_hist<<<dim3(gp, L.nslots), 256, 0, st>>>(L.jobs, L.slots, L.counts, mask);
  sort_tile_sums<<<dim3(std::min(ntiles, 4 * L.num_sms), L.nslots), 256, 0, st>>>(L.jobs, L.slots, mask);
  sort_scan_parts<<<L.nslots, 256, 0, st>>>(L.jobs, L.slots, mask);
  sort_apply<<<dim3(std::min(ntiles, 4 * L.num_sms), L.nslots), 256, 0, st>>>(L.jobs, L.slots, mask);
  sort_scatter<<<dim3(gp, L.nslots), 256, 0, st>>>(L.jobs, L.slots, L.counts, mask);
  sort_swap<<<(L.nslots + 255) / 256, 256, 0, st>>>(L.slots_mut, mask, L.nslots);
  return 7;
}
