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

__global__ void sort_zero(const JobDev* jobs, const SlotDev* slots, const uint8_t* mask, int* aux) {
  const int s = blockIdx.y;
  if (!mask[s]) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) aux[4 * s + 3] = 0;   // descents, counted by sort_hist
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

// A warp takes kSortRounds x 32 consecutive particles per iteration, lane-striped (round r,
// lane l: particle 32 r + l), and issues all their loads before any dependent work, so each
// warp keeps kSortRounds coalesced requests per array in flight.
constexpr int kSortRounds = 4;
constexpr int kSortItem = 32 * kSortRounds;

// Histogram of cell keys, one atomic per warp segment of equal keys.  With count_descents, also
// the particles whose key is below their predecessor's (within a warp iteration's 4 x 32), one
// atomic per CTA into aux[4 s + 3].
__global__ void __launch_bounds__(256) sort_hist(const JobDev* jobs, const SlotDev* slots, const int* counts,
                                                 const uint8_t* mask, int* aux, int count_descents) {
  const int s = blockIdx.y;
  if (!mask[s]) return;
  const SlotDev& S = slots[s];
  const JobDev& J = jobs[S.job];
  const int n = counts[s];
  const uint32_t ncells = (uint32_t)(J.ncx * J.ncy);
  const uint32_t* __restrict__ cell = S.cell;
  int* const cnt = S.cell_count;
  const int ncx = J.ncx;
  const int lane = lane_id();
  const int nitems = (n + kSortItem - 1) / kSortItem;
  int descents = 0;
  for (int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < nitems; it += (gridDim.x * blockDim.x) >> 5) {
    uint32_t key[kSortRounds];
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
      const int p = it * kSortItem + 32 * r + lane;
      key[r] = p < n ? dense_key(__ldg(cell + p), ncx, ncells) : kNoKey;
    }
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
      int first, last;
      run_segment(key[r], first, last);
      if (lane == last && key[r] != kNoKey) atomicAdd(cnt + key[r], last - first + 1);
      if (count_descents) {
        uint32_t prev = __shfl_up_sync(0xffffffffu, key[r], 1);
        const uint32_t wrap = r > 0 ? __shfl_sync(0xffffffffu, key[r > 0 ? r - 1 : 0], 31) : kNoKey;
        if (lane == 0) prev = wrap;
        descents += (key[r] != kNoKey && prev != kNoKey && key[r] < prev) ? 1 : 0;
      }
    }
  }
  if (count_descents) {
    __shared__ int block_desc;
    if (threadIdx.x == 0) block_desc = 0;
    __syncthreads();
    const int w = __reduce_add_sync(0xffffffffu, descents);
    if (lane == 0 && w) atomicAdd(&block_desc, w);
    __syncthreads();
    if (threadIdx.x == 0 && block_desc) atomicAdd(aux + 4 * s + 3, block_desc);
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
// segment of equal keys returns the segment's first position.  Every field of the warp's
// kSortRounds x 32 particles is loaded before the atomics, so loads and atomics overlap; the
// stores of a round are consecutive across lanes where the order was kept since the last sort.
__global__ void sort_scatter(const JobDev* jobs, const SlotDev* slots, const int* counts, const uint8_t* mask) {
  const int s = blockIdx.y;
  if (!mask[s]) return;
  const SlotDev& S = slots[s];
  const JobDev& J = jobs[S.job];
  const int n = counts[s];
  const uint32_t ncells = (uint32_t)(J.ncx * J.ncy);
  const int ncx = J.ncx;
  const uint32_t* __restrict__ cell = S.cell;
  const float* __restrict__ fx = S.fx;
  const float* __restrict__ fy = S.fy;
  const float* __restrict__ vx = S.vx;
  const float* __restrict__ vy = S.vy;
  const float* __restrict__ vz = S.vz;
  const uint32_t* __restrict__ pid = S.pid;
  uint32_t* const cell_b = S.cell_b;
  float* const fx_b = S.fx_b;
  float* const fy_b = S.fy_b;
  float* const vx_b = S.vx_b;
  float* const vy_b = S.vy_b;
  float* const vz_b = S.vz_b;
  uint32_t* const pid_b = S.pid_b;
  int* const cnt = S.cell_count;
  const int lane = lane_id();
  const int nitems = (n + kSortItem - 1) / kSortItem;
  for (int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < nitems; it += (gridDim.x * blockDim.x) >> 5) {
    uint32_t c[kSortRounds], pd[kSortRounds], key[kSortRounds];
    float a[kSortRounds], b[kSortRounds], u[kSortRounds], v[kSortRounds], w[kSortRounds];
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
      const int p = it * kSortItem + 32 * r + lane;
      const int q = p < n ? p : 0;
      c[r] = __ldcs(cell + q); a[r] = __ldcs(fx + q); b[r] = __ldcs(fy + q);
      u[r] = __ldcs(vx + q); v[r] = __ldcs(vy + q); w[r] = __ldcs(vz + q); pd[r] = __ldcs(pid + q);
      key[r] = p < n ? dense_key(c[r], ncx, ncells) : kNoKey;
    }
    int at[kSortRounds];
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
      int first, last;
      run_segment(key[r], first, last);
      int base = 0;
      if (lane == last && key[r] != kNoKey) base = atomicAdd(cnt + key[r], last - first + 1);
      at[r] = __shfl_sync(0xffffffffu, base, last) + lane - first;
    }
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r)
      if (key[r] != kNoKey) {
        const int d = at[r];
        cell_b[d] = c[r]; fx_b[d] = a[r]; fy_b[d] = b[r];
        vx_b[d] = u[r]; vy_b[d] = v[r]; vz_b[d] = w[r]; pid_b[d] = pd[r];
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

// Slots of the mask whose particles are nearly in cell order (descents below 1/32 of the
// particles) leave the mask: their histogram is not scanned and they are not moved.
__global__ void sort_filter_kernel(uint8_t* mask, const int* counts, const int* aux, int nslots) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots || !mask[s]) return;
  if (aux[4 * s + 3] < (counts[s] >> kSortDisorderShift)) mask[s] = 0;
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

int launch_sort(const EngineLaunch& L, uint8_t* mask, int max_cells, int max_particles, bool by_disorder,
                cudaStream_t st) {
  if (L.nslots == 0) return 0;
  const int ncells = max_cells + 1;
  const int ntiles = (ncells + kTile - 1) / kTile;
  const int gz = std::min(std::max((ncells + 255) / 256, 1), 4 * L.num_sms);
  const int gp = std::min(std::max((max_particles + 255) / 256, 1), 8 * L.num_sms);
  sort_zero<<<dim3(gz, L.nslots), 256, 0, st>>>(L.jobs, L.slots, mask, L.aux);
  sort_hist<<<dim3(gp, L.nslots), 256, 0, st>>>(L.jobs, L.slots, L.counts, mask, L.aux, by_disorder ? 1 : 0);
  if (by_disorder) sort_filter_kernel<<<(L.nslots + 255) / 256, 256, 0, st>>>(mask, L.counts, L.aux, L.nslots);
  sort_tile_sums<<<dim3(std::min(ntiles, 4 * L.num_sms), L.nslots), 256, 0, st>>>(L.jobs, L.slots, mask);
  sort_scan_parts<<<L.nslots, 256, 0, st>>>(L.jobs, L.slots, mask);
  sort_apply<<<dim3(std::min(ntiles, 4 * L.num_sms), L.nslots), 256, 0, st>>>(L.jobs, L.slots, mask);
  sort_scatter<<<dim3(gp, L.nslots), 256, 0, st>>>(L.jobs, L.slots, L.counts, mask);
  sort_swap<<<(L.nslots + 255) / 256, 256, 0, st>>>(L.slots_mut, mask, L.nslots);
  return by_disorder ? 8 : 7;
}
