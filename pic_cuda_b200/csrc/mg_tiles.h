// mg_tiles.h — shapes of the multigrid tile kernels' shared-memory tiles, shared by the host
// (which encodes one tensor map per tile shape and array) and the kernels (which load the
// tiles with cp.async.bulk.tensor).
//
// A tile covers grid columns gx0 .. gx0 + W - 1.  A tensor-map load must start at a column
// that is a multiple of 4 (16 bytes of FP32), so the box starts `off` columns to the left of
// gx0 and is BW >= off + W columns wide (a multiple of 4); the tile's node (0, 0) sits at
// shared float `off` of the box, and the box's row length BW is the tile's row pitch.  Every
// level array therefore has a row pitch that is a multiple of 4 floats (JobDev::pl).
#pragma once

namespace mgt {

constexpr int kTC = 16;   // down-leg tile: 16 x 16 coarse nodes (32 x 32 owned fine nodes)
constexpr int kTU = 32;   // up-leg tile: 32 x 32 owned fine nodes

__host__ __device__ constexpr int round4(int v) { return (v + 3) & ~3; }
// columns between an origin 32 k - a (k any integer) and the multiple of 4 at or below it
__host__ __device__ constexpr int align_off(int a) { return (4 - (a % 4)) % 4; }

// Down leg of NU pre-sweeps: tile origin gx0 = 2 ic0 - 2 - 2 NU (ic0 a multiple of kTC).
__host__ __device__ constexpr int down_w(int nu) { return 2 * kTC + 3 + 4 * nu; }
__host__ __device__ constexpr int down_off(int nu) { return align_off(2 + 2 * nu); }
// Row pitch of the down-leg tiles and the sweep's row-group width: at two pre-sweeps (tile
// width 43) a 56-float pitch with 48-thread groups (7 of them idle) cuts the half-sweeps' bank
// wavefronts by a quarter for a fifth more iterations, a net gain measured on B200 (V-cycle
// 454 -> 440 us at 4097^2); other smoothing counts keep the smallest pitch.
__host__ __device__ constexpr int down_bw(int nu) { return nu == 2 ? 56 : round4(down_off(nu) + down_w(nu)); }
__host__ __device__ constexpr int down_group(int nu) { return nu == 2 ? 48 : down_w(nu) - 2; }

// Up leg of NU post-sweeps, X = 1 on level 0 (one more node of halo for the FP64 defect):
// tile origin gx0 = i0 - 2 NU - X (i0 a multiple of kTU); the coarse tile starts at column
// floor(gx0 / 2) = i0 / 2 - ceil((2 NU + X) / 2).
__host__ __device__ constexpr int up_w(int nu, int x) { return kTU + 4 * nu + 2 * x; }
__host__ __device__ constexpr int up_off(int nu, int x) { return align_off(2 * nu + x); }
// Row pitch BW of the up-leg tiles.  At two post-sweeps (tile widths 40 and 42) a pitch of 52
// floats (20 mod 32 banks) with row groups of up_group = 40 threads puts the accesses of every
// warp of a half-sweep, including warps that straddle two row groups, in distinct banks
// (the smallest pitch, 40 or 48, gives 1.5-1.6 wavefronts per access; V-cycle 490 -> 453 us
// at 4097^2 on B200); other smoothing counts keep the smallest pitch and one thread per
// interior column.
__host__ __device__ constexpr int up_bw(int nu, int x) { return nu == 2 ? 52 : round4(up_off(nu, x) + up_w(nu, x)); }
__host__ __device__ constexpr int up_group(int nu, int x) { return nu == 2 ? 40 : up_w(nu, x) - 2; }
__host__ __device__ constexpr int up_cw(int nu, int x) { return up_w(nu, x) / 2 + 2; }
__host__ __device__ constexpr int up_coff(int nu, int x) { return align_off((2 * nu + x + 1) / 2); }
__host__ __device__ constexpr int up_cbw(int nu, int x) { return round4(up_coff(nu, x) + up_cw(nu, x)); }

// Tensor maps of one level (JobDev::tmaps + kTmapsPerLevel * l + index).
enum {
  kMapDownF = 0,    // f_l, box down_bw x down_w
  kMapDownF0b = 1,  // level 0's second right-hand side, same box
  kMapUpE = 2,      // e_l, box up_bw x up_w
  kMapUpF = 3,      // f_l, same box
  kMapUpF0b = 4,    // level 0's second right-hand side, same box
  kMapUpC = 5,      // the coarser correction read by the up leg (e or eu of level l + 1), box up_cbw x up_cw
  kTmapsPerLevel = 6
};

}  // namespace mgt
