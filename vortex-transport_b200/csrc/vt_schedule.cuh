// Tile schedule of the stage kernel: which elements form each tile and which
// faces each tile evaluates. Built once per mesh.
//
// A tile is two runs of up to 32 consecutive elements. On the reference's
// structured mesh (Meshgeneration.cpp:57-117: cell (j, row) holds elements
// 2(row*nx + j) and +1) a tile is 16 cells of two adjacent rows, so the faces
// between the two rows are evaluated once inside the tile; on any other mesh a
// tile is 64 consecutive elements.
#pragma once

#include <vector>

#include "vt_device.cuh"

namespace vt {

// Two-row tiles of the reference's structured mesh with nx x ny cells (nx a
// multiple of kTileRun / 2 and ny even); empty otherwise.
inline std::vector<int4> grid_tiles(int nx, int ny) {
  std::vector<int4> tiles;
  constexpr int cells = kTileRun / 2;  // cells per run
  if (nx < 1 || ny < 1 || nx % cells || ny % 2) return tiles;
  for (int rp = 0; rp < ny / 2; ++rp)
    for (int j = 0; j < nx / cells; ++j) {
      const int s0 = 2 * nx * (2 * rp) + kTileRun * j;
      tiles.push_back(make_int4(s0, kTileRun, s0 + 2 * nx, kTileRun));
    }
  return tiles;
}

// grid_tiles when `conn`/`type` are exactly the reference's periodic
// structured mesh; empty otherwise.
inline std::vector<int4> structured_tiles(int K, const int32_t* type, const int32_t* conn) {
  std::vector<int4> tiles;
  if (K < 2 || conn[1] < 1) return tiles;
  const int nx = (conn[1] + 1) / 2;  // element 0's left neighbour is 2 nx - 1
  if (nx < 1 || K % (2 * nx)) return tiles;
  const int ny = K / (2 * nx);
  for (int i = 0; i < K; ++i) {
    const int left = i % (2 * nx) == 0 ? i - 1 + 2 * nx : i - 1;
    const int right = (i + 1) % (2 * nx) == 0 ? i + 1 - 2 * nx : i + 1;
    // the reference's three loops, later ones overwriting earlier ones
    int vert;
    if (i >= 2 * nx * (ny - 1)) vert = i % 2 == 0 ? i + 1 - 2 * nx : i - 1 - 2 * nx * (ny - 1);
    else if (i >= 2 * nx) vert = i % 2 == 0 ? i + 1 - 2 * nx : i - 1 + 2 * nx;
    else vert = i % 2 == 0 ? i + 1 + 2 * nx * (ny - 1) : i - 1 + 2 * nx;
    if (type[i] != i % 2 || conn[3 * i] != right || conn[3 * i + 1] != left || conn[3 * i + 2] != vert)
      return tiles;
  }
  return grid_tiles(nx, ny);
}

__global__ void contiguous_tiles_kernel(int4* tiles, int K, int ntiles) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  const int s0 = t * kTileElems, s1 = s0 + kTileRun;
  const int l0 = min(kTileRun, K - s0), l1 = max(0, min(kTileRun, K - s1));
  tiles[t] = make_int4(s0, l0, s1, l1);
}

// One block of 256 threads per tile: every (element, side) of the tile is a
// candidate; it is evaluated here when the neighbour is outside the tile or
// has a larger index. Grouped by how the outer state is found -- a partner in
// the tile, a side-0 neighbour staged in shared memory, any other neighbour
// read from global memory -- so that a warp's work items take one path, and
// in (element, side) order within a group.
//
// The stage kernel gives work item w = item * nfq + q to thread w mod 256, so
// with nw = n * nfq > 256 the threads below L = nw mod 256 (or all, when L is
// 0) take one item more than the rest. The items of the last group wait on
// global loads; they are placed on threads with one item fewer (item indices
// from ceil(L / nfq) on, in the first round) when they fit there, so that
// their latency does not lengthen the face phase.
__global__ void build_tile_items_kernel(const int4* __restrict__ tiles, const int4* __restrict__ nbr,
                                        int* __restrict__ items, int* __restrict__ count, int nfq) {
  __shared__ int warp_n[3][8];
  const int tile = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int4 run = tiles[tile];
  bool take = false;
  int code = 0, cls = 0;
  if (t < kMaxItems) {
    const int el = t / 3, s = t % 3;
    const int pos = el % kTileRun;
    const bool second = el >= kTileRun;
    const int e = (second ? run.z : run.x) + pos;
    if (pos < (second ? run.w : run.y)) {
      const int4 n4 = nbr[e];
      const int nb = s == 0 ? n4.x : (s == 1 ? n4.y : n4.z);
      int nl = -1;
      if (nb >= run.x && nb < run.x + run.y) nl = nb - run.x;
      else if (nb >= run.z && nb < run.z + run.w) nl = kTileRun + nb - run.z;
      const bool inside = nl >= 0 && nb != e;
      take = !inside || e < nb;
      code = el | (s << 8) | (inside ? (1 << 10) | (nl << 11) : 0);
      cls = inside ? 0 : (s == 0 ? 1 : 2);
    }
  }
  unsigned m[3];
  for (int k = 0; k < 3; ++k) {
    m[k] = __ballot_sync(0xffffffffu, take && cls == k);
    if (lane == 0) warp_n[k][warp] = __popc(m[k]);
  }
  __syncthreads();
  int n_cls[3] = {0, 0, 0};
  for (int k = 0; k < 3; ++k)
    for (int w = 0; w < 8; ++w) n_cls[k] += warp_n[k][w];
  const int n = n_cls[0] + n_cls[1] + n_cls[2];
  // where the global-gather group goes: item index k0, or after the others
  const int T = 4 * kTileElems, nw = n * nfq;
  const int L = nw % T;
  const int k0 = nfq > 0 ? (L + nfq - 1) / nfq : 0;
  const bool move = nw > T && L > 0 && (k0 + n_cls[2]) * nfq <= T && k0 <= n_cls[0] + n_cls[1];
  int rank = 0;  // position within the (class 0, class 1, class 2) order
  for (int k = 0; k < cls; ++k) rank += n_cls[k];
  for (int w = 0; w < warp; ++w) rank += warp_n[cls][w];
  rank += __popc(m[cls] & ((1u << lane) - 1u));
  int slot = rank;
  if (move) {
    if (cls == 2) slot = k0 + (rank - n_cls[0] - n_cls[1]);
    else if (rank >= k0) slot = rank + n_cls[2];
  }
  if (take) items[static_cast<long long>(tile) * kMaxItems + slot] = code;
  if (t == 0) count[tile] = n;
}

}  // namespace vt
