// The fused RK stage kernel, tiled through shared memory.
//
// A persistent block walks tiles of 64 elements (two runs of 32 consecutive
// elements, see StageArgs) and advances each through one stage of the nodal
// DG scheme (Evolve.cpp:135-308, numerical_flux Numericalflux.cpp:13-157,
// stage update Timestepping.cpp:85-306 / :39-82). The state crosses HBM once
// per stage:
//
//   0. prefetch (TMA bulk prefetch into L2) the next tile's state rows,
//             geometry and neighbour rows, and this tile's RK base and
//             accumulator rows, so the dependent loads below hit L2;
//   1. load   the tile's state (2*Np double2 rows), the neighbours across
//             side 0 (their p+1 side nodes), the neighbour table and the
//             tile's face list into shared memory;
//   2. faces  one work item per (face, Gauss point) from the list built once
//             at set-up (vt_schedule.cuh). A face between two tile elements
//             is evaluated once, by the element with the smaller index, and
//             written to both elements' slots (the partner sees -F at the
//             mirrored point nfq-1-q, its outward normal being -n); a face
//             leaving the tile is evaluated by each side, as in the reference;
//   3. lift   4 threads per element, one conserved component each: surface
//             term -(len_s/detJ) LIFT_s F_s into Np accumulators;
//   4. flux   the nodal Euler flux of every node, contracted with the inverse
//             Jacobian, once, into shared memory;
//   5. volume D_xi G_xi + D_eta G_eta, then the RK stage update written back.
//
// The reference's mass-inverse apply is folded into D and LIFT on the host.
// Shared-memory rows are padded by one element so that rows that differ by a
// multiple of 128 bytes do not fall into the same banks.
#pragma once

#include "vt_device.cuh"

namespace vt {

__host__ __device__ constexpr int align16(int b) { return (b + 15) / 16 * 16; }

template <int P, int NFQ>
struct TileLayout {
  static constexpr int E = kTileElems;
  static constexpr int NP = np_of_p(P);
  static constexpr int NE = P + 1;
  static constexpr int ES = E + 1;  // padded row length (elements)
  static constexpr int kFBDoubles = (3 * 4 * NFQ > NP * 8 ? 3 * 4 * NFQ : NP * 8) * ES;
  // byte offsets into dynamic shared memory, each 16-byte aligned
  static constexpr int kS = 0;                                   // double2 [2NP][ES]
  static constexpr int kH = align16(kS + 2 * NP * ES * 16);      // double2 [2NE][ES]
  static constexpr int kFB = align16(kH + 2 * NE * ES * 16);     // double [3][4][NFQ][ES] | [NP][8][ES]
  static constexpr int kTP = align16(kFB + kFBDoubles * 8);      // double [3][NFQ][NE]
  static constexpr int kTM = align16(kTP + 3 * NFQ * NE * 8);    // double [3][NFQ][NE]
  static constexpr int kNB = align16(kTM + 3 * NFQ * NE * 8);    // int4 [E]
  static constexpr int kEL = align16(kNB + E * 16);              // int [E] global element index
  static constexpr int kItems = align16(kEL + E * 4);            // int [kMaxItems]
  static constexpr int kBytes = align16(kItems + kMaxItems * 4);
};

// L2 prefetch of [p, p + bytes) through the TMA unit; bytes is a multiple of
// 16 and p is 16-byte aligned (every row start of the SoA layout is).
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Thread r (< 2 runs x rows) issues one row-run prefetch. `next`: the stage
// input, geometry and neighbour rows of tile `run`; otherwise this tile's
// accumulator and base rows (when the stage reads them).
template <int NP>
__device__ __forceinline__ void prefetch_runs(const StageArgs& a, const int4 run, bool next, int r) {
  const long long KP = a.Kpad;
  const int which = r & 1;
  r >>= 1;
  const int start = which ? run.z : run.x;
  const int len = which ? run.w : run.y;
  if (len <= 0) return;
  const unsigned bytes = static_cast<unsigned>(len) * 16u;
  if (next) {
    if (r < 2 * NP) prefetch_l2(a.in + r * KP + start, bytes);
    else if (r < 2 * NP + 7) prefetch_l2(a.geo + (r - 2 * NP) * KP + start, bytes);
    else if (r == 2 * NP + 7) prefetch_l2(a.nbr + start, bytes);
    return;
  }
  if (r < 2 * NP) {
    if (a.stage >= 1 && a.stage <= 3) prefetch_l2(a.acc + r * KP + start, bytes);
  } else if (r < 4 * NP) {
    if (a.stage == 1 || a.stage == 2) prefetch_l2(a.base + (r - 2 * NP) * KP + start, bytes);
  }
}

template <int P, int NFQ>
// Three 256-thread blocks per SM (<= 80 registers per thread) keep 24 warps
// resident alongside 3 x ~75 KB of shared memory.
__global__ void __launch_bounds__(4 * kTileElems, 3) tile_stage_kernel(const StageArgs a,
                                                                        const StageOps<P, NFQ> ops) {
  using L = TileLayout<P, NFQ>;
  constexpr int E = L::E;
  constexpr int NP = L::NP;
  constexpr int NE = L::NE;
  constexpr int ES = L::ES;
  constexpr int T = 4 * E;
  extern __shared__ __align__(16) unsigned char smem[];
  double2* S = reinterpret_cast<double2*>(smem + L::kS);
  double2* H = reinterpret_cast<double2*>(smem + L::kH);
  double* FB = reinterpret_cast<double*>(smem + L::kFB);
  double* TP = reinterpret_cast<double*>(smem + L::kTP);
  double* TM = reinterpret_cast<double*>(smem + L::kTM);
  int4* NB = reinterpret_cast<int4*>(smem + L::kNB);
  int* EL = reinterpret_cast<int*>(smem + L::kEL);
  int* items = reinterpret_cast<int*>(smem + L::kItems);

  const int t = threadIdx.x;
  const long long KP = a.Kpad;

  {
    const double* tp = &ops.tp[0][0][0];
    const double* tm = &ops.tm[0][0][0];
    for (int l = t; l < 3 * NFQ * NE; l += T) {
      TP[l] = tp[l];
      TM[l] = tm[l];
    }
  }

  for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    const int4 run = __ldg(a.tiles + tile);
    const int nitems = __ldg(a.tile_count + tile);

    // ---- 0. prefetch ------------------------------------------------------------
    if (t < 64) {
      if (tile + gridDim.x < a.ntiles) prefetch_runs<NP>(a, __ldg(a.tiles + tile + gridDim.x), true, t);
    } else if (t < 64 + 8 * NP) {
      prefetch_runs<NP>(a, run, false, t - 64);
    }

    // ---- 1. load ------------------------------------------------------------------
    {
      const int col = t % E, grp = t / E;
      const int pos = col % kTileRun;
      const bool second = col >= kTileRun;
      const int e = (second ? run.z : run.x) + pos;
      const bool valid = pos < (second ? run.w : run.y);
      int4 nb = make_int4(0, 0, 0, 0);
      if (valid) nb = __ldg(a.nbr + e);
      if (grp == 0) {
        NB[col] = nb;
        EL[col] = valid ? e : -1;
      }
#pragma unroll
      for (int r = grp; r < 2 * NP; r += 4)
        S[r * ES + col] = valid ? __ldg(a.in + r * KP + e) : make_double2(1.0, 0.0);
#pragma unroll
      for (int r = grp; r < 2 * NE; r += 4)  // side 0 nodes are nodes 0..P: rows 0..2P+1
        H[r * ES + col] = valid ? __ldg(a.in + r * KP + nb.x) : make_double2(1.0, 0.0);
      const int* src = a.tile_items + static_cast<long long>(tile) * kMaxItems;
      for (int i = t; i < nitems; i += T) items[i] = __ldg(src + i);
    }
    __syncthreads();

    // ---- 2. faces ----------------------------------------------------------------------
    for (int w = t; w < nitems * NFQ; w += T) {
      const int it = items[w / NFQ];
      const int q = w % NFQ;
      const int el = it & 0xff, s = (it >> 8) & 3;
      const bool mirror = (it >> 10) & 1;
      const int nl = (it >> 11) & 0xff;
      const int e = EL[el];
      const double2 n = __ldg(a.geo + (2 + s) * KP + e);
      const int4 nb4 = NB[el];
      const int nb = s == 0 ? nb4.x : (s == 1 ? nb4.y : nb4.z);
      double up[4] = {0, 0, 0, 0}, um[4] = {0, 0, 0, 0};
#pragma unroll
      for (int k = 0; k < NE; ++k) {
        const int node = s == 0 ? edge_node(P, 0, k) : (s == 1 ? edge_node(P, 1, k) : edge_node(P, 2, k));
        const double cp = TP[(s * NFQ + q) * NE + k];
        const double cm = TM[(s * NFQ + q) * NE + k];
        const double2 o0 = S[(2 * node) * ES + el], o1 = S[(2 * node + 1) * ES + el];
        double2 n0, n1;
        if (mirror) {
          n0 = S[(2 * node) * ES + nl];
          n1 = S[(2 * node + 1) * ES + nl];
        } else if (s == 0) {
          n0 = H[(2 * k) * ES + el];
          n1 = H[(2 * k + 1) * ES + el];
        } else {
          n0 = __ldg(a.in + (2 * node) * KP + nb);
          n1 = __ldg(a.in + (2 * node + 1) * KP + nb);
        }
        up[0] = fma(cp, o0.x, up[0]);
        up[1] = fma(cp, o0.y, up[1]);
        up[2] = fma(cp, o1.x, up[2]);
        up[3] = fma(cp, o1.y, up[3]);
        um[0] = fma(cm, n0.x, um[0]);
        um[1] = fma(cm, n0.y, um[1]);
        um[2] = fma(cm, n1.x, um[2]);
        um[3] = fma(cm, n1.y, um[3]);
      }
      double f[4];
      const int code = roe_flux(up, um, n.x, n.y, f);
      if (code) record_error(a, NFQ, e, q, s, code);
#pragma unroll
      for (int c = 0; c < 4; ++c) FB[((s * 4 + c) * NFQ + q) * ES + el] = f[c];
      if (mirror) {
#pragma unroll
        for (int c = 0; c < 4; ++c) FB[((s * 4 + c) * NFQ + (NFQ - 1 - q)) * ES + nl] = -f[c];
      }
    }
    __syncthreads();

    // ---- 3. lift: thread (element el, component c) --------------------------------------
    const int c = t / E;  // uniform per warp
    const int el = t % E;
    const int e = EL[el];
    const bool valid = e >= 0;
    const int eg = valid ? e : run.x;
    double r[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) r[i] = 0.0;
    {
      const double2 lsa = __ldg(a.geo + 5 * KP + eg);
      const double2 lsb = __ldg(a.geo + 6 * KP + eg);
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const double ls = s == 0 ? lsa.x : (s == 1 ? lsa.y : lsb.x);
#pragma unroll
        for (int q = 0; q < NFQ; ++q) {
          const double fs = ls * FB[((s * 4 + c) * NFQ + q) * ES + el];
#pragma unroll
          for (int i = 0; i < NP; ++i) r[i] = fma(-ops.lift[s][i][q], fs, r[i]);
        }
      }
    }
    __syncthreads();

    // ---- 4. nodal flux of every node, once: G[j][0..3] xi, G[j][4..7] eta ---------------
    if (P > 0) {
      double* G = FB;
      const double2 j0 = __ldg(a.geo + 0 * KP + eg);
      const double2 j1 = __ldg(a.geo + 1 * KP + eg);
      for (int j = c; j < NP; j += 4) {
        const double2 s0 = S[(2 * j) * ES + el], s1 = S[(2 * j + 1) * ES + el];
        const double sv[4] = {s0.x, s0.y, s1.x, s1.y};
        double gxi[4], geta[4];
        contravariant_flux(sv, j0.x, j0.y, j1.x, j1.y, gxi, geta);
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          G[(j * 8 + cc) * ES + el] = gxi[cc];
          G[(j * 8 + 4 + cc) * ES + el] = geta[cc];
        }
      }
      __syncthreads();

      // ---- 5a. volume ------------------------------------------------------------------
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        const double gx = G[(j * 8 + c) * ES + el];
        const double gy = G[(j * 8 + 4 + c) * ES + el];
#pragma unroll
        for (int i = 0; i < NP; ++i) r[i] = fma(ops.D[0][i][j], gx, fma(ops.D[1][i][j], gy, r[i]));
      }
    }

    // ---- 5b. stage update: component c of every node ----------------------------------
    if (valid) {
      const int h = c >> 1, part = c & 1;
      const long long off0 = (h * KP + e) * 2 + part;  // node 0; node i adds i * 4 * KP
      const double* base = reinterpret_cast<const double*>(a.base) + off0;
      double* acc = reinterpret_cast<double*>(a.acc) + off0;
      double* out = reinterpret_cast<double*>(a.out) + off0;
      const double* sv = reinterpret_cast<const double*>(S + h * ES + el) + part;
      const long long step = 4 * KP;  // doubles between node rows of the same pair
      switch (a.stage) {
        case 0:
#pragma unroll
          for (int i = 0; i < NP; ++i) {
            const double u = sv[i * 4 * ES];
            acc[i * step] = fma(a.c_acc, r[i], u);
            out[i * step] = fma(a.c_out, r[i], u);
          }
          break;
        case 1:
        case 2:
#pragma unroll
          for (int i = 0; i < NP; ++i) {
            acc[i * step] = fma(a.c_acc, r[i], acc[i * step]);
            out[i * step] = fma(a.c_out, r[i], __ldg(base + i * step));
          }
          break;
        case 3:
#pragma unroll
          for (int i = 0; i < NP; ++i) out[i * step] = fma(a.c_out, r[i], acc[i * step]);
          break;
        case kStageEuler:
#pragma unroll
          for (int i = 0; i < NP; ++i) out[i * step] = fma(a.c_out, r[i], sv[i * 4 * ES]);
          break;
        default:
#pragma unroll
          for (int i = 0; i < NP; ++i) out[i * step] = r[i];
          break;
      }
    }
    __syncthreads();  // the next tile reuses the shared buffers
  }

  if (a.stage == 3 || a.stage == kStageEuler) {
    if (t == 0) {
      __threadfence();
      const unsigned long long done = atomicAdd(&a.err[2], 1ull);
      if (done == gridDim.x - 1) {
        a.err[2] = 0ull;
        atomicAdd(&a.err[1], 1ull);
      }
    }
  }
}

}  // namespace vt
