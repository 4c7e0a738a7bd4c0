// The fused RK stage kernel, tiled through shared memory.
//
// One block advances a tile of E consecutive elements through one stage of
// the nodal DG scheme (Evolve.cpp:135-308, numerical_flux Numericalflux.cpp:13-157,
// stage update Timestepping.cpp:85-306 / :39-82). The state crosses HBM once:
//
//   1. load   the tile's state (2*Np double2 rows x E, coalesced), the
//             neighbours across side 0 (their p+1 side nodes) and the
//             neighbour table into shared memory;
//   2. faces  one work item per (edge, Gauss point). An edge between two tile
//             elements is evaluated once, by the element with the smaller
//             index, and its flux is written to both elements' slots (the
//             partner sees -F at the mirrored point nfq-1-q, its outward
//             normal being -n); an edge leaving the tile is evaluated by each
//             side, as in the reference;
//   3. lift   4 threads per element, one conserved component each: surface
//             term -(len_s/detJ) LIFT_s F_s into 10 accumulators;
//   4. flux   the nodal Euler flux, contracted with the inverse Jacobian, of
//             every node, once, into shared memory;
//   5. volume D_xi G_xi + D_eta G_eta, then the RK stage update written back.
//
// The reference's mass-inverse apply is folded into D and LIFT on the host.
#pragma once

#include "vt_device.cuh"

namespace vt {

__host__ __device__ constexpr int align16(int b) { return (b + 15) / 16 * 16; }

template <int P, int NFQ, int E>
struct TileLayout {
  static constexpr int NP = np_of_p(P);
  static constexpr int NE = P + 1;
  // byte offsets into dynamic shared memory, each 16-byte aligned
  static constexpr int kS = 0;                                        // double2 [2NP][E]
  static constexpr int kH = align16(kS + 2 * NP * E * 16);            // double2 [2NE][E]
  static constexpr int kFB = align16(kH + 2 * NE * E * 16);           // double [3][NFQ][4][E] | [NP][8][E]
  static constexpr int kFBBytes = (3 * NFQ * 4 > NP * 8 ? 3 * NFQ * 4 : NP * 8) * E * 8;
  static constexpr int kTP = align16(kFB + kFBBytes);                 // double [3][NFQ][NE]
  static constexpr int kTM = align16(kTP + 3 * NFQ * NE * 8);         // double [3][NFQ][NE]
  static constexpr int kNB = align16(kTM + 3 * NFQ * NE * 8);         // int4 [E]
  static constexpr int kItems = align16(kNB + E * 16);                // int [3E]
  static constexpr int kCount = align16(kItems + 3 * E * 4);          // int [32]
  static constexpr int kBytes = align16(kCount + 32 * 4);
};

template <int P, int NFQ, int E>
__global__ void __launch_bounds__(4 * E) tile_stage_kernel(const StageArgs a, const StageOps<P, NFQ> ops) {
  using L = TileLayout<P, NFQ, E>;
  constexpr int NP = L::NP;
  constexpr int NE = L::NE;
  constexpr int T = 4 * E;
  extern __shared__ __align__(16) unsigned char smem[];
  double2* S = reinterpret_cast<double2*>(smem + L::kS);
  double2* H = reinterpret_cast<double2*>(smem + L::kH);
  double* FB = reinterpret_cast<double*>(smem + L::kFB);
  double* TP = reinterpret_cast<double*>(smem + L::kTP);
  double* TM = reinterpret_cast<double*>(smem + L::kTM);
  int4* NB = reinterpret_cast<int4*>(smem + L::kNB);
  int* items = reinterpret_cast<int*>(smem + L::kItems);
  int* counts = reinterpret_cast<int*>(smem + L::kCount);

  const int t = threadIdx.x;
  const int e0 = blockIdx.x * E;
  const long long KP = a.Kpad;

  // ---- 1. load ---------------------------------------------------------------
  {
    const int col = t % E, grp = t / E;
    const int e = e0 + col;
    const bool valid = e < a.K;
    int4 nb = make_int4(e, e, e, 0);
    if (valid) nb = __ldg(a.nbr + e);
    if (grp == 0) NB[col] = nb;
#pragma unroll
    for (int r = grp; r < 2 * NP; r += 4)
      S[r * E + col] = valid ? __ldg(a.in + r * KP + e) : make_double2(1.0, 0.0);
#pragma unroll
    for (int r = grp; r < 2 * NE; r += 4) {
      // side 0 nodes are nodes 0..P: rows 0..2P+1
      H[r * E + col] = valid ? __ldg(a.in + r * KP + nb.x) : make_double2(1.0, 0.0);
    }
    const double* tp = &ops.tp[0][0][0];
    const double* tm = &ops.tm[0][0][0];
    for (int l = t; l < 3 * NFQ * NE; l += T) {
      TP[l] = tp[l];
      TM[l] = tm[l];
    }
  }
  __syncthreads();

  // ---- edge list: (element, side) pairs this tile evaluates ------------------
  {
    const int lane = t & 31, warp = t >> 5;
    bool take = false;
    int code = 0;
    if (t < 3 * E) {
      const int el = t / 3, s = t % 3;
      if (e0 + el < a.K) {
        const int4 nb4 = NB[el];
        const int nb = s == 0 ? nb4.x : (s == 1 ? nb4.y : nb4.z);
        const int nl = nb - e0;
        const bool inside = nl >= 0 && nl < E;
        take = !inside || (e0 + el < nb);
        code = el | (s << 8) | ((inside && nb != e0 + el) ? (1 << 10) : 0);
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, take);
    if (lane == 0) counts[warp] = __popc(m);
    __syncthreads();
    int base = 0;
    for (int w = 0; w < warp; ++w) base += counts[w];
    if (take) items[base + __popc(m & ((1u << lane) - 1u))] = code;
    __syncthreads();
    if (t == 0) {
      int n = 0;
      for (int w = 0; w < T / 32; ++w) n += counts[w];
      counts[T / 32] = n;
    }
    __syncthreads();
  }
  const int nitems = counts[T / 32];

  // ---- 2. faces ------------------------------------------------------------------
  for (int w = t; w < nitems * NFQ; w += T) {
    const int it = items[w / NFQ];
    const int q = w % NFQ;
    const int el = it & 0xff, s = (it >> 8) & 3;
    const bool mirror = (it >> 10) & 1;
    const int e = e0 + el;
    const int4 nb4 = NB[el];
    const int nb = s == 0 ? nb4.x : (s == 1 ? nb4.y : nb4.z);
    const int nl = nb - e0;
    const bool inside = nl >= 0 && nl < E;
    double up[4] = {0, 0, 0, 0}, um[4] = {0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < NE; ++k) {
      const int node = s == 0 ? edge_node(P, 0, k) : (s == 1 ? edge_node(P, 1, k) : edge_node(P, 2, k));
      const double cp = TP[(s * NFQ + q) * NE + k];
      const double cm = TM[(s * NFQ + q) * NE + k];
      const double2 o0 = S[(2 * node) * E + el], o1 = S[(2 * node + 1) * E + el];
      double2 n0, n1;
      if (inside) {
        n0 = S[(2 * node) * E + nl];
        n1 = S[(2 * node + 1) * E + nl];
      } else if (s == 0) {
        n0 = H[(2 * k) * E + el];
        n1 = H[(2 * k + 1) * E + el];
      } else {
        n0 = __ldg(a.in + (2 * node) * KP + nb);
        n1 = __ldg(a.in + (2 * node + 1) * KP + nb);
      }
      up[0] += cp * o0.x;
      up[1] += cp * o0.y;
      up[2] += cp * o1.x;
      up[3] += cp * o1.y;
      um[0] += cm * n0.x;
      um[1] += cm * n0.y;
      um[2] += cm * n1.x;
      um[3] += cm * n1.y;
    }
    const double2 n = __ldg(a.geo + (2 + s) * KP + e);
    double f[4];
    const int code = roe_flux(up, um, n.x, n.y, f);
    if (code) record_error(a, NFQ, e, q, s, code);
#pragma unroll
    for (int c = 0; c < 4; ++c) FB[((s * NFQ + q) * 4 + c) * E + el] = f[c];
    if (mirror) {
#pragma unroll
      for (int c = 0; c < 4; ++c) FB[((s * NFQ + (NFQ - 1 - q)) * 4 + c) * E + nl] = -f[c];
    }
  }
  __syncthreads();

  // ---- 3. lift: thread (element el, component c) ----------------------------------
  const int c = t / E;  // uniform per warp
  const int el = t % E;
  const int e = e0 + el;
  const bool valid = e < a.K;
  double r[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) r[i] = 0.0;
  {
    const double2 lsa = __ldg(a.geo + 5 * KP + (valid ? e : 0));
    const double2 lsb = __ldg(a.geo + 6 * KP + (valid ? e : 0));
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const double ls = s == 0 ? lsa.x : (s == 1 ? lsa.y : lsb.x);
#pragma unroll
      for (int q = 0; q < NFQ; ++q) {
        const double fs = ls * FB[((s * NFQ + q) * 4 + c) * E + el];
#pragma unroll
        for (int i = 0; i < NP; ++i) r[i] -= ops.lift[s][i][q] * fs;
      }
    }
  }
  __syncthreads();

  // ---- 4. nodal flux of every node, once: G[j][0..3] xi, G[j][4..7] eta ------
  double* G = FB;
  if (P > 0) {
    const double2 j0 = __ldg(a.geo + 0 * KP + (valid ? e : 0));
    const double2 j1 = __ldg(a.geo + 1 * KP + (valid ? e : 0));
#pragma unroll
    for (int j = c; j < NP; j += 4) {
      const double2 s0 = S[(2 * j) * E + el], s1 = S[(2 * j + 1) * E + el];
      const double sv[4] = {s0.x, s0.y, s1.x, s1.y};
      double gxi[4], geta[4];
      contravariant_flux(sv, j0.x, j0.y, j1.x, j1.y, gxi, geta);
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) {
        G[(j * 8 + cc) * E + el] = gxi[cc];
        G[(j * 8 + 4 + cc) * E + el] = geta[cc];
      }
    }
    __syncthreads();

    // ---- 5a. volume ------------------------------------------------------------------
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      const double gx = G[(j * 8 + c) * E + el];
      const double gy = G[(j * 8 + 4 + c) * E + el];
#pragma unroll
      for (int i = 0; i < NP; ++i) r[i] += ops.D[0][i][j] * gx + ops.D[1][i][j] * gy;
    }
  }

  // ---- 5b. stage update: component c of every node ------------------------------------
  if (valid) {
    const int h = c >> 1, part = c & 1;
    const double* base = reinterpret_cast<const double*>(a.base);
    double* acc = reinterpret_cast<double*>(a.acc);
    double* out = reinterpret_cast<double*>(a.out);
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const long long idx = (((2 * i + h) * KP) + e) * 2 + part;
      const double2 sv = S[(2 * i + h) * E + el];
      const double u = part ? sv.y : sv.x;
      switch (a.stage) {
        case 0:
          acc[idx] = u + a.c_acc * r[i];
          out[idx] = u + a.c_out * r[i];
          break;
        case 1:
        case 2:
          acc[idx] = acc[idx] + a.c_acc * r[i];
          out[idx] = __ldg(base + idx) + a.c_out * r[i];
          break;
        case 3:
          out[idx] = acc[idx] + a.c_out * r[i];
          break;
        case kStageEuler:
          out[idx] = u + a.c_out * r[i];
          break;
        default:
          out[idx] = r[i];
          break;
      }
    }
  }

  if (a.stage == 3 || a.stage == kStageEuler) {
    __syncthreads();
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
