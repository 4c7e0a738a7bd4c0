// The fused RK stage kernel: right-hand side of the nodal DG discretisation
// (Evolve.cpp:135-308 with numerical_flux, Numericalflux.cpp:13-157) and the
// stage update of Timestepping.cpp:85-306 / :39-82 in one pass, so each stage
// reads its input state once from HBM and writes its outputs once.
//
// One thread per element. Volume term: nodal flux -> contravariant flux ->
// D_xi, D_eta (Np x Np). Surface term: for each side, traces of own and
// neighbour state at the Gauss points from the p + 1 nodes on that side, Roe
// flux, lift back with (len / detJ) * LIFT_s. The reference's mass-inverse
// apply is folded into D and LIFT on the host.
#pragma once

#include "vt_device.cuh"

namespace vt {

template <int P, int NFQ>
__global__ void __launch_bounds__(128) stage_kernel(const StageArgs a, const StageOps<P, NFQ> ops) {
  constexpr int NP = np_of_p(P);
  constexpr int NE = P + 1;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const long long KP = a.Kpad;

  if (e < a.K) {
    double u[NP][4];
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const double2 v0 = __ldg(a.in + (2 * i) * KP + e);
      const double2 v1 = __ldg(a.in + (2 * i + 1) * KP + e);
      u[i][0] = v0.x;
      u[i][1] = v0.y;
      u[i][2] = v1.x;
      u[i][3] = v1.y;
    }
    const int4 nb = __ldg(a.nbr + e);
    const double2 lsa = __ldg(a.geo + 5 * KP + e);
    const double2 lsb = __ldg(a.geo + 6 * KP + e);

    double r[NP][4];
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int c = 0; c < 4; ++c) r[i][c] = 0.0;

    // ---- surface term -----------------------------------------------------
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const int ne = s == 0 ? nb.x : (s == 1 ? nb.y : nb.z);
      double un[NE][4];
#pragma unroll
      for (int k = 0; k < NE; ++k) {
        const int node = edge_node(P, s, k);
        const double2 v0 = __ldg(a.in + (2 * node) * KP + ne);
        const double2 v1 = __ldg(a.in + (2 * node + 1) * KP + ne);
        un[k][0] = v0.x;
        un[k][1] = v0.y;
        un[k][2] = v1.x;
        un[k][3] = v1.y;
      }
      const double2 n = __ldg(a.geo + (2 + s) * KP + e);
      const double ls = s == 0 ? lsa.x : (s == 1 ? lsa.y : lsb.x);
#pragma unroll
      for (int q = 0; q < NFQ; ++q) {
        double up[4], um[4], f[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          double ap = 0.0, am = 0.0;
#pragma unroll
          for (int k = 0; k < NE; ++k) {
            ap += ops.tp[s][q][k] * u[edge_node(P, s, k)][c];
            am += ops.tm[s][q][k] * un[k][c];
          }
          up[c] = ap;
          um[c] = am;
        }
        const int code = roe_flux(up, um, n.x, n.y, f);
        if (code) record_error(a, NFQ, e, q, s, code);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const double fs = ls * f[c];
#pragma unroll
          for (int i = 0; i < NP; ++i) r[i][c] -= ops.lift[s][i][q] * fs;
        }
      }
    }

    // ---- volume term ------------------------------------------------------
    if (P > 0) {
      const double2 j0 = __ldg(a.geo + 0 * KP + e);
      const double2 j1 = __ldg(a.geo + 1 * KP + e);
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        double gxi[4], geta[4];
        contravariant_flux(u[j], j0.x, j0.y, j1.x, j1.y, gxi, geta);
#pragma unroll
        for (int i = 0; i < NP; ++i)
#pragma unroll
          for (int c = 0; c < 4; ++c) r[i][c] += ops.D[0][i][j] * gxi[c] + ops.D[1][i][j] * geta[c];
      }
    }

    // ---- stage update -----------------------------------------------------
#pragma unroll
    for (int i = 0; i < NP; ++i) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const long long idx = (2 * i + h) * KP + e;
        const double r0 = r[i][2 * h], r1 = r[i][2 * h + 1];
        const double s0 = u[i][2 * h], s1 = u[i][2 * h + 1];
        switch (a.stage) {
          case 0: {  // k1: acc = U + dt/6 k, next = U + dt/2 k
            a.acc[idx] = make_double2(s0 + a.c_acc * r0, s1 + a.c_acc * r1);
            a.out[idx] = make_double2(s0 + a.c_out * r0, s1 + a.c_out * r1);
            break;
          }
          case 1:
          case 2: {  // k2, k3: acc += dt/3 k, next = U + c k
            const double2 ac = a.acc[idx];
            const double2 b = __ldg(a.base + idx);
            a.acc[idx] = make_double2(ac.x + a.c_acc * r0, ac.y + a.c_acc * r1);
            a.out[idx] = make_double2(b.x + a.c_out * r0, b.y + a.c_out * r1);
            break;
          }
          case 3: {  // k4: U = acc + dt/6 k
            const double2 ac = a.acc[idx];
            a.out[idx] = make_double2(ac.x + a.c_out * r0, ac.y + a.c_out * r1);
            break;
          }
          case kStageEuler:
            a.out[idx] = make_double2(s0 + a.c_out * r0, s1 + a.c_out * r1);
            break;
          default:
            a.out[idx] = make_double2(r0, r1);
            break;
        }
      }
    }
  }

  // Step counter for the error key: the last block of a step's final stage
  // advances it, after every block of that stage has read it.
  if (a.stage == 3 || a.stage == kStageEuler) {
    __syncthreads();
    if (threadIdx.x == 0) {
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
