// Device-side building blocks of the stepper: state layout, folded operators,
// Roe flux, nodal flux and the first-error record.
//
// HBM layout of a state vector (U, a stage, the RK accumulator): structure of
// arrays of double2, row r = 2*i + h for node i and component pair h
// (h = 0: rho, rho u; h = 1: rho v, rho E), element e in the column:
//   state[r * Kpad + e]
// A warp touching 32 consecutive elements of one row reads 512 contiguous
// bytes; one element's state is 2*Np 16-byte loads.
#pragma once

#include <cuda.h>

#include <cstdint>

namespace vt {

constexpr double kGamma = 1.4;
// (gamma - 1) exactly as the reference forms it (1.4 - 1.0 = 0.3999999999999999).
constexpr double kGm1 = 1.4 - 1.0;

__host__ __device__ constexpr int np_of_p(int p) { return (p + 1) * (p + 2) / 2; }

// Node numbering of Meshgeneration.cpp:208-216: j (eta) outer, i (xi) inner.
__host__ __device__ constexpr int node_id(int p, int i, int j) { return j * (p + 1) - j * (j - 1) / 2 + i; }

// k-th node (0..p) on side s of the reference triangle: s = 0 is the side
// eta = 0 (reference side 1), s = 1 is xi + eta = 1 (side 2), s = 2 is
// xi = 0 (side 3). Only these p + 1 basis functions are non-zero on the side.
__host__ __device__ constexpr int edge_node(int p, int s, int k) {
  return s == 0 ? node_id(p, k, 0) : (s == 1 ? node_id(p, p - k, k) : node_id(p, 0, k));
}

// Operators shared by all elements, folded on the host (vt_solver.cu):
//   D[0] = M_ref^-1 S_xi, D[1] = M_ref^-1 S_eta          (volume term)
//   lift[s][i][q] = sum_j M_ref^-1[i][j] phi+_s(q)_j w_q  (surface term)
//   tp[s][q][k], tm[s][q][k]: own / neighbour basis at face point q restricted
//   to the p + 1 nodes of side s.
// Passed by value as a kernel parameter, so every coefficient is an immediate
// constant-bank operand of the FMA that uses it.
template <int P, int NFQ>
struct StageOps {
  static constexpr int NP = np_of_p(P);
  static constexpr int NE = P + 1;
  double D[2][NP][NP];
  double lift[3][NP][NFQ];
  double tp[3][NFQ][NE];
  double tm[3][NFQ][NE];
};

// What one stage launch reads and writes. Geometry rows (double2, Kpad each):
//   0: (Jinv00, Jinv01)  1: (Jinv10, Jinv11)  2..4: normal of side 0..2
//   5: (len0/detJ, len1/detJ)  6: (len2/detJ, 0)
// nbr[e] = (neighbour across side 0, 1, 2, unused).
//
// Tiles: tiles[t] = (start0, len0, start1, len1), two runs of consecutive
// elements (local columns 0..31 and 32..63). tile_items[t * kMaxItems + i],
// i < tile_count[t], lists the (element, side) faces tile t evaluates:
//   bits 0-7 local element, 8-9 side, 10 mirror (the neighbour is in the tile
//   and receives -F), 11-18 the neighbour's local column when mirrored.
struct StageArgs {
  const double2* in;    // state the right-hand side is evaluated on
  const double2* base;  // U_n (RK4 stages 1, 2)
  double2* acc;         // RK4 accumulator X (written by stage 1, read by stage 3; vt_tile.cuh)
  double2* out;         // next stage state / new U / the right-hand side itself
  const double2* geo;
  const int4* nbr;
  const int4* tiles;
  const int* tile_items;
  const int* tile_count;
  const double* tile_dt;  // per-tile time step (batched problems), or null: c_* hold dt
  unsigned long long* err;  // [0] first-error key, [1] steps done, [2] blocks done
  long long Kpad;
  int K;
  int ntiles;
  int stage;     // 0..3 RK4 stages, 4 forward Euler, 5 right-hand side only
  double c_acc;  // accumulator coefficient (stage 1)
  double c_out;  // output coefficient
  // Test hook of the bounded waits (vt_test_bulk_wait): polls of the tile's
  // mbarrier before a wait gives up (0: the default bound), and bit 0 of
  // test_flags issues no state copies at all, so every wait gives up.
  unsigned wait_tries = 0;
  int test_flags = 0;
  // RK4 stages 0-2 that only produce the next stage state (a step rerun to
  // keep its stage states): stage 1 does not form the accumulator
  int no_acc = 0;
  // 2-D tensor maps of in / acc / base, [2 Np rows] x [2 Kpad doubles], box of
  // 2 Np rows x 64 doubles (one 32-element run); encoded on the host by the
  // launcher, read by the tensor copies through this grid-constant parameter
  CUtensorMap map_in, map_acc, map_base;
};

enum : int { kTestNoCopies = 1 };

constexpr int kTileRun = 32;            // elements per run
constexpr int kTileElems = 2 * kTileRun;  // elements per tile
constexpr int kMaxItems = 3 * kTileElems;

enum : int { kStageEuler = 4, kStageRhs = 5 };

// Warp mappings of the stage kernel (vt_tile.cuh): one thread per (element,
// component), or per (element, component pair, node half).
enum : int { kMapComponent = 0, kMapPair = 1 };

// First-error key: (stage epoch << 40) | (((e * nfq + q) * 3 + s) * 4 + code).
// The minimum over all failures is the failure the reference's serial loop
// meets first: earliest stage, then element, face point, side, check.
__device__ __forceinline__ void record_error(const StageArgs& a, int nfq, int e, int q, int s,
                                             int code) {
  const unsigned long long steps = *(volatile unsigned long long*)&a.err[1];
  const int slot = a.stage < 4 ? a.stage : 0;
  const unsigned long long epoch = steps * 4ull + static_cast<unsigned long long>(slot);
  const unsigned long long local =
      ((static_cast<unsigned long long>(e) * nfq + q) * 3ull + s) * 4ull + code;
  atomicMin(&a.err[0], (epoch << 40) | local);
}

// 1/x for the positive, normal x of the flux formulas (densities, Roe-average
// terms): the hardware reciprocal estimate (rcp.approx.ftz.f64, relative error
// about 1e-6 measured on B200) refined by two Newton-Raphson steps
// r <- r + r (1 - x r), each of which squares the relative error, so the
// result is within rounding of 1/x. This is the textbook Newton iteration for
// the reciprocal with the residual 1 - x r formed by one fused multiply-add,
// as in P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Develop. 34(1), 1990, and his book
// "IA-64 and Elementary Functions" (2000), ch. 8. It matched 1.0 / x bit for
// bit on 2.4 million inputs in [2^-10, 2^10] (tests/test_gpu_reciprocal.py
// bounds the difference at one ulp). Zero, subnormal and non-finite x are not
// handled (those states are non-physical and reported by the flux's checks).
__device__ __forceinline__ double recip_nr(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
}

// Roe flux with the reference's entropy fix and its squared "sound speed"
// ci = c2^2 (Numericalflux.cpp:13-157), rearranged to need one reciprocal for
// both densities, one square root and two further reciprocals per call
// (recip_nr), and to fold constant factors into fused multiply-adds:
//   p = (gamma-1) (rhoE - (m_x u + m_y v) / 2) with u = m_x / rho,
//   1/rhoL = rhoR / (rhoL rhoR), sqrt(rhoR / rhoL) = sqrt(rhoR * (1 / rhoL)),
//   1 / eps = 10 / ci, the entropy fix's halving taken into its constants,
//   the normal velocity u.n = (m.n) / rho with m.n shared with the mass flux,
//   and each flux component as 0.5 (central part - dissipation) with the two
//   pressures added once.
// Equal to the reference's expression up to rounding (about 6e-16 relative
// after two RK4 steps at 768 x 768 cells, p = 3, against the unfused form;
// 0.5% fewer cycles per step there). Returns the reference's error code
// (1 left state, 2 right state, 3 c2 <= 0) or 0.
__device__ __forceinline__ int roe_flux(const double* uL, const double* uR, double nx, double ny,
                                        double* f) {
  const double rL = uL[0];
  const double rR = uR[0];
  const double irLR = recip_nr(rL * rR);
  const double irL = rR * irLR;
  const double irR = rL * irLR;
  const double vxL = uL[1] * irL, vyL = uL[2] * irL;
  const double mnL = uL[1] * nx + uL[2] * ny;
  const double unL = mnL * irL;
  const double pL = kGm1 * fma(-0.5, uL[1] * vxL + uL[2] * vyL, uL[3]);
  int code = 0;
  if ((pL <= 0) || (rL <= 0)) code = 1;
  const double rHL = uL[3] + pL;
  const double HL = rHL * irL;

  const double vxR = uR[1] * irR, vyR = uR[2] * irR;
  const double mnR = uR[1] * nx + uR[2] * ny;
  const double unR = mnR * irR;
  const double pR = kGm1 * fma(-0.5, uR[1] * vxR + uR[2] * vyR, uR[3]);
  if (code == 0 && ((pR <= 0) || (rR <= 0))) code = 2;
  const double rHR = uR[3] + pR;
  const double HR = rHR * irR;

  const double du0 = uR[0] - uL[0], du1 = uR[1] - uL[1], du2 = uR[2] - uL[2], du3 = uR[3] - uL[3];

  const double di = sqrt(rR * irL);
  const double d1 = recip_nr(1.0 + di);
  const double ui = fma(di, vxR, vxL) * d1;
  const double vi = fma(di, vyR, vyL) * d1;
  const double Hi = fma(di, HR, HL) * d1;
  const double af = 0.5 * (ui * ui + vi * vi);
  const double ucp = ui * nx + vi * ny;
  const double c2 = kGm1 * (Hi - af);
  if (code == 0 && c2 <= 0) code = 3;
  const double ci = c2 * c2;
  const double ci1 = recip_nr(ci);

  // eigenvalue moduli with the entropy fix |l| < eps -> (eps + l^2/eps) / 2, eps = ci / 10,
  // the halving folded into the constants
  const double eps = 0.1 * ci, heps = 0.05 * ci, hieps = 5.0 * ci1;
  const double l0r = ucp + ci, l1r = ucp - ci;
  const double l0 = fabs(l0r) < eps ? fma(l0r * l0r, hieps, heps) : fabs(l0r);
  const double l1 = fabs(l1r) < eps ? fma(l1r * l1r, hieps, heps) : fabs(l1r);
  const double l3 = fabs(ucp) < eps ? fma(ucp * ucp, hieps, heps) : fabs(ucp);
  const double s1l3 = fma(0.5, l0 + l1, -l3);  // s1 - l3
  const double s2 = 0.5 * (l0 - l1);
  const double G1 = kGm1 * (fma(af, du0, du3) - ui * du1 - vi * du2);
  const double G2 = fma(-ucp, du0, du1 * nx + du2 * ny);
  const double C1 = fma(G1 * s1l3, ci1, G2 * s2) * ci1;
  const double C2 = fma(G1 * s2, ci1, G2 * s1l3);
  const double pLR = pL + pR;
  f[0] = 0.5 * ((mnL + mnR) - fma(l3, du0, C1));
  f[1] = 0.5 * (fma(uL[1], unL, fma(uR[1], unR, pLR * nx)) - fma(l3, du1, fma(C1, ui, C2 * nx)));
  f[2] = 0.5 * (fma(uL[2], unL, fma(uR[2], unR, pLR * ny)) - fma(l3, du2, fma(C1, vi, C2 * ny)));
  f[3] = 0.5 * (fma(rHL, unL, rHR * unR) - fma(l3, du3, fma(C1, Hi, C2 * ucp)));
  return code;
}

// Nodal Euler flux of one node's state (the formula of Timestepping.cpp:141-158)
// contracted with the inverse Jacobian rows: gxi = Jinv00 Fx + Jinv01 Fy,
// geta = Jinv10 Fx + Jinv11 Fy.
__device__ __forceinline__ void contravariant_flux(const double* s, double j00, double j01,
                                                   double j10, double j11, double* gxi,
                                                   double* geta) {
  const double ir = recip_nr(s[0]);
  const double vx = s[1] * ir, vy = s[2] * ir;
  const double p = kGm1 * (s[3] - 0.5 * (s[1] * vx + s[2] * vy));
  const double rH = s[3] + p;
  const double fx[4] = {s[1], s[1] * vx + p, s[2] * vx, rH * vx};
  const double fy[4] = {s[2], s[1] * vy, s[2] * vy + p, rH * vy};
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    gxi[c] = j00 * fx[c] + j01 * fy[c];
    geta[c] = j10 * fx[c] + j11 * fy[c];
  }
}

}  // namespace vt
