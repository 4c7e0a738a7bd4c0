// Kernels of the discrete adjoint and the tangent-linear model.
//
// One reverse RK4 stage (the transpose of one stage's right-hand side at the
// stage state U, applied to the stage adjoint a) is two launches:
//
//   adjoint_face_kernel     thread (element e, side s, face point q): a block
//                           is 32 consecutive elements of one side s, a warp
//                           one face point q:
//                           bF = -(len_s / detJ) sa * sum_i lift[s][i][q] a_i
//                           (transposed lift and mass inverse), then the
//                           transposed Roe Jacobian at (U+, U-) gives the face
//                           adjoints of the own trace (bp) and of the
//                           neighbour's trace (bm);
//   adjoint_element_kernel  thread (element e, node j): the transposed volume
//                           operator sum_i D[d][i][j] a_i, the transposed nodal
//                           flux Jacobian at U_j, and the transposed traces of
//                           the own faces (tp, bp of e) and of the neighbours'
//                           faces (tm, bm of the neighbour across side s, whose
//                           side s faces e), then the reverse RK4 combine.
//
// On meshes whose faces take the edge-once form the whole reverse stage is
// one launch instead, adjoint_tile_kernel (vt_adjoint_tile.cuh).
//
// Both read the state through the SoA-of-double2 layout of the stage kernel,
// so a warp's 32 consecutive elements are contiguous 512-byte rows. The
// face adjoints bp/bm hold 2 double2 rows per (s, q) face point:
//   bp[((s * NFQ + q) * 2 + h) * Kpad + e]
#pragma once

#include "vt_adjoint.cuh"
#include "vt_device.cuh"

namespace vt {

struct AdjArgs {
  const double2* U;       // stage state the right-hand side was evaluated on
  const double2* a;       // stage adjoint (multiplied by sa)
  const double2* lam;     // adjoint of U_{n+1}, or null when lam_coef = 0 and a_out is null
  const double2* acc_in;  // running adjoint of U_n, or null
  double2* acc_out;       // acc_in + lam_coef * lam + g
  double2* a_out;         // cl * lam + cg * g, or null
  double2* bp;            // face adjoints, own trace
  double2* bm;            // face adjoints, neighbour trace
  const double2* geo;
  const int4* nbr;
  // Per-element time steps (a batch group with uneven steps), or null: then
  // sa (when sa_dt is set), cl and cg are fractions of the element's step.
  const double* elem_dt;
  int sa_dt;
  // The stage kernel's tile schedule (adjoint_tile_kernel) and error words.
  const int4* tiles;
  const int* tile_items;
  const int* tile_count;
  int ntiles;
  unsigned long long* err;
  long long Kpad;
  int K;
  double sa, lam_coef, cl, cg;
  // 2-D tensor maps of U and a (adjoint_tile_kernel only), as the stage
  // kernel's: [2 Np rows] x [2 Kpad doubles], a box of one 32-element run;
  // encoded on the host by the launcher
  CUtensorMap map_U, map_a;
};

constexpr int kAdjRun = 32;  // elements per block (one per lane)

template <int P, int NFQ>
__global__ void __launch_bounds__(kAdjRun * NFQ)
    adjoint_face_kernel(const AdjArgs a, const StageOps<P, NFQ> o) {
  constexpr int NP = np_of_p(P), NE = P + 1;
  const int e = blockIdx.x * kAdjRun + threadIdx.x;
  if (e >= a.K) return;
  const int s = blockIdx.y, q = threadIdx.y;  // uniform per block / warp
  const int w = s * NFQ + q;
  const long long KP = a.Kpad;
  const int4 nb4 = __ldg(a.nbr + e);
  const int nb = s == 0 ? nb4.x : (s == 1 ? nb4.y : nb4.z);
  double up[4] = {0.0, 0.0, 0.0, 0.0}, um[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int k = 0; k < NE; ++k) {
    const int node = edge_node(P, s, k);
    const double cp = o.tp[s][q][k], cm = o.tm[s][q][k];
    const double2 x0 = __ldg(a.U + (2 * node) * KP + e), x1 = __ldg(a.U + (2 * node + 1) * KP + e);
    const double2 y0 = __ldg(a.U + (2 * node) * KP + nb), y1 = __ldg(a.U + (2 * node + 1) * KP + nb);
    up[0] = fma(cp, x0.x, up[0]);
    up[1] = fma(cp, x0.y, up[1]);
    up[2] = fma(cp, x1.x, up[2]);
    up[3] = fma(cp, x1.y, up[3]);
    um[0] = fma(cm, y0.x, um[0]);
    um[1] = fma(cm, y0.y, um[1]);
    um[2] = fma(cm, y1.x, um[2]);
    um[3] = fma(cm, y1.y, um[3]);
  }
  double bf[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    const double l = o.lift[s][i][q];
    const double2 a0 = __ldg(a.a + (2 * i) * KP + e), a1 = __ldg(a.a + (2 * i + 1) * KP + e);
    bf[0] = fma(l, a0.x, bf[0]);
    bf[1] = fma(l, a0.y, bf[1]);
    bf[2] = fma(l, a1.x, bf[2]);
    bf[3] = fma(l, a1.y, bf[3]);
  }
  const double2 lsa = __ldg(a.geo + 5 * KP + e), lsb = __ldg(a.geo + 6 * KP + e);
  const double sa = (a.elem_dt && a.sa_dt) ? a.sa * __ldg(a.elem_dt + e) : a.sa;
  const double sc = -(s == 0 ? lsa.x : (s == 1 ? lsa.y : lsb.x)) * sa;
#pragma unroll
  for (int c = 0; c < 4; ++c) bf[c] *= sc;
  const double2 n = __ldg(a.geo + (2 + s) * KP + e);
  double bu[4] = {0.0, 0.0, 0.0, 0.0}, bv[4] = {0.0, 0.0, 0.0, 0.0};
  roe_flux_vjp(up, um, n.x, n.y, bf, bu, bv);
  const long long r0 = static_cast<long long>(2 * w) * KP + e;
  a.bp[r0] = make_double2(bu[0], bu[1]);
  a.bp[r0 + KP] = make_double2(bu[2], bu[3]);
  a.bm[r0] = make_double2(bv[0], bv[1]);
  a.bm[r0 + KP] = make_double2(bv[2], bv[3]);
}

template <int P, int NFQ>
__global__ void __launch_bounds__(kAdjRun * np_of_p(P), 3)
    adjoint_element_kernel(const AdjArgs a, const StageOps<P, NFQ> o) {
  constexpr int NP = np_of_p(P), NE = P + 1;
  __shared__ double2 sA[2 * NP][kAdjRun];  // the block's stage adjoints, row pair j loaded by warp j
  const int e = blockIdx.x * kAdjRun + threadIdx.x;
  const int j = threadIdx.y;  // node, uniform per warp
  const long long KP = a.Kpad;
  // every global operand of this thread is requested before the barrier
  const long long r0 = (2 * j) * KP + e, r1 = r0 + KP;
  double2 u0 = make_double2(1.0, 0.0), u1 = make_double2(0.0, 0.0), j0 = u1, j1 = u1, l0 = u1, l1 = u1, c0 = u1,
          c1 = u1;
  int4 nb4 = make_int4(0, 0, 0, 0);
  if (e < a.K) {
    sA[2 * j][threadIdx.x] = __ldg(a.a + (2 * j) * KP + e);
    sA[2 * j + 1][threadIdx.x] = __ldg(a.a + (2 * j + 1) * KP + e);
    u0 = __ldg(a.U + r0);
    u1 = __ldg(a.U + r1);
    j0 = __ldg(a.geo + 0 * KP + e);
    j1 = __ldg(a.geo + 1 * KP + e);
    nb4 = __ldg(a.nbr + e);
    if (a.lam_coef != 0.0 || a.a_out) {
      l0 = a.lam[r0];
      l1 = a.lam[r1];
    }
    if (a.acc_in) {
      c0 = a.acc_in[r0];
      c1 = a.acc_in[r1];
    }
  }
  __syncthreads();
  if (e >= a.K) return;
  double g[4] = {0.0, 0.0, 0.0, 0.0};
  if (P > 0) {
    double bx[4] = {0.0, 0.0, 0.0, 0.0}, by[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const double d0 = o.D[0][i][j], d1 = o.D[1][i][j];
      const double2 a0 = sA[2 * i][threadIdx.x], a1 = sA[2 * i + 1][threadIdx.x];
      bx[0] = fma(d0, a0.x, bx[0]);
      bx[1] = fma(d0, a0.y, bx[1]);
      bx[2] = fma(d0, a1.x, bx[2]);
      bx[3] = fma(d0, a1.y, bx[3]);
      by[0] = fma(d1, a0.x, by[0]);
      by[1] = fma(d1, a0.y, by[1]);
      by[2] = fma(d1, a1.x, by[2]);
      by[3] = fma(d1, a1.y, by[3]);
    }
    const double sa = (a.elem_dt && a.sa_dt) ? a.sa * __ldg(a.elem_dt + e) : a.sa;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      bx[c] *= sa;
      by[c] *= sa;
    }
    const double sv[4] = {u0.x, u0.y, u1.x, u1.y};
    contravariant_vjp(sv, j0.x, j0.y, j1.x, j1.y, bx, by, g);
  }
  // two-sided faces: own bp (tp) and the neighbour's bm (tm)
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const int nb = s == 0 ? nb4.x : (s == 1 ? nb4.y : nb4.z);
#pragma unroll
    for (int k = 0; k < NE; ++k) {
      if (edge_node(P, s, k) != j) continue;  // uniform per warp
#pragma unroll
      for (int q = 0; q < NFQ; ++q) {
        const long long r0 = static_cast<long long>(2 * (s * NFQ + q)) * KP;
        const double cp = o.tp[s][q][k], cm = o.tm[s][q][k];
        const double2 p0 = __ldg(a.bp + r0 + e), p1 = __ldg(a.bp + r0 + KP + e);
        g[0] = fma(cp, p0.x, g[0]);
        g[1] = fma(cp, p0.y, g[1]);
        g[2] = fma(cp, p1.x, g[2]);
        g[3] = fma(cp, p1.y, g[3]);
        const double2 m0 = __ldg(a.bm + r0 + nb), m1 = __ldg(a.bm + r0 + KP + nb);
        g[0] = fma(cm, m0.x, g[0]);
        g[1] = fma(cm, m0.y, g[1]);
        g[2] = fma(cm, m1.x, g[2]);
        g[3] = fma(cm, m1.y, g[3]);
      }
    }
  }
  const double lam[4] = {l0.x, l0.y, l1.x, l1.y};
  double acc[4] = {c0.x, c0.y, c1.x, c1.y};
#pragma unroll
  for (int c = 0; c < 4; ++c) acc[c] = fma(a.lam_coef, lam[c], acc[c]) + g[c];
  if (a.a_out) {
    const double h = a.elem_dt ? __ldg(a.elem_dt + e) : 1.0;
    const double cl = a.elem_dt ? a.cl * h : a.cl, cg = a.elem_dt ? a.cg * h : a.cg;
    double an[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) an[c] = fma(cl, lam[c], cg * g[c]);
    a.a_out[r0] = make_double2(an[0], an[1]);
    a.a_out[r1] = make_double2(an[2], an[3]);
  }
  a.acc_out[r0] = make_double2(acc[0], acc[1]);
  a.acc_out[r1] = make_double2(acc[2], acc[3]);
}

// dR = R'(U) V for all elements, one thread per element, on dual numbers:
// the right-hand side restated element by element (volume, traces, Roe flux,
// lift) with every quantity carrying its derivative along V.
template <int P, int NFQ>
__global__ void __launch_bounds__(128)
    rhs_jvp_kernel(const double2* __restrict__ U, const double2* __restrict__ V, double2* __restrict__ dR,
                   const double2* __restrict__ geo, const int4* __restrict__ nbr, long long KP, int K,
                   const StageOps<P, NFQ> o) {
  constexpr int NP = np_of_p(P), NE = P + 1;
  using D1 = Dual<1>;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= K) return;
  D1 u[NP][4], r[NP][4];
  for (int i = 0; i < NP; ++i) {
    const double2 x0 = U[(2 * i) * KP + e], x1 = U[(2 * i + 1) * KP + e];
    const double2 v0 = V[(2 * i) * KP + e], v1 = V[(2 * i + 1) * KP + e];
    const double xs[4] = {x0.x, x0.y, x1.x, x1.y}, vs[4] = {v0.x, v0.y, v1.x, v1.y};
    for (int c = 0; c < 4; ++c) {
      u[i][c] = D1(xs[c]);
      u[i][c].d[0] = vs[c];
      r[i][c] = D1(0.0);
    }
  }
  if (P > 0) {
    const double2 j0 = geo[0 * KP + e], j1 = geo[1 * KP + e];
    for (int j = 0; j < NP; ++j) {
      D1 gxi[4], geta[4];
      contravariant_flux_t(u[j], j0.x, j0.y, j1.x, j1.y, gxi, geta);
      for (int i = 0; i < NP; ++i)
        for (int c = 0; c < 4; ++c) r[i][c] = r[i][c] + (o.D[0][i][j] * gxi[c] + o.D[1][i][j] * geta[c]);
    }
  }
  const int4 nb4 = nbr[e];
  const double2 lsa = geo[5 * KP + e], lsb = geo[6 * KP + e];
  for (int s = 0; s < 3; ++s) {
    const int nb = s == 0 ? nb4.x : (s == 1 ? nb4.y : nb4.z);
    const double ls = s == 0 ? lsa.x : (s == 1 ? lsa.y : lsb.x);
    const double2 n = geo[(2 + s) * KP + e];
    D1 un[NE][4];
    for (int k = 0; k < NE; ++k) {
      const int node = edge_node(P, s, k);
      const double2 x0 = U[(2 * node) * KP + nb], x1 = U[(2 * node + 1) * KP + nb];
      const double2 v0 = V[(2 * node) * KP + nb], v1 = V[(2 * node + 1) * KP + nb];
      const double xs[4] = {x0.x, x0.y, x1.x, x1.y}, vs[4] = {v0.x, v0.y, v1.x, v1.y};
      for (int c = 0; c < 4; ++c) {
        un[k][c] = D1(xs[c]);
        un[k][c].d[0] = vs[c];
      }
    }
    for (int q = 0; q < NFQ; ++q) {
      D1 up[4], um[4], f[4];
      for (int k = 0; k < NE; ++k) {
        const int node = edge_node(P, s, k);
        for (int c = 0; c < 4; ++c) {
          up[c] = up[c] + o.tp[s][q][k] * u[node][c];
          um[c] = um[c] + o.tm[s][q][k] * un[k][c];
        }
      }
      roe_flux_t(up, um, n.x, n.y, f);
      for (int i = 0; i < NP; ++i)
        for (int c = 0; c < 4; ++c) r[i][c] = r[i][c] - o.lift[s][i][q] * (ls * f[c]);
    }
  }
  for (int i = 0; i < NP; ++i) {
    dR[(2 * i) * KP + e] = make_double2(r[i][0].d[0], r[i][1].d[0]);
    dR[(2 * i + 1) * KP + e] = make_double2(r[i][2].d[0], r[i][3].d[0]);
  }
}

// out = cx x + cy y + cz z over n double2 entries (null operands are skipped).
__global__ void lincomb_kernel(double2* out, const double2* x, double cx, const double2* y, double cy,
                               const double2* z, double cz, long long n) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double2 r = make_double2(0.0, 0.0);
  if (x) {
    const double2 v = x[i];
    r.x = cx * v.x;
    r.y = cx * v.y;
  }
  if (y) {
    const double2 v = y[i];
    r.x = fma(cy, v.x, r.x);
    r.y = fma(cy, v.y, r.y);
  }
  if (z) {
    const double2 v = z[i];
    r.x = fma(cz, v.x, r.x);
    r.y = fma(cz, v.y, r.y);
  }
  out[i] = r;
}

}  // namespace vt
