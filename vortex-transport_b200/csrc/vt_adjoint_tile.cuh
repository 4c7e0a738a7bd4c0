// One reverse RK stage fused into one kernel on the stage kernel's tiles.
//
// The transpose of the stage right-hand side R at the stage state U applied to
// the stage adjoint a (times sa), g = R'(U)^T (sa a), followed by the reverse
// RK4 combine of adjoint_element_kernel, for meshes on which the face phase
// may take the edge-once form (a face's flux is evaluated once for both
// sides: F(u-, u+, -n) = -F(u+, u-, n)). A persistent block walks the forward
// stage kernel's tiles (64 elements, two runs, vt_schedule.cuh) and keeps every
// intermediate in shared memory, so nothing but the state, the adjoints and
// the geometry crosses HBM:
//
//   1. load   the tile's stage state and stage adjoint by one 2-D TMA tensor
//             copy each per run (issued during the previous tile); the
//             side-0 neighbours' side nodes, the neighbour table and the face
//             list by cp.async during the previous tile;
//   2. lift^T thread (element, component): the lifted face adjoint
//             bF(s, q) = -(len_s/detJ) sa sum_i LIFT_s[i][q] a_i at every face
//             point (the transpose of the lift and of the folded mass inverse);
//   3. faces  one work item per face point of the tile's face list. A face
//             between two tile elements is taken once: the transposed Roe
//             Jacobian at (U+, U-) applied to bF_e(q) - bF_nb(nfq-1-q) gives
//             the adjoints of both traces, each written over its element's bF
//             slot. A face leaving the tile is taken by each side, with the
//             neighbour's bF recomputed from its stage adjoint, and gives the
//             own trace's adjoint only (the neighbour's tile takes the other);
//   4. traces^T  thread (element, component): the trace adjoints onto the
//             side nodes (transposed trace weights) into Np accumulators; then
//             the transposed volume operator sa sum_i D[d][i][j] a_i per node;
//   5. flux^T the transposed nodal flux Jacobian of every node (its state in
//             shared memory), once; the state tile is then free and the next
//             tile's copies are issued;
//   6. combine acc_out = acc_in + lam_coef lam + g, a_out = cl lam + cg g,
//             thread (element, component pair, node half) after the
//             components of g meet in shared memory.
//
// As in the stage kernel, from phase 4 on every shared-memory access stays
// within an element's four threads, so the barriers after phases 4a, 4b and 5
// are per-run named barriers and each run issues its own next copies; the load
// phase has no block barrier (phase 2 reads and writes only the thread's own
// column, phase 3 comes after a barrier), and a tile ends with a
// per-run barrier (the next tile's phase 2 reuses rows that this tile's phase
// 6 reads in other warps of the same run).
//
// Every wait on the mbarrier is bounded; a wait that gives up sets bit 1 of
// err[3] and the block stops taking tiles.
#pragma once

#include "vt_adjoint.cuh"
#include "vt_adjoint_kernels.cuh"
#include "vt_tile.cuh"

namespace vt {

// The stage kernel's shared-memory layout plus the two operator tables the
// face phase indexes at run time (side and face point differ across a warp)
// and the stage adjoint tile, which arrives by tensor copy like the state
// tile (both [2 runs][2 Np rows][32 elements] of double2, 128-byte aligned).
template <int P, int NFQ>
struct AdjTileLayout {
  using Base = TileLayout<P, NFQ>;
  static constexpr int NP = Base::NP;
  static constexpr int NE = Base::NE;
  static constexpr int kTP = align16(Base::kBytes);            // double [3][NFQ][NE] own trace weights
  static constexpr int kLF = align16(kTP + 3 * NFQ * NE * 8);  // double [3][NP][NFQ] LIFT
  static constexpr int kA = (kLF + 3 * NP * NFQ * 8 + 127) / 128 * 128;  // double2 [2][2NP][32] stage adjoint
  static constexpr int kBytes = kA + 2 * 2 * NP * kTileRun * 16;
};

// Lane 0 of warp `which` announces its run's two boxes (stage state and stage
// adjoint) on the tile's mbarrier and issues both tensor copies.
template <int NP>
__device__ __forceinline__ void issue_adj_run_copies(const AdjArgs& a, const int4 run, int which, double2* S,
                                                     double2* A, unsigned long long* bar, int lane) {
  if (lane != 0) return;
  const int start = which ? run.z : run.x, len = which ? run.w : run.y;
  fence_proxy_async_smem();
  mbar_arrive_expect_tx(bar, len > 0 ? 2u * 2u * NP * kTileRun * 16u : 0u);
  if (len > 0) {
    tensor_g2s(S + which * 2 * NP * kTileRun, &a.map_U, 2 * start, 0, bar);
    tensor_g2s(A + which * 2 * NP * kTileRun, &a.map_a, 2 * start, 0, bar);
  }
}

// Two 256-thread blocks per SM: the transposed Roe Jacobian needs about 128
// registers per thread; capped at 80 (three blocks) it spills 416 bytes and the
// reverse stage runs 18% slower. Two blocks leave shared memory for the stage
// adjoint tile (about 96 KB per block at p = 3).
//
// Loads follow the stage kernel: the tile's stage state and stage adjoint
// arrive by one 2-D tensor copy each per run, issued when that run finished
// the previous tile's transposed nodal flux; the next tile's descriptor, face
// list, face count, neighbour table and side-0 neighbour rows go straight to
// shared memory by cp.async, so no register holds them across a tile.
template <int P, int NFQ>
__global__ void __launch_bounds__(4 * kTileElems, 2) adjoint_tile_kernel(const __grid_constant__ AdjArgs a,
                                                                          const StageOps<P, NFQ> ops) {
  using B = TileLayout<P, NFQ>;
  using L = AdjTileLayout<P, NFQ>;
  constexpr int E = B::E;
  constexpr int NP = B::NP;
  constexpr int NE = B::NE;
  constexpr int ES = B::ES;
  constexpr int T = 4 * E;
  extern __shared__ __align__(128) unsigned char smem[];
  double2* S = reinterpret_cast<double2*>(smem + B::kS);  // stage state tile, sidx layout
  double2* H = reinterpret_cast<double2*>(smem + B::kH);
  double* FB = reinterpret_cast<double*>(smem + B::kFB);
  double* TM = reinterpret_cast<double*>(smem + B::kTM);
  int4* NB = reinterpret_cast<int4*>(smem + B::kNB);
  int* EL = reinterpret_cast<int*>(smem + B::kEL);
  int* items = reinterpret_cast<int*>(smem + B::kItems);
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem + B::kBar);
  int* abort_flag = reinterpret_cast<int*>(smem + B::kBar + 8);
  int* NITEMS = reinterpret_cast<int*>(smem + B::kBar + 12);  // the tile's face count
  int4* RUNS = reinterpret_cast<int4*>(smem + B::kRuns);      // tile descriptor, one copy per run
  int4* NEXT = reinterpret_cast<int4*>(smem + B::kNext);      // next tile's descriptor, per run
  double* TP = reinterpret_cast<double*>(smem + L::kTP);
  double* LF = reinterpret_cast<double*>(smem + L::kLF);
  double2* A = reinterpret_cast<double2*>(smem + L::kA);  // stage adjoint tile, sidx layout
  const double* Ad = reinterpret_cast<const double*>(A);

  const int t = threadIdx.x;
  const int col = t % E, grp = t / E;
  const int lane = t & 31;
  const long long KP = a.Kpad;
  const int G = gridDim.x;

  {
    const double* tm = &ops.tm[0][0][0];
    const double* tp = &ops.tp[0][0][0];
    const double* lf = &ops.lift[0][0][0];
    for (int l = t; l < 3 * NFQ * NE; l += T) {
      TM[l] = tm[l];
      TP[l] = tp[l];
    }
    for (int l = t; l < 3 * NP * NFQ; l += T) LF[l] = lf[l];
  }
  if (t == 0) {
    mbar_init(bar, 2);
    *abort_flag = 0;
  }
  __syncthreads();

  // the first tile: descriptor, face count, and by cp.async its face list,
  // neighbour table and side-0 neighbour rows; then its tensor copies
  int tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  if (t == 0) *NITEMS = __ldg(a.tile_count + tile);
  {
    const int4 run = __ldg(a.tiles + tile);
    if (lane == 0 && t < 64) RUNS[t >> 5] = run;
    const int pos = col % kTileRun;
    const bool second = col >= kTileRun;
    const bool valid = pos < (second ? run.w : run.y);
    const int4* nsrc = a.nbr + (second ? run.z : run.x) + pos;
    const int nbx = valid ? __ldg(&nsrc->x) : 0;
    if (grp == 0) {
      if (valid) cp_async16(NB + col, nsrc);
      else NB[col] = make_int4(0, 0, 0, 0);
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int r = grp + 4 * k;
      if (r < 2 * NE) {
        if (valid) cp_async16(H + r * ES + col, a.U + r * KP + nbx);
        else H[r * ES + col] = make_double2(1.0, 0.0);
      }
    }
    if (t < kMaxItems) cp_async4(items + t, a.tile_items + static_cast<long long>(tile) * kMaxItems + t);
    cp_async_commit();
    if (t < 64) issue_adj_run_copies<NP>(a, run, t >> 5, S, A, bar, lane);
  }
  __syncthreads();
  unsigned parity = 0;

  for (; tile < a.ntiles; tile += G) {
    const bool has_next = tile + G < a.ntiles;

    // ---- 1. load ------------------------------------------------------------------
    // the next tile's descriptor, by cp.async into the run's own slot (waited
    // for before the barrier after phase 2, copied into RUNS after the faces)
    if (lane == 0 && t < 64 && has_next) cp_async16(NEXT + (t >> 5), a.tiles + tile + G);
    const int c = grp;  // uniform per warp
    const int el = col;
    int e;
    {
      const int4 run = RUNS[(t >> 5) & 1];
      const int pos = col % kTileRun;
      const bool second = col >= kTileRun;
      e = pos < (second ? run.w : run.y) ? (second ? run.z : run.x) + pos : -1;
      if (grp == 0) EL[col] = e;
    }
    const bool valid = e >= 0;
    {
      bool ok = false;
      for (unsigned n = 0; n < kMaxWaitTries && !ok; ++n) ok = mbar_try_wait(bar, parity);
      if (!ok) {
        atomicOr(&a.err[3], 2ull);
        *abort_flag = 1;
      }
    }
    parity ^= 1u;

    // ---- 2. lifted face adjoints bF[s][c][q][el], thread (element el, component c) ----
    const double sa = valid && a.elem_dt && a.sa_dt ? a.sa * __ldg(a.elem_dt + e) : a.sa;
    {
      double lam[NP];
      double2 lsa = make_double2(0.0, 0.0), lsb = lsa;
#pragma unroll
      for (int i = 0; i < NP; ++i) lam[i] = valid ? Ad[sidx<NP>(2 * i + (c >> 1), el) * 2 + (c & 1)] : 0.0;
      if (valid) {
        lsa = __ldg(a.geo + 5 * KP + e);
        lsb = __ldg(a.geo + 6 * KP + e);
      }
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const double sc = -(s == 0 ? lsa.x : (s == 1 ? lsa.y : lsb.x)) * sa;
#pragma unroll
        for (int q = 0; q < NFQ; ++q) {
          double v = 0.0;
#pragma unroll
          for (int i = 0; i < NP; ++i) v = fma(ops.lift[s][i][q], lam[i], v);
          FB[((s * 4 + c) * NFQ + q) * ES + el] = sc * v;
        }
      }
    }
    cp_async_wait_all();  // this thread's cp.async copies of the tile's face list and neighbour rows
    __syncthreads();
    if (*abort_flag) break;

    // ---- 3. faces: transposed Roe Jacobian; the trace adjoints overwrite bF ----------
    const int nitems = *NITEMS;
    for (int w = t; w < nitems * NFQ; w += T) {
      const int it = items[w / NFQ];
      const int q = w % NFQ;
      const int fl = it & 0xff, s = (it >> 8) & 3;
      const bool mirror = (it >> 10) & 1;
      const int nl = (it >> 11) & 0xff;
      const int qm = NFQ - 1 - q;
      const int fe = EL[fl];
      const double2 n = __ldg(a.geo + (2 + s) * KP + fe);
      double up[4] = {0.0, 0.0, 0.0, 0.0}, um[4] = {0.0, 0.0, 0.0, 0.0}, bn[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int k = 0; k < NE; ++k) {
        const int node = s == 0 ? edge_node(P, 0, k) : (s == 1 ? edge_node(P, 1, k) : edge_node(P, 2, k));
        const double cp = TP[(s * NFQ + q) * NE + k];
        const double2 x0 = S[sidx<NP>(2 * node, fl)], x1 = S[sidx<NP>(2 * node + 1, fl)];
        up[0] = fma(cp, x0.x, up[0]);
        up[1] = fma(cp, x0.y, up[1]);
        up[2] = fma(cp, x1.x, up[2]);
        up[3] = fma(cp, x1.y, up[3]);
      }
      if (mirror) {
        // the partner's own trace at its point nfq-1-q, as the stage kernel reads it
#pragma unroll
        for (int k = 0; k < NE; ++k) {
          const int node = s == 0 ? edge_node(P, 0, k) : (s == 1 ? edge_node(P, 1, k) : edge_node(P, 2, k));
          const double cm = TP[(s * NFQ + qm) * NE + k];
          const double2 y0 = S[sidx<NP>(2 * node, nl)], y1 = S[sidx<NP>(2 * node + 1, nl)];
          um[0] = fma(cm, y0.x, um[0]);
          um[1] = fma(cm, y0.y, um[1]);
          um[2] = fma(cm, y1.x, um[2]);
          um[3] = fma(cm, y1.y, um[3]);
        }
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) bn[cc] = FB[((s * 4 + cc) * NFQ + qm) * ES + nl];
      } else {
        const int4 nb4 = NB[fl];
        const int nb = s == 0 ? nb4.x : (s == 1 ? nb4.y : nb4.z);
#pragma unroll
        for (int k = 0; k < NE; ++k) {
          const int node = s == 0 ? edge_node(P, 0, k) : (s == 1 ? edge_node(P, 1, k) : edge_node(P, 2, k));
          const double cm = TM[(s * NFQ + q) * NE + k];
          double2 y0, y1;
          if (s == 0) {
            y0 = H[(2 * k) * ES + fl];
            y1 = H[(2 * k + 1) * ES + fl];
          } else {
            y0 = __ldg(a.U + (2 * node) * KP + nb);
            y1 = __ldg(a.U + (2 * node + 1) * KP + nb);
          }
          um[0] = fma(cm, y0.x, um[0]);
          um[1] = fma(cm, y0.y, um[1]);
          um[2] = fma(cm, y1.x, um[2]);
          um[3] = fma(cm, y1.y, um[3]);
        }
        // the neighbour's lifted adjoint at its point nfq-1-q, formed as its own tile forms it
        const double san = a.elem_dt && a.sa_dt ? a.sa * __ldg(a.elem_dt + nb) : a.sa;
        const double* gn = reinterpret_cast<const double*>(a.geo + (s < 2 ? 5 : 6) * KP + nb);
        const double sc = -__ldg(gn + (s == 1 ? 1 : 0)) * san;
        double v[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          const double l = LF[(s * NP + i) * NFQ + qm];
          const double2 a0 = __ldg(a.a + (2 * i) * KP + nb), a1 = __ldg(a.a + (2 * i + 1) * KP + nb);
          v[0] = fma(l, a0.x, v[0]);
          v[1] = fma(l, a0.y, v[1]);
          v[2] = fma(l, a1.x, v[2]);
          v[3] = fma(l, a1.y, v[3]);
        }
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) bn[cc] = sc * v[cc];
      }
      double bf[4], bu[4] = {0.0, 0.0, 0.0, 0.0}, bv[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) bf[cc] = FB[((s * 4 + cc) * NFQ + q) * ES + fl] - bn[cc];
      roe_flux_vjp(up, um, n.x, n.y, bf, bu, bv);
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) FB[((s * 4 + cc) * NFQ + q) * ES + fl] = bu[cc];
      if (mirror) {
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) FB[((s * 4 + cc) * NFQ + qm) * ES + nl] = bv[cc];
      }
    }
    __syncthreads();

    // next tile's metadata: the face list and count of this tile are no longer
    // read, so the next tile's go to shared memory now, and the next
    // descriptor into RUNS (read again after this run's next barrier)
    if (lane == 0 && t < 64) RUNS[t >> 5] = has_next ? NEXT[t >> 5] : make_int4(0, 0, 0, 0);
    if (has_next) {
      if (t < kMaxItems) cp_async4(items + t, a.tile_items + static_cast<long long>(tile + G) * kMaxItems + t);
      if (t == kMaxItems) cp_async4(NITEMS, a.tile_count + tile + G);
    }

    // ---- 4a. trace adjoints onto the side nodes, component c --------------------------
    double g[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) g[i] = 0.0;
#pragma unroll
    for (int s = 0; s < 3; ++s)
#pragma unroll
      for (int q = 0; q < NFQ; ++q) {
        const double b = FB[((s * 4 + c) * NFQ + q) * ES + el];
#pragma unroll
        for (int k = 0; k < NE; ++k) g[edge_node(P, s, k)] = fma(ops.tp[s][q][k], b, g[edge_node(P, s, k)]);
      }
    run_sync(t);

    // the next tile's neighbour table, now that the run's barrier has made its
    // descriptor visible; it lands during phases 4b and 5
    if (has_next && grp == 0) {
      const int4 nr = RUNS[col >= kTileRun];
      const int pos = col % kTileRun;
      if (pos < (col >= kTileRun ? nr.w : nr.y)) cp_async16(NB + col, a.nbr + (col >= kTileRun ? nr.z : nr.x) + pos);
      else NB[col] = make_int4(0, 0, 0, 0);
    }

    // ---- 4b. transposed volume operator: rows j*8 + c (xi), j*8 + 4 + c (eta) ---------
    double* Gs = FB;
    if (P > 0) {
      double lam[NP];
#pragma unroll
      for (int i = 0; i < NP; ++i) lam[i] = valid ? Ad[sidx<NP>(2 * i + (c >> 1), el) * 2 + (c & 1)] : 0.0;
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        double bx = 0.0, by = 0.0;
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          bx = fma(ops.D[0][i][j], lam[i], bx);
          by = fma(ops.D[1][i][j], lam[i], by);
        }
        Gs[(j * 8 + c) * ES + el] = bx * sa;
        Gs[(j * 8 + 4 + c) * ES + el] = by * sa;
      }
    }
    run_sync(t);

    // ---- 5. transposed nodal flux Jacobian of every node, in place over the xi rows ----
    if (P > 0) {
      const int eg = valid ? e : 0;
      const double2 j0 = __ldg(a.geo + 0 * KP + eg);
      const double2 j1 = __ldg(a.geo + 1 * KP + eg);
      for (int j = c; j < NP; j += 4) {
        const double2 s0 = S[sidx<NP>(2 * j, el)], s1 = S[sidx<NP>(2 * j + 1, el)];
        const double sv[4] = {s0.x, s0.y, s1.x, s1.y};
        double bx[4], by[4], gv[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          bx[cc] = Gs[(j * 8 + cc) * ES + el];
          by[cc] = Gs[(j * 8 + 4 + cc) * ES + el];
        }
        contravariant_vjp(sv, j0.x, j0.y, j1.x, j1.y, bx, by, gv);
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) Gs[(j * 8 + cc) * ES + el] = gv[cc];
      }
    }
    // the neighbour table has landed; the barrier shows it to the column's other threads
    if (grp == 0) cp_async_wait_all();
    run_sync(t);

    // this run's columns of the state and adjoint tiles are free: start its
    // next copies and the next tile's side-0 neighbour rows
    if (has_next) {
      if (t < 64) issue_adj_run_copies<NP>(a, RUNS[t >> 5], t >> 5, S, A, bar, lane);
      const int4 nr = RUNS[col >= kTileRun];
      const bool nvalid = col % kTileRun < (col >= kTileRun ? nr.w : nr.y);
      const int nbx = NB[col].x;
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int rr = grp + 4 * k;
        if (rr < 2 * NE) {
          if (nvalid) cp_async16(H + rr * ES + col, a.U + rr * KP + nbx);
          else H[rr * ES + col] = make_double2(1.0, 0.0);
        }
      }
    }
    cp_async_commit();

    // ---- 6. reverse RK combine -------------------------------------------------------------
    // the thread's component adjoints meet their pair partner's in shared memory
    // (rows i*8 + c of the flux^T buffer, own column), then thread (el, h, half)
    // combines component pair h of half of the nodes with 16-byte accesses, as
    // the stage kernel's pair mapping does: half the load and store
    // instructions of a per-component combine, on whole 16-byte pairs
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const double gi = P > 0 ? g[i] + Gs[(i * 8 + c) * ES + el] : g[i];
      Gs[(i * 8 + c) * ES + el] = gi;
    }
    run_sync(t);
    if (valid) {
      constexpr int NH = (NP + 1) / 2;
      const int h = grp & 1, half = grp >> 1;
      const double hh = a.elem_dt ? __ldg(a.elem_dt + e) : 1.0;
      const double cl = a.elem_dt ? a.cl * hh : a.cl, cg = a.elem_dt ? a.cg * hh : a.cg;
      const bool need_lam = a.lam_coef != 0.0 || a.a_out;
      // every load before the first store: acc_in and acc_out are the same
      // array in three of the four reverse stages, so loads that follow a
      // store could not be moved above it and each would wait on its own
      // round trip to L2
      double2 lv[NH], av[NH];
#pragma unroll
      for (int k = 0; k < NH; ++k) {
        const int i = half * NH + k;
        if (i < NP) {
          const long long x = (2 * i + h) * KP + e;
          lv[k] = need_lam ? a.lam[x] : make_double2(0.0, 0.0);
          av[k] = a.acc_in ? a.acc_in[x] : make_double2(0.0, 0.0);
        }
      }
#pragma unroll
      for (int k = 0; k < NH; ++k) {
        const int i = half * NH + k;
        if (i < NP) {
          const long long x = (2 * i + h) * KP + e;
          const double2 gi = make_double2(Gs[(i * 8 + 2 * h) * ES + el], Gs[(i * 8 + 2 * h + 1) * ES + el]);
          a.acc_out[x] = make_double2(fma(a.lam_coef, lv[k].x, av[k].x) + gi.x, fma(a.lam_coef, lv[k].y, av[k].y) + gi.y);
          if (a.a_out) a.a_out[x] = make_double2(fma(cl, lv[k].x, cg * gi.x), fma(cl, lv[k].y, cg * gi.y));
        }
      }
    }
    // the four warps of a run hold different components of the same elements:
    // none may start the next tile's phase 2 (which reuses rows of the face /
    // flux buffer) before the others are done with this tile's
    run_sync(t);
  }

  cp_async_wait_all();  // none may land after the block has left
  if (*abort_flag) {
    // the bulk copies of a tile whose wait gave up may still land: wait for
    // them once more, with the same bound, before the block leaves
    for (unsigned n = 0; n < kMaxWaitTries; ++n)
      if (mbar_try_wait(bar, parity ^ 1u)) break;
  }
}

}  // namespace vt
