// The fused RK stage kernel, tiled through shared memory.
//
// A persistent block walks tiles of 64 elements (two runs of 32 consecutive
// elements, see StageArgs) and advances each through one stage of the nodal
// DG scheme (Evolve.cpp:135-308, numerical_flux Numericalflux.cpp:13-157,
// stage update Timestepping.cpp:85-306 / :39-82). The state crosses HBM once
// per stage:
//
//   1. load   the tile's state arrives in shared memory by one 2-D TMA tensor
//             copy per run (cp.async.bulk.tensor: 2 Np rows x 32 elements,
//             completion on an mbarrier), issued when that run finished the
//             previous tile's flux phase; the side-0 neighbours' side nodes,
//             the neighbour table and the tile's face list were copied into
//             shared memory during the previous tile as well, by cp.async
//             (global to shared without registers), once the previous tile's
//             faces no longer needed those buffers;
//   2. traces 4 threads per element, one conserved component each, evaluate
//             the element's own trace at every face point from the p+1 side
//             nodes (coefficients are immediates);
//   3. faces  one work item per (face, Gauss point) from the list built once
//             at set-up (vt_schedule.cuh), sorted so warps stay on one path.
//             A face between two tile elements is evaluated once, by the
//             element with the smaller index: its outer state is the partner's
//             own trace at the mirrored point nfq-1-q, and the flux is written
//             over both traces (the partner gets -F, its outward normal being
//             -n). A face leaving the tile is evaluated by each side, as in
//             the reference, with the outer trace from the neighbour's nodes;
//   4. lift   4 threads per element, one conserved component each: surface
//             term -(len_s/detJ) LIFT_s F_s into Np accumulators;
//   5. flux   the nodal Euler flux of every node, contracted with the inverse
//             Jacobian, once, into shared memory; the state tile is then free
//             and the next tile's copies are issued;
//   6. volume D_xi G_xi + D_eta G_eta, then the RK stage update written back.
//
// From phase 4 on, every shared-memory access stays within an element's four
// threads, which lie in the four warps of equal parity (warps 0, 2, 4, 6 hold
// the first run's elements, 1, 3, 5, 7 the second's). So the barriers after
// phases 4 and 5 are per-run 128-thread named barriers, and each run issues its
// own next copies (the tile's mbarrier expects one arrival per run). The load
// phase has no block barrier either: the traces read only the thread's own
// column of the state tile, which its own wait on the mbarrier covers, and the
// face list, neighbour rows and element indices written there are first read
// in phase 3, after the barrier that follows the traces. A tile ends with a
// per-run barrier: the four warps of a run hold different components of the
// same elements, and the next tile's traces reuse rows of the buffer that this
// tile's volume phase reads. So the two halves of a block run apart from phase
// 4 of one tile to the end of the next tile's trace phase.
//
// Registers are the kernel's scarcest resource (80 per thread for three blocks
// per SM), so nothing about the next tile is held in registers across a tile:
// its neighbour rows, neighbour table and face list go straight to shared
// memory by cp.async, and the tile descriptor (the two runs) is kept in shared
// memory, one copy per run, written after the face phase by the run's first
// warp and read behind the run's own barriers. Holding them in registers cost
// 176 bytes of spill stores per thread, whose reloads missed the small L1 that
// three 73 KB blocks leave; staged this way 16 bytes remain and a step at
// 768 x 768, p = 3 is 12% faster, with bit-identical results.
//
// The tile's RK operand rows are prefetched into L2 by tensor prefetches (one
// per run and vector) when the tile starts, and its geometry rows into L1. One
// tensor instruction per run replaced 2 Np per-row bulk copies and prefetches
// (4% faster at 768 x 768, p = 3): the TMA unit's instruction issue, not its
// bandwidth, was what the per-row form paid for.
// The reference's mass-inverse apply is folded into D and LIFT on the host.
// The face and flux buffers' rows are padded by one element so that rows that
// differ by a multiple of 128 bytes do not fall into the same banks (the face
// phase reads several rows and columns per warp instruction); the state tile
// is dense per run, as the tensor copies write it (each warp instruction reads
// 32 consecutive elements of one row).
//
// Every wait on the mbarrier is bounded; a wait that gives up sets bit 1 of
// err[3], and the block stops taking tiles. StageArgs::wait_tries and
// test_flags (vt_test_bulk_wait) let a test shorten the bound and issue no
// copies, so that the give-up path runs without any copy in flight.
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
  static constexpr int kS = 0;  // double2 [2NP][ES]; the stage kernel's tensor copies use it as [2][2NP][32]
  static constexpr int kH = align16(kS + 2 * NP * ES * 16);      // double2 [2NE][ES]
  static constexpr int kFB = align16(kH + 2 * NE * ES * 16);     // double [3][4][NFQ][ES] | [NP][8][ES]
  static constexpr int kTM = align16(kFB + kFBDoubles * 8);      // double [3][NFQ][NE]
  static constexpr int kNB = align16(kTM + 3 * NFQ * NE * 8);    // int4 [E]
  static constexpr int kEL = align16(kNB + E * 16);              // int [E] global element index
  static constexpr int kItems = align16(kEL + E * 4);            // int [kMaxItems]
  static constexpr int kBar = align16(kItems + kMaxItems * 4);   // mbarrier (8 B), abort flag, face count
  static constexpr int kRuns = kBar + 16;                        // int4 [2] tile descriptor, one copy per run
  static constexpr int kNext = kRuns + 32;                       // int4 [2] next tile's descriptor, per run
  static constexpr int kBytes = align16(kNext + 32);
};

// ---- TMA unit ------------------------------------------------------------------
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// true once the phase with parity `parity` has completed.
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Global-to-shared copies that bypass the registers (cp.async, completed per
// thread by cp.async.wait_all): 16 bytes (both addresses 16-byte aligned,
// cached in L2 only) or 4 bytes.
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(__cvta_generic_to_global(src))
               : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(__cvta_generic_to_global(src))
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

constexpr unsigned kMaxWaitTries = 1u << 22;

// Shared-memory index of (row, element column) of the state tile: each run's
// tensor box lands dense, [2 Np rows][32 elements] per run.
template <int NP>
__device__ __forceinline__ int sidx(int row, int el) {
  return ((el >> 5) * 2 * NP + row) * kTileRun + (el & (kTileRun - 1));
}

__device__ __forceinline__ void tensor_g2s(void* dst, const CUtensorMap* map, int x, int y, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_addr(dst)), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tensor_prefetch_l2(const CUtensorMap* map, int x, int y) {
  asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];"
               ::"l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y) : "memory");
}

// Lane 0 of warp `which` announces the run's box and issues its one tensor copy.
template <int NP>
__device__ __forceinline__ void issue_run_tensor_copy(const CUtensorMap* map, const int4 run, int which,
                                                      double2* S, unsigned long long* bar, int lane, int test_flags) {
  if (test_flags & kTestNoCopies) return;  // test hook: nothing arrives, every wait gives up
  if (lane != 0) return;
  const int start = which ? run.z : run.x, len = which ? run.w : run.y;
  fence_proxy_async_smem();
  mbar_arrive_expect_tx(bar, len > 0 ? 2u * NP * kTileRun * 16u : 0u);
  if (len > 0) tensor_g2s(S + which * 2 * NP * kTileRun, map, 2 * start, 0, bar);
}

// Barrier of the four warps that hold one run's elements (warps of equal parity).
__device__ __forceinline__ void run_sync(int t) {
  if ((t >> 5) & 1) asm volatile("bar.sync 2, 128;" ::: "memory");
  else asm volatile("bar.sync 1, 128;" ::: "memory");
}

// ---- warp mappings -------------------------------------------------------------------
// Thread t of a block holds element column el = t % 64 and group g = t / 64
// (uniform per warp; warps of equal parity hold one run). Two mappings of the
// work onto (el, g), chosen per order p (StageKernel, vt_launch.cu):
//   component (kMapComponent): g is the conserved component c; the thread
//     forms every face point's trace and every node's update of component c;
//   pair (kMapPair): g = (half, h) with h the component pair of the HBM
//     layout ((rho, rho u) or (rho v, rho E)); the thread forms both
//     components of pair h for half of the face points (traces) and half of
//     the nodes (lift, volume, update): [0, QH) / [0, NH) or the rest, with
//     QH = ceil(nfq / 2), NH = ceil(Np / 2). Shared- and global-memory
//     accesses are then 16 bytes wide (half the load/store instructions) for
//     the same floating-point work.
// The face buffer holds the same bytes either way: [s][c][q][el] doubles for
// the component mapping, [s][q][h][el] double2 for the pair mapping (and the
// nodal flux [j][8][el] doubles or [j][4][el] double2).
template <int P, int NFQ, int HALF>
__device__ __forceinline__ void pair_traces(const StageOps<P, NFQ>& ops, const double2* S, double2* FB2, int h,
                                            int el) {
  constexpr int NP = np_of_p(P), NE = P + 1, ES = kTileElems + 1, QH = (NFQ + 1) / 2;
  constexpr int q0 = HALF * QH, q1 = (HALF + 1) * QH < NFQ ? (HALF + 1) * QH : NFQ;
  double2 u[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) u[i] = S[sidx<NP>(2 * i + h, el)];
#pragma unroll
  for (int s = 0; s < 3; ++s)
#pragma unroll
    for (int q = q0; q < q1; ++q) {
      double vx = 0.0, vy = 0.0;
#pragma unroll
      for (int k = 0; k < NE; ++k) {
        vx = fma(ops.tp[s][q][k], u[edge_node(P, s, k)].x, vx);
        vy = fma(ops.tp[s][q][k], u[edge_node(P, s, k)].y, vy);
      }
      FB2[((s * NFQ + q) * 2 + h) * ES + el] = make_double2(vx, vy);
    }
}

template <int P, int NFQ, int HALF>
__device__ __forceinline__ void pair_lift(const StageOps<P, NFQ>& ops, const double2* FB2, int h, int el,
                                          double2 lsa, double2 lsb, double2* r) {
  constexpr int NP = np_of_p(P), ES = kTileElems + 1, NH = (NP + 1) / 2, base = HALF * NH;
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const double ls = s == 0 ? lsa.x : (s == 1 ? lsa.y : lsb.x);
#pragma unroll
    for (int q = 0; q < NFQ; ++q) {
      const double2 f = FB2[((s * NFQ + q) * 2 + h) * ES + el];
      const double fx = ls * f.x, fy = ls * f.y;
#pragma unroll
      for (int i = 0; i < NH; ++i)
        if (base + i < NP) {
          r[i].x = fma(-ops.lift[s][base + i][q], fx, r[i].x);
          r[i].y = fma(-ops.lift[s][base + i][q], fy, r[i].y);
        }
    }
  }
}

template <int P, int NFQ, int HALF>
__device__ __forceinline__ void pair_volume(const StageOps<P, NFQ>& ops, const double2* G2, int h, int el,
                                            double2* r) {
  constexpr int NP = np_of_p(P), ES = kTileElems + 1, NH = (NP + 1) / 2, base = HALF * NH;
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const double2 gx = G2[(j * 4 + h) * ES + el];
    const double2 gy = G2[(j * 4 + 2 + h) * ES + el];
#pragma unroll
    for (int i = 0; i < NH; ++i)
      if (base + i < NP) {
        r[i].x = fma(ops.D[0][base + i][j], gx.x, fma(ops.D[1][base + i][j], gy.x, r[i].x));
        r[i].y = fma(ops.D[0][base + i][j], gx.y, fma(ops.D[1][base + i][j], gy.y, r[i].y));
      }
  }
}

// Stage 3's U3 / (3 c_out) (f = 1 / (3 c_out)) added to pair h of this half's
// node accumulators, from the state tile.
template <int P, int HALF>
__device__ __forceinline__ void pair_fold(const double2* S, int h, int el, double f, double2* r) {
  constexpr int NP = np_of_p(P), NH = (NP + 1) / 2, base = HALF * NH;
#pragma unroll
  for (int i = 0; i < NH; ++i)
    if (base + i < NP) r[i] = make_double2(fma(f, S[sidx<NP>(2 * (base + i) + h, el)].x, r[i].x),
                                           fma(f, S[sidx<NP>(2 * (base + i) + h, el)].y, r[i].y));
}

// Non-coherent loads issued where they are written, so that the stage
// update's first operand is in flight during the volume phase (the compiler
// would otherwise sink them to their use), and so that stage 1's re-read of
// its input stays in the update (plain loads were hoisted and spilled). They
// do not allocate in L1: three
// 73 KB blocks leave about 30 KB of it, which the tile's geometry rows and the
// face phase's neighbour rows use, and each operand row is read once (0.2%
// faster at 768 x 768, p = 3).
__device__ __forceinline__ double ld_early(const double* p) {
  double v;
  asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double2 ld_early2(const double2* p) {
  double2 v;
  asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}

// The RK4 step in 12 state-vector passes. Classical RK4 (Timestepping.cpp:85-306)
// with k_i the right-hand side at stage i's input has the stage states
// U1 = U + dt/2 k1, U2 = U + dt/2 k2, U3 = U + dt k3, and since
// dt/6 k1 = (U1 - U)/3 and dt/3 k3 = (U3 - U)/3 its new state is
// X + U3/3 + dt/6 k4 with X = (U + U1)/3 + dt/3 k2:
//   stage 0: reads U,              writes U1
//   stage 1: reads U1, U (and U1 again from L2), writes U2 and X
//   stage 2: reads U2, U,          writes U3
//   stage 3: reads U3, X,          writes U_{n+1}
// against 16 passes when the accumulator is carried through every stage. The
// stage states are formed as before, bit for bit; only the last stage's sum is
// grouped differently (rounding level). Stage 3 adds U3/3 by starting its
// accumulators at U3/(3 c_out) while the state tile is still in shared memory.
// The coefficient ratios are classical RK4's: (dt/6)/(dt/2) = (dt/3)/dt = 1/3.
constexpr double kThird = 1.0 / 3.0;

// The stage's read-only operand that the update needs besides the
// accumulator: U_n (stage 0, forward Euler), X (stage 3) or the base U_n
// (stages 1, 2); none for the bare right-hand side.
__device__ __forceinline__ const double2* first_operand(const StageArgs& a) {
  return (a.stage == 0 || a.stage == kStageEuler) ? a.in : (a.stage == 3 ? a.acc : a.base);
}

__device__ __forceinline__ double2 fma2(double c, double2 r, double2 u) {
  return make_double2(fma(c, r.x, u.x), fma(c, r.y, u.y));
}

// Stage update of pair h of this half's nodes; pre holds first_operand's values.
// The stage's outputs are written with streaming stores (st.global.cs, evict
// first): where the stage is memory-bound its vectors exceed L2, and evicting
// them first keeps the rows that tiles in flight still read there (neighbour
// rows, prefetched operand rows); 0.3% faster at 768 x 768, p = 3.
template <int P, int HALF>
__device__ __forceinline__ void pair_update(const StageArgs& a, int e, int h, double c_acc, double c_out,
                                            const double2* r, const double2* pre) {
  constexpr int NP = np_of_p(P), NH = (NP + 1) / 2;
  const long long KP = a.Kpad;
  const long long o = (2 * HALF * NH + h) * KP + e;  // row 2 * node + h of this half's first node
  constexpr int N = NP - HALF * NH < NH ? NP - HALF * NH : NH;  // nodes of this half
  switch (a.stage) {
    case 1: {
      if (!a.no_acc) {
        // X = (U_n + U1) / 3 + c_acc k2, U1 being this stage's input, re-read
        // here (its tile was copied one tile ago and is still in L2) by loads
        // that stay where they are written (plain loads of the read-only
        // input were hoisted and spilled); every row is read before the first
        // store, since a load that follows a store to another array cannot be
        // moved above it
        double2 iv[NH];
#pragma unroll
        for (int i = 0; i < N; ++i) iv[i] = ld_early2(a.in + o + i * 2 * KP);
#pragma unroll
        for (int i = 0; i < N; ++i)
          __stcs(a.acc + (o + i * 2 * KP),
                 fma2(c_acc, r[i], make_double2((pre[i].x + iv[i].x) * kThird, (pre[i].y + iv[i].y) * kThird)));
      }
#pragma unroll
      for (int i = 0; i < N; ++i) __stcs(a.out + (o + i * 2 * KP), fma2(c_out, r[i], pre[i]));
      break;
    }
    case 0:
    case 2:
    case 3:
    case kStageEuler:
#pragma unroll
      for (int i = 0; i < N; ++i) __stcs(a.out + (o + i * 2 * KP), fma2(c_out, r[i], pre[i]));
      break;
    default:
#pragma unroll
      for (int i = 0; i < N; ++i) __stcs(a.out + (o + i * 2 * KP), r[i]);
      break;
  }
}

template <int P, int NFQ, int MAP>
// Three 256-thread blocks per SM (<= 80 registers per thread) keep 24 warps
// resident alongside 3 x ~75 KB of shared memory.
__global__ void __launch_bounds__(4 * kTileElems, 3) tile_stage_kernel(const __grid_constant__ StageArgs a,
                                                                        const StageOps<P, NFQ> ops) {
  using L = TileLayout<P, NFQ>;
  constexpr int E = L::E;
  constexpr int NP = L::NP;
  constexpr int NE = L::NE;
  constexpr int ES = L::ES;
  constexpr int T = 4 * E;
  constexpr bool PAIR = MAP == kMapPair;
  extern __shared__ __align__(128) unsigned char smem[];
  double2* S = reinterpret_cast<double2*>(smem + L::kS);
  double2* H = reinterpret_cast<double2*>(smem + L::kH);
  double* FB = reinterpret_cast<double*>(smem + L::kFB);
  double2* FB2 = reinterpret_cast<double2*>(smem + L::kFB);
  double* TM = reinterpret_cast<double*>(smem + L::kTM);
  int4* NB = reinterpret_cast<int4*>(smem + L::kNB);
  int* EL = reinterpret_cast<int*>(smem + L::kEL);
  int* items = reinterpret_cast<int*>(smem + L::kItems);
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem + L::kBar);
  int* abort_flag = reinterpret_cast<int*>(smem + L::kBar + 8);
  int* NITEMS = reinterpret_cast<int*>(smem + L::kBar + 12);  // the tile's face count
  int4* RUNS = reinterpret_cast<int4*>(smem + L::kRuns);
  int4* NEXT = reinterpret_cast<int4*>(smem + L::kNext);

  const int t = threadIdx.x;
  const int col = t % E, grp = t / E;  // load mapping; also (element, group) later
  const int lane = t & 31;
  const long long KP = a.Kpad;
  const int G = gridDim.x;
  const unsigned max_tries = a.wait_tries ? a.wait_tries : kMaxWaitTries;

  {
    const double* tm = &ops.tm[0][0][0];
    for (int l = t; l < 3 * NFQ * NE; l += T) TM[l] = tm[l];
  }
  if (t == 0) {
    mbar_init(bar, 2);
    *abort_flag = 0;
  }
  __syncthreads();

  // the first tile: its descriptor (one copy per run), face count, and by
  // cp.async its face list, neighbour table and side-0 neighbour rows; then
  // its state copies
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
        if (valid) cp_async16(H + r * ES + col, a.in + r * KP + nbx);
        else H[r * ES + col] = make_double2(1.0, 0.0);
      }
    }
    if (t < kMaxItems) cp_async4(items + t, a.tile_items + static_cast<long long>(tile) * kMaxItems + t);
    cp_async_commit();
    if (t < 64) issue_run_tensor_copy<NP>(&a.map_in, run, t >> 5, S, bar, lane, a.test_flags);
  }
  __syncthreads();
  unsigned parity = 0;

  for (; tile < a.ntiles; tile += G) {
    const bool has_next = tile + G < a.ntiles;
    const int4 run = RUNS[(t >> 5) & 1];

    // ---- prefetch: this tile's RK operand rows into L2 (read in phase 6) and its
    // geometry rows into L1. The next tile's state is not prefetched: its bulk
    // copies, issued in phase 5, read it from HBM themselves (prefetching it
    // as well was 1.6% slower) -------------------------------------------------
    if (t >= 64 && t < 68) {
      const int which = t & 1, vec = (t - 64) >> 1;  // vec 0: acc, 1: base
      const int start = which ? run.z : run.x, len = which ? run.w : run.y;
      if (len > 0) {
        if (vec == 0 && a.stage == 3) tensor_prefetch_l2(&a.map_acc, 2 * start, 0);
        if (vec == 1 && (a.stage == 1 || a.stage == 2)) tensor_prefetch_l2(&a.map_base, 2 * start, 0);
      }
    } else if (t >= 64 + 8 * NP && t < 64 + 8 * NP + 56) {
      // this tile's 7 geometry rows into L1 (4 lines per 32-element run)
      const int l = t - 64 - 8 * NP, row = l >> 3, which = (l >> 2) & 1, line = l & 3;
      const int start = which ? run.z : run.x, len = which ? run.w : run.y;
      if (line * 8 < len) prefetch_l1(a.geo + row * KP + start + line * 8);
    }

    // ---- 1. load ------------------------------------------------------------------
    // the next tile's descriptor, by cp.async into the run's own slot (lane 0
    // of warp 0 or 1 issues, waits before the barrier after the traces and
    // copies it into RUNS after the faces), so no register holds it across the
    // trace and face phases
    if (lane == 0 && t < 64 && has_next) cp_async16(NEXT + (t >> 5), a.tiles + tile + G);
    {
      const int pos = col % kTileRun;
      const bool second = col >= kTileRun;
      const bool valid = pos < (second ? run.w : run.y);
      if (grp == 0) EL[col] = valid ? (second ? run.z : run.x) + pos : -1;
    }
    {
      bool ok = false;
      for (unsigned n = 0; n < max_tries && !ok; ++n) ok = mbar_try_wait(bar, parity);
      if (!ok) {
        atomicOr(&a.err[3], 2ull);
        *abort_flag = 1;
      }
    }
    parity ^= 1u;

    // ---- 2. own traces at every face point -------------------------------------------
    if constexpr (PAIR) {
      if (grp >> 1) pair_traces<P, NFQ, 1>(ops, S, FB2, grp & 1, col);
      else pair_traces<P, NFQ, 0>(ops, S, FB2, grp & 1, col);
    } else {
      const int cc = grp, el = col;
      const double* Sd = reinterpret_cast<const double*>(S);
      double u[NP];
#pragma unroll
      for (int i = 0; i < NP; ++i) u[i] = Sd[sidx<NP>(2 * i + (cc >> 1), el) * 2 + (cc & 1)];
#pragma unroll
      for (int s = 0; s < 3; ++s)
#pragma unroll
        for (int q = 0; q < NFQ; ++q) {
          double v = 0.0;
#pragma unroll
          for (int k = 0; k < NE; ++k) v = fma(ops.tp[s][q][k], u[edge_node(P, s, k)], v);
          FB[((s * 4 + cc) * NFQ + q) * ES + el] = v;
        }
    }
    cp_async_wait_all();  // this thread's cp.async copies of the tile's face list and neighbour rows
    __syncthreads();
    if (*abort_flag) break;

    // ---- 3. faces: the flux overwrites the traces it consumed ----------------------------
    const int nitems = *NITEMS;
    for (int w = t; w < nitems * NFQ; w += T) {
      const int it = items[w / NFQ];
      const int q = w % NFQ;
      const int el = it & 0xff, s = (it >> 8) & 3;
      const bool mirror = (it >> 10) & 1;
      const int nl = (it >> 11) & 0xff;
      const int qm = NFQ - 1 - q;
      const int e = EL[el];
      const double2 n = __ldg(a.geo + (2 + s) * KP + e);
      double up[4], um[4];
      if constexpr (PAIR) {
        const double2 x0 = FB2[((s * NFQ + q) * 2) * ES + el], x1 = FB2[((s * NFQ + q) * 2 + 1) * ES + el];
        up[0] = x0.x, up[1] = x0.y, up[2] = x1.x, up[3] = x1.y;
      } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) up[c] = FB[((s * 4 + c) * NFQ + q) * ES + el];
      }
      if (mirror) {
        if constexpr (PAIR) {
          const double2 y0 = FB2[((s * NFQ + qm) * 2) * ES + nl], y1 = FB2[((s * NFQ + qm) * 2 + 1) * ES + nl];
          um[0] = y0.x, um[1] = y0.y, um[2] = y1.x, um[3] = y1.y;
        } else {
#pragma unroll
          for (int c = 0; c < 4; ++c) um[c] = FB[((s * 4 + c) * NFQ + qm) * ES + nl];
        }
      } else {
        const int4 nb4 = NB[el];
        const int nb = s == 0 ? nb4.x : (s == 1 ? nb4.y : nb4.z);
#pragma unroll
        for (int c = 0; c < 4; ++c) um[c] = 0.0;
#pragma unroll
        for (int k = 0; k < NE; ++k) {
          const int node = s == 0 ? edge_node(P, 0, k) : (s == 1 ? edge_node(P, 1, k) : edge_node(P, 2, k));
          const double cm = TM[(s * NFQ + q) * NE + k];
          double2 n0, n1;
          if (s == 0) {
            n0 = H[(2 * k) * ES + el];
            n1 = H[(2 * k + 1) * ES + el];
          } else {
            n0 = __ldg(a.in + (2 * node) * KP + nb);
            n1 = __ldg(a.in + (2 * node + 1) * KP + nb);
          }
          um[0] = fma(cm, n0.x, um[0]);
          um[1] = fma(cm, n0.y, um[1]);
          um[2] = fma(cm, n1.x, um[2]);
          um[3] = fma(cm, n1.y, um[3]);
        }
      }
      double f[4];
      const int code = roe_flux(up, um, n.x, n.y, f);
      if (code) record_error(a, NFQ, e, q, s, code);
      if constexpr (PAIR) {
        FB2[((s * NFQ + q) * 2) * ES + el] = make_double2(f[0], f[1]);
        FB2[((s * NFQ + q) * 2 + 1) * ES + el] = make_double2(f[2], f[3]);
        if (mirror) {
          FB2[((s * NFQ + qm) * 2) * ES + nl] = make_double2(-f[0], -f[1]);
          FB2[((s * NFQ + qm) * 2 + 1) * ES + nl] = make_double2(-f[2], -f[3]);
        }
      } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) FB[((s * 4 + c) * NFQ + q) * ES + el] = f[c];
        if (mirror) {
#pragma unroll
          for (int c = 0; c < 4; ++c) FB[((s * 4 + c) * NFQ + qm) * ES + nl] = -f[c];
        }
      }
    }
    __syncthreads();

    // next tile's metadata. The face list and face count of this tile are no
    // longer read, so the next tile's go to shared memory now (the item rows
    // are kMaxItems wide, so the copy need not wait for the item count), and
    // the next descriptor into RUNS; the descriptor copies are read again
    // after this run's next barrier (the neighbour table's copy below, the
    // copy issue after the nodal flux, and the next tile's start).
    if (lane == 0 && t < 64) RUNS[t >> 5] = has_next ? NEXT[t >> 5] : make_int4(0, 0, 0, 0);
    if (has_next) {
      if (t < kMaxItems) cp_async4(items + t, a.tile_items + static_cast<long long>(tile + G) * kMaxItems + t);
      if (t == kMaxItems) cp_async4(NITEMS, a.tile_count + tile + G);
    }

    // ---- 4. lift ---------------------------------------------------------------------------
    const int el = col;
    const int e = EL[el];
    const bool valid = e >= 0;
    const int eg = valid ? e : 0;
    constexpr int NH = (NP + 1) / 2;
    constexpr int NR = PAIR ? NH : NP;  // accumulators: double2 per node pair, or one double per node
    double2 r2[PAIR ? NH : 1];
    double r[PAIR ? 1 : NP];
    {
      const double2 lsa = __ldg(a.geo + 5 * KP + eg);
      const double2 lsb = __ldg(a.geo + 6 * KP + eg);
      if constexpr (PAIR) {
#pragma unroll
        for (int i = 0; i < NH; ++i) r2[i] = make_double2(0.0, 0.0);
        if (grp >> 1) pair_lift<P, NFQ, 1>(ops, FB2, grp & 1, el, lsa, lsb, r2);
        else pair_lift<P, NFQ, 0>(ops, FB2, grp & 1, el, lsa, lsb, r2);
      } else {
        const int c = grp;
#pragma unroll
        for (int i = 0; i < NP; ++i) r[i] = 0.0;
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
    }
    // stage 3: U3 / (3 c_out) into the accumulators while the state tile still
    // holds U3 (the update then writes X + c_out (k4 + U3 / (3 c_out)))
    if (a.stage == 3 && valid) {
      const double dtt = a.tile_dt ? __ldg(a.tile_dt + tile) : 1.0;
      const double f = kThird / (a.c_out * dtt);
      if constexpr (PAIR) {
        if (grp >> 1) pair_fold<P, 1>(S, grp & 1, el, f, r2);
        else pair_fold<P, 0>(S, grp & 1, el, f, r2);
      } else {
        const int c = grp;
        const double* Sd = reinterpret_cast<const double*>(S);
#pragma unroll
        for (int i = 0; i < NP; ++i) r[i] = fma(f, Sd[sidx<NP>(2 * i + (c >> 1), el) * 2 + (c & 1)], r[i]);
      }
    }
    (void)NR;
    run_sync(t);

    // the next tile's neighbour table, now that the run's barrier has made its
    // descriptor visible; it lands during the nodal flux phase
    if (has_next && grp == 0) {
      const int4 nr = RUNS[col >= kTileRun];
      const int pos = col % kTileRun;
      if (pos < (col >= kTileRun ? nr.w : nr.y)) cp_async16(NB + col, a.nbr + (col >= kTileRun ? nr.z : nr.x) + pos);
      else NB[col] = make_int4(0, 0, 0, 0);
    }

    // ---- 5. nodal flux of every node, once, contracted with the inverse Jacobian --------
    if (P > 0) {
      const double2 j0 = __ldg(a.geo + 0 * KP + eg);
      const double2 j1 = __ldg(a.geo + 1 * KP + eg);
      for (int j = grp; j < NP; j += 4) {
        const double2 s0 = S[sidx<NP>(2 * j, el)], s1 = S[sidx<NP>(2 * j + 1, el)];
        const double sv[4] = {s0.x, s0.y, s1.x, s1.y};
        double gxi[4], geta[4];
        contravariant_flux(sv, j0.x, j0.y, j1.x, j1.y, gxi, geta);
        if constexpr (PAIR) {  // G2[j][0..1] xi pairs, G2[j][2..3] eta pairs
          FB2[(j * 4 + 0) * ES + el] = make_double2(gxi[0], gxi[1]);
          FB2[(j * 4 + 1) * ES + el] = make_double2(gxi[2], gxi[3]);
          FB2[(j * 4 + 2) * ES + el] = make_double2(geta[0], geta[1]);
          FB2[(j * 4 + 3) * ES + el] = make_double2(geta[2], geta[3]);
        } else {  // G[j][0..3] xi, G[j][4..7] eta
#pragma unroll
          for (int cc = 0; cc < 4; ++cc) {
            FB[(j * 8 + cc) * ES + el] = gxi[cc];
            FB[(j * 8 + 4 + cc) * ES + el] = geta[cc];
          }
        }
      }
    }
    // the neighbour table has landed; the barrier shows it to the column's other threads
    if (grp == 0) cp_async_wait_all();
    run_sync(t);

    // this run's columns of the state tile are free: start its next copies and neighbour rows
    if (has_next) {
      if (t < 64) issue_run_tensor_copy<NP>(&a.map_in, RUNS[t >> 5], t >> 5, S, bar, lane, a.test_flags);
      // the next tile's side-0 neighbours, from the descriptor and neighbour
      // table already in shared memory (held in registers across the lift and
      // the nodal flux they were spilled, and their global load waited on)
      const int4 nr = RUNS[col >= kTileRun];
      const bool nvalid = col % kTileRun < (col >= kTileRun ? nr.w : nr.y);
      const int nbx = NB[col].x;
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int rr = grp + 4 * k;
        if (rr < 2 * NE) {
          if (nvalid) cp_async16(H + rr * ES + col, a.in + rr * KP + nbx);
          else H[rr * ES + col] = make_double2(1.0, 0.0);
        }
      }
    }
    cp_async_commit();

    // the stage update's first operand, requested now so that it is in flight
    // during the volume phase
    const bool upd = valid && a.stage != kStageRhs;
    const double2* src = first_operand(a);
    double2 pre2[PAIR ? NH : 1];
    double pre[PAIR ? 1 : NP];
    if constexpr (PAIR) {
      const int h = grp & 1, half = grp >> 1;
      const long long o = (2 * half * NH + h) * KP + eg;
#pragma unroll
      for (int i = 0; i < NH; ++i)
        pre2[i] = upd && half * NH + i < NP ? ld_early2(src + o + i * 2 * KP) : make_double2(0.0, 0.0);
    } else {
      const int c = grp;
      const double* s1 = reinterpret_cast<const double*>(src) + ((c >> 1) * KP + eg) * 2 + (c & 1);
#pragma unroll
      for (int i = 0; i < NP; ++i) pre[i] = upd ? ld_early(s1 + i * 4 * KP) : 0.0;
    }

    // ---- 6a. volume D_xi G_xi + D_eta G_eta --------------------------------------------
    if (P > 0) {
      if constexpr (PAIR) {
        if (grp >> 1) pair_volume<P, NFQ, 1>(ops, FB2, grp & 1, el, r2);
        else pair_volume<P, NFQ, 0>(ops, FB2, grp & 1, el, r2);
      } else {
        const int c = grp;
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          const double gx = FB[(j * 8 + c) * ES + el];
          const double gy = FB[(j * 8 + 4 + c) * ES + el];
#pragma unroll
          for (int i = 0; i < NP; ++i) r[i] = fma(ops.D[0][i][j], gx, fma(ops.D[1][i][j], gy, r[i]));
        }
      }
    }

    // ---- 6b. stage update ------------------------------------------------------------------
    if (valid) {
      const double dtt = a.tile_dt ? __ldg(a.tile_dt + tile) : 1.0;
      const double c_acc = a.c_acc * dtt, c_out = a.c_out * dtt;
      if constexpr (PAIR) {
        if (grp >> 1) pair_update<P, 1>(a, e, grp & 1, c_acc, c_out, r2, pre2);
        else pair_update<P, 0>(a, e, grp & 1, c_acc, c_out, r2, pre2);
      } else {
        const int c = grp, h = c >> 1, part = c & 1;
        const long long off0 = (h * KP + e) * 2 + part;  // node 0; node i adds i * 4 * KP
        double* acc = reinterpret_cast<double*>(a.acc) + off0;
        double* out = reinterpret_cast<double*>(a.out) + off0;
        const long long step = 4 * KP;  // doubles between node rows of the same pair
        switch (a.stage) {
          case 1: {
            if (!a.no_acc) {  // X = (U_n + U1) / 3 + c_acc k2, as in pair_update
              const double* in = reinterpret_cast<const double*>(a.in) + off0;
              double iv[NP];  // all reads before the first store
#pragma unroll
              for (int i = 0; i < NP; ++i) iv[i] = ld_early(in + i * step);
#pragma unroll
              for (int i = 0; i < NP; ++i) __stcs(acc + i * step, fma(c_acc, r[i], (pre[i] + iv[i]) * kThird));
            }
#pragma unroll
            for (int i = 0; i < NP; ++i) __stcs(out + i * step, fma(c_out, r[i], pre[i]));
            break;
          }
          case 0:
          case 2:
          case 3:
          case kStageEuler:
#pragma unroll
            for (int i = 0; i < NP; ++i) __stcs(out + i * step, fma(c_out, r[i], pre[i]));
            break;
          default:
#pragma unroll
            for (int i = 0; i < NP; ++i) __stcs(out + i * step, r[i]);
            break;
        }
      }
    }
    // the four warps of a run work on the same elements: none may start the
    // next tile's traces (which reuse rows of the face / flux buffer) before
    // the others are done with this tile's volume phase
    run_sync(t);
  }

  cp_async_wait_all();  // none may land after the block has left
  if (*abort_flag) {
    // the bulk copies of a tile whose wait gave up may still land: wait for
    // them once more, with the same bound, before the block leaves
    for (unsigned n = 0; n < max_tries; ++n)
      if (mbar_try_wait(bar, parity ^ 1u)) break;
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
