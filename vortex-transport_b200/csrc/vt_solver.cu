// C ABI of the device solver (include/vortex_b200.h, "drop-in boundary").
//
// vt_create folds the reference-space operators into the per-stage kernel
// parameter block and uploads packed per-element geometry; vt_step_rk4 replays
// a captured CUDA graph of the four fused stage kernels once per step.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/vortex_b200.h"
#include "vt_common.h"
#include "vt_ctx.h"
#include "vt_precompute.h"
#include "vt_launch.h"

namespace vt {
namespace {

std::vector<double> fold_operators(int p, int nfq, const double* minv, const double* stiff,
                                   const double* line, const double* phi_plus,
                                   const double* phi_minus) {
  std::vector<double> ops(static_cast<size_t>(stage_ops_doubles(p, nfq)));
  fold_stage_operators(p, nfq, minv, stiff, line, phi_plus, phi_minus, ops.data());
  return ops;
}

// Host AoS (K x Np x 4) <-> device SoA-of-double2 rows, through a shared
// memory tile of 32 elements so both sides stay coalesced.
constexpr int kTileE = 32;

__global__ void aos_to_soa_kernel(const double2* __restrict__ aos, double2* __restrict__ soa, int K,
                                  int Np, long long Kpad) {
  extern __shared__ double2 tile[];
  const int R = 2 * Np;
  const int e0 = blockIdx.x * kTileE;
  const int ne = min(kTileE, K - e0);
  for (int l = threadIdx.x; l < ne * R; l += blockDim.x) tile[l] = aos[static_cast<long long>(e0) * R + l];
  __syncthreads();
  for (int l = threadIdx.x; l < kTileE * R; l += blockDim.x) {
    const int r = l / kTileE, j = l % kTileE;
    if (j < ne) soa[r * Kpad + e0 + j] = tile[j * R + r];
  }
}

__global__ void soa_to_aos_kernel(const double2* __restrict__ soa, double2* __restrict__ aos, int K,
                                  int Np, long long Kpad) {
  extern __shared__ double2 tile[];
  const int R = 2 * Np;
  const int e0 = blockIdx.x * kTileE;
  const int ne = min(kTileE, K - e0);
  for (int l = threadIdx.x; l < kTileE * R; l += blockDim.x) {
    const int r = l / kTileE, j = l % kTileE;
    if (j < ne) tile[j * R + r] = soa[r * Kpad + e0 + j];
  }
  __syncthreads();
  for (int l = threadIdx.x; l < ne * R; l += blockDim.x) aos[static_cast<long long>(e0) * R + l] = tile[l];
}

// Conservation totals: per block, sum over its elements of detJ * W . U in a
// fixed order; a second single-block pass sums the partials in a fixed order.
__global__ void totals_partial_kernel(const double2* __restrict__ U, const double2* __restrict__ geo,
                                      const double* __restrict__ W, int K, int Np, long long Kpad,
                                      double* __restrict__ partial) {
  __shared__ double red[4][256];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[4] = {0, 0, 0, 0};
  if (e < K) {
    const double detj = geo[6 * Kpad + e].y;
    for (int i = 0; i < Np; ++i) {
      const double2 a = U[(2 * i) * Kpad + e], b = U[(2 * i + 1) * Kpad + e];
      acc[0] += W[i] * a.x;
      acc[1] += W[i] * a.y;
      acc[2] += W[i] * b.x;
      acc[3] += W[i] * b.y;
    }
    for (int c = 0; c < 4; ++c) acc[c] *= detj;
  }
  for (int c = 0; c < 4; ++c) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int c = 0; c < 4; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) partial[blockIdx.x * 4 + threadIdx.x] = red[threadIdx.x][0];
}

// The L2 difference of two states in the form of the reference's
// post-processing script (plottools/l2stateerror.py:65-98): per element the
// squared nodal differences, interpolated at the area-rule points (bq: nq x Np
// basis values), integrated with the rule weights and det J. Per-block partial
// sums in a fixed order, summed by totals_final_kernel.
__global__ void l2_partial_kernel(const double2* __restrict__ U, const double2* __restrict__ V,
                                  const double2* __restrict__ geo, const double* __restrict__ bq,
                                  const double* __restrict__ wq, int nq, int K, int Np, long long Kpad,
                                  double* __restrict__ partial) {
  __shared__ double red[4][256];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[4] = {0, 0, 0, 0};
  if (e < K) {
    double del[10][4];
    for (int j = 0; j < Np; ++j) {
      const double2 a = U[(2 * j) * Kpad + e], b = U[(2 * j + 1) * Kpad + e];
      const double2 c = V[(2 * j) * Kpad + e], d = V[(2 * j + 1) * Kpad + e];
      const double x[4] = {a.x - c.x, a.y - c.y, b.x - d.x, b.y - d.y};
      for (int k = 0; k < 4; ++k) del[j][k] = x[k] * x[k];
    }
    for (int k = 0; k < 4; ++k) {
      double s = 0.0;
      for (int q = 0; q < nq; ++q) {
        double v = 0.0;
        for (int j = 0; j < Np; ++j) v += del[j][k] * bq[q * Np + j];
        s += wq[q] * v;
      }
      acc[k] = geo[6 * Kpad + e].y * s;
    }
  }
  for (int c = 0; c < 4; ++c) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int c = 0; c < 4; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) partial[blockIdx.x * 4 + threadIdx.x] = red[threadIdx.x][0];
}

// The isentropic vortex (Element.cpp:134-179 formula, parameters from `ic`).
__device__ void vortex_point(const vt_vortex& c, double x, double y, double t, double* s) {
  const double dx = x - c.x0 - c.U_infty * t, dy = y - c.y0 - c.V_infty * t;
  const double f0 = 1.0 - (dx * dx + dy * dy) / (c.rc * c.rc);
  const double f1 = 1.0 - c.epsilon * c.epsilon * (c.gamma - 1) * (c.M_infty * c.M_infty) * exp(f0) /
                              (8.0 * (M_PI * M_PI));
  const double f2 = c.epsilon * (c.U_infty * c.U_infty + c.V_infty * c.V_infty) * exp(f0 / 2.0) / (2.0 * M_PI * c.rc);
  const double rho = c.rho_infty * pow(f1, 1.0 / (c.gamma - 1.0));
  const double u = c.U_infty - f2 * dy, v = c.V_infty + f2 * dx;
  const double p = c.p_infty * pow(f1, c.gamma / (c.gamma - 1.0));
  const double E = p / (rho * (c.gamma - 1.0)) + (u * u + v * v) / 2.0;
  s[0] = rho;
  s[1] = rho * u;
  s[2] = rho * v;
  s[3] = rho * E;
}

// L2 projection of the vortex onto each element's basis (Element.cpp:180-326):
// b_i = sum_q detJ phi_i(q) u(x_q) w_q, U_i = sum_j (M_ref^-1_ij / detJ) b_j, with
// x_q the affine image of the area-rule point. One thread per element; tab
// holds the basis at the points (nq x Np), the weights (nq), the points (nq x 2)
// and M_ref^-1 (Np x Np).
__global__ void project_vortex_kernel(const double* __restrict__ verts, const double2* __restrict__ geo,
                                      const double* __restrict__ tab, int nq, const vt_vortex ic, double t, int K,
                                      int Np, long long Kpad, double2* __restrict__ U) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= K) return;
  const double* bq = tab;
  const double* wq = tab + nq * Np;
  const double* pq = wq + nq;
  const double* minv = pq + 2 * nq;
  const double* v = verts + 6 * static_cast<long long>(e);
  const double det = geo[6 * Kpad + e].y;
  double b[10][4];
  for (int i = 0; i < Np; ++i)
    for (int k = 0; k < 4; ++k) b[i][k] = 0.0;
  for (int q = 0; q < nq; ++q) {
    const double xi = pq[2 * q], eta = pq[2 * q + 1];
    const double h0 = 1.0 - xi - eta;
    const double x = v[0] * h0 + v[2] * xi + v[4] * eta;
    const double y = v[1] * h0 + v[3] * xi + v[5] * eta;
    double s[4];
    vortex_point(ic, x, y, t, s);
    for (int i = 0; i < Np; ++i)
      for (int k = 0; k < 4; ++k) b[i][k] += det * bq[q * Np + i] * s[k] * wq[q];
  }
  for (int i = 0; i < Np; ++i) {
    double r[4] = {0, 0, 0, 0};
    for (int j = 0; j < Np; ++j)
      for (int k = 0; k < 4; ++k) r[k] += (minv[i * Np + j] / det) * b[j][k];
    U[(2 * i) * Kpad + e] = make_double2(r[0], r[1]);
    U[(2 * i + 1) * Kpad + e] = make_double2(r[2], r[3]);
  }
}

// ---- the reference's structured periodic mesh, generated on the device --------
// Meshgeneration.cpp:16-186 and Element.cpp:54-93 per element, with the
// parameter block's float arithmetic kept where the reference has it (the
// grid spacing and origin are float expressions widened to double). sin, cos
// and pow are CUDA's, so perturbed vertices agree with the host's (glibc) to
// rounding; connectivity is exact.
struct GridSpec {
  int nx, ny;
  double gx0, gy0, esx, esy;  // origin and spacing, as the reference rounds them
  float pg;                    // perturb_grid
  double nodes_ref[20];        // Np x 2 reference nodes
};

__device__ void grid_point(const GridSpec& g, int a, int b, double* x, double* y) {
  // products and sums rounded one at a time, as the host build (no contraction) does
  const double gx = __dadd_rn(g.gx0, __dmul_rn(g.esx, b)), gy = __dadd_rn(g.gy0, __dmul_rn(g.esy, a));
  const int inner = (a == 0 ? 0 : 1) * (a == g.ny ? 0 : 1) * (b == 0 ? 0 : 1) * (b == g.nx ? 0 : 1);
  const float ip = static_cast<float>(inner) * g.pg;
  const double cx = __dmul_rn(__dmul_rn(static_cast<double>(ip), 0.2), g.esx);
  const double cy = __dmul_rn(__dmul_rn(static_cast<double>(ip), 0.2), g.esy);
  *x = __dadd_rn(gx, __dmul_rn(cx, sin(pow(gx + 6, gy + 6))));
  *y = __dadd_rn(gy, __dmul_rn(cy, cos(pow(gy + 6, gx + 6))));
}

// One thread per element: vertices, packed geometry rows, side-ordered
// neighbours, and (when U is given) the nodal vortex state at the nodes.
__global__ void structured_mesh_kernel(const GridSpec g, int Np, long long Kpad, double* __restrict__ verts,
                                       double2* __restrict__ geo, int4* __restrict__ nbr, const vt_vortex ic,
                                       double2* __restrict__ U) {
  const int K = 2 * g.nx * g.ny;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= K) return;
  const int nx = g.nx, ny = g.ny;
  const int cell = e >> 1, r = cell / nx, j = cell % nx;
  const bool even = (e & 1) == 0;
  // vertex grid points (row, column): n1, n2 = n1 -+ 1, n3 = the partner's n2
  const int va[3] = {even ? r : r + 1, even ? r : r + 1, even ? r + 1 : r};
  const int vb[3] = {even ? j : j + 1, even ? j + 1 : j, even ? j : j + 1};
  double v[6];
  for (int k = 0; k < 3; ++k) grid_point(g, va[k], vb[k], &v[2 * k], &v[2 * k + 1]);
  for (int k = 0; k < 6; ++k) verts[6ll * e + k] = v[k];
  const double x0 = v[0], y0 = v[1], x1 = v[2], y1 = v[3], x2 = v[4], y2 = v[5];
  const double j00 = x1 - x0, j01 = x2 - x0, j10 = y1 - y0, j11 = y2 - y0;
  const double det = __dsub_rn(__dmul_rn(j00, j11), __dmul_rn(j10, j01));
  const double rdet = 1 / det;
  const double i00 = __dmul_rn(rdet, y2 - y0), i01 = __dmul_rn(rdet, x0 - x2);
  const double i10 = __dmul_rn(rdet, y0 - y1), i11 = __dmul_rn(rdet, x1 - x0);
  const double l0 = pow(__dadd_rn(__dmul_rn(x1 - x0, x1 - x0), __dmul_rn(y1 - y0, y1 - y0)), 0.5);
  const double l1 = pow(__dadd_rn(__dmul_rn(x2 - x1, x2 - x1), __dmul_rn(y2 - y1, y2 - y1)), 0.5);
  const double l2 = pow(__dadd_rn(__dmul_rn(x0 - x2, x0 - x2), __dmul_rn(y0 - y2, y0 - y2)), 0.5);
  geo[0 * Kpad + e] = make_double2(i00, i01);
  geo[1 * Kpad + e] = make_double2(i10, i11);
  geo[2 * Kpad + e] = make_double2((y1 - y0) / l0, -1 * (x1 - x0) / l0);
  geo[3 * Kpad + e] = make_double2((y2 - y1) / l1, -1 * (x2 - x1) / l1);
  geo[4 * Kpad + e] = make_double2((y0 - y2) / l2, -1 * (x0 - x2) / l2);
  geo[5 * Kpad + e] = make_double2(l0 / det, l1 / det);
  geo[6 * Kpad + e] = make_double2(l2 / det, det);
  const int left = e % (2 * nx) == 0 ? e - 1 + 2 * nx : e - 1;
  const int right = (e + 1) % (2 * nx) == 0 ? e + 1 - 2 * nx : e + 1;
  int vert;
  if (e >= 2 * nx * (ny - 1)) vert = even ? e + 1 - 2 * nx : e - 1 - 2 * nx * (ny - 1);
  else if (e >= 2 * nx) vert = even ? e + 1 - 2 * nx : e - 1 + 2 * nx;
  else vert = even ? e + 1 + 2 * nx * (ny - 1) : e - 1 + 2 * nx;
  nbr[e] = even ? make_int4(vert, right, left, 0) : make_int4(vert, left, right, 0);
  if (!U) return;
  for (int i = 0; i < Np; ++i) {  // nodal initial condition (Element.cpp:124-179)
    const double xi = g.nodes_ref[2 * i], eta = g.nodes_ref[2 * i + 1], h0 = 1.0 - xi - eta;
    double s4[4];
    const double px = __dadd_rn(__dadd_rn(__dmul_rn(x0, h0), __dmul_rn(x1, xi)), __dmul_rn(x2, eta));
    const double py = __dadd_rn(__dadd_rn(__dmul_rn(y0, h0), __dmul_rn(y1, xi)), __dmul_rn(y2, eta));
    vortex_point(ic, px, py, 0.0, s4);
    U[(2 * i) * Kpad + e] = make_double2(s4[0], s4[1]);
    U[(2 * i + 1) * Kpad + e] = make_double2(s4[2], s4[3]);
  }
}

__global__ void totals_final_kernel(const double* __restrict__ partial, int nblocks,
                                    double* __restrict__ out) {
  __shared__ double red[4][256];
  double acc[4] = {0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int c = 0; c < 4; ++c) acc[c] += partial[b * 4 + c];
  for (int c = 0; c < 4; ++c) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int c = 0; c < 4; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[threadIdx.x] = red[threadIdx.x][0];
}

}  // namespace

std::string cuda_msg(const char* what, cudaError_t e) {
  return std::string(what) + ": " + cudaGetErrorString(e);
}

}  // namespace vt

namespace {

using vt::fail;

template <typename T>
cudaError_t alloc(T** p, size_t bytes) {
  return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}

void release(vt_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  vt::adjoint_release(c);
  if (c->rk4_graph) cudaGraphExecDestroy(c->rk4_graph);
  void* bufs[] = {c->U,  c->A,     c->Sa,  c->Sb,         c->R,          c->geo,     c->nbr,
                  c->err, c->aos,  c->W,   c->partial,    c->tot,        c->tiles,   c->tile_items,
                  c->tile_count};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

}  // namespace

namespace vt {

vt::StageArgs stage_args(vt_ctx* c, const double2* in, const double2* base, double2* acc, double2* out,
                         int stage, double c_acc, double c_out) {
  vt::StageArgs a;
  a.in = in;
  a.base = base;
  a.acc = acc;
  a.out = out;
  a.geo = c->geo;
  a.nbr = c->nbr;
  a.tiles = c->tiles;
  a.tile_items = c->tile_items;
  a.tile_dt = c->tile_dt;
  a.tile_count = c->tile_count;
  a.ntiles = c->ntiles;
  a.err = c->err;
  a.Kpad = c->Kpad;
  a.K = c->K;
  a.stage = stage;
  a.c_acc = c_acc;
  a.c_out = c_out;
  a.wait_tries = c->test_wait_tries;
  a.test_flags = c->test_flags;
  return a;
}

cudaError_t enqueue_rk4_step(vt_ctx* c, double dt) {
  cudaError_t e;
  const double* ops = c->ops.data();
  if ((e = c->launch(stage_args(c, c->U, c->U, c->A, c->Sa, 0, (1.0 / 6) * dt, 0.5 * dt), ops, c->max_blocks, c->stream))) return e;
  if ((e = c->launch(stage_args(c, c->Sa, c->U, c->A, c->Sb, 1, (1.0 / 3) * dt, 0.5 * dt), ops, c->max_blocks, c->stream))) return e;
  if ((e = c->launch(stage_args(c, c->Sb, c->U, c->A, c->Sa, 2, (1.0 / 3) * dt, dt), ops, c->max_blocks, c->stream))) return e;
  return c->launch(stage_args(c, c->Sa, c->U, c->A, c->U, 3, 0.0, (1.0 / 6) * dt), ops, c->max_blocks, c->stream);
}

cudaError_t reset_error_words(vt_ctx* c) {
  cudaError_t e = cudaMemsetAsync(c->err, 0xFF, sizeof(unsigned long long), c->stream);
  if (e) return e;
  return cudaMemsetAsync(c->err + 1, 0, 3 * sizeof(unsigned long long), c->stream);
}

// Waits for the stream, decodes the first-error key and advances the clock.
int finish(vt_ctx* c, int nsteps, double dt) {
  unsigned long long words[4] = {~0ull, 0, 0, 0};
  cudaError_t e = cudaMemcpyAsync(words, c->err, sizeof(words), cudaMemcpyDeviceToHost, c->stream);
  if (!e) e = cudaStreamSynchronize(c->stream);
  if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("step", e));
  for (int s = 0; s < nsteps; ++s) c->time += dt;  // Element::time += t_step per step
  c->last = vt_error_info{};
  if (words[3] & 2ull)
    return fail(VT_ERR_CUDA, "stage kernel: a bulk-copy wait gave up (the state is not valid)");
  const unsigned long long key = words[0];
  if (key == ~0ull) return VT_OK;
  c->last = vt::decode_error_key(key, c->nfq);
  return fail(c->last.code, "Non-physical state (code " + std::to_string(c->last.code) + ") at element " +
                                std::to_string(c->last.element) + ", step " + std::to_string(c->last.step) +
                                ", stage " + std::to_string(c->last.stage));
}

int ensure_aos(vt_ctx* c) {
  if (c->aos) return VT_OK;
  cudaError_t e = alloc(&c->aos, sizeof(double) * 4 * static_cast<size_t>(c->K) * c->Np);
  return e ? fail(VT_ERR_NO_MEMORY, vt::cuda_msg("staging buffer", e)) : VT_OK;
}

cudaError_t aos_to_soa(vt_ctx* c, const double* src, double2* dst) {
  const int blocks = (c->K + vt::kTileE - 1) / vt::kTileE;
  const size_t smem = sizeof(double2) * vt::kTileE * 2 * c->Np;
  vt::aos_to_soa_kernel<<<blocks, 256, smem, c->stream>>>(reinterpret_cast<const double2*>(src), dst, c->K,
                                                          c->Np, c->Kpad);
  return cudaGetLastError();
}

cudaError_t soa_to_aos(vt_ctx* c, const double2* src, double* dst) {
  const int blocks = (c->K + vt::kTileE - 1) / vt::kTileE;
  const size_t smem = sizeof(double2) * vt::kTileE * 2 * c->Np;
  vt::soa_to_aos_kernel<<<blocks, 256, smem, c->stream>>>(src, reinterpret_cast<double2*>(dst), c->K, c->Np,
                                                          c->Kpad);
  return cudaGetLastError();
}

}  // namespace vt

using vt::aos_to_soa;
using vt::enqueue_rk4_step;
using vt::ensure_aos;
using vt::finish;
using vt::reset_error_words;
using vt::soa_to_aos;
using vt::stage_args;

extern "C" {

vt_ctx* vt_create(const vt_mesh_desc* d, int device, int* status) {
  auto set = [&](int s) {
    if (status) *status = s;
  };
  if (!d || !d->element_type || !d->neighbours || !d->det_jacobian || !d->inv_jacobian || !d->normals ||
      !d->side_lengths || !d->inv_mass_ref || !d->stiffness_ref || !d->line_quadrature || !d->phi_plus ||
      !d->phi_minus) {
    set(fail(VT_ERR_INVALID, "vt_create: null descriptor field"));
    return nullptr;
  }
  if (d->p < 0 || d->p > 3) {
    set(fail(VT_ERR_UNSUPPORTED, "vt_create: p must be 0..3"));
    return nullptr;
  }
  if (d->n_line_points < 1 || d->n_line_points > 10) {
    set(fail(VT_ERR_UNSUPPORTED, "vt_create: n_line_points must be 1..10"));
    return nullptr;
  }
  if (d->n_elements < 1) {
    set(fail(VT_ERR_INVALID, "vt_create: n_elements must be positive"));
    return nullptr;
  }
  const int K = d->n_elements;
  for (int n = 0; n < 3 * K; ++n)
    if (d->neighbours[n] < 0 || d->neighbours[n] >= K) {
      set(fail(VT_ERR_INVALID, "vt_create: neighbour index out of range at element " + std::to_string(n / 3)));
      return nullptr;
    }
  cudaError_t e = cudaSetDevice(device);
  if (e) {
    set(fail(VT_ERR_CUDA, vt::cuda_msg("cudaSetDevice", e)));
    return nullptr;
  }
  auto* c = new vt_ctx();
  c->device = device;
  c->p = d->p;
  c->Np = vt::np_of(d->p);
  c->nfq = d->n_line_points;
  c->K = K;
  c->Kpad = (static_cast<long long>(K) + 127) / 128 * 128;
  const vt::StageKernel sk = vt::select_kernel(c->p, c->nfq);
  c->launch = sk.launch;
  int per_sm = 0, sms = 0;
  if ((e = vt::tensor_maps_available()) || (e = sk.configure(&per_sm)) ||
      (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device))) {
    set(fail(VT_ERR_CUDA, vt::cuda_msg("stage kernel attributes", e)));
    delete c;
    return nullptr;
  }
  c->max_blocks = sms * (per_sm > 0 ? per_sm : 1);
  c->ops = vt::fold_operators(c->p, c->nfq, d->inv_mass_ref, d->stiffness_ref, d->line_quadrature,
                              d->phi_plus, d->phi_minus);
  c->minv_ref.assign(d->inv_mass_ref, d->inv_mass_ref + c->Np * c->Np);

  // packed geometry and side-ordered neighbours (Evolve.cpp:167-202)
  const long long KP = c->Kpad;
  std::vector<double2> geo(7 * static_cast<size_t>(KP), make_double2(0.0, 0.0));
  std::vector<int4> nbr(static_cast<size_t>(KP), make_int4(0, 0, 0, 0));
  for (int n = 0; n < K; ++n) {
    const double* ji = d->inv_jacobian + 4 * static_cast<size_t>(n);
    const double* nv = d->normals + 6 * static_cast<size_t>(n);
    const double* ln = d->side_lengths + 3 * static_cast<size_t>(n);
    const double det = d->det_jacobian[n];
    geo[0 * KP + n] = make_double2(ji[0], ji[1]);
    geo[1 * KP + n] = make_double2(ji[2], ji[3]);
    for (int s = 0; s < 3; ++s) geo[(2 + s) * KP + n] = make_double2(nv[2 * s], nv[2 * s + 1]);
    geo[5 * KP + n] = make_double2(ln[0] / det, ln[1] / det);
    geo[6 * KP + n] = make_double2(ln[2] / det, det);
    const int right = d->neighbours[3 * n], left = d->neighbours[3 * n + 1], vert = d->neighbours[3 * n + 2];
    nbr[n] = d->element_type[n] == 0 ? make_int4(vert, right, left, 0) : make_int4(vert, left, right, 0);
  }
  // side s of an element faces side s of its neighbour (Evolve.cpp:167-202 on
  // the reference mesh); the adjoint's gather of neighbour face terms needs it
  c->side_pairing = true;
  for (int n = 0; n < K && c->side_pairing; ++n) {
    const int4 b = nbr[n];
    c->side_pairing = nbr[b.x].x == n && nbr[b.y].y == n && nbr[b.z].z == n;
  }
  // W_i = integral of phi_i = sum_j M_ref[i][j] (the basis sums to one)
  std::vector<double> m(d->inv_mass_ref, d->inv_mass_ref + c->Np * c->Np), W(c->Np, 0.0);
  vt::invert_gauss_jordan(c->Np, &m);
  for (int i = 0; i < c->Np; ++i)
    for (int j = 0; j < c->Np; ++j) W[i] += m[i * c->Np + j];

  const size_t state_bytes = sizeof(double2) * 2 * c->Np * static_cast<size_t>(KP);
  const int tot_blocks = (K + 255) / 256;
  if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) || (e = alloc(&c->U, state_bytes)) ||
      (e = alloc(&c->A, state_bytes)) || (e = alloc(&c->Sa, state_bytes)) || (e = alloc(&c->Sb, state_bytes)) ||
      (e = alloc(&c->geo, geo.size() * sizeof(double2))) || (e = alloc(&c->nbr, nbr.size() * sizeof(int4))) ||
      (e = alloc(&c->err, 4 * sizeof(unsigned long long))) || (e = alloc(&c->W, sizeof(double) * c->Np)) ||
      (e = alloc(&c->partial, sizeof(double) * 4 * tot_blocks)) || (e = alloc(&c->tot, sizeof(double) * 4))) {
    const bool oom = e == cudaErrorMemoryAllocation;
    set(fail(oom ? VT_ERR_NO_MEMORY : VT_ERR_CUDA, vt::cuda_msg("vt_create", e)));
    release(c);
    return nullptr;
  }
  if ((e = cudaMemcpy(c->geo, geo.data(), geo.size() * sizeof(double2), cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(c->nbr, nbr.data(), nbr.size() * sizeof(int4), cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(c->W, W.data(), sizeof(double) * c->Np, cudaMemcpyHostToDevice)) ||
      (e = cudaMemset(c->U, 0, state_bytes)) || (e = cudaMemset(c->A, 0, state_bytes)) ||
      (e = cudaMemset(c->Sa, 0, state_bytes)) || (e = cudaMemset(c->Sb, 0, state_bytes))) {
    set(fail(VT_ERR_CUDA, vt::cuda_msg("vt_create upload", e)));
    release(c);
    return nullptr;
  }
  // tile schedule: two-row tiles on the reference's structured mesh, runs of
  // consecutive elements otherwise; then each tile's face list
  {
    const std::vector<int4> runs = vt::structured_tile_runs(K, d->element_type, d->neighbours);
    c->ntiles = runs.empty() ? (K + vt::kTileElems - 1) / vt::kTileElems : static_cast<int>(runs.size());
    if ((e = alloc(&c->tiles, sizeof(int4) * c->ntiles)) ||
        (e = alloc(&c->tile_items, sizeof(int) * vt::kMaxItems * static_cast<size_t>(c->ntiles))) ||
        (e = alloc(&c->tile_count, sizeof(int) * c->ntiles))) {
      set(fail(e == cudaErrorMemoryAllocation ? VT_ERR_NO_MEMORY : VT_ERR_CUDA, vt::cuda_msg("tiles", e)));
      release(c);
      return nullptr;
    }
    if (runs.empty())
      e = vt::launch_contiguous_tiles(c->tiles, K, c->ntiles, c->stream);
    else
      e = cudaMemcpyAsync(c->tiles, runs.data(), sizeof(int4) * runs.size(), cudaMemcpyHostToDevice, c->stream);
    if (!e) e = vt::launch_build_tile_items(c->tiles, c->nbr, c->tile_items, c->tile_count, c->ntiles, c->nfq, c->stream);
    if (!e) e = cudaStreamSynchronize(c->stream);
    if (e) {
      set(fail(VT_ERR_CUDA, vt::cuda_msg("tile schedule", e)));
      release(c);
      return nullptr;
    }
  }
  set(VT_OK);
  return c;
}

vt_ctx* vt_create_structured(const vt_params* prm, const vt_vortex* ic_in, int device, int* status) {
  auto set = [&](int s) {
    if (status) *status = s;
  };
  if (!prm) {
    set(fail(VT_ERR_INVALID, "vt_create_structured: null parameters"));
    return nullptr;
  }
  if (prm->p < 0 || prm->p > 3 || prm->integration_order < 0 || prm->integration_order > 19 ||
      (prm->U_initialization_type != 0 && prm->U_initialization_type != 1)) {
    set(fail(VT_ERR_UNSUPPORTED, "vt_create_structured: p, integration_order or U_initialization_type out of range"));
    return nullptr;
  }
  const int nx = prm->num_element_in_x, ny = prm->num_element_in_y;
  if (nx < 1 || ny < 1 || 2.0 * nx * ny > 2147483647.0 / 64) {
    set(fail(VT_ERR_INVALID, "vt_create_structured: num_element_in_x/y out of range"));
    return nullptr;
  }
  // With one row of cells the reference's periodic vertical-neighbour formula
  // (Meshgeneration.cpp:94-117) gives every even element a negative index, a
  // mesh vt_create rejects as well; the device set-up never builds one.
  if (ny < 2) {
    set(fail(VT_ERR_INVALID, "vt_create_structured: num_element_in_y must be at least 2 (the reference's "
                             "vertical neighbour of a single row is out of range)"));
    return nullptr;
  }
  const vt_vortex ic = ic_in ? *ic_in : vt::default_vortex();
  // reference-space tables (host, a few KB)
  const int p = prm->p, Np = vt::np_of(p);
  std::vector<double> line, area, minv, pp, pm;
  vt::line_rule(prm->integration_order, &line);
  vt::area_rule(prm->integration_order, &area);
  const std::vector<double> nodes_ref = vt::reference_nodes(p);
  if (!vt::inverse_mass_reference(p, area, &minv)) {
    set(fail(VT_ERR_UNSUPPORTED, "vt_create_structured: the reference mass matrix is singular for this rule"));
    return nullptr;
  }
  const std::vector<double> stiff = vt::stiffness_reference(p, area);
  vt::face_tables(p, line, &pp, &pm);
  const int nfq = static_cast<int>(line.size() / 2);
  if (nfq < 1 || nfq > 10) {
    set(fail(VT_ERR_UNSUPPORTED, "vt_create_structured: n_line_points must be 1..10"));
    return nullptr;
  }
  cudaError_t e = cudaSetDevice(device);
  if (e) {
    set(fail(VT_ERR_CUDA, vt::cuda_msg("cudaSetDevice", e)));
    return nullptr;
  }
  auto* c = new vt_ctx();
  c->device = device;
  c->p = p;
  c->Np = Np;
  c->nfq = nfq;
  c->K = 2 * nx * ny;
  c->Kpad = (static_cast<long long>(c->K) + 127) / 128 * 128;
  const vt::StageKernel sk = vt::select_kernel(p, nfq);
  c->launch = sk.launch;
  int per_sm = 0, sms = 0;
  if ((e = vt::tensor_maps_available()) || (e = sk.configure(&per_sm)) ||
      (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device))) {
    set(fail(VT_ERR_CUDA, vt::cuda_msg("stage kernel attributes", e)));
    delete c;
    return nullptr;
  }
  c->max_blocks = sms * (per_sm > 0 ? per_sm : 1);
  c->ops = vt::fold_operators(p, nfq, minv.data(), stiff.data(), line.data(), pp.data(), pm.data());
  c->minv_ref = minv;
  c->side_pairing = true;
  std::vector<double> m(minv), W(Np, 0.0);
  vt::invert_gauss_jordan(Np, &m);
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Np; ++j) W[i] += m[i * Np + j];

  const long long KP = c->Kpad;
  const size_t state_bytes = sizeof(double2) * 2 * Np * static_cast<size_t>(KP);
  const int tot_blocks = (c->K + 255) / 256;
  double* verts = nullptr;
  if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) || (e = alloc(&c->U, state_bytes)) ||
      (e = alloc(&c->A, state_bytes)) || (e = alloc(&c->Sa, state_bytes)) || (e = alloc(&c->Sb, state_bytes)) ||
      (e = alloc(&c->geo, sizeof(double2) * 7 * KP)) || (e = alloc(&c->nbr, sizeof(int4) * KP)) ||
      (e = alloc(&c->err, 4 * sizeof(unsigned long long))) || (e = alloc(&c->W, sizeof(double) * Np)) ||
      (e = alloc(&c->partial, sizeof(double) * 4 * tot_blocks)) || (e = alloc(&c->tot, sizeof(double) * 4)) ||
      (e = alloc(&verts, sizeof(double) * 6 * static_cast<size_t>(c->K)))) {
    set(fail(e == cudaErrorMemoryAllocation ? VT_ERR_NO_MEMORY : VT_ERR_CUDA, vt::cuda_msg("vt_create_structured", e)));
    if (verts) cudaFree(verts);
    release(c);
    return nullptr;
  }
  // grid origin and spacing as the reference rounds them (float, then widened)
  vt::GridSpec g{};
  g.nx = nx;
  g.ny = ny;
  const float esxf = prm->domain_x / nx, esyf = prm->domain_y / ny;
  const float gx0f = -1 * prm->domain_x / 2, gy0f = -1 * prm->domain_y / 2;
  g.esx = esxf;
  g.esy = esyf;
  g.gx0 = gx0f;
  g.gy0 = gy0f;
  g.pg = prm->perturb_grid;
  for (int i = 0; i < 2 * Np; ++i) g.nodes_ref[i] = nodes_ref[i];
  // the projected initial condition's table: basis at the area points, weights, points, M_ref^-1
  const int nq = static_cast<int>(area.size() / 3);
  std::vector<double> tab(static_cast<size_t>(nq) * (Np + 3) + Np * Np);
  for (int q = 0; q < nq; ++q) {
    vt::basis(p, area[3 * q], area[3 * q + 1], &tab[static_cast<size_t>(q) * Np]);
    tab[static_cast<size_t>(nq) * Np + q] = area[3 * q + 2];
    tab[static_cast<size_t>(nq) * (Np + 1) + 2 * q] = area[3 * q];
    tab[static_cast<size_t>(nq) * (Np + 1) + 2 * q + 1] = area[3 * q + 1];
  }
  std::copy(minv.begin(), minv.end(), tab.begin() + static_cast<size_t>(nq) * (Np + 3));
  double* dtab = nullptr;
  if (!e) e = cudaMemsetAsync(c->U, 0, state_bytes, c->stream);
  if (!e) e = cudaMemsetAsync(c->A, 0, state_bytes, c->stream);
  if (!e) e = cudaMemsetAsync(c->Sa, 0, state_bytes, c->stream);
  if (!e) e = cudaMemsetAsync(c->Sb, 0, state_bytes, c->stream);
  if (!e) e = cudaMemsetAsync(c->geo, 0, sizeof(double2) * 7 * KP, c->stream);
  if (!e) e = cudaMemsetAsync(c->nbr, 0, sizeof(int4) * KP, c->stream);
  if (!e) e = cudaMemcpyAsync(c->W, W.data(), sizeof(double) * Np, cudaMemcpyHostToDevice, c->stream);
  if (!e) {
    vt::structured_mesh_kernel<<<(c->K + 127) / 128, 128, 0, c->stream>>>(
        g, Np, KP, verts, c->geo, c->nbr, ic, prm->U_initialization_type == 0 ? c->U : nullptr);
    e = cudaGetLastError();
  }
  if (!e && prm->U_initialization_type == 1) {
    e = alloc(&dtab, sizeof(double) * tab.size());
    if (!e) e = cudaMemcpyAsync(dtab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, c->stream);
    if (!e) {
      vt::project_vortex_kernel<<<(c->K + 127) / 128, 128, 0, c->stream>>>(verts, c->geo, dtab, nq, ic, 0.0, c->K, Np,
                                                                          KP, c->U);
      e = cudaGetLastError();
    }
  }
  // tiles: two-row runs of the structured mesh, or runs of consecutive elements
  const std::vector<int4> runs = vt::grid_tile_runs(nx, ny);
  c->ntiles = runs.empty() ? (c->K + vt::kTileElems - 1) / vt::kTileElems : static_cast<int>(runs.size());
  if (!e) e = alloc(&c->tiles, sizeof(int4) * c->ntiles);
  if (!e) e = alloc(&c->tile_items, sizeof(int) * vt::kMaxItems * static_cast<size_t>(c->ntiles));
  if (!e) e = alloc(&c->tile_count, sizeof(int) * c->ntiles);
  if (!e) {
    if (runs.empty())
      e = vt::launch_contiguous_tiles(c->tiles, c->K, c->ntiles, c->stream);
    else
      e = cudaMemcpyAsync(c->tiles, runs.data(), sizeof(int4) * runs.size(), cudaMemcpyHostToDevice, c->stream);
  }
  if (!e) e = vt::launch_build_tile_items(c->tiles, c->nbr, c->tile_items, c->tile_count, c->ntiles, c->nfq, c->stream);
  if (!e) e = cudaStreamSynchronize(c->stream);
  cudaFree(verts);
  if (dtab) cudaFree(dtab);
  if (e) {
    set(fail(e == cudaErrorMemoryAllocation ? VT_ERR_NO_MEMORY : VT_ERR_CUDA, vt::cuda_msg("vt_create_structured", e)));
    release(c);
    return nullptr;
  }
  set(VT_OK);
  return c;
}

void vt_destroy(vt_ctx* c) { release(c); }

int vt_upload_state_device(vt_ctx* c, const double* dU) {
  if (!c || !dU) return fail(VT_ERR_INVALID, "null argument");
  if (!vt::aligned_to(dU, 16)) return fail(VT_ERR_INVALID, "vt_upload_state_device: dU is not 16-byte aligned");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  cudaError_t e = aos_to_soa(c, dU, c->U);
  if (!e) e = cudaStreamSynchronize(c->stream);
  return e ? fail(VT_ERR_CUDA, vt::cuda_msg("upload", e)) : VT_OK;
}

int vt_upload_state(vt_ctx* c, const double* U) {
  if (!c || !U) return fail(VT_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  int st = ensure_aos(c);
  if (st) return st;
  cudaError_t e = cudaMemcpyAsync(c->aos, U, sizeof(double) * 4 * static_cast<size_t>(c->K) * c->Np,
                                  cudaMemcpyHostToDevice, c->stream);
  if (!e) e = aos_to_soa(c, reinterpret_cast<const double*>(c->aos), c->U);
  if (!e) e = cudaStreamSynchronize(c->stream);
  return e ? fail(VT_ERR_CUDA, vt::cuda_msg("upload", e)) : VT_OK;
}

int vt_download_state_device(vt_ctx* c, double* dU) {
  if (!c || !dU) return fail(VT_ERR_INVALID, "null argument");
  if (!vt::aligned_to(dU, 16)) return fail(VT_ERR_INVALID, "vt_download_state_device: dU is not 16-byte aligned");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  cudaError_t e = soa_to_aos(c, c->U, dU);
  if (!e) e = cudaStreamSynchronize(c->stream);
  return e ? fail(VT_ERR_CUDA, vt::cuda_msg("download", e)) : VT_OK;
}

int vt_download_state(vt_ctx* c, double* U, double* F) {
  if (!c || !U) return fail(VT_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  int st = ensure_aos(c);
  if (st) return st;
  cudaError_t e = soa_to_aos(c, c->U, reinterpret_cast<double*>(c->aos));
  if (!e)
    e = cudaMemcpyAsync(U, c->aos, sizeof(double) * 4 * static_cast<size_t>(c->K) * c->Np,
                        cudaMemcpyDeviceToHost, c->stream);
  if (!e) e = cudaStreamSynchronize(c->stream);
  if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("download", e));
  if (F) vt::flux_from_state(c->K, c->Np, U, F);
  return VT_OK;
}

static int rk4_enqueue(vt_ctx* c, double dt, int nsteps) {
  cudaError_t e = reset_error_words(c);
  if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("reset", e));
  if (!c->rk4_graph || c->rk4_graph_dt != dt) {
    if (c->rk4_graph) {
      cudaGraphExecDestroy(c->rk4_graph);
      c->rk4_graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    if (!e) {
      const cudaError_t le = enqueue_rk4_step(c, dt);
      e = cudaStreamEndCapture(c->stream, &g);
      if (le) e = le;
    }
    if (!e) e = cudaGraphInstantiate(&c->rk4_graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("graph capture", e));
    c->rk4_graph_dt = dt;
  }
  for (int s = 0; s < nsteps; ++s)
    if ((e = cudaGraphLaunch(c->rk4_graph, c->stream))) return fail(VT_ERR_CUDA, vt::cuda_msg("graph launch", e));
  c->pending_steps += nsteps;
  c->pending_dt = dt;
  return VT_OK;
}

int vt_step_rk4_async(vt_ctx* c, double dt, int nsteps) {
  if (!c || nsteps < 0) return fail(VT_ERR_INVALID, "bad argument");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (c->pending_steps) return fail(VT_ERR_INVALID, "a previous async step is not synchronised");
  return rk4_enqueue(c, dt, nsteps);
}

int vt_synchronize(vt_ctx* c) {
  if (!c) return fail(VT_ERR_INVALID, "null context");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  const int n = c->pending_steps;
  c->pending_steps = 0;
  return finish(c, n, c->pending_dt);
}

int vt_step_rk4(vt_ctx* c, double dt, int nsteps) {
  if (!c || nsteps < 0) return fail(VT_ERR_INVALID, "bad argument");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (c->pending_steps) return fail(VT_ERR_INVALID, "a previous async step is not synchronised");
  int st = rk4_enqueue(c, dt, nsteps);
  if (st) return st;
  c->pending_steps = 0;
  return finish(c, nsteps, dt);
}

int vt_step_euler(vt_ctx* c, double dt, int nsteps) {
  if (!c || nsteps < 0) return fail(VT_ERR_INVALID, "bad argument");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (c->pending_steps) return fail(VT_ERR_INVALID, "a previous async step is not synchronised");
  cudaError_t e = reset_error_words(c);
  for (int s = 0; s < nsteps && !e; ++s) {
    // double buffer: the neighbours of an element read the old state
    e = c->launch(stage_args(c, c->U, c->U, c->A, c->Sa, vt::kStageEuler, 0.0, dt), c->ops.data(),
                  c->max_blocks, c->stream);
    std::swap(c->U, c->Sa);
  }
  if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("euler", e));
  // the RK4 graph captured the old buffer roles
  if (nsteps % 2 && c->rk4_graph) {
    cudaGraphExecDestroy(c->rk4_graph);
    c->rk4_graph = nullptr;
  }
  return finish(c, nsteps, dt);
}

int vt_rhs(vt_ctx* c, double* Udot) {
  if (!c || !Udot) return fail(VT_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  int st = ensure_aos(c);
  if (st) return st;
  cudaError_t e = cudaSuccess;
  if (!c->R) e = alloc(&c->R, sizeof(double2) * 2 * c->Np * static_cast<size_t>(c->Kpad));
  if (!e) e = reset_error_words(c);
  if (!e)
    e = c->launch(stage_args(c, c->U, c->U, c->A, c->R, vt::kStageRhs, 0.0, 0.0), c->ops.data(),
                  c->max_blocks, c->stream);
  if (!e) e = soa_to_aos(c, c->R, reinterpret_cast<double*>(c->aos));
  if (!e)
    e = cudaMemcpyAsync(Udot, c->aos, sizeof(double) * 4 * static_cast<size_t>(c->K) * c->Np,
                        cudaMemcpyDeviceToHost, c->stream);
  if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("rhs", e));
  return finish(c, 0, 0.0);
}

int vt_last_error(const vt_ctx* c, vt_error_info* out) {
  if (!c || !out) return fail(VT_ERR_INVALID, "null argument");
  *out = c->last;
  return VT_OK;
}

double vt_get_time(const vt_ctx* c) { return c ? c->time : 0.0; }

int vt_set_time(vt_ctx* c, double t) {
  if (!c) return fail(VT_ERR_INVALID, "null context");
  c->time = t;
  return VT_OK;
}

int vt_totals(vt_ctx* c, double* out) {
  if (!c || !out) return fail(VT_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  const int blocks = (c->K + 255) / 256;
  vt::totals_partial_kernel<<<blocks, 256, 0, c->stream>>>(c->U, c->geo, c->W, c->K, c->Np, c->Kpad, c->partial);
  vt::totals_final_kernel<<<1, 256, 0, c->stream>>>(c->partial, blocks, c->tot);
  cudaError_t e = cudaGetLastError();
  if (!e) e = cudaMemcpyAsync(out, c->tot, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (!e) e = cudaStreamSynchronize(c->stream);
  return e ? fail(VT_ERR_CUDA, vt::cuda_msg("totals", e)) : VT_OK;
}

int vt_l2_error(vt_ctx* c, int nq, const double* area_quad, const double* U_ref, int device_pointers, double* out) {
  if (!c || nq < 1 || !area_quad || !U_ref || !out) return fail(VT_ERR_INVALID, "vt_l2_error: bad argument");
  if (device_pointers && !vt::aligned_to(U_ref, 16))
    return fail(VT_ERR_INVALID, "vt_l2_error: the device array U_ref is not 16-byte aligned");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  const int Np = c->Np;
  std::vector<double> tab(static_cast<size_t>(nq) * (Np + 1));
  for (int q = 0; q < nq; ++q) {
    vt::basis(c->p, area_quad[3 * q], area_quad[3 * q + 1], &tab[static_cast<size_t>(q) * Np]);
    tab[static_cast<size_t>(nq) * Np + q] = area_quad[3 * q + 2];
  }
  double* dtab = nullptr;
  cudaError_t e = alloc(&dtab, sizeof(double) * tab.size());
  if (!e) e = cudaMemcpyAsync(dtab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, c->stream);
  if (!e && !device_pointers) {
    const int st = ensure_aos(c);
    if (st) {
      cudaFree(dtab);
      return st;
    }
    e = cudaMemcpyAsync(c->aos, U_ref, sizeof(double) * 4 * static_cast<size_t>(c->K) * Np, cudaMemcpyHostToDevice,
                        c->stream);
  }
  if (!e) e = aos_to_soa(c, device_pointers ? U_ref : reinterpret_cast<const double*>(c->aos), c->Sa);
  const int blocks = (c->K + 255) / 256;
  if (!e) {
    vt::l2_partial_kernel<<<blocks, 256, 0, c->stream>>>(c->U, c->Sa, c->geo, dtab, dtab + static_cast<size_t>(nq) * Np,
                                                          nq, c->K, Np, c->Kpad, c->partial);
    vt::totals_final_kernel<<<1, 256, 0, c->stream>>>(c->partial, blocks, c->tot);
    e = cudaGetLastError();
  }
  double tot[4] = {0, 0, 0, 0};
  if (!e) e = cudaMemcpyAsync(tot, c->tot, sizeof(tot), cudaMemcpyDeviceToHost, c->stream);
  if (!e) e = cudaStreamSynchronize(c->stream);
  if (dtab) cudaFree(dtab);
  if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("l2 error", e));
  for (int k = 0; k < 4; ++k) out[k] = std::sqrt((1.0 / 25.0) * tot[k]);
  return VT_OK;
}

int vt_project_vortex(vt_ctx* c, const double* vertices, const vt_vortex* ic, double t, int nq,
                      const double* area_quad) {
  if (!c || !vertices || !ic || nq < 1 || !area_quad) return fail(VT_ERR_INVALID, "vt_project_vortex: bad argument");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  const int Np = c->Np;
  std::vector<double> tab(static_cast<size_t>(nq) * (Np + 3) + Np * Np);
  for (int q = 0; q < nq; ++q) {
    vt::basis(c->p, area_quad[3 * q], area_quad[3 * q + 1], &tab[static_cast<size_t>(q) * Np]);
    tab[static_cast<size_t>(nq) * Np + q] = area_quad[3 * q + 2];
    tab[static_cast<size_t>(nq) * (Np + 1) + 2 * q] = area_quad[3 * q];
    tab[static_cast<size_t>(nq) * (Np + 1) + 2 * q + 1] = area_quad[3 * q + 1];
  }
  std::copy(c->minv_ref.begin(), c->minv_ref.end(), tab.begin() + static_cast<size_t>(nq) * (Np + 3));
  double *dtab = nullptr, *dverts = nullptr;
  const size_t vbytes = sizeof(double) * 6 * static_cast<size_t>(c->K);
  cudaError_t e = alloc(&dtab, sizeof(double) * tab.size());
  if (!e) e = alloc(&dverts, vbytes);
  if (!e) e = cudaMemcpyAsync(dtab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, c->stream);
  if (!e) e = cudaMemcpyAsync(dverts, vertices, vbytes, cudaMemcpyHostToDevice, c->stream);
  if (!e) {
    vt::project_vortex_kernel<<<(c->K + 127) / 128, 128, 0, c->stream>>>(dverts, c->geo, dtab, nq, *ic, t, c->K, Np,
                                                                        c->Kpad, c->U);
    e = cudaGetLastError();
  }
  if (!e) e = cudaStreamSynchronize(c->stream);
  if (dtab) cudaFree(dtab);
  if (dverts) cudaFree(dverts);
  return e ? fail(VT_ERR_CUDA, vt::cuda_msg("project vortex", e)) : VT_OK;
}

int vt_save_state(vt_ctx* c, const char* path) {
  if (!c || !path) return fail(VT_ERR_INVALID, "vt_save_state: null argument");
  std::vector<double> U(4 * static_cast<size_t>(c->K) * c->Np);
  const int st = vt_download_state(c, U.data(), nullptr);
  return st ? st : vt_write_state_file(path, c->p, c->K, c->time, U.data());
}

int vt_load_state(vt_ctx* c, const char* path) {
  if (!c || !path) return fail(VT_ERR_INVALID, "vt_load_state: null argument");
  int p = 0, K = 0;
  double t = 0.0;
  int st = vt_state_file_info(path, &p, &K, &t);
  if (st) return st;
  if (p != c->p || K != c->K)
    return fail(VT_ERR_INVALID, "vt_load_state: the file holds p=" + std::to_string(p) + ", K=" + std::to_string(K) +
                                    ", the context p=" + std::to_string(c->p) + ", K=" + std::to_string(c->K));
  std::vector<double> U(4 * static_cast<size_t>(K) * c->Np);
  if ((st = vt_read_state_file(path, U.data()))) return st;
  if ((st = vt_upload_state(c, U.data()))) return st;
  c->time = t;
  return VT_OK;
}

void* vt_stream(vt_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

int vt_set_stage_mapping(vt_ctx* c, int mapping) {
  if (!c || (mapping != vt::kMapComponent && mapping != vt::kMapPair))
    return fail(VT_ERR_INVALID, "vt_set_stage_mapping: mapping must be 0 (component) or 1 (pair)");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  const vt::StageKernel sk = vt::select_kernel(c->p, c->nfq, mapping);
  int per_sm = 0, sms = 0;
  cudaError_t e = sk.configure(&per_sm);
  if (!e) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("vt_set_stage_mapping", e));
  c->launch = sk.launch;
  c->map = mapping;
  c->max_blocks = sms * (per_sm > 0 ? per_sm : 1);
  if (c->rk4_graph) {  // the captured step holds the old kernel
    cudaGraphExecDestroy(c->rk4_graph);
    c->rk4_graph = nullptr;
  }
  vt::adjoint_invalidate_graphs(c);
  return VT_OK;
}

int vt_get_stage_mapping(const vt_ctx* c) { return c ? c->map : -1; }

int vt_test_bulk_wait(vt_ctx* c, unsigned tries, int issue_no_copies) {
  if (!c) return fail(VT_ERR_INVALID, "vt_test_bulk_wait: null context");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->test_wait_tries = tries;
  c->test_flags = issue_no_copies ? vt::kTestNoCopies : 0;
  if (c->rk4_graph) {  // the captured step holds the old kernel arguments
    cudaGraphExecDestroy(c->rk4_graph);
    c->rk4_graph = nullptr;
  }
  return VT_OK;
}

int vt_profile_rk4_stages(vt_ctx* c, double dt, int reps, float* ms) {
  if (!c || !ms || reps < 1) return fail(VT_ERR_INVALID, "bad argument");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  cudaEvent_t ev[5];
  for (auto& x : ev) cudaEventCreate(&x);
  double acc[4] = {0, 0, 0, 0};
  cudaError_t e = reset_error_words(c);
  const double* ops = c->ops.data();
  for (int r = 0; r < reps && !e; ++r) {
    const vt::StageArgs args[4] = {stage_args(c, c->U, c->U, c->A, c->Sa, 0, (1.0 / 6) * dt, 0.5 * dt),
                                   stage_args(c, c->Sa, c->U, c->A, c->Sb, 1, (1.0 / 3) * dt, 0.5 * dt),
                                   stage_args(c, c->Sb, c->U, c->A, c->Sa, 2, (1.0 / 3) * dt, dt),
                                   stage_args(c, c->Sa, c->U, c->A, c->U, 3, 0.0, (1.0 / 6) * dt)};
    cudaEventRecord(ev[0], c->stream);
    for (int s = 0; s < 4 && !e; ++s) {
      e = c->launch(args[s], ops, c->max_blocks, c->stream);
      cudaEventRecord(ev[s + 1], c->stream);
    }
    if (!e) e = cudaEventSynchronize(ev[4]);
    for (int s = 0; s < 4 && !e; ++s) {
      float t = 0;
      cudaEventElapsedTime(&t, ev[s], ev[s + 1]);
      acc[s] += t;
    }
  }
  for (auto& x : ev) cudaEventDestroy(x);
  if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("profile", e));
  for (int s = 0; s < 4; ++s) ms[s] = static_cast<float>(acc[s] / reps);
  return finish(c, reps, dt);
}

}  // extern "C"
