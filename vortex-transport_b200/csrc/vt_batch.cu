// Batched ensemble: many independent vortex problems advanced together
// (vt_batch_* in include/vortex_b200.h). The reference runs one problem per
// process; this has no reference counterpart beyond the per-problem stepper.
//
// Instances with the same polynomial order and the same reference operators
// (p, line rule, mass/stiffness tables) form a group. A group is one ragged
// element array: the instances' elements are concatenated, their neighbour ids
// shifted by the instance's offset, and their tiles (the same tiles a single
// instance would get, so the arithmetic per element is identical) listed one
// after another, each tile carrying its instance's time step. One launch of the
// stage kernel per group and stage advances every instance of the group; one
// CUDA graph holds a whole RK4 step of all groups.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/vortex_b200.h"
#include "vt_common.h"
#include "vt_ctx.h"
#include "vt_launch.h"
#include "vt_precompute.h"

namespace vt {
namespace {

template <typename T>
cudaError_t dalloc(T** p, size_t bytes) {
  return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}

// instance AoS (K_i x Np x 4) <-> group SoA rows at an element offset
__global__ void batch_aos_to_soa(const double2* __restrict__ aos, double2* __restrict__ soa, int K, int Np,
                                 long long Kpad, long long offset) {
  const long long l = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (l >= static_cast<long long>(K) * 2 * Np) return;
  const int e = static_cast<int>(l / (2 * Np)), r = static_cast<int>(l % (2 * Np));
  soa[r * Kpad + offset + e] = aos[l];
}

__global__ void batch_soa_to_aos(const double2* __restrict__ soa, double2* __restrict__ aos, int K, int Np,
                                 long long Kpad, long long offset) {
  const long long l = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (l >= static_cast<long long>(K) * 2 * Np) return;
  const int e = static_cast<int>(l / (2 * Np)), r = static_cast<int>(l % (2 * Np));
  aos[l] = soa[r * Kpad + offset + e];
}

std::vector<double> fold(int p, int nfq, const vt_mesh_desc& d) {
  std::vector<double> ops(static_cast<size_t>(stage_ops_doubles(p, nfq)));
  fold_stage_operators(p, nfq, d.inv_mass_ref, d.stiffness_ref, d.line_quadrature, d.phi_plus, d.phi_minus,
                       ops.data());
  return ops;
}

// the reference-space tables that decide which group an instance joins
std::vector<double> table_key(const vt_mesh_desc& d) {
  const int Np = np_of(d.p), nfq = d.n_line_points;
  std::vector<double> k;
  k.insert(k.end(), d.inv_mass_ref, d.inv_mass_ref + Np * Np);
  k.insert(k.end(), d.stiffness_ref, d.stiffness_ref + 2 * Np * Np);
  k.insert(k.end(), d.line_quadrature, d.line_quadrature + 2 * nfq);
  k.insert(k.end(), d.phi_plus, d.phi_plus + 3 * Np * nfq);
  k.insert(k.end(), d.phi_minus, d.phi_minus + 3 * Np * nfq);
  return k;
}

struct Group {
  int p = 0, nfq = 0, Np = 0;
  long long K = 0, Kpad = 0;
  int ntiles = 0;
  std::vector<int> members;
  std::vector<long long> offset;  // element offset of each member
  std::vector<int> tile_begin;    // first tile of each member
  std::vector<double> ops;
  StageKernel kern;
  int max_blocks = 0;
  double2 *U = nullptr, *A = nullptr, *Sa = nullptr, *Sb = nullptr, *geo = nullptr;
  int4 *nbr = nullptr, *tiles = nullptr;
  int *items = nullptr, *count = nullptr;
  double* tile_dt = nullptr;
  unsigned long long* err = nullptr;
};

}  // namespace
}  // namespace vt

struct vt_batch {
  std::mutex mu;
  int device = 0;
  int n = 0;
  cudaStream_t stream = nullptr;
  std::vector<vt::Group> groups;
  std::vector<int> group_of, index_in_group, K_of;
  double2* staging = nullptr;  // largest instance, AoS
  size_t staging_bytes = 0;
  cudaGraphExec_t graph = nullptr;
  // one stream per group: the groups' stage chains are independent and run as
  // concurrent branches of the step graph, so one group's wave tail overlaps
  // the next group's work
  std::vector<cudaStream_t> gstreams;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  int sms = 0, per_sm = 0;
  std::vector<double> dt;  // per instance
  int last_instance = -1;
  vt_error_info last{};
  // one solver context per group over the group's own buffers, for the adjoint,
  // with each group's per-element time steps
  std::vector<vt_ctx*> views;
  std::vector<double*> view_dt;
};

namespace {

using vt::fail;

void release(vt_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  for (vt_ctx* v : b->views) {
    vt::adjoint_release(v);
    if (v->aos) cudaFree(v->aos);
    delete v;
  }
  for (double* p : b->view_dt)
    if (p) cudaFree(p);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (cudaStream_t st : b->gstreams)
    if (st) cudaStreamDestroy(st);
  for (cudaEvent_t ev : b->join)
    if (ev) cudaEventDestroy(ev);
  if (b->fork) cudaEventDestroy(b->fork);
  for (auto& g : b->groups) {
    void* bufs[] = {g.U, g.A, g.Sa, g.Sb, g.geo, g.nbr, g.tiles, g.items, g.count, g.tile_dt, g.err};
    for (void* p : bufs)
      if (p) cudaFree(p);
  }
  if (b->staging) cudaFree(b->staging);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

vt::StageArgs group_args(vt::Group& g, const double2* in, double2* out, int stage, double k_acc, double k_out) {
  vt::StageArgs a;
  a.in = in;
  a.base = g.U;
  a.acc = g.A;
  a.out = out;
  a.geo = g.geo;
  a.nbr = g.nbr;
  a.tiles = g.tiles;
  a.tile_items = g.items;
  a.tile_count = g.count;
  a.tile_dt = g.tile_dt;
  a.err = g.err;
  a.Kpad = g.Kpad;
  a.K = static_cast<int>(g.K);
  a.ntiles = g.ntiles;
  a.stage = stage;
  a.c_acc = k_acc;
  a.c_out = k_out;
  return a;
}

// The four stage launches of one RK4 step of group g on stream st; the
// coefficients are fractions of each tile's dt.
cudaError_t enqueue_group_step(vt::Group& g, cudaStream_t st) {
  const double* ops = g.ops.data();
  cudaError_t e = g.kern.launch(group_args(g, g.U, g.Sa, 0, 1.0 / 6, 0.5), ops, g.max_blocks, st);
  if (!e) e = g.kern.launch(group_args(g, g.Sa, g.Sb, 1, 1.0 / 3, 0.5), ops, g.max_blocks, st);
  if (!e) e = g.kern.launch(group_args(g, g.Sb, g.Sa, 2, 1.0 / 3, 1.0), ops, g.max_blocks, st);
  if (!e) e = g.kern.launch(group_args(g, g.Sa, g.U, 3, 0.0, 1.0 / 6), ops, g.max_blocks, st);
  return e;
}

// One RK4 step of every group. The groups are independent problems: each
// group's chain of four stages runs on its own stream, forked from and joined
// back into the batch stream, so that in the captured graph they are parallel
// branches and the GPU starts one group's blocks while another group's last
// tiles finish.
cudaError_t enqueue_step(vt_batch* b) {
  if (b->groups.size() == 1) return enqueue_group_step(b->groups[0], b->stream);
  cudaError_t e = cudaEventRecord(b->fork, b->stream);
  for (size_t gi = 0; gi < b->groups.size() && !e; ++gi) {
    e = cudaStreamWaitEvent(b->gstreams[gi], b->fork, 0);
    if (!e) e = enqueue_group_step(b->groups[gi], b->gstreams[gi]);
    if (!e) e = cudaEventRecord(b->join[gi], b->gstreams[gi]);
  }
  for (size_t gi = 0; gi < b->groups.size() && !e; ++gi) e = cudaStreamWaitEvent(b->stream, b->join[gi], 0);
  return e;
}

cudaError_t reset_errors(vt_batch* b) {
  cudaError_t e = cudaSuccess;
  for (auto& g : b->groups) {
    if (!e) e = cudaMemsetAsync(g.err, 0xFF, sizeof(unsigned long long), b->stream);
    if (!e) e = cudaMemsetAsync(g.err + 1, 0, 3 * sizeof(unsigned long long), b->stream);
  }
  return e;
}

int capture(vt_batch* b) {
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  cudaGraph_t gr = nullptr;
  cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
  if (!e) {
    const cudaError_t le = enqueue_step(b);
    e = cudaStreamEndCapture(b->stream, &gr);
    if (le) e = le;
  }
  if (!e) e = cudaGraphInstantiate(&b->graph, gr, 0);
  if (gr) cudaGraphDestroy(gr);
  return e ? fail(VT_ERR_CUDA, vt::cuda_msg("batch graph", e)) : VT_OK;
}

int upload_dt(vt_batch* b) {
  for (auto& g : b->groups) {
    std::vector<double> tdt(g.ntiles);
    for (size_t m = 0; m < g.members.size(); ++m) {
      const int end = m + 1 < g.members.size() ? g.tile_begin[m + 1] : g.ntiles;
      for (int t = g.tile_begin[m]; t < end; ++t) tdt[t] = b->dt[g.members[m]];
    }
    cudaError_t e =
        cudaMemcpyAsync(g.tile_dt, tdt.data(), sizeof(double) * g.ntiles, cudaMemcpyHostToDevice, b->stream);
    if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("batch dt", e));
    if ((e = cudaStreamSynchronize(b->stream))) return fail(VT_ERR_CUDA, vt::cuda_msg("batch dt", e));
  }
  return VT_OK;
}

// A vt_ctx over a group's buffers (not owning them), so the single-problem
// adjoint runs on the group's ragged element array: one launch per stage for
// all its instances. The group's tiles and face lists are the ones the batch
// steps with; the time step is uniform within the group.
int ensure_views(vt_batch* b) {
  if (b->views.size() == b->groups.size()) return VT_OK;
  for (size_t gi = b->views.size(); gi < b->groups.size(); ++gi) {
    vt::Group& G = b->groups[gi];
    auto* c = new vt_ctx();
    c->device = b->device;
    c->p = G.p;
    c->Np = G.Np;
    c->nfq = G.nfq;
    c->K = static_cast<int>(G.K);
    c->Kpad = G.Kpad;
    c->max_blocks = G.max_blocks;
    c->stream = b->stream;
    c->U = G.U;
    c->A = G.A;
    c->Sa = G.Sa;
    c->Sb = G.Sb;
    c->geo = G.geo;
    c->nbr = G.nbr;
    c->tiles = G.tiles;
    c->tile_items = G.items;
    c->tile_count = G.count;
    c->ntiles = G.ntiles;
    c->err = G.err;
    c->ops = G.ops;
    c->launch = G.kern.launch;
    c->map = G.kern.map;
    c->tile_dt = G.tile_dt;
    double* edt = nullptr;
    const cudaError_t ea = cudaMalloc(reinterpret_cast<void**>(&edt), sizeof(double) * static_cast<size_t>(G.K));
    if (ea) {
      delete c;
      return fail(ea == cudaErrorMemoryAllocation ? VT_ERR_NO_MEMORY : VT_ERR_CUDA,
                  vt::cuda_msg("batch adjoint set-up", ea));
    }
    c->elem_dt = edt;
    b->view_dt.push_back(edt);
    std::vector<int4> nb(static_cast<size_t>(G.K));
    const cudaError_t e = cudaMemcpy(nb.data(), G.nbr, sizeof(int4) * nb.size(), cudaMemcpyDeviceToHost);
    if (e) {
      delete c;
      return fail(VT_ERR_CUDA, vt::cuda_msg("batch adjoint set-up", e));
    }
    c->side_pairing = true;
    for (size_t n = 0; n < nb.size() && c->side_pairing; ++n)
      c->side_pairing = nb[nb[n].x].x == static_cast<int>(n) && nb[nb[n].y].y == static_cast<int>(n) &&
                        nb[nb[n].z].z == static_cast<int>(n);
    b->views.push_back(c);
  }
  return VT_OK;
}

}  // namespace

extern "C" {

vt_batch* vt_batch_create(const vt_mesh_desc* descs, int n, int device, int* status) {
  auto set = [&](int s) {
    if (status) *status = s;
  };
  if (!descs || n < 1) {
    set(fail(VT_ERR_INVALID, "vt_batch_create: no instances"));
    return nullptr;
  }
  for (int i = 0; i < n; ++i) {
    const vt_mesh_desc& d = descs[i];
    if (!d.element_type || !d.neighbours || !d.det_jacobian || !d.inv_jacobian || !d.normals ||
        !d.side_lengths || !d.inv_mass_ref || !d.stiffness_ref || !d.line_quadrature || !d.phi_plus ||
        !d.phi_minus || d.n_elements < 1) {
      set(fail(VT_ERR_INVALID, "vt_batch_create: incomplete descriptor for instance " + std::to_string(i)));
      return nullptr;
    }
    if (d.p < 0 || d.p > 3 || d.n_line_points < 1 || d.n_line_points > 10) {
      set(fail(VT_ERR_UNSUPPORTED, "vt_batch_create: p or n_line_points out of range"));
      return nullptr;
    }
    for (int k = 0; k < 3 * d.n_elements; ++k)
      if (d.neighbours[k] < 0 || d.neighbours[k] >= d.n_elements) {
        set(fail(VT_ERR_INVALID, "vt_batch_create: neighbour out of range in instance " + std::to_string(i)));
        return nullptr;
      }
  }
  cudaError_t e = cudaSetDevice(device);
  if (e) {
    set(fail(VT_ERR_CUDA, vt::cuda_msg("cudaSetDevice", e)));
    return nullptr;
  }
  auto* b = new vt_batch();
  b->device = device;
  b->n = n;
  b->group_of.assign(n, -1);
  b->index_in_group.assign(n, -1);
  b->K_of.assign(n, 0);
  b->dt.assign(n, 0.0);
  // group instances by (p, nfq, reference tables)
  std::map<std::pair<std::pair<int, int>, std::vector<double>>, int> gid;
  for (int i = 0; i < n; ++i) {
    const vt_mesh_desc& d = descs[i];
    auto key = std::make_pair(std::make_pair(d.p, d.n_line_points), vt::table_key(d));
    auto it = gid.find(key);
    int g;
    if (it == gid.end()) {
      g = static_cast<int>(b->groups.size());
      gid.emplace(key, g);
      b->groups.emplace_back();
      vt::Group& G = b->groups.back();
      G.p = d.p;
      G.nfq = d.n_line_points;
      G.Np = vt::np_of(d.p);
      G.ops = vt::fold(d.p, d.n_line_points, d);
    } else {
      g = it->second;
    }
    vt::Group& G = b->groups[g];
    b->group_of[i] = g;
    b->index_in_group[i] = static_cast<int>(G.members.size());
    b->K_of[i] = d.n_elements;
    G.members.push_back(i);
    G.offset.push_back(G.K);
    G.K += d.n_elements;
  }
  if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) ||
      (e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device)) ||
      (e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming))) {
    set(fail(VT_ERR_CUDA, vt::cuda_msg("vt_batch_create", e)));
    release(b);
    return nullptr;
  }
  b->gstreams.assign(b->groups.size(), nullptr);
  b->join.assign(b->groups.size(), nullptr);
  for (size_t gi = 0; gi < b->groups.size() && !e; ++gi) {
    e = cudaStreamCreateWithFlags(&b->gstreams[gi], cudaStreamNonBlocking);
    if (!e) e = cudaEventCreateWithFlags(&b->join[gi], cudaEventDisableTiming);
  }
  if (e) {
    set(fail(VT_ERR_CUDA, vt::cuda_msg("vt_batch_create streams", e)));
    release(b);
    return nullptr;
  }
  size_t max_inst_bytes = 0;
  for (auto& G : b->groups) {
    G.kern = vt::select_kernel(G.p, G.nfq);
    int per_sm = 0;
    if ((e = vt::tensor_maps_available()) || (e = G.kern.configure(&per_sm))) {
      set(fail(VT_ERR_CUDA, vt::cuda_msg("stage kernel attributes", e)));
      release(b);
      return nullptr;
    }
    G.max_blocks = b->sms * (per_sm > 0 ? per_sm : 1);
    G.Kpad = (G.K + 127) / 128 * 128;
    const long long KP = G.Kpad;
    // packed geometry, shifted neighbours and per-member tiles
    std::vector<double2> geo(7 * static_cast<size_t>(KP), make_double2(0.0, 0.0));
    std::vector<int4> nbr(static_cast<size_t>(KP), make_int4(0, 0, 0, 0));
    std::vector<int4> tiles;
    for (size_t m = 0; m < G.members.size(); ++m) {
      const vt_mesh_desc& d = descs[G.members[m]];
      const int off = static_cast<int>(G.offset[m]);
      max_inst_bytes = std::max(max_inst_bytes, sizeof(double) * 4 * static_cast<size_t>(d.n_elements) * G.Np);
      for (int k = 0; k < d.n_elements; ++k) {
        const long long n_ = off + k;
        const double* ji = d.inv_jacobian + 4 * static_cast<size_t>(k);
        const double* nv = d.normals + 6 * static_cast<size_t>(k);
        const double* ln = d.side_lengths + 3 * static_cast<size_t>(k);
        const double det = d.det_jacobian[k];
        geo[0 * KP + n_] = make_double2(ji[0], ji[1]);
        geo[1 * KP + n_] = make_double2(ji[2], ji[3]);
        for (int s = 0; s < 3; ++s) geo[(2 + s) * KP + n_] = make_double2(nv[2 * s], nv[2 * s + 1]);
        geo[5 * KP + n_] = make_double2(ln[0] / det, ln[1] / det);
        geo[6 * KP + n_] = make_double2(ln[2] / det, det);
        const int right = d.neighbours[3 * k] + off, left = d.neighbours[3 * k + 1] + off,
                  vert = d.neighbours[3 * k + 2] + off;
        nbr[n_] = d.element_type[k] == 0 ? make_int4(vert, right, left, 0) : make_int4(vert, left, right, 0);
      }
      G.tile_begin.push_back(static_cast<int>(tiles.size()));
      std::vector<int4> runs = vt::structured_tile_runs(d.n_elements, d.element_type, d.neighbours);
      if (runs.empty())
        for (int s0 = 0; s0 < d.n_elements; s0 += vt::kTileElems) {
          const int l0 = std::min(vt::kTileRun, d.n_elements - s0);
          const int l1 = std::max(0, std::min(vt::kTileRun, d.n_elements - s0 - vt::kTileRun));
          runs.push_back(make_int4(s0, l0, s0 + vt::kTileRun, l1));
        }
      for (const int4& r : runs) tiles.push_back(make_int4(r.x + off, r.y, r.z + off, r.w));
    }
    G.ntiles = static_cast<int>(tiles.size());
    const size_t state_bytes = sizeof(double2) * 2 * G.Np * static_cast<size_t>(KP);
    if ((e = vt::dalloc(&G.U, state_bytes)) || (e = vt::dalloc(&G.A, state_bytes)) ||
        (e = vt::dalloc(&G.Sa, state_bytes)) || (e = vt::dalloc(&G.Sb, state_bytes)) ||
        (e = vt::dalloc(&G.geo, geo.size() * sizeof(double2))) || (e = vt::dalloc(&G.nbr, nbr.size() * sizeof(int4))) ||
        (e = vt::dalloc(&G.tiles, tiles.size() * sizeof(int4))) ||
        (e = vt::dalloc(&G.items, sizeof(int) * vt::kMaxItems * tiles.size())) ||
        (e = vt::dalloc(&G.count, sizeof(int) * tiles.size())) ||
        (e = vt::dalloc(&G.tile_dt, sizeof(double) * tiles.size())) ||
        (e = vt::dalloc(&G.err, 4 * sizeof(unsigned long long)))) {
      set(fail(e == cudaErrorMemoryAllocation ? VT_ERR_NO_MEMORY : VT_ERR_CUDA, vt::cuda_msg("vt_batch_create", e)));
      release(b);
      return nullptr;
    }
    if ((e = cudaMemcpy(G.geo, geo.data(), geo.size() * sizeof(double2), cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(G.nbr, nbr.data(), nbr.size() * sizeof(int4), cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(G.tiles, tiles.data(), tiles.size() * sizeof(int4), cudaMemcpyHostToDevice)) ||
        (e = cudaMemset(G.U, 0, state_bytes)) || (e = cudaMemset(G.A, 0, state_bytes)) ||
        (e = cudaMemset(G.Sa, 0, state_bytes)) || (e = cudaMemset(G.Sb, 0, state_bytes)) ||
        (e = cudaMemset(G.tile_dt, 0, sizeof(double) * tiles.size())) ||
        (e = vt::launch_build_tile_items(G.tiles, G.nbr, G.items, G.count, G.ntiles, G.nfq, b->stream)) ||
        (e = cudaStreamSynchronize(b->stream))) {
      set(fail(VT_ERR_CUDA, vt::cuda_msg("vt_batch_create upload", e)));
      release(b);
      return nullptr;
    }
  }
  if ((e = vt::dalloc(&b->staging, max_inst_bytes))) {
    set(fail(VT_ERR_NO_MEMORY, vt::cuda_msg("vt_batch_create staging", e)));
    release(b);
    return nullptr;
  }
  b->staging_bytes = max_inst_bytes;
  set(VT_OK);
  return b;
}

void vt_batch_destroy(vt_batch* b) { release(b); }

int vt_batch_size(const vt_batch* b) { return b ? b->n : 0; }

int vt_batch_groups(const vt_batch* b) { return b ? static_cast<int>(b->groups.size()) : 0; }

int vt_batch_upload_state(vt_batch* b, int i, const double* U) {
  if (!b || !U || i < 0 || i >= b->n) return fail(VT_ERR_INVALID, "vt_batch_upload_state: bad argument");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  vt::Group& G = b->groups[b->group_of[i]];
  const int K = b->K_of[i];
  const size_t bytes = sizeof(double) * 4 * static_cast<size_t>(K) * G.Np;
  cudaError_t e = cudaMemcpyAsync(b->staging, U, bytes, cudaMemcpyHostToDevice, b->stream);
  const long long nrow = static_cast<long long>(K) * 2 * G.Np;
  if (!e) {
    vt::batch_aos_to_soa<<<static_cast<int>((nrow + 255) / 256), 256, 0, b->stream>>>(
        b->staging, G.U, K, G.Np, G.Kpad, G.offset[b->index_in_group[i]]);
    e = cudaGetLastError();
  }
  if (!e) e = cudaStreamSynchronize(b->stream);
  return e ? fail(VT_ERR_CUDA, vt::cuda_msg("vt_batch_upload_state", e)) : VT_OK;
}

int vt_batch_download_state(vt_batch* b, int i, double* U, double* F) {
  if (!b || !U || i < 0 || i >= b->n) return fail(VT_ERR_INVALID, "vt_batch_download_state: bad argument");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  vt::Group& G = b->groups[b->group_of[i]];
  const int K = b->K_of[i];
  const size_t bytes = sizeof(double) * 4 * static_cast<size_t>(K) * G.Np;
  const long long nrow = static_cast<long long>(K) * 2 * G.Np;
  vt::batch_soa_to_aos<<<static_cast<int>((nrow + 255) / 256), 256, 0, b->stream>>>(
      G.U, b->staging, K, G.Np, G.Kpad, G.offset[b->index_in_group[i]]);
  cudaError_t e = cudaGetLastError();
  if (!e) e = cudaMemcpyAsync(U, b->staging, bytes, cudaMemcpyDeviceToHost, b->stream);
  if (!e) e = cudaStreamSynchronize(b->stream);
  if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("vt_batch_download_state", e));
  if (F) vt::flux_from_state(K, G.Np, U, F);
  return VT_OK;
}

int vt_batch_upload_state_device(vt_batch* b, int i, const double* dU) {
  if (!b || !dU || i < 0 || i >= b->n) return fail(VT_ERR_INVALID, "vt_batch_upload_state_device: bad argument");
  if (!vt::aligned_to(dU, 16)) return fail(VT_ERR_INVALID, "vt_batch_upload_state_device: dU is not 16-byte aligned");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  vt::Group& G = b->groups[b->group_of[i]];
  const int K = b->K_of[i];
  const long long nrow = static_cast<long long>(K) * 2 * G.Np;
  vt::batch_aos_to_soa<<<static_cast<int>((nrow + 255) / 256), 256, 0, b->stream>>>(
      reinterpret_cast<const double2*>(dU), G.U, K, G.Np, G.Kpad, G.offset[b->index_in_group[i]]);
  cudaError_t e = cudaGetLastError();
  if (!e) e = cudaStreamSynchronize(b->stream);
  return e ? fail(VT_ERR_CUDA, vt::cuda_msg("vt_batch_upload_state_device", e)) : VT_OK;
}

int vt_batch_download_state_device(vt_batch* b, int i, double* dU) {
  if (!b || !dU || i < 0 || i >= b->n) return fail(VT_ERR_INVALID, "vt_batch_download_state_device: bad argument");
  if (!vt::aligned_to(dU, 16)) return fail(VT_ERR_INVALID, "vt_batch_download_state_device: dU is not 16-byte aligned");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  vt::Group& G = b->groups[b->group_of[i]];
  const int K = b->K_of[i];
  const long long nrow = static_cast<long long>(K) * 2 * G.Np;
  vt::batch_soa_to_aos<<<static_cast<int>((nrow + 255) / 256), 256, 0, b->stream>>>(
      G.U, reinterpret_cast<double2*>(dU), K, G.Np, G.Kpad, G.offset[b->index_in_group[i]]);
  cudaError_t e = cudaGetLastError();
  if (!e) e = cudaStreamSynchronize(b->stream);
  return e ? fail(VT_ERR_CUDA, vt::cuda_msg("vt_batch_download_state_device", e)) : VT_OK;
}

int vt_batch_set_dt(vt_batch* b, const double* dt) {
  if (!b || !dt) return fail(VT_ERR_INVALID, "vt_batch_set_dt: bad argument");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  b->dt.assign(dt, dt + b->n);
  return upload_dt(b);
}

int vt_batch_step_rk4(vt_batch* b, int nsteps) {
  if (!b || nsteps < 0) return fail(VT_ERR_INVALID, "vt_batch_step_rk4: bad argument");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  cudaError_t e = reset_errors(b);
  if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("batch reset", e));
  if (!b->graph) {
    const int st = capture(b);
    if (st) return st;
  }
  for (int s = 0; s < nsteps; ++s)
    if ((e = cudaGraphLaunch(b->graph, b->stream))) return fail(VT_ERR_CUDA, vt::cuda_msg("batch launch", e));
  if ((e = cudaStreamSynchronize(b->stream))) return fail(VT_ERR_CUDA, vt::cuda_msg("batch step", e));
  // first failure over groups: earliest stage, then instance order
  b->last = vt_error_info{};
  b->last_instance = -1;
  unsigned long long best_epoch = ~0ull;
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    vt::Group& G = b->groups[gi];
    unsigned long long w[4];
    if ((e = cudaMemcpy(w, G.err, sizeof(w), cudaMemcpyDeviceToHost))) return fail(VT_ERR_CUDA, "batch errors");
    if (w[3] & 2ull) return fail(VT_ERR_CUDA, "stage kernel: a bulk-copy wait gave up (the state is not valid)");
    if (w[0] == ~0ull) continue;
    const unsigned long long epoch = w[0] >> 40;
    vt_error_info info = vt::decode_error_key(w[0], G.nfq);
    const long long ge = info.element;  // element of the group's ragged array
    const size_t m = std::upper_bound(G.offset.begin(), G.offset.end(), ge) - G.offset.begin() - 1;
    info.element = static_cast<int>(ge - G.offset[m]);
    const int inst = G.members[m];
    if (epoch < best_epoch || (epoch == best_epoch && inst < b->last_instance)) {
      best_epoch = epoch;
      b->last = info;
      b->last_instance = inst;
    }
  }
  if (b->last_instance < 0) return VT_OK;
  return fail(b->last.code, "Non-physical state (code " + std::to_string(b->last.code) + ") in instance " +
                                std::to_string(b->last_instance) + " at element " + std::to_string(b->last.element));
}

int vt_batch_adjoint_forward(vt_batch* b, int nsteps, int nsnapshots) {
  if (!b || nsteps < 1 || nsnapshots < 1) return fail(VT_ERR_INVALID, "vt_batch_adjoint_forward: bad argument");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  int st = ensure_views(b);
  if (st) return st;
  b->last = vt_error_info{};
  b->last_instance = -1;
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    vt::Group& G = b->groups[gi];
    vt_ctx* c = b->views[gi];
    // each element steps with its instance's time step (the tiles already carry it)
    std::vector<double> edt(static_cast<size_t>(G.K));
    for (size_t m = 0; m < G.members.size(); ++m)
      std::fill(edt.begin() + G.offset[m], edt.begin() + G.offset[m] + b->K_of[G.members[m]], b->dt[G.members[m]]);
    cudaError_t e = cudaMemcpyAsync(b->view_dt[gi], edt.data(), sizeof(double) * edt.size(), cudaMemcpyHostToDevice,
                                    b->stream);
    if (!e) e = cudaStreamSynchronize(b->stream);
    if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("batch adjoint time steps", e));
    c->max_blocks = G.max_blocks;
    st = vt_adjoint_forward(c, 1.0, nsteps, nsnapshots);
    if (st > 0) {  // map the group element to its instance
      vt_error_info info{};
      vt_last_error(c, &info);
      const size_t m = std::upper_bound(G.offset.begin(), G.offset.end(), static_cast<long long>(info.element)) -
                       G.offset.begin() - 1;
      info.element -= static_cast<int>(G.offset[m]);
      b->last = info;
      b->last_instance = G.members[m];
      return fail(st, "Non-physical state (code " + std::to_string(st) + ") in instance " +
                          std::to_string(b->last_instance) + " at element " + std::to_string(info.element));
    }
    if (st) return st;
  }
  return VT_OK;
}

// Reverse sweep of every group; the instances' blocks are gathered into group
// order (host arrays, or device arrays when device_pointers is set).
static int batch_backward(vt_batch* b, const double* dJdU_T, double* dJdU_0, int device_pointers);

int vt_batch_adjoint_backward(vt_batch* b, const double* dJdU_T, double* dJdU_0) {
  return batch_backward(b, dJdU_T, dJdU_0, 0);
}

int vt_batch_adjoint_backward_device(vt_batch* b, const double* dJdU_T, double* dJdU_0) {
  return batch_backward(b, dJdU_T, dJdU_0, 1);
}

static int batch_backward(vt_batch* b, const double* dJdU_T, double* dJdU_0, int device_pointers) {
  if (!b || !dJdU_T || !dJdU_0) return fail(VT_ERR_INVALID, "vt_batch_adjoint_backward: null argument");
  if (device_pointers && !(vt::aligned_to(dJdU_T, 8) && vt::aligned_to(dJdU_0, 8)))
    return fail(VT_ERR_INVALID, "vt_batch_adjoint_backward_device: device arrays must be 8-byte aligned");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  if (b->views.size() != b->groups.size()) return fail(VT_ERR_INVALID, "vt_batch_adjoint_backward: no forward sweep");
  std::vector<size_t> off(b->n + 1, 0);  // instance offsets in the concatenated arrays (doubles)
  for (int i = 0; i < b->n; ++i)
    off[i + 1] = off[i] + 4 * static_cast<size_t>(b->K_of[i]) * b->groups[b->group_of[i]].Np;
  std::vector<double> gin, gout;
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    vt::Group& G = b->groups[gi];
    const size_t per = 4 * static_cast<size_t>(G.Np);
    if (device_pointers) {
      // group-order device buffers: the view's staging array and a scratch copy
      double *din = nullptr, *dout = nullptr;
      cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&din), 2 * sizeof(double) * per * G.K);
      if (e) return fail(e == cudaErrorMemoryAllocation ? VT_ERR_NO_MEMORY : VT_ERR_CUDA, vt::cuda_msg("batch adjoint", e));
      dout = din + per * G.K;
      for (size_t m = 0; m < G.members.size() && !e; ++m) {
        const int i = G.members[m];
        e = cudaMemcpyAsync(din + per * G.offset[m], dJdU_T + off[i], sizeof(double) * (off[i + 1] - off[i]),
                            cudaMemcpyDeviceToDevice, b->stream);
      }
      if (!e) e = cudaStreamSynchronize(b->stream);
      int st = e ? fail(VT_ERR_CUDA, vt::cuda_msg("batch adjoint gather", e)) : VT_OK;
      if (!st) st = vt_adjoint_backward(b->views[gi], din, dout, 1);
      for (size_t m = 0; m < G.members.size() && !st && !e; ++m) {
        const int i = G.members[m];
        e = cudaMemcpyAsync(dJdU_0 + off[i], dout + per * G.offset[m], sizeof(double) * (off[i + 1] - off[i]),
                            cudaMemcpyDeviceToDevice, b->stream);
      }
      if (!st && !e) e = cudaStreamSynchronize(b->stream);
      cudaFree(din);
      if (st) return st;
      if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("batch adjoint scatter", e));
      continue;
    }
    gin.resize(per * G.K);
    gout.resize(per * G.K);
    for (size_t m = 0; m < G.members.size(); ++m) {
      const int i = G.members[m];
      std::memcpy(gin.data() + per * G.offset[m], dJdU_T + off[i], sizeof(double) * (off[i + 1] - off[i]));
    }
    const int st = vt_adjoint_backward(b->views[gi], gin.data(), gout.data(), 0);
    if (st) return st;
    for (size_t m = 0; m < G.members.size(); ++m) {
      const int i = G.members[m];
      std::memcpy(dJdU_0 + off[i], gout.data() + per * G.offset[m], sizeof(double) * (off[i + 1] - off[i]));
    }
  }
  return VT_OK;
}

int vt_batch_adjoint_info(const vt_batch* b, int group, vt_checkpoint_info* out) {
  if (!b || !out || group < 0 || group >= static_cast<int>(b->views.size()))
    return fail(VT_ERR_INVALID, "vt_batch_adjoint_info: bad argument");
  return vt_adjoint_info(b->views[group], out);
}

int vt_batch_last_error(const vt_batch* b, int* instance, vt_error_info* out) {
  if (!b || !out) return fail(VT_ERR_INVALID, "bad argument");
  *out = b->last;
  if (instance) *instance = b->last_instance;
  return VT_OK;
}

// Times `trials` RK4 steps (after one untimed) of group G alone with its
// current kernel and grid; the group's state must be saved by the caller.
static float time_group_steps(vt_batch* b, vt::Group& G, int trials, cudaEvent_t e0, cudaEvent_t e1) {
  float tot = 0;
  for (int r = 0; r < trials + 1; ++r) {
    cudaEventRecord(e0, b->stream);
    enqueue_group_step(G, b->stream);
    cudaEventRecord(e1, b->stream);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r) tot += ms;  // the first repetition warms up
  }
  return tot;
}

int vt_batch_autotune(vt_batch* b, int trials, int* blocks_per_sm_out, int* mapping_out) {
  if (!b || trials < 1) return fail(VT_ERR_INVALID, "vt_batch_autotune: bad argument");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  // candidates per group: both warp mappings of the stage kernel (one thread
  // per component, or per component pair and node half) x persistent grids of
  // SMs x {1 .. resident limit} blocks; the state is restored afterwards so
  // tuning does not advance the solution
  std::vector<std::vector<double2>> saved;
  for (auto& G : b->groups) {
    const size_t state = 2 * G.Np * static_cast<size_t>(G.Kpad);
    saved.emplace_back(state);
    if (cudaMemcpy(saved.back().data(), G.U, state * sizeof(double2), cudaMemcpyDeviceToHost))
      return fail(VT_ERR_CUDA, "autotune save");
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    vt::Group& G = b->groups[gi];
    vt::StageKernel best_k = G.kern;
    int best_b = 1;
    float best_ms = 1e30f;
    for (int map : {vt::kMapComponent, vt::kMapPair}) {
      const vt::StageKernel k = vt::select_kernel(G.p, G.nfq, map);
      int limit = 0;
      if (k.configure(&limit)) continue;
      G.kern = k;
      for (int bps = 1; bps <= std::max(1, limit); ++bps) {
        G.max_blocks = b->sms * bps;
        const float ms = time_group_steps(b, G, trials, e0, e1);
        if (ms < best_ms) {
          best_ms = ms;
          best_b = bps;
          best_k = k;
        }
      }
    }
    G.kern = best_k;
    G.max_blocks = b->sms * best_b;
    if (blocks_per_sm_out) blocks_per_sm_out[gi] = best_b;
    if (mapping_out) mapping_out[gi] = best_k.map;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    vt::Group& G = b->groups[gi];
    if (cudaMemcpy(G.U, saved[gi].data(), saved[gi].size() * sizeof(double2), cudaMemcpyHostToDevice))
      return fail(VT_ERR_CUDA, "autotune restore");
  }
  for (size_t gi = 0; gi < b->views.size(); ++gi) {  // the adjoint's group views step with the chosen kernels
    vt_ctx* v = b->views[gi];
    v->launch = b->groups[gi].kern.launch;
    v->map = b->groups[gi].kern.map;
    v->max_blocks = b->groups[gi].max_blocks;
    vt::adjoint_invalidate_graphs(v);
  }
  return capture(b);
}

int vt_batch_set_mapping(vt_batch* b, const int* mapping) {
  if (!b || !mapping) return fail(VT_ERR_INVALID, "bad argument");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    if (mapping[gi] != vt::kMapComponent && mapping[gi] != vt::kMapPair)
      return fail(VT_ERR_INVALID, "vt_batch_set_mapping: mapping must be 0 (component) or 1 (pair)");
    vt::Group& G = b->groups[gi];
    const vt::StageKernel k = vt::select_kernel(G.p, G.nfq, mapping[gi]);
    int limit = 0;
    const cudaError_t e = k.configure(&limit);
    if (e) return fail(VT_ERR_CUDA, vt::cuda_msg("vt_batch_set_mapping", e));
    G.kern = k;
    G.max_blocks = std::min(G.max_blocks, b->sms * std::max(1, limit));
    if (gi < b->views.size()) {
      b->views[gi]->launch = k.launch;
      b->views[gi]->map = k.map;
      b->views[gi]->max_blocks = G.max_blocks;
      vt::adjoint_invalidate_graphs(b->views[gi]);
    }
  }
  return capture(b);
}

int vt_batch_time_groups(vt_batch* b, int reps, float* ms_per_step) {
  if (!b || reps < 1 || !ms_per_step) return fail(VT_ERR_INVALID, "vt_batch_time_groups: bad argument");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) || cudaEventCreate(&e1)) return fail(VT_ERR_CUDA, "vt_batch_time_groups: events");
  int st = VT_OK;
  for (size_t gi = 0; gi < b->groups.size() && !st; ++gi) {
    vt::Group& G = b->groups[gi];
    // the group's state is saved and restored, so timing does not advance the solution
    const size_t state = 2 * G.Np * static_cast<size_t>(G.Kpad);
    std::vector<double2> saved(state);
    cudaError_t e = cudaMemcpy(saved.data(), G.U, state * sizeof(double2), cudaMemcpyDeviceToHost);
    if (!e) e = enqueue_group_step(G, b->stream);  // warm-up
    if (!e) e = cudaEventRecord(e0, b->stream);
    for (int r = 0; r < reps && !e; ++r) e = enqueue_group_step(G, b->stream);
    if (!e) e = cudaEventRecord(e1, b->stream);
    if (!e) e = cudaEventSynchronize(e1);
    float ms = 0;
    if (!e) e = cudaEventElapsedTime(&ms, e0, e1);
    if (!e) e = cudaMemcpy(G.U, saved.data(), state * sizeof(double2), cudaMemcpyHostToDevice);
    if (e) st = fail(VT_ERR_CUDA, vt::cuda_msg("vt_batch_time_groups", e));
    ms_per_step[gi] = ms / reps;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

int vt_batch_set_blocks_per_sm(vt_batch* b, const int* blocks_per_sm) {
  if (!b || !blocks_per_sm) return fail(VT_ERR_INVALID, "bad argument");
  std::lock_guard<std::mutex> lk(b->mu);
  cudaSetDevice(b->device);
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    int limit = 0;
    b->groups[gi].kern.configure(&limit);
    const int bps = std::max(1, std::min(blocks_per_sm[gi], std::max(1, limit)));
    b->groups[gi].max_blocks = b->sms * bps;
  }
  return capture(b);
}

int vt_batch_group_info(const vt_batch* b, int g, int* p, int* n_instances, int64_t* n_elements) {
  if (!b || g < 0 || g >= static_cast<int>(b->groups.size())) return fail(VT_ERR_INVALID, "bad group");
  if (p) *p = b->groups[g].p;
  if (n_instances) *n_instances = static_cast<int>(b->groups[g].members.size());
  if (n_elements) *n_elements = b->groups[g].K;
  return VT_OK;
}

}  // extern "C"
