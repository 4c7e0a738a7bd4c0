// RK4 stepping that allocates no device memory (vt_step_rk4_noalloc in
// include/vortex_b200.h).
//
// Some callers cannot call cudaMalloc: code that runs while another component
// owns every device allocation (a memory pool or arena handed out by a host
// framework), real-time loops where a cudaMalloc/cudaFree would synchronise
// the device and stall the loop, and plugins that are only allowed to touch
// buffers their host passes in. For them this file keeps the stepper's
// scratch -- the packed geometry and neighbour rows, the tile schedule, the state in the
// kernel's layout, the RK accumulator, the two stage buffers and the error
// words -- in one file-scope __device__ array of kScratchBytes, which every
// GPU that loads the library holds until the process exits. The caller passes
// the inputs (the mesh arrays and U, in device memory) and the output U.
//
// The array is shared by every call on a device and keeps the last call's
// contents; each call clears the words that must start at zero. Two calls
// whose work overlaps on the GPU (different streams, or different host
// threads on one stream) race on the array.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/vortex_b200.h"
#include "vt_common.h"
#include "vt_precompute.h"
#include "vt_launch.h"

namespace vt {
namespace {

constexpr size_t kScratchBytes = VT_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Per-device set-up, done by the first call on a device with that device
// current: the SM count for the persistent grid. The device address of
// g_scratch (the host-side symbol is only a stand-in) is looked up on every
// call instead of being cached, so a context re-created after cudaDeviceReset
// (which may load the module at another address) gets the current one.
struct DeviceSetup {
  bool done = false;
  int sms = 0;
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mu;

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

struct Carve {
  long long Kpad;
  int ntiles;
  size_t err, geo, nbr, tiles, items, count, U, A, Sa, Sb, total;
};

Carve carve(int p, int K) {
  Carve c;
  c.Kpad = (static_cast<long long>(K) + 127) / 128 * 128;
  const size_t state = sizeof(double2) * 2 * np_of(p) * static_cast<size_t>(c.Kpad);
  c.err = 0;
  c.geo = align256(c.err + 4 * sizeof(unsigned long long));
  c.nbr = align256(c.geo + sizeof(double2) * 7 * static_cast<size_t>(c.Kpad));
  c.ntiles = (K + kTileElems - 1) / kTileElems;
  c.tiles = align256(c.nbr + sizeof(int4) * static_cast<size_t>(c.Kpad));
  c.items = align256(c.tiles + sizeof(int4) * static_cast<size_t>(c.ntiles));
  c.count = align256(c.items + sizeof(int) * kMaxItems * static_cast<size_t>(c.ntiles));
  c.U = align256(c.count + sizeof(int) * static_cast<size_t>(c.ntiles));
  c.A = align256(c.U + state);
  c.Sa = align256(c.A + state);
  c.Sb = align256(c.Sa + state);
  c.total = align256(c.Sb + state);
  return c;
}

// Packs the caller's per-element device arrays (vt_mesh_desc layouts) into the
// kernel's geometry and side-ordered neighbour rows; flags bad neighbour ids.
__global__ void pack_geometry_kernel(vt_device_mesh m, double2* geo, int4* nbr, long long KP,
                                     unsigned long long* err) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= m.n_elements) return;
  const double* ji = m.inv_jacobian + 4 * static_cast<size_t>(n);
  const double* nv = m.normals + 6 * static_cast<size_t>(n);
  const double* ln = m.side_lengths + 3 * static_cast<size_t>(n);
  const double det = m.det_jacobian[n];
  geo[0 * KP + n] = make_double2(ji[0], ji[1]);
  geo[1 * KP + n] = make_double2(ji[2], ji[3]);
  for (int s = 0; s < 3; ++s) geo[(2 + s) * KP + n] = make_double2(nv[2 * s], nv[2 * s + 1]);
  geo[5 * KP + n] = make_double2(ln[0] / det, ln[1] / det);
  geo[6 * KP + n] = make_double2(ln[2] / det, det);
  int right = m.neighbours[3 * n], left = m.neighbours[3 * n + 1], vert = m.neighbours[3 * n + 2];
  const int K = m.n_elements;
  if (right < 0 || right >= K || left < 0 || left >= K || vert < 0 || vert >= K) {
    atomicOr(&err[3], 1ull);
    right = left = vert = n;
  }
  nbr[n] = m.element_type[n] == 0 ? make_int4(vert, right, left, 0) : make_int4(vert, left, right, 0);
}

__global__ void gather_soa_kernel(const double2* __restrict__ aos, double2* __restrict__ soa, int K, int Np,
                                  long long KP) {
  const long long l = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (l >= static_cast<long long>(K) * 2 * Np) return;
  const int r = static_cast<int>(l / K), e = static_cast<int>(l % K);
  soa[r * KP + e] = aos[static_cast<long long>(e) * 2 * Np + r];
}

__global__ void scatter_aos_kernel(const double2* __restrict__ soa, double2* __restrict__ aos, int K, int Np,
                                   long long KP) {
  const long long l = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (l >= static_cast<long long>(K) * 2 * Np) return;
  const int r = static_cast<int>(l / K), e = static_cast<int>(l % K);
  aos[static_cast<long long>(e) * 2 * Np + r] = soa[r * KP + e];
}

// The operator block of StageOps<P, NFQ> (at most 740 doubles), folded on the
// host into a fixed-size stack buffer by the solver's own fold.
constexpr int kMaxOps = 2 * 10 * 10 + 3 * 10 * 10 + 2 * 3 * 10 * 4;

}  // namespace
}  // namespace vt

extern "C" {

size_t vt_noalloc_scratch_bytes(int p, int n_elements) {
  if (p < 0 || p > 3 || n_elements < 1) return 0;
  return vt::carve(p, n_elements).total;
}

int vt_step_rk4_noalloc(const vt_device_mesh* m, const double* dU_in, double* dU_out, double dt, int nsteps,
                        void* stream, vt_error_info* err) {
  using vt::fail;
  if (err) *err = vt_error_info{};
  if (!m || !dU_in || !dU_out || nsteps < 0)
    return fail(VT_ERR_INVALID, "vt_step_rk4_noalloc: null argument or negative step count");
  if (!m->element_type || !m->neighbours || !m->det_jacobian || !m->inv_jacobian || !m->normals ||
      !m->side_lengths || !m->inv_mass_ref || !m->stiffness_ref || !m->line_quadrature || !m->phi_plus ||
      !m->phi_minus)
    return fail(VT_ERR_INVALID, "vt_step_rk4_noalloc: null mesh field");
  if (m->p < 0 || m->p > 3 || m->n_line_points < 1 || m->n_line_points > 10 || m->n_elements < 1)
    return fail(VT_ERR_UNSUPPORTED, "vt_step_rk4_noalloc: p must be 0..3, n_line_points 1..10, n_elements > 0");
  const vt::Carve cv = vt::carve(m->p, m->n_elements);
  if (cv.total > vt::kScratchBytes)
    return fail(VT_ERR_INVALID, "vt_step_rk4_noalloc: the problem needs " + std::to_string(cv.total) +
                                    " bytes of scratch, more than the fixed " +
                                    std::to_string(vt::kScratchBytes) + " (use vt_create for larger meshes)");
  // the kernels read the states as double2 and the mesh arrays as doubles / ints:
  // reject misaligned views before any device work
  if (!vt::aligned_to(dU_in, 16) || !vt::aligned_to(dU_out, 16))
    return fail(VT_ERR_INVALID, "vt_step_rk4_noalloc: dU_in and dU_out must be 16-byte aligned");
  if (!vt::aligned_to(m->element_type, 4) || !vt::aligned_to(m->neighbours, 4) ||
      !vt::aligned_to(m->det_jacobian, 8) || !vt::aligned_to(m->inv_jacobian, 8) ||
      !vt::aligned_to(m->normals, 8) || !vt::aligned_to(m->side_lengths, 8))
    return fail(VT_ERR_INVALID, "vt_step_rk4_noalloc: a mesh array is misaligned for its element type");
  const vt::StageKernel pk = vt::select_kernel(m->p, m->n_line_points);

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e) return fail(VT_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= vt::kMaxDevices) return fail(VT_ERR_UNSUPPORTED, "device index out of range");
  vt::DeviceSetup* ds = &vt::g_setup[dev];
  {
    std::lock_guard<std::mutex> lk(vt::g_setup_mu);
    if (!ds->done) {
      e = cudaDeviceGetAttribute(&ds->sms, cudaDevAttrMultiProcessorCount, dev);
      if (e) return fail(VT_ERR_CUDA, std::string("device attribute: ") + cudaGetErrorString(e));
      ds->done = true;
    }
  }
  // the device address of the scratch array on the current device (a lookup,
  // no allocation); the host-side symbol g_scratch is only a stand-in
  void* scratch_ptr = nullptr;
  e = cudaGetSymbolAddress(&scratch_ptr, vt::g_scratch);
  if (e || !scratch_ptr)
    return fail(VT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  int per_sm = 0;
  if ((e = vt::tensor_maps_available()) || (e = pk.configure(&per_sm)))
    return fail(VT_ERR_CUDA, std::string("kernel attributes: ") + cudaGetErrorString(e));
  const int max_blocks = ds->sms * (per_sm > 0 ? per_sm : 1);

  unsigned char* base = static_cast<unsigned char*>(scratch_ptr);
  auto* errw = reinterpret_cast<unsigned long long*>(base + cv.err);
  auto* geo = reinterpret_cast<double2*>(base + cv.geo);
  auto* nbr = reinterpret_cast<int4*>(base + cv.nbr);
  auto* tiles = reinterpret_cast<int4*>(base + cv.tiles);
  auto* items = reinterpret_cast<int*>(base + cv.items);
  auto* count = reinterpret_cast<int*>(base + cv.count);
  auto* U = reinterpret_cast<double2*>(base + cv.U);
  auto* A = reinterpret_cast<double2*>(base + cv.A);
  auto* Sa = reinterpret_cast<double2*>(base + cv.Sa);
  auto* Sb = reinterpret_cast<double2*>(base + cv.Sb);
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int K = m->n_elements, Np = vt::np_of(m->p);

  double ops[vt::kMaxOps];
  vt::fold_stage_operators(m->p, m->n_line_points, m->inv_mass_ref, m->stiffness_ref, m->line_quadrature,
                           m->phi_plus, m->phi_minus, ops);

  // error key to "none", step and block counters and the neighbour flag to zero
  if ((e = cudaMemsetAsync(errw, 0xFF, sizeof(unsigned long long), st)) ||
      (e = cudaMemsetAsync(errw + 1, 0, 3 * sizeof(unsigned long long), st)))
    return fail(VT_ERR_CUDA, std::string("scratch reset: ") + cudaGetErrorString(e));
  vt::pack_geometry_kernel<<<(K + 255) / 256, 256, 0, st>>>(*m, geo, nbr, cv.Kpad, errw);
  if ((e = vt::launch_contiguous_tiles(tiles, K, cv.ntiles, st)) ||
      (e = vt::launch_build_tile_items(tiles, nbr, items, count, cv.ntiles, m->n_line_points, st)))
    return fail(VT_ERR_CUDA, std::string("tile schedule: ") + cudaGetErrorString(e));
  const long long nrow = static_cast<long long>(K) * 2 * Np;
  const int tb = static_cast<int>((nrow + 255) / 256);
  vt::gather_soa_kernel<<<tb, 256, 0, st>>>(reinterpret_cast<const double2*>(dU_in), U, K, Np, cv.Kpad);
  if ((e = cudaGetLastError())) return fail(VT_ERR_CUDA, std::string("pack: ") + cudaGetErrorString(e));

  auto args = [&](const double2* in, double2* out, int stage, double c_acc, double c_out) {
    vt::StageArgs a;
    a.in = in;
    a.base = U;
    a.acc = A;
    a.out = out;
    a.geo = geo;
    a.nbr = nbr;
    a.tiles = tiles;
    a.tile_items = items;
    a.tile_dt = nullptr;
    a.tile_count = count;
    a.ntiles = cv.ntiles;
    a.err = errw;
    a.Kpad = cv.Kpad;
    a.K = K;
    a.stage = stage;
    a.c_acc = c_acc;
    a.c_out = c_out;
    return a;
  };
  for (int s = 0; s < nsteps && !e; ++s) {
    if (!e) e = pk.launch(args(U, Sa, 0, (1.0 / 6) * dt, 0.5 * dt), ops, max_blocks, st);
    if (!e) e = pk.launch(args(Sa, Sb, 1, (1.0 / 3) * dt, 0.5 * dt), ops, max_blocks, st);
    if (!e) e = pk.launch(args(Sb, Sa, 2, (1.0 / 3) * dt, dt), ops, max_blocks, st);
    if (!e) e = pk.launch(args(Sa, U, 3, 0.0, (1.0 / 6) * dt), ops, max_blocks, st);
  }
  if (!e) {
    vt::scatter_aos_kernel<<<tb, 256, 0, st>>>(U, reinterpret_cast<double2*>(dU_out), K, Np, cv.Kpad);
    e = cudaGetLastError();
  }
  unsigned long long words[4] = {~0ull, 0, 0, 0};
  if (!e) e = cudaMemcpyAsync(words, errw, sizeof(words), cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaStreamSynchronize(st);
  if (e) return fail(VT_ERR_CUDA, std::string("vt_step_rk4_noalloc: ") + cudaGetErrorString(e));
  if (words[3] & 1ull) return fail(VT_ERR_INVALID, "vt_step_rk4_noalloc: neighbour index out of range");
  if (words[3] & 2ull) return fail(VT_ERR_CUDA, "vt_step_rk4_noalloc: a bulk-copy wait gave up");
  if (words[0] == ~0ull) return VT_OK;
  const vt_error_info info = vt::decode_error_key(words[0], m->n_line_points);
  if (err) *err = info;
  return fail(info.code, "Non-physical state (code " + std::to_string(info.code) + ") at element " +
                             std::to_string(info.element));
}

}  // extern "C"
