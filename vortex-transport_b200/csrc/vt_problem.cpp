// C ABI of the host precompute (include/vortex_b200.h, "input file",
// "initial condition" and "host precompute" sections).
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "vt_common.h"
#include "vt_precompute.h"

namespace vt {

namespace {
thread_local std::string g_message;
}

int fail(int status, const std::string& msg) {
  g_message = msg;
  return status;
}

void clear_message() { g_message.clear(); }

}  // namespace vt

struct vt_problem {
  vt_params prm;
  vt_vortex ic;
  vt::Mesh mesh;
  int Np = 0;
  std::vector<double> nodes_ref, nodes_phys, line, area, minv, stiff, phi_plus, phi_minus;
  std::vector<double> jac, jinv, detj, detjinv, normals, sides;
  std::vector<double> U0, F0;
};

extern "C" {

const char* vt_last_message(void) { return vt::g_message.c_str(); }

int vt_parse_input(const char* text, vt_params* out) {
  if (!text || !out) return vt::fail(VT_ERR_INVALID, "vt_parse_input: null argument");
  std::string msg;
  const int st = vt::parse_input_text(text, out, &msg);
  if (st != VT_OK) return vt::fail(st, msg);
  return VT_OK;
}

int vt_read_input_file(const char* path, vt_params* out) {
  if (!path || !out) return vt::fail(VT_ERR_INVALID, "vt_read_input_file: null argument");
  std::ifstream f(path);
  if (!f.is_open()) return vt::fail(VT_ERR_INVALID, std::string("unable to open input file '") + path + "'");
  std::stringstream ss;
  ss << f.rdbuf();
  return vt_parse_input(ss.str().c_str(), out);
}

void vt_default_vortex(vt_vortex* out) {
  if (out) *out = vt::default_vortex();
}

vt_problem* vt_problem_create(const vt_params* prm, const vt_vortex* ic, int* status) {
  auto set = [&](int s) {
    if (status) *status = s;
  };
  if (!prm) {
    set(vt::fail(VT_ERR_INVALID, "vt_problem_create: null parameters"));
    return nullptr;
  }
  if (prm->p < 0 || prm->p > 3) {
    set(vt::fail(VT_ERR_UNSUPPORTED, "p must be 0..3 (Lagrangebasis.cpp:53-56)"));
    return nullptr;
  }
  if (prm->integration_order < 0 || prm->integration_order > 19) {
    set(vt::fail(VT_ERR_UNSUPPORTED, "integration_order must be 0..19"));
    return nullptr;
  }
  if (prm->num_element_in_x < 1 || prm->num_element_in_y < 1 ||
      2.0 * prm->num_element_in_x * prm->num_element_in_y > 2147483647.0 / 64) {
    set(vt::fail(VT_ERR_INVALID, "num_element_in_x/y out of range"));
    return nullptr;
  }
  if (prm->U_initialization_type != 0 && prm->U_initialization_type != 1) {
    set(vt::fail(VT_ERR_UNSUPPORTED, "U_initialization_type must be 0 or 1 (Element.cpp:327-330)"));
    return nullptr;
  }
  auto* pb = new vt_problem();
  pb->prm = *prm;
  pb->ic = ic ? *ic : vt::default_vortex();
  const int p = prm->p;
  pb->Np = vt::np_of(p);
  vt::line_rule(prm->integration_order, &pb->line);
  vt::area_rule(prm->integration_order, &pb->area);
  pb->mesh = vt::generate_mesh(*prm);
  pb->nodes_ref = vt::reference_nodes(p);
  if (!vt::inverse_mass_reference(p, pb->area, &pb->minv)) {
    delete pb;
    set(vt::fail(VT_ERR_UNSUPPORTED, "integration_order " + std::to_string(prm->integration_order) +
                                         " is too low for p=" + std::to_string(p) +
                                         ": the reference mass matrix is singular"));
    return nullptr;
  }
  pb->stiff = vt::stiffness_reference(p, pb->area);
  vt::face_tables(p, pb->line, &pb->phi_plus, &pb->phi_minus);
  const int K = pb->mesh.K;
  pb->jac.resize(4 * static_cast<size_t>(K));
  pb->jinv.resize(4 * static_cast<size_t>(K));
  pb->detj.resize(K);
  pb->detjinv.resize(K);
  pb->normals.resize(6 * static_cast<size_t>(K));
  pb->sides.resize(3 * static_cast<size_t>(K));
  for (int n = 0; n < K; ++n)
    vt::element_geometry(&pb->mesh.verts[6 * static_cast<size_t>(n)], &pb->jac[4 * n], &pb->jinv[4 * n],
                         &pb->detj[n], &pb->detjinv[n], &pb->normals[6 * static_cast<size_t>(n)],
                         &pb->sides[3 * static_cast<size_t>(n)]);
  const int st = vt::initial_condition(*prm, pb->ic, pb->mesh, pb->nodes_ref, pb->area, pb->minv, 0.0,
                                       &pb->U0, &pb->F0, &pb->nodes_phys);
  if (st != VT_OK) {
    delete pb;
    set(vt::fail(st, "initial condition failed"));
    return nullptr;
  }
  set(VT_OK);
  return pb;
}

void vt_problem_destroy(vt_problem* pb) { delete pb; }

int vt_problem_get_info(const vt_problem* pb, vt_problem_info* out) {
  if (!pb || !out) return vt::fail(VT_ERR_INVALID, "null argument");
  out->K = pb->mesh.K;
  out->p = pb->prm.p;
  out->Np = pb->Np;
  out->nfq = static_cast<int>(pb->line.size() / 2);
  out->nqa = static_cast<int>(pb->area.size() / 3);
  out->nx = pb->mesh.nx;
  out->ny = pb->mesh.ny;
  return VT_OK;
}

int vt_problem_get_array(const vt_problem* pb, const char* name, void* dst, size_t bytes) {
  if (!pb || !name || !dst) return vt::fail(VT_ERR_INVALID, "null argument");
  const void* src = nullptr;
  size_t n = 0;
  auto take_d = [&](const std::vector<double>& v) {
    src = v.data();
    n = v.size() * sizeof(double);
  };
  auto take_i = [&](const std::vector<int32_t>& v) {
    src = v.data();
    n = v.size() * sizeof(int32_t);
  };
  const std::string k(name);
  if (k == "vertices") take_d(pb->mesh.verts);
  else if (k == "conn") take_i(pb->mesh.conn);
  else if (k == "type") take_i(pb->mesh.type);
  else if (k == "nodes_ref") take_d(pb->nodes_ref);
  else if (k == "nodes_phys") take_d(pb->nodes_phys);
  else if (k == "line_quad") take_d(pb->line);
  else if (k == "area_quad") take_d(pb->area);
  else if (k == "minv_ref") take_d(pb->minv);
  else if (k == "stiff_ref") take_d(pb->stiff);
  else if (k == "phi_plus") take_d(pb->phi_plus);
  else if (k == "phi_minus") take_d(pb->phi_minus);
  else if (k == "jac") take_d(pb->jac);
  else if (k == "jinv") take_d(pb->jinv);
  else if (k == "detj") take_d(pb->detj);
  else if (k == "detjinv") take_d(pb->detjinv);
  else if (k == "normals") take_d(pb->normals);
  else if (k == "sides") take_d(pb->sides);
  else if (k == "U0") take_d(pb->U0);
  else if (k == "F0") take_d(pb->F0);
  else return vt::fail(VT_ERR_INVALID, "unknown array name '" + k + "'");
  if (bytes != n)
    return vt::fail(VT_ERR_INVALID, "array '" + k + "' has " + std::to_string(n) + " bytes, got " +
                                        std::to_string(bytes));
  std::memcpy(dst, src, n);
  return VT_OK;
}

int vt_problem_mesh_desc(const vt_problem* pb, vt_mesh_desc* d) {
  if (!pb || !d) return vt::fail(VT_ERR_INVALID, "null argument");
  d->p = pb->prm.p;
  d->n_elements = pb->mesh.K;
  d->n_line_points = static_cast<int32_t>(pb->line.size() / 2);
  d->element_type = pb->mesh.type.data();
  d->neighbours = pb->mesh.conn.data();
  d->det_jacobian = pb->detj.data();
  d->inv_jacobian = pb->jinv.data();
  d->normals = pb->normals.data();
  d->side_lengths = pb->sides.data();
  d->inv_mass_ref = pb->minv.data();
  d->stiffness_ref = pb->stiff.data();
  d->line_quadrature = pb->line.data();
  d->phi_plus = pb->phi_plus.data();
  d->phi_minus = pb->phi_minus.data();
  return VT_OK;
}

int vt_flux_from_state(int K, int p, const double* U, double* F) {
  if (!U || !F || K < 0 || p < 0 || p > 3) return vt::fail(VT_ERR_INVALID, "bad argument");
  vt::flux_from_state(K, vt::np_of(p), U, F);
  return VT_OK;
}

int vt_problem_exact_state(const vt_problem* pb, double t, double* U) {
  if (!pb || !U) return vt::fail(VT_ERR_INVALID, "vt_problem_exact_state: null argument");
  vt::exact_vortex(pb->prm, pb->ic, pb->nodes_phys, t, U);
  return VT_OK;
}

// State file: "VTSTATE" + NUL, int32 version (1), p, K, Np, float64 time, then
// K x Np x 4 float64 (the reference's element-major U layout), little-endian
// as the host writes it.
namespace {
constexpr char kStateMagic[8] = {'V', 'T', 'S', 'T', 'A', 'T', 'E', '\0'};
struct StateHeader {
  char magic[8];
  int32_t version, p, K, Np;
  double time;
};
static_assert(sizeof(StateHeader) == 32, "state header layout");
}  // namespace

int vt_write_state_file(const char* path, int p, int K, double time, const double* U) {
  if (!path || !U || p < 0 || p > 3 || K < 1) return vt::fail(VT_ERR_INVALID, "vt_write_state_file: bad argument");
  StateHeader h{};
  std::memcpy(h.magic, kStateMagic, 8);
  h.version = 1;
  h.p = p;
  h.K = K;
  h.Np = vt::np_of(p);
  h.time = time;
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) return vt::fail(VT_ERR_INVALID, std::string("vt_write_state_file: cannot open '") + path + "'");
  f.write(reinterpret_cast<const char*>(&h), sizeof(h));
  f.write(reinterpret_cast<const char*>(U), static_cast<std::streamsize>(sizeof(double) * 4 * static_cast<size_t>(K) * h.Np));
  if (!f) return vt::fail(VT_ERR_INVALID, std::string("vt_write_state_file: write failed on '") + path + "'");
  return VT_OK;
}

int vt_state_file_info(const char* path, int* p, int* K, double* time) {
  if (!path) return vt::fail(VT_ERR_INVALID, "vt_state_file_info: null path");
  std::ifstream f(path, std::ios::binary);
  StateHeader h{};
  if (!f || !f.read(reinterpret_cast<char*>(&h), sizeof(h)))
    return vt::fail(VT_ERR_INVALID, std::string("vt_state_file_info: cannot read '") + path + "'");
  if (std::memcmp(h.magic, kStateMagic, 8) != 0 || h.version != 1 || h.p < 0 || h.p > 3 || h.K < 1 ||
      h.Np != vt::np_of(h.p))
    return vt::fail(VT_ERR_INVALID, std::string("vt_state_file_info: '") + path + "' is not a state file");
  f.seekg(0, std::ios::end);
  const std::streamoff want = static_cast<std::streamoff>(sizeof(h) + sizeof(double) * 4 * static_cast<size_t>(h.K) * h.Np);
  if (f.tellg() != want) return vt::fail(VT_ERR_INVALID, std::string("vt_state_file_info: '") + path + "' has the wrong size");
  if (p) *p = h.p;
  if (K) *K = h.K;
  if (time) *time = h.time;
  return VT_OK;
}

int vt_read_state_file(const char* path, double* U) {
  int p = 0, K = 0;
  double t = 0;
  int st = vt_state_file_info(path, &p, &K, &t);
  if (st) return st;
  if (!U) return vt::fail(VT_ERR_INVALID, "vt_read_state_file: null output");
  std::ifstream f(path, std::ios::binary);
  f.seekg(sizeof(StateHeader));
  if (!f.read(reinterpret_cast<char*>(U), static_cast<std::streamsize>(sizeof(double) * 4 * static_cast<size_t>(K) * vt::np_of(p))))
    return vt::fail(VT_ERR_INVALID, std::string("vt_read_state_file: cannot read '") + path + "'");
  return VT_OK;
}

}  // extern "C"
