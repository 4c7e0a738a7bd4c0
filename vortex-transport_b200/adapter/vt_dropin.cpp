// Reference-side adapter: the same signature as the reference's stepper
//
//     void rk4(Element*, Evolve_element*, double& t_step, const int& n_elements);
//     void forward_euler(Element*, Evolve_element*, double& t_step, const int& n_elements);
//
// (Timestepping.H:8-9), implemented on the B200 through the C ABI of
// libvortex_b200.so. It is compiled together with the reference's own objects
// (it includes Element.H and Evolve.H), so a driver switches with one call
// site: `rk4(...)` -> `vt_rk4_dropin(...)` at main.cpp:165.
//
// On the first call it packs what the element loop reads from the Element and
// Evolve_element arrays into a vt_mesh_desc, creates the device context and
// uploads U. Each call then advances one step on the GPU; the state stays on
// the device. The reference driver reads the Element objects only when it
// dumps them (write_output, main.cpp:172-178), so the driver's write_output
// call sites are redirected as well (-Dwrite_output=vt_write_output_dropin,
// adapter/Makefile): before a dump, U (and F, with the reference's flux
// formula) and Element::time are written back into the Element objects, and
// the reference's own write_output then writes them. A driver that reads the
// Elements at other times calls vt_dropin_sync(elements) first.
//
// The reference-space operators are not stored in Element; they are recovered
// from element 0's physical ones, which the reference builds as
// M^-1_phys = M^-1_ref / detJ and S_phys = detJ (S_xi J^-1_0d + S_eta J^-1_1d)
// (Element.cpp:96-116): exact up to one rounding each.
//
// A non-physical state ends the process with the reference's message and exit
// status (Numericalflux.cpp:42-115).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "Element.H"
#include "Evolve.H"
#include "Utilities.H"
#include "vortex_b200.h"

namespace {

struct Dropin {
  vt_ctx* ctx = nullptr;
  const Element* elements = nullptr;
  int K = 0, Np = 0, p = 0;
  bool stale = false;  // the device state is ahead of the Element objects
  std::vector<double> U, F;
};

Dropin g;

void fail_exit(const char* what) {
  std::fprintf(stderr, "vt_dropin: %s: %s\n", what, vt_last_message());
  std::exit(EXIT_FAILURE);
}

void create(Element* el, Evolve_element* ev, int K) {
  const int p = el[0].p, Np = (p + 1) * (p + 2) / 2;
  const int nfq = static_cast<int>(ev[0].gau_integ_line.size());
  std::vector<int32_t> type(K), nbr(3 * static_cast<size_t>(K));
  std::vector<double> det(K), jinv(4 * static_cast<size_t>(K)), nrm(6 * static_cast<size_t>(K)),
      len(3 * static_cast<size_t>(K));
  for (int n = 0; n < K; ++n) {
    type[n] = el[n].type;
    nbr[3 * n + 0] = el[n].right_element;
    nbr[3 * n + 1] = el[n].left_element;
    nbr[3 * n + 2] = el[n].vertical_element;
    det[n] = el[n].determinant_jacobian;
    for (int r = 0; r < 2; ++r)
      for (int c = 0; c < 2; ++c) jinv[4 * n + 2 * r + c] = el[n].inverse_jacobian[r][c];
    for (int s = 0; s < 3; ++s) {
      nrm[6 * n + 2 * s + 0] = el[n].units_vectors_perpendicular_to_element_boundary[s][0];
      nrm[6 * n + 2 * s + 1] = el[n].units_vectors_perpendicular_to_element_boundary[s][1];
      len[3 * n + s] = el[n].sides_lenght[s];
    }
  }
  // reference-space operators from element 0 (see the header comment)
  const Element& e0 = el[0];
  const double d = e0.determinant_jacobian;
  const double j00 = e0.inverse_jacobian[0][0], j01 = e0.inverse_jacobian[0][1];
  const double j10 = e0.inverse_jacobian[1][0], j11 = e0.inverse_jacobian[1][1];
  const double jdet = j00 * j11 - j10 * j01;
  std::vector<double> minv(Np * Np), stiff(2 * Np * Np);
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Np; ++j) {
      minv[i * Np + j] = e0.inverse_mass_matrix_physical_space[i][j] * d;
      const double sx = e0.stiffness_matrix_physical_space[0][i][j] / d;
      const double sy = e0.stiffness_matrix_physical_space[1][i][j] / d;
      // [j00 j10; j01 j11] [s_xi; s_eta] = [sx; sy]
      stiff[(0 * Np + i) * Np + j] = (j11 * sx - j10 * sy) / jdet;
      stiff[(1 * Np + i) * Np + j] = (j00 * sy - j01 * sx) / jdet;
    }
  std::vector<double> line(2 * static_cast<size_t>(nfq)), pp(3 * static_cast<size_t>(Np) * nfq),
      pm(pp.size());
  for (int q = 0; q < nfq; ++q) {
    line[2 * q] = ev[0].gau_integ_line[q][0];
    line[2 * q + 1] = ev[0].gau_integ_line[q][1];
  }
  const std::vector<std::vector<double>>* plus[3] = {&ev[0].plus_phi_in_quadrature_points_side_1,
                                                     &ev[0].plus_phi_in_quadrature_points_side_2,
                                                     &ev[0].plus_phi_in_quadrature_points_side_3};
  const std::vector<std::vector<double>>* minus[3] = {&ev[0].minus_phi_in_quadrature_points_side_1,
                                                      &ev[0].minus_phi_in_quadrature_points_side_2,
                                                      &ev[0].minus_phi_in_quadrature_points_side_3};
  for (int s = 0; s < 3; ++s)
    for (int j = 0; j < Np; ++j)
      for (int q = 0; q < nfq; ++q) {
        pp[(s * Np + j) * nfq + q] = (*plus[s])[j][q];
        pm[(s * Np + j) * nfq + q] = (*minus[s])[j][q];
      }
  vt_mesh_desc desc;
  desc.p = p;
  desc.n_elements = K;
  desc.n_line_points = nfq;
  desc.element_type = type.data();
  desc.neighbours = nbr.data();
  desc.det_jacobian = det.data();
  desc.inv_jacobian = jinv.data();
  desc.normals = nrm.data();
  desc.side_lengths = len.data();
  desc.inv_mass_ref = minv.data();
  desc.stiffness_ref = stiff.data();
  desc.line_quadrature = line.data();
  desc.phi_plus = pp.data();
  desc.phi_minus = pm.data();
  int st = 0;
  const char* dev = std::getenv("VT_DEVICE");
  g.ctx = vt_create(&desc, dev ? std::atoi(dev) : 0, &st);
  if (!g.ctx) fail_exit("vt_create");
  g.elements = el;
  g.K = K;
  g.Np = Np;
  g.p = p;
  g.U.resize(4 * static_cast<size_t>(K) * Np);
  g.F.resize(8 * static_cast<size_t>(K) * Np);
  for (int n = 0; n < K; ++n)
    for (int i = 0; i < Np; ++i)
      for (int k = 0; k < 4; ++k) g.U[(static_cast<size_t>(n) * Np + i) * 4 + k] = el[n].hidrodynamics_vector_U[i][k];
  if (vt_upload_state(g.ctx, g.U.data()) != VT_OK) fail_exit("vt_upload_state");
  vt_set_time(g.ctx, el[0].time);
}

void write_back(Element* el) {
  if (vt_download_state(g.ctx, g.U.data(), g.F.data()) != VT_OK) fail_exit("vt_download_state");
  const double t = vt_get_time(g.ctx);
  for (int n = 0; n < g.K; ++n) {
    for (int i = 0; i < g.Np; ++i) {
      const size_t a = static_cast<size_t>(n) * g.Np + i;
      for (int k = 0; k < 4; ++k) el[n].hidrodynamics_vector_U[i][k] = g.U[4 * a + k];
      for (int dd = 0; dd < 2; ++dd)
        for (int k = 0; k < 4; ++k) el[n].hidrodynamics_vector_F[i][dd][k] = g.F[8 * a + 4 * dd + k];
    }
    el[n].time = t;
  }
  g.stale = false;
}

void step(Element* el, Evolve_element* ev, double dt, int K, bool rk4) {
  if (!g.ctx || g.elements != el || g.K != K) {
    if (g.ctx) vt_destroy(g.ctx);
    create(el, ev, K);
  }
  const int st = rk4 ? vt_step_rk4(g.ctx, dt, 1) : vt_step_euler(g.ctx, dt, 1);
  if (st == VT_ERR_NONPHYSICAL_LEFT || st == VT_ERR_NONPHYSICAL_RIGHT || st == VT_ERR_NONPHYSICAL_C2) {
    vt_error_info info;
    vt_last_error(g.ctx, &info);
    std::fprintf(stderr, "%d. Error: Non-physical state! \n", st);
    std::printf(" element %d, face point %d, side %d\n", info.element, info.point, info.side + 1);
    std::exit(EXIT_FAILURE);
  }
  if (st != VT_OK) fail_exit(rk4 ? "vt_step_rk4" : "vt_step_euler");
  g.stale = true;
}

}  // namespace

void vt_dropin_sync(Element* elemts) {
  if (g.ctx && g.stale && g.elements == elemts) write_back(elemts);
}

// The driver's dumps: bring the Element objects up to date from the device,
// then the reference's own writer (Utilities.cpp:65-77).
void vt_write_output_dropin(Element* elemts, const int& total_num_elements, const int& step_num) {
  vt_dropin_sync(elemts);
  write_output(elemts, total_num_elements, step_num);
}

void vt_rk4_dropin(Element* elemts, Evolve_element* evo_elemts, double& t_step, const int& n_elements) {
  step(elemts, evo_elemts, t_step, n_elements, true);
}

void vt_forward_euler_dropin(Element* elemts, Evolve_element* evo_elemts, double& t_step,
                             const int& n_elements) {
  step(elemts, evo_elemts, t_step, n_elements, false);
}
