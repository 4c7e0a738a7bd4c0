// Host-side precompute of the reference's operators and mesh, restated in C++.
//
// Everything the reference computes once before its time loop (main.cpp:96-147)
// and hands to the stepper: input-file keys, structured periodic mesh and
// connectivity, reference nodes, Lagrange basis, quadrature rules, reference
// mass-inverse and stiffness matrices, per-element geometry, face basis tables
// and the isentropic-vortex initial condition. Arithmetic follows the
// reference's expressions (including its float/double conversions) so the
// results match the reference bit for bit; see each function for the lines.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/vortex_b200.h"

namespace vt {

constexpr int np_of(int p) { return (p + 1) * (p + 2) / 2; }

// Parameters.cpp:12-64 on the text of an input file. Returns VT_OK or
// VT_ERR_INVALID with a message naming the offending key.
int parse_input_text(const std::string& text, vt_params* out, std::string* msg);

// Quadraturerule.cpp:13-181: Gauss-Legendre on [0, 1], rows (sigma, weight).
bool line_rule(int integration_order, std::vector<double>* rows);
// Quadraturerule.cpp:183-662: Dunavant rule on the reference triangle, rows
// (xi, eta, weight); weights sum to the triangle area 1/2.
bool area_rule(int integration_order, std::vector<double>* rows);

// Lagrangebasis.cpp:12-63 / :66-147. phi has Np entries, grad Np x 2.
bool basis(int p, double xi, double eta, double* phi);
bool basis_gradient(int p, double xi, double eta, double* grad);

// Meshgeneration.cpp:188-220: Np x 2 (xi, eta), j (eta) outer, i (xi) inner.
std::vector<double> reference_nodes(int p);

// Preevolve.cpp:15-78 and :86-144.
// Returns false when the rule is too coarse for p and the mass matrix is
// exactly singular (the reference then carries inf/nan operators).
bool inverse_mass_reference(int p, const std::vector<double>& area, std::vector<double>* minv);
std::vector<double> stiffness_reference(int p, const std::vector<double>& area);

// Gauss-Jordan elimination with partial pivoting, in place on an n x n row-major
// matrix; returns false if singular.
bool invert_gauss_jordan(int n, std::vector<double>* a);

struct Mesh {
  int nx = 0, ny = 0, K = 0;
  std::vector<double> verts;  // K x 3 x 2, vertex 0 at the right angle, counter-clockwise
  std::vector<int32_t> conn;  // K x 3: right, left, vertical neighbour
  std::vector<int32_t> type;  // K: 0 right angle down, 1 up
};

// Meshgeneration.cpp:16-186 (without the grid/ text files).
Mesh generate_mesh(const vt_params& prm);

// Element.cpp:54-93 for one element: jac/jinv [00,01,10,11], normals 3 x 2, sides 3.
void element_geometry(const double* v, double* jac, double* jinv, double* detj,
                      double* detjinv, double* normals, double* sides);

// Evolve.cpp:76-132: 3 x Np x nfq tables of the basis at the face points, own
// side (plus) and as seen from the neighbour (minus).
void face_tables(int p, const std::vector<double>& line, std::vector<double>* plus,
                 std::vector<double>* minus);

// Element.cpp:119-179 (type 0, nodal) and :180-326 (type 1, L2 projection),
// with the vortex parameters taken from `ic` instead of hard-coded literals.
// U is K x Np x 4 and F is K x Np x 2 x 4.
int initial_condition(const vt_params& prm, const vt_vortex& ic, const Mesh& mesh,
                      const std::vector<double>& nodes_ref, const std::vector<double>& area,
                      const std::vector<double>& minv_ref, double time, std::vector<double>* U,
                      std::vector<double>* F, std::vector<double>* nodes_phys);

// The exactly translated vortex at time t at the physical nodes (K x Np x 2),
// U = K x Np x 4: the formula of Element.cpp:134-179 with the centre moved by
// (U_infty, V_infty) t and taken as the nearest periodic image of each node on
// the domain_x x domain_y torus (the reference's formula does not wrap).
void exact_vortex(const vt_params& prm, const vt_vortex& ic, const std::vector<double>& nodes_phys, double t,
                  double* U);

// Nodal flux of a state (Timestepping.cpp:141-158 formula), F = K x Np x 2 x 4.
void flux_from_state(int K, int Np, const double* U, double* F);

// The reference's vortex literals (Element.cpp:134-143).
vt_vortex default_vortex();

}  // namespace vt
