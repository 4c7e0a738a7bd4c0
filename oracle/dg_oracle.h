/* Test infrastructure: the ORACLE. Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load it, and only as the checker.
 *
 * CPU restatement of the reference's nodal-DG right-hand side and explicit
 * steppers over flat arrays, written to perform the reference's floating-point
 * operations in the reference's order (libm pow() where the reference calls
 * pow(), no FMA contraction), so that on x86-64 it reproduces the reference's
 * -O2 build bit for bit. Each function cites the reference lines it restates.
 *
 * Array layouts (row-major, element-major like the reference's nested vectors):
 *   U      K x Np x 4          hidrodynamics_vector_U   (Element.H:30)
 *   F      K x Np x 2 x 4      hidrodynamics_vector_F   (Element.H:31)
 *   verts  K x 3 x 2           mesh.element_coordinates (Meshgeneration.H:9)
 *   conn   K x 3 (right, left, vertical)                (Meshgeneration.cpp:140-146)
 *   type   K (0: right angle down, 1: up)               (Meshgeneration.cpp:84-88)
 *   minv_ref   Np x Np, stiff_ref 2 x Np x Np           (Preevolve.cpp:15-144)
 *   phi_plus / phi_minus   3 x Np x nfq                 (Evolve.cpp:76-132)
 *   line_quad  nfq x 2 (sigma, weight)                  (Quadraturerule.cpp:13-181)
 */
#ifndef VT_DG_ORACLE_H
#define VT_DG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int K, p, Np, nfq;
  const double* verts;
  const int* conn;
  const int* type;
  const double* minv_ref;
  const double* stiff_ref;
  const double* phi_plus;
  const double* phi_minus;
  const double* line_quad;
} vto_mesh;

/* Error report with the reference's exit conditions (Numericalflux.cpp:42-115):
 * code 1 left state pL<=0 or rL<=0, 2 right state, 3 Roe c2<=0. The first
 * failure in the reference's serial order (element, quadrature point, side). */
typedef struct {
  int code;
  int element;
  int point;
  int side;
} vto_error;

/* Element::build_jacobians (Element.cpp:54-93) for every element:
 * jac/jinv K x 4 ([00,01,10,11]), detj/detjinv K, normals K x 3 x 2, sides K x 3. */
void vto_geometry(const vto_mesh* m, double* jac, double* jinv, double* detj, double* detjinv,
                  double* normals, double* sides);

/* numerical_flux (Numericalflux.cpp:13-157). Returns 0 or the error code. */
int vto_numerical_flux(const double* uL, const double* uR, const double* n, double* flux);

/* evolve_elem (Timestepping.cpp:18-36): Udot = DG_time_derivative_U, K x Np x 4. */
int vto_rhs(const vto_mesh* m, const double* U, const double* F, double* Udot, vto_error* err);

/* Nodal flux refresh used after every stage (Timestepping.cpp:141-158). */
void vto_flux_from_state(int K, int Np, const double* U, double* F);

/* forward_euler (Timestepping.cpp:39-82) and rk4 (Timestepping.cpp:85-306),
 * nsteps times, in place on U and F. Stops at the first non-physical state,
 * as the reference does (it exits), and returns its code. */
int vto_forward_euler(const vto_mesh* m, double* U, double* F, double dt, int nsteps, vto_error* err);
int vto_rk4(const vto_mesh* m, double* U, double* F, double dt, int nsteps, vto_error* err);

/* plottools/l2stateerror.py:30-98 on full-precision states: interpolate the
 * squared nodal differences to the area rule, integrate with detJ, and return
 * sqrt(integral / 25) per component in out[4]. basis_q is nqa x Np (the Lagrange
 * basis at the area points), area_quad nqa x 3 (xi, eta, weight). */
void vto_l2_state_error(int K, int Np, int nqa, const double* basis_q, const double* area_quad,
                        const double* detj, const double* Ua, const double* Ub, double* out);

/* Conservation totals sum_e detJ_e sum_i W_i U_e,i,c with W_i = sum_q w_q phi_i(q). */
void vto_totals(int K, int Np, int nqa, const double* basis_q, const double* area_quad,
                const double* detj, const double* U, double* out);

#ifdef __cplusplus
}
#endif
#endif
