/* Test infrastructure: the ORACLE (see dg_oracle.h). Never linked into the
 * product. Restates the reference's hot path over flat arrays, keeping its
 * floating-point operation order so results are bit-identical to the reference
 * built with g++ -O2 (no FMA contraction on x86-64). */
#include "dg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define GAMMA 1.4

static inline double vx(const vto_mesh* m, int n, int a) { return m->verts[(n * 3 + a) * 2 + 0]; }
static inline double vy(const vto_mesh* m, int n, int a) { return m->verts[(n * 3 + a) * 2 + 1]; }

/* Element::build_jacobians, Element.cpp:54-93 */
static void element_geometry(const vto_mesh* m, int n, double* jac, double* jinv, double* detj,
                             double* detjinv, double* nrm, double* sides) {
  const double x0 = vx(m, n, 0), y0 = vy(m, n, 0);
  const double x1 = vx(m, n, 1), y1 = vy(m, n, 1);
  const double x2 = vx(m, n, 2), y2 = vy(m, n, 2);
  jac[0] = x1 - x0;
  jac[1] = x2 - x0;
  jac[2] = y1 - y0;
  jac[3] = y2 - y0;
  const double det = jac[0] * jac[3] - jac[2] * jac[1];
  *detj = det;
  jinv[0] = (1 / det) * (y2 - y0);
  jinv[1] = (1 / det) * (x0 - x2);
  jinv[2] = (1 / det) * (y0 - y1);
  jinv[3] = (1 / det) * (x1 - x0);
  *detjinv = jinv[0] * jinv[3] - jinv[2] * jinv[1];
  const double l0 = pow(pow(x1 - x0, 2) + pow(y1 - y0, 2), 0.5);
  const double l1 = pow(pow(x2 - x1, 2) + pow(y2 - y1, 2), 0.5);
  const double l2 = pow(pow(x0 - x2, 2) + pow(y0 - y2, 2), 0.5);
  nrm[0] = (y1 - y0) / l0;
  nrm[2] = (y2 - y1) / l1;
  nrm[4] = (y0 - y2) / l2;
  nrm[1] = -1 * (x1 - x0) / l0;
  nrm[3] = -1 * (x2 - x1) / l1;
  nrm[5] = -1 * (x0 - x2) / l2;
  sides[0] = l0;
  sides[1] = l1;
  sides[2] = l2;
}

void vto_geometry(const vto_mesh* m, double* jac, double* jinv, double* detj, double* detjinv,
                  double* normals, double* sides) {
  for (int n = 0; n < m->K; ++n)
    element_geometry(m, n, jac + 4 * n, jinv + 4 * n, detj + n, detjinv + n, normals + 6 * n,
                     sides + 3 * n);
}

/* numerical_flux, Numericalflux.cpp:13-157 */
int vto_numerical_flux(const double* u_left, const double* u_right, const double* nv, double* flux) {
  const double gamma = GAMMA;
  const double gmi = gamma - 1.0;

  const double rL = u_left[0];
  const double uL = u_left[1] / rL;
  const double vL = u_left[2] / rL;
  const double unL = uL * nv[0] + vL * nv[1];
  const double qL = pow(pow(u_left[1], 2) + pow(u_left[2], 2), 0.5) / rL;
  const double pL = (gamma - 1) * (u_left[3] - 0.5 * rL * pow(qL, 2));
  if ((pL <= 0) || (rL <= 0)) return 1;
  const double rHL = u_left[3] + pL;
  const double HL = rHL / rL;
  double FL[4];
  FL[0] = rL * unL;
  FL[1] = u_left[1] * unL + pL * nv[0];
  FL[2] = u_left[2] * unL + pL * nv[1];
  FL[3] = rHL * unL;

  const double rR = u_right[0];
  const double uR = u_right[1] / rR;
  const double vR = u_right[2] / rR;
  const double unR = uR * nv[0] + vR * nv[1];
  const double qR = pow(pow(u_right[1], 2) + pow(u_right[2], 2), 0.5) / rR;
  const double pR = (gamma - 1) * (u_right[3] - 0.5 * rR * pow(qR, 2));
  if ((pR <= 0) || (rR <= 0)) return 2;
  const double rHR = u_right[3] + pR;
  const double HR = rHR / rR;
  double FR[4];
  FR[0] = rR * unR;
  FR[1] = u_right[1] * unR + pR * nv[0];
  FR[2] = u_right[2] * unR + pR * nv[1];
  FR[3] = rHR * unR;

  double du[4];
  for (int k = 0; k < 4; ++k) du[k] = u_right[k] - u_left[k];

  const double di = pow(rR / rL, 0.5);
  const double d1 = 1.0 / (1.0 + di);
  const double ui = (di * uR + uL) * d1;
  const double vi = (di * vR + vL) * d1;
  const double Hi = (di * HR + HL) * d1;
  const double af = 0.5 * (ui * ui + vi * vi);
  const double ucp = ui * nv[0] + vi * nv[1];
  const double c2 = gmi * (Hi - af);
  if (c2 <= 0) return 3;
  /* The reference squares c2 here (ci = c^4, not c); kept as is. */
  const double ci = pow(c2, 2);
  const double ci1 = 1.0 / ci;

  double l[3];
  l[0] = ucp + ci;
  l[1] = ucp - ci;
  l[2] = ucp;
  const double epsilon = ci * 0.1;
  for (int i = 0; i < 3; ++i)
    if ((l[i] < epsilon) && (l[i] > -1 * epsilon)) l[i] = 0.5 * (epsilon + l[i] * l[i] / epsilon);
  for (int i = 0; i < 3; ++i) l[i] = fabs(l[i]);
  const double l3 = l[2];
  const double s1 = 0.5 * (l[0] + l[1]);
  const double s2 = 0.5 * (l[0] - l[1]);
  const double G1 = gmi * (af * du[0] - ui * du[1] - vi * du[2] + du[3]);
  const double G2 = -1 * ucp * du[0] + du[1] * nv[0] + du[2] * nv[1];
  const double C1 = G1 * (s1 - l3) * ci1 * ci1 + G2 * s2 * ci1;
  const double C2 = G1 * s2 * ci1 + G2 * (s1 - l3);
  flux[0] = 0.5 * (FL[0] + FR[0]) - 0.5 * (l3 * du[0] + C1);
  flux[1] = 0.5 * (FL[1] + FR[1]) - 0.5 * (l3 * du[1] + C1 * ui + C2 * nv[0]);
  flux[2] = 0.5 * (FL[2] + FR[2]) - 0.5 * (l3 * du[2] + C1 * vi + C2 * nv[1]);
  flux[3] = 0.5 * (FL[3] + FR[3]) - 0.5 * (l3 * du[3] + C1 * Hi + C2 * ucp);
  return 0;
}

#define NP_MAX 10
#define NFQ_MAX 10

/* One element's DG_time_derivative_U: the six Evolve_element calls of
 * evolve_elem (Timestepping.cpp:29-34), Evolve.cpp:135-308. Returns 0 or an
 * error code, reporting the first failing (point, side) like the serial loop
 * of compute_numerical_flux (Evolve.cpp:215-221). */
static int element_rhs(const vto_mesh* m, int n, const double* U, const double* F, double* out,
                       int* fail_q, int* fail_s) {
  const int Np = m->Np, nq = m->nfq;
  double jac[4], jinv[4], det, detinv, nrm[6], sides[3];
  element_geometry(m, n, jac, jinv, &det, &detinv, nrm, sides);

  /* neighbour on each side (Evolve.cpp:167-202) */
  int nb[3];
  const int right = m->conn[3 * n + 0], left = m->conn[3 * n + 1], vert = m->conn[3 * n + 2];
  nb[0] = vert;
  if (m->type[n] == 0) { nb[1] = right; nb[2] = left; }
  else { nb[1] = left; nb[2] = right; }

  /* compute_U_plus_minus, Evolve.cpp:135-204 */
  double Up[3][NFQ_MAX][4], Um[3][NFQ_MAX][4];
  const double* Uo = U + (size_t)n * Np * 4;
  for (int q = 0; q < nq; ++q)
    for (int s = 0; s < 3; ++s) {
      const double* Un = U + (size_t)nb[s] * Np * 4;
      for (int k = 0; k < 4; ++k) {
        double ap = 0.0, am = 0.0;
        for (int j = 0; j < Np; ++j) {
          ap += m->phi_plus[(s * Np + j) * nq + q] * Uo[j * 4 + k];
          am += m->phi_minus[(s * Np + j) * nq + q] * Un[j * 4 + k];
        }
        Up[s][q][k] = ap;
        Um[s][q][k] = am;
      }
    }

  /* compute_numerical_flux, Evolve.cpp:207-222 */
  double Fl[3][NFQ_MAX][4];
  for (int q = 0; q < nq; ++q)
    for (int s = 0; s < 3; ++s) {
      const int st = vto_numerical_flux(Up[s][q], Um[s][q], nrm + 2 * s, Fl[s][q]);
      if (st) { *fail_q = q; *fail_s = s; return st; }
    }

  /* integrate_numerical_flux, Evolve.cpp:225-251 */
  double L[NP_MAX][4];
  for (int i = 0; i < Np; ++i)
    for (int k = 0; k < 4; ++k) {
      double a = 0.0;
      for (int j = 0; j < nq; ++j) {
        const double w = m->line_quad[2 * j + 1];
        a += sides[0] * m->phi_plus[(0 * Np + i) * nq + j] * Fl[0][j][k] * w;
        a += sides[1] * m->phi_plus[(1 * Np + i) * nq + j] * Fl[1][j][k] * w;
        a += sides[2] * m->phi_plus[(2 * Np + i) * nq + j] * Fl[2][j][k] * w;
      }
      L[i][k] = a;
    }

  /* Element::build_stiffness_matrix (Element.cpp:107-116) folded into
   * compute_stiffness_vector (Evolve.cpp:254-272) */
  const double* Fo = F + (size_t)n * Np * 8;
  double S[NP_MAX][4];
  for (int i = 0; i < Np; ++i)
    for (int k = 0; k < 4; ++k) {
      double a = 0.0;
      for (int j = 0; j < Np; ++j) {
        const double sxi = m->stiff_ref[(0 * Np + i) * Np + j];
        const double seta = m->stiff_ref[(1 * Np + i) * Np + j];
        const double Sx = det * (sxi * jinv[0] + seta * jinv[2]);
        const double Sy = det * (sxi * jinv[1] + seta * jinv[3]);
        a += Sx * Fo[(j * 2 + 0) * 4 + k] + Sy * Fo[(j * 2 + 1) * 4 + k];
      }
      S[i][k] = a;
    }

  /* compute_residual_vector (Evolve.cpp:275-287), then
   * Element::build_mass_matrix_inverse (Element.cpp:96-104) with
   * compute_time_derivative_U (Evolve.cpp:290-308) */
  double R[NP_MAX][4];
  for (int i = 0; i < Np; ++i)
    for (int k = 0; k < 4; ++k) R[i][k] = S[i][k] - L[i][k];
  for (int i = 0; i < Np; ++i)
    for (int k = 0; k < 4; ++k) {
      double a = 0.0;
      for (int j = 0; j < Np; ++j) a += (m->minv_ref[i * Np + j] / det) * R[j][k];
      out[i * 4 + k] = a;
    }
  return 0;
}

int vto_rhs(const vto_mesh* m, const double* U, const double* F, double* Udot, vto_error* err) {
  const int K = m->K, Np = m->Np;
  int first = K;
  int code = 0, fq = -1, fs = -1;
#pragma omp parallel for schedule(static)
  for (int n = 0; n < K; ++n) {
    int q = -1, s = -1;
    const int st = element_rhs(m, n, U, F, Udot + (size_t)n * Np * 4, &q, &s);
    if (st) {
#pragma omp critical
      {
        if (n < first) { first = n; code = st; fq = q; fs = s; }
      }
    }
  }
  if (err) {
    err->code = code;
    err->element = code ? first : -1;
    err->point = fq;
    err->side = fs;
  }
  return code;
}

/* Timestepping.cpp:141-158 (identical blocks after every stage) */
void vto_flux_from_state(int K, int Np, const double* U, double* F) {
  const double gamma = GAMMA;
#pragma omp parallel for schedule(static)
  for (int n = 0; n < K; ++n)
    for (int i = 0; i < Np; ++i) {
      const double* u = U + ((size_t)n * Np + i) * 4;
      double* f = F + ((size_t)n * Np + i) * 8;
      const double rho = u[0];
      const double uu = u[1] / rho;
      const double v = u[2] / rho;
      const double E = u[3] / rho;
      const double p = rho * (gamma - 1) * (E - (pow(uu, 2) + pow(v, 2)) / 2);
      const double H = E + p / rho;
      f[0] = rho * uu;
      f[1] = rho * pow(uu, 2) + p;
      f[2] = rho * uu * v;
      f[3] = rho * uu * H;
      f[4] = rho * v;
      f[5] = rho * uu * v;
      f[6] = rho * pow(v, 2) + p;
      f[7] = rho * v * H;
    }
}

int vto_forward_euler(const vto_mesh* m, double* U, double* F, double dt, int nsteps, vto_error* err) {
  const size_t N = (size_t)m->K * m->Np * 4;
  double* Ud = (double*)malloc(N * sizeof(double));
  int st = 0;
  for (int step = 0; step < nsteps && !st; ++step) {
    st = vto_rhs(m, U, F, Ud, err);
    if (st) break;
    /* Timestepping.cpp:51-57 */
#pragma omp parallel for schedule(static)
    for (size_t a = 0; a < N; ++a) U[a] += dt * Ud[a];
    vto_flux_from_state(m->K, m->Np, U, F);
  }
  free(Ud);
  return st;
}

int vto_rk4(const vto_mesh* m, double* U, double* F, double dt, int nsteps, vto_error* err) {
  const size_t N = (size_t)m->K * m->Np * 4;
  double* U0 = (double*)malloc(N * sizeof(double));
  double* Ud = (double*)malloc(N * sizeof(double));
  double* k1 = (double*)malloc(N * sizeof(double));
  double* k2 = (double*)malloc(N * sizeof(double));
  double* k3 = (double*)malloc(N * sizeof(double));
  int st = 0;
  for (int step = 0; step < nsteps; ++step) {
    memcpy(U0, U, N * sizeof(double)); /* Timestepping.cpp:105-114 */
    /* k1, Timestepping.cpp:125-160 */
    if ((st = vto_rhs(m, U, F, Ud, err))) break;
#pragma omp parallel for schedule(static)
    for (size_t a = 0; a < N; ++a) {
      k1[a] = dt * Ud[a];
      U[a] = U0[a] + k1[a] / 2.0;
    }
    vto_flux_from_state(m->K, m->Np, U, F);
    /* k2, Timestepping.cpp:167-202 */
    if ((st = vto_rhs(m, U, F, Ud, err))) break;
#pragma omp parallel for schedule(static)
    for (size_t a = 0; a < N; ++a) {
      k2[a] = dt * Ud[a];
      U[a] = U0[a] + k2[a] / 2.0;
    }
    vto_flux_from_state(m->K, m->Np, U, F);
    /* k3, Timestepping.cpp:209-244 */
    if ((st = vto_rhs(m, U, F, Ud, err))) break;
#pragma omp parallel for schedule(static)
    for (size_t a = 0; a < N; ++a) {
      k3[a] = dt * Ud[a];
      U[a] = U0[a] + k3[a];
    }
    vto_flux_from_state(m->K, m->Np, U, F);
    /* k4 and the combine, Timestepping.cpp:251-301 */
    if ((st = vto_rhs(m, U, F, Ud, err))) break;
#pragma omp parallel for schedule(static)
    for (size_t a = 0; a < N; ++a) {
      const double k4 = dt * Ud[a];
      U[a] = U0[a] + (1.0 / 6.0) * (k1[a] + 2 * k2[a] + 2 * k3[a] + k4);
    }
    vto_flux_from_state(m->K, m->Np, U, F);
  }
  free(U0);
  free(Ud);
  free(k1);
  free(k2);
  free(k3);
  return st;
}

/* plottools/l2stateerror.py:30-98 (p taken from the problem instead of the
 * script's hard-coded 3, states at full precision instead of 6-decimal text) */
void vto_l2_state_error(int K, int Np, int nqa, const double* basis_q, const double* area_quad,
                        const double* detj, const double* Ua, const double* Ub, double* out) {
  double integral[4] = {0, 0, 0, 0};
  for (int n = 0; n < K; ++n) {
    double del[NP_MAX][4];
    for (int j = 0; j < Np; ++j)
      for (int c = 0; c < 4; ++c) {
        const double d = Ub[((size_t)n * Np + j) * 4 + c] - Ua[((size_t)n * Np + j) * 4 + c];
        del[j][c] = d * d;
      }
    for (int c = 0; c < 4; ++c) {
      double acc = 0.0;
      for (int q = 0; q < nqa; ++q) {
        double v = 0.0;
        for (int j = 0; j < Np; ++j) v += del[j][c] * basis_q[q * Np + j];
        acc += area_quad[3 * q + 2] * v;
      }
      integral[c] += detj[n] * acc;
    }
  }
  for (int c = 0; c < 4; ++c) out[c] = sqrt((1.0 / 25.0) * integral[c]);
}

void vto_totals(int K, int Np, int nqa, const double* basis_q, const double* area_quad,
                const double* detj, const double* U, double* out) {
  double W[NP_MAX];
  for (int j = 0; j < Np; ++j) {
    double a = 0.0;
    for (int q = 0; q < nqa; ++q) a += area_quad[3 * q + 2] * basis_q[q * Np + j];
    W[j] = a;
  }
  long double tot[4] = {0, 0, 0, 0};
  for (int n = 0; n < K; ++n)
    for (int c = 0; c < 4; ++c) {
      double a = 0.0;
      for (int j = 0; j < Np; ++j) a += W[j] * U[((size_t)n * Np + j) * 4 + c];
      tot[c] += (long double)detj[n] * a;
    }
  for (int c = 0; c < 4; ++c) out[c] = (double)tot[c];
}
