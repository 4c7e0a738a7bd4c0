// Host precompute; see vt_precompute.h. Each block cites the reference lines it
// restates. Expressions keep the reference's evaluation order and its
// float/double conversions, because the operators feed a solver whose results
// are compared with the reference's to 1e-12.
#include "vt_precompute.h"

#include <cmath>
#include <cstdlib>
#include <sstream>
#include <stdexcept>
#include <unordered_map>

namespace vt {

// ---------------------------------------------------------------------------
// Parameters.cpp:12-64
// ---------------------------------------------------------------------------
int parse_input_text(const std::string& text, vt_params* out, std::string* msg) {
  std::unordered_map<std::string, std::string> kv;
  std::istringstream in(text);
  std::string line;
  while (std::getline(in, line)) {
    const size_t pos = line.find('=');
    if (pos != std::string::npos) kv[line.substr(0, pos)] = line.substr(pos + 1);
  }
  const char* key = "";
  try {
    vt_params p;
    key = "p"; p.p = std::stoi(kv[key]);
    key = "domain_x"; p.domain_x = std::stof(kv[key]);
    key = "domain_y"; p.domain_y = std::stof(kv[key]);
    key = "num_element_in_x"; p.num_element_in_x = std::stoi(kv[key]);
    key = "num_element_in_y"; p.num_element_in_y = std::stoi(kv[key]);
    // std::stoi, as the reference does: "0.2" reads as 0 (Parameters.cpp:55).
    key = "perturb_grid"; p.perturb_grid = static_cast<float>(std::stoi(kv[key]));
    key = "integration_order"; p.integration_order = std::stoi(kv[key]);
    key = "simulation_time"; p.simulation_time = std::stof(kv[key]);
    key = "number_time_steps"; p.number_time_steps = std::stoi(kv[key]);
    key = "simulation_time";
    p.time_step = std::stod(kv["simulation_time"]) / std::stod(kv["number_time_steps"]);
    key = "write_every_steps"; p.write_every_steps = std::stoi(kv[key]);
    key = "U_initialization_type"; p.U_initialization_type = std::stoi(kv[key]);
    key = "stepping_method"; p.stepping_method = std::stoi(kv[key]);
    *out = p;
  } catch (const std::exception&) {
    if (msg) *msg = std::string("input file: missing or malformed key '") + key + "'";
    return VT_ERR_INVALID;
  }
  return VT_OK;
}

// ---------------------------------------------------------------------------
// Quadrature tables. These have to equal the reference's to the last digit
// (Quadraturerule.cpp:13-181 and :183-662): they are the published
// Gauss-Legendre and Dunavant (1985) values rounded to 15 decimals, and the
// operators built from them are compared bit for bit.
// ---------------------------------------------------------------------------
namespace {

struct LineRule {
  int n;
  double x[10], w[10];
};

const LineRule kLine[10] = {
    {1, {0.500000000000000}, {1.000000000000000}},
    {2, {0.211324865405187, 0.788675134594813}, {0.500000000000000, 0.500000000000000}},
    {3, {0.112701665379258, 0.500000000000000, 0.887298334620742},
     {0.277777777777778, 0.444444444444444, 0.277777777777778}},
    {4, {0.069431844202974, 0.330009478207572, 0.669990521792428, 0.930568155797026},
     {0.173927422568727, 0.326072577431273, 0.326072577431273, 0.173927422568727}},
    {5, {0.046910077030668, 0.230765344947158, 0.500000000000000, 0.769234655052841,
         0.953089922969332},
     {0.118463442528095, 0.239314335249683, 0.284444444444444, 0.239314335249683,
      0.118463442528095}},
    {6, {0.033765242898424, 0.169395306766868, 0.380690406958402, 0.619309593041598,
         0.830604693233132, 0.966234757101576},
     {0.085662246189585, 0.180380786524069, 0.233956967286345, 0.233956967286345,
      0.180380786524069, 0.085662246189585}},
    {7, {0.025446043828621, 0.129234407200303, 0.297077424311301, 0.500000000000000,
         0.702922575688699, 0.870765592799697, 0.974553956171379},
     {0.064742483084435, 0.139852695744638, 0.190915025252560, 0.208979591836735,
      0.190915025252560, 0.139852695744638, 0.064742483084435}},
    {8, {0.019855071751232, 0.101666761293187, 0.237233795041836, 0.408282678752175,
         0.591717321247825, 0.762766204958164, 0.898333238706813, 0.980144928248768},
     {0.050614268145188, 0.111190517226687, 0.156853322938944, 0.181341891689181,
      0.181341891689181, 0.156853322938944, 0.111190517226687, 0.050614268145188}},
    {9, {0.015919880246187, 0.081984446336682, 0.193314283649705, 0.337873288298096,
         0.500000000000000, 0.662126711701905, 0.806685716350295, 0.918015553663318,
         0.984080119753813},
     {0.040637194180787, 0.090324080347429, 0.130305348201468, 0.156173538520001,
      0.165119677500630, 0.156173538520001, 0.130305348201468, 0.090324080347429,
      0.040637194180787}},
    {10, {0.013046735741414, 0.067468316655508, 0.160295215850488, 0.283302302935376,
          0.425562830509184, 0.574437169490816, 0.716697697064624, 0.839704784149512,
          0.932531683344492, 0.986953264258586},
     {0.033335672154344, 0.074725674575290, 0.109543181257991, 0.134633359654998,
      0.147762112357376, 0.147762112357376, 0.134633359654998, 0.109543181257991,
      0.074725674575290, 0.033335672154344}},
};

// A Dunavant rule as symmetry orbits. kind 1: centroid (a, a); kind 3: the
// points (a,b), (b,b), (b,a); kind 6: (a,b), (b,c), (c,a), (b,a), (c,b), (a,c).
// This expansion order is the order of the reference's point lists.
struct Orbit {
  int kind;
  double a, b, c, w;
};

struct AreaRule {
  int norbits;
  Orbit o[6];
};

constexpr double kThird = 0.333333333333333;

const AreaRule kArea[10] = {
    {1, {{1, kThird, 0, 0, 0.500000000000000}}},
    {1, {{3, 0.666666666666667, 0.166666666666667, 0, 0.166666666666666}}},
    {2, {{1, kThird, 0, 0, -0.281250000000000}, {3, 0.6, 0.2, 0, 0.260416666666667}}},
    {2, {{3, 0.108103018168070, 0.445948490915965, 0, 0.111690794839005},
         {3, 0.816847572980459, 0.091576213509771, 0, 0.054975871827661}}},
    {3, {{1, kThird, 0, 0, 0.112500000000000},
         {3, 0.059715871789770, 0.470142064105115, 0, 0.066197076394253},
         {3, 0.797426985353087, 0.101286507323456, 0, 0.062969590272414}}},
    {3, {{3, 0.501426509658179, 0.249286745170910, 0, 0.058393137863189},
         {3, 0.873821971016996, 0.063089014491502, 0, 0.025422453185103},
         {6, 0.053145049844817, 0.310352451033784, 0.636502499121399, 0.041425537809187}}},
    {4, {{1, kThird, 0, 0, -0.074785022233841},
         {3, 0.479308067841920, 0.260345966079040, 0, 0.087807628716604},
         {3, 0.869739794195568, 0.065130102902216, 0, 0.026673617804419},
         {6, 0.048690315425316, 0.312865496004874, 0.638444188569810, 0.038556880445128}}},
    {5, {{1, kThird, 0, 0, 0.072157803838894},
         {3, 0.081414823414554, 0.459292588292723, 0, 0.047545817133642},
         {3, 0.658861384496480, 0.170569307751760, 0, 0.051608685267359},
         {3, 0.898905543365938, 0.050547228317031, 0, 0.016229248811599},
         {6, 0.008394777409958, 0.263112829634638, 0.728492392955404, 0.013615157087217}}},
    {6, {{1, kThird, 0, 0, 0.048567898141400},
         {3, 0.020634961602525, 0.489682519198738, 0, 0.015667350113570},
         {3, 0.125820817014127, 0.437089591492937, 0, 0.038913770502387},
         {3, 0.623592928761935, 0.188203535619033, 0, 0.039823869463605},
         {3, 0.910540973211095, 0.044729513394453, 0, 0.012788837829349},
         {6, 0.036838412054736, 0.221962989160766, 0.741198598784498, 0.021641769688645}}},
    {6, {{1, kThird, 0, 0, 0.045408995191377},
         {3, 0.028844733232685, 0.485577633383657, 0, 0.018362978878233},
         {3, 0.781036849029926, 0.109481575485037, 0, 0.022660529717764},
         {6, 0.141707219414880, 0.307939838764121, 0.550352941820999, 0.036378958422710},
         {6, 0.025003534762686, 0.246672560639903, 0.728323904597411, 0.014163621265528},
         {6, 0.009540815400299, 0.066803251012200, 0.923655933587500, 0.004710833481867}}},
};

}  // namespace

bool line_rule(int io, std::vector<double>* rows) {
  if (io < 0 || io > 19) return false;
  // IntOrder2Rule (Quadraturerule.cpp:125): order 2k and 2k+1 -> k+1 points.
  const LineRule& r = kLine[io / 2];
  rows->resize(2 * r.n);
  for (int i = 0; i < r.n; ++i) {
    (*rows)[2 * i] = r.x[i];
    (*rows)[2 * i + 1] = r.w[i];
  }
  return true;
}

bool area_rule(int io, std::vector<double>* rows) {
  if (io < 0 || io > 19) return false;
  // IntOrder2Rule (Quadraturerule.cpp:590) is the identity above order 1 up to
  // order 10. Orders 11-19 select rules 12-19 in the reference; the degree-10
  // rule used here instead already integrates every p <= 3 mass and stiffness
  // integrand (degree <= 6) exactly, so only the 15-digit table rounding differs.
  const int rule = io <= 1 ? 1 : (io <= 10 ? io : 10);
  const AreaRule& r = kArea[rule - 1];
  rows->clear();
  auto push = [&](double x, double y, double w) {
    rows->push_back(x);
    rows->push_back(y);
    rows->push_back(w);
  };
  for (int k = 0; k < r.norbits; ++k) {
    const Orbit& o = r.o[k];
    if (o.kind == 1) {
      push(o.a, o.a, o.w);
    } else if (o.kind == 3) {
      push(o.a, o.b, o.w);
      push(o.b, o.b, o.w);
      push(o.b, o.a, o.w);
    } else {
      push(o.a, o.b, o.w);
      push(o.b, o.c, o.w);
      push(o.c, o.a, o.w);
      push(o.b, o.a, o.w);
      push(o.c, o.b, o.w);
      push(o.a, o.c, o.w);
    }
  }
  return true;
}

// ---------------------------------------------------------------------------
// Lagrangebasis.cpp:12-147. The equispaced Lagrange polynomials on the
// reference triangle, written term by term in the reference's order so that
// the evaluated values are identical.
// ---------------------------------------------------------------------------
bool basis(int p, double xi, double eta, double* phi) {
  switch (p) {
    case 0:
      phi[0] = 1.0;
      return true;
    case 1:
      phi[0] = 1.0 - xi - eta;
      phi[1] = xi;
      phi[2] = eta;
      return true;
    case 2:
      phi[0] = 1.0 - 3.0 * xi - 3.0 * eta + 2.0 * xi * xi + 4.0 * xi * eta + 2.0 * eta * eta;
      phi[1] = 4.0 * xi - 4.0 * xi * xi - 4.0 * xi * eta;
      phi[2] = -xi + 2.0 * xi * xi;
      phi[3] = 4.0 * eta - 4.0 * xi * eta - 4.0 * eta * eta;
      phi[4] = 4.0 * xi * eta;
      phi[5] = -eta + 2.0 * eta * eta;
      return true;
    case 3:
      phi[0] = 1.0 - 11.0 / 2.0 * xi - 11.0 / 2.0 * eta + 9.0 * xi * xi + 18.0 * xi * eta +
               9.0 * eta * eta - 9.0 / 2.0 * xi * xi * xi - 27.0 / 2.0 * xi * xi * eta -
               27.0 / 2.0 * xi * eta * eta - 9.0 / 2.0 * eta * eta * eta;
      phi[1] = 9.0 * xi - 45.0 / 2.0 * xi * xi - 45.0 / 2.0 * xi * eta + 27.0 / 2.0 * xi * xi * xi +
               27.0 * xi * xi * eta + 27.0 / 2.0 * xi * eta * eta;
      phi[2] = -9.0 / 2.0 * xi + 18.0 * xi * xi + 9.0 / 2.0 * xi * eta - 27.0 / 2.0 * xi * xi * xi -
               27.0 / 2.0 * xi * xi * eta;
      phi[3] = xi - 9.0 / 2.0 * xi * xi + 9.0 / 2.0 * xi * xi * xi;
      phi[4] = 9.0 * eta - 45.0 / 2.0 * xi * eta - 45.0 / 2.0 * eta * eta +
               27.0 / 2.0 * xi * xi * eta + 27.0 * xi * eta * eta + 27.0 / 2.0 * eta * eta * eta;
      phi[5] = 27.0 * xi * eta - 27.0 * xi * xi * eta - 27.0 * xi * eta * eta;
      phi[6] = -9.0 / 2.0 * xi * eta + 27.0 / 2.0 * xi * xi * eta;
      phi[7] = -9.0 / 2.0 * eta + 9.0 / 2.0 * xi * eta + 18.0 * eta * eta -
               27.0 / 2.0 * xi * eta * eta - 27.0 / 2.0 * eta * eta * eta;
      phi[8] = -9.0 / 2.0 * xi * eta + 27.0 / 2.0 * xi * eta * eta;
      phi[9] = eta - 9.0 / 2.0 * eta * eta + 9.0 / 2.0 * eta * eta * eta;
      return true;
    default:
      return false;
  }
}

bool basis_gradient(int p, double xi, double eta, double* g) {
  // g[2*j + d]: d 0 = d/dxi, 1 = d/deta
  switch (p) {
    case 0:
      g[0] = 0.0;
      g[1] = 0.0;
      return true;
    case 1:
      g[0] = -1.0; g[2] = 1.0; g[4] = 0.0;
      g[1] = -1.0; g[3] = 0.0; g[5] = 1.0;
      return true;
    case 2:
      g[0] = -3.0 + 4.0 * xi + 4.0 * eta;
      g[2] = 4.0 - 8.0 * xi - 4.0 * eta;
      g[4] = -1.0 + 4.0 * xi;
      g[6] = -4.0 * eta;
      g[8] = 4.0 * eta;
      g[10] = 0.0;
      g[1] = -3.0 + 4.0 * xi + 4.0 * eta;
      g[3] = -4.0 * xi;
      g[5] = 0.0;
      g[7] = 4.0 - 4.0 * xi - 8.0 * eta;
      g[9] = 4.0 * xi;
      g[11] = -1.0 + 4.0 * eta;
      return true;
    case 3:
      g[0] = -11.0 / 2.0 + 18.0 * xi + 18.0 * eta - 27.0 / 2.0 * xi * xi - 27.0 * xi * eta -
             27.0 / 2.0 * eta * eta;
      g[2] = 9.0 - 45.0 * xi - 45.0 / 2.0 * eta + 81.0 / 2.0 * xi * xi + 54.0 * xi * eta +
             27.0 / 2.0 * eta * eta;
      g[4] = -9.0 / 2.0 + 36.0 * xi + 9.0 / 2.0 * eta - 81.0 / 2.0 * xi * xi - 27.0 * xi * eta;
      g[6] = 1.0 - 9.0 * xi + 27.0 / 2.0 * xi * xi;
      g[8] = -45.0 / 2.0 * eta + 27.0 * xi * eta + 27.0 * eta * eta;
      g[10] = 27.0 * eta - 54.0 * xi * eta - 27.0 * eta * eta;
      g[12] = -9.0 / 2.0 * eta + 27.0 * xi * eta;
      g[14] = 9.0 / 2.0 * eta - 27.0 / 2.0 * eta * eta;
      g[16] = -9.0 / 2.0 * eta + 27.0 / 2.0 * eta * eta;
      g[18] = 0.0;
      g[1] = -11.0 / 2.0 + 18.0 * xi + 18.0 * eta - 27.0 / 2.0 * xi * xi - 27.0 * xi * eta -
             27.0 / 2.0 * eta * eta;
      g[3] = -45.0 / 2.0 * xi + 27.0 * xi * xi + 27.0 * xi * eta;
      g[5] = 9.0 / 2.0 * xi - 27.0 / 2.0 * xi * xi;
      g[7] = 0.0;
      g[9] = 9.0 - 45.0 / 2.0 * xi - 45.0 * eta + 27.0 / 2.0 * xi * xi + 54.0 * xi * eta +
             81.0 / 2.0 * eta * eta;
      g[11] = 27.0 * xi - 27.0 * xi * xi - 54.0 * xi * eta;
      g[13] = -9.0 / 2.0 * xi + 27.0 / 2.0 * xi * xi;
      g[15] = -9.0 / 2.0 + 9.0 / 2.0 * xi + 36.0 * eta - 27.0 * xi * eta - 81.0 / 2.0 * eta * eta;
      g[17] = -9.0 / 2.0 * xi + 27.0 * xi * eta;
      g[19] = 1.0 - 9.0 * eta + 27.0 / 2.0 * eta * eta;
      return true;
    default:
      return false;
  }
}

std::vector<double> reference_nodes(int p) {
  std::vector<double> r(2 * np_of(p), 0.0);
  if (p == 0) return r;  // single node at (0, 0)
  const double h = 1.0 / p;
  int c = 0;
  for (int j = 0; j < p + 1; ++j)
    for (int i = 0; i < p + 1; ++i)
      if (i + j < p + 1) {
        r[2 * c] = h * i;
        r[2 * c + 1] = h * j;
        ++c;
      }
  return r;
}

// ---------------------------------------------------------------------------
// Preevolve.cpp:15-144
// ---------------------------------------------------------------------------
bool invert_gauss_jordan(int n, std::vector<double>* m) {
  std::vector<double>& a = *m;
  std::vector<double> inv(static_cast<size_t>(n) * n, 0.0);
  for (int i = 0; i < n; ++i) inv[i * n + i] = 1.0;
  for (int col = 0; col < n; ++col) {
    int piv = col;
    double best = std::fabs(a[col * n + col]);
    for (int r = col + 1; r < n; ++r) {
      const double v = std::fabs(a[r * n + col]);
      if (v > best) {
        best = v;
        piv = r;
      }
    }
    if (best == 0.0) return false;
    if (piv != col)
      for (int j = 0; j < n; ++j) {
        std::swap(a[col * n + j], a[piv * n + j]);
        std::swap(inv[col * n + j], inv[piv * n + j]);
      }
    const double d = a[col * n + col];
    for (int j = 0; j < n; ++j) {
      a[col * n + j] /= d;
      inv[col * n + j] /= d;
    }
    for (int r = 0; r < n; ++r) {
      if (r == col) continue;
      const double f = a[r * n + col];
      if (f == 0.0) continue;
      for (int j = 0; j < n; ++j) {
        a[r * n + j] -= f * a[col * n + j];
        inv[r * n + j] -= f * inv[col * n + j];
      }
    }
  }
  a.swap(inv);
  return true;
}

bool inverse_mass_reference(int p, const std::vector<double>& area, std::vector<double>* minv) {
  const int Np = np_of(p), nq = static_cast<int>(area.size() / 3);
  std::vector<double> phi(static_cast<size_t>(Np) * nq), tmp(Np);
  for (int q = 0; q < nq; ++q) {
    basis(p, area[3 * q], area[3 * q + 1], tmp.data());
    for (int j = 0; j < Np; ++j) phi[j * nq + q] = tmp[j];
  }
  std::vector<double> mass(static_cast<size_t>(Np) * Np);
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Np; ++j) {
      double s = 0;
      for (int n = 0; n < nq; ++n) s += phi[i * nq + n] * phi[j * nq + n] * area[3 * n + 2];
      mass[i * Np + j] = s;
    }
  const bool ok = invert_gauss_jordan(Np, &mass);
  minv->swap(mass);
  return ok;
}

std::vector<double> stiffness_reference(int p, const std::vector<double>& area) {
  const int Np = np_of(p), nq = static_cast<int>(area.size() / 3);
  std::vector<double> phi(static_cast<size_t>(Np) * nq), grad(static_cast<size_t>(Np) * nq * 2);
  std::vector<double> t1(Np), t2(2 * Np);
  for (int q = 0; q < nq; ++q) {
    basis(p, area[3 * q], area[3 * q + 1], t1.data());
    basis_gradient(p, area[3 * q], area[3 * q + 1], t2.data());
    for (int j = 0; j < Np; ++j) {
      phi[j * nq + q] = t1[j];
      grad[(j * nq + q) * 2 + 0] = t2[2 * j + 0];
      grad[(j * nq + q) * 2 + 1] = t2[2 * j + 1];
    }
  }
  std::vector<double> s(2 * static_cast<size_t>(Np) * Np);
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Np; ++j) {
      double s0 = 0, s1 = 0;
      for (int n = 0; n < nq; ++n) {
        s0 += grad[(i * nq + n) * 2 + 0] * phi[j * nq + n] * area[3 * n + 2];
        s1 += grad[(i * nq + n) * 2 + 1] * phi[j * nq + n] * area[3 * n + 2];
      }
      s[(0 * Np + i) * Np + j] = s0;
      s[(1 * Np + i) * Np + j] = s1;
    }
  return s;
}

// ---------------------------------------------------------------------------
// Meshgeneration.cpp:16-186. Note the float arithmetic the reference does on
// its float parameters (domain size, perturbation) before widening to double.
// ---------------------------------------------------------------------------
Mesh generate_mesh(const vt_params& prm) {
  Mesh m;
  const int nx = prm.num_element_in_x, ny = prm.num_element_in_y;
  m.nx = nx;
  m.ny = ny;
  m.K = 2 * nx * ny;
  std::vector<double> gx(nx + 1), gy(ny + 1);
  const double esx = prm.domain_x / nx;  // float division, widened
  const double esy = prm.domain_y / ny;
  for (int i = 0; i < nx + 1; ++i) gx[i] = -1 * prm.domain_x / 2 + esx * i;
  for (int i = 0; i < ny + 1; ++i) gy[i] = -1 * prm.domain_y / 2 + esy * i;

  std::vector<double> px(static_cast<size_t>(nx + 1) * (ny + 1)), py(px.size());
  int c = 0;
  for (int i = 0; i < ny + 1; ++i)
    for (int j = 0; j < nx + 1; ++j) {
      const int inner = (i == 0 ? 0 : 1) * (i == ny ? 0 : 1) * (j == 0 ? 0 : 1) * (j == nx ? 0 : 1);
      px[c] = gx[j] + inner * prm.perturb_grid * 0.2 * esx * std::sin(std::pow(gx[j] + 6, gy[i] + 6));
      py[c] = gy[i] + inner * prm.perturb_grid * 0.2 * esy * std::cos(std::pow(gy[i] + 6, gx[j] + 6));
      ++c;
    }

  const int K = m.K;
  std::vector<int> n1(K), n2(K), n3(K);
  c = 0;
  for (int i = 1; i < ny + 1; ++i)
    for (int j = 0; j < nx; ++j) {
      n1[c++] = j + (nx + 1) * (i - 1);
      n1[c++] = (j + (nx + 1) * i) + 1;
    }
  for (int i = 0; i < K; ++i) n2[i] = n1[i] + (i % 2 == 0 ? 1 : -1);
  for (int i = 0; i < K; ++i) n3[i] = n2[(i % 2 == 0 ? i + 1 : i - 1)];

  m.type.resize(K);
  for (int i = 0; i < K; ++i) m.type[i] = (i % 2 == 0 ? 0 : 1);

  std::vector<int> left(K), right(K), vert(K);
  for (int i = 0; i < K; ++i) left[i] = (i % (2 * nx) == 0 ? i - 1 + 2 * nx : i - 1);
  for (int i = 0; i < K; ++i) right[i] = ((i + 1) % (2 * nx) == 0 ? i + 1 - 2 * nx : i + 1);
  for (int i = 0; i < 2 * nx; ++i)
    vert[i] = (i % 2 == 0 ? i + 1 + 2 * nx * (ny - 1) : i - 1 + 2 * nx);
  for (int i = 2 * nx; i < 2 * nx * (ny - 1); ++i)
    vert[i] = (i % 2 == 0 ? i + 1 - 2 * nx : i - 1 + 2 * nx);
  for (int i = 2 * nx * (ny - 1); i < K; ++i)
    vert[i] = (i % 2 == 0 ? i + 1 - 2 * nx : i - 1 - 2 * nx * (ny - 1));

  m.verts.resize(static_cast<size_t>(K) * 6);
  m.conn.resize(static_cast<size_t>(K) * 3);
  for (int i = 0; i < K; ++i) {
    const int ids[3] = {n1[i], n2[i], n3[i]};
    for (int a = 0; a < 3; ++a) {
      m.verts[(i * 3 + a) * 2 + 0] = px[ids[a]];
      m.verts[(i * 3 + a) * 2 + 1] = py[ids[a]];
    }
    m.conn[i * 3 + 0] = right[i];
    m.conn[i * 3 + 1] = left[i];
    m.conn[i * 3 + 2] = vert[i];
  }
  return m;
}

// ---------------------------------------------------------------------------
// Element.cpp:54-93
// ---------------------------------------------------------------------------
void element_geometry(const double* v, double* jac, double* jinv, double* detj, double* detjinv,
                      double* nrm, double* sides) {
  const double x0 = v[0], y0 = v[1], x1 = v[2], y1 = v[3], x2 = v[4], y2 = v[5];
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
  const double l0 = std::pow(std::pow(x1 - x0, 2) + std::pow(y1 - y0, 2), 0.5);
  const double l1 = std::pow(std::pow(x2 - x1, 2) + std::pow(y2 - y1, 2), 0.5);
  const double l2 = std::pow(std::pow(x0 - x2, 2) + std::pow(y0 - y2, 2), 0.5);
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

// ---------------------------------------------------------------------------
// Evolve.cpp:76-132
// ---------------------------------------------------------------------------
void face_tables(int p, const std::vector<double>& line, std::vector<double>* plus,
                 std::vector<double>* minus) {
  const int Np = np_of(p), nq = static_cast<int>(line.size() / 2);
  plus->assign(3 * static_cast<size_t>(Np) * nq, 0.0);
  minus->assign(plus->size(), 0.0);
  double ph[6][10];
  for (int q = 0; q < nq; ++q) {
    const double s = line[2 * q];
    basis(p, s, 0.0, ph[0]);
    basis(p, 1.0 - s, 0.0, ph[1]);
    basis(p, 1.0 - s, s, ph[2]);
    basis(p, s, 1.0 - s, ph[3]);
    basis(p, 0.0, 1.0 - s, ph[4]);
    basis(p, 0.0, s, ph[5]);
    for (int side = 0; side < 3; ++side)
      for (int j = 0; j < Np; ++j) {
        (*plus)[(side * Np + j) * nq + q] = ph[2 * side][j];
        (*minus)[(side * Np + j) * nq + q] = ph[2 * side + 1][j];
      }
  }
}

// ---------------------------------------------------------------------------
// Element.cpp:119-333
// ---------------------------------------------------------------------------
vt_vortex default_vortex() {
  vt_vortex v;
  v.rho_infty = 1.0;
  v.rc = 1.0;
  v.epsilon = 0.3;
  v.gamma = 1.4;
  v.M_infty = 0.5;
  v.p_infty = 20.0 / 7.0;
  v.U_infty = 1.0 / std::pow(2.0, 0.5);
  v.V_infty = 1.0 / std::pow(2.0, 0.5);
  v.x0 = 0.0;
  v.y0 = 0.0;
  return v;
}

namespace {

// Element.cpp:151-160: the vortex's primitive state at (x, y, t).
void vortex_state(const vt_vortex& c, double x, double y, double t, double* rho, double* u,
                  double* v, double* p) {
  const double f0 = 1.0 - (std::pow(x - c.x0 - c.U_infty * t, 2.0) +
                           std::pow(y - c.y0 - c.V_infty * t, 2.0)) / std::pow(c.rc, 2.0);
  const double f1 = 1.0 - std::pow(c.epsilon, 2.0) * (c.gamma - 1) * std::pow(c.M_infty, 2.0) *
                              std::exp(f0) / (8.0 * std::pow(M_PI, 2.0));
  const double f2 = c.epsilon * (std::pow(c.U_infty, 2.0) + std::pow(c.V_infty, 2.0)) *
                    std::exp(f0 / 2.0) / (2.0 * M_PI * c.rc);
  *rho = c.rho_infty * std::pow(f1, 1.0 / (c.gamma - 1.0));
  *u = c.U_infty - f2 * (y - c.y0 - c.V_infty * t);
  *v = c.V_infty + f2 * (x - c.x0 - c.U_infty * t);
  *p = c.p_infty * std::pow(f1, c.gamma / (c.gamma - 1.0));
}

void reference_to_physical(const double* vtx, double xi, double eta, double* x, double* y) {
  // Lagrangebasis.cpp:150-165 with the p = 1 basis
  const double ph0 = 1.0 - xi - eta, ph1 = xi, ph2 = eta;
  *x = vtx[0] * ph0 + vtx[2] * ph1 + vtx[4] * ph2;
  *y = vtx[1] * ph0 + vtx[3] * ph1 + vtx[5] * ph2;
}

}  // namespace

void exact_vortex(const vt_params& prm, const vt_vortex& ic, const std::vector<double>& nodes_phys, double t,
                  double* U) {
  const double Lx = prm.domain_x, Ly = prm.domain_y;
  const size_t n = nodes_phys.size() / 2;
  for (size_t a = 0; a < n; ++a) {
    double x = nodes_phys[2 * a], y = nodes_phys[2 * a + 1];
    // shift the node by whole periods so it lies within half a period of the centre
    x -= Lx * std::nearbyint((x - ic.x0 - ic.U_infty * t) / Lx);
    y -= Ly * std::nearbyint((y - ic.y0 - ic.V_infty * t) / Ly);
    double rho, u, v, pr;
    vortex_state(ic, x, y, t, &rho, &u, &v, &pr);
    const double E = pr / (rho * (ic.gamma - 1.0)) + (std::pow(u, 2.0) + std::pow(v, 2.0)) / 2.0;
    U[4 * a + 0] = rho;
    U[4 * a + 1] = rho * u;
    U[4 * a + 2] = rho * v;
    U[4 * a + 3] = rho * E;
  }
}

void flux_from_state(int K, int Np, const double* U, double* F) {
  const double gamma = 1.4;
  for (size_t a = 0; a < static_cast<size_t>(K) * Np; ++a) {
    const double* s = U + 4 * a;
    double* f = F + 8 * a;
    const double rho = s[0];
    const double u = s[1] / rho;
    const double v = s[2] / rho;
    const double E = s[3] / rho;
    const double p = rho * (gamma - 1) * (E - (std::pow(u, 2) + std::pow(v, 2)) / 2);
    const double H = E + p / rho;
    f[0] = rho * u;
    f[1] = rho * std::pow(u, 2) + p;
    f[2] = rho * u * v;
    f[3] = rho * u * H;
    f[4] = rho * v;
    f[5] = rho * u * v;
    f[6] = rho * std::pow(v, 2) + p;
    f[7] = rho * v * H;
  }
}

int initial_condition(const vt_params& prm, const vt_vortex& ic, const Mesh& mesh,
                      const std::vector<double>& nodes_ref, const std::vector<double>& area,
                      const std::vector<double>& minv_ref, double time, std::vector<double>* U,
                      std::vector<double>* F, std::vector<double>* nodes_phys) {
  const int K = mesh.K, p = prm.p, Np = np_of(p);
  U->assign(static_cast<size_t>(K) * Np * 4, 0.0);
  F->assign(static_cast<size_t>(K) * Np * 8, 0.0);
  nodes_phys->assign(static_cast<size_t>(K) * Np * 2, 0.0);
  for (int n = 0; n < K; ++n) {
    const double* vtx = &mesh.verts[static_cast<size_t>(n) * 6];
    for (int i = 0; i < Np; ++i)  // Element.cpp:48-50
      reference_to_physical(vtx, nodes_ref[2 * i], nodes_ref[2 * i + 1],
                            &(*nodes_phys)[(static_cast<size_t>(n) * Np + i) * 2],
                            &(*nodes_phys)[(static_cast<size_t>(n) * Np + i) * 2 + 1]);
  }
  if (prm.U_initialization_type == 0) {
    // direct nodal interpolation, Element.cpp:124-179
    for (int n = 0; n < K; ++n)
      for (int i = 0; i < Np; ++i) {
        const size_t a = static_cast<size_t>(n) * Np + i;
        double rho, u, v, pr;
        vortex_state(ic, (*nodes_phys)[2 * a], (*nodes_phys)[2 * a + 1], time, &rho, &u, &v, &pr);
        const double E = pr / (rho * (ic.gamma - 1.0)) + (std::pow(u, 2.0) + std::pow(v, 2.0)) / 2.0;
        const double H = E + pr / rho;
        double* s = &(*U)[4 * a];
        double* f = &(*F)[8 * a];
        s[0] = rho;
        s[1] = rho * u;
        s[2] = rho * v;
        s[3] = rho * E;
        f[0] = rho * u;
        f[1] = rho * std::pow(u, 2) + pr;
        f[2] = rho * u * v;
        f[3] = rho * u * H;
        f[4] = rho * v;
        f[5] = rho * u * v;
        f[6] = rho * std::pow(v, 2) + pr;
        f[7] = rho * v * H;
      }
    return VT_OK;
  }
  if (prm.U_initialization_type == 1) {
    // L2 projection, Element.cpp:180-326
    const int nq = static_cast<int>(area.size() / 3);
    std::vector<double> phi(static_cast<size_t>(Np) * nq), tmp(Np), ue(static_cast<size_t>(nq) * 4);
    for (int q = 0; q < nq; ++q) {
      basis(p, area[3 * q], area[3 * q + 1], tmp.data());
      for (int j = 0; j < Np; ++j) phi[j * nq + q] = tmp[j];
    }
    for (int n = 0; n < K; ++n) {
      const double* vtx = &mesh.verts[static_cast<size_t>(n) * 6];
      double jac[4], jinv[4], det, detinv, nrm[6], sides[3];
      element_geometry(vtx, jac, jinv, &det, &detinv, nrm, sides);
      for (int q = 0; q < nq; ++q) {
        double x, y, rho, u, v, pr;
        reference_to_physical(vtx, area[3 * q], area[3 * q + 1], &x, &y);
        vortex_state(ic, x, y, time, &rho, &u, &v, &pr);
        const double E = pr / (rho * (ic.gamma - 1.0)) + (std::pow(u, 2.0) + std::pow(v, 2.0)) / 2.0;
        ue[4 * q + 0] = rho;
        ue[4 * q + 1] = rho * u;
        ue[4 * q + 2] = rho * v;
        ue[4 * q + 3] = rho * E;
      }
      double b[10][4];
      for (int i = 0; i < Np; ++i)
        for (int k = 0; k < 4; ++k) {
          double s = 0.0;
          for (int j = 0; j < nq; ++j) s += det * phi[i * nq + j] * ue[4 * j + k] * area[3 * j + 2];
          b[i][k] = s;
        }
      for (int i = 0; i < Np; ++i)
        for (int k = 0; k < 4; ++k) {
          double s = 0.0;
          for (int j = 0; j < Np; ++j) s += (minv_ref[i * Np + j] / det) * b[j][k];
          (*U)[(static_cast<size_t>(n) * Np + i) * 4 + k] = s;
        }
    }
    // Element.cpp:306-323 uses the IC's gamma in the flux formula
    const double gamma = ic.gamma;
    for (size_t a = 0; a < static_cast<size_t>(K) * Np; ++a) {
      const double* s = &(*U)[4 * a];
      double* f = &(*F)[8 * a];
      const double rho = s[0];
      const double u = s[1] / rho;
      const double v = s[2] / rho;
      const double E = s[3] / rho;
      const double pr = rho * (gamma - 1) * (E - (std::pow(u, 2) + std::pow(v, 2)) / 2);
      const double H = E + pr / rho;
      f[0] = rho * u;
      f[1] = rho * std::pow(u, 2) + pr;
      f[2] = rho * u * v;
      f[3] = rho * u * H;
      f[4] = rho * v;
      f[5] = rho * u * v;
      f[6] = rho * std::pow(v, 2) + pr;
      f[7] = rho * v * H;
    }
    return VT_OK;
  }
  return VT_ERR_UNSUPPORTED;
}

}  // namespace vt
