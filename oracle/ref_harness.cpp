// Test infrastructure: driver around the UNMODIFIED reference sources.
//
// Built by oracle/Makefile into oracle/_ref/vt_ref_harness from the reference's
// own translation units (Meshgeneration, Element, Lagrangebasis,
// Quadraturerule, Preevolve, Evolve, Numericalflux, Timestepping, Parameters).
// It replaces only two things:
//   * main.cpp:81-197 -> this file: same init sequence (main.cpp:96-147) and
//     the same time loop (main.cpp:154-170), minus the text dumps;
//   * Utilities.cpp (text output, `rm -rf` via system()) -> no-op stubs below,
//     because per-element text files are out of scope and would dominate the
//     run time on large meshes.
// It dumps every precomputed operator and the state at full precision as raw
// little-endian binary files (the reference's own dumps are 6-decimal text,
// Element.cpp:346-361), which is how the golden fixtures under tests/golden/
// are produced and how the reference's CPU speed is timed.
//
// Options (all optional; defaults reproduce input_files/input except
// integration_order=10):
//   --input FILE      parse FILE with the reference's read_input_files
//                     (Parameters.cpp:12-64); later options override it
//   --nx N --ny N --p P --io IO --domain-x X --domain-y Y
//   --perturb F       float perturb_grid (bypasses std::stoi, Parameters.cpp:55)
//   --init-type T     U_initialization_type (0 nodal, 1 L2 projection)
//   --stepping M      0 forward Euler, 1 RK4
//   --dt DT           time step (default simulation_time / number_time_steps)
//   --steps N         number of steps
//   --load-state DIR  replace the initial U (and F) by DIR/U0.f64 (+ F0.f64)
//   --dump DIR        write binary dumps into DIR
//   --dump-every N    also write U after every N steps (U_step<n>.f64)
//   --rhs             dump the RHS (DG_time_derivative_U) of the initial state
//   --no-ops          skip the per-element operator dumps
//   --time            print one JSON timing line for the stepping loop
//   --warmup N        with --time: N untimed steps before the timed --steps
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <sys/stat.h>

#ifdef VORTEX_USE_OPENMP
#include <omp.h>
#endif

#include "Element.H"
#include "Evolve.H"
#include "Meshgeneration.H"
#include "Parameters.H"
#include "Preevolve.H"
#include "Quadraturerule.H"
#include "Timestepping.H"
#include "Utilities.H"

// ---- Utilities.cpp replacements (I/O out of scope) -------------------------
void writeToFile(const std::string&, const std::vector<std::string>&) {}
void clean_create_directory(const std::string&) {}
void write_output(Element*, const int&, const int&) {}

namespace {

void die(const char* msg) {
  std::fprintf(stderr, "vt_ref_harness: %s\n", msg);
  std::exit(2);
}

void write_raw(const std::string& path, const void* data, size_t bytes) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) die(("cannot write " + path).c_str());
  if (bytes && std::fwrite(data, 1, bytes, f) != bytes) die("short write");
  std::fclose(f);
}

bool read_raw(const std::string& path, void* data, size_t bytes) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  const size_t got = std::fread(data, 1, bytes, f);
  std::fclose(f);
  if (got != bytes) die(("size mismatch reading " + path).c_str());
  return true;
}

void dump_f64(const std::string& dir, const char* name, const std::vector<double>& v) {
  write_raw(dir + "/" + name + ".f64", v.data(), v.size() * sizeof(double));
}

void dump_i32(const std::string& dir, const char* name, const std::vector<int>& v) {
  write_raw(dir + "/" + name + ".i32", v.data(), v.size() * sizeof(int));
}

std::vector<double> gather_U(const Element* el, int K, int Np) {
  std::vector<double> out(static_cast<size_t>(K) * Np * 4);
  for (int n = 0; n < K; ++n)
    for (int i = 0; i < Np; ++i)
      for (int k = 0; k < 4; ++k)
        out[(static_cast<size_t>(n) * Np + i) * 4 + k] = el[n].hidrodynamics_vector_U[i][k];
  return out;
}

std::vector<double> gather_F(const Element* el, int K, int Np) {
  std::vector<double> out(static_cast<size_t>(K) * Np * 8);
  for (int n = 0; n < K; ++n)
    for (int i = 0; i < Np; ++i)
      for (int d = 0; d < 2; ++d)
        for (int k = 0; k < 4; ++k)
          out[((static_cast<size_t>(n) * Np + i) * 2 + d) * 4 + k] =
              el[n].hidrodynamics_vector_F[i][d][k];
  return out;
}

}  // namespace

int main(int argc, char** argv) {
  parameters parms;
  parms.p = 3;
  parms.domain_x = 10.0f;
  parms.domain_y = 10.0f;
  parms.num_element_in_x = 8;
  parms.num_element_in_y = 8;
  parms.perturb_grid = 0.0f;
  parms.integration_order = 10;
  parms.simulation_time = 14.14213562373f;
  parms.number_time_steps = 10000;
  parms.time_step = std::stod("14.14213562373") / std::stod("10000");
  parms.write_every_steps = 250;
  parms.U_initialization_type = 0;
  parms.stepping_method = 1;

  std::string dump_dir, load_dir;
  int dump_every = 0, warmup = 0;
  bool want_rhs = false, want_ops = true, want_time = false;
  bool dt_given = false;
  double dt = 0.0;

  for (int a = 1; a < argc; ++a) {
    auto next = [&](void) -> const char* {
      if (a + 1 >= argc) die("missing option value");
      return argv[++a];
    };
    const char* o = argv[a];
    if (!std::strcmp(o, "--input")) {
      const char* path = next();
      char* fake[2] = {argv[0], const_cast<char*>(path)};
      parms = read_input_files(2, fake);
    } else if (!std::strcmp(o, "--nx")) parms.num_element_in_x = std::atoi(next());
    else if (!std::strcmp(o, "--ny")) parms.num_element_in_y = std::atoi(next());
    else if (!std::strcmp(o, "--p")) parms.p = std::atoi(next());
    else if (!std::strcmp(o, "--io")) parms.integration_order = std::atoi(next());
    else if (!std::strcmp(o, "--domain-x")) parms.domain_x = std::strtof(next(), nullptr);
    else if (!std::strcmp(o, "--domain-y")) parms.domain_y = std::strtof(next(), nullptr);
    else if (!std::strcmp(o, "--perturb")) parms.perturb_grid = std::strtof(next(), nullptr);
    else if (!std::strcmp(o, "--init-type")) parms.U_initialization_type = std::atoi(next());
    else if (!std::strcmp(o, "--stepping")) parms.stepping_method = std::atoi(next());
    else if (!std::strcmp(o, "--dt")) { dt = std::strtod(next(), nullptr); dt_given = true; }
    else if (!std::strcmp(o, "--steps")) parms.number_time_steps = std::atoi(next());
    else if (!std::strcmp(o, "--load-state")) load_dir = next();
    else if (!std::strcmp(o, "--dump")) dump_dir = next();
    else if (!std::strcmp(o, "--dump-every")) dump_every = std::atoi(next());
    else if (!std::strcmp(o, "--rhs")) want_rhs = true;
    else if (!std::strcmp(o, "--no-ops")) want_ops = false;
    else if (!std::strcmp(o, "--time")) want_time = true;
    else if (!std::strcmp(o, "--warmup")) warmup = std::atoi(next());
    else die((std::string("unknown option ") + o).c_str());
  }
  if (dt_given) parms.time_step = dt;
  if (!dump_dir.empty()) mkdir(dump_dir.c_str(), 0755);

  const int K = 2 * parms.num_element_in_x * parms.num_element_in_y;
  const int p = parms.p;
  const int Np = (p + 1) * (p + 2) / 2;

  const auto t0 = std::chrono::steady_clock::now();

  // ---- init: main.cpp:99-147 ----------------------------------------------
  mesh simulation_mesh = generate_mesh(parms);
  std::vector<std::vector<double>> gl = gauss_line_integral(parms.integration_order);
  std::vector<std::vector<double>> ga = gauss_area_integral(parms.integration_order);
  std::vector<std::vector<double>> nodes_ref = generate_nodes_reference_space(parms);
  std::vector<std::vector<double>> minv = inverse_mass_matrix_reference_space(p, ga);
  std::vector<std::vector<std::vector<double>>> stiff = sitffness_matrix_reference_space(p, ga);

  Element* elements = new Element[K];
#ifdef VORTEX_USE_OPENMP
#pragma omp parallel for default(shared) schedule(runtime)
#endif
  for (int i = 0; i < K; ++i) {
    elements[i] = Element(i, simulation_mesh, nodes_ref, p);
    elements[i].build_jacobians();
    elements[i].build_mass_matrix_inverse(minv);
    elements[i].build_stiffness_matrix(stiff);
    elements[i].initialize_hydrodinamics(parms.U_initialization_type, ga);
  }

  if (!load_dir.empty()) {
    std::vector<double> U(static_cast<size_t>(K) * Np * 4);
    if (!read_raw(load_dir + "/U0.f64", U.data(), U.size() * sizeof(double)))
      die("--load-state needs U0.f64");
    std::vector<double> F(static_cast<size_t>(K) * Np * 8);
    const bool haveF = read_raw(load_dir + "/F0.f64", F.data(), F.size() * sizeof(double));
    for (int n = 0; n < K; ++n)
      for (int i = 0; i < Np; ++i) {
        for (int k = 0; k < 4; ++k)
          elements[n].hidrodynamics_vector_U[i][k] = U[(static_cast<size_t>(n) * Np + i) * 4 + k];
        if (haveF)
          for (int d = 0; d < 2; ++d)
            for (int k = 0; k < 4; ++k)
              elements[n].hidrodynamics_vector_F[i][d][k] =
                  F[((static_cast<size_t>(n) * Np + i) * 2 + d) * 4 + k];
      }
    if (!haveF) die("--load-state needs F0.f64 as well (the reference keeps F as state)");
  }

  Evolve_element* evolve_elements = new Evolve_element[K];
#ifdef VORTEX_USE_OPENMP
#pragma omp parallel for default(shared) schedule(runtime)
#endif
  for (int i = 0; i < K; ++i) {
    evolve_elements[i] = Evolve_element(&elements[i], &elements[elements[i].right_element],
                                        &elements[elements[i].left_element],
                                        &elements[elements[i].vertical_element], gl, p);
    evolve_elements[i].evaluate_basis_in_quadrature_poits();
  }
  const auto t1 = std::chrono::steady_clock::now();

  if (!dump_dir.empty()) {
    std::vector<double> v;
    std::vector<int> iv;
    // mesh
    v.assign(static_cast<size_t>(K) * 6, 0.0);
    for (int n = 0; n < K; ++n)
      for (int a = 0; a < 3; ++a)
        for (int d = 0; d < 2; ++d) v[(n * 3 + a) * 2 + d] = simulation_mesh.element_coordinates[n][a][d];
    dump_f64(dump_dir, "vertices", v);
    iv.assign(static_cast<size_t>(K) * 3, 0);
    for (int n = 0; n < K; ++n)
      for (int a = 0; a < 3; ++a) iv[n * 3 + a] = simulation_mesh.elements_at_boundary[n][a];
    dump_i32(dump_dir, "conn", iv);
    iv.assign(simulation_mesh.element_type.begin(), simulation_mesh.element_type.end());
    dump_i32(dump_dir, "type", iv);
    // reference-space data
    v.clear();
    for (auto& r : nodes_ref) v.insert(v.end(), r.begin(), r.end());
    dump_f64(dump_dir, "nodes_ref", v);
    v.clear();
    for (auto& r : gl) v.insert(v.end(), r.begin(), r.end());
    dump_f64(dump_dir, "line_quad", v);
    v.clear();
    for (auto& r : ga) v.insert(v.end(), r.begin(), r.end());
    dump_f64(dump_dir, "area_quad", v);
    v.clear();
    for (auto& r : minv) v.insert(v.end(), r.begin(), r.end());
    dump_f64(dump_dir, "minv_ref", v);
    v.clear();
    for (auto& m : stiff)
      for (auto& r : m) v.insert(v.end(), r.begin(), r.end());
    dump_f64(dump_dir, "stiff_ref", v);
    // per-element geometry (Element.cpp:54-93)
    std::vector<double> jac(static_cast<size_t>(K) * 4), jinv(static_cast<size_t>(K) * 4),
        detj(K), detinv(K), nrm(static_cast<size_t>(K) * 6), sides(static_cast<size_t>(K) * 3),
        xyz(static_cast<size_t>(K) * Np * 2);
    for (int n = 0; n < K; ++n) {
      const Element& e = elements[n];
      for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 2; ++c) {
          jac[n * 4 + r * 2 + c] = e.jacobian[r][c];
          jinv[n * 4 + r * 2 + c] = e.inverse_jacobian[r][c];
        }
      detj[n] = e.determinant_jacobian;
      detinv[n] = e.determinant_inverse_jacobian;
      for (int s = 0; s < 3; ++s) {
        nrm[n * 6 + s * 2 + 0] = e.units_vectors_perpendicular_to_element_boundary[s][0];
        nrm[n * 6 + s * 2 + 1] = e.units_vectors_perpendicular_to_element_boundary[s][1];
        sides[n * 3 + s] = e.sides_lenght[s];
      }
      for (int i = 0; i < Np; ++i) {
        xyz[(static_cast<size_t>(n) * Np + i) * 2 + 0] = e.nods_coords_phys_space[i][0];
        xyz[(static_cast<size_t>(n) * Np + i) * 2 + 1] = e.nods_coords_phys_space[i][1];
      }
    }
    dump_f64(dump_dir, "jac", jac);
    dump_f64(dump_dir, "jinv", jinv);
    dump_f64(dump_dir, "detj", detj);
    dump_f64(dump_dir, "detjinv", detinv);
    dump_f64(dump_dir, "normals", nrm);
    dump_f64(dump_dir, "sides", sides);
    dump_f64(dump_dir, "nodes_phys", xyz);
    if (want_ops) {
      std::vector<double> mp(static_cast<size_t>(K) * Np * Np), sp(static_cast<size_t>(K) * 2 * Np * Np);
      for (int n = 0; n < K; ++n)
        for (int i = 0; i < Np; ++i)
          for (int j = 0; j < Np; ++j) {
            mp[(static_cast<size_t>(n) * Np + i) * Np + j] = elements[n].inverse_mass_matrix_physical_space[i][j];
            for (int d = 0; d < 2; ++d)
              sp[((static_cast<size_t>(n) * 2 + d) * Np + i) * Np + j] =
                  elements[n].stiffness_matrix_physical_space[d][i][j];
          }
      dump_f64(dump_dir, "minv_phys", mp);
      dump_f64(dump_dir, "stiff_phys", sp);
    }
    // face basis tables (Evolve.cpp:76-132); identical for every element
    {
      const Evolve_element& ev = evolve_elements[0];
      const int nq = static_cast<int>(gl.size());
      const std::vector<std::vector<double>>* plus[3] = {&ev.plus_phi_in_quadrature_points_side_1,
                                                         &ev.plus_phi_in_quadrature_points_side_2,
                                                         &ev.plus_phi_in_quadrature_points_side_3};
      const std::vector<std::vector<double>>* minus[3] = {&ev.minus_phi_in_quadrature_points_side_1,
                                                          &ev.minus_phi_in_quadrature_points_side_2,
                                                          &ev.minus_phi_in_quadrature_points_side_3};
      std::vector<double> pp(static_cast<size_t>(3) * Np * nq), mm(static_cast<size_t>(3) * Np * nq);
      for (int s = 0; s < 3; ++s)
        for (int j = 0; j < Np; ++j)
          for (int q = 0; q < nq; ++q) {
            pp[(s * Np + j) * nq + q] = (*plus[s])[j][q];
            mm[(s * Np + j) * nq + q] = (*minus[s])[j][q];
          }
      dump_f64(dump_dir, "phi_plus", pp);
      dump_f64(dump_dir, "phi_minus", mm);
    }
    dump_f64(dump_dir, "U0", gather_U(elements, K, Np));
    dump_f64(dump_dir, "F0", gather_F(elements, K, Np));
  }

  if (want_rhs) {
    // One RHS evaluation on the initial state, as evolve_elem does
    // (Timestepping.cpp:18-36); the reference keeps it static, so the six
    // member calls are repeated here in the same order.
    for (int n = 0; n < K; ++n) {
      evolve_elements[n].compute_U_plus_minus();
      evolve_elements[n].compute_numerical_flux();
      evolve_elements[n].integrate_numerical_flux();
      evolve_elements[n].compute_stiffness_vector();
      evolve_elements[n].compute_residual_vector();
      evolve_elements[n].compute_time_derivative_U();
    }
    if (!dump_dir.empty()) {
      std::vector<double> r(static_cast<size_t>(K) * Np * 4);
      for (int n = 0; n < K; ++n)
        for (int i = 0; i < Np; ++i)
          for (int k = 0; k < 4; ++k)
            r[(static_cast<size_t>(n) * Np + i) * 4 + k] = evolve_elements[n].DG_time_derivative_U[i][k];
      dump_f64(dump_dir, "rhs0", r);
    }
  }

  // untimed warm-up steps (first touch of the per-step temporaries)
  for (int a = 0; a < warmup; ++a) {
    if (parms.stepping_method == 0) forward_euler(elements, evolve_elements, parms.time_step, K);
    else rk4(elements, evolve_elements, parms.time_step, K);
  }

  // ---- time loop: main.cpp:154-170 ----------------------------------------
  const auto t2 = std::chrono::steady_clock::now();
  for (int a = 1; a < parms.number_time_steps + 1; ++a) {
    if (parms.stepping_method == 0) {
      forward_euler(elements, evolve_elements, parms.time_step, K);
    } else if (parms.stepping_method == 1) {
      rk4(elements, evolve_elements, parms.time_step, K);
    } else {
      die("unsupported stepping_method");
    }
    if (!dump_dir.empty() && dump_every > 0 && a % dump_every == 0) {
      dump_f64(dump_dir, ("U_step" + std::to_string(a)).c_str(), gather_U(elements, K, Np));
    }
  }
  const auto t3 = std::chrono::steady_clock::now();

  if (!dump_dir.empty()) {
    dump_f64(dump_dir, "U_final", gather_U(elements, K, Np));
    dump_f64(dump_dir, "F_final", gather_F(elements, K, Np));
    FILE* f = std::fopen((dump_dir + "/meta.json").c_str(), "w");
    if (!f) die("cannot write meta.json");
    std::fprintf(f,
                 "{\"K\": %d, \"p\": %d, \"Np\": %d, \"nfq\": %d, \"nqa\": %d, \"nx\": %d, \"ny\": %d,"
                 " \"io\": %d, \"domain_x\": %.9g, \"domain_y\": %.9g, \"perturb_grid\": %.9g,"
                 " \"init_type\": %d, \"stepping\": %d, \"dt\": %.17g, \"steps\": %d,"
                 " \"time\": %.17g, \"dump_every\": %d}\n",
                 K, p, Np, static_cast<int>(gl.size()), static_cast<int>(ga.size()),
                 parms.num_element_in_x, parms.num_element_in_y, parms.integration_order,
                 static_cast<double>(parms.domain_x), static_cast<double>(parms.domain_y),
                 static_cast<double>(parms.perturb_grid), parms.U_initialization_type,
                 parms.stepping_method, parms.time_step, parms.number_time_steps,
                 elements[0].time, dump_every);
    std::fclose(f);
  }

  if (want_time) {
    int threads = 1;
#ifdef VORTEX_USE_OPENMP
    threads = omp_get_max_threads();
#endif
    const double init_s = std::chrono::duration<double>(t1 - t0).count();
    const double step_s = std::chrono::duration<double>(t3 - t2).count();
    const int stages = parms.stepping_method == 1 ? 4 : 1;
    const double dof_stages = static_cast<double>(K) * Np * stages * parms.number_time_steps;
    std::printf(
        "{\"K\": %d, \"p\": %d, \"Np\": %d, \"steps\": %d, \"stepping\": %d, \"threads\": %d,"
        " \"init_s\": %.6f, \"stepping_s\": %.6f, \"dof_stages_per_s\": %.6e}\n",
        K, p, Np, parms.number_time_steps, parms.stepping_method, threads, init_s, step_s,
        step_s > 0 ? dof_stages / step_s : 0.0);
  }
  return 0;
}
