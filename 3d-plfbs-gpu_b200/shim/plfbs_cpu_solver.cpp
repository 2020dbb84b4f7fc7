// Drop-in body of the reference's CPU Solver entry point.
//
// Compile this file in the reference's source tree in place of Solver.cpp and
// link against libplfbs.so. It keeps the class and the signature that
// program.cpp calls when <gpu_solver>0</gpu_solver> (Solver.h:18-37,
// program.cpp:111-113):
//
//   void Solver::General_Purpose_Solver_mk_i(unstructured_mesh&, Solution&,
//       Boundary_Conditions&, external_forces&, global_variables&,
//       domain_geometry&, initial_conditions&, unstructured_bcs&, int mg,
//       Solution& residual, int fmg, post_processing&)
//
// (program.cpp references no other member of Solver), and runs the time step
// through libplfbs with PLFBS_FLAVOUR_CPU_SOLVER: the CPU Solver's boundary
// types, upwinding and body-force sign (Solver.cpp:88-590,840-1274), in FP64.
// The host side follows Solver.cpp: error.txt and the console line every
// output_step steps with Solution::output below a decade threshold, the
// convergence exit with the host post-processing, and the final state in
// soln (interior cells only: the CPU Solver never writes the ghost cells of
// soln). Constant time stepping only (time_stepping local/min/talts is not
// taken). Like the GPU shim it never calls exit(), and it writes the final
// state losslessly to <output_file>/state.bin (4 x (n_cells + n_bc) doubles:
// rho, u, v, w; ghost cells as soln holds them).
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "Solver.h"
#include "plfbs.h"
#include "plfbs_shim_common.hpp"
#include "residuals.h"
#include "tecplot_output.h"

Solver::Solver() {}
Solver::~Solver() {}

void Solver::General_Purpose_Solver_mk_i(unstructured_mesh& Mesh, Solution& soln,
                                         Boundary_Conditions& bcs, external_forces& source,
                                         global_variables& globals, domain_geometry& domain,
                                         initial_conditions& init_conds,
                                         unstructured_bcs& quad_bcs_orig, int mg,
                                         Solution& residual, int fmg, post_processing& pp) {
  (void)source;
  (void)quad_bcs_orig;
  (void)residual;
  const int C = Mesh.get_n_cells(), B = Mesh.get_num_bc(), T = Mesh.get_total_cells();
  if (globals.time_stepping != "constant") {
    std::cout << "plfbs: time_stepping " << globals.time_stepping
              << " is not taken (constant only)" << std::endl;
    return;
  }
  plfbs_shim::Owned o;
  const plfbs_mesh_view mv = plfbs_shim::mesh_view(Mesh, o);
  const plfbs_bc_view bv = plfbs_shim::bc_view(bcs, B, o);
  const plfbs_ibm_view iv = {0, nullptr, nullptr, 0.0, 0.0, 0.0, 0};  // the CPU Solver has no IBM
  const plfbs_config cfg =
      plfbs_shim::config(globals, domain, init_conds, PLFBS_FLAVOUR_CPU_SOLVER);

  plfbs_ctx* ctx = nullptr;
  int rc = plfbs_create(&cfg, &mv, &bv, &iv, 0, &ctx);
  if (rc) {
    plfbs_shim::report(nullptr, "plfbs_create", rc);
    return;
  }
  std::vector<double> rho(T), u(T), v(T), w(T);
  for (int i = 0; i < T; i++) {
    rho[i] = soln.get_rho(i);
    u[i] = soln.get_u(i);
    v[i] = soln.get_v(i);
    w[i] = soln.get_w(i);
  }
  auto pull = [&]() {  // soln.update of the interior cells (Solver.cpp:434)
    std::vector<double> r(T), a(T), b(T), c(T);
    if (plfbs_get_state(ctx, r.data(), a.data(), b.data(), c.data(), T) == PLFBS_OK)
      for (int i = 0; i < C; i++) {
        rho[i] = r[i];
        u[i] = a[i];
        v[i] = b[i];
        w[i] = c[i];
        soln.update(r[i], a[i], b[i], c[i], i);
      }
  };
  rc = plfbs_set_state(ctx, rho.data(), u.data(), v.data(), w.data(), T);
  if (rc) {
    plfbs_shim::report(ctx, "plfbs_set_state", rc);
    plfbs_destroy(ctx);
    return;
  }

  std::ofstream error_output((globals.output_file + "/error.txt").c_str(), std::ios::out);
  plfbs_shim::RunLog run_log(globals.output_file + "/run.jsonl", Mesh.get_n_cells());
  const char* exit_kind = "out_of_time";
  tecplot_output<double> tecplot;
  Solution residual_worker(T), temp_soln(T);
  gradients grads(T);
  grads.pre_fill_LHS_and_RHS_matrix(bcs, Mesh, domain, soln, globals);  // for post-processing
  Solution wall_shear_stress(Mesh.get_n_wall_cells());
  std::vector<double> delta_t_local(C, globals.time_marching_step), local_fneq(T, 0.0);

  const long long timesteps = (long long)std::ceil(globals.simulation_length);
  const double delta_t = globals.time_marching_step;
  const int out_step = globals.output_step > 0 ? globals.output_step : 1;
  double output_residual_threshold = 0;
  std::vector<double> hist;
  long long t = 0;
  bool converged = false;
  while (t < timesteps) {
    // run up to and including the next output step (t % output_step == 1)
    long long next = t;
    while (next < timesteps - 1 && !(mg == 0 && next % out_step == 1)) next++;
    const long long n = next - t + 1;
    hist.assign(6 * (size_t)n, 0.0);
    plfbs_stats st;
    rc = plfbs_run(ctx, n, &st, hist.data());
    if (rc && rc != PLFBS_ERR_DIVERGED) {
      exit_kind = "error";
      plfbs_shim::report(ctx, "plfbs_run", rc);
      break;
    }
    const long long ran = st.steps_run;
    const long long last = t + ran - 1;
    if (mg == 0 && last % out_step == 1 && ran > 0) {  // Solver.cpp:501-515
      pull();
      run_log.step(last, st);
      error_output << last << ", " << st.max_error << ", " << st.rho_rms << ", " << st.u_rms
                   << ", " << st.v_rms << ", " << st.w_rms << " , FMG cycle: " << fmg << std::endl;
      std::cout << "time t=" << last * delta_t << " error e =" << st.max_error
                << " delta_t:" << delta_t << std::endl;
      if (st.max_error < std::pow(10, output_residual_threshold)) {
        tecplot.tecplot_output_unstructured_soln(globals, Mesh, soln, bcs, last * delta_t, pp,
                                                 residual_worker, delta_t_local.data(),
                                                 local_fneq.data());
        output_residual_threshold = output_residual_threshold - 1;
        soln.output(globals.output_file, globals, domain);
      }
    }
    t += ran;
    if (rc == PLFBS_ERR_DIVERGED) {
      exit_kind = "diverged";  // the NaN / rho > 1000 exits, Solver.cpp:448-490
      plfbs_shim::report(ctx, "time step", rc);
      break;
    }
    if (st.converged) {
      converged = true;
      exit_kind = "converged";
      break;
    }
    if (ran < n) break;
  }
  pull();
  error_output.close();
  if (converged) {  // Solver.cpp:522-536
    if (mg == 0) {
      std::cout << "convergence" << std::endl;
      std::cout << "time t=" << (t - 1) * delta_t << std::endl;
      temp_soln.clone(soln);
      temp_soln.update_unstructured_bcs(bcs, Mesh, domain, (int)(t - 1));
      grads.Get_LS_Gradients(bcs, Mesh, domain, temp_soln, globals);
      pp.cylinder_post_processing(Mesh, globals, grads, bcs, temp_soln, domain,
                                  wall_shear_stress);
      tecplot.tecplot_output_unstructured_soln(globals, Mesh, soln, bcs, (t - 1) * delta_t, pp,
                                               residual_worker, delta_t_local.data(),
                                               local_fneq.data());
    }
  } else {  // Solver.cpp:565-572
    std::cout << "out of time" << std::endl;
    temp_soln.clone(soln);
    pp.cylinder_post_processing(Mesh, globals, grads, bcs, temp_soln, domain, wall_shear_stress);
    tecplot.tecplot_output_unstructured_soln(globals, Mesh, soln, bcs, timesteps * delta_t, pp,
                                             residual_worker, delta_t_local.data(),
                                             local_fneq.data());
  }
  run_log.end(exit_kind, t, pp.drag_coef, pp.lift_coef);
  // lossless copy of the final state (the text output keeps 6 digits)
  if (FILE* f = std::fopen((globals.output_file + "/state.bin").c_str(), "wb")) {
    std::fwrite(rho.data(), sizeof(double), T, f);
    std::fwrite(u.data(), sizeof(double), T, f);
    std::fwrite(v.data(), sizeof(double), T, f);
    std::fwrite(w.data(), sizeof(double), T, f);
    std::fclose(f);
  }
  plfbs_destroy(ctx);
}
