// Drop-in body of the reference's GPU solver entry point.
//
// Compile this file in the reference's source tree in place of Solver_gpu.cu
// (plus LBFS.cu, immersed_boundary_method.cu and common_kernels.cu, which it
// makes unnecessary) and link against libplfbs.so. It keeps the class and the
// signature that program.cpp calls (Solver_gpu.h:28-31, program.cpp:107-109):
//
//   void gpu_solver::General_Purpose_Solver_mk_i(unstructured_mesh&, Solution&,
//       Boundary_Conditions&, external_forces&, global_variables&,
//       domain_geometry&, initial_conditions&, unstructured_bcs&, int mg,
//       Solution& residual, int fmg, post_processing&,
//       std::vector<lagrangian_object>&)
//
// and reproduces the host side of Solver_gpu.cu:150-917: the marshalling of
// mesh, boundary conditions and Lagrangian objects (here into the plain views
// of include/plfbs.h), the time loop with its output every output_step steps
// (error.txt, console line, Tecplot calls, Solution::output below a decade
// threshold), the convergence exit with the host post-processing, and
// soln.clone of the final state. All arithmetic of the time step runs in
// libplfbs (FP64). Unlike the reference it never calls exit(): a failed
// library call prints plfbs_last_error() and returns with soln unchanged
// since the last output. In addition it writes the final state losslessly to
// <output_file>/state.bin (4 x (n_cells + n_bc) doubles: rho, u, v, w).
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "Solver_gpu.h"
#include "plfbs.h"
#include "plfbs_shim_common.hpp"
#include "residuals.h"
#include "tecplot_output.h"

gpu_solver::gpu_solver() {}
gpu_solver::~gpu_solver() {}

using plfbs_shim::Owned;
using plfbs_shim::report;

void gpu_solver::General_Purpose_Solver_mk_i(
    unstructured_mesh& Mesh, Solution& soln, Boundary_Conditions& bcs, external_forces& source,
    global_variables& globals, domain_geometry& domain, initial_conditions& init_conds,
    unstructured_bcs& quad_bcs_orig, int mg, Solution& residual, int fmg, post_processing& pp,
    std::vector<lagrangian_object>& object_vec) {
  (void)source;
  (void)quad_bcs_orig;
  const int C = Mesh.get_n_cells();
  const int B = Mesh.get_num_bc(), T = Mesh.get_total_cells();
  Owned o;
  const plfbs_mesh_view mv = plfbs_shim::mesh_view(Mesh, o);
  const plfbs_bc_view bv = plfbs_shim::bc_view(bcs, B, o);
  // --- Lagrangian objects (Solver_gpu.cu:1469-1499) ---------------------------
  int N = 0;
  for (auto& obj : object_vec) N += obj.num_nodes;
  o.xref.resize(3 * (size_t)N);
  o.x.resize(3 * (size_t)N);
  {
    int n = 0;
    for (auto& obj : object_vec)
      for (int j = 0; j < obj.num_nodes; j++, n++) {
        o.xref[3 * n] = obj.node_x_ref[j];
        o.xref[3 * n + 1] = obj.node_y_ref[j];
        o.xref[3 * n + 2] = obj.node_z_ref[j];
        o.x[3 * n] = obj.node_x[j];
        o.x[3 * n + 1] = obj.node_y[j];
        o.x[3 * n + 2] = obj.node_z[j];
      }
  }
  plfbs_ibm_view iv = {N, o.xref.data(), o.x.data(), 0.0, 0.0, 0.0, 0};
  if (!object_vec.empty()) {
    iv.stiffness = object_vec[0].stiffness;
    iv.radius = object_vec[0].radius;
    iv.depth = object_vec[0].depth;
    iv.object_nodes = object_vec[0].num_nodes;
  }
  const plfbs_config cfg = plfbs_shim::config(globals, domain, init_conds, PLFBS_FLAVOUR_GPU);

  plfbs_ctx* ctx = nullptr;
  int rc = plfbs_create(&cfg, &mv, &bv, &iv, 0, &ctx);
  if (rc) {
    report(nullptr, "plfbs_create", rc);
    return;
  }
  std::vector<double> rho(T), u(T), v(T), w(T);
  for (int i = 0; i < T; i++) {  // soln_to_double, Solver_gpu.cu:1646-1659
    rho[i] = soln.get_rho(i);
    u[i] = soln.get_u(i);
    v[i] = soln.get_v(i);
    w[i] = soln.get_w(i);
  }
  auto pull = [&]() {  // soln.clone(temp_soln)
    if (plfbs_get_state(ctx, rho.data(), u.data(), v.data(), w.data(), T) == PLFBS_OK)
      for (int i = 0; i < T; i++) soln.update(rho[i], u[i], v[i], w[i], i);
  };
  rc = plfbs_set_state(ctx, rho.data(), u.data(), v.data(), w.data(), T);
  if (rc) {
    report(ctx, "plfbs_set_state", rc);
    plfbs_destroy(ctx);
    return;
  }

  std::ofstream error_output((globals.output_file + "/error.txt").c_str(), std::ios::out);
  plfbs_shim::RunLog run_log(globals.output_file + "/run.jsonl", Mesh.get_n_cells());
  const char* exit_kind = "out_of_time";
  tecplot_output<double> tecplot;
  Solution residual_worker(T);
  gradients grads(T);
  grads.pre_fill_LHS_and_RHS_matrix(bcs, Mesh, domain, soln, globals);  // for post-processing
  Solution wall_shear_stress(Mesh.get_n_wall_cells());
  std::vector<double> delta_t_local(C, globals.time_marching_step), local_fneq(T, 0.0);
  std::vector<double> nx(3 * (size_t)N), nvel(3 * (size_t)N), nforce(3 * (size_t)N);
  auto node_arrays = [&](std::vector<double>& a, int c) {
    std::vector<double> r(N);
    for (int n = 0; n < N; n++) r[n] = a[3 * n + c];
    return r;
  };
  auto output_objects = [&](double t) {
    if (N == 0 || object_vec.empty()) return;
    plfbs_get_nodes(ctx, nx.data(), nvel.data(), nforce.data(), N);
    auto vx = node_arrays(nvel, 0), vy = node_arrays(nvel, 1), vz = node_arrays(nvel, 2);
    auto px = node_arrays(nx, 0), py = node_arrays(nx, 1), pz = node_arrays(nx, 2);
    auto fx = node_arrays(nforce, 0), fy = node_arrays(nforce, 1), fz = node_arrays(nforce, 2);
    tecplot.tecplot_output_lagrangian_object_gpu(
        vx.data(), vy.data(), vz.data(), px.data(), py.data(), pz.data(), fx.data(), fy.data(),
        fz.data(), globals, domain, t, object_vec[0].name, object_vec[0].num_nodes,
        object_vec[0].depth_nodes, object_vec[0].radial_nodes);
  };

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
      report(ctx, "plfbs_run", rc);
      break;
    }
    const long long ran = st.steps_run;
    const long long last = t + ran - 1;
    const double max_error = st.max_error;
    if (mg == 0 && last % out_step == 1 && ran > 0) {  // Solver_gpu.cu:844-868
      pull();
      run_log.step(last, st);
      error_output << last << ", " << max_error << ", " << st.rho_rms << ", " << st.u_rms << ", "
                   << st.v_rms << ", " << st.w_rms << " , FMG cycle: " << fmg << std::endl;
      std::cout << "time t=" << last * delta_t << " error e =" << max_error
                << " delta_t:" << delta_t << std::endl;
      if (max_error < std::pow(10, output_residual_threshold)) {
        tecplot.tecplot_output_unstructured_soln(globals, Mesh, soln, bcs, last, pp,
                                                 residual_worker, delta_t_local.data(),
                                                 local_fneq.data());
        output_objects(last);
        output_residual_threshold = output_residual_threshold - 1;
        soln.output(globals.output_file, globals, domain);
      }
    }
    t += ran;
    if (rc == PLFBS_ERR_DIVERGED) {
      exit_kind = "diverged";
      report(ctx, "time step", rc);
      break;
    }
    if (st.converged) {  // Solver_gpu.cu:870-895
      converged = true;
      exit_kind = "converged";
      break;
    }
    if (ran < n) break;
  }
  pull();
  error_output.close();
  if (converged) {
    if (mg == 0) {
      std::cout << "convergence" << std::endl;
      std::cout << "time t=" << (t - 1) * delta_t << std::endl;
      soln.update_unstructured_bcs(bcs, Mesh, domain, (int)(t - 1));
      grads.Get_LS_Gradients(bcs, Mesh, domain, soln, globals);
      pp.cylinder_post_processing(Mesh, globals, grads, bcs, soln, domain, wall_shear_stress);
      tecplot.tecplot_output_unstructured_soln(globals, Mesh, soln, bcs, t - 1, pp,
                                               residual_worker, delta_t_local.data(),
                                               local_fneq.data());
      output_objects((double)timesteps);
    }
  } else {
    std::cout << "out of time" << std::endl;
    pp.cylinder_post_processing(Mesh, globals, grads, bcs, soln, domain, wall_shear_stress);
    tecplot.tecplot_output_unstructured_soln(globals, Mesh, soln, bcs, timesteps, pp,
                                             residual_worker, delta_t_local.data(),
                                             local_fneq.data());
    output_objects((double)timesteps);
  }
  run_log.end(exit_kind, t, pp.drag_coef, pp.lift_coef);
  // lossless checkpoint of the final state (the text output keeps 6 digits)
  if (FILE* f = std::fopen((globals.output_file + "/state.bin").c_str(), "wb")) {
    std::fwrite(rho.data(), sizeof(double), T, f);
    std::fwrite(u.data(), sizeof(double), T, f);
    std::fwrite(v.data(), sizeof(double), T, f);
    std::fwrite(w.data(), sizeof(double), T, f);
    std::fclose(f);
  }
  (void)residual;
  plfbs_destroy(ctx);
}
