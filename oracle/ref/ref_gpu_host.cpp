// ORACLE / TEST INFRASTRUCTURE — never part of the product path.
//
// Host-serial execution of the reference's own CUDA kernels. This file
// #includes the reference's unmodified device sources (LBFS.cu,
// common_kernels.cu, immersed_boundary_method.cu) through the host shims in
// shims/: execution-space qualifiers vanish and the launch builtins describe a
// single thread (blockIdx = threadIdx = 0, blockDim = gridDim = 1), so every
// grid-stride loop of a reference kernel visits all of its items in index order
// and every FP64 CAS "atomic" becomes an ordered read-modify-write.
//
// It then supplies gpu_solver::General_Purpose_Solver_mk_i, the entry point
// that program.cpp calls when <gpu_solver>1</gpu_solver> (program.cpp:107-109),
// by restating the orchestration of Solver_gpu.cu:150-917: the same marshalling
// (Solver_gpu.cu:629-660, 1434-1659), the same kernel sequence per time step
// (Solver_gpu.cu:664-833) and the same convergence test (Solver_gpu.cu:870).
// Linked with the reference's other sources this yields oracle/_ref/plfbs_ref:
// the reference program whose GPU path runs on the host. Environment variable
// PLFBS_REF_DUMP=<dir> makes it write .npy dumps of the marshalled inputs, of the
// intermediate arrays of the first RK stage and of the final state, which the
// tests use as golden vectors.

#include <math.h>
#include <cmath>
using std::abs;  // device code resolves abs(double) to fabs; make the host agree

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "Solver_gpu.h"
#include "residuals.h"

// LBFS.cu's unused check_error kernel (LBFS.cu:1733-1765) issues a device
// trap through inline asm, which is not host assembly; it is never called here.
#define asm(...) ((void)0)
#include "LBFS.cu"
#include "common_kernels.cu"
#include "immersed_boundary_method.cu"
#undef asm

namespace {

// Minimal .npy (format 1.0) writer: little-endian, C order.
void write_npy(const std::string& path, const char* descr, const void* data,
               size_t elem_size, const std::vector<size_t>& shape) {
  std::string shp = "(";
  size_t n = 1;
  for (size_t i = 0; i < shape.size(); ++i) {
    shp += std::to_string(shape[i]);
    shp += (shape.size() == 1) ? "," : (i + 1 < shape.size() ? ", " : "");
    n *= shape[i];
  }
  shp += ")";
  std::string hdr = std::string("{'descr': '") + descr +
                    "', 'fortran_order': False, 'shape': " + shp + ", }";
  size_t total = 10 + hdr.size() + 1;
  size_t pad = (64 - total % 64) % 64;
  hdr.append(pad, ' ');
  hdr.push_back('\n');
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    std::fprintf(stderr, "plfbs_ref: cannot write %s\n", path.c_str());
    std::exit(3);
  }
  const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
  std::fwrite(magic, 1, 8, f);
  uint16_t hl = (uint16_t)hdr.size();
  std::fwrite(&hl, 2, 1, f);
  std::fwrite(hdr.data(), 1, hdr.size(), f);
  if (n) std::fwrite(data, elem_size, n, f);
  std::fclose(f);
}

void dump_d(const std::string& dir, const char* name, const double* p,
            std::vector<size_t> shape) {
  if (dir.empty()) return;
  write_npy(dir + "/" + name + ".npy", "<f8", p, 8, shape);
}
void dump_i(const std::string& dir, const char* name, const int* p,
            std::vector<size_t> shape) {
  if (dir.empty()) return;
  write_npy(dir + "/" + name + ".npy", "<i4", p, 4, shape);
}

// D3Q15 weights in the order of Solver_gpu.cu:1024-1045.
void fill_lattice_weights() {
  for (int k = 0; k < 15; k++) {
    if (k > 0 && k < 7)
      lattice_weight[k] = 1.0 / 9.0;
    else if (k > 6)
      lattice_weight[k] = 1.0 / 72.0;
    else
      lattice_weight[k] = 2.0 / 9.0;
  }
}

}  // namespace

gpu_solver::gpu_solver() {}
gpu_solver::~gpu_solver() {}

void gpu_solver::General_Purpose_Solver_mk_i(
    unstructured_mesh& Mesh, Solution& soln, Boundary_Conditions& bcs,
    external_forces& source, global_variables& globals, domain_geometry& domain,
    initial_conditions& init_conds, unstructured_bcs& quad_bcs_orig, int mg,
    Solution& residual, int fmg, post_processing& pp,
    std::vector<lagrangian_object>& object_vec) {
  const char* dump_env = std::getenv("PLFBS_REF_DUMP");
  const std::string dump = dump_env ? dump_env : "";
  const int n_cells = Mesh.get_n_cells();
  const int n_faces = Mesh.get_n_faces();
  const int n_nb = Mesh.get_n_neighbours();
  const int n_bc = Mesh.get_num_bc();
  const int total = Mesh.get_total_cells();

  gradients grads(total);
  Solution wall_shear_stress(Mesh.get_n_wall_cells());
  grads.pre_fill_LHS_and_RHS_matrix(bcs, Mesh, domain, soln, globals);  // Solver_gpu.cu:479

  // Marshalling, Solver_gpu.cu:629-660 (the GPU path assumes 6 neighbours per cell).
  std::vector<double4> temp_soln(total), soln_t0(total), soln_t1(total);
  std::vector<double> cell_volume(total), surface_area(n_faces), streaming_dt(n_faces);
  std::vector<int> stencil((size_t)n_cells * 6), owner(n_faces), neighbour(n_faces);
  std::vector<double3> centroid(total), face_normal(n_faces), face_centroid(n_faces);
  std::vector<double3> d_cfl_areas(total), RHS((size_t)n_cells * 6);
  std::vector<double> L[9];
  for (auto& v : L) v.resize(n_cells);
  std::vector<double4> bcs_arr(n_bc);
  std::vector<int> rho_type(n_bc), vel_type(n_bc);
  std::vector<double3> grad_rho(total), grad_u(total), grad_v(total), grad_w(total);
  std::vector<double> res_rho(total), res_u(total), res_v(total), res_w(total);
  std::vector<double4> res_face(n_faces);
  std::vector<double> local_fneq(total), dt_local(total);
  std::vector<double> force_x(total), force_y(total), force_z(total);

  for (int i = 0; i < total; i++) {
    temp_soln[i] = make_double4(soln.get_u(i), soln.get_v(i), soln.get_w(i), soln.get_rho(i));
    cell_volume[i] = Mesh.get_cell_volume(i);
    centroid[i] = make_double3(Mesh.get_centroid_x(i), Mesh.get_centroid_y(i),
                               Mesh.get_centroid_z(i));
  }
  for (int i = 0; i < n_cells; i++) {
    if (Mesh.gradient_cells[i].size() != 6) {
      std::fprintf(stderr, "plfbs_ref: the reference GPU path needs 6 neighbours per cell\n");
      std::exit(4);
    }
    for (int j = 0; j < 6; j++) stencil[i * 6 + j] = Mesh.gradient_cells[i][j];
    L[0][i] = grads.LHS_xx[i]; L[1][i] = grads.LHS_xy[i]; L[2][i] = grads.LHS_xz[i];
    L[3][i] = grads.LHS_yx[i]; L[4][i] = grads.LHS_yy[i]; L[5][i] = grads.LHS_yz[i];
    L[6][i] = grads.LHS_zx[i]; L[7][i] = grads.LHS_zy[i]; L[8][i] = grads.LHS_zz[i];
    for (int j = 0; j < 6; j++)
      RHS[i * 6 + j] = make_double3(grads.RHS_x[i * 6 + j], grads.RHS_y[i * 6 + j],
                                    grads.RHS_z[i * 6 + j]);
    double ax = 0, ay = 0, az = 0;  // populate_cfl_areas, Solver_gpu.cu:1271-1304
    for (size_t f = 0; f < Mesh.gradient_faces[i].size(); f++) {
      int face = Mesh.gradient_faces[i][f];
      ax = ax + fabs(Mesh.get_face_i(face) * Mesh.get_face_area(face));
      ay = ay + fabs(Mesh.get_face_j(face) * Mesh.get_face_area(face));
      az = az + fabs(Mesh.get_face_k(face) * Mesh.get_face_area(face));
    }
    d_cfl_areas[i] = make_double3(ax / 2, ay / 2, az / 2);
  }
  for (int f = 0; f < n_faces; f++) {
    owner[f] = Mesh.get_mesh_owner(f);
    neighbour[f] = Mesh.get_mesh_neighbour(f);
    surface_area[f] = Mesh.get_face_area(f);
    streaming_dt[f] = Mesh.get_delta_t_face(f);
    face_normal[f] = make_double3(Mesh.get_face_i(f), Mesh.get_face_j(f), Mesh.get_face_k(f));
    face_centroid[f] = make_double3(Mesh.get_face_x(f), Mesh.get_face_y(f), Mesh.get_face_z(f));
  }
  for (int b = 0; b < n_bc; b++) {
    bcs_arr[b] = make_double4(bcs.get_u(b), bcs.get_v(b), bcs.get_w(b), bcs.get_rho(b));
    rho_type[b] = bcs.get_rho_type(b);
    vel_type[b] = bcs.get_vel_type(b);
  }

  // Lagrangian objects, Solver_gpu.cu:331-391 and 1469-1499.
  int n_nodes = 0;
  for (auto& o : object_vec) n_nodes += o.num_nodes;
  std::vector<double> ox_ref(n_nodes), oy_ref(n_nodes), oz_ref(n_nodes), ox(n_nodes),
      oy(n_nodes), oz(n_nodes), ox0(n_nodes), oy0(n_nodes), oz0(n_nodes), ovx(n_nodes),
      ovy(n_nodes), ovz(n_nodes), ofx(n_nodes), ofy(n_nodes), ofz(n_nodes);
  {
    int n = 0;
    for (auto& o : object_vec)
      for (int j = 0; j < o.num_nodes; j++, n++) {
        ox_ref[n] = o.node_x_ref[j]; ox[n] = o.node_x[j]; ox0[n] = o.node_x[j];
        oy_ref[n] = o.node_y_ref[j]; oy[n] = o.node_y[j]; oy0[n] = o.node_y[j];
        oz_ref[n] = o.node_z_ref[j]; oz[n] = o.node_z[j]; oz0[n] = o.node_z[j];
      }
  }

  fill_lattice_weights();
  const double delta_t = globals.time_marching_step;
  const int timesteps = (int)ceil(globals.simulation_length);
  const double delta_x = domain.dt * 2;
  const double3 mesh_lengths = make_double3(domain.X, domain.Y, domain.Z);
  const double3 mesh_origin = make_double3(domain.origin_x, domain.origin_y, domain.origin_z);
  const double tol = globals.tolerance;

  if (!dump.empty()) {
    int hdr[5] = {n_cells, n_faces, n_nb, n_bc, total};
    dump_i(dump, "sizes", hdr, {5});
    dump_i(dump, "owner", owner.data(), {(size_t)n_faces});
    dump_i(dump, "neighbour", neighbour.data(), {(size_t)n_faces});
    dump_i(dump, "stencil", stencil.data(), {(size_t)n_cells, 6});
    dump_d(dump, "face_area", surface_area.data(), {(size_t)n_faces});
    dump_d(dump, "streaming_dt", streaming_dt.data(), {(size_t)n_faces});
    dump_d(dump, "face_normal", &face_normal[0].x, {(size_t)n_faces, 3});
    dump_d(dump, "face_centroid", &face_centroid[0].x, {(size_t)n_faces, 3});
    dump_d(dump, "cell_volume", cell_volume.data(), {(size_t)total});
    dump_d(dump, "cell_centroid", &centroid[0].x, {(size_t)total, 3});
    std::vector<double> lhs((size_t)n_cells * 9);
    for (int i = 0; i < n_cells; i++)
      for (int k = 0; k < 9; k++) lhs[(size_t)i * 9 + k] = L[k][i];
    dump_d(dump, "lhs_inv", lhs.data(), {(size_t)n_cells, 3, 3});
    dump_d(dump, "rhs_w", &RHS[0].x, {(size_t)n_cells, 6, 3});
    dump_d(dump, "bc_value", &bcs_arr[0].x, {(size_t)n_bc, 4});
    dump_i(dump, "bc_rho_type", rho_type.data(), {(size_t)n_bc});
    dump_i(dump, "bc_vel_type", vel_type.data(), {(size_t)n_bc});
    dump_d(dump, "state_init", &temp_soln[0].x, {(size_t)total, 4});
    dump_d(dump, "node_init", ox.data(), {(size_t)n_nodes});
    double par[8] = {globals.visc, globals.pre_conditioned_gamma, delta_t, domain.dt,
                     init_conds.pressure_gradient, domain.Y, globals.max_velocity, globals.ref_rho};
    dump_d(dump, "params", par, {8});
  }

  std::vector<double> history;  // per step: t, max_error, rho, u, v, w rms
  clone_a_to_b(n_cells, temp_soln.data(), soln_t1.data());  // Solver_gpu.cu:664
  int t_done = timesteps;
  bool converged = false;
  for (int t = 0; t < timesteps; t++) {
    clone_a_to_b(n_cells, soln_t1.data(), soln_t0.data());
    get_cfl_device(n_cells, temp_soln.data(), cell_volume.data(), dt_local.data(),
                   d_cfl_areas.data(), globals.time_marching_step, globals.max_velocity,
                   globals.pre_conditioned_gamma, globals.visc, globals.gpu_time_stepping);
    // IBM, Solver_gpu.cu:690-713
    interpolate_velocities_on_nodes(n_nodes, ovx.data(), ovy.data(), ovz.data(), ox.data(),
                                    oy.data(), oz.data(), mesh_origin, mesh_lengths, delta_x,
                                    temp_soln.data(), n_cells);
    update_node_positions_rk4(n_nodes, ovx.data(), ovy.data(), ovz.data(), ox.data(), oy.data(),
                              oz.data(), delta_t, object_vec[0].num_nodes, ox0.data(),
                              oy0.data(), oz0.data());
    fill_double(n_cells, force_x.data(), init_conds.pressure_gradient);
    fill_zero(n_cells, force_y.data());
    fill_zero(n_cells, force_z.data());
    update_node_forces(n_nodes, ofx.data(), ofy.data(), ofz.data(), ox.data(), oy.data(),
                       oz.data(), ox_ref.data(), oy_ref.data(), oz_ref.data(),
                       object_vec[0].stiffness, object_vec[0].radius, globals.PI,
                       object_vec[0].num_nodes, ovx.data(), ovy.data(), ovz.data(), delta_t,
                       object_vec[0].depth);
    spread_forces_on_structured_grid(n_nodes, ofx.data(), ofy.data(), ofz.data(), ox.data(),
                                     oy.data(), oz.data(), mesh_origin, mesh_lengths, delta_x,
                                     force_x.data(), force_y.data(), force_z.data(), n_cells);
    if (t == 0 && !dump.empty()) {
      std::vector<double> f3((size_t)n_cells * 3);
      for (int i = 0; i < n_cells; i++) {
        f3[i * 3] = force_x[i]; f3[i * 3 + 1] = force_y[i]; f3[i * 3 + 2] = force_z[i];
      }
      dump_d(dump, "s0_force", f3.data(), {(size_t)n_cells, 3});
      std::vector<double> nd((size_t)n_nodes * 9);
      for (int n = 0; n < n_nodes; n++) {
        double v[9] = {ox[n], oy[n], oz[n], ovx[n], ovy[n], ovz[n], ofx[n], ofy[n], ofz[n]};
        for (int k = 0; k < 9; k++) nd[(size_t)n * 9 + k] = v[k];
      }
      dump_d(dump, "s0_nodes", nd.data(), {(size_t)n_nodes, 9});
    }
    for (int rk = 0; rk < 4; rk++) {  // Solver_gpu.cu:720-813
      update_unstructured_bcs(n_bc, n_nb, n_cells, owner.data(), rho_type.data(),
                              vel_type.data(), temp_soln.data(), bcs_arr.data(),
                              centroid.data(), domain.Y);
      fill_zero(n_cells, res_rho.data());
      fill_zero(n_cells, res_u.data());
      fill_zero(n_cells, res_v.data());
      fill_zero(n_cells, res_w.data());
      get_interior_gradients(n_cells, stencil.data(), temp_soln.data(), RHS.data(),
                             L[0].data(), L[1].data(), L[2].data(), L[3].data(), L[4].data(),
                             L[5].data(), L[6].data(), L[7].data(), L[8].data(),
                             grad_rho.data(), grad_u.data(), grad_v.data(), grad_w.data());
      get_bc_gradients(n_bc, n_nb, n_cells, owner.data(), rho_type.data(), vel_type.data(),
                       temp_soln.data(), face_normal.data(), centroid.data(), bcs_arr.data(),
                       grad_rho.data(), grad_u.data(), grad_v.data(), grad_w.data());
      calc_face_flux(n_faces, temp_soln.data(), cell_volume.data(), surface_area.data(),
                     owner.data(), neighbour.data(), centroid.data(), face_centroid.data(),
                     face_normal.data(), streaming_dt.data(), grad_rho.data(), grad_u.data(),
                     grad_v.data(), grad_w.data(), n_cells, (1 / globals.pre_conditioned_gamma),
                     local_fneq.data(), globals.visc, res_rho.data(), res_u.data(),
                     res_v.data(), res_w.data(), res_face.data(), rho_type.data(),
                     vel_type.data(), bcs_arr.data(), globals.PI);
      add(n_cells, res_u.data(), force_x.data());
      add(n_cells, res_v.data(), force_y.data());
      add(n_cells, res_w.data(), force_z.data());
      if (t == 0 && rk == 0 && !dump.empty()) {
        dump_d(dump, "s0_state_bc", &temp_soln[0].x, {(size_t)total, 4});
        std::vector<double> g((size_t)total * 12);
        for (int i = 0; i < total; i++) {
          double v[12] = {grad_rho[i].x, grad_rho[i].y, grad_rho[i].z, grad_u[i].x,
                          grad_u[i].y,   grad_u[i].z,   grad_v[i].x,   grad_v[i].y,
                          grad_v[i].z,   grad_w[i].x,   grad_w[i].y,   grad_w[i].z};
          for (int k = 0; k < 12; k++) g[(size_t)i * 12 + k] = v[k];
        }
        dump_d(dump, "s0_grad", g.data(), {(size_t)total, 12});
        dump_d(dump, "s0_face_flux", &res_face[0].x, {(size_t)n_faces, 4});
        std::vector<double> r((size_t)n_cells * 4);
        for (int i = 0; i < n_cells; i++) {
          r[i * 4] = res_u[i]; r[i * 4 + 1] = res_v[i]; r[i * 4 + 2] = res_w[i];
          r[i * 4 + 3] = res_rho[i];
        }
        dump_d(dump, "s0_residual", r.data(), {(size_t)n_cells, 4});
      }
      time_integration(n_cells, rk, 4, dt_local.data(), soln_t0.data(), soln_t1.data(),
                       temp_soln.data(), res_rho.data(), res_u.data(), res_v.data(),
                       res_w.data());
      if (t == 0 && rk == 0 && !dump.empty())
        dump_d(dump, "s0_state_rk", &temp_soln[0].x, {(size_t)total, 4});
    }
    // square + total<256> + l2_norm_rms_moukallad, Solver_gpu.cu:820-833
    double s[4] = {0, 0, 0, 0};
    for (int i = 0; i < n_cells; i++) {
      s[0] += res_rho[i] * res_rho[i];
      s[1] += res_u[i] * res_u[i];
      s[2] += res_v[i] * res_v[i];
      s[3] += res_w[i] * res_w[i];
    }
    residuals conv;
    conv.reset();
    conv.l2_norm_rms_moukallad(globals, &s[0], &s[1], &s[2], &s[3], 1, n_cells);
    double row[6] = {(double)t, conv.max_error(), conv.rho_rms, conv.u_rms, conv.v_rms,
                     conv.w_rms};
    history.insert(history.end(), row, row + 6);
    if (conv.max_error() < tol) {  // Solver_gpu.cu:870
      t_done = t + 1;
      converged = true;
      break;
    }
  }
  soln.clone(temp_soln.data());
  double wall_forces[2] = {0.0, 0.0};
  if (converged) {
    // Solver_gpu.cu:881-884: host ghost update, host gradients, wall forces
    soln.update_unstructured_bcs(bcs, Mesh, domain, t_done - 1);
    grads.Get_LS_Gradients(bcs, Mesh, domain, soln, globals);
    pp.cylinder_post_processing(Mesh, globals, grads, bcs, soln, domain, wall_shear_stress);
    wall_forces[0] = pp.drag_coef;
    wall_forces[1] = pp.lift_coef;
  }
  if (!dump.empty()) {
    dump_d(dump, "final_state", &temp_soln[0].x, {(size_t)total, 4});
    dump_d(dump, "final_t1", &soln_t1[0].x, {(size_t)total, 4});
    dump_d(dump, "history", history.data(), {history.size() / 6, 6});
    int steps[1] = {t_done};
    dump_i(dump, "steps_done", steps, {1});
    std::vector<double> nd((size_t)n_nodes * 9);
    for (int n = 0; n < n_nodes; n++) {
      double v[9] = {ox[n], oy[n], oz[n], ovx[n], ovy[n], ovz[n], ofx[n], ofy[n], ofz[n]};
      for (int k = 0; k < 9; k++) nd[(size_t)n * 9 + k] = v[k];
    }
    dump_d(dump, "final_nodes", nd.data(), {(size_t)n_nodes, 9});
    dump_d(dump, "wall_forces", wall_forces, {2});  // Cd, Cl (zero unless converged)
  }
  (void)source; (void)quad_bcs_orig; (void)mg; (void)residual; (void)fmg;
}
