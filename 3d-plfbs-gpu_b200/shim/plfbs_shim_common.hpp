// Marshalling shared by the drop-in shims (plfbs_gpu_solver.cpp for the
// reference's GPU entry point, plfbs_cpu_solver.cpp for its CPU Solver): the
// reference's mesh, boundary-condition and global objects into the plain views
// of include/plfbs.h (what Solver_gpu.cu:629-660 marshals, with the gradient
// stencil as CSR).
#ifndef PLFBS_SHIM_COMMON_HPP
#define PLFBS_SHIM_COMMON_HPP

#include <cmath>
#include <cstdio>
#include <iostream>
#include <string>
#include <vector>

#include "Boundary_Conditions.h"
#include "domain_geometry.h"
#include "global_variables.h"
#include "initial_conditions.h"
#include "plfbs.h"
#include "unstructured_mesh.h"

namespace plfbs_shim {

struct Owned {
  std::vector<int32_t> owner, neighbour, st_off, st_cells, st_faces, rho_type, vel_type;
  std::vector<double> area, normal, fcen, sdt, vol, ccen, bcval, xref, x;
};

inline int gradient_mode(const std::string& s) {
  // gradients.cpp:259-265
  if (s == "hybrid") return PLFBS_GRAD_HYBRID;
  if (s == "LS") return PLFBS_GRAD_LS;
  return PLFBS_GRAD_GREEN_GAUSS;
}

inline void report(plfbs_ctx* ctx, const char* what, int rc) {
  std::cout << "plfbs: " << what << " failed (" << rc << "): " << plfbs_last_error(ctx)
            << std::endl;
}

// Mesh (Solver_gpu.cu:629-651).
inline plfbs_mesh_view mesh_view(unstructured_mesh& Mesh, Owned& o) {
  const int C = Mesh.get_n_cells(), F = Mesh.get_n_faces(), Fi = Mesh.get_n_neighbours();
  const int T = Mesh.get_total_cells();
  o.owner.resize(F);
  o.neighbour.resize(F);
  o.area.resize(F);
  o.sdt.resize(F);
  o.normal.resize(3 * (size_t)F);
  o.fcen.resize(3 * (size_t)F);
  for (int f = 0; f < F; f++) {
    o.owner[f] = Mesh.get_mesh_owner(f);
    o.neighbour[f] = Mesh.get_mesh_neighbour(f);
    o.area[f] = Mesh.get_face_area(f);
    o.sdt[f] = Mesh.get_delta_t_face(f);
    o.normal[3 * f] = Mesh.get_face_i(f);
    o.normal[3 * f + 1] = Mesh.get_face_j(f);
    o.normal[3 * f + 2] = Mesh.get_face_k(f);
    o.fcen[3 * f] = Mesh.get_face_x(f);
    o.fcen[3 * f + 1] = Mesh.get_face_y(f);
    o.fcen[3 * f + 2] = Mesh.get_face_z(f);
  }
  o.vol.resize(T);
  o.ccen.resize(3 * (size_t)T);
  for (int i = 0; i < T; i++) {
    o.vol[i] = Mesh.get_cell_volume(i);
    o.ccen[3 * i] = Mesh.get_centroid_x(i);
    o.ccen[3 * i + 1] = Mesh.get_centroid_y(i);
    o.ccen[3 * i + 2] = Mesh.get_centroid_z(i);
  }
  o.st_off.assign(1, 0);
  for (int i = 0; i < C; i++) {
    for (size_t j = 0; j < Mesh.gradient_cells[i].size(); j++) {
      o.st_cells.push_back(Mesh.gradient_cells[i][j]);
      o.st_faces.push_back(Mesh.gradient_faces[i][j]);
    }
    o.st_off.push_back((int32_t)o.st_cells.size());
  }
  return plfbs_mesh_view{C, F, Fi, o.owner.data(), o.neighbour.data(), o.area.data(),
                         o.normal.data(), o.fcen.data(), o.sdt.data(), o.vol.data(),
                         o.ccen.data(), o.st_off.data(), o.st_cells.data(), o.st_faces.data()};
}

// Boundary conditions (Solver_gpu.cu:653-655).
inline plfbs_bc_view bc_view(Boundary_Conditions& bcs, int B, Owned& o) {
  o.rho_type.resize(B);
  o.vel_type.resize(B);
  o.bcval.resize(4 * (size_t)B);
  for (int b = 0; b < B; b++) {
    o.rho_type[b] = bcs.get_rho_type(b);
    o.vel_type[b] = bcs.get_vel_type(b);
    o.bcval[4 * b] = bcs.get_u(b);
    o.bcval[4 * b + 1] = bcs.get_v(b);
    o.bcval[4 * b + 2] = bcs.get_w(b);
    o.bcval[4 * b + 3] = bcs.get_rho(b);
  }
  return plfbs_bc_view{o.rho_type.data(), o.vel_type.data(), o.bcval.data()};
}

// The scalar configuration from the reference's globals.
inline plfbs_config config(global_variables& globals, domain_geometry& domain,
                           initial_conditions& init_conds, int flavour) {
  plfbs_config cfg = {};
  cfg.visc = globals.visc;
  cfg.gamma = globals.pre_conditioned_gamma;
  cfg.time_marching_step = globals.time_marching_step;
  cfg.domain_dt = domain.dt;
  cfg.max_velocity = globals.max_velocity;
  cfg.ref_rho = globals.ref_rho;
  cfg.tolerance = globals.tolerance;
  cfg.pressure_gradient = init_conds.pressure_gradient;
  cfg.channel_height = domain.Y;
  cfg.origin[0] = domain.origin_x;
  cfg.origin[1] = domain.origin_y;
  cfg.origin[2] = domain.origin_z;
  cfg.lengths[0] = domain.X;
  cfg.lengths[1] = domain.Y;
  cfg.lengths[2] = domain.Z;
  cfg.gradient_mode = gradient_mode(globals.gradient_calc_type);
  cfg.precision = PLFBS_FP64;
  cfg.renumber = 1;
  cfg.flavour = flavour;
  return cfg;
}

// JSON-lines run log, <output_file>/run.jsonl: one record per output step
// (the residual norms the reference writes to error.txt, plus the device time
// of the steps since the previous record and the throughput they give) and a
// last record with the exit (converged, out_of_time, diverged or error) and the
// drag and lift coefficients post-processing computed.
class RunLog {
 public:
  RunLog(const std::string& path, long long cells) : f_(std::fopen(path.c_str(), "w")), cells_(cells) {}
  ~RunLog() {
    if (f_) std::fclose(f_);
  }
  RunLog(const RunLog&) = delete;
  RunLog& operator=(const RunLog&) = delete;
  void step(long long t, const plfbs_stats& st) {
    if (!f_) return;
    const double mcups = st.kernel_ms > 0 ? (double)cells_ * st.steps_run / (st.kernel_ms * 1e3) : 0.0;
    std::fprintf(f_,
                 "{\"step\": %lld, \"max_error\": %s, \"rho_rms\": %s, \"u_rms\": %s, "
                 "\"v_rms\": %s, \"w_rms\": %s, \"steps_run\": %lld, \"kernel_ms\": %s, "
                 "\"mcell_updates_per_s\": %s}\n",
                 t, num(st.max_error).c_str(), num(st.rho_rms).c_str(), num(st.u_rms).c_str(),
                 num(st.v_rms).c_str(), num(st.w_rms).c_str(), (long long)st.steps_run,
                 num(st.kernel_ms).c_str(), num(mcups).c_str());
    std::fflush(f_);
  }
  void end(const char* exit, long long steps, double cd, double cl) {
    if (!f_) return;
    std::fprintf(f_, "{\"exit\": \"%s\", \"steps\": %lld, \"cd\": %s, \"cl\": %s}\n", exit,
                 steps, num(cd).c_str(), num(cl).c_str());
    std::fflush(f_);
  }

 private:
  // JSON has no NaN or infinity: those are written as null
  static std::string num(double v) {
    if (!std::isfinite(v)) return "null";
    char b[32];
    std::snprintf(b, sizeof b, "%.17g", v);
    return b;
  }
  FILE* f_;
  long long cells_;
};

}  // namespace plfbs_shim

#endif  // PLFBS_SHIM_COMMON_HPP
