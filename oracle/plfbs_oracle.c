/*
 * ORACLE — TEST INFRASTRUCTURE ONLY. Plain-C, serial, FP64 restatement of the
 * reference's GPU time step (CHRG-Developer/3D-PLFBS-GPU, src/LBFS.cu,
 * src/immersed_boundary_method.cu, src/common_kernels.cu, orchestrated as in
 * src/Solver_gpu.cu:664-870) plus the least-squares weight precompute
 * (src/gradients.cpp:149-313). Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py use it, as the checker; the product never
 * links or calls it.
 *
 * Pinned against the reference itself: tests/golden/ holds dumps of the
 * reference's own kernels (compiled from its sources and run on the host by
 * oracle/ref/) and the tests compare this restatement with them.
 *
 * The one generalisation: the gradient stencil is a CSR list (any number of
 * face neighbours per cell) where the reference hard-codes 6
 * (LBFS.cu:1549-1556); on hex meshes the two are the same computation.
 * Everything else follows the reference formula by formula, including its
 * quirks: the strict ghost test neighbour > n_cells (LBFS.cu:356), the
 * determinant typo (gradients.cpp:282-284), RK alpha = {1, .5, .5, 1}
 * (LBFS.cu:1467), the +-0.001 dt dead band (LBFS.cu:353-354) and the Neumann
 * ghost gradient g (1 - |n|) (LBFS.cu:1366-1368).
 *
 * flavour = 1 restates the reference's CPU Solver instead (src/Solver.cpp:88-590
 * and 840-1274, gradients.cpp:395-506 and 592-648, Solution.cpp:759-833):
 * boundary types rho 1, 2, 6, 7 and velocity 1, 2, 6, 8; Dirichlet ghost
 * gradients along the face normal, Neumann g (1 - n); on boundary faces the
 * owner's gradient on the owner side; lattice nodes on the strict sign of
 * e . n (no dead band, e . n = 0 takes the owner side); body force
 * -pressure_gradient; no IBM. Pinned against the CPU Solver's own final states
 * (tests/golden/cpu_*.npz).
 *
 * State layout: 4 doubles per cell (u, v, w, rho), cells then ghosts.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int n_cells, n_faces, n_internal;
  const int *owner, *neighbour;          /* [F]; boundary neighbour = C + f - F_i */
  const double *face_area;               /* [F] */
  const double *face_normal;             /* [3F] */
  const double *face_centroid;           /* [3F] */
  const double *streaming_dt;            /* [F] */
  const double *cell_volume;             /* [C+B] */
  const double *cell_centroid;           /* [3(C+B)] */
  const int *st_off, *st_cells, *st_faces; /* CSR gradient stencil over interior cells */
  const int *bc_rho_type, *bc_vel_type;  /* [B] */
  const double *bc_value;                /* [4B] u, v, w, rho */
  const double *lhs_inv;                 /* [9C] row-major inverse LHS */
  const double *rhs;                     /* [3 nnz] per stencil entry */
  double visc, gamma, dt, domain_dt, pressure_gradient, channel_height;
  double max_velocity, ref_rho, tolerance;
  double origin[3], lengths[3];
  int n_nodes, object_nodes;
  const double *node_ref;                /* [3N] x_ref, y_ref, z_ref interleaved */
  double stiffness, radius, depth;
  int flavour;                           /* 0: the GPU kernels; 1: the CPU Solver */
} oracle_problem;

typedef struct {
  double *state;      /* [4(C+B)] in/out */
  double *t0, *t1;    /* [4C] RK start / accumulator (in/out) */
  double *node_x;     /* [3N] positions (in/out) */
  double *node_x0;    /* [3N] (in/out) */
  double *node_vel;   /* [3N] out */
  double *node_force; /* [3N] out */
  double *force;      /* [3C] out: body force per cell */
  double *grad;       /* [12(C+B)] out: rho, u, v, w gradients */
  double *face_flux;  /* [4F] out: x, y, z momentum flux, mass flux */
  double *residual;   /* [4C] out: u, v, w, rho residual of the last stage */
  double *history;    /* [6 * steps] out: t, max_error, rho, u, v, w rms */
  int stage;          /* stages done so far (in/out); rk = stage % 4 */
} oracle_state;

static const double W0 = 2.0 / 9.0, W1 = 1.0 / 9.0, W7 = 1.0 / 72.0;
/* D3Q15 lattice, Solver_gpu.cu:1024-1026 */
static const int EX[15] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
static const int EY[15] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, -1, 1, 1, -1};
static const int EZ[15] = {0, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 1, -1, 1, -1};

static double wgt(int k) { return k == 0 ? W0 : (k < 7 ? W1 : W7); }

/* -------------------------------------------------------------------------
 * Least-squares weights, gradients.cpp:214-313 (beta_0 by mode, LHS/RHS
 * contributions :149-210, inverse by cofactors with the reference's
 * determinant typo :282-284). mode: 0 = LS, 1 = hybrid, 2 = Green-Gauss;
 * | 0x100 uses the true determinant instead (an extension for skewed cells).
 * ------------------------------------------------------------------------- */
int oracle_ls_weights(int n_cells, const int *off, const int *st_cells, const int *st_faces,
                      const int *owner, const double *face_area, const double *face_normal,
                      const double *face_centroid, const double *cell_volume,
                      const double *cell_centroid, int mode, double *lhs_inv, double *rhs) {
  for (int i = 0; i < n_cells; i++) {
    double L[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double max_area = 0.0, max_disp = 0.0;
    const double *ci = cell_centroid + 3 * i;
    for (int e = off[i]; e < off[i + 1]; e++) {
      int i1 = st_cells[e], f = st_faces[e];
      if (face_area[f] > max_area) max_area = face_area[f];
      const double *c1 = cell_centroid + 3 * i1;
      double dx = c1[0] - ci[0], dy = c1[1] - ci[1], dz = c1[2] - ci[2];
      double disp = sqrt(dx * dx + dy * dy + dz * dz);
      if (disp > max_disp) max_disp = disp;
    }
    double aspect = 2 * fabs(max_disp) * max_area / cell_volume[i];
    double beta;
    if ((mode & 0xff) == 1)
      beta = (2 / aspect) < 1.0 ? (2 / aspect) : 1.0;
    else if ((mode & 0xff) == 0)
      beta = 1.0;
    else
      beta = 0.0;
    L[0] = L[0] + 2 * (1 - beta) * cell_volume[i];
    L[4] = L[4] + 2 * (1 - beta) * cell_volume[i];
    L[8] = L[8] + 2 * (1 - beta) * cell_volume[i];
    for (int e = off[i]; e < off[i + 1]; e++) {
      int i1 = st_cells[e], f = st_faces[e];
      const double *fc = face_centroid + 3 * f, *n = face_normal + 3 * f;
      double dx = fc[0] - ci[0], dy = fc[1] - ci[1], dz = fc[2] - ci[2];
      double l_norm = dx * n[0] + dy * n[1] + dz * n[2];
      const double *c1 = cell_centroid + 3 * i1;
      dx = c1[0] - ci[0];
      dy = c1[1] - ci[1];
      dz = c1[2] - ci[2];
      double Ld = sqrt(pow(dx, 2.0) + pow(dy, 2.0) + pow(dz, 2.0));
      double s = face_area[f];
      double L_norm = dx * n[0] + dy * n[1] + dz * n[2];
      double alpha_w = pow(2 * l_norm / L_norm, 2.0);
      double w = alpha_w * s / Ld;
      L[0] = L[0] + w * dx * dx * beta;
      L[1] = L[1] + w * dx * dy * beta;
      L[2] = L[2] + w * dx * dz * beta;
      L[3] = L[3] + w * dy * dx * beta;
      L[4] = L[4] + w * dy * dy * beta;
      L[5] = L[5] + w * dy * dz * beta;
      L[6] = L[6] + w * dz * dx * beta;
      L[7] = L[7] + w * dz * dy * beta;
      L[8] = L[8] + w * dz * dz * beta;
      double sgn = (owner[f] == i) ? 1.0 : -1.0;
      if (sgn > 0) {
        rhs[3 * e + 0] = beta * w * dx + 2 * (1 - beta) * 0.5 * n[0] * s;
        rhs[3 * e + 1] = beta * w * dy + 2 * (1 - beta) * 0.5 * n[1] * s;
        rhs[3 * e + 2] = beta * w * dz + 2 * (1 - beta) * 0.5 * n[2] * s;
      } else {
        rhs[3 * e + 0] = beta * w * dx + 2 * (1 - beta) * 0.5 * n[0] * -1 * s;
        rhs[3 * e + 1] = beta * w * dy + 2 * (1 - beta) * 0.5 * n[1] * -1 * s;
        rhs[3 * e + 2] = beta * w * dz + 2 * (1 - beta) * 0.5 * n[2] * -1 * s;
      }
    }
    /* the reference's determinant, typo included: (yz - zx) where the
       cofactor expansion has -(yx zz - yz zx); mode bit 0x100 asks for the
       true determinant */
    double det = (mode & 0x100)
                     ? L[0] * (L[4] * L[8] - L[5] * L[7]) - L[1] * (L[3] * L[8] - L[5] * L[6]) +
                           L[2] * (L[3] * L[7] - L[4] * L[6])
                     : L[0] * (L[4] * L[8] - L[5] * L[7]) + L[1] * (L[3] * L[8] - L[5] - L[6]) +
                           L[2] * (L[3] * L[7] - L[4] * L[6]);
    double a = L[0], b = L[1], c = L[2], d = L[3], e_ = L[4], f_ = L[5], g = L[6], h = L[7],
           k = L[8];
    double *o = lhs_inv + 9 * i;
    o[0] = 1 / det * (e_ * k - f_ * h);
    o[1] = 1 / det * (c * h - b * k);
    o[2] = 1 / det * (b * f_ - c * e_);
    o[3] = 1 / det * (f_ * g - d * k);
    o[4] = 1 / det * (a * k - c * g);
    o[5] = 1 / det * (c * d - a * f_);
    o[6] = 1 / det * (d * h - e_ * g);
    o[7] = 1 / det * (b * g - a * h);
    o[8] = 1 / det * (a * e_ - b * d);
  }
  return 0;
}

/* ---- ghost states, LBFS.cu:1228-1301 ----------------------------------- */
static void update_bcs(const oracle_problem *p, double *q) {
  const int C = p->n_cells, Fi = p->n_internal, B = p->n_faces - p->n_internal;
  double H2 = p->channel_height * 0.5;
  double H = p->channel_height, H4 = H * H * H * H;
  for (int b = 0; b < B; b++) {
    int j = C + b, o = p->owner[Fi + b];
    const double *nbq = q + 4 * o, *bc = p->bc_value + 4 * b;
    double *g = q + 4 * j;
    if (p->flavour == 1) { /* Solution::update_unstructured_bcs, Solution.cpp:759-833 */
      int rt = p->bc_rho_type[b], vt = p->bc_vel_type[b];
      if (rt == 1)
        g[3] = bc[3] - (nbq[3] - bc[3]);
      else if (rt == 2)
        g[3] = nbq[3] + 0.0 * bc[3];
      else if (rt == 6 || rt == 7)
        g[3] = bc[3];
      for (int c = 0; c < 3; c++) {
        if (vt == 1)
          g[c] = bc[c] - (nbq[c] - bc[c]);
        else if (vt == 2)
          g[c] = nbq[c] + 0.0 * bc[c];
        else if (vt == 6)
          g[c] = bc[c] * 1.0;
        else if (vt == 8)
          g[c] = c == 1 ? -nbq[c] : nbq[c];
      }
      continue;
    }
    if (p->bc_rho_type[b] == 1)
      g[3] = bc[3] - (nbq[3] - bc[3]);
    else if (p->bc_rho_type[b] == 2)
      g[3] = nbq[3];
    if (p->bc_vel_type[b] == 1) {
      for (int c = 0; c < 3; c++) g[c] = bc[c] - (nbq[c] - bc[c]);
    } else if (p->bc_vel_type[b] == 2) {
      for (int c = 0; c < 3; c++) g[c] = nbq[c];
    } else if (p->bc_vel_type[b] == 9) {
      const double *cc = p->cell_centroid + 3 * j;
      double ut = 16 * bc[0] * (H2 + cc[1]) * (H2 - cc[1]) * (H2 + cc[2]) * (H2 - cc[2]) / H4;
      g[0] = ut - (nbq[0] - ut);
      g[1] = bc[1] - (nbq[1] - bc[1]);
      g[2] = bc[2] - (nbq[2] - bc[2]);
    }
  }
}

/* ---- interior LS gradients, LBFS.cu:1419-1451 and 1526-1589 ------------ */
static void interior_gradients(const oracle_problem *p, const double *q, double *grad) {
  for (int i = 0; i < p->n_cells; i++) {
    double R[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}}; /* rho, u, v, w */
    const double *qi = q + 4 * i;
    for (int e = p->st_off[i]; e < p->st_off[i + 1]; e++) {
      const double *q1 = q + 4 * p->st_cells[e], *W = p->rhs + 3 * e;
      double d[4] = {q1[3] - qi[3], q1[0] - qi[0], q1[1] - qi[1], q1[2] - qi[2]};
      for (int f = 0; f < 4; f++)
        for (int c = 0; c < 3; c++) R[f][c] = R[f][c] + W[c] * d[f];
    }
    const double *L = p->lhs_inv + 9 * i;
    for (int f = 0; f < 4; f++)
      for (int r = 0; r < 3; r++)
        grad[12 * i + 3 * f + r] = L[3 * r] * R[f][0] + L[3 * r + 1] * R[f][1] + L[3 * r + 2] * R[f][2];
  }
}

/* ---- ghost gradients, LBFS.cu:1306-1416 -------------------------------- */
static void bc_gradients(const oracle_problem *p, const double *q, double *grad) {
  const int C = p->n_cells, Fi = p->n_internal, B = p->n_faces - p->n_internal;
  for (int b = 0; b < B; b++) {
    int face = Fi + b, o = p->owner[face], j = C + b;
    const double *n = p->face_normal + 3 * face;
    const double *cn = p->cell_centroid + 3 * o, *cb = p->cell_centroid + 3 * j;
    const double *bc = p->bc_value + 4 * b, *s = q + 4 * o;
    double dx = cb[0] - cn[0], dy = cb[1] - cn[1], dz = cb[2] - cn[2];
    double dmag = sqrt(pow(dx, 2.0) + pow(dy, 2.0) + pow(dz, 2.0));
    double nv[3] = {dx / dmag, dy / dmag, dz / dmag};
    double dq[4] = {2 * (bc[3] - s[3]), 2 * (bc[0] - s[0]), 2 * (bc[1] - s[1]), 2 * (bc[2] - s[2])};
    double *gj = grad + 12 * j;
    const double *go = grad + 12 * o;
    if (p->flavour == 1) { /* Get_LS_Gradients / get_ghost_grads, gradients.cpp:395-506,592-648 */
      int rt = p->bc_rho_type[b], vt = p->bc_vel_type[b];
      for (int c = 0; c < 3; c++) {
        if (rt == 1) gj[c] = dq[0] / dmag * n[c];
        else if (rt == 2) gj[c] = go[c] * (1 - n[c]);
        else if (rt == 6) gj[c] = 0.0;
        else if (rt == 7) gj[c] = go[c];
      }
      for (int f = 1; f < 4; f++)
        for (int c = 0; c < 3; c++) {
          if (vt == 1 || vt == 8) gj[3 * f + c] = dq[f] / dmag * n[c];
          else if (vt == 2) gj[3 * f + c] = go[3 * f + c] * (1 - n[c]);
          else if (vt == 6) gj[3 * f + c] = 0.0;
        }
      continue;
    }
    if (p->bc_rho_type[b] == 1) {
      for (int c = 0; c < 3; c++) gj[c] = dq[0] / dmag * nv[c];
    } else if (p->bc_rho_type[b] == 2) {
      for (int c = 0; c < 3; c++) gj[c] = go[c] * (1 - fabs(n[c]));
    }
    if (p->bc_vel_type[b] == 1 || p->bc_vel_type[b] == 9) {
      for (int f = 1; f < 4; f++)
        for (int c = 0; c < 3; c++) gj[3 * f + c] = dq[f] / dmag * nv[c];
    } else if (p->bc_vel_type[b] == 2) {
      for (int f = 1; f < 4; f++)
        for (int c = 0; c < 3; c++) gj[3 * f + c] = go[3 * f + c] * (1 - fabs(n[c]));
    }
  }
}

/* ---- face flux, LBFS.cu:1592-1710 with populate_lattice_macros (:330-938),
 *      populate_feq (:942-1038), calculate_flux_at_interface (:1042-1223) --- */
static void face_fluxes(const oracle_problem *p, const double *q, const double *grad,
                        double *flux, double *res) {
  const int C = p->n_cells;
  const double pg = 1.0 / p->gamma;
  for (int face = 0; face < p->n_faces; face++) {
    int i = p->owner[face], nb = p->neighbour[face];
    const double *c1 = p->cell_centroid + 3 * i, *c2 = p->cell_centroid + 3 * nb;
    const double *xf = p->face_centroid + 3 * face, *n = p->face_normal + 3 * face;
    double A = p->face_area[face], dt = p->streaming_dt[face];
    const double *g1 = grad + 12 * i, *g2 = grad + 12 * nb;
    const double *qo = q + 4 * i, *qn = q + 4 * nb;
    double t1[3] = {c1[0] - xf[0], c1[1] - xf[1], c1[2] - xf[2]};
    double t2[3] = {c2[0] - xf[0], c2[1] - xf[1], c2[2] - xf[2]};
    /* per field f (0 rho, 1 u, 2 v, 3 w): owner-side, neighbour-side and
       centre values, and the gradients used on each side */
    double side_i[4], side_n[4], centre[4];
    double G1[4][3], G2[4][3], G3[4][3];
    const int qi_idx[4] = {3, 0, 1, 2};
    double d1 = 0.001 * dt;
    if (nb > C) { /* boundary: strict test, LBFS.cu:356 */
      int b = nb - C;
      const double *bc = p->bc_value + 4 * b;
      int rt = p->bc_rho_type[b], vt = p->bc_vel_type[b];
      for (int f = 0; f < 4; f++) {
        double dotv = t1[0] * g2[3 * f] + t1[1] * g2[3 * f + 1] + t1[2] * g2[3 * f + 2];
        double v;
        if (f == 0)
          v = (rt == 1) ? bc[3] : qo[3] - dotv;
        else if (p->flavour == 1) /* populate_lattice_macros, Solver.cpp:862-904 */
          v = (vt == 1) ? bc[f - 1] : (vt == 8 ? (f == 2 ? 0.0 : qo[qi_idx[f]]) : qo[qi_idx[f]] - dotv);
        else
          v = (vt == 1 || vt == 9) ? bc[f - 1] : qo[qi_idx[f]] - dotv;
        centre[f] = side_i[f] = side_n[f] = v;
        /* the GPU kernels use the ghost gradient on both sides (LBFS.cu:398-401),
           the CPU Solver the owner's on the owner side */
        for (int c = 0; c < 3; c++) {
          G2[f][c] = G3[f][c] = g2[3 * f + c];
          G1[f][c] = p->flavour == 1 ? g1[3 * f + c] : g2[3 * f + c];
        }
      }
    } else {
      for (int f = 0; f < 4; f++) {
        double a = qo[qi_idx[f]] - (t1[0] * g1[3 * f] + t1[1] * g1[3 * f + 1] + t1[2] * g1[3 * f + 2]);
        double bb = qn[qi_idx[f]] - (t2[0] * g2[3 * f] + t2[1] * g2[3 * f + 1] + t2[2] * g2[3 * f + 2]);
        side_i[f] = a;
        side_n[f] = bb;
        centre[f] = (a + bb) * 0.5;
        for (int c = 0; c < 3; c++) {
          G1[f][c] = g1[3 * f + c];
          G2[f][c] = g2[3 * f + c];
          G3[f][c] = (g1[3 * f + c] + g2[3 * f + c]) * 0.5;
        }
      }
    }
    /* lattice node values: node k sits at x_f - e_k dt; the upwind side is
       chosen by the sign of e_k . n for the first node of each opposite pair */
    double lat[4][15];
    for (int f = 0; f < 4; f++) lat[f][0] = centre[f];
    for (int k = 1; k < 15; k += 2) {
      double s = EX[k] * n[0] + EY[k] * n[1] + EZ[k] * n[2];
      for (int f = 0; f < 4; f++) {
        double ek_g1 = EX[k] * G1[f][0] + EY[k] * G1[f][1] + EZ[k] * G1[f][2];
        double ek_g2 = EX[k] * G2[f][0] + EY[k] * G2[f][1] + EZ[k] * G2[f][2];
        double ek_g3 = EX[k] * G3[f][0] + EY[k] * G3[f][1] + EZ[k] * G3[f][2];
        if (p->flavour == 1) { /* strict sign, Solver.cpp:929-1271 */
          if (s > 0) {
            lat[f][k] = side_i[f] - ek_g1 * dt;
            lat[f][k + 1] = side_n[f] + ek_g2 * dt;
          } else if (s < 0) {
            lat[f][k] = side_n[f] - ek_g2 * dt;
            lat[f][k + 1] = side_i[f] + ek_g1 * dt;
          } else {
            lat[f][k] = side_i[f] - ek_g1 * dt;
            lat[f][k + 1] = side_i[f] + ek_g1 * dt;
          }
        } else if (s > d1) {
          lat[f][k] = side_i[f] - ek_g1 * dt;
          lat[f][k + 1] = side_n[f] + ek_g2 * dt;
        } else if (s < -d1) {
          lat[f][k] = side_n[f] - ek_g2 * dt;
          lat[f][k + 1] = side_i[f] + ek_g1 * dt;
        } else {
          lat[f][k] = centre[f] - ek_g3 * dt;
          lat[f][k + 1] = centre[f] + ek_g3 * dt;
        }
      }
    }
    /* equilibrium at every lattice node, populate_feq */
    double feq[15];
    for (int k = 0; k < 15; k++) {
      double r = lat[0][k], u = lat[1][k], v = lat[2][k], w = lat[3][k];
      double eu = EX[k] * u + EY[k] * v + EZ[k] * w;
      double usq = (u * u + v * v + w * w) * pg;
      feq[k] = wgt(k) * r * (1.0 + 3.0 * eu + 4.5 * eu * eu * pg - 1.5 * usq);
    }
    double rhoI = 0, m[3] = {0, 0, 0};
    for (int k = 0; k < 15; k++) {
      rhoI += feq[k];
      m[0] += EX[k] * feq[k];
      m[1] += EY[k] * feq[k];
      m[2] += EZ[k] * feq[k];
    }
    double uI[3] = {1 / rhoI * m[0], 1 / rhoI * m[1], 1 / rhoI * m[2]};
    /* calculate_flux_at_interface: relax towards the interface equilibrium */
    double tau = p->visc * 3 / dt * pg;
    double usqI = (uI[0] * uI[0] + uI[1] * uI[1] + uI[2] * uI[2]) * pg;
    double fk[15];
    for (int k = 1; k < 15; k++) {
      double eu = EX[k] * uI[0] + EY[k] * uI[1] + EZ[k] * uI[2];
      double fe = wgt(k) * rhoI * (1.0 + 3.0 * eu + 4.5 * eu * eu * pg - 1.5 * usqI);
      fk[k] = fe - tau * (fe - feq[k]);
    }
    double Fm[3] = {0, 0, 0}, P[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int k = 1; k < 15; k++) {
      int e[3] = {EX[k], EY[k], EZ[k]};
      for (int a = 0; a < 3; a++) {
        Fm[a] += e[a] * fk[k];
        for (int b2 = 0; b2 < 3; b2++) P[a][b2] += e[a] * e[b2] * fk[k];
      }
    }
    double *out = flux + 4 * face;
    out[3] = (Fm[0] * n[0] + Fm[1] * n[1] + Fm[2] * n[2]) * A;
    for (int a = 0; a < 3; a++) out[a] = (P[0][a] * n[0] + P[1][a] * n[1] + P[2][a] * n[2]) * A;
    /* residual accumulation (the reference's 8 atomics, here in face order);
       ghost-cell residuals are never read, so only interior cells are kept */
    double Vi = p->cell_volume[i];
    for (int a = 0; a < 4; a++) res[4 * i + a] += -out[a] / Vi;
    if (nb < C) {
      double Vn = p->cell_volume[nb];
      for (int a = 0; a < 4; a++) res[4 * nb + a] += out[a] / Vn;
    }
  }
}

/* ---- IBM, immersed_boundary_method.cu:13-90, 161-190, 244-295, 299-375 ---- */
static void ibm_step(const oracle_problem *p, oracle_state *s) {
  const int C = p->n_cells, N = p->n_nodes;
  const double dx = p->domain_dt * 2;
  int xc = (int)(p->lengths[0] / dx), yc = (int)(p->lengths[1] / dx);
  double inv3 = 1 / dx / dx / dx;
  for (int c = 0; c < C; c++) {
    s->force[3 * c] = p->pressure_gradient;
    s->force[3 * c + 1] = 0.0;
    s->force[3 * c + 2] = 0.0;
  }
  /* interpolate at the old positions */
  for (int nd = 0; nd < N; nd++) {
    double *x = s->node_x + 3 * nd, *v = s->node_vel + 3 * nd;
    double r[3] = {(x[0] - p->origin[0]) / dx, fabs((x[1] - p->origin[1]) / dx),
                   fabs((x[2] - p->origin[2]) / dx)};
    int lo[3];
    for (int a = 0; a < 3; a++) lo[a] = (int)round(r[a]) - 1;
    v[0] = v[1] = v[2] = 0.0;
    for (int i = lo[0]; i <= lo[0] + 1; i++)
      for (int j = lo[1]; j <= lo[1] + 1; j++)
        for (int k = lo[2]; k <= lo[2] + 1; k++) {
          int cell = i + j * xc + k * yc * xc;
          if (cell < C && cell >= 0) {
            double wx = 1 - fabs(i + 0.5 - r[0]), wy = 1 - fabs(j + 0.5 - r[1]),
                   wz = 1 - fabs(k + 0.5 - r[2]);
            const double *q = s->state + 4 * cell;
            v[0] += q[0] * wx * wy * wz * inv3;
            v[1] += q[1] * wx * wy * wz * inv3;
            v[2] += q[2] * wx * wy * wz * inv3;
          }
        }
  }
  /* advect and store x0 */
  for (int nd = 0; nd < N; nd++)
    for (int a = 0; a < 3; a++) {
      s->node_x[3 * nd + a] = s->node_x0[3 * nd + a] + s->node_vel[3 * nd + a] * p->dt;
      s->node_x0[3 * nd + a] = s->node_x[3 * nd + a];
    }
  /* penalty force F = -k A (x - x_ref), A = 2 pi r depth / N_object */
  double area = 2 * acos(-1.0) * p->radius / p->object_nodes * p->depth;
  for (int nd = 0; nd < N; nd++)
    for (int a = 0; a < 3; a++)
      s->node_force[3 * nd + a] =
          (-p->stiffness * area * (s->node_x[3 * nd + a] - p->node_ref[3 * nd + a]));
  /* spread with the same kernel at the new positions */
  for (int nd = 0; nd < N; nd++) {
    double *x = s->node_x + 3 * nd, *F = s->node_force + 3 * nd;
    double r[3] = {(x[0] - p->origin[0]) / dx, fabs((x[1] - p->origin[1]) / dx),
                   fabs((x[2] - p->origin[2]) / dx)};
    int lo[3];
    for (int a = 0; a < 3; a++) lo[a] = (int)round(r[a]) - 1;
    for (int i = lo[0]; i <= lo[0] + 1; i++)
      for (int j = lo[1]; j <= lo[1] + 1; j++)
        for (int k = lo[2]; k <= lo[2] + 1; k++) {
          int cell = i + j * xc + k * yc * xc;
          if (cell < C && cell >= 0) {
            double wx = 1 - fabs(i + 0.5 - r[0]), wy = 1 - fabs(j + 0.5 - r[1]),
                   wz = 1 - fabs(k + 0.5 - r[2]);
            for (int a = 0; a < 3; a++) s->force[3 * cell + a] += F[a] * wx * wy * wz * inv3;
          }
        }
  }
}

/* ---- RK stage update, LBFS.cu:1457-1521 --------------------------------- */
static void time_integration(const oracle_problem *p, oracle_state *s, int rk) {
  static const double alpha[4] = {1.0, 0.5, 0.5, 1.0};
  static const double beta[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
  const double dt = p->dt;
  for (int i = 0; i < p->n_cells; i++) {
    const double *t0 = s->t0 + 4 * i, *R = s->residual + 4 * i;
    double *t1 = s->t1 + 4 * i, *q = s->state + 4 * i;
    double f1 = t0[3] + R[3] * dt * alpha[rk];
    double f2 = t0[0] + (R[0]) * dt * alpha[rk];
    double f3 = t0[1] + (R[1]) * dt * alpha[rk];
    double f4 = t0[2] + (R[2]) * dt * alpha[rk];
    f2 = f2 / f1;
    f3 = f3 / f1;
    f4 = f4 / f1;
    t1[3] = t1[3] + dt * beta[rk] * R[3];
    t1[0] = t1[0] + dt * beta[rk] * R[0];
    t1[1] = t1[1] + dt * beta[rk] * R[1];
    t1[2] = t1[2] + dt * beta[rk] * R[2];
    if (rk == 3) {
      q[3] = t1[3];
      q[0] = t1[0] / t1[3];
      q[1] = t1[1] / t1[3];
      q[2] = t1[2] / t1[3];
    } else {
      q[3] = f1;
      q[0] = f2;
      q[1] = f3;
      q[2] = f4;
    }
  }
}

/* Copy the interior state into the RK accumulator (Solver_gpu.cu:664). */
void oracle_init_t1(const oracle_problem *p, oracle_state *s) {
  memcpy(s->t1, s->state, sizeof(double) * 4 * (size_t)p->n_cells);
}

/* Run n_stages RK stages (4 per time step) starting at s->stage. At the start
 * of each step: t0 = t1 and the IBM update (Solver_gpu.cu:671-713). After the
 * 4th stage: residual rms (Solver_gpu.cu:820-833, residuals.cpp:95-147) into
 * s->history, and, if stop_on_convergence, return once max_error < tolerance
 * (Solver_gpu.cu:870). Returns the number of completed steps in this call. */
int oracle_run(const oracle_problem *p, oracle_state *s, int n_stages, int stop_on_convergence) {
  const int C = p->n_cells;
  double *res = s->residual;
  int steps = 0;
  for (int g = 0; g < n_stages; g++) {
    int rk = s->stage % 4;
    if (rk == 0) {
      memcpy(s->t0, s->t1, sizeof(double) * 4 * (size_t)C);
      if (p->flavour == 1) { /* force = -pressure_gradient on u, Solver.cpp:213,410,424 */
        for (int i = 0; i < C; i++) {
          s->force[3 * i] = -p->pressure_gradient;
          s->force[3 * i + 1] = s->force[3 * i + 2] = 0.0;
        }
      } else {
        ibm_step(p, s);
      }
    }
    update_bcs(p, s->state);
    memset(res, 0, sizeof(double) * 4 * (size_t)C);
    interior_gradients(p, s->state, s->grad);
    bc_gradients(p, s->state, s->grad);
    face_fluxes(p, s->state, s->grad, s->face_flux, res);
    for (int i = 0; i < C; i++)
      for (int a = 0; a < 3; a++) res[4 * i + a] = res[4 * i + a] + s->force[3 * i + a];
    time_integration(p, s, rk);
    s->stage++;
    if (rk == 3) {
      double sq[4] = {0, 0, 0, 0};
      for (int i = 0; i < C; i++)
        for (int a = 0; a < 4; a++) sq[a] += res[4 * i + a] * res[4 * i + a];
      double mom = p->ref_rho * p->max_velocity;
      double rho_rms = sqrt(sq[3] / C) / p->ref_rho;
      double u_rms = sqrt(sq[0] / C) / mom, v_rms = sqrt(sq[1] / C) / mom,
             w_rms = sqrt(sq[2] / C) / mom;
      double me = fmax(fmax(w_rms, u_rms), v_rms);
      double *h = s->history + 6 * steps;
      h[0] = (double)(s->stage / 4 - 1);
      h[1] = me;
      h[2] = rho_rms;
      h[3] = u_rms;
      h[4] = v_rms;
      h[5] = w_rms;
      steps++;
      if (stop_on_convergence && me < p->tolerance) break;
    }
  }
  return steps;
}
