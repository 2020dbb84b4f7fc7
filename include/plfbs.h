/*
 * plfbs.h — C ABI of the B200 LBFS explicit time step.
 *
 * Drop-in for the GPU path of CHRG-Developer/3D-PLFBS-GPU:
 *   gpu_solver::General_Purpose_Solver_mk_i(unstructured_mesh&, Solution&,
 *       Boundary_Conditions&, external_forces&, global_variables&,
 *       domain_geometry&, initial_conditions&, unstructured_bcs&, int mg,
 *       Solution& residual, int fmg, post_processing&,
 *       std::vector<lagrangian_object>&)          (src/Solver_gpu.h:28-31,
 *                                                   src/Solver_gpu.cu:150-917)
 * called from program.cpp:107-109. A thin C++ shim with that exact signature
 * copies the mesh/BC/object getters into the plain views below and drives
 * create -> set_state -> run -> get_state -> destroy.
 *
 * Conventions: all arrays are borrowed for the duration of the call only and
 * use the caller's numbering (cells 0..C-1, then one ghost per boundary face,
 * ghost index C + f - F_i for boundary face f, as unstructured_mesh assigns,
 * unstructured_mesh.cpp:1346-1375). Per-cell state is four doubles (u, v, w,
 * rho). Every function returns PLFBS_OK (0) or a negative status; it never
 * exits the process and never traps the GPU; plfbs_last_error() explains the
 * last failure. A context is single-threaded and bound to one device;
 * different contexts may be used from different threads, and the message of a
 * failure without a context (plfbs_last_error(NULL)) is kept per thread.
 */
#ifndef PLFBS_H
#define PLFBS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  PLFBS_OK = 0,
  PLFBS_ERR_ARG = -1,         /* null pointer, bad size */
  PLFBS_ERR_MESH = -2,        /* inconsistent mesh arrays */
  PLFBS_ERR_BC = -3,          /* boundary type the GPU path does not define */
  PLFBS_ERR_CUDA = -4,        /* CUDA runtime error (message in last_error) */
  PLFBS_ERR_DIVERGED = -5,    /* NaN residual or rho > 1000 (Solver.cpp:448-493) */
  PLFBS_ERR_NO_DEVICE = -6,   /* no CUDA device / device not sm_100 */
  PLFBS_ERR_STATE = -7,       /* call out of order */
  PLFBS_ERR_TIMEOUT = -8      /* a bounded wait ran out; the launched steps are still in flight */
};

/* Gradient weighting, gradients.cpp:259-265 ("LS", "hybrid", anything else = GG).
 * OR-ing PLFBS_GRAD_EXACT_INVERSE inverts the LS matrix with the true
 * determinant instead of the one gradients.cpp:282-284 computes (which drops a
 * product and a sign in its second term). The two agree when the matrix has no
 * xy/yx coupling (axis-aligned hexes); on skewed or tetrahedral cells the
 * as-written determinant can flip the sign of the inverse and the scheme
 * diverges. Default (flag clear): the reference's arithmetic. */
enum {
  PLFBS_GRAD_LS = 0,
  PLFBS_GRAD_HYBRID = 1,
  PLFBS_GRAD_GREEN_GAUSS = 2,
  PLFBS_GRAD_EXACT_INVERSE = 0x100
};

/* Which of the reference's two solvers the step reproduces.
 * PLFBS_FLAVOUR_GPU: its CUDA kernels (LBFS.cu), the path Solver_gpu.cu runs:
 *   boundary types 1, 2 and 9, the +-0.001 dt dead band with face averages,
 *   the ghost gradient on both sides of a boundary face, Neumann 1 - |n|,
 *   body force +pressure_gradient, IBM.
 * PLFBS_FLAVOUR_CPU_SOLVER: its CPU Solver (Solver.cpp:88-590,840-1274 with
 *   gradients.cpp:319-506,592-648 and Solution.cpp:759-833): strict-sign
 *   upwinding (a lattice node on a face-parallel direction from the owner
 *   side), owner gradients on the owner side of a boundary face, Dirichlet
 *   ghost gradients along the face normal, Neumann 1 - n, rho types 1, 2, 6
 *   ("inlet", the value) and 7 ("wall", the value with the owner's gradient),
 *   velocity types 1, 2, 6 ("inlet") and 8 ("symmetry-x", (u, -v, w)), body
 *   force -pressure_gradient; FP64 only, no IBM (the CPU Solver has none).
 *   Periodic boundaries (3) are not taken: the reference's partner search reads
 *   an uninitialised cell index (Boundary_Conditions.cpp:426-444); nor rho type
 *   8, whose ghost gradient the reference never writes. */
enum { PLFBS_FLAVOUR_GPU = 0, PLFBS_FLAVOUR_CPU_SOLVER = 1 };

/* Arithmetic of the time step. */
enum {
  PLFBS_FP64 = 0,            /* the reference's FP64 semantics */
  PLFBS_FP32_DEVIATION = 1   /* FP32 state/flux, rho stored as rho - rho0,
                                velocity scaled by the reference velocity;
                                FP64 weights built then stored FP32, FP64
                                reductions and node positions */
};

/* Pre-processed mesh: what unstructured_mesh exposes (unstructured_mesh.h:15-47)
 * and what Solver_gpu.cu marshals (Solver_gpu.cu:629-651). B = n_faces - n_internal. */
typedef struct {
  int32_t n_cells;            /* C  = get_n_cells() */
  int32_t n_faces;            /* F  = get_n_faces() */
  int32_t n_internal;         /* F_i = get_n_neighbours(); faces [F_i, F) are boundary */
  const int32_t* owner;       /* [F] get_mesh_owner */
  const int32_t* neighbour;   /* [F] get_mesh_neighbour (boundary: C + f - F_i) */
  const double* face_area;    /* [F] get_face_area */
  const double* face_normal;  /* [3F] get_face_i/j/k, unit, owner -> neighbour */
  const double* face_centroid;/* [3F] get_face_x/y/z */
  const double* streaming_dt; /* [F] get_delta_t_face */
  const double* cell_volume;  /* [C+B] get_cell_volume */
  const double* cell_centroid;/* [3(C+B)] get_centroid_x/y/z */
  const int32_t* stencil_offsets; /* [C+1] CSR over gradient_cells / gradient_faces */
  const int32_t* stencil_cells;   /* [nnz] gradient_cells[i][*] */
  const int32_t* stencil_faces;   /* [nnz] gradient_faces[i][*] */
} plfbs_mesh_view;

/* A raw OpenFOAM polyMesh (what unstructured_mesh reads from points, faces,
 * owner and neighbour, unstructured_mesh.cpp:300-305 and the face loops after
 * it): internal faces first, then the boundary faces patch by patch. */
typedef struct {
  int32_t n_points;
  int32_t n_faces;
  int32_t n_internal;           /* faces with a neighbour */
  int32_t n_cells;
  const float* points;          /* [3 n_points] x, y, z (read as float, unstructured_mesh.h:50) */
  const int32_t* face_offsets;  /* [n_faces + 1] into face_points; every face has >= 3 vertices */
  const int32_t* face_points;   /* [face_offsets[n_faces]] vertex indices */
  const int32_t* owner;         /* [n_faces] */
  const int32_t* neighbour;     /* [n_internal] */
} plfbs_polymesh_view;

/* Caller-allocated outputs of plfbs_polymesh_geometry, sized as the arrays of
 * the mesh view above; B = n_faces - n_internal, nnz = 2 n_internal + B. */
typedef struct {
  int32_t* owner;             /* [F] */
  int32_t* neighbour;         /* [F] (boundary: C + f - F_i) */
  double* face_area;          /* [F] */
  double* face_normal;        /* [3F] */
  double* face_centroid;      /* [3F] */
  double* streaming_dt;       /* [F] */
  double* cell_volume;        /* [C+B] (ghosts 0) */
  double* cell_centroid;      /* [3(C+B)] */
  int32_t* stencil_offsets;   /* [C+1] */
  int32_t* stencil_cells;     /* [nnz] */
  int32_t* stencil_faces;     /* [nnz] */
} plfbs_mesh_arrays;

/* Boundary conditions per boundary face (Boundary_Conditions, marshalled as in
 * Solver_gpu.cu:653-655). Supported on the GPU path: rho_type 1 (Dirichlet) or
 * 2 (Neumann); vel_type 1 (Dirichlet), 2 (Neumann) or 9 (parabolic inlet). */
typedef struct {
  const int32_t* rho_type;    /* [B] */
  const int32_t* vel_type;    /* [B] */
  const double* value;        /* [4B] u, v, w, rho (get_u/v/w/rho) */
} plfbs_bc_view;

/* Lagrangian nodes of all objects (Solver_gpu.cu:1469-1499). Force area uses
 * object 0's stiffness/radius/depth/num_nodes, as Solver_gpu.cu:708-709 does.
 * n_nodes may be 0 (no immersed body). */
typedef struct {
  int32_t n_nodes;
  const double* x_ref;        /* [3N] interleaved x, y, z reference positions */
  const double* x;            /* [3N] interleaved current positions */
  double stiffness, radius, depth;
  int32_t object_nodes;       /* object_vec[0].num_nodes */
} plfbs_ibm_view;

typedef struct {
  double visc;                /* globals.visc */
  double gamma;               /* globals.pre_conditioned_gamma */
  double time_marching_step;  /* globals.time_marching_step (the RK dt) */
  double domain_dt;           /* domain.dt (streaming dt; IBM spacing = 2 domain.dt) */
  double max_velocity;        /* globals.max_velocity */
  double ref_rho;             /* globals.ref_rho */
  double tolerance;           /* globals.tolerance */
  double pressure_gradient;   /* init_conds.pressure_gradient (body force x) */
  double channel_height;      /* domain.Y (parabolic inlet, LBFS.cu:1286) */
  double origin[3];           /* domain.origin_x/y/z */
  double lengths[3];          /* domain.X/Y/Z */
  int32_t gradient_mode;      /* PLFBS_GRAD_*, optionally | PLFBS_GRAD_EXACT_INVERSE */
  int32_t precision;          /* PLFBS_FP64 or PLFBS_FP32_DEVIATION */
  int32_t renumber;           /* 0: caller's cell order; 1: reverse Cuthill-McKee (host
                                 breadth-first search); 2: the same order built on the
                                 device; faces are reordered for locality in every case */
  int32_t flavour;            /* PLFBS_FLAVOUR_*: whose reconstruction and boundary tables */
} plfbs_config;

typedef struct {
  int64_t steps_done;         /* time steps completed by this context */
  int32_t converged;          /* max_error < tolerance reached */
  int32_t status;             /* PLFBS_OK or PLFBS_ERR_DIVERGED */
  double max_error;           /* residuals::max_error() of the last step */
  double rho_rms, u_rms, v_rms, w_rms; /* l2_norm_rms_moukallad of the last step */
  double kernel_ms;           /* device time of the run() call (CUDA events) */
  int64_t steps_run;          /* steps completed by this run() call */
} plfbs_stats;

typedef struct plfbs_ctx plfbs_ctx;

/* The pre-processed mesh of a polyMesh, computed on `device`:
 * unstructured_mesh::generate_internal_mesh (unstructured_mesh.cpp:1133-1233)
 * with calc_face_delta_t (:979-983) and the ghost cells of
 * populate_ghost_cell_from_foam_face (:1346-1375). Faces are fanned from
 * vertex 0: area, area-weighted centroid and unit normal from the triangles'
 * cross products; cell volumes from the tetrahedra (a . (b-a) x (c-a)) / 6,
 * owner + and neighbour -; cell centroids as the area-weighted mean of their
 * faces' centroids; streaming dt = min(sqrt(A)/2, 3 visc / (gamma fneq_min))
 * (no cap when fneq_min is 0); the stencil lists each cell's faces in face
 * order. Every sum runs in the reference's order, so the arrays equal the
 * reference's bit for bit. Fills `out` (host memory) for plfbs_create. */
int plfbs_polymesh_geometry(const plfbs_polymesh_view* mesh, double visc, double gamma,
                            double fneq_min, int32_t device, plfbs_mesh_arrays* out);

/* Replaces the setup half of Solver_gpu.cu:150-662: validates the views,
 * builds the least-squares weights (gradients.cpp:214-313), renumbers for
 * locality, uploads everything to `device` and captures one time step in a
 * CUDA graph. The mesh arrays are copied to the device first and checked
 * there (the same checks, first failing index and message as on the host
 * threads, which check them when `device` is absent); from page-locked host
 * memory the copies set the pace. The initial state is all zeros until
 * plfbs_set_state. */
int plfbs_create(const plfbs_config* cfg, const plfbs_mesh_view* mesh,
                 const plfbs_bc_view* bc, const plfbs_ibm_view* ibm, int device,
                 plfbs_ctx** out);

/* soln_to_double (Solver_gpu.cu:1646-1659) + the RK seed (Solver_gpu.cu:664):
 * n_total = C + B values per array, caller numbering. Resets the step count. */
int plfbs_set_state(plfbs_ctx* ctx, const double* rho, const double* u, const double* v,
                    const double* w, int64_t n_total);

/* Starts a run from a field that is not uniform flow (a previous solution, a
 * prediction). Like plfbs_set_state, except that the RK accumulators are
 * seeded with the conserved variables (rho u, rho v, rho w, rho): the
 * reference seeds them with the velocity state (Solver_gpu.cu:664), which is
 * exact only where rho = 1 and perturbs a near-converged field by |rho - 1|.
 * node_x [n_nodes][3] (or NULL to keep the current positions) sets the IBM
 * node positions. Resets the step count. No counterpart in the reference. */
int plfbs_warm_start(plfbs_ctx* ctx, const double* rho, const double* u, const double* v,
                     const double* w, int64_t n_total, const double* node_x, int32_t n_nodes);

/* Drag and lift coefficients over the wall faces of a body-fitted mesh, as
 * post_processing::cylinder_post_processing (post_processing.cpp:50-173)
 * computes them at the end of a run (Solver_gpu.cu:881-884), on the device
 * and from the current state: the ghost states and the gradients are
 * recomputed first, and the wall ghost gradients follow the reference's host
 * rules (Dirichlet velocity 2 (u_b - u_o) / |d| times the face normal,
 * Neumann the owner's gradient times (1 - n)). wall_bc [n_wall] lists the
 * walls as boundary-face indices in the caller's numbering (the reference's
 * bc_types[i] == "wall"); their velocity type must be 1 or 2. Normalisation
 * of the reference: Cd = 2 D / (rho_ref U^2 Y Z), Cl = 2 L / (rho_ref U^2 X Z)
 * with X, Y, Z = plfbs_config.lengths. Leaves the step state unchanged. */
int plfbs_wall_forces(plfbs_ctx* ctx, const int32_t* wall_bc, int32_t n_wall, double* cd,
                      double* cl);

/* Lossless checkpoint at a step boundary (replaces the 6-digit text output of
 * Solution::output, Solution.cpp:221-251, as a restart source): the state,
 * the RK accumulator, the IBM nodes and the run status, in the caller's
 * numbering and the context's precision. plfbs_load_checkpoint into a context
 * created from the same mesh, boundary conditions and precision continues the
 * run bit for bit (IBM force spreading uses atomics, whose order can vary).
 * The image is plfbs_checkpoint_bytes long; a mesh fingerprint, the sizes
 * and the precision are checked on load. No counterpart in the reference. */
int plfbs_checkpoint_bytes(plfbs_ctx* ctx, int64_t* bytes);
int plfbs_save_checkpoint(plfbs_ctx* ctx, void* buf, int64_t bytes);
int plfbs_load_checkpoint(plfbs_ctx* ctx, const void* buf, int64_t bytes);

/* The time loop of Solver_gpu.cu:667-898: up to max_steps steps, stopping after
 * the first step whose max_error < tolerance (Solver_gpu.cu:870). Synchronous.
 * history (optional, may be NULL) receives 6 doubles per completed step:
 * step index, max_error, rho_rms, u_rms, v_rms, w_rms. */
int plfbs_run(plfbs_ctx* ctx, int64_t max_steps, plfbs_stats* stats, double* history);

/* Bounded waits (the reference waits without limit and exits on a CUDA error,
 * Solver_gpu.cu:1419-1431). With a limit of `seconds` > 0, plfbs_run waits at
 * most that long for each batch of up to 2048 launched steps; when it runs out
 * it returns PLFBS_ERR_TIMEOUT without stats or history, and the batch stays
 * in flight: until it ends, every call on the context but plfbs_wait and
 * plfbs_destroy returns PLFBS_ERR_TIMEOUT. plfbs_wait waits at most `seconds`
 * (0: only asks) and returns PLFBS_OK once the steps have ended; the context
 * then carries on from them (their residual history is not returned; their
 * steps count in the next stats). 0 (the default) waits without limit.
 * plfbs_destroy always waits for work in flight. */
int plfbs_set_timeout(plfbs_ctx* ctx, double seconds);
int plfbs_wait(plfbs_ctx* ctx, double seconds);

/* soln.clone(temp_soln) (Solver_gpu.cu:846,872,904): C + B values per array. */
int plfbs_get_state(plfbs_ctx* ctx, double* rho, double* u, double* v, double* w,
                    int64_t n_total);

/* Lagrangian node positions, velocities and forces, 3N each (interleaved xyz). */
int plfbs_get_nodes(plfbs_ctx* ctx, double* x, double* vel, double* force, int32_t n_nodes);

/* Immersed-body drag and lift: -sum(node force) projected on x and y,
 * normalised by 0.5 rho_ref U^2 * frontal_area. No reference counterpart
 * (the reference never reduces IBM forces); returns PLFBS_ERR_STATE without nodes. */
int plfbs_get_body_force(plfbs_ctx* ctx, double frontal_area, double* cd, double* cl);

/* Introspection for parity tests (caller numbering). plfbs_run_stages advances
 * by RK stages (4 per time step; the IBM update runs before each step's first
 * stage) with individual kernel launches instead of the step graph. The
 * getters return the last stage's interior-cell gradients [12C] (rho, u, v, w,
 * each x, y, z), face fluxes [4F] (x, y, z momentum, mass) and residuals [4C]
 * (u, v, w, rho); residuals are only recorded after plfbs_set_debug(ctx, 1). */
int plfbs_set_debug(plfbs_ctx* ctx, int enable);
int plfbs_run_stages(plfbs_ctx* ctx, int64_t n_stages);
int plfbs_get_gradients(plfbs_ctx* ctx, double* grad, int32_t n_cells);
int plfbs_get_face_flux(plfbs_ctx* ctx, double* flux, int32_t n_faces);
int plfbs_get_residual(plfbs_ctx* ctx, double* res, int32_t n_cells);

/* The layout the device built, for tests, in device numbering: sizes[4] =
 * (K stencil slots, K2 gather slots per cell, unique face records and unique
 * cell weight sets of the compact layout in use, 0 where it is not); cell_order [C] and face_order
 * [F] give the caller's cell / face of each device cell / face; stencil_nbr
 * [K*C] and stencil_w [3][K*C] (x, y, z weights, widened from FP32 in the
 * FP32 form) hold slot k of device cell i at k*C + i, neighbour -1 in empty
 * slots (device numbering, ghosts C + device boundary index); gather [K2*C]
 * holds (device face << 1) | (cell is the neighbour), -1 empty. Every array
 * pointer may be NULL; call with only `sizes` first to size the others. */
int plfbs_get_layout(plfbs_ctx* ctx, int32_t* sizes, int32_t* cell_order, int32_t* face_order,
                     int32_t* stencil_nbr, double* stencil_w, int32_t* gather);

/* Host-only: the cell order plfbs_create uses (order[new] = caller cell): the
 * identity for renumber 0, reverse Cuthill-McKee over the internal faces for
 * renumber 1 and 2 (start cells by ascending degree, neighbours by ascending degree,
 * both stable). Needs owner, neighbour and the sizes of `mesh` only. */
int plfbs_cell_order(const plfbs_mesh_view* mesh, int32_t renumber, int32_t* order);

/* Host-only: the least-squares weights as gradients::pre_fill_LHS_and_RHS_matrix
 * computes them (gradients.cpp:214-313, determinant as written at :282-284):
 * lhs_inv [9C] row-major, rhs [3 nnz] per stencil entry. The mesh is checked
 * first as plfbs_create checks it (PLFBS_ERR_ARG / PLFBS_ERR_MESH with the first
 * failing index). No GPU needed. */
int plfbs_ls_weights(const plfbs_mesh_view* mesh, int32_t gradient_mode, double* lhs_inv,
                     double* rhs);

/* Per-kernel device time: advances n_steps time steps launching each kernel
 * between CUDA events and returns the summed milliseconds per kernel kind in
 * ms[4] = {ibm, gradient, flux, update}. For profiling; the state advances. */
int plfbs_profile_steps(plfbs_ctx* ctx, int64_t n_steps, double* ms);

/* Per-kernel device time without launch gaps: each kernel kind launched
 * `launches` times back to back between two CUDA events, mean milliseconds
 * per launch in ms[5] = {ibm, gradient, flux, update (mean of the four RK
 * stages), finish (the residual reduction)}; one step costs about
 * ibm + 4 (gradient + flux + update) + finish. The kernels' outputs that a
 * later step reads (state, RK accumulators, body force, nodes, run status)
 * are copied aside on the device first and put back afterwards, so the run
 * continues as if nothing had happened. For profiling; no reference
 * counterpart. */
int plfbs_profile_kernels(plfbs_ctx* ctx, int64_t launches, double* ms);

/* FP64 fused multiply-add throughput of a device, measured (GFLOP/s, two per
 * FMA): a one-wave kernel of independent FMA chains, best of five timed
 * launches. The denominator of a kernel's FP64-pipe fraction; changes no
 * device setting. No reference counterpart. */
int plfbs_fp64_fma_peak(int32_t device, double* gflops);

/* Which FP64 flux kernel the step uses: 0 = one thread per face gathering its
 * cells' state and gradients itself (the default); 1 = internal faces staged
 * through shared memory by a producer warp's tile::gather4 bulk tensor copies
 * (TMA), consumer warps computing from shared memory, boundary faces as in 0.
 * Both compute the same flux bit for bit. PLFBS_ERR_ARG for FP32 contexts. */
int plfbs_set_flux_kernel(plfbs_ctx* ctx, int32_t kind);

/* Contexts store bitwise-equal face records (normal, area, streaming dt,
 * centroid offsets, relaxation factor) and cells' gradient-weight sets once,
 * each face or cell keeping an index, when a table holds at most 1/8 of the
 * items (structured regions of a mesh repeat their geometry): the kernels
 * read 4 bytes per face and per cell instead of 96 and 24 K (FP32: 48 and
 * 12 K). On by default where available; 0 reads the per-item arrays (the
 * same bits, so the same results). PLFBS_ERR_ARG when the mesh has no compact
 * layout. */
int plfbs_set_layout_compression(plfbs_ctx* ctx, int32_t on);

/* Device bytes held by the context. */
int plfbs_memory_bytes(plfbs_ctx* ctx, int64_t* bytes);

/* Residual norms with no device allocation. No counterpart in the reference.
 * For callers that cannot let a library call cudaMalloc while they run: an
 * application under a fixed device-memory budget that reserves everything at
 * start-up (an allocation mid-run may fail, and cudaMalloc may synchronise the
 * device), or a host framework whose caching allocator must own all device
 * memory. From residuals the caller keeps in device memory ([4 n_cells]:
 * u, v, w, rho per cell, as plfbs_get_residual lays them out) it writes
 * out[5] = {max_error, rho_rms, u_rms, v_rms, w_rms} (device memory) with the
 * normalisation of plfbs_run's last RK stage (residuals.cpp:95-147),
 * asynchronously on `stream` (a cudaStream_t, NULL for the default stream).
 * Its only scratch is a file-scope __device__ array of 65,792 bytes (2048
 * block partials + a counter) that every GPU loading this library holds until
 * exit, so n_cells is limited to 8,388,608; larger inputs are rejected with
 * PLFBS_ERR_ARG. A call made outside stream capture looks up that array's
 * device address in the current context with cudaGetSymbolAddress; a call
 * under capture reuses the address the last uncaptured call on that device
 * found, so make the first call on each device before any stream capture
 * (and one again after a device reset). All calls share the array: calls
 * that overlap on the GPU (other streams, other host threads) race and must
 * be serialised by the caller. Errors are reported through
 * plfbs_last_error(NULL). */
int plfbs_residual_norms_noalloc(const double* residual, int64_t n_cells, double ref_rho,
                                 double max_velocity, double* out, void* stream);

const char* plfbs_last_error(const plfbs_ctx* ctx);  /* ctx may be NULL: this thread's last error */

/* Frees the context (replaces the end of General_Purpose_Solver_mk_i; the
 * reference never frees its managed buffers). Its device arrays return to a
 * per-device memory pool of this library, which keeps them for the next
 * plfbs_create on that device instead of unmapping them. */
void plfbs_destroy(plfbs_ctx* ctx);

/* Returns the memory cached in this library's pool for `device` to the driver
 * (contexts still alive keep theirs), and frees the pinned host status and
 * staging buffers destroyed contexts left for reuse. No counterpart in the
 * reference.
 * Errors are reported through plfbs_last_error(NULL). */
int plfbs_release_cached(int32_t device);

const char* plfbs_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PLFBS_H */
