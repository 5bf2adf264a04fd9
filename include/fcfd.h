/*
 * fcfd.h — C ABI of the B200 residual / Newton-Krylov library (libfcfd_b200.so).
 *
 * Free CFD has no plugin or FFI layer: its residual path is a set of C++
 * member functions of NavierStokes/RANS reading process-global state
 * (src/navier_stokes/ns.h:57-64, src/rans/rans.h:40-45).  Each entry point
 * below names the reference routine(s) it stands in for.  Conventions:
 *   - every function returns an int status (FCFD_OK = 0) and never exits;
 *     fcfd_last_error() returns a message for the calling thread;
 *   - cell arrays are in the reference's cell order (Grid::create_nodes_cells,
 *     src/grid/grid_create_elements.cc:27-182), AoS [cell][5] = (p,u,v,w,T)
 *     primitive gauge variables (src/navier_stokes/ns.cc:356-361);
 *   - face arrays are in the reference's face order (Grid::create_faces,
 *     src/grid/grid_create_elements.cc:184-412);
 *   - host pointers unless FCFD_DEVICE_PTRS is passed in `flags`;
 *   - a context owns its device buffers and one CUDA stream; it is not
 *     thread-safe; separate contexts may run concurrently.
 */
#ifndef FCFD_H
#define FCFD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum fcfd_status {
  FCFD_OK = 0,
  FCFD_ERR_INPUT = 1,          /* bad deck / argument (reference: cerr + exit(1)) */
  FCFD_ERR_MESH = 2,           /* mesh could not be built (e.g. unassigned boundary face) */
  FCFD_ERR_DIVERGED = 3,       /* NaN/Inf in an update (reference: ns.cc:349-355 MPI_Abort) */
  FCFD_ERR_NOT_CONVERGED = 4,  /* Newton / Krylov iteration cap reached */
  FCFD_ERR_CUDA = 5,           /* CUDA runtime error */
  FCFD_ERR_TIMEOUT = 6,        /* a bounded device wait ran out */
  FCFD_ERR_UNSUPPORTED = 7,    /* option outside the restated path */
  FCFD_ERR_BC = 8              /* boundary condition failure (e.g. supersonic inlet without state) */
};

enum fcfd_flags {
  FCFD_DEVICE_PTRS = 1, /* input/output pointers are device pointers on the context's device */
  FCFD_JVP_FP32 = 4,    /* fcfd_jvp: evaluate the tangent chain in FP32 (value and derivative) */
  FCFD_NO_SYNC = 8      /* fcfd_partition_residual with device pointers: enqueue only, no host
                           synchronisation; a BC error stays flagged on the device until
                           fcfd_ctx_check (or the next synchronising call) reports it */
};

enum fcfd_precision { FCFD_FP64 = 0, FCFD_FP32 = 1 };

typedef struct fcfd_case fcfd_case;
typedef struct fcfd_mesh fcfd_mesh;
typedef struct fcfd_ctx fcfd_ctx;

/* CELL-type raw grid, same meaning as GridRawData (src/grid/grid.h:61-78):
 * node coordinates, CGNS-ordered element connectivity (4/6/8-node cells),
 * and per boundary region the node ids on it (region b is BC_{b+1}). */
typedef struct fcfd_raw_mesh {
  int32_t n_nodes;
  const double *xyz;          /* [n_nodes][3] */
  int32_t n_cells;
  const int32_t *conn_index;  /* [n_cells+1] */
  const int32_t *conn;        /* [conn_index[n_cells]] */
  int32_t n_bc;
  const int32_t *bc_index;    /* [n_bc+1] */
  const int32_t *bc_nodes;    /* [bc_index[n_bc]] */
} fcfd_raw_mesh;

const char *fcfd_last_error(void);
const char *fcfd_version(void);

/* Parse an input deck (+ <material>.mat beside it).  Replaces read_inputs()
 * (src/read_inputs.cc:28-218), InputFile (src/inputs/inputs.cc:37-345),
 * MATERIAL::set (src/material/material.cc:29-106) and NavierStokes::set_bcs
 * (src/navier_stokes/ns_set_bcs.cc:25-140). */
int fcfd_case_from_deck(const char *deck_path, fcfd_case **out);
void fcfd_case_destroy(fcfd_case *cs);
/* dv[13] = gamma, R, Pref, Tref, Minf, limiter threshold, mu, lambda,
 *          sutherland mu_ref, T_ref, S, Pr, (unused 0)
 * iv[7+4*n_bc] = flux, limiter, order, sutherland, prandtl, n_bc, dimension,
 *                then per BC: type, kind, specified, thermalType           */
int fcfd_case_summary(const fcfd_case *cs, double *dv, int32_t *iv, int32_t iv_len);

/* Build connectivity, geometry and stencils.  Replaces Grid::setup
 * (src/grid/grid.cc:55-82), set_bcs (src/set_bcs.cc:35-260),
 * set_lengthScales (src/main.cc:456-491), face_interpolation_weights
 * (src/face_interpolation_weights.cc:32-138) and gradient_maps/lsqr_grad_map
 * (src/gradient_maps.cc:39-78, src/lsqr_grad_map.cc:32-99). */
int fcfd_mesh_create(const fcfd_raw_mesh *raw, const fcfd_case *cs, fcfd_mesh **out);
void fcfd_mesh_destroy(fcfd_mesh *m);
/* Read a Tecplot FEPolyhedron grid file (the deck's `format=tecplot`,
 * Grid::readTEC src/grid/grid_reader_tec.cc:36-278) and build the mesh from
 * its faces (Grid::create_faces2, grid_create_elements.cc:444-553): face
 * order, parent / neighbour = the file's left / right elements, boundary
 * regions from the boundary zones in file order (BC_1 = first zone).  Faces
 * have 3 or 4 nodes.  bc_names (may be NULL) receives the zone names,
 * newline-separated. */
int fcfd_mesh_from_tecplot(const char *path, const fcfd_case *cs, fcfd_mesh **out, char *bc_names, int32_t bc_names_len);
/* out[8] = n_cells, n_faces, n_ghosts, n_total, n_nodes, stencil entries,
 *          cell-face entries, neighbour entries */
int fcfd_mesh_sizes(const fcfd_mesh *m, int64_t *out);
/* Reference-order integer connectivity (for bit-exact parity checks). */
int fcfd_mesh_connectivity(const fcfd_mesh *m, int32_t *face_parent, int32_t *face_neighbor, int32_t *face_bc,
                           int32_t *face_nodes /* [nf][4], -1 pad */, int32_t *cell_face_index,
                           int32_t *cell_faces, int32_t *nbr_index, int32_t *nbrs, int32_t *grad_index,
                           int32_t *grad_keys);
/* Geometry in reference order (ghost cells follow interior cells). */
int fcfd_mesh_geometry(const fcfd_mesh *m, double *face_normal, double *face_area, double *face_centroid,
                       double *face_avg /* [nf][2] */, double *cell_centroid, double *cell_volume,
                       double *cell_length, double *cell_wall_distance, double *length_scale);

/* Least-squares gradient data per interior cell: cofactors[nc][7] =
 * (C00,C01,C02,C11,C12,C22,det) of the weighted normal matrix and
 * self_weight[nc][3], the weight of the cell's own value
 * (lsqr_grad_map, src/lsqr_grad_map.cc:74-96). */
int fcfd_mesh_lsq(const fcfd_mesh *m, double *cofactors, double *self_weight);

/* Stored gradient-map weights, weights[E][3] in the order of the stencil
 * keys of fcfd_mesh_connectivity (grad_index / grad_keys): built when some
 * cell takes the curvilinear map (curvilinear_grad_map.cc:28-228, the
 * reference's default for hexahedra and prisms, read_inputs.cc:47-48); the
 * least-squares cells of such a mesh store lsqr_grad_map's weights
 * (lsqr_grad_map.cc:86-96).  FCFD_ERR_UNSUPPORTED for a mesh without
 * curvilinear cells (its least-squares weights are rebuilt on the device). */
int fcfd_mesh_grad_weights(const fcfd_mesh *m, double *weights);

/* Reverse Cuthill-McKee order of the interior cells over the face-neighbour
 * graph: perm[new] = old, nc entries.  The reference takes its cell order
 * from the grid file's element order, or from ParMETIS when partitioned
 * (grid_partition.cc:25-141); it has no renumbering for locality.  A caller
 * with an unordered grid (a face-based Tecplot file, a shuffled export)
 * lists the elements in this order and builds the mesh again: every face's
 * gathers then touch nearby cells.  Deterministic (ties to the lower index).
 * Host only. */
int fcfd_mesh_rcm(const fcfd_mesh *m, int32_t *perm);

/* Create a device context on CUDA device `device`. */
int fcfd_ctx_create(const fcfd_mesh *m, const fcfd_case *cs, int device, fcfd_ctx **out);
void fcfd_ctx_destroy(fcfd_ctx *ctx);

/* Gradient arithmetic.  By default the LSQ gradient is evaluated bit-exactly
 * (the reference's rounded sums, src/lsqr_grad_map.cc:86-94, src/variable/variable.h:194-202)
 * when the limiter decides on the sign of rounding noise (minmod,
 * Barth-Jespersen, VK with threshold 0) and in a fused form equal to it up to
 * rounding otherwise.  exact=1 forces the bit-exact form for every limiter. */
int fcfd_ctx_set_exact_gradients(fcfd_ctx *ctx, int exact);

/* Gradient + limiter kernel (calc_cell_grads + calc_limiter, ns.cc:301-336,
 * ns_limiters.cc): 0 automatic (1), 1 per cell (one or,
 * on small meshes, two threads per cell gathering each stencil cell from
 * L2), 2 per tile of 128 consecutive cells with the states and centroids the
 * tile's stencils and faces name staged in shared memory once (same
 * arithmetic), 3 per cell with the fused least-squares sums over folded
 * stencils: the ghosts of z-normal symmetry faces (the front and back planes
 * of one-layer meshes) hold their parents' states with w negated, so their
 * terms join their parents' entries (27 entries become 9; equal to the
 * unfolded sum to rounding; continuous limiters only, the bit-exact path is
 * unchanged; measured no faster than 1 on the benchmark cylinder, since the
 * stencil loop does not set that kernel's time).  FCFD_ERR_UNSUPPORTED for a
 * kind the mesh does not have. */
int fcfd_ctx_set_gradient_kernel(fcfd_ctx *ctx, int kind);

/* on = 1 (the default): the residual chain's gradient and face kernels are
 * programmatic dependent launches, scheduled while their predecessor in the
 * stream finishes and waiting on the device for its results, so a
 * kernel boundary costs less than a full drain and launch; 0: ordinary
 * launches.  The results are the same bits either way. */
int fcfd_ctx_set_launch_overlap(fcfd_ctx *ctx, int32_t on);

/* The gradient kernel the residual runs: out[0] = 1 per cell, 2 tiles, 3
 * per cell over folded stencils; out[1] = folded stencil entries (0 if not
 * built); out[2] = 1 for the fused (continuous-limiter) gradient, 0 for the
 * bit-exact one. */
int fcfd_ctx_gradient_info(const fcfd_ctx *ctx, int64_t *out);

/* Spatial residual R(W) = sum over faces of +/-(F_diffusive - F_convective)
 * for the interior-cell state W[nc][5].  Replaces the residual part of
 * NavierStokes::assemble_linear_system (src/navier_stokes/ns_assemble_linear_system.cc:34-140)
 * preceded by update_boundaries (reconstructed, first-order ghost update as at
 * initialise, ns.cc:93), calc_cell_grads (ns.cc:301-336) and calc_limiter
 * (ns_limiters.cc:26-248).  R[nc][5]. */
int fcfd_residual(fcfd_ctx *ctx, const double *W, double *R, int flags);
/* Per-stage outputs of the last fcfd_residual call (reference order):
 * grads[nc][15] (p,u,v,w,T gradients), limiter[nc][5], ghost[n_ghosts][5],
 * mdot[nf] (Variable mdot, ns_assemble_linear_system.cc:123), weightL[nf]. */
int fcfd_last_stages(fcfd_ctx *ctx, double *grads, double *limiter, double *ghost, double *mdot, double *weightL);
/* Local time step, update_time_step (src/time_step.cc:143-224):
 * mode 0 = CFL_LOCAL (dt_c = cfl*l_c/(|V|+a)), mode 1 = CFL_MAX (global min). */
int fcfd_local_dt(fcfd_ctx *ctx, const double *W, double cfl, int mode, double *dt, int flags);

/* Forward-tangent (JVP) of the residual: JV = (dR/dW) V for a direction
 * V[nc][5], evaluated by the same kernels on dual numbers (exact derivative
 * of the discrete residual, not a finite difference).  Optionally returns
 * R(W) too (R may be NULL).  Replaces the finite-difference Jacobian columns
 * of NavierStokes::get_jacobians (ns_assemble_linear_system.cc:197-267) in a
 * matrix-free Newton-Krylov solve. */
int fcfd_jvp(fcfd_ctx *ctx, const double *W, const double *V, double *R, double *JV, int flags);

/* Adjoint (VJP) of the residual: Wbar = (dR/dW)^T Rbar for a cotangent
 * Rbar[nc][5]; the backward half of the (fcfd_jvp, fcfd_vjp) pair, exact for
 * the discrete residual (the branches taken at W).  The reference has no
 * adjoint; the map it transposes is the residual of
 * NavierStokes::assemble_linear_system (ns_assemble_linear_system.cc:34-140)
 * with calc_cell_grads (ns.cc:301-336) and calc_limiter (ns_limiters.cc). */
int fcfd_vjp(fcfd_ctx *ctx, const double *W, const double *Rbar, double *Wbar, int flags);

/* k-omega RANS residual for the state W[nc][5] and K[nc][2] = (k, omega):
 * R[nc][5] is the NS residual with the eddy viscosity mu_t in the viscous
 * flux (ns_diffusive_face_flux.cc:36-39), RK[nc][2] the k and omega
 * right-hand side of RANS::terms (rans_terms.cc:39-275) with the eddy
 * viscosity of rans_update_eddy_viscosity.cc:26-56 and the fixed BC values of
 * rans_set_bcs.cc:25-83.  Only model=k-omega; FCFD_ERR_INPUT if the case has
 * no turbulence section. */
int fcfd_rans_residual(fcfd_ctx *ctx, const double *W, const double *K, double *R, double *RK, int flags);
/* Device time (CUDA events) of the coupled NS + k-omega residual on the
 * state of the last fcfd_rans_residual call: out[0] ms per evaluation,
 * out[1] the NS part, out[2] the k-omega part; the L2 cache is flushed before
 * each evaluation when flush_l2 != 0.  Benchmark entry point, no counterpart
 * in the reference. */
int fcfd_time_rans(fcfd_ctx *ctx, int reps, int flush_l2, double *out, int out_len);
/* Forward tangent of the coupled residual: (JV, JVK) = d(R, RK)/d(W, K)
 * applied to (V[nc][5], VK[nc][2]), evaluated by the same kernels as
 * fcfd_rans_residual on dual numbers (the eddy viscosity, the k-omega fluxes
 * and sources and their coupling into the NS viscous flux all carry the
 * tangent).  R and RK (both or neither) receive the residual.  flags may
 * add FCFD_JVP_FP32: the tangent chain in single precision (as fcfd_jvp). */
int fcfd_rans_jvp(fcfd_ctx *ctx, const double *W, const double *K, const double *V, const double *VK, double *R,
                  double *RK, double *JV, double *JVK, int flags);
/* Adjoint of the coupled residual, the backward half of the (fcfd_rans_jvp,
 * fcfd_rans_vjp) pair: (Wbar[nc][5], Kbar[nc][2]) = (d(R, RK)/d(W, K))^T
 * (Rbar[nc][5], RKbar[nc][2]), exact for the discrete residual (the branches
 * taken at W, K).  Reverses the eddy viscosity (rans_update_eddy_viscosity.cc
 * :26-56), its face values, the k-omega gradients, face fluxes and sources
 * (rans_terms.cc:39-275), their coupling into the NS viscous flux
 * (ns_diffusive_face_flux.cc:36-39) and the NS residual as fcfd_vjp does.
 * Deterministic (every accumulation has a fixed order). */
int fcfd_rans_vjp(fcfd_ctx *ctx, const double *W, const double *K, const double *Rbar, const double *RKbar,
                  double *Wbar, double *Kbar, int flags);
/* Domain decomposition: one rank's part of the residual.  Replaces the
 * partition-ghost exchange of the reference's MPI runs
 * (NavierStokes::mpi_update_ghost_primitives / mpi_update_ghost_gradients,
 * navier_stokes/ns_mpi.cc:62-140, called from ns.cc:92-115) and the extrema
 * all-reduce of find_min_max (ns.cc:425-427).  A rank owns the global cells
 * [lo, hi).  fcfd_partition_sets (host only, no device needed) returns
 * counts[4] = {cells whose gradient is formed, faces whose flux is formed,
 * halo cells, ghosts updated} and, where the arrays are not NULL, the
 * gradient cells, the faces and the halo cells (not owned; their states must
 * be current before phase 1; ascending global ids).  Gradients are
 * recomputed on the halo, so only states are exchanged.
 *
 * fcfd_ctx_set_partition selects the range on a context (lo = hi = 0: none;
 * FCFD_ERR_UNSUPPORTED for k-omega cases).
 * fcfd_partition_extrema (phase 1) loads W [nc][5] and returns ext[8]: the
 * VK limiter's extrema over the owned cells (max p, min p, max u, min u,
 * max v, min v, max p and min p below the last cell; -inf/+inf where empty),
 * to be combined over the ranks with max (even slots) and min (odd slots).
 * fcfd_partition_residual (phase 2) takes the combined ext and writes rows
 * [lo, hi) of R [nc][5]: bit for bit the single-domain residual's rows.
 * With FCFD_DEVICE_PTRS, W, ext and R are device pointers; phase 1 then only
 * enqueues work on the context's stream (fcfd_ctx_stream), so the caller can
 * all-reduce ext on that stream and call phase 2 without a host round trip
 * (phase 2 synchronises once and reports BC errors of both phases). */
int fcfd_partition_sets(const fcfd_mesh *mesh, const fcfd_case *cs, int lo, int hi, int counts[4], int *grad_cells,
                        int *faces, int *halo);
int fcfd_ctx_set_partition(fcfd_ctx *ctx, int lo, int hi);
int fcfd_partition_extrema(fcfd_ctx *ctx, const double *W, double ext[8], int flags);
int fcfd_partition_residual(fcfd_ctx *ctx, const double ext[8], double *R, int flags);
/* The CUDA stream (cudaStream_t) the context's work is enqueued on. */
int fcfd_ctx_stream(const fcfd_ctx *ctx, void **stream);
/* Waits for the context's stream and reports (and clears) a boundary-condition
 * error flagged by work enqueued without synchronisation (FCFD_NO_SYNC):
 * FCFD_ERR_BC, or FCFD_OK. */
int fcfd_ctx_check(fcfd_ctx *ctx);

/* Fixed BC values of the RANS variables, per BC region: kw_fixed, k, omega,
 * mut_fixed, mu_t (5 doubles each; out_len >= 5 * number of regions). */
int fcfd_rans_bcs(const fcfd_ctx *ctx, double *out, int32_t out_len);

/* Boundary loads and their adjoint gradient.  force[3] = sum over the faces
 * of every BC region b with bit b of bc_mask set of the convective minus
 * diffusive momentum flux times area (the loads of
 * ns_assemble_linear_system.cc:108-119: pressure + viscous force on the
 * region).  If dJdW is not NULL it receives d(force . dir)/dW [nc][5] (e.g.
 * dir = freestream direction: the drag gradient). */
int fcfd_drag(fcfd_ctx *ctx, const double *W, uint32_t bc_mask, const double *dir, double *force, double *dJdW,
              int flags);

/* Options of the device Newton-Krylov solve. */
typedef struct fcfd_newton_opts {
  int32_t max_newton;     /* Newton (pseudo-time) steps, default 200 */
  double tol;             /* stop when |R_mass|_2 <= tol * |R_mass(W0)|_2 */
  int32_t krylov_dim;     /* GMRES basis size m (one cycle per Newton step), default 30 */
  double krylov_rtol;     /* GMRES relative tolerance, default 1e-2 */
  double cfl0;            /* initial CFL (time marching ramp initial) */
  double cfl_growth;      /* ramp growth per step (cfl_mode 0) */
  double cfl_max;         /* CFL cap */
  int32_t cfl_mode;       /* 0: reference ramp (time_step.cc:146-156); 1: CFL0 * (|R0|/|R|)^ser_exponent */
  double ser_exponent;
  int32_t jvp_mode;       /* 0: finite-difference J.v of the FP64 residual; 1: tangent (dual-number)
                             kernels with the limiter held fixed (frozen-limiter Jacobian);
                             2: tangent kernels, exact (limiter differentiated too);
                             3: as 2 with the tangent chain in FP32 (mixed precision: the FP64
                                residual stays the outer Newton residual);
                             4: as 1 (limiter held fixed) with the tangent chain in FP32 */
  int32_t fp32_krylov;    /* 1: Krylov basis, preconditioner couplings, vectors and Gauss-Seidel
                             arithmetic in FP32 (dot products and Gram-Schmidt in FP64) */
  double max_seconds;     /* wall-clock cap (0: none) */
  int32_t precond_sweeps; /* symmetric multicolour block Gauss-Seidel sweeps on the first-order
                             operator (0: block-Jacobi, the block diagonal only) */
  int32_t krylov_cycles;  /* GMRES(m) restarts per Newton step (default 1) */
  int32_t stop_all_rows;  /* 1: stop only when the momentum (x,y,z together) and energy residual
                             norms have also dropped by tol from their initial values */
  int32_t gs_launch;      /* Gauss-Seidel sweeps: 0 one launch per colour update (default); 1 all colour
                             updates of a preconditioner application in one cooperative launch with
                             grid barriers between them (couplings staged in shared memory where they
                             fit; a barrier that waits too long ends the solve with FCFD_ERR_TIMEOUT) */
  int32_t precond_ilu0;   /* 1: block ILU(0) of the first-order operator in the multicolour order
                             (modified diagonal blocks, one forward and one backward colour sweep)
                             instead of block Jacobi / Gauss-Seidel; precond_sweeps is ignored.  The
                             reference's PETSc default for its FGMRES (ns_petsc_functions.cc:25-83) is
                             block Jacobi with ILU(0) inside each process's block */
  int32_t local_relax;    /* 0: the whole update is scaled so that p and T change by at most 20 % in
                             every cell; 1: each cell's update is scaled on its own to that bound
                             (local under-relaxation: cells far from a shock or a wake take full
                             steps), inactive once every cell's change is below the bound */
  int32_t startup_steps;  /* > 0: before the Newton steps, up to this many explicit steps (forward
                             Euler in the primitive variables with local time steps at cfl0,
                             (V P/dt) dW = R per cell) until the mass residual has dropped by
                             startup_drop; for start-up transients that a linearised implicit step
                             does not keep physical (an impulsively started hypersonic flow) */
  double startup_drop;    /* explicit start-up target drop (default 1e-3) */
} fcfd_newton_opts;

typedef struct fcfd_newton_report {
  int32_t status, newton_iterations, krylov_iterations, pad;
  double res0, res_final, wall_seconds, last_cfl;
  double history[512];    /* |R_mass| / |R_mass(W0)| per Newton step */
  double rows_final[3];   /* final / initial norm of the mass, momentum and energy residual */
  double seconds_to_tol;  /* wall time when |R_mass| first dropped by tol */
  double seconds_history[512]; /* wall time at each history[] entry */
  double kw_final[2];     /* fcfd_rans_newton_solve: final / initial norm of the k and omega residuals */
  int32_t startup_steps;  /* explicit start-up steps taken (fcfd_newton_opts.startup_steps) */
  int32_t pad2;
} fcfd_newton_report;

/* Mixed-precision residual: fcfd_residual's R(W) with the face pass in FP32
 * where the flow is smooth and in FP64 at shocks.  Ghost states, gradients,
 * limiters and the gather stay FP64 (the reference's minmod / Barth-Jespersen
 * decisions on one-layer meshes follow the sign of the FP64 gradient's
 * rounding noise); a face whose two cell-centre absolute pressures differ by
 * more than the factor shock_ratio runs in FP64, so the equation of state
 * (material.cc:108-153) and the flux's pressure terms across a captured
 * shock keep FP64; every other face evaluates reconstruction, equation of
 * state, convective and viscous flux in FP32 and its face difference is
 * summed in FP64.  shock_ratio < 1 sends every face to the FP64 pass.
 * *n_fp64_faces (may be null) receives the number of FP64 faces.  No
 * counterpart in the reference (its residual is FP64 throughout). */
int fcfd_residual_mixed(fcfd_ctx *ctx, const double *W, double *R, double shock_ratio, int32_t flags,
                        int64_t *n_fp64_faces);

/* Device time of the mixed-precision chain on the state of the last residual
 * call: out[0] = mean ms per evaluation over reps (L2 flushed before each
 * when flush_l2), out[1] = FP64 faces of the last evaluation. */
int fcfd_time_residual_mixed(fcfd_ctx *ctx, int32_t reps, int32_t flush_l2, double shock_ratio, double *out);

/* Steady solve R(W) = 0 by pseudo-transient matrix-free Newton-Krylov on the
 * device: (V P/dt - dR/dW) dW = R(W), W += dW, with P = cons2prim
 * (ns_time_terms.cc:26-56), local dt (time_step.cc:143-224), block-Jacobi
 * preconditioner from first-order face Jacobians (get_jacobians,
 * ns_assemble_linear_system.cc:197-267) and GMRES(m) with FP64
 * Gram-Schmidt.  Replaces NavierStokes::solve's assemble + PETSc FGMRES
 * (ns.cc:104-118, ns_petsc_functions.cc:85-110).  W[nc][5] host, in/out.
 * Returns FCFD_ERR_NOT_CONVERGED / FCFD_ERR_DIVERGED with the report filled. */
int fcfd_newton_solve(fcfd_ctx *ctx, double *W, const fcfd_newton_opts *opts, fcfd_newton_report *report);

/* Diagonal blocks V P/dt - J_cc of the implicit operator at the state W[nc][5]
 * and local time steps dt[nc] (both host): the matrix the block
 * preconditioner of fcfd_newton_solve / fcfd_run inverts.  Replaces the
 * diagonal of the matrix that NavierStokes::time_terms (P V / dt,
 * ns_time_terms.cc:107-186 with cons2prim 26-56) and assemble_linear_system's
 * first-order Jacobian (get_jacobians, ns_assemble_linear_system.cc:142-267)
 * build; here J_cc is the exact derivative of the first-order face fluxes
 * (the reference takes finite differences).  blocks[nc][5][5], row =
 * equation (mass, momentum x/y/z, energy), column = primitive (p,u,v,w,T). */
int fcfd_diag_blocks(fcfd_ctx *ctx, const double *W, const double *dt, double *blocks);

/* Time-term blocks V P/dt of the implicit operator at the state W[nc][5] and
 * local time steps dt[nc] (host): NavierStokes::time_terms
 * (ns_time_terms.cc:107-186, cons2prim 26-56).  blocks[nc][5][5], the layout
 * of fcfd_diag_blocks.  A caller that forms (V P/dt - dR/dW) z itself (a
 * domain-decomposed solver) applies these to z. */
int fcfd_time_terms(fcfd_ctx *ctx, const double *W, const double *dt, double *blocks);

/* Coupled steady solve of the flow and k-omega residuals (turbulent decks):
 * pseudo-transient Newton-Krylov on X = (p,u,v,w,T,k,omega) per cell, one
 * system where the reference solves NavierStokes::solve and then RANS::solve
 * (ns.cc:104-118, rans.cc:85-98), each with its own time terms
 * (ns_time_terms.cc:107-186, rans_time_terms.cc:25-87).  J.v by a finite
 * difference of the FP64 coupled residual (jvp_mode 0) or the coupled tangent
 * chain in FP32 (any other jvp_mode); block-Jacobi preconditioner (the flow
 * blocks from first-order face Jacobians with the eddy viscosity, a diagonal
 * for k and omega); GMRES(krylov_dim), one cycle per step, FP64 Gram-Schmidt.
 * Uses tol, max_newton, krylov_dim, krylov_rtol, cfl0, cfl_max,
 * cfl_mode (SER on the mass residual, or 2: on the largest per-equation
 * drop), ser_exponent, max_seconds and
 * stop_all_rows (all seven equations instead of the mass residual alone).
 * W[nc][5] and K[nc][2] host, in/out; k and omega are kept at or above the
 * deck's klowlimit / omegalowlimit. */
int fcfd_rans_newton_solve(fcfd_ctx *ctx, double *W, double *K, const fcfd_newton_opts *opts,
                           fcfd_newton_report *report);

/* Deck-driven time loop (main.cc:294-438) for one laminar or Euler grid,
 * replacing the reference's main program after set-up.  Per time step:
 * update_time_step (time_step.cc:143-224: CFL ramp, schedule file, FIXED /
 * CFL_MAX / CFL_LOCAL step, max CFL, physical time), one implicit
 * backward-Euler step (NavierStokes::solve, ns.cc:104-118) solved by GMRES
 * with the deck's navierstokes relative tolerance, absolute tolerance (in the
 * row-scaled norm) and maximum iterations (one cycle), W += dW, the residual
 * of update_variables (ns.cc:338-396), a convergence.dat line (main.cc:
 * 351-369: step, grid, time, max CFL, linear iterations, residual), loads files
 * volume_output/loads_grid_1_BC_<b>.dat (write_loads, write_volume_output.cc:
 * 65-85) every loadfrequency steps, restart files every restartfrequency
 * steps, at the last step and when a file named dump_restart appears in the
 * run directory (write_restart.cc:45-100), and every updatefrequency steps a
 * re-read of the deck's timemarching section.  The implicit operator is the
 * full Jacobian (jvp_mode as in fcfd_newton_opts), preconditioned by the
 * first-order one; the reference solves with its first-order FD Jacobian.
 * Turbulent decks and pseudo-time sub-iterations return
 * FCFD_ERR_UNSUPPORTED; a NaN/Inf update returns FCFD_ERR_DIVERGED (the
 * reference aborts).  W[nc][5] host, in/out. */
typedef struct fcfd_run_opts {
  const char *work_dir;   /* run directory (the reference's working directory); NULL: "." */
  int32_t restart_step;   /* > 0: read restart/<step>/ from work_dir and continue with step+1 */
  int32_t max_steps;      /* > 0: overrides timemarching -> numberofsteps */
  int32_t jvp_mode;       /* J.v of the implicit operator, as in fcfd_newton_opts */
  int32_t fp32_krylov;    /* as in fcfd_newton_opts */
  int32_t precond_sweeps; /* as in fcfd_newton_opts */
  int32_t echo;           /* 1: also print the reference's screen lines to stdout */
  double *K;              /* turbulent decks: k and omega per cell [nc][2], in/out (required); the
                             time step is then one coupled implicit solve on (p,u,v,w,T,k,omega)
                             where the reference solves the flow and then the k-omega system
                             (ns.cc:104-118, rans.cc:85-98); convergence.dat adds the k-omega
                             iterations and residual (main.cc:351-361), restart files k, omega, mu_t */
} fcfd_run_opts;

typedef struct fcfd_run_report {
  int32_t status, steps, krylov_iterations, pad;
  double time, res, wall_seconds;
} fcfd_run_report;

int fcfd_run(fcfd_ctx *ctx, double *W, const fcfd_run_opts *opts, fcfd_run_report *report);

/* Restart files in the reference's layout under <dir>/restart/ (dir NULL:
 * "."): partitionMap_<gid>.dat, <step>/time.dat and raw native-endian doubles
 * per cell <step>/{dt,p,V,T[,k,omega,mu_t]}.<gid> (write_restart.cc:45-100,
 * ns_write_restart.cc:25-35, rans_write_restart.cc:25-35,
 * Variable::dump_cell_data variable.h:229-245).  gid = the grid number of
 * the file names (1 for grid_1); one partition, global id of cell c = c.
 * first_res[3] = the NS residual normalisations, rans_first_res[2] the RANS
 * ones (NULL writes -1 -1); W[nc][5] = (p,u,v,w,T); dt[nc] may be NULL;
 * K[nc][2] = (k, omega) and mu_t[nc] may be NULL (laminar). */
int fcfd_restart_write(const char *dir, int32_t gid, int32_t step, double time, const double *first_res,
                       const double *rans_first_res, int32_t n_cells, int32_t n_nodes, const double *W,
                       const double *dt, const double *K, const double *mu_t);
/* Reads the files fcfd_restart_write (or the reference) wrote, placing each
 * value by the global cell id of the partition map (read_restart.cc:44-102,
 * Variable::read_cell_data variable.h:248-271).  Any output may be NULL
 * except W. */
int fcfd_restart_read(const char *dir, int32_t gid, int32_t step, int32_t n_cells, double *time, double *first_res,
                      double *rans_first_res, double *W, double *K, double *mu_t);

/* Device timing of the residual: runs `reps` residual evaluations on the
 * resident state (captured in one CUDA graph) and returns per-kernel average
 * milliseconds: out[0] total per residual, out[1..] per kernel (see fcfd.cu). */
int fcfd_time_residual(fcfd_ctx *ctx, int reps, int flush_l2, double *out, int out_len);

/* Allocation-free CFL_MAX local time step, for callers that cannot call
 * cudaMalloc (host applications that own all device memory through their own
 * pool, code that must not allocate once set up).  No counterpart in the
 * reference.  Same result as fcfd_local_dt(mode 1) but with no context: all
 * pointers are device pointers, W[n_cells][5] = (p,u,v,w,T), length[n_cells]
 * = cell length scales, dt[n_cells] output; gas_R, Pref, Tref as in the deck;
 * stream may be NULL (legacy default stream).  The scratch for the global
 * minimum is a file-scope __device__ array of 4096+32 doubles, so n_cells is
 * limited to 1,048,576 (larger sizes return FCFD_ERR_INPUT).  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress);
 * make that first call before any stream capture.  That address is kept for
 * the life of the process: after cudaDeviceReset on a device the library must
 * not be called on that device again.  A cell whose time step is NaN is left
 * out of the minimum, as std::min leaves it out in update_time_step
 * (time_step.cc:181-186); fcfd_local_dt does the same.  A CUDA error already
 * pending on the calling thread is reported (FCFD_ERR_CUDA) without launching
 * and without clearing it.  Every call shares the one array: calls that
 * overlap on the GPU race and must be serialised. */
int fcfd_local_dt_cflmax_noalloc(const double *W, const double *length, int32_t n_cells, double gamma, double gas_R,
                                 double Pref, double Tref, double cfl, double *dt, void *stream);

/* Point fluxes in the reference's rotated-frame signature
 * (roe_flux ns_roe.cc:25, AUSMplusUP_flux ns_ausm_plus_up.cc:35,
 * vanLeer_flux ns_vanleer.cc:25, SD_SLAU_flux ns_sd_slau.cc:37), flux
 * numbered as ns.h:48-53 (1 Roe, 2 Van Leer, 3 AUSM+up, 4 SD-SLAU).  The
 * Steger-Warming flux (5) needs the face's wall distance and dissipation
 * factor and is not offered here (FCFD_ERR_UNSUPPORTED); it runs inside the
 * residual.  L/R = (p,u,v,w,T) face states,
 * n = unit normal; out[5] = xyz flux per unit area (convective_face_flux
 * ns_convective_face_flux.cc:32-59 without the area factor).  Material is
 * given by gamma, R and the gauge offsets Pref/Tref. */
int fcfd_point_flux(int flux, const double *L, const double *R, const double *n, double gamma, double gas_R,
                    double Pref, double Tref, double Minf, double *out, double *weightL);

#ifdef __cplusplus
}
#endif
#endif /* FCFD_H */
