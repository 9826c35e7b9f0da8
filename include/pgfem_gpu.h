/*
 * pgfem_gpu.h -- C ABI of the B200 (sm_100a) element-assembly path.
 *
 * Drop-in replacement for PGFem3D's FP64 constitutive-model assembly: the
 * per-quadrature-point constitutive update, the element residual and the
 * consistent tangent of the 1-field total-Lagrangian element, scattered into
 * the CSR operator whose pattern Psparse_ApAi builds.  Reference paths are
 * relative to the PGFem3D source tree.
 *
 * Conventions (mirroring the reference):
 *  - every entry point returns int; 0 = success, negative = usage / CUDA
 *    error (PGFEM_GPU_E*), never a trap or abort;
 *  - element failures are counted, not raised: a pgfem_gpu_status holds the
 *    counts the reference accumulates into its `err` / INFO word
 *    (src/constitutive_model.cc:3443-3448 inverted elements,
 *    :2682-2687 non-normal stiffness diagonal, and local-solver
 *    non-convergence of the integration algorithm);
 *  - arrays are caller-owned; 3x3 tensors are row-major [9]; element vectors
 *    are node-major; element matrices use idx_K order
 *    (include/index_macros.h:25-26); DOF ids follow the reference: >0 free
 *    (1-based), 0 fixed, <0 prescribed (value u_presc[-id-1]);
 *  - one context per host thread; a context owns its CUDA stream, device
 *    copies of the mesh in structure-of-arrays form, the element->CSR map and
 *    the per-quadrature-point state at t_n and t_{n+1}.
 */
#ifndef PGFEM_GPU_H
#define PGFEM_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define PGFEM_GPU_OK 0
#define PGFEM_GPU_EINVAL (-1)   /* bad argument */
#define PGFEM_GPU_ECUDA (-2)    /* CUDA runtime error */
#define PGFEM_GPU_ENOMEM (-3)   /* device allocation failed */
#define PGFEM_GPU_EPATTERN (-4) /* CSR pattern does not hold an element block */
#define PGFEM_GPU_ENODEV (-5)   /* no usable sm_100 device */
#define PGFEM_GPU_ELIMIT (-6)   /* size beyond a fixed limit of the entry point */
#define PGFEM_GPU_ETIMEOUT (-7) /* a bounded device-side wait ran out (kernel returned early) */
#define PGFEM_GPU_EFORMAT (-8)  /* input file missing or malformed (pgfem_input_last_error says where) */

/* Constitutive models (the Model_parameters families on the path). */
enum {
  PGFEM_MODEL_HE = 0, /* HE_PARAM, src/plasticity_model_none.cc */
  PGFEM_MODEL_J2 = 1, /* CM_J2P_PARAM, src/cm_j2_plasticity.cc (damage off) */
  PGFEM_MODEL_CP = 2  /* CP_PARAM, src/plasticity_model.cc */
};

/* Doubles of per-quadrature-point state (one time level) in the host AoS
 * exchange format: HE 0; J2 10 = Cp^-1 (9) + eqps; CP 10 = pF (9) + g. */
int pgfem_gpu_state_size(int model);

/* Scatter modes:
 *  ATOMIC  FP64 atomic adds of every element entry (default);
 *  COLOUR  element colours with plain adds (deterministic summation order). */
enum { PGFEM_SCATTER_ATOMIC = 0, PGFEM_SCATTER_COLOUR = 1 };

typedef struct {
  int model;
  double E, nu;          /* isotropic elasticity (neo-Hookean: G = E/2(1+nu), kappa per src/hommat.cc:58-61) */
  double sigma_y, H;     /* J2: yield stress, linear isotropic hardening modulus */
  double gamma_dot_0, m; /* CP flow: gamma_dot = gamma_dot_0 sgn(tau) |tau/g|^(1/m) */
  double G0, g0, gs_0, gamma_dot_s, w; /* CP saturation hardening */
  double cp_tol;         /* CP local residual tolerance */
  int cp_max_iter;       /* CP local iteration cap */
  int dev_pot;           /* HE deviatoric potential, the reference's devPotFlag (src/new_potentials.cc:79-156):
                            0 or 1 Mooney-Rivlin with m01 = 0 (neo-Hookean, m10 = G/2); 2 linear,
                            S_dev = G (C - I) (devStress_Linear :364-375).  HE only; 2 runs the
                            per-node element kernel on every R/K path. */
  int vol_pot;           /* HE and J2 volumetric potential U(J), the reference's volPotFlag
                            (src/new_potentials.cc:185-300, 553-640): 99 (or <= 0) U_Common
                            0.5 (J-1)^2; 2 Doll-Schweizerhof 0.5 (exp(J-1) - ln J - 1); 3
                            Doll-Schweizerhof 0.5 (J-1) ln J.  Other values: PGFEM_GPU_EINVAL. */
} pgfem_material_desc;

typedef struct {
  long nn, ne;
  int nne;              /* 4 (linear tet, 1 qp) or 10 (quadratic tet, 4 qp) */
  const double *X;      /* nn*3 reference coordinates */
  const int *conn;      /* ne*nne node ids (0-based) */
  const long *dof_id;   /* nn*3 DOF ids (reference convention) */
  long ndof;            /* free DOFs = CSR rows */
  long npres;           /* prescribed values */
  const double *F0;     /* 9: macro deformation added to F (FE2, src/constitutive_model.cc:247-252) or NULL */
  const double *R_cp;   /* ne*9 crystal rotations (CP) or NULL */
} pgfem_mesh_desc;

typedef struct {
  long inverted;        /* J <= 0 at a quadrature point */
  long nonconverged;    /* local constitutive solver failed */
  long bad_diagonal;    /* non-normal stiffness diagonal */
  long other;
} pgfem_gpu_status;

typedef struct pgfem_gpu_ctx pgfem_gpu_ctx;

/* ---- setup (host) -------------------------------------------------------- */

/* generate_local_dof_ids (src/generate_dof_ids.cc:69-171, 306-412): on input
 * id[] holds codes (0 free, 1 fixed, <0 prescribed); on output the DOF ids.
 * Pr[n] = periodic master node or -1 (may be NULL).  Returns #free DOFs. */
long pgfem_generate_dof_ids(long nn, long ne, int nne, const int *conn, const long *Pr, long *id);

/* Psparse_ApAi (src/Psparse_ApAi.cc:238-670) for one rank: Ap[ndof+1] and
 * the sorted column ids Ai[nnz].  With Ai == NULL only Ap is filled.
 * Returns nnz (or a negative error). */
long pgfem_psparse_apai(long ne, int nne, const int *conn, const long *id, long ndof, int *Ap,
                        int *Ai);

/* Structured unit-cube mesh, n^3 cells of 6 tets each (nne 4 or 10); nodes
 * lexicographic on the vertex (nne 4) or half-cell (nne 10) lattice.  Call
 * with X == NULL to get the sizes.  Pr (may be NULL) receives the periodic
 * master of each node when periodic != 0, else -1. */
int pgfem_mesh_box_tet(int n, int nne, int periodic, long *nn, long *ne, double *X, int *conn,
                       long *Pr);

/* ---- context ------------------------------------------------------------- */

/* Builds the device copy and the element->CSR node-block map from the
 * caller's Ap/Ai (src/Psparse_ApAi.cc pattern) and validates it. */
int pgfem_gpu_create(const pgfem_mesh_desc *mesh, const pgfem_material_desc *mat, const int *Ap,
                     const int *Ai, long nrows, pgfem_gpu_ctx **ctx);
int pgfem_gpu_destroy(pgfem_gpu_ctx *ctx);
int pgfem_gpu_set_scatter_mode(pgfem_gpu_ctx *ctx, int mode);
/* Tests of the failure path (no counterpart in the reference): the bound of
 * the producer/consumer hand-off waits of the linear-tet R+K kernel (seconds,
 * default 2) and, with stall_next_assembly, the next such assembly's producer
 * warps withhold their first hand-off: the consumers' waits run out, every
 * warp leaves its loop (no trap), status.other counts it, and later calls are
 * unaffected. */
int pgfem_gpu_set_wait_test(pgfem_gpu_ctx *ctx, double limit_s, int stall_next_assembly);

/* ---- surface loads (Neumann boundary conditions) ------------------------
 * Replaces the NeumannBoundaryElement lists (include/PGFem3D_data_structure.h:
 * 32-120, built by construct_list_of_boundary_elements,
 * src/PGFem3D_data_structure.cc:825-895, from the NBC/<physics>.nbc features
 * read in src/read_input_file.cc:168-214) and their quasi-static terms
 * (compute_Neumann_boundary_conditions, src/fd_residuals.cc:123-273;
 * compute_Neumann_boundary_conditions_stiffnes_mat, src/stiffmat_fd.cc:
 * 359-500), which every residual and R+K call and the element-level calls
 * then add after the element integrals.
 * Face k: element elem[k] (0-based), local face face[k] (0..3, FEMLIB's
 * Tet2Tri numbering: {0,2,1}, {0,1,3}, {1,2,3}, {0,3,2}), feature feature[k].
 * Feature f: load_type[f] values (1: pressure p along the face's unit
 * normal, 2 or 3: traction components), load_np1[3f .. 3f+2] at t_{n+1} (the
 * host evaluates the load functions; unused entries are ignored).  nface = 0
 * clears.  Returns PGFEM_GPU_EINVAL for an element, face, feature or type out
 * of range.  set_neumann_loads replaces only the values (same nfeature). */
int pgfem_gpu_set_neumann(pgfem_gpu_ctx *ctx, long nface, const long *elem, const int *face,
                          const int *feature, int nfeature, const int *load_type, const double *load_np1);
int pgfem_gpu_set_neumann_loads(pgfem_gpu_ctx *ctx, int nfeature, const double *load_np1);
/* The same features' values at t_n and t_{n-1} (3 per feature), which the
 * transient call (pgfem_gpu_assemble_RK_transient) needs when faces are set:
 * it applies the surface loads at the two mid points, as the reference's
 * compute_Neumann_boundary_conditions(_stiffnes_mat) do with inertia
 * (src/fd_residuals.cc:123-273, src/stiffmat_fd.cc:359-500; the loads at the
 * three times from NBE compute_load_values, src/fd_residuals.cc:505-507). */
int pgfem_gpu_set_neumann_load_history(pgfem_gpu_ctx *ctx, int nfeature, const double *load_n,
                                       const double *load_nm1);

/* ---- three-field (CM3F) element -----------------------------------------
 * The constitutive-model element with one pressure P and one volume theta per
 * element (analysis type CM3F: get_3f_pressure_volume_number,
 * src/three_field_element.cc:1399-1409; the element loop of
 * src/constitutive_model.cc:695-881 with CM_ThreeField,
 * src/constitutive_model_3f.cc:185-491, and the static condensation
 * condense_K_3F_to_1F / condense_F_3F_to_1F, src/condense.cc:300-385), for
 * quadratic tets and the hyperelastic model -- and this library's J2 model,
 * whose isochoric return map is unchanged by the element's volume -- on the
 * default R+K path (atomic scatter), total Lagrangian, quasi-static.  set_three_field gives P and
 * theta per element (host arrays of ne, element order; theta > 0) and switches
 * every later R+K and residual call of the context to the condensed
 * three-field element; NULL, NULL switches back.  PGFEM_GPU_EINVAL for other
 * elements or models, and, while it is on, for the element-level calls.
 * get_three_field reads P and theta back.
 * three_field_increments: the local update after a displacement increment du
 * (free-DOF vector; compute_d_theta_dP, src/constitutive_model_3f.cc:494-549)
 * -- dP, d_theta per element from the blocks at u; the caller adds them.
 * three_field_update_device: the same on device buffers; with d_out NULL the
 * increments are added to the context's P and theta (what the device Newton
 * step, pgfem_gpu_newton_step, does after each solve while three-field is on),
 * else written to d_out (2 ne: dP, then d_theta). */
int pgfem_gpu_set_three_field(pgfem_gpu_ctx *ctx, const double *P, const double *theta);
int pgfem_gpu_get_three_field(pgfem_gpu_ctx *ctx, double *P, double *theta);
int pgfem_gpu_three_field_enabled(const pgfem_gpu_ctx *ctx);
int pgfem_gpu_three_field_increments(pgfem_gpu_ctx *ctx, const double *u, const double *u_presc,
                                     const double *du, double *dP, double *dtheta, pgfem_gpu_status *st);
int pgfem_gpu_three_field_update_device(pgfem_gpu_ctx *ctx, const double *d_u, const double *d_u_presc,
                                        const double *d_du, double *d_out, void *stream);
/* Three-field transient (hyperelastic; residuals_el_constitutive_model_w_inertia_3f
 * / stiffness_el_constitutive_model_w_inertia_3f, src/constitutive_model.cc:
 * 2190-2395, 2960-3229).  The context keeps P and theta at t_n and t_{n-1}
 * per element: set_three_field starts them at its values the first time,
 * set_three_field_history sets them, and commit_state moves t_n to t_{n-1}
 * and the current P, theta to t_n.  pgfem_gpu_assemble_RK_transient on a
 * three-field context (0 < alpha < 1) evaluates the newer mid point at
 * u_{n+alpha}, P = mid(P_n, P), theta = mid(theta_n, theta) and the older one
 * at u_{n-1+alpha}, mid(P_{n-1}, P_n), mid(theta_{n-1}, theta_n), combines the
 * residuals (R_u, R_p, R_t) with -dt_np1 (1 - alpha) and -dt_n alpha, the blocks
 * of the newer point with -dt_np1 alpha (1 - alpha), condenses, and adds the
 * inertia terms.  three_field_increments_transient: the local update after a
 * displacement increment du with those combined blocks (dP, d_theta per
 * element; the caller adds them). */
int pgfem_gpu_set_three_field_history(pgfem_gpu_ctx *ctx, const double *P_n, const double *theta_n,
                                      const double *P_nm1, const double *theta_nm1);
int pgfem_gpu_three_field_increments_transient(pgfem_gpu_ctx *ctx, const double *u_np1, const double *u_n,
                                               const double *u_nm1, const double *presc_np1,
                                               const double *presc_n, const double *presc_nm1, const double *du,
                                               double alpha, double dt_np1, double dt_n, double *dP,
                                               double *dtheta, pgfem_gpu_status *st);

/* Device bytes held by the context (mesh, map, state, scratch). */
long pgfem_gpu_device_bytes(const pgfem_gpu_ctx *ctx);
long pgfem_gpu_nnz(const pgfem_gpu_ctx *ctx);

/* ---- state (Model_parameters::set_init_vals / update_state_vars /
 *      reset_state_vars, src/constitutive_model.cc:1337-1497) ------------- */
int pgfem_gpu_set_state(pgfem_gpu_ctx *ctx, const double *state_n); /* AoS ne*nint*ns, host */
int pgfem_gpu_get_state(pgfem_gpu_ctx *ctx, int level, double *state); /* level 0: t_n, 1: t_{n+1},
                                                                          2: t_{n-1} (crystal plasticity) */
/* Crystal plasticity keeps the state at t_{n-1} too (get_pF(m, pF, 0), the
 * transient element's older mid point): set_state sets all three levels,
 * set_state_nm1 only t_{n-1} (AoS nqp*10; PGFEM_GPU_EINVAL for other models),
 * commit moves n to n-1 before n+1 to n, and a crystal-plasticity restart
 * file sets it from its pF_{n-1}, g_{n-1} fields. */
int pgfem_gpu_set_state_nm1(pgfem_gpu_ctx *ctx, const double *state_nm1);
int pgfem_gpu_commit_state(pgfem_gpu_ctx *ctx); /* (n-1 <- n,) n <- n+1 */
int pgfem_gpu_reset_state(pgfem_gpu_ctx *ctx);  /* n+1 <- n */

/* ---- assembly (host buffers; synchronous) --------------------------------
 * fd_residuals_MP (include/fd_residuals.h:39-51) and stiffmat_fd_MP
 * (include/stiffmat_fd.h:72-83) for one rank: R[ndof] and K[nnz] (aligned
 * with Ai) are overwritten; u is the free-DOF displacement (u_np1 + d_u),
 * u_presc the prescribed values (may be NULL when npres == 0).  The
 * constitutive update runs once and writes the state at t_{n+1}. */
int pgfem_gpu_assemble_R(pgfem_gpu_ctx *ctx, const double *u, const double *u_presc, double dt,
                         double *R, pgfem_gpu_status *st);
int pgfem_gpu_assemble_RK(pgfem_gpu_ctx *ctx, const double *u, const double *u_presc, double dt,
                          double *R, double *K, pgfem_gpu_status *st);

/* ---- assembly (device buffers; asynchronous on `stream`) -----------------
 * Same operation with device pointers; nothing is synchronised.  The failure
 * counts accumulate on the device until pgfem_gpu_read_status. */
int pgfem_gpu_assemble_RK_device(pgfem_gpu_ctx *ctx, const double *d_u, const double *d_u_presc,
                                 double dt, double *d_R, double *d_K, void *stream);
int pgfem_gpu_read_status(pgfem_gpu_ctx *ctx, pgfem_gpu_status *st, int clear);
/* Transient (inertia) element, mid-point rule: what fd_residuals_MP /
 * stiffmat_fd_MP compute when the material density exceeds 1e-16
 * (src/fd_residuals.cc:494-500, src/stiffmat_fd.cc:549-565; residual_with_inertia
 * / stiffness_with_inertia, src/dynamics.cc:183-432, with the CM parts of
 * src/constitutive_model.cc:1905-2170, 2803-2958).  Host buffers: free-DOF
 * displacements and prescribed values at t_{n+1}, t_n, t_{n-1}; alpha of the
 * mid-point rule (0..1), dt_np1 = t_{n+1} - t_n, dt_n = t_n - t_{n-1}, the
 * density rho.  Output R[ndof] and K[nnz] (K may be NULL):
 *   R = -dt_np1 (1 - alpha) R(u_{n+alpha}) - dt_n alpha R(u_{n-1+alpha}) - f_i
 *   K = -M / dt_np1 - alpha (1 - alpha) dt_np1 K(u_{n+alpha})
 * with R(u), K(u) the quasi-static element integrals, f_i the inertia force of
 * rho (dt_n u_{n+1} - (dt_np1 + dt_n) u_n + dt_np1 u_{n-1}) / (dt_np1 dt_n) and M
 * the consistent mass (rho N_A N_C) on the element's own quadrature rule.  With
 * |rho| < 1e-16 this is the quasi-static R, K at u_{n+1}, as in the reference.
 * Crystal plasticity (linear tets): the point update runs at u_{n+1} from the
 * state at t_n (the state at t_{n+1} is written, as by assemble_RK), and each
 * mid point takes the mid-point plastic part, pF = mid(pF_n, pF_{n+1}) and
 * mid(pF_{n-1}, pF_n) with the context's state at t_{n-1}, M = pF^-1 and the
 * factor det pF (residuals_el_constitutive_model_n_plus_alpha); K is the
 * derivative of that R in u_{n+1} through F and pF_{n+1}.  Surface loads at
 * the two mid points as pgfem_gpu_set_neumann_load_history sets them.
 * Hyperelastic (one- and three-field) and crystal-plasticity contexts
 * without macro deformation or mesh groups (PGFEM_GPU_EINVAL otherwise; the
 * three-field form below needs 0 < alpha < 1).  The
 * status counts inverted elements at both mid points. */
int pgfem_gpu_assemble_RK_transient(pgfem_gpu_ctx *ctx, const double *u_np1, const double *u_n,
                                    const double *u_nm1, const double *presc_np1, const double *presc_n,
                                    const double *presc_nm1, double alpha, double dt_np1, double dt_n, double rho,
                                    double *R, double *K, pgfem_gpu_status *st);
/* The same on device buffers (free-DOF displacements d_u_* [ndof], prescribed
 * values d_presc_* [npres], outputs d_R [ndof], d_K [nnz] or NULL), enqueued
 * on stream (a cudaStream_t; NULL is the default stream, as for
 * pgfem_gpu_assemble_RK_device); no copies, no synchronisation; the
 * status accumulates until pgfem_gpu_read_status clears it. */
int pgfem_gpu_assemble_RK_transient_device(pgfem_gpu_ctx *ctx, const double *d_u_np1, const double *d_u_n,
                                           const double *d_u_nm1, const double *d_presc_np1,
                                           const double *d_presc_n, const double *d_presc_nm1, double alpha,
                                           double dt_np1, double dt_n, double rho, double *d_R, double *d_K,
                                           void *stream);
/* Launch count of the kernels of one assemble_RK call (for accounting). */
int pgfem_gpu_launches_per_assembly(const pgfem_gpu_ctx *ctx);

/* ---- measurement ---------------------------------------------------------
 * With timing on, every assembly records CUDA events on its stream around
 * the element-assembly kernel launch(es) only.  pgfem_gpu_kernel_time
 * synchronises, returns the summed kernel time (ms) and the number of timed
 * calls since the last reset.  No counterpart in the reference (its CLOCK()
 * timers, src/Newton_Raphson.cc:419-439, wrap whole assemblies). */
int pgfem_gpu_set_timing(pgfem_gpu_ctx *ctx, int on);
int pgfem_gpu_kernel_time(pgfem_gpu_ctx *ctx, double *ms, long *ncalls, int reset);

/* FP64 FMA throughput of the current device (TFLOP/s), measured by an FMA
 * chain kernel over every SM; the FP64 roofline denominator.  No counterpart
 * in the reference. */
int pgfem_gpu_fp64_peak(double *tflops);

/* Compute capability the library's kernels were compiled for, as reported by
 * the CUDA runtime for one of them (major * 10 + minor: 100 for sm_100a).  No
 * counterpart in the reference. */
int pgfem_gpu_binary_version(int *version);

/* ---- crystal plasticity local solver -------------------------------------
 * Initial guess of the local Newton per quadrature point (host AoS nqp*10:
 * M0 = pF_n pF_{n+1}^-1 guess (9), g guess); NULL restores the elastic
 * predictor (M = I, g = g_n).  The plain solve always remains the fallback:
 * a point whose Newton from the guess fails is counted as non-converged.
 * No counterpart in the reference. */
int pgfem_gpu_set_cp_guess(pgfem_gpu_ctx *ctx, const double *guess);
/* Per-point local Newton iteration counts (nqp) and slip increments
 * dt*gamma_dot_a (nqp*12, may be NULL) of the last assembly. */
int pgfem_gpu_get_cp_iterations(pgfem_gpu_ctx *ctx, int *iters, double *dgam);

/* ---- element level (batched over an element list) -----------------------
 * stiffness_el_constitutive_model / residuals_el_constitutive_model
 * (include/constitutive_model.h:1003-1049), exported under the element
 * entry-point names of the dispatch they replace (stiffmatel_fd,
 * include/stiffmatel_fd.h:18-40; resid_on_elem, include/resid_on_elem.h:19-38).
 * lk: nel*(nne*3)^2 idx_K order; fe: nel*nne*3.  The state at t_{n+1} of the
 * listed elements is updated. */
int pgfem_gpu_stiffmatel_fd(pgfem_gpu_ctx *ctx, long nel, const long *elems, const double *u,
                            const double *u_presc, double dt, double *lk, double *fe,
                            pgfem_gpu_status *st);
int pgfem_gpu_resid_on_elem(pgfem_gpu_ctx *ctx, long nel, const long *elems, const double *u,
                            const double *u_presc, double dt, double *fe, pgfem_gpu_status *st);

/* ---- constitutive level ---------------------------------------------------
 * Model_parameters::integration_algorithm + update_elasticity
 * (include/constitutive_model.h:266-272, 242-757) batched over nqp points:
 * from F (nqp*9) and the state at t_n (nqp*ns, AoS) compute the state at
 * t_{n+1}, the PK2 stress S (nqp*9) and the material tangent L = 2 dS/dC
 * (nqp*81, idx_4 order; may be NULL).  R_cp: nqp*9 rotations (CP) or NULL.
 * qp_status (may be NULL): 0 ok, 1 inverted, 2 non-converged.  Host buffers. */
int pgfem_gpu_cm_integrate(const pgfem_material_desc *mat, long nqp, const double *F, double dt,
                           const double *R_cp, const double *state_n, double *state_np1,
                           double *S, double *L, int *qp_status);

/* ---- crystal plasticity point update that allocates nothing --------------
 * No counterpart in the reference.  For callers that must not call
 * cudaMalloc: code running under another framework's memory pool (the pool
 * owns the device memory, so a raw allocation bypasses it or fails), work on
 * a latency-critical path where cudaMalloc's implicit device-wide
 * synchronisation is unacceptable, and hosts that forbid allocation after
 * start-up.  The local Newton of the CP model (the same kernel the CP
 * assembly runs) for nqp <= 4096 points on caller-owned DEVICE buffers, all
 * component-major (SoA): d_F [9][nqp], d_R_cp [9][nqp] crystal rotations,
 * d_state_n / d_state_np1 [10][nqp] (pF 9, g), optional d_dgam [12][nqp]
 * slip increments dt*gamma_dot_a and d_iters [nqp] Newton iteration counts.
 * Asynchronous on `stream` unless st != NULL, in which case the call waits
 * for the stream and returns the failure counts (so st must be NULL while
 * the stream is being captured into a graph: PGFEM_GPU_EINVAL otherwise).
 * Its working memory (about 3.4 MB: per-point Newton record, ticket counter,
 * failure counters) is one fixed array in the library's device image, held
 * by every GPU that loads the library until the process exits; each call
 * zeroes the counters it needs.  Consequences:
 *  - nqp > 4096 returns PGFEM_GPU_ELIMIT (split larger batches);
 *  - calls that overlap on the GPU (different streams or host threads on the
 *    same device) share the array and race: order them on one stream;
 *  - the first call on each device performs a one-time set-up (looks up the
 *    array's device address, sets the kernel's shared-memory limit); make
 *    that first call before any stream capture;
 *  - the set-up is kept per device ordinal, for the device's primary context
 *    (the CUDA runtime's default): call it from threads that use the primary
 *    context, not from a driver-API context created with cuCtxCreate. */
int pgfem_gpu_cp_integrate_noalloc(const pgfem_material_desc *mat, long nqp, const double *d_F,
                                   const double *d_R_cp, const double *d_state_n, double dt,
                                   double *d_state_np1, double *d_dgam, int *d_iters,
                                   pgfem_gpu_status *st, void *stream);

/* ---- batches of independent meshes (FE2 micro-structures) ---------------
 * The context's mesh may be the union of independent meshes (e.g. the
 * periodic RVEs of all macro points, src/stiffmat_fd.cc:1010-1128 assembles
 * them one at a time): elements of group g are [elem_off[g], elem_off[g+1])
 * and see the macro deformation F0[9g..9g+8] (added to F like
 * cm_add_macro_F, src/constitutive_model.cc:247-252) instead of mesh->F0.
 * The CSR is block diagonal over the groups (one Psparse_ApAi pattern over
 * the union).  HE and J2. */
int pgfem_gpu_set_mesh_groups(pgfem_gpu_ctx *ctx, int ngroups, const long *elem_off, const double *F0);
/* Launch schedule of the linear-tet element kernel: elements per block
 * (16, 32, 64; 0 = default 32) and work stealing (grab > 0: a persistent
 * grid claims `grab` blocks of elements at a time from a counter; 0 = static
 * grid-stride order).  No counterpart in the reference. */
int pgfem_gpu_set_schedule(pgfem_gpu_ctx *ctx, int elems_per_block, int grab);
int pgfem_gpu_get_schedule(const pgfem_gpu_ctx *ctx, int *elems_per_block, int *grab);
/* One R+K assembly on device buffers captured as a CUDA graph (the
 * context's stream; the capture runs the assembly once uncaptured first).
 * Replays recompute R and K from the current contents of d_u / d_u_presc
 * and the context state.  No counterpart in the reference. */
typedef struct pgfem_gpu_graph pgfem_gpu_graph;
int pgfem_gpu_graph_create(pgfem_gpu_ctx *ctx, const double *d_u, const double *d_u_presc, double dt,
                           double *d_R, double *d_K, pgfem_gpu_graph **graph);
int pgfem_gpu_graph_launch(pgfem_gpu_graph *graph, void *stream);
int pgfem_gpu_graph_destroy(pgfem_gpu_graph *graph);
/* Times every schedule (3 block sizes x 5 steal sizes) as captured graphs,
 * `reps` replays each, keeps the fastest and reports it.  Linear tets. */
int pgfem_gpu_autotune(pgfem_gpu_ctx *ctx, const double *d_u, const double *d_u_presc, double dt, double *d_R,
                       double *d_K, int reps, int *best_elems_per_block, int *best_grab, double *best_ms);

/* ---- learned warm start of the CP local Newton ----------------------------
 * No counterpart in the reference (its Newton starts from the elastic
 * predictor, src/plasticity_model.cc:1148-1224).  A 34 -> 128 -> 128 -> 128
 * (GELU) -> 12 network maps per-point features to the slip increments
 * dt*gamma_dot_a; only the initial guess of the FP64 Newton is taken from it.
 * Features (row of 34 FP32): F_{n+1} F_n^-1 - I (9) and pF_n - I (9), both in
 * the lattice frame of the point's crystal (R^T A R), the 12 slip resistances
 * (g_n for every system of this model), lattice quaternion (4, w >= 0).  BF16 tensor-core (tcgen05) GEMMs, FP32 accumulation; trained on
 * the GPU by the library's own fused forward/backward kernel and Adam.
 * Parameter vector (FP32, 39,052): W1[128][34] b1 W2[128][128] b2 W3 b3
 * W4[12][128] b4.  Device pointers are marked d_. */
typedef struct pgfem_mlp pgfem_mlp;
typedef struct {
  int epochs, batch;        /* batch: samples per Adam step (>= 128) */
  float lr, lr_min;         /* cosine decay from lr to lr_min over all steps */
  float beta1, beta2, eps;  /* Adam */
  unsigned long long seed;  /* shuffling */
} pgfem_mlp_train_opts;
long pgfem_mlp_num_params(void);
int pgfem_mlp_create(unsigned long long seed, pgfem_mlp **m); /* Glorot-uniform weights, zero biases */
int pgfem_mlp_destroy(pgfem_mlp *m);
int pgfem_mlp_set_params(pgfem_mlp *m, const float *params);  /* host; resets the Adam moments */
int pgfem_mlp_get_params(const pgfem_mlp *m, float *params);
/* inputs are normalised as (x - x_mean) / x_std, outputs scaled by y_std */
int pgfem_mlp_set_scaling(pgfem_mlp *m, const float *x_mean, const float *x_std, const float *y_std);
int pgfem_mlp_get_scaling(const pgfem_mlp *m, float *x_mean, float *x_inv_std, float *y_std);
/* scaling from data: feature mean / standard deviation, target RMS */
int pgfem_mlp_fit_scaling(pgfem_mlp *m, long n, const float *d_x, const float *d_t);
int pgfem_mlp_predict_device(pgfem_mlp *m, long n, const float *d_x, float *d_y, void *stream);
/* Tests of the failure path (no counterpart in the reference): the bound of
 * the network kernels' tensor-core completion waits (seconds, default 2) and,
 * with stall_next_forward, the next forward pass withholds each CTA's first
 * MMA chain so that its wait runs out: the kernel returns early (TMEM released,
 * no trap) and the call reports PGFEM_GPU_ETIMEOUT; later calls are unaffected. */
int pgfem_mlp_set_wait_test(pgfem_mlp *m, double limit_s, int stall_next_forward);
int pgfem_mlp_predict(pgfem_mlp *m, long n, const float *x, float *y); /* host buffers */
/* loss 1/(2n) sum |out - t/y_std|^2 over all n rows and its gradient (host buffers) */
int pgfem_mlp_loss_grad(pgfem_mlp *m, long n, const float *x, const float *t, float *grad, double *loss);
/* Adam over shuffled mini-batches of the n pairs; epoch_loss[epochs] (may be NULL) */
int pgfem_mlp_train_device(pgfem_mlp *m, long n, const float *d_x, const float *d_t,
                           const pgfem_mlp_train_opts *opts, double *epoch_loss);

/* Newton iterations allowed from a guess (set_cp_guess or the network) before
 * the point restarts from the elastic predictor with the full cp_max_iter
 * budget; 0 (default) = cp_max_iter.  Iteration counts report both runs. */
int pgfem_gpu_set_cp_warm_limit(pgfem_gpu_ctx *ctx, int k);
/* Attach (m != NULL) or detach the network: each CP assembly then computes
 * the features on the device, runs the tcgen05 forward pass and starts the
 * FP64 Newton from the predicted slip (M0 = I - sum dgam_a P_a, g0 from the
 * hardening update).  The tolerance is unchanged; the cold start remains the
 * fallback.  The network must live on the context's device and outlive use. */
int pgfem_gpu_set_cp_surrogate(pgfem_gpu_ctx *ctx, pgfem_mlp *m);
/* Training pairs of the last assembly: features (d_x, nqp x 34) and the
 * converged slip increments (d_t, nqp x 12), device FP32 buffers. */
int pgfem_gpu_cp_training_pairs(pgfem_gpu_ctx *ctx, float *d_x, float *d_t);
/* Points of the last assembly that fell back to the cold start. */
int pgfem_gpu_get_cp_fallbacks(pgfem_gpu_ctx *ctx, long *n);

/* ---- linear solve and Newton-Raphson on the device ------------------------
 * The consumer of K.  The reference solves K dd_u = f with hypre
 * (src/solvers/hypre/Hypre.cc:147-194): GMRES (src/solvers/hypre/GMRes.cc, the
 * default) or BiCGSTAB (src/solvers/hypre/BCGStab.cc), preconditioned by
 * diagonal scaling (src/solvers/hypre/ScaleDiag.cc: 1/K_ii, 1.1 where
 * |K_ii| <= 1e-5), inside its Newton-Raphson loop
 * (src/Newton_Raphson.cc:931-1330).  A solver holds the CSR pattern on the
 * device (Ap, Ai of one rank, columns sorted, column id = row id on the
 * diagonal) and its Krylov work vectors; K values are passed per call.
 * Solver and preconditioner ids keep the values of the reference's
 * enumerations (include/enumerations.h:35-45, 87-94). */
enum { PGFEM_SOLVER_GMRES = 0, PGFEM_SOLVER_BCG_STAB = 1 };      /* SOLVER_GMRES, SOLVER_BCG_STAB */
enum { PGFEM_PRECOND_NONE = 4, PGFEM_PRECOND_DIAG_SCALE = 5 };  /* PRECOND_NONE, PRECOND_DIAG_SCALE */
#define PGFEM_GMRES_MAX_KDIM 1000 /* largest Krylov dimension of a GMRES solver (ELIMIT beyond) */

typedef struct {
  int solver;      /* PGFEM_SOLVER_GMRES or PGFEM_SOLVER_BCG_STAB */
  int precond;     /* PGFEM_PRECOND_NONE or PGFEM_PRECOND_DIAG_SCALE */
  int maxit;       /* iteration cap (the reference's -maxit, default 1000) */
  int kdim;        /* GMRES restart length (-kdim, default 500); the basis takes (kdim + 1) * nrows doubles */
  double tol;      /* relative residual ||b - K x|| / ||b|| to reach (sol->err) */
  int check_every; /* iterations queued between host convergence checks; <= 0: 8 */
} pgfem_solver_opts;

typedef struct {
  int iters;       /* iterations (GMRES: Arnoldi steps over all cycles; SOLVER_INFO n_iter) */
  double res_norm; /* final relative residual (GMRES: ||b - K x|| / ||b|| recomputed; BiCGSTAB: of the
                      recurrence) (SOLVER_INFO res_norm) */
  int converged;   /* the method's residual reached tol */
  int breakdown;   /* a denominator vanished or a value was not finite */
} pgfem_solve_info;

typedef struct pgfem_gpu_solver pgfem_gpu_solver;

/* Copies the pattern to the device and allocates the work vectors; EPATTERN
 * when a column id is out of range, ELIMIT for kdim > PGFEM_GMRES_MAX_KDIM,
 * ENODEV without an sm_100 device. */
int pgfem_gpu_solver_create(const int *Ap, const int *Ai, long nrows, const pgfem_solver_opts *opts,
                            pgfem_gpu_solver **solver);
int pgfem_gpu_solver_destroy(pgfem_gpu_solver *solver);
long pgfem_gpu_solver_device_bytes(const pgfem_gpu_solver *solver);
/* y = K x on `stream` (device pointers; asynchronous). */
int pgfem_gpu_spmv(pgfem_gpu_solver *solver, const double *d_K, const double *d_x, double *d_y, void *stream);
/* K x = b by the solver's method; d_x holds the initial guess on entry.
 * Synchronises `stream` at each convergence check. */
int pgfem_gpu_solve(pgfem_gpu_solver *solver, const double *d_K, const double *d_b, double *d_x,
                    pgfem_solve_info *info, void *stream);

#define PGFEM_NEWTON_HISTORY 32
typedef struct {
  int iter_max;         /* Newton iteration cap (sol->iter_max) */
  double nor_min;       /* converged when ||R|| / ||R_0|| <= nor_min (sol->nor_min) */
  double computer_zero; /* ... or when ||R|| <= computer_zero (sol->computer_zero) */
} pgfem_newton_opts;

typedef struct {
  int iters;          /* Newton iterations (solves) taken */
  int converged;
  int lin_iters;      /* BiCGSTAB iterations summed over the solves */
  int lin_failed;     /* a linear solve missed its tolerance */
  long elem_failures; /* element/point failures reported by the assemblies */
  double nor, nor2;   /* last ||R|| / ||R_0|| and ||R|| */
  double nor_hist[PGFEM_NEWTON_HISTORY]; /* ||R|| / ||R_0|| per iteration */
} pgfem_newton_info;

/* One load step of full Newton-Raphson (stiffness every iteration, no line
 * search): from the free-DOF displacement d_u (updated in place) and the
 * prescribed values of the step, assemble R and K on the device
 * (pgfem_gpu_assemble_RK_device), solve K du = -R with the solver, u += du,
 * until the reference's test nor = ||R|| / ||R_0|| <= nor_min or
 * ||R|| <= computer_zero (src/Newton_Raphson.cc:1203-1217, 1323).  The state
 * at t_{n+1} in the context is the one of the last assembly: commit it with
 * pgfem_gpu_commit_state after a converged step.  Returns a negative code
 * on usage/CUDA errors; non-convergence is reported in info. */
int pgfem_gpu_newton_step(pgfem_gpu_ctx *ctx, pgfem_gpu_solver *solver, double *d_u, const double *d_u_presc,
                          double dt, const pgfem_newton_opts *opts, pgfem_newton_info *info, void *stream);

/* ---- input files (host only) ----------------------------------------------
 * Readers of PGFem3D's own input files, so that the reference's inputs drive
 * this library: mesh files <base><r>.in of read_input_file
 * (src/read_input_file.cc:268-415, non-legacy formats), solver files
 * (read_solver_file, :556-700), model_params.in (read_model_parameters_list,
 * src/constitutive_model.cc:1171-1309) and crystal orientation files
 * (plasticity_model_read_orientations, src/plasticity_model.cc:1260-1337).
 * Errors: PGFEM_GPU_EFORMAT with a message from pgfem_input_last_error(). */
const char *pgfem_input_last_error(void);

typedef struct pgfem_input pgfem_input;
typedef struct {
  long nn, ne;          /* merged mesh */
  int nne;              /* 4 or 10 (one element type per mesh) */
  long npres;           /* prescribed values (support code -k takes defl[k-1]) */
  int nmat;             /* material lines */
  long nconc, norient;  /* material geometry sizes */
  long lin_maxit;       /* header line 2: linear solver iterations, tolerance, zero */
  double lin_err, lim_zero;
  long nln, nel_s, nel_v; /* nodal / surface / volume load counts (not applied on this path) */
  long nperiodic;       /* nodes that are periodic images of another (pgfem_input_get_periodic) */
} pgfem_input_info;

/* Reads <base><r>.in for r = 0..nparts-1 and merges the partitions into one
 * mesh: a partition-boundary node (Gnn >= 0) is one node whichever files list
 * it at the same position, an interior node (Gnn = -1) belongs to its file;
 * nodes that share a global number at different positions are periodic
 * images (periodic micro-structures), kept as nodes of their own and linked to
 * the first image (pgfem_input_get_periodic).  Nodes are numbered in order of
 * first appearance (partition, then local id), elements partition by
 * partition.  Partitions must agree on supports, prescribed values and
 * materials.  The supports come from the mesh files. */
int pgfem_input_read_mesh(const char *base, int nparts, pgfem_input **out);
/* The same with the supports and prescribed values of a BC directory
 * (src/read_input_file.cc:320-360): <bc_base>_<r>.bc per partition and
 * <bc_base>.bcv (e.g. bc_base = "<input dir>/BC/Mechanical"); the mesh files'
 * own supports sections are read and ignored, as the reference does. */
int pgfem_input_read_mesh_bc(const char *base, int nparts, const char *bc_base, pgfem_input **out);
/* Multiphysics meshes: one supports section per physics in the order of
 * multiphysics.in, ndim[k] codes per node (1 heat transfer, 3 mechanics);
 * section `mech` (ndim 3) is kept.  With bc_base the mesh file holds a single
 * supports section, which the BC directory's files replace (the reference's
 * layout, src/read_input_file.cc:320-360). */
int pgfem_input_read_mesh_mp(const char *base, int nparts, const char *bc_base, int nphys, const int *ndim,
                             int mech, pgfem_input **out);
/* multiphysics.in (read_multiphysics_settings, src/PGFem3D_data_structure.cc:
 * 680-780): per physics in file order its id (0 mechanical, 1 thermal) and
 * degrees of freedom per node; n = number of physics. */
int pgfem_input_read_multiphysics(const char *path, int max_phys, int *ids, int *ndim, int *n);
int pgfem_input_get_info(const pgfem_input *in, pgfem_input_info *info);
/* X[nn*3], conn[ne*nne] (0-based merged ids), codes[nn*3] support codes
 * (0 free, 1 fixed, -k prescribed: the pgfem_generate_dof_ids input),
 * defl[npres]. */
int pgfem_input_get_mesh(const pgfem_input *in, double *X, int *conn, long *codes, double *defl);
/* Per element (each may be NULL): mat[ne*2], hom[ne*2] (matrix, fibre),
 * partition and id within the partition. */
int pgfem_input_get_elements(const pgfem_input *in, long *mat, long *hom, int *part, long *local_id);
/* vals[nmat*13] = Ex Ey Ez Gyz Gxz Gxy nyz nxz nxy ax ay az sig, and the
 * potential flags (devPotFlag, volPotFlag) per material. */
int pgfem_input_get_materials(const pgfem_input *in, double *vals, int *dev_pot, int *vol_pot);
/* Crystal orientations <base>_<r>.in (one per partition): angles[ne*3]
 * (phi, theta, psi) per merged element, NAN where no line sets one; a line
 * with a negative element id sets every element of material `ip` of its
 * partition.  euler_type: the file's "# EulerAngleType: k" (0 if absent). */
int pgfem_input_read_orientations(const pgfem_input *in, const char *base, double *angles, int *euler_type);
/* Partition `part` of the merged mesh: its node and element counts and the
 * merged id of each of its local nodes (node_map[nn], may be NULL); its
 * elements are the merged elements [sum of earlier ne, + ne).  This is what
 * maps per-rank files (restart files, outputs) onto the merged mesh. */
int pgfem_input_get_partition(const pgfem_input *in, int part, long *nn, long *ne, long *node_map);
/* Pr[nn]: periodic master of each node or -1 (the pgfem_generate_dof_ids Pr input). */
int pgfem_input_get_periodic(const pgfem_input *in, long *Pr);
/* The boundary feature of each element face, read from the element lines
 * (bnd_type[4], bnd_id[4], src/element.cc:168-199): bnd_type[ne*4] and
 * bnd_id[ne*4] (each may be NULL), merged element order, local faces 0..3. */
int pgfem_input_get_element_faces(const pgfem_input *in, int *bnd_type, int *bnd_id);
void pgfem_input_destroy(pgfem_input *in);

/* Surface-load files: <ipath>/NBC/<physics>.nbc (read_Neumann_boundary_conditions,
 * src/read_input_file.cc:168-214): a feature count, then per feature its
 * type, id, number of load values (1 pressure, 2..3 traction) and one file
 * name per value, whose first line is the load as an expression of time t
 * (read_loads, src/PGFem3D_data_structure.cc:934-948).  A missing directory
 * or file means no surface loads (an empty set, as in the reference).  The
 * reference evaluates the expressions with the exprtk library
 * (string_function_of_time, src/utils.cc:3423-3440); this library evaluates
 * the arithmetic subset pgfem_load_expression documents and rejects the rest
 * (EFORMAT).  A feature listed twice is rejected too: the reference would
 * then load face 0 of the element with feature 0 (its list has more rows
 * than flagged faces, src/PGFem3D_data_structure.cc:870-891). */
typedef struct pgfem_nbc pgfem_nbc;
int pgfem_input_read_nbc(const char *ipath, const char *physics, pgfem_nbc **out);
/* Feature count and, per feature (arrays may be NULL), type, id, load type. */
int pgfem_nbc_get_features(const pgfem_nbc *nbc, int *nfeature, int *ftype, int *fid, int *load_type);
/* The loaded faces of the mesh (construct_list_of_boundary_elements,
 * src/PGFem3D_data_structure.cc:825-895): every element face whose
 * (bnd_type, bnd_id) is a feature's (type, id), in element then face order;
 * nface receives the count (elem/face/feature may be NULL to count first).
 * The arrays are pgfem_gpu_set_neumann's. */
int pgfem_nbc_faces(const pgfem_nbc *nbc, const pgfem_input *in, long *nface, long *elem, int *face, int *feature);
/* The features' load values at time t (compute_load_values,
 * src/PGFem3D_data_structure.cc:956-972): load[nfeature*3], entries past a
 * feature's load type 0; pgfem_gpu_set_neumann_loads' input. */
int pgfem_nbc_load_values(const pgfem_nbc *nbc, double t, double *load);
void pgfem_nbc_destroy(pgfem_nbc *nbc);
/* One load expression at time t (names case-insensitive, comments # and //
 * to the end of the line and slash-star blocks skipped): numbers, t, pi,
 * epsilon, inf, true, false;
 * + - * / % ^ (right associative, above unary minus), comparisons (< <= > >=
 * == = != <>), and / or / not (also && || & |), c ? a : b; functions if(c,a,b),
 * min, max (1 or more arguments), clamp(lo,x,hi), pow, atan2, hypot, mod, abs,
 * sgn, sqrt, exp, log, log10, log2, floor, ceil, round, trunc, frac, sin, cos,
 * tan, asin, acos, atan, sinh, cosh, tanh; an optional trailing ';'. */
int pgfem_load_expression(const char *expr, double t, double *value);
/* R = Az(psi) Ay(theta) Ax(phi), right-handed rotations about the axes (the
 * composition the reference states at src/plasticity_model.cc:1252-1255; its
 * rotation_matrix_of_Euler_angles lives in an absent library).  With this R
 * the reference's crystal plasticity tension case (EulerAngleType 0)
 * reproduces its own restart output; the transpose does not.  Other
 * EulerAngleType values select conventions of that library that no reference
 * output pins; callers check the type pgfem_input_read_orientations returns. */
int pgfem_euler_rotation(long n, const double *angles, double *R);

typedef struct {
  double nor_min;        /* Newton tolerance */
  long iter_max, npres, FNR;
  double dAL0, dALMAX;   /* arc length (FNR 2, 3) */
  int physicsno, max_NR_staggering, max_subdivision; /* FNR 4 */
  long nt;               /* time steps: times[nt+1] */
  long n_print;          /* output steps */
  long n_load;           /* steps with a load increment */
  long n_incr;           /* increments per load step (npd, or npres when npd < 0) */
} pgfem_solver_file;
/* Reads a solver file; arrays may be NULL (call once with NULL for the
 * sizes): times[nt+1], print_steps[n_print], load_steps[n_load],
 * load_incr[n_load*n_incr], the prescribed-value increments the reference
 * reads while stepping, one per prescribed value of the mesh: pass the
 * mesh's npres as npd (the header's npres is a different count).  A file that
 * ends after the output steps has its load history in a load directory, which
 * is not read (n_load = 0). */
int pgfem_input_read_solver_file(const char *path, long npd, pgfem_solver_file *sf, double *times,
                                 long *print_steps, long *load_steps, double *load_incr);

/* ---- restart files --------------------------------------------------------
 * One rank's restart file in the reference's layout (write_restart_constitutive_model /
 * read_restart_constitutive_model, src/restart.cc:187-300): per node the pairs
 * "u_nm1 u_n" of x, y, z (total displacements, prescribed values included),
 * then per element its point count and per point the model block of
 * write_restart: HE (src/plasticity_model_none.cc:298-311) Fn, Fnm1 = 18
 * doubles; CP (src/plasticity_model.cc:883-942) Fn, Fnm1, pFn, pFnm1,
 * tau_n[12], gamma_dot_n[12], g_n, g_nm1, L_n, L_nm1 = 64 doubles; J2
 * (src/cm_j2_plasticity.cc:784-808) Fn, pSn, Fnm1, pSnm1, w, X, H, ep_n, ep_nm1,
 * gam_n, gam_nm1, the damage flag = 47 doubles.  File name convention of the reference:
 * <dir>/STEP_<step %06d>/<name>_<rank>_<step>.res. */
int pgfem_restart_block_size(int model);
/* Host-only formatting / parsing: u_nm1, u_n nodal AoS (nn*3), blocks
 * (ne*n_ip*block_size).  The parser rejects a file whose node, element or
 * point counts do not match (EFORMAT). */
int pgfem_restart_format(const char *path, long nn, long ne, int n_ip, int model, const double *u_nm1,
                         const double *u_n, const double *blocks);
int pgfem_restart_parse(const char *path, long nn, long ne, int n_ip, int model, double *u_nm1, double *u_n,
                        double *blocks);
/* One file per partition of a merged mesh, as the reference's ranks write
 * them: <name>_<r>_<step>.res with the partition's nodes (its node map) and
 * elements, from merged nodal u_nm1, u_n (nn*3) and blocks (ne*n_ip*block). */
int pgfem_restart_write_partitions(const pgfem_input *in, const char *name, int step, int model, int n_ip,
                                   const double *u_nm1, const double *u_n, const double *blocks);
/* Context level.  Write: u_nm1, u_n free-DOF displacements at t_{n-1}, t_n
 * with their prescribed values; F per point is computed from them on the
 * device; CP pFn, g_n from the committed state (t_n) and pFnm1, g_nm1 from
 * state_nm1 (host AoS nqp*10 as pgfem_gpu_get_state, the state before the
 * last commit; NULL = the state at t_n); tau_n and gamma_dot_n from F_n, pF_n
 * and g_n (pgfem_cp_resolved_shear); L_n, L_nm1 (a multiplier of the
 * reference's integrator) written as 0.  J2: the plastic stress of
 * the reference's block is pS = G (I - Cp^-1) of this path's state (zero in
 * the initial state, as the reference initialises it), ep_n / ep_nm1 the
 * equivalent plastic strain, gam_n = sqrt(3/2) (ep_n - ep_nm1), the damage
 * variables w, X, H, gam_nm1 and the damage flag 0 (damage is not carried).
 * Read: returns the free-DOF displacements u_nm1, u_n (the caller's vectors)
 * and sets the state at t_n from the file (CP: pFn, g_n and F at t_n; J2:
 * Cp^-1 = I - pSn / G and ep_n); the other fields are not used. */
int pgfem_gpu_write_restart(pgfem_gpu_ctx *ctx, const char *path, const double *u_nm1, const double *u_n,
                            const double *presc_nm1, const double *presc_n, const double *state_nm1);
/* Host: the crystal plasticity restart fields tau_n and gamma_dot_n of n
 * points from F (n*9), pF (n*9), g (n) and the crystal rotation R (n*9), all
 * row-major: tau = s . (Ce S) n per slip system at Ce = pF^-T F^T F pF^-1 and
 * gamma_dot = gamma_dot_0 (tau/g) |tau/g|^(1/m - 1), written (n*12 each) in the
 * order and sign of the systems in the reference's restart files (the order of
 * its integrator, taken from its own output: every element of its crystal
 * plasticity tension case).  gdot may be NULL. */
int pgfem_cp_resolved_shear(const pgfem_material_desc *mat, long n, const double *F, const double *pF,
                            const double *g, const double *R, double *tau, double *gdot);
int pgfem_gpu_read_restart(pgfem_gpu_ctx *ctx, const char *path, double *u_nm1, double *u_n);

/* model_type values of model_params.in (include/constitutive_model.h:42-54) */
enum {
  PGFEM_CM_HYPER_ELASTICITY = 0,
  PGFEM_CM_CRYSTAL_PLASTICITY = 1,
  PGFEM_CM_BPA_PLASTICITY = 2,
  PGFEM_CM_ISO_VISCOUS_DAMAGE = 3,
  PGFEM_CM_J2_PLASTICITY_DAMAGE = 4,
  PGFEM_CM_UQCM = 100
};
typedef struct {
  int mat_id, model_type, uq;
  int np;                 /* parameters in p: CP 7 (gamma_dot_0 m G0 g0 gs_0 gamma_dot_s w);
                             J2 14 (beta hp k0, mu w_max P1 P2 Yin, da db_p db_m va vb_p vb_m) */
  double p[16];
  int unit_cell;          /* CP slip system */
  int ort_option[3];      /* CP orientation option (2: from files ort_file_<r>.in; 3: ort_angles) */
  char ort_file[256];
  double ort_angles[3];
  int solver_set;         /* CP local solver block present */
  int max_itr_stag, max_itr_hardening, max_itr_M, max_subdivision;
  double tol_hardening, tol_M, computer_zero;
} pgfem_model_params;
/* Reads up to max_entries entries (n = entries in the file). */
int pgfem_input_read_model_params(const char *path, int max_entries, pgfem_model_params *out, int *n);
/* Material of a J2 entry (CM_J2P_PARAM::read_param, src/cm_j2_plasticity.cc:
 * 865-932): E, nu and vol_pot (volPotFlag) from the mesh file's material line,
 * sigma_y = k0 and H = hp from the entry (yield function ||dev tau|| -
 * sqrt(2/3) (k0 + hp ep), linear isotropic hardening).  Returns
 * PGFEM_GPU_EINVAL for beta != 0 (only the reference driver's beta = 0 is
 * carried) and for active damage (mu != 0); the damage parameters are
 * otherwise unused (damage off). */
int pgfem_input_j2_material(const pgfem_model_params *mp, double E, double nu, int vol_pot,
                            pgfem_material_desc *out);

#ifdef __cplusplus
}
#endif
#endif
