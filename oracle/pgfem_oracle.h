/*
 * pgfem_oracle.h -- CPU oracle for the PGFem3D element-assembly hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates, on the CPU and in plain
 * C++, the reference algorithms that the GPU product replaces.  It is used by
 * tests/, by __graft_entry__.smoke() and by the cpu_baseline / reference arm
 * of bench.py as the checker and as the timed CPU baseline.  The product path
 * (pgfem-3d_b200/) never links, loads or calls it.
 *
 * Parity status: the in-tree parts (FEMLIB shape functions and quadrature,
 * the constitutive-model element integrals, DOF numbering, the CSR pattern,
 * the Mooney-Rivlin / U_Common potentials, the crystal-plasticity flow and
 * hardening laws) follow the reference line by line and are pinned by the
 * reference's own structure and by known-answer tests.  The J2 return map and
 * the crystal-plasticity local solver of the reference live in an external
 * library that is absent from the reference tree, so those two are
 * restatements of the published algorithms: parity against the reference is
 * unpinned for them (see the per-function comments).
 */
#ifndef PGFEM_ORACLE_H
#define PGFEM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_MODEL_HE = 0, ORC_MODEL_J2 = 1, ORC_MODEL_CP = 2 };

/* Number of doubles of per-quadrature-point state for each model (one time
 * level).  HE: none.  J2: Cp^{-1} (9, row-major) + eqps (1).
 * CP: pFn (9) + slip resistance g_n (1). */
int orc_state_size(int model);

typedef struct {
  int model;
  double E, nu;                 /* isotropic elasticity */
  double sigma_y, H;            /* J2: initial yield stress, linear isotropic hardening */
  /* CP power-law flow + saturation hardening */
  double gamma_dot_0, m, G0, g0, gs_0, gamma_dot_s, w;
  double cp_tol;                /* local-Newton residual tolerance */
  int cp_max_iter;              /* local-Newton iteration cap */
  int dev_pot;                  /* deviatoric potential flag of src/new_potentials.cc:79-156:
                                   1 (or 0) Mooney-Rivlin with m10 = G/2, m01 = 0 (neo-Hookean),
                                   2 Linear (S_dev = G (C - I)) */
  int vol_pot;                  /* volumetric potential flag (src/new_potentials.cc:185-300, 553-640):
                                   99 (or <= 0) U_Common, 2 / 3 Doll-Schweizerhof; HE and J2 */
} orc_material;

typedef struct {
  long nn, ne;
  int nne;                      /* 4 (linear tet) or 10 (quadratic tet) */
  const double *X;              /* nn*3 reference coordinates, node-major */
  const int *conn;              /* ne*nne node ids, element-major */
  const long *id;               /* nn*3 DOF ids: >0 free (1-based), 0 fixed, <0 prescribed */
  long ndof;                    /* number of free DOFs */
  const int *Ap, *Ai;           /* CSR pattern of the free DOFs (0-based) */
  const double *F0;             /* macro deformation-gradient increment added to F (FE2), or NULL */
  const double *R_cp;           /* CP: ne*9 crystal rotation per element (row-major), or NULL */
  /* Neumann faces (surface loads), or nbc_off == NULL for none: the faces of
   * element e are k = nbc_off[e] .. nbc_off[e+1]-1, each with its local face
   * nbc_face[k] (0..3, FEMLIB's Tet2Tri numbering), the number of load values
   * nbc_type[k] (1: pressure along the face normal, 2 or 3: traction) and the
   * values at t_{n+1} nbc_load[3k .. 3k+2].  Added to the element's residual and
   * stiffness after the element integrals (src/fd_residuals.cc:123-273,
   * src/stiffmat_fd.cc:359-500). */
  const long *nbc_off;
  const int *nbc_face;
  const int *nbc_type;
  const double *nbc_load;
  /* the same faces' values at t_n and t_{n-1} (3k .. 3k+2), read by the
   * transient element only (may be NULL otherwise) */
  const double *nbc_load_n;
  const double *nbc_load_nm1;
} orc_problem;

/* Reference: src/generate_dof_ids.cc:69-171 (generate_local_dof_ids) and
 * :306-412 (generate_local_dof_ids_on_elem).  id[] holds the input codes
 * (0 free, 1 fixed, <0 prescribed) and receives the DOF ids.  Pr[n] is the
 * periodic master node of n or -1.  Returns the number of free DOFs. */
long orc_generate_dof_ids(long nn, long ne, int nne, const int *conn,
                          const long *Pr, long *id);

/* Reference: src/Psparse_ApAi.cc:161-213 (countDof/mapDof), :327-366 (row
 * sort + dedupe), :639-658 (Ap prefix, Ai).  Single rank.  With Ai == NULL
 * only Ap is filled and nnz is returned. */
long orc_psparse_apai(long ne, int nne, const int *conn, const long *id,
                      long ndof, int *Ap, int *Ai);

/* One constitutive update at one quadrature point, the equivalent of
 * run_integration_algorithm followed by update_elasticity
 * (src/constitutive_model.cc:1100-1129, 1139-1164).  Outputs the PK2 stress
 * S (9) and the material tangent L = 2 dS/dC (81, idx_4 order) at the
 * elastic deformation, and the state at n+1.  For CP it also returns pF_{n+1}
 * (9) in pFnp1 and dM/du support data is handled inside orc_element.
 * Returns a non-zero error count on failure. */
int orc_cm_update(const orc_material *mat, const double *F, double dt,
                  const double *Rcp, const double *state_n,
                  double *state_np1, double *S, double *L, int *iters);

/* Element residual fe (nne*3) and stiffness lk ((nne*3)^2, idx_K order) of
 * element e through the constitutive-model 1-field path
 * (src/constitutive_model.cc:3322-3539, 2474-2692, 1520-1662).  u_e is the
 * element displacement (nne*3, node-major), state_n/state_np1 point at the
 * element's nint state records.  lk may be NULL. */
int orc_element(const orc_problem *P, const orc_material *mat, long e,
                const double *u_e, double dt, const double *state_n,
                double *state_np1, double *fe, double *lk);

/* Global assembly: R (ndof) and K values (nnz, aligned with Ai), the
 * equivalent of fd_residuals_MP + stiffmat_fd_MP on one rank
 * (src/fd_residuals.cc:468-636, 58-73; src/stiffmat_fd.cc:831-993;
 * src/PLoc_Sparse.cc:15-175).  u is the free-DOF displacement vector,
 * u_presc the prescribed values (indexed by -id-1, may be NULL).  Elements
 * [e0, e1) only; R and K are accumulated (caller zeroes them).  K may be NULL.
 * nthreads > 1 runs element colours in parallel (deterministic per colour).
 * iter_hist (may be NULL) receives per-qp local-iteration counts (CP). */
int orc_assemble(const orc_problem *P, const orc_material *mat,
                 const double *u, const double *u_presc, double dt,
                 const double *state_n, double *state_np1, double *R,
                 double *K, long e0, long e1, int nthreads, int *iters);

/* Three-field (CM3F) element of the hyperelastic and J2 models (one pressure
 * and one volume per element, condensed; J2 state per point at t_n in, t_{n+1}
 * out, as in orc_element): element residual/stiffness at (u_e, P,
 * theta); blk (may be NULL) receives fp, ft, Ktp, Ktt, Kup[3 nne]. */
int orc_element_3f(const orc_problem *P, const orc_material *mat, long e, const double *u_e,
                   double Pe, double theta, const double *state_n, double *state_np1, double *fe,
                   double *lk, double *blk);
/* Its global assembly (R, K accumulated; K may be NULL), and the element
 * pressure / volume increments after a displacement increment du. */
int orc_assemble_3f(const orc_problem *P, const orc_material *mat, const double *u,
                    const double *u_presc, const double *Pe, const double *theta, const double *state_n,
                    double *state_np1, double *R, double *K);
int orc_update_3f(const orc_problem *P, const orc_material *mat, const double *u, const double *u_presc,
                  const double *du, const double *Pe, const double *theta, const double *state_n,
                  double *dP, double *dtheta);

/* Same element integrals in the algebraically identical B-matrix form (the
 * "best CPU algorithm" baseline).  Same arguments as orc_assemble. */
int orc_assemble_bform(const orc_problem *P, const orc_material *mat,
                       const double *u, const double *u_presc, double dt,
                       const double *state_n, double *state_np1, double *R,
                       double *K, long e0, long e1, int nthreads);

/* Crystal-plasticity point updates over nqp points: F (nqp*9), rotations
 * Rcp (nqp*9), state at t_n (nqp*10: pF_n 9, g_n).  M0/g_guess (may be NULL)
 * give the Newton's initial guess per point (NULL: elastic predictor).
 * Outputs the state at t_{n+1} (nqp*10), the iteration counts, the slip
 * increments dt*gamma_dot_a (nqp*12, may be NULL) and a convergence flag.
 * With a guess, the Newton gets warm_k iterations from it (0: cp_max_iter)
 * before restarting from the elastic predictor; fallback[q] (may be NULL)
 * flags those restarts and iters counts both runs.
 * Returns the number of points that failed. */
long orc_cp_update_batch(const orc_material *mat, long nqp, const double *F, double dt, const double *Rcp,
                         const double *state_n, const double *M0, const double *g_guess,
                         double *state_np1, int *iters, double *dgam, int *converged, int warm_k,
                         int *fallback);

/* Transient (inertia, mid-point rule) R and K of the hyperelastic 1-field
 * element (residual_with_inertia / stiffness_with_inertia,
 * src/dynamics.cc:183-432, with the CM parts of src/constitutive_model.cc:
 * 1905-2170, 2803-2958), which the reference runs when the density exceeds
 * 1e-16.  Displacements (free DOFs) and prescribed values at t_{n+1}, t_n and
 * t_{n-1}; alpha of the mid-point rule, the step sizes dt_{n+1} = t_{n+1} - t_n
 * and dt_n = t_n - t_{n-1}, the density.  R and K are accumulated (caller
 * zeroes them); K may be NULL.  HE only (returns 1 otherwise). */
int orc_assemble_transient(const orc_problem *P, const orc_material *mat, const double *u_np1,
                           const double *u_n, const double *u_nm1, const double *p_np1,
                           const double *p_n, const double *p_nm1, double alpha, double dt_np1,
                           double dt_n, double rho, double *R, double *K);

/* The same with the per-point state: crystal plasticity (state AoS 10 per
 * point: pF, g) takes the state at t_{n-1} and t_n, runs the point update at
 * F_{n+1} (state_np1 out, may be NULL) and evaluates each mid point with the
 * mid-point plastic part; HE ignores the state.  Returns 1 for other models. */
int orc_assemble_transient_state(const orc_problem *P, const orc_material *mat, const double *u_np1,
                                 const double *u_n, const double *u_nm1, const double *p_np1,
                                 const double *p_n, const double *p_nm1, double alpha, double dt_np1,
                                 double dt_n, double rho, const double *state_nm1, const double *state_n,
                                 double *state_np1, double *R, double *K);

/* Number of quadrature points per element for nne (1 for 4, 4 for 10). */
int orc_nint(int nne);

#ifdef __cplusplus
}
#endif
#endif
