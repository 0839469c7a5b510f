/*
 * ORACLE — test infrastructure only.  A plain-C, double-precision restatement of
 * the reference ZLLBM single-level LBM time step (collide, pull-stream, domain
 * boundary conditions), used by the tests, the smoke check and the CPU
 * baseline leg of the benchmark as the checker.  The product never links it.
 *
 * Parity pin: the restatement is checked bit-for-bit against dumps produced by
 * the reference itself (built from its own sources with a single-rank MPI
 * stand-in, oracle/Makefile + oracle/ref_harness.cpp); the committed fixtures
 * live in tests/golden/.
 *
 * Node layout: the reference's stored nodes of one uniform level, x fastest,
 * n[0] * n[1] * n[2] nodes (n = cells + 1 per axis: the reference stores both
 * the minimum and the maximum plane, grid/grid_manager3d.cpp:106-112), each
 * with q populations contiguous: f[(node) * q + iq].
 */
#ifndef ZLLBM_ORACLE_ZL_PORT_H_
#define ZLLBM_ORACLE_ZL_PORT_H_
#ifdef __cplusplus
extern "C" {
#endif

enum { ZLP_BC_NONE = 0, ZLP_BC_BOUNCE_BACK = 1, ZLP_BC_PERIODIC = 2, ZLP_BC_NONEQ_EXTRAP = 3,
       ZLP_BC_CONVECTIVE = 4 /* no counterpart in the reference, see apply_face */ };
enum { ZLP_SRT = 0, ZLP_MRT = 1 };
enum { ZLP_LES_OFF = 0, ZLP_LES_SMAGORINSKY = 1 };

typedef struct zlp_level {
    int dims;            /* 2 (D2Q9) or 3 (D3Q19) */
    int n[3];            /* stored nodes per axis; n[2] = 1 in 2D */
    int collision;       /* ZLP_SRT / ZLP_MRT */
    int level;           /* refinement level, dt = 2^-level */
    double nu;           /* lattice viscosity at the background level */
    double rho0;         /* default density (bounce-back wall term, NEQ boundary density) */
    int bc_kind[6];      /* faces in the order xmin, xmax, ymin, ymax, zmin, zmax */
    double bc_vel[6][3]; /* wall / boundary velocity per face */
    int les;             /* ZLP_LES_* ; Smagorinsky with tau_eff = tau0 + tau_sgs */
    double les_cs;       /* Smagorinsky constant (the reference hard-wires 0.16) */
    int has_force;       /* constant body force (Guo forcing) */
    double force[3];
    /* per-node force (GridNodeLbm::force_ of one force group, nodes x 3, x y z) added to the
       constant force in the collision (GetAllForcesForANode, lbm_solver_interface.cpp:132-144);
       NULL: none.  The boundary faces see the constant force only. */
    const double* node_force;
} zlp_level;

/* Advance `steps` time steps in place.  f is the post-stream state (the
 * reference's f_), fc the post-collision state (f_collide_); both are read
 * (missing neighbours keep stale values) and written.  Returns 0 on success. */
int zlp_run(const zlp_level* cfg, double* f, double* fc, int steps);

/* Macroscopic fields of every node (rho[n], u[n * dims]), recomputed from f
 * the way the reference's output does (lbm_grid_interface.cpp:614-657). */
int zlp_macros(const zlp_level* cfg, const double* f, double* rho, double* u);

/* Equilibrium populations, reference arithmetic order (lbm_solver_interface.cpp:374-435). */
void zlp_feq(int dims, double rho, const double* u, double* feq);

/* The MRT collision matrix M^-1 S M built in the reference's loop order
 * (collision_model/lbm_collision_model_mrt.cpp:63-82); out is q*q row-major. */
void zlp_mrt_matrix(int dims, double tau, double* out);

/* The Smagorinsky increment tau_sgs (les_models/lbm_les_smagorinsky.cpp:22-94) for one node,
   with the constant C = 18 cs^2; force and u are read only when has_force is set. */
double zlp_smag_tau_sgs(int dims, const double* f, const double* feq, double tau0, double dt, double cs,
                        int has_force, const double* force, const double* u);

/* Relaxation time at a level, tau = 3 nu / dt + 0.5 (lbm_collision_models.cpp:114-118). */
double zlp_tau(double nu, int level);

#ifdef __cplusplus
}
#endif
#endif  /* ZLLBM_ORACLE_ZL_PORT_H_ */
