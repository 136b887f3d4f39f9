/*
 * oracle.h -- CPU restatement of paraCLAWs' 2D wave-propagation finite-volume step.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load this library, and only as the checker or as the timed CPU
 * stand-in for the reference.  The product path (paraclaws_b200) never calls it.
 *
 * parity unpinned: the reference is Fortran + MPI + LAPACK and cannot be compiled in this
 * image (no Fortran compiler, no MPI, empty mpidcl/VTKFortran submodules) and it ships no
 * tests or golden outputs.  This restatement follows the reference source line by line
 * (citations below, paths relative to the reference project) and is pinned only by
 * hand-derived known-answer tests and by a cross-check of its closed-form wave speeds
 * against LAPACK dgeev (eigen_mode = 1).
 */
#ifndef PARACLAWS_ORACLE_H
#define PARACLAWS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* All fields of control.in (utility/MOD_IO.f90:61-94) that the hot path reads, plus the
 * build's extensions.  Order matters: oracle.py mirrors this layout with ctypes. */
typedef struct orc_params {
    int m_xi, m_eta;
    int num_ghost;                       /* must be 2 */
    int higher_order;                    /* add_higher_order_flux_correction */
    int use_limiter;
    int limiter_method;                  /* 1 minmod, 2 superbee, 3 van Leer, 4 MC (by code) */
    int bc_xi_lower, bc_xi_upper, bc_eta_lower, bc_eta_upper;  /* 1 wall, 2 zero grad., 3 const. grad. */
    int n_snapshots;
    int adaptive;
    int eigen_mode;                      /* 0 closed form, 1 LAPACK dgeev + BLAS dgemv */
    int num_equations;                   /* components per cell, 1 .. ORC_MAX_EQ (0: 3) */
    double xi_min, xi_max, eta_min, eta_max;
    double grav;
    double t_start, t_final, dt_initial;
    double cfl_limit, dt_min, dt_max, growth, shrink;
    long long max_accepted;              /* build extension: stop after this many accepted steps (0 = off) */
} orc_params;

typedef struct orc orc_t;

enum {
    ORC_OK = 0,
    ORC_ERR_NAN = -1,          /* NaN in a Jacobian (examples/.../SMOD_jakobian.f90:55-68) */
    ORC_ERR_NEG_DEPTH = -2,    /* h < 0: complex eigenvalues (utility/SMOD_eigenvalue_problem.f90:72-83) */
    ORC_ERR_BADARG = -5,
    ORC_ERR_FATAL_DT = -7,     /* end_program in updateTime (time_control/MOD_time_control.f90:213-231) */
    ORC_ERR_LAPACK = -8
};

int    orc_load_lapack(const char* so_path);   /* dlopen a LAPACK exporting <prefix>dgeev_/dgemv_ */
orc_t* orc_create(const orc_params* p);
void   orc_destroy(orc_t* o);
int    orc_status(const orc_t* o);
void   orc_set_threads(int n);
int    orc_get_threads(void);

/* state in the reference layout vars(num_equations, -1:m_xi+2, -1:m_eta+2), column-major */
void orc_set_state(orc_t* o, const double* vars);
void orc_get_state(const orc_t* o, double* vars);

/* mesh metrics (same padded layout, one value per cell) */
void orc_get_mesh(const orc_t* o, double* xi, double* eta, double* kappa, double* lr_xi, double* lr_eta);
/* a non-zero source_function for tests of the source hook: phi = (0, -c*hu, -c*hv) (linear
   friction), integrated by integrate_source_term (solver/MOD_solve.f90:295-336); c = 0 is the
   dam break's phi = 0 */
void orc_set_friction(orc_t* o, double c);
/* Equation modules (getJakobi of user_subroutines/MOD_user_subroutines.f90 and the eigenvalues
   of its Jacobian), restated in oracle.c for the checker.  The ids are the ones the library's
   pcl_set_equation takes, so a test passes the same id to both; num_equations of the module
   must be the context's. */
enum {
    ORC_EQ_OWN_SWE = 0,    /* the dam-break shallow water, g from orc_params (3 equations) */
    ORC_EQ_SWE = 1,        /* the same Jacobian with g = p0 (3) */
    ORC_EQ_ACOUSTICS = 2,  /* linear acoustics (p, u, v), p0 = K, p1 = rho (3) */
    ORC_EQ_ADVECTION = 3,  /* q_t + a q_x + b q_y = 0, p0 = a, p1 = b (1) */
    ORC_EQ_BURGERS = 4,    /* Jacobian q in both directions (1) */
    ORC_EQ_SWE_TRACER = 5  /* (h, hu, hv, hc): shallow water carrying a tracer, p0 = g (4) */
};
#define ORC_MAX_EQ 4
int orc_module_num_equations(int module);
int orc_set_equation(orc_t* o, int module, double p0, double p1);
/* replace capacity and face length ratios by those of a mapped grid (finalize_mesh of a user
   mapping, SMOD_mesh_manipulation.f90:147-173); cell centres stay computational */
void orc_set_mesh(orc_t* o, const double* kappa, const double* lr_xi, const double* lr_eta);

int    orc_update_rank_boundaries(orc_t* o);
int    orc_solve_dimensional_split(orc_t* o, int* ierr);
int    orc_sweep(orc_t* o, int ixy, double* cfl_sweep);   /* one sweep, for unit parity */

/* time control (time_control/MOD_time_control.f90) */
int    orc_update_time(orc_t* o, int step_valid);
void   orc_reset_cfl(orc_t* o);
void   orc_set_dt(orc_t* o, double dt);
void   orc_set_time_state(orc_t* o, double time, double dt, double cfl, int snapshot_index);
void   orc_get_time_state(const orc_t* o, double* out8, int* out4);
   /* out8 = {time, dt, dt_previous, CFL, CFL_previous_timestep, time_final, next snapshot time, 0}
      out4 = {snapshot index (1-based), snapshot_exception, n_snapshots, 0} */

/* main loop of main.f90:193-283.  One log row per attempted step:
   log_d[k*4 + {0,1,2,3}] = {dt used, CFL of the attempt, time after, dt after}
   log_i[k*2 + {0,1}]     = {ierr (1 accept / -1 reject), snapshot index after} */
int orc_run(orc_t* o, long long max_attempts, double* log_d, int* log_i, long long log_cap,
            long long* n_attempts, long long* n_accepted);

/* known-answer helpers */
int    orc_hll_interface(int ixy, const double* qL, const double* qR, double grav, int eigen_mode,
                         double* lambda2, double* waves6);
double orc_limiter_phi(int method, double r);

#ifdef __cplusplus
}
#endif
#endif
