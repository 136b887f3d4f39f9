/*
 * oracle.c -- CPU restatement of paraCLAWs' 2D wave-propagation finite-volume step
 * (single MPI rank), in the reference's loop order and operation order.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU stand-in for the
 * reference.  Nothing in the product links or calls this file.
 *
 * parity unpinned (see oracle.h): the reference cannot be built in this image.
 *
 * Build: cc -O2 -ffp-contract=off -fopenmp -fPIC -shared (oracle/Makefile).  No FMA
 * contraction, so every expression rounds exactly where the Fortran source rounds when it is
 * evaluated left to right without contraction (reference Makefile:74-78 builds with
 * -march=native -O3, which lets gfortran contract; that build is not bit-reproducible).
 *
 * Array layout: the reference's column-major AoS vars(neq, -1:m_xi+2, -1:m_eta+2)
 * (domain/SMOD_domain_allocation.f90:94) with neq = num_equations components fastest (the dam
 * break: h, hu, hv), then i, then j.  Work arrays keep the reference's shapes
 * (solver/MOD_work_arrays.f90:61-69) with num_waves = 2: HLL writes two waves, and the
 * reference's further waves (num_waves > 2) stay zero after every flash_work_to_zero.
 *
 * Eigen modes for the HLL wave speed (solver/SMOD_approximate_Riemann_solvers.f90:63-72):
 *   0  closed form of the shallow-water Jacobian: eigenvalues u-c, u, u+c with
 *      u = hu/h (xi sweep) or hv/h (eta sweep) and c = sqrt(g*h); flux J.q in the order of
 *      reference BLAS dgemv ('N': y = 0; y += x(j)*A(:,j) for j = 1..n).
 *   1  LAPACK dgeev (jobvl='N', jobvr='V', workspace query + heap work array per call, as
 *      utility/SMOD_eigenvalue_problem.f90:33-88) and BLAS dgemv (utility/
 *      SMOD_matrix_operations.f90:108-113), loaded with orc_load_lapack().  This is the
 *      faithful cost model of the reference and its closest runnable arithmetic.
 */
#include "oracle.h"

#include <dlfcn.h>
#include <stdio.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define UD_PRECISION 1e-10 /* constant/MOD_constants.f90:18 */
#define NWAVES 2

/* ------------------------------------------------------------------------------------- */
/* LAPACK / BLAS through dlopen (gfortran calling convention: hidden string lengths)      */
/* ------------------------------------------------------------------------------------- */
typedef void (*dgeev_fn)(const char*, const char*, const int*, double*, const int*, double*, double*,
                         double*, const int*, double*, const int*, double*, const int*, int*, size_t,
                         size_t);
typedef void (*dgemv_fn)(const char*, const int*, const int*, const double*, const double*, const int*,
                         const double*, const int*, const double*, double*, const int*, size_t);
static dgeev_fn p_dgeev = NULL;
static dgemv_fn p_dgemv = NULL;

int orc_load_lapack(const char* so_path)
{
    void* h = dlopen(so_path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return ORC_ERR_LAPACK;
    const char* prefixes[] = {"scipy_", "", NULL};
    for (int k = 0; prefixes[k]; ++k) {
        char n1[64], n2[64], n3[96];
        snprintf(n1, sizeof n1, "%sdgeev_", prefixes[k]);
        snprintf(n2, sizeof n2, "%sdgemv_", prefixes[k]);
        void* a = dlsym(h, n1);
        void* b = dlsym(h, n2);
        if (a && b) {
            p_dgeev = (dgeev_fn)a;
            p_dgemv = (dgemv_fn)b;
            /* one BLAS thread per caller: the OpenMP loops above own the parallelism
               (the reference's set_env.sh:18-28 pins its BLAS to one thread as well) */
            snprintf(n3, sizeof n3, "%sopenblas_set_num_threads", prefixes[k]);
            void (*setn)(int) = (void (*)(int))dlsym(h, n3);
            if (setn) setn(1);
            return ORC_OK;
        }
    }
    return ORC_ERR_LAPACK;
}

/* ------------------------------------------------------------------------------------- */
/* Types                                                                                  */
/* ------------------------------------------------------------------------------------- */
typedef struct {
    /* time_control/MOD_time_control.f90:16-66 */
    double time, time_initial, time_final;
    double dt, dt_previous, dt_max, dt_min;
    double* snapshot_intervals;
    int current_snapshot_index; /* 1-based */
    int number_of_snapshots;
    double time_precision, CFL, CFL_target, CFL_previous_timestep;
    double timestep_shrink_limit, timestep_growth_limit, emergency_shrink_ratio;
    int adaptive_timestepping, snapshot_exception;
} tctl_t;

struct orc {
    orc_params p;
    int ni, nj; /* padded extents m+4 */
    double d_xi, d_eta;
    double *vars, *vars_old;
    double *xi, *eta, *kappa, *lr_xi, *lr_eta;
    /* work arrays */
    double *lambda, *waves, *Am, *Ap, *f, *wn2l, *wn2r;
    tctl_t t;
    int status;
    double friction; /* source_function phi = (0, -c hu, -c hv); 0: phi = 0 */
    int eq;          /* equation module (ORC_EQ_*) */
    int neq;         /* num_equations: components per cell */
    double eqp[2];
};

#define CID(o, i, j) ((size_t)((j) + 1) * (size_t)(o)->ni + (size_t)((i) + 1))
#define Q(o, me, i, j) (o)->vars[CID(o, i, j) * (size_t)(o)->neq + (size_t)(me)]
#define LAM(o, mw, i, j) (o)->lambda[CID(o, i, j) * NWAVES + (size_t)(mw)]
#define WAV(o, me, mw, i, j) (o)->waves[(CID(o, i, j) * NWAVES + (size_t)(mw)) * (size_t)(o)->neq + (size_t)(me)]
#define AM(o, me, i, j) (o)->Am[CID(o, i, j) * (size_t)(o)->neq + (size_t)(me)]
#define AP(o, me, i, j) (o)->Ap[CID(o, i, j) * (size_t)(o)->neq + (size_t)(me)]
#define FC(o, me, i, j) (o)->f[CID(o, i, j) * (size_t)(o)->neq + (size_t)(me)]
#define WNL(o, mw, i, j) (o)->wn2l[CID(o, i, j) * NWAVES + (size_t)(mw)]
#define WNR(o, mw, i, j) (o)->wn2r[CID(o, i, j) * NWAVES + (size_t)(mw)]
#define KAP(o, i, j) (o)->kappa[CID(o, i, j)]

static void set_status(orc_t* o, int s)
{
    /* keep the most severe: NaN before negative depth before anything else */
#pragma omp critical(orc_status)
    {
        if (o->status == ORC_OK || s == ORC_ERR_NAN) o->status = s;
    }
}

void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
int orc_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------------------- */
/* Mesh: domain/SMOD_mesh_manipulation.f90:14-178 with the identity coordinate mapping     */
/* (user_subroutines/SMOD_coordinate_mapping.f90:35-43)                                   */
/* ------------------------------------------------------------------------------------- */
static double norm2_2(double a, double b)
{
    /* Fortran NORM2 of a 2-vector.  The uniform mapping always has one zero component, for
       which every NORM2 implementation returns |other| exactly. */
    if (a == 0.0) return fabs(b);
    if (b == 0.0) return fabs(a);
    return sqrt(a * a + b * b);
}

static void build_mesh(orc_t* o)
{
    const orc_params* p = &o->p;
    o->d_xi = (p->xi_max - p->xi_min) / p->m_xi;     /* :28 */
    o->d_eta = (p->eta_max - p->eta_min) / p->m_eta; /* :29 */
    for (int j = -1; j <= p->m_eta + 2; ++j) {
        for (int i = -1; i <= p->m_xi + 2; ++i) {
            double xc[6], yc[6];
            xc[1] = p->xi_min + (double)(i - 1) * o->d_xi; /* :36 */
            xc[2] = xc[1] + o->d_xi;
            xc[3] = xc[2];
            xc[4] = xc[1];
            xc[5] = xc[1];
            yc[1] = p->eta_min + (double)(j - 1) * o->d_eta; /* :43 */
            yc[2] = yc[1];
            yc[3] = yc[2] + o->d_eta;
            yc[4] = yc[3];
            yc[5] = yc[1];
            size_t c = CID(o, i, j);
            o->xi[c] = p->xi_min + (double)(i - 1) * o->d_xi + o->d_xi / 2;    /* :50 */
            o->eta[c] = p->eta_min + (double)(j - 1) * o->d_eta + o->d_eta / 2; /* :51 */
            /* finalize_mesh :147-173 */
            double fdx = xc[4] - xc[1], fdy = yc[4] - yc[1];
            o->lr_xi[c] = norm2_2(fdx, fdy) / o->d_eta;
            fdx = xc[2] - xc[1];
            fdy = yc[2] - yc[1];
            o->lr_eta[c] = norm2_2(fdx, fdy) / o->d_xi;
            double area = 0.0;
            for (int m = 1; m <= 4; ++m) area = area + (0.5 * (yc[m] + yc[m + 1])) * (xc[m] - xc[m + 1]);
            o->kappa[c] = area / (o->d_xi * o->d_eta);
        }
    }
}

/* ------------------------------------------------------------------------------------- */
/* Time control: time_control/MOD_time_control.f90                                      */
/* ------------------------------------------------------------------------------------- */
static int tctl_init(tctl_t* t, const orc_params* p)
{
    /* initialize :70-151 */
    t->time_initial = p->t_start;
    t->time_final = p->t_final;
    t->time = p->t_start;
    t->dt = p->dt_initial;
    t->dt_previous = p->dt_initial;
    t->dt_max = p->dt_max;
    t->dt_min = p->dt_min;
    t->adaptive_timestepping = p->adaptive ? 1 : 0;
    if (t->dt_min > t->dt_max) return ORC_ERR_BADARG; /* :114-119 */
    t->number_of_snapshots = p->n_snapshots < 1 ? 1 : p->n_snapshots;
    t->snapshot_intervals = (double*)malloc(sizeof(double) * (size_t)t->number_of_snapshots);
    double si = (t->time_final - t->time_initial) / t->number_of_snapshots;
    for (int i = 1; i <= t->number_of_snapshots; ++i) t->snapshot_intervals[i - 1] = t->time_initial + i * si;
    t->snapshot_intervals[t->number_of_snapshots - 1] = t->time_final;
    t->current_snapshot_index = 1;
    t->CFL = 0.0;
    t->CFL_previous_timestep = 0.0;
    t->CFL_target = p->cfl_limit;
    t->time_precision = 0.01;
    t->timestep_growth_limit = p->growth;
    t->timestep_shrink_limit = p->shrink;
    t->emergency_shrink_ratio = 0.25;
    t->snapshot_exception = 0;
    return ORC_OK;
}

static double tctl_next_snapshot(const tctl_t* t)
{
    /* the reference never reads past the last snapshot: its loop ends at time_final */
    int k = t->current_snapshot_index;
    if (k > t->number_of_snapshots) k = t->number_of_snapshots;
    return t->snapshot_intervals[k - 1];
}

static int tctl_update_time(tctl_t* t, int step_valid)
{
    /* updateTime :153-243 */
    double change_factor, dt_step;
    t->dt_previous = t->dt;
    dt_step = t->dt;
    if (step_valid) {
        if (t->adaptive_timestepping) {
            if (t->CFL > 0.0)
                change_factor = t->CFL_target / t->CFL;
            else
                change_factor = 1.0;
            if (change_factor >= t->timestep_growth_limit)
                change_factor = t->timestep_growth_limit;
            else if (fabs(change_factor - 1.0) <= t->time_precision)
                change_factor = 1.0;
            dt_step = t->dt_previous * change_factor;
        }
        double ts = tctl_next_snapshot(t);
        if (t->time + dt_step > ts) {
            dt_step = ts - t->time;
            t->snapshot_exception = 1;
        } else {
            t->snapshot_exception = 0;
        }
    } else {
        if (!t->adaptive_timestepping) return ORC_ERR_FATAL_DT; /* :213-216 */
        dt_step = t->emergency_shrink_ratio * t->dt;
    }
    if (dt_step > t->dt_max) dt_step = t->dt_max;
    if (dt_step < t->dt_min) {
        if (!t->adaptive_timestepping && !t->snapshot_exception) return ORC_ERR_FATAL_DT; /* :228-231 */
        dt_step = t->dt_min;
    }
    if (step_valid) t->time = t->time + dt_step;
    t->dt = dt_step;
    return ORC_OK;
}

static int tctl_valid(const tctl_t* t)
{
    /* check_timestep_validity :262-268 */
    return t->CFL_target / t->CFL >= t->timestep_shrink_limit;
}

/* ------------------------------------------------------------------------------------- */
/* Equation module: examples/2D_dam_break/cartesian/SMOD_jakobian.f90:16-71               */
/* J stored column-major, J[(col-1)*3 + (row-1)] as Fortran jakobi(row, col).             */
/* ------------------------------------------------------------------------------------- */
static int jakobi(int ixy, const double* q, double g, double* J)
{
    const double h = q[0], hu = q[1], hv = q[2];
    for (int k = 0; k < 9; ++k) J[k] = 0.0;
#define JS(r, c) J[((c)-1) * 3 + ((r)-1)]
    if (ixy == 1) {
        JS(1, 1) = 0.0; JS(1, 2) = 1.0; JS(1, 3) = 0.0;
        JS(2, 1) = -((hu * hu) / (h * h)) + g * h; JS(2, 2) = (2.0 * hu) / h; JS(2, 3) = 0.0;
        JS(3, 1) = -((hu * hv) / (h * h)); JS(3, 2) = hv / h; JS(3, 3) = hu / h;
    } else {
        JS(1, 1) = 0.0; JS(1, 2) = 0.0; JS(1, 3) = 1.0;
        JS(2, 1) = -((hu * hv) / (h * h)); JS(2, 2) = hv / h; JS(2, 3) = hu / h;
        JS(3, 1) = -((hv * hv) / (h * h)) + g * h; JS(3, 2) = 0.0; JS(3, 3) = (2.0 * hv) / h;
    }
#undef JS
    for (int k = 0; k < 9; ++k)
        if (isnan(J[k])) return ORC_ERR_NAN;
    return ORC_OK;
}

/* ------------------------------------------------------------------------------------- */
/* Other equation modules: the caller's physics through the getJakobi interface            */
/* (user_subroutines/MOD_user_subroutines.f90), n = num_equations, J column-major n x n as   */
/* Fortran jakobi(row, col) = J[(col-1)*n + (row-1)], with the eigenvalues                   */
/* calculateEigenSolution would find (closed form in eigen mode 0, dgeev in mode 1).         */
/* Restated here for the checker from each module's equations, independently of the         */
/* library's own module code.                                                              */
/* ------------------------------------------------------------------------------------- */
int orc_module_num_equations(int eq)
{
    switch (eq) {
    case ORC_EQ_OWN_SWE: case ORC_EQ_SWE: case ORC_EQ_ACOUSTICS: return 3;
    case ORC_EQ_ADVECTION: case ORC_EQ_BURGERS: return 1;
    case ORC_EQ_SWE_TRACER: return 4;
    default: return 0;
    }
}

/* the component a reflective wall negates on xi (ixy 1) / eta (ixy 2) sides; -1: mirror all */
static int module_wall(int eq, int ixy)
{
    return (eq == ORC_EQ_ADVECTION || eq == ORC_EQ_BURGERS) ? -1 : ixy;
}

static int module_jakobi(int eq, const double* prm, int ixy, const double* q, double g, double* J)
{
    const int n = orc_module_num_equations(eq);
    if (eq == ORC_EQ_OWN_SWE || eq == ORC_EQ_SWE) return jakobi(ixy, q, eq == ORC_EQ_SWE ? prm[0] : g, J);
    for (int k = 0; k < n * n; ++k) J[k] = 0.0;
#define JN(r, c) J[((c)-1) * n + ((r)-1)]
    if (eq == ORC_EQ_ACOUSTICS) {
        /* p_t + K (u_x + v_y) = 0, rho u_t + p_x = 0, rho v_t + p_y = 0 */
        const double K = prm[0], rho = prm[1];
        if (ixy == 1) {
            JN(1, 2) = K;
            JN(2, 1) = 1.0 / rho;
        } else {
            JN(1, 3) = K;
            JN(3, 1) = 1.0 / rho;
        }
    } else if (eq == ORC_EQ_ADVECTION) {
        /* q_t + a q_x + b q_y = 0 */
        JN(1, 1) = ixy == 1 ? prm[0] : prm[1];
    } else if (eq == ORC_EQ_BURGERS) {
        /* Jacobian q in both directions */
        JN(1, 1) = q[0];
    } else if (eq == ORC_EQ_SWE_TRACER) {
        /* the dam break's rows plus the transport of hc: flux (n hc)/h with n the normal momentum */
        const double h = q[0], hu = q[1], hv = q[2], hc = q[3], gg = prm[0];
        if (ixy == 1) {
            JN(1, 1) = 0.0; JN(1, 2) = 1.0; JN(1, 3) = 0.0; JN(1, 4) = 0.0;
            JN(2, 1) = -((hu * hu) / (h * h)) + gg * h; JN(2, 2) = (2.0 * hu) / h;
            JN(3, 1) = -((hu * hv) / (h * h)); JN(3, 2) = hv / h; JN(3, 3) = hu / h;
            JN(4, 1) = -((hu * hc) / (h * h)); JN(4, 2) = hc / h; JN(4, 4) = hu / h;
        } else {
            JN(1, 3) = 1.0;
            JN(2, 1) = -((hu * hv) / (h * h)); JN(2, 2) = hv / h; JN(2, 3) = hu / h;
            JN(3, 1) = -((hv * hv) / (h * h)) + gg * h; JN(3, 3) = (2.0 * hv) / h;
            JN(4, 1) = -((hv * hc) / (h * h)); JN(4, 3) = hc / h; JN(4, 4) = hv / h;
        }
    }
#undef JN
    for (int k = 0; k < n * n; ++k)
        if (isnan(J[k])) return ORC_ERR_NAN;
    return ORC_OK;
}

/* closed-form eigenvalues of a module's Jacobian (real; the order does not matter to HLL) */
static int module_eigen(int eq, const double* prm, int ixy, const double* q, double g, double* lam)
{
    if (eq == ORC_EQ_OWN_SWE || eq == ORC_EQ_SWE || eq == ORC_EQ_SWE_TRACER) {
        const double gg = eq == ORC_EQ_OWN_SWE ? g : prm[0];
        const double h = q[0];
        if (h < 0.0) return ORC_ERR_NEG_DEPTH;
        const double u = (ixy == 1 ? q[1] : q[2]) / h;
        const double c = sqrt(gg * h);
        lam[0] = u - c;
        lam[1] = u;
        lam[2] = u + c;
        if (eq == ORC_EQ_SWE_TRACER) lam[3] = u;
        return ORC_OK;
    }
    if (eq == ORC_EQ_ACOUSTICS) {
        const double c = sqrt(prm[0] / prm[1]);
        lam[0] = -c;
        lam[1] = 0.0;
        lam[2] = c;
        return ORC_OK;
    }
    lam[0] = eq == ORC_EQ_BURGERS ? q[0] : (ixy == 1 ? prm[0] : prm[1]);
    return ORC_OK;
}

/* reference BLAS dgemv('N', n, n, 1.0, A, n, x, 1, 0.0, y, 1) */
static void matvec(int mode, int n, const double* A, const double* x, double* y)
{
    if (mode == 1) {
        const int one = 1;
        const double alpha = 1.0, beta = 0.0;
        p_dgemv("N", &n, &n, &alpha, A, &n, x, &one, &beta, y, &one, 1);
        return;
    }
    for (int r = 0; r < n; ++r) y[r] = 0.0;
    for (int c = 0; c < n; ++c) {
        const double temp = x[c];
        for (int r = 0; r < n; ++r) y[r] = y[r] + temp * A[c * n + r];
    }
}

/* calculateEigenSolution in eigen mode 1: LAPACK dgeev on the n x n Jacobian
   (utility/SMOD_eigenvalue_problem.f90:33-88) */
static int eigen_dgeev(int n, const double* J, double* lam)
{
    const int one = 1;
    double A[ORC_MAX_EQ * ORC_MAX_EQ], wr[ORC_MAX_EQ], wi[ORC_MAX_EQ], vl[1] = {0},
        vr[ORC_MAX_EQ * ORC_MAX_EQ], wq[1] = {0};
    int info = 0, lwork = -1;
    memcpy(A, J, sizeof(double) * (size_t)(n * n));
    memset(vr, 0, sizeof vr);
    memset(wr, 0, sizeof wr);
    memset(wi, 0, sizeof wi);
    double* work = (double*)malloc(sizeof(double));
    p_dgeev("N", "V", &n, A, &n, wr, wi, vl, &one, vr, &n, wq, &lwork, &info, 1, 1);
    lwork = (int)wq[0];
    free(work);
    work = (double*)calloc((size_t)(lwork > 1 ? lwork : 1), sizeof(double));
    p_dgeev("N", "V", &n, A, &n, wr, wi, vl, &one, vr, &n, work, &lwork, &info, 1, 1);
    free(work);
    for (int k = 0; k < n; ++k) {
        if (wi[k] > UD_PRECISION) return ORC_ERR_NEG_DEPTH; /* :72-83 */
        lam[k] = wr[k];
    }
    return ORC_OK;
}

/* HLL: solver/SMOD_approximate_Riemann_solvers.f90:15-102 for one interface, n components */
static int hll_core_eq(int eq, const double* prm, int ixy, const double* qL, const double* qR, double g, int mode,
                       double* lam2, double* W /* [mw*n+me] */)
{
    const int n = orc_module_num_equations(eq);
    double JL[ORC_MAX_EQ * ORC_MAX_EQ], JR[ORC_MAX_EQ * ORC_MAX_EQ], lL[ORC_MAX_EQ], lR[ORC_MAX_EQ],
        fL[ORC_MAX_EQ], fR[ORC_MAX_EQ];
    int st = ORC_OK, s;
    for (int k = 0; k < n; ++k) lL[k] = lR[k] = 0.0;
    if ((s = module_jakobi(eq, prm, ixy, qL, g, JL)) != ORC_OK) st = s;
    if ((s = module_jakobi(eq, prm, ixy, qR, g, JR)) != ORC_OK) st = s;
    if (st != ORC_OK) {
        lam2[0] = lam2[1] = 0.0;
        for (int k = 0; k < 2 * n; ++k) W[k] = 0.0;
        return st;
    }
    if (mode == 1) {
        if ((s = eigen_dgeev(n, JL, lL)) != ORC_OK) st = s;
        if ((s = eigen_dgeev(n, JR, lR)) != ORC_OK) st = s;
    } else {
        if ((s = module_eigen(eq, prm, ixy, qL, g, lL)) != ORC_OK) st = s;
        if ((s = module_eigen(eq, prm, ixy, qR, g, lR)) != ORC_OK) st = s;
    }
    /* s2 = maxval([abs(lambda_left), abs(lambda_right)]) :66 */
    double s2 = fabs(lL[0]);
    for (int k = 1; k < n; ++k) s2 = fabs(lL[k]) > s2 ? fabs(lL[k]) : s2;
    for (int k = 0; k < n; ++k) s2 = fabs(lR[k]) > s2 ? fabs(lR[k]) : s2;
    double s1 = -s2;
    lam2[1] = s2;
    lam2[0] = s1;
    for (int k = 0; k < n; ++k) fL[k] = fR[k] = 0.0;
    if (fabs(lam2[0]) > UD_PRECISION && fabs(lam2[1]) > UD_PRECISION) {
        matvec(mode, n, JL, qL, fL);
        matvec(mode, n, JR, qR, fR);
        for (int me = 0; me < n; ++me) {
            double qi = (((fR[me] - fL[me]) - s2 * qR[me]) + s1 * qL[me]) / ((UD_PRECISION + s1) - s2);
            W[0 * n + me] = qi - qL[me];
            W[1 * n + me] = qR[me] - qi;
        }
    } else {
        lam2[0] = lam2[1] = 0.0;
        for (int k = 0; k < 2 * n; ++k) W[k] = 0.0;
    }
    return st;
}

static int hll_core(int ixy, const double* qL, const double* qR, double g, int mode, double* lam2, double* W)
{
    return hll_core_eq(ORC_EQ_OWN_SWE, NULL, ixy, qL, qR, g, mode, lam2, W);
}

int orc_hll_interface(int ixy, const double* qL, const double* qR, double grav, int eigen_mode, double* lambda2,
                      double* waves6)
{
    if (eigen_mode == 1 && !p_dgeev) return ORC_ERR_LAPACK;
    return hll_core(ixy, qL, qR, grav, eigen_mode, lambda2, waves6);
}

static void wave_decomposition(orc_t* o, int ixy, int i, int j)
{
    double qL[ORC_MAX_EQ], qR[ORC_MAX_EQ], lam2[2], W[2 * ORC_MAX_EQ];
    const int il = ixy == 1 ? i - 1 : i, jl = ixy == 1 ? j : j - 1;
    for (int me = 0; me < o->neq; ++me) {
        qL[me] = Q(o, me, il, jl);
        qR[me] = Q(o, me, i, j);
    }
    int st = hll_core_eq(o->eq, o->eqp, ixy, qL, qR, o->p.grav, o->p.eigen_mode, lam2, W);
    if (st != ORC_OK) set_status(o, st);
    LAM(o, 0, i, j) = lam2[0];
    LAM(o, 1, i, j) = lam2[1];
    for (int mw = 0; mw < 2; ++mw)
        for (int me = 0; me < o->neq; ++me) WAV(o, me, mw, i, j) = W[mw * o->neq + me];
}

/* split_flux: solver/MOD_flux_calculation.f90:82-121 */
static void split_flux(orc_t* o)
{
    const int mx = o->p.m_xi, my = o->p.m_eta;
#pragma omp parallel for collapse(2)
    for (int j = 0; j <= my + 1; ++j)
        for (int i = 0; i <= mx + 1; ++i)
            for (int mw = 0; mw < 2; ++mw) {
                const double s = LAM(o, mw, i, j);
                for (int me = 0; me < o->neq; ++me) {
                    const double w = WAV(o, me, mw, i, j);
                    const double mask = s < 0.0 ? 1.0 : 0.0;
                    AM(o, me, i, j) = AM(o, me, i, j) + mask * s * w;
                    AP(o, me, i, j) = AP(o, me, i, j) + (1.0 - mask) * s * w;
                }
            }
}

/* integrate_flux_difference: solver/MOD_solve.f90:177-238 */
static void integrate_flux_difference(orc_t* o, int ixy)
{
    const int mx = o->p.m_xi, my = o->p.m_eta;
    const double delta = ixy == 1 ? o->d_xi : o->d_eta;
    const double dtod = o->t.dt / delta;
#pragma omp parallel for collapse(2)
    for (int j = 1; j <= my; ++j)
        for (int i = 1; i <= mx; ++i) {
            double lrl, lrr;
            if (ixy == 1) {
                lrl = o->lr_xi[CID(o, i, j)];
                lrr = o->lr_xi[CID(o, i + 1, j)];
            } else {
                lrl = o->lr_eta[CID(o, i, j)];
                lrr = o->lr_eta[CID(o, i, j + 1)];
            }
            for (int me = 0; me < o->neq; ++me) {
                const double amr = ixy == 1 ? AM(o, me, i + 1, j) : AM(o, me, i, j + 1);
                Q(o, me, i, j) = Q(o, me, i, j) - dtod / KAP(o, i, j) * (lrl * AP(o, me, i, j) + lrr * amr);
            }
        }
}

/* limiter: solver/MOD_flux_correction.f90:17-125 (serial in the reference) */
double orc_limiter_phi(int method, double r)
{
    switch (method) {
    case 1: return fmax(0.0, fmin(1.0, r));
    case 2: return fmax(fmax(0.0, fmin(1.0, 2.0 * r)), fmin(2.0, r));
    case 3: return (r + fabs(r)) / (1.0 + fabs(r));
    case 4: return fmax(0.0, fmin(fmin((1.0 + r) / 2.0, 2.0), 2.0 * r));
    default: return NAN;
    }
}

static void limiter(orc_t* o, int ixy)
{
    const int mx = o->p.m_xi, my = o->p.m_eta;
    if (!o->p.use_limiter) return;
    if (ixy == 1) {
        const int i = 0;
        for (int j = 1; j <= my; ++j)
            for (int mw = 0; mw < 2; ++mw)
                for (int me = 0; me < o->neq; ++me)
                    WNR(o, mw, i, j) = WNR(o, mw, i, j) + WAV(o, me, mw, i, j) * WAV(o, me, mw, i + 1, j);
    } else {
        const int j = 0;
        for (int i = 1; i <= mx; ++i)
            for (int mw = 0; mw < 2; ++mw)
                for (int me = 0; me < o->neq; ++me)
                    WNR(o, mw, i, j) = WNR(o, mw, i, j) + WAV(o, me, mw, i, j) * WAV(o, me, mw, i, j + 1);
    }
    for (int j = 1; j <= my; ++j)
        for (int i = 1; i <= mx; ++i)
            for (int mw = 0; mw < 2; ++mw) {
                double wnorm2 = 0.0;
                WNL(o, mw, i, j) = ixy == 1 ? WNR(o, mw, i - 1, j) : WNR(o, mw, i, j - 1);
                WNR(o, mw, i, j) = 0.0;
                const int ir = i + (ixy == 1 ? 1 : 0), jr = j + (ixy == 1 ? 0 : 1);
                for (int me = 0; me < o->neq; ++me) {
                    wnorm2 = wnorm2 + WAV(o, me, mw, i, j) * WAV(o, me, mw, i, j);
                    WNR(o, mw, i, j) = WNR(o, mw, i, j) + WAV(o, me, mw, i, j) * WAV(o, me, mw, ir, jr);
                }
                const double up = LAM(o, mw, i, j) > 0.0 ? WNL(o, mw, i, j) : WNR(o, mw, i, j);
                const double r = up / wnorm2;
                const double phi = orc_limiter_phi(o->p.limiter_method, r);
                if (!(fabs(wnorm2) <= UD_PRECISION))
                    for (int me = 0; me < o->neq; ++me) WAV(o, me, mw, i, j) = phi * WAV(o, me, mw, i, j);
            }
}

/* second_order_flux_correction: solver/MOD_flux_correction.f90:127-187 */
static void second_order_flux_correction(orc_t* o, int ixy)
{
    const int mx = o->p.m_xi, my = o->p.m_eta;
    const double delta = ixy == 1 ? o->d_xi : o->d_eta;
    const double dtod = o->t.dt / delta;
    const int jlo = ixy == 1 ? 1 : 0, jhi = ixy == 1 ? my : my + 1;
    const int ilo = ixy == 1 ? 0 : 1, ihi = ixy == 1 ? mx + 1 : mx;
#pragma omp parallel for collapse(2)
    for (int j = jlo; j <= jhi; ++j)
        for (int i = ilo; i <= ihi; ++i) {
            const double kb = ixy == 1 ? 0.5 * (KAP(o, i - 1, j) + KAP(o, i, j)) : 0.5 * (KAP(o, i, j - 1) + KAP(o, i, j));
            for (int mw = 0; mw < 2; ++mw) {
                const double al = fabs(LAM(o, mw, i, j));
                for (int me = 0; me < o->neq; ++me)
                    FC(o, me, i, j) = FC(o, me, i, j) + 0.5 * al * (1.0 - al * dtod / kb) * WAV(o, me, mw, i, j);
            }
        }
}

/* integrator_flux_correction_increment: solver/MOD_solve.f90:240-293 */
static void integrator_flux_correction_increment(orc_t* o, int ixy)
{
    const int mx = o->p.m_xi, my = o->p.m_eta;
    const double delta = ixy == 1 ? o->d_xi : o->d_eta;
    const double dtod = o->t.dt / delta;
#pragma omp parallel for collapse(2)
    for (int j = 1; j <= my; ++j)
        for (int i = 1; i <= mx; ++i)
            for (int me = 0; me < o->neq; ++me) {
                const double fr = ixy == 1 ? FC(o, me, i + 1, j) : FC(o, me, i, j + 1);
                Q(o, me, i, j) = Q(o, me, i, j) - dtod / KAP(o, i, j) * (fr - FC(o, me, i, j));
            }
}

/* flash_work_to_zero: solver/MOD_work_arrays.f90:78-109 */
static void flash_work_to_zero(orc_t* o)
{
    const size_t nc = (size_t)o->ni * (size_t)o->nj;
#pragma omp parallel for
    for (long long c = 0; c < (long long)nc; ++c) {
        for (int mw = 0; mw < 2; ++mw) {
            o->wn2l[c * 2 + mw] = 0.0;
            o->wn2r[c * 2 + mw] = 0.0;
            o->lambda[c * 2 + mw] = 0.0;
            for (int me = 0; me < o->neq; ++me) {
                o->Am[c * o->neq + me] = 0.0;
                o->Ap[c * o->neq + me] = 0.0;
                o->waves[(c * 2 + mw) * o->neq + me] = 0.0;
                o->f[c * o->neq + me] = 0.0;
            }
        }
    }
}

/* one sweep of solve_dimensional_split (solver/MOD_solve.f90:69-105 / 122-157); returns the
   sweep's CFL_local contribution */
static double sweep(orc_t* o, int ixy)
{
    const int mx = o->p.m_xi, my = o->p.m_eta;
    double cfl_local = 0.0;
    const double dt = o->t.dt;
    if (ixy == 1) {
#pragma omp parallel for reduction(max : cfl_local)
        for (int j = 1; j <= my; ++j)
            for (int i = 0; i <= mx + 1; ++i) {
                wave_decomposition(o, 1, i, j);
                for (int mw = 0; mw < 2; ++mw) cfl_local = fmax(cfl_local, LAM(o, mw, i, j) * dt / o->d_xi);
            }
    } else {
#pragma omp parallel for reduction(max : cfl_local)
        for (int i = 1; i <= mx; ++i)
            for (int j = 0; j <= my + 1; ++j) {
                wave_decomposition(o, 2, i, j);
                for (int mw = 0; mw < 2; ++mw) cfl_local = fmax(cfl_local, LAM(o, mw, i, j) * dt / o->d_eta);
            }
    }
    split_flux(o);
    integrate_flux_difference(o, ixy);
    if (o->p.higher_order) {
        limiter(o, ixy);
        second_order_flux_correction(o, ixy);
        integrator_flux_correction_increment(o, ixy);
    }
    return cfl_local;
}

int orc_sweep(orc_t* o, int ixy, double* cfl_sweep)
{
    double c = sweep(o, ixy);
    flash_work_to_zero(o);
    if (cfl_sweep) *cfl_sweep = c;
    return o->status;
}

int orc_solve_dimensional_split(orc_t* o, int* ierr)
{
    double cfl_local;
    *ierr = -1;
    if (o->eq < 0) return ORC_ERR_BADARG; /* num_equations != 3 needs a module */
    cfl_local = sweep(o, 1);
    o->t.CFL = fmax(o->t.CFL, cfl_local); /* update_max_CFL */
    flash_work_to_zero(o);
    if (o->status != ORC_OK) return o->status;
    if (!tctl_valid(&o->t)) {
        *ierr = -1;
        return ORC_OK;
    }
    cfl_local = fmax(cfl_local, sweep(o, 2)); /* CFL_local is not reset between sweeps */
    o->t.CFL = fmax(o->t.CFL, cfl_local);
    flash_work_to_zero(o);
    if (o->status != ORC_OK) return o->status;
    *ierr = tctl_valid(&o->t) ? 1 : -1;
    return ORC_OK;
}

/* ------------------------------------------------------------------------------------- */
/* Boundary conditions: user_subroutines/SMOD_boundary_conditions.f90:58-213              */
/* code 1 (BC_USER; the reference aborts) is filled here with a reflective wall:  */
/* mirror the two nearest interior cells and negate the normal momentum.                   */
/* ------------------------------------------------------------------------------------- */
static double deriv_2p(double x1, double x2, double y1, double y2) { return (y2 - y1) / (x2 - x1); }

int orc_update_rank_boundaries(orc_t* o)
{
    const int mx = o->p.m_xi, my = o->p.m_eta;
    const int bcs[4] = {o->p.bc_xi_lower, o->p.bc_xi_upper, o->p.bc_eta_lower, o->p.bc_eta_upper};
    for (int k = 0; k < 4; ++k)
        if (bcs[k] < 1 || bcs[k] > 3) return ORC_ERR_BADARG;
    const int wx = module_wall(o->eq, 1), wy = module_wall(o->eq, 2); /* wall: negated components */
    /* left */
    for (int j = 1; j <= my; ++j)
        for (int i = -1; i <= 0; ++i)
            for (int me = 0; me < o->neq; ++me) {
                double v;
                if (bcs[0] == 2) v = Q(o, me, 1, j);
                else if (bcs[0] == 3)
                    v = Q(o, me, 1, j) + deriv_2p(o->xi[CID(o, 1, j)], o->xi[CID(o, 2, j)], Q(o, me, 1, j), Q(o, me, 2, j)) *
                                             (o->xi[CID(o, i, j)] - o->xi[CID(o, 1, j)]);
                else v = me == wx ? -Q(o, me, 1 - i, j) : Q(o, me, 1 - i, j);
                Q(o, me, i, j) = v;
            }
    /* right */
    for (int j = 1; j <= my; ++j)
        for (int i = mx + 1; i <= mx + 2; ++i)
            for (int me = 0; me < o->neq; ++me) {
                double v;
                if (bcs[1] == 2) v = Q(o, me, mx, j);
                else if (bcs[1] == 3)
                    v = Q(o, me, mx, j) + deriv_2p(o->xi[CID(o, mx - 1, j)], o->xi[CID(o, mx, j)], Q(o, me, mx - 1, j), Q(o, me, mx, j)) *
                                              (o->xi[CID(o, i, j)] - o->xi[CID(o, mx, j)]);
                else v = me == wx ? -Q(o, me, 2 * mx + 1 - i, j) : Q(o, me, 2 * mx + 1 - i, j);
                Q(o, me, i, j) = v;
            }
    /* bottom */
    for (int j = -1; j <= 0; ++j)
        for (int i = 1; i <= mx; ++i)
            for (int me = 0; me < o->neq; ++me) {
                double v;
                if (bcs[2] == 2) v = Q(o, me, i, 1);
                else if (bcs[2] == 3)
                    v = Q(o, me, i, 1) + deriv_2p(o->eta[CID(o, i, 1)], o->eta[CID(o, i, 2)], Q(o, me, i, 1), Q(o, me, i, 2)) *
                                             (o->eta[CID(o, i, j)] - o->eta[CID(o, i, 1)]);
                else v = me == wy ? -Q(o, me, i, 1 - j) : Q(o, me, i, 1 - j);
                Q(o, me, i, j) = v;
            }
    /* top */
    for (int j = my + 1; j <= my + 2; ++j)
        for (int i = 1; i <= mx; ++i)
            for (int me = 0; me < o->neq; ++me) {
                double v;
                if (bcs[3] == 2) v = Q(o, me, i, my);
                else if (bcs[3] == 3)
                    v = Q(o, me, i, my) + deriv_2p(o->eta[CID(o, i, my - 1)], o->eta[CID(o, i, my)], Q(o, me, i, my - 1), Q(o, me, i, my)) *
                                              (o->eta[CID(o, i, j)] - o->eta[CID(o, i, my)]);
                else v = me == wy ? -Q(o, me, i, 2 * my + 1 - j) : Q(o, me, i, 2 * my + 1 - j);
                Q(o, me, i, j) = v;
            }
    return ORC_OK;
}

/* ------------------------------------------------------------------------------------- */
/* Lifecycle                                                                              */
/* ------------------------------------------------------------------------------------- */
orc_t* orc_create(const orc_params* p)
{
    if (p->m_xi < 2 || p->m_eta < 2 || p->num_ghost != 2) return NULL;
    if (p->higher_order && p->use_limiter && (p->limiter_method < 1 || p->limiter_method > 4)) return NULL;
    if (p->eigen_mode == 1 && !p_dgeev) return NULL;
    const int neq = p->num_equations == 0 ? 3 : p->num_equations;
    if (neq < 1 || neq > ORC_MAX_EQ) return NULL;
    orc_t* o = (orc_t*)calloc(1, sizeof(orc_t));
    o->p = *p;
    o->neq = neq;
    o->eq = neq == 3 ? ORC_EQ_OWN_SWE : -1;
    o->ni = p->m_xi + 4;
    o->nj = p->m_eta + 4;
    const size_t nc = (size_t)o->ni * (size_t)o->nj;
    o->vars = (double*)calloc(nc * (size_t)o->neq, sizeof(double));
    o->vars_old = (double*)calloc(nc * (size_t)o->neq, sizeof(double));
    o->xi = (double*)calloc(nc, sizeof(double));
    o->eta = (double*)calloc(nc, sizeof(double));
    o->kappa = (double*)calloc(nc, sizeof(double));
    o->lr_xi = (double*)calloc(nc, sizeof(double));
    o->lr_eta = (double*)calloc(nc, sizeof(double));
    o->lambda = (double*)calloc(nc * NWAVES, sizeof(double));
    o->waves = (double*)calloc(nc * NWAVES * (size_t)o->neq, sizeof(double));
    o->Am = (double*)calloc(nc * (size_t)o->neq, sizeof(double));
    o->Ap = (double*)calloc(nc * (size_t)o->neq, sizeof(double));
    o->f = (double*)calloc(nc * (size_t)o->neq, sizeof(double));
    o->wn2l = (double*)calloc(nc * NWAVES, sizeof(double));
    o->wn2r = (double*)calloc(nc * NWAVES, sizeof(double));
    build_mesh(o);
    if (tctl_init(&o->t, p) != ORC_OK) {
        orc_destroy(o);
        return NULL;
    }
    o->status = ORC_OK;
    return o;
}

void orc_destroy(orc_t* o)
{
    if (!o) return;
    free(o->vars); free(o->vars_old); free(o->xi); free(o->eta); free(o->kappa); free(o->lr_xi);
    free(o->lr_eta); free(o->lambda); free(o->waves); free(o->Am); free(o->Ap); free(o->f);
    free(o->wn2l); free(o->wn2r); free(o->t.snapshot_intervals);
    free(o);
}

int orc_status(const orc_t* o) { return o->status; }

void orc_set_state(orc_t* o, const double* vars)
{
    memcpy(o->vars, vars, sizeof(double) * (size_t)o->ni * (size_t)o->nj * (size_t)o->neq);
}
void orc_get_state(const orc_t* o, double* vars)
{
    memcpy(vars, o->vars, sizeof(double) * (size_t)o->ni * (size_t)o->nj * (size_t)o->neq);
}
void orc_get_mesh(const orc_t* o, double* xi, double* eta, double* kappa, double* lr_xi, double* lr_eta)
{
    const size_t n = sizeof(double) * (size_t)o->ni * (size_t)o->nj;
    if (xi) memcpy(xi, o->xi, n);
    if (eta) memcpy(eta, o->eta, n);
    if (kappa) memcpy(kappa, o->kappa, n);
    if (lr_xi) memcpy(lr_xi, o->lr_xi, n);
    if (lr_eta) memcpy(lr_eta, o->lr_eta, n);
}

void orc_set_friction(orc_t* o, double c) { o->friction = c; }

int orc_set_equation(orc_t* o, int module, double p0, double p1)
{
    if (orc_module_num_equations(module) != o->neq) return ORC_ERR_BADARG;
    o->eq = module;
    o->eqp[0] = p0;
    o->eqp[1] = p1;
    return ORC_OK;
}

void orc_set_mesh(orc_t* o, const double* kappa, const double* lr_xi, const double* lr_eta)
{
    const size_t n = sizeof(double) * (size_t)o->ni * (size_t)o->nj;
    memcpy(o->kappa, kappa, n);
    memcpy(o->lr_xi, lr_xi, n);
    memcpy(o->lr_eta, lr_eta, n);
}

int orc_update_time(orc_t* o, int step_valid) { return tctl_update_time(&o->t, step_valid); }
void orc_reset_cfl(orc_t* o)
{
    o->t.CFL_previous_timestep = o->t.CFL; /* reset_CFL :270-279 */
    o->t.CFL = 0.0;
}
void orc_set_dt(orc_t* o, double dt) { o->t.dt = dt; }
void orc_set_time_state(orc_t* o, double time, double dt, double cfl, int snapshot_index)
{
    o->t.time = time;
    o->t.dt = dt;
    o->t.CFL = cfl;
    o->t.current_snapshot_index = snapshot_index;
}

void orc_get_time_state(const orc_t* o, double* out8, int* out4)
{
    out8[0] = o->t.time;
    out8[1] = o->t.dt;
    out8[2] = o->t.dt_previous;
    out8[3] = o->t.CFL;
    out8[4] = o->t.CFL_previous_timestep;
    out8[5] = o->t.time_final;
    out8[6] = tctl_next_snapshot(&o->t);
    out8[7] = 0.0;
    out4[0] = o->t.current_snapshot_index;
    out4[1] = o->t.snapshot_exception;
    out4[2] = o->t.number_of_snapshots;
    out4[3] = 0;
}

/* main loop: main.f90:193-283 */
int orc_run(orc_t* o, long long max_attempts, double* log_d, int* log_i, long long log_cap, long long* n_attempts,
            long long* n_accepted)
{
    const size_t nbytes = sizeof(double) * (size_t)o->ni * (size_t)o->nj * (size_t)o->neq;
    long long att = 0, acc = 0;
    int rc = ORC_OK;
    if (o->eq < 0) return ORC_ERR_BADARG;
    while (o->t.time < o->t.time_final) {
        if (o->p.max_accepted > 0 && acc >= o->p.max_accepted) break;
        if (max_attempts > 0 && att >= max_attempts) break;
        const double dt_used = o->t.dt;
        int ierr = 0;
        memcpy(o->vars_old, o->vars, nbytes); /* solution_old = solution :201 */
        rc = orc_solve_dimensional_split(o, &ierr);
        if (rc != ORC_OK) break;
        const double cfl = o->t.CFL;
        if (ierr < 0) {
            rc = tctl_update_time(&o->t, 0);
            memcpy(o->vars, o->vars_old, nbytes); /* :221 */
            orc_reset_cfl(o);
        } else {
            /* integrate_source_term (MOD_solve.f90:295-336): with phi = 0 it is q + 0*dt, no change
               for finite q; with friction q_p = q_p + phi_p*dt per interior cell, j outer */
            if (o->friction != 0.0 && o->neq == 3) {
                const double dt = o->t.dt; /* get_dt(): updateTime has not run yet */
                for (int j = 1; j <= o->p.m_eta; ++j)
                    for (int i = 1; i <= o->p.m_xi; ++i) {
                        const double phi[3] = {0.0, -o->friction * Q(o, 1, i, j), -o->friction * Q(o, 2, i, j)};
                        for (int me = 0; me < 3; ++me) Q(o, me, i, j) = Q(o, me, i, j) + phi[me] * dt;
                    }
            }
            orc_update_rank_boundaries(o);
            rc = tctl_update_time(&o->t, 1);
            if (rc == ORC_OK && o->t.time >= tctl_next_snapshot(&o->t) &&
                o->t.current_snapshot_index <= o->t.number_of_snapshots)
                o->t.current_snapshot_index += 1; /* :256-268 */
            orc_reset_cfl(o);
            acc++;
        }
        if (log_d && att < log_cap) {
            log_d[att * 4 + 0] = dt_used;
            log_d[att * 4 + 1] = cfl;
            log_d[att * 4 + 2] = o->t.time;
            log_d[att * 4 + 3] = o->t.dt;
            log_i[att * 2 + 0] = ierr;
            log_i[att * 2 + 1] = o->t.current_snapshot_index;
        }
        att++;
        if (rc != ORC_OK) break;
    }
    if (n_attempts) *n_attempts = att;
    if (n_accepted) *n_accepted = acc;
    return rc;
}
