/* pcl_equations.h -- equation modules of the generic FP64 sweeps: the getJakobi interface of the
 * reference (user_subroutines/MOD_user_subroutines.f90, examples/.../SMOD_jakobian.f90:16-71,
 * an N x N Jacobian for num_equations = N) with the eigenvalues calculateEigenSolution would find
 * (utility/SMOD_eigenvalue_problem.f90), written out in closed form.  The step itself is the
 * reference's for any module: flux J(q).q in BLAS dgemv order, HLL with s2 = max |eigenvalue|
 * over both cells and two waves (solver/SMOD_approximate_Riemann_solvers.f90:15-102, arrays
 * sized by num_equations at :34-44), the limiter and the correction on N components.
 *
 * The reference picks its equation module when it is built (a USER_DIR source replaces the
 * example's jakobian submodule) and sizes the state by num_equations from control.in
 * (utility/MOD_IO.f90:61, constant/MOD_solver_parameters.f90:14,38); here a module is a case of
 * the functions below, compiled into the library and chosen per context with pcl_set_equation,
 * and the context's state has as many planes as control.in's num_equations.  Adding a module
 * means adding a case to each function and rebuilding.
 *
 * Built without contraction everywhere.
 */
#ifndef PCL_EQUATIONS_H
#define PCL_EQUATIONS_H

#include <math.h>

#ifdef __CUDACC__
#define PCL_EQ_FN __host__ __device__ static inline
#else
#define PCL_EQ_FN static inline
#endif

/* module ids */
#define PCL_EQ_SHALLOW_WATER 0         /* the dam-break module; the specialised kernels */
#define PCL_EQ_SHALLOW_WATER_GENERIC 1 /* the same Jacobian through the generic path */
#define PCL_EQ_ACOUSTICS 2             /* linear acoustics q = (p, u, v), params (K, rho) */
#define PCL_EQ_ADVECTION 3             /* one equation q_t + a q_x + b q_y = 0, params (a, b) */
#define PCL_EQ_BURGERS 4               /* one equation with J = q in both directions */
#define PCL_EQ_SHALLOW_WATER_TRACER 5  /* four equations (h, hu, hv, hc): shallow water carrying
                                          a passive tracer c, params (g) */
#define PCL_EQ_COUNT 6
#define PCL_EQ_MAX_EQUATIONS 4         /* the largest num_equations a module has */

/* num_equations of a module (0: unknown module) */
PCL_EQ_FN int pcl_eq_num_equations(int module)
{
    switch (module) {
    case PCL_EQ_SHALLOW_WATER:
    case PCL_EQ_SHALLOW_WATER_GENERIC:
    case PCL_EQ_ACOUSTICS: return 3;
    case PCL_EQ_ADVECTION:
    case PCL_EQ_BURGERS: return 1;
    case PCL_EQ_SHALLOW_WATER_TRACER: return 4;
    default: return 0;
    }
}

/* The component a reflective wall (boundary code 1) negates on a side of sweep direction dir
 * (1 xi, 2 eta): the normal momentum or velocity; -1 when the module has no wall. */
PCL_EQ_FN int pcl_eq_wall_component(int module, int dir)
{
    switch (module) {
    case PCL_EQ_SHALLOW_WATER:
    case PCL_EQ_SHALLOW_WATER_GENERIC:
    case PCL_EQ_ACOUSTICS:
    case PCL_EQ_SHALLOW_WATER_TRACER: return dir;
    default: return -1;
    }
}

/* J(q) for sweep direction dir (1 xi, 2 eta), column-major n x n with n = num_equations
 * (J[(col-1)*n + (row-1)], the Fortran jakobi(row, col)).  prm: module parameters (shallow
 * water: prm[0] = g).  Returns 0, or 1 when an entry is NaN (getJakobi's trap,
 * examples/2D_dam_break/cartesian/SMOD_jakobian.f90:55-70). */
PCL_EQ_FN int pcl_eq_jacobian(int module, int dir, const double* q, const double* prm, double* J)
{
    const int n = pcl_eq_num_equations(module);
    int k;
    for (k = 0; k < n * n; ++k) J[k] = 0.0;
    if (module == PCL_EQ_SHALLOW_WATER || module == PCL_EQ_SHALLOW_WATER_GENERIC) {
        /* SMOD_jakobian.f90:44-53 */
        const double h = q[0], hu = q[1], hv = q[2], g = prm[0];
        if (dir == 1) {
            J[1] = -((hu * hu) / (h * h)) + g * h; J[4] = (2.0 * hu) / h;
            J[2] = -((hu * hv) / (h * h));         J[5] = hv / h;          J[8] = hu / h;
            J[3] = 1.0;
        } else {
            J[1] = -((hu * hv) / (h * h)); J[4] = hv / h; J[7] = hu / h;
            J[2] = -((hv * hv) / (h * h)) + g * h;        J[8] = (2.0 * hv) / h;
            J[6] = 1.0;
        }
    } else if (module == PCL_EQ_ACOUSTICS) {
        /* p_t + K (u_x + v_y) = 0, u_t + p_x / rho = 0, v_t + p_y / rho = 0 */
        const double K = prm[0], rho = prm[1];
        if (dir == 1) {
            J[3] = K;          /* (1, 2) */
            J[1] = 1.0 / rho;  /* (2, 1) */
        } else {
            J[6] = K;          /* (1, 3) */
            J[2] = 1.0 / rho;  /* (3, 1) */
        }
    } else if (module == PCL_EQ_ADVECTION) {
        J[0] = dir == 1 ? prm[0] : prm[1];
    } else if (module == PCL_EQ_BURGERS) {
        J[0] = q[0];
    } else if (module == PCL_EQ_SHALLOW_WATER_TRACER) {
        /* the dam-break Jacobian in rows 1-3 and the tracer row of (hc)_t + (u hc)_x + (v hc)_y = 0:
           row 4 = [-(n hc)/h^2, 0 or hc/h in the normal-momentum column, 0, n/h] */
        const double h = q[0], hu = q[1], hv = q[2], hc = q[3], g = prm[0];
#define JT(r, c) J[((c)-1) * 4 + ((r)-1)]
        if (dir == 1) {
            JT(1, 2) = 1.0;
            JT(2, 1) = -((hu * hu) / (h * h)) + g * h; JT(2, 2) = (2.0 * hu) / h;
            JT(3, 1) = -((hu * hv) / (h * h)); JT(3, 2) = hv / h; JT(3, 3) = hu / h;
            JT(4, 1) = -((hu * hc) / (h * h)); JT(4, 2) = hc / h; JT(4, 4) = hu / h;
        } else {
            JT(1, 3) = 1.0;
            JT(2, 1) = -((hu * hv) / (h * h)); JT(2, 2) = hv / h; JT(2, 3) = hu / h;
            JT(3, 1) = -((hv * hv) / (h * h)) + g * h; JT(3, 3) = (2.0 * hv) / h;
            JT(4, 1) = -((hv * hc) / (h * h)); JT(4, 3) = hc / h; JT(4, 4) = hv / h;
        }
#undef JT
    }
    for (k = 0; k < n * n; ++k)
        if (isnan(J[k])) return 1;
    return 0;
}

/* The eigenvalues of J(q), n of them (real parts; the order is irrelevant: HLL takes
 * max |lambda|).  Returns 0, or 1 when they are complex (calculateEigenSolution's abort,
 * SMOD_eigenvalue_problem.f90:72-83). */
PCL_EQ_FN int pcl_eq_eigenvalues(int module, int dir, const double* q, const double* prm, double* lam)
{
    if (module == PCL_EQ_SHALLOW_WATER || module == PCL_EQ_SHALLOW_WATER_GENERIC ||
        module == PCL_EQ_SHALLOW_WATER_TRACER) {
        /* the tracer adds a second eigenvalue u (the contact) */
        const double h = q[0];
        const double u = (dir == 1 ? q[1] : q[2]) / h;
        const double c = sqrt(prm[0] * h);
        lam[0] = u - c;
        lam[1] = u;
        lam[2] = u + c;
        if (module == PCL_EQ_SHALLOW_WATER_TRACER) lam[3] = u;
        return h < 0.0 ? 1 : 0;
    }
    if (module == PCL_EQ_ACOUSTICS) {
        const double c = sqrt(prm[0] / prm[1]);
        lam[0] = -c;
        lam[1] = 0.0;
        lam[2] = c;
        return 0;
    }
    if (module == PCL_EQ_ADVECTION) {
        lam[0] = dir == 1 ? prm[0] : prm[1];
        return 0;
    }
    if (module == PCL_EQ_BURGERS) {
        lam[0] = q[0];
        return 0;
    }
    return 0;
}

#endif /* PCL_EQUATIONS_H */
