/* pcl_equations.h -- equation modules of the generic FP64 sweeps: the getJakobi interface of the
 * reference (user_subroutines/MOD_user_subroutines.f90, examples/.../SMOD_jakobian.f90) with the
 * eigenvalues calculateEigenSolution would find (utility/SMOD_eigenvalue_problem.f90), written
 * out in closed form.  The step itself is the reference's for any module: flux J(q).q in BLAS
 * dgemv order, HLL with s2 = max |eigenvalue| over both cells, two waves, limiter, correction.
 *
 * The reference picks its equation module when it is built (a USER_DIR source replaces the
 * example's jakobian submodule); here a module is a case of the two functions below, compiled
 * into the library and chosen per context with pcl_set_equation.  Adding one means adding a
 * case to both functions and rebuilding.  Three equations, two waves (num_equations = 3,
 * num_waves = 2 in control.in).
 *
 * Plain C99 so that the CPU oracle can include it too (the module is the caller's definition
 * of the physics, not part of the step under test).  Built without contraction everywhere.
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
#define PCL_EQ_COUNT 3

/* J(q) for sweep direction dir (1 xi, 2 eta), column-major 3 x 3 (J[(col-1)*3 + (row-1)], the
 * Fortran jakobi(row, col)).  prm: module parameters (shallow water: prm[0] = g).  Returns 0, or
 * 1 when an entry is NaN (getJakobi's trap, examples/2D_dam_break/cartesian/SMOD_jakobian.f90:55-70). */
PCL_EQ_FN int pcl_eq_jacobian(int module, int dir, const double* q, const double* prm, double* J)
{
    int k;
    for (k = 0; k < 9; ++k) J[k] = 0.0;
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
    }
    for (k = 0; k < 9; ++k)
        if (isnan(J[k])) return 1;
    return 0;
}

/* The eigenvalues of J(q) (real parts, the order is irrelevant: HLL takes max |lambda|).  Returns
 * 0, or 1 when they are complex (calculateEigenSolution's abort, SMOD_eigenvalue_problem.f90:72-83). */
PCL_EQ_FN int pcl_eq_eigenvalues(int module, int dir, const double* q, const double* prm, double* lam)
{
    if (module == PCL_EQ_SHALLOW_WATER || module == PCL_EQ_SHALLOW_WATER_GENERIC) {
        const double h = q[0];
        const double u = (dir == 1 ? q[1] : q[2]) / h;
        const double c = sqrt(prm[0] * h);
        lam[0] = u - c;
        lam[1] = u;
        lam[2] = u + c;
        return h < 0.0 ? 1 : 0;
    }
    if (module == PCL_EQ_ACOUSTICS) {
        const double c = sqrt(prm[0] / prm[1]);
        lam[0] = -c;
        lam[1] = 0.0;
        lam[2] = c;
        return 0;
    }
    lam[0] = lam[1] = lam[2] = 0.0;
    return 0;
}

#endif /* PCL_EQUATIONS_H */
