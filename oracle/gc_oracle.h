/* CPU oracle for the gridcalc periodic-grid hot path: a plain-C restatement
 * of the reference algorithms, used ONLY as test infrastructure (the parity
 * checker in tests/, the smoke check, and the CPU baseline leg of bench.py).
 * The product path never links or calls it.
 *
 * Every routine follows the reference arithmetic order tap by tap (no FMA
 * contraction: build with -ffp-contract=off), so on identical inputs it
 * reproduces the reference bit for bit; tests/test_oracle.py pins that
 * against the reference compiled from its own headers and against the
 * committed golden vectors in tests/golden/.
 *
 * Layout: i-fastest linear index i + Nx*(j + Ny*k) (core/Grid.hpp:132-137).
 * Vector fields: three planes (x, y, z component), N values each.
 * Order 6 has no reference counterpart (the reference specialises only
 * orders 2 and 4); its weight tables are the standard central-difference
 * ones and are pinned by the Taylor-moment and convergence tests instead.
 *
 * Return codes: 0 ok; 1 invalid argument (message via oc_last_error()).
 */
#ifndef GC_ORACLE_H
#define GC_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

const char* oc_last_error(void);

/* Stencil weight tables (unscaled).  kind: 1 = first derivative,
 * 2 = second derivative, 3 = third derivative, 4 = fourth derivative.
 * Returns the radius, or -1 for an unknown (kind, order); fills
 * weights[0 .. 2*radius]. */
int oc_weights(int kind, int order, double* weights);

int oc_laplacian(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                 const double* in, double* out);
int oc_gradient(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                const double* in, double* out3);
int oc_divergence(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                  const double* in3, double* out);
/* diff/Gradient.hpp:100-137: Vec3d (3 planes) -> Mat3d (9 planes, 3*row + col). */
int oc_gradient_vec(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                    const double* v3, double* out9);
/* diff/Divergence.hpp:100-135: Mat3d (9 planes, 3*row + col) -> Vec3d (3 planes). */
int oc_divergence_mat(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                      const double* m9, double* out3);
/* diff/detail/MultiIndexDerivative.hpp:96-137 (the 31 named partials). */
int oc_mixed(int ax, int ay, int az, int order, int nx, int ny, int nz, double hx, double hy, double hz,
             const double* f, double* out);
int oc_biharmonic(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                  const double* in, double* out);
/* Returns 0, 1 (axis extent) or 2 (D not strictly positive; *bad_index set). */
int oc_cell_laplacian(int nx, int ny, int nz, double hx, double hy, double hz,
                      const double* psi, const double* D, double* out, int64_t* bad_index);

double oc_sum_pairwise(const double* x, size_t n);
double oc_sum_neumaier(const double* x, size_t n);
double oc_integrate(int nx, int ny, int nz, double hx, double hy, double hz,
                    const double* in, int kahan);

/* func::evaluate with a general callable (func/Functional.hpp:88-148 scalar,
 * :183-220 vector), the callable given as a straight-line register program:
 * op 0 const, 1 input a, 2 add, 3 sub, 4 mul, 5 div, 6 neg, 7 abs, 8 sqrt,
 * 9 std::min, 10 std::max; value = r[dst] of the last instruction.  Inputs:
 * scalar psi, grad x/y/z, lap, biharmonic (order 2) up to the arity; vector
 * u x/y/z then M(row, col) = d_col u_row at 3 + 3*row + col.  Returns 0, 1
 * (axis extent) or 3 (malformed program). */
typedef struct oc_instr { int16_t op, dst, a, b; double value; } oc_instr;
int oc_evaluate_program(int components, int arity, int nx, int ny, int nz, double hx, double hy, double hz,
                        const double* field, const oc_instr* prog, int n_instr, int kahan, double* result);

int oc_ch_rhs(int order, double M, double kappa, int nx, int ny, int nz, double hx,
              double hy, double hz, const double* psi, double* out);
/* integrator: 0 = explicit Euler, 1 = RK4.  psi advanced in place. */
int oc_ch_integrate(int order, double M, double kappa, int nx, int ny, int nz, double hx,
                    double hy, double hz, double* psi, double dt, int n_steps, int integrator);
double oc_ch_free_energy(int nx, int ny, int nz, double hx, double hy, double hz,
                         const double* psi, double kappa);
double oc_ch_gradient_energy(int nx, int ny, int nz, double hx, double hy, double hz,
                             const double* psi);
double oc_ch_mean(int nx, int ny, int nz, double hx, double hy, double hz, const double* psi);

/* Largest harmonic-mean face D over the +x/+y/+z faces (solve/Diffusion.hpp:187-207). */
double oc_d_max_face(int nx, int ny, int nz, const double* D);
int oc_diffuse_const(int nx, int ny, int nz, double hx, double hy, double hz, double* psi,
                     double D, double dt, int n_steps, int integrator);
int oc_diffuse_fvm(int nx, int ny, int nz, double hx, double hy, double hz, double* psi,
                   const double* D, double dt, int n_steps, int integrator);

#ifdef __cplusplus
}
#endif
#endif
