/*
 * CPU oracle for the B200 tensor-algebra library -- TEST INFRASTRUCTURE ONLY.
 *
 * A float64 restatement, in plain C, of RoughPy's dense free-tensor
 * algorithms (roughpy_compute/ headers).  Only the test suite, the smoke
 * check and the CPU-baseline leg of the benchmark load it, and only as the
 * checker.  The product library never links or calls it.
 *
 * Pinned against: golden vectors generated by the reference's own
 * `roughpy.compute` extension (built from its sources by oracle/Makefile,
 * fixtures in tests/golden/), and the known-answer tests in the reference's
 * tests/compute suite.
 *
 * Layout: degree-major dense tensors, degree_begin[k] = (w^k - 1)/(w - 1).
 * Degree bounds: max = -1 means depth; min defaults to 0.
 */
#ifndef RPYB_ORACLE_H
#define RPYB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

int64_t orc_tensor_size(int width, int depth);

/* out += lhs * rhs; bounds = {out_min,out_max,lhs_min,lhs_max,rhs_min,rhs_max} or NULL */
void orc_ft_fma(int width, int depth, double* out, const double* lhs, const double* rhs,
                const int32_t* bounds);
/* lhs <- scale * (lhs * rhs); bounds = {lhs_min,lhs_max,rhs_min,rhs_max} or NULL */
void orc_ft_inplace_mul(int width, int depth, double* lhs, const double* rhs,
                        const int32_t* bounds, double scale);
void orc_ft_exp(int width, int depth, double* out, const double* arg, int out_depth);
void orc_ft_fmexp(int width, int depth, double* out, const double* mul, const double* expo,
                  int out_depth);
/* out must hold its incoming contents (zeros for the plain logarithm) */
void orc_ft_log(int width, int depth, double* out, const double* arg, int out_depth,
                int arg_depth);
void orc_ft_antipode(int width, int depth, double* out, const double* arg);
void orc_ft_adjoint_left_mul(int width, int depth, double* out, const double* op,
                             const double* arg, int out_depth, int op_depth, int arg_depth);
/* Chen product of exp(x_t) over `len` rows of `width` increments (fmexp chain). */
void orc_signature(int width, int depth, int64_t len, const double* inc, double* out);

#ifdef __cplusplus
}
#endif

#endif
