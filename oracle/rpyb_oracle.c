/*
 * CPU oracle (float64) -- TEST INFRASTRUCTURE ONLY; see rpyb_oracle.h.
 *
 * Each routine restates the reference algorithm step for step, in the same
 * order of floating-point operations, so that the oracle agrees with the
 * reference's own roughpy.compute build to the last few ulps:
 *   orc_ft_fma          roughpy_compute/dense/basic/free_tensor_fma.hpp:13-53
 *   orc_ft_inplace_mul  roughpy_compute/dense/basic/free_tensor_inplace_mul.hpp:13-87
 *   orc_ft_exp          roughpy_compute/dense/intermediate/free_tensor_exp.hpp:13-37
 *   orc_ft_fmexp        roughpy_compute/dense/intermediate/free_tensor_fmexp.hpp:15-40
 *   orc_ft_log          roughpy_compute/dense/intermediate/free_tensor_log.hpp:12-39
 *   orc_ft_antipode     roughpy_compute/dense/basic/free_tensor_antipode.hpp:50-100
 *   orc_ft_adjoint_left_mul roughpy_compute/dense/basic/free_tensor_adjoint_left_mul.hpp:11-77
 *   orc_signature       algebra/src/lite_context.h:542-563 (fmexp chain)
 */
#include "rpyb_oracle.h"

#include <stdlib.h>
#include <string.h>

#define ORC_MAX_DEPTH 32

typedef struct {
    int64_t db[ORC_MAX_DEPTH + 2];
    int width;
    int depth;
} Geom;

static void geom_init(Geom* g, int width, int depth)
{
    g->width = width;
    g->depth = depth;
    g->db[0] = 0;
    for (int i = 1; i <= depth + 1; ++i) g->db[i] = 1 + (int64_t)width * g->db[i - 1];
}

/* a view: data pointer with [min, max] degree bounds */
typedef struct {
    double* p;
    int mn, mx;
} View;

static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

static int clampmax(int m, int depth) { return (m < 0 || m > depth) ? depth : m; }

int64_t orc_tensor_size(int width, int depth)
{
    Geom g;
    geom_init(&g, width, depth);
    return g.db[depth + 1];
}

/* ft_fma: levels from the top down, lhs degree from high to low, rank-1 blocks */
static void fma_views(const Geom* g, View out, View lhs, View rhs)
{
    const int out_min = imax(1, out.mn);
    for (int od = out.mx; od >= out_min; --od) {
        const int lmax = imin(lhs.mx, od - rhs.mn);
        const int lmin = imax(lhs.mn, od - rhs.mx);
        double* of = out.p + g->db[od];
        for (int ld = lmax; ld >= lmin; --ld) {
            const int rd = od - ld;
            const double* lf = lhs.p + g->db[ld];
            const double* rf = rhs.p + g->db[rd];
            const int64_t ls = g->db[ld + 1] - g->db[ld];
            const int64_t rs = g->db[rd + 1] - g->db[rd];
            for (int64_t i = 0; i < ls; ++i)
                for (int64_t j = 0; j < rs; ++j) of[i * rs + j] += lf[i] * rf[j];
        }
    }
    if (out.mn == 0 && lhs.mn == 0 && rhs.mn == 0) out.p[0] += lhs.p[0] * rhs.p[0];
}

void orc_ft_fma(int width, int depth, double* out, const double* lhs, const double* rhs,
                const int32_t* bounds)
{
    Geom g;
    geom_init(&g, width, depth);
    int b[6] = {0, -1, 0, -1, 0, -1};
    if (bounds) for (int i = 0; i < 6; ++i) b[i] = bounds[i];
    View o = {out, b[0], clampmax(b[1], depth)};
    View l = {(double*)lhs, b[2], clampmax(b[3], depth)};
    View r = {(double*)rhs, b[4], clampmax(b[5], depth)};
    fma_views(&g, o, l, r);
}

/* in-place multiply with op(x) = x * scale applied to every term */
static void inplace_mul_views(const Geom* g, View lhs, View rhs, double scale)
{
    for (int od = lhs.mx; od >= imax(1, lhs.mn); --od) {
        const int ldmin = imax(lhs.mn, od - rhs.mx);
        const int ldmax = od - imax(1, rhs.mn);
        double* of = lhs.p + g->db[od];
        const int64_t os = g->db[od + 1] - g->db[od];
        if (rhs.mn == 0) {
            for (int64_t i = 0; i < os; ++i) of[i] = (of[i] * rhs.p[0]) * scale;
        } else {
            for (int64_t i = 0; i < os; ++i) of[i] = 0.0;
        }
        for (int ld = ldmax; ld >= ldmin; --ld) {
            const int rd = od - ld;
            const double* lf = lhs.p + g->db[ld];
            const double* rf = rhs.p + g->db[rd];
            const int64_t ls = g->db[ld + 1] - g->db[ld];
            const int64_t rs = g->db[rd + 1] - g->db[rd];
            for (int64_t i = 0; i < ls; ++i)
                for (int64_t j = 0; j < rs; ++j) of[i * rs + j] += (lf[i] * rf[j]) * scale;
        }
    }
    if (lhs.mn == 0 && rhs.mn == 0) lhs.p[0] = (lhs.p[0] * rhs.p[0]) * scale;
    else if (lhs.mn == 0) lhs.p[0] = 0.0;
}

void orc_ft_inplace_mul(int width, int depth, double* lhs, const double* rhs,
                        const int32_t* bounds, double scale)
{
    Geom g;
    geom_init(&g, width, depth);
    int b[4] = {0, -1, 0, -1};
    if (bounds) for (int i = 0; i < 4; ++i) b[i] = bounds[i];
    View l = {lhs, b[0], clampmax(b[1], depth)};
    View r = {(double*)rhs, b[2], clampmax(b[3], depth)};
    inplace_mul_views(&g, l, r, scale);
}

void orc_ft_exp(int width, int depth, double* out, const double* arg, int out_depth)
{
    Geom g;
    geom_init(&g, width, depth);
    const int M = clampmax(out_depth, depth);
    out[0] = 1.0;
    for (int deg = M; deg > 0; --deg) {
        const int ml = M - deg + 1;
        View o = {out, 0, ml};
        View a = {(double*)arg, 1, imin(M, ml)};
        inplace_mul_views(&g, o, a, 1.0 / (double)deg);
        out[0] += 1.0;
    }
}

void orc_ft_fmexp(int width, int depth, double* out, const double* mul, const double* expo,
                  int out_depth)
{
    Geom g;
    geom_init(&g, width, depth);
    const int M = clampmax(out_depth, depth);
    const int64_t n = g.db[M + 1];
    memcpy(out, mul, sizeof(double) * (size_t)n);
    for (int deg = M; deg > 0; --deg) {
        const int ml = M - deg + 1;
        View o = {out, 0, ml};
        View x = {(double*)expo, 1, imin(M, ml)};
        inplace_mul_views(&g, o, x, 1.0 / (double)deg);
        for (int64_t i = 0; i < n; ++i) out[i] += mul[i];
    }
}

void orc_ft_log(int width, int depth, double* out, const double* arg, int out_depth,
                int arg_depth)
{
    Geom g;
    geom_init(&g, width, depth);
    const int M = clampmax(out_depth, depth);
    const int Ma = clampmax(arg_depth, depth);
    for (int deg = M; deg > 0; --deg) {
        const int ml = M - deg + 1;
        if (deg % 2 == 0) out[0] -= 1.0 / (double)deg;
        else out[0] += 1.0 / (double)deg;
        View o = {out, 0, ml};
        View a = {(double*)arg, 1, imin(Ma, ml)};
        inplace_mul_views(&g, o, a, 1.0);
    }
}

void orc_ft_antipode(int width, int depth, double* out, const double* arg)
{
    Geom g;
    geom_init(&g, width, depth);
    out[0] = arg[0];
    for (int k = 1; k <= depth; ++k) {
        const int64_t n = g.db[k + 1] - g.db[k];
        const double sgn = (k % 2) ? -1.0 : 1.0;
        for (int64_t i = 0; i < n; ++i) {
            int64_t x = i, rev = 0;
            for (int q = 0; q < k; ++q) {
                rev = rev * width + x % width;
                x /= width;
            }
            out[g.db[k] + rev] = sgn * arg[g.db[k] + i];
        }
    }
}

void orc_ft_adjoint_left_mul(int width, int depth, double* out, const double* op,
                             const double* arg, int out_depth, int op_depth, int arg_depth)
{
    Geom g;
    geom_init(&g, width, depth);
    const int omax = clampmax(out_depth, depth);
    const int pmax = clampmax(op_depth, depth);
    const int amax = clampmax(arg_depth, depth);
    const int ahi = imin(amax - 0, omax);
    const int alo = imax(0 - pmax, 0);
    for (int ad = ahi; ad >= alo; --ad) {
        const int odmin = imax(ad - pmax, 0);
        const int odmax = imin(ad - 0, omax);
        const double* af = arg + g.db[ad];
        for (int od = odmax; od >= odmin; --od) {
            const int pd = ad - od;
            const double* pf = op + g.db[pd];
            double* of = out + g.db[od];
            const int64_t os = g.db[od + 1] - g.db[od];
            const int64_t ps = g.db[pd + 1] - g.db[pd];
            for (int64_t j = 0; j < ps; ++j) {
                const double v = pf[j];
                for (int64_t i = 0; i < os; ++i) of[i] += v * af[i + j * os];
            }
        }
    }
}

void orc_signature(int width, int depth, int64_t len, const double* inc, double* out)
{
    Geom g;
    geom_init(&g, width, depth);
    const int64_t n = g.db[depth + 1];
    memset(out, 0, sizeof(double) * (size_t)n);
    out[0] = 1.0;
    if (depth == 0) return;
    double* x = (double*)calloc((size_t)n, sizeof(double));
    double* tmp = (double*)malloc(sizeof(double) * (size_t)n);
    for (int64_t t = 0; t < len; ++t) {
        for (int a = 0; a < width; ++a) x[1 + a] = inc[t * width + a];
        orc_ft_fmexp(width, depth, tmp, out, x, -1);
        memcpy(out, tmp, sizeof(double) * (size_t)n);
    }
    free(tmp);
    free(x);
}
