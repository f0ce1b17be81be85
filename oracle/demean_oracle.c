/*
 * ORACLE -- test infrastructure only.  Nothing in the product links, loads or
 * calls this file; tests/, __graft_entry__.smoke() and the CPU-baseline leg of
 * bench.py use it as the checker.
 *
 * A plain-C, single-threaded restatement of the reference's CPU absorber for
 * the demeaning path (reisportela/xhdfe-xfe):
 *
 *   oracle_sweep        one Gauss-Seidel projection sweep: for each FE dim d
 *                       in `order`, v -= D_d (D_d' W D_d)^-1 D_d' W v on every
 *                       column (src/fe_absorption_cuda.cu:3070 run_demean,
 *                       CPU packed_demean_grouped src/fe_absorption.cpp:5718-5830)
 *   oracle_demean_map   the accelerated alternating-projection loop the
 *                       reference runs by default: Irons-Tuck extrapolation
 *                       with the "honest" stop ||G(gx)-gx|| <= tol*max(1,||gx||)
 *                       (src/fe_absorption.cpp:6598-6780 packed_accel_phase;
 *                       stats src/fe_absorption.cpp:5242-5268, update :5365-5392)
 *                       with the divergence safeguard (coef = 0 while the
 *                       post-sweep norm exceeds 4x its running minimum).
 *                       accel == 0 runs plain Gauss-Seidel sweeps and stops on
 *                       the same criterion.
 *   oracle_certify      the explicit normal-equation certificate
 *                       abs_residual = max_c ||D'W v~_c||_2 and
 *                       abs_residual_rel = max_c ||D'W v~_c|| / (||D'W||_F ||v_c||)
 *                       (src/fe_absorption.cpp:14942-15190)
 *
 * Arrays: v is column-major n x C (the outcome first), gids holds D arrays of
 * n dense ids back to back, G[d] the number of levels, w the weights or NULL.
 * Sums run in long double where the reference uses long double, else double.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static void group_means(int64_t n, const double* col, const int32_t* g, int32_t G,
                        const double* w, double* sum, double* wsum) {
    memset(sum, 0, sizeof(double) * (size_t)G);
    memset(wsum, 0, sizeof(double) * (size_t)G);
    for (int64_t i = 0; i < n; ++i) {
        const double wi = w ? w[i] : 1.0;
        sum[g[i]] += wi * col[i];
        wsum[g[i]] += wi;
    }
    for (int32_t k = 0; k < G; ++k) sum[k] = wsum[k] > 0.0 ? sum[k] / wsum[k] : 0.0;
}

/* One Gauss-Seidel sweep over the dims in `order` (NULL: 0..D-1). */
void oracle_sweep(int64_t n, int C, double* v, int D, const int32_t* gids, const int32_t* G,
                  const double* w, const int32_t* order) {
    int32_t Gmax = 1;
    for (int d = 0; d < D; ++d)
        if (G[d] > Gmax) Gmax = G[d];
    double* mean = (double*)malloc(sizeof(double) * (size_t)Gmax);
    double* wsum = (double*)malloc(sizeof(double) * (size_t)Gmax);
    for (int j = 0; j < D; ++j) {
        const int d = order ? order[j] : j;
        const int32_t* g = gids + (size_t)d * (size_t)n;
        for (int c = 0; c < C; ++c) {
            double* col = v + (size_t)c * (size_t)n;
            group_means(n, col, g, G[d], w, mean, wsum);
            for (int64_t i = 0; i < n; ++i) col[i] -= mean[g[i]];
        }
    }
    free(mean);
    free(wsum);
}

static double sumsq(const double* a, int64_t m) {
    double s = 0.0;
    for (int64_t i = 0; i < m; ++i) s += a[i] * a[i];
    return s;
}

/* Returns 1 when converged.  v is overwritten with the within transform. */
int oracle_demean_map(int64_t n, int C, double* v, int D, const int32_t* gids,
                      const int32_t* G, const double* w, const int32_t* order, double tol,
                      int max_iter, int accel, int* iters_out) {
    const int64_t m = n * (int64_t)C;
    int converged = 0;
    int it = 0;
    if (D == 0) {
        if (iters_out) *iters_out = 0;
        return 1;
    }
    if (!accel) {
        double* prev = (double*)malloc(sizeof(double) * (size_t)m);
        for (it = 0; it < max_iter; ++it) {
            memcpy(prev, v, sizeof(double) * (size_t)m);
            oracle_sweep(n, C, v, D, gids, G, w, order);
            double d1 = 0.0;
            for (int64_t i = 0; i < m; ++i) {
                const double d = v[i] - prev[i];
                d1 += d * d;
            }
            const double nv = sqrt(sumsq(v, m));
            if (sqrt(d1) <= tol * (nv > 1.0 ? nv : 1.0)) {
                converged = 1;
                ++it;
                break;
            }
        }
        free(prev);
        if (iters_out) *iters_out = it;
        return converged;
    }
    double* x = v; /* cur */
    double* gx = (double*)malloc(sizeof(double) * (size_t)m);
    double* ggx = (double*)malloc(sizeof(double) * (size_t)m);
    double prev_norm = sqrt(sumsq(x, m));
    double best = prev_norm;
    int suspended = 0;
    memcpy(gx, x, sizeof(double) * (size_t)m);
    oracle_sweep(n, C, gx, D, gids, G, w, order);
    for (it = 0; it < max_iter; ++it) {
        memcpy(ggx, gx, sizeof(double) * (size_t)m);
        oracle_sweep(n, C, ggx, D, gids, G, w, order);
        double vprod = 0.0, ssq = 0.0, d1sq = 0.0;
        for (int64_t i = 0; i < m; ++i) {
            const double dgx = ggx[i] - gx[i];
            const double d2 = dgx - gx[i] + x[i];
            vprod += dgx * d2;
            ssq += d2 * d2;
            d1sq += dgx * dgx;
        }
        if (sqrt(d1sq) <= tol * (prev_norm > 1.0 ? prev_norm : 1.0)) {
            memcpy(x, ggx, sizeof(double) * (size_t)m);
            converged = 1;
            ++it;
            break;
        }
        if (ssq == 0.0) {
            memcpy(x, gx, sizeof(double) * (size_t)m);
            converged = 1;
            ++it;
            break;
        }
        const double coef = suspended ? 0.0 : vprod / ssq;
        for (int64_t i = 0; i < m; ++i) {
            const double nx = ggx[i] - coef * (ggx[i] - gx[i]);
            x[i] = nx;
            gx[i] = nx;
        }
        oracle_sweep(n, C, gx, D, gids, G, w, order);
        const double cur = sqrt(sumsq(gx, m));
        prev_norm = cur;
        if (cur <= best) {
            best = cur;
            suspended = 0;
        } else if (cur > 4.0 * best) {
            suspended = 1;
        }
    }
    if (!converged) memcpy(x, gx, sizeof(double) * (size_t)m);
    free(gx);
    free(ggx);
    if (iters_out) *iters_out = it;
    return converged;
}

void oracle_certify(int64_t n, int C, const double* v_orig, const double* v_tilde, int D,
                    const int32_t* gids, const int32_t* G, const double* w, double* abs_out,
                    double* rel_out) {
    long double opn = 0.0L;
    long double* res = (long double*)calloc((size_t)C, sizeof(long double));
    int32_t Gmax = 1;
    for (int d = 0; d < D; ++d)
        if (G[d] > Gmax) Gmax = G[d];
    double* s = (double*)malloc(sizeof(double) * (size_t)Gmax);
    for (int d = 0; d < D; ++d) {
        const int32_t* g = gids + (size_t)d * (size_t)n;
        for (int64_t i = 0; i < n; ++i) {
            const double wi = w ? w[i] : 1.0;
            opn += (long double)(wi * wi);
        }
        for (int c = 0; c < C; ++c) {
            const double* col = v_tilde + (size_t)c * (size_t)n;
            memset(s, 0, sizeof(double) * (size_t)G[d]);
            for (int64_t i = 0; i < n; ++i) s[g[i]] += (w ? w[i] : 1.0) * col[i];
            double q = 0.0;
            for (int32_t k = 0; k < G[d]; ++k) q += s[k] * s[k];
            res[c] += (long double)q;
        }
    }
    double amax = 0.0, rmax = 0.0;
    const double opnorm = sqrt((double)opn);
    for (int c = 0; c < C; ++c) {
        const double a = sqrt((double)(res[c] > 0 ? res[c] : 0));
        const double on = sqrt(sumsq(v_orig + (size_t)c * (size_t)n, n));
        const double sc = opnorm * on;
        double r = 0.0;
        if (sc > 0.0) r = a / sc;
        else if (a > 0.0) r = 1.7976931348623157e308;
        if (a > amax) amax = a;
        if (r > rmax) rmax = r;
    }
    free(s);
    free(res);
    *abs_out = amax;
    *rel_out = rmax;
}

/* Tightly converged projection for pinning: IT-MAP to `tol` (e.g. 1e-14). */
int oracle_project(int64_t n, int C, double* v, int D, const int32_t* gids, const int32_t* G,
                   const double* w, double tol, int max_iter, int* iters_out) {
    return oracle_demean_map(n, C, v, D, gids, G, w, NULL, tol, max_iter, 1, iters_out);
}
