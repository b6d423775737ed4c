/*
 * grav_oracle.c -- CPU restatement of StarSmasher's FP64 gravity path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests,
 * the smoke check and the CPU-baseline leg of the benchmark load it.  The
 * GPU library never links or calls it, and nothing in the product path falls
 * back to it.
 *
 * What it restates (paths relative to the reference project):
 *   parallel_bleeding_edge/src/cpu_grav.f:1-381   get_gravity_using_cpus
 *       FP64 triangle j >= i with Newton's third law (massratio = m_i/m_j),
 *       the three softening kernels (nkernel 0 cubic spline :43-158,
 *       1 Wendland C6 :159-269, 2 Wendland C4 :270-376) and the zero-distance
 *       rule (:138-145, :249-256, :356-363).
 *   parallel_bleeding_edge/src/main.f:296-349       gravquant
 *       the split of the triangle's rows over workers by interaction count
 *       (here: OpenMP threads instead of MPI ranks; thread-private
 *       accumulators summed at the end in thread order, like mpi_reduce at
 *       balAV3.f:436-442).
 *   parallel_bleeding_edge/src/grav.f:15-18
 *       the caller's softening convention: range2 = 4 hp^2, negated for
 *       point masses (u == 0).  The oracle takes range2 like the GPU ABI and
 *       recovers twohp = sqrt(|range2|) (exact: sqrt(fl(x*x)) == |x| in IEEE
 *       double), fourhp2 = |range2| and the point-mass flag range2 > 0.
 *
 * Two drivers:
 *   oracle_triangle  -- the faithful CPU algorithm (timed CPU baseline).
 *   oracle_rows      -- per-row full j loop, same pair formulas evaluated from
 *                       the row particle's side, Neumaier-compensated sums;
 *                       the error oracle (rows can be a subset, so it also
 *                       scales to N = 1,048,576).
 *
 * Zero-distance rule, stated for one row a receiving from source b with
 * r2 == 0 (what the triangle produces, cpu_grav.f:138-145, :149-156):
 *   b == a : -c   * flag_a           * (m_a/H_a + m_a/H_a)   (added twice)
 *   b != a : -c/2 * flag_{min(a,b)}  * (m_b/H_a + m_b/H_b)
 * with c = 1.4, 1.9140625, 1.71875 for nkernel 0, 1, 2 and H = 2 hp.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_OK 0
#define ORACLE_EINVAL 1
#define ORACLE_ENOMEM 2

static const double SELF_C[3] = {1.4, 1.9140625, 1.71875};

/* Near-field pair (r2 < max(H_i^2, H_j^2)), cpu_grav.f:71-157 (nkernel 0),
 * :187-268 (1), :298-375 (2).  Returns gacc (multiplies dr) and gpot.  The
 * r2 == 0 case is left to the caller (it depends on which side is lower). */
static inline void near_pair(int nkernel, double r2, double rinv,
                             double amj, double twohpi, double fourhpi2,
                             double twohpj, double fourhpj2,
                             double mrinv1, double mrinv3,
                             double *gacc, double *gpot)
{
    double invq1, invq2, qq1, qq2;
    invq1 = rinv * twohpi;
    invq2 = rinv * twohpj;
    qq1 = 1.0 / invq1;
    qq2 = 1.0 / invq2;
    double q21 = qq1 * qq1, q22 = qq2 * qq2;
    double q31 = qq1 * q21, q32 = qq2 * q22;
    double invq21 = invq1 * invq1, invq22 = invq2 * invq2;
    double invq31 = invq1 * invq21, invq32 = invq2 * invq22;
    double mj11 = amj / twohpi, mj12 = amj / twohpj;
    double mj21 = mj11 / fourhpi2, mj22 = mj12 / fourhpj2;
    double g1 = (r2 <= fourhpi2) ? 1.0 : 0.0;
    double g2 = (r2 <= fourhpj2) ? 1.0 : 0.0;
    double acc1, acc2, pot1, pot2;
    if (nkernel == 0) {
        /* cubic spline, cpu_grav.f:91-118 */
        if (qq1 < 0.5) {
            acc1 = 10.666666666667 + q21 * (32.0 * qq1 - 38.4);
            pot1 = -2.8 + q21 * (5.333333333333 + q21 * (6.4 * qq1 - 9.6));
        } else {
            acc1 = 21.333333333333 - 48.0 * qq1 + 38.4 * q21
                 - 10.666666666667 * q31 - 0.066666666667 * invq31;
            pot1 = -3.2 + 0.066666666667 * invq1
                 + q21 * (10.666666666667 + qq1 * (-16.0 + qq1 * (9.6 - 2.133333333333 * qq1)));
        }
        if (qq2 < 0.5) {
            acc2 = 10.666666666667 + q22 * (32.0 * qq2 - 38.4);
            pot2 = -2.8 + q22 * (5.333333333333 + q22 * (6.4 * qq2 - 9.6));
        } else {
            acc2 = 21.333333333333 - 48.0 * qq2 + 38.4 * q22
                 - 10.666666666667 * q32 - 0.066666666667 * invq32;
            pot2 = -3.2 + 0.066666666667 * invq2
                 + q22 * (10.666666666667 + qq2 * (-16.0 + qq2 * (9.6 - 2.133333333333 * qq2)));
        }
        *gacc = 0.5 * (g1 * mj21 * acc1 + (1.0 - g1) * mrinv3 + g2 * mj22 * acc2 + (1.0 - g2) * mrinv3);
        *gpot = 0.5 * (g1 * mj11 * pot1 + (g1 - 1.0) * mrinv1 + g2 * mj12 * pot2 + (g2 - 1.0) * mrinv1);
    } else if (nkernel == 1) {
        /* Wendland C6 (3,3), cpu_grav.f:210-248 */
        acc1 = 28.4375 + q21 * ((-187.6875) + q21 * (804.375 + q21 * ((-4379.375) + qq1 * (9009.0 + qq1 * ((-8957.8125) + qq1 * (5005.0 + qq1 * ((-1515.9375) + 195.0 * qq1)))))));
        acc2 = 28.4375 + q22 * ((-187.6875) + q22 * (804.375 + q22 * ((-4379.375) + qq2 * (9009.0 + qq2 * ((-8957.8125) + qq2 * (5005.0 + qq2 * ((-1515.9375) + 195.0 * qq2)))))));
        pot1 = g1 > 0.0 ? (-3.828125) + q21 * (14.21875 + q21 * ((-46.921875) + q21 * (134.0625 + q21 * ((-547.421875) + qq1 * (1001.0 + qq1 * ((-895.78125) + qq1 * (455.0 + qq1 * ((-126.328125) + 15.0 * qq1)))))))) : 0.0;
        pot2 = g2 > 0.0 ? (-3.828125) + q22 * (14.21875 + q22 * ((-46.921875) + q22 * (134.0625 + q22 * ((-547.421875) + qq2 * (1001.0 + qq2 * ((-895.78125) + qq2 * (455.0 + qq2 * ((-126.328125) + 15.0 * qq2)))))))) : 0.0;
        *gacc = 0.5 * (g1 * mj21 * acc1 + (1.0 - g1) * mrinv3 + g2 * mj22 * acc2 + (1.0 - g2) * mrinv3);
        *gpot = 0.5 * (mj11 * pot1 + (g1 - 1.0) * mrinv1 + mj12 * pot2 + (g2 - 1.0) * mrinv1);
    } else {
        /* Wendland C4, cpu_grav.f:321-355 */
        acc1 = 20.625 + q21 * ((-115.5) + q21 * (618.75 + qq1 * ((-1155.0) + qq1 * (962.5 + qq1 * ((-396.0) + 65.625 * qq1)))));
        acc2 = 20.625 + q22 * ((-115.5) + q22 * (618.75 + qq2 * ((-1155.0) + qq2 * (962.5 + qq2 * ((-396.0) + 65.625 * qq2)))));
        pot1 = g1 > 0.0 ? (-3.4375) + q21 * (10.3125 + q21 * ((-28.875) + q21 * (103.125 + qq1 * ((-165.0) + qq1 * (120.3125 + qq1 * ((-44.0) + 6.5625 * qq1)))))) : 0.0;
        pot2 = g2 > 0.0 ? (-3.4375) + q22 * (10.3125 + q22 * ((-28.875) + q22 * (103.125 + qq2 * ((-165.0) + qq2 * (120.3125 + qq2 * ((-44.0) + 6.5625 * qq2)))))) : 0.0;
        *gacc = 0.5 * (g1 * mj21 * acc1 + (1.0 - g1) * mrinv3 + g2 * mj22 * acc2 + (1.0 - g2) * mrinv3);
        *gpot = 0.5 * (mj11 * pot1 + (g1 - 1.0) * mrinv1 + mj12 * pot2 + (g2 - 1.0) * mrinv1);
    }
}

static int check_inputs(int n, const double *m, const double *range2, int nkernel)
{
    if (n < 0 || nkernel < 0 || nkernel > 2) return ORACLE_EINVAL;
    for (int i = 0; i < n; i++)
        if (!(m[i] > 0.0) || range2[i] == 0.0 || isnan(range2[i])) return ORACLE_EINVAL;
    return ORACLE_OK;
}

/* gravquant (main.f:296-349): row boundaries so that worker k gets about
 * n(n+1)/2/nworkers triangle interactions over rows [lo, hi).  Here the row
 * range is [i_lo, i_hi) of a possibly partial triangle; rows are 0-based. */
static void split_triangle_rows(int n, int i_lo, int i_hi, int nworkers, int *bounds)
{
    double total = 0.0;
    for (int i = i_lo; i < i_hi; i++) total += (double)(n - i);
    bounds[0] = i_lo;
    int w = 0;
    double acc = 0.0;
    for (int i = i_lo; i < i_hi && w < nworkers - 1; i++) {
        acc += (double)(n - i);
        if (acc + (double)((n - i - 1) / 2) >= (w + 1.0) * total / nworkers) {
            bounds[++w] = i + 1;
        }
    }
    while (w < nworkers - 1) bounds[++w] = i_hi;
    bounds[nworkers] = i_hi;
}

/*
 * Faithful triangle (cpu_grav.f:17-378).  Rows [i_lo, i_hi) (0-based) are
 * processed; each pair (i, j >= i) updates i and j.  Outputs are zeroed over
 * the whole length n first (cpu_grav.f:17-22) and hold the sum over all
 * workers.  Returns 0, or an error code for invalid input.
 */
int oracle_triangle(int n, const double *x, const double *y, const double *z,
                    const double *m, const double *range2, int nkernel,
                    int i_lo, int i_hi, int nthreads,
                    double *gx, double *gy, double *gz, double *grpot)
{
    int rc = check_inputs(n, m, range2, nkernel);
    if (rc) return rc;
    if (i_lo < 0 || i_hi > n || i_lo > i_hi) return ORACLE_EINVAL;
    if (nthreads < 1) nthreads = 1;
    for (int i = 0; i < n; i++) { gx[i] = gy[i] = gz[i] = grpot[i] = 0.0; }
    if (i_hi == i_lo) return ORACLE_OK;
    if (nthreads > i_hi - i_lo) nthreads = i_hi - i_lo;

    const double cself = SELF_C[nkernel];
    const size_t span = (size_t)(n - i_lo);      /* j only reaches [i_lo, n) */
    double *priv = (double *)malloc(sizeof(double) * 4 * span * (size_t)nthreads);
    int *bounds = (int *)malloc(sizeof(int) * (nthreads + 1));
    if (!priv || !bounds) { free(priv); free(bounds); return ORACLE_ENOMEM; }
    split_triangle_rows(n, i_lo, i_hi, nthreads, bounds);

#pragma omp parallel num_threads(nthreads)
    {
#ifdef _OPENMP
        int t = omp_get_thread_num();
#else
        int t = 0;
#endif
        double *px = priv + (size_t)t * 4 * span;
        double *py = px + span, *pz = py + span, *pp = pz + span;
        memset(px, 0, sizeof(double) * 4 * span);
        for (int i = bounds[t]; i < bounds[t + 1]; i++) {
            const double ami = m[i];
            const double fourhpi2 = fabs(range2[i]);
            const double twohpi = sqrt(fourhpi2);
            const int ui = range2[i] > 0.0;
            const size_t ii = (size_t)(i - i_lo);
            for (int j = i; j < n; j++) {
                const size_t jj = (size_t)(j - i_lo);
                double dr1 = x[j] - x[i];
                double dr2 = y[j] - y[i];
                double dr3 = z[j] - z[i];
                double r2 = dr1 * dr1 + dr2 * dr2 + dr3 * dr3;
                double rinv = 1.0 / sqrt(r2);
                double rinv2 = rinv * rinv;
                double amj = m[j];
                double fourhpj2 = fabs(range2[j]);
                double twohpj = sqrt(fourhpj2);
                double massratio = ami / amj;
                double mrinv1 = rinv * amj;
                double mrinv3 = rinv2 * mrinv1;
                double gacc, gpot;
                if (r2 >= fmax(fourhpi2, fourhpj2)) {
                    gacc = mrinv3;
                    gpot = -mrinv1;
                } else if (r2 > 0.0) {
                    near_pair(nkernel, r2, rinv, amj, twohpi, fourhpi2, twohpj, fourhpj2,
                              mrinv1, mrinv3, &gacc, &gpot);
                } else {
                    gacc = 0.0;
                    gpot = ui ? -0.5 * cself * (amj / twohpi + amj / twohpj) : 0.0;
                }
                double dgx = gacc * dr1, dgy = gacc * dr2, dgz = gacc * dr3;
                px[ii] += dgx; px[jj] -= dgx * massratio;
                py[ii] += dgy; py[jj] -= dgy * massratio;
                pz[ii] += dgz; pz[jj] -= dgz * massratio;
                pp[ii] += gpot; pp[jj] += gpot * massratio;
            }
        }
    }
    /* reduce in worker order (deterministic, like mpi_reduce) */
    for (int t = 0; t < nthreads; t++) {
        const double *px = priv + (size_t)t * 4 * span;
        const double *py = px + span, *pz = py + span, *pp = pz + span;
        for (size_t k = 0; k < span; k++) {
            gx[i_lo + k] += px[k]; gy[i_lo + k] += py[k];
            gz[i_lo + k] += pz[k]; grpot[i_lo + k] += pp[k];
        }
    }
    free(priv);
    free(bounds);
    return ORACLE_OK;
}

/* Neumaier compensated accumulator */
typedef struct { double s, c; } nsum;
static inline void nadd(nsum *a, double v)
{
    double t = a->s + v;
    if (fabs(a->s) >= fabs(v)) a->c += (a->s - t) + v;
    else a->c += (v - t) + a->s;
    a->s = t;
}

/*
 * Row form: for each listed row a (0-based), sum over all j of the pair
 * contribution of j to a, evaluated from a's side with the cpu_grav.f pair
 * formulas, Neumaier-compensated.  Equal to the triangle up to rounding.
 */
int oracle_rows(int n, const double *x, const double *y, const double *z,
                const double *m, const double *range2, int nkernel,
                int nrows, const int *rows, int nthreads,
                double *ax, double *ay, double *az, double *pot)
{
    int rc = check_inputs(n, m, range2, nkernel);
    if (rc) return rc;
    for (int k = 0; k < nrows; k++) if (rows[k] < 0 || rows[k] >= n) return ORACLE_EINVAL;
    if (nthreads < 1) nthreads = 1;
    const double cself = SELF_C[nkernel];

#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 4)
    for (int k = 0; k < nrows; k++) {
        const int i = rows[k];
        const double fourhpi2 = fabs(range2[i]);
        const double twohpi = sqrt(fourhpi2);
        nsum sx = {0, 0}, sy = {0, 0}, sz = {0, 0}, sp = {0, 0};
        for (int j = 0; j < n; j++) {
            double dr1 = x[j] - x[i];
            double dr2 = y[j] - y[i];
            double dr3 = z[j] - z[i];
            double r2 = dr1 * dr1 + dr2 * dr2 + dr3 * dr3;
            double amj = m[j];
            double fourhpj2 = fabs(range2[j]);
            double twohpj = sqrt(fourhpj2);
            double gacc, gpot;
            if (r2 >= fmax(fourhpi2, fourhpj2)) {
                double rinv = 1.0 / sqrt(r2);
                double mrinv1 = rinv * amj;
                gacc = rinv * rinv * mrinv1;
                gpot = -mrinv1;
            } else if (r2 > 0.0) {
                double rinv = 1.0 / sqrt(r2);
                double mrinv1 = rinv * amj;
                double mrinv3 = rinv * rinv * mrinv1;
                near_pair(nkernel, r2, rinv, amj, twohpi, fourhpi2, twohpj, fourhpj2,
                          mrinv1, mrinv3, &gacc, &gpot);
            } else {
                gacc = 0.0;
                if (j == i) {
                    gpot = range2[i] > 0.0 ? -cself * (amj / twohpi + amj / twohpj) : 0.0;
                } else {
                    int lo = i < j ? i : j;
                    gpot = range2[lo] > 0.0 ? -0.5 * cself * (amj / twohpi + amj / twohpj) : 0.0;
                }
            }
            nadd(&sx, gacc * dr1);
            nadd(&sy, gacc * dr2);
            nadd(&sz, gacc * dr3);
            nadd(&sp, gpot);
        }
        ax[k] = sx.s + sx.c;
        ay[k] = sy.s + sy.c;
        az[k] = sz.s + sz.c;
        pot[k] = sp.s + sp.c;
    }
    return ORACLE_OK;
}

/* Row split of the GPU path across gravity ranks, main.f:283-295:
 * gravstride = (n-1)/nranks + 1; rank r owns 1-based rows
 * [gravstride*r + 1, min(gravstride*(r+1), n)].  Writes 0-based [lo, hi). */
void oracle_gpu_row_split(int n, int nranks, int rank, int *lo, int *hi)
{
    int stride = (n - 1) / nranks + 1;
    int l = stride * rank;
    int h = l + stride;
    if (h > n) h = n;
    if (l > n) l = n;
    *lo = l;
    *hi = h;
}

/* Triangle row split across CPU gravity ranks (main.f:296-349), 0-based
 * bounds[0..nranks]. */
void oracle_cpu_row_split(int n, int nranks, int *bounds)
{
    split_triangle_rows(n, 0, n, nranks, bounds);
}

int oracle_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
