// sg_internal.cuh -- shared layout, device helpers and the FP64 pair formulas
// of the B200 gravity library.  Paths in citations are inside the reference
// project (StarSmasher).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sg {

// ------------------------------------------------------------------ layout
constexpr int META_J = 64;        // particles per j-tile metadata record
constexpr int PAD_J = 256;        // per-set padding of the sorted arrays
constexpr double FAR_POS = 1.0e15;  // position of padding slots (mass 0)
constexpr int MAX_SETS = 1 << 20;

// One independent particle set (one star model / collision snapshot).
struct SetDesc {
    int n;         // particles in the set
    int off;       // first particle in the caller's concatenated arrays
    int poff;      // first slot of the set in the padded sorted arrays
    int npad;      // padded length (multiple of PAD_J)
    int ioff;      // first entry of the set's rows in the row list
    int ni;        // rows computed for this set
    int i_lo;      // rows are set-local original indices [i_lo, i_lo + ni)
    int tile_off;  // first i-tile of the set (global i-tile index)
    int ntiles;    // i-tiles of the set
    int meta_off;  // first j metadata record of the set
    int slot_off;  // first partial slot of the set (refine plans: of its items)
    int nchunks;   // j-chunks per i-tile (the main plan: the most of any tile)
    int light_off; // refine plans, sets with few listed rows: first row-chunk item
    int light_nch; // ... and source chunks per row (0: the set's rows use tiles)
};

// One unit of the persistent kernels' device-side queue.
struct WorkItem {
    int set;     // set index
    int tile;    // set-local i-tile
    int jb, je;  // set-local sorted slots [jb, je), multiples of the j-tile
    int chunk;   // j-chunk index within the i-tile
    int slot;    // partial-sum slot of this item
    int pad_[2];
};

// Padded, spatially sorted SoA copies of the inputs.
struct SortedF64 {
    double *x, *y, *z, *m, *h2;  // h2 = |range2| = H^2 with H = 2 hp
    int *orig;                   // global index in the caller's arrays (-1: pad)
    unsigned char *flag;         // range2 > 0 (the particle has self-potential)
};
struct SortedF32 {
    float *xh, *xl, *yh, *yl, *zh, *zl;  // hi + lo float pairs of the FP64 positions
    float *m, *h2;
};
// Bounding box and largest H^2 of META_J consecutive sorted slots.
struct JMeta {
    float cx, cy, cz;   // box centre
    float ex, ey, ez;   // half extents (negative: no particle)
    float h2max;
    float pad_;
};
// Centre of an i-tile's bounding box as float hi + lo pairs.
struct ITileMeta {
    float chx, chy, chz, clx, cly, clz;
    float pad_[2];
};

// Error flag bits written by device code.
enum : int {
    DEVERR_INPUT = 1,
    DEVERR_TIMEOUT = 2,
    DEVERR_TREE = 4,  // tree walk: traversal stack full
    DEVERR_TREE_CAP = 8,  // captured tree call: node array or heavy-group list full
};

// Self-potential constants c of the zero-distance rule (cpu_grav.f:141,
// :252, :359 use c/2 because the triangle adds the self pair twice).
__host__ __device__ inline double self_c(int nkernel)
{
    return nkernel == 0 ? 1.4 : (nkernel == 1 ? 1.9140625 : 1.71875);
}

// ------------------------------------------------------ FP64 pair formulas
// Contribution of source j to row i, evaluated from i's side in FP64 with the
// cpu_grav.f formulas (far: :59-70; near: :71-157 / :187-268 / :298-375).
// dr = x_j - x_i.  r2 == 0 uses the triangle's zero-distance rule restated
// per row: i == j gives -c*flag_i*(m/H_i + m/H_j); distinct coincident
// particles give -c/2 * flag_{lower original index} * (m_j/H_i + m_j/H_j).
struct PairOut { double ax, ay, az, pot; };

// The near-field pair evaluated with the CPU path's operations in the CPU
// path's order (cpu_grav.f:71-157 nkernel 0, :187-268 nkernel 1, :298-375
// nkernel 2): every product, sum, quotient and square root is an explicit
// IEEE round-to-nearest operation (no contraction into FMA), so a near pair
// gives the same bits as the CPU path does for the same r2, rinv, H.  Near
// pairs are rare (r < max H), so their cost does not matter, and near q = 1
// the kernel polynomials cancel by up to ~1e4: a last-bit difference in
// their inputs would otherwise show as a ~1e-12 relative difference on a
// particle whose acceleration cancels.
#define SG_M(a, b) __dmul_rn((a), (b))
#define SG_A(a, b) __dadd_rn((a), (b))
#define SG_S(a, b) __dsub_rn((a), (b))
#define SG_D(a, b) __ddiv_rn((a), (b))

__device__ __forceinline__ void near_kernel_f64(int nkernel, double r2, double rinv, double amj,
                                                double twohpi, double fourhpi2, double twohpj,
                                                double fourhpj2, double mrinv1, double mrinv3,
                                                double &gacc, double &gpot)
{
    const double invq1 = SG_M(rinv, twohpi), invq2 = SG_M(rinv, twohpj);
    const double qq1 = SG_D(1.0, invq1), qq2 = SG_D(1.0, invq2);
    const double q21 = SG_M(qq1, qq1), q22 = SG_M(qq2, qq2);
    const double q31 = SG_M(qq1, q21), q32 = SG_M(qq2, q22);
    const double invq21 = SG_M(invq1, invq1), invq22 = SG_M(invq2, invq2);
    const double invq31 = SG_M(invq1, invq21), invq32 = SG_M(invq2, invq22);
    const double mj11 = SG_D(amj, twohpi), mj12 = SG_D(amj, twohpj);
    const double mj21 = SG_D(mj11, fourhpi2), mj22 = SG_D(mj12, fourhpj2);
    const double g1 = (r2 <= fourhpi2) ? 1.0 : 0.0;
    const double g2 = (r2 <= fourhpj2) ? 1.0 : 0.0;
    double acc1, acc2, pot1, pot2;
    // 0.5 * (g1 mj21 acc1 + (1 - g1) mrinv3 + g2 mj22 acc2 + (1 - g2) mrinv3), left to right
    auto gsum = [&](double a1, double a2, double w1, double w2, double far1, double far2) {
        double t = SG_M(SG_M(g1, w1), a1);
        t = SG_A(t, far1);
        t = SG_A(t, SG_M(SG_M(g2, w2), a2));
        t = SG_A(t, far2);
        return SG_M(0.5, t);
    };
    if (nkernel == 0) {
        auto spline = [&](double q, double q2, double q3, double iq, double iq3, double &acc, double &pot) {
            if (q < 0.5) {
                acc = SG_A(10.666666666667, SG_M(q2, SG_S(SG_M(32.0, q), 38.4)));
                pot = SG_A(-2.8, SG_M(q2, SG_A(5.333333333333, SG_M(q2, SG_S(SG_M(6.4, q), 9.6)))));
            } else {
                double a = SG_S(21.333333333333, SG_M(48.0, q));
                a = SG_A(a, SG_M(38.4, q2));
                a = SG_S(a, SG_M(10.666666666667, q3));
                acc = SG_S(a, SG_M(0.066666666667, iq3));
                const double inner =
                    SG_A(10.666666666667,
                         SG_M(q, SG_A(-16.0, SG_M(q, SG_S(9.6, SG_M(2.133333333333, q))))));
                pot = SG_A(SG_A(-3.2, SG_M(0.066666666667, iq)), SG_M(q2, inner));
            }
        };
        spline(qq1, q21, q31, invq1, invq31, acc1, pot1);
        spline(qq2, q22, q32, invq2, invq32, acc2, pot2);
        gacc = gsum(acc1, acc2, mj21, mj22, SG_M(SG_S(1.0, g1), mrinv3), SG_M(SG_S(1.0, g2), mrinv3));
        double t = SG_M(SG_M(g1, mj11), pot1);
        t = SG_A(t, SG_M(SG_S(g1, 1.0), mrinv1));
        t = SG_A(t, SG_M(SG_M(g2, mj12), pot2));
        t = SG_A(t, SG_M(SG_S(g2, 1.0), mrinv1));
        gpot = SG_M(0.5, t);
    } else {
        auto wend = [&](double q, double q2, double g, double &acc, double &pot) {
            if (nkernel == 1) {
                double a = SG_A(-1515.9375, SG_M(195.0, q));
                a = SG_A(5005.0, SG_M(q, a));
                a = SG_A(-8957.8125, SG_M(q, a));
                a = SG_A(9009.0, SG_M(q, a));
                a = SG_A(-4379.375, SG_M(q, a));
                a = SG_A(804.375, SG_M(q2, a));
                a = SG_A(-187.6875, SG_M(q2, a));
                acc = SG_A(28.4375, SG_M(q2, a));
                double p = SG_A(-126.328125, SG_M(15.0, q));
                p = SG_A(455.0, SG_M(q, p));
                p = SG_A(-895.78125, SG_M(q, p));
                p = SG_A(1001.0, SG_M(q, p));
                p = SG_A(-547.421875, SG_M(q, p));
                p = SG_A(134.0625, SG_M(q2, p));
                p = SG_A(-46.921875, SG_M(q2, p));
                p = SG_A(14.21875, SG_M(q2, p));
                pot = g > 0.0 ? SG_A(-3.828125, SG_M(q2, p)) : 0.0;
            } else {
                double a = SG_A(-396.0, SG_M(65.625, q));
                a = SG_A(962.5, SG_M(q, a));
                a = SG_A(-1155.0, SG_M(q, a));
                a = SG_A(618.75, SG_M(q, a));
                a = SG_A(-115.5, SG_M(q2, a));
                acc = SG_A(20.625, SG_M(q2, a));
                double p = SG_A(-44.0, SG_M(6.5625, q));
                p = SG_A(120.3125, SG_M(q, p));
                p = SG_A(-165.0, SG_M(q, p));
                p = SG_A(103.125, SG_M(q, p));
                p = SG_A(-28.875, SG_M(q2, p));
                p = SG_A(10.3125, SG_M(q2, p));
                pot = g > 0.0 ? SG_A(-3.4375, SG_M(q2, p)) : 0.0;
            }
        };
        wend(qq1, q21, g1, acc1, pot1);
        wend(qq2, q22, g2, acc2, pot2);
        gacc = gsum(acc1, acc2, mj21, mj22, SG_M(SG_S(1.0, g1), mrinv3), SG_M(SG_S(1.0, g2), mrinv3));
        double t = SG_M(mj11, pot1);
        t = SG_A(t, SG_M(SG_S(g1, 1.0), mrinv1));
        t = SG_A(t, SG_M(mj12, pot2));
        t = SG_A(t, SG_M(SG_S(g2, 1.0), mrinv1));
        gpot = SG_M(0.5, t);
    }
}

// FP64 pair of row slot ip and source slot jp given their separation dr
// (x_j - x_i), the source mass and both H^2; the zero-distance rule reads
// the flags and original indices of the sorted layout.  Evaluated like the
// CPU path's row form: r2 summed without contraction, rinv = 1/sqrt(r2),
// twohp = sqrt(H^2).
static __device__ __forceinline__ PairOut pair_f64_core(const SortedF64 &D, int nkernel, int ip,
                                                        int jp, double dr1, double dr2, double dr3,
                                                        double amj, double fourhpi2,
                                                        double fourhpj2)
{
    const double r2 = SG_A(SG_A(SG_M(dr1, dr1), SG_M(dr2, dr2)), SG_M(dr3, dr3));
    double gacc, gpot;
    if (r2 >= fmax(fourhpi2, fourhpj2)) {
        const double rinv = SG_D(1.0, __dsqrt_rn(r2));
        const double mrinv1 = SG_M(rinv, amj);
        gacc = SG_M(SG_M(rinv, rinv), mrinv1);
        gpot = -mrinv1;
    } else if (r2 > 0.0) {
        const double rinv = SG_D(1.0, __dsqrt_rn(r2));
        const double mrinv1 = SG_M(rinv, amj);
        const double mrinv3 = SG_M(SG_M(rinv, rinv), mrinv1);
        near_kernel_f64(nkernel, r2, rinv, amj, __dsqrt_rn(fourhpi2), fourhpi2,
                        __dsqrt_rn(fourhpj2), fourhpj2, mrinv1, mrinv3, gacc, gpot);
    } else {
        gacc = 0.0;
        const double twohpi = __dsqrt_rn(fourhpi2), twohpj = __dsqrt_rn(fourhpj2);
        const double s = SG_A(SG_D(amj, twohpi), SG_D(amj, twohpj));  // m/H_i + m/H_j
        const double c = self_c(nkernel);
        if (ip == jp) {
            gpot = D.flag[ip] ? SG_M(-c, s) : 0.0;
        } else {
            const int lo = D.orig[ip] < D.orig[jp] ? ip : jp;
            gpot = D.flag[lo] ? SG_M(SG_M(-0.5, c), s) : 0.0;
        }
    }
    PairOut o;
    o.ax = SG_M(gacc, dr1);
    o.ay = SG_M(gacc, dr2);
    o.az = SG_M(gacc, dr3);
    o.pot = gpot;
    return o;
}

// The same near-field formulas from reciprocals ih = 1/H = rsqrt(H^2) where
// the CPU path divides (qq = 1/invq, amj/twohp, mj1/fourhp2), with
// contraction allowed: equal to near_kernel_f64 up to last-bit roundings, at a
// fraction of its cost and register use.  The split-FP32 kernel's near pairs
// (their positions are the 48-bit hi + lo pairs anyway) and the tree mode (an
// approximation) use it.
__device__ __forceinline__ void near_kernel_fast(int nkernel, double r2, double rinv,
                                                double amj, double ihi, double fourhpi2,
                                                double ihj, double fourhpj2,
                                                double mrinv1, double mrinv3,
                                                double &gacc, double &gpot)
{
    const double r = r2 * rinv;
    const double twohpi = fourhpi2 * ihi, twohpj = fourhpj2 * ihj;
    const double invq1 = rinv * twohpi, invq2 = rinv * twohpj;
    const double qq1 = r * ihi, qq2 = r * ihj;
    const double q21 = qq1 * qq1, q22 = qq2 * qq2;
    const double mj11 = amj * ihi, mj12 = amj * ihj;
    const double mj21 = mj11 * (ihi * ihi), mj22 = mj12 * (ihj * ihj);
    const double g1 = (r2 <= fourhpi2) ? 1.0 : 0.0;
    const double g2 = (r2 <= fourhpj2) ? 1.0 : 0.0;
    double acc1, acc2, pot1, pot2;
    if (nkernel == 0) {
        const double q31 = qq1 * q21, q32 = qq2 * q22;
        const double invq31 = invq1 * invq1 * invq1, invq32 = invq2 * invq2 * invq2;
        if (qq1 < 0.5) {
            acc1 = 10.666666666667 + q21 * (32.0 * qq1 - 38.4);
            pot1 = -2.8 + q21 * (5.333333333333 + q21 * (6.4 * qq1 - 9.6));
        } else {
            acc1 = 21.333333333333 - 48.0 * qq1 + 38.4 * q21 - 10.666666666667 * q31
                 - 0.066666666667 * invq31;
            pot1 = -3.2 + 0.066666666667 * invq1
                 + q21 * (10.666666666667 + qq1 * (-16.0 + qq1 * (9.6 - 2.133333333333 * qq1)));
        }
        if (qq2 < 0.5) {
            acc2 = 10.666666666667 + q22 * (32.0 * qq2 - 38.4);
            pot2 = -2.8 + q22 * (5.333333333333 + q22 * (6.4 * qq2 - 9.6));
        } else {
            acc2 = 21.333333333333 - 48.0 * qq2 + 38.4 * q22 - 10.666666666667 * q32
                 - 0.066666666667 * invq32;
            pot2 = -3.2 + 0.066666666667 * invq2
                 + q22 * (10.666666666667 + qq2 * (-16.0 + qq2 * (9.6 - 2.133333333333 * qq2)));
        }
        gacc = 0.5 * (g1 * mj21 * acc1 + (1.0 - g1) * mrinv3 + g2 * mj22 * acc2 + (1.0 - g2) * mrinv3);
        gpot = 0.5 * (g1 * mj11 * pot1 + (g1 - 1.0) * mrinv1 + g2 * mj12 * pot2 + (g2 - 1.0) * mrinv1);
    } else if (nkernel == 1) {
        acc1 = 28.4375 + q21 * ((-187.6875) + q21 * (804.375 + q21 * ((-4379.375) + qq1 * (9009.0 + qq1 * ((-8957.8125) + qq1 * (5005.0 + qq1 * ((-1515.9375) + 195.0 * qq1)))))));
        acc2 = 28.4375 + q22 * ((-187.6875) + q22 * (804.375 + q22 * ((-4379.375) + qq2 * (9009.0 + qq2 * ((-8957.8125) + qq2 * (5005.0 + qq2 * ((-1515.9375) + 195.0 * qq2)))))));
        pot1 = g1 > 0.0 ? (-3.828125) + q21 * (14.21875 + q21 * ((-46.921875) + q21 * (134.0625 + q21 * ((-547.421875) + qq1 * (1001.0 + qq1 * ((-895.78125) + qq1 * (455.0 + qq1 * ((-126.328125) + 15.0 * qq1)))))))) : 0.0;
        pot2 = g2 > 0.0 ? (-3.828125) + q22 * (14.21875 + q22 * ((-46.921875) + q22 * (134.0625 + q22 * ((-547.421875) + qq2 * (1001.0 + qq2 * ((-895.78125) + qq2 * (455.0 + qq2 * ((-126.328125) + 15.0 * qq2)))))))) : 0.0;
        gacc = 0.5 * (g1 * mj21 * acc1 + (1.0 - g1) * mrinv3 + g2 * mj22 * acc2 + (1.0 - g2) * mrinv3);
        gpot = 0.5 * (mj11 * pot1 + (g1 - 1.0) * mrinv1 + mj12 * pot2 + (g2 - 1.0) * mrinv1);
    } else {
        acc1 = 20.625 + q21 * ((-115.5) + q21 * (618.75 + qq1 * ((-1155.0) + qq1 * (962.5 + qq1 * ((-396.0) + 65.625 * qq1)))));
        acc2 = 20.625 + q22 * ((-115.5) + q22 * (618.75 + qq2 * ((-1155.0) + qq2 * (962.5 + qq2 * ((-396.0) + 65.625 * qq2)))));
        pot1 = g1 > 0.0 ? (-3.4375) + q21 * (10.3125 + q21 * ((-28.875) + q21 * (103.125 + qq1 * ((-165.0) + qq1 * (120.3125 + qq1 * ((-44.0) + 6.5625 * qq1)))))) : 0.0;
        pot2 = g2 > 0.0 ? (-3.4375) + q22 * (10.3125 + q22 * ((-28.875) + q22 * (103.125 + qq2 * ((-165.0) + qq2 * (120.3125 + qq2 * ((-44.0) + 6.5625 * qq2)))))) : 0.0;
        gacc = 0.5 * (g1 * mj21 * acc1 + (1.0 - g1) * mrinv3 + g2 * mj22 * acc2 + (1.0 - g2) * mrinv3);
        gpot = 0.5 * (mj11 * pot1 + (g1 - 1.0) * mrinv1 + mj12 * pot2 + (g2 - 1.0) * mrinv1);
    }
}

// pair_f64_core with near_kernel_fast (the split-FP32 kernel's near pairs).
static __device__ __forceinline__ PairOut pair_f64_fast(const SortedF64 &D, int nkernel, int ip,
                                                        int jp, double dr1, double dr2, double dr3,
                                                        double amj, double fourhpi2,
                                                        double fourhpj2)
{
    const double r2 = dr1 * dr1 + dr2 * dr2 + dr3 * dr3;
    double gacc, gpot;
    if (r2 >= fmax(fourhpi2, fourhpj2)) {
        const double rinv = rsqrt(r2);
        const double mrinv1 = rinv * amj;
        gacc = rinv * rinv * mrinv1;
        gpot = -mrinv1;
    } else if (r2 > 0.0) {
        const double rinv = rsqrt(r2);
        const double mrinv1 = rinv * amj;
        const double mrinv3 = rinv * rinv * mrinv1;
        near_kernel_fast(nkernel, r2, rinv, amj, rsqrt(fourhpi2), fourhpi2, rsqrt(fourhpj2),
                        fourhpj2, mrinv1, mrinv3, gacc, gpot);
    } else {
        gacc = 0.0;
        const double s = amj * (rsqrt(fourhpi2) + rsqrt(fourhpj2));  // m/H_i + m/H_j
        const double c = self_c(nkernel);
        if (ip == jp) {
            gpot = D.flag[ip] ? -c * s : 0.0;
        } else {
            const int lo = D.orig[ip] < D.orig[jp] ? ip : jp;
            gpot = D.flag[lo] ? -0.5 * c * s : 0.0;
        }
    }
    PairOut o;
    o.ax = gacc * dr1;
    o.ay = gacc * dr2;
    o.az = gacc * dr3;
    o.pot = gpot;
    return o;
}

// Full FP64 pair from sorted slots ip (row) and jp (source).
static __device__ __noinline__ PairOut pair_f64_slots(const SortedF64 D, int nkernel, int ip, int jp)
{
    const double xi = D.x[ip], yi = D.y[ip], zi = D.z[ip];
    return pair_f64_core(D, nkernel, ip, jp, D.x[jp] - xi, D.y[jp] - yi, D.z[jp] - zi, D.m[jp],
                         D.h2[ip], D.h2[jp]);
}

// ----------------------------------------------------- packed FP32 (sm_100)
// Two FP32 lanes in one 64-bit register; one instruction issues both
// (add/sub/mul/fma .f32x2, PTX ISA 8.6, sm_100+).
typedef unsigned long long f2;

__device__ __forceinline__ f2 pk(float lo, float hi)
{
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void upk(f2 v, float &lo, float &hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2 add2(f2 a, f2 b)
{
    f2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b)
{
    f2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b)
{
    f2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c)
{
    f2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
__device__ __forceinline__ float rsqrt_approx(float x)
{
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Error-free transformation a + b = s + e (Knuth TwoSum).
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e)
{
    s = __fadd_rn(a, b);
    const float bp = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bp)), __fsub_rn(b, bp));
}
// Compensated accumulator (hi, lo): add v.
__device__ __forceinline__ void ff_add(float &hi, float &lo, float v)
{
    float s, e;
    two_sum(hi, v, s, e);
    hi = s;
    lo = __fadd_rn(lo, e);
}
// Add a double into a compensated float accumulator (hi and lo parts).
__device__ __forceinline__ void ff_add_d(float &hi, float &lo, double v)
{
    const float vh = __double2float_rn(v);
    const float vl = __double2float_rn(v - (double)vh);
    ff_add(hi, lo, vh);
    lo = __fadd_rn(lo, vl);
}

// ------------------------------------------ bulk async copies (TMA, 1-D)
// Global -> shared bulk copies completing on an mbarrier (no multicast).
// Source and destination must be 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
// Make barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for phase `parity` of an mbarrier; gives up after `limit` polls
// (each try_wait itself suspends for a hardware-bounded time) and returns
// false, so a lost completion becomes an error status instead of a hang.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t limit)
{
    for (uint32_t it = 0; it < limit; it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Monotone map of doubles to uint64 for atomicMin/atomicMax.
__device__ __forceinline__ unsigned long long dkey(double v)
{
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dkey_inv(unsigned long long k)
{
    unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

}  // namespace sg
