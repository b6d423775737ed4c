// sg_f32sym.cu -- split-FP32 direct summation with mutual updates (sm_100a).
//
// The reference's CPU path evaluates each unordered pair once and applies it
// to both particles (cpu_grav.f: the j >= i triangle with the x m_i/m_j
// update).  This kernel does the same on the GPU: a row tile sums its own
// rows against the sources of its own slots (the diagonal, one-sided) and
// against every later source; the later pairs also give the source j the
// mirrored terms, -m_i f(r) dr and the potential m_i phi.  Per pair, in
// packed f32x2 arithmetic (two sources per instruction):
//     dr = x_j' - x_i',  r2 = dr.dr,  y = rsqrt.approx(r2),  y3 = y^3
//     row i:    acc += (m_j y3) dr,  pot += m_j y
//     source j: acc += (m_i y3) dr,  pot += m_i y       (negated at the merge)
// 18 FMA-pipe lane-ops and one MUFU per pair, two interactions: 9 lane-ops
// per interaction against 13 for the one-sided kernel.
//
// Organisation: the one-sided kernel's (sg_f32.cu) warp-specialised CTA, with
// one producer warp staging 128-source tiles by bulk async copies into an
// mbarrier ring and W consumer warps holding K rows per thread.  A staged
// tile is laid out as source PAIRS (x0 x1 y0 y1 | z0 z1 m0 m1).  Within a
// sub-block of 32 pairs, lane u at step s works on pair (u + s) mod 32, so
// every lane touches every pair once; the source's mirrored sums travel with
// it, one lane down per step (shuffles), and after 32 steps lane u holds the
// warp's complete sums for pair u.  Those are converted to integers at a
// tile-local scale and added into the stage's shared-memory accumulators
// (exact, so independent of the warps' order); when the consumers release
// the stage, the producer adds them into the global per-slot sums (two int64
// words, see sg_internal.cuh) and clears them.  Near pairs (r < band max H)
// are masked out of the FP32 sums, flagged, and evaluated in FP64 after the
// tile, one pair per lane, for both particles.
// Reference kernel replaced: dev_compute_forces / dev_force_ij_nkernel*
// (parallel_bleeding_edge/src/SPHgrav_lib2/grav_force_direct.cu:55-502), with
// the pair symmetry of get_gravity_using_cpus (cpu_grav.f:1-381).
#include <type_traits>
#include "sg_launch.h"

namespace sg {

template <int W, int K, int TJ, int NS>
struct SymSmem {
    static constexpr int NT = W * 32;
    static constexpr int NMETA = TJ / META_J;
    static constexpr int NSB = TJ / 64;  // sub-blocks of 32 source pairs per tile
    static constexpr int NMW = TJ / 32;  // near-mask words per row: 16 steps x 2 sources each
    // raw stage (bulk-copy target): 8 float arrays x_hi x_lo y_hi y_lo z_hi z_lo
    // m H^2, 2 double arrays m H^2, 1 int array (the slots' exponent words)
    static constexpr int RAWSTAGE = 8 * TJ * 4 + 2 * TJ * 8 + TJ * 4;
    static constexpr int RAW = 0;
    static constexpr int META = RAW + NS * RAWSTAGE;
    // computed stage: XY float4[TJ/2] (x0 x1 y0 y1), ZM float4[TJ/2] (z0 z1 m0 m1),
    // H float[TJ] ((band H)^2), EA int[TJ], EP int[TJ] (tile-local exponents)
    static constexpr int COMPSTAGE = 28 * TJ;
    static constexpr int COMP = META + NS * NMETA * 32;
    static constexpr int BOX = COMP + NS * COMPSTAGE;
    static constexpr int ACC = BOX + NS * 32;           // [K*8][NT] floats
    static constexpr int NBITS = ACC + K * 8 * NT * 4;  // [K*NMW][NT] uint32 near masks
    static constexpr int COOP = NBITS + K * NMW * NT * 4;
    static constexpr int COOP_RES = 128 * 8;            // per warp: 4 x 32 doubles ...
    static constexpr int COOP_BUF = 32 * 32 * 2;        // ... and up to 32 x 32 entries
    static constexpr int ROW = COOP + W * (COOP_RES + COOP_BUF);  // [K][5][NT] double
    static constexpr int JACC = ROW + K * 5 * NT * 8;   // [NS][5][TJ] long long
    static constexpr int JT = JACC + NS * 5 * TJ * 8;   // [NS] int2: slot base, mirrored
    static constexpr int BAR = JT + NS * 8;
    static constexpr int ITEM = BAR + 3 * NS * 8;
    static constexpr int BYTES = ITEM + 16;
    static constexpr uint32_t TX = RAWSTAGE + NMETA * 32;  // bytes per tile
};

// Rows farther than this many H from their i-tile centre get an infinite error
// scale (the FP64 refine recomputes them), as in the one-sided kernel.
constexpr float SYM_SHIFT_H = 8.f;

// Add one lane's pair sums (sources j0 = 2p, j1 = 2p + 1) into the stage's
// integer accumulators at the tile-local scales.
__device__ __forceinline__ void sym_add_pair(long long *jacc, int tj, const int *ea, const int *ep,
                                             int p, f2 jx, f2 jy, f2 jz, f2 jp)
{
    f2 gg = mul2(jx, jx);
    gg = fma2(jy, jy, gg);
    gg = fma2(jz, jz, gg);
    float v[5][2];
    upk(jx, v[0][0], v[0][1]);
    upk(jy, v[1][0], v[1][1]);
    upk(jz, v[2][0], v[2][1]);
    upk(jp, v[3][0], v[3][1]);
    upk(gg, v[4][0], v[4][1]);
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int j = 2 * p + h;
        const int e = ea[j];
        if (e == SYM_E_NONE) continue;
        const float sa = exp2f_int(e), sp = exp2f_int(ep[j]);
        atomicAdd(reinterpret_cast<unsigned long long *>(jacc + j),
                  (unsigned long long)__float2ll_rn(v[0][h] * sa));
        atomicAdd(reinterpret_cast<unsigned long long *>(jacc + tj + j),
                  (unsigned long long)__float2ll_rn(v[1][h] * sa));
        atomicAdd(reinterpret_cast<unsigned long long *>(jacc + 2 * tj + j),
                  (unsigned long long)__float2ll_rn(v[2][h] * sa));
        atomicAdd(reinterpret_cast<unsigned long long *>(jacc + 3 * tj + j),
                  (unsigned long long)__float2ll_rn(v[3][h] * sp));
        atomicAdd(reinterpret_cast<unsigned long long *>(jacc + 4 * tj + j),
                  (unsigned long long)__double2ll_rn((double)v[4][h] *
                                                     exp2d_int(2 * e - SYM_LOCAL_BITS)));
    }
}

// Rows of one thread for near_sym.
template <int K>
struct RowSlots {
    int ip[K];
};

// Warp-cooperative FP64 evaluation of the near pairs (r < band max H) the
// checked loop flagged for one staged tile.  Mask word wd = k * NMW + w of a
// lane covers its row k and steps 16 (w & 1) .. 16 (w & 1) + 15 of sub-block
// w >> 1: bit 2 s' + h is source 2 ((lane + 16 (w & 1) + s') mod 32 + 32 (w >> 1)) + h.
// The set bits of all lanes are compacted in lane order, evaluated one pair
// per lane (row data from the FP64 row cache, source data from the raw
// staged tile) as unit-mass terms; each owner sums its rows' results in list
// order (deterministic) and folds them once per row into its compensated
// accumulators, and, for sources past the row tile, every lane adds the
// mirrored terms of its pair into the stage's integer accumulators.  Sources
// below tile-local index jlo (the previous row tile's) are excluded.
template <int K, int TJ, int NT>
__device__ __noinline__ void near_sym(const SortedF64 D, int nkernel, int jbase, int jlo,
                                      RowSlots<K> rs_, uint32_t wsum, const uint32_t *nbits,
                                      const double *s_row, float *s_acc, const float *rs,
                                      const int *ea, const int *ep, long long *jacc, bool mirror,
                                      unsigned short *cbuf, double *res)
{
    constexpr int NMW = TJ / 32;
    constexpr unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, wb = tid - lane;
    const double *rd = reinterpret_cast<const double *>(rs + 8 * TJ);
    uint32_t rem = __reduce_or_sync(FULL, wsum);
    int kcur = -1;
    double sx = 0.0, sy = 0.0, sz = 0.0, sp = 0.0;
    double2 *res2 = reinterpret_cast<double2 *>(res);  // [32] (a_x, a_y), then [32] (a_z, pot)
    auto fold_row = [&]() {
        if (sx != 0.0 || sy != 0.0 || sz != 0.0 || sp != 0.0) {
            float *acc = s_acc + (kcur * 8) * NT + tid;
            ff_add_d(acc[0], acc[4 * NT], sx);
            ff_add_d(acc[NT], acc[5 * NT], sy);
            ff_add_d(acc[2 * NT], acc[6 * NT], sz);
            ff_add_d(acc[3 * NT], acc[7 * NT], -sp);  // accumulators hold -pot
        }
    };
    while (rem) {
        const int wd = __ffs(rem) - 1;
        rem &= rem - 1;
        const int k = wd / NMW, w = wd - k * NMW;
        if (k != kcur) {
            if (kcur >= 0) fold_row();
            kcur = k;
            sx = sy = sz = sp = 0.0;
        }
        const uint32_t m = ((wsum >> wd) & 1u) ? nbits[wd * NT + tid] : 0u;
        const int c = __popc(m);
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(FULL, incl, 31);
        const int excl = incl - c;
        {
            uint32_t mm = m;
            for (int p = excl; mm; p++) {
                const int b = __ffs(mm) - 1;
                mm &= mm - 1;
                cbuf[p] = (unsigned short)((lane << 5) | b);
            }
        }
        __syncwarp();
        int ipk = rs_.ip[0];
#pragma unroll
        for (int kk = 1; kk < K; kk++)
            if (k == kk) ipk = rs_.ip[kk];
        const double *rowk = s_row + (k * 5) * NT + wb;
        const int s0 = 16 * (w & 1), sb = w >> 1;
        for (int base = 0; base < total; base += 32) {
            const int g = base + lane;
            const int ent = g < total ? (int)cbuf[g] : lane << 5;
            const int ow = ent >> 5, bit = ent & 31;
            const int ipo = __shfl_sync(FULL, ipk, ow);
            const int j = 2 * (((ow + s0 + (bit >> 1)) & 31) + 32 * sb) + (bit & 1);
            if (g < total && j < jlo) {
                // an excluded source (the previous row tile's): no term
                res2[lane] = make_double2(0.0, 0.0);
                res2[32 + lane] = make_double2(0.0, 0.0);
            } else if (g < total) {
                const double *row = rowk + ow;
                const double xj = (double)rs[j] + (double)rs[TJ + j];
                const double yj = (double)rs[2 * TJ + j] + (double)rs[3 * TJ + j];
                const double zj = (double)rs[4 * TJ + j] + (double)rs[5 * TJ + j];
                const PairOut o = pair_f64_fast(D, nkernel, ipo, jbase + j, xj - row[0],
                                                yj - row[NT], zj - row[2 * NT], 1.0, row[3 * NT],
                                                rd[TJ + j]);
                const double mj = rd[j];
                res2[lane] = make_double2(mj * o.ax, mj * o.ay);
                res2[32 + lane] = make_double2(mj * o.az, mj * o.pot);
                if (mirror && ea[j] != SYM_E_NONE) {
                    // the source's terms, stored negated: +m_i f dr and -m_i phi
                    const double mi = row[4 * NT];
                    const double sa = exp2d_int(ea[j]), spp = exp2d_int(ep[j]);
                    atomicAdd(reinterpret_cast<unsigned long long *>(jacc + j),
                              (unsigned long long)__double2ll_rn(mi * o.ax * sa));
                    atomicAdd(reinterpret_cast<unsigned long long *>(jacc + TJ + j),
                              (unsigned long long)__double2ll_rn(mi * o.ay * sa));
                    atomicAdd(reinterpret_cast<unsigned long long *>(jacc + 2 * TJ + j),
                              (unsigned long long)__double2ll_rn(mi * o.az * sa));
                    atomicAdd(reinterpret_cast<unsigned long long *>(jacc + 3 * TJ + j),
                              (unsigned long long)__double2ll_rn(-mi * o.pot * spp));
                }
            }
            __syncwarp();
            const int e1 = min(incl, base + 32);
            int e = max(excl, base);
            double tx = 0.0, ty = 0.0, tz = 0.0, tp = 0.0;
            for (; e + 1 < e1; e += 2) {
                const double2 a0 = res2[e - base], b0 = res2[32 + e - base];
                const double2 a1 = res2[e + 1 - base], b1 = res2[33 + e - base];
                sx += a0.x; sy += a0.y; sz += b0.x; sp += b0.y;
                tx += a1.x; ty += a1.y; tz += b1.x; tp += b1.y;
            }
            if (e < e1) {
                const double2 a0 = res2[e - base], b0 = res2[32 + e - base];
                sx += a0.x; sy += a0.y; sz += b0.x; sp += b0.y;
            }
            sx += tx; sy += ty; sz += tz; sp += tp;
            __syncwarp();
        }
    }
    if (kcur >= 0) fold_row();
}

// One step of the rotated pair loop for K rows: the pair's two sources against
// each row; row sums into ax/ay/az/tp, the sources' mirrored sums into
// jx/jy/jz/jp.  CHECK masks pairs with r^2 < max(h2i, the source's (band H)^2)
// (y = 0) and sets their bits (bit shift + h) in nb[k].
template <int K, bool CHECK>
__device__ __forceinline__ void sym_step(const ulonglong2 XY, const ulonglong2 ZM, float2 H2,
                                         const f2 *xi, const f2 *yi, const f2 *zi, const f2 *mi,
                                         const float *h2i, f2 *ax, f2 *ay, f2 *az, f2 *tp,
                                         f2 &jx, f2 &jy, f2 &jz, f2 &jp, uint32_t *nb, int shift)
{
#pragma unroll
    for (int k = 0; k < K; k++) {
        const f2 dx = sub2(XY.x, xi[k]), dy = sub2(XY.y, yi[k]), dz = sub2(ZM.x, zi[k]);
        f2 r2 = mul2(dx, dx);
        r2 = fma2(dy, dy, r2);
        r2 = fma2(dz, dz, r2);
        float ra, rb;
        upk(r2, ra, rb);
        float ya = rsqrt_approx(ra), yb = rsqrt_approx(rb);
        if (CHECK) {
            const bool na = ra < fmaxf(h2i[k], H2.x);
            const bool nb2 = rb < fmaxf(h2i[k], H2.y);
            if (na) ya = 0.f;
            if (nb2) yb = 0.f;
            nb[k] |= ((na ? 1u : 0u) | (nb2 ? 2u : 0u)) << shift;
        }
        const f2 y0 = pk(ya, yb);
        const f2 y3 = mul2(y0, mul2(y0, y0));
        const f2 w = mul2(ZM.y, y3);
        ax[k] = fma2(w, dx, ax[k]);
        ay[k] = fma2(w, dy, ay[k]);
        az[k] = fma2(w, dz, az[k]);
        tp[k] = fma2(ZM.y, y0, tp[k]);
        const f2 v = mul2(mi[k], y3);
        jx = fma2(v, dx, jx);
        jy = fma2(v, dy, jy);
        jz = fma2(v, dz, jz);
        jp = fma2(mi[k], y0, jp);
    }
}

template <int W, int K, int TJ, int NS>
__global__ void __launch_bounds__((W + 1) * 32, 1) k_f32sym(ComputeArgs a)
{
    static_assert(TJ % 64 == 0, "j-tile must hold whole sub-blocks of 32 source pairs");
    using L = SymSmem<W, K, TJ, NS>;
    constexpr int NT = L::NT;
    constexpr int ITILE = NT * K;
    constexpr int NMETA = L::NMETA;
    static_assert(NMETA >= 1 && NMETA <= 32 && (NMETA & (NMETA - 1)) == 0,
                  "tile box reduction: one record per lane, a power of two");
    constexpr int NSB = L::NSB, NMW = L::NMW;
    static_assert(K * NMW <= 32, "one summary bit per near-mask word");
    constexpr uint32_t WAIT_LIMIT = 1u << 22;
    constexpr unsigned FULL = 0xffffffffu;

    extern __shared__ __align__(128) unsigned char smem[];
    JMeta *s_meta = reinterpret_cast<JMeta *>(smem + L::META);
    TileBox *s_box = reinterpret_cast<TileBox *>(smem + L::BOX);
    float *s_acc = reinterpret_cast<float *>(smem + L::ACC);
    uint32_t *s_nbits = reinterpret_cast<uint32_t *>(smem + L::NBITS);
    double *s_row = reinterpret_cast<double *>(smem + L::ROW);  // [K][5][NT]: x y z H^2 m
    long long *s_jacc = reinterpret_cast<long long *>(smem + L::JACC);
    int2 *s_jt = reinterpret_cast<int2 *>(smem + L::JT);
    uint64_t *bar_raw = reinterpret_cast<uint64_t *>(smem + L::BAR);
    uint64_t *bar_full = bar_raw + NS;
    uint64_t *bar_empty = bar_full + NS;
    int *s_item = reinterpret_cast<int *>(smem + L::ITEM);

    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const bool producer = (warp == W);
    const SortedF64 D = a.D;
    const SortedF32 F = a.F;
    const int nitems = a.nitems_dev ? *a.nitems_dev : a.nitems;

    if (tid == 0) {
        for (int s = 0; s < NS; s++) {
            mbar_init(&bar_raw[s], 1);
            mbar_init(&bar_full[s], 32);
            mbar_init(&bar_empty[s], NT);
        }
        fence_mbar_init();
    }
    for (int i = tid; i < NS * 5 * TJ; i += (W + 1) * 32) s_jacc[i] = 0ll;
    for (int i = tid; i < NS; i += (W + 1) * 32) s_jt[i] = make_int2(0, 0);
    __syncthreads();

    uint32_t g = 0;
    bool failed = false;
    bool pending[NS];
    uint32_t pend_par[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) { pending[s] = false; pend_par[s] = 0u; }

    auto stage_raw = [&](int s) -> const float * {
        return reinterpret_cast<const float *>(smem + L::RAW + s * L::RAWSTAGE);
    };
    auto stage_comp = [&](int s) -> unsigned char * { return smem + L::COMP + s * L::COMPSTAGE; };
    // bulk copies of set-local slots [jt, jt+TJ) (ring tile gt) into raw stage gt % NS
    auto issue = [&](const SetDesc &S, int jt, uint32_t gt) {
        const int b = gt % NS;
        float *dst = reinterpret_cast<float *>(smem + L::RAW + b * L::RAWSTAGE);
        double *dstd = reinterpret_cast<double *>(dst + 8 * TJ);
        int *dsti = reinterpret_cast<int *>(dstd + 2 * TJ);
        const int s0 = S.poff + jt;
        pending[b] = true;
        pend_par[b] = (gt / NS) & 1;
        fence_mbar_init();
        mbar_arrive_expect_tx(&bar_raw[b], L::TX);
        const float *src[8] = {F.xh, F.xl, F.yh, F.yl, F.zh, F.zl, F.m, F.h2};
#pragma unroll
        for (int k = 0; k < 8; k++) bulk_g2s(dst + k * TJ, src[k] + s0, TJ * 4, &bar_raw[b]);
        bulk_g2s(dstd, D.m + s0, TJ * 8, &bar_raw[b]);
        bulk_g2s(dstd + TJ, D.h2 + s0, TJ * 8, &bar_raw[b]);
        bulk_g2s(dsti, a.jword + s0, TJ * 4, &bar_raw[b]);
        bulk_g2s(s_meta + b * NMETA, a.jmeta + S.meta_off + jt / META_J, NMETA * 32, &bar_raw[b]);
    };
    // producer warp: add stage b's integer sums into the global per-slot sums and clear them
    auto flush = [&](int b) {
        const int2 jt = s_jt[b];
        long long *sj = s_jacc + b * 5 * TJ;
        if (jt.y) {
            const int *eg = reinterpret_cast<const int *>(stage_raw(b) + 8 * TJ + 4 * TJ);
            const unsigned char *cs = stage_comp(b);
            const int *ea = reinterpret_cast<const int *>(cs + 20 * TJ);
            const int *ep = reinterpret_cast<const int *>(cs + 24 * TJ);
            const size_t js = a.jstride;
            for (int j = lane; j < TJ; j += 32) {
                const int wg = eg[j];
                const int Ea = sym_exp_acc(wg), Ep = sym_exp_pot(wg);
                if (Ea == SYM_E_NONE || ea[j] == SYM_E_NONE) continue;
                unsigned long long *gp =
                    reinterpret_cast<unsigned long long *>(a.jacc) + (size_t)jt.x + j;
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    long long hi, lo;
                    sym_split(sj[c * TJ + j], c < 3 ? Ea - ea[j] : Ep - ep[j], hi, lo);
                    if (hi) atomicAdd(gp + (2 * c) * js, (unsigned long long)hi);
                    if (lo) atomicAdd(gp + (2 * c + 1) * js, (unsigned long long)lo);
                }
                const long long g2 = sym_shift(sj[4 * TJ + j],
                                               2 * (Ea - ea[j]) - (SYM_G2_SHIFT - SYM_LOCAL_BITS));
                if (g2) atomicAdd(gp + 8 * js, (unsigned long long)g2);
            }
        }
        for (int i = lane; i < 5 * TJ; i += 32) sj[i] = 0ll;
        __syncwarp();
    };

    for (int iter = 0;; iter++) {
        if (tid == 0) s_item[iter & 1] = atomicAdd(a.head, 1);
        if (__syncthreads_or(failed)) break;
        const int it = s_item[iter & 1];
        if (it >= nitems) break;
        const WorkItem Wk = a.items[it];
        const SetDesc S = a.sets[Wk.set];
        const ITileMeta C = a.imeta[S.tile_off + Wk.tile];
        const int ntile = (Wk.je - Wk.jb) / TJ;
        // set-local slots: the row tile's own [row_lo, mirror_from) are summed
        // one-sided; slots below row_lo (the tail of the previous row tile, in
        // a j-tile that straddles) are excluded; slots from mirror_from on get
        // the mirrored terms
        const int row_lo = Wk.tile * ITILE;
        const int mirror_from = row_lo + ITILE;

        if (producer) {
            // ------------------------------------------------ producer warp
            auto issue_tile = [&](int t, uint32_t gt) {
                const int b = gt % NS;
                if (gt >= (uint32_t)NS) flush(b);  // the stage's previous tile, released
                const int jt = Wk.jb + t * TJ;
                if (lane == 0) {
                    s_jt[b] = make_int2(S.poff + jt, jt + TJ > mirror_from ? 1 : 0);
                    issue(S, jt, gt);
                }
                __syncwarp();
            };
            if (ntile > 0) {
                const bool ok = mbar_wait_bounded(&bar_empty[g % NS], ((g / NS) & 1) ^ 1, WAIT_LIMIT);
                if (!__all_sync(FULL, ok)) {
                    if (lane == 0) atomicOr(a.err, DEVERR_TIMEOUT);
                    failed = true;
                } else {
                    issue_tile(0, g);
                }
            }
            for (int t = 0; t < ntile && !failed; t++) {
                const uint32_t gt = g + t;
                const int s = gt % NS;
                bool ok = true;
                if (t + 1 < ntile) {
                    const uint32_t gn = gt + 1;
                    ok = mbar_wait_bounded(&bar_empty[gn % NS], ((gn / NS) & 1) ^ 1, WAIT_LIMIT);
                    if (__all_sync(FULL, ok)) issue_tile(t + 1, gn);
                }
                ok = ok && mbar_wait_bounded(&bar_raw[s], (gt / NS) & 1, WAIT_LIMIT);
                if (ok && lane == 0) pending[s] = false;
                if (!__all_sync(FULL, ok)) {
                    if (lane == 0) atomicOr(a.err, DEVERR_TIMEOUT);
                    failed = true;
                    break;
                }
                // rewrite the tile as source pairs relative to the i-tile centre,
                // with the tile-local exponents of the mirrored sums
                const float4 *rb4 = reinterpret_cast<const float4 *>(stage_raw(s));
                const int4 *eg4 = reinterpret_cast<const int4 *>(stage_raw(s) + 8 * TJ + 4 * TJ);
                unsigned char *cs = stage_comp(s);
                float4 *xy = reinterpret_cast<float4 *>(cs);
                float4 *zm = reinterpret_cast<float4 *>(cs + 8 * TJ);
                float4 *hh = reinterpret_cast<float4 *>(cs + 16 * TJ);
                int4 *ea4 = reinterpret_cast<int4 *>(cs + 20 * TJ);
                int4 *ep4 = reinterpret_cast<int4 *>(cs + 24 * TJ);
                constexpr int T4 = TJ / 4;
                auto rel = [](float4 h, float4 l, float ch, float cl) {
                    return make_float4(__fadd_rn(__fsub_rn(h.x, ch), __fsub_rn(l.x, cl)),
                                       __fadd_rn(__fsub_rn(h.y, ch), __fsub_rn(l.y, cl)),
                                       __fadd_rn(__fsub_rn(h.z, ch), __fsub_rn(l.z, cl)),
                                       __fadd_rn(__fsub_rn(h.w, ch), __fsub_rn(l.w, cl)));
                };
                const float inv_hmin = C.h2min > 0.f ? __frcp_rn(C.h2min) : INFINITY;
                const float rs_hmin = C.h2min > 0.f ? rsqrtf(C.h2min) : INFINITY;
                const int jt = Wk.jb + t * TJ;
                for (int j = lane; j < T4; j += 32) {
                    const float4 x = rel(rb4[j], rb4[T4 + j], C.chx, C.clx);
                    const float4 y = rel(rb4[2 * T4 + j], rb4[3 * T4 + j], C.chy, C.cly);
                    const float4 z = rel(rb4[4 * T4 + j], rb4[5 * T4 + j], C.chz, C.clz);
                    float4 m = rb4[6 * T4 + j];
                    const float4 h = rb4[7 * T4 + j];
                    const int jl = jt + 4 * j;  // set-local slot of the first of the four
                    if (jl < row_lo) {          // excluded sources carry no mass
                        if (jl + 0 < row_lo) m.x = 0.f;
                        if (jl + 1 < row_lo) m.y = 0.f;
                        if (jl + 2 < row_lo) m.z = 0.f;
                        if (jl + 3 < row_lo) m.w = 0.f;
                    }
                    xy[2 * j] = make_float4(x.x, x.y, y.x, y.y);
                    xy[2 * j + 1] = make_float4(x.z, x.w, y.z, y.w);
                    zm[2 * j] = make_float4(z.x, z.y, m.x, m.y);
                    zm[2 * j + 1] = make_float4(z.z, z.w, m.z, m.w);
                    hh[j] = make_float4(a.band2 * h.x, a.band2 * h.y, a.band2 * h.z, a.band2 * h.w);
                    const int4 wg = eg4[j];
                    const int wv[4] = {wg.x, wg.y, wg.z, wg.w};
                    const float hv[4] = {h.x, h.y, h.z, h.w};
                    int eav[4], epv[4];
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const int Ea = sym_exp_acc(wv[q]), Ep = sym_exp_pot(wv[q]);
                        if (Ea == SYM_E_NONE || Ep == SYM_E_NONE || jl + q < mirror_from) {
                            eav[q] = epv[q] = SYM_E_NONE;
                            continue;
                        }
                        // tile-local bounds (the row tile's mass and smallest H); a
                        // bound that is not finite falls back to the global one,
                        // valid because the tile's mass and H lie within the set's
                        const float ba = SYM_BOUND * C.mass * (__frcp_rn(hv[q]) + inv_hmin);
                        const float bp = SYM_BOUND * C.mass * (rsqrtf(hv[q]) + rs_hmin);
                        eav[q] = max(sym_local_exp(ba, Ea - (SYM_GLOBAL_BITS - SYM_LOCAL_BITS)),
                                     Ea - SYM_LO_BITS);
                        epv[q] = max(sym_local_exp(bp, Ep - (SYM_GLOBAL_BITS - SYM_LOCAL_BITS)),
                                     Ep - SYM_LO_BITS);
                    }
                    ea4[j] = make_int4(eav[0], eav[1], eav[2], eav[3]);
                    ep4[j] = make_int4(epv[0], epv[1], epv[2], epv[3]);
                }
                // the tile's box relative to the centre (as in the one-sided kernel)
                {
                    float lo[3] = {INFINITY, INFINITY, INFINITY};
                    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
                    float h2m = 0.f;
                    int empty = 1;
                    if (lane < NMETA) {
                        const JMeta M = s_meta[s * NMETA + lane];
                        if (M.ex >= 0.f) {
                            empty = 0;
                            const float c3[3] = {C.chx, C.chy, C.chz};
                            const float mc[3] = {M.cx, M.cy, M.cz}, me[3] = {M.ex, M.ey, M.ez};
#pragma unroll
                            for (int d = 0; d < 3; d++) {
                                const float rc = mc[d] - c3[d];
                                const float e = me[d] + 9.5367e-7f * (fabsf(mc[d]) + fabsf(c3[d]) + me[d]);
                                lo[d] = rc - e;
                                hi[d] = rc + e;
                            }
                            h2m = a.band2 * M.h2max * 1.000001f;
                        }
                    }
#pragma unroll
                    for (int o = 1; o < NMETA; o <<= 1) {
#pragma unroll
                        for (int d = 0; d < 3; d++) {
                            lo[d] = fminf(lo[d], __shfl_xor_sync(FULL, lo[d], o));
                            hi[d] = fmaxf(hi[d], __shfl_xor_sync(FULL, hi[d], o));
                        }
                        h2m = fmaxf(h2m, __shfl_xor_sync(FULL, h2m, o));
                        empty &= __shfl_xor_sync(FULL, empty, o);
                    }
                    if (lane == 0) {
                        TileBox B;
                        B.empty = empty;
                        B.h2max = h2m;
                        for (int d = 0; d < 3; d++) { B.lo[d] = lo[d]; B.hi[d] = hi[d]; }
                        s_box[s] = B;
                    }
                }
                __syncwarp();
                mbar_arrive(&bar_full[s]);
            }
        } else {
            // ----------------------------------------------- consumer warps
            int ip[K];
            bool act[K], shifted[K];
            f2 xi[K], yi[K], zi[K], mi[K], g2[K];
            float h2i[K];
            float wlo[3] = {INFINITY, INFINITY, INFINITY};
            float whi[3] = {-INFINITY, -INFINITY, -INFINITY};
            float wh2 = 0.f;
#pragma unroll
            for (int k = 0; k < K; k++) {
                const int li = warp * 32 * K + k * 32 + lane;
                const int r = Wk.tile * ITILE + li;
                act[k] = r < S.ni;
                ip[k] = act[k] ? a.ilist[S.ioff + r] : 0;
                float x = 1.0e15f, y = 1.0e15f, z = -1.0e15f, h2 = 0.f, m = 0.f;
                if (act[k]) {
                    const int sl = ip[k];
                    x = __fadd_rn(__fsub_rn(F.xh[sl], C.chx), __fsub_rn(F.xl[sl], C.clx));
                    y = __fadd_rn(__fsub_rn(F.yh[sl], C.chy), __fsub_rn(F.yl[sl], C.cly));
                    z = __fadd_rn(__fsub_rn(F.zh[sl], C.chz), __fsub_rn(F.zl[sl], C.clz));
                    h2 = a.band2 * F.h2[sl];
                    m = F.m[sl];
                    double *rw = s_row + (k * 5) * NT + tid;
                    rw[0] = (double)F.xh[sl] + (double)F.xl[sl];
                    rw[NT] = (double)F.yh[sl] + (double)F.yl[sl];
                    rw[2 * NT] = (double)F.zh[sl] + (double)F.zl[sl];
                    rw[3 * NT] = D.h2[sl];
                    rw[4 * NT] = D.m[sl];
                    wlo[0] = fminf(wlo[0], x); whi[0] = fmaxf(whi[0], x);
                    wlo[1] = fminf(wlo[1], y); whi[1] = fmaxf(whi[1], y);
                    wlo[2] = fminf(wlo[2], z); whi[2] = fmaxf(whi[2], z);
                    wh2 = fmaxf(wh2, h2);
                }
                xi[k] = pk(x, x);
                yi[k] = pk(y, y);
                zi[k] = pk(z, z);
                mi[k] = pk(m, m);
                h2i[k] = h2;
                g2[k] = pk(0.f, 0.f);
                shifted[k] = act[k] && x * x + y * y + z * z > SYM_SHIFT_H * SYM_SHIFT_H * F.h2[ip[k]];
#pragma unroll
                for (int c = 0; c < 8; c++) s_acc[(k * 8 + c) * NT + tid] = 0.f;
            }
#pragma unroll
            for (int d = 0; d < 3; d++) {
                for (int o = 16; o > 0; o >>= 1) {
                    wlo[d] = fminf(wlo[d], __shfl_xor_sync(FULL, wlo[d], o));
                    whi[d] = fmaxf(whi[d], __shfl_xor_sync(FULL, whi[d], o));
                }
            }
            for (int o = 16; o > 0; o >>= 1) wh2 = fmaxf(wh2, __shfl_xor_sync(FULL, wh2, o));
            const bool warp_rows = wlo[0] <= whi[0];
            wh2 = wh2 * 1.00001f;
            float slack[3];
#pragma unroll
            for (int d = 0; d < 3; d++) slack[d] = 9.5367e-7f * fmaxf(fabsf(wlo[d]), fabsf(whi[d]));
            const int src_lane = (lane + 1) & 31;

            for (int t = 0; t < ntile; t++) {
                const uint32_t gt = g + t;
                const int s = gt % NS;
                const bool ok = mbar_wait_bounded(&bar_full[s], (gt / NS) & 1, WAIT_LIMIT);
                if (!__all_sync(FULL, ok)) {
                    if (lane == 0) atomicOr(a.err, DEVERR_TIMEOUT);
                    failed = true;
                    break;
                }
                const unsigned char *cs = stage_comp(s);
                const ulonglong2 *s_xy = reinterpret_cast<const ulonglong2 *>(cs);
                const ulonglong2 *s_zm = reinterpret_cast<const ulonglong2 *>(cs + 8 * TJ);
                const float2 *s_h = reinterpret_cast<const float2 *>(cs + 16 * TJ);
                const int *s_ea = reinterpret_cast<const int *>(cs + 20 * TJ);
                const int *s_ep = reinterpret_cast<const int *>(cs + 24 * TJ);
                long long *jacc = s_jacc + s * 5 * TJ;
                const int jt = Wk.jb + t * TJ;
                const bool mirror = jt + TJ > mirror_from;
                // warps without rows (the end of a set's last row tile) add nothing
                if (warp_rows) {
                    const TileBox B = s_box[s];
                    bool far = B.empty;
                    if (!far) {
                        float d2 = 0.f;
#pragma unroll
                        for (int d = 0; d < 3; d++) {
                            float gap = fmaxf(B.lo[d] - whi[d], wlo[d] - B.hi[d]) - slack[d];
                            gap = fmaxf(gap, 0.f);
                            d2 = fmaf(gap, gap, d2);
                        }
                        far = d2 > fmaxf(wh2, B.h2max) * 1.0001f;
                    }
                    f2 tx[K], ty[K], tz[K], tp[K];
#pragma unroll
                    for (int k = 0; k < K; k++) tx[k] = ty[k] = tz[k] = tp[k] = pk(0.f, 0.f);
                    uint32_t wsum = 0;
                    // the sub-block loop, with or without the per-pair near test
                    auto run = [&](auto check_tag) {
                        constexpr bool CHECK = decltype(check_tag)::value;
                        for (int sb = 0; sb < NSB; sb++) {
                            f2 jx = pk(0.f, 0.f), jy = jx, jz = jx, jp = jx;
                            uint32_t nb[K];
#pragma unroll
                            for (int k = 0; k < K; k++) nb[k] = 0u;
#pragma unroll
                            for (int s8 = 0; s8 < 4; s8++) {
                                f2 ax[K], ay[K], az[K];
#pragma unroll
                                for (int k = 0; k < K; k++) ax[k] = ay[k] = az[k] = pk(0.f, 0.f);
#pragma unroll
                                for (int u = 0; u < 8; u++) {
                                    const int st = s8 * 8 + u;
                                    const int p = sb * 32 + ((lane + st) & 31);
                                    const ulonglong2 XY = s_xy[p], ZM = s_zm[p];
                                    const float2 H2 = CHECK ? s_h[p] : make_float2(0.f, 0.f);
                                    sym_step<K, CHECK>(XY, ZM, H2, xi, yi, zi, mi, h2i, ax, ay, az,
                                                       tp, jx, jy, jz, jp, nb, 2 * (st & 15));
                                    jx = __shfl_sync(FULL, jx, src_lane);
                                    jy = __shfl_sync(FULL, jy, src_lane);
                                    jz = __shfl_sync(FULL, jz, src_lane);
                                    jp = __shfl_sync(FULL, jp, src_lane);
                                    if (CHECK && (st & 15) == 15) {
                                        const int wd = 2 * sb + (st >> 4);
#pragma unroll
                                        for (int k = 0; k < K; k++) {
                                            if (act[k] && nb[k]) {
                                                s_nbits[(k * NMW + wd) * NT + tid] = nb[k];
                                                wsum |= 1u << (k * NMW + wd);
                                            }
                                            nb[k] = 0u;
                                        }
                                    }
                                }
#pragma unroll
                                for (int k = 0; k < K; k++) {
                                    tx[k] = add2(tx[k], ax[k]);
                                    ty[k] = add2(ty[k], ay[k]);
                                    tz[k] = add2(tz[k], az[k]);
                                }
                            }
                            // lane holds the warp's sums for pair sb * 32 + lane
                            if (mirror)
                                sym_add_pair(jacc, TJ, s_ea, s_ep, sb * 32 + lane, jx, jy, jz, jp);
                        }
                    };
                    if (far)
                        run(std::false_type{});
                    else
                        run(std::true_type{});
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        g2[k] = fma2(tx[k], tx[k], g2[k]);
                        g2[k] = fma2(ty[k], ty[k], g2[k]);
                        g2[k] = fma2(tz[k], tz[k], g2[k]);
                        float *acc = s_acc + (k * 8) * NT + tid;
                        fold(acc, acc + 4 * NT, tx[k]);
                        fold(acc + NT, acc + 5 * NT, ty[k]);
                        fold(acc + 2 * NT, acc + 6 * NT, tz[k]);
                        fold(acc + 3 * NT, acc + 7 * NT, tp[k]);
                    }
                    if (!far && __any_sync(FULL, wsum != 0u)) {
                        unsigned char *cb = smem + L::COOP + warp * (L::COOP_RES + L::COOP_BUF);
                        RowSlots<K> rsl;
#pragma unroll
                        for (int k = 0; k < K; k++) rsl.ip[k] = ip[k];
                        near_sym<K, TJ, NT>(D, a.nkernel, S.poff + jt, row_lo - jt, rsl, wsum,
                                            s_nbits, s_row, s_acc, stage_raw(s), s_ea, s_ep, jacc,
                                            mirror,
                                            reinterpret_cast<unsigned short *>(cb + L::COOP_RES),
                                            reinterpret_cast<double *>(cb));
                    }
                }
                mbar_arrive(&bar_empty[s]);
            }
            if (!failed) {
                __syncwarp();
                const size_t slot = (size_t)Wk.slot;
                double *p = a.partials + slot * 4 * ITILE;
#pragma unroll
                for (int k = 0; k < K; k++) {
                    if (!act[k]) continue;
                    const int li = warp * 32 * K + k * 32 + lane;
                    if (a.gpart) {
                        float ga, gb;
                        upk(g2[k], ga, gb);
                        a.gpart[slot * ITILE + li] = shifted[k] ? INFINITY : ga + gb;
                    }
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        const float h = s_acc[(k * 8 + c) * NT + tid];
                        const float l = s_acc[(k * 8 + 4 + c) * NT + tid];
                        p[c * ITILE + li] = ((double)h + (double)l) * (c < 3 ? 1.0 : -1.0);
                    }
                }
            }
        }
        g += ntile;
    }
    // the last tiles' stages: wait for their release, then flush them; never
    // leave with bulk copies in flight into this CTA's shared memory
    if (producer) {
        if (!failed) {
            const uint32_t first = g > (uint32_t)NS ? g - NS : 0u;
            for (uint32_t gt = first; gt < g; gt++) {
                const bool ok = mbar_wait_bounded(&bar_empty[gt % NS], (gt / NS) & 1, WAIT_LIMIT);
                if (!__all_sync(FULL, ok)) {
                    if (lane == 0) atomicOr(a.err, DEVERR_TIMEOUT);
                    break;
                }
                flush(gt % NS);
            }
        }
        if (lane == 0)
            for (int b = 0; b < NS; b++)
                if (pending[b]) mbar_wait_bounded(&bar_raw[b], pend_par[b], WAIT_LIMIT);
    }
}

// name, consumer warps W, rows per thread K, j-tile TJ, stages NS.  (13 warps
// leave 128 registers per thread, one SMSP holding four of them; 12 or fewer
// allow 168.)
#define SG_SYM_VARIANTS(X)                                  \
    X(11, 2, 128, 6, "f32sym_w11_k2_tj128_ns6")            \
    X(11, 3, 128, 6, "f32sym_w11_k3_tj128_ns6")            \
    X(8, 4, 128, 6, "f32sym_w8_k4_tj128_ns6")              \
    X(12, 2, 128, 6, "f32sym_w12_k2_tj128_ns6")

#define SG_INFO(W, K, TJ, NS, NAME) {1, (W + 1) * 32, K, 1, TJ, 0, NAME, W * 32 * K, 1},
static const VariantInfo kSymVariants[] = {SG_SYM_VARIANTS(SG_INFO)};
#undef SG_INFO
#define SG_PTR(W, K, TJ, NS, NAME) (const void *)k_f32sym<W, K, TJ, NS>,
static const void *kSymKernels[] = {SG_SYM_VARIANTS(SG_PTR)};
#undef SG_PTR
#define SG_SMEM(W, K, TJ, NS, NAME) SymSmem<W, K, TJ, NS>::BYTES,
static const int kSymSmem[] = {SG_SYM_VARIANTS(SG_SMEM)};
#undef SG_SMEM
constexpr int kNSym = sizeof(kSymVariants) / sizeof(kSymVariants[0]);

int sym_variant_count() { return kNSym; }
const VariantInfo &sym_variant_info(int v) { return kSymVariants[v]; }
const void *sym_kernel(int v) { return kSymKernels[v]; }
int sym_smem_bytes(int v) { return kSymSmem[v]; }

cudaError_t sym_prepare(int v)
{
    constexpr int MAXDEV = 64;
    static std::atomic<bool> done[MAXDEV][kNSym];
    if (v < 0 || v >= kNSym) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const bool track = dev >= 0 && dev < MAXDEV;
    if (track && done[dev][v].load(std::memory_order_acquire)) return cudaSuccess;
    e = cudaFuncSetAttribute(kSymKernels[v], cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kSymSmem[v]);
    if (e == cudaSuccess && track) done[dev][v].store(true, std::memory_order_release);
    return e;
}

cudaError_t launch_sym(int v, int grid, const ComputeArgs &a, cudaStream_t st)
{
    cudaError_t e = sym_prepare(v);
    if (e != cudaSuccess) return e;
    int idx = 0;
#define SG_CASE(W, K, TJ, NS, NAME)                                                        \
    if (v == idx) {                                                                        \
        k_f32sym<W, K, TJ, NS><<<grid, (W + 1) * 32, SymSmem<W, K, TJ, NS>::BYTES, st>>>(a); \
        ++g_launches;                                                                      \
        return cudaGetLastError();                                                         \
    }                                                                                      \
    ++idx;
    SG_SYM_VARIANTS(SG_CASE)
#undef SG_CASE
    return cudaErrorInvalidValue;
}

}  // namespace sg
