// sg_f32.cu -- split-FP32 direct-summation kernel for sm_100a.
//
// Per pair (far field, the >99.9% case at large N), in packed f32x2
// arithmetic so one instruction evaluates two (row, source) pairs:
//     dr   = x_j' - x_i'                    (tile-relative coordinates)
//     r2   = dr.dr
//     y    = rsqrt.approx(r2)
//     pot += m_j y                          (accumulated as +m/r, negated at the end)
//     acc += (m_j y)(y y) dr
// 13 FMA-pipe lane-ops and one MUFU per pair.  The `_newton` variants add one
// Newton step, Y = y (r2 y^2 - 3) = -2/r, accumulating -2 m_j/r and
// -8 m_j dr/r^3 (exact power-of-two scales removed at the end): 16 lane-ops.
// Measured against FP64 on every benchmark workload the step does not make
// the FP32 sums more accurate (its own two roundings cost more than the
// ~1e-7 rsqrt.approx error it removes: RMS 3.2e-8 without vs 3.7e-8 with at
// N=1M), so the defaults leave it out.
//
// CTA organisation (warp-specialised, persistent over a device queue of
// (set, i-tile, j-chunk) items):
//   * one producer warp: issues 1-D bulk async copies (cp.async.bulk, the
//     TMA engine; no multicast) of each j-tile's SoA arrays x_hi, x_lo, y_hi,
//     y_lo, z_hi, z_lo, m, H^2, FP64 m and H^2, and bounding-box records into
//     an NS-stage raw ring, waits for their mbarrier transaction count,
//     rewrites the tile as i-tile-relative floats into the stage's computed
//     part and signals the stage "full";
//   * W consumer warps: each owns 32*K/Q rows in registers, waits for a full
//     stage, sums the tile, and signals it "empty".  Consumers never meet at
//     a CTA-wide barrier inside an item, so warps that hit near-field pairs
//     may run behind the others by up to NS-1 tiles.  W = 12 puts three
//     consumer warps on every SMSP; with W = 15 the producer's SMSP has one
//     fewer, and its warps finish tiles early and wait on the ring.
//   * every mbarrier wait is a bounded poll; a timeout sets an error bit and
//     the CTA leaves at the next item boundary after its copies have landed.
//
// Precision design:
//   * positions arrive as float hi + lo pairs of the FP64 inputs; rows and
//     staged sources are re-expressed relative to the i-tile's centre c:
//     x' = (x_hi - c_hi) + (x_lo - c_lo), a few flops per staged particle
//     instead of per pair.
//   * acceleration sums run in FP32 over sub-blocks (8 terms per
//     accumulator lane), are added into a per-tile FP32 sum that folds into
//     compensated (TwoSum, "Kahan") float hi/lo accumulators in shared memory
//     once per tile; the potential terms, all of one sign, go straight into
//     the tile sum in the far loop.  Per row the kernel also keeps G^2, the
//     sum over tiles of |FP32 tile sum|^2 (the scale of the FP32 rounding
//     error), for the FP64 refine of ill-conditioned rows (sg_refine.cu).
//   * pairs with r < band max(H_i, H_j) (band 1 by default) are masked out
//     of the FP32 sums by the checked loop, flagged in per-thread bit masks,
//     and evaluated after the tile's FP32 loop in FP64 with the CPU-path
//     formulas, one pair per lane of the warp (near_eval), then folded into
//     the same accumulators: the softened near field, whose reference
//     polynomials cancel by up to ~1e4 near q = 1 (a larger band also moves
//     the largest Newtonian terms, see ComputeArgs::band2).  A warp skips the
//     per-pair test (the far loop) for a tile when the bounding boxes of its
//     rows and of the tile are farther apart than band max(H) of both.
//   * per (row, j-chunk) results leave the CTA as FP64 partial sums merged in
//     chunk order (k_merge).
// Reference kernel replaced: dev_compute_forces / dev_force_ij_nkernel*
// (parallel_bleeding_edge/src/SPHgrav_lib2/grav_force_direct.cu:55-502).
#include "sg_launch.h"

namespace sg {

struct TileBox {
    float lo[3], hi[3];
    float h2max;
    int empty;
};

template <bool NEWTON>
struct Scales {
    // accumulated value * scale = physical value
    static constexpr float acc = NEWTON ? -0.125f : 1.0f;
    static constexpr float pot = NEWTON ? 0.5f : -1.0f;
};

__device__ __forceinline__ void geom2(f2 xj, f2 yj, f2 zj, f2 xi, f2 yi, f2 zi, f2 &dx, f2 &dy,
                                      f2 &dz, f2 &r2)
{
    dx = sub2(xj, xi);
    dy = sub2(yj, yi);
    dz = sub2(zj, zi);
    r2 = mul2(dx, dx);
    r2 = fma2(dy, dy, r2);
    r2 = fma2(dz, dz, r2);
}

template <bool NEWTON>
__device__ __forceinline__ void accum2(f2 dx, f2 dy, f2 dz, f2 r2, f2 mj, f2 &ax, f2 &ay,
                                       f2 &az, f2 &pp)
{
    float ra, rb;
    upk(r2, ra, rb);
    const f2 y0 = pk(rsqrt_approx(ra), rsqrt_approx(rb));
    const f2 ysq = mul2(y0, y0);
    f2 mr, mr3;
    if (NEWTON) {
        const f2 t = fma2(r2, ysq, pk(-3.0f, -3.0f));  // -(3 - r2 y0^2)
        const f2 yn = mul2(y0, t);                       // -2 y1
        mr = mul2(mj, yn);                               // -2 m y1
        const f2 y2 = mul2(yn, yn);                      // 4 y1^2
        mr3 = mul2(mr, y2);                              // -8 m y1^3
    } else {
        mr = mul2(mj, y0);
        mr3 = mul2(mr, ysq);
    }
    ax = fma2(mr3, dx, ax);
    ay = fma2(mr3, dy, ay);
    az = fma2(mr3, dz, az);
    pp = add2(pp, mr);
}

// Fold a packed FP32 partial into a compensated accumulator pair in shared memory.
__device__ __forceinline__ void fold(float *hi, float *lo, f2 v)
{
    float a, b;
    upk(v, a, b);
    float h = *hi, l = *lo;
    ff_add(h, l, a);
    ff_add(h, l, b);
    *hi = h;
    *lo = l;
}

// Near-field pair (r^2 < max H^2) in FP64, folded into the row's
// compensated accumulators acc[c * stride] (hi) / acc[(4 + c) * stride] (lo),
// in the accumulators' scaled units.
// The source's data come from the staged raw tile `rs` (index j): the hi + lo
// position pair (a 48-bit representation of the FP64 position, exact in
// double) and its FP64 mass and H^2.  The row's data come from the caller's
// shared-memory row cache `row` = {x, y, z, H^2} (stride `rstride`), its
// position rebuilt from its own hi + lo pair the same way, so coincident
// particles give dr == 0 exactly.
// Warp-cooperative FP64 evaluation of the near pairs (r < band * max H) that
// the checked loop flagged for one staged j-tile.  Each thread holds one 16-bit
// mask per (row k, sub-block sb) of its sources (bit = 4u + 2h + e for source
// j = 4 (phase + (sb*SUBQ + u) Q) + 2h + e, the checked loop's order); `wsum`
// marks its non-empty masks.  Per mask index (uniform over the warp) the set
// bits of all lanes are compacted into `cbuf` in lane order, evaluated one
// pair per lane (the row's data from the FP64 row cache of the owning thread,
// the source's from the raw staged tile: hi + lo position pair, FP64 m, H^2),
// and every owner sums its own results in list order in FP64, then folds the
// sums once per row into its compensated accumulators: deterministic, and
// all lanes busy whatever the distribution of near pairs over the rows.
template <int K, int Q, int TJ, int NT, bool NEWTON>
__device__ __noinline__ void near_eval(const SortedF64 D, int nkernel, int jbase, int ip0,
                                       int ip1, uint32_t wsum, const unsigned short *nbits,
                                       const double *s_row, float *s_acc, const float *rs,
                                       unsigned short *cbuf, double *res)
{
    constexpr int SUBQ = 4;
    constexpr int NSB = TJ / (16 * Q);
    constexpr double SA = Scales<NEWTON>::acc, SP = Scales<NEWTON>::pot;
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
            ff_add_d(acc[0], acc[4 * NT], sx / SA);
            ff_add_d(acc[NT], acc[5 * NT], sy / SA);
            ff_add_d(acc[2 * NT], acc[6 * NT], sz / SA);
            ff_add_d(acc[3 * NT], acc[7 * NT], sp / SP);
        }
    };
    while (rem) {
        const int wd = __ffs(rem) - 1;
        rem &= rem - 1;
        const int k = wd / NSB, sb = wd - k * NSB;
        if (k != kcur) {
            if (kcur >= 0) fold_row();
            kcur = k;
            sx = sy = sz = sp = 0.0;
        }
        const uint32_t m = ((wsum >> wd) & 1u) ? (uint32_t)nbits[wd * NT + tid] : 0u;
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
                cbuf[p] = (unsigned short)((lane << 4) | b);
            }
        }
        __syncwarp();
        const int ipk = (K > 1 && k) ? ip1 : ip0;
        const double *rowk = s_row + (k * 4) * NT + wb;
        for (int base = 0; base < total; base += 32) {
            const int g = base + lane;
            const int ent = g < total ? (int)cbuf[g] : lane << 4;
            const int ow = ent >> 4, bit = ent & 15;
            const int ipo = __shfl_sync(FULL, ipk, ow);
            if (g < total) {
                const int j = 4 * ((ow % Q) + (sb * SUBQ + (bit >> 2)) * Q) + (bit & 3);
                const double *row = rowk + ow;
                const double xj = (double)rs[j] + (double)rs[TJ + j];
                const double yj = (double)rs[2 * TJ + j] + (double)rs[3 * TJ + j];
                const double zj = (double)rs[4 * TJ + j] + (double)rs[5 * TJ + j];
                const PairOut o = pair_f64_fast(D, nkernel, ipo, jbase + j, xj - row[0],
                                                yj - row[NT], zj - row[2 * NT], rd[j], row[3 * NT],
                                                rd[TJ + j]);
                res2[lane] = make_double2(o.ax, o.ay);
                res2[32 + lane] = make_double2(o.az, o.pot);
            }
            __syncwarp();
            // this owner's entries of the round, in order, two at a time into
            // two partial sums (halves the dependent-add chains)
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

// Pairs with r < band * max(H_i, H_j) take the FP64 path (ComputeArgs::band2 =
// band^2, >= 1; default band 1, sphgrav_set_fp64_band).  Below H that is the
// softened near field (reference polynomials, which cancel in FP32); a band
// above 1 also moves the Newtonian terms between H and band*H, the largest
// far-field terms, to FP64.  The rows whose FP32 sums are ill-conditioned
// anyway (acceleration that cancels) are recomputed in FP64 by the refine,
// which is why band 1 suffices.  Scaling H^2 by band2 only moves pairs
// between two correct evaluations; with band2 >= 1 every r < H pair stays on
// the FP64 path.

// Shared-memory layout of one CTA (dynamic shared memory, byte offsets).
template <int W, int K, int Q, int TJ, int NS>
struct WsSmem {
    static constexpr int NT = W * 32;
    static constexpr int NMETA = TJ / META_J;
    // raw stage (TMA target): 8 float arrays x_hi x_lo y_hi y_lo z_hi z_lo m H^2,
    // then 2 double arrays m, H^2
    static constexpr int RAWSTAGE = 8 * TJ * 4 + 2 * TJ * 8;
    static constexpr int RAW = 0;                          // [NS] raw stages
    static constexpr int META = RAW + NS * RAWSTAGE;       // [NS][NMETA] JMeta (TMA targets)
    static constexpr int COMP = META + NS * NMETA * 32;    // [NS][5][TJ] floats
    static constexpr int BOX = COMP + NS * 5 * TJ * 4;     // [NS] TileBox
    static constexpr int ACC = BOX + NS * 32;              // [K*8][NT] floats
    static constexpr int NSB = TJ / (16 * Q);              // 16-source sub-blocks per thread
    static constexpr int NBITS = ACC + K * 8 * NT * 4;     // [K*NSB][NT] ushort near masks
    static constexpr int COOP = NBITS + (K * NSB * NT * 2 + 15) / 16 * 16;  // [W] near_eval buffers
    static constexpr int COOP_RES = 128 * 8;               // per warp: 4 x 32 doubles ...
    static constexpr int COOP_BUF = 32 * 16 * 2;           // ... and up to 32 x 16 entries
    static constexpr int ROW = COOP + W * (COOP_RES + COOP_BUF);  // [K][4][NT] double
    static constexpr int BAR = ROW + K * 4 * NT * 8;       // 3*NS mbarriers
    static constexpr int ITEM = BAR + 3 * NS * 8;          // 2 ints
    static constexpr int BYTES = ITEM + 16;
    static constexpr uint32_t TX = RAWSTAGE + NMETA * 32;  // bytes per tile
};

// Rows farther than SHIFT_H * H from their i-tile centre are listed for the
// FP64 refine (measured on the collision sweep: the coordinate shift stays
// below 1.3e-7 relative for |x'| < 8 H, reaches ~1e-6 beyond 24 H; 0-0.3% of
// the rows of the benchmark workloads lie beyond 8 H).
constexpr float SHIFT_H = 8.f;

// Phase accounting (diagnostic build, -DSG_PHASES): every warp reads clock64
// at its phase boundaries and lane 0 adds the elapsed cycles into a shared
// per-warp row, flushed to ComputeArgs::phases when the CTA leaves.
#ifdef SG_PHASES
bool phases_built() { return true; }
#define PH_MARK(i)                                                              \
    do {                                                                        \
        const long long t_ = clock64();                                         \
        if (lane == 0) s_ph[warp][(i)] += (unsigned long long)(t_ - ph_t);      \
        ph_t = t_;                                                              \
    } while (0)
#define PH_COUNT(i)                                 \
    do {                                            \
        if (lane == 0) s_ph[warp][(i)] += 1ull;     \
    } while (0)
#else
bool phases_built() { return false; }
#define PH_MARK(i) do {} while (0)
#define PH_COUNT(i) do {} while (0)
#endif

template <int W, int K, int Q, int TJ, int NS, bool NEWTON, int FQ>
__global__ void __launch_bounds__((W + 1) * 32) k_f32split(ComputeArgs a)
{
    static_assert(32 % Q == 0, "threads per row must divide a warp");
    constexpr int SUBQ = 4;                // quads per checked-loop sub-block (8 sources per lane)
    static_assert((TJ / 4) % (Q * SUBQ) == 0, "j-tile must hold whole sub-blocks");
    // far loop: FQ quads per sub-block (2 FQ sources per packed lane in one
    // FP32 FMA chain before the sub-block sum is added to the tile sum)
    static_assert((TJ / 4) % (Q * FQ) == 0, "j-tile must hold whole far sub-blocks");
    static_assert(TJ % 32 == 0, "producer lanes split the tile");
    using L = WsSmem<W, K, Q, TJ, NS>;
    constexpr int NT = L::NT;              // consumer threads
    constexpr int RPW = 32 / Q;            // row groups per warp
    constexpr int ITILE = NT * K / Q;      // rows per i-tile
    constexpr int NMETA = L::NMETA;
    static_assert(NMETA >= 1 && NMETA <= 32 && (NMETA & (NMETA - 1)) == 0,
                  "tile box reduction: one record per lane, a power of two");
    constexpr float SA = Scales<NEWTON>::acc, SP = Scales<NEWTON>::pot;
    constexpr uint32_t WAIT_LIMIT = 1u << 22;
    constexpr int NSB = L::NSB;
    static_assert(K * NSB <= 32, "one summary bit per near mask");
    static_assert(K <= 2, "near_eval takes the row slots of at most two rows");

    extern __shared__ __align__(128) unsigned char smem[];
    JMeta *s_meta = reinterpret_cast<JMeta *>(smem + L::META);
    float *comp = reinterpret_cast<float *>(smem + L::COMP);
    TileBox *s_box = reinterpret_cast<TileBox *>(smem + L::BOX);
    float *s_acc = reinterpret_cast<float *>(smem + L::ACC);
    unsigned short *s_nbits = reinterpret_cast<unsigned short *>(smem + L::NBITS);
    double *s_row = reinterpret_cast<double *>(smem + L::ROW);  // [K][4][NT]: x y z H^2
    uint64_t *bar_raw = reinterpret_cast<uint64_t *>(smem + L::BAR);  // [NS]
    uint64_t *bar_full = bar_raw + NS;                                 // [NS]
    uint64_t *bar_empty = bar_full + NS;                               // [NS]
    int *s_item = reinterpret_cast<int *>(smem + L::ITEM);             // [2]

    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const bool producer = (warp == W);
    const int grp = lane / Q, phase = lane % Q;
    const SortedF64 D = a.D;
    const SortedF32 F = a.F;
    const int nitems = a.nitems_dev ? *a.nitems_dev : a.nitems;
#ifdef SG_PHASES
    __shared__ unsigned long long s_ph[W + 1][PHASE_COUNTERS];
    for (int i = tid; i < (W + 1) * PHASE_COUNTERS; i += NT) (&s_ph[0][0])[i] = 0ull;
#endif

    if (tid == 0) {
        for (int s = 0; s < NS; s++) {
            mbar_init(&bar_raw[s], 1);     // TMA transaction count
            mbar_init(&bar_full[s], 32);   // every producer lane arrives
            mbar_init(&bar_empty[s], NT);  // every consumer thread arrives
        }
        fence_mbar_init();
    }
    __syncthreads();
#ifdef SG_PHASES
    long long ph_t = clock64();
#endif

    uint32_t g = 0;                        // tiles this CTA has passed through its ring
    bool failed = false;
    bool pending[NS];                      // producer lane 0: raw copies in flight per stage
    uint32_t pend_par[NS];                 // ... and the barrier phase they complete
#pragma unroll
    for (int s = 0; s < NS; s++) { pending[s] = false; pend_par[s] = 0u; }

    // bulk copies of set-local slots [jt, jt+TJ) (ring tile gt) into raw stage gt % NS;
    // the caller has seen that stage's consumers release it
    auto issue = [&](const SetDesc &S, int jt, uint32_t gt) {
        const int b = gt % NS;
        float *dst = reinterpret_cast<float *>(smem + L::RAW + b * L::RAWSTAGE);
        double *dstd = reinterpret_cast<double *>(dst + 8 * TJ);
        const int s0 = S.poff + jt;
        pending[b] = true;
        pend_par[b] = (gt / NS) & 1;
        fence_mbar_init();  // order earlier generic reads of the stage before the async writes
        mbar_arrive_expect_tx(&bar_raw[b], L::TX);
        const float *src[8] = {F.xh, F.xl, F.yh, F.yl, F.zh, F.zl, F.m, F.h2};
#pragma unroll
        for (int k = 0; k < 8; k++) bulk_g2s(dst + k * TJ, src[k] + s0, TJ * 4, &bar_raw[b]);
        bulk_g2s(dstd, D.m + s0, TJ * 8, &bar_raw[b]);
        bulk_g2s(dstd + TJ, D.h2 + s0, TJ * 8, &bar_raw[b]);
        bulk_g2s(s_meta + b * NMETA, a.jmeta + S.meta_off + jt / META_J, NMETA * 32, &bar_raw[b]);
    };
    auto stage_raw = [&](int s) -> const float * {
        return reinterpret_cast<const float *>(smem + L::RAW + s * L::RAWSTAGE);
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
        PH_MARK(producer ? PH_PROD_WAIT : PH_ITEM);

        if (producer) {
            // ------------------------------------------------ producer warp
            // A stage (raw tile + computed tile) is reused for ring tile gt once the
            // consumers released tile gt - NS: wait for that before each bulk copy.
            if (ntile > 0) {
                const bool ok = mbar_wait_bounded(&bar_empty[g % NS], ((g / NS) & 1) ^ 1, WAIT_LIMIT);
                PH_MARK(PH_PROD_WAIT);
                if (!__all_sync(0xffffffffu, ok)) {
                    if (lane == 0) atomicOr(a.err, DEVERR_TIMEOUT);
                    failed = true;
                } else if (lane == 0) {
                    issue(S, Wk.jb, g);
                }
                PH_MARK(PH_PROD_WORK);
            }
            for (int t = 0; t < ntile && !failed; t++) {
                const uint32_t gt = g + t;
                const int s = gt % NS;
                bool ok = true;
                if (t + 1 < ntile) {
                    const uint32_t gn = gt + 1;
                    ok = mbar_wait_bounded(&bar_empty[gn % NS], ((gn / NS) & 1) ^ 1, WAIT_LIMIT);
                    PH_MARK(PH_PROD_WAIT);
                    if (__all_sync(0xffffffffu, ok) && lane == 0) issue(S, Wk.jb + (t + 1) * TJ, gn);
                    PH_MARK(PH_PROD_WORK);
                }
                ok = ok && mbar_wait_bounded(&bar_raw[s], (gt / NS) & 1, WAIT_LIMIT);
                PH_MARK(PH_PROD_WAIT);
                if (ok && lane == 0) pending[s] = false;
                if (!__all_sync(0xffffffffu, ok)) {
                    if (lane == 0) atomicOr(a.err, DEVERR_TIMEOUT);
                    failed = true;
                    break;
                }
                // rewrite the tile relative to the i-tile centre (four sources
                // per lane and step, 16-byte shared-memory accesses)
                const float4 *rb4 = reinterpret_cast<const float4 *>(stage_raw(s));
                float4 *cx4 = reinterpret_cast<float4 *>(comp + s * 5 * TJ);
                constexpr int T4 = TJ / 4;
                auto rel = [](float4 h, float4 l, float ch, float cl) {
                    return make_float4(__fadd_rn(__fsub_rn(h.x, ch), __fsub_rn(l.x, cl)),
                                       __fadd_rn(__fsub_rn(h.y, ch), __fsub_rn(l.y, cl)),
                                       __fadd_rn(__fsub_rn(h.z, ch), __fsub_rn(l.z, cl)),
                                       __fadd_rn(__fsub_rn(h.w, ch), __fsub_rn(l.w, cl)));
                };
#pragma unroll
                for (int j = lane; j < T4; j += 32) {
                    cx4[j] = rel(rb4[j], rb4[T4 + j], C.chx, C.clx);
                    cx4[T4 + j] = rel(rb4[2 * T4 + j], rb4[3 * T4 + j], C.chy, C.cly);
                    cx4[2 * T4 + j] = rel(rb4[4 * T4 + j], rb4[5 * T4 + j], C.chz, C.clz);
                    cx4[3 * T4 + j] = rb4[6 * T4 + j];
                    const float4 h = rb4[7 * T4 + j];
                    cx4[4 * T4 + j] = make_float4(a.band2 * h.x, a.band2 * h.y, a.band2 * h.z,
                                                  a.band2 * h.w);  // (band H)^2
                }
                // the tile's box relative to the centre: one record per lane,
                // then a min/max reduction over the NMETA lanes (exact, so
                // independent of the order)
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
                                // rounding of the float centres and of the staged
                                // coordinates: widen by 2^-20 of the magnitudes
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
                            lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
                            hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
                        }
                        h2m = fmaxf(h2m, __shfl_xor_sync(0xffffffffu, h2m, o));
                        empty &= __shfl_xor_sync(0xffffffffu, empty, o);
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
                PH_MARK(PH_PROD_WORK);
            }
        } else {
            // ----------------------------------------------- consumer warps
            int ip[K];
            bool act[K];
            f2 xi[K], yi[K], zi[K];
            f2 g2[K];  // sum over tiles of |FP32 tile sum|^2 per packed lane (error scale)
            bool shifted[K];  // row far from the i-tile centre (see below)
            float h2i[K];
            float wlo[3] = {INFINITY, INFINITY, INFINITY};
            float whi[3] = {-INFINITY, -INFINITY, -INFINITY};
            float wh2 = 0.f;
#pragma unroll
            for (int k = 0; k < K; k++) {
                const int li = warp * RPW * K + k * RPW + grp;
                const int r = Wk.tile * ITILE + li;
                act[k] = r < S.ni;
                ip[k] = act[k] ? a.ilist[S.ioff + r] : 0;
                float x = 1.0e15f, y = 1.0e15f, z = -1.0e15f, h2 = 0.f;
                if (act[k]) {
                    const int sl = ip[k];
                    x = __fadd_rn(__fsub_rn(F.xh[sl], C.chx), __fsub_rn(F.xl[sl], C.clx));
                    y = __fadd_rn(__fsub_rn(F.yh[sl], C.chy), __fsub_rn(F.yl[sl], C.cly));
                    z = __fadd_rn(__fsub_rn(F.zh[sl], C.chz), __fsub_rn(F.zl[sl], C.clz));
                    h2 = a.band2 * F.h2[sl];
                    // FP64 row data for the deferred near pairs
                    double *rw = s_row + (k * 4) * NT + tid;
                    rw[0] = (double)F.xh[sl] + (double)F.xl[sl];
                    rw[NT] = (double)F.yh[sl] + (double)F.yl[sl];
                    rw[2 * NT] = (double)F.zh[sl] + (double)F.zl[sl];
                    rw[3 * NT] = D.h2[sl];
                    wlo[0] = fminf(wlo[0], x); whi[0] = fmaxf(whi[0], x);
                    wlo[1] = fminf(wlo[1], y); whi[1] = fmaxf(whi[1], y);
                    wlo[2] = fminf(wlo[2], z); whi[2] = fmaxf(whi[2], z);
                    wh2 = fmaxf(wh2, h2);
                }
                xi[k] = pk(x, x);
                yi[k] = pk(y, y);
                zi[k] = pk(z, z);
                h2i[k] = h2;
                g2[k] = pk(0.f, 0.f);
                // The FP32 rounding of a row's tile-relative coordinate shifts the
                // row by up to ~1e-7 |x'|, a coherent error (tidal field times the
                // shift) that grows with |x'| / H; i-tiles whose rows span a
                // space-filling-curve exit leave a few rows tens of H from the
                // centre.  Such rows (|x'| > SHIFT_H H) get an infinite error
                // scale, so the refine recomputes them in FP64.
                shifted[k] = act[k] && x * x + y * y + z * z > SHIFT_H * SHIFT_H * F.h2[ip[k]];
#pragma unroll
                for (int c = 0; c < 8; c++) s_acc[(k * 8 + c) * NT + tid] = 0.f;
            }
#pragma unroll
            for (int d = 0; d < 3; d++) {
                for (int o = 16; o > 0; o >>= 1) {
                    wlo[d] = fminf(wlo[d], __shfl_xor_sync(0xffffffffu, wlo[d], o));
                    whi[d] = fmaxf(whi[d], __shfl_xor_sync(0xffffffffu, whi[d], o));
                }
            }
            for (int o = 16; o > 0; o >>= 1) wh2 = fmaxf(wh2, __shfl_xor_sync(0xffffffffu, wh2, o));
            const bool warp_rows = wlo[0] <= whi[0];
            wh2 = wh2 * 1.00001f;
            float slack[3];
#pragma unroll
            for (int d = 0; d < 3; d++) slack[d] = 9.5367e-7f * fmaxf(fabsf(wlo[d]), fabsf(whi[d]));
            PH_MARK(PH_ROWS);
            PH_COUNT(PH_N_ITEMS);

            for (int t = 0; t < ntile; t++) {
                const uint32_t gt = g + t;
                const int s = gt % NS;
                const bool ok = mbar_wait_bounded(&bar_full[s], (gt / NS) & 1, WAIT_LIMIT);
                PH_MARK(PH_WAIT_FULL);
                if (!__all_sync(0xffffffffu, ok)) {
                    if (lane == 0) atomicOr(a.err, DEVERR_TIMEOUT);
                    failed = true;
                    break;
                }
                const float *s_x = comp + s * 5 * TJ;
                const float *s_y = s_x + TJ, *s_z = s_y + TJ, *s_m = s_z + TJ, *s_h = s_m + TJ;
                const int jt = Wk.jb + t * TJ;
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
                    // tile sums: two levels (8-source sub-blocks -> tile)
                    f2 tx[K], ty[K], tz[K], tp[K];
#pragma unroll
                    for (int k = 0; k < K; k++) tx[k] = ty[k] = tz[k] = tp[k] = pk(0.f, 0.f);
                    uint32_t wsum = 0;  // non-empty near masks of this thread (bit k*NSB + sb)

                    if (far) {
                        // the potential terms are all positive (no cancellation), so
                        // they go straight into the tile sum; the acceleration
                        // components, which cancel, keep the sub-block sums
                        for (int base = phase; base < TJ / 4; base += Q * FQ) {
                            f2 ax[K], ay[K], az[K];
#pragma unroll
                            for (int k = 0; k < K; k++) ax[k] = ay[k] = az[k] = pk(0.f, 0.f);
#pragma unroll  // whole sub-block: +5% at N=1M over unroll 2
                            for (int u = 0; u < FQ; u++) {
                                const int qd = base + u * Q;
                                const ulonglong2 X = *reinterpret_cast<const ulonglong2 *>(&s_x[4 * qd]);
                                const ulonglong2 Y = *reinterpret_cast<const ulonglong2 *>(&s_y[4 * qd]);
                                const ulonglong2 Z = *reinterpret_cast<const ulonglong2 *>(&s_z[4 * qd]);
                                const ulonglong2 M = *reinterpret_cast<const ulonglong2 *>(&s_m[4 * qd]);
#pragma unroll
                                for (int k = 0; k < K; k++) {
                                    f2 dx, dy, dz, r2;
                                    geom2(X.x, Y.x, Z.x, xi[k], yi[k], zi[k], dx, dy, dz, r2);
                                    accum2<NEWTON>(dx, dy, dz, r2, M.x, ax[k], ay[k], az[k], tp[k]);
                                    geom2(X.y, Y.y, Z.y, xi[k], yi[k], zi[k], dx, dy, dz, r2);
                                    accum2<NEWTON>(dx, dy, dz, r2, M.y, ax[k], ay[k], az[k], tp[k]);
                                }
                            }
#pragma unroll
                            for (int k = 0; k < K; k++) {
                                tx[k] = add2(tx[k], ax[k]);
                                ty[k] = add2(ty[k], ay[k]);
                                tz[k] = add2(tz[k], az[k]);
                            }
                        }
                    } else {
                        // near pairs are masked here and flagged in this thread's
                        // per-(row, sub-block) masks; FP64 evaluation runs after the loop
                        for (int base = phase, sb = 0; base < TJ / 4; base += Q * SUBQ, sb++) {
                            f2 ax[K], ay[K], az[K], pp[K];
                            uint32_t mb[K];
#pragma unroll
                            for (int k = 0; k < K; k++) {
                                ax[k] = ay[k] = az[k] = pp[k] = pk(0.f, 0.f);
                                mb[k] = 0u;
                            }
                            for (int u = 0; u < SUBQ; u++) {
                                const int qd = base + u * Q;
                                const ulonglong2 X = *reinterpret_cast<const ulonglong2 *>(&s_x[4 * qd]);
                                const ulonglong2 Y = *reinterpret_cast<const ulonglong2 *>(&s_y[4 * qd]);
                                const ulonglong2 Z = *reinterpret_cast<const ulonglong2 *>(&s_z[4 * qd]);
                                const ulonglong2 M = *reinterpret_cast<const ulonglong2 *>(&s_m[4 * qd]);
                                const float4 H = *reinterpret_cast<const float4 *>(&s_h[4 * qd]);
#pragma unroll
                                for (int k = 0; k < K; k++) {
#pragma unroll
                                    for (int h = 0; h < 2; h++) {
                                        f2 dx, dy, dz, r2;
                                        geom2(h ? X.y : X.x, h ? Y.y : Y.x, h ? Z.y : Z.x, xi[k],
                                              yi[k], zi[k], dx, dy, dz, r2);
                                        f2 mj = h ? M.y : M.x;
                                        float ra, rb;
                                        upk(r2, ra, rb);
                                        const float ha = h ? H.z : H.x, hb = h ? H.w : H.y;
                                        const bool na = ra < fmaxf(h2i[k], ha);
                                        const bool nb = rb < fmaxf(h2i[k], hb);
                                        if (na || nb) {
                                            mb[k] |= ((na ? 1u : 0u) | (nb ? 2u : 0u)) << (4 * u + 2 * h);
                                            float ma, mb;
                                            upk(mj, ma, mb);
                                            mj = pk(na ? 0.f : ma, nb ? 0.f : mb);
                                            r2 = pk(na ? 1.f : ra, nb ? 1.f : rb);
                                        }
                                        accum2<NEWTON>(dx, dy, dz, r2, mj, ax[k], ay[k], az[k], pp[k]);
                                    }
                                }
                            }
#pragma unroll
                            for (int k = 0; k < K; k++) {
                                tx[k] = add2(tx[k], ax[k]);
                                ty[k] = add2(ty[k], ay[k]);
                                tz[k] = add2(tz[k], az[k]);
                                tp[k] = add2(tp[k], pp[k]);
                                if (act[k] && mb[k]) {
                                    s_nbits[(k * NSB + sb) * NT + tid] = (unsigned short)mb[k];
                                    wsum |= 1u << (k * NSB + sb);
                                }
                            }
                        }
                    }
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
                    PH_MARK(far ? PH_FAR : PH_CHECKED);
                    PH_COUNT(far ? PH_N_FAR : PH_N_CHECKED);
                    // deferred near-field pairs in FP64 (far is uniform over the warp)
                    if (!far && __any_sync(0xffffffffu, wsum != 0u)) {
                        unsigned char *cb = smem + L::COOP + warp * (L::COOP_RES + L::COOP_BUF);
                        near_eval<K, Q, TJ, NT, NEWTON>(
                            D, a.nkernel, S.poff + jt, ip[0], ip[K > 1 ? K - 1 : 0], wsum, s_nbits,
                            s_row, s_acc, stage_raw(s),
                            reinterpret_cast<unsigned short *>(cb + L::COOP_RES),
                            reinterpret_cast<double *>(cb));
                        PH_MARK(PH_NEAR);
                        PH_COUNT(PH_N_NEAR);
                    }
                }
                mbar_arrive(&bar_empty[s]);
            }
            if (!failed) {
                // combine the Q threads of a row (fixed order), convert, write FP64 partials
                __syncwarp();
                const size_t slot = (size_t)Wk.slot;
                double *p = a.partials + slot * 4 * ITILE;
                if (a.gpart) {
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        float ga, gb;
                        upk(g2[k], ga, gb);
                        float gs = ga + gb;
#pragma unroll
                        for (int o = 1; o < Q; o <<= 1) gs += __shfl_xor_sync(0xffffffffu, gs, o);
                        if (phase == 0 && act[k])
                            a.gpart[slot * ITILE + warp * RPW * K + k * RPW + grp] =
                                shifted[k] ? INFINITY : gs * (SA * SA);
                    }
                }
                if (phase == 0) {
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        if (!act[k]) continue;
                        const int li = warp * RPW * K + k * RPW + grp;
#pragma unroll
                        for (int c = 0; c < 4; c++) {
                            float h = s_acc[(k * 8 + c) * NT + tid];
                            float l = s_acc[(k * 8 + 4 + c) * NT + tid];
                            for (int ph = 1; ph < Q; ph++) {
                                ff_add(h, l, s_acc[(k * 8 + c) * NT + tid + ph]);
                                l = __fadd_rn(l, s_acc[(k * 8 + 4 + c) * NT + tid + ph]);
                            }
                            p[c * ITILE + li] = ((double)h + (double)l) * (double)(c < 3 ? SA : SP);
                        }
                    }
                }
            }
            PH_MARK(PH_END);
        }
        g += ntile;
    }
#ifdef SG_PHASES
    if (a.phases && lane == 0)
        for (int i = 0; i < PHASE_COUNTERS; i++) atomicAdd(a.phases + i, s_ph[warp][i]);
#endif
    // never leave with bulk copies in flight into this CTA's shared memory
    if (producer && lane == 0) {
        for (int b = 0; b < NS; b++)
            if (pending[b]) mbar_wait_bounded(&bar_raw[b], pend_par[b], WAIT_LIMIT);
    }
}

// name, consumer warps W, rows per thread K, threads per row Q, j-tile TJ,
// stages NS, Newton step, quads per far-loop sub-block FQ.  (Two far
// sub-blocks per loop iteration were measured slower: 1M 511.7 vs 488.7 ms.)
#define SG_F32_VARIANTS(X)                                              \
    X(12, 2, 1, 256, 7, false, 4, "f32split_w12_k2_q1_tj256_ns7")        \
    X(15, 2, 1, 256, 4, false, 4, "f32split_w15_k2_q1_tj256")            \
    X(12, 1, 1, 256, 7, false, 4, "f32split_w12_k1_q1_tj256_ns7")        \
    X(15, 1, 2, 256, 4, false, 4, "f32split_w15_k1_q2_tj256")            \
    X(8, 1, 4, 256, 4, false, 4, "f32split_w8_k1_q4_tj256")              \
    X(12, 1, 4, 256, 7, false, 4, "f32split_w12_k1_q4_tj256_ns7")        \
    X(15, 2, 1, 256, 4, true, 4, "f32split_w15_k2_q1_tj256_newton")      \
    X(15, 1, 2, 256, 4, true, 4, "f32split_w15_k1_q2_tj256_newton")      \
    X(8, 1, 4, 256, 4, true, 4, "f32split_w8_k1_q4_tj256_newton")        \
    X(12, 2, 1, 256, 7, false, 8, "f32split_w12_k2_q1_tj256_ns7_fq8")    \
    X(12, 1, 1, 256, 7, false, 8, "f32split_w12_k1_q1_tj256_ns7_fq8")

#define SG_INFO(W, K, Q, TJ, NS, NW, FQ, NAME) {1, (W + 1) * 32, K, Q, TJ, NW ? 1 : 0, NAME, W * 32 * K / Q},
static const VariantInfo kF32Variants[] = {SG_F32_VARIANTS(SG_INFO)};
#undef SG_INFO
#define SG_PTR(W, K, Q, TJ, NS, NW, FQ, NAME) (const void *)k_f32split<W, K, Q, TJ, NS, NW, FQ>,
static const void *kF32Kernels[] = {SG_F32_VARIANTS(SG_PTR)};
#undef SG_PTR
#define SG_SMEM(W, K, Q, TJ, NS, NW, FQ, NAME) WsSmem<W, K, Q, TJ, NS>::BYTES,
static const int kF32Smem[] = {SG_F32_VARIANTS(SG_SMEM)};
#undef SG_SMEM
constexpr int kNF32 = sizeof(kF32Variants) / sizeof(kF32Variants[0]);

int f32_variant_count() { return kNF32; }
const VariantInfo &f32_variant_info(int v) { return kF32Variants[v]; }
const void *f32_kernel(int v) { return kF32Kernels[v]; }
int f32_smem_bytes(int v) { return kF32Smem[v]; }

// Opt in to more than 48 KB of dynamic shared memory (once per variant and
// device; the attribute belongs to the device's context).
cudaError_t f32_prepare(int v)
{
    constexpr int MAXDEV = 64;
    static std::atomic<bool> done[MAXDEV][kNF32];
    if (v < 0 || v >= kNF32) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const bool track = dev >= 0 && dev < MAXDEV;
    if (track && done[dev][v].load(std::memory_order_acquire)) return cudaSuccess;
    e = cudaFuncSetAttribute(kF32Kernels[v], cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kF32Smem[v]);
    if (e == cudaSuccess && track) done[dev][v].store(true, std::memory_order_release);
    return e;
}

cudaError_t launch_f32(int v, int grid, const ComputeArgs &a, cudaStream_t st)
{
    cudaError_t e = f32_prepare(v);
    if (e != cudaSuccess) return e;
    int idx = 0;
#define SG_CASE(W, K, Q, TJ, NS, NW, FQ, NAME)                                                \
    if (v == idx) {                                                                           \
        k_f32split<W, K, Q, TJ, NS, NW, FQ><<<grid, (W + 1) * 32, WsSmem<W, K, Q, TJ, NS>::BYTES, st>>>(a); \
        ++g_launches;                                                                         \
        return cudaGetLastError();                                                            \
    }                                                                                         \
    ++idx;
    SG_F32_VARIANTS(SG_CASE)
#undef SG_CASE
    return cudaErrorInvalidValue;
}

}  // namespace sg
