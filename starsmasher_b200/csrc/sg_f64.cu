// sg_f64.cu -- plain FP64 direct-summation kernel.
//
// Same pair formulas and branch rule as the reference's CPU path
// (parallel_bleeding_edge/src/cpu_grav.f:46-157): Newtonian when
// r^2 >= max(H_i^2, H_j^2), otherwise the softened pair of pair_f64_slots.
// Work decomposition (persistent CTAs over a device queue of
// (set, i-tile, j-chunk) items):
//   * K rows per thread kept in registers (a warp owns 32 K consecutive
//     sorted rows, so its rows form a compact box), NT threads per CTA;
//   * j-tiles of TJ sources staged in shared memory as SoA doubles
//     (x, y, z, m, H^2) by 1-D bulk async copies (cp.async.bulk, the TMA
//     engine; no multicast) into an NS-stage ring completing on mbarriers,
//     together with the tile's bounding-box records;
//   * per (warp, tile) a box test: when every pair of the warp's rows with
//     the tile's sources is Newtonian (r^2 > max H^2 for all of them), the
//     tile runs a loop without the per-pair branch;
//   * per row, each j-tile's plain FP64 sums fold into TwoSum-compensated
//     running sums; one FP64 partial sum per (row, j-chunk), merged in chunk
//     order by k_merge.
// Far pairs take 1/r from the PTX rsqrt.approx.ftz.f64 seed y0 refined by one
// third-order step of the series (1 - e)^(-1/2) = 1 + e/2 + 3e^2/8 + O(e^3),
// e = 1 - r^2 y0^2 (Householder's method for x^(-1/2)): 5 FP64 operations
// to full precision.
#include "sg_launch.h"

namespace sg {

__device__ __forceinline__ double rsqrt_approx_f64(double x)
{
    double r;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    return r;
}

// 1/sqrt(r2) for r2 > 0 (normal range): seed and one third-order correction.
__device__ __forceinline__ double rsqrt_f64(double r2)
{
    const double y0 = rsqrt_approx_f64(r2);
    const double e = fma(-(r2 * y0), y0, 1.0);
    const double q = e * fma(e, 0.375, 0.5);
    return fma(y0, q, y0);
}

// Resident blocks per SM the register budget is sized for: 64K registers /
// (NT * MINB) per thread (K = 1: 128, K = 2: 170, K >= 3: 255 at NT = 128).
// MB > 0 overrides the count.
template <int NT, int K, int MB>
struct F64Occ {
    static constexpr int MINB = MB > 0 ? MB : (K >= 3 ? 2 : (K == 2 ? 3 : 4)) * 128 / NT;
};

template <int NT, int K, int TJ, int NS, int U, int MB>
__global__ void __launch_bounds__(NT, F64Occ<NT, K, MB>::MINB) k_fp64(ComputeArgs a)
{
    static_assert(TJ % META_J == 0, "j-tile must hold whole metadata records");
    constexpr int ITILE = NT * K;
    constexpr int NMETA = TJ / META_J;
    constexpr uint32_t TX = 5 * TJ * 8 + NMETA * (uint32_t)sizeof(JMeta);
    constexpr uint32_t WAIT_LIMIT = 1u << 22;
    __shared__ __align__(128) double s_src[NS][5][TJ];  // x y z m H^2
    __shared__ __align__(16) JMeta s_meta[NS][NMETA];
    __shared__ __align__(8) uint64_t s_bar[NS];
    __shared__ double s_lo[4][K][NT];  // low parts of the compensated running sums
    __shared__ int s_item;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const SortedF64 D = a.D;
    const int nitems = a.nitems_dev ? *a.nitems_dev : a.nitems;

    if (tid == 0) {
        for (int s = 0; s < NS; s++) mbar_init(&s_bar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();

    uint32_t g = 0;          // tiles this CTA has passed through its ring
    bool failed = false;
    bool pending[NS];        // thread 0: copies in flight per stage ...
    uint32_t pend_par[NS];   // ... and the phase they complete
#pragma unroll
    for (int s = 0; s < NS; s++) { pending[s] = false; pend_par[s] = 0u; }

    // bulk copies of set-local sorted slots [jt, jt + TJ) into stage gt % NS
    auto issue = [&](const SetDesc &S, int jt, uint32_t gt) {
        const int b = gt % NS;
        const int s0 = S.poff + jt;
        pending[b] = true;
        pend_par[b] = (gt / NS) & 1;
        fence_mbar_init();  // earlier generic reads of the stage before the async writes
        mbar_arrive_expect_tx(&s_bar[b], TX);
        const double *src[5] = {D.x, D.y, D.z, D.m, D.h2};
#pragma unroll
        for (int q = 0; q < 5; q++) bulk_g2s(s_src[b][q], src[q] + s0, TJ * 8, &s_bar[b]);
        bulk_g2s(s_meta[b], a.jmeta + S.meta_off + jt / META_J, NMETA * (uint32_t)sizeof(JMeta),
                 &s_bar[b]);
    };

    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.head, 1);
        if (__syncthreads_or(failed)) break;
        const int it = s_item;
        if (it >= nitems) break;
        const WorkItem W = a.items[it];
        const SetDesc S = a.sets[W.set];
        const int ntile = (W.je - W.jb) / TJ;
        if (tid == 0)
            for (int t = 0; t < NS && t < ntile; t++) issue(S, W.jb + t * TJ, g + t);

        int ip[K];
        bool act[K];
        double xi[K], yi[K], zi[K], hi2[K];
        double ax[K], ay[K], az[K], pot[K];  // this j-tile's sums
        double sh[K][4];                     // compensated running sums: high parts (low: s_lo)
        double wlo[3] = {INFINITY, INFINITY, INFINITY}, whi[3] = {-INFINITY, -INFINITY, -INFINITY};
        double wh2 = 0.0;
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int r = W.tile * ITILE + warp * 32 * K + k * 32 + lane;
            act[k] = r < S.ni;
            ip[k] = act[k] ? a.ilist[S.ioff + r] : -1;
            xi[k] = act[k] ? D.x[ip[k]] : FAR_POS;
            yi[k] = act[k] ? D.y[ip[k]] : FAR_POS;
            zi[k] = act[k] ? D.z[ip[k]] : -FAR_POS;
            hi2[k] = act[k] ? D.h2[ip[k]] : 0.0;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                sh[k][c] = 0.0;
                s_lo[c][k][tid] = 0.0;
            }
            if (act[k]) {
                wlo[0] = fmin(wlo[0], xi[k]); whi[0] = fmax(whi[0], xi[k]);
                wlo[1] = fmin(wlo[1], yi[k]); whi[1] = fmax(whi[1], yi[k]);
                wlo[2] = fmin(wlo[2], zi[k]); whi[2] = fmax(whi[2], zi[k]);
                wh2 = fmax(wh2, hi2[k]);
            }
        }
#pragma unroll
        for (int d = 0; d < 3; d++) {
            for (int o = 16; o > 0; o >>= 1) {
                wlo[d] = fmin(wlo[d], __shfl_xor_sync(0xffffffffu, wlo[d], o));
                whi[d] = fmax(whi[d], __shfl_xor_sync(0xffffffffu, whi[d], o));
            }
        }
        for (int o = 16; o > 0; o >>= 1) wh2 = fmax(wh2, __shfl_xor_sync(0xffffffffu, wh2, o));
        const bool warp_rows = wlo[0] <= whi[0];
        // the warp's box in FP32, rounded outward, for the per-tile far test
        // (FP32 keeps the test off the FP64 pipe, which the pair loop saturates)
        float flo[3], fhi[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            flo[d] = warp_rows ? __double2float_rd(wlo[d]) : 0.f;
            fhi[d] = warp_rows ? __double2float_ru(whi[d]) : 0.f;
        }
        const float fwh2 = __double2float_ru(wh2);

        for (int t = 0; t < ntile; t++) {
            const uint32_t gt = g + t;
            const int s = gt % NS;
            const bool ok = mbar_wait_bounded(&s_bar[s], (gt / NS) & 1, WAIT_LIMIT);
            if (ok && tid == 0) pending[s] = false;
            if (ok && warp_rows) {
                const double *sx = s_src[s][0], *sy = s_src[s][1], *sz = s_src[s][2];
                const double *sm = s_src[s][3], *shj = s_src[s][4];
#pragma unroll
                for (int k = 0; k < K; k++) ax[k] = ay[k] = az[k] = pot[k] = 0.0;
                // box test: the gap between the warp's rows and each record's
                // box bounds r from below; far when it exceeds every H.  In
                // FP32 with the gap shrunk by 2^-20 of the coordinates'
                // magnitude and the squared gap by 1e-5, which covers the
                // roundings of the box arithmetic.
                bool far = true;
#pragma unroll
                for (int r = 0; r < NMETA; r++) {
                    const JMeta M = s_meta[s][r];
                    if (M.ex < 0.f) continue;  // no particle
                    const float c[3] = {M.cx, M.cy, M.cz}, e[3] = {M.ex, M.ey, M.ez};
                    float d2 = 0.f;
#pragma unroll
                    for (int d = 0; d < 3; d++) {
                        const float slack = 9.5367e-7f * (fabsf(c[d]) + e[d] + fabsf(flo[d]) + fabsf(fhi[d]));
                        const float gap = fmaxf(0.f, fmaxf((c[d] - e[d]) - fhi[d], flo[d] - (c[d] + e[d])) - slack);
                        d2 = fmaf(gap, gap, d2);
                    }
                    far = far && d2 > fmaxf(fwh2, M.h2max) * 1.00001f;
                }
                if (far) {
#pragma unroll U
                    for (int j = 0; j < TJ; j++) {
                        const double xj = sx[j], yj = sy[j], zj = sz[j], mj = sm[j];
#pragma unroll
                        for (int k = 0; k < K; k++) {
                            const double dx = xj - xi[k], dy = yj - yi[k], dz = zj - zi[k];
                            const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
                            const double y = rsqrt_f64(r2);
                            const double mr = mj * y;
                            const double mr3 = mr * (y * y);
                            ax[k] = fma(mr3, dx, ax[k]);
                            ay[k] = fma(mr3, dy, ay[k]);
                            az[k] = fma(mr3, dz, az[k]);
                            pot[k] -= mr;
                        }
                    }
                } else {
                    const int jt = W.jb + t * TJ;
                    for (int j = 0; j < TJ; j++) {
                        const double xj = sx[j], yj = sy[j], zj = sz[j], mj = sm[j], hj = shj[j];
#pragma unroll
                        for (int k = 0; k < K; k++) {
                            const double dx = xj - xi[k], dy = yj - yi[k], dz = zj - zi[k];
                            const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
                            if (r2 >= fmax(hi2[k], hj)) {
                                const double y = rsqrt_f64(r2);
                                const double mr = mj * y;
                                const double mr3 = mr * (y * y);
                                ax[k] = fma(mr3, dx, ax[k]);
                                ay[k] = fma(mr3, dy, ay[k]);
                                az[k] = fma(mr3, dz, az[k]);
                                pot[k] -= mr;
                            } else if (act[k]) {
                                const PairOut o = pair_f64_slots(D, a.nkernel, ip[k], S.poff + jt + j);
                                ax[k] += o.ax;
                                ay[k] += o.ay;
                                az[k] += o.az;
                                pot[k] += o.pot;
                            }
                        }
                    }
                }
                // the tile's sums (a few hundred terms, plain FP64) go into the
                // row's compensated running sums: FP64 rounding then grows with
                // the tile sums, not with a running sum over the whole j-range
                // (which at a particle whose acceleration cancels is much
                // larger than the result)
#pragma unroll
                for (int k = 0; k < K; k++) {
                    const double tv[4] = {ax[k], ay[k], az[k], pot[k]};
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        const double hsum = sh[k][c] + tv[c];
                        const double bp = hsum - sh[k][c];
                        s_lo[c][k][tid] += (sh[k][c] - (hsum - bp)) + (tv[c] - bp);
                        sh[k][c] = hsum;
                    }
                }
            }
            // every thread is done with stage s (or a wait gave up)
            if (__syncthreads_or(!ok)) {
                if (tid == 0) atomicOr(a.err, DEVERR_TIMEOUT);
                failed = true;
                break;
            }
            if (tid == 0 && t + NS < ntile) issue(S, W.jb + (t + NS) * TJ, gt + NS);
        }
        g += ntile;
        if (failed) break;

        double *p = a.partials + (size_t)W.slot * 4 * ITILE;
#pragma unroll
        for (int k = 0; k < K; k++) {
            if (act[k]) {
                const int li = warp * 32 * K + k * 32 + lane;
                p[li] = sh[k][0] + s_lo[0][k][tid];
                p[ITILE + li] = sh[k][1] + s_lo[1][k][tid];
                p[2 * ITILE + li] = sh[k][2] + s_lo[2][k][tid];
                p[3 * ITILE + li] = sh[k][3] + s_lo[3][k][tid];
            }
        }
    }
    // never leave with bulk copies in flight into this CTA's shared memory
    if (tid == 0) {
        for (int b = 0; b < NS; b++)
            if (pending[b]) mbar_wait_bounded(&s_bar[b], pend_par[b], WAIT_LIMIT);
    }
}

// name, threads NT, rows per thread K, j-tile TJ, stages NS, far-loop unroll U,
// resident blocks per SM the registers are sized for MB (0: by K and NT).
// Variants 0 and 12 (one row per thread, 128- or 64-source tiles) also
// recompute the split-FP32 refine rows (64-source tiles for sets of at most
// 65,536 particles: shorter j-chunks spread a few rows' near pairs over more
// blocks).
#define SG_F64_VARIANTS(X)                                   \
    X(128, 1, 128, 3, 2, 0, "fp64_nt128_k1_tj128")           \
    X(128, 2, 128, 3, 2, 0, "fp64_nt128_k2_tj128")           \
    X(128, 4, 128, 3, 2, 0, "fp64_nt128_k4_tj128")           \
    X(256, 1, 128, 3, 2, 0, "fp64_nt256_k1_tj128")           \
    X(128, 2, 256, 3, 2, 0, "fp64_nt128_k2_tj256")           \
    X(128, 4, 256, 3, 2, 0, "fp64_nt128_k4_tj256")           \
    X(128, 2, 256, 3, 4, 0, "fp64_nt128_k2_tj256_u4")        \
    X(128, 3, 256, 3, 2, 0, "fp64_nt128_k3_tj256")           \
    X(64, 2, 256, 3, 2, 0, "fp64_nt64_k2_tj256")             \
    X(32, 2, 128, 3, 2, 0, "fp64_nt32_k2_tj128")             \
    X(128, 2, 256, 3, 1, 4, "fp64_nt128_k2_tj256_u1_b4")     \
    X(64, 3, 256, 3, 2, 0, "fp64_nt64_k3_tj256")             \
    X(128, 1, 64, 3, 2, 0, "fp64_nt128_k1_tj64")            \
    X(32, 1, 128, 3, 2, 0, "fp64_nt32_k1_tj128")             \
    X(64, 1, 128, 3, 2, 0, "fp64_nt64_k1_tj128")

#define SG_INFO(NT, K, TJ, NS, U, MB, NAME) {0, NT, K, 1, TJ, 0, NAME, NT * K},
static const VariantInfo kF64Variants[] = {SG_F64_VARIANTS(SG_INFO)};
#undef SG_INFO
#define SG_PTR(NT, K, TJ, NS, U, MB, NAME) (const void *)k_fp64<NT, K, TJ, NS, U, MB>,
static const void *kF64Kernels[] = {SG_F64_VARIANTS(SG_PTR)};
#undef SG_PTR
constexpr int kNF64 = sizeof(kF64Variants) / sizeof(kF64Variants[0]);

int f64_variant_count() { return kNF64; }
const VariantInfo &f64_variant_info(int v) { return kF64Variants[v]; }
const void *f64_kernel(int v) { return kF64Kernels[v]; }

cudaError_t launch_f64(int v, int grid, const ComputeArgs &a, cudaStream_t st)
{
    int idx = 0;
#define SG_CASE(NT, K, TJ, NS, U, MB, NAME)                        \
    if (v == idx) {                                                \
        k_fp64<NT, K, TJ, NS, U, MB><<<grid, NT, 0, st>>>(a);      \
        ++g_launches;                                              \
        return cudaGetLastError();                                 \
    }                                                              \
    ++idx;
    SG_F64_VARIANTS(SG_CASE)
#undef SG_CASE
    return cudaErrorInvalidValue;
}

}  // namespace sg
