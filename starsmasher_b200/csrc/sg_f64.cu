// sg_f64.cu -- plain FP64 direct-summation kernel.
//
// Same pair formulas and branch rule as the reference's CPU path
// (parallel_bleeding_edge/src/cpu_grav.f:46-157): Newtonian when
// r^2 >= max(H_i^2, H_j^2), otherwise the softened pair of pair_f64_slots.
// Work decomposition (persistent CTAs over a device queue of
// (set, i-tile, j-chunk) items):
//   * K rows per thread kept in registers, NT threads per CTA;
//   * j-tiles of TJ particles staged in shared memory as SoA doubles
//     (x, y, z, m, H^2), the next tile prefetched into registers while the
//     current one is summed;
//   * one FP64 partial sum per (row, j-chunk), merged in chunk order by
//     k_merge.
#include "sg_launch.h"

namespace sg {

template <int NT, int K, int TJ>
__global__ void __launch_bounds__(NT) k_fp64(ComputeArgs a)
{
    static_assert(TJ % NT == 0, "j-tile must be a multiple of the block");
    constexpr int ITILE = NT * K;
    constexpr int LPT = TJ / NT;  // j loads per thread per tile
    __shared__ double s_x[TJ], s_y[TJ], s_z[TJ], s_m[TJ], s_h[TJ];
    __shared__ int s_item;
    const int tid = threadIdx.x;
    const SortedF64 D = a.D;

    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.head, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= a.nitems) break;
        const WorkItem W = a.items[it];
        const SetDesc S = a.sets[W.set];

        int ip[K];
        bool act[K];
        double xi[K], yi[K], zi[K], hi2[K];
        double ax[K], ay[K], az[K], pot[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int r = W.tile * ITILE + k * NT + tid;
            act[k] = r < S.ni;
            ip[k] = act[k] ? a.ilist[S.ioff + r] : -1;
            xi[k] = act[k] ? D.x[ip[k]] : FAR_POS;
            yi[k] = act[k] ? D.y[ip[k]] : FAR_POS;
            zi[k] = act[k] ? D.z[ip[k]] : -FAR_POS;
            hi2[k] = act[k] ? D.h2[ip[k]] : 0.0;
            ax[k] = ay[k] = az[k] = pot[k] = 0.0;
        }

        // register prefetch of the first tile
        double px[LPT], py[LPT], pz[LPT], pm[LPT], ph[LPT];
#pragma unroll
        for (int l = 0; l < LPT; l++) {
            const int slot = S.poff + W.jb + l * NT + tid;
            px[l] = D.x[slot]; py[l] = D.y[slot]; pz[l] = D.z[slot];
            pm[l] = D.m[slot]; ph[l] = D.h2[slot];
        }
        for (int jt = W.jb; jt < W.je; jt += TJ) {
#pragma unroll
            for (int l = 0; l < LPT; l++) {
                const int t = l * NT + tid;
                s_x[t] = px[l]; s_y[t] = py[l]; s_z[t] = pz[l]; s_m[t] = pm[l]; s_h[t] = ph[l];
            }
            __syncthreads();
            if (jt + TJ < W.je) {
#pragma unroll
                for (int l = 0; l < LPT; l++) {
                    const int slot = S.poff + jt + TJ + l * NT + tid;
                    px[l] = D.x[slot]; py[l] = D.y[slot]; pz[l] = D.z[slot];
                    pm[l] = D.m[slot]; ph[l] = D.h2[slot];
                }
            }
#pragma unroll 2
            for (int j = 0; j < TJ; j++) {
                const double xj = s_x[j], yj = s_y[j], zj = s_z[j], mj = s_m[j], hj = s_h[j];
#pragma unroll
                for (int k = 0; k < K; k++) {
                    const double dx = xj - xi[k], dy = yj - yi[k], dz = zj - zi[k];
                    const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
                    if (r2 >= fmax(hi2[k], hj)) {
                        const double rinv = rsqrt(r2);
                        const double mr = mj * rinv;
                        const double mr3 = mr * rinv * rinv;
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
            __syncthreads();
        }

        double *p = a.partials + (size_t)(S.slot_off + W.tile * S.nchunks + W.chunk) * 4 * ITILE;
#pragma unroll
        for (int k = 0; k < K; k++) {
            if (act[k]) {
                const int li = k * NT + tid;
                p[li] = ax[k];
                p[ITILE + li] = ay[k];
                p[2 * ITILE + li] = az[k];
                p[3 * ITILE + li] = pot[k];
            }
        }
    }
}

static const VariantInfo kF64Variants[] = {
    {0, 128, 1, 1, 128, 0, "fp64_nt128_k1_tj128", 128},
    {0, 256, 1, 1, 256, 0, "fp64_nt256_k1_tj256", 256},
    {0, 128, 2, 1, 128, 0, "fp64_nt128_k2_tj128", 256},
};
static const void *kF64Kernels[] = {
    (const void *)k_fp64<128, 1, 128>,
    (const void *)k_fp64<256, 1, 256>,
    (const void *)k_fp64<128, 2, 128>,
};
constexpr int kNF64 = sizeof(kF64Variants) / sizeof(kF64Variants[0]);

int f64_variant_count() { return kNF64; }
const VariantInfo &f64_variant_info(int v) { return kF64Variants[v]; }
const void *f64_kernel(int v) { return kF64Kernels[v]; }

cudaError_t launch_f64(int v, int grid, const ComputeArgs &a, cudaStream_t st)
{
    switch (v) {
    case 0: k_fp64<128, 1, 128><<<grid, 128, 0, st>>>(a); break;
    case 1: k_fp64<256, 1, 256><<<grid, 256, 0, st>>>(a); break;
    case 2: k_fp64<128, 2, 128><<<grid, 128, 0, st>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    ++g_launches;
    return cudaGetLastError();
}

}  // namespace sg
