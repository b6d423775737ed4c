// sg_prep.cu -- per-call preparation of the device-resident particle layout,
// the ordered merge of partial sums, the potential-energy diagnostic and the
// kick kernel of device-resident sweeps.
//
// Layout produced per call (all on the device):
//   * per-set bounding boxes -> 3 x bits Hilbert-curve keys with the set
//     index above them -> one radix sort of all particles: particles of a
//     set stay contiguous and in set order, spatially sorted inside the set
//     along a Hilbert curve (consecutive cells are face neighbours, so every
//     run of consecutive particles -- an i-tile, a j-tile -- is spatially
//     compact; a Morton order jumps across octant boundaries, and an i-tile
//     across such a jump put rows far from the tile centre, where the FP32
//     rounding of their tile-relative coordinates shifted them measurably);
//   * padded sorted SoA arrays (each set padded to a multiple of PAD_J with
//     mass-0 slots far away): FP64 copies for the FP64 kernel and the
//     near-field pairs, FP32 hi+lo position pairs for the split kernel;
//   * the row list (sorted slots of the rows to compute), i-tile centres and
//     j-tile bounding boxes used to skip the near-field test.
#include <cub/cub.cuh>
#include "sg_launch.h"

namespace sg {

std::atomic<unsigned long long> g_launches{0};

static inline unsigned grid_for(long long n, int block, int cap)
{
    long long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

// ------------------------------------------------------------- validation
// The reference asserts mass > 0 and range2 != 0 on the host
// (grav_force_direct.cu:601-602); here the check runs on the device and sets
// an error bit read back at the next synchronisation.
__global__ void k_validate(InputsDev in, int n, int *err)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const double x = in.x[p], y = in.y[p], z = in.z[p], m = in.m[p], r2 = in.r2[p];
        const bool ok = isfinite(x) && isfinite(y) && isfinite(z) && isfinite(m) && m > 0.0 &&
                        isfinite(r2) && r2 != 0.0;
        if (!ok) atomicOr(err, DEVERR_INPUT);
    }
}

cudaError_t launch_validate(const InputsDev &in, int ntot, int *err, cudaStream_t st)
{
    if (ntot <= 0) return cudaSuccess;
    k_validate<<<grid_for(ntot, 256, 4096), 256, 0, st>>>(in, ntot, err);
    ++g_launches;
    return cudaGetLastError();
}

// ------------------------------------------------------------ bounding box
__global__ void k_bbox_init(unsigned long long *bbox, int nsets)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 6 * nsets) bbox[t] = (t % 6) < 3 ? ~0ull : 0ull;
}

__global__ void k_bbox(const SetDesc *sets, InputsDev in, unsigned long long *bbox)
{
    const SetDesc S = sets[blockIdx.y];
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S.n; k += gridDim.x * blockDim.x) {
        const int p = S.off + k;
        const double v[3] = {in.x[p], in.y[p], in.z[p]};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            lo[d] = fmin(lo[d], v[d]);
            hi[d] = fmax(hi[d], v[d]);
        }
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
            hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
        }
    }
    if ((threadIdx.x & 31) == 0 && lo[0] <= hi[0]) {
        unsigned long long *b = bbox + 6 * blockIdx.y;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            atomicMin(b + d, dkey(lo[d]));
            atomicMax(b + 3 + d, dkey(hi[d]));
        }
    }
}

cudaError_t launch_bbox(const SetDesc *sets, int nsets, int max_n, const InputsDev &in,
                        unsigned long long *bbox, cudaStream_t st)
{
    k_bbox_init<<<grid_for(6 * nsets, 256, 1 << 20), 256, 0, st>>>(bbox, nsets);
    ++g_launches;
    dim3 grid(grid_for(max_n, 256, 64), nsets);
    k_bbox<<<grid, 256, 0, st>>>(sets, in, bbox);
    ++g_launches;
    return cudaGetLastError();
}

// ----------------------------------------------------------- Hilbert keys
__device__ __forceinline__ unsigned long long spread3(unsigned long long v)
{
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

// Index of cell (x0, x1, x2) (bits per axis) on the 3-D Hilbert curve, after
// J. Skilling, "Programming the Hilbert curve", AIP Conf. Proc. 707 (2004):
// the axes are transformed in place (undo the excess work of the inverse
// map, then Gray-encode) and the transposed form is interleaved into the
// index.  The top 3 L bits of the index name the level-L octree cell, as
// those of a Morton key do, so cells are contiguous key ranges.
__device__ __forceinline__ unsigned long long hilbert3(unsigned x0, unsigned x1, unsigned x2,
                                                       int bits)
{
    unsigned X[3] = {x0, x1, x2};
    const unsigned M = 1u << (bits - 1);
    for (unsigned Q = M; Q > 1; Q >>= 1) {
        const unsigned P = Q - 1;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            if (X[i] & Q) {
                X[0] ^= P;
            } else {
                const unsigned t = (X[0] ^ X[i]) & P;
                X[0] ^= t;
                X[i] ^= t;
            }
        }
    }
    X[1] ^= X[0];
    X[2] ^= X[1];
    unsigned t = 0;
    for (unsigned Q = M; Q > 1; Q >>= 1)
        if (X[2] & Q) t ^= Q - 1;
    X[0] ^= t;
    X[1] ^= t;
    X[2] ^= t;
    return (spread3(X[0]) << 2) | (spread3(X[1]) << 1) | spread3(X[2]);
}

__global__ void k_sfc_keys(const SetDesc *sets, InputsDev in, const unsigned long long *bbox,
                           int bits, unsigned long long *keys, int *vals)
{
    const int s = blockIdx.y;
    const SetDesc S = sets[s];
    const unsigned long long *b = bbox + 6 * s;
    double lo[3], scale[3];
    const double cells = (double)((1u << bits) - 1);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        lo[d] = dkey_inv(b[d]);
        const double ext = dkey_inv(b[3 + d]) - lo[d];
        scale[d] = ext > 0.0 ? cells / ext : 0.0;
    }
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S.n; k += gridDim.x * blockDim.x) {
        const int p = S.off + k;
        const double v[3] = {in.x[p], in.y[p], in.z[p]};
        unsigned q[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            double c = (v[d] - lo[d]) * scale[d];
            q[d] = (unsigned)fmin(fmax(c, 0.0), cells);
        }
        keys[p] = ((unsigned long long)s << (3 * bits)) | hilbert3(q[0], q[1], q[2], bits);
        vals[p] = p;
    }
}

cudaError_t launch_sfc_keys(const SetDesc *sets, int nsets, int max_n, const InputsDev &in,
                          const unsigned long long *bbox, int bits_per_axis,
                          unsigned long long *keys, int *vals, cudaStream_t st)
{
    dim3 grid(grid_for(max_n, 256, 1024), nsets);
    k_sfc_keys<<<grid, 256, 0, st>>>(sets, in, bbox, bits_per_axis, keys, vals);
    ++g_launches;
    return cudaGetLastError();
}

size_t sort_temp_bytes(int ntot, int end_bit)
{
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const unsigned long long *)nullptr,
                                    (unsigned long long *)nullptr, (const int *)nullptr,
                                    (int *)nullptr, ntot, 0, end_bit);
    return bytes;
}

cudaError_t launch_sort(void *temp, size_t temp_bytes, const unsigned long long *keys_in,
                        unsigned long long *keys_out, const int *vals_in, int *vals_out,
                        int ntot, int end_bit, cudaStream_t st)
{
    // CUB's onesweep radix sort: a handful of kernels per call.
    g_launches += 1 + (end_bit + 7) / 8;
    return cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, vals_in,
                                           vals_out, ntot, 0, end_bit, st);
}

// ------------------------------------------------------------------ gather
__global__ void k_gather(const SetDesc *sets, InputsDev in, const int *sorted_vals,
                         SortedF64 D, SortedF32 F)
{
    const SetDesc S = sets[blockIdx.y];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S.npad; k += gridDim.x * blockDim.x) {
        const int slot = S.poff + k;
        if (k < S.n) {
            const int p = sorted_vals[S.off + k];
            const double x = in.x[p], y = in.y[p], z = in.z[p], m = in.m[p], r2 = in.r2[p];
            D.x[slot] = x;
            D.y[slot] = y;
            D.z[slot] = z;
            D.m[slot] = m;
            D.h2[slot] = fabs(r2);
            D.orig[slot] = p;
            D.flag[slot] = r2 > 0.0 ? 1 : 0;
            // split of the FP64 positions into float hi + lo pairs
            const float xh = __double2float_rn(x), yh = __double2float_rn(y),
                        zh = __double2float_rn(z);
            F.xh[slot] = xh;
            F.xl[slot] = __double2float_rn(x - (double)xh);
            F.yh[slot] = yh;
            F.yl[slot] = __double2float_rn(y - (double)yh);
            F.zh[slot] = zh;
            F.zl[slot] = __double2float_rn(z - (double)zh);
            F.m[slot] = __double2float_rn(m);
            F.h2[slot] = __double2float_rn(fabs(r2));
        } else {
            D.x[slot] = FAR_POS;
            D.y[slot] = FAR_POS;
            D.z[slot] = FAR_POS;
            D.m[slot] = 0.0;
            D.h2[slot] = 0.0;
            D.orig[slot] = -1;
            D.flag[slot] = 0;
            F.xh[slot] = (float)FAR_POS;
            F.xl[slot] = 0.f;
            F.yh[slot] = (float)FAR_POS;
            F.yl[slot] = 0.f;
            F.zh[slot] = (float)FAR_POS;
            F.zl[slot] = 0.f;
            F.m[slot] = 0.f;
            F.h2[slot] = 0.f;
        }
    }
}

cudaError_t launch_gather(const SetDesc *sets, int nsets, int max_npad, const InputsDev &in,
                          const int *sorted_vals, SortedF64 D, SortedF32 F, cudaStream_t st)
{
    dim3 grid(grid_for(max_npad, 256, 1024), nsets);
    k_gather<<<grid, 256, 0, st>>>(sets, in, sorted_vals, D, F);
    ++g_launches;
    return cudaGetLastError();
}

// ---------------------------------------------------------------- row list
__global__ void k_rows_full(const SetDesc *sets, int *ilist)
{
    const SetDesc S = sets[blockIdx.y];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S.n; k += gridDim.x * blockDim.x)
        ilist[S.ioff + k] = S.poff + k;
}

cudaError_t launch_rows_full(const SetDesc *sets, int nsets, int max_n, int *ilist,
                             cudaStream_t st)
{
    dim3 grid(grid_for(max_n, 256, 1024), nsets);
    k_rows_full<<<grid, 256, 0, st>>>(sets, ilist);
    ++g_launches;
    return cudaGetLastError();
}

struct InRows {
    const int *orig;
    int off, lo, hi;
    __device__ __forceinline__ bool operator()(const int slot) const
    {
        const int o = orig[slot] - off;
        return o >= lo && o < hi;
    }
};

size_t select_temp_bytes(int n)
{
    size_t bytes = 0;
    cub::DeviceSelect::If(nullptr, bytes, cub::CountingInputIterator<int>(0), (int *)nullptr,
                          (int *)nullptr, n, InRows{nullptr, 0, 0, 0});
    return bytes;
}

cudaError_t launch_rows_range(const SetDesc &S, const SortedF64 D, int *ilist, int *nsel_dev,
                              void *temp, size_t temp_bytes, cudaStream_t st)
{
    g_launches += 2;
    return cub::DeviceSelect::If(temp, temp_bytes, cub::CountingInputIterator<int>(S.poff),
                                 ilist + S.ioff, nsel_dev, S.n,
                                 InRows{D.orig, S.off, S.i_lo, S.i_lo + S.ni}, st);
}

// ------------------------------------------------------------ tile metadata
__global__ void k_itile_meta(const SetDesc *sets, const int *tile_set, int itile,
                             const int *ilist, SortedF64 D, ITileMeta *meta)
{
    const int t = blockIdx.x;
    const SetDesc S = sets[tile_set[t]];
    const int lt = t - S.tile_off;
    const int r0 = lt * itile;
    const int r1 = min(S.ni, r0 + itile);
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
        const int slot = ilist[S.ioff + r];
        const double v[3] = {D.x[slot], D.y[slot], D.z[slot]};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            lo[d] = fmin(lo[d], v[d]);
            hi[d] = fmax(hi[d], v[d]);
        }
    }
    __shared__ double s_lo[3][32], s_hi[3][32];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
            hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
        }
        if ((threadIdx.x & 31) == 0) {
            s_lo[d][threadIdx.x >> 5] = lo[d];
            s_hi[d][threadIdx.x >> 5] = hi[d];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        double c[3];
        for (int d = 0; d < 3; d++) {
            double l = s_lo[d][0], h = s_hi[d][0];
            for (int w = 1; w < nw; w++) {
                l = fmin(l, s_lo[d][w]);
                h = fmax(h, s_hi[d][w]);
            }
            c[d] = l <= h ? 0.5 * (l + h) : 0.0;
        }
        ITileMeta M;
        M.chx = __double2float_rn(c[0]);
        M.chy = __double2float_rn(c[1]);
        M.chz = __double2float_rn(c[2]);
        M.clx = __double2float_rn(c[0] - (double)M.chx);
        M.cly = __double2float_rn(c[1] - (double)M.chy);
        M.clz = __double2float_rn(c[2] - (double)M.chz);
        M.pad_[0] = M.pad_[1] = 0.f;
        meta[t] = M;
    }
}

cudaError_t launch_itile_meta(const SetDesc *sets, int nsets, int ntiles_total,
                              const int *tile_set, int itile, const int *ilist,
                              const SortedF64 D, ITileMeta *meta, cudaStream_t st)
{
    (void)nsets;
    if (ntiles_total <= 0) return cudaSuccess;
    k_itile_meta<<<ntiles_total, 128, 0, st>>>(sets, tile_set, itile, ilist, D, meta);
    ++g_launches;
    return cudaGetLastError();
}

// One warp per META_J slots.
__global__ void k_jmeta(const SetDesc *sets, int nmeta_total, const int *meta_set, SortedF64 D,
                        JMeta *meta)
{
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (r >= nmeta_total) return;
    const int lane = threadIdx.x & 31;
    const SetDesc S = sets[meta_set[r]];
    const int k0 = (r - S.meta_off) * META_J;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    double h2max = 0.0;
    for (int k = k0 + lane; k < k0 + META_J; k += 32) {
        if (k < S.n) {
            const int slot = S.poff + k;
            const double v[3] = {D.x[slot], D.y[slot], D.z[slot]};
#pragma unroll
            for (int d = 0; d < 3; d++) {
                lo[d] = fmin(lo[d], v[d]);
                hi[d] = fmax(hi[d], v[d]);
            }
            h2max = fmax(h2max, D.h2[slot]);
        }
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
            hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
        }
    }
    for (int o = 16; o > 0; o >>= 1) h2max = fmax(h2max, __shfl_xor_sync(0xffffffffu, h2max, o));
    if (lane == 0) {
        JMeta M;
        if (lo[0] <= hi[0]) {
            // centre rounded to float; the half extents absorb that rounding
            // and are rounded up, so the box still holds every particle.
            const double c[3] = {0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1]), 0.5 * (lo[2] + hi[2])};
            float cf[3], ef[3];
            for (int d = 0; d < 3; d++) {
                cf[d] = __double2float_rn(c[d]);
                const double e = 0.5 * (hi[d] - lo[d]) + fabs(c[d] - (double)cf[d]);
                ef[d] = __double2float_ru(e * (1.0 + 1e-6) + 1e-30);
            }
            M.cx = cf[0]; M.cy = cf[1]; M.cz = cf[2];
            M.ex = ef[0]; M.ey = ef[1]; M.ez = ef[2];
            M.h2max = __double2float_ru(h2max);
        } else {
            M.cx = M.cy = M.cz = 0.f;
            M.ex = M.ey = M.ez = -1.f;
            M.h2max = 0.f;
        }
        M.pad_ = 0.f;
        meta[r] = M;
    }
}

cudaError_t launch_jmeta(const SetDesc *sets, int nsets, int nmeta_total, const int *meta_set,
                         const SortedF64 D, JMeta *meta, cudaStream_t st)
{
    (void)nsets;
    if (nmeta_total <= 0) return cudaSuccess;
    k_jmeta<<<grid_for((long long)nmeta_total * 32, 256, 1 << 30), 256, 0, st>>>(
        sets, nmeta_total, meta_set, D, meta);
    ++g_launches;
    return cudaGetLastError();
}

// ------------------------------------------------------------------ merge
// Block-wide sum of one double per thread in a fixed order (tree over the
// thread index); the result is valid in thread 0.
__device__ double block_sum_fixed(double w)
{
    __shared__ double s_w[1024];
    s_w[threadIdx.x] = w;
    __syncthreads();
    for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
        if (threadIdx.x < o) s_w[threadIdx.x] += s_w[threadIdx.x + o];
        __syncthreads();
    }
    return s_w[0];
}

// Ordered second pass: row sums over the j-chunks in chunk order (the result
// does not depend on which block computed which chunk), scatter to the
// caller's order, and the per-tile sum of m_i * phi_i in a fixed order.
// Split-FP32 calls also merge the rows' error scales G^2 (sum over j-tiles of
// |FP32 tile sum|^2) and append every row with G^2 > thresh2 |a|^2 to its
// set's refine list, rlist[S.ioff + k], k counted in rcount[set].
__global__ void k_merge(const SetDesc *sets, const int *tile_set, const int2 *tile_slots, int itile,
                        const int *ilist, SortedF64 D, const double *partials, OutputsDev out,
                        double *wtile, MergeRefine R)
{
    const int t = blockIdx.x;
    const int set = tile_set[t];
    const SetDesc S = sets[set];
    const int2 ts = tile_slots[t];  // first partial slot, j-chunks of this tile
    const int lt = t - S.tile_off;
    const int r0 = lt * itile;
    const int nrow = min(itile, S.ni - r0);
    double w = 0.0;
    for (int li = threadIdx.x; li < nrow; li += blockDim.x) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        float g2 = 0.f;
        for (int c = 0; c < ts.y; c++) {
            const size_t slot = (size_t)(ts.x + c);
            const double *p = partials + slot * 4 * itile;
#pragma unroll
            for (int q = 0; q < 4; q++) acc[q] += p[q * itile + li];
            if (R.gpart) g2 += R.gpart[slot * itile + li];
        }
        const int slot = ilist[S.ioff + r0 + li];
        const int o = D.orig[slot];
        out.ax[o] = acc[0];
        out.ay[o] = acc[1];
        out.az[o] = acc[2];
        out.pot[o] = acc[3];
        w += D.m[slot] * acc[3];
        if (R.gpart) {
            const double a2 = acc[0] * acc[0] + acc[1] * acc[1] + acc[2] * acc[2];
            if (R.rlist && (double)g2 > R.thresh2 * a2) {
                const int k = atomicAdd(&R.rcount[set], 1);
                R.rlist[S.ioff + k] = slot;
            }
            if (R.scale) R.scale[o] = sqrt((double)g2);
        }
    }
    const double wt = block_sum_fixed(w);
    if (threadIdx.x == 0 && wtile) wtile[t] = wt;
}

cudaError_t launch_merge(const SetDesc *sets, const int *tile_set, const int2 *tile_slots,
                         int ntiles_total, int itile, const int *ilist, const SortedF64 D,
                         const double *partials, OutputsDev out, double *wtile,
                         const MergeRefine &R, cudaStream_t st)
{
    if (ntiles_total <= 0) return cudaSuccess;
    k_merge<<<ntiles_total, 256, 0, st>>>(sets, tile_set, tile_slots, itile, ilist, D, partials,
                                          out, wtile, R);
    ++g_launches;
    return cudaGetLastError();
}

// Per-tile sum of m_i * phi_i from the outputs (caller order), in the order of
// k_merge; used after rows were replaced by the FP64 refine.
__global__ void k_wtile_out(const SetDesc *sets, const int *tile_set, int itile, const int *ilist,
                            SortedF64 D, const double *pot, double *wtile)
{
    const int t = blockIdx.x;
    const SetDesc S = sets[tile_set[t]];
    const int lt = t - S.tile_off;
    const int r0 = lt * itile;
    const int nrow = min(itile, S.ni - r0);
    double w = 0.0;
    for (int li = threadIdx.x; li < nrow; li += blockDim.x) {
        const int slot = ilist[S.ioff + r0 + li];
        w += D.m[slot] * pot[D.orig[slot]];
    }
    const double wt = block_sum_fixed(w);
    if (threadIdx.x == 0) wtile[t] = wt;
}

cudaError_t launch_wtile_out(const SetDesc *sets, const int *tile_set, int ntiles_total, int itile,
                             const int *ilist, const SortedF64 D, const double *pot, double *wtile,
                             cudaStream_t st)
{
    if (ntiles_total <= 0) return cudaSuccess;
    k_wtile_out<<<ntiles_total, 256, 0, st>>>(sets, tile_set, itile, ilist, D, pot, wtile);
    ++g_launches;
    return cudaGetLastError();
}

// W = 1/2 sum m_i phi_i per set (output.f:232-252): one block per set sums
// the set's tile sums, thread k over tiles k, k + blockDim, ... in order,
// then a fixed tree over the threads.
__global__ void k_wsum(const SetDesc *sets, int nsets, const double *wtile, double *W)
{
    const int s = blockIdx.x;
    if (s >= nsets) return;
    const SetDesc S = sets[s];
    double w = 0.0;
    for (int t = threadIdx.x; t < S.ntiles; t += blockDim.x) w += wtile[S.tile_off + t];
    const double tot = block_sum_fixed(w);
    if (threadIdx.x == 0) W[s] = 0.5 * tot;
}

cudaError_t launch_wsum(const SetDesc *sets, int nsets, const double *wtile, double *W,
                        cudaStream_t st)
{
    if (nsets <= 0) return cudaSuccess;
    k_wsum<<<nsets, 128, 0, st>>>(sets, nsets, wtile, W);
    ++g_launches;
    return cudaGetLastError();
}

// ------------------------------------------------------------------- kick
// Counter-based normal deviates: splitmix64 of (seed, call, particle, k)
// gives uniform 53-bit doubles; Box-Muller turns two of them into a pair of
// normals.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double u01(unsigned long long h)
{
    return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);  // (0, 1)
}

__global__ void k_kick(int n, double *x, double *y, double *z, double sigma,
                       unsigned long long seed, const unsigned long long *counter)
{
    const unsigned long long c = *counter;
    const unsigned long long base = splitmix64(seed ^ splitmix64(c + 0x632be59bd9b4e019ull));
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const unsigned long long h = splitmix64(base + (unsigned long long)p * 4ull);
        const double u1 = u01(h), u2 = u01(splitmix64(h + 1)), u3 = u01(splitmix64(h + 2)),
                     u4 = u01(splitmix64(h + 3));
        const double ra = sqrt(-2.0 * log(u1)), rb = sqrt(-2.0 * log(u3));
        const double ta = 6.283185307179586 * u2, tb = 6.283185307179586 * u4;
        x[p] += sigma * ra * cos(ta);
        y[p] += sigma * ra * sin(ta);
        z[p] += sigma * rb * cos(tb);
    }
}
__global__ void k_kick_advance(unsigned long long *counter) { *counter += 1; }

// ------------------------------------------- Fortran caller's range2 (grav.f:15-18)
// range2 = 4 hp^2, negated for point masses (u == 0)
__global__ void k_range2(int n, const double *hp, const double *u, double *range2)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double r = 4.0 * hp[i] * hp[i];
        range2[i] = u[i] == 0.0 ? -r : r;
    }
}

cudaError_t launch_range2(int n, const double *hp, const double *u, double *range2, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    k_range2<<<grid_for(n, 256, 4096), 256, 0, st>>>(n, hp, u, range2);
    ++g_launches;
    return cudaGetLastError();
}

cudaError_t launch_kick(int n, double *x, double *y, double *z, double sigma,
                        unsigned long long seed, unsigned long long *counter, cudaStream_t st)
{
    if (n > 0) {
        k_kick<<<grid_for(n, 256, 4096), 256, 0, st>>>(n, x, y, z, sigma, seed, counter);
        ++g_launches;
    }
    k_kick_advance<<<1, 1, 0, st>>>(counter);
    ++g_launches;
    return cudaGetLastError();
}

// --------------------------------------------------------- FP32 FMA probe
// Eight independent packed-FMA chains per thread: issue-bound on the FMA
// pipe, the ceiling the split kernel's roofline fraction is quoted against.
__global__ void k_fp32_probe(int iters, float *sink)
{
    f2 a[8];
    const float s = 1.0f + 1e-7f * threadIdx.x;
#pragma unroll
    for (int c = 0; c < 8; c++) a[c] = pk(s * (c + 1), s * (c + 2));
    const f2 mul = pk(0.999999f, 0.9999995f), add = pk(1e-7f, 2e-7f);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int c = 0; c < 8; c++) a[c] = fma2(a[c], mul, add);
    }
    float acc = 0.f;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        float lo, hi;
        upk(a[c], lo, hi);
        acc += lo + hi;
    }
    if (acc == 12345.678f) sink[blockIdx.x] = acc;
}

cudaError_t launch_fp32_probe(int iters, int blocks, float *sink, cudaStream_t st)
{
    k_fp32_probe<<<blocks, 256, 0, st>>>(iters, sink);
    ++g_launches;
    return cudaGetLastError();
}

// ------------------------------------------------------- FP64 FMA probe
// Eight independent DFMA chains per thread: the FP64 pipe's throughput.
__global__ void k_fp64_probe(int iters, float *sink)
{
    double a[8];
    const double s = 1.0 + 1e-9 * threadIdx.x;
#pragma unroll
    for (int c = 0; c < 8; c++) a[c] = s * (c + 1);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int c = 0; c < 8; c++) a[c] = fma(a[c], 0.9999999999, 1e-10);
    }
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c < 8; c++) acc += a[c];
    if (acc == 12345.678) sink[blockIdx.x] = (float)acc;
}

// ------------------------------------------- device timeout self-test
// One warp waits, through the pair kernels' bounded mbarrier poll, on a
// barrier that nothing arrives on; after `polls` polls it records
// DEVERR_TIMEOUT the way a pair kernel does and returns.
__global__ void k_wait_selftest(uint32_t polls, int *err)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncwarp();
    const bool ok = mbar_wait_bounded(&bar, 0, polls);
    if (!__all_sync(0xffffffffu, ok) && threadIdx.x == 0) atomicOr(err, DEVERR_TIMEOUT);
}

cudaError_t launch_wait_selftest(uint32_t polls, int *err, cudaStream_t st)
{
    k_wait_selftest<<<1, 32, 0, st>>>(polls, err);
    ++g_launches;
    return cudaGetLastError();
}

cudaError_t launch_fp64_probe(int iters, int blocks, float *sink, cudaStream_t st)
{
    k_fp64_probe<<<blocks, 256, 0, st>>>(iters, sink);
    ++g_launches;
    return cudaGetLastError();
}

}  // namespace sg
