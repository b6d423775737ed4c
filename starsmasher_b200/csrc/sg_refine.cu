// sg_refine.cu -- FP64 recomputation of the rows whose split-FP32 sums may
// miss the 1e-6 accuracy target.
//
// The split-FP32 kernel accumulates, per row, G^2 = sum over its j-tiles of
// |FP32 tile sum|^2.  The FP32 rounding of the tile sums (the dominant error
// term: the sub-block sums add into a 256-source tile sum in FP32) and of the
// terms behaves like a random walk of size ~1e-7 G, so a row whose
// acceleration cancels (|a| a few % of its G) can reach a relative error of
// several 1e-6 even though its absolute error is ordinary.  The kernel also
// marks (G = infinity) the rows lying more than 8 H from their i-tile centre,
// whose FP32 tile-relative coordinate is rounded by enough to shift the row
// measurably.  k_merge lists the rows with G > T |a| per set; this file
// plans, on the device, an FP64 pass
// over exactly those rows (k_fp64 over a device-written work list, so the
// call needs no host round trip and stays graph-capturable) and scatters its
// results over the FP32 ones.
//
// Sets with few listed rows (at most REFINE_LIGHT_ROWS) take another route:
// a tile of 128 rows would hold a handful of them, and each row would walk its
// sources one after another, the near pairs (IEEE division and square root)
// setting the time.  There one warp takes one (row, source chunk) item, its
// lanes striding over the chunk's sources (k_refine_light).
//
// Determinism: the list order within a set depends on the merge's atomics,
// but a row's FP64 sum depends only on its own pairs and on the chunk bounds,
// which depend on the per-set counts alone; chunk sums merge in chunk order.
#include "sg_launch.h"

namespace sg {

constexpr int PLAN_NT = 1024;
constexpr int REFINE_LIGHT_ROWS = 32;     // a set with at most this many listed rows: row-chunk items
constexpr int REFINE_LIGHT_MIN_J = 512;   // sources per row-chunk item, at least (16 per lane)
constexpr int REFINE_LIGHT_MAX_CH = 256;  // source chunks per light row, at most

// Exclusive block scan of one long long per thread (Hillis-Steele in shared
// memory); returns the thread's prefix and writes the total to *total.
__device__ long long block_exclusive_scan(long long v, long long *total)
{
    __shared__ long long s[PLAN_NT];
    const int t = threadIdx.x;
    s[t] = v;
    __syncthreads();
    for (int o = 1; o < blockDim.x; o <<= 1) {
        const long long add = t >= o ? s[t - o] : 0;
        __syncthreads();
        s[t] += add;
        __syncthreads();
    }
    const long long incl = s[t];
    *total = s[blockDim.x - 1];
    __syncthreads();
    return incl - v;
}

// Sources per refine chunk: at least min_j (the host's choice: 256 sources
// with 128-source tiles, 64 with 64-source tiles for small sets), so a few
// listed rows still spread over many blocks (a listed row can have most of
// its set within its softening length, e.g. a point-mass core, and pay the
// near-pair path, one pair after another, for most sources).
__device__ __forceinline__ int refine_chunks(const SetDesc &S, int tj, int min_j, int nch_global)
{
    const int jtiles = (S.n + tj - 1) / tj;
    const int by_len = max(1, (int)(((long long)jtiles * tj) / min_j));
    return max(1, min(nch_global, min(by_len, max(1, jtiles))));
}

__global__ void __launch_bounds__(PLAN_NT) k_refine_plan(const SetDesc *sets, int nsets,
                                                          const int *rcount, int itile, int tj,
                                                          int min_j, int target, int max_items,
                                                          SetDesc *rsets, WorkItem *items,
                                                          int *nitems, WorkItem *litems,
                                                          int *nlight, int *err)
{
    const int t = threadIdx.x;
    const int per = (nsets + blockDim.x - 1) / blockDim.x;
    const int s0 = min(nsets, t * per), s1 = min(nsets, s0 + per);
    auto light = [&](int r) { return r > 0 && r <= REFINE_LIGHT_ROWS; };
    // pass 1: refine tiles and light rows of this thread's sets
    long long tiles = 0, lrows = 0;
    for (int s = s0; s < s1; s++) {
        const int r = min(rcount[s], sets[s].ni);
        if (light(r)) lrows += r;
        else tiles += (r + itile - 1) / itile;
    }
    long long total_tiles = 0, total_lrows = 0;
    block_exclusive_scan(tiles, &total_tiles);
    block_exclusive_scan(lrows, &total_lrows);
    const int nch_global = total_tiles > 0 ? (int)max(1ll, (long long)target / total_tiles) : 1;
    const int nchl_global =
        (int)min((long long)REFINE_LIGHT_MAX_CH, max(1ll, REFINE_LIGHT_CAP / max(1ll, total_lrows)));
    auto light_chunks = [&](const SetDesc &S) {
        return max(1, min(nchl_global, S.n / REFINE_LIGHT_MIN_J));
    };
    // pass 2: items of this thread's sets
    long long cnt = 0, lcnt = 0;
    for (int s = s0; s < s1; s++) {
        const int r = min(rcount[s], sets[s].ni);
        if (light(r)) lcnt += (long long)r * light_chunks(sets[s]);
        else cnt += (long long)((r + itile - 1) / itile) * refine_chunks(sets[s], tj, min_j, nch_global);
    }
    long long total_items = 0, total_light = 0;
    long long base = block_exclusive_scan(cnt, &total_items);
    long long lbase = block_exclusive_scan(lcnt, &total_light);
    if (total_items > max_items || total_light > REFINE_LIGHT_CAP) {
        if (t == 0) {
            atomicOr(err, DEVERR_INPUT);
            *nitems = 0;
            *nlight = 0;
        }
        return;
    }
    // pass 3: the refine descriptors of this thread's sets (slot_off = the
    // set's first tile item, light_off its first row-chunk item)
    for (int s = s0; s < s1; s++) {
        SetDesc S = sets[s];
        const int r = min(rcount[s], S.ni);
        const bool lt = light(r);
        const int nt = lt ? 0 : (r + itile - 1) / itile;
        const int nch = refine_chunks(S, tj, min_j, nch_global);
        S.ni = r;
        S.ntiles = nt;
        S.nchunks = nch;
        S.slot_off = (int)base;
        S.light_off = (int)lbase;
        S.light_nch = lt ? light_chunks(S) : 0;
        rsets[s] = S;
        base += (long long)nt * nch;
        lbase += lt ? (long long)r * S.light_nch : 0;
    }
    __syncthreads();  // rsets visible to the whole block
    // pass 4: the items, spread over all threads (one set can own them all):
    // item k belongs to the last set whose slot_off <= k (a set without
    // items has the slot_off of the next set that has some, so the last
    // such set is never empty)
    for (long long k = t; k < total_items; k += blockDim.x) {
        int lo = 0, hi = nsets - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (rsets[mid].slot_off <= k) lo = mid; else hi = mid - 1;
        }
        const SetDesc S = rsets[lo];
        const int local = (int)(k - S.slot_off);
        const int it = local / S.nchunks, c = local - it * S.nchunks;
        const int jtiles = (S.n + tj - 1) / tj;
        WorkItem w;
        w.set = lo;
        w.tile = it;
        w.chunk = c;
        w.slot = (int)k;  // = S.slot_off + it * S.nchunks + c
        w.jb = (int)((long long)jtiles * c / S.nchunks) * tj;
        w.je = (int)((long long)jtiles * (c + 1) / S.nchunks) * tj;
        w.pad_[0] = w.pad_[1] = 0;
        items[k] = w;
    }
    // pass 5: the row-chunk items (the same search on light_off)
    for (long long k = t; k < total_light; k += blockDim.x) {
        int lo = 0, hi = nsets - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (rsets[mid].light_off <= k) lo = mid; else hi = mid - 1;
        }
        const SetDesc S = rsets[lo];
        const int local = (int)(k - S.light_off);
        const int row = local / S.light_nch, c = local - row * S.light_nch;
        WorkItem w;
        w.set = lo;
        w.tile = row;  // the row's index in the set's listed rows
        w.chunk = c;
        w.slot = (int)k;
        w.jb = (int)((long long)S.n * c / S.light_nch);
        w.je = (int)((long long)S.n * (c + 1) / S.light_nch);
        w.pad_[0] = w.pad_[1] = 0;
        litems[k] = w;
    }
    if (t == 0) {
        *nitems = (int)total_items;
        *nlight = (int)total_light;
    }
}

// One warp per (listed row, source chunk) item of a light set: lanes stride
// over the chunk's sources with the CPU path's pair formulas, then a fixed
// butterfly sums the lanes; lpart[item][4] receives the chunk's sums.
__global__ void __launch_bounds__(256) k_refine_light(const SetDesc *rsets, const WorkItem *items,
                                                     const int *nitems, const int *rlist,
                                                     SortedF64 D, int nkernel, double *lpart)
{
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int n_it = *nitems;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n_it; k += nw) {
        const WorkItem w = items[k];
        const SetDesc S = rsets[w.set];
        const int i = rlist[S.ioff + w.tile];
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int j = S.poff + w.jb + lane; j < S.poff + w.je; j += 32) {
            const PairOut o = pair_f64_slots(D, nkernel, i, j);
            acc[0] += o.ax;
            acc[1] += o.ay;
            acc[2] += o.az;
            acc[3] += o.pot;
        }
#pragma unroll
        for (int q = 0; q < 4; q++)
            for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < 4; q++) lpart[(size_t)k * 4 + q] = acc[q];
        }
    }
}

cudaError_t launch_refine_light(const SetDesc *rsets, const WorkItem *items, const int *nitems,
                                const int *rlist, const SortedF64 &D, int nkernel, double *lpart,
                                int sm_count, cudaStream_t st)
{
    k_refine_light<<<sm_count * 8, 256, 0, st>>>(rsets, items, nitems, rlist, D, nkernel, lpart);
    ++g_launches;
    return cudaGetLastError();
}

cudaError_t launch_refine_plan(const SetDesc *sets, int nsets, const int *rcount, int itile,
                               int tj, int min_j, int target, int max_items, SetDesc *rsets,
                               WorkItem *items, int *nitems, WorkItem *litems, int *nlight,
                               int *err, cudaStream_t st)
{
    k_refine_plan<<<1, PLAN_NT, 0, st>>>(sets, nsets, rcount, itile, tj, min_j, target, max_items,
                                         rsets, items, nitems, litems, nlight, err);
    ++g_launches;
    return cudaGetLastError();
}

// One warp per refined row: lane l sums chunks l, l + 32, ... in order, then
// a fixed shuffle tree combines the lanes (deterministic).
__global__ void k_refine_merge(const SetDesc *sets, const SetDesc *rsets, const int *tile_set,
                               int itile_main, int itile_ref, const int *rcount, const int *rlist,
                               SortedF64 D, const double *rpart, const double *lpart,
                               OutputsDev out)
{
    const int t = blockIdx.x;
    const int set = tile_set[t];
    const SetDesc S = sets[set];
    const int r = min(rcount[set], S.ni);
    const int lt = t - S.tile_off;
    const int l0 = lt * itile_main, l1 = min(r, l0 + itile_main);
    if (l0 >= l1) return;
    const SetDesc RS = rsets[set];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int li = l0 + warp; li < l1; li += nw) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        if (RS.light_nch > 0) {  // row-chunk items
            for (int c = lane; c < RS.light_nch; c += 32) {
                const double *p = lpart + (size_t)(RS.light_off + li * RS.light_nch + c) * 4;
#pragma unroll
                for (int q = 0; q < 4; q++) acc[q] += p[q];
            }
        } else {
            const int rt = li / itile_ref, ri = li - rt * itile_ref;
            for (int c = lane; c < RS.nchunks; c += 32) {
                const double *p = rpart + (size_t)(RS.slot_off + rt * RS.nchunks + c) * 4 * itile_ref;
#pragma unroll
                for (int q = 0; q < 4; q++) acc[q] += p[q * itile_ref + ri];
            }
        }
#pragma unroll
        for (int q = 0; q < 4; q++)
            for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
        if (lane == 0) {
            const int o = D.orig[rlist[S.ioff + li]];
            out.ax[o] = acc[0];
            out.ay[o] = acc[1];
            out.az[o] = acc[2];
            out.pot[o] = acc[3];
        }
    }
}

cudaError_t launch_refine_merge(const SetDesc *sets, const SetDesc *rsets, const int *tile_set,
                                int ntiles_main, int itile_main, int itile_ref, const int *rcount,
                                const int *rlist, const SortedF64 D, const double *rpart,
                                const double *lpart, OutputsDev out, cudaStream_t st)
{
    if (ntiles_main <= 0) return cudaSuccess;
    k_refine_merge<<<ntiles_main, 128, 0, st>>>(sets, rsets, tile_set, itile_main, itile_ref,
                                                rcount, rlist, D, rpart, lpart, out);
    ++g_launches;
    return cudaGetLastError();
}

}  // namespace sg
