// sg_launch.h -- host-side launch interface between the context code and the
// kernels.  Every function enqueues on `st` and returns the launch status.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include "sg_internal.cuh"

namespace sg {

extern unsigned long long g_launches;  // kernels launched by the library

// Input arrays in the caller's (original) order, device pointers.
struct InputsDev {
    const double *x, *y, *z, *m, *r2;
};
// Outputs in the caller's order, device pointers (rows only are written).
struct OutputsDev {
    double *ax, *ay, *az, *pot;
};

// --- preparation (sg_prep.cu)
cudaError_t launch_validate(const InputsDev &in, int ntot, int *err, cudaStream_t st);
cudaError_t launch_bbox(const SetDesc *sets, int nsets, int max_n, const InputsDev &in,
                        unsigned long long *bbox /* 6 per set */, cudaStream_t st);
cudaError_t launch_morton(const SetDesc *sets, int nsets, int max_n, const InputsDev &in,
                          const unsigned long long *bbox, int bits_per_axis,
                          unsigned long long *keys, int *vals, cudaStream_t st);
size_t sort_temp_bytes(int ntot, int end_bit);
cudaError_t launch_sort(void *temp, size_t temp_bytes, const unsigned long long *keys_in,
                        unsigned long long *keys_out, const int *vals_in, int *vals_out,
                        int ntot, int end_bit, cudaStream_t st);
cudaError_t launch_gather(const SetDesc *sets, int nsets, int max_npad, const InputsDev &in,
                          const int *sorted_vals, SortedF64 D, SortedF32 F, cudaStream_t st);
// Row list.  full_rows: every set computes all its particles.  Otherwise one
// set with rows [i_lo, i_lo + ni) selected in sorted order.
cudaError_t launch_rows_full(const SetDesc *sets, int nsets, int max_n, int *ilist,
                             cudaStream_t st);
size_t select_temp_bytes(int n);
cudaError_t launch_rows_range(const SetDesc &set_host, const SortedF64 D, int *ilist,
                              int *nsel_dev, void *temp, size_t temp_bytes, cudaStream_t st);
cudaError_t launch_itile_meta(const SetDesc *sets, int nsets, int ntiles_total,
                              const int *tile_set, int itile, const int *ilist,
                              const SortedF64 D, ITileMeta *meta, cudaStream_t st);
cudaError_t launch_jmeta(const SetDesc *sets, int nsets, int nmeta_total, const int *meta_set,
                         const SortedF64 D, JMeta *meta, cudaStream_t st);

// --- compute kernels (sg_f64.cu, sg_f32.cu)
struct ComputeArgs {
    const SetDesc *sets;
    const WorkItem *items;
    int nitems;
    int *head;           // queue head, zeroed before the launch
    SortedF64 D;
    SortedF32 F;
    const int *ilist;
    const ITileMeta *imeta;
    const JMeta *jmeta;
    double *partials;    // [slot][4][itile]
    int *err;
    int nkernel;
    int itile;
    float band2;         // split-FP32: pairs with r^2 < band2 * max(H^2) use FP64 (>= 1)
};

struct VariantInfo {
    int precision;  // 0 fp64, 1 f32 split
    int nt;         // threads per block
    int k;          // rows per thread
    int q;          // threads per row
    int tj;         // j-tile
    int newton;     // one Newton step on rsqrt (f32 only)
    const char *name;
    int rows;       // rows per i-tile
    int itile() const { return rows; }
};
int variant_count(int precision);
const VariantInfo &variant_info(int precision, int v);
// Resident blocks per SM of variant v (queried once per process).
int variant_occupancy(int precision, int v);
cudaError_t launch_compute(int precision, int v, int grid, const ComputeArgs &a, cudaStream_t st);

// --- merge and diagnostics (sg_prep.cu)
cudaError_t launch_merge(const SetDesc *sets, const int *tile_set, int ntiles_total, int itile,
                         const int *ilist, const SortedF64 D, const double *partials,
                         OutputsDev out, double *wtile, cudaStream_t st);
cudaError_t launch_wsum(const SetDesc *sets, int nsets, const double *wtile, double *W,
                        cudaStream_t st);
cudaError_t launch_range2(int n, const double *hp, const double *u, double *range2, cudaStream_t st);
cudaError_t launch_kick(int n, double *x, double *y, double *z, double sigma,
                        unsigned long long seed, unsigned long long *counter, cudaStream_t st);
cudaError_t launch_fp32_probe(int iters, int blocks, float *sink, cudaStream_t st);
cudaError_t launch_fp64_probe(int iters, int blocks, float *sink, cudaStream_t st);
cudaError_t launch_wait_selftest(uint32_t polls, int *err, cudaStream_t st);

}  // namespace sg
