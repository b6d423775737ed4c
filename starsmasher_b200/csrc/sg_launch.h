// sg_launch.h -- host-side launch interface between the context code and the
// kernels.  Every function enqueues on `st` and returns the launch status.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <atomic>
#include "sg_internal.cuh"

namespace sg {

// Kernels launched by the library; atomic because entry points on different
// contexts (or the allocation-free one) may run on several host threads.
extern std::atomic<unsigned long long> g_launches;

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
cudaError_t launch_sfc_keys(const SetDesc *sets, int nsets, int max_n, const InputsDev &in,
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
    double *partials;    // [slot][4][itile], slot = WorkItem::slot
    // split-FP32: [slot][itile] sum over the item's j-tiles of |FP32 tile sum|^2
    // (acceleration components, both packed lanes): the scale of the FP32
    // rounding error of the row, merged into the refine test (nullable)
    float *gpart;
    // when non-null the item count is read here instead of `nitems` (work
    // lists planned on the device, e.g. the FP64 refine of flagged rows)
    const int *nitems_dev;
    int *err;
    int nkernel;
    int itile;
    float band2;         // split-FP32: pairs with r^2 < band2 * max(H^2) use FP64 (>= 1)
    // split-FP32 built with -DSG_PHASES: [PHASE_COUNTERS] clock64 cycles per
    // phase summed over warps (see the Phase enum); nullptr = not counted
    unsigned long long *phases = nullptr;
};

// Phase accounting of the split-FP32 kernel (a diagnostic build: the pair
// kernel compiled with -DSG_PHASES).  Consumer and producer warps sum the
// SM cycles they spend in each phase; counts are per warp.
enum Phase {
    PH_ITEM = 0,      // consumer: queue fetch and the CTA barrier at an item start
    PH_ROWS,          // consumer: loading the item's rows, warp box
    PH_WAIT_FULL,     // consumer: waiting for a staged tile
    PH_FAR,           // consumer: far loop + tile fold
    PH_CHECKED,       // consumer: checked loop (near pairs masked) + tile fold
    PH_NEAR,          // consumer: near_eval (FP64 pairs)
    PH_END,           // consumer: combining and writing the item's partials
    PH_PROD_WAIT,     // producer: waiting for a free stage or for its copies
    PH_PROD_WORK,     // producer: issuing copies, rewriting tiles, tile boxes
    PH_N_FAR,         // count: far (warp, tile) pairs
    PH_N_CHECKED,     // count: checked (warp, tile) pairs
    PH_N_NEAR,        // count: near_eval calls
    PH_N_ITEMS,       // count: items started per consumer warp
    PHASE_COUNTERS = 16
};
bool phases_built();

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
// Refine test of the merge (split-FP32 calls): rows whose error scale G^2
// exceeds thresh2 * |a|^2 are listed for the FP64 refine.
struct MergeRefine {
    const float *gpart = nullptr;  // [slot][itile] G^2 partials; null: no test
    double thresh2 = 0.0;          // T^2
    int *rcount = nullptr;         // [nsets] rows listed per set (zeroed before the merge)
    int *rlist = nullptr;          // listed sorted slots; set s at [S.ioff, S.ioff + S.ni)
    double *scale = nullptr;       // optional: G per row in the caller's order
};
// tile_slots[t] = (first partial slot, j-chunk count) of global i-tile t.
cudaError_t launch_merge(const SetDesc *sets, const int *tile_set, const int2 *tile_slots,
                         int ntiles_total, int itile, const int *ilist, const SortedF64 D,
                         const double *partials, OutputsDev out, double *wtile,
                         const MergeRefine &R, cudaStream_t st);
cudaError_t launch_wtile_out(const SetDesc *sets, const int *tile_set, int ntiles_total, int itile,
                             const int *ilist, const SortedF64 D, const double *pot, double *wtile,
                             cudaStream_t st);

// --- FP64 refine of the listed rows (sg_refine.cu)
// Plans the refine on the device from the per-set counts: for set s the rows
// rlist[S.ioff, S.ioff + rcount[s]) in tiles of `itile` rows, every tile
// split into the same number of j-chunks (enough items to fill `target`
// persistent blocks, at least 256 sources per chunk), one partial slot per
// item.  Writes rsets (copies of sets with ni, ntiles, nchunks, slot_off of
// the refine), the items and their count.  At most max_items items are
// written; a plan that would need more sets DEVERR_INPUT (never expected:
// the host sizes max_items for every row flagged).
// Row-chunk items (sets with at most 32 listed rows: one warp per row and
// source chunk) a refine plan may hold.
constexpr int REFINE_LIGHT_CAP = 65536;
cudaError_t launch_refine_plan(const SetDesc *sets, int nsets, const int *rcount, int itile,
                               int tj, int min_j, int target, int max_items, SetDesc *rsets,
                               WorkItem *items, int *nitems, WorkItem *litems, int *nlight,
                               int *err, cudaStream_t st);
cudaError_t launch_refine_light(const SetDesc *rsets, const WorkItem *items, const int *nitems,
                                const int *rlist, const SortedF64 &D, int nkernel, double *lpart,
                                int sm_count, cudaStream_t st);
// Scatter the refined rows: chunk sums in chunk order, written over the
// split-FP32 results in the caller's order.  Launched over the main plan's
// tiles (grid ntiles_main); tile t covers refine-list entries
// [lt * itile_main, (lt + 1) * itile_main) of its set.
cudaError_t launch_refine_merge(const SetDesc *sets, const SetDesc *rsets, const int *tile_set,
                                int ntiles_main, int itile_main, int itile_ref, const int *rcount,
                                const int *rlist, const SortedF64 D, const double *rpart,
                                const double *lpart, OutputsDev out, cudaStream_t st);
cudaError_t launch_wsum(const SetDesc *sets, int nsets, const double *wtile, double *W,
                        cudaStream_t st);
cudaError_t launch_range2(int n, const double *hp, const double *u, double *range2, cudaStream_t st);
cudaError_t launch_kick(int n, double *x, double *y, double *z, double sigma,
                        unsigned long long seed, unsigned long long *counter, cudaStream_t st);
cudaError_t launch_fp32_probe(int iters, int blocks, float *sink, cudaStream_t st);
cudaError_t launch_fp64_probe(int iters, int blocks, float *sink, cudaStream_t st);
cudaError_t launch_wait_selftest(uint32_t polls, int *err, cudaStream_t st);

// --- Barnes-Hut octree (sg_tree.cu)
constexpr int TREE_LEAF = 16;    // a node with more particles splits
constexpr int TREE_LEVELS = 21;  // key bits per axis (one octree level per 3-bit digit)
// device level table: [L] first node of level L (L = 0..TREE_LEVELS + 1), then a
// node-capacity overflow flag
constexpr int TREE_LV_OVERFLOW = TREE_LEVELS + 2;
constexpr int TREE_LV_SIZE = TREE_LEVELS + 3;
constexpr int TREE_STACK = 8192; // traversal stack entries per warp
constexpr int TREE_GROUP = 32;   // a walking group: a maximal node with <= 32 particles
constexpr int TREE_BUDGET = 8192;  // particles within the largest H of a group's box (each
                                   // tested pair by pair) before the group is handed to the
                                   // direct FP64 sum; a typical group has ~500-800
constexpr int TREE_HEAVY_CHUNKS = 1024;  // most source chunks of a heavy group's direct sum
// Heavy groups a captured (device-counted) tree call can hand to the direct
// sum; more set DEVERR_TREE_CAP.  Partial sums: (4096 + cap) chunks.
constexpr int TREE_HEAVY_CAP = 4096;
// Source chunks per heavy group: about 4096 blocks in all, at least 2048 sources
// each, 1..TREE_HEAVY_CHUNKS (n: the largest set's particles).
__host__ __device__ inline int tree_heavy_chunks(int nheavy, int n)
{
    int c = (4096 + nheavy - 1) / (nheavy > 0 ? nheavy : 1);
    if (c > n / 2048) c = n / 2048;
    return c < 1 ? 1 : (c > TREE_HEAVY_CHUNKS ? TREE_HEAVY_CHUNKS : c);
}

struct TreeNode {
    int start, end;     // sorted-slot range of its particles
    int child, nchild;  // first child (children are contiguous), count; 0: leaf
};
struct NodeGeom {      // bounding box and opening data (48 bytes)
    double cx, cy, cz; // box centre
    float hx, hy, hz;  // half sizes, rounded up
    float op2;         // (l / theta)^2, l = edge length
    float h2max;       // largest H^2 of its particles
    float pad_;
};
struct NodeMP {        // multipoles (64 bytes)
    double mx, my, mz; // centre of mass
    double m;          // mass
    float q[6];        // traceless quadrupole 3 S - tr(S) I about the centre of
                       // mass (S the second moment): xx yy zz xy xz yz
    float pad_[2];
};
struct TreeBuildArgs {
    int n;                           // particles (all sets)
    int levels;                      // key digits per set: bits per axis (<= TREE_LEVELS)
    int nroots;                      // sets: level 0 holds one root per set
    const SetDesc *sets;             // root s spans [sets[s].poff, sets[s].poff + sets[s].n)
    const unsigned long long *keys;  // Hilbert keys by sorted slot (set index in the top bits)
    TreeNode *nodes;
    int cap;                         // node capacity
    int *cnt, *off;                  // per-level scratch (n + 1 entries)
    unsigned char *gflag;            // per node: a walking group (maximal with <= TREE_GROUP)
    int *lv;                         // device level table (TREE_LV_SIZE ints)
    void *scan_temp;
    size_t scan_temp_bytes;
};
struct TreeWalkArgs {
    const TreeNode *nodes;
    const NodeGeom *geom;
    const NodeMP *mp;
    SortedF64 D;
    int n, ngroups, nkernel;   // n: result stride (sorted slots, pads included)
    const int *ngroups_dev;    // when non-null the group count is read here
    int nroots;                // roots are nodes [0, nroots), one per set
    const int2 *groups;  // [ngroups] sorted-slot ranges (start, end), end - start <= 32
    int *head;       // group counter (zeroed before the launch)
    int *heavy;      // [ngroups] groups handed to the direct sum ...
    int *nheavy;     // ... and their count (zeroed before the launch)
    int *stack;      // TREE_STACK entries per walking warp
    int stack_cap;
    double *out;     // [4][n] in sorted order
    int *err;
};
size_t tree_scan_temp_bytes(int n);
// Slot-indexed keys of every set's particles (pads are in no node).
cudaError_t tree_slot_keys(const SetDesc *sets, int nsets, int max_n,
                           const unsigned long long *keys_sorted, unsigned long long *keys_slot,
                           cudaStream_t st);
// Octree build: issues levels [level_begin, level_end) without a host wait
// (level 0 also sets up the root); t.lv receives the level table (nodes of
// level l are [lv[l], lv[l + 1])) and a flag set when `cap` nodes do not
// suffice (the caller regrows the node array and builds again).
cudaError_t tree_build_levels(const TreeBuildArgs &t, int level_begin, int level_end,
                              cudaStream_t st);
// Counts that the host either knows (eager calls: read back) or leaves on the
// device (calls inside a graph capture): `dev` non-null means "read it there",
// `host` then bounds it (grids are sized for the bound, kernels loop).
struct DevCount {
    int host;
    const int *dev;
    __device__ int get() const { return dev ? *dev : host; }
};
// Lists the walking groups (order not significant); *ngroups via `count`.
cudaError_t tree_groups(DevCount nn, const TreeNode *nodes, const unsigned char *gflag,
                        int2 *glist, int *count, cudaStream_t st);
// Groups sorted by descending largest H^2 of their particles (walking order).
size_t tree_order_temp_bytes(int ng);
cudaError_t tree_order_groups(DevCount ng, const int2 *glist, int2 *ordered, const double *h2,
                              unsigned *keys_in, unsigned *keys_out, void *temp, size_t temp_bytes,
                              cudaStream_t st);
// Node properties; acc_buf: tree_acc_bytes(nn) of scratch.  Levels
// [0, depth) are combined bottom-up; their node ranges are read from the
// device level table lv (level_start, when given, sizes the grids exactly).
size_t tree_acc_bytes(int nn);
cudaError_t tree_props(DevCount nn, const TreeNode *nodes, const SortedF64 &D, double theta,
                       const int *lv, const int *level_start, int depth, int level_bound,
                       void *acc_buf, NodeGeom *geom, NodeMP *mp, cudaStream_t st);
int tree_walk_warps(int sm_count);
cudaError_t tree_walk(const TreeWalkArgs &a, int sm_count, cudaStream_t st);
cudaError_t tree_scatter(int nslots, int i_lo, int ni, const double *res, const int *orig,
                         const OutputsDev &out, cudaStream_t st);
// W of every set (one block per set, fixed order); res stride nslots.
cudaError_t tree_wsum(const SetDesc *sets, int nsets, int nslots, const double *res,
                      const double *m, double *W, cudaStream_t st);
// Direct FP64 sums over the group's own set for the groups the walk handed
// over (*nheavy on the device, at most `cap`; more set DEVERR_TREE_CAP).
// max_n: the largest set; nheavy_host > 0 sizes the grid exactly.
cudaError_t tree_heavy(int nheavy_host, const int *nheavy, int cap, const int *heavy,
                       const int2 *groups, const TreeNode *nodes, int nroots, const SortedF64 &D,
                       int nslots, int max_n, int nkernel, double *partials, double *out, int *err,
                       cudaStream_t st);
// Partial-sum doubles tree_heavy needs for up to `cap` heavy groups.
size_t tree_heavy_partials(int cap, int max_n);
// Raises DEVERR_TREE_CAP when the build ran out of nodes (lv overflow flag).
cudaError_t tree_check_build(const int *lv, int *err, cudaStream_t st);

}  // namespace sg
