// sg_api.cu -- host runtime of the B200 gravity library: contexts, device
// buffers, work plans, the per-call pipeline, the legacy Fortran ABI, the
// batch and capture entry points and the autotuner.
//
// Reference host code replaced (parallel_bleeding_edge/src/SPHgrav_lib2/):
//   grav_force_direct.cu:504-646  SPHgrav_direct / SPHgrav:: marshalling.  The
//     reference re-allocates its buffers and converts positions to float on
//     the host every call; here buffers grow once and stay on the device, the
//     conversion, sort and tiling run as kernels, and host<->device copies
//     are one contiguous transfer each way.
//   grav_force_direct.cu:648-677  the C-ABI (same symbols below).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>
#include "sg_launch.h"
#include "../../include/sphgrav_b200.h"

namespace sg {
int f64_variant_count();
const VariantInfo &f64_variant_info(int v);
const void *f64_kernel(int v);
cudaError_t launch_f64(int v, int grid, const ComputeArgs &a, cudaStream_t st);
int f32_variant_count();
const VariantInfo &f32_variant_info(int v);
const void *f32_kernel(int v);
int f32_smem_bytes(int v);
cudaError_t f32_prepare(int v);
cudaError_t launch_f32(int v, int grid, const ComputeArgs &a, cudaStream_t st);

int variant_count(int precision) { return precision == 0 ? f64_variant_count() : f32_variant_count(); }
const VariantInfo &variant_info(int precision, int v)
{
    return precision == 0 ? f64_variant_info(v) : f32_variant_info(v);
}
int variant_occupancy(int precision, int v)
{
    // contexts on different host threads may ask at once
    static std::mutex mu;
    static std::map<std::pair<int, int>, int> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_pair(precision, v);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int nb = 0;
    const void *k = precision == 0 ? f64_kernel(v) : f32_kernel(v);
    size_t dyn = 0;
    if (precision == 1) {
        f32_prepare(v);
        dyn = (size_t)f32_smem_bytes(v);
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, variant_info(precision, v).nt, dyn) !=
        cudaSuccess)
        nb = 1;
    if (nb < 1) nb = 1;
    cache[key] = nb;
    return nb;
}
cudaError_t launch_compute(int precision, int v, int grid, const ComputeArgs &a, cudaStream_t st)
{
    return precision == 0 ? launch_f64(v, grid, a, st) : launch_f32(v, grid, a, st);
}
}  // namespace sg

using namespace sg;

// ------------------------------------------------------------------ errors
static thread_local std::string g_errmsg;

static int set_err(int status, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_errmsg = buf;
    return status;
}

#define CUDA_TRY(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            return set_err(e_ == cudaErrorMemoryAllocation ? SPHGRAV_ERR_OUT_OF_MEMORY        \
                                                           : SPHGRAV_ERR_CUDA,                \
                           "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,         \
                           __LINE__);                                                         \
        }                                                                                     \
    } while (0)

#define TRY(call)                 \
    do {                          \
        int s_ = (call);          \
        if (s_ != SPHGRAV_OK) return s_; \
    } while (0)

// ----------------------------------------------------------- device buffers
template <class T>
struct DBuf {
    T *p = nullptr;
    size_t cap = 0;
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

struct PinnedBuf {
    void *p = nullptr;
    size_t cap = 0;
    void release()
    {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
};

struct Plan {
    bool valid = false;
    // key
    std::vector<int> offsets;
    bool full_rows = true;
    int i_lo = 0, ni = 0, precision = -1, variant = -1;
    bool tree = false;  // Barnes-Hut call: the octree's levels are the full curve key
    // derived
    int nsets = 0, ntot = 0, npad_tot = 0, rows_tot = 0, ntiles = 0, nmeta = 0, nitems = 0;
    int nslots = 0, itile = 0, tj = 0, max_n = 0, max_npad = 0, bits = 21, end_bit = 63;
    int grid = 1, nchunks_max = 1;
    std::vector<SetDesc> sets;
    std::vector<int> tile_set, meta_set;
    std::vector<int2> tile_slots;  // per i-tile: first partial slot, j-chunk count
    std::vector<WorkItem> items;
    // set of global i-tile t (binary search over the sets' tile offsets)
    int tile_set_of(int t) const
    {
        int lo = 0, hi = nsets - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (sets[mid].tile_off <= t) lo = mid; else hi = mid - 1;
        }
        return lo;
    }
};

// A captured graph bakes in the context's work plan and buffer addresses.
// The context counts every change of either (`epoch`); a graph replays only
// while the count is the one it was captured at and the context is alive.
struct sphgrav_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t stream = nullptr;
    int device = 0;
    sphgrav_ctx *ctx = nullptr;  // null once the context is destroyed
    unsigned long long epoch = 0;
};

// Default refine threshold T of split-FP32 calls: rows whose error scale G
// (the root sum of squares of their FP32 tile sums) exceeds T |a| are
// recomputed in FP64.
static const double kRefineDefault = 1.0;

struct sphgrav_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    bool capturing = false;
    unsigned long long epoch = 1;       // bumped by every plan rebuild and buffer reallocation
    std::set<sphgrav_graph *> graphs;   // live graphs captured from this context

    DBuf<double> in;    // 5 * cap: x y z m range2 (caller order)
    DBuf<double> out;   // 4 * cap: ax ay az pot (caller order)
    size_t io_cap = 0;
    DBuf<unsigned long long> keys_in, keys_out, bbox;
    DBuf<int> vals_in, vals_out, ilist, nsel, tile_set, meta_set, head, err;
    DBuf<char> sort_temp, sel_temp;
    DBuf<double> d64;   // 5 * pcap: x y z m h2 (sorted, padded)
    DBuf<int> orig;
    DBuf<unsigned char> flag;
    DBuf<float> f32;    // 8 * pcap
    size_t pcap = 0;
    DBuf<SetDesc> sets;
    DBuf<int2> tile_slots;
    DBuf<ITileMeta> imeta;
    DBuf<JMeta> jmeta;
    DBuf<WorkItem> items;
    DBuf<double> partials, wtile, wdev;
    DBuf<unsigned long long> kick_counter;
    DBuf<double> range2;  // sphgrav_gravforce_device: range2 built on the device

    // FP64 refine of split-FP32 rows whose error scale G exceeds refine_T |a|
    double refine_T = kRefineDefault;  // 0: off
    bool keep_scale = false;           // keep G per row (sphgrav_error_scale)
    int scale_n = 0;                   // rows of the kept G (0: none)
    int refine_nsets = 0;              // sets of the last split-FP32 call (rcount entries)
    DBuf<float> gpart;                 // [slot][itile] G^2 partials
    DBuf<int> rcount, rlist, rnitems, rhead, rnlight;
    DBuf<SetDesc> rsets;
    DBuf<WorkItem> ritems, rlitems;  // tile items; row-chunk items of sets with few rows
    DBuf<double> rpart, scale, rlpart;  // rlpart: row-chunk partials [item][4]

    // Barnes-Hut mode (SPHGRAV_TREE)
    double theta = 0.3;   // opening angle (gpu_init_dev_ passes it; main.f:269)
    int tree_groups_last = 0, tree_heavy_last = 0;  // walking groups of the last tree call,
                                                    // and those handed to the direct sum
    DBuf<TreeNode> tnodes;
    DBuf<NodeGeom> tgeom;
    DBuf<NodeMP> tmp;
    DBuf<int> tcnt, toff, tstack, tgcount, theavy, tlv;
    DBuf<double> theavy_part, tacc;
    DBuf<unsigned char> tgflag;
    DBuf<int2> tglist, tgorder;
    DBuf<unsigned long long> tkeys;  // Hilbert keys by sorted slot (batches)
    DBuf<unsigned char> tscan;
    DBuf<double> tres, twsum;
    DBuf<float> probe_sink;

    PinnedBuf h_in, h_out, h_err;
    Plan plan;

    // legacy call in flight
    bool pending = false;
    int pend_n = 0, pend_i0 = 0, pend_ni = 0;
    int pend_nsets = 0;
    double *pend_user[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t ev_start = nullptr, ev_done = nullptr;

    int forced_variant[2] = {-1, -1};
    std::map<int, std::string> tuned[2];  // N bucket -> variant name

    // kernel timing (sphgrav_profile_*)
    double fp64_band = 1.0;  // split-FP32: FP64 for r < fp64_band * max(H)
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;
    size_t prof_used = 0;
    // phase cycles of the split-FP32 kernel (diagnostic build only)
    DBuf<unsigned long long> phases;
};

template <class T>
static int ensure(sphgrav_ctx *c, DBuf<T> &b, size_t n, const char *what)
{
    if (n <= b.cap && b.p) return SPHGRAV_OK;
    if (c->capturing)
        return set_err(SPHGRAV_ERR_PROTOCOL,
                       "buffer '%s' must grow to %zu elements during a graph capture; call the "
                       "entry point once with the same sizes before capturing",
                       what, n);
    size_t want = std::max<size_t>(n, (size_t)(b.cap * 1.25));
    if (want == 0) want = 1;
    ++c->epoch;
    b.release();
    CUDA_TRY(cudaMalloc((void **)&b.p, want * sizeof(T)));
    b.cap = want;
    return SPHGRAV_OK;
}

static int ensure_pinned(sphgrav_ctx *c, PinnedBuf &b, size_t bytes)
{
    if (bytes <= b.cap && b.p) return SPHGRAV_OK;
    if (c->capturing) return set_err(SPHGRAV_ERR_PROTOCOL, "host staging cannot grow during capture");
    size_t want = std::max<size_t>(bytes, (size_t)(b.cap * 1.25));
    ++c->epoch;
    b.release();
    CUDA_TRY(cudaMallocHost(&b.p, want));
    b.cap = want;
    return SPHGRAV_OK;
}

static int use_device(sphgrav_ctx *c)
{
    int cur = -1;
    CUDA_TRY(cudaGetDevice(&cur));
    if (cur != c->device) CUDA_TRY(cudaSetDevice(c->device));
    return SPHGRAV_OK;
}

// ------------------------------------------------------- variant choice
static const int kMinChunkJ = 2048;  // shortest j-chunk worth a partial slot
// The FP64 kernel's items are slower per source, so a short chunk still
// outweighs its partial slot; small sets need them to fill the GPU (16K:
// 1,024 items of 2,048 sources left a third of the SMs idle at the end).
static const int kMinChunkJ64 = 512;
// FP64 variant that recomputes the refine-listed rows (few rows per set: the
// smallest row tile)
static const int kRefineVariant = 0;
// ... and for sets of at most kRefineSmallN particles the 64-source-tile
// shape with 64-source chunks (16K: 22 rows refined in 76 us with 256-source
// chunks; their near pairs, one after another per row, set the time)
static const int kRefineVariantSmall = 12;
static const int kRefineSmallN = 65536;
static int refine_variant(const Plan &P) { return P.max_n <= kRefineSmallN ? kRefineVariantSmall : kRefineVariant; }

static int ceil_log2(long long v)
{
    int b = 0;
    while ((1ll << b) < v) b++;
    return b;
}

static int bucket_of(const std::vector<int> &offsets, bool full_rows, int ni)
{
    double s1 = 0.0, s2 = 0.0;
    for (size_t s = 0; s + 1 < offsets.size(); s++) {
        double n = offsets[s + 1] - offsets[s];
        double rows = full_rows ? n : ni;
        s1 += rows;
        s2 += rows * n;
    }
    double nw = s1 > 0 ? s2 / s1 : 1.0;
    return (int)std::floor(std::log2(std::max(1.0, nw)));
}

static int variant_by_name(int precision, const std::string &name)
{
    for (int v = 0; v < variant_count(precision); v++)
        if (name == variant_info(precision, v).name) return v;
    return -1;
}

static int choose_variant(sphgrav_ctx *c, int precision, const std::vector<int> &offsets,
                          bool full_rows, int ni)
{
    if (c->forced_variant[precision] >= 0) return c->forced_variant[precision];
    const int b = bucket_of(offsets, full_rows, ni);
    auto it = c->tuned[precision].find(b);
    if (it != c->tuned[precision].end()) {
        int v = variant_by_name(precision, it->second);
        if (v >= 0) return v;
    }
    const bool batch = offsets.size() > 2;
    // FP64 (kernel ms on B200), 128-source tiles throughout.  One-warp CTAs
    // wait only on their own warp at the per-tile stage release.
    //   single sets 2^13..2^16: one-warp CTAs, one row per thread (16K: 0.80
    //     vs 0.81 for 4-warp CTAs; 32K: 1.93 vs 2.18 for two rows per
    //     thread; 64K: 6.13 vs 6.32)
    //   from 2^17, and batches from 2^15: one-warp CTAs, two rows per thread
    //     (131K: 21.9 vs 23.1 for one row; 262K: 81.9 vs 88.0; 1M: 1235 vs
    //     1356; the batch of 4K-131K models: 156 vs 170; the 16 collision
    //     snapshots: 1396 vs 1535)
    //   below: 4-warp CTAs, one row per thread
    if (precision == SPHGRAV_FP64) {
        if (b >= 17 || (batch && b >= 15)) return 9;
        if (!batch && b >= 13) return 13;
        return 0;
    }
    // split-FP32 defaults by pair-weighted mean N = 2^b, from sweeps on B200
    // (pair-kernel ms of the chosen shape vs the runner-up):
    //   b >= 20, and batches from 2^18: W12K2Q1, 7 stages (1M: 488.5; the
    //                                 16 collision snapshots, mean 317K: 562
    //                                 vs 579 for W12K1Q1, whole call 587 vs 595)
    //   17..19, and batches from 2^15: W12K1Q1, 7 stages (131K: 9.28 vs 9.65
    //                                 for W15K1Q2; the batch of 4K-131K models,
    //                                 mean 61K: 64.7 vs 67.3; 262K collision:
    //                                 35.40 vs 35.42 for W12K2Q1, whose
    //                                 768-row tiles leave more rows beyond
    //                                 8 H of their centre for the FP64
    //                                 refine: 2,357 rows, whole call 37.5 ms)
    //   15..16   W15K1Q2             (32K: 0.791 vs 0.827; 64K: 2.52 vs 2.58)
    //   13..14   W12K1Q4, 7 stages   (8K: 0.135 vs 0.142; 16K: 0.307 vs 0.302 for
    //                                 W15K1Q2, whose 240-row tiles leave 69 rows
    //                                 for the FP64 refine against 22: whole call
    //                                 0.51 vs 0.63 ms)
    //   <= 12    W8K1Q4              (4K: 75 vs 72 G pairs/s)
    // Twelve consumer warps put the same number of consumers on every SMSP;
    // all without the Newton step on rsqrt.approx: in FP32 the step's own
    // roundings cost more than it corrects (RMS error 3.2e-8 vs 3.7e-8 at
    // N=1M, 2.7e-8 vs 4.4e-8 at N=16K, max error equal or lower on every
    // workload) and it is 3 of 16 FMA-pipe lane-ops per pair.
    if (b >= 20 || (batch && b >= 18)) return 0;
    if (b >= 17 || (batch && b >= 15)) return 2;
    if (b >= 15) return 3;
    if (b >= 13) return 5;
    return 4;
}

// ------------------------------------------------------------------ plan
// The work plan of one call: host-only arithmetic (resident = persistent CTAs
// of the variant on the device), so it also runs without a GPU
// (sphgrav_plan_preview).
static int build_plan(int resident, const std::vector<int> &offsets, bool full_rows, int i_lo,
                      int ni, int precision, int variant, Plan &P, bool tree = false)
{
    const VariantInfo &V = variant_info(precision, variant);
    P = Plan();
    P.offsets = offsets;
    P.full_rows = full_rows;
    P.i_lo = i_lo;
    P.ni = ni;
    P.precision = precision;
    P.variant = variant;
    P.tree = tree;
    P.nsets = (int)offsets.size() - 1;
    P.itile = V.itile();
    P.tj = V.tj;
    long long poff = 0, ioff = 0, toff = 0, moff = 0;
    for (int s = 0; s < P.nsets; s++) {
        SetDesc d{};
        memset(&d, 0, sizeof(d));
        d.n = offsets[s + 1] - offsets[s];
        d.off = offsets[s];
        d.poff = (int)poff;
        d.npad = (d.n + PAD_J - 1) / PAD_J * PAD_J;
        d.ioff = (int)ioff;
        d.ni = full_rows ? d.n : ni;
        d.i_lo = full_rows ? 0 : i_lo;
        d.tile_off = (int)toff;
        d.ntiles = (d.ni + P.itile - 1) / P.itile;
        d.meta_off = (int)moff;
        poff += d.npad;
        ioff += d.ni;
        toff += d.ntiles;
        moff += d.npad / META_J;
        P.max_n = std::max(P.max_n, d.n);
        P.max_npad = std::max(P.max_npad, d.npad);
        P.sets.push_back(d);
    }
    if (poff > 0x7fffffffll - PAD_J) return set_err(SPHGRAV_ERR_TOO_LARGE, "too many particles");
    P.ntot = offsets.back() - offsets.front();
    P.npad_tot = (int)poff;
    P.rows_tot = (int)ioff;
    P.ntiles = (int)toff;
    P.nmeta = (int)moff;
    const int target = 4 * resident;
    const int min_chunk = precision == SPHGRAV_FP64 ? kMinChunkJ64 : kMinChunkJ;
    // One set: items are all alike, so pick the chunk count whose item count
    // fills the last wave of persistent CTAs best (ties: fewer chunks).
    int single_nch = 0;
    if (P.nsets == 1 && P.ntiles > 0) {
        const SetDesc &d = P.sets[0];
        const int jtiles = (d.n + P.tj - 1) / P.tj;
        const int maxch = std::max(1, std::min(jtiles, std::min(64, (int)(((long long)jtiles * P.tj) / min_chunk))));
        // item costs differ (near-field work is uneven), so small sets want
        // several items per CTA for the queue to balance them
        const int nch_min = std::min(maxch, std::max(1, (3 * resident + P.ntiles - 1) / P.ntiles));
        double best = -1.0;
        for (int nch = nch_min; nch <= maxch; nch++) {
            const double waves = (double)P.ntiles * nch / resident;
            const double eff = waves / std::ceil(waves) - 0.002 * nch;  // small per-chunk cost
            if (eff > best + 1e-9) { best = eff; single_nch = nch; }
        }
    }
    // Chunk counts per i-tile.  Few tiles (<= 2 waves of persistent CTAs),
    // or the FP64 kernel: every tile of a set gets the same count, enough
    // items for the queue to balance (one set: the count that fills the last
    // wave best).  Split-FP32 with many tiles: every tile is one whole-j-range
    // item, except the TAIL_DIV-th part of a wave of tiles that comes last
    // in the longest-first order, which is cut into 4 chunks: the queue still
    // ends on small items, and the FP64 partial sums (written per item,
    // merged by k_merge) stay about the size of the outputs instead of 4x.
    // (The FP64 kernel keeps chunks everywhere: a row tile holding a point
    // mass with a large H, like the red giant's core, pays the serial near-
    // pair path for most of the set and must not be one item.)
    constexpr int TAIL_DIV = 2, TAIL_CHUNKS = 4;
    std::vector<int> tile_nch(P.ntiles, 1);
    auto set_maxch = [&](const SetDesc &d) {
        const int jtiles = (d.n + P.tj - 1) / P.tj;
        return std::max(1, std::min(jtiles, (int)(((long long)jtiles * P.tj) / min_chunk)));
    };
    if (P.ntiles <= 2 * resident || precision != SPHGRAV_F32SPLIT) {
        for (int s = 0; s < P.nsets; s++) {
            const SetDesc &d = P.sets[s];
            int nch = P.ntiles > 0 ? (target + P.ntiles - 1) / P.ntiles : 1;
            nch = std::max(1, std::min(nch, set_maxch(d)));
            if (single_nch > 0) nch = single_nch;
            for (int t = 0; t < d.ntiles; t++) tile_nch[d.tile_off + t] = nch;
        }
    } else {
        // whole-tile costs, longest first (stable: ties keep set and tile order)
        std::vector<std::pair<long long, int>> order;
        order.reserve(P.ntiles);
        for (const SetDesc &d : P.sets)
            for (int t = 0; t < d.ntiles; t++)
                order.push_back({(long long)std::min(P.itile, d.ni - t * P.itile) * d.npad,
                                 d.tile_off + t});
        std::stable_sort(order.begin(), order.end(),
                         [](const std::pair<long long, int> &a, const std::pair<long long, int> &b) {
                             return a.first > b.first;
                         });
        const int tail = std::max(1, resident / TAIL_DIV);
        for (int k = P.ntiles - tail; k < P.ntiles; k++) {
            const int t = order[k].second;
            tile_nch[t] = std::min(TAIL_CHUNKS, set_maxch(P.sets[P.tile_set_of(t)]));
        }
    }
    int slot = 0;
    P.nchunks_max = 1;
    struct Cost { long long cost; WorkItem w; };
    std::vector<Cost> items;
    for (int s = 0; s < P.nsets; s++) {
        SetDesc &d = P.sets[s];
        const int jtiles = (d.n + P.tj - 1) / P.tj;
        d.nchunks = 1;
        d.slot_off = slot;
        for (int t = 0; t < d.ntiles; t++) {
            const int rows = std::min(P.itile, d.ni - t * P.itile);
            const int nch = tile_nch[d.tile_off + t];
            P.tile_slots.push_back({slot, nch});
            d.nchunks = std::max(d.nchunks, nch);
            for (int ch = 0; ch < nch; ch++) {
                WorkItem w;
                memset(&w, 0, sizeof(w));
                w.set = s;
                w.tile = t;
                w.chunk = ch;
                w.slot = slot + ch;
                w.jb = (int)((long long)jtiles * ch / nch) * P.tj;
                w.je = (int)((long long)jtiles * (ch + 1) / nch) * P.tj;
                items.push_back({(long long)rows * (w.je - w.jb), w});
            }
            slot += nch;
        }
        P.nchunks_max = std::max(P.nchunks_max, d.nchunks);
        for (int t = 0; t < d.ntiles; t++) P.tile_set.push_back(s);
        for (int r = 0; r < d.npad / META_J; r++) P.meta_set.push_back(s);
    }
    // longest first: the dynamic queue then balances like LPT scheduling
    std::stable_sort(items.begin(), items.end(),
                     [](const Cost &a, const Cost &b) { return a.cost > b.cost; });
    for (auto &it : items) P.items.push_back(it.w);
    P.nitems = (int)P.items.size();
    P.nslots = slot;
    P.grid = std::max(1, std::min(P.nitems, resident));
    const int setbits = ceil_log2(std::max(1, P.nsets));
    // Curve-key bits per axis.  The octree's levels are the key's 3-bit
    // digits, so tree calls keep 21.  For the direct sums every 8 key bits
    // cost the sort a pass, which matters only for small sets: up to 65,536
    // particles they take cells just fine enough that particles rarely
    // share one (2^(3b) cells, about 2^15 per particle, at least 2^10 per
    // axis; 16K: 4 passes instead of 8).  Larger sets keep 21 bits: a curve
    // of another order has another orientation, so it tiles a centred star
    // differently (on the 1M red giant 18 refined rows instead of 8, RMS
    // error 6.2e-8 instead of 4.7e-8), for a sort that is < 0.1% of the call.
    const int want = (tree || P.max_n > 65536)
                         ? 21
                         : std::max(10, (ceil_log2(std::max(2, P.max_n)) + 2) / 3 + 5);
    P.bits = std::min(std::min(21, want), (64 - setbits) / 3);
    P.end_bit = 3 * P.bits + setbits;
    P.valid = true;
    return SPHGRAV_OK;
}

static bool plan_matches(const Plan &P, const std::vector<int> &offsets, bool full_rows, int i_lo,
                         int ni, int precision, int variant, bool tree)
{
    return P.valid && P.offsets == offsets && P.full_rows == full_rows &&
           (full_rows || (P.i_lo == i_lo && P.ni == ni)) && P.precision == precision &&
           P.variant == variant && P.tree == tree;
}

static int prepare(sphgrav_ctx *c, const std::vector<int> &offsets, bool full_rows, int i_lo,
                   int ni, int precision, int variant, bool tree = false)
{
    if (!plan_matches(c->plan, offsets, full_rows, i_lo, ni, precision, variant, tree)) {
        if (c->capturing)
            return set_err(SPHGRAV_ERR_PROTOCOL,
                           "work plan changed during a graph capture; call the entry point once "
                           "with the same sizes before capturing");
        Plan P;
        TRY(build_plan(variant_occupancy(precision, variant) * c->sm_count, offsets, full_rows,
                       i_lo, ni, precision, variant, P, tree));
        ++c->epoch;  // graphs captured under the old plan must not replay
        TRY(ensure(c, c->sets, std::max(1, P.nsets), "sets"));
        TRY(ensure(c, c->tile_set, std::max(1, P.ntiles), "tile_set"));
        TRY(ensure(c, c->tile_slots, std::max(1, P.ntiles), "tile_slots"));
        TRY(ensure(c, c->meta_set, std::max(1, P.nmeta), "meta_set"));
        TRY(ensure(c, c->items, std::max(1, P.nitems), "items"));
        CUDA_TRY(cudaMemcpyAsync(c->sets.p, P.sets.data(), sizeof(SetDesc) * P.nsets,
                                 cudaMemcpyHostToDevice, c->stream));
        if (P.ntiles) {
            CUDA_TRY(cudaMemcpyAsync(c->tile_set.p, P.tile_set.data(), sizeof(int) * P.ntiles,
                                     cudaMemcpyHostToDevice, c->stream));
            CUDA_TRY(cudaMemcpyAsync(c->tile_slots.p, P.tile_slots.data(), sizeof(int2) * P.ntiles,
                                     cudaMemcpyHostToDevice, c->stream));
        }
        if (P.nmeta)
            CUDA_TRY(cudaMemcpyAsync(c->meta_set.p, P.meta_set.data(), sizeof(int) * P.nmeta,
                                     cudaMemcpyHostToDevice, c->stream));
        if (P.nitems)
            CUDA_TRY(cudaMemcpyAsync(c->items.p, P.items.data(), sizeof(WorkItem) * P.nitems,
                                     cudaMemcpyHostToDevice, c->stream));
        // pageable-source copies are staged before return; the vectors may change after
        c->plan = std::move(P);
    }
    const Plan &P = c->plan;
    const size_t np = std::max(1, P.npad_tot);
    if (np > c->pcap || !c->d64.p) {
        TRY(ensure(c, c->d64, 5 * np, "sorted fp64"));
        TRY(ensure(c, c->orig, np, "orig"));
        TRY(ensure(c, c->flag, np, "flag"));
        TRY(ensure(c, c->f32, 8 * np, "sorted f32"));
        c->pcap = np;
    }
    const size_t nt = std::max(1, P.ntot);
    TRY(ensure(c, c->keys_in, nt, "keys"));
    TRY(ensure(c, c->keys_out, nt, "keys"));
    TRY(ensure(c, c->vals_in, nt, "vals"));
    TRY(ensure(c, c->vals_out, nt, "vals"));
    TRY(ensure(c, c->ilist, std::max(1, P.rows_tot), "rows"));
    TRY(ensure(c, c->bbox, 6 * (size_t)std::max(1, P.nsets), "bbox"));
    TRY(ensure(c, c->imeta, std::max(1, P.ntiles), "itile meta"));
    TRY(ensure(c, c->jmeta, std::max(1, P.nmeta), "jtile meta"));
    TRY(ensure(c, c->partials, (size_t)std::max(1, P.nslots) * 4 * P.itile, "partials"));
    TRY(ensure(c, c->wtile, std::max(1, P.ntiles), "wtile"));
    TRY(ensure(c, c->wdev, std::max(1, P.nsets), "W"));
    if (P.precision == SPHGRAV_F32SPLIT && (c->refine_T > 0.0 || c->keep_scale)) {
        TRY(ensure(c, c->gpart, (size_t)std::max(1, P.nslots) * P.itile, "error-scale partials"));
        TRY(ensure(c, c->rcount, std::max(1, P.nsets), "refine counts"));
        TRY(ensure(c, c->rlist, std::max(1, P.rows_tot), "refine rows"));
        TRY(ensure(c, c->rsets, std::max(1, P.nsets), "refine sets"));
        TRY(ensure(c, c->rnitems, 1, "refine items"));
        TRY(ensure(c, c->rhead, 1, "refine head"));
        const int rv = refine_variant(P);
        const VariantInfo &V = variant_info(SPHGRAV_FP64, rv);
        long long tiles = 0;
        for (const SetDesc &d : P.sets) tiles += (d.ni + V.itile() - 1) / V.itile();
        const long long target = 4ll * variant_occupancy(SPHGRAV_FP64, rv) * c->sm_count;
        const size_t cap = (size_t)std::max(1ll, std::max(tiles, target));
        TRY(ensure(c, c->ritems, cap, "refine items"));
        TRY(ensure(c, c->rpart, cap * 4 * V.itile(), "refine partials"));
        TRY(ensure(c, c->rlitems, REFINE_LIGHT_CAP, "refine row-chunk items"));
        TRY(ensure(c, c->rlpart, 4 * (size_t)REFINE_LIGHT_CAP, "refine row-chunk partials"));
        TRY(ensure(c, c->rnlight, 1, "refine row-chunk items"));
        if (c->keep_scale) TRY(ensure(c, c->scale, std::max(1, P.ntot), "error scale"));
    }
    const size_t sb = sort_temp_bytes(P.ntot, P.end_bit);
    TRY(ensure(c, c->sort_temp, std::max<size_t>(sb, 1), "sort temp"));
    if (!P.full_rows) {
        const size_t selb = select_temp_bytes(P.ntot);
        TRY(ensure(c, c->sel_temp, std::max<size_t>(selb, 1), "select temp"));
    }
    return SPHGRAV_OK;
}

static SortedF64 sorted64(sphgrav_ctx *c)
{
    SortedF64 D;
    const size_t np = c->pcap;
    D.x = c->d64.p;
    D.y = D.x + np;
    D.z = D.y + np;
    D.m = D.z + np;
    D.h2 = D.m + np;
    D.orig = c->orig.p;
    D.flag = c->flag.p;
    return D;
}

static SortedF32 sorted32(sphgrav_ctx *c)
{
    SortedF32 F;
    const size_t np = c->pcap;
    F.xh = c->f32.p;
    F.xl = F.xh + np;
    F.yh = F.xl + np;
    F.yl = F.yh + np;
    F.zh = F.yl + np;
    F.zl = F.zh + np;
    F.m = F.zl + np;
    F.h2 = F.m + np;
    return F;
}

// The per-call pipeline on device-resident inputs and outputs.
// Barnes-Hut mode: the preparation of the direct path (validation, Hilbert
// sort, gather), then the octree, its multipoles, the group walk and the
// scatter of the requested rows.  One particle set per call.
static int run_tree(sphgrav_ctx *c, const std::vector<int> &offsets, bool full_rows, int i_lo,
                    int ni, const InputsDev &in, const OutputsDev &out, double *W, int nkernel)
{
    TRY(prepare(c, offsets, full_rows, i_lo, ni, SPHGRAV_FP64, 0, true));
    const Plan &P = c->plan;
    cudaStream_t st = c->stream;
    const int n = P.ntot, nslots = P.npad_tot, nsets = P.nsets;
    if (n == 0) {
        if (W && nsets > 0) CUDA_TRY(cudaMemsetAsync(W, 0, sizeof(double) * nsets, st));
        return SPHGRAV_OK;
    }
    // Inside a graph capture every count stays on the device: all key levels
    // are issued, grids are sized for bounds and kernels read the counts
    // there; buffers must already have the sizes an eager call of the same
    // sizes gave them (ensure refuses to grow during a capture).
    const bool dev = c->capturing;
    SortedF64 D = sorted64(c);
    SortedF32 F = sorted32(c);
    CUDA_TRY(launch_validate(in, n, c->err.p, st));
    CUDA_TRY(launch_bbox(c->sets.p, P.nsets, P.max_n, in, c->bbox.p, st));
    CUDA_TRY(launch_sfc_keys(c->sets.p, P.nsets, P.max_n, in, c->bbox.p, P.bits, c->keys_in.p,
                           c->vals_in.p, st));
    CUDA_TRY(launch_sort(c->sort_temp.p, c->sort_temp.cap, c->keys_in.p, c->keys_out.p,
                         c->vals_in.p, c->vals_out.p, n, P.end_bit, st));
    CUDA_TRY(launch_gather(c->sets.p, P.nsets, P.max_npad, in, c->vals_out.p, D, F, st));
    // the tree indexes sorted slots; with one set they are the sorted order
    const unsigned long long *keys = c->keys_out.p;
    if (nsets > 1) {
        TRY(ensure(c, c->tkeys, (size_t)nslots, "tree keys"));
        CUDA_TRY(tree_slot_keys(c->sets.p, nsets, P.max_n, c->keys_out.p, c->tkeys.p, st));
        keys = c->tkeys.p;
    }
    TRY(ensure(c, c->tcnt, (size_t)n + 1, "tree scratch"));
    TRY(ensure(c, c->toff, (size_t)n + 1, "tree scratch"));
    // scan scratch, also for a walking-order sort of up to n groups (the
    // bound a captured call sorts)
    TRY(ensure(c, c->tscan, std::max(tree_scan_temp_bytes(n + 1), tree_order_temp_bytes(n)),
               "tree scan"));
    TRY(ensure(c, c->tnodes, std::max<size_t>(c->tnodes.cap, 2 * (size_t)n + 64 + nsets), "tree nodes"));
    // walking groups: runs of sibling nodes with <= TREE_GROUP particles
    TRY(ensure(c, c->tglist, (size_t)n, "tree groups"));
    TRY(ensure(c, c->tgorder, (size_t)n, "tree groups"));
    TRY(ensure(c, c->theavy, (size_t)n, "tree heavy groups"));
    TRY(ensure(c, c->tgcount, 2, "tree groups"));  // [0] groups, [1] heavy groups
    TRY(ensure(c, c->tlv, TREE_LV_SIZE, "tree levels"));
    const int levels = P.bits;
    TreeBuildArgs t;
    t.n = n;
    t.levels = levels;
    t.nroots = nsets;
    t.sets = c->sets.p;
    t.keys = keys;
    t.cnt = c->tcnt.p;
    t.off = c->toff.p;
    t.scan_temp = c->tscan.p;
    t.scan_temp_bytes = c->tscan.cap;
    t.lv = c->tlv.p;
    int lvh[TREE_LV_SIZE];
    DevCount nn{0, nullptr};
    int depth = 0;
    if (!dev) {
        // Eager: TREE_BATCH levels at a time; one read-back of the level
        // table per batch shows whether the tree has ended (an empty level)
        // or the node array is full (it is regrown and the build repeated).
        constexpr int TREE_BATCH = 4;
        for (;;) {
            TRY(ensure(c, c->tgflag, c->tnodes.cap, "tree groups"));
            t.nodes = c->tnodes.p;
            t.cap = (int)std::min<size_t>(c->tnodes.cap, 0x7fffffff);
            t.gflag = c->tgflag.p;
            bool overflow = false;
            for (int l0 = 0; l0 < levels; l0 += TREE_BATCH) {
                const int l1 = std::min(l0 + TREE_BATCH, levels);
                CUDA_TRY(tree_build_levels(t, l0, l1, st));
                CUDA_TRY(cudaMemcpyAsync(lvh, c->tlv.p, sizeof(lvh), cudaMemcpyDeviceToHost, st));
                CUDA_TRY(cudaStreamSynchronize(st));
                overflow = lvh[TREE_LV_OVERFLOW] != 0;
                nn.host = lvh[l1 + 1];  // end of level l1, the last one written
                depth = l1;
                if (overflow || lvh[l1 + 1] == lvh[l1]) break;  // level l1 is empty
            }
            if (!overflow) break;
            TRY(ensure(c, c->tnodes, 2 * c->tnodes.cap, "tree nodes"));
        }
        while (depth > 0 && lvh[depth + 1] == lvh[depth]) depth--;  // deepest non-empty level
        // room for a captured call of these sizes: twice this tree's nodes
        const size_t room = std::min<size_t>(c->tnodes.cap, 2 * (size_t)nn.host + 1024);
        TRY(ensure(c, c->tgeom, room, "tree geometry"));
        TRY(ensure(c, c->tmp, room, "tree multipoles"));
        TRY(ensure(c, c->tacc, tree_acc_bytes((int)room) / sizeof(double), "tree node sums"));
    } else {
        // Captured: every level, no read-back; the node capacity is what the
        // eager call left (twice its tree); a replay whose tree needs more
        // raises DEVERR_TREE_CAP (SPHGRAV_ERR_TOO_LARGE at the next sync)
        const size_t cap = std::min({c->tnodes.cap, c->tgflag.cap, c->tgeom.cap, c->tmp.cap,
                                     c->tacc.cap * sizeof(double) / tree_acc_bytes(1)});
        if (cap < (size_t)nsets + 1 || !c->tgflag.p || !c->tgeom.p)
            return set_err(SPHGRAV_ERR_PROTOCOL,
                           "capture a tree call only after an eager tree call of the same sizes");
        t.nodes = c->tnodes.p;
        t.cap = (int)std::min<size_t>(cap, 0x7fffffff);
        t.gflag = c->tgflag.p;
        CUDA_TRY(tree_build_levels(t, 0, levels, st));
        CUDA_TRY(tree_check_build(c->tlv.p, c->err.p, st));
        nn = DevCount{t.cap, c->tlv.p + levels + 1};
        depth = levels;
    }
    CUDA_TRY(tree_groups(nn, c->tnodes.p, c->tgflag.p, c->tglist.p, c->tgcount.p, st));
    DevCount ng{n, c->tgcount.p};
    if (!dev) {
        CUDA_TRY(cudaMemcpyAsync(&ng.host, c->tgcount.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        ng.dev = nullptr;
    }
    // walking order: largest H first (the build's scratch holds the sort keys)
    CUDA_TRY(tree_order_groups(ng, c->tglist.p, c->tgorder.p, D.h2, (unsigned *)c->tcnt.p,
                               (unsigned *)c->toff.p, c->tscan.p, c->tscan.cap, st));
    CUDA_TRY(tree_props(nn, c->tnodes.p, D, c->theta, c->tlv.p, dev ? nullptr : lvh, depth, n,
                        c->tacc.p, c->tgeom.p, c->tmp.p, st));
    TRY(ensure(c, c->tstack, (size_t)tree_walk_warps(c->sm_count) * TREE_STACK, "tree stack"));
    TRY(ensure(c, c->tres, 4 * (size_t)nslots, "tree results"));
    // heavy groups' partial sums: room for TREE_HEAVY_CAP groups (a captured
    // call's bound), more when an eager call finds more
    TRY(ensure(c, c->theavy_part, tree_heavy_partials(TREE_HEAVY_CAP, P.max_n), "tree heavy sums"));
    CUDA_TRY(cudaMemsetAsync(c->head.p, 0, sizeof(int), st));
    TreeWalkArgs a;
    a.nodes = c->tnodes.p;
    a.geom = c->tgeom.p;
    a.mp = c->tmp.p;
    a.D = D;
    a.n = nslots;
    a.ngroups = ng.host;
    a.ngroups_dev = ng.dev;
    a.nroots = nsets;
    a.groups = c->tgorder.p;
    CUDA_TRY(cudaMemsetAsync(c->tgcount.p + 1, 0, sizeof(int), st));
    a.heavy = c->theavy.p;
    a.nheavy = c->tgcount.p + 1;
    a.nkernel = nkernel;
    a.head = c->head.p;
    a.stack = c->tstack.p;
    a.stack_cap = TREE_STACK;
    a.out = c->tres.p;
    a.err = c->err.p;
    const bool timed = c->profiling && !dev;
    if (timed) {
        if (c->prof_used == c->prof_events.size()) {
            cudaEvent_t e0, e1;
            CUDA_TRY(cudaEventCreate(&e0));
            CUDA_TRY(cudaEventCreate(&e1));
            c->prof_events.push_back({e0, e1});
        }
        CUDA_TRY(cudaEventRecord(c->prof_events[c->prof_used].first, st));
    }
    CUDA_TRY(tree_walk(a, c->sm_count, st));
    // groups whose particles' softening spheres hold too many particles: the
    // direct FP64 sum over their own set
    int nheavy = -1;
    if (!dev) {
        CUDA_TRY(cudaMemcpyAsync(&nheavy, c->tgcount.p + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        if (nheavy > TREE_HEAVY_CAP)
            TRY(ensure(c, c->theavy_part, tree_heavy_partials(nheavy, P.max_n), "tree heavy sums"));
    }
    if (dev || nheavy > 0) {
        const int hcap = dev ? TREE_HEAVY_CAP : std::max(nheavy, TREE_HEAVY_CAP);
        CUDA_TRY(tree_heavy(dev ? 0 : nheavy, c->tgcount.p + 1, hcap, c->theavy.p, c->tgorder.p,
                            c->tnodes.p, nsets, D, nslots, P.max_n, nkernel, c->theavy_part.p,
                            c->tres.p, c->err.p, st));
    }
    c->tree_groups_last = dev ? -1 : ng.host;
    c->tree_heavy_last = nheavy;
    if (timed) CUDA_TRY(cudaEventRecord(c->prof_events[c->prof_used++].second, st));
    CUDA_TRY(tree_scatter(nslots, full_rows ? 0 : i_lo, full_rows ? n : ni, c->tres.p, D.orig, out,
                          st));
    if (W) CUDA_TRY(tree_wsum(c->sets.p, nsets, nslots, c->tres.p, D.m, W, st));
    return SPHGRAV_OK;
}

// FP64 recomputation of the rows the merge listed (split-FP32 calls): a
// device-written plan, the FP64 kernel over it, and the scatter of the
// refined rows over the split-FP32 ones.  No host round trip.
static int run_refine(sphgrav_ctx *c, int nkernel, const SortedF64 &D, const OutputsDev &out)
{
    const Plan &P = c->plan;
    cudaStream_t st = c->stream;
    const int v = refine_variant(P);
    const VariantInfo &V = variant_info(SPHGRAV_FP64, v);
    const int resident = variant_occupancy(SPHGRAV_FP64, v) * c->sm_count;
    const int min_j = v == kRefineVariantSmall ? 64 : 256;  // sources per refine chunk, at least
    CUDA_TRY(launch_refine_plan(c->sets.p, P.nsets, c->rcount.p, V.itile(), V.tj, min_j, 4 * resident,
                                (int)std::min<size_t>(c->ritems.cap, 0x7fffffff), c->rsets.p,
                                c->ritems.p, c->rnitems.p, c->rlitems.p, c->rnlight.p, c->err.p,
                                st));
    CUDA_TRY(cudaMemsetAsync(c->rhead.p, 0, sizeof(int), st));
    // sets with few listed rows: one warp per (row, source chunk)
    CUDA_TRY(launch_refine_light(c->rsets.p, c->rlitems.p, c->rnlight.p, c->rlist.p, D, nkernel,
                                 c->rlpart.p, c->sm_count, st));
    ComputeArgs a{};
    a.sets = c->rsets.p;
    a.items = c->ritems.p;
    a.nitems = 0;
    a.nitems_dev = c->rnitems.p;
    a.head = c->rhead.p;
    a.D = D;
    a.F = sorted32(c);
    a.ilist = c->rlist.p;
    a.jmeta = c->jmeta.p;
    a.partials = c->rpart.p;
    a.gpart = nullptr;
    a.err = c->err.p;
    a.nkernel = nkernel;
    a.itile = V.itile();
    a.band2 = 1.f;
    CUDA_TRY(launch_compute(SPHGRAV_FP64, v, resident, a, st));
    CUDA_TRY(launch_refine_merge(c->sets.p, c->rsets.p, c->tile_set.p, P.ntiles, P.itile, V.itile(),
                                 c->rcount.p, c->rlist.p, D, c->rpart.p, c->rlpart.p, out, st));
    return SPHGRAV_OK;
}

static int run_device(sphgrav_ctx *c, const std::vector<int> &offsets, bool full_rows, int i_lo,
                      int ni, const InputsDev &in, const OutputsDev &out, double *W, int nkernel,
                      int precision)
{
    if (nkernel < 0 || nkernel > 2)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "nkernel must be 0, 1 or 2 (got %d)", nkernel);
    if (precision == SPHGRAV_TREE)
        return run_tree(c, offsets, full_rows, i_lo, ni, in, out, W, nkernel);
    if (precision != SPHGRAV_FP64 && precision != SPHGRAV_F32SPLIT)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "unknown precision %d", precision);
    const int variant = choose_variant(c, precision, offsets, full_rows, ni);
    TRY(prepare(c, offsets, full_rows, i_lo, ni, precision, variant));
    const Plan &P = c->plan;
    cudaStream_t st = c->stream;
    if (P.ntot == 0) return SPHGRAV_OK;
    SortedF64 D = sorted64(c);
    SortedF32 F = sorted32(c);
    CUDA_TRY(launch_validate(in, P.ntot, c->err.p, st));
    CUDA_TRY(launch_bbox(c->sets.p, P.nsets, P.max_n, in, c->bbox.p, st));
    CUDA_TRY(launch_sfc_keys(c->sets.p, P.nsets, P.max_n, in, c->bbox.p, P.bits, c->keys_in.p,
                           c->vals_in.p, st));
    CUDA_TRY(launch_sort(c->sort_temp.p, c->sort_temp.cap, c->keys_in.p, c->keys_out.p,
                         c->vals_in.p, c->vals_out.p, P.ntot, P.end_bit, st));
    CUDA_TRY(launch_gather(c->sets.p, P.nsets, P.max_npad, in, c->vals_out.p, D, F, st));
    if (P.full_rows) {
        CUDA_TRY(launch_rows_full(c->sets.p, P.nsets, P.max_n, c->ilist.p, st));
    } else {
        CUDA_TRY(launch_rows_range(P.sets[0], D, c->ilist.p, c->nsel.p, c->sel_temp.p,
                                   c->sel_temp.cap, st));
    }
    if (precision == SPHGRAV_F32SPLIT)
        CUDA_TRY(launch_itile_meta(c->sets.p, P.nsets, P.ntiles, c->tile_set.p, P.itile,
                                   c->ilist.p, D, c->imeta.p, st));
    // source boxes: both kernels skip the per-pair near test on far tiles
    CUDA_TRY(launch_jmeta(c->sets.p, P.nsets, P.nmeta, c->meta_set.p, D, c->jmeta.p, st));
    CUDA_TRY(cudaMemsetAsync(c->head.p, 0, sizeof(int), st));
    ComputeArgs a{};
    a.sets = c->sets.p;
    a.items = c->items.p;
    a.nitems = P.nitems;
    a.head = c->head.p;
    a.D = D;
    a.F = F;
    a.ilist = c->ilist.p;
    a.imeta = c->imeta.p;
    a.jmeta = c->jmeta.p;
    a.partials = c->partials.p;
    a.err = c->err.p;
    a.nkernel = nkernel;
    a.itile = P.itile;
    a.band2 = (float)(c->fp64_band * c->fp64_band);
    a.nitems_dev = nullptr;
    const bool refine = precision == SPHGRAV_F32SPLIT && c->refine_T > 0.0;
    const bool want_g = precision == SPHGRAV_F32SPLIT && (refine || c->keep_scale);
    a.gpart = want_g ? c->gpart.p : nullptr;
    const bool timed = c->profiling && !c->capturing && P.nitems > 0;
    if (timed && precision == SPHGRAV_F32SPLIT && phases_built()) {
        if (!c->phases.p) {
            TRY(ensure(c, c->phases, PHASE_COUNTERS, "phase counters"));
            CUDA_TRY(cudaMemsetAsync(c->phases.p, 0, sizeof(unsigned long long) * PHASE_COUNTERS, st));
        }
        a.phases = c->phases.p;
    }
    if (timed) {
        if (c->prof_used == c->prof_events.size()) {
            cudaEvent_t e0, e1;
            CUDA_TRY(cudaEventCreate(&e0));
            CUDA_TRY(cudaEventCreate(&e1));
            c->prof_events.push_back({e0, e1});
        }
        CUDA_TRY(cudaEventRecord(c->prof_events[c->prof_used].first, st));
    }
    if (P.nitems > 0) CUDA_TRY(launch_compute(precision, P.variant, P.grid, a, st));
    if (timed) CUDA_TRY(cudaEventRecord(c->prof_events[c->prof_used++].second, st));
    MergeRefine R;
    c->scale_n = 0;
    if (want_g) {
        R.gpart = c->gpart.p;
        R.scale = c->keep_scale ? c->scale.p : nullptr;
        c->scale_n = c->keep_scale ? P.ntot : 0;
    }
    if (refine) {
        R.thresh2 = c->refine_T * c->refine_T;
        R.rcount = c->rcount.p;
        R.rlist = c->rlist.p;
        CUDA_TRY(cudaMemsetAsync(c->rcount.p, 0, sizeof(int) * P.nsets, st));
    }
    c->refine_nsets = refine ? P.nsets : 0;
    CUDA_TRY(launch_merge(c->sets.p, c->tile_set.p, c->tile_slots.p, P.ntiles, P.itile, c->ilist.p,
                          D, c->partials.p, out, refine ? nullptr : c->wtile.p, R, st));
    if (refine) TRY(run_refine(c, nkernel, D, out));
    if (W && refine)
        CUDA_TRY(launch_wtile_out(c->sets.p, c->tile_set.p, P.ntiles, P.itile, c->ilist.p, D,
                                  out.pot, c->wtile.p, st));
    if (W) CUDA_TRY(launch_wsum(c->sets.p, P.nsets, c->wtile.p, W, st));
    return SPHGRAV_OK;
}

static int read_device_error(sphgrav_ctx *c)
{
    int e = 0;
    CUDA_TRY(cudaMemcpy(&e, c->err.p, sizeof(int), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemset(c->err.p, 0, sizeof(int)));
    if (e & DEVERR_INPUT)
        return set_err(SPHGRAV_ERR_INVALID_INPUT,
                       "invalid particle data (mass <= 0, range2 == 0 or a non-finite value)");
    if (e & DEVERR_TIMEOUT) return set_err(SPHGRAV_ERR_DEVICE_TIMEOUT, "device wait timed out");
    if (e & DEVERR_TREE)
        return set_err(SPHGRAV_ERR_TOO_LARGE, "tree walk: traversal stack full (theta too small for N?)");
    if (e & DEVERR_TREE_CAP)
        return set_err(SPHGRAV_ERR_TOO_LARGE,
                       "captured tree call: the tree outgrew the node array or the heavy-group "
                       "list sized by the eager call before the capture; capture again");
    return SPHGRAV_OK;
}

// Host-side check of the inputs, the reference's asserts
// (grav_force_direct.cu:601-602) as a status.
static bool particle_ok(int i, const double *const a[5])
{
    const double m = a[3][i], r2 = a[4][i];
    return m > 0.0 && std::isfinite(m) && r2 != 0.0 && std::isfinite(r2) && std::isfinite(a[0][i]) &&
           std::isfinite(a[1][i]) && std::isfinite(a[2][i]);
}

static int report_bad_particle(int i, const double *const a[5])
{
    const double m = a[3][i], r2 = a[4][i];
    if (!(m > 0.0) || !std::isfinite(m))
        return set_err(SPHGRAV_ERR_INVALID_INPUT, "mass[%d] = %g must be > 0", i, m);
    if (r2 == 0.0 || !std::isfinite(r2))
        return set_err(SPHGRAV_ERR_INVALID_INPUT, "range2[%d] = %g must be non-zero", i, r2);
    return set_err(SPHGRAV_ERR_INVALID_INPUT, "position of particle %d is not finite", i);
}

// Host passes over the caller's (pageable) arrays -- copies into and out of
// the pinned staging buffers, input validation -- run on up to 8 threads
// once they are a few MB: a single thread moves ~5-10 GB/s, which at
// N = 1M made the staging a few percent of a host-array call.
static int host_threads(size_t bytes)
{
    if (bytes < ((size_t)4 << 20)) return 1;
    const unsigned hc = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(hc ? hc : 1u, 8u));
}

// f(i0, i1, t) over nt contiguous ranges of [0, n); ranges that get no
// thread (thread creation failed) run on the calling thread.
template <class F>
static void parallel_ranges(int n, int nt, const F &f)
{
    auto lo = [&](int t) { return (int)((long long)n * t / nt); };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; t++) {
        try {
            th.emplace_back(f, lo(t), lo(t + 1), t);
        } catch (...) {
            break;
        }
    }
    for (int t = (int)th.size() + 1; t < nt; t++) f(lo(t), lo(t + 1), t);
    f(0, lo(1), 0);
    for (auto &x : th) x.join();
}

static int check_host_inputs(int n, const double *x, const double *y, const double *z,
                             const double *m, const double *r2)
{
    const double *a[5] = {x, y, z, m, r2};
    const int nt = host_threads(5 * sizeof(double) * (size_t)n);
    std::vector<int> first(nt, n);
    parallel_ranges(n, nt, [&](int i0, int i1, int t) {
        for (int i = i0; i < i1; i++)
            if (!particle_ok(i, a)) { first[t] = i; break; }
    });
    const int bad = *std::min_element(first.begin(), first.end());
    return bad < n ? report_bad_particle(bad, a) : SPHGRAV_OK;
}

// Copy count arrays of n doubles (src[q] + off) to dst[q] + doff, in parallel
// slices of the index range.
static void copy_arrays(int count, int n, double *const *dst, size_t doff, const double *const *src,
                        size_t soff)
{
    parallel_ranges(n, host_threads(count * sizeof(double) * (size_t)n), [&](int i0, int i1, int) {
        for (int q = 0; q < count; q++)
            memcpy(dst[q] + doff + i0, src[q] + soff + i0, sizeof(double) * (size_t)(i1 - i0));
    });
}

// Context-owned input (5 arrays) and output (4 arrays) buffers of io_cap
// elements each, for the host-buffer entry points and the tuner.
static int ensure_io(sphgrav_ctx *c, int n)
{
    if ((size_t)n > c->io_cap || !c->in.p || !c->out.p) {
        const size_t want = std::max<size_t>(std::max(n, 1), c->io_cap);
        TRY(ensure(c, c->in, 5 * want, "inputs"));
        TRY(ensure(c, c->out, 4 * want, "outputs"));
        c->io_cap = want;
    }
    return SPHGRAV_OK;
}

// Copy host inputs (length n) to the context's device input buffer.
static int upload_inputs(sphgrav_ctx *c, int n, const double *x, const double *y, const double *z,
                         const double *m, const double *r2, InputsDev &in)
{
    TRY(ensure_io(c, n));
    TRY(ensure_pinned(c, c->h_in, 5 * sizeof(double) * std::max(n, 1)));
    double *h = (double *)c->h_in.p;
    const double *src[5] = {x, y, z, m, r2};
    double *dst[5];
    for (int a = 0; a < 5; a++) dst[a] = h + (size_t)a * n;
    copy_arrays(5, n, dst, 0, src, 0);
    const size_t cap = c->io_cap;
    if (n > 0)  // the device buffer holds 5 arrays of io_cap: one strided copy
        CUDA_TRY(cudaMemcpy2DAsync(c->in.p, sizeof(double) * cap, h, sizeof(double) * n,
                                   sizeof(double) * n, 5, cudaMemcpyHostToDevice, c->stream));
    in.x = c->in.p;
    in.y = in.x + cap;
    in.z = in.y + cap;
    in.m = in.z + cap;
    in.r2 = in.m + cap;
    return SPHGRAV_OK;
}

static OutputsDev ctx_outputs(sphgrav_ctx *c)
{
    OutputsDev o;
    const size_t cap = c->io_cap;
    o.ax = c->out.p;
    o.ay = o.ax + cap;
    o.az = o.ay + cap;
    o.pot = o.az + cap;
    return o;
}

// ------------------------------------------------------------ public API
extern "C" {

const char *sphgrav_status_string(int s)
{
    switch (s) {
    case SPHGRAV_OK: return "ok";
    case SPHGRAV_ERR_INVALID_ARGUMENT: return "invalid argument";
    case SPHGRAV_ERR_INVALID_INPUT: return "invalid particle data";
    case SPHGRAV_ERR_CUDA: return "CUDA error";
    case SPHGRAV_ERR_NO_DEVICE: return "no CUDA device";
    case SPHGRAV_ERR_OUT_OF_MEMORY: return "out of device memory";
    case SPHGRAV_ERR_PROTOCOL: return "call protocol violated";
    case SPHGRAV_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
    case SPHGRAV_ERR_TOO_LARGE: return "size beyond a documented limit";
    case SPHGRAV_ERR_UNSUPPORTED: return "not built into this library";
    default: return "unknown status";
    }
}

const char *sphgrav_last_error_message(void) { return g_errmsg.c_str(); }
unsigned long long sphgrav_launch_count(void) { return g_launches; }

int sphgrav_variant_count(int precision)
{
    if (precision != SPHGRAV_FP64 && precision != SPHGRAV_F32SPLIT) return 0;
    return variant_count(precision);
}
const char *sphgrav_variant_name(int precision, int v)
{
    if (v < 0 || v >= sphgrav_variant_count(precision)) return "";
    return variant_info(precision, v).name;
}

int sphgrav_create(sphgrav_ctx **out, int device)
{
    if (!out) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx pointer is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return set_err(SPHGRAV_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= ndev)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "device %d out of range (%d devices)", device, ndev);
    CUDA_TRY(cudaSetDevice(device));
    sphgrav_ctx *c = new sphgrav_ctx();
    c->device = device;
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    int st = SPHGRAV_OK;
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev_start) != cudaSuccess || cudaEventCreate(&c->ev_done) != cudaSuccess) {
        st = set_err(SPHGRAV_ERR_CUDA, "stream/event creation failed: %s",
                     cudaGetErrorString(cudaGetLastError()));
    }
    c->stream = c->own_stream;
    if (st == SPHGRAV_OK) st = ensure(c, c->head, 1, "head");
    if (st == SPHGRAV_OK) st = ensure(c, c->err, 1, "err");
    if (st == SPHGRAV_OK) st = ensure(c, c->nsel, 1, "nsel");
    if (st == SPHGRAV_OK) st = ensure(c, c->kick_counter, 1, "kick counter");
    if (st == SPHGRAV_OK) st = ensure_pinned(c, c->h_err, sizeof(int));
    if (st == SPHGRAV_OK && (cudaMemset(c->err.p, 0, sizeof(int)) != cudaSuccess ||
                             cudaMemset(c->kick_counter.p, 0, sizeof(unsigned long long)) != cudaSuccess))
        st = set_err(SPHGRAV_ERR_CUDA, "memset failed");
    if (st != SPHGRAV_OK) {
        sphgrav_destroy(c);
        return st;
    }
    *out = c;
    return SPHGRAV_OK;
}

int sphgrav_destroy(sphgrav_ctx *c)
{
    if (!c) return SPHGRAV_OK;
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != c->device) cudaSetDevice(c->device);
    if (c->own_stream) cudaStreamSynchronize(c->own_stream);
    if (c->stream && c->stream != c->own_stream) cudaStreamSynchronize(c->stream);
    for (sphgrav_graph *G : c->graphs) G->ctx = nullptr;  // they refuse to launch from now on
    c->graphs.clear();
    c->in.release(); c->out.release(); c->keys_in.release(); c->keys_out.release();
    c->bbox.release(); c->vals_in.release(); c->vals_out.release(); c->ilist.release();
    c->nsel.release(); c->tile_set.release(); c->tile_slots.release(); c->meta_set.release();
    c->head.release();
    c->err.release(); c->sort_temp.release(); c->sel_temp.release(); c->d64.release();
    c->orig.release(); c->flag.release(); c->f32.release(); c->sets.release();
    c->imeta.release(); c->jmeta.release(); c->items.release(); c->partials.release();
    c->wtile.release(); c->wdev.release(); c->kick_counter.release(); c->probe_sink.release();
    c->range2.release();
    c->gpart.release(); c->rcount.release(); c->rlist.release(); c->rnitems.release();
    c->rhead.release(); c->rsets.release(); c->ritems.release(); c->rpart.release();
    c->rnlight.release(); c->rlitems.release(); c->rlpart.release();
    c->scale.release(); c->phases.release();
    c->tnodes.release(); c->tgeom.release(); c->tmp.release(); c->tcnt.release(); c->tkeys.release();
    c->toff.release(); c->tstack.release(); c->tscan.release(); c->tres.release();
    c->twsum.release(); c->tgcount.release(); c->tgflag.release(); c->tglist.release();
    c->tgorder.release(); c->tlv.release();
    c->theavy.release(); c->theavy_part.release(); c->tacc.release();
    c->h_in.release(); c->h_out.release(); c->h_err.release();
    for (auto &e : c->prof_events) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    if (c->ev_start) cudaEventDestroy(c->ev_start);
    if (c->ev_done) cudaEventDestroy(c->ev_done);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return SPHGRAV_OK;
}

int sphgrav_set_stream(sphgrav_ctx *c, void *stream)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (c->capturing) return set_err(SPHGRAV_ERR_PROTOCOL, "cannot change stream during capture");
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return SPHGRAV_OK;
}

int sphgrav_sync(sphgrav_ctx *c)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    TRY(use_device(c));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return read_device_error(c);
}

int sphgrav_forces_device(sphgrav_ctx *c, int n, int i_begin, int ni, const double *x,
                          const double *y, const double *z, const double *mass,
                          const double *range2, int nkernel, int precision, double *ax,
                          double *ay, double *az, double *pot, double *W)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (n < 0 || i_begin < 0 || ni < 0 || i_begin + (long long)ni > n)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "bad sizes n=%d i_begin=%d ni=%d", n, i_begin, ni);
    if (n > 0 && (!x || !y || !z || !mass || !range2 || !ax || !ay || !az || !pot))
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "NULL data pointer");
    TRY(use_device(c));
    std::vector<int> offs = {0, n};
    const bool full = (i_begin == 0 && ni == n);
    InputsDev in = {x, y, z, mass, range2};
    OutputsDev out = {ax, ay, az, pot};
    if (W && n == 0) CUDA_TRY(cudaMemsetAsync(W, 0, sizeof(double), c->stream));
    return run_device(c, offs, full, i_begin, ni, in, out, W, nkernel, precision);
}

int sphgrav_batch_forces_device(sphgrav_ctx *c, int nsets, const int *offsets, const double *x,
                                const double *y, const double *z, const double *mass,
                                const double *range2, int nkernel, int precision, double *ax,
                                double *ay, double *az, double *pot, double *W_per_set)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (nsets <= 0 || nsets > MAX_SETS || !offsets)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "nsets must be in [1, %d]", MAX_SETS);
    std::vector<int> offs(offsets, offsets + nsets + 1);
    if (offs[0] != 0) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "offsets[0] must be 0");
    for (int s = 0; s < nsets; s++)
        if (offs[s + 1] < offs[s]) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "offsets must not decrease");
    if (offs.back() > 0 && (!x || !y || !z || !mass || !range2 || !ax || !ay || !az || !pot))
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "NULL data pointer");
    TRY(use_device(c));
    InputsDev in = {x, y, z, mass, range2};
    OutputsDev out = {ax, ay, az, pot};
    return run_device(c, offs, true, 0, 0, in, out, W_per_set, nkernel, precision);
}

int sphgrav_batch_forces(sphgrav_ctx *c, int nsets, const int *offsets, const double *x,
                         const double *y, const double *z, const double *mass,
                         const double *range2, int nkernel, int precision, double *ax, double *ay,
                         double *az, double *pot, double *W_per_set)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (c->capturing) return set_err(SPHGRAV_ERR_PROTOCOL, "host-buffer calls cannot be captured");
    if (nsets <= 0 || nsets > MAX_SETS || !offsets)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "nsets must be in [1, %d]", MAX_SETS);
    const int n = offsets[nsets];
    if (offsets[0] != 0 || n < 0) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "bad offsets");
    for (int s = 0; s < nsets; s++)
        if (offsets[s + 1] < offsets[s]) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "offsets must not decrease");
    if (n > 0 && (!x || !y || !z || !mass || !range2 || !ax || !ay || !az || !pot))
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "NULL data pointer");
    TRY(use_device(c));
    TRY(check_host_inputs(n, x, y, z, mass, range2));
    InputsDev in;
    TRY(upload_inputs(c, n, x, y, z, mass, range2, in));
    OutputsDev out = ctx_outputs(c);
    std::vector<int> offs(offsets, offsets + nsets + 1);
    TRY(ensure(c, c->wdev, nsets, "W"));
    TRY(run_device(c, offs, true, 0, 0, in, out, c->wdev.p, nkernel, precision));
    TRY(ensure_pinned(c, c->h_out, sizeof(double) * (4 * (size_t)n + nsets)));
    double *h = (double *)c->h_out.p;
    if (n > 0)  // 4 output arrays of io_cap: one strided copy
        CUDA_TRY(cudaMemcpy2DAsync(h, sizeof(double) * n, c->out.p, sizeof(double) * c->io_cap,
                                   sizeof(double) * n, 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemcpyAsync(h + 4 * (size_t)n, c->wdev.p, sizeof(double) * nsets,
                             cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    TRY(read_device_error(c));
    double *dst[4] = {ax, ay, az, pot};
    const double *src[4] = {h, h + (size_t)n, h + 2 * (size_t)n, h + 3 * (size_t)n};
    copy_arrays(4, n, dst, 0, src, 0);
    if (W_per_set) memcpy(W_per_set, h + 4 * (size_t)n, sizeof(double) * nsets);
    return SPHGRAV_OK;
}

int sphgrav_firsthalf(sphgrav_ctx *c, int n, int i_begin, int ni, const double *x, const double *y,
                      const double *z, const double *mass, const double *range2, int nkernel,
                      int precision)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (c->capturing) return set_err(SPHGRAV_ERR_PROTOCOL, "host-buffer calls cannot be captured");
    if (c->pending)
        return set_err(SPHGRAV_ERR_PROTOCOL, "firsthalf called twice without lasthalf");
    if (n < 0 || i_begin < 0 || ni < 0 || i_begin + (long long)ni > n)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "bad sizes n=%d i_begin=%d ni=%d", n, i_begin, ni);
    if (n > 0 && (!x || !y || !z || !mass || !range2))
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "NULL data pointer");
    TRY(use_device(c));
    TRY(check_host_inputs(n, x, y, z, mass, range2));
    CUDA_TRY(cudaEventRecord(c->ev_start, c->stream));
    InputsDev in;
    TRY(upload_inputs(c, n, x, y, z, mass, range2, in));
    OutputsDev out = ctx_outputs(c);
    std::vector<int> offs = {0, n};
    const bool full = (i_begin == 0 && ni == n);
    TRY(run_device(c, offs, full, i_begin, ni, in, out, nullptr, nkernel, precision));
    TRY(ensure_pinned(c, c->h_out, sizeof(double) * 4 * (size_t)std::max(ni, 1)));
    double *h = (double *)c->h_out.p;
    if (ni > 0)  // the row slice of the 4 output arrays: one strided copy
        CUDA_TRY(cudaMemcpy2DAsync(h, sizeof(double) * ni, c->out.p + i_begin,
                                   sizeof(double) * c->io_cap, sizeof(double) * ni, 4,
                                   cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->h_err.p, c->err.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemsetAsync(c->err.p, 0, sizeof(int), c->stream));
    CUDA_TRY(cudaEventRecord(c->ev_done, c->stream));
    c->pending = true;
    c->pend_n = n;
    c->pend_i0 = i_begin;
    c->pend_ni = ni;
    return SPHGRAV_OK;
}

int sphgrav_lasthalf(sphgrav_ctx *c, double *ax, double *ay, double *az, double *pot)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (!c->pending) return set_err(SPHGRAV_ERR_PROTOCOL, "lasthalf called without firsthalf");
    c->pending = false;
    TRY(use_device(c));
    CUDA_TRY(cudaEventSynchronize(c->ev_done));
    const int e = *(int *)c->h_err.p;
    if (e & DEVERR_INPUT) return set_err(SPHGRAV_ERR_INVALID_INPUT, "invalid particle data");
    if (e & DEVERR_TIMEOUT) return set_err(SPHGRAV_ERR_DEVICE_TIMEOUT, "device wait timed out");
    if (e & DEVERR_TREE)
        return set_err(SPHGRAV_ERR_TOO_LARGE, "tree walk: traversal stack full (theta too small for N?)");
    if (e & DEVERR_TREE_CAP)
        return set_err(SPHGRAV_ERR_TOO_LARGE, "tree: node array or heavy-group list full");
    const int ni = c->pend_ni, i0 = c->pend_i0;
    if (ni > 0 && (!ax || !ay || !az || !pot))
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "NULL output pointer");
    const double *h = (const double *)c->h_out.p;
    double *dst[4] = {ax, ay, az, pot};
    const double *src[4] = {h, h + (size_t)ni, h + 2 * (size_t)ni, h + 3 * (size_t)ni};
    copy_arrays(4, ni, dst, (size_t)i0, src, 0);
    return SPHGRAV_OK;
}

int sphgrav_gravforce(sphgrav_ctx *c, int ntot, int ngrav_lower, int ngrav_upper, const double *x,
                      const double *y, const double *z, const double *am, const double *hp,
                      const double *u, int nkernel, int precision, double *gx, double *gy,
                      double *gz, double *grpot)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (ntot < 0 || ngrav_lower < 1 || ngrav_upper < ngrav_lower - 1 || ngrav_upper > ntot)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "bad row range [%d, %d] of %d", ngrav_lower,
                       ngrav_upper, ntot);
    if (ntot > 0 && (!hp || !u)) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "NULL hp or u");
    std::vector<double> range2(ntot);
    for (int i = 0; i < ntot; i++) {  // grav.f:15-18
        range2[i] = 4 * hp[i] * hp[i];
        if (u[i] == 0.0) range2[i] = -range2[i];
    }
    const int len = ngrav_upper - ngrav_lower + 1;  // grav.f:23
    TRY(sphgrav_firsthalf(c, ntot, ngrav_lower - 1, len, x, y, z, am, range2.data(), nkernel,
                          precision));
    return sphgrav_lasthalf(c, gx, gy, gz, grpot);
}

int sphgrav_gravforce_device(sphgrav_ctx *c, int ntot, int ngrav_lower, int ngrav_upper,
                             const double *x, const double *y, const double *z, const double *am,
                             const double *hp, const double *u, int nkernel, int precision,
                             double *gx, double *gy, double *gz, double *grpot)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (ntot < 0 || ngrav_lower < 1 || ngrav_upper < ngrav_lower - 1 || ngrav_upper > ntot)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "bad row range [%d, %d] of %d", ngrav_lower,
                       ngrav_upper, ntot);
    if (ntot > 0 && (!hp || !u)) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "NULL hp or u");
    TRY(use_device(c));
    TRY(ensure(c, c->range2, std::max(ntot, 1), "range2"));
    CUDA_TRY(launch_range2(ntot, hp, u, c->range2.p, c->stream));  // grav.f:15-18
    const int len = ngrav_upper - ngrav_lower + 1;                   // grav.f:23
    return sphgrav_forces_device(c, ntot, ngrav_lower - 1, len, x, y, z, am, c->range2.p, nkernel,
                                 precision, gx, gy, gz, grpot, nullptr);
}

// ------------------------------------------------------ sweeps & capture
int sphgrav_kick_positions_device(sphgrav_ctx *c, int n, double *x, double *y, double *z,
                                  double sigma, unsigned long long seed)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (n < 0 || (n > 0 && (!x || !y || !z)))
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "bad kick arguments");
    TRY(use_device(c));
    CUDA_TRY(launch_kick(n, x, y, z, sigma, seed, c->kick_counter.p, c->stream));
    return SPHGRAV_OK;
}

int sphgrav_kick_reset(sphgrav_ctx *c, unsigned long long v)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (c->capturing) return set_err(SPHGRAV_ERR_PROTOCOL, "kick_reset cannot be captured");
    TRY(use_device(c));
    CUDA_TRY(cudaMemcpyAsync(c->kick_counter.p, &v, sizeof(v), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return SPHGRAV_OK;
}

// Captures are thread-local: while this thread captures, destroying a graph
// (an unsafe call during a capture, which would invalidate it) is deferred
// until its last capture ends.  A garbage-collected graph handle from an
// earlier capture is the usual case.
static thread_local int t_captures = 0;
static thread_local std::vector<sphgrav_graph *> t_deferred_graphs;

static void destroy_graph_now(sphgrav_graph *G)
{
    if (G->exec) cudaGraphExecDestroy(G->exec);
    if (G->graph) cudaGraphDestroy(G->graph);
    delete G;
}

int sphgrav_capture_begin(sphgrav_ctx *c)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (c->capturing) return set_err(SPHGRAV_ERR_PROTOCOL, "capture already active");
    TRY(use_device(c));
    CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    c->capturing = true;
    ++t_captures;
    return SPHGRAV_OK;
}

int sphgrav_capture_end(sphgrav_ctx *c, sphgrav_graph **out)
{
    if (!c || !out) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!c->capturing) return set_err(SPHGRAV_ERR_PROTOCOL, "no capture active");
    c->capturing = false;
    TRY(use_device(c));
    cudaGraph_t g = nullptr;
    const cudaError_t ended = cudaStreamEndCapture(c->stream, &g);
    if (--t_captures == 0) {  // no capture left on this thread: release deferred graphs
        for (sphgrav_graph *D : t_deferred_graphs) destroy_graph_now(D);
        t_deferred_graphs.clear();
    }
    CUDA_TRY(ended);
    sphgrav_graph *G = new sphgrav_graph();
    G->graph = g;
    G->stream = c->stream;
    G->device = c->device;
    G->ctx = c;
    G->epoch = c->epoch;
    cudaError_t e = cudaGraphInstantiate(&G->exec, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        delete G;
        return set_err(SPHGRAV_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
    }
    c->graphs.insert(G);
    *out = G;
    return SPHGRAV_OK;
}

int sphgrav_graph_valid(const sphgrav_graph *G)
{
    return G && G->ctx && G->ctx->epoch == G->epoch ? 1 : 0;
}

int sphgrav_graph_launch(sphgrav_graph *G, int repeats)
{
    if (!G || repeats < 0) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "bad graph launch");
    if (!G->ctx) return set_err(SPHGRAV_ERR_PROTOCOL, "the graph's context was destroyed");
    if (G->ctx->epoch != G->epoch)
        return set_err(SPHGRAV_ERR_PROTOCOL,
                       "the context's work plan, buffers or settings changed after this graph was "
                       "captured (a call with other sizes, precision or variant, or a new FP64 "
                       "band, refine threshold, error-scale setting or theta); capture it again");
    for (int r = 0; r < repeats; r++) {
        CUDA_TRY(cudaGraphLaunch(G->exec, G->stream));
        ++g_launches;
    }
    return SPHGRAV_OK;
}

int sphgrav_graph_destroy(sphgrav_graph *G)
{
    if (!G) return SPHGRAV_OK;
    if (G->ctx) G->ctx->graphs.erase(G);
    G->ctx = nullptr;
    if (t_captures > 0) {
        t_deferred_graphs.push_back(G);
        return SPHGRAV_OK;
    }
    destroy_graph_now(G);
    return SPHGRAV_OK;
}

// ----------------------------------------------------------------- tuning
int sphgrav_force_variant(sphgrav_ctx *c, int precision, int variant)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (precision != SPHGRAV_FP64 && precision != SPHGRAV_F32SPLIT)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "unknown precision %d", precision);
    if (variant < -1 || variant >= variant_count(precision))
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "variant %d out of range", variant);
    c->forced_variant[precision] = variant;
    return SPHGRAV_OK;
}

int sphgrav_autotune(sphgrav_ctx *c, int nsets, const int *offsets, const double *x,
                     const double *y, const double *z, const double *mass, const double *range2,
                     int nkernel, int precision)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (c->capturing) return set_err(SPHGRAV_ERR_PROTOCOL, "cannot tune during capture");
    if (precision != SPHGRAV_FP64 && precision != SPHGRAV_F32SPLIT)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "unknown precision %d", precision);
    if (nsets <= 0 || !offsets) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "bad sets");
    TRY(use_device(c));
    const int n = offsets[nsets];
    TRY(ensure_io(c, n));
    OutputsDev out = ctx_outputs(c);
    InputsDev in = {x, y, z, mass, range2};
    std::vector<int> offs(offsets, offsets + nsets + 1);
    const int saved = c->forced_variant[precision];
    float best_ms = 1e30f;
    int best = -1;
    for (int v = 0; v < variant_count(precision); v++) {
        const VariantInfo &V = variant_info(precision, v);
        if (precision == SPHGRAV_F32SPLIT && V.newton) continue;  // same numerics as the defaults
        c->forced_variant[precision] = v;
        int st = run_device(c, offs, true, 0, 0, in, out, nullptr, nkernel, precision);
        if (st != SPHGRAV_OK) { c->forced_variant[precision] = saved; return st; }
        float ms_min = 1e30f;
        for (int r = 0; r < 2; r++) {
            CUDA_TRY(cudaEventRecord(c->ev_start, c->stream));
            st = run_device(c, offs, true, 0, 0, in, out, nullptr, nkernel, precision);
            if (st != SPHGRAV_OK) { c->forced_variant[precision] = saved; return st; }
            CUDA_TRY(cudaEventRecord(c->ev_done, c->stream));
            CUDA_TRY(cudaEventSynchronize(c->ev_done));
            float ms = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&ms, c->ev_start, c->ev_done));
            ms_min = std::min(ms_min, ms);
        }
        if (ms_min < best_ms) { best_ms = ms_min; best = v; }
    }
    c->forced_variant[precision] = saved;
    TRY(read_device_error(c));
    if (best >= 0) c->tuned[precision][bucket_of(offs, true, 0)] = variant_info(precision, best).name;
    return SPHGRAV_OK;
}

int sphgrav_tuning_save(sphgrav_ctx *c, const char *path)
{
    if (!c || !path) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "NULL argument");
    FILE *f = fopen(path, "w");
    if (!f) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "cannot open %s for writing", path);
    fprintf(f, "{\"format\": \"sphgrav_b200-tuning-1\", \"entries\": [");
    bool first = true;
    for (int p = 0; p < 2; p++)
        for (auto &kv : c->tuned[p]) {
            fprintf(f, "%s\n  {\"precision\": %d, \"bucket\": %d, \"variant\": \"%s\"}",
                    first ? "" : ",", p, kv.first, kv.second.c_str());
            first = false;
        }
    fprintf(f, "\n]}\n");
    fclose(f);
    return SPHGRAV_OK;
}

int sphgrav_tuning_load(sphgrav_ctx *c, const char *path)
{
    if (!c || !path) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "NULL argument");
    FILE *f = fopen(path, "r");
    if (!f) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "cannot open %s", path);
    std::string s;
    char buf[4096];
    size_t k;
    while ((k = fread(buf, 1, sizeof(buf), f)) > 0) s.append(buf, k);
    fclose(f);
    if (s.find("sphgrav_b200-tuning-1") == std::string::npos)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "%s is not a tuning file", path);
    size_t pos = 0;
    int loaded = 0;
    while ((pos = s.find("{\"precision\"", pos)) != std::string::npos) {
        int p = -1, b = 0;
        char name[128] = {0};
        if (sscanf(s.c_str() + pos, "{\"precision\": %d, \"bucket\": %d, \"variant\": \"%127[^\"]\"}",
                   &p, &b, name) == 3 &&
            (p == 0 || p == 1) && variant_by_name(p, name) >= 0) {
            c->tuned[p][b] = name;
            loaded++;
        }
        pos += 12;
    }
    (void)loaded;
    return SPHGRAV_OK;
}

int sphgrav_last_plan_info(sphgrav_ctx *c, int *nitems, int *nchunks_max, int *variant)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (nitems) *nitems = c->plan.nitems;
    if (nchunks_max) *nchunks_max = c->plan.nchunks_max;
    if (variant) *variant = c->plan.variant;
    return SPHGRAV_OK;
}

int sphgrav_plan_preview(int nsets, const int *offsets, int precision, int variant, int resident,
                         int *nitems, int *nslots, int *items, int cap)
{
    if (nsets <= 0 || nsets > MAX_SETS || !offsets || !nitems || !nslots || resident <= 0)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "plan_preview: bad arguments");
    if ((precision != SPHGRAV_FP64 && precision != SPHGRAV_F32SPLIT) || variant < 0 ||
        variant >= variant_count(precision))
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "plan_preview: unknown precision or variant");
    std::vector<int> offs(offsets, offsets + nsets + 1);
    if (offs[0] != 0) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "offsets[0] must be 0");
    for (int s = 0; s < nsets; s++)
        if (offs[s + 1] < offs[s]) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "offsets must not decrease");
    Plan P;
    TRY(build_plan(resident, offs, true, 0, 0, precision, variant, P));
    *nitems = P.nitems;
    *nslots = P.nslots;
    if (items) {
        const int m = std::min(cap, P.nitems);
        for (int k = 0; k < m; k++) {
            const WorkItem &w = P.items[k];
            int *o = items + 6 * (size_t)k;
            o[0] = w.set; o[1] = w.tile; o[2] = w.chunk; o[3] = w.slot; o[4] = w.jb; o[5] = w.je;
        }
    }
    return SPHGRAV_OK;
}

int sphgrav_set_fp64_band(sphgrav_ctx *c, double factor)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (!(factor >= 1.0 && factor <= 16.0))
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "fp64 band factor %g outside [1, 16]", factor);
    if (c->capturing) return set_err(SPHGRAV_ERR_PROTOCOL, "cannot change the FP64 band during capture");
    if (factor != c->fp64_band) ++c->epoch;  // captured graphs hold the old band
    c->fp64_band = factor;
    return SPHGRAV_OK;
}

int sphgrav_set_refine(sphgrav_ctx *c, double threshold)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (!(threshold >= 0.0 && threshold <= 1e6))
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "refine threshold %g outside [0, 1e6]", threshold);
    if (c->capturing) return set_err(SPHGRAV_ERR_PROTOCOL, "cannot change the refine test during capture");
    if (threshold != c->refine_T) ++c->epoch;  // captured graphs hold the old test
    c->refine_T = threshold;
    return SPHGRAV_OK;
}

int sphgrav_last_refine_rows(sphgrav_ctx *c, long long *rows)
{
    if (!c || !rows) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "NULL argument");
    TRY(use_device(c));
    *rows = 0;
    if (c->refine_nsets <= 0) return SPHGRAV_OK;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    std::vector<int> cnt(c->refine_nsets);
    CUDA_TRY(cudaMemcpy(cnt.data(), c->rcount.p, sizeof(int) * cnt.size(), cudaMemcpyDeviceToHost));
    long long t = 0;
    for (int v : cnt) t += v;
    *rows = t;
    return SPHGRAV_OK;
}

int sphgrav_keep_error_scale(sphgrav_ctx *c, int on)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (c->capturing) return set_err(SPHGRAV_ERR_PROTOCOL, "cannot change this during capture");
    if ((on != 0) != c->keep_scale) ++c->epoch;  // captured graphs write (or not) the scale
    c->keep_scale = on != 0;
    if (!c->keep_scale) c->scale_n = 0;
    return SPHGRAV_OK;
}

int sphgrav_error_scale(sphgrav_ctx *c, int n, double *G)
{
    if (!c || (n > 0 && !G)) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n != c->scale_n)
        return set_err(SPHGRAV_ERR_PROTOCOL,
                       "no error scale of %d rows kept (last split-FP32 call kept %d)", n, c->scale_n);
    TRY(use_device(c));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (n > 0) CUDA_TRY(cudaMemcpy(G, c->scale.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return SPHGRAV_OK;
}

int sphgrav_profile_enable(sphgrav_ctx *c, int on)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    c->profiling = on != 0;
    return SPHGRAV_OK;
}

int sphgrav_profile_read(sphgrav_ctx *c, double *kernel_ms, int *launches)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    TRY(use_device(c));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    double total = 0.0;
    for (size_t k = 0; k < c->prof_used; k++) {
        float ms = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&ms, c->prof_events[k].first, c->prof_events[k].second));
        total += ms;
    }
    if (kernel_ms) *kernel_ms = total;
    if (launches) *launches = (int)c->prof_used;
    c->prof_used = 0;
    return SPHGRAV_OK;
}

int sphgrav_phase_read(sphgrav_ctx *c, unsigned long long *counters, int n)
{
    if (!c || !counters || n < (int)PHASE_COUNTERS)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "need room for %d counters", (int)PHASE_COUNTERS);
    if (!phases_built())
        return set_err(SPHGRAV_ERR_UNSUPPORTED,
                       "phase accounting needs the library built with -DSG_PHASES "
                       "(python -m starsmasher_b200.build --phases)");
    TRY(use_device(c));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < (int)PHASE_COUNTERS; i++) counters[i] = 0ull;
    if (c->phases.p) {
        CUDA_TRY(cudaMemcpy(counters, c->phases.p, sizeof(unsigned long long) * PHASE_COUNTERS,
                            cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemset(c->phases.p, 0, sizeof(unsigned long long) * PHASE_COUNTERS));
    }
    return SPHGRAV_OK;
}

int sphgrav_fp32_peak_probe(sphgrav_ctx *c, int iters, double *tflops)
{
    if (!c || !tflops || iters <= 0) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "bad probe arguments");
    TRY(use_device(c));
    const int blocks = c->sm_count * 8;
    TRY(ensure(c, c->probe_sink, blocks, "probe"));
    CUDA_TRY(launch_fp32_probe(std::min(iters, 1000), blocks, c->probe_sink.p, c->stream));
    CUDA_TRY(cudaEventRecord(c->ev_start, c->stream));
    CUDA_TRY(launch_fp32_probe(iters, blocks, c->probe_sink.p, c->stream));
    CUDA_TRY(cudaEventRecord(c->ev_done, c->stream));
    CUDA_TRY(cudaEventSynchronize(c->ev_done));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, c->ev_start, c->ev_done));
    const double flops = (double)blocks * 256.0 * iters * 8 * 2 * 2;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return SPHGRAV_OK;
}

int sphgrav_selftest_wait_timeout(sphgrav_ctx *c, int polls)
{
    if (!c || polls <= 0 || polls > (1 << 16))
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "polls must be in [1, 65536]");
    if (c->capturing) return set_err(SPHGRAV_ERR_PROTOCOL, "the self-test cannot be captured");
    TRY(use_device(c));
    CUDA_TRY(launch_wait_selftest((uint32_t)polls, c->err.p, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return read_device_error(c);
}

int sphgrav_fp64_peak_probe(sphgrav_ctx *c, int iters, double *tflops)
{
    if (!c || !tflops || iters <= 0) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "bad probe arguments");
    TRY(use_device(c));
    const int blocks = c->sm_count * 8;
    TRY(ensure(c, c->probe_sink, blocks, "probe"));
    CUDA_TRY(launch_fp64_probe(std::min(iters, 1000), blocks, c->probe_sink.p, c->stream));
    CUDA_TRY(cudaEventRecord(c->ev_start, c->stream));
    CUDA_TRY(launch_fp64_probe(iters, blocks, c->probe_sink.p, c->stream));
    CUDA_TRY(cudaEventRecord(c->ev_done, c->stream));
    CUDA_TRY(cudaEventSynchronize(c->ev_done));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, c->ev_start, c->ev_done));
    const double flops = (double)blocks * 256.0 * iters * 8 * 2;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return SPHGRAV_OK;
}

// -------------------------------------------------- legacy Fortran ABI
static sphgrav_ctx *g_legacy = nullptr;
static int g_legacy_device = -1;
static int g_legacy_precision = -1;
static double g_legacy_theta = 0.3;

static void legacy_fail(const char *where, int st)
{
    fprintf(stderr, "sphgrav_b200: %s failed: %s: %s\n", where, sphgrav_status_string(st),
            sphgrav_last_error_message());
    abort();
}

static int legacy_precision()
{
    if (g_legacy_precision < 0) {
        const char *e = getenv("SPHGRAV_PRECISION");
        g_legacy_precision = (e && (!strcmp(e, "fp64") || !strcmp(e, "FP64"))) ? SPHGRAV_FP64
                             : (e && (!strcmp(e, "tree") || !strcmp(e, "TREE"))) ? SPHGRAV_TREE
                                                                                 : SPHGRAV_F32SPLIT;
    }
    return g_legacy_precision;
}

static sphgrav_ctx *legacy_ctx()
{
    if (!g_legacy) {
        int dev = g_legacy_device;
        if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) dev = 0;
        int st = sphgrav_create(&g_legacy, dev);
        if (st != SPHGRAV_OK) legacy_fail("context creation", st);
        st = sphgrav_set_theta(g_legacy, g_legacy_theta);
        if (st != SPHGRAV_OK) legacy_fail("gpu_init_dev_ theta", st);
    }
    return g_legacy;
}

int sphgrav_set_theta(sphgrav_ctx *c, double theta)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (!(theta >= 0.0 && theta <= 2.0))
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "theta must be in [0, 2] (got %g)", theta);
    if (c->capturing) return set_err(SPHGRAV_ERR_PROTOCOL, "cannot change theta during capture");
    if (theta != c->theta) ++c->epoch;  // captured tree graphs hold the old angle
    c->theta = theta;
    return SPHGRAV_OK;
}

int sphgrav_tree_stats(sphgrav_ctx *c, int *groups, int *heavy)
{
    if (!c) return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (groups) *groups = c->tree_groups_last;
    if (heavy) *heavy = c->tree_heavy_last;
    return SPHGRAV_OK;
}

int sphgrav_legacy_set_precision(int precision)
{
    if (precision != SPHGRAV_FP64 && precision != SPHGRAV_F32SPLIT && precision != SPHGRAV_TREE)
        return set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "unknown precision %d", precision);
    g_legacy_precision = precision;
    return SPHGRAV_OK;
}

void gpu_init_dev_(int *myrank, double *theta)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
        legacy_fail("gpu_init_dev_", set_err(SPHGRAV_ERR_NO_DEVICE, "no CUDA device"));
    const int dev = myrank ? *myrank : 0;
    if (dev < 0 || dev >= ndev)
        legacy_fail("gpu_init_dev_", set_err(SPHGRAV_ERR_INVALID_ARGUMENT, "device %d of %d", dev, ndev));
    if (g_legacy && g_legacy->device != dev) {
        sphgrav_destroy(g_legacy);
        g_legacy = nullptr;
    }
    g_legacy_device = dev;
    if (cudaSetDevice(dev) != cudaSuccess)
        legacy_fail("gpu_init_dev_", set_err(SPHGRAV_ERR_CUDA, "cudaSetDevice(%d) failed", dev));
    // the opening angle of the tree mode (the direct modes do not use it)
    if (theta) g_legacy_theta = *theta;
    if (g_legacy) sphgrav_set_theta(g_legacy, g_legacy_theta);
}

void firsthalf_grav_forces_(int *n, int *n_lower, int *my_length, double *px, double *py,
                            double *pz, double *mass, double *range2, int *q, int *nkernel)
{
    (void)q;  // threads per particle: chosen by the library's tuning instead
    sphgrav_ctx *c = legacy_ctx();
    int st = sphgrav_firsthalf(c, *n, *n_lower - 1, *my_length, px, py, pz, mass, range2,
                               *nkernel, legacy_precision());
    if (st != SPHGRAV_OK) legacy_fail("firsthalf_grav_forces_", st);
}

void lasthalf_grav_forces_(int *n, double *ax, double *ay, double *az, double *pot, int *myrank)
{
    (void)n;
    (void)myrank;  // never read: the Fortran callers pass five arguments
    sphgrav_ctx *c = legacy_ctx();
    int st = sphgrav_lasthalf(c, ax, ay, az, pot);
    if (st != SPHGRAV_OK) legacy_fail("lasthalf_grav_forces_", st);
    if (getenv("SPHGRAV_VERBOSE")) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev_start, c->ev_done);
        fprintf(stderr, " >>> SPHgrav_lib took %g sec\n", ms * 1e-3);
    }
}

}  // extern "C"
