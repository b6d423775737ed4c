// sg_tree.cu -- Barnes-Hut octree gravity for sm_100a: the approximate
// alternative that the reference ships as a drop-in library with the same
// C-ABI (misc/SPHgravtree_lib: grav_force_tree.cu over libSequoia), written
// here from its semantics:
//   * an octree over the Hilbert-sorted particles (an octree cell is a
//     contiguous key range); a node splits while it holds more than
//     TREE_LEAF particles (the reference: 64);
//   * every node carries its mass, centre of mass and second moment about
//     it (monopole + quadrupole, as libSequoia's body_node), built bottom-up
//     in FP64; the walk uses the traceless quadrupole 3S - tr(S)I;
//   * particles are walked in groups, one warp each: the children of every
//     node with more than 32 particles, consecutive small siblings merged up
//     to 32 (a leaf that cannot split is cut into chunks of 32), the groups
//     with the largest H first; a node is opened when the gap between the
//     group's and the node's bounding boxes is at most l / theta, l the
//     node's edge length (libSequoia's minimum-distance criterion,
//     compute_properties.cu:339, dev_shared_traverse_functions.cu:311-337);
//     theta comes from gpu_init_dev_ (main.f:269-270 passes 0.3).  It is
//     also opened when the gap is at most max(H) of the node's or the
//     group's particles, so every pair closer than the softening length is
//     evaluated particle by particle with the softened kernel (the reference
//     leaves that test out, INDSOFT); with theta -> 0 the walk is therefore
//     the direct sum;
//   * accepted nodes interact through the quadrupole expansion in FP32;
//     particles of opened leaves that lie farther than every H from the
//     group's box are Newtonian FP32 pairs without a per-pair test, the
//     others are tested pair by pair: FP32 when Newtonian, FP64 with the
//     CPU-path formulas (pair_f64_fast) for r < max(H_i, H_j) and r = 0;
//   * a group with more than TREE_BUDGET tested particles (a dense region
//     inside a softening sphere, e.g. a point-mass core with a large H)
//     leaves the walk and gets the direct FP64 sum over all particles
//     instead, spread over many CTAs (k_tree_heavy).
// Construction is level by level with prefix sums.  Atomics only order the
// group list and hand groups to warps; every sum has a fixed order, so the
// results are bit-for-bit reproducible.
#include "sg_launch.h"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>

namespace sg {

// ---------------------------------------------------------------- build
__device__ __forceinline__ int lower_bound_key(const unsigned long long *keys, int lo, int hi,
                                               unsigned long long v)
{
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (keys[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Children of node i of level `level` (keys of its particles share their
// set index and top 3*level spatial key bits): the eight 3-bit digits of
// level + 1 split its sorted range; b[0..8] are the digit boundaries.
// `levels` = the keys' bits per axis (digits per set).
__device__ __forceinline__ void child_bounds(const TreeNode &T, int level, int levels,
                                             const unsigned long long *keys, int b[9])
{
    const int sh = 3 * (levels - 1 - level);  // digit of level + 1
    const unsigned long long base = (keys[T.start] >> (sh + 3)) << (sh + 3);
    b[0] = T.start;
    b[8] = T.end;
    for (int d = 1; d < 8; d++)
        b[d] = lower_bound_key(keys, b[d - 1], T.end, base | ((unsigned long long)d << sh));
}

// Level bounds live on the device (lv[L] = first node of level L, lv[L + 1]
// its end; lv[TREE_LV_OVERFLOW] set when the node array is too small), so the
// host issues every level without waiting.  Level L has at most `bound`
// nodes (min(roots 8^L, n)); counts are written for the whole bound, zero past
// the level's end, so that one fixed-size scan gives the child offsets.
__global__ void k_tree_count(int level, int levels, int bound, const int *lv,
                             const TreeNode *nodes, const unsigned long long *keys, int *cnt)
{
    const int l0 = lv[level], l1 = lv[level + 1];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < bound; j += gridDim.x * blockDim.x) {
        const int i = l0 + j;
        int c = 0;
        if (i < l1) {
            const TreeNode T = nodes[i];
            if (T.end - T.start > TREE_LEAF && level < levels) {
                int b[9];
                child_bounds(T, level, levels, keys, b);
                for (int d = 0; d < 8; d++) c += b[d + 1] > b[d] ? 1 : 0;
            }
        }
        cnt[j] = c;
    }
}

// One thread: the end of level + 1 from the scan; past the capacity the
// overflow flag is set and the tree stops at this level.
__global__ void k_tree_next(int level, int cap, int *lv, const int *cnt, const int *off)
{
    const int count = lv[level + 1] - lv[level];
    const long long total = count > 0 ? (long long)off[count - 1] + cnt[count - 1] : 0;
    if (lv[level + 1] + total > cap) {
        lv[TREE_LV_OVERFLOW] = 1;
        lv[level + 2] = lv[level + 1];
    } else {
        lv[level + 2] = lv[level + 1] + (int)total;
    }
}

__device__ void emit_children(int i, int l0, int level, int levels, int next_base,
                              TreeNode *nodes, const unsigned long long *keys, const int *cnt,
                              const int *off, unsigned char *gflag)
{
    const int c = cnt[i - l0];
    if (c == 0) return;
    TreeNode T = nodes[i];
    int b[9];
    child_bounds(T, level, levels, keys, b);
    int k = next_base + off[i - l0];
    T.child = k;
    T.nchild = c;
    nodes[i] = T;
    // Children of a node too big to be a group become groups, consecutive
    // small siblings merged (curve order) while they total <= TREE_GROUP:
    // gflag of a run's first child = the run's length in nodes.
    const bool big = T.end - T.start > TREE_GROUP;
    int run = -1, run_len = 0, run_n = 0;
    for (int d = 0; d < 8; d++) {
        if (b[d + 1] > b[d]) {
            TreeNode C;
            C.start = b[d];
            C.end = b[d + 1];
            C.child = 0;
            C.nchild = 0;
            const int cn = C.end - C.start;
            gflag[k] = 0;
            if (big && cn <= TREE_GROUP) {
                if (run >= 0 && run_n + cn <= TREE_GROUP) {
                    run_len++;
                    run_n += cn;
                } else {
                    if (run >= 0) gflag[run] = (unsigned char)run_len;
                    run = k;
                    run_len = 1;
                    run_n = cn;
                }
            } else if (run >= 0) {
                gflag[run] = (unsigned char)run_len;
                run = -1;
            }
            nodes[k++] = C;
        }
    }
    if (run >= 0) gflag[run] = (unsigned char)run_len;
}

__global__ void k_tree_emit(int level, int levels, const int *lv, TreeNode *nodes,
                            const unsigned long long *keys, const int *cnt, const int *off,
                            unsigned char *gflag)
{
    const int l0 = lv[level], l1 = lv[level + 1];
    if (lv[level + 2] == l1) return;  // no children (or no room: overflow is flagged)
    for (int i = l0 + blockIdx.x * blockDim.x + threadIdx.x; i < l1;
         i += gridDim.x * blockDim.x)
        emit_children(i, l0, level, levels, l1, nodes, keys, cnt, off, gflag);
}

// Walking groups: runs of consecutive sibling nodes that together hold at
// most TREE_GROUP particles (each a maximal such node or merged with its
// neighbours), and TREE_GROUP-particle chunks of the (coincident-particle)
// leaves that hold more; each particle lies in exactly one.  Atomic order:
// results do not depend on which warp walks which group.
__global__ void k_tree_groups(DevCount nnc, const TreeNode *nodes, const unsigned char *gflag,
                              int2 *glist, int *count)
{
    const int nn = nnc.get();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const TreeNode T = nodes[i];
        if (gflag[i]) {
            glist[atomicAdd(count, 1)] = make_int2(T.start, nodes[i + gflag[i] - 1].end);
        } else if (T.nchild == 0 && T.end - T.start > TREE_GROUP) {
            for (int b = T.start; b < T.end; b += TREE_GROUP)
                glist[atomicAdd(count, 1)] = make_int2(b, min(b + TREE_GROUP, T.end));
        }
    }
}

// Level 0: one root per set over the set's sorted slots (its pads excluded);
// a set of at most TREE_GROUP particles is one walking group.
__global__ void k_tree_roots(TreeNode *nodes, const SetDesc *sets, int nsets,
                             unsigned char *gflag, int *lv)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0) {
        lv[0] = 0;
        lv[1] = nsets;
        lv[TREE_LV_OVERFLOW] = 0;
    }
    if (s >= nsets) return;
    const SetDesc S = sets[s];
    gflag[s] = S.n > 0 && S.n <= TREE_GROUP;
    TreeNode R;
    R.start = S.poff;
    R.end = S.poff + S.n;
    R.child = 0;
    R.nchild = 0;
    nodes[s] = R;
}

// Root (set) of a sorted slot: the last root starting at or before it.
// Roots are in set order; an empty set's root never holds a group.
__device__ __forceinline__ int root_of(const TreeNode *nodes, int nroots, int slot)
{
    int lo = 0, hi = nroots - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (nodes[mid].start <= slot) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ------------------------------------------------------------ properties
// Leaves from their particles (one warp each, fixed-order butterfly sums),
// inner nodes from their children in child order, deepest level first
// (masses and centres of mass combined, second moments moved to the new
// centre by the parallel-axis rule), all in FP64: reproducible, and every
// level costs one short launch instead of a pass over its particles.
struct NodeAcc {
    double m, c[3];   // mass, centre of mass
    double lo[3], hi[3];
    double s[6];      // second moment about c: xx yy zz xy xz yz
    double h2max;
};

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__global__ void k_tree_leaf_acc(DevCount nnc, const TreeNode *nodes, SortedF64 D, NodeAcc *acc)
{
    const int nn = nnc.get();
    const int lane = threadIdx.x & 31;
    const int nw = gridDim.x * (blockDim.x >> 5);
    for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < nn; i += nw) {
        const TreeNode T = nodes[i];
        if (T.nchild > 0) continue;
        double m = 0.0, mx = 0.0, my = 0.0, mz = 0.0, h2 = 0.0;
        double nlo[3] = {-INFINITY, -INFINITY, -INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int s = T.start + lane; s < T.end; s += 32) {
            const double w = D.m[s], x = D.x[s], y = D.y[s], z = D.z[s];
            m += w;
            mx += w * x;
            my += w * y;
            mz += w * z;
            h2 = fmax(h2, D.h2[s]);
            nlo[0] = fmax(nlo[0], -x); nlo[1] = fmax(nlo[1], -y); nlo[2] = fmax(nlo[2], -z);
            hi[0] = fmax(hi[0], x);    hi[1] = fmax(hi[1], y);    hi[2] = fmax(hi[2], z);
        }
        m = warp_sum(m);
        mx = warp_sum(mx);
        my = warp_sum(my);
        mz = warp_sum(mz);
        h2 = warp_max(h2);
        for (int d = 0; d < 3; d++) {
            nlo[d] = warp_max(nlo[d]);
            hi[d] = warp_max(hi[d]);
        }
        // massless nodes sit at their box centre
        const double cx = m > 0.0 ? mx / m : 0.5 * (hi[0] - nlo[0]);
        const double cy = m > 0.0 ? my / m : 0.5 * (hi[1] - nlo[1]);
        const double cz = m > 0.0 ? mz / m : 0.5 * (hi[2] - nlo[2]);
        double q[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int s = T.start + lane; s < T.end; s += 32) {
            const double w = D.m[s], x = D.x[s] - cx, y = D.y[s] - cy, z = D.z[s] - cz;
            q[0] += w * x * x;
            q[1] += w * y * y;
            q[2] += w * z * z;
            q[3] += w * x * y;
            q[4] += w * x * z;
            q[5] += w * y * z;
        }
        for (int k = 0; k < 6; k++) q[k] = warp_sum(q[k]);
        if (lane == 0) {
            NodeAcc A;
            A.m = m;
            A.c[0] = cx; A.c[1] = cy; A.c[2] = cz;
            for (int d = 0; d < 3; d++) {
                A.lo[d] = -nlo[d];
                A.hi[d] = hi[d];
            }
            for (int k = 0; k < 6; k++) A.s[k] = q[k];
            A.h2max = h2;
            acc[i] = A;
        }
    }
}

__global__ void k_tree_inner_acc(int level, const int *lv, const TreeNode *nodes, NodeAcc *acc)
{
    const int l0 = lv[level], l1 = lv[level + 1];
    for (int i = l0 + blockIdx.x * blockDim.x + threadIdx.x; i < l1; i += gridDim.x * blockDim.x) {
        const TreeNode T = nodes[i];
        if (T.nchild == 0) continue;
        NodeAcc A;
        A.m = 0.0;
        double mc[3] = {0.0, 0.0, 0.0};
        A.h2max = 0.0;
        for (int d = 0; d < 3; d++) {
            A.lo[d] = INFINITY;
            A.hi[d] = -INFINITY;
        }
        for (int k = 0; k < T.nchild; k++) {
            const NodeAcc &C = acc[T.child + k];
            A.m += C.m;
            for (int d = 0; d < 3; d++) {
                mc[d] += C.m * C.c[d];
                A.lo[d] = fmin(A.lo[d], C.lo[d]);
                A.hi[d] = fmax(A.hi[d], C.hi[d]);
            }
            A.h2max = fmax(A.h2max, C.h2max);
        }
        for (int d = 0; d < 3; d++) A.c[d] = A.m > 0.0 ? mc[d] / A.m : 0.5 * (A.lo[d] + A.hi[d]);
        for (int q = 0; q < 6; q++) A.s[q] = 0.0;
        for (int k = 0; k < T.nchild; k++) {
            const NodeAcc &C = acc[T.child + k];
            const double dx = C.c[0] - A.c[0], dy = C.c[1] - A.c[1], dz = C.c[2] - A.c[2];
            A.s[0] += C.s[0] + C.m * dx * dx;
            A.s[1] += C.s[1] + C.m * dy * dy;
            A.s[2] += C.s[2] + C.m * dz * dz;
            A.s[3] += C.s[3] + C.m * dx * dy;
            A.s[4] += C.s[4] + C.m * dx * dz;
            A.s[5] += C.s[5] + C.m * dy * dz;
        }
        acc[i] = A;
    }
}

__global__ void k_tree_finalize(DevCount nnc, const NodeAcc *acc, double theta, NodeGeom *geom,
                                NodeMP *mp)
{
    const int nn = nnc.get();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const NodeAcc A = acc[i];
        NodeGeom G;
        G.cx = 0.5 * (A.lo[0] + A.hi[0]);
        G.cy = 0.5 * (A.lo[1] + A.hi[1]);
        G.cz = 0.5 * (A.lo[2] + A.hi[2]);
        // half sizes rounded up by 2^-20 of the coordinates' magnitude, so
        // that float rounding never lets a node look farther than it is
        const double c3[3] = {G.cx, G.cy, G.cz};
        float hs[3];
        double hmax = 0.0;
        for (int d = 0; d < 3; d++) {
            const double h = 0.5 * (A.hi[d] - A.lo[d]);
            hs[d] = (float)(h + 9.5367e-7 * (fabs(c3[d]) + h));
            hmax = fmax(hmax, h);
        }
        G.hx = hs[0];
        G.hy = hs[1];
        G.hz = hs[2];
        const double l = 2.0 * hmax;  // edge length
        G.op2 = l > 0.0 ? (theta > 0.0 ? (float)((l / theta) * (l / theta)) : INFINITY) : 0.f;
        G.h2max = (float)A.h2max * 1.000001f;
        G.pad_ = 0.f;
        geom[i] = G;
        NodeMP P;
        P.mx = A.c[0];
        P.my = A.c[1];
        P.mz = A.c[2];
        P.m = A.m;
        // traceless quadrupole Q = 3 S - tr(S) I
        const double tr = A.s[0] + A.s[1] + A.s[2];
        P.q[0] = (float)(3.0 * A.s[0] - tr);
        P.q[1] = (float)(3.0 * A.s[1] - tr);
        P.q[2] = (float)(3.0 * A.s[2] - tr);
        for (int q = 3; q < 6; q++) P.q[q] = (float)(3.0 * A.s[q]);
        P.pad_[0] = P.pad_[1] = 0.f;
        mp[i] = P;
    }
}

// -------------------------------------------------------------------- walk
constexpr int WALK_WARPS = 4;
constexpr int CELL_CAP = 64;  // < 32 pending + 32 appended per step
constexpr int PART_CAP = 64;

__global__ void __launch_bounds__(WALK_WARPS * 32) k_tree_walk(TreeWalkArgs a)
{
    // accepted nodes, group-relative: {x y z M} {Qxx Qyy Qzz Qxy} {Qxz Qyz - -}
    __shared__ float4 s_cell[WALK_WARPS][3][CELL_CAP];
    // particles farther than any H from the whole group: {x y z m}
    __shared__ float4 s_far[WALK_WARPS][PART_CAP];
    // the other particles: x y z m H^2 and their sorted slot
    __shared__ float s_part[WALK_WARPS][5][PART_CAP];
    __shared__ int s_pslot[WALK_WARPS][PART_CAP];
    __shared__ int s_q[WALK_WARPS][64];           // FP64 pairs: owner lane << 8 | entry
    __shared__ double s_qres[WALK_WARPS][4][32];  // their results
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    int *stack = a.stack + (size_t)(blockIdx.x * WALK_WARPS + w) * a.stack_cap;
    const SortedF64 D = a.D;
    float4(*cl)[CELL_CAP] = s_cell[w];
    float4 *fl = s_far[w];
    float(*pl)[PART_CAP] = s_part[w];
    int *ps = s_pslot[w];
    int *q = s_q[w];
    double(*qr)[32] = s_qres[w];
    const int ngroups = a.ngroups_dev ? *a.ngroups_dev : a.ngroups;

    for (;;) {
        int g = 0;
        if (lane == 0) g = atomicAdd(a.head, 1);
        g = __shfl_sync(FULL, g, 0);
        if (g >= ngroups) break;
        const int2 grp = a.groups[g];
        const int s0 = grp.x;
        const int s = s0 + lane;
        const bool act = s < grp.y;
        const int sr = act ? s : s0;  // inactive lanes mirror the group's first particle
        const double px = D.x[sr], py = D.y[sr], pz = D.z[sr];
        double lo[3] = {px, py, pz}, hi[3] = {px, py, pz};
        float gh2 = act ? (float)D.h2[s] : 0.f;
        for (int o = 16; o > 0; o >>= 1) {
            for (int d = 0; d < 3; d++) {
                lo[d] = fmin(lo[d], __shfl_xor_sync(FULL, lo[d], o));
                hi[d] = fmax(hi[d], __shfl_xor_sync(FULL, hi[d], o));
            }
            gh2 = fmaxf(gh2, __shfl_xor_sync(FULL, gh2, o));
        }
        gh2 *= 1.000001f;
        const double cx = 0.5 * (lo[0] + hi[0]), cy = 0.5 * (lo[1] + hi[1]),
                     cz = 0.5 * (lo[2] + hi[2]);
        const float ghx = (float)(0.5 * (hi[0] - lo[0]) * (1.0 + 1e-6) + 1e-30);
        const float ghy = (float)(0.5 * (hi[1] - lo[1]) * (1.0 + 1e-6) + 1e-30);
        const float ghz = (float)(0.5 * (hi[2] - lo[2]) * (1.0 + 1e-6) + 1e-30);
        const float xi = (float)(px - cx), yi = (float)(py - cy), zi = (float)(pz - cz);
        const float h2i = act ? (float)D.h2[s] : 0.f;
        // sums: each list flush in FP32, flushes and FP64 near pairs in FP64
        double fx = 0.0, fy = 0.0, fz = 0.0, fp = 0.0;
        int ncell = 0, nfar = 0, npart = 0, top = 1;
        int taken = 0;  // tested-list entries of this group so far
        bool overflow = false, heavy = false;
        // the walk starts at the root of the group's own set
        if (lane == 0) stack[0] = a.nroots > 1 ? root_of(a.nodes, a.nroots, s0) : 0;
        __syncwarp();

        // Every accepted node's box is disjoint from the group's (its gap is
        // above zero), so r > 0 for every lane, the idle ones included (they
        // mirror a particle of the group): no lane needs a guard.
        //   a = M d/r^3 - Q d/r^5 + 2.5 (d.Q.d) d/r^7,  phi = -M/r - 0.5 (d.Q.d)/r^5
        auto eval_cells = [&]() {
            float ax = 0.f, ay = 0.f, az = 0.f, sx = 0.f, sy = 0.f, sz = 0.f, pm = 0.f, pq = 0.f;
#pragma unroll 2  // measured: -15% walk time at theta 0.5, N = 1M (with the far loop's 4)
            for (int e = 0; e < ncell; e++) {
                const float4 A = cl[0][e], B = cl[1][e], C = cl[2][e];
                const float dx = A.x - xi, dy = A.y - yi, dz = A.z - zi;
                const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                const float ri = rsqrtf(r2);
                const float ri2 = ri * ri, ri3 = ri2 * ri, ri5 = ri3 * ri2;
                // Q d with B = (Qxx, Qyy, Qzz, Qxy), C = (Qxz, Qyz)
                const float qx = fmaf(C.x, dz, fmaf(B.w, dy, B.x * dx));
                const float qy = fmaf(C.y, dz, fmaf(B.y, dy, B.w * dx));
                const float qz = fmaf(B.z, dz, fmaf(C.y, dy, C.x * dx));
                const float dqd = fmaf(dz, qz, fmaf(dy, qy, dx * qx));
                const float c = fmaf(2.5f * dqd, ri2 * ri5, A.w * ri3);
                ax = fmaf(c, dx, ax);
                ay = fmaf(c, dy, ay);
                az = fmaf(c, dz, az);
                sx = fmaf(ri5, qx, sx);
                sy = fmaf(ri5, qy, sy);
                sz = fmaf(ri5, qz, sz);
                pm = fmaf(A.w, ri, pm);
                pq = fmaf(dqd, ri5, pq);
            }
            fx += (double)(ax - sx);
            fy += (double)(ay - sy);
            fz += (double)(az - sz);
            fp -= (double)(pm + 0.5f * pq);
            ncell = 0;
            __syncwarp();
        };
        // Far particles: Newtonian FP32 pairs, no per-pair test (r > 0 as above).
        auto eval_far = [&]() {
            float ax = 0.f, ay = 0.f, az = 0.f, pot = 0.f;
#pragma unroll 4
            for (int e = 0; e < nfar; e++) {
                const float4 P = fl[e];
                const float dx = P.x - xi, dy = P.y - yi, dz = P.z - zi;
                const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                const float ri = rsqrtf(r2);
                const float mr = P.w * ri;
                const float mr3 = mr * ri * ri;
                ax = fmaf(mr3, dx, ax);
                ay = fmaf(mr3, dy, ay);
                az = fmaf(mr3, dz, az);
                pot += mr;
            }
            fx += ax;
            fy += ay;
            fz += az;
            fp -= pot;
            nfar = 0;
            __syncwarp();
        };
        // FP64 pairs queued as (owner lane, list entry), evaluated one per lane
        // and summed by each owner in queue order
        auto eval_queue = [&](int cnt) {
            if (lane < cnt) {
                const int o = q[lane] >> 8, e = q[lane] & 255;
                const int si = s0 + o, j = ps[e];
                const PairOut r = pair_f64_fast(D, a.nkernel, si, j, D.x[j] - D.x[si],
                                                D.y[j] - D.y[si], D.z[j] - D.z[si], D.m[j],
                                                D.h2[si], D.h2[j]);
                qr[0][lane] = r.ax;
                qr[1][lane] = r.ay;
                qr[2][lane] = r.az;
                qr[3][lane] = r.pot;
            }
            __syncwarp();
            for (int t = 0; t < cnt; t++) {
                if ((q[t] >> 8) == lane) {
                    fx += qr[0][t];
                    fy += qr[1][t];
                    fz += qr[2][t];
                    fp += qr[3][t];
                }
            }
            __syncwarp();
        };
        // Particles that may lie within some H of some lane: tested per pair,
        // softened (or r = 0) pairs go to the FP64 queue.
        auto eval_parts = [&]() {
            float ax = 0.f, ay = 0.f, az = 0.f, pot = 0.f;
            int nq = 0;
            for (int e = 0; e < npart; e++) {
                const float dx = pl[0][e] - xi, dy = pl[1][e] - yi, dz = pl[2][e] - zi;
                const float r2 = dx * dx + dy * dy + dz * dz;
                const bool near = act && !(r2 >= fmaxf(h2i, pl[4][e]));
                if (act && !near) {
                    const float ri = rsqrtf(r2);
                    const float mr = pl[3][e] * ri;
                    const float mr3 = mr * ri * ri;
                    ax += mr3 * dx;
                    ay += mr3 * dy;
                    az += mr3 * dz;
                    pot -= mr;
                }
                const unsigned nm = __ballot_sync(FULL, near);
                if (near) q[nq + __popc(nm & below)] = (lane << 8) | e;
                nq += __popc(nm);
                __syncwarp();
                if (nq >= 32) {
                    eval_queue(32);
                    const int rest = nq - 32;  // < 32: move them to the front
                    const int v = lane < rest ? q[32 + lane] : 0;
                    __syncwarp();
                    if (lane < rest) q[lane] = v;
                    nq = rest;
                    __syncwarp();
                }
            }
            if (nq > 0) eval_queue(nq);
            fx += ax;
            fy += ay;
            fz += az;
            fp += pot;
            npart = 0;
            __syncwarp();
        };

        while (top > 0 && !heavy) {
            const int nb = min(top, 32);
            top -= nb;
            const int node = lane < nb ? stack[top + lane] : -1;
            __syncwarp();  // popped before the pushes below overwrite the slots
            bool cell = false, leaf_open = false;
            int nch = 0, ch0 = 0;
            if (node >= 0) {
                const NodeGeom G = a.geom[node];
                const float gx = fmaxf(0.f, (float)fabs(G.cx - cx) - (G.hx + ghx));
                const float gy = fmaxf(0.f, (float)fabs(G.cy - cy) - (G.hy + ghy));
                const float gz = fmaxf(0.f, (float)fabs(G.cz - cz) - (G.hz + ghz));
                const float d2 = gx * gx + gy * gy + gz * gz;
                const bool open = d2 <= G.op2 || d2 <= fmaxf(G.h2max, gh2);
                const TreeNode T = a.nodes[node];
                cell = !open;
                if (open) {
                    if (T.nchild > 0) {
                        nch = T.nchild;
                        ch0 = T.child;
                    } else {
                        leaf_open = true;
                    }
                }
            }
            // accepted nodes join the cell list (group-relative coordinates)
            const unsigned cm = __ballot_sync(FULL, cell);
            if (cell) {
                const int p = ncell + __popc(cm & below);
                const NodeMP P = a.mp[node];
                cl[0][p] = make_float4((float)(P.mx - cx), (float)(P.my - cy), (float)(P.mz - cz),
                                       (float)P.m);
                cl[1][p] = make_float4(P.q[0], P.q[1], P.q[2], P.q[3]);
                cl[2][p] = make_float4(P.q[4], P.q[5], 0.f, 0.f);
            }
            ncell += __popc(cm);
            __syncwarp();
            if (ncell >= 32) eval_cells();
            // opened inner nodes push their children
            int incl = nch;
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += v;
            }
            const int pushed = __shfl_sync(FULL, incl, 31);
            if (top + pushed > a.stack_cap) {
                overflow = true;
                break;
            }
            for (int c = 0; c < nch; c++) stack[top + incl - nch + c] = ch0 + c;
            top += pushed;
            __syncwarp();
            // opened leaves: their particles join the far list or the tested list
            unsigned lm = __ballot_sync(FULL, leaf_open);
            while (lm) {
                const int src = __ffs(lm) - 1;
                lm &= lm - 1;
                const int ln = __shfl_sync(FULL, node, src);
                const TreeNode T = a.nodes[ln];
                for (int b = T.start; b < T.end; b += 32) {
                    const int j = b + lane;
                    const bool has = j < T.end;
                    bool far = false;
                    float ex = 0.f, ey = 0.f, ez = 0.f, em = 0.f, eh2 = 0.f;
                    if (has) {
                        ex = (float)(D.x[j] - cx);
                        ey = (float)(D.y[j] - cy);
                        ez = (float)(D.z[j] - cz);
                        em = (float)D.m[j];
                        eh2 = (float)D.h2[j] * 1.000001f;
                        // a lower bound of the particle's distance to the group's
                        // box (1e-6 covers the FP32 roundings of ex and this sum)
                        const float bx = fmaxf(0.f, fabsf(ex) * (1.f - 1e-6f) - ghx);
                        const float by = fmaxf(0.f, fabsf(ey) * (1.f - 1e-6f) - ghy);
                        const float bz = fmaxf(0.f, fabsf(ez) * (1.f - 1e-6f) - ghz);
                        far = (bx * bx + by * by + bz * bz) * 0.9999f > fmaxf(eh2, gh2);
                    }
                    const unsigned fm = __ballot_sync(FULL, has && far);
                    const unsigned tm = __ballot_sync(FULL, has && !far);
                    if (has && far) fl[nfar + __popc(fm & below)] = make_float4(ex, ey, ez, em);
                    if (has && !far) {
                        const int p = npart + __popc(tm & below);
                        pl[0][p] = ex;
                        pl[1][p] = ey;
                        pl[2][p] = ez;
                        pl[3][p] = em;
                        pl[4][p] = eh2;
                        ps[p] = j;
                    }
                    nfar += __popc(fm);
                    npart += __popc(tm);
                    taken += __popc(tm);
                    __syncwarp();
                    if (taken > TREE_BUDGET) {
                        heavy = true;  // hand the group to the direct sum
                        break;
                    }
                    if (nfar >= 32) eval_far();
                    if (npart >= 32) eval_parts();
                }
                if (heavy) break;
            }
        }
        if (heavy) {
            if (lane == 0) a.heavy[atomicAdd(a.nheavy, 1)] = g;
            __syncwarp();
            continue;
        }
        if (ncell > 0) eval_cells();
        if (nfar > 0) eval_far();
        if (npart > 0) eval_parts();
        if (overflow && lane == 0) atomicOr(a.err, DEVERR_TREE);
        if (act) {
            a.out[s] = fx;
            a.out[a.n + s] = fy;
            a.out[2 * a.n + s] = fz;
            a.out[3 * a.n + s] = fp;
        }
    }
}

// Direct FP64 sum of a heavy group: block (h, c) sums the group's <= 32
// particles (lane = row) over source chunk c (the block's warps take
// interleaved sources); warps combine in order, chunks merge in order.
constexpr int HEAVY_WARPS = 8;
// Block b works on (heavy group, source chunk) pairs b, b + grid, ...: chunk c
// of the group's own set, one row per lane, sources split over the warps.
// The chunk count follows the number of heavy groups (read on the device).
__global__ void __launch_bounds__(HEAVY_WARPS * 32)
k_tree_heavy(const int *nheavy_p, int cap, const int *heavy, const int2 *groups,
             const TreeNode *nodes, int nroots, SortedF64 D, int max_n, int nkernel,
             double *partials, int *err)
{
    __shared__ double sh[HEAVY_WARPS][4][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nh_all = *nheavy_p;
    if (nh_all > cap && blockIdx.x == 0 && threadIdx.x == 0) atomicOr(err, DEVERR_TREE_CAP);
    const int nheavy = min(nh_all, cap);
    const int nchunks = tree_heavy_chunks(nheavy, max_n);
    for (int b = blockIdx.x; b < nheavy * nchunks; b += gridDim.x) {
        const int h = b / nchunks, c = b % nchunks;
        const int2 grp = groups[heavy[h]];
        const TreeNode R = nodes[nroots > 1 ? root_of(nodes, nroots, grp.x) : 0];
        const int ns = R.end - R.start;
        const int si = grp.x + lane;
        const bool act = si < grp.y;
        const int jb = R.start + (int)((long long)ns * c / nchunks);
        const int je = R.start + (int)((long long)ns * (c + 1) / nchunks);
        double sx = 0.0, sy = 0.0, sz = 0.0, sp = 0.0;
        if (act) {
            const double xi = D.x[si], yi = D.y[si], zi = D.z[si], h2i = D.h2[si];
            for (int j = jb + w; j < je; j += HEAVY_WARPS) {
                const PairOut o = pair_f64_fast(D, nkernel, si, j, D.x[j] - xi, D.y[j] - yi,
                                                D.z[j] - zi, D.m[j], h2i, D.h2[j]);
                sx += o.ax;
                sy += o.ay;
                sz += o.az;
                sp += o.pot;
            }
        }
        __syncthreads();  // the previous pair's reduction has read sh
        sh[w][0][lane] = sx;
        sh[w][1][lane] = sy;
        sh[w][2][lane] = sz;
        sh[w][3][lane] = sp;
        __syncthreads();
        if (w == 0) {
            for (int q = 0; q < 4; q++) {
                double v = sh[0][q][lane];
                for (int k = 1; k < HEAVY_WARPS; k++) v += sh[k][q][lane];
                partials[(((size_t)h * nchunks + c) * 4 + q) * 32 + lane] = v;
            }
        }
    }
}

// warp q of a block: quantity q of heavy group h, chunks in order
__global__ void k_tree_heavy_merge(const int *nheavy_p, int cap, const int *heavy,
                                   const int2 *groups, int max_n, const double *partials,
                                   int nslots, double *out)
{
    const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
    const int nheavy = min(*nheavy_p, cap);
    const int nchunks = tree_heavy_chunks(nheavy, max_n);
    for (int h = blockIdx.x; h < nheavy; h += gridDim.x) {
        const int2 grp = groups[heavy[h]];
        const int si = grp.x + lane;
        if (si >= grp.y) continue;
        double v = 0.0;
        for (int c = 0; c < nchunks; c++)
            v += partials[(((size_t)h * nchunks + c) * 4 + q) * 32 + lane];
        out[(size_t)q * nslots + si] = v;
    }
}

size_t tree_heavy_partials(int cap, int max_n)
{
    // nheavy * tree_heavy_chunks(nheavy, .) <= 4096 + nheavy for every nheavy <= cap
    (void)max_n;
    return ((size_t)4096 + (size_t)cap) * 4 * 32;
}

cudaError_t tree_heavy(int nheavy_host, const int *nheavy, int cap, const int *heavy,
                       const int2 *groups, const TreeNode *nodes, int nroots, const SortedF64 &D,
                       int nslots, int max_n, int nkernel, double *partials, double *out, int *err,
                       cudaStream_t st)
{
    // eager calls know the count: one block per (group, chunk); captured
    // calls size the grid for the most chunks any count can give
    const int blocks = nheavy_host > 0
                           ? std::min(nheavy_host, cap) * tree_heavy_chunks(std::min(nheavy_host, cap), max_n)
                           : 4096;
    k_tree_heavy<<<blocks, HEAVY_WARPS * 32, 0, st>>>(nheavy, cap, heavy, groups, nodes, nroots, D,
                                                     max_n, nkernel, partials, err);
    ++g_launches;
    const int mblocks = nheavy_host > 0 ? std::min(nheavy_host, cap) : 256;
    k_tree_heavy_merge<<<mblocks, 128, 0, st>>>(nheavy, cap, heavy, groups, max_n, partials, nslots,
                                               out);
    ++g_launches;
    return cudaGetLastError();
}

// Sorted-order results to the caller's rows [i_lo, i_lo + ni) (pad slots,
// orig < 0, are skipped).
__global__ void k_tree_scatter(int nslots, int i_lo, int ni, const double *res, const int *orig,
                               OutputsDev out)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nslots; s += gridDim.x * blockDim.x) {
        const int p = orig[s];
        if (p < i_lo || p >= i_lo + ni) continue;
        out.ax[p] = res[s];
        out.ay[p] = res[nslots + s];
        out.az[p] = res[2 * nslots + s];
        out.pot[p] = res[3 * nslots + s];
    }
}

// W = 1/2 sum m phi over each set's particles: one block per set, fixed order.
__global__ void k_tree_wsum(const SetDesc *sets, int nslots, const double *res, const double *m,
                            double *W)
{
    __shared__ double part[1024];
    const SetDesc S = sets[blockIdx.x];
    double w = 0.0;
    for (int k = threadIdx.x; k < S.n; k += blockDim.x)
        w += m[S.poff + k] * res[3 * (size_t)nslots + S.poff + k];
    part[threadIdx.x] = w;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) W[blockIdx.x] = 0.5 * part[0];
}

cudaError_t tree_wsum(const SetDesc *sets, int nsets, int nslots, const double *res,
                      const double *m, double *W, cudaStream_t st)
{
    if (nsets <= 0) return cudaSuccess;
    k_tree_wsum<<<nsets, 1024, 0, st>>>(sets, nslots, res, m, W);
    ++g_launches;
    return cudaGetLastError();
}

// Keys by sorted slot: set s's particles sit at slots [poff, poff + n) and
// at [off, off + n) of the sorted key array.
__global__ void k_tree_slot_keys(const SetDesc *sets, const unsigned long long *keys_sorted,
                                 unsigned long long *keys_slot)
{
    const SetDesc S = sets[blockIdx.y];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S.n; k += gridDim.x * blockDim.x)
        keys_slot[S.poff + k] = keys_sorted[S.off + k];
}

cudaError_t tree_slot_keys(const SetDesc *sets, int nsets, int max_n,
                           const unsigned long long *keys_sorted, unsigned long long *keys_slot,
                           cudaStream_t st)
{
    if (nsets <= 0 || max_n <= 0) return cudaSuccess;
    const dim3 grid(std::min((max_n + 255) / 256, 1024), nsets);
    k_tree_slot_keys<<<grid, 256, 0, st>>>(sets, keys_sorted, keys_slot);
    ++g_launches;
    return cudaGetLastError();
}

__global__ void k_tree_check_build(const int *lv, int *err)
{
    if (lv[TREE_LV_OVERFLOW]) atomicOr(err, DEVERR_TREE_CAP);
}

cudaError_t tree_check_build(const int *lv, int *err, cudaStream_t st)
{
    k_tree_check_build<<<1, 1, 0, st>>>(lv, err);
    ++g_launches;
    return cudaGetLastError();
}

// --------------------------------------------------------------- driver
size_t tree_scan_temp_bytes(int n)
{
    size_t b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b, (const int *)nullptr, (int *)nullptr, std::max(n, 1));
    return b;
}

cudaError_t tree_build_levels(const TreeBuildArgs &t, int level_begin, int level_end,
                              cudaStream_t st)
{
    if (level_begin == 0) {
        k_tree_roots<<<(t.nroots + 127) / 128, 128, 0, st>>>(t.nodes, t.sets, t.nroots, t.gflag, t.lv);
        ++g_launches;
    }
    for (int level = level_begin; level < level_end; level++) {
        // level has at most min(roots * 8^level, n) nodes
        const long long fan = level < 20 ? (1ll << (3 * level)) : (1ll << 60);
        const long long b = (long long)t.nroots * std::min(fan, (long long)t.n);
        const int bound = (int)std::max(1ll, std::min(b, (long long)std::max(t.n, 1)));
        const int blocks = std::min((bound + 255) / 256, 4096);
        k_tree_count<<<blocks, 256, 0, st>>>(level, t.levels, bound, t.lv, t.nodes, t.keys, t.cnt);
        ++g_launches;
        size_t tb = t.scan_temp_bytes;
        const cudaError_t e = cub::DeviceScan::ExclusiveSum(t.scan_temp, tb, t.cnt, t.off, bound, st);
        if (e != cudaSuccess) return e;
        ++g_launches;
        k_tree_next<<<1, 1, 0, st>>>(level, t.cap, t.lv, t.cnt, t.off);
        ++g_launches;
        k_tree_emit<<<blocks, 256, 0, st>>>(level, t.levels, t.lv, t.nodes, t.keys, t.cnt, t.off,
                                            t.gflag);
        ++g_launches;
    }
    return cudaGetLastError();
}

static int grid_for(DevCount c, int per_block, int cap_blocks)
{
    return std::max(1, std::min((std::max(c.host, 1) + per_block - 1) / per_block, cap_blocks));
}

cudaError_t tree_groups(DevCount nn, const TreeNode *nodes, const unsigned char *gflag,
                        int2 *glist, int *count, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    k_tree_groups<<<grid_for(nn, 256, 4096), 256, 0, st>>>(nn, nodes, gflag, glist, count);
    ++g_launches;
    return cudaGetLastError();
}

// Walking order: the largest H first.  Every particle within H of a group
// is tested pair by pair, so those groups walk longest; started first, they
// do not leave one warp running after the rest (results do not depend on the
// order: each group's sums are its own).  Entries past the group count (a
// device count bounded by ng.host) get key 0 and sort last.
__global__ void k_tree_group_keys(DevCount ngc, int bound, const int2 *glist, const double *h2,
                                  unsigned *keys)
{
    const int ng = ngc.get();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= bound) return;
    double m = 0.0;
    if (g < ng) {
        const int2 r = glist[g];
        for (int s = r.x; s < r.y; s++) m = fmax(m, h2[s]);
    }
    // non-negative floats order as their bits; a group always keys above
    // the unused entries, even if its H^2 rounds to a float 0
    keys[g] = g < ng ? max(__float_as_uint((float)m), 1u) : 0u;
}

size_t tree_order_temp_bytes(int ng)
{
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, (const unsigned *)nullptr,
                                              (unsigned *)nullptr, (const int2 *)nullptr,
                                              (int2 *)nullptr, std::max(ng, 1));
    return bytes;
}

cudaError_t tree_order_groups(DevCount ng, const int2 *glist, int2 *ordered, const double *h2,
                              unsigned *keys_in, unsigned *keys_out, void *temp, size_t temp_bytes,
                              cudaStream_t st)
{
    if (ng.host <= 0) return cudaSuccess;
    k_tree_group_keys<<<(ng.host + 255) / 256, 256, 0, st>>>(ng, ng.host, glist, h2, keys_in);
    ++g_launches;
    size_t tb = temp_bytes;
    const cudaError_t e = cub::DeviceRadixSort::SortPairsDescending(temp, tb, keys_in, keys_out,
                                                                    glist, ordered, ng.host, 0, 32,
                                                                    st);
    ++g_launches;
    return e != cudaSuccess ? e : cudaGetLastError();
}

size_t tree_acc_bytes(int nn) { return (size_t)nn * sizeof(NodeAcc); }

cudaError_t tree_props(DevCount nn, const TreeNode *nodes, const SortedF64 &D, double theta,
                       const int *lv, const int *level_start, int depth, int level_bound,
                       void *acc_buf, NodeGeom *geom, NodeMP *mp, cudaStream_t st)
{
    NodeAcc *acc = (NodeAcc *)acc_buf;
    k_tree_leaf_acc<<<grid_for(nn, 8, 148 * 16), 256, 0, st>>>(nn, nodes, D, acc);
    ++g_launches;
    for (int l = depth - 1; l >= 0; l--) {
        // a level's node count: exact when the host read the level table,
        // else bounded (grid-stride)
        const int cnt = level_start ? level_start[l + 1] - level_start[l] : level_bound;
        if (level_start && cnt <= 0) continue;
        k_tree_inner_acc<<<std::max(1, std::min((cnt + 127) / 128, 148 * 8)), 128, 0, st>>>(
            l, lv, nodes, acc);
        ++g_launches;
    }
    k_tree_finalize<<<grid_for(nn, 256, 148 * 16), 256, 0, st>>>(nn, acc, theta, geom, mp);
    ++g_launches;
    return cudaGetLastError();
}

int tree_walk_warps(int sm_count) { return sm_count * 8 * WALK_WARPS; }

cudaError_t tree_walk(const TreeWalkArgs &a, int sm_count, cudaStream_t st)
{
    k_tree_walk<<<sm_count * 8, WALK_WARPS * 32, 0, st>>>(a);
    ++g_launches;
    return cudaGetLastError();
}

cudaError_t tree_scatter(int nslots, int i_lo, int ni, const double *res, const int *orig,
                         const OutputsDev &out, cudaStream_t st)
{
    k_tree_scatter<<<std::max(1, std::min((nslots + 255) / 256, 4096)), 256, 0, st>>>(
        nslots, i_lo, ni, res, orig, out);
    ++g_launches;
    return cudaGetLastError();
}

}  // namespace sg
