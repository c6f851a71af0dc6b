// Pieces shared by the FP32 (CUDA-core) and BF16 (tcgen05) fused projection
// kernels: the workspace layout, the per-item segment table filled from the
// slot-bucketed segment list, the TMA staging of a slot's planes, and the
// bit-exact per-sample geometry.
#pragma once

#include <algorithm>

#include "atdf_common.cuh"

namespace atdf {

constexpr int kSegItem = 128;         // segments per work item
constexpr int kLineWin = 64;          // line-gradient window entries per line
constexpr int kSegTabArrays = 17;     // per-segment arrays of the per-item segment table
constexpr int kSegMapCap = 4096;      // samples of an item covered by the sample -> segment map
constexpr int kSegTabFloats = kSegTabArrays * (kSegItem + 4) + 16 + kSegMapCap / 4;  // + the item's box, the map

// ---------------------------------------------------------------------------
// workspace
// ---------------------------------------------------------------------------
struct Ws {
    int64_t* ray_seg_offset;
    int64_t* ray_sample_offset;
    int64_t* totals;
    int32_t* node;
    float* tmin;
    float* tmax;
    int32_t* nsamp;
    int32_t* ray;
    int32_t* first;
    float* seg_partial;
    int32_t* bucket;
    int32_t* slot_offset;  // [nslot + 2]
    int32_t* slot_cursor;  // [nslot + 1]: bucket cursors, then the queue's slot order
    int32_t* item_offset;  // [nslot + 2]
    int32_t* counters;     // [8]: the queues' positions (0, 1), the item queue's length (4)
    int2* item_queue;      // (slot, item of the slot) in the slot queue's order
    int64_t cap;
    int64_t nslot;
};

static int64_t seg_capacity(int64_t R, int max_depth)
{
    int64_t per = 3 * ((int64_t)1 << std::min(std::max(max_depth, 0), 20)) + 3;
    per = std::min<int64_t>(per, ATDF_MAX_HITS);
    return std::max<int64_t>(R * per, 1);
}

static size_t carve(char*& p, size_t bytes)
{
    size_t off = (size_t)p;
    p += (bytes + 255) & ~(size_t)255;
    return off;
}

// Lays the workspace out from base (nullptr: only the size).
static size_t ws_layout(int64_t R, int max_depth, int64_t nslot, char* base, Ws* w)
{
    const int64_t cap = seg_capacity(R, max_depth);
    char* p = base;
    Ws x;
    x.ray_seg_offset = (int64_t*)carve(p, (R + 1) * 8);
    x.ray_sample_offset = (int64_t*)carve(p, (R + 1) * 8);
    x.totals = (int64_t*)carve(p, 4 * 8);
    x.node = (int32_t*)carve(p, cap * 4);
    x.tmin = (float*)carve(p, cap * 4);
    x.tmax = (float*)carve(p, cap * 4);
    x.nsamp = (int32_t*)carve(p, cap * 4);
    x.ray = (int32_t*)carve(p, cap * 4);
    x.first = (int32_t*)carve(p, cap * 4);
    x.seg_partial = (float*)carve(p, cap * 4);
    x.bucket = (int32_t*)carve(p, cap * 4);
    x.slot_offset = (int32_t*)carve(p, (nslot + 2) * 4);
    x.slot_cursor = (int32_t*)carve(p, (nslot + 1) * 4);
    x.item_offset = (int32_t*)carve(p, (nslot + 2) * 4);
    x.counters = (int32_t*)carve(p, 8 * 4);
    x.item_queue = (int2*)carve(p, (nslot + 3 + cap / kSegItem) * 8);
    x.cap = cap;
    x.nslot = nslot;
    if (w) *w = x;
    return (size_t)(p - base);
}

static atdf_segments_t ws_segments(const Ws& w)
{
    atdf_segments_t s;
    s.ray_seg_offset = w.ray_seg_offset;
    s.ray_sample_offset = w.ray_sample_offset;
    s.node = w.node;
    s.tmin = w.tmin;
    s.tmax = w.tmax;
    s.nsamp = w.nsamp;
    s.ray = w.ray;
    s.first = w.first;
    s.capacity = w.cap;
    s.totals = w.totals;
    return s;
}

__device__ __forceinline__ int64_t seg_slot(const atdf_field_t& f, int64_t num_nodes, int32_t node)
{
    if (node < 0 || node >= num_nodes) return f.num_slots;
    const int64_t s = f.leaf_slot[node];
    return (s < 0 || s >= f.num_slots) ? f.num_slots : s;
}

// ---------------------------------------------------------------------------
// TMA bulk copies and a bounded mbarrier wait
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tma_bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Bounded wait (about a second of try_wait rounds); false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase)
{
    for (int i = 0; i < (1 << 22); ++i)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

struct FusedParams {
    atdf_tree_t tree;
    atdf_field_t field;
    atdf_mlp_t mlp;
    const float* origin;
    const float* dir;
    int64_t R;
    uint64_t seed;
    Ws ws;
    const float* grad_image;
    atdf_field_grad_t gfield;
    atdf_mlp_grad_t gmlp;
    int32_t* err;
    int plane_off[4];    // element offsets of the three planes in shared memory (+ total)
    int plane_pitch[3];  // texels per shared-memory row of each plane (>= plane_w)
    int gplane_off[4];   // float offsets of the unpadded FP32 plane-gradient copy (+ total)
    float roi_inv;     // 1 / (roi_max.x - roi_min.x) when a power of two, else 0
    // Caller-placed samples (null: the uniform per-node rule): t and weight
    // of every sample in canonical order, indexed by the ray's sample offset
    // plus the segment's first sample plus j.
    const float* xt;
    const float* xw;
    // Forward only (nullable): rho * w of each sample added into kBins equal
    // bins of its segment, [segment][kBins].
    float* bins;
};

constexpr int kBins = ATDF_PROPOSAL_BINS;

// Per-item segment table in shared memory. The segments of a plane slot's
// item share one leaf, whose box is kept once (box: min[3], size[3], inverse
// size[3] when a power of two else 0, then the node id).
struct SegTab {
    int* start;  // [kSegItem + 1]
    int* node;
    int* n;
    int* id;
    float* tmin;
    float* tmax;
    float* step;  // (tmax - tmin) / n
    float* acc;   // forward partial integral / backward dI of the ray
    int* first;     // global index of the segment's first sample (caller-placed samples)
    float* org[3];  // the segment's ray: origin and direction
    float* dir[3];
    unsigned* key_lo;  // the ray's jitter key (low and high 32 bits)
    unsigned* key_hi;
    float* box;
    unsigned char* map;  // segment of each sample (items of at most kSegMapCap samples)
};

__device__ __forceinline__ SegTab seg_tab(float* base)
{
    constexpr int S = kSegItem + 4;
    SegTab t;
    int* ib = reinterpret_cast<int*>(base);
    t.start = ib;
    t.node = ib + S;
    t.n = ib + 2 * S;
    t.id = ib + 3 * S;
    t.tmin = base + 4 * S;
    t.tmax = base + 5 * S;
    t.step = base + 6 * S;
    t.acc = base + 7 * S;
    t.first = ib + 8 * S;
    for (int k = 0; k < 3; ++k) {
        t.org[k] = base + (9 + k) * S;
        t.dir[k] = base + (12 + k) * S;
    }
    t.key_lo = reinterpret_cast<unsigned*>(base + 15 * S);
    t.key_hi = reinterpret_cast<unsigned*>(base + 16 * S);
    t.box = base + 17 * S;
    t.map = reinterpret_cast<unsigned char*>(t.box + 16);
    return t;
}

// Takes the next work item; fills the segment table; issues the plane TMA
// when the item starts a new slot. Returns the item's slot, or -1 when the
// queue is empty. Items of up to map_cap (<= kSegMapCap) samples get the
// sample -> segment byte map, larger ones a binary search.
// sample_state(permute = true) visits a work item's samples in the order
// k -> k * 104729 mod total (a permutation: the prime exceeds any item's
// sample count). Consecutive samples, which share a warp, then come from
// different rays and depths in the leaf and touch different texels, so their
// shared-memory atomics do not collide the way the samples along one ray
// would. The FP32 kernels and the 16-channel tensor-core backward use it; the
// tensor-core forwards and the 24-channel backward visit samples in order
// (gathers along a ray share texels; that backward rotates its atomics
// instead).
constexpr int kSamplePermPrime = 104729;

struct ItemInfo {
    int64_t slot;
    int nseg;
    int total;
    double inv_total;  // 1 / total (for the sample permutation)
    bool first;        // first item of its slot: the slot's planes were just requested
    bool last;         // last item of its slot
    int slot_items;    // work items of the slot
    bool use_map;      // total <= kSegMapCap: the table's map gives each sample's segment
};

// (k * kSamplePermPrime) mod total without a 64-bit integer division: the
// product is below 2^34 and exact in double, the quotient estimate from the
// reciprocal is off by at most one, and q * total and the remainder are exact.
__device__ __forceinline__ int perm_index(int k, int total, double inv_total)
{
    const double kp = (double)k * (double)kSamplePermPrime;
    const double q = floor(kp * inv_total);
    double r = kp - q * (double)total;
    if (r < 0.0)
        r += (double)total;
    else if (r >= (double)total)
        r -= (double)total;
    return (int)r;
}

// Work is handed out by leaf slot: a CTA takes the next slot with segments
// from the queue (counters[queue] counts slots) and then walks that slot's
// work items of up to kSegItem segments itself, so each slot's planes are
// staged once and its gradient copy is zeroed and written back once, by one
// CTA, with plain stores. s_ctl[4..6] hold the CTA's current slot and its
// next / end item (thread 0 only; init_item_queue sets them), s_ctl[7] the
// slot's item count.
__device__ __forceinline__ void init_item_queue(int* s_ctl)
{
    s_ctl[4] = -1;
    s_ctl[5] = 0;
    s_ctl[6] = 0;
    s_ctl[7] = 0;
}

// by_item (the forwards, which keep no per-slot state between items): work
// is handed out by item from the item queue (the slot queue's order, each
// slot's items in a row), so the items of a large slot spread over several
// CTAs; a CTA stages a slot's planes when its next item is of another slot.
__device__ __forceinline__ ItemInfo next_item(const FusedParams& p, int queue, float* sm, SegTab tab, uint64_t* bar,
                                              int* s_ctl, bool want_dI, int map_cap = kSegMapCap,
                                              bool by_item = false)
{
    const Ws& w = p.ws;
    const int tid = threadIdx.x;
    if (tid < 32) {
        if (tid == 0 && by_item) {
            int slot = -1, b0 = 0, nseg = 0, flags = 0;
            const int q = atomicAdd(&w.counters[queue], 1);
            if (q < w.counters[4]) {
                const int2 e = w.item_queue[q];
                slot = e.x;
                const int nit = w.item_offset[slot + 1] - w.item_offset[slot];
                if (slot != s_ctl[4]) {
                    s_ctl[4] = slot;
                    flags |= 1;
                    if (slot < w.nslot) {
                        const int esz = p.field.dtype == ATDF_BF16 ? 2 : 4;
                        uint32_t bytes = 0;
                        for (int m = 0; m < 3; ++m)
                            bytes += (uint32_t)(p.field.plane_h[m] * p.field.plane_w[m] * p.field.channels * esz);
                        mbar_expect_tx(bar, bytes);
                        flags |= 4;
                    }
                }
                const int cnt = w.slot_offset[slot + 1] - w.slot_offset[slot];
                const int per = (cnt + nit - 1) / nit;
                b0 = w.slot_offset[slot] + e.y * per;
                nseg = min(b0 + per, w.slot_offset[slot + 1]) - b0;
                if (e.y == nit - 1) flags |= 2;
                s_ctl[7] = nit;
            }
            s_ctl[0] = slot;
            s_ctl[1] = b0;
            s_ctl[2] = nseg;
            s_ctl[3] = flags;
        } else if (tid == 0) {
            int slot = -1, b0 = 0, nseg = 0, flags = 0;
            if (s_ctl[5] >= s_ctl[6]) {  // the current slot is done: take the next one with work
                const int nslots = (int)w.nslot + 1;  // plane slots + the out-of-ROI bucket
                s_ctl[4] = -1;
                while (true) {
                    const int q = atomicAdd(&w.counters[queue], 1);
                    if (q >= nslots) break;
                    const int sl = w.slot_cursor[q];  // largest slots first (slot_order_kernel)
                    const int i0 = w.item_offset[sl], i1 = w.item_offset[sl + 1];
                    if (i1 > i0) {
                        s_ctl[4] = sl;
                        s_ctl[5] = i0;
                        s_ctl[6] = i1;
                        s_ctl[7] = i1 - i0;
                        flags |= 1;
                        break;
                    }
                }
                if (s_ctl[4] >= 0 && s_ctl[4] < w.nslot) {
                    // plane_off counts elements of the plane type (4 or 2 bytes)
                    const int esz = p.field.dtype == ATDF_BF16 ? 2 : 4;
                    uint32_t bytes = 0;
                    for (int m = 0; m < 3; ++m)
                        bytes += (uint32_t)(p.field.plane_h[m] * p.field.plane_w[m] * p.field.channels * esz);
                    mbar_expect_tx(bar, bytes);
                    flags |= 4;  // warp 0 issues the slot's plane copies below
                }
            }
            if (s_ctl[4] >= 0 && s_ctl[5] < s_ctl[6]) {
                slot = s_ctl[4];
                const int it = s_ctl[5]++;
                // the slot's segments in s_ctl[7] items of equal size (<= kSegItem)
                const int cnt = w.slot_offset[slot + 1] - w.slot_offset[slot];
                const int per = (cnt + s_ctl[7] - 1) / s_ctl[7];
                b0 = w.slot_offset[slot] + (it - w.item_offset[slot]) * per;
                const int b1 = min(b0 + per, w.slot_offset[slot + 1]);
                nseg = b1 - b0;
                if (s_ctl[5] == s_ctl[6]) flags |= 2;
            }
            s_ctl[0] = slot;
            s_ctl[1] = b0;
            s_ctl[2] = nseg;
            s_ctl[3] = flags;
        }
        __syncwarp();
        if (s_ctl[3] & 4) {  // a new plane slot: its three planes, the copies spread over warp 0's lanes
            const int64_t sl = s_ctl[4];
            const int esz = p.field.dtype == ATDF_BF16 ? 2 : 4;
            fence_proxy_async();
            // copy c of plane m: its whole plane (unpadded) or its row c (padded)
            int c0 = 0;
            for (int m = 0; m < 3; ++m) {
                const int64_t pf = (int64_t)p.field.plane_h[m] * p.field.plane_w[m] * p.field.channels;
                char* dst = reinterpret_cast<char*>(sm) + (size_t)p.plane_off[m] * esz;
                const char* src = reinterpret_cast<const char*>(p.field.plane[m]) + (size_t)sl * pf * esz;
                const bool padded = p.plane_pitch[m] != p.field.plane_w[m];
                const int ncopy = padded ? p.field.plane_h[m] : 1;
                const uint32_t row = (uint32_t)(p.field.plane_w[m] * p.field.channels * esz);
                const uint32_t pitch = (uint32_t)(p.plane_pitch[m] * p.field.channels * esz);
                for (int c = ((tid - c0) % 32 + 32) % 32; c < ncopy; c += 32) {
                    if (padded)
                        tma_bulk_load(dst + (size_t)c * pitch, src + (size_t)c * row, row, bar);
                    else
                        tma_bulk_load(dst, src, (uint32_t)(pf * esz), bar);
                }
                c0 += ncopy;
            }
        }
    }
    __syncthreads();
    ItemInfo info;
    info.slot = s_ctl[0];
    info.nseg = s_ctl[2];
    info.first = (s_ctl[3] & 1) != 0;
    info.last = (s_ctl[3] & 2) != 0;
    info.slot_items = s_ctl[7];
    info.total = 0;
    info.inv_total = 0.0;
    info.use_map = false;
    if (info.slot < 0) return info;
    const int b0 = s_ctl[1];
    if (tid < info.nseg) {
        const int sid = w.bucket[b0 + tid];
        tab.id[tid] = sid;
        tab.node[tid] = w.node[sid];
        tab.n[tid] = w.nsamp[sid];
        const float tmin = w.tmin[sid], tmax = w.tmax[sid];
        const int n = w.nsamp[sid], node = w.node[sid];
        tab.tmin[tid] = tmin;
        tab.tmax[tid] = tmax;
        tab.step[tid] = __fdiv_rn(__fsub_rn(tmax, tmin), (float)n);  // sample_t's step
        tab.acc[tid] = want_dI ? p.grad_image[w.ray[sid]] : 0.0f;
        tab.first[tid] = p.xt ? (int)(w.ray_sample_offset[w.ray[sid]] + w.first[sid]) : 0;
        const int r = w.ray[sid];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            tab.org[k][tid] = p.origin[3 * r + k];
            tab.dir[k][tid] = p.dir[3 * r + k];
        }
        const uint64_t key = p.seed ? jitter_key(p.seed, r) : 0ull;
        tab.key_lo[tid] = (unsigned)key;
        tab.key_hi[tid] = (unsigned)(key >> 32);
        if (tid == 0) {  // the item's leaf (segment 0's; other leaves read the tree)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float mn = p.tree.node_position_min[3 * node + k], mx = p.tree.node_position_max[3 * node + k];
                const float sz = __fsub_rn(mx, mn);
                tab.box[k] = mn;
                tab.box[3 + k] = sz;
                tab.box[6 + k] = pow2_reciprocal(sz);
            }
            reinterpret_cast<int*>(tab.box)[9] = node;
        }
    }
    __syncthreads();
    if (tid < 32) {
        // exclusive scan of the sample counts (kSegItem = 128: four per lane)
        constexpr int PL = kSegItem / 32;
        int v[PL];
        int s = 0;
#pragma unroll
        for (int q = 0; q < PL; ++q) {
            const int i = PL * tid + q;
            v[q] = i < info.nseg ? tab.n[i] : 0;
            s += v[q];
        }
        int incl = s;
        for (int off = 1; off < 32; off <<= 1) {
            const int x = __shfl_up_sync(0xffffffffu, incl, off);
            if (tid >= off) incl += x;
        }
        int ex = incl - s;
#pragma unroll
        for (int q = 0; q < PL; ++q) {
            tab.start[PL * tid + q] = ex;
            ex += v[q];
        }
        if (tid == 31) tab.start[kSegItem] = incl;
    }
    __syncthreads();
    info.total = tab.start[info.nseg];
    info.inv_total = info.total > 0 ? 1.0 / (double)info.total : 0.0;
    // sample -> segment map (one byte per sample), in place of a binary
    // search of the count scan per sample
    info.use_map = info.total <= map_cap;
    if (info.use_map && tid < info.nseg) {
        const int b = tab.start[tid], e = tab.start[tid + 1];
        for (int k = b; k < e; ++k) tab.map[k] = (unsigned char)tid;
    }
    __syncthreads();
    return info;
}

// Geometry of sample k of the current item (computed by all 8 threads of the
// sample): segment index, weight, position.
struct SampleState {
    int si;
    float w;
    float t;
    float pos[3];
    int node;
};

__device__ __forceinline__ int find_seg(const SegTab& tab, int nseg, int k)
{
    int lo = 0, hi = nseg;  // start[lo] <= k < start[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (tab.start[mid] <= k)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// sample_t with the segment's step precomputed (same operations).
__device__ __forceinline__ float sample_t_step(float tmin, float step, int j, float a)
{
    const float t1 = __fadd_rn(tmin, __fmul_rn((float)j, step));
    const float t2 = __fadd_rn(tmin, __fmul_rn((float)(j + 1), step));
    const float oma = __fsub_rn(1.0f, a);
    return __fadd_rn(__fmul_rn(t1, oma), __fmul_rn(t2, a));
}

// permute: visit the item's samples in the permuted order (kernels that
// scatter with shared-memory atomics); without it sample k is the item's k-th
// (consecutive rows walk along a ray, so their gathers share texels).
__device__ __forceinline__ SampleState sample_state(const FusedParams& p, const SegTab& tab, const ItemInfo& it,
                                                    int k, bool permute = true)
{
    SampleState s;
    const int kk = permute && it.total < kSamplePermPrime ? perm_index(k, it.total, it.inv_total) : k;
    s.si = it.use_map ? (int)tab.map[kk] : find_seg(tab, it.nseg, kk);
    const int j = kk - tab.start[s.si];
    const int n = tab.n[s.si];
    s.node = tab.node[s.si];
    const float tmin = tab.tmin[s.si], tmax = tab.tmax[s.si], step = tab.step[s.si];
    float t;
    if (p.xt) {
        const int gi = tab.first[s.si] + j;
        t = p.xt[gi];
        s.w = p.xw[gi];
    } else {
        // jitter hash of (seed, ray, node, j) from the ray's key in the table
        // (sample_a's value: the same hash, or 0.5 without a seed)
        const uint64_t key = ((uint64_t)tab.key_hi[s.si] << 32) | tab.key_lo[s.si];
        auto a = [&](int jj) { return p.seed ? jitter_keyed(key, s.node, jj) : 0.5f; };
        t = sample_t_step(tmin, step, j, a(j));
        const float tp = j > 0 ? sample_t_step(tmin, step, j - 1, a(j - 1)) : 0.0f;
        const float tn = j < n - 1 ? sample_t_step(tmin, step, j + 1, a(j + 1)) : 0.0f;
        s.w = sample_w(tmin, tmax, n, j, tp, t, tn);
    }
    s.t = t;
#pragma unroll
    for (int k2 = 0; k2 < 3; ++k2) s.pos[k2] = __fadd_rn(tab.org[k2][s.si], __fmul_rn(tab.dir[k2][s.si], t));
    return s;
}

// sample_geo with the segment's box from the table and division-free
// coordinates where the divisor is a power of two (bit-identical).
__device__ __forceinline__ SampleGeo sample_geo_fast(const FusedParams& p, const SegTab& tab, int node,
                                                     const float pos[3])
{
    float loc[3];
    if (node == reinterpret_cast<const int*>(tab.box)[9]) {
#pragma unroll
        for (int k = 0; k < 3; ++k) loc[k] = local_coord_fast(pos[k], tab.box[k], tab.box[3 + k], tab.box[6 + k]);
    } else {  // a slot shared by several leaves: this sample's box from the tree
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float mn = p.tree.node_position_min[3 * node + k], mx = p.tree.node_position_max[3 * node + k];
            const float sz = __fsub_rn(mx, mn);
            loc[k] = local_coord_fast(pos[k], mn, sz, pow2_reciprocal(sz));
        }
    }
    SampleGeo g;
    g.pu[0] = loc[1];
    g.pv[0] = loc[2];
    g.pu[1] = loc[0];
    g.pv[1] = loc[2];
    g.pu[2] = loc[0];
    g.pv[2] = loc[1];
    const float a = __fsub_rn(pos[0], p.field.roi_min[0]);
    const float b = __fmul_rn(2.0f, a);
    const float c = p.roi_inv != 0.0f ? __fmul_rn(b, p.roi_inv)
                                      : __fdiv_rn(b, __fsub_rn(p.field.roi_max[0], p.field.roi_min[0]));
    g.lu[0] = __fsub_rn(c, 1.0f);
    g.lu[1] = loc[1];
    g.lu[2] = pos[2];
    return g;
}

// Adds rho * w of a sample at t into its segment's bins (forward, optional).
__device__ __forceinline__ void add_to_bins(const FusedParams& p, const SegTab& tab, int si, float t, float v)
{
    const float tmin = tab.tmin[si], len = tab.tmax[si] - tmin;
    int b = len > 0.0f ? (int)((t - tmin) / len * (float)kBins) : 0;
    b = b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
    atomicAdd(&p.bins[(int64_t)tab.id[si] * kBins + b], v);
}

// BF16 tensor-core variants: 16 channels (fused_tc.cu) and 24 channels
// (fused_tc24.cu); launch_tc_* dispatch on the field's channel count.
bool tc_supported(const atdf_field_t* f, const atdf_mlp_t* m);
bool tc24_supported(const atdf_field_t* f, const atdf_mlp_t* m);
int launch_tc_forward(const FusedParams& p, cudaStream_t st);
int launch_tc_backward(const FusedParams& p, cudaStream_t st);
int launch_tc24_forward(const FusedParams& p, cudaStream_t st);
int launch_tc24_backward(const FusedParams& p, cudaStream_t st);

}  // namespace atdf
