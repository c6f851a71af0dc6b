// HyperTree ray/leaf intersection, canonical segment lists, sample emission,
// local coordinates and point location for sm_100a.
//
// Reference: hyperacorn/csrc/structure/HyperTree.cu:237-259 (local samples),
// :266-514 (ComputeRaySamples), :516-610 (CreateSamplesForRays),
// :1339-1525 (NodeIdForPositionGPU); HyperTree.h:338-380 (slab test).
//
// The reference tests every active leaf against every ray (one CTA per ray,
// O(leaves) per ray). Here one warp walks the tree top-down: a child's box lies
// inside its parent's and the float slab test is monotone in the box bounds,
// so a subtree whose box the ray misses holds no leaf the reference would hit;
// leaves are then tested with the reference's own test and grazing rule.
// Hits are sorted by (tmin, node id), the canonical order of the reference's
// unordered append.

#include "atdf_common.cuh"

namespace atdf {

// Exclusive scan of n values with one 1024-thread block: each thread owns a
// contiguous chunk, loads it 8 values at a time (the loads of a group are in
// flight together; chunks of up to 16 stay in registers for the write-back),
// then a warp-shuffle scan of the chunk sums and one of the 32 warp totals.
template <typename T>
__device__ __forceinline__ void block_scan_exclusive(T* data, int64_t n, T* total, T* warp_sums)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t per = div_up(n, 1024);
    const int64_t b = min(n, (int64_t)tid * per), e = min(n, b + per);
    constexpr int KEEP = 17;  // 16384 rays + 1 offsets per 1024 threads
    T keep[KEEP];
    T s = 0;
    if (per <= KEEP) {
#pragma unroll
        for (int k = 0; k < KEEP; ++k) keep[k] = b + k < e ? data[b + k] : T(0);
#pragma unroll
        for (int k = 0; k < KEEP; ++k) s += keep[k];
    } else {
        for (int64_t i = b; i < e; i += 8) {
            T v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = i + k < e ? data[i + k] : T(0);
#pragma unroll
            for (int k = 0; k < 8; ++k) s += v[k];
        }
    }
    T incl = s;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const T x = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += x;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const T ws = warp_sums[lane];
        T wi = ws;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const T x = __shfl_up_sync(0xffffffffu, wi, off);
            if (lane >= off) wi += x;
        }
        warp_sums[lane] = wi - ws;  // exclusive warp offsets
        if (lane == 31 && total) *total = wi;
    }
    __syncthreads();
    T run = warp_sums[warp] + incl - s;
    if (per <= KEEP) {
#pragma unroll
        for (int k = 0; k < KEEP; ++k)
            if (b + k < e) {
                data[b + k] = run;
                run += keep[k];
            }
    } else {
        for (int64_t i = b; i < e; i += 8) {
            T v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = i + k < e ? data[i + k] : T(0);
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if (i + k < e) {
                    data[i + k] = run;
                    run += v[k];
                }
        }
    }
    __syncthreads();  // warp_sums is reused by a second scan in the same block
}

__global__ void scan_exclusive_i64_kernel(int64_t* data, int64_t n, int64_t* total)
{
    __shared__ int64_t ws[32];
    block_scan_exclusive<int64_t>(data, n, total, ws);
}

// Two arrays of the same length in one launch (blocks 0 and 1).
__global__ void scan2_exclusive_i64_kernel(int64_t* a, int64_t* b, int64_t n)
{
    __shared__ int64_t ws[32];
    block_scan_exclusive<int64_t>(blockIdx.x == 0 ? a : b, n, nullptr, ws);
}

__global__ void scan_exclusive_i32_kernel(int32_t* data, int64_t n, int32_t* total)
{
    __shared__ int32_t ws[32];
    block_scan_exclusive<int32_t>(data, n, total, ws);
}

// bit 0: active leaf; bit 1: some descendant is an active leaf. Bits only
// grow, so the sweep converges in max_depth + 1 rounds; 64 rounds bound it.
__global__ void tree_flags_kernel(const int32_t* active, const int32_t* children, int ns, int64_t num_nodes,
                                  uint8_t* flags, int32_t* err)
{
    __shared__ int changed;
    for (int64_t i = threadIdx.x; i < num_nodes; i += blockDim.x) flags[i] = active[i] == 1 ? 1 : 0;
    __syncthreads();
    int round = 0;
    for (; round < 64; ++round) {
        if (threadIdx.x == 0) changed = 0;
        __syncthreads();
        for (int64_t i = threadIdx.x; i < num_nodes; i += blockDim.x) {
            uint8_t f = flags[i];
            uint8_t nf = f;
            for (int k = 0; k < ns; ++k) {
                int c = children[i * ns + k];
                if (c < 0) continue;
                if (c >= num_nodes) {
                    set_err(err, ATDF_DEVERR_INDEX);
                    continue;
                }
                if (((volatile uint8_t*)flags)[c] & 3) nf |= 2;
            }
            if (nf != f) {
                flags[i] = nf;
                changed = 1;
            }
        }
        __syncthreads();
        if (!changed) break;
        __syncthreads();
    }
    if (round == 64 && threadIdx.x == 0) set_err(err, ATDF_DEVERR_TREE);
}

constexpr int kSegWarps = 8;

// Modes of ray_segments_kernel.
enum SegMode {
    kSegCount = 0,      // per-ray segment and sample counts
    kSegWrite = 1,      // traverse again, write the canonical segments at the scanned offsets
    kSegCountKeep = 2,  // counts, and the ray's sorted hits kept in scratch (kept_per entries per ray)
    kSegWriteKept = 3,  // write the canonical segments from the kept hits (no traversal)
};

// One warp per ray.
template <int MODE>
__global__ void __launch_bounds__(kSegWarps * 32)
    ray_segments_kernel(atdf_tree_t tree, const float* __restrict__ origin, const float* __restrict__ dir, int64_t R,
                        int M, atdf_segments_t segs, int32_t* err, uint32_t* kept_lo, uint32_t* kept_hi,
                        int64_t kept_per)
{
    constexpr bool WRITE = MODE == kSegWrite || MODE == kSegWriteKept;
    constexpr bool TRAVERSE = MODE != kSegWriteKept;
    __shared__ uint64_t keys[kSegWarps][ATDF_MAX_HITS];
    __shared__ int32_t front[kSegWarps][2][ATDF_MAX_HITS];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int64_t r = (int64_t)blockIdx.x * kSegWarps + warp;
    if (!WRITE && blockIdx.x == 0 && threadIdx.x == 0) {
        segs.ray_seg_offset[R] = 0;
        segs.ray_sample_offset[R] = 0;
    }
    if (r >= R) return;

    float o[3], d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        o[k] = origin[3 * r + k];
        d[k] = dir[3 * r + k];
    }
    const float* pmin = tree.node_position_min;
    const float* pmax = tree.node_position_max;
    const int ns = tree.ns;

    uint64_t* key = keys[warp];
    int nhit = 0;
    int64_t nsamp = 0;
    bool overflow = false;

    if constexpr (!TRAVERSE) {  // the hits kept by the counting pass, already sorted
        nhit = (int)(segs.ray_seg_offset[r + 1] - segs.ray_seg_offset[r]);
        const int kmax = (int)(kept_per < ATDF_MAX_HITS ? kept_per : ATDF_MAX_HITS);
        nhit = max(0, min(nhit, kmax));
        for (int i = lane; i < nhit; i += 32)
            key[i] = ((uint64_t)kept_hi[r * kept_per + i] << 32) | kept_lo[r * kept_per + i];
        __syncwarp();
    } else {
    // root
    int nfront = 0;
    int cur = 0;
    {
        uint8_t f = tree.node_flags[0];
        float tmin, tmax;
        bool hit = (f & 3) ? intersect_box(pmin, pmax, o, d, tmin, tmax) : false;
        if (f & 1) {
            if (hit && !((double)__fsub_rn(tmax, tmin) < 1e-5)) {
                nhit = 1;
                if (lane == 0) {
                    nsamp = seg_num_samples(pmin, pmax, tmin, tmax, M);
                    key[0] = ((uint64_t)float_key(tmin) << 32) | 0u;
                }
            }
        } else if ((f & 2) && hit) {
            nfront = 1;
            if (lane == 0) front[warp][0][0] = 0;
        }
    }
    __syncwarp();

    // breadth-first descent, one level per round
    for (int level = 0; nfront > 0 && level < 64; ++level) {
        const int32_t* fr = front[warp][cur];
        int32_t* nx = front[warp][cur ^ 1];
        int nnext = 0;
        const int pairs = nfront * ns;
        for (int base = 0; base < pairs; base += 32) {
            const int p = base + lane;
            bool leaf_hit = false, node_hit = false;
            int child = -1;
            float tmin = 0, tmax = 0;
            if (p < pairs) {
                const int parent = fr[p / ns];
                child = tree.node_children[(int64_t)parent * ns + (p % ns)];
                if (child >= tree.num_nodes) {
                    set_err(err, ATDF_DEVERR_INDEX);
                    child = -1;
                }
                if (child >= 0) {
                    const uint8_t f = tree.node_flags[child];
                    if (f & 3) {
                        const bool hit = intersect_box(pmin + 3 * (int64_t)child, pmax + 3 * (int64_t)child, o, d,
                                                       tmin, tmax);
                        if (f & 1)
                            leaf_hit = hit && !((double)__fsub_rn(tmax, tmin) < 1e-5);
                        else
                            node_hit = hit;
                    }
                }
            }
            const unsigned lb = __ballot_sync(0xffffffffu, leaf_hit);
            const unsigned nb = __ballot_sync(0xffffffffu, node_hit);
            const int lpos = nhit + __popc(lb & ((1u << lane) - 1));
            const int npos = nnext + __popc(nb & ((1u << lane) - 1));
            if (leaf_hit) {
                if (lpos < ATDF_MAX_HITS) {
                    key[lpos] = ((uint64_t)float_key(tmin) << 32) | (uint32_t)child;
                    nsamp += seg_num_samples(pmin + 3 * (int64_t)child, pmax + 3 * (int64_t)child, tmin, tmax, M);
                }
            }
            if (node_hit && npos < ATDF_MAX_HITS) nx[npos] = child;
            nhit += __popc(lb);
            nnext += __popc(nb);
            if (nhit > ATDF_MAX_HITS || nnext > ATDF_MAX_HITS) overflow = true;
            nhit = min(nhit, ATDF_MAX_HITS);
            nnext = min(nnext, ATDF_MAX_HITS);
        }
        __syncwarp();
        nfront = nnext;
        cur ^= 1;
    }
    if (overflow && lane == 0) set_err(err, ATDF_DEVERR_HIT_OVERFLOW);

    // warp total of samples (each lane summed its own hits)
    for (int off = 16; off > 0; off >>= 1) nsamp += __shfl_xor_sync(0xffffffffu, nsamp, off);
    }

    if constexpr (!WRITE) {
        if (lane == 0) {
            segs.ray_seg_offset[r] = nhit;
            segs.ray_sample_offset[r] = nsamp;
            atomicMax((unsigned long long*)&segs.totals[2], (unsigned long long)nsamp);
            atomicMax((unsigned long long*)&segs.totals[3], (unsigned long long)nhit);
        }
        if constexpr (MODE == kSegCount) return;
    }

    if constexpr (TRAVERSE) {
        // sort the hits by (tmin, node): bitonic sort of the padded key array
        int npow = 32;
        while (npow < nhit) npow <<= 1;
        for (int i = nhit + lane; i < npow; i += 32) key[i] = ~0ull;
        __syncwarp();
        for (int k = 2; k <= npow; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = lane; i < npow; i += 32) {
                    const int ixj = i ^ j;
                    if (ixj > i) {
                        const uint64_t a = key[i], b = key[ixj];
                        const bool up = (i & k) == 0;
                        if ((a > b) == up) {
                            key[i] = b;
                            key[ixj] = a;
                        }
                    }
                }
                __syncwarp();
            }
        }
    }

    if constexpr (MODE == kSegCountKeep) {  // keep the sorted hits for the writing pass
        if (nhit > kept_per) {
            if (lane == 0) set_err(err, ATDF_DEVERR_SEG_CAPACITY);
            return;
        }
        for (int i = lane; i < nhit; i += 32) {
            kept_lo[r * kept_per + i] = (uint32_t)key[i];
            kept_hi[r * kept_per + i] = (uint32_t)(key[i] >> 32);
        }
        return;
    }

    const int64_t seg0 = segs.ray_seg_offset[r];
    if (seg0 + nhit > segs.capacity) {
        if (lane == 0) set_err(err, ATDF_DEVERR_SEG_CAPACITY);
        return;
    }
    // each lane owns up to 8 consecutive sorted hits
    constexpr int PER = ATDF_MAX_HITS / 32;
    int nloc[PER];
    int lsum = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int i = lane * PER + q;
        nloc[q] = 0;
        if (i < nhit) {
            int node = (int)(key[i] & 0xffffffffu);
            if (node < 0 || node >= tree.num_nodes) {  // kept hits of a ray that overflowed its slots
                set_err(err, ATDF_DEVERR_INDEX);
                node = 0;
            }
            float tmin, tmax;
            intersect_box(pmin + 3 * (int64_t)node, pmax + 3 * (int64_t)node, o, d, tmin, tmax);
            nloc[q] = seg_num_samples(pmin + 3 * (int64_t)node, pmax + 3 * (int64_t)node, tmin, tmax, M);
            const int64_t s = seg0 + i;
            segs.node[s] = node;
            segs.tmin[s] = tmin;
            segs.tmax[s] = tmax;
            segs.nsamp[s] = nloc[q];
            segs.ray[s] = (int32_t)r;
        }
        lsum += nloc[q];
    }
    int incl = lsum;
    for (int off = 1; off < 32; off <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += v;
    }
    int run = incl - lsum;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int i = lane * PER + q;
        if (i < nhit) segs.first[seg0 + i] = run;
        run += nloc[q];
    }
}

// One warp per ray: the SampleList of the ray's segments.
__global__ void __launch_bounds__(256)
    emit_samples_kernel(atdf_segments_t segs, int64_t R, const float* __restrict__ origin,
                        const float* __restrict__ dir, const float* __restrict__ rnd, uint64_t seed, float* out_pos,
                        float* out_t, float* out_w, int64_t* out_ray, int64_t* out_local, int64_t* out_node,
                        int64_t cap, int32_t* err)
{
    const int lane = threadIdx.x & 31;
    const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= R) return;
    const int64_t sb = segs.ray_seg_offset[r], se = segs.ray_seg_offset[r + 1];
    const int64_t base = segs.ray_sample_offset[r];
    if (se - sb > 0 && se > segs.capacity) return;  // flagged by the segment pass
    float o[3], d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        o[k] = origin[3 * r + k];
        d[k] = dir[3 * r + k];
    }
    for (int64_t s = sb; s < se; ++s) {
        const int n = segs.nsamp[s];
        const int node = segs.node[s];
        const float tmin = segs.tmin[s], tmax = segs.tmax[s];
        const int64_t g0 = base + segs.first[s];
        for (int j = lane; j < n; j += 32) {
            const int64_t g = g0 + j;
            if (g >= cap) {
                set_err(err, ATDF_DEVERR_SAMPLE_CAPACITY);
                continue;
            }
            const float t = sample_t(tmin, tmax, n, j, sample_a(rnd, g, seed, (int32_t)r, node, j));
            const float tp = j > 0 ? sample_t(tmin, tmax, n, j - 1, sample_a(rnd, g - 1, seed, (int32_t)r, node, j - 1))
                                   : 0.0f;
            const float tn = j < n - 1
                                 ? sample_t(tmin, tmax, n, j + 1, sample_a(rnd, g + 1, seed, (int32_t)r, node, j + 1))
                                 : 0.0f;
            out_t[g] = t;
            out_w[g] = sample_w(tmin, tmax, n, j, tp, t, tn);
#pragma unroll
            for (int k = 0; k < 3; ++k) out_pos[3 * g + k] = __fadd_rn(o[k], __fmul_rn(d[k], t));
            out_ray[g] = r;
            out_local[g] = segs.first[s] + j;
            out_node[g] = node;
        }
    }
}

__global__ void local_samples_kernel(const float* __restrict__ pos, const int64_t* __restrict__ node, int64_t P,
                                     int64_t group, const float* __restrict__ pmin, const float* __restrict__ pmax,
                                     int64_t num_nodes, float* out, int32_t* err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const int64_t nd = node[group > 1 ? i / group : i];
    if (nd < 0 || nd >= num_nodes) {
        set_err(err, ATDF_DEVERR_INDEX);
        return;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) out[3 * i + k] = local_coord(pos[3 * i + k], pmin[3 * nd + k], pmax[3 * nd + k]);
}

__global__ void node_id_kernel(atdf_tree_t tree, const int64_t* __restrict__ active_ids, const float* __restrict__ pos,
                               int64_t P, int64_t* out_id, float* out_mask, int32_t* err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const float p0 = pos[3 * i], p1 = pos[3 * i + 1], p2 = pos[3 * i + 2];
    const float* mn = tree.node_position_min;
    const float* mx = tree.node_position_max;
    int64_t cur = 0, res = -1;
    for (int it = 0; it < 64; ++it) {
        if (tree.node_active[cur] > 0) {
            res = cur;
            break;
        }
        const int64_t prev = cur;
        bool missing = false;
        for (int k = 0; k < tree.ns; ++k) {
            const int c = tree.node_children[cur * tree.ns + k];
            if (c == -1) {
                missing = true;
                break;
            }
            if (c < 0 || c >= tree.num_nodes) {
                set_err(err, ATDF_DEVERR_INDEX);
                missing = true;
                break;
            }
            if (mn[3 * c] <= p0 && mx[3 * c] >= p0 && mn[3 * c + 1] <= p1 && mx[3 * c + 1] >= p1 &&
                mn[3 * c + 2] <= p2 && mx[3 * c + 2] >= p2) {
                cur = c;
                break;
            }
        }
        if (missing || cur == prev) break;
    }
    if (res < 0) {
        out_id[i] = active_ids[0];
        out_mask[i] = 0.0f;
    } else {
        out_id[i] = res;
        out_mask[i] = 1.0f;
    }
}

// Launch helpers shared with the fused path. kept_lo / kept_hi (nullable):
// scratch of R * kept_per entries each where the counting pass keeps every
// ray's sorted hits, so that the writing pass does not traverse the tree again.
int launch_ray_segments(const atdf_tree_t& tree, const float* origin, const float* dir, int64_t R, int M,
                        const atdf_segments_t& segs, int32_t* err, cudaStream_t st, uint32_t* kept_lo = nullptr,
                        uint32_t* kept_hi = nullptr, int64_t kept_per = 0)
{
    ATDF_CUDA_TRY(cudaMemsetAsync(segs.totals, 0, 4 * sizeof(int64_t), st));
    const int64_t blocks = div_up(R, kSegWarps);
    const bool keep = kept_lo && kept_hi && kept_per > 0;
    if (R > 0) {
        if (keep)
            ray_segments_kernel<kSegCountKeep><<<(unsigned)blocks, kSegWarps * 32, 0, st>>>(
                tree, origin, dir, R, M, segs, err, kept_lo, kept_hi, kept_per);
        else
            ray_segments_kernel<kSegCount><<<(unsigned)blocks, kSegWarps * 32, 0, st>>>(tree, origin, dir, R, M, segs,
                                                                                       err, nullptr, nullptr, 0);
        ATDF_LAUNCH_CHECK();
    } else {
        ATDF_CUDA_TRY(cudaMemsetAsync(segs.ray_seg_offset, 0, sizeof(int64_t), st));
        ATDF_CUDA_TRY(cudaMemsetAsync(segs.ray_sample_offset, 0, sizeof(int64_t), st));
    }
    scan2_exclusive_i64_kernel<<<2, 1024, 0, st>>>(segs.ray_seg_offset, segs.ray_sample_offset, R + 1);
    ATDF_LAUNCH_CHECK();
    ATDF_CUDA_TRY(cudaMemcpyAsync(&segs.totals[0], &segs.ray_seg_offset[R], sizeof(int64_t),
                                  cudaMemcpyDeviceToDevice, st));
    ATDF_CUDA_TRY(cudaMemcpyAsync(&segs.totals[1], &segs.ray_sample_offset[R], sizeof(int64_t),
                                  cudaMemcpyDeviceToDevice, st));
    if (R > 0) {
        if (keep)
            ray_segments_kernel<kSegWriteKept><<<(unsigned)blocks, kSegWarps * 32, 0, st>>>(
                tree, origin, dir, R, M, segs, err, kept_lo, kept_hi, kept_per);
        else
            ray_segments_kernel<kSegWrite><<<(unsigned)blocks, kSegWarps * 32, 0, st>>>(tree, origin, dir, R, M, segs,
                                                                                       err, nullptr, nullptr, 0);
        ATDF_LAUNCH_CHECK();
    }
    return ATDF_OK;
}

}  // namespace atdf

using namespace atdf;

extern "C" {

const char* atdf_status_string(int status)
{
    switch (status) {
        case ATDF_OK: return "ok";
        case ATDF_ERR_INVALID_ARGUMENT: return "invalid argument";
        case ATDF_ERR_UNSUPPORTED: return "unsupported configuration";
        case ATDF_ERR_WORKSPACE: return "workspace too small";
        case ATDF_ERR_CUDA: return "CUDA launch failed";
        default: return "unknown status";
    }
}

int atdf_version(void) { return 100; }

int atdf_tree_flags(const int32_t* node_active, const int32_t* node_children, int32_t ns, int64_t num_nodes,
                    uint8_t* node_flags, int32_t* dev_error, atdf_stream_t stream)
{
    if (!node_active || !node_children || !node_flags || num_nodes <= 0 || (ns != 4 && ns != 8))
        return ATDF_ERR_INVALID_ARGUMENT;
    tree_flags_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(node_active, node_children, ns, num_nodes, node_flags,
                                                            dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

static bool tree_ok(const atdf_tree_t* t)
{
    return t && t->node_position_min && t->node_position_max && t->node_children && t->node_flags &&
           t->num_nodes > 0 && (t->ns == 4 || t->ns == 8);
}

int atdf_ray_segments(const atdf_tree_t* tree, const float* ray_origin, const float* ray_direction, int64_t num_rays,
                      int32_t max_samples_per_node, const atdf_segments_t* segs, int32_t* dev_error,
                      atdf_stream_t stream)
{
    if (!tree_ok(tree) || !segs || num_rays < 0 || (num_rays > 0 && (!ray_origin || !ray_direction)) ||
        max_samples_per_node < 0 || !segs->ray_seg_offset || !segs->ray_sample_offset || !segs->totals)
        return ATDF_ERR_INVALID_ARGUMENT;
    if (num_rays >= (int64_t)1 << 31) return ATDF_ERR_UNSUPPORTED;
    return launch_ray_segments(*tree, ray_origin, ray_direction, num_rays, max_samples_per_node, *segs, dev_error,
                               (cudaStream_t)stream);
}

int atdf_emit_samples(const atdf_segments_t* segs, int64_t num_rays, const float* ray_origin,
                      const float* ray_direction, const float* sample_rnd, uint64_t jitter_seed, float* out_position,
                      float* out_t, float* out_weight, int64_t* out_ray_index, int64_t* out_local_index,
                      int64_t* out_node_id, int64_t sample_capacity, int32_t* dev_error, atdf_stream_t stream)
{
    if (!segs || num_rays < 0) return ATDF_ERR_INVALID_ARGUMENT;
    if (num_rays == 0) return ATDF_OK;
    // with no capacity the outputs may be null; the kernel only flags overflow
    if (sample_capacity > 0 &&
        (!out_position || !out_t || !out_weight || !out_ray_index || !out_local_index || !out_node_id))
        return ATDF_ERR_INVALID_ARGUMENT;
    const int64_t threads = num_rays * 32;
    emit_samples_kernel<<<(unsigned)div_up(threads, 256), 256, 0, (cudaStream_t)stream>>>(
        *segs, num_rays, ray_origin, ray_direction, sample_rnd, jitter_seed, out_position, out_t, out_weight,
        out_ray_index, out_local_index, out_node_id, sample_capacity, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_local_samples(const float* position, const int64_t* node, int64_t num_points, int64_t group,
                       const float* node_position_min, const float* node_position_max, int64_t num_nodes,
                       float* out_local, int32_t* dev_error, atdf_stream_t stream)
{
    if (num_points < 0 || (num_points > 0 && (!position || !node || !node_position_min || !node_position_max ||
                                              !out_local)))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (num_points == 0) return ATDF_OK;
    local_samples_kernel<<<(unsigned)div_up(num_points, 256), 256, 0, (cudaStream_t)stream>>>(
        position, node, num_points, group, node_position_min, node_position_max, num_nodes, out_local, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_node_id_for_position(const atdf_tree_t* tree, const int64_t* active_node_ids, const float* position,
                              int64_t num_points, int64_t* out_node_id, float* out_mask, int32_t* dev_error,
                              atdf_stream_t stream)
{
    if (!tree || !tree->node_active || !tree->node_children || !active_node_ids || num_points < 0 ||
        (num_points > 0 && (!position || !out_node_id || !out_mask)))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (num_points == 0) return ATDF_OK;
    node_id_kernel<<<(unsigned)div_up(num_points, 256), 256, 0, (cudaStream_t)stream>>>(
        *tree, active_node_ids, position, num_points, out_node_id, out_mask, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

}  // extern "C"
