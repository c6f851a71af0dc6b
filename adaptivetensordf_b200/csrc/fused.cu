// Fused leaf-major forward projection and its hand-written adjoint (FP32,
// CUDA cores) for sm_100a.
//
// One training step of the reference runs CreateSamplesForRays, then
// SampleVolumeIndirect (six gathers + products), DecodeFeatures (FCBlock +
// softplus) and IntegrateSamplesXRay (index_add_), materialising every [S, .]
// intermediate in HBM, and autograd replays them backwards with atomics into
// the factor-grid gradients (hyperacorn/csrc/geometry/geometry.cpp:828-1019,
// geometry_tensor_qo.cpp:257-380, modules/IndirectGridSample2D.cu:175-393).
//
// Here:
//  1. ray_segments (sampler.cu) lists every ray's leaf segments in canonical
//     order; no per-sample array is ever written.
//  2. Segments are bucketed by plane slot and cut into work items of at most
//     kSegItem segments.
//  3. A persistent kernel takes items from an atomic queue. Per item it
//     stages the slot's three factor planes in shared memory with TMA bulk
//     copies, expands the segments into samples 32 at a time, gathers the VM
//     features from shared memory, runs the decoder as register-tiled
//     shared-memory GEMMs and sums density * weight per segment.
//  4. A per-ray pass adds the segment partials in t order.
//  The backward kernel recomputes each sample (no stored activations), runs
//  the decoder backward as tile GEMMs with the weight gradients held in
//  registers across items, scatters the feature gradient into a shared-memory
//  copy of the slot's plane gradients and flushes it with vector atomics.

#include <algorithm>

#include "fused_common.cuh"

namespace atdf {

int launch_ray_segments(const atdf_tree_t& tree, const float* origin, const float* dir, int64_t R, int M,
                        const atdf_segments_t& segs, int32_t* err, cudaStream_t st, uint32_t* kept_lo = nullptr,
                        uint32_t* kept_hi = nullptr, int64_t kept_per = 0);

// The workspace's bucket and segment-partial arrays (R * per entries, idle
// until the segments exist) hold the segment pass's kept hits.
static int launch_ray_segments_ws(const atdf_tree_t& tree, const float* origin, const float* dir, int64_t R, int M,
                                  const Ws& w, int32_t* err, cudaStream_t st)
{
    const int64_t per = R > 0 ? w.cap / R : 0;
    return launch_ray_segments(tree, origin, dir, R, M, ws_segments(w), err, st, reinterpret_cast<uint32_t*>(w.bucket),
                               reinterpret_cast<uint32_t*>(w.seg_partial), per);
}

constexpr int kThreads = 256;
constexpr int kT = 32;                // samples per tile
constexpr int kSPT = kThreads / kT;   // threads per sample
// ---------------------------------------------------------------------------
// bucketing by plane slot
// ---------------------------------------------------------------------------
// A segment whose node id or plane slot is out of range sets the index bit
// and joins the out-of-ROI bucket (zero features, no gradient).
__global__ void bucket_count_kernel(Ws w, atdf_field_t f, int64_t num_nodes, int32_t* err)
{
    const int64_t nseg = min(w.totals[0], w.cap);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nseg; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t nd = w.node[i];
        if (nd < 0 || nd >= num_nodes || f.leaf_slot[nd] >= f.num_slots) set_err(err, ATDF_DEVERR_INDEX);
        atomicAdd(&w.slot_offset[seg_slot(f, num_nodes, nd)], 1);
    }
}

__global__ void bucket_scatter_kernel(Ws w, atdf_field_t f, int64_t num_nodes)
{
    const int64_t nseg = min(w.totals[0], w.cap);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nseg; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = seg_slot(f, num_nodes, w.node[i]);
        const int pos = w.slot_offset[s] + atomicAdd(&w.slot_cursor[s], 1);
        w.bucket[pos] = (int32_t)i;
    }
}

// Order of the slot queue: slots by descending segment count, so that the
// largest slots start first and the kernels' tail holds the smallest ones
// (longest-processing-time-first scheduling of the slot-sticky work). A
// counting sort on min(segments / 2, 255) in one block; it writes into
// slot_cursor, whose bucketing role has ended.
__global__ void slot_order_kernel(Ws w)
{
    __shared__ int hist[256];
    const int n = (int)w.nslot + 1;
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < n; s += blockDim.x)
        atomicAdd(&hist[255 - min((w.slot_offset[s + 1] - w.slot_offset[s]) >> 1, 255)], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int i = 0; i < 256; ++i) {
            const int c = hist[i];
            hist[i] = run;
            run += c;
        }
    }
    __syncthreads();
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
        const int pos = atomicAdd(&hist[255 - min((w.slot_offset[s + 1] - w.slot_offset[s]) >> 1, 255)], 1);
        w.slot_cursor[pos] = s;
    }
}

__global__ void item_count_kernel(Ws w)
{
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s <= w.nslot + 1;
         s += (int64_t)gridDim.x * blockDim.x) {
        if (s == w.nslot + 1) {
            w.item_offset[s] = 0;
        } else {
            const int cnt = w.slot_offset[s + 1] - w.slot_offset[s];
            w.item_offset[s] = (cnt + kSegItem - 1) / kSegItem;
        }
    }
}

// The item queue of the forwards: for each slot in the slot queue's order
// (slot_cursor) its items (slot, 0 .. n - 1), at the exclusive prefix of the
// item counts in that order; counters[4] = the number of items. One block.
__global__ void item_queue_kernel(Ws w)
{
    __shared__ int warp_sum[32];
    __shared__ int s_base;
    const int n = (int)w.nslot + 1;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    for (int c0 = 0; c0 < n; c0 += blockDim.x) {
        const int q = c0 + threadIdx.x;
        int sl = -1, ni = 0;
        if (q < n) {
            sl = w.slot_cursor[q];
            ni = w.item_offset[sl + 1] - w.item_offset[sl];
        }
        int incl = ni;
        for (int off = 1; off < 32; off <<= 1) {
            const int x = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += x;
        }
        if (lane == 31) warp_sum[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            int v = lane < nw ? warp_sum[lane] : 0;
            for (int off = 1; off < 32; off <<= 1) {
                const int x = __shfl_up_sync(0xffffffffu, v, off);
                if (lane >= off) v += x;
            }
            if (lane < nw) warp_sum[lane] = v;  // inclusive over warps
        }
        __syncthreads();
        const int pos = s_base + (wid > 0 ? warp_sum[wid - 1] : 0) + incl - ni;
        for (int i = 0; i < ni; ++i) w.item_queue[pos + i] = make_int2(sl, i);
        __syncthreads();
        if (threadIdx.x == 0) s_base += warp_sum[nw - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) w.counters[4] = s_base;
}

// Zeroes the plane gradients of the slots that no segment touches; the
// tensor-core backward writes every touched slot's gradient itself.
__global__ void zero_untouched_slots_kernel(Ws w, atdf_field_grad_t g, atdf_field_t f)
{
    for (int64_t s = blockIdx.x; s < w.nslot; s += gridDim.x) {
        if (w.item_offset[s + 1] > w.item_offset[s]) continue;
        for (int m = 0; m < 3; ++m) {
            const int64_t pf = (int64_t)f.plane_h[m] * f.plane_w[m] * f.channels;
            float* dst = g.plane[m] + s * pf;
            for (int64_t i = threadIdx.x; i < pf; i += blockDim.x) dst[i] = 0.0f;
        }
    }
}

// Per-ray sum of the segment partials, in segment (t) order.
__global__ void ray_reduce_kernel(Ws w, int64_t R, float* image)
{
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    const int64_t b = w.ray_seg_offset[r], e = w.ray_seg_offset[r + 1];
    float acc = 0.0f;
    if (e <= w.cap)
        for (int64_t s = b; s < e; ++s) acc = __fadd_rn(acc, w.seg_partial[s]);
    image[r] = acc;
}

// ---------------------------------------------------------------------------
// register-tiled shared-memory GEMM: acc[i][j] += sum_k A[k][row0+i] B[k][col0+j]
// ---------------------------------------------------------------------------
template <int N>
__device__ __forceinline__ void ldv(float (&v)[N], const float* p)
{
    if constexpr (N == 4) {
        const float4 t = *reinterpret_cast<const float4*>(p);
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    } else if constexpr (N == 2) {
        const float2 t = *reinterpret_cast<const float2*>(p);
        v[0] = t.x;
        v[1] = t.y;
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) v[i] = p[i];
    }
}

// Thread tiling of an M x N output over 256 threads.
template <int M, int N>
struct Map {
    static constexpr int PER = M * N / kThreads;
    static constexpr int RM = PER >= 16 ? 4 : (PER == 3 || PER == 1) ? 1 : 2;
    static constexpr int CN = PER / RM;
    static constexpr int TX = N / CN;
    static constexpr int TY = M / RM;
    static_assert(PER >= 1 && RM * CN == PER && TX * TY == kThreads && N % CN == 0 && M % RM == 0, "tile map");
};

// Thread coordinates of the tile map. RF (row-fast): consecutive threads own
// consecutive output rows, which makes k-major ([col][row]) epilogue stores
// conflict-free; otherwise consecutive threads own consecutive columns.
template <int M, int N, bool RF>
__device__ __forceinline__ void tile_coords(int& tx, int& ty)
{
    using Mp = Map<M, N>;
    if (RF) {
        ty = threadIdx.x % Mp::TY;
        tx = threadIdx.x / Mp::TY;
    } else {
        tx = threadIdx.x % Mp::TX;
        ty = threadIdx.x / Mp::TX;
    }
}

template <int M, int N, bool RF = false>
__device__ __forceinline__ void gemm(float (&acc)[Map<M, N>::RM][Map<M, N>::CN], const float* At, int lda,
                                     const float* Bt, int ldb, int K)
{
    using Mp = Map<M, N>;
    int tx, ty;
    tile_coords<M, N, RF>(tx, ty);
    const float* a = At + ty * Mp::RM;
    const float* b = Bt + tx * Mp::CN;
#pragma unroll 4
    for (int k = 0; k < K; ++k) {
        float av[Mp::RM], bv[Mp::CN];
        ldv<Mp::RM>(av, a + k * lda);
        ldv<Mp::CN>(bv, b + k * ldb);
#pragma unroll
        for (int i = 0; i < Mp::RM; ++i)
#pragma unroll
            for (int j = 0; j < Mp::CN; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
}

template <int M, int N>
__device__ __forceinline__ void zero(float (&acc)[Map<M, N>::RM][Map<M, N>::CN])
{
#pragma unroll
    for (int i = 0; i < Map<M, N>::RM; ++i)
#pragma unroll
        for (int j = 0; j < Map<M, N>::CN; ++j) acc[i][j] = 0.0f;
}

// ---------------------------------------------------------------------------
// fused kernels
// ---------------------------------------------------------------------------
template <int C, int MODE, int H, int NH>
struct Cfg {
    static constexpr int F = MODE ? 3 * C : C;
    static constexpr int CPT = C / kSPT;
    static_assert(C % kSPT == 0, "channels must be a multiple of 8");
    static_assert(NH == 1 || NH == 2, "one or two hidden layers");
};

// Shared-memory carve-up (floats, every region 16-byte aligned).
template <int C, int MODE, int H, int NH, bool BWD>
struct Smem {
    using K = Cfg<C, MODE, H, NH>;
    static constexpr int F = K::F;
    __host__ __device__ static constexpr int a4(int x) { return (x + 3) & ~3; }
    int planes, gplanes, gline, w0t, w0, b0, w1t, w1, b1, wl, bl, xt, xs, a0t, h0t, h0s, a1t, h1s, sw, sdi, sz, sseg,
        segi, total;
    __host__ __device__ Smem(int plane_floats)
    {
        int o = 0;
        planes = o;
        o += a4(plane_floats);
        gplanes = o;
        if (BWD) o += a4(plane_floats);
        gline = o;
        if (BWD) o += 3 * kLineWin * C;
        w0t = o;
        o += F * H;
        w0 = o;
        if (BWD) o += F * H;
        b0 = o;
        o += a4(H);
        w1t = o;
        if (NH == 2) o += H * H;
        w1 = o;
        if (NH == 2 && BWD) o += H * H;
        b1 = o;
        if (NH == 2) o += a4(H);
        wl = o;
        o += a4(H);
        bl = o;
        o += 4;
        xt = o;
        o += F * kT;
        xs = o;
        if (BWD) o += F * kT;
        a0t = o;
        if (BWD) o += H * kT;
        h0t = o;
        o += H * kT;
        h0s = o;
        if (BWD) o += H * kT;
        a1t = o;
        if (NH == 2) o += H * kT;
        h1s = o;
        if (NH == 2 && BWD) o += H * kT;
        sw = o;
        o += kT;
        sdi = o;
        o += kT;
        sz = o;
        o += kT;
        sseg = o;
        o += kT;
        segi = o;
        o += kSegTabFloats;
        total = o;
    }
};

// Gathered values of one sample for channels q*CPT .. q*CPT+CPT-1.
template <int CPT>
struct Gathered {
    float mat[3][CPT];
    float vec[3][CPT];
};

template <int C, int CPT>
__device__ __forceinline__ void gather_sample(const FusedParams& p, const float* sm, const SampleGeo& g, int q,
                                              Gathered<CPT>& out)
{
    const int c0 = q * CPT;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        const int Hm = p.field.plane_h[m], Wm = p.field.plane_w[m], L = p.field.line_len[m];
        const Corner2 k = corners2(g.pu[m], g.pv[m], Hm, Wm);
        const Corner1 l = corners1(g.lu[m], L);
        const float* P = sm + p.plane_off[m];
        const float* V = (const float*)p.field.line[m];
        float vnw[CPT], vne[CPT], vsw[CPT], vse[CPT], v0[CPT], v1[CPT];
        ldv<CPT>(vnw, P + (k.y0 * Wm + k.x0) * C + c0);
        ldv<CPT>(vne, P + (k.y0 * Wm + k.x1) * C + c0);
        ldv<CPT>(vsw, P + (k.y1 * Wm + k.x0) * C + c0);
        ldv<CPT>(vse, P + (k.y1 * Wm + k.x1) * C + c0);
#pragma unroll
        for (int cc = 0; cc < CPT; ++cc) {
            v0[cc] = __ldg(V + l.x0 * C + c0 + cc);
            v1[cc] = __ldg(V + l.x1 * C + c0 + cc);
            out.mat[m][cc] = bilerp(k, vnw[cc], vne[cc], vsw[cc], vse[cc]);
            out.vec[m][cc] = lerp1(l, v0[cc], v1[cc]);
        }
    }
}

template <int C, int MODE, int CPT>
__device__ __forceinline__ void features_of(const Gathered<CPT>& g, float (&f)[MODE ? 3 * CPT : CPT])
{
#pragma unroll
    for (int cc = 0; cc < CPT; ++cc) {
        if (MODE) {
#pragma unroll
            for (int m = 0; m < 3; ++m) f[m * CPT + cc] = __fmul_rn(g.mat[m][cc], g.vec[m][cc]);
        } else {
            float acc = __fmul_rn(g.mat[0][cc], g.vec[0][cc]);
            acc = __fadd_rn(acc, __fmul_rn(g.mat[1][cc], g.vec[1][cc]));
            acc = __fadd_rn(acc, __fmul_rn(g.mat[2][cc], g.vec[2][cc]));
            f[cc] = acc;
        }
    }
}

// feature index of local channel cc of thread q (plane m in cat mode)
template <int C, int MODE, int CPT>
__device__ __forceinline__ int feat_index(int q, int m, int cc)
{
    return MODE ? m * C + q * CPT + cc : q * CPT + cc;
}

// Loads the decoder weights into shared memory (k-major copies for the
// forward GEMMs, row-major copies for the backward).
template <int C, int MODE, int H, int NH, bool BWD>
__device__ void load_weights(const FusedParams& p, float* sm, const Smem<C, MODE, H, NH, BWD>& L)
{
    constexpr int F = Cfg<C, MODE, H, NH>::F;
    const atdf_mlp_t& m = p.mlp;
    for (int i = threadIdx.x; i < F * H; i += kThreads) {
        const int o = i / F, k = i % F;  // W0 [H][F]
        const float v = m.weight[0][i];
        sm[L.w0t + k * H + o] = v;
        if (BWD) sm[L.w0 + i] = v;
    }
    for (int i = threadIdx.x; i < H; i += kThreads) sm[L.b0 + i] = m.bias[0][i];
    if (NH == 2) {
        for (int i = threadIdx.x; i < H * H; i += kThreads) {
            const int o = i / H, k = i % H;
            const float v = m.weight[1][i];
            sm[L.w1t + k * H + o] = v;
            if (BWD) sm[L.w1 + i] = v;
        }
        for (int i = threadIdx.x; i < H; i += kThreads) sm[L.b1 + i] = m.bias[1][i];
    }
    for (int i = threadIdx.x; i < H; i += kThreads) sm[L.wl + i] = m.weight[NH][i];
    if (threadIdx.x == 0) sm[L.bl] = m.bias[NH][0];
}

// Epilogue of a forward layer: pre = acc + b; writes act(pre) k-major (and
// the pre-activation / a sample-major copy when requested).
template <int M, int N, bool RF = false>
__device__ __forceinline__ void store_layer(const float (&acc)[Map<M, N>::RM][Map<M, N>::CN], const float* bias,
                                            int act, float beta, float* out_t, float* pre_t, float* out_s)
{
    using Mp = Map<M, N>;
    int tx, ty;
    tile_coords<M, N, RF>(tx, ty);
#pragma unroll
    for (int i = 0; i < Mp::RM; ++i)
#pragma unroll
        for (int j = 0; j < Mp::CN; ++j) {
            const int row = ty * Mp::RM + i, col = tx * Mp::CN + j;
            const float pre = acc[i][j] + bias[col];
            const float h = act_fwd(act, pre, beta);
            if (out_t) out_t[col * M + row] = h;
            if (pre_t) pre_t[col * M + row] = pre;
            if (out_s) out_s[row * N + col] = h;
        }
}

// Last layer z[s] = sum_k Hs_t[k][s] W[k] + b, 8 threads per sample.
template <int H>
__device__ __forceinline__ float last_layer(const float* ht, const float* wl, float bl, int s, int q)
{
    float acc = 0.0f;
#pragma unroll
    for (int i = 0; i < H / kSPT; ++i) {
        const int k = q + kSPT * i;
        acc = fmaf(ht[k * kT + s], wl[k], acc);
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 4);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    return acc + bl;
}

template <int C, int MODE, int H, int NH>
__global__ void __launch_bounds__(kThreads) fused_forward_kernel(FusedParams p)
{
    using K = Cfg<C, MODE, H, NH>;
    constexpr int F = K::F, CPT = K::CPT, NF = MODE ? 3 * CPT : CPT;
    extern __shared__ __align__(16) float sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int s_ctl[8];
    const Smem<C, MODE, H, NH, false> L(p.plane_off[3]);
    const int tid = threadIdx.x;
    const int s = tid / kSPT, q = tid % kSPT;
    if (tid == 0) {
        mbar_init(&bar, 1);
        init_item_queue(s_ctl);
    }
    load_weights<C, MODE, H, NH, false>(p, sm, L);
    __syncthreads();
    SegTab tab = seg_tab(sm + L.segi);
    uint32_t phase = 0;
    const float beta = p.mlp.softplus_beta;
    const int hact = p.mlp.hidden_activation, lact = p.mlp.last_activation;
    while (true) {
        const ItemInfo it = next_item(p, 0, sm, tab, &bar, s_ctl, false);
        if (it.slot < 0) break;
        const bool real = it.slot < p.ws.nslot;
        if (real && it.first) {
            if (!mbar_wait(&bar, phase)) {
                set_err(p.err, ATDF_DEVERR_TREE);
                mbar_wait(&bar, phase);
                return;
            }
            phase ^= 1;
        }
        for (int t0 = 0; t0 < it.total; t0 += kT) {
            const int k = t0 + s;
            const bool valid = k < it.total;
            float f[NF];
#pragma unroll
            for (int i = 0; i < NF; ++i) f[i] = 0.0f;
            float w = 0.0f, ts = 0.0f;
            int si = -1;
            if (valid) {
                const SampleState st = sample_state(p, tab, it, k);
                w = st.w;
                ts = st.t;
                si = st.si;
                if (real) {
                    const SampleGeo g = sample_geo_fast(p, tab, st.node, st.pos);
                    Gathered<CPT> ga;
                    gather_sample<C, CPT>(p, sm, g, q, ga);
                    features_of<C, MODE, CPT>(ga, f);
                }
            }
#pragma unroll
            for (int m = 0; m < (MODE ? 3 : 1); ++m)
#pragma unroll
                for (int cc = 0; cc < CPT; ++cc) sm[L.xt + feat_index<C, MODE, CPT>(q, m, cc) * kT + s] = f[m * CPT + cc];
            if (q == 0) {
                sm[L.sw + s] = w;
                reinterpret_cast<int*>(sm + L.sseg)[s] = si;
            }
            __syncthreads();
            {
                float acc[Map<kT, H>::RM][Map<kT, H>::CN];
                zero<kT, H>(acc);
                gemm<kT, H, true>(acc, sm + L.xt, kT, sm + L.w0t, H, F);
                store_layer<kT, H, true>(acc, sm + L.b0, hact, beta, sm + L.h0t, nullptr, nullptr);
            }
            __syncthreads();
            const float* hlast = sm + L.h0t;
            if (NH == 2) {
                float acc[Map<kT, H>::RM][Map<kT, H>::CN];
                zero<kT, H>(acc);
                gemm<kT, H, true>(acc, sm + L.h0t, kT, sm + L.w1t, H, H);
                store_layer<kT, H, true>(acc, sm + L.b1, hact, beta, sm + L.a1t, nullptr, nullptr);
                __syncthreads();
                hlast = sm + L.a1t;
            }
            const float z = last_layer<H>(hlast, sm + L.wl, sm[L.bl], s, q);
            if (q == 0 && valid) {
                const float rho = act_fwd(lact, z, beta);
                atomicAdd(&tab.acc[si], __fmul_rn(rho, w));
                if (p.bins) add_to_bins(p, tab, si, ts, __fmul_rn(rho, w));
            }
            __syncthreads();
        }
        if (tid < it.nseg) p.ws.seg_partial[tab.id[tid]] = tab.acc[tid];
        __syncthreads();
    }
}

template <int C, int MODE, int H, int NH>
__global__ void __launch_bounds__(kThreads, 1) fused_backward_kernel(FusedParams p)
{
    using K = Cfg<C, MODE, H, NH>;
    constexpr int F = K::F, CPT = K::CPT, NF = MODE ? 3 * CPT : CPT;
    extern __shared__ __align__(16) float sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int s_ctl[8];
    __shared__ int s_lo[3];
    const Smem<C, MODE, H, NH, true> L(p.plane_off[3]);
    const int tid = threadIdx.x;
    const int s = tid / kSPT, q = tid % kSPT;
    if (tid == 0) {
        mbar_init(&bar, 1);
        init_item_queue(s_ctl);
    }
    load_weights<C, MODE, H, NH, true>(p, sm, L);
    __syncthreads();
    SegTab tab = seg_tab(sm + L.segi);
    uint32_t phase = 0;
    const float beta = p.mlp.softplus_beta;
    const int hact = p.mlp.hidden_activation, lact = p.mlp.last_activation;
    const int plane_floats = p.plane_off[3];

    // decoder-gradient accumulators held across items
    float gW0[Map<H, F>::RM][Map<H, F>::CN];
    zero<H, F>(gW0);
    float gW1[Map<H, H>::RM][Map<H, H>::CN];
    zero<H, H>(gW1);
    constexpr int PARTS = kThreads / H;  // bias / last-layer partial sums
    constexpr int SPP = kT / PARTS;
    const int bn = tid % H, bpart = tid / H;
    float gb0 = 0.0f, gb1 = 0.0f, gwl = 0.0f;
    double gbl = 0.0;  // one scalar summed over every sample: FP64 against cancellation

    while (true) {
        const ItemInfo it = next_item(p, 1, sm, tab, &bar, s_ctl, true);
        if (it.slot < 0) break;
        const bool real = it.slot < p.ws.nslot;
        // a slot's first item: zero its gradient copy, set up the line windows
        if (real && it.first) {
            for (int i = tid * 4; i < plane_floats; i += kThreads * 4)
                *reinterpret_cast<float4*>(sm + L.gplanes + i) = make_float4(0.f, 0.f, 0.f, 0.f);
            for (int i = tid; i < 3 * kLineWin * C; i += kThreads) sm[L.gline + i] = 0.0f;
            if (tid < 3) {
                const float* bmin = tab.box;  // the item's leaf (segment 0's)
                const int Ln = p.field.line_len[tid];
                int lo = 0;
                if (Ln > kLineWin) {
                    const float u = tid == 0 ? roi_coord(bmin[0], p.field.roi_min[0], p.field.roi_max[0])
                                             : (tid == 2 ? bmin[2] : -1.0f);
                    lo = (int)floorf(((u + 1.0f) / 2.0f) * (float)(Ln - 1)) - 2;
                    lo = max(0, min(lo, Ln - kLineWin));
                }
                s_lo[tid] = lo;
            }
            if (!mbar_wait(&bar, phase)) {
                set_err(p.err, ATDF_DEVERR_TREE);
                mbar_wait(&bar, phase);
                return;
            }
            phase ^= 1;
        }
        __syncthreads();
        for (int t0 = 0; t0 < it.total; t0 += kT) {
            const int k = t0 + s;
            const bool valid = k < it.total;
            float f[NF];
#pragma unroll
            for (int i = 0; i < NF; ++i) f[i] = 0.0f;
            float w = 0.0f, dIw = 0.0f;
            SampleGeo g;
            if (valid) {
                const SampleState st = sample_state(p, tab, it, k);
                w = st.w;
                dIw = __fmul_rn(tab.acc[st.si], st.w);
                if (real) {
                    g = sample_geo_fast(p, tab, st.node, st.pos);
                    Gathered<CPT> ga;
                    gather_sample<C, CPT>(p, sm, g, q, ga);
                    features_of<C, MODE, CPT>(ga, f);
                }
            }
#pragma unroll
            for (int m = 0; m < (MODE ? 3 : 1); ++m)
#pragma unroll
                for (int cc = 0; cc < CPT; ++cc) {
                    const int fi = feat_index<C, MODE, CPT>(q, m, cc);
                    sm[L.xt + fi * kT + s] = f[m * CPT + cc];
                    sm[L.xs + s * F + fi] = f[m * CPT + cc];
                }
            if (q == 0) {
                sm[L.sw + s] = w;
                sm[L.sdi + s] = valid ? dIw : 0.0f;
            }
            __syncthreads();
            // ---- forward recompute ----
            {
                float acc[Map<kT, H>::RM][Map<kT, H>::CN];
                zero<kT, H>(acc);
                gemm<kT, H, true>(acc, sm + L.xt, kT, sm + L.w0t, H, F);
                store_layer<kT, H, true>(acc, sm + L.b0, hact, beta, sm + L.h0t, sm + L.a0t, sm + L.h0s);
            }
            __syncthreads();
            const float* hlast_s;
            if (NH == 2) {
                float acc[Map<kT, H>::RM][Map<kT, H>::CN];
                zero<kT, H>(acc);
                gemm<kT, H>(acc, sm + L.h0t, kT, sm + L.w1t, H, H);
                store_layer<kT, H>(acc, sm + L.b1, hact, beta, nullptr, sm + L.a1t, sm + L.h1s);
                __syncthreads();
                hlast_s = sm + L.h1s;
            } else {
                hlast_s = sm + L.h0s;
            }
            // last layer from the sample-major copy: z, dz
            {
                float acc = 0.0f;
#pragma unroll
                for (int i = 0; i < H / kSPT; ++i) {
                    const int kk = q + kSPT * i;
                    acc = fmaf(hlast_s[s * H + kk], sm[L.wl + kk], acc);
                }
                acc += __shfl_xor_sync(0xffffffffu, acc, 4);
                acc += __shfl_xor_sync(0xffffffffu, acc, 2);
                acc += __shfl_xor_sync(0xffffffffu, acc, 1);
                const float z = acc + sm[L.bl];
                if (q == 0) sm[L.sz + s] = sm[L.sdi + s] * act_grad(lact, z, beta);
            }
            __syncthreads();
            // last-layer gradients (partial sums per thread)
#pragma unroll
            for (int i = 0; i < SPP; ++i) {
                const int ss = bpart * SPP + i;
                gwl = fmaf(sm[L.sz + ss], hlast_s[ss * H + bn], gwl);
            }
            if (tid < kT) gbl += (double)sm[L.sz + tid];
            __syncthreads();
            // dA of the last hidden layer: dz * Wl * act'(pre); k-major (in
            // place of the pre-activation) and sample-major copies
            float* dAt = NH == 2 ? sm + L.a1t : sm + L.a0t;
            float* dAs = NH == 2 ? sm + L.h1s : sm + L.h0s;
            for (int e = tid; e < H * kT; e += kThreads) {
                const int n = e / kT, ss = e % kT;
                const float g = sm[L.sz + ss] * sm[L.wl + n] * act_grad(hact, dAt[e], beta);
                dAt[e] = g;
                dAs[ss * H + n] = g;
            }
            __syncthreads();
            if (NH == 2) {
                // dW1 += dA1^T H0 ; db1 ; dH0 = dA1 W1 -> dA0
                gemm<H, H>(gW1, sm + L.h1s, H, sm + L.h0s, H, kT);
#pragma unroll
                for (int i = 0; i < SPP; ++i) gb1 += sm[L.h1s + (bpart * SPP + i) * H + bn];
                float acc[Map<kT, H>::RM][Map<kT, H>::CN];
                zero<kT, H>(acc);
                gemm<kT, H>(acc, sm + L.a1t, kT, sm + L.w1, H, H);
                __syncthreads();
                using Mp = Map<kT, H>;
                const int tx = tid % Mp::TX, ty = tid / Mp::TX;
#pragma unroll
                for (int i = 0; i < Mp::RM; ++i)
#pragma unroll
                    for (int j = 0; j < Mp::CN; ++j) {
                        const int row = ty * Mp::RM + i, col = tx * Mp::CN + j;
                        const float g = acc[i][j] * act_grad(hact, sm[L.a0t + col * kT + row], beta);
                        sm[L.a0t + col * kT + row] = g;
                        sm[L.h0s + row * H + col] = g;
                    }
                __syncthreads();
            }
            // dW0 += dA0^T X ; db0 ; dX = dA0 W0
            gemm<H, F>(gW0, sm + L.h0s, H, sm + L.xs, F, kT);
#pragma unroll
            for (int i = 0; i < SPP; ++i) gb0 += sm[L.h0s + (bpart * SPP + i) * H + bn];
            {
                float acc[Map<kT, F>::RM][Map<kT, F>::CN];
                zero<kT, F>(acc);
                gemm<kT, F>(acc, sm + L.a0t, kT, sm + L.w0, F, H);
                __syncthreads();
                using Mp = Map<kT, F>;
                const int tx = tid % Mp::TX, ty = tid / Mp::TX;
#pragma unroll
                for (int i = 0; i < Mp::RM; ++i)
#pragma unroll
                    for (int j = 0; j < Mp::CN; ++j)
                        sm[L.xs + (ty * Mp::RM + i) * F + tx * Mp::CN + j] = acc[i][j];
            }
            __syncthreads();
            // scatter dX into the shared plane-gradient copy and line windows
            if (valid && real) {
                const int c0 = q * CPT;
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    const int Hm = p.field.plane_h[m], Wm = p.field.plane_w[m], Ln = p.field.line_len[m];
                    const Corner2 kc = corners2(g.pu[m], g.pv[m], Hm, Wm);
                    const Corner1 l = corners1(g.lu[m], Ln);
                    const float* P = sm + p.plane_off[m];
                    float* GP = sm + L.gplanes + p.plane_off[m];
                    const float* V = (const float*)p.field.line[m];
                    const int lo = s_lo[m];
#pragma unroll
                    for (int cc = 0; cc < CPT; ++cc) {
                        const int c = c0 + cc;
                        const float gf = sm[L.xs + s * F + (MODE ? m * C + c : c)];
                        const float mat = bilerp(kc, P[(kc.y0 * Wm + kc.x0) * C + c], P[(kc.y0 * Wm + kc.x1) * C + c],
                                                 P[(kc.y1 * Wm + kc.x0) * C + c], P[(kc.y1 * Wm + kc.x1) * C + c]);
                        const float vec = lerp1(l, __ldg(V + l.x0 * C + c), __ldg(V + l.x1 * C + c));
                        const float gm = __fmul_rn(gf, vec), gv = __fmul_rn(gf, mat);
                        atomicAdd(&GP[(kc.y0 * Wm + kc.x0) * C + c], __fmul_rn(kc.w_nw, gm));
                        atomicAdd(&GP[(kc.y0 * Wm + kc.x1) * C + c], __fmul_rn(kc.w_ne, gm));
                        atomicAdd(&GP[(kc.y1 * Wm + kc.x0) * C + c], __fmul_rn(kc.w_sw, gm));
                        atomicAdd(&GP[(kc.y1 * Wm + kc.x1) * C + c], __fmul_rn(kc.w_se, gm));
                        const int i0 = l.x0 - lo, i1 = l.x1 - lo;
                        const float g0 = __fmul_rn(l.w0, gv), g1 = __fmul_rn(l.w1, gv);
                        if (i0 >= 0 && i0 < kLineWin)
                            atomicAdd(&sm[L.gline + (m * kLineWin + i0) * C + c], g0);
                        else
                            atomicAdd(&p.gfield.line[m][l.x0 * C + c], g0);
                        if (i1 >= 0 && i1 < kLineWin)
                            atomicAdd(&sm[L.gline + (m * kLineWin + i1) * C + c], g1);
                        else
                            atomicAdd(&p.gfield.line[m][l.x1 * C + c], g1);
                    }
                }
            }
            __syncthreads();
        }
        // a slot's last item: store its plane gradients (this CTA owns the
        // slot) and flush the line windows
        if (real && it.last) {
            for (int m = 0; m < 3; ++m) {
                const int pf = p.field.plane_h[m] * p.field.plane_w[m] * C;
                float* dst = p.gfield.plane[m] + it.slot * (int64_t)pf;
                const float* src = sm + L.gplanes + p.plane_off[m];
                for (int i = tid * 4; i < pf; i += kThreads * 4)
                    *reinterpret_cast<float4*>(dst + i) = *reinterpret_cast<const float4*>(src + i);
                const int Ln = p.field.line_len[m];
                const int lo = s_lo[m];
                for (int i = tid; i < kLineWin * C; i += kThreads) {
                    const int e = lo + i / C;
                    const float v = sm[L.gline + m * kLineWin * C + i];
                    if (e < Ln && v != 0.0f) atomicAdd(&p.gfield.line[m][e * C + (i % C)], v);
                }
            }
        }
        __syncthreads();
    }

    // flush the decoder gradients
    {
        using Mp = Map<H, F>;
        const int tx = tid % Mp::TX, ty = tid / Mp::TX;
#pragma unroll
        for (int i = 0; i < Mp::RM; ++i)
#pragma unroll
            for (int j = 0; j < Mp::CN; ++j)
                atomicAdd(&p.gmlp.weight[0][(ty * Mp::RM + i) * F + tx * Mp::CN + j], gW0[i][j]);
    }
    if (NH == 2) {
        using Mp = Map<H, H>;
        const int tx = tid % Mp::TX, ty = tid / Mp::TX;
#pragma unroll
        for (int i = 0; i < Mp::RM; ++i)
#pragma unroll
            for (int j = 0; j < Mp::CN; ++j)
                atomicAdd(&p.gmlp.weight[1][(ty * Mp::RM + i) * H + tx * Mp::CN + j], gW1[i][j]);
        atomicAdd(&p.gmlp.bias[1][bn], gb1);
    }
    atomicAdd(&p.gmlp.bias[0][bn], gb0);
    atomicAdd(&p.gmlp.weight[NH][bn], gwl);
    static_assert(kT == 32, "the last-layer bias partials live in warp 0");
    if (tid < 32) {
        for (int off = 16; off > 0; off >>= 1) gbl += __shfl_down_sync(0xffffffffu, gbl, off);
        if (tid == 0) atomicAdd(&p.gmlp.bias[NH][0], (float)gbl);
    }
}

// ---------------------------------------------------------------------------
// node-error scoring: one warp per segment, FP64 sums
// ---------------------------------------------------------------------------
__global__ void node_error_kernel(Ws w, const float* __restrict__ prl, int cout, int64_t R, uint64_t seed,
                                  double* ls, double* wsum, int64_t num_nodes, int32_t* err)
{
    const int lane = threadIdx.x & 31;
    const int64_t nseg = min(w.totals[0], w.cap);
    for (int64_t sidx = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; sidx < nseg;
         sidx += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int n = w.nsamp[sidx], node = w.node[sidx], r = w.ray[sidx];
        const float tmin = w.tmin[sidx], tmax = w.tmax[sidx];
        double acc = 0.0;
        for (int j = lane; j < n; j += 32) {
            const float t = sample_t(tmin, tmax, n, j, sample_a(nullptr, 0, seed, r, node, j));
            const float tp = j > 0 ? sample_t(tmin, tmax, n, j - 1, sample_a(nullptr, 0, seed, r, node, j - 1)) : 0.f;
            const float tn = j < n - 1 ? sample_t(tmin, tmax, n, j + 1, sample_a(nullptr, 0, seed, r, node, j + 1))
                                       : 0.f;
            acc += (double)sample_w(tmin, tmax, n, j, tp, t, tn);
        }
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (lane == 0) {
            if (node < 0 || node >= num_nodes) {
                set_err(err, ATDF_DEVERR_INDEX);
                continue;
            }
            double l = 0.0;
            for (int c = 0; c < cout; ++c) l += (double)prl[c * R + r];
            l /= (double)cout;
            atomicAdd(&ls[node], l * acc);
            atomicAdd(&wsum[node], acc);
        }
    }
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
using KernelFn = void (*)(FusedParams);

struct Variant {
    int C, mode, H, NH;
    KernelFn fwd, bwd;
    int (*smem)(int, bool);
};

template <int C, int MODE, int H, int NH>
static int smem_bytes(int plane_floats, bool bwd)
{
    if (bwd) return Smem<C, MODE, H, NH, true>(plane_floats).total * 4;
    return Smem<C, MODE, H, NH, false>(plane_floats).total * 4;
}

#define ATDF_VARIANT(C, M, H, NH) \
    {C, M, H, NH, fused_forward_kernel<C, M, H, NH>, fused_backward_kernel<C, M, H, NH>, smem_bytes<C, M, H, NH>}

static const Variant kVariants[] = {
    ATDF_VARIANT(8, 0, 32, 1),  ATDF_VARIANT(8, 0, 64, 1),  ATDF_VARIANT(8, 0, 64, 2),
    ATDF_VARIANT(16, 0, 32, 1), ATDF_VARIANT(16, 0, 64, 1), ATDF_VARIANT(16, 0, 64, 2),
    ATDF_VARIANT(8, 1, 64, 2),  ATDF_VARIANT(8, 1, 32, 1),
};

static const Variant* find_variant(const atdf_field_t* f, const atdf_mlp_t* m)
{
    const int nh = m->num_layers - 1;
    if (nh < 1 || nh > 2 || m->dims[m->num_layers] != 1) return nullptr;
    const int H = m->dims[1];
    if (nh == 2 && m->dims[2] != H) return nullptr;
    const int F = f->mode ? 3 * f->channels : f->channels;
    if (m->dims[0] != F) return nullptr;
    for (const Variant& v : kVariants)
        if (v.C == f->channels && v.mode == f->mode && v.H == H && v.NH == nh) return &v;
    return nullptr;
}

static int max_smem_optin()
{
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

static int prepare(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp, const float* origin,
                   const float* dir, int64_t R, void* workspace, size_t ws_bytes, FusedParams& p,
                   const Variant*& var)
{
    if (!tree || !field || !mlp || !workspace || R < 0 || (R > 0 && (!origin || !dir)))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (!field->leaf_slot) return ATDF_ERR_INVALID_ARGUMENT;
    var = nullptr;
    if (field->dtype == ATDF_BF16) {
        if (!tc_supported(field, mlp)) return ATDF_ERR_UNSUPPORTED;
    } else if (field->dtype == ATDF_F32) {
        var = find_variant(field, mlp);
        if (!var) return ATDF_ERR_UNSUPPORTED;
    } else {
        return ATDF_ERR_UNSUPPORTED;
    }
    for (int l = 0; l < mlp->num_layers; ++l)
        if (!mlp->weight[l] || !mlp->bias[l]) return ATDF_ERR_INVALID_ARGUMENT;
    // The 16-channel BF16 tensor-core kernels keep each plane in shared
    // memory with rows padded to a pitch of 2 mod 4 texels (texel = 16
    // channels = 32 bytes): the four corners of a bilinear footprint then
    // have texel indices of all four residues mod 4 and fill distinct bank
    // groups. The 24-channel ones keep the planes unpadded.
    int off = 0, goff = 0;
    for (int m = 0; m < 3; ++m) {
        if (!field->plane[m] || !field->line[m] || ((uintptr_t)field->plane[m] & 15) ||
            ((uintptr_t)field->line[m] & 15))
            return ATDF_ERR_UNSUPPORTED;
        const int W = field->plane_w[m];
        p.plane_pitch[m] = (field->dtype == ATDF_BF16 && field->channels == 16) ? W + ((2 - W) & 3) : W;
        p.plane_off[m] = off;
        off += field->plane_h[m] * p.plane_pitch[m] * field->channels;
        p.gplane_off[m] = goff;
        goff += field->plane_h[m] * W * field->channels;
    }
    p.plane_off[3] = off;
    p.gplane_off[3] = goff;
    p.roi_inv = pow2_reciprocal(field->roi_max[0] - field->roi_min[0]);
    const size_t need = ws_layout(R, tree->max_depth, field->num_slots, nullptr, nullptr);
    if (ws_bytes < need) return ATDF_ERR_WORKSPACE;
    ws_layout(R, tree->max_depth, field->num_slots, (char*)workspace, &p.ws);
    p.tree = *tree;
    p.field = *field;
    p.mlp = *mlp;
    p.origin = origin;
    p.dir = dir;
    p.R = R;
    p.grad_image = nullptr;
    p.xt = nullptr;
    p.xw = nullptr;
    p.bins = nullptr;
    return ATDF_OK;
}

static int launch_persistent(KernelFn fn, int smem, const FusedParams& p, cudaStream_t st)
{
    if (smem > max_smem_optin()) return ATDF_ERR_UNSUPPORTED;
    ATDF_CUDA_TRY(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ATDF_CUDA_TRY(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared));
    int dev = 0, sms = 0, per = 0;
    ATDF_CUDA_TRY(cudaGetDevice(&dev));
    ATDF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    ATDF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)fn, kThreads, smem));
    if (per < 1) return ATDF_ERR_UNSUPPORTED;
    fn<<<sms * per, kThreads, smem, st>>>(p);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}


// Forward projection. compute_segments: derive the ray/leaf segments (and the
// uniform per-node sample counts) into the workspace; otherwise use the
// segments already there (atdf_project_segments) with caller-placed samples.
static int project_forward(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                           const float* ray_origin, const float* ray_direction, int64_t num_rays,
                           int32_t max_samples_per_node, uint64_t jitter_seed, bool compute_segments,
                           const float* xt, const float* xw, float* bins, float* image, void* workspace,
                           size_t workspace_bytes, int32_t* dev_error, cudaStream_t s)
{
    FusedParams p;
    const Variant* var = nullptr;
    int st = prepare(tree, field, mlp, ray_origin, ray_direction, num_rays, workspace, workspace_bytes, p, var);
    if (st != ATDF_OK) return st;
    if (!image) return ATDF_ERR_INVALID_ARGUMENT;
    if (num_rays >= ((int64_t)1 << 31)) return ATDF_ERR_UNSUPPORTED;
    p.seed = jitter_seed;
    p.err = dev_error;
    p.xt = xt;
    p.xw = xw;
    p.bins = bins;
    const Ws& w = p.ws;
    if (compute_segments) {
        st = launch_ray_segments_ws(*tree, ray_origin, ray_direction, num_rays, max_samples_per_node, w, dev_error,
                                    s);
        if (st != ATDF_OK) return st;
    }
    if (bins) ATDF_CUDA_TRY(cudaMemsetAsync(bins, 0, (size_t)w.cap * kBins * sizeof(float), s));
    ATDF_CUDA_TRY(cudaMemsetAsync(w.slot_offset, 0, (w.nslot + 2) * 4, s));
    ATDF_CUDA_TRY(cudaMemsetAsync(w.slot_cursor, 0, (w.nslot + 1) * 4, s));
    ATDF_CUDA_TRY(cudaMemsetAsync(w.counters, 0, 8 * 4, s));
    bucket_count_kernel<<<592, 256, 0, s>>>(w, *field, tree->num_nodes, dev_error);
    ATDF_LAUNCH_CHECK();
    scan_exclusive_i32_kernel<<<1, 1024, 0, s>>>(w.slot_offset, w.nslot + 2, nullptr);
    ATDF_LAUNCH_CHECK();
    bucket_scatter_kernel<<<592, 256, 0, s>>>(w, *field, tree->num_nodes);
    ATDF_LAUNCH_CHECK();
    item_count_kernel<<<(unsigned)div_up(w.nslot + 2, 256), 256, 0, s>>>(w);
    ATDF_LAUNCH_CHECK();
    slot_order_kernel<<<1, 1024, 0, s>>>(w);
    ATDF_LAUNCH_CHECK();
    scan_exclusive_i32_kernel<<<1, 1024, 0, s>>>(w.item_offset, w.nslot + 2, nullptr);
    ATDF_LAUNCH_CHECK();
    if (!var) {  // the tensor-core forwards take work by item
        item_queue_kernel<<<1, 1024, 0, s>>>(w);
        ATDF_LAUNCH_CHECK();
    }
    st = var ? launch_persistent(var->fwd, var->smem(p.plane_off[3], false), p, s) : launch_tc_forward(p, s);
    if (st != ATDF_OK) return st;
    if (num_rays > 0) {
        ray_reduce_kernel<<<(unsigned)div_up(num_rays, 256), 256, 0, s>>>(w, num_rays, image);
        ATDF_LAUNCH_CHECK();
    }
    return ATDF_OK;
}

// Backward (recomputes every sample; reuses the forward's workspace).
static int project_backward(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                            const float* ray_origin, const float* ray_direction, int64_t num_rays,
                            uint64_t jitter_seed, const float* xt, const float* xw, const float* grad_image,
                            const atdf_field_grad_t* grad_field, const atdf_mlp_grad_t* grad_mlp, void* workspace,
                            size_t workspace_bytes, int32_t* dev_error, cudaStream_t s)
{
    FusedParams p;
    const Variant* var = nullptr;
    int st = prepare(tree, field, mlp, ray_origin, ray_direction, num_rays, workspace, workspace_bytes, p, var);
    if (st != ATDF_OK) return st;
    if (!grad_image || !grad_field || !grad_mlp) return ATDF_ERR_INVALID_ARGUMENT;
    for (int m = 0; m < 3; ++m)
        if (!grad_field->plane[m] || !grad_field->line[m] || ((uintptr_t)grad_field->plane[m] & 15))
            return ATDF_ERR_INVALID_ARGUMENT;
    for (int l = 0; l < mlp->num_layers; ++l)
        if (!grad_mlp->weight[l] || !grad_mlp->bias[l]) return ATDF_ERR_INVALID_ARGUMENT;
    p.seed = jitter_seed;
    p.err = dev_error;
    p.grad_image = grad_image;
    p.gfield = *grad_field;
    p.gmlp = *grad_mlp;
    p.xt = xt;
    p.xw = xw;
    for (int m = 0; m < 3; ++m) {
        // the tensor-core backward writes the plane gradient of every slot
        // it touches (zeroing it first) and the rest is zeroed below
        if (var) {
            const size_t pf = (size_t)field->plane_h[m] * field->plane_w[m] * field->channels * field->num_slots;
            ATDF_CUDA_TRY(cudaMemsetAsync(grad_field->plane[m], 0, pf * 4, s));
        }
        ATDF_CUDA_TRY(
            cudaMemsetAsync(grad_field->line[m], 0, (size_t)field->line_len[m] * field->channels * 4, s));
    }
    if (!var && p.ws.nslot > 0) {
        zero_untouched_slots_kernel<<<(unsigned)std::min<int64_t>(p.ws.nslot, 592), 256, 0, s>>>(p.ws, *grad_field,
                                                                                                *field);
        ATDF_LAUNCH_CHECK();
    }
    for (int l = 0; l < mlp->num_layers; ++l) {
        ATDF_CUDA_TRY(cudaMemsetAsync(grad_mlp->weight[l], 0, (size_t)mlp->dims[l] * mlp->dims[l + 1] * 4, s));
        ATDF_CUDA_TRY(cudaMemsetAsync(grad_mlp->bias[l], 0, (size_t)mlp->dims[l + 1] * 4, s));
    }
    ATDF_CUDA_TRY(cudaMemsetAsync(p.ws.counters + 1, 0, 4, s));
    return var ? launch_persistent(var->bwd, var->smem(p.plane_off[3], true), p, s) : launch_tc_backward(p, s);
}

}  // namespace atdf

using namespace atdf;

extern "C" {

int atdf_project_workspace_size(int64_t num_rays, int32_t max_depth, int32_t ns, int64_t num_slots,
                                int32_t out_channels, size_t* bytes)
{
    if (!bytes || num_rays < 0 || max_depth < 0 || num_slots < 0 || (ns != 4 && ns != 8) || out_channels != 1)
        return ATDF_ERR_INVALID_ARGUMENT;
    *bytes = ws_layout(num_rays, max_depth, num_slots, nullptr, nullptr);
    return ATDF_OK;
}

int atdf_project_forward(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                         const float* ray_origin, const float* ray_direction, int64_t num_rays,
                         int32_t max_samples_per_node, uint64_t jitter_seed, float* image, void* workspace,
                         size_t workspace_bytes, int32_t* dev_error, atdf_stream_t stream)
{
    return project_forward(tree, field, mlp, ray_origin, ray_direction, num_rays, max_samples_per_node, jitter_seed,
                           true, nullptr, nullptr, nullptr, image, workspace, workspace_bytes, dev_error,
                           (cudaStream_t)stream);
}

int atdf_project_forward_segmented(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                                   const float* ray_origin, const float* ray_direction, int64_t num_rays,
                                   uint64_t jitter_seed, float* image, void* workspace, size_t workspace_bytes,
                                   int32_t* dev_error, atdf_stream_t stream)
{
    return project_forward(tree, field, mlp, ray_origin, ray_direction, num_rays, 0, jitter_seed, false, nullptr,
                           nullptr, nullptr, image, workspace, workspace_bytes, dev_error, (cudaStream_t)stream);
}

int atdf_project_forward_binned(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                                const float* ray_origin, const float* ray_direction, int64_t num_rays,
                                int32_t max_samples_per_node, uint64_t jitter_seed, float* image, float* seg_bins,
                                void* workspace, size_t workspace_bytes, int32_t* dev_error, atdf_stream_t stream)
{
    if (!seg_bins) return ATDF_ERR_INVALID_ARGUMENT;
    return project_forward(tree, field, mlp, ray_origin, ray_direction, num_rays, max_samples_per_node, jitter_seed,
                           true, nullptr, nullptr, seg_bins, image, workspace, workspace_bytes, dev_error,
                           (cudaStream_t)stream);
}

int atdf_project_segments(const atdf_tree_t* tree, const float* ray_origin, const float* ray_direction,
                          int64_t num_rays, int32_t max_samples_per_node, int64_t num_slots, void* workspace,
                          size_t workspace_bytes, atdf_segments_t* view, int32_t* dev_error, atdf_stream_t stream)
{
    if (!tree || !workspace || !view || num_rays < 0 || num_slots < 0 ||
        (num_rays > 0 && (!ray_origin || !ray_direction)))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (num_rays >= ((int64_t)1 << 31)) return ATDF_ERR_UNSUPPORTED;
    const size_t need = ws_layout(num_rays, tree->max_depth, num_slots, nullptr, nullptr);
    if (workspace_bytes < need) return ATDF_ERR_WORKSPACE;
    Ws w;
    ws_layout(num_rays, tree->max_depth, num_slots, (char*)workspace, &w);
    *view = ws_segments(w);
    return launch_ray_segments_ws(*tree, ray_origin, ray_direction, num_rays, max_samples_per_node, w, dev_error,
                                  (cudaStream_t)stream);
}

int atdf_project_segment_view(int64_t num_rays, int32_t max_depth, int64_t num_slots, void* workspace,
                              size_t workspace_bytes, atdf_segments_t* view)
{
    if (!workspace || !view || num_rays < 0 || max_depth < 0 || num_slots < 0) return ATDF_ERR_INVALID_ARGUMENT;
    const size_t need = ws_layout(num_rays, max_depth, num_slots, nullptr, nullptr);
    if (workspace_bytes < need) return ATDF_ERR_WORKSPACE;
    Ws w;
    ws_layout(num_rays, max_depth, num_slots, (char*)workspace, &w);
    *view = ws_segments(w);
    return ATDF_OK;
}

int atdf_project_forward_samples(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                                 const float* ray_origin, const float* ray_direction, int64_t num_rays,
                                 const float* sample_t, const float* sample_w, float* image, void* workspace,
                                 size_t workspace_bytes, int32_t* dev_error, atdf_stream_t stream)
{
    if (num_rays > 0 && (!sample_t || !sample_w)) return ATDF_ERR_INVALID_ARGUMENT;
    return project_forward(tree, field, mlp, ray_origin, ray_direction, num_rays, 0, 0, false, sample_t, sample_w,
                           nullptr, image, workspace, workspace_bytes, dev_error, (cudaStream_t)stream);
}

int atdf_project_backward(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                          const float* ray_origin, const float* ray_direction, int64_t num_rays,
                          int32_t max_samples_per_node, uint64_t jitter_seed, const float* grad_image,
                          const atdf_field_grad_t* grad_field, const atdf_mlp_grad_t* grad_mlp, void* workspace,
                          size_t workspace_bytes, int32_t* dev_error, atdf_stream_t stream)
{
    (void)max_samples_per_node;
    return project_backward(tree, field, mlp, ray_origin, ray_direction, num_rays, jitter_seed, nullptr, nullptr,
                            grad_image, grad_field, grad_mlp, workspace, workspace_bytes, dev_error,
                            (cudaStream_t)stream);
}

int atdf_project_backward_samples(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                                  const float* ray_origin, const float* ray_direction, int64_t num_rays,
                                  const float* sample_t, const float* sample_w, const float* grad_image,
                                  const atdf_field_grad_t* grad_field, const atdf_mlp_grad_t* grad_mlp,
                                  void* workspace, size_t workspace_bytes, int32_t* dev_error, atdf_stream_t stream)
{
    if (num_rays > 0 && (!sample_t || !sample_w)) return ATDF_ERR_INVALID_ARGUMENT;
    return project_backward(tree, field, mlp, ray_origin, ray_direction, num_rays, 0, sample_t, sample_w, grad_image,
                            grad_field, grad_mlp, workspace, workspace_bytes, dev_error, (cudaStream_t)stream);
}

int atdf_project_node_error(const atdf_tree_t* tree, const float* ray_origin, const float* ray_direction,
                            int64_t num_rays, int32_t max_samples_per_node, uint64_t jitter_seed,
                            const float* per_ray_loss, int32_t out_channels, double* loss_sum, double* weight_sum,
                            void* workspace, size_t workspace_bytes, int32_t* dev_error, atdf_stream_t stream)
{
    (void)ray_origin;
    (void)ray_direction;
    (void)max_samples_per_node;
    if (!tree || !per_ray_loss || !loss_sum || !weight_sum || !workspace || out_channels <= 0 || num_rays < 0)
        return ATDF_ERR_INVALID_ARGUMENT;
    Ws w;
    // the slot count does not move the segment arrays; any value gives them
    const size_t need = ws_layout(num_rays, tree->max_depth, 0, nullptr, nullptr);
    if (workspace_bytes < need) return ATDF_ERR_WORKSPACE;
    ws_layout(num_rays, tree->max_depth, 0, (char*)workspace, &w);
    cudaStream_t s = (cudaStream_t)stream;
    ATDF_CUDA_TRY(cudaMemsetAsync(loss_sum, 0, tree->num_nodes * sizeof(double), s));
    ATDF_CUDA_TRY(cudaMemsetAsync(weight_sum, 0, tree->num_nodes * sizeof(double), s));
    node_error_kernel<<<1184, 256, 0, s>>>(w, per_ray_loss, out_channels, num_rays, jitter_seed, loss_sum, weight_sum,
                                           tree->num_nodes, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

}  // extern "C"
