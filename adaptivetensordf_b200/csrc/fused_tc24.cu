// Fused leaf-major projection with BF16 factor planes and the decoder on the
// 5th-generation tensor cores, forward and hand-written adjoint, for 24
// channels ("add", rank-24 VM): decoder 24 -> 64 -> 64 -> 1 (the reference's
// FCBlock default with one hidden layer of 64 over the 24 VM features;
// hyperacorn/csrc/geometry/Modules.h:68-109, feature count from
// grid_features, geometry_tensor_qo.cpp:10-36).
//
// The tile pipeline is the one of the 16-channel kernels (fused_tc.cu) with
// two changes forced by the wider texel:
//   * K of the first layer and N of its adjoint (dX) are padded from 24 to 32
//     channels: the feature buffer holds X in columns 64..87, a ones column
//     at 88 (bias gradients through the weight-gradient MMA) and zeros up to
//     95; W0 is kept as [64][32] with zero columns 24..31. The padding adds
//     exact zeros, so the result equals the 24-channel product.
//   * The backward keeps the slot's planes (41.6 KB) and their fixed-point
//     gradient copy (83 KB) in shared memory, which leaves room for one
//     128-row tile at a time, with three threads per sample row (384
//     threads). Thread group g of a row owns the 8 channels [8g, 8g + 8) (one
//     16-byte piece of a 48-byte texel) in the feature gather and scatters
//     them to all four bilinear corners itself, so no per-row scratch is
//     shared between the threads; groups 0 and 1 also own the hidden columns
//     [32g, 32g + 32) of the decoder's epilogues, while group 2 waits.
// The line-gradient MMA has N = 72 columns padded to 80 (the columns past 72
// of its output are not read).

#include <cuda_bf16.h>

#include "fused_common.cuh"
#include "tc.cuh"
#include "tc_common.cuh"

namespace atdf {
namespace tc24 {

using tcf::corner_texel;
using tcf::ld16;
using tcf::pack_bf16;
using tcf::sigmoid_tanh;
using tcf::silu;
using tcf::silu_grad;
using tcf::store_bf16x8;
using tcf::trow;
using tcf::unpack_bf16x8;
using tcf::wait_mma;

constexpr int kC = 24;
constexpr int kCP = 32;          // channels padded to a multiple of 16 (K of layer 0, N of dX)
constexpr int kH = 64;
constexpr int kRows = 128;       // samples per tile
constexpr int kHBCols = 96;      // backward feature buffer: H0 (64) | X (24) | ones | zero pad
constexpr int kHBColsF = 64;     // forward: X in columns 0..31 (24..31 zero), then H0 over it
constexpr int kXCol = 64;
constexpr int kOnesCol = 88;
constexpr int kGCols = 128;      // dA1 (64) | dA0 (64)
// The backward keeps a window of kLineRows rows of each line per slot: the
// rows of the line values it reads (staged in shared memory) and of the line
// gradients it accumulates (in TMEM, by the line MMA). A leaf of depth d spans
// 256 / 2^d cells of a 256-entry line, so 40 rows cover depth-3 leaves (32
// cells, both taps and a rounding margin); samples outside the window read
// and add to global memory. Line m's taps are columns 40 m .. 40 m + 39 of the
// line MMA's A operand: five 16-byte groups, which thread group m zeroes and
// fills for its row.
constexpr int kLineRows = 40;    // 3 x 40 = 120 <= 128 rows of the line MMA
constexpr int kLineN = 80;       // N of the line-gradient MMA (3 * 24 = 72, padded)
constexpr int kThreadsF = 256;   // forward: two halves of 128 rows, one thread per row
constexpr int kThreadsB = 384;   // backward: one half of 128 rows, three threads per row
// The shared fixed-point gradient keeps each texel's 24 channels at a pitch
// of 25 words: texel * 24 mod 32 takes only 4 values, so the atomics of a
// warp (random texels, one channel) would meet in 4 banks; with an odd pitch
// they spread over all 32.
constexpr int kGP = 25;
constexpr int kMapCapF = 2048;    // forward: items of up to this many samples use the byte map
constexpr uint32_t kTmemF = 256;  // columns per forward CTA (two CTAs per SM)
constexpr uint32_t kTmemB = 512;  // columns per backward CTA (one CTA per SM)

__device__ __forceinline__ uint32_t hb_off(int s, int c) { return tc::mnmajor_off(c, s, kHBCols); }
__device__ __forceinline__ uint32_t hbf_off(int s, int c) { return tc::mnmajor_off(c, s, kHBColsF); }
__device__ __forceinline__ uint32_t g_off(int s, int c) { return tc::mnmajor_off(c, s, kGCols); }
__device__ __forceinline__ uint32_t w0_off(int n, int f) { return tc::kmajor_off(n, f, kCP); }
__device__ __forceinline__ uint32_t w1_off(int n, int k) { return tc::kmajor_off(n, k, kH); }

struct Smem24 {
    uint32_t planes, w0, w1, bias, hb[2], g, gplanes, lwin, segi, total;
    // gplane_elems: the unpadded plane-gradient elements (texels x 24)
    __host__ __device__ Smem24(int plane_elems, int gplane_elems, bool bwd)
    {
        auto al = [](uint32_t x) { return (x + 127u) & ~127u; };
        uint32_t o = 0;
        planes = o;
        o = al(o + plane_elems * 2);
        w0 = o;
        o = al(o + kH * kCP * 2);
        w1 = o;
        o = al(o + kH * kH * 2);
        bias = o;  // b0[64] b1[64] w2[64] b2
        o = al(o + (3 * kH + 4) * 4);
        hb[0] = o;
        o = al(o + kRows * (bwd ? kHBCols : kHBColsF) * 2);
        hb[1] = o;
        if (!bwd) o = al(o + kRows * kHBColsF * 2);
        g = o;
        if (bwd) o = al(o + kRows * kGCols * 2);
        gplanes = o;
        if (bwd) o = al(o + ((gplane_elems / kC * kGP + 3) & ~3) * 4);
        lwin = o;  // BF16 rows of the slot's line windows
        o = al(o + 3 * kLineRows * kC * 2);
        segi = o;
        // the forward's table keeps a sample -> segment map of kMapCapF
        // samples only, which lets two forward CTAs share an SM
        o = al(o + (bwd ? kSegTabFloats : kSegTabFloats - (kSegMapCap - kMapCapF) / 4) * 4);
        total = o;
    }
};

__device__ __forceinline__ void load_weights(const FusedParams& p, unsigned char* sm, const Smem24& L)
{
    const atdf_mlp_t& m = p.mlp;
    for (int i = threadIdx.x; i < kH * kCP; i += blockDim.x) {
        const int n = i / kCP, f = i % kCP;
        const float v = f < kC ? m.weight[0][n * kC + f] : 0.0f;
        *reinterpret_cast<__nv_bfloat16*>(sm + L.w0 + w0_off(n, f)) = __float2bfloat16_rn(v);
    }
    for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) {
        const int n = i / kH, k = i % kH;
        *reinterpret_cast<__nv_bfloat16*>(sm + L.w1 + w1_off(n, k)) = __float2bfloat16_rn(m.weight[1][i]);
    }
    float* bias = reinterpret_cast<float*>(sm + L.bias);
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        bias[i] = m.bias[0][i];
        bias[kH + i] = m.bias[1][i];
        bias[2 * kH + i] = m.weight[2][i];
    }
    if (threadIdx.x == 0) bias[3 * kH] = m.bias[2][0];
}

// Columns 88..95 of a feature buffer: the ones column (used by the
// weight-gradient MMA; zero weight in W0) and zeros.
__device__ __forceinline__ void init_pad_columns(unsigned char* hb, int rows_per_thread_start, int stride)
{
    for (int s = rows_per_thread_start; s < kRows; s += stride) {
        float v[8] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        store_bf16x8(hb + hb_off(s, kOnesCol), v);
    }
}

// Layer 0 (K = 32 over X | ones | zeros, or X | zeros; W0's columns 24..31
// are zero) of a feature buffer of COLS columns with X at column XCOL.
template <int COLS, int XCOL>
__device__ __forceinline__ void issue_l0(const unsigned char* sm, const Smem24& L, uint32_t hb, uint32_t d0)
{
    const uint32_t abase = tc::smem_addr(sm + hb + (XCOL / 8) * 128), bbase = tc::smem_addr(sm + L.w0);
#pragma unroll
    for (int j = 0; j < kCP / 16; ++j) {
        const uint64_t a = tc::smem_desc(abase + j * 256, 128, (COLS / 8) * 128);
        const uint64_t b = tc::smem_desc(bbase + j * 256, 128, (kCP / 8) * 128);
        tc::mma_bf16(d0, a, b, tc::idesc_bf16(kRows, kH, 0, 0), j > 0);
    }
}

template <int COLS>
__device__ __forceinline__ void issue_l1(const unsigned char* sm, const Smem24& L, uint32_t hb, uint32_t d1)
{
    const uint32_t abase = tc::smem_addr(sm + hb), bbase = tc::smem_addr(sm + L.w1);
#pragma unroll
    for (int j = 0; j < kH / 16; ++j) {
        const uint64_t a = tc::smem_desc(abase + j * 256, 128, (COLS / 8) * 128);
        const uint64_t b = tc::smem_desc(bbase + j * 256, 128, (kH / 8) * 128);
        tc::mma_bf16(d1, a, b, tc::idesc_bf16(kRows, kH, 0, 0), j > 0);
    }
}

// ---------------------------------------------------------------------------
// forward: one thread per sample row, two halves of 128 rows
// ---------------------------------------------------------------------------
__device__ __forceinline__ void half_barrier(int h) { asm volatile("bar.sync %0, 128;" ::"r"(1 + h) : "memory"); }

// First row of line m's window for the slot whose leaf box (min, size) is
// `box`: two rows below the leaf's first cell, clamped to the line.
__device__ __forceinline__ int line_window_lo(const FusedParams& p, const float* box, int m)
{
    const int Ln = p.field.line_len[m];
    if (Ln <= kLineRows) return 0;
    // x line: the ROI-normalised x; z line: the raw z; y line: the local y
    const float u = m == 0 ? roi_coord(box[0], p.field.roi_min[0], p.field.roi_max[0]) : (m == 2 ? box[2] : -1.0f);
    const int lo = (int)floorf(((u + 1.0f) * 0.5f) * (float)(Ln - 1)) - 2;
    return max(0, min(lo, Ln - kLineRows));
}

// Stages rows lo .. lo + kLineRows - 1 of each line (3 x 16 bytes per row)
// into LW and records lo in s_lo (the item's leaf box is segment 0's).
__device__ __forceinline__ void stage_line_windows(const FusedParams& p, const float* box, unsigned char* LW,
                                                   int* s_lo)
{
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        const int lo = line_window_lo(p, box, m);
        if (threadIdx.x == 0) s_lo[m] = lo;
        const int n16 = 3 * min(kLineRows, p.field.line_len[m] - lo);
        const uint4* src = reinterpret_cast<const uint4*>(reinterpret_cast<const unsigned char*>(p.field.line[m]) +
                                                          (size_t)lo * (kC * 2));
        uint4* dst = reinterpret_cast<uint4*>(LW + m * (kLineRows * kC * 2));
        for (int i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = __ldg(src + i);
    }
}

// VM feature of one sample, all 24 channels: planes (BF16, shared memory) and
// lines (BF16, the slot's window in shared memory when both taps are inside
// it, else global), plane 2 first, corners in order.
__device__ __forceinline__ void gather24(const FusedParams& p, const unsigned char* sm, const unsigned char* LW,
                                         const int* s_lo, const SampleGeo& g, float (&f)[kC])
{
#pragma unroll
    for (int m = 2; m >= 0; --m) {
        const int Hm = p.field.plane_h[m], Wm = p.field.plane_w[m], L = p.field.line_len[m];
        const int Wp = p.plane_pitch[m];
        const Corner2 k = corners2(g.pu[m], g.pv[m], Hm, Wm);
        const Corner1 l = corners1(g.lu[m], L);
        const unsigned char* P = sm + (size_t)p.plane_off[m] * 2;
        const int r0 = l.x0 - s_lo[m], r1 = l.x1 - s_lo[m];
        const bool inwin = (unsigned)r0 < (unsigned)kLineRows && (unsigned)r1 < (unsigned)kLineRows;
        const unsigned char* V0 = inwin ? LW + (size_t)m * (kLineRows * kC * 2) + r0 * (kC * 2)
                                        : reinterpret_cast<const unsigned char*>(p.field.line[m]) + l.x0 * (kC * 2);
        const unsigned char* V1 = inwin ? LW + (size_t)m * (kLineRows * kC * 2) + r1 * (kC * 2)
                                        : reinterpret_cast<const unsigned char*>(p.field.line[m]) + l.x1 * (kC * 2);
        float ma[kC];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float w;
            const unsigned char* tx = P + corner_texel(k, j, Wp, w) * (kC * 2);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                float u[8];
                unpack_bf16x8(*reinterpret_cast<const uint4*>(tx + 16 * q), u);
#pragma unroll
                for (int i = 0; i < 8; ++i) ma[8 * q + i] = j == 0 ? u[i] * w : fmaf(u[i], w, ma[8 * q + i]);
            }
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            float v0[8], v1[8];
            unpack_bf16x8(*reinterpret_cast<const uint4*>(V0 + 16 * q), v0);
            unpack_bf16x8(*reinterpret_cast<const uint4*>(V1 + 16 * q), v1);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const float ve = fmaf(v0[i], l.w0, v1[i] * l.w1);
                f[8 * q + i] = m == 2 ? ma[8 * q + i] * ve : fmaf(ma[8 * q + i], ve, f[8 * q + i]);
            }
        }
    }
}

__global__ void __launch_bounds__(kThreadsF, 2) tc24_forward_kernel(FusedParams p)
{
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar_tma;
    __shared__ __align__(8) uint64_t bar_mma[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_ctl[8];
    __shared__ int s_lo[3];
    const Smem24 L(p.plane_off[3], p.gplane_off[3], false);
    const int tid = threadIdx.x, h = tid / kRows, t = tid % kRows;
    if (tid < 32) tc::tmem_alloc(&s_tmem, kTmemF);
    if (tid == 0) {
        mbar_init(&bar_tma, 1);
        init_item_queue(s_ctl);
        mbar_init(&bar_mma[0], 1);
        mbar_init(&bar_mma[1], 1);
    }
    load_weights(p, sm, L);
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = s_tmem + (uint32_t)(h * 128);
    const uint32_t d0 = tbase, d1 = tbase + 64;
    SegTab tab = seg_tab(reinterpret_cast<float*>(sm + L.segi));
    const float* bias = reinterpret_cast<const float*>(sm + L.bias);
    const float beta = p.mlp.softplus_beta;
    const int lact = p.mlp.last_activation;
    unsigned char* hbh = sm + L.hb[h];
    uint32_t tma_phase = 0, mma_phase = 0;
    bool alive = true;
    while (alive) {
        const ItemInfo it = next_item(p, 0, reinterpret_cast<float*>(sm), tab, &bar_tma, s_ctl, false, kMapCapF, true);
        if (it.slot < 0) break;
        const bool real = it.slot < p.ws.nslot;
        if (real && it.first) {
            stage_line_windows(p, tab.box, sm + L.lwin, s_lo);
            if (!mbar_wait(&bar_tma, tma_phase)) {
                set_err(p.err, ATDF_DEVERR_TREE);
                mbar_wait(&bar_tma, tma_phase);
                alive = false;
            }
            tma_phase ^= 1;
        }
        alive = __syncthreads_and(alive);
        for (int t0 = h * kRows; alive && t0 < it.total; t0 += 2 * kRows) {
            const int k = t0 + t;
            const bool valid = k < it.total;
            float f[kC];
#pragma unroll
            for (int i = 0; i < kC; ++i) f[i] = 0.0f;
            float w = 0.0f, ts = 0.0f;
            int si = -1;
            if (valid) {
                const SampleState st = sample_state(p, tab, it, k, false);
                w = st.w;
                ts = st.t;
                si = st.si;
                if (real) {
                    const SampleGeo g = sample_geo_fast(p, tab, st.node, st.pos);
                    gather24(p, sm, sm + L.lwin, s_lo, g, f);
                }
            }
#pragma unroll
            for (int q = 0; q < 3; ++q) store_bf16x8(hbh + hbf_off(t, 8 * q), f + 8 * q);
            {
                const float zero[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                store_bf16x8(hbh + hbf_off(t, kC), zero);  // K padding (the previous tile's H0 there)
            }
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            half_barrier(h);
            if (t == 0) {
                tc::fence_after_sync();
                issue_l0<kHBColsF, 0>(sm, L, L.hb[h], d0);
                tc::commit(&bar_mma[h]);
            }
            alive = wait_mma(&bar_mma[h], mma_phase, p.err);
            // H0 = silu(D0 + b0) into HB columns 0..63
#pragma unroll
            for (int j = 0; j < kH / 16; ++j) {
                float v[16], bb[16];
                tc::ld_32x32b_x16(trow(d0, 16 * j), v);
                ld16(bias + 16 * j, bb);
                tc::wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = silu(v[i] + bb[i]);
                store_bf16x8(hbh + hbf_off(t, 16 * j), v);
                store_bf16x8(hbh + hbf_off(t, 16 * j + 8), v + 8);
            }
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            half_barrier(h);
            if (t == 0) {
                tc::fence_after_sync();
                issue_l1<kHBColsF>(sm, L, L.hb[h], d1);
                tc::commit(&bar_mma[h]);
            }
            alive = wait_mma(&bar_mma[h], mma_phase, p.err) && alive;
            float z = bias[3 * kH];
#pragma unroll
            for (int j = 0; j < kH / 16; ++j) {
                float v[16], bb[16], ww[16];
                tc::ld_32x32b_x16(trow(d1, 16 * j), v);
                ld16(bias + kH + 16 * j, bb);
                ld16(bias + 2 * kH + 16 * j, ww);
                tc::wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) z = fmaf(silu(v[i] + bb[i]), ww[i], z);
            }
            // the samples' contributions to their segments: the rows of a
            // warp hold consecutive samples, so each segment's samples form
            // a run of lanes; a segmented scan leaves each run's sum in its
            // last lane, which adds it to the segment's entry
            const float v = valid ? act_fwd(lact, z, beta) * w : 0.0f;
            {
                const int lane = t & 31;
                float run = v;
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const float o = __shfl_up_sync(0xffffffffu, run, off);
                    const int ko = __shfl_up_sync(0xffffffffu, si, off);
                    if (lane >= off && ko == si) run += o;
                }
                const int next = __shfl_down_sync(0xffffffffu, si, 1);
                if (valid && (lane == 31 || next != si)) atomicAdd(&tab.acc[si], run);
            }
            if (valid && p.bins) add_to_bins(p, tab, si, ts, v);
            tc::fence_before_sync();
            half_barrier(h);
        }
        alive = __syncthreads_and(alive);
        if (tid < it.nseg) p.ws.seg_partial[tab.id[tid]] = tab.acc[tid];
        __syncthreads();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid < 32) tc::tmem_dealloc(s_tmem, kTmemF);
}

// ---------------------------------------------------------------------------
// backward: one half of 128 rows, two threads per row (group g = tid / 128)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cta_barrier() { asm volatile("bar.sync 1, 384;" ::: "memory"); }

// Plane (bilinear) and line (linear) values of plane / line m for the 8
// channels of group g (channels 8g .. 8g + 7) of one sample. The line rows
// come from the slot's window in shared memory (LW: kLineRows rows of 24
// BF16 channels from row lo) when both taps are inside it.
__device__ __forceinline__ void gather8(const FusedParams& p, const unsigned char* sm, const unsigned char* LW,
                                        int lo, const SampleGeo& g, int m, int grp, float (&mat)[8],
                                        float (&vec)[8])
{
    const int Hm = p.field.plane_h[m], Wm = p.field.plane_w[m], L = p.field.line_len[m];
    const int Wp = p.plane_pitch[m];
    const Corner2 k = corners2(g.pu[m], g.pv[m], Hm, Wm);
    const Corner1 l = corners1(g.lu[m], L);
    const unsigned char* P = sm + (size_t)p.plane_off[m] * 2 + 16 * grp;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float w, u[8];
        unpack_bf16x8(*reinterpret_cast<const uint4*>(P + corner_texel(k, j, Wp, w) * (kC * 2)), u);
#pragma unroll
        for (int i = 0; i < 8; ++i) mat[i] = j == 0 ? u[i] * w : fmaf(u[i], w, mat[i]);
    }
    const int r0 = l.x0 - lo, r1 = l.x1 - lo;
    uint4 q0, q1;
    if ((unsigned)r0 < (unsigned)kLineRows && (unsigned)r1 < (unsigned)kLineRows) {
        const unsigned char* V = LW + (size_t)m * (kLineRows * kC * 2) + 16 * grp;
        q0 = *reinterpret_cast<const uint4*>(V + r0 * (kC * 2));
        q1 = *reinterpret_cast<const uint4*>(V + r1 * (kC * 2));
    } else {
        const unsigned char* V = reinterpret_cast<const unsigned char*>(p.field.line[m]) + 16 * grp;
        q0 = __ldg(reinterpret_cast<const uint4*>(V + l.x0 * (kC * 2)));
        q1 = __ldg(reinterpret_cast<const uint4*>(V + l.x1 * (kC * 2)));
    }
    float v0[8], v1[8];
    unpack_bf16x8(q0, v0);
    unpack_bf16x8(q1, v1);
#pragma unroll
    for (int i = 0; i < 8; ++i) vec[i] = fmaf(v0[i], l.w0, v1[i] * l.w1);
}

__global__ void __launch_bounds__(kThreadsB, 1) tc24_backward_kernel(FusedParams p)
{
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar_tma;
    __shared__ __align__(8) uint64_t bar_mma;
    __shared__ uint32_t s_tmem;
    __shared__ int s_ctl[8];
    __shared__ int s_lo[3];
    __shared__ float s_z[2][kRows];  // partial last-layer sums [group 0 / 1][row]
    // the next tile's sample states, computed by group 2 while groups 0 and 1
    // run the decoder's epilogues: SampleGeo (9 values), weight, segment
    __shared__ float s_pre[10][kRows];
    __shared__ int s_pre_si[kRows];
    __shared__ int s_pre_node[kRows];
    // fixed-point plane-gradient accumulation of the current slot
    __shared__ float s_tcum;    // sum of |contribution| over the slot's tiles so far
    __shared__ float s_tfirst;  // the same over its first tile (scale choice)
    __shared__ float s_scale;   // the slot's scale (a power of two; 0 = not chosen yet)
    __shared__ int s_fb;        // a tile of the slot went to global memory in FP32
    const Smem24 L(p.plane_off[3], p.gplane_off[3], true);
    const int tid = threadIdx.x, grp = tid >> 7, t = tid & (kRows - 1), lane = tid & 31;
    const bool mlp = grp < 2;   // the group owns hidden columns
    const int col0 = 32 * grp;  // hidden columns of groups 0 and 1
    const bool issuer = tid == 0;
    if (tid < 32) tc::tmem_alloc(&s_tmem, kTmemB);
    if (tid == 0) {
        mbar_init(&bar_tma, 1);
        init_item_queue(s_ctl);
        mbar_init(&bar_mma, 1);
    }
    load_weights(p, sm, L);
    init_pad_columns(sm + L.hb[0], tid, kThreadsB);
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = s_tmem;
    // TMEM: D0 / dX (0..63), D1 / dH0 (64..127), the weight-gradient
    // accumulator (128..223), the BF16 plane values of the feature step
    // (256 + 12 g .. + 11), the slot's line-gradient accumulator (320..399;
    // row m * kLineRows + i, columns 24 m + c) and the FP32 line values of the
    // feature step (400 + 24 g .. + 23)
    const uint32_t d0 = tbase, d1 = tbase + 64, dacc = tbase + 128, dline = tbase + 320;
    const uint32_t stash = tbase + 256 + 12 * grp, vstash = tbase + 400 + 24 * grp;
    // per-row sums of dz * H1 over all tiles (the last layer's weight
    // gradient before the sum over rows): group 0 at 224..255, group 1 at
    // 472..503
    const uint32_t dw2 = grp == 0 ? tbase + 224 : tbase + 472;
    SegTab tab = seg_tab(reinterpret_cast<float*>(sm + L.segi));
    const float* bias = reinterpret_cast<const float*>(sm + L.bias);
    const float beta = p.mlp.softplus_beta;
    const int lact = p.mlp.last_activation;
    // the slot's plane gradients in shared memory: plane m's texels from
    // gpo[m], kGP words each
    const int gpl_words = (p.gplane_off[3] / kC * kGP + 3) & ~3;
    const int gpo[3] = {p.gplane_off[0] / kC * kGP, p.gplane_off[1] / kC * kGP, p.gplane_off[2] / kC * kGP};
    int* gpl = reinterpret_cast<int*>(sm + L.gplanes);
    unsigned char* lw = sm + L.lwin;
    unsigned char* hb = sm + L.hb[0];
    unsigned char* gb = sm + L.g;
    uint32_t tma_phase = 0, mma_phase = 0;
    bool alive = true, had_tile = false;
    float gb2 = 0.f;             // group 0: this row's sum of dz over all tiles
    float scale = 0.f;           // the slot's fixed-point scale
    int ntiles = 0;              // tiles of the slot
    bool lacc = false;           // the line MMA has written the slot's accumulator
    bool gzero = false;          // the slot's global gradient has been zeroed (its first FP32 tile)
    while (alive) {
        const ItemInfo it = next_item(p, 1, reinterpret_cast<float*>(sm), tab, &bar_tma, s_ctl, true);
        if (it.slot < 0) break;
        const bool real = it.slot < p.ws.nslot;
        if (real && it.first) {
            for (int i = tid * 4; i < gpl_words; i += kThreadsB * 4)
                *reinterpret_cast<int4*>(gpl + i) = make_int4(0, 0, 0, 0);
            gzero = false;
            if (tid == 0) {
                s_tcum = 0.f;
                s_tfirst = 0.f;
                s_scale = 0.f;
                s_fb = 0;
            }
            scale = 0.f;
            ntiles = 0;
            lacc = false;
            stage_line_windows(p, tab.box, lw, s_lo);
            if (!mbar_wait(&bar_tma, tma_phase)) {
                set_err(p.err, ATDF_DEVERR_TREE);
                mbar_wait(&bar_tma, tma_phase);
                alive = false;
            }
            tma_phase ^= 1;
        }
        alive = __syncthreads_and(alive);
        const bool scale_set = s_scale != 0.f;
        if (scale_set) scale = s_scale;
        for (int t0 = 0; alive && t0 < it.total; t0 += kRows) {
            const bool handshake = !scale_set && t0 == 0;
            const int k = t0 + t;
            const bool valid = k < it.total;
            // features (own 8 channels); the plane values (BF16) and the line
            // values (FP32) go to TMEM for the scatter
            SampleGeo g;
            float w = 0.0f;
            int si = -1;
            bool act = false;
            if (t0 > 0) {  // computed during the previous tile
                si = s_pre_si[t];
                w = s_pre[9][t];
                act = real && valid;
                if (act) {
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        g.pu[q] = s_pre[q][t];
                        g.pv[q] = s_pre[3 + q][t];
                        g.lu[q] = s_pre[6 + q][t];
                    }
                }
            } else if (valid) {
                const SampleState st = sample_state(p, tab, it, k, false);
                w = st.w;
                si = st.si;
                if (real) {
                    g = sample_geo_fast(p, tab, st.node, st.pos);
                    act = true;
                }
            }
            float f[8];
#pragma unroll
            for (int m = 2; m >= 0; --m) {
                float mat[8], vec[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) mat[i] = vec[i] = 0.0f;
                if (act) gather8(p, sm, lw, s_lo[m], g, m, grp, mat, vec);
#pragma unroll
                for (int i = 0; i < 8; ++i) f[i] = m == 2 ? mat[i] * vec[i] : fmaf(mat[i], vec[i], f[i]);
                uint32_t pk[4], vb[8];
#pragma unroll
                for (int i = 0; i < 4; ++i) pk[i] = pack_bf16(mat[2 * i], mat[2 * i + 1]);
#pragma unroll
                for (int i = 0; i < 8; ++i) vb[i] = __float_as_uint(vec[i]);
                tc::st_32x32b_x4(trow(stash + 4 * m, 0), pk);
                tc::st_32x32b_x8(trow(vstash + 8 * m, 0), vb);
            }
            store_bf16x8(hb + hb_off(t, kXCol + 8 * grp), f);
            const float dIw = valid ? tab.acc[si] * w : 0.0f;
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            cta_barrier();
            if (issuer) {
                tc::fence_after_sync();
                issue_l0<kHBCols, kXCol>(sm, L, L.hb[0], d0);
                tc::commit(&bar_mma);
            }
            alive = wait_mma(&bar_mma, mma_phase, p.err);
            // H0 = silu(D0 + b0), this group's 32 columns
            if (mlp) {
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    float v[16], bb[16];
                    tc::ld_32x32b_x16(trow(d0, col0 + 16 * j), v);
                    ld16(bias + col0 + 16 * j, bb);
                    tc::wait_ld();
#pragma unroll
                    for (int i = 0; i < 16; ++i) v[i] = silu(v[i] + bb[i]);
                    store_bf16x8(hb + hb_off(t, col0 + 16 * j), v);
                    store_bf16x8(hb + hb_off(t, col0 + 16 * j + 8), v + 8);
                }
            }
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            cta_barrier();
            if (issuer) {
                tc::fence_after_sync();
                issue_l1<kHBCols>(sm, L, L.hb[0], d1);
                tc::commit(&bar_mma);
            }
            alive = wait_mma(&bar_mma, mma_phase, p.err) && alive;
            // last layer: partial z over this group's columns
            float a1[32];
            __half2 gpk[16];
            if (mlp) {
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    float v[16], bb[16];
                    tc::ld_32x32b_x16(trow(d1, col0 + 16 * j), v);
                    ld16(bias + kH + col0 + 16 * j, bb);
                    tc::wait_ld();
#pragma unroll
                    for (int i = 0; i < 16; ++i) a1[16 * j + i] = v[i] + bb[i];
                }
                float zp = 0.f;
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    float ww[16];
                    ld16(bias + 2 * kH + col0 + 16 * j, ww);
#pragma unroll
                    for (int i = 0; i < 16; i += 2) {
                        const float x0 = a1[16 * j + i], x1 = a1[16 * j + i + 1];
                        const float s0 = sigmoid_tanh(x0), s1 = sigmoid_tanh(x1);
                        const float h0 = x0 * s0, h1 = x1 * s1;
                        gpk[(16 * j + i) >> 1] = __floats2half2_rn(s0 * (1.0f + x0 * (1.0f - s0)),
                                                                   s1 * (1.0f + x1 * (1.0f - s1)));
                        a1[16 * j + i] = h0;
                        a1[16 * j + i + 1] = h1;
                        zp = fmaf(h0, ww[i], zp);
                        zp = fmaf(h1, ww[i + 1], zp);
                    }
                }
                s_z[grp][t] = zp;
                // the two partial sums of a row meet within its quarter of
                // the rows (warps q and q + 4); group 2 goes on without them
                asm volatile("bar.sync %0, 64;" ::"r"(2 + ((tid >> 5) & 3)) : "memory");
            }
            if (mlp) {
                const float z = s_z[0][t] + s_z[1][t] + bias[3 * kH];
                const float dz = dIw * act_grad(lact, z, beta);
                // dA1 = dz w2 silu'(A1) into G columns col0..col0+31
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    float ww[16], da[16];
                    ld16(bias + 2 * kH + col0 + 16 * j, ww);
#pragma unroll
                    for (int i = 0; i < 16; i += 2) {
                        const float2 gg = __half22float2(gpk[(16 * j + i) >> 1]);
                        da[i] = dz * ww[i] * gg.x;
                        da[i + 1] = dz * ww[i + 1] * gg.y;
                    }
                    store_bf16x8(gb + g_off(t, col0 + 16 * j), da);
                    store_bf16x8(gb + g_off(t, col0 + 16 * j + 8), da + 8);
                }
                // last-layer weight gradient: this row's dz * H1 added to its
                // running sums in TMEM (summed over rows at the end)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    float acc[16];
                    if (had_tile) {
                        tc::ld_32x32b_x16(trow(dw2, 16 * j), acc);
                        tc::wait_ld();
                    }
#pragma unroll
                    for (int i = 0; i < 16; ++i) acc[i] = had_tile ? fmaf(dz, a1[16 * j + i], acc[i]) : dz * a1[16 * j + i];
                    tc::st_32x32b_x16(trow(dw2, 16 * j), acc);
                }
                gb2 += dz;
            } else if (t0 + kRows < it.total) {
                // group 2, part 1: the next tile's sample states (position
                // and leaf parked in the line-coordinate slots and s_pre_node)
                const int k2 = t0 + kRows + t;
                int si2 = -1;
                float w2 = 0.0f;
                if (k2 < it.total) {
                    const SampleState st = sample_state(p, tab, it, k2, false);
                    si2 = st.si;
                    w2 = st.w;
#pragma unroll
                    for (int q = 0; q < 3; ++q) s_pre[6 + q][t] = st.pos[q];
                    s_pre_node[t] = st.node;
                }
                s_pre[9][t] = w2;
                s_pre_si[t] = si2;
            }
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            cta_barrier();
            if (issuer) {  // dH0 = dA1 W1 into the D1 columns
                tc::fence_after_sync();
                const uint32_t abase = tc::smem_addr(gb), bbase = tc::smem_addr(sm + L.w1);
#pragma unroll
                for (int j = 0; j < kH / 16; ++j) {
                    const uint64_t a = tc::smem_desc(abase + j * 256, 128, (kGCols / 8) * 128);
                    const uint64_t b = tc::smem_desc(bbase + j * 2 * (kH / 8) * 128, (kH / 8) * 128, 128);
                    tc::mma_bf16(d1, a, b, tc::idesc_bf16(kRows, kH, 0, 1), j > 0);
                }
                tc::commit(&bar_mma);
            }
            alive = wait_mma(&bar_mma, mma_phase, p.err) && alive;
            // dA0 = dH0 silu'(A0) into G columns 64 + col0.. (A0 = D0 + b0)
            if (mlp) {
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    float gv[16], av[16], da[16], bb[16];
                    tc::ld_32x32b_x16(trow(d1, col0 + 16 * j), gv);
                    tc::ld_32x32b_x16(trow(d0, col0 + 16 * j), av);
                    ld16(bias + col0 + 16 * j, bb);
                    tc::wait_ld();
#pragma unroll
                    for (int i = 0; i < 16; ++i) da[i] = gv[i] * silu_grad(av[i] + bb[i]);
                    store_bf16x8(gb + g_off(t, kH + col0 + 16 * j), da);
                    store_bf16x8(gb + g_off(t, kH + col0 + 16 * j + 8), da + 8);
                }
            } else if (real && t0 + kRows < it.total && s_pre_si[t] >= 0) {
                // group 2, part 2: the next tile's plane and line coordinates
                const float pos[3] = {s_pre[6][t], s_pre[7][t], s_pre[8][t]};
                const SampleGeo g2 = sample_geo_fast(p, tab, s_pre_node[t], pos);
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    s_pre[q][t] = g2.pu[q];
                    s_pre[3 + q][t] = g2.pv[q];
                    s_pre[6 + q][t] = g2.lu[q];
                }
            }
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            cta_barrier();
            if (issuer) {
                tc::fence_after_sync();
                // dX = dA0 W0 into the D0 columns 0..31 (24..31 are zero)
                const uint32_t abase = tc::smem_addr(gb + (kH / 8) * 128), bbase = tc::smem_addr(sm + L.w0);
#pragma unroll
                for (int j = 0; j < kH / 16; ++j) {
                    const uint64_t a = tc::smem_desc(abase + j * 256, 128, (kGCols / 8) * 128);
                    const uint64_t b = tc::smem_desc(bbase + j * 2 * (kCP / 8) * 128, (kCP / 8) * 128, 128);
                    tc::mma_bf16(d0, a, b, tc::idesc_bf16(kRows, kCP, 0, 1), j > 0);
                }
                // [dW1 db1; dW0 db0] += [dA1 | dA0]^T [H0 | X | 1]
                const uint32_t gbase = tc::smem_addr(gb), hbase = tc::smem_addr(hb);
#pragma unroll
                for (int j = 0; j < kRows / 16; ++j) {
                    const uint64_t a = tc::smem_desc(gbase + j * 2 * (kGCols / 8) * 128, (kGCols / 8) * 128, 128);
                    const uint64_t b = tc::smem_desc(hbase + j * 2 * (kHBCols / 8) * 128, (kHBCols / 8) * 128, 128);
                    tc::mma_bf16(dacc, a, b, tc::idesc_bf16(kRows, kHBCols, 1, 1), (had_tile || j > 0) ? 1u : 0u);
                }
                tc::commit(&bar_mma);
            }
            had_tile = true;
            alive = wait_mma(&bar_mma, mma_phase, p.err) && alive;
            // scatter, phase 1: dX * plane values as the line MMA's B operand
            // (HB columns 24 m + c), the tap column of the line MMA's A operand
            // (group 0), and dX * line values (the plane-gradient
            // contributions) in registers
            float dx[8];
            uint32_t pkr[3][4];
            tc::wait_st();  // the feature step's TMEM stores of the plane and line values
            tc::ld_32x32b_x8(trow(d0, 8 * grp), dx);
#pragma unroll
            for (int m = 0; m < 3; ++m) tc::ld_32x32b_x4(trow(stash + 4 * m, 0), pkr[m]);
            tc::wait_ld();
            float gv[3][8];
            if (real) {
                {
                    const uint4 z4 = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
                    for (int q = 0; q < kLineRows / 8; ++q)
                        *reinterpret_cast<uint4*>(gb + g_off(t, kLineRows * grp + 8 * q)) = z4;
                }
                float tsum = 0.f;  // sum of |dX * line value| of this thread's 24 values
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    float lv[8], vec[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) gv[m][i] = lv[i] = 0.f;
                    tc::ld_32x32b_x8(trow(vstash + 8 * m, 0), vec);
                    tc::wait_ld();
                    if (valid) {
                        float mat[8];
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const float2 x = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&pkr[m][i]));
                            mat[2 * i] = x.x;
                            mat[2 * i + 1] = x.y;
                        }
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            gv[m][i] = dx[i] * vec[i];
                            tsum += fabsf(gv[m][i]);
                            lv[i] = dx[i] * mat[i];
                        }
                        const Corner1 l = corners1(g.lu[m], p.field.line_len[m]);
                        const int lo = s_lo[m];
                        const int i0 = l.x0 - lo, i1 = l.x1 - lo;
                        if (i0 >= 0 && i0 < kLineRows && i1 >= 0 && i1 < kLineRows) {
                            if (grp == m) {
                                if (i0 == i1) {
                                    *reinterpret_cast<__nv_bfloat16*>(gb + g_off(t, m * kLineRows + i0)) =
                                        __float2bfloat16_rn(l.w0 + l.w1);
                                } else {
                                    *reinterpret_cast<__nv_bfloat16*>(gb + g_off(t, m * kLineRows + i0)) =
                                        __float2bfloat16_rn(l.w0);
                                    *reinterpret_cast<__nv_bfloat16*>(gb + g_off(t, m * kLineRows + i1)) =
                                        __float2bfloat16_rn(l.w1);
                                }
                            }
                        } else {  // outside the slot's window: straight to global
#pragma unroll
                            for (int i = 0; i < 8; ++i) {
                                const int c = 8 * grp + i;
                                atomicAdd(&p.gfield.line[m][l.x0 * kC + c], l.w0 * lv[i]);
                                atomicAdd(&p.gfield.line[m][l.x1 * kC + c], l.w1 * lv[i]);
                            }
                        }
                    }
                    store_bf16x8(hb + hb_off(t, kC * m + 8 * grp), lv);
                }
                // The bilinear weights of a sample sum to 1, so the tile adds at
                // most sum |dX * line value| to any texel of the slot.
#pragma unroll
                for (int off = 16; off >= 1; off >>= 1) tsum += __shfl_xor_sync(0xffffffffu, tsum, off);
                if (lane == 0) {
                    atomicAdd(&s_tcum, tsum);
                    if (handshake) atomicAdd(&s_tfirst, tsum);
                }
                tc::fence_smem_to_async();
                tc::fence_before_sync();
                cta_barrier();
                if (handshake) {
                    // scale = 2^e with the slot's expected total near 2^28
                    // (its tiles estimated from this item)
                    const float first = s_tfirst;
                    const float tiles = fmaxf(1.f, ceilf((float)it.total * (float)it.slot_items / (float)kRows));
                    int e = 20;
                    if (first > 0.f) e = ilogbf(268435456.0f / (first * tiles));
                    scale = ldexpf(1.0f, max(-100, min(e, 100)));
                    if (tid == 0) s_scale = scale;
                }
                // Overflow guard: the slot's values stay below 2^30 in
                // magnitude (sum of its scaled |contributions| plus half a unit
                // of rounding per contribution); a tile beyond that goes to
                // global memory in FP32.
                ++ntiles;
                const bool to_smem =
                    s_tcum * scale + (float)ntiles * (0.5f * kRows * 3 * 4 * kC) <= 1073741824.0f;
                if (!to_smem && issuer) s_fb = 1;
                if (!to_smem && !gzero) {
                    // the slot's first tile in FP32 (the same decision in every
                    // thread): its global gradient starts at zero (the caller
                    // does not clear it), then tiles and the flush add to it
                    for (int m = 0; m < 3; ++m) {
                        const int pf = p.field.plane_h[m] * p.field.plane_w[m] * kC;
                        float* dst = p.gfield.plane[m] + it.slot * (int64_t)pf;
                        for (int i = tid * 4; i < pf; i += kThreadsB * 4)
                            *reinterpret_cast<float4*>(dst + i) = make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                    __syncthreads();
                    gzero = true;
                }
                if (issuer) {  // line gradients of the tile into the slot's accumulator (overlaps the atomics)
                    tc::fence_after_sync();
                    const uint32_t abase = tc::smem_addr(gb), bbase = tc::smem_addr(hb);
#pragma unroll
                    for (int j = 0; j < kRows / 16; ++j) {
                        const uint64_t a =
                            tc::smem_desc(abase + j * 2 * (kGCols / 8) * 128, (kGCols / 8) * 128, 128);
                        const uint64_t b =
                            tc::smem_desc(bbase + j * 2 * (kHBCols / 8) * 128, (kHBCols / 8) * 128, 128);
                        tc::mma_bf16(dline, a, b, tc::idesc_bf16(kRows, kLineN, 1, 1), (lacc || j > 0) ? 1u : 0u);
                    }
                    tc::commit(&bar_mma);
                }
                lacc = true;
                // scatter, phase 2: the group's 8 channels to the four
                // corners, as fixed-point integers (shared-memory integer
                // atomics run several times faster than FP32 ones). A warp's
                // rows are consecutive samples of a ray, several in one cell:
                // lane l takes the corners from (l mod 4) on and the channels
                // from (l / 4 mod 8) on, so up to 32 lanes in one cell add to
                // 32 different words at each step.
                if (valid && to_smem) {
                    const int crot = (lane >> 2) & 7;
#pragma unroll
                    for (int m = 0; m < 3; ++m) {
                        const int Hm = p.field.plane_h[m], Wm = p.field.plane_w[m];
                        const Corner2 kc = corners2(g.pu[m], g.pv[m], Hm, Wm);
                        // gr[i] = gv[m][(i + crot) mod 8] (a three-stage rotation)
                        float gr[8];
#pragma unroll
                        for (int i = 0; i < 8; ++i) gr[i] = gv[m][i];
#pragma unroll
                        for (int b = 0; b < 3; ++b) {
                            const bool on = (crot >> b) & 1;
                            float nx[8];
#pragma unroll
                            for (int i = 0; i < 8; ++i) nx[i] = on ? gr[(i + (1 << b)) & 7] : gr[i];
#pragma unroll
                            for (int i = 0; i < 8; ++i) gr[i] = nx[i];
                        }
                        int* GP = gpl + gpo[m] + 8 * grp;
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            float wj;
                            const int tx = corner_texel(kc, (j + lane) & 3, Wm, wj) * kGP;
                            const float ws = wj * scale;
#pragma unroll
                            for (int i = 0; i < 8; ++i)
                                atomicAdd(&GP[tx + ((i + crot) & 7)], __float2int_rn(ws * gr[i]));
                        }
                    }
                }
                // a tile beyond the fixed-point range: FP32 atomics to the
                // slot's global gradient (rare; kept out of the unrolled code)
                if (valid && !to_smem) {
#pragma unroll
                    for (int m = 0; m < 3; ++m) {
                        const int Hm = p.field.plane_h[m], Wm = p.field.plane_w[m];
                        const Corner2 kc = corners2(g.pu[m], g.pv[m], Hm, Wm);
                        float* GG = p.gfield.plane[m] + it.slot * (int64_t)(Hm * Wm * kC);
#pragma unroll 1
                        for (int j = 0; j < 4; ++j) {
                            float wj;
                            const int tx = corner_texel(kc, j, Wm, wj) * kC;
#pragma unroll
                            for (int i = 0; i < 8; ++i) atomicAdd(&GG[tx + 8 * grp + i], wj * gv[m][i]);
                        }
                    }
                }
                alive = wait_mma(&bar_mma, mma_phase, p.err) && alive;
            }
            tc::fence_before_sync();
            cta_barrier();
        }
        alive = __syncthreads_and(alive);
        if (real && it.last) {
            // this CTA owns the slot: plain stores, unless a tile went to
            // global memory directly
            const float sc = s_scale, inv = sc > 0.f ? 1.0f / sc : 0.f;  // exact: a power of two
            const bool fb = s_fb != 0;
            for (int m = 0; m < 3; ++m) {
                const int pf = p.field.plane_h[m] * p.field.plane_w[m] * kC;
                float* dst = p.gfield.plane[m] + it.slot * (int64_t)pf;
                const int* src = gpl + gpo[m];
                for (int i = tid * 4; i < pf; i += kThreadsB * 4) {
                    // 4 channels of one texel (24 is a multiple of 4)
                    const int* e = src + (i / kC) * kGP + i % kC;
                    const int4 q = make_int4(e[0], e[1], e[2], e[3]);
                    const float4 v =
                        make_float4((float)q.x * inv, (float)q.y * inv, (float)q.z * inv, (float)q.w * inv);
                    if (fb)
                        atomicAdd(reinterpret_cast<float4*>(dst + i), v);
                    else
                        *reinterpret_cast<float4*>(dst + i) = v;
                }
            }
            // the slot's line gradients: TMEM row m * kLineRows + i holds row
            // s_lo[m] + i of line m in columns 24 m .. 24 m + 23
            if (lacc) {
                tc::fence_after_sync();
                float v0[8], v1[8], v2[8];
                tc::ld_32x32b_x8(trow(dline, 8 * grp), v0);
                tc::ld_32x32b_x8(trow(dline, kC + 8 * grp), v1);
                tc::ld_32x32b_x8(trow(dline, 2 * kC + 8 * grp), v2);
                tc::wait_ld();
                tc::fence_before_sync();
                if (t < 3 * kLineRows) {
                    const int m = t / kLineRows, i = t % kLineRows;
                    const int e = s_lo[m] + i;
                    if (e < p.field.line_len[m]) {
                        float* dst = p.gfield.line[m] + e * kC + 8 * grp;
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const float v = m == 0 ? v0[q] : (m == 1 ? v1[q] : v2[q]);
                            if (v != 0.0f) atomicAdd(dst + q, v);
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    // decoder gradients from the TMEM accumulator rows (group g reads columns
    // 32g .. 32g + 31): rows 0..63 hold dW1 (columns 0..63) and db1 (column
    // 88), rows 64..127 dW0 (columns 64..87) and db0 (column 88)
    if (had_tile) {
        tc::fence_after_sync();
#pragma unroll
        for (int jj = 0; jj < 2; ++jj) {
            const int j = 2 * grp + jj;
            float v[16];
            tc::ld_32x32b_x16(trow(dacc, 16 * j), v);
            tc::wait_ld();
            if (t < kH) {
                if (j < 4)
#pragma unroll
                    for (int i = 0; i < 16; ++i) atomicAdd(&p.gmlp.weight[1][t * kH + 16 * j + i], v[i]);
                if (j == 5) atomicAdd(&p.gmlp.bias[1][t], v[kOnesCol - 80]);
            } else {
                const int n = t - kH;
                if (j == 4)
#pragma unroll
                    for (int i = 0; i < 16; ++i) atomicAdd(&p.gmlp.weight[0][n * kC + i], v[i]);
                if (j == 5) {
#pragma unroll
                    for (int i = 0; i < 8; ++i) atomicAdd(&p.gmlp.weight[0][n * kC + 16 + i], v[i]);
                    atomicAdd(&p.gmlp.bias[0][n], v[kOnesCol - 80]);
                }
            }
        }
    }
    // last layer: the rows' running sums reduced over the warp's 32 rows,
    // halving the value set each round (lane l ends with one column)
    if (mlp && had_tile) {
        float a[32];
        tc::ld_32x32b_x16(trow(dw2, 0), *reinterpret_cast<float(*)[16]>(a));
        tc::ld_32x32b_x16(trow(dw2, 16), *reinterpret_cast<float(*)[16]>(a + 16));
        tc::wait_ld();
        int n = 32;
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) {
            const bool upper = (lane & off) != 0;
            n >>= 1;
#pragma unroll
            for (int kk = 0; kk < 16; ++kk) {
                if (kk < n) {
                    const float send = upper ? a[kk] : a[kk + n];
                    const float keep = upper ? a[kk + n] : a[kk];
                    a[kk] = keep + __shfl_xor_sync(0xffffffffu, send, off);
                }
            }
        }
        int colbits = 0;
        for (int off = 16, b = 0; off >= 1; off >>= 1, ++b)
            if (lane & off) colbits |= (32 >> (b + 1));
        atomicAdd(&p.gmlp.weight[2][col0 + colbits], a[0]);
        if (grp == 0) {
            float s = gb2;
#pragma unroll
            for (int off = 16; off >= 1; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
            if (lane == 0) atomicAdd(&p.gmlp.bias[2][0], s);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid < 32) tc::tmem_dealloc(s_tmem, kTmemB);
}

}  // namespace tc24

bool tc24_supported(const atdf_field_t* f, const atdf_mlp_t* m)
{
    return f->dtype == ATDF_BF16 && f->channels == tc24::kC && f->mode == 0 && m->num_layers == 3 &&
           m->dims[0] == tc24::kC && m->dims[1] == tc24::kH && m->dims[2] == tc24::kH && m->dims[3] == 1 &&
           m->hidden_activation == ATDF_ACT_SILU;
}

static int launch24(void (*fn)(FusedParams), bool bwd, const FusedParams& p, cudaStream_t st)
{
    const int smem = (int)tc24::Smem24(p.plane_off[3], p.gplane_off[3], bwd).total;
    int dev = 0, optin = 0, sms = 0, per = 0;
    ATDF_CUDA_TRY(cudaGetDevice(&dev));
    ATDF_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (smem > optin) return ATDF_ERR_UNSUPPORTED;
    ATDF_CUDA_TRY(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ATDF_CUDA_TRY(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared));
    ATDF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int threads = bwd ? tc24::kThreadsB : tc24::kThreadsF;
    ATDF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)fn, threads, smem));
    if (per < 1) return ATDF_ERR_UNSUPPORTED;
    // the forward fits two CTAs per SM (shared memory, 2 x 256 TMEM columns);
    // the backward one (its shared memory, all 512 TMEM columns)
    int smem_sm = 0;
    ATDF_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    per = bwd ? 1 : std::max(1, std::min(2, smem_sm / (smem + 1024)));
    fn<<<sms * per, threads, smem, st>>>(p);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int launch_tc24_forward(const FusedParams& p, cudaStream_t st)
{
    return launch24(tc24::tc24_forward_kernel, false, p, st);
}
int launch_tc24_backward(const FusedParams& p, cudaStream_t st)
{
    return launch24(tc24::tc24_backward_kernel, true, p, st);
}

}  // namespace atdf
