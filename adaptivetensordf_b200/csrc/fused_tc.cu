// Fused leaf-major projection with BF16 factor planes and the decoder on the
// 5th-generation tensor cores (tcgen05, FP32 accumulation in TMEM), forward
// and hand-written adjoint, for sm_100a. Shape: C = 16 channels ("add"),
// decoder 16 -> 64 -> 64 -> 1 (the reference's FCBlock default with one
// hidden layer of 64; hyperacorn/csrc/geometry/Modules.h:68-109).
//
// A forward CTA has two halves of 128 threads; each half owns a 128-sample
// tile, one thread per sample (= one TMEM lane / accumulator row). A backward
// CTA has two halves of 256 threads, two per sample row, each of the pair
// taking half the channels and half the hidden columns. Both halves share the
// work item's planes (staged by TMA) and, in the backward, its shared
// plane-gradient copy. Per tile:
//   forward  X[128x16] -> D0 = X W0^T -> H0 = silu(D0 + b0)
//            D1 = H0 W1^T -> silu(D1 + b1) . w2 + b2 -> softplus -> rho * w
//   backward dz, dA1 = dz w2 silu'(A1);   dH0 = dA1 W1 -> dA0 = dH0 silu'(A0)
//            dX = dA0 W0 -> scatter into the plane gradients
//            [dW1 db1; dW0 db0] += [dA1 | dA0]^T [H0 | X | 1]   (one M=128 MMA,
//            accumulated in TMEM across every tile of the CTA)
// All MMA operands use the no-swizzle core-matrix layouts of tc.cuh, chosen
// so one buffer serves several GEMMs: the buffer HB [128 x 96] (H0 | X | 1)
// is the A operand of both forward layers (K-major views) and the B operand
// of the weight-gradient MMA (MN-major); G [128 x 128] (dA1 | dA0) is the A
// operand of dH0 and dX (K-major views) and of the weight-gradient MMA
// (MN-major). W0 / W1 in [out][in] order are the K-major B of the forward
// layers and, unchanged, the MN-major B of the backward ones.

#include <cuda_bf16.h>

#include "fused_common.cuh"
#include "tc.cuh"
#include "tc_common.cuh"

namespace atdf {
namespace tcf {

constexpr int kC = 16;
constexpr int kH = 64;
constexpr int kRows = 128;          // samples per tile
constexpr int kThreadsTC = 256;     // two halves
constexpr int kHBCols = 96;         // H0 (64) | X (16) | ones | zero pad
constexpr int kGCols = 128;         // dA1 (64) | dA0 (64)
constexpr int kLineWinTC = 32;      // line-gradient window entries per line (shared memory)
constexpr int kLineRowsTC = 21;     // rows per line in the line-gradient MMA (3 lines <= 64 rows)
constexpr uint32_t kTmemFwd = 256;  // columns per CTA (2 CTAs per SM)
constexpr uint32_t kTmemBwd = 512;

__device__ __forceinline__ uint32_t hb_off(int s, int c) { return tc::mnmajor_off(c, s, kHBCols); }
__device__ __forceinline__ uint32_t g_off(int s, int c) { return tc::mnmajor_off(c, s, kGCols); }
__device__ __forceinline__ uint32_t w0_off(int n, int f) { return tc::kmajor_off(n, f, kC); }
__device__ __forceinline__ uint32_t w1_off(int n, int k) { return tc::kmajor_off(n, k, kH); }

struct TCSmem {
    uint32_t planes, w0, w1, bias, hb[2], g[2], gplanes, gline, segi, total;
    __host__ __device__ TCSmem(int plane_elems, int gplane_elems, bool bwd)
    {
        auto al = [](uint32_t x) { return (x + 127u) & ~127u; };
        uint32_t o = 0;
        planes = o;
        o = al(o + plane_elems * 2);
        w0 = o;
        o = al(o + kH * kC * 2);
        w1 = o;
        o = al(o + kH * kH * 2);
        bias = o;  // b0[64] b1[64] w2[64] b2
        o = al(o + (3 * kH + 4) * 4);
        for (int h = 0; h < 2; ++h) {
            hb[h] = o;
            o = al(o + kRows * kHBCols * 2);
        }
        for (int h = 0; h < 2; ++h) {
            g[h] = o;
            if (bwd) o = al(o + kRows * kGCols * 2);
        }
        gplanes = o;
        if (bwd) o = al(o + gplane_elems * 4);
        gline = o;
        if (bwd) o = al(o + 3 * kLineWinTC * kC * 4);
        segi = o;
        o = al(o + kSegTabFloats * 4);
        total = o;
    }
};

__device__ __forceinline__ void half_barrier(int h) { asm volatile("bar.sync %0, 128;" ::"r"(1 + h) : "memory"); }

// Corner visited first by this lane. A texel (16 BF16 channels) spans two
// 16-byte bank groups, and with the pitch at 2 mod 4 the corners' texel
// indices are r, r + 1, r + 2, r + 3 mod 4 (r of corner 0), so the 8
// (corner, half) chunks of a footprint fill all 8 groups of a 128-byte bank
// row. 16-byte loads are served per 8-lane phase; lane p of a phase starts
// at the corner of residue sel(p) and walks the corners in residue order,
// which spreads one instruction's loads of the phase over distinct groups.
__device__ __forceinline__ int first_corner(const Corner2& k, int Wp, int sel)
{
    return (sel - (k.y0 * Wp + k.x0)) & 3;
}

// VM feature of one sample (16 channels) from the BF16 planes in shared
// memory (padded rows) and the BF16 lines in global memory: fa = channels
// 8 * hf .. 8 * hf + 7, fb = the other eight, hf = lane mod 2. Lane p of an
// 8-lane phase loads at step j the corner of residue p / 2 + j, first half
// hf, then half 1 - hf: 8 distinct bank groups per instruction and phase.
__device__ __forceinline__ void gather_features(const FusedParams& p, const unsigned char* sm, const SampleGeo& g,
                                                float (&fa)[8], float (&fb)[8])
{
    const int lane = threadIdx.x & 31, hf = lane & 1;
#pragma unroll
    for (int m = 2; m >= 0; --m) {
        const int Hm = p.field.plane_h[m], Wm = p.field.plane_w[m], L = p.field.line_len[m];
        const int Wp = p.plane_pitch[m];
        const Corner2 k = corners2(g.pu[m], g.pv[m], Hm, Wm);
        const Corner1 l = corners1(g.lu[m], L);
        const unsigned char* P = sm + (size_t)p.plane_off[m] * 2;
        const uint4* V = reinterpret_cast<const uint4*>(p.field.line[m]);
        const int c0 = first_corner(k, Wp, (lane & 7) >> 1);
        float ma[8], mb[8];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float w;
            const unsigned char* tx = P + corner_texel(k, (c0 + j) & 3, Wp, w) * (kC * 2);
            float u[8], v[8];
            unpack_bf16x8(*reinterpret_cast<const uint4*>(tx + 16 * hf), u);
            unpack_bf16x8(*reinterpret_cast<const uint4*>(tx + 16 * (hf ^ 1)), v);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                ma[i] = j == 0 ? u[i] * w : fmaf(u[i], w, ma[i]);
                mb[i] = j == 0 ? v[i] * w : fmaf(v[i], w, mb[i]);
            }
        }
        float va0[8], va1[8], vb0[8], vb1[8];
        unpack_bf16x8(__ldg(V + l.x0 * 2 + hf), va0);
        unpack_bf16x8(__ldg(V + l.x1 * 2 + hf), va1);
        unpack_bf16x8(__ldg(V + l.x0 * 2 + (hf ^ 1)), vb0);
        unpack_bf16x8(__ldg(V + l.x1 * 2 + (hf ^ 1)), vb1);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float vea = fmaf(va0[i], l.w0, va1[i] * l.w1), veb = fmaf(vb0[i], l.w0, vb1[i] * l.w1);
            fa[i] = m == 2 ? ma[i] * vea : fmaf(ma[i], vea, fa[i]);
            fb[i] = m == 2 ? mb[i] * veb : fmaf(mb[i], veb, fb[i]);
        }
    }
}

__device__ __forceinline__ void load_weights_tc(const FusedParams& p, unsigned char* sm, const TCSmem& L)
{
    const atdf_mlp_t& m = p.mlp;
    for (int i = threadIdx.x; i < kH * kC; i += blockDim.x) {
        const int n = i / kC, f = i % kC;
        *reinterpret_cast<__nv_bfloat16*>(sm + L.w0 + w0_off(n, f)) = __float2bfloat16_rn(m.weight[0][i]);
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

// Forward layer-0 / layer-1 MMAs of one half (issued by one thread).
__device__ __forceinline__ void issue_l0(const unsigned char* sm, const TCSmem& L, int h, uint32_t d0)
{
    const uint64_t a = tc::smem_desc(tc::smem_addr(sm + L.hb[h] + (kH / 8) * 128), 128, 12 * 128);
    const uint64_t b = tc::smem_desc(tc::smem_addr(sm + L.w0), 128, (kC / 8) * 128);
    tc::mma_bf16(d0, a, b, tc::idesc_bf16(kRows, kH, 0, 0), 0);
}

__device__ __forceinline__ void issue_l1(const unsigned char* sm, const TCSmem& L, int h, uint32_t d1)
{
    const uint32_t abase = tc::smem_addr(sm + L.hb[h]), bbase = tc::smem_addr(sm + L.w1);
#pragma unroll
    for (int j = 0; j < kH / 16; ++j) {
        const uint64_t a = tc::smem_desc(abase + j * 256, 128, 12 * 128);
        const uint64_t b = tc::smem_desc(bbase + j * 256, 128, (kH / 8) * 128);
        tc::mma_bf16(d1, a, b, tc::idesc_bf16(kRows, kH, 0, 0), j > 0);
    }
}

// Forward sample features of tile row t into HB (X columns); returns validity.
// The forward walks an item's samples in order: a warp's rows follow one ray,
// so their plane gathers and segment-table reads share addresses.
__device__ __forceinline__ bool tile_features(const FusedParams& p, unsigned char* sm, const TCSmem& L,
                                              const SegTab& tab, const ItemInfo& it, bool real, int h, int k,
                                              int t, float& w, int& si, SampleGeo& g, float& ts)
{
    const bool valid = k < it.total;
    float fa[8], fb[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) fa[i] = fb[i] = 0.0f;
    w = 0.0f;
    ts = 0.0f;
    si = -1;
    if (valid) {
        const SampleState st = sample_state(p, tab, it, k, false);
        w = st.w;
        ts = st.t;
        si = st.si;
        if (real) {
            g = sample_geo_fast(p, tab, st.node, st.pos);
            gather_features(p, sm, g, fa, fb);
        }
    }
    const int hf = threadIdx.x & 1;
    store_bf16x8(sm + L.hb[h] + hb_off(t, kH + 8 * hf), fa);
    store_bf16x8(sm + L.hb[h] + hb_off(t, kH + 8 * (hf ^ 1)), fb);
    return valid;
}

// Layer-0 epilogue: H0 = silu(D0 + b0) into HB columns 0..63.
__device__ __forceinline__ void epilogue_l0(unsigned char* sm, const TCSmem& L, int h, int t, uint32_t d0)
{
    const float* b0 = reinterpret_cast<const float*>(sm + L.bias);
#pragma unroll
    for (int j = 0; j < kH / 16; ++j) {
        float v[16], bb[16];
        tc::ld_32x32b_x16(trow(d0, 16 * j), v);
        ld16(b0 + 16 * j, bb);
        tc::wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = silu(v[i] + bb[i]);
        store_bf16x8(sm + L.hb[h] + hb_off(t, 16 * j), v);
        store_bf16x8(sm + L.hb[h] + hb_off(t, 16 * j + 8), v + 8);
    }
}

__global__ void __launch_bounds__(kThreadsTC, 2) tc_forward_kernel(FusedParams p)
{
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar_tma;
    __shared__ __align__(8) uint64_t bar_mma[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_ctl[8];
    const TCSmem L(p.plane_off[3], p.gplane_off[3], false);
    const int tid = threadIdx.x, h = tid / kRows, t = tid % kRows;
    if (tid < 32) tc::tmem_alloc(&s_tmem, kTmemFwd);
    if (tid == 0) {
        mbar_init(&bar_tma, 1);
        init_item_queue(s_ctl);
        mbar_init(&bar_mma[0], 1);
        mbar_init(&bar_mma[1], 1);
    }
    load_weights_tc(p, sm, L);
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
    uint32_t tma_phase = 0, mma_phase = 0;
    bool alive = true;
    while (alive) {
        const ItemInfo it = next_item(p, 0, reinterpret_cast<float*>(sm), tab, &bar_tma, s_ctl, false, kSegMapCap, true);
        if (it.slot < 0) break;
        const bool real = it.slot < p.ws.nslot;
        if (real && it.first) {
            if (!mbar_wait(&bar_tma, tma_phase)) {
                set_err(p.err, ATDF_DEVERR_TREE);
                mbar_wait(&bar_tma, tma_phase);
                alive = false;
            }
            tma_phase ^= 1;
        }
        alive = __syncthreads_and(alive);
        for (int t0 = h * kRows; alive && t0 < it.total; t0 += 2 * kRows) {
            float w, ts;
            int si;
            SampleGeo g;
            const bool valid = tile_features(p, sm, L, tab, it, real, h, t0 + t, t, w, si, g, ts);
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            half_barrier(h);
            if (t == 0) {
                tc::fence_after_sync();
                issue_l0(sm, L, h, d0);
                tc::commit(&bar_mma[h]);
            }
            alive = wait_mma(&bar_mma[h], mma_phase, p.err);
            epilogue_l0(sm, L, h, t, d0);
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            half_barrier(h);
            if (t == 0) {
                tc::fence_after_sync();
                issue_l1(sm, L, h, d1);
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
            // each segment's run of lanes summed by a segmented warp scan,
            // its last lane adding the run to the segment's entry
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
    if (tid < 32) tc::tmem_dealloc(s_tmem, kTmemFwd);
}

// ---------------------------------------------------------------------------
// Backward with two threads per sample row: 512 threads = two halves x two
// channel groups of 128 threads. Group g of a half owns channels 8g..8g+7 of
// the features and columns 32g..32g+31 of every 64-wide layer, so each
// thread carries half the registers of the 256-thread kernel and an SM runs
// 16 warps instead of 8 within the same shared memory and TMEM (a 256-thread
// version with one thread per row ran 4.9 ms where this one runs 4.0 ms on
// 16384 rays of the depth-4 workload).
// ---------------------------------------------------------------------------
constexpr int kThreadsB2 = 512;

__device__ __forceinline__ void half_barrier2(int h) { asm volatile("bar.sync %0, 256;" ::"r"(1 + h) : "memory"); }

// Bilinear plane values and linear line values of plane / line m for the 8
// channels cb..cb+7 of one sample (cb is the same across a warp, so one
// 8-lane phase can reach 4 of the 8 bank groups: lanes p and p + 4 of a
// phase share a corner residue, two loads per group).
__device__ __forceinline__ void gather_half(const FusedParams& p, const unsigned char* sm, const SampleGeo& g, int m,
                                            int cb, float (&mat)[8], float (&vec)[8])
{
    const int Hm = p.field.plane_h[m], Wm = p.field.plane_w[m], L = p.field.line_len[m];
    const int Wp = p.plane_pitch[m];
    const Corner2 k = corners2(g.pu[m], g.pv[m], Hm, Wm);
    const Corner1 l = corners1(g.lu[m], L);
    const unsigned char* P = sm + (size_t)p.plane_off[m] * 2 + cb * 2;
    const uint4* V = reinterpret_cast<const uint4*>(p.field.line[m]);
    const int c0 = first_corner(k, Wp, threadIdx.x & 3);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float w, u[8];
        const int tx = corner_texel(k, (c0 + j) & 3, Wp, w);
        unpack_bf16x8(*reinterpret_cast<const uint4*>(P + tx * (kC * 2)), u);
#pragma unroll
        for (int i = 0; i < 8; ++i) mat[i] = j == 0 ? u[i] * w : fmaf(u[i], w, mat[i]);
    }
    float v0[8], v1[8];
    unpack_bf16x8(__ldg(V + l.x0 * 2 + (cb >> 3)), v0);
    unpack_bf16x8(__ldg(V + l.x1 * 2 + (cb >> 3)), v1);
#pragma unroll
    for (int i = 0; i < 8; ++i) vec[i] = fmaf(v0[i], l.w0, v1[i] * l.w1);
}

// Linear line values of line m for the 8 channels cb..cb+7 of one sample.
__device__ __forceinline__ void line_half(const FusedParams& p, const SampleGeo& g, int m, int cb, float (&vec)[8])
{
    const Corner1 l = corners1(g.lu[m], p.field.line_len[m]);
    const uint4* V = reinterpret_cast<const uint4*>(p.field.line[m]);
    float v0[8], v1[8];
    unpack_bf16x8(__ldg(V + l.x0 * 2 + (cb >> 3)), v0);
    unpack_bf16x8(__ldg(V + l.x1 * 2 + (cb >> 3)), v1);
#pragma unroll
    for (int i = 0; i < 8; ++i) vec[i] = fmaf(v0[i], l.w0, v1[i] * l.w1);
}

// Features (channels cb..cb+7) of tile row t into HB; returns validity.
// The bilinear plane values are kept (as BF16) in 12 TMEM columns at stash
// for the scatter of the same tile, which then does not gather them again.
__device__ __forceinline__ bool tile_features_half(const FusedParams& p, unsigned char* sm, const TCSmem& L,
                                                   const SegTab& tab, const ItemInfo& it, bool real, int h, int k,
                                                   int t, int cb, uint32_t stash, float& w, int& si, SampleGeo& g)
{
    const bool valid = k < it.total;
    float f[8];
    uint32_t pk[3][4];
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = 0.0f;
#pragma unroll
    for (int m = 0; m < 3; ++m) pk[m][0] = pk[m][1] = pk[m][2] = pk[m][3] = 0u;
    w = 0.0f;
    si = -1;
    if (valid) {
        const SampleState st = sample_state(p, tab, it, k, false);
        w = st.w;
        si = st.si;
        if (real) {
            g = sample_geo_fast(p, tab, st.node, st.pos);
            // planes 2, 1, 0, as in gather_features
#pragma unroll
            for (int m = 2; m >= 0; --m) {
                float mat[8], vec[8];
                gather_half(p, sm, g, m, cb, mat, vec);
#pragma unroll
                for (int i = 0; i < 8; ++i) f[i] = m == 2 ? mat[i] * vec[i] : fmaf(mat[i], vec[i], f[i]);
#pragma unroll
                for (int i = 0; i < 4; ++i) pk[m][i] = pack_bf16(mat[2 * i], mat[2 * i + 1]);
            }
        }
    }
    store_bf16x8(sm + L.hb[h] + hb_off(t, kH + cb), f);
#pragma unroll
    for (int m = 0; m < 3; ++m) tc::st_32x32b_x4(stash + 4 * m, pk[m]);
    return valid;
}

// Scratch float j (0..47) of sample t: HB columns 48..79 for j < 16, G
// columns 64..127 (free once the dX and dW MMAs have read them) for the rest.
__device__ __forceinline__ float* scratch2(unsigned char* hbh, unsigned char* gh, int t, int j)
{
    if (j < 16) return reinterpret_cast<float*>(hbh + hb_off(t, 48 + 8 * (j >> 2)) + (j & 3) * 4);
    const int q = j - 16;
    return reinterpret_cast<float*>(gh + g_off(t, 64 + 8 * (q >> 2)) + (q & 3) * 4);
}

__global__ void __launch_bounds__(kThreadsB2, 1) tc_backward2_kernel(FusedParams p)
{
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar_tma;
    __shared__ __align__(8) uint64_t bar_mma[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_ctl[8];
    __shared__ int s_lo[3];
    __shared__ float s_z[2][2][kRows];  // partial last-layer sums [half][group][row]
    // fixed-point plane-gradient accumulation of the current slot
    __shared__ float s_tcum[2];    // per half: sum of |contribution| over the slot's tiles so far
    __shared__ float s_tfirst[2];  // per half: the same over its first tile (scale choice)
    __shared__ float s_scale;      // the slot's scale (a power of two; 0 = not chosen yet)
    __shared__ int s_fb;           // a tile of the slot went to global memory in FP32
    const TCSmem L(p.plane_off[3], p.gplane_off[3], true);
    const int tid = threadIdx.x, h = tid >> 8, grp = (tid >> 7) & 1, t = tid & (kRows - 1), lane = tid & 31;
    const int cb = 8 * grp;       // channels of this group
    const int col0 = 32 * grp;    // hidden columns of this group
    const bool issuer = (tid & 255) == 0;
    if (tid < 32) tc::tmem_alloc(&s_tmem, kTmemBwd);
    if (tid == 0) {
        mbar_init(&bar_tma, 1);
        init_item_queue(s_ctl);
        mbar_init(&bar_mma[0], 1);
        mbar_init(&bar_mma[1], 1);
    }
    load_weights_tc(p, sm, L);
    // ones column (80) and zero padding (81..95) of both HB buffers
    for (int i = tid; i < 2 * kRows; i += kThreadsB2) {
        const int hh = i / kRows, s = i % kRows;
        float v[8] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        store_bf16x8(sm + L.hb[hh] + hb_off(s, 80), v);
        v[0] = 0.f;
        store_bf16x8(sm + L.hb[hh] + hb_off(s, 88), v);
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = s_tmem + (uint32_t)(h * 256);
    const uint32_t d0 = tbase, d1 = tbase + 64, dacc = tbase + 128;
    const uint32_t stash = trow(tbase + 224 + 12 * grp, 0);  // this thread's row, 12 columns
    SegTab tab = seg_tab(reinterpret_cast<float*>(sm + L.segi));
    const float* bias = reinterpret_cast<const float*>(sm + L.bias);
    const float beta = p.mlp.softplus_beta;
    const int lact = p.mlp.last_activation;
    const int C = kC;
    const int gplane_elems = p.gplane_off[3];
    int* gpl = reinterpret_cast<int*>(sm + L.gplanes);  // the slot's plane gradients, fixed point
    float* gln = reinterpret_cast<float*>(sm + L.gline);
    unsigned char* hbh = sm + L.hb[h];
    unsigned char* gh = sm + L.g[h];
    uint32_t tma_phase = 0, mma_phase = 0;
    bool alive = true, had_tile = false;
    float gw2 = 0.f, gb2 = 0.f;  // lane owns one last-layer column of its group
    const int crot = 2 * (lane & 7) + ((lane >> 3) & 1) + 2 * (lane >> 4);
    float scale = 0.f;  // the slot's fixed-point scale
    int ntiles = 0;     // tiles of this half in the slot
    while (alive) {
        const ItemInfo it = next_item(p, 1, reinterpret_cast<float*>(sm), tab, &bar_tma, s_ctl, true);
        if (it.slot < 0) break;
        const bool real = it.slot < p.ws.nslot;
        if (real && it.first) {
            for (int i = tid * 4; i < gplane_elems; i += kThreadsB2 * 4)
                *reinterpret_cast<int4*>(gpl + i) = make_int4(0, 0, 0, 0);
            // the slot's global gradient starts at zero (the caller does not
            // clear it): a tile that overflows the fixed-point range adds to it
            for (int m = 0; m < 3; ++m) {
                const int pf = p.field.plane_h[m] * p.field.plane_w[m] * C;
                float* dst = p.gfield.plane[m] + it.slot * (int64_t)pf;
                for (int i = tid * 4; i < pf; i += kThreadsB2 * 4)
                    *reinterpret_cast<float4*>(dst + i) = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            if (tid == 0) {
                s_tcum[0] = s_tcum[1] = 0.f;
                s_tfirst[0] = s_tfirst[1] = 0.f;
                s_scale = 0.f;
                s_fb = 0;
            }
            scale = 0.f;
            ntiles = 0;
            for (int i = tid; i < 3 * kLineWinTC * C; i += kThreadsB2) gln[i] = 0.0f;
            if (tid < 3) {
                const float* bmin = tab.box;  // the item's leaf (segment 0's)
                const int Ln = p.field.line_len[tid];
                int lo = 0;
                if (Ln > kLineRowsTC) {
                    const float u = tid == 0 ? roi_coord(bmin[0], p.field.roi_min[0], p.field.roi_max[0])
                                             : (tid == 2 ? bmin[2] : -1.0f);
                    lo = (int)floorf(((u + 1.0f) * 0.5f) * (float)(Ln - 1)) - 2;
                    lo = max(0, min(lo, Ln - kLineRowsTC));
                }
                s_lo[tid] = lo;
            }
            if (!mbar_wait(&bar_tma, tma_phase)) {
                set_err(p.err, ATDF_DEVERR_TREE);
                mbar_wait(&bar_tma, tma_phase);
                alive = false;
            }
            tma_phase ^= 1;
        }
        alive = __syncthreads_and(alive);
        // The scale is chosen once per slot, at the first tile of each half
        // (both halves together when the item gives both a tile), from the
        // measured contributions of those tiles; later items read it.
        const bool scale_set = s_scale != 0.f;
        if (scale_set) scale = s_scale;
        const bool both = it.total > kRows;
        for (int t0 = h * kRows; alive && t0 < it.total; t0 += 2 * kRows) {
            const bool handshake = !scale_set && t0 == h * kRows;
            SampleGeo g;
            float w;
            int si;
            const bool valid = tile_features_half(p, sm, L, tab, it, real, h, t0 + t, t, cb, stash, w, si, g);
            const float dIw = valid ? tab.acc[si] * w : 0.0f;
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            half_barrier2(h);
            if (issuer) {
                tc::fence_after_sync();
                issue_l0(sm, L, h, d0);
                tc::commit(&bar_mma[h]);
            }
            alive = wait_mma(&bar_mma[h], mma_phase, p.err);
            // H0 = silu(D0 + b0), this group's 32 columns
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                float v[16], bb[16];
                tc::ld_32x32b_x16(trow(d0, col0 + 16 * j), v);
                ld16(bias + col0 + 16 * j, bb);
                tc::wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = silu(v[i] + bb[i]);
                store_bf16x8(hbh + hb_off(t, col0 + 16 * j), v);
                store_bf16x8(hbh + hb_off(t, col0 + 16 * j + 8), v + 8);
            }
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            half_barrier2(h);
            if (issuer) {
                tc::fence_after_sync();
                issue_l1(sm, L, h, d1);
                tc::commit(&bar_mma[h]);
            }
            alive = wait_mma(&bar_mma[h], mma_phase, p.err) && alive;
            // last layer: partial z over this group's columns
            float a1[32];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                float v[16], bb[16];
                tc::ld_32x32b_x16(trow(d1, col0 + 16 * j), v);
                ld16(bias + kH + col0 + 16 * j, bb);
                tc::wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) a1[16 * j + i] = v[i] + bb[i];
            }
            // one logistic per element: a1 becomes silu(A1), gpk keeps
            // silu'(A1) (in [-0.1, 1.1]) as packed FP16 for dA1
            float zp = 0.f;
            __half2 gpk[16];
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
            s_z[h][grp][t] = zp;
            // a row's two partial sums meet within its quarter of the half's
            // rows (warps 8 h + q and 8 h + 4 + q)
            asm volatile("bar.sync %0, 64;" ::"r"(4 + 4 * h + ((tid >> 5) & 3)) : "memory");
            const float z = s_z[h][0][t] + s_z[h][1][t] + bias[3 * kH];
            const float dz = dIw * act_grad(lact, z, beta);
            // dA1 = dz w2 silu'(A1) into G columns col0..col0+31
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                float ww[16], da[16];
                ld16(bias + 2 * kH + col0 + 16 * j, ww);
#pragma unroll
                for (int i = 0; i < 16; i += 2) {
                    const float2 g = __half22float2(gpk[(16 * j + i) >> 1]);
                    da[i] = dz * ww[i] * g.x;
                    da[i + 1] = dz * ww[i + 1] * g.y;
                }
                store_bf16x8(gh + g_off(t, col0 + 16 * j), da);
                store_bf16x8(gh + g_off(t, col0 + 16 * j + 8), da + 8);
            }
            // last-layer weight gradient: reduce dz * silu(a1[k]) over the
            // warp's 32 rows, halving the value set each round; the lane ends
            // with one column
            {
#pragma unroll
                for (int k = 0; k < 32; ++k) a1[k] = dz * a1[k];
                int n = 32;
#pragma unroll
                for (int off = 16; off >= 1; off >>= 1) {
                    const bool upper = (lane & off) != 0;
                    n >>= 1;
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        if (k < n) {
                            const float send = upper ? a1[k] : a1[k + n];
                            const float keep = upper ? a1[k + n] : a1[k];
                            a1[k] = keep + __shfl_xor_sync(0xffffffffu, send, off);
                        }
                    }
                }
                gw2 += a1[0];
                if (grp == 0) {
                    float s = dz;
#pragma unroll
                    for (int off = 16; off >= 1; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
                    if (lane == 0) gb2 += s;
                }
            }
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            half_barrier2(h);
            if (issuer) {  // dH0 = dA1 W1 into the D1 columns
                tc::fence_after_sync();
                const uint32_t abase = tc::smem_addr(gh), bbase = tc::smem_addr(sm + L.w1);
#pragma unroll
                for (int j = 0; j < kH / 16; ++j) {
                    const uint64_t a = tc::smem_desc(abase + j * 256, 128, (kGCols / 8) * 128);
                    const uint64_t b = tc::smem_desc(bbase + j * 2 * (kH / 8) * 128, (kH / 8) * 128, 128);
                    tc::mma_bf16(d1, a, b, tc::idesc_bf16(kRows, kH, 0, 1), j > 0);
                }
                tc::commit(&bar_mma[h]);
            }
            alive = wait_mma(&bar_mma[h], mma_phase, p.err) && alive;
            // dA0 = dH0 silu'(A0) into G columns 64 + col0.. (A0 = D0 + b0)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                float gv[16], av[16], da[16], bb[16];
                tc::ld_32x32b_x16(trow(d1, col0 + 16 * j), gv);
                tc::ld_32x32b_x16(trow(d0, col0 + 16 * j), av);
                ld16(bias + col0 + 16 * j, bb);
                tc::wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) da[i] = gv[i] * silu_grad(av[i] + bb[i]);
                store_bf16x8(gh + g_off(t, kH + col0 + 16 * j), da);
                store_bf16x8(gh + g_off(t, kH + col0 + 16 * j + 8), da + 8);
            }
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            half_barrier2(h);
            if (issuer) {
                tc::fence_after_sync();
                // dX = dA0 W0 into the D0 columns 0..15
                const uint32_t abase = tc::smem_addr(gh + (kH / 8) * 128), bbase = tc::smem_addr(sm + L.w0);
#pragma unroll
                for (int j = 0; j < kH / 16; ++j) {
                    const uint64_t a = tc::smem_desc(abase + j * 256, 128, (kGCols / 8) * 128);
                    const uint64_t b = tc::smem_desc(bbase + j * 2 * (kC / 8) * 128, (kC / 8) * 128, 128);
                    tc::mma_bf16(d0, a, b, tc::idesc_bf16(kRows, kC, 0, 1), j > 0);
                }
                // [dW1 db1; dW0 db0] += [dA1 | dA0]^T [H0 | X | 1]
                const uint32_t gbase = tc::smem_addr(gh), hbase = tc::smem_addr(hbh);
#pragma unroll
                for (int j = 0; j < kRows / 16; ++j) {
                    const uint64_t a = tc::smem_desc(gbase + j * 2 * (kGCols / 8) * 128, (kGCols / 8) * 128, 128);
                    const uint64_t b = tc::smem_desc(hbase + j * 2 * (kHBCols / 8) * 128, (kHBCols / 8) * 128, 128);
                    tc::mma_bf16(dacc, a, b, tc::idesc_bf16(kRows, kHBCols, 1, 1), (had_tile || j > 0) ? 1u : 0u);
                }
                tc::commit(&bar_mma[h]);
            }
            had_tile = true;
            alive = wait_mma(&bar_mma[h], mma_phase, p.err) && alive;
            // scatter, phase 1 (own channels): dX * line values into the
            // scratch row, dX * plane values as the line MMA's B operand, and
            // (group 0) the tap column of the line MMA's A operand
            float dx[8];
            uint32_t pk[3][4];  // BF16 bilinear plane values kept by the feature step
            tc::ld_32x32b_x8(trow(d0, cb), dx);
            tc::wait_st();
#pragma unroll
            for (int m = 0; m < 3; ++m) tc::ld_32x32b_x4(stash + 4 * m, pk[m]);
            tc::wait_ld();
            if (real) {
                if (grp == 0) {
                    const uint4 z4 = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
                    for (int q = 0; q < 8; ++q) *reinterpret_cast<uint4*>(gh + g_off(t, 8 * q)) = z4;
                }
                float tsum = 0.f;  // sum of |dX * line value| of this thread's 24 values
                if (valid) {
#pragma unroll
                    for (int m = 0; m < 3; ++m) {
                        const int Ln = p.field.line_len[m];
                        float mat[8], vec[8], lv[8], gv[8];
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const float2 x = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&pk[m][i]));
                            mat[2 * i] = x.x;
                            mat[2 * i + 1] = x.y;
                        }
                        line_half(p, g, m, cb, vec);
#pragma unroll
                        for (int c = 0; c < 8; ++c) {
                            gv[c] = dx[c] * vec[c];
                            tsum += fabsf(gv[c]);
                        }
#pragma unroll
                        for (int q = 0; q < 2; ++q)
                            *reinterpret_cast<float4*>(scratch2(hbh, gh, t, 16 * m + cb + 4 * q)) =
                                make_float4(gv[4 * q], gv[4 * q + 1], gv[4 * q + 2], gv[4 * q + 3]);
#pragma unroll
                        for (int c = 0; c < 8; ++c) lv[c] = dx[c] * mat[c];
                        store_bf16x8(hbh + hb_off(t, 16 * m + cb), lv);
                        const Corner1 l = corners1(g.lu[m], Ln);
                        const int lo = s_lo[m];
                        const int i0 = l.x0 - lo, i1 = l.x1 - lo;
                        if (i0 >= 0 && i0 < kLineRowsTC && i1 >= 0 && i1 < kLineRowsTC) {
                            if (grp == 0) {
                                if (i0 == i1) {
                                    *reinterpret_cast<__nv_bfloat16*>(gh + g_off(t, m * kLineRowsTC + i0)) =
                                        __float2bfloat16_rn(l.w0 + l.w1);
                                } else {
                                    *reinterpret_cast<__nv_bfloat16*>(gh + g_off(t, m * kLineRowsTC + i0)) =
                                        __float2bfloat16_rn(l.w0);
                                    *reinterpret_cast<__nv_bfloat16*>(gh + g_off(t, m * kLineRowsTC + i1)) =
                                        __float2bfloat16_rn(l.w1);
                                }
                            }
                        } else {  // outside the item's window: straight to global
                            for (int c = 0; c < 8; ++c) {
                                atomicAdd(&p.gfield.line[m][l.x0 * C + cb + c], l.w0 * lv[c]);
                                atomicAdd(&p.gfield.line[m][l.x1 * C + cb + c], l.w1 * lv[c]);
                            }
                        }
                    }
                }
                // The bilinear weights of a sample sum to 1, so the tile adds at
                // most sum |dX * line value| to any texel of the slot.
#pragma unroll
                for (int off = 16; off >= 1; off >>= 1) tsum += __shfl_xor_sync(0xffffffffu, tsum, off);
                if (lane == 0) {
                    atomicAdd(&s_tcum[h], tsum);
                    if (handshake) atomicAdd(&s_tfirst[h], tsum);
                }
                tc::fence_smem_to_async();
                tc::fence_before_sync();
                if (handshake && both)
                    asm volatile("bar.sync 3, 512;" ::: "memory");
                else
                    half_barrier2(h);
                if (handshake) {
                    // scale = 2^e with the slot's expected total near 2^28 per
                    // half (the tiles of this half estimated from this item)
                    const float first = both ? 0.5f * (s_tfirst[0] + s_tfirst[1]) : s_tfirst[0];
                    const float tiles = fmaxf(1.f, ceilf((float)it.total * (float)it.slot_items / (2.f * kRows)));
                    int e = 20;
                    if (first > 0.f) e = ilogbf(268435456.0f / (first * tiles));
                    scale = ldexpf(1.0f, max(-100, min(e, 100)));
                    if (tid == 0) s_scale = scale;
                }
                // Overflow guard: a half may bring the slot's values at most
                // to 2^30 in magnitude (sum of its scaled |contributions| plus
                // half a unit of rounding per contribution); a tile beyond
                // that goes to global memory in FP32.
                ++ntiles;
                const bool to_smem =
                    s_tcum[h] * scale + (float)ntiles * (0.5f * kRows * 3 * 4 * kC) <= 1073741824.0f;
                if (!to_smem && issuer) s_fb = 1;
                if (issuer) {  // line gradients of the tile (overlaps the plane atomics)
                    tc::fence_after_sync();
                    const uint32_t abase = tc::smem_addr(gh), bbase = tc::smem_addr(hbh);
#pragma unroll
                    for (int j = 0; j < kRows / 16; ++j) {
                        const uint64_t a =
                            tc::smem_desc(abase + j * 2 * (kGCols / 8) * 128, (kGCols / 8) * 128, 128);
                        const uint64_t b =
                            tc::smem_desc(bbase + j * 2 * (kHBCols / 8) * 128, (kHBCols / 8) * 128, 128);
                        tc::mma_bf16(d1, a, b, tc::idesc_bf16(kRows, 3 * kC, 1, 1), j > 0 ? 1u : 0u);
                    }
                    tc::commit(&bar_mma[h]);
                }
                // scatter, phase 2: plane gradients as fixed-point integers
                // (shared-memory integer atomics run several times faster than
                // FP32 ones); group 0 adds the two upper corners, group 1 the
                // two lower ones. A texel's 16 channels fill one half of the
                // 32 banks (the half given by the parity of its index), and the two corners of a row have
                // opposite parities: lanes 0-15 take first the corner in banks
                // 0-15, lanes 16-31 the one in banks 16-31, and channel
                // (r + crot) mod 16 with crot a permutation of 0..15 within
                // each half-warp, so every warp-wide atomic touches 32 distinct
                // banks. crot mod 4 also differs among the four lanes that share
                // lane mod 8, which keeps the scratch-row reads conflict-free.
                if (valid) {
#pragma unroll 1
                    for (int m = 0; m < 3; ++m) {
                        const int Hm = p.field.plane_h[m], Wm = p.field.plane_w[m];
                        const Corner2 kc = corners2(g.pu[m], g.pv[m], Hm, Wm);
                        const int ya = grp == 0 ? kc.y0 : kc.y1;
                        const float wl = grp == 0 ? kc.w_nw : kc.w_sw, wr = grp == 0 ? kc.w_ne : kc.w_se;
                        const int tl = ya * Wm + kc.x0, tr = ya * Wm + kc.x1;
                        const bool swap = (tl & 1) != (lane >> 4);
                        const int ta = (swap ? tr : tl) * C, tb = (swap ? tl : tr) * C;
                        const float wa = swap ? wr : wl, wb = swap ? wl : wr;
                        if (to_smem) {
                            int* GP = gpl + p.gplane_off[m];
                            const float was = wa * scale, wbs = wb * scale;
#pragma unroll 4
                            for (int r = 0; r < kC; ++r) {
                                const int c = (r + crot) & (kC - 1);
                                const float v = *scratch2(hbh, gh, t, 16 * m + c);
                                atomicAdd(&GP[ta + c], __float2int_rn(was * v));
                                atomicAdd(&GP[tb + c], __float2int_rn(wbs * v));
                            }
                        } else {
                            float* GG = p.gfield.plane[m] + it.slot * (int64_t)(Hm * Wm * C);
                            for (int r = 0; r < kC; ++r) {
                                const float v = *scratch2(hbh, gh, t, 16 * m + r);
                                atomicAdd(&GG[ta + r], wa * v);
                                atomicAdd(&GG[tb + r], wb * v);
                            }
                        }
                    }
                }
                alive = wait_mma(&bar_mma[h], mma_phase, p.err) && alive;
                float v0[8], v1[8], v2[8];
                tc::ld_32x32b_x8(trow(d1, cb), v0);
                tc::ld_32x32b_x8(trow(d1, kC + cb), v1);
                tc::ld_32x32b_x8(trow(d1, 2 * kC + cb), v2);
                tc::wait_ld();
                if (t < 3 * kLineRowsTC) {
                    const int m = t / kLineRowsTC, i = t % kLineRowsTC;
                    float* dst = gln + (m * kLineWinTC + i) * C + cb;
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        const float v = m == 0 ? v0[c] : (m == 1 ? v1[c] : v2[c]);
                        if (v != 0.0f) atomicAdd(dst + c, v);
                    }
                }
            }
            tc::fence_before_sync();
            half_barrier2(h);
        }
        alive = __syncthreads_and(alive);
        if (real && it.last) {
            // this CTA owns the slot: plain stores, unless a tile went to
            // global memory directly
            const float sc = s_scale, inv = sc > 0.f ? 1.0f / sc : 0.f;  // exact: a power of two
            const bool fb = s_fb != 0;
            for (int m = 0; m < 3; ++m) {
                const int pf = p.field.plane_h[m] * p.field.plane_w[m] * C;
                float* dst = p.gfield.plane[m] + it.slot * (int64_t)pf;
                const int* src = gpl + p.gplane_off[m];
                for (int i = tid * 4; i < pf; i += kThreadsB2 * 4) {
                    const int4 q = *reinterpret_cast<const int4*>(src + i);
                    const float4 v = make_float4((float)q.x * inv, (float)q.y * inv, (float)q.z * inv, (float)q.w * inv);
                    if (fb)
                        atomicAdd(reinterpret_cast<float4*>(dst + i), v);
                    else
                        *reinterpret_cast<float4*>(dst + i) = v;
                }
                const int Ln = p.field.line_len[m];
                const int lo = s_lo[m];
                for (int i = tid; i < kLineWinTC * C; i += kThreadsB2) {
                    const int e = lo + i / C;
                    const float v = gln[m * kLineWinTC * C + i];
                    if (e < Ln && v != 0.0f) atomicAdd(&p.gfield.line[m][e * C + (i % C)], v);
                }
            }
        }
        __syncthreads();
    }
    // decoder gradients: the TMEM accumulator rows of this half (group 0 reads
    // columns 0..47, group 1 columns 48..95)
    if (had_tile) {
        tc::fence_after_sync();
#pragma unroll
        for (int jj = 0; jj < 3; ++jj) {
            const int j = 3 * grp + jj;
            float v[16];
            tc::ld_32x32b_x16(trow(dacc, 16 * j), v);
            tc::wait_ld();
            if (t < kH) {  // rows 0..63: dW1 (cols 0..63), db1 (col 80)
                if (j < 4)
#pragma unroll
                    for (int i = 0; i < 16; ++i) atomicAdd(&p.gmlp.weight[1][t * kH + 16 * j + i], v[i]);
                if (j == 5) atomicAdd(&p.gmlp.bias[1][t], v[0]);
            } else {  // rows 64..127: dW0 (cols 64..79), db0 (col 80)
                const int n = t - kH;
                if (j == 4)
#pragma unroll
                    for (int i = 0; i < 16; ++i) atomicAdd(&p.gmlp.weight[0][n * kC + i], v[i]);
                if (j == 5) atomicAdd(&p.gmlp.bias[0][n], v[0]);
            }
        }
    }
    // last layer: lane l's column within its group's 32, by the halving order above
    {
        int colbits = 0;
        for (int off = 16, b = 0; off >= 1; off >>= 1, ++b)
            if (lane & off) colbits |= (32 >> (b + 1));
        atomicAdd(&p.gmlp.weight[2][col0 + colbits], gw2);
        if (grp == 0 && lane == 0) atomicAdd(&p.gmlp.bias[2][0], gb2);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid < 32) tc::tmem_dealloc(s_tmem, kTmemBwd);
}

}  // namespace tcf

bool tc_supported(const atdf_field_t* f, const atdf_mlp_t* m)
{
    if (tc24_supported(f, m)) return true;
    return f->dtype == ATDF_BF16 && f->channels == tcf::kC && f->mode == 0 && m->num_layers == 3 &&
           m->dims[0] == tcf::kC && m->dims[1] == tcf::kH && m->dims[2] == tcf::kH && m->dims[3] == 1 &&
           m->hidden_activation == ATDF_ACT_SILU;
}

static int max_optin()
{
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

static int launch_tc(void (*fn)(FusedParams), bool bwd, const FusedParams& p, cudaStream_t st,
                     int threads = tcf::kThreadsTC)
{
    const int smem = (int)tcf::TCSmem(p.plane_off[3], p.gplane_off[3], bwd).total;
    if (smem > max_optin()) return ATDF_ERR_UNSUPPORTED;
    ATDF_CUDA_TRY(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    // without an explicit carveout the occupancy query assumes a smaller
    // shared-memory partition and reports one forward CTA per SM
    ATDF_CUDA_TRY(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared));
    int dev = 0, sms = 0, per = 0;
    ATDF_CUDA_TRY(cudaGetDevice(&dev));
    ATDF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    ATDF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)fn, threads, smem));
    if (per < 1) return ATDF_ERR_UNSUPPORTED;
    // TMEM: 256 columns per forward CTA, 512 per backward CTA (512 per SM).
    // The forward fits two CTAs per SM by shared memory and registers
    // (launch bounds); the occupancy query reports one, so size it here.
    int smem_sm = 0;
    ATDF_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    per = bwd ? 1 : std::max(1, std::min(2, smem_sm / (smem + 1024)));
    fn<<<sms * per, threads, smem, st>>>(p);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int launch_tc_forward(const FusedParams& p, cudaStream_t st)
{
    if (p.field.channels == 24) return launch_tc24_forward(p, st);
    return launch_tc(tcf::tc_forward_kernel, false, p, st);
}
// The backward runs two threads per sample row (512 threads per CTA).
int launch_tc_backward(const FusedParams& p, cudaStream_t st)
{
    if (p.field.channels == 24) return launch_tc24_backward(p, st);
    return launch_tc(tcf::tc_backward2_kernel, true, p, st, tcf::kThreadsB2);
}

}  // namespace atdf
