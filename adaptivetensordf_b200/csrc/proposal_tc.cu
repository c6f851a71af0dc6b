// The proposal MLP (16 -> 64 -> 64 -> 64 -> 33, SiLU hidden, identity last)
// on the 5th-generation tensor cores: BF16 operands in shared memory, FP32
// accumulation in TMEM, 128 segment rows per tile (one TMEM lane per row).
//
// Forward (128 threads, one per row):
//   X[128x16] -> Z0 = X W0^T -> A0 = silu(Z0 + b0) -> ... -> A2 -> A2 W3^T + b3
// Backward (256 threads, two per row, each taking half of a layer's columns):
//   recompute Z0..Z2 (kept in TMEM) and A0..A2 (BF16, shared), then
//   dZ3 = dlogits,  dA_{l} = dZ_{l+1} W_{l+1},  dZ_l = dA_l * silu'(Z_l + b_l)
//   [dW3 db3; dW2 db2] += [dZ3 | dZ2]^T [A2 | A1 | 1]     (one M = 128 MMA)
//   [dW1 db1; dW0 db0] += [dZ1 | dZ0]^T [A0 | X  | 1]     (one M = 128 MMA)
// accumulated in TMEM across all tiles of the CTA (the off-diagonal blocks
// of the two products are computed and ignored) and added to the global
// gradients once per CTA. The buffers use the no-swizzle core-matrix layouts
// of tc.cuh, so each serves as a K-major operand of the layer GEMMs and, as
// the same bytes, as an MN-major operand of the weight-gradient GEMMs:
//   HBQ [128 x 96]  = A0 (0..63) | X (64..79) | 1 (80) | 0
//   HBP [128 x 144] = A2 (0..63) | A1 (64..127) | 1 (128) | 0
//   GP  [128 x 128] = dZ3 (0..32, zero to 63) | dZ2 (64..127)
//   GQ  [128 x 128] = dZ1 (0..63) | dZ0 (64..127)
// and the weights W_l [out][in] BF16 (K-major for the forward, MN-major for
// dA = dZ W), W3 padded to 64 output rows with zeros.
//
// The FP32 CUDA-core kernels of proposal.cu compute the same functions for
// 1 to 3 hidden layers; these take the BF16 rounding of the operands (the
// tolerance of the BF16 form) in exchange for the tensor-core throughput.

#include <cuda_bf16.h>

#include <algorithm>

#include "fused_common.cuh"
#include "tc.cuh"

namespace atdf {
namespace ptc {

constexpr int kIn = ATDF_PROPOSAL_INPUTS;   // 16
constexpr int kOut = ATDF_PROPOSAL_OUTPUTS; // 33
constexpr int kH = 64;
constexpr int kRows = 128;
constexpr int kOutN = 48;                   // forward last-layer N (33 padded to a multiple of 16)
constexpr int kHBQ = 96, kHBP = 144, kG = 128;
constexpr uint32_t kTmemFwd = 64;
constexpr uint32_t kTmemBwd = 512;
// backward TMEM columns
constexpr uint32_t kZ0 = 0, kZ1 = 64, kZ2 = 128, kD = 192, kDP = 256, kDQ = 400;

struct Mlp4 {
    const float* w[4];
    const float* b[4];
    float* gw[4];
    float* gb[4];
};

// shared-memory byte offsets
constexpr uint32_t kW0 = 0;
constexpr uint32_t kW1 = kW0 + kH * kIn * 2;
constexpr uint32_t kW2 = kW1 + kH * kH * 2;
constexpr uint32_t kW3 = kW2 + kH * kH * 2;
constexpr uint32_t kBias = kW3 + kH * kH * 2;          // b0 b1 b2 b3, 64 floats each
constexpr uint32_t kBufs = kBias + 4 * kH * 4;
// forward buffers
constexpr uint32_t kFX = kBufs;                        // [128 x 16]
constexpr uint32_t kFA = kFX + kRows * kIn * 2;        // [128 x 64]
constexpr uint32_t kFStage = kFA + kRows * kH * 2;     // [128 x 33] float
constexpr uint32_t kFwdSmem = kFStage + kRows * kOut * 4;
// backward buffers
constexpr uint32_t kBHBQ = kBufs;
constexpr uint32_t kBHBP = kBHBQ + kRows * kHBQ * 2;
constexpr uint32_t kBGP = kBHBP + kRows * kHBP * 2;
constexpr uint32_t kBGQ = kBGP + kRows * kG * 2;
constexpr uint32_t kBwdSmem = kBGQ + kRows * kG * 2;
static_assert(kFwdSmem <= 227 * 1024 && kBwdSmem <= 227 * 1024, "shared memory");
static_assert(kDQ + kHBQ <= kTmemBwd, "TMEM columns");

__device__ __forceinline__ uint32_t trow(uint32_t base, uint32_t col)
{
    const int warp = threadIdx.x >> 5;
    return base + ((uint32_t)(32 * (warp & 3)) << 16) + col;
}

__device__ __forceinline__ uint32_t pack2(float a, float b)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void st8(unsigned char* dst, const float* v)
{
    *reinterpret_cast<uint4*>(dst) = make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]),
                                                 pack2(v[6], v[7]));
}

// Logistic function from the hardware tanh approximation (one MUFU op,
// ~2^-11 relative error, below the BF16 rounding of the activations).
__device__ __forceinline__ float sig(float z)
{
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(0.5f * z));
    return fmaf(0.5f, y, 0.5f);
}
__device__ __forceinline__ float silu_f(float z) { return z * sig(z); }
__device__ __forceinline__ float dsilu(float z)
{
    const float s = sig(z);
    return s * (1.0f + z * (1.0f - s));
}

// Weights as BF16 K-major [out][in] (W3 padded to 64 rows), biases FP32.
// Four consecutive inputs per load (rows of 16 or 64 floats, 16-byte
// aligned), eight loads in flight per thread: this runs once per CTA, and a
// chain of dependent global loads here would cost more than a tile.
__device__ void load_weights(const Mlp4& m, unsigned char* sm, int nthreads)
{
    constexpr int kQ0 = kH * kIn / 4, kQh = kH * kH / 4, kQ = kQ0 + 3 * kQh;  // float4s of W0 and W1..W3
    for (int e0 = threadIdx.x; e0 < kQ; e0 += 8 * nthreads) {
        float4 v[8];
        int l[8], n[8], k[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * nthreads;
            l[u] = e < kQ0 ? 0 : 1 + (e - kQ0) / kQh;
            const int Kl = l[u] == 0 ? kIn : kH;
            const int q = l[u] == 0 ? e : (e - kQ0) % kQh;
            n[u] = (4 * q) / Kl;
            k[u] = (4 * q) % Kl;
            const int O = l[u] == 3 ? kOut : kH;
            v[u] = (e < kQ && n[u] < O) ? *reinterpret_cast<const float4*>(m.w[l[u]] + n[u] * Kl + k[u])
                                        : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (e0 + u * nthreads >= kQ) continue;
            const uint32_t off = l[u] == 0 ? kW0 : l[u] == 1 ? kW1 : l[u] == 2 ? kW2 : kW3;
            const int Kl = l[u] == 0 ? kIn : kH;
            *reinterpret_cast<uint2*>(sm + off + tc::kmajor_off(n[u], k[u], Kl)) =
                make_uint2(pack2(v[u].x, v[u].y), pack2(v[u].z, v[u].w));
        }
    }
    float* b = reinterpret_cast<float*>(sm + kBias);
    for (int i = threadIdx.x; i < 4 * kH; i += nthreads) {
        const int l = i / kH, o = i % kH;
        b[i] = o < (l == 3 ? kOut : kH) ? m.b[l][o] : 0.0f;
    }
}

__device__ __forceinline__ void ld16(const float* src, float (&v)[16])
{
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 x = *reinterpret_cast<const float4*>(src + 4 * q);
        v[4 * q] = x.x;
        v[4 * q + 1] = x.y;
        v[4 * q + 2] = x.z;
        v[4 * q + 3] = x.w;
    }
}

// D = A[128 x K] W^T with A K-major at a_addr (row pitch a_cols) and W
// K-major [N][K]: one MMA per 16 columns of K.
__device__ __forceinline__ void gemm_kmajor(uint32_t d, uint32_t a_addr, int a_cols, uint32_t w_addr, int K, int N)
{
    for (int j = 0; j < K / 16; ++j) {
        const uint64_t a = tc::smem_desc(a_addr + j * 256, 128, (a_cols / 8) * 128);
        const uint64_t b = tc::smem_desc(w_addr + j * 256, 128, (K / 8) * 128);
        tc::mma_bf16(d, a, b, tc::idesc_bf16(kRows, N, 0, 0), j > 0);
    }
}

// D = dZ[128 x 64] W with dZ K-major at a_addr (row pitch kG) and W [64
// out][64 in] read MN-major (N = in, K = out).
__device__ __forceinline__ void gemm_back(uint32_t d, uint32_t a_addr, uint32_t w_addr)
{
    for (int j = 0; j < kH / 16; ++j) {
        const uint64_t a = tc::smem_desc(a_addr + j * 256, 128, (kG / 8) * 128);
        const uint64_t b = tc::smem_desc(w_addr + j * 2 * (kH / 8) * 128, (kH / 8) * 128, 128);
        tc::mma_bf16(d, a, b, tc::idesc_bf16(kRows, kH, 0, 1), j > 0);
    }
}

// D (+)= G^T HB over the 128 rows: G [128 x 128] and HB [128 x N] both read MN-major.
__device__ __forceinline__ void gemm_wgrad(uint32_t d, uint32_t g_addr, uint32_t hb_addr, int N, bool acc)
{
    for (int j = 0; j < kRows / 16; ++j) {
        const uint64_t a = tc::smem_desc(g_addr + j * 2 * (kG / 8) * 128, (kG / 8) * 128, 128);
        const uint64_t b = tc::smem_desc(hb_addr + j * 2 * (N / 8) * 128, (N / 8) * 128, 128);
        tc::mma_bf16(d, a, b, tc::idesc_bf16(kRows, N, 1, 1), (acc || j > 0) ? 1u : 0u);
    }
}

__device__ __forceinline__ bool wait_bar(uint64_t* bar, uint32_t& phase, int32_t* err)
{
    const bool ok = mbar_wait(bar, phase);
    phase ^= 1;
    if (!ok) set_err(err, ATDF_DEVERR_TREE);
    tc::fence_after_sync();
    return ok;
}

// After a timed-out wait (alive false, block-uniform): the issuing thread
// commits once more, so the barrier's next phase completes when every MMA it
// issued has, and the block waits for that (bounded) before freeing TMEM.
__device__ __forceinline__ void drain_on_timeout(bool alive, uint64_t* bar, uint32_t phase, bool issuer)
{
    if (alive) return;
    if (issuer) tc::commit(bar);
    mbar_wait(bar, phase);
}

__device__ __forceinline__ void to_async_and_sync()
{
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
}

// Hidden-layer epilogue of `ncol` columns from col0: A = silu(Z + b) -> BF16
// at column dst_col0 of a K-major buffer with row pitch pitch.
__device__ __forceinline__ void hidden_epilogue(unsigned char* sm, uint32_t zaddr, const float* b, int col0, int ncol,
                                                unsigned char* buf, int pitch, int dst_col0, int t)
{
    for (int j = 0; j < ncol / 16; ++j) {
        float v[16], bb[16];
        tc::ld_32x32b_x16(trow(zaddr, col0 + 16 * j), v);
        ld16(b + col0 + 16 * j, bb);
        tc::wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = silu_f(v[i] + bb[i]);
        st8(buf + tc::kmajor_off(t, dst_col0 + 16 * j, pitch), v);
        st8(buf + tc::kmajor_off(t, dst_col0 + 16 * j + 8, pitch), v + 8);
    }
}

__global__ void __launch_bounds__(kRows) prop_tc_forward_kernel(Mlp4 m, const int64_t* __restrict__ count,
                                                                const float* __restrict__ x, float* __restrict__ out,
                                                                int32_t* err)
{
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t s_tmem;
    const int t = threadIdx.x;
    if (t < 32) tc::tmem_alloc(&s_tmem, kTmemFwd);
    if (t == 0) mbar_init(&bar, 1);
    load_weights(m, sm, kRows);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t d = s_tmem;
    const float* bias = reinterpret_cast<const float*>(sm + kBias);
    float* stage = reinterpret_cast<float*>(sm + kFStage);
    const uint32_t xa = tc::smem_addr(sm + kFX), aa = tc::smem_addr(sm + kFA);
    const int64_t nrows = *count;
    uint32_t phase = 0;
    bool alive = true;
    // this thread's row of the next tile, loaded while the current one runs
    float v[16];
    auto fetch = [&](int64_t r0) {
        const int64_t row = r0 + t;
        if (row < nrows)
            ld16(x + row * kIn, v);
        else
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = 0.0f;
    };
    fetch((int64_t)blockIdx.x * kRows);
    for (int64_t row0 = (int64_t)blockIdx.x * kRows; alive && row0 < nrows; row0 += (int64_t)gridDim.x * kRows) {
        st8(sm + kFX + tc::kmajor_off(t, 0, kIn), v);
        st8(sm + kFX + tc::kmajor_off(t, 8, kIn), v + 8);
        fetch(row0 + (int64_t)gridDim.x * kRows);
#pragma unroll 1
        for (int l = 0; l < 4; ++l) {
            to_async_and_sync();
            if (t == 0) {
                if (l == 0)
                    gemm_kmajor(d, xa, kIn, tc::smem_addr(sm + kW0), kIn, kH);
                else
                    gemm_kmajor(d, aa, kH, tc::smem_addr(sm + (l == 1 ? kW1 : l == 2 ? kW2 : kW3)), kH,
                                l == 3 ? kOutN : kH);
                tc::commit(&bar);
            }
            alive = wait_bar(&bar, phase, err) && alive;
            if (l < 3) {
                hidden_epilogue(sm, d, bias + l * kH, 0, kH, sm + kFA, kH, 0, t);
            } else {
                for (int j = 0; j < kOutN / 16; ++j) {
                    float o[16], bb[16];
                    tc::ld_32x32b_x16(trow(d, 16 * j), o);
                    ld16(bias + 3 * kH + 16 * j, bb);
                    tc::wait_ld();
#pragma unroll
                    for (int i = 0; i < 16; ++i)
                        if (16 * j + i < kOut) stage[t * kOut + 16 * j + i] = o[i] + bb[i];
                }
            }
        }
        tc::fence_before_sync();
        __syncthreads();
        // coalesced copy of the tile's logits
        const int nvalid = nrows - row0 < kRows ? (int)(nrows - row0) : kRows;
        for (int e = t; e < nvalid * kOut; e += kRows) out[row0 * kOut + e] = stage[e];
        alive = __syncthreads_and(alive);
    }
    drain_on_timeout(alive, &bar, phase, t == 0);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (t < 32) tc::tmem_dealloc(s_tmem, kTmemFwd);
}

__global__ void __launch_bounds__(2 * kRows, 1) prop_tc_backward_kernel(Mlp4 m, const int64_t* __restrict__ count,
                                                                       const float* __restrict__ x,
                                                                       const float* __restrict__ gout, int32_t* err)
{
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, h = tid / kRows, t = tid % kRows;
    if (tid < 32) tc::tmem_alloc(&s_tmem, kTmemBwd);
    if (tid == 0) mbar_init(&bar, 1);
    load_weights(m, sm, 2 * kRows);
    unsigned char* HBQ = sm + kBHBQ;
    unsigned char* HBP = sm + kBHBP;
    unsigned char* GP = sm + kBGP;
    unsigned char* GQ = sm + kBGQ;
    // constant columns: the ones column and its zero padding of HBQ and HBP
    {
        float c[8] = {h == 0 ? 1.0f : 0.0f, 0, 0, 0, 0, 0, 0, 0}, z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        st8(HBQ + tc::kmajor_off(t, 80 + 8 * h, kHBQ), h == 0 ? c : z);
        st8(HBP + tc::kmajor_off(t, 128 + 8 * h, kHBP), h == 0 ? c : z);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = s_tmem;
    const float* bias = reinterpret_cast<const float*>(sm + kBias);
    const uint32_t hbq = tc::smem_addr(HBQ), hbp = tc::smem_addr(HBP), gp = tc::smem_addr(GP), gq = tc::smem_addr(GQ);
    const int64_t nrows = *count;
    const int c0 = 32 * h;  // this thread's half of a 64-column layer
    uint32_t phase = 0;
    bool alive = true, had_tile = false;
    // this thread's X half (8 features) and dZ3 half (32 logits, zero past
    // 33) of the next tile, loaded while the current one runs
    float xv[8], gv[32];
    auto fetch = [&](int64_t r0) {
        const int64_t row = r0 + t;
        const bool in = row < nrows;
#pragma unroll
        for (int i = 0; i < 8; ++i) xv[i] = in ? x[row * kIn + 8 * h + i] : 0.0f;
#pragma unroll
        for (int i = 0; i < 32; ++i) gv[i] = (in && c0 + i < kOut) ? gout[row * kOut + c0 + i] : 0.0f;
    };
    fetch((int64_t)blockIdx.x * kRows);
    for (int64_t row0 = (int64_t)blockIdx.x * kRows; alive && row0 < nrows; row0 += (int64_t)gridDim.x * kRows) {
        st8(HBQ + tc::kmajor_off(t, 64 + 8 * h, kHBQ), xv);
#pragma unroll
        for (int q = 0; q < 4; ++q) st8(GP + tc::kmajor_off(t, c0 + 8 * q, kG), gv + 8 * q);
        fetch(row0 + (int64_t)gridDim.x * kRows);
        // forward: Z0, Z1, Z2 into TMEM, A0 -> HBQ, A1 -> HBP[64..], A2 -> HBP[0..]
        to_async_and_sync();
        if (tid == 0) {
            gemm_kmajor(tm + kZ0, hbq + (64 / 8) * 128, kHBQ, tc::smem_addr(sm + kW0), kIn, kH);
            tc::commit(&bar);
        }
        alive = wait_bar(&bar, phase, err) && alive;
        hidden_epilogue(sm, tm + kZ0, bias, c0, 32, HBQ, kHBQ, c0, t);
        to_async_and_sync();
        if (tid == 0) {
            gemm_kmajor(tm + kZ1, hbq, kHBQ, tc::smem_addr(sm + kW1), kH, kH);
            tc::commit(&bar);
        }
        alive = wait_bar(&bar, phase, err) && alive;
        hidden_epilogue(sm, tm + kZ1, bias + kH, c0, 32, HBP, kHBP, 64 + c0, t);
        to_async_and_sync();
        if (tid == 0) {
            gemm_kmajor(tm + kZ2, hbp + (64 / 8) * 128, kHBP, tc::smem_addr(sm + kW2), kH, kH);
            // dA2 = dZ3 W3 does not depend on the forward
            gemm_back(tm + kD, gp, tc::smem_addr(sm + kW3));
            tc::commit(&bar);
        }
        alive = wait_bar(&bar, phase, err) && alive;
        hidden_epilogue(sm, tm + kZ2, bias + 2 * kH, c0, 32, HBP, kHBP, c0, t);
        // dZ_l = dA_l * silu'(Z_l + b_l) for l = 2, 1, 0
#pragma unroll 1
        for (int l = 2; l >= 0; --l) {
            unsigned char* dst = l == 2 ? GP + 0 : GQ;
            const int dcol = l == 2 ? 64 : l == 1 ? 0 : 64;
            const uint32_t zcol = l == 2 ? kZ2 : l == 1 ? kZ1 : kZ0;
            for (int j = 0; j < 2; ++j) {
                float da[16], z[16], bb[16];
                tc::ld_32x32b_x16(trow(tm + kD, c0 + 16 * j), da);
                tc::ld_32x32b_x16(trow(tm + zcol, c0 + 16 * j), z);
                ld16(bias + l * kH + c0 + 16 * j, bb);
                tc::wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) da[i] *= dsilu(z[i] + bb[i]);
                st8(dst + tc::kmajor_off(t, dcol + c0 + 16 * j, kG), da);
                st8(dst + tc::kmajor_off(t, dcol + c0 + 16 * j + 8, kG), da + 8);
            }
            to_async_and_sync();
            if (tid == 0) {
                if (l == 2) {
                    gemm_back(tm + kD, gp + (64 / 8) * 128, tc::smem_addr(sm + kW2));  // dA1 = dZ2 W2
                    gemm_wgrad(tm + kDP, gp, hbp, kHBP, had_tile);                   // [dW3;dW2]
                } else if (l == 1) {
                    gemm_back(tm + kD, gq, tc::smem_addr(sm + kW1));  // dA0 = dZ1 W1
                } else {
                    gemm_wgrad(tm + kDQ, gq, hbq, kHBQ, had_tile);   // [dW1;dW0]
                }
                tc::commit(&bar);
            }
            // the last wait also covers the weight-gradient MMAs that read the buffers
            alive = wait_bar(&bar, phase, err) && alive;
        }
        had_tile = true;
        alive = __syncthreads_and(alive);
    }
    // Add this CTA's weight gradients: D_P lanes 0..63 = layer 3 (rows < 33),
    // 64..127 = layer 2; D_Q lanes 0..63 = layer 1, 64..127 = layer 0.
    if (alive && had_tile) {
        const int lane = t;  // TMEM lane of this thread
        const bool lo = lane < 64;
        const int o = lo ? lane : lane - 64;
        {  // D_P
            float* gw = lo ? m.gw[3] : m.gw[2];
            float* gb = lo ? m.gb[3] : m.gb[2];
            const bool ok = !lo || o < kOut;
            const int ncol0 = lo ? 0 : 64;
            for (int j = 0; j < 2; ++j) {
                float v[16];
                tc::ld_32x32b_x16(trow(tm + kDP, ncol0 + c0 + 16 * j), v);
                tc::wait_ld();
                if (ok)
#pragma unroll
                    for (int i = 0; i < 16; ++i) atomicAdd(&gw[o * kH + c0 + 16 * j + i], v[i]);
            }
            if (h == 0) {
                float v[16];
                tc::ld_32x32b_x16(trow(tm + kDP, 128), v);
                tc::wait_ld();
                if (ok) atomicAdd(&gb[o], v[0]);
            }
        }
        {  // D_Q
            if (lo) {
                for (int j = 0; j < 2; ++j) {
                    float v[16];
                    tc::ld_32x32b_x16(trow(tm + kDQ, c0 + 16 * j), v);
                    tc::wait_ld();
#pragma unroll
                    for (int i = 0; i < 16; ++i) atomicAdd(&m.gw[1][o * kH + c0 + 16 * j + i], v[i]);
                }
            } else {
                float v[16];
                tc::ld_32x32b_x16(trow(tm + kDQ, 64), v);
                tc::wait_ld();
#pragma unroll
                for (int i = 0; i < 8; ++i) atomicAdd(&m.gw[0][o * kIn + 8 * h + i], v[8 * h + i]);
            }
            if (h == 0) {
                float v[16];
                tc::ld_32x32b_x16(trow(tm + kDQ, 80), v);
                tc::wait_ld();
                atomicAdd(lo ? &m.gb[1][o] : &m.gb[0][o], v[0]);
            }
        }
    }
    drain_on_timeout(alive, &bar, phase, tid == 0);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid < 32) tc::tmem_dealloc(s_tmem, kTmemBwd);
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

static int check_mlp(const atdf_mlp_t* m)
{
    if (!m || m->num_layers != 4 || m->dims[0] != kIn || m->dims[4] != kOut) return ATDF_ERR_UNSUPPORTED;
    for (int l = 1; l < 4; ++l)
        if (m->dims[l] != kH) return ATDF_ERR_UNSUPPORTED;
    if (m->hidden_activation != ATDF_ACT_SILU || m->last_activation != ATDF_ACT_ID) return ATDF_ERR_UNSUPPORTED;
    for (int l = 0; l < 4; ++l)
        if (!m->weight[l] || !m->bias[l] || !aligned16(m->weight[l])) return ATDF_ERR_INVALID_ARGUMENT;
    return ATDF_OK;
}

static int sm_count(int& sms)
{
    int dev = 0;
    ATDF_CUDA_TRY(cudaGetDevice(&dev));
    ATDF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return ATDF_OK;
}

}  // namespace ptc
}  // namespace atdf

using namespace atdf;
using namespace atdf::ptc;

extern "C" {

int atdf_proposal_mlp_forward_bf16(const atdf_mlp_t* mlp, const atdf_segments_t* segments, const float* features,
                                   float* logits, int32_t* dev_error, atdf_stream_t stream)
{
    if (!segments || !segments->totals || !features || !logits || !dev_error || !aligned16(features))
        return ATDF_ERR_INVALID_ARGUMENT;
    int st = check_mlp(mlp);
    if (st != ATDF_OK) return st;
    Mlp4 m{};
    for (int l = 0; l < 4; ++l) {
        m.w[l] = mlp->weight[l];
        m.b[l] = mlp->bias[l];
    }
    int sms = 0;
    if ((st = sm_count(sms)) != ATDF_OK) return st;
    ATDF_CUDA_TRY(cudaFuncSetAttribute((const void*)prop_tc_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kFwdSmem));
    const int64_t tiles = std::max<int64_t>(1, div_up(segments->capacity, kRows));
    const unsigned grid = (unsigned)std::min<int64_t>(tiles, (int64_t)sms * 3);
    prop_tc_forward_kernel<<<grid, kRows, kFwdSmem, (cudaStream_t)stream>>>(m, segments->totals, features, logits,
                                                                            dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_proposal_mlp_backward_bf16(const atdf_mlp_t* mlp, const atdf_segments_t* segments, const float* features,
                                    const float* grad_logits, const atdf_mlp_grad_t* grad_mlp, int32_t* dev_error,
                                    atdf_stream_t stream)
{
    if (!segments || !segments->totals || !features || !grad_logits || !grad_mlp || !dev_error)
        return ATDF_ERR_INVALID_ARGUMENT;
    int st = check_mlp(mlp);
    if (st != ATDF_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    Mlp4 m{};
    for (int l = 0; l < 4; ++l) {
        if (!grad_mlp->weight[l] || !grad_mlp->bias[l]) return ATDF_ERR_INVALID_ARGUMENT;
        m.w[l] = mlp->weight[l];
        m.b[l] = mlp->bias[l];
        m.gw[l] = grad_mlp->weight[l];
        m.gb[l] = grad_mlp->bias[l];
        ATDF_CUDA_TRY(cudaMemsetAsync(m.gw[l], 0, (size_t)mlp->dims[l] * mlp->dims[l + 1] * sizeof(float), s));
        ATDF_CUDA_TRY(cudaMemsetAsync(m.gb[l], 0, (size_t)mlp->dims[l + 1] * sizeof(float), s));
    }
    int sms = 0;
    if ((st = sm_count(sms)) != ATDF_OK) return st;
    ATDF_CUDA_TRY(cudaFuncSetAttribute((const void*)prop_tc_backward_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBwdSmem));
    const int64_t tiles = std::max<int64_t>(1, div_up(segments->capacity, kRows));
    const unsigned grid = (unsigned)std::min<int64_t>(tiles, (int64_t)sms);
    prop_tc_backward_kernel<<<grid, 2 * kRows, kBwdSmem, s>>>(m, segments->totals, features, grad_logits, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

}  // extern "C"
