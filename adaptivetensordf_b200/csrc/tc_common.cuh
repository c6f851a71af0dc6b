// Device helpers shared by the tensor-core projection kernels (fused_tc.cu
// for 16 channels, fused_tc24.cu for 24): bounded MMA waits, BF16 packing,
// the logistic function from the hardware tanh approximation, bilinear
// corner addressing and the TMEM row address of a thread.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "fused_common.cuh"
#include "tc.cuh"

namespace atdf {
namespace tcf {

__device__ __forceinline__ bool wait_mma(uint64_t* bar, uint32_t& phase, int32_t* err)
{
    const bool ok = mbar_wait(bar, phase);
    phase ^= 1;
    if (!ok) set_err(err, ATDF_DEVERR_TREE);
    tc::fence_after_sync();
    return ok;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void unpack_bf16x8(const uint4& u, float* f)
{
    const __nv_bfloat162* p = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 x = __bfloat1622float2(p[i]);
        f[2 * i] = x.x;
        f[2 * i + 1] = x.y;
    }
}

// 8 FP32 values -> 8 BF16 at a 16-byte aligned shared address.
__device__ __forceinline__ void store_bf16x8(unsigned char* dst, const float* v)
{
    uint4 u;
    u.x = pack_bf16(v[0], v[1]);
    u.y = pack_bf16(v[2], v[3]);
    u.z = pack_bf16(v[4], v[5]);
    u.w = pack_bf16(v[6], v[7]);
    *reinterpret_cast<uint4*>(dst) = u;
}

// Logistic function from the hardware tanh approximation (one MUFU op,
// ~2^-11 relative error, below the BF16 rounding of the activations).
__device__ __forceinline__ float sigmoid_tanh(float x)
{
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(0.5f * x));
    return fmaf(0.5f, y, 0.5f);
}
__device__ __forceinline__ float silu(float x) { return x * sigmoid_tanh(x); }
__device__ __forceinline__ float silu_grad(float x)
{
    const float s = sigmoid_tanh(x);
    return s * (1.0f + x * (1.0f - s));
}

// 16 consecutive floats of the bias block (16-byte aligned) into registers.
__device__ __forceinline__ void ld16(const float* src, float (&v)[16])
{
    const float4* s4 = reinterpret_cast<const float4*>(src);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 x = s4[q];
        v[4 * q] = x.x;
        v[4 * q + 1] = x.y;
        v[4 * q + 2] = x.z;
        v[4 * q + 3] = x.w;
    }
}

// Texel index (padded rows of pitch Wp) and weight of corner o of a bilinear
// footprint: 0 = (y0, x0), 1 = (y0, x1), 2 = (y1, x0), 3 = (y1, x1).
__device__ __forceinline__ int corner_texel(const Corner2& k, int o, int Wp, float& w)
{
    w = o == 0 ? k.w_nw : (o == 1 ? k.w_ne : (o == 2 ? k.w_sw : k.w_se));
    return ((o & 2) ? k.y1 : k.y0) * Wp + ((o & 1) ? k.x1 : k.x0);
}

// TMEM address of this thread's accumulator row at column col of a half.
__device__ __forceinline__ uint32_t trow(uint32_t base, int col)
{
    const int warp = threadIdx.x >> 5;
    return base + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)col;
}

}  // namespace tcf
}  // namespace atdf
