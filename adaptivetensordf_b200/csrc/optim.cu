// Adam step over one parameter tensor that also writes the parameter's BF16
// working copy, so that the BF16 form's training step reads and writes each
// parameter's optimizer state once (torch.optim.Adam's update followed by a
// separate FP32 -> BF16 cast pass reads the parameters a second time).
//
// The update is torch.optim.Adam's (no amsgrad, L2 weight decay added to
// the gradient), the optimizer the reference builds for the grid and decoder
// parameters (geometry_tensor_qo.cpp:79-81, 209-220):
//   g' = g + wd * p
//   m  = b1 * m + (1 - b1) * g'
//   v  = b2 * v + (1 - b2) * g'^2
//   p -= (lr / (1 - b1^t)) * m / (sqrt(v) / sqrt(1 - b2^t) + eps)
// One pass, HBM-bound: 16 bytes read and 12 written per element (+2 for the
// BF16 copy).

#include <cuda_bf16.h>

#include <cmath>

#include "atdf_common.cuh"

namespace atdf {

struct AdamArgs {
    float lr_t;        // lr / (1 - b1^t)
    float b1, b2, eps;
    float inv_sqrt_bc2;  // 1 / sqrt(1 - b2^t)
    float wd;
};

__device__ __forceinline__ float adam_one(float& p, float g, float& m, float& v, const AdamArgs& a)
{
    const float gg = a.wd != 0.0f ? fmaf(a.wd, p, g) : g;
    m = fmaf(a.b1, m, (1.0f - a.b1) * gg);
    v = fmaf(a.b2, v, (1.0f - a.b2) * gg * gg);
    const float denom = fmaf(sqrtf(v), a.inv_sqrt_bc2, a.eps);
    p = p - a.lr_t * m / denom;
    return p;
}

// vec: all five arrays 16-byte aligned, n4 = n / 4 float4 groups, the rest
// element by element.
__global__ void adam_kernel(int64_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, __nv_bfloat16* __restrict__ pb, AdamArgs a, bool vec)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t done = 0;
    if (vec) {
        const int64_t n4 = n / 4;
        for (int64_t i = t; i < n4; i += stride) {
            float4 pp = reinterpret_cast<float4*>(p)[i];
            const float4 gg = reinterpret_cast<const float4*>(g)[i];
            float4 mm = reinterpret_cast<float4*>(m)[i];
            float4 vv = reinterpret_cast<float4*>(v)[i];
            adam_one(pp.x, gg.x, mm.x, vv.x, a);
            adam_one(pp.y, gg.y, mm.y, vv.y, a);
            adam_one(pp.z, gg.z, mm.z, vv.z, a);
            adam_one(pp.w, gg.w, mm.w, vv.w, a);
            reinterpret_cast<float4*>(p)[i] = pp;
            reinterpret_cast<float4*>(m)[i] = mm;
            reinterpret_cast<float4*>(v)[i] = vv;
            if (pb) {
                __nv_bfloat162 lo = __floats2bfloat162_rn(pp.x, pp.y), hi = __floats2bfloat162_rn(pp.z, pp.w);
                uint2 w;
                w.x = *reinterpret_cast<uint32_t*>(&lo);
                w.y = *reinterpret_cast<uint32_t*>(&hi);
                reinterpret_cast<uint2*>(pb)[i] = w;
            }
        }
        done = n4 * 4;
    }
    for (int64_t i = done + t; i < n; i += stride) {
        float pp = p[i], mm = m[i], vv = v[i];
        adam_one(pp, g[i], mm, vv, a);
        p[i] = pp;
        m[i] = mm;
        v[i] = vv;
        if (pb) pb[i] = __float2bfloat16_rn(pp);
    }
}

// Several parameter tensors in one launch: tensor k owns the blocks
// [first_block[k], first_block[k + 1]) (in proportion to its size, at least
// one), which run adam_kernel's loop over it.
constexpr int kAdamMulti = 16;
struct AdamMulti {
    int count;
    int first_block[kAdamMulti + 1];
    int64_t n[kAdamMulti];
    float* p[kAdamMulti];
    const float* g[kAdamMulti];
    float* m[kAdamMulti];
    float* v[kAdamMulti];
    __nv_bfloat16* pb[kAdamMulti];
    AdamArgs a[kAdamMulti];
    bool vec[kAdamMulti];
};

__global__ void adam_multi_kernel(AdamMulti t)
{
    int k = 0;
    while (k + 1 < t.count && (int)blockIdx.x >= t.first_block[k + 1]) ++k;
    const int b = blockIdx.x - t.first_block[k], nb = t.first_block[k + 1] - t.first_block[k];
    const int64_t n = t.n[k];
    float* __restrict__ p = t.p[k];
    const float* __restrict__ g = t.g[k];
    float* __restrict__ m = t.m[k];
    float* __restrict__ v = t.v[k];
    __nv_bfloat16* __restrict__ pb = t.pb[k];
    const AdamArgs a = t.a[k];
    const int64_t stride = (int64_t)nb * blockDim.x;
    const int64_t i0 = (int64_t)b * blockDim.x + threadIdx.x;
    int64_t done = 0;
    if (t.vec[k]) {
        const int64_t n4 = n / 4;
        for (int64_t i = i0; i < n4; i += stride) {
            float4 pp = reinterpret_cast<float4*>(p)[i];
            const float4 gg = reinterpret_cast<const float4*>(g)[i];
            float4 mm = reinterpret_cast<float4*>(m)[i];
            float4 vv = reinterpret_cast<float4*>(v)[i];
            adam_one(pp.x, gg.x, mm.x, vv.x, a);
            adam_one(pp.y, gg.y, mm.y, vv.y, a);
            adam_one(pp.z, gg.z, mm.z, vv.z, a);
            adam_one(pp.w, gg.w, mm.w, vv.w, a);
            reinterpret_cast<float4*>(p)[i] = pp;
            reinterpret_cast<float4*>(m)[i] = mm;
            reinterpret_cast<float4*>(v)[i] = vv;
            if (pb) {
                __nv_bfloat162 lo = __floats2bfloat162_rn(pp.x, pp.y), hi = __floats2bfloat162_rn(pp.z, pp.w);
                uint2 w;
                w.x = *reinterpret_cast<uint32_t*>(&lo);
                w.y = *reinterpret_cast<uint32_t*>(&hi);
                reinterpret_cast<uint2*>(pb)[i] = w;
            }
        }
        done = n4 * 4;
    }
    for (int64_t i = done + i0; i < n; i += stride) {
        float pp = p[i], mm = m[i], vv = v[i];
        adam_one(pp, g[i], mm, vv, a);
        p[i] = pp;
        m[i] = mm;
        v[i] = vv;
        if (pb) pb[i] = __float2bfloat16_rn(pp);
    }
}

static int adam_args(const atdf_adam_tensor_t& t, AdamArgs& a, bool& vec)
{
    if (t.n < 0 || t.step < 1 || (t.n > 0 && (!t.param || !t.grad || !t.exp_avg || !t.exp_avg_sq)))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (!(t.beta1 >= 0.0f && t.beta1 < 1.0f && t.beta2 >= 0.0f && t.beta2 < 1.0f && t.eps >= 0.0f))
        return ATDF_ERR_INVALID_ARGUMENT;
    const double bc1 = 1.0 - std::pow((double)t.beta1, (double)t.step);
    const double bc2 = 1.0 - std::pow((double)t.beta2, (double)t.step);
    a.lr_t = (float)(t.lr / bc1);
    a.b1 = t.beta1;
    a.b2 = t.beta2;
    a.eps = t.eps;
    a.inv_sqrt_bc2 = (float)(1.0 / std::sqrt(bc2));
    a.wd = t.weight_decay;
    auto al16 = [](const void* q) { return ((uintptr_t)q & 15) == 0; };
    vec = al16(t.param) && al16(t.grad) && al16(t.exp_avg) && al16(t.exp_avg_sq) &&
          (!t.param_bf16 || ((uintptr_t)t.param_bf16 & 7) == 0);
    return ATDF_OK;
}

}  // namespace atdf

using namespace atdf;

extern "C" int atdf_adam_step_multi(int32_t count, const atdf_adam_tensor_t* tensors, atdf_stream_t stream)
{
    if (count < 0 || (count > 0 && !tensors)) return ATDF_ERR_INVALID_ARGUMENT;
    int dev = 0, sms = 0;
    ATDF_CUDA_TRY(cudaGetDevice(&dev));
    ATDF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t budget = (int64_t)sms * 8;  // blocks per launch, as for one large tensor
    for (int32_t c0 = 0; c0 < count; c0 += kAdamMulti) {
        AdamMulti t{};
        int64_t work[kAdamMulti], total = 0;
        for (int k = 0; k < kAdamMulti && c0 + k < count; ++k) {
            const atdf_adam_tensor_t& s = tensors[c0 + k];
            const int st = adam_args(s, t.a[t.count], t.vec[t.count]);
            if (st != ATDF_OK) return st;
            if (s.n == 0) continue;
            const int j = t.count++;
            t.n[j] = s.n;
            t.p[j] = s.param;
            t.g[j] = s.grad;
            t.m[j] = s.exp_avg;
            t.v[j] = s.exp_avg_sq;
            t.pb[j] = reinterpret_cast<__nv_bfloat16*>(s.param_bf16);
            work[j] = div_up(t.vec[j] ? div_up(s.n, 4) : s.n, 256);
            total += work[j];
        }
        if (t.count == 0) continue;
        int blocks = 0;
        for (int j = 0; j < t.count; ++j) {
            t.first_block[j] = blocks;
            const int64_t share = total > budget ? work[j] * budget / total : work[j];
            blocks += (int)std::max<int64_t>(1, std::min<int64_t>(share, work[j]));
        }
        t.first_block[t.count] = blocks;
        adam_multi_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(t);
        ATDF_LAUNCH_CHECK();
    }
    return ATDF_OK;
}

extern "C" int atdf_adam_step(int64_t n, float* param, const float* grad, float* exp_avg, float* exp_avg_sq,
                              void* param_bf16, float lr, float beta1, float beta2, float eps, float weight_decay,
                              int64_t step, atdf_stream_t stream)
{
    if (n < 0 || step < 1 || (n > 0 && (!param || !grad || !exp_avg || !exp_avg_sq))) return ATDF_ERR_INVALID_ARGUMENT;
    if (!(beta1 >= 0.0f && beta1 < 1.0f && beta2 >= 0.0f && beta2 < 1.0f && eps >= 0.0f))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (n == 0) return ATDF_OK;
    AdamArgs a;
    const double bc1 = 1.0 - std::pow((double)beta1, (double)step);
    const double bc2 = 1.0 - std::pow((double)beta2, (double)step);
    a.lr_t = (float)(lr / bc1);
    a.b1 = beta1;
    a.b2 = beta2;
    a.eps = eps;
    a.inv_sqrt_bc2 = (float)(1.0 / std::sqrt(bc2));
    a.wd = weight_decay;
    auto al16 = [](const void* q) { return ((uintptr_t)q & 15) == 0; };
    const bool vec = al16(param) && al16(grad) && al16(exp_avg) && al16(exp_avg_sq) &&
                     (!param_bf16 || ((uintptr_t)param_bf16 & 7) == 0);
    int dev = 0, sms = 0;
    ATDF_CUDA_TRY(cudaGetDevice(&dev));
    ATDF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t want = div_up(vec ? div_up(n, 4) : n, 256);
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * 8));
    adam_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(n, param, grad, exp_avg, exp_avg_sq,
                                                          reinterpret_cast<__nv_bfloat16*>(param_bf16), a, vec);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}
