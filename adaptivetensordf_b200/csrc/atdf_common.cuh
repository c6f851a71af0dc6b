// Device helpers shared by the sm_100a kernels of libatdf_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "atdf.h"

#define ATDF_CUDA_TRY(expr)                             \
    do {                                                \
        cudaError_t _e = (expr);                        \
        if (_e != cudaSuccess) return ATDF_ERR_CUDA;    \
    } while (0)

#define ATDF_LAUNCH_CHECK()                             \
    do {                                                \
        if (cudaGetLastError() != cudaSuccess) return ATDF_ERR_CUDA; \
    } while (0)

namespace atdf {

__device__ __forceinline__ void set_err(int32_t* e, int32_t bit)
{
    if (e) atomicOr(e, bit);
}

__host__ __device__ __forceinline__ int64_t div_up(int64_t a, int64_t b) { return (a + b - 1) / b; }

// ---------------------------------------------------------------------------
// Exact restatements with one rounding per source operation (no contraction):
// the integer outputs of the sampler (hit lists, sample counts) and the
// sample t / weight / position values depend on them bit for bit.
// ---------------------------------------------------------------------------

// IntersectBoxRayPrecise (hyperacorn/csrc/structure/HyperTree.h:338-380).
__device__ __forceinline__ bool intersect_box(const float* bmin, const float* bmax, const float o[3], const float d[3],
                                              float& tmin, float& tmax)
{
    double t_near = -236436436.0;
    double t_far = 43637575.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float mn = bmin[i], mx = bmax[i];
        if (d[i] == 0.0f) {
            if ((o[i] < mn) || (o[i] >= mx)) return false;
        } else {
            float T1 = __fdiv_rn(__fsub_rn(mn, o[i]), d[i]);
            float T2 = __fdiv_rn(__fsub_rn(mx, o[i]), d[i]);
            if (T1 > T2) {
                float tmp = T1;
                T1 = T2;
                T2 = tmp;
            }
            if ((double)T1 > t_near) t_near = T1;
            if ((double)T2 < t_far) t_far = T2;
            if ((t_near > t_far) || (t_far < 0)) return false;
        }
    }
    tmin = (float)t_near;
    tmax = (float)t_far;
    return true;
}

// Sample count of one leaf hit (HyperTree.cu:344-355), iCeil = ceiling.
__device__ __forceinline__ int seg_num_samples(const float* bmin, const float* bmax, float tmin, float tmax, int M)
{
    float dx = __fsub_rn(bmax[0], bmin[0]);
    float dy = __fsub_rn(bmax[1], bmin[1]);
    float dz = __fsub_rn(bmax[2], bmin[2]);
    float sq = __fmul_rn(dx, dx);
    sq = __fadd_rn(sq, __fmul_rn(dy, dy));
    sq = __fadd_rn(sq, __fmul_rn(dz, dz));
    float diag = __fsqrt_rn(sq);
    float dis = __fsub_rn(tmax, tmin);
    float rel = __fdiv_rn(dis, diag);
    float prod = __fmul_rn(rel, (float)M);
    return (int)ceilf(prod);
}

// t of sample j of a segment (HyperTree.cu:448-461).
__device__ __forceinline__ float sample_t(float tmin, float tmax, int n, int j, float a)
{
    float dis = __fsub_rn(tmax, tmin);
    float step = __fdiv_rn(dis, (float)n);
    float t1 = __fadd_rn(tmin, __fmul_rn((float)j, step));
    float t2 = __fadd_rn(tmin, __fmul_rn((float)(j + 1), step));
    float oma = __fsub_rn(1.0f, a);
    return __fadd_rn(__fmul_rn(t1, oma), __fmul_rn(t2, a));
}

// Jitter hash: uniform [0, 1) keyed by (seed, ray, node, j), from the
// SplitMix64 finaliser (Steele, Lea, Flood 2014). Same bits as the oracle.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
// The jitter hash in two stages: the ray's key, then the sample's value.
__device__ __forceinline__ uint64_t jitter_key(uint64_t seed, int32_t ray)
{
    return mix64(seed + 0x9e3779b97f4a7c15ULL * (uint64_t)(uint32_t)ray);
}
__device__ __forceinline__ float jitter_keyed(uint64_t key, int32_t node, int32_t j)
{
    const uint64_t k = mix64(key ^ (((uint64_t)(uint32_t)node << 32) | (uint64_t)(uint32_t)j));
    return (float)(k >> 40) * (1.0f / 16777216.0f);
}
__device__ __forceinline__ float jitter(uint64_t seed, int32_t ray, int32_t node, int32_t j)
{
    return jitter_keyed(jitter_key(seed, ray), node, j);
}

// Interval value a of sample j: explicit array, hash, or the midpoint.
__device__ __forceinline__ float sample_a(const float* rnd, int64_t idx, uint64_t seed, int32_t ray, int32_t node,
                                          int32_t j)
{
    if (rnd) return rnd[idx];
    if (seed) return jitter(seed, ray, node, j);
    return 0.5f;
}

// Weight of sample j from its neighbours' t (HyperTree.cu:495-512).
__device__ __forceinline__ float sample_w(float tmin, float tmax, int n, int j, float t_prev, float t, float t_next)
{
    float lo = (j == 0) ? tmin : __fmul_rn(__fadd_rn(t_prev, t), 0.5f);
    float hi = (j == n - 1) ? tmax : __fmul_rn(__fadd_rn(t_next, t), 0.5f);
    return __fsub_rn(hi, lo);
}

// Leaf-local coordinate (HyperTree.cu:253).
__device__ __forceinline__ float local_coord(float x, float mn, float mx)
{
    float size = __fsub_rn(mx, mn);
    float b = __fdiv_rn(__fsub_rn(x, mn), size);
    return __fsub_rn(__fmul_rn(b, 2.0f), 1.0f);
}

// Same value as local_coord when inv_size is nonzero: it is only set when the
// size is a power of two, and then (x - mn) / size and (x - mn) * (1 / size)
// are the same exact scaling.
__device__ __forceinline__ float local_coord_fast(float x, float mn, float size, float inv_size)
{
    float a = __fsub_rn(x, mn);
    float b = inv_size != 0.0f ? __fmul_rn(a, inv_size) : __fdiv_rn(a, size);
    return __fsub_rn(__fmul_rn(b, 2.0f), 1.0f);
}

// 1 / x when x is a power of two (exactly representable reciprocal), else 0.
__host__ __device__ __forceinline__ float pow2_reciprocal(float x)
{
    int e = 0;
    const float m = frexpf(x, &e);
    return (x > 0.0f && m == 0.5f) ? ldexpf(1.0f, 1 - e) : 0.0f;
}

// ROI-normalised x line coordinate (geometry_tensor_qo.cpp:293).
__device__ __forceinline__ float roi_coord(float x, float rmin, float rmax)
{
    float a = __fsub_rn(x, rmin);
    float b = __fmul_rn(2.0f, a);
    float range = __fsub_rn(rmax, rmin);
    return __fsub_rn(__fdiv_rn(b, range), 1.0f);
}

// Bilinear corners of IndirectGridSample2D (IndirectGridSample2D.cu:36-92):
// align_corners=True, weights from the unclamped corners, clamped indices.
struct Corner2 {
    int x0, x1, y0, y1;
    float w_nw, w_ne, w_sw, w_se;
    float ix, iy;
    float fx0, fx1, fy0, fy1;
};
__device__ __forceinline__ Corner2 corners2(float u, float v, int H, int W)
{
    Corner2 c;
    // (u + 1) / 2 as a multiplication by 0.5: both round the same exact value
    float ix = __fmul_rn(__fmul_rn(__fadd_rn(u, 1.0f), 0.5f), (float)(W - 1));
    float iy = __fmul_rn(__fmul_rn(__fadd_rn(v, 1.0f), 0.5f), (float)(H - 1));
    int x0 = (int)floorf(ix), y0 = (int)floorf(iy);
    int x1 = x0 + 1, y1 = y0 + 1;
    c.fx0 = (float)x0;
    c.fx1 = (float)x1;
    c.fy0 = (float)y0;
    c.fy1 = (float)y1;
    c.w_nw = __fmul_rn(__fsub_rn(c.fx1, ix), __fsub_rn(c.fy1, iy));
    c.w_ne = __fmul_rn(__fsub_rn(ix, c.fx0), __fsub_rn(c.fy1, iy));
    c.w_sw = __fmul_rn(__fsub_rn(c.fx1, ix), __fsub_rn(iy, c.fy0));
    c.w_se = __fmul_rn(__fsub_rn(ix, c.fx0), __fsub_rn(iy, c.fy0));
    c.ix = ix;
    c.iy = iy;
    c.x0 = min(W - 1, max(x0, 0));
    c.x1 = min(W - 1, max(x1, 0));
    c.y0 = min(H - 1, max(y0, 0));
    c.y1 = min(H - 1, max(y1, 0));
    return c;
}

// Linear corners of IndirectGridSample1D (IndirectGridSample1D.cu:29-45).
struct Corner1 {
    int x0, x1;
    float w0, w1, ix, fx0, fx1;
};
__device__ __forceinline__ Corner1 corners1(float u, int W)
{
    Corner1 c;
    float ix = __fmul_rn(__fmul_rn(__fadd_rn(u, 1.0f), 0.5f), (float)(W - 1));
    int x0 = (int)floorf(ix);
    c.fx0 = (float)x0;
    c.fx1 = (float)(x0 + 1);
    c.w0 = __fsub_rn(c.fx1, ix);
    c.w1 = __fsub_rn(ix, c.fx0);
    c.ix = ix;
    c.x0 = min(W - 1, max(x0, 0));
    c.x1 = min(W - 1, max(x0 + 1, 0));
    return c;
}

// Bilinear value with the reference's accumulation order (nw, ne, sw, se).
__device__ __forceinline__ float bilerp(const Corner2& c, float vnw, float vne, float vsw, float vse)
{
    float acc = __fmul_rn(vnw, c.w_nw);
    acc = __fadd_rn(acc, __fmul_rn(vne, c.w_ne));
    acc = __fadd_rn(acc, __fmul_rn(vsw, c.w_sw));
    acc = __fadd_rn(acc, __fmul_rn(vse, c.w_se));
    return acc;
}
__device__ __forceinline__ float lerp1(const Corner1& c, float v0, float v1)
{
    return __fadd_rn(__fmul_rn(v0, c.w0), __fmul_rn(v1, c.w1));
}

struct SampleGeo {
    float pu[3], pv[3], lu[3];
};

// geometry_tensor_qo.cpp:280-298: plane coordinates from the leaf-local
// position; x line at the ROI-normalised x, y line at the local y, z line at
// the raw global z.
__device__ __forceinline__ SampleGeo sample_geo(const float p[3], const float* bmin, const float* bmax,
                                                const float* roi_min, const float* roi_max)
{
    float loc[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) loc[k] = local_coord(p[k], bmin[k], bmax[k]);
    SampleGeo g;
    g.pu[0] = loc[1];
    g.pv[0] = loc[2];
    g.pu[1] = loc[0];
    g.pv[1] = loc[2];
    g.pu[2] = loc[0];
    g.pv[2] = loc[1];
    g.lu[0] = roi_coord(p[0], roi_min[0], roi_max[0]);
    g.lu[1] = loc[1];
    g.lu[2] = p[2];
    return g;
}

// ---------------------------------------------------------------------------
// Activations (FCBlock hidden activation, DecodeFeatures last activation).
// ---------------------------------------------------------------------------
// Logistic function with the fast exponential and divide intrinsics (a few
// ulp; the decoder tolerance is 1e-5 relative).
__device__ __forceinline__ float sigmoidf_(float x) { return __fdividef(1.0f, 1.0f + __expf(-x)); }

__device__ __forceinline__ float act_fwd(int a, float x, float beta)
{
    switch (a) {
        case ATDF_ACT_RELU: return x > 0.0f ? x : 0.0f;
        case ATDF_ACT_SILU: return x * sigmoidf_(x);
        case ATDF_ACT_SIGMOID: return sigmoidf_(x);
        case ATDF_ACT_SOFTPLUS: return (x * beta > 20.0f) ? x : log1pf(expf(x * beta)) / beta;
        case ATDF_ACT_LEAKYRELU: return x > 0.0f ? x : x * 0.01f;
        case ATDF_ACT_ABS: return fabsf(x);
        case ATDF_ACT_TANH: return tanhf(x);
        default: return x;
    }
}

__device__ __forceinline__ float act_grad(int a, float x, float beta)
{
    switch (a) {
        case ATDF_ACT_RELU: return x > 0.0f ? 1.0f : 0.0f;
        case ATDF_ACT_SILU: {
            float s = sigmoidf_(x);
            return s * (1.0f + x * (1.0f - s));
        }
        case ATDF_ACT_SIGMOID: {
            float s = sigmoidf_(x);
            return s * (1.0f - s);
        }
        case ATDF_ACT_SOFTPLUS: {
            if (x * beta > 20.0f) return 1.0f;
            float z = expf(x * beta);
            return z / (z + 1.0f);
        }
        case ATDF_ACT_LEAKYRELU: return x > 0.0f ? 1.0f : 0.01f;
        case ATDF_ACT_ABS: return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f);
        case ATDF_ACT_TANH: {
            float t = tanhf(x);
            return 1.0f - t * t;
        }
        default: return 1.0f;
    }
}

// Order-preserving key of a float (+0 and -0 map to the same key).
__device__ __forceinline__ uint32_t float_key(float f)
{
    uint32_t u = __float_as_uint(f + 0.0f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Single-block exclusive scan of n int64 values in place; writes the total to
// *total (if non-null). Launched with 1024 threads.
__global__ void scan_exclusive_i64_kernel(int64_t* data, int64_t n, int64_t* total);
__global__ void scan_exclusive_i32_kernel(int32_t* data, int64_t n, int32_t* total);

}  // namespace atdf
