// Photometric calibration of projected ray integrals (the reference's "tone
// mapper"): PhotometricCalibrationImpl::forward
// (hyperacorn/csrc/modules/ToneMapper.cpp:161-201) with the camera response
// of CameraResponseNetImpl::forward (:32-97), and the adjoint of both, one
// kernel each way instead of the reference's chain of index_select,
// grid_sample and elementwise tensor ops. Per element (channel c, ray r):
//
//   x  = I[c, r] + exposure_bias[img]    or   I[c, r] * exposure_factor[img]
//   x += bilinear(sensor_bias, uv[r])         border padding, align_corners = false
//   y  = bilinear(response, x / range)        border padding, align_corners = true
//        + (x - range) [x > range]            the leak, training mode only
//
// Both bilinear lookups follow torch's grid sampler (the reference calls
// torch::nn::functional::grid_sample, PyTorch 1.9.1): coordinates unnormalised
// from [-1, 1], clamped to [0, size - 1], corners outside the map skipped, and
// in the adjoint a zero coordinate gradient on and beyond the clamp bounds.
// Every FP32 operation of the forward and of the per-element adjoint is
// rounded on its own (no contraction), in the order the reference's ops apply
// them, so a plain FP32 restatement reproduces the outputs bit for bit; the
// parameter gradients are sums over rays (shared-memory atomics per block,
// then one global atomic per touched entry), equal to a sequential sum within
// FP32 rounding.

#include <algorithm>

#include "atdf_common.cuh"

namespace atdf {

struct ToneParams {
    int num_images, exposure_mode;
    const float* exposure;
    int sw, sh;
    const float* sensor;
    int P;
    const float* response;
    float range, inv_range;
    int leak;
};

// grid_sample's source coordinate, align_corners = false: ((g + 1) size - 1) / 2
__device__ __forceinline__ float unnorm_edges(float g, int size)
{
    return __fdiv_rn(__fsub_rn(__fmul_rn(__fadd_rn(g, 1.0f), (float)size), 1.0f), 2.0f);
}

// align_corners = true: ((g + 1) / 2) (size - 1)
__device__ __forceinline__ float unnorm_corners(float g, int size)
{
    return __fmul_rn(__fdiv_rn(__fadd_rn(g, 1.0f), 2.0f), (float)(size - 1));
}

__device__ __forceinline__ float clamp_border(float x, int size) { return fminf((float)(size - 1), fmaxf(x, 0.0f)); }

// The sensor-bias tap of ray r: corner indices (−1 = outside the map) and weights
struct SensorTap {
    int i[4];
    float w[4];
};

__device__ __forceinline__ SensorTap sensor_tap(const ToneParams& tp, float u, float v)
{
    const float gx = __fsub_rn(__fmul_rn(u, 2.0f), 1.0f);
    const float gy = __fsub_rn(__fmul_rn(v, 2.0f), 1.0f);
    const float ix = clamp_border(unnorm_edges(gx, tp.sw), tp.sw);
    const float iy = clamp_border(unnorm_edges(gy, tp.sh), tp.sh);
    const float x0 = floorf(ix), y0 = floorf(iy);
    const float x1 = x0 + 1.0f, y1 = y0 + 1.0f;
    const int ix0 = (int)x0, iy0 = (int)y0;
    const bool xin = ix0 + 1 < tp.sw, yin = iy0 + 1 < tp.sh;
    SensorTap t;
    // nw, ne, sw, se: torch's corner order
    t.w[0] = __fmul_rn(__fsub_rn(x1, ix), __fsub_rn(y1, iy));
    t.w[1] = __fmul_rn(__fsub_rn(ix, x0), __fsub_rn(y1, iy));
    t.w[2] = __fmul_rn(__fsub_rn(x1, ix), __fsub_rn(iy, y0));
    t.w[3] = __fmul_rn(__fsub_rn(ix, x0), __fsub_rn(iy, y0));
    t.i[0] = iy0 * tp.sw + ix0;
    t.i[1] = xin ? iy0 * tp.sw + ix0 + 1 : -1;
    t.i[2] = yin ? (iy0 + 1) * tp.sw + ix0 : -1;
    t.i[3] = xin && yin ? (iy0 + 1) * tp.sw + ix0 + 1 : -1;
    return t;
}

// The response lookup of value x: the left tap, its weights, and the clamp
// gradient of the coordinate (0 on and beyond the bounds).
struct ResponseTap {
    int i0;
    bool right;  // the right tap lies inside the curve
    float wl, wr, grad_clip;
};

__device__ __forceinline__ ResponseTap response_tap(const ToneParams& tp, float x)
{
    const float t = __fsub_rn(__fmul_rn(__fmul_rn(x, tp.inv_range), 2.0f), 1.0f);
    const float raw = unnorm_corners(t, tp.P);
    const float ix = clamp_border(raw, tp.P);
    const float x0 = floorf(ix);
    ResponseTap rt;
    rt.i0 = (int)x0;
    rt.right = rt.i0 + 1 < tp.P;
    // the curve is one row high: the vertical weight (iy_se - iy) is exactly 1
    rt.wl = __fsub_rn(x0 + 1.0f, ix);
    rt.wr = __fsub_rn(ix, x0);
    rt.grad_clip = (raw <= 0.0f || raw >= (float)(tp.P - 1)) ? 0.0f : 1.0f;
    return rt;
}

// x after exposure and sensor bias; false for an image id outside the table
__device__ __forceinline__ bool pre_response(const ToneParams& tp, float I, int img, const SensorTap* st, float& x)
{
    if (tp.exposure_mode != ATDF_EXPOSURE_NONE) {
        if (img < 0 || img >= tp.num_images) return false;
        const float e = __ldg(tp.exposure + img);
        x = tp.exposure_mode == ATDF_EXPOSURE_FACTOR ? __fmul_rn(I, e) : __fadd_rn(I, e);
    } else {
        x = I;
    }
    if (st) {
        float val = 0.0f;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (st->i[k] >= 0) val = __fadd_rn(val, __fmul_rn(__ldg(tp.sensor + st->i[k]), st->w[k]));
        x = __fadd_rn(x, val);
    }
    return true;
}

__global__ void tone_forward_kernel(ToneParams tp, int64_t C, int64_t R, const float* __restrict__ integral,
                                    const float* __restrict__ uv, const int32_t* __restrict__ image_id,
                                    float* __restrict__ out, int32_t* err)
{
    const int64_t n = C * R;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e % R;
        SensorTap st;
        if (tp.sw > 0) st = sensor_tap(tp, uv[2 * r], uv[2 * r + 1]);
        float x;
        if (!pre_response(tp, integral[e], image_id ? image_id[r] : 0, tp.sw > 0 ? &st : nullptr, x)) {
            set_err(err, ATDF_DEVERR_INDEX);
            out[e] = __int_as_float(0x7fffffff);
            continue;
        }
        if (tp.P > 0) {
            const ResponseTap rt = response_tap(tp, x);
            float y = __fmul_rn(__ldg(tp.response + rt.i0), rt.wl);
            if (rt.right) y = __fadd_rn(y, __fmul_rn(__ldg(tp.response + rt.i0 + 1), rt.wr));
            if (tp.leak && x > tp.range) y = __fadd_rn(y, __fsub_rn(x, tp.range));
            x = y;
        }
        out[e] = x;
    }
}

// Gradients of the calibration: grad_integral is written; the parameter
// gradients (any may be null) are added to. SMEM: per-block accumulators for
// the exposure table, the sensor map and the curve in shared memory.
template <bool SMEM>
__global__ void tone_backward_kernel(ToneParams tp, int64_t C, int64_t R, const float* __restrict__ integral,
                                     const float* __restrict__ uv, const int32_t* __restrict__ image_id,
                                     const float* __restrict__ grad_out, float* __restrict__ grad_integral,
                                     float* grad_exposure, float* grad_sensor, float* grad_response, int32_t* err)
{
    extern __shared__ float acc[];
    const int ne = grad_exposure ? tp.num_images : 0;
    const int ns = grad_sensor ? tp.sw * tp.sh : 0;
    const int np = grad_response ? tp.P : 0;
    float* ge = SMEM ? acc : grad_exposure;
    float* gs = SMEM ? acc + ne : grad_sensor;
    float* gr = SMEM ? acc + ne + ns : grad_response;
    if (SMEM) {
        for (int i = threadIdx.x; i < ne + ns + np; i += blockDim.x) acc[i] = 0.0f;
        __syncthreads();
    }
    const int64_t n = C * R;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e % R;
        const int img = image_id ? image_id[r] : 0;
        SensorTap st;
        if (tp.sw > 0) st = sensor_tap(tp, uv[2 * r], uv[2 * r + 1]);
        const float I = integral[e];
        float x;
        if (!pre_response(tp, I, img, tp.sw > 0 ? &st : nullptr, x)) {
            set_err(err, ATDF_DEVERR_INDEX);
            if (grad_integral) grad_integral[e] = 0.0f;
            continue;
        }
        const float g = grad_out[e];
        float dx = g;
        if (tp.P > 0) {
            const ResponseTap rt = response_tap(tp, x);
            const float vl = __ldg(tp.response + rt.i0);
            if (np) atomicAdd(gr + rt.i0, __fmul_rn(rt.wl, g));
            float gix = __fsub_rn(0.0f, __fmul_rn(vl, g));
            if (rt.right) {
                if (np) atomicAdd(gr + rt.i0 + 1, __fmul_rn(rt.wr, g));
                gix = __fadd_rn(gix, __fmul_rn(__ldg(tp.response + rt.i0 + 1), g));
            }
            const float mult = __fmul_rn(__fdiv_rn((float)(tp.P - 1), 2.0f), rt.grad_clip);
            const float dgrid = __fmul_rn(mult, gix);
            dx = __fmul_rn(__fmul_rn(dgrid, 2.0f), tp.inv_range);
            if (tp.leak && x > tp.range) dx = __fadd_rn(dx, g);
        }
        if (tp.sw > 0 && ns) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (st.i[k] >= 0) atomicAdd(gs + st.i[k], __fmul_rn(st.w[k], dx));
        }
        float dI = dx;
        if (tp.exposure_mode == ATDF_EXPOSURE_FACTOR) {
            if (ne) atomicAdd(ge + img, __fmul_rn(dx, I));
            dI = __fmul_rn(dx, __ldg(tp.exposure + img));
        } else if (tp.exposure_mode == ATDF_EXPOSURE_BIAS) {
            if (ne) atomicAdd(ge + img, dx);
        }
        if (grad_integral) grad_integral[e] = dI;
    }
    if (SMEM) {
        __syncthreads();
        for (int i = threadIdx.x; i < ne + ns + np; i += blockDim.x) {
            const float v = acc[i];
            if (v == 0.0f) continue;
            if (i < ne)
                atomicAdd(grad_exposure + i, v);
            else if (i < ne + ns)
                atomicAdd(grad_sensor + (i - ne), v);
            else
                atomicAdd(grad_response + (i - ne - ns), v);
        }
    }
}

// CameraResponseNetImpl::ParamLoss (ToneMapper.cpp:98-111): f = P sqrt(1e-5);
// target t_0 = 0, t_{P-1} = range, t_i = (r_{i+1} + r_{i-1}) / 2; loss =
// sum_i (f r_i - f t_i)^2 with the gradient through both r and t. One block.
__global__ void tone_response_loss_kernel(int P, const float* __restrict__ r, float range, float f, float* loss,
                                          float* grad, const float* grad_scale)
{
    __shared__ double part[32];
    const float scale = grad_scale ? *grad_scale : 1.0f;
    auto target = [&](int i) -> float {
        if (i == 0) return 0.0f;
        if (i == P - 1) return range;
        return __fmul_rn(__fadd_rn(r[i + 1], r[i - 1]), 0.5f);
    };
    // d loss / d (f r_i), times the caller's scale
    auto da = [&](int i) -> float {
        const float d = __fsub_rn(__fmul_rn(r[i], f), __fmul_rn(target(i), f));
        return __fmul_rn(__fmul_rn(2.0f, d), scale);
    };
    double s = 0.0;
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const float d = __fsub_rn(__fmul_rn(r[i], f), __fmul_rn(target(i), f));
        s += (double)d * (double)d;
        if (grad) {
            float gi = __fmul_rn(da(i), f);
            // r_i feeds the targets of its neighbours i - 1 and i + 1 (interior entries only)
            float gt = 0.0f;
            if (i - 1 >= 1 && i - 1 <= P - 2) gt = __fadd_rn(gt, __fmul_rn(__fmul_rn(-da(i - 1), f), 0.5f));
            if (i + 1 >= 1 && i + 1 <= P - 2) gt = __fadd_rn(gt, __fmul_rn(__fmul_rn(-da(i + 1), f), 0.5f));
            grad[i] += __fadd_rn(gi, gt);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
        if (loss) *loss = (float)t;
    }
}

static int tone_params(const atdf_tone_mapper_t* tm, int64_t channels, ToneParams& tp)
{
    if (!tm || tm->num_images < 0 || tm->sensor_w < 0 || tm->sensor_h < 0 || tm->response_params < 0)
        return ATDF_ERR_INVALID_ARGUMENT;
    if (tm->exposure_mode != ATDF_EXPOSURE_NONE && tm->exposure_mode != ATDF_EXPOSURE_BIAS &&
        tm->exposure_mode != ATDF_EXPOSURE_FACTOR)
        return ATDF_ERR_INVALID_ARGUMENT;
    if (tm->exposure_mode != ATDF_EXPOSURE_NONE && (!tm->exposure || tm->num_images < 1))
        return ATDF_ERR_INVALID_ARGUMENT;
    if ((tm->sensor_w > 0) != (tm->sensor_h > 0) || (tm->sensor_w > 0 && !tm->sensor_bias))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (tm->response_params == 1 || (tm->response_params > 1 && (!tm->response || !(tm->response_range > 0.0f))))
        return ATDF_ERR_INVALID_ARGUMENT;
    // the curve has one channel (CameraResponseNet(25, 1, ...), ToneMapper.cpp:40-43 asserts the match)
    if (tm->response_params > 1 && channels != 1) return ATDF_ERR_UNSUPPORTED;
    tp.num_images = tm->num_images;
    tp.exposure_mode = tm->exposure_mode;
    tp.exposure = tm->exposure;
    tp.sw = tm->sensor_w;
    tp.sh = tm->sensor_h;
    tp.sensor = tm->sensor_bias;
    tp.P = tm->response_params;
    tp.response = tm->response;
    tp.range = tm->response_range;
    tp.inv_range = tp.P > 0 ? 1.0f / tm->response_range : 0.0f;
    tp.leak = tm->leak != 0;
    return ATDF_OK;
}

static unsigned tone_blocks(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>(div_up(n, 256), 148 * 8)); }

}  // namespace atdf

using namespace atdf;

extern "C" {

int atdf_tone_map_forward(const atdf_tone_mapper_t* tm, int64_t channels, int64_t num_rays, const float* integral,
                          const float* uv, const int32_t* image_id, float* out, int32_t* dev_error,
                          atdf_stream_t stream)
{
    ToneParams tp;
    if (channels < 1 || num_rays < 0) return ATDF_ERR_INVALID_ARGUMENT;
    const int st = tone_params(tm, channels, tp);
    if (st != ATDF_OK) return st;
    if (num_rays == 0) return ATDF_OK;
    if (!integral || !out || !dev_error || (tp.sw > 0 && !uv) || (tp.exposure_mode != ATDF_EXPOSURE_NONE && !image_id))
        return ATDF_ERR_INVALID_ARGUMENT;
    const int64_t n = channels * num_rays;
    tone_forward_kernel<<<tone_blocks(n), 256, 0, (cudaStream_t)stream>>>(tp, channels, num_rays, integral, uv,
                                                                         image_id, out, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_tone_map_backward(const atdf_tone_mapper_t* tm, int64_t channels, int64_t num_rays, const float* integral,
                           const float* uv, const int32_t* image_id, const float* grad_out, float* grad_integral,
                           float* grad_exposure, float* grad_sensor_bias, float* grad_response, int32_t* dev_error,
                           atdf_stream_t stream)
{
    ToneParams tp;
    if (channels < 1 || num_rays < 0) return ATDF_ERR_INVALID_ARGUMENT;
    const int st = tone_params(tm, channels, tp);
    if (st != ATDF_OK) return st;
    if (num_rays == 0) return ATDF_OK;
    if (!integral || !grad_out || !dev_error || (tp.sw > 0 && !uv) ||
        (tp.exposure_mode != ATDF_EXPOSURE_NONE && !image_id))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (tp.exposure_mode == ATDF_EXPOSURE_NONE) grad_exposure = nullptr;
    if (tp.sw == 0) grad_sensor_bias = nullptr;
    if (tp.P == 0) grad_response = nullptr;
    const int64_t n = channels * num_rays;
    const int64_t floats = (grad_exposure ? (int64_t)tp.num_images : 0) +
                           (grad_sensor_bias ? (int64_t)tp.sw * tp.sh : 0) + (grad_response ? (int64_t)tp.P : 0);
    const unsigned blocks = tone_blocks(n);
    cudaStream_t s = (cudaStream_t)stream;
    if (floats * 4 <= 48 * 1024) {
        tone_backward_kernel<true><<<blocks, 256, (size_t)floats * 4, s>>>(
            tp, channels, num_rays, integral, uv, image_id, grad_out, grad_integral, grad_exposure, grad_sensor_bias,
            grad_response, dev_error);
    } else {
        tone_backward_kernel<false><<<blocks, 256, 0, s>>>(tp, channels, num_rays, integral, uv, image_id, grad_out,
                                                           grad_integral, grad_exposure, grad_sensor_bias,
                                                           grad_response, dev_error);
    }
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_tone_response_loss(int32_t response_params, const float* response, float response_range, float* loss,
                            float* grad_response, const float* grad_scale, atdf_stream_t stream)
{
    if (response_params < 2 || !response || (!loss && !grad_response)) return ATDF_ERR_INVALID_ARGUMENT;
    const float f = (float)((double)response_params * sqrt(1e-5));
    tone_response_loss_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(response_params, response, response_range, f,
                                                                   loss, grad_response, grad_scale);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

}  // extern "C"
