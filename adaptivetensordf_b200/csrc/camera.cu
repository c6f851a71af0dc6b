// Rays of detector pixels from the tilt series' camera poses: the reference's
// SceneBase::GetRays (hyperacorn/csrc/data/SceneBase.cpp:369-450) for its two
// camera models, fused into one kernel (the reference composes UVToPixel,
// CameraModelModule::Unproject, a quaternion rotation kernel and tensor
// arithmetic, CameraPose.h:14-30, CameraPose.cu:469-479).
//
//   px      = uv * (w - 1)            (align_corners)   | uv * w - 0.5   (FP32, as UVToPixel)
//   c       = (px - (cx, cy)) / (fx, fy)                                 (FP64 from here on)
//   orthographic: dir = R (0, 0, 1);  origin = R (c.x, c.y, 0) + t_vol - sqrt(2) dir
//   pinhole:      dir = R normalize(c.x, c.y, 1);  origin = translation[image]
//
// R is the image's unit quaternion (x, y, z, w); q p = p + w s + u x s with
// u = (x, y, z), s = 2 (u x p). Every FP64 operation is rounded on its own
// (no contraction), so a plain double restatement reproduces the results.
// Outputs are rounded to FP32 at the end, as the reference does.

#include <algorithm>

#include "atdf_common.cuh"

namespace atdf {

struct D3 {
    double x, y, z;
};

__device__ __forceinline__ D3 cross(const D3& a, const D3& b)
{
    return {__dsub_rn(__dmul_rn(a.y, b.z), __dmul_rn(a.z, b.y)), __dsub_rn(__dmul_rn(a.z, b.x), __dmul_rn(a.x, b.z)),
            __dsub_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x))};
}

__device__ __forceinline__ D3 rotate(const double* q, const D3& p)
{
    const D3 u{q[0], q[1], q[2]};
    D3 s = cross(u, p);
    s = {__dadd_rn(s.x, s.x), __dadd_rn(s.y, s.y), __dadd_rn(s.z, s.z)};
    const D3 us = cross(u, s);
    const double w = q[3];
    return {__dadd_rn(__dadd_rn(p.x, __dmul_rn(w, s.x)), us.x), __dadd_rn(__dadd_rn(p.y, __dmul_rn(w, s.y)), us.y),
            __dadd_rn(__dadd_rn(p.z, __dmul_rn(w, s.z)), us.z)};
}

__global__ void camera_rays_kernel(int64_t n, const float* __restrict__ uv, const int32_t* __restrict__ image_id,
                                   const int32_t* __restrict__ camera_id, const double* __restrict__ rotation,
                                   const double* __restrict__ translation, int64_t num_images,
                                   const double* __restrict__ intrinsics, int64_t num_cameras, int w, int h,
                                   int align_corners, int model, float tvx, float tvy, float tvz,
                                   float* __restrict__ origin, float* __restrict__ direction, int32_t* err)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int img = image_id[i];
        const int cam = camera_id ? camera_id[i] : 0;
        if (img < 0 || img >= num_images || cam < 0 || cam >= num_cameras) {
            set_err(err, ATDF_DEVERR_INDEX);
            continue;
        }
        const float u = uv[2 * i], v = uv[2 * i + 1];
        const float px = align_corners ? __fmul_rn(u, (float)(w - 1)) : __fsub_rn(__fmul_rn(u, (float)w), 0.5f);
        const float py = align_corners ? __fmul_rn(v, (float)(h - 1)) : __fsub_rn(__fmul_rn(v, (float)h), 0.5f);
        const double* K = intrinsics + 5 * (int64_t)cam;  // fx fy cx cy s
        const double cx = __ddiv_rn(__dsub_rn((double)px, K[2]), K[0]);
        const double cy = __ddiv_rn(__dsub_rn((double)py, K[3]), K[1]);
        const double* q = rotation + 4 * (int64_t)img;
        D3 o, d;
        if (model == ATDF_CAMERA_ORTHOGRAPHIC) {
            d = rotate(q, D3{0.0, 0.0, 1.0});
            const D3 p = rotate(q, D3{cx, cy, 0.0});
            const double r2 = 1.4142135623730951;  // sqrt(2) rounded to double
            o = {__dsub_rn(__dadd_rn(p.x, (double)tvx), __dmul_rn(d.x, r2)),
                 __dsub_rn(__dadd_rn(p.y, (double)tvy), __dmul_rn(d.y, r2)),
                 __dsub_rn(__dadd_rn(p.z, (double)tvz), __dmul_rn(d.z, r2))};
        } else {
            const double nrm = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(cx, cx), __dmul_rn(cy, cy)), 1.0));
            d = rotate(q, D3{__ddiv_rn(cx, nrm), __ddiv_rn(cy, nrm), __ddiv_rn(1.0, nrm)});
            const double* t = translation + 3 * (int64_t)img;
            o = {t[0], t[1], t[2]};
        }
        origin[3 * i] = __double2float_rn(o.x);
        origin[3 * i + 1] = __double2float_rn(o.y);
        origin[3 * i + 2] = __double2float_rn(o.z);
        direction[3 * i] = __double2float_rn(d.x);
        direction[3 * i + 1] = __double2float_rn(d.y);
        direction[3 * i + 2] = __double2float_rn(d.z);
    }
}

// SceneBase::PointInAnyImage (hyperacorn/csrc/data/SceneBase.cu:13-97): a
// point is marked when it lies in the ROI box (closed bounds on its FP32
// value, BoxContainsPoint, HyperTree.h:382-392) and its projection rounds to a
// pixel inside the w x h image of at least one pose. The view position is
// R^T (p - t) in FP64 (the pose's unit quaternion R conjugated, t its
// translation or zero), the pixel is (fx v.x + cx, fy v.y + cy) for the
// orthographic camera and (fx v.x / v.z + cx, fy v.y / v.z + cy) for the
// pinhole one (the skew set to zero as the reference does), rounded half away
// from zero. One thread per point, images in order until one contains it.
__global__ void point_in_any_image_kernel(int64_t n, const float* __restrict__ pts,
                                          const double* __restrict__ rotation, const double* __restrict__ translation,
                                          int64_t num_images, const double* __restrict__ K, int model, int w, int h,
                                          float3 rmin, float3 rmax, float* __restrict__ mask)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float x = pts[3 * i], y = pts[3 * i + 1], z = pts[3 * i + 2];
        float m = 0.0f;
        if (!(rmin.x > x || rmax.x < x || rmin.y > y || rmax.y < y || rmin.z > z || rmax.z < z)) {
            for (int64_t a = 0; a < num_images && m == 0.0f; ++a) {
                const double* q = rotation + 4 * a;
                const double qi[4] = {-q[0], -q[1], -q[2], q[3]};
                D3 pt{(double)x, (double)y, (double)z};
                if (translation) {
                    const double* t = translation + 3 * a;
                    pt = {__dsub_rn(pt.x, t[0]), __dsub_rn(pt.y, t[1]), __dsub_rn(pt.z, t[2])};
                }
                const D3 v = rotate(qi, pt);
                double px, py;
                if (model == ATDF_CAMERA_ORTHOGRAPHIC) {
                    px = __dadd_rn(__dmul_rn(K[0], v.x), K[2]);
                    py = __dadd_rn(__dmul_rn(K[1], v.y), K[3]);
                } else {
                    px = __dadd_rn(__dmul_rn(K[0], __ddiv_rn(v.x, v.z)), K[2]);
                    py = __dadd_rn(__dmul_rn(K[1], __ddiv_rn(v.y, v.z)), K[3]);
                }
                const double rx = round(px), ry = round(py);
                if (rx >= 0.0 && rx < (double)w && ry >= 0.0 && ry < (double)h) m = 1.0f;
            }
        }
        mask[i] = m;
    }
}

}  // namespace atdf

using namespace atdf;

extern "C" int atdf_point_in_any_image(int64_t n, const float* points, const double* rotation,
                                       const double* translation, int64_t num_images, const double* intrinsics,
                                       int32_t width, int32_t height, int32_t model, const float* roi_min,
                                       const float* roi_max, float* mask, atdf_stream_t stream)
{
    if (n < 0 || width < 1 || height < 1 || num_images < 1 || !roi_min || !roi_max) return ATDF_ERR_INVALID_ARGUMENT;
    if (model != ATDF_CAMERA_PINHOLE && model != ATDF_CAMERA_ORTHOGRAPHIC) return ATDF_ERR_INVALID_ARGUMENT;
    if (n > 0 && (!points || !rotation || !intrinsics || !mask)) return ATDF_ERR_INVALID_ARGUMENT;
    if (n == 0) return ATDF_OK;
    const unsigned blocks = (unsigned)std::min<int64_t>(div_up(n, 256), 148 * 16);
    point_in_any_image_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(
        n, points, rotation, translation, num_images, intrinsics, model, width, height,
        make_float3(roi_min[0], roi_min[1], roi_min[2]), make_float3(roi_max[0], roi_max[1], roi_max[2]), mask);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

extern "C" int atdf_camera_rays(int64_t n, const float* uv, const int32_t* image_id, const int32_t* camera_id,
                                const double* rotation, const double* translation, int64_t num_images,
                                const double* intrinsics, int64_t num_cameras, int32_t width, int32_t height,
                                int32_t align_corners, int32_t model, const float* volume_translation,
                                float* origin, float* direction, int32_t* dev_error, atdf_stream_t stream)
{
    if (n < 0 || width < 1 || height < 1 || num_images < 1 || num_cameras < 1) return ATDF_ERR_INVALID_ARGUMENT;
    if (model != ATDF_CAMERA_PINHOLE && model != ATDF_CAMERA_ORTHOGRAPHIC) return ATDF_ERR_INVALID_ARGUMENT;
    if (n > 0 && (!uv || !image_id || !rotation || !intrinsics || !origin || !direction || !dev_error))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (model == ATDF_CAMERA_PINHOLE && n > 0 && !translation) return ATDF_ERR_INVALID_ARGUMENT;
    if (n == 0) return ATDF_OK;
    const float tv[3] = {volume_translation ? volume_translation[0] : 0.0f,
                         volume_translation ? volume_translation[1] : 0.0f,
                         volume_translation ? volume_translation[2] : 0.0f};
    const unsigned blocks = (unsigned)std::min<int64_t>(div_up(n, 256), 148 * 16);
    camera_rays_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(
        n, uv, image_id, camera_id, rotation, translation, num_images, intrinsics, num_cameras, width, height,
        align_corners, model, tv[0], tv[1], tv[2], origin, direction, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}
