// Line integrals of a voxel volume along rays, in FP64 with exact
// intersection lengths (Siddon's method, traversed voxel by voxel in the
// incremental form of Amanatides & Woo). This generates the training
// projections of the synthetic tilt series from a voxelised phantom; the
// reference reads measured tilt series instead
// (hyperacorn/csrc/data/SceneBase.cpp:904-1000).
#include <cuda_runtime.h>
#include <math.h>

#include "atdf.h"
#include "atdf_common.cuh"

namespace atdf {

struct SiddonGrid {
    const float* vol;  // [nz][ny][nx]
    int n[3];          // nx, ny, nz
    double bmin[3], bmax[3], h[3];
};

__global__ void siddon_kernel(SiddonGrid g, const float* __restrict__ origin, const float* __restrict__ dir,
                              int64_t R, double* __restrict__ out)
{
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    double o[3], d[3];
    for (int a = 0; a < 3; ++a) {
        o[a] = (double)origin[3 * r + a];
        d[a] = (double)dir[3 * r + a];
    }
    double t0 = -INFINITY, t1 = INFINITY;
    for (int a = 0; a < 3; ++a) {
        if (d[a] == 0.0) {
            if (o[a] < g.bmin[a] || o[a] >= g.bmax[a]) {
                out[r] = 0.0;
                return;
            }
        } else {
            const double ta = (g.bmin[a] - o[a]) / d[a], tb = (g.bmax[a] - o[a]) / d[a];
            t0 = fmax(t0, fmin(ta, tb));
            t1 = fmin(t1, fmax(ta, tb));
        }
    }
    if (!(t0 < t1)) {
        out[r] = 0.0;
        return;
    }
    // voxel containing the point just inside the entry face
    int idx[3], step[3];
    const double tin = t0 + 1e-9 * (t1 - t0);
    for (int a = 0; a < 3; ++a) {
        const double u = (o[a] + d[a] * tin - g.bmin[a]) / g.h[a];
        int i = (int)floor(u);
        idx[a] = i < 0 ? 0 : (i >= g.n[a] ? g.n[a] - 1 : i);
        step[a] = d[a] > 0 ? 1 : -1;
    }
    double acc = 0.0, t = t0;
    const int max_steps = g.n[0] + g.n[1] + g.n[2] + 3;
    for (int it = 0; it < max_steps && t < t1; ++it) {
        // parameter of the next voxel face crossed on each axis, recomputed
        // from the voxel index so that rounding does not accumulate
        double tn = t1;
        int axis = -1;
        for (int a = 0; a < 3; ++a) {
            if (d[a] == 0.0) continue;
            const double face = g.bmin[a] + (double)(idx[a] + (step[a] > 0 ? 1 : 0)) * g.h[a];
            const double ta = (face - o[a]) / d[a];
            if (ta < tn) {
                tn = ta;
                axis = a;
            }
        }
        if (tn > t) {
            const int64_t v = ((int64_t)idx[2] * g.n[1] + idx[1]) * g.n[0] + idx[0];
            acc += (tn - t) * (double)g.vol[v];
            t = tn;
        }
        if (axis < 0) break;
        idx[axis] += step[axis];
        if (idx[axis] < 0 || idx[axis] >= g.n[axis]) break;
    }
    out[r] = acc;
}

}  // namespace atdf

using namespace atdf;

extern "C" int atdf_siddon_project(const float* volume, int32_t nx, int32_t ny, int32_t nz, const double* box_min,
                                   const double* box_max, const float* ray_origin, const float* ray_direction,
                                   int64_t num_rays, double* out, atdf_stream_t stream)
{
    if (num_rays < 0 || nx <= 0 || ny <= 0 || nz <= 0 || !box_min || !box_max) return ATDF_ERR_INVALID_ARGUMENT;
    if (num_rays == 0) return ATDF_OK;
    if (!volume || !ray_origin || !ray_direction || !out) return ATDF_ERR_INVALID_ARGUMENT;
    SiddonGrid g;
    g.vol = volume;
    g.n[0] = nx;
    g.n[1] = ny;
    g.n[2] = nz;
    for (int a = 0; a < 3; ++a) {
        if (!(box_max[a] > box_min[a])) return ATDF_ERR_INVALID_ARGUMENT;
        g.bmin[a] = box_min[a];
        g.bmax[a] = box_max[a];
        g.h[a] = (box_max[a] - box_min[a]) / g.n[a];
    }
    const int threads = 128;
    siddon_kernel<<<(unsigned)((num_rays + threads - 1) / threads), threads, 0, (cudaStream_t)stream>>>(
        g, ray_origin, ray_direction, num_rays, out);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}
