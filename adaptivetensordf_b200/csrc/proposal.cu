// Learned proposal sampler: per ray/leaf segment a small MLP predicts a
// piecewise-constant density over 32 equal bins of the segment and the
// segment's mass, from the segment's leaf-local entry and exit points, its
// relative length and the leaf's occupancy (whole leaf and 8 octants). A
// ray's sample budget is split over its segments by predicted mass, and each
// segment's samples are placed by stratified inverse-CDF sampling of its bin
// density and weighted by their Voronoi cells along the segment, the
// quadrature the uniform sampler uses (HyperTree.cu:495-512), so dense
// placement refines the quadrature where the density is. The network is trained on the bins of rho * w that the
// uniform sampler's forward pass produces (atdf_project_forward_binned), and
// those bins also refresh the occupancy.
//
// The reference has no proposal sampler: it places max_samples_per_node
// uniform (optionally jittered) samples in every leaf a ray crosses
// (hyperacorn/csrc/structure/HyperTree.cu:266-514). Segments and sample
// offsets keep the reference's canonical per-ray layout.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>

#include "atdf.h"
#include "atdf_common.cuh"

namespace atdf {

constexpr int kPropBins = ATDF_PROPOSAL_BINS;
constexpr int kPropOut = ATDF_PROPOSAL_OUTPUTS;
constexpr int kPropIn = ATDF_PROPOSAL_INPUTS;
constexpr int kPropOcc = ATDF_PROPOSAL_OCC;

__device__ __forceinline__ float softplus1(float x) { return x > 20.0f ? x : log1pf(__expf(x)); }

__device__ __forceinline__ int octant_of(float x, float y, float z)
{
    return (x > 0.0f ? 1 : 0) | (y > 0.0f ? 2 : 0) | (z > 0.0f ? 4 : 0);
}

__global__ void proposal_features_kernel(atdf_tree_t tree, atdf_segments_t segs, const float* __restrict__ origin,
                                         const float* __restrict__ dir, const float* __restrict__ occupancy,
                                         float* __restrict__ feat, int32_t* err)
{
    const int64_t nseg = segs.totals[0];
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += (int64_t)gridDim.x * blockDim.x) {
        const int node = segs.node[s], r = segs.ray[s];
        float* f = feat + s * kPropIn;
        if (node < 0 || node >= tree.num_nodes) {
            set_err(err, ATDF_DEVERR_INDEX);
            for (int k = 0; k < kPropIn; ++k) f[k] = 0.0f;
            continue;
        }
        const float t0 = segs.tmin[s], t1 = segs.tmax[s];
        float diag2 = 0.0f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float mn = tree.node_position_min[3 * node + k], mx = tree.node_position_max[3 * node + k];
            const float o = origin[3 * r + k], d = dir[3 * r + k];
            const float inv = 2.0f / (mx - mn);
            f[k] = (o + d * t0 - mn) * inv - 1.0f;
            f[3 + k] = (o + d * t1 - mn) * inv - 1.0f;
            diag2 += (mx - mn) * (mx - mn);
        }
        f[6] = (t1 - t0) * rsqrtf(diag2);
        const float* oc = occupancy ? occupancy + (int64_t)node * kPropOcc : nullptr;
        f[7] = oc ? oc[8] : 0.0f;
#pragma unroll
        for (int q = 0; q < 8; ++q) f[8 + q] = oc ? oc[q] : 0.0f;
    }
}

// ---------------------------------------------------------------------------
// Proposal MLP: 16 -> 64 x NH (SiLU) -> 33, 64-row tiles in shared memory,
// register micro-tiles of 4 rows x 4 outputs. Activations are stored
// feature-major with a row stride of 65 floats; weights [out][in + 1], the
// last layer's outputs padded to 64 with zeros.
// ---------------------------------------------------------------------------
constexpr int kPT = 64;        // rows per tile
constexpr int kPS = kPT + 1;   // feature-major row stride
constexpr int kPH = 64;        // hidden width (and padded output width)
constexpr int kPThreads = 256;

struct PropMlp {
    const float* w[ATDF_MAX_LAYERS];
    const float* b[ATDF_MAX_LAYERS];
    float* gw[ATDF_MAX_LAYERS];
    float* gb[ATDF_MAX_LAYERS];
};

__host__ __device__ constexpr int prop_wfloats(int NH) { return kPH * (kPropIn + 1) + NH * kPH * (kPH + 1); }

// Weights (layer l at offset woff(l)) and biases into shared memory.
template <int NH>
__device__ __forceinline__ int woff(int l)
{
    return l == 0 ? 0 : kPH * (kPropIn + 1) + (l - 1) * kPH * (kPH + 1);
}

template <int NH>
__device__ void prop_load_weights(const PropMlp& m, float* sW, float* sB)
{
    for (int l = 0; l <= NH; ++l) {
        const int K = l == 0 ? kPropIn : kPH, O = l == NH ? kPropOut : kPH;
        float* W = sW + woff<NH>(l);
        for (int e = threadIdx.x; e < kPH * (K + 1); e += kPThreads) {
            const int o = e / (K + 1), k = e % (K + 1);
            W[e] = (o < O && k < K) ? m.w[l][o * K + k] : 0.0f;
        }
        for (int o = threadIdx.x; o < kPH; o += kPThreads) sB[l * kPH + o] = o < O ? m.b[l][o] : 0.0f;
    }
}

// acc[i][j] = sum_k in[k][rg + 16 i] * W[cg * 4 + j][k]
template <int K>
__device__ __forceinline__ void prop_gemm(const float* in, const float* W, float (&acc)[4][4])
{
    const int rg = threadIdx.x % 16, cg = threadIdx.x / 16;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
#pragma unroll 4
    for (int k = 0; k < K; ++k) {
        float a[4], w[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = in[k * kPS + rg + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; ++j) w[j] = W[(cg * 4 + j) * (K + 1) + k];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], w[j], acc[i][j]);
    }
}

__device__ __forceinline__ void prop_load_tile(const float* __restrict__ x, int64_t row0, int64_t nrows, float* X)
{
    for (int e = threadIdx.x; e < kPT * kPropIn; e += kPThreads) {
        const int r = e / kPropIn, k = e % kPropIn;
        const int64_t row = row0 + r;
        X[k * kPS + r] = row < nrows ? x[row * kPropIn + k] : 0.0f;
    }
}

template <int NH>
__global__ void __launch_bounds__(kPThreads) proposal_mlp_fwd_kernel(PropMlp m, const int64_t* __restrict__ count,
                                                                     const float* __restrict__ x,
                                                                     float* __restrict__ out)
{
    extern __shared__ float psm[];
    float* sW = psm;
    float* sB = sW + prop_wfloats(NH);
    float* X = sB + (NH + 1) * kPH;
    float* buf[2] = {X + kPropIn * kPS, X + kPropIn * kPS + kPH * kPS};
    prop_load_weights<NH>(m, sW, sB);
    const int64_t nrows = *count;
    const int rg = threadIdx.x % 16, cg = threadIdx.x / 16;
    for (int64_t row0 = (int64_t)blockIdx.x * kPT; row0 < nrows; row0 += (int64_t)gridDim.x * kPT) {
        __syncthreads();
        prop_load_tile(x, row0, nrows, X);
        __syncthreads();
        const float* in = X;
#pragma unroll
        for (int l = 0; l <= NH; ++l) {
            float acc[4][4];
            if (l == 0)
                prop_gemm<kPropIn>(in, sW + woff<NH>(0), acc);
            else
                prop_gemm<kPH>(in, sW + woff<NH>(l), acc);
            if (l < NH) {
                float* o = buf[l & 1];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float z = acc[i][j] + sB[l * kPH + cg * 4 + j];
                        o[(cg * 4 + j) * kPS + rg + 16 * i] = act_fwd(ATDF_ACT_SILU, z, 1.0f);
                    }
                __syncthreads();
                in = o;
            } else {
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int64_t row = row0 + rg + 16 * i;
                    if (row >= nrows) continue;
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int c = cg * 4 + j;
                        if (c < kPropOut) out[row * kPropOut + c] = acc[i][j] + sB[l * kPH + c];
                    }
                }
            }
        }
    }
}

template <int NH>
__host__ __device__ constexpr int prop_bwd_floats()
{
    return prop_wfloats(NH) + (NH + 1) * kPH + kPropIn * kPS + 2 * NH * kPH * kPS + 2 * kPH * kPS;
}

template <int NH>
__global__ void __launch_bounds__(kPThreads, 1) proposal_mlp_bwd_kernel(PropMlp m, const int64_t* __restrict__ count,
                                                                        const float* __restrict__ x,
                                                                        const float* __restrict__ gout)
{
    extern __shared__ float psm[];
    float* sW = psm;
    float* sB = sW + prop_wfloats(NH);
    float* X = sB + (NH + 1) * kPH;
    float* Z = X + kPropIn * kPS;       // [NH][64][kPS] pre-activations
    float* A = Z + NH * kPH * kPS;      // [NH][64][kPS] activations
    float* D[2] = {A + NH * kPH * kPS, A + NH * kPH * kPS + kPH * kPS};
    prop_load_weights<NH>(m, sW, sB);
    const int64_t nrows = *count;
    const int tid = threadIdx.x, rg = tid % 16, cg = tid / 16;
    // weight-gradient accumulators, kept across tiles
    float g0[4];        // layer 0: k = tid % 16, outputs (tid / 16) * 4 + j
    float gh[NH][16];   // layers 1..NH: [4 i + j] = (output cg * 4 + j, input rg + 16 i)
    float gbias[NH + 1];
#pragma unroll
    for (int j = 0; j < 4; ++j) g0[j] = 0.0f;
#pragma unroll
    for (int l = 0; l < NH; ++l)
#pragma unroll
        for (int j = 0; j < 16; ++j) gh[l][j] = 0.0f;
#pragma unroll
    for (int l = 0; l <= NH; ++l) gbias[l] = 0.0f;

    for (int64_t row0 = (int64_t)blockIdx.x * kPT; row0 < nrows; row0 += (int64_t)gridDim.x * kPT) {
        __syncthreads();
        prop_load_tile(x, row0, nrows, X);
        // dZ of the last layer: dlogits, padded to 64 outputs; rows past the end are zero
        for (int e = tid; e < kPT * kPH; e += kPThreads) {
            const int r = e / kPH, c = e % kPH;
            const int64_t row = row0 + r;
            D[NH & 1][c * kPS + r] = (row < nrows && c < kPropOut) ? gout[row * kPropOut + c] : 0.0f;
        }
        __syncthreads();
        // forward, keeping pre-activations and activations of the hidden layers
#pragma unroll
        for (int l = 0; l < NH; ++l) {
            float acc[4][4];
            if (l == 0)
                prop_gemm<kPropIn>(X, sW + woff<NH>(0), acc);
            else
                prop_gemm<kPH>(A + (l - 1) * kPH * kPS, sW + woff<NH>(l), acc);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int e = (cg * 4 + j) * kPS + rg + 16 * i;
                    const float z = acc[i][j] + sB[l * kPH + cg * 4 + j];
                    Z[l * kPH * kPS + e] = z;
                    A[l * kPH * kPS + e] = act_fwd(ATDF_ACT_SILU, z, 1.0f);
                }
            __syncthreads();
        }
        // backward through the layers
#pragma unroll
        for (int l = NH; l >= 0; --l) {
            const float* dz = D[l & 1];
            const float* in = l == 0 ? X : A + (l - 1) * kPH * kPS;
            if (l == 0) {
                const int k = tid % kPropIn, og = tid / kPropIn;
                for (int r = 0; r < kPT; ++r) {
                    const float a = in[k * kPS + r];
#pragma unroll
                    for (int j = 0; j < 4; ++j) g0[j] = fmaf(a, dz[(og * 4 + j) * kPS + r], g0[j]);
                }
            } else {
                // 4 x 4 outer products per row: 16 FMAs for 8 shared loads (the
                // inputs rg + 16 i sit 65 floats apart: distinct banks)
#pragma unroll 4
                for (int r = 0; r < kPT; ++r) {
                    float a[4], d[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) a[i] = in[(rg + 16 * i) * kPS + r];
#pragma unroll
                    for (int j = 0; j < 4; ++j) d[j] = dz[(cg * 4 + j) * kPS + r];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) gh[l - 1][4 * i + j] = fmaf(a[i], d[j], gh[l - 1][4 * i + j]);
                }
            }
            if (tid < kPH) {
                float s = 0.0f;
                for (int r = 0; r < kPT; ++r) s += dz[tid * kPS + r];
                gbias[l] += s;
            }
            if (l > 0) {
                // dA[k][r] = sum_o W[o][k] dZ[o][r]; dZ_prev = dA * silu'(Z_prev)
                const float* W = sW + woff<NH>(l);
                float acc[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
#pragma unroll 4
                for (int o = 0; o < kPH; ++o) {
                    float a[4], w[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) a[i] = dz[o * kPS + rg + 16 * i];
#pragma unroll
                    for (int j = 0; j < 4; ++j) w[j] = W[o * (kPH + 1) + cg * 4 + j];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], w[j], acc[i][j]);
                }
                float* dprev = D[(l - 1) & 1];
                const float* zprev = Z + (l - 1) * kPH * kPS;
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int e = (cg * 4 + j) * kPS + rg + 16 * i;
                        dprev[e] = acc[i][j] * act_grad(ATDF_ACT_SILU, zprev[e], 1.0f);
                    }
            }
            __syncthreads();
        }
    }
    // flush this CTA's gradients
    {
        const int k = tid % kPropIn, og = tid / kPropIn;
#pragma unroll
        for (int j = 0; j < 4; ++j) atomicAdd(&m.gw[0][(og * 4 + j) * kPropIn + k], g0[j]);
    }
#pragma unroll
    for (int l = 1; l <= NH; ++l) {
        const int O = l == NH ? kPropOut : kPH;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int o = cg * 4 + j, k = rg + 16 * i;
                if (o < O) atomicAdd(&m.gw[l][o * kPH + k], gh[l - 1][4 * i + j]);
            }
    }
    if (tid < kPH) {
#pragma unroll
        for (int l = 0; l <= NH; ++l) {
            const int O = l == NH ? kPropOut : kPH;
            if (tid < O) atomicAdd(&m.gb[l][tid], gbias[l]);
        }
    }
}

// ---------------------------------------------------------------------------
// allocation, sampling, loss, occupancy
// ---------------------------------------------------------------------------
// Allocation weight of a segment: len * (predicted mean density)^power.
__device__ __forceinline__ float alloc_weight(const float* lg, float len, float power)
{
    const float dens = softplus1(lg[kPropBins]);
    return power == 0.0f ? len : len * __powf(fmaxf(dens, 1e-20f), power);
}

// One warp per ray, a lane per segment (in chunks of 32): sample counts of
// the ray's segments from the predicted densities; writes nsamp, first
// (within the ray, a warp scan) and the ray's total into
// ray_sample_offset[r] (scanned afterwards).
__global__ void proposal_allocate_kernel(atdf_segments_t segs, int64_t R, const float* __restrict__ logits,
                                         int32_t budget, float mass_mix, float mass_power)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < R; r += warps) {
        const int64_t b = segs.ray_seg_offset[r], e = segs.ray_seg_offset[r + 1];
        const int nseg = (int)(e - b);
        float msum = 0.0f, lsum = 0.0f;
        for (int64_t s = b + lane; s < e; s += 32) {
            const float len = segs.tmax[s] - segs.tmin[s];
            msum += alloc_weight(logits + s * kPropOut, len, mass_power);
            lsum += len;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            msum += __shfl_xor_sync(0xffffffffu, msum, o);
            lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        }
        const int spare = budget > nseg ? budget - nseg : 0;
        int run = 0;
        for (int64_t s0 = b; s0 < e; s0 += 32) {
            const int64_t s = s0 + lane;
            int n = 0;
            if (s < e) {
                const float len = segs.tmax[s] - segs.tmin[s];
                const float m = alloc_weight(logits + s * kPropOut, len, mass_power);
                float share = lsum > 0.0f ? len / lsum : 1.0f / (float)nseg;
                if (msum > 0.0f) share = (1.0f - mass_mix) * (m / msum) + mass_mix * share;
                n = 1 + (int)floorf((float)spare * share + 0.5f);
            }
            int incl = n;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            if (s < e) {
                segs.nsamp[s] = n;
                segs.first[s] = run + incl - n;
            }
            run += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) {
            segs.ray_sample_offset[r] = run;
            atomicMax((unsigned long long*)&segs.totals[2], (unsigned long long)run);
        }
    }
}

// Bin probabilities of a segment: softmax of power * (the 32 logits), i.e.
// the predicted bin distribution raised to power and renormalised, mixed
// with the uniform density.
__device__ __forceinline__ void bin_probs(const float* lg, float bin_mix, float* p, float power = 1.0f)
{
    float mx = lg[0];
    for (int b = 1; b < kPropBins; ++b) mx = fmaxf(mx, lg[b]);
    float sum = 0.0f;
    for (int b = 0; b < kPropBins; ++b) {
        p[b] = __expf(power * (lg[b] - mx));
        sum += p[b];
    }
    const float inv = (1.0f - bin_mix) / sum, u = bin_mix / (float)kPropBins;
    for (int b = 0; b < kPropBins; ++b) p[b] = p[b] * inv + u;
}

// One thread per segment. The bin probabilities live in shared memory, one
// column per thread (the bin search indexes them by a run-time bin, which in
// a register array would go to local memory).
constexpr int kSampThreads = 256;

__global__ void __launch_bounds__(kSampThreads) proposal_samples_kernel(atdf_segments_t segs,
                                                                        const float* __restrict__ logits,
                                                                        float bin_mix, float bin_power, uint64_t seed,
                                                                        int weight_rule,
                                                                        float* __restrict__ sample_t,
                                                                        float* __restrict__ sample_w, int64_t capacity,
                                                                        int32_t* err)
{
    __shared__ float s_p[kPropBins * kSampThreads];
    float* p = s_p + threadIdx.x;  // bin b at p[b * kSampThreads]
    const int64_t nseg = segs.totals[0];
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += (int64_t)gridDim.x * blockDim.x) {
        const int n = segs.nsamp[s], r = segs.ray[s], node = segs.node[s];
        if (n <= 0) continue;
        const int64_t base = segs.ray_sample_offset[r] + segs.first[s];
        if (base < 0 || base + n > capacity) {
            set_err(err, ATDF_DEVERR_SAMPLE_CAPACITY);
            continue;
        }
        {
            float q[kPropBins];
            bin_probs(logits + s * kPropOut, bin_mix, q, bin_power);
#pragma unroll
            for (int b = 0; b < kPropBins; ++b) p[b * kSampThreads] = q[b];
        }
        const float t0 = segs.tmin[s], t1 = segs.tmax[s];
        const float binw = (t1 - t0) / (float)kPropBins;
        int bcur = 0;
        float cdf = 0.0f;  // CDF at the start of bin bcur
        // t of sample j; j increases, so the bin search only moves forward
        auto place = [&](int j) {
            const float a = seed ? jitter(seed, r, node, j) : 0.5f;
            const float u = ((float)j + a) / (float)n;
            while (bcur < kPropBins - 1 && cdf + p[bcur * kSampThreads] <= u) {
                cdf += p[bcur * kSampThreads];
                ++bcur;
            }
            float frac = (u - cdf) / p[bcur * kSampThreads];
            frac = fminf(fmaxf(frac, 0.0f), 1.0f);
            const float t = t0 + ((float)bcur + frac) * binw;
            return fminf(fmaxf(t, t0), t1);
        };
        if (weight_rule == ATDF_PROPOSAL_WEIGHTS_IMPORTANCE) {
            // importance weights: sample j stands for probability 1 / n of q,
            // whose density in its bin b is p_b / binw, so w = binw / (n p_b)
            // and sum_j w_j rho(t_j) estimates the segment integral without
            // bias when the jitter is uniform
            const float inv_n = 1.0f / (float)n;
            for (int j = 0; j < n; ++j) {
                sample_t[base + j] = place(j);
                sample_w[base + j] = binw * inv_n / p[bcur * kSampThreads];
            }
            continue;
        }
        // weights: the Voronoi cells of the placed samples within the segment,
        // the rule the uniform sampler applies to its own samples
        float t_prev = 0.0f, t_cur = place(0);
        for (int j = 0; j < n; ++j) {
            const float t_next = j + 1 < n ? place(j + 1) : 0.0f;
            sample_t[base + j] = t_cur;
            sample_w[base + j] = atdf::sample_w(t0, t1, n, j, t_prev, t_cur, t_next);
            t_prev = t_cur;
            t_cur = t_next;
        }
    }
}

// Proposal loss per segment against the uniform pass's bins of rho * w:
// cross-entropy of the normalised bins against the bin probabilities
// (without the uniform mixture), plus mass_weight * (log(m_hat + d) -
// log(m + d))^2 with m_hat = softplus(logit_32) * len; averaged over
// segments. Adds each bin's target mass and length into its leaf octant
// (bin centre between the features' entry and exit points) and the leaf.
__global__ void proposal_loss_kernel(atdf_segments_t segs, const float* __restrict__ feat,
                                     const float* __restrict__ bins, const float* __restrict__ logits,
                                     float mass_weight, float* __restrict__ dlogits, double* loss, double* node_mass,
                                     double* node_len, int64_t num_nodes, int32_t* err)
{
    const int64_t nseg = segs.totals[0];
    const float invG = nseg > 0 ? 1.0f / (float)nseg : 0.0f;
    double local = 0.0;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += (int64_t)gridDim.x * blockDim.x) {
        const float* lg = logits + s * kPropOut;
        const float* h = bins + s * kPropBins;
        const float* f = feat + s * kPropIn;
        float* d = dlogits + s * kPropOut;
        float p[kPropBins];
        bin_probs(lg, 0.0f, p);
        float m = 0.0f;
        for (int b = 0; b < kPropBins; ++b) m += fmaxf(h[b], 0.0f);
        float ce = 0.0f;
        for (int b = 0; b < kPropBins; ++b) {
            const float hb = m > 0.0f ? fmaxf(h[b], 0.0f) / m : 0.0f;
            if (m > 0.0f) ce -= hb * __logf(fmaxf(p[b], 1e-30f));
            d[b] = m > 0.0f ? (p[b] - hb) * invG : 0.0f;
        }
        const float len = segs.tmax[s] - segs.tmin[s];
        const float z = lg[kPropBins];
        const float mh = softplus1(z) * len;
        const float delta = 1e-4f;
        const float e = __logf(mh + delta) - __logf(m + delta);
        const float sig = 1.0f / (1.0f + __expf(-z));
        d[kPropBins] = mass_weight * 2.0f * e / (mh + delta) * len * sig * invG;
        local += (double)((ce + mass_weight * e * e) * invG);
        const int node = segs.node[s];
        if (node < 0 || node >= num_nodes) {
            set_err(err, ATDF_DEVERR_INDEX);
            continue;
        }
        float om[8], ol[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) om[q] = ol[q] = 0.0f;
        const float binw = len / (float)kPropBins;
        for (int b = 0; b < kPropBins; ++b) {
            const float c = ((float)b + 0.5f) / (float)kPropBins;
            const int q = octant_of(f[0] + c * (f[3] - f[0]), f[1] + c * (f[4] - f[1]), f[2] + c * (f[5] - f[2]));
            om[q] += fmaxf(h[b], 0.0f);
            ol[q] += binw;
        }
        double* nm = node_mass + (int64_t)node * kPropOcc;
        double* nl = node_len + (int64_t)node * kPropOcc;
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (ol[q] > 0.0f) {
                atomicAdd(&nm[q], (double)om[q]);
                atomicAdd(&nl[q], (double)ol[q]);
            }
        atomicAdd(&nm[8], (double)m);
        atomicAdd(&nl[8], (double)len);
    }
    // warp-reduce the loss before one atomic per warp
    for (int off = 16; off > 0; off >>= 1) local += __shfl_down_sync(0xffffffffu, local, off);
    if ((threadIdx.x & 31) == 0 && local != 0.0) atomicAdd(loss, local);
}

__global__ void proposal_occupancy_kernel(const double* node_mass, const double* node_len, int64_t n,
                                          float* occupancy)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (node_len[i] > 0.0) occupancy[i] = (float)(node_mass[i] / node_len[i]);
}

static unsigned seg_blocks(int64_t capacity)
{
    const int64_t b = div_up(capacity, 256);
    return (unsigned)std::min<int64_t>(std::max<int64_t>(b, 1), 148 * 16);
}

static int prop_hidden_layers(const atdf_mlp_t* m)
{
    if (!m || m->num_layers < 2 || m->num_layers > 4) return -1;
    if (m->dims[0] != kPropIn || m->dims[m->num_layers] != kPropOut) return -1;
    for (int l = 1; l < m->num_layers; ++l)
        if (m->dims[l] != kPH) return -1;
    if (m->hidden_activation != ATDF_ACT_SILU || m->last_activation != ATDF_ACT_ID) return -1;
    for (int l = 0; l < m->num_layers; ++l)
        if (!m->weight[l] || !m->bias[l]) return -1;
    return m->num_layers - 1;
}

template <int NH>
static int launch_prop_fwd(const PropMlp& pm, const atdf_segments_t& s, const float* x, float* out, cudaStream_t st)
{
    const int smem = (prop_wfloats(NH) + (NH + 1) * kPH + kPropIn * kPS + 2 * kPH * kPS) * 4;
    auto fn = proposal_mlp_fwd_kernel<NH>;
    ATDF_CUDA_TRY(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int dev = 0, sms = 0, per = 0;
    ATDF_CUDA_TRY(cudaGetDevice(&dev));
    ATDF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    ATDF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)fn, kPThreads, smem));
    const int64_t tiles = std::max<int64_t>(1, div_up(s.capacity, kPT));
    const unsigned grid = (unsigned)std::min<int64_t>(tiles, (int64_t)sms * std::max(per, 1));
    fn<<<grid, kPThreads, smem, st>>>(pm, s.totals, x, out);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

template <int NH>
static int launch_prop_bwd(const PropMlp& pm, const atdf_segments_t& s, const float* x, const float* g,
                           cudaStream_t st)
{
    const int smem = prop_bwd_floats<NH>() * 4;
    auto fn = proposal_mlp_bwd_kernel<NH>;
    ATDF_CUDA_TRY(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int dev = 0, sms = 0;
    ATDF_CUDA_TRY(cudaGetDevice(&dev));
    ATDF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t tiles = std::max<int64_t>(1, div_up(s.capacity, kPT));
    const unsigned grid = (unsigned)std::min<int64_t>(tiles, (int64_t)sms);
    fn<<<grid, kPThreads, smem, st>>>(pm, s.totals, x, g);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

}  // namespace atdf

using namespace atdf;

extern "C" {

int atdf_proposal_features(const atdf_tree_t* tree, const atdf_segments_t* segments, const float* ray_origin,
                           const float* ray_direction, const float* occupancy, float* features, int32_t* dev_error,
                           atdf_stream_t stream)
{
    if (!tree || !segments || !ray_origin || !ray_direction || !features || !segments->totals)
        return ATDF_ERR_INVALID_ARGUMENT;
    proposal_features_kernel<<<seg_blocks(segments->capacity), 256, 0, (cudaStream_t)stream>>>(
        *tree, *segments, ray_origin, ray_direction, occupancy, features, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_proposal_mlp_forward(const atdf_mlp_t* mlp, const atdf_segments_t* segments, const float* features,
                              float* logits, atdf_stream_t stream)
{
    if (!segments || !segments->totals || !features || !logits) return ATDF_ERR_INVALID_ARGUMENT;
    const int nh = prop_hidden_layers(mlp);
    if (nh < 1) return ATDF_ERR_UNSUPPORTED;
    PropMlp pm{};
    for (int l = 0; l < mlp->num_layers; ++l) {
        pm.w[l] = mlp->weight[l];
        pm.b[l] = mlp->bias[l];
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (nh == 1) return launch_prop_fwd<1>(pm, *segments, features, logits, s);
    if (nh == 2) return launch_prop_fwd<2>(pm, *segments, features, logits, s);
    return launch_prop_fwd<3>(pm, *segments, features, logits, s);
}

int atdf_proposal_mlp_backward(const atdf_mlp_t* mlp, const atdf_segments_t* segments, const float* features,
                               const float* grad_logits, const atdf_mlp_grad_t* grad_mlp, atdf_stream_t stream)
{
    if (!segments || !segments->totals || !features || !grad_logits || !grad_mlp) return ATDF_ERR_INVALID_ARGUMENT;
    const int nh = prop_hidden_layers(mlp);
    if (nh < 1) return ATDF_ERR_UNSUPPORTED;
    PropMlp pm{};
    cudaStream_t s = (cudaStream_t)stream;
    for (int l = 0; l < mlp->num_layers; ++l) {
        if (!grad_mlp->weight[l] || !grad_mlp->bias[l]) return ATDF_ERR_INVALID_ARGUMENT;
        pm.w[l] = mlp->weight[l];
        pm.b[l] = mlp->bias[l];
        pm.gw[l] = grad_mlp->weight[l];
        pm.gb[l] = grad_mlp->bias[l];
        ATDF_CUDA_TRY(cudaMemsetAsync(pm.gw[l], 0, (size_t)mlp->dims[l] * mlp->dims[l + 1] * sizeof(float), s));
        ATDF_CUDA_TRY(cudaMemsetAsync(pm.gb[l], 0, (size_t)mlp->dims[l + 1] * sizeof(float), s));
    }
    if (nh == 1) return launch_prop_bwd<1>(pm, *segments, features, grad_logits, s);
    if (nh == 2) return launch_prop_bwd<2>(pm, *segments, features, grad_logits, s);
    return launch_prop_bwd<3>(pm, *segments, features, grad_logits, s);
}

int atdf_proposal_allocate(const atdf_segments_t* segments, int64_t num_rays, const float* logits, int32_t budget,
                           float mass_mix, float mass_power, atdf_stream_t stream)
{
    if (!segments || !logits || num_rays < 0 || budget < 1 || !(mass_mix >= 0.0f && mass_mix <= 1.0f) ||
        !(mass_power >= 0.0f && mass_power <= 1.0f))
        return ATDF_ERR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    ATDF_CUDA_TRY(cudaMemsetAsync(&segments->totals[2], 0, sizeof(int64_t), s));
    if (num_rays > 0) {
        const unsigned blocks = (unsigned)std::min<int64_t>(div_up(num_rays, 8), 148 * 16);  // 8 rays per block
        proposal_allocate_kernel<<<blocks, 256, 0, s>>>(*segments, num_rays, logits, budget, mass_mix, mass_power);
        ATDF_LAUNCH_CHECK();
    }
    ATDF_CUDA_TRY(cudaMemsetAsync(&segments->ray_sample_offset[num_rays], 0, sizeof(int64_t), s));
    scan_exclusive_i64_kernel<<<1, 1024, 0, s>>>(segments->ray_sample_offset, num_rays + 1, nullptr);
    ATDF_LAUNCH_CHECK();
    ATDF_CUDA_TRY(cudaMemcpyAsync(&segments->totals[1], &segments->ray_sample_offset[num_rays], sizeof(int64_t),
                                  cudaMemcpyDeviceToDevice, s));
    return ATDF_OK;
}

int atdf_proposal_samples(const atdf_segments_t* segments, const float* logits, float bin_mix, float bin_power,
                          uint64_t seed, int32_t weight_rule, float* sample_t, float* sample_w,
                          int64_t sample_capacity, int32_t* dev_error, atdf_stream_t stream)
{
    if (!segments || !logits || !sample_t || !sample_w || sample_capacity < 0 ||
        !(bin_mix > 0.0f && bin_mix <= 1.0f) || !(bin_power >= 0.0f && bin_power <= 1.0f) ||
        (weight_rule != ATDF_PROPOSAL_WEIGHTS_VORONOI && weight_rule != ATDF_PROPOSAL_WEIGHTS_IMPORTANCE))
        return ATDF_ERR_INVALID_ARGUMENT;
    proposal_samples_kernel<<<seg_blocks(segments->capacity), kSampThreads, 0, (cudaStream_t)stream>>>(
        *segments, logits, bin_mix, bin_power, seed, weight_rule, sample_t, sample_w, sample_capacity, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_proposal_loss(const atdf_segments_t* segments, const float* features, const float* seg_bins,
                       const float* logits, float mass_weight, float* grad_logits, double* loss, double* node_mass,
                       double* node_len, int64_t num_nodes, int32_t* dev_error, atdf_stream_t stream)
{
    if (!segments || !features || !seg_bins || !logits || !grad_logits || !loss || !node_mass || !node_len ||
        num_nodes < 0)
        return ATDF_ERR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    ATDF_CUDA_TRY(cudaMemsetAsync(loss, 0, sizeof(double), s));
    ATDF_CUDA_TRY(cudaMemsetAsync(node_mass, 0, num_nodes * kPropOcc * sizeof(double), s));
    ATDF_CUDA_TRY(cudaMemsetAsync(node_len, 0, num_nodes * kPropOcc * sizeof(double), s));
    proposal_loss_kernel<<<seg_blocks(segments->capacity), 256, 0, s>>>(*segments, features, seg_bins, logits,
                                                                       mass_weight, grad_logits, loss, node_mass,
                                                                       node_len, num_nodes, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_proposal_occupancy(const double* node_mass, const double* node_len, int64_t num_nodes, float* occupancy,
                            atdf_stream_t stream)
{
    if (!node_mass || !node_len || !occupancy || num_nodes < 0) return ATDF_ERR_INVALID_ARGUMENT;
    if (num_nodes == 0) return ATDF_OK;
    const int64_t n = num_nodes * kPropOcc;
    proposal_occupancy_kernel<<<(unsigned)div_up(n, 256), 256, 0, (cudaStream_t)stream>>>(node_mass, node_len, n,
                                                                                          occupancy);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

}  // extern "C"
