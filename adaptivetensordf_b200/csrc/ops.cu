// Unfused drop-in operators of the projection path for sm_100a: the two
// indirect grid-sample ops, GradientCorrection's backward, the VM feature
// field, the decoder MLP, the X-ray line integral, node-error scoring and the
// MSE loss. They keep the reference's per-op interfaces so callers can swap
// them in one at a time; the fused leaf-major path lives in fused.cu.
//
// Reference: hyperacorn/csrc/modules/IndirectGridSample2D.cu:22-393,
// IndirectGridSample1D.cu:20-140, GradientCorrection.cu:22-48;
// hyperacorn/csrc/geometry/geometry_tensor_qo.cpp:257-380, Modules.h:23-149,
// geometry.cpp:33-53,176-253,977-1019.

#include "atdf_common.cuh"

namespace atdf {

// ---------------------------------------------------------------------------
// grid sample 2D / 1D (one thread per sample, channels in a loop)
// ---------------------------------------------------------------------------
__global__ void gs2_fwd_kernel(const float* __restrict__ grid, int64_t N, int64_t C, int H, int W, int64_t sN,
                               int64_t sC, int64_t sH, int64_t sW, const int64_t* __restrict__ index,
                               const float* __restrict__ uv, int64_t S, float* __restrict__ out, int32_t* err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S) return;
    const int64_t n = index[i];
    if (n < 0 || n >= N) {
        set_err(err, ATDF_DEVERR_INDEX);
        for (int64_t c = 0; c < C; ++c) out[i * C + c] = 0.0f;
        return;
    }
    const Corner2 k = corners2(uv[2 * i], uv[2 * i + 1], H, W);
    const float* g = grid + n * sN;
    for (int64_t c = 0; c < C; ++c) {
        const float* gc = g + c * sC;
        out[i * C + c] = bilerp(k, gc[k.y0 * sH + k.x0 * sW], gc[k.y0 * sH + k.x1 * sW], gc[k.y1 * sH + k.x0 * sW],
                                gc[k.y1 * sH + k.x1 * sW]);
    }
}

__global__ void gs2_bwd_kernel(const float* __restrict__ grid, int64_t N, int64_t C, int H, int W, int64_t sN,
                               int64_t sC, int64_t sH, int64_t sW, const int64_t* __restrict__ index,
                               const float* __restrict__ uv, int64_t S, const float* __restrict__ gout,
                               float* __restrict__ ggrid, float* __restrict__ guv, int32_t* err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S) return;
    const int64_t n = index[i];
    if (n < 0 || n >= N) {
        set_err(err, ATDF_DEVERR_INDEX);
        return;
    }
    const Corner2 k = corners2(uv[2 * i], uv[2 * i + 1], H, W);
    const float* g = grid + n * sN;
    float* gg = ggrid ? ggrid + n * C * H * W : nullptr;
    float gix = 0.0f, giy = 0.0f;
    const float ay1 = __fsub_rn(k.fy1, k.iy), ay0 = __fsub_rn(k.iy, k.fy0);
    const float ax1 = __fsub_rn(k.fx1, k.ix), ax0 = __fsub_rn(k.ix, k.fx0);
    for (int64_t c = 0; c < C; ++c) {
        const float go = gout[i * C + c];
        const float* gc = g + c * sC;
        if (gg) {
            float* ggc = gg + c * H * W;
            atomicAdd(&ggc[k.y0 * W + k.x0], __fmul_rn(k.w_nw, go));
            atomicAdd(&ggc[k.y0 * W + k.x1], __fmul_rn(k.w_ne, go));
            atomicAdd(&ggc[k.y1 * W + k.x0], __fmul_rn(k.w_sw, go));
            atomicAdd(&ggc[k.y1 * W + k.x1], __fmul_rn(k.w_se, go));
        }
        const float vnw = gc[k.y0 * sH + k.x0 * sW], vne = gc[k.y0 * sH + k.x1 * sW];
        const float vsw = gc[k.y1 * sH + k.x0 * sW], vse = gc[k.y1 * sH + k.x1 * sW];
        // IndirectGridSample2D.cu:354-367, one rounding per operation
        gix = __fadd_rn(gix, __fmul_rn(__fmul_rn(__fmul_rn(-1.0f, vnw), ay1), go));
        gix = __fadd_rn(gix, __fmul_rn(__fmul_rn(vne, ay1), go));
        gix = __fadd_rn(gix, __fmul_rn(__fmul_rn(__fmul_rn(-1.0f, vsw), ay0), go));
        gix = __fadd_rn(gix, __fmul_rn(__fmul_rn(vse, ay0), go));
        giy = __fadd_rn(giy, __fmul_rn(__fmul_rn(__fmul_rn(-1.0f, vnw), ax1), go));
        giy = __fadd_rn(giy, __fmul_rn(__fmul_rn(__fmul_rn(-1.0f, vne), ax0), go));
        giy = __fadd_rn(giy, __fmul_rn(__fmul_rn(vsw, ax1), go));
        giy = __fadd_rn(giy, __fmul_rn(__fmul_rn(vse, ax0), go));
    }
    if (guv) {
        guv[2 * i] = __fadd_rn(guv[2 * i], __fdiv_rn(__fmul_rn(gix, (float)(W - 1)), 2.0f));
        guv[2 * i + 1] = __fadd_rn(guv[2 * i + 1], __fdiv_rn(__fmul_rn(giy, (float)(H - 1)), 2.0f));
    }
}

__global__ void gs1_fwd_kernel(const float* __restrict__ grid, int64_t N, int64_t C, int W, int64_t sN, int64_t sC,
                               int64_t sW, const int64_t* __restrict__ index, const float* __restrict__ uv, int64_t S,
                               float* __restrict__ out, int32_t* err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S) return;
    const int64_t n = index[i];
    if (n < 0 || n >= N) {
        set_err(err, ATDF_DEVERR_INDEX);
        for (int64_t c = 0; c < C; ++c) out[i * C + c] = 0.0f;
        return;
    }
    const Corner1 k = corners1(uv[i], W);
    const float* g = grid + n * sN;
    for (int64_t c = 0; c < C; ++c) out[i * C + c] = lerp1(k, g[c * sC + k.x0 * sW], g[c * sC + k.x1 * sW]);
}

__global__ void gs1_bwd_kernel(const float* __restrict__ grid, int64_t N, int64_t C, int W, int64_t sN, int64_t sC,
                               int64_t sW, const int64_t* __restrict__ index, const float* __restrict__ uv, int64_t S,
                               const float* __restrict__ gout, float* __restrict__ ggrid, float* __restrict__ guv,
                               int32_t* err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S) return;
    const int64_t n = index[i];
    if (n < 0 || n >= N) {
        set_err(err, ATDF_DEVERR_INDEX);
        return;
    }
    const Corner1 k = corners1(uv[i], W);
    const float* g = grid + n * sN;
    float* gg = ggrid ? ggrid + n * C * W : nullptr;
    float gix = 0.0f;
    const float a1 = __fsub_rn(k.fx1, k.ix), a0 = __fsub_rn(k.ix, k.fx0);
    for (int64_t c = 0; c < C; ++c) {
        const float go = gout[i * C + c];
        if (gg) {
            atomicAdd(&gg[c * W + k.x0], __fmul_rn(k.w0, go));
            atomicAdd(&gg[c * W + k.x1], __fmul_rn(k.w1, go));
        }
        const float v0 = g[c * sC + k.x0 * sW], v1 = g[c * sC + k.x1 * sW];
        gix = __fadd_rn(gix, __fmul_rn(__fmul_rn(__fmul_rn(-1.0f, v0), a1), go));
        gix = __fadd_rn(gix, __fmul_rn(__fmul_rn(v1, a0), go));
    }
    if (guv) guv[i] = __fadd_rn(guv[i], __fdiv_rn(__fmul_rn(gix, (float)(W - 1)), 2.0f));
}

__global__ void gradcorr_bwd_kernel(const float* __restrict__ dir, const int64_t* __restrict__ ray, int64_t R,
                                    const float* __restrict__ gin, int64_t S, float* __restrict__ gout, int32_t* err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S) return;
    const int64_t r = ray[i];
    if (r < 0 || r >= R) {
        set_err(err, ATDF_DEVERR_INDEX);
        return;
    }
    const float d0 = dir[3 * r], d1 = dir[3 * r + 1], d2 = dir[3 * r + 2];
    const float g0 = gin[3 * i], g1 = gin[3 * i + 1], g2 = gin[3 * i + 2];
    // grad - grad.dot(direction) * direction, one rounding per operation
    // (the dot product summed left to right), so the result is reproducible
    const float dot = __fadd_rn(__fadd_rn(__fmul_rn(g0, d0), __fmul_rn(g1, d1)), __fmul_rn(g2, d2));
    gout[3 * i] = __fsub_rn(g0, __fmul_rn(dot, d0));
    gout[3 * i + 1] = __fsub_rn(g1, __fmul_rn(dot, d1));
    gout[3 * i + 2] = __fsub_rn(g2, __fmul_rn(dot, d2));
}

// ---------------------------------------------------------------------------
// VM feature field, FP32, channels-last (one thread per sample)
// ---------------------------------------------------------------------------
__global__ void vm_fwd_kernel(atdf_field_t f, const float* __restrict__ pmin, const float* __restrict__ pmax,
                              int64_t num_nodes, const float* __restrict__ pos, const int64_t* __restrict__ node,
                              int64_t S, float* __restrict__ out, int32_t* err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S) return;
    const int C = f.channels;
    const int F = f.mode ? 3 * C : C;
    float* o = out + i * F;
    const int64_t nd = node[i];
    if (nd < 0 || nd >= num_nodes) {
        set_err(err, ATDF_DEVERR_INDEX);
        for (int c = 0; c < F; ++c) o[c] = 0.0f;
        return;
    }
    const int64_t slot = f.leaf_slot[nd];
    if (slot < 0 || slot >= f.num_slots) {
        if (slot >= f.num_slots) set_err(err, ATDF_DEVERR_INDEX);
        for (int c = 0; c < F; ++c) o[c] = 0.0f;
        return;
    }
    const float p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    const SampleGeo g = sample_geo(p, pmin + 3 * nd, pmax + 3 * nd, f.roi_min, f.roi_max);
    for (int m = 0; m < 3; ++m) {
        const int H = f.plane_h[m], W = f.plane_w[m], L = f.line_len[m];
        const Corner2 k = corners2(g.pu[m], g.pv[m], H, W);
        const Corner1 l = corners1(g.lu[m], L);
        const float* P = (const float*)f.plane[m] + slot * (int64_t)H * W * C;
        const float* V = (const float*)f.line[m];
        for (int c = 0; c < C; ++c) {
            const float mat = bilerp(k, P[(k.y0 * W + k.x0) * C + c], P[(k.y0 * W + k.x1) * C + c],
                                     P[(k.y1 * W + k.x0) * C + c], P[(k.y1 * W + k.x1) * C + c]);
            const float vec = lerp1(l, V[l.x0 * C + c], V[l.x1 * C + c]);
            const float prod = __fmul_rn(mat, vec);
            if (f.mode)
                o[m * C + c] = prod;
            else
                o[c] = m == 0 ? prod : __fadd_rn(o[c], prod);
        }
    }
}

__global__ void vm_bwd_kernel(atdf_field_t f, const float* __restrict__ pmin, const float* __restrict__ pmax,
                              int64_t num_nodes, const float* __restrict__ pos, const int64_t* __restrict__ node,
                              int64_t S, const float* __restrict__ gout, atdf_field_grad_t gr, int32_t* err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S) return;
    const int C = f.channels;
    const int F = f.mode ? 3 * C : C;
    const int64_t nd = node[i];
    if (nd < 0 || nd >= num_nodes) {
        set_err(err, ATDF_DEVERR_INDEX);
        return;
    }
    const int64_t slot = f.leaf_slot[nd];
    if (slot < 0 || slot >= f.num_slots) return;
    const float p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    const SampleGeo g = sample_geo(p, pmin + 3 * nd, pmax + 3 * nd, f.roi_min, f.roi_max);
    const float* go = gout + i * F;
    for (int m = 0; m < 3; ++m) {
        const int H = f.plane_h[m], W = f.plane_w[m], L = f.line_len[m];
        const Corner2 k = corners2(g.pu[m], g.pv[m], H, W);
        const Corner1 l = corners1(g.lu[m], L);
        const int64_t pbase = slot * (int64_t)H * W * C;
        const float* P = (const float*)f.plane[m] + pbase;
        const float* V = (const float*)f.line[m];
        float* GP = gr.plane[m] ? gr.plane[m] + pbase : nullptr;
        float* GV = gr.line[m];
        for (int c = 0; c < C; ++c) {
            const float gf = f.mode ? go[m * C + c] : go[c];
            const float mat = bilerp(k, P[(k.y0 * W + k.x0) * C + c], P[(k.y0 * W + k.x1) * C + c],
                                     P[(k.y1 * W + k.x0) * C + c], P[(k.y1 * W + k.x1) * C + c]);
            const float vec = lerp1(l, V[l.x0 * C + c], V[l.x1 * C + c]);
            const float gm = __fmul_rn(gf, vec), gv = __fmul_rn(gf, mat);
            if (GP) {
                atomicAdd(&GP[(k.y0 * W + k.x0) * C + c], __fmul_rn(k.w_nw, gm));
                atomicAdd(&GP[(k.y0 * W + k.x1) * C + c], __fmul_rn(k.w_ne, gm));
                atomicAdd(&GP[(k.y1 * W + k.x0) * C + c], __fmul_rn(k.w_sw, gm));
                atomicAdd(&GP[(k.y1 * W + k.x1) * C + c], __fmul_rn(k.w_se, gm));
            }
            if (GV) {
                atomicAdd(&GV[l.x0 * C + c], __fmul_rn(l.w0, gv));
                atomicAdd(&GV[l.x1 * C + c], __fmul_rn(l.w1, gv));
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Decoder MLP, one thread per row (reference-compatible unfused path)
// ---------------------------------------------------------------------------
constexpr int kMlpMaxWidth = 256;

__global__ void mlp_fwd_kernel(atdf_mlp_t m, const float* __restrict__ x, int64_t S, float* __restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S) return;
    float buf[2][kMlpMaxWidth];
    const int in0 = m.dims[0];
    for (int k = 0; k < in0; ++k) buf[0][k] = x[i * in0 + k];
    int cur = 0;
    for (int l = 0; l < m.num_layers; ++l) {
        const int in = m.dims[l], on = m.dims[l + 1];
        const bool last = l == m.num_layers - 1;
        const float* Wl = m.weight[l];
        for (int o = 0; o < on; ++o) {
            float acc = 0.0f;
            for (int k = 0; k < in; ++k) acc = fmaf(buf[cur][k], Wl[o * in + k], acc);
            acc += m.bias[l][o];
            buf[cur ^ 1][o] = act_fwd(last ? m.last_activation : m.hidden_activation, acc, m.softplus_beta);
        }
        cur ^= 1;
    }
    const int on = m.dims[m.num_layers];
    for (int o = 0; o < on; ++o) out[i * on + o] = buf[cur][o];
}

constexpr int kMlpMaxPre = 1024;

__global__ void mlp_bwd_kernel(atdf_mlp_t m, const float* __restrict__ x, int64_t S, const float* __restrict__ gout,
                               float* __restrict__ gx, atdf_mlp_grad_t gr)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S) return;
    float pre[kMlpMaxPre];
    float g[2][kMlpMaxWidth];
    int po[ATDF_MAX_LAYERS + 1];
    po[0] = 0;
    for (int l = 0; l < m.num_layers; ++l) po[l + 1] = po[l] + m.dims[l + 1];
    const int in0 = m.dims[0];
    // forward keeping pre-activations
    for (int l = 0; l < m.num_layers; ++l) {
        const int in = m.dims[l], on = m.dims[l + 1];
        const float* Wl = m.weight[l];
        for (int o = 0; o < on; ++o) {
            float acc = 0.0f;
            for (int k = 0; k < in; ++k) {
                const float xin = l == 0 ? x[i * in0 + k]
                                         : act_fwd(m.hidden_activation, pre[po[l - 1] + k], m.softplus_beta);
                acc = fmaf(xin, Wl[o * in + k], acc);
            }
            pre[po[l] + o] = acc + m.bias[l][o];
        }
    }
    const int L = m.num_layers;
    int cur = 0;
    for (int o = 0; o < m.dims[L]; ++o) g[cur][o] = gout[i * m.dims[L] + o];
    for (int l = L - 1; l >= 0; --l) {
        const int in = m.dims[l], on = m.dims[l + 1];
        const int a = l == L - 1 ? m.last_activation : m.hidden_activation;
        for (int o = 0; o < on; ++o) g[cur][o] *= act_grad(a, pre[po[l] + o], m.softplus_beta);
        const float* Wl = m.weight[l];
        for (int o = 0; o < on; ++o) {
            const float gp = g[cur][o];
            if (gr.bias[l]) atomicAdd(&gr.bias[l][o], gp);
            if (gr.weight[l] && gp != 0.0f) {
                for (int k = 0; k < in; ++k) {
                    const float xin = l == 0 ? x[i * in0 + k]
                                             : act_fwd(m.hidden_activation, pre[po[l - 1] + k], m.softplus_beta);
                    atomicAdd(&gr.weight[l][o * in + k], gp * xin);
                }
            }
        }
        for (int k = 0; k < in; ++k) {
            float acc = 0.0f;
            for (int o = 0; o < on; ++o) acc = fmaf(g[cur][o], Wl[o * in + k], acc);
            g[cur ^ 1][k] = acc;
        }
        cur ^= 1;
    }
    if (gx)
        for (int k = 0; k < in0; ++k) gx[i * in0 + k] = g[cur][k];
}

// ---------------------------------------------------------------------------
// line integral, node-error scoring, MSE loss
// ---------------------------------------------------------------------------
__global__ void integrate_kernel(const float* __restrict__ vals, const float* __restrict__ w,
                                 const int64_t* __restrict__ ray, int64_t S, int C, int64_t R, float* img,
                                 int32_t* err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S) return;
    const int64_t r = ray[i];
    if (r < 0 || r >= R) {
        set_err(err, ATDF_DEVERR_INDEX);
        return;
    }
    const float wi = w[i];
    for (int c = 0; c < C; ++c) atomicAdd(&img[c * R + r], __fmul_rn(vals[i * C + c], wi));
}

__global__ void node_loss_kernel(const float* __restrict__ prl, int C, int64_t R, const int64_t* __restrict__ ray,
                                 const int64_t* __restrict__ node, const float* __restrict__ w, int64_t S,
                                 int64_t num_nodes, double* ls, double* ws, int32_t* err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S) return;
    const int64_t r = ray[i], nd = node[i];
    if (r < 0 || r >= R || nd < 0 || nd >= num_nodes) {
        set_err(err, ATDF_DEVERR_INDEX);
        return;
    }
    double l = 0.0;
    for (int c = 0; c < C; ++c) l += (double)prl[c * R + r];
    l /= (double)C;
    const double wi = (double)w[i];
    atomicAdd(&ls[nd], l * wi);
    atomicAdd(&ws[nd], wi);
}

__global__ void mse_kernel(const float* __restrict__ img, const float* __restrict__ tgt, int64_t n, float scale,
                           double* loss, float* __restrict__ gimg, float* __restrict__ prl)
{
    __shared__ double red[256];
    double acc = 0.0;
    const float gs = scale * 2.0f / (float)n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float d = img[i] - tgt[i];
        acc += (double)d * (double)d;
        if (gimg) gimg[i] = gs * d;
        if (prl) prl[i] = d * d;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0 && loss) atomicAdd(loss, red[0] * (double)scale / (double)n);
}

}  // namespace atdf

using namespace atdf;

static inline unsigned blocks_for(int64_t n, int t = 256) { return (unsigned)div_up(n, t); }

extern "C" {

int atdf_grid_sample2d_forward(const float* grid, int64_t N, int64_t C, int64_t H, int64_t W,
                               const int64_t* s, const int64_t* index, const float* uv, int64_t S, float* out,
                               int32_t* dev_error, atdf_stream_t stream)
{
    if (!grid || !s || N <= 0 || C <= 0 || H <= 0 || W <= 0 || S < 0 || (S > 0 && (!index || !uv || !out)))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (S == 0) return ATDF_OK;
    gs2_fwd_kernel<<<blocks_for(S), 256, 0, (cudaStream_t)stream>>>(grid, N, C, (int)H, (int)W, s[0], s[1], s[2],
                                                                    s[3], index, uv, S, out, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_grid_sample2d_backward(const float* grid, int64_t N, int64_t C, int64_t H, int64_t W, const int64_t* s,
                                const int64_t* index, const float* uv, int64_t S, const float* grad_out,
                                float* grad_grid, float* grad_uv, int32_t* dev_error, atdf_stream_t stream)
{
    if (!grid || !s || N <= 0 || C <= 0 || H <= 0 || W <= 0 || S < 0 || (S > 0 && (!index || !uv || !grad_out)))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (S == 0) return ATDF_OK;
    gs2_bwd_kernel<<<blocks_for(S), 256, 0, (cudaStream_t)stream>>>(grid, N, C, (int)H, (int)W, s[0], s[1], s[2],
                                                                    s[3], index, uv, S, grad_out, grad_grid, grad_uv,
                                                                    dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_grid_sample1d_forward(const float* grid, int64_t N, int64_t C, int64_t W, const int64_t* s,
                               const int64_t* index, const float* uv, int64_t S, float* out, int32_t* dev_error,
                               atdf_stream_t stream)
{
    if (!grid || !s || N <= 0 || C <= 0 || W <= 0 || S < 0 || (S > 0 && (!index || !uv || !out)))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (S == 0) return ATDF_OK;
    gs1_fwd_kernel<<<blocks_for(S), 256, 0, (cudaStream_t)stream>>>(grid, N, C, (int)W, s[0], s[1], s[2], index, uv,
                                                                    S, out, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_grid_sample1d_backward(const float* grid, int64_t N, int64_t C, int64_t W, const int64_t* s,
                                const int64_t* index, const float* uv, int64_t S, const float* grad_out,
                                float* grad_grid, float* grad_uv, int32_t* dev_error, atdf_stream_t stream)
{
    if (!grid || !s || N <= 0 || C <= 0 || W <= 0 || S < 0 || (S > 0 && (!index || !uv || !grad_out)))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (S == 0) return ATDF_OK;
    gs1_bwd_kernel<<<blocks_for(S), 256, 0, (cudaStream_t)stream>>>(grid, N, C, (int)W, s[0], s[1], s[2], index, uv,
                                                                    S, grad_out, grad_grid, grad_uv, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_gradient_correction_backward(const float* ray_direction, const int64_t* ray_index, int64_t num_rays,
                                      const float* grad_in, int64_t S, float* grad_out, int32_t* dev_error,
                                      atdf_stream_t stream)
{
    if (S < 0 || (S > 0 && (!ray_direction || !ray_index || !grad_in || !grad_out))) return ATDF_ERR_INVALID_ARGUMENT;
    if (S == 0) return ATDF_OK;
    gradcorr_bwd_kernel<<<blocks_for(S), 256, 0, (cudaStream_t)stream>>>(ray_direction, ray_index, num_rays, grad_in,
                                                                         S, grad_out, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

static bool field_ok(const atdf_field_t* f)
{
    if (!f || f->channels <= 0 || (f->mode != 0 && f->mode != 1) || !f->leaf_slot) return false;
    for (int m = 0; m < 3; ++m)
        if (!f->plane[m] || !f->line[m] || f->plane_h[m] <= 0 || f->plane_w[m] <= 0 || f->line_len[m] <= 0)
            return false;
    return true;
}

int atdf_vm_features_forward(const atdf_field_t* field, const float* pmin, const float* pmax, int64_t num_nodes,
                             const float* position, const int64_t* node_id, int64_t S, float* out, int32_t* dev_error,
                             atdf_stream_t stream)
{
    if (!field_ok(field) || !pmin || !pmax || S < 0 || (S > 0 && (!position || !node_id || !out)))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (field->dtype != ATDF_F32) return ATDF_ERR_UNSUPPORTED;
    if (S == 0) return ATDF_OK;
    vm_fwd_kernel<<<blocks_for(S, 128), 128, 0, (cudaStream_t)stream>>>(*field, pmin, pmax, num_nodes, position,
                                                                         node_id, S, out, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_vm_features_backward(const atdf_field_t* field, const float* pmin, const float* pmax, int64_t num_nodes,
                              const float* position, const int64_t* node_id, int64_t S, const float* grad_features,
                              const atdf_field_grad_t* grad, int32_t* dev_error, atdf_stream_t stream)
{
    if (!field_ok(field) || !pmin || !pmax || !grad || S < 0 || (S > 0 && (!position || !node_id || !grad_features)))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (field->dtype != ATDF_F32) return ATDF_ERR_UNSUPPORTED;
    if (S == 0) return ATDF_OK;
    vm_bwd_kernel<<<blocks_for(S, 128), 128, 0, (cudaStream_t)stream>>>(*field, pmin, pmax, num_nodes, position,
                                                                         node_id, S, grad_features, *grad, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

static bool mlp_ok(const atdf_mlp_t* m)
{
    if (!m || m->num_layers <= 0 || m->num_layers > ATDF_MAX_LAYERS) return false;
    int total = 0;
    for (int l = 0; l <= m->num_layers; ++l) {
        if (m->dims[l] <= 0 || m->dims[l] > kMlpMaxWidth) return false;
        if (l > 0) total += m->dims[l];
    }
    for (int l = 0; l < m->num_layers; ++l)
        if (!m->weight[l] || !m->bias[l]) return false;
    return total <= kMlpMaxPre;
}

int atdf_mlp_forward(const atdf_mlp_t* mlp, const float* x, int64_t S, float* out, atdf_stream_t stream)
{
    if (!mlp_ok(mlp) || S < 0 || (S > 0 && (!x || !out))) return ATDF_ERR_INVALID_ARGUMENT;
    if (S == 0) return ATDF_OK;
    mlp_fwd_kernel<<<blocks_for(S, 128), 128, 0, (cudaStream_t)stream>>>(*mlp, x, S, out);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_mlp_backward(const atdf_mlp_t* mlp, const float* x, int64_t S, const float* grad_out, float* grad_x,
                      const atdf_mlp_grad_t* grad, atdf_stream_t stream)
{
    if (!mlp_ok(mlp) || !grad || S < 0 || (S > 0 && (!x || !grad_out))) return ATDF_ERR_INVALID_ARGUMENT;
    if (S == 0) return ATDF_OK;
    mlp_bwd_kernel<<<blocks_for(S, 64), 64, 0, (cudaStream_t)stream>>>(*mlp, x, S, grad_out, grad_x, *grad);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_integrate_xray(const float* values, const float* weight, const int64_t* ray_index, int64_t S,
                        int32_t channels, int64_t num_rays, float* image, int32_t* dev_error, atdf_stream_t stream)
{
    if (S < 0 || channels <= 0 || num_rays < 0 || (S > 0 && (!values || !weight || !ray_index || !image)))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (S == 0) return ATDF_OK;
    integrate_kernel<<<blocks_for(S), 256, 0, (cudaStream_t)stream>>>(values, weight, ray_index, S, channels, num_rays,
                                                                      image, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_accumulate_loss_per_node(const float* per_ray_loss, int32_t channels, int64_t num_rays,
                                  const int64_t* ray_index, const int64_t* node_id, const float* weight, int64_t S,
                                  int64_t num_nodes, double* loss_sum, double* weight_sum, int32_t* dev_error,
                                  atdf_stream_t stream)
{
    if (S < 0 || channels <= 0 || !loss_sum || !weight_sum ||
        (S > 0 && (!per_ray_loss || !ray_index || !node_id || !weight)))
        return ATDF_ERR_INVALID_ARGUMENT;
    if (S == 0) return ATDF_OK;
    node_loss_kernel<<<blocks_for(S), 256, 0, (cudaStream_t)stream>>>(per_ray_loss, channels, num_rays, ray_index,
                                                                      node_id, weight, S, num_nodes, loss_sum,
                                                                      weight_sum, dev_error);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

int atdf_mse_loss(const float* image, const float* target, int64_t count, float scale, double* loss,
                  float* grad_image, float* per_ray_loss, atdf_stream_t stream)
{
    if (count < 0 || (count > 0 && (!image || !target))) return ATDF_ERR_INVALID_ARGUMENT;
    if (loss) ATDF_CUDA_TRY(cudaMemsetAsync(loss, 0, sizeof(double), (cudaStream_t)stream));
    if (count == 0) return ATDF_OK;
    const int64_t nb = div_up(count, 256);
    const unsigned blocks = (unsigned)(nb < 1184 ? nb : 1184);
    mse_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(image, target, count, scale, loss, grad_image, per_ray_loss);
    ATDF_LAUNCH_CHECK();
    return ATDF_OK;
}

}  // extern "C"
