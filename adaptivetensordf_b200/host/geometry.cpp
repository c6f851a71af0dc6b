// Operator surface of the projection path over libatdf_b200.so:
// IndirectGridSample2D/1D and GradientCorrection (custom autograd ops of
// hyperacorn/csrc/modules/), IntegrateSamplesXRay, AccumulateSampleLossPerNode,
// DecodeFeatures (hyperacorn/csrc/geometry/geometry.cpp), the VM field of
// GeometryTensorQO (geometry_tensor_qo.cpp:257-390) and the fused projection
// with its hand-written adjoint.
#include <ATen/cuda/CUDAContext.h>
#include <cuda_runtime_api.h>

#include "atdf_host.h"

using torch::Tensor;
using torch::autograd::AutogradContext;
using torch::autograd::tensor_list;

namespace atdf_host {

static cudaStream_t cur_stream() { return at::cuda::getCurrentCUDAStream().stream(); }
static atdf_stream_t stream_arg() { return (atdf_stream_t)cur_stream(); }

#define ATDF_CHECK_CUDA(t) TORCH_CHECK((t).is_cuda(), #t " must be a CUDA tensor (there is no CPU path)")

static Tensor err_word(const torch::Device& dev)
{
    return torch::zeros({1}, torch::TensorOptions().dtype(torch::kInt32).device(dev));
}

int activation_id(const std::string& a)
{
    if (a == "id" || a == "none") return ATDF_ACT_ID;
    if (a == "relu") return ATDF_ACT_RELU;
    if (a == "silu") return ATDF_ACT_SILU;
    if (a == "sigmoid") return ATDF_ACT_SIGMOID;
    if (a == "softplus") return ATDF_ACT_SOFTPLUS;
    if (a == "leakyrelu") return ATDF_ACT_LEAKYRELU;
    if (a == "abs") return ATDF_ACT_ABS;
    if (a == "tanh") return ATDF_ACT_TANH;
    TORCH_CHECK(false, "unknown activation '", a, "'");
    return 0;
}

// ---------------------------------------------------------------------------
// IndirectGridSample2D / 1D (IndirectGridSample2D.cu:408-492,
// IndirectGridSample1D.cu:153-220)
// ---------------------------------------------------------------------------
class GridSample2DFn : public torch::autograd::Function<GridSample2DFn> {
   public:
    static Tensor forward(AutogradContext* ctx, Tensor grid, Tensor index, Tensor uv)
    {
        ATDF_CHECK_CUDA(grid);
        ATDF_CHECK_CUDA(index);
        ATDF_CHECK_CUDA(uv);
        TORCH_CHECK(grid.dim() == 4 && index.dim() == 1 && uv.dim() == 2 && uv.size(1) == 2,
                    "IndirectGridSample2D: grid [N,C,H,W], index [S], uv [S,2]");
        TORCH_CHECK(grid.scalar_type() == torch::kFloat32 && uv.scalar_type() == torch::kFloat32, "float32 required");
        auto idx = index.to(torch::kLong).contiguous();
        auto u = uv.contiguous();
        const int64_t S = idx.size(0), C = grid.size(1);
        auto out = torch::zeros({S, C}, grid.options().memory_format(torch::MemoryFormat::Contiguous));
        int64_t st[4] = {grid.stride(0), grid.stride(1), grid.stride(2), grid.stride(3)};
        auto err = err_word(grid.device());
        check_status(atdf_grid_sample2d_forward(grid.data_ptr<float>(), grid.size(0), C, grid.size(2), grid.size(3), st,
                                                idx.data_ptr<int64_t>(), u.data_ptr<float>(), S, out.data_ptr<float>(),
                                                err.data_ptr<int32_t>(), stream_arg()),
                     "IndirectGridSample2D");
        // data-dependent problems (an index out of range) raise here, as the
        // reference checks for errors after every op (CUDA_SYNC_CHECK_ERROR)
        check_dev_error(err, "IndirectGridSample2D");
        ctx->save_for_backward({grid, idx, u});
        ctx->saved_data["err"] = err;
        return out;
    }
    static tensor_list backward(AutogradContext* ctx, tensor_list go)
    {
        auto s = ctx->get_saved_variables();
        auto grid = s[0], idx = s[1], u = s[2];
        auto g = go[0].contiguous();
        auto ggrid = torch::zeros(grid.sizes(), grid.options().memory_format(torch::MemoryFormat::Contiguous));
        auto guv = torch::zeros_like(u);
        int64_t st[4] = {grid.stride(0), grid.stride(1), grid.stride(2), grid.stride(3)};
        auto err = ctx->saved_data["err"].toTensor();
        check_status(atdf_grid_sample2d_backward(grid.data_ptr<float>(), grid.size(0), grid.size(1), grid.size(2),
                                                 grid.size(3), st, idx.data_ptr<int64_t>(), u.data_ptr<float>(),
                                                 idx.size(0), g.data_ptr<float>(), ggrid.data_ptr<float>(),
                                                 guv.data_ptr<float>(), err.data_ptr<int32_t>(), stream_arg()),
                     "IndirectGridSample2D backward");
        check_dev_error(err, "IndirectGridSample2D backward");
        return {ggrid, Tensor(), guv};
    }
};

class GridSample1DFn : public torch::autograd::Function<GridSample1DFn> {
   public:
    static Tensor forward(AutogradContext* ctx, Tensor grid, Tensor index, Tensor uv)
    {
        ATDF_CHECK_CUDA(grid);
        ATDF_CHECK_CUDA(index);
        ATDF_CHECK_CUDA(uv);
        TORCH_CHECK(grid.dim() == 4 && grid.size(3) == 1 && index.dim() == 1 && uv.dim() == 2 && uv.size(1) == 1,
                    "IndirectGridSample1D: grid [N,C,W,1], index [S], uv [S,1]");
        TORCH_CHECK(grid.scalar_type() == torch::kFloat32 && uv.scalar_type() == torch::kFloat32, "float32 required");
        auto idx = index.to(torch::kLong).contiguous();
        auto u = uv.contiguous();
        const int64_t S = idx.size(0), C = grid.size(1);
        auto out = torch::zeros({S, C}, grid.options().memory_format(torch::MemoryFormat::Contiguous));
        int64_t st[3] = {grid.stride(0), grid.stride(1), grid.stride(2)};
        auto err = err_word(grid.device());
        check_status(atdf_grid_sample1d_forward(grid.data_ptr<float>(), grid.size(0), C, grid.size(2), st,
                                                idx.data_ptr<int64_t>(), u.data_ptr<float>(), S, out.data_ptr<float>(),
                                                err.data_ptr<int32_t>(), stream_arg()),
                     "IndirectGridSample1D");
        check_dev_error(err, "IndirectGridSample1D");
        ctx->save_for_backward({grid, idx, u});
        ctx->saved_data["err"] = err;
        return out;
    }
    static tensor_list backward(AutogradContext* ctx, tensor_list go)
    {
        auto s = ctx->get_saved_variables();
        auto grid = s[0], idx = s[1], u = s[2];
        auto g = go[0].contiguous();
        auto ggrid = torch::zeros(grid.sizes(), grid.options().memory_format(torch::MemoryFormat::Contiguous));
        auto guv = torch::zeros_like(u);
        int64_t st[3] = {grid.stride(0), grid.stride(1), grid.stride(2)};
        auto err = ctx->saved_data["err"].toTensor();
        check_status(atdf_grid_sample1d_backward(grid.data_ptr<float>(), grid.size(0), grid.size(1), grid.size(2), st,
                                                 idx.data_ptr<int64_t>(), u.data_ptr<float>(), idx.size(0),
                                                 g.data_ptr<float>(), ggrid.data_ptr<float>(), guv.data_ptr<float>(),
                                                 err.data_ptr<int32_t>(), stream_arg()),
                     "IndirectGridSample1D backward");
        check_dev_error(err, "IndirectGridSample1D backward");
        return {ggrid, Tensor(), guv};
    }
};

Tensor IndirectGridSample2D(Tensor multi_grid, Tensor index, Tensor uv)
{
    return GridSample2DFn::apply(multi_grid, index, uv);
}
Tensor IndirectGridSample1D(Tensor multi_grid, Tensor index, Tensor uv)
{
    return GridSample1DFn::apply(multi_grid, index, uv);
}

// GradientCorrection (GradientCorrection.cu:63-119): identity forward,
// backward removes the gradient component along the ray.
class GradCorrFn : public torch::autograd::Function<GradCorrFn> {
   public:
    static Tensor forward(AutogradContext* ctx, Tensor pos, Tensor dir, Tensor ray_index)
    {
        ATDF_CHECK_CUDA(pos);
        ctx->save_for_backward({dir.contiguous(), ray_index.to(torch::kLong).contiguous()});
        return pos.clone();
    }
    static tensor_list backward(AutogradContext* ctx, tensor_list go)
    {
        auto s = ctx->get_saved_variables();
        auto g = go[0].contiguous();
        auto out = torch::empty_like(g);
        auto err = err_word(g.device());
        check_status(atdf_gradient_correction_backward(s[0].data_ptr<float>(), s[1].data_ptr<int64_t>(), s[0].size(0),
                                                       g.data_ptr<float>(), g.size(0), out.data_ptr<float>(),
                                                       err.data_ptr<int32_t>(), stream_arg()),
                     "GradientCorrection backward");
        check_dev_error(err, "GradientCorrection backward");
        return {out, Tensor(), Tensor()};
    }
};

Tensor GradientCorrection(Tensor sample_position, Tensor ray_direction, Tensor ray_index)
{
    return GradCorrFn::apply(sample_position, ray_direction, ray_index);
}

// ---------------------------------------------------------------------------
// IntegrateSamplesXRay (geometry.cpp:977-1019)
// ---------------------------------------------------------------------------
class IntegrateFn : public torch::autograd::Function<IntegrateFn> {
   public:
    static Tensor forward(AutogradContext* ctx, Tensor values, Tensor weight, Tensor ray_index, int64_t C, int64_t R)
    {
        ATDF_CHECK_CUDA(values);
        auto v = values.reshape({-1, C}).contiguous();
        auto w = weight.reshape({-1}).contiguous();
        auto r = ray_index.reshape({-1}).to(torch::kLong).contiguous();
        auto img = torch::zeros({C, R}, v.options());
        auto err = err_word(v.device());
        check_status(atdf_integrate_xray(v.data_ptr<float>(), w.data_ptr<float>(), r.data_ptr<int64_t>(), v.size(0),
                                         (int32_t)C, R, img.data_ptr<float>(), err.data_ptr<int32_t>(), stream_arg()),
                     "IntegrateSamplesXRay");
        check_dev_error(err, "IntegrateSamplesXRay");
        ctx->save_for_backward({v, w, r});
        ctx->saved_data["vshape"] = values.sizes().vec();
        ctx->saved_data["wshape"] = weight.sizes().vec();
        return img;
    }
    static tensor_list backward(AutogradContext* ctx, tensor_list go)
    {
        auto s = ctx->get_saved_variables();
        auto v = s[0], w = s[1], r = s[2];
        auto g = go[0].index_select(1, r).t();  // [S, C]
        auto gv = (g * w.unsqueeze(1)).reshape(ctx->saved_data["vshape"].toIntVector());
        auto gw = (g * v).sum(1).reshape(ctx->saved_data["wshape"].toIntVector());
        return {gv, gw, Tensor(), Tensor(), Tensor()};
    }
};

Tensor IntegrateSamplesXRay(Tensor sample_values, Tensor integration_weight, Tensor ray_index, int num_channels,
                            int64_t num_rays)
{
    if (sample_values.numel() == 0)
        return torch::zeros({num_channels, num_rays}, sample_values.options());
    TORCH_CHECK(sample_values.dim() == integration_weight.dim(), "IntegrateSamplesXRay: rank mismatch");
    return IntegrateFn::apply(sample_values, integration_weight, ray_index, num_channels, num_rays);
}

std::pair<Tensor, Tensor> AccumulateSampleLossPerNode(const SampleList& samples, Tensor per_ray_loss, int64_t num_nodes)
{
    ATDF_CHECK_CUDA(per_ray_loss);
    auto prl = per_ray_loss.dim() == 1 ? per_ray_loss.unsqueeze(0) : per_ray_loss;
    prl = prl.to(torch::kFloat32).contiguous();
    auto dopt = prl.options().dtype(torch::kFloat64);
    auto ls = torch::zeros({num_nodes}, dopt), ws = torch::zeros({num_nodes}, dopt);
    auto r = samples.ray_index.reshape({-1}).contiguous();
    auto n = samples.node_id.reshape({-1}).contiguous();
    auto w = samples.weight.reshape({-1}).contiguous();
    auto err = err_word(prl.device());
    check_status(atdf_accumulate_loss_per_node(prl.data_ptr<float>(), (int32_t)prl.size(0), prl.size(1),
                                               r.data_ptr<int64_t>(), n.data_ptr<int64_t>(), w.data_ptr<float>(),
                                               w.size(0), num_nodes, ls.data_ptr<double>(), ws.data_ptr<double>(),
                                               err.data_ptr<int32_t>(), stream_arg()),
                 "AccumulateSampleLossPerNode");
    check_dev_error(err, "AccumulateSampleLossPerNode");
    return {ls, ws};
}

std::tuple<Tensor, Tensor> MseLossAndGrad(Tensor image, Tensor target, double scale)
{
    ATDF_CHECK_CUDA(image);
    auto im = image.contiguous(), tg = target.to(image.device()).reshape(image.sizes()).contiguous();
    auto loss = torch::zeros({}, im.options().dtype(torch::kFloat64));
    auto grad = torch::empty_like(im);
    check_status(atdf_mse_loss(im.data_ptr<float>(), tg.data_ptr<float>(), im.numel(), (float)scale,
                               loss.data_ptr<double>(), grad.data_ptr<float>(), nullptr, stream_arg()),
                 "MseLoss");
    return {loss, grad};
}

Tensor SiddonProject(Tensor volume, Tensor origin, Tensor direction, std::vector<double> box_min,
                     std::vector<double> box_max)
{
    ATDF_CHECK_CUDA(volume);
    TORCH_CHECK(volume.dim() == 3 && volume.scalar_type() == torch::kFloat32, "volume: [nz, ny, nx] float");
    TORCH_CHECK(box_min.size() == 3 && box_max.size() == 3, "box_min / box_max: 3 values each");
    auto v = volume.contiguous();
    auto o = origin.to(v.device()).to(torch::kFloat32).contiguous();
    auto d = direction.to(v.device()).to(torch::kFloat32).contiguous();
    TORCH_CHECK(o.dim() == 2 && o.size(1) == 3 && d.sizes() == o.sizes(), "origin / direction: [R, 3]");
    auto out = torch::empty({o.size(0)}, v.options().dtype(torch::kFloat64));
    check_status(atdf_siddon_project(v.data_ptr<float>(), (int32_t)v.size(2), (int32_t)v.size(1),
                                     (int32_t)v.size(0), box_min.data(), box_max.data(), o.data_ptr<float>(),
                                     d.data_ptr<float>(), o.size(0), out.data_ptr<double>(), stream_arg()),
                 "SiddonProject");
    return out;
}

// ---------------------------------------------------------------------------
// Decoder (FCBlock + DecodeFeatures) through a flat parameter vector
// ---------------------------------------------------------------------------
static std::vector<int64_t> layer_dims(const Decoder& dec)
{
    std::vector<int64_t> dims;
    TORCH_CHECK(!dec.weight.empty() && dec.weight.size() == dec.bias.size() &&
                    (int)dec.weight.size() <= ATDF_MAX_LAYERS,
                "Decoder: 1..8 layers with one bias each");
    dims.push_back(dec.weight[0].size(1));
    for (auto& w : dec.weight) dims.push_back(w.size(0));
    return dims;
}

static Tensor flat_params(const Decoder& dec)
{
    std::vector<Tensor> parts;
    for (size_t l = 0; l < dec.weight.size(); ++l) {
        parts.push_back(dec.weight[l].reshape({-1}));
        parts.push_back(dec.bias[l].reshape({-1}));
    }
    return torch::cat(parts).contiguous();
}

// MLP view whose weights point into the flat vector.
static atdf_mlp_t mlp_view(const std::vector<int64_t>& dims, const float* flat, int act, int last, float beta)
{
    atdf_mlp_t m;
    std::memset(&m, 0, sizeof(m));
    m.num_layers = (int32_t)dims.size() - 1;
    int64_t off = 0;
    for (int l = 0; l <= m.num_layers; ++l) m.dims[l] = (int32_t)dims[l];
    for (int l = 0; l < m.num_layers; ++l) {
        m.weight[l] = flat + off;
        off += dims[l] * dims[l + 1];
        m.bias[l] = flat + off;
        off += dims[l + 1];
    }
    m.hidden_activation = act;
    m.last_activation = last;
    m.softplus_beta = beta;
    return m;
}

static atdf_mlp_grad_t mlp_grad_view(const std::vector<int64_t>& dims, float* flat)
{
    atdf_mlp_grad_t g;
    std::memset(&g, 0, sizeof(g));
    int64_t off = 0;
    for (size_t l = 0; l + 1 < dims.size(); ++l) {
        g.weight[l] = flat + off;
        off += dims[l] * dims[l + 1];
        g.bias[l] = flat + off;
        off += dims[l + 1];
    }
    return g;
}

atdf_mlp_t Decoder::view() const
{
    TORCH_CHECK(false, "Decoder::view: use the flat parameter vector");
    return atdf_mlp_t{};
}

class MlpFn : public torch::autograd::Function<MlpFn> {
   public:
    static Tensor forward(AutogradContext* ctx, Tensor x, Tensor flat, std::vector<int64_t> dims, int64_t act,
                          int64_t last, double beta)
    {
        ATDF_CHECK_CUDA(x);
        auto xc = x.reshape({-1, dims[0]}).contiguous();
        auto m = mlp_view(dims, flat.data_ptr<float>(), (int)act, (int)last, (float)beta);
        auto out = torch::empty({xc.size(0), dims.back()}, xc.options());
        check_status(atdf_mlp_forward(&m, xc.data_ptr<float>(), xc.size(0), out.data_ptr<float>(), stream_arg()),
                     "DecodeFeatures");
        ctx->save_for_backward({xc, flat});
        ctx->saved_data["dims"] = dims;
        ctx->saved_data["act"] = act;
        ctx->saved_data["last"] = last;
        ctx->saved_data["beta"] = beta;
        ctx->saved_data["xshape"] = x.sizes().vec();
        auto oshape = x.sizes().vec();
        oshape.back() = dims.back();
        return out.reshape(oshape);
    }
    static tensor_list backward(AutogradContext* ctx, tensor_list go)
    {
        auto s = ctx->get_saved_variables();
        auto xc = s[0], flat = s[1];
        auto dims = ctx->saved_data["dims"].toIntVector();
        auto m = mlp_view(dims, flat.data_ptr<float>(), (int)ctx->saved_data["act"].toInt(),
                          (int)ctx->saved_data["last"].toInt(), (float)ctx->saved_data["beta"].toDouble());
        auto g = go[0].reshape({-1, dims.back()}).contiguous();
        auto gflat = torch::zeros_like(flat);
        auto gx = torch::empty_like(xc);
        auto gv = mlp_grad_view(dims, gflat.data_ptr<float>());
        check_status(atdf_mlp_backward(&m, xc.data_ptr<float>(), xc.size(0), g.data_ptr<float>(), gx.data_ptr<float>(),
                                       &gv, stream_arg()),
                     "DecodeFeatures backward");
        return {gx.reshape(ctx->saved_data["xshape"].toIntVector()), gflat, Tensor(), Tensor(), Tensor(), Tensor()};
    }
};

Tensor DecodeFeatures(const Decoder& dec, Tensor features)
{
    auto dims = layer_dims(dec);
    return MlpFn::apply(features, flat_params(dec), dims, activation_id(dec.activation),
                        activation_id(dec.last_activation), dec.softplus_beta);
}

// ---------------------------------------------------------------------------
// VM field
// ---------------------------------------------------------------------------
static Tensor channels_last(const Tensor& t)
{
    return t.is_contiguous(torch::MemoryFormat::ChannelsLast) ? t : t.contiguous(torch::MemoryFormat::ChannelsLast);
}

static atdf_field_t field_view(const GeometryTensorQO& g, const std::vector<Tensor>& planes,
                               const std::vector<Tensor>& lines)
{
    atdf_field_t f;
    std::memset(&f, 0, sizeof(f));
    f.channels = (int32_t)planes[0].size(1);
    TORCH_CHECK(g.tensor_op == "add" || g.tensor_op == "cat", "tensor_op must be add or cat");
    f.mode = g.tensor_op == "cat" ? 1 : 0;
    f.dtype = ATDF_F32;
    for (int m = 0; m < 3; ++m) {
        TORCH_CHECK(planes[m].dim() == 4 && planes[m].size(1) == f.channels && planes[m].size(0) == planes[0].size(0),
                    "planes must be [N, C, H, W] with a common N and C");
        TORCH_CHECK(lines[m].dim() == 4 && lines[m].size(1) == f.channels && lines[m].size(3) == 1,
                    "lines must be [1, C, L, 1]");
        TORCH_CHECK(planes[m].scalar_type() == torch::kFloat32 && lines[m].scalar_type() == torch::kFloat32,
                    "planes / lines must be float32");
        TORCH_CHECK(planes[m].is_contiguous(torch::MemoryFormat::ChannelsLast) &&
                        lines[m].is_contiguous(torch::MemoryFormat::ChannelsLast),
                    "planes / lines must be channels-last");
        f.plane[m] = planes[m].data_ptr<float>();
        f.plane_h[m] = (int32_t)planes[m].size(2);
        f.plane_w[m] = (int32_t)planes[m].size(3);
        f.line[m] = lines[m].data_ptr<float>();
        f.line_len[m] = (int32_t)lines[m].size(2);
        f.roi_min[m] = (float)g.roi_min[m];
        f.roi_max[m] = (float)g.roi_max[m];
    }
    TORCH_CHECK(g.leaf_slot.defined() && g.leaf_slot.is_cuda() && g.leaf_slot.scalar_type() == torch::kLong &&
                    g.leaf_slot.is_contiguous(),
                "leaf_slot must be a contiguous CUDA long tensor");
    f.leaf_slot = g.leaf_slot.data_ptr<int64_t>();
    f.num_slots = planes[0].size(0);
    return f;
}

void GeometryTensorQO::RefreshLowPrecision()
{
    torch::NoGradGuard ng;
    bool fresh = planes_bf16.size() != 3 || lines_bf16.size() != 3;
    for (int m = 0; m < 3 && !fresh; ++m)
        fresh = planes_bf16[m].sizes() != planes[m].sizes() || lines_bf16[m].sizes() != lines[m].sizes();
    if (fresh) {
        planes_bf16.clear();
        lines_bf16.clear();
    }
    for (int m = 0; m < 3; ++m) {
        if (fresh) {
            planes_bf16.push_back(torch::empty(planes[m].sizes(), planes[m].options().dtype(torch::kBFloat16))
                                      .contiguous(torch::MemoryFormat::ChannelsLast));
            lines_bf16.push_back(torch::empty(lines[m].sizes(), lines[m].options().dtype(torch::kBFloat16))
                                     .contiguous(torch::MemoryFormat::ChannelsLast));
        }
        planes_bf16[m].copy_(planes[m]);
        lines_bf16[m].copy_(lines[m]);
    }
}

Tensor GeometryTensorQO::error_word(const torch::Device& dev)
{
    if (!fused_error.defined() || fused_error.device() != dev) fused_error = err_word(dev);
    return fused_error;
}

void GeometryTensorQO::CheckErrors()
{
    if (!fused_error.defined()) return;
    auto e = fused_error.clone();
    fused_error.zero_();
    check_dev_error(e, "ProjectRays");
}

// Field view over the BF16 working copies (the shapes are the FP32 ones).
static atdf_field_t field_view_bf16(const GeometryTensorQO& g, const std::vector<Tensor>& planes32)
{
    TORCH_CHECK(g.planes_bf16.size() == 3 && g.lines_bf16.size() == 3,
                "precision bf16: call RefreshLowPrecision() after creating or updating the parameters");
    atdf_field_t f;
    std::memset(&f, 0, sizeof(f));
    f.channels = (int32_t)planes32[0].size(1);
    f.mode = g.tensor_op == "cat" ? 1 : 0;
    f.dtype = ATDF_BF16;
    for (int m = 0; m < 3; ++m) {
        const auto& p = g.planes_bf16[m];
        const auto& l = g.lines_bf16[m];
        TORCH_CHECK(p.sizes() == planes32[m].sizes() && p.is_contiguous(torch::MemoryFormat::ChannelsLast) &&
                        l.is_contiguous(torch::MemoryFormat::ChannelsLast) && p.scalar_type() == torch::kBFloat16,
                    "BF16 working copies out of date: call RefreshLowPrecision()");
        f.plane[m] = p.data_ptr();
        f.plane_h[m] = (int32_t)p.size(2);
        f.plane_w[m] = (int32_t)p.size(3);
        f.line[m] = l.data_ptr();
        f.line_len[m] = (int32_t)l.size(2);
        f.roi_min[m] = (float)g.roi_min[m];
        f.roi_max[m] = (float)g.roi_max[m];
    }
    f.leaf_slot = g.leaf_slot.data_ptr<int64_t>();
    f.num_slots = planes32[0].size(0);
    return f;
}

static atdf_field_t fused_field_view(const GeometryTensorQO& g, const std::vector<Tensor>& planes,
                                     const std::vector<Tensor>& lines);

atdf_field_t GeometryTensorQO::view() const
{
    std::vector<Tensor> p, l;
    for (int m = 0; m < 3; ++m) {
        p.push_back(channels_last(planes[m]));
        l.push_back(channels_last(lines[m]));
    }
    return field_view(*this, p, l);
}

static atdf_field_grad_t field_grad_view(std::vector<Tensor>& gp, std::vector<Tensor>& gl)
{
    atdf_field_grad_t g;
    for (int m = 0; m < 3; ++m) {
        g.plane[m] = gp[m].data_ptr<float>();
        g.line[m] = gl[m].data_ptr<float>();
    }
    return g;
}

class VmFeatureFn : public torch::autograd::Function<VmFeatureFn> {
   public:
    static Tensor forward(AutogradContext* ctx, Tensor pos, Tensor node, Tensor p0, Tensor p1, Tensor p2, Tensor l0,
                          Tensor l1, Tensor l2, int64_t geo_ptr, int64_t tree_ptr)
    {
        auto* geo = reinterpret_cast<GeometryTensorQO*>(geo_ptr);
        auto* tree = reinterpret_cast<HyperTreeBase*>(tree_ptr);
        std::vector<Tensor> P{p0, p1, p2}, L{l0, l1, l2};
        auto f = field_view(*geo, P, L);
        auto pc = pos.contiguous(), nc = node.to(torch::kLong).contiguous();
        const int64_t S = nc.size(0);
        const int F = f.mode ? 3 * f.channels : f.channels;
        auto out = torch::empty({S, F}, pc.options());
        auto err = err_word(pc.device());
        check_status(atdf_vm_features_forward(&f, tree->node_position_min.data_ptr<float>(),
                                              tree->node_position_max.data_ptr<float>(), tree->NumNodes(),
                                              pc.data_ptr<float>(), nc.data_ptr<int64_t>(), S, out.data_ptr<float>(),
                                              err.data_ptr<int32_t>(), stream_arg()),
                     "SampleVolumeIndirect_feature");
        check_dev_error(err, "SampleVolumeIndirect_feature");
        ctx->save_for_backward({pc, nc, p0, p1, p2, l0, l1, l2});
        ctx->saved_data["geo"] = geo_ptr;
        ctx->saved_data["tree"] = tree_ptr;
        return out;
    }
    static tensor_list backward(AutogradContext* ctx, tensor_list go)
    {
        auto s = ctx->get_saved_variables();
        auto* geo = reinterpret_cast<GeometryTensorQO*>(ctx->saved_data["geo"].toInt());
        auto* tree = reinterpret_cast<HyperTreeBase*>(ctx->saved_data["tree"].toInt());
        std::vector<Tensor> P{s[2], s[3], s[4]}, L{s[5], s[6], s[7]};
        auto f = field_view(*geo, P, L);
        std::vector<Tensor> gp, gl;
        for (int m = 0; m < 3; ++m) {
            gp.push_back(torch::zeros_like(P[m]));  // keeps channels-last strides
            gl.push_back(torch::zeros_like(L[m]));
        }
        auto gv = field_grad_view(gp, gl);
        auto g = go[0].contiguous();
        auto err = err_word(g.device());
        check_status(atdf_vm_features_backward(&f, tree->node_position_min.data_ptr<float>(),
                                               tree->node_position_max.data_ptr<float>(), tree->NumNodes(),
                                               s[0].data_ptr<float>(), s[1].data_ptr<int64_t>(), s[1].size(0),
                                               g.data_ptr<float>(), &gv, err.data_ptr<int32_t>(), stream_arg()),
                     "SampleVolumeIndirect_feature backward");
        check_dev_error(err, "SampleVolumeIndirect_feature backward");
        return {Tensor(), Tensor(), gp[0], gp[1], gp[2], gl[0], gl[1], gl[2], Tensor(), Tensor()};
    }
};

Tensor GeometryTensorQO::SampleVolumeIndirect_feature(HyperTreeBase& tree, Tensor global_coordinate, Tensor node_id)
{
    if (global_coordinate.numel() == 0) return global_coordinate;
    ATDF_CHECK_CUDA(global_coordinate);
    std::vector<Tensor> P, L;
    for (int m = 0; m < 3; ++m) {
        P.push_back(channels_last(planes[m]));
        L.push_back(channels_last(lines[m]));
    }
    return VmFeatureFn::apply(global_coordinate.reshape({-1, 3}), node_id.reshape({-1}), P[0], P[1], P[2], L[0], L[1],
                              L[2], reinterpret_cast<int64_t>(this), reinterpret_cast<int64_t>(&tree));
}

Tensor GeometryTensorQO::SampleVolumeIndirect(HyperTreeBase& tree, Tensor global_coordinate, Tensor node_id)
{
    if (global_coordinate.numel() == 0) return global_coordinate;
    auto feat = SampleVolumeIndirect_feature(tree, global_coordinate, node_id);
    return DecodeFeatures(decoder, feat).contiguous();
}

std::tuple<Tensor, Tensor, Tensor> GeometryTensorQO::ComputeImage(HyperTreeBase& tree, const SampleList& samples,
                                                                  int num_channels, int64_t num_pixels,
                                                                  bool use_decoder)
{
    (void)use_decoder;
    auto out = SampleVolumeIndirect(tree, samples.global_coordinate, samples.node_id);
    auto image = IntegrateSamplesXRay(out, samples.weight.unsqueeze(1), samples.ray_index, num_channels, num_pixels);
    return {image, Tensor(), Tensor()};
}

static atdf_field_t fused_field_view(const GeometryTensorQO& g, const std::vector<Tensor>& planes,
                                     const std::vector<Tensor>& lines)
{
    if (g.precision == "bf16") return field_view_bf16(g, planes);
    TORCH_CHECK(g.precision == "fp32", "precision must be fp32 or bf16");
    return field_view(g, planes, lines);
}

// ---------------------------------------------------------------------------
// Fused projection with the hand-written adjoint
// ---------------------------------------------------------------------------
struct ProjectArgs {
    GeometryTensorQO* geo;
    HyperTreeBase* tree;
    int M;
    uint64_t seed;
    Tensor bins;    // uniform samples: also bin rho * w per segment (optional)
    Tensor ws;      // workspace to use (required with placed samples)
    Tensor xt, xw;  // caller-placed samples: t and weight per sample
    bool segmented = false;  // ws already holds the uniform segments of these rays (atdf_project_segments)
    Tensor err;              // device error word to use (optional)
};

class ProjectFn : public torch::autograd::Function<ProjectFn> {
   public:
    static Tensor forward(AutogradContext* ctx, Tensor origin, Tensor dir, Tensor p0, Tensor p1, Tensor p2, Tensor l0,
                          Tensor l1, Tensor l2, Tensor flat, int64_t args_ptr)
    {
        auto* a = reinterpret_cast<ProjectArgs*>(args_ptr);
        std::vector<Tensor> P{p0, p1, p2}, L{l0, l1, l2};
        auto f = fused_field_view(*a->geo, P, L);
        auto dims = layer_dims(a->geo->decoder);
        const int act = activation_id(a->geo->decoder.activation), last = activation_id(a->geo->decoder.last_activation);
        const float beta = (float)a->geo->decoder.softplus_beta;
        auto m = mlp_view(dims, flat.data_ptr<float>(), act, last, beta);
        auto t = a->tree->view();
        auto o = origin.contiguous(), d = dir.contiguous();
        const int64_t R = o.size(0);
        size_t bytes = 0;
        check_status(atdf_project_workspace_size(R, t.max_depth, t.ns, f.num_slots, (int32_t)dims.back(), &bytes),
                     "atdf_project_workspace_size");
        const bool placed = a->xt.defined();
        TORCH_CHECK(!placed || a->ws.defined(), "ProjectRays: placed samples need their workspace");
        auto ws = a->ws.defined() ? a->ws : torch::empty({(int64_t)bytes}, o.options().dtype(torch::kUInt8));
        TORCH_CHECK((size_t)ws.numel() >= bytes, "ProjectRays: workspace too small");
        auto img = torch::empty({dims.back(), R}, o.options());
        auto err = a->err.defined() ? a->err : a->geo->error_word(o.device());
        if (placed) {
            check_status(atdf_project_forward_samples(&t, &f, &m, o.data_ptr<float>(), d.data_ptr<float>(), R,
                                                      a->xt.data_ptr<float>(), a->xw.data_ptr<float>(),
                                                      img.data_ptr<float>(), ws.data_ptr(), (size_t)ws.numel(),
                                                      err.data_ptr<int32_t>(), stream_arg()),
                         "ProjectRays forward (placed samples)");
            ctx->saved_data["xt"] = a->xt;
            ctx->saved_data["xw"] = a->xw;
        } else if (a->bins.defined()) {
            check_status(atdf_project_forward_binned(&t, &f, &m, o.data_ptr<float>(), d.data_ptr<float>(), R, a->M,
                                                     a->seed, img.data_ptr<float>(), a->bins.data_ptr<float>(),
                                                     ws.data_ptr(), (size_t)ws.numel(), err.data_ptr<int32_t>(),
                                                     stream_arg()),
                         "ProjectRays forward (binned)");
        } else if (a->segmented) {
            check_status(atdf_project_forward_segmented(&t, &f, &m, o.data_ptr<float>(), d.data_ptr<float>(), R,
                                                        a->seed, img.data_ptr<float>(), ws.data_ptr(),
                                                        (size_t)ws.numel(), err.data_ptr<int32_t>(), stream_arg()),
                         "ProjectRays forward (segmented)");
        } else {
            check_status(atdf_project_forward(&t, &f, &m, o.data_ptr<float>(), d.data_ptr<float>(), R, a->M, a->seed,
                                              img.data_ptr<float>(), ws.data_ptr(), (size_t)ws.numel(),
                                              err.data_ptr<int32_t>(), stream_arg()),
                         "ProjectRays forward");
        }
        ctx->save_for_backward({o, d, p0, p1, p2, l0, l1, l2, flat});
        ctx->saved_data["ws"] = ws;
        ctx->saved_data["err"] = err;
        ctx->saved_data["M"] = (int64_t)a->M;
        ctx->saved_data["seed"] = (int64_t)a->seed;
        ctx->saved_data["geo"] = reinterpret_cast<int64_t>(a->geo);
        ctx->saved_data["tree"] = reinterpret_cast<int64_t>(a->tree);
        return img;
    }
    static tensor_list backward(AutogradContext* ctx, tensor_list go)
    {
        auto s = ctx->get_saved_variables();
        auto* geo = reinterpret_cast<GeometryTensorQO*>(ctx->saved_data["geo"].toInt());
        auto* tree = reinterpret_cast<HyperTreeBase*>(ctx->saved_data["tree"].toInt());
        std::vector<Tensor> P{s[2], s[3], s[4]}, L{s[5], s[6], s[7]};
        auto flat = s[8];
        auto f = fused_field_view(*geo, P, L);
        auto dims = layer_dims(geo->decoder);
        auto m = mlp_view(dims, flat.data_ptr<float>(), activation_id(geo->decoder.activation),
                          activation_id(geo->decoder.last_activation), (float)geo->decoder.softplus_beta);
        auto t = tree->view();
        auto ws = ctx->saved_data["ws"].toTensor();
        auto err = ctx->saved_data["err"].toTensor();
        std::vector<Tensor> gp, gl;
        for (int k = 0; k < 3; ++k) {
            gp.push_back(torch::empty_like(P[k]));
            gl.push_back(torch::empty_like(L[k]));
        }
        auto gfv = field_grad_view(gp, gl);
        auto gflat = torch::empty_like(flat);
        auto gmv = mlp_grad_view(dims, gflat.data_ptr<float>());
        auto gi = go[0].contiguous();
        if (ctx->saved_data.count("xt")) {
            auto xt = ctx->saved_data["xt"].toTensor(), xw = ctx->saved_data["xw"].toTensor();
            check_status(atdf_project_backward_samples(&t, &f, &m, s[0].data_ptr<float>(), s[1].data_ptr<float>(),
                                                       s[0].size(0), xt.data_ptr<float>(), xw.data_ptr<float>(),
                                                       gi.data_ptr<float>(), &gfv, &gmv, ws.data_ptr(),
                                                       (size_t)ws.numel(), err.data_ptr<int32_t>(), stream_arg()),
                         "ProjectRays backward (placed samples)");
        } else {
            check_status(atdf_project_backward(&t, &f, &m, s[0].data_ptr<float>(), s[1].data_ptr<float>(),
                                               s[0].size(0), (int32_t)ctx->saved_data["M"].toInt(),
                                               (uint64_t)ctx->saved_data["seed"].toInt(), gi.data_ptr<float>(), &gfv,
                                               &gmv, ws.data_ptr(), (size_t)ws.numel(), err.data_ptr<int32_t>(),
                                               stream_arg()),
                         "ProjectRays backward");
        }
        return {Tensor(), Tensor(), gp[0], gp[1], gp[2], gl[0], gl[1], gl[2], gflat, Tensor()};
    }
};

// The forward reads args only while it runs; the backward uses saved data.
// The current stream waits for the last parameter update (params_ready).
static void wait_params(const GeometryTensorQO& geo)
{
    if (geo.params_ready == 0) return;
    TORCH_CHECK(cudaStreamWaitEvent(cur_stream(), reinterpret_cast<cudaEvent_t>(geo.params_ready), 0) == cudaSuccess,
                "waiting for params_ready failed");
}

static Tensor project_apply(GeometryTensorQO& geo, ProjectArgs& args, const RayList& rays)
{
    ATDF_CHECK_CUDA(rays.origin);
    if (geo.params_ready != 0 && !args.ws.defined() && !args.bins.defined()) {
        // segments first (rays and tree only), then wait for the parameters
        auto t = args.tree->view();
        auto o = rays.origin.contiguous(), d = rays.direction.contiguous();
        const int64_t R = o.size(0), slots = geo.planes[0].size(0);
        size_t bytes = 0;
        check_status(atdf_project_workspace_size(R, t.max_depth, t.ns, slots, 1, &bytes),
                     "atdf_project_workspace_size");
        args.ws = torch::empty({(int64_t)bytes}, o.options().dtype(torch::kUInt8));
        args.err = geo.error_word(o.device());
        atdf_segments_t view;
        check_status(atdf_project_segments(&t, o.data_ptr<float>(), d.data_ptr<float>(), R, args.M, slots,
                                           args.ws.data_ptr(), bytes, &view, args.err.data_ptr<int32_t>(),
                                           stream_arg()),
                     "ProjectRays segments");
        args.segmented = true;
    }
    wait_params(geo);
    std::vector<Tensor> P, L;
    for (int m = 0; m < 3; ++m) {
        P.push_back(channels_last(geo.planes[m]));
        L.push_back(channels_last(geo.lines[m]));
    }
    return ProjectFn::apply(rays.origin, rays.direction, P[0], P[1], P[2], L[0], L[1], L[2], flat_params(geo.decoder),
                            reinterpret_cast<int64_t>(&args));
}

Tensor GeometryTensorQO::ProjectRays(HyperTreeBase& tree, const RayList& rays, int max_samples_per_node,
                                     uint64_t jitter_seed)
{
    ProjectArgs args{this, &tree, max_samples_per_node, jitter_seed, {}, {}, {}, {}};
    return project_apply(*this, args, rays);
}

std::tuple<Tensor, Tensor, Tensor> GeometryTensorQO::ProjectNodeError(HyperTreeBase& tree, const RayList& rays,
                                                                      int max_samples_per_node, uint64_t jitter_seed,
                                                                      Tensor target)
{
    torch::NoGradGuard ng;
    ATDF_CHECK_CUDA(rays.origin);
    wait_params(*this);
    std::vector<Tensor> P, L;
    for (int m = 0; m < 3; ++m) {
        P.push_back(channels_last(planes[m]));
        L.push_back(channels_last(lines[m]));
    }
    auto f = fused_field_view(*this, P, L);
    auto dims = layer_dims(decoder);
    auto flat = flat_params(decoder);
    auto m = mlp_view(dims, flat.data_ptr<float>(), activation_id(decoder.activation),
                      activation_id(decoder.last_activation), (float)decoder.softplus_beta);
    auto t = tree.view();
    auto o = rays.origin.contiguous(), d = rays.direction.contiguous();
    const int64_t R = o.size(0);
    size_t bytes = 0;
    check_status(atdf_project_workspace_size(R, t.max_depth, t.ns, f.num_slots, (int32_t)dims.back(), &bytes),
                 "atdf_project_workspace_size");
    auto ws = torch::empty({(int64_t)bytes}, o.options().dtype(torch::kUInt8));
    auto img = torch::empty({dims.back(), R}, o.options());
    auto err = err_word(o.device());
    check_status(atdf_project_forward(&t, &f, &m, o.data_ptr<float>(), d.data_ptr<float>(), R, max_samples_per_node,
                                      jitter_seed, img.data_ptr<float>(), ws.data_ptr(), bytes,
                                      err.data_ptr<int32_t>(), stream_arg()),
                 "ProjectNodeError forward");
    auto tg = target.to(img.device()).reshape(img.sizes()).to(torch::kFloat32).contiguous();
    auto prl = torch::empty_like(img);
    check_status(atdf_mse_loss(img.data_ptr<float>(), tg.data_ptr<float>(), img.numel(), 1.0f, nullptr, nullptr,
                               prl.data_ptr<float>(), stream_arg()),
                 "per-ray loss");
    auto dopt = o.options().dtype(torch::kFloat64);
    auto ls = torch::empty({tree.NumNodes()}, dopt), wsum = torch::empty({tree.NumNodes()}, dopt);
    check_status(atdf_project_node_error(&t, o.data_ptr<float>(), d.data_ptr<float>(), R, max_samples_per_node,
                                         jitter_seed, prl.data_ptr<float>(), (int32_t)dims.back(),
                                         ls.data_ptr<double>(), wsum.data_ptr<double>(), ws.data_ptr(), bytes,
                                         err.data_ptr<int32_t>(), stream_arg()),
                 "ProjectNodeError");
    check_dev_error(err, "ProjectNodeError");
    return {img, ls, wsum};
}

// ---------------------------------------------------------------------------
// Learned proposal sampler
// ---------------------------------------------------------------------------
static std::vector<int64_t> proposal_dims(const std::vector<Tensor>& weight)
{
    std::vector<int64_t> dims{weight[0].size(1)};
    for (auto& w : weight) dims.push_back(w.size(0));
    return dims;
}

static Tensor proposal_flat(const std::vector<Tensor>& weight, const std::vector<Tensor>& bias)
{
    std::vector<Tensor> parts;
    for (size_t l = 0; l < weight.size(); ++l) {
        parts.push_back(weight[l].detach().reshape({-1}));
        parts.push_back(bias[l].detach().reshape({-1}));
    }
    return torch::cat(parts).contiguous();
}

ProposalSampler::ProposalSampler(int64_t num_nodes, int64_t hidden, int64_t hidden_layers, int64_t seed,
                                 const std::string& device)
{
    TORCH_CHECK(hidden == 64 && hidden_layers >= 1 && hidden_layers <= 3,
                "ProposalSampler: hidden width 64 with 1..3 hidden layers");
    auto gen = at::make_generator<at::CPUGeneratorImpl>((uint64_t)seed);
    std::vector<int64_t> dims{ATDF_PROPOSAL_INPUTS};
    for (int64_t l = 0; l < hidden_layers; ++l) dims.push_back(hidden);
    dims.push_back(ATDF_PROPOSAL_OUTPUTS);
    auto opt = torch::TensorOptions().dtype(torch::kFloat32);
    for (size_t l = 0; l + 1 < dims.size(); ++l) {
        // torch Linear-style init: Kaiming-normal weights (fan_in), uniform bias
        auto w = at::normal(0.0, std::sqrt(2.0 / (double)dims[l]), {dims[l + 1], dims[l]}, gen, opt);
        const double bound = 1.0 / std::sqrt((double)dims[l]);
        auto b = at::empty({dims[l + 1]}, opt).uniform_(-bound, bound, gen);
        if (l + 2 == dims.size()) w.mul_(0.1);  // start near the uniform proposal
        weight.push_back(w.to(torch::Device(device)).set_requires_grad(true));
        bias.push_back(b.to(torch::Device(device)).set_requires_grad(true));
    }
    occupancy = torch::zeros({num_nodes, ATDF_PROPOSAL_OCC}, opt.device(torch::Device(device)));
}

bool ProposalSampler::tensor_core_mlp() const
{
    TORCH_CHECK(precision == "fp32" || precision == "bf16", "ProposalSampler.precision: \"fp32\" or \"bf16\"");
    TORCH_CHECK(precision == "fp32" || weight.size() == 4,
                "ProposalSampler: the tensor-core MLP (precision \"bf16\") has 3 hidden layers");
    return precision == "bf16";
}

std::vector<Tensor> ProposalSampler::parameters() const
{
    std::vector<Tensor> p;
    for (size_t l = 0; l < weight.size(); ++l) {
        p.push_back(weight[l]);
        p.push_back(bias[l]);
    }
    return p;
}

Tensor ProposalSampler::logits_for(HyperTreeBase& tree, const atdf_segments_t& view, const RayList& rays,
                                   Tensor* features_out)
{
    auto t = tree.view();
    auto o = rays.origin.contiguous(), d = rays.direction.contiguous();
    const int64_t cap = std::max<int64_t>(view.capacity, 1);
    auto feat = torch::empty({cap, ATDF_PROPOSAL_INPUTS}, o.options());
    auto err = err_word(o.device());
    TORCH_CHECK(occupancy.size(0) == tree.NumNodes(), "ProposalSampler: occupancy has one row per tree node");
    check_status(atdf_proposal_features(&t, &view, o.data_ptr<float>(), d.data_ptr<float>(),
                                        occupancy.data_ptr<float>(), feat.data_ptr<float>(), err.data_ptr<int32_t>(),
                                        stream_arg()),
                 "atdf_proposal_features");
    auto dims = proposal_dims(weight);
    flat_ = proposal_flat(weight, bias);
    auto m = mlp_view(dims, flat_.data_ptr<float>(), ATDF_ACT_SILU, ATDF_ACT_ID, 1.0f);
    auto logits = torch::empty({cap, ATDF_PROPOSAL_OUTPUTS}, o.options());
    if (tensor_core_mlp())
        check_status(atdf_proposal_mlp_forward_bf16(&m, &view, feat.data_ptr<float>(), logits.data_ptr<float>(),
                                                    err.data_ptr<int32_t>(), stream_arg()),
                     "atdf_proposal_mlp_forward_bf16");
    else
        check_status(atdf_proposal_mlp_forward(&m, &view, feat.data_ptr<float>(), logits.data_ptr<float>(),
                                               stream_arg()),
                     "atdf_proposal_mlp_forward");
    err_ = err;
    if (features_out) *features_out = feat;
    return logits;
}

Tensor ProposalSampler::Project(HyperTreeBase& tree, GeometryTensorQO& geo, const RayList& rays, uint64_t jitter_seed)
{
    ATDF_CHECK_CUDA(rays.origin);
    auto t = tree.view();
    auto o = rays.origin.contiguous(), d = rays.direction.contiguous();
    const int64_t R = o.size(0);
    const int64_t slots = geo.planes[0].size(0);
    size_t bytes = 0;
    check_status(atdf_project_workspace_size(R, t.max_depth, t.ns, slots, 1, &bytes), "atdf_project_workspace_size");
    auto ws = torch::empty({(int64_t)bytes}, o.options().dtype(torch::kUInt8));
    auto err = err_word(o.device());
    atdf_segments_t view;
    check_status(atdf_project_segments(&t, o.data_ptr<float>(), d.data_ptr<float>(), R, 1, slots, ws.data_ptr(), bytes,
                                       &view, err.data_ptr<int32_t>(), stream_arg()),
                 "atdf_project_segments");
    auto logits = logits_for(tree, view, rays, nullptr);
    check_status(atdf_proposal_allocate(&view, R, logits.data_ptr<float>(), (int32_t)budget, (float)mass_mix,
                                        (float)mass_power, stream_arg()),
                 "atdf_proposal_allocate");
    // a ray gets at most budget + its segment count samples: no host read needed
    const int64_t cap = R * budget + view.capacity;
    auto xt = torch::empty({std::max<int64_t>(cap, 1)}, o.options());
    auto xw = torch::empty_like(xt);
    check_status(atdf_proposal_samples(&view, logits.data_ptr<float>(), (float)bin_mix, (float)bin_power,
                                       jitter_seed, importance_weights ? ATDF_PROPOSAL_WEIGHTS_IMPORTANCE
                                                                       : ATDF_PROPOSAL_WEIGHTS_VORONOI,
                                       xt.data_ptr<float>(), xw.data_ptr<float>(), cap,
                                       err.data_ptr<int32_t>(), stream_arg()),
                 "atdf_proposal_samples");
    ProjectArgs args{&geo, &tree, 0, 0, {}, ws, xt, xw};
    auto img = project_apply(geo, args, rays);
    if (check_errors) {
        check_dev_error(err, "ProposalSampler::Project");
        check_dev_error(err_, "atdf_proposal_features");
    }
    return img;
}

Tensor ProposalSampler::ProjectUniformBinned(HyperTreeBase& tree, GeometryTensorQO& geo, const RayList& rays,
                                             int max_samples_per_node, uint64_t jitter_seed)
{
    ATDF_CHECK_CUDA(rays.origin);
    auto t = tree.view();
    const int64_t R = rays.origin.size(0);
    const int64_t slots = geo.planes[0].size(0);
    size_t bytes = 0;
    check_status(atdf_project_workspace_size(R, t.max_depth, t.ns, slots, 1, &bytes), "atdf_project_workspace_size");
    auto ws = torch::empty({(int64_t)bytes}, rays.origin.options().dtype(torch::kUInt8));
    atdf_segments_t view;
    check_status(atdf_project_segment_view(R, t.max_depth, slots, ws.data_ptr(), bytes, &view),
                 "atdf_project_segment_view");
    // bins [segment capacity][32], indexed like the workspace's segment arrays
    auto bins = torch::empty({view.capacity, ATDF_PROPOSAL_BINS}, rays.origin.options());
    ProjectArgs args{&geo, &tree, max_samples_per_node, jitter_seed, bins, ws, {}, {}};
    auto img = project_apply(geo, args, rays);
    last_ws_ = ws;
    last_bins_ = bins;
    last_rays_ = RayList{rays.origin.contiguous(), rays.direction.contiguous()};
    last_slots_ = slots;
    return img;
}

Tensor ProposalSampler::ComputeGradients(HyperTreeBase& tree)
{
    TORCH_CHECK(last_ws_.defined(), "ProposalSampler::ComputeGradients: run ProjectUniformBinned first");
    torch::NoGradGuard ng;
    auto t = tree.view();
    const int64_t R = last_rays_.origin.size(0);
    atdf_segments_t view;
    check_status(atdf_project_segment_view(R, t.max_depth, last_slots_, last_ws_.data_ptr(),
                                           (size_t)last_ws_.numel(), &view),
                 "atdf_project_segment_view");
    Tensor feat;
    auto logits = logits_for(tree, view, last_rays_, &feat);
    const int64_t nn = tree.NumNodes();
    auto dopt = last_bins_.options().dtype(torch::kFloat64);
    auto loss = torch::empty({}, dopt);
    auto node_mass = torch::empty({nn, ATDF_PROPOSAL_OCC}, dopt), node_len = torch::empty({nn, ATDF_PROPOSAL_OCC}, dopt);
    auto dlogits = torch::empty_like(logits);
    auto err = err_word(last_ws_.device());
    check_status(atdf_proposal_loss(&view, feat.data_ptr<float>(), last_bins_.data_ptr<float>(),
                                    logits.data_ptr<float>(), (float)mass_weight, dlogits.data_ptr<float>(),
                                    loss.data_ptr<double>(), node_mass.data_ptr<double>(), node_len.data_ptr<double>(),
                                    nn, err.data_ptr<int32_t>(), stream_arg()),
                 "atdf_proposal_loss");
    auto dims = proposal_dims(weight);
    auto m = mlp_view(dims, flat_.data_ptr<float>(), ATDF_ACT_SILU, ATDF_ACT_ID, 1.0f);
    auto gflat = torch::empty_like(flat_);
    auto gm = mlp_grad_view(dims, gflat.data_ptr<float>());
    if (tensor_core_mlp())
        check_status(atdf_proposal_mlp_backward_bf16(&m, &view, feat.data_ptr<float>(), dlogits.data_ptr<float>(), &gm,
                                                     err.data_ptr<int32_t>(), stream_arg()),
                     "atdf_proposal_mlp_backward_bf16");
    else
        check_status(atdf_proposal_mlp_backward(&m, &view, feat.data_ptr<float>(), dlogits.data_ptr<float>(), &gm,
                                                stream_arg()),
                     "atdf_proposal_mlp_backward");
    int64_t off = 0;
    for (size_t l = 0; l < weight.size(); ++l) {
        const int64_t nw = weight[l].numel(), nb = bias[l].numel();
        weight[l].mutable_grad() = gflat.slice(0, off, off + nw).view(weight[l].sizes());
        off += nw;
        bias[l].mutable_grad() = gflat.slice(0, off, off + nb);
        off += nb;
    }
    check_status(atdf_proposal_occupancy(node_mass.data_ptr<double>(), node_len.data_ptr<double>(), nn,
                                         occupancy.data_ptr<float>(), stream_arg()),
                 "atdf_proposal_occupancy");
    if (check_errors) check_dev_error(err, "atdf_proposal_loss");
    return loss;
}

}  // namespace atdf_host
