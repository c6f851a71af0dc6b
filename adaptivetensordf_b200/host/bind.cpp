// Python bindings of the C++ host layer (used by tests/, bench.py and users
// who drive the path from Python). The C++ API in atdf_host.h is the
// reference-facing surface; this file only exposes it.
#include <torch/extension.h>

#include <optional>

#include "atdf_host.h"

namespace py = pybind11;
using namespace atdf_host;

static RayList make_rays(torch::Tensor origin, torch::Tensor direction)
{
    RayList r;
    r.origin = origin;
    r.direction = direction;
    return r;
}

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m)
{
    m.doc() = "B200 (sm_100a) forward-projection path of the adaptive tensorial density field reconstructor";

    py::class_<RayList>(m, "RayList")
        .def(py::init(&make_rays), py::arg("origin"), py::arg("direction"))
        .def_readwrite("origin", &RayList::origin)
        .def_readwrite("direction", &RayList::direction)
        .def("size", &RayList::size);

    py::class_<SampleList>(m, "SampleList")
        .def(py::init<>())
        .def_readwrite("max_samples_per_ray", &SampleList::max_samples_per_ray)
        .def_readwrite("global_coordinate", &SampleList::global_coordinate)
        .def_readwrite("ray_t", &SampleList::ray_t)
        .def_readwrite("weight", &SampleList::weight)
        .def_readwrite("ray_index", &SampleList::ray_index)
        .def_readwrite("local_index_in_ray", &SampleList::local_index_in_ray)
        .def_readwrite("node_id", &SampleList::node_id)
        .def("size", &SampleList::size);

    py::class_<SegmentList>(m, "SegmentList")
        .def_readonly("ray_seg_offset", &SegmentList::ray_seg_offset)
        .def_readonly("ray_sample_offset", &SegmentList::ray_sample_offset)
        .def_readonly("node", &SegmentList::node)
        .def_readonly("nsamp", &SegmentList::nsamp)
        .def_readonly("ray", &SegmentList::ray)
        .def_readonly("first", &SegmentList::first)
        .def_readonly("tmin", &SegmentList::tmin)
        .def_readonly("tmax", &SegmentList::tmax)
        .def_readonly("num_segments", &SegmentList::num_segments)
        .def_readonly("num_samples", &SegmentList::num_samples)
        .def_readonly("max_samples_per_ray", &SegmentList::max_samples_per_ray)
        .def_readonly("max_segments_per_ray", &SegmentList::max_segments_per_ray);

    py::class_<HyperTreeBase>(m, "HyperTreeBase")
        .def(py::init<int, int>(), py::arg("d"), py::arg("max_depth"))
        .def("settree", &HyperTreeBase::settree, py::arg("use_quad"), py::arg("y_min") = -1.0f,
             py::arg("y_max") = 1.0f)
        .def("SetActive", &HyperTreeBase::SetActive)
        .def("UpdateActive", &HyperTreeBase::UpdateActive)
        .def("to", [](HyperTreeBase& t, const std::string& dev) { t.to(torch::Device(dev)); })
        .def("NumNodes", &HyperTreeBase::NumNodes)
        .def("NumActiveNodes", &HyperTreeBase::NumActiveNodes)
        .def("NS", &HyperTreeBase::NS)
        .def("RaySegments", &HyperTreeBase::RaySegments)
        .def("CreateSamplesForRays", &HyperTreeBase::CreateSamplesForRays, py::arg("rays"),
             py::arg("max_samples_per_node"), py::arg("interval_jitter"))
        .def(
            "CreateSamplesForRaysWithRnd",
            [](HyperTreeBase& t, const RayList& rays, int M, std::optional<torch::Tensor> rnd, uint64_t seed) {
                return t.CreateSamplesForRaysWithRnd(rays, M, rnd ? *rnd : torch::Tensor(), seed);
            },
            py::arg("rays"), py::arg("max_samples_per_node"), py::arg("rnd"), py::arg("jitter_seed") = 0)
        .def("ComputeLocalSamples", &HyperTreeBase::ComputeLocalSamples)
        .def("NodeIdForPositionGPU", &HyperTreeBase::NodeIdForPositionGPU)
        .def("SetErrorForActiveNodes", &HyperTreeBase::SetErrorForActiveNodes)
        .def("OptimizeStructure", &HyperTreeBase::OptimizeStructure, py::arg("max_active_nodes"),
             py::arg("error_merge_factor") = 1.1, py::arg("error_split_factor") = 0.75)
        .def_readonly("max_depth", &HyperTreeBase::max_depth)
        .def_readonly("use_quad_tree", &HyperTreeBase::use_quad_tree)
        .def_readwrite("node_parent", &HyperTreeBase::node_parent)
        .def_readwrite("node_children", &HyperTreeBase::node_children)
        .def_readwrite("node_position_min", &HyperTreeBase::node_position_min)
        .def_readwrite("node_position_max", &HyperTreeBase::node_position_max)
        .def_readwrite("node_scale", &HyperTreeBase::node_scale)
        .def_readwrite("node_error", &HyperTreeBase::node_error)
        .def_readwrite("node_max_density", &HyperTreeBase::node_max_density)
        .def_readwrite("node_active", &HyperTreeBase::node_active)
        .def_readwrite("node_culled", &HyperTreeBase::node_culled)
        .def_readwrite("node_depth", &HyperTreeBase::node_depth)
        .def_readwrite("node_active_prefix_sum", &HyperTreeBase::node_active_prefix_sum)
        .def_readwrite("active_node_ids", &HyperTreeBase::active_node_ids)
        .def_readonly("node_flags", &HyperTreeBase::node_flags);

    py::class_<GeometryTensorQO>(m, "GeometryTensorQO")
        .def(py::init<>())
        .def_readwrite("planes", &GeometryTensorQO::planes)
        .def_readwrite("lines", &GeometryTensorQO::lines)
        .def_readwrite("leaf_slot", &GeometryTensorQO::leaf_slot)
        .def_readwrite("roi_min", &GeometryTensorQO::roi_min)
        .def_readwrite("roi_max", &GeometryTensorQO::roi_max)
        .def_readwrite("tensor_op", &GeometryTensorQO::tensor_op)
        .def_readwrite("precision", &GeometryTensorQO::precision)
        .def_readwrite("params_ready", &GeometryTensorQO::params_ready)
        .def_readonly("planes_bf16", &GeometryTensorQO::planes_bf16)
        .def_readonly("lines_bf16", &GeometryTensorQO::lines_bf16)
        .def("RefreshLowPrecision", &GeometryTensorQO::RefreshLowPrecision)
        .def("CheckErrors", &GeometryTensorQO::CheckErrors)
        .def_property(
            "decoder_weight", [](GeometryTensorQO& g) { return g.decoder.weight; },
            [](GeometryTensorQO& g, std::vector<torch::Tensor> v) { g.decoder.weight = v; })
        .def_property(
            "decoder_bias", [](GeometryTensorQO& g) { return g.decoder.bias; },
            [](GeometryTensorQO& g, std::vector<torch::Tensor> v) { g.decoder.bias = v; })
        .def_property(
            "activation", [](GeometryTensorQO& g) { return g.decoder.activation; },
            [](GeometryTensorQO& g, std::string v) { g.decoder.activation = v; })
        .def_property(
            "last_activation", [](GeometryTensorQO& g) { return g.decoder.last_activation; },
            [](GeometryTensorQO& g, std::string v) { g.decoder.last_activation = v; })
        .def_property(
            "softplus_beta", [](GeometryTensorQO& g) { return g.decoder.softplus_beta; },
            [](GeometryTensorQO& g, double v) { g.decoder.softplus_beta = v; })
        .def("SampleVolumeIndirect_feature", &GeometryTensorQO::SampleVolumeIndirect_feature)
        .def("SampleVolumeIndirect", &GeometryTensorQO::SampleVolumeIndirect)
        .def("ComputeImage", &GeometryTensorQO::ComputeImage, py::arg("tree"), py::arg("samples"),
             py::arg("num_channels"), py::arg("num_pixels"), py::arg("use_decoder") = true)
        .def("ProjectRays", &GeometryTensorQO::ProjectRays, py::arg("tree"), py::arg("rays"),
             py::arg("max_samples_per_node"), py::arg("jitter_seed") = 0)
        .def("ProjectNodeError", &GeometryTensorQO::ProjectNodeError, py::arg("tree"), py::arg("rays"),
             py::arg("max_samples_per_node"), py::arg("jitter_seed"), py::arg("target"));

    py::class_<ProposalSampler>(m, "ProposalSampler")
        .def(py::init<int64_t, int64_t, int64_t, int64_t, const std::string&>(), py::arg("num_nodes"),
             py::arg("hidden") = 64, py::arg("hidden_layers") = 3, py::arg("seed") = 1005,
             py::arg("device") = std::string("cuda"))
        .def("Project", &ProposalSampler::Project, py::arg("tree"), py::arg("geo"), py::arg("rays"),
             py::arg("jitter_seed") = 0)
        .def("ProjectUniformBinned", &ProposalSampler::ProjectUniformBinned, py::arg("tree"), py::arg("geo"),
             py::arg("rays"), py::arg("max_samples_per_node"), py::arg("jitter_seed") = 0)
        .def("ComputeGradients", &ProposalSampler::ComputeGradients, py::arg("tree"))
        .def("parameters", &ProposalSampler::parameters)
        .def_readwrite("weight", &ProposalSampler::weight)
        .def_readwrite("bias", &ProposalSampler::bias)
        .def_readwrite("occupancy", &ProposalSampler::occupancy)
        .def_readwrite("budget", &ProposalSampler::budget)
        .def_readwrite("mass_mix", &ProposalSampler::mass_mix)
        .def_readwrite("bin_mix", &ProposalSampler::bin_mix)
        .def_readwrite("mass_weight", &ProposalSampler::mass_weight)
        .def_readwrite("mass_power", &ProposalSampler::mass_power)
        .def_readwrite("bin_power", &ProposalSampler::bin_power)
        .def_readwrite("importance_weights", &ProposalSampler::importance_weights)
        .def_readwrite("check_errors", &ProposalSampler::check_errors)
        .def_readwrite("precision", &ProposalSampler::precision);

    m.def("IndirectGridSample2D", &IndirectGridSample2D);
    m.def("IndirectGridSample1D", &IndirectGridSample1D);
    m.def("GradientCorrection", &GradientCorrection);
    m.def("IntegrateSamplesXRay", &IntegrateSamplesXRay);
    m.def("AccumulateSampleLossPerNode", &AccumulateSampleLossPerNode);
    m.def("MseLossAndGrad", &MseLossAndGrad);
    m.def("SiddonProject", &SiddonProject, py::arg("volume"), py::arg("origin"), py::arg("direction"),
          py::arg("box_min") = std::vector<double>{-1, -1, -1}, py::arg("box_max") = std::vector<double>{1, 1, 1});
    m.def(
        "DecodeFeatures",
        [](std::vector<torch::Tensor> weight, std::vector<torch::Tensor> bias, std::string act, std::string last,
           double beta, torch::Tensor x) {
            Decoder d;
            d.weight = weight;
            d.bias = bias;
            d.activation = act;
            d.last_activation = last;
            d.softplus_beta = beta;
            return DecodeFeatures(d, x);
        },
        py::arg("weight"), py::arg("bias"), py::arg("activation"), py::arg("last_activation"),
        py::arg("softplus_beta"), py::arg("features"));
    m.def("version", []() { return atdf_version(); });
}
