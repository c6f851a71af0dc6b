// C++ / libtorch host layer over the C ABI of libatdf_b200.so. It keeps the
// reference's operator surface (hyperacorn/csrc/structure/HyperTree.h,
// HelperStructs.h, modules/IndirectGridSample{1D,2D}.h, GradientCorrection.h,
// geometry/geometry.h, geometry_tensor_qo.h, Modules.h): same names, argument
// meaning and tensor shapes. Every entry point requires CUDA tensors and fails
// with a c10::Error otherwise; there is no CPU path.
#pragma once

#include <torch/torch.h>

#include <string>
#include <tuple>
#include <vector>

#include "atdf.h"

namespace atdf_host {

// RayList (HelperStructs.h:103-175): origin / direction [R, 3] float.
struct RayList {
    torch::Tensor origin;
    torch::Tensor direction;
    int64_t size() const { return origin.size(0); }
};

// SampleList (HelperStructs.h:231-297), in canonical order (ray-major, then
// leaf segments by (tmin, node id), then sample index).
struct SampleList {
    int64_t max_samples_per_ray = 0;
    torch::Tensor global_coordinate;   // [S, 3] float
    torch::Tensor ray_t;               // [S] float
    torch::Tensor weight;              // [S] float
    torch::Tensor ray_index;           // [S] long
    torch::Tensor local_index_in_ray;  // [S] long
    torch::Tensor node_id;             // [S] long
    int64_t size() const { return weight.defined() ? weight.size(0) : 0; }
};

// Ray/leaf segments (one entry per ray/leaf hit) in canonical order.
struct SegmentList {
    torch::Tensor ray_seg_offset, ray_sample_offset;  // [R + 1] long
    torch::Tensor node, nsamp, ray, first;            // [G] int
    torch::Tensor tmin, tmax;                         // [G] float
    int64_t num_segments = 0, num_samples = 0, max_samples_per_ray = 0, max_segments_per_ray = 0;
};

// HyperTreeBaseImpl (HyperTree.h:395-561): a complete 2^d-ary tree stored as
// flat tensors (node_position_min/max, node_children, node_active, ...).
class HyperTreeBase {
   public:
    HyperTreeBase(int d, int max_depth);
    void settree(bool use_quad, float y_min, float y_max);
    void SetActive(int depth);
    void UpdateActive();
    void to(torch::Device device);

    int64_t NumNodes() const { return node_position_min.size(0); }
    int64_t NumActiveNodes() const { return active_node_ids.size(0); }
    int D() const { return d; }
    int NS() const { return use_quad_tree ? (1 << (d - 1)) : (1 << d); }

    SegmentList RaySegments(const RayList& rays, int max_samples_per_node);
    SampleList CreateSamplesForRays(const RayList& rays, int max_samples_per_node, bool interval_jitter);
    SampleList CreateSamplesForRaysWithRnd(const RayList& rays, int max_samples_per_node, torch::Tensor rnd,
                                           uint64_t jitter_seed);
    torch::Tensor ComputeLocalSamples(torch::Tensor global_samples, torch::Tensor node_indices);
    std::tuple<torch::Tensor, torch::Tensor> NodeIdForPositionGPU(torch::Tensor global_samples);
    void SetErrorForActiveNodes(torch::Tensor error, const std::string& strategy);
    // Tree structure optimisation (HyperTreeStructureOptimizer.cpp:5-392,
    // an OR-Tools MIP in the reference) solved exactly on the host by dynamic
    // programming over the active-leaf count: split / merge / keep active
    // leaves under a budget of active leaves, costs from node_error and
    // node_max_density. Returns whether the structure changed (then the active
    // set, prefix sums and flags are updated).
    bool OptimizeStructure(int64_t max_active_nodes, double error_merge_factor = 1.1,
                           double error_split_factor = 0.75);

    atdf_tree_t view() const;  // C view (device pointers)

    int d, max_depth;
    bool use_quad_tree = false;
    torch::Tensor node_parent, node_children, node_position_min, node_position_max, node_scale, node_error,
        node_max_density, node_active, node_culled, node_depth, node_active_prefix_sum, active_node_ids,
        node_flags;
};

// Custom ops (modules/IndirectGridSample2D.h:24, IndirectGridSample1D.h:24,
// GradientCorrection.h).
torch::Tensor IndirectGridSample2D(torch::Tensor multi_grid, torch::Tensor index, torch::Tensor uv);
torch::Tensor IndirectGridSample1D(torch::Tensor multi_grid, torch::Tensor index, torch::Tensor uv);
torch::Tensor GradientCorrection(torch::Tensor sample_position, torch::Tensor ray_direction,
                                 torch::Tensor ray_index);

// NeuralGeometry::IntegrateSamplesXRay (geometry.h:269-270): [C, R].
torch::Tensor IntegrateSamplesXRay(torch::Tensor sample_values, torch::Tensor integration_weight,
                                   torch::Tensor ray_index, int num_channels, int64_t num_rays);

// Decoder (FCBlock, Modules.h:23-149, + DecodeFeatures, geometry.cpp:176-253).
struct Decoder {
    std::vector<torch::Tensor> weight, bias;  // weight[l] [out, in]
    std::string activation = "silu";
    std::string last_activation = "softplus";
    double softplus_beta = 2.0;
    atdf_mlp_t view() const;
};
torch::Tensor DecodeFeatures(const Decoder& dec, torch::Tensor features);

// GeometryTensorQO (geometry_tensor_qo.h): VM planes / lines + decoder.
// Planes are parameters of shape [N, C, H, W] (m = yz, xz, xy) kept in
// channels-last memory format; lines [1, C, L, 1] with C innermost.
struct GeometryTensorQO {
    std::vector<torch::Tensor> planes, lines;  // 3 each
    torch::Tensor leaf_slot;                   // [num_nodes] long, -1 outside the ROI
    std::vector<double> roi_min{-1, -1, -1}, roi_max{1, 1, 1};
    std::string tensor_op = "add";
    Decoder decoder;
    // "fp32": the fused path reads the FP32 planes / lines. "bf16": it reads
    // BF16 working copies (planes_bf16 / lines_bf16, refreshed from the FP32
    // parameters by RefreshLowPrecision) and runs the decoder on the tensor
    // cores; gradients still flow to the FP32 parameters.
    std::string precision = "fp32";
    std::vector<torch::Tensor> planes_bf16, lines_bf16;
    // A cudaEvent_t (as an integer; 0 = none) that marks the end of the last
    // parameter update when that update ran on another stream (an optimizer
    // step). ProjectRays then runs the ray/leaf segment pass, which does not
    // read the parameters, before the current stream waits for the event.
    int64_t params_ready = 0;
    void RefreshLowPrecision();
    // Device error word of the fused projection (ProjectRays), accumulated
    // over calls so that the hot path never reads it back. CheckErrors()
    // reads it (one synchronisation), clears it and raises if a kernel set a
    // bit (an index out of range, a capacity exceeded); a training loop calls
    // it where it synchronises anyway (an evaluation).
    torch::Tensor fused_error;
    torch::Tensor error_word(const torch::Device& dev);
    void CheckErrors();

    atdf_field_t view() const;
    torch::Tensor SampleVolumeIndirect_feature(HyperTreeBase& tree, torch::Tensor global_coordinate,
                                               torch::Tensor node_id);
    torch::Tensor SampleVolumeIndirect(HyperTreeBase& tree, torch::Tensor global_coordinate, torch::Tensor node_id);
    // HierarchicalNeuralGeometry::ComputeImage (geometry.h:335, geometry.cpp:
    // 828-914), unfused: (image [C, R], ratio, ratio_inv). As in the
    // reference's indirect-sampling path, ratio and ratio_inv are undefined
    // and use_decoder has no effect (it only steers the batched path).
    std::tuple<torch::Tensor, torch::Tensor, torch::Tensor> ComputeImage(HyperTreeBase& tree,
                                                                         const SampleList& samples, int num_channels,
                                                                         int64_t num_pixels, bool use_decoder = true);
    // Fused forward projection with the hand-written adjoint.
    torch::Tensor ProjectRays(HyperTreeBase& tree, const RayList& rays, int max_samples_per_node,
                              uint64_t jitter_seed);
    // Node-error scoring of a fused forward (FP64 per-node sums).
    std::tuple<torch::Tensor, torch::Tensor, torch::Tensor> ProjectNodeError(HyperTreeBase& tree,
                                                                             const RayList& rays,
                                                                             int max_samples_per_node,
                                                                             uint64_t jitter_seed,
                                                                             torch::Tensor target);
};

// Learned proposal sampler (no counterpart in the reference, which places
// max_samples_per_node uniform samples in every crossed leaf,
// HyperTree.cu:266-514). A small MLP maps each ray/leaf segment (leaf-local
// entry and exit points, the relative length, the leaf's occupancy as a whole
// and per octant) to a 32-bin sample density over the segment and the
// segment's mass; each ray's budget of samples is split by predicted mass and
// drawn by stratified inverse-CDF sampling, weighted by the samples' Voronoi
// cells (the uniform sampler's quadrature) or, with importance_weights, by
// 1 / (n q) (an unbiased estimate of each segment's integral under uniform
// jitter). The network trains online on the bins of rho * w
// of uniform passes (ProjectUniformBinned), which also judge it. No call
// reads device memory back to the host unless check_errors is set.
class ProposalSampler {
   public:
    ProposalSampler(int64_t num_nodes, int64_t hidden, int64_t hidden_layers, int64_t seed, const std::string& device);

    // Projection through proposal-placed samples (autograd over field + decoder).
    torch::Tensor Project(HyperTreeBase& tree, GeometryTensorQO& geo, const RayList& rays, uint64_t jitter_seed);
    // Uniform projection (ProjectRays) that also keeps the per-segment bins
    // of rho * w as the proposal's next training target.
    torch::Tensor ProjectUniformBinned(HyperTreeBase& tree, GeometryTensorQO& geo, const RayList& rays,
                                       int max_samples_per_node, uint64_t jitter_seed);
    // Proposal loss on the last binned pass; sets weight[l].grad() and
    // bias[l].grad() and refreshes the leaf occupancy. Returns the loss
    // (device FP64 scalar).
    torch::Tensor ComputeGradients(HyperTreeBase& tree);
    std::vector<torch::Tensor> parameters() const;

    std::vector<torch::Tensor> weight, bias;  // [out, in] / [out], FP32
    torch::Tensor occupancy;                  // [num_nodes, 9] float: 8 octants + whole leaf
    int64_t budget = 64;
    double mass_mix = 0.25, bin_mix = 0.2, mass_weight = 0.1;
    double mass_power = 0.5, bin_power = 0.5;  // sample density ~ predicted density^power
    bool check_errors = false;  // read the device error words after each call (synchronises)
    bool importance_weights = false;  // sample weights 1 / (n q) instead of Voronoi cells
    // "fp32": the MLP on CUDA cores in FP32; "bf16": on the tensor cores
    // (tcgen05, BF16 operands), 3 hidden layers only
    std::string precision = "fp32";

   private:
    bool tensor_core_mlp() const;
    torch::Tensor logits_for(HyperTreeBase& tree, const atdf_segments_t& view, const RayList& rays,
                             torch::Tensor* features_out);
    torch::Tensor last_ws_, last_bins_, flat_, err_;
    RayList last_rays_;
    int64_t last_slots_ = 0;
};

// AccumulateSampleLossPerNode (geometry.h:326-327) in FP64.
std::pair<torch::Tensor, torch::Tensor> AccumulateSampleLossPerNode(const SampleList& samples,
                                                                    torch::Tensor per_ray_loss, int64_t num_nodes);

// Fused MSE loss + gradient of an image against a target.
std::tuple<torch::Tensor, torch::Tensor> MseLossAndGrad(torch::Tensor image, torch::Tensor target, double scale);

// FP64 Siddon line integrals of a voxel volume [nz, ny, nx] over the box
// [box_min, box_max] (synthetic tilt series; SceneBase.cpp:904-1000 reads
// measured ones instead).
torch::Tensor SiddonProject(torch::Tensor volume, torch::Tensor origin, torch::Tensor direction,
                            std::vector<double> box_min, std::vector<double> box_max);

int activation_id(const std::string& name);
void check_status(int status, const char* what);
void check_dev_error(torch::Tensor err, const char* what);

}  // namespace atdf_host
