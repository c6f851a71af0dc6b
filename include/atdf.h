/*
 * atdf.h - C ABI of the B200 (sm_100a) forward-projection library
 * (libatdf_b200.so) for the adaptive tensorial density field reconstructor.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream,
 * launches asynchronously on that stream and returns an atdf_status. Nothing
 * here allocates device memory: callers pass outputs and, where stated, a
 * workspace whose size is queried first. Kernels report data-dependent
 * problems (an index out of range, a capacity overflow) by OR-ing bits into a
 * caller-provided device word (dev_error, see ATDF_DEVERR_*) and skipping the
 * offending access; they never trap.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   hyperacorn/csrc/structure/HyperTree.h:463      CreateSamplesForRays
 *   hyperacorn/csrc/structure/HyperTree.h:432      ComputeLocalSamples
 *   hyperacorn/csrc/structure/HyperTree.h:444      NodeIdForPositionGPU
 *   hyperacorn/csrc/modules/IndirectGridSample2D.h:24  IndirectGridSample2D
 *   hyperacorn/csrc/modules/IndirectGridSample1D.h:24  IndirectGridSample1D
 *   hyperacorn/csrc/modules/GradientCorrection.h       GradientCorrection
 *   hyperacorn/csrc/geometry/geometry_tensor_qo.h:32   SampleVolumeIndirect
 *   hyperacorn/csrc/geometry/Modules.h:23              FCBlock (+ DecodeFeatures)
 *   hyperacorn/csrc/geometry/geometry.h:269-270        IntegrateSamplesXRay
 *   hyperacorn/csrc/geometry/geometry.h:326-327        AccumulateSampleLossPerNode
 *   hyperacorn/csrc/geometry/geometry.h:335            ComputeImage (fused form)
 *   hyperacorn/csrc/modules/ToneMapper.cpp:161-201     PhotometricCalibration (tone mapper)
 */
#ifndef ATDF_H
#define ATDF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same type as cudaStream_t. */
typedef struct CUstream_st* atdf_stream_t;

typedef enum {
    ATDF_OK = 0,
    ATDF_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad size or shape */
    ATDF_ERR_UNSUPPORTED = 2,      /* a configuration this build does not implement */
    ATDF_ERR_WORKSPACE = 3,        /* workspace smaller than the queried size */
    ATDF_ERR_CUDA = 4              /* a CUDA launch failed (cudaGetLastError) */
} atdf_status;

/* Bits OR-ed into *dev_error by kernels. */
#define ATDF_DEVERR_HIT_OVERFLOW 0x1   /* a ray hit more than ATDF_MAX_HITS leaves */
#define ATDF_DEVERR_SEG_CAPACITY 0x2   /* segment output capacity exceeded */
#define ATDF_DEVERR_SAMPLE_CAPACITY 0x4 /* sample output capacity exceeded */
#define ATDF_DEVERR_INDEX 0x8          /* an index outside its array (access skipped) */
#define ATDF_DEVERR_TREE 0x10          /* tree flags did not converge / malformed tree */

/* Largest number of leaves one ray may cross (the reference's limit,
 * HyperTree.cu:280, max_intersections = 256). */
#define ATDF_MAX_HITS 256

#define ATDF_MAX_LAYERS 8

/* Activations (Saiga ActivationFromString names used by FCBlock and
 * DecodeFeatures; softplus uses softplus_beta and torch's threshold 20). */
typedef enum {
    ATDF_ACT_ID = 0,
    ATDF_ACT_RELU = 1,
    ATDF_ACT_SILU = 2,
    ATDF_ACT_SIGMOID = 3,
    ATDF_ACT_SOFTPLUS = 4,
    ATDF_ACT_LEAKYRELU = 5,
    ATDF_ACT_ABS = 6,
    ATDF_ACT_TANH = 7
} atdf_activation;

typedef enum { ATDF_F32 = 0, ATDF_BF16 = 1 } atdf_dtype;

/* HyperTree buffers (HyperTree.h:522-556), device pointers. node_flags comes
 * from atdf_tree_flags: bit 0 = active leaf, bit 1 = subtree holds an active
 * leaf. Children are -1 where absent; a child's box lies inside its parent's
 * (HyperTree.cpp settree), which the ray traversal relies on. */
typedef struct {
    const float* node_position_min; /* [num_nodes, 3] */
    const float* node_position_max; /* [num_nodes, 3] */
    const int32_t* node_children;   /* [num_nodes, ns] */
    const int32_t* node_active;     /* [num_nodes] */
    const uint8_t* node_flags;      /* [num_nodes] */
    int64_t num_nodes;
    int32_t ns; /* 8 (octree) or 4 (quad tree) */
    int32_t max_depth;
} atdf_tree_t;

/* Ray/leaf segments in canonical order: ray-major, and within a ray by
 * (tmin, node id). Segment arrays have `capacity` entries. totals (device,
 * 4 x int64): [0] segments, [1] samples, [2] max samples of one ray,
 * [3] max segments of one ray. */
typedef struct {
    int64_t* ray_seg_offset;    /* [num_rays + 1] */
    int64_t* ray_sample_offset; /* [num_rays + 1] */
    int32_t* node;              /* leaf node id */
    float* tmin;
    float* tmax;
    int32_t* nsamp;             /* samples in the segment */
    int32_t* ray;               /* ray index */
    int32_t* first;             /* index of the first sample within its ray */
    int64_t capacity;
    int64_t* totals;
} atdf_segments_t;

/* Vector-matrix factor field of GeometryTensorQO (geometry_tensor_qo.cpp:
 * 257-380). Planes m = yz, xz, xy are stored channels-last:
 * plane[m][slot][h][w][c] (the reference's [N, C, H, W] with C innermost);
 * lines m = x, y, z are line[m][l][c] (the reference's [1, C, L, 1] with C
 * innermost). leaf_slot maps a node id to its plane slot, -1 outside the ROI
 * (whose features are zero, as in the reference with a ground-truth volume).
 * mode 0 = "add" (F = C features), 1 = "cat" (F = 3C). */
typedef struct {
    int32_t channels;
    int32_t mode;
    int32_t dtype; /* atdf_dtype of planes and lines */
    const void* plane[3];
    int32_t plane_h[3];
    int32_t plane_w[3];
    const void* line[3];
    int32_t line_len[3];
    const int64_t* leaf_slot; /* [num_nodes] */
    int64_t num_slots;
    float roi_min[3];
    float roi_max[3];
} atdf_field_t;

/* FP32 gradients of the field, same channels-last layouts as atdf_field_t. */
typedef struct {
    float* plane[3];
    float* line[3];
} atdf_field_grad_t;

/* Decoder MLP (FCBlock): layers y = act(x W^T + b); the hidden activation
 * follows every layer but the last, the last activation (DecodeFeatures)
 * follows the last. weight[l] is [dims[l+1], dims[l]] (torch Linear). */
typedef struct {
    int32_t num_layers;
    int32_t dims[ATDF_MAX_LAYERS + 1];
    const float* weight[ATDF_MAX_LAYERS];
    const float* bias[ATDF_MAX_LAYERS];
    int32_t hidden_activation;
    int32_t last_activation;
    float softplus_beta;
} atdf_mlp_t;

typedef struct {
    float* weight[ATDF_MAX_LAYERS];
    float* bias[ATDF_MAX_LAYERS];
} atdf_mlp_grad_t;

const char* atdf_status_string(int status);
int atdf_version(void);

/* ---- HyperTree ----------------------------------------------------------
 * node_flags for atdf_tree_t. No reference counterpart (the reference tests
 * every active leaf per ray, HyperTree.cu:320-359); see atdf_ray_segments. */
int atdf_tree_flags(const int32_t* node_active, const int32_t* node_children, int32_t ns, int64_t num_nodes,
                    uint8_t* node_flags, int32_t* dev_error, atdf_stream_t stream);

/* Replaces the intersection half of ComputeRaySamples
 * (hyperacorn/csrc/structure/HyperTree.cu:266-371, launched from
 * CreateSamplesForRays, HyperTree.cu:516-553): all active leaves hit by each
 * ray (IntersectBoxRayPrecise, HyperTree.h:338-380; hits shorter than 1e-5
 * skipped), with n = ceil(|tmax - tmin| / |box diagonal| * max_samples_per_node)
 * samples each. Found by a descent of the tree that tests exactly the leaves
 * the reference tests (a child's box lies inside its parent's). */
int atdf_ray_segments(const atdf_tree_t* tree, const float* ray_origin, const float* ray_direction, int64_t num_rays,
                      int32_t max_samples_per_node, const atdf_segments_t* segs, int32_t* dev_error,
                      atdf_stream_t stream);

/* Replaces the sample half of ComputeRaySamples (HyperTree.cu:434-513) and
 * the position recomputation of CreateSamplesForRays (HyperTree.cu:558-603):
 * writes the SampleList arrays in canonical order. sample_rnd (nullable,
 * [num_samples]) is the interval jitter; without it, jitter_seed != 0 draws
 * it from the hash shared with the fused path, and jitter_seed == 0 uses the
 * midpoint. Outputs have sample_capacity entries. */
int atdf_emit_samples(const atdf_segments_t* segs, int64_t num_rays, const float* ray_origin,
                      const float* ray_direction, const float* sample_rnd, uint64_t jitter_seed, float* out_position,
                      float* out_t, float* out_weight, int64_t* out_ray_index, int64_t* out_local_index,
                      int64_t* out_node_id, int64_t sample_capacity, int32_t* dev_error, atdf_stream_t stream);

/* ComputeLocalSamples (HyperTree.cu:237-259): (x - min) / (max - min) * 2 - 1.
 * group > 1: point i uses node[i / group] (the [G, g, 3] + [G] form). */
int atdf_local_samples(const float* position, const int64_t* node, int64_t num_points, int64_t group,
                       const float* node_position_min, const float* node_position_max, int64_t num_nodes,
                       float* out_local, int32_t* dev_error, atdf_stream_t stream);

/* NodeIdForPositionGPU (HyperTree.cu:1339-1400,1468-1525). */
int atdf_node_id_for_position(const atdf_tree_t* tree, const int64_t* active_node_ids, const float* position,
                              int64_t num_points, int64_t* out_node_id, float* out_mask, int32_t* dev_error,
                              atdf_stream_t stream);

/* ---- gathers (IndirectGridSample2D.cu / IndirectGridSample1D.cu) --------
 * grid is [N, C, H, W] (1D: [N, C, W, 1]) with arbitrary element strides
 * grid_stride = {sN, sC, sH, sW}. align_corners = True, border clamp.
 * Backward ACCUMULATES into grad_grid (contiguous [N, C, H, W]) and grad_uv. */
int atdf_grid_sample2d_forward(const float* grid, int64_t N, int64_t C, int64_t H, int64_t W,
                               const int64_t* grid_stride, const int64_t* index, const float* uv, int64_t num_samples,
                               float* out, int32_t* dev_error, atdf_stream_t stream);
int atdf_grid_sample2d_backward(const float* grid, int64_t N, int64_t C, int64_t H, int64_t W,
                                const int64_t* grid_stride, const int64_t* index, const float* uv,
                                int64_t num_samples, const float* grad_out, float* grad_grid, float* grad_uv,
                                int32_t* dev_error, atdf_stream_t stream);
int atdf_grid_sample1d_forward(const float* grid, int64_t N, int64_t C, int64_t W, const int64_t* grid_stride,
                               const int64_t* index, const float* uv, int64_t num_samples, float* out,
                               int32_t* dev_error, atdf_stream_t stream);
int atdf_grid_sample1d_backward(const float* grid, int64_t N, int64_t C, int64_t W, const int64_t* grid_stride,
                                const int64_t* index, const float* uv, int64_t num_samples, const float* grad_out,
                                float* grad_grid, float* grad_uv, int32_t* dev_error, atdf_stream_t stream);

/* GradientCorrection backward (GradientCorrection.cu:22-48): g - (g.d) d. */
int atdf_gradient_correction_backward(const float* ray_direction, const int64_t* ray_index, int64_t num_rays,
                                      const float* grad_in, int64_t num_samples, float* grad_out, int32_t* dev_error,
                                      atdf_stream_t stream);

/* ---- field / decoder / integral (unfused SampleVolumeIndirect path) ---- */
/* SampleVolumeIndirect_feature (geometry_tensor_qo.cpp:257-380), FP32 field:
 * features [S, F] at sample positions in node ids. */
int atdf_vm_features_forward(const atdf_field_t* field, const float* node_position_min,
                             const float* node_position_max, int64_t num_nodes, const float* position,
                             const int64_t* node_id, int64_t num_samples, float* out_features, int32_t* dev_error,
                             atdf_stream_t stream);
/* Adjoint of the above: ACCUMULATES into grad (FP32, channels-last). */
int atdf_vm_features_backward(const atdf_field_t* field, const float* node_position_min,
                              const float* node_position_max, int64_t num_nodes, const float* position,
                              const int64_t* node_id, int64_t num_samples, const float* grad_features,
                              const atdf_field_grad_t* grad, int32_t* dev_error, atdf_stream_t stream);

/* FCBlock::forward (Modules.h:137) + DecodeFeatures last activation
 * (geometry.cpp:176-253): out [S, dims[num_layers]]. Hidden widths <= 256. */
int atdf_mlp_forward(const atdf_mlp_t* mlp, const float* x, int64_t num_rows, float* out, atdf_stream_t stream);
/* Adjoint: writes grad_x [S, dims[0]] (nullable), ACCUMULATES grad. */
int atdf_mlp_backward(const atdf_mlp_t* mlp, const float* x, int64_t num_rows, const float* grad_out, float* grad_x,
                      const atdf_mlp_grad_t* grad, atdf_stream_t stream);

/* IntegrateSamplesXRay (geometry.cpp:977-1019): ACCUMULATES
 * image[c, ray[s]] += values[s, c] * weight[s]; image is [C, num_rays]. */
int atdf_integrate_xray(const float* values, const float* weight, const int64_t* ray_index, int64_t num_samples,
                        int32_t channels, int64_t num_rays, float* image, int32_t* dev_error, atdf_stream_t stream);

/* AccumulateSampleLossPerNode (geometry.cpp:33-53) in FP64: ACCUMULATES
 * loss_sum[node[s]] += mean_c(per_ray_loss[c, ray[s]]) * weight[s] and
 * weight_sum[node[s]] += weight[s]. */
int atdf_accumulate_loss_per_node(const float* per_ray_loss, int32_t channels, int64_t num_rays,
                                  const int64_t* ray_index, const int64_t* node_id, const float* weight,
                                  int64_t num_samples, int64_t num_nodes, double* loss_sum, double* weight_sum,
                                  int32_t* dev_error, atdf_stream_t stream);

/* ---- fused projection (ComputeImage with CreateSamplesForRays,
 * SampleVolumeIndirect, DecodeFeatures and IntegrateSamplesXRay in one
 * leaf-major pass; geometry.cpp:828-914) -------------------------------- */

/* Workspace for the fused entry points, for num_rays rays through a tree of
 * max_depth with num_slots plane slots. The workspace carries the ray/leaf
 * segments from atdf_project_forward to atdf_project_backward and
 * atdf_project_node_error: pass the same workspace, rays and tree to them. */
int atdf_project_workspace_size(int64_t num_rays, int32_t max_depth, int32_t ns, int64_t num_slots,
                                int32_t out_channels, size_t* bytes);

/* Forward projection image [Cout, num_rays] (Cout = mlp->dims[last]).
 * jitter_seed = 0: midpoint samples; else the interval jitter hash. */
int atdf_project_forward(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                         const float* ray_origin, const float* ray_direction, int64_t num_rays,
                         int32_t max_samples_per_node, uint64_t jitter_seed, float* image, void* workspace,
                         size_t workspace_bytes, int32_t* dev_error, atdf_stream_t stream);

/* atdf_project_forward in two calls: atdf_project_segments (below) first
 * writes the ray/leaf segments and their uniform sample counts into the
 * workspace, then this call projects them. The segment pass reads only the
 * rays and the tree, so a caller can run it while the factors are still
 * being updated (an optimizer step on another stream) and make the stream
 * wait for that update between the two calls. The results equal
 * atdf_project_forward's. */
int atdf_project_forward_segmented(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                                   const float* ray_origin, const float* ray_direction, int64_t num_rays,
                                   uint64_t jitter_seed, float* image, void* workspace, size_t workspace_bytes,
                                   int32_t* dev_error, atdf_stream_t stream);

/* Hand-written adjoint of atdf_project_forward given grad_image [Cout, R]:
 * OVERWRITES grad_field (FP32, channels-last) and grad_mlp. Recomputes every
 * sample (no stored activations); reuses the forward's segments from the
 * workspace. */
int atdf_project_backward(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                          const float* ray_origin, const float* ray_direction, int64_t num_rays,
                          int32_t max_samples_per_node, uint64_t jitter_seed, const float* grad_image,
                          const atdf_field_grad_t* grad_field, const atdf_mlp_grad_t* grad_mlp, void* workspace,
                          size_t workspace_bytes, int32_t* dev_error, atdf_stream_t stream);

/* Mean-squared-error loss of image [Cout, R] against target and its gradient:
 * loss (device double) = scale * mean((image - target)^2), grad_image =
 * scale * 2 (image - target) / (Cout R); per_ray_loss [Cout, R] (nullable)
 * = (image - target)^2 (hyper_train.cpp:1019-1069, MSE branch). */
int atdf_mse_loss(const float* image, const float* target, int64_t count, float scale, double* loss,
                  float* grad_image, float* per_ray_loss, atdf_stream_t stream);

/* Node-error scoring after atdf_project_forward (same workspace): OVERWRITES
 * loss_sum / weight_sum [num_nodes] with the FP64 per-node sums of
 * AccumulateSampleLossPerNode for per_ray_loss [Cout, R]. */
int atdf_project_node_error(const atdf_tree_t* tree, const float* ray_origin, const float* ray_direction,
                            int64_t num_rays, int32_t max_samples_per_node, uint64_t jitter_seed,
                            const float* per_ray_loss, int32_t out_channels, double* loss_sum, double* weight_sum,
                            void* workspace, size_t workspace_bytes, int32_t* dev_error, atdf_stream_t stream);

/* ---- learned proposal sampler --------------------------------------------
 * No counterpart in the reference, which always places max_samples_per_node
 * uniform samples in every crossed leaf (HyperTree.cu:266-514). A proposal
 * MLP (ATDF_PROPOSAL_INPUTS -> 64 x (1..3) SiLU -> ATDF_PROPOSAL_OUTPUTS)
 * maps each ray/leaf segment to 32 bin logits of a piecewise-constant sample
 * density over the segment plus one mass logit (predicted integral =
 * softplus(logit) * segment length). Leaf occupancy is kept per node as
 * ATDF_PROPOSAL_OCC floats: the mean density of its 8 octants (index = x>0
 * | (y>0)<<1 | (z>0)<<2 in leaf-local coordinates) and of the whole leaf. */
#define ATDF_PROPOSAL_BINS 32
#define ATDF_PROPOSAL_OUTPUTS 33
#define ATDF_PROPOSAL_INPUTS 16
#define ATDF_PROPOSAL_OCC 9

/* atdf_project_forward that also adds each sample's rho * w into 32 equal
 * bins of its segment: seg_bins [segment capacity][32] (zero-filled by the
 * call; capacity and order as in the workspace's segment view). */
int atdf_project_forward_binned(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                                const float* ray_origin, const float* ray_direction, int64_t num_rays,
                                int32_t max_samples_per_node, uint64_t jitter_seed, float* image, float* seg_bins,
                                void* workspace, size_t workspace_bytes, int32_t* dev_error, atdf_stream_t stream);

/* Ray/leaf segments (with the uniform per-node sample counts) into a fused
 * workspace sized by atdf_project_workspace_size; *view receives the
 * workspace's segment arrays. A caller may then overwrite nsamp, first,
 * ray_sample_offset and totals[1..2] (atdf_proposal_allocate does) and
 * project with caller-placed samples. */
int atdf_project_segments(const atdf_tree_t* tree, const float* ray_origin, const float* ray_direction,
                          int64_t num_rays, int32_t max_samples_per_node, int64_t num_slots, void* workspace,
                          size_t workspace_bytes, atdf_segments_t* view, int32_t* dev_error, atdf_stream_t stream);

/* The segment arrays inside a fused workspace (no device work). */
int atdf_project_segment_view(int64_t num_rays, int32_t max_depth, int64_t num_slots, void* workspace,
                              size_t workspace_bytes, atdf_segments_t* view);

/* Forward projection over the workspace's segments with caller-placed
 * samples: sample_t / sample_w [total samples] in canonical order (index =
 * ray_sample_offset[ray] + first[segment] + j). */
int atdf_project_forward_samples(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                                 const float* ray_origin, const float* ray_direction, int64_t num_rays,
                                 const float* sample_t, const float* sample_w, float* image, void* workspace,
                                 size_t workspace_bytes, int32_t* dev_error, atdf_stream_t stream);

/* Adjoint of atdf_project_forward_samples (same workspace and samples). */
int atdf_project_backward_samples(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                                  const float* ray_origin, const float* ray_direction, int64_t num_rays,
                                  const float* sample_t, const float* sample_w, const float* grad_image,
                                  const atdf_field_grad_t* grad_field, const atdf_mlp_grad_t* grad_mlp,
                                  void* workspace, size_t workspace_bytes, int32_t* dev_error, atdf_stream_t stream);

/* Proposal inputs per segment, features [segment capacity][16]: leaf-local
 * entry point (3), leaf-local exit point (3), segment length / leaf
 * diagonal, the leaf's mean occupancy, its 8 octant occupancies
 * (occupancy [num_nodes][9], nullable: zeros). Rows from totals[0] on are
 * untouched. */
int atdf_proposal_features(const atdf_tree_t* tree, const atdf_segments_t* segments, const float* ray_origin,
                           const float* ray_direction, const float* occupancy, float* features, int32_t* dev_error,
                           atdf_stream_t stream);

/* The proposal MLP over the totals[0] segment rows (count read on the
 * device): logits [capacity][33] = MLP(features). mlp: 16 -> 64 x (1..3) ->
 * 33, SiLU hidden, identity last (else ATDF_ERR_UNSUPPORTED). */
int atdf_proposal_mlp_forward(const atdf_mlp_t* mlp, const atdf_segments_t* segments, const float* features,
                              float* logits, atdf_stream_t stream);

/* Its adjoint: OVERWRITES grad_mlp with the weight and bias gradients for
 * grad_logits [capacity][33] (rows < totals[0]). */
int atdf_proposal_mlp_backward(const atdf_mlp_t* mlp, const atdf_segments_t* segments, const float* features,
                               const float* grad_logits, const atdf_mlp_grad_t* grad_mlp, atdf_stream_t stream);

/* The same two functions on the tensor cores (tcgen05, BF16 operands, FP32
 * accumulation) for the 3-hidden-layer network 16 -> 64 -> 64 -> 64 -> 33
 * (else ATDF_ERR_UNSUPPORTED): results within BF16 rounding of the FP32
 * kernels above. The weights and the features must be 16-byte aligned
 * (ATDF_ERR_INVALID_ARGUMENT otherwise). A bounded wait that runs out sets
 * ATDF_DEVERR_TREE. */
int atdf_proposal_mlp_forward_bf16(const atdf_mlp_t* mlp, const atdf_segments_t* segments, const float* features,
                                   float* logits, int32_t* dev_error, atdf_stream_t stream);
int atdf_proposal_mlp_backward_bf16(const atdf_mlp_t* mlp, const atdf_segments_t* segments, const float* features,
                                    const float* grad_logits, const atdf_mlp_grad_t* grad_mlp, int32_t* dev_error,
                                    atdf_stream_t stream);

/* Splits a budget of samples per ray over its segments: n = 1 +
 * round((budget - segments of the ray) * share), share = (1 - mass_mix) *
 * weight share + mass_mix * length share, weight = length * (predicted mean
 * density)^mass_power (mass_power in [0, 1]: 0 is the uniform per-length
 * rule, 1 allocates by predicted mass, 1/2 minimises the error of stratified
 * sampling when a segment's variation scales with its density). Overwrites
 * nsamp, first, ray_sample_offset, totals[1] (samples) and totals[2] (max
 * per ray). A ray gets at most budget + its segment count samples. */
int atdf_proposal_allocate(const atdf_segments_t* segments, int64_t num_rays, const float* logits, int32_t budget,
                           float mass_mix, float mass_power, atdf_stream_t stream);

/* Sample t and weight of every segment's nsamp samples: stratified
 * inverse-CDF draws u_j = (j + a_j) / n (a_j the interval jitter hash of
 * seed, 0.5 for seed 0) from q = (1 - bin_mix) softmax(bin_power * bin
 * logits) + bin_mix / 32 over 32 equal bins (the predicted distribution
 * raised to bin_power in [0, 1]; bin_mix in (0, 1] keeps samples
 * everywhere). weight_rule ATDF_PROPOSAL_WEIGHTS_VORONOI: the samples'
 * Voronoi cells within the segment, the rule of the uniform sampler
 * (HyperTree.cu:495-512), so with uniform q the result is the uniform
 * per-node quadrature with these counts; ATDF_PROPOSAL_WEIGHTS_IMPORTANCE:
 * w_j = 1 / (n q(t_j)) (bin width / (n p_bin)), the importance weights under
 * which sum_j w_j rho(t_j) is an unbiased estimate of the segment integral
 * for uniform jitter. */
#define ATDF_PROPOSAL_WEIGHTS_VORONOI 0
#define ATDF_PROPOSAL_WEIGHTS_IMPORTANCE 1
int atdf_proposal_samples(const atdf_segments_t* segments, const float* logits, float bin_mix, float bin_power,
                          uint64_t seed, int32_t weight_rule, float* sample_t, float* sample_w,
                          int64_t sample_capacity, int32_t* dev_error, atdf_stream_t stream);

/* Training loss of the proposal against seg_bins of a uniform binned forward
 * on the same segments: mean over segments of the cross-entropy of the
 * normalised bins vs softmax(bin logits) plus mass_weight * (log(m_hat +
 * 1e-4) - log(m + 1e-4))^2. Writes grad_logits (rows < totals[0]),
 * OVERWRITES *loss (device double) and node_mass / node_len [num_nodes][9]
 * with the target mass and crossed length per leaf octant and leaf (FP64;
 * bin centres placed by the features' entry / exit points). */
int atdf_proposal_loss(const atdf_segments_t* segments, const float* features, const float* seg_bins,
                       const float* logits, float mass_weight, float* grad_logits, double* loss, double* node_mass,
                       double* node_len, int64_t num_nodes, int32_t* dev_error, atdf_stream_t stream);

/* occupancy[i] = node_mass[i] / node_len[i] where node_len[i] > 0, over
 * num_nodes * 9 entries; other entries are kept. */
int atdf_proposal_occupancy(const double* node_mass, const double* node_len, int64_t num_nodes, float* occupancy,
                            atdf_stream_t stream);

/* ---- rays of detector pixels ---------------------------------------------
 * SceneBase::GetRays (SceneBase.cpp:369-450) with UVToPixel
 * (CameraPose.h:14-30) and CameraModelModule::Unproject (CameraPose.cu:469-479)
 * for n pixels: uv [n,2] in [0,1] (pixel centres at (i + 0.5) / w without
 * align_corners), image_id [n], camera_id [n] (nullable: camera 0); per image
 * rotation [num_images,4] unit quaternions (x, y, z, w) and translation
 * [num_images,3] (pinhole only, nullable otherwise); per camera intrinsics
 * [num_cameras,5] = fx fy cx cy s; volume_translation: host float[3]
 * (orthographic only, nullable = 0). FP64 arithmetic, FP32 outputs
 * origin / direction [n,3]. An out-of-range image or camera index sets
 * ATDF_DEVERR_INDEX and leaves that ray unwritten. */
#define ATDF_CAMERA_PINHOLE 0
#define ATDF_CAMERA_ORTHOGRAPHIC 1
int atdf_camera_rays(int64_t n, const float* uv, const int32_t* image_id, const int32_t* camera_id,
                     const double* rotation, const double* translation, int64_t num_images, const double* intrinsics,
                     int64_t num_cameras, int32_t width, int32_t height, int32_t align_corners, int32_t model,
                     const float* volume_translation, float* origin, float* direction, int32_t* dev_error,
                     atdf_stream_t stream);

/* SceneBase::PointInAnyImage (hyperacorn/csrc/data/SceneBase.cu:13-97), the
 * visibility mask of the per-leaf max-density grid: mask[i] = 1 when point i
 * ([n, 3] float) lies in the ROI box [roi_min, roi_max] (host float[3] each,
 * closed bounds) and projects to a pixel of at least one of the num_images
 * poses (rotation [num_images, 4] unit quaternions x y z w, translation
 * [num_images, 3] or null = 0; view = R^T (p - t), intrinsics [5] = fx fy cx
 * cy s with the skew ignored, pixel rounded half away from zero, inside
 * [0, width) x [0, height)); else 0. */
int atdf_point_in_any_image(int64_t n, const float* points, const double* rotation, const double* translation,
                            int64_t num_images, const double* intrinsics, int32_t width, int32_t height,
                            int32_t model, const float* roi_min, const float* roi_max, float* mask,
                            atdf_stream_t stream);

/* ---- optimizer step ------------------------------------------------------
 * Replaces the torch::optim::Adam step the reference builds for the grid and
 * decoder parameters (geometry_tensor_qo.cpp:79-81, 209-220): torch's Adam
 * update (no amsgrad; weight_decay is L2 added to the gradient) over n FP32
 * elements of one parameter, in place on param, exp_avg and exp_avg_sq;
 * step is the 1-based step count after this update (bias corrections
 * 1 - beta^step). param_bf16 (nullable) receives the updated parameter
 * rounded to BF16, the working copy of the BF16 form, in the same pass. All
 * arrays share one element order (any dense layout, the same for all). */
int atdf_adam_step(int64_t n, float* param, const float* grad, float* exp_avg, float* exp_avg_sq, void* param_bf16,
                   float lr, float beta1, float beta2, float eps, float weight_decay, int64_t step,
                   atdf_stream_t stream);

/* atdf_adam_step for `count` parameter tensors (each with its own sizes,
 * hyper-parameters and step) in one launch per 16 tensors. */
typedef struct {
    int64_t n;
    float* param;
    const float* grad;
    float* exp_avg;
    float* exp_avg_sq;
    void* param_bf16; /* nullable */
    float lr, beta1, beta2, eps, weight_decay;
    int64_t step;
} atdf_adam_tensor_t;
int atdf_adam_step_multi(int32_t count, const atdf_adam_tensor_t* tensors, atdf_stream_t stream);

/* ---- photometric calibration (the tone mapper) ------------------------------
 * Replaces PhotometricCalibrationImpl::forward
 * (hyperacorn/csrc/modules/ToneMapper.cpp:161-201) with its camera response
 * CameraResponseNetImpl::forward (:32-97) and the autograd adjoint of both.
 * Per element (channel c, ray r) of the projected integrals I [channels, R]:
 *   x  = I + exposure[image_id[r]]  (ATDF_EXPOSURE_BIAS, exposure_mult = false)
 *      | I * exposure[image_id[r]]  (ATDF_EXPOSURE_FACTOR, exposure_mult = true)
 *   x += bilinear(sensor_bias [sensor_h, sensor_w], uv[r])   (border, align_corners = false)
 *   y  = bilinear(response [response_params], x / range)   (border, align_corners = true)
 *      + (x - range) when leak and x > range                (training mode)
 * with torch grid_sample semantics for both lookups; uv [R, 2] in [0, 1]
 * (u along the width). A disabled part has mode NONE / size 0. The response
 * curve has one channel: with it, channels must be 1 (ATDF_ERR_UNSUPPORTED
 * otherwise, as the reference asserts). An image id outside [0, num_images)
 * sets ATDF_DEVERR_INDEX and yields NaN (forward) / a zero gradient. */
#define ATDF_EXPOSURE_NONE 0
#define ATDF_EXPOSURE_BIAS 1
#define ATDF_EXPOSURE_FACTOR 2
typedef struct {
    int32_t num_images;
    int32_t exposure_mode;    /* ATDF_EXPOSURE_* */
    const float* exposure;    /* [num_images]: the bias or the factor */
    int32_t sensor_w, sensor_h; /* sensor-bias map size; 0 = disabled */
    const float* sensor_bias; /* [sensor_h, sensor_w] */
    int32_t response_params;  /* samples of the response curve (>= 2); 0 = disabled */
    const float* response;    /* [response_params] */
    float response_range;     /* the curve spans inputs [0, range] */
    int32_t leak;             /* 1: add the leak above the range (training mode) */
} atdf_tone_mapper_t;

int atdf_tone_map_forward(const atdf_tone_mapper_t* tm, int64_t channels, int64_t num_rays, const float* integral,
                          const float* uv, const int32_t* image_id, float* out, int32_t* dev_error,
                          atdf_stream_t stream);

/* The adjoint of atdf_tone_map_forward for grad_out [channels, R]:
 * grad_integral [channels, R] is written (may be null); grad_exposure
 * [num_images], grad_sensor_bias [sensor_h, sensor_w] and grad_response
 * [response_params] are ADDED to (each may be null when not wanted). */
int atdf_tone_map_backward(const atdf_tone_mapper_t* tm, int64_t channels, int64_t num_rays, const float* integral,
                           const float* uv, const int32_t* image_id, const float* grad_out, float* grad_integral,
                           float* grad_exposure, float* grad_sensor_bias, float* grad_response, int32_t* dev_error,
                           atdf_stream_t stream);

/* The response curve's smoothness loss, CameraResponseNetImpl::ParamLoss
 * (ToneMapper.cpp:98-111): with f = P sqrt(1e-5) and targets t_0 = 0,
 * t_{P-1} = range, t_i = (r_{i-1} + r_{i+1}) / 2, loss = sum_i (f r_i - f t_i)^2.
 * *loss (device float, may be null) is written; (*grad_scale) * d loss / d r
 * is ADDED to grad_response (may be null); grad_scale is a device float (the
 * upstream gradient of the loss), null for 1. */
int atdf_tone_response_loss(int32_t response_params, const float* response, float response_range, float* loss,
                            float* grad_response, const float* grad_scale, atdf_stream_t stream);

/* ---- forward projection without device allocation ----------------------
 * No counterpart in the reference (it allocates with torch on every call).
 * For callers that cannot call cudaMalloc (a plugin whose host framework owns
 * every device allocation, or a loop where an allocation would synchronise
 * the device): atdf_project_forward with its workspace taken from a static
 * device array of ATDF_NOALLOC_SCRATCH_BYTES (16 MiB) that every GPU loading
 * the library holds until exit. A problem whose workspace
 * (atdf_project_workspace_size) exceeds it is rejected with
 * ATDF_ERR_WORKSPACE before any launch; at depth 4 that is about 10,000
 * rays per call. Every call looks the array's address up in the current
 * context (cudaGetSymbolAddress, no device work); the first call in a context
 * loads the library's module there, so make that first call on each device
 * before any stream capture. All calls share the array: calls that overlap on
 * the GPU race. Inputs and outputs are the caller's, as in
 * atdf_project_forward. It is forward only: the segments it leaves in the
 * array are not a workspace that atdf_project_backward can take, so a caller
 * that needs gradients uses atdf_project_forward with its own workspace. */
#define ATDF_NOALLOC_SCRATCH_BYTES (16u << 20)
int atdf_project_forward_noalloc(const atdf_tree_t* tree, const atdf_field_t* field, const atdf_mlp_t* mlp,
                                 const float* ray_origin, const float* ray_direction, int64_t num_rays,
                                 int32_t max_samples_per_node, uint64_t jitter_seed, float* image,
                                 int32_t* dev_error, atdf_stream_t stream);

/* ---- synthetic tilt series ------------------------------------------------
 * FP64 line integrals of a voxel volume [nz][ny][nx] (float) spanning the box
 * [box_min, box_max] (host double[3] each) along num_rays rays (origin /
 * direction [R, 3] float): out[r] = sum over traversed voxels of (exit t -
 * entry t) * value, i.e. exact intersection lengths in units of t. Generates
 * the projections that the reference reads from measured tilt series
 * (hyperacorn/csrc/data/SceneBase.cpp:904-1000). */
int atdf_siddon_project(const float* volume, int32_t nx, int32_t ny, int32_t nz, const double* box_min,
                        const double* box_max, const float* ray_origin, const float* ray_direction,
                        int64_t num_rays, double* out, atdf_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* ATDF_H */
