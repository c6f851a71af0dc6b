// Forward projection for callers that cannot allocate device memory.
//
// atdf_project_forward needs a caller-provided workspace (ray/leaf segments,
// slot buckets, work queue). Some callers cannot call cudaMalloc to make one:
// a plugin running inside a host framework or inference engine that owns every
// device allocation and forbids its plugins from allocating, or a
// latency-critical loop where a cudaMalloc would synchronise the device. For
// them, atdf_project_forward_noalloc takes its workspace from a fixed array in
// device memory that this library defines, so it allocates nothing.
//
// The array has ATDF_NOALLOC_SCRATCH_BYTES bytes; every GPU that loads the
// library holds it until the process exits. All calls share it and it keeps
// the previous call's contents: the projection clears what must start at zero
// (counters, bucket counts) on every call, and calls whose work overlaps on
// the GPU (two streams, or two host threads) race on it.

#include "atdf_common.cuh"

static __device__ __align__(256) unsigned char g_project_scratch[ATDF_NOALLOC_SCRATCH_BYTES];

namespace {
// Device address of the array in the current device's current context. In
// host code the name g_project_scratch is only a host-side stand-in, so the
// address is looked up with that device current. The address belongs to a
// CUDA context, not to a device ordinal: a caller that runs in a context of
// its own, or calls again after cudaDeviceReset, gets another one. So it is
// looked up on every call (a host-side table lookup once the library's
// module is loaded in the context; the first call in a context loads it) and
// never cached.
int scratch_address(void** out)
{
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_project_scratch) != cudaSuccess || !p) return ATDF_ERR_CUDA;
    *out = p;
    return ATDF_OK;
}
}  // namespace

extern "C" int atdf_project_forward_noalloc(const atdf_tree_t* tree, const atdf_field_t* field,
                                            const atdf_mlp_t* mlp, const float* ray_origin,
                                            const float* ray_direction, int64_t num_rays,
                                            int32_t max_samples_per_node, uint64_t jitter_seed, float* image,
                                            int32_t* dev_error, atdf_stream_t stream)
{
    if (!tree || !field || !mlp || mlp->num_layers <= 0 || mlp->num_layers > ATDF_MAX_LAYERS)
        return ATDF_ERR_INVALID_ARGUMENT;
    size_t need = 0;
    const int st = atdf_project_workspace_size(num_rays, tree->max_depth, tree->ns, field->num_slots,
                                               mlp->dims[mlp->num_layers], &need);
    if (st != ATDF_OK) return st;
    if (need > (size_t)ATDF_NOALLOC_SCRATCH_BYTES) return ATDF_ERR_WORKSPACE;
    void* scratch = nullptr;
    const int sa = scratch_address(&scratch);
    if (sa != ATDF_OK) return sa;
    return atdf_project_forward(tree, field, mlp, ray_origin, ray_direction, num_rays, max_samples_per_node,
                                jitter_seed, image, scratch, (size_t)ATDF_NOALLOC_SCRATCH_BYTES, dev_error, stream);
}
