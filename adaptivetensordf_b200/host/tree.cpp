// HyperTreeBase: the reference's HyperTreeBaseImpl surface
// (hyperacorn/csrc/structure/HyperTree.h:395-561, HyperTree.cpp:298-705,
// HyperTree.cu:237-259,516-610,1339-1525) over libatdf_b200.so.
#include <ATen/cuda/CUDAContext.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "atdf_host.h"

namespace atdf_host {

static cudaStream_t cur_stream() { return at::cuda::getCurrentCUDAStream().stream(); }

void check_status(int status, const char* what)
{
    TORCH_CHECK(status == ATDF_OK, what, " failed: ", atdf_status_string(status));
}

void check_dev_error(torch::Tensor err, const char* what)
{
    const int v = err.item<int>();
    TORCH_CHECK(v == 0, what, ": device error flags ", v,
                (v & ATDF_DEVERR_HIT_OVERFLOW) ? " [a ray hit more than 256 leaves]" : "",
                (v & ATDF_DEVERR_SEG_CAPACITY) ? " [segment capacity exceeded]" : "",
                (v & ATDF_DEVERR_SAMPLE_CAPACITY) ? " [sample capacity exceeded]" : "",
                (v & ATDF_DEVERR_INDEX) ? " [index out of range]" : "", (v & ATDF_DEVERR_TREE) ? " [tree]" : "");
}

HyperTreeBase::HyperTreeBase(int d_, int max_depth_) : d(d_), max_depth(max_depth_)
{
    TORCH_CHECK(d == 3, "HyperTreeBase: only d = 3 is supported (the reference kernels are 3D)");
}

// settree (HyperTree.cpp:298-525): breadth-first numbering; child i takes the
// upper half on split axis k iff bit k of i is set; the quad tree splits x and
// z only and spans [y_min, y_max] in y.
void HyperTreeBase::settree(bool use_quad, float y_min, float y_max)
{
    use_quad_tree = use_quad;
    const int ns = NS();
    const int split_dims = use_quad ? d - 1 : d;
    int64_t num_nodes = 0;
    for (int i = 0; i <= max_depth; ++i) {
        int64_t n = 1;
        for (int j = 0; j < i; ++j) n *= ns;
        num_nodes += n;
    }
    node_parent = torch::empty({num_nodes}, torch::kInt32);
    node_children = -torch::ones({num_nodes, ns}, torch::kInt32);
    node_position_min = torch::empty({num_nodes, d}, torch::kFloat32);
    node_position_max = torch::empty({num_nodes, d}, torch::kFloat32);
    node_scale = torch::empty({num_nodes}, torch::kFloat32);
    node_error = -torch::ones({num_nodes}, torch::kFloat32);
    node_max_density = -torch::ones({num_nodes}, torch::kFloat32);
    node_active = torch::zeros({num_nodes}, torch::kInt32);
    node_culled = torch::zeros({num_nodes}, torch::kInt32);
    node_depth = torch::zeros({num_nodes}, torch::kInt32);

    float* pmin = node_position_min.data_ptr<float>();
    float* pmax = node_position_max.data_ptr<float>();
    int32_t* ch = node_children.data_ptr<int32_t>();
    int32_t* dep = node_depth.data_ptr<int32_t>();
    int32_t* par = node_parent.data_ptr<int32_t>();
    float* sc = node_scale.data_ptr<float>();
    auto set_node = [&](int64_t id, int64_t parent, const float* mn, const float* mx, int depth) {
        float scale = ((float)depth / (max_depth)) * 2 - 1;
        if (max_depth == 0) scale = 0;
        for (int k = 0; k < d; ++k) {
            pmin[id * d + k] = mn[k];
            pmax[id * d + k] = mx[k];
        }
        if (use_quad) {
            pmin[id * d + 1] = y_min;
            pmax[id * d + 1] = y_max;
        }
        dep[id] = depth;
        par[id] = (int32_t)parent;
        sc[id] = scale;
    };
    int64_t current = 0;
    const float rmin[3] = {-1, -1, -1}, rmax[3] = {1, 1, 1};
    set_node(current++, -1, rmin, rmax, 0);
    int64_t start_layer = 0;
    for (int depth = 1; depth <= max_depth; ++depth) {
        const int64_t n = current - start_layer;
        for (int64_t j = 0; j < n; ++j) {
            const int64_t node = start_layer + j;
            float mn[3], mx[3], center[3];
            for (int k = 0; k < d; ++k) {
                mn[k] = pmin[node * d + k];
                mx[k] = pmax[node * d + k];
                center[k] = (mn[k] + mx[k]) * 0.5f;
            }
            for (int i = 0; i < ns; ++i) {
                float cmn[3] = {mn[0], mn[1], mn[2]}, cmx[3] = {mx[0], mx[1], mx[2]};
                for (int k = 0; k < split_dims; ++k) {
                    const int axis = (split_dims == 2 && k == 1) ? 2 : k;
                    if (((i >> k) & 1) == 0) {
                        cmn[axis] = mn[axis];
                        cmx[axis] = center[axis];
                    } else {
                        cmn[axis] = center[axis];
                        cmx[axis] = mx[axis];
                    }
                }
                ch[node * ns + i] = (int32_t)current;
                set_node(current++, node, cmn, cmx, depth);
            }
        }
        start_layer = current - n * ns;
    }
    active_node_ids = torch::zeros({1}, torch::kLong);
    SetActive(0);
}

void HyperTreeBase::SetActive(int depth)
{
    node_active = (node_depth == depth).to(torch::kInt32);
    UpdateActive();
}

// UpdateActive (HyperTree.cpp:550-588): ascending active ids, the active
// prefix sum (-1 for inactive nodes), and the traversal flags.
void HyperTreeBase::UpdateActive()
{
    auto dev = node_position_min.device();
    auto act = node_active.to(torch::kCPU).contiguous();
    auto cul = node_culled.to(torch::kCPU).contiguous();
    TORCH_CHECK((act * cul).sum().item<int64_t>() == 0, "UpdateActive: a culled node is active");
    const int64_t n = act.size(0);
    const int32_t* a = act.data_ptr<int32_t>();
    std::vector<int64_t> ids, pref(n, -1);
    for (int64_t i = 0; i < n; ++i)
        if (a[i] == 1) {
            pref[i] = (int64_t)ids.size();
            ids.push_back(i);
        }
    active_node_ids = torch::from_blob(ids.data(), {(int64_t)ids.size()}, torch::kLong).clone().to(dev);
    node_active_prefix_sum = torch::from_blob(pref.data(), {n}, torch::kLong).clone().to(dev);
    node_active = node_active.to(dev);
    if (dev.is_cuda()) {
        node_flags = torch::zeros({n}, torch::TensorOptions().dtype(torch::kUInt8).device(dev));
        auto err = torch::zeros({1}, torch::TensorOptions().dtype(torch::kInt32).device(dev));
        auto ac = node_active.contiguous();
        auto chd = node_children.to(dev).contiguous();
        check_status(atdf_tree_flags(ac.data_ptr<int32_t>(), chd.data_ptr<int32_t>(), NS(), n,
                                     node_flags.data_ptr<uint8_t>(), err.data_ptr<int32_t>(),
                                     (atdf_stream_t)cur_stream()),
                     "atdf_tree_flags");
        check_dev_error(err, "atdf_tree_flags");
    } else {
        // host sweep (children have larger ids than their parent)
        auto chd = node_children.contiguous();
        const int32_t* c = chd.data_ptr<int32_t>();
        std::vector<uint8_t> fl(n, 0);
        for (int64_t i = n - 1; i >= 0; --i) {
            uint8_t f = a[i] == 1 ? 1 : 0;
            for (int k = 0; k < NS(); ++k) {
                const int32_t cc = c[i * NS() + k];
                if (cc >= 0 && cc < n && (fl[cc] & 3)) f |= 2;
            }
            fl[i] = f;
        }
        node_flags = torch::from_blob(fl.data(), {n}, torch::kUInt8).clone();
    }
}

void HyperTreeBase::to(torch::Device device)
{
    node_parent = node_parent.to(device);
    node_children = node_children.to(device);
    node_position_min = node_position_min.to(device);
    node_position_max = node_position_max.to(device);
    node_scale = node_scale.to(device);
    node_error = node_error.to(device);
    node_max_density = node_max_density.to(device);
    node_active = node_active.to(device);
    node_culled = node_culled.to(device);
    node_depth = node_depth.to(device);
    UpdateActive();
}

atdf_tree_t HyperTreeBase::view() const
{
    TORCH_CHECK(node_position_min.is_cuda(), "HyperTreeBase: the tree must be on a CUDA device (call to('cuda'))");
    TORCH_CHECK(node_flags.defined() && node_flags.is_cuda(), "HyperTreeBase: flags missing, call UpdateActive()");
    TORCH_CHECK(node_position_min.is_contiguous() && node_position_max.is_contiguous() &&
                    node_children.is_contiguous() && node_active.is_contiguous(),
                "HyperTreeBase: buffers must be contiguous");
    TORCH_CHECK(node_children.scalar_type() == torch::kInt32 && node_active.scalar_type() == torch::kInt32,
                "HyperTreeBase: node_children / node_active must be int32");
    atdf_tree_t t;
    t.node_position_min = node_position_min.data_ptr<float>();
    t.node_position_max = node_position_max.data_ptr<float>();
    t.node_children = node_children.data_ptr<int32_t>();
    t.node_active = node_active.data_ptr<int32_t>();
    t.node_flags = node_flags.data_ptr<uint8_t>();
    t.num_nodes = NumNodes();
    t.ns = NS();
    t.max_depth = max_depth;
    return t;
}

static void check_rays(const RayList& rays)
{
    TORCH_CHECK(rays.origin.is_cuda() && rays.direction.is_cuda(), "rays must be CUDA tensors (no CPU path)");
    TORCH_CHECK(rays.origin.dim() == 2 && rays.origin.size(1) == 3 && rays.direction.sizes() == rays.origin.sizes(),
                "rays: origin and direction must be [R, 3]");
    TORCH_CHECK(rays.origin.scalar_type() == torch::kFloat32 && rays.direction.scalar_type() == torch::kFloat32,
                "rays must be float32");
}

static int64_t segment_capacity(int64_t R, int max_depth)
{
    int64_t per = 3 * ((int64_t)1 << std::min(std::max(max_depth, 0), 20)) + 3;
    per = std::min<int64_t>(per, ATDF_MAX_HITS);
    return std::max<int64_t>(R * per, 1);
}

SegmentList HyperTreeBase::RaySegments(const RayList& rays, int max_samples_per_node)
{
    check_rays(rays);
    auto t = view();
    auto dev = node_position_min.device();
    const int64_t R = rays.size();
    auto o = rays.origin.contiguous(), dr = rays.direction.contiguous();
    const int64_t cap = segment_capacity(R, max_depth);
    auto li = torch::TensorOptions().dtype(torch::kLong).device(dev);
    auto ii = torch::TensorOptions().dtype(torch::kInt32).device(dev);
    auto fi = torch::TensorOptions().dtype(torch::kFloat32).device(dev);
    SegmentList s;
    s.ray_seg_offset = torch::empty({R + 1}, li);
    s.ray_sample_offset = torch::empty({R + 1}, li);
    s.node = torch::empty({cap}, ii);
    s.nsamp = torch::empty({cap}, ii);
    s.ray = torch::empty({cap}, ii);
    s.first = torch::empty({cap}, ii);
    s.tmin = torch::empty({cap}, fi);
    s.tmax = torch::empty({cap}, fi);
    auto totals = torch::zeros({4}, li);
    auto err = torch::zeros({1}, ii);
    atdf_segments_t sv;
    sv.ray_seg_offset = s.ray_seg_offset.data_ptr<int64_t>();
    sv.ray_sample_offset = s.ray_sample_offset.data_ptr<int64_t>();
    sv.node = s.node.data_ptr<int32_t>();
    sv.tmin = s.tmin.data_ptr<float>();
    sv.tmax = s.tmax.data_ptr<float>();
    sv.nsamp = s.nsamp.data_ptr<int32_t>();
    sv.ray = s.ray.data_ptr<int32_t>();
    sv.first = s.first.data_ptr<int32_t>();
    sv.capacity = cap;
    sv.totals = totals.data_ptr<int64_t>();
    check_status(atdf_ray_segments(&t, o.data_ptr<float>(), dr.data_ptr<float>(), R, max_samples_per_node, &sv,
                                   err.data_ptr<int32_t>(), (atdf_stream_t)cur_stream()),
                 "atdf_ray_segments");
    // the reference also reads the sample count back here (HyperTree.cu:550)
    auto th = totals.cpu();
    check_dev_error(err, "CreateSamplesForRays");
    const int64_t* tv = th.data_ptr<int64_t>();
    s.num_segments = tv[0];
    s.num_samples = tv[1];
    s.max_samples_per_ray = tv[2];
    s.max_segments_per_ray = tv[3];
    s.node = s.node.slice(0, 0, s.num_segments);
    s.nsamp = s.nsamp.slice(0, 0, s.num_segments);
    s.ray = s.ray.slice(0, 0, s.num_segments);
    s.first = s.first.slice(0, 0, s.num_segments);
    s.tmin = s.tmin.slice(0, 0, s.num_segments);
    s.tmax = s.tmax.slice(0, 0, s.num_segments);
    return s;
}

SampleList HyperTreeBase::CreateSamplesForRaysWithRnd(const RayList& rays, int max_samples_per_node,
                                                      torch::Tensor rnd, uint64_t jitter_seed)
{
    SegmentList sg = RaySegments(rays, max_samples_per_node);
    auto dev = node_position_min.device();
    const int64_t S = sg.num_samples;
    const int64_t R = rays.size();
    auto fo = torch::TensorOptions().dtype(torch::kFloat32).device(dev);
    auto lo = torch::TensorOptions().dtype(torch::kLong).device(dev);
    SampleList list;
    list.global_coordinate = torch::empty({S, 3}, fo);
    list.ray_t = torch::empty({S}, fo);
    list.weight = torch::empty({S}, fo);
    list.ray_index = torch::empty({S}, lo);
    list.local_index_in_ray = torch::empty({S}, lo);
    list.node_id = torch::empty({S}, lo);
    list.max_samples_per_ray = sg.max_samples_per_ray;
    const float* rp = nullptr;
    torch::Tensor rc;
    if (rnd.defined()) {
        TORCH_CHECK(rnd.is_cuda() && rnd.scalar_type() == torch::kFloat32 && rnd.numel() >= S,
                    "interval jitter must be a CUDA float tensor with one value per sample");
        rc = rnd.contiguous();
        rp = rc.data_ptr<float>();
    }
    atdf_segments_t sv;
    sv.ray_seg_offset = sg.ray_seg_offset.data_ptr<int64_t>();
    sv.ray_sample_offset = sg.ray_sample_offset.data_ptr<int64_t>();
    sv.node = sg.node.data_ptr<int32_t>();
    sv.tmin = sg.tmin.data_ptr<float>();
    sv.tmax = sg.tmax.data_ptr<float>();
    sv.nsamp = sg.nsamp.data_ptr<int32_t>();
    sv.ray = sg.ray.data_ptr<int32_t>();
    sv.first = sg.first.data_ptr<int32_t>();
    sv.capacity = sg.num_segments;
    sv.totals = nullptr;
    auto err = torch::zeros({1}, torch::TensorOptions().dtype(torch::kInt32).device(dev));
    auto o = rays.origin.contiguous(), d = rays.direction.contiguous();
    check_status(atdf_emit_samples(&sv, R, o.data_ptr<float>(), d.data_ptr<float>(), rp, jitter_seed,
                                   list.global_coordinate.data_ptr<float>(), list.ray_t.data_ptr<float>(),
                                   list.weight.data_ptr<float>(), list.ray_index.data_ptr<int64_t>(),
                                   list.local_index_in_ray.data_ptr<int64_t>(), list.node_id.data_ptr<int64_t>(), S,
                                   err.data_ptr<int32_t>(), (atdf_stream_t)cur_stream()),
                 "atdf_emit_samples");
    check_dev_error(err, "CreateSamplesForRays");
    return list;
}

// CreateSamplesForRays (HyperTree.cu:516-610). With interval_jitter the jitter
// is uniform [0, 1) per sample (the reference's rand_like, :533).
SampleList HyperTreeBase::CreateSamplesForRays(const RayList& rays, int max_samples_per_node, bool interval_jitter)
{
    if (!interval_jitter) return CreateSamplesForRaysWithRnd(rays, max_samples_per_node, torch::Tensor(), 0);
    SegmentList sg = RaySegments(rays, max_samples_per_node);
    auto rnd = torch::rand({std::max<int64_t>(sg.num_samples, 1)},
                           torch::TensorOptions().dtype(torch::kFloat32).device(node_position_min.device()));
    return CreateSamplesForRaysWithRnd(rays, max_samples_per_node, rnd, 0);
}

torch::Tensor HyperTreeBase::ComputeLocalSamples(torch::Tensor global_samples, torch::Tensor node_indices)
{
    TORCH_CHECK(global_samples.is_cuda() && node_indices.is_cuda(), "ComputeLocalSamples: CUDA tensors required");
    TORCH_CHECK(global_samples.size(-1) == 3, "ComputeLocalSamples: last dimension must be 3");
    int64_t group = 1;
    if (global_samples.dim() == 3 && node_indices.dim() == 1) {
        TORCH_CHECK(node_indices.size(0) == global_samples.size(0), "ComputeLocalSamples: [G, g, 3] needs node [G]");
        group = global_samples.size(1);
    } else {
        TORCH_CHECK(node_indices.numel() * 3 == global_samples.numel(), "ComputeLocalSamples: size mismatch");
    }
    auto g = global_samples.to(torch::kFloat32).contiguous();
    auto n = node_indices.to(torch::kLong).contiguous();
    auto out = torch::empty_like(g);
    auto err = torch::zeros({1}, torch::TensorOptions().dtype(torch::kInt32).device(g.device()));
    check_status(atdf_local_samples(g.data_ptr<float>(), n.data_ptr<int64_t>(), g.numel() / 3, group,
                                    node_position_min.data_ptr<float>(), node_position_max.data_ptr<float>(),
                                    NumNodes(), out.data_ptr<float>(), err.data_ptr<int32_t>(),
                                    (atdf_stream_t)cur_stream()),
                 "atdf_local_samples");
    return out;
}

std::tuple<torch::Tensor, torch::Tensor> HyperTreeBase::NodeIdForPositionGPU(torch::Tensor global_samples)
{
    TORCH_CHECK(global_samples.is_cuda(), "NodeIdForPositionGPU: CUDA tensor required");
    auto t = view();
    auto p = global_samples.reshape({-1, 3}).to(torch::kFloat32).contiguous();
    const int64_t P = p.size(0);
    auto ids = torch::zeros({P}, p.options().dtype(torch::kLong));
    auto mask = torch::zeros({P}, p.options());
    auto err = torch::zeros({1}, p.options().dtype(torch::kInt32));
    check_status(atdf_node_id_for_position(&t, active_node_ids.data_ptr<int64_t>(), p.data_ptr<float>(), P,
                                           ids.data_ptr<int64_t>(), mask.data_ptr<float>(), err.data_ptr<int32_t>(),
                                           (atdf_stream_t)cur_stream()),
                 "atdf_node_id_for_position");
    return {ids, mask};
}

// SetErrorForActiveNodes (HyperTree.cpp:607-647).
void HyperTreeBase::SetErrorForActiveNodes(torch::Tensor error, const std::string& strategy)
{
    TORCH_CHECK(error.sizes() == node_error.sizes(), "SetErrorForActiveNodes: size mismatch");
    error = error.to(node_error.device()).to(torch::kFloat32);
    auto active_float = node_active.to(torch::kFloat32);
    auto inactive = 1 - active_float;
    auto invalid_errors = (node_error < 0).to(torch::kFloat32);
    error = active_float * error;
    if (strategy == "override") {
        node_error = node_error * inactive + error;
    } else if (strategy == "min") {
        error = error + inactive * 1000000;
        auto filtered = node_error + (invalid_errors * active_float) * 1000000;
        node_error = torch::min(filtered, error);
    } else {
        TORCH_CHECK(false, "SetErrorForActiveNodes: unknown strategy ", strategy);
    }
}

// ---------------------------------------------------------------------------
// Structure optimisation. The reference solves a mixed-integer program with
// OR-Tools / CBC (HyperTreeStructureOptimizer.cpp:5-392): every active leaf
// chooses none / split / merge, where a merge takes all siblings of a group
// whose members are all active or culled (:146-182), a split needs children
// (:102-106, :185-196), the cost of a choice is error x max density with the
// split and merge predictions of :211-323 (none: own error at own density;
// split: error_split_factor x own error at own density; merge:
// error_merge_factor x the siblings' error sum at their max density), and the
// active-leaf count after the change (none 1, split its non-culled children,
// merge 1 per group) must stay within max_active_nodes (:136-206).
//
// The program is a multiple-choice knapsack over independent items: each
// mergeable sibling group (merge, or each member none / split) and each other
// active leaf (none / split). It is solved exactly by dynamic programming
// over the leaf count: per group a table of the cheapest member choices for
// every count, plus the merge at count 1; then the groups and leaves are
// combined count by count, keeping each item's choice for the backtrack.
// When no choice meets the budget the smallest possible leaf count is taken.
// ---------------------------------------------------------------------------
namespace {

// Cost of a set of choices and how many leaves or groups they change: among
// choices whose costs agree to 1e-12 the one with fewer changes is preferred
// (no change without a gain).
struct Score {
    double cost;
    int changes;
};

bool better(const Score& a, const Score& b)
{
    const double inf = std::numeric_limits<double>::infinity();
    if (b.cost == inf) return a.cost < inf;
    if (a.cost == inf) return false;
    const double tol = 1e-12 * std::max(std::fabs(a.cost), std::fabs(b.cost));
    if (a.cost < b.cost - tol) return true;
    if (b.cost < a.cost - tol) return false;
    return a.changes < b.changes;
}

// Leaf choices: none (count 1) and, when it has live children, split.
struct LeafItem {
    int64_t node;
    double none, split;
    int live;  // non-culled children (0: cannot split)
};

}  // namespace

bool HyperTreeBase::OptimizeStructure(int64_t max_active_nodes, double error_merge_factor,
                                      double error_split_factor)
{
    auto dev = node_position_min.device();
    auto act_t = node_active.to(torch::kCPU).contiguous().clone();
    auto cul_t = node_culled.to(torch::kCPU).contiguous();
    auto chd_t = node_children.to(torch::kCPU).contiguous();
    auto err_t = node_error.to(torch::kCPU).to(torch::kFloat64).contiguous();
    auto den_t = node_max_density.to(torch::kCPU).to(torch::kFloat64).contiguous();
    const int64_t n = act_t.size(0);
    const int ns = NS();
    int32_t* act = act_t.data_ptr<int32_t>();
    const int32_t* cul = cul_t.data_ptr<int32_t>();
    const int32_t* chd = chd_t.data_ptr<int32_t>();
    const double* err = err_t.data_ptr<double>();
    const double* den = den_t.data_ptr<double>();
    auto e_of = [&](int64_t i) { return err[i] > 0 ? err[i] : 0.0; };
    // a density never computed (negative) counts as 1
    auto d_of = [&](int64_t i) { return den[i] >= 0 ? den[i] : 1.0; };
    auto leaf_item = [&](int64_t i) {
        LeafItem it{i, e_of(i) * d_of(i), 0.0, 0};
        if (chd[i * ns] >= 0) {
            for (int k = 0; k < ns; ++k) it.live += cul[chd[i * ns + k]] ? 0 : 1;
            it.split = error_split_factor * e_of(i) * d_of(i);
        }
        return it;
    };

    // items: mergeable groups (members + merge cost) and single leaves
    struct Group {
        int64_t parent;  // -1: a single leaf
        std::vector<LeafItem> members;
        double merge;
    };
    std::vector<Group> items;
    std::vector<char> in_group(n, 0);
    for (int64_t p = 0; p < n; ++p) {
        if (chd[p * ns] < 0 || act[p] == 1) continue;
        int active = 0, culled = 0;
        for (int k = 0; k < ns; ++k) {
            const int32_t c = chd[p * ns + k];
            active += act[c] == 1;
            culled += (act[c] != 1 && cul[c]) ? 1 : 0;
        }
        if (active == 0 || active + culled != ns) continue;
        Group g{p, {}, 0.0};
        double esum = 0, dmax = 0;
        for (int k = 0; k < ns; ++k) {
            const int32_t c = chd[p * ns + k];
            if (act[c] != 1) continue;
            g.members.push_back(leaf_item(c));
            esum += e_of(c);
            dmax = std::max(dmax, d_of(c));
            in_group[c] = 1;
        }
        g.merge = error_merge_factor * esum * dmax;
        items.push_back(std::move(g));
    }
    for (int64_t i = 0; i < n; ++i) {
        if (act[i] != 1) continue;
        if (!in_group[i]) items.push_back(Group{-1, {leaf_item(i)}, 0.0});
    }

    // per item: the cheapest member choices for every leaf count (member
    // sub-table with its own backtrack), plus the merge at count 1
    const Score none_yet{std::numeric_limits<double>::infinity(), 0};
    auto reachable = [](const Score& x) { return x.cost < std::numeric_limits<double>::infinity(); };
    struct Table {
        int hi;                               // counts 1..hi
        std::vector<Score> score;             // [hi + 1]
        std::vector<char> merged;             // the count-1 entry is the merge
        std::vector<std::vector<char>> pick;  // [member][count]: member splits
    };
    std::vector<Table> tables(items.size());
    int64_t lo_total = 0, hi_total = 0;
    for (size_t gi = 0; gi < items.size(); ++gi) {
        const Group& g = items[gi];
        Table& t = tables[gi];
        int hi = 0;
        for (const LeafItem& m : g.members) hi += std::max(1, m.live);
        std::vector<Score> cur(hi + 1, none_yet), nxt(hi + 1, none_yet);
        cur[0] = Score{0.0, 0};
        t.pick.assign(g.members.size(), std::vector<char>(hi + 1, 0));
        int reach = 0;
        for (size_t mi = 0; mi < g.members.size(); ++mi) {
            const LeafItem& m = g.members[mi];
            std::fill(nxt.begin(), nxt.end(), none_yet);
            for (int b = 0; b <= reach; ++b) {
                if (!reachable(cur[b])) continue;
                const Score keep{cur[b].cost + m.none, cur[b].changes};
                if (better(keep, nxt[b + 1])) {
                    nxt[b + 1] = keep;
                    t.pick[mi][b + 1] = 0;
                }
                const Score split{cur[b].cost + m.split, cur[b].changes + 1};
                if (m.live > 0 && better(split, nxt[b + m.live])) {
                    nxt[b + m.live] = split;
                    t.pick[mi][b + m.live] = 1;
                }
            }
            reach += std::max(1, m.live);
            std::swap(cur, nxt);
        }
        t.hi = hi;
        t.score = cur;
        t.merged.assign(hi + 1, 0);
        if (g.parent >= 0 && better(Score{g.merge, 1}, t.score[1])) {
            t.score[1] = Score{g.merge, 1};
            t.merged[1] = 1;
        }
        int lo = hi;
        for (int b = 1; b <= hi; ++b)
            if (reachable(t.score[b])) lo = std::min(lo, b);
        lo_total += lo;
        hi_total += hi;
    }
    const int64_t B = std::max<int64_t>(std::min<int64_t>(max_active_nodes, hi_total), lo_total);

    // combine the items count by count: best[b] = cheapest choices at count b
    std::vector<Score> best(B + 1, none_yet), next(B + 1, none_yet);
    best[0] = Score{0.0, 0};
    std::vector<std::vector<int32_t>> choice(items.size());  // count taken by item gi at total b
    int64_t reach = 0;
    for (size_t gi = 0; gi < items.size(); ++gi) {
        const Table& t = tables[gi];
        std::fill(next.begin(), next.end(), none_yet);
        choice[gi].assign(B + 1, -1);
        for (int64_t b = 0; b <= std::min(reach, B); ++b) {
            if (!reachable(best[b])) continue;
            for (int c = 1; c <= t.hi && b + c <= B; ++c) {
                if (!reachable(t.score[c])) continue;
                const Score v{best[b].cost + t.score[c].cost, best[b].changes + t.score[c].changes};
                if (better(v, next[b + c])) {
                    next[b + c] = v;
                    choice[gi][b + c] = c;
                }
            }
        }
        reach += t.hi;
        std::swap(best, next);
    }
    int64_t bstar = -1;
    for (int64_t b = 0; b <= B; ++b)
        if (reachable(best[b]) && (bstar < 0 || better(best[b], best[bstar]))) bstar = b;
    TORCH_CHECK(bstar >= 0, "OptimizeStructure: no feasible leaf count");

    // backtrack and apply
    bool changed = false;
    int64_t b = bstar;
    for (size_t gi = items.size(); gi-- > 0;) {
        const Group& g = items[gi];
        const Table& t = tables[gi];
        const int c = choice[gi][b];
        TORCH_CHECK(c >= 1, "OptimizeStructure: backtrack failed");
        b -= c;
        if (t.merged[c]) {
            for (const LeafItem& m : g.members) act[m.node] = 0;
            act[g.parent] = 1;
            changed = true;
            continue;
        }
        int r = c;
        for (size_t mi = g.members.size(); mi-- > 0;) {
            const LeafItem& m = g.members[mi];
            if (t.pick[mi][r]) {
                act[m.node] = 0;
                for (int k = 0; k < ns; ++k) {
                    const int32_t ch = chd[m.node * ns + k];
                    if (!cul[ch]) act[ch] = 1;
                }
                r -= m.live;
                changed = true;
            } else {
                r -= 1;
            }
        }
    }
    if (changed) {
        node_active = act_t.to(dev);
        UpdateActive();
    }
    return changed;
}

}  // namespace atdf_host
