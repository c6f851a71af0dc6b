// HyperTreeBase: the reference's HyperTreeBaseImpl surface
// (hyperacorn/csrc/structure/HyperTree.h:395-561, HyperTree.cpp:298-705,
// HyperTree.cu:237-259,516-610,1339-1525) over libatdf_b200.so.
#include <ATen/cuda/CUDAContext.h>

#include <algorithm>
#include <cstring>
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
// Tree structure optimisation. The reference solves a mixed-integer program
// with OR-Tools / CBC (HyperTreeStructureOptimizer.cpp:5-392): every active
// leaf chooses none / split / merge (all active siblings together), the cost
// of a choice is error x max density with the split and merge predictions of
// :211-323 (split: error_split_factor x own error; merge: error_merge_factor x
// the siblings' error sum, at the siblings' max density), and the active-leaf
// count after the change must stay within max_active_nodes (:146-206). OR-Tools
// is not available, so the same program is solved greedily: merges with the
// smallest cost increase per freed leaf until the budget holds, then splits
// by gain per added leaf, paying for a split with cheaper merges while that
// lowers the objective.
// ---------------------------------------------------------------------------
bool HyperTreeBase::OptimizeStructure(int64_t max_active_nodes, double error_merge_factor,
                                      double error_split_factor)
{
    auto dev = node_position_min.device();
    auto act_t = node_active.to(torch::kCPU).contiguous().clone();
    auto cul_t = node_culled.to(torch::kCPU).contiguous();
    auto chd_t = node_children.to(torch::kCPU).contiguous();
    auto par_t = node_parent.to(torch::kCPU).contiguous();
    auto err_t = node_error.to(torch::kCPU).to(torch::kFloat64).contiguous();
    auto den_t = node_max_density.to(torch::kCPU).to(torch::kFloat64).contiguous();
    const int64_t n = act_t.size(0);
    const int ns = NS();
    int32_t* act = act_t.data_ptr<int32_t>();
    const int32_t* cul = cul_t.data_ptr<int32_t>();
    const int32_t* chd = chd_t.data_ptr<int32_t>();
    const int32_t* par = par_t.data_ptr<int32_t>();
    const double* err = err_t.data_ptr<double>();
    const double* den = den_t.data_ptr<double>();
    auto e_of = [&](int64_t i) { return err[i] > 0 ? err[i] : 0.0; };
    // a density never computed (negative) counts as 1
    auto d_of = [&](int64_t i) { return den[i] >= 0 ? den[i] : 1.0; };

    struct Split {
        int64_t node;
        double gain;
        int cost;  // leaves added
    };
    struct Merge {
        int64_t parent;
        double loss;
        int freed;  // leaves removed
    };
    std::vector<Split> splits;
    std::vector<Merge> merges;
    int64_t count = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (act[i] != 1) continue;
        ++count;
        if (chd[i * ns] >= 0) {
            int live = 0;
            for (int k = 0; k < ns; ++k) live += cul[chd[i * ns + k]] ? 0 : 1;
            if (live > 0) {
                const double none = e_of(i) * d_of(i);
                const double split = error_split_factor * e_of(i) * d_of(i);
                splits.push_back({i, none - split, live - 1});
            }
        }
    }
    for (int64_t p = 0; p < n; ++p) {
        if (chd[p * ns] < 0) continue;
        int active = 0, culled = 0;
        double esum = 0, dmax = 0, none = 0;
        for (int k = 0; k < ns; ++k) {
            const int32_t c = chd[p * ns + k];
            if (act[c] == 1) {
                ++active;
                esum += e_of(c);
                dmax = std::max(dmax, d_of(c));
                none += e_of(c) * d_of(c);
            } else if (cul[c]) {
                ++culled;
            }
        }
        if (active == 0 || active + culled != ns) continue;
        merges.push_back({p, error_merge_factor * esum * dmax - none, active - 1});
    }
    std::sort(splits.begin(), splits.end(), [](const Split& a, const Split& b) {
        return a.gain * std::max(b.cost, 1) > b.gain * std::max(a.cost, 1);
    });
    std::sort(merges.begin(), merges.end(), [](const Merge& a, const Merge& b) {
        return a.loss * std::max(b.freed, 1) < b.loss * std::max(a.freed, 1);
    });
    std::vector<char> split_taken(n, 0), merge_taken(n, 0), blocked(n, 0);  // blocked: parent of a split leaf
    size_t mi = 0;
    auto next_merge = [&]() -> int64_t {
        while (mi < merges.size() && (blocked[merges[mi].parent] || merge_taken[merges[mi].parent])) ++mi;
        return mi < merges.size() ? (int64_t)mi : -1;
    };
    // 1. meet the budget
    while (count > max_active_nodes) {
        const int64_t k = next_merge();
        if (k < 0) break;
        merge_taken[merges[k].parent] = 1;
        count -= merges[k].freed;
        ++mi;
    }
    // 2. splits, paid for by merges when the budget is full
    for (const Split& sp : splits) {
        if (sp.gain <= 0) break;
        const int64_t parent = par[sp.node];
        if (parent >= 0 && merge_taken[parent]) continue;  // its sibling group is being merged
        if (count + sp.cost <= max_active_nodes) {
            split_taken[sp.node] = 1;
            if (parent >= 0) blocked[parent] = 1;
            count += sp.cost;
            continue;
        }
        // merges needed to make room, cheapest first, none involving this leaf
        const char was_blocked = parent >= 0 ? blocked[parent] : 0;
        if (parent >= 0) blocked[parent] = 1;
        std::vector<int64_t> pick;
        double loss = 0;
        int64_t freed = 0;
        size_t save = mi;
        while (count + sp.cost - freed > max_active_nodes) {
            const int64_t k = next_merge();
            if (k < 0) break;
            pick.push_back(k);
            loss += merges[k].loss;
            freed += merges[k].freed;
            ++mi;
        }
        if (count + sp.cost - freed <= max_active_nodes && loss < sp.gain) {
            for (int64_t k : pick) merge_taken[merges[k].parent] = 1;
            split_taken[sp.node] = 1;
            count += sp.cost - freed;
        } else {
            mi = save;
            if (parent >= 0) blocked[parent] = was_blocked;
            break;
        }
    }
    bool changed = false;
    for (int64_t i = 0; i < n; ++i) {
        if (split_taken[i]) {
            act[i] = 0;
            for (int k = 0; k < ns; ++k) {
                const int32_t c = chd[i * ns + k];
                if (!cul[c]) act[c] = 1;
            }
            changed = true;
        }
        if (merge_taken[i]) {
            for (int k = 0; k < ns; ++k) act[chd[i * ns + k]] = 0;
            act[i] = 1;
            changed = true;
        }
    }
    if (changed) {
        node_active = act_t.to(dev);
        UpdateActive();
    }
    return changed;
}

}  // namespace atdf_host
