// CPU oracle for the differentiable forward-projection path of the adaptive
// tensorial density field reconstructor (HyperAcorn / adaptivetensordf).
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product links or calls this file:
// only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
// the shared library built from it, and only as the checker / the timed CPU
// baseline.
//
// PARITY UNPINNED: the reference ships no tests, fixtures or golden vectors,
// and it cannot be compiled here (it needs Saiga, Eigen, OR-Tools and a
// libtorch 1.9.1 source build that are not vendored, plus several of its own
// headers that are missing from its tree). This file restates the reference's
// arithmetic from its source lines, cited per function, and is checked against
// closed-form known answers and central finite differences in tests/.
//
// Conventions shared with the CUDA path (each is a documented restatement
// choice, not an observed reference output):
//  * Intersections of one ray are ordered by (tmin, node id). The reference
//    appends them with a shared-memory atomic and leaves its sort disabled
//    (hyperacorn/csrc/structure/HyperTree.cu:341,373-374), so its order is
//    nondeterministic; this is the canonical form of its output.
//  * The sample position / t / weight arithmetic is done with one rounding per
//    source-level operation (no contraction), compiled with -ffp-contract=off.
//  * iCeil(x) is the ceiling converted to int (Saiga a9c60bd, not vendored).
//
// Layouts: planes are the reference's [N, C, H, W] (contiguous); lines are
// [1, C, L, 1] (contiguous); sample arrays are structure-of-arrays.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

enum {
    ORC_ACT_ID = 0,
    ORC_ACT_RELU = 1,
    ORC_ACT_SILU = 2,
    ORC_ACT_SIGMOID = 3,
    ORC_ACT_SOFTPLUS = 4,
    ORC_ACT_LEAKYRELU = 5,
    ORC_ACT_ABS = 6,
    ORC_ACT_TANH = 7,
};

// ---------------------------------------------------------------------------
// Tree construction: hyperacorn/csrc/structure/HyperTree.cpp:298-525
// (settree). Nodes are numbered breadth first; child i of a node takes the
// upper half on split axis k iff bit k of i is set. The octree splits x,y,z
// (NS = 8); the "quad" tree splits x and z only (NS = 4) and every node spans
// [y_min, y_max] in y. Returns the node count; arrays may be null to query it.
// ---------------------------------------------------------------------------
int64_t orc_tree_build(int max_depth, int quad, float y_min, float y_max, float* pmin, float* pmax,
                       int32_t* children, int32_t* depth, int32_t* parent)
{
    const int d = 3;
    const int NS = quad ? 4 : 8;
    const int split_dims = quad ? 2 : 3;
    int64_t num_nodes = 0;
    for (int i = 0; i <= max_depth; ++i) {
        int64_t n = 1;
        for (int j = 0; j < i; ++j) n *= NS;
        num_nodes += n;
    }
    if (!pmin) return num_nodes;

    auto set_node = [&](int64_t id, int64_t par, const float* mn, const float* mx, int dep) {
        for (int k = 0; k < d; ++k) {
            pmin[id * d + k] = mn[k];
            pmax[id * d + k] = mx[k];
        }
        if (quad) {
            pmin[id * d + 1] = y_min;
            pmax[id * d + 1] = y_max;
        }
        depth[id] = dep;
        parent[id] = (int32_t)par;
    };
    for (int64_t i = 0; i < num_nodes * NS; ++i) children[i] = -1;

    int64_t current = 0;
    float rmin[3] = {-1, -1, -1}, rmax[3] = {1, 1, 1};
    set_node(current++, -1, rmin, rmax, 0);
    int64_t start_layer = 0;
    for (int dep = 1; dep <= max_depth; ++dep) {
        int64_t n = current - start_layer;
        for (int64_t j = 0; j < n; ++j) {
            int64_t node = start_layer + j;
            float mn[3], mx[3], center[3];
            for (int k = 0; k < d; ++k) {
                mn[k] = pmin[node * d + k];
                mx[k] = pmax[node * d + k];
                center[k] = (mn[k] + mx[k]) * 0.5f;
            }
            for (int i = 0; i < NS; ++i) {
                float cmn[3] = {mn[0], mn[1], mn[2]}, cmx[3] = {mx[0], mx[1], mx[2]};
                for (int k = 0; k < split_dims; ++k) {
                    int axis = (split_dims == 2 && k == 1) ? 2 : k;
                    if (((i >> k) & 1) == 0) {
                        cmn[axis] = mn[axis];
                        cmx[axis] = center[axis];
                    } else {
                        cmn[axis] = center[axis];
                        cmx[axis] = mx[axis];
                    }
                }
                children[node * NS + i] = (int32_t)current;
                set_node(current++, node, cmn, cmx, dep);
            }
        }
        start_layer = current - n * NS;
    }
    return num_nodes;
}

// ---------------------------------------------------------------------------
// Slab test: hyperacorn/csrc/structure/HyperTree.h:338-380
// (IntersectBoxRayPrecise). Float divisions, double running interval, early
// exit, parallel rays rejected outside [min, max).
// ---------------------------------------------------------------------------
int orc_intersect_box(const float* bmin, const float* bmax, const float* o, const float* dir, float* out_tmin,
                      float* out_tmax)
{
    double t_near = -236436436;
    double t_far = 43637575;
    for (int i = 0; i < 3; i++) {
        if (dir[i] == 0) {
            if ((o[i] < bmin[i]) || (o[i] >= bmax[i])) {
                *out_tmin = 0;
                *out_tmax = 0;
                return 0;
            }
        } else {
            float T_1 = (bmin[i] - o[i]) / dir[i];
            float T_2 = (bmax[i] - o[i]) / dir[i];
            if (T_1 > T_2) {
                float tmp = T_1;
                T_1 = T_2;
                T_2 = tmp;
            }
            if (T_1 > t_near) t_near = T_1;
            if (T_2 < t_far) t_far = T_2;
            if ((t_near > t_far) || (t_far < 0)) {
                *out_tmin = 0;
                *out_tmax = 0;
                return 0;
            }
        }
    }
    *out_tmin = (float)t_near;
    *out_tmax = (float)t_far;
    return 1;
}

// Per-leaf sample count: hyperacorn/csrc/structure/HyperTree.cu:344-355.
static int seg_num_samples(const float* bmin, const float* bmax, float tmin, float tmax, int M)
{
    float dx = bmax[0] - bmin[0], dy = bmax[1] - bmin[1], dz = bmax[2] - bmin[2];
    float sq = dx * dx;
    sq = sq + dy * dy;
    sq = sq + dz * dz;
    float diag = std::sqrt(sq);
    float dis = tmax - tmin;
    float rel_dis = dis / diag;
    float prod = rel_dis * (float)M;
    return (int)std::ceil(prod);
}

struct Hit {
    float tmin, tmax;
    int32_t node;
    int32_t n;
};

static void ray_hits(const float* pmin, const float* pmax, const int64_t* active, int64_t A, const float* o,
                     const float* d, int M, std::vector<Hit>& hits)
{
    hits.clear();
    for (int64_t i = 0; i < A; ++i) {
        int64_t node = active[i];
        float tmin, tmax;
        int hit = orc_intersect_box(pmin + 3 * node, pmax + 3 * node, o, d, &tmin, &tmax);
        // HyperTree.cu:332-337: grazing hits (length < 1e-5) are skipped.
        if ((double)(tmax - tmin) < 1e-5) continue;
        if (hit) {
            Hit h;
            h.tmin = tmin;
            h.tmax = tmax;
            h.node = (int32_t)node;
            h.n = seg_num_samples(pmin + 3 * node, pmax + 3 * node, tmin, tmax, M);
            hits.push_back(h);
        }
    }
    std::sort(hits.begin(), hits.end(), [](const Hit& a, const Hit& b) {
        if (a.tmin != b.tmin) return a.tmin < b.tmin;
        return a.node < b.node;
    });
}

// ---------------------------------------------------------------------------
// Ray/leaf segments: hyperacorn/csrc/structure/HyperTree.cu:266-371 (the
// intersection half of ComputeRaySamples). For every ray, every active node is
// slab tested; each hit becomes one segment (node, tmin, tmax, n samples).
// Segments are written ray-major in canonical (tmin, node) order at offsets
// given by the exclusive scan of the per-ray segment counts. seg_first is the
// index of the segment's first sample within its ray (local_index_in_ray).
// Returns the total segment count; nothing is written when it exceeds cap.
// ray_seg_count / ray_samp_count ([R]) are always written.
// ---------------------------------------------------------------------------
int64_t orc_ray_segments(const float* pmin, const float* pmax, const int64_t* active, int64_t A,
                         const float* origin, const float* dir, int64_t R, int M, int64_t* ray_seg_count,
                         int64_t* ray_samp_count, int64_t cap, int32_t* seg_node, float* seg_tmin, float* seg_tmax,
                         int32_t* seg_n, int32_t* seg_ray, int32_t* seg_first)
{
#pragma omp parallel
    {
        std::vector<Hit> hits;
#pragma omp for schedule(dynamic, 16)
        for (int64_t r = 0; r < R; ++r) {
            ray_hits(pmin, pmax, active, A, origin + 3 * r, dir + 3 * r, M, hits);
            int64_t ns = 0;
            for (auto& h : hits) ns += h.n;
            ray_seg_count[r] = (int64_t)hits.size();
            ray_samp_count[r] = ns;
        }
    }
    std::vector<int64_t> off(R + 1, 0);
    for (int64_t r = 0; r < R; ++r) off[r + 1] = off[r] + ray_seg_count[r];
    int64_t total = off[R];
    if (total > cap || !seg_node) return total;
#pragma omp parallel
    {
        std::vector<Hit> hits;
#pragma omp for schedule(dynamic, 16)
        for (int64_t r = 0; r < R; ++r) {
            ray_hits(pmin, pmax, active, A, origin + 3 * r, dir + 3 * r, M, hits);
            int64_t s = off[r];
            int32_t first = 0;
            for (auto& h : hits) {
                seg_node[s] = h.node;
                seg_tmin[s] = h.tmin;
                seg_tmax[s] = h.tmax;
                seg_n[s] = h.n;
                seg_ray[s] = (int32_t)r;
                seg_first[s] = first;
                first += h.n;
                ++s;
            }
        }
    }
    return total;
}

// t of sample j of a segment: HyperTree.cu:448-461 (one rounding per op).
static inline float sample_t(float tmin, float tmax, int n, int j, float a)
{
    float dis = tmax - tmin;
    float step = dis / (float)n;
    float t1 = tmin + (float)j * step;
    float t2 = tmin + (float)(j + 1) * step;
    float oma = 1.0f - a;
    float p1 = t1 * oma;
    float p2 = t2 * a;
    return p1 + p2;
}

// ---------------------------------------------------------------------------
// Sample emission: HyperTree.cu:434-513 (t, weights) and :558-603 (the ATen
// recomputation pos = origin[ray] + dir[ray] * t, one rounding per op).
// Samples are written ray-major, segment by segment, at the running offset.
// rnd (nullable) holds the interval jitter of each output sample; without it
// the midpoint a = 0.5 is used (HyperTree.cu:456-460).
// ---------------------------------------------------------------------------
void orc_emit_samples(int64_t nseg, const int32_t* seg_node, const float* seg_tmin, const float* seg_tmax,
                      const int32_t* seg_n, const int32_t* seg_ray, const int32_t* seg_first, const float* origin,
                      const float* dir, const float* rnd, float* out_pos, float* out_t, float* out_w,
                      int64_t* out_ray, int64_t* out_local, int64_t* out_node)
{
    std::vector<int64_t> off(nseg + 1, 0);
    for (int64_t s = 0; s < nseg; ++s) off[s + 1] = off[s] + seg_n[s];
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t s = 0; s < nseg; ++s) {
        int n = seg_n[s];
        int64_t base = off[s];
        float tmin = seg_tmin[s], tmax = seg_tmax[s];
        for (int j = 0; j < n; ++j) {
            float a = rnd ? rnd[base + j] : 0.5f;
            out_t[base + j] = sample_t(tmin, tmax, n, j, a);
        }
        int r = seg_ray[s];
        for (int j = 0; j < n; ++j) {
            float t = out_t[base + j];
            float lo = (j == 0) ? tmin : (out_t[base + j - 1] + t) * 0.5f;
            float hi = (j == n - 1) ? tmax : (out_t[base + j + 1] + t) * 0.5f;
            out_w[base + j] = hi - lo;
            for (int k = 0; k < 3; ++k) {
                float dt = dir[3 * r + k] * t;
                out_pos[3 * (base + j) + k] = origin[3 * r + k] + dt;
            }
            out_ray[base + j] = r;
            out_local[base + j] = seg_first[s] + j;
            out_node[base + j] = seg_node[s];
        }
    }
}

// ---------------------------------------------------------------------------
// Jitter hash shared with the fused CUDA path: a uniform value in [0, 1) keyed
// by (seed, ray, node, sample index in segment), built from the SplitMix64
// finaliser (Steele, Lea, Flood 2014).
// ---------------------------------------------------------------------------
static inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
float orc_jitter(uint64_t seed, int32_t ray, int32_t node, int32_t j)
{
    uint64_t k = mix64(seed + 0x9e3779b97f4a7c15ULL * (uint64_t)(uint32_t)ray);
    k = mix64(k ^ ((uint64_t)(uint32_t)node << 32 | (uint64_t)(uint32_t)j));
    return (float)(k >> 40) * (1.0f / 16777216.0f);
}

void orc_jitter_for_segments(uint64_t seed, int64_t nseg, const int32_t* seg_node, const int32_t* seg_n,
                             const int32_t* seg_ray, float* out)
{
    int64_t o = 0;
    for (int64_t s = 0; s < nseg; ++s)
        for (int j = 0; j < seg_n[s]; ++j) out[o++] = orc_jitter(seed, seg_ray[s], seg_node[s], j);
}

// ---------------------------------------------------------------------------
// Leaf-local coordinates: HyperTree.cu:237-259 (ComputeLocalSamples):
// (x - min[node]) / (max - min) * 2 - 1, one rounding per ATen op.
// group > 1 means node[i / group] (the [G, g, 3] + [G] form).
// ---------------------------------------------------------------------------
void orc_local_samples(int64_t P, const float* pos, const int64_t* node, int64_t group, const float* pmin,
                       const float* pmax, float* out)
{
    for (int64_t i = 0; i < P; ++i) {
        int64_t nd = node[group > 1 ? i / group : i];
        for (int k = 0; k < 3; ++k) {
            float mn = pmin[3 * nd + k], mx = pmax[3 * nd + k];
            float size = mx - mn;
            float a = pos[3 * i + k] - mn;
            float b = a / size;
            float c = b * 2.0f;
            out[3 * i + k] = c - 1.0f;
        }
    }
}

// ---------------------------------------------------------------------------
// Point -> active leaf: HyperTree.cu:1339-1400,1468-1525
// (ActiveNodeIdForGlobalPosition + ComputeNodeId). Descends into the first
// child whose closed box contains the point; -1 becomes (active_ids[0], 0).
// ---------------------------------------------------------------------------
void orc_node_id_for_position(int64_t P, const float* pos, const float* pmin, const float* pmax,
                              const int32_t* children, int ns, const int32_t* node_active, int64_t first_active,
                              int64_t* out_id, float* out_mask)
{
    for (int64_t i = 0; i < P; ++i) {
        const float* p = pos + 3 * i;
        int64_t cur = 0;
        int64_t res = -1;
        while (true) {
            int64_t nid = cur;
            if (node_active[cur] > 0) {
                res = cur;
                break;
            }
            bool missing = false;
            for (int cid = 0; cid < ns; ++cid) {
                int c = children[cur * ns + cid];
                if (c == -1) {
                    missing = true;
                    break;
                }
                if (pmin[3 * c + 0] <= p[0] && pmax[3 * c + 0] >= p[0] && pmin[3 * c + 1] <= p[1] &&
                    pmax[3 * c + 1] >= p[1] && pmin[3 * c + 2] <= p[2] && pmax[3 * c + 2] >= p[2]) {
                    cur = c;
                    break;
                }
            }
            if (missing || cur == nid) {
                res = -1;
                break;
            }
        }
        if (res < 0) {
            out_id[i] = first_active;
            out_mask[i] = 0;
        } else {
            out_id[i] = res;
            out_mask[i] = 1;
        }
    }
}

}  // extern "C"

// ===========================================================================
// Templated field / decoder arithmetic (float and double instantiations).
// ===========================================================================

template <typename T>
struct Corner2 {
    int x0, x1, y0, y1;  // clamped
    T w_nw, w_ne, w_sw, w_se;
    T ix, iy;
    int ix0, iy0;  // unclamped floor
};

// Bilinear corner weights of IndirectGridSample2DForwardCUDAKernel,
// hyperacorn/csrc/modules/IndirectGridSample2D.cu:36-92 (align_corners=True,
// weights from unclamped corners, indices clamped to the border).
template <typename T>
static inline Corner2<T> corners2(T u, T v, int H, int W)
{
    Corner2<T> c;
    T ix = ((u + T(1)) / T(2)) * T(W - 1);
    T iy = ((v + T(1)) / T(2)) * T(H - 1);
    int x0 = (int)std::floor(ix), y0 = (int)std::floor(iy);
    int x1 = x0 + 1, y1 = y0 + 1;
    c.w_nw = (T(x1) - ix) * (T(y1) - iy);
    c.w_ne = (ix - T(x0)) * (T(y1) - iy);
    c.w_sw = (T(x1) - ix) * (iy - T(y0));
    c.w_se = (ix - T(x0)) * (iy - T(y0));
    c.ix = ix;
    c.iy = iy;
    c.ix0 = x0;
    c.iy0 = y0;
    auto clip = [](int a, int lim) { return std::min(lim - 1, std::max(a, 0)); };
    c.x0 = clip(x0, W);
    c.x1 = clip(x1, W);
    c.y0 = clip(y0, H);
    c.y1 = clip(y1, H);
    return c;
}

template <typename T>
struct Corner1 {
    int x0, x1;
    T w0, w1, ix;
    int ix0;
};

// Linear weights of IndirectGridSample1DForwardCUDAKernel,
// hyperacorn/csrc/modules/IndirectGridSample1D.cu:29-45.
template <typename T>
static inline Corner1<T> corners1(T u, int W)
{
    Corner1<T> c;
    T ix = ((u + T(1)) / T(2)) * T(W - 1);
    int x0 = (int)std::floor(ix);
    int x1 = x0 + 1;
    c.w0 = T(x1) - ix;
    c.w1 = ix - T(x0);
    c.ix = ix;
    c.ix0 = x0;
    c.x0 = std::min(W - 1, std::max(x0, 0));
    c.x1 = std::min(W - 1, std::max(x1, 0));
    return c;
}

// grid [N, C, H, W]
template <typename T>
static void gs2_fwd(const T* grid, int64_t C, int H, int W, int64_t n, T u, T v, T* out)
{
    auto c = corners2<T>(u, v, H, W);
    const T* g = grid + n * C * H * W;
    for (int64_t ch = 0; ch < C; ++ch) {
        const T* gc = g + ch * H * W;
        T acc = 0;
        acc += gc[c.y0 * W + c.x0] * c.w_nw;
        acc += gc[c.y0 * W + c.x1] * c.w_ne;
        acc += gc[c.y1 * W + c.x0] * c.w_sw;
        acc += gc[c.y1 * W + c.x1] * c.w_se;
        out[ch] = acc;
    }
}

// Backward of the 2D gather: IndirectGridSample2D.cu:175-393.
template <typename T>
static void gs2_bwd(const T* grid, int64_t C, int H, int W, int64_t n, T u, T v, const T* gout, T* ggrid,
                    T* gu, T* gv)
{
    auto c = corners2<T>(u, v, H, W);
    const T* g = grid + n * C * H * W;
    T* gg = ggrid ? ggrid + n * C * H * W : nullptr;
    T gix = 0, giy = 0;
    T ix = c.ix, iy = c.iy;
    T fx0 = T(c.ix0), fx1 = T(c.ix0 + 1), fy0 = T(c.iy0), fy1 = T(c.iy0 + 1);
    for (int64_t ch = 0; ch < C; ++ch) {
        T go = gout[ch];
        const T* gc = g + ch * H * W;
        if (gg) {
            T* ggc = gg + ch * H * W;
            ggc[c.y0 * W + c.x0] += c.w_nw * go;
            ggc[c.y0 * W + c.x1] += c.w_ne * go;
            ggc[c.y1 * W + c.x0] += c.w_sw * go;
            ggc[c.y1 * W + c.x1] += c.w_se * go;
        }
        T v_nw = gc[c.y0 * W + c.x0], v_ne = gc[c.y0 * W + c.x1];
        T v_sw = gc[c.y1 * W + c.x0], v_se = gc[c.y1 * W + c.x1];
        gix += T(-1) * v_nw * (fy1 - iy) * go;
        gix += v_ne * (fy1 - iy) * go;
        gix += T(-1) * v_sw * (iy - fy0) * go;
        gix += v_se * (iy - fy0) * go;
        giy += T(-1) * v_nw * (fx1 - ix) * go;
        giy += T(-1) * v_ne * (ix - fx0) * go;
        giy += v_sw * (fx1 - ix) * go;
        giy += v_se * (ix - fx0) * go;
    }
    *gu += gix * T(W - 1) / T(2);
    *gv += giy * T(H - 1) / T(2);
}

// line [N, C, W, 1]
template <typename T>
static void gs1_fwd(const T* grid, int64_t C, int W, int64_t n, T u, T* out)
{
    auto c = corners1<T>(u, W);
    const T* g = grid + n * C * W;
    for (int64_t ch = 0; ch < C; ++ch) {
        T acc = 0;
        acc += g[ch * W + c.x0] * c.w0;
        acc += g[ch * W + c.x1] * c.w1;
        out[ch] = acc;
    }
}

// Backward of the 1D gather: IndirectGridSample1D.cu:80-140.
template <typename T>
static void gs1_bwd(const T* grid, int64_t C, int W, int64_t n, T u, const T* gout, T* ggrid, T* gu)
{
    auto c = corners1<T>(u, W);
    const T* g = grid + n * C * W;
    T* gg = ggrid ? ggrid + n * C * W : nullptr;
    T gix = 0;
    T fx0 = T(c.ix0), fx1 = T(c.ix0 + 1);
    for (int64_t ch = 0; ch < C; ++ch) {
        T go = gout[ch];
        if (gg) {
            gg[ch * W + c.x0] += c.w0 * go;
            gg[ch * W + c.x1] += c.w1 * go;
        }
        T v0 = g[ch * W + c.x0], v1 = g[ch * W + c.x1];
        gix += T(-1) * v0 * (fx1 - c.ix) * go;
        gix += v1 * (c.ix - fx0) * go;
    }
    *gu += gix * T(W - 1) / T(2);
}

// Field description (reference layouts, element type T).
template <typename T>
struct Field {
    int C;
    int cat;  // 0: "add" (F = C), 1: "cat" (F = 3C)
    const T* plane[3];  // yz, xz, xy : [Nslot, C, H, W]
    int ph[3], pw[3];
    const T* line[3];  // x, y, z : [1, C, L, 1]
    int ll[3];
    const int64_t* leaf_slot;  // node -> plane slot, -1 outside the ROI
    const float* pmin;
    const float* pmax;
    float roi_min[3], roi_max[3];
};

// Coordinates fed to the six gathers of one sample:
// hyperacorn/csrc/geometry/geometry_tensor_qo.cpp:280-298. Planes use
// leaf-local (y,z), (x,z), (x,y); the x line the ROI-normalised global x, the
// y line the leaf-local y, the z line the raw global z.
template <typename T>
struct SampleCoords {
    T pu[3], pv[3];
    T lu[3];
};

template <typename T>
static SampleCoords<T> sample_coords(const Field<T>& f, const float* pos, int64_t node)
{
    T loc[3];
    for (int k = 0; k < 3; ++k) {
        T mn = (T)f.pmin[3 * node + k], mx = (T)f.pmax[3 * node + k];
        T size = mx - mn;
        T a = (T)pos[k] - mn;
        T b = a / size;
        T c = b * T(2);
        loc[k] = c - T(1);
    }
    SampleCoords<T> s;
    s.pu[0] = loc[1];
    s.pv[0] = loc[2];
    s.pu[1] = loc[0];
    s.pv[1] = loc[2];
    s.pu[2] = loc[0];
    s.pv[2] = loc[1];
    T gx = (T)pos[0];
    T a = gx - (T)f.roi_min[0];
    T b = T(2) * a;
    T range = (T)f.roi_max[0] - (T)f.roi_min[0];
    s.lu[0] = b / range - T(1);
    s.lu[1] = loc[1];
    s.lu[2] = (T)pos[2];
    return s;
}

template <typename T>
static inline int field_F(const Field<T>& f)
{
    return f.cat ? 3 * f.C : f.C;
}

// VM feature of one sample: geometry_tensor_qo.cpp:302-327 ("cat" and "add").
template <typename T>
static void field_feature(const Field<T>& f, const float* pos, int64_t node, T* out)
{
    int C = f.C;
    int F = field_F(f);
    int64_t slot = f.leaf_slot[node];
    if (slot < 0) {
        for (int i = 0; i < F; ++i) out[i] = 0;
        return;
    }
    auto s = sample_coords(f, pos, node);
    std::vector<T> mat(C), vec(C);
    for (int m = 0; m < 3; ++m) {
        gs2_fwd<T>(f.plane[m], C, f.ph[m], f.pw[m], slot, s.pu[m], s.pv[m], mat.data());
        gs1_fwd<T>(f.line[m], C, f.ll[m], 0, s.lu[m], vec.data());
        for (int c = 0; c < C; ++c) {
            T prod = mat[c] * vec[c];
            if (f.cat)
                out[m * C + c] = prod;
            else if (m == 0)
                out[c] = prod;
            else
                out[c] = out[c] + prod;
        }
    }
}

// Adjoint of field_feature for one sample: accumulates plane / line grads.
template <typename T>
static void field_feature_bwd(const Field<T>& f, const float* pos, int64_t node, const T* gfeat, T* const* gplane,
                              T* const* gline)
{
    int C = f.C;
    int64_t slot = f.leaf_slot[node];
    if (slot < 0) return;
    auto s = sample_coords(f, pos, node);
    std::vector<T> mat(C), vec(C), gm(C), gv(C);
    for (int m = 0; m < 3; ++m) {
        gs2_fwd<T>(f.plane[m], C, f.ph[m], f.pw[m], slot, s.pu[m], s.pv[m], mat.data());
        gs1_fwd<T>(f.line[m], C, f.ll[m], 0, s.lu[m], vec.data());
        for (int c = 0; c < C; ++c) {
            T g = f.cat ? gfeat[m * C + c] : gfeat[c];
            gm[c] = g * vec[c];
            gv[c] = g * mat[c];
        }
        T du = 0, dv = 0, dl = 0;
        gs2_bwd<T>(f.plane[m], C, f.ph[m], f.pw[m], slot, s.pu[m], s.pv[m], gm.data(), gplane[m], &du, &dv);
        gs1_bwd<T>(f.line[m], C, f.ll[m], 0, s.lu[m], gv.data(), gline[m], &dl);
    }
}

// Decoder: hyperacorn/csrc/geometry/Modules.h:23-149 (FCBlock: torch Linear
// layers y = x W^T + b, hidden activation after every layer but the last) and
// hyperacorn/csrc/geometry/geometry.cpp:176-253 (DecodeFeatures: last
// activation, softplus with beta and torch's threshold 20).
template <typename T>
struct Mlp {
    int n_layers;
    const int* dims;  // n_layers + 1
    const T* const* W;  // W[l] : [dims[l+1], dims[l]]
    const T* const* b;  // b[l] : [dims[l+1]]
    int act;
    int last_act;
    T beta;
};

template <typename T>
static inline T sigm(T x)
{
    return T(1) / (T(1) + std::exp(-x));
}

template <typename T>
static inline T act_fwd(int a, T x, T beta)
{
    switch (a) {
        case ORC_ACT_RELU: return x > 0 ? x : T(0);
        case ORC_ACT_SILU: return x * sigm(x);
        case ORC_ACT_SIGMOID: return sigm(x);
        case ORC_ACT_SOFTPLUS: return (x * beta > T(20)) ? x : std::log1p(std::exp(x * beta)) / beta;
        case ORC_ACT_LEAKYRELU: return x > 0 ? x : x * T(0.01);
        case ORC_ACT_ABS: return std::abs(x);
        case ORC_ACT_TANH: return std::tanh(x);
        default: return x;
    }
}

// d act / d x evaluated at the pre-activation x.
template <typename T>
static inline T act_grad(int a, T x, T beta)
{
    switch (a) {
        case ORC_ACT_RELU: return x > 0 ? T(1) : T(0);
        case ORC_ACT_SILU: {
            T s = sigm(x);
            return s * (T(1) + x * (T(1) - s));
        }
        case ORC_ACT_SIGMOID: {
            T s = sigm(x);
            return s * (T(1) - s);
        }
        case ORC_ACT_SOFTPLUS: {
            if (x * beta > T(20)) return T(1);
            T z = std::exp(x * beta);
            return z / (z + T(1));
        }
        case ORC_ACT_LEAKYRELU: return x > 0 ? T(1) : T(0.01);
        case ORC_ACT_ABS: return x > 0 ? T(1) : (x < 0 ? T(-1) : T(0));
        case ORC_ACT_TANH: {
            T t = std::tanh(x);
            return T(1) - t * t;
        }
        default: return T(1);
    }
}

// Forward of one row; keeps the pre-activations of every layer in pre
// (concatenated, size sum(dims[1..])).
template <typename T>
static void mlp_row(const Mlp<T>& m, const T* x, T* pre, T* out)
{
    std::vector<T> cur(x, x + m.dims[0]), nxt;
    int64_t po = 0;
    for (int l = 0; l < m.n_layers; ++l) {
        int in = m.dims[l], on = m.dims[l + 1];
        nxt.assign(on, 0);
        for (int o = 0; o < on; ++o) {
            T acc = 0;
            for (int i = 0; i < in; ++i) acc += cur[i] * m.W[l][o * in + i];
            acc += m.b[l][o];
            if (pre) pre[po + o] = acc;
            bool last = (l == m.n_layers - 1);
            nxt[o] = last ? act_fwd<T>(m.last_act, acc, m.beta) : act_fwd<T>(m.act, acc, m.beta);
        }
        po += on;
        cur.swap(nxt);
    }
    for (int o = 0; o < m.dims[m.n_layers]; ++o) out[o] = cur[o];
}

// Backward of one row: accumulates dW, db and writes dx.
template <typename T>
static void mlp_row_bwd(const Mlp<T>& m, const T* x, const T* gout, T* const* dW, T* const* db, T* dx)
{
    int64_t total = 0;
    for (int l = 1; l <= m.n_layers; ++l) total += m.dims[l];
    std::vector<T> pre(total), outv(m.dims[m.n_layers]);
    mlp_row(m, x, pre.data(), outv.data());
    std::vector<int64_t> po(m.n_layers + 1, 0);
    for (int l = 0; l < m.n_layers; ++l) po[l + 1] = po[l] + m.dims[l + 1];
    std::vector<T> g(gout, gout + m.dims[m.n_layers]);
    for (int l = m.n_layers - 1; l >= 0; --l) {
        int in = m.dims[l], on = m.dims[l + 1];
        bool last = (l == m.n_layers - 1);
        std::vector<T> gpre(on);
        for (int o = 0; o < on; ++o) gpre[o] = g[o] * act_grad<T>(last ? m.last_act : m.act, pre[po[l] + o], m.beta);
        // input of this layer
        std::vector<T> inp(in);
        if (l == 0) {
            for (int i = 0; i < in; ++i) inp[i] = x[i];
        } else {
            for (int i = 0; i < in; ++i) inp[i] = act_fwd<T>(m.act, pre[po[l - 1] + i], m.beta);
        }
        if (dW)
            for (int o = 0; o < on; ++o)
                for (int i = 0; i < in; ++i) dW[l][o * in + i] += gpre[o] * inp[i];
        if (db)
            for (int o = 0; o < on; ++o) db[l][o] += gpre[o];
        std::vector<T> gin(in, 0);
        for (int o = 0; o < on; ++o)
            for (int i = 0; i < in; ++i) gin[i] += gpre[o] * m.W[l][o * in + i];
        g.swap(gin);
    }
    if (dx)
        for (int i = 0; i < m.dims[0]; ++i) dx[i] = g[i];
}

template <typename T>
static Field<T> make_field(int C, int cat, const T* const* planes, const int* ph, const int* pw, const T* const* lines,
                           const int* ll, const int64_t* leaf_slot, const float* pmin, const float* pmax,
                           const float* roi_min, const float* roi_max)
{
    Field<T> f;
    f.C = C;
    f.cat = cat;
    for (int m = 0; m < 3; ++m) {
        f.plane[m] = planes[m];
        f.ph[m] = ph[m];
        f.pw[m] = pw[m];
        f.line[m] = lines[m];
        f.ll[m] = ll[m];
        f.roi_min[m] = roi_min[m];
        f.roi_max[m] = roi_max[m];
    }
    f.leaf_slot = leaf_slot;
    f.pmin = pmin;
    f.pmax = pmax;
    return f;
}

template <typename T>
static Mlp<T> make_mlp(int n_layers, const int* dims, const T* const* W, const T* const* b, int act, int last_act,
                       double beta)
{
    Mlp<T> m;
    m.n_layers = n_layers;
    m.dims = dims;
    m.W = W;
    m.b = b;
    m.act = act;
    m.last_act = last_act;
    m.beta = (T)beta;
    return m;
}

// Line integral: hyperacorn/csrc/geometry/geometry.cpp:977-1019
// (IntegrateSamplesXRay): I[c, ray] += value[s, c] * weight[s].
template <typename T>
static void project_fwd(const Field<T>& f, const Mlp<T>& m, int64_t S, const float* pos, const float* w,
                        const int64_t* ray, const int64_t* node, int64_t R, T* image)
{
    int F = field_F(f);
    int Co = m.dims[m.n_layers];
    for (int64_t i = 0; i < Co * R; ++i) image[i] = 0;
    std::vector<T> feat(F), out(Co);
    for (int64_t s = 0; s < S; ++s) {
        field_feature<T>(f, pos + 3 * s, node[s], feat.data());
        mlp_row<T>(m, feat.data(), nullptr, out.data());
        for (int c = 0; c < Co; ++c) {
            T v = out[c] * (T)w[s];
            image[c * R + ray[s]] += v;
        }
    }
}

// Adjoint of project_fwd given dL/dimage: the autograd chain of the reference
// (index_add_^T = gather, mul, DecodeFeatures, FCBlock, the VM products and the
// two gather ops' backward kernels).
template <typename T>
static void project_bwd(const Field<T>& f, const Mlp<T>& m, int64_t S, const float* pos, const float* w,
                        const int64_t* ray, const int64_t* node, int64_t R, const T* gimage, T* const* gplane,
                        T* const* gline, T* const* dW, T* const* db)
{
    int F = field_F(f);
    int Co = m.dims[m.n_layers];
    std::vector<T> feat(F), gout(Co), gfeat(F);
    for (int64_t s = 0; s < S; ++s) {
        field_feature<T>(f, pos + 3 * s, node[s], feat.data());
        for (int c = 0; c < Co; ++c) gout[c] = gimage[c * R + ray[s]] * (T)w[s];
        mlp_row_bwd<T>(m, feat.data(), gout.data(), dW, db, gfeat.data());
        field_feature_bwd<T>(f, pos + 3 * s, node[s], gfeat.data(), gplane, gline);
    }
}

#define ORC_FIELD_ARGS(T)                                                                                       \
    int C, int cat, const T* const *planes, const int *ph, const int *pw, const T *const *lines, const int *ll, \
        const int64_t *leaf_slot, const float *pmin, const float *pmax, const float *roi_min, const float *roi_max
#define ORC_FIELD_PASS C, cat, planes, ph, pw, lines, ll, leaf_slot, pmin, pmax, roi_min, roi_max
#define ORC_MLP_ARGS(T) \
    int n_layers, const int *dims, const T *const *W, const T *const *b, int act, int last_act, double beta
#define ORC_MLP_PASS n_layers, dims, W, b, act, last_act, beta

#define ORC_INSTANTIATE(T, SUF)                                                                                      \
    extern "C" void orc_grid_sample2d_fwd_##SUF(const T* grid, int64_t N, int64_t C, int H, int W,                  \
                                                const int64_t* index, const T* uv, int64_t S, T* out)               \
    {                                                                                                                \
        (void)N;                                                                                                     \
        _Pragma("omp parallel for") for (int64_t i = 0; i < S; ++i)                                                  \
            gs2_fwd<T>(grid, C, H, W, index[i], uv[2 * i], uv[2 * i + 1], out + i * C);                              \
    }                                                                                                                \
    extern "C" void orc_grid_sample2d_bwd_##SUF(const T* grid, int64_t N, int64_t C, int H, int W,                  \
                                                const int64_t* index, const T* uv, int64_t S, const T* gout,        \
                                                T* ggrid, T* guv)                                                    \
    {                                                                                                                \
        (void)N;                                                                                                     \
        for (int64_t i = 0; i < S; ++i)                                                                              \
            gs2_bwd<T>(grid, C, H, W, index[i], uv[2 * i], uv[2 * i + 1], gout + i * C, ggrid, guv + 2 * i,          \
                       guv + 2 * i + 1);                                                                             \
    }                                                                                                                \
    extern "C" void orc_grid_sample1d_fwd_##SUF(const T* grid, int64_t N, int64_t C, int W, const int64_t* index,   \
                                                const T* uv, int64_t S, T* out)                                      \
    {                                                                                                                \
        (void)N;                                                                                                     \
        _Pragma("omp parallel for") for (int64_t i = 0; i < S; ++i)                                                  \
            gs1_fwd<T>(grid, C, W, index[i], uv[i], out + i * C);                                                    \
    }                                                                                                                \
    extern "C" void orc_grid_sample1d_bwd_##SUF(const T* grid, int64_t N, int64_t C, int W, const int64_t* index,   \
                                                const T* uv, int64_t S, const T* gout, T* ggrid, T* guv)             \
    {                                                                                                                \
        (void)N;                                                                                                     \
        for (int64_t i = 0; i < S; ++i) gs1_bwd<T>(grid, C, W, index[i], uv[i], gout + i * C, ggrid, guv + i);      \
    }                                                                                                                \
    extern "C" void orc_vm_features_##SUF(ORC_FIELD_ARGS(T), int64_t S, const float* pos, const int64_t* node, T* out)  \
    {                                                                                                                \
        auto f = make_field<T>(ORC_FIELD_PASS);                                                                      \
        int F = field_F(f);                                                                                          \
        _Pragma("omp parallel for") for (int64_t s = 0; s < S; ++s)                                                  \
            field_feature<T>(f, pos + 3 * s, node[s], out + s * F);                                                  \
    }                                                                                                                \
    extern "C" void orc_vm_features_bwd_##SUF(ORC_FIELD_ARGS(T), int64_t S, const float* pos, const int64_t* node,      \
                                              const T* gout, T* const* gplane, T* const* gline)                      \
    {                                                                                                                \
        auto f = make_field<T>(ORC_FIELD_PASS);                                                                      \
        int F = field_F(f);                                                                                          \
        for (int64_t s = 0; s < S; ++s) field_feature_bwd<T>(f, pos + 3 * s, node[s], gout + s * F, gplane, gline); \
    }                                                                                                                \
    extern "C" void orc_mlp_fwd_##SUF(ORC_MLP_ARGS(T), int64_t S, const T* x, T* out)                                  \
    {                                                                                                                \
        auto m = make_mlp<T>(ORC_MLP_PASS);                                                                          \
        int in = dims[0], on = dims[n_layers];                                                                       \
        _Pragma("omp parallel for") for (int64_t s = 0; s < S; ++s)                                                  \
            mlp_row<T>(m, x + s * in, nullptr, out + s * on);                                                        \
    }                                                                                                                \
    extern "C" void orc_mlp_bwd_##SUF(ORC_MLP_ARGS(T), int64_t S, const T* x, const T* gout, T* const* dW,             \
                                      T* const* db, T* dx)                                                           \
    {                                                                                                                \
        auto m = make_mlp<T>(ORC_MLP_PASS);                                                                          \
        int in = dims[0], on = dims[n_layers];                                                                       \
        for (int64_t s = 0; s < S; ++s)                                                                              \
            mlp_row_bwd<T>(m, x + s * in, gout + s * on, dW, db, dx ? dx + s * in : nullptr);                        \
    }                                                                                                                \
    extern "C" void orc_project_fwd_##SUF(ORC_FIELD_ARGS(T), ORC_MLP_ARGS(T), int64_t S, const float* pos,                 \
                                          const float* w, const int64_t* ray, const int64_t* node, int64_t R,        \
                                          T* image)                                                                  \
    {                                                                                                                \
        auto f = make_field<T>(ORC_FIELD_PASS);                                                                      \
        auto m = make_mlp<T>(ORC_MLP_PASS);                                                                          \
        project_fwd<T>(f, m, S, pos, w, ray, node, R, image);                                                        \
    }                                                                                                                \
    extern "C" void orc_project_bwd_##SUF(ORC_FIELD_ARGS(T), ORC_MLP_ARGS(T), int64_t S, const float* pos,                 \
                                          const float* w, const int64_t* ray, const int64_t* node, int64_t R,        \
                                          const T* gimage, T* const* gplane, T* const* gline, T* const* dW,          \
                                          T* const* db)                                                              \
    {                                                                                                                \
        auto f = make_field<T>(ORC_FIELD_PASS);                                                                      \
        auto m = make_mlp<T>(ORC_MLP_PASS);                                                                          \
        project_bwd<T>(f, m, S, pos, w, ray, node, R, gimage, gplane, gline, dW, db);                                \
    }

ORC_INSTANTIATE(float, f32)
ORC_INSTANTIATE(double, f64)

// ---------------------------------------------------------------------------
// One plain-method training step on the CPU (fwd + MSE loss + bwd), the timed
// CPU baseline: segments and samples of every ray (interval jitter from
// orc_jitter keyed by seed, or the midpoint when seed == 0), the field and
// decoder per sample, the line integral per ray, loss = mean((I - y)^2) and the
// adjoint into zero-initialised gradient buffers. Rays are processed in
// parallel with one private gradient copy per thread, reduced at the end.
// Returns the loss; writes the image [Co, R].
// ---------------------------------------------------------------------------
template <typename T>
static double train_step(const float* pmin, const float* pmax, const int64_t* active, int64_t A, const float* origin,
                         const float* dir, const float* target, int64_t R, int M, uint64_t seed, const Field<T>& f,
                         const Mlp<T>& m, const int64_t* plane_numel, const int64_t* line_numel, T* image,
                         T* const* gplane, T* const* gline, T* const* dW, T* const* db)
{
    int F = field_F(f);
    int Co = m.dims[m.n_layers];
    // forward, ray-parallel
    std::vector<std::vector<float>> spos(R), sw(R);
    std::vector<std::vector<int64_t>> snode(R);
#pragma omp parallel
    {
        std::vector<Hit> hits;
        std::vector<T> feat(F), out(Co);
        std::vector<float> ts;
#pragma omp for schedule(dynamic, 8)
        for (int64_t r = 0; r < R; ++r) {
            const float* o = origin + 3 * r;
            const float* d = dir + 3 * r;
            ray_hits(pmin, pmax, active, A, o, d, M, hits);
            auto& P = spos[r];
            auto& W = sw[r];
            auto& N = snode[r];
            P.clear();
            W.clear();
            N.clear();
            for (auto& h : hits) {
                ts.resize(h.n);
                for (int j = 0; j < h.n; ++j) {
                    float a = seed ? orc_jitter(seed, (int32_t)r, h.node, j) : 0.5f;
                    ts[j] = sample_t(h.tmin, h.tmax, h.n, j, a);
                }
                for (int j = 0; j < h.n; ++j) {
                    float t = ts[j];
                    float lo = (j == 0) ? h.tmin : (ts[j - 1] + t) * 0.5f;
                    float hi = (j == h.n - 1) ? h.tmax : (ts[j + 1] + t) * 0.5f;
                    W.push_back(hi - lo);
                    for (int k = 0; k < 3; ++k) P.push_back(o[k] + d[k] * t);
                    N.push_back(h.node);
                }
            }
            for (int c = 0; c < Co; ++c) image[c * R + r] = 0;
            for (size_t s = 0; s < W.size(); ++s) {
                field_feature<T>(f, &P[3 * s], N[s], feat.data());
                mlp_row<T>(m, feat.data(), nullptr, out.data());
                for (int c = 0; c < Co; ++c) image[c * R + r] += out[c] * (T)W[s];
            }
        }
    }
    double loss = 0;
    std::vector<T> gimage(Co * R);
    for (int64_t i = 0; i < Co * R; ++i) {
        double diff = (double)image[i] - (double)target[i];
        loss += diff * diff;
        gimage[i] = (T)(2.0 * diff / (double)(Co * R));
    }
    loss /= (double)(Co * R);
    // backward, ray-parallel with private gradients
    int nthreads = 1;
#pragma omp parallel
    {
#pragma omp single
        {
#ifdef _OPENMP
            nthreads = omp_get_num_threads();
#endif
        }
    }
    int64_t pn[3] = {plane_numel[0], plane_numel[1], plane_numel[2]};
    int64_t ln[3] = {line_numel[0], line_numel[1], line_numel[2]};
    std::vector<int64_t> wn(m.n_layers), bn(m.n_layers);
    for (int l = 0; l < m.n_layers; ++l) {
        wn[l] = (int64_t)m.dims[l] * m.dims[l + 1];
        bn[l] = m.dims[l + 1];
    }
    std::vector<std::vector<T>> priv(nthreads);
    int64_t tot = 0;
    for (int k = 0; k < 3; ++k) tot += pn[k] + ln[k];
    for (int l = 0; l < m.n_layers; ++l) tot += wn[l] + bn[l];
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        auto& buf = priv[tid];
        buf.assign(tot, T(0));
        std::vector<T*> gp(3), gl(3), gW(m.n_layers), gb(m.n_layers);
        T* p = buf.data();
        for (int k = 0; k < 3; ++k) {
            gp[k] = p;
            p += pn[k];
        }
        for (int k = 0; k < 3; ++k) {
            gl[k] = p;
            p += ln[k];
        }
        for (int l = 0; l < m.n_layers; ++l) {
            gW[l] = p;
            p += wn[l];
            gb[l] = p;
            p += bn[l];
        }
        std::vector<T> feat(F), gout(Co), gfeat(F);
#pragma omp for schedule(dynamic, 8)
        for (int64_t r = 0; r < R; ++r) {
            auto& P = spos[r];
            auto& W = sw[r];
            auto& N = snode[r];
            for (size_t s = 0; s < W.size(); ++s) {
                field_feature<T>(f, &P[3 * s], N[s], feat.data());
                for (int c = 0; c < Co; ++c) gout[c] = gimage[c * R + r] * (T)W[s];
                mlp_row_bwd<T>(m, feat.data(), gout.data(), gW.data(), gb.data(), gfeat.data());
                field_feature_bwd<T>(f, &P[3 * s], N[s], gfeat.data(), gp.data(), gl.data());
            }
        }
    }
    // reduce
    for (int th = 0; th < nthreads; ++th) {
        const T* p = priv[th].data();
        for (int k = 0; k < 3; ++k) {
            for (int64_t i = 0; i < pn[k]; ++i) gplane[k][i] += p[i];
            p += pn[k];
        }
        for (int k = 0; k < 3; ++k) {
            for (int64_t i = 0; i < ln[k]; ++i) gline[k][i] += p[i];
            p += ln[k];
        }
        for (int l = 0; l < m.n_layers; ++l) {
            for (int64_t i = 0; i < wn[l]; ++i) dW[l][i] += p[i];
            p += wn[l];
            for (int64_t i = 0; i < bn[l]; ++i) db[l][i] += p[i];
            p += bn[l];
        }
    }
    return loss;
}

extern "C" double orc_train_step_f32(const float* pmin, const float* pmax, const int64_t* active, int64_t A,
                                     const float* origin, const float* dir, const float* target, int64_t R, int M,
                                     uint64_t seed, int C, int cat, const float* const* planes, const int* ph,
                                     const int* pw, const float* const* lines, const int* ll,
                                     const int64_t* leaf_slot, const float* roi_min, const float* roi_max,
                                     int n_layers, const int* dims, const float* const* W, const float* const* b,
                                     int act, int last_act, double beta, const int64_t* plane_numel,
                                     const int64_t* line_numel, float* image, float* const* gplane,
                                     float* const* gline, float* const* dW, float* const* db)
{
    auto f = make_field<float>(C, cat, planes, ph, pw, lines, ll, leaf_slot, pmin, pmax, roi_min, roi_max);
    auto m = make_mlp<float>(n_layers, dims, W, b, act, last_act, beta);
    return train_step<float>(pmin, pmax, active, A, origin, dir, target, R, M, seed, f, m, plane_numel, line_numel,
                             image, gplane, gline, dW, db);
}

extern "C" int orc_num_threads()
{
    int n = 1;
#ifdef _OPENMP
    n = omp_get_max_threads();
#endif
    return n;
}

// ---------------------------------------------------------------------------
// Node-error scoring: hyperacorn/csrc/geometry/geometry.cpp:33-53
// (AccumulateSampleLossPerNode): per-ray loss averaged over channels, gathered
// by ray index, times the sample weight, scattered into per-node sums of loss
// and of weight. Accumulated in double.
// ---------------------------------------------------------------------------
extern "C" void orc_accumulate_loss_per_node(int64_t S, const int64_t* ray, const int64_t* node, const float* w,
                                             const float* per_ray_loss, int64_t C, int64_t R, int64_t num_nodes,
                                             double* loss_sum, double* weight_sum)
{
    for (int64_t i = 0; i < num_nodes; ++i) {
        loss_sum[i] = 0;
        weight_sum[i] = 0;
    }
    for (int64_t s = 0; s < S; ++s) {
        double l = 0;
        for (int64_t c = 0; c < C; ++c) l += (double)per_ray_loss[c * R + ray[s]];
        l /= (double)C;
        loss_sum[node[s]] += l * (double)w[s];
        weight_sum[node[s]] += (double)w[s];
    }
}
