// ORACLE — test infrastructure only (see oracle_core.hpp). Restates
// crates/core/src/bvh.rs (binned SAH, traversal) and crates/core/src/lbvh.rs.
#include "oracle_scene.hpp"
#include <algorithm>
#include <numeric>
#include <sstream>

namespace oracle {

Aabb triangle_bounds(const GpuTriangle& t, const float* pos) {  // bvh.rs:202-210
    Aabb b;
    uint32_t idx[3] = {t.i0, t.i1, t.i2};
    for (uint32_t i : idx) b.grow_point(Vec3(pos[4 * i], pos[4 * i + 1], pos[4 * i + 2]));
    b.pad();
    return b;
}

static const int BINS = 12;
static const float TRAVERSAL_COST = 1.0f, INTERSECT_COST = 1.0f;
static const size_t MIN_LEAF = 2;

static inline size_t bin_index(float c, float axis_min, float scale) {  // bvh.rs:608-612
    return std::min<size_t>((size_t)f2usize((c - axis_min) * scale), BINS - 1);
}

Bvh Bvh::build(const std::vector<GpuTriangle>& tris, const std::vector<float>& pos) {
    std::vector<Aabb> b(tris.size());
    for (size_t i = 0; i < tris.size(); ++i) b[i] = triangle_bounds(tris[i], pos.data());
    return build_over_bounds(b);
}

// bvh.rs:245-459
Bvh Bvh::build_over_bounds(const std::vector<Aabb>& bounds_in) {
    Bvh out;
    if (bounds_in.empty()) return out;
    size_t n = bounds_in.size();
    std::vector<Vec3> centroid(n);
    for (size_t i = 0; i < n; ++i) centroid[i] = bounds_in[i].centroid();
    std::vector<uint32_t> pi(n);
    for (size_t i = 0; i < n; ++i) pi[i] = (uint32_t)i;
    std::vector<GpuBvhNode> nodes;
    nodes.reserve(2 * n);
    auto fresh = [] {
        GpuBvhNode g;
        for (int a = 0; a < 3; ++a) { g.bounds_min[a] = INFINITY; g.bounds_max[a] = -INFINITY; }
        g.left_first = 0;
        g.count = 0;
        return g;
    };
    nodes.push_back(fresh());
    struct Item { size_t node, start, count, depth; };
    std::vector<Item> stack{{0, 0, n, 0}};
    while (!stack.empty()) {
        Item it = stack.back();
        stack.pop_back();
        Aabb bounds, cb;
        for (size_t k = it.start; k < it.start + it.count; ++k) {
            bounds.grow(bounds_in[pi[k]]);
            cb.grow_point(centroid[pi[k]]);
        }
        bounds.min.to(nodes[it.node].bounds_min);
        bounds.max.to(nodes[it.node].bounds_max);
        auto make_leaf = [&] {
            nodes[it.node].left_first = (uint32_t)it.start;
            nodes[it.node].count = (uint32_t)it.count;
        };
        if (it.count <= MIN_LEAF) { make_leaf(); continue; }
        Vec3 extent = cb.max - cb.min;
        int axis = (extent.x > extent.y && extent.x > extent.z) ? 0 : (extent.y > extent.z ? 1 : 2);
        if (extent[axis] <= 0.0f) { make_leaf(); continue; }
        float scale = (float)BINS / extent[axis];
        Aabb bin_b[BINS];
        uint32_t bin_c[BINS] = {0};
        for (size_t k = it.start; k < it.start + it.count; ++k) {
            size_t b = bin_index(centroid[pi[k]][axis], cb.min[axis], scale);
            bin_c[b] += 1;
            bin_b[b].grow(bounds_in[pi[k]]);
        }
        float left_area[BINS - 1], right_area[BINS - 1];
        uint32_t left_count[BINS - 1], right_count[BINS - 1];
        Aabb acc;
        uint32_t cnt = 0;
        for (int i = 0; i < BINS - 1; ++i) {
            acc.grow(bin_b[i]);
            cnt += bin_c[i];
            left_area[i] = acc.surface_area();
            left_count[i] = cnt;
        }
        acc = Aabb();
        cnt = 0;
        for (int i = BINS - 1; i >= 1; --i) {
            acc.grow(bin_b[i]);
            cnt += bin_c[i];
            right_area[i - 1] = acc.surface_area();
            right_count[i - 1] = cnt;
        }
        float parent_area = bounds.surface_area();
        float best_cost = INFINITY;
        int best = -1;
        for (int i = 0; i < BINS - 1; ++i) {
            if (left_count[i] == 0 || right_count[i] == 0) continue;
            float cost = TRAVERSAL_COST +
                         (left_area[i] * (float)left_count[i] + right_area[i] * (float)right_count[i]) /
                             parent_area * INTERSECT_COST;
            if (cost < best_cost) { best_cost = cost; best = i; }
        }
        float leaf_cost = (float)it.count * INTERSECT_COST;
        if (best < 0 || best_cost >= leaf_cost) { make_leaf(); continue; }
        size_t split_bin = (size_t)best + 1;
        size_t i = it.start, j = it.start + it.count;
        while (i < j) {
            size_t b = bin_index(centroid[pi[i]][axis], cb.min[axis], scale);
            if (b < split_bin) {
                ++i;
            } else {
                --j;
                std::swap(pi[i], pi[j]);
            }
        }
        size_t left_n = i - it.start;
        size_t left_idx = nodes.size();
        nodes.push_back(fresh());
        nodes.push_back(fresh());
        nodes[it.node].left_first = (uint32_t)left_idx;
        nodes[it.node].count = 0;
        stack.push_back({left_idx, it.start, left_n, it.depth + 1});
        stack.push_back({left_idx + 1, it.start + left_n, it.count - left_n, it.depth + 1});
    }
    out.nodes = std::move(nodes);
    out.prim_indices = std::move(pi);
    return out;
}

float Bvh::sah_cost() const {  // bvh.rs:470-493
    if (nodes.empty()) return 0.0f;
    float root_area = node_aabb(nodes[0]).surface_area();
    if (root_area <= 0.0f) return 0.0f;
    float total = 0.0f;
    for (const GpuBvhNode& n : nodes) {
        float area = node_aabb(n).surface_area();
        float own = n.count == 0 ? TRAVERSAL_COST : (float)n.count * INTERSECT_COST;
        total += area / root_area * own;
    }
    return total;
}

void Bvh::compact_primitives(std::vector<GpuTriangle>& tris) {  // bvh.rs:517-528
    std::vector<GpuTriangle> re(tris.size());
    for (size_t i = 0; i < prim_indices.size(); ++i) re[i] = tris[prim_indices[i]];
    tris = re;
    for (size_t i = 0; i < prim_indices.size(); ++i) prim_indices[i] = (uint32_t)i;
}

std::vector<std::string> Bvh::validate(size_t tc) const {  // bvh.rs:544-606
    std::vector<std::string> problems;
    if (nodes.empty()) {
        if (tc > 0) problems.push_back("triangles but no nodes");
        return problems;
    }
    std::vector<uint32_t> seen(tc, 0);
    for (size_t i = 0; i < nodes.size(); ++i) {
        const GpuBvhNode& n = nodes[i];
        if (n.count == 0) {
            size_t l = n.left_first;
            if (l + 1 >= nodes.size()) { problems.push_back("out-of-range children"); continue; }
            Aabb p = node_aabb(n);
            float eps = 1e-3f * fmax_(std::sqrt(p.surface_area()), 1.0f);
            for (size_t c : {l, l + 1}) {
                Aabb cbx = node_aabb(nodes[c]);
                bool ok = cbx.is_empty() ||
                          (p.min.x <= cbx.min.x + eps && p.min.y <= cbx.min.y + eps &&
                           p.min.z <= cbx.min.z + eps && p.max.x >= cbx.max.x - eps &&
                           p.max.y >= cbx.max.y - eps && p.max.z >= cbx.max.z - eps);
                if (!ok) {
                    std::ostringstream os;
                    os << "node " << i << " does not contain child " << c;
                    problems.push_back(os.str());
                }
            }
        } else {
            size_t s = n.left_first, e = s + n.count;
            if (e > prim_indices.size()) { problems.push_back("leaf range out of bounds"); continue; }
            for (size_t k = s; k < e; ++k) {
                if (prim_indices[k] >= tc) problems.push_back("leaf references out-of-range prim");
                else seen[prim_indices[k]] += 1;
            }
        }
    }
    size_t missing = 0, dup = 0;
    for (uint32_t c : seen) { missing += c == 0; dup += c > 1; }
    if (missing) problems.push_back(std::to_string(missing) + " triangles are in no leaf");
    if (dup) problems.push_back(std::to_string(dup) + " triangles appear in more than one leaf");
    return problems;
}

static inline void tri_pos(const GpuTriangle& t, const float* pos, Vec3& a, Vec3& b, Vec3& c) {
    a = Vec3(pos[4 * t.i0], pos[4 * t.i0 + 1], pos[4 * t.i0 + 2]);
    b = Vec3(pos[4 * t.i1], pos[4 * t.i1 + 1], pos[4 * t.i1 + 2]);
    c = Vec3(pos[4 * t.i2], pos[4 * t.i2 + 1], pos[4 * t.i2 + 2]);
}

bool brute_force_intersect(const GpuTriangle* tris, size_t n, const float* pos, const Ray& ray,
                           float tmin, float tmax, TriHit& out) {  // bvh.rs:975-997
    bool found = false;
    float closest = tmax;
    for (size_t i = 0; i < n; ++i) {
        Vec3 a, b, c;
        tri_pos(tris[i], pos, a, b, c);
        float t, u, v;
        if (intersect_triangle(a, b, c, ray, tmin, closest, t, u, v)) {
            closest = t;
            out = TriHit{t, u, v, (uint32_t)i};
            found = true;
        }
    }
    return found;
}

static const size_t MAX_STACK = 64;

// bvh.rs:1045-1130
bool Bvh::intersect(const GpuTriangle* tris, const float* pos, const Ray& ray, float tmin,
                    float tmax, TraversalStats& st, TriHit& out) const {
    if (nodes.empty()) return false;
    Vec3 inv = safe_inv_dir(ray.dir);
    bool found = false;
    float closest = tmax;
    uint32_t stack[MAX_STACK];
    size_t sp = 0;
    uint32_t node = 0;
    for (;;) {
        const GpuBvhNode& n = nodes[node];
        st.node_visits += 1;
        if (n.count > 0) {
            for (uint32_t k = n.left_first; k < n.left_first + n.count; ++k) {
                uint32_t p = prim_indices[k];
                Vec3 a, b, c;
                tri_pos(tris[p], pos, a, b, c);
                st.triangle_tests += 1;
                float t, u, v;
                if (intersect_triangle(a, b, c, ray, tmin, closest, t, u, v)) {
                    closest = t;
                    out = TriHit{t, u, v, p};
                    found = true;
                }
            }
        } else {
            uint32_t c0 = n.left_first, c1 = c0 + 1;
            float d0, d1;
            bool h0 = node_aabb(nodes[c0]).hit(ray.origin, inv, tmin, closest, d0);
            bool h1 = node_aabb(nodes[c1]).hit(ray.origin, inv, tmin, closest, d1);
            if (h0 && h1) {
                uint32_t nearc = d0 <= d1 ? c0 : c1, farc = d0 <= d1 ? c1 : c0;
                if (sp < MAX_STACK) stack[sp++] = farc;
                node = nearc;
                continue;
            } else if (h0) {
                node = c0;
                continue;
            } else if (h1) {
                node = c1;
                continue;
            }
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    return found;
}

// bvh.rs:1137-1193
bool Bvh::occluded(const GpuTriangle* tris, const float* pos, const Ray& ray, float tmin,
                   float tmax) const {
    if (nodes.empty()) return false;
    Vec3 inv = safe_inv_dir(ray.dir);
    uint32_t stack[MAX_STACK];
    size_t sp = 0;
    uint32_t node = 0;
    for (;;) {
        const GpuBvhNode& n = nodes[node];
        if (n.count > 0) {
            for (uint32_t k = n.left_first; k < n.left_first + n.count; ++k) {
                Vec3 a, b, c;
                tri_pos(tris[prim_indices[k]], pos, a, b, c);
                float t, u, v;
                if (intersect_triangle(a, b, c, ray, tmin, tmax, t, u, v)) return true;
            }
        } else {
            uint32_t c0 = n.left_first, c1 = c0 + 1;
            float d;
            bool h0 = node_aabb(nodes[c0]).hit(ray.origin, inv, tmin, tmax, d);
            bool h1 = node_aabb(nodes[c1]).hit(ray.origin, inv, tmin, tmax, d);
            if (h0) {
                if (h1 && sp < MAX_STACK) stack[sp++] = c1;
                node = c0;
                continue;
            }
            if (h1) {
                node = c1;
                continue;
            }
        }
        if (sp == 0) return false;
        node = stack[--sp];
    }
}

// ---------------------------------------------------------------- lbvh.rs
uint32_t expand_bits(uint32_t v) {  // lbvh.rs:72-79
    uint32_t x = v & 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}
uint32_t morton3d(Vec3 p) {  // lbvh.rs:93-101
    const float SCALE = 1023.0f;
    auto q = [&](float v) { return f2u(clampf(v * SCALE, 0.0f, SCALE)); };
    return (expand_bits(q(p.x)) << 2) | (expand_bits(q(p.y)) << 1) | expand_bits(q(p.z));
}
Vec3 lbvh_normalise(Vec3 p, const Aabb& b) {  // lbvh.rs:109-117
    Vec3 e = b.max - b.min;
    auto f = [](float v, float lo, float ex) { return ex > 0.0f ? (v - lo) / ex : 0.5f; };
    return Vec3(f(p.x, b.min.x, e.x), f(p.y, b.min.y, e.y), f(p.z, b.min.z, e.z));
}
int32_t longest_common_prefix(const uint32_t* codes, int64_t n, int32_t i, int32_t j) {
    // lbvh.rs:149-159
    if (j < 0 || j >= n) return -1;
    uint32_t a = codes[i], b = codes[j];
    if (a == b) return 32 + leading_zeros((uint32_t)i ^ (uint32_t)j);
    return leading_zeros(a ^ b);
}

// lbvh.rs:211-292
static void build_hierarchy(const std::vector<uint32_t>& codes, std::vector<uint32_t>& karras,
                            std::vector<uint32_t>& parent) {
    int64_t n = (int64_t)codes.size();
    karras.assign(2 * (n - 1), 0);
    parent.assign(2 * n - 1, 0xFFFFFFFFu);
    uint32_t leaf_base = (uint32_t)(n - 1);
    const uint32_t* c = codes.data();
    auto delta = [&](int32_t i, int32_t j) { return longest_common_prefix(c, n, i, j); };
    for (int32_t i = 0; i < (int32_t)(n - 1); ++i) {
        int32_t dd = delta(i, i + 1) - delta(i, i - 1);
        int32_t d = (dd > 0) - (dd < 0);
        int32_t delta_min = delta(i, i - d);
        int32_t l_max = 2;
        while (delta(i, i + l_max * d) > delta_min) l_max *= 2;
        int32_t l = 0;
        for (int32_t t = l_max / 2; t >= 1; t /= 2)
            if (delta(i, i + (l + t) * d) > delta_min) l += t;
        int32_t j = i + l * d;
        int32_t first = std::min(i, j), last = std::max(i, j);
        int32_t delta_node = delta(i, j);
        int32_t s = 0, t = l;
        while (t > 1) {
            t = (t + 1) / 2;
            if (delta(i, i + (s + t) * d) > delta_node) s += t;
        }
        int32_t split = i + s * d + std::min(d, 0);
        uint32_t left = split == first ? leaf_base + (uint32_t)split : (uint32_t)split;
        uint32_t right = split + 1 == last ? leaf_base + (uint32_t)(split + 1) : (uint32_t)(split + 1);
        karras[2 * i] = left;
        karras[2 * i + 1] = right;
        parent[left] = (uint32_t)i;
        parent[right] = (uint32_t)i;
    }
}

// lbvh.rs:315-406
static void relayout(const std::vector<uint32_t>& karras, const std::vector<uint32_t>& subtree,
                     const std::vector<uint32_t>& sorted, const std::vector<Aabb>& bounds, size_t n,
                     size_t max_leaf, Bvh& out) {
    uint32_t leaf_base = (uint32_t)(n - 1);
    std::vector<GpuBvhNode>& nodes = out.nodes;
    std::vector<uint32_t>& prims = out.prim_indices;
    nodes.clear();
    prims.clear();
    auto gather = [&](uint32_t root) {
        std::vector<uint32_t> st{root};
        while (!st.empty()) {
            uint32_t id = st.back();
            st.pop_back();
            if (id >= leaf_base) {
                prims.push_back(sorted[id - leaf_base]);
            } else {
                st.push_back(karras[2 * id + 1]);
                st.push_back(karras[2 * id]);
            }
        }
    };
    auto size_of = [&](uint32_t id) -> size_t { return id >= leaf_base ? 1 : subtree[id]; };
    auto mk = [](const Aabb& b, uint32_t lf, uint32_t cnt) {
        GpuBvhNode g;
        b.min.to(g.bounds_min);
        b.max.to(g.bounds_max);
        g.left_first = lf;
        g.count = cnt;
        return g;
    };
    nodes.push_back(GpuBvhNode{});
    struct It { uint32_t id; size_t slot; };
    std::vector<It> st{{0u, 0}};
    while (!st.empty()) {
        It it = st.back();
        st.pop_back();
        const Aabb& b = bounds[it.id];
        size_t count = size_of(it.id);
        if (it.id >= leaf_base || count <= max_leaf) {
            uint32_t first = (uint32_t)prims.size();
            gather(it.id);
            uint32_t got = (uint32_t)prims.size() - first;
            nodes[it.slot] = mk(b, first, got);
            continue;
        }
        size_t left_slot = nodes.size();
        nodes.push_back(GpuBvhNode{});
        nodes.push_back(GpuBvhNode{});
        nodes[it.slot] = mk(b, (uint32_t)left_slot, 0);
        st.push_back({karras[2 * it.id + 1], left_slot + 1});
        st.push_back({karras[2 * it.id], left_slot});
    }
}

// lbvh.rs:422-538, over arbitrary boxes (the triangle path computes the
// padded triangle boxes first).
LbvhStages lbvh_build_over_bounds(const std::vector<Aabb>& tb, size_t max_leaf) {
    LbvhStages S;
    max_leaf = std::max<size_t>(max_leaf, 1);
    size_t n = tb.size();
    S.tri_bounds = tb;
    if (n == 0) return S;
    for (const Aabb& b : tb) S.centroid_bounds.grow_point(b.centroid());
    S.codes.resize(n);
    for (size_t i = 0; i < n; ++i) S.codes[i] = morton3d(lbvh_normalise(tb[i].centroid(), S.centroid_bounds));
    S.order.resize(n);
    std::iota(S.order.begin(), S.order.end(), 0u);
    std::stable_sort(S.order.begin(), S.order.end(), [&](uint32_t a, uint32_t b) {
        return S.codes[a] != S.codes[b] ? S.codes[a] < S.codes[b] : a < b;
    });
    S.sorted_codes.resize(n);
    for (size_t i = 0; i < n; ++i) S.sorted_codes[i] = S.codes[S.order[i]];
    if (n == 1) {
        GpuBvhNode g;
        tb[0].min.to(g.bounds_min);
        tb[0].max.to(g.bounds_max);
        g.left_first = 0;
        g.count = 1;
        S.tree.nodes = {g};
        S.tree.prim_indices = {0};
        S.node_bounds = {tb[0]};
        S.parent = {0xFFFFFFFFu};
        return S;
    }
    build_hierarchy(S.sorted_codes, S.karras, S.parent);
    uint32_t leaf_base = (uint32_t)(n - 1);
    S.node_bounds.assign(2 * n - 1, Aabb());
    S.subtree_size.assign(n - 1, 0);
    std::vector<uint32_t> visits(n - 1, 0);
    for (size_t leaf = 0; leaf < n; ++leaf) S.node_bounds[leaf_base + leaf] = tb[S.order[leaf]];
    for (size_t leaf = 0; leaf < n; ++leaf) {
        uint32_t node = S.parent[leaf_base + leaf];
        while (node != 0xFFFFFFFFu) {
            visits[node] += 1;
            if (visits[node] == 1) break;
            uint32_t l = S.karras[2 * node], r = S.karras[2 * node + 1];
            Aabb b = S.node_bounds[l];
            b.grow(S.node_bounds[r]);
            S.node_bounds[node] = b;
            auto sz = [&](uint32_t id) { return id >= leaf_base ? 1u : S.subtree_size[id]; };
            S.subtree_size[node] = sz(l) + sz(r);
            node = S.parent[node];
        }
    }
    relayout(S.karras, S.subtree_size, S.order, S.node_bounds, n, max_leaf, S.tree);
    return S;
}

LbvhStages lbvh_build(const std::vector<GpuTriangle>& tris, const std::vector<float>& pos,
                      size_t max_leaf) {
    std::vector<Aabb> tb(tris.size());
    for (size_t i = 0; i < tris.size(); ++i) tb[i] = triangle_bounds(tris[i], pos.data());
    return lbvh_build_over_bounds(tb, max_leaf);
}

}  // namespace oracle
