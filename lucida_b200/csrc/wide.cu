// Compressed 8-wide BVH, collapsed on the device from the binary tree that
// the traversal layout is derived from (the device LBVH, or a caller's tree).
// No counterpart in Lucida, whose kernels walk the binary GpuBvhNode array
// (bvh.rs:1045-1193); this is a re-layout of the same tree for the wide
// traversal in scene_dev.cuh (node format documented there).
//
// Build, level by level (one launch per level of the wide tree, plus a
// one-thread launch that advances the level range):
//   * a task is a binary internal node, or a leaf chunk (a binary leaf with
//     more than 4 triangles, 28 at a time); each task becomes one wide node;
//   * an internal task opens children greedily, largest surface area first,
//     until it has 8 children or none can be opened (a leaf with <= 4
//     triangles stays a leaf slot, and a node holds at most 32 triangles);
//     leaf slots of 2+ triangles compete for the free slots by area too,
//     splitting into the two subsets of least area x triangles, each under
//     the box of its own triangles;
//   * children are placed in slots by octant (greedy assignment of children
//     to the corner they lie towards), internal children get consecutive
//     wide indices in slot order, leaf triangles consecutive soup slots;
//   * quantization in double: origin two quanta below the node's box, one
//     quantum of slack outside every child box, so quantized boxes contain the
//     binary boxes (which carry the reference's magnitude-relative padding).
// Node and soup slots are claimed with atomics, so the layout order depends
// on scheduling; traversal results do not (slot order is deterministic and a
// hit reports the triangle's leaf-order index stored in the soup).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "ctx.cuh"

namespace luc {
namespace {

constexpr uint32_t kSmallLeaf = 4;   // leaves up to this size are leaf slots
constexpr uint32_t kChunkTris = 28;  // triangles per leaf chunk node before chaining
constexpr uint32_t kNodeTris = 32;   // triangle budget of one wide node
// Priority of splitting a leaf slot against opening an internal child of the
// same area: the displaced-sphere frame ran 324 / 335 / 341 / 341 / 340
// Mpaths/s at weights 1 / 2 / 4 / 8 / 16 (3.96 triangle tests and 14.2 node
// visits per closest-hit ray at 4).
constexpr float kLeafSplitWeight = 4.0f;
// The same for the BLASes of two-level scenes (negative: leaf slots are never
// split). The instanced frame (4096 instances of 16 meshes, 1920x1080, 8 spp)
// took 777 / 759 / 753 / 758 ms with weights -1 / 0 / 1 / 4 under nested
// walks; under the lock-step walk it runs 68.5 / 72.5 / 74.4 Mpaths/s at
// -1 / 1 / 4 (11.8 -> 8.6 triangle tests per ray from 1 to 4).
constexpr float kBlasLeafSplitWeight = 4.0f;
constexpr uint32_t kKindInternal = 0, kKindChunk = 1;

// ctr words
constexpr int kWcBegin = 0, kWcEnd = 1, kWcAlloc = 2, kWcSoup = 3, kWcErr = 4, kWcWords = 8;
constexpr uint32_t kErrTree = 1, kErrCapacity = 2;

struct Child {
    float lo[3], hi[3];
    uint32_t node;   // binary node index (box source)
    uint32_t first, count;
    uint32_t kind;   // 0 internal binary node, 1 chunk (internal wide child), 2 leaf slot
    uint32_t sub;    // leaf slot: its triangles, bit i = triangle first + i (count = popc)
};

__device__ __forceinline__ void node_box(const float4* nodes, uint32_t i, Child& c) {
    float4 a = nodes[2 * (size_t)i], b = nodes[2 * (size_t)i + 1];
    c.lo[0] = a.x; c.lo[1] = a.y; c.lo[2] = a.z;
    c.hi[0] = b.x; c.hi[1] = b.y; c.hi[2] = b.z;
}

// Child record for binary node i (internal, small leaf or big leaf).
__device__ __forceinline__ bool make_child(const float4* nodes, uint32_t num_nodes, uint32_t num_tris, uint32_t i,
                                           Child& c) {
    if (i >= num_nodes) return false;
    node_box(nodes, i, c);
    const uint32_t lf = __float_as_uint(nodes[2 * (size_t)i].w), cnt = __float_as_uint(nodes[2 * (size_t)i + 1].w);
    c.node = i;
    if (cnt == 0) {
        c.kind = kKindInternal;
        c.first = lf;
        c.count = 0;
        return lf + 1u < num_nodes && lf > i;  // children after their parent (preorder)
    }
    if ((uint64_t)lf + cnt > num_tris) return false;
    c.first = lf;
    c.count = cnt;
    c.kind = cnt <= kSmallLeaf ? 2u : kKindChunk;
    c.sub = cnt <= kSmallLeaf ? (1u << cnt) - 1u : 0u;
    return true;
}

// Leaf slots hold up to 4 triangles of one binary leaf (a subset `sub` of
// [first, first + 4), leaf order), under the union of their padded bounds,
// as the binary tree's own leaf boxes are made.
__device__ __forceinline__ float box_half_area(const float lo[3], const float hi[3]) {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return dx * dy + dy * dz + dz * dx;
}
struct LeafBoxes {
    float lo[kSmallLeaf][3], hi[kSmallLeaf][3];
};
__device__ __forceinline__ void leaf_boxes(const GpuTriangle* __restrict__ tris, const float4* __restrict__ pos,
                                           const Child& c, LeafBoxes& b) {
    for (uint32_t i = 0; i < kSmallLeaf; ++i)
        if (c.sub >> i & 1u) {
            const GpuTriangle t = tris[c.first + i];
            padded_tri_box(pos[t.i0], pos[t.i1], pos[t.i2], b.lo[i], b.hi[i]);
        }
}
__device__ __forceinline__ void subset_box(const LeafBoxes& b, uint32_t sub, float lo[3], float hi[3]) {
    for (int a = 0; a < 3; ++a) {
        lo[a] = INFINITY;
        hi[a] = -INFINITY;
    }
    for (uint32_t i = 0; i < kSmallLeaf; ++i)
        if (sub >> i & 1u)
            for (int a = 0; a < 3; ++a) {
                lo[a] = fminf(lo[a], b.lo[i][a]);
                hi[a] = fmaxf(hi[a], b.hi[i][a]);
            }
}
// Split leaf slot c (2 or more triangles) into the two subsets with the
// least surface-area cost (area x triangles, summed); l and r get their
// boxes.
__device__ __forceinline__ void split_leaf(const GpuTriangle* __restrict__ tris, const float4* __restrict__ pos,
                                           const Child& c, Child& l, Child& r) {
    LeafBoxes b;
    leaf_boxes(tris, pos, c, b);
    const uint32_t low = c.sub & (0u - c.sub);
    float best = INFINITY;
    uint32_t best_s = low;
    // Subsets holding the lowest triangle, short of all of them.
    for (uint32_t sset = c.sub; sset; sset = (sset - 1u) & c.sub) {
        if (!(sset & low) || sset == c.sub) continue;
        float lo[3], hi[3];
        subset_box(b, sset, lo, hi);
        float cost = box_half_area(lo, hi) * (float)__popc(sset);
        subset_box(b, c.sub ^ sset, lo, hi);
        cost += box_half_area(lo, hi) * (float)__popc(c.sub ^ sset);
        if (cost < best) {
            best = cost;
            best_s = sset;
        }
    }
    l = c;
    r = c;
    l.sub = best_s;
    r.sub = c.sub ^ best_s;
    l.count = __popc(l.sub);
    r.count = __popc(r.sub);
    subset_box(b, l.sub, l.lo, l.hi);
    subset_box(b, r.sub, r.lo, r.hi);
}

__device__ __forceinline__ float half_area(const Child& c) {
    float dx = c.hi[0] - c.lo[0], dy = c.hi[1] - c.lo[1], dz = c.hi[2] - c.lo[2];
    return dx * dy + dy * dz + dz * dx;
}

// Task k = binary root roots[k] (wide node k); map[roots[k]] = k when given.
__global__ void k_wide_init(const float4* __restrict__ nodes, uint32_t num_nodes, const uint32_t* __restrict__ roots,
                            uint32_t nroots, uint4* __restrict__ tasks, uint32_t* __restrict__ map,
                            uint32_t* __restrict__ ctr) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0) {
        ctr[kWcBegin] = 0;
        ctr[kWcEnd] = nroots;
        ctr[kWcAlloc] = nroots;
        ctr[kWcSoup] = 0;
        ctr[kWcErr] = 0;
    }
    if (k >= nroots) return;
    const uint32_t r = roots[k];
    if (r >= num_nodes) {
        atomicOr(ctr + kWcErr, kErrTree);
        tasks[k] = make_uint4(0u, 0u, 0u, kKindChunk);  // empty chunk: no reads
        return;
    }
    const uint32_t cnt = __float_as_uint(nodes[2 * (size_t)r + 1].w), lf = __float_as_uint(nodes[2 * (size_t)r].w);
    tasks[k] = cnt == 0 ? make_uint4(r, lf, 0u, kKindInternal) : make_uint4(r, lf, cnt, kKindChunk);
    if (map) map[r] = k;
}

__global__ void k_wide_advance(uint32_t* __restrict__ ctr) {
    ctr[kWcBegin] = ctr[kWcEnd];
    ctr[kWcEnd] = ctr[kWcAlloc];
}

// kTlas: the binary tree is a TLAS whose leaves hold at most kSmallLeaf
// instances (primitive indices); leaf slots are never split and the soup is
// `isoup`, one primitive index per entry, instead of triangle records.
template <bool kTlas>
__global__ void __launch_bounds__(128) k_wide_level(const float4* __restrict__ nodes, uint32_t num_nodes,
                                                    const float4* __restrict__ soup, uint32_t num_tris,
                                                    const GpuTriangle* __restrict__ tri_idx,
                                                    const float4* __restrict__ tri_pos, float leaf_weight,
                                                    uint4* __restrict__ tasks, float4* __restrict__ wnodes,
                                                    float4* __restrict__ wsoup, uint32_t* __restrict__ isoup,
                                                    uint32_t cap, uint32_t* __restrict__ ctr) {
    if (ctr[kWcErr]) return;  // a failed level ends the build
    // Claims past the capacity failed (and flagged); never read beyond it.
    const uint32_t begin = ctr[kWcBegin], end = min(ctr[kWcEnd], cap);
    for (uint32_t w = begin + blockIdx.x * blockDim.x + threadIdx.x; w < end; w += gridDim.x * blockDim.x) {
        const uint4 task = tasks[w];
        Child ch[8];
        uint32_t n = 0;
        bool ok = true;
        if (task.w == kKindInternal) {
            ok = make_child(nodes, num_nodes, num_tris, task.y, ch[0]) &&
                 make_child(nodes, num_nodes, num_tris, task.y + 1u, ch[1]);
            n = 2;
            uint32_t tris = (ch[0].kind == 2u ? ch[0].count : 0u) + (ch[1].kind == 2u ? ch[1].count : 0u);
            // Open the largest child while the node has room: an internal
            // child into its two children, a leaf slot of 2+ triangles into
            // two slots of fewer triangles under their own boxes (the binary
            // tree's leaves hold up to 4 triangles under one box); leaf
            // areas count leaf_weight times.
            while (ok && n < 8) {
                int best = -1;
                float best_a = -1.0f;
                for (uint32_t k = 0; k < n; ++k) {
                    if (ch[k].kind == 2u) {
                        const float a =
                            ch[k].count >= 2u && leaf_weight >= 0.0f ? half_area(ch[k]) * leaf_weight : -1.0f;
                        if (a > best_a) {
                            best = (int)k;
                            best_a = a;
                        }
                        continue;
                    }
                    if (ch[k].kind != kKindInternal) continue;
                    float a = half_area(ch[k]);
                    if (a > best_a) {
                        // The grandchildren's small leaves must fit the triangle budget.
                        Child l, r;
                        if (!make_child(nodes, num_nodes, num_tris, ch[k].first, l) ||
                            !make_child(nodes, num_nodes, num_tris, ch[k].first + 1u, r)) {
                            ok = false;
                            break;
                        }
                        uint32_t add = (l.kind == 2u ? l.count : 0u) + (r.kind == 2u ? r.count : 0u);
                        if (tris + add > kNodeTris) continue;
                        best = (int)k;
                        best_a = a;
                    }
                }
                if (!ok || best < 0) break;
                if (ch[best].kind == 2u) {
                    Child l, r;
                    split_leaf(tri_idx, tri_pos, ch[best], l, r);
                    ch[best] = l;
                    ch[n++] = r;
                    continue;
                }
                Child l, r;
                make_child(nodes, num_nodes, num_tris, ch[best].first, l);
                make_child(nodes, num_nodes, num_tris, ch[best].first + 1u, r);
                tris += (l.kind == 2u ? l.count : 0u) + (r.kind == 2u ? r.count : 0u);
                ch[best] = l;
                ch[n++] = r;
            }
        } else if (kTlas) {
            // A TLAS whose root is a leaf: one slot under the leaf's box.
            if (task.z == 0 || task.z > kSmallLeaf) {
                atomicOr(ctr + kWcErr, kErrTree);
                continue;
            }
            node_box(nodes, task.x, ch[0]);
            ch[0].node = task.x;
            ch[0].first = task.y;
            ch[0].count = task.z;
            ch[0].kind = 2u;
            ch[0].sub = (1u << task.z) - 1u;
            n = 1;
        } else {
            // Leaf chunk: up to 7 (or 8, for the last) slots of 4 triangles,
            // every slot with the binary leaf's box; the rest chains on.
            Child box;
            node_box(nodes, task.x, box);
            uint32_t first = task.y, rem = task.z;
            const uint32_t here = rem <= kNodeTris ? rem : kChunkTris;
            for (uint32_t k = 0; k < here; k += kSmallLeaf) {
                ch[n].node = task.x;
                ch[n].first = first + k;
                ch[n].count = min(kSmallLeaf, here - k);
                ch[n].kind = 2u;
                ch[n].sub = (1u << ch[n].count) - 1u;
                LeafBoxes lb;  // each slot under its own triangles' box
                leaf_boxes(tri_idx, tri_pos, ch[n], lb);
                subset_box(lb, ch[n].sub, ch[n].lo, ch[n].hi);
                ++n;
            }
            if (rem > here) {
                ch[n] = box;
                ch[n].node = task.x;
                ch[n].first = first + here;
                ch[n].count = rem - here;
                ch[n].kind = kKindChunk;
                ++n;
            }
        }
        if (kTlas)
            for (uint32_t k = 0; k < n; ++k) ok = ok && ch[k].kind != kKindChunk;  // leaves of <= 4 instances only
        if (!ok) {
            atomicOr(ctr + kWcErr, kErrTree);
            continue;
        }
        // Node box and octant slot assignment.
        float lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = ch[0].lo[a];
            hi[a] = ch[0].hi[a];
            for (uint32_t k = 1; k < n; ++k) {
                lo[a] = fminf(lo[a], ch[k].lo[a]);
                hi[a] = fmaxf(hi[a], ch[k].hi[a]);
            }
        }
        float cost[8][8];
        for (uint32_t k = 0; k < n; ++k) {
            float v[3];
            for (int a = 0; a < 3; ++a) v[a] = (ch[k].lo[a] + ch[k].hi[a]) - (lo[a] + hi[a]);
            for (uint32_t s = 0; s < 8; ++s)
                cost[k][s] = -((s & 1u ? v[0] : -v[0]) + (s & 2u ? v[1] : -v[1]) + (s & 4u ? v[2] : -v[2]));
        }
        int slot_of[8];
        uint32_t used_slots = 0, done = 0;
        for (uint32_t r = 0; r < n; ++r) {
            float bc = 3.4e38f;
            int bk = -1, bs = -1;
            for (uint32_t k = 0; k < n; ++k) {
                if (done & (1u << k)) continue;
                for (uint32_t s = 0; s < 8; ++s) {
                    if (used_slots & (1u << s)) continue;
                    if (cost[k][s] < bc || bk < 0) {
                        bc = cost[k][s];
                        bk = (int)k;
                        bs = (int)s;
                    }
                }
            }
            slot_of[bk] = bs;
            done |= 1u << bk;
            used_slots |= 1u << bs;
        }
        int child_at[8];
        for (int s = 0; s < 8; ++s) child_at[s] = -1;
        for (uint32_t k = 0; k < n; ++k) child_at[slot_of[k]] = (int)k;
        uint32_t imask = 0, ntri = 0;
        for (int s = 0; s < 8; ++s) {
            const int k = child_at[s];
            if (k < 0) continue;
            if (ch[k].kind == 2u) ntri += ch[k].count;
            else imask |= 1u << s;
        }
        const uint32_t nint = __popc(imask);
        const uint32_t cbase = nint ? atomicAdd(ctr + kWcAlloc, nint) : 0u;
        const uint32_t tbase = ntri ? atomicAdd(ctr + kWcSoup, ntri) : 0u;
        if ((nint && (uint64_t)cbase + nint > cap) || (uint64_t)tbase + ntri > num_tris) {
            atomicOr(ctr + kWcErr, kErrCapacity);
            continue;
        }
        // Quantization (double: exact for these magnitudes).
        uint32_t ebits = 0;
        float p[3];
        double scale[3], inv_scale[3];
        for (int a = 0; a < 3; ++a) {
            const double ext = (double)hi[a] - (double)lo[a];
            int ex = -126;
            if (ext > 0.0) {
                int e2;
                frexp(ext / 250.0, &e2);  // ext / 250 < 2^e2
                ex = max(-126, min(120, e2));
            }
            // No finer than 1/64 of the coordinates' ulp: the loop below then
            // needs at most a few coarsening steps.
            const double mag = fmax(fabs((double)lo[a]), fabs((double)hi[a]));
            if (mag > 0.0) {
                int em;
                frexp(mag, &em);  // ulp(mag) = 2^(em - 24)
                ex = max(ex, min(120, em - 24 - 6));
            }
            // Origin at least two quanta below the box, rounded down to float;
            // coarsen the grid until the box's top plane fits in 253 quanta
            // (the float origin can sit up to an ulp of the coordinates lower).
            float pf = 0.0f;
            for (;;) {
                scale[a] = ldexp(1.0, ex);
                inv_scale[a] = ldexp(1.0, -ex);  // x / 2^ex == x * 2^-ex exactly: no double divisions
                const double pd = (double)lo[a] - 2.0 * scale[a];
                pf = (float)pd;
                if ((double)pf > pd) pf = nextafterf(pf, -3.4e38f);
                if (ex >= 120 || ceil(((double)hi[a] - (double)pf) * inv_scale[a]) + 1.0 <= 253.0) break;
                ++ex;
            }
            p[a] = pf;
            ebits |= (uint32_t)(ex + 127) << (8 * a);
        }
        ebits |= imask << 24;
        uint32_t qlo[3][2] = {{0, 0}, {0, 0}, {0, 0}}, qhi[3][2] = {{0, 0}, {0, 0}, {0, 0}}, cntmask = 0;
        uint32_t off = 0, rank = 0;
        for (int s = 0; s < 8; ++s) {
            const int k = child_at[s];
            uint32_t l8[3], h8[3];
            if (k < 0) {
                for (int a = 0; a < 3; ++a) {
                    l8[a] = 255u;  // empty: near plane beyond far plane, never hit
                    h8[a] = 0u;
                }
            } else {
                for (int a = 0; a < 3; ++a) {
                    double ql = floor(((double)ch[k].lo[a] - (double)p[a]) * inv_scale[a]) - 1.0;
                    double qh = ceil(((double)ch[k].hi[a] - (double)p[a]) * inv_scale[a]) + 1.0;
                    l8[a] = (uint32_t)fmax(0.0, fmin(255.0, ql));
                    h8[a] = (uint32_t)fmax(0.0, fmin(255.0, qh));
                }
                if (ch[k].kind == 2u) {
                    cntmask |= ((1u << ch[k].count) - 1u) << (4 * s);  // nibble s: the slot's triangles
                    uint32_t i = 0;
                    for (uint32_t bits = ch[k].sub; bits; bits &= bits - 1u, ++i) {
                        const uint32_t t = ch[k].first + (uint32_t)(__ffs(bits) - 1);
                        if (kTlas) {
                            isoup[tbase + off + i] = t;
                            continue;
                        }
                        const size_t src = 3 * (size_t)t, dst = 3 * (size_t)(tbase + off + i);
                        float4 q0 = soup[src];
                        q0.w = __uint_as_float(t);
                        wsoup[dst] = q0;
                        wsoup[dst + 1] = soup[src + 1];
                        wsoup[dst + 2] = soup[src + 2];
                    }
                    off += ch[k].count;
                } else {
                    tasks[cbase + rank] = ch[k].kind == kKindInternal
                                              ? make_uint4(ch[k].node, ch[k].first, 0u, kKindInternal)
                                              : make_uint4(ch[k].node, ch[k].first, ch[k].count, kKindChunk);
                    ++rank;
                }
            }
            for (int a = 0; a < 3; ++a) {
                qlo[a][s >> 2] |= l8[a] << (8 * (s & 3));
                qhi[a][s >> 2] |= h8[a] << (8 * (s & 3));
            }
        }
        float4* o = wnodes + 5 * (size_t)w;
        o[0] = make_float4(p[0], p[1], p[2], __uint_as_float(ebits));
        o[1] = make_float4(__uint_as_float(cbase), __uint_as_float(tbase), __uint_as_float(cntmask), 0.0f);
        o[2] = make_float4(__uint_as_float(qlo[0][0]), __uint_as_float(qlo[0][1]), __uint_as_float(qlo[1][0]),
                           __uint_as_float(qlo[1][1]));
        o[3] = make_float4(__uint_as_float(qlo[2][0]), __uint_as_float(qlo[2][1]), __uint_as_float(qhi[0][0]),
                           __uint_as_float(qhi[0][1]));
        o[4] = make_float4(__uint_as_float(qhi[1][0]), __uint_as_float(qhi[1][1]), __uint_as_float(qhi[2][0]),
                           __uint_as_float(qhi[2][1]));
    }
}

}  // namespace
}  // namespace luc

// Collapse the resident binary tree (c->nodes, c->soup in leaf order) into
// c->wnodes / c->wsoup: one wide tree per root in `roots` (host array; wide
// node k is the root of the tree of roots[k]), whose trees must together
// cover every triangle. With `map`, c->blas_wide[roots[k]] = k (two-level
// scenes reach a BLAS's wide tree from its binary root). Leaves
// c->wide_nodes = 0 (binary traversal) when a tree is deeper than the level
// budget or the trees miss triangles; fails on a malformed tree.
int32_t luc_build_wide_roots(luc_ctx* c, const uint32_t* roots, uint32_t nroots, bool map, uint32_t num_nodes,
                             uint32_t num_tris) {
    using namespace luc;
    c->wide_nodes = 0;
    if (!num_nodes || !num_tris || !nroots) return LUC_OK;
    const uint64_t cap = 2ull * num_nodes + num_tris / kChunkTris + nroots + 8;
    if (cap > 0x7FFFFFFFull) return LUC_OK;
    cudaStream_t s = c->stream;
    LUC_CUDA(c, c->wnodes.ensure(cap * 80), "alloc wide nodes");
    LUC_CUDA(c, c->wsoup.ensure((size_t)num_tris * 48), "alloc wide soup");
    LUC_CUDA(c, c->wtasks.ensure(cap * 16), "alloc wide tasks");
    LUC_CUDA(c, c->wctr.ensure(kWcWords * 4), "alloc wide counters");
    LUC_CUDA(c, upload(c->wroots, roots, nroots, s), "upload wide roots");
    uint32_t* wmap = nullptr;
    if (map) {
        LUC_CUDA(c, c->blas_wide.ensure((size_t)num_nodes * 4), "alloc wide root map");
        LUC_CUDA(c, cudaMemsetAsync(c->blas_wide.p, 0xFF, (size_t)num_nodes * 4, s), "clear wide root map");
        wmap = c->blas_wide.as<uint32_t>();
    }
    uint32_t* ctr = c->wctr.as<uint32_t>();
    k_wide_init<<<(nroots + 127) / 128, 128, 0, s>>>(c->nodes.as<float4>(), num_nodes, c->wroots.as<uint32_t>(),
                                                      nroots, c->wtasks.as<uint4>(), wmap, ctr);
    const int grid = c->num_sms * 8;
    constexpr int kLevelsPerSync = 12, kMaxLevels = 240;
    uint32_t h[kWcWords] = {};
    for (int level = 0; level < kMaxLevels; level += kLevelsPerSync) {
        for (int k = 0; k < kLevelsPerSync; ++k) {
            k_wide_level<false><<<grid, 128, 0, s>>>(c->nodes.as<float4>(), num_nodes, c->soup.as<float4>(), num_tris,
                                              c->tris.as<GpuTriangle>(), c->positions.as<float4>(),
                                              map ? kBlasLeafSplitWeight : kLeafSplitWeight, c->wtasks.as<uint4>(), c->wnodes.as<float4>(), c->wsoup.as<float4>(),
                                              nullptr, (uint32_t)cap, ctr);
            k_wide_advance<<<1, 1, 0, s>>>(ctr);
        }
        LUC_CUDA(c, cudaGetLastError(), "wide build");
        LUC_CUDA(c, cudaMemcpyAsync(h, ctr, sizeof(h), cudaMemcpyDeviceToHost, s), "wide build counters");
        LUC_CUDA(c, cudaStreamSynchronize(s), "wide build");
        if (h[kWcErr] & kErrTree) return luc_fail(c, LUC_ERR_VALIDATION, "BVH: malformed tree (wide collapse)");
        if (h[kWcErr]) return LUC_OK;  // capacity: keep the binary traversal
        if (h[kWcBegin] == h[kWcEnd]) break;
    }
    if (h[kWcBegin] != h[kWcEnd] || h[kWcSoup] != num_tris) return LUC_OK;  // too deep: binary traversal
    c->wide_nodes = h[kWcAlloc];
    return LUC_OK;
}

// Collapse the TLAS (binary nodes [root, num_nodes) of c->nodes, leaves of at
// most 4 instances whose primitive indices lie below prim_bound) into
// c->twnodes / c->twsoup (one primitive index per leaf entry), the same
// 8-wide format as the BLASes' trees. *ok is false (binary TLAS traversal)
// when the leaves are larger or the tree is deeper than the level budget.
int32_t luc_build_wide_tlas(luc_ctx* c, uint32_t root, uint32_t num_nodes, uint32_t prim_bound, uint32_t ninst,
                            bool* ok) {
    using namespace luc;
    *ok = false;
    if (!ninst || c->tlas_leaf > kSmallLeaf || root >= num_nodes) return LUC_OK;
    const uint64_t cap = 2ull * (num_nodes - root) + 8;
    cudaStream_t s = c->stream;
    LUC_CUDA(c, c->twnodes.ensure(cap * 80), "alloc wide tlas");
    LUC_CUDA(c, c->twsoup.ensure((size_t)prim_bound * 4), "alloc wide tlas soup");
    LUC_CUDA(c, c->wtasks.ensure(cap * 16), "alloc wide tasks");
    LUC_CUDA(c, c->wctr.ensure(kWcWords * 4), "alloc wide counters");
    LUC_CUDA(c, upload(c->wroots, &root, 1, s), "upload wide roots");
    uint32_t* ctr = c->wctr.as<uint32_t>();
    k_wide_init<<<1, 128, 0, s>>>(c->nodes.as<float4>(), num_nodes, c->wroots.as<uint32_t>(), 1,
                                  c->wtasks.as<uint4>(), nullptr, ctr);
    const int grid = c->num_sms * 2;
    constexpr int kLevels = 16;  // 4^16 instances deep at 2 children per level: far beyond any TLAS here
    for (int level = 0; level < kLevels; ++level) {
        k_wide_level<true><<<grid, 128, 0, s>>>(c->nodes.as<float4>(), num_nodes, nullptr, prim_bound, nullptr,
                                                nullptr, -1.0f, c->wtasks.as<uint4>(), c->twnodes.as<float4>(),
                                                nullptr, c->twsoup.as<uint32_t>(), (uint32_t)cap, ctr);
        k_wide_advance<<<1, 1, 0, s>>>(ctr);
    }
    LUC_CUDA(c, cudaGetLastError(), "wide tlas");
    uint32_t h[kWcWords] = {};
    LUC_CUDA(c, cudaMemcpyAsync(h, ctr, sizeof(h), cudaMemcpyDeviceToHost, s), "wide tlas counters");
    LUC_CUDA(c, cudaStreamSynchronize(s), "wide tlas");
    if (h[kWcErr] & kErrTree) return luc_fail(c, LUC_ERR_VALIDATION, "TLAS: malformed tree (wide collapse)");
    *ok = h[kWcErr] == 0 && h[kWcBegin] == h[kWcEnd] && h[kWcSoup] == ninst;
    return LUC_OK;
}

int32_t luc_build_wide(luc_ctx* c, uint32_t num_nodes, uint32_t num_tris) {
    const uint32_t root = 0;
    return luc_build_wide_roots(c, &root, 1, false, num_nodes, num_tris);
}
