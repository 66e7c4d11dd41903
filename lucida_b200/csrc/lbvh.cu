// GPU LBVH builder and radix sort on sm_100a (crates/core/src/lbvh.rs,
// crates/gpu/src/lbvh.rs; shaders/lbvh/*.wgsl):
//
//   triangle bounds (padded, bvh.rs:100-111)  -> k_tri_bounds
//   centroid bounds (exact min/max)           -> k_cbounds_partial/final
//   30-bit Morton codes (lbvh.rs:72-131)       -> k_morton
//   stable sort of (code, index)               -> onesweep LSD radix sort,
//                                                 8-bit digits, decoupled look-back
//   Karras hierarchy (lbvh.rs:211-292)         -> k_karras, one thread per node
//   bottom-up fit + subtree sizes (:490-525)   -> k_fit, one atomic per node
//   relayout, collapse <= 4 (:315-406)         -> k_relayout: preorder ranks from
//                                                 per-subtree internal counts, so
//                                                 the DFS order the CPU produces
//                                                 is reproduced without a stack
//
// Every stage is integer or exact-min/max/IEEE work compiled with
// --fmad=false, so each is bit-identical to the CPU builder. The relayout,
// which the reference runs on the host after a readback (Lbvh::from_parts),
// runs on the device here.
#include "ctx.cuh"
#include "sort_kernels.cuh"

namespace luc {

constexpr uint32_t kNone = 0xFFFFFFFFu;

// ---------------------------------------------------------------- bounds
__global__ void k_tri_bounds(const GpuTriangle* __restrict__ tris, const float4* __restrict__ pos, uint32_t n,
                             float* __restrict__ boxes) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        GpuTriangle t = tris[i];
        float lo[3], hi[3];
        padded_tri_box(pos[t.i0], pos[t.i1], pos[t.i2], lo, hi);
        float* o = boxes + 6 * (size_t)i;
        o[0] = lo[0]; o[1] = lo[1]; o[2] = lo[2]; o[3] = hi[0]; o[4] = hi[1]; o[5] = hi[2];
    }
}

__device__ __forceinline__ void centroid(const float* b, float& x, float& y, float& z) {
    x = (b[0] + b[3]) * 0.5f;
    y = (b[1] + b[4]) * 0.5f;
    z = (b[2] + b[5]) * 0.5f;
}

// Exact min/max of the centroids: per-block partials, then one block.
__global__ void k_cbounds_partial(const float* __restrict__ boxes, uint32_t n, float* __restrict__ partial) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float c[3];
        centroid(boxes + 6 * (size_t)i, c[0], c[1], c[2]);
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(lo[k], c[k]);
            hi[k] = fmaxf(hi[k], c[k]);
        }
    }
    __shared__ float s[6][256];
    for (int k = 0; k < 3; ++k) {
        s[k][threadIdx.x] = lo[k];
        s[3 + k][threadIdx.x] = hi[k];
    }
    __syncthreads();
    for (uint32_t w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 3; ++k) {
                s[k][threadIdx.x] = fminf(s[k][threadIdx.x], s[k][threadIdx.x + w]);
                s[3 + k][threadIdx.x] = fmaxf(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 6; ++k) partial[6 * blockIdx.x + k] = s[k][0];
}
__global__ void k_cbounds_final(const float* __restrict__ partial, uint32_t nb, float* __restrict__ out) {
    __shared__ float s[6][256];
    float v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x)
        for (int k = 0; k < 6; ++k) v[k] = k < 3 ? fminf(v[k], partial[6 * i + k]) : fmaxf(v[k], partial[6 * i + k]);
    for (int k = 0; k < 6; ++k) s[k][threadIdx.x] = v[k];
    __syncthreads();
    for (uint32_t w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 6; ++k)
                s[k][threadIdx.x] = k < 3 ? fminf(s[k][threadIdx.x], s[k][threadIdx.x + w])
                                          : fmaxf(s[k][threadIdx.x], s[k][threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x < 6) out[threadIdx.x] = s[threadIdx.x][0];
}

// ---------------------------------------------------------------- Morton
__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {  // lbvh.rs:72-79
    uint32_t x = v & 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}
__device__ __forceinline__ float norm_axis(float v, float lo, float hi) {  // lbvh.rs:109-117
    float e = hi - lo;
    return e > 0.0f ? (v - lo) / e : 0.5f;
}
__device__ __forceinline__ uint32_t quantise(float v) {  // lbvh.rs:93-97
    return f2u(clampf(v * 1023.0f, 0.0f, 1023.0f));
}
__global__ void k_morton(const float* __restrict__ boxes, uint32_t n, const float* __restrict__ cb,
                         uint32_t* __restrict__ keys, uint32_t* __restrict__ vals, uint32_t* __restrict__ codes) {
    float lo0 = cb[0], lo1 = cb[1], lo2 = cb[2], hi0 = cb[3], hi1 = cb[4], hi2 = cb[5];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float x, y, z;
        centroid(boxes + 6 * (size_t)i, x, y, z);
        uint32_t code = (expand_bits(quantise(norm_axis(x, lo0, hi0))) << 2) |
                        (expand_bits(quantise(norm_axis(y, lo1, hi1))) << 1) |
                        expand_bits(quantise(norm_axis(z, lo2, hi2)));
        keys[i] = code;
        vals[i] = i;
        codes[i] = code;
    }
}

// ---------------------------------------------------------------- onesweep sort
// Stable LSD radix sort of (u32 key, u32 value), 8-bit digits, 4 passes.
// One histogram pass counts all four digits at once; each pass then sorts a
// 4096-key tile per block by digit in shared memory (stable), publishes the
// tile's per-digit counts, and resolves each digit's global start by
// decoupled look-back over the preceding tiles. Tile ids come from an atomic
// counter, so every tile a block waits on has already started.

__global__ void k_hist4(const uint32_t* __restrict__ keys, uint32_t n, uint32_t* __restrict__ hist) {
    __shared__ uint32_t sh[4][256];
    for (int t = threadIdx.x; t < 1024; t += blockDim.x) (&sh[0][0])[t] = 0;
    __syncthreads();
    auto count = [&](uint32_t k) {
        atomicAdd(&sh[0][k & 255u], 1u);
        atomicAdd(&sh[1][(k >> 8) & 255u], 1u);
        atomicAdd(&sh[2][(k >> 16) & 255u], 1u);
        atomicAdd(&sh[3][k >> 24], 1u);
    };
    // 16-byte loads where the array allows them (the scratch arrays are
    // 256-byte aligned); the last n % 4 keys one at a time.
    const uint32_t n4 = ((reinterpret_cast<uintptr_t>(keys) & 15u) == 0) ? n / 4 : 0;
    const uint4* k4 = reinterpret_cast<const uint4*>(keys);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += gridDim.x * blockDim.x) {
        uint4 v = k4[i];
        count(v.x);
        count(v.y);
        count(v.z);
        count(v.w);
    }
    for (uint32_t i = 4 * n4 + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) count(keys[i]);
    __syncthreads();
    for (int t = threadIdx.x; t < 1024; t += blockDim.x) {
        uint32_t v = (&sh[0][0])[t];
        if (v) atomicAdd(hist + t, v);
    }
}
// Exclusive scan of each pass's 256 digit counts (one block of 256 threads).
__global__ void k_hist_scan(const uint32_t* __restrict__ hist, uint32_t* __restrict__ offsets) {
    __shared__ uint32_t s[256];
    for (int p = 0; p < 4; ++p) {
        uint32_t v = hist[p * 256 + threadIdx.x];
        s[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < 256; off <<= 1) {
            uint32_t t = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
            __syncthreads();
            s[threadIdx.x] += t;
            __syncthreads();
        }
        offsets[p * 256 + threadIdx.x] = s[threadIdx.x] - v;
        __syncthreads();
    }
}

// Look-back status words are read and written at GPU scope (past the
// incoherent L1). A word packs its flag with its count, so it is seen whole.
__device__ __forceinline__ uint32_t ld_status(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_status(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// The exclusive prefix of digit `tid` over the tiles before `tile`: walks
// back from tile - 1, kLookWin status rows per round trip (each read is one
// coalesced row segment per warp), adding aggregates until an inclusive
// prefix ends the walk; an unpublished word stops the round and the next
// round re-reads from there. Publishes this tile's inclusive prefix.
__device__ __forceinline__ uint32_t look_back(uint32_t* status, uint32_t tile, uint32_t tid, uint32_t total,
                                              uint32_t spin_limit, uint32_t* err) {
    if (tile == 0) return 0;  // published inclusive with the aggregate
    uint32_t excl = 0, spins = 0;
    int64_t j = (int64_t)tile - 1;  // the next predecessor to account for
    while (j >= 0) {
        const int64_t j0 = j;
        uint32_t e[kLookWin];
#pragma unroll
        for (int v = 0; v < kLookWin; ++v) e[v] = j0 - v >= 0 ? ld_status(status + (size_t)(j0 - v) * 256 + tid) : 0u;
        bool stop = false, done = false;
#pragma unroll
        for (int v = 0; v < kLookWin; ++v) {
            const uint32_t flag = e[v] & ~kCountMask;
            if (!stop && j0 - v >= 0) {
                if (flag == 0) {
                    stop = true;
                } else {
                    excl += e[v] & kCountMask;
                    j = j0 - v - 1;
                    if (flag == kFlagInc) stop = done = true;
                }
            }
        }
        if (done) break;
        if (stop && ++spins > spin_limit) {  // bounded wait: report, never hang
            atomicExch(err, 1u);
            break;
        }
    }
    st_status(status + (size_t)tile * 256 + tid, (excl + total) | kFlagInc);
    return excl;
}

// One pass, by persistent blocks that take tiles from the counter in turn.
// Per 4096-key tile (16 keys a thread in warp-striped order): count the
// tile's digits per warp and publish the tile's per-digit aggregate at once,
// so that later tiles' look-backs find it early; scan the counts into each
// (warp, digit)'s first position in the digit-sorted tile; rank every key
// into the shared-memory tile (lanes holding the same digit find one another
// through a per-digit lane mask that each sets a bit in, which keeps ties in
// input order); then take the next tile and load its keys and values into
// the registers the ranking freed, while this tile looks back for its
// digits' global starts and writes each digit's run out contiguously. 64
// registers and 45 KB of shared memory hold four blocks per SM.
__global__ void __launch_bounds__(kSortThreads, 4) k_onesweep(const uint32_t* __restrict__ kin,
                                                           const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
                                                           uint32_t* __restrict__ vout, uint32_t n, int shift,
                                                           const uint32_t* __restrict__ digit_offsets,
                                                           uint32_t* status, uint32_t* tile_counter, uint32_t* err,
                                                           uint32_t spin_limit) {
    constexpr uint32_t kWarps = kSortThreads / 32;
    __shared__ uint32_t s_tile, s_next_tile;
    __shared__ uint16_t s_next[kWarps][256];  // next tile position of each (warp, digit) while ranking
    __shared__ uint32_t s_lanes[kWarps][256]; // lanes of one key slot holding each digit (zero between slots)
    __shared__ uint32_t s_base[256];          // global destination minus tile position, per digit
    __shared__ uint32_t s_wsum[kWarps];
    __shared__ uint32_t s_keys[kTile], s_vals[kTile];
    uint32_t(*s_count)[256] = reinterpret_cast<uint32_t(*)[256]>(s_vals);  // digit counts, before the ranking
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    const uint32_t offs = digit_offsets[tid];
    for (uint32_t t = tid; t < kWarps * 256; t += kSortThreads) (&s_lanes[0][0])[t] = 0;
    if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    uint32_t tile = s_tile;
    uint32_t key[kSortKpt], val[kSortKpt];
    auto load = [&](uint32_t t) {
        const uint32_t base = t * kTile + warp * (32u * kSortKpt);
#pragma unroll
        for (int k = 0; k < kSortKpt; ++k) {
            const uint32_t idx = base + k * 32u + lane;
            const bool valid = idx < n;
            key[k] = valid ? kin[idx] : 0u;
            val[k] = valid ? vin[idx] : 0u;
        }
    };
    if (tile < tiles) load(tile);
    while (tile < tiles) {
        const uint32_t wbase = tile * kTile + warp * (32u * kSortKpt);
        for (uint32_t t = tid; t < kWarps * 256; t += kSortThreads) (&s_count[0][0])[t] = 0;
        if (tid == 0) s_next_tile = atomicAdd(tile_counter, 1u);  // read after the ranking
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kSortKpt; ++k)
            if (wbase + k * 32u + lane < n) atomicAdd(&s_count[warp][(key[k] >> shift) & 255u], 1u);
        __syncthreads();
        // Thread `tid` owns digit `tid`: its count per warp and in the tile;
        // the aggregate goes out before anything else.
        uint32_t wc[kWarps], total = 0;
#pragma unroll
        for (uint32_t w = 0; w < kWarps; ++w) {
            wc[w] = s_count[w][tid];
            total += wc[w];
        }
        st_status(status + (size_t)tile * 256 + tid, total | (tile == 0 ? kFlagInc : kFlagAgg));
        // Exclusive scan of the digit totals over the tile: where each
        // digit's run starts in the digit-sorted tile.
        uint32_t x = total;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (lane == 31) s_wsum[warp] = x;
        __syncthreads();  // also: every count is read before the values overwrite them
        uint32_t start = x - total;
#pragma unroll
        for (uint32_t w = 0; w < kWarps; ++w) start += w < warp ? s_wsum[w] : 0u;
        uint32_t run = start;
#pragma unroll
        for (uint32_t w = 0; w < kWarps; ++w) {
            s_next[w][tid] = (uint16_t)run;
            run += wc[w];
        }
        __syncthreads();
        // Rank each key slot: its lanes holding one digit are numbered in
        // lane order after the warp's earlier slots; the key lands in its
        // position.
        const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
        for (int k = 0; k < kSortKpt; ++k) {
            const bool valid = wbase + k * 32u + lane < n;
            const uint32_t digit = (key[k] >> shift) & 255u;
            if (valid) atomicOr(&s_lanes[warp][digit], 1u << lane);
            __syncwarp();
            const uint32_t peers = valid ? s_lanes[warp][digit] : 0u;
            const uint32_t before = valid ? s_next[warp][digit] : 0u;
            __syncwarp();
            if (valid && lane == (uint32_t)(__ffs(peers) - 1)) {
                s_next[warp][digit] = (uint16_t)(before + __popc(peers));
                s_lanes[warp][digit] = 0u;
            }
            __syncwarp();
            const uint32_t local = before + __popc(peers & lt);
            if (valid) {
                s_keys[local] = key[k];
                s_vals[local] = val[k];
            }
        }
        // The next tile's keys and values load while this tile looks back.
        const uint32_t next = s_next_tile;
        if (next < tiles) load(next);
        const uint32_t excl = look_back(status, tile, tid, total, spin_limit, err);
        s_base[tid] = offs + excl - start;
        __syncthreads();
        const uint32_t first_key = tile * kTile;
        const uint32_t count = min(kTile, n - first_key);
        for (uint32_t i = tid; i < count; i += kSortThreads) {
            const uint32_t kk = s_keys[i];
            const uint32_t dst = s_base[(kk >> shift) & 255u] + i;
            // In bounds whenever the pass's input matches the histogram; a
            // pass after one whose look-back gave up may not, and writes
            // nothing outside the arrays.
            if (dst < n) {
                kout[dst] = kk;
                vout[dst] = s_vals[i];
            }
        }
        __syncthreads();  // the tile's shared memory is read before the next tile's counts reuse it
        tile = next;
    }
}

// ---------------------------------------------------------------- Karras
__device__ __forceinline__ int lcp(const uint32_t* __restrict__ c, int64_t n, int32_t i, int32_t j) {
    if (j < 0 || j >= n) return -1;
    uint32_t a = c[i], b = c[j];
    if (a == b) return 32 + __clz((uint32_t)i ^ (uint32_t)j);
    return __clz(a ^ b);
}
// lbvh.rs:211-292: node i finds its direction, range and split alone.
__global__ void k_karras(const uint32_t* __restrict__ codes, uint32_t n, uint32_t* __restrict__ karras,
                         uint32_t* __restrict__ parent, uint32_t* __restrict__ first_of) {
    const int64_t nn = n;
    const uint32_t leaf_base = n - 1;
    for (uint32_t ui = blockIdx.x * blockDim.x + threadIdx.x; ui < n - 1; ui += gridDim.x * blockDim.x) {
        int32_t i = (int32_t)ui;
        int32_t dd = lcp(codes, nn, i, i + 1) - lcp(codes, nn, i, i - 1);
        int32_t d = (dd > 0) - (dd < 0);
        int32_t dmin = lcp(codes, nn, i, i - d);
        int32_t lmax = 2;
        while (lcp(codes, nn, i, i + lmax * d) > dmin) lmax *= 2;
        int32_t l = 0;
        for (int32_t t = lmax / 2; t >= 1; t /= 2)
            if (lcp(codes, nn, i, i + (l + t) * d) > dmin) l += t;
        int32_t j = i + l * d;
        int32_t first = min(i, j), last = max(i, j);
        int32_t dnode = lcp(codes, nn, i, j);
        int32_t s = 0, t = l;
        while (t > 1) {
            t = (t + 1) / 2;
            if (lcp(codes, nn, i, i + (s + t) * d) > dnode) s += t;
        }
        int32_t split = i + s * d + min(d, 0);
        uint32_t left = split == first ? leaf_base + (uint32_t)split : (uint32_t)split;
        uint32_t right = split + 1 == last ? leaf_base + (uint32_t)(split + 1) : (uint32_t)(split + 1);
        karras[2 * ui] = left;
        karras[2 * ui + 1] = right;
        parent[left] = ui;
        parent[right] = ui;
        first_of[ui] = (uint32_t)first;
    }
}

// Bottom-up fit (lbvh.rs:490-525): the second child to arrive at a node
// unions both boxes and continues upward. Also counts, per node, how many
// nodes of its subtree stay internal after the <= max_leaf collapse.
__global__ void k_fit(const float* __restrict__ boxes, const uint32_t* __restrict__ order, uint32_t n,
                      const uint32_t* __restrict__ karras, const uint32_t* __restrict__ parent, float* nbounds,
                      uint32_t* subtree, uint32_t* icount, uint32_t* visits, uint32_t* err, uint32_t max_leaf) {
    const uint32_t leaf_base = n - 1;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float* b = boxes + 6 * (size_t)order[k];
        float* o = nbounds + 6 * (size_t)(leaf_base + k);
        for (int q = 0; q < 6; ++q) o[q] = b[q];
        uint32_t node = parent[leaf_base + k];
        uint32_t steps = 0;
        while (node != kNone) {
            if (node >= leaf_base || ++steps > n) {  // a malformed tree: report, never loop
                atomicExch(err, 2u);
                break;
            }
            __threadfence();
            if (atomicAdd(visits + node, 1u) == 0u) break;
            __threadfence();
            uint32_t l = karras[2 * node], r = karras[2 * node + 1];
            const float* bl = nbounds + 6 * (size_t)l;
            const float* br = nbounds + 6 * (size_t)r;
            float* bo = nbounds + 6 * (size_t)node;
            for (int q = 0; q < 3; ++q) bo[q] = fminf(__ldcg(bl + q), __ldcg(br + q));
            for (int q = 3; q < 6; ++q) bo[q] = fmaxf(__ldcg(bl + q), __ldcg(br + q));
            uint32_t sl = l >= leaf_base ? 1u : __ldcg(subtree + l), sr = r >= leaf_base ? 1u : __ldcg(subtree + r);
            uint32_t il = l >= leaf_base ? 0u : __ldcg(icount + l), ir = r >= leaf_base ? 0u : __ldcg(icount + r);
            uint32_t size = sl + sr;
            subtree[node] = size;
            icount[node] = size > max_leaf ? 1u + il + ir : 0u;
            node = parent[node];
        }
    }
}

// Relayout (lbvh.rs:315-406) without a stack. Node x that stays internal
// after the collapse gets preorder rank r(x) among such nodes (left subtree
// before right, the order the CPU's push-right-then-left DFS visits them);
// its children occupy slots 1 + 2 r(x) and 2 + 2 r(x). r(x) is the number of
// internal ancestors plus, for every ancestor whose right subtree holds x,
// the internal-node count of that ancestor's left subtree. Leaves gather
// their sorted range, so prim_indices is the sorted order itself and a
// leaf's first index is its range start.
__global__ void k_relayout(const uint32_t* __restrict__ karras, const uint32_t* __restrict__ parent,
                           const uint32_t* __restrict__ first_of, const uint32_t* __restrict__ subtree,
                           const uint32_t* __restrict__ icount, const float* __restrict__ nbounds, uint32_t n,
                           float4* __restrict__ nodes, uint32_t* err, uint32_t max_leaf) {
    const uint32_t leaf_base = n - 1;
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < n - 1; x += gridDim.x * blockDim.x) {
        if (subtree[x] <= max_leaf) continue;
        uint32_t r = 0, cur = x, steps = 0;
        while (cur != 0) {
            uint32_t p = parent[cur];
            if (p >= leaf_base || ++steps > n) {
                atomicExch(err, 3u);
                break;
            }
            uint32_t pl = karras[2 * p];
            r += 1u + (karras[2 * p + 1] == cur && pl < leaf_base ? icount[pl] : 0u);
            cur = p;
        }
        if (x == 0) {
            const float* b = nbounds;
            nodes[0] = make_float4(b[0], b[1], b[2], __uint_as_float(1u));
            nodes[1] = make_float4(b[3], b[4], b[5], __uint_as_float(0u));
        }
        for (uint32_t side = 0; side < 2; ++side) {
            uint32_t c = karras[2 * x + side];
            uint32_t slot = 1u + 2u * r + side;
            bool leaf = c >= leaf_base;
            uint32_t size = leaf ? 1u : subtree[c];
            const float* b = nbounds + 6 * (size_t)c;
            uint32_t lf, cnt;
            if (leaf || size <= max_leaf) {
                lf = leaf ? c - leaf_base : first_of[c];
                cnt = size;
            } else {
                uint32_t pl = karras[2 * x];
                uint32_t rc = r + 1u + (side == 1 && pl < leaf_base ? icount[pl] : 0u);
                lf = 1u + 2u * rc;
                cnt = 0u;
            }
            nodes[2 * slot] = make_float4(b[0], b[1], b[2], __uint_as_float(lf));
            nodes[2 * slot + 1] = make_float4(b[3], b[4], b[5], __uint_as_float(cnt));
        }
    }
}
// Root collapsed into one leaf (n <= max_leaf) or n == 1.
__global__ void k_root_leaf(const float* __restrict__ b, uint32_t n, float4* __restrict__ nodes) {
    nodes[0] = make_float4(b[0], b[1], b[2], __uint_as_float(0u));
    nodes[1] = make_float4(b[3], b[4], b[5], __uint_as_float(n));
}

__global__ void k_gather_tris(const GpuTriangle* __restrict__ src, GpuTriangle* __restrict__ dst,
                              const uint32_t* __restrict__ order, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[order[i]];
}

inline int grid_for(uint64_t n, int threads, int sms) {
    uint64_t b = (n + threads - 1) / threads;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, (uint64_t)sms * 32));
}

}  // namespace luc

using namespace luc;

int32_t luc_triangle_boxes_device(luc_ctx* c, const GpuTriangle* tris, const float4* pos, uint32_t n) {
    LUC_CUDA(c, c->lb_boxes.ensure((size_t)n * 6 * sizeof(float)), "alloc boxes");
    if (n) k_tri_bounds<<<grid_for(n, 256, c->num_sms), 256, 0, c->stream>>>(tris, pos, n, c->lb_boxes.as<float>());
    LUC_CUDA(c, cudaGetLastError(), "triangle bounds");
    return LUC_OK;
}

int32_t luc_radix_sort_device(luc_ctx* c, uint32_t n) {
    if (n <= 1) return LUC_OK;
    if (n > kCountMask) return luc_fail(c, LUC_ERR_VALIDATION, "sort: more than 2^30-1 keys");
    cudaStream_t s = c->stream;
    uint32_t tiles = (n + kTile - 1) / kTile;
    LUC_CUDA(c, c->lb_keys2.ensure((size_t)n * 4), "alloc sort");
    LUC_CUDA(c, c->lb_vals2.ensure((size_t)n * 4), "alloc sort");
    LUC_CUDA(c, c->lb_hist.ensure((4 * 256 + 4 * 256 + 8) * 4), "alloc sort");
    // One status row more than the tiles: the look-back test hook (below)
    // numbers the tiles from 1.
    LUC_CUDA(c, c->lb_look.ensure((size_t)(tiles + 1) * 256 * 4), "alloc sort");
    uint32_t* hist = c->lb_hist.as<uint32_t>();
    uint32_t* offs = hist + 1024;
    uint32_t* tcount = hist + 2048;  // [0..3] one tile counter per pass, [4] error flag
    cudaMemsetAsync(hist, 0, (2048 + 8) * 4, s);
    // Test hook (luc_debug_waits, LUC_DEBUG_SORT_ORPHAN_TILE): the first
    // pass's tile counter starts at 1, so tile 0 never runs and tile 1's
    // look-back waits on a flag nothing sets until `spin` polls run out.
    uint32_t spin = kSpinLimit;
    bool orphan = false;
    if (c->dbg_mode == LUC_DEBUG_SORT_ORPHAN_TILE) {
        orphan = true;
        const uint32_t one = 1;
        LUC_CUDA(c, cudaMemcpyAsync(tcount, &one, 4, cudaMemcpyHostToDevice, s), "debug tile counter");
        LUC_CUDA(c, cudaStreamSynchronize(s), "debug tile counter");
        spin = c->dbg_limit;
        c->dbg_mode = 0;
    }
    k_hist4<<<grid_for(n, 256, c->num_sms), 256, 0, s>>>(c->lb_keys.as<uint32_t>(), n, hist);
    k_hist_scan<<<1, 256, 0, s>>>(hist, offs);
    uint32_t *ka = c->lb_keys.as<uint32_t>(), *va = c->lb_vals.as<uint32_t>();
    uint32_t *kb = c->lb_keys2.as<uint32_t>(), *vb = c->lb_vals2.as<uint32_t>();
    // The test hook runs the first pass alone: it is made to fail.
    const int passes = orphan ? 1 : 4;
    for (int p = 0; p < passes; ++p) {
        cudaMemsetAsync(c->lb_look.p, 0, (size_t)(tiles + 1) * 256 * 4, s);
        k_onesweep<<<onesweep_grid(tiles, c->num_sms), kSortThreads, 0, s>>>(
            ka, va, kb, vb, n, 8 * p, offs + 256 * p, c->lb_look.as<uint32_t>(), tcount + p, tcount + 4,
            p == 0 ? spin : kSpinLimit);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    // Four passes: the result is back in lb_keys / lb_vals.
    LUC_CUDA(c, cudaGetLastError(), "radix sort");
    uint32_t errflag = 0;
    LUC_CUDA(c, cudaMemcpyAsync(&errflag, tcount + 4, 4, cudaMemcpyDeviceToHost, s), "sort status");
    LUC_CUDA(c, cudaStreamSynchronize(s), "radix sort");
    if (errflag) return luc_fail(c, LUC_ERR_VALIDATION, "radix sort: look-back wait gave up");
    return LUC_OK;
}

// LBVH over the n boxes in lb_boxes -> lb_nodes (tree), lb_vals (order),
// lb_codes (codes in input order), lb_karras / lb_parent / lb_nbounds /
// lb_subtree, lb_misc[0..6) centroid bounds.
int32_t luc_lbvh_device(luc_ctx* c, uint32_t n, uint32_t* num_nodes, uint32_t max_leaf) {
    cudaStream_t s = c->stream;
    *num_nodes = 0;
    if (n == 0) return LUC_OK;
    const int sms = c->num_sms;
    uint32_t nb = (uint32_t)std::min<uint64_t>((n + 255) / 256, 1024);
    LUC_CUDA(c, c->lb_misc.ensure((6 + 6 * (size_t)nb + 1) * 4), "alloc lbvh");
    LUC_CUDA(c, c->lb_keys.ensure((size_t)n * 4), "alloc lbvh");
    LUC_CUDA(c, c->lb_vals.ensure((size_t)n * 4), "alloc lbvh");
    LUC_CUDA(c, c->lb_codes.ensure((size_t)n * 4), "alloc lbvh");
    LUC_CUDA(c, c->lb_nodes.ensure((size_t)(2 * n) * sizeof(GpuBvhNode)), "alloc lbvh");
    float* cb = c->lb_misc.as<float>();
    k_cbounds_partial<<<nb, 256, 0, s>>>(c->lb_boxes.as<float>(), n, cb + 6);
    k_cbounds_final<<<1, 256, 0, s>>>(cb + 6, nb, cb);
    k_morton<<<grid_for(n, 256, sms), 256, 0, s>>>(c->lb_boxes.as<float>(), n, cb, c->lb_keys.as<uint32_t>(),
                                                   c->lb_vals.as<uint32_t>(), c->lb_codes.as<uint32_t>());
    LUC_CUDA(c, cudaGetLastError(), "morton");
    int32_t rc = luc_radix_sort_device(c, n);
    if (rc) return rc;
    if (n <= max_leaf) {
        // The whole tree collapses into the root leaf (Lbvh::build n == 1, or
        // relayout with count <= max_leaf at the root). Its bounds are the
        // union of every box, which the fit computes for n > 1.
        if (n == 1) {
            k_root_leaf<<<1, 1, 0, s>>>(c->lb_boxes.as<float>(), 1, c->lb_nodes.as<float4>());
            LUC_CUDA(c, c->lb_nbounds.ensure(6 * 4), "alloc lbvh");
            LUC_CUDA(c, cudaMemcpyAsync(c->lb_nbounds.p, c->lb_boxes.p, 24, cudaMemcpyDeviceToDevice, s), "lbvh");
            *num_nodes = 1;
            LUC_CUDA(c, cudaGetLastError(), "lbvh root");
            return LUC_OK;
        }
    }
    LUC_CUDA(c, c->lb_karras.ensure((size_t)2 * (n - 1) * 4), "alloc lbvh");
    LUC_CUDA(c, c->lb_parent.ensure((size_t)(2 * n - 1) * 4), "alloc lbvh");
    LUC_CUDA(c, c->lb_rank.ensure((size_t)(n - 1) * 4), "alloc lbvh");
    LUC_CUDA(c, c->lb_nbounds.ensure((size_t)(2 * n - 1) * 6 * 4), "alloc lbvh");
    LUC_CUDA(c, c->lb_subtree.ensure((size_t)(n - 1) * 4), "alloc lbvh");
    LUC_CUDA(c, c->lb_icount.ensure((size_t)(n - 1) * 4), "alloc lbvh");
    LUC_CUDA(c, c->lb_flags.ensure((size_t)(n - 1) * 4), "alloc lbvh");
    cudaMemsetAsync(c->lb_parent.p, 0xFF, (size_t)(2 * n - 1) * 4, s);
    cudaMemsetAsync(c->lb_flags.p, 0, (size_t)(n - 1) * 4, s);
    uint32_t* errp = (uint32_t*)(c->lb_misc.as<float>() + 6 + 6 * (size_t)nb);
    cudaMemsetAsync(errp, 0, 4, s);
    k_karras<<<grid_for(n - 1, 256, sms), 256, 0, s>>>(c->lb_keys.as<uint32_t>(), n, c->lb_karras.as<uint32_t>(),
                                                       c->lb_parent.as<uint32_t>(), c->lb_rank.as<uint32_t>());
    k_fit<<<grid_for(n, 256, sms), 256, 0, s>>>(c->lb_boxes.as<float>(), c->lb_vals.as<uint32_t>(), n,
                                                c->lb_karras.as<uint32_t>(), c->lb_parent.as<uint32_t>(),
                                                c->lb_nbounds.as<float>(), c->lb_subtree.as<uint32_t>(),
                                                c->lb_icount.as<uint32_t>(), c->lb_flags.as<uint32_t>(), errp,
                                                max_leaf);
    if (n <= max_leaf) {
        k_root_leaf<<<1, 1, 0, s>>>(c->lb_nbounds.as<float>(), n, c->lb_nodes.as<float4>());
        *num_nodes = 1;
    } else {
        k_relayout<<<grid_for(n - 1, 256, sms), 256, 0, s>>>(
            c->lb_karras.as<uint32_t>(), c->lb_parent.as<uint32_t>(), c->lb_rank.as<uint32_t>(),
            c->lb_subtree.as<uint32_t>(), c->lb_icount.as<uint32_t>(), c->lb_nbounds.as<float>(), n,
            c->lb_nodes.as<float4>(), errp, max_leaf);
        uint32_t root_internal = 0;
        LUC_CUDA(c, cudaMemcpyAsync(&root_internal, c->lb_icount.p, 4, cudaMemcpyDeviceToHost, s), "lbvh count");
        *num_nodes = 1u + 2u * root_internal;
    }
    uint32_t errv = 0;
    LUC_CUDA(c, cudaMemcpyAsync(&errv, errp, 4, cudaMemcpyDeviceToHost, s), "lbvh status");
    LUC_CUDA(c, cudaStreamSynchronize(s), "lbvh");
    if (errv) return luc_fail(c, LUC_ERR_VALIDATION, "lbvh: malformed hierarchy (status " + std::to_string(errv) + ")");
    LUC_CUDA(c, cudaGetLastError(), "lbvh");
    return LUC_OK;
}

int32_t luc_gather_triangles(luc_ctx* c, const GpuTriangle* src, GpuTriangle* dst, const uint32_t* order, uint32_t n) {
    if (n) k_gather_tris<<<grid_for(n, 256, c->num_sms), 256, 0, c->stream>>>(src, dst, order, n);
    LUC_CUDA(c, cudaGetLastError(), "gather triangles");
    return LUC_OK;
}

static int32_t copy_out(luc_ctx* c, uint32_t n, uint32_t num_nodes, luc_lbvh_out* o) {
    cudaStream_t s = c->stream;
    auto d2h = [&](void* dst, const DevBuf& src, size_t bytes) -> cudaError_t {
        if (!dst || bytes == 0) return cudaSuccess;
        return cudaMemcpyAsync(dst, src.p, bytes, cudaMemcpyDeviceToHost, s);
    };
    LUC_CUDA(c, d2h(o->codes, c->lb_codes, (size_t)n * 4), "read codes");
    LUC_CUDA(c, d2h(o->order, c->lb_vals, (size_t)n * 4), "read order");
    LUC_CUDA(c, d2h(o->prim_indices, c->lb_vals, (size_t)n * 4), "read prim indices");
    LUC_CUDA(c, d2h(o->scene_bounds, c->lb_misc, 24), "read scene bounds");
    LUC_CUDA(c, d2h(o->nodes, c->lb_nodes, (size_t)num_nodes * sizeof(GpuBvhNode)), "read nodes");
    if (n > 1) {
        LUC_CUDA(c, d2h(o->karras, c->lb_karras, (size_t)2 * (n - 1) * 4), "read karras");
        LUC_CUDA(c, d2h(o->parent, c->lb_parent, (size_t)(2 * n - 1) * 4), "read parent");
        LUC_CUDA(c, d2h(o->node_bounds, c->lb_nbounds, (size_t)(2 * n - 1) * 24), "read bounds");
        LUC_CUDA(c, d2h(o->subtree_size, c->lb_subtree, (size_t)(n - 1) * 4), "read subtree");
    } else if (n == 1) {
        if (o->parent) o->parent[0] = kNone;
        LUC_CUDA(c, d2h(o->node_bounds, c->lb_nbounds, 24), "read bounds");
    }
    LUC_CUDA(c, cudaStreamSynchronize(s), "lbvh readback");
    o->num_nodes = num_nodes;
    return LUC_OK;
}

extern "C" {

int32_t luc_lbvh_build(luc_ctx* c, const GpuTriangle* tris, uint32_t n, const float* positions, uint32_t nv,
                       luc_lbvh_out* out) {
    if (!c || !out || (n && (!tris || !positions))) return LUC_ERR_VALIDATION;
    cudaSetDevice(c->device);
    for (uint32_t i = 0; i < n; ++i)
        if (tris[i].i0 >= nv || tris[i].i1 >= nv || tris[i].i2 >= nv)
            return luc_fail(c, LUC_ERR_VALIDATION, "triangle " + std::to_string(i) + " indexes out of range");
    cudaStream_t s = c->stream;
    LUC_CUDA(c, c->lb_tris.ensure((size_t)n * sizeof(GpuTriangle)), "alloc");
    LUC_CUDA(c, c->lb_pos.ensure((size_t)nv * 16), "alloc");
    if (n) LUC_CUDA(c, cudaMemcpyAsync(c->lb_tris.p, tris, (size_t)n * 16, cudaMemcpyHostToDevice, s), "upload");
    if (nv) LUC_CUDA(c, cudaMemcpyAsync(c->lb_pos.p, positions, (size_t)nv * 16, cudaMemcpyHostToDevice, s), "upload");
    int32_t rc = luc_triangle_boxes_device(c, c->lb_tris.as<GpuTriangle>(), c->lb_pos.as<float4>(), n);
    if (rc) return rc;
    uint32_t nn = 0;
    rc = luc_lbvh_device(c, n, &nn);
    if (rc) return rc;
    return copy_out(c, n, nn, out);
}

int32_t luc_lbvh_build_boxes(luc_ctx* c, const float* boxes, uint32_t n, luc_lbvh_out* out) {
    if (!c || !out || (n && !boxes)) return LUC_ERR_VALIDATION;
    cudaSetDevice(c->device);
    LUC_CUDA(c, c->lb_boxes.ensure((size_t)n * 24), "alloc");
    if (n) LUC_CUDA(c, cudaMemcpyAsync(c->lb_boxes.p, boxes, (size_t)n * 24, cudaMemcpyHostToDevice, c->stream), "upload");
    uint32_t nn = 0;
    int32_t rc = luc_lbvh_device(c, n, &nn);
    if (rc) return rc;
    return copy_out(c, n, nn, out);
}

int32_t luc_sort_u32(luc_ctx* c, const uint32_t* keys, const uint32_t* vals, uint32_t n, uint32_t* ko, uint32_t* vo) {
    if (!c || (n && (!keys || !vals || !ko || !vo))) return LUC_ERR_VALIDATION;
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    LUC_CUDA(c, c->lb_keys.ensure((size_t)n * 4), "alloc");
    LUC_CUDA(c, c->lb_vals.ensure((size_t)n * 4), "alloc");
    if (n) {
        LUC_CUDA(c, cudaMemcpyAsync(c->lb_keys.p, keys, (size_t)n * 4, cudaMemcpyHostToDevice, s), "upload");
        LUC_CUDA(c, cudaMemcpyAsync(c->lb_vals.p, vals, (size_t)n * 4, cudaMemcpyHostToDevice, s), "upload");
    }
    int32_t rc = luc_radix_sort_device(c, n);
    if (rc) return rc;
    if (n) {
        LUC_CUDA(c, cudaMemcpyAsync(ko, c->lb_keys.p, (size_t)n * 4, cudaMemcpyDeviceToHost, s), "readback");
        LUC_CUDA(c, cudaMemcpyAsync(vo, c->lb_vals.p, (size_t)n * 4, cudaMemcpyDeviceToHost, s), "readback");
    }
    LUC_CUDA(c, cudaStreamSynchronize(s), "sort");
    return LUC_OK;
}

// Sorts caller device arrays in place (copies through the context's
// scratch; the caller's arrays hold the result on return).
int32_t luc_sort_u32_dev(luc_ctx* c, void* keys_dev, void* vals_dev, uint32_t n) {
    if (!c || (n && (!keys_dev || !vals_dev))) return LUC_ERR_VALIDATION;
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    LUC_CUDA(c, c->lb_keys.ensure((size_t)n * 4), "alloc");
    LUC_CUDA(c, c->lb_vals.ensure((size_t)n * 4), "alloc");
    if (n) {
        LUC_CUDA(c, cudaMemcpyAsync(c->lb_keys.p, keys_dev, (size_t)n * 4, cudaMemcpyDeviceToDevice, s), "copy");
        LUC_CUDA(c, cudaMemcpyAsync(c->lb_vals.p, vals_dev, (size_t)n * 4, cudaMemcpyDeviceToDevice, s), "copy");
    }
    int32_t rc = luc_radix_sort_device(c, n);
    if (rc) return rc;
    if (n) {
        LUC_CUDA(c, cudaMemcpyAsync(keys_dev, c->lb_keys.p, (size_t)n * 4, cudaMemcpyDeviceToDevice, s), "copy");
        LUC_CUDA(c, cudaMemcpyAsync(vals_dev, c->lb_vals.p, (size_t)n * 4, cudaMemcpyDeviceToDevice, s), "copy");
    }
    LUC_CUDA(c, cudaStreamSynchronize(s), "sort");
    return LUC_OK;
}

}  // extern "C"
