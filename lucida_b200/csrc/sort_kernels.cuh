// The onesweep radix-sort kernels (defined in lbvh.cu), for the files that
// drive them.
#pragma once
#include <cstdint>

namespace luc {

constexpr int kSortThreads = 256;
constexpr int kSortKpt = 16;
constexpr uint32_t kTile = kSortThreads * kSortKpt;  // keys per block tile
constexpr uint32_t kFlagAgg = 1u << 30, kFlagInc = 2u << 30, kCountMask = (1u << 30) - 1u;
constexpr uint32_t kSpinLimit = 1u << 24;
constexpr int kLookWin = 4;  // look-back predecessors read per round trip
constexpr int kOnesweepBlocksPerSm = 4;

// k_onesweep's grid: persistent blocks, four per SM (what 64 registers and
// 45 KB of shared memory allow), at most one per tile.
inline unsigned onesweep_grid(uint32_t tiles, int sms) {
    const uint32_t g = (uint32_t)sms * kOnesweepBlocksPerSm;
    return tiles < g ? tiles : g;
}

// Digit histograms of all four 8-bit passes (hist: 4 x 256, zeroed by the caller).
__global__ void k_hist4(const uint32_t* __restrict__ keys, uint32_t n, uint32_t* __restrict__ hist);
// Exclusive scan of each pass's 256 counts into offsets (one block of 256 threads).
__global__ void k_hist_scan(const uint32_t* __restrict__ hist, uint32_t* __restrict__ offsets);
// One stable pass over digit (key >> shift) & 255, by onesweep_grid(tiles)
// persistent blocks; `status` (tiles x 256) and `tile_counter` must be zero
// on entry; *err is set if a look-back wait gives
// up after `spin_limit` polls of a predecessor that has not published
// (kSpinLimit in every product call).
__global__ void __launch_bounds__(kSortThreads, 4) k_onesweep(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                           uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, uint32_t n, int shift,
                           const uint32_t* __restrict__ digit_offsets, uint32_t* status, uint32_t* tile_counter,
                           uint32_t* err, uint32_t spin_limit);

}  // namespace luc
