// Device-bounded stable LSD radix sort (onesweep) of 64-bit keys with int32
// values, used by the LBVH build to order surfels along the Morton curve.
//
// The emitted count is read on the device, so a sort needs no host
// synchronisation and can be captured in a CUDA graph.  One histogram launch
// covers every pass; each onesweep launch handles one 8-bit digit: a
// partition of kSortTile keys ranks its keys stably with warp match/ballot,
// publishes per-digit counts, resolves its global offsets by decoupled
// look-back over earlier partitions and scatters through shared memory so
// that stores are coalesced.  Keys are either used as they are
// (SortKeyMap.raw) or mapped to the composite (tile, depth_bits - near_bits)
// digits of the tile-intersection keys.
#include "vgr_kernels.h"

namespace vgr {

constexpr uint64_t kSortDescAggregate = 1ull << 62;
constexpr uint64_t kSortDescInclusive = 2ull << 62;
constexpr uint64_t kSortDescCount = (1ull << 62) - 1;

__device__ __forceinline__ int64_t sort_count(const SortParams& p) {
  int64_t n = p.counters[1];
  if (n > p.capacity) n = p.capacity;
  if (n < 0) n = 0;
  return n;
}

__global__ void __launch_bounds__(kSortThreads) sort_histogram_kernel(SortParams p) {
  __shared__ uint32_t s_hist[kMaxSortPasses][kRadixBins];
  const int tid = threadIdx.x;
  for (int i = tid; i < kMaxSortPasses * kRadixBins; i += kSortThreads) {
    (&s_hist[0][0])[i] = 0u;
  }
  __syncthreads();
  const int64_t n = sort_count(p);
  const int64_t parts = (n + kSortTile - 1) / kSortTile;
  uint64_t* desc = reinterpret_cast<uint64_t*>(p.scratch + p.layout.sort_desc);
  const int64_t max_parts = p.layout.max_partitions;
  for (int64_t part = blockIdx.x; part < parts; part += gridDim.x) {
    // Clear this partition's look-back descriptors of every pass.
    for (int i = tid; i < p.passes * kRadixBins; i += kSortThreads) {
      const int pass = i / kRadixBins;
      const int digit = i - pass * kRadixBins;
      desc[(static_cast<int64_t>(pass) * max_parts + part) * kRadixBins + digit] = 0ull;
    }
    const int64_t begin = part * kSortTile;
    for (int k = 0; k < kSortItems; ++k) {
      const int64_t idx = begin + k * kSortThreads + tid;
      if (idx < n) {
        const uint64_t ck = composite_key(p.keys_in[idx], p.map);
        for (int pass = 0; pass < p.passes; ++pass) {
          atomicAdd(&s_hist[pass][(ck >> (pass * kRadixBits)) & (kRadixBins - 1)], 1u);
        }
      }
    }
  }
  __syncthreads();
  uint32_t* hist = reinterpret_cast<uint32_t*>(p.scratch + p.layout.sort_hist);
  for (int i = tid; i < p.passes * kRadixBins; i += kSortThreads) {
    const uint32_t v = (&s_hist[0][0])[i];
    if (v) atomicAdd(hist + i, v);
  }
}

__global__ void __launch_bounds__(kSortThreads, 3) sort_onesweep_kernel(SortParams p) {
  constexpr int kWarps = kSortThreads / 32;
  __shared__ uint32_t s_warp_hist[kWarps][kRadixBins];
  extern __shared__ __align__(16) unsigned char s_dynamic[];
  uint64_t* s_keys = reinterpret_cast<uint64_t*>(s_dynamic);
  int32_t* s_vals = reinterpret_cast<int32_t*>(s_dynamic + kSortTile * sizeof(uint64_t));
  __shared__ uint32_t s_global_excl[kRadixBins];
  __shared__ uint64_t s_scatter_base[kRadixBins];
  __shared__ uint32_t s_digit_start[kRadixBins];
  __shared__ uint32_t s_scan[kWarps];
  __shared__ int64_t s_part;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  ScratchHeader* header = reinterpret_cast<ScratchHeader*>(p.scratch + p.layout.header);
  uint64_t* desc = reinterpret_cast<uint64_t*>(p.scratch + p.layout.sort_desc) +
                   static_cast<int64_t>(p.pass) * p.layout.max_partitions * kRadixBins;
  const int64_t n = sort_count(p);
  const int64_t parts = (n + kSortTile - 1) / kSortTile;
  const int shift = p.pass * kRadixBits;

  // Exclusive scan of this pass's global digit histogram (one digit/thread).
  {
    const uint32_t* hist =
        reinterpret_cast<const uint32_t*>(p.scratch + p.layout.sort_hist) + p.pass * kRadixBins;
    uint32_t v = hist[tid];
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) s_scan[warp] = incl;
    __syncthreads();
    uint32_t wp = 0;
    for (int w = 0; w < warp; ++w) wp += s_scan[w];
    s_global_excl[tid] = wp + incl - v;
    __syncthreads();
  }

  while (true) {
    if (tid == 0) s_part = atomicAdd(&header->sort_queue[p.pass], 1u);
    for (int i = tid; i < kWarps * kRadixBins; i += kSortThreads) (&s_warp_hist[0][0])[i] = 0u;
    __syncthreads();
    const int64_t part = s_part;
    if (part >= parts) break;
    const int64_t begin = part * kSortTile;

    // Items in (warp, k, lane) order; digit and in-warp rank packed as
    // digit << 16 | rank (digit 0x1ff marks an item past the end).
    uint64_t keys[kSortItems];
    int32_t vals[kSortItems];
    uint32_t dr[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
      const int64_t idx = begin + warp * (kSortItems * 32) + k * 32 + lane;
      const bool valid = idx < n;
      keys[k] = valid ? p.keys_in[idx] : 0ull;
      vals[k] = valid ? p.values_in[idx] : 0;
    }
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
      const int64_t idx = begin + warp * (kSortItems * 32) + k * 32 + lane;
      const bool valid = idx < n;
      const uint32_t d = valid
          ? static_cast<uint32_t>((composite_key(keys[k], p.map) >> shift) & (kRadixBins - 1))
          : (kRadixBins + lane);  // unique per lane: matches nothing valid
      const uint32_t peers = __match_any_sync(0xffffffffu, d);
      uint32_t old = 0;
      if (valid) old = s_warp_hist[warp][d];
      __syncwarp();
      if (valid && lane == (__ffs(peers) - 1)) s_warp_hist[warp][d] = old + __popc(peers);
      __syncwarp();
      dr[k] = valid ? ((d << 16) | (old + __popc(peers & lt))) : (0x1ffu << 16);
    }
    __syncthreads();
    // Per digit: exclusive prefix across warps and the partition total.
    const int d = tid;  // kSortThreads == kRadixBins
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t t = s_warp_hist[w][d];
      s_warp_hist[w][d] = total;
      total += t;
    }
    uint64_t* my_desc = desc + part * kRadixBins + d;
    if (part == 0) {
      st_release_u64(my_desc, kSortDescInclusive | total);
    } else {
      st_release_u64(my_desc, kSortDescAggregate | total);
    }
    // Block exclusive scan of totals over digits (for the shared reorder).
    {
      uint32_t incl = total;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (lane == 31) s_scan[warp] = incl;
      __syncthreads();
      uint32_t wp = 0;
      for (int w = 0; w < warp; ++w) wp += s_scan[w];
      s_digit_start[d] = wp + incl - total;
    }
    // Decoupled look-back for digit d.
    uint64_t prefix = 0;
    if (part > 0) {
      int64_t j = part - 1;
      uint32_t spins = 0;
      while (j >= 0) {
        const uint64_t v = ld_acquire_u64(desc + j * kRadixBins + d);
        const uint64_t flag = v >> 62;
        if (flag == 0) {
          if (++spins > kSpinLimit) {
            atomicOr(&header->status, kDeviceErrorLookback);
            break;
          }
          continue;
        }
        prefix += v & kSortDescCount;
        if (flag == 2) break;
        --j;
      }
      st_release_u64(my_desc, kSortDescInclusive | (prefix + total));
    }
    s_scatter_base[d] = static_cast<uint64_t>(s_global_excl[d]) + prefix;
    __syncthreads();
    // Reorder the partition by digit in shared memory.
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
      const uint32_t dk = dr[k] >> 16;
      if (dk < kRadixBins) {
        const uint32_t pos = s_digit_start[dk] + s_warp_hist[warp][dk] + (dr[k] & 0xffffu);
        s_keys[pos] = keys[k];
        s_vals[pos] = vals[k];
      }
    }
    __syncthreads();
    const int64_t remaining = n - begin;
    const int count = remaining < kSortTile ? static_cast<int>(remaining) : kSortTile;
    for (int i = tid; i < count; i += kSortThreads) {
      const uint64_t key = s_keys[i];
      const uint32_t dk =
          static_cast<uint32_t>((composite_key(key, p.map) >> shift) & (kRadixBins - 1));
      const uint64_t g = s_scatter_base[dk] + (i - s_digit_start[dk]);
      if (g < static_cast<uint64_t>(n)) {
        p.keys_out[g] = key;
        p.values_out[g] = s_vals[i];
      }
    }
    __syncthreads();
  }
}

}  // namespace vgr
