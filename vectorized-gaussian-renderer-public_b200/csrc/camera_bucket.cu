// Tile-bucket sort of the tile intersections and the tile ranges.
//
// The reference orders the 64-bit keys (global tile << 32 | float bits of
// depth) with a host count read plus CUB DeviceRadixSort
// (src/isaacsim_gaussian_renderer/native/renderer_cuda.cu:3215-3269), or in
// its deterministic mode with count/scan/scatter/segmented sort
// (:1831-1906, :1944-1971, :3288-3381), then derives the tile ranges
// (:1908-1942).  Both produce the order (tile, depth bits, Gaussian id).
//
// Here the tile is never a radix digit.  The projection kernel counts each
// tile's keys while it emits them, so after one scan of the counts every
// tile's range [start, end) is known before any key moves:
//   tile_span_*_kernel    counts -> starts, ends (= scatter cursors), active
//                         tile count and the bucket total;
//   bucket_scatter_kernel one read of the emitted keys, each (depth bits,
//                         record index) pair claims a slot of its tile's
//                         bucket with an atomic cursor;
//   tile_sort_kernel      one CTA per tile orders its bucket by (depth bits,
//                         record index) - in shared memory when it holds at
//                         most kTileSortCap pairs, else split by depth
//                         through global memory into runs sorted in shared
//                         memory - and writes the sorted keys and record
//                         indices.
// Within a tile the record index increases with the Gaussian id (records are
// compacted in Gaussian order per camera), so (depth bits, record) is the
// reference order, and it is a total order: the arbitrary order in which the
// atomic cursors fill a bucket does not reach the result, and no step of the
// tile sort needs to be stable.
//
// Traffic per key: 12 bytes read and 8 written by the scatter, 8 read and 12
// written by the tile sort, against 24 bytes per radix pass (6 passes for a
// 44-bit key at 64 cameras of 640x480) of the global sort.
#include <type_traits>

#include "../../include/vgr_b200.h"
#include "vgr_kernels.h"

namespace vgr {
namespace {

constexpr int kTsWarps = kTileSortThreads / 32;
constexpr uint32_t kNoDigit = 0xffffu;
static_assert(kTileSortThreads == kRadixBins, "one digit per thread in the digit scans");
static_assert(kTileSortCap <= 65536, "ranks are packed in 16 bits");

struct RankSmem {
  uint32_t warp_hist[kTsWarps][kRadixBins];
  uint32_t digit_start[kRadixBins];
  uint32_t scan[kTsWarps];
};

// Digit of one LSD pass over a bucket entry (depth bits << 32 | record
// index, so that integer order is the reference order), relative to the
// tile's minimum of the word.
struct PassDigit {
  int use_record;
  uint32_t base;
  int shift;
  __device__ __forceinline__ uint32_t operator()(uint64_t v) const {
    const uint32_t word = use_record ? static_cast<uint32_t>(v) : static_cast<uint32_t>(v >> 32);
    return ((word - base) >> shift) & (kRadixBins - 1);
  }
};

__device__ __forceinline__ int bit_length_u32(uint32_t v) { return v ? 32 - __clz(v) : 0; }

// Stable rank of one chunk of m items held warp-blocked in registers: item k
// of lane l in warp w is chunk element (w * K + k) * 32 + l.  On return
// warp_hist[w][d] is the count of digit d in warps < w, digit_start[d] the
// count of digits < d, dr[k] = digit << 16 | rank among the warp's earlier
// items of that digit, and the result is this thread's digit total.
// warp_hist must be zero on entry.
template <int kItems>
__device__ __forceinline__ uint32_t rank_chunk(const uint64_t (&it)[kItems], uint32_t (&dr)[kItems],
                                               int K, int m, PassDigit dig, RankSmem& s) {
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    if (k >= K) break;
    const int idx = (warp * K + k) * 32 + lane;
    const bool valid = idx < m;
    const uint32_t d = valid ? dig(it[k]) : (kRadixBins + lane);
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t old = 0;
    if (valid) old = s.warp_hist[warp][d];
    __syncwarp();
    if (valid && lane == __ffs(peers) - 1) s.warp_hist[warp][d] = old + __popc(peers);
    __syncwarp();
    dr[k] = valid ? ((d << 16) | (old + __popc(peers & lt))) : (kNoDigit << 16);
  }
  __syncthreads();
  const int d = tid;
  uint32_t total = 0;
#pragma unroll
  for (int w = 0; w < kTsWarps; ++w) {
    const uint32_t t = s.warp_hist[w][d];
    s.warp_hist[w][d] = total;
    total += t;
  }
  uint32_t incl = total;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s.scan[warp] = incl;
  __syncthreads();
  uint32_t wp = 0;
#pragma unroll
  for (int w = 0; w < kTsWarps; ++w) wp += w < warp ? s.scan[w] : 0u;
  s.digit_start[d] = wp + incl - total;
  __syncthreads();
  return total;
}

// Block-wide min/max of four words; every thread gets the result.
__device__ __forceinline__ void block_minmax(uint32_t& dmin, uint32_t& dmax, uint32_t& rmin,
                                             uint32_t& rmax, uint32_t (*s)[kTsWarps]) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  dmin = __reduce_min_sync(0xffffffffu, dmin);
  dmax = __reduce_max_sync(0xffffffffu, dmax);
  rmin = __reduce_min_sync(0xffffffffu, rmin);
  rmax = __reduce_max_sync(0xffffffffu, rmax);
  if (lane == 0) {
    s[0][warp] = dmin;
    s[1][warp] = dmax;
    s[2][warp] = rmin;
    s[3][warp] = rmax;
  }
  __syncthreads();
#pragma unroll
  for (int w = 0; w < kTsWarps; ++w) {
    dmin = min(dmin, s[0][w]);
    dmax = max(dmax, s[1][w]);
    rmin = min(rmin, s[2][w]);
    rmax = max(rmax, s[3][w]);
  }
}

}  // namespace

// Counts -> exclusive starts, cursors, active tiles and bucket total, in
// three passes over spans of kTileScanSpan tiles (one CTA per span; a
// single CTA walking every tile took 0.21 ms on a 154k-tile frame).
namespace {

// Sum of a block's values (all threads get it).
template <int kThreads>
__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* s_warp) {
  v = __reduce_add_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = v;
  __syncthreads();
  uint32_t total = 0;
#pragma unroll
  for (int w = 0; w < kThreads / 32; ++w) total += s_warp[w];
  __syncthreads();
  return total;
}

}  // namespace

// Pass 1: each CTA sums its span's counts into the span's first tile_starts
// slot (free until pass 3 writes the span) and adds its active tiles to the
// frame's total.
__global__ void __launch_bounds__(kTileSpanThreads) tile_span_sum_kernel(BucketParams p) {
  __shared__ uint32_t s_warp[kTileSpanThreads / 32];
  ScratchHeader* header = reinterpret_cast<ScratchHeader*>(p.scratch + p.layout.header);
  const uint32_t* counts = reinterpret_cast<const uint32_t*>(p.tile_ends);
  const int64_t first = static_cast<int64_t>(blockIdx.x) * kTileScanSpan;
  uint32_t sum = 0, active = 0;
#pragma unroll
  for (int k = 0; k < kTileScanItems; ++k) {
    const int64_t t = first + k * kTileSpanThreads + threadIdx.x;
    const uint32_t c = t < p.tile_count ? counts[t] : 0u;
    sum += c;
    active += c != 0u ? 1u : 0u;
  }
  sum = block_sum<kTileSpanThreads>(sum, s_warp);
  active = block_sum<kTileSpanThreads>(active, s_warp);
  if (threadIdx.x == 0 && first < p.tile_count) {
    p.tile_starts[first] = static_cast<int32_t>(sum);
    if (active) atomicAdd(&header->active_tiles, active);
  }
}

// Pass 2 (one CTA): exclusive scan of the span sums in place, the bucket
// total and the frame counters.
__global__ void __launch_bounds__(kTileScanThreads) tile_span_scan_kernel(BucketParams p, int64_t spans) {
  __shared__ uint32_t s_warp[kTileScanThreads / 32];
  __shared__ uint32_t s_carry;
  ScratchHeader* header = reinterpret_cast<ScratchHeader*>(p.scratch + p.layout.header);
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  if (tid == 0) s_carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < spans; base += kTileScanThreads) {
    const int64_t s = base + tid;
    const uint32_t v = s < spans ? static_cast<uint32_t>(p.tile_starts[s * kTileScanSpan]) : 0u;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = s_warp[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += t;
      }
      s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t carry = s_carry;
    if (s < spans) p.tile_starts[s * kTileScanSpan] = static_cast<int32_t>(carry + (warp > 0 ? s_warp[warp - 1] : 0u) + incl - v);
    __syncthreads();
    if (tid == kTileScanThreads - 1) s_carry = carry + s_warp[kTileScanThreads / 32 - 1];
    __syncthreads();
  }
  if (tid == 0) {
    header->bucket_total = s_carry;
    p.counters[VGR_COUNTER_ACTIVE_TILES] = static_cast<int64_t>(header->active_tiles);
    // Frame counters from the projection's reservations.
    const uint64_t tv = header->visible_total;
    const uint64_t ti = header->isect_total;
    const uint64_t vcap = static_cast<uint64_t>(p.visible_capacity);
    const uint64_t icap = static_cast<uint64_t>(p.capacity);
    p.counters[0] = static_cast<int64_t>(tv);
    p.counters[1] = static_cast<int64_t>(ti);
    p.counters[2] = tv > vcap ? static_cast<int64_t>(tv - vcap) : 0;
    p.counters[3] = ti > icap ? static_cast<int64_t>(ti - icap) : 0;
  }
}

// Pass 3: each CTA scans its span (thread t holds tiles [16 t, 16 t + 16)
// of it) from the span's offset and writes starts and cursors.  The offset
// sits in the span's first starts slot, read before any thread writes.
__global__ void __launch_bounds__(kTileSpanThreads) tile_span_apply_kernel(BucketParams p) {
  __shared__ uint32_t s_warp[kTileSpanThreads / 32];
  __shared__ uint32_t s_offset;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int64_t span_first = static_cast<int64_t>(blockIdx.x) * kTileScanSpan;
  if (tid == 0) s_offset = static_cast<uint32_t>(p.tile_starts[span_first]);
  const uint32_t* counts = reinterpret_cast<const uint32_t*>(p.tile_ends);
  const int64_t tiles = p.tile_count;
  const int64_t first = span_first + static_cast<int64_t>(tid) * kTileScanItems;
  uint32_t c[kTileScanItems];
  uint32_t sum = 0;
#pragma unroll
  for (int k = 0; k < kTileScanItems; ++k) {
    c[k] = first + k < tiles ? counts[first + k] : 0u;
    sum += c[k];
  }
  uint32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  uint32_t prefix = s_offset + incl - sum;
#pragma unroll
  for (int w = 0; w < kTileSpanThreads / 32; ++w) prefix += w < warp ? s_warp[w] : 0u;
#pragma unroll
  for (int k = 0; k < kTileScanItems; ++k) {
    if (first + k < tiles) {
      p.tile_starts[first + k] = static_cast<int32_t>(prefix);
      p.tile_ends[first + k] = static_cast<int32_t>(prefix);
    }
    prefix += c[k];
  }
}

// Each emitted key claims a slot in its tile's bucket; keys whose tile is out
// of range (records past the visible capacity) go after the buckets.  A warp
// handles 32 consecutive keys at a time: lanes whose keys share a tile (the
// keys of neighbouring records, which the projection emits side by side)
// claim their slots with one atomic by the group's first lane, which hands
// out base + rank.  A thread claims the slots of kBatch keys before it
// stores any of them, so the claims of its batch are in flight together.
__global__ void __launch_bounds__(256, 4) bucket_scatter_kernel(BucketParams p) {
  constexpr int kBatch = 8;
  ScratchHeader* header = reinterpret_cast<ScratchHeader*>(p.scratch + p.layout.header);
  int64_t n = p.counters[1];
  if (n > p.capacity) n = p.capacity;
  if (n < 0) n = 0;
  const uint32_t bucket_total = header->bucket_total;
  uint32_t* cursors = reinterpret_cast<uint32_t*>(p.tile_ends);
  const uint64_t tiles = static_cast<uint64_t>(p.tile_count);
  const int lane = threadIdx.x & 31;
  const uint32_t below = lanemask_lt();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x * kBatch;
  // Warp-uniform loop: every lane runs the same iterations (the shuffles
  // below take the full mask); keys past n are masked per lane.
  for (int64_t wbase = static_cast<int64_t>(blockIdx.x) * blockDim.x * kBatch + (threadIdx.x & ~31);
       wbase < n; wbase += stride) {
    uint64_t key[kBatch];
    int32_t value[kBatch];
    uint64_t pos[kBatch];
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      const int64_t i = wbase + b * static_cast<int64_t>(blockDim.x) + lane;
      key[b] = i < n ? p.keys_in[i] : ~0ull;
      value[b] = i < n ? p.values_in[i] : 0;
    }
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      const int64_t i = wbase + b * static_cast<int64_t>(blockDim.x) + lane;
      const bool valid = i < n;
      const uint64_t tile = valid ? key[b] >> 32 : ~0ull;
      const uint32_t peers = __match_any_sync(0xffffffffu, tile);
      const int leader = __ffs(peers) - 1;
      uint32_t claim = 0u;
      if (valid && lane == leader) {
        const uint32_t count = static_cast<uint32_t>(__popc(peers));
        claim = tile < tiles ? atomicAdd(cursors + tile, count)
                             : bucket_total + atomicAdd(&header->tail_cursor, count);
      }
      claim = __shfl_sync(0xffffffffu, claim, leader);
      pos[b] = valid ? static_cast<uint64_t>(claim) + static_cast<uint64_t>(__popc(peers & below)) : ~0ull;
    }
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      if (pos[b] >= static_cast<uint64_t>(n)) continue;
      if ((key[b] >> 32) < tiles) {
        p.keys_out[pos[b]] = (key[b] << 32) | static_cast<uint32_t>(value[b]);
      } else {
        p.keys_out[pos[b]] = ~0ull;
        p.values_out[pos[b]] = value[b];
      }
    }
  }
}

// One CTA per tile: order the bucket by (depth bits, Gaussian id).
//
// Buckets of at most kTileSortCap entries stay in shared memory: one split
// of the bucket's depth range into 2048 sub-ranges with shared-memory
// counters, a scatter by split, and every entry ranked within its split by
// its own thread (the work of a dense split is spread over the threads that
// hold its entries).  A bucket whose largest split exceeds kMaxRankSplit
// (many equal or nearly equal depths) is sorted by stable LSD passes over
// the depth bits instead, after which runs of equal depth bits are ordered
// by Gaussian id.
// Buckets above kTileSortCap are split the same way through global memory
// into runs of whole splits that fit in shared memory, and each run is then
// sorted like a small bucket (split again by its own depth range); only a
// single split above kTileSortCap takes chunked LSD passes through global
// memory.
namespace {

struct TileSortSmem {
  __align__(16) uint64_t items[kTileSortCap];
  __align__(16) union {
    RankSmem rank;
    uint32_t split[1 << kTileSortSplitBits];
  } u;
  __align__(16) uint32_t off[1 << kTileSortSplitBits];
  uint32_t base[kRadixBins];
  uint32_t minmax[4][kTsWarps];
  uint32_t scan[kTsWarps];
  uint32_t big[kTsWarps];
  uint32_t run_count;
  uint32_t queue_base;
};

// Orders one tile's bucket.  kLarge false: buckets of at most kTileSortCap
// entries (larger ones are left to the large pass); kLarge true: the larger
// buckets only.
template <bool kLarge>
__device__ __forceinline__ void sort_tile(const BucketParams& p, int64_t tile, TileSortSmem& sm) {
  constexpr int kSplitBits = kTileSortSplitBits;
  constexpr int kSplits = 1 << kSplitBits;
  constexpr int kSplitsPerThread = kSplits / kTileSortThreads;
  constexpr uint32_t kMaxRankSplit = 256;   // longest split whose entries are ranked
  static_assert(kSplitsPerThread == 8, "two uint4 loads of split counters per thread");
  uint64_t (&s_items)[kTileSortCap] = sm.items;
  auto& s_u = sm.u;
  uint32_t (&s_off)[kSplits] = sm.off;
  uint32_t (&s_base)[kRadixBins] = sm.base;
  uint32_t (&s_minmax)[4][kTsWarps] = sm.minmax;
  uint32_t (&s_scan)[kTsWarps] = sm.scan;
  uint32_t (&s_big)[kTsWarps] = sm.big;
  uint32_t& s_run_count = sm.run_count;

  const int64_t start = p.tile_starts[tile];
  const int64_t end = p.tile_ends[tile];
  if (start < 0 || end > p.capacity || end - start <= 0) return;
  const int n = static_cast<int>(end - start);
  if ((n > kTileSortCap) != kLarge) return;  // the other pass's bucket
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const uint64_t key_tile = static_cast<uint64_t>(tile) << 32;
  uint64_t* bucket = p.keys_out + start;

  if (n == 1) {
    if (tid == 0) {
      const uint64_t v = bucket[0];
      p.keys_out[start] = key_tile | (v >> 32);
      p.values_out[start] = static_cast<int32_t>(static_cast<uint32_t>(v));
    }
    return;
  }

  uint64_t it[kTileSortItems];
  uint32_t dr[kTileSortItems];

  // Order of two entries of this tile: depth bits, then Gaussian id (the
  // reference's tie-break; ids are unique within a camera, so the order is
  // total).  The id is read from the record only when the depths are equal.
  const Record* records = p.records;
  auto gaussian_id = [&](uint64_t e) -> uint32_t {
    return __float_as_uint(__ldg(&records[static_cast<uint32_t>(e)].b).w);
  };
  auto greater = [&](uint64_t a, uint64_t b) -> bool {
    const uint32_t da = static_cast<uint32_t>(a >> 32);
    const uint32_t db = static_cast<uint32_t>(b >> 32);
    if (da != db) return da > db;
    return gaussian_id(a) > gaussian_id(b);
  };

  // Stable LSD of count <= kTileSortCap entries read from src, leaving them
  // sorted in s_items.  by_gid false: passes over the depth bits only (equal
  // depths keep the order of src).  by_gid true: passes over the Gaussian id
  // (placed in the high word for the passes), then over the depth bits.
  // Items are held warp-blocked (element (w * K + k) * 32 + l) for the stable
  // ranking; s_u.rank must be free (not holding split counters).
  auto lsd_run = [&](const uint64_t* src, int count, auto by_gid_tag) {
    constexpr bool by_gid = decltype(by_gid_tag)::value;
    const int K = (count + kTileSortThreads - 1) / kTileSortThreads;
    for (int i = tid; i < kTsWarps * kRadixBins; i += kTileSortThreads) {
      (&s_u.rank.warp_hist[0][0])[i] = 0u;
    }
    uint32_t gl = 0xffffffffu, gh = 0u, dl = 0xffffffffu, dh = 0u;
#pragma unroll
    for (int k = 0; k < kTileSortItems; ++k) {
      if (k >= K) break;
      const int idx = (warp * K + k) * 32 + lane;
      if (idx < count) {
        const uint64_t v = src[idx];
        if constexpr (by_gid) {
          const uint32_t g = gaussian_id(v);
          it[k] = (static_cast<uint64_t>(g) << 32) | static_cast<uint32_t>(v);
          gl = min(gl, g);
          gh = max(gh, g);
        } else {
          it[k] = v;
        }
        dl = min(dl, static_cast<uint32_t>(v >> 32));
        dh = max(dh, static_cast<uint32_t>(v >> 32));
      }
    }
    block_minmax(gl, gh, dl, dh, s_minmax);
    __syncthreads();  // s_minmax is reused by the next run
    auto pass = [&](PassDigit dig) {
      rank_chunk(it, dr, K, count, dig, s_u.rank);
#pragma unroll
      for (int k = 0; k < kTileSortItems; ++k) {
        if (k >= K) break;
        const uint32_t d = dr[k] >> 16;
        if (d != kNoDigit) {
          s_items[s_u.rank.digit_start[d] + s_u.rank.warp_hist[warp][d] + (dr[k] & 0xffffu)] = it[k];
        }
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < kTileSortItems; ++k) {
        if (k >= K) break;
        const int idx = (warp * K + k) * 32 + lane;
        if (idx < count) it[k] = s_items[idx];
      }
#pragma unroll
      for (int w = 0; w < kTsWarps; ++w) s_u.rank.warp_hist[w][tid] = 0u;
      __syncthreads();
    };
    const int passes_d = (bit_length_u32(dh - dl) + kRadixBits - 1) / kRadixBits;
    if constexpr (by_gid) {
      const int passes_g = (bit_length_u32(gh - gl) + kRadixBits - 1) / kRadixBits;
      for (int q = 0; q < passes_g; ++q) pass(PassDigit{0, gl, q * kRadixBits});
#pragma unroll
      for (int k = 0; k < kTileSortItems; ++k) {
        if (k >= K) break;
        const int idx = (warp * K + k) * 32 + lane;
        if (idx < count) {
          const uint32_t r = static_cast<uint32_t>(it[k]);
          const uint32_t depth = __float_as_uint(__ldg(&records[r].b).z);
          it[k] = (static_cast<uint64_t>(depth) << 32) | r;
        }
      }
    }
    for (int q = 0; q < passes_d; ++q) pass(PassDigit{0, dl, q * kRadixBits});
#pragma unroll
    for (int k = 0; k < kTileSortItems; ++k) {
      if (k >= K) break;
      const int idx = (warp * K + k) * 32 + lane;
      if (idx < count) s_items[idx] = it[k];
    }
    __syncthreads();
  };

  // Stable LSD by the depth bits, then runs of equal depth bits ordered by
  // Gaussian id: each run is insertion-sorted by the thread that finds its
  // first entry; a run longer than kMaxTieRun sends the whole range through
  // the LSD passes again with the Gaussian id as the second key.
  auto lsd_sort = [&](const uint64_t* src, int count) {
    constexpr int kMaxTieRun = 32;
    if (tid == 0) s_run_count = 0u;  // read after the barriers inside lsd_run
    lsd_run(src, count, std::false_type{});
    auto depth_at = [&](int i) { return static_cast<uint32_t>(s_items[i] >> 32); };
    auto run_end = [&](int i) {
      // End of the run of equal depth bits that starts at i, or -1 when i
      // does not start a run of two or more.
      const uint32_t d = depth_at(i);
      if ((i > 0 && depth_at(i - 1) == d) || i + 1 >= count || depth_at(i + 1) != d) return -1;
      int e = i + 2;
      while (e < count && e - i <= kMaxTieRun && depth_at(e) == d) ++e;
      return e;
    };
    // Runs of two or more are listed as (start, end) pairs in the split
    // counters' storage, which is free once lsd_run returns.
    uint32_t* s_runs = s_u.split;
    constexpr int kMaxRuns = kSplits / 2;
    bool long_run = false;
    for (int i = tid; i < count; i += kTileSortThreads) {
      const int e = run_end(i);
      if (e < 0) continue;
      const uint32_t slot = e - i > kMaxTieRun ? kMaxRuns : atomicAdd(&s_run_count, 1u);
      if (slot < kMaxRuns) {
        s_runs[2 * slot] = i;
        s_runs[2 * slot + 1] = e;
      } else {
        long_run = true;
      }
    }
    if (__syncthreads_or(long_run)) {
      lsd_run(src, count, std::true_type{});
      return;
    }
    const int nruns = static_cast<int>(s_run_count);
    for (int r = tid; r < nruns; r += kTileSortThreads) {
      const int lo = static_cast<int>(s_runs[2 * r]);
      const int hi = static_cast<int>(s_runs[2 * r + 1]);
      for (int a = lo + 1; a < hi; ++a) {
        const uint64_t v = s_items[a];
        int b = a - 1;
        while (b >= lo && gaussian_id(s_items[b]) > gaussian_id(v)) {
          s_items[b + 1] = s_items[b];
          --b;
        }
        s_items[b + 1] = v;
      }
    }
    __syncthreads();
  };

  // Writes entry s_items[i] of a group of splits to the output at its sorted
  // place: its split occupies s_items[lo, hi) (splits in depth order), and
  // its rank is the number of the split's entries that order before it
  // (depth bits, then Gaussian id where depths are equal - read only then;
  // ids are unique within a camera, so ranks are too).  Every entry is
  // ranked by its own thread: the work of a split is spread over the
  // threads holding its entries instead of one thread per split.
  auto place = [&](int i, int lo, int hi, int64_t out_base) {
    const uint64_t v = s_items[i];
    const uint32_t d = static_cast<uint32_t>(v >> 32);
    // Entries of the split below d, and equal to d (the entry itself
    // included): the depth words alone, four per iteration.
    const uint32_t* words = reinterpret_cast<const uint32_t*>(s_items) + 1;
    int rank = 0, equal = 0;
    int f = lo;
    for (; f + 4 <= hi; f += 4) {
      const uint32_t d0 = words[2 * f], d1 = words[2 * f + 2], d2 = words[2 * f + 4], d3 = words[2 * f + 6];
      rank += (d0 < d) + (d1 < d) + (d2 < d) + (d3 < d);
      equal += (d0 == d) + (d1 == d) + (d2 == d) + (d3 == d);
    }
    for (; f < hi; ++f) {
      const uint32_t df = words[2 * f];
      rank += df < d;
      equal += df == d;
    }
    if (equal > 1) {
      const uint32_t g = gaussian_id(v);
      for (int f = lo; f < hi; ++f) {
        const uint64_t w = s_items[f];
        if (f != i && static_cast<uint32_t>(w >> 32) == d && gaussian_id(w) < g) ++rank;
      }
    }
    const int64_t out = out_base + lo + rank;
    p.keys_out[out] = key_tile | (v >> 32);
    p.values_out[out] = static_cast<int32_t>(static_cast<uint32_t>(v));
  };

  // Sorts count <= kTileSortCap entries read from src (a bucket, or a run of
  // whole splits of a long bucket) and writes them to the output from
  // out_base on: split them by the top kSplitBits bits of their own depth
  // range with shared-memory counters, scatter them into s_items by split,
  // then rank every entry within its split (place).  A split above
  // kMaxRankSplit entries (many equal or nearly equal depths) sends the
  // entries through stable LSD passes instead, after which runs of equal
  // depth bits are ordered by Gaussian id.  The split offsets live in the
  // counters' storage, so s_off (a long bucket's own splits) is left alone.
  auto sort_resident = [&](const uint64_t* src, int count, int64_t out_base) {
    uint32_t dmin = 0xffffffffu, dmax = 0u, rmin = 0xffffffffu, rmax = 0u;
    const int K = (count + kTileSortThreads - 1) / kTileSortThreads;
#pragma unroll
    for (int k = 0; k < kTileSortItems; ++k) {
      if (k >= K) break;
      const int i = k * kTileSortThreads + tid;
      if (i < count) {
        it[k] = src[i];
        const uint32_t dw = static_cast<uint32_t>(it[k] >> 32);
        const uint32_t rw = static_cast<uint32_t>(it[k]);
        dmin = min(dmin, dw);
        dmax = max(dmax, dw);
        rmin = min(rmin, rw);
        rmax = max(rmax, rw);
      }
    }
    for (int b = tid; b < kSplits; b += kTileSortThreads) s_u.split[b] = 0u;
    block_minmax(dmin, dmax, rmin, rmax, s_minmax);
    const int range_bits = bit_length_u32(dmax - dmin);
    const int shift = range_bits > kSplitBits ? range_bits - kSplitBits : 0;
#pragma unroll
    for (int k = 0; k < kTileSortItems; ++k) {
      if (k >= K) break;
      if (k * kTileSortThreads + tid < count) {
        const uint32_t sp = (static_cast<uint32_t>(it[k] >> 32) - dmin) >> shift;
        dr[k] = (sp << 16) | atomicAdd(&s_u.split[sp], 1u);
      }
    }
    __syncthreads();
    // Exclusive offsets of the splits; thread t owns splits [8t, 8t + 8).
    // Also the largest split.
    uint32_t c[kSplitsPerThread];
    {
      const uint4 lo = reinterpret_cast<const uint4*>(s_u.split)[tid * 2];
      const uint4 hi = reinterpret_cast<const uint4*>(s_u.split)[tid * 2 + 1];
      c[0] = lo.x; c[1] = lo.y; c[2] = lo.z; c[3] = lo.w;
      c[4] = hi.x; c[5] = hi.y; c[6] = hi.z; c[7] = hi.w;
    }
    uint32_t sum = 0, big = 0;
#pragma unroll
    for (int j = 0; j < kSplitsPerThread; ++j) {
      sum += c[j];
      big = max(big, c[j]);
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    big = __reduce_max_sync(0xffffffffu, big);
    if (lane == 31) s_scan[warp] = incl;
    if (lane == 0) s_big[warp] = big;
    __syncthreads();  // every thread has read its counters
    uint32_t prefix = incl - sum;
#pragma unroll
    for (int w = 0; w < kTsWarps; ++w) {
      prefix += w < warp ? s_scan[w] : 0u;
      big = max(big, s_big[w]);
    }
    if (big <= kMaxRankSplit) {
      uint32_t off[kSplitsPerThread];
#pragma unroll
      for (int j = 0; j < kSplitsPerThread; ++j) {
        off[j] = prefix;
        prefix += c[j];
      }
      uint32_t* split_off = s_u.split;
      reinterpret_cast<uint4*>(split_off)[tid * 2] = make_uint4(off[0], off[1], off[2], off[3]);
      reinterpret_cast<uint4*>(split_off)[tid * 2 + 1] = make_uint4(off[4], off[5], off[6], off[7]);
      __syncthreads();
#pragma unroll
      for (int k = 0; k < kTileSortItems; ++k) {
        if (k >= K) break;
        if (k * kTileSortThreads + tid < count) {
          s_items[split_off[dr[k] >> 16] + (dr[k] & 0xffffu)] = it[k];
        }
      }
      __syncthreads();
      // Every entry goes straight to its sorted place (src was read into
      // registers before the barriers above, so it may be the output).
      for (int i = tid; i < count; i += kTileSortThreads) {
        const uint32_t sp = (static_cast<uint32_t>(s_items[i] >> 32) - dmin) >> shift;
        const int lo = static_cast<int>(split_off[sp]);
        const int hi = sp + 1 < static_cast<uint32_t>(kSplits) ? static_cast<int>(split_off[sp + 1]) : count;
        place(i, lo, hi, out_base);
      }
      __syncthreads();  // s_items and the offsets are reused by the caller
      return;
    }
    // ------------------------------------------- stable LSD in shared memory
    __syncthreads();  // the split counters share storage with the rank state
    lsd_sort(src, count);
    for (int i = tid; i < count; i += kTileSortThreads) {
      const uint64_t v = s_items[i];
      p.keys_out[out_base + i] = key_tile | (v >> 32);
      p.values_out[out_base + i] = static_cast<int32_t>(static_cast<uint32_t>(v));
    }
    __syncthreads();
  };

  if (n <= kTileSortCap) {
    sort_resident(bucket, n, start);
    return;
  }

  // ------------------------------------------------------------ large buckets
  // Split by the top kSplitBits bits of the tile's depth range through global
  // memory (count, then scatter into the same range of the temp buffer with
  // shared-memory cursors), then sort runs of whole splits in shared memory,
  // each like a small bucket.
  {
    uint32_t dlo = 0xffffffffu, dhi = 0u, rlo = 0xffffffffu, rhi = 0u;
    // The bucket passes below keep kLoads independent loads in flight per
    // thread (the large path is latency-bound on its global reads).
    constexpr int kLoads = 8;
    constexpr int kStep = kLoads * kTileSortThreads;
    for (int b = tid; b < kSplits; b += kTileSortThreads) s_u.split[b] = 0u;
    for (int i0 = tid; i0 < n; i0 += kStep) {
      uint32_t dw[kLoads];
#pragma unroll
      for (int u = 0; u < kLoads; ++u) {
        const int i = i0 + u * kTileSortThreads;
        dw[u] = i < n ? static_cast<uint32_t>(bucket[i] >> 32) : dlo;
      }
#pragma unroll
      for (int u = 0; u < kLoads; ++u) {
        if (i0 + u * kTileSortThreads < n) {
          dlo = min(dlo, dw[u]);
          dhi = max(dhi, dw[u]);
        }
      }
    }
    block_minmax(dlo, dhi, rlo, rhi, s_minmax);
    const int range_bits = bit_length_u32(dhi - dlo);
    const int shift = range_bits > kSplitBits ? range_bits - kSplitBits : 0;
    for (int i0 = tid; i0 < n; i0 += kStep) {
      uint32_t dw[kLoads];
#pragma unroll
      for (int u = 0; u < kLoads; ++u) {
        const int i = i0 + u * kTileSortThreads;
        dw[u] = i < n ? static_cast<uint32_t>(bucket[i] >> 32) : 0u;
      }
#pragma unroll
      for (int u = 0; u < kLoads; ++u) {
        if (i0 + u * kTileSortThreads < n) atomicAdd(&s_u.split[(dw[u] - dlo) >> shift], 1u);
      }
    }
    __syncthreads();
    uint32_t c[kSplitsPerThread];
    {
      const uint4 lo4 = reinterpret_cast<const uint4*>(s_u.split)[tid * 2];
      const uint4 hi4 = reinterpret_cast<const uint4*>(s_u.split)[tid * 2 + 1];
      c[0] = lo4.x; c[1] = lo4.y; c[2] = lo4.z; c[3] = lo4.w;
      c[4] = hi4.x; c[5] = hi4.y; c[6] = hi4.z; c[7] = hi4.w;
    }
    uint32_t sum = 0, big = 0;
#pragma unroll
    for (int j = 0; j < kSplitsPerThread; ++j) {
      sum += c[j];
      big = max(big, c[j]);
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    big = __reduce_max_sync(0xffffffffu, big);
    if (lane == 31) s_scan[warp] = incl;
    if (lane == 0) s_big[warp] = big;
    __syncthreads();
    uint32_t prefix = incl - sum;
#pragma unroll
    for (int w = 0; w < kTsWarps; ++w) {
      prefix += w < warp ? s_scan[w] : 0u;
      big = max(big, s_big[w]);
    }
    if (big <= static_cast<uint32_t>(kTileSortCap)) {
      uint32_t off[kSplitsPerThread];
#pragma unroll
      for (int j = 0; j < kSplitsPerThread; ++j) {
        off[j] = prefix;
        prefix += c[j];
      }
      __syncthreads();  // every thread has read its counters
      reinterpret_cast<uint4*>(s_off)[tid * 2] = make_uint4(off[0], off[1], off[2], off[3]);
      reinterpret_cast<uint4*>(s_off)[tid * 2 + 1] = make_uint4(off[4], off[5], off[6], off[7]);
      reinterpret_cast<uint4*>(s_u.split)[tid * 2] = make_uint4(off[0], off[1], off[2], off[3]);
      reinterpret_cast<uint4*>(s_u.split)[tid * 2 + 1] = make_uint4(off[4], off[5], off[6], off[7]);
      __syncthreads();
      uint64_t* split_buf = p.temp + start;
      for (int i0 = tid; i0 < n; i0 += kStep) {
        uint64_t v[kLoads];
#pragma unroll
        for (int u = 0; u < kLoads; ++u) {
          const int i = i0 + u * kTileSortThreads;
          v[u] = i < n ? bucket[i] : 0ull;
        }
#pragma unroll
        for (int u = 0; u < kLoads; ++u) {
          if (i0 + u * kTileSortThreads < n) {
            split_buf[atomicAdd(&s_u.split[(static_cast<uint32_t>(v[u] >> 32) - dlo) >> shift], 1u)] = v[u];
          }
        }
      }
      __syncthreads();
      // Runs of whole splits that fit in shared memory, in split order.
      int first = 0;
      while (first < kSplits) {
        const int base = static_cast<int>(s_off[first]);
        int lo = first + 1, hi = kSplits;  // the run is [first, last): largest last in [lo, hi]
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          const int end_mid = mid < kSplits ? static_cast<int>(s_off[mid]) : n;
          if (end_mid - base <= kTileSortCap) lo = mid; else hi = mid - 1;
        }
        const int last = lo;
        const int count = (last < kSplits ? static_cast<int>(s_off[last]) : n) - base;
        sort_resident(split_buf + base, count, start + base);
        first = last;
      }
      return;
    }
    __syncthreads();  // the split counters share storage with the rank state below
  }

  // A single split above kTileSortCap (many equal or nearly equal depths):
  // stable chunked LSD through global memory, ping-ponging between the bucket
  // and the same range of the temp buffer: passes over the Gaussian id
  // (placed in the high word), then over the depth bits.
  constexpr int kChunkItems = 8;
  constexpr int kChunk = kTileSortThreads * kChunkItems;
  for (int i = tid; i < kTsWarps * kRadixBins; i += kTileSortThreads) {
    (&s_u.rank.warp_hist[0][0])[i] = 0u;
  }
  uint32_t gmin = 0xffffffffu, gmax = 0u, dmin = 0xffffffffu, dmax = 0u;
  for (int i = tid; i < n; i += kTileSortThreads) {
    const uint64_t v = bucket[i];
    const uint32_t dw = static_cast<uint32_t>(v >> 32);
    const uint32_t g = gaussian_id(v);
    dmin = min(dmin, dw);
    dmax = max(dmax, dw);
    gmin = min(gmin, g);
    gmax = max(gmax, g);
    bucket[i] = (static_cast<uint64_t>(g) << 32) | static_cast<uint32_t>(v);
  }
  block_minmax(gmin, gmax, dmin, dmax, s_minmax);
  const int passes_g = (bit_length_u32(gmax - gmin) + kRadixBits - 1) / kRadixBits;
  const int passes_d = (bit_length_u32(dmax - dmin) + kRadixBits - 1) / kRadixBits;
  uint64_t* src = bucket;
  uint64_t* dst = p.temp + start;
  for (int q = 0; q < passes_g + passes_d; ++q) {
    if (q == passes_g) {
      // Switch the high word from the Gaussian id to the depth bits.
      __syncthreads();
      for (int i = tid; i < n; i += kTileSortThreads) {
        const uint32_t r = static_cast<uint32_t>(src[i]);
        src[i] = (static_cast<uint64_t>(__float_as_uint(__ldg(&records[r].b).z)) << 32) | r;
      }
    }
    const PassDigit dig = q < passes_g ? PassDigit{0, gmin, q * kRadixBits}
                                       : PassDigit{0, dmin, (q - passes_g) * kRadixBits};
    s_base[tid] = 0u;
    __syncthreads();
    for (int i = tid; i < n; i += kTileSortThreads) atomicAdd(&s_base[dig(src[i])], 1u);
    __syncthreads();
    {
      const uint32_t v = s_base[tid];
      uint32_t incl = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (lane == 31) s_scan[warp] = incl;
      __syncthreads();
      uint32_t wp = 0;
#pragma unroll
      for (int w = 0; w < kTsWarps; ++w) wp += w < warp ? s_scan[w] : 0u;
      s_base[tid] = wp + incl - v;
      __syncthreads();
    }
    for (int cb = 0; cb < n; cb += kChunk) {
      const int m = n - cb < kChunk ? n - cb : kChunk;
      uint64_t ci[kChunkItems];
      uint32_t cr[kChunkItems];
#pragma unroll
      for (int k = 0; k < kChunkItems; ++k) {
        const int idx = (warp * kChunkItems + k) * 32 + lane;
        ci[k] = idx < m ? src[cb + idx] : 0ull;
      }
      const uint32_t total = rank_chunk(ci, cr, kChunkItems, m, dig, s_u.rank);
#pragma unroll
      for (int k = 0; k < kChunkItems; ++k) {
        const uint32_t d = cr[k] >> 16;
        if (d != kNoDigit) dst[s_base[d] + s_u.rank.warp_hist[warp][d] + (cr[k] & 0xffffu)] = ci[k];
      }
      __syncthreads();
      s_base[tid] += total;
#pragma unroll
      for (int w = 0; w < kTsWarps; ++w) s_u.rank.warp_hist[w][tid] = 0u;
      __syncthreads();
    }
    uint64_t* t = src;
    src = dst;
    dst = t;
  }
  if (passes_d == 0) {
    // No depth pass ran: the high word still holds the Gaussian id.
    __syncthreads();
    for (int i = tid; i < n; i += kTileSortThreads) {
      const uint32_t r = static_cast<uint32_t>(src[i]);
      src[i] = (static_cast<uint64_t>(__float_as_uint(__ldg(&records[r].b).z)) << 32) | r;
    }
  }
  __syncthreads();
  for (int i = tid; i < n; i += kTileSortThreads) {
    const uint64_t v = src[i];
    p.keys_out[start + i] = key_tile | (v >> 32);
    p.values_out[start + i] = static_cast<int32_t>(static_cast<uint32_t>(v));
  }
}

}  // namespace

// Lists the tiles whose buckets exceed kTileSortCap (in any order) in
// p.large_list, their number in ScratchHeader::large_tile_count.  The list
// lives in the emitted record-index buffer, which the scatter has consumed.
__global__ void __launch_bounds__(256) large_tile_list_kernel(BucketParams p) {
  ScratchHeader* header = reinterpret_cast<ScratchHeader*>(p.scratch + p.layout.header);
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  bool large = false;
  if (t < p.tile_count) {
    const int64_t s = p.tile_starts[t];
    const int64_t e = p.tile_ends[t];
    large = s >= 0 && e <= p.capacity && e - s > kTileSortCap;
  }
  const uint32_t mask = __ballot_sync(0xffffffffu, large);
  uint32_t base = 0;
  if ((threadIdx.x & 31) == 0 && mask) base = atomicAdd(&header->large_tile_count, __popc(mask));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (large) p.large_list[base + __popc(mask & lanemask_lt())] = static_cast<int32_t>(t);
}

// One launch for both kinds of bucket.  The first p.large_workers CTAs are
// persistent workers for the buckets above kTileSortCap: each takes one
// listed tile at a time from ScratchHeader::large_tile_queue and sorts it.
// They are dispatched first, so the long buckets start at once and the rest
// of the grid (CTA p.large_workers + t sorts tile t when its bucket holds at
// most kTileSortCap entries) fills in behind them.  A ragged frame of
// cameras inside dense scenes keeps most of its intersections in a few long
// buckets of neighbouring tiles; with one CTA per tile in tile order they
// ran as a tail at the end of the grid.
// Four resident CTAs per SM: a 64-register cap (five CTAs, the most the
// shared-memory footprint allows, cap registers at 48 and spilled about
// 2 KB per thread to local memory; four measured 5.26 -> 4.56 ms on the
// 1,024-camera ragged frame, three 5.11 ms).
__global__ void __launch_bounds__(kTileSortThreads, 4) tile_sort_kernel(BucketParams p) {
  __shared__ TileSortSmem sm;
  const int64_t workers = p.large_workers;
  if (static_cast<int64_t>(blockIdx.x) >= workers) {
    sort_tile<false>(p, static_cast<int64_t>(blockIdx.x) - workers, sm);
    return;
  }
  ScratchHeader* header = reinterpret_cast<ScratchHeader*>(p.scratch + p.layout.header);
  const uint32_t listed = header->large_tile_count;
  while (true) {
    if (threadIdx.x == 0) sm.queue_base = atomicAdd(&header->large_tile_queue, 1u);
    __syncthreads();
    const uint32_t index = sm.queue_base;
    __syncthreads();  // thread 0 rewrites the ticket only after every thread read it
    if (index >= listed) break;
    sort_tile<true>(p, p.large_list[index], sm);
    __syncthreads();  // shared staging is reused by the next bucket
  }
}

}  // namespace vgr
