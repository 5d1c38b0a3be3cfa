// Stream compaction / re-indexing of the working LP and the general transpose.
//
// Reference: apply_plan_to_working_lp / compact_csr_by_masks_gpu
// (cpp/src/presolve/gpu_presolve.cu:95-436,715-770,1793-1930) and
// transpose_csr64 (cpp/src/presolve/transpose64.cu:54-117).
//
// Materialisation compacts A and A^T with the same row/column maps.  A^T is
// kept row-sorted, and the old->new maps are monotone, so compacting A^T gives
// exactly cusparseCsr2cscEx2(compact(A)): the per-apply transpose becomes a
// second streaming pass.  The general transpose below is only needed for an
// input A^T that is not row-sorted and for matrices rebuilt by a rule.
#include "engine.cuh"
#include "sort.hpp"

#include <algorithm>
#include <utility>

namespace gpp {

namespace {

__global__ void mask_to_int(const uint8_t* __restrict__ keep, int32_t n, int32_t* __restrict__ out) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = keep[i] != 0;
}
__global__ void prefix_to_map(const uint8_t* __restrict__ keep, const int32_t* __restrict__ prefix, int32_t n,
                              int32_t* __restrict__ old_to_new) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    old_to_new[i] = keep[i] ? prefix[i] : -1;
}

// ---- entry-tiled compaction -------------------------------------------------
//
// The stored entries are cut into tiles of kCompactTile consecutive positions,
// one block per tile and kCompactPer consecutive positions per thread, so the
// index and value streams are read with 128-bit loads whatever the row
// lengths.  A tile learns the row of each of its entries without a search:
// the rows whose pointer falls inside the tile mark their start positions in
// shared memory, and a block scan of the marks counts the row starts at or
// before every position.  The copy is a stream compaction in stored order, so
// a kept entry's output position is the number of kept entries before it.
// One pass does it: tiles are handed out in order by a ticket counter, each
// tile publishes its kept count as soon as it knows it, and looks back over
// its predecessors' published counts (a decoupled look-back) for its output
// offset; its block scan then places each kept entry and each kept row's new
// pointer.
constexpr int kCompactPer = 8;
constexpr int kCompactTile = kThreads * kCompactPer;

// first_row[t]: the first row whose pointer is at or past t * kCompactTile
// (rows when there is none).  Row r takes the tiles whose start lies in
// (ptr[r - 1], ptr[r]]; the virtual row `rows` takes the tiles past the last
// row's pointer.
__global__ void compact_tile_rows(int rows, const offset_t* __restrict__ ptr, int tiles,
                                  int32_t* __restrict__ first_row) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r <= rows; r += gridDim.x * blockDim.x) {
    const int64_t lo = r == 0 ? 0 : int64_t(ptr[r - 1]) / kCompactTile + 1;
    int64_t hi = r == rows ? int64_t(tiles) - 1 : int64_t(ptr[r]) / kCompactTile;
    if (hi > tiles - 1) hi = tiles - 1;
    for (int64_t t = lo; t <= hi; ++t) first_row[t] = r;
  }
}

// Exclusive scan of one value per thread over the block; the block total goes
// to *total.  `warp_sums` holds kThreads / 32 ints of shared memory.
__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_sums, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += y;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  int before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < kThreads / 32; ++w) {
    const int sw = warp_sums[w];
    before += w < warp ? sw : 0;
    all += sw;
  }
  __syncthreads();
  *total = all;
  return before + incl - v;
}

template <bool kVec>
__device__ __forceinline__ void load_tile_cols(const int32_t* __restrict__ p, int avail, int (&col)[kCompactPer]) {
  if (kVec && avail >= kCompactPer) {
    const int4 a = __ldcs(reinterpret_cast<const int4*>(p));
    const int4 b = __ldcs(reinterpret_cast<const int4*>(p) + 1);
    col[0] = a.x; col[1] = a.y; col[2] = a.z; col[3] = a.w;
    col[4] = b.x; col[5] = b.y; col[6] = b.z; col[7] = b.w;
  } else {
#pragma unroll
    for (int k = 0; k < kCompactPer; ++k) col[k] = k < avail ? __ldcs(p + k) : -1;
  }
}
template <bool kVec>
__device__ __forceinline__ void load_tile_vals(const double* __restrict__ p, int avail, double (&v)[kCompactPer]) {
  if (kVec && avail >= kCompactPer) {
#pragma unroll
    for (int k = 0; k < kCompactPer / 2; ++k) {
      const double2 d = __ldcs(reinterpret_cast<const double2*>(p) + k);
      v[2 * k] = d.x;
      v[2 * k + 1] = d.y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < kCompactPer; ++k) v[k] = k < avail ? __ldcs(p + k) : 0.0;
  }
}

// Kept-entry mask of this thread's kCompactPer positions: the entry exists,
// its row is kept and its (remapped) inner index is kept.  `col` holds the
// inner indices already mapped (-1 for a dropped or missing entry).
__device__ __forceinline__ unsigned tile_kept_mask(int r0, int64_t base, int len, const offset_t* __restrict__ ptr,
                                                   int r1, const int32_t* __restrict__ outer_map,
                                                   const int (&col)[kCompactPer], int* marker, int* warp_sums) {
  const int p0 = int(threadIdx.x) * kCompactPer;
  // Row starts inside the tile.
#pragma unroll
  for (int k = 0; k < kCompactPer; ++k) marker[p0 + k] = 0;
  __syncthreads();
  for (int r = r0 + int(threadIdx.x); r < r1; r += kThreads) {
    const int64_t pos = int64_t(ptr[r]) - base;
    if (pos < len) atomicAdd(marker + pos, 1);
  }
  __syncthreads();
  int mk[kCompactPer], local = 0;
#pragma unroll
  for (int k = 0; k < kCompactPer; ++k) {
    mk[k] = marker[p0 + k];
    local += mk[k];
  }
  int total;
  int row = r0 - 1 + block_exclusive_scan(local, warp_sums, &total);
  unsigned mask = 0;
  int cached_row = -1, cached_keep = -1;
#pragma unroll
  for (int k = 0; k < kCompactPer; ++k) {
    row += mk[k];
    if (p0 + k < len && col[k] >= 0) {
      if (row != cached_row) {
        cached_row = row;
        cached_keep = outer_map[row];
      }
      if (cached_keep >= 0) mask |= 1u << k;
    }
  }
  return mask;
}

// Tile status words: the top two bits say what the low 62 hold (an aggregate:
// the tile's own kept count; an inclusive count: the kept entries of every
// tile up to and including it).  Zero means nothing published yet.
constexpr unsigned long long kTileAggregate = 1ull << 62, kTileInclusive = 2ull << 62;
constexpr unsigned long long kTileValue = (1ull << 62) - 1;
// Polls of one predecessor before a look-back gives up (well over a second;
// a predecessor that holds a ticket is running and publishes within
// microseconds).  Giving up sets the error word, which the host checks.
constexpr int kLookbackPolls = 1 << 22;

__device__ __forceinline__ unsigned long long ld_tile_status(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_tile_status(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Kept entries before tile t, by warp 0: 32 predecessors per round, summing
// aggregates back to the nearest inclusive count (before tile 0: zero).
__device__ __forceinline__ int64_t tile_lookback(const unsigned long long* status, int t, int32_t* err) {
  const int lane = threadIdx.x & 31;
  int64_t before = 0;
  for (int end = t - 1;; end -= 32) {
    const int j = end - lane;
    unsigned long long st = kTileInclusive;
    if (j >= 0) {
      st = ld_tile_status(status + j);
      for (int polls = 1; (st >> 62) == 0; ++polls) {
        if (polls == kLookbackPolls) {
          atomicExch(err, 1);
          st = kTileInclusive;
          break;
        }
        __nanosleep(64);
        st = ld_tile_status(status + j);
      }
    }
    const unsigned incl = __ballot_sync(0xffffffffu, (st >> 62) == 2);
    const int first = incl ? __ffs(incl) - 1 : 32;
    unsigned long long v = lane <= first ? (st & kTileValue) : 0ull;
#pragma unroll
    for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    before += int64_t(v);
    if (incl) return before;
  }
}

// One pass: result[0] receives the kept total, result[1] is set if a
// look-back gave up.  `status` holds tiles words and then the ticket counter,
// all zero at launch.
template <bool kVec>
__global__ void __launch_bounds__(kThreads)
compact_tiles(offset_t nnz, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
              const double* __restrict__ val, const int32_t* __restrict__ outer_map,
              const int32_t* __restrict__ inner_map, const int32_t* __restrict__ first_row, int rows, int tiles,
              unsigned long long* status, int32_t outer_new, offset_t* __restrict__ out_ptr,
              int32_t* __restrict__ out_idx, double* __restrict__ out_val, int32_t* result) {
  // `marker` is free once the rows are known and then stages the kept
  // indices; `stage_val` the kept values.  The stores go out coalesced.
  __shared__ __align__(16) int marker[kCompactTile];
  __shared__ __align__(16) double stage_val[kCompactTile];
  __shared__ int warp_sums[kThreads / 32];
  __shared__ int thread_before[kThreads];
  __shared__ unsigned thread_mask[kThreads];
  __shared__ int ticket;
  __shared__ long long tile_before;
  const int p0 = int(threadIdx.x) * kCompactPer;
  for (;;) {
    if (threadIdx.x == 0) ticket = int(atomicAdd(status + tiles, 1ull));
    __syncthreads();
    const int t = ticket;
    if (t >= tiles) return;   // block-uniform
    const int64_t base = int64_t(t) * kCompactTile;
    const int len = int(min(int64_t(kCompactTile), int64_t(nnz) - base));
    int col[kCompactPer];
    double v[kCompactPer];
    load_tile_cols<kVec>(idx + base + p0, len - p0, col);
    load_tile_vals<kVec>(val + base + p0, len - p0, v);
    const int r0 = first_row[t], r1 = t + 1 < tiles ? first_row[t + 1] : rows;
#pragma unroll
    for (int k = 0; k < kCompactPer; ++k) col[k] = col[k] >= 0 ? inner_map[col[k]] : -1;
    const unsigned mask = tile_kept_mask(r0, base, len, ptr, r1, outer_map, col, marker, warp_sums);
    int total;
    const int before = block_exclusive_scan(__popc(mask), warp_sums, &total);
    if (threadIdx.x < 32) {
      if (threadIdx.x == 0)
        st_tile_status(status + t, (t == 0 ? kTileInclusive : kTileAggregate) | (unsigned long long)total);
      const int64_t ahead = t == 0 ? 0 : tile_lookback(status, t, result + 1);
      if (threadIdx.x == 0) {
        if (t > 0) st_tile_status(status + t, kTileInclusive | (unsigned long long)(ahead + total));
        tile_before = ahead;
      }
    }
    int o = before;
#pragma unroll
    for (int k = 0; k < kCompactPer; ++k)
      if (mask >> k & 1u) {
        marker[o] = col[k];
        stage_val[o] = v[k];
        ++o;
      }
    thread_before[threadIdx.x] = before;
    thread_mask[threadIdx.x] = mask;
    __syncthreads();
    const int64_t tile_out = tile_before;
    for (int q = int(threadIdx.x); q < total; q += kThreads) {
      out_idx[tile_out + q] = marker[q];
      out_val[tile_out + q] = stage_val[q];
    }
    // New row pointers of the kept rows that start in this tile: the kept
    // entries before the row's first position.
    for (int r = r0 + int(threadIdx.x); r < r1; r += kThreads) {
      const int nr = outer_map[r];
      if (nr < 0) continue;
      const int64_t pos = int64_t(ptr[r]) - base;
      int kept_before = total;
      if (pos < len) {
        const int q = int(pos) / kCompactPer, j = int(pos) % kCompactPer;
        kept_before = thread_before[q] + __popc(thread_mask[q] & ((1u << j) - 1u));
      }
      out_ptr[nr] = offset_t(tile_out + kept_before);
    }
    if (t == tiles - 1 && threadIdx.x == 0) {
      out_ptr[outer_new] = offset_t(tile_out + total);
      result[0] = int32_t(tile_out + total);
    }
    __syncthreads();   // the staging buffers and the ticket are reused by the next tile
  }
}

__global__ void histogram(const int32_t* __restrict__ idx, offset_t nnz, int32_t* __restrict__ counts) {
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz; p += int64_t(gridDim.x) * blockDim.x)
    atomicAdd(counts + idx[p], 1);
}
// Longest column (the histogram's largest count), one atomic per warp.
__global__ void longest_count(const int32_t* __restrict__ counts, int n, int32_t* __restrict__ out) {
  int32_t best = 0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) best = max(best, counts[j]);
  best = __reduce_max_sync(0xffffffffu, best);
  if ((threadIdx.x & 31) == 0 && best > 0) atomicMax(out, best);
}
// Short-column transpose: each stored position goes to a slot of its column
// through an atomic cursor (slot order within a column is arbitrary), then
// every column's positions are put back in ascending order, which is the
// stored (row-major) order: the same result as the stable sort.
constexpr int kShortColumn = 64;
__global__ void place_positions(offset_t nnz, const int32_t* __restrict__ idx, int32_t* __restrict__ cursor,
                                int32_t* __restrict__ pos) {
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz; p += int64_t(gridDim.x) * blockDim.x)
    pos[atomicAdd(cursor + idx[p], 1)] = int32_t(p);
}
__global__ void order_columns(int n, const offset_t* __restrict__ ptr, int32_t* __restrict__ pos) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const offset_t first = ptr[j];
    const int len = int(ptr[j + 1] - first);
    if (len < 2) continue;
    int32_t a[kShortColumn];
    for (int k = 0; k < len; ++k) a[k] = pos[first + k];
    for (int k = 1; k < len; ++k) {   // insertion sort: columns hold at most kShortColumn entries
      const int32_t v = a[k];
      int q = k - 1;
      while (q >= 0 && a[q] > v) { a[q + 1] = a[q]; --q; }
      a[q + 1] = v;
    }
    for (int k = 0; k < len; ++k) pos[first + k] = a[k];
  }
}
// Column keys and entry positions of M, in stored (row-major) order.
__global__ void transpose_keys(offset_t nnz, const int32_t* __restrict__ idx, uint64_t* __restrict__ keys,
                               int32_t* __restrict__ pos) {
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz; p += int64_t(gridDim.x) * blockDim.x) {
    keys[p] = uint64_t(uint32_t(idx[p]));
    pos[p] = int32_t(p);
  }
}
// Row of every stored entry: one warp per row writes its run.
__global__ void row_of_entry(int rows, const offset_t* __restrict__ ptr, int32_t* __restrict__ row) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += warps)
    for (offset_t p = ptr[r] + lane; p < ptr[r + 1]; p += 32) row[p] = r;
}
// Entries in (column, row) order: gather their rows and values.
__global__ void transpose_gather(offset_t nnz, const int32_t* __restrict__ pos, const int32_t* __restrict__ row,
                                 const double* __restrict__ val, int32_t* __restrict__ out_idx,
                                 double* __restrict__ out_val) {
  for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < nnz; q += int64_t(gridDim.x) * blockDim.x) {
    const int32_t p = pos[q];
    out_idx[q] = row[p];
    out_val[q] = val[p];
  }
}

// Four rows per warp, eight lanes per row, each lane comparing the pairs
// (p - 1, p) of its stride.
__global__ void check_sorted(int rows, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                             int32_t* bad) {
  const int g = threadIdx.x & 7;
  const int groups = gridDim.x * (blockDim.x >> 3);
  for (int r = blockIdx.x * (blockDim.x >> 3) + (threadIdx.x >> 3); r < rows; r += groups)
    for (offset_t p = ptr[r] + 1 + g; p < ptr[r + 1]; p += 8)
      if (idx[p - 1] >= idx[p]) { atomicExch(bad, 1); break; }
}

// Structure of an uploaded CSR: pointers start at 0, end at nnz and never
// decrease; every inner index lies in [0, cols).  Any violation sets *bad.
__global__ void check_csr_structure(int rows, int cols, offset_t nnz, const offset_t* __restrict__ ptr,
                                    const int32_t* __restrict__ idx, int32_t* bad) {
  const int64_t top = int64_t(rows) + 1 > int64_t(nnz) ? int64_t(rows) + 1 : int64_t(nnz);
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < top; i += int64_t(gridDim.x) * blockDim.x) {
    bool fail = false;
    if (i <= rows) {
      const offset_t p = ptr[i];
      if (i == 0 ? p != 0 : p < ptr[i - 1]) fail = true;
      if (i == rows && p != nnz) fail = true;
    }
    if (i < nnz) {
      const int32_t c = idx[i];
      if (c < 0 || c >= cols) fail = true;
    }
    if (fail) atomicExch(bad, 1);
  }
}

__global__ void gather_kernel(double* __restrict__ dst, const double* __restrict__ src,
                              const int32_t* __restrict__ map, int32_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const int k = map[i];
    if (k >= 0) dst[k] = src[i];
  }
}
__global__ void compose_kernel(int32_t* __restrict__ next, const int32_t* __restrict__ prev,
                               const int32_t* __restrict__ map, int32_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const int k = map[i];
    if (k >= 0) next[k] = prev[i];
  }
}

// Old -> new maps of the row and the column masks together, straight from
// the byte masks: one launch counts the kept items of every tile of
// kMapTile items (row tiles first, then column tiles), a second gives each
// kept item its rank (earlier tiles' counts plus a block scan) and writes -1
// for a dropped one; the last tile of each mask writes its total.
constexpr int kMapTile = 8 * kThreads;

__device__ __forceinline__ int block_sum_i32(int v, int* sh) {
  for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  int t = 0;
  for (int w = 0; w < kThreads / 32; ++w) t += sh[w];
  __syncthreads();
  return t;
}

struct MaskPair {
  const uint8_t* keep[2];
  int32_t n[2];
  int32_t tiles0;          // tiles of the first mask; the second's follow
  int32_t* map[2];
};

__global__ void __launch_bounds__(kThreads) map_tile_counts(MaskPair mp, int32_t* __restrict__ tile_counts) {
  __shared__ int sh[kThreads / 32];
  const int side = int(blockIdx.x) < mp.tiles0 ? 0 : 1;
  const int tile = side ? int(blockIdx.x) - mp.tiles0 : int(blockIdx.x);
  const int64_t base = int64_t(tile) * kMapTile + int64_t(threadIdx.x) * 8;
  int c = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) c += base + k < mp.n[side] && mp.keep[side][base + k] != 0;
  c = block_sum_i32(c, sh);
  if (threadIdx.x == 0) tile_counts[blockIdx.x] = c;
}

__global__ void __launch_bounds__(kThreads) map_tile_ranks(MaskPair mp, const int32_t* __restrict__ tile_counts,
                                                           int32_t* __restrict__ totals) {
  __shared__ int sh[kThreads / 32];
  __shared__ int warp_incl[kThreads / 32];
  const int side = int(blockIdx.x) < mp.tiles0 ? 0 : 1;
  const int first_tile = side ? mp.tiles0 : 0;
  const int tile = int(blockIdx.x) - first_tile;
  int offset = 0;
  for (int k = first_tile + int(threadIdx.x); k < int(blockIdx.x); k += kThreads) offset += tile_counts[k];
  offset = block_sum_i32(offset, sh);
  const int64_t base = int64_t(tile) * kMapTile + int64_t(threadIdx.x) * 8;
  const uint8_t* keep = mp.keep[side];
  const int32_t n = mp.n[side];
  uint8_t kept[8];
  int local = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    kept[k] = base + k < n && keep[base + k] != 0;
    local += kept[k];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = local;
  for (int off = 1; off < 32; off <<= 1) {
    const int peer = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += peer;
  }
  if (lane == 31) warp_incl[warp] = incl;
  __syncthreads();
  int before = 0;
  for (int w = 0; w < warp; ++w) before += warp_incl[w];
  int run = offset + before + incl - local;
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if (base + k < n) {
      mp.map[side][base + k] = kept[k] ? run : -1;
      run += kept[k];
    }
  const int tiles_side = side ? int(gridDim.x) - mp.tiles0 : mp.tiles0;
  if (tile == tiles_side - 1 && threadIdx.x == kThreads - 1) totals[side] = run;
}

}  // namespace

int32_t build_old_to_new(const uint8_t* keep, int32_t n, int32_t* old_to_new, cudaStream_t s) {
  if (n == 0) return 0;
  DBuf<int32_t> prefix(size_t(n) + 1, s);
  GPP_LAUNCH(mask_to_int, grid_stride_blocks(n), kThreads, 0, s, keep, n, prefix.p);
  exclusive_scan_i32(prefix.p, prefix.p, n, s);
  GPP_LAUNCH(prefix_to_map, grid_stride_blocks(n), kThreads, 0, s, keep, prefix.p, n, old_to_new);
  return read_scalar(prefix.p + n);
}

std::pair<int32_t, int32_t> build_old_to_new_pair(const uint8_t* keep_row, int32_t m, int32_t* row_map,
                                                  const uint8_t* keep_col, int32_t n, int32_t* col_map,
                                                  cudaStream_t s) {
  const int32_t tr = (m + kMapTile - 1) / kMapTile, tc = (n + kMapTile - 1) / kMapTile;
  if (tr + tc == 0) return {0, 0};
  MaskPair mp{{keep_row, keep_col}, {m, n}, tr, {row_map, col_map}};
  DBuf<int32_t> counts(size_t(tr + tc), s);
  Status st;
  st.clear(2);   // a mask of no items keeps its total at 0
  GPP_LAUNCH(map_tile_counts, tr + tc, kThreads, 0, s, mp, counts.p);
  GPP_LAUNCH(map_tile_ranks, tr + tc, kThreads, 0, s, mp, counts.p, st.d);
  const int32_t* t = st.read(2);
  return {t[0], t[1]};
}

DevCsr compact_csr_queued(const DevCsr& M, const int32_t* outer_map, int32_t outer_new, const int32_t* inner_map,
                          int32_t inner_new, cudaStream_t s, int32_t* result, int64_t* profile_record) {
  DevCsr out;
  out.rows = outer_new;
  out.cols = inner_new;
  out.nnz = -1;
  out.ptr = dalloc<offset_t>(size_t(outer_new) + 1);
  *profile_record = -1;
  if (outer_new == 0 || inner_new == 0 || M.nnz == 0) {
    check(cudaMemsetAsync(out.ptr, 0, sizeof(offset_t) * (size_t(outer_new) + 1), s), "compact empty ptr");
    check(cudaMemsetAsync(result, 0, 2 * sizeof(int32_t), s), "compact empty result");
    return out;
  }
  // The kept entries are at most the stored ones: the outputs are sized for
  // those, so nothing waits for the kept count before the copy.
  out.idx = dalloc<int32_t>(size_t(M.nnz));
  out.val = dalloc<double>(size_t(M.nnz));
  const int tiles = int((int64_t(M.nnz) + kCompactTile - 1) / kCompactTile);
  DBuf<int32_t> first_row(size_t(tiles), s);
  DBuf<unsigned long long> status(size_t(tiles) + 1, s);   // tile words, then the ticket counter
  status.zero();
  check(cudaMemsetAsync(result, 0, 2 * sizeof(int32_t), s), "compact result");
  GPP_LAUNCH(compact_tile_rows, grid_stride_blocks(int64_t(M.rows) + 1), kThreads, 0, s, M.rows, M.ptr, tiles,
             first_row.p);
  // 128-bit loads need 16-byte aligned index and value arrays (always so for
  // the engine's own matrices; a caller's input may be offset).
  const bool vec = reinterpret_cast<uintptr_t>(M.idx) % 16 == 0 && reinterpret_cast<uintptr_t>(M.val) % 16 == 0;
  // Reads; the writes (4 (outer_new + 1) + 12 nnz') are added to the launch's
  // profile record once the kept count is known.
  const double read_bytes = 4.0 * (M.rows + 1) + 12.0 * M.nnz + 4.0 * M.rows + 4.0 * M.cols + 4.0 * tiles;
  const int grid = std::min(tiles, kNumSMs * 5);   // resident blocks at its register budget
  if (vec)
    GPP_LAUNCH_BYTES(compact_tiles<true>, read_bytes, grid, kThreads, 0, s, M.nnz, M.ptr, M.idx, M.val, outer_map,
                     inner_map, first_row.p, M.rows, tiles, status.p, outer_new, out.ptr, out.idx, out.val, result);
  else
    GPP_LAUNCH_BYTES(compact_tiles<false>, read_bytes, grid, kThreads, 0, s, M.nnz, M.ptr, M.idx, M.val, outer_map,
                     inner_map, first_row.p, M.rows, tiles, status.p, outer_new, out.ptr, out.idx, out.val, result);
  *profile_record = profile_last();
  return out;
}

void compact_csr_finish(DevCsr& out, const int32_t* result_host, int64_t profile_record) {
  if (result_host[1]) throw CudaError("compaction: a tile's look-back timed out waiting for its predecessors");
  out.nnz = out.rows > 0 && out.cols > 0 ? offset_t(result_host[0]) : 0;
  profile_add_bytes(profile_record, 4.0 * (out.rows + 1) + 12.0 * out.nnz);
}

DevCsr compact_csr(const DevCsr& M, const int32_t* outer_map, int32_t outer_new, const int32_t* inner_map,
                   int32_t inner_new, cudaStream_t s) {
  Status st;
  int64_t rec = -1;
  DevCsr out = compact_csr_queued(M, outer_map, outer_new, inner_map, inner_new, s, st.d, &rec);
  compact_csr_finish(out, st.read(2), rec);
  return out;
}

DevCsr transpose_csr(const DevCsr& M, cudaStream_t s) {
  DevCsr t;
  t.rows = M.cols;
  t.cols = M.rows;
  t.nnz = M.nnz;
  t.ptr = dalloc<offset_t>(size_t(t.rows) + 1);
  if (M.nnz > 0) {
    t.idx = dalloc<int32_t>(size_t(M.nnz));
    t.val = dalloc<double>(size_t(M.nnz));
  }
  transpose_csr_into(M, t, s);
  return t;
}

void transpose_csr_into(const DevCsr& M, const DevCsr& t, cudaStream_t s) {
  // Entries ordered by column, each column in stored (row-major) order,
  // i.e. ascending rows (duplicates in stored order): the row-sorted CSR of
  // M^T.  Short columns (all at most kShortColumn long) use atomic slots and
  // a per-column sort of the positions; otherwise a stable radix sort.
  if (M.nnz == 0) {
    check(cudaMemsetAsync(t.ptr, 0, sizeof(offset_t) * (size_t(t.rows) + 1), s), "transpose empty");
    return;
  }
  DBuf<int32_t> cnt(size_t(t.rows) + 1, s);
  cnt.zero();
  const int g = grid_stride_blocks(M.nnz);
  GPP_LAUNCH(histogram, g, kThreads, 0, s, M.idx, M.nnz, cnt.p);
  exclusive_scan_i32(cnt.p, t.ptr, t.rows, s);
  DBuf<int32_t> pos(size_t(M.nnz), s), row(size_t(M.nnz), s);
  Status st;
  st.clear(1);
  GPP_LAUNCH(longest_count, grid_stride_blocks(t.rows), kThreads, 0, s, cnt.p, t.rows, st.d);
  if (st.read(1)[0] <= kShortColumn) {
    DBuf<int32_t> cursor(size_t(t.rows), s);
    check(cudaMemcpyAsync(cursor.p, t.ptr, sizeof(int32_t) * size_t(t.rows), cudaMemcpyDeviceToDevice, s),
          "transpose cursors");
    GPP_LAUNCH(place_positions, g, kThreads, 0, s, M.nnz, M.idx, cursor.p, pos.p);
    GPP_LAUNCH(order_columns, grid_stride_blocks(t.rows), kThreads, 0, s, t.rows, t.ptr, pos.p);
  } else {
    DBuf<uint64_t> keys(size_t(M.nnz), s);
    GPP_LAUNCH(transpose_keys, g, kThreads, 0, s, M.nnz, M.idx, keys.p, pos.p);
    radix_sort_pairs(keys.p, pos.p, M.nnz, s);
  }
  GPP_LAUNCH(row_of_entry, std::max(1, std::min((M.rows + 7) / 8, kNumSMs * 16)), kThreads, 0, s, M.rows, M.ptr,
             row.p);
  GPP_LAUNCH(transpose_gather, g, kThreads, 0, s, M.nnz, pos.p, row.p, M.val, t.idx, t.val);
}

bool csr_structure_valid(const DevCsr& M, cudaStream_t s) {
  if (M.rows < 0 || M.cols < 0 || M.nnz < 0) return false;
  Status st;
  st.clear(1);
  GPP_LAUNCH(check_csr_structure, grid_stride_blocks(std::max<int64_t>(M.rows + 1, M.nnz)), kThreads, 0, s, M.rows,
             M.cols, M.nnz, M.ptr, M.idx, st.d);
  return st.read(1)[0] == 0;
}

bool rows_strictly_sorted(const DevCsr& M, cudaStream_t s) {
  if (M.rows <= 0 || M.nnz <= 1) return true;
  // A matrix does not change between materialisations, so the answer is kept
  // with its cached schedule.
  const RowSchedule& sch = stored_schedule(M);
  if (sch.sorted >= 0) return sch.sorted != 0;
  DBuf<int32_t> bad(1, s);
  bad.zero();
  GPP_LAUNCH(check_sorted, std::max(1, std::min((M.rows + 31) / 32, kNumSMs * 16)), kThreads, 0, s, M.rows, M.ptr,
             M.idx, bad.p);
  sch.sorted = read_scalar(bad.p) == 0 ? 1 : 0;
  return sch.sorted != 0;
}

void gather_by_map(double* dst, const double* src, const int32_t* old_to_new, int32_t n_old, cudaStream_t s) {
  GPP_LAUNCH(gather_kernel, grid_stride_blocks(n_old), kThreads, 0, s, dst, src, old_to_new, n_old);
}

void compose_map(int32_t* next, const int32_t* prev, const int32_t* old_to_new, int32_t n_old, cudaStream_t s) {
  GPP_LAUNCH(compose_kernel, grid_stride_blocks(n_old), kThreads, 0, s, next, prev, old_to_new, n_old);
}

void free_csr(DevCsr& M) {
  forget_schedule(M.ptr);
  dfree(M.ptr);
  dfree(M.idx);
  dfree(M.val);
  M = DevCsr{};
}

}  // namespace gpp
