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

// Copy roles.  Rows of up to kLongRow stored entries go four to a warp,
// eight lanes per row, the warp's four rows consecutive (so its loads and
// stores cover one contiguous stretch of the matrix); longer rows take a whole
// block.  Entries are copied in stored order, so the schedule is free.
// First of the four consecutive rows of this warp in the group role.
__device__ __forceinline__ int warp_first_row(int block) {
  return (block * (kThreads / 32) + int(threadIdx.x >> 5)) * 4;
}

// Count kept entries of kept rows: short rows by thread, medium by warp,
// long by block (roles as in live.cu).
__global__ void __launch_bounds__(kThreads)
count_kept(int rows, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
           const int32_t* __restrict__ outer_map, const int32_t* __restrict__ inner_map,
           const int32_t* __restrict__ medium, const int32_t* __restrict__ longq,
           const int32_t* __restrict__ counts, int short_blocks, int medium_blocks,
           int32_t* __restrict__ out_counts) {
  __shared__ int scount[8];
  const int b = blockIdx.x;
  if (b < short_blocks) {
    const int stride_ = short_blocks * blockDim.x;
    int r_next = b * blockDim.x + threadIdx.x;
    offset_t first_next = r_next < rows ? ptr[r_next] : 0, last_next = r_next < rows ? ptr[r_next + 1] : 0;
    for (int r = r_next; r < rows; r += stride_) {
      const offset_t first = first_next, last = last_next;
      r_next = r + stride_;   // the next row's pointers, one iteration ahead
      first_next = r_next < rows ? ptr[r_next] : 0;
      last_next = r_next < rows ? ptr[r_next + 1] : 0;
      if (last - first > kShortRow) continue;
      const int nr = outer_map[r];
      if (nr < 0) continue;
      // All (at most 8) index loads, then all map gathers, in flight together.
      int col[kShortRow];
#pragma unroll
      for (int k = 0; k < kShortRow; ++k) col[k] = first + k < last ? __ldcs(idx + first + k) : -1;
      int c = 0;
#pragma unroll
      for (int k = 0; k < kShortRow; ++k) c += col[k] >= 0 && inner_map[col[k]] >= 0;
      out_counts[nr] = c;
    }
    return;
  }
  if (b < short_blocks + medium_blocks) {
    // Four medium rows per warp, eight lanes each.
    const int g = threadIdx.x & 7;
    const int nwarps = medium_blocks * (kThreads / 32);
    for (int q0 = ((b - short_blocks) * (kThreads / 32) + (threadIdx.x >> 5)) * 4; q0 < counts[0]; q0 += nwarps * 4) {
      const int q = q0 + ((threadIdx.x & 31) >> 3);
      int nr = -1, c = 0;
      if (q < counts[0]) {
        const int r = medium[q];
        nr = outer_map[r];
        if (nr >= 0)
          for (offset_t p = ptr[r] + g; p < ptr[r + 1]; p += 8) c += inner_map[__ldcs(idx + p)] >= 0;
      }
      for (int off = 4; off; off >>= 1) c += __shfl_down_sync(0xffffffffu, c, off, 8);
      if (g == 0 && nr >= 0) out_counts[nr] = c;
    }
    return;
  }
  const int lb = b - short_blocks - medium_blocks, nlong = gridDim.x - short_blocks - medium_blocks;
  for (int q = lb; q < counts[1]; q += nlong) {
    const int r = longq[q];
    const int nr = outer_map[r];
    if (nr < 0) continue;  // block-uniform
    int c = 0;
    for (offset_t p = ptr[r] + threadIdx.x; p < ptr[r + 1]; p += kThreads) c += inner_map[__ldcs(idx + p)] >= 0;
    for (int off = 16; off; off >>= 1) c += __shfl_down_sync(0xffffffffu, c, off);
    if ((threadIdx.x & 31) == 0) scount[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < 8; ++w) c += scount[w];
      out_counts[nr] = c;
    }
    __syncthreads();
  }
}

// Stable copy of kept entries (order preserving), remapping inner indices.
// In the group role a ballot over the group's eight lanes ranks the kept
// entries of each round of eight stored entries; every lane runs the warp's
// largest number of rounds, so the ballots stay warp-uniform.
__global__ void __launch_bounds__(kThreads)
copy_kept(int rows, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
          const double* __restrict__ val, const int32_t* __restrict__ outer_map,
          const int32_t* __restrict__ inner_map, const int32_t* __restrict__ longq,
          const int32_t* __restrict__ counts, int group_blocks, const offset_t* __restrict__ out_ptr,
          int32_t* __restrict__ out_idx, double* __restrict__ out_val) {
  __shared__ int wcount[8];
  const int b = blockIdx.x;
  if (b < group_blocks) {
    const int g = threadIdx.x & 7;
    const unsigned shift = unsigned(threadIdx.x & 24);
    const int stride = group_blocks * kThreads / 8;
    for (int r0 = warp_first_row(b); r0 < rows; r0 += stride) {
      const int r = r0 + int((threadIdx.x & 31) >> 3);
      offset_t first = 0, end = 0, w = 0;
      if (r < rows) {
        const offset_t a = ptr[r], e = ptr[r + 1];
        const int nr = e - a > kLongRow ? -1 : outer_map[r];
        if (nr >= 0) {
          first = a;
          end = e;
          w = out_ptr[nr];
        }
      }
      const int rounds = __reduce_max_sync(0xffffffffu, int((end - first + 7) >> 3));
      // Four rounds per step: their index loads, then their column-map
      // gathers and value loads, are all in flight before the first ballot.
      constexpr int kBatch = 4;
      for (int k0 = 0; k0 < rounds; k0 += kBatch) {
        int col[kBatch];
        double v[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
          const offset_t p = first + offset_t(k0 + u) * 8 + g;
          col[u] = k0 + u < rounds && p < end ? __ldcs(idx + p) : -1;
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
          const offset_t p = first + offset_t(k0 + u) * 8 + g;
          col[u] = col[u] >= 0 ? inner_map[col[u]] : -1;
          v[u] = col[u] >= 0 ? __ldcs(val + p) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
          if (k0 + u >= rounds) break;   // warp-uniform
          const unsigned bits = (__ballot_sync(0xffffffffu, col[u] >= 0) >> shift) & 0xFFu;
          if (col[u] >= 0) {
            const offset_t o = w + __popc(bits & ((1u << g) - 1u));
            out_idx[o] = col[u];
            out_val[o] = v[u];
          }
          w += __popc(bits);
        }
      }
    }
    return;
  }
  const int lb = b - group_blocks, nlong = gridDim.x - group_blocks;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int q = lb; q < counts[1]; q += nlong) {
    const int r = longq[q];
    const int nr = outer_map[r];
    if (nr < 0) continue;
    offset_t w = out_ptr[nr];
    for (offset_t chunk = ptr[r]; chunk < ptr[r + 1]; chunk += kThreads) {
      const offset_t p = chunk + threadIdx.x;
      const int c = p < ptr[r + 1] ? inner_map[__ldcs(idx + p)] : -1;
      const unsigned mask = __ballot_sync(0xffffffffu, c >= 0);
      if (lane == 0) wcount[warp] = __popc(mask);
      __syncthreads();
      int before = 0, total = 0;
      for (int k = 0; k < 8; ++k) { before += k < warp ? wcount[k] : 0; total += wcount[k]; }
      if (c >= 0) {
        const offset_t o = w + before + __popc(mask & ((1u << lane) - 1u));
        out_idx[o] = c;
        out_val[o] = __ldcs(val + p);
      }
      w += total;
      __syncthreads();
    }
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

int roles_long(int rows) { return std::min<int>(kNumSMs * 4, rows); }

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

DevCsr compact_csr(const DevCsr& M, const int32_t* outer_map, int32_t outer_new, const int32_t* inner_map,
                   int32_t inner_new, cudaStream_t s, int64_t known_nnz) {
  DevCsr out;
  out.rows = outer_new;
  out.cols = inner_new;
  out.ptr = dalloc<offset_t>(size_t(outer_new) + 1);
  if (outer_new == 0 || inner_new == 0 || M.nnz == 0) {
    check(cudaMemsetAsync(out.ptr, 0, sizeof(offset_t) * (size_t(outer_new) + 1), s), "compact empty ptr");
    return out;
  }
  const RowSchedule& sch = stored_schedule(M);
  const int gb = std::max(1, std::min((M.rows + 31) / 32, kNumSMs * 16));
  const int lb = roles_long(M.rows);
  // Counting reads only: short rows one per thread (more rows in flight),
  // medium rows four per warp, long rows one per block.
  const int sb = grid_stride_blocks(M.rows, kThreads, 16), mb = std::min<int>(kNumSMs * 8, (M.rows + 7) / 8);
  DBuf<int32_t> counts(size_t(outer_new) + 1, s);
  const double count_bytes = 4.0 * (M.rows + 1) + 4.0 * M.nnz + 4.0 * M.rows + 4.0 * M.cols + 4.0 * outer_new;
  GPP_LAUNCH_BYTES(count_kept, count_bytes, sb + mb + lb, kThreads, 0, s, M.rows, M.ptr, M.idx, outer_map, inner_map,
                   sch.medium.p, sch.long_rows.p, sch.counts.p, sb, mb, counts.p);
  exclusive_scan_i32(counts.p, out.ptr, outer_new, s);
  out.nnz = known_nnz >= 0 ? offset_t(known_nnz) : read_scalar(out.ptr + outer_new);
  out.idx = dalloc<int32_t>(size_t(out.nnz));
  out.val = dalloc<double>(size_t(out.nnz));
  const double copy_bytes = 4.0 * (M.rows + 1) + 12.0 * M.nnz + 4.0 * M.rows + 4.0 * M.cols +
                            4.0 * (outer_new + 1) + 12.0 * out.nnz;
  GPP_LAUNCH_BYTES(copy_kept, copy_bytes, gb + lb, kThreads, 0, s, M.rows, M.ptr, M.idx, M.val, outer_map,
                   inner_map, sch.long_rows.p, sch.counts.p, gb, out.ptr, out.idx, out.val);
  return out;
}

DevCsr transpose_csr(const DevCsr& M, cudaStream_t s) {
  // Entries ordered by column, each column in stored (row-major) order,
  // i.e. ascending rows (duplicates in stored order): the row-sorted CSR of
  // M^T.  Short columns (all at most kShortColumn long) use atomic slots and
  // a per-column sort of the positions; otherwise a stable radix sort.
  DevCsr t;
  t.rows = M.cols;
  t.cols = M.rows;
  t.nnz = M.nnz;
  t.ptr = dalloc<offset_t>(size_t(t.rows) + 1);
  if (M.nnz == 0) {
    check(cudaMemsetAsync(t.ptr, 0, sizeof(offset_t) * (size_t(t.rows) + 1), s), "transpose empty");
    return t;
  }
  t.idx = dalloc<int32_t>(size_t(M.nnz));
  t.val = dalloc<double>(size_t(M.nnz));
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
  return t;
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
