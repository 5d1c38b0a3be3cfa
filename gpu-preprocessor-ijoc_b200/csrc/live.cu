// Live-structure kernels: row schedules, live statistics, row activity
// summaries and column max |a|.
//
// Reference: cpp/src/presolve/gpu_presolve_kernels.cu:96-517,744-809.
// Each kernel is ONE launch whose blocks split into three roles: a
// thread-per-row pass over short rows, warp-per-row over the medium queue and
// block-per-row over the long queue.  Masked traversals hand every lane the
// live entries with live rank == lane (mod width), exactly the sequence a
// physically compacted row would give, so the floating-point association of
// the activity sums is the reference's:
//   short  : sequential left-to-right sum,
//   medium : 32 lane partials, shfl_down tree 16,8,4,2,1 (own + peer),
//   long   : 256 lane partials, per-warp shfl tree 1,2,4,8,16 then warp
//            aggregates added in warp order (cub::BlockReduce default).
#include "engine.cuh"
#include "live_visit.cuh"

#include <array>

namespace gpp {

namespace {

__device__ __forceinline__ int row_len(const offset_t* ptr, const int32_t* live_deg, int row) {
  return live_deg ? live_deg[row] : int(ptr[row + 1] - ptr[row]);
}

__global__ void classify_rows(const offset_t* __restrict__ ptr, int m, const int32_t* __restrict__ live_deg,
                              int32_t* __restrict__ medium, int32_t* __restrict__ longq,
                              int32_t* __restrict__ counts) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  const int len = row < m ? row_len(ptr, live_deg, row) : 0;
  for (int g = 0; g < 2; ++g) {
    const bool sel = row < m && (g == 0 ? (len > kShortRow && len <= kLongRow) : len > kLongRow);
    const int at = block_append(counts + g, sel);
    if (sel) (g == 0 ? medium : longq)[at] = row;
  }
}

template <class T>
__device__ __forceinline__ T warp_sum_down(T v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, off);
  return v;
}

// cub::BlockReduce<T,256>::Sum order; result valid in thread 0.
template <class T>
__device__ __forceinline__ T block_sum_cub_order(T v, T* warp_aggs) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const T peer = __shfl_down_sync(0xffffffffu, v, off);
    if (lane + off <= 31) v = v + peer;
  }
  if (lane == 0) warp_aggs[threadIdx.x >> 5] = v;
  __syncthreads();
  T total = v;
  if (threadIdx.x == 0) {
    total = warp_aggs[0];
#pragma unroll
    for (int w = 1; w < 8; ++w) total = total + warp_aggs[w];
  }
  __syncthreads();
  return total;
}

template <bool Plain>
struct ActivityTerm {
  const int32_t* idx;
  const double* val;
  const double2* lu;
  double zero_tol;
  L2Hints hint;
  // The term of live stored entry p whose column bounds are b.
  __device__ __forceinline__ void operator()(offset_t p, double2 b, double& lo, double& hi, int& ni, int& pi) const {
    add(ld_stream(val + p, hint.stream), b, lo, hi, ni, pi);   // streamed once: keep L2 for the gathered bounds
  }
  __device__ __forceinline__ void add(double a, double2 b, double& lo, double& hi, int& ni, int& pi) const {
    if constexpr (Plain) {
      // Plain sums of the redundant-row test: infinities propagate.
      lo += a >= 0.0 ? a * b.x : a * b.y;
      hi += a >= 0.0 ? a * b.y : a * b.x;
      return;
    }
    if (fabs(a) <= zero_tol) return;
    const double tlo = a >= 0.0 ? a * b.x : a * b.y;
    const double thi = a >= 0.0 ? a * b.y : a * b.x;
    if (isfinite(tlo)) lo += tlo; else if (tlo < 0.0) ++ni;
    if (isfinite(thi)) hi += thi; else if (thi > 0.0) ++pi;
  }
  __device__ __forceinline__ double2 bounds(offset_t p) const {
    return ld_keep(lu + ld_stream(idx + p, hint.stream), hint.keep);
  }
  // One live entry as the reference's lane partial holds it when the lane
  // sees no other entry: 0.0 + term (or 0.0 when the term is skipped), plus
  // the infinite-term counts.
  __device__ __forceinline__ void slot(double a, double2 b, double& plo, double& phi, int& ni, int& pi) const {
    plo = 0.0;
    phi = 0.0;
    if constexpr (Plain) {
      plo = plo + (a >= 0.0 ? a * b.x : a * b.y);
      phi = phi + (a >= 0.0 ? a * b.y : a * b.x);
      return;
    }
    if (fabs(a) <= zero_tol) return;
    const double tlo = a >= 0.0 ? a * b.x : a * b.y;
    const double thi = a >= 0.0 ? a * b.y : a * b.x;
    if (isfinite(tlo)) plo = plo + tlo; else if (tlo < 0.0) ++ni;
    if (isfinite(thi)) phi = phi + thi; else if (thi > 0.0) ++pi;
  }
};

// Medium rows of at most 32 stored entries (most rows of the random family
// hold 9-32) take eight lanes each, four rows per warp.  For such a row the
// reference's warp association is fixed by live rank k alone: lane k holds
// p[k] = 0.0 + term k (0.0 past the live length), and the shfl_down tree
// 16,8,4,2,1 leaves in lane l < 8, after its first two steps,
// (p[l] + p[l+16]) + (p[l+8] + p[l+24]); the tree 4,2,1 over those eight
// lanes finishes the sum with the same roundings.  So lane l of a group forms
// exactly that value and the group runs the last three steps.  Terms are
// staged in shared memory at their live rank, so masked rows give the same
// sums.
constexpr int kGroupRowMax = 32;

template <bool Plain>
__global__ void __launch_bounds__(kThreads)
activity_kernel(int m, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                const double* __restrict__ val, const double2* __restrict__ lu, double zero_tol,
                const uint8_t* __restrict__ keep_row, const int32_t* __restrict__ live_deg,
                const int32_t* __restrict__ medium, const int32_t* __restrict__ longq,
                const int32_t* __restrict__ counts, int short_blocks, int medium_blocks,
                double* __restrict__ min_fin, double* __restrict__ max_fin, int32_t* __restrict__ min_inf,
                int32_t* __restrict__ max_inf) {
  __shared__ int slots[256];
  __shared__ int warp_counts[8];
  __shared__ double dagg[8];
  __shared__ int iagg[8];
  __shared__ double group_lo[(kThreads / 32) * 4 * kGroupRowMax];
  __shared__ double group_hi[(kThreads / 32) * 4 * kGroupRowMax];
  const ActivityTerm<Plain> term{idx, val, lu, zero_tol, l2_hints()};
  const auto live_at = [&](offset_t p) { return !removed_column(term.bounds(p)); };
  const int b = blockIdx.x;
  if (b < short_blocks) {
    // The next row's pointers and live length are loaded one iteration ahead.
    const int stride = short_blocks * blockDim.x;
    int i_next = b * blockDim.x + threadIdx.x;
    offset_t first_next = i_next < m ? ptr[i_next] : 0, last_next = i_next < m ? ptr[i_next + 1] : 0;
    int len_next = i_next < m && live_deg ? live_deg[i_next] : int(last_next - first_next);
    for (int i = i_next; i < m; i += stride) {
      const offset_t first = first_next, last = last_next;
      const int len = len_next;
      i_next = i + stride;
      first_next = i_next < m ? ptr[i_next] : 0;
      last_next = i_next < m ? ptr[i_next + 1] : 0;
      len_next = i_next < m && live_deg ? live_deg[i_next] : int(last_next - first_next);
      if (len > kShortRow) continue;
      double lo = 0.0, hi = 0.0;
      int ni = 0, pi = 0;
      if (keep_row && !keep_row[i]) {
      } else if (last - first <= kShortRow) {
        // All loads of the (at most 8) entries first, then the sequential sum.
        int col[kShortRow];
        double a[kShortRow];
        double2 bnd[kShortRow];
#pragma unroll
        for (int k = 0; k < kShortRow; ++k) {
          col[k] = first + k < last ? ld_stream(idx + first + k, term.hint.stream) : -1;
          a[k] = first + k < last ? ld_stream(val + first + k, term.hint.stream) : 0.0;
        }
#pragma unroll
        for (int k = 0; k < kShortRow; ++k)
          bnd[k] = col[k] >= 0 ? ld_keep(lu + col[k], term.hint.keep) : make_double2(0.0, 0.0);
#pragma unroll
        for (int k = 0; k < kShortRow; ++k)
          if (col[k] >= 0 && !removed_column(bnd[k])) term.add(a[k], bnd[k], lo, hi, ni, pi);
      } else {
        for (offset_t p = first; p < last; ++p) {
          const double2 bnd = term.bounds(p);
          if (!removed_column(bnd)) term(p, bnd, lo, hi, ni, pi);
        }
      }
      min_fin[i] = lo; max_fin[i] = hi;
      if (min_inf) { min_inf[i] = ni; max_inf[i] = pi; }
    }
    return;
  }
  if (b < short_blocks + medium_blocks) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane >> 3, gl = lane & 7;
    const int nwarps = medium_blocks * (kThreads / 32);
    const int count = counts[0];
    double* glo = group_lo + (warp * 4 + grp) * kGroupRowMax;
    double* ghi = group_hi + (warp * 4 + grp) * kGroupRowMax;
    const auto full_row = [&](int row) {
      double lo = 0.0, hi = 0.0;
      int ni = 0, pi = 0;
      const offset_t first = ptr[row], last = ptr[row + 1];
      const bool all_live = live_deg && live_deg[row] == int(last - first);
      if (!keep_row || keep_row[row])
        live_visit_by<32>(first, last, all_live, live_at, slots + warp * 32, nullptr,
                          [&](offset_t p) { term(p, term.bounds(p), lo, hi, ni, pi); });
      lo = warp_sum_down(lo); hi = warp_sum_down(hi); ni = warp_sum_down(ni); pi = warp_sum_down(pi);
      if (lane == 0) {
        min_fin[row] = lo; max_fin[row] = hi;
        if (min_inf) { min_inf[row] = ni; max_inf[row] = pi; }
      }
    };
    // The row ids and row pointers of later iterations are loaded ahead (the
    // queue entry two iterations ahead, the pointers one ahead), so each
    // iteration's critical path starts at its entries instead of at the queue.
    const int step = nwarps * 4;
    const int q_first = ((b - short_blocks) * (kThreads / 32) + warp) * 4 + grp;
    int row_next = q_first < count ? medium[q_first] : 0;
    int row_after = q_first + step < count ? medium[q_first + step] : 0;
    offset_t first_next = q_first < count ? ptr[row_next] : 0, last_next = q_first < count ? ptr[row_next + 1] : 0;
    for (int q0 = ((b - short_blocks) * (kThreads / 32) + warp) * 4; q0 < count; q0 += step) {
      const int q = q0 + grp;
      const bool have = q < count;
      const int row = row_next;
      const offset_t first = first_next, last = last_next;
      row_next = row_after;
      first_next = q + step < count ? ptr[row_next] : 0;
      last_next = q + step < count ? ptr[row_next + 1] : 0;
      row_after = q + 2 * step < count ? medium[q + 2 * step] : 0;
      const bool kept = have && (!keep_row || keep_row[row]);
      const bool grouped = have && (!kept || last - first <= kGroupRowMax);
      const offset_t end = grouped && kept ? last : first;
      // Every load of the row's (up to) four entries per lane first.
      int col[4];
      double a[4];
      double2 bnd[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const offset_t p = first + gl + 8 * j;
        col[j] = p < end ? ld_stream(idx + p, term.hint.stream) : -1;
        a[j] = p < end ? ld_stream(val + p, term.hint.stream) : 0.0;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j)
        bnd[j] = col[j] >= 0 ? ld_keep(lu + col[j], term.hint.keep) : make_double2(0.0, 0.0);
      // Live mask over the group's 32 stored positions: bit (8j + gl) is
      // stored entry gl + 8j.
      unsigned live_mask = 0;
      bool live[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        live[j] = col[j] >= 0 && !removed_column(bnd[j]);
        live_mask |= ((__ballot_sync(0xffffffffu, live[j]) >> (grp * 8)) & 0xffu) << (8 * j);
      }
      int ni = 0, pi = 0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (!live[j]) continue;
        double plo, phi;
        term.slot(a[j], bnd[j], plo, phi, ni, pi);
        const int rank = __popc(live_mask & ((1u << (gl + 8 * j)) - 1u));
        glo[rank] = plo;
        ghi[rank] = phi;
      }
      __syncwarp();
      const int nlive = __popc(live_mask);
      const auto at = [&](const double* v, int r) { return r < nlive ? v[r] : 0.0; };
      double lo = (at(glo, gl) + at(glo, gl + 16)) + (at(glo, gl + 8) + at(glo, gl + 24));
      double hi = (at(ghi, gl) + at(ghi, gl + 16)) + (at(ghi, gl + 8) + at(ghi, gl + 24));
      __syncwarp();
#pragma unroll
      for (int off = 4; off > 0; off >>= 1) {
        lo = lo + __shfl_down_sync(0xffffffffu, lo, off, 8);
        hi = hi + __shfl_down_sync(0xffffffffu, hi, off, 8);
        ni = ni + __shfl_down_sync(0xffffffffu, ni, off, 8);
        pi = pi + __shfl_down_sync(0xffffffffu, pi, off, 8);
      }
      if (grouped && gl == 0) {
        min_fin[row] = lo; max_fin[row] = hi;
        if (min_inf) { min_inf[row] = ni; max_inf[row] = pi; }
      }
      // Longer medium rows: one warp each, as before.
      unsigned rest = __ballot_sync(0xffffffffu, have && !grouped && gl == 0);
      while (rest) {
        const int src = __ffs(rest) - 1;
        rest &= rest - 1;
        full_row(__shfl_sync(0xffffffffu, row, src));
      }
    }
    return;
  }
  const int lb = b - short_blocks - medium_blocks;
  const int nlong = gridDim.x - short_blocks - medium_blocks;
  const int count = counts[1];
  for (int q = lb; q < count; q += nlong) {
    const int row = longq[q];
    double lo = 0.0, hi = 0.0;
    int ni = 0, pi = 0;
    const offset_t first = ptr[row], last = ptr[row + 1];
    const bool all_live = live_deg && live_deg[row] == int(last - first);
    if (!keep_row || keep_row[row])
      live_visit_by<256>(first, last, all_live, live_at, slots, warp_counts,
                         [&](offset_t p) { term(p, term.bounds(p), lo, hi, ni, pi); });
    lo = block_sum_cub_order(lo, dagg);
    hi = block_sum_cub_order(hi, dagg);
    ni = block_sum_cub_order(ni, iagg);
    pi = block_sum_cub_order(pi, iagg);
    if (threadIdx.x == 0) {
      min_fin[row] = lo; max_fin[row] = hi;
      if (min_inf) { min_inf[row] = ni; max_inf[row] = pi; }
    }
    __syncthreads();
  }
}

__global__ void pack_bounds_kernel(int n, const double* __restrict__ l, const double* __restrict__ u,
                                   const uint8_t* __restrict__ keep, double2* __restrict__ lu) {
  const double removed = __longlong_as_double(static_cast<long long>(kRemovedColumnBits));
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    lu[j] = !keep || keep[j] ? make_double2(l[j], u[j]) : make_double2(removed, removed);
}

// Live degree / singleton support.  Counts and the max live position are
// order independent, so the roles follow stored length.
__device__ __forceinline__ void stats_write(int row, bool active, int count, offset_t position,
                                            const int32_t* idx, const double* val, int32_t* degree,
                                            uint8_t* empty, uint8_t* singleton, int32_t* support,
                                            double* coefficient, unsigned long long* total) {
  if (degree) degree[row] = count;
  if (empty) empty[row] = active && count == 0;
  if (singleton) singleton[row] = active && count == 1;
  if (support) support[row] = count == 1 ? idx[position] : -1;
  if (coefficient) coefficient[row] = count == 1 ? val[position] : 0.0;
  if (total && count) atomicAdd(total, (unsigned long long)count);
}

__global__ void __launch_bounds__(kThreads)
live_stats_kernel(int rows, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                  const double* __restrict__ val, const uint8_t* __restrict__ keep_outer,
                  const uint8_t* __restrict__ keep_inner, const int32_t* __restrict__ medium,
                  const int32_t* __restrict__ longq, const int32_t* __restrict__ counts, int short_blocks,
                  int medium_blocks, int32_t* degree, uint8_t* empty, uint8_t* singleton,
                  int32_t* support, double* coefficient, unsigned long long* total) {
  __shared__ int scount[8];
  __shared__ long long spos[8];
  __shared__ unsigned long long stotal[8];
  const int b = blockIdx.x;
  unsigned long long acc = 0;  // live entries seen by this thread, added once per block
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
      const bool active = !keep_outer || keep_outer[r];
      int count = 0;
      offset_t pos = -1;
      if (active)
        for (offset_t p = first; p < last; ++p)
          if (!keep_inner || keep_inner[__ldcs(idx + p)]) { ++count; pos = p; }
      stats_write(r, active, count, pos, idx, val, degree, empty, singleton, support, coefficient, nullptr);
      acc += unsigned(count);
    }
  } else if (b < short_blocks + medium_blocks) {
    // Four medium rows per warp, eight lanes each: counts and the last live
    // position are order-free, and four rows' loads are in flight at once.
    const int g = threadIdx.x & 7;
    const int nwarps = medium_blocks * (kThreads / 32);
    const int nmedium = counts[0];
    for (int q0 = ((b - short_blocks) * (kThreads / 32) + (threadIdx.x >> 5)) * 4; q0 < nmedium; q0 += nwarps * 4) {
      const int q = q0 + ((threadIdx.x & 31) >> 3);
      int r = -1, count = 0;
      bool active = false;
      long long pos = -1;
      if (q < nmedium) {
        r = medium[q];
        active = !keep_outer || keep_outer[r];
        if (active)
          for (offset_t p = ptr[r] + g; p < ptr[r + 1]; p += 8)
            if (!keep_inner || keep_inner[__ldcs(idx + p)]) { ++count; pos = p; }
      }
      for (int off = 4; off; off >>= 1) {
        count += __shfl_down_sync(0xffffffffu, count, off, 8);
        pos = max(pos, __shfl_down_sync(0xffffffffu, pos, off, 8));
      }
      if (g == 0 && r >= 0) {
        stats_write(r, active, count, offset_t(pos), idx, val, degree, empty, singleton, support, coefficient, nullptr);
        acc += unsigned(count);
      }
    }
  } else {
    const int lb = b - short_blocks - medium_blocks, nlong = gridDim.x - short_blocks - medium_blocks;
    for (int q = lb; q < counts[1]; q += nlong) {
      const int r = longq[q];
      const bool active = !keep_outer || keep_outer[r];
      int count = 0;
      long long pos = -1;
      if (active)
        for (offset_t p = ptr[r] + threadIdx.x; p < ptr[r + 1]; p += kThreads)
          if (!keep_inner || keep_inner[__ldcs(idx + p)]) { ++count; pos = p; }
      for (int off = 16; off; off >>= 1) {
        count += __shfl_down_sync(0xffffffffu, count, off);
        pos = max(pos, __shfl_down_sync(0xffffffffu, pos, off));
      }
      if ((threadIdx.x & 31) == 0) { scount[threadIdx.x >> 5] = count; spos[threadIdx.x >> 5] = pos; }
      __syncthreads();
      if (threadIdx.x == 0) {
        for (int w = 1; w < 8; ++w) { count += scount[w]; pos = max(pos, spos[w]); }
        stats_write(r, active, count, offset_t(pos), idx, val, degree, empty, singleton, support, coefficient, nullptr);
        acc += unsigned(count);
      }
      __syncthreads();
    }
  }
  if (!total) return;
  for (int off = 16; off; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) stotal[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < 8; ++w) t += stotal[w];
    if (t) atomicAdd(total, t);
  }
}

__global__ void __launch_bounds__(kThreads)
col_max_kernel(int rows, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
               const double* __restrict__ val, const uint8_t* __restrict__ keep_row,
               const int32_t* __restrict__ medium, const int32_t* __restrict__ longq,
               const int32_t* __restrict__ counts, int short_blocks, int medium_blocks, double* out) {
  __shared__ double smax[8];
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
      // All (at most 8) loads first; the max is order-free.
      int row[kShortRow];
      double a[kShortRow];
#pragma unroll
      for (int k = 0; k < kShortRow; ++k) {
        row[k] = first + k < last ? __ldcs(idx + first + k) : -1;
        a[k] = first + k < last ? __ldcs(val + first + k) : 0.0;
      }
      double v = 0.0;
#pragma unroll
      for (int k = 0; k < kShortRow; ++k)
        if (row[k] >= 0 && (!keep_row || keep_row[row[k]])) v = fmax(v, fabs(a[k]));
      out[r] = v;
    }
    return;
  }
  if (b < short_blocks + medium_blocks) {
    // Four medium rows per warp, eight lanes each (the max is order-free).
    const int g = threadIdx.x & 7;
    const int nwarps = medium_blocks * (kThreads / 32);
    const int nmedium = counts[0];
    for (int q0 = ((b - short_blocks) * (kThreads / 32) + (threadIdx.x >> 5)) * 4; q0 < nmedium; q0 += nwarps * 4) {
      const int q = q0 + ((threadIdx.x & 31) >> 3);
      int r = -1;
      double v = 0.0;
      if (q < nmedium) {
        r = medium[q];
        for (offset_t p = ptr[r] + g; p < ptr[r + 1]; p += 8)
          if (!keep_row || keep_row[__ldcs(idx + p)]) v = fmax(v, fabs(__ldcs(val + p)));
      }
      for (int off = 4; off; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off, 8));
      if (g == 0 && r >= 0) out[r] = v;
    }
    return;
  }
  const int lb = b - short_blocks - medium_blocks, nlong = gridDim.x - short_blocks - medium_blocks;
  for (int q = lb; q < counts[1]; q += nlong) {
    const int r = longq[q];
    double v = 0.0;
    for (offset_t p = ptr[r] + threadIdx.x; p < ptr[r + 1]; p += kThreads)
      if (!keep_row || keep_row[idx[p]]) v = fmax(v, fabs(val[p]));
    for (int off = 16; off; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < 8; ++w) v = fmax(v, smax[w]);
      out[r] = v;
    }
    __syncthreads();
  }
}

struct Roles {
  int short_blocks, medium_blocks, long_blocks;
};
Roles roles_for(int rows) {
  Roles r;
  r.short_blocks = grid_stride_blocks(rows, kThreads, 16);
  r.medium_blocks = std::min<int>(kNumSMs * 8, (rows + 7) / 8);
  r.long_blocks = std::min<int>(kNumSMs * 4, rows);
  return r;
}

struct ScheduleCache {
  std::array<RowSchedule, 2> slots;
  unsigned next = 0;
  uint64_t epoch = 1;
};
// Thread-lifetime caches are deliberately never destroyed: their device
// buffers live until process exit, when the driver reclaims them, so no CUDA
// call runs during thread-exit destruction (whose order relative to the
// engine stream is unspecified).
ScheduleCache& schedule_cache() {
  static thread_local ScheduleCache* c = [] {
    ctx();
    return new ScheduleCache;
  }();
  return *c;
}

}  // namespace

namespace {
// Row r writes the tiles whose first stored position, or last one (the last
// tile ends at nnz - 1), falls in [ptr[r], ptr[r+1]): every tile gets both
// rows with no search, in one pass over the row pointers.
__global__ void tile_rows_kernel(int rows, offset_t nnz, const offset_t* __restrict__ ptr, int2* __restrict__ tile_rows) {
  constexpr int64_t T = kEntryTile;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    const int64_t a = ptr[r], b = ptr[r + 1];
    if (a == b) continue;
    for (int64_t t = (a + T - 1) / T; t * T < b; ++t) tile_rows[t].x = r;
    for (int64_t t = (a + T) / T - 1; (t + 1) * T <= b; ++t) tile_rows[t].y = r;
    if (b == nnz) tile_rows[(nnz - 1) / T].y = r;
  }
}
}  // namespace

void build_schedule(RowSchedule& s, const DevCsr& M, const int32_t* live_degrees, cudaStream_t st) {
  const size_t rows = size_t(std::max(M.rows, 1));
  if (s.medium.n < rows) s.medium.alloc(rows, st);
  if (s.long_rows.n < rows) s.long_rows.alloc(rows, st);
  if (s.counts.n < 2) s.counts.alloc(2, st);
  check(cudaMemsetAsync(s.counts.p, 0, 2 * sizeof(int32_t), st), "schedule counts");
  GPP_LAUNCH(classify_rows, blocks_for(M.rows), kThreads, 0, st, M.ptr, M.rows, live_degrees, s.medium.p,
             s.long_rows.p, s.counts.p);
  s.tiles = 0;
  s.sorted = -1;
  if (!live_degrees && M.rows > 0 && M.nnz > 0) {
    s.tiles = (int64_t(M.nnz) + kEntryTile - 1) / kEntryTile;
    if (s.tile_rows.n < size_t(s.tiles)) s.tile_rows.alloc(size_t(s.tiles), st);
    GPP_LAUNCH(tile_rows_kernel, grid_stride_blocks(M.rows), kThreads, 0, st, M.rows, M.nnz, M.ptr, s.tile_rows.p);
  }
  s.ptr = M.ptr;
  s.rows = M.rows;
  s.nnz = M.nnz;
  s.epoch = live_degrees ? 0 : schedule_cache().epoch;
}

const RowSchedule& stored_schedule(const DevCsr& M) {
  auto& c = schedule_cache();
  for (auto& s : c.slots)
    if (s.epoch == c.epoch && s.ptr == M.ptr && s.rows == M.rows && s.nnz == M.nnz) return s;
  auto& s = c.slots[c.next++ % c.slots.size()];
  build_schedule(s, M, nullptr, ctx().stream);
  return s;
}

void invalidate_schedules() { ++schedule_cache().epoch; }

void forget_schedule(const offset_t* ptr) {
  if (!ptr) return;
  for (auto& s : schedule_cache().slots)
    if (s.ptr == ptr) s.ptr = nullptr;
}

void live_stats_side(const DevCsr& M, const uint8_t* keep_outer, const uint8_t* keep_inner, int32_t* degree,
                     uint8_t* empty, uint8_t* singleton, int32_t* support, double* coefficient,
                     unsigned long long* total, cudaStream_t s) {
  if (!M.rows) return;
  const RowSchedule& sch = stored_schedule(M);
  const Roles r = roles_for(M.rows);
  // Algorithmic bytes: row pointers, inner indices, both masks, five outputs.
  const double bytes = 4.0 * (M.rows + 1) + 4.0 * M.nnz + (keep_outer ? M.rows : 0) + (keep_inner ? M.cols : 0) +
                       double(M.rows) * ((degree ? 4 : 0) + (empty ? 1 : 0) + (singleton ? 1 : 0) +
                                         (support ? 4 : 0) + (coefficient ? 8 : 0));
  GPP_LAUNCH_BYTES(live_stats_kernel, bytes, r.short_blocks + r.medium_blocks + r.long_blocks, kThreads, 0, s, M.rows,
             M.ptr, M.idx, M.val, keep_outer, keep_inner, sch.medium.p, sch.long_rows.p, sch.counts.p,
             r.short_blocks, r.medium_blocks, degree, empty, singleton, support, coefficient, total);
}

void allocate_stats(Stats& st, int32_t m, int32_t n) {
  auto s = ctx().stream;
  st.row_nnz.alloc(size_t(m), s); st.empty_row.alloc(size_t(m), s); st.singleton_row.alloc(size_t(m), s);
  st.srow_col.alloc(size_t(m), s); st.srow_val.alloc(size_t(m), s);
  st.col_nnz.alloc(size_t(n), s); st.empty_col.alloc(size_t(n), s); st.singleton_col.alloc(size_t(n), s);
  st.scol_row.alloc(size_t(n), s); st.scol_val.alloc(size_t(n), s);
  st.live_nnz.alloc(1, s);
  st.seen_row.alloc(size_t(m), s); st.seen_col.alloc(size_t(n), s);
  st.dirty_row.alloc(size_t(m), s); st.dirty_col.alloc(size_t(n), s);
  st.dirty_row.zero(); st.dirty_col.zero();
  st.deleted.alloc(size_t(m) + size_t(n), s);
  st.counters.alloc(2, s);
  st.valid = false;
}

namespace {

// ---- incremental refresh ---------------------------------------------------
//
// Masks only lose entries between two materialisations, so the statistics of
// the current masks follow from those of the previous ones: a deleted row
// takes one off the degree of every still-kept column it touches (and a
// deleted column likewise for rows), the live total drops by the entries that
// stopped being live, and only rows / columns whose degree changed need their
// empty / singleton flags and singleton support recomputed.  The result is
// the full recount's exactly (integer counts, and the support of a degree-1
// row is its only live entry).

// Rows (first m) and columns (next n) whose mask went from kept to deleted.
__global__ void inc_deleted(int m, int n, const uint8_t* __restrict__ seen_row, const uint8_t* __restrict__ keep_row,
                            const uint8_t* __restrict__ seen_col, const uint8_t* __restrict__ keep_col,
                            int32_t* __restrict__ list, int32_t* counters) {
  const int stride = gridDim.x * blockDim.x;
  const int top = (max(m, n) + stride - 1) / stride * stride;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < top; i += stride) {
    const bool dr = i < m && seen_row[i] && !keep_row[i];
    const bool dc = i < n && seen_col[i] && !keep_col[i];
    const int pr = block_append(counters, dr);
    if (dr) list[pr] = i;
    const int pc = block_append(counters + 1, dc);
    if (dc) list[m + pc] = i;
  }
}

// One warp per deleted outer item: its own statistics are reset, and every
// still-kept inner item it touches loses one degree and is marked dirty.
// `total` (rows only) drops by the item's old degree; `cross_total` (columns
// only) drops by one per kept row it leaves.
__global__ void inc_walk(const int32_t* __restrict__ list, const int32_t* __restrict__ count, const offset_t* __restrict__ ptr,
                         const int32_t* __restrict__ idx, const uint8_t* __restrict__ keep_inner,
                         int32_t* __restrict__ degree, uint8_t* __restrict__ empty, uint8_t* __restrict__ singleton,
                         int32_t* __restrict__ support, double* __restrict__ coefficient,
                         int32_t* __restrict__ inner_degree, uint8_t* __restrict__ inner_dirty,
                         unsigned long long* total, unsigned long long* cross_total) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int k = *count;
  for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < k; w += warps) {
    const int r = list[w];
    unsigned int left = 0;
    for (offset_t p = ptr[r] + lane; p < ptr[r + 1]; p += 32) {
      const int c = idx[p];
      if (keep_inner[c]) {
        atomicSub(inner_degree + c, 1);
        inner_dirty[c] = 1;
        ++left;
      }
    }
    for (int off = 16; off; off >>= 1) left += __shfl_down_sync(0xffffffffu, left, off);
    if (lane == 0) {
      if (total) atomicAdd(total, 0ULL - (unsigned long long)degree[r]);
      if (cross_total && left) atomicAdd(cross_total, 0ULL - (unsigned long long)left);
      degree[r] = 0; empty[r] = 0; singleton[r] = 0; support[r] = -1; coefficient[r] = 0.0;
    }
  }
}

// Flags of the dirty kept items; a degree-1 item finds its only live entry.
__global__ void inc_fix(int rows, const offset_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                        const double* __restrict__ val, const uint8_t* __restrict__ keep_outer,
                        const uint8_t* __restrict__ keep_inner, uint8_t* __restrict__ dirty,
                        const int32_t* __restrict__ degree, uint8_t* __restrict__ empty,
                        uint8_t* __restrict__ singleton, int32_t* __restrict__ support,
                        double* __restrict__ coefficient) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    if (!dirty[r]) continue;
    dirty[r] = 0;
    if (!keep_outer[r]) continue;
    const int d = degree[r];
    empty[r] = d == 0;
    singleton[r] = d == 1;
    int sup = -1;
    double coef = 0.0;
    if (d == 1)
      for (offset_t p = ptr[r]; p < ptr[r + 1]; ++p)
        if (keep_inner[idx[p]]) { sup = idx[p]; coef = val[p]; }
    support[r] = sup;
    coefficient[r] = coef;
  }
}

}  // namespace

void refresh_stats(Stats& st, const WorkingLp& lp, const Plan& plan) {
  // refresh_live_stats (gpu_presolve_kernels.cu:493-517).
  auto s = ctx().stream;
  const int m = lp.m(), n = lp.n();
  if (!st.valid) {
    // A full recount normally follows a fresh plan, whose masks keep every
    // row and column (the host knows: Plan::all_kept): then the counts are
    // the stored lengths, and the sweeps run without masks (no index or mask
    // reads), with the same results.
    const uint8_t* keep_row = plan.all_kept ? nullptr : plan.keep_row.p;
    const uint8_t* keep_col = plan.all_kept ? nullptr : plan.keep_col.p;
    st.live_nnz.zero();
    live_stats_side(lp.A, keep_row, keep_col, st.row_nnz.p, st.empty_row.p, st.singleton_row.p, st.srow_col.p,
                    st.srow_val.p, st.live_nnz.p, s);
    live_stats_side(lp.AT, keep_col, keep_row, st.col_nnz.p, st.empty_col.p, st.singleton_col.p, st.scol_row.p,
                    st.scol_val.p, nullptr, s);
  } else {
    st.counters.zero();
    GPP_LAUNCH(inc_deleted, grid_stride_blocks(std::max(m, n)), kThreads, 0, s, m, n, st.seen_row.p, plan.keep_row.p,
               st.seen_col.p, plan.keep_col.p, st.deleted.p, st.counters.p);
    const int g = kNumSMs * 8;
    GPP_LAUNCH(inc_walk, g, kThreads, 0, s, st.deleted.p, st.counters.p, lp.A.ptr, lp.A.idx, plan.keep_col.p,
               st.row_nnz.p, st.empty_row.p, st.singleton_row.p, st.srow_col.p, st.srow_val.p, st.col_nnz.p,
               st.dirty_col.p, st.live_nnz.p, nullptr);
    GPP_LAUNCH(inc_walk, g, kThreads, 0, s, st.deleted.p + m, st.counters.p + 1, lp.AT.ptr, lp.AT.idx,
               plan.keep_row.p, st.col_nnz.p, st.empty_col.p, st.singleton_col.p, st.scol_row.p, st.scol_val.p,
               st.row_nnz.p, st.dirty_row.p, nullptr, st.live_nnz.p);
    GPP_LAUNCH(inc_fix, grid_stride_blocks(m), kThreads, 0, s, m, lp.A.ptr, lp.A.idx, lp.A.val, plan.keep_row.p,
               plan.keep_col.p, st.dirty_row.p, st.row_nnz.p, st.empty_row.p, st.singleton_row.p, st.srow_col.p,
               st.srow_val.p);
    GPP_LAUNCH(inc_fix, grid_stride_blocks(n), kThreads, 0, s, n, lp.AT.ptr, lp.AT.idx, lp.AT.val, plan.keep_col.p,
               plan.keep_row.p, st.dirty_col.p, st.col_nnz.p, st.empty_col.p, st.singleton_col.p, st.scol_row.p,
               st.scol_val.p);
  }
  st.seen_row.copy_from(plan.keep_row.p, size_t(m));
  st.seen_col.copy_from(plan.keep_col.p, size_t(n));
  st.valid = true;
}

void pack_bounds(const double* l, const double* u, const uint8_t* keep_col, int32_t n, double2* lu,
                 cudaStream_t s) {
  if (n <= 0) return;
  GPP_LAUNCH_BYTES(pack_bounds_kernel, 33.0 * n, grid_stride_blocks(n), kThreads, 0, s, n, l, u, keep_col, lu);
}

namespace {
template <bool Plain>
void launch_activity(const DevCsr& A, const double2* lu, double zero_tol, const uint8_t* keep_row,
                     const int32_t* live_deg, double* lo, double* hi, int32_t* ni, int32_t* pi, double out_bytes,
                     cudaStream_t s) {
  static thread_local RowSchedule* live_schedule = new RowSchedule;  // never destroyed (see schedule_cache)
  const RowSchedule* sch;
  if (live_deg) {
    build_schedule(*live_schedule, A, live_deg, s);
    sch = live_schedule;
  } else {
    sch = &stored_schedule(A);
  }
  const Roles r = roles_for(A.rows);
  // Algorithmic bytes (each array charged once): row pointers, column indices
  // and values, packed column bounds, row mask, live degrees, the outputs.
  const double bytes = 4.0 * (A.rows + 1) + 12.0 * A.nnz + 16.0 * A.cols + (keep_row ? A.rows : 0) +
                       (live_deg ? 4.0 * A.rows : 0) + out_bytes * A.rows;
  const int grid = r.short_blocks + r.medium_blocks + r.long_blocks;
  if constexpr (Plain)
    GPP_LAUNCH_BYTES(activity_kernel<true>, bytes, grid, kThreads, 0, s, A.rows, A.ptr, A.idx, A.val, lu, zero_tol,
                     keep_row, live_deg, sch->medium.p, sch->long_rows.p, sch->counts.p, r.short_blocks,
                     r.medium_blocks, lo, hi, ni, pi);
  else
    GPP_LAUNCH_BYTES(activity_kernel<false>, bytes, grid, kThreads, 0, s, A.rows, A.ptr, A.idx, A.val, lu, zero_tol,
                     keep_row, live_deg, sch->medium.p, sch->long_rows.p, sch->counts.p, r.short_blocks,
                     r.medium_blocks, lo, hi, ni, pi);
}
}  // namespace

void row_activity_summary_packed(const DevCsr& A, const double2* lu, double zero_tol, const uint8_t* keep_row,
                                 const int32_t* live_deg, double* min_fin, double* max_fin, int32_t* min_inf,
                                 int32_t* max_inf, cudaStream_t s) {
  // compute_row_activity_summary (gpu_presolve_kernels.cu:744-787).
  if (!A.rows) return;
  launch_activity<false>(A, lu, zero_tol, keep_row, live_deg, min_fin, max_fin, min_inf, max_inf, 24.0, s);
}

void row_activity_summary(const DevCsr& A, const double* l, const double* u, double zero_tol,
                          const uint8_t* keep_row, const uint8_t* keep_col, const int32_t* live_deg,
                          double* min_fin, double* max_fin, int32_t* min_inf, int32_t* max_inf,
                          cudaStream_t s) {
  if (!A.rows) return;
  DBuf<double2> lu(size_t(std::max(A.cols, 1)), s);
  pack_bounds(l, u, keep_col, A.cols, lu.p, s);
  row_activity_summary_packed(A, lu.p, zero_tol, keep_row, live_deg, min_fin, max_fin, min_inf, max_inf, s);
}

void row_plain_minmax(const DevCsr& A, const double* l, const double* u, const uint8_t* keep_row,
                      const uint8_t* keep_col, const int32_t* live_deg, double* row_min, double* row_max,
                      cudaStream_t s) {
  // Row sums of the redundant-row rule (rule_infeasible_and_redundant_rows.cu:46-156).
  if (!A.rows) return;
  DBuf<double2> lu(size_t(std::max(A.cols, 1)), s);
  pack_bounds(l, u, keep_col, A.cols, lu.p, s);
  launch_activity<true>(A, lu.p, 0.0, keep_row, live_deg, row_min, row_max, nullptr, nullptr, 16.0, s);
}

void col_max_abs(const DevCsr& AT, const uint8_t* keep_row, double* out, cudaStream_t s) {
  // compute_col_max_abs (gpu_presolve_kernels.cu:789-809).
  if (!AT.rows) return;
  const RowSchedule& sch = stored_schedule(AT);
  const Roles r = roles_for(AT.rows);
  const double bytes = 4.0 * (AT.rows + 1) + 12.0 * AT.nnz + (keep_row ? AT.cols : 0) + 8.0 * AT.rows;
  GPP_LAUNCH_BYTES(col_max_kernel, bytes, r.short_blocks + r.medium_blocks + r.long_blocks, kThreads, 0, s, AT.rows,
             AT.ptr, AT.idx, AT.val, keep_row, sch.medium.p, sch.long_rows.p, sch.counts.p, r.short_blocks,
             r.medium_blocks, out);
}

}  // namespace gpp
