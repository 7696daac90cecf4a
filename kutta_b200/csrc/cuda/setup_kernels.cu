// AMG setup on the device: the pairwise aggregation and the coarse pattern
// and entry map of src/kutta/linalg/amg.cpp:25-174, reproducing the host
// (sequential) results exactly.
//
// Pairing (amg.cpp:25-75) is a greedy pass in row order: an unassigned row
// takes its strongest unassigned neighbour. Rows below i are always assigned
// when i is reached, so row i's choice is the first entry of its preference
// list (candidates j > i, strongest first, lowest column on ties) that no
// leader k < i has taken, and i is a leader unless a leader k < i took it.
// These equations are triangular (row i reads only rows below it), so they
// have one solution, the sequential result, and a state that one Jacobi sweep
// leaves unchanged is that solution. The sweeps run on the device until one
// changes nothing (about 50 on 3-D meshes of 10^4-10^6 rows).
//
// The coarse operator's pattern and entry map (amg.cpp:77-158): per
// aggregate, the (coarse column, canonical entry, source entry) triples of its
// members' entries, sorted; the values then come from the refresh kernels
// (k_galerkin, k_m_matrix_diagonal), whose compensated sums over the entry
// map are the setup's own.
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "kernels.hpp"

namespace kb2 {
namespace {
using namespace dev;

#define ROWS(i, n) \
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

// ---- exclusive scan: out[0..n] with out[n] the total ------------------------
constexpr int kScanBlock = 1024;

__device__ __forceinline__ int warp_inclusive(int x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  return x;
}

// Exclusive scan of one value per thread of a 1024-thread block; returns the
// thread's exclusive prefix and writes the block total to *total.
__device__ int block_exclusive(int v, int* total) {
  __shared__ int warp_sums[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int x = warp_inclusive(v);
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) warp_sums[lane] = warp_inclusive(warp_sums[lane]);
  __syncthreads();
  const int prefix = x - v + (warp > 0 ? warp_sums[warp - 1] : 0);
  if (threadIdx.x == 0) *total = warp_sums[31];
  __syncthreads();
  return prefix;
}

__global__ void k_scan_blocks(int n, const int* __restrict__ in, int* __restrict__ out,
                              int* __restrict__ block_sums) {
  __shared__ int total;
  const int i = blockIdx.x * kScanBlock + threadIdx.x;
  const int v = i < n ? in[i] : 0;
  const int prefix = block_exclusive(v, &total);
  if (i < n) out[i] = prefix;
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

// One block: exclusive scan of the block sums in place; out[n] = the total.
__global__ void k_scan_sums(int blocks, int* __restrict__ block_sums, int n, int* __restrict__ out) {
  __shared__ int total;
  const int per = (blocks + kScanBlock - 1) / kScanBlock;
  const int first = threadIdx.x * per;
  int local = 0;
  for (int k = 0; k < per && first + k < blocks; ++k) local += block_sums[first + k];
  int running = block_exclusive(local, &total);
  for (int k = 0; k < per && first + k < blocks; ++k) {
    const int v = block_sums[first + k];
    block_sums[first + k] = running;
    running += v;
  }
  if (threadIdx.x == 0) out[n] = total;
}

__global__ void k_scan_add(int n, int* __restrict__ out, const int* __restrict__ block_sums) {
  const int i = blockIdx.x * kScanBlock + threadIdx.x;
  if (i < n) out[i] += block_sums[blockIdx.x];
}

// ---- pairing -----------------------------------------------------------------
constexpr int kNone = 0x7F7F7F7F;  // "no owner" (memset byte 0x7F), above every row index
// Pairing state per row: -3 left out (no nonzero neighbour, first pass),
// -2 taken by a leader, -1 leader without partner, j >= 0 leader paired with j.
constexpr int kLeftOut = -3, kTaken = -2, kAlone = -1;

// Entry (row, column) of a sorted CSR row, or -1.
__device__ __forceinline__ int find_entry(const int* __restrict__ rows, const int* __restrict__ cols,
                                          int row, int column) {
  int lo = rows[row], hi = rows[row + 1];
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (cols[mid] < column) lo = mid + 1;
    else hi = mid;
  }
  return lo < rows[row + 1] && cols[lo] == column ? lo : -1;
}

// Strength max(|a_ij|, |a_ji|) of the entry j of row i (symmetric pattern).
__device__ __forceinline__ float strength(const int* __restrict__ rows, const int* __restrict__ cols,
                                          const float* __restrict__ vals, int i, int j) {
  const int t = find_entry(rows, cols, cols[j], i);
  const float a = fabsf(vals[j]);
  const float b = t >= 0 ? fabsf(vals[t]) : 0.0f;
  return a > b ? a : b;
}

// Strongest off-diagonal strength of row i.
__device__ float strongest_of(const int* __restrict__ rows, const int* __restrict__ cols,
                              const float* __restrict__ vals, int i) {
  float best = 0.0f;
  for (int j = rows[i]; j < rows[i + 1]; ++j)
    if (cols[j] != i) {
      const float w = strength(rows, cols, vals, i, j);
      best = w > best ? w : best;
    }
  return best;
}

// A candidate: j != i, nonzero strength, w >= threshold * strongest (in
// double, amg.cpp:61-62).
__device__ __forceinline__ bool strong(float w, float strongest, double threshold) {
  return w != 0.0f && static_cast<double>(w) >= threshold * static_cast<double>(strongest);
}

__global__ void k_pair_count(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                             const float* __restrict__ vals, double threshold, int exclude_isolated,
                             int* __restrict__ count, int* __restrict__ state) {
  ROWS(i, n) {
    const float top = strongest_of(rows, cols, vals, i);
    int c = 0;
    for (int j = rows[i]; j < rows[i + 1]; ++j)
      if (cols[j] > i && strong(strength(rows, cols, vals, i, j), top, threshold)) ++c;
    count[i] = c;
    state[i] = (exclude_isolated && top == 0.0f) ? kLeftOut : kAlone;
  }
}

// Preference list of row i at pref[offsets[i]..]: candidates j > i ordered by
// strength descending, then column ascending (the greedy pass's strict >
// over columns in order keeps the lowest column among equal strengths).
__global__ void k_pair_fill(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                            const float* __restrict__ vals, double threshold,
                            const int* __restrict__ offsets, unsigned long long* __restrict__ keys,
                            int* __restrict__ pref) {
  ROWS(i, n) {
    const float top = strongest_of(rows, cols, vals, i);
    const int first = offsets[i];
    int c = first;
    for (int j = rows[i]; j < rows[i + 1]; ++j) {
      if (cols[j] <= i) continue;
      const float w = strength(rows, cols, vals, i, j);
      if (!strong(w, top, threshold)) continue;
      // w >= 0: the complement of its bits orders strengths descending.
      const unsigned long long key =
          (static_cast<unsigned long long>(~__float_as_uint(w)) << 32) |
          static_cast<unsigned>(cols[j]);
      int k = c++;
      while (k > first && keys[k - 1] > key) {
        keys[k] = keys[k - 1];
        --k;
      }
      keys[k] = key;
    }
    for (int k = first; k < c; ++k) pref[k] = static_cast<int>(keys[k] & 0xFFFFFFFFull);
  }
}

__global__ void k_pair_claims(int n, const int* __restrict__ state, int* __restrict__ owner) {
  ROWS(i, n) {
    const int p = state[i];
    if (p >= 0) atomicMin(owner + p, i);
  }
}

// One Jacobi sweep of the pairing equations; changed[0] set if any row moved.
__global__ void k_pair_update(int n, const int* __restrict__ offsets, const int* __restrict__ pref,
                              const int* __restrict__ owner, const int* __restrict__ state,
                              int* __restrict__ next, int* __restrict__ changed) {
  ROWS(i, n) {
    const int old = state[i];
    int p = old;
    if (old != kLeftOut) {
      if (owner[i] != kNone) {
        p = kTaken;
      } else {
        p = kAlone;
        for (int k = offsets[i]; k < offsets[i + 1]; ++k) {
          const int j = pref[k];
          if (owner[j] >= i) {  // no leader below i has taken j
            p = j;
            break;
          }
        }
      }
    }
    next[i] = p;
    if (p != old) changed[0] = 1;
  }
}

__global__ void k_pair_leaders(int n, const int* __restrict__ state, int* __restrict__ flag) {
  ROWS(i, n) flag[i] = state[i] >= kAlone ? 1 : 0;
}

// Aggregate numbers in leader order (amg.cpp:68-72).
__global__ void k_pair_assign(int n, const int* __restrict__ state, const int* __restrict__ owner,
                              const int* __restrict__ id, int* __restrict__ aggregate) {
  ROWS(i, n) {
    const int p = state[i];
    aggregate[i] = p >= kAlone ? id[i] : (p == kTaken ? id[owner[i]] : -1);
  }
}

// ---- singleton absorption (mixed hierarchy) -----------------------------------
__global__ void k_aggregate_sizes(int n, const int* __restrict__ aggregate, int* __restrict__ size) {
  ROWS(i, n) {
    const int g = aggregate[i];
    if (g >= 0) atomicAdd(size + g, 1);
  }
}

// One Jacobi sweep of the absorption pass: a row alone in its aggregate joins
// the pair of its strongest strongly coupled neighbour (strict > over columns
// in order). A neighbour below i is seen where it already went (cur); one
// above i where it started (map0), as in the sequential pass. Only original
// pairs (size0 >= 2) accept rows, and they never shrink.
__global__ void k_absorb_update(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                                const int* __restrict__ diag, const float* __restrict__ vals,
                                double threshold, double coupling, const int* __restrict__ map0,
                                const int* __restrict__ size0, const int* __restrict__ cur,
                                int* __restrict__ next, int* __restrict__ changed) {
  ROWS(i, n) {
    const int own = map0[i];
    int g_best = own;
    if (own >= 0 && size0[own] == 1) {
      const float top = strongest_of(rows, cols, vals, i);
      const double di = fabs(static_cast<double>(vals[diag[i]]));
      float weight = 0.0f;
      for (int j = rows[i]; j < rows[i + 1]; ++j) {
        const int c = cols[j];
        if (c == i) continue;
        const float w = strength(rows, cols, vals, i, j);
        if (w == 0.0f) continue;
        const int g = c < i ? cur[c] : map0[c];
        const double dj = fabs(static_cast<double>(vals[diag[c]]));
        if (g >= 0 && g != own && size0[g] >= 2 && w > weight &&
            static_cast<double>(w) >= threshold * static_cast<double>(top) &&
            static_cast<double>(w) >= coupling * sqrt(di * dj)) {
          g_best = g;
          weight = w;
        }
      }
    }
    next[i] = g_best;
    if (g_best != cur[i]) changed[0] = 1;
  }
}

__global__ void k_mark_used(int n, const int* __restrict__ aggregate, int* __restrict__ used) {
  ROWS(i, n) {
    const int g = aggregate[i];
    if (g >= 0) used[g] = 1;
  }
}

// map[i] = table[map[i]] for map[i] >= 0 (renumbering, and composing passes).
__global__ void k_compose(int n, int* __restrict__ map, const int* __restrict__ table) {
  ROWS(i, n) {
    const int g = map[i];
    if (g >= 0) map[i] = table[g];
  }
}

// ---- coarse pattern and entry map ----------------------------------------------
// Members per aggregate and their triples: size[g] += 1, triples[g] += the
// member's entries whose column is aggregated.
__global__ void k_coarsen_count(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                                const int* __restrict__ aggregate, int* __restrict__ size,
                                int* __restrict__ triples) {
  ROWS(i, n) {
    const int g = aggregate[i];
    if (g < 0) continue;
    int c = 0;
    for (int j = rows[i]; j < rows[i + 1]; ++j)
      if (aggregate[cols[j]] >= 0) ++c;
    atomicAdd(size + g, 1);
    atomicAdd(triples + g, c);
  }
}

__global__ void k_place_members(int n, const int* __restrict__ aggregate,
                                const int* __restrict__ offsets, int* __restrict__ cursor,
                                int* __restrict__ members) {
  ROWS(i, n) {
    const int g = aggregate[i];
    if (g >= 0) members[offsets[g] + atomicAdd(cursor + g, 1)] = i;
  }
}

// Members of each aggregate in row order (amg.cpp:88-91 fills them so).
__global__ void k_sort_members(int nc, const int* __restrict__ offsets, int* __restrict__ members) {
  ROWS(g, nc) {
    const int first = offsets[g], last = offsets[g + 1];
    for (int a = first + 1; a < last; ++a) {
      const int v = members[a];
      int k = a;
      while (k > first && members[k - 1] > v) {
        members[k] = members[k - 1];
        --k;
      }
      members[k] = v;
    }
  }
}

__device__ __forceinline__ bool triple_less(int4 a, int4 b) {
  if (a.x != b.x) return a.x < b.x;
  if (a.y != b.y) return a.y < b.y;
  return a.z < b.z;
}

// Triples (coarse column, canonical entry, source entry) of aggregate g,
// sorted (amg.cpp:96-112); unique[g] = its number of coarse columns. For an
// M-matrix the canonical entry of (i, c) is the smaller of its own position
// and its transpose's, so opposite coarse entries sum in the same order.
__global__ void k_coarsen_triples(int nc, const int* __restrict__ rows,
                                  const int* __restrict__ cols, const int* __restrict__ aggregate,
                                  const int* __restrict__ member_offsets,
                                  const int* __restrict__ members,
                                  const int* __restrict__ triple_offsets, int m_matrix,
                                  int4* __restrict__ triples, int* __restrict__ unique) {
  ROWS(g, nc) {
    const int first = triple_offsets[g];
    int c = first;
    for (int m = member_offsets[g]; m < member_offsets[g + 1]; ++m) {
      const int i = members[m];
      for (int j = rows[i]; j < rows[i + 1]; ++j) {
        const int target = aggregate[cols[j]];
        if (target < 0) continue;
        int canonical = j;
        if (m_matrix) {
          const int t = find_entry(rows, cols, cols[j], i);
          if (t >= 0 && t < canonical) canonical = t;
        }
        const int4 v = make_int4(target, canonical, j, 0);
        int k = c++;
        while (k > first && triple_less(v, triples[k - 1])) {
          triples[k] = triples[k - 1];
          --k;
        }
        triples[k] = v;
      }
    }
    int u = 0;
    for (int k = first; k < c; ++k)
      if (k == first || triples[k].x != triples[k - 1].x) ++u;
    unique[g] = u;
  }
}

// Coarse columns, diagonal positions and the entry map: entry e of the coarse
// operator sums the sources entries[entry_offsets[e] .. entry_offsets[e+1]).
__global__ void k_coarsen_fill(int nc, const int* __restrict__ triple_offsets,
                               const int4* __restrict__ triples, const int* __restrict__ coarse_rows,
                               int* __restrict__ coarse_cols, int* __restrict__ coarse_diag,
                               int* __restrict__ entry_offsets, int* __restrict__ entries) {
  ROWS(g, nc) {
    int e = coarse_rows[g] - 1;
    for (int k = triple_offsets[g]; k < triple_offsets[g + 1]; ++k) {
      const int4 t = triples[k];
      if (k == triple_offsets[g] || t.x != triples[k - 1].x) {
        ++e;
        coarse_cols[e] = t.x;
        entry_offsets[e] = k;
        if (t.x == g) coarse_diag[g] = e;
      }
      entries[k] = t.z;
    }
  }
}

// 1 in flag[0] if some entry (i, j) has no transpose (j, i).
__global__ void k_pattern_symmetric(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                                    int* __restrict__ flag) {
  ROWS(i, n) {
    for (int j = rows[i]; j < rows[i + 1]; ++j)
      if (find_entry(rows, cols, cols[j], i) < 0) flag[0] = 1;
  }
}

int scan_blocks(int n) { return (n + kScanBlock - 1) / kScanBlock; }

}  // namespace

namespace launch {

void exclusive_scan(int n, const int* in, int* out, int* block_sums, cudaStream_t s) {
  const int blocks = scan_blocks(n > 0 ? n : 1);
  ++counter;
  k_scan_blocks<<<blocks, kScanBlock, 0, s>>>(n, in, out, block_sums);
  ++counter;
  k_scan_sums<<<1, kScanBlock, 0, s>>>(blocks, block_sums, n, out);
  ++counter;
  k_scan_add<<<blocks, kScanBlock, 0, s>>>(n, out, block_sums);
}
int scan_scratch(int n) { return scan_blocks(n > 0 ? n : 1); }

void pattern_symmetric(int n, const int* rows, const int* cols, int* flag, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_pattern_symmetric<<<grid_for(n), kBlock, 0, s>>>(n, rows, cols, flag);
}
void pair_count(int n, const int* rows, const int* cols, const float* vals, double threshold,
                int exclude_isolated, int* count, int* state, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_pair_count<<<grid_for(n), kBlock, 0, s>>>(n, rows, cols, vals, threshold, exclude_isolated,
                                              count, state);
}
void pair_fill(int n, const int* rows, const int* cols, const float* vals, double threshold,
               const int* offsets, unsigned long long* keys, int* pref, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_pair_fill<<<grid_for(n), kBlock, 0, s>>>(n, rows, cols, vals, threshold, offsets, keys, pref);
}
void pair_sweep(int n, const int* offsets, const int* pref, int* owner, const int* state,
                int* next, int* changed, cudaStream_t s) {
  if (n <= 0) return;
  // Errors of the memset surface with the next checked call, as launch errors do.
  (void)cudaMemsetAsync(owner, 0x7F, sizeof(int) * static_cast<std::size_t>(n), s);
  ++counter;
  k_pair_claims<<<grid_for(n), kBlock, 0, s>>>(n, state, owner);
  ++counter;
  k_pair_update<<<grid_for(n), kBlock, 0, s>>>(n, offsets, pref, owner, state, next, changed);
}
void pair_leaders(int n, const int* state, int* flag, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_pair_leaders<<<grid_for(n), kBlock, 0, s>>>(n, state, flag);
}
void pair_assign(int n, const int* state, const int* owner, const int* id, int* aggregate,
                 cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_pair_assign<<<grid_for(n), kBlock, 0, s>>>(n, state, owner, id, aggregate);
}
void aggregate_sizes(int n, const int* aggregate, int* size, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_aggregate_sizes<<<grid_for(n), kBlock, 0, s>>>(n, aggregate, size);
}
void absorb_sweep(int n, const int* rows, const int* cols, const int* diag, const float* vals,
                  double threshold, double coupling, const int* map0, const int* size0,
                  const int* cur, int* next, int* changed, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_absorb_update<<<grid_for(n), kBlock, 0, s>>>(n, rows, cols, diag, vals, threshold, coupling,
                                                 map0, size0, cur, next, changed);
}
void mark_used(int n, const int* aggregate, int* used, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_mark_used<<<grid_for(n), kBlock, 0, s>>>(n, aggregate, used);
}
void compose(int n, int* map, const int* table, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_compose<<<grid_for(n), kBlock, 0, s>>>(n, map, table);
}
void coarsen_count(int n, const int* rows, const int* cols, const int* aggregate, int* size,
                   int* triples, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_coarsen_count<<<grid_for(n), kBlock, 0, s>>>(n, rows, cols, aggregate, size, triples);
}
void place_members(int n, const int* aggregate, const int* offsets, int* cursor, int* members,
                   cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_place_members<<<grid_for(n), kBlock, 0, s>>>(n, aggregate, offsets, cursor, members);
}
void sort_members(int nc, const int* offsets, int* members, cudaStream_t s) {
  if (nc <= 0) return;
  ++counter;
  k_sort_members<<<grid_for(nc), kBlock, 0, s>>>(nc, offsets, members);
}
void coarsen_triples(int nc, const int* rows, const int* cols, const int* aggregate,
                     const int* member_offsets, const int* members, const int* triple_offsets,
                     int m_matrix, int4* triples, int* unique, cudaStream_t s) {
  if (nc <= 0) return;
  ++counter;
  k_coarsen_triples<<<grid_for(nc), kBlock, 0, s>>>(nc, rows, cols, aggregate, member_offsets,
                                                    members, triple_offsets, m_matrix, triples,
                                                    unique);
}
void coarsen_fill(int nc, const int* triple_offsets, const int4* triples, const int* coarse_rows,
                  int* coarse_cols, int* coarse_diag, int* entry_offsets, int* entries,
                  cudaStream_t s) {
  if (nc <= 0) return;
  ++counter;
  k_coarsen_fill<<<grid_for(nc), kBlock, 0, s>>>(nc, triple_offsets, triples, coarse_rows,
                                                 coarse_cols, coarse_diag, entry_offsets, entries);
}

}  // namespace launch
}  // namespace kb2
