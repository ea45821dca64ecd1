// libaq.so: the simulator object, binning and grid kernels, and the C ABI
// of the substep (include/aq.h).  The fused substep kernel k_step lives in
// aq_kernels.cuh (see there for the data layout and the algorithm).
//
// Per substep: one k_step launch (grid_op of the accumulated grid as each
// tile is staged, G2P of substep k, P2G of substep k+1 into the other grid,
// which a memset clears first).  Every sort_interval substeps the records
// are re-binned: k_bin (cell key and rank), an exclusive scan of the
// per-cell counts, k_scatter (records and ids into block-wide slot-major
// order), k_items_count + k_items (one work item per occupied block, the
// fullest blocks first).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_run_length_encode.cuh>
#include <cub/device/device_scan.cuh>
#include <new>
#include <string>
#include <vector>

#include "aq_common.cuh"
#include "aq_jit.h"
#include "aq_kernels.cuh"

namespace aq {

// ------------------------------------------------------------ binning

template <int D, class R>
__global__ void __launch_bounds__(256) k_bin(const __grid_constant__ aq_layout L, const SimK<R> K,
                                             const uint64_t* __restrict__ words, int64_t n,
                                             int32_t* __restrict__ keys, int32_t* __restrict__ ranks,
                                             int32_t* __restrict__ cell_count, unsigned* __restrict__ status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const GRec w{words, i, K.W};
  unsigned fl = 0;
  int b[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < D; ++d) b[d] = base_of<R>(decode_slot<R>(L, d, w), K, d, fl);
  constexpr int BS = Geo<D>::BS;
  int key;
  if (D == 3) {
    // cells of a block ordered z fastest, then x, then y: eight consecutive
    // cells then map to distinct 16-byte bank groups of the shared tiles
    // (node stride 1 in z, XS = 4 mod 8 in x)
    const int blk = ((b[0] / BS) * K.nb[1] + b[1] / BS) * K.nb[2] + b[2] / BS;
    key = blk * 64 + ((b[1] % BS) * BS + b[0] % BS) * BS + b[2] % BS;
  } else {
    const int blk = (b[0] / BS) * K.nb[1] + b[1] / BS;
    key = blk * 64 + (b[0] % BS) * BS + b[1] % BS;
  }
  keys[i] = key;
  ranks[i] = atomicAdd(&cell_count[key], 1);
  if (fl) atomicOr(status, fl);
}

// Move every record to its sorted position.  A block's records are ordered
// slot-major over the whole block: first the first record of every cell of
// the block (in cell order), then the second record of every cell, and so
// on.  k_step's warps take this sequence 32 records at a time, so the lanes
// of a warp are in different cells except where a slot holds fewer than 32
// cells.  A warp moves one group of 32 records (grouped storage,
// grec_word): it reads the group's word pairs with coalesced 16-byte loads
// and writes each record's pairs to its destination as 16-byte vectors.
constexpr int SCATTER_T = 128;

__global__ void __launch_bounds__(SCATTER_T) k_scatter(const uint64_t* __restrict__ win,
                                                       const int32_t* __restrict__ pin, uint64_t* __restrict__ wout,
                                                       int32_t* __restrict__ pout, const int32_t* __restrict__ keys,
                                                       const int32_t* __restrict__ ranks,
                                                       const int32_t* __restrict__ start, int64_t n, int W) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t i0 = (int64_t)blockIdx.x * SCATTER_T + warp * 32;  // first record of a group
  const int64_t i = i0 + lane;
  if (i >= n) return;
  const int32_t p = __ldg(pin + i);
  const int key = keys[i];
  const int rk = ranks[i];  // rank of the record in its cell
  const int64_t c0 = (int64_t)(key >> 6) * 64;
  const int myc = key & 63;
  // records before this one: min(count, rk) of every cell, plus one more
  // for every earlier cell that has an rk-th record; with mask_r the cells
  // holding more than r records, that is the sum of popc(mask_r) over
  // r < rk plus popc(mask_rk) below cell myc.
  int64_t b0;
  int t = 0;
  const unsigned am = __activemask();
  const int64_t c0_first = __shfl_sync(am, c0, 0);
  if (am == 0xffffffffu && __all_sync(am, c0 == c0_first)) {
    // the whole warp in one block (the usual case: records come in the
    // previous binning's block order): the warp builds mask_r rank by rank
    // from two cells per lane, one ballot pair per rank
    const int* sc = start + c0;
    const int n_lo = __ldg(sc + lane + 1) - __ldg(sc + lane);
    const int n_hi = __ldg(sc + lane + 33) - __ldg(sc + lane + 32);
    b0 = __ldg(sc);
    const int rmax = (int)__reduce_max_sync(am, (unsigned)rk);
    const unsigned long long below = (1ull << myc) - 1ull;
    int acc = 0;
    for (int r = 0; r <= rmax; ++r) {
      const unsigned long long m =
          (unsigned long long)__ballot_sync(am, n_lo > r) | ((unsigned long long)__ballot_sync(am, n_hi > r) << 32);
      if (r == rk) t = acc + __popcll(m & below);
      acc += __popcll(m);
    }
  } else {
    // lanes of several blocks (or a partial warp): each lane alone.  The
    // block's 65 offsets are read as int4 vectors (start is 256-byte
    // aligned, c0 a multiple of 64).
    const int4* st4 = reinterpret_cast<const int4*>(start + c0);
    int4 v = __ldg(st4);
    b0 = v.x;
#pragma unroll 4
    for (int q = 0; q < 16; ++q) {
      const int4 nv = q < 15 ? __ldg(st4 + q + 1) : make_int4(__ldg(start + c0 + 64), 0, 0, 0);
      const int ss[5] = {v.x, v.y, v.z, v.w, nv.x};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = 4 * q + j, nk = ss[j + 1] - ss[j];
        t += min(nk, rk) + ((k < myc && nk > rk) ? 1 : 0);
      }
      v = nv;
    }
  }
  const int64_t dst = b0 + t;
  const uint64_t* g = win + i0 * W;  // the group's words (i0 is a multiple of 32)
  uint64_t* go = wout + (dst >> 5) * 32 * (int64_t)W;
  const int lo = (int)(dst & 31), W2 = W & ~1;
  for (int k = 0; k < W2; k += 2)
    *reinterpret_cast<ulonglong2*>(go + (k >> 1) * 64 + 2 * lo) =
        __ldg(reinterpret_cast<const ulonglong2*>(g + (k >> 1) * 64 + 2 * lane));
  if (W & 1) go[W2 * 32 + lo] = __ldg(g + W2 * 32 + lane);
  pout[dst] = p;
}

// One work item per occupied cell block: (block, first record, count),
// ordered by decreasing count in buckets of 16 records (largest first, so
// that the persistent CTAs that claim items end on small ones).
// item_info: [0] item count, [1, 1 + IB) bucket sizes, [1 + IB, 1 + 2 IB)
// bucket fill cursors; zeroed before k_items_count.
constexpr int IB = 64;

__device__ __forceinline__ int item_bucket(int c) { return IB - 1 - min(IB - 1, (c - 1) >> 4); }

__global__ void k_items_count(const int32_t* __restrict__ start, int nblk, int32_t* __restrict__ item_info) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblk) return;
  const int c = start[(int64_t)(b + 1) * 64] - start[(int64_t)b * 64];
  if (c > 0) atomicAdd(item_info + 1 + item_bucket(c), 1);
}

// blk_of (sparse grids): the grid block of each compact block index, else null
__global__ void k_items(const int32_t* __restrict__ start, int nblk, int4* __restrict__ items,
                        int32_t* __restrict__ item_info, const int32_t* __restrict__ blk_of) {
  __shared__ int off[IB];
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int k = 0; k < IB; ++k) {
      off[k] = acc;
      acc += item_info[1 + k];
    }
    if (blockIdx.x == 0) item_info[0] = acc;
  }
  __syncthreads();
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblk) return;
  const int s = start[(int64_t)b * 64], c = start[(int64_t)(b + 1) * 64] - s;
  if (c <= 0) return;
  const int k = item_bucket(c);
  items[off[k] + atomicAdd(item_info + 1 + IB + k, 1)] = make_int4(blk_of ? blk_of[b] : b, s, c, 0);
}

// ------------------------------------------------- sparse-grid binning
// The dense binning above counts records per cell of the whole grid; a
// sparse grid's index space can be far larger than the particles need, so
// its binning works on occupied blocks only:
//   k_sbin       grid block and cell-in-block of every record
//   radix sort   records by grid block (CUB), run-length encoding of the
//                sorted blocks: the occupied blocks, their record counts
//   k_occ_keys   compact key (occupied block, cell) and rank in the cell
//   k_cstart     per occupied block, the exclusive scan of its 64 cell
//                counts from the block's first record
// then k_scatter and the work items as in the dense case, with the compact
// keys and offsets; k_activate hands out pool slots to the 3^D blocks
// around every occupied block.

template <int D, class R>
__global__ void __launch_bounds__(256) k_sbin(const __grid_constant__ aq_layout L, const SimK<R> K,
                                              const uint64_t* __restrict__ words, int64_t n,
                                              uint32_t* __restrict__ blk_out, int32_t* __restrict__ cslot,
                                              int32_t* __restrict__ iota, unsigned* __restrict__ status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const GRec w{words, i, K.W};
  unsigned fl = 0;
  int b[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < D; ++d) b[d] = base_of<R>(decode_slot<R>(L, d, w), K, d, fl);
  constexpr int BS = Geo<D>::BS;
  blk_out[i] = (uint32_t)block_of<D>(K.nb, b[0], b[1], b[2]);
  // the dense keys' cell order inside a block (k_bin)
  cslot[i] = D == 3 ? ((b[1] % BS) * BS + b[0] % BS) * BS + b[2] % BS : (b[0] % BS) * BS + b[1] % BS;
  iota[i] = (int32_t)i;
  if (fl) atomicOr(status, fl);
}

// occupied block of sorted record j by binary search in the blocks' first
// records; compact key o * 64 + cell and rank within the cell
__global__ void k_occ_keys(const int32_t* __restrict__ order, const int32_t* __restrict__ cslot,
                           const int32_t* __restrict__ occ_first, const int32_t* __restrict__ n_occ_p, int64_t n,
                           int32_t* __restrict__ keys, int32_t* __restrict__ ranks, int32_t* __restrict__ ccount) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  int lo = 0, hi = *n_occ_p - 1;  // last o with occ_first[o] <= j
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (occ_first[mid] <= j)
      lo = mid;
    else
      hi = mid - 1;
  }
  const int p = order[j];
  const int key = lo * 64 + cslot[p];
  keys[p] = key;
  ranks[p] = atomicAdd(&ccount[key], 1);
}

// one warp per occupied block: cstart[o * 64 + k] = first record of the
// block + the counts of its cells before k; cstart[n_occ * 64] = n
__global__ void k_cstart(const int32_t* __restrict__ ccount, const int32_t* __restrict__ occ_first,
                         const int32_t* __restrict__ n_occ_p, int64_t n, int32_t* __restrict__ cstart) {
  const int n_occ = *n_occ_p;
  const int lane = threadIdx.x & 31;
  const int o = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (o >= n_occ) {
    if (o == n_occ && lane == 0) cstart[(int64_t)n_occ * 64] = (int32_t)n;
    return;
  }
  const int c0 = ccount[(int64_t)o * 64 + 2 * lane], c1 = ccount[(int64_t)o * 64 + 2 * lane + 1];
  int x = c0 + c1;
#pragma unroll
  for (int k = 1; k < 32; k <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, k);
    if (lane >= k) x += y;
  }
  const int before = occ_first[o] + x - c0 - c1;
  cstart[(int64_t)o * 64 + 2 * lane] = before;
  cstart[(int64_t)o * 64 + 2 * lane + 1] = before + c0;
}

// Empty the pools for a new set of active blocks: zero the slots handed out
// so far in both pools, and their table entries
template <class R4>
__global__ void k_pool_reset(int32_t* __restrict__ bptr, int32_t* __restrict__ pool_blk,
                             const int32_t* __restrict__ n_alloc, int cap, R4* __restrict__ p0, R4* __restrict__ p1) {
  const int used = min(*n_alloc, cap);
  R4 z;
  z.x = z.y = z.z = z.w = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)used * 64;
       i += (int64_t)gridDim.x * blockDim.x) {
    p0[i] = z;
    p1[i] = z;
    if ((i & 63) == 0) {
      const int64_t s = i >> 6;
      if (pool_blk[s] >= 0) bptr[pool_blk[s]] = -1;
      pool_blk[s] = -1;
    }
  }
}

// zero the slots handed out so far in one pool (the P2G target)
template <class R4>
__global__ void k_pool_clear(const int32_t* __restrict__ n_alloc, int cap, R4* __restrict__ pool) {
  const int used = min(*n_alloc, cap);
  R4 z;
  z.x = z.y = z.z = z.w = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)used * 64;
       i += (int64_t)gridDim.x * blockDim.x)
    pool[i] = z;
}

// Pool slots for the 3^D grid blocks around every occupied block, in two
// passes so that a block wanted by several occupied neighbours takes one
// slot: pass 0 marks every wanted block (-2; all writers store the same
// value), pass 1 lets the one thread whose compare-and-swap moves the mark
// on (-2 -> -3) take a slot for it.
template <int D>
__device__ __forceinline__ int64_t around_block(const int32_t* occ_blk, int NN, int64_t t, int nb0, int nb1,
                                                int nb2) {
  const int o = (int)(t / NN), e = (int)(t - (int64_t)o * NN);
  const int blk = occ_blk[o];
  int b0, b1, b2 = 0;
  if (D == 3) {
    b2 = blk % nb2;
    b1 = (blk / nb2) % nb1;
    b0 = blk / nb2 / nb1;
  } else {
    b1 = blk % nb1;
    b0 = blk / nb1;
  }
  const int c0 = b0 + (D == 3 ? e / 9 : e / 3) - 1, c1 = b1 + (D == 3 ? (e / 3) % 3 : e % 3) - 1,
            c2 = D == 3 ? b2 + e % 3 - 1 : 0;
  if (c0 < 0 || c0 >= nb0 || c1 < 0 || c1 >= nb1 || (D == 3 && (c2 < 0 || c2 >= nb2))) return -1;
  return D == 3 ? ((int64_t)c0 * nb1 + c1) * nb2 + c2 : (int64_t)c0 * nb1 + c1;
}

template <int D>
__global__ void k_activate(const int32_t* __restrict__ occ_blk, const int32_t* __restrict__ n_occ_p, int nb0, int nb1,
                           int nb2, int32_t* __restrict__ bptr, int32_t* __restrict__ n_alloc,
                           int32_t* __restrict__ pool_blk, int cap, unsigned* __restrict__ status, int pass) {
  constexpr int NN = D == 3 ? 27 : 9;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)*n_occ_p * NN) return;
  const int64_t nbk = around_block<D>(occ_blk, NN, t, nb0, nb1, nb2);
  if (nbk < 0) return;
  if (pass == 0) {
    bptr[nbk] = -2;
    return;
  }
  if (atomicCAS(bptr + nbk, -2, -3) != -2) return;  // another thread takes this block
  const int slot = atomicAdd(n_alloc, 1);
  if (slot < cap) {
    pool_blk[slot] = (int32_t)nbk;
    bptr[nbk] = slot;
  } else {
    bptr[nbk] = -1;
    atomicOr(status, AQ_ST_POOL_FULL);
  }
}

// node masses of a sparse grid as a dense float array (zero where no block)
template <int D, class R4>
__global__ void k_grid_mass_sparse(const R4* __restrict__ pool, const int32_t* __restrict__ bptr, int r0, int r1,
                                   int r2, int nb1, int nb2, float* __restrict__ out, int64_t n) {
  const int nb[3] = {0, nb1, nb2};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int i0, i1, i2 = 0;
    if (D == 3) {
      i2 = (int)(i % r2);
      i1 = (int)((i / r2) % r1);
      i0 = (int)(i / r2 / r1);
    } else {
      i1 = (int)(i % r1);
      i0 = (int)(i / r1);
    }
    const int sl = bptr[block_of<D>(nb, i0, i1, i2)];
    out[i] = sl >= 0 ? (float)pool[node_in_slot<D>(sl, i0, i1, i2)].x : 0.f;
  }
}

// Exclusive scan of n int32 counts into out[0..n] (out[n] = total), in
// tiles of 4096: per-tile sums, one CTA scans the tile sums, per-tile scan.
constexpr int SCAN_T = 1024, SCAN_V = 4, SCAN_TILE = SCAN_T * SCAN_V;

__device__ __forceinline__ int block_excl_scan(int v, int* sh, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    sh[lane] = s;
  }
  __syncthreads();
  total = sh[(blockDim.x >> 5) - 1];
  const int r = x - v + (warp ? sh[warp - 1] : 0);
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_sums(const int32_t* __restrict__ in, int64_t n,
                                                      int32_t* __restrict__ sums) {
  __shared__ int sh[32];
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_V;
  int v = 0;
#pragma unroll
  for (int k = 0; k < SCAN_V; ++k) v += base + k < n ? in[base + k] : 0;
  int total;
  block_excl_scan(v, sh, total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_top(int32_t* __restrict__ sums, int nt, int32_t* __restrict__ out,
                                                     int64_t n) {
  __shared__ int sh[32];
  const int per = (nt + SCAN_T - 1) / SCAN_T;
  const int b = threadIdx.x * per;
  int v = 0;
  for (int k = 0; k < per; ++k) v += b + k < nt ? sums[b + k] : 0;
  int total;
  int run = block_excl_scan(v, sh, total);
  for (int k = 0; k < per; ++k) {
    if (b + k < nt) {
      const int s = sums[b + k];
      sums[b + k] = run;
      run += s;
    }
  }
  if (threadIdx.x == 0) out[n] = total;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_apply(const int32_t* __restrict__ in, int64_t n,
                                                       const int32_t* __restrict__ offs, int32_t* __restrict__ out) {
  __shared__ int sh[32];
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_V;
  int loc[SCAN_V], v = 0;
#pragma unroll
  for (int k = 0; k < SCAN_V; ++k) {
    loc[k] = base + k < n ? in[base + k] : 0;
    v += loc[k];
  }
  int total;
  int run = block_excl_scan(v, sh, total) + offs[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_V; ++k) {
    if (base + k < n) out[base + k] = run;
    run += loc[k];
  }
}

// decode records into particle order
template <class T>
__global__ void __launch_bounds__(128) k_get_state(const __grid_constant__ aq_layout L,
                                                   const uint64_t* __restrict__ words,
                                                   const int32_t* __restrict__ pid, T* __restrict__ out, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int ns = L.n_slots;
  const GRec w{words, i, L.n_words};
  const int64_t dst = pid[i];
  for (int s = 0; s < ns; ++s) out[dst * ns + s] = (T)decode_slot<double>(L, s, w);
}

// Records from the simulator's grouped storage to contiguous records in
// particle order (record i goes to out[pid[i]]).
// base: the id of out's first record (a streamed chunk's first particle).
__global__ void k_words_ungroup(const uint64_t* __restrict__ in, const int32_t* __restrict__ pid,
                                uint64_t* __restrict__ out, int64_t n, int W, int64_t base = 0) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t a = pid[i] - base;
  for (int j = 0; j < W; ++j) out[a * W + j] = in[grec_word(i, j, W)];
}

// Contiguous records (record i at in[i W]) into grouped storage, same order,
// from grouped position base on (appended records: base = records already
// stored; the words of records below base are not touched).
__global__ void k_words_group(const uint64_t* __restrict__ in, uint64_t* __restrict__ out, int64_t n, int W,
                              int64_t base = 0) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int j = 0; j < W; ++j) out[grec_word(base + i, j, W)] = in[i * W + j];
}

// Grouped records back to the order of their ids (record i to grouped
// position pid[i] - base): a streamed chunk from its binned order to
// particle order.
__global__ void k_words_unpermute(const uint64_t* __restrict__ in, const int32_t* __restrict__ pid,
                                  uint64_t* __restrict__ out, int64_t n, int W, int64_t base) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t a = pid[i] - base;
  for (int j = 0; j < W; ++j) out[grec_word(a, j, W)] = in[grec_word(i, j, W)];
}

__global__ void k_iota(int32_t* p, int64_t n, int64_t base = 0) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = (int32_t)(base + i);
}

// Node masses (component 0 of the row-major m, m v grid) as float.
template <class R4>
__global__ void k_grid_mass(const R4* __restrict__ g, float* __restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)g[i].x;
}

template <int D, class R>
__global__ void __launch_bounds__(256) k_loss(const __grid_constant__ aq_layout L, const SimK<R> K,
                                              const uint64_t* __restrict__ words, int64_t n, double* out) {
  __shared__ double sh[8];
  double acc = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const GRec w{words, i, K.W};
    double vv = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const double v = (double)decode_slot<R>(L, D + d, w);
      vv += v * v;
    }
    if (D == 3)
      acc += 0.5 * (double)K.p_mass * vv + (double)K.grav * (double)K.p_mass * (double)decode_slot<R>(L, 1, w);
    else
      acc += vv;
  }
#pragma unroll
  for (int k = 16; k; k >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, k);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += sh[k];
    atomicAdd(out, s);
  }
}

// Per-slot statistics of the decoded state (features of the sensitivity
// surrogate).  blockIdx.y is the slot; out[slot * 5 + k] accumulates
// k = 0: sum |v|, 1: sum v, 2: sum v^2, 3: max |v| (as the bit pattern of a
// non-negative double, which orders like the value), 4: sum |v - ref|
// (ref: n x n_slots values in particle order, or null).
template <class T>
__global__ void __launch_bounds__(256) k_field_stats(const __grid_constant__ aq_layout L,
                                                     const uint64_t* __restrict__ words,
                                                     const int32_t* __restrict__ pid, const T* __restrict__ ref,
                                                     int64_t n, double* __restrict__ out) {
  __shared__ double sh[8][5];
  const int s = blockIdx.y, ns = L.n_slots;
  double a[5] = {0, 0, 0, 0, 0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = decode_slot<double>(L, s, GRec{words, i, L.n_words});
    const double av = fabs(v);
    a[0] += av;
    a[1] += v;
    a[2] += v * v;
    a[3] = fmax(a[3], av);
    if (ref) a[4] += fabs(v - (double)ref[(int64_t)pid[i] * ns + s]);
  }
#pragma unroll
  for (int k = 16; k; k >>= 1) {
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const double o = __shfl_xor_sync(0xffffffffu, a[j], k);
      a[j] = j == 3 ? fmax(a[j], o) : a[j] + o;
    }
  }
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
    for (int j = 0; j < 5; ++j) sh[warp][j] = a[j];
  __syncthreads();
  if (threadIdx.x < 5) {
    const int j = threadIdx.x;
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = j == 3 ? fmax(t, sh[w][j]) : t + sh[w][j];
    if (j == 3)
      atomicMax(reinterpret_cast<unsigned long long*>(out + s * 5 + 3), (unsigned long long)__double_as_longlong(t));
    else
      atomicAdd(out + s * 5 + j, t);
  }
}

// ------------------------------------------------------------------ host

struct SimBase {
  virtual ~SimBase() {}
  virtual int substeps(int n, cudaStream_t st) = 0;
  virtual int loss(double* h, cudaStream_t st) = 0;
  virtual int sort(cudaStream_t st) = 0;
  virtual size_t smem_bytes(bool reg_record) const = 0;
  virtual void set_collider(const aq_sim* sim) = 0;
  virtual int setup_kernel(bool col) = 0;
  virtual int load_chunk(int64_t c, cudaStream_t st) = 0;
};

}  // namespace aq

struct aq_sim {
  aq_params P;
  aq_layout L;
  int W = 0, WS = 0, NS = 0, D = 0;
  int64_t n = 0;    // active records
  int64_t cap = 0;  // records the device buffers hold (n_particles at creation)
  uint64_t* words[2] = {nullptr, nullptr};
  int32_t* pid[2] = {nullptr, nullptr};
  int cur = 0;
  void* grid[2] = {nullptr, nullptr};
  int64_t ncell = 0, nkeys = 0;
  int nblk = 0;
  int32_t *keys = nullptr, *ranks = nullptr, *cell_count = nullptr, *cell_start = nullptr, *scan_sums = nullptr;
  int4* items = nullptr;
  int32_t* n_items = nullptr;  // [0] item count, then k_items' bucket sizes and cursors
  int32_t* item_ctr = nullptr;  // [2] k_step's item claim counters
  int64_t step_launches = 0;
  int64_t max_items = 0;
  unsigned* status = nullptr;
  unsigned long long* fallbacks = nullptr;
  double *rmax = nullptr, *rmin = nullptr;
  double* dloss = nullptr;
  double* dstats = nullptr;  // aq_sim_field_stats accumulators
  // SDF collider (aq_sim_set_collider): caller-owned volumes and its motion
  int col_on = 0, col_center = 0, col_dims[3] = {0, 0, 0}, col_off[3] = {0, 0, 0};
  const float* col_sdf = nullptr;
  const float* col_nrm = nullptr;
  double col_theta = 0, col_height = 0, col_omega = 0, col_rate = 0;
  int col_node_cv = 0;  // collider velocity from the node (sdf_collision_no_arg) instead of the rotated index
  // sparse grid (P.sparse): block table, node pools (grid[] points at them)
  // and the buffers of the sparse binning; all but the pools and the
  // occupancy-sized arrays live in the slab
  int32_t* bptr = nullptr;      // grid block -> pool slot, -1: none
  int32_t* n_alloc = nullptr;   // [0] slots handed out, [1] occupied blocks of the last binning
  int32_t* pool_blk = nullptr;  // pool slot -> grid block (-1: free)
  int pool_cap = 0;             // node blocks per pool
  int64_t occ_cap = 0;          // occupied blocks ccount / cstart are sized for
  int32_t *ccount = nullptr, *cstart = nullptr;
  uint32_t *sblk = nullptr, *sblk_sorted = nullptr;
  int32_t *order_in = nullptr, *order = nullptr, *cslot = nullptr;
  int32_t *occ_blk = nullptr, *occ_len = nullptr, *occ_first = nullptr;
  void* cub_tmp = nullptr;
  size_t cub_bytes = 0;
  int blk_bits = 1;  // bits of a grid block index (radix sort)
  void* slab = nullptr;      // the one device allocation all buffers above live in
  int ranges_on = 0;
  // streamed (out-of-core) mode, aq_sim_create_streamed: the records of all
  // n_total particles live in pinned host memory, chunk c (particles
  // c * chunk onward) from h_words + c * grouped_words(chunk, W), in particle
  // order in the device's grouped layout, so particle ids never cross the
  // link; every pass over the particles moves each chunk through the device
  // buffers, where n is then that chunk's count.  words_dl: the chunk put
  // back in particle order for its download.  chunk 0: in-core.
  int64_t chunk = 0;
  int64_t n_total = 0;
  uint64_t* h_words = nullptr;
  uint64_t* words_dl = nullptr;
  // uploads alternate between two buffers (the slab's first record buffer
  // and words_up2), so an upload never waits for the binning of the chunk
  // before; the slab's second record buffer takes the binned chunk
  uint64_t* words_up[2] = {nullptr, nullptr};
  uint64_t* words_binned = nullptr;
  int up_par = 0;
  cudaEvent_t ev_read[2] = {nullptr, nullptr};  // the binning that last read words_up[k]
  // uploads and downloads run on their own streams beside the kernels
  cudaStream_t up_st = nullptr, down_st = nullptr;
  cudaEvent_t ev_start = nullptr, ev_up = nullptr, ev_ready = nullptr, ev_down = nullptr;
  std::vector<cudaEvent_t> ev_chunk_down;  // per chunk: its last download (its host words are final)
  int64_t step = 0;
  int last_grid = 0;  // grid[] holding the P2G sums of the latest substep
  int since_sort = 0;
  bool sorted = false;
  int64_t launches = 0;
  int step_grid = 0;
  size_t step_smem = 0;  // dynamic shared memory of the k_step in use
  void* jit_fn = nullptr;  // CUfunction of the layout-specialized k_step, or null
  std::string jit_error;
  aq::SimBase* impl = nullptr;
  // kernel timing (aq_sim_profile_*): event pairs per kernel kind
  static constexpr int PROF_CAP = 8192;
  int prof_on = 0;
  cudaEvent_t* prof_ev[2] = {nullptr, nullptr};  // [PROF_CAP * 2]
  int prof_n[2] = {0, 0};
};

namespace aq {

template <int D, bool HF, bool HM, class R>
static int setup_step_kernel(aq_sim* s, size_t smem_jit, size_t smem_aot, bool col);

template <int D, bool HF, bool HM, class R>
struct SimImpl final : SimBase {
  aq_sim* s;
  SimK<R> K;
  explicit SimImpl(aq_sim* sim) : s(sim) {
    const aq_params& P = sim->P;
    memset(&K, 0, sizeof(K));
    for (int d = 0; d < 3; ++d) {
      K.res[d] = d < D ? P.res[d] : 1;
      K.nb[d] = d < D ? (P.res[d] + Geo<D>::BS - 1) / Geo<D>::BS : 1;
      K.lb[d] = P.lb[d];
      K.ub[d] = P.ub[d];
      K.clip_lo[d] = (R)(P.lb[d] * P.dx);
      K.clip_hi[d] = (R)(P.ub[d] * P.dx);
    }
    K.W = sim->W;
    K.WS = sim->WS;
    K.friction = P.use_friction;
    K.bound_clip = P.use_bound_clip;
    K.n_mat = P.n_materials < 1 ? 1 : P.n_materials;
    K.inv_dx = (R)(1.0 / P.dx);
    K.dx = (R)P.dx;
    K.dt = (R)P.dt;
    K.p_mass = (R)P.p_mass;
    K.stress_coef = (R)(-(P.dt * P.p_vol * 4.0 * (1.0 / P.dx) * (1.0 / P.dx)));
    K.four_inv_dx = (R)(4.0 * (1.0 / P.dx));
    K.grav = (R)P.gravity;
    for (int m = 0; m < AQ_MAX_MATERIALS; ++m) {
      K.mat_kind[m] = P.mat[m].kind;
      K.mu[m] = (R)P.mat[m].mu;
      K.lam[m] = (R)P.mat[m].lam;
    }
  }

  int setup_kernel(bool col) override {
    return setup_step_kernel<D, HF, HM, R>(s, smem_bytes(jit_reg_record(s->L)), smem_bytes(false), col);
  }

  void set_collider(const aq_sim* c) override {
    const aq_params& P = c->P;
    K.col_on = c->col_on && D == 3;
    K.col_n = c->col_center;
    for (int k = 0; k < 3; ++k) {
      K.col_dims[k] = c->col_dims[k];
      K.col_off[k] = c->col_off[k];
      K.col_lo[k] = (int)P.lb[k];
      K.col_hi[k] = (int)P.ub[k];
    }
    K.col_sdf = c->col_sdf;
    K.col_nrm = c->col_nrm;
    K.col_omega = (R)c->col_omega;
    K.col_node_cv = c->col_node_cv;
  }

  // the grid tile and the warp tiles, plus a record slot per thread unless
  // the kernel keeps records in registers (layout-specialized build)
  size_t smem_bytes(bool reg_record) const override {
    const size_t b = sizeof(typename R4T<R>::type) * (NWARP + 1) * Geo<D>::TNP;
    return b + (reg_record ? 0 : sizeof(uint64_t) * (size_t)CH * s->WS);
  }

  int sort(cudaStream_t st) override {
    if (s->P.sparse) return sort_sparse(st);
    aq_sim* S_ = s;
    const int64_t n = S_->n;
    AQ_CUDA_TRY(cudaMemsetAsync(S_->cell_count, 0, sizeof(int32_t) * S_->nkeys, st));
    AQ_CUDA_TRY(cudaMemsetAsync(S_->n_items, 0, sizeof(int32_t) * (1 + 2 * IB), st));
    k_bin<D, R><<<grid_for(n, 256), 256, 0, st>>>(S_->L, K, S_->words[S_->cur], n, S_->keys, S_->ranks, S_->cell_count,
                                                  S_->status);
    const int nt = (int)((S_->nkeys + SCAN_TILE - 1) / SCAN_TILE);
    k_scan_sums<<<nt, SCAN_T, 0, st>>>(S_->cell_count, S_->nkeys, S_->scan_sums);
    k_scan_top<<<1, SCAN_T, 0, st>>>(S_->scan_sums, nt, S_->cell_start, S_->nkeys);
    k_scan_apply<<<nt, SCAN_T, 0, st>>>(S_->cell_count, S_->nkeys, S_->scan_sums, S_->cell_start);
    const int nxt = 1 - S_->cur;
    k_scatter<<<grid_for(n, SCATTER_T), SCATTER_T, 0, st>>>(S_->words[S_->cur], S_->pid[S_->cur], S_->words[nxt], S_->pid[nxt],
                                                S_->keys, S_->ranks, S_->cell_start, n, S_->W);
    k_items_count<<<grid_for(S_->nblk, 256), 256, 0, st>>>(S_->cell_start, S_->nblk, S_->n_items);
    k_items<<<grid_for(S_->nblk, 256), 256, 0, st>>>(S_->cell_start, S_->nblk, S_->items, S_->n_items, nullptr);
    AQ_CUDA_TRY(cudaGetLastError());
    S_->cur = nxt;
    S_->launches += 7;
    S_->since_sort = 0;
    S_->sorted = true;
    return AQ_OK;
  }

  // Grow a device buffer (contents dropped) to at least `need` elements.
  template <class T>
  static int grow(T*& p, int64_t& cap_elems, int64_t need) {
    if (need <= cap_elems && p) return AQ_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap_elems = 0;
    const cudaError_t e = cudaMalloc((void**)&p, sizeof(T) * (size_t)need);
    if (e != cudaSuccess) {
      set_last_cuda_error(e, "cudaMalloc (sparse grid)");
      return AQ_E_NOMEM;
    }
    cap_elems = need;
    return AQ_OK;
  }

  // Binning of a sparse grid: see the kernels' comment.  Reads the number of
  // occupied blocks back to the host (one synchronization per re-binning) to
  // size the per-block arrays and the pools.
  int sort_sparse(cudaStream_t st) {
    aq_sim* S_ = s;
    const int64_t n = S_->n;
    k_sbin<D, R><<<grid_for(n, 256), 256, 0, st>>>(S_->L, K, S_->words[S_->cur], n, S_->sblk, S_->cslot,
                                                   S_->order_in, S_->status);
    size_t tb = S_->cub_bytes;
    AQ_CUDA_TRY(cub::DeviceRadixSort::SortPairs(S_->cub_tmp, tb, S_->sblk, S_->sblk_sorted, S_->order_in, S_->order,
                                                (int)n, 0, S_->blk_bits, st));
    tb = S_->cub_bytes;
    AQ_CUDA_TRY(cub::DeviceRunLengthEncode::Encode(S_->cub_tmp, tb, S_->sblk_sorted,
                                                   reinterpret_cast<uint32_t*>(S_->occ_blk), S_->occ_len,
                                                   S_->n_alloc + 1, (int)n, st));
    int32_t n_occ = 0;
    AQ_CUDA_TRY(cudaMemcpyAsync(&n_occ, S_->n_alloc + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    AQ_CUDA_TRY(cudaStreamSynchronize(st));
    if (n_occ < 1 || (int64_t)n_occ * 64 + 1 > 0x7fffffffLL) return AQ_E_LIMIT;  // compact keys are int32
    tb = S_->cub_bytes;
    AQ_CUDA_TRY(cub::DeviceScan::ExclusiveSum(S_->cub_tmp, tb, S_->occ_len, S_->occ_first, n_occ, st));
    int rc;
    int64_t cc = S_->occ_cap, cs = S_->occ_cap;
    if (n_occ > S_->occ_cap) {
      const int64_t want = (int64_t)n_occ + n_occ / 4 + 64;
      cc = cs = 0;
      if ((rc = grow(S_->ccount, cc, want * 64))) return rc;
      if ((rc = grow(S_->cstart, cs, want * 64 + 1))) return rc;
      S_->occ_cap = want;
    }
    AQ_CUDA_TRY(cudaMemsetAsync(S_->ccount, 0, sizeof(int32_t) * 64 * (size_t)n_occ, st));
    k_occ_keys<<<grid_for(n, 256), 256, 0, st>>>(S_->order, S_->cslot, S_->occ_first, S_->n_alloc + 1, n, S_->keys,
                                                S_->ranks, S_->ccount);
    k_cstart<<<grid_for(((int64_t)n_occ + 1) * 32, 256), 256, 0, st>>>(S_->ccount, S_->occ_first, S_->n_alloc + 1, n,
                                                                       S_->cstart);
    const int nxt = 1 - S_->cur;
    k_scatter<<<grid_for(n, SCATTER_T), SCATTER_T, 0, st>>>(
        S_->words[S_->cur], S_->pid[S_->cur], S_->words[nxt], S_->pid[nxt], S_->keys, S_->ranks, S_->cstart, n, S_->W);
    AQ_CUDA_TRY(cudaMemsetAsync(S_->n_items, 0, sizeof(int32_t) * (1 + 2 * IB), st));
    k_items_count<<<grid_for(n_occ, 256), 256, 0, st>>>(S_->cstart, n_occ, S_->n_items);
    k_items<<<grid_for(n_occ, 256), 256, 0, st>>>(S_->cstart, n_occ, S_->items, S_->n_items, S_->occ_blk);
    // the active blocks: empty the pools, then the 3^D blocks around every
    // occupied block; pools grow (dropping their contents, which the next
    // launch rebuilds from the records) when the new set may not fit
    typedef typename R4T<R>::type R4;
    const int nn = D == 3 ? 27 : 9;
    k_pool_reset<R4><<<num_sms() * 4, 256, 0, st>>>(S_->bptr, S_->pool_blk, S_->n_alloc, S_->pool_cap,
                                                    (R4*)S_->grid[0], (R4*)S_->grid[1]);
    AQ_CUDA_TRY(cudaMemsetAsync(S_->n_alloc, 0, sizeof(int32_t), st));
    const int64_t need = std::min<int64_t>((int64_t)nn * n_occ, S_->nblk);  // activated blocks, at most
    if (need > S_->pool_cap) {
      AQ_CUDA_TRY(cudaStreamSynchronize(st));
      // slack beyond the block count: slots lost to write races during the
      // interval (claim_slot) must not starve the blocks that need one
      const int64_t want =
          std::min<int64_t>(std::min<int64_t>(need + need / 4 + 256, (int64_t)S_->nblk + 256), 0x7fffffffLL);
      for (int k = 0; k < 2; ++k) {
        if (S_->grid[k]) cudaFree(S_->grid[k]);
        S_->grid[k] = nullptr;
      }
      if (S_->pool_blk) cudaFree(S_->pool_blk);
      S_->pool_blk = nullptr;
      S_->pool_cap = 0;
      for (int k = 0; k < 2; ++k) {
        const cudaError_t e = cudaMalloc(&S_->grid[k], sizeof(R4) * 64 * (size_t)want);
        if (e != cudaSuccess) {
          set_last_cuda_error(e, "cudaMalloc (sparse grid pool)");
          return AQ_E_NOMEM;
        }
        AQ_CUDA_TRY(cudaMemsetAsync(S_->grid[k], 0, sizeof(R4) * 64 * (size_t)want, st));
      }
      AQ_CUDA_TRY(cudaMalloc((void**)&S_->pool_blk, sizeof(int32_t) * (size_t)want));
      AQ_CUDA_TRY(cudaMemsetAsync(S_->pool_blk, 0xff, sizeof(int32_t) * (size_t)want, st));
      S_->pool_cap = (int)want;
    }
    for (int pass = 0; pass < 2; ++pass)
      k_activate<D><<<grid_for((int64_t)n_occ * nn, 256), 256, 0, st>>>(S_->occ_blk, S_->n_alloc + 1, K.nb[0],
                                                                         K.nb[1], K.nb[2], S_->bptr, S_->n_alloc,
                                                                         S_->pool_blk, S_->pool_cap, S_->status, pass);
    AQ_CUDA_TRY(cudaGetLastError());
    S_->cur = nxt;
    S_->launches += 10;
    S_->since_sort = 0;
    S_->sorted = true;
    return AQ_OK;
  }

  // clear = false: gout already holds this pass's sums of earlier chunks
  // (streamed mode clears it once per pass)
  int launch_step(int do_g2p, int do_p2g, void* gin, void* gout, cudaStream_t st, bool clear = true) {
    // the P2G target starts at zero (profiled as the grid pass)
    if (do_p2g && clear && (rc_ = clear_grid(gout, st))) return rc_;
    aq_sim* S_ = s;
    StepArgs a;
    memset(&a, 0, sizeof(a));
    a.words = S_->words[S_->cur];
    a.pid = S_->pid[S_->cur];
    a.items = S_->items;
    a.n_items = S_->n_items;
    // two claim counters alternate between launches; each launch zeroes the
    // one the next launch uses (both start at zero)
    a.item_ctr = S_->item_ctr + (S_->step_launches & 1);
    a.item_ctr_next = S_->item_ctr + ((S_->step_launches + 1) & 1);
    ++S_->step_launches;
    a.grid_in = gin;
    a.grid_out = gout;
    a.status = S_->status;
    a.fallbacks = S_->fallbacks;
    a.rmax = S_->rmax;
    a.rmin = S_->rmin;
    a.sk = step_key(S_->P.seed, S_->step);
    a.do_g2p = do_g2p;
    a.do_p2g = do_p2g;
    a.ranges = S_->ranges_on;
    a.raw_in = do_g2p;  // grid_in holds the previous P2G sums; grid_op runs as the tile is staged
    K.bptr = S_->bptr;
    K.n_alloc = S_->n_alloc;
    K.pool_blk = S_->pool_blk;
    K.pool_cap = S_->pool_cap;
    K.col_c = (R)cos(S_->col_theta);
    K.col_s = (R)sin(S_->col_theta);
    K.col_yshift = (int)(S_->col_height / S_->P.dx + 0.5);
    const bool prof = S_->prof_on && S_->prof_n[0] < aq_sim::PROF_CAP;
    if (prof) AQ_CUDA_TRY(cudaEventRecord(S_->prof_ev[0][2 * S_->prof_n[0]], st));
    if (S_->jit_fn) {
      void* args[] = {(void*)&S_->L, (void*)&K, (void*)&a};
      if (jit_launch(S_->jit_fn, S_->step_grid, CH, S_->step_smem, st, args) != AQ_OK) {
        set_last_cuda_error(cudaErrorLaunchFailure, "cuLaunchKernel(k_step)");
        return AQ_E_CUDA;
      }
    } else if (S_->P.sparse) {
      k_step<D, HF, HM, R, RtLayout, true, true><<<S_->step_grid, CH, S_->step_smem, st>>>(S_->L, K, a);
      AQ_CUDA_TRY(cudaGetLastError());
    } else {
      k_step<D, HF, HM, R, RtLayout><<<S_->step_grid, CH, S_->step_smem, st>>>(S_->L, K, a);
      AQ_CUDA_TRY(cudaGetLastError());
    }
    if (prof) AQ_CUDA_TRY(cudaEventRecord(S_->prof_ev[0][2 * S_->prof_n[0]++ + 1], st));
    S_->launches += 1;
    return AQ_OK;
  }

  int rc_ = 0;
  int clear_grid(void* g, cudaStream_t st) {
    const bool prof = s->prof_on && s->prof_n[1] < aq_sim::PROF_CAP;
    if (prof) AQ_CUDA_TRY(cudaEventRecord(s->prof_ev[1][2 * s->prof_n[1]], st));
    if (s->P.sparse) {
      k_pool_clear<typename R4T<R>::type><<<num_sms() * 4, 256, 0, st>>>(s->n_alloc, s->pool_cap,
                                                                        (typename R4T<R>::type*)g);
      AQ_CUDA_TRY(cudaGetLastError());
    } else {
      AQ_CUDA_TRY(cudaMemsetAsync(g, 0, sizeof(typename R4T<R>::type) * s->ncell, st));
    }
    if (prof) AQ_CUDA_TRY(cudaEventRecord(s->prof_ev[1][2 * s->prof_n[1]++ + 1], st));
    return AQ_OK;
  }

  // ------------------------------------------------ streamed (out-of-core)
  int64_t n_chunks() const { return (s->n_total + s->chunk - 1) / s->chunk; }
  int64_t chunk_count(int64_t c) const { return std::min(s->chunk, s->n_total - c * s->chunk); }
  uint64_t* chunk_words(int64_t c) const { return s->h_words + c * grouped_words(s->chunk, s->W); }

  // chunk c from host memory into the current device buffers, ids set to
  // its particles' (particle order); the loss and aq_sim_stream_get_words
  int load_chunk(int64_t c, cudaStream_t st) override {
    s->n = chunk_count(c);
    AQ_CUDA_TRY(cudaMemcpyAsync(s->words[s->cur], chunk_words(c), sizeof(uint64_t) * grouped_words(s->n, s->W),
                                cudaMemcpyHostToDevice, st));
    k_iota<<<grid_for(s->n, 256), 256, 0, st>>>(s->pid[s->cur], s->n, c * s->chunk);
    AQ_CUDA_TRY(cudaGetLastError());
    return AQ_OK;
  }

  // One pass of k_step over every chunk: upload (particle order), bin (the
  // chunk's own items), step, put back in particle order, download (not
  // after a P2G-only step, which changes no record).  The P2G target is
  // cleared once for the pass; all chunks add into it and read the same
  // complete G2P source.  Kernels run on st, uploads on up_st, downloads on
  // down_st, over four buffers: chunk c goes up into words_up[c's parity],
  // free once the binning of chunk c - 2 read it; its binning writes
  // words_binned, where it steps (after chunk c - 1 was put back in order
  // from there); it is put back in order into words_dl once chunk c - 1 has
  // come down from there.  So the uploads, the kernels and the downloads of
  // neighbouring chunks overlap, and an upload waits for no kernel of the
  // chunk before it.
  // chained: the previous pass of the same chain ran just before: uploads
  // wait only for the binnings that read their buffers and for their own
  // chunks' downloads of that pass, so the first upload overlaps that
  // pass's last kernels and download.  last: the chain ends with this pass,
  // whose downloads st then waits for (within a chain only the next
  // put-back waits for them).
  int stream_pass(int do_g2p, int do_p2g, void* gin, void* gout, cudaStream_t st, bool chained, bool last) {
    aq_sim* S_ = s;
    int rc;
    const int64_t nc = n_chunks();
    if (do_p2g && (rc = clear_grid(gout, st))) return rc;
    AQ_CUDA_TRY(cudaEventRecord(S_->ev_start, st));
    // not chained: every upload after whatever st did before this pass
    if (!chained) AQ_CUDA_TRY(cudaStreamWaitEvent(S_->up_st, S_->ev_start, 0));
    AQ_CUDA_TRY(cudaStreamWaitEvent(S_->down_st, S_->ev_start, 0));
    for (int64_t c = 0; c < nc; ++c) {
      const int par = S_->up_par;
      S_->up_par ^= 1;
      uint64_t* X = S_->words_up[par];
      const int64_t m = chunk_count(c), base = c * S_->chunk;
      AQ_CUDA_TRY(cudaStreamWaitEvent(S_->up_st, S_->ev_read[par], 0));      // the buffer is free
      AQ_CUDA_TRY(cudaStreamWaitEvent(S_->up_st, S_->ev_chunk_down[c], 0));  // the host words are final
      AQ_CUDA_TRY(cudaMemcpyAsync(X, chunk_words(c), sizeof(uint64_t) * grouped_words(m, S_->W),
                                  cudaMemcpyHostToDevice, S_->up_st));
      AQ_CUDA_TRY(cudaEventRecord(S_->ev_up, S_->up_st));
      // bin from X (ids: the chunk's particles in order) into words_binned
      S_->words[0] = X;
      S_->words[1] = S_->words_binned;
      S_->cur = 0;
      k_iota<<<grid_for(m, 256), 256, 0, st>>>(S_->pid[0], m, base);
      AQ_CUDA_TRY(cudaGetLastError());
      S_->launches += 1;
      AQ_CUDA_TRY(cudaStreamWaitEvent(st, S_->ev_up, 0));
      S_->n = m;
      if ((rc = sort(st))) return rc;  // words[0] -> words[1], cur = 1
      AQ_CUDA_TRY(cudaEventRecord(S_->ev_read[par], st));
      if ((rc = launch_step(do_g2p, do_p2g, gin, gout, st, false))) return rc;
      if (!do_g2p) continue;  // a P2G-only pass leaves the records as they are: nothing to take down
      AQ_CUDA_TRY(cudaStreamWaitEvent(st, S_->ev_down, 0));  // words_dl may still be going down
      k_words_unpermute<<<grid_for(m, 256), 256, 0, st>>>(S_->words[S_->cur], S_->pid[S_->cur], S_->words_dl, m,
                                                          S_->W, base);
      AQ_CUDA_TRY(cudaGetLastError());
      S_->launches += 1;
      AQ_CUDA_TRY(cudaEventRecord(S_->ev_ready, st));
      AQ_CUDA_TRY(cudaStreamWaitEvent(S_->down_st, S_->ev_ready, 0));
      AQ_CUDA_TRY(cudaMemcpyAsync(chunk_words(c), S_->words_dl, sizeof(uint64_t) * grouped_words(m, S_->W),
                                  cudaMemcpyDeviceToHost, S_->down_st));
      AQ_CUDA_TRY(cudaEventRecord(S_->ev_down, S_->down_st));
      AQ_CUDA_TRY(cudaEventRecord(S_->ev_chunk_down[c], S_->down_st));
    }
    if (last) AQ_CUDA_TRY(cudaStreamWaitEvent(st, S_->ev_down, 0));  // the host store is complete when st gets here
    return AQ_OK;
  }

  // The fused chain of substeps() over streamed chunks: a P2G pass, one
  // fused pass per substep, a final G2P pass (n + 1 passes for n substeps);
  // each chunk is re-binned on every pass, which costs little beside the
  // host transfers that bound this mode.
  int stream_substeps(int n, cudaStream_t st) {
    aq_sim* S_ = s;
    int rc, a = 0;
    if ((rc = stream_pass(0, 1, nullptr, S_->grid[a], st, false, false))) return rc;
    for (int k = 0; k < n; ++k) {
      const int b = 1 - a;
      if (k + 1 < n) {
        if ((rc = stream_pass(1, 1, S_->grid[a], S_->grid[b], st, true, false))) return rc;
        a = b;
      } else {
        if ((rc = stream_pass(1, 0, S_->grid[a], nullptr, st, true, true))) return rc;
        S_->last_grid = a;
      }
      ++S_->step;
      S_->col_theta += S_->col_omega * S_->P.dt;
      S_->col_height += S_->col_rate * S_->P.dt;
    }
    return AQ_OK;
  }

  int substeps(int n, cudaStream_t st) override {
    aq_sim* S_ = s;
    if (S_->chunk) return stream_substeps(n, st);
    const int interval = S_->P.sort_interval < 1 ? 1 : S_->P.sort_interval;
    int rc;
    while (n > 0) {
      if (!S_->sorted || S_->since_sort >= interval) {
        if ((rc = sort(st))) return rc;
      }
      int m = interval - S_->since_sort;
      if (m > n) m = n;
      // P2G of the first substep, then per substep one fused launch: grid_op
      // applied while staging the tile, G2P, P2G of the next substep into
      // the other (cleared) grid
      int a = 0;
      if ((rc = launch_step(0, 1, nullptr, S_->grid[a], st))) return rc;
      for (int k = 0; k < m; ++k) {
        const int b = 1 - a;
        if (k + 1 < m) {
          if ((rc = launch_step(1, 1, S_->grid[a], S_->grid[b], st))) return rc;
          a = b;
        } else {
          if ((rc = launch_step(1, 0, S_->grid[a], nullptr, st))) return rc;
          S_->last_grid = a;
        }
        ++S_->step;
        // step_collider (mpm_solver.py:1542-1547) after every substep
        S_->col_theta += S_->col_omega * S_->P.dt;
        S_->col_height += S_->col_rate * S_->P.dt;
      }
      S_->since_sort += m;
      n -= m;
    }
    return AQ_OK;
  }

  int loss(double* h, cudaStream_t st) override {
    AQ_CUDA_TRY(cudaMemsetAsync(s->dloss, 0, sizeof(double), st));
    if (s->chunk) {  // streamed: the sum over every chunk
      for (int64_t c = 0; c < n_chunks(); ++c) {
        int rc;
        if ((rc = load_chunk(c, st))) return rc;
        k_loss<D, R><<<num_sms() * 4, 256, 0, st>>>(s->L, K, s->words[s->cur], s->n, s->dloss);
        AQ_CUDA_TRY(cudaGetLastError());
      }
    } else {
      k_loss<D, R><<<num_sms() * 4, 256, 0, st>>>(s->L, K, s->words[s->cur], s->n, s->dloss);
      AQ_CUDA_TRY(cudaGetLastError());
    }
    AQ_CUDA_TRY(cudaMemcpyAsync(h, s->dloss, sizeof(double), cudaMemcpyDeviceToHost, st));
    AQ_CUDA_TRY(cudaStreamSynchronize(st));
    return AQ_OK;
  }
};

// Compile (NVRTC, layout as a constant; with or without the collider) or
// select the library's own k_step, and size its persistent grid.
template <int D, bool HF, bool HM, class R>
static int setup_step_kernel(aq_sim* s, size_t smem_jit, size_t smem_aot, bool col) {
  int occ = 0;
  s->jit_fn = nullptr;
  if (s->P.jit) {
    const size_t smem = smem_jit;
    s->jit_fn = jit_k_step(D, HF, HM, sizeof(R) == 8, col, s->P.sparse != 0, s->L, &s->jit_error);
    if (s->jit_fn && (jit_set_smem(s->jit_fn, (int)smem) != AQ_OK || jit_occupancy(s->jit_fn, CH, smem, &occ) != AQ_OK)) {
      s->jit_fn = nullptr;
      s->jit_error = "cuFuncSetAttribute/occupancy failed";
    }
    s->step_smem = smem;
  }
  if (!s->jit_fn) {
    const size_t smem = smem_aot;
    s->step_smem = smem;
    if (s->P.sparse) {
      AQ_CUDA_TRY(cudaFuncSetAttribute(k_step<D, HF, HM, R, RtLayout, true, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      AQ_CUDA_TRY(
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_step<D, HF, HM, R, RtLayout, true, true>, CH, smem));
    } else {
      AQ_CUDA_TRY(cudaFuncSetAttribute(k_step<D, HF, HM, R, RtLayout>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
      AQ_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_step<D, HF, HM, R, RtLayout>, CH, smem));
    }
  }
  if (occ < 1) occ = 1;
  s->step_grid = occ * num_sms();
  return AQ_OK;
}

template <int D, bool HF, bool HM, class R>
static int make_impl(aq_sim* s) {
  auto* im = new (std::nothrow) SimImpl<D, HF, HM, R>(s);
  if (!im) return AQ_E_NOMEM;
  s->impl = im;
  const size_t smem = im->smem_bytes(false);
  if (smem > 227 * 1024) return AQ_E_LIMIT;
  return setup_step_kernel<D, HF, HM, R>(s, im->smem_bytes(jit_reg_record(s->L)), smem, false);
}

template <int D, class R>
static int make_impl_d(aq_sim* s) {
  const bool hf = s->P.has_F != 0, hm = s->P.has_mat != 0;
  if (hf && hm) return make_impl<D, true, true, R>(s);
  if (hf) return make_impl<D, true, false, R>(s);
  if (hm) return make_impl<D, false, true, R>(s);
  return make_impl<D, false, false, R>(s);
}

static void free_sim(aq_sim* s) {
  if (!s) return;
  delete s->impl;
  for (int k = 0; k < 2; ++k) {
    if (s->prof_ev[k]) {
      for (int j = 0; j < 2 * aq_sim::PROF_CAP; ++j) cudaEventDestroy(s->prof_ev[k][j]);
      delete[] s->prof_ev[k];
    }
  }
  if (s->P.sparse) {
    for (int k = 0; k < 2; ++k)
      if (s->grid[k]) cudaFree(s->grid[k]);
    if (s->pool_blk) cudaFree(s->pool_blk);
    if (s->ccount) cudaFree(s->ccount);
    if (s->cstart) cudaFree(s->cstart);
    if (s->cub_tmp) cudaFree(s->cub_tmp);
  }
  if (s->slab) cudaFree(s->slab);
  if (s->h_words) cudaFreeHost(s->h_words);
  if (s->words_dl) cudaFree(s->words_dl);
  if (s->words_up[1]) cudaFree(s->words_up[1]);
  for (cudaEvent_t ev : {s->ev_start, s->ev_up, s->ev_read[0], s->ev_read[1], s->ev_ready, s->ev_down})
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : s->ev_chunk_down)
    if (ev) cudaEventDestroy(ev);
  if (s->up_st) cudaStreamDestroy(s->up_st);
  if (s->down_st) cudaStreamDestroy(s->down_st);
  delete s;
}

}  // namespace aq

using namespace aq;

extern "C" {

int aq_sim_create(const aq_params* P, const aq_layout* L, aq_sim** out) {
  if (!P || !L || !out) return AQ_E_ARG;
  *out = nullptr;
  const int D = P->dim;
  if (D != 2 && D != 3) return AQ_E_ARG;
  if (P->precision != 0 && P->precision != 1) return AQ_E_ARG;
  if (P->n_particles < 1 || P->n_particles > 0x7fffffffLL) return AQ_E_ARG;
  for (int d = 0; d < D; ++d)
    if (P->res[d] < 3 || P->res[d] > 8192) return AQ_E_ARG;
  if (!(P->dx > 0) || !(P->dt > 0)) return AQ_E_ARG;
  const int ns = 2 * D + D * D + (P->has_F ? D * D : 1) + (P->has_mat ? 1 : 0);
  if (L->n_slots != ns) return AQ_E_LAYOUT;
  if (P->n_materials < 0 || P->n_materials > AQ_MAX_MATERIALS) return AQ_E_ARG;
  for (int m = 0; m < (P->n_materials ? P->n_materials : 1); ++m) {
    const int k = P->mat[m].kind;
    if (k != AQ_MAT_FLUID && k != AQ_MAT_ELASTIC && k != AQ_MAT_COROTATED) return AQ_E_ARG;
    if (!P->has_F && k != AQ_MAT_FLUID) return AQ_E_LAYOUT;
  }

  aq_sim* s = new (std::nothrow) aq_sim();
  if (!s) return AQ_E_NOMEM;
  s->P = *P;
  s->L = *L;
  s->D = D;
  s->W = L->n_words;
  s->WS = L->n_words | 1;  // odd shared-memory stride: conflict-free 8-byte accesses
  s->NS = ns;
  s->n = P->n_particles;
  s->cap = P->n_particles;
  int nb[3] = {1, 1, 1};
  const int BS = D == 3 ? 4 : 8;
  s->ncell = 1;
  for (int d = 0; d < D; ++d) {
    nb[d] = (P->res[d] + BS - 1) / BS;
    s->ncell *= P->res[d];
  }
  const int64_t nblk64 = (int64_t)nb[0] * nb[1] * nb[2];
  if (P->sparse && nblk64 > 0x7fffffffLL) {
    delete s;
    return AQ_E_LIMIT;  // block indices of a sparse grid are int32
  }
  if (!P->sparse && nblk64 * 64 > 0x7fffffffLL) {
    delete s;
    return AQ_E_LIMIT;  // the dense binning's cell keys are int32
  }
  s->nblk = (int)nblk64;
  s->nkeys = P->sparse ? 0 : (int64_t)s->nblk * 64;
  s->max_items = P->sparse ? std::min<int64_t>(s->nblk, P->n_particles) + 1 : (int64_t)s->nblk + 1;
  const size_t rsz = P->precision ? sizeof(double) : sizeof(float);
  const int64_t n = s->n;
  const int nt = (int)((s->nkeys + SCAN_TILE - 1) / SCAN_TILE);
  cudaError_t e = cudaSuccess;
  // every buffer is carved from one device allocation (one cudaMalloc per
  // simulator, one cudaFree at destroy), each on a 256-byte boundary
  struct Part {
    void** p;
    size_t off;
  };
  Part parts[40];
  int nparts = 0;
  size_t total = 0;
  bool too_many = false;
  auto alloc = [&](void** p, size_t bytes) {
    if (nparts >= (int)(sizeof(parts) / sizeof(parts[0]))) {  // reported below
      too_many = true;
      return;
    }
    parts[nparts++] = Part{p, total};
    total += (bytes + 255) & ~(size_t)255;
  };
  alloc((void**)&s->words[0], sizeof(uint64_t) * (grouped_words(n, s->W) + 2));
  alloc((void**)&s->words[1], sizeof(uint64_t) * (grouped_words(n, s->W) + 2));
  alloc((void**)&s->pid[0], sizeof(int32_t) * n);
  alloc((void**)&s->pid[1], sizeof(int32_t) * n);
  alloc((void**)&s->keys, sizeof(int32_t) * n);
  alloc((void**)&s->ranks, sizeof(int32_t) * n);
  if (P->sparse) {  // block table and sparse binning; the pools are sized at the first binning
    alloc((void**)&s->bptr, sizeof(int32_t) * (size_t)s->nblk);
    alloc((void**)&s->n_alloc, 2 * sizeof(int32_t));
    alloc((void**)&s->sblk, sizeof(uint32_t) * n);
    alloc((void**)&s->sblk_sorted, sizeof(uint32_t) * n);
    alloc((void**)&s->order_in, sizeof(int32_t) * n);
    alloc((void**)&s->order, sizeof(int32_t) * n);
    alloc((void**)&s->cslot, sizeof(int32_t) * n);
    alloc((void**)&s->occ_blk, sizeof(int32_t) * n);
    alloc((void**)&s->occ_len, sizeof(int32_t) * n);
    alloc((void**)&s->occ_first, sizeof(int32_t) * n);
  } else {
    alloc(&s->grid[0], rsz * 4 * s->ncell);
    alloc(&s->grid[1], rsz * 4 * s->ncell);
    alloc((void**)&s->cell_count, sizeof(int32_t) * s->nkeys);
    alloc((void**)&s->cell_start, sizeof(int32_t) * (s->nkeys + 1));
    alloc((void**)&s->scan_sums, sizeof(int32_t) * (nt + 1));
  }
  alloc((void**)&s->items, sizeof(int4) * s->max_items);
  alloc((void**)&s->n_items, sizeof(int32_t) * (1 + 2 * IB));
  alloc((void**)&s->item_ctr, 2 * sizeof(int32_t));
  alloc((void**)&s->status, sizeof(unsigned));
  alloc((void**)&s->fallbacks, sizeof(unsigned long long));
  alloc((void**)&s->rmax, sizeof(double) * AQ_MAX_SLOTS);
  alloc((void**)&s->rmin, sizeof(double) * AQ_MAX_SLOTS);
  alloc((void**)&s->dloss, sizeof(double));
  alloc((void**)&s->dstats, sizeof(double) * 5 * AQ_MAX_SLOTS);
  if (too_many) {  // a buffer was left out: the list above outgrew parts
    free_sim(s);
    return AQ_E_LIMIT;
  }
  e = cudaMalloc(&s->slab, total);
  if (e == cudaSuccess)
    for (int k = 0; k < nparts; ++k) *parts[k].p = static_cast<char*>(s->slab) + parts[k].off;
  if (e != cudaSuccess) {
    s->slab = nullptr;
    set_last_cuda_error(e, "cudaMalloc");
    free_sim(s);
    return AQ_E_NOMEM;
  }
  if (P->sparse) {
    e = cudaMemset(s->bptr, 0xff, sizeof(int32_t) * (size_t)s->nblk);
    if (e == cudaSuccess) e = cudaMemset(s->n_alloc, 0, 2 * sizeof(int32_t));
    // scratch of the radix sort, run-length encoding and scan over n records
    size_t b1 = 0, b2 = 0, b3 = 0;
    while (s->blk_bits < 31 && (int64_t(1) << s->blk_bits) < s->nblk) ++s->blk_bits;
    if (e == cudaSuccess)
      e = cub::DeviceRadixSort::SortPairs(nullptr, b1, s->sblk, s->sblk_sorted, s->order_in, s->order, (int)n, 0,
                                          s->blk_bits);
    if (e == cudaSuccess)
      e = cub::DeviceRunLengthEncode::Encode(nullptr, b2, s->sblk_sorted, reinterpret_cast<uint32_t*>(s->occ_blk),
                                             s->occ_len, s->n_alloc + 1, (int)n);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, b3, s->occ_len, s->occ_first, (int)n);
    s->cub_bytes = std::max(std::max(b1, b2), std::max(b3, (size_t)256));
    if (e == cudaSuccess) e = cudaMalloc(&s->cub_tmp, s->cub_bytes);
  } else {
    e = cudaMemset(s->grid[0], 0, rsz * 4 * s->ncell);
    if (e == cudaSuccess) e = cudaMemset(s->grid[1], 0, rsz * 4 * s->ncell);
  }
  if (e == cudaSuccess) e = cudaMemset(s->words[0], 0, sizeof(uint64_t) * (grouped_words(n, s->W) + 2));
  if (e == cudaSuccess) e = cudaMemset(s->status, 0, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(s->fallbacks, 0, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(s->item_ctr, 0, 2 * sizeof(int32_t));
  if (e != cudaSuccess) {
    set_last_cuda_error(e, "cudaMemset");
    free_sim(s);
    return AQ_E_CUDA;
  }
  k_iota<<<grid_for(n, 256), 256>>>(s->pid[0], n);
  int rc;
  if (D == 3)
    rc = P->precision ? make_impl_d<3, double>(s) : make_impl_d<3, float>(s);
  else
    rc = P->precision ? make_impl_d<2, double>(s) : make_impl_d<2, float>(s);
  if (rc == AQ_OK) {
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      set_last_cuda_error(e, "aq_sim_create");
      rc = AQ_E_CUDA;
    }
  }
  if (rc != AQ_OK) {
    free_sim(s);
    return rc;
  }
  *out = s;
  return AQ_OK;
}

int aq_sim_create_streamed(const aq_params* P, const aq_layout* L, int64_t chunk, aq_sim** out) {
  if (!P || !L || !out || chunk < 1) return AQ_E_ARG;
  *out = nullptr;
  if (P->sparse) return AQ_E_ARG;  // streamed chunks bin on a dense grid
  const int64_t n_total = P->n_particles;
  if (n_total < 1 || n_total > 0x7fffffffLL) return AQ_E_ARG;
  if (chunk > n_total) chunk = n_total;
  aq_params Q = *P;
  Q.n_particles = chunk;  // the device buffers hold one chunk
  aq_sim* s = nullptr;
  int rc = aq_sim_create(&Q, L, &s);
  if (rc != AQ_OK) return rc;
  const int64_t nc = (n_total + chunk - 1) / chunk;
  const size_t wbytes = sizeof(uint64_t) * (size_t)(nc * grouped_words(chunk, s->W));
  cudaError_t e = cudaMallocHost((void**)&s->h_words, wbytes);
  if (e != cudaSuccess) {
    set_last_cuda_error(e, "cudaMallocHost");
    free_sim(s);
    return AQ_E_NOMEM;
  }
  e = cudaMalloc((void**)&s->words_dl, sizeof(uint64_t) * (size_t)(grouped_words(chunk, s->W) + 2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&s->words_up[1], sizeof(uint64_t) * (size_t)(grouped_words(chunk, s->W) + 2));
  if (e != cudaSuccess) {
    set_last_cuda_error(e, "cudaMalloc");
    free_sim(s);
    return AQ_E_NOMEM;
  }
  s->words_up[0] = s->words[0];
  s->words_binned = s->words[1];
  e = cudaStreamCreateWithFlags(&s->up_st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->down_st, cudaStreamNonBlocking);
  for (cudaEvent_t* ev : {&s->ev_start, &s->ev_up, &s->ev_read[0], &s->ev_read[1], &s->ev_ready, &s->ev_down})
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  s->ev_chunk_down.assign((size_t)nc, nullptr);
  for (int64_t c = 0; c < nc && e == cudaSuccess; ++c)
    e = cudaEventCreateWithFlags(&s->ev_chunk_down[c], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    set_last_cuda_error(e, "cudaStreamCreate/cudaEventCreate");
    free_sim(s);
    return AQ_E_CUDA;
  }
  memset(s->h_words, 0, wbytes);
  s->chunk = chunk;
  s->n_total = n_total;
  *out = s;
  return AQ_OK;
}

int aq_sim_stream_set_words(aq_sim* s, const uint64_t* h_words, void* stream) {
  if (!s || !h_words) return AQ_E_ARG;
  if (!s->chunk) return AQ_E_STATE;
  cudaStream_t st = as_stream(stream);
  AQ_CUDA_TRY(cudaStreamSynchronize(st));  // no pass still reads or writes the host store
  const int64_t nc = (s->n_total + s->chunk - 1) / s->chunk;
  uint64_t* tmp = s->words[1 - s->cur];
  for (int64_t c = 0; c < nc; ++c) {
    const int64_t base = c * s->chunk, m = std::min(s->chunk, s->n_total - base);
    AQ_CUDA_TRY(cudaMemcpyAsync(tmp, h_words + base * s->W, sizeof(uint64_t) * m * s->W, cudaMemcpyHostToDevice, st));
    k_words_group<<<grid_for(m, 256), 256, 0, st>>>(tmp, s->words[s->cur], m, s->W);
    AQ_CUDA_TRY(cudaGetLastError());
    AQ_CUDA_TRY(cudaMemcpyAsync(s->h_words + c * grouped_words(s->chunk, s->W), s->words[s->cur],
                                sizeof(uint64_t) * grouped_words(m, s->W), cudaMemcpyDeviceToHost, st));
    s->launches += 1;
  }
  AQ_CUDA_TRY(cudaStreamSynchronize(st));
  s->sorted = false;
  return AQ_OK;
}

int aq_sim_stream_get_words(aq_sim* s, uint64_t* h_words, void* stream) {
  if (!s || !h_words) return AQ_E_ARG;
  if (!s->chunk) return AQ_E_STATE;
  cudaStream_t st = as_stream(stream);
  const int64_t nc = (s->n_total + s->chunk - 1) / s->chunk;
  uint64_t* tmp = s->words[1 - s->cur];
  for (int64_t c = 0; c < nc; ++c) {
    const int64_t base = c * s->chunk, m = std::min(s->chunk, s->n_total - base);
    int rc;
    if ((rc = s->impl->load_chunk(c, st))) return rc;  // particle order, ids base, base + 1, ...
    k_words_ungroup<<<grid_for(m, 256), 256, 0, st>>>(s->words[s->cur], s->pid[s->cur], tmp, m, s->W, base);
    AQ_CUDA_TRY(cudaGetLastError());
    AQ_CUDA_TRY(cudaMemcpyAsync(h_words + base * s->W, tmp, sizeof(uint64_t) * m * s->W, cudaMemcpyDeviceToHost, st));
    s->launches += 1;
  }
  AQ_CUDA_TRY(cudaStreamSynchronize(st));
  return AQ_OK;
}

int aq_sim_set_count(aq_sim* s, int64_t n) {
  if (!s) return AQ_E_ARG;
  if (s->chunk) return AQ_E_STATE;
  if (n < 1 || n > s->cap) return AQ_E_ARG;
  s->n = n;
  s->sorted = false;
  return AQ_OK;
}

int aq_sim_append(aq_sim* s, const void* values, int32_t values_f64, int64_t count, void* stream) {
  if (!s || !values || count < 1) return AQ_E_ARG;
  if (s->chunk) return AQ_E_STATE;
  if (count > s->cap - s->n) return AQ_E_LIMIT;
  cudaStream_t st = as_stream(stream);
  const int64_t base = s->n;
  int32_t* ids = s->pid[s->cur] + base;
  k_iota<<<grid_for(count, 256), 256, 0, st>>>(ids, count, base);
  AQ_CUDA_TRY(cudaGetLastError());
  // contiguous records into the other buffer (scratch between binnings),
  // then grouped behind the stored ones
  uint64_t* tmp = s->words[1 - s->cur];
  int rc = aq_encode(&s->L, values, values_f64, tmp, count, ids, s->P.seed, -1, nullptr, stream);
  if (rc != AQ_OK) return rc;
  k_words_group<<<grid_for(count, 256), 256, 0, st>>>(tmp, s->words[s->cur], count, s->W, base);
  AQ_CUDA_TRY(cudaGetLastError());
  s->n = base + count;
  s->sorted = false;
  s->launches += 3;
  return AQ_OK;
}

int aq_sim_count(const aq_sim* s, int64_t* h_n, int64_t* h_cap) {
  if (!s || !h_n || !h_cap) return AQ_E_ARG;
  *h_n = s->chunk ? s->n_total : s->n;
  *h_cap = s->chunk ? s->n_total : s->cap;
  return AQ_OK;
}

int aq_sim_stream_chunks(const aq_sim* s, int64_t* h_chunk, int64_t* h_n_total) {
  if (!s || !h_chunk || !h_n_total) return AQ_E_ARG;
  *h_chunk = s->chunk;
  *h_n_total = s->chunk ? s->n_total : s->n;
  return AQ_OK;
}

int aq_sim_destroy(aq_sim* s) {
  if (!s) return AQ_E_ARG;
  cudaDeviceSynchronize();
  free_sim(s);
  return AQ_OK;
}

int aq_sim_set_state(aq_sim* s, const void* values, int32_t values_f64, void* stream) {
  if (!s || !values) return AQ_E_ARG;
  if (s->chunk) return AQ_E_STATE;  // streamed: the state is in host memory
  cudaStream_t st = as_stream(stream);
  k_iota<<<grid_for(s->n, 256), 256, 0, st>>>(s->pid[s->cur], s->n);
  AQ_CUDA_TRY(cudaGetLastError());
  // contiguous records into the other buffer, then grouped into the current
  uint64_t* tmp = s->words[1 - s->cur];
  int rc = aq_encode(&s->L, values, values_f64, tmp, s->n, nullptr, s->P.seed, -1, nullptr, stream);
  if (rc != AQ_OK) return rc;
  k_words_group<<<grid_for(s->n, 256), 256, 0, st>>>(tmp, s->words[s->cur], s->n, s->W);
  AQ_CUDA_TRY(cudaGetLastError());
  s->sorted = false;
  s->launches += 3;
  return AQ_OK;
}

int aq_sim_get_state(aq_sim* s, void* values, int32_t values_f64, void* stream) {
  if (!s || !values) return AQ_E_ARG;
  if (s->chunk) return AQ_E_STATE;  // streamed: the state is in host memory
  cudaStream_t st = as_stream(stream);
  if (values_f64)
    k_get_state<double><<<grid_for(s->n, 128), 128, 0, st>>>(s->L, s->words[s->cur], s->pid[s->cur], (double*)values,
                                                             s->n);
  else
    k_get_state<float><<<grid_for(s->n, 128), 128, 0, st>>>(s->L, s->words[s->cur], s->pid[s->cur], (float*)values,
                                                            s->n);
  AQ_CUDA_TRY(cudaGetLastError());
  s->launches += 1;
  return AQ_OK;
}

int aq_sim_set_collider(aq_sim* s, const float* d_sdf, const float* d_normal, const int32_t* dims,
                        const int32_t* offset, int32_t center, double theta, double height, double omega,
                        double height_rate) {
  if (!s) return AQ_E_ARG;
  if (!d_sdf) {
    s->col_on = 0;
  } else {
    if (s->D != 3 || !d_normal || !dims || !offset) return AQ_E_ARG;
    for (int k = 0; k < 3; ++k)
      if (dims[k] < 1) return AQ_E_ARG;
    s->col_on = 1;
    s->col_center = center;
    s->col_sdf = d_sdf;
    s->col_nrm = d_normal;
    for (int k = 0; k < 3; ++k) {
      s->col_dims[k] = dims[k];
      s->col_off[k] = offset[k];
    }
  }
  s->col_theta = theta;
  s->col_height = height;
  s->col_omega = omega;
  s->col_rate = height_rate;
  s->impl->set_collider(s);
  // the layout-specialized kernel is built with the collider only when one is set
  if (s->P.jit) return s->impl->setup_kernel(s->col_on != 0);
  return AQ_OK;
}

int aq_sim_collider_pose(aq_sim* s, double theta, double height) {
  if (!s) return AQ_E_ARG;
  s->col_theta = theta;
  s->col_height = height;
  return AQ_OK;
}

int aq_sim_collider_velocity_mode(aq_sim* s, int32_t from_node) {
  if (!s || (from_node != 0 && from_node != 1)) return AQ_E_ARG;
  s->col_node_cv = from_node;
  s->impl->set_collider(s);
  return AQ_OK;
}

int aq_sim_sparse_blocks(aq_sim* s, int64_t* h_slots, int64_t* h_occupied, void* stream) {
  if (!s || !h_slots || !h_occupied) return AQ_E_ARG;
  if (!s->P.sparse) return AQ_E_STATE;
  cudaStream_t st = as_stream(stream);
  int32_t v[2] = {0, 0};
  AQ_CUDA_TRY(cudaMemcpyAsync(v, s->n_alloc, sizeof(v), cudaMemcpyDeviceToHost, st));
  AQ_CUDA_TRY(cudaStreamSynchronize(st));
  *h_slots = std::min<int64_t>(v[0], s->pool_cap);
  *h_occupied = v[1];
  return AQ_OK;
}

int aq_sim_collider_get(aq_sim* s, double* h_theta, double* h_height) {
  if (!s || !h_theta || !h_height) return AQ_E_ARG;
  *h_theta = s->col_theta;
  *h_height = s->col_height;
  return AQ_OK;
}

int aq_sim_field_stats(aq_sim* s, const void* ref, int32_t ref_f64, double* h_out, void* stream) {
  if (!s || !h_out) return AQ_E_ARG;
  if (s->chunk) return AQ_E_STATE;  // streamed: the state is in host memory
  cudaStream_t st = as_stream(stream);
  AQ_CUDA_TRY(cudaMemsetAsync(s->dstats, 0, sizeof(double) * 5 * AQ_MAX_SLOTS, st));
  const unsigned nb = (unsigned)std::min<int64_t>(grid_for(s->n, 256), (int64_t)num_sms() * 4);
  const dim3 grid(nb > 0 ? nb : 1, s->NS);
  if (ref_f64)
    k_field_stats<double><<<grid, 256, 0, st>>>(s->L, s->words[s->cur], s->pid[s->cur], (const double*)ref, s->n,
                                                s->dstats);
  else
    k_field_stats<float><<<grid, 256, 0, st>>>(s->L, s->words[s->cur], s->pid[s->cur], (const float*)ref, s->n,
                                               s->dstats);
  AQ_CUDA_TRY(cudaGetLastError());
  s->launches += 1;
  AQ_CUDA_TRY(cudaMemcpyAsync(h_out, s->dstats, sizeof(double) * 5 * s->NS, cudaMemcpyDeviceToHost, st));
  AQ_CUDA_TRY(cudaStreamSynchronize(st));
  return AQ_OK;
}

int aq_sim_set_words(aq_sim* s, const uint64_t* words, void* stream) {
  if (!s || !words) return AQ_E_ARG;
  if (s->chunk) return AQ_E_STATE;  // streamed: the state is in host memory
  cudaStream_t st = as_stream(stream);
  k_iota<<<grid_for(s->n, 256), 256, 0, st>>>(s->pid[s->cur], s->n);
  k_words_group<<<grid_for(s->n, 256), 256, 0, st>>>(words, s->words[s->cur], s->n, s->W);
  AQ_CUDA_TRY(cudaGetLastError());
  s->sorted = false;
  s->launches += 2;
  return AQ_OK;
}

int aq_sim_get_words(aq_sim* s, uint64_t* words, void* stream) {
  if (!s || !words) return AQ_E_ARG;
  if (s->chunk) return AQ_E_STATE;  // streamed: the state is in host memory
  cudaStream_t st = as_stream(stream);
  k_words_ungroup<<<grid_for(s->n, 256), 256, 0, st>>>(s->words[s->cur], s->pid[s->cur], words, s->n, s->W);
  AQ_CUDA_TRY(cudaGetLastError());
  s->launches += 1;
  return AQ_OK;
}

int aq_sim_substeps(aq_sim* s, int32_t n, void* stream) {
  if (!s || n < 0) return AQ_E_ARG;
  if (n == 0) return AQ_OK;
  return s->impl->substeps(n, as_stream(stream));
}

int aq_sim_grid_mass(aq_sim* s, float* d_out, void* stream) {
  if (!s || !d_out) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  const unsigned nb = (unsigned)std::min<int64_t>(grid_for(s->ncell, 256), (int64_t)num_sms() * 8);
  if (s->P.sparse) {
    const int r0 = s->P.res[0], r1 = s->P.res[1], r2 = s->D == 3 ? s->P.res[2] : 1;
    const int bs = s->D == 3 ? 4 : 8;
    const int nb1 = (r1 + bs - 1) / bs, nb2 = s->D == 3 ? (r2 + bs - 1) / bs : 1;
    const void* g = s->grid[s->last_grid];
    if (!g) return AQ_E_STATE;  // no substep has run yet
    if (s->D == 3 && s->P.precision)
      k_grid_mass_sparse<3><<<nb, 256, 0, st>>>((const double4*)g, s->bptr, r0, r1, r2, nb1, nb2, d_out, s->ncell);
    else if (s->D == 3)
      k_grid_mass_sparse<3><<<nb, 256, 0, st>>>((const float4*)g, s->bptr, r0, r1, r2, nb1, nb2, d_out, s->ncell);
    else if (s->P.precision)
      k_grid_mass_sparse<2><<<nb, 256, 0, st>>>((const double4*)g, s->bptr, r0, r1, r2, nb1, nb2, d_out, s->ncell);
    else
      k_grid_mass_sparse<2><<<nb, 256, 0, st>>>((const float4*)g, s->bptr, r0, r1, r2, nb1, nb2, d_out, s->ncell);
    AQ_CUDA_TRY(cudaGetLastError());
    s->launches += 1;
    return AQ_OK;
  }
  if (s->P.precision)
    k_grid_mass<<<nb, 256, 0, st>>>((const double4*)s->grid[s->last_grid], d_out, s->ncell);
  else
    k_grid_mass<<<nb, 256, 0, st>>>((const float4*)s->grid[s->last_grid], d_out, s->ncell);
  AQ_CUDA_TRY(cudaGetLastError());
  s->launches += 1;
  return AQ_OK;
}

int aq_sim_loss(aq_sim* s, int32_t kind, double* h_out, void* stream) {
  if (!s || !h_out || kind != 0) return AQ_E_ARG;
  s->launches += 1;
  return s->impl->loss(h_out, as_stream(stream));
}

int aq_sim_ranges_enable(aq_sim* s, int32_t on, void* stream) {
  if (!s) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  if (on) {
    double mx[AQ_MAX_SLOTS], mn[AQ_MAX_SLOTS];
    for (int k = 0; k < AQ_MAX_SLOTS; ++k) {
      mx[k] = -INFINITY;
      mn[k] = INFINITY;
    }
    AQ_CUDA_TRY(cudaMemcpyAsync(s->rmax, mx, sizeof(mx), cudaMemcpyHostToDevice, st));
    AQ_CUDA_TRY(cudaMemcpyAsync(s->rmin, mn, sizeof(mn), cudaMemcpyHostToDevice, st));
    AQ_CUDA_TRY(cudaStreamSynchronize(st));
  }
  s->ranges_on = on ? 1 : 0;
  return AQ_OK;
}

int aq_sim_ranges_get(aq_sim* s, double* h_max, double* h_min, void* stream) {
  if (!s || !h_max || !h_min) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  AQ_CUDA_TRY(cudaMemcpyAsync(h_max, s->rmax, sizeof(double) * s->NS, cudaMemcpyDeviceToHost, st));
  AQ_CUDA_TRY(cudaMemcpyAsync(h_min, s->rmin, sizeof(double) * s->NS, cudaMemcpyDeviceToHost, st));
  AQ_CUDA_TRY(cudaStreamSynchronize(st));
  return AQ_OK;
}

int aq_sim_status(aq_sim* s, uint32_t* h_flags, int64_t* h_fallbacks, int32_t clear, void* stream) {
  if (!s) return AQ_E_ARG;
  cudaStream_t st = as_stream(stream);
  unsigned f = 0;
  unsigned long long fb = 0;
  AQ_CUDA_TRY(cudaMemcpyAsync(&f, s->status, sizeof(f), cudaMemcpyDeviceToHost, st));
  AQ_CUDA_TRY(cudaMemcpyAsync(&fb, s->fallbacks, sizeof(fb), cudaMemcpyDeviceToHost, st));
  if (clear) {
    AQ_CUDA_TRY(cudaMemsetAsync(s->status, 0, sizeof(unsigned), st));
    AQ_CUDA_TRY(cudaMemsetAsync(s->fallbacks, 0, sizeof(unsigned long long), st));
  }
  AQ_CUDA_TRY(cudaStreamSynchronize(st));
  if (h_flags) *h_flags = f;
  if (h_fallbacks) *h_fallbacks = (int64_t)fb;
  return AQ_OK;
}

int aq_sim_step_count(const aq_sim* s, int64_t* h_out) {
  if (!s || !h_out) return AQ_E_ARG;
  *h_out = s->step;
  return AQ_OK;
}

int aq_sim_set_step_count(aq_sim* s, int64_t step) {
  if (!s || step < 0) return AQ_E_ARG;
  s->step = step;
  return AQ_OK;
}

int aq_sim_kernel_is_jit(const aq_sim* s, int32_t* h_out) {
  if (!s || !h_out) return AQ_E_ARG;
  *h_out = s->jit_fn ? 1 : 0;
  return AQ_OK;
}

int aq_sim_launches(const aq_sim* s, int64_t* h_out) {
  if (!s || !h_out) return AQ_E_ARG;
  *h_out = s->launches;
  return AQ_OK;
}

int aq_sim_profile_enable(aq_sim* s, int32_t on) {
  if (!s) return AQ_E_ARG;
  if (on) {
    for (int k = 0; k < 2; ++k) {
      if (!s->prof_ev[k]) {
        s->prof_ev[k] = new (std::nothrow) cudaEvent_t[2 * aq_sim::PROF_CAP];
        if (!s->prof_ev[k]) return AQ_E_NOMEM;
        for (int j = 0; j < 2 * aq_sim::PROF_CAP; ++j) AQ_CUDA_TRY(cudaEventCreate(&s->prof_ev[k][j]));
      }
      s->prof_n[k] = 0;
    }
  }
  s->prof_on = on ? 1 : 0;
  return AQ_OK;
}

int aq_sim_profile_get(aq_sim* s, int32_t which, double* h_total_ms, int64_t* h_launches) {
  if (!s || which < 0 || which > 1 || !h_total_ms || !h_launches) return AQ_E_ARG;
  double tot = 0.0;
  const int n = s->prof_n[which];
  for (int j = 0; j < n; ++j) {
    AQ_CUDA_TRY(cudaEventSynchronize(s->prof_ev[which][2 * j + 1]));
    float ms = 0.f;
    AQ_CUDA_TRY(cudaEventElapsedTime(&ms, s->prof_ev[which][2 * j], s->prof_ev[which][2 * j + 1]));
    tot += ms;
  }
  s->prof_n[which] = 0;
  *h_total_ms = tot;
  *h_launches = n;
  return AQ_OK;
}

}  // extern "C"
