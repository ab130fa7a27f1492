// Tree build with its point work on the GPU.
//
// The same tree as build_tree (fgt_tree.cpp), which follows the reference's
// pts_tree_build / pts_tree_fix_lr / pts_tree_sort (pts_tree2d4.f,
// pts_tree3d.f): the box-level steps (which boxes refine, level restriction,
// reorganisation, colleagues, depth-first leaf ranks) stay on the host and are
// shared with the host build; every step that touches all points runs here:
//   - the bounding box (pts_tree_boxsize0's min / max);
//   - each refinement level: every point of a refined box moves to its child
//     (coordinate minus centre < 0 goes to the lower child, as
//     sort_pts_to_children) and the children's source counts are summed with
//     warp-aggregated atomics; the host reads the counts back to decide the
//     next level;
//   - after the level restriction, every point descends to its final leaf;
//   - the stable sort of the points by the depth-first rank of their leaf
//     (pts_tree_sort keeps the input order inside a leaf), done as a stable
//     LSD radix sort (CUB) of (rank, input index), and the per-leaf counts
//     that give every box its point range.
// The permutations stay on the device; only box-level arrays cross the bus.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "fgt_device.hpp"
#include "fgt_plan.hpp"

namespace fgtb {
namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

#define CKD(x)                          \
  do {                                  \
    cudaError_t e_ = (x);               \
    if (e_ != cudaSuccess) return e_;   \
  } while (0)

__device__ __forceinline__ int child_slot_d(const double* x, const double* c, int D) {
  int j = 0;
  for (int d = 0; d < D; d++)
    if (!(x[d] - c[d] < 0)) j |= 1 << d;
  return j;
}

// Per-block minimum and maximum of each coordinate (blockDim = 256);
// part[6 block + d] = min, part[6 block + 3 + d] = max.  Four points per
// thread and step, so that several loads are in flight.
template <int DIM>
__global__ void __launch_bounds__(256) k_bbox(const double* __restrict__ x, int n, double* __restrict__ part) {
  __shared__ double smn[DIM][8], smx[DIM][8];
  double mn[DIM], mx[DIM];
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    mn[d] = INFINITY;
    mx[d] = -INFINITY;
  }
  const long long tot = (long long)n * DIM, stride = (long long)gridDim.x * 256 * 4;
  for (long long e = ((long long)blockIdx.x * 256 * 4 + threadIdx.x); e < tot; e += stride) {
    double v[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const long long q = e + (long long)u * 256;
      v[u] = q < tot ? x[q] : NAN;
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const long long q = e + (long long)u * 256;
      if (q < tot) {
        const int d = (int)(q % DIM);
#pragma unroll
        for (int dd = 0; dd < DIM; dd++)
          if (d == dd) {
            mn[dd] = fmin(mn[dd], v[u]);
            mx[dd] = fmax(mx[dd], v[u]);
          }
      }
    }
  }
#pragma unroll
  for (int d = 0; d < DIM; d++)
    for (int off = 16; off > 0; off >>= 1) {
      mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], off));
      mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], off));
    }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      smn[d][w] = mn[d];
      smx[d][w] = mx[d];
    }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; d++) {
      double lo = INFINITY, hi = -INFINITY;
      if (d < DIM)
        for (int k = 0; k < 8; k++) {
          lo = fmin(lo, smn[d][k]);
          hi = fmax(hi, smx[d][k]);
        }
      part[6 * blockIdx.x + d] = lo;
      part[6 * blockIdx.x + 3 + d] = hi;
    }
}

// One refinement level: a point in a refined box [a, b] of the level moves to
// its child; cnt[c - c0] counts the sources of each new box.
__global__ void __launch_bounds__(256) k_refine(const double* __restrict__ x, int n, int dim,
                                                int* __restrict__ pbox, int a, int b,
                                                const int* __restrict__ fc, const double* __restrict__ cen,
                                                int c0, int* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int c = -1;
  if (i < n) {
    const int box = pbox[i];
    if (box >= a && box <= b) {
      const int f = fc[box - a];
      if (f >= 0) {
        c = f + child_slot_d(x + (size_t)dim * i, cen + (size_t)(box - a) * dim, dim);
        pbox[i] = c;
      }
    }
  }
  const unsigned m = __match_any_sync(0xffffffffu, c);
  if (c >= 0 && (int)(threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(cnt + (c - c0), __popc(m));
}

// Working order of the refinement: a Morton key of depth L (x the lowest
// bit of each level's digit, as the child numbering) per point, so that the
// points of a box are contiguous and warps aggregate their count atomics.
__global__ void k_morton(const double* __restrict__ x, int n, int dim, double lx, double ly, double lz,
                         double scale, int L, unsigned long long* __restrict__ key, int* __restrict__ id) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double lo[3] = {lx, ly, lz};
  const long long top = (1LL << L) - 1;
  unsigned long long k = 0;
  for (int d = 0; d < dim; d++) {
    const double v = floor((x[(size_t)dim * i + d] - lo[d]) * scale);
    const long long c = v < 0 ? 0 : v > (double)top ? top : (long long)v;
    for (int b = 0; b < L; b++) k |= (unsigned long long)((c >> b) & 1) << (dim * b + d);
  }
  key[i] = k;
  id[i] = i;
}
__global__ void k_gather_x(const double* __restrict__ x, const int* __restrict__ id, int n, int dim,
                           double* __restrict__ xs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long j = id[i];
  for (int d = 0; d < dim; d++) xs[(size_t)dim * i + d] = x[dim * j + d];
}
__global__ void k_scatter_box(const int* __restrict__ pw, const int* __restrict__ id, int n,
                              int* __restrict__ pbox) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) pbox[id[i]] = pw[i];
}

__global__ void k_remap(int* __restrict__ pbox, int n, const int* __restrict__ idmap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) pbox[i] = idmap[pbox[i]];
}

// Descent to the final leaf (from start[i], or the root), its depth-first
// rank as the sort key, and the per-leaf counts.  The descent is bounded by
// the number of levels; a point that does not reach a leaf sets *err.
__global__ void __launch_bounds__(256) k_locate(const double* __restrict__ x, int n, int dim,
                                                const int* __restrict__ start, const int* __restrict__ nchild,
                                                const int* __restrict__ child, const double* __restrict__ cen,
                                                int nch, int maxdepth, const int* __restrict__ rank,
                                                int* __restrict__ key, int* __restrict__ idx,
                                                int* __restrict__ leafcnt, int* __restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int r = -1;
  if (i < n) {
    int b = start ? start[i] : 0;
    const double* p = x + (size_t)dim * i;
    for (int it = 0; it <= maxdepth && nchild[b] > 0; it++) {
      const int c = child[(size_t)b * nch + child_slot_d(p, cen + (size_t)b * dim, dim)];
      if (c < 0) break;
      b = c;
    }
    r = nchild[b] == 0 ? rank[b] : -1;
    if (r < 0) {
      atomicExch(err, 1);
      r = 0;
    }
    key[i] = r;
    idx[i] = i;
  }
  const unsigned m = __match_any_sync(0xffffffffu, i < n ? r : -1);
  if (i < n && (int)(threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(leafcnt + r, __popc(m));
}

// Exact child digits of every point: the descent from the root for L levels
// with the tree's own centre arithmetic (a child's centre is its parent's
// plus or minus a quarter of the parent's size, the test is coordinate minus
// centre < 0 as sort_pts_to_children), packed most significant level first.
// Every box the refinement can create is a contiguous range of these keys in
// sorted order, and sorted order is the depth-first order of the leaves.
template <int DIM>
__global__ void __launch_bounds__(256) k_exact_key(const double* __restrict__ x, int n, double cx, double cy,
                                                   double cz, double bs0, int L,
                                                   unsigned long long* __restrict__ key, int* __restrict__ id) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double p[DIM], c[DIM];
  const double c3[3] = {cx, cy, cz};
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    p[d] = x[(size_t)DIM * i + d];
    c[d] = c3[d];
  }
  double bs = bs0;
  unsigned long long k = 0;
  for (int l = 0; l < L; l++) {
    int j = 0;
#pragma unroll
    for (int d = 0; d < DIM; d++)
      if (!(p[d] - c[d] < 0)) j |= 1 << d;
    k = (k << DIM) | (unsigned long long)j;
    bs = bs / 2;  // size of the child level
    const double h = bs / 2;
#pragma unroll
    for (int d = 0; d < DIM; d++) c[d] = c[d] + (((j >> d) & 1) ? h : -h);
  }
  key[i] = k;
  id[i] = i;
}

// First position in [lo, hi) whose digit (key >> shift) & (nch - 1) is >= v,
// found by one warp: every round the 32 lanes probe 32 increasing positions
// of the remaining range and a ballot keeps the interval between the last
// probe below v and the first at or above it (the digits are nondecreasing
// there: the range is one box of the level above the digit), so a range of
// n keys takes about log32(n) rounds of independent loads.  Called by all 32
// lanes with the same arguments; every lane returns the position.
__device__ __forceinline__ int warp_digit_lower_bound(const unsigned long long* __restrict__ key, int lo, int hi,
                                                      int shift, int nch, int v) {
  const int lane = threadIdx.x & 31;
  int a = lo, b = hi;  // positions < a are below v; position b is at or above v (or b == hi)
  for (int round = 0; round < 8 && b - a > 32; round++) {
    const long long span = b - a;
    const int p = a + (int)(span * lane / 32);  // lane 0 probes a; a < p < b otherwise
    const bool below = (int)((key[p] >> shift) & (unsigned long long)(nch - 1)) < v;
    const int c = __popc(__ballot_sync(0xffffffffu, below));  // lanes 0 .. c-1 are below
    const int pa = __shfl_sync(0xffffffffu, p, (c + 31) & 31);
    const int pb = __shfl_sync(0xffffffffu, p, c & 31);
    if (c == 0) return a;
    b = c < 32 ? pb : b;
    a = pa + 1;
  }
  const int p = a + lane;
  const bool below = p < b && (int)((key[p] >> shift) & (unsigned long long)(nch - 1)) < v;
  return a + __popc(__ballot_sync(0xffffffffu, below));
}

// Key ranges of the children of the boxes [a, a + nlev) of one level of the
// finished tree (child[box * NCH + j]), from the parents' ranges: one warp
// per (box, digit v = 1 .. NCH-1) finds where the children's digit reaches
// v; child v - 1 ends and child v starts there, child 0 starts at the
// parent's start and child NCH-1 ends at its end.
template <int DIM>
__global__ void __launch_bounds__(256) k_child_bounds(const unsigned long long* __restrict__ key, int shift, int a,
                                                      int nlev, const int* __restrict__ child, int* __restrict__ r0,
                                                      int* __restrict__ r1) {
  constexpr int NCH = 1 << DIM;
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  const long long nw = (long long)nlev * (NCH - 1);
  for (long long w = (long long)blockIdx.x * wpb + (threadIdx.x >> 5); w < nw; w += (long long)gridDim.x * wpb) {
    const int i = (int)(w / (NCH - 1)), v = (int)(w - (long long)i * (NCH - 1)) + 1, box = a + i;
    const int* ch = child + (size_t)box * NCH;
    const int cprev = ch[v - 1], cv = ch[v];
    if (cprev < 0 && cv < 0) continue;  // (warp-uniform)
    const int lo = r0[box], hi = r1[box];
    const int bnd = warp_digit_lower_bound(key, lo, hi, shift, NCH, v);
    if (lane == 0) {
      if (cprev >= 0) r1[cprev] = bnd;
      if (cv >= 0) r0[cv] = bnd;
      if (v == 1 && cprev >= 0) r0[cprev] = lo;
      if (v == NCH - 1 && cv >= 0) r1[cv] = hi;
    }
  }
}

// Sort key of the final point order: the depth-first rank r of the leaf
// whose key range [r0, r1) holds sorted position k, scattered to the
// point's input index, with the input index as the value (a stable sort on
// the rank keeps the input order inside a leaf).  One warp per leaf; the
// leaves' ranges tile the sorted positions.  (A segmented sort of each
// leaf's input indices is slower: the leaves of clustered inputs hold
// thousands of points, and large segments are sorted one block each.)
__global__ void __launch_bounds__(256) k_position_rank(const int* __restrict__ r0, const int* __restrict__ r1,
                                                       const int* __restrict__ leaf_of_rank, int nleaf,
                                                       const int* __restrict__ wid, int* __restrict__ rk,
                                                       int* __restrict__ idx) {
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  for (int r = blockIdx.x * wpb + (threadIdx.x >> 5); r < nleaf; r += gridDim.x * wpb) {
    const int leaf = leaf_of_rank[r], lo = r0[leaf], hi = r1[leaf];
    for (int k = lo + lane; k < hi; k += 32) {
      rk[wid[k]] = r;
      idx[k] = k;
    }
  }
}
__global__ void k_root_range(int* r0, int* r1, int n) {
  r0[0] = 0;
  r1[0] = n;
}

// ---- refinement on the device (exact-key form) ----
// lev[2 l], lev[2 l + 1]: first and last box of level l (last < first: empty);
// lev[2 nslot]: the box count.  Box arrays hold the tree as the host builds
// it (tree_refine_level): level by level, the children of a refined box
// consecutive, refined boxes in box order.
__global__ void k_ref_init(int* lev, int nslot, int* r0, int* r1, int* par, int* nchild, int* child, int* level,
                           double* cen, int nch, int dim, double cx, double cy, double cz, int n, int* ncoll,
                           int* coll, int nco) {
  ncoll[0] = 1;
  coll[0] = 0;
  for (int q = 1; q < nco; q++) coll[q] = -1;
  for (int i = 0; i < nslot; i++) {
    lev[2 * i] = 0;
    lev[2 * i + 1] = -1;
  }
  lev[1] = 0;
  lev[2 * nslot] = 1;
  r0[0] = 0;
  r1[0] = n;
  par[0] = -1;
  nchild[0] = 0;
  level[0] = 0;
  for (int j = 0; j < nch; j++) child[j] = -1;
  const double c[3] = {cx, cy, cz};
  for (int d = 0; d < dim; d++) cen[d] = c[d];
}
// ---- multi-block exclusive scans of 0/1 flags (blockDim 256) ----
// Block k of G handles the items [k chunk, min(n, (k + 1) chunk)), chunk =
// ceil(n / G): a counting pass writes each block's count to part[k], one
// block scans part[] (k_scan_top), and a ranking pass adds each block's
// offset to the block-wide prefix of its items.
__device__ __forceinline__ int block_reduce256(int v, int* sw) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if (lane == 0) sw[w] = v;
  __syncthreads();
  int t = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) t += sw[k];
  __syncthreads();
  return t;
}
// exclusive prefix of v over the block; *total the block's sum
__device__ __forceinline__ int block_excl_scan256(int v, int* sw, int& total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int x = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += x;
  }
  if (lane == 31) sw[w] = incl;
  __syncthreads();
  int before = 0, t = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int x = sw[k];
    before += k < w ? x : 0;
    t += x;
  }
  __syncthreads();
  total = t;
  return before + incl - v;
}
// exclusive scan of part[0, G) in place (G <= 4096, one block of 1024);
// the sum goes to *total, and with lev (the refinement) it makes the id
// range of level l + 1: nch children per flagged box after the current boxes
__global__ void __launch_bounds__(1024) k_scan_top(int* __restrict__ part, int G, int* __restrict__ total,
                                                   int* __restrict__ lev, int l, int nslot, int nch) {
  __shared__ int sw[32];
  const int per = (G + 1023) / 1024, i0 = min(G, (int)threadIdx.x * per), i1 = min(G, i0 + per);
  int v = 0;
  for (int i = i0; i < i1; i++) v += part[i];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int x = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += x;
  }
  if (lane == 31) sw[w] = incl;
  __syncthreads();
  int before = 0, t = 0;
  for (int k = 0; k < 32; k++) {
    before += k < w ? sw[k] : 0;
    t += sw[k];
  }
  int run = before + incl - v;
  for (int i = i0; i < i1; i++) {
    const int x = part[i];
    part[i] = run;
    run += x;
  }
  if (threadIdx.x == 0) {
    if (total) *total = t;
    if (lev && t > 0) {
      const int nb = lev[2 * nslot];
      lev[2 * (l + 1)] = nb;
      lev[2 * (l + 1) + 1] = nb + nch * t - 1;
      lev[2 * nslot] = nb + nch * t;
    }
  }
}
// refinement, level l: flag[i] = box first + i holds more than thr sources;
// part[block] = the block's count
__global__ void __launch_bounds__(256) k_ref_count(const int* __restrict__ lev, int l, const int* __restrict__ r0,
                                                   const int* __restrict__ r1, int thr, int* __restrict__ flag,
                                                   int* __restrict__ part) {
  __shared__ int sw[8];
  const int first = lev[2 * l], n = max(0, lev[2 * l + 1] - first + 1);
  const int chunk = (n + gridDim.x - 1) / gridDim.x, i0 = blockIdx.x * chunk, i1 = min(n, i0 + chunk);
  int c = 0;
  for (int i = i0 + threadIdx.x; i < i1; i += 256) {
    const int f = r1[first + i] - r0[first + i] > thr;
    flag[i] = f;
    c += f;
  }
  c = block_reduce256(c, sw);
  if (threadIdx.x == 0) part[blockIdx.x] = c;
}
// pos[i] = the rank of flagged box first + i among the level's flagged boxes
__global__ void __launch_bounds__(256) k_ref_rank(const int* __restrict__ lev, int l, const int* __restrict__ flag,
                                                  const int* __restrict__ part, int* __restrict__ pos) {
  __shared__ int sw[8];
  const int first = lev[2 * l], n = max(0, lev[2 * l + 1] - first + 1);
  const int chunk = (n + gridDim.x - 1) / gridDim.x, i0 = blockIdx.x * chunk, i1 = min(n, i0 + chunk);
  int carry = part[blockIdx.x];
  for (int base = i0; base < i1; base += 256) {  // (block-uniform)
    const int i = base + threadIdx.x;
    const int v = i < i1 ? flag[i] : 0;
    int tot;
    const int ex = block_excl_scan256(v, sw, tot);
    if (i < i1) pos[i] = carry + ex;
    carry += tot;
  }
}
// blocks of a flag scan over n items (at most 4096, 2048 items or more each)
static int scan_blocks(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 2047) / 2048, 1184)); }

// The children of the refined boxes of level l: structure, centres (the
// parent's plus or minus h, a quarter of the parent's size, in each
// dimension) and key ranges.  One warp per (refined box, digit v = 1 ..
// NCH-1): the warp finds where the children's digit reaches v
// (warp_digit_lower_bound), lane 0 writes child v - 1 (and lane 1 child
// NCH-1 for the last digit).
template <int DIM>
__device__ __forceinline__ void ref_child(int b, int c, int j, int l, double h, int* __restrict__ par,
                                          int* __restrict__ nchild, int* __restrict__ child, int* __restrict__ level,
                                          double* __restrict__ cen) {
  constexpr int NCH = 1 << DIM;
  child[(size_t)b * NCH + j] = c;
  par[c] = b;
  level[c] = l + 1;
  nchild[c] = 0;
#pragma unroll
  for (int q = 0; q < NCH; q++) child[(size_t)c * NCH + q] = -1;
#pragma unroll
  for (int d = 0; d < DIM; d++) cen[(size_t)c * DIM + d] = cen[(size_t)b * DIM + d] + (((j >> d) & 1) ? h : -h);
}
template <int DIM>
__global__ void __launch_bounds__(256) k_ref_children(const int* __restrict__ lev, int l,
                                                      const int* __restrict__ flag, const int* __restrict__ pos,
                                                      const unsigned long long* __restrict__ key, int shift, double h,
                                                      int* __restrict__ r0, int* __restrict__ r1,
                                                      int* __restrict__ par, int* __restrict__ nchild,
                                                      int* __restrict__ child, int* __restrict__ level,
                                                      double* __restrict__ cen) {
  constexpr int NCH = 1 << DIM;
  const int first = lev[2 * l], n = lev[2 * l + 1] - first + 1, c0 = lev[2 * (l + 1)];
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  const long long nw = (long long)n * (NCH - 1);
  for (long long w = (long long)blockIdx.x * wpb + (threadIdx.x >> 5); w < nw; w += (long long)gridDim.x * wpb) {
    const int bi = (int)(w / (NCH - 1)), v = (int)(w - (long long)bi * (NCH - 1)) + 1;
    if (!flag[bi]) continue;  // (warp-uniform)
    const int b = first + bi, cb = c0 + NCH * pos[bi];
    const int lo = r0[b], hi = r1[b];
    const int bnd = warp_digit_lower_bound(key, lo, hi, shift, NCH, v);
    if (lane == 0) {
      ref_child<DIM>(b, cb + v - 1, v - 1, l, h, par, nchild, child, level, cen);
      r1[cb + v - 1] = bnd;
      r0[cb + v] = bnd;
      if (v == 1) {
        r0[cb] = lo;
        nchild[b] = NCH;
      }
    } else if (lane == 1 && v == NCH - 1) {
      ref_child<DIM>(b, cb + NCH - 1, NCH - 1, l, h, par, nchild, child, level, cen);
      r1[cb + NCH - 1] = hi;
    }
  }
}

// Colleagues of box b (computecoll, tree_routs4.f:100-211, as colleagues_box
// in fgt_tree.cpp): the children of the parent's colleagues whose centres lie
// within lim of the box's in every dimension, in the parent's colleague
// order then child order; unused slots -1.  One warp per box: lane q tests
// the children of the parent's colleague q (nco <= 32), and a prefix sum of
// the lanes' counts places them.  When a colleague has all its children,
// child j's coordinate d is that of child 0 or child 2^d (bit d of j), so
// two centres per dimension decide all of them.
template <int DIM>
__device__ __forceinline__ void colleagues_warp(int b, double lim, int nco, const int* __restrict__ par,
                                                const int* __restrict__ child, const double* __restrict__ cen,
                                                int* __restrict__ ncoll, int* __restrict__ coll) {
  constexpr int NCH = 1 << DIM;
  const int lane = threadIdx.x & 31;
  const int dad = par[b];
  const int nc = ncoll[dad];
  double cb[DIM];
#pragma unroll
  for (int d = 0; d < DIM; d++) cb[d] = cen[(size_t)b * DIM + d];
  int ch[NCH];
  unsigned mask = 0;
  const int jb = lane < nc ? coll[(size_t)dad * nco + lane] : -1;
  if (jb >= 0) {
    bool all = true;
#pragma unroll
    for (int j = 0; j < NCH; j++) {
      ch[j] = child[(size_t)jb * NCH + j];
      all = all && ch[j] >= 0;
    }
    if (all) {
      unsigned pass0 = 0u, pass1 = 0u;
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        if (fabs(cen[(size_t)ch[0] * DIM + d] - cb[d]) <= lim) pass0 |= 1u << d;
        if (fabs(cen[(size_t)ch[1 << d] * DIM + d] - cb[d]) <= lim) pass1 |= 1u << d;
      }
#pragma unroll
      for (int j = 0; j < NCH; j++) {
        const unsigned ok = (pass1 & (unsigned)j) | (pass0 & ~(unsigned)j);
        if ((ok & (NCH - 1u)) == NCH - 1u) mask |= 1u << j;
      }
    } else {
#pragma unroll
      for (int j = 0; j < NCH; j++) {
        if (ch[j] < 0) continue;
        bool ok = true;
#pragma unroll
        for (int d = 0; d < DIM; d++) ok = ok && fabs(cen[(size_t)ch[j] * DIM + d] - cb[d]) <= lim;
        if (ok) mask |= 1u << j;
      }
    }
  }
  const int cnt = __popc(mask);
  int incl = cnt;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += v;
  }
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  int o = incl - cnt;
#pragma unroll
  for (int j = 0; j < NCH; j++)
    if ((mask >> j) & 1u) {
      if (o < nco) coll[(size_t)b * nco + o] = ch[j];
      o++;
    }
  const int kept = min(total, nco);
  for (int q = kept + lane; q < nco; q += 32) coll[(size_t)b * nco + q] = -1;
  if (lane == 0) ncoll[b] = kept;
}
// the boxes of level l (ids from lev)
template <int DIM>
__global__ void __launch_bounds__(256) k_ref_colleagues(const int* __restrict__ lev, int l, double lim, int nco,
                                                        const int* __restrict__ par, const int* __restrict__ child,
                                                        const double* __restrict__ cen, int* __restrict__ ncoll,
                                                        int* __restrict__ coll) {
  const int first = lev[2 * l], n = lev[2 * l + 1] - first + 1, wpb = blockDim.x >> 5;
  for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); w < n; w += gridDim.x * wpb)
    colleagues_warp<DIM>(first + w, lim, nco, par, child, cen, ncoll, coll);
}

// ---- level restriction on the device (pts_tree_fix_lr, pts_tree2d4.f:693-996,
// as Builder::fix_lr in fgt_tree.cpp) ----
// Boxes keep their creation ids until the end: the original boxes, then the
// first pass's new boxes level by level, then the second pass's; every
// level is at most three contiguous id ranges ("LrRanges"), in the order the
// host build numbers them after each reorganisation.  The final renumbering
// and the colleagues of the finished tree follow at the end.
struct LrRanges {
  int a[3], b[3];  // ranges [a[i], b[i]] (empty when b < a)
};
__device__ __forceinline__ bool lr_touch(const double* __restrict__ cen, int dim, int x, int y, double lim) {
  for (int d = 0; d < dim; d++)
    if (!(fabs(cen[(size_t)x * dim + d] - cen[(size_t)y * dim + d]) <= lim)) return false;
  return true;
}
__device__ __forceinline__ int lr_box(const LrRanges& R, int i) {  // i-th box of the concatenated ranges, or -1
  for (int r = 0; r < 3; r++) {
    const int n = R.b[r] - R.a[r] + 1;
    if (n <= 0) continue;
    if (i < n) return R.a[r] + i;
    i -= n;
  }
  return -1;
}
__host__ __device__ __forceinline__ int lr_count(const LrRanges& R) {
  int n = 0;
  for (int r = 0; r < 3; r++) n += R.b[r] >= R.a[r] ? R.b[r] - R.a[r] + 1 : 0;
  return n;
}
// first flag pass: a leaf colleague of a grandparent that touches the parent
// of a box two levels down is flagged 1 (0 -> 1 only, so the order of the
// boxes does not matter); boxes [b0, b1], dist per level l of the box
__global__ void k_lr_flag1(int b0, int b1, const int* __restrict__ level, const double* __restrict__ dist1,
                           const int* __restrict__ par, const int* __restrict__ nchild,
                           const int* __restrict__ ncoll, const int* __restrict__ coll, int nco,
                           const double* __restrict__ cen, int dim, int* __restrict__ flag) {
  for (int b = b0 + blockIdx.x * blockDim.x + threadIdx.x; b <= b1; b += gridDim.x * blockDim.x) {
    const double dist = dist1[level[b]];
    const int dad = par[b], gd = par[dad];
    for (int i = 0; i < ncoll[gd]; i++) {
      const int jb = coll[(size_t)gd * nco + i];
      if (nchild[jb] == 0 && flag[jb] == 0 && lr_touch(cen, dim, jb, dad, dist)) atomicCAS(flag + jb, 0, 1);
    }
  }
}
// second flag pass, one level: a flagged box flags the leaf colleagues of its
// parent that touch it (0 -> 2)
__global__ void k_lr_flag2(int b0, int b1, double dist, const int* __restrict__ par,
                           const int* __restrict__ nchild, const int* __restrict__ ncoll,
                           const int* __restrict__ coll, int nco, const double* __restrict__ cen, int dim,
                           int* __restrict__ flag) {
  for (int b = b0 + blockIdx.x * blockDim.x + threadIdx.x; b <= b1; b += gridDim.x * blockDim.x) {
    const int f = flag[b];
    if (f != 1 && f != 2) continue;
    const int dad = par[b];
    for (int i = 0; i < ncoll[dad]; i++) {
      const int jb = coll[(size_t)dad * nco + i];
      if (nchild[jb] == 0 && flag[jb] == 0 && lr_touch(cen, dim, jb, b, dist)) atomicCAS(flag + jb, 0, 2);
    }
  }
}
// updateflags (tree_routs4.f:217-326) over the boxes of one level: a box
// flagged 3 keeps flag 1 when a child of one of its colleagues has children
// and touches it, else 0
__global__ void k_lr_update(LrRanges R, double dist, const int* __restrict__ nchild,
                            const int* __restrict__ child, int nch, const int* __restrict__ ncoll,
                            const int* __restrict__ coll, int nco, const double* __restrict__ cen, int dim,
                            int* __restrict__ flag) {
  const int n = lr_count(R);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int box = lr_box(R, i);
    if (flag[box] != 3) continue;
    int f = 0;
    for (int q = 0; q < ncoll[box] && f == 0; q++) {
      const int jb = coll[(size_t)box * nco + q];
      for (int j = 0; j < nch; j++) {
        const int kb = child[(size_t)jb * nch + j];
        if (kb >= 0 && nchild[kb] > 0 && lr_touch(cen, dim, kb, box, dist)) {
          f = 1;
          break;
        }
      }
    }
    flag[box] = f;
  }
}
// Rank of every flagged box (flag > 0) among the flagged boxes of the
// concatenated ranges, by the multi-block scan above: per-block counts,
// k_scan_top (the total to *total), ranks pos[i] by position i.
__global__ void __launch_bounds__(256) k_lr_count(LrRanges R, const int* __restrict__ flag, int* __restrict__ part) {
  __shared__ int sw[8];
  const int n = lr_count(R);
  const int chunk = (n + gridDim.x - 1) / gridDim.x, i0 = blockIdx.x * chunk, i1 = min(n, i0 + chunk);
  int c = 0;
  for (int i = i0 + threadIdx.x; i < i1; i += 256) c += flag[lr_box(R, i)] > 0;
  c = block_reduce256(c, sw);
  if (threadIdx.x == 0) part[blockIdx.x] = c;
}
__global__ void __launch_bounds__(256) k_lr_rank(LrRanges R, const int* __restrict__ flag,
                                                 const int* __restrict__ part, int* __restrict__ pos) {
  __shared__ int sw[8];
  const int n = lr_count(R);
  const int chunk = (n + gridDim.x - 1) / gridDim.x, i0 = blockIdx.x * chunk, i1 = min(n, i0 + chunk);
  int carry = part[blockIdx.x];
  for (int base = i0; base < i1; base += 256) {  // (block-uniform)
    const int i = base + threadIdx.x;
    const int v = i < i1 ? (flag[lr_box(R, i)] > 0) : 0;
    int tot;
    const int ex = block_excl_scan256(v, sw, tot);
    if (i < i1) pos[i] = carry + ex;
    carry += tot;
  }
}
// tree_refine_boxes_flag (tree_routs4.f:334-388): the flagged boxes of the
// concatenated ranges get nch children each, from id base on, in the ranges'
// order; a child is flagged 3 when its parent's flag is 1.  hsz[l] is a
// quarter of the size of level l (the children's centre offset).
__global__ void k_lr_children(LrRanges R, const int* __restrict__ pos, int base, int nch, int dim,
                              const double* __restrict__ hsz, int* __restrict__ level, int* __restrict__ par,
                              int* __restrict__ nchild, int* __restrict__ child, double* __restrict__ cen,
                              int* __restrict__ flag, int cap, int* __restrict__ err) {
  const int n = lr_count(R);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * nch;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / nch), j = (int)(t - (long long)i * nch);
    const int box = lr_box(R, i);
    const int f = flag[box];
    if (f <= 0) continue;
    const int c = base + nch * pos[i] + j;
    if (c < base || c >= cap) {  // a rank out of the counted range: recorded, not written
      atomicExch(err, 1);
      continue;
    }
    const int l = level[box];
    if (j == 0) nchild[box] = nch;
    child[(size_t)box * nch + j] = c;
    par[c] = box;
    level[c] = l + 1;
    nchild[c] = 0;
    for (int q = 0; q < nch; q++) child[(size_t)c * nch + q] = -1;
    const double h = hsz[l];
    for (int d = 0; d < dim; d++) cen[(size_t)c * dim + d] = cen[(size_t)box * dim + d] + (((j >> d) & 1) ? h : -h);
    flag[c] = f == 1 ? 3 : 0;
  }
}
// colleagues of the boxes of the concatenated ranges (colleagues_warp)
template <int DIM>
__global__ void __launch_bounds__(256) k_lr_colleagues(LrRanges R, double lim, int nco, const int* __restrict__ par,
                                                       const int* __restrict__ child, const double* __restrict__ cen,
                                                       int* __restrict__ ncoll, int* __restrict__ coll) {
  const int n = lr_count(R), wpb = blockDim.x >> 5;
  for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); w < n; w += gridDim.x * wpb)
    colleagues_warp<DIM>(lr_box(R, w), lim, nco, par, child, cen, ncoll, coll);
}
__global__ void k_lr_gather(const int* __restrict__ src, const int* __restrict__ idx, int n, int* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = src[idx[k]];
}
// flags other than 3 back to 0
__global__ void k_lr_keep3(int n, int* __restrict__ flag) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x)
    if (flag[b] != 3) flag[b] = 0;
}
// final numbering: creation id -> final id from a table of (first creation
// id, last, first final id) ranges sorted by creation id
__global__ void k_lr_map(const int* __restrict__ tab, int ntab, int n, int* __restrict__ map) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x) {
    int lo = 0, hi = ntab - 1;  // last range whose first id is <= b
    while (lo < hi) {
      const int m = (lo + hi + 1) >> 1;
      if (tab[3 * m] <= b) lo = m;
      else hi = m - 1;
    }
    map[b] = tab[3 * lo + 2] + (b - tab[3 * lo]);
  }
}
__global__ void k_lr_scatter(int n, const int* __restrict__ map, int nch, int dim, const int* __restrict__ level,
                             const int* __restrict__ par, const int* __restrict__ nchild,
                             const int* __restrict__ child, const double* __restrict__ cen, int* __restrict__ level2,
                             int* __restrict__ par2, int* __restrict__ nchild2, int* __restrict__ child2,
                             double* __restrict__ cen2) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x) {
    const int f = map[b];
    level2[f] = level[b];
    par2[f] = par[b] >= 0 ? map[par[b]] : -1;
    nchild2[f] = nchild[b];
    for (int j = 0; j < nch; j++) {
      const int c = child[(size_t)b * nch + j];
      child2[(size_t)f * nch + j] = c >= 0 ? map[c] : -1;
    }
    for (int d = 0; d < dim; d++) cen2[(size_t)f * dim + d] = cen[(size_t)b * dim + d];
  }
}

// ---- modified list1 on the device (build_list1 in fgt_tree.cpp:
// tree_routs4.f:715-879 in 2D, tree_routs3d.f:511-619 in 3D) ----
// list(X) = [the symmetric entries b, in increasing id | X's own entries in
// its loop order]; own entries are written by X's thread, symmetric ones
// through per-box atomic cursors and then sorted (a handful per box).
struct L1Tree {
  const int *level, *par, *nchild, *child, *ncoll, *coll;
  const double* cen;
  const double* bsz;  // box size per level
  int nch, nco, dim, npw;
};
template <class Own, class Sym>
__device__ __forceinline__ void l1_visit(const L1Tree& T, int b, Own&& own, Sym&& sym) {
  if (T.nchild[b] != 0) return;
  const int l = T.level[b];
  for (int i = 0; i < T.ncoll[b]; i++) {
    const int jb = T.coll[(size_t)b * T.nco + i];
    if (l >= T.npw || T.nchild[jb] == 0) {
      own(jb);
      continue;
    }
    const double dist = 1.05 * (T.bsz[l] + T.bsz[l + 1]) / 2.0;
    for (int j = 0; j < T.nch; j++) {
      const int kb = T.child[(size_t)jb * T.nch + j];
      if (kb < 0) continue;
      bool near = true;
      for (int d = 0; d < T.dim; d++)
        if (!(fabs(T.cen[(size_t)kb * T.dim + d] - T.cen[(size_t)b * T.dim + d]) < dist)) near = false;
      if (near) {
        own(kb);
        if (T.dim == 2) sym(kb);
      }
    }
  }
  if (T.dim == 3) {  // coarser leaf neighbours: the parent's leaf colleagues
    const int dad = T.par[b];
    const double dist = 1.05 * (T.bsz[l] + T.bsz[l - 1]) / 2.0;
    for (int i = 0; i < T.ncoll[dad]; i++) {
      const int jb = T.coll[(size_t)dad * T.nco + i];
      if (T.nchild[jb] != 0) continue;
      bool near = true;
      for (int d = 0; d < T.dim; d++)
        if (!(fabs(T.cen[(size_t)jb * T.dim + d] - T.cen[(size_t)b * T.dim + d]) < dist)) near = false;
      if (near) own(jb);
    }
  }
}
// counts over the visited boxes [b_lo, b_hi]; a leaf root lists itself
__global__ void k_l1_count(L1Tree T, int b_lo, int b_hi, int* __restrict__ nown, int* __restrict__ nsym) {
  if (blockIdx.x == 0 && threadIdx.x == 0 && T.nchild[0] == 0) nown[0] = 1;
  for (int b = b_lo + blockIdx.x * blockDim.x + threadIdx.x; b <= b_hi; b += gridDim.x * blockDim.x) {
    int n = 0;
    l1_visit(T, b, [&](int) { n++; }, [&](int kb) { atomicAdd(nsym + kb, 1); });
    nown[b] = n;
  }
}
__global__ void k_l1_sum(int nb, const int* __restrict__ nown, const int* __restrict__ nsym, int* __restrict__ cnt) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= nb; b += gridDim.x * blockDim.x)
    cnt[b] = b < nb ? nown[b] + nsym[b] : 0;
}
__global__ void k_l1_fill(L1Tree T, int b_lo, int b_hi, const int* __restrict__ l1off, const int* __restrict__ nsym,
                          int* __restrict__ scur, int* __restrict__ l1) {
  if (blockIdx.x == 0 && threadIdx.x == 0 && T.nchild[0] == 0) l1[l1off[0] + nsym[0]] = 0;
  for (int b = b_lo + blockIdx.x * blockDim.x + threadIdx.x; b <= b_hi; b += gridDim.x * blockDim.x) {
    int pos = l1off[b] + nsym[b];
    l1_visit(T, b, [&](int v) { l1[pos++] = v; }, [&](int kb) { l1[atomicAdd(scur + kb, 1)] = b; });
  }
}
// the symmetric block of every list in increasing id (insertion sort)
__global__ void k_l1_sortsym(int nb, const int* __restrict__ l1off, const int* __restrict__ nsym,
                             int* __restrict__ l1) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    int* a = l1 + l1off[b];
    const int n = nsym[b];
    for (int i = 1; i < n; i++) {
      const int v = a[i];
      int j = i - 1;
      while (j >= 0 && a[j] > v) {
        a[j + 1] = a[j];
        j--;
      }
      a[j + 1] = v;
    }
  }
}
// ifhung: the leaves with sources at levels 0 .. the cut (ids 0 .. s_hi)
__global__ void k_l1_hung(int s_hi, const int* __restrict__ nchild, const int* __restrict__ s0,
                          const int* __restrict__ s1, unsigned char* __restrict__ hung) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= s_hi; b += gridDim.x * blockDim.x)
    hung[b] = nchild[b] == 0 && s1[b] - s0[b] > 0;
}

// ---- near-field task arrays on the device (the host's build_near_tasks) ----
// (A, S) pairs of the list1 entries of the near-field source boxes S (levels
// 0 .. the cut, ids 0 .. s_hi), in S-major order
__global__ void k_near_count(int s_hi, const unsigned char* __restrict__ ifhung, const int* __restrict__ l1off,
                             int* __restrict__ cnt) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s <= s_hi) cnt[s] = ifhung[s] ? l1off[s + 1] - l1off[s] : 0;
}
__global__ void k_near_pairs(int s_hi, const unsigned char* __restrict__ ifhung, const int* __restrict__ l1off,
                             const int* __restrict__ l1, const int* __restrict__ pfx, int* __restrict__ keyA,
                             int* __restrict__ valS, int* __restrict__ cntA) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s > s_hi || !ifhung[s]) return;
  int q = pfx[s];
  for (int k = l1off[s]; k < l1off[s + 1]; k++, q++) {
    keyA[q] = l1[k];
    valS[q] = s;
    atomicAdd(cntA + l1[k], 1);
  }
}
// sources and ranges summed down the ancestor chains, one level
__global__ void k_near_cum(int a, int n, const int* __restrict__ parent, const int* __restrict__ ioff,
                           const int* __restrict__ into, const int* __restrict__ s0, const int* __restrict__ s1,
                           int* __restrict__ cum_r, long long* __restrict__ cum_ns) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = a + i, p = parent[b];
  long long ns = 0;
  for (int k = ioff[b]; k < ioff[b + 1]; k++) ns += s1[into[k]] - s0[into[k]];
  cum_r[b] = ioff[b + 1] - ioff[b] + (p >= 0 ? cum_r[p] : 0);
  cum_ns[b] = ns + (p >= 0 ? cum_ns[p] : 0);
}
// per leaf: its ranges (cum_r per evaluated set) and tasks (<= 32 points)
__global__ void k_near_sizes(int nb, const int* __restrict__ nchild, const int* __restrict__ cum_r,
                             const int* __restrict__ s0, const int* __restrict__ s1, const int* __restrict__ t0,
                             const int* __restrict__ t1, int set0, int set1, long long* __restrict__ rcnt,
                             long long* __restrict__ tcnt) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  long long r = 0, tk = 0;
  if (nchild[b] == 0 && cum_r[b] > 0) {
    const int n0 = s1[b] - s0[b], n1 = t1[b] - t0[b];
    if (set0 && n0 > 0) { r += cum_r[b]; tk += (n0 + 31) / 32; }
    if (set1 && n1 > 0) { r += cum_r[b]; tk += (n1 + 31) / 32; }
  }
  rcnt[b] = r;
  tcnt[b] = tk;
}
__global__ void k_near_fill(int nb, const int* __restrict__ nchild, const int* __restrict__ parent,
                            const int* __restrict__ cum_r, const long long* __restrict__ cum_ns,
                            const int* __restrict__ ioff, const int* __restrict__ into, const int* __restrict__ s0,
                            const int* __restrict__ s1, const int* __restrict__ t0, const int* __restrict__ t1,
                            int set0, int set1, const long long* __restrict__ roff, const long long* __restrict__ toff,
                            DirTask* __restrict__ dir, SrcRange* __restrict__ src,
                            unsigned long long* __restrict__ pairs) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb || nchild[b] != 0 || cum_r[b] == 0) return;
  long long ro = roff[b], to = toff[b];
  unsigned long long pr = 0;
  for (int set = 0; set < 2; set++) {
    const int n = set == 0 ? s1[b] - s0[b] : t1[b] - t0[b];
    if (!(set == 0 ? set0 : set1) || n == 0) continue;
    const int i0 = set == 0 ? s0[b] : t0[b];
    const int off = (int)ro;
    for (int a = b; a >= 0; a = parent[a])
      for (int k = ioff[a]; k < ioff[a + 1]; k++) {
        const int sb = into[k];
        src[ro++] = SrcRange{s0[sb], s1[sb] - s0[sb]};
      }
    for (int c = 0; c < n; c += 32) dir[to++] = DirTask{set, i0 + c, min(32, n - c), off, cum_r[b]};
    pr += (unsigned long long)cum_ns[b] * (unsigned long long)n;
  }
  if (pr) atomicAdd(pairs, pr);
}

// Device scratch of one build, stream-ordered on the build's stream (no
// device-wide synchronisation) and freed at the end of the build.
struct Scratch {
  cudaStream_t st;
  std::vector<void*> ptrs;
  explicit Scratch(cudaStream_t s) : st(s) {}
  ~Scratch() {
    for (void* p : ptrs) cudaFreeAsync(p, st);
  }
  template <typename T>
  cudaError_t get(T** out, size_t n) {
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, std::max<size_t>(n, 1) * sizeof(T), st);
    if (e != cudaSuccess) return e;
    ptrs.push_back(p);
    *out = static_cast<T*>(p);
    return cudaSuccess;
  }
};

// Pinned staging of the build's transfers of box arrays: copies from or to
// pageable vectors go through the driver's bounce buffers at a fraction of
// the link rate.  The stage grows and keeps its old buffers until the thread
// exits (freeing pinned memory would wait for the whole device).
struct PinnedStage {
  char* p = nullptr;
  size_t cap = 0;
  std::vector<char*> old;
  ~PinnedStage() {
    if (p) cudaFreeHost(p);
    for (char* q : old) cudaFreeHost(q);
  }
  char* get(size_t n) {
    if (n > cap) {
      if (p) old.push_back(p);
      p = nullptr;
      const size_t want = std::max({n + n / 4, 2 * cap, (size_t)4 << 20});
      cap = 0;
      if (cudaHostAlloc(reinterpret_cast<void**>(&p), want, cudaHostAllocPortable) != cudaSuccess) {
        (void)cudaGetLastError();
        p = nullptr;
        return nullptr;
      }
      cap = want;
    }
    return p;
  }
};
thread_local PinnedStage g_stage;

// One batch of transfers through the stage (sized up front); finish()
// synchronises the stream and copies the downloads out, after which the
// stage may be reused.  Without pinned memory the copies go direct.
struct StagedBatch {
  cudaStream_t st;
  char* base = nullptr;
  size_t used = 0, cap = 0;
  struct Out {
    void* dst;
    size_t off, bytes;
  };
  std::vector<Out> outs;
  StagedBatch(cudaStream_t s, size_t total) : st(s), cap(total) { base = g_stage.get(total); }
  size_t take(size_t b) {
    const size_t off = (used + 255) & ~size_t(255);
    used = off + b;
    return off;
  }
  template <typename T>
  cudaError_t down(T* dst, const T* dev, size_t n) {
    const size_t b = n * sizeof(T);
    if (b == 0) return cudaSuccess;
    if (!base || ((used + 255) & ~size_t(255)) + b > cap) return cudaMemcpyAsync(dst, dev, b, cudaMemcpyDeviceToHost, st);
    const size_t off = take(b);
    outs.push_back({dst, off, b});
    return cudaMemcpyAsync(base + off, dev, b, cudaMemcpyDeviceToHost, st);
  }
  template <typename T>
  cudaError_t up(T* dev, const T* src, size_t n) {
    const size_t b = n * sizeof(T);
    if (b == 0) return cudaSuccess;
    if (!base || ((used + 255) & ~size_t(255)) + b > cap) return cudaMemcpyAsync(dev, src, b, cudaMemcpyHostToDevice, st);
    const size_t off = take(b);
    memcpy(base + off, src, b);
    return cudaMemcpyAsync(dev, base + off, b, cudaMemcpyHostToDevice, st);
  }
  // the same once `ev` (recorded after the downloads) has completed, while
  // the stream goes on with later work
  cudaError_t finish_at(cudaEvent_t ev) {
    cudaError_t e = cudaEventSynchronize(ev);
    if (e != cudaSuccess) return e;
#pragma omp parallel for schedule(dynamic, 1) if (used > (2u << 20))
    for (long long i = 0; i < (long long)outs.size(); i++) memcpy(outs[i].dst, base + outs[i].off, outs[i].bytes);
    outs.clear();
    return cudaSuccess;
  }
  cudaError_t finish() {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
#pragma omp parallel for schedule(dynamic, 1) if (used > (2u << 20))
    for (long long i = 0; i < (long long)outs.size(); i++) memcpy(outs[i].dst, base + outs[i].off, outs[i].bytes);
    outs.clear();
    return cudaSuccess;
  }
};
// blocks of 256 threads for one warp per item (the kernels stride beyond)
static int grid_warps(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 7) / 8, 2368)); }

static size_t staged_bytes(std::initializer_list<size_t> b) {
  size_t t = 0;
  for (size_t x : b) t += (x + 255) & ~size_t(255);
  return t;
}

template <typename T>
cudaError_t upload(T* dst, const T* src, size_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  return cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, st);
}

cudaError_t device_bbox(const double* d_src, int ns, const double* d_trg, int nt, int dim, double* mn,
                        double* mx, cudaStream_t st) {
  Scratch S(st);
  const int nb = 592;
  double* part = nullptr;
  CKD(S.get(&part, (size_t)12 * nb));
  if (dim == 2) {
    k_bbox<2><<<nb, 256, 0, st>>>(d_src, ns, part);
    k_bbox<2><<<nb, 256, 0, st>>>(d_trg, nt, part + 6 * nb);
  } else {
    k_bbox<3><<<nb, 256, 0, st>>>(d_src, ns, part);
    k_bbox<3><<<nb, 256, 0, st>>>(d_trg, nt, part + 6 * nb);
  }
  std::vector<double> h((size_t)12 * nb);
  CKD(cudaMemcpyAsync(h.data(), part, h.size() * 8, cudaMemcpyDeviceToHost, st));
  CKD(cudaStreamSynchronize(st));
  for (int d = 0; d < dim; d++) {
    double lo = INFINITY, hi = -INFINITY;
    for (int k = 0; k < 2 * nb; k++) {
      lo = std::min(lo, h[6 * (size_t)k + d]);
      hi = std::max(hi, h[6 * (size_t)k + 3 + d]);
    }
    mn[d] = lo;
    mx[d] = hi;
  }
  return cudaGetLastError();
}

// Sorts one point set into tree order: perm (device) and per-box ranges.
cudaError_t sort_points_device(const Tree& t, const double* d_x, int n, const int* d_start,
                               const int* d_nchild, const int* d_child, const double* d_cen,
                               const int* d_rank, int nleaf, const std::vector<int>& leaf_of_rank,
                               int* d_perm, std::vector<int>& r0, std::vector<int>& r1, cudaStream_t st) {
  Scratch S(st);
  int *key = nullptr, *key2 = nullptr, *idx = nullptr, *cnt = nullptr, *err = nullptr;
  CKD(S.get(&key, n));
  CKD(S.get(&key2, n));
  CKD(S.get(&idx, n));
  CKD(S.get(&cnt, nleaf));
  CKD(S.get(&err, 1));
  CKD(cudaMemsetAsync(cnt, 0, sizeof(int) * nleaf, st));
  CKD(cudaMemsetAsync(err, 0, sizeof(int), st));
  if (n > 0)
    k_locate<<<(n + 255) / 256, 256, 0, st>>>(d_x, n, t.dim, d_start, d_nchild, d_child, d_cen, t.nch,
                                                t.nlevels + 1, d_rank, key, idx, cnt, err);
  int bits = 1;
  while ((1 << bits) < nleaf) bits++;
  size_t tmp = 0;
  CKD(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key, key2, idx, d_perm, n, 0, bits, st));
  void* dtmp = nullptr;
  CKD(S.get(reinterpret_cast<char**>(&dtmp), tmp));
  CKD(cub::DeviceRadixSort::SortPairs(dtmp, tmp, key, key2, idx, d_perm, n, 0, bits, st));
  std::vector<int> lc(nleaf);
  int herr = 0;
  CKD(cudaMemcpyAsync(lc.data(), cnt, sizeof(int) * nleaf, cudaMemcpyDeviceToHost, st));
  CKD(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKD(cudaStreamSynchronize(st));
  if (herr) {
    fprintf(stderr, "fgt device tree: a point did not reach a leaf (%d points)\n", n);
    return cudaErrorLaunchFailure;
  }
  tree_ranges(t, lc, leaf_of_rank, r0, r1);
  return cudaGetLastError();
}

}  // namespace

cudaError_t build_plan_device_bbox(const double* d_src, int ns, const double* d_trg, int nt, int dim,
                                   double* mn, double* mx, cudaStream_t st) {
  return device_bbox(d_src, ns, d_trg, nt, dim, mn, mx, st);
}

// Upper bound of the box count of the refinement (per level in *per_level):
// level l + 1 holds nch children of each box of level l that holds more than
// thr sources, and at most ns / (thr + 1) boxes can.
long long key_tree_capacity(const TreeSetup& ts, int dim, int ns, std::vector<long long>* per_level) {
  const int nch = 1 << dim;
  std::vector<long long> b(ts.nlmax + 2, 0);
  b[0] = 1;
  long long tot = 1;
  for (int l = 0; l < ts.nlmax && tot < (1LL << 40); l++) {
    const int thr = l < ts.levcut ? ts.ndiv0 : ts.ndiv;
    b[l + 1] = nch * std::min<long long>(b[l], (long long)ns / (thr + 1));
    tot += b[l + 1];
  }
  if (per_level) *per_level = b;
  return tot;
}
constexpr long long kKeyTreeMaxBoxes = 1LL << 24;

// The tree from the exact child digits of the sources (k_exact_key), for
// trees whose depth fits a 64-bit key (31 levels in 2D, 21 in 3D): one sort
// of the keys, after which every refinement level is a warp search per
// (refined box, child digit) inside the parent's range, and the final point order
// is the key order with the input order restored inside each leaf.  No pass
// over the points per level, and the same tree, ranges and permutations as
// the per-level refinement below.
cudaError_t build_tree_device_keys(Tree& t, int dim, const double* d_src, int ns, const double* d_trg, int nt,
                                   bool same, const TreeSetup& ts, int* d_isrc, int* d_itarg, cudaStream_t st,
                                   HostPlan::DevTree* keep) {
  const bool dbg = getenv("FGT_TREE_TIMING") != nullptr;
  const double tA = now_s();
  tree_init(t, dim, ts.bs0, ts.cen0, ts.nlmax);
  Scratch S(st);
  const int L = ts.nlmax, nch = 1 << dim;
  unsigned long long *key = nullptr, *skey = nullptr;
  int *wid0 = nullptr, *wid = nullptr;
  CKD(S.get(&key, ns));
  CKD(S.get(&skey, ns));
  CKD(S.get(&wid0, ns));
  CKD(S.get(&wid, ns));
  if (dim == 2)
    k_exact_key<2><<<(ns + 255) / 256, 256, 0, st>>>(d_src, ns, ts.cen0[0], ts.cen0[1], ts.cen0[2], ts.bs0, L, key,
                                                     wid0);
  else
    k_exact_key<3><<<(ns + 255) / 256, 256, 0, st>>>(d_src, ns, ts.cen0[0], ts.cen0[1], ts.cen0[2], ts.bs0, L, key,
                                                     wid0);
  {
    size_t tmp = 0;
    CKD(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key, skey, wid0, wid, ns, 0, dim * L, st));
    char* dtmp = nullptr;
    CKD(S.get(&dtmp, tmp));
    CKD(cub::DeviceRadixSort::SortPairs(dtmp, tmp, key, skey, wid0, wid, ns, 0, dim * L, st));
  }
  if (dbg) CKD(cudaStreamSynchronize(st));
  const double tK = now_s();
  // refinement on source counts (idivflag = 0), pts_tree2d4.f:495-563: every
  // level on the device (flags, the refined boxes' ranks, the children and
  // their key ranges), no host round trip; the box arrays come back once
  const int nslot = L + 1;
  std::vector<long long> bound;
  const long long cap = key_tree_capacity(ts, dim, ns, &bound);
  long long maxlev = 1;
  for (long long v : bound) maxlev = std::max(maxlev, v);
  int *r0 = nullptr, *r1 = nullptr, *dpar = nullptr, *dnch = nullptr, *dchild = nullptr, *dlevel = nullptr;
  int *dflag = nullptr, *dpos = nullptr, *dlev = nullptr;
  double* dcen = nullptr;
  CKD(S.get(&r0, cap));
  CKD(S.get(&r1, cap));
  CKD(S.get(&dpar, cap));
  CKD(S.get(&dnch, cap));
  CKD(S.get(&dchild, (size_t)cap * nch));
  CKD(S.get(&dlevel, cap));
  CKD(S.get(&dcen, (size_t)cap * dim));
  CKD(S.get(&dflag, maxlev));
  CKD(S.get(&dpos, maxlev));
  CKD(S.get(&dlev, 2 * nslot + 1));
  int* dpart = nullptr;
  CKD(S.get(&dpart, 1184));
  const int nco = t.nco;
  int *dncoll = nullptr, *dcoll = nullptr;
  CKD(S.get(&dncoll, cap));
  CKD(S.get(&dcoll, (size_t)cap * nco));
  k_ref_init<<<1, 1, 0, st>>>(dlev, nslot, r0, r1, dpar, dnch, dchild, dlevel, dcen, nch, dim, ts.cen0[0],
                              ts.cen0[1], ts.cen0[2], ns, dncoll, dcoll, nco);
  {
    double bs = ts.bs0;
    for (int l = 0; l <= ts.nlmax - 1; l++) {
      const int thr = l < ts.levcut ? ts.ndiv0 : ts.ndiv;
      const int g1 = scan_blocks(bound[l]);
      k_ref_count<<<g1, 256, 0, st>>>(dlev, l, r0, r1, thr, dflag, dpart);
      k_scan_top<<<1, 1024, 0, st>>>(dpart, g1, nullptr, dlev, l, nslot, nch);
      k_ref_rank<<<g1, 256, 0, st>>>(dlev, l, dflag, dpart, dpos);
      bs = bs / 2;  // size of level l + 1, as tree_refine_level
      const int g2 = grid_warps(bound[l] * (nch - 1));
      if (dim == 2)
        k_ref_children<2><<<g2, 256, 0, st>>>(dlev, l, dflag, dpos, skey, dim * (L - 1 - l), bs / 2, r0, r1, dpar,
                                              dnch, dchild, dlevel, dcen);
      else
        k_ref_children<3><<<g2, 256, 0, st>>>(dlev, l, dflag, dpos, skey, dim * (L - 1 - l), bs / 2, r0, r1, dpar,
                                              dnch, dchild, dlevel, dcen);
    }
  }
  // colleagues of every level (the level restriction starts from them)
  {
    double bs = ts.bs0;
    for (int l = 1; l <= ts.nlmax; l++) {
      bs = bs / 2;
      const int g = grid_warps(bound[l]);
      if (dim == 2)
        k_ref_colleagues<2><<<g, 256, 0, st>>>(dlev, l, (double)1.05f * bs, nco, dpar, dchild, dcen, dncoll, dcoll);
      else
        k_ref_colleagues<3><<<g, 256, 0, st>>>(dlev, l, (double)1.05f * bs, nco, dpar, dchild, dcen, dncoll, dcoll);
    }
  }
  CKD(cudaGetLastError());
  std::vector<int> hlev(2 * nslot + 1);
  CKD(cudaMemcpyAsync(hlev.data(), dlev, sizeof(int) * hlev.size(), cudaMemcpyDeviceToHost, st));
  CKD(cudaStreamSynchronize(st));
  const int nbr = hlev[2 * nslot];
  if (nbr > cap) {
    fprintf(stderr, "fgt device tree: %d boxes exceed the capacity %lld (%d sources, %d levels)\n", nbr, cap, ns,
            ts.nlmax);
    return cudaErrorLaunchFailure;
  }
  int lev = 0;
  while (lev + 1 <= ts.nlmax && hlev[2 * (lev + 1) + 1] >= hlev[2 * (lev + 1)]) lev++;
  const double tB = now_s();
  // level restriction on the device (pts_tree_fix_lr, pts_tree2d4.f:693-996)
  std::vector<int> lf0(lev + 1), ll0(lev + 1);
  for (int l = 0; l <= lev; l++) {
    lf0[l] = hlev[2 * l];
    ll0[l] = hlev[2 * l + 1];
  }
  std::vector<double> bsz(lev + 3);
  bsz[0] = ts.bs0;
  for (int l = 1; l < (int)bsz.size(); l++) bsz[l] = bsz[l - 1] / 2;
  int nbc = nbr;  // boxes so far (creation ids)
  // LR arrays, growable
  struct LrA {
    int *par = nullptr, *nch = nullptr, *child = nullptr, *level = nullptr, *ncoll = nullptr, *coll = nullptr,
        *flag = nullptr, *pos = nullptr;
    double* cen = nullptr;
    size_t cap = 0;
  } A;
  auto lr_alloc = [&](LrA& X, size_t c) -> cudaError_t {
    X.cap = c;
    CKD(S.get(&X.par, c));
    CKD(S.get(&X.nch, c));
    CKD(S.get(&X.child, c * nch));
    CKD(S.get(&X.level, c));
    CKD(S.get(&X.ncoll, c));
    CKD(S.get(&X.coll, c * nco));
    CKD(S.get(&X.flag, c));
    CKD(S.get(&X.pos, c));
    CKD(S.get(&X.cen, c * dim));
    return cudaSuccess;
  };
  auto lr_copy = [&](LrA& X, const int* par_, const int* nch_, const int* child_, const int* level_,
                     const int* ncoll_, const int* coll_, const int* flag_, const double* cen_, size_t n,
                     const int* pos_ = nullptr) -> cudaError_t {
    auto cp = [&](void* d, const void* s_, size_t b) {
      return b ? cudaMemcpyAsync(d, s_, b, cudaMemcpyDeviceToDevice, st) : cudaSuccess;
    };
    CKD(cp(X.par, par_, 4 * n));
    CKD(cp(X.nch, nch_, 4 * n));
    CKD(cp(X.child, child_, 4 * n * nch));
    CKD(cp(X.level, level_, 4 * n));
    CKD(cp(X.ncoll, ncoll_, 4 * n));
    CKD(cp(X.coll, coll_, 4 * n * nco));
    if (flag_) CKD(cp(X.flag, flag_, 4 * n));
    if (pos_) CKD(cp(X.pos, pos_, 4 * n));
    CKD(cp(X.cen, cen_, 8 * n * dim));
    return cudaSuccess;
  };
  auto lr_grow = [&](size_t need) -> cudaError_t {
    if (need <= A.cap) return cudaSuccess;
    LrA B;
    CKD(lr_alloc(B, std::max(need, 2 * A.cap)));
    // the ranks of the scan that precedes every growth are copied too
    CKD(lr_copy(B, A.par, A.nch, A.child, A.level, A.ncoll, A.coll, A.flag, A.cen, nbc, A.pos));
    A = B;
    return cudaSuccess;
  };
  CKD(lr_alloc(A, (size_t)nbr + std::max<size_t>(nbr / 4, 4096)));
  CKD(lr_copy(A, dpar, dnch, dchild, dlevel, dncoll, dcoll, nullptr, dcen, nbr));
  CKD(cudaMemsetAsync(A.flag, 0, sizeof(int) * A.cap, st));
  // ranges per level: the original boxes, the first pass's, the second's
  std::vector<LrRanges> RL(lev + 2);
  for (int l = 0; l <= lev + 1; l++)
    for (int r = 0; r < 3; r++) {
      RL[l].a[r] = 0;
      RL[l].b[r] = -1;
    }
  for (int l = 0; l <= lev; l++) {
    RL[l].a[0] = lf0[l];
    RL[l].b[0] = ll0[l];
  }
  int* d_tot = nullptr;
  double *d_dist1 = nullptr, *d_hsz = nullptr;
  CKD(S.get(&d_tot, 64));
  CKD(cudaMemsetAsync(d_tot, 0, 64 * sizeof(int), st));
  CKD(S.get(&d_dist1, lev + 3));
  CKD(S.get(&d_hsz, lev + 3));
  auto grid_for = [](long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 1184)); };
  int* d_part = nullptr;
  CKD(S.get(&d_part, 1184));
  // ranks of the flagged boxes of R into A.pos, their number to d_tot[0]
  auto lr_scan = [&](const LrRanges& R) {
    const int g = scan_blocks(lr_count(R));
    k_lr_count<<<g, 256, 0, st>>>(R, A.flag, d_part);
    k_scan_top<<<1, 1024, 0, st>>>(d_part, g, d_tot, nullptr, 0, 0, 0);
    k_lr_rank<<<g, 256, 0, st>>>(R, A.flag, d_part, A.pos);
  };
  auto lr_colleagues = [&](const LrRanges& R, double lim) {
    const int g = grid_warps(lr_count(R));
    if (dim == 2) k_lr_colleagues<2><<<g, 256, 0, st>>>(R, lim, nco, A.par, A.child, A.cen, A.ncoll, A.coll);
    else k_lr_colleagues<3><<<g, 256, 0, st>>>(R, lim, nco, A.par, A.child, A.cen, A.ncoll, A.coll);
  };
  if (lev >= 2) {
    std::vector<double> dist1(lev + 3, 0.0), hsz(lev + 3, 0.0);
    for (int l = 2; l <= lev; l++) dist1[l] = 1.05 * (bsz[l - 1] + bsz[l - 2]) / 2.0;
    for (int l = 0; l <= lev; l++) hsz[l] = bsz[l + 1] / 2;
    CKD(upload(d_dist1, dist1.data(), dist1.size(), st));
    CKD(upload(d_hsz, hsz.data(), hsz.size(), st));
    // flag passes
    k_lr_flag1<<<grid_for(ll0[lev] - lf0[2] + 1), 256, 0, st>>>(lf0[2], ll0[lev], A.level, d_dist1, A.par, A.nch,
                                                                A.ncoll, A.coll, nco, A.cen, dim, A.flag);
    for (int l = lev; l >= 1; l--)
      k_lr_flag2<<<grid_for(ll0[l] - lf0[l] + 1), 256, 0, st>>>(lf0[l], ll0[l], 1.05 * (bsz[l] + bsz[l - 1]) / 2.0,
                                                                 A.par, A.nch, A.ncoll, A.coll, nco, A.cen, dim,
                                                                 A.flag);
    // first refinement pass: flagged boxes of levels 1 .. lev-2, in id order
    if (lev >= 3) {
      LrRanges R;
      for (int r = 0; r < 3; r++) { R.a[r] = 0; R.b[r] = -1; }
      R.a[0] = lf0[1];
      R.b[0] = ll0[lev - 2];
      lr_scan(R);
      // exclusive ranks at the first box of each level 1 .. lev-2
      std::vector<int> idx(lev - 2);
      for (int l = 1; l <= lev - 2; l++) idx[l - 1] = lf0[l] - lf0[1];
      int* d_idx = nullptr;
      CKD(S.get(&d_idx, idx.size()));
      CKD(upload(d_idx, idx.data(), idx.size(), st));
      k_lr_gather<<<1, 64, 0, st>>>(A.pos, d_idx, (int)idx.size(), d_tot + 1);
      std::vector<int> rk(lev - 1);
      CKD(cudaMemcpyAsync(rk.data(), d_tot, sizeof(int) * rk.size(), cudaMemcpyDeviceToHost, st));
      CKD(cudaStreamSynchronize(st));
      const int total = rk[0];
      // rank at level l's first box: rk[l] (l = 1 .. lev-2); level l's flagged boxes: up to the next
      std::vector<int> at(lev);
      for (int l = 1; l <= lev - 2; l++) at[l] = rk[l];
      at[lev - 1] = total;
      if (total > 0) {
        CKD(lr_grow((size_t)nbc + (size_t)nch * total));
        k_lr_children<<<grid_for((long long)lr_count(R) * nch), 256, 0, st>>>(R, A.pos, nbc, nch, dim, d_hsz, A.level,
                                                                             A.par, A.nch, A.child, A.cen, A.flag,
                                                                             nbc + nch * total, d_tot + 60);
        for (int l = 1; l <= lev - 2; l++) {
          RL[l + 1].a[1] = nbc + nch * at[l];
          RL[l + 1].b[1] = nbc + nch * at[l + 1] - 1;
        }
        nbc += nch * total;
      }
    }
    // colleagues after the first pass (computecoll on that tree)
    for (int l = 1; l <= lev; l++)
      lr_colleagues(RL[l], (double)1.05f * bsz[l]);
    k_lr_keep3<<<grid_for(nbc), 256, 0, st>>>(nbc, A.flag);
    // second pass, level by level (updateflags, then refinement in the
    // order old boxes, this pass's boxes)
    for (int l = 2; l <= lev - 2; l++) {
      k_lr_update<<<grid_for(lr_count(RL[l])), 256, 0, st>>>(RL[l], 1.05 * (bsz[l] + bsz[l + 1]) / 2.0, A.nch,
                                                             A.child, nch, A.ncoll, A.coll, nco, A.cen, dim, A.flag);
      lr_scan(RL[l]);
      int total = 0;
      CKD(cudaMemcpyAsync(&total, d_tot, sizeof(int), cudaMemcpyDeviceToHost, st));
      CKD(cudaStreamSynchronize(st));
      if (total <= 0) continue;
      CKD(lr_grow((size_t)nbc + (size_t)nch * total));
      k_lr_children<<<grid_for((long long)lr_count(RL[l]) * nch), 256, 0, st>>>(RL[l], A.pos, nbc, nch, dim, d_hsz,
                                                                               A.level, A.par, A.nch, A.child, A.cen,
                                                                               A.flag, nbc + nch * total, d_tot + 60);
      RL[l + 1].a[2] = nbc;
      RL[l + 1].b[2] = nbc + nch * total - 1;
      LrRanges Rn;
      for (int r = 0; r < 3; r++) { Rn.a[r] = 0; Rn.b[r] = -1; }
      Rn.a[0] = RL[l + 1].a[2];
      Rn.b[0] = RL[l + 1].b[2];
      lr_colleagues(Rn, (double)1.05f * bsz[l + 1]);
      nbc += nch * total;
    }
  }
  CKD(cudaGetLastError());
  {
    int lr_err = 0;
    CKD(cudaMemcpyAsync(&lr_err, d_tot + 60, sizeof(int), cudaMemcpyDeviceToHost, st));
    CKD(cudaStreamSynchronize(st));
    if (lr_err) {
      fprintf(stderr, "fgt device tree: level restriction child id out of range (%d boxes, %d sources)\n", nbc, ns);
      return cudaErrorLaunchFailure;
    }
  }
  // final numbering: per level the original boxes, then each pass's
  std::vector<int> tab, nlevb(lev + 1, 0);
  {
    std::vector<std::array<int, 3>> rows;
    int fin = 0;
    for (int l = 0; l <= lev; l++) {
      t.lfirst[l] = fin;
      for (int r = 0; r < 3; r++) {
        const int a = RL[l].a[r], b = RL[l].b[r];
        if (b < a) continue;
        rows.push_back({a, b, fin});
        fin += b - a + 1;
      }
      t.llast[l] = fin - 1;
    }
    std::sort(rows.begin(), rows.end());
    for (auto& r : rows) tab.insert(tab.end(), {r[0], r[1], r[2]});
    if (fin != nbc) {
      fprintf(stderr, "fgt device tree: renumbering covers %d of %d boxes (%d sources)\n", fin, nbc, ns);
      return cudaErrorLaunchFailure;
    }
  }
  const int nb = nbc;
  int *d_tab = nullptr, *d_map = nullptr, *d_nchild = nullptr, *d_child = nullptr, *d_par2 = nullptr,
      *d_level2 = nullptr, *d_ncoll2 = nullptr, *d_coll2 = nullptr, *d_lev2 = nullptr;
  double* d_cen2 = nullptr;
  int *fr0 = nullptr, *fr1 = nullptr;  // the finished tree's key ranges
  CKD(S.get(&d_tab, tab.size()));
  CKD(S.get(&d_map, nb));
  CKD(S.get(&d_lev2, 2 * nslot + 1));
  if (keep) {  // one allocation that outlives this build
    const size_t ib = (((size_t)nb * 4) + 255) & ~size_t(255);
    const size_t bytes = ib * (7 + (size_t)nch + nco) + ((((size_t)nb * dim * 8) + 255) & ~size_t(255));
    char* m = nullptr;
    CKD(cudaMallocAsync(reinterpret_cast<void**>(&m), bytes, st));
    keep->mem = m;
    auto take = [&](size_t b) { char* p = m; m += (b + 255) & ~size_t(255); return p; };
    d_level2 = reinterpret_cast<int*>(take((size_t)nb * 4));
    d_par2 = reinterpret_cast<int*>(take((size_t)nb * 4));
    d_nchild = reinterpret_cast<int*>(take((size_t)nb * 4));
    d_ncoll2 = reinterpret_cast<int*>(take((size_t)nb * 4));
    fr0 = reinterpret_cast<int*>(take((size_t)nb * 4));
    fr1 = reinterpret_cast<int*>(take((size_t)nb * 4));
    d_child = reinterpret_cast<int*>(take((size_t)nb * 4 * nch));
    d_coll2 = reinterpret_cast<int*>(take((size_t)nb * 4 * nco));
    d_cen2 = reinterpret_cast<double*>(take((size_t)nb * 8 * dim));
    keep->level = d_level2;
    keep->parent = d_par2;
    keep->nchild = d_nchild;
    keep->child = d_child;
    keep->ncoll = d_ncoll2;
    keep->coll = d_coll2;
    keep->centers = d_cen2;
    keep->s0 = fr0;
    keep->s1 = fr1;
  } else {
    CKD(S.get(&d_nchild, nb));
    CKD(S.get(&d_child, (size_t)nb * nch));
    CKD(S.get(&d_par2, nb));
    CKD(S.get(&d_level2, nb));
    CKD(S.get(&d_cen2, (size_t)nb * dim));
    CKD(S.get(&d_ncoll2, nb));
    CKD(S.get(&d_coll2, (size_t)nb * nco));
    CKD(S.get(&fr0, nb));
    CKD(S.get(&fr1, nb));
  }
  CKD(upload(d_tab, tab.data(), tab.size(), st));
  k_lr_map<<<grid_for(nb), 256, 0, st>>>(d_tab, (int)tab.size() / 3, nb, d_map);
  k_lr_scatter<<<grid_for(nb), 256, 0, st>>>(nb, d_map, nch, dim, A.level, A.par, A.nch, A.child, A.cen, d_level2,
                                             d_par2, d_nchild, d_child, d_cen2);
  // colleagues of the finished tree (computecoll), the root's as before
  {
    std::vector<int> lv(2 * nslot + 1, 0);
    for (int l = 0; l < nslot; l++) {
      lv[2 * l] = 0;
      lv[2 * l + 1] = -1;
    }
    for (int l = 0; l <= lev; l++) {
      lv[2 * l] = t.lfirst[l];
      lv[2 * l + 1] = t.llast[l];
    }
    lv[2 * nslot] = nb;
    CKD(upload(d_lev2, lv.data(), lv.size(), st));
    CKD(cudaMemcpyAsync(d_ncoll2, A.ncoll, sizeof(int), cudaMemcpyDeviceToDevice, st));
    CKD(cudaMemcpyAsync(d_coll2, A.coll, sizeof(int) * nco, cudaMemcpyDeviceToDevice, st));
    for (int l = 1; l <= lev; l++) {
      const int g = grid_warps(t.llast[l] - t.lfirst[l] + 1);
      if (dim == 2)
        k_ref_colleagues<2><<<g, 256, 0, st>>>(d_lev2, l, (double)1.05f * bsz[l], nco, d_par2, d_child, d_cen2,
                                               d_ncoll2, d_coll2);
      else
        k_ref_colleagues<3><<<g, 256, 0, st>>>(d_lev2, l, (double)1.05f * bsz[l], nco, d_par2, d_child, d_cen2,
                                               d_ncoll2, d_coll2);
    }
  }
  CKD(cudaGetLastError());
  t.nboxes = nb;
  t.nlevels = lev;
  t.level.resize(nb);
  t.parent.resize(nb);
  t.nchild.resize(nb);
  t.child.resize((size_t)nb * nch);
  t.centers.resize((size_t)nb * dim);
  t.ncoll.resize(nb);
  t.coll.resize((size_t)nb * nco);
  {
    const size_t i4 = sizeof(int) * (size_t)nb;
    StagedBatch X(st, staged_bytes({i4, i4, i4, i4 * nch, sizeof(double) * (size_t)nb * dim, i4, i4 * nco}));
    CKD(X.down(t.level.data(), d_level2, nb));
    CKD(X.down(t.parent.data(), d_par2, nb));
    CKD(X.down(t.nchild.data(), d_nchild, nb));
    CKD(X.down(t.child.data(), d_child, (size_t)nb * nch));
    CKD(X.down(t.centers.data(), d_cen2, (size_t)nb * dim));
    CKD(X.down(t.ncoll.data(), d_ncoll2, nb));
    CKD(X.down(t.coll.data(), d_coll2, (size_t)nb * nco));
    CKD(X.finish());
  }
  for (int l = 1; l <= lev; l++) t.boxsize[l] = bsz[l];
  t.boxsize.resize(lev + 1);
  t.lfirst.resize(lev + 1);
  t.llast.resize(lev + 1);
  const double tC = now_s();
  std::vector<int> dfs_rank, leaf_of_rank;
  tree_leaf_ranks(t, dfs_rank, leaf_of_rank);
  const int nleaf = (int)leaf_of_rank.size();
  int* d_lor = nullptr;
  CKD(S.get(&d_lor, nleaf));
  CKD(upload(d_lor, leaf_of_rank.data(), nleaf, st));
  // ranges of the finished tree (the level restriction added boxes and
  // renumbered), level by level from the root
  r0 = fr0;
  r1 = fr1;
  k_root_range<<<1, 1, 0, st>>>(r0, r1, ns);
  for (int l = 0; l < t.nlevels; l++) {
    const int a = t.lfirst[l], n = t.llast[l] - a + 1;
    if (n <= 0) continue;
    const int g = grid_warps((long long)n * (nch - 1));
    if (dim == 2) k_child_bounds<2><<<g, 256, 0, st>>>(skey, dim * (L - 1 - l), a, n, d_child, r0, r1);
    else k_child_bounds<3><<<g, 256, 0, st>>>(skey, dim * (L - 1 - l), a, n, d_child, r0, r1);
  }
  t.s0.assign(nb, 0);
  t.s1.assign(nb, 0);
  StagedBatch Xr(st, staged_bytes({sizeof(int) * (size_t)nb, sizeof(int) * (size_t)nb}));
  CKD(Xr.down(t.s0.data(), r0, nb));
  CKD(Xr.down(t.s1.data(), r1, nb));
  // the host needs the ranges next; the point order (below) is read only by
  // the device plan, later on the same stream
  struct Ev {
    cudaEvent_t e = nullptr;
    ~Ev() {
      if (e) cudaEventDestroy(e);
    }
  } ranges_done;
  CKD(cudaEventCreateWithFlags(&ranges_done.e, cudaEventDisableTiming));
  CKD(cudaEventRecord(ranges_done.e, st));
  // final order: leaf rank of each sorted position, to input order, stable sort
  {
    int *rk = nullptr, *rk2 = nullptr, *idx = nullptr;
    CKD(S.get(&rk, ns));
    CKD(S.get(&rk2, ns));
    CKD(S.get(&idx, ns));
    k_position_rank<<<grid_warps(nleaf), 256, 0, st>>>(r0, r1, d_lor, nleaf, wid, rk, idx);
    int bits = 1;
    while ((1 << bits) < nleaf) bits++;
    size_t tmp = 0;
    CKD(cub::DeviceRadixSort::SortPairs(nullptr, tmp, rk, rk2, idx, d_isrc, ns, 0, bits, st));
    char* dtmp = nullptr;
    CKD(S.get(&dtmp, tmp));
    CKD(cub::DeviceRadixSort::SortPairs(dtmp, tmp, rk, rk2, idx, d_isrc, ns, 0, bits, st));
  }
  const double tD = now_s();
  if (same && nt > 0) CKD(cudaMemcpyAsync(d_itarg, d_isrc, sizeof(int) * nt, cudaMemcpyDeviceToDevice, st));
  CKD(Xr.finish_at(ranges_done.e));
  if (same) {
    t.t0 = t.s0;
    t.t1 = t.s1;
  } else {
    int* d_rank = nullptr;
    double* d_centers = nullptr;
    CKD(S.get(&d_rank, nb));
    CKD(S.get(&d_centers, (size_t)nb * dim));
    {
      StagedBatch X(st, staged_bytes({sizeof(int) * (size_t)nb, sizeof(double) * (size_t)nb * dim}));
      CKD(X.up(d_rank, dfs_rank.data(), nb));
      CKD(X.up(d_centers, t.centers.data(), (size_t)nb * dim));
      CKD(X.finish());
    }
    CKD(sort_points_device(t, d_trg, nt, nullptr, d_nchild, d_child, d_centers, d_rank, nleaf, leaf_of_rank,
                           d_itarg, t.t0, t.t1, st));
  }
  if (dbg) CKD(cudaStreamSynchronize(st));
  if (dbg)
    fprintf(stderr,
            "device tree (keys): keys+sort %.4f refine %.4f (%d levels, %d boxes) lr %.4f ranks+sort_s %.4f "
            "sort_t %.4f\n",
            tK - tA, tB - tK, lev, nbr, tC - tB, tD - tC, now_s() - tD);
  return cudaGetLastError();
}

cudaError_t build_tree_device(Tree& t, int dim, const double* d_src, int ns, const double* d_trg, int nt,
                              bool same, const TreeSetup& ts, int* d_isrc, int* d_itarg,
                              cudaStream_t st, HostPlan::DevTree* keep) {
  if (ns > 0 && ts.nlmax >= 1 && ts.nlmax <= (dim == 2 ? 31 : 21) && !getenv("FGT_TREE_LEVELWISE") &&
      key_tree_capacity(ts, dim, ns, nullptr) <= kKeyTreeMaxBoxes)
    return build_tree_device_keys(t, dim, d_src, ns, d_trg, nt, same, ts, d_isrc, d_itarg, st, keep);
  const bool dbg = getenv("FGT_TREE_TIMING") != nullptr;
  const double tA = now_s();
  tree_init(t, dim, ts.bs0, ts.cen0, ts.nlmax);
  Scratch S(st);
  int* pbox = nullptr;
  CKD(S.get(&pbox, ns));
  // the refinement runs on a copy of the sources in Morton order (pw[i] is
  // the box of working point i, wid[i] its input index); the child choice
  // is the centre comparison either way, so the tree does not depend on it
  int *pw = nullptr, *wid = nullptr, *wid0 = nullptr;
  unsigned long long *mk = nullptr, *mk2 = nullptr;
  double* xs = nullptr;
  CKD(S.get(&pw, ns));
  CKD(S.get(&wid, ns));
  CKD(S.get(&wid0, ns));
  CKD(S.get(&mk, ns));
  CKD(S.get(&mk2, ns));
  CKD(S.get(&xs, (size_t)ns * dim));
  CKD(cudaMemsetAsync(pw, 0, sizeof(int) * std::max(ns, 1), st));
  if (ns > 0) {
    const int L = std::max(1, std::min(ts.nlmax, dim == 2 ? 31 : 21));
    const double lo[3] = {ts.cen0[0] - ts.bs0 / 2, ts.cen0[1] - ts.bs0 / 2, ts.cen0[2] - ts.bs0 / 2};
    k_morton<<<(ns + 255) / 256, 256, 0, st>>>(d_src, ns, dim, lo[0], lo[1], lo[2],
                                                std::ldexp(1.0, L) / ts.bs0, L, mk, wid0);
    size_t tmp = 0;
    CKD(cub::DeviceRadixSort::SortPairs(nullptr, tmp, mk, mk2, wid0, wid, ns, 0, dim * L, st));
    char* dtmp = nullptr;
    CKD(S.get(&dtmp, tmp));
    CKD(cub::DeviceRadixSort::SortPairs(dtmp, tmp, mk, mk2, wid0, wid, ns, 0, dim * L, st));
    k_gather_x<<<(ns + 255) / 256, 256, 0, st>>>(d_src, wid, ns, dim, xs);
  }
  // refinement on source counts (idivflag = 0), pts_tree2d4.f:495-563
  std::vector<int> count(1, ns), fc;
  int* d_fc = nullptr;
  double* d_cen = nullptr;
  int* d_cnt = nullptr;
  size_t cap_lev = 0, cap_new = 0;
  int lev;
  double th = 0, tw = 0;
  for (lev = 0; lev <= ts.nlmax - 1; lev++) {
    const int a = t.lfirst[lev], b = t.llast[lev];
    const int thr = lev < ts.levcut ? ts.ndiv0 : ts.ndiv;
    const double th0 = now_s();
    if (tree_refine_level(t, lev, thr, count, fc) == 0) break;
    th += now_s() - th0;
    const int c0 = t.lfirst[lev + 1], nnew = t.nboxes - c0, nlev = b - a + 1;
    if ((size_t)nlev > cap_lev) {
      cap_lev = (size_t)nlev * 2;
      CKD(S.get(&d_fc, cap_lev));
      CKD(S.get(&d_cen, cap_lev * dim));
    }
    if ((size_t)nnew > cap_new) {
      cap_new = (size_t)nnew * 2;
      CKD(S.get(&d_cnt, cap_new));
    }
    CKD(upload(d_fc, fc.data(), nlev, st));
    CKD(upload(d_cen, t.centers.data() + (size_t)a * dim, (size_t)nlev * dim, st));
    CKD(cudaMemsetAsync(d_cnt, 0, sizeof(int) * nnew, st));
    if (ns > 0) k_refine<<<(ns + 255) / 256, 256, 0, st>>>(xs, ns, dim, pw, a, b, d_fc, d_cen, c0, d_cnt);
    count.resize(t.nboxes, 0);
    CKD(cudaMemcpyAsync(count.data() + c0, d_cnt, sizeof(int) * nnew, cudaMemcpyDeviceToHost, st));
    const double tw0 = now_s();
    CKD(cudaStreamSynchronize(st));
    tw += now_s() - tw0;
  }
  if (dbg) fprintf(stderr, "refine levels %d host %.4f wait %.4f\n", lev, th, tw);
  if (ns > 0) k_scatter_box<<<(ns + 255) / 256, 256, 0, st>>>(pw, wid, ns, pbox);
  const double tB = now_s();
  std::vector<int> idmap;
  tree_finish(t, lev, idmap);
  const double tC = now_s();
  int* d_map = nullptr;
  CKD(S.get(&d_map, idmap.size()));
  CKD(upload(d_map, idmap.data(), idmap.size(), st));
  if (ns > 0) k_remap<<<(ns + 255) / 256, 256, 0, st>>>(pbox, ns, d_map);
  std::vector<int> dfs_rank, leaf_of_rank;
  tree_leaf_ranks(t, dfs_rank, leaf_of_rank);
  const int nb = t.nboxes, nleaf = (int)leaf_of_rank.size();
  int *d_nchild = nullptr, *d_child = nullptr, *d_rank = nullptr;
  double* d_centers = nullptr;
  CKD(S.get(&d_nchild, nb));
  CKD(S.get(&d_child, (size_t)nb * t.nch));
  CKD(S.get(&d_rank, nb));
  CKD(S.get(&d_centers, (size_t)nb * dim));
  CKD(upload(d_nchild, t.nchild.data(), nb, st));
  CKD(upload(d_child, t.child.data(), (size_t)nb * t.nch, st));
  CKD(upload(d_rank, dfs_rank.data(), nb, st));
  CKD(upload(d_centers, t.centers.data(), (size_t)nb * dim, st));
  const double tD = now_s();
  CKD(sort_points_device(t, d_src, ns, pbox, d_nchild, d_child, d_centers, d_rank, nleaf, leaf_of_rank,
                         d_isrc, t.s0, t.s1, st));
  const double tE = now_s();
  if (same) {
    if (nt > 0) CKD(cudaMemcpyAsync(d_itarg, d_isrc, sizeof(int) * nt, cudaMemcpyDeviceToDevice, st));
    t.t0 = t.s0;
    t.t1 = t.s1;
  } else {
    CKD(sort_points_device(t, d_trg, nt, nullptr, d_nchild, d_child, d_centers, d_rank, nleaf,
                           leaf_of_rank, d_itarg, t.t0, t.t1, st));
  }
  CKD(cudaStreamSynchronize(st));
  if (dbg)
    fprintf(stderr, "device tree: refine %.4f lr %.4f ranks+upload %.4f sort_s %.4f sort_t %.4f\n", tB - tA,
            tC - tB, tD - tC, tE - tD, now_s() - tE);
  return cudaGetLastError();
}

cudaError_t build_plan_device(HostPlan& H, int dim, int nd, double delta, double eps, int ns,
                              const double* d_src, int nt, const double* d_trg, bool same, int ifpgh,
                              int ifpghtarg, int* d_isrc, int* d_itarg, cudaStream_t st,
                              int ifcharge, int ifdipole) {
  const double tstart = now_s();
  H.same_points = same;
  double mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
  CKD(device_bbox(d_src, ns, d_trg, same ? 0 : nt, dim, mn, mx, st));
  int npwlevel;
  double bs0, cen0[3] = {0, 0, 0};
  boxsize0_bbox(dim, delta, eps, mn, mx, &npwlevel, &bs0, cen0);
  TreeSetup ts;
  if (!plan_begin(H, dim, nd, delta, eps, ns, nt, ifpgh, ifpghtarg, npwlevel, bs0, cen0, ts, ifcharge,
                  ifdipole)) {
    H.host_tree_s = now_s() - tstart;
    return cudaSuccess;
  }
  CKD(build_tree_device(H.tree, dim, d_src, ns, d_trg, nt, same, ts, d_isrc, d_itarg, st,
                        H.defer_near ? &H.dtree : nullptr));
  H.host_tree_s = now_s() - tstart;
  if (H.defer_near && H.dtree.mem) {
    // the near-field arrays on the GPU, driven from a second host thread
    // beside the host's far-field tasks (its kernels go to the same stream;
    // this thread makes no CUDA call meanwhile)
    int dev = 0;
    CKD(cudaGetDevice(&dev));
    cudaError_t near_err = cudaSuccess;
    plan_end(H, [&] {
      try {
        const double tn = now_s();
        near_err = cudaSetDevice(dev);
        if (near_err == cudaSuccess) near_err = build_near_tasks_device(H, st);
        if (getenv("FGT_TREE_TIMING")) fprintf(stderr, "near-field tasks (device, beside): %.4f\n", now_s() - tn);
      } catch (const std::bad_alloc&) {
        near_err = cudaErrorMemoryAllocation;
      }
    });
    H.near_built = true;
    return near_err;
  }
  plan_end(H);
  return cudaSuccess;
}


// The near-field task arrays of a built host plan on the GPU, in the order of
// the host's build_near_tasks (fgt_plan.cpp): for every leaf, its source
// ranges (the ifhung source boxes whose list1 holds the leaf or one of its
// ancestors, leaf first, each box's sources in increasing box id) once per
// evaluated point set, and its tasks of <= 32 points, leaves in box order.
// The transpose of list1 is a stable radix sort of the (A, S) pairs by A.
cudaError_t build_near_tasks_device(HostPlan& H, cudaStream_t st) {
  const Params& P = H.P;
  const Tree& t = H.tree;
  const Lists& L = H.lists;
  const int nb = t.nboxes, npl = P.npwlevel;
  const int nlevend = npl < P.nlevels ? npl : P.nlevels;
  const int s_hi = nlevend >= 0 ? t.llast[nlevend] : -1;
  const int set0 = P.ifpgh >= 1, set1 = P.ifpghtarg >= 1;
  (void)L;
  Scratch S(st);
  const int nch = t.nch, nco = t.nco, dim = t.dim, nlv = (int)t.boxsize.size();
  int *d_par = nullptr, *d_nch = nullptr, *d_s0 = nullptr, *d_s1 = nullptr, *d_t0 = nullptr, *d_t1 = nullptr,
      *d_level = nullptr, *d_child = nullptr, *d_ncoll = nullptr, *d_coll = nullptr;
  double *d_cen = nullptr, *d_bsz = nullptr;
  unsigned char* d_hung = nullptr;
  CKD(S.get(&d_bsz, nlv + 1));
  CKD(S.get(&d_hung, nb));
  const HostPlan::DevTree& K = H.dtree;
  const bool tsame = t.t0.size() == t.s0.size() && t.t1.size() == t.s1.size() &&
                     std::memcmp(t.t0.data(), t.s0.data(), sizeof(int) * nb) == 0 &&
                     std::memcmp(t.t1.data(), t.s1.data(), sizeof(int) * nb) == 0;
  if (K.mem) {  // the tree build's arrays, still on the device
    d_par = K.parent;
    d_nch = K.nchild;
    d_s0 = K.s0;
    d_s1 = K.s1;
    d_level = K.level;
    d_child = K.child;
    d_ncoll = K.ncoll;
    d_coll = K.coll;
    d_cen = K.centers;
    if (tsame) {
      d_t0 = d_s0;
      d_t1 = d_s1;
    } else {
      CKD(S.get(&d_t0, nb));
      CKD(S.get(&d_t1, nb));
    }
    // small copies, straight from the host arrays (this may run on a thread
    // of its own, whose pinned stage would be allocated for the one call)
    CKD(upload(d_bsz, t.boxsize.data(), nlv, st));
    if (!tsame) {
      CKD(upload(d_t0, t.t0.data(), nb, st));
      CKD(upload(d_t1, t.t1.data(), nb, st));
    }
  } else {
    CKD(S.get(&d_par, nb));
    CKD(S.get(&d_nch, nb));
    CKD(S.get(&d_s0, nb));
    CKD(S.get(&d_s1, nb));
    CKD(S.get(&d_t0, nb));
    CKD(S.get(&d_t1, nb));
    CKD(S.get(&d_level, nb));
    CKD(S.get(&d_child, (size_t)nb * nch));
    CKD(S.get(&d_ncoll, nb));
    CKD(S.get(&d_coll, (size_t)nb * nco));
    CKD(S.get(&d_cen, (size_t)nb * dim));
    const size_t i4 = sizeof(int) * (size_t)nb;
    StagedBatch X(st, staged_bytes({i4, i4, i4, i4, i4, i4, i4, i4 * nch, i4, i4 * nco, 8 * (size_t)nb * dim,
                                    8 * (size_t)nlv}));
    CKD(X.up(d_par, t.parent.data(), nb));
    CKD(X.up(d_nch, t.nchild.data(), nb));
    CKD(X.up(d_s0, t.s0.data(), nb));
    CKD(X.up(d_s1, t.s1.data(), nb));
    CKD(X.up(d_t0, t.t0.data(), nb));
    CKD(X.up(d_t1, t.t1.data(), nb));
    CKD(X.up(d_level, t.level.data(), nb));
    CKD(X.up(d_child, t.child.data(), (size_t)nb * nch));
    CKD(X.up(d_ncoll, t.ncoll.data(), nb));
    CKD(X.up(d_coll, t.coll.data(), (size_t)nb * nco));
    CKD(X.up(d_cen, t.centers.data(), (size_t)nb * dim));
    CKD(X.up(d_bsz, t.boxsize.data(), nlv));
    // the stage is reused below only after this batch's copies (finish)
    CKD(X.finish());
  }
  // list1 of the boxes at levels 1 .. min(nlevels, cut) and the ifhung flags
  const int lmax = std::min(t.nlevels, nlevend);
  const int b_hi = lmax >= 1 ? t.llast[lmax] : -1, b_lo = t.nlevels >= 1 ? t.lfirst[1] : 1;
  int *d_nown = nullptr, *d_nsym = nullptr, *d_l1cnt = nullptr, *d_l1off = nullptr, *d_l1 = nullptr,
      *d_scur = nullptr;
  CKD(S.get(&d_nown, nb));
  CKD(S.get(&d_nsym, nb));
  CKD(S.get(&d_l1cnt, nb + 1));
  CKD(S.get(&d_l1off, nb + 1));
  CKD(S.get(&d_scur, nb));
  CKD(cudaMemsetAsync(d_nown, 0, sizeof(int) * nb, st));
  CKD(cudaMemsetAsync(d_nsym, 0, sizeof(int) * nb, st));
  L1Tree LT{d_level, d_par, d_nch, d_child, d_ncoll, d_coll, d_cen, d_bsz, nch, nco, dim, npl};
  const int gv = (int)std::max<long long>(1, std::min<long long>(((long long)b_hi - b_lo + 1 + 255) / 256, 1184));
  const int gb = (int)std::max<long long>(1, std::min<long long>(((long long)nb + 1 + 255) / 256, 1184));
  k_l1_count<<<gv, 256, 0, st>>>(LT, b_lo, b_hi, d_nown, d_nsym);
  k_l1_sum<<<gb, 256, 0, st>>>(nb, d_nown, d_nsym, d_l1cnt);
  {
    size_t tmp = 0;
    CKD(cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_l1cnt, d_l1off, nb + 1, st));
    char* dt = nullptr;
    CKD(S.get(&dt, tmp));
    CKD(cub::DeviceScan::ExclusiveSum(dt, tmp, d_l1cnt, d_l1off, nb + 1, st));
  }
  int ne = 0;
  CKD(cudaMemcpyAsync(&ne, d_l1off + nb, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKD(cudaStreamSynchronize(st));
  CKD(S.get(&d_l1, std::max(ne, 1)));
  CKD(cudaMemcpyAsync(d_scur, d_l1off, sizeof(int) * nb, cudaMemcpyDeviceToDevice, st));
  k_l1_fill<<<gv, 256, 0, st>>>(LT, b_lo, b_hi, d_l1off, d_nsym, d_scur, d_l1);
  if (dim == 2) k_l1_sortsym<<<gb, 256, 0, st>>>(nb, d_l1off, d_nsym, d_l1);
  if (s_hi >= 0) k_l1_hung<<<(s_hi + 256) / 256, 256, 0, st>>>(s_hi, d_nch, d_s0, d_s1, d_hung);
  // (A, S) pairs, stable sort by A: into[] = the S of each A in increasing id
  int *d_cnt = nullptr, *d_pfx = nullptr, *d_keyA = nullptr, *d_valS = nullptr, *d_keyA2 = nullptr,
      *d_into = nullptr, *d_cntA = nullptr, *d_ioff = nullptr;
  const int nsrcbox = s_hi + 1;
  CKD(S.get(&d_cnt, nsrcbox + 1));
  CKD(S.get(&d_pfx, nsrcbox + 1));
  CKD(S.get(&d_cntA, nb + 1));
  CKD(S.get(&d_ioff, nb + 1));
  CKD(cudaMemsetAsync(d_cntA, 0, sizeof(int) * (nb + 1), st));
  int npairs = 0;
  if (nsrcbox > 0) {
    k_near_count<<<(nsrcbox + 255) / 256, 256, 0, st>>>(s_hi, d_hung, d_l1off, d_cnt);
    CKD(cudaMemsetAsync(d_cnt + nsrcbox, 0, sizeof(int), st));
    size_t tmp = 0;
    CKD(cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_cnt, d_pfx, nsrcbox + 1, st));
    char* dt = nullptr;
    CKD(S.get(&dt, tmp));
    CKD(cub::DeviceScan::ExclusiveSum(dt, tmp, d_cnt, d_pfx, nsrcbox + 1, st));
    CKD(cudaMemcpyAsync(&npairs, d_pfx + nsrcbox, sizeof(int), cudaMemcpyDeviceToHost, st));
    CKD(cudaStreamSynchronize(st));
  }
  CKD(S.get(&d_keyA, npairs));
  CKD(S.get(&d_valS, npairs));
  CKD(S.get(&d_keyA2, npairs));
  CKD(S.get(&d_into, npairs));
  if (npairs > 0) {
    k_near_pairs<<<(nsrcbox + 255) / 256, 256, 0, st>>>(s_hi, d_hung, d_l1off, d_l1, d_pfx, d_keyA, d_valS, d_cntA);
    int bits = 1;
    while ((1 << bits) < nb) bits++;
    size_t tmp = 0;
    CKD(cub::DeviceRadixSort::SortPairs(nullptr, tmp, d_keyA, d_keyA2, d_valS, d_into, npairs, 0, bits, st));
    char* dt = nullptr;
    CKD(S.get(&dt, tmp));
    CKD(cub::DeviceRadixSort::SortPairs(dt, tmp, d_keyA, d_keyA2, d_valS, d_into, npairs, 0, bits, st));
  }
  {
    size_t tmp = 0;
    CKD(cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_cntA, d_ioff, nb + 1, st));
    char* dt = nullptr;
    CKD(S.get(&dt, tmp));
    CKD(cub::DeviceScan::ExclusiveSum(dt, tmp, d_cntA, d_ioff, nb + 1, st));
  }
  // sums down the ancestor chains, level by level
  int* d_cumr = nullptr;
  long long* d_cumns = nullptr;
  CKD(S.get(&d_cumr, nb));
  CKD(S.get(&d_cumns, nb));
  for (int l = 0; l <= P.nlevels; l++) {
    const int a = t.lfirst[l], n = t.llast[l] - a + 1;
    if (n > 0)
      k_near_cum<<<(n + 255) / 256, 256, 0, st>>>(a, n, d_par, d_ioff, d_into, d_s0, d_s1, d_cumr, d_cumns);
  }
  // sizes, offsets (in box order), totals
  long long *d_rc = nullptr, *d_tc = nullptr, *d_roff = nullptr, *d_toff = nullptr;
  unsigned long long* d_pairs = nullptr;
  CKD(S.get(&d_rc, nb + 1));
  CKD(S.get(&d_tc, nb + 1));
  CKD(S.get(&d_roff, nb + 1));
  CKD(S.get(&d_toff, nb + 1));
  CKD(S.get(&d_pairs, 1));
  k_near_sizes<<<(nb + 255) / 256, 256, 0, st>>>(nb, d_nch, d_cumr, d_s0, d_s1, d_t0, d_t1, set0, set1, d_rc, d_tc);
  CKD(cudaMemsetAsync(d_rc + nb, 0, sizeof(long long), st));
  CKD(cudaMemsetAsync(d_tc + nb, 0, sizeof(long long), st));
  CKD(cudaMemsetAsync(d_pairs, 0, sizeof(unsigned long long), st));
  {
    size_t tmp = 0, tmp2 = 0;
    CKD(cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_rc, d_roff, nb + 1, st));
    CKD(cub::DeviceScan::ExclusiveSum(nullptr, tmp2, d_tc, d_toff, nb + 1, st));
    char* dt = nullptr;
    CKD(S.get(&dt, std::max(tmp, tmp2)));
    CKD(cub::DeviceScan::ExclusiveSum(dt, tmp, d_rc, d_roff, nb + 1, st));
    CKD(cub::DeviceScan::ExclusiveSum(dt, tmp2, d_tc, d_toff, nb + 1, st));
  }
  long long tot[2] = {0, 0};
  CKD(cudaMemcpyAsync(&tot[0], d_roff + nb, sizeof(long long), cudaMemcpyDeviceToHost, st));
  CKD(cudaMemcpyAsync(&tot[1], d_toff + nb, sizeof(long long), cudaMemcpyDeviceToHost, st));
  CKD(cudaStreamSynchronize(st));
  // the output arrays outlive this build (until the plan copies them)
  HostPlan::DevNear& out = H.dnear;
  const size_t bd = ((size_t)tot[1] * sizeof(DirTask) + 255) & ~size_t(255);
  const size_t bs = (size_t)tot[0] * sizeof(SrcRange);
  void* mem = nullptr;
  CKD(cudaMallocAsync(&mem, std::max<size_t>(bd + bs, 256), st));
  out.mem = mem;
  out.dir = reinterpret_cast<DirTask*>(mem);
  out.src = reinterpret_cast<SrcRange*>(static_cast<char*>(mem) + bd);
  out.ndir = tot[1];
  out.nsrc = tot[0];
  k_near_fill<<<(nb + 255) / 256, 256, 0, st>>>(nb, d_nch, d_par, d_cumr, d_cumns, d_ioff, d_into, d_s0, d_s1, d_t0,
                                                d_t1, set0, set1, d_roff, d_toff, out.dir, out.src, d_pairs);
  unsigned long long pairs = 0;
  CKD(cudaMemcpyAsync(&pairs, d_pairs, sizeof(pairs), cudaMemcpyDeviceToHost, st));
  CKD(cudaStreamSynchronize(st));
  H.direct_pairs = (long long)pairs;
  H.dir.clear();
  H.dir_src.clear();
  if (H.dtree.mem) {  // the tree arrays are not read after this (stream-ordered release)
    CKD(cudaFreeAsync(H.dtree.mem, st));
    H.dtree = HostPlan::DevTree();
  }
  return cudaGetLastError();
}

void device_near_free(HostPlan& H, cudaStream_t st) {
  if (H.dnear.mem) cudaFreeAsync(H.dnear.mem, st);
  if (H.dtree.mem) cudaFreeAsync(H.dtree.mem, st);
  H.dnear = HostPlan::DevNear();
  H.dtree = HostPlan::DevTree();
}

}  // namespace fgtb
