// CUDA stages of the plane-wave FGT for sm_100a.
//
// (a) form     : per leaf, Hermite coefficients of its sources and the
//                Hermite -> plane-wave transform (g2dformhc_vec + g2dh2pw_real_vec,
//                g3dformhc_vec + g3dh2pw_real_vec), or the direct tensor-product
//                exponential sum (g3dformpwc_vec) where the reference uses it.
// (b) shifts   : diagonal plane-wave translations (g2dshiftpw_vec,
//                g2dcopypwexp_vec): merge up to the cut level, mp -> loc over the
//                plane-wave list, split down to the leaves.  HBM-bound.
// (c) eval     : per leaf, plane wave -> Taylor (g2dpw2local_real_vec) and
//                Taylor evaluation (g2dlevalp_vec), or direct plane-wave
//                evaluation (g2dpwevalp_vec) on the levels the reference picks.
// (d) direct   : near-field Gaussian sum with the reference cutoff
//                (g2d_directcp_vec / g3d_directcp_vec), target-centric.
//
// Expansions are complex FP64 in the reference layouts: 2D pw(npw/2, npw),
// 3D pw(npw, npw, npw/2), one block of nexp per (box slot, density).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <type_traits>

#include "fgt_device.hpp"
#include "fgt_kcommon.cuh"

namespace fgtb {

namespace {

// ------------------------------------------------------------ sort / unsort
// Tree order: out row i = in row perm[i] (dreorderf, fmmcommon2d.f:3-26);
// coordinates and charges of a point move together.
__global__ void k_gather_pts(const double* __restrict__ x, const double* __restrict__ q,
                             double* __restrict__ xs, double* __restrict__ qs,
                             const int* __restrict__ perm, int n, int dim, int nd, int vec) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const long long p = perm[i];
    if (x == nullptr) {
    } else if (dim == 2 && vec) {
      reinterpret_cast<double2*>(xs)[i] = reinterpret_cast<const double2*>(x)[p];
    } else {
      for (int d = 0; d < dim; d++) xs[(long long)i * dim + d] = x[p * dim + d];
    }
    if (q)
      for (int c = 0; c < nd; c++) qs[(long long)i * nd + c] = q[p * nd + c];
  }
}
// Diagonal translation tables from their 1D factors (merge_split_pw_matrices,
// pw_translation_matrices): merge row (l nch + jc) for parents at level l,
// entry e = prod_d (child jc on the + side along d ? conj(v) : v) with
// v = ww[node_d(e)][nlevels - l]; mp->loc row s = (ox+1) + 3 (oy+1) [+ 9 (oz+1)],
// entry prod_d (o_d = 0 ? 1 : o_d > 0 ? w1 : conj(w1)).  Products are formed
// left to right without contraction, (ac - bd, ad + bc).
__device__ __forceinline__ double2 cmul_rn(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__global__ void k_shift_tables(int dim, int npw, int nexp, int nlevels, int lstart, int nms,
                               const double2* __restrict__ ww, const double2* __restrict__ w1,
                               double2* __restrict__ wms, double2* __restrict__ wsh) {
  const int nch = 1 << dim, n2 = npw / 2, ns3 = dim == 2 ? 9 : 27;
  const long long nm = (long long)(nlevels + 1) * nch * nexp, total = nm + (long long)ns3 * nexp;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const bool merge = i < nm;
    const long long r = merge ? i / nexp : (i - nm) / nexp;
    const int e = (int)((merge ? i : i - nm) % nexp);
    int node[3];
    if (dim == 2) {
      node[0] = e % n2;
      node[1] = e / n2;
    } else {
      node[0] = e % npw;
      node[1] = (e / npw) % npw;
      node[2] = e / (npw * npw);
    }
    double2 f = make_double2(1.0, 0.0);
    if (merge) {
      const int l = (int)(r / nch), jc = (int)(r % nch);
      if (l < lstart || l > nlevels - 1) {
        wms[i] = make_double2(0.0, 0.0);
        continue;
      }
      const int klev = nlevels - l;
      for (int d = 0; d < dim; d++) {
        double2 v = ww[node[d] * (nms + 1) + klev];
        if ((jc >> d) & 1) v.y = -v.y;
        f = cmul_rn(f, v);
      }
      wms[i] = f;
    } else {
      const int s = (int)r;
      const int o[3] = {s % 3 - 1, (s / 3) % 3 - 1, s / 9 - 1};
      for (int d = 0; d < dim; d++) {
        double2 v = o[d] == 0 ? make_double2(1.0, 0.0) : w1[node[d]];
        if (o[d] < 0) v.y = -v.y;
        f = cmul_rn(f, v);
      }
      wsh[i - nm] = f;
    }
  }
}

// *bad = 1 when any of x[0, n) is not finite
__global__ void k_all_finite(const double* __restrict__ x, size_t n, int* __restrict__ bad) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (!isfinite(x[i])) *bad = 1;
}
// qs[i] = q[perm[i]] for one density (the charges of every execute): four
// independent random reads in flight per thread
__global__ void __launch_bounds__(256) k_gather1(const double* __restrict__ q, const int* __restrict__ perm, int n,
                                                 double* __restrict__ qs) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += 4 * stride) {
    int p[4];
    double v[4];
#pragma unroll
    for (int u = 0; u < 4; u++) p[u] = i + u * stride < n ? perm[i + u * stride] : -1;
#pragma unroll
    for (int u = 0; u < 4; u++) v[u] = p[u] >= 0 ? q[p[u]] : 0.0;
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (p[u] >= 0) qs[i + u * stride] = v[u];
  }
}
// inv[perm[i]] = i
__global__ void k_invperm(const int* __restrict__ perm, int n, int* __restrict__ inv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) inv[perm[i]] = i;
}
// Caller order: out row j = in row iperm[j] (dreorderi / dreorderiv,
// fmmcommon2d.f:29-90), written as a gather so the stores stay coalesced.
// A sorted row is `stride` doubles; out takes the w doubles from `off`.
__global__ void k_unsort(const double* __restrict__ in, double* __restrict__ out,
                         const int* __restrict__ iperm, int n, int stride, int off, int w) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const long long p = iperm[j];
    for (int c = 0; c < w; c++) out[(long long)j * w + c] = in[p * stride + off + c];
  }
}

// ------------------------------------------------------------ (a) form, 2D
// One CTA (256 threads) per (leaf, density).
//   H[j + Pp k] = sum_i q_i x_i^j y_i^k / sqrt(j! k!)      (g2dformhc_vec)
// is a small (P x n) * (n x P) product: the rows x^j/sqrt(j!) and
// q y^k/sqrt(k!) of a chunk of sources are built in shared memory with the
// 1/sqrt(j) table, each thread keeps a 4x4 register tile of H and the chunk's
// sources are split over G thread groups (split-K), reduced at the end.  Then
// the two 1D Hermite -> plane-wave passes (g2dh2pw_real_vec,
// g2drouts.f:1276-1326) run in shared memory.
// With dipoles each source contributes two columns (as k_form2d_mma):
// (hx, q hy + v2 dhy) and (v1 dhx, hy), dh_j = sqrt(j) dsq h_(j-1).
__global__ void __launch_bounds__(256) k_form2d(KP k, const FormTask* __restrict__ tasks,
                                                const double* __restrict__ isq, int ch) {
  const FormTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  const int Pn = T.p + 1, n2 = k.n2, npw = k.npw;
  const int tpd = (Pn + 3) >> 2, Pp = tpd * 4, ntiles = tpd * tpd;
  const int G = 256 / ntiles;
  extern __shared__ double sm[];
  double* xs = sm;                     // [ch][Pp]
  double* ys = xs + ch * Pp;           // [ch][Pp]
  double* part = ys + ch * Pp;         // [G][Pp*Pp]
  double* H = part;                    // reduced H overwrites group 0
  double2* px = reinterpret_cast<double2*>(part + G * Pp * Pp);  // [Pn][n2]
  const double cx = k.centers[2 * T.box], cy = k.centers[2 * T.box + 1];
  const int tid = threadIdx.x, tile = tid % ntiles, g = tid / ntiles;
  const int jb = (tile % tpd) * 4, kb = (tile / tpd) * 4;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
  const int vc = k.ifdipole ? 2 : 1;     // columns per source
  const int chs = k.ifdipole ? ch / 2 : ch;  // sources per chunk
  for (int s0c = 0; s0c < T.n; s0c += chs) {
    const int ms = min(chs, T.n - s0c), m = vc * ms;
    for (int r = tid; r < 2 * m; r += 256) {
      const int t = r >> 1, kind = r & 1;
      const int i = T.s0 + s0c + t / vc;
      const double v = kind == 0 ? (k.src[2 * i] - cx) * k.dsq : (k.src[2 * i + 1] - cy) * k.dsq;
      double* row = (kind ? ys : xs) + t * Pp;
      if (!k.ifdipole) {
        double w = kind == 0 ? 1.0 : k.chg[(size_t)i * k.nd + ind];
        row[0] = w;
        for (int j = 1; j < Pn; j++) {
          w = w * v * isq[j];
          row[j] = w;
        }
      } else {
        // a h_j + b dh_j for the column's factor
        double dv[2];
        src_dipole<2>(k, i, ind, dv);
        const bool c1 = t & 1;
        double a, b;
        if (kind == 0) { a = c1 ? 0.0 : 1.0; b = c1 ? dv[0] : 0.0; }
        else { a = c1 ? 1.0 : src_charge(k, i, ind); b = c1 ? 0.0 : dv[1]; }
        double h = 1.0;
        row[0] = a;
        for (int j = 1; j < Pn; j++) {
          const double dh = j * isq[j] * k.dsq * h;
          h = h * v * isq[j];
          row[j] = fma(a, h, b * dh);
        }
      }
      for (int j = Pn; j < Pp; j++) row[j] = 0.0;
    }
    __syncthreads();
    if (g < G) {
      for (int t = g; t < m; t += G) {
        const double2 x01 = *reinterpret_cast<const double2*>(xs + t * Pp + jb);
        const double2 x23 = *reinterpret_cast<const double2*>(xs + t * Pp + jb + 2);
        const double2 y01 = *reinterpret_cast<const double2*>(ys + t * Pp + kb);
        const double2 y23 = *reinterpret_cast<const double2*>(ys + t * Pp + kb + 2);
        const double xa[4] = {x01.x, x01.y, x23.x, x23.y};
        const double ya[4] = {y01.x, y01.y, y23.x, y23.y};
#pragma unroll
        for (int b = 0; b < 4; b++)
#pragma unroll
          for (int a = 0; a < 4; a++) acc[a][b] = fma(ya[b], xa[a], acc[a][b]);
      }
    }
    __syncthreads();
  }
  if (g < G) {
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) part[g * Pp * Pp + (jb + a) + Pp * (kb + b)] = acc[a][b];
  }
  __syncthreads();
  for (int e = tid; e < Pp * Pp; e += 256) {
    double v = 0.0;
    for (int q = 0; q < G; q++) v += part[q * Pp * Pp + e];
    H[e] = v;  // element e is read and written by this thread only
  }
  __syncthreads();
  // x pass: px[j2][k2] = sum_j1 h2x(j1,k2) i^j1 H[j1][j2], k2 over the positive half
  for (int idx = tid; idx < Pn * n2; idx += 256) {
    const int j2 = idx / n2, k2 = idx - j2 * n2;
    double2 a = make_double2(0.0, 0.0);
    for (int j1 = 0; j1 < Pn; j1++) addrot(a, k.h2x[j1 * npw + k2] * H[j1 + Pp * j2], j1);
    px[idx] = a;
  }
  __syncthreads();
  // y pass over the full node set, written to the leaf's multipole slot
  double2* out = k.mp + ((size_t)T.slot * k.nd + ind) * k.nexp;
  for (int e = tid; e < k.nexp; e += 256) {
    const int k1 = e / n2, k2 = e - k1 * n2;
    double2 a = make_double2(0.0, 0.0);
    for (int j2 = 0; j2 < Pn; j2++) {
      const double h = k.h2x[j2 * npw + k1];
      const double2 z = rot(px[j2 * n2 + k2], j2);
      a.x = fma(h, z.x, a.x);
      a.y = fma(h, z.y, a.y);
    }
    out[e] = a;
  }
}

// ------------------------------------------------------------ (a) form, 3D Hermite
// Persistent CTAs; H (P^3) in shared memory, accumulated by (j,k) pairs with
// the P values of l in registers; the three 1D passes go through this CTA's
// scratch slab in global memory (z pass, y pass, x pass into the slot).
template <int MAXP>
__global__ void __launch_bounds__(256) k_form3d_hermite(KP k, const FormTask* __restrict__ tasks,
                                                        int ntasks, double2* __restrict__ scratch,
                                                        size_t slab, const double* __restrict__ isq) {
  extern __shared__ double sm[];
  const int npw = k.npw, n2 = k.n2;
  double2* T1 = scratch + slab * blockIdx.x;
  for (int w = blockIdx.x; w < ntasks * k.nd; w += gridDim.x) {
    const FormTask T = tasks[w / k.nd];
    const int ind = w % k.nd;
    const int Pn = T.p + 1, P2 = Pn * Pn, P3 = P2 * Pn;
    double* H = sm;
    double* X = H + P3;
    double* Y = X + FORM_CH * Pn;
    double* Z = Y + FORM_CH * Pn;
    const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1],
                 cz = k.centers[3 * T.box + 2];
    for (int e = threadIdx.x; e < P3; e += blockDim.x) H[e] = 0.0;
    __syncthreads();
    // dipoles: three columns per source (dip3_coef), 10 sources per chunk
    const int vc = k.ifdipole ? 3 : 1, chs = FORM_CH / vc;
    for (int c0 = 0; c0 < T.n; c0 += chs) {
      const int m = vc * min(chs, T.n - c0);
      if (threadIdx.x < m) {
        const int i = T.s0 + c0 + threadIdx.x / vc;
        const double x = (k.src[3 * i] - cx) * k.dsq, y = (k.src[3 * i + 1] - cy) * k.dsq,
                     z = (k.src[3 * i + 2] - cz) * k.dsq;
        double* xr = X + threadIdx.x * Pn;
        double* yr = Y + threadIdx.x * Pn;
        double* zr = Z + threadIdx.x * Pn;
        if (!k.ifdipole) {
          double xv = 1.0, yv = 1.0, zv = k.chg[(size_t)i * k.nd + ind];
          xr[0] = xv; yr[0] = yv; zr[0] = zv;
          for (int j = 1; j < Pn; j++) {
            double sj = sqrt((double)j);
            xv = xv * x / sj; yv = yv * y / sj; zv = zv * z / sj;
            xr[j] = xv; yr[j] = yv; zr[j] = zv;
          }
        } else {
          double dv[3], a, b;
          src_dipole<3>(k, i, ind, dv);
          const double q = src_charge(k, i, ind), cv[3] = {x, y, z};
          double* rows[3] = {xr, yr, zr};
          for (int d = 0; d < 3; d++) {
            dip3_coef(threadIdx.x % vc, d, q, dv, a, b);
            dip_row(rows[d], 1, Pn, cv[d], a, b, k.dsq, isq);
          }
        }
      }
      __syncthreads();
      for (int pr = threadIdx.x; pr < P2; pr += blockDim.x) {
        const int j = pr % Pn, kk = pr / Pn;
        double acc[MAXP];
#pragma unroll
        for (int l = 0; l < MAXP; l++) acc[l] = l < Pn ? H[j + Pn * (kk + Pn * l)] : 0.0;
        for (int t = 0; t < m; t++) {
          const double a = X[t * Pn + j] * Y[t * Pn + kk];
          const double* zr = Z + t * Pn;
#pragma unroll
          for (int l = 0; l < MAXP; l++)
            if (l < Pn) acc[l] = fma(a, zr[l], acc[l]);
        }
#pragma unroll
        for (int l = 0; l < MAXP; l++)
          if (l < Pn) H[j + Pn * (kk + Pn * l)] = acc[l];
      }
      __syncthreads();
    }
    // z pass: T1[(j3 + P j2) n2 + k1] = sum_j1 A(j1,k1) i^j1 H[j3 + P(j2 + P j1)]
    // (k1 over the first half of the ascending 3D nodes, as pwexp(:,:,npw/2))
    double2* T2 = T1 + (size_t)P2 * n2;
    for (int idx = threadIdx.x; idx < P2 * n2; idx += blockDim.x) {
      const int k1 = idx % n2, jj = idx / n2;
      double2 a = make_double2(0.0, 0.0);
      for (int j1 = 0; j1 < Pn; j1++) addrot(a, k.h2x[j1 * npw + k1] * H[jj + P2 * j1], j1);
      T1[idx] = a;
    }
    __syncthreads();
    // y pass: T2[(j3 npw + k2) n2 + k1] = sum_j2 A(j2,k2) i^j2 T1[(j3 + P j2) n2 + k1]
    for (int idx = threadIdx.x; idx < Pn * npw * n2; idx += blockDim.x) {
      const int k1 = idx % n2, r = idx / n2, k2 = r % npw, j3 = r / npw;
      double2 a = make_double2(0.0, 0.0);
      for (int j2 = 0; j2 < Pn; j2++) {
        const double h = k.h2x[j2 * npw + k2];
        const double2 z = rot(T1[(j3 + Pn * j2) * n2 + k1], j2);
        a.x = fma(h, z.x, a.x);
        a.y = fma(h, z.y, a.y);
      }
      T2[idx] = a;
    }
    __syncthreads();
    // x pass into the slot: pw[k3 + npw (k2 + npw k1)]
    double2* out = k.mp + ((size_t)T.slot * k.nd + ind) * k.nexp;
    for (int e = threadIdx.x; e < k.nexp; e += blockDim.x) {
      const int k3 = e % npw, r = e / npw, k2 = r % npw, k1 = r / npw;
      double2 a = make_double2(0.0, 0.0);
      for (int j3 = 0; j3 < Pn; j3++) {
        const double h = k.h2x[j3 * npw + k3];
        const double2 z = rot(T2[(j3 * npw + k2) * n2 + k1], j3);
        a.x = fma(h, z.x, a.x);
        a.y = fma(h, z.y, a.y);
      }
      out[e] = a;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ (a) form, 2D on FP64 MMA
// Hermite block of a leaf, H[j][k] = sum_t q_t x_t^j y_t^k (g2dformhc_vec,
// g2drouts.f:100-168, without the 1/sqrt(j! k!) factors, which k_h2pw2d
// folds into its tables), on the FP64 tensor cores: mma.sync.m8n8k4.f64 takes
// four sources per step (K = 4) into NT x NT tiles of 8 x 8 (P <= 8 NT).
// Fragment layout (PTX ISA, m8n8k4 .f64): A element (row = lane/4, col =
// lane%4), B element (row = lane%4, col = lane/4), accumulator pair (row =
// lane/4, col = 2 (lane%4) + i).  The powers x^j and q y^j of a block of 32
// sources are built once per source (one lane each) in a per-warp
// shared-memory stage laid out [j][source] with a row stride of 36 doubles, so
// each fragment load is two conflict-free wavefronts.  Four warps split the
// leaf's sources; their tiles are summed in shared memory and the P x P block
// goes to the leaf's slot of the Hermite buffer.
__device__ __forceinline__ void dmma_884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Leading dimensions (in doubles) of zero-padded shared-memory operands of
// the m8n8k4 FP64 MMA: an A operand with K columns is stored with a stride of
// 4 (mod 16) and a B operand with N columns with a stride of 8 (mod 16), so
// the eight rows (A) or four rows (B) that a fragment load touches fall in
// distinct bank pairs: two wavefronts per load, the minimum for 256 bytes.
__host__ __device__ __forceinline__ int mma_lda(int K) { return K <= 4 ? 4 : ((K + 11) & ~15) + 4; }
__host__ __device__ __forceinline__ int mma_ldb(int N) { return ((N + 7) & ~15) + 8; }

// Warp-level C = A B (+ C2 = A2 B2 on the same tiles when TWO) on the FP64
// MMA with row-major, zero-padded operands in shared memory: A is
// (8 Mt) x (4 Ks), B is (4 Ks) x (8 Nt).  out(i, j, c0, c1 [, d0, d1])
// receives row i, columns j and j + 1 (j even) of C (and C2).  Two
// accumulator sets alternate over the K steps.
template <bool TWO, class Out>
__device__ __forceinline__ void warp_gemm(const double* A, int lda, const double* B, int ldb,
                                          const double* A2, const double* B2, int Mt, int Nt, int Ks,
                                          Out out) {
  const int lane = threadIdx.x & 31, r = lane >> 2, c = lane & 3;
  for (int mt = 0; mt < Mt; mt++)
  for (int nt = 0; nt < Nt; nt++) {
    const int ao = (8 * mt + r) * lda + c, bo = c * ldb + 8 * nt + r;
    double d0 = 0.0, d1 = 0.0, e0 = 0.0, e1 = 0.0;
    double f0 = 0.0, f1 = 0.0, g0 = 0.0, g1 = 0.0;
    for (int ks = 0; ks < Ks; ks++) {
      const int ak = ao + 4 * ks, bk = bo + 4 * ks * ldb;
      if (ks & 1) {
        dmma_884(e0, e1, A[ak], B[bk]);
        if (TWO) dmma_884(g0, g1, A2[ak], B2[bk]);
      } else {
        dmma_884(d0, d1, A[ak], B[bk]);
        if (TWO) dmma_884(f0, f1, A2[ak], B2[bk]);
      }
    }
    if (TWO) out(8 * mt + r, 8 * nt + 2 * c, d0 + e0, d1 + e1, f0 + g0, f1 + g1);
    else out(8 * mt + r, 8 * nt + 2 * c, d0 + e0, d1 + e1, 0.0, 0.0);
  }
}

// With dipoles (DIP) the source derivative enters as a second column per
// source (g2dformhd_vec / g2dformhcd_vec, g2drouts.f:173-338; in the
// unnormalised powers here d/dX x^j = j dsq x^(j-1)):
//   column 0: X = x^j,               Y = q y^k + v2 k dsq y^(k-1)
//   column 1: X = v1 j dsq x^(j-1),  Y = y^k
// (v = dipstr * n), so a block of 32 columns holds 16 sources.
template <int NT, bool DIP>
__global__ void __launch_bounds__(128) k_form2d_mma(KP k, const FormTask* __restrict__ tasks,
                                                    const long long* __restrict__ hoff,
                                                    double* __restrict__ hbuf) {
  constexpr int PP = 8 * NT, SW = 36, WS = 2 * PP * SW;  // per-warp staging [2][PP][SW]
  const FormTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  const int Pn = T.p + 1;
  extern __shared__ double smf[];
  double* stg = smf;                                          // [4][WS]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double cx = k.centers[2 * T.box], cy = k.centers[2 * T.box + 1];
  const int j0 = lane >> 2, tl = lane & 3;
  double* X = stg + warp * WS;  // X[j][s] = x_s^j, Y[j][s] = q_s y_s^j
  double* Y = X + PP * SW;
  double c[2][NT][NT][2];
#pragma unroll
  for (int h = 0; h < 2; h++)
#pragma unroll
    for (int a = 0; a < NT; a++)
#pragma unroll
      for (int b = 0; b < NT; b++) c[h][a][b][0] = c[h][a][b][1] = 0.0;
  // each warp takes blocks of 32 sources in turn: every lane builds the
  // powers of one source in shared memory, then the warp runs up to eight
  // K = 4 steps of the FP64 MMA over the block, alternating two accumulator
  // sets so consecutive steps are independent
  constexpr int SPB = DIP ? 16 : 32;  // sources per 32-column block
  for (int base = SPB * warp; base < T.n; base += 4 * SPB) {
    const int sl = DIP ? lane >> 1 : lane;
    double x = 0.0, y = 0.0, q = 0.0, v[2] = {0.0, 0.0};
    if (base + sl < T.n) {
      const int i = T.s0 + base + sl;
      const double2 pt = reinterpret_cast<const double2*>(k.src)[i];
      x = (pt.x - cx) * k.dsq;
      y = (pt.y - cy) * k.dsq;
      if (DIP) {
        q = src_charge(k, i, ind);
        src_dipole<2>(k, i, ind, v);
      } else {
        q = k.chg[(size_t)i * k.nd + ind];
      }
    }
    if (!DIP) {
      double xp = 1.0, yp = q;
#pragma unroll
      for (int j = 0; j < PP; j++) {
        X[j * SW + lane] = xp;
        Y[j * SW + lane] = yp;
        xp *= x;
        yp *= y;
      }
    } else {
      // column (lane & 1): powers and their derivatives, one pass
      const bool c1 = lane & 1;
      const double ax = c1 ? 0.0 : 1.0, bx = c1 ? v[0] * k.dsq : 0.0;
      const double ay = c1 ? 1.0 : q, by = c1 ? 0.0 : v[1] * k.dsq;
      double xp = 1.0, yp = 1.0, xm = 0.0, ym = 0.0;  // x^j, j x^(j-1)
#pragma unroll
      for (int j = 0; j < PP; j++) {
        X[j * SW + lane] = fma(ax, xp, bx * xm);
        Y[j * SW + lane] = fma(ay, yp, by * ym);
        xm = fma(xm, x, xp);  // (j+1) x^j = j x^(j-1) x + x^j
        ym = fma(ym, y, yp);
        xp *= x;
        yp *= y;
      }
    }
    __syncwarp();
    const int ncol = DIP ? 2 * min(SPB, T.n - base) : T.n - base;
    const int nst = min(8, (ncol + 3) >> 2);
    for (int st = 0; st < nst; st += 2) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        if (st + h < nst) {
          const int col = 4 * (st + h) + tl;
          double av[NT], bv[NT];
#pragma unroll
          for (int a = 0; a < NT; a++) {
            av[a] = X[(8 * a + j0) * SW + col];
            bv[a] = Y[(8 * a + j0) * SW + col];
          }
#pragma unroll
          for (int a = 0; a < NT; a++)
#pragma unroll
            for (int b = 0; b < NT; b++) dmma_884(c[h][a][b][0], c[h][a][b][1], av[a], bv[b]);
        }
      }
    }
    __syncwarp();
  }
  // tile (a, b) holds H'[j = 8a + lane/4][k = 8b + 2 (lane%4) + i]; each warp
  // writes its sum into its own staging area, then the four are added and
  // the leaf's P x P block is stored row-major (x power j, y power k)
  double* part = X;
#pragma unroll
  for (int a = 0; a < NT; a++)
#pragma unroll
    for (int b = 0; b < NT; b++)
#pragma unroll
      for (int i = 0; i < 2; i++)
        part[(8 * a + j0) + PP * (8 * b + 2 * tl + i)] = c[0][a][b][i] + c[1][a][b][i];
  __syncthreads();
  double* hb = hbuf + hoff[blockIdx.x] + (size_t)ind * Pn * Pn;
  for (int e = threadIdx.x; e < Pn * Pn; e += 128) {
    const int j = e / Pn, kk = e - j * Pn, f = j + PP * kk;
    hb[e] = stg[f] + stg[WS + f] + stg[2 * WS + f] + stg[3 * WS + f];
  }
}

// Hermite -> plane wave (g2dh2pw_real_vec, g2drouts.f:1242-1329), one warp
// per leaf, the two 1D passes on the leaf's P x P block H[j1][j2] as FP64 MMA
// products:
//   px[k2][j2]  = sum_j1 i^j1 hx[j1][k2] H[j1][j2]           (pass 1)
//   pw[k1][k2]  = sum_j2 hx[j2][k1] (i^j2 px[k2][j2])         (pass 2)
// with hx[j][k] = h2x[j][k] / sqrt(j!).  Pass 1 splits i^j1 by parity: the even
// rows of H give Re px and the odd rows Im px, through the table signed by
// (j mod 4 < 2 ? + : -), so it is two real products on the same tiles.  Pass 2
// is one real product with B[j2][2 k2 + c] = component c of i^j2 px[k2][j2].
// The tables are shared by the CTA's warps (all leaves of a launch have one
// order); operands are zero padded to whole tiles.
struct H2pwDims {
  int Pn, Ph, Mp, Kp, Np, Kq, Nq, Mq;  // see k_h2pw2d
  int ldS, ldH, ldP, ldU;
  int tab, warp;  // doubles: CTA tables, per-warp area
  __host__ __device__ H2pwDims(int P, int npw) {
    const int n2 = npw / 2;
    Pn = P;
    Ph = (Pn + 1) / 2;
    Mp = (n2 + 7) & ~7;     // pass 1 rows: k2
    Kp = (Ph + 3) & ~3;     // pass 1 depth: j1 of one parity
    Np = (Pn + 7) & ~7;     // pass 1 columns: j2 (also the rows of the pass 2 operand)
    Kq = (Pn + 3) & ~3;     // pass 2 depth: j2
    Nq = (npw + 7) & ~7;    // pass 2 columns: (k2, re/im)
    Mq = (npw + 7) & ~7;    // pass 2 rows: k1
    ldS = mma_lda(Kp);
    ldH = mma_ldb(Np);
    ldP = mma_ldb(Nq > 2 * Mp ? Nq : 2 * Mp);
    ldU = mma_lda(Kq);
    tab = 2 * Mp * ldS + Mq * ldU;
    warp = Np * ldP;
  }
};

// Tables of k_h2pw2d for order P (built on the host, copied to shared
// memory): HSe[k2][i] = s(2i) hx[2i][k2], HSo[k2][i] = s(2i+1) hx[2i+1][k2]
// with s(j) = (j mod 4 < 2 ? 1 : -1), and HUT[k1][j2] = hx[j2][k1].
void build_h2pw_table(const HostPlan& H, int Pn, std::vector<double>& out) {
  const int npw = H.P.npw, n2 = npw / 2;
  const H2pwDims Z(Pn, npw);
  std::vector<double> cf(Pn + 1, 1.0);
  for (int j = 1; j <= Pn; j++) cf[j] = cf[j - 1] / std::sqrt((double)j);
  auto hx = [&](int j, int kk) { return H.h2x[(size_t)j * npw + kk] * cf[j]; };
  const size_t base = out.size();
  out.resize(base + Z.tab, 0.0);
  double* HSe = out.data() + base;
  double* HSo = HSe + Z.Mp * Z.ldS;
  double* HUT = HSo + Z.Mp * Z.ldS;
  for (int k2 = 0; k2 < n2; k2++)
    for (int i = 0; 2 * i < Pn; i++) {
      const int je = 2 * i, jo = 2 * i + 1;
      HSe[k2 * Z.ldS + i] = (je & 2) ? -hx(je, k2) : hx(je, k2);
      if (jo < Pn) HSo[k2 * Z.ldS + i] = (jo & 2) ? -hx(jo, k2) : hx(jo, k2);
    }
  for (int k1 = 0; k1 < npw; k1++)
    for (int j2 = 0; j2 < Pn; j2++) HUT[k1 * Z.ldU + j2] = hx(j2, k1);
}

template <int KQ>  // pass 2 depth in steps of 4: KQ = ceil(P / 4)
__global__ void __launch_bounds__(128) k_h2pw2d(KP k, const FormTask* __restrict__ tasks, int ntask,
                                                const long long* __restrict__ hoff,
                                                const double* __restrict__ hbuf,
                                                const double* __restrict__ tab) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int t = blockIdx.x * 4 + warp;
  if (t >= ntask) return;  // no CTA-wide barrier in this kernel
  const FormTask T = tasks[t];
  const int npw = k.npw, n2 = k.n2;
  const H2pwDims Z(T.p + 1, npw);
  const int Pn = Z.Pn;
  extern __shared__ double sh2[];
  double* PB = sh2 + warp * Z.Np * Z.ldP;    // [Np][ldP]
  const double* HSe = tab;                   // [Mp][ldS], read through L1
  const double* HSo = HSe + Z.Mp * Z.ldS;    // [Mp][ldS]
  const double* HUT = HSo + Z.Mp * Z.ldS;    // [Mq][ldU]
  const int ind = blockIdx.y;
  const double* H = hbuf + hoff[t] + (size_t)ind * Pn * Pn;
  const int r = lane >> 2, c = lane & 3;
  // pass 1: (Re, Im) px[k2][j2] on the same tiles, B operands He[i][j2] =
  // H[2i][j2] and Ho[i][j2] = H[2i+1][j2] read straight from the block;
  // PB[j2][2 k2 + c] = i^j2 px (padded rows and columns come out zero)
  for (int nt = 0; nt < Z.Np / 8; nt++) {
    const int j2b = 8 * nt + r;
    for (int mt = 0; mt < Z.Mp / 8; mt++) {
      const double* ae = HSe + (8 * mt + r) * Z.ldS + c;
      const double* ao = HSo + (8 * mt + r) * Z.ldS + c;
      double re0 = 0.0, re1 = 0.0, im0 = 0.0, im1 = 0.0;
      for (int ks = 0; ks < Z.Kp / 4; ks++) {
        const int i = 4 * ks + c, je = 2 * i, jo = 2 * i + 1;
        const double be = (je < Pn && j2b < Pn) ? __ldg(H + je * Pn + j2b) : 0.0;
        const double bo = (jo < Pn && j2b < Pn) ? __ldg(H + jo * Pn + j2b) : 0.0;
        dmma_884(re0, re1, __ldg(ae + 4 * ks), be);
        dmma_884(im0, im1, __ldg(ao + 4 * ks), bo);
      }
      const int k2 = 8 * mt + r, j2 = 8 * nt + 2 * c;
      const double2 z0 = rot_bf(make_double2(re0, im0), j2);
      const double2 z1 = rot_bf(make_double2(re1, im1), j2 + 1);
      PB[j2 * Z.ldP + 2 * k2] = z0.x;
      PB[j2 * Z.ldP + 2 * k2 + 1] = z0.y;
      PB[(j2 + 1) * Z.ldP + 2 * k2] = z1.x;
      PB[(j2 + 1) * Z.ldP + 2 * k2 + 1] = z1.y;
    }
  }
  __syncwarp();
  // pass 2: pw[k1][k2] = sum_j2 hx[j2][k1] PB[j2][(k2, c)]
  double2* out = k.mp + ((size_t)T.slot * k.nd + ind) * k.nexp;
  for (int mt = 0; mt < Z.Mq / 8; mt++) {
    const double* ap = HUT + (8 * mt + r) * Z.ldU + c;
    double a[KQ];
#pragma unroll
    for (int ks = 0; ks < KQ; ks++) a[ks] = __ldg(ap + 4 * ks);
    for (int nt = 0; nt < Z.Nq / 8; nt++) {
      const double* bp = PB + c * Z.ldP + 8 * nt + r;
      double d0 = 0.0, d1 = 0.0, e0 = 0.0, e1 = 0.0;
#pragma unroll
      for (int ks = 0; ks < KQ; ks++) {
        if (ks & 1) dmma_884(e0, e1, a[ks], bp[4 * ks * Z.ldP]);
        else dmma_884(d0, d1, a[ks], bp[4 * ks * Z.ldP]);
      }
      const int k1 = 8 * mt + r, n = 8 * nt + 2 * c;
      if (k1 < npw && n < npw) out[k1 * n2 + (n >> 1)] = make_double2(d0 + e0, d1 + e1);
    }
  }
}

// ------------------------------------------------------------ (a) form, 3D, two kernels
// Kernel A: one CTA per chunk of <= FORM3_CHK sources of a leaf; the chunk's
// Hermite block H[j + P (k + P l)] (g3dformhc_vec, g3drouts.f:109-192) is
// accumulated in shared memory -- each thread owns (j,k) pairs and keeps the
// P values of l in registers -- and written to its slot of the partial buffer.
// Kernel B: one CTA per leaf sums the leaf's partial blocks in chunk order
// (deterministic) and runs the separable Hermite -> plane-wave transform
// (g3dh2pw_real_vec, g3drouts.f:1565-1685) in shared memory: z pass over the
// stored half, then y and x passes over the positive half using the mirror
// symmetry A(j, mirror k) = (-1)^j A(j, k) of the ascending node set.

// The chunk's Hermite block on the FP64 tensor cores: H[j][(k, l)] =
// sum_t x_t^j (q_t y_t^k z_t^l) (with the 1/sqrt(j!) factors, g3dformhc_vec,
// g3drouts.f:109-192) is one product with M = j (MT tiles of 8), N = the
// P^2 pairs (k, l) and K = the sources, four per mma.m8n8k4 step.  Sources
// are staged 64 at a time as power rows in shared memory (row stride 68: the
// A fragments are conflict-free); a B element is y^k q z^l, one multiply of
// two staged powers, with (k, l) of the lane's column fixed per tile.  The
// eight warps split the N tiles (up to four each per pass over the sources).
// The partial block goes to the chunk's slot of the Hermite buffer, laid out
// H[j + P (k + P l)] as k_form3d_h2pw reads it.
// With dipoles (DIP) every source stages three columns (dip3_coef), 21
// sources (63 columns) per batch.
template <int MT, bool DIP>
__global__ void __launch_bounds__(256) k_form3d_mma(KP k, const FormTask* __restrict__ tasks,
                                                    const FormChunk* __restrict__ chunks,
                                                    double* __restrict__ hbuf, const double* __restrict__ isq) {
  constexpr int SB = 64, SW = 68, NTW = 4;
  constexpr int VC = DIP ? 3 : 1, SBS = SB / VC;  // columns per source, sources per batch
  const FormChunk C = chunks[blockIdx.x];
  const FormTask T = tasks[C.task];
  const int ind = blockIdx.y;
  const int Pn = T.p + 1, P2 = Pn * Pn, P3 = P2 * Pn, ntiles = (P2 + 7) / 8;
  extern __shared__ double sm[];
  double* X = sm;                // [8 MT][SW]
  double* Y = X + 8 * MT * SW;   // [Pn][SW]
  double* Z = Y + Pn * SW;       // [Pn][SW], times q
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, r = lane >> 2, c = lane & 3;
  const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1], cz = k.centers[3 * T.box + 2];
  for (int e = threadIdx.x; e < (8 * MT - Pn) * SW; e += blockDim.x) X[Pn * SW + e] = 0.0;
  double* out = hbuf + ((size_t)C.hoff * k.nd + (size_t)ind * P3);
  for (int base = 0; base < ntiles; base += 8 * NTW) {
    double acc[MT][NTW][2];
    int ko[NTW], lo_[NTW];
#pragma unroll
    for (int i = 0; i < NTW; i++) {
      const int n = 8 * (base + warp + 8 * i) + r;
      ko[i] = n < P2 ? (n % Pn) * SW : -1;
      lo_[i] = n < P2 ? (n / Pn) * SW : 0;
#pragma unroll
      for (int mt = 0; mt < MT; mt++) acc[mt][i][0] = acc[mt][i][1] = 0.0;
    }
    for (int c0 = 0; c0 < C.n; c0 += SBS) {
      const int m = VC * min(SBS, C.n - c0);
      __syncthreads();
      for (int job = threadIdx.x; job < 3 * SB; job += blockDim.x) {
        const int t = job / 3, d = job - 3 * t;
        double* row = (d == 0 ? X : d == 1 ? Y : Z) + t;
        if (!DIP) {
          double v = 0.0, w = 0.0;
          if (t < m) {
            const int i = C.s0 + c0 + t;
            v = (k.src[3 * i + d] - (d == 0 ? cx : d == 1 ? cy : cz)) * k.dsq;
            w = d == 2 ? k.chg[(size_t)i * k.nd + ind] : 1.0;
          }
          row[0] = w;
          for (int j = 1; j < Pn; j++) {
            w = w * v * isq[j];
            row[j * SW] = w;
          }
        } else {
          double v = 0.0, a = 0.0, b = 0.0;
          if (t < m) {
            const int i = C.s0 + c0 + t / VC;
            v = (k.src[3 * i + d] - (d == 0 ? cx : d == 1 ? cy : cz)) * k.dsq;
            double dv[3];
            src_dipole<3>(k, i, ind, dv);
            dip3_coef(t % VC, d, src_charge(k, i, ind), dv, a, b);
          }
          dip_row(row, SW, Pn, v, a, b, k.dsq, isq);
        }
      }
      __syncthreads();
      const int nst = (m + 3) >> 2;
      for (int st = 0; st < nst; st++) {
        const int s = 4 * st + c;
        double a[MT];
#pragma unroll
        for (int mt = 0; mt < MT; mt++) a[mt] = X[(8 * mt + r) * SW + s];
#pragma unroll
        for (int i = 0; i < NTW; i++) {
          if (base + warp + 8 * i < ntiles) {
            const double b = ko[i] >= 0 ? Y[ko[i] + s] * Z[lo_[i] + s] : 0.0;
#pragma unroll
            for (int mt = 0; mt < MT; mt++) dmma_884(acc[mt][i][0], acc[mt][i][1], a[mt], b);
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < NTW; i++) {
      const int nt = base + warp + 8 * i;
      if (nt >= ntiles) continue;
#pragma unroll
      for (int mt = 0; mt < MT; mt++) {
        const int j = 8 * mt + r;
#pragma unroll
        for (int ii = 0; ii < 2; ii++) {
          const int n = 8 * nt + 2 * c + ii;
          if (j < Pn && n < P2) out[j + Pn * n] = acc[mt][i][ii];
        }
      }
    }
  }
}

__global__ void __launch_bounds__(512) k_form3d_h2pw(KP k, const FormTask* __restrict__ tasks,
                                                     const int* __restrict__ cbeg,
                                                     const FormChunk* __restrict__ chunks,
                                                     const double* __restrict__ hbuf) {
  const int tk = blockIdx.x, ind = blockIdx.y;
  const FormTask T = tasks[tk];
  const int npw = k.npw, n2 = k.n2;
  const int Pn = T.p + 1, P2 = Pn * Pn, P3 = P2 * Pn;
  extern __shared__ double sm[];
  // region A: H, later T2 [(j3 npw + k2) n2 + k1]; region B: T1 [(j3 + P j2) n2 + k1];
  // then the signed table hs[j][k] = h2x[j][k] (j mod 4 < 2 ? 1 : -1).  The
  // factor i^j of each pass is then a sign (in hs) times 1 (even j) or i
  // (odd j): even and odd j are summed apart, E + i O, and the mirror node
  // of k (A(j, mirror k) = (-1)^j A(j, k)) gets E - i O.
  const size_t szA = max((size_t)P3, (size_t)2 * Pn * npw * n2);
  double* H = sm;
  double2* T2 = reinterpret_cast<double2*>(sm);
  double2* T1 = reinterpret_cast<double2*>(sm + ((szA + 1) & ~size_t(1)));
  double* hs = reinterpret_cast<double*>(T1 + (size_t)P2 * n2);
  for (int e = threadIdx.x; e < Pn * npw; e += blockDim.x) {
    const int j = e / npw;
    hs[e] = (j & 2) ? -k.h2x[e] : k.h2x[e];
  }
  for (int e = threadIdx.x; e < P3; e += blockDim.x) {
    double v = 0.0;
    for (int c = cbeg[tk]; c < cbeg[tk + 1]; c++) v += hbuf[(size_t)chunks[c].hoff * k.nd + (size_t)ind * P3 + e];
    H[e] = v;
  }
  __syncthreads();
  // z pass over the stored half (the first n2 ascending nodes)
  for (int idx = threadIdx.x; idx < P2 * n2; idx += blockDim.x) {
    const int k1 = idx % n2, jj = idx / n2;
    double ev = 0.0, od = 0.0;
    int j1 = 0;
    for (; j1 + 1 < Pn; j1 += 2) {
      ev = fma(hs[j1 * npw + k1], H[jj + P2 * j1], ev);
      od = fma(hs[(j1 + 1) * npw + k1], H[jj + P2 * (j1 + 1)], od);
    }
    if (j1 < Pn) ev = fma(hs[j1 * npw + k1], H[jj + P2 * j1], ev);
    T1[idx] = make_double2(ev, od);
  }
  __syncthreads();
  // y pass over the positive half k2 = n2 + m and its mirror n2 - 1 - m
  for (int idx = threadIdx.x; idx < Pn * n2 * n2; idx += blockDim.x) {
    const int k1 = idx % n2, r = idx / n2, m = r % n2, j3 = r / n2;
    const int kp = n2 + m, km = n2 - 1 - m;
    double2 E = make_double2(0.0, 0.0), O = make_double2(0.0, 0.0);
    const double2* zc = T1 + (size_t)j3 * n2 + k1;
    int j2 = 0;
    for (; j2 + 1 < Pn; j2 += 2) {
      const double he = hs[j2 * npw + kp], ho = hs[(j2 + 1) * npw + kp];
      const double2 ze = zc[(size_t)Pn * j2 * n2], zo = zc[(size_t)Pn * (j2 + 1) * n2];
      E.x = fma(he, ze.x, E.x);
      E.y = fma(he, ze.y, E.y);
      O.x = fma(ho, zo.x, O.x);
      O.y = fma(ho, zo.y, O.y);
    }
    if (j2 < Pn) {
      const double he = hs[j2 * npw + kp];
      const double2 ze = zc[(size_t)Pn * j2 * n2];
      E.x = fma(he, ze.x, E.x);
      E.y = fma(he, ze.y, E.y);
    }
    T2[((size_t)j3 * npw + kp) * n2 + k1] = make_double2(E.x - O.y, E.y + O.x);
    T2[((size_t)j3 * npw + km) * n2 + k1] = make_double2(E.x + O.y, E.y - O.x);
  }
  __syncthreads();
  double2* out = k.mp + ((size_t)T.slot * k.nd + ind) * k.nexp;
  // x pass into the slot, positive half k3 = n2 + m and mirror
  for (int idx = threadIdx.x; idx < n2 * npw * n2; idx += blockDim.x) {
    const int m = idx % n2, r = idx / n2, k2 = r % npw, k1 = r / npw;
    const int kp = n2 + m, km = n2 - 1 - m;
    double2 E = make_double2(0.0, 0.0), O = make_double2(0.0, 0.0);
    const double2* zc = T2 + (size_t)k2 * n2 + k1;
    const size_t zs = (size_t)npw * n2;
    int j3 = 0;
    for (; j3 + 1 < Pn; j3 += 2) {
      const double he = hs[j3 * npw + kp], ho = hs[(j3 + 1) * npw + kp];
      const double2 ze = zc[zs * j3], zo = zc[zs * (j3 + 1)];
      E.x = fma(he, ze.x, E.x);
      E.y = fma(he, ze.y, E.y);
      O.x = fma(ho, zo.x, O.x);
      O.y = fma(ho, zo.y, O.y);
    }
    if (j3 < Pn) {
      const double he = hs[j3 * npw + kp];
      const double2 ze = zc[zs * j3];
      E.x = fma(he, ze.x, E.x);
      E.y = fma(he, ze.y, E.y);
    }
    const size_t base = (size_t)npw * (k2 + (size_t)npw * k1);
    out[base + kp] = make_double2(E.x - O.y, E.y + O.x);
    out[base + km] = make_double2(E.x + O.y, E.y - O.x);
  }
}

// k_form3d_h2pw_mma: the transform of k_form3d_h2pw with its three passes on
// the FP64 tensor cores.  Each pass is a real product against the signed node
// table hs, the even and odd j in separate k-steps so that i^j becomes E + i O
// and the mirror node gets E - i O from the same accumulators (K = j, KS
// k-steps of 4 per parity):
//   z pass  E/O[m][kz]   = sum_l  H[m][l] hs[l][kz],        m = jx + P jy, kz < n2
//           -> T1[jy][(jx, kz)] = E + i O                    (M = P^2, N = n2)
//   y pass  E/O[m][col]  = sum_jy hs[jy][n2 + m] T1[jy][col], col = (jx, kz, re/im)
//           -> T2[jx][(ky, kz)], ky = n2 + m and n2 - 1 - m  (M = n2, N = 2 P n2)
//   x pass  E/O[m][col]  = sum_jx hs[jx][n2 + m] T2[jx][col], col = (ky, kz, re/im)
//           -> the slot, kx = n2 + m and n2 - 1 - m          (M = n2, N = 2 npw n2)
// The y and x passes run per 8-row tile t of the node half: the y pass of tile
// t fills T2 with its 16 ky and the x pass of tile t drains it, so T2 holds 16
// ky instead of npw.  The node tables are register fragments, loaded once per
// CTA (a launch covers one order); rows j >= P are zero fragments, not loads.
// Row strides are 4 (mod 8) doubles, so the rows two apart that one fragment
// reads fall in opposite halves of the banks.  Persistent CTAs of 8 warps, two
// per SM at the orders of eps >= 1e-6, stride over the leaves of the order
// group; where shared memory allows, the next leaf's Hermite block is copied
// into its own buffer with cp.async while the y and x passes of the current
// leaf run (else it is staged over T2 at the leaf's start).  Each warp takes
// two N tiles per step (independent accumulator chains in flight).
struct H3Dims {
  int ldh, ld1, ld2;
  size_t total_pf, total_ov;  // doubles: H in its own buffer (prefetched) / H over T2
  __host__ __device__ H3Dims(int Pn, int n2) {
    ldh = ((Pn * Pn + 3) & ~7) + 4;
    ld1 = 8 * ((2 * Pn * n2 + 7) / 8) + 4;
    ld2 = 32 * n2 + 4;
    total_pf = (size_t)Pn * (ld1 + ld2 + ldh) + 8;
    const size_t t2 = (size_t)Pn * ld2, hb = (size_t)Pn * ldh + 8;
    total_ov = (size_t)Pn * ld1 + (t2 > hb ? t2 : hb);
  }
};

// Stage the Hermite block of task tk (the sum of its chunk partials) into H
// with row stride ldh, row l of P^2 doubles per warp: a single partial block
// by asynchronous copies (16 bytes where the rows allow; waited for by the
// caller), several by plain loads in chunk order.
// The task's chunk range [cb0, cb1) and its first chunk's offset hoff0 are
// loaded by the caller ahead of time.
__device__ __forceinline__ void h2pw_stage(const KP& k, int ind, int Pn, int ldh, int cb0, int cb1, long long hoff0,
                                           const FormChunk* __restrict__ chunks, const double* __restrict__ hbuf,
                                           double* H) {
  const int P2 = Pn * Pn, P3 = P2 * Pn, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (cb1 - cb0 == 1) {
    const double* src = hbuf + (size_t)hoff0 * k.nd + (size_t)ind * P3;
    const unsigned dst = (unsigned)__cvta_generic_to_shared(H);
    if (((P2 | (int)(reinterpret_cast<size_t>(src) >> 3)) & 1) == 0) {
      for (int l = threadIdx.x >> 5; l < Pn; l += nw)
        for (int m = 2 * lane; m < P2; m += 64)
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + 8u * (unsigned)(l * ldh + m)),
                       "l"(src + l * P2 + m) : "memory");
    } else {
      for (int l = threadIdx.x >> 5; l < Pn; l += nw)
        for (int m = lane; m < P2; m += 32)
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst + 8u * (unsigned)(l * ldh + m)),
                       "l"(src + l * P2 + m) : "memory");
    }
  } else {
    for (int l = threadIdx.x >> 5; l < Pn; l += nw)
      for (int m = lane; m < P2; m += 32) {
        double v = 0.0;
        for (int ch = cb0; ch < cb1; ch++) v += hbuf[(size_t)chunks[ch].hoff * k.nd + (size_t)ind * P3 + l * P2 + m];
        H[l * ldh + m] = v;
      }
  }
}

// q / d for 0 <= q < 1115 and 1 <= d <= 64, with mg = ceil(2^16 / d)
__device__ __forceinline__ int div16(int q, int mg) { return (q * mg) >> 16; }

template <int KS, int MT>
__global__ void __launch_bounds__(256, (KS * MT <= 4) ? 2 : 1)
    k_form3d_h2pw_mma(KP k, const FormTask* __restrict__ tasks, int ntask, const int* __restrict__ cbeg,
                      const FormChunk* __restrict__ chunks, const double* __restrict__ hbuf, bool pf) {
  const int ind = blockIdx.y;
  const int npw = k.npw, n2 = k.n2;
  const int Pn = tasks[0].p + 1, P2 = Pn * Pn;
  const int mgP = (65536 + Pn - 1) / Pn, mgN = (65536 + n2 - 1) / n2;  // div16 factors
  const H3Dims Z(Pn, n2);
  extern __shared__ double sm[];
  double* T1 = sm;                       // [Pn][ld1]: (jx, kz, re/im)
  double* T2 = T1 + (size_t)Pn * Z.ld1;  // [Pn][ld2]: (kyl, kz, re/im)
  // H [Pn][ldh] (+ 8: the last M tile's rows past P^2): its own buffer when
  // pf (the next leaf's block is prefetched), else over T2 (staged per leaf)
  double* H = pf ? T2 + (size_t)Pn * Z.ld2 : T2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, r = lane >> 2, c = lane & 3;
  int tk = blockIdx.x;
  if (tk >= ntask) return;
  // chunk range and first partial block of the current task
  int cb0 = cbeg[tk], cb1 = cbeg[tk + 1];
  long long hoff0 = chunks[cb0].hoff;
  if (pf) h2pw_stage(k, ind, Pn, Z.ldh, cb0, cb1, hoff0, chunks, hbuf, H);
  // B fragments of the stored-half table for the z pass (B[k = j][n = kz]) and
  // A fragments of the positive-half table for the y and x passes (A[m][k = j])
  double hz[MT][2][KS], hn[MT][2][KS];
#pragma unroll
  for (int t = 0; t < MT; t++)
#pragma unroll
    for (int par = 0; par < 2; par++)
#pragma unroll
      for (int s = 0; s < KS; s++) {
        const int j = 8 * s + 2 * c + par, m = 8 * t + r;
        const bool ok = j < Pn && m < n2;
        const double sg = (j & 2) ? -1.0 : 1.0;
        hz[t][par][s] = ok ? sg * k.h2x[j * npw + m] : 0.0;
        hn[t][par][s] = ok ? sg * k.h2x[j * npw + n2 + m] : 0.0;
      }
  const int mtiles = (P2 + 7) / 8, nt1 = (2 * Pn * n2 + 7) / 8;
  for (; tk < ntask; tk += gridDim.x) {
    if (!pf) h2pw_stage(k, ind, Pn, Z.ldh, cb0, cb1, hoff0, chunks, hbuf, H);  // T2 is free: the last pass ended in a barrier
    // the next task's chunk range and first block offset, loaded while this one runs
    const int tn = tk + gridDim.x;
    if (tn < ntask) {
      cb0 = cbeg[tn];
      cb1 = cbeg[tn + 1];
      hoff0 = chunks[cb0].hoff;
    }
    const int slot = tasks[tk].slot;
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    // z pass: H -> T1
    for (int mt = warp; mt < mtiles; mt += 8) {
      const int m = 8 * mt + r;
      double a[2][KS];
#pragma unroll
      for (int par = 0; par < 2; par++)
#pragma unroll
        for (int s = 0; s < KS; s++) {
          const int j = 8 * s + 2 * c + par;
          a[par][s] = j < Pn ? H[m + j * Z.ldh] : 0.0;
        }
      const int jy = div16(m, mgP), jx = m - jy * Pn;
#pragma unroll
      for (int t = 0; t < MT; t++) {
        double e0 = 0.0, e1 = 0.0, o0 = 0.0, o1 = 0.0;
#pragma unroll
        for (int s = 0; s < KS; s++) {
          dmma_884(e0, e1, a[0][s], hz[t][0][s]);
          dmma_884(o0, o1, a[1][s], hz[t][1][s]);
        }
        const int kz = 8 * t + 2 * c;  // the lane's accumulator columns kz, kz + 1
        if (m < P2) {
          double* row = T1 + jy * Z.ld1 + 2 * (jx * n2 + kz);
          if (kz < n2) *reinterpret_cast<double2*>(row) = make_double2(e0, o0);
          if (kz + 1 < n2) *reinterpret_cast<double2*>(row + 2) = make_double2(e1, o1);
        }
      }
    }
    __syncthreads();
    // the next leaf's Hermite block lands while this leaf's y and x passes run
    if (pf && tn < ntask) h2pw_stage(k, ind, Pn, Z.ldh, cb0, cb1, hoff0, chunks, hbuf, H);
    double2* out = k.mp + ((size_t)slot * k.nd + ind) * k.nexp;
#pragma unroll
    for (int t = 0; t < MT; t++) {
      const int nv = min(8, n2 - 8 * t);  // node rows of tile t
      // y pass of tile t into T2[jx][(kyl n2 + kz)], kyl = 2 i (ky = n2 + 8t + i) or 2 i + 1 (ky = n2 - 1 - 8t - i)
      for (int nt0 = warp; nt0 < nt1; nt0 += 16) {
        double b[2][2][KS], acc[2][4];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int col = 8 * (nt0 + 8 * h) + r;
          const bool ok = nt0 + 8 * h < nt1;
#pragma unroll
          for (int par = 0; par < 2; par++)
#pragma unroll
            for (int s = 0; s < KS; s++) {
              const int j = 8 * s + 2 * c + par;
              b[h][par][s] = (ok && j < Pn) ? T1[j * Z.ld1 + col] : 0.0;
            }
          acc[h][0] = acc[h][1] = acc[h][2] = acc[h][3] = 0.0;
        }
#pragma unroll
        for (int s = 0; s < KS; s++)
#pragma unroll
          for (int h = 0; h < 2; h++) {
            dmma_884(acc[h][0], acc[h][1], hn[t][0][s], b[h][0][s]);
            dmma_884(acc[h][2], acc[h][3], hn[t][1][s], b[h][1][s]);
          }
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int q = 4 * (nt0 + 8 * h) + c;  // the lane's complex column (jx, kz)
          if (r < nv && q < Pn * n2) {
            const int jx = div16(q, mgN), kz = q - jx * n2;
            double* row = T2 + jx * Z.ld2 + 2 * kz + 4 * n2 * r;
            *reinterpret_cast<double2*>(row) = make_double2(acc[h][0] - acc[h][3], acc[h][1] + acc[h][2]);
            *reinterpret_cast<double2*>(row + 2 * n2) = make_double2(acc[h][0] + acc[h][3], acc[h][1] - acc[h][2]);
          }
        }
      }
      __syncthreads();
      // x pass of tile t: all node rows of kx against T2's columns (kyl, kz)
      const int nq = 2 * nv * n2, nt2 = (2 * nq + 7) / 8;
      for (int nt0 = warp; nt0 < nt2; nt0 += 16) {
        double b[2][2][KS], acc[2][MT][4];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int col = 8 * (nt0 + 8 * h) + r;
          const bool ok = nt0 + 8 * h < nt2;
#pragma unroll
          for (int par = 0; par < 2; par++)
#pragma unroll
            for (int s = 0; s < KS; s++) {
              const int j = 8 * s + 2 * c + par;
              b[h][par][s] = (ok && j < Pn) ? T2[j * Z.ld2 + col] : 0.0;
            }
#pragma unroll
          for (int u = 0; u < MT; u++) acc[h][u][0] = acc[h][u][1] = acc[h][u][2] = acc[h][u][3] = 0.0;
        }
#pragma unroll
        for (int s = 0; s < KS; s++)
#pragma unroll
          for (int h = 0; h < 2; h++)
#pragma unroll
            for (int u = 0; u < MT; u++) {
              dmma_884(acc[h][u][0], acc[h][u][1], hn[u][0][s], b[h][0][s]);
              dmma_884(acc[h][u][2], acc[h][u][3], hn[u][1][s], b[h][1][s]);
            }
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int q = 4 * (nt0 + 8 * h) + c;  // the lane's complex column (kyl, kz)
          if (q < nq) {
            const int kyl = div16(q, mgN), kz = q - kyl * n2, i = kyl >> 1;
            const int ky = (kyl & 1) ? n2 - 1 - 8 * t - i : n2 + 8 * t + i;
            double2* o = out + npw * (ky + npw * kz);
#pragma unroll
            for (int u = 0; u < MT; u++) {
              const int mx = 8 * u + r;
              if (mx < n2) {
                o[n2 + mx] = make_double2(acc[h][u][0] - acc[h][u][3], acc[h][u][1] + acc[h][u][2]);
                o[n2 - 1 - mx] = make_double2(acc[h][u][0] + acc[h][u][3], acc[h][u][1] - acc[h][u][2]);
              }
            }
          }
        }
      }
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------ (c) eval, 2D Taylor in two kernels
// k_pw2taylor2d: one warp per evaluation leaf converts the leaf's plane-wave
// expansion L[j2 + n2 j1] into the real Taylor block (g2dpw2local_real_vec,
// g2drouts.f:1417-1540)
//     lx[k2][j1] = i^k2 sum_j2 x2l[k2][j2] L[j2 + n2 j1]                     (pass A)
//     lo[k1][k2] = 2 Re( i^k1 sum_{j1 < n2} x2l[k1][j1] (lx[k2][j1] + (-1)^k1 lx[k2][j1 + n2]) )
// once per leaf, as FP64 MMA products, and stores it row-major with the even
// row length E >= P (zero padded) for k_eval2d_horner.  Pass A is one real
// product with B[j2][2 j1 + c] = component c of L[j2 + n2 j1].  2 Re(i^k1 a)
// keeps a.x (even k1) or a.y (odd k1), so pass B is two real products: even
// k1 against be[j1][k2] = Re(lx[k2][j1] + lx[k2][j1+n2]), odd k1 against
// bo[j1][k2] = Im(lx[k2][j1] - lx[k2][j1+n2]).  Operands are zero padded to
// whole tiles; the x2l tables are shared by the CTA's warps (all leaves of a
// launch have one order).
struct ConvDims {
  int Pn, E, Ph, M1, K1, N1, M2, N2;
  int ldX, ldA2, ldB2;
  int tab, warp;  // doubles: CTA tables, per-warp area
  __host__ __device__ ConvDims(int P, int npw) {
    const int n2 = npw / 2;
    Pn = P;
    E = (Pn + 1) & ~1;
    Ph = (Pn + 1) / 2;
    M1 = (Pn + 7) & ~7;        // pass A rows: k2
    K1 = (n2 + 3) & ~3;        // pass A depth j2, pass B depth j1
    N1 = (4 * n2 + 7) & ~7;    // pass A columns: (j1, {re, im} of j1 and of j1 + n2)
    M2 = (Ph + 7) & ~7;        // pass B rows: k1 of one parity
    N2 = M1;                   // pass B columns: k2
    ldX = mma_lda(K1);
    ldA2 = mma_lda(K1);
    ldB2 = mma_ldb(N2);
    tab = M1 * ldX + 2 * M2 * ldA2;
    warp = 2 * K1 * ldB2 + 2 * (n2 + npw);  // be, bo, the fused split's phases (double2 [n2 + npw])
  }
};
constexpr int CONV_MAXKS = 12;  // largest pass A depth in steps of 4: n2 <= 48

// Tables of k_pw2taylor2d for order P: XA[k2][j2] = x2l[k2][j2],
// AE[i][j1] = x2l[2i][j1], AO[i][j1] = x2l[2i+1][j1], zero padded.
void build_conv_table(const HostPlan& H, int Pn, std::vector<double>& out) {
  const int npw = H.P.npw, n2 = npw / 2;
  const ConvDims Z(Pn, npw);
  const size_t base = out.size();
  out.resize(base + Z.tab, 0.0);
  double* XA = out.data() + base;
  double* AE = XA + Z.M1 * Z.ldX;
  double* AO = AE + Z.M2 * Z.ldA2;
  for (int r = 0; r < Pn; r++)
    for (int c = 0; c < n2; c++) {
      XA[r * Z.ldX + c] = H.x2l[(size_t)r * npw + c];
      if (r % 2 == 0) AE[(r / 2) * Z.ldA2 + c] = H.x2l[(size_t)r * npw + c];
      else AO[(r / 2) * Z.ldA2 + c] = H.x2l[(size_t)r * npw + c];
    }
}

// With f32, each coefficient is stored as the FP32 pair (c, c) in its FP64
// slot instead (the layout k_eval2d_horner_f32 reads: a row's float4 m holds
// (c_2m, c_2m, c_2m+1, c_2m+1)), so the mixed evaluation needs no
// conversion pass of its own.
template <int KS>  // pass A depth in steps of 4: KS = ceil(n2 / 4)
__global__ void __launch_bounds__(128) k_pw2taylor2d(KP k, const ConvTask* __restrict__ tasks, int ntask,
                                                     double* __restrict__ lo_all,
                                                     const double* __restrict__ tab, int f32) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int t = blockIdx.x * nw + warp;
  if (t >= ntask) return;  // no CTA-wide barrier in this kernel
  const ConvTask T = tasks[t];
  const int n2 = k.n2;
  const ConvDims Z(T.p + 1, k.npw);
  const int Pn = Z.Pn, E = Z.E;
  extern __shared__ double s1[];
  const double* XA = tab;                 // [M1][ldX], read through L1
  const double* AE = XA + Z.M1 * Z.ldX;   // [M2][ldA2]
  const double* AO = AE + Z.M2 * Z.ldA2;  // [M2][ldA2]
  double* BE = s1 + warp * Z.warp;        // [K1][ldB2]: be[j1][k2]
  double* BO = BE + Z.K1 * Z.ldB2;        // [K1][ldB2]: bo[j1][k2]
  double2* PHX = reinterpret_cast<double2*>(BO + Z.K1 * Z.ldB2);  // fused split: [n2] x phases, then
  double2* PHY = PHX + n2;                                         // [npw] y phases
  // rows of be / bo that pass A does not write
  for (int rr = Z.N1 / 4; rr < Z.K1; rr++)
    for (int c = lane; c < Z.ldB2; c += 32) {
      BE[rr * Z.ldB2 + c] = 0.0;
      BO[rr * Z.ldB2 + c] = 0.0;
    }
  const int ind = blockIdx.y;
  const double* Ld = reinterpret_cast<const double*>(k.loc + ((size_t)T.slot * k.nd + ind) * k.nexp);
  const int r = lane >> 2, c = lane & 3;
  // the split fused (T.fused: T.slot is the cut-level ancestor's expansion):
  // the leaf's coefficient (j2, J) is the ancestor's times
  // exp(i (t_j2 sh0 + t_J sh1)), t_m = x2l[1][m] the nodes, sh the leaf
  // centre minus the ancestor's over sqrt(delta)
  if (T.fused) {
    for (int m = lane; m < n2 + k.npw; m += 32) {
      double sn, cs;
      sincos(k.x2l[k.npw + (m < n2 ? m : m - n2)] * T.sh[m < n2 ? 0 : 1], &sn, &cs);
      PHX[m] = make_double2(cs, sn);
    }
    __syncwarp();
  }
  // pass A: B[j2][n], n = 4 j1 + {re, im of L[.][j1], re, im of L[.][j1 + n2]},
  // read straight from the leaf's expansion (it stays in L1 across the tiles).
  // The accumulator pair of lane (r, c) in tile (mt, nt) is row k2 = 8 mt + r,
  // j1 = 2 nt + c/2: lx[k2][j1] for even c, lx[k2][j1 + n2] for odd c; the
  // partner lane (c xor 1) holds the other, so one exchange forms be and bo.
  for (int nt = 0; nt < Z.N1 / 8; nt++) {
    double bk[KS];
    {
      const int j1 = 2 * nt + (r >> 2), q = r & 3;
      const bool ok = j1 < n2;
      const int J = j1 + (q >> 1) * n2;  // the y node of this lane's column
      const double* bp = Ld + 2 * (c + n2 * J) + (q & 1);
      if (T.fused) {
#pragma unroll
        for (int ks = 0; ks < KS; ks++) {
          const int j2 = 4 * ks + c;
          bk[ks] = 0.0;
          if (ok && j2 < n2) {
            const double2 L = __ldg(reinterpret_cast<const double2*>(Ld) + j2 + n2 * J);
            const double2 v = cmul_rn(L, cmul_rn(PHX[j2], PHY[J]));
            bk[ks] = (q & 1) ? v.y : v.x;
          }
        }
      } else {
#pragma unroll
        for (int ks = 0; ks < KS; ks++) bk[ks] = (ok && 4 * ks + c < n2) ? __ldg(bp + 8 * ks) : 0.0;
      }
    }
    for (int mt = 0; mt < Z.M1 / 8; mt++) {
      const double* ap = XA + (8 * mt + r) * Z.ldX + c;
      double d0 = 0.0, d1 = 0.0, e0 = 0.0, e1 = 0.0;
#pragma unroll
      for (int ks = 0; ks < KS; ks++) {
        if (ks & 1) dmma_884(e0, e1, __ldg(ap + 4 * ks), bk[ks]);
        else dmma_884(d0, d1, __ldg(ap + 4 * ks), bk[ks]);
      }
      const int k2 = 8 * mt + r, j1 = 2 * nt + (c >> 1);
      const double2 z = rot_bf(make_double2(d0 + e0, d1 + e1), k2);
      const double px = __shfl_xor_sync(FULL_MASK, z.x, 1), py = __shfl_xor_sync(FULL_MASK, z.y, 1);
      if ((c & 1) == 0) BE[j1 * Z.ldB2 + k2] = z.x + px;  // Re(lx[j1] + lx[j1 + n2])
      else BO[j1 * Z.ldB2 + k2] = py - z.y;               // Im(lx[j1] - lx[j1 + n2])
    }
  }
  __syncwarp();
  // pass B: 2 Re(i^k1 ...) = 2 {x, -y, -x, y}[k1 mod 4]
  double* out = lo_all + T.off + (size_t)ind * Pn * E;
  float2* out2 = reinterpret_cast<float2*>(out);
  auto put = [&](int e, double v) {
    if (f32) out2[e] = make_float2((float)v, (float)v);
    else out[e] = v;
  };
  warp_gemm<true>(AE, Z.ldA2, BE, Z.ldB2, AO, BO, Z.M2 / 8, Z.N2 / 8, KS,  // A through L1
                  [&](int i, int k2, double e0, double e1, double o0, double o1) {
                    const double se = (i & 1) ? -2.0 : 2.0, so = -se;
                    const int ke = 2 * i, ko = 2 * i + 1;
                    if (ke < Pn) {
                      if (k2 < E) put(ke * E + k2, se * e0);
                      if (k2 + 1 < E) put(ke * E + k2 + 1, se * e1);
                    }
                    if (ko < Pn) {
                      if (k2 < E) put(ko * E + k2, so * o0);
                      if (k2 + 1 < E) put(ko * E + k2 + 1, so * o1);
                    }
                  });
}

// k_eval2d_horner: one CTA (128 threads) per chunk of <= 256 points of an
// evaluation leaf; the leaf's Taylor block (P rows of E = 2 NP2) is staged in
// shared memory and each thread evaluates two points (g2dlevalp_vec,
// g2drouts.f:847-900):
//     pot += sum_k1 y^k1 sum_k2 lo[k1][k2] x^k2,
// Horner in x along each row (coefficient pairs read as double2), then in y.
// Plain FP64 FMAs: on B200 the FP64 FMA pipe and the FP64 MMA share one
// throughput, and Horner at the exact order does P (E - 1) + P FMAs a point
// where the 8 x 8 x 4 MMA pads P up to a multiple of 8 in both dimensions.
// PGH > 1 carries the derivative chains of the Horner sums (hstep, hrow),
// the gradient and Hessian of g2dlevalg_vec / g2dlevalh_vec
// (g2drouts.f:905-1085).
template <int NP2, int PGH>
__global__ void __launch_bounds__(128) k_eval2d_horner(KP k, const HornerTask* __restrict__ tasks,
                                                       const double* __restrict__ lo_all) {
  constexpr int NC = ncomp<2, PGH>();
  const HornerTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y, Pn = T.p + 1;
  extern __shared__ double2 lo2[];  // [Pn][NP2]
  const double2* src = reinterpret_cast<const double2*>(lo_all + T.off + (size_t)ind * Pn * 2 * NP2);
  for (int e = threadIdx.x; e < Pn * NP2; e += blockDim.x) lo2[e] = src[e];
  __syncthreads();
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const int nc = T.set ? k.nc_t : k.nc_s;
  const double cx = k.centers[2 * T.box], cy = k.centers[2 * T.box + 1];
  const int ta = threadIdx.x, tb = threadIdx.x + 128;
  if (ta >= T.n) return;
  const bool two = tb < T.n;
  const double2 pa = reinterpret_cast<const double2*>(pts)[T.i0 + ta];
  const double2 pb = reinterpret_cast<const double2*>(pts)[T.i0 + (two ? tb : ta)];
  const double x0 = (pa.x - cx) * k.dsq, y0 = (pa.y - cy) * k.dsq;
  const double x1 = (pb.x - cx) * k.dsq, y1 = (pb.y - cy) * k.dsq;
  Hor2 a0, a1;
  for (int k1 = Pn - 1; k1 >= 0; k1--) {
    const double2* rw = lo2 + k1 * NP2;
    const double2 ct = rw[NP2 - 1];
    double s0 = ct.y, s1 = ct.y, u0 = 0.0, u1 = 0.0, w0 = 0.0, w1 = 0.0;
    hstep<PGH>(s0, u0, w0, x0, ct.x);
    hstep<PGH>(s1, u1, w1, x1, ct.x);
#pragma unroll
    for (int m = NP2 - 2; m >= 0; m--) {
      const double2 c = rw[m];
      hstep<PGH>(s0, u0, w0, x0, c.y);
      hstep<PGH>(s1, u1, w1, x1, c.y);
      hstep<PGH>(s0, u0, w0, x0, c.x);
      hstep<PGH>(s1, u1, w1, x1, c.x);
    }
    hrow<PGH>(a0, y0, s0, u0, w0);
    hrow<PGH>(a1, y1, s1, u1, w1);
  }
  double v[NC];
  hemit<PGH>(a0, k.dsq, v);
  add_out<NC>(out, T.i0 + ta, k.nd, nc, ind, v);
  if (two) {
    hemit<PGH>(a1, k.dsq, v);
    add_out<NC>(out, T.i0 + tb, k.nd, nc, ind, v);
  }
}

// Orders above 64 (rows longer than 64): the same evaluation with a runtime
// row length.
template <int PGH>
__global__ void __launch_bounds__(128) k_eval2d_horner_any(KP k, const HornerTask* __restrict__ tasks,
                                                           const double* __restrict__ lo_all) {
  constexpr int NC = ncomp<2, PGH>();
  const HornerTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y, Pn = T.p + 1, E = (Pn + 1) & ~1;
  extern __shared__ double lo1[];  // [Pn][E]
  const double* src = lo_all + T.off + (size_t)ind * Pn * E;
  for (int e = threadIdx.x; e < Pn * E; e += blockDim.x) lo1[e] = src[e];
  __syncthreads();
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const int nc = T.set ? k.nc_t : k.nc_s;
  const double cx = k.centers[2 * T.box], cy = k.centers[2 * T.box + 1];
  for (int t = threadIdx.x; t < T.n; t += blockDim.x) {
    const double2 pa = reinterpret_cast<const double2*>(pts)[T.i0 + t];
    double v[NC];
    horner2_rt<PGH>(lo1, E, Pn, (pa.x - cx) * k.dsq, (pa.y - cy) * k.dsq, k.dsq, v);
    add_out<NC>(out, T.i0 + t, k.nd, nc, ind, v);
  }
}

// ------------------------------------------------------------ (c) eval, 3D Taylor in two kernels
// k_pw2taylor3d: one CTA per evaluation leaf converts the leaf's plane-wave
// expansion L[(m1 npw + m2) npw + m3] (m1 over the stored half) into the real
// Taylor block (g3dpw2local_real_vec, g3drouts.f:1774-1938)
//   S1[m2][a]    = i^a  sum_m3 x2l[a][m3] L[m1][m2][m3]        (pass 1, per m1)
//   U2[a][b][m1] = i^b  sum_m2 x2l[b][m2] S1[m2][a]            (pass 2, per m1)
//   lo[c][b][a]  = 2 Re( i^c sum_{m1 < n2} x2l[c][m1] U2[a][b][m1] )   (pass 3)
// as FP64 MMA products.  Passes 1 and 2 run slice by slice over m1 (the
// warps take the slices in turn), so the only large intermediate is U2,
// kept as its real and imaginary parts: pass 3 is two real products, even c
// against Re U2 and odd c against Im U2 (2 Re(i^c z) keeps z.x or z.y).
// Pass 1 reads L straight from the expansion pool: a fragment is four runs of
// 64 contiguous bytes.  The real and imaginary parts of a pass-1 or pass-2
// result sit in the lanes r and r xor 1 of the accumulator layout (rows
// interleave re / im), so one exchange pairs them for the rotation.
struct Conv3Dims {
  int Pn, E, n2, npw;
  int N1, K1, M1;       // pass 1: N1 = a (padded), K1 = m3, M1 = (m2, re/im)
  int M2, K2;           // pass 2: M2 = (a, re/im), K2 = m2, N = N1 (b)
  int M3, K3, N3;       // pass 3: M3 = (a, b) compact, K3 = m1, N3 = c of one parity
  int ldT, ldA2, ldU, ldB3;
  int tab, warp, shared;  // doubles: CTA tables, per-warp area, shared U2
  __host__ __device__ Conv3Dims(int P, int npw_) {
    Pn = P;
    npw = npw_;
    n2 = npw / 2;
    E = (Pn + 1) & ~1;
    N1 = (Pn + 7) & ~7;
    K1 = (npw + 3) & ~3;
    M1 = (2 * npw + 7) & ~7;
    M2 = 2 * N1;
    K2 = K1;
    M3 = (Pn * Pn + 7) & ~7;
    K3 = (n2 + 3) & ~3;
    N3 = (((Pn + 1) / 2) + 7) & ~7;
    ldT = mma_ldb(N1);
    ldA2 = mma_lda(K2);
    ldU = mma_lda(K3);
    ldB3 = mma_ldb(N3);
    tab = K1 * ldT + 2 * K3 * ldB3;
    warp = M2 * ldA2;
    shared = 2 * M3 * ldU;
  }
};

// Shared memory of k_pw2taylor3d with nw warps (the tables and one pass-2
// operand per warp; U2 lives in the CTA's global scratch, conv3_scratch).
size_t conv3_smem_bytes(int Pn, int npw, int nw) {
  const Conv3Dims Z(Pn, npw);
  return ((size_t)Z.tab + (size_t)nw * Z.warp) * 8;
}
// Doubles of U2 (real and imaginary parts) per CTA.
size_t conv3_scratch(int Pn, int npw) {
  const Conv3Dims Z(Pn, npw);
  return (size_t)Z.shared;
}

// Tables of k_pw2taylor3d for order P: XT[m][n] = x2l[n][m] (m < npw, n < P),
// B3e[m1][i] = x2l[2i][m1], B3o[m1][i] = x2l[2i+1][m1] (m1 < n2), zero padded.
void build_conv3_table(const HostPlan& H, int Pn, std::vector<double>& out) {
  const int npw = H.P.npw, n2 = npw / 2;
  const Conv3Dims Z(Pn, npw);
  const size_t base = out.size();
  out.resize(base + Z.tab, 0.0);
  double* XT = out.data() + base;
  double* B3e = XT + Z.K1 * Z.ldT;
  double* B3o = B3e + Z.K3 * Z.ldB3;
  for (int m = 0; m < npw; m++)
    for (int n = 0; n < Pn; n++) XT[m * Z.ldT + n] = H.x2l[(size_t)n * npw + m];
  for (int m1 = 0; m1 < n2; m1++)
    for (int c = 0; c < Pn; c++) {
      double* B = (c & 1) ? B3o : B3e;
      B[m1 * Z.ldB3 + c / 2] = H.x2l[(size_t)c * npw + m1];
    }
}

// Persistent CTAs: the launch's tasks (one order) are taken in turn; U2
// (the pass-3 operand, 2 P^2 n2 doubles) lives in the CTA's slice of uscr
// (global memory, L2-resident), so shared memory holds only the tables and
// one pass-2 operand per warp and several CTAs fit on an SM.
template <int KS1>  // pass 1 depth in steps of 4: KS1 = ceil(npw / 4)
__global__ void __launch_bounds__(128) k_pw2taylor3d(KP k, const ConvTask* __restrict__ tasks, int ntask,
                                                     double* __restrict__ lo_all,
                                                     const double* __restrict__ tab,
                                                     double* __restrict__ uscr, size_t uper) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int r = lane >> 2, c = lane & 3;
  const int ind = blockIdx.y;
  const Conv3Dims Z(tasks[0].p + 1, k.npw);
  const int Pn = Z.Pn, E = Z.E, npw = Z.npw, n2 = Z.n2;
  extern __shared__ double s3[];
  double* XT = s3;                                 // [K1][ldT]
  double* B3e = XT + Z.K1 * Z.ldT;                 // [K3][ldB3]
  double* B3o = B3e + Z.K3 * Z.ldB3;
  double* A2 = s3 + Z.tab + warp * Z.warp;         // [M2][ldA2]
  double* Ure = uscr + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * uper;  // [M3][ldU]
  double* Uim = Ure + Z.M3 * Z.ldU;
  for (int e = threadIdx.x; e < Z.tab; e += blockDim.x) s3[e] = tab[e];
  // every task writes the same entries of U2; the rest (padding) stays zero
  for (int e = threadIdx.x; e < 2 * Z.M3 * Z.ldU; e += blockDim.x) Ure[e] = 0.0;
  __syncthreads();
  for (int task = blockIdx.x; task < ntask; task += gridDim.x) {
    const ConvTask T = tasks[task];
    const double* Ld = reinterpret_cast<const double*>(k.loc + ((size_t)T.slot * k.nd + ind) * k.nexp);
    for (int m1 = warp; m1 < n2; m1 += nw) {
      // pass 1: rows (m2, re/im) of the slice, columns a
      for (int mt = 0; mt < Z.M1 / 8; mt++) {
        const int row = 8 * mt + r, m2 = row >> 1, comp = row & 1;
        const bool rok = m2 < npw;
        const double* ap = Ld + ((size_t)(m1 * npw + m2) * npw) * 2 + comp;
        double av[KS1];
#pragma unroll
        for (int ks = 0; ks < KS1; ks++) {
          const int m3 = 4 * ks + c;
          av[ks] = (rok && m3 < npw) ? __ldg(ap + 2 * m3) : 0.0;
        }
        for (int nt = 0; nt < Z.N1 / 8; nt++) {
          const double* bp = XT + c * Z.ldT + 8 * nt + r;
          double d0 = 0.0, d1 = 0.0, e0 = 0.0, e1 = 0.0;
#pragma unroll
          for (int ks = 0; ks < KS1; ks++) {
            if (ks & 1) dmma_884(e0, e1, av[ks], bp[4 * ks * Z.ldT]);
            else dmma_884(d0, d1, av[ks], bp[4 * ks * Z.ldT]);
          }
          d0 += e0;
          d1 += e1;
          // lane r holds comp (r & 1) of S1[m2][a0], S1[m2][a0 + 1]; r xor 1 the other
          const double o0 = __shfl_xor_sync(FULL_MASK, d0, 4), o1 = __shfl_xor_sync(FULL_MASK, d1, 4);
          const int a0 = 8 * nt + 2 * c;
          const double2 z0 = rot_bf(comp ? make_double2(o0, d0) : make_double2(d0, o0), a0);
          const double2 z1 = rot_bf(comp ? make_double2(o1, d1) : make_double2(d1, o1), a0 + 1);
          if (m2 < Z.K2) {
            if (comp == 0) {
              A2[(2 * a0) * Z.ldA2 + m2] = z0.x;
              A2[(2 * a0 + 1) * Z.ldA2 + m2] = z0.y;
            } else {
              A2[(2 * a0 + 2) * Z.ldA2 + m2] = z1.x;
              A2[(2 * a0 + 3) * Z.ldA2 + m2] = z1.y;
            }
          }
        }
      }
      __syncwarp();
      // pass 2: rows (a, re/im), columns b; U2[a][b][m1] into Ure / Uim
      for (int mt = 0; mt < Z.M2 / 8; mt++) {
        const double* ap = A2 + (8 * mt + r) * Z.ldA2 + c;
        for (int nt = 0; nt < Z.N1 / 8; nt++) {
          const double* bp = XT + c * Z.ldT + 8 * nt + r;
          double d0 = 0.0, d1 = 0.0, e0 = 0.0, e1 = 0.0;
          for (int ks = 0; ks < Z.K2 / 4; ks += 2) {
            dmma_884(d0, d1, ap[4 * ks], bp[4 * ks * Z.ldT]);
            if (ks + 1 < Z.K2 / 4) dmma_884(e0, e1, ap[4 * ks + 4], bp[(4 * ks + 4) * Z.ldT]);
          }
          d0 += e0;
          d1 += e1;
          const double o0 = __shfl_xor_sync(FULL_MASK, d0, 4), o1 = __shfl_xor_sync(FULL_MASK, d1, 4);
          const int row = 8 * mt + r, a = row >> 1, comp = row & 1, b0 = 8 * nt + 2 * c;
          const double2 z0 = rot_bf(comp ? make_double2(o0, d0) : make_double2(d0, o0), b0);
          const double2 z1 = rot_bf(comp ? make_double2(o1, d1) : make_double2(d1, o1), b0 + 1);
          if (a < Pn) {
            if (comp == 0 && b0 < Pn) {
              Ure[(a * Pn + b0) * Z.ldU + m1] = z0.x;
              Uim[(a * Pn + b0) * Z.ldU + m1] = z0.y;
            }
            if (comp == 1 && b0 + 1 < Pn) {
              Ure[(a * Pn + b0 + 1) * Z.ldU + m1] = z1.x;
              Uim[(a * Pn + b0 + 1) * Z.ldU + m1] = z1.y;
            }
          }
        }
      }
      __syncwarp();
    }
    __syncthreads();
    // pass 3: lo[c][b][a] = 2 {x, -y, -x, y}[c mod 4] of sum_m1 x2l[c][m1] U2[a][b][m1]
    double* out = lo_all + T.off + (size_t)ind * Pn * Pn * E;
    for (int mt = warp; mt < Z.M3 / 8; mt += nw) {
      const double* ae = Ure + (8 * mt + r) * Z.ldU + c;
      const double* ao = Uim + (8 * mt + r) * Z.ldU + c;
      for (int nt = 0; nt < Z.N3 / 8; nt++) {
        const double* be = B3e + c * Z.ldB3 + 8 * nt + r;
        const double* bo = B3o + c * Z.ldB3 + 8 * nt + r;
        double e0 = 0.0, e1 = 0.0, o0 = 0.0, o1 = 0.0;
        for (int ks = 0; ks < Z.K3 / 4; ks++) {
          dmma_884(e0, e1, ae[4 * ks], be[4 * ks * Z.ldB3]);
          dmma_884(o0, o1, ao[4 * ks], bo[4 * ks * Z.ldB3]);
        }
        const int q = 8 * mt + r;
        if (q >= Pn * Pn) continue;
        const int a = q / Pn, b = q - a * Pn;
        const double ev[2] = {e0, e1}, od[2] = {o0, o1};
#pragma unroll
        for (int i = 0; i < 2; i++) {
          const int ce = 2 * (8 * nt + 2 * c + i), co = ce + 1;
          if (ce < Pn) out[((size_t)ce * Pn + b) * E + a] = ((ce & 3) == 2 ? -2.0 : 2.0) * ev[i];
          if (co < Pn) out[((size_t)co * Pn + b) * E + a] = ((co & 3) == 1 ? -2.0 : 2.0) * od[i];
        }
      }
    }
    if (E > Pn)  // the padding column of every row
      for (int e = threadIdx.x; e < Pn * Pn; e += blockDim.x) out[(size_t)e * E + Pn] = 0.0;
    __syncthreads();  // U2 of this task is read until here
  }
}

// k_pw2taylor3d_mma: the conversion of k_pw2taylor3d for orders P <= 16 with
// the mirror symmetry of the node set used in both full dimensions and the
// node tables as register fragments.  With the signed table
// tx[a][m] = x2l[a][m] (-1)^(a/2) over the first half m < n2 and mirror node
// mb = npw - 1 - m (x2l[a][mb] = (-1)^a x2l[a][m]), a sum over all nodes is
//   i^a sum_m x2l[a][m] L[m] = tx[a][.] (L[m] + L[mb])        (a even)
//                            = i tx[a][.] (L[m] - L[mb])      (a odd),
// so every pass is two real products of depth n2 (KS k-steps of 4):
//   x pass  S1[m1][m2][a] from the staged slices of L     (M = a, N = (m1, m2, re/im))
//   y pass  S2[m1][b][a]  from S1, same table in b         (M = b, N = (m1, a, re/im))
//   z pass  lo[c][b][a] += 2 Re(i^c tx[c][m1] S2[m1][b][a]): even c against
//           Re S2, odd c against -Im S2, K = the four slices m1 of a group
// The leaf is taken four z slices (one z k-step) at a time: the slices are
// copied into shared memory with cp.async (the next group's copy overlaps
// the y and z passes of this one), and the z accumulators stay in registers
// across the groups (each warp owns up to four of the ceil(P^2 / 8) column
// tiles).  Row strides: staged slices 8 (mod 16) doubles (the fragment's
// re/im pairs of four rows are conflict-free), S1 and S2 4 (mod 8).
// Persistent CTAs of 8 warps, two per SM, over the leaves of one order.
struct C3Dims {
  int ldL, ld1, ld2;
  size_t total;  // doubles
  __host__ __device__ C3Dims(int Pn, int npw) {
    ldL = ((2 * npw + 7) & ~15) + 8;
    ld1 = 8 * Pn + 4;
    ld2 = 8 * ((Pn * Pn + 7) / 8) + 4;
    total = (size_t)4 * npw * ldL + (size_t)npw * ld1 + (size_t)8 * ld2 + (size_t)2 * (2 * npw + npw / 2);
  }
};
// The fused split's phase tables of one task (x and y over all npw nodes, z
// over the stored half) into ph (double2 [2 npw + n2]); node t_m = x2l[1][m].
__device__ __forceinline__ void conv_phases(const KP& k, const ConvTask& T, double2* ph) {
  const int npw = k.npw, n2 = k.n2;
  for (int e = threadIdx.x; e < 2 * npw + n2; e += blockDim.x) {
    const int d = e < npw ? 0 : e < 2 * npw ? 1 : 2, m = e - d * npw;
    double sn, cs;
    sincos(k.x2l[npw + m] * T.sh[d], &sn, &cs);
    ph[e] = make_double2(cs, sn);
  }
}
// Multiplies staged slices (rows (m1, m2) of npw complex m3, row stride ldL
// doubles, slices m1 = m1_0 .. m1_0 + ns - 1) by the task's phases.
__device__ __forceinline__ void conv_apply_phases(double* Lb, int ldL, int npw, int m1_0, int ns,
                                                  const double2* ph) {
  const int n = ns * npw * npw;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const int row = e / npw, m3 = e - row * npw, m1 = m1_0 + row / npw, m2 = row - (row / npw) * npw;
    double2* z = reinterpret_cast<double2*>(Lb + (size_t)row * ldL + 2 * m3);
    *z = cmul(*z, cmul(ph[m3], cmul(ph[npw + m2], ph[2 * npw + m1])));
  }
}

template <int KS>
__global__ void __launch_bounds__(256, 2) k_pw2taylor3d_mma(KP k, const ConvTask* __restrict__ tasks, int ntask,
                                                            double* __restrict__ lo_all) {
  constexpr int NTW = 4;  // z-pass column tiles per warp (ceil(16^2 / 8) / 8)
  const int ind = blockIdx.y;
  const int npw = k.npw, n2 = k.n2;
  const int Pn = tasks[0].p + 1, E = (Pn + 1) & ~1, P2 = Pn * Pn;
  const int mgN = (65536 + npw - 1) / npw, mgP = (65536 + Pn - 1) / Pn;  // div16 factors
  const C3Dims Z(Pn, npw);
  extern __shared__ double sm[];
  double* Lb = sm;                                  // [4 m1][npw m2][ldL]: (m3, re/im)
  double* S1 = Lb + (size_t)4 * npw * Z.ldL;        // [npw m2][ld1]: (m1, a, re/im)
  double* S2r = S1 + (size_t)npw * Z.ld1;           // [4 m1][ld2]: (b, a)
  double* S2i = S2r + 4 * Z.ld2;
  double2* PH = reinterpret_cast<double2*>(S2i + 4 * Z.ld2);  // fused split: [2 npw + n2] phases
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, r = lane >> 2, c = lane & 3;
  int tk = blockIdx.x;
  if (tk >= ntask) return;
  // A fragments: tx[par][s] = table row 2 r + par, node 4 s + c
  double tx[2][KS];
#pragma unroll
  for (int par = 0; par < 2; par++)
#pragma unroll
    for (int s = 0; s < KS; s++) {
      const int a = 2 * r + par, m = 4 * s + c;
      tx[par][s] = (a < Pn && m < n2) ? (((a >> 1) & 1) ? -k.x2l[a * npw + m] : k.x2l[a * npw + m]) : 0.0;
    }
  // copy the slices 4 g .. 4 g + 3 of the expansion in the given slot (rows of npw complex)
  auto stage = [&](int slot, int g) {
    const double* L = reinterpret_cast<const double*>(k.loc + ((size_t)slot * k.nd + ind) * k.nexp) +
                      (size_t)8 * g * npw * npw;
    const int rows = min(4, n2 - 4 * g) * npw;
    const unsigned dst = (unsigned)__cvta_generic_to_shared(Lb);
    for (int row = warp; row < rows; row += 8)
      for (int u = lane; u < npw; u += 32)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + 8u * (unsigned)(row * Z.ldL + 2 * u)),
                     "l"(L + (size_t)row * 2 * npw + 2 * u) : "memory");
  };
  int slot = tasks[tk].slot;
  stage(slot, 0);
  double acc[NTW][2][2];
#pragma unroll
  for (int i = 0; i < NTW; i++) acc[i][0][0] = acc[i][0][1] = acc[i][1][0] = acc[i][1][1] = 0.0;
  const int ntZ = (P2 + 7) / 8;
  for (; tk < ntask; tk += gridDim.x) {
    const int tn = tk + gridDim.x;
    const int nslot = tn < ntask ? tasks[tn].slot : 0;
    const long long off = tasks[tk].off;
    const bool fused = tasks[tk].fused;
    if (fused) conv_phases(k, tasks[tk], PH);
    for (int g = 0; g < KS; g++) {
      const int ns = min(4, n2 - 4 * g);
      asm volatile("cp.async.wait_all;" ::: "memory");
      __syncthreads();
      if (fused) {  // the ancestor's slices become the leaf's: the split, fused
        conv_apply_phases(Lb, Z.ldL, npw, 4 * g, ns, PH);
        __syncthreads();
      }
      // x pass: columns (m1, m2, re/im) of the staged slices
      const int ntX = (ns * npw * 2 + 7) / 8;
      for (int nt = warp; nt < ntX; nt += 8) {
        const int col = 8 * nt + r;
        const double* bp = Lb + (col >> 1) * Z.ldL + (col & 1);
        double e0 = 0.0, e1 = 0.0, o0 = 0.0, o1 = 0.0;
#pragma unroll
        for (int s = 0; s < KS; s++) {
          const int m = 4 * s + c;
          double v1 = 0.0, v2 = 0.0;
          if (m < n2) {
            v1 = bp[2 * m];
            v2 = bp[2 * (npw - 1 - m)];
          }
          dmma_884(e0, e1, tx[0][s], v1 + v2);
          dmma_884(o0, o1, tx[1][s], v1 - v2);
        }
        const int q = 4 * nt + c;  // the lane's complex column (m1, m2)
        if (q < ns * npw) {
          const int m1 = div16(q, mgN), m2 = q - m1 * npw;
          double* o = S1 + m2 * Z.ld1 + 2 * (m1 * Pn + 2 * r);
          if (2 * r < Pn) *reinterpret_cast<double2*>(o) = make_double2(e0, e1);
          if (2 * r + 1 < Pn) *reinterpret_cast<double2*>(o + 2) = make_double2(-o1, o0);
        }
      }
      __syncthreads();
      // the slices are consumed: copy the next group's (or the next leaf's first)
      if (g + 1 < KS) stage(slot, g + 1);
      else if (tn < ntask) stage(nslot, 0);
      // y pass: columns (m1, a, re/im)
      const int ntY = (ns * Pn * 2 + 7) / 8;
      for (int nt = warp; nt < ntY; nt += 8) {
        const int col = 8 * nt + r;
        double e0 = 0.0, e1 = 0.0, o0 = 0.0, o1 = 0.0;
#pragma unroll
        for (int s = 0; s < KS; s++) {
          const int m = 4 * s + c;
          double v1 = 0.0, v2 = 0.0;
          if (m < n2) {
            v1 = S1[m * Z.ld1 + col];
            v2 = S1[(npw - 1 - m) * Z.ld1 + col];
          }
          dmma_884(e0, e1, tx[0][s], v1 + v2);
          dmma_884(o0, o1, tx[1][s], v1 - v2);
        }
        const int q = 4 * nt + c;  // the lane's complex column (m1, a)
        if (q < ns * Pn) {
          const int m1 = div16(q, mgP), a = q - m1 * Pn;
          const int o = m1 * Z.ld2 + 2 * r * Pn + a;
          if (2 * r < Pn) {
            S2r[o] = e0;
            S2i[o] = e1;
          }
          if (2 * r + 1 < Pn) {
            S2r[o + Pn] = -o1;
            S2i[o + Pn] = o0;
          }
        }
      }
      __syncthreads();
      // z pass: k-step g of the accumulators, rows c = 2 r + par, columns (b, a)
      double te = tx[0][0], to = tx[1][0];
#pragma unroll
      for (int s = 1; s < KS; s++)
        if (s == g) {
          te = tx[0][s];
          to = tx[1][s];
        }
#pragma unroll
      for (int i = 0; i < NTW; i++) {
        const int nt = warp + 8 * i;
        if (nt < ntZ) {
          const double br = c < ns ? S2r[c * Z.ld2 + 8 * nt + r] : 0.0;
          const double bi = c < ns ? S2i[c * Z.ld2 + 8 * nt + r] : 0.0;
          dmma_884(acc[i][0][0], acc[i][0][1], te, br);
          dmma_884(acc[i][1][0], acc[i][1][1], to, bi);
        }
      }
    }
    // lo[c][b][a] = 2 acc (even c), -2 acc (odd c); rows of E doubles
    double* out = lo_all + off + (size_t)ind * P2 * E;
#pragma unroll
    for (int i = 0; i < NTW; i++) {
      const int nt = warp + 8 * i;
#pragma unroll
      for (int ii = 0; ii < 2; ii++) {
        const int q = 8 * nt + 2 * c + ii;
        if (nt < ntZ && q < P2) {
          const int b = div16(q, mgP), a = q - b * Pn;
          if (2 * r < Pn) out[((2 * r) * Pn + b) * E + a] = 2.0 * acc[i][0][ii];
          if (2 * r + 1 < Pn) out[((2 * r + 1) * Pn + b) * E + a] = -2.0 * acc[i][1][ii];
        }
        acc[i][0][ii] = acc[i][1][ii] = 0.0;
      }
    }
    if (E > Pn)  // the padding column of every row
      for (int e = threadIdx.x; e < P2; e += blockDim.x) out[(size_t)e * E + Pn] = 0.0;
    slot = nslot;
  }
}

// k_pw2taylor3d_mma2: the same conversion for orders 17..32 (two 8-row tiles
// of each parity).  The z accumulators of these orders do not fit in
// registers, so S2 keeps every z slice (Re and Im, n2 rows of P^2) and the z
// pass runs once per leaf after the x and y passes of all its slice groups;
// a group is gs slices (4, 2 or 1, the largest whose shared memory fits).
// One CTA of 8 warps per SM, persistent over the leaves of one order.
struct C3Dims2 {
  int gs, ldL, ld1, ld2;
  size_t total;  // doubles
  __host__ __device__ C3Dims2(int Pn, int npw, int gs_) {
    const int n2 = npw / 2;
    gs = gs_;
    ldL = ((2 * npw + 7) & ~15) + 8;
    ld1 = 8 * ((2 * gs * Pn + 7) / 8) + 4;
    ld2 = 8 * ((Pn * Pn + 7) / 8) + 4;
    total = (size_t)gs * npw * ldL + (size_t)npw * ld1 + (size_t)2 * n2 * ld2 + (size_t)2 * (2 * npw + n2);
  }
};

template <int KS>
__global__ void __launch_bounds__(256, 1) k_pw2taylor3d_mma2(KP k, const ConvTask* __restrict__ tasks, int ntask,
                                                             double* __restrict__ lo_all, int gs) {
  const int ind = blockIdx.y;
  const int npw = k.npw, n2 = k.n2;
  const int Pn = tasks[0].p + 1, E = (Pn + 1) & ~1, P2 = Pn * Pn;
  const int mgN = (65536 + npw - 1) / npw, mgP = (65536 + Pn - 1) / Pn;  // div16 factors
  const C3Dims2 Z(Pn, npw, gs);
  extern __shared__ double sm[];
  double* Lb = sm;                                  // [gs m1][npw m2][ldL]: (m3, re/im)
  double* S1 = Lb + (size_t)gs * npw * Z.ldL;       // [npw m2][ld1]: (m1, a, re/im)
  double* S2r = S1 + (size_t)npw * Z.ld1;           // [n2 m1][ld2]: (b, a)
  double* S2i = S2r + (size_t)n2 * Z.ld2;
  double2* PH = reinterpret_cast<double2*>(S2i + (size_t)n2 * Z.ld2);  // fused split: [2 npw + n2] phases
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, r = lane >> 2, c = lane & 3;
  int tk = blockIdx.x;
  if (tk >= ntask) return;
  // A fragments: tx[u][par][s] = table row 2 (8 u + r) + par, node 4 s + c
  double tx[2][2][KS];
#pragma unroll
  for (int u = 0; u < 2; u++)
#pragma unroll
    for (int par = 0; par < 2; par++)
#pragma unroll
      for (int s = 0; s < KS; s++) {
        const int a = 2 * (8 * u + r) + par, m = 4 * s + c;
        tx[u][par][s] =
            (a < Pn && m < n2) ? (((a >> 1) & 1) ? -k.x2l[a * npw + m] : k.x2l[a * npw + m]) : 0.0;
      }
  const int ng = (n2 + gs - 1) / gs;
  auto stage = [&](int slot, int g) {
    const double* L = reinterpret_cast<const double*>(k.loc + ((size_t)slot * k.nd + ind) * k.nexp) +
                      (size_t)2 * gs * g * npw * npw;
    const int rows = min(gs, n2 - gs * g) * npw;
    const unsigned dst = (unsigned)__cvta_generic_to_shared(Lb);
    for (int row = warp; row < rows; row += 8)
      for (int u = lane; u < npw; u += 32)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + 8u * (unsigned)(row * Z.ldL + 2 * u)),
                     "l"(L + (size_t)row * 2 * npw + 2 * u) : "memory");
  };
  int slot = tasks[tk].slot;
  stage(slot, 0);
  const int ntZ = (P2 + 7) / 8;
  for (; tk < ntask; tk += gridDim.x) {
    const int tn = tk + gridDim.x;
    const int nslot = tn < ntask ? tasks[tn].slot : 0;
    const long long off = tasks[tk].off;
    const bool fused = tasks[tk].fused;
    if (fused) conv_phases(k, tasks[tk], PH);
    for (int g = 0; g < ng; g++) {
      const int ns = min(gs, n2 - gs * g);
      asm volatile("cp.async.wait_all;" ::: "memory");
      __syncthreads();
      if (fused) {  // the ancestor's slices become the leaf's: the split, fused
        conv_apply_phases(Lb, Z.ldL, npw, gs * g, ns, PH);
        __syncthreads();
      }
      // x pass: columns (m1, m2, re/im) of the staged slices
      const int ntX = (ns * npw * 2 + 7) / 8;
      for (int nt = warp; nt < ntX; nt += 8) {
        const int col = 8 * nt + r;
        const double* bp = Lb + (col >> 1) * Z.ldL + (col & 1);
        double acc[2][4];
#pragma unroll
        for (int u = 0; u < 2; u++) acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0.0;
#pragma unroll
        for (int s = 0; s < KS; s++) {
          const int m = 4 * s + c;
          double v1 = 0.0, v2 = 0.0;
          if (m < n2) {
            v1 = bp[2 * m];
            v2 = bp[2 * (npw - 1 - m)];
          }
#pragma unroll
          for (int u = 0; u < 2; u++) {
            dmma_884(acc[u][0], acc[u][1], tx[u][0][s], v1 + v2);
            dmma_884(acc[u][2], acc[u][3], tx[u][1][s], v1 - v2);
          }
        }
        const int q = 4 * nt + c;  // the lane's complex column (m1, m2)
        if (q < ns * npw) {
          const int m1 = div16(q, mgN), m2 = q - m1 * npw;
#pragma unroll
          for (int u = 0; u < 2; u++) {
            const int a = 2 * (8 * u + r);
            double* o = S1 + m2 * Z.ld1 + 2 * (m1 * Pn + a);
            if (a < Pn) *reinterpret_cast<double2*>(o) = make_double2(acc[u][0], acc[u][1]);
            if (a + 1 < Pn) *reinterpret_cast<double2*>(o + 2) = make_double2(-acc[u][3], acc[u][2]);
          }
        }
      }
      __syncthreads();
      // the slices are consumed: copy the next group's (or the next leaf's first)
      if (g + 1 < ng) stage(slot, g + 1);
      else if (tn < ntask) stage(nslot, 0);
      // y pass: columns (m1, a, re/im) into the z slices gs g + m1 of S2
      const int ntY = (ns * Pn * 2 + 7) / 8;
      for (int nt = warp; nt < ntY; nt += 8) {
        const int col = 8 * nt + r;
        double acc[2][4];
#pragma unroll
        for (int u = 0; u < 2; u++) acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0.0;
#pragma unroll
        for (int s = 0; s < KS; s++) {
          const int m = 4 * s + c;
          double v1 = 0.0, v2 = 0.0;
          if (m < n2) {
            v1 = S1[m * Z.ld1 + col];
            v2 = S1[(npw - 1 - m) * Z.ld1 + col];
          }
#pragma unroll
          for (int u = 0; u < 2; u++) {
            dmma_884(acc[u][0], acc[u][1], tx[u][0][s], v1 + v2);
            dmma_884(acc[u][2], acc[u][3], tx[u][1][s], v1 - v2);
          }
        }
        const int q = 4 * nt + c;  // the lane's complex column (m1, a)
        if (q < ns * Pn) {
          const int m1 = div16(q, mgP), a = q - m1 * Pn;
#pragma unroll
          for (int u = 0; u < 2; u++) {
            const int b = 2 * (8 * u + r);
            const int o = (gs * g + m1) * Z.ld2 + b * Pn + a;
            if (b < Pn) {
              S2r[o] = acc[u][0];
              S2i[o] = acc[u][1];
            }
            if (b + 1 < Pn) {
              S2r[o + Pn] = -acc[u][3];
              S2i[o + Pn] = acc[u][2];
            }
          }
        }
      }
    }
    __syncthreads();
    // z pass over all slices: rows c = 2 (8 u + r) + par, columns (b, a)
    double* out = lo_all + off + (size_t)ind * P2 * E;
    for (int nt = warp; nt < ntZ; nt += 8) {
      double acc[2][2][2];
#pragma unroll
      for (int u = 0; u < 2; u++) acc[u][0][0] = acc[u][0][1] = acc[u][1][0] = acc[u][1][1] = 0.0;
#pragma unroll
      for (int s = 0; s < KS; s++) {
        const int m1 = 4 * s + c;
        const double br = m1 < n2 ? S2r[m1 * Z.ld2 + 8 * nt + r] : 0.0;
        const double bi = m1 < n2 ? S2i[m1 * Z.ld2 + 8 * nt + r] : 0.0;
#pragma unroll
        for (int u = 0; u < 2; u++) {
          dmma_884(acc[u][0][0], acc[u][0][1], tx[u][0][s], br);
          dmma_884(acc[u][1][0], acc[u][1][1], tx[u][1][s], bi);
        }
      }
#pragma unroll
      for (int ii = 0; ii < 2; ii++) {
        const int q = 8 * nt + 2 * c + ii;
        if (q < P2) {
          const int b = div16(q, mgP), a = q - b * Pn;
#pragma unroll
          for (int u = 0; u < 2; u++) {
            const int ce = 2 * (8 * u + r);
            if (ce < Pn) out[(ce * Pn + b) * E + a] = 2.0 * acc[u][0][ii];
            if (ce + 1 < Pn) out[((ce + 1) * Pn + b) * E + a] = -2.0 * acc[u][1][ii];
          }
        }
      }
    }
    if (E > Pn)  // the padding column of every row
      for (int e = threadIdx.x; e < P2; e += blockDim.x) out[(size_t)e * E + Pn] = 0.0;
    slot = nslot;
  }
}

// k_eval3d_sep: potential at a leaf's points straight from its plane-wave
// local expansion, for the plane-wave route (g3dpwevalp_vec,
// g3drouts.f:2268-2362) and for Taylor-route leaves whose order exceeds the
// conversion kernels (g3dpw2local_real_vec + g3dlevalp_vec).  Both are
//   pot = 2 Re sum_{m1 < n2} Z[m1](z) sum_{m2} Y[m2](y) sum_{m3} X[m3](x) L[m1][m2][m3]
// with X[m](x) = exp(i t_m x) on the plane-wave route and, on the Taylor
// route, its series truncated at the order, sum_{a<P} x2l[a][m] (i x)^a: the
// Taylor block lo[c][b][a] of the conversion contracted with x^a y^b z^c is
// exactly this sum, evaluated without forming the P^3 block.  One CTA per
// task; points in blocks of 32 whose phase tables sit in shared memory; a
// thread takes rows (m1, m2) of the expansion for four points (L read once
// per block, through the read-only cache), and the partial sums are reduced
// in a fixed order.  Potentials only (the derivative variants keep their own
// kernels).
constexpr int SEP_NPB = 32;
// xt: the x2l table of the order, staged in shared memory ([a][m], npw per row)
__device__ __forceinline__ double2 sep_phase(const KP& k, bool taylor, int m, double u, int Pn,
                                             const double* xt) {
  const double t = (2 * (m - k.n2) + 1) * k.t1;
  if (!taylor) return cexpi(t * u);
  // sum_{a<P} x2l[a][m] (i u)^a by Horner in (i u)
  double re = xt[(Pn - 1) * k.npw + m], im = 0.0;
  for (int a = Pn - 2; a >= 0; a--) {
    const double nr = fma(-im, u, xt[a * k.npw + m]);
    im = re * u;
    re = nr;
  }
  return make_double2(re, im);
}
template <bool TAYLOR>
__global__ void __launch_bounds__(256, 2) k_eval3d_sep(KP k, const EvalTask* __restrict__ tasks) {
  const EvalTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  const int npw = k.npw, n2 = k.n2, Pn = T.p + 1, tid = threadIdx.x;
  const double2* L = k.loc + ((size_t)T.slot * k.nd + ind) * k.nexp;
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const int nc = T.set ? k.nc_t : k.nc_s;
  const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1], cz = k.centers[3 * T.box + 2];
  extern __shared__ double2 sep_sh[];
  double2* X = sep_sh;                      // [npw][SEP_NPB]
  double2* Y = X + npw * SEP_NPB;           // [npw][SEP_NPB]
  double2* Zt = Y + npw * SEP_NPB;          // [n2][SEP_NPB]
  double2* part = Zt + n2 * SEP_NPB;        // [256][4] partial sums
  double* xt = reinterpret_cast<double*>(part + 256 * 4);  // Taylor route: x2l rows a < P
  if (TAYLOR)
    for (int e = tid; e < Pn * npw; e += blockDim.x) xt[e] = k.x2l[e];
  const int nrow = n2 * npw;
  __syncthreads();
  for (int p0 = 0; p0 < T.n; p0 += SEP_NPB) {
    const int np = min(SEP_NPB, T.n - p0);
    for (int e = tid; e < (2 * npw + n2) * SEP_NPB; e += blockDim.x) {
      const int m = e / SEP_NPB, pt = e % SEP_NPB;
      const int d = m < npw ? 0 : m < 2 * npw ? 1 : 2, node = d == 0 ? m : d == 1 ? m - npw : m - 2 * npw;
      double2 v = make_double2(0.0, 0.0);
      if (pt < np) {
        const double u = (pts[3 * (T.i0 + p0 + pt) + d] - (d == 0 ? cx : d == 1 ? cy : cz)) * k.dsq;
        v = sep_phase(k, TAYLOR, node, u, Pn, xt);
      }
      // X, Y and Zt are consecutive; point 4 g + j sits at j * 8 + g of its
      // row, so the eight point groups of one j are one 128-byte line
      X[m * SEP_NPB + (pt & 3) * 8 + (pt >> 2)] = v;
    }
    __syncthreads();
    const int npg = (np + 3) / 4, rstep = blockDim.x / npg;
    const int pg = tid % npg, rs = tid / npg;
    double2 acc[4];
#pragma unroll
    for (int j = 0; j < 4; j++) acc[j] = make_double2(0.0, 0.0);
    if (rs < rstep) {
      int m1 = 0, m2 = rs;
      while (m2 >= npw) {
        m2 -= npw;
        m1++;
      }
      for (int row = rs; row < nrow; row += rstep) {
        const double2* Lr = L + (size_t)row * npw;
        double2 s[4];
#pragma unroll
        for (int j = 0; j < 4; j++) s[j] = make_double2(0.0, 0.0);
        // eight coefficients loaded before their products (loads in flight)
        int m3 = 0;
        for (; m3 + 8 <= npw; m3 += 8) {
          double2 l[8];
#pragma unroll
          for (int u = 0; u < 8; u++) l[u] = __ldg(Lr + m3 + u);
#pragma unroll
          for (int u = 0; u < 8; u++) {
            const double2* xp = X + (m3 + u) * SEP_NPB + pg;
#pragma unroll
            for (int j = 0; j < 4; j++) s[j] = cfma(l[u], xp[8 * j], s[j]);
          }
        }
        for (; m3 < npw; m3++) {
          const double2 l = __ldg(Lr + m3);
          const double2* xp = X + m3 * SEP_NPB + pg;
#pragma unroll
          for (int j = 0; j < 4; j++) s[j] = cfma(l, xp[8 * j], s[j]);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const double2 yz = cmul(Y[m2 * SEP_NPB + 8 * j + pg], Zt[m1 * SEP_NPB + 8 * j + pg]);
          acc[j] = cfma(s[j], yz, acc[j]);
        }
        m2 += rstep;
        while (m2 >= npw) {
          m2 -= npw;
          m1++;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) part[tid * 4 + j] = acc[j];
    __syncthreads();
    if (tid < np) {
      const int g = tid >> 2, j = tid & 3;
      double re = 0.0;
      for (int r = 0; r < rstep; r++) re += part[(r * npg + g) * 4 + j].x;
      const double v = 2.0 * re;
      add_out<1>(out, T.i0 + p0 + tid, k.nd, nc, ind, &v);
    }
    __syncthreads();
  }
}

// k_eval3d_horner: one CTA (128 threads) per chunk of <= 256 points of an
// evaluation leaf; the leaf's Taylor block lo[c][b][a] (rows of E = 2 NP2)
// is staged in shared memory and each thread evaluates two points by Horner
// in x along each row, then in y, then in z (g3dlevalp_vec,
// g3drouts.f:1045-1107), plain FP64 FMAs at the exact order.
// Horner over the planes and rows of a staged block for NPT points at once,
// NR rows of a plane in flight (independent x chains: instruction-level
// parallelism for leaves of few points), the rows then folded into the y
// chain in row order: the same operations in the same order per point as
// one row at a time.
template <int NP2, int PGH, int NPT, int NR>
__device__ __forceinline__ void horner3_block(const double2* lo3, int Pn, const double* x, const double* y,
                                              const double* z, Hor3* a) {
  for (int cc = Pn - 1; cc >= 0; cc--) {
    Hor2 q[NPT];
    for (int b = Pn - 1; b >= 0; b -= NR) {
      double s[NR][NPT], u[NR][NPT], w[NR][NPT];
      const double2* rw[NR];
#pragma unroll
      for (int r = 0; r < NR; r++) {
        rw[r] = lo3 + (cc * Pn + (b - r >= 0 ? b - r : b)) * NP2;  // past row 0: a copy, not folded
        const double2 ct = rw[r][NP2 - 1];
#pragma unroll
        for (int p = 0; p < NPT; p++) {
          s[r][p] = ct.y;
          u[r][p] = w[r][p] = 0.0;
          hstep<PGH>(s[r][p], u[r][p], w[r][p], x[p], ct.x);
        }
      }
#pragma unroll
      for (int m = NP2 - 2; m >= 0; m--) {
#pragma unroll
        for (int r = 0; r < NR; r++) {
          const double2 cf = rw[r][m];
#pragma unroll
          for (int p = 0; p < NPT; p++) hstep<PGH>(s[r][p], u[r][p], w[r][p], x[p], cf.y);
#pragma unroll
          for (int p = 0; p < NPT; p++) hstep<PGH>(s[r][p], u[r][p], w[r][p], x[p], cf.x);
        }
      }
#pragma unroll
      for (int r = 0; r < NR; r++)
        if (b - r >= 0)
#pragma unroll
          for (int p = 0; p < NPT; p++) hrow<PGH>(q[p], y[p], s[r][p], u[r][p], w[r][p]);
    }
#pragma unroll
    for (int p = 0; p < NPT; p++) hplane<PGH>(a[p], z[p], q[p]);
  }
}

template <int NP2, int PGH>
__global__ void __launch_bounds__(128) k_eval3d_horner(KP k, const HornerTask* __restrict__ tasks,
                                                       const double* __restrict__ lo_all) {
  constexpr int NC = ncomp<3, PGH>();
  const HornerTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y, Pn = T.p + 1;
  extern __shared__ double2 lo3[];  // [Pn][Pn][NP2]
  const double2* src = reinterpret_cast<const double2*>(lo_all + T.off + (size_t)ind * Pn * Pn * 2 * NP2);
  for (int e = threadIdx.x; e < Pn * Pn * NP2; e += blockDim.x) lo3[e] = src[e];
  __syncthreads();
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const int nc = T.set ? k.nc_t : k.nc_s;
  const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1], cz = k.centers[3 * T.box + 2];
  const int ta = threadIdx.x, tb = threadIdx.x + 128;
  if (ta >= T.n) return;
  const int pa = T.i0 + ta;
  double v[NC];
  if (T.n <= 128) {
    // one point per thread, four rows in flight
    const double x = (pts[3 * pa] - cx) * k.dsq, y = (pts[3 * pa + 1] - cy) * k.dsq, z = (pts[3 * pa + 2] - cz) * k.dsq;
    Hor3 a[1];
    horner3_block<NP2, PGH, 1, 4>(lo3, Pn, &x, &y, &z, a);
    hemit<PGH>(a[0], k.dsq, v);
    add_out<NC>(out, pa, k.nd, nc, ind, v);
    return;
  }
  // two points per thread, two rows in flight
  const bool two = tb < T.n;
  const int pb = T.i0 + (two ? tb : ta);
  const double x[2] = {(pts[3 * pa] - cx) * k.dsq, (pts[3 * pb] - cx) * k.dsq};
  const double y[2] = {(pts[3 * pa + 1] - cy) * k.dsq, (pts[3 * pb + 1] - cy) * k.dsq};
  const double z[2] = {(pts[3 * pa + 2] - cz) * k.dsq, (pts[3 * pb + 2] - cz) * k.dsq};
  Hor3 a[2];
  horner3_block<NP2, PGH, 2, 2>(lo3, Pn, x, y, z, a);
  hemit<PGH>(a[0], k.dsq, v);
  add_out<NC>(out, pa, k.nd, nc, ind, v);
  if (two) {
    hemit<PGH>(a[1], k.dsq, v);
    add_out<NC>(out, pb, k.nd, nc, ind, v);
  }
}

// ------------------------------------------------------------ (c) eval, 3D Taylor in shared memory
// One CTA per chunk of an evaluation leaf: plane wave -> Taylor
// (g3dpw2local_real_vec, g3drouts.f:1774-1938) with x and y passes over the
// positive half (mirror pre-add) and the z pass over the stored half, then
// Horner evaluation, two points per thread.
template <int PGH>
__global__ void __launch_bounds__(512) k_eval3d_taylor_smem(KP k, const EvalTask* __restrict__ tasks) {
  constexpr int NC = ncomp<3, PGH>();
  const EvalTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  const int npw = k.npw, n2 = k.n2;
  const int Pn = T.p + 1, P2 = Pn * Pn;
  extern __shared__ double sm[];
  const size_t szA = max((size_t)2 * Pn * npw * n2, (size_t)P2 * Pn);
  double2* U1 = reinterpret_cast<double2*>(sm);                       // [(a npw + m2) n2 + m1]
  double* lo = sm;                                                    // overwrites U1
  double2* U2 = reinterpret_cast<double2*>(sm + ((szA + 1) & ~size_t(1)));  // [(a P + b) n2 + m1]
  const double2* L = k.loc + ((size_t)T.slot * k.nd + ind) * k.nexp;
  for (int idx = threadIdx.x; idx < Pn * npw * n2; idx += blockDim.x) {
    const int m1 = idx % n2, r = idx / n2, m2 = r % npw, a = r / npw;
    const double2* row = L + (size_t)npw * (m2 + (size_t)npw * m1);
    const double sg = (a & 1) ? -1.0 : 1.0;
    double2 s = make_double2(0.0, 0.0);
    for (int m = 0; m < n2; m++) {
      const double h = k.x2l[a * npw + n2 + m];
      const double2 u = row[n2 + m], v = row[n2 - 1 - m];
      s.x = fma(h, fma(sg, v.x, u.x), s.x);
      s.y = fma(h, fma(sg, v.y, u.y), s.y);
    }
    U1[idx] = rot(s, a);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < P2 * n2; idx += blockDim.x) {
    const int m1 = idx % n2, r = idx / n2, b = r % Pn, a = r / Pn;
    const double sg = (b & 1) ? -1.0 : 1.0;
    double2 s = make_double2(0.0, 0.0);
    for (int m = 0; m < n2; m++) {
      const double h = k.x2l[b * npw + n2 + m];
      const double2 u = U1[((size_t)a * npw + n2 + m) * n2 + m1], v = U1[((size_t)a * npw + n2 - 1 - m) * n2 + m1];
      s.x = fma(h, fma(sg, v.x, u.x), s.x);
      s.y = fma(h, fma(sg, v.y, u.y), s.y);
    }
    U2[idx] = rot(s, b);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < P2 * Pn; idx += blockDim.x) {
    const int a = idx % Pn, r = idx / Pn, b = r % Pn, c = r / Pn;
    double2 s = make_double2(0.0, 0.0);
    for (int m1 = 0; m1 < n2; m1++) {
      const double h = k.x2l[c * npw + m1];
      const double2 v = U2[((size_t)a * Pn + b) * n2 + m1];
      s.x = fma(h, v.x, s.x);
      s.y = fma(h, v.y, s.y);
    }
    lo[idx] = 2.0 * rot(s, c).x;
  }
  __syncthreads();
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const int nc = T.set ? k.nc_t : k.nc_s;
  const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1], cz = k.centers[3 * T.box + 2];
  for (int i = threadIdx.x; i < T.n; i += blockDim.x) {
    const int ip = T.i0 + i;
    double v[NC];
    horner3_rt<PGH>(lo, Pn, Pn, (pts[3 * ip] - cx) * k.dsq, (pts[3 * ip + 1] - cy) * k.dsq,
                    (pts[3 * ip + 2] - cz) * k.dsq, k.dsq, v);
    add_out<NC>(out, ip, k.nd, nc, ind, v);
  }
}

// ------------------------------------------------------------ (a) form, 3D direct
// pw[k3,k2,k1] = sum_i q_i w(k3) e^{-i t x} w(k2) e^{-i t y} w(k1) e^{-i t z}
// (g3dformpwc_vec, g3drouts.f:1950-2038).  One CTA per (leaf, density);
// sources in chunks of FORM_CH, each with its three factor rows built once
// in shared memory; a thread owns expansion rows (k1, k2) for one block of 8
// consecutive k3 (its block fixed, its rows strided), so each source costs
// one row product and 8 complex FMAs per item, and the chunks' sums are added
// to the slot in chunk order.
__global__ void __launch_bounds__(256) k_form3d_pw(KP k, const FormTask* __restrict__ tasks) {
  const FormTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  const int npw = k.npw, n2 = k.n2;
  extern __shared__ double sm[];
  double2* F1 = reinterpret_cast<double2*>(sm);      // [FORM_CH][npw] (+ 8 padding)
  double2* F2 = F1 + FORM_CH * npw + 8;                // [FORM_CH][npw]
  double2* F3 = F2 + FORM_CH * npw;                    // [FORM_CH][n2], charge folded in
  const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1], cz = k.centers[3 * T.box + 2];
  double2* out = k.mp + ((size_t)T.slot * k.nd + ind) * k.nexp;
  // this thread's k3 block and first row; rows advance by rstep.  The block
  // is the slow index, so a warp's lanes share it (the k3 factors are
  // broadcast loads) and take consecutive rows
  const int nmb = (npw + 7) / 8, rstep = blockDim.x / nmb, mb = threadIdx.x / rstep;
  const int row0 = threadIdx.x - mb * rstep, nrow = n2 * npw;
  // dipoles (g3dformpwd_vec / g3dformpwcd_vec, g3drouts.f:2042-2262): three
  // columns per source, the factor of one dimension times v_d (-i t dsq)
  // in each (as dip3_coef), 10 sources per chunk
  const int vc = k.ifdipole ? 3 : 1, chs = FORM_CH / vc;
  for (int c0 = 0; c0 < T.n; c0 += chs) {
    const int m = vc * min(chs, T.n - c0);
    __syncthreads();
    if (threadIdx.x < m) {
      const int i = T.s0 + c0 + threadIdx.x / vc, col = threadIdx.x % vc;
      const double x = (k.src[3 * i] - cx) * k.dsq, y = (k.src[3 * i + 1] - cy) * k.dsq,
                   z = (k.src[3 * i + 2] - cz) * k.dsq;
      double dv[3] = {0.0, 0.0, 0.0}, ca[3], cb[3];
      if (k.ifdipole) src_dipole<3>(k, i, ind, dv);
      const double q = k.ifdipole ? src_charge(k, i, ind) : k.chg[(size_t)i * k.nd + ind];
      for (int d = 0; d < 3; d++) dip3_coef(col, d, q, dv, ca[d], cb[d]);
      // positive node m: t = (2m+1) t1 at index n2+m; its mirror n2-1-m
      double2 ex = cexpi(-k.t1 * x), ey = cexpi(-k.t1 * y), ez = cexpi(-k.t1 * z);
      const double2 exx = cmul(ex, ex), eyy = cmul(ey, ey), ezz = cmul(ez, ez);
      double2* f1 = F1 + threadIdx.x * npw;
      double2* f2 = F2 + threadIdx.x * npw;
      double2* f3 = F3 + threadIdx.x * n2;
      for (int mm = 0; mm < n2; mm++) {
        const double w = k.ws[n2 + mm];
        double2 a = make_double2(ex.x * w, ex.y * w), b = make_double2(ey.x * w, ey.y * w),
                c = make_double2(ez.x * w * q, ez.y * w * q);
        if (k.ifdipole) {
          // ca f + cb f (-i t dsq) per dimension, f = w e^{-i t x}
          const double td = (2 * mm + 1) * k.t1 * k.dsq;
          auto mix = [td](double2 f, double p0, double p1) {
            return make_double2(fma(p0, f.x, p1 * td * f.y), fma(p0, f.y, -p1 * td * f.x));
          };
          a = mix(a, ca[0], cb[0]);
          b = mix(b, ca[1], cb[1]);
          c = mix(make_double2(ez.x * w, ez.y * w), ca[2], cb[2]);
        }
        f1[n2 + mm] = a; f1[n2 - 1 - mm] = make_double2(a.x, -a.y);
        f2[n2 + mm] = b; f2[n2 - 1 - mm] = make_double2(b.x, -b.y);
        f3[n2 - 1 - mm] = make_double2(c.x, -c.y);
        ex = cmul(ex, exx); ey = cmul(ey, eyy); ez = cmul(ez, ezz);
      }
    }
    __syncthreads();
    if (mb >= nmb) continue;
    int i1 = 0, i2 = row0;
    while (i2 >= npw) {
      i2 -= npw;
      i1++;
    }
    for (int row = row0; row < nrow; row += rstep) {
      double2 acc[8];
#pragma unroll
      for (int j = 0; j < 8; j++) acc[j] = make_double2(0.0, 0.0);
      for (int t = 0; t < m; t++) {
        const double2 yz = cmul(F2[t * npw + i2], F3[t * n2 + i1]);
        const double2* f1 = F1 + t * npw + 8 * mb;
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] = cfma(f1[j], yz, acc[j]);
      }
      double2* o = out + (size_t)row * npw + 8 * mb;
#pragma unroll
      for (int j = 0; j < 8; j++)
        if (8 * mb + j < npw) {
          if (c0 == 0) {
            o[j] = acc[j];
          } else {
            const double2 p = o[j];
            o[j] = make_double2(p.x + acc[j].x, p.y + acc[j].y);
          }
        }
      i2 += rstep;
      while (i2 >= npw) {
        i2 -= npw;
        i1++;
      }
    }
  }
  if (T.n == 0)  // no sources: a zero expansion
    for (int e = threadIdx.x; e < k.nexp; e += blockDim.x) out[e] = make_double2(0.0, 0.0);
}

// 2D plane-wave expansion of a box formed directly from its sources: the
// exact sum that the NUFFT scheme computes with a type-1 NUFFT
// (g2dformpwc_vec, 2d/nufft/src/g2drouts.f:1234-1307),
//   mp[a + n2 b] = sum_s q_s ws_a ws_b exp(-i (t_a x_s + t_b y_s)),
// a over the n2 positive x nodes, b over every y node (positive half first,
// the layout of the plane-wave form and of k_eval2d).  One CTA per (box,
// density); per chunk of FORM_CH sources the first threads build one
// source's factor rows each in shared memory (the phases by the recurrence
// e^{-i t1 x} (e^{-2 i t1 x})^m, the charge folded into the x row), then
// every thread sums its own coefficients over the chunk.
__global__ void __launch_bounds__(256) k_form2d_pw(KP k, const FormTask* __restrict__ tasks) {
  const FormTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  const int npw = k.npw, n2 = k.n2, nexp = k.nexp;
  extern __shared__ double sm[];
  double2* FX = reinterpret_cast<double2*>(sm);  // [FORM_CH][n2]
  double2* FY = FX + FORM_CH * n2;               // [FORM_CH][npw]
  const double cx = k.centers[2 * T.box], cy = k.centers[2 * T.box + 1];
  double2* out = k.mp + ((size_t)T.slot * k.nd + ind) * nexp;
  for (int c0 = 0; c0 < T.n; c0 += FORM_CH) {
    const int m = min(FORM_CH, T.n - c0);
    __syncthreads();
    if (threadIdx.x < m) {
      const int i = T.s0 + c0 + threadIdx.x;
      const double x = (k.src[2 * i] - cx) * k.dsq, y = (k.src[2 * i + 1] - cy) * k.dsq;
      const double q = k.chg[(size_t)i * k.nd + ind];
      double2 ex = cexpi(-k.t1 * x), ey = cexpi(-k.t1 * y);
      const double2 exx = cmul(ex, ex), eyy = cmul(ey, ey);
      double2* fx = FX + threadIdx.x * n2;
      double2* fy = FY + threadIdx.x * npw;
      for (int mm = 0; mm < n2; mm++) {
        const double w = k.ws[mm];  // node (2 mm + 1) t1; the weights are even in t
        fx[mm] = make_double2(ex.x * w * q, ex.y * w * q);
        const double2 b = make_double2(ey.x * w, ey.y * w);
        fy[mm] = b;
        fy[n2 + mm] = make_double2(b.x, -b.y);
        ex = cmul(ex, exx);
        ey = cmul(ey, eyy);
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nexp; e += blockDim.x) {
      const int a = e % n2, b = e / n2;
      double2 acc = make_double2(0.0, 0.0);
      for (int t = 0; t < m; t++) acc = cfma(FX[t * n2 + a], FY[t * npw + b], acc);
      if (c0 == 0) {
        out[e] = acc;
      } else {
        const double2 p = out[e];
        out[e] = make_double2(p.x + acc.x, p.y + acc.y);
      }
    }
  }
  if (T.n == 0)  // no sources: a zero expansion
    for (int e = threadIdx.x; e < nexp; e += blockDim.x) out[e] = make_double2(0.0, 0.0);
}

// ------------------------------------------------------------ (b) shifts
// merge: parent = sum over its children of child * W (g2dshiftpw_vec)
__global__ void k_merge(KP k, const MergeGroup* __restrict__ groups, const ShiftTask* __restrict__ tasks) {
  const MergeGroup G = groups[blockIdx.x];
  const size_t per = (size_t)k.nd * k.nexp;
  for (size_t e = (size_t)blockIdx.y * blockDim.x + threadIdx.x; e < per; e += (size_t)gridDim.y * blockDim.x) {
    const int ee = (int)(e % k.nexp);
    double2 a = make_double2(0.0, 0.0);
    for (int t = G.beg; t < G.beg + G.cnt; t++) {
      const ShiftTask S = tasks[t];
      a = cfma(k.mp[(size_t)S.src * per + e], k.wms[(size_t)S.table * k.nexp + ee], a);
    }
    k.mp[(size_t)G.dst * per + e] = a;
  }
}
// mp -> loc at the cut level: sum over the plane-wave list plus the box's own
// multipole (g2dshiftpw_vec + g2dcopypwexp_vec, fgt2d.f:1048-1060)
__global__ void k_m2l(KP k, const M2LTask* __restrict__ tasks, const M2LNbr* __restrict__ nbr) {
  const M2LTask T = tasks[blockIdx.x];
  const size_t per = (size_t)k.nd * k.nexp;
  for (size_t e = (size_t)blockIdx.y * blockDim.x + threadIdx.x; e < per; e += (size_t)gridDim.y * blockDim.x) {
    const int ee = (int)(e % k.nexp);
    double2 a = make_double2(0.0, 0.0);
    for (int t = T.off; t < T.off + T.cnt; t++) {
      const M2LNbr N = nbr[t];
      a = cfma(k.mp[(size_t)N.mp * per + e], k.wsh[(size_t)N.shift * k.nexp + ee], a);
    }
    if (T.self_mp >= 0) {
      const double2 s = k.mp[(size_t)T.self_mp * per + e];
      a.x += s.x;
      a.y += s.y;
    }
    k.loc[(size_t)T.loc * per + e] = a;
  }
}
// One CTA per (task, block of SHU * 256 coefficients), every density in
// turn; a thread's SHU loads of the parent and of the table are issued
// before the first product.
constexpr int SHU = 4;
// split: child = parent * conj(W), W the merge factor of that child
__global__ void __launch_bounds__(256) k_split(KP k, const ShiftTask* __restrict__ tasks) {
  const ShiftTask S = tasks[blockIdx.x];
  const size_t per = (size_t)k.nd * k.nexp;
  const int e0 = blockIdx.y * 256 * SHU + threadIdx.x;
  const double2* w = k.wms + (size_t)S.table * k.nexp;
  for (int ind = 0; ind < k.nd; ind++) {
    const double2* src = k.loc + (size_t)S.src * per + (size_t)ind * k.nexp;
    double2* dst = k.loc + (size_t)S.dst * per + (size_t)ind * k.nexp;
    double2 a[SHU], b[SHU];
#pragma unroll
    for (int u = 0; u < SHU; u++) {
      const int e = e0 + 256 * u;
      if (e < k.nexp) {
        a[u] = src[e];
        b[u] = __ldg(w + e);
      }
    }
#pragma unroll
    for (int u = 0; u < SHU; u++) {
      const int e = e0 + 256 * u;
      if (e < k.nexp) dst[e] = cmulc(a[u], b[u]);
    }
  }
}

// ------------------------------------------------------------ (c) eval, plane-wave route derivatives
// A pair of nodes +t, -t with coefficients A (of e^{itx}) and B (of e^{-itx})
// contributes A w + B conj(w), w = e^{itx}; its x derivatives are
// i t (A w - B conj(w)) and -t^2 (A w + B conj(w)).  PwAcc keeps
//   S0 = sum (A w + B w*),  S1 = sum t (A w - B w*),  S2 = sum t^2 (A w + B w*)
// (the derivative orders the evaluation needs), so that d/dx = i S1 and
// d2/dx2 = -S2 (the ww1x / ww1xx factors of g2dpwevalg_vec / g2dpwevalh_vec,
// g2drouts.f:1973-2200, and g3dpwevalg/h_vec, g3drouts.f:2369-2660).
template <int ORD>
struct PwAcc {
  double2 s[ORD + 1];
  __device__ __forceinline__ PwAcc() {
#pragma unroll
    for (int i = 0; i <= ORD; i++) s[i] = make_double2(0.0, 0.0);
  }
  // add A w + B conj(w) at node t
  __device__ __forceinline__ void add(double2 A, double2 B, double2 w, double t) {
    if (ORD == 0) {  // the potential alone: two complex FMAs
      s[0] = cfmac(B, w, cfma(A, w, s[0]));
      return;
    }
    const double2 p = cmul(A, w), m = cmulc(B, w);  // A w, B conj(w)
    const double2 sp = make_double2(p.x + m.x, p.y + m.y);
    s[0].x += sp.x;
    s[0].y += sp.y;
    if (ORD >= 1) {
      s[1].x = fma(t, p.x - m.x, s[1].x);
      s[1].y = fma(t, p.y - m.y, s[1].y);
    }
    if (ORD >= 2) {
      const double t2 = t * t;
      s[2].x = fma(t2, sp.x, s[2].x);
      s[2].y = fma(t2, sp.y, s[2].y);
    }
  }
};

// ------------------------------------------------------------ (c) eval, 2D plane-wave route
// One CTA per (leaf, point set, density): direct plane-wave sum at every point
// with e^{i t x} built by the recurrence of g2dpwevalp_vec (g2drouts.f:1887-1966),
// on the levels where the reference picks it (nlocal > 50, fgt2d.f:1166).
// The stored half is x > 0; y runs over both signs.  With z_j = sum over x
// nodes of e^{i t_x x} t_x^a (y-sum of derivative order b), the outputs are
//   pot = 2 Re z(0,0), g_x = -2 Im z(1,0), g_y = -2 Im z(0,1),
//   h_xx = -2 Re z(2,0), h_xy = -2 Re z(1,1), h_yy = -2 Re z(0,2)
// times dsq per derivative.
template <int PGH>
__global__ void __launch_bounds__(256) k_eval2d(KP k, const EvalTask* __restrict__ tasks) {
  constexpr int NC = ncomp<2, PGH>(), ORD = PGH - 1;
  const EvalTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  const int n2 = k.n2;
  const double2* L = k.loc + ((size_t)T.slot * k.nd + ind) * k.nexp;
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const int nc = T.set ? k.nc_t : k.nc_s;
  const double cx = k.centers[2 * T.box], cy = k.centers[2 * T.box + 1];
  for (int i = threadIdx.x; i < T.n; i += blockDim.x) {
    const int ip = T.i0 + i;
    const double x = (pts[2 * ip] - cx) * k.dsq, y = (pts[2 * ip + 1] - cy) * k.dsq;
    const double2 ex = cexpi(k.t1 * x), ey = cexpi(k.t1 * y);
    const double2 exx = cmul(ex, ex), eyy = cmul(ey, ey);
    // z[0] = (0,0), z[1] = (1,0), z[2] = (0,1), z[3] = (2,0), z[4] = (1,1), z[5] = (0,2)
    double2 z[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) z[c] = make_double2(0.0, 0.0);
    double2 w1 = ex;
    for (int kx = 0; kx < n2; kx++) {
      const double tx = (2 * kx + 1) * k.t1;
      PwAcc<ORD> sy;
      double2 w2 = ey;
      for (int ky = 0; ky < n2; ky++) {
        sy.add(L[kx + n2 * ky], L[kx + n2 * (ky + n2)], w2, (2 * ky + 1) * k.t1);
        w2 = cmul(w2, eyy);
      }
      const double2 a0 = cmul(sy.s[0], w1);
      z[0].x += a0.x;
      z[0].y += a0.y;
      if (PGH >= 2) {
        const double2 a1 = cmul(sy.s[ORD >= 1 ? 1 : 0], w1);
        z[1].x = fma(tx, a0.x, z[1].x);
        z[1].y = fma(tx, a0.y, z[1].y);
        z[2].x += a1.x;
        z[2].y += a1.y;
        if (PGH >= 3) {
          const double2 a2 = cmul(sy.s[ORD >= 2 ? 2 : 0], w1);
          z[3].x = fma(tx * tx, a0.x, z[3].x);
          z[4].x = fma(tx, a1.x, z[4].x);
          z[5].x += a2.x;
        }
      }
      w1 = cmul(w1, exx);
    }
    double v[NC];
    v[0] = 2.0 * z[0].x;
    if (PGH >= 2) {
      v[1] = -2.0 * z[1].y * k.dsq;
      v[2] = -2.0 * z[2].y * k.dsq;
    }
    if (PGH >= 3) {
      const double d2 = k.dsq * k.dsq;
      v[3] = -2.0 * z[3].x * d2;
      v[4] = -2.0 * z[4].x * d2;
      v[5] = -2.0 * z[5].x * d2;
    }
    add_out<NC>(out, ip, k.nd, nc, ind, v);
  }
}

// ------------------------------------------------------------ (c) eval, 3D
// Taylor route, persistent CTAs: plane wave -> Taylor through the scratch
// slab (x, y passes) and a z pass into shared memory
// (g3dpw2local_real_vec, g3drouts.f:1774-1938), then Horner evaluation.
template <int PGH>
__global__ void __launch_bounds__(256) k_eval3d_taylor(KP k, const EvalTask* __restrict__ tasks, int ntasks,
                                                       double2* __restrict__ scratch, size_t slab) {
  constexpr int NC = ncomp<3, PGH>();
  const int npw = k.npw, n2 = k.n2;
  double2* U1 = scratch + slab * blockIdx.x;
  for (int w = blockIdx.x; w < ntasks * k.nd; w += gridDim.x) {
    const EvalTask T = tasks[w / k.nd];
    const int ind = w % k.nd;
    const int Pn = T.p + 1, P2 = Pn * Pn;
    double2* U2 = U1 + (size_t)Pn * npw * n2;
    double* lo = reinterpret_cast<double*>(U2 + (size_t)P2 * n2);  // [P^3]
    const double2* L = k.loc + ((size_t)T.slot * k.nd + ind) * k.nexp;
    // x pass: U1[(a npw + m2) n2 + m1] = i^a sum_m3 x2l(m3,a) L[m3 + npw (m2 + npw m1)]
    for (int idx = threadIdx.x; idx < Pn * npw * n2; idx += blockDim.x) {
      const int m1 = idx % n2, r = idx / n2, m2 = r % npw, a = r / npw;
      double2 s = make_double2(0.0, 0.0);
      const double2* row = L + (size_t)npw * (m2 + (size_t)npw * m1);
      for (int m3 = 0; m3 < npw; m3++) {
        const double h = k.x2l[a * npw + m3];
        const double2 v = row[m3];
        s.x = fma(h, v.x, s.x);
        s.y = fma(h, v.y, s.y);
      }
      U1[idx] = rot(s, a);
    }
    __syncthreads();
    // y pass: U2[(a P + b) n2 + m1] = i^b sum_m2 x2l(m2,b) U1[(a npw + m2) n2 + m1]
    for (int idx = threadIdx.x; idx < P2 * n2; idx += blockDim.x) {
      const int m1 = idx % n2, r = idx / n2, b = r % Pn, a = r / Pn;
      double2 s = make_double2(0.0, 0.0);
      for (int m2 = 0; m2 < npw; m2++) {
        const double h = k.x2l[b * npw + m2];
        const double2 v = U1[((size_t)a * npw + m2) * n2 + m1];
        s.x = fma(h, v.x, s.x);
        s.y = fma(h, v.y, s.y);
      }
      U2[idx] = rot(s, b);
    }
    __syncthreads();
    // z pass over the half: lo[a + P (b + P c)] = 2 Re(i^c sum_m1 x2l(m1,c) U2[(a P + b) n2 + m1])
    for (int idx = threadIdx.x; idx < P2 * Pn; idx += blockDim.x) {
      const int a = idx % Pn, r = idx / Pn, b = r % Pn, c = r / Pn;
      double2 s = make_double2(0.0, 0.0);
      for (int m1 = 0; m1 < n2; m1++) {
        const double h = k.x2l[c * npw + m1];
        const double2 v = U2[((size_t)a * Pn + b) * n2 + m1];
        s.x = fma(h, v.x, s.x);
        s.y = fma(h, v.y, s.y);
      }
      lo[idx] = 2.0 * rot(s, c).x;
    }
    __syncthreads();
    const double* pts = T.set ? k.trg : k.src;
    double* out = T.set ? k.pottarg : k.pot;
    const int nc = T.set ? k.nc_t : k.nc_s;
    const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1], cz = k.centers[3 * T.box + 2];
    for (int i = threadIdx.x; i < T.n; i += blockDim.x) {
      const int ip = T.i0 + i;
      double v[NC];
      horner3_rt<PGH>(lo, Pn, Pn, (pts[3 * ip] - cx) * k.dsq, (pts[3 * ip + 1] - cy) * k.dsq,
                      (pts[3 * ip + 2] - cz) * k.dsq, k.dsq, v);
      add_out<NC>(out, ip, k.nd, nc, ind, v);
    }
    __syncthreads();
  }
}

// PW route (g3dpwevalp_vec, g3drouts.f:2268-2362): one CTA per task.  x and y
// run over both signs (PwAcc), z over the stored half, whose nodes are
// negative: e^{-i t z} has z derivatives -i t and -t^2.  With Y(a,b) the x/y
// sums of derivative orders a, b and F(a,b) = sum_z Y(a,b) e^{-itz},
// G(a,b) = sum_z t Y(a,b) e^{-itz}, Gz2 = sum_z t^2 Y(0,0) e^{-itz}:
//   pot = 2 Re F00, g = (-2 Im F10, -2 Im F01, 2 Im G00),
//   h_xx, h_yy, h_zz = -2 Re F20, -2 Re F02, -2 Re Gz2,
//   h_xy, h_xz, h_yz = -2 Re F11, 2 Re G10, 2 Re G01   (times dsq per derivative).
template <int PGH>
__global__ void __launch_bounds__(256) k_eval3d_pw(KP k, const EvalTask* __restrict__ tasks) {
  constexpr int NC = ncomp<3, PGH>(), ORD = PGH - 1;
  const EvalTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  const int npw = k.npw, n2 = k.n2;
  const double2* L = k.loc + ((size_t)T.slot * k.nd + ind) * k.nexp;
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const int nc = T.set ? k.nc_t : k.nc_s;
  const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1], cz = k.centers[3 * T.box + 2];
  for (int i = threadIdx.x; i < T.n; i += blockDim.x) {
    const int ip = T.i0 + i;
    const double x = (pts[3 * ip] - cx) * k.dsq, y = (pts[3 * ip + 1] - cy) * k.dsq,
                 z = (pts[3 * ip + 2] - cz) * k.dsq;
    const double2 ex = cexpi(k.t1 * x), ey = cexpi(k.t1 * y), ez = cexpi(k.t1 * z);
    const double2 exx = cmul(ex, ex), eyy = cmul(ey, ey), ezz = cmul(ez, ez);
    // acc: [0] F00, [1] F10, [2] F01, [3] G00, [4] F20, [5] F02, [6] Gz2, [7] F11, [8] G10, [9] G01
    double2 acc[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) acc[c] = make_double2(0.0, 0.0);
    double2 w3 = ez;
    for (int mz = 0; mz < n2; mz++) {
      // z index n2-1-mz holds node -(2 mz + 1) t1
      const double tz = (2 * mz + 1) * k.t1;
      // Y[b][a]: y order b of the x order a sums
      PwAcc<ORD> Y[ORD + 1];
      double2 w2 = ey;
      for (int my = 0; my < n2; my++) {
        const double ty = (2 * my + 1) * k.t1;
        const double2* rp = L + (size_t)npw * ((n2 + my) + (size_t)npw * (n2 - 1 - mz));
        const double2* rm = L + (size_t)npw * ((n2 - 1 - my) + (size_t)npw * (n2 - 1 - mz));
        PwAcc<ORD> sp, sn;
        double2 w1 = ex;
        for (int mx = 0; mx < n2; mx++) {
          const double tx = (2 * mx + 1) * k.t1;
          sp.add(rp[n2 + mx], rp[n2 - 1 - mx], w1, tx);
          sn.add(rm[n2 + mx], rm[n2 - 1 - mx], w1, tx);
          w1 = cmul(w1, exx);
        }
#pragma unroll
        for (int a = 0; a <= ORD; a++) Y[a].add(sp.s[a], sn.s[a], w2, ty);
        w2 = cmul(w2, eyy);
      }
      // conj(w3) factors
      const double2 f00 = cmulc(Y[0].s[0], w3);
      acc[0].x += f00.x;
      acc[0].y += f00.y;
      if (PGH >= 2) {
        const double2 f10 = cmulc(Y[ORD >= 1 ? 1 : 0].s[0], w3), f01 = cmulc(Y[0].s[ORD >= 1 ? 1 : 0], w3);
        acc[1].y += f10.y;
        acc[2].y += f01.y;
        acc[3].y = fma(tz, f00.y, acc[3].y);
        if (PGH >= 3) {
          const double2 f20 = cmulc(Y[ORD >= 2 ? 2 : 0].s[0], w3), f02 = cmulc(Y[0].s[ORD >= 2 ? 2 : 0], w3);
          const double2 f11 = cmulc(Y[ORD >= 1 ? 1 : 0].s[ORD >= 1 ? 1 : 0], w3);
          acc[4].x += f20.x;
          acc[5].x += f02.x;
          acc[6].x = fma(tz * tz, f00.x, acc[6].x);
          acc[7].x += f11.x;
          acc[8].x = fma(tz, f10.x, acc[8].x);
          acc[9].x = fma(tz, f01.x, acc[9].x);
        }
      }
      w3 = cmul(w3, ezz);
    }
    double v[NC];
    v[0] = 2.0 * acc[0].x;
    if (PGH >= 2) {
      v[1] = -2.0 * acc[1].y * k.dsq;
      v[2] = -2.0 * acc[2].y * k.dsq;
      v[3] = 2.0 * acc[3].y * k.dsq;
    }
    if (PGH >= 3) {
      const double d2 = k.dsq * k.dsq;
      v[4] = -2.0 * acc[4].x * d2;
      v[5] = -2.0 * acc[5].x * d2;
      v[6] = -2.0 * acc[6].x * d2;
      v[7] = -2.0 * acc[7].x * d2;
      v[8] = 2.0 * acc[8].x * d2;
      v[9] = 2.0 * acc[9].x * d2;
    }
    add_out<NC>(out, ip, k.nd, nc, ind, v);
  }
}

// ------------------------------------------------------------ (d) near field
// Source list of a near-field task: the concatenation of its source ranges
// (leaves of its list1).  A warp walks it in batches of at most CAP sources:
// ranges are read 32 at a time (one per lane) and prefix-summed with
// shuffles; for the batch starting at b0 each lane maps its slots
// b0 + lane + 32 u to source indices by a binary search over the lanes'
// prefixes, so all loads of a batch can be in flight together (a range at a
// time would serialise one load round trip per range).
// ------------------------------------------------------------ (d) near field, kernels
// One warp per chunk of <= 32 evaluation points (g2d_directcp_vec,
// g2ddirect.f:32-76; g3d_directcp_vec, g3ddirect.f:3-49): the chunk's source
// ranges are staged through the warp's shared memory in batches of 256, and
// g lanes per point (g n <= 32) split the sources of that point.
// pot += q exp(-r^2/delta) when r^2 < dmax, all in FP64; with PGH > 1 the
// gradient and Hessian per pair as g2d_directcg/ch_vec (g2ddirect.f:83-212)
// and g3d_directcg/ch_vec (g3ddirect.f:56-203): with rfac = -2/delta and
// d = target - source, grad += rfac d_i r, hess_ii += (rfac + (rfac d_i)^2) r,
// hess_ij += (rfac d_i)(rfac d_j) r, r = q exp(-|d|^2/delta).
template <int DIM, int PGH>
__device__ __forceinline__ void pair_terms(double* acc, double r, const double* d, double rfac) {
  acc[0] += r;
  if (PGH >= 2) {
    double g[DIM];
#pragma unroll
    for (int i = 0; i < DIM; i++) {
      g[i] = rfac * d[i];
      acc[1 + i] = fma(g[i], r, acc[1 + i]);
    }
    if (PGH >= 3) {
      double* h = acc + 1 + DIM;
      if (DIM == 2) {
        h[0] = fma(fma(g[0], g[0], rfac), r, h[0]);
        h[1] = fma(g[0] * g[1], r, h[1]);
        h[2] = fma(fma(g[1], g[1], rfac), r, h[2]);
      } else {
        h[0] = fma(fma(g[0], g[0], rfac), r, h[0]);
        h[1] = fma(fma(g[1], g[1], rfac), r, h[1]);
        h[2] = fma(fma(g[DIM - 1], g[DIM - 1], rfac), r, h[2]);
        h[3] = fma(g[0] * g[1], r, h[3]);
        h[4] = fma(g[0] * g[DIM - 1], r, h[4]);
        h[5] = fma(g[1] * g[DIM - 1], r, h[5]);
      }
    }
  }
}
// Dipole terms per pair (g2d_directd{p,g,h}_vec, g2ddirect.f:217-420, and
// g3d_directd*_vec, g3ddirect.f:207-435), v = dipstr n, e = exp(-r^2/delta):
// with R = 2/delta, u = R (t - s), rinc = u.v,
//   pot += rinc e,  grad_a += g_a e with g_a = R v_a - rinc u_a,
//   hess_aa += (-R (u_a v_a + rinc) - g_a u_a) e,  hess_ab += (-R u_a v_b - g_a u_b) e.
template <int DIM, int PGH>
__device__ __forceinline__ void dip_terms(double* acc, double e, const double* d, const double* v,
                                          double R) {
  double u[DIM], rinc = 0.0;
#pragma unroll
  for (int a = 0; a < DIM; a++) {
    u[a] = R * d[a];
    rinc = fma(u[a], v[a], rinc);
  }
  acc[0] = fma(rinc, e, acc[0]);
  if (PGH >= 2) {
    double g[DIM];
#pragma unroll
    for (int a = 0; a < DIM; a++) {
      g[a] = fma(R, v[a], -rinc * u[a]);
      acc[1 + a] = fma(g[a], e, acc[1 + a]);
    }
    if (PGH >= 3) {
      double* h = acc + 1 + DIM;
      auto hd = [&](int a) { return -R * (u[a] * v[a] + rinc) - g[a] * u[a]; };
      auto ho = [&](int a, int b) { return -R * u[a] * v[b] - g[a] * u[b]; };
      if (DIM == 2) {
        h[0] = fma(hd(0), e, h[0]);
        h[1] = fma(ho(0, 1), e, h[1]);
        h[2] = fma(hd(1), e, h[2]);
      } else {
        h[0] = fma(hd(0), e, h[0]);
        h[1] = fma(hd(1), e, h[1]);
        h[2] = fma(hd(DIM - 1), e, h[2]);
        h[3] = fma(ho(0, 1), e, h[3]);
        h[4] = fma(ho(0, DIM - 1), e, h[4]);
        h[5] = fma(ho(1, DIM - 1), e, h[5]);
      }
    }
  }
}
// DIP: charges (when present) and dipoles, staged with the dipole vectors;
// 128 sources per batch so the staging stays within static shared memory.
template <int DIM, int PGH, bool DIP>
__global__ void __launch_bounds__(128) k_direct(KP k, const DirTask* __restrict__ tasks, int ntask,
                                                const SrcRange* __restrict__ ranges) {
  constexpr int NC = ncomp<DIM, PGH>();
  constexpr int CAP = DIP ? 128 : 256;  // sources staged per warp and batch
  constexpr int ROWS = DIP ? 2 * DIM + 1 : DIM + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * 4 + warp;
  __shared__ double ssm[4][ROWS * CAP];
  if (w >= ntask) return;  // whole warp leaves; no block-wide barrier below
  const DirTask T = tasks[w];
  const int ind = blockIdx.y;
  double* sx = ssm[warp];
  double* sy = sx + CAP;
  double* sz = sy + CAP;
  double* sq = sz + (DIM == 3 ? CAP : 0);
  double* sv = sq + CAP;  // [DIM][CAP] dipole vectors (DIP)
  // g lanes per point (g * n <= 32) split the sources of that point
  int g = 1;
  while (g * 2 * T.n <= 32) g *= 2;
  const int tt = lane / g, sub = lane - tt * g;
  const bool act = tt < T.n;
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const int nc = T.set ? k.nc_t : k.nc_s;
  const int ip = T.i0 + (act ? tt : 0);
  const double tx = pts[DIM * ip], ty = pts[DIM * ip + 1];
  const double tz = DIM == 3 ? pts[DIM * ip + 2] : 0.0;
  const double ninv = -1.0 / k.delta, rfac = -2.0 / k.delta;
  double acc[NC];
#pragma unroll
  for (int c = 0; c < NC; c++) acc[c] = 0.0;
  for (int rc = 0; rc < T.cnt; rc += 32) {
    const RangeChunk C = load_range_chunk(ranges, T.off, T.cnt, rc, lane);
    for (int b0 = 0; b0 < C.tot; b0 += CAP) {
      const int m = min(CAP, C.tot - b0);
      int js[CAP / 32];
#pragma unroll
      for (int u = 0; u < CAP / 32; u++) js[u] = range_slot_source(C, b0 + lane + 32 * u);
      __syncwarp();
#pragma unroll
      for (int u = 0; u < CAP / 32; u++) {
        const int t = lane + 32 * u;
        if (t < m) {
          const int j = js[u];
          sx[t] = k.src[DIM * j];
          sy[t] = k.src[DIM * j + 1];
          if (DIM == 3) sz[t] = k.src[DIM * j + 2];
          if (DIP) {
            sq[t] = src_charge(k, j, ind);
            double v[DIM];
            src_dipole<DIM>(k, j, ind, v);
#pragma unroll
            for (int a = 0; a < DIM; a++) sv[a * CAP + t] = v[a];
          } else {
            sq[t] = k.chg[(size_t)j * k.nd + ind];
          }
        }
      }
      __syncwarp();
      if (act) {
#pragma unroll 4
        for (int t = sub; t < m; t += g) {
          const double dx = tx - sx[t], dy = ty - sy[t];
          double rr = fma(dx, dx, dy * dy);
          double dz = 0.0;
          if (DIM == 3) {
            dz = tz - sz[t];
            rr = fma(dz, dz, rr);
          }
          if (rr < k.dmax) {
            if (DIP) {
              const double e = exp(rr * ninv), d[3] = {dx, dy, dz};
              double v[DIM];
#pragma unroll
              for (int a = 0; a < DIM; a++) v[a] = sv[a * CAP + t];
              if (PGH == 1) acc[0] = fma(e, sq[t], acc[0]);
              else pair_terms<DIM, PGH>(acc, e * sq[t], d, rfac);
              dip_terms<DIM, PGH>(acc, e, d, v, -rfac);
            } else if (PGH == 1) {
              acc[0] = fma(exp(rr * ninv), sq[t], acc[0]);
            } else {
              const double d[3] = {dx, dy, dz};
              pair_terms<DIM, PGH>(acc, exp(rr * ninv) * sq[t], d, rfac);
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int c = 0; c < NC; c++)
    for (int o = 1; o < g; o <<= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
  if (act && sub == 0) add_out<NC>(out, ip, k.nd, nc, ind, acc);
}

// Scaled coordinates of the mixed near field, once per plan: (x - c) cs with
// c the root box's centre, as an FP32 pair (hi, lo) per dimension.
__global__ void k_mixed_coords(const double* __restrict__ x, int n, int dim, double c0, double c1, double c2,
                               double cs, float* __restrict__ f) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int d = 0; d < dim; d++) {
      const double v = (x[(size_t)dim * i + d] - (d == 0 ? c0 : d == 1 ? c1 : c2)) * cs;
      const float h = (float)v;
      f[(size_t)2 * dim * i + 2 * d] = h;
      f[(size_t)2 * dim * i + 2 * d + 1] = (float)(v - (double)h);
    }
}

// Mixed form of the near field (eps >= 1e-6): the same task structure with
// the pair arithmetic in FP32.  Coordinates are taken relative to the root
// box's centre, scaled by sqrt(log2(e) / delta) and split into a float pair
// (hi, lo) once per plan (k_mixed_coords), so dx = (t_hi - s_hi) + (t_lo -
// s_lo) carries about FP32 relative accuracy in dx itself (the hi parts of
// nearby points subtract exactly; the lo parts hold the rest to 2^-48 of the
// coordinate); the Gaussian is then
// 2^-(dx^2 + dy^2 (+ dz^2)) by ex2.approx.  Each lane holds NTL = 4 targets,
// so a staged source is read from shared memory once for four pairs; g lanes
// per target group (g * groups <= 32) split the sources.  Groups of four
// sources are summed in FP32 per target and added into FP64 accumulators.
// With PGH > 1 the FP32 partials are, per target, sum e q, sum e q d_i and
// (PGH = 3) sum e q d_i d_j in the scaled differences d = (x_t - x_s) cs;
// they become the gradient rfac/cs sum e q d_i and the Hessian
// rfac sum e q + (rfac/cs)^2 sum e q d_i^2 (diagonal), (rfac/cs)^2 sum e q d_i d_j
// in FP64 (the per-pair terms of g2d_directch_vec / g3d_directch_vec).
template <int DIM, int PGH>
__global__ void __launch_bounds__(128) k_direct_mixed(KP k, const DirTask* __restrict__ tasks, int ntask,
                                                      const SrcRange* __restrict__ ranges, double cs,
                                                      float amax) {
  constexpr int CAP = 256, NTL = PGH == 1 ? 4 : PGH == 2 ? 2 : 1;
  constexpr int NC = ncomp<DIM, PGH>();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * 4 + warp;
  __shared__ float fsm[4][(2 * DIM + 1) * CAP];
  if (w >= ntask) return;  // whole warp leaves; no block-wide barrier below
  const DirTask T = tasks[w];
  const int ind = blockIdx.y;
  float* sh = fsm[warp];           // [DIM][CAP] hi parts
  float* sl = sh + DIM * CAP;      // [DIM][CAP] lo parts
  float* sq = sl + DIM * CAP;      // [CAP] charges
  const int ngr = (T.n + NTL - 1) / NTL;
  int g = 1;
  while (g * 2 * ngr <= 32) g *= 2;
  const int tt = lane / g, sub = lane - tt * g;
  const bool act = tt < ngr;
  double* out = T.set ? k.pottarg : k.pot;
  const int nc = T.set ? k.nc_t : k.nc_s;
  const float* fp = T.set ? k.ftrg : k.fsrc;  // the points' FP32 (hi, lo) coordinates
  float th[NTL][DIM], tl[NTL][DIM];
  double acc[NTL][NC];
#pragma unroll
  for (int v = 0; v < NTL; v++) {
#pragma unroll
    for (int c = 0; c < NC; c++) acc[v][c] = 0.0;
    const int it = min(tt * NTL + v, T.n - 1);
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      th[v][d] = fp[(size_t)2 * DIM * (T.i0 + it) + 2 * d];
      tl[v][d] = fp[(size_t)2 * DIM * (T.i0 + it) + 2 * d + 1];
    }
  }
  for (int rc = 0; rc < T.cnt; rc += 32) {
   const RangeChunk C = load_range_chunk(ranges, T.off, T.cnt, rc, lane);
   for (int b0 = 0; b0 < C.tot; b0 += CAP) {
    const int m = min(CAP, C.tot - b0);
    int js[CAP / 32];
#pragma unroll
    for (int u = 0; u < CAP / 32; u++) js[u] = range_slot_source(C, b0 + lane + 32 * u);
    __syncwarp();
#pragma unroll
    for (int u = 0; u < CAP / 32; u++) {
      const int t = lane + 32 * u;
      if (t < m) {
        const int j = js[u];
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          const float2 hl = reinterpret_cast<const float2*>(k.fsrc)[(size_t)DIM * j + d];
          sh[d * CAP + t] = hl.x;
          sl[d * CAP + t] = hl.y;
        }
        sq[t] = (float)k.chg[(size_t)j * k.nd + ind];
      }
    }
    __syncwarp();
    if (act) {
      for (int t = sub; t < m; t += 4 * g) {
        float part[NTL][NC];
#pragma unroll
        for (int v = 0; v < NTL; v++)
#pragma unroll
          for (int c = 0; c < NC; c++) part[v][c] = 0.0f;
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int tu = t + u * g;
          if (tu < m) {
            float sH[DIM], sL[DIM];
#pragma unroll
            for (int d = 0; d < DIM; d++) {
              sH[d] = sh[d * CAP + tu];
              sL[d] = sl[d * CAP + tu];
            }
            const float q = sq[tu];
#pragma unroll
            for (int v = 0; v < NTL; v++) {
              float a = 0.0f, dd[DIM];
#pragma unroll
              for (int d = 0; d < DIM; d++) {
                dd[d] = (th[v][d] - sH[d]) + (tl[v][d] - sL[d]);
                a = fmaf(dd[d], dd[d], a);
              }
              const float e = ex2_approx(-a);
              if (PGH == 1) {
                part[v][0] = a < amax ? fmaf(e, q, part[v][0]) : part[v][0];
              } else if (a < amax) {
                const float r = e * q;
                part[v][0] += r;
#pragma unroll
                for (int d = 0; d < DIM; d++) part[v][1 + d] = fmaf(dd[d], r, part[v][1 + d]);
                if (PGH >= 3) {
                  float* h = part[v] + 1 + DIM;
                  if (DIM == 2) {
                    h[0] = fmaf(dd[0] * dd[0], r, h[0]);
                    h[1] = fmaf(dd[0] * dd[1], r, h[1]);
                    h[2] = fmaf(dd[1] * dd[1], r, h[2]);
                  } else {
                    h[0] = fmaf(dd[0] * dd[0], r, h[0]);
                    h[1] = fmaf(dd[1] * dd[1], r, h[1]);
                    h[2] = fmaf(dd[DIM - 1] * dd[DIM - 1], r, h[2]);
                    h[3] = fmaf(dd[0] * dd[1], r, h[3]);
                    h[4] = fmaf(dd[0] * dd[DIM - 1], r, h[4]);
                    h[5] = fmaf(dd[1] * dd[DIM - 1], r, h[5]);
                  }
                }
              }
            }
          }
        }
#pragma unroll
        for (int v = 0; v < NTL; v++)
#pragma unroll
          for (int c = 0; c < NC; c++) acc[v][c] += (double)part[v][c];
      }
    }
   }
  }
#pragma unroll
  for (int v = 0; v < NTL; v++)
#pragma unroll
    for (int c = 0; c < NC; c++)
      for (int o2 = 1; o2 < g; o2 <<= 1) acc[v][c] += __shfl_xor_sync(0xffffffffu, acc[v][c], o2);
  if (act && sub == 0) {
    // scaled sums -> physical: d = dx cs, rfac = -2/delta
    const double rfac = -2.0 / k.delta, c1 = rfac / cs, c2 = c1 * c1;
#pragma unroll
    for (int v = 0; v < NTL; v++) {
      const int it = tt * NTL + v;
      if (it >= T.n) continue;
      double w[NC];
      w[0] = acc[v][0];
      if (PGH >= 2)
#pragma unroll
        for (int d = 0; d < DIM; d++) w[1 + d] = c1 * acc[v][1 + d];
      if (PGH >= 3) {
        const double* h = acc[v] + 1 + DIM;
        double* hw = w + 1 + DIM;
        if (DIM == 2) {
          hw[0] = fma(c2, h[0], rfac * w[0]);
          hw[1] = c2 * h[1];
          hw[2] = fma(c2, h[2], rfac * w[0]);
        } else {
          hw[0] = fma(c2, h[0], rfac * w[0]);
          hw[1] = fma(c2, h[1], rfac * w[0]);
          hw[2] = fma(c2, h[2], rfac * w[0]);
          hw[3] = c2 * h[3];
          hw[4] = c2 * h[4];
          hw[5] = c2 * h[5];
        }
      }
      add_out<NC>(out, T.i0 + it, k.nd, nc, ind, w);
    }
  }
}

// ------------------------------------------------------------ large delta
// local[j + P k (+ P^2 l)] = sum_i q h_j(x) h_k(y) (h_l(z)) with
// h_j(x) = H_j(x) e^{-x^2} / j! (g2dformlc_vec, g2drouts.f:621-681), one
// partial sum per CTA added into the global array.
// Dipoles (g2dformld_vec / g3dformld_vec, g2drouts.f:685-840,
// g3drouts.f:857-1040) add columns with the source derivative of one
// factor, dh_j = -(j+1) dsq h_(j+1): 2D (hx, q hy + v2 dhy), (v1 dhx, hy);
// 3D as dip3_coef with these h and dh.
template <int DIM>
__global__ void __launch_bounds__(256) k_ld_form(KP k, int ns, int p, const double3 c3,
                                                 double* __restrict__ local, double* __restrict__ partial) {
  const double cen[3] = {c3.x, c3.y, c3.z};
  const int Pn = p + 1;
  const int nent = DIM == 2 ? Pn * Pn : Pn * Pn * Pn;
  extern __shared__ double sm[];
  double* hx = sm;                    // [FORM_CH][Pn]
  double* hy = hx + FORM_CH * Pn;
  double* hz = hy + FORM_CH * Pn;
  const int ind = blockIdx.y;
  const int per = (ns + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per, i1 = min(ns, i0 + per);
  const int vc = k.ifdipole ? DIM : 1, chs = FORM_CH / vc;
  for (int e0 = 0; e0 < nent; e0 += 256 * 4) {
    double acc[4] = {0, 0, 0, 0};
    for (int c0 = i0; c0 < i1; c0 += chs) {
      const int m = vc * min(chs, i1 - c0);
      __syncthreads();
      if (threadIdx.x < m) {
        const int i = c0 + threadIdx.x / vc, col = threadIdx.x % vc;
        double v[3];
        for (int d = 0; d < DIM; d++) v[d] = (k.src[DIM * i + d] - cen[d]) * k.dsq;
        if (!k.ifdipole) {
          for (int d = 0; d < DIM; d++) {
            double* h = (d == 0 ? hx : d == 1 ? hy : hz) + threadIdx.x * Pn;
            const double f = exp(-v[d] * v[d]);
            h[0] = f;
            if (Pn > 1) h[1] = 2.0 * v[d] * f;
            for (int j = 1; j < Pn - 1; j++) h[j + 1] = 2.0 * (v[d] * h[j] - h[j - 1]) / (j + 1);
          }
          double* hl = (DIM == 2 ? hy : hz) + threadIdx.x * Pn;
          const double q = k.chg[(size_t)i * k.nd + ind];
          for (int j = 0; j < Pn; j++) hl[j] *= q;
        } else {
          double dv[3] = {0.0, 0.0, 0.0}, a, b;
          src_dipole<DIM>(k, i, ind, dv);
          const double q = src_charge(k, i, ind);
          for (int d = 0; d < DIM; d++) {
            if (DIM == 2) {  // columns (hx, q hy + v2 dhy) and (v1 dhx, hy)
              a = d == 0 ? (col ? 0.0 : 1.0) : (col ? 1.0 : q);
              b = d == 0 ? (col ? dv[0] : 0.0) : (col ? 0.0 : dv[1]);
            } else {
              dip3_coef(col, d, q, dv, a, b);
            }
            // h_0 .. h_Pn by the recurrence, row_j = a h_j - b (j+1) dsq h_(j+1)
            double* row = (d == 0 ? hx : d == 1 ? hy : hz) + threadIdx.x * Pn;
            const double f = exp(-v[d] * v[d]);
            double hm = f, hc = 2.0 * v[d] * f;  // h_j, h_(j+1)
            for (int j = 0; j < Pn; j++) {
              row[j] = fma(a, hm, -b * (j + 1.0) * k.dsq * hc);
              const double hn = 2.0 * (v[d] * hc - hm) / (j + 2);
              hm = hc;
              hc = hn;
            }
          }
        }
      }
      __syncthreads();
      for (int t = 0; t < m; t++) {
#pragma unroll
        for (int s = 0; s < 4; s++) {
          const int e = e0 + threadIdx.x + s * 256;
          if (e < nent) {
            const int a = e % Pn, b = (e / Pn) % Pn, c = e / (Pn * Pn);
            double v = hx[t * Pn + a] * hy[t * Pn + b];
            if (DIM == 3) v *= hz[t * Pn + c];
            acc[s] += v;
          }
        }
      }
    }
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const int e = e0 + threadIdx.x + s * 256;
      if (e >= nent) continue;
      if (partial) partial[((size_t)ind * gridDim.x + blockIdx.x) * nent + e] = acc[s];
      else atomicAdd(local + (size_t)ind * nent + e, acc[s]);
    }
  }
}
// local = sum of the per-CTA partial blocks, in CTA order (deterministic)
__global__ void k_ld_sum(int nent, int nparts, const double* __restrict__ partial, double* __restrict__ local) {
  const int ind = blockIdx.y;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nent; e += gridDim.x * blockDim.x) {
    double a = 0.0;
    for (int c = 0; c < nparts; c++) a += partial[((size_t)ind * nparts + c) * nent + e];
    local[(size_t)ind * nent + e] = a;
  }
}
// Taylor evaluation at every point (g2dlevalp/g/h_vec, g3dlevalp/g/h_vec);
// outputs in the caller's layout: pot(nd, n), grad(nd, dim, n), hess(nd, H, n).
template <int DIM, int PGH>
__global__ void k_ld_eval(KP k, int n, const double* __restrict__ pts, double* __restrict__ pot,
                          double* __restrict__ grad, double* __restrict__ hess, int p,
                          const double3 c3, const double* __restrict__ local) {
  const double cen[3] = {c3.x, c3.y, c3.z};
  constexpr int NC = ncomp<DIM, PGH>(), NH = nhess<DIM>();
  const int Pn = p + 1;
  const int nent = DIM == 2 ? Pn * Pn : Pn * Pn * Pn;
  const int ind = blockIdx.y, nd = k.nd;
  const double* lo = local + (size_t)ind * nent;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double x = (pts[DIM * i] - cen[0]) * k.dsq, y = (pts[DIM * i + 1] - cen[1]) * k.dsq;
    double v[NC];
    if (DIM == 2) horner2_rt<PGH>(lo, Pn, Pn, x, y, k.dsq, v);
    else horner3_rt<PGH>(lo, Pn, Pn, x, y, (pts[DIM * i + 2] - cen[DIM - 1]) * k.dsq, k.dsq, v);
    pot[(size_t)i * nd + ind] = v[0];
    if (PGH >= 2)
#pragma unroll
      for (int d = 0; d < DIM; d++) grad[((size_t)i * DIM + d) * nd + ind] = v[1 + d];
    if (PGH >= 3)
#pragma unroll
      for (int c = 0; c < NH; c++) hess[((size_t)i * NH + c) * nd + ind] = v[1 + DIM + c];
  }
}

// ------------------------------------------------------------ FP64 MMA throughput probe
// Eight independent m8n8k4 f64 accumulator chains per warp, `iters` steps:
// 8 * 256 * iters FMAs per warp.  Used to measure the FP64 tensor-core
// denominator of the 2D form/eval roofline on the running GPU.
__global__ void __launch_bounds__(128) k_probe_dmma(double* out, int iters) {
  double c[8][2];
  const double a = 1.0 + 1e-9 * threadIdx.x, b = 1.0 - 1e-9 * blockIdx.x;
#pragma unroll
  for (int i = 0; i < 8; i++) c[i][0] = c[i][1] = 0.0;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < 8; i++) dmma_884(c[i][0], c[i][1], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 8; i++) s += c[i][0] + c[i][1];
  if (s == 12345.678) out[0] = s;  // keeps the chains live
}

// ------------------------------------------------------------ host helpers
template <typename T, typename A>
cudaError_t put(char*& cur, T*& dst, const std::vector<T, A>& v, cudaStream_t s) {
  dst = reinterpret_cast<T*>(cur);
  size_t b = (v.size() * sizeof(T) + 255) & ~size_t(255);
  cur += b;
  if (v.empty()) return cudaSuccess;
  return cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}
template <typename T, typename A>
size_t bytes_of(const std::vector<T, A>& v) {
  return (v.size() * sizeof(T) + 255) & ~size_t(255);
}
size_t al(size_t b) { return (b + 255) & ~size_t(255); }

// Arrays placed one after another in the device arena (as put() does) and
// copied up together: the host data is gathered, by the host threads, into
// a pinned mirror of the arena range, which goes up in one asynchronous copy.
// The mirror belongs to the calling thread and is reused; the caller
// synchronises the stream before the thread stages again.
struct Staged {
  struct Item {
    size_t off, bytes;
    const void* src;
  };
  std::vector<Item> items;
  size_t span = 0;
  template <typename T, typename A>
  void add(char*& cur, T*& dst, const std::vector<T, A>& v) {
    dst = reinterpret_cast<T*>(cur);
    const size_t b = v.size() * sizeof(T);
    if (b) items.push_back({span, b, v.data()});
    span += (b + 255) & ~size_t(255);
    cur += (b + 255) & ~size_t(255);
  }
  cudaError_t upload(char* dev, cudaStream_t s) {
    if (span == 0) return cudaSuccess;
    // A mirror that grows keeps its old buffers until the thread exits:
    // cudaFreeHost waits for the whole device, which would stall this
    // request behind every other stream's work (the server's workers).
    struct Mirror {
      char* p = nullptr;
      size_t cap = 0;
      std::vector<char*> old;
      ~Mirror() {
        if (p) cudaFreeHost(p);
        for (char* q : old) cudaFreeHost(q);
      }
    };
    thread_local Mirror m;
    if (m.cap < span) {
      if (m.p) m.old.push_back(m.p);
      m.p = nullptr;
      const size_t want = std::max(std::max(span + span / 4, 2 * m.cap), (size_t)16 << 20);
      m.cap = 0;
      cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&m.p), want, cudaHostAllocPortable);
      if (e != cudaSuccess) {
        m.p = nullptr;
        (void)cudaGetLastError();
        // no pinned memory: the arrays go up one by one from where they are
        for (const Item& it : items) {
          e = cudaMemcpyAsync(dev + it.off, it.src, it.bytes, cudaMemcpyHostToDevice, s);
          if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
      }
      m.cap = want;
    }
    // copy in 1 MB pieces so that large arrays are split over the threads
    // (the mirror's address is taken here: m is the calling thread's own)
    char* const mirror = m.p;
    std::vector<std::pair<size_t, size_t>> pieces;  // (item, piece offset)
    for (size_t i = 0; i < items.size(); i++)
      for (size_t o = 0; o < items[i].bytes; o += (1 << 20)) pieces.push_back({i, o});
#pragma omp parallel for schedule(dynamic, 1) if (span > (4u << 20))
    for (long long q = 0; q < (long long)pieces.size(); q++) {
      const Item& it = items[pieces[q].first];
      const size_t o = pieces[q].second, n = std::min<size_t>(1 << 20, it.bytes - o);
      memcpy(mirror + it.off + o, static_cast<const char*>(it.src) + o, n);
    }
    return cudaMemcpyAsync(dev, mirror, span, cudaMemcpyHostToDevice, s);
  }
};


}  // namespace

#define CK(x)                               \
  do {                                      \
    cudaError_t e_ = (x);                   \
    if (e_ != cudaSuccess) return e_;       \
  } while (0)

// Shared memory of k_form3d_h2pw (the SIMT passes) at order Pn.
size_t form3_simt_smem(int Pn_, int npw) {
  const size_t Pn = Pn_, n2 = npw / 2, P3 = Pn * Pn * Pn;
  const size_t szA = std::max(P3, 2 * Pn * npw * n2);
  return (((szA + 1) & ~size_t(1)) + 2 * Pn * Pn * n2 + Pn * npw) * 8;
}
// Stable sort of tasks by (route, order): a counting sort (the keys are few
// small integers), linear in the number of tasks.
template <typename Task>
std::vector<Task> route_order_sort(const std::vector<Task>& in) {
  // the tasks come level by level, so runs of one key are long: count and
  // place whole runs (a per-task counter increment is a dependency chain
  // through one memory cell when most tasks share a key)
  auto key = [](const Task& t) { return 4096 * t.route + t.p; };
  std::vector<std::pair<size_t, size_t>> runs;  // [begin, end)
  int kmax = 0;
  for (size_t i = 0; i < in.size();) {
    size_t j = i + 1;
    const int k = key(in[i]);
    while (j < in.size() && key(in[j]) == k) j++;
    runs.push_back({i, j});
    kmax = std::max(kmax, k);
    i = j;
  }
  std::vector<size_t> cnt((size_t)kmax + 2, 0);
  for (const auto& r : runs) cnt[key(in[r.first]) + 1] += r.second - r.first;
  for (size_t i = 1; i < cnt.size(); i++) cnt[i] += cnt[i - 1];
  std::vector<Task> out(in.size());
  for (const auto& r : runs) {
    size_t& at = cnt[key(in[r.first])];
    std::copy(in.begin() + r.first, in.begin() + r.second, out.begin() + at);
    at += r.second - r.first;
  }
  return out;
}
// Whether the 3D Hermite form of order Pn runs on the shared-memory kernels:
// k_form3d_mma's staging ((8 ceil(P/8) + 2 P) power rows of 68 doubles) and
// one of the Hermite -> PW kernels (tensor-core or SIMT passes).
bool form3_fits(int Pn, int npw) {
  const size_t lim = 227 * 1024;
  const size_t shA = ((size_t)8 * ((Pn + 7) / 8) + 2 * Pn) * 68 * 8;
  if (Pn > 32 || shA > lim) return false;
  const H3Dims Z(Pn, npw / 2);
  const bool mma = (Pn + 7) / 8 <= 4 && (npw / 2 + 7) / 8 <= 4 && std::min(Z.total_pf, Z.total_ov) * 8 <= lim;
  return mma || form3_simt_smem(Pn, npw) <= lim;
}

cudaError_t device_pool_setup() {
  // keep freed stream-ordered allocations in the device's default pool
  // instead of returning them at every synchronisation (process-local
  // runtime state, once per device)
  static std::mutex mu;
  static bool done[64] = {false};
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev >= 0 && dev < 64 && !done[dev]) {
    cudaMemPool_t pool;
    CK(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t thr = UINT64_MAX;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    done[dev] = true;
  }
  return cudaSuccess;
}

cudaError_t device_plan_create(const HostPlan& H, DevicePlan& D, const int* d_isrc, const int* d_itarg,
                               cudaStream_t pst, size_t* size_only) {
  const auto tnow = [] {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  };
  const double tin = tnow();
  double tp[8];
  int np_ = 0;
  D = DevicePlan();
  D.P = H.P;
  const Params& P = H.P;
  D.nboxes = H.tree.nboxes;
  D.nch = 1 << P.dim;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&D.sm_count, cudaDevAttrMultiProcessorCount, dev));
  double tq[8];
  int nq = 0;
  tq[nq++] = tnow();
  // order form and eval tasks by route so each kernel gets a contiguous range
  // (then by order; stable)
  const std::vector<FormTask> form = route_order_sort(H.form);
  D.nform = (int)form.size();
  for (auto& f : form) {
    (f.route == ROUTE_PW ? D.form_pw_n : D.form_hermite_n)++;
    if (f.route == ROUTE_HERMITE) D.form_pmax = std::max(D.form_pmax, f.p);
  }
  const std::vector<EvalTask> ev = route_order_sort(H.eval);
  D.neval = (int)ev.size();
  for (auto& e : ev) {
    (e.route == ROUTE_PW ? D.eval_pw_n : D.eval_taylor_n)++;
    if (e.route == ROUTE_TAYLOR) D.eval_pmax = std::max(D.eval_pmax, e.p);
  }
  tq[nq++] = tnow();
  // launch groups of equal order among the Hermite form / Taylor eval tasks
  for (int t = 0; t < D.form_hermite_n;) {
    int u = t;
    while (u < D.form_hermite_n && form[u].p == form[t].p) u++;
    D.form_groups.push_back({form[t].p, t, u});
    t = u;
  }

  // dominant form group (most sources) for the per-kernel roofline of the bench
  if (P.dim == 2) {
    long long best = -1;
    for (size_t gi = 0; gi < D.form_groups.size(); gi++) {
      const OrderGroup& G = D.form_groups[gi];
      long long n = 0;
      for (int t = G.beg; t < G.end; t++) n += form[t].n;
      const double Pn = G.p + 1;
      D.group_flops.push_back(2.0 * (double)n * Pn * Pn * P.nd);
      D.group_alg_flops.push_back(4.0 * (double)n * P.npw * P.npw * P.nd);
      if (G.p + 1 <= 32 && n > best) { best = n; D.dom_form_group = (int)gi; }
    }
  }
  tp[np_++] = tnow();
  // 2D Taylor evaluation: one conversion per leaf slot, point chunks of <= 256
  std::vector<ConvTask> conv;
  std::vector<HornerTask> horner;
  size_t lo_doubles = 0;
  // 3D: the same two kernels for the Taylor tasks whose order's shared-memory
  // needs fit (k_eval3d_horner is instantiated for rows of up to 30
  // coefficients); the tasks are sorted by order, so these are a prefix and
  // the higher orders take the direct separable evaluation (k_eval3d_sep) or,
  // with derivatives, the fallback kernels
  if (P.dim == 3 && !P.all_direct) {
    int t = 0;
    while (t < D.eval_taylor_n && ev[t].p + 1 <= 30 && conv3_smem_bytes(ev[t].p + 1, P.npw, 4) <= 200 * 1024 &&
           (P.npw + 3) / 4 <= CONV_MAXKS)
      t++;
    D.eval3_nsplit = t;
  }
  D.eval3_split = D.eval3_nsplit > 0;
  const int split_pmax = D.eval3_split ? ev[D.eval3_nsplit - 1].p : -1;
  // The split is fused into the conversion kernels (2D: all; 3D: those that
  // stage the expansion in shared memory, orders <= 32): they read the
  // cut-level ancestor's local expansion and apply the leaf's phases
  // (ConvTask.sh)
  // 2D: every conversion (k_pw2taylor2d) applies the fused split itself
  auto conv_fusable = [&](int Pn) {
    if (P.dim == 2) return true;
    const int ksm = (P.npw / 2 + 3) / 4;
    if (ksm > 8) return false;
    if (Pn <= 16) return C3Dims(Pn, P.npw).total * 8 <= 227 * 1024;
    if (Pn > 32) return false;
    int gs2 = 4;
    while (gs2 > 1 && C3Dims2(Pn, P.npw, gs2).total * 8 > 227 * 1024) gs2 >>= 1;
    return C3Dims2(Pn, P.npw, gs2).total * 8 <= 227 * 1024;
  };
  const int lcut = std::max(P.npwlevel, 0);
  std::vector<uint8_t> fused_leaf(H.tree.nboxes, 0);
  tq[nq++] = tnow();
  if ((P.dim == 2 || D.eval3_split) && !P.all_direct) {
    const int ntay = P.dim == 2 ? D.eval_taylor_n : D.eval3_nsplit;
    // the conversion of leaf slot s, made by its first task: (ConvTask, the
    // fused split), the same for either way of filling below
    auto make_conv = [&](const EvalTask& e, long long off) {
      const long long Pn = e.p + 1;
      ConvTask ct{e.slot, e.p, off};
      if (conv_fusable((int)Pn) && H.tree.level[e.box] > lcut) {
        int a = e.box;
        while (H.tree.level[a] > lcut) a = H.tree.parent[a];
        if (a >= 0 && H.loc_slot[a] >= 0) {
          ct.slot = H.loc_slot[a];
          ct.fused = 1;
          for (int d = 0; d < P.dim; d++) ct.sh[d] = (H.tree.c(e.box, d) - H.tree.c(a, d)) * P.dsq;
          fused_leaf[e.box] = 1;
        }
      }
      return ct;
    };
    auto lo_size = [&](const EvalTask& e) {
      const long long Pn = e.p + 1, E = (Pn + 1) & ~1LL;
      return (size_t)(P.nd * Pn * E * (P.dim == 3 ? Pn : 1));
    };
    // The tasks of one leaf are consecutive (the builder emits them leaf by
    // leaf and the route sort is stable): then every slot's first task starts
    // a run, the conversions and chunk lists are laid out by prefix sums and
    // filled in parallel.  Otherwise the serial loop below does the same.
    std::vector<int> cidx(ntay + 1, 0);
    std::vector<long long> hidx(ntay + 1, 0);
    bool runs = true;
    {
      std::vector<uint8_t> seen(std::max(H.nloc, 1), 0);
      for (int t = 0; t < ntay; t++) {
        const bool first = t == 0 || ev[t].slot != ev[t - 1].slot;
        if (first) {
          if (seen[ev[t].slot]) runs = false;
          seen[ev[t].slot] = 1;
        }
        cidx[t + 1] = cidx[t] + first;
        hidx[t + 1] = hidx[t] + (ev[t].n + 255) / 256;
      }
    }
    if (runs) {
      const int ncv = cidx[ntay];
      std::vector<long long> coff(ncv + 1, 0);
      for (int t = 0; t < ntay; t++)
        if (cidx[t + 1] != cidx[t]) coff[cidx[t] + 1] = (long long)lo_size(ev[t]);
      for (int c = 0; c < ncv; c++) coff[c + 1] += coff[c];
      lo_doubles = (size_t)coff[ncv];
      conv.resize(ncv);
      horner.resize(hidx[ntay]);
#pragma omp parallel for schedule(static) if (ntay > 4096)
      for (int t = 0; t < ntay; t++) {
        const EvalTask& e = ev[t];
        const int c = cidx[t + 1] - 1;  // this task's slot's conversion
        if (cidx[t + 1] != cidx[t]) conv[c] = make_conv(e, coff[c]);
        long long h = hidx[t];
        for (int k = 0; k < e.n; k += 256) horner[h++] = {e.box, e.set, e.i0 + k, std::min(256, e.n - k), e.p, coff[c]};
      }
    }
    std::vector<long long> slot_off(runs ? 1 : std::max(H.nloc, 1), -1);
    if (!runs) {
      conv.reserve(ntay);
      horner.reserve(hidx[ntay]);
    }
    for (int t = 0; t < ntay && !runs; t++) {
      const EvalTask& e = ev[t];
      if (slot_off[e.slot] < 0) {
        slot_off[e.slot] = (long long)lo_doubles;
        conv.push_back(make_conv(e, (long long)lo_doubles));
        lo_doubles += lo_size(e);
      }
      for (int c = 0; c < e.n; c += 256)
        horner.push_back({e.box, e.set, e.i0 + c, std::min(256, e.n - c), e.p, slot_off[e.slot]});
    }
    tq[nq++] = tnow();
    // conv and horner are in order of p (the Taylor tasks are sorted by p)
    for (size_t t = 0; t < conv.size();) {
      size_t u = t;
      while (u < conv.size() && conv[u].p == conv[t].p) u++;
      D.conv_groups.push_back({conv[t].p, (int)t, (int)u});
      t = u;
    }
    for (size_t t = 0; t < horner.size();) {
      size_t u = t;
      while (u < horner.size() && horner[u].p == horner[t].p) u++;
      D.horner_groups.push_back({horner[t].p, (int)t, (int)u});
      t = u;
    }
  }
  tp[np_++] = tnow();
  // padded operand tables of the 2D MMA transforms, one per order group
  std::vector<double> tables;
  if (P.dim == 2 && !P.all_direct) {
    for (OrderGroup& G : D.form_groups)
      if (G.p + 1 <= 32) {
        G.tab = (long long)tables.size();
        build_h2pw_table(H, G.p + 1, tables);
      }
    for (OrderGroup& G : D.conv_groups) {
      G.tab = (long long)tables.size();
      build_conv_table(H, G.p + 1, tables);
    }
  }
  if (D.eval3_split)
    for (OrderGroup& G : D.conv_groups) {
      G.tab = (long long)tables.size();
      build_conv3_table(H, G.p + 1, tables);
    }
  tp[np_++] = tnow();
  // merge groups: consecutive tasks with the same destination
  std::vector<MergeGroup> groups;
  D.merge_beg.assign(P.nlevels + 1, 0);
  D.merge_end.assign(P.nlevels + 1, 0);
  for (int l = 0; l <= P.nlevels && !H.merge_beg.empty(); l++) {
    D.merge_beg[l] = (int)groups.size();
    for (int t = H.merge_beg[l]; t < H.merge_end[l];) {
      int u = t;
      while (u < H.merge_end[l] && H.merge[u].dst == H.merge[t].dst) u++;
      groups.push_back({H.merge[t].dst, t, u - t});
      t = u;
    }
    D.merge_end[l] = (int)groups.size();
  }
  tp[np_++] = tnow();
  // the split tasks still needed: the boxes on the path from the cut level
  // to every evaluation leaf whose conversion does not fuse the split
  std::vector<ShiftTask> split_kept;
  {
    const Tree& tr = H.tree;
    std::vector<uint8_t> need(tr.nboxes, 0);
    for (int t = 0; t < (int)H.eval.size(); t++) {
      int b = H.eval[t].box;
      if (fused_leaf[b]) continue;
      while (b >= 0 && tr.level[b] > lcut && !need[b]) {
        need[b] = 1;
        b = tr.parent[b];
      }
    }
    std::vector<int> loc_box(std::max(H.nloc, 1), -1);
    for (int b = 0; b < tr.nboxes; b++)
      if (H.loc_slot[b] >= 0) loc_box[H.loc_slot[b]] = b;
    D.split_beg.assign(H.split_beg.size(), 0);
    D.split_end.assign(H.split_end.size(), 0);
    for (size_t l = 0; l < H.split_beg.size(); l++) {
      D.split_beg[l] = (int)split_kept.size();
      for (int i = H.split_beg[l]; i < H.split_end[l]; i++)
        if (need[loc_box[H.split[i].dst]]) split_kept.push_back(H.split[i]);
      D.split_end[l] = (int)split_kept.size();
    }
    std::vector<uint8_t> rd(std::max(H.nloc, 1), 0), wr(std::max(H.nloc, 1), 0);
    long long nrw = 0;
    for (const ShiftTask& x : split_kept) {
      nrw += !rd[x.src] + !wr[x.dst];
      rd[x.src] = wr[x.dst] = 1;
    }
    D.split_bytes = 16LL * P.nexp * P.nd * nrw;
  }
  D.nm2l = (int)H.m2l.size();
  D.ndir = (int)(H.dnear.mem ? H.dnear.ndir : (long long)H.dir.size());
  D.nmp = H.nmp;
  D.nloc = H.nloc;
  D.direct_pairs = H.direct_pairs;
  D.form_sources = H.form_sources;
  D.eval_points = H.eval_points;
  tp[np_++] = tnow();
  // 3D: shared-memory paths when the largest order fits, else the scratch path
  std::vector<FormChunk> fchunks;
  std::vector<int> fcbeg;
  size_t hbuf_doubles = 0;
  // 2D: Hermite blocks of the MMA form (orders <= 31), nd P^2 doubles per leaf
  std::vector<long long> form_hoff;
  if (P.dim == 2 && !P.all_direct) {
    form_hoff.assign(form.size(), 0);
    for (int t = 0; t < D.form_hermite_n; t++) {
      const long long Pn = form[t].p + 1;
      if (Pn > 32) continue;
      form_hoff[t] = (long long)hbuf_doubles;
      hbuf_doubles += (size_t)(P.nd * Pn * Pn);
    }
  }
  if (P.dim == 3 && !P.all_direct) {
    const size_t lim = 227 * 1024;
    const int n2 = P.npw / 2;
    if (D.form_hermite_n > 0) {
      // the Hermite block kernel and one of the two Hermite -> PW kernels
      // take the tasks whose order fits their shared memory (a prefix: the
      // tasks are sorted by order); the rest take the scratch fallback
      int t = 0;
      while (t < D.form_hermite_n && form3_fits(form[t].p + 1, P.npw)) t++;
      D.form3_nsplit = t;
      D.form3_smem = t > 0;
      if (D.form3_smem) {
        long long hoff = 0;
        for (int t = 0; t < D.form3_nsplit; t++) {
          fcbeg.push_back((int)fchunks.size());
          const FormTask& f = form[t];
          long long p3 = (long long)(f.p + 1) * (f.p + 1) * (f.p + 1);
          for (int c = 0; c < f.n; c += 4096) {
            fchunks.push_back({t, f.s0 + c, std::min(4096, f.n - c), hoff});
            hoff += p3;
          }
        }
        fcbeg.push_back((int)fchunks.size());
        hbuf_doubles = (size_t)hoff * P.nd;
        D.nfchunks = (int)fchunks.size();
        // chunk ranges of equal order (the tasks are sorted by order)
        long long best = -1;
        for (size_t t = 0; t < fchunks.size();) {
          size_t u = t;
          const int pt = form[fchunks[t].task].p;
          long long n = 0;
          while (u < fchunks.size() && form[fchunks[u].task].p == pt) n += fchunks[u++].n;
          const double Pn = pt + 1;
          D.group_flops.push_back(2.0 * (double)n * Pn * Pn * Pn * P.nd);
          D.group_alg_flops.push_back(4.0 * (double)n * P.npw * P.npw * P.npw * P.nd);
          if (n > best) { best = n; D.dom_fchunk_group = (int)D.fchunk_groups.size(); }
          D.fchunk_groups.push_back({pt, (int)t, (int)u});
          t = u;
        }
      }
    }
    if (D.eval_taylor_n > 0) {
      const size_t Pn = D.eval_pmax + 1;
      size_t szA = std::max(2 * Pn * P.npw * n2, Pn * Pn * Pn);
      D.eval3_sh = (((szA + 1) & ~size_t(1)) + 2 * Pn * Pn * n2) * 8;
      // the fallback kernels run only on the Taylor tasks beyond the split
      // kernels' orders, and only with derivatives
      const bool fallback = D.eval3_nsplit < D.eval_taylor_n && std::max(P.ifpgh, P.ifpghtarg) >= 2;
      D.eval3_smem = D.eval3_sh <= lim || !fallback;
    }
  }
  // scratch for the 3D separable transforms (fallback path)
  const bool form3_fallback = P.dim == 3 && D.form3_nsplit < D.form_hermite_n;
  if (P.dim == 3 && !P.all_direct && (form3_fallback || !D.eval3_smem)) {
    size_t slab = 0;
    int n2 = P.npw / 2;
    if (form3_fallback)
      for (auto& f : form)
        if (f.route == ROUTE_HERMITE) slab = std::max(slab, (size_t)(f.p + 1) * (f.p + 1) * n2 + (size_t)(f.p + 1) * P.npw * n2);
    if (!D.eval3_smem)
      for (auto& e : ev)
        if (e.route == ROUTE_TAYLOR) {
        size_t Pn = e.p + 1;
        slab = std::max(slab, Pn * P.npw * n2 + Pn * Pn * n2 + (Pn * Pn * Pn + 1) / 2);
      }
    D.scratch_per_cta = (slab + 15) & ~size_t(15);
    D.scratch_ctas = D.scratch_per_cta ? D.sm_count * 2 : 0;
  }
  if (D.eval3_split) {
    D.uscr_per_cta = (conv3_scratch(split_pmax + 1, P.npw) + 31) & ~size_t(31);
    D.conv3_ctas = D.sm_count * 4;
  }
  size_t ns = P.ns, nt = P.nt, nd = P.nd, dim = P.dim;
  // FP32 coordinates of the mixed near field (charges only)
  const bool fmix = D.ndir > 0 && !P.ifdipole;
  // diagonal translation tables (formed on the device)
  const size_t n_wms = P.all_direct ? 0 : (size_t)(P.nlevels + 1) * D.nch * P.nexp;
  const size_t n_wsh = P.all_direct ? 0 : (size_t)(P.dim == 2 ? 9 : 27) * P.nexp;
  size_t total = bytes_of(H.box_centers) + bytes_of(H.h2x) + bytes_of(H.x2l) + al(n_wms * 16) + al(n_wsh * 16) + al(H.ww.size() * 8) + al(H.w1.size() * 8) + 2 * al((size_t)P.ns * 4) + 2 * al((size_t)P.nt * 4) +
                 al((size_t)(std::max(P.ntermmax, 1) + 2) * 8) + al(32 * 8) +
                 bytes_of(form) + bytes_of(groups) + bytes_of(H.merge) + bytes_of(split_kept) +
                 bytes_of(H.m2l) + bytes_of(H.m2l_nbr) + bytes_of(ev) + bytes_of(H.dir) +
                 al((size_t)H.dnear.ndir * sizeof(DirTask)) + al((size_t)H.dnear.nsrc * sizeof(SrcRange)) +
                 bytes_of(H.dir_src) + al((size_t)H.nmp * nd * P.nexp * 16) +
                 al((size_t)H.nloc * nd * P.nexp * 16) + al(ns * dim * 8) + al(ns * nd * 8) +
                 al(nt * dim * 8) + al(ns * nd * out_comps(dim, P.ifpgh) * 8) +
                 (fmix ? al(ns * dim * 8) + al((P.ifpghtarg > 0 ? nt : 0) * dim * 8) : 0) +
                 al(P.ifdipole ? ns * dim * 8 : 0) + al(P.ifdipole ? ns * nd * 8 : 0) +
                 al(nt * nd * out_comps(dim, P.ifpghtarg) * 8) +
                 al((size_t)D.scratch_ctas * D.scratch_per_cta * 16) + bytes_of(fchunks) +
                 al((size_t)D.conv3_ctas * nd * D.uscr_per_cta * 8) +
                 bytes_of(fcbeg) + al(hbuf_doubles * 8) + bytes_of(form_hoff) + bytes_of(tables) + bytes_of(conv) + bytes_of(horner) +
                 al(lo_doubles * 8) + 4096;
  D.bytes = total;
  if (size_only) {
    *size_only = total;
    return cudaSuccess;
  }
  const double tm0 = tnow();
  D.stream = pst;
  CK(device_pool_setup());
  CK(cudaMallocAsync(reinterpret_cast<void**>(&D.base), total, pst));
  const double tm1 = tnow();
  char* cur = D.base;
  cudaStream_t s = pst;
  // Everything that goes up from the host, laid out in the arena as it
  // comes, goes in one copy from a pinned mirror of that range (filled by the
  // host threads); no pageable copy (each would wait for the stream) and no
  // synchronisation here: the kernels below follow the copy on the stream.
  std::vector<double2> ww(H.ww.size() / 2), w1(H.w1.size() / 2);
  memcpy(ww.data(), H.ww.data(), H.ww.size() * 8);
  memcpy(w1.data(), H.w1.data(), H.w1.size() * 8);
  std::vector<double> isq(std::max(P.ntermmax, 1) + 2, 0.0);
  for (size_t j = 1; j < isq.size(); j++) isq[j] = 1.0 / std::sqrt((double)j);
  std::vector<double> cfac(32);
  cfac[0] = 1.0;
  for (int j = 1; j < 32; j++) cfac[j] = cfac[j - 1] / std::sqrt((double)j);
  double2 *d_ww = nullptr, *d_w1 = nullptr;
  {
    char* const b0 = cur;
    Staged st;
    st.add(cur, D.centers, H.box_centers);
    st.add(cur, D.h2x, H.h2x);
    st.add(cur, D.x2l, H.x2l);
    st.add(cur, d_ww, ww);
    st.add(cur, d_w1, w1);
    st.add(cur, D.isq, isq);
    st.add(cur, D.cfac, cfac);
    st.add(cur, D.form, form);
    st.add(cur, D.mgroups, groups);
    st.add(cur, D.merge, H.merge);
    st.add(cur, D.split, split_kept);
    st.add(cur, D.m2l, H.m2l);
    st.add(cur, D.m2l_nbr, H.m2l_nbr);
    st.add(cur, D.eval, ev);
    if (!H.dnear.mem) {  // else built on the device: copied after this block
      st.add(cur, D.dir, H.dir);
      st.add(cur, D.dir_src, H.dir_src);
    }
    st.add(cur, D.fchunks, fchunks);
    st.add(cur, D.fcbeg, fcbeg);
    st.add(cur, D.form_hoff, form_hoff);
    st.add(cur, D.tables, tables);
    st.add(cur, D.conv, conv);
    st.add(cur, D.horner, horner);
    CK(st.upload(b0, s));
  }
  // translation tables formed on the device from their 1D factors
  D.wms = reinterpret_cast<double2*>(cur); cur += al(n_wms * 16);
  D.wsh = reinterpret_cast<double2*>(cur); cur += al(n_wsh * 16);
  if (n_wms > 0) {
    const long long tot = (long long)(n_wms + n_wsh);
    const int blocks = (int)std::min<long long>((tot + 255) / 256, (long long)D.sm_count * 16);
    k_shift_tables<<<blocks, 256, 0, s>>>(P.dim, P.npw, P.nexp, P.nlevels, std::max(P.nlevstart, 0), H.nms,
                                          d_ww, d_w1, D.wms, D.wsh);
    CK(cudaGetLastError());
  }
  if (d_isrc) {
    // permutations built on the device (fgt_devtree.cu): copy, invert there;
    // targets that are the sources share the sources' arrays
    auto carve = [&](int*& dst, size_t n) {
      dst = reinterpret_cast<int*>(cur);
      cur += al(n * 4);
    };
    const bool same = H.same_points && P.nt == P.ns;
    carve(D.isrc, P.ns);
    carve(D.isrc_inv, P.ns);
    if (same) {
      D.itarg = D.isrc;
      D.itarg_inv = D.isrc_inv;
    } else {
      carve(D.itarg, P.nt);
      carve(D.itarg_inv, P.nt);
    }
    if (P.ns > 0) {
      CK(cudaMemcpyAsync(D.isrc, d_isrc, (size_t)P.ns * 4, cudaMemcpyDeviceToDevice, pst));
      k_invperm<<<(P.ns + 255) / 256, 256, 0, pst>>>(D.isrc, P.ns, D.isrc_inv);
    }
    if (P.nt > 0 && !same) {
      CK(cudaMemcpyAsync(D.itarg, d_itarg, (size_t)P.nt * 4, cudaMemcpyDeviceToDevice, pst));
      k_invperm<<<(P.nt + 255) / 256, 256, 0, pst>>>(D.itarg, P.nt, D.itarg_inv);
    }
  } else {
    CK(put(cur, D.isrc, H.tree.isrc, s));
    CK(put(cur, D.itarg, H.tree.itarg, s));
    std::vector<int> inv(H.tree.isrc.size());
    for (size_t i = 0; i < inv.size(); i++) inv[H.tree.isrc[i]] = (int)i;
    CK(put(cur, D.isrc_inv, inv, s));
    CK(cudaStreamSynchronize(s));
    inv.assign(H.tree.itarg.size(), 0);
    for (size_t i = 0; i < inv.size(); i++) inv[H.tree.itarg[i]] = (int)i;
    CK(put(cur, D.itarg_inv, inv, s));
  }
  if (H.dnear.mem) {
    D.dir = reinterpret_cast<DirTask*>(cur);
    cur += al((size_t)H.dnear.ndir * sizeof(DirTask));
    D.dir_src = reinterpret_cast<SrcRange*>(cur);
    cur += al((size_t)H.dnear.nsrc * sizeof(SrcRange));
    if (H.dnear.ndir)
      CK(cudaMemcpyAsync(D.dir, H.dnear.dir, (size_t)H.dnear.ndir * sizeof(DirTask), cudaMemcpyDeviceToDevice, s));
    if (H.dnear.nsrc)
      CK(cudaMemcpyAsync(D.dir_src, H.dnear.src, (size_t)H.dnear.nsrc * sizeof(SrcRange), cudaMemcpyDeviceToDevice,
                         s));
  }
  D.lo = reinterpret_cast<double*>(cur); cur += al(lo_doubles * 8);
  D.hbuf = reinterpret_cast<double*>(cur); cur += al(hbuf_doubles * 8);
  D.mp = reinterpret_cast<double2*>(cur); cur += al((size_t)H.nmp * nd * P.nexp * 16);
  D.loc = reinterpret_cast<double2*>(cur); cur += al((size_t)H.nloc * nd * P.nexp * 16);
  D.ssort = reinterpret_cast<double*>(cur); cur += al(ns * dim * 8);
  D.csort = reinterpret_cast<double*>(cur); cur += al(ns * nd * 8);
  D.nsort = reinterpret_cast<double*>(cur); cur += al(P.ifdipole ? ns * dim * 8 : 0);
  D.dsort = reinterpret_cast<double*>(cur); cur += al(P.ifdipole ? ns * nd * 8 : 0);
  D.tsort = reinterpret_cast<double*>(cur); cur += al(nt * dim * 8);
  if (fmix) {
    D.fsrc = reinterpret_cast<float*>(cur); cur += al(ns * dim * 8);
    D.ftrg = reinterpret_cast<float*>(cur); cur += al((P.ifpghtarg > 0 ? nt : 0) * dim * 8);
  }
  D.psort = reinterpret_cast<double*>(cur); cur += al(ns * nd * out_comps(dim, P.ifpgh) * 8);
  D.ptsort = reinterpret_cast<double*>(cur); cur += al(nt * nd * out_comps(dim, P.ifpghtarg) * 8);
  D.scratch = reinterpret_cast<double2*>(cur); cur += al((size_t)D.scratch_ctas * D.scratch_per_cta * 16);
  D.uscr = reinterpret_cast<double*>(cur); cur += al((size_t)D.conv3_ctas * nd * D.uscr_per_cta * 8);
  CK(cudaStreamSynchronize(s));
  if (getenv("FGT_TREE_TIMING"))
    fprintf(stderr, "device plan prep parts: sort %.4f conv %.4f tables %.4f merge %.4f split %.4f rest %.4f"
            " (device %.4f route sorts %.4f groups %.4f conv loop %.4f)\n",
            tp[0] - tin, tp[1] - tp[0], tp[2] - tp[1], tp[3] - tp[2], tp[4] - tp[3], tm0 - tp[4], tq[0] - tin,
            tq[1] - tq[0], tq[2] - tq[1], nq > 3 ? tq[3] - tq[2] : 0.0);
  if (getenv("FGT_TREE_TIMING"))
    fprintf(stderr, "device plan: prep %.4f malloc %.4f upload %.4f (%zu bytes); eval tasks: taylor %d "
            "(conversion %d, max order %d) pw %d; form tasks: hermite %d (shared memory %d, max order %d) pw %d\n",
            tm0 - tin, tm1 - tm0, tnow() - tm1, total, D.eval_taylor_n,
            P.dim == 3 ? D.eval3_nsplit : D.eval_taylor_n, D.eval_pmax + 1, D.eval_pw_n, D.form_hermite_n,
            P.dim == 3 ? D.form3_nsplit : D.form_hermite_n, D.form_pmax + 1, D.form_pw_n);
  return cudaSuccess;
}

void device_plan_destroy(DevicePlan& D) {
  if (D.base) cudaFreeAsync(D.base, D.stream);
  D.base = nullptr;
}

static KP make_kp(const DevicePlan& D) {
  KP k;
  const Params& P = D.P;
  k.dim = P.dim; k.nd = P.nd; k.npw = P.npw; k.n2 = P.npw / 2; k.nexp = P.nexp;
  k.dsq = P.dsq; k.delta = P.delta; k.dmax = P.dmax;
  k.t1 = P.npw > 0 ? 0.5 * P.pmax / (P.npw / 2) : 0.0;
  k.centers = D.centers; k.h2x = D.h2x; k.x2l = D.x2l; k.ws = nullptr;
  k.wms = D.wms; k.wsh = D.wsh; k.mp = D.mp; k.loc = D.loc;
  k.src = D.ssort; k.chg = D.csort; k.trg = D.tsort; k.pot = D.psort; k.pottarg = D.ptsort;
  k.nc_s = out_comps(P.dim, P.ifpgh);
  k.nc_t = out_comps(P.dim, P.ifpghtarg);
  k.ifcharge = P.ifcharge;
  k.ifdipole = P.ifdipole;
  k.dnrm = D.nsort;
  k.dstr = D.dsort;
  k.fsrc = D.fsrc;
  k.ftrg = D.ftrg;
  return k;
}

// node weights for the direct 3D form kernel live in the x2l/h2x neighbourhood:
// ws(k) = h2x[0 * npw + k] (j = 0 row of h2x is ws_k).
cudaError_t device_check_finite(const double* x, size_t n, int* d_flag, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  int dev = 0, sms = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const size_t blocks = std::min<size_t>((n + 255) / 256, (size_t)sms * 8);
  k_all_finite<<<(unsigned)blocks, 256, 0, st>>>(x, n, d_flag);
  return cudaGetLastError();
}

cudaError_t device_plan_set_points(DevicePlan& D, const double* src, const double* trg,
                                   cudaStream_t st) {
  const Params& P = D.P;
  const int gb = std::max(1, std::min(8 * D.sm_count, (std::max(P.ns, P.nt) + 255) / 256));
  if (P.ns > 0) {
    const int vec = (reinterpret_cast<uintptr_t>(src) & 15) == 0;
    k_gather_pts<<<gb, 256, 0, st>>>(src, nullptr, D.ssort, nullptr, D.isrc, P.ns, P.dim, P.nd, vec);
  }
  if (P.nt > 0 && P.ifpghtarg > 0) {
    const int vec = (reinterpret_cast<uintptr_t>(trg) & 15) == 0;
    k_gather_pts<<<gb, 256, 0, st>>>(trg, nullptr, D.tsort, nullptr, D.itarg, P.nt, P.dim, P.nd, vec);
  }
  if (D.fsrc) {
    const double cs = std::sqrt(1.4426950408889634 / P.delta);
    if (P.ns > 0)
      k_mixed_coords<<<gb, 256, 0, st>>>(D.ssort, P.ns, P.dim, P.cen0[0], P.cen0[1], P.cen0[2], cs, D.fsrc);
    if (P.nt > 0 && P.ifpghtarg > 0)
      k_mixed_coords<<<gb, 256, 0, st>>>(D.tsort, P.nt, P.dim, P.cen0[0], P.cen0[1], P.cen0[2], cs, D.ftrg);
  }
  return cudaGetLastError();
}

// Runs launch(std::integral_constant<int, G>) with G = pgh in {1, 2, 3}.
template <class F>
cudaError_t with_pgh(int pgh, F&& launch) {
  switch (pgh) {
    case 1: return launch(std::integral_constant<int, 1>());
    case 2: return launch(std::integral_constant<int, 2>());
    case 3: return launch(std::integral_constant<int, 3>());
    default: return cudaErrorNotSupported;
  }
}

cudaError_t device_plan_execute(DevicePlan& D, const Inputs& in, const Outputs& outs,
                                int precision, cudaStream_t st, StageTimes* times, int phase) {
  const Params& P = D.P;
  // phase 1: gather, form, merge (every mp expansion up to the cut level);
  // phase 2: mp -> loc, split, eval, near field, scatter; 0: both
  const bool ph1 = phase != 2, ph2 = phase != 1;
  KP k = make_kp(D);
  // the derivative order the kernels compute: the larger of the two sets'
  const int pgh = std::max(1, std::max(P.ifpgh, P.ifpghtarg));
  // mixed form of stages (a) and (c): FP32 arithmetic with FP64 accumulation
  // in the 2D Hermite block and Taylor evaluation (charges, potentials)
  const bool mixed_ac = precision == PREC_MIXED && !P.ifdipole;
  k.ws = D.h2x;  // row j = 0 of h2x holds the weights
  const int nd = P.nd;
  cudaEvent_t ev[9], dev0 = nullptr, dev1 = nullptr;
  if (times) {
    for (int i = 0; i < 9; i++) CK(cudaEventCreate(&ev[i]));
    CK(cudaEventCreate(&dev0));
    CK(cudaEventCreate(&dev1));
    times->dom_ms = 0;
    times->dom_flops = 0;
    times->dom_alg_flops = 0;
    times->dom_name[0] = 0;
  }
  auto mark = [&](int i) { if (times) cudaEventRecord(ev[i], st); };
  long long launches = 0;
  mark(0);
  // charges into tree order (coordinates were sorted once, at plan set-up)
  const int gb = std::max(1, std::min(8 * D.sm_count, (std::max(P.ns, P.nt) + 255) / 256));
  if (ph1 && P.ns > 0 && P.ifcharge) {
    if (nd == 1) k_gather1<<<gb, 256, 0, st>>>(in.charge, D.isrc, P.ns, D.csort);
    else k_gather_pts<<<gb, 256, 0, st>>>(nullptr, in.charge, nullptr, D.csort, D.isrc, P.ns, P.dim, nd, 0);
    launches++;
  }
  if (ph1 && P.ns > 0 && P.ifdipole) {  // directions and strengths of the dipoles
    k_gather_pts<<<gb, 256, 0, st>>>(in.rnormal, in.dipstr, D.nsort, D.dsort, D.isrc, P.ns, P.dim, nd, 0);
    launches++;
  }
  if (ph1 && P.ifpgh > 0 && P.ns > 0) CK(cudaMemsetAsync(D.psort, 0, (size_t)P.ns * nd * k.nc_s * 8, st));
  if (ph1 && P.ifpghtarg > 0 && P.nt > 0) CK(cudaMemsetAsync(D.ptsort, 0, (size_t)P.nt * nd * k.nc_t * 8, st));
  mark(1);
  const int n2 = P.npw / 2;
  const int echunks = (int)std::min<long long>(65535, ((long long)nd * P.nexp + 255) / 256);
  const int schunks = (P.nexp + 256 * SHU - 1) / (256 * SHU);  // k_split: every density per block
  if (!P.all_direct) {
   if (ph1) {
    // (a) form
    if (P.dim == 2 && D.form_hermite_n > 0) {
      for (size_t gi = 0; gi < D.form_groups.size(); gi++) {
        const OrderGroup& G = D.form_groups[gi];
        const int Pn = G.p + 1;
        dim3 g(G.end - G.beg, nd);
        const FormTask* tk = D.form + G.beg;
        const bool dom = times && (int)gi == D.dom_form_group;
        if (dom) cudaEventRecord(dev0, st);
        if (Pn <= 32) {
#define FORM_MMA(NT)                                                                              \
  do {                                                                                            \
    const size_t sh = (size_t)4 * 2 * (8 * NT) * 36 * 8;                                          \
    if (P.ifdipole) {                                                                             \
      CK(smem_limit(k_form2d_mma<NT, true>)); \
      k_form2d_mma<NT, true><<<g, 128, sh, st>>>(k, tk, D.form_hoff + G.beg, D.hbuf);             \
    } else {                                                                                      \
      CK(smem_limit(k_form2d_mma<NT, false>)); \
      k_form2d_mma<NT, false><<<g, 128, sh, st>>>(k, tk, D.form_hoff + G.beg, D.hbuf);            \
    }                                                                                             \
  } while (0)
          if (mixed_ac && Pn <= 16) CK(launch_form2d_f32(k, tk, G.end - G.beg, nd, D.form_hoff + G.beg, D.hbuf, Pn, st));
          else if (Pn <= 8) FORM_MMA(1);
          else if (Pn <= 16) FORM_MMA(2);
          else if (Pn <= 24) FORM_MMA(3);
          else FORM_MMA(4);
#undef FORM_MMA
          if (dom) {
            cudaEventRecord(dev1, st);
            if (mixed_ac && Pn <= 16) snprintf(times->dom_name, sizeof(times->dom_name), "k_form2d_f32");
            else snprintf(times->dom_name, sizeof(times->dom_name), "k_form2d_mma<%d>", (Pn + 7) / 8);
            times->dom_flops = D.group_flops[gi];
            times->dom_alg_flops = D.group_alg_flops[gi];
          }
          const int nt = G.end - G.beg;
          const H2pwDims Z(Pn, P.npw);
          const size_t sh2 = 4 * (size_t)Z.warp * 8;
          if (sh2 > 227 * 1024) return cudaErrorNotSupported;
          const dim3 hg((nt + 3) / 4, nd);
          switch (Z.Kq / 4) {
#define H2PW_CASE(N)                                                                              \
  case N:                                                                                         \
    CK(smem_limit(k_h2pw2d<N>)); \
    k_h2pw2d<N><<<hg, 128, sh2, st>>>(k, tk, nt, D.form_hoff + G.beg, D.hbuf, D.tables + G.tab);  \
    break;
            H2PW_CASE(1) H2PW_CASE(2) H2PW_CASE(3) H2PW_CASE(4) H2PW_CASE(5) H2PW_CASE(6)
            H2PW_CASE(7) H2PW_CASE(8)
#undef H2PW_CASE
            default: return cudaErrorNotSupported;
          }
          launches++;
        } else {
          const int tpd = (Pn + 3) / 4, Pp = 4 * tpd;
          if (tpd * tpd > 256) return cudaErrorNotSupported;
          const int ch = Pp <= 32 ? 128 : 64;
          size_t sh = ((size_t)2 * ch * Pp + 4096 + 2 * (size_t)Pn * n2) * 8;
          CK(smem_limit(k_form2d));
          k_form2d<<<g, 256, sh, st>>>(k, tk, D.isq, ch);
        }
        launches++;
      }
    }
    if (P.dim == 3 && D.form_hermite_n > 0 && D.form3_smem) {
      for (size_t gi = 0; gi < D.fchunk_groups.size(); gi++) {
        const OrderGroup& G = D.fchunk_groups[gi];
        const int Pn = G.p + 1, mt = (Pn + 7) / 8;
        const bool dom = times && (int)gi == D.dom_fchunk_group;
        if (dom) cudaEventRecord(dev0, st);
        const size_t sh = ((size_t)8 * mt + 2 * Pn) * 68 * 8;
        const dim3 fg(G.end - G.beg, nd);
        const FormChunk* ch = D.fchunks + G.beg;
        // The tcgen05 Hermite blocks (BF16 x 3) only on request: building
        // their Pn^2 split operand rows per source costs more than the FP64
        // DMMA kernel's whole block (3D blobs, Pn = 14: form 4.2 vs 3.45 ms),
        // so the mixed form keeps the FP64 blocks by default.
        const bool tc_form = getenv("FGT_FORM3D_TC") != nullptr;
        if (mixed_ac && tc_form && form3d_tc_supported(Pn)) {
          // mixed form: the Hermite blocks as BF16 x 3 tensor-core products
          CK(launch_form3d_tc(k, D.form, ch, G.end - G.beg, nd, Pn, D.hbuf, D.isq, st));
          if (dom) {
            cudaEventRecord(dev1, st);
            snprintf(times->dom_name, sizeof(times->dom_name), "k_form3d_tc<%d>", Pn);
            times->dom_flops = D.group_flops[gi];
            times->dom_alg_flops = D.group_alg_flops[gi];
          }
          launches++;
          continue;
        }
        switch (mt) {
#define FORM3_CASE(N)                                                                             \
  case N:                                                                                         \
    if (P.ifdipole) {                                                                             \
      CK(smem_limit(k_form3d_mma<N, true>)); \
      k_form3d_mma<N, true><<<fg, 256, sh, st>>>(k, D.form, ch, D.hbuf, D.isq);                   \
    } else {                                                                                      \
      CK(smem_limit(k_form3d_mma<N, false>)); \
      k_form3d_mma<N, false><<<fg, 256, sh, st>>>(k, D.form, ch, D.hbuf, D.isq);                  \
    }                                                                                             \
    break;
          FORM3_CASE(1) FORM3_CASE(2) FORM3_CASE(3) FORM3_CASE(4)
#undef FORM3_CASE
          default: return cudaErrorNotSupported;
        }
        if (dom) {
          cudaEventRecord(dev1, st);
          snprintf(times->dom_name, sizeof(times->dom_name), "k_form3d_mma<%d>", mt);
          times->dom_flops = D.group_flops[gi];
          times->dom_alg_flops = D.group_alg_flops[gi];
        }
        launches++;
      }
      // Hermite -> plane wave per order group: tensor-core passes where the
      // order and node count fit their fragments and shared memory
      for (const OrderGroup& G : D.form_groups) {
        if (G.beg >= D.form3_nsplit) break;  // the scratch fallback's orders
        const int Pn = G.p + 1, ks = (Pn + 7) / 8, mt = (P.npw / 2 + 7) / 8;
        const H3Dims Z3(Pn, P.npw / 2);
        const bool pf = Z3.total_pf * 8 <= 227 * 1024;
        const size_t sh = (pf ? Z3.total_pf : Z3.total_ov) * 8;
        const int ntk = G.end - G.beg;
        const dim3 hg(ntk, nd);
        const FormTask* ft = D.form + G.beg;
        const int* cb = D.fcbeg + G.beg;
        // persistent CTAs: as many as fit on the SMs at once
        const dim3 pg(D.pgrid(ntk, ks * mt <= 4 && 2 * (sh + 1024) <= 228 * 1024 ? 2 : 1), nd);
        if (ks <= 4 && mt <= 4 && sh <= 227 * 1024) {
          switch (4 * (ks - 1) + mt - 1) {
#define H2PW_CASE(KS_, MT_)                                                                        \
  case 4 * (KS_ - 1) + MT_ - 1:                                                                    \
    CK(smem_limit(k_form3d_h2pw_mma<KS_, MT_>)); \
    k_form3d_h2pw_mma<KS_, MT_><<<pg, 256, sh, st>>>(k, ft, ntk, cb, D.fchunks, D.hbuf, pf);       \
    break;
            H2PW_CASE(1, 1) H2PW_CASE(1, 2) H2PW_CASE(1, 3) H2PW_CASE(1, 4)
            H2PW_CASE(2, 1) H2PW_CASE(2, 2) H2PW_CASE(2, 3) H2PW_CASE(2, 4)
            H2PW_CASE(3, 1) H2PW_CASE(3, 2) H2PW_CASE(3, 3) H2PW_CASE(3, 4)
            H2PW_CASE(4, 1) H2PW_CASE(4, 2) H2PW_CASE(4, 3) H2PW_CASE(4, 4)
#undef H2PW_CASE
            default: return cudaErrorNotSupported;
          }
        } else {
          const size_t shb = form3_simt_smem(Pn, P.npw);
          CK(smem_limit(k_form3d_h2pw));
          k_form3d_h2pw<<<hg, 512, shb, st>>>(k, ft, cb, D.fchunks, D.hbuf);
        }
        launches++;
      }
    }
    if (P.dim == 3 && D.form3_nsplit < D.form_hermite_n) {
      // scratch fallback for the orders above the shared-memory kernels
      const FormTask* ft = D.form + D.form3_nsplit;
      const int nft = D.form_hermite_n - D.form3_nsplit;
      int Pn = D.form_pmax + 1;
      size_t sh = ((size_t)Pn * Pn * Pn + 3 * FORM_CH * Pn) * 8;
      if (Pn > 32 || sh > 227 * 1024) return cudaErrorNotSupported;
      int grid = std::min(D.scratch_ctas, 2 * D.psm());
      if (Pn <= 16) {
        CK(smem_limit(k_form3d_hermite<16>));
        k_form3d_hermite<16><<<grid, 256, sh, st>>>(k, ft, nft, D.scratch, D.scratch_per_cta, D.isq);
      } else {
        CK(smem_limit(k_form3d_hermite<32>));
        k_form3d_hermite<32><<<grid, 256, sh, st>>>(k, ft, nft, D.scratch, D.scratch_per_cta, D.isq);
      }
      launches++;
    }
    if (P.dim == 3 && D.form_pw_n > 0) {
      size_t sh = ((size_t)FORM_CH * (2 * P.npw + n2) + 8) * 16;
      CK(smem_limit(k_form3d_pw));
      k_form3d_pw<<<dim3(D.form_pw_n, nd), 256, sh, st>>>(k, D.form + D.form_hermite_n);
      launches++;
    }
    if (P.dim == 2 && D.form_pw_n > 0) {  // the NUFFT scheme's direct form
      const size_t sh = (size_t)FORM_CH * (P.npw + n2) * 16;
      if (sh > 227 * 1024) return cudaErrorNotSupported;
      CK(smem_limit(k_form2d_pw));
      k_form2d_pw<<<dim3(D.form_pw_n, nd), 256, sh, st>>>(k, D.form + D.form_hermite_n);
      launches++;
    }
    mark(2);
    // (b) merge, bottom-up
    for (int l = P.nlevels - 1; l >= P.nlevstart; l--) {
      int ng = D.merge_end[l] - D.merge_beg[l];
      if (ng <= 0) continue;
      k_merge<<<dim3(ng, echunks), 256, 0, st>>>(k, D.mgroups + D.merge_beg[l], D.merge);
      launches++;
    }
   }  // phase 1
    mark(3);
   if (ph2) {
    if (D.nm2l > 0) {
      k_m2l<<<dim3(D.nm2l, echunks), 256, 0, st>>>(k, D.m2l, D.m2l_nbr);
      launches++;
    }
    mark(4);
    for (int l = P.nlevstart; l <= P.nlevels - 1; l++) {
      int nsp = D.split_end[l] - D.split_beg[l];
      if (nsp <= 0) continue;
      k_split<<<dim3(nsp, schunks), 256, 0, st>>>(k, D.split + D.split_beg[l]);
      launches++;
    }
    mark(5);
    // (c) eval
    if (P.dim == 2 && D.neval > 0) {
      for (const OrderGroup& G : D.conv_groups) {
        const int Pn = G.p + 1, nt = G.end - G.beg;
        const ConvDims Z(Pn, P.npw);
        if (Z.K1 / 4 > CONV_MAXKS) return cudaErrorNotSupported;
        int nw = 4;
        while (nw > 1 && (size_t)nw * Z.warp * 8 > 100 * 1024) nw >>= 1;
        const size_t sh = (size_t)nw * Z.warp * 8;
        if (sh > 227 * 1024) return cudaErrorNotSupported;
        const dim3 cg((nt + nw - 1) / nw, nd);
        // the blocks the mixed evaluation reads (the condition of its launch below)
        const int f32 = mixed_ac && pgh == 1 && (Pn + 1) / 2 <= 16;
        switch (Z.K1 / 4) {
#define CONV_CASE(N)                                                                              \
  case N:                                                                                         \
    CK(smem_limit(k_pw2taylor2d<N>)); \
    k_pw2taylor2d<N><<<cg, 32 * nw, sh, st>>>(k, D.conv + G.beg, nt, D.lo, D.tables + G.tab, f32);  \
    break;
          CONV_CASE(1) CONV_CASE(2) CONV_CASE(3) CONV_CASE(4) CONV_CASE(5) CONV_CASE(6)
          CONV_CASE(7) CONV_CASE(8) CONV_CASE(9) CONV_CASE(10) CONV_CASE(11) CONV_CASE(12)
#undef CONV_CASE
          default: return cudaErrorNotSupported;
        }
        launches++;
      }
      for (const OrderGroup& G : D.horner_groups) {
        const int Pn = G.p + 1, np2 = (Pn + 1) / 2;
        const dim3 g(G.end - G.beg, nd);
        const HornerTask* tk = D.horner + G.beg;
        const size_t sh = (size_t)Pn * np2 * 16;
        if (sh > 227 * 1024) return cudaErrorNotSupported;
        if (mixed_ac && pgh == 1 && np2 <= 16) {
          CK(launch_eval2d_horner_f32(k, tk, G.end - G.beg, nd, Pn, D.lo, st));
          launches++;
          continue;
        }
        {
          const cudaError_t e_pgh = with_pgh(pgh, [&](auto G) -> cudaError_t {
          constexpr int PG = decltype(G)::value;
          switch (np2) {
#define HORNER_CASE(N)                                                                            \
  case N:                                                                                         \
    CK(smem_limit(k_eval2d_horner<N, PG>)); \
    k_eval2d_horner<N, PG><<<g, 128, sh, st>>>(k, tk, D.lo);                                      \
    break;
            HORNER_CASE(1) HORNER_CASE(2) HORNER_CASE(3) HORNER_CASE(4) HORNER_CASE(5) HORNER_CASE(6)
            HORNER_CASE(7) HORNER_CASE(8) HORNER_CASE(9) HORNER_CASE(10) HORNER_CASE(11) HORNER_CASE(12)
            HORNER_CASE(13) HORNER_CASE(14) HORNER_CASE(15) HORNER_CASE(16) HORNER_CASE(17) HORNER_CASE(18)
            HORNER_CASE(19) HORNER_CASE(20) HORNER_CASE(21) HORNER_CASE(22) HORNER_CASE(23) HORNER_CASE(24)
            HORNER_CASE(25) HORNER_CASE(26) HORNER_CASE(27) HORNER_CASE(28) HORNER_CASE(29) HORNER_CASE(30)
            HORNER_CASE(31) HORNER_CASE(32)
#undef HORNER_CASE
            default:
              CK(smem_limit(k_eval2d_horner_any<PG>));
              k_eval2d_horner_any<PG><<<g, 128, sh, st>>>(k, tk, D.lo);
          }
          return cudaSuccess;
        });
          CK(e_pgh);
        }
        launches++;
      }
      if (D.eval_pw_n > 0) {
        {
          const cudaError_t e_pgh = with_pgh(pgh, [&](auto G) -> cudaError_t {
          k_eval2d<decltype(G)::value><<<dim3(D.eval_pw_n, nd), 256, 0, st>>>(k, D.eval + D.eval_taylor_n);
          return cudaSuccess;
        });
          CK(e_pgh);
        }
        launches++;
      }
    }
    if (P.dim == 3 && D.eval3_split) {
      for (const OrderGroup& G : D.conv_groups) {
        const int Pn = G.p + 1, nt = G.end - G.beg;
        const int nw = 4;
        const size_t sh = conv3_smem_bytes(Pn, P.npw, nw);
        const dim3 cg(std::min(nt, std::min(D.conv3_ctas, 4 * D.psm())), nd);
        const int n2 = P.npw / 2, ksm = (n2 + 3) / 4;
        const size_t shm = C3Dims(Pn, P.npw).total * 8;
        if (Pn <= 16 && ksm <= 8 && shm <= 227 * 1024) {
          const dim3 pg(D.pgrid(nt, 2 * (shm + 1024) <= 228 * 1024 ? 2 : 1), nd);
          switch (ksm) {
#define CONV3M_CASE(N)                                                                            \
  case N:                                                                                         \
    CK(smem_limit(k_pw2taylor3d_mma<N>)); \
    k_pw2taylor3d_mma<N><<<pg, 256, shm, st>>>(k, D.conv + G.beg, nt, D.lo);                      \
    break;
            CONV3M_CASE(1) CONV3M_CASE(2) CONV3M_CASE(3) CONV3M_CASE(4)
            CONV3M_CASE(5) CONV3M_CASE(6) CONV3M_CASE(7) CONV3M_CASE(8)
#undef CONV3M_CASE
            default: return cudaErrorNotSupported;
          }
          launches++;
          continue;
        }
        int gs2 = 4;
        while (gs2 > 1 && C3Dims2(Pn, P.npw, gs2).total * 8 > 227 * 1024) gs2 >>= 1;
        const size_t shm2 = C3Dims2(Pn, P.npw, gs2).total * 8;
        if (Pn > 16 && Pn <= 32 && ksm <= 8 && shm2 <= 227 * 1024) {
          const dim3 pg(D.pgrid(nt, 1), nd);
          switch (ksm) {
#define CONV3M2_CASE(N)                                                                           \
  case N:                                                                                         \
    CK(smem_limit(k_pw2taylor3d_mma2<N>)); \
    k_pw2taylor3d_mma2<N><<<pg, 256, shm2, st>>>(k, D.conv + G.beg, nt, D.lo, gs2);               \
    break;
            CONV3M2_CASE(1) CONV3M2_CASE(2) CONV3M2_CASE(3) CONV3M2_CASE(4)
            CONV3M2_CASE(5) CONV3M2_CASE(6) CONV3M2_CASE(7) CONV3M2_CASE(8)
#undef CONV3M2_CASE
            default: return cudaErrorNotSupported;
          }
          launches++;
          continue;
        }
        switch ((P.npw + 3) / 4) {
#define CONV3_CASE(N)                                                                             \
  case N:                                                                                         \
    CK(smem_limit(k_pw2taylor3d<N>)); \
    k_pw2taylor3d<N><<<cg, 32 * nw, sh, st>>>(k, D.conv + G.beg, nt, D.lo, D.tables + G.tab,      \
                                              D.uscr, D.uscr_per_cta);                            \
    break;
          CONV3_CASE(1) CONV3_CASE(2) CONV3_CASE(3) CONV3_CASE(4) CONV3_CASE(5) CONV3_CASE(6)
          CONV3_CASE(7) CONV3_CASE(8) CONV3_CASE(9) CONV3_CASE(10) CONV3_CASE(11) CONV3_CASE(12)
#undef CONV3_CASE
          default: return cudaErrorNotSupported;
        }
        launches++;
      }
      for (const OrderGroup& G : D.horner_groups) {
        const int Pn = G.p + 1, np2 = (Pn + 1) / 2;
        const dim3 g(G.end - G.beg, nd);
        const HornerTask* tk = D.horner + G.beg;
        const size_t sh = (size_t)Pn * Pn * np2 * 16;
        if (sh > 227 * 1024) return cudaErrorNotSupported;
        if (mixed_ac && pgh == 1 && eval3d_tc_supported(Pn)) {
          // mixed form: the Taylor evaluation as BF16 x 3 tensor-core products
          CK(launch_eval3d_tc(k, tk, G.end - G.beg, nd, Pn, D.lo, st));
          launches++;
          continue;
        }
        {
          const cudaError_t e_pgh = with_pgh(pgh, [&](auto G) -> cudaError_t {
          constexpr int PG = decltype(G)::value;
          switch (np2) {
#define HORNER3_CASE(N)                                                                           \
  case N:                                                                                         \
    CK(smem_limit(k_eval3d_horner<N, PG>)); \
    k_eval3d_horner<N, PG><<<g, 128, sh, st>>>(k, tk, D.lo);                                      \
    break;
            HORNER3_CASE(1) HORNER3_CASE(2) HORNER3_CASE(3) HORNER3_CASE(4) HORNER3_CASE(5)
            HORNER3_CASE(6) HORNER3_CASE(7) HORNER3_CASE(8) HORNER3_CASE(9) HORNER3_CASE(10)
            HORNER3_CASE(11) HORNER3_CASE(12) HORNER3_CASE(13) HORNER3_CASE(14) HORNER3_CASE(15)
#undef HORNER3_CASE
            default: return cudaErrorNotSupported;
          }
          return cudaSuccess;
        });
          CK(e_pgh);
        }
        launches++;
      }
    }
    // 3D Taylor tasks beyond the conversion kernels' orders, and the
    // plane-wave route: the direct separable evaluation for potentials
    const int nbig = P.dim == 3 ? D.eval_taylor_n - D.eval3_nsplit : 0;
    const size_t sh_sep = ((size_t)(2 * P.npw + P.npw / 2) * SEP_NPB + 256 * 4) * 16 +
                          (size_t)(D.eval_pmax + 1) * P.npw * 8;
    if (nbig > 0 && pgh == 1) {
      CK(smem_limit(k_eval3d_sep<true>));
      k_eval3d_sep<true><<<dim3(nbig, nd), 256, sh_sep, st>>>(k, D.eval + D.eval3_nsplit);
      launches++;
    } else if (nbig > 0 && D.eval3_smem) {
      {
          const cudaError_t e_pgh = with_pgh(pgh, [&](auto G) -> cudaError_t {
        constexpr int PG = decltype(G)::value;
        CK(smem_limit(k_eval3d_taylor_smem<PG>));
        k_eval3d_taylor_smem<PG><<<dim3(nbig, nd), 512, D.eval3_sh, st>>>(k, D.eval + D.eval3_nsplit);
        return cudaSuccess;
      });
          CK(e_pgh);
        }
      launches++;
    } else if (nbig > 0) {
      {
          const cudaError_t e_pgh = with_pgh(pgh, [&](auto G) -> cudaError_t {
        k_eval3d_taylor<decltype(G)::value><<<std::min(D.scratch_ctas, 2 * D.psm()), 256, 0, st>>>(k, D.eval + D.eval3_nsplit, nbig,
                                                                           D.scratch, D.scratch_per_cta);
        return cudaSuccess;
      });
          CK(e_pgh);
        }
      launches++;
    }
    if (P.dim == 3 && D.eval_pw_n > 0 && pgh == 1) {
      CK(smem_limit(k_eval3d_sep<false>));
      k_eval3d_sep<false><<<dim3(D.eval_pw_n, nd), 256, sh_sep, st>>>(k, D.eval + D.eval_taylor_n);
      launches++;
    } else if (P.dim == 3 && D.eval_pw_n > 0) {
      {
          const cudaError_t e_pgh = with_pgh(pgh, [&](auto G) -> cudaError_t {
        k_eval3d_pw<decltype(G)::value><<<dim3(D.eval_pw_n, nd), 256, 0, st>>>(k, D.eval + D.eval_taylor_n);
        return cudaSuccess;
      });
          CK(e_pgh);
        }
      launches++;
    }
   }  // phase 2
  } else {
    mark(2); mark(3); mark(4); mark(5);
  }
  mark(6);
  // (d) near field
  if (ph2 && D.ndir > 0) {
    dim3 g((D.ndir + 3) / 4, nd);
    // dipoles take the FP64 near field (the mixed form is charges only)
    const bool mixed = precision == PREC_MIXED && !P.ifdipole;
    const double l2e = 1.4426950408889634;
    const double cs = std::sqrt(l2e / P.delta);
    const float amax = (float)(P.dmax * l2e / P.delta);
    if (mixed && pgh == 1) {
      // potentials only: the packed-FP32 kernel
      CK(launch_direct_mixed_x2(k, D.dir, D.ndir, nd, D.dir_src, amax, st));
    } else {
          const cudaError_t e_pgh = with_pgh(pgh, [&](auto G) -> cudaError_t {
      constexpr int PG = decltype(G)::value;
      if (P.dim == 2) {
        if (mixed) k_direct_mixed<2, PG><<<g, 128, 0, st>>>(k, D.dir, D.ndir, D.dir_src, cs, amax);
        else if (P.ifdipole) k_direct<2, PG, true><<<g, 128, 0, st>>>(k, D.dir, D.ndir, D.dir_src);
        else k_direct<2, PG, false><<<g, 128, 0, st>>>(k, D.dir, D.ndir, D.dir_src);
      } else {
        if (mixed) k_direct_mixed<3, PG><<<g, 128, 0, st>>>(k, D.dir, D.ndir, D.dir_src, cs, amax);
        else if (P.ifdipole) k_direct<3, PG, true><<<g, 128, 0, st>>>(k, D.dir, D.ndir, D.dir_src);
        else k_direct<3, PG, false><<<g, 128, 0, st>>>(k, D.dir, D.ndir, D.dir_src);
      }
      return cudaSuccess;
    });
          CK(e_pgh);
        }
    launches++;
  }
  mark(7);
  // sorted rows [nc][nd] -> pot (nd, n), grad (nd, dim, n), hess (nd, H, n)
  const int nh = P.dim == 2 ? 3 : 6;
  auto unsort = [&](const double* in, const int* inv, int n, int nc, double* pot, double* grad,
                    double* hess) {
    if (pot) {
      // one density, one component per point: the same random gather
      if (nd == 1 && nc == 1) k_gather1<<<gb, 256, 0, st>>>(in, inv, n, pot);
      else k_unsort<<<gb, 256, 0, st>>>(in, pot, inv, n, nc * nd, 0, nd);
      launches++;
    }
    if (nc > 1 && grad) {
      k_unsort<<<gb, 256, 0, st>>>(in, grad, inv, n, nc * nd, nd, P.dim * nd);
      launches++;
    }
    if (nc > 1 + P.dim && hess) {
      k_unsort<<<gb, 256, 0, st>>>(in, hess, inv, n, nc * nd, (1 + P.dim) * nd, nh * nd);
      launches++;
    }
  };
  if (ph2 && P.ifpgh > 0 && P.ns > 0) unsort(D.psort, D.isrc_inv, P.ns, k.nc_s, outs.pot, outs.grad, outs.hess);
  if (ph2 && P.ifpghtarg > 0 && P.nt > 0)
    unsort(D.ptsort, D.itarg_inv, P.nt, k.nc_t, outs.pottarg, outs.gradtarg, outs.hesstarg);
  mark(8);
  D.launches = launches;
  CK(cudaGetLastError());
  if (times) {
    CK(cudaEventSynchronize(ev[8]));
    // stage i spans marks i..i+1; the shift stages merge/m2l/split are 2..5
    float t[8];
    for (int i = 0; i < 8; i++) cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]);
    for (int i = 0; i < 8; i++) times->ms[i] = t[i];
    if (times->dom_name[0]) cudaEventElapsedTime(&times->dom_ms, dev0, dev1);
    for (int i = 0; i < 9; i++) cudaEventDestroy(ev[i]);
    cudaEventDestroy(dev0);
    cudaEventDestroy(dev1);
  }
  return cudaSuccess;
}

cudaError_t probe_fp64_mma(double* tflops) {
  int dev = 0, sms = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int iters = 4096, blocks = sms * 16;
  k_probe_dmma<<<blocks, 128>>>(nullptr, 64);  // warm-up
  CK(cudaEventRecord(e0));
  k_probe_dmma<<<blocks, 128>>>(nullptr, iters);
  CK(cudaEventRecord(e1));
  CK(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const double fma = (double)blocks * 4 * 8 * 256 * iters;
  *tflops = 2.0 * fma / (ms * 1e-3) / 1e12;
  return cudaGetLastError();
}

size_t large_delta_work_doubles(const Params& P, bool deterministic) {
  const size_t Pn = P.nlocal0 + 1;
  const size_t nent = P.dim == 2 ? Pn * Pn : Pn * Pn * Pn;
  return (size_t)P.nd * nent * (deterministic ? 1 + LD_PARTS : 1);
}

cudaError_t large_delta_execute(const Params& P, const double* src, const Inputs& in,
                                const double* trg, const Outputs& outs, double* work,
                                cudaStream_t st, bool deterministic) {
  KP k;
  memset(&k, 0, sizeof(k));
  k.dim = P.dim; k.nd = P.nd; k.dsq = P.dsq; k.delta = P.delta;
  k.src = src; k.chg = in.charge;
  k.ifcharge = P.ifcharge; k.ifdipole = P.ifdipole;
  k.dnrm = in.rnormal; k.dstr = in.dipstr;  // caller order: this path sorts nothing
  int p = P.nlocal0;
  int Pn = p + 1;
  size_t nent = P.dim == 2 ? (size_t)Pn * Pn : (size_t)Pn * Pn * Pn;
  // the centre travels by value in the kernel arguments (no host->device copy)
  const double3 cen = make_double3(P.cen0[0], P.cen0[1], P.dim == 3 ? P.cen0[2] : 0.0);
  double* local = work;
  CK(cudaMemsetAsync(local, 0, nent * P.nd * sizeof(double), st));
  size_t sh = 3 * FORM_CH * Pn * 8;
  if (sh > 227 * 1024) return cudaErrorNotSupported;
  if (sh > 48 * 1024) {
    CK(smem_limit(k_ld_form<2>));
    CK(smem_limit(k_ld_form<3>));
  }
  // deterministic: per-CTA partial blocks after the local block, summed in
  // CTA order; otherwise atomic accumulation (last-bit order dependence)
  double* partial = deterministic ? local + nent * P.nd : nullptr;
  int blocks = std::max(1, std::min(deterministic ? LD_PARTS : 1024, (P.ns + 255) / 256));
  if (P.ns > 0) {
    if (P.dim == 2) k_ld_form<2><<<dim3(blocks, P.nd), 256, sh, st>>>(k, P.ns, p, cen, local, partial);
    else k_ld_form<3><<<dim3(blocks, P.nd), 256, sh, st>>>(k, P.ns, p, cen, local, partial);
    if (deterministic) {
      const int sb = std::max(1, std::min(1024, (int)((nent + 255) / 256)));
      k_ld_sum<<<dim3(sb, P.nd), 256, 0, st>>>((int)nent, blocks, partial, local);
    }
  }
  auto ev = [&](const double* pts, int n, int pgh, double* pot, double* grad, double* hess) -> cudaError_t {
    if (n <= 0 || pgh <= 0) return cudaSuccess;
    int b = std::max(1, std::min(4096, (n + 255) / 256));
    return with_pgh(pgh, [&](auto G) -> cudaError_t {
      constexpr int PG = decltype(G)::value;
      if (P.dim == 2) k_ld_eval<2, PG><<<dim3(b, P.nd), 256, 0, st>>>(k, n, pts, pot, grad, hess, p, cen, local);
      else k_ld_eval<3, PG><<<dim3(b, P.nd), 256, 0, st>>>(k, n, pts, pot, grad, hess, p, cen, local);
      return cudaSuccess;
    });
  };
  CK(ev(trg, P.nt, P.ifpghtarg, outs.pottarg, outs.gradtarg, outs.hesstarg));
  CK(ev(src, P.ns, P.ifpgh, outs.pot, outs.grad, outs.hess));
  return cudaGetLastError();
}


// ------------------------------------------------------------ allocation-free large-delta call
// Some callers cannot let this library allocate device memory: codes that
// hand over device arrays from their own pool and run under a fixed memory
// budget, and latency-critical loops that must not pay for cudaMalloc, which
// can synchronise the whole device.  For them the large-delta transform (one
// Taylor local about a given centre, the reference's fgt2d_large_delta /
// fgt3d_large_delta) runs with its only scratch -- the local expansion -- in
// this fixed device array.  Every device that loads the
// library holds it (512 KB) until the process exits; every call shares it, so
// calls that overlap on the GPU race; each call clears what it accumulates.
namespace {
constexpr size_t kNoAllocScratchDoubles = 65536;
__device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles + 8];
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[64] = {nullptr};
}  // namespace

size_t large_delta_noalloc_capacity() { return kNoAllocScratchDoubles; }

cudaError_t large_delta_noalloc(const Params& P, const double* src, const double* chg,
                                const double* trg, double* pot, double* pottarg, cudaStream_t st) {
  const size_t Pn = (size_t)P.nlocal0 + 1;
  const size_t nent = P.dim == 2 ? Pn * Pn : Pn * Pn * Pn;
  if (P.nlocal0 < 0 || nent * P.nd > kNoAllocScratchDoubles) return cudaErrorInvalidValue;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  double* work = nullptr;
  {
    // the host name of the array is not a device address: its address on
    // this device is looked up once, with this device current
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* ptr = nullptr;
      CK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
      g_noalloc_ptr[dev] = static_cast<double*>(ptr);
    }
    work = g_noalloc_ptr[dev];
  }
  // the source staging of the local-expansion kernel grows with the order
  const int sh = (int)(3 * FORM_CH * Pn * 8);
  if (sh > 48 * 1024) {
    CK(smem_limit(k_ld_form<2>));
    CK(smem_limit(k_ld_form<3>));
  }
  // large_delta_execute clears the local expansion (work[0..nd*nent)) on the
  // stream before accumulating into it; the centre goes by value in the
  // kernel arguments, so the call makes no host->device copy
  Outputs o;
  o.pot = pot;
  o.pottarg = pottarg;
  Inputs in;
  in.charge = chg;
  return large_delta_execute(P, src, in, trg, o, work, st, false);
}

}  // namespace fgtb
