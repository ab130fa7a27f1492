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
#include <cstdio>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "fgt_device.hpp"

namespace fgtb {

namespace {

constexpr int FORM_CH = 32;    // sources staged per chunk in the form kernels

struct KP {
  int dim, nd, npw, n2, nexp;
  double dsq, delta, dmax, t1;
  const double* centers;
  const double* h2x;
  const double* x2l;
  const double* ws;
  const double2* wms;
  const double2* wsh;
  double2* mp;
  double2* loc;
  const double* src;
  const double* chg;
  const double* trg;
  double* pot;
  double* pottarg;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {  // c + a b
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 cfmac(double2 a, double2 b, double2 c) {  // c + a conj(b)
  return make_double2(fma(a.x, b.x, fma(a.y, b.y, c.x)), fma(a.y, b.x, fma(-a.x, b.y, c.y)));
}
// z * i^j
__device__ __forceinline__ double2 rot(double2 z, int j) {
  switch (j & 3) {
    case 0: return z;
    case 1: return make_double2(-z.y, z.x);
    case 2: return make_double2(-z.x, -z.y);
    default: return make_double2(z.y, -z.x);
  }
}
// a + v * i^j for real v
__device__ __forceinline__ void addrot(double2& a, double v, int j) {
  switch (j & 3) {
    case 0: a.x += v; break;
    case 1: a.y += v; break;
    case 2: a.x -= v; break;
    default: a.y -= v; break;
  }
}
__device__ __forceinline__ double2 cexpi(double th) {
  double s, c;
  sincos(th, &s, &c);
  return make_double2(c, s);
}
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

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
// Caller order: out row j = in row iperm[j] (dreorderi, fmmcommon2d.f:29-56),
// written as a gather so the stores stay coalesced.
__global__ void k_unsort(const double* __restrict__ in, double* __restrict__ out,
                         const int* __restrict__ iperm, int n, int nd) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const long long p = iperm[j];
    for (int c = 0; c < nd; c++) out[(long long)j * nd + c] = in[p * nd + c];
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
  for (int c0 = 0; c0 < T.n; c0 += ch) {
    const int m = min(ch, T.n - c0);
    for (int r = tid; r < 2 * m; r += 256) {
      const int t = r >> 1, kind = r & 1;
      const int i = T.s0 + c0 + t;
      double v, w;
      if (kind == 0) { v = (k.src[2 * i] - cx) * k.dsq; w = 1.0; }
      else { v = (k.src[2 * i + 1] - cy) * k.dsq; w = k.chg[(size_t)i * k.nd + ind]; }
      double* row = (kind ? ys : xs) + t * Pp;
      row[0] = w;
      for (int j = 1; j < Pn; j++) {
        w = w * v * isq[j];
        row[j] = w;
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
                                                        size_t slab) {
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
    for (int c0 = 0; c0 < T.n; c0 += FORM_CH) {
      const int m = min(FORM_CH, T.n - c0);
      if (threadIdx.x < m) {
        const int i = T.s0 + c0 + threadIdx.x;
        const double x = (k.src[3 * i] - cx) * k.dsq, y = (k.src[3 * i + 1] - cy) * k.dsq,
                     z = (k.src[3 * i + 2] - cz) * k.dsq;
        double* xr = X + threadIdx.x * Pn;
        double* yr = Y + threadIdx.x * Pn;
        double* zr = Z + threadIdx.x * Pn;
        double xv = 1.0, yv = 1.0, zv = k.chg[(size_t)i * k.nd + ind];
        xr[0] = xv; yr[0] = yv; zr[0] = zv;
        for (int j = 1; j < Pn; j++) {
          double sj = sqrt((double)j);
          xv = xv * x / sj; yv = yv * y / sj; zv = zv * z / sj;
          xr[j] = xv; yr[j] = yv; zr[j] = zv;
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
// Same product as k_form2d, H (P x P, P <= 8 NT) = sum_t x_t^j (q_t y_t^k),
// on the FP64 tensor cores: mma.sync.m8n8k4.f64 takes four sources per step
// (K = 4) into NT x NT tiles of 8 x 8.  Fragment layout (PTX ISA, m8n8k4
// .f64): A element (row = lane/4, col = lane%4), B element (row = lane%4,
// col = lane/4), accumulator pair (row = lane/4, col = 2 (lane%4) + i).  Lane
// (j0 = lane/4, t = lane%4) therefore needs x_t^(j0 + 8 m) / sqrt((j0+8m)!)
// and q_t y_t^(j0 + 8 m) / sqrt(..) for m < NT, built from x, x^2, x^4, x^8.
// Four warps split the leaf's sources; their tiles are summed in shared
// memory, then the Hermite -> plane-wave passes run as in k_form2d.
__device__ __forceinline__ void dmma_884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <int NT>
__global__ void __launch_bounds__(128) k_form2d_mma(KP k, const FormTask* __restrict__ tasks,
                                                    const double* __restrict__ cfac) {
  constexpr int PP = 8 * NT;
  const FormTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  const int Pn = T.p + 1, n2 = k.n2, npw = k.npw;
  __shared__ double part[4][PP * PP];
  __shared__ double cf[PP];
  extern __shared__ double2 px[];  // [Pn][n2], then the h2x table [Pn][npw]
  double* hx = reinterpret_cast<double*>(px + Pn * n2);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x < PP) cf[threadIdx.x] = cfac[threadIdx.x];
  for (int e = threadIdx.x; e < Pn * npw; e += 128) hx[e] = k.h2x[e];
  __syncthreads();
  const double cx = k.centers[2 * T.box], cy = k.centers[2 * T.box + 1];
  const int j0 = lane >> 2, tl = lane & 3;
  double c[NT][NT][2], c2[NT][NT][2];
#pragma unroll
  for (int a = 0; a < NT; a++)
#pragma unroll
    for (int b = 0; b < NT; b++) c[a][b][0] = c[a][b][1] = c2[a][b][0] = c2[a][b][1] = 0.0;
  double cj[NT];
#pragma unroll
  for (int m = 0; m < NT; m++) cj[m] = cf[j0 + 8 * m];
  // each warp takes steps of four sources: two steps (eight sources) per
  // iteration as independent chains, warps interleaved
  auto rows = [&](int t, double* av, double* bv) {
    double x = 0.0, y = 0.0, q = 0.0;
    if (t < T.n) {
      const int i = T.s0 + t;
      x = (k.src[2 * i] - cx) * k.dsq;
      y = (k.src[2 * i + 1] - cy) * k.dsq;
      q = k.chg[(size_t)i * k.nd + ind];
    }
    const double x2 = x * x, x4 = x2 * x2, x8 = x4 * x4;
    const double y2 = y * y, y4 = y2 * y2, y8 = y4 * y4;
    double xa = (j0 & 1) ? x : 1.0, ya = (j0 & 1) ? y : 1.0;
    if (j0 & 2) { xa *= x2; ya *= y2; }
    if (j0 & 4) { xa *= x4; ya *= y4; }
    ya *= q;
#pragma unroll
    for (int m = 0; m < NT; m++) {
      av[m] = xa * cj[m];
      bv[m] = ya * cj[m];
      xa *= x8;
      ya *= y8;
    }
  };
  for (int t0 = 8 * warp; t0 < T.n; t0 += 32) {
    double av0[NT], bv0[NT], av1[NT], bv1[NT];
    rows(t0 + tl, av0, bv0);
    rows(t0 + 4 + tl, av1, bv1);
#pragma unroll
    for (int a = 0; a < NT; a++)
#pragma unroll
      for (int b = 0; b < NT; b++) {
        dmma_884(c[a][b][0], c[a][b][1], av0[a], bv0[b]);
        dmma_884(c2[a][b][0], c2[a][b][1], av1[a], bv1[b]);
      }
  }
#pragma unroll
  for (int a = 0; a < NT; a++)
#pragma unroll
    for (int b = 0; b < NT; b++) {
      c[a][b][0] += c2[a][b][0];
      c[a][b][1] += c2[a][b][1];
    }
  // tile (a, b) holds H[j = 8a + lane/4][k = 8b + 2 (lane%4) + i]
#pragma unroll
  for (int a = 0; a < NT; a++)
#pragma unroll
    for (int b = 0; b < NT; b++)
#pragma unroll
      for (int i = 0; i < 2; i++) part[warp][(8 * a + j0) + PP * (8 * b + 2 * tl + i)] = c[a][b][i];
  __syncthreads();
  for (int e = threadIdx.x; e < PP * PP; e += 128)
    part[0][e] = part[0][e] + part[1][e] + part[2][e] + part[3][e];
  __syncthreads();
  const double* H = part[0];
  for (int idx = threadIdx.x; idx < Pn * n2; idx += 128) {
    const int j2 = idx / n2, k2 = idx - j2 * n2;
    double2 a = make_double2(0.0, 0.0);
    for (int j1 = 0; j1 < Pn; j1++) addrot(a, hx[j1 * npw + k2] * H[j1 + PP * j2], j1);
    px[idx] = a;
  }
  __syncthreads();
  double2* out = k.mp + ((size_t)T.slot * k.nd + ind) * k.nexp;
  for (int e = threadIdx.x; e < k.nexp; e += 128) {
    const int k1 = e / n2, k2 = e - k1 * n2;
    double2 a = make_double2(0.0, 0.0);
    for (int j2 = 0; j2 < Pn; j2++) {
      const double h = hx[j2 * npw + k1];
      const double2 z = rot(px[j2 * n2 + k2], j2);
      a.x = fma(h, z.x, a.x);
      a.y = fma(h, z.y, a.y);
    }
    out[e] = a;
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

template <int MAXP>
__global__ void __launch_bounds__(256) k_form3d_acc(KP k, const FormTask* __restrict__ tasks,
                                                    const FormChunk* __restrict__ chunks,
                                                    double* __restrict__ hbuf, const double* __restrict__ isq,
                                                    int sub) {
  const FormChunk C = chunks[blockIdx.x];
  const FormTask T = tasks[C.task];
  const int ind = blockIdx.y;
  const int Pn = T.p + 1, P2 = Pn * Pn, P3 = P2 * Pn;
  extern __shared__ double sm[];
  double* H = sm;
  double* X = H + P3;
  double* Y = X + sub * Pn;
  double* Z = Y + sub * Pn;
  const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1], cz = k.centers[3 * T.box + 2];
  for (int e = threadIdx.x; e < P3; e += blockDim.x) H[e] = 0.0;
  for (int c0 = 0; c0 < C.n; c0 += sub) {
    const int m = min(sub, C.n - c0);
    __syncthreads();
    for (int r = threadIdx.x; r < 3 * m; r += blockDim.x) {
      const int t = r / 3, d = r - 3 * t;
      const int i = C.s0 + c0 + t;
      const double v = (k.src[3 * i + d] - (d == 0 ? cx : d == 1 ? cy : cz)) * k.dsq;
      double w = d == 2 ? k.chg[(size_t)i * k.nd + ind] : 1.0;
      double* row = (d == 0 ? X : d == 1 ? Y : Z) + t * Pn;
      row[0] = w;
      for (int j = 1; j < Pn; j++) {
        w = w * v * isq[j];
        row[j] = w;
      }
    }
    __syncthreads();
    for (int pr = threadIdx.x; pr < P2; pr += blockDim.x) {
      const int j = pr % Pn, kk = pr / Pn;
      double acc[MAXP];
#pragma unroll
      for (int l = 0; l < MAXP; l++) acc[l] = l < Pn ? H[pr + P2 * l] : 0.0;
      for (int t = 0; t < m; t++) {
        const double a = X[t * Pn + j] * Y[t * Pn + kk];
        const double* zr = Z + t * Pn;
#pragma unroll
        for (int l = 0; l < MAXP; l++)
          if (l < Pn) acc[l] = fma(a, zr[l], acc[l]);
      }
#pragma unroll
      for (int l = 0; l < MAXP; l++)
        if (l < Pn) H[pr + P2 * l] = acc[l];
    }
  }
  __syncthreads();
  double* out = hbuf + ((size_t)C.hoff * k.nd + (size_t)ind * P3);
  for (int e = threadIdx.x; e < P3; e += blockDim.x) out[e] = H[e];
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
  // region A: H, later T2 [(j3 npw + k2) n2 + k1]; region B: T1 [(j3 + P j2) n2 + k1]
  const size_t szA = max((size_t)P3, (size_t)2 * Pn * npw * n2);
  double* H = sm;
  double2* T2 = reinterpret_cast<double2*>(sm);
  double2* T1 = reinterpret_cast<double2*>(sm + ((szA + 1) & ~size_t(1)));
  for (int e = threadIdx.x; e < P3; e += blockDim.x) {
    double v = 0.0;
    for (int c = cbeg[tk]; c < cbeg[tk + 1]; c++) v += hbuf[(size_t)chunks[c].hoff * k.nd + (size_t)ind * P3 + e];
    H[e] = v;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < P2 * n2; idx += blockDim.x) {
    const int k1 = idx % n2, jj = idx / n2;
    double2 a = make_double2(0.0, 0.0);
    for (int j1 = 0; j1 < Pn; j1++) addrot(a, k.h2x[j1 * npw + k1] * H[jj + P2 * j1], j1);
    T1[idx] = a;
  }
  __syncthreads();
  // y pass over the positive half k2 = n2 + m and its mirror n2 - 1 - m
  for (int idx = threadIdx.x; idx < Pn * n2 * n2; idx += blockDim.x) {
    const int k1 = idx % n2, r = idx / n2, m = r % n2, j3 = r / n2;
    const int kp = n2 + m, km = n2 - 1 - m;
    double2 ev = make_double2(0.0, 0.0), od = make_double2(0.0, 0.0);
    for (int j2 = 0; j2 < Pn; j2++) {
      const double h = k.h2x[j2 * npw + kp];
      const double2 z = rot(T1[(j3 + Pn * j2) * n2 + k1], j2);
      double2& acc = (j2 & 1) ? od : ev;
      acc.x = fma(h, z.x, acc.x);
      acc.y = fma(h, z.y, acc.y);
    }
    T2[((size_t)j3 * npw + kp) * n2 + k1] = make_double2(ev.x + od.x, ev.y + od.y);
    T2[((size_t)j3 * npw + km) * n2 + k1] = make_double2(ev.x - od.x, ev.y - od.y);
  }
  __syncthreads();
  double2* out = k.mp + ((size_t)T.slot * k.nd + ind) * k.nexp;
  // x pass into the slot, positive half k3 = n2 + m and mirror
  for (int idx = threadIdx.x; idx < n2 * npw * n2; idx += blockDim.x) {
    const int m = idx % n2, r = idx / n2, k2 = r % npw, k1 = r / npw;
    const int kp = n2 + m, km = n2 - 1 - m;
    double2 ev = make_double2(0.0, 0.0), od = make_double2(0.0, 0.0);
    for (int j3 = 0; j3 < Pn; j3++) {
      const double h = k.h2x[j3 * npw + kp];
      const double2 z = rot(T2[((size_t)j3 * npw + k2) * n2 + k1], j3);
      double2& acc = (j3 & 1) ? od : ev;
      acc.x = fma(h, z.x, acc.x);
      acc.y = fma(h, z.y, acc.y);
    }
    const size_t base = (size_t)npw * (k2 + (size_t)npw * k1);
    out[base + kp] = make_double2(ev.x + od.x, ev.y + od.y);
    out[base + km] = make_double2(ev.x - od.x, ev.y - od.y);
  }
}

// ------------------------------------------------------------ (c) eval, 2D Taylor on FP64 MMA
// One CTA (4 warps) per chunk of an evaluation leaf.  The leaf's plane-wave
// expansion is staged in shared memory and converted to the Taylor block
// lo[k2 + LD k1] (g2dpw2local_real_vec); then for eight points per warp step
//     E[t][k1] = sum_k2 x_t^k2 lo[k2][k1]      (mma.m8n8k4.f64, K = 4 per step)
//     pot_t   += sum_k1 E[t][k1] y_t^k1         (per lane, then two shuffles)
// The B fragments of lo stay in registers for the whole chunk.
template <int NT>
__global__ void __launch_bounds__(128) k_eval2d_mma(KP k, const EvalTask* __restrict__ tasks) {
  constexpr int PP = 8 * NT, LD = PP + 1;
  const EvalTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  const int npw = k.npw, n2 = k.n2, Pn = T.p + 1;
  extern __shared__ double sm[];
  double* lo = sm;                                   // [PP][LD], zero padded
  double2* lx = reinterpret_cast<double2*>(sm + ((PP * LD + 1) & ~1));  // [Pn][npw]
  double2* Ls = lx + Pn * npw;                       // [nexp]
  double* xl = reinterpret_cast<double*>(Ls + k.nexp);  // [Pn][npw]
  const double2* L = k.loc + ((size_t)T.slot * k.nd + ind) * k.nexp;
  for (int e = threadIdx.x; e < k.nexp; e += 128) Ls[e] = L[e];
  for (int e = threadIdx.x; e < PP * LD; e += 128) lo[e] = 0.0;
  for (int e = threadIdx.x; e < Pn * npw; e += 128) xl[e] = k.x2l[e];
  __syncthreads();
  for (int idx = threadIdx.x; idx < Pn * npw; idx += 128) {
    const int k2 = idx / npw, j1 = idx - k2 * npw;
    double2 a = make_double2(0.0, 0.0);
    for (int j2 = 0; j2 < n2; j2++) {
      const double h = xl[k2 * npw + j2];
      const double2 v = Ls[j2 + n2 * j1];
      a.x = fma(h, v.x, a.x);
      a.y = fma(h, v.y, a.y);
    }
    lx[idx] = rot(a, k2);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < Pn * Pn; idx += 128) {
    const int k1 = idx / Pn, k2 = idx - k1 * Pn;
    const double sg = (k1 & 1) ? -1.0 : 1.0;
    double2 a = make_double2(0.0, 0.0);
    for (int j1 = 0; j1 < n2; j1++) {
      const double h = xl[k1 * npw + j1];
      const double2 u = lx[k2 * npw + j1], v = lx[k2 * npw + j1 + n2];
      a.x = fma(h, fma(sg, v.x, u.x), a.x);
      a.y = fma(h, fma(sg, v.y, u.y), a.y);
    }
    lo[k2 + LD * k1] = 2.0 * rot(a, k1).x;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r4 = lane >> 2, c4 = lane & 3;
  // B fragment (row = k2 = 4 ks + c4, col = k1 = 8 b + r4)
  double bf[2 * NT][NT];
#pragma unroll
  for (int ks = 0; ks < 2 * NT; ks++)
#pragma unroll
    for (int b = 0; b < NT; b++) bf[ks][b] = lo[(4 * ks + c4) + LD * (8 * b + r4)];
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const double cx = k.centers[2 * T.box], cy = k.centers[2 * T.box + 1];
  // two groups of eight points per warp iteration (independent MMA chains)
  auto point = [&](int ta, double& x, double& y) {
    x = 0.0;
    y = 0.0;
    if (ta < T.n) {
      const int ip = T.i0 + ta;
      x = (pts[2 * ip] - cx) * k.dsq;
      y = (pts[2 * ip + 1] - cy) * k.dsq;
    }
  };
  auto finish = [&](int ta, double y, double (*c)[2]) {
    const double y2 = y * y, y8 = (y2 * y2) * (y2 * y2);
    double yb = (c4 & 1) ? y2 : 1.0;
    if (c4 & 2) yb *= y2 * y2;
    double r = 0.0;
#pragma unroll
    for (int b = 0; b < NT; b++) {
      r = fma(c[b][0], yb, r);
      r = fma(c[b][1], yb * y, r);
      yb *= y8;
    }
    r += __shfl_xor_sync(0xffffffffu, r, 1);
    r += __shfl_xor_sync(0xffffffffu, r, 2);
    if (c4 == 0 && ta < T.n) out[(size_t)(T.i0 + ta) * k.nd + ind] += r;
  };
  for (int t0 = 16 * warp; t0 < T.n; t0 += 64) {
    const int ta0 = t0 + r4, ta1 = t0 + 8 + r4;
    double x0, y0, x1, y1;
    point(ta0, x0, y0);
    point(ta1, x1, y1);
    const double x20 = x0 * x0, x40 = x20 * x20, x21 = x1 * x1, x41 = x21 * x21;
    double xa0 = (c4 & 1) ? x0 : 1.0, xa1 = (c4 & 1) ? x1 : 1.0;
    if (c4 & 2) { xa0 *= x20; xa1 *= x21; }
    double c0[NT][2], c1[NT][2];
#pragma unroll
    for (int b = 0; b < NT; b++) c0[b][0] = c0[b][1] = c1[b][0] = c1[b][1] = 0.0;
#pragma unroll
    for (int ks = 0; ks < 2 * NT; ks++) {
#pragma unroll
      for (int b = 0; b < NT; b++) {
        dmma_884(c0[b][0], c0[b][1], xa0, bf[ks][b]);
        dmma_884(c1[b][0], c1[b][1], xa1, bf[ks][b]);
      }
      xa0 *= x40;
      xa1 *= x41;
    }
    finish(ta0, y0, c0);
    finish(ta1, y1, c1);
  }
}

// ------------------------------------------------------------ (c) eval, 3D Taylor in shared memory
// One CTA per chunk of an evaluation leaf: plane wave -> Taylor
// (g3dpw2local_real_vec, g3drouts.f:1774-1938) with x and y passes over the
// positive half (mirror pre-add) and the z pass over the stored half, then
// Horner evaluation, two points per thread.
__global__ void __launch_bounds__(512) k_eval3d_taylor_smem(KP k, const EvalTask* __restrict__ tasks) {
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
  const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1], cz = k.centers[3 * T.box + 2];
  for (int i0 = threadIdx.x; i0 < T.n; i0 += 2 * blockDim.x) {
    const int i1 = i0 + blockDim.x;
    const bool two = i1 < T.n;
    const int p0 = T.i0 + i0, p1 = T.i0 + (two ? i1 : i0);
    const double x0 = (pts[3 * p0] - cx) * k.dsq, y0 = (pts[3 * p0 + 1] - cy) * k.dsq, z0 = (pts[3 * p0 + 2] - cz) * k.dsq;
    const double x1 = (pts[3 * p1] - cx) * k.dsq, y1 = (pts[3 * p1 + 1] - cy) * k.dsq, z1 = (pts[3 * p1 + 2] - cz) * k.dsq;
    double rz0 = 0.0, rz1 = 0.0;
    for (int c = Pn - 1; c >= 0; c--) {
      double ry0 = 0.0, ry1 = 0.0;
      for (int b = Pn - 1; b >= 0; b--) {
        const double* row = lo + Pn * (b + Pn * c);
        double rx0 = 0.0, rx1 = 0.0;
        for (int a = Pn - 1; a >= 0; a--) {
          const double cf = row[a];
          rx0 = fma(rx0, x0, cf);
          rx1 = fma(rx1, x1, cf);
        }
        ry0 = fma(ry0, y0, rx0);
        ry1 = fma(ry1, y1, rx1);
      }
      rz0 = fma(rz0, z0, ry0);
      rz1 = fma(rz1, z1, ry1);
    }
    out[(size_t)p0 * k.nd + ind] += rz0;
    if (two) out[(size_t)p1 * k.nd + ind] += rz1;
  }
}

// ------------------------------------------------------------ (a) form, 3D direct
// pw[k3,k2,k1] = sum_i q_i w(k3) e^{-i t x} w(k2) e^{-i t y} w(k1) e^{-i t z}
// (g3dformpwc_vec, g3drouts.f:1950-2038).  One CTA per (leaf, density);
// entries in passes of 4 per thread, sources staged with their factor rows.
__global__ void __launch_bounds__(256) k_form3d_pw(KP k, const FormTask* __restrict__ tasks) {
  const FormTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  const int npw = k.npw, n2 = k.n2;
  extern __shared__ double sm[];
  double2* F1 = reinterpret_cast<double2*>(sm);      // [FORM_CH][npw]
  double2* F2 = F1 + FORM_CH * npw;                    // [FORM_CH][npw]
  double2* F3 = F2 + FORM_CH * npw;                    // [FORM_CH][n2], charge folded in
  const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1], cz = k.centers[3 * T.box + 2];
  double2* out = k.mp + ((size_t)T.slot * k.nd + ind) * k.nexp;
  for (int e0 = 0; e0 < k.nexp; e0 += 4 * 256) {
    double2 acc[4];
    int i3[4], i2[4], i1[4];
#pragma unroll
    for (int s = 0; s < 4; s++) {
      acc[s] = make_double2(0.0, 0.0);
      int e = e0 + threadIdx.x + s * 256;
      if (e >= k.nexp) e = 0;
      i3[s] = e % npw;
      i2[s] = (e / npw) % npw;
      i1[s] = e / (npw * npw);
    }
    for (int c0 = 0; c0 < T.n; c0 += FORM_CH) {
      const int m = min(FORM_CH, T.n - c0);
      __syncthreads();
      if (threadIdx.x < m) {
        const int i = T.s0 + c0 + threadIdx.x;
        const double x = (k.src[3 * i] - cx) * k.dsq, y = (k.src[3 * i + 1] - cy) * k.dsq,
                     z = (k.src[3 * i + 2] - cz) * k.dsq;
        const double q = k.chg[(size_t)i * k.nd + ind];
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
          f1[n2 + mm] = a; f1[n2 - 1 - mm] = make_double2(a.x, -a.y);
          f2[n2 + mm] = b; f2[n2 - 1 - mm] = make_double2(b.x, -b.y);
          f3[n2 - 1 - mm] = make_double2(c.x, -c.y);
          ex = cmul(ex, exx); ey = cmul(ey, eyy); ez = cmul(ez, ezz);
        }
      }
      __syncthreads();
      for (int t = 0; t < m; t++) {
#pragma unroll
        for (int s = 0; s < 4; s++) {
          const double2 yz = cmul(F2[t * npw + i2[s]], F3[t * n2 + i1[s]]);
          acc[s] = cfma(F1[t * npw + i3[s]], yz, acc[s]);
        }
      }
    }
#pragma unroll
    for (int s = 0; s < 4; s++) {
      int e = e0 + threadIdx.x + s * 256;
      if (e < k.nexp) out[e] = acc[s];
    }
  }
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
// split: child = parent * conj(W), W the merge factor of that child
__global__ void k_split(KP k, const ShiftTask* __restrict__ tasks) {
  const ShiftTask S = tasks[blockIdx.x];
  const size_t per = (size_t)k.nd * k.nexp;
  for (size_t e = (size_t)blockIdx.y * blockDim.x + threadIdx.x; e < per; e += (size_t)gridDim.y * blockDim.x) {
    const int ee = (int)(e % k.nexp);
    k.loc[(size_t)S.dst * per + e] = cmulc(k.loc[(size_t)S.src * per + e], k.wms[(size_t)S.table * k.nexp + ee]);
  }
}

// ------------------------------------------------------------ (c) eval, 2D
// One CTA per (leaf, point set, density).  Taylor route: plane wave ->
// Taylor in shared memory (g2drouts.f:1449-1535), then Horner evaluation of
// sum_{k1,k2} L[k2 + P k1] x^k2 y^k1.  PW route: direct plane-wave sum with
// e^{i t x} built by the recurrence of g2dpwevalp_vec.
__global__ void __launch_bounds__(256) k_eval2d(KP k, const EvalTask* __restrict__ tasks) {
  const EvalTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  const int npw = k.npw, n2 = k.n2;
  const double2* L = k.loc + ((size_t)T.slot * k.nd + ind) * k.nexp;
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const double cx = k.centers[2 * T.box], cy = k.centers[2 * T.box + 1];
  extern __shared__ double sm[];
  if (T.route == ROUTE_TAYLOR) {
    const int Pn = T.p + 1;
    double2* lx = reinterpret_cast<double2*>(sm);   // [Pn][npw]
    double* lo = sm + 2 * Pn * npw;                  // [Pn][Pn]
    for (int idx = threadIdx.x; idx < Pn * npw; idx += blockDim.x) {
      const int k2 = idx / npw, j1 = idx - k2 * npw;
      double2 a = make_double2(0.0, 0.0);
      for (int j2 = 0; j2 < n2; j2++) {
        const double h = k.x2l[k2 * npw + j2];
        const double2 v = L[j2 + n2 * j1];
        a.x = fma(h, v.x, a.x);
        a.y = fma(h, v.y, a.y);
      }
      lx[idx] = rot(a, k2);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < Pn * Pn; idx += blockDim.x) {
      const int k1 = idx / Pn, k2 = idx - k1 * Pn;
      const double sg = (k1 & 1) ? -1.0 : 1.0;
      double2 a = make_double2(0.0, 0.0);
      for (int j1 = 0; j1 < n2; j1++) {
        const double h = k.x2l[k1 * npw + j1];
        const double2 u = lx[k2 * npw + j1], v = lx[k2 * npw + j1 + n2];
        a.x = fma(h, fma(sg, v.x, u.x), a.x);
        a.y = fma(h, fma(sg, v.y, u.y), a.y);
      }
      lo[k2 + Pn * k1] = 2.0 * rot(a, k1).x;
    }
    __syncthreads();
    // Horner in x within a row, then in y; two points per thread for two
    // independent FMA chains
    for (int i0 = threadIdx.x; i0 < T.n; i0 += 2 * blockDim.x) {
      const int i1 = i0 + blockDim.x;
      const bool two = i1 < T.n;
      const int p0 = T.i0 + i0, p1 = T.i0 + (two ? i1 : i0);
      const double x0 = (pts[2 * p0] - cx) * k.dsq, y0 = (pts[2 * p0 + 1] - cy) * k.dsq;
      const double x1 = (pts[2 * p1] - cx) * k.dsq, y1 = (pts[2 * p1 + 1] - cy) * k.dsq;
      double r0 = 0.0, r1 = 0.0;
      for (int k1 = Pn - 1; k1 >= 0; k1--) {
        double s0 = 0.0, s1 = 0.0;
        const double* row = lo + Pn * k1;
        for (int k2 = Pn - 1; k2 >= 0; k2--) {
          const double c = row[k2];
          s0 = fma(s0, x0, c);
          s1 = fma(s1, x1, c);
        }
        r0 = fma(r0, y0, s0);
        r1 = fma(r1, y1, s1);
      }
      out[(size_t)p0 * k.nd + ind] += r0;
      if (two) out[(size_t)p1 * k.nd + ind] += r1;
    }
  } else {
    for (int i = threadIdx.x; i < T.n; i += blockDim.x) {
      const int ip = T.i0 + i;
      const double x = (pts[2 * ip] - cx) * k.dsq, y = (pts[2 * ip + 1] - cy) * k.dsq;
      const double2 ex = cexpi(k.t1 * x), ey = cexpi(k.t1 * y);
      const double2 exx = cmul(ex, ex), eyy = cmul(ey, ey);
      double2 z = make_double2(0.0, 0.0), w1 = ex;
      for (int kx = 0; kx < n2; kx++) {
        double2 s = make_double2(0.0, 0.0), w2 = ey;
        for (int ky = 0; ky < n2; ky++) {
          s = cfma(L[kx + n2 * ky], w2, s);
          s = cfmac(L[kx + n2 * (ky + n2)], w2, s);
          w2 = cmul(w2, eyy);
        }
        z = cfma(s, w1, z);
        w1 = cmul(w1, exx);
      }
      out[(size_t)ip * k.nd + ind] += 2.0 * z.x;
    }
  }
}

// ------------------------------------------------------------ (c) eval, 3D
// Taylor route, persistent CTAs: plane wave -> Taylor through the scratch
// slab (x, y passes) and a z pass into shared memory
// (g3dpw2local_real_vec, g3drouts.f:1774-1938), then Horner evaluation.
__global__ void __launch_bounds__(256) k_eval3d_taylor(KP k, const EvalTask* __restrict__ tasks, int ntasks,
                                                       double2* __restrict__ scratch, size_t slab) {
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
    const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1], cz = k.centers[3 * T.box + 2];
    for (int i = threadIdx.x; i < T.n; i += blockDim.x) {
      const int ip = T.i0 + i;
      const double x = (pts[3 * ip] - cx) * k.dsq, y = (pts[3 * ip + 1] - cy) * k.dsq,
                   z = (pts[3 * ip + 2] - cz) * k.dsq;
      double rz = 0.0;
      for (int c = Pn - 1; c >= 0; c--) {
        double ry = 0.0;
        for (int b = Pn - 1; b >= 0; b--) {
          const double* row = lo + Pn * (b + Pn * c);
          double rx = 0.0;
          for (int a = Pn - 1; a >= 0; a--) rx = fma(rx, x, row[a]);
          ry = fma(ry, y, rx);
        }
        rz = fma(rz, z, ry);
      }
      out[(size_t)ip * k.nd + ind] += rz;
    }
    __syncthreads();
  }
}

// PW route (g3dpwevalp_vec, g3drouts.f:2268-2362): one CTA per task.
__global__ void __launch_bounds__(256) k_eval3d_pw(KP k, const EvalTask* __restrict__ tasks) {
  const EvalTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  const int npw = k.npw, n2 = k.n2;
  const double2* L = k.loc + ((size_t)T.slot * k.nd + ind) * k.nexp;
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1], cz = k.centers[3 * T.box + 2];
  for (int i = threadIdx.x; i < T.n; i += blockDim.x) {
    const int ip = T.i0 + i;
    const double x = (pts[3 * ip] - cx) * k.dsq, y = (pts[3 * ip + 1] - cy) * k.dsq,
                 z = (pts[3 * ip + 2] - cz) * k.dsq;
    const double2 ex = cexpi(k.t1 * x), ey = cexpi(k.t1 * y), ez = cexpi(k.t1 * z);
    const double2 exx = cmul(ex, ex), eyy = cmul(ey, ey), ezz = cmul(ez, ez);
    double2 acc = make_double2(0.0, 0.0), w3 = ez;
    for (int mz = 0; mz < n2; mz++) {
      // z index n2-1-mz holds node -(2 mz + 1) t1
      double2 sy = make_double2(0.0, 0.0), w2 = ey;
      for (int my = 0; my < n2; my++) {
        const double2* rp = L + (size_t)npw * ((n2 + my) + (size_t)npw * (n2 - 1 - mz));
        const double2* rm = L + (size_t)npw * ((n2 - 1 - my) + (size_t)npw * (n2 - 1 - mz));
        double2 sp = make_double2(0.0, 0.0), sn = make_double2(0.0, 0.0), w1 = ex;
        for (int mx = 0; mx < n2; mx++) {
          sp = cfma(rp[n2 + mx], w1, sp);
          sp = cfmac(rp[n2 - 1 - mx], w1, sp);
          sn = cfma(rm[n2 + mx], w1, sn);
          sn = cfmac(rm[n2 - 1 - mx], w1, sn);
          w1 = cmul(w1, exx);
        }
        sy = cfma(sp, w2, sy);
        sy = cfmac(sn, w2, sy);
        w2 = cmul(w2, eyy);
      }
      acc = cfmac(sy, w3, acc);
      w3 = cmul(w3, ezz);
    }
    out[(size_t)ip * k.nd + ind] += 2.0 * acc.x;
  }
}

// ------------------------------------------------------------ (d) near field
// One CTA per chunk of <= 128 evaluation points; every source range of the
// chunk is staged through shared memory.  pot += q exp(-r^2/delta) when
// r^2 < dmax.  MIXED computes exp in FP32 on the SFU (ex2.approx) from an
// FP64 argument and accumulates in FP64.
template <int DIM, bool MIXED>
__global__ void __launch_bounds__(128) k_direct(KP k, const DirTask* __restrict__ tasks, int ntask,
                                                const SrcRange* __restrict__ ranges) {
  constexpr int CAP = 256;  // sources staged per warp and batch
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * 4 + warp;
  __shared__ double ssm[4][(DIM + 1) * CAP];
  if (w >= ntask) return;  // whole warp leaves; no block-wide barrier below
  const DirTask T = tasks[w];
  const int ind = blockIdx.y;
  double* sx = ssm[warp];
  double* sy = sx + CAP;
  double* sz = sy + CAP;
  double* sq = sz + (DIM == 3 ? CAP : 0);
  // g lanes per point (g * n <= 32) split the sources of that point
  int g = 1;
  while (g * 2 * T.n <= 32) g *= 2;
  const int tt = lane / g, sub = lane - tt * g;
  const bool act = tt < T.n;
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const int ip = T.i0 + (act ? tt : 0);
  const double tx = pts[DIM * ip], ty = pts[DIM * ip + 1];
  const double tz = DIM == 3 ? pts[DIM * ip + 2] : 0.0;
  const double ninv = -1.0 / k.delta;
  const double nl2 = -1.4426950408889634 / k.delta;
  double acc = 0.0;
  int r = 0, roff = 0;
  while (r < T.cnt) {
    int m = 0;
    __syncwarp();
    while (r < T.cnt && m < CAP) {
      const SrcRange R = ranges[T.off + r];
      const int take = min(CAP - m, R.n - roff);
      for (int t = lane; t < take; t += 32) {
        const int j = R.s0 + roff + t;
        sx[m + t] = k.src[DIM * j];
        sy[m + t] = k.src[DIM * j + 1];
        if (DIM == 3) sz[m + t] = k.src[DIM * j + 2];
        sq[m + t] = k.chg[(size_t)j * k.nd + ind];
      }
      m += take;
      roff += take;
      if (roff == R.n) { r++; roff = 0; }
    }
    __syncwarp();
    if (act) {
#pragma unroll 4
      for (int t = sub; t < m; t += g) {
        const double dx = tx - sx[t], dy = ty - sy[t];
        double rr = fma(dx, dx, dy * dy);
        if (DIM == 3) {
          const double dz = tz - sz[t];
          rr = fma(dz, dz, rr);
        }
        if (rr < k.dmax) {
          if (MIXED) acc = fma((double)ex2_approx((float)(rr * nl2)), sq[t], acc);
          else acc = fma(exp(rr * ninv), sq[t], acc);
        }
      }
    }
  }
  for (int o = 1; o < g; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (act && sub == 0) out[(size_t)ip * k.nd + ind] += acc;
}

// ------------------------------------------------------------ large delta
// local[j + P k (+ P^2 l)] = sum_i q h_j(x) h_k(y) (h_l(z)) with
// h_j(x) = H_j(x) e^{-x^2} / j! (g2dformlc_vec, g2drouts.f:621-681), one
// partial sum per CTA added into the global array.
template <int DIM>
__global__ void __launch_bounds__(256) k_ld_form(KP k, int ns, int p, const double* __restrict__ cen,
                                                 double* __restrict__ local) {
  const int Pn = p + 1;
  const int nent = DIM == 2 ? Pn * Pn : Pn * Pn * Pn;
  extern __shared__ double sm[];
  double* hx = sm;                    // [FORM_CH][Pn]
  double* hy = hx + FORM_CH * Pn;
  double* hz = hy + FORM_CH * Pn;
  const int ind = blockIdx.y;
  const int per = (ns + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per, i1 = min(ns, i0 + per);
  for (int e0 = 0; e0 < nent; e0 += 256 * 4) {
    double acc[4] = {0, 0, 0, 0};
    for (int c0 = i0; c0 < i1; c0 += FORM_CH) {
      const int m = min(FORM_CH, i1 - c0);
      __syncthreads();
      if (threadIdx.x < m) {
        const int i = c0 + threadIdx.x;
        double v[3];
        for (int d = 0; d < DIM; d++) v[d] = (k.src[DIM * i + d] - cen[d]) * k.dsq;
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
      if (e < nent) atomicAdd(local + (size_t)ind * nent + e, acc[s]);
    }
  }
}
template <int DIM>
__global__ void k_ld_eval(KP k, int n, const double* __restrict__ pts, double* __restrict__ out, int p,
                          const double* __restrict__ cen, const double* __restrict__ local) {
  const int Pn = p + 1;
  const int nent = DIM == 2 ? Pn * Pn : Pn * Pn * Pn;
  const int ind = blockIdx.y;
  const double* lo = local + (size_t)ind * nent;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double x = (pts[DIM * i] - cen[0]) * k.dsq, y = (pts[DIM * i + 1] - cen[1]) * k.dsq;
    const double z = DIM == 3 ? (pts[DIM * i + 2] - cen[2]) * k.dsq : 0.0;
    double rz = 0.0;
    for (int c = (DIM == 3 ? Pn - 1 : 0); c >= 0; c--) {
      double ry = 0.0;
      for (int b = Pn - 1; b >= 0; b--) {
        const double* row = lo + Pn * (b + Pn * c);
        double rx = 0.0;
        for (int a = Pn - 1; a >= 0; a--) rx = fma(rx, x, row[a]);
        ry = fma(ry, y, rx);
      }
      rz = DIM == 3 ? fma(rz, z, ry) : ry;
    }
    out[(size_t)i * k.nd + ind] = rz;
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
template <typename T>
cudaError_t put(char*& cur, T*& dst, const std::vector<T>& v, cudaStream_t s) {
  dst = reinterpret_cast<T*>(cur);
  size_t b = (v.size() * sizeof(T) + 255) & ~size_t(255);
  cur += b;
  if (v.empty()) return cudaSuccess;
  return cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}
template <typename T>
size_t bytes_of(const std::vector<T>& v) {
  return (v.size() * sizeof(T) + 255) & ~size_t(255);
}
size_t al(size_t b) { return (b + 255) & ~size_t(255); }


}  // namespace

#define CK(x)                               \
  do {                                      \
    cudaError_t e_ = (x);                   \
    if (e_ != cudaSuccess) return e_;       \
  } while (0)

cudaError_t device_plan_create(const HostPlan& H, DevicePlan& D) {
  D = DevicePlan();
  D.P = H.P;
  const Params& P = H.P;
  D.nboxes = H.tree.nboxes;
  D.nch = 1 << P.dim;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&D.sm_count, cudaDevAttrMultiProcessorCount, dev));
  // order form and eval tasks by route so each kernel gets a contiguous range
  std::vector<FormTask> form = H.form;
  std::stable_sort(form.begin(), form.end(), [](const FormTask& a, const FormTask& b) {
    return a.route != b.route ? a.route < b.route : a.p < b.p;
  });
  D.nform = (int)form.size();
  for (auto& f : form) {
    (f.route == ROUTE_PW ? D.form_pw_n : D.form_hermite_n)++;
    if (f.route == ROUTE_HERMITE) D.form_pmax = std::max(D.form_pmax, f.p);
  }
  std::vector<EvalTask> ev = H.eval;
  std::stable_sort(ev.begin(), ev.end(), [](const EvalTask& a, const EvalTask& b) {
    return a.route != b.route ? a.route < b.route : a.p < b.p;
  });
  D.neval = (int)ev.size();
  for (auto& e : ev) {
    (e.route == ROUTE_PW ? D.eval_pw_n : D.eval_taylor_n)++;
    if (e.route == ROUTE_TAYLOR) D.eval_pmax = std::max(D.eval_pmax, e.p);
  }
  // launch groups of equal order among the Hermite form / Taylor eval tasks
  for (int t = 0; t < D.form_hermite_n;) {
    int u = t;
    while (u < D.form_hermite_n && form[u].p == form[t].p) u++;
    D.form_groups.push_back({form[t].p, t, u});
    t = u;
  }
  for (int t = 0; t < D.eval_taylor_n;) {
    int u = t;
    while (u < D.eval_taylor_n && ev[u].p == ev[t].p) u++;
    D.eval_groups.push_back({ev[t].p, t, u});
    t = u;
  }
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
  D.split_beg = H.split_beg;
  D.split_end = H.split_end;
  D.nm2l = (int)H.m2l.size();
  D.ndir = (int)H.dir.size();
  D.nmp = H.nmp;
  D.nloc = H.nloc;
  D.direct_pairs = H.direct_pairs;
  D.form_sources = H.form_sources;
  D.eval_points = H.eval_points;
  // 3D: shared-memory paths when the largest order fits, else the scratch path
  std::vector<FormChunk> fchunks;
  std::vector<int> fcbeg;
  size_t hbuf_doubles = 0;
  if (P.dim == 3 && !P.all_direct) {
    const size_t lim = 227 * 1024;
    const int n2 = P.npw / 2;
    if (D.form_hermite_n > 0) {
      const size_t Pn = D.form_pmax + 1, P3 = Pn * Pn * Pn;
      size_t szA = std::max(P3, 2 * Pn * P.npw * n2);
      D.form3_shB = (((szA + 1) & ~size_t(1)) + 2 * Pn * Pn * n2) * 8;
      D.form3_sub = (P3 + 3 * 64 * Pn) * 8 <= lim ? 64 : 32;
      D.form3_shA = (P3 + 3 * (size_t)D.form3_sub * Pn) * 8;
      D.form3_smem = D.form3_shB <= lim && D.form3_shA <= lim;
      if (D.form3_smem) {
        long long hoff = 0;
        for (int t = 0; t < D.form_hermite_n; t++) {
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
      }
    }
    if (D.eval_taylor_n > 0) {
      const size_t Pn = D.eval_pmax + 1;
      size_t szA = std::max(2 * Pn * P.npw * n2, Pn * Pn * Pn);
      D.eval3_sh = (((szA + 1) & ~size_t(1)) + 2 * Pn * Pn * n2) * 8;
      D.eval3_smem = D.eval3_sh <= lim;
    }
  }
  // scratch for the 3D separable transforms (fallback path)
  if (P.dim == 3 && !P.all_direct && (!D.form3_smem || !D.eval3_smem)) {
    size_t slab = 0;
    int n2 = P.npw / 2;
    if (!D.form3_smem)
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
  size_t ns = P.ns, nt = P.nt, nd = P.nd, dim = P.dim;
  size_t total = bytes_of(H.box_centers) + bytes_of(H.h2x) + bytes_of(H.x2l) + al(H.wms.size() * 8) +
                 al(H.wsh.size() * 8) + 2 * al(H.tree.isrc.size() * 4) + 2 * al(H.tree.itarg.size() * 4) +
                 al((size_t)(std::max(P.ntermmax, 1) + 2) * 8) + al(32 * 8) +
                 bytes_of(form) + bytes_of(groups) + bytes_of(H.merge) + bytes_of(H.split) +
                 bytes_of(H.m2l) + bytes_of(H.m2l_nbr) + bytes_of(ev) + bytes_of(H.dir) +
                 bytes_of(H.dir_src) + al((size_t)H.nmp * nd * P.nexp * 16) +
                 al((size_t)H.nloc * nd * P.nexp * 16) + al(ns * dim * 8) + al(ns * nd * 8) +
                 al(nt * dim * 8) + al(ns * nd * 8) + al(nt * nd * 8) +
                 al((size_t)D.scratch_ctas * D.scratch_per_cta * 16) + bytes_of(fchunks) +
                 bytes_of(fcbeg) + al(hbuf_doubles * 8) + 4096;
  D.bytes = total;
  CK(cudaMalloc(&D.base, total));
  char* cur = D.base;
  cudaStream_t s = 0;
  CK(put(cur, D.centers, H.box_centers, s));
  CK(put(cur, D.h2x, H.h2x, s));
  CK(put(cur, D.x2l, H.x2l, s));
  {
    std::vector<double2> w(H.wms.size() / 2), v(H.wsh.size() / 2);
    memcpy(w.data(), H.wms.data(), H.wms.size() * 8);
    memcpy(v.data(), H.wsh.data(), H.wsh.size() * 8);
    CK(put(cur, D.wms, w, s));
    CK(put(cur, D.wsh, v, s));
    CK(cudaStreamSynchronize(s));
  }
  CK(put(cur, D.isrc, H.tree.isrc, s));
  CK(put(cur, D.itarg, H.tree.itarg, s));
  {
    std::vector<int> inv(H.tree.isrc.size());
    for (size_t i = 0; i < inv.size(); i++) inv[H.tree.isrc[i]] = (int)i;
    CK(put(cur, D.isrc_inv, inv, s));
    CK(cudaStreamSynchronize(s));
    inv.assign(H.tree.itarg.size(), 0);
    for (size_t i = 0; i < inv.size(); i++) inv[H.tree.itarg[i]] = (int)i;
    CK(put(cur, D.itarg_inv, inv, s));
    std::vector<double> isq(std::max(P.ntermmax, 1) + 2, 0.0);
    for (size_t j = 1; j < isq.size(); j++) isq[j] = 1.0 / std::sqrt((double)j);
    CK(put(cur, D.isq, isq, s));
    std::vector<double> cfac(32);
    cfac[0] = 1.0;
    for (int j = 1; j < 32; j++) cfac[j] = cfac[j - 1] / std::sqrt((double)j);
    CK(put(cur, D.cfac, cfac, s));
    CK(cudaStreamSynchronize(s));
  }
  CK(put(cur, D.form, form, s));
  CK(put(cur, D.mgroups, groups, s));
  CK(put(cur, D.merge, H.merge, s));
  CK(put(cur, D.split, H.split, s));
  CK(put(cur, D.m2l, H.m2l, s));
  CK(put(cur, D.m2l_nbr, H.m2l_nbr, s));
  CK(put(cur, D.eval, ev, s));
  CK(put(cur, D.dir, H.dir, s));
  CK(put(cur, D.dir_src, H.dir_src, s));
  CK(put(cur, D.fchunks, fchunks, s));
  CK(put(cur, D.fcbeg, fcbeg, s));
  D.hbuf = reinterpret_cast<double*>(cur); cur += al(hbuf_doubles * 8);
  D.mp = reinterpret_cast<double2*>(cur); cur += al((size_t)H.nmp * nd * P.nexp * 16);
  D.loc = reinterpret_cast<double2*>(cur); cur += al((size_t)H.nloc * nd * P.nexp * 16);
  D.ssort = reinterpret_cast<double*>(cur); cur += al(ns * dim * 8);
  D.csort = reinterpret_cast<double*>(cur); cur += al(ns * nd * 8);
  D.tsort = reinterpret_cast<double*>(cur); cur += al(nt * dim * 8);
  D.psort = reinterpret_cast<double*>(cur); cur += al(ns * nd * 8);
  D.ptsort = reinterpret_cast<double*>(cur); cur += al(nt * nd * 8);
  D.scratch = reinterpret_cast<double2*>(cur); cur += al((size_t)D.scratch_ctas * D.scratch_per_cta * 16);
  CK(cudaStreamSynchronize(s));
  return cudaSuccess;
}

void device_plan_destroy(DevicePlan& D) {
  if (D.base) cudaFree(D.base);
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
  return k;
}

// node weights for the direct 3D form kernel live in the x2l/h2x neighbourhood:
// ws(k) = h2x[0 * npw + k] (j = 0 row of h2x is ws_k).
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
  return cudaGetLastError();
}

cudaError_t device_plan_execute(DevicePlan& D, const double* chg, double* pot, double* pottarg,
                                int precision, cudaStream_t st, StageTimes* times) {
  const Params& P = D.P;
  KP k = make_kp(D);
  k.ws = D.h2x;  // row j = 0 of h2x holds the weights
  const int nd = P.nd;
  cudaEvent_t ev[9];
  if (times)
    for (int i = 0; i < 9; i++) CK(cudaEventCreate(&ev[i]));
  auto mark = [&](int i) { if (times) cudaEventRecord(ev[i], st); };
  long long launches = 0;
  mark(0);
  // charges into tree order (coordinates were sorted once, at plan set-up)
  const int gb = std::max(1, std::min(8 * D.sm_count, (std::max(P.ns, P.nt) + 255) / 256));
  if (P.ns > 0) {
    k_gather_pts<<<gb, 256, 0, st>>>(nullptr, chg, nullptr, D.csort, D.isrc, P.ns, P.dim, nd, 0);
    launches++;
  }
  if (P.ifpgh > 0 && P.ns > 0) CK(cudaMemsetAsync(D.psort, 0, (size_t)P.ns * nd * 8, st));
  if (P.ifpghtarg > 0 && P.nt > 0) CK(cudaMemsetAsync(D.ptsort, 0, (size_t)P.nt * nd * 8, st));
  mark(1);
  const int n2 = P.npw / 2;
  if (!P.all_direct) {
    // (a) form
    if (P.dim == 2 && D.form_hermite_n > 0) {
      for (const OrderGroup& G : D.form_groups) {
        const int Pn = G.p + 1;
        dim3 g(G.end - G.beg, nd);
        const FormTask* tk = D.form + G.beg;
        if (Pn <= 32) {
          size_t sh = (size_t)Pn * n2 * 16 + (size_t)Pn * P.npw * 8;
#define FORM_MMA(NT)                                                                              \
  do {                                                                                            \
    CK(cudaFuncSetAttribute(k_form2d_mma<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh)); \
    k_form2d_mma<NT><<<g, 128, sh, st>>>(k, tk, D.cfac);                                          \
  } while (0)
          if (Pn <= 8) FORM_MMA(1);
          else if (Pn <= 16) FORM_MMA(2);
          else if (Pn <= 24) FORM_MMA(3);
          else FORM_MMA(4);
#undef FORM_MMA
        } else {
          const int tpd = (Pn + 3) / 4, Pp = 4 * tpd;
          if (tpd * tpd > 256) return cudaErrorNotSupported;
          const int ch = Pp <= 32 ? 128 : 64;
          size_t sh = ((size_t)2 * ch * Pp + 4096 + 2 * (size_t)Pn * n2) * 8;
          CK(cudaFuncSetAttribute(k_form2d, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
          k_form2d<<<g, 256, sh, st>>>(k, tk, D.isq, ch);
        }
        launches++;
      }
    }
    if (P.dim == 3 && D.form_hermite_n > 0 && D.form3_smem) {
      const int Pn = D.form_pmax + 1;
      if (Pn <= 16) {
        CK(cudaFuncSetAttribute(k_form3d_acc<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D.form3_shA));
        k_form3d_acc<16><<<dim3(D.nfchunks, nd), 256, D.form3_shA, st>>>(k, D.form, D.fchunks, D.hbuf, D.isq, D.form3_sub);
      } else {
        CK(cudaFuncSetAttribute(k_form3d_acc<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D.form3_shA));
        k_form3d_acc<32><<<dim3(D.nfchunks, nd), 256, D.form3_shA, st>>>(k, D.form, D.fchunks, D.hbuf, D.isq, D.form3_sub);
      }
      CK(cudaFuncSetAttribute(k_form3d_h2pw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D.form3_shB));
      k_form3d_h2pw<<<dim3(D.form_hermite_n, nd), 512, D.form3_shB, st>>>(k, D.form, D.fcbeg, D.fchunks, D.hbuf);
      launches += 2;
    } else if (P.dim == 3 && D.form_hermite_n > 0) {
      int Pn = D.form_pmax + 1;
      size_t sh = ((size_t)Pn * Pn * Pn + 3 * FORM_CH * Pn) * 8;
      if (Pn > 32 || sh > 227 * 1024) return cudaErrorNotSupported;
      int grid = D.scratch_ctas;
      if (Pn <= 16) {
        CK(cudaFuncSetAttribute(k_form3d_hermite<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
        k_form3d_hermite<16><<<grid, 256, sh, st>>>(k, D.form, D.form_hermite_n, D.scratch, D.scratch_per_cta);
      } else {
        CK(cudaFuncSetAttribute(k_form3d_hermite<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
        k_form3d_hermite<32><<<grid, 256, sh, st>>>(k, D.form, D.form_hermite_n, D.scratch, D.scratch_per_cta);
      }
      launches++;
    }
    if (P.dim == 3 && D.form_pw_n > 0) {
      size_t sh = (size_t)FORM_CH * (2 * P.npw + n2) * 16;
      CK(cudaFuncSetAttribute(k_form3d_pw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
      k_form3d_pw<<<dim3(D.form_pw_n, nd), 256, sh, st>>>(k, D.form + D.form_hermite_n);
      launches++;
    }
    mark(2);
    // (b) merge, bottom-up
    int echunks = (int)std::min<long long>(65535, ((long long)nd * P.nexp + 255) / 256);
    for (int l = P.nlevels - 1; l >= P.nlevstart; l--) {
      int ng = D.merge_end[l] - D.merge_beg[l];
      if (ng <= 0) continue;
      k_merge<<<dim3(ng, echunks), 256, 0, st>>>(k, D.mgroups + D.merge_beg[l], D.merge);
      launches++;
    }
    mark(3);
    if (D.nm2l > 0) {
      k_m2l<<<dim3(D.nm2l, echunks), 256, 0, st>>>(k, D.m2l, D.m2l_nbr);
      launches++;
    }
    mark(4);
    for (int l = P.nlevstart; l <= P.nlevels - 1; l++) {
      int nsp = D.split_end[l] - D.split_beg[l];
      if (nsp <= 0) continue;
      k_split<<<dim3(nsp, echunks), 256, 0, st>>>(k, D.split + D.split_beg[l]);
      launches++;
    }
    mark(5);
    // (c) eval
    if (P.dim == 2 && D.neval > 0) {
      for (const OrderGroup& G : D.eval_groups) {
        const int Pn = G.p + 1;
        dim3 g(G.end - G.beg, nd);
        const EvalTask* tk = D.eval + G.beg;
        if (Pn <= 32) {
#define EVAL_MMA(NT)                                                                              \
  do {                                                                                            \
    size_t sh = ((size_t)((8 * NT * (8 * NT + 1) + 1) & ~1) + 2 * (size_t)Pn * P.npw + 2 * (size_t)P.nexp + (size_t)Pn * P.npw) * 8; \
    CK(cudaFuncSetAttribute(k_eval2d_mma<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh)); \
    k_eval2d_mma<NT><<<g, 128, sh, st>>>(k, tk);                                                  \
  } while (0)
          if (Pn <= 8) EVAL_MMA(1);
          else if (Pn <= 16) EVAL_MMA(2);
          else if (Pn <= 24) EVAL_MMA(3);
          else EVAL_MMA(4);
#undef EVAL_MMA
        } else {
          size_t sh = (2 * (size_t)Pn * P.npw + (size_t)Pn * Pn) * 8;
          CK(cudaFuncSetAttribute(k_eval2d, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
          k_eval2d<<<g, 256, sh, st>>>(k, tk);
        }
        launches++;
      }
      if (D.eval_pw_n > 0) {
        k_eval2d<<<dim3(D.eval_pw_n, nd), 256, 0, st>>>(k, D.eval + D.eval_taylor_n);
        launches++;
      }
    }
    if (P.dim == 3 && D.eval_taylor_n > 0 && D.eval3_smem) {
      CK(cudaFuncSetAttribute(k_eval3d_taylor_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D.eval3_sh));
      k_eval3d_taylor_smem<<<dim3(D.eval_taylor_n, nd), 512, D.eval3_sh, st>>>(k, D.eval);
      launches++;
    } else if (P.dim == 3 && D.eval_taylor_n > 0) {
      k_eval3d_taylor<<<D.scratch_ctas, 256, 0, st>>>(k, D.eval, D.eval_taylor_n, D.scratch, D.scratch_per_cta);
      launches++;
    }
    if (P.dim == 3 && D.eval_pw_n > 0) {
      k_eval3d_pw<<<dim3(D.eval_pw_n, nd), 256, 0, st>>>(k, D.eval + D.eval_taylor_n);
      launches++;
    }
  } else {
    mark(2); mark(3); mark(4); mark(5);
  }
  mark(6);
  // (d) near field
  if (D.ndir > 0) {
    dim3 g((D.ndir + 3) / 4, nd);
    bool mixed = precision == PREC_MIXED;
    if (P.dim == 2) {
      if (mixed) k_direct<2, true><<<g, 128, 0, st>>>(k, D.dir, D.ndir, D.dir_src);
      else k_direct<2, false><<<g, 128, 0, st>>>(k, D.dir, D.ndir, D.dir_src);
    } else {
      if (mixed) k_direct<3, true><<<g, 128, 0, st>>>(k, D.dir, D.ndir, D.dir_src);
      else k_direct<3, false><<<g, 128, 0, st>>>(k, D.dir, D.ndir, D.dir_src);
    }
    launches++;
  }
  mark(7);
  if (P.ifpgh > 0 && P.ns > 0) {
    k_unsort<<<gb, 256, 0, st>>>(D.psort, pot, D.isrc_inv, P.ns, nd);
    launches++;
  }
  if (P.ifpghtarg > 0 && P.nt > 0) {
    k_unsort<<<gb, 256, 0, st>>>(D.ptsort, pottarg, D.itarg_inv, P.nt, nd);
    launches++;
  }
  mark(8);
  D.launches = launches;
  CK(cudaGetLastError());
  if (times) {
    CK(cudaEventSynchronize(ev[8]));
    // stage i spans marks i..i+1; the shift stages merge/m2l/split are 2..5
    float t[8];
    for (int i = 0; i < 8; i++) cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]);
    for (int i = 0; i < 8; i++) times->ms[i] = t[i];
    for (int i = 0; i < 9; i++) cudaEventDestroy(ev[i]);
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

cudaError_t large_delta_execute(const Params& P, const double* src, const double* chg,
                                const double* trg, double* pot, double* pottarg, double* work,
                                cudaStream_t st) {
  KP k;
  memset(&k, 0, sizeof(k));
  k.dim = P.dim; k.nd = P.nd; k.dsq = P.dsq; k.delta = P.delta;
  k.src = src; k.chg = chg;
  int p = P.nlocal0;
  int Pn = p + 1;
  size_t nent = P.dim == 2 ? (size_t)Pn * Pn : (size_t)Pn * Pn * Pn;
  double* cen = work;
  double* local = work + 4;
  CK(cudaMemcpyAsync(cen, P.cen0, 3 * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(local, 0, nent * P.nd * sizeof(double), st));
  size_t sh = 3 * FORM_CH * Pn * 8;
  if (sh > 227 * 1024) return cudaErrorNotSupported;
  if (sh > 48 * 1024) {
    CK(cudaFuncSetAttribute(k_ld_form<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
    CK(cudaFuncSetAttribute(k_ld_form<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
  }
  int blocks = std::max(1, std::min(1024, (P.ns + 255) / 256));
  if (P.ns > 0) {
    if (P.dim == 2) k_ld_form<2><<<dim3(blocks, P.nd), 256, sh, st>>>(k, P.ns, p, cen, local);
    else k_ld_form<3><<<dim3(blocks, P.nd), 256, sh, st>>>(k, P.ns, p, cen, local);
  }
  auto ev = [&](const double* pts, int n, double* out) {
    if (n <= 0) return;
    int b = std::max(1, std::min(4096, (n + 255) / 256));
    if (P.dim == 2) k_ld_eval<2><<<dim3(b, P.nd), 256, 0, st>>>(k, n, pts, out, p, cen, local);
    else k_ld_eval<3><<<dim3(b, P.nd), 256, 0, st>>>(k, n, pts, out, p, cen, local);
  };
  if (P.ifpghtarg == 1) ev(trg, P.nt, pottarg);
  if (P.ifpgh == 1) ev(src, P.ns, pot);
  return cudaGetLastError();
}


// ------------------------------------------------------------ allocation-free large-delta call
// Some callers cannot let this library allocate device memory: codes that
// hand over device arrays from their own pool and run under a fixed memory
// budget, and latency-critical loops that must not pay for cudaMalloc, which
// can synchronise the whole device.  For them the large-delta transform (one
// Taylor local about a given centre, the reference's fgt2d_large_delta /
// fgt3d_large_delta) runs with its only scratch -- the centre and the local
// expansion -- in this fixed device array.  Every device that loads the
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
    CK(cudaFuncSetAttribute(k_ld_form<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sh));
    CK(cudaFuncSetAttribute(k_ld_form<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, sh));
  }
  // large_delta_execute copies the centre into work[0..2] and clears the
  // local expansion in work[4..] before accumulating into it
  return large_delta_execute(P, src, chg, trg, pot, pottarg, work, st);
}

}  // namespace fgtb
