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
#include <cstring>

#include "fgt_device.hpp"

namespace fgtb {

namespace {

constexpr int FORM_CH = 32;    // sources staged per chunk in the form kernels
constexpr int DIR_T = 128;     // threads (targets) per near-field task

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
__global__ void k_gather(const double* __restrict__ in, double* __restrict__ out,
                         const int* __restrict__ perm, long long n, int w) {
  long long tot = n * w;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot;
       i += (long long)gridDim.x * blockDim.x) {
    long long r = i / w;
    int c = (int)(i - r * w);
    out[i] = in[(long long)perm[r] * w + c];
  }
}
__global__ void k_scatter(const double* __restrict__ in, double* __restrict__ out,
                          const int* __restrict__ perm, long long n, int w) {
  long long tot = n * w;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot;
       i += (long long)gridDim.x * blockDim.x) {
    long long r = i / w;
    int c = (int)(i - r * w);
    out[(long long)perm[r] * w + c] = in[i];
  }
}

// ------------------------------------------------------------ (a) form, 2D
// One CTA per (leaf, density).  H[j + P k] = sum_i q_i x_i^j y_i^k / sqrt(j! k!)
// accumulated in registers (MAXE entries per thread), then the two 1D
// Hermite -> plane-wave passes in shared memory (g2drouts.f:1276-1326).
template <int MAXE>
__global__ void __launch_bounds__(256) k_form2d_hermite(KP k, const FormTask* __restrict__ tasks) {
  const FormTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  const int Pn = T.p + 1, n2 = k.n2, npw = k.npw, nent = Pn * Pn;
  extern __shared__ double sm[];
  double* xs = sm;
  double* ys = xs + FORM_CH * Pn;
  double* H = ys + FORM_CH * Pn;
  double2* px = reinterpret_cast<double2*>(H + ((nent + 1) & ~1));
  const double cx = k.centers[2 * T.box], cy = k.centers[2 * T.box + 1];
  double acc[MAXE];
  int oj[MAXE], ok[MAXE];
#pragma unroll
  for (int s = 0; s < MAXE; s++) {
    int e = threadIdx.x + s * 256;
    acc[s] = 0.0;
    oj[s] = e % Pn;
    ok[s] = e / Pn;
  }
  for (int c0 = 0; c0 < T.n; c0 += FORM_CH) {
    const int m = min(FORM_CH, T.n - c0);
    if (threadIdx.x < m) {
      const int i = T.s0 + c0 + threadIdx.x;
      const double x = (k.src[2 * i] - cx) * k.dsq, y = (k.src[2 * i + 1] - cy) * k.dsq;
      double* xr = xs + threadIdx.x * Pn;
      double* yr = ys + threadIdx.x * Pn;
      double xv = 1.0, yv = k.chg[(size_t)i * k.nd + ind];
      xr[0] = xv;
      yr[0] = yv;
      for (int j = 1; j < Pn; j++) {
        double sj = sqrt((double)j);
        xv = xv * x / sj;
        yv = yv * y / sj;
        xr[j] = xv;
        yr[j] = yv;
      }
    }
    __syncthreads();
    for (int t = 0; t < m; t++) {
      const double* xr = xs + t * Pn;
      const double* yr = ys + t * Pn;
#pragma unroll
      for (int s = 0; s < MAXE; s++)
        if (threadIdx.x + s * 256 < nent) acc[s] = fma(yr[ok[s]], xr[oj[s]], acc[s]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int s = 0; s < MAXE; s++)
    if (threadIdx.x + s * 256 < nent) H[threadIdx.x + s * 256] = acc[s];
  __syncthreads();
  // x pass: px[j2][k2] = sum_j1 h2x(j1,k2) i^j1 H[j1][j2], k2 over the positive half
  for (int idx = threadIdx.x; idx < Pn * n2; idx += 256) {
    const int j2 = idx / n2, k2 = idx - j2 * n2;
    double2 a = make_double2(0.0, 0.0);
    for (int j1 = 0; j1 < Pn; j1++) addrot(a, k.h2x[j1 * npw + k2] * H[j1 + Pn * j2], j1);
    px[idx] = a;
  }
  __syncthreads();
  // y pass over the full node set, written to the leaf's multipole slot
  double2* out = k.mp + ((size_t)T.slot * k.nd + ind) * k.nexp;
  for (int e = threadIdx.x; e < k.nexp; e += 256) {
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
    for (int i = threadIdx.x; i < T.n; i += blockDim.x) {
      const int ip = T.i0 + i;
      const double x = (pts[2 * ip] - cx) * k.dsq, y = (pts[2 * ip + 1] - cy) * k.dsq;
      double r = 0.0;
      for (int k1 = Pn - 1; k1 >= 0; k1--) {
        double s = 0.0;
        const double* row = lo + Pn * k1;
        for (int k2 = Pn - 1; k2 >= 0; k2--) s = fma(s, x, row[k2]);
        r = fma(r, y, s);
      }
      out[(size_t)ip * k.nd + ind] += r;
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
__global__ void __launch_bounds__(DIR_T) k_direct(KP k, const DirTask* __restrict__ tasks,
                                                  const SrcRange* __restrict__ ranges) {
  const DirTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y;
  __shared__ double sx[DIR_T], sy[DIR_T], sz[DIM == 3 ? DIR_T : 1], sq[DIR_T];
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const bool act = threadIdx.x < T.n;
  const int ip = T.i0 + threadIdx.x;
  double tx = 0, ty = 0, tz = 0;
  if (act) {
    tx = pts[DIM * ip];
    ty = pts[DIM * ip + 1];
    if (DIM == 3) tz = pts[DIM * ip + 2];
  }
  const double ninv = -1.0 / k.delta;
  const double nl2 = -1.4426950408889634 / k.delta;
  double acc = 0.0;
  for (int r = 0; r < T.cnt; r++) {
    const SrcRange R = ranges[T.off + r];
    for (int c0 = 0; c0 < R.n; c0 += DIR_T) {
      const int m = min(DIR_T, R.n - c0);
      __syncthreads();
      if (threadIdx.x < m) {
        const int j = R.s0 + c0 + threadIdx.x;
        sx[threadIdx.x] = k.src[DIM * j];
        sy[threadIdx.x] = k.src[DIM * j + 1];
        if (DIM == 3) sz[threadIdx.x] = k.src[DIM * j + 2];
        sq[threadIdx.x] = k.chg[(size_t)j * k.nd + ind];
      }
      __syncthreads();
      if (act) {
        for (int t = 0; t < m; t++) {
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
  }
  if (act) out[(size_t)ip * k.nd + ind] += acc;
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

int form2d_maxe(int pmax) {
  int need = ((pmax + 1) * (pmax + 1) + 255) / 256;
  if (need <= 4) return 4;
  if (need <= 16) return 16;
  if (need <= 40) return 40;
  return -1;
}

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
  std::stable_sort(form.begin(), form.end(), [](const FormTask& a, const FormTask& b) { return a.route < b.route; });
  D.nform = (int)form.size();
  for (auto& f : form) {
    (f.route == ROUTE_PW ? D.form_pw_n : D.form_hermite_n)++;
    if (f.route == ROUTE_HERMITE) D.form_pmax = std::max(D.form_pmax, f.p);
  }
  std::vector<EvalTask> ev = H.eval;
  std::stable_sort(ev.begin(), ev.end(), [](const EvalTask& a, const EvalTask& b) { return a.route < b.route; });
  D.neval = (int)ev.size();
  for (auto& e : ev) {
    (e.route == ROUTE_PW ? D.eval_pw_n : D.eval_taylor_n)++;
    if (e.route == ROUTE_TAYLOR) D.eval_pmax = std::max(D.eval_pmax, e.p);
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
  // scratch for the 3D separable transforms
  if (P.dim == 3 && !P.all_direct) {
    size_t slab = 0;
    int n2 = P.npw / 2;
    for (auto& f : form)
      if (f.route == ROUTE_HERMITE) slab = std::max(slab, (size_t)(f.p + 1) * (f.p + 1) * n2 + (size_t)(f.p + 1) * P.npw * n2);
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
                 al(H.wsh.size() * 8) + al(H.tree.isrc.size() * 4) + al(H.tree.itarg.size() * 4) +
                 bytes_of(form) + bytes_of(groups) + bytes_of(H.merge) + bytes_of(H.split) +
                 bytes_of(H.m2l) + bytes_of(H.m2l_nbr) + bytes_of(ev) + bytes_of(H.dir) +
                 bytes_of(H.dir_src) + al((size_t)H.nmp * nd * P.nexp * 16) +
                 al((size_t)H.nloc * nd * P.nexp * 16) + al(ns * dim * 8) + al(ns * nd * 8) +
                 al(nt * dim * 8) + al(ns * nd * 8) + al(nt * nd * 8) +
                 al((size_t)D.scratch_ctas * D.scratch_per_cta * 16) + 4096;
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
  CK(put(cur, D.form, form, s));
  CK(put(cur, D.mgroups, groups, s));
  CK(put(cur, D.merge, H.merge, s));
  CK(put(cur, D.split, H.split, s));
  CK(put(cur, D.m2l, H.m2l, s));
  CK(put(cur, D.m2l_nbr, H.m2l_nbr, s));
  CK(put(cur, D.eval, ev, s));
  CK(put(cur, D.dir, H.dir, s));
  CK(put(cur, D.dir_src, H.dir_src, s));
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
cudaError_t device_plan_execute(DevicePlan& D, const double* src, const double* chg,
                                const double* trg, double* pot, double* pottarg, int precision,
                                cudaStream_t st, StageTimes* times) {
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
  // gather into tree order
  if (P.ns > 0) {
    k_gather<<<std::min<long long>(4096, ((long long)P.ns * P.dim + 255) / 256), 256, 0, st>>>(src, D.ssort, D.isrc, P.ns, P.dim);
    k_gather<<<std::min<long long>(4096, ((long long)P.ns * nd + 255) / 256), 256, 0, st>>>(chg, D.csort, D.isrc, P.ns, nd);
    launches += 2;
  }
  if (P.nt > 0 && P.ifpghtarg > 0) {
    k_gather<<<std::min<long long>(4096, ((long long)P.nt * P.dim + 255) / 256), 256, 0, st>>>(trg, D.tsort, D.itarg, P.nt, P.dim);
    launches++;
  }
  if (P.ifpgh > 0 && P.ns > 0) CK(cudaMemsetAsync(D.psort, 0, (size_t)P.ns * nd * 8, st));
  if (P.ifpghtarg > 0 && P.nt > 0) CK(cudaMemsetAsync(D.ptsort, 0, (size_t)P.nt * nd * 8, st));
  mark(1);
  const int n2 = P.npw / 2;
  if (!P.all_direct) {
    // (a) form
    if (P.dim == 2 && D.form_hermite_n > 0) {
      int pm = D.form_pmax;
      int Pn = pm + 1;
      size_t sh = (2 * FORM_CH * Pn + ((Pn * Pn + 1) & ~1) + 2 * Pn * n2) * 8;
      int me = form2d_maxe(pm);
      dim3 g(D.form_hermite_n, nd);
      if (me == 4) {
        CK(cudaFuncSetAttribute(k_form2d_hermite<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
        k_form2d_hermite<4><<<g, 256, sh, st>>>(k, D.form);
      } else if (me == 16) {
        CK(cudaFuncSetAttribute(k_form2d_hermite<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
        k_form2d_hermite<16><<<g, 256, sh, st>>>(k, D.form);
      } else if (me == 40) {
        CK(cudaFuncSetAttribute(k_form2d_hermite<40>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
        k_form2d_hermite<40><<<g, 256, sh, st>>>(k, D.form);
      } else {
        return cudaErrorNotSupported;
      }
      launches++;
    }
    if (P.dim == 3 && D.form_hermite_n > 0) {
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
      int Pn = D.eval_pmax + 1;
      size_t sh = (2 * (size_t)Pn * P.npw + (size_t)Pn * Pn) * 8;
      CK(cudaFuncSetAttribute(k_eval2d, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
      k_eval2d<<<dim3(D.neval, nd), 256, sh, st>>>(k, D.eval);
      launches++;
    }
    if (P.dim == 3 && D.eval_taylor_n > 0) {
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
    dim3 g(D.ndir, nd);
    bool mixed = precision == PREC_MIXED;
    if (P.dim == 2) {
      if (mixed) k_direct<2, true><<<g, DIR_T, 0, st>>>(k, D.dir, D.dir_src);
      else k_direct<2, false><<<g, DIR_T, 0, st>>>(k, D.dir, D.dir_src);
    } else {
      if (mixed) k_direct<3, true><<<g, DIR_T, 0, st>>>(k, D.dir, D.dir_src);
      else k_direct<3, false><<<g, DIR_T, 0, st>>>(k, D.dir, D.dir_src);
    }
    launches++;
  }
  mark(7);
  if (P.ifpgh > 0 && P.ns > 0) {
    k_scatter<<<std::min<long long>(4096, ((long long)P.ns * nd + 255) / 256), 256, 0, st>>>(D.psort, pot, D.isrc, P.ns, nd);
    launches++;
  }
  if (P.ifpghtarg > 0 && P.nt > 0) {
    k_scatter<<<std::min<long long>(4096, ((long long)P.nt * nd + 255) / 256), 256, 0, st>>>(D.ptsort, pottarg, D.itarg, P.nt, nd);
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

}  // namespace fgtb
