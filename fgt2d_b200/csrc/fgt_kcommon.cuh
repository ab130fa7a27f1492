// Device-side definitions shared by the CUDA translation units of the
// library: the kernel parameter block, complex helpers, the dipole factor
// rows, output layout and the Horner steps of the Taylor evaluation.
#pragma once
#include <cuda_runtime.h>

#include "fgt_device.hpp"

namespace fgtb {

constexpr int FORM_CH = 32;    // sources staged per chunk in the form kernels
constexpr int LD_PARTS = 256;  // CTAs (partial blocks) of the deterministic large-delta form
constexpr unsigned FULL_MASK = 0xffffffffu;

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
  double* pot;      // sorted outputs of the sources: per point [nc_s][nd]
  double* pottarg;  // sorted outputs of the targets: per point [nc_t][nd]
  int nc_s, nc_t;   // components per density written: 1 (pot), 1 + dim (+ grad), + H (+ Hessian)
  int ifcharge, ifdipole;
  const double* dnrm;  // sorted dipole directions (ns, dim)
  const double* dstr;  // sorted dipole strengths (ns, nd)
  const float* fsrc;   // mixed near field: scaled coordinates as FP32 (hi, lo), [dim][2] per point
  const float* ftrg;
};

// Source weights of density ind at sorted source i: the charge (0 without
// charges) and the dipole vector dipstr * n (zeros without dipoles).
__device__ __forceinline__ double src_charge(const KP& k, long long i, int ind) {
  return k.ifcharge ? k.chg[i * k.nd + ind] : 0.0;
}
template <int DIM>
__device__ __forceinline__ void src_dipole(const KP& k, long long i, int ind, double* v) {
  const double s = k.dstr[i * k.nd + ind];
#pragma unroll
  for (int d = 0; d < DIM; d++) v[d] = s * k.dnrm[i * DIM + d];
}

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
// z * i^j without a branch on j (lanes of a warp hold different j)
__device__ __forceinline__ double2 rot_bf(double2 z, int j) {
  const double a = (j & 1) ? -z.y : z.x, b = (j & 1) ? z.x : z.y;
  return (j & 2) ? make_double2(-a, -b) : make_double2(a, b);
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
// Packed FP32 pairs on the sm_100 f32x2 pipe: one instruction computes both
// lanes of a float2 (d.x = a.x b.x + c.x, d.y = a.y b.y + c.y), each rounded
// as the scalar FP32 operation.
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
      "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// A staged factor row of a dipole source column: a h_j + b dh_j for j < Pn
// at stride `st`, with h_j = v^j / sqrt(j!) and dh_j = sqrt(j) dsq h_(j-1)
// (the source-coordinate derivative, g3dformhd_vec's dxhx).
__device__ __forceinline__ void dip_row(double* row, int st, int Pn, double v, double a, double b,
                                        double dsq, const double* __restrict__ isq) {
  double h = 1.0;
  row[0] = a;
  for (int j = 1; j < Pn; j++) {
    const double dh = j * isq[j] * dsq * h;
    h = h * v * isq[j];
    row[j * st] = fma(a, h, b * dh);
  }
}
// The three columns of a 3D dipole source (g3dformhd_vec / g3dformhcd_vec,
// g3drouts.f:197-405): H += hx hy (q hz + v3 dhz) + hx dhy (v2 hz) + dhx hy (v1 hz).
// Coefficients (a, b) of the factor along d (0 x, 1 y, 2 z) in column c.
__device__ __forceinline__ void dip3_coef(int c, int d, double q, const double* v, double& a,
                                          double& b) {
  if (d == 2) {
    a = c == 0 ? q : c == 1 ? v[1] : v[0];
    b = c == 0 ? v[2] : 0.0;
  } else {
    const bool deriv = (d == 1 && c == 1) || (d == 0 && c == 2);
    a = deriv ? 0.0 : 1.0;
    b = deriv ? 1.0 : 0.0;
  }
}

// ------------------------------------------------------------ outputs: potential, gradient, Hessian
// PGH = 1 potential, 2 + gradient, 3 + Hessian (the reference's ifpgh).  The
// components of one density at one point are, in order, pot, d/dx, d/dy
// (, d/dz), then the Hessian in the reference's order: 2D xx, xy, yy
// (g2dlevalh_vec); 3D xx, yy, zz, xy, xz, yz (g3dlevalh_vec).  A sorted
// output row holds the nc components of all nd densities, [nc][nd].
template <int DIM>
__host__ __device__ constexpr int nhess() { return DIM == 2 ? 3 : 6; }
template <int DIM, int PGH>
__host__ __device__ constexpr int ncomp() { return PGH >= 3 ? 1 + DIM + nhess<DIM>() : PGH == 2 ? 1 + DIM : 1; }

// out row ip += v[0 .. nc) for density ind (nc <= NC: the set's own count)
template <int NC>
__device__ __forceinline__ void add_out(double* __restrict__ out, long long ip, int nd, int nc, int ind,
                                        const double* v) {
#pragma unroll
  for (int c = 0; c < NC; c++)
    if (c < nc) out[(ip * nc + c) * nd + ind] += v[c];
}

// Horner with derivative chains.  One step with coefficient c of a
// polynomial in x carries s, s' and s''/2:
//   s''/2 <- s''/2 x + s',  s' <- s' x + s,  s <- s x + c.
template <int PGH>
__device__ __forceinline__ void hstep(double& s, double& sx, double& sxx, double x, double c) {
  if (PGH >= 3) sxx = fma(sxx, x, sx);
  if (PGH >= 2) sx = fma(sx, x, s);
  s = fma(s, x, c);
}
// Sums over the rows of a 2D block, r = sum_k y^k s_k(x), with the x chains
// of the rows: r, r_x, r_y, r_xx/2, r_xy, r_yy/2.
struct Hor2 {
  double r = 0, rx = 0, ry = 0, rxx = 0, rxy = 0, ryy = 0;
};
template <int PGH>
__device__ __forceinline__ void hrow(Hor2& a, double y, double s, double sx, double sxx) {
  if (PGH >= 3) {
    a.ryy = fma(a.ryy, y, a.ry);
    a.rxy = fma(a.rxy, y, a.rx);
    a.rxx = fma(a.rxx, y, sxx);
  }
  if (PGH >= 2) {
    a.ry = fma(a.ry, y, a.r);
    a.rx = fma(a.rx, y, sx);
  }
  a.r = fma(a.r, y, s);
}
// Sums over the planes of a 3D block with the planes' 2D chains.
struct Hor3 {
  double r = 0, rx = 0, ry = 0, rz = 0, rxx = 0, ryy = 0, rzz = 0, rxy = 0, rxz = 0, ryz = 0;
};
template <int PGH>
__device__ __forceinline__ void hplane(Hor3& a, double z, const Hor2& q) {
  if (PGH >= 3) {
    a.rzz = fma(a.rzz, z, a.rz);
    a.rxz = fma(a.rxz, z, a.rx);
    a.ryz = fma(a.ryz, z, a.ry);
    a.rxx = fma(a.rxx, z, q.rxx);
    a.ryy = fma(a.ryy, z, q.ryy);
    a.rxy = fma(a.rxy, z, q.rxy);
  }
  if (PGH >= 2) {
    a.rz = fma(a.rz, z, a.r);
    a.rx = fma(a.rx, z, q.rx);
    a.ry = fma(a.ry, z, q.ry);
  }
  a.r = fma(a.r, z, q.r);
}
// Components in physical coordinates: the expansion variable is
// (x - c) dsq, so each derivative carries a factor dsq.
template <int PGH>
__device__ __forceinline__ void hemit(const Hor2& a, double dsq, double* v) {
  v[0] = a.r;
  if (PGH >= 2) {
    v[1] = a.rx * dsq;
    v[2] = a.ry * dsq;
  }
  if (PGH >= 3) {
    const double d2 = dsq * dsq;
    v[3] = 2.0 * a.rxx * d2;
    v[4] = a.rxy * d2;
    v[5] = 2.0 * a.ryy * d2;
  }
}
template <int PGH>
__device__ __forceinline__ void hemit(const Hor3& a, double dsq, double* v) {
  v[0] = a.r;
  if (PGH >= 2) {
    v[1] = a.rx * dsq;
    v[2] = a.ry * dsq;
    v[3] = a.rz * dsq;
  }
  if (PGH >= 3) {
    const double d2 = dsq * dsq;
    v[4] = 2.0 * a.rxx * d2;
    v[5] = 2.0 * a.ryy * d2;
    v[6] = 2.0 * a.rzz * d2;
    v[7] = a.rxy * d2;
    v[8] = a.rxz * d2;
    v[9] = a.ryz * d2;
  }
}
// Runtime-order evaluation of a real Taylor block: 2D lo[b ld + a],
// 3D lo[(c Pn + b) ld + a] (a, b, c the powers of x, y, z).
template <int PGH>
__device__ void horner2_rt(const double* lo, int ld, int Pn, double x, double y, double dsq, double* v) {
  Hor2 a;
  for (int b = Pn - 1; b >= 0; b--) {
    const double* row = lo + (size_t)b * ld;
    double s = row[Pn - 1], sx = 0.0, sxx = 0.0;
    for (int m = Pn - 2; m >= 0; m--) hstep<PGH>(s, sx, sxx, x, row[m]);
    hrow<PGH>(a, y, s, sx, sxx);
  }
  hemit<PGH>(a, dsq, v);
}
template <int PGH>
__device__ void horner3_rt(const double* lo, int ld, int Pn, double x, double y, double z, double dsq,
                           double* v) {
  Hor3 a;
  for (int c = Pn - 1; c >= 0; c--) {
    Hor2 q;
    for (int b = Pn - 1; b >= 0; b--) {
      const double* row = lo + ((size_t)c * Pn + b) * ld;
      double s = row[Pn - 1], sx = 0.0, sxx = 0.0;
      for (int m = Pn - 2; m >= 0; m--) hstep<PGH>(s, sx, sxx, x, row[m]);
      hrow<PGH>(q, y, s, sx, sxx);
    }
    hplane<PGH>(a, z, q);
  }
  hemit<PGH>(a, dsq, v);
}

// ------------------------------------------------------------ (d) near field: source ranges
// A near-field task's sources are a list of ranges; a warp reads up to 32
// ranges at a time and maps slots of their concatenation to source indices.
// Raises a kernel's dynamic shared-memory limit to the most the device
// allows beside the kernel's static shared memory; every launch then asks
// for its own size below it.  Setting each launch's own size instead would
// let concurrent plans (a server's worker threads) lower the limit under one
// another's launches, which then fail with an invalid-argument error.  The
// limit only ever rises, so concurrent calls agree.
template <typename K>
cudaError_t smem_limit(K* kernel) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa;
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess) return e;
  const int lim = optin - (int)fa.sharedSizeBytes;
  if (fa.maxDynamicSharedSizeBytes >= lim) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}

struct RangeChunk {
  int nr, excl, s0, tot;  // ranges in the chunk; this lane's exclusive prefix and start; chunk size
};
__device__ __forceinline__ RangeChunk load_range_chunk(const SrcRange* __restrict__ ranges, int off,
                                                       int cnt, int rc, int lane) {
  RangeChunk C;
  C.nr = min(32, cnt - rc);
  int rn = 0;
  C.s0 = 0;
  if (lane < C.nr) {
    const SrcRange R = ranges[off + rc + lane];
    rn = R.n;
    C.s0 = R.s0;
  }
  int inc = rn;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(FULL_MASK, inc, o);
    if (lane >= o) inc += v;
  }
  C.excl = inc - rn;
  C.tot = __shfl_sync(FULL_MASK, inc, 31);
  return C;
}
// source index of slot s (0 <= s < C.tot) of the chunk; all lanes must call
__device__ __forceinline__ int range_slot_source(const RangeChunk& C, int s) {
  int lo = 0, hi = C.nr;
#pragma unroll
  for (int it = 0; it < 5; it++) {
    const int mid = (lo + hi) >> 1;
    if (__shfl_sync(FULL_MASK, C.excl, mid) <= s) lo = mid;
    else hi = mid;
  }
  return __shfl_sync(FULL_MASK, C.s0, lo) + (s - __shfl_sync(FULL_MASK, C.excl, lo));
}

// Mixed-form kernels (fgt_mixed.cu).  2D Hermite block in FP32 for the
// leaves of one order group (Pn <= 16), written as the plain form's FP64
// block at hbuf + hoff[task].
cudaError_t launch_form2d_f32(const KP& k, const FormTask* tasks, int ntask, int nd,
                              const long long* hoff, double* hbuf, int Pn, cudaStream_t st);
// Mixed near field of potentials (charges) on the packed FP32 pipe.
cudaError_t launch_direct_mixed_x2(const KP& k, const DirTask* tasks, int ntask, int nd,
                                   const SrcRange* ranges, float amax, cudaStream_t st);
// 2D Taylor evaluation of potentials in FP32 (Pn <= 32) for the point chunks
// of one order group, added into the sorted outputs; the group's Taylor
// blocks must have been written in FP32 pairs (k_pw2taylor2d with f32).
cudaError_t launch_eval2d_horner_f32(const KP& k, const HornerTask* tasks, int ntask, int nd, int Pn,
                                     const double* lo, cudaStream_t st);

// Tensor-core kernels (fgt_tc.cu).  3D Taylor evaluation of potentials as
// BF16 x 3 tcgen05 products for the point chunks of one order group.
bool eval3d_tc_supported(int Pn);
cudaError_t launch_eval3d_tc(const KP& k, const HornerTask* tasks, int ntask, int nd, int Pn,
                             const double* lo, cudaStream_t st);
// 3D Hermite partial blocks of the source chunks of one order group as BF16 x 3
// tcgen05 products (the plain form's k_form3d_mma output layout).
bool form3d_tc_supported(int Pn);
cudaError_t launch_form3d_tc(const KP& k, const FormTask* tasks, const FormChunk* chunks, int nchunk,
                             int nd, int Pn, double* hbuf, const double* isq, cudaStream_t st);

}  // namespace fgtb
