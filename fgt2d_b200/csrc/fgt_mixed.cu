// Mixed-form (eps >= 1e-6) kernels of stages (a) and (c) in 2D: the Hermite
// block of a leaf and the Taylor evaluation at its points in FP32 arithmetic
// with FP64 accumulation across chunks, in place of the FP64 kernels that the
// plain form runs.  Inputs and outputs are the plain form's (FP64 Hermite and
// Taylor blocks, FP64 point outputs), so the shifts, the transforms and the
// near field are unchanged around them.
#include <cuda_runtime.h>

#include "fgt_kcommon.cuh"

namespace fgtb {

namespace {

// ------------------------------------------------------------ (a) form, 2D, FP32
// H[j][k] = sum_i x_i^j (q_i y_i^k) over a leaf's sources (the unnormalised
// powers of g2dformhc_vec, g2drouts.f:100-168, with x, y relative to the leaf
// centre and scaled by 1/sqrt(delta); 1/sqrt(j! k!) is applied by the
// Hermite -> plane-wave tables), orders Pn <= 16.
//
// One CTA per (leaf, density), 128 threads.  The leaf's sources go through
// in chunks of 128: each thread forms the 16 powers x^j and q y^k of one
// source in FP32 (the offsets from the centre are taken in FP64 first) and
// stages them in shared memory; then lane (h, a, b) of warp w accumulates the
// 4 x 4 tile H[4a..4a+3][4b..4b+3] over the 16 sources w*32 + 2m + h of the
// chunk (two float4 broadcast loads per 16 FMAs) and adds the FP32 tile into
// FP64 accumulators after each chunk, so an FP32 sum never runs over more
// than 16 terms.  The 8 partial blocks (warp, half) are added in a fixed
// order at the end: results do not depend on scheduling.
constexpr int F2_SW = 20;  // floats per staged source row: conflict-free float4 stores and loads

__global__ void __launch_bounds__(128) k_form2d_f32(KP k, const FormTask* __restrict__ tasks,
                                                    const long long* __restrict__ hoff,
                                                    double* __restrict__ hbuf) {
  __shared__ __align__(16) float stage[2 * 128 * F2_SW];  // X rows then Y rows; aliased by the reduction
  float* X = stage;
  float* Y = stage + 128 * F2_SW;
  const FormTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y, Pn = T.p + 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int h = lane >> 4, a = (lane >> 2) & 3, b = lane & 3;
  const double cx = k.centers[2 * T.box], cy = k.centers[2 * T.box + 1];
  double acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) acc[r][c] = 0.0;
  for (int base = 0; base < T.n; base += 128) {
    {
      const int i = base + threadIdx.x;
      float xf = 0.f, yf = 0.f, qf = 0.f;
      if (i < T.n) {
        const long long is = (long long)T.s0 + i;
        const double2 pt = reinterpret_cast<const double2*>(k.src)[is];
        xf = (float)((pt.x - cx) * k.dsq);
        yf = (float)((pt.y - cy) * k.dsq);
        qf = (float)k.chg[is * k.nd + ind];
      }
      float xp = i < T.n ? 1.f : 0.f, yp = qf;
      float4* xr = reinterpret_cast<float4*>(X + threadIdx.x * F2_SW);
      float4* yr = reinterpret_cast<float4*>(Y + threadIdx.x * F2_SW);
#pragma unroll
      for (int q4 = 0; q4 < 4; q4++) {
        float4 xv, yv;
        xv.x = xp; yv.x = yp; xp *= xf; yp *= yf;
        xv.y = xp; yv.y = yp; xp *= xf; yp *= yf;
        xv.z = xp; yv.z = yp; xp *= xf; yp *= yf;
        xv.w = xp; yv.w = yp; xp *= xf; yp *= yf;
        xr[q4] = xv;
        yr[q4] = yv;
      }
    }
    __syncthreads();
    float c32[4][4];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int c = 0; c < 4; c++) c32[r][c] = 0.f;
    const int nsrc = min(16, (T.n - base - warp * 32 - h + 1) / 2);  // valid sources of this half-warp
#pragma unroll 4
    for (int m = 0; m < nsrc; m++) {
      const int s = warp * 32 + 2 * m + h;
      const float4 xv = reinterpret_cast<const float4*>(X + s * F2_SW)[a];
      const float4 yv = reinterpret_cast<const float4*>(Y + s * F2_SW)[b];
      const float xs[4] = {xv.x, xv.y, xv.z, xv.w}, ys[4] = {yv.x, yv.y, yv.z, yv.w};
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) c32[r][c] = fmaf(xs[r], ys[c], c32[r][c]);
    }
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[r][c] += (double)c32[r][c];
    __syncthreads();
  }
  double* red = reinterpret_cast<double*>(stage);  // [8][16][16]
  const int part = warp * 2 + h;
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) red[part * 256 + (4 * a + r) * 16 + 4 * b + c] = acc[r][c];
  __syncthreads();
  double* hb = hbuf + hoff[blockIdx.x] + (size_t)ind * Pn * Pn;
  for (int e = threadIdx.x; e < Pn * Pn; e += 128) {
    const int j = e / Pn, kk = e - j * Pn, f = j * 16 + kk;
    double s = 0.0;
#pragma unroll
    for (int p = 0; p < 8; p++) s += red[p * 256 + f];
    hb[e] = s;
  }
}

// ------------------------------------------------------------ (c) eval, 2D Taylor, FP32
// pot += sum_k y^k sum_j L[k][j] x^j (g2dlevalp_vec, g2drouts.f:847-900) for
// a chunk of <= 256 points of one leaf, two points per thread.  The block is
// converted to FP32 once per CTA; each row's polynomial in x runs in FP32
// (Pn FMAs), the outer polynomial in y and the output in FP64.
template <int NP2>
__global__ void __launch_bounds__(128) k_eval2d_horner_f32(KP k, const HornerTask* __restrict__ tasks,
                                                           const double* __restrict__ lo_all) {
  const HornerTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y, Pn = T.p + 1;
  extern __shared__ float2 lf[];  // [Pn][NP2] coefficient pairs (x^(2m), x^(2m+1))
  const double2* src = reinterpret_cast<const double2*>(lo_all + T.off + (size_t)ind * Pn * 2 * NP2);
  for (int e = threadIdx.x; e < Pn * NP2; e += blockDim.x) {
    const double2 v = src[e];
    lf[e] = make_float2((float)v.x, (float)v.y);
  }
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
  const float x0 = (float)((pa.x - cx) * k.dsq), x1 = (float)((pb.x - cx) * k.dsq);
  const double y0 = (pa.y - cy) * k.dsq, y1 = (pb.y - cy) * k.dsq;
  double r0 = 0.0, r1 = 0.0;
  for (int k1 = Pn - 1; k1 >= 0; k1--) {
    const float2* rw = lf + k1 * NP2;
    const float2 ct = rw[NP2 - 1];
    float s0 = fmaf(ct.y, x0, ct.x), s1 = fmaf(ct.y, x1, ct.x);
#pragma unroll
    for (int m = NP2 - 2; m >= 0; m--) {
      const float2 c = rw[m];
      s0 = fmaf(s0, x0, c.y);
      s1 = fmaf(s1, x1, c.y);
      s0 = fmaf(s0, x0, c.x);
      s1 = fmaf(s1, x1, c.x);
    }
    r0 = fma(r0, y0, (double)s0);
    r1 = fma(r1, y1, (double)s1);
  }
  out[((long long)(T.i0 + ta) * nc) * k.nd + ind] += r0;
  if (two) out[((long long)(T.i0 + tb) * nc) * k.nd + ind] += r1;
}

}  // namespace

cudaError_t launch_form2d_f32(const KP& k, const FormTask* tasks, int ntask, int nd,
                              const long long* hoff, double* hbuf, int Pn, cudaStream_t st) {
  if (Pn > 16 || ntask <= 0) return Pn > 16 ? cudaErrorInvalidValue : cudaSuccess;
  k_form2d_f32<<<dim3(ntask, nd), 128, 0, st>>>(k, tasks, hoff, hbuf);
  return cudaGetLastError();
}

cudaError_t launch_eval2d_horner_f32(const KP& k, const HornerTask* tasks, int ntask, int nd, int Pn,
                                     const double* lo, cudaStream_t st) {
  if (ntask <= 0) return cudaSuccess;
  const int np2 = (Pn + 1) / 2;
  const size_t sh = (size_t)Pn * np2 * sizeof(float2);
  const dim3 g(ntask, nd);
  switch (np2) {
#define HF32_CASE(N)                                                   \
  case N:                                                              \
    k_eval2d_horner_f32<N><<<g, 128, sh, st>>>(k, tasks, lo);          \
    break;
    HF32_CASE(1) HF32_CASE(2) HF32_CASE(3) HF32_CASE(4) HF32_CASE(5) HF32_CASE(6) HF32_CASE(7)
    HF32_CASE(8) HF32_CASE(9) HF32_CASE(10) HF32_CASE(11) HF32_CASE(12) HF32_CASE(13) HF32_CASE(14)
    HF32_CASE(15) HF32_CASE(16)
#undef HF32_CASE
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace fgtb
