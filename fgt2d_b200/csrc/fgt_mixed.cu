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
// One CTA per (leaf, density), 128 threads; each warp runs its own pipeline
// over batches of 32 sources (warp w takes sources 32 w + 128 c): every lane
// forms the 16 powers x^j and q y^k of one source in FP32 (the offsets from
// the centre are taken in FP64 first) into the warp's staging rows, then
// lane (h, a, b) accumulates the 4 x 4 tile H[4a..4a+3][4b..4b+3] over the 16
// sources 2m + h of the batch (two float4 broadcast loads per 16 FMAs) and
// adds the FP32 tile into FP64 accumulators after the batch, so an FP32 sum
// never runs over more than 16 terms.  The next batch's coordinates and
// charge are loaded before the current batch is summed.  The 8 partial
// blocks (warp, half) are added in a fixed order at the end: results do not
// depend on scheduling.
constexpr int F2_SW = 20;  // floats per staged y row: conflict-free float4 stores and loads
constexpr int F2_SX = 36;  // floats per staged x row (each power twice): conflict-free float4 access

__global__ void __launch_bounds__(128) k_form2d_f32(KP k, const FormTask* __restrict__ tasks,
                                                    const long long* __restrict__ hoff,
                                                    double* __restrict__ hbuf) {
  __shared__ __align__(16) float stage[4][32 * (F2_SX + F2_SW)];  // per warp: X rows, Y rows; aliased by the reduction
  const FormTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y, Pn = T.p + 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int h = lane >> 4, a = (lane >> 2) & 3, b = lane & 3;
  float* X = stage[warp];              // [32][F2_SX]: x^j twice, (x^0, x^0, x^1, x^1, ...)
  float* Y = stage[warp] + 32 * F2_SX;  // [32][F2_SW]: q y^k
  const double cx = k.centers[2 * T.box], cy = k.centers[2 * T.box + 1];
  double acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) acc[r][c] = 0.0;
  auto fetch = [&](int i, double2& pt, double& q) {
    if (i < T.n) {
      const long long is = (long long)T.s0 + i;
      pt = reinterpret_cast<const double2*>(k.src)[is];
      q = k.chg[is * k.nd + ind];
    } else {
      pt = make_double2(cx, cy);
      q = 0.0;
    }
  };
  double2 pt;
  double q;
  fetch(32 * warp + lane, pt, q);
  for (int base = 32 * warp; base < T.n; base += 128) {
    {
      const float xf = (float)((pt.x - cx) * k.dsq), yf = (float)((pt.y - cy) * k.dsq);
      float xp = base + lane < T.n ? 1.f : 0.f, yp = (float)q;
      float4* xr = reinterpret_cast<float4*>(X + lane * F2_SX);
      float4* yr = reinterpret_cast<float4*>(Y + lane * F2_SW);
#pragma unroll
      for (int q4 = 0; q4 < 4; q4++) {
        float4 xa, xb, yv;
        xa.x = xa.y = xp; yv.x = yp; xp *= xf; yp *= yf;
        xa.z = xa.w = xp; yv.y = yp; xp *= xf; yp *= yf;
        xb.x = xb.y = xp; yv.z = yp; xp *= xf; yp *= yf;
        xb.z = xb.w = xp; yv.w = yp; xp *= xf; yp *= yf;
        xr[2 * q4] = xa;
        xr[2 * q4 + 1] = xb;
        yr[q4] = yv;
      }
    }
    fetch(base + 128 + lane, pt, q);  // the next batch's source, in flight while this one is summed
    __syncwarp();
    // c2[r][h2] = (H[4a+r][4b+2h2], H[4a+r][4b+2h2+1]) on the packed FP32 pipe
    float2 c2[4][2];
#pragma unroll
    for (int r = 0; r < 4; r++) c2[r][0] = c2[r][1] = make_float2(0.f, 0.f);
    const int nsrc = min(16, (T.n - base - h + 1) / 2);  // valid sources of this half-warp
#pragma unroll 4
    for (int m = 0; m < nsrc; m++) {
      const int s = 2 * m + h;
      const float4 xa = reinterpret_cast<const float4*>(X + s * F2_SX)[2 * a];
      const float4 xb = reinterpret_cast<const float4*>(X + s * F2_SX)[2 * a + 1];
      const float4 yv = reinterpret_cast<const float4*>(Y + s * F2_SW)[b];
      const float2 xs[4] = {make_float2(xa.x, xa.y), make_float2(xa.z, xa.w), make_float2(xb.x, xb.y),
                            make_float2(xb.z, xb.w)};
      const float2 y01 = make_float2(yv.x, yv.y), y23 = make_float2(yv.z, yv.w);
#pragma unroll
      for (int r = 0; r < 4; r++) {
        c2[r][0] = ffma2(xs[r], y01, c2[r][0]);
        c2[r][1] = ffma2(xs[r], y23, c2[r][1]);
      }
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
      acc[r][0] += (double)c2[r][0].x;
      acc[r][1] += (double)c2[r][0].y;
      acc[r][2] += (double)c2[r][1].x;
      acc[r][3] += (double)c2[r][1].y;
    }
    __syncwarp();
  }
  __syncthreads();
  double* red = reinterpret_cast<double*>(&stage[0][0]);  // [8][16][16] doubles = 16 KB of the 28 KB
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
// a chunk of <= 256 points of one leaf, two points per thread.  The leaf's
// Taylor block comes from k_pw2taylor2d already in FP32, each coefficient as
// the pair (c, c) (row k: float4 m = (c_2m, c_2m, c_2m+1, c_2m+1)), and is
// copied to shared memory as it is (no conversion).  Each row's polynomial
// in x runs in FP32 (Pn FMAs), the outer polynomial in y and the output in
// FP64.  (Reading the rows straight from global memory, every thread the
// same addresses, made the evaluation 1.7x slower than staging them.)
template <int NP2>
__global__ void __launch_bounds__(128) k_eval2d_horner_f32(KP k, const HornerTask* __restrict__ tasks,
                                                           const double* __restrict__ lo_all) {
  const HornerTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y, Pn = T.p + 1;
  extern __shared__ float4 lf[];  // [Pn][NP2]
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const int nc = T.set ? k.nc_t : k.nc_s;
  const double cx = k.centers[2 * T.box], cy = k.centers[2 * T.box + 1];
  const int ta = threadIdx.x, tb = threadIdx.x + 128;
  const bool one = ta < T.n, two = tb < T.n;
  // the points are loaded before the block, so both loads are in flight together
  const double2 pa = reinterpret_cast<const double2*>(pts)[T.i0 + (one ? ta : 0)];
  const double2 pb = reinterpret_cast<const double2*>(pts)[T.i0 + (two ? tb : 0)];
  const float4* src = reinterpret_cast<const float4*>(lo_all + T.off + (size_t)ind * Pn * 2 * NP2);
  for (int e = threadIdx.x; e < Pn * NP2; e += blockDim.x) lf[e] = src[e];
  __syncthreads();
  if (!one) return;
  const float2 x01 = make_float2((float)((pa.x - cx) * k.dsq), (float)((pb.x - cx) * k.dsq));
  const double y0 = (pa.y - cy) * k.dsq, y1 = (pb.y - cy) * k.dsq;
  double r0 = 0.0, r1 = 0.0;
  for (int k1 = Pn - 1; k1 >= 0; k1--) {
    const float4* rw = lf + k1 * NP2;
    const float4 ct = rw[NP2 - 1];
    float2 s = ffma2(make_float2(ct.z, ct.w), x01, make_float2(ct.x, ct.y));
#pragma unroll
    for (int m = NP2 - 2; m >= 0; m--) {
      const float4 c = rw[m];
      s = ffma2(s, x01, make_float2(c.z, c.w));
      s = ffma2(s, x01, make_float2(c.x, c.y));
    }
    r0 = fma(r0, y0, (double)s.x);
    r1 = fma(r1, y1, (double)s.y);
  }
  out[((long long)(T.i0 + ta) * nc) * k.nd + ind] += r0;
  if (two) out[((long long)(T.i0 + tb) * nc) * k.nd + ind] += r1;
}

// ------------------------------------------------------------ (d) near field, packed FP32
// The mixed near field of potentials (g2d_directcp_vec, g2ddirect.f:32-76;
// g3d_directcp_vec, g3ddirect.f:3-49) on the packed f32x2 pipe.  Same task
// structure and arithmetic as the scalar mixed kernel: coordinates relative
// to the root centre, scaled by sqrt(log2 e / delta) and held as FP32
// (hi, lo) pairs, dx = (t_hi - s_hi) + (t_lo - s_lo), 2^-|dx|^2 by
// ex2.approx, pot += q 2^-|dx|^2 when |dx|^2 < amax (the reference cutoff),
// groups of four sources summed in FP32 and added into FP64.  Each lane
// holds four targets as two packed pairs, so every subtraction, square and
// accumulation serves two targets; a staged source is kept in shared memory
// with each value twice, (s, s), ready as the other operand of a pair.
template <int DIM>
__global__ void __launch_bounds__(128) k_direct_mixed_x2(KP k, const DirTask* __restrict__ tasks, int ntask,
                                                         const SrcRange* __restrict__ ranges, float amax) {
  constexpr int CAP = 128;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * 4 + warp;
  __shared__ float2 fsm[4][(2 * DIM + 1) * CAP];
  if (w >= ntask) return;  // whole warp leaves; no block-wide barrier below
  const DirTask T = tasks[w];
  const int ind = blockIdx.y;
  float2* sh = fsm[warp];          // [DIM][CAP] (hi, hi)
  float2* sl = sh + DIM * CAP;     // [DIM][CAP] (lo, lo)
  float2* sq = sl + DIM * CAP;     // [CAP] (q, q)
  const int ngr = (T.n + 3) / 4;
  int g = 1;
  while (g * 2 * ngr <= 32) g *= 2;
  const int tt = lane / g, sub = lane - tt * g;
  const bool act = tt < ngr;
  double* out = T.set ? k.pottarg : k.pot;
  const int nc = T.set ? k.nc_t : k.nc_s;
  const float* fp = T.set ? k.ftrg : k.fsrc;
  float2 th[2][DIM], tl[2][DIM];  // targets (4 tt, 4 tt + 1) and (4 tt + 2, 4 tt + 3)
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int p = 0; p < 2; p++) {
    const int i0 = min(tt * 4 + 2 * p, T.n - 1), i1 = min(tt * 4 + 2 * p + 1, T.n - 1);
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      th[p][d] = make_float2(fp[(size_t)2 * DIM * (T.i0 + i0) + 2 * d], fp[(size_t)2 * DIM * (T.i0 + i1) + 2 * d]);
      tl[p][d] = make_float2(fp[(size_t)2 * DIM * (T.i0 + i0) + 2 * d + 1],
                             fp[(size_t)2 * DIM * (T.i0 + i1) + 2 * d + 1]);
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
            sh[d * CAP + t] = make_float2(hl.x, hl.x);
            sl[d * CAP + t] = make_float2(hl.y, hl.y);
          }
          const float q = (float)k.chg[(size_t)j * k.nd + ind];
          sq[t] = make_float2(q, q);
        }
      }
      __syncwarp();
      if (act) {
        for (int t = sub; t < m; t += 4 * g) {
          float2 part[2] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const int tu = t + u * g;
            if (tu < m) {
              float2 sH[DIM], sL[DIM];
#pragma unroll
              for (int d = 0; d < DIM; d++) {
                sH[d] = sh[d * CAP + tu];
                sL[d] = sl[d * CAP + tu];
              }
              const float2 q2 = sq[tu];
#pragma unroll
              for (int p = 0; p < 2; p++) {
                float2 dd = fadd2(fsub2(th[p][0], sH[0]), fsub2(tl[p][0], sL[0]));
                float2 a = fmul2(dd, dd);
#pragma unroll
                for (int d = 1; d < DIM; d++) {
                  dd = fadd2(fsub2(th[p][d], sH[d]), fsub2(tl[p][d], sL[d]));
                  a = ffma2(dd, dd, a);
                }
                const float2 e = make_float2(a.x < amax ? ex2_approx(-a.x) : 0.f,
                                             a.y < amax ? ex2_approx(-a.y) : 0.f);
                part[p] = ffma2(e, q2, part[p]);
              }
            }
          }
          acc[0] += (double)part[0].x;
          acc[1] += (double)part[0].y;
          acc[2] += (double)part[1].x;
          acc[3] += (double)part[1].y;
        }
      }
    }
  }
#pragma unroll
  for (int v = 0; v < 4; v++)
    for (int o2 = 1; o2 < g; o2 <<= 1) acc[v] += __shfl_xor_sync(0xffffffffu, acc[v], o2);
  if (act && sub == 0) {
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const int it = tt * 4 + v;
      if (it < T.n) out[((size_t)(T.i0 + it) * nc) * k.nd + ind] += acc[v];
    }
  }
}

}  // namespace

cudaError_t launch_direct_mixed_x2(const KP& k, const DirTask* tasks, int ntask, int nd,
                                   const SrcRange* ranges, float amax, cudaStream_t st) {
  if (ntask <= 0) return cudaSuccess;
  const dim3 g((ntask + 3) / 4, nd);
  if (k.dim == 2) k_direct_mixed_x2<2><<<g, 128, 0, st>>>(k, tasks, ntask, ranges, amax);
  else k_direct_mixed_x2<3><<<g, 128, 0, st>>>(k, tasks, ntask, ranges, amax);
  return cudaGetLastError();
}

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
  const size_t sh = (size_t)Pn * np2 * sizeof(float4);
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
