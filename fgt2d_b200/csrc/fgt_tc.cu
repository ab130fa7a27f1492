// Mixed-form kernels on the fifth-generation tensor cores (tcgen05, sm_100a).
//
// 3D Taylor evaluation (g3dlevalp_vec, g3drouts.f:1045-1107) as a
// compensated BF16 x 3 product:  for the points t of a leaf and its Taylor
// block L[c][b][a] (powers a of x, b of y, c of z),
//     C[t][(c, b)] = sum_a x_t^a L[c][b][a]                 (tensor cores)
//     pot(t)      += sum_c z_t^c sum_b y_t^b C[t][(c, b)]   (epilogue)
// M = 128 points per tile (one TMEM lane each), K = 16 powers of x, N = the
// Pn^2 (c, b) pairs rounded up to 16.  Both operands are split exactly into
// three BF16 pieces (tc::split3) and the six piece products of order <= 2
// accumulate in FP32 in TMEM, which carries ~2^-22 of each product: FP32
// accuracy.  The epilogue runs in FP32 per plane c and adds the planes in FP64.
//
// Also: a self-test of the tensor-core path (one BF16 x 3 GEMM tile against
// an FP64 product on the host) for diagnostics and tests.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "fgt_kcommon.cuh"
#include "fgt_tc.cuh"

#define CK(x)                         \
  do {                                \
    cudaError_t e_ = (x);             \
    if (e_ != cudaSuccess) return e_; \
  } while (0)

namespace fgtb {

namespace {

// device error flag of the tensor-core kernels: set when a wait on an MMA
// completion gives up (the kernel then frees its TMEM and returns)
__device__ int g_tc_error = 0;
constexpr uint32_t kWaitLimit = 1u << 24;  // polls of one mbarrier wait (seconds at most)

template <int PN>
struct Eval3Dims {
  static constexpr int NCOL = PN * PN;
  // the (c, b) rows go through the tensor cores in NPASS passes of NP rows
  // (a multiple of 16, <= 128), so one accumulator of NP <= 128 TMEM columns
  // serves every pass and four CTAs fit the 512 columns of an SM
  static constexpr int NPASS = (NCOL + 127) / 128;
  static constexpr int NP = ((NCOL + NPASS - 1) / NPASS + 15) / 16 * 16;
  static constexpr int N = NP * NPASS;                         // B rows staged (zero past NCOL)
  static constexpr int TCOLS = NP <= 32 ? 32 : NP <= 64 ? 64 : 128;
  static constexpr int A_BYTES = 128 * 32;                     // one piece
  static constexpr int B_BYTES = N * 32;                       // one piece
  static constexpr int SMEM = 3 * A_BYTES + 3 * B_BYTES;
  static constexpr int PER_SM = 512 / TCOLS < 4 ? 512 / TCOLS : 4;  // CTAs holding TMEM at once
};

// One CTA (128 threads) per chunk of <= 256 points of a leaf.  The points'
// coordinates and their current outputs are loaded first (both tiles), so
// those loads are in flight while the Taylor block is split into its BF16
// pieces.  Each tile of 128 points then runs NPASS passes: six MMAs into
// the accumulator, one commit, and the pass's epilogue (TMEM loads issued
// in groups before one wait, the y contraction per plane c in FP32).
template <int PN>
__global__ void __launch_bounds__(128) k_eval3d_tc(KP k, const HornerTask* __restrict__ tasks,
                                                   const double* __restrict__ lo_all) {
  using D = Eval3Dims<PN>;
  static_assert(PN <= 16, "order above the single-K-step tile");
  extern __shared__ __align__(1024) unsigned char smraw[];
  unsigned char* Ab = smraw;                    // 3 pieces x [128 rows][16] bf16
  unsigned char* Bb = smraw + 3 * D::A_BYTES;   // 3 pieces x [N rows][16] bf16
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  const HornerTask T = tasks[blockIdx.x];
  const int ind = blockIdx.y, tid = threadIdx.x, warp = tid >> 5;
  constexpr int E = (PN + 1) & ~1;
  const double* L = lo_all + T.off + (size_t)ind * PN * PN * E;
  const double* pts = T.set ? k.trg : k.src;
  double* out = T.set ? k.pottarg : k.pot;
  const int nc = T.set ? k.nc_t : k.nc_s;
  const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1], cz = k.centers[3 * T.box + 2];
  // this thread's points (tile 0 and tile 1) and their outputs, loaded up front
  double px[2], py[2], pz[2], po[2];
#pragma unroll
  for (int u = 0; u < 2; u++) {
    const int r = u * 128 + tid;
    const long long ip = (long long)T.i0 + (r < T.n ? r : 0);
    px[u] = pts[3 * ip];
    py[u] = pts[3 * ip + 1];
    pz[u] = pts[3 * ip + 2];
    po[u] = r < T.n ? out[(ip * nc) * k.nd + ind] : 0.0;
  }

  if (warp == 0) tc::tmem_alloc(&tslot, D::TCOLS);
  if (tid == 0) tc::mbar_init(&mbar, 1);
  // B operand: row n = c * PN + b, column a (zero for a >= PN and n >= PN^2);
  // each thread takes whole 8-column halves of rows: one 16-byte store per piece
  for (int e = tid; e < D::N * 2; e += 128) {
    const int n = e >> 1, h = e & 1;
    uint32_t w0[4], w1[4], w2[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int a0 = 8 * h + 2 * q, a1 = a0 + 1;
      const float v0 = (n < D::NCOL && a0 < PN) ? (float)L[(size_t)n * E + a0] : 0.f;
      const float v1 = (n < D::NCOL && a1 < PN) ? (float)L[(size_t)n * E + a1] : 0.f;
      uint16_t x0, x1, x2, y0, y1, y2;
      tc::split3(v0, x0, x1, x2);
      tc::split3(v1, y0, y1, y2);
      w0[q] = x0 | (uint32_t)y0 << 16;
      w1[q] = x1 | (uint32_t)y1 << 16;
      w2[q] = x2 | (uint32_t)y2 << 16;
    }
    const uint32_t o = tc::op_off(n, 8 * h);
    *reinterpret_cast<uint4*>(Bb + o) = make_uint4(w0[0], w0[1], w0[2], w0[3]);
    *reinterpret_cast<uint4*>(Bb + D::B_BYTES + o) = make_uint4(w1[0], w1[1], w1[2], w1[3]);
    *reinterpret_cast<uint4*>(Bb + 2 * D::B_BYTES + o) = make_uint4(w2[0], w2[1], w2[2], w2[3]);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tslot;
  const uint32_t aS = tc::smem_u32(Ab), bS = tc::smem_u32(Bb);
  constexpr uint32_t idesc = tc::idesc_bf16(128, D::NP);
  const uint32_t tl = tmem + ((uint32_t)(32 * warp) << 16);  // this warp's TMEM lanes
  bool ok = true;
  uint32_t phase = 0;
  const int ntile = (T.n + 127) / 128;
  for (int tile = 0; tile < ntile && ok; tile++) {
    const int r = tile * 128 + tid;
    const bool valid = r < T.n;
    // (selects, not indexing: the per-tile values stay in registers)
    const double qx = tile ? px[1] : px[0], qy = tile ? py[1] : py[0], qz = tile ? pz[1] : pz[0];
    const double qo = tile ? po[1] : po[0];
    const float x = (float)((qx - cx) * k.dsq), y = (float)((qy - cy) * k.dsq);
    const double z = (qz - cz) * k.dsq;
    // A operand row tid: x^a for a < PN (zero rows for missing points)
    {
      float xp = valid ? 1.f : 0.f;
      uint16_t p0[16], p1[16], p2[16];
#pragma unroll
      for (int a = 0; a < 16; a++) {
        tc::split3(a < PN ? xp : 0.f, p0[a], p1[a], p2[a]);
        xp *= x;
      }
#pragma unroll
      for (int kc = 0; kc < 2; kc++) {
        uint32_t w0[4], w1[4], w2[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int a = 8 * kc + 2 * q;
          w0[q] = p0[a] | (uint32_t)p0[a + 1] << 16;
          w1[q] = p1[a] | (uint32_t)p1[a + 1] << 16;
          w2[q] = p2[a] | (uint32_t)p2[a + 1] << 16;
        }
        const uint32_t o = tc::op_off(tid, 8 * kc);
        *reinterpret_cast<uint4*>(Ab + o) = make_uint4(w0[0], w0[1], w0[2], w0[3]);
        *reinterpret_cast<uint4*>(Ab + D::A_BYTES + o) = make_uint4(w1[0], w1[1], w1[2], w1[3]);
        *reinterpret_cast<uint4*>(Ab + 2 * D::A_BYTES + o) = make_uint4(w2[0], w2[1], w2[2], w2[3]);
      }
    }
    float yp[PN], s[PN];
    {
      float q = 1.f;
#pragma unroll
      for (int b = 0; b < PN; b++) {
        yp[b] = q;
        q *= y;
        s[b] = 0.f;
      }
    }
    tc::fence_async_smem();
#pragma unroll
    for (int pass = 0; pass < D::NPASS; pass++) {
      tc::fence_before_sync();
      __syncthreads();  // A written (first pass) / the previous pass's TMEM reads done
      if (tid == 0) {
        tc::fence_after_sync();
#pragma unroll
        for (int i = 0; i < 6; i++) {
          const tc::SplitPair sp = tc::split_pair(i);
          tc::mma_bf16(tmem, tc::smem_desc(aS + sp.a * D::A_BYTES),
                       tc::smem_desc(bS + sp.b * D::B_BYTES + pass * (D::NP / 8) * tc::kSBO), idesc,
                       i > 0 ? 1u : 0u);
        }
        tc::mma_commit(&mbar);
      }
      __syncwarp();
      const bool timed_out = !tc::mbar_wait(&mbar, phase, kWaitLimit);
      phase ^= 1u;
      if (__syncthreads_or(timed_out)) {
        ok = false;
        if (tid == 0) atomicExch(&g_tc_error, 1);
        tc::mbar_wait(&mbar, phase ^ 1u, kWaitLimit);  // let the MMAs in flight drain before TMEM is freed
        break;
      }
      tc::fence_after_sync();
      // epilogue of the pass: columns n = pass * NP + j of this warp's lanes,
      // two 16-column loads in flight per wait
#pragma unroll
      for (int g4 = 0; g4 < D::NP / 16; g4 += 2) {
        constexpr int NG = D::NP / 16;
        uint32_t v[2][16];
#pragma unroll
        for (int u = 0; u < 2; u++)
          if (g4 + u < NG) tc::tmem_ld16_nowait(tl + 16 * (g4 + u), v[u]);
        tc::tmem_wait_ld();
#pragma unroll
        for (int u = 0; u < 2; u++)
          if (g4 + u < NG) tc::tmem_fix(v[u]);
#pragma unroll
        for (int u = 0; u < 2; u++)
#pragma unroll
          for (int i = 0; i < 16; i++) {
            const int n = pass * D::NP + 16 * (g4 + u) + i;
            if (g4 + u < NG && n < D::NCOL) s[n / PN] = fmaf(__uint_as_float(v[u][i]), yp[n % PN], s[n / PN]);
          }
      }
    }
    if (!ok) break;
    double pot = 0.0;
#pragma unroll
    for (int c = PN - 1; c >= 0; c--) pot = fma(pot, z, (double)s[c]);
    if (valid) out[(((long long)T.i0 + r) * nc) * k.nd + ind] = qo + pot;
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tmem, D::TCOLS);
}

// ---- 3D Hermite block (g3dformhc_vec, g3drouts.f:109-192) as BF16 x 3 products
// H[j][(l, k)] = sum_i hx_j(x_i) hy_k(y_i) q_i hz_l(z_i) over a chunk of a
// leaf's sources, h_j(v) = v^j / sqrt(j!) with v = (x - c) / sqrt(delta), as
// the tensor-core product D[(l, k)][j] = sum_i A[(l, k)][i] B[j][i]:
// M = the Pn^2 (l, k) rows in two 128-row tiles, N = 16 powers of x, K = 16
// sources per step.  Per step the 48 first threads form the sources' three
// power rows (x's go straight into the B pieces, y's and q z's into shared
// memory), then every thread forms its A rows (l, k) as products, splits
// them into three BF16 pieces and stores them; one thread issues the six
// piece products per tile.  The operand buffers alternate between steps so
// the next step's rows are formed while the tensor cores work.  Every four
// steps (64 sources) the FP32 accumulators are read from TMEM and added into
// FP64 registers and the next step starts a fresh sum, so no FP32 sum runs
// over more than 24 tensor-core accumulations.  Output: the chunk's partial
// block out[j + Pn (k + Pn l)] in FP64, the plain form's layout.
template <int PN>
struct Form3Dims {
  static constexpr int P2 = PN * PN;
  static constexpr int MT = P2 > 128 ? 2 : 1;     // 128-row tiles of (l, k)
  static constexpr int NT = 128 * MT;             // threads: one A row each
  static constexpr int A_BYTES = 128 * MT * 32;  // one piece, one buffer
  static constexpr int B_BYTES = 16 * 32;        // one piece, one buffer
  static constexpr int BUF = 3 * A_BYTES + 3 * B_BYTES;
  static constexpr int SMEM = 2 * BUF;
  static constexpr int TCOLS = 32;               // tile t accumulates in columns 16 t .. 16 t + 15
  static constexpr int FLUSH = 4;                // steps between TMEM -> FP64 flushes
  static constexpr int SW = 20;                  // floats per staged power row (conflict-free float4 reads)
};

template <int PN>
__global__ void __launch_bounds__(Form3Dims<PN>::NT) k_form3d_tc(KP k, const FormTask* __restrict__ tasks,
                                                                const FormChunk* __restrict__ chunks,
                                                                double* __restrict__ hbuf,
                                                                const double* __restrict__ isq) {
  using D = Form3Dims<PN>;
  static_assert(PN <= 16, "order above the single-N-tile form");
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ uint64_t mbar[2];
  __shared__ uint32_t tslot;
  __shared__ __align__(16) float Yt[16][D::SW];  // [power][source of the step]
  __shared__ __align__(16) float Zt[16][D::SW];
  const FormChunk C = chunks[blockIdx.x];
  const FormTask T = tasks[C.task];
  const int ind = blockIdx.y, tid = threadIdx.x, warp = tid >> 5;
  const double cx = k.centers[3 * T.box], cy = k.centers[3 * T.box + 1], cz = k.centers[3 * T.box + 2];

  if (warp == 0) tc::tmem_alloc(&tslot, D::TCOLS);
  if (tid == 0) {
    tc::mbar_init(&mbar[0], 1);
    tc::mbar_init(&mbar[1], 1);
  }
  // this thread's A row n = (l, k) (tile n / 128, lane n % 128); rows >= Pn^2
  // stay zero in both buffers
  const int n = tid, l = n / PN, kk = n - l * PN;
  const bool row_ok = n < D::P2;
  if (!row_ok)
    for (int buf = 0; buf < 2; buf++)
      for (int piece = 0; piece < 3; piece++)
        for (int kc = 0; kc < 2; kc++)
          *reinterpret_cast<uint4*>(smraw + buf * D::BUF + piece * D::A_BYTES + tc::op_off(n, 8 * kc)) =
              make_uint4(0u, 0u, 0u, 0u);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tslot;
  double acc[16];
#pragma unroll
  for (int j = 0; j < 16; j++) acc[j] = 0.0;
  constexpr uint32_t idesc = tc::idesc_bf16(128, 16);
  const int nstep = (C.n + 15) / 16;
  bool ok = true;
  // phase-1 inputs of thread (source i, dimension d): its coordinate offset
  // and weight for the current step, loaded one step ahead
  const int pi = tid & 15, pd = tid >> 4;
  auto load_src = [&](int step, float& v, float& w) {
    v = 0.f;
    w = 0.f;
    const int si = step * 16 + pi;
    if (tid < 48 && si < C.n) {
      const long long is = (long long)C.s0 + si;
      v = (float)((k.src[3 * is + pd] - (pd == 0 ? cx : pd == 1 ? cy : cz)) * k.dsq);
      w = pd == 2 ? (float)k.chg[is * k.nd + ind] : 1.f;
    }
  };
  float vnext, wnext;
  load_src(0, vnext, wnext);
  for (int s = 0; s < nstep; s++) {
    const int b = s & 1;
    unsigned char* Ab = smraw + b * D::BUF;
    unsigned char* Bb = Ab + 3 * D::A_BYTES;
    // buffer b was last read by step s - 2
    if (s >= 2) {
      const bool to = !tc::mbar_wait(&mbar[b], ((s - 2) >> 1) & 1, kWaitLimit);
      if (__syncthreads_or(to)) { ok = false; break; }
    }
    // phase 1: the step's sources, one (source, dimension) per thread; the
    // next step's inputs are requested before this step's powers are formed
    if (tid < 48) {
      const int i = pi, d = pd;
      const float v = vnext;
      float w = wnext;
      if (s + 1 < nstep) load_src(s + 1, vnext, wnext);
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const float val = j < PN ? w : 0.f;
        if (d == 0) {
          uint16_t b0, b1, b2;
          tc::split3(val, b0, b1, b2);
          const uint32_t o = tc::op_off(j, i);
          *reinterpret_cast<uint16_t*>(Bb + o) = b0;
          *reinterpret_cast<uint16_t*>(Bb + D::B_BYTES + o) = b1;
          *reinterpret_cast<uint16_t*>(Bb + 2 * D::B_BYTES + o) = b2;
        } else if (d == 1) {
          Yt[j][i] = val;
        } else {
          Zt[j][i] = val;
        }
        if (j + 1 < PN) w = w * v * (float)isq[j + 1];  // isq holds 1/sqrt(j) for j <= the largest order + 1
      }
    }
    __syncthreads();
    // phase 2: this thread's A row (l, k): the 16 sources' products, split
    if (row_ok) {
      const float4* yr = reinterpret_cast<const float4*>(Yt[kk]);
      const float4* zr = reinterpret_cast<const float4*>(Zt[l]);
#pragma unroll
      for (int kc = 0; kc < 2; kc++) {
        const float4 y0 = yr[2 * kc], y1 = yr[2 * kc + 1], z0 = zr[2 * kc], z1 = zr[2 * kc + 1];
        const float v[8] = {y0.x * z0.x, y0.y * z0.y, y0.z * z0.z, y0.w * z0.w,
                            y1.x * z1.x, y1.y * z1.y, y1.z * z1.z, y1.w * z1.w};
        uint32_t w0[4], w1[4], w2[4];
#pragma unroll
        for (int h = 0; h < 4; h++) {
          uint16_t a0, a1, a2, c0, c1, c2;
          tc::split3(v[2 * h], a0, a1, a2);
          tc::split3(v[2 * h + 1], c0, c1, c2);
          w0[h] = a0 | (uint32_t)c0 << 16;
          w1[h] = a1 | (uint32_t)c1 << 16;
          w2[h] = a2 | (uint32_t)c2 << 16;
        }
        const uint32_t o = tc::op_off(n, 8 * kc);
        *reinterpret_cast<uint4*>(Ab + o) = make_uint4(w0[0], w0[1], w0[2], w0[3]);
        *reinterpret_cast<uint4*>(Ab + D::A_BYTES + o) = make_uint4(w1[0], w1[1], w1[2], w1[3]);
        *reinterpret_cast<uint4*>(Ab + 2 * D::A_BYTES + o) = make_uint4(w2[0], w2[1], w2[2], w2[3]);
      }
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t aS = tc::smem_u32(Ab), bS = tc::smem_u32(Bb);
      const bool fresh = (s % D::FLUSH) == 0;
#pragma unroll
      for (int t = 0; t < D::MT; t++)
#pragma unroll
        for (int i = 0; i < 6; i++) {
          const tc::SplitPair sp = tc::split_pair(i);
          // tile t's rows start 128 t rows (16 8-row groups) into each A piece
          tc::mma_bf16(tmem + 16 * t, tc::smem_desc(aS + sp.a * D::A_BYTES + t * 16 * tc::kSBO),
                       tc::smem_desc(bS + sp.b * D::B_BYTES), idesc, (fresh && i == 0) ? 0u : 1u);
        }
      tc::mma_commit(&mbar[b]);
    }
    __syncwarp();
    if ((s % D::FLUSH) == D::FLUSH - 1 || s == nstep - 1) {
      const bool to = !tc::mbar_wait(&mbar[b], (s >> 1) & 1, kWaitLimit);
      if (__syncthreads_or(to)) { ok = false; break; }
      tc::fence_after_sync();
      // warp w reads lanes 32 (w % 4) .. of tile w / 4: this thread's row n
      uint32_t v[16];
      tc::tmem_ld16_nowait(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + 16 * (warp >> 2), v);
      tc::tmem_wait_ld();
      tc::tmem_fix(v);
#pragma unroll
      for (int j = 0; j < 16; j++) acc[j] += (double)__uint_as_float(v[j]);
      tc::fence_before_sync();
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(&g_tc_error, 1);
    // let the MMAs in flight drain before TMEM is freed
    tc::mbar_wait(&mbar[0], 0, kWaitLimit);
    tc::mbar_wait(&mbar[1], 0, kWaitLimit);
  } else if (row_ok) {
    double* out = hbuf + ((size_t)C.hoff * k.nd + (size_t)ind * PN * D::P2);
#pragma unroll
    for (int j = 0; j < PN; j++) out[j + PN * n] = acc[j];
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tmem, D::TCOLS);
}

// ---- self-test: D = A B^T for A (128 x 16), B (N x 16) FP32 values split
// into three BF16 pieces, against an FP64 product on the host
__global__ void __launch_bounds__(128) k_tc_selftest(const float* __restrict__ A, const float* __restrict__ B,
                                                     int N, float* __restrict__ D) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5;
  unsigned char* Ab = smraw;
  unsigned char* Bb = smraw + 3 * 4096;
  const int bbytes = N * 32;
  if (warp == 0) tc::tmem_alloc(&tslot, 256);
  if (tid == 0) tc::mbar_init(&mbar, 1);
  for (int e = tid; e < 128 * 16; e += 128) {
    uint16_t b0, b1, b2;
    tc::split3(A[e], b0, b1, b2);
    const uint32_t o = tc::op_off(e >> 4, e & 15);
    *reinterpret_cast<uint16_t*>(Ab + o) = b0;
    *reinterpret_cast<uint16_t*>(Ab + 4096 + o) = b1;
    *reinterpret_cast<uint16_t*>(Ab + 8192 + o) = b2;
  }
  for (int e = tid; e < N * 16; e += 128) {
    uint16_t b0, b1, b2;
    tc::split3(B[e], b0, b1, b2);
    const uint32_t o = tc::op_off(e >> 4, e & 15);
    *reinterpret_cast<uint16_t*>(Bb + o) = b0;
    *reinterpret_cast<uint16_t*>(Bb + bbytes + o) = b1;
    *reinterpret_cast<uint16_t*>(Bb + 2 * bbytes + o) = b2;
  }
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tslot;
  if (tid == 0) {
    const uint32_t aS = tc::smem_u32(Ab), bS = tc::smem_u32(Bb);
    const uint32_t idesc = tc::idesc_bf16(128, N);
    for (int i = 0; i < 6; i++) {
      const tc::SplitPair sp = tc::split_pair(i);
      tc::mma_bf16(tmem, tc::smem_desc(aS + sp.a * 4096), tc::smem_desc(bS + sp.b * bbytes), idesc,
                   i > 0 ? 1u : 0u);
    }
    tc::mma_commit(&mbar);
  }
  __syncwarp();
  const bool timed_out = !tc::mbar_wait(&mbar, 0, kWaitLimit);
  if (!__syncthreads_or(timed_out)) {
    tc::fence_after_sync();
    for (int ch = 0; ch < N / 16; ch++) {
      float v[16];
      tc::tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + 16 * ch, v);
      for (int i = 0; i < 16; i++) D[(size_t)tid * N + 16 * ch + i] = v[i];
    }
  } else {
    if (tid == 0) atomicExch(&g_tc_error, 1);
    tc::mbar_wait(&mbar, 0, kWaitLimit);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tmem, 256);
}

}  // namespace

bool eval3d_tc_supported(int Pn) { return Pn >= 1 && Pn <= 16; }
bool form3d_tc_supported(int Pn) { return Pn >= 1 && Pn <= 16; }

cudaError_t launch_form3d_tc(const KP& k, const FormTask* tasks, const FormChunk* chunks, int nchunk,
                             int nd, int Pn, double* hbuf, const double* isq, cudaStream_t st) {
  if (nchunk <= 0) return cudaSuccess;
  const dim3 g(nchunk, nd);
  switch (Pn) {
#define F3TC_CASE(P_)                                                                                  \
  case P_: {                                                                                           \
    const int sh = Form3Dims<P_>::SMEM + 1024;                                                         \
    CK(smem_limit(k_form3d_tc<P_>));       \
    k_form3d_tc<P_><<<g, Form3Dims<P_>::NT, sh, st>>>(k, tasks, chunks, hbuf, isq);                    \
    break;                                                                                             \
  }
    F3TC_CASE(1) F3TC_CASE(2) F3TC_CASE(3) F3TC_CASE(4) F3TC_CASE(5) F3TC_CASE(6) F3TC_CASE(7)
    F3TC_CASE(8) F3TC_CASE(9) F3TC_CASE(10) F3TC_CASE(11) F3TC_CASE(12) F3TC_CASE(13) F3TC_CASE(14)
    F3TC_CASE(15) F3TC_CASE(16)
#undef F3TC_CASE
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_eval3d_tc(const KP& k, const HornerTask* tasks, int ntask, int nd, int Pn,
                             const double* lo, cudaStream_t st) {
  if (ntask <= 0) return cudaSuccess;
  const dim3 g(ntask, nd);
  switch (Pn) {
#define EV3TC_CASE(P_)                                                                                   \
  case P_: {                                                                                             \
    using D = Eval3Dims<P_>;                                                                             \
    /* TMEM: PER_SM CTAs hold their columns on one SM at a time; the shared memory request keeps */       \
    /* more CTAs off the SM instead of waiting in tcgen05.alloc */                                        \
    const int sh = std::max(D::SMEM + 1024, (228 * 1024) / (D::PER_SM + 1) + 1024);                      \
    CK(smem_limit(k_eval3d_tc<P_>));         \
    k_eval3d_tc<P_><<<g, 128, sh, st>>>(k, tasks, lo);                                                   \
    break;                                                                                               \
  }
    EV3TC_CASE(1) EV3TC_CASE(2) EV3TC_CASE(3) EV3TC_CASE(4) EV3TC_CASE(5) EV3TC_CASE(6) EV3TC_CASE(7)
    EV3TC_CASE(8) EV3TC_CASE(9) EV3TC_CASE(10) EV3TC_CASE(11) EV3TC_CASE(12) EV3TC_CASE(13)
    EV3TC_CASE(14) EV3TC_CASE(15) EV3TC_CASE(16)
#undef EV3TC_CASE
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t tc_error_flag(int* flag, bool clear) {
  CK(cudaMemcpyFromSymbol(flag, g_tc_error, sizeof(int)));
  if (clear) {
    const int z = 0;
    CK(cudaMemcpyToSymbol(g_tc_error, &z, sizeof(int)));
  }
  return cudaSuccess;
}

cudaError_t tc_selftest(int N, double* max_rel_err) {
  if (N < 16 || N > 256 || N % 16) return cudaErrorInvalidValue;
  std::vector<float> A(128 * 16), B((size_t)N * 16);
  uint32_t s = 12345u;
  auto rnd = [&]() {
    s = s * 1664525u + 1013904223u;
    return (float)((s >> 8) * (1.0 / 16777216.0)) * 2.f - 1.f;
  };
  for (auto& v : A) v = rnd();
  for (auto& v : B) v = rnd();
  float *dA = nullptr, *dB = nullptr, *dD = nullptr;
  CK(cudaMalloc(&dA, A.size() * 4));
  CK(cudaMalloc(&dB, B.size() * 4));
  CK(cudaMalloc(&dD, (size_t)128 * N * 4));
  CK(cudaMemcpy(dA, A.data(), A.size() * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dB, B.data(), B.size() * 4, cudaMemcpyHostToDevice));
  const int sh = 3 * 4096 + 3 * N * 32 + 1024;
  CK(smem_limit(k_tc_selftest));
  k_tc_selftest<<<1, 128, sh>>>(dA, dB, N, dD);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  std::vector<float> D((size_t)128 * N);
  CK(cudaMemcpy(D.data(), dD, D.size() * 4, cudaMemcpyDeviceToHost));
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dD);
  double num = 0, den = 0;
  for (int m = 0; m < 128; m++)
    for (int n = 0; n < N; n++) {
      double ex = 0;
      for (int kk = 0; kk < 16; kk++) ex += (double)A[m * 16 + kk] * (double)B[(size_t)n * 16 + kk];
      const double d = D[(size_t)m * N + n] - ex;
      num = std::max(num, std::fabs(d));
      den = std::max(den, std::fabs(ex));
    }
  *max_rel_err = num / (den > 0 ? den : 1.0);
  int flag = 0;
  CK(tc_error_flag(&flag, true));
  return flag ? cudaErrorTimeout : cudaSuccess;
}

}  // namespace fgtb
