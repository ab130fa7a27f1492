// Host plan construction: tree, lists, expansion lengths, translation tables
// and the flattened task arrays of the four GPU stages.
//
// The set-up follows the driver and the start of the main routine of the
// reference: fgt2d.f:125-400 / fgt2dmain fgt2d.f:695-857 (2D) and
// fgt3d.f:127-414 / fgt3dmain fgt3d.f:690-900 (3D).
#include "fgt_plan.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <thread>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace fgtb {

namespace {
typedef std::complex<double> cplx;
double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

// Translation tables and 1D matrices (pw_translation_matrices,
// merge_split_pw_matrices, g2drh2xmat, g2drx2lmat and 3D twins).
static void build_tables(HostPlan& H) {
  Params& P = H.P;
  const Tree& t = H.tree;
  int D = P.dim, npw = P.npw, n2 = npw / 2, nch = 1 << D;
  double pi = 4.0 * std::atan(1.0);
  // get_pwnodes: 2D +half then -half (g2drouts.f:2205); 3D ascending (g3drouts.f:2669)
  H.ts.assign(npw, 0.0);
  H.ws.assign(npw, 0.0);
  double h = P.pmax / n2, w = h / (2.0 * std::sqrt(pi));
  for (int j = 0; j < npw; j++) {
    double tj = D == 2 ? (j < n2 ? (j + 0.5) * h : -((j - n2) + 0.5) * h) : (j - n2 + 0.5) * h;
    H.ts[j] = tj;
    H.ws[j] = w * std::exp(-tj * tj / 4);
  }
  int tm = P.ntermmax;
  H.h2x.assign((size_t)(tm + 1) * npw, 0.0);
  H.x2l.assign((size_t)(tm + 1) * npw, 0.0);
  {
    std::vector<double> fac(tm + 1), fac2(tm + 1);
    fac[0] = fac2[0] = 1;
    for (int i = 1; i <= tm; i++) {
      fac[i] = fac[i - 1] / std::sqrt((double)i);
      fac2[i] = fac2[i - 1] * i;
    }
    for (int j = 0; j <= tm; j++)
      for (int k = 0; k < npw; k++) {
        H.h2x[(size_t)j * npw + k] = H.ws[k] * __builtin_powi(-H.ts[k], j) * fac[j];
        H.x2l[(size_t)j * npw + k] = __builtin_powi(H.ts[k], j) / fac2[j];
      }
  }
  // 1D factors of the diagonal translation tables; the tables themselves
  // (nexp entries per row) are formed on the device (device_plan_create).
  // Merge factors: child slot j merged into its parent, the parent-child
  // offset at level l being boxsize(l+1)/2; ww(k) = exp(i t xmin2)^(2^(k-1))
  // as in merge_split_pw_matrices (g2drouts.f:2326-2332).
  cplx I(0, 1);
  int nms = std::max(P.nlevels - std::max(P.npwlevel, 0), 1);
  H.nms = nms;
  double xmin2 = t.boxsize[P.nlevels] / std::sqrt(P.delta) / 2;
  H.ww.assign((size_t)npw * (nms + 1) * 2, 0.0);
  for (int j = 0; j < npw; j++) {
    cplx z = std::exp(I * H.ts[j] * xmin2);
    for (int k = 1; k <= nms; k++) {
      H.ww[2 * ((size_t)j * (nms + 1) + k)] = z.real();
      H.ww[2 * ((size_t)j * (nms + 1) + k) + 1] = z.imag();
      z = z * z;
    }
  }
  // mp->loc factors (pw_translation_matrices): exp(i t xmin), xmin = boxsize(cut)
  double xmin = (P.npwlevel >= 0 ? t.boxsize[P.npwlevel] : 0.0) / std::sqrt(P.delta);
  H.w1.assign((size_t)npw * 2, 0.0);
  for (int j = 0; j < npw; j++) {
    cplx v = std::exp(I * H.ts[j] * xmin);
    H.w1[2 * j] = v.real();
    H.w1[2 * j + 1] = v.imag();
  }
  (void)nch;
}

// (d) near field, target-centric: for every leaf, the ifhung source boxes
// whose list1 holds the leaf or one of its ancestors (fgt2d.f:1287-1333);
// the same in both schemes
static void build_near_tasks(HostPlan& H) {
  const Params& P = H.P;
  const Tree& t = H.tree;
  const Lists& L = H.lists;
  const int nb = t.nboxes, npl = P.npwlevel;
  H.dir.clear();
  H.dir_src.clear();
  double tn[6];
  tn[0] = now();
  // box A -> source boxes S with A in list1(S), as CSR in the order of S
  // (a transpose of the list1 CSR: the S range is cut into one chunk per
  // thread, each thread counts and then places its entries through its own
  // cursors, laid out chunk after chunk, so every segment lists S in
  // increasing box id whatever the thread count)
  std::vector<int> ioff(nb + 1, 0), into;
  int nlevend = npl < P.nlevels ? npl : P.nlevels;
  const int s_hi = nlevend >= 0 ? t.llast[nlevend] : -1;  // levels 0..nlevend are ids 0..s_hi
  {
    int nth = 1;
#ifdef _OPENMP
    if (s_hi > 8192) nth = std::max(1, std::min(omp_get_max_threads(), 8));
#endif
    // per-thread cursors, left uninitialised here (each thread clears its own)
    std::unique_ptr<int[]> cur_buf(new int[(size_t)nth * nb]);
    int* const curp = cur_buf.get();
    auto cur = [&](size_t i) -> int& { return curp[i]; };
    const int chunk = (s_hi + 1 + nth - 1) / nth;
#pragma omp parallel num_threads(nth) if (nth > 1)
    {
#ifdef _OPENMP
      const int th = omp_get_thread_num();
#else
      const int th = 0;
#endif
      int* const c = curp + (size_t)th * nb;
      std::fill(c, c + nb, 0);
      const int s0 = th * chunk, s1 = std::min(s_hi + 1, s0 + chunk);
      for (int s = s0; s < s1; s++)
        if (L.ifhung[s])
          for (int k = L.l1off[s]; k < L.l1off[s + 1]; k++) c[L.l1[k]]++;
#pragma omp barrier
#pragma omp for schedule(static)
      for (int a = 0; a < nb; a++) {
        int n = 0;
        for (int q = 0; q < nth; q++) n += cur((size_t)q * nb + a);
        ioff[a + 1] = n;
      }
#pragma omp single
      {
        for (int a = 0; a < nb; a++) ioff[a + 1] += ioff[a];
        into.assign(ioff[nb], 0);
      }
#pragma omp for schedule(static)
      for (int a = 0; a < nb; a++) {
        int pos = ioff[a];
        for (int q = 0; q < nth; q++) {
          const int n = cur((size_t)q * nb + a);
          cur((size_t)q * nb + a) = pos;
          pos += n;
        }
      }
      for (int s = s0; s < s1; s++)
        if (L.ifhung[s])
          for (int k = L.l1off[s]; k < L.l1off[s + 1]; k++) into[c[L.l1[k]]++] = s;
    }
  }
  // per leaf: its source ranges (ancestors' segments, leaf first) once per
  // evaluated point set, and its tasks of <= CH points; counted per leaf,
  // placed by prefix sums in box order, filled in parallel
  const int CH = 32;  // one warp per task
  const bool sets[2] = {P.ifpgh >= 1, P.ifpghtarg >= 1};
  // ranges and sources summed down the ancestor chains, level by level
  tn[1] = now();
  std::vector<long long> cum_ns(nb, 0);
  std::vector<int> cum_r(nb, 0);
  for (int l = 0; l <= P.nlevels; l++) {
#pragma omp parallel for schedule(static) if (t.llast[l] - t.lfirst[l] > 4096)
    for (int b = t.lfirst[l]; b <= t.llast[l]; b++) {
      int r = ioff[b + 1] - ioff[b];
      long long ns_ = 0;
      for (int k = ioff[b]; k < ioff[b + 1]; k++) ns_ += t.ns(into[k]);
      const int a = t.parent[b];
      cum_r[b] = r + (a >= 0 ? cum_r[a] : 0);
      cum_ns[b] = ns_ + (a >= 0 ? cum_ns[a] : 0);
    }
  }
  tn[2] = now();
  std::vector<int> nr(nb, 0);
  std::vector<long long> roff(nb + 1, 0), toff(nb + 1, 0);
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; b++) {
    if (t.nchild[b] != 0 || cum_r[b] == 0) continue;
    const int r = cum_r[b];
    nr[b] = r;
    int nset = 0, nt_ = 0;
    for (int set = 0; set < 2; set++) {
      const int n = set == 0 ? t.ns(b) : t.nt(b);
      if (!sets[set] || n == 0) continue;
      nset++;
      nt_ += (n + CH - 1) / CH;
    }
    roff[b + 1] = (long long)r * nset;
    toff[b + 1] = nt_;
  }
  for (int b = 0; b < nb; b++) {
    roff[b + 1] += roff[b];
    toff[b + 1] += toff[b];
  }
  H.dir_src.resize(roff[nb]);
  H.dir.resize(toff[nb]);
  long long pairs = 0;
  tn[3] = now();
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : pairs)
  for (int b = 0; b < nb; b++) {
    if (nr[b] == 0) continue;
    long long ro = roff[b], to = toff[b];
    for (int set = 0; set < 2; set++) {
      const int n = set == 0 ? t.ns(b) : t.nt(b);
      if (!sets[set] || n == 0) continue;
      const int i0 = set == 0 ? t.s0[b] : t.t0[b];
      const int off = (int)ro;
      for (int a = b; a >= 0; a = t.parent[a])
        for (int k = ioff[a]; k < ioff[a + 1]; k++) H.dir_src[ro++] = {t.s0[into[k]], t.ns(into[k])};
      for (int c = 0; c < n; c += CH) H.dir[to++] = {set, i0 + c, std::min(CH, n - c), off, nr[b]};
      pairs += cum_ns[b] * n;
    }
  }
  H.direct_pairs = pairs;
  if (getenv("FGT_TREE_TIMING"))
    fprintf(stderr, "near-field parts: csr %.4f cum %.4f offsets %.4f fill %.4f\n", tn[1] - tn[0], tn[2] - tn[1],
            tn[3] - tn[2], now() - tn[3]);
}

// Flattens the tree into the stage task arrays.
static void build_tasks(HostPlan& H) {
  double tq[16];
  int nq = 0;
  tq[nq++] = now();
  Params& P = H.P;
  const Tree& t = H.tree;
  int nb = t.nboxes, D = P.dim, nch = t.nch, nco = t.nco;
  int npl = P.npwlevel, nls = P.nlevstart;
  auto relevant = [&](int b) {
    return (P.ifpghtarg > 0 ? t.nt(b) : 0) + (P.ifpgh > 0 ? t.ns(b) : 0);
  };
  // the plane-wave list of a cut-level box (gt2d_computelistpw_slow /
  // gt3d_computelistpw): its colleagues other than itself, in 3D the
  // non-leaf ones, in colleague order
  auto pw_keep = [&](int b, int jb) { return jb != b && (D == 2 || t.nchild[jb] > 0); };
  // iflocal (fgt2d.f:790-814): a cut-level leaf with a non-leaf colleague
  std::vector<uint8_t> ifl;
  if (npl >= 0 && npl <= P.nlevels) {
    const int a = t.lfirst[npl], z = t.llast[npl];
    ifl.assign(z - a + 1, 0);
#pragma omp parallel for schedule(static) if (z - a > 4096)
    for (int b = a; b <= z; b++)
      if (t.nchild[b] == 0)
        for (int i = 0; i < t.ncoll[b]; i++)
          if (t.nchild[t.coll[(size_t)b * nco + i]] > 0) {
            ifl[b - a] = 1;
            break;
          }
  }
  auto iflocal = [&](int b) { return ifl[b - t.lfirst[npl]] != 0; };  // b at the cut level
  H.mp_slot.assign(nb, -1);
  H.loc_slot.assign(nb, -1);
  H.nmp = H.nloc = 0;
  H.form.clear(); H.merge.clear(); H.split.clear(); H.m2l.clear(); H.m2l_nbr.clear();
  H.eval.clear();
  H.merge_beg.assign(P.nlevels + 1, 0);
  H.merge_end.assign(P.nlevels + 1, 0);
  H.split_beg.assign(P.nlevels + 1, 0);
  H.split_end.assign(P.nlevels + 1, 0);
  H.form_sources = H.eval_points = 0;
  if (!P.all_direct) {
    // capacities from the box count (untouched until filled)
    H.form.reserve(nb);
    H.merge.reserve(nb);
    H.split.reserve(nb);
    H.eval.reserve((size_t)nb + (size_t)(P.ns + P.nt) / 2048 + 16);
    for (int l = nls; l <= P.nlevels; l++)
      for (int b = t.lfirst[l]; b <= t.llast[l]; b++) {
        bool leaf = t.nchild[b] == 0;
        if (t.ns(b) > 0 && !(leaf && l == npl)) H.mp_slot[b] = H.nmp++;
        if (relevant(b) > 0 && !(leaf && l == npl && !iflocal(b))) H.loc_slot[b] = H.nloc++;
      }
    // (a) form, levels nlevels .. max(npwlevel+1, 0) (fgt2d.f:871)
    for (int l = P.nlevels; l >= std::max(npl + 1, 0); l--) {
      int p = H.nlocal[l];
      int route = ROUTE_HERMITE;
      if (D == 3) {
        double r1 = (p + 1.0) / P.npw, r3 = r1 * r1 * r1;
        route = r3 >= 3 ? ROUTE_PW : ROUTE_HERMITE;  // fgt3d.f:931-940
      }
      for (int b = t.lfirst[l]; b <= t.llast[l]; b++) {
        if (t.nchild[b] != 0 || t.ns(b) <= 0) continue;
        int r = route;
        if (D == 3 && route == ROUTE_PW && t.ns(b) > 1000000) r = ROUTE_HERMITE;
        // a 3D Hermite block of more than 29^3 coefficients does not fit in
        // shared memory; the exact exponential sum replaces it there
        if (D == 3 && r == ROUTE_HERMITE && p + 1 > 29) r = ROUTE_PW;
        H.form.push_back({b, t.s0[b], t.ns(b), H.mp_slot[b], p, r});
        H.form_sources += t.ns(b);
      }
    }
    // (b) merge, parents at levels nlevels-1 .. nlevstart
    for (int l = P.nlevels - 1; l >= nls; l--) {
      H.merge_beg[l] = (int)H.merge.size();
      for (int b = t.lfirst[l]; b <= t.llast[l]; b++) {
        if (H.mp_slot[b] < 0 || t.nchild[b] == 0) continue;
        for (int j = 0; j < nch; j++) {
          int c = t.ch(b, j);
          if (c >= 0 && H.mp_slot[c] >= 0) H.merge.push_back({H.mp_slot[b], H.mp_slot[c], l * nch + j});
        }
      }
      H.merge_end[l] = (int)H.merge.size();
    }
    tq[nq++] = now();
    // (b) mp -> loc at the cut level
    // in box order, the list's boxes with a multipole in list order; tasks
    // and neighbours counted per box, placed by prefix sums, filled in parallel
    double xmin = npl >= 0 ? t.boxsize[npl] : 1.0;
    {
      const int a = t.lfirst[nls], z = t.llast[nls], nc = z - a + 1;
      std::vector<int> tix(nc + 1, 0), nix(nc + 1, 0);
#pragma omp parallel for schedule(static) if (nc > 4096)
      for (int b = a; b <= z; b++) {
        if (H.loc_slot[b] < 0) continue;
        int n = 0;
        for (int i = 0; i < t.ncoll[b]; i++) {
          const int j = t.coll[(size_t)b * nco + i];
          n += pw_keep(b, j) && H.mp_slot[j] >= 0;
        }
        tix[b - a + 1] = 1;
        nix[b - a + 1] = n;
      }
      for (int i = 0; i < nc; i++) {
        tix[i + 1] += tix[i];
        nix[i + 1] += nix[i];
      }
      H.m2l.resize(tix[nc]);
      H.m2l_nbr.resize(nix[nc]);
#pragma omp parallel for schedule(static) if (nc > 4096)
      for (int b = a; b <= z; b++) {
        if (H.loc_slot[b] < 0) continue;
        int q = nix[b - a];
        M2LTask mt{H.loc_slot[b], H.mp_slot[b], q, 0};
        for (int i = 0; i < t.ncoll[b]; i++) {
          const int j = t.coll[(size_t)b * nco + i];
          if (!pw_keep(b, j) || H.mp_slot[j] < 0) continue;
          int s = 0, mul = 1;
          for (int d = 0; d < D; d++) {
            int o = (int)std::lround((t.c(b, d) - t.c(j, d)) / xmin);
            s += (o + 1) * mul;
            mul *= 3;
          }
          H.m2l_nbr[q++] = {H.mp_slot[j], s};
          mt.cnt++;
        }
        H.m2l[tix[b - a]] = mt;
      }
    }
    tq[nq++] = now();
    // (b) split, parents at levels nlevstart .. nlevels-1
    for (int l = nls; l <= P.nlevels - 1; l++) {
      H.split_beg[l] = (int)H.split.size();
      for (int b = t.lfirst[l]; b <= t.llast[l]; b++) {
        if (H.loc_slot[b] < 0 || t.nchild[b] == 0) continue;
        for (int j = 0; j < nch; j++) {
          int c = t.ch(b, j);
          if (c >= 0 && H.loc_slot[c] >= 0) H.split.push_back({H.loc_slot[c], H.loc_slot[b], l * nch + j});
        }
      }
      H.split_end[l] = (int)H.split.size();
    }
    // (c) evaluation leaves (fgt2d.f:1141-1271 / fgt3d.f:1283-1446)
    for (int l = nls; l <= P.nlevels; l++) {
      int p = H.nlocal[l];
      bool pw;
      if (D == 2) pw = p > 50;
      else {
        double r1 = (p + 1.0) / P.npw, r3 = r1 * r1 * r1;
        pw = r3 >= 3;
      }
      for (int b = t.lfirst[l]; b <= t.llast[l]; b++) {
        if (t.nchild[b] != 0 || H.loc_slot[b] < 0) continue;
        if (l == npl && !iflocal(b)) continue;
        int route = pw ? ROUTE_PW : ROUTE_TAYLOR;
        if (D == 3 && pw && t.ns(b) + t.nt(b) >= 1000000) route = ROUTE_TAYLOR;
        // big leaves are cut into chunks so that no CTA serialises a
        // 10^4-point leaf; each chunk rebuilds the leaf's Taylor expansion
        const int evch = D == 2 ? 2048 : 2048;
        for (int set = 1; set >= 0; set--) {
          if (set == 1 && !(P.ifpghtarg >= 1 && t.nt(b) > 0)) continue;
          if (set == 0 && !(P.ifpgh >= 1 && t.ns(b) > 0)) continue;
          int i0 = set ? t.t0[b] : t.s0[b], n = set ? t.nt(b) : t.ns(b);
          for (int c = 0; c < n; c += evch)
            H.eval.push_back({b, set, i0 + c, std::min(evch, n - c), H.loc_slot[b], p, route});
          H.eval_points += n;
        }
      }
    }
  }
  tq[nq++] = now();
  // flops of the routes taken: Hermite block (2 n P^d) and its separable
  // transform, or the direct exponential sum (8 n nexp); Taylor conversion
  // and evaluation (2 P^d per point) or direct plane-wave evaluation
  {
    const double n2 = P.npw / 2, npw = P.npw, nexp = P.nexp;
    H.form_route_flops = 0;
    for (auto& f : H.form) {
      const double Pn = f.p + 1;
      if (f.route == ROUTE_HERMITE) {
        if (D == 2) H.form_route_flops += 2 * f.n * Pn * Pn + 4 * Pn * Pn * n2 + 4 * Pn * nexp;
        else H.form_route_flops += 2 * f.n * Pn * Pn * Pn + 4 * Pn * Pn * Pn * n2 + 4 * Pn * Pn * npw * n2 + 4 * Pn * nexp;
      } else {
        H.form_route_flops += 8.0 * f.n * nexp;
      }
    }
    H.form_route_flops *= P.nd;
    H.eval_route_flops = 0;
    for (auto& e : H.eval) {
      const double Pn = e.p + 1;
      if (e.route == ROUTE_TAYLOR) {
        if (D == 2) H.eval_route_flops += 4 * Pn * npw * n2 + 4 * Pn * Pn * n2 + 2 * e.n * Pn * Pn;
        else H.eval_route_flops += 4 * Pn * npw * npw * n2 + 4 * Pn * Pn * npw * n2 + 4 * Pn * Pn * Pn * n2 + 2 * e.n * Pn * Pn * Pn;
      } else {
        H.eval_route_flops += 8.0 * e.n * nexp;
      }
    }
    H.eval_route_flops *= P.nd;
  }
  // algorithmic bytes of the shift stages: each distinct expansion read once,
  // each written once, 16 bytes per complex coefficient
  {
    long long per = 16LL * P.nexp * P.nd;
    std::vector<char> seen;
    long long c = 0;
    auto start = [&](int n) {
      seen.assign(n, 0);
      c = 0;
    };
    auto see = [&](int v) {
      if (v >= 0 && !seen[v]) { seen[v] = 1; c++; }
    };
    long long ra, rb;
    start(H.nmp); for (auto& s : H.merge) see(s.src); ra = c;
    start(H.nmp); for (auto& s : H.merge) see(s.dst); rb = c;
    H.shift_bytes[0] = per * (ra + rb);
    start(H.nmp); for (auto& m : H.m2l) see(m.self_mp); for (auto& n : H.m2l_nbr) see(n.mp); ra = c;
    start(H.nloc); for (auto& m : H.m2l) see(m.loc); rb = c;
    H.shift_bytes[1] = per * (ra + rb);
    start(H.nloc); for (auto& s : H.split) see(s.src); ra = c;
    start(H.nloc); for (auto& s : H.split) see(s.dst); rb = c;
    H.shift_bytes[2] = per * (ra + rb);
  }
  tq[nq++] = now();
  if (getenv("FGT_TREE_TIMING")) {
    fprintf(stderr, "far-field tasks:");
    for (int i = 1; i < nq; i++) fprintf(stderr, " %.4f", tq[i] - tq[i - 1]);
    fprintf(stderr, "\n");
  }
  (void)D;
}

// The NUFFT scheme (2d/nufft/src/fgt2d.f:695-1060, 3d/nufft/src/fgt3d.f
// twin): at the cut level (the root level when the cut is above it) a box
// with more than ndiv sources forms its plane-wave expansion from all its
// sources (the exact sum of the type-1 NUFFT, route PW), which is also its
// own local expansion; the boxes with evaluation points add the shifted
// expansions of their colleagues that have children (listpw of the scheme,
// which then hold more than ndiv sources) and evaluate the sum at every
// point of the box (the exact sum of the type-2 NUFFT, route PW) when they
// have such a colleague or an expansion of their own.  No merge, no split;
// the near field is the plane-wave scheme's.
static void build_tasks_nufft(HostPlan& H) {
  Params& P = H.P;
  const Tree& t = H.tree;
  const int nb = t.nboxes, D = P.dim;
  const int ndiv = D == 2 ? 80 : 100;  // fgt2d.f:162, fgt3d.f:165
  const int lc = P.nlevstart;
  H.mp_slot.assign(nb, -1);
  H.loc_slot.assign(nb, -1);
  H.nmp = H.nloc = 0;
  H.form.clear(); H.merge.clear(); H.split.clear(); H.m2l.clear(); H.m2l_nbr.clear();
  H.eval.clear();
  H.merge_beg.assign(P.nlevels + 1, 0);
  H.merge_end.assign(P.nlevels + 1, 0);
  H.split_beg.assign(P.nlevels + 1, 0);
  H.split_end.assign(P.nlevels + 1, 0);
  H.form_sources = H.eval_points = 0;
  H.form_route_flops = H.eval_route_flops = 0;
  H.shift_bytes[0] = H.shift_bytes[1] = H.shift_bytes[2] = 0;
  if (!P.all_direct && lc <= P.nlevels) {
    const int a0 = t.lfirst[lc], a1 = t.llast[lc];
    auto big = [&](int b) { return t.ns(b) > ndiv; };
    auto pw_nbr = [&](int b, int jb) { return jb != b && t.nchild[jb] > 0; };
    auto npts = [&](int b) { return (P.ifpghtarg > 0 ? t.nt(b) : 0) + (P.ifpgh > 0 ? t.ns(b) : 0); };
    for (int b = a0; b <= a1; b++)
      if (big(b)) H.mp_slot[b] = H.nmp++;
    for (int b = a0; b <= a1; b++) {
      if (npts(b) <= 0) continue;
      bool any = big(b);
      for (int i = 0; i < t.ncoll[b] && !any; i++) any = pw_nbr(b, t.coll[(size_t)b * t.nco + i]);
      if (any) H.loc_slot[b] = H.nloc++;
    }
    // form (fgt2d.f:824-900)
    for (int b = a0; b <= a1; b++)
      if (H.mp_slot[b] >= 0) {
        H.form.push_back({b, t.s0[b], t.ns(b), H.mp_slot[b], 0, ROUTE_PW});
        H.form_sources += t.ns(b);
      }
    // mp -> loc (fgt2d.f:918-958): own expansion plus the colleagues'
    const double xmin = t.boxsize[lc];
    for (int b = a0; b <= a1; b++) {
      if (H.loc_slot[b] < 0) continue;
      M2LTask mt{H.loc_slot[b], H.mp_slot[b], (int)H.m2l_nbr.size(), 0};
      for (int i = 0; i < t.ncoll[b]; i++) {
        const int j = t.coll[(size_t)b * t.nco + i];
        if (!pw_nbr(b, j) || H.mp_slot[j] < 0) continue;
        int s = 0, mul = 1;
        for (int d = 0; d < D; d++) {
          const int o = (int)std::lround((t.c(b, d) - t.c(j, d)) / xmin);
          s += (o + 1) * mul;
          mul *= 3;
        }
        H.m2l_nbr.push_back({H.mp_slot[j], s});
        mt.cnt++;
      }
      H.m2l.push_back(mt);
    }
    // evaluation at every point of the box (fgt2d.f:973-1047)
    for (int b = a0; b <= a1; b++) {
      if (H.loc_slot[b] < 0) continue;
      for (int set = 1; set >= 0; set--) {
        if (set == 1 && !(P.ifpghtarg >= 1 && t.nt(b) > 0)) continue;
        if (set == 0 && !(P.ifpgh >= 1 && t.ns(b) > 0)) continue;
        const int i0 = set ? t.t0[b] : t.s0[b], n = set ? t.nt(b) : t.ns(b);
        for (int c = 0; c < n; c += 2048)
          H.eval.push_back({b, set, i0 + c, std::min(2048, n - c), H.loc_slot[b], 0, ROUTE_PW});
        H.eval_points += n;
      }
    }
    H.form_route_flops = 8.0 * (double)H.form_sources * P.nexp * P.nd;
    H.eval_route_flops = 8.0 * (double)H.eval_points * P.nexp * P.nd;
    const long long per = 16LL * P.nexp * P.nd;
    H.shift_bytes[1] = per * ((long long)H.nmp + H.nloc);
  }
}

static void finish_plan(HostPlan& H) {
  Params& P = H.P;
  Tree& t = H.tree;
  double t0 = now();
  t.npwlevel = P.npwlevel;
  if (H.defer_near) H.lists = Lists();  // list1 is built on the device with the near-field tasks
  else build_lists(t, H.lists);
  double t1 = now();
  H.host_lists_s = t1 - t0;
  if (!P.all_direct) build_tables(H);
  if (P.scheme == 1) build_tasks_nufft(H);
  else build_tasks(H);
  const double tn = now();
  if (!H.defer_near) build_near_tasks(H);
  if (getenv("FGT_TREE_TIMING"))
    fprintf(stderr, "near-field tasks: %.4f (dir %zu ranges %zu)\n", now() - tn, H.dir.size(), H.dir_src.size());
  H.box_centers = t.centers;
  H.host_plan_s = now() - t1;
}

int build_host_plan_from_tree(HostPlan& H, const Params& P0, const std::vector<int>& nlocal,
                              double pmax, int npw) {
  H.P = P0;
  Params& P = H.P;
  H.nlocal = nlocal;
  P.pmax = pmax;
  P.npw = npw;
  P.nlevels = H.tree.nlevels;
  P.nlevstart = std::max(P.npwlevel, 0);
  P.all_direct = P.npwlevel >= P.nlevels;
  P.nexp = P.dim == 2 ? npw * npw / 2 : npw * npw * npw / 2;
  P.ntermmax = 0;
  for (int v : nlocal) P.ntermmax = std::max(P.ntermmax, v);
  P.dsq = 1.0 / std::sqrt(P.delta);
  P.dmax = P.dim == 2 ? std::log(1.0 / (P.eps / 90)) * P.delta : std::log(1.0 / P.eps) * P.delta;
  finish_plan(H);
  return 0;
}

bool plan_begin(HostPlan& H, int dim, int nd, double delta, double eps, int ns, int nt, int ifpgh,
                int ifpghtarg, int npwlevel, double bs0, const double* cen0, TreeSetup& ts,
                int ifcharge, int ifdipole) {
  Params& P = H.P;
  P = Params();
  P.scheme = H.scheme;
  P.dim = dim; P.nd = nd; P.delta = delta; P.eps = eps; P.ns = ns; P.nt = nt;
  P.ifpgh = ifpgh; P.ifpghtarg = ifpghtarg;
  P.ifcharge = ifcharge; P.ifdipole = ifdipole;
  P.dsq = 1.0 / std::sqrt(delta);
  P.dmax = dim == 2 ? std::log(1.0 / (eps / 90)) * delta : std::log(1.0 / eps) * delta;
  P.npwlevel = npwlevel;
  for (int d = 0; d < 3; d++) P.cen0[d] = cen0[d];
  if (npwlevel < -2) {  // fgt2d.f:133-150: one Taylor local about the box centre
    P.large_delta = true;
    int nl0 = hlterms(dim, bs0, delta, eps, 0);
    P.nlocal0 = nl0 + std::max(ifpgh, ifpghtarg) - 1;
    return false;
  }
  // fgt2d.f:158-162 / fgt3d.f:161-165 (3D NUFFT scheme: ndiv0 = 20)
  ts.ndiv0 = dim == 2 ? 10 : (P.scheme == 1 ? 20 : 40);
  ts.ndiv = dim == 2 ? 80 : 100;
  const int hcap = dim == 2 ? 18 : 15;
  int nlmax = npwlevel + 4, nls = std::max(npwlevel, 0);
  double bsize = bs0 / std::ldexp(1.0, nls);
  int nl0 = 0;
  for (int i = nls; i <= 100; i++) {  // fgt2d.f:175-186
    nl0 = hlterms(dim, bsize, delta, eps, nl0);
    if (nl0 <= hcap) { nlmax = i; break; }
    bsize /= 2;
  }
  // the NUFFT scheme's tree stops one level below the cut (2d/nufft
  // fgt2d.f:188, 3d/nufft fgt3d.f:192)
  if (P.scheme == 1 && npwlevel >= 0) nlmax = npwlevel + 1;
  P.nlmax = nlmax;
  ts.levcut = npwlevel;
  ts.nlmax = nlmax;
  ts.bs0 = bs0;
  for (int d = 0; d < 3; d++) ts.cen0[d] = cen0[d];
  return true;
}

void plan_end(HostPlan& H, const std::function<void()>& beside) {
  Params& P = H.P;
  const int dim = P.dim;
  Tree& t = H.tree;
  const int nls = std::max(P.npwlevel, 0);
  P.nlevels = t.nlevels;
  P.nlevstart = nls;
  P.all_direct = P.npwlevel >= t.nlevels;
  H.nlocal.assign(t.nlevels + 1, 0);
  // fgt2d.f:339-347: orders raised by the dipole and derivative orders
  int nadd = P.ifdipole + std::max(P.ifpgh, P.ifpghtarg);
  for (int i = nls; i <= t.nlevels; i++) {
    H.nlocal[i] = hlterms(dim, t.boxsize[i], P.delta, P.eps, 0);
    if (P.ifdipole == 1 || P.ifpgh >= 2 || P.ifpghtarg >= 2) H.nlocal[i] += nadd;
  }
  P.ntermmax = 0;
  for (int v : H.nlocal) P.ntermmax = std::max(P.ntermmax, v);
  double pweps = nadd > 2 ? P.eps / 100 : P.eps;
  pwterms(2 * t.bs0 / std::pow(2.0, nls), P.delta, pweps, &P.pmax, &P.npw);
  P.nexp = dim == 2 ? P.npw * P.npw / 2 : P.npw * P.npw * P.npw / 2;
  if (!beside) {
    finish_plan(H);
    return;
  }
  std::thread th(beside);
  try {
    finish_plan(H);
  } catch (...) {
    th.join();
    throw;
  }
  th.join();
}

int build_host_plan(HostPlan& H, int dim, int nd, double delta, double eps, int ns,
                    const double* sources, int nt, const double* targ, int ifpgh, int ifpghtarg,
                    int nthreads, int ifcharge, int ifdipole) {
  double tstart = now();
  int npwlevel;
  double bs0, cen0[3] = {0, 0, 0};
  boxsize0(dim, delta, eps, sources, ns, targ, nt, &npwlevel, &bs0, cen0);
  TreeSetup ts;
  if (!plan_begin(H, dim, nd, delta, eps, ns, nt, ifpgh, ifpghtarg, npwlevel, bs0, cen0, ts, ifcharge,
                  ifdipole)) {
    H.host_tree_s = now() - tstart;
    return 0;
  }
  build_tree(H.tree, dim, sources, ns, targ, nt, ts.ndiv, ts.ndiv0, ts.levcut, ts.nlmax, ts.bs0, ts.cen0,
             nthreads);
  H.host_tree_s = now() - tstart;
  plan_end(H);
  return 0;
}

}  // namespace fgtb
