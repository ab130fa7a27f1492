// ORACLE -- test infrastructure only.
//
// A CPU restatement, routine by routine, of the plane-wave point Gauss
// transform of flatironinstitute/fgt2d (directories 2d/planewave and
// 3d/planewave, legacy Fortran).  It exists to check the CUDA product path and
// to provide the timed CPU baseline.  Nothing in the product library links,
// loads or calls this file; only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py do.
//
// Pinning: the reference cannot be compiled here (no Fortran compiler), so the
// restatement is pinned against the reference's own known-answer test: FGT vs
// an FP64 direct sum, relative l2 error (test_fgt2d.f:161-174, 204-225;
// test_fgt3d.f:142-171), on the reference test inputs regenerated with the
// restated hkrand/DLARAN generator (hkrand.f:3-19, dlaran.f:1-89).
//
// Conventions: arrays that mirror Fortran arrays keep 1-based box ids and
// column-major layouts so that each loop can be read beside the Fortran line
// it follows.  Charges and/or dipoles (ifcharge, ifdipole in {0,1}) with
// potentials, gradients and Hessians (ifpgh, ifpghtarg in {0..3}) are
// restated; other flag values return ORC_UNSUPPORTED.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cplx;

namespace {

enum { ORC_OK = 0, ORC_BADARG = 1, ORC_UNSUPPORTED = 2 };

// Fortran default-real literals used in the reference (single precision).
const double F105 = (double)1.05f;   // computecoll, tree_routs4.f:195
const double F109 = (double)1.09f;   // g2dhlterms, g2dterms.f:54

inline double powi(double x, int n) { return __builtin_powi(x, n); }

// ---------------------------------------------------------------- RNG
// dlaran.f:1-89: multiplicative congruential generator mod 2^48,
// multiplier 33952834046453 held as four 12-bit digits.
double dlaran(int* s) {
  const int M1 = 494, M2 = 322, M3 = 2508, M4 = 2549, IPW2 = 4096;
  const double R = 1.0 / IPW2;
  int it4 = s[3] * M4;
  int it3 = it4 / IPW2;
  it4 -= IPW2 * it3;
  it3 += s[2] * M4 + s[3] * M3;
  int it2 = it3 / IPW2;
  it3 -= IPW2 * it2;
  it2 += s[1] * M4 + s[2] * M3 + s[3] * M2;
  int it1 = it2 / IPW2;
  it2 -= IPW2 * it1;
  it1 += s[0] * M4 + s[1] * M3 + s[2] * M2 + s[3] * M1;
  it1 %= IPW2;
  s[0] = it1; s[1] = it2; s[2] = it3; s[3] = it4;
  return R * ((double)it1 + R * ((double)it2 + R * ((double)it3 + R * (double)it4)));
}
int g_hkseed[4] = {0, 0, 0, 1};

// ---------------------------------------------------------------- terms
// g2dterms.f:19-64 / g3dterms.f:13-58 (identical formulas)
int hlterms(int ndim, double bsize, double delta, double eps, int nterms_in) {
  int nterms = nterms_in;
  double e1 = std::exp(1.0);
  double r = bsize / std::sqrt(2.0 * delta);
  int p0 = (int)(e1 * r * r) + 1;
  double rk = F109 * std::pow(8 * std::atan(1.0), -0.25);
  for (int p = p0; p <= 300; p++) {
    double rp = r * std::sqrt(e1 / p);
    double error = ndim * rk * std::pow(p * 1.0, -0.25) * powi(rp, p) / (1 - rp);
    if (error < eps) { nterms = p; break; }
  }
  return nterms;
}
// g2dterms.f:71-133
void pwterms(double bsize, double delta, double eps, double* pmax, int* npw) {
  double pi = 4.0 * std::atan(1.0);
  double rmax = bsize / std::sqrt(delta);
  double d = std::sqrt(std::log(1.0 / eps));
  *pmax = 2.0 * d;
  double h = 2 * pi / (rmax + d);
  int n = (int)(*pmax / h);
  *npw = 2 * n;
}

// pts_tree2d4.f:1187-1258 / pts_tree3d.f:1597-1685
template <int D>
void boxsize0(double delta, double eps, const double* src, int ns,
              const double* trg, int nt, int* levcut, double* bs0, double* cen0) {
  double mn[3], mx[3];
  for (int d = 0; d < D; d++) mn[d] = mx[d] = src[d];
  for (int i = 0; i < ns; i++)
    for (int d = 0; d < D; d++) {
      double v = src[D * i + d];
      if (v < mn[d]) mn[d] = v;
      if (v > mx[d]) mx[d] = v;
    }
  for (int i = 0; i < nt; i++)
    for (int d = 0; d < D; d++) {
      double v = trg[D * i + d];
      if (v < mn[d]) mn[d] = v;
      if (v > mx[d]) mx[d] = v;
    }
  double b = mx[0] - mn[0];
  for (int d = 1; d < D; d++)
    if (mx[d] - mn[d] > b) b = mx[d] - mn[d];
  for (int d = 0; d < D; d++) cen0[d] = (mn[d] + mx[d]) / 2;
  double dc = std::sqrt(delta * std::log(1.0 / eps));
  double dl = std::log(b / dc) / std::log(2.0);
  int lc = (int)dl;
  *bs0 = b;
  *levcut = lc;
  if (b < dc) return;
  *bs0 = (double)(1 << (lc + 1)) * dc;
  *levcut = lc + 1;
}

// ---------------------------------------------------------------- tree
template <int D>
struct Tree {
  static const int NCH = 1 << D;
  static const int NCO = (D == 2) ? 9 : 27;
  int nlevels = 0, nboxes = 0;
  std::vector<int> laddr;                 // laddr[2l], laddr[2l+1]
  std::vector<int> ilevel, iparent, nchild, ichild, nnbors, nbors;  // index by box (1-based)
  std::vector<double> centers;            // centers[D*b + d]
  std::vector<double> boxsize;
  void grow(int nb) {
    if ((int)ilevel.size() > nb) return;
    int n = std::max(nb + 1, (int)(ilevel.size() * 2));
    ilevel.resize(n, 0); iparent.resize(n, -1); nchild.resize(n, 0);
    ichild.resize((size_t)n * NCH, -1); centers.resize((size_t)n * D, 0.0);
  }
  int& ch(int b, int j) { return ichild[(size_t)b * NCH + (j - 1)]; }
  double& c(int b, int d) { return centers[(size_t)b * D + d]; }
  int& L(int l, int k) { return laddr[2 * l + k]; }
};

// child j (1-based) offset sign per dimension: tree_routs4.f:34-39,
// tree_routs3d.f:28-38
inline double child_sign(int j, int d) { return (((j - 1) >> d) & 1) ? 1.0 : -1.0; }

// tree_refine_boxes, tree_routs4.f:9-56 / tree_routs3d.f:9-63
template <int D>
void refine_boxes(Tree<D>& t, const std::vector<int>& irefine, int ifirst, int nbloc,
                  double bs, int& nbctr, int nlctr) {
  const int NCH = Tree<D>::NCH;
  int cnt = 0;
  for (int i = 0; i < nbloc; i++) cnt += irefine[i];
  t.grow(nbctr + cnt * NCH + 1);
  int isum = 0;
  for (int i = 0; i < nbloc; i++) {
    int ibox = ifirst + i;
    if (irefine[i] == 1) {
      isum++;
      int nbl = nbctr + (isum - 1) * NCH;
      t.nchild[ibox] = NCH;
      for (int j = 1; j <= NCH; j++) {
        int jbox = nbl + j;
        for (int d = 0; d < D; d++) t.c(jbox, d) = t.c(ibox, d) + child_sign(j, d) * bs / 2;
        t.iparent[jbox] = ibox;
        t.nchild[jbox] = 0;
        for (int l = 1; l <= NCH; l++) t.ch(jbox, l) = -1;
        t.ch(ibox, j) = jbox;
        t.ilevel[jbox] = nlctr;
      }
    }
  }
  nbctr += cnt * NCH;
}

// tree_refine_boxes_flag, tree_routs4.f:334-388
template <int D>
void refine_boxes_flag(Tree<D>& t, std::vector<int>& iflag, int ifirst, int nbloc,
                       double bs, int& nbctr, int nlctr) {
  const int NCH = Tree<D>::NCH;
  int cnt = 0;
  for (int i = 0; i < nbloc; i++) cnt += (iflag[ifirst + i] > 0);
  t.grow(nbctr + cnt * NCH + 1);
  if ((int)iflag.size() < (int)t.ilevel.size()) iflag.resize(t.ilevel.size(), 0);
  int isum = 0;
  for (int i = 0; i < nbloc; i++) {
    int ibox = ifirst + i;
    if (iflag[ibox] > 0) {
      isum++;
      int nbl = nbctr + (isum - 1) * NCH;
      t.nchild[ibox] = NCH;
      for (int j = 1; j <= NCH; j++) {
        int jbox = nbl + j;
        for (int d = 0; d < D; d++) t.c(jbox, d) = t.c(ibox, d) + child_sign(j, d) * bs / 2;
        t.iparent[jbox] = ibox;
        t.nchild[jbox] = 0;
        for (int l = 1; l <= NCH; l++) t.ch(jbox, l) = -1;
        t.ch(ibox, j) = jbox;
        t.ilevel[jbox] = nlctr + 1;
        if (iflag[ibox] == 1) iflag[jbox] = 3;
        if (iflag[ibox] == 2) iflag[jbox] = 0;
      }
    }
  }
  nbctr += cnt * NCH;
}

// sort_pts_to_children, pts_tree2d4.f:594-689 / pts_tree3d.f:662-851.
// The reference's passes amount to a stable partition of the box's range by
// child index, children in order 1..NCH; a point whose coordinate equals the
// centre goes to the upper child.
template <int D>
void sort_pts_to_children(Tree<D>& t, int ibox, const double* x, std::vector<int>& ix,
                          std::vector<int>& ixse) {
  const int NCH = Tree<D>::NCH;
  int s = ixse[2 * ibox], e = ixse[2 * ibox + 1];
  std::vector<int> bucket[8];
  for (int i = s; i <= e; i++) {
    int p = ix[i];
    int j = 0;
    for (int d = 0; d < D; d++)
      if (!(x[D * (p - 1) + d] - t.c(ibox, d) < 0)) j |= 1 << d;
    bucket[j].push_back(p);
  }
  int pos = s;
  for (int j = 0; j < NCH; j++) {
    int jbox = t.ch(ibox, j + 1);
    ixse[2 * jbox] = pos;
    for (int p : bucket[j]) ix[pos++] = p;
    ixse[2 * jbox + 1] = pos - 1;
  }
}

// computecoll, tree_routs4.f:100-211 / tree_routs3d.f:108-220
template <int D>
void computecoll(Tree<D>& t) {
  const int NCH = Tree<D>::NCH, NCO = Tree<D>::NCO;
  t.nnbors.assign(t.nboxes + 1, 0);
  t.nbors.assign((size_t)(t.nboxes + 1) * NCO, -1);
  t.nnbors[1] = 1;
  t.nbors[(size_t)1 * NCO] = 1;
  for (int ilev = 1; ilev <= t.nlevels; ilev++) {
    for (int ibox = t.L(ilev, 0); ibox <= t.L(ilev, 1); ibox++) {
      int dad = t.iparent[ibox];
      for (int i = 0; i < t.nnbors[dad]; i++) {
        int jbox = t.nbors[(size_t)dad * NCO + i];
        for (int j = 1; j <= NCH; j++) {
          int kbox = t.ch(jbox, j);
          if (kbox > 0) {
            bool ok = true;
            for (int d = 0; d < D; d++)
              if (!(std::fabs(t.c(kbox, d) - t.c(ibox, d)) <= F105 * t.boxsize[ilev])) ok = false;
            if (ok) {
              t.nbors[(size_t)ibox * NCO + t.nnbors[ibox]] = kbox;
              t.nnbors[ibox]++;
            }
          }
        }
      }
    }
  }
}

// updateflags, tree_routs4.f:217-326
template <int D>
void updateflags(Tree<D>& t, int curlev, int a, int b, std::vector<int>& iflag) {
  const int NCH = Tree<D>::NCH, NCO = Tree<D>::NCO;
  double distest = 1.05 * (t.boxsize[curlev] + t.boxsize[curlev + 1]) / 2.0;
  for (int ibox = a; ibox <= b; ibox++) {
    if (iflag[ibox] != 3) continue;
    iflag[ibox] = 0;
    for (int i = 0; i < t.nnbors[ibox]; i++) {
      int jbox = t.nbors[(size_t)ibox * NCO + i];
      bool hit = false;
      for (int j = 1; j <= NCH; j++) {
        int kbox = t.ch(jbox, j);
        if (kbox > 0 && t.nchild[kbox] > 0) {
          int ict = 0;
          for (int d = 0; d < D; d++)
            if (std::fabs(t.c(kbox, d) - t.c(ibox, d)) <= distest) ict++;
          if (ict == D) { iflag[ibox] = 1; hit = true; break; }
        }
      }
      if (hit) break;
    }
  }
}

// pts_tree_reorg, pts_tree2d4.f:1001-1150
template <int D>
void reorg(Tree<D>& t, std::vector<int>& laddrtail, std::vector<int>& iflag) {
  const int NCH = Tree<D>::NCH;
  int nb = t.nboxes;
  Tree<D> o = t;  // copy of the old arrays
  std::vector<int> tiflag(iflag.begin(), iflag.begin() + nb + 1);
  std::vector<int> tladdr = t.laddr;
  std::vector<int> map(nb + 1, 0);
  for (int ilev = 0; ilev <= 1 && ilev <= t.nlevels; ilev++)
    for (int ibox = tladdr[2 * ilev]; ibox <= tladdr[2 * ilev + 1]; ibox++) map[ibox] = ibox;
  if (t.nlevels >= 2) {
    int cur = tladdr[4];
    for (int ilev = 2; ilev <= t.nlevels; ilev++) {
      t.L(ilev, 0) = cur;
      for (int pass = 0; pass < 2; pass++) {
        int a = pass == 0 ? tladdr[2 * ilev] : laddrtail[2 * ilev];
        int b = pass == 0 ? tladdr[2 * ilev + 1] : laddrtail[2 * ilev + 1];
        for (int ibox = a; ibox <= b; ibox++) {
          t.ilevel[cur] = o.ilevel[ibox];
          t.nchild[cur] = o.nchild[ibox];
          for (int d = 0; d < D; d++) t.c(cur, d) = o.c(ibox, d);
          iflag[cur] = tiflag[ibox];
          map[ibox] = cur;
          cur++;
        }
      }
      t.L(ilev, 1) = cur - 1;
    }
  }
  for (int ibox = 1; ibox <= nb; ibox++) {
    if (o.iparent[ibox] == -1) t.iparent[map[ibox]] = -1;
    if (o.iparent[ibox] > 0) t.iparent[map[ibox]] = map[o.iparent[ibox]];
    for (int i = 1; i <= NCH; i++) {
      int c = o.ch(ibox, i);
      if (c == -1) t.ch(map[ibox], i) = -1;
      if (c > 0) t.ch(map[ibox], i) = map[c];
    }
  }
}

// pts_tree_fix_lr, pts_tree2d4.f:693-996 / pts_tree3d.f:855-1168
template <int D>
void fix_lr(Tree<D>& t) {
  const int NCH = Tree<D>::NCH, NCO = Tree<D>::NCO;
  int nlev = t.nlevels;
  std::vector<int> iflag(t.nboxes + 1, 0);
  for (int ilev = nlev; ilev >= 2; ilev--) {
    double distest = 1.05 * (t.boxsize[ilev - 1] + t.boxsize[ilev - 2]) / 2.0;
    for (int ibox = t.L(ilev, 0); ibox <= t.L(ilev, 1); ibox++) {
      int idad = t.iparent[ibox], igd = t.iparent[idad];
      for (int i = 0; i < t.nnbors[igd]; i++) {
        int jbox = t.nbors[(size_t)igd * NCO + i];
        if (t.nchild[jbox] == 0 && iflag[jbox] == 0) {
          int ict = 0;
          for (int d = 0; d < D; d++)
            if (std::fabs(t.c(jbox, d) - t.c(idad, d)) <= distest) ict++;
          if (ict == D) iflag[jbox] = 1;
        }
      }
    }
  }
  for (int ilev = nlev; ilev >= 1; ilev--) {
    double distest = 1.05 * (t.boxsize[ilev] + t.boxsize[ilev - 1]) / 2.0;
    for (int ibox = t.L(ilev, 0); ibox <= t.L(ilev, 1); ibox++) {
      if (iflag[ibox] == 1 || iflag[ibox] == 2) {
        int idad = t.iparent[ibox];
        for (int i = 0; i < t.nnbors[idad]; i++) {
          int jbox = t.nbors[(size_t)idad * NCO + i];
          if (t.nchild[jbox] == 0 && iflag[jbox] == 0) {
            int ict = 0;
            for (int d = 0; d < D; d++)
              if (std::fabs(t.c(jbox, d) - t.c(ibox, d)) <= distest) ict++;
            if (ict == D) iflag[jbox] = 2;
          }
        }
      }
    }
  }
  std::vector<int> tail(2 * (nlev + 1));
  for (int l = 0; l <= nlev; l++) { tail[2 * l] = 0; tail[2 * l + 1] = -1; }
  int nb = t.nboxes;
  for (int ilev = 1; ilev <= nlev - 2; ilev++) {
    tail[2 * (ilev + 1)] = nb + 1;
    int nbloc = t.L(ilev, 1) - t.L(ilev, 0) + 1;
    refine_boxes_flag(t, iflag, t.L(ilev, 0), nbloc, t.boxsize[ilev + 1], nb, ilev);
    tail[2 * (ilev + 1) + 1] = nb;
  }
  t.nboxes = nb;
  iflag.resize(std::max((size_t)nb + 1, iflag.size()), 0);
  reorg(t, tail, iflag);
  computecoll(t);
  for (int ibox = 1; ibox <= nb; ibox++)
    if (iflag[ibox] != 3) iflag[ibox] = 0;
  for (int l = 0; l <= nlev; l++) { tail[2 * l] = 0; tail[2 * l + 1] = -1; }
  for (int ilev = 2; ilev <= nlev - 2; ilev++) {
    updateflags(t, ilev, t.L(ilev, 0), t.L(ilev, 1), iflag);
    updateflags(t, ilev, tail[2 * ilev], tail[2 * ilev + 1], iflag);
    tail[2 * (ilev + 1)] = nb + 1;
    int nbloc = t.L(ilev, 1) - t.L(ilev, 0) + 1;
    refine_boxes_flag(t, iflag, t.L(ilev, 0), nbloc, t.boxsize[ilev + 1], nb, ilev);
    nbloc = tail[2 * ilev + 1] - tail[2 * ilev] + 1;
    refine_boxes_flag(t, iflag, tail[2 * ilev], nbloc, t.boxsize[ilev + 1], nb, ilev);
    tail[2 * (ilev + 1) + 1] = nb;
    t.nboxes = nb;
    if ((int)t.nnbors.size() < nb + 1) {
      t.nnbors.resize(nb + 1, 0);
      t.nbors.resize((size_t)(nb + 1) * NCO, -1);
    }
    for (int ibox = tail[2 * (ilev + 1)]; ibox <= tail[2 * (ilev + 1) + 1]; ibox++) {
      t.nnbors[ibox] = 0;
      int idad = t.iparent[ibox];
      for (int i = 0; i < t.nnbors[idad]; i++) {
        int jbox = t.nbors[(size_t)idad * NCO + i];
        for (int j = 1; j <= NCH; j++) {
          int kbox = t.ch(jbox, j);
          if (kbox > 0) {
            bool ok = true;
            for (int d = 0; d < D; d++)
              if (!(std::fabs(t.c(kbox, d) - t.c(ibox, d)) <= F105 * t.boxsize[ilev + 1])) ok = false;
            if (ok) {
              t.nbors[(size_t)ibox * NCO + t.nnbors[ibox]] = kbox;
              t.nnbors[ibox]++;
            }
          }
        }
      }
    }
  }
  t.nboxes = nb;
  iflag.resize(std::max((size_t)nb + 1, iflag.size()), 0);
  reorg(t, tail, iflag);
  computecoll(t);
}

// pts_tree_build (pts_tree2d4.f:363-590) with the level bound that
// pts_tree_mem (pts_tree2d4.f:34-356) would return, then pts_tree_sort
// (pts_tree2d4.f:1157-1181) of sources and targets.
template <int D>
void build_tree(Tree<D>& t, const double* src, int ns, const double* trg, int nt, int ndiv,
                int ndiv0, int levcut, int nlmax, double bs0, const double* cen0,
                std::vector<int>& isrc, std::vector<int>& isrcse, std::vector<int>& itarg,
                std::vector<int>& itargse) {
  const int NCH = Tree<D>::NCH;
  t.boxsize.assign(std::max(nlmax, 0) + 2, 0.0);
  t.laddr.assign(2 * (std::max(nlmax, 0) + 2), 0);
  t.grow(1);
  t.boxsize[0] = bs0;
  for (int d = 0; d < D; d++) t.c(1, d) = cen0[d];
  t.L(0, 0) = 1; t.L(0, 1) = 1;
  t.ilevel[1] = 0; t.iparent[1] = -1; t.nchild[1] = 0;
  for (int j = 1; j <= NCH; j++) t.ch(1, j) = -1;
  std::vector<int> xs(ns + 1), xt(nt + 1);
  std::vector<int> sse(4, 0), tse(4, 0);
  sse[2] = 1; sse[3] = ns; tse[2] = 1; tse[3] = nt;
  for (int i = 1; i <= ns; i++) xs[i] = i;
  for (int i = 1; i <= nt; i++) xt[i] = i;
  int nbctr = 1;
  int ilev;
  for (ilev = 0; ilev <= nlmax - 1; ilev++) {
    int ifirst = t.L(ilev, 0), ilast = t.L(ilev, 1);
    int nbloc = ilast - ifirst + 1;
    std::vector<int> irefine(nbloc, 0);
    int any = 0;
    for (int i = 0; i < nbloc; i++) {
      int ibox = ifirst + i;
      int nn = sse[2 * ibox + 1] - sse[2 * ibox] + 1;  // idivflag = 0
      if (ilev < levcut) { if (nn > ndiv0) irefine[i] = 1; }
      else { if (nn > ndiv) irefine[i] = 1; }
      any = std::max(any, irefine[i]);
    }
    if (any == 1) {
      t.boxsize[ilev + 1] = t.boxsize[ilev] / 2;
      t.L(ilev + 1, 0) = nbctr + 1;
      refine_boxes(t, irefine, ifirst, nbloc, t.boxsize[ilev + 1], nbctr, ilev + 1);
      sse.resize(2 * (nbctr + 1), 0);
      tse.resize(2 * (nbctr + 1), 0);
      for (int i = 0; i < nbloc; i++) {
        if (irefine[i] == 1) {
          sort_pts_to_children(t, ifirst + i, src, xs, sse);
          sort_pts_to_children(t, ifirst + i, trg, xt, tse);
        }
      }
      t.L(ilev + 1, 1) = nbctr;
    } else {
      break;
    }
  }
  t.nboxes = nbctr;
  t.nlevels = ilev;
  computecoll(t);
  if (t.nlevels >= 2) fix_lr(t);
  // pts_tree_sort for sources and targets on the final tree
  for (int pass = 0; pass < 2; pass++) {
    const double* x = pass == 0 ? src : trg;
    int n = pass == 0 ? ns : nt;
    std::vector<int>& ix = pass == 0 ? isrc : itarg;
    std::vector<int>& ixse = pass == 0 ? isrcse : itargse;
    ix.assign(n + 1, 0);
    ixse.assign(2 * (t.nboxes + 1), 0);
    for (int i = 1; i <= n; i++) ix[i] = i;
    ixse[2] = 1; ixse[3] = n;
    for (int l = 0; l <= t.nlevels - 1; l++)
      for (int ibox = t.L(l, 0); ibox <= t.L(l, 1); ibox++)
        if (t.nchild[ibox] > 0) sort_pts_to_children(t, ibox, x, ix, ixse);
  }
}

// ---------------------------------------------------------------- lists
// 2D compute_modified_list1, tree_routs4.f:715-879
void modified_list1_2d(Tree<2>& t, int npwlevel, std::vector<std::vector<int>>& list1) {
  const int NCO = 9;
  list1.assign(t.nboxes + 1, std::vector<int>());
  if (t.nchild[1] == 0) list1[1].push_back(1);
  for (int ilev = 1; ilev <= t.nlevels; ilev++) {
    for (int ibox = t.L(ilev, 0); ibox <= t.L(ilev, 1); ibox++) {
      if (t.nchild[ibox] != 0) continue;
      for (int i = 0; i < t.nnbors[ibox]; i++) {
        int jbox = t.nbors[(size_t)ibox * NCO + i];
        if (ilev >= npwlevel) {
          list1[ibox].push_back(jbox);
        } else if (t.nchild[jbox] == 0) {
          list1[ibox].push_back(jbox);
        } else {
          double distest = 1.05 * (t.boxsize[ilev] + t.boxsize[ilev + 1]) / 2.0;
          for (int j = 1; j <= t.nchild[jbox]; j++) {
            int kbox = t.ch(jbox, j);
            double xd = std::fabs(t.c(kbox, 0) - t.c(ibox, 0));
            double yd = std::fabs(t.c(kbox, 1) - t.c(ibox, 1));
            if (xd < distest && yd < distest) {
              list1[ibox].push_back(kbox);
              list1[kbox].push_back(ibox);
            }
          }
        }
      }
    }
  }
}

// 3D compute_modified_list1, tree_routs3d.f:511-619
void modified_list1_3d(Tree<3>& t, int npwlevel, std::vector<std::vector<int>>& list1) {
  const int NCO = 27;
  list1.assign(t.nboxes + 1, std::vector<int>());
  if (t.nchild[1] == 0) list1[1].push_back(1);
  for (int ilev = 1; ilev <= t.nlevels; ilev++) {
    for (int ibox = t.L(ilev, 0); ibox <= t.L(ilev, 1); ibox++) {
      int dad = t.iparent[ibox];
      if (t.nchild[ibox] != 0) continue;
      for (int i = 0; i < t.nnbors[ibox]; i++) {
        int jbox = t.nbors[(size_t)ibox * NCO + i];
        if (ilev >= npwlevel) {
          list1[ibox].push_back(jbox);
        } else if (t.nchild[jbox] == 0) {
          list1[ibox].push_back(jbox);
        } else {
          double distest = 1.05 * (t.boxsize[ilev] + t.boxsize[ilev + 1]) / 2.0 * 1;
          for (int j = 1; j <= 8; j++) {
            int kbox = t.ch(jbox, j);
            if (kbox > 0) {
              double xd = std::fabs(t.c(kbox, 0) - t.c(ibox, 0));
              double yd = std::fabs(t.c(kbox, 1) - t.c(ibox, 1));
              double zd = std::fabs(t.c(kbox, 2) - t.c(ibox, 2));
              if (xd < distest && yd < distest && zd < distest) list1[ibox].push_back(kbox);
            }
          }
        }
      }
      for (int i = 0; i < t.nnbors[dad]; i++) {
        int jbox = t.nbors[(size_t)dad * NCO + i];
        if (t.nchild[jbox] == 0) {
          double distest = 1.05 * (t.boxsize[ilev] + t.boxsize[ilev - 1]) / 2.0 * 1;
          double xd = std::fabs(t.c(jbox, 0) - t.c(ibox, 0));
          double yd = std::fabs(t.c(jbox, 1) - t.c(ibox, 1));
          double zd = std::fabs(t.c(jbox, 2) - t.c(ibox, 2));
          if (xd < distest && yd < distest && zd < distest) list1[ibox].push_back(jbox);
        }
      }
    }
  }
}

// gt2d_computelistpw_slow, tree_routs4.f:907-972
void listpw_2d(Tree<2>& t, int npwlevel, std::vector<std::vector<int>>& lpw) {
  lpw.assign(t.nboxes + 1, std::vector<int>());
  int nls = std::max(npwlevel, 0);
  for (int ilev = nls; ilev <= t.nlevels; ilev++)
    for (int ibox = t.L(ilev, 0); ibox <= t.L(ilev, 1); ibox++) {
      if (ilev == npwlevel) {
        for (int i = 0; i < t.nnbors[ibox]; i++) {
          int jbox = t.nbors[(size_t)ibox * 9 + i];
          if (jbox != ibox) lpw[ibox].push_back(jbox);
        }
      } else if (ilev > std::max(npwlevel, 0)) {
        int dad = t.iparent[ibox];
        for (int i = 1; i <= t.nchild[dad]; i++) {
          int jbox = t.ch(dad, i);
          if (jbox != ibox) lpw[ibox].push_back(jbox);
        }
      }
    }
}

// gt3d_computelistpw, tree_routs3d.f:644-719
void listpw_3d(Tree<3>& t, int npwlevel, std::vector<std::vector<int>>& lpw) {
  lpw.assign(t.nboxes + 1, std::vector<int>());
  int nls = std::max(npwlevel, 0);
  for (int ilev = nls; ilev <= t.nlevels; ilev++)
    for (int ibox = t.L(ilev, 0); ibox <= t.L(ilev, 1); ibox++) {
      if (ilev == npwlevel) {
        for (int i = 0; i < t.nnbors[ibox]; i++) {
          int jbox = t.nbors[(size_t)ibox * 27 + i];
          if (jbox != ibox && t.nchild[jbox] > 0) lpw[ibox].push_back(jbox);
        }
      } else if (ilev > std::max(npwlevel, 0)) {
        int dad = t.iparent[ibox];
        for (int i = 1; i <= 8; i++) {
          int jbox = t.ch(dad, i);
          if (jbox > 0 && jbox != ibox) lpw[ibox].push_back(jbox);
        }
      }
    }
}

// ---------------------------------------------------------------- PW tables
// get_pwnodes, g2drouts.f:2205-2225 (2D order: +half then -half)
void pwnodes_2d(double pmax, int npw, std::vector<double>& ws, std::vector<double>& ts) {
  double pi = 4.0 * std::atan(1.0);
  int npw2 = npw / 2;
  double h = pmax / npw2, w = h / (2.0 * std::sqrt(pi));
  ws.assign(npw + 1, 0); ts.assign(npw + 1, 0);
  for (int j = 1; j <= npw2; j++) {
    ts[j] = (j - 0.5) * h;
    ws[j] = w * std::exp(-ts[j] * ts[j] / 4);
    ts[j + npw2] = -ts[j];
    ws[j + npw2] = ws[j];
  }
}
// get_pwnodes, g3drouts.f:2669-2690 (3D order: ascending, negatives first)
void pwnodes_3d(double pmax, int npw, std::vector<double>& ws, std::vector<double>& ts) {
  double pi = 4.0 * std::atan(1.0);
  int npw2 = npw / 2;
  double h = pmax / npw2, w = h / (2.0 * std::sqrt(pi));
  ws.assign(npw + 1, 0); ts.assign(npw + 1, 0);
  for (int j = -npw2; j <= npw2 - 1; j++) {
    int k = j + npw2 + 1;
    ts[k] = (j + 0.5) * h;
    ws[k] = w * std::exp(-ts[k] * ts[k] / 4);
  }
}

// ---------------------------------------------------------------- 2D expansions
// g2dformhc_vec, g2drouts.f:100-168.  ffexp(0:p,0:p,nd)
void g2dformhc(int nd, double delta, const double* src, int ns, const double* chg,
               const double* cent, int p, double* ff) {
  int P = p + 1;
  std::fill(ff, ff + (size_t)P * P * nd, 0.0);
  std::vector<double> xp(P), yp(P);
  double dsq = 1.0 / std::sqrt(delta);
  for (int i = 0; i < ns; i++) {
    double x = (src[2 * i] - cent[0]) * dsq, y = (src[2 * i + 1] - cent[1]) * dsq;
    xp[0] = 1.0; yp[0] = 1.0;
    for (int k = 1; k <= p; k++) {
      double tmp = std::sqrt((double)k);
      xp[k] = xp[k - 1] * x / tmp;
      yp[k] = yp[k - 1] * y / tmp;
    }
    for (int ind = 0; ind < nd; ind++) {
      double q = chg[nd * i + ind];
      for (int k = 0; k <= p; k++) {
        double yt = q * yp[k];
        for (int j = 0; j <= p; j++) ff[(size_t)ind * P * P + j + P * k] += yt * xp[j];
      }
    }
  }
}
// Dipole terms of g2dformhd_vec / g2dformhcd_vec (g2drouts.f:173-338), added
// to ff: with hx_j = x^j/sqrt(j!) and dxhx_j = j dsq hx_{j-1}/sqrt(j) (the
// derivative in the source coordinate),
//   ff(j,k) += dipstr (n1 dxhx_j hy_k + n2 hx_j dyhy_k).
void g2dformhd_add(int nd, double delta, const double* src, int ns, const double* rn,
                   const double* ds, const double* cent, int p, double* ff) {
  int P = p + 1;
  std::vector<double> hx(P), hy(P), dxhx(P), dyhy(P);
  double dsq = 1.0 / std::sqrt(delta);
  for (int i = 0; i < ns; i++) {
    double x = (src[2 * i] - cent[0]) * dsq, y = (src[2 * i + 1] - cent[1]) * dsq;
    hx[0] = 1.0; hy[0] = 1.0; dxhx[0] = 0.0; dyhy[0] = 0.0;
    for (int j1 = 1; j1 <= p; j1++) {
      double tmp = std::sqrt((double)j1);
      hy[j1] = hy[j1 - 1] * y / tmp;
      hx[j1] = hx[j1 - 1] * x / tmp;
      dxhx[j1] = j1 * dsq * hx[j1 - 1] / tmp;
      dyhy[j1] = j1 * dsq * hy[j1 - 1] / tmp;
    }
    for (int ind = 0; ind < nd; ind++) {
      for (int k = 0; k <= p; k++) {
        double d1 = hy[k] * rn[2 * i] * ds[nd * i + ind];
        double d2 = dyhy[k] * rn[2 * i + 1] * ds[nd * i + ind];
        for (int j = 0; j <= p; j++) ff[(size_t)ind * P * P + j + P * k] += dxhx[j] * d1 + hx[j] * d2;
      }
    }
  }
}
// g2dh2pw_real_vec, g2drouts.f:1242-1329.  h2x(npw,0:p), pw(npw/2,npw,nd) +=
void g2dh2pw(int nd, int p, int npw, const double* h2x, const double* hexp, cplx* pw) {
  int P = p + 1, n2 = npw / 2;
  cplx eye(0, 1);
  std::vector<cplx> pxhy((size_t)P * n2);
  for (int ind = 0; ind < nd; ind++) {
    const double* H = hexp + (size_t)ind * P * P;
    for (int k2 = 1; k2 <= n2; k2++)
      for (int j2 = 0; j2 <= p; j2++) {
        cplx c[4] = {0, 0, 0, 0};
        for (int r = 0; r < 4; r++)
          for (int j1 = r; j1 <= p; j1 += 4) c[r] += h2x[(k2 - 1) + npw * j1] * H[j1 + P * j2];
        pxhy[j2 + P * (k2 - 1)] = c[0] - c[2] + eye * (c[1] - c[3]);
      }
    cplx* out = pw + (size_t)ind * n2 * npw;
    for (int k1 = 1; k1 <= npw; k1++)
      for (int k2 = 1; k2 <= n2; k2++) {
        cplx c[4] = {0, 0, 0, 0};
        for (int r = 0; r < 4; r++)
          for (int j2 = r; j2 <= p; j2 += 4) c[r] += h2x[(k1 - 1) + npw * j2] * pxhy[j2 + P * (k2 - 1)];
        out[(k2 - 1) + n2 * (k1 - 1)] += c[0] - c[2] + eye * (c[1] - c[3]);
      }
  }
}
// g2dpw2local_real_vec, g2drouts.f:1417-1540.  local(0:p,0:p,nd) =
void g2dpw2local(int nd, int p, int npw, const double* pw2l, const cplx* pw, double* local) {
  int P = p + 1, n2 = npw / 2;
  cplx eye(0, 1);
  std::vector<cplx> lx((size_t)P * npw);
  for (int ind = 0; ind < nd; ind++) {
    const cplx* W = pw + (size_t)ind * n2 * npw;
    double* Lo = local + (size_t)ind * P * P;
    for (int k2 = 0; k2 <= p; k2++)
      for (int j1 = 1; j1 <= npw; j1++) {
        cplx cd = 0;
        for (int j2 = 1; j2 <= n2; j2++) cd += pw2l[(j2 - 1) + npw * k2] * W[(j2 - 1) + n2 * (j1 - 1)];
        int m = k2 % 4;
        lx[k2 + P * (j1 - 1)] = m == 0 ? cd : m == 1 ? cd * eye : m == 2 ? -cd : -eye * cd;
      }
    for (int k1 = 0; k1 <= p; k1++) {
      int m = k1 % 4;
      for (int k2 = 0; k2 <= p; k2++) {
        cplx cd = 0;
        for (int j1 = 1; j1 <= n2; j1++) {
          cplx a = lx[k2 + P * (j1 - 1)], b = lx[k2 + P * (j1 + n2 - 1)];
          cd += pw2l[(j1 - 1) + npw * k1] * ((m % 2 == 0) ? (a + b) : (a - b));
        }
        double v = m == 0 ? cd.real() * 2 : m == 1 ? -cd.imag() * 2 : m == 2 ? -cd.real() * 2 : cd.imag() * 2;
        Lo[k2 + P * k1] = v;
      }
    }
  }
}
// g2dlevalp_vec / g2dlevalg_vec / g2dlevalh_vec, g2drouts.f:847-1085:
// potential (pgh = 1), + gradient (2), + Hessian (3, order xx, xy, yy).
// grad(nd, 2, nt) and hess(nd, 3, nt) as in the reference.
void g2dleval(int nd, double delta, const double* cent, int p, const double* local,
              const double* trg, int nt, int pgh, double* pot, double* grad, double* hess) {
  int P = p + 1;
  double dsq = 1.0 / std::sqrt(delta);
  std::vector<double> xp(P + 1), yp(P + 1), xpx(P + 1), ypy(P + 1), xpxx(P + 1), ypyy(P + 1);
  for (int it = 0; it < nt; it++) {
    double x = (trg[2 * it] - cent[0]) * dsq, y = (trg[2 * it + 1] - cent[1]) * dsq;
    xp[0] = 1; yp[0] = 1;
    for (int i = 1; i <= p; i++) { xp[i] = x * xp[i - 1]; yp[i] = y * yp[i - 1]; }
    if (pgh >= 2) {
      xpx[0] = 0; ypy[0] = 0;
      for (int i = 1; i <= p; i++) { xpx[i] = i * xp[i - 1] * dsq; ypy[i] = i * yp[i - 1] * dsq; }
    }
    if (pgh >= 3) {
      xpxx[0] = ypyy[0] = xpxx[1] = ypyy[1] = 0;
      for (int i = 2; i <= p; i++) {
        xpxx[i] = (double)(i * (i - 1)) * xp[i - 2] * dsq * dsq;
        ypyy[i] = (double)(i * (i - 1)) * yp[i - 2] * dsq * dsq;
      }
    }
    for (int ind = 0; ind < nd; ind++) {
      const double* Lo = local + (size_t)ind * P * P;
      double dd = 0, g1 = 0, g2 = 0, h1 = 0, h2 = 0, h3 = 0;
      for (int j1 = 0; j1 <= p; j1++) {
        double d2 = 0, d2x = 0, d2xx = 0;
        for (int j2 = 0; j2 <= p; j2++) {
          d2 += Lo[j2 + P * j1] * xp[j2];
          if (pgh >= 2) d2x += Lo[j2 + P * j1] * xpx[j2];
          if (pgh >= 3) d2xx += Lo[j2 + P * j1] * xpxx[j2];
        }
        dd += d2 * yp[j1];
        if (pgh >= 2) { g1 += d2x * yp[j1]; g2 += d2 * ypy[j1]; }
        if (pgh >= 3) { h1 += d2xx * yp[j1]; h2 += d2x * ypy[j1]; h3 += d2 * ypyy[j1]; }
      }
      pot[nd * it + ind] += dd;
      if (pgh >= 2) {
        grad[ind + nd * (0 + 2 * (size_t)it)] += g1;
        grad[ind + nd * (1 + 2 * (size_t)it)] += g2;
      }
      if (pgh >= 3) {
        hess[ind + nd * (0 + 3 * (size_t)it)] += h1;
        hess[ind + nd * (1 + 3 * (size_t)it)] += h2;
        hess[ind + nd * (2 + 3 * (size_t)it)] += h3;
      }
    }
  }
}
// g2dpwevalp_vec / g2dpwevalg_vec / g2dpwevalh_vec, g2drouts.f:1887-2200
void g2dpweval(int nd, double delta, const double* cent, int npw, const double* ts,
               const cplx* pw, const double* trg, int nt, int pgh, double* pot, double* grad,
               double* hess) {
  cplx eye(0, 1);
  double dsq = 1.0 / std::sqrt(delta);
  int n2 = npw / 2;
  std::vector<cplx> w1(npw + 1), w2(npw + 1), w1x(npw + 1), w2y(npw + 1), w1xx(npw + 1), w2yy(npw + 1);
  for (int it = 0; it < nt; it++) {
    double x = (trg[2 * it] - cent[0]) * dsq, y = (trg[2 * it + 1] - cent[1]) * dsq;
    cplx qqx = std::exp(eye * ts[1] * x), qqy = std::exp(eye * ts[1] * y);
    cplx q1 = qqx, q2 = qqy;
    qqx = qqx * qqx; qqy = qqy * qqy;
    for (int j1 = 1; j1 <= n2; j1++) {
      w1[j1] = q1; w2[j1] = q2;
      w1[j1 + n2] = std::conj(w1[j1]);
      w2[j1 + n2] = std::conj(w2[j1]);
      if (pgh >= 2) {
        w1x[j1] = eye * ts[j1] * dsq * w1[j1];
        w2y[j1] = eye * ts[j1] * dsq * w2[j1];
        w1x[j1 + n2] = std::conj(w1x[j1]);
        w2y[j1 + n2] = std::conj(w2y[j1]);
      }
      if (pgh >= 3) {
        w1xx[j1] = eye * ts[j1] * dsq * w1x[j1];
        w2yy[j1] = eye * ts[j1] * dsq * w2y[j1];
        w1xx[j1 + n2] = std::conj(w1xx[j1]);
        w2yy[j1 + n2] = std::conj(w2yy[j1]);
      }
      q1 = q1 * qqx; q2 = q2 * qqy;
    }
    for (int ind = 0; ind < nd; ind++) {
      const cplx* W = pw + (size_t)ind * n2 * npw;
      cplx z = 0, zx = 0, zy = 0, zxx = 0, zxy = 0, zyy = 0;
      for (int j2 = 1; j2 <= npw; j2++) {
        cplx c = 0, cx = 0, cxx = 0;
        for (int j1 = 1; j1 <= n2; j1++) {
          const cplx wv = W[(j1 - 1) + n2 * (j2 - 1)];
          c += wv * w1[j1];
          if (pgh >= 2) cx += wv * w1x[j1];
          if (pgh >= 3) cxx += wv * w1xx[j1];
        }
        z += c * w2[j2];
        if (pgh >= 2) { zx += cx * w2[j2]; zy += c * w2y[j2]; }
        if (pgh >= 3) { zxx += cxx * w2[j2]; zxy += cx * w2y[j2]; zyy += c * w2yy[j2]; }
      }
      pot[nd * it + ind] += z.real() * 2;
      if (pgh >= 2) {
        grad[ind + nd * (0 + 2 * (size_t)it)] += zx.real() * 2;
        grad[ind + nd * (1 + 2 * (size_t)it)] += zy.real() * 2;
      }
      if (pgh >= 3) {
        hess[ind + nd * (0 + 3 * (size_t)it)] += zxx.real() * 2;
        hess[ind + nd * (1 + 3 * (size_t)it)] += zxy.real() * 2;
        hess[ind + nd * (2 + 3 * (size_t)it)] += zyy.real() * 2;
      }
    }
  }
}
// The 2D plane-wave expansion of a box formed directly from its sources:
// the quantity that g2dformpwc_vec of the NUFFT scheme (2d/nufft/src/
// g2drouts.f:1234-1307) computes with a type-1 NUFFT (finufft2d1many),
// here as the exact sum, in this restatement's 2D layout pw(npw/2, npw)
// (x nodes of the positive half first index, every y node second):
//   pw(k2, k1) += q ws(k2) ws(k1) exp(-i (ts(k2) x + ts(k1) y)).
void g2dformpwc(int nd, double delta, const double* src, int ns, const double* chg,
                const double* cent, int npw, const double* ws, const double* ts, cplx* pw) {
  cplx eye(0, 1);
  double dsq = 1.0 / std::sqrt(delta);
  int n2 = npw / 2;
  std::vector<cplx> w1(npw + 1), w2(npw + 1);
  for (int i = 0; i < ns; i++) {
    double x = (src[2 * i] - cent[0]) * dsq, y = (src[2 * i + 1] - cent[1]) * dsq;
    for (int j = 1; j <= npw; j++) {
      w1[j] = ws[j] * std::exp(-eye * ts[j] * x);
      w2[j] = ws[j] * std::exp(-eye * ts[j] * y);
    }
    for (int ind = 0; ind < nd; ind++) {
      double q = chg[nd * i + ind];
      cplx* out = pw + (size_t)ind * n2 * npw;
      for (int k1 = 1; k1 <= npw; k1++) {
        cplx yq = q * w2[k1];
        for (int k2 = 1; k2 <= n2; k2++) out[(k2 - 1) + n2 * (k1 - 1)] += yq * w1[k2];
      }
    }
  }
}
// g2dformlc_vec, g2drouts.f:621-681 (local accumulated, caller zeroes)
void g2dformlc(int nd, double delta, const double* src, int ns, const double* chg,
               const double* cent, int p, double* local) {
  int P = p + 1;
  double dsq = 1.0 / std::sqrt(delta);
  std::vector<double> hx(P + 1), hy(P + 1);
  for (int i = 0; i < ns; i++) {
    double x = (src[2 * i] - cent[0]) * dsq, y = (src[2 * i + 1] - cent[1]) * dsq;
    double fx = std::exp(-x * x), fy = std::exp(-y * y);
    hx[0] = fx; hy[0] = fy; hx[1] = 2.0 * x * fx; hy[1] = 2.0 * y * fy;
    for (int j = 1; j <= p - 1; j++) {
      hx[j + 1] = 2.0 * (x * hx[j] - hx[j - 1]) / (j + 1);
      hy[j + 1] = 2.0 * (y * hy[j] - hy[j - 1]) / (j + 1);
    }
    for (int ind = 0; ind < nd; ind++) {
      double q = chg[nd * i + ind];
      for (int j1 = 0; j1 <= p; j1++) {
        double yt = q * hy[j1];
        for (int j2 = 0; j2 <= p; j2++) local[(size_t)ind * P * P + j2 + P * j1] += yt * hx[j2];
      }
    }
  }
}
// Dipole terms of g2dformld_vec / g2dformlcd_vec (g2drouts.f:685-840): the
// Hermite functions h_j = H_j(x) e^{-x^2}/j! and dh_j = -(j+1) dsq h_{j+1}.
void g2dformld_add(int nd, double delta, const double* src, int ns, const double* rn,
                   const double* ds, const double* cent, int p, double* local) {
  int P = p + 1;
  double dsq = 1.0 / std::sqrt(delta);
  std::vector<double> hx(P + 1), hy(P + 1), dhx(P), dhy(P);
  for (int i = 0; i < ns; i++) {
    double x = (src[2 * i] - cent[0]) * dsq, y = (src[2 * i + 1] - cent[1]) * dsq;
    double fx = std::exp(-x * x), fy = std::exp(-y * y);
    hx[0] = fx; hy[0] = fy; hx[1] = 2.0 * x * fx; hy[1] = 2.0 * y * fy;
    for (int j = 1; j <= p; j++) {
      hx[j + 1] = 2.0 * (x * hx[j] - hx[j - 1]) / (j + 1);
      hy[j + 1] = 2.0 * (y * hy[j] - hy[j - 1]) / (j + 1);
    }
    for (int j = 0; j <= p; j++) {
      dhx[j] = -hx[j + 1] * dsq * (j + 1.0);
      dhy[j] = -hy[j + 1] * dsq * (j + 1.0);
    }
    for (int ind = 0; ind < nd; ind++) {
      double r1 = rn[2 * i] * ds[nd * i + ind], r2 = rn[2 * i + 1] * ds[nd * i + ind];
      for (int j1 = 0; j1 <= p; j1++) {
        double ry1 = hy[j1] * r1, ry2 = dhy[j1] * r2;
        for (int j2 = 0; j2 <= p; j2++) local[(size_t)ind * P * P + j2 + P * j1] += dhx[j2] * ry1 + hx[j2] * ry2;
      }
    }
  }
}

// ---------------------------------------------------------------- 3D expansions
// g3dformhc_vec, g3drouts.f:109-192.  ffexp(0:p,0:p,0:p,nd)
void g3dformhc(int nd, double delta, const double* src, int ns, const double* chg,
               const double* cent, int p, double* ff) {
  int P = p + 1;
  size_t PP = (size_t)P * P * P;
  std::fill(ff, ff + PP * nd, 0.0);
  std::vector<double> xp(P), yp(P), zp(P), sqk(P);
  double dsq = 1.0 / std::sqrt(delta);
  for (int k = 1; k <= p; k++) sqk[k] = std::sqrt((double)k);
  for (int i = 0; i < ns; i++) {
    double x = (src[3 * i] - cent[0]) * dsq, y = (src[3 * i + 1] - cent[1]) * dsq,
           z = (src[3 * i + 2] - cent[2]) * dsq;
    xp[0] = yp[0] = zp[0] = 1.0;
    for (int k = 1; k <= p; k++) {
      xp[k] = xp[k - 1] * x / sqk[k];
      yp[k] = yp[k - 1] * y / sqk[k];
      zp[k] = zp[k - 1] * z / sqk[k];
    }
    for (int ind = 0; ind < nd; ind++) {
      double q = chg[nd * i + ind];
      double* F = ff + PP * ind;
      for (int l = 0; l <= p; l++) {
        double zt = q * zp[l];
        for (int k = 0; k <= p; k++) {
          double rt = zt * yp[k];
          for (int j = 0; j <= p; j++) F[j + P * (k + (size_t)P * l)] += rt * xp[j];
        }
      }
    }
  }
}
// g3dh2pw_real_vec, g3drouts.f:1565-1685.  h2x(0:p,npw), pw(npw,npw,npw/2,nd) +=
void g3dh2pw(int nd, int p, int npw, const double* h2x, const double* hexp, cplx* pw) {
  int P = p + 1, n2 = npw / 2;
  cplx eye(0, 1);
  std::vector<cplx> a((size_t)npw * P * P), b((size_t)npw * npw * P);
  auto HX = [&](int j, int k) { return h2x[j + (size_t)P * (k - 1)]; };
  for (int ind = 0; ind < nd; ind++) {
    const double* H = hexp + (size_t)ind * P * P * P;
    for (int j1 = 0; j1 <= p; j1++)
      for (int j2 = 0; j2 <= p; j2++)
        for (int k3 = 1; k3 <= n2; k3++) {
          cplx c[4] = {0, 0, 0, 0};
          for (int r = 0; r < 4; r++)
            for (int j3 = r; j3 <= p; j3 += 4) c[r] += HX(j3, k3) * H[j3 + P * (j2 + (size_t)P * j1)];
          cplx ce = c[0] - c[2], co = eye * (c[1] - c[3]);
          a[(k3 - 1) + npw * (j2 + (size_t)P * j1)] = ce + co;
          a[(npw - k3) + npw * (j2 + (size_t)P * j1)] = ce - co;
        }
    for (int j1 = 0; j1 <= p; j1++)
      for (int k2 = 1; k2 <= n2; k2++)
        for (int k3 = 1; k3 <= npw; k3++) {
          cplx c[4] = {0, 0, 0, 0};
          for (int r = 0; r < 4; r++)
            for (int j2 = r; j2 <= p; j2 += 4) c[r] += HX(j2, k2) * a[(k3 - 1) + npw * (j2 + (size_t)P * j1)];
          cplx ce = c[0] - c[2], co = eye * (c[1] - c[3]);
          b[(k3 - 1) + npw * ((k2 - 1) + (size_t)npw * j1)] = ce + co;
          b[(k3 - 1) + npw * ((npw - k2) + (size_t)npw * j1)] = ce - co;
        }
    cplx* out = pw + (size_t)ind * npw * npw * n2;
    for (int k1 = 1; k1 <= n2; k1++)
      for (int k2 = 1; k2 <= npw; k2++)
        for (int k3 = 1; k3 <= npw; k3++) {
          cplx c[4] = {0, 0, 0, 0};
          for (int r = 0; r < 4; r++)
            for (int j1 = r; j1 <= p; j1 += 4) c[r] += HX(j1, k1) * b[(k3 - 1) + npw * ((k2 - 1) + (size_t)npw * j1)];
          out[(k3 - 1) + npw * ((k2 - 1) + (size_t)npw * (k1 - 1))] += c[0] - c[2] + eye * (c[1] - c[3]);
        }
  }
}
// g3dformpwc_vec, g3drouts.f:1950-2038
void g3dformpwc(int nd, double delta, const double* src, int ns, const double* chg,
                const double* cent, int npw, const double* ws, const double* ts, cplx* pw) {
  cplx eye(0, 1);
  double dsq = 1.0 / std::sqrt(delta);
  int n2 = npw / 2;
  std::vector<cplx> w1(npw + 1), w2(npw + 1), w3(npw + 1);
  for (int i = 0; i < ns; i++) {
    double x = (src[3 * i] - cent[0]) * dsq, y = (src[3 * i + 1] - cent[1]) * dsq,
           z = (src[3 * i + 2] - cent[2]) * dsq;
    cplx qx = std::exp(-eye * ts[n2 + 1] * x), qy = std::exp(-eye * ts[n2 + 1] * y),
         qz = std::exp(-eye * ts[n2 + 1] * z);
    cplx q1 = qx, q2 = qy, q3 = qz;
    qx = qx * qx; qy = qy * qy; qz = qz * qz;
    for (int j1 = n2 + 1; j1 <= npw; j1++) {
      w1[j1] = q1 * ws[j1]; w2[j1] = q2 * ws[j1]; w3[j1] = q3 * ws[j1];
      q1 = q1 * qx; q2 = q2 * qy; q3 = q3 * qz;
      w1[npw - j1 + 1] = std::conj(w1[j1]);
      w2[npw - j1 + 1] = std::conj(w2[j1]);
      w3[npw - j1 + 1] = std::conj(w3[j1]);
    }
    for (int ind = 0; ind < nd; ind++) {
      double q = chg[nd * i + ind];
      cplx* out = pw + (size_t)ind * npw * npw * n2;
      for (int j3 = 1; j3 <= n2; j3++) {
        cplx zt = q * w3[j3];
        for (int j2 = 1; j2 <= npw; j2++) {
          cplx yt = zt * w2[j2];
          for (int j1 = 1; j1 <= npw; j1++) out[(j1 - 1) + npw * ((j2 - 1) + (size_t)npw * (j3 - 1))] += yt * w1[j1];
        }
      }
    }
  }
}
// Dipole terms of g3dformhd_vec / g3dformhcd_vec (g3drouts.f:197-405)
void g3dformhd_add(int nd, double delta, const double* src, int ns, const double* rn,
                   const double* ds, const double* cent, int p, double* ff) {
  int P = p + 1;
  size_t PP = (size_t)P * P * P;
  std::vector<double> hx(P), hy(P), hz(P), dxhx(P), dyhy(P), dzhz(P), sqk(P);
  double dsq = 1.0 / std::sqrt(delta);
  for (int k = 1; k <= p; k++) sqk[k] = std::sqrt((double)k);
  for (int i = 0; i < ns; i++) {
    double x = (src[3 * i] - cent[0]) * dsq, y = (src[3 * i + 1] - cent[1]) * dsq,
           z = (src[3 * i + 2] - cent[2]) * dsq;
    hx[0] = hy[0] = hz[0] = 1.0;
    dxhx[0] = dyhy[0] = dzhz[0] = 0.0;
    for (int j1 = 1; j1 <= p; j1++) {
      hy[j1] = hy[j1 - 1] * y / sqk[j1];
      hx[j1] = hx[j1 - 1] * x / sqk[j1];
      hz[j1] = hz[j1 - 1] * z / sqk[j1];
      dxhx[j1] = j1 * dsq * hx[j1 - 1] / sqk[j1];
      dyhy[j1] = j1 * dsq * hy[j1 - 1] / sqk[j1];
      dzhz[j1] = j1 * dsq * hz[j1 - 1] / sqk[j1];
    }
    for (int ind = 0; ind < nd; ind++) {
      double r1 = rn[3 * i] * ds[nd * i + ind], r2 = rn[3 * i + 1] * ds[nd * i + ind],
             r3 = rn[3 * i + 2] * ds[nd * i + ind];
      double* F = ff + PP * ind;
      for (int l = 0; l <= p; l++) {
        double d1 = hz[l] * r1, d2 = hz[l] * r2, d3 = dzhz[l] * r3;
        for (int k = 0; k <= p; k++) {
          double c1 = hy[k] * d1, c2 = dyhy[k] * d2 + hy[k] * d3;
          for (int j = 0; j <= p; j++) F[j + P * (k + (size_t)P * l)] += dxhx[j] * c1 + hx[j] * c2;
        }
      }
    }
  }
}
// Dipole terms of g3dformpwd_vec / g3dformpwcd_vec (g3drouts.f:2042-2262):
// the node factors times -i t dsq (the source-coordinate derivative).
void g3dformpwd_add(int nd, double delta, const double* src, int ns, const double* rn,
                    const double* ds, const double* cent, int npw, const double* ws,
                    const double* ts, cplx* pw) {
  cplx eye(0, 1);
  double dsq = 1.0 / std::sqrt(delta);
  int n2 = npw / 2;
  std::vector<cplx> w1(npw + 1), w2(npw + 1), w3(npw + 1), w1x(npw + 1), w2y(npw + 1), w3z(npw + 1);
  for (int i = 0; i < ns; i++) {
    double x = (src[3 * i] - cent[0]) * dsq, y = (src[3 * i + 1] - cent[1]) * dsq,
           z = (src[3 * i + 2] - cent[2]) * dsq;
    cplx qx = std::exp(-eye * ts[n2 + 1] * x), qy = std::exp(-eye * ts[n2 + 1] * y),
         qz = std::exp(-eye * ts[n2 + 1] * z);
    cplx q1 = qx, q2 = qy, q3 = qz;
    qx = qx * qx; qy = qy * qy; qz = qz * qz;
    for (int j1 = n2 + 1; j1 <= npw; j1++) {
      w1[j1] = q1 * ws[j1]; w2[j1] = q2 * ws[j1]; w3[j1] = q3 * ws[j1];
      q1 = q1 * qx; q2 = q2 * qy; q3 = q3 * qz;
      w1[npw - j1 + 1] = std::conj(w1[j1]);
      w2[npw - j1 + 1] = std::conj(w2[j1]);
      w3[npw - j1 + 1] = std::conj(w3[j1]);
    }
    for (int j1 = 1; j1 <= npw; j1++) {
      cplx zt = -eye * ts[j1] * dsq;
      w1x[j1] = w1[j1] * zt; w2y[j1] = w2[j1] * zt; w3z[j1] = w3[j1] * zt;
    }
    for (int ind = 0; ind < nd; ind++) {
      double r1 = rn[3 * i] * ds[nd * i + ind], r2 = rn[3 * i + 1] * ds[nd * i + ind],
             r3 = rn[3 * i + 2] * ds[nd * i + ind];
      cplx* out = pw + (size_t)ind * npw * npw * n2;
      for (int j3 = 1; j3 <= n2; j3++) {
        cplx rz1 = w3[j3] * r1, rz2 = w3[j3] * r2, rz3 = w3z[j3] * r3;
        for (int j2 = 1; j2 <= npw; j2++) {
          cplx ry1 = rz1 * w2[j2], ry2 = rz2 * w2y[j2] + rz3 * w2[j2];
          for (int j1 = 1; j1 <= npw; j1++)
            out[(j1 - 1) + npw * ((j2 - 1) + (size_t)npw * (j3 - 1))] += w1x[j1] * ry1 + w1[j1] * ry2;
        }
      }
    }
  }
}
// g3dpw2local_real_vec, g3drouts.f:1774-1938.  pw2l(npw,0:p)
void g3dpw2local(int nd, int p, int npw, const double* pw2l, const cplx* pw, double* local) {
  int P = p + 1, n2 = npw / 2;
  cplx eye(0, 1);
  auto XL = [&](int j, int k) { return pw2l[(j - 1) + (size_t)npw * k]; };
  auto rot = [&](int k, cplx cd) { int m = k % 4; return m == 0 ? cd : m == 1 ? cd * eye : m == 2 ? -cd : -eye * cd; };
  std::vector<cplx> a((size_t)P * npw * n2), b((size_t)P * P * n2);
  for (int ind = 0; ind < nd; ind++) {
    const cplx* W = pw + (size_t)ind * npw * npw * n2;
    double* Lo = local + (size_t)ind * P * P * P;
    for (int j1 = 1; j1 <= n2; j1++)
      for (int j2 = 1; j2 <= npw; j2++)
        for (int k3 = 0; k3 <= p; k3++) {
          cplx cd = 0;
          for (int j3 = 1; j3 <= n2; j3++) {
            cplx u = W[(j3 - 1) + npw * ((j2 - 1) + (size_t)npw * (j1 - 1))];
            cplx v = W[(npw - j3) + npw * ((j2 - 1) + (size_t)npw * (j1 - 1))];
            cd += XL(j3, k3) * ((k3 % 2 == 0) ? (u + v) : (u - v));
          }
          a[k3 + P * ((j2 - 1) + (size_t)npw * (j1 - 1))] = rot(k3, cd);
        }
    for (int j1 = 1; j1 <= n2; j1++)
      for (int k2 = 0; k2 <= p; k2++)
        for (int k3 = 0; k3 <= p; k3++) {
          cplx cd = 0;
          for (int j2 = 1; j2 <= n2; j2++) {
            cplx u = a[k3 + P * ((j2 - 1) + (size_t)npw * (j1 - 1))];
            cplx v = a[k3 + P * ((npw - j2) + (size_t)npw * (j1 - 1))];
            cd += XL(j2, k2) * ((k2 % 2 == 0) ? (u + v) : (u - v));
          }
          b[k3 + P * (k2 + (size_t)P * (j1 - 1))] = rot(k2, cd);
        }
    for (int k1 = 0; k1 <= p; k1++) {
      int m = k1 % 4;
      for (int k2 = 0; k2 <= p; k2++)
        for (int k3 = 0; k3 <= p; k3++) {
          cplx cd = 0;
          for (int j1 = 1; j1 <= n2; j1++) cd += XL(j1, k1) * b[k3 + P * (k2 + (size_t)P * (j1 - 1))];
          double v = m == 0 ? cd.real() * 2 : m == 1 ? -cd.imag() * 2 : m == 2 ? -cd.real() * 2 : cd.imag() * 2;
          Lo[k3 + P * (k2 + (size_t)P * k1)] = v;
        }
    }
  }
}
// g3dlevalp_vec / g3dlevalg_vec / g3dlevalh_vec, g3drouts.f:1045-1360:
// Hessian order xx, yy, zz, xy, xz, yz.
void g3dleval(int nd, double delta, const double* cent, int p, const double* local,
              const double* trg, int nt, int pgh, double* pot, double* grad, double* hess) {
  int P = p + 1;
  double dsq = 1.0 / std::sqrt(delta);
  std::vector<double> xp(P + 1), yp(P + 1), zp(P + 1), xpx(P + 1), ypy(P + 1), zpz(P + 1),
      xpxx(P + 1), ypyy(P + 1), zpzz(P + 1);
  for (int it = 0; it < nt; it++) {
    double x = (trg[3 * it] - cent[0]) * dsq, y = (trg[3 * it + 1] - cent[1]) * dsq,
           z = (trg[3 * it + 2] - cent[2]) * dsq;
    xp[0] = yp[0] = zp[0] = 1;
    for (int i = 1; i <= p; i++) { xp[i] = x * xp[i - 1]; yp[i] = y * yp[i - 1]; zp[i] = z * zp[i - 1]; }
    if (pgh >= 2) {
      xpx[0] = ypy[0] = zpz[0] = 0;
      for (int i = 1; i <= p; i++) {
        xpx[i] = i * xp[i - 1] * dsq; ypy[i] = i * yp[i - 1] * dsq; zpz[i] = i * zp[i - 1] * dsq;
      }
    }
    if (pgh >= 3) {
      xpxx[0] = ypyy[0] = zpzz[0] = xpxx[1] = ypyy[1] = zpzz[1] = 0;
      for (int i = 2; i <= p; i++) {
        const double c = (double)(i * (i - 1));
        xpxx[i] = c * xp[i - 2] * dsq * dsq;
        ypyy[i] = c * yp[i - 2] * dsq * dsq;
        zpzz[i] = c * zp[i - 2] * dsq * dsq;
      }
    }
    for (int ind = 0; ind < nd; ind++) {
      const double* Lo = local + (size_t)ind * P * P * P;
      double dd = 0, g1 = 0, g2 = 0, g3 = 0, h11 = 0, h22 = 0, h33 = 0, h12 = 0, h13 = 0, h23 = 0;
      for (int j1 = 0; j1 <= p; j1++) {
        double d1 = 0, d1x = 0, d1y = 0, d1xx = 0, d1yy = 0, d1xy = 0;
        for (int j2 = 0; j2 <= p; j2++) {
          double d2 = 0, d2x = 0, d2xx = 0;
          for (int j3 = 0; j3 <= p; j3++) {
            const double l = Lo[j3 + P * (j2 + (size_t)P * j1)];
            d2 += l * xp[j3];
            if (pgh >= 2) d2x += l * xpx[j3];
            if (pgh >= 3) d2xx += l * xpxx[j3];
          }
          d1 += d2 * yp[j2];
          if (pgh >= 2) { d1x += d2x * yp[j2]; d1y += d2 * ypy[j2]; }
          if (pgh >= 3) { d1xx += d2xx * yp[j2]; d1xy += d2x * ypy[j2]; d1yy += d2 * ypyy[j2]; }
        }
        dd += d1 * zp[j1];
        if (pgh >= 2) { g1 += d1x * zp[j1]; g2 += d1y * zp[j1]; g3 += d1 * zpz[j1]; }
        if (pgh >= 3) {
          h11 += d1xx * zp[j1]; h22 += d1yy * zp[j1]; h12 += d1xy * zp[j1];
          h13 += d1x * zpz[j1]; h23 += d1y * zpz[j1]; h33 += d1 * zpzz[j1];
        }
      }
      pot[nd * it + ind] += dd;
      if (pgh >= 2) {
        double g[3] = {g1, g2, g3};
        for (int k = 0; k < 3; k++) grad[ind + nd * (k + 3 * (size_t)it)] += g[k];
      }
      if (pgh >= 3) {
        double h[6] = {h11, h22, h33, h12, h13, h23};
        for (int k = 0; k < 6; k++) hess[ind + nd * (k + 6 * (size_t)it)] += h[k];
      }
    }
  }
}
// g3dpwevalp_vec / g3dpwevalg_vec / g3dpwevalh_vec, g3drouts.f:2268-2660
void g3dpweval(int nd, double delta, const double* cent, int npw, const double* ts,
               const cplx* pw, const double* trg, int nt, int pgh, double* pot, double* grad,
               double* hess) {
  cplx eye(0, 1);
  double dsq = 1.0 / std::sqrt(delta);
  int n2 = npw / 2;
  std::vector<cplx> w1(npw + 1), w2(npw + 1), w3(npw + 1), w1x(npw + 1), w2y(npw + 1),
      w3z(npw + 1), w1xx(npw + 1), w2yy(npw + 1), w3zz(npw + 1);
  for (int it = 0; it < nt; it++) {
    double x = (trg[3 * it] - cent[0]) * dsq, y = (trg[3 * it + 1] - cent[1]) * dsq,
           z = (trg[3 * it + 2] - cent[2]) * dsq;
    cplx qx = std::exp(eye * ts[n2 + 1] * x), qy = std::exp(eye * ts[n2 + 1] * y),
         qz = std::exp(eye * ts[n2 + 1] * z);
    cplx q1 = qx, q2 = qy, q3 = qz;
    qx = qx * qx; qy = qy * qy; qz = qz * qz;
    for (int j1 = n2 + 1; j1 <= npw; j1++) {
      const int m = npw - j1 + 1;
      w1[j1] = q1; w2[j1] = q2; w3[j1] = q3;
      w1[m] = std::conj(w1[j1]); w2[m] = std::conj(w2[j1]); w3[m] = std::conj(w3[j1]);
      const cplx zt = eye * ts[j1] * dsq;
      if (pgh >= 2) {
        w1x[j1] = zt * w1[j1]; w2y[j1] = zt * w2[j1]; w3z[j1] = zt * w3[j1];
        w1x[m] = std::conj(w1x[j1]); w2y[m] = std::conj(w2y[j1]); w3z[m] = std::conj(w3z[j1]);
      }
      if (pgh >= 3) {
        w1xx[j1] = zt * w1x[j1]; w2yy[j1] = zt * w2y[j1]; w3zz[j1] = zt * w3z[j1];
        w1xx[m] = std::conj(w1xx[j1]); w2yy[m] = std::conj(w2yy[j1]); w3zz[m] = std::conj(w3zz[j1]);
      }
      q1 = q1 * qx; q2 = q2 * qy; q3 = q3 * qz;
    }
    for (int ind = 0; ind < nd; ind++) {
      const cplx* W = pw + (size_t)ind * npw * npw * n2;
      cplx dd = 0, g1 = 0, g2 = 0, g3 = 0, h11 = 0, h22 = 0, h33 = 0, h12 = 0, h13 = 0, h23 = 0;
      for (int j3 = 1; j3 <= n2; j3++) {
        cplx d1 = 0, d1x = 0, d1y = 0, d1xx = 0, d1yy = 0, d1xy = 0;
        for (int j2 = 1; j2 <= npw; j2++) {
          cplx d2 = 0, d2x = 0, d2xx = 0;
          for (int j1 = 1; j1 <= npw; j1++) {
            const cplx wv = W[(j1 - 1) + npw * ((j2 - 1) + (size_t)npw * (j3 - 1))];
            d2 += wv * w1[j1];
            if (pgh >= 2) d2x += wv * w1x[j1];
            if (pgh >= 3) d2xx += wv * w1xx[j1];
          }
          d1 += d2 * w2[j2];
          if (pgh >= 2) { d1x += d2x * w2[j2]; d1y += d2 * w2y[j2]; }
          if (pgh >= 3) { d1xx += d2xx * w2[j2]; d1xy += d2x * w2y[j2]; d1yy += d2 * w2yy[j2]; }
        }
        dd += d1 * w3[j3];
        if (pgh >= 2) { g1 += d1x * w3[j3]; g2 += d1y * w3[j3]; g3 += d1 * w3z[j3]; }
        if (pgh >= 3) {
          h11 += d1xx * w3[j3]; h22 += d1yy * w3[j3]; h12 += d1xy * w3[j3];
          h13 += d1x * w3z[j3]; h23 += d1y * w3z[j3]; h33 += d1 * w3zz[j3];
        }
      }
      pot[nd * it + ind] += dd.real() * 2;
      if (pgh >= 2) {
        cplx g[3] = {g1, g2, g3};
        for (int k = 0; k < 3; k++) grad[ind + nd * (k + 3 * (size_t)it)] += g[k].real() * 2;
      }
      if (pgh >= 3) {
        cplx h[6] = {h11, h22, h33, h12, h13, h23};
        for (int k = 0; k < 6; k++) hess[ind + nd * (k + 6 * (size_t)it)] += h[k].real() * 2;
      }
    }
  }
}
// g3dformlc_vec, g3drouts.f:784-850.  The reference assigns the z offset to y
// at g3drouts.f:810 (so its z offset is never set); the intended tensor
// product x,y,z is restated here.
void g3dformlc(int nd, double delta, const double* src, int ns, const double* chg,
               const double* cent, int p, double* local) {
  int P = p + 1;
  double dsq = 1.0 / std::sqrt(delta);
  std::vector<double> hx(P + 1), hy(P + 1), hz(P + 1);
  for (int i = 0; i < ns; i++) {
    double x = (src[3 * i] - cent[0]) * dsq, y = (src[3 * i + 1] - cent[1]) * dsq,
           z = (src[3 * i + 2] - cent[2]) * dsq;
    double fx = std::exp(-x * x), fy = std::exp(-y * y), fz = std::exp(-z * z);
    hx[0] = fx; hy[0] = fy; hz[0] = fz;
    hx[1] = 2 * x * fx; hy[1] = 2 * y * fy; hz[1] = 2 * z * fz;
    for (int j = 1; j <= p - 1; j++) {
      hx[j + 1] = 2.0 * (x * hx[j] - hx[j - 1]) / (j + 1);
      hy[j + 1] = 2.0 * (y * hy[j] - hy[j - 1]) / (j + 1);
      hz[j + 1] = 2.0 * (z * hz[j] - hz[j - 1]) / (j + 1);
    }
    for (int ind = 0; ind < nd; ind++) {
      double q = chg[nd * i + ind];
      double* Lo = local + (size_t)ind * P * P * P;
      for (int j1 = 0; j1 <= p; j1++) {
        double zt = q * hz[j1];
        for (int j2 = 0; j2 <= p; j2++) {
          double yt = zt * hy[j2];
          for (int j3 = 0; j3 <= p; j3++) Lo[j3 + P * (j2 + (size_t)P * j1)] += yt * hx[j3];
        }
      }
    }
  }
}
// Dipole terms of g3dformld_vec / g3dformlcd_vec (g3drouts.f:857-1040)
void g3dformld_add(int nd, double delta, const double* src, int ns, const double* rn,
                   const double* ds, const double* cent, int p, double* local) {
  int P = p + 1;
  double dsq = 1.0 / std::sqrt(delta);
  std::vector<double> h[3], dh[3];
  for (int d = 0; d < 3; d++) { h[d].resize(P + 1); dh[d].resize(P); }
  for (int i = 0; i < ns; i++) {
    for (int d = 0; d < 3; d++) {
      double v = (src[3 * i + d] - cent[d]) * dsq, f = std::exp(-v * v);
      h[d][0] = f;
      h[d][1] = 2.0 * v * f;
      for (int j = 1; j <= p; j++) h[d][j + 1] = 2.0 * (v * h[d][j] - h[d][j - 1]) / (j + 1);
      for (int j = 0; j <= p; j++) dh[d][j] = -h[d][j + 1] * dsq * (j + 1.0);
    }
    for (int ind = 0; ind < nd; ind++) {
      double r1 = rn[3 * i] * ds[nd * i + ind], r2 = rn[3 * i + 1] * ds[nd * i + ind],
             r3 = rn[3 * i + 2] * ds[nd * i + ind];
      double* Lo = local + (size_t)ind * P * P * P;
      for (int j1 = 0; j1 <= p; j1++) {
        double z1 = h[2][j1] * r1, z2 = h[2][j1] * r2, z3 = dh[2][j1] * r3;
        for (int j2 = 0; j2 <= p; j2++) {
          double c1 = h[1][j2] * z1, c2 = dh[1][j2] * z2 + h[1][j2] * z3;
          for (int j3 = 0; j3 <= p; j3++) Lo[j3 + P * (j2 + (size_t)P * j1)] += dh[0][j3] * c1 + h[0][j3] * c2;
        }
      }
    }
  }
}

// g2d_directcp/cg/ch_vec (g2ddirect.f:32-212) / g3d_directcp/cg/ch_vec
// (g3ddirect.f:3-203): pot (pgh = 1), + grad (2), + Hessian (3) with
// rfac = -2/delta, d_x = rfac dx, d_xx = rfac + d_x^2, d_xy = d_x d_y.
// Hessian order 2D xx, xy, yy; 3D xx, yy, zz, xy, xz, yz.
template <int D>
void directc(int nd, double delta, double dmax, const double* src, int ns, const double* chg,
             const double* trg, int nt, int pgh, double* pot, double* grad, double* hess) {
  const int NH = D == 2 ? 3 : 6;
  const double rfac = -2.0 / delta;
  for (int it = 0; it < nt; it++)
    for (int i = 0; i < ns; i++) {
      double rr = 0, df[3] = {0, 0, 0};
      for (int d = 0; d < D; d++) {
        df[d] = trg[D * it + d] - src[D * i + d];
        rr += df[d] * df[d];
      }
      if (rr < dmax) {
        double r = std::exp(-rr / delta);
        double g[3], h[6];
        for (int d = 0; d < D; d++) g[d] = rfac * df[d];
        if (D == 2) {
          h[0] = rfac + g[0] * g[0]; h[1] = g[0] * g[1]; h[2] = rfac + g[1] * g[1];
        } else {
          h[0] = rfac + g[0] * g[0]; h[1] = rfac + g[1] * g[1]; h[2] = rfac + g[2] * g[2];
          h[3] = g[0] * g[1]; h[4] = g[0] * g[2]; h[5] = g[1] * g[2];
        }
        for (int ii = 0; ii < nd; ii++) {
          double v = r * chg[nd * i + ii];
#pragma omp atomic
          pot[nd * it + ii] += v;
          if (pgh >= 2)
            for (int d = 0; d < D; d++) {
              double w = g[d] * v;
#pragma omp atomic
              grad[ii + nd * (d + D * (size_t)it)] += w;
            }
          if (pgh >= 3)
            for (int c = 0; c < NH; c++) {
              double w = h[c] * v;
#pragma omp atomic
              hess[ii + nd * (c + NH * (size_t)it)] += w;
            }
        }
      }
    }
}

// Dipole terms of g2d_directd{p,g,h}_vec / g2d_directcd{p,g,h}_vec
// (g2ddirect.f:217-658) and g3d_directd*/cd*_vec (g3ddirect.f:207-708):
// with R = 2/delta, u = R (t - s), rinc = u.n,
//   pot  += rinc e dipstr,  grad_a += (R n_a - rinc u_a) e dipstr,
//   hess_aa += (-R (u_a n_a + rinc) - g_a u_a) e dipstr,
//   hess_ab += (-R u_a n_b - g_a u_b) e dipstr   (g_a the grad factor).
template <int D>
void directd(int nd, double delta, double dmax, const double* src, int ns, const double* rn,
             const double* ds, const double* trg, int nt, int pgh, double* pot, double* grad,
             double* hess) {
  const int NH = D == 2 ? 3 : 6;
  const double R = 2.0 / delta;
  for (int it = 0; it < nt; it++)
    for (int i = 0; i < ns; i++) {
      double rr = 0, df[3] = {0, 0, 0};
      for (int d = 0; d < D; d++) {
        df[d] = trg[D * it + d] - src[D * i + d];
        rr += df[d] * df[d];
      }
      if (!(rr < dmax)) continue;
      double e = std::exp(-rr / delta), u[3], n[3], g[3], h[6];
      double rinc = 0;
      for (int d = 0; d < D; d++) {
        u[d] = R * df[d];
        n[d] = rn[D * i + d];
        rinc += u[d] * n[d];
      }
      for (int d = 0; d < D; d++) g[d] = n[d] * R - rinc * u[d];
      auto hd = [&](int a) { return -R * (u[a] * n[a] + rinc) - g[a] * u[a]; };
      auto ho = [&](int a, int b) { return -R * u[a] * n[b] - g[a] * u[b]; };
      if (D == 2) {
        h[0] = hd(0); h[1] = ho(0, 1); h[2] = hd(1);
      } else {
        h[0] = hd(0); h[1] = hd(1); h[2] = hd(2); h[3] = ho(0, 1); h[4] = ho(0, 2); h[5] = ho(1, 2);
      }
      for (int ii = 0; ii < nd; ii++) {
        double v = e * ds[nd * i + ii];
        double w = rinc * v;
#pragma omp atomic
        pot[nd * it + ii] += w;
        if (pgh >= 2)
          for (int d = 0; d < D; d++) {
            double gv = g[d] * v;
#pragma omp atomic
            grad[ii + nd * (d + D * (size_t)it)] += gv;
          }
        if (pgh >= 3)
          for (int c = 0; c < NH; c++) {
            double hv = h[c] * v;
#pragma omp atomic
            hess[ii + nd * (c + NH * (size_t)it)] += hv;
          }
      }
    }
}

// ---------------------------------------------------------------- drivers
struct Result {
  int npwlevel = 0, nlevels = 0, nboxes = 0, npw = 0, nlmax = 0;
  double bs0 = 0;
  long long nleaf_direct = 0;
};

// Expansions of chosen boxes (0-based ids) copied out after the shifts of
// the plane-wave scheme (multipole after merge, local after split), for the
// intermediate-stage comparison with the product.
struct Probe {
  int nbox = 0;
  const int* boxes = nullptr;
  cplx* mp = nullptr;  // [nbox][nd * nexp]
  cplx* lo = nullptr;
  int* has = nullptr;  // [nbox]: 1 when the box has expansions (levels >= the cut)
};

// fgt2d (fgt2d.f:19-462) + fgt2dmain (fgt2d.f:468-1348) and the 3D twins
// (fgt3d.f:19-477, 483-1527).  Output arrays are overwritten.
//
// nufft = 1 restates the NUFFT scheme of 2d/nufft and 3d/nufft instead
// (fgt2d.f / fgt3d.f there): the tree stops one level below the cut level
// (fgt2d.f:188, fgt3d.f:192; 3D ndiv0 = 20, fgt3d.f:161), the boxes of the
// cut level with more than ndiv sources form their plane-wave expansion
// from all their sources (type-1 NUFFT there, the exact sum here), the
// expansions are shifted between cut-level colleagues, evaluated at every
// point of the cut-level boxes that have one (type-2 NUFFT there, exact
// here), and the rest is the same direct interaction.
template <int D>
int fgt_run(int nd, double delta, double eps, int ns, const double* sources, int ifcharge,
            const double* charge, int ifdipole, const double* rnormal, const double* dipstr,
            int ifpgh, double* pot, double* grad, double* hess,
            int nt, const double* targ, int ifpghtarg, double* pottarg, double* gradtarg,
            double* hesstarg, Result* res, int nufft = 0, Probe* probe = nullptr) {
  const int NCH = Tree<D>::NCH;
  const int NH = D == 2 ? 3 : 6;
  if (nd < 1 || !(delta > 0) || !(eps > 0) || ns < 0 || nt < 0) return ORC_BADARG;
  if (ifcharge < 0 || ifcharge > 1 || ifdipole < 0 || ifdipole > 1) return ORC_UNSUPPORTED;
  if (ifpgh < 0 || ifpgh > 3 || ifpghtarg < 0 || ifpghtarg > 3) return ORC_UNSUPPORTED;
  // fgt2d.f:238-322: outputs zeroed per flag
  if (ifpgh >= 1) std::fill(pot, pot + (size_t)nd * ns, 0.0);
  if (ifpgh >= 2) std::fill(grad, grad + (size_t)nd * D * ns, 0.0);
  if (ifpgh >= 3) std::fill(hess, hess + (size_t)nd * NH * ns, 0.0);
  if (ifpghtarg >= 1) std::fill(pottarg, pottarg + (size_t)nd * nt, 0.0);
  if (ifpghtarg >= 2) std::fill(gradtarg, gradtarg + (size_t)nd * D * nt, 0.0);
  if (ifpghtarg >= 3) std::fill(hesstarg, hesstarg + (size_t)nd * NH * nt, 0.0);
  if (ns == 0) return ORC_OK;

  int npwlevel;
  double bs0, cen0[3];
  boxsize0<D>(delta, eps, sources, ns, targ, nt, &npwlevel, &bs0, cen0);
  if (res) { res->npwlevel = npwlevel; res->bs0 = bs0; }

  if (npwlevel < -2) {  // fgt2d.f:133-150 / fgt3d.f:136-154, large-delta path
    int nl0 = hlterms(D, bs0, delta, eps, 0);
    nl0 = nl0 + std::max(ifpgh, ifpghtarg) - 1;
    int P = nl0 + 1;
    size_t LL = (size_t)nd * (D == 2 ? P * P : P * P * P);
    std::vector<double> local(LL, 0.0);
    if (D == 2) {
      if (ifcharge) g2dformlc(nd, delta, sources, ns, charge, cen0, nl0, local.data());
      if (ifdipole) g2dformld_add(nd, delta, sources, ns, rnormal, dipstr, cen0, nl0, local.data());
      if (ifpghtarg >= 1) g2dleval(nd, delta, cen0, nl0, local.data(), targ, nt, ifpghtarg, pottarg, gradtarg, hesstarg);
      if (ifpgh >= 1) g2dleval(nd, delta, cen0, nl0, local.data(), sources, ns, ifpgh, pot, grad, hess);
    } else {
      if (ifcharge) g3dformlc(nd, delta, sources, ns, charge, cen0, nl0, local.data());
      if (ifdipole) g3dformld_add(nd, delta, sources, ns, rnormal, dipstr, cen0, nl0, local.data());
      if (ifpghtarg >= 1) g3dleval(nd, delta, cen0, nl0, local.data(), targ, nt, ifpghtarg, pottarg, gradtarg, hesstarg);
      if (ifpgh >= 1) g3dleval(nd, delta, cen0, nl0, local.data(), sources, ns, ifpgh, pot, grad, hess);
    }
    return ORC_OK;
  }

  if (nufft && D == 2 && ifdipole) return ORC_UNSUPPORTED;
  const int ndiv0 = D == 2 ? 10 : (nufft ? 20 : 40), ndiv = D == 2 ? 80 : 100, hcap = D == 2 ? 18 : 15;
  int nlmax = npwlevel + 4;
  int nlevstart = std::max(npwlevel, 0);
  double bsize = bs0 / (double)(1 << nlevstart);
  int nlocal0 = 0;
  for (int i = nlevstart; i <= 100; i++) {
    nlocal0 = hlterms(D, bsize, delta, eps, nlocal0);
    if (nlocal0 <= hcap) { nlmax = i; break; }
    bsize = bsize / 2;
  }
  if (nufft && npwlevel >= 0) nlmax = npwlevel + 1;
  Tree<D> t;
  std::vector<int> isrc, isrcse, itarg, itargse;
  build_tree<D>(t, sources, ns, targ, nt, ndiv, ndiv0, npwlevel, nlmax, bs0, cen0, isrc, isrcse,
                itarg, itargse);
  int nlevels = t.nlevels, nboxes = t.nboxes;
  if (res) { res->nlevels = nlevels; res->nboxes = nboxes; res->nlmax = nlmax; }

  std::vector<int> nlocal(nlevels + 1, 0);
  int nadd = ifdipole + std::max(ifpgh, ifpghtarg);
  for (int i = std::max(npwlevel, 0); i <= nlevels; i++) {
    nlocal[i] = hlterms(D, t.boxsize[i], delta, eps, nlocal[i]);
    if (ifdipole == 1 || ifpgh >= 2 || ifpghtarg >= 2) nlocal[i] += nadd;
  }
  int ntermmax = 0;
  for (int i = 0; i <= nlevels; i++) ntermmax = std::max(ntermmax, nlocal[i]);
  double pmax;
  int npw;
  {
    double bsz = 2 * bs0 / std::pow(2.0, std::max(npwlevel, 0));
    double pweps = eps;
    if (nadd > 2) pweps = pweps / 100;
    pwterms(bsz, delta, pweps, &pmax, &npw);
  }
  if (res) res->npw = npw;

  // dreorderf
  std::vector<double> ssort((size_t)D * ns), csort((size_t)nd * ns), tsort((size_t)D * nt);
  std::vector<double> rsort(ifdipole ? (size_t)D * ns : 0), dsort(ifdipole ? (size_t)nd * ns : 0);
  for (int i = 0; i < ns; i++) {
    const size_t o = isrc[i + 1] - 1;
    for (int d = 0; d < D; d++) ssort[(size_t)D * i + d] = sources[(size_t)D * o + d];
    if (ifcharge)
      for (int k = 0; k < nd; k++) csort[(size_t)nd * i + k] = charge[(size_t)nd * o + k];
    if (ifdipole) {
      for (int d = 0; d < D; d++) rsort[(size_t)D * i + d] = rnormal[(size_t)D * o + d];
      for (int k = 0; k < nd; k++) dsort[(size_t)nd * i + k] = dipstr[(size_t)nd * o + k];
    }
  }
  for (int i = 0; i < nt; i++)
    for (int d = 0; d < D; d++) tsort[(size_t)D * i + d] = targ[(size_t)D * (itarg[i + 1] - 1) + d];
  std::vector<double> psort((size_t)nd * ns, 0.0), ptsort((size_t)nd * nt, 0.0);
  std::vector<double> gsort(ifpgh >= 2 ? (size_t)nd * D * ns : 0, 0.0),
      hsort(ifpgh >= 3 ? (size_t)nd * NH * ns : 0, 0.0),
      gtsort(ifpghtarg >= 2 ? (size_t)nd * D * nt : 0, 0.0),
      htsort(ifpghtarg >= 3 ? (size_t)nd * NH * nt : 0, 0.0);
  // sorted output pointers of the points from index i of either set
  auto PT = [&](int i) { return ptsort.data() + (size_t)nd * i; };
  auto GT = [&](int i) { return gtsort.data() + (size_t)nd * D * i; };
  auto HT = [&](int i) { return htsort.data() + (size_t)nd * NH * i; };
  auto PS = [&](int i) { return psort.data() + (size_t)nd * i; };
  auto GS = [&](int i) { return gsort.data() + (size_t)nd * D * i; };
  auto HS = [&](int i) { return hsort.data() + (size_t)nd * NH * i; };

  auto NS = [&](int b) { return isrcse[2 * b + 1] - isrcse[2 * b] + 1; };
  auto NT = [&](int b) { return itargse[2 * b + 1] - itargse[2 * b] + 1; };
  auto S0 = [&](int b) { return isrcse[2 * b] - 1; };   // 0-based first source
  auto T0 = [&](int b) { return itargse[2 * b] - 1; };

  // ---- fgt2dmain
  int nlevend = (npwlevel < nlevels) ? npwlevel : nlevels;
  std::vector<int> ifhung(nboxes + 1, 0);
  for (int ilev = 0; ilev <= nlevend; ilev++)
    for (int ibox = t.L(ilev, 0); ibox <= t.L(ilev, 1); ibox++)
      if (t.nchild[ibox] == 0 && NS(ibox) > 0 && (!nufft || NS(ibox) <= ndiv)) ifhung[ibox] = 1;
  std::vector<std::vector<int>> list1;
  if constexpr (D == 2) modified_list1_2d(t, npwlevel, list1);
  else modified_list1_3d(t, npwlevel, list1);

  if (npwlevel < nlevels) {
    std::vector<double> ws, ts;
    if (D == 2) pwnodes_2d(pmax, npw, ws, ts); else pwnodes_3d(pmax, npw, ws, ts);
    int n2 = npw / 2;
    size_t nexp = D == 2 ? (size_t)npw * npw / 2 : (size_t)npw * npw * npw / 2;
    cplx eye(0, 1);
    // pw_translation_matrices (nmax = 1), g2drouts.f:2235 / g3drouts.f:2697
    // index (jx+1) + 3 (jy+1) [+ 9 (jz+1)]
    int n3 = D == 2 ? 9 : 27;
    std::vector<cplx> wsh(nexp * n3);
    {
      double xmin = (npwlevel >= 0 ? t.boxsize[npwlevel] : 0.0) / std::sqrt(delta);
      std::vector<cplx> ww((size_t)(npw + 1) * 3);
      for (int j = 1; j <= npw; j++) {
        cplx z = std::exp(eye * ts[j] * xmin);
        ww[3 * j + 1] = 1.0;
        ww[3 * j + 2] = z;
        ww[3 * j + 0] = std::conj(z);
      }
      for (int s = 0; s < n3; s++) {
        int kx = s % 3, ky = (s / 3) % 3, kz = s / 9;
        cplx* W = wsh.data() + nexp * s;
        if (D == 2) {
          for (int j1 = 1; j1 <= npw; j1++)
            for (int j2 = 1; j2 <= n2; j2++) W[(j2 - 1) + n2 * (j1 - 1)] = ww[3 * j2 + kx] * ww[3 * j1 + ky];
        } else {
          size_t j = 0;
          for (int j1 = 1; j1 <= n2; j1++)
            for (int j2 = 1; j2 <= npw; j2++)
              for (int j3 = 1; j3 <= npw; j3++) W[j++] = ww[3 * j3 + kx] * ww[3 * j2 + ky] * ww[3 * j1 + kz];
        }
      }
    }
    // merge_split_pw_matrices, g2drouts.f:2294-2350 / g3drouts.f:2760-2840
    int nmaxms = nlevels - std::max(npwlevel, 0);
    std::vector<cplx> wms(nexp * NCH * std::max(nmaxms, 1));
    {
      double xmin2 = t.boxsize[nlevels] / std::sqrt(delta) / 2;
      std::vector<cplx> ww((size_t)(npw + 1) * (nmaxms + 1));
      for (int j = 1; j <= npw; j++) {
        cplx z = std::exp(eye * ts[j] * xmin2);
        for (int k = 1; k <= nmaxms; k++) { ww[(size_t)j * (nmaxms + 1) + k] = z; z = z * z; }
      }
      auto W1 = [&](int j, int k, bool m) { cplx v = ww[(size_t)j * (nmaxms + 1) + k]; return m ? std::conj(v) : v; };
      for (int k = 1; k <= nmaxms; k++)
        for (int q = 1; q <= NCH; q++) {
          // quadrant q: 2D 1 pp, 2 pm, 3 mp, 4 mm (x then y); 3D adds z (1-4 p, 5-8 m)
          bool mx = (q - 1) & 2, my = (q - 1) & 1, mz = (q - 1) & 4;
          cplx* W = wms.data() + nexp * ((q - 1) + (size_t)NCH * (k - 1));
          if (D == 2) {
            for (int j1 = 1; j1 <= npw; j1++)
              for (int j2 = 1; j2 <= n2; j2++) W[(j2 - 1) + n2 * (j1 - 1)] = W1(j2, k, mx) * W1(j1, k, my);
          } else {
            size_t j = 0;
            for (int j1 = 1; j1 <= n2; j1++)
              for (int j2 = 1; j2 <= npw; j2++)
                for (int j3 = 1; j3 <= npw; j3++) W[j++] = W1(j3, k, mx) * W1(j2, k, my) * W1(j1, k, mz);
          }
        }
    }
    // 1D matrices rh2x, rx2l (g2drouts.f:1645,1731; g3drouts.f:3019,3106)
    std::vector<double> rh2x((size_t)npw * (ntermmax + 1)), rx2l((size_t)npw * (ntermmax + 1));
    {
      std::vector<double> fac(ntermmax + 1), fac2(ntermmax + 1);
      fac[0] = 1; fac2[0] = 1;
      for (int i = 1; i <= ntermmax; i++) { fac[i] = fac[i - 1] / std::sqrt((double)i); fac2[i] = fac2[i - 1] * i; }
      for (int j = 0; j <= ntermmax; j++)
        for (int i = 1; i <= npw; i++) {
          double hv = ws[i] * powi(-ts[i], j) * fac[j];
          if (D == 2) rh2x[(i - 1) + (size_t)npw * j] = hv;
          else rh2x[j + (size_t)(ntermmax + 1) * (i - 1)] = hv;
          rx2l[(i - 1) + (size_t)npw * j] = powi(ts[i], j) / fac2[j];
        }
    }
    // iflocal (fgt2d.f:790-814)
    std::vector<int> iflocal(nboxes + 1, 0);
    if (npwlevel >= 0 && npwlevel <= nlevels)
      for (int jbox = t.L(npwlevel, 0); jbox <= t.L(npwlevel, 1); jbox++)
        if (t.nchild[jbox] == 0)
          for (int i = 0; i < t.nnbors[jbox]; i++)
            if (t.nchild[t.nbors[(size_t)jbox * Tree<D>::NCO + i]] > 0) { iflocal[jbox] = 1; break; }
    std::vector<std::vector<int>> lpw;
    if constexpr (D == 2) listpw_2d(t, npwlevel, lpw);
    else listpw_3d(t, npwlevel, lpw);
    // g2dmpalloc (fgt2d.f:1518-1610): mp then loc blocks, levels nlevstart..nlevels
    std::vector<long long> iaddr(2 * (nboxes + 1), -1);
    long long pos = 0;
    for (int pass = 0; pass < 2; pass++)
      for (int i = nlevstart; i <= nlevels; i++)
        for (int ibox = t.L(i, 0); ibox <= t.L(i, 1); ibox++) { iaddr[2 * ibox + pass] = pos; pos += (long long)nexp * nd; }
    std::vector<cplx> rml(pos, cplx(0, 0));
    auto MP = [&](int b) { return rml.data() + iaddr[2 * b]; };
    auto LO = [&](int b) { return rml.data() + iaddr[2 * b + 1]; };
    auto shift = [&](const cplx* a, cplx* b, const cplx* w) {
      for (int ind = 0; ind < nd; ind++)
        for (size_t j = 0; j < nexp; j++) b[ind * nexp + j] += a[ind * nexp + j] * w[j];
    };
    if (nufft) {
      // NUFFT scheme, steps 1-3 at the cut level (the level of the cut when
      // it is >= 0; the reference leaves npwlevel in {-2, -1} undefined, the
      // root level is used here)
      const int lc = nlevstart;
      const double xmin = t.boxsize[lc];
      auto big = [&](int b) { return NS(b) > ndiv; };
      // listpw of the NUFFT scheme: the cut level's colleagues with children
      // (2d/nufft/src/common/tree_routs4.f:940-953, tree_routs3d.f gt3d_computelistpw)
      auto lpwn = [&](int ibox) {
        std::vector<int> v;
        for (int i = 0; i < t.nnbors[ibox]; i++) {
          int jbox = t.nbors[(size_t)ibox * Tree<D>::NCO + i];
          if (jbox != ibox && t.nchild[jbox] > 0) v.push_back(jbox);
        }
        return v;
      };
      // step 1 (fgt2d.f:824-900 / fgt3d.f:860-960): form, and the copy into
      // the box's own local expansion
#pragma omp parallel for schedule(dynamic)
      for (int ibox = t.L(lc, 0); ibox <= t.L(lc, 1); ibox++) {
        if (!big(ibox)) continue;
        const double* sp = ssort.data() + (size_t)D * S0(ibox);
        const double* q = csort.data() + (size_t)nd * S0(ibox);
        const double* c = &t.centers[(size_t)D * ibox];
        if (D == 2) {
          g2dformpwc(nd, delta, sp, NS(ibox), q, c, npw, ws.data(), ts.data(), MP(ibox));
        } else {
          if (ifcharge) g3dformpwc(nd, delta, sp, NS(ibox), q, c, npw, ws.data(), ts.data(), MP(ibox));
          if (ifdipole)
            g3dformpwd_add(nd, delta, sp, NS(ibox), rsort.data() + (size_t)D * S0(ibox),
                           dsort.data() + (size_t)nd * S0(ibox), c, npw, ws.data(), ts.data(), MP(ibox));
        }
        for (size_t j = 0; j < (size_t)nd * nexp; j++) LO(ibox)[j] += MP(ibox)[j];
      }
      // step 2 (fgt2d.f:918-958 / fgt3d.f:990-1030): shifts from the colleagues
#pragma omp parallel for schedule(dynamic)
      for (int ibox = t.L(lc, 0); ibox <= t.L(lc, 1); ibox++) {
        int npts = 0;
        if (ifpghtarg > 0) npts += NT(ibox);
        if (ifpgh > 0) npts += NS(ibox);
        if (npts <= 0) continue;
        for (int jbox : lpwn(ibox)) {
          if (!big(jbox)) continue;
          int jx = (int)std::lround((t.c(ibox, 0) - t.c(jbox, 0)) / xmin);
          int jy = (int)std::lround((t.c(ibox, 1) - t.c(jbox, 1)) / xmin);
          int jz = D == 3 ? (int)std::lround((t.c(ibox, 2) - t.c(jbox, 2)) / xmin) : -1;
          shift(MP(jbox), LO(ibox), wsh.data() + nexp * ((jx + 1) + 3 * (jy + 1) + 9 * (jz + 1)));
        }
      }
      // step 3 (fgt2d.f:973-1047 / fgt3d.f:1045-1130): evaluation at every
      // point of the boxes with a listpw entry or an expansion of their own
#pragma omp parallel for schedule(dynamic)
      for (int ibox = t.L(lc, 0); ibox <= t.L(lc, 1); ibox++) {
        if (lpwn(ibox).empty() && !big(ibox)) continue;
        const double* c = &t.centers[(size_t)D * ibox];
        const int i0 = T0(ibox), j0 = S0(ibox), nts = NT(ibox), nss = NS(ibox);
        if (nts > 0 && ifpghtarg >= 1) {
          if (D == 2) g2dpweval(nd, delta, c, npw, ts.data(), LO(ibox), tsort.data() + 2 * (size_t)i0, nts, ifpghtarg, PT(i0), GT(i0), HT(i0));
          else g3dpweval(nd, delta, c, npw, ts.data(), LO(ibox), tsort.data() + 3 * (size_t)i0, nts, ifpghtarg, PT(i0), GT(i0), HT(i0));
        }
        if (nss > 0 && ifpgh >= 1) {
          if (D == 2) g2dpweval(nd, delta, c, npw, ts.data(), LO(ibox), ssort.data() + 2 * (size_t)j0, nss, ifpgh, PS(j0), GS(j0), HS(j0));
          else g3dpweval(nd, delta, c, npw, ts.data(), LO(ibox), ssort.data() + 3 * (size_t)j0, nss, ifpgh, PS(j0), GS(j0), HS(j0));
        }
      }
    } else {
    // step 1: form mp (fgt2d.f:871-959 / fgt3d.f:899-1098)
    for (int ilev = nlevels; ilev >= std::max(npwlevel + 1, 0); ilev--) {
      int p = nlocal[ilev], P = p + 1;
      int nptsswitch = 0;
      if (D == 3) {
        double r1 = (p + 1.0) / npw, r2 = r1 * r1, r3 = r1 * r2;
        nptsswitch = (r3 >= 3) ? 1000000 : 0;
      }
      std::vector<double> rh2xt;
      if (D == 3) {
        rh2xt.resize((size_t)P * npw);
        for (int j1 = 1; j1 <= npw; j1++)
          for (int j2 = 0; j2 <= p; j2++) rh2xt[j2 + (size_t)P * (j1 - 1)] = rh2x[j2 + (size_t)(ntermmax + 1) * (j1 - 1)];
      }
#pragma omp parallel for schedule(dynamic)
      for (int ibox = t.L(ilev, 0); ibox <= t.L(ilev, 1); ibox++) {
        int npts = NS(ibox);
        if (t.nchild[ibox] != 0 || npts <= 0) continue;
        const double* s = ssort.data() + (size_t)D * S0(ibox);
        const double* q = csort.data() + (size_t)nd * S0(ibox);
        const double* rn = rsort.data() + (size_t)D * S0(ibox);
        const double* dp = dsort.data() + (size_t)nd * S0(ibox);
        const double* c = &t.centers[(size_t)D * ibox];
        // g2dformhc/hd/hcd_vec by ifcharge/ifdipole (fgt2d.f:882-954)
        if (D == 2) {
          std::vector<double> hexp((size_t)P * P * nd, 0.0);
          if (ifcharge) g2dformhc(nd, delta, s, npts, q, c, p, hexp.data());
          if (ifdipole) g2dformhd_add(nd, delta, s, npts, rn, dp, c, p, hexp.data());
          g2dh2pw(nd, p, npw, rh2x.data(), hexp.data(), MP(ibox));
        } else if (npts > nptsswitch) {
          std::vector<double> hexp((size_t)P * P * P * nd, 0.0);
          if (ifcharge) g3dformhc(nd, delta, s, npts, q, c, p, hexp.data());
          if (ifdipole) g3dformhd_add(nd, delta, s, npts, rn, dp, c, p, hexp.data());
          g3dh2pw(nd, p, npw, rh2xt.data(), hexp.data(), MP(ibox));
        } else {
          if (ifcharge) g3dformpwc(nd, delta, s, npts, q, c, npw, ws.data(), ts.data(), MP(ibox));
          if (ifdipole) g3dformpwd_add(nd, delta, s, npts, rn, dp, c, npw, ws.data(), ts.data(), MP(ibox));
        }
      }
    }
    // step 2: merge mp (fgt2d.f:976-1009 / fgt3d.f:1114-1155)
    for (int ilev = nlevels - 1; ilev >= nlevstart; ilev--) {
#pragma omp parallel for schedule(dynamic)
      for (int ibox = t.L(ilev, 0); ibox <= t.L(ilev, 1); ibox++)
        for (int i = 1; i <= t.nchild[ibox]; i++) {
          int jbox = t.ch(ibox, i);
          if (NS(jbox) <= 0) continue;
          int q = 0;
          double dx = t.c(ibox, 0) - t.c(jbox, 0), dy = t.c(ibox, 1) - t.c(jbox, 1);
          double dz = D == 3 ? t.c(ibox, 2) - t.c(jbox, 2) : 1.0;
          if (dx > 0 && dy > 0 && dz > 0) q = 1;
          else if (dx > 0 && dy < 0 && dz > 0) q = 2;
          else if (dx < 0 && dy > 0 && dz > 0) q = 3;
          else if (dx < 0 && dy < 0 && dz > 0) q = 4;
          else if (dx > 0 && dy > 0 && dz < 0) q = 5;
          else if (dx > 0 && dy < 0 && dz < 0) q = 6;
          else if (dx < 0 && dy > 0 && dz < 0) q = 7;
          else if (dx < 0 && dy < 0 && dz < 0) q = 8;
          shift(MP(jbox), MP(ibox), wms.data() + nexp * ((q - 1) + (size_t)NCH * (nlevels - ilev - 1)));
        }
    }
    // step 3: mp to loc at the cut level (fgt2d.f:1026-1064 / fgt3d.f:1172-1209)
    {
      double xmin = npwlevel >= 0 ? t.boxsize[npwlevel] : 1.0;
      int ilev = nlevstart;
#pragma omp parallel for schedule(dynamic)
      for (int ibox = t.L(ilev, 0); ibox <= t.L(ilev, 1); ibox++) {
        int npts = 0;
        if (ifpghtarg > 0) npts += NT(ibox);
        if (ifpgh > 0) npts += NS(ibox);
        if (npts <= 0) continue;
        for (int jbox : lpw[ibox]) {
          int jx = (int)std::lround((t.c(ibox, 0) - t.c(jbox, 0)) / xmin);
          int jy = (int)std::lround((t.c(ibox, 1) - t.c(jbox, 1)) / xmin);
          int jz = D == 3 ? (int)std::lround((t.c(ibox, 2) - t.c(jbox, 2)) / xmin) : -1;
          int s = (jx + 1) + 3 * (jy + 1) + 9 * (jz + 1);
          shift(MP(jbox), LO(ibox), wsh.data() + nexp * s);
        }
        for (int ind = 0; ind < nd; ind++)
          for (size_t j = 0; j < nexp; j++) LO(ibox)[ind * nexp + j] += MP(ibox)[ind * nexp + j];
      }
    }
    // step 4: split loc (fgt2d.f:1082-1125 / fgt3d.f:1227-1276)
    for (int ilev = nlevstart; ilev <= nlevels - 1; ilev++) {
#pragma omp parallel for schedule(dynamic)
      for (int ibox = t.L(ilev, 0); ibox <= t.L(ilev, 1); ibox++) {
        int npts = 0;
        if (ifpghtarg > 0) npts += NT(ibox);
        if (ifpgh > 0) npts += NS(ibox);
        if (npts <= 0) continue;
        for (int i = 1; i <= t.nchild[ibox]; i++) {
          int jbox = t.ch(ibox, i);
          int q = 0;
          double dx = t.c(jbox, 0) - t.c(ibox, 0), dy = t.c(jbox, 1) - t.c(ibox, 1);
          double dz = D == 3 ? t.c(jbox, 2) - t.c(ibox, 2) : 1.0;
          if (dx > 0 && dy > 0 && dz > 0) q = 1;
          else if (dx > 0 && dy < 0 && dz > 0) q = 2;
          else if (dx < 0 && dy > 0 && dz > 0) q = 3;
          else if (dx < 0 && dy < 0 && dz > 0) q = 4;
          else if (dx > 0 && dy > 0 && dz < 0) q = 5;
          else if (dx > 0 && dy < 0 && dz < 0) q = 6;
          else if (dx < 0 && dy > 0 && dz < 0) q = 7;
          else if (dx < 0 && dy < 0 && dz < 0) q = 8;
          shift(LO(ibox), LO(jbox), wms.data() + nexp * ((q - 1) + (size_t)NCH * (nlevels - ilev - 1)));
        }
      }
    }
    if (probe)
      for (int i = 0; i < probe->nbox; i++) {
        const int b = probe->boxes[i] + 1;
        const bool ok = b >= 1 && b <= nboxes && iaddr[2 * b] >= 0;
        probe->has[i] = ok;
        if (!ok) continue;
        std::copy(MP(b), MP(b) + (size_t)nd * nexp, probe->mp + (size_t)i * nd * nexp);
        std::copy(LO(b), LO(b) + (size_t)nd * nexp, probe->lo + (size_t)i * nd * nexp);
      }
    // step 5: evaluate (fgt2d.f:1141-1271 / fgt3d.f:1283-1446)
    for (int ilev = nlevstart; ilev <= nlevels; ilev++) {
      int p = nlocal[ilev], P = p + 1;
      bool pweval;
      if (D == 2) {
        pweval = p > 50;  // nlocalswitch, fgt2d.f:855
      } else {
        double r1 = (p + 1.0) / npw, r2 = r1 * r1, r3 = r1 * r2;
        pweval = r3 >= 3;  // nptsswitch 1e6 vs 0, fgt3d.f:1302-1311
      }
#pragma omp parallel for schedule(dynamic)
      for (int ibox = t.L(ilev, 0); ibox <= t.L(ilev, 1); ibox++) {
        if (ilev == npwlevel && iflocal[ibox] == 0) continue;
        if (t.nchild[ibox] != 0) continue;
        int nts = NT(ibox), nss = NS(ibox);
        if (nts + nss <= 0) continue;
        const double* c = &t.centers[(size_t)D * ibox];
        bool usepw = pweval && (D == 2 || nts + nss < 1000000);
        if (usepw) {
          const int i0 = T0(ibox), j0 = S0(ibox);
          if (nts > 0 && ifpghtarg >= 1) {
            if (D == 2) g2dpweval(nd, delta, c, npw, ts.data(), LO(ibox), tsort.data() + 2 * (size_t)i0, nts, ifpghtarg, PT(i0), GT(i0), HT(i0));
            else g3dpweval(nd, delta, c, npw, ts.data(), LO(ibox), tsort.data() + 3 * (size_t)i0, nts, ifpghtarg, PT(i0), GT(i0), HT(i0));
          }
          if (nss > 0 && ifpgh >= 1) {
            if (D == 2) g2dpweval(nd, delta, c, npw, ts.data(), LO(ibox), ssort.data() + 2 * (size_t)j0, nss, ifpgh, PS(j0), GS(j0), HS(j0));
            else g3dpweval(nd, delta, c, npw, ts.data(), LO(ibox), ssort.data() + 3 * (size_t)j0, nss, ifpgh, PS(j0), GS(j0), HS(j0));
          }
        } else {
          std::vector<double> local((size_t)nd * (D == 2 ? P * P : P * P * P));
          if (D == 2) g2dpw2local(nd, p, npw, rx2l.data(), LO(ibox), local.data());
          else g3dpw2local(nd, p, npw, rx2l.data(), LO(ibox), local.data());
          const int i0 = T0(ibox), j0 = S0(ibox);
          if (nts > 0 && ifpghtarg >= 1) {
            if (D == 2) g2dleval(nd, delta, c, p, local.data(), tsort.data() + 2 * (size_t)i0, nts, ifpghtarg, PT(i0), GT(i0), HT(i0));
            else g3dleval(nd, delta, c, p, local.data(), tsort.data() + 3 * (size_t)i0, nts, ifpghtarg, PT(i0), GT(i0), HT(i0));
          }
          if (nss > 0 && ifpgh >= 1) {
            if (D == 2) g2dleval(nd, delta, c, p, local.data(), ssort.data() + 2 * (size_t)j0, nss, ifpgh, PS(j0), GS(j0), HS(j0));
            else g3dleval(nd, delta, c, p, local.data(), ssort.data() + 3 * (size_t)j0, nss, ifpgh, PS(j0), GS(j0), HS(j0));
          }
        }
      }
    }
    }  // plane-wave scheme
  }
  // step 6: direct (fgt2d.f:1287-1333, cutoff eps/90; fgt3d.f:1466-1512, cutoff eps)
  {
    double dmax = D == 2 ? std::log(1.0 / (eps / 90)) * delta : std::log(1.0 / eps) * delta;
    long long nhung = 0;
    for (int ilev = 0; ilev <= nlevend; ilev++) {
#pragma omp parallel for schedule(dynamic) reduction(+ : nhung)
      for (int jbox = t.L(ilev, 0); jbox <= t.L(ilev, 1); jbox++) {
        if (ifhung[jbox] != 1) continue;
        nhung++;
        const double* s = ssort.data() + (size_t)D * S0(jbox);
        const double* q = csort.data() + (size_t)nd * S0(jbox);
        const double* rn = rsort.data() + (size_t)D * S0(jbox);
        const double* dp = dsort.data() + (size_t)nd * S0(jbox);
        int nsj = NS(jbox);
        // fgt2dpart_direct_vec: charge and dipole terms (fgt2d.f:1354-1512)
        for (int ibox : list1[jbox]) {
          const int i0 = T0(ibox), j0 = S0(ibox);
          if (NT(ibox) > 0 && ifpghtarg >= 1) {
            const double* tp = tsort.data() + (size_t)D * i0;
            if (ifcharge) directc<D>(nd, delta, dmax, s, nsj, q, tp, NT(ibox), ifpghtarg, PT(i0), GT(i0), HT(i0));
            if (ifdipole) directd<D>(nd, delta, dmax, s, nsj, rn, dp, tp, NT(ibox), ifpghtarg, PT(i0), GT(i0), HT(i0));
          }
          if (NS(ibox) > 0 && ifpgh >= 1) {
            const double* sp = ssort.data() + (size_t)D * j0;
            if (ifcharge) directc<D>(nd, delta, dmax, s, nsj, q, sp, NS(ibox), ifpgh, PS(j0), GS(j0), HS(j0));
            if (ifdipole) directd<D>(nd, delta, dmax, s, nsj, rn, dp, sp, NS(ibox), ifpgh, PS(j0), GS(j0), HS(j0));
          }
        }
      }
    }
    if (res) res->nleaf_direct = nhung;
  }
  // dreorderi: un-permute outputs
  // (dreorderi / dreorderiv, fgt2d.f:430-458)
  auto unsort = [&](int n, const std::vector<int>& perm, int w, const std::vector<double>& in, double* out) {
    for (int i = 0; i < n; i++)
      for (int k = 0; k < w; k++) out[(size_t)w * (perm[i + 1] - 1) + k] = in[(size_t)w * i + k];
  };
  if (ifpgh >= 1) unsort(ns, isrc, nd, psort, pot);
  if (ifpgh >= 2) unsort(ns, isrc, nd * D, gsort, grad);
  if (ifpgh >= 3) unsort(ns, isrc, nd * NH, hsort, hess);
  if (ifpghtarg >= 1) unsort(nt, itarg, nd, ptsort, pottarg);
  if (ifpghtarg >= 2) unsort(nt, itarg, nd * D, gtsort, gradtarg);
  if (ifpghtarg >= 3) unsort(nt, itarg, nd * NH, htsort, hesstarg);
  return ORC_OK;
}

// Tree snapshot exported for the product-vs-oracle tree comparison.
struct TreeOut {
  int dim, nlevels, nboxes, npwlevel;
  std::vector<int> laddr, ilevel, iparent, nchild, ichild, nnbors, nbors, isrc, isrcse, itarg, itargse;
  std::vector<double> centers, boxsize;
};

template <int D>
TreeOut* tree_snapshot(double delta, double eps, int ns, const double* src, int nt, const double* trg) {
  int npwlevel;
  double bs0, cen0[3];
  boxsize0<D>(delta, eps, src, ns, trg, nt, &npwlevel, &bs0, cen0);
  if (npwlevel < -2) return nullptr;
  const int ndiv0 = D == 2 ? 10 : 40, ndiv = D == 2 ? 80 : 100, hcap = D == 2 ? 18 : 15;
  int nlmax = npwlevel + 4, nlevstart = std::max(npwlevel, 0);
  double bsize = bs0 / (double)(1 << nlevstart);
  int nl0 = 0;
  for (int i = nlevstart; i <= 100; i++) {
    nl0 = hlterms(D, bsize, delta, eps, nl0);
    if (nl0 <= hcap) { nlmax = i; break; }
    bsize /= 2;
  }
  Tree<D> t;
  TreeOut* o = new TreeOut();
  build_tree<D>(t, src, ns, trg, nt, ndiv, ndiv0, npwlevel, nlmax, bs0, cen0, o->isrc, o->isrcse, o->itarg, o->itargse);
  o->dim = D; o->nlevels = t.nlevels; o->nboxes = t.nboxes; o->npwlevel = npwlevel;
  o->laddr.assign(t.laddr.begin(), t.laddr.begin() + 2 * (t.nlevels + 1));
  int nb = t.nboxes;
  o->ilevel.assign(t.ilevel.begin() + 1, t.ilevel.begin() + nb + 1);
  o->iparent.assign(t.iparent.begin() + 1, t.iparent.begin() + nb + 1);
  o->nchild.assign(t.nchild.begin() + 1, t.nchild.begin() + nb + 1);
  o->ichild.assign(t.ichild.begin() + Tree<D>::NCH, t.ichild.begin() + (size_t)(nb + 1) * Tree<D>::NCH);
  o->nnbors.assign(t.nnbors.begin() + 1, t.nnbors.begin() + nb + 1);
  o->nbors.assign(t.nbors.begin() + Tree<D>::NCO, t.nbors.begin() + (size_t)(nb + 1) * Tree<D>::NCO);
  o->centers.assign(t.centers.begin() + D, t.centers.begin() + (size_t)(nb + 1) * D);
  o->boxsize.assign(t.boxsize.begin(), t.boxsize.begin() + t.nlevels + 1);
  o->isrc.erase(o->isrc.begin());
  o->itarg.erase(o->itarg.begin());
  o->isrcse.erase(o->isrcse.begin(), o->isrcse.begin() + 2);
  o->itargse.erase(o->itargse.begin(), o->itargse.begin() + 2);
  return o;
}

}  // namespace

// ---------------------------------------------------------------- C ABI (ctypes)
extern "C" {

void orc_hkrand_reset(void) { g_hkseed[0] = 0; g_hkseed[1] = 0; g_hkseed[2] = 0; g_hkseed[3] = 1; }
// hkrand(0) n times (hkrand.f:3-19 with iseed_hk = 0)
void orc_hkrand(long long n, double* out) {
  for (long long i = 0; i < n; i++) out[i] = dlaran(g_hkseed);
}
int orc_hlterms(int ndim, double bsize, double delta, double eps) { return hlterms(ndim, bsize, delta, eps, -1); }
void orc_pwterms(double bsize, double delta, double eps, double* pmax, int* npw) { pwterms(bsize, delta, eps, pmax, npw); }
void orc_boxsize0(int dim, double delta, double eps, int ns, const double* src, int nt,
                  const double* trg, int* levcut, double* bs0, double* cen0) {
  if (dim == 2) boxsize0<2>(delta, eps, src, ns, trg, nt, levcut, bs0, cen0);
  else boxsize0<3>(delta, eps, src, ns, trg, nt, levcut, bs0, cen0);
}

// Full transform, the reference's calling sequence minus the dipole/grad/hess
// arrays.  info (optional, int[8]): npwlevel, nlevels, nboxes, npw, nlmax, ndirect leaves.
int orc_fgt_pgh(int dim, int nd, double delta, double eps, int ns, const double* sources,
                int ifcharge, const double* charge, int ifdipole, int ifpgh, double* pot,
                double* grad, double* hess, int nt, const double* targ, int ifpghtarg,
                double* pottarg, double* gradtarg, double* hesstarg, int* info, int nthreads);
int orc_fgt_full(int dim, int nd, double delta, double eps, int ns, const double* sources,
                 int ifcharge, const double* charge, int ifdipole, const double* rnormal,
                 const double* dipstr, int ifpgh, double* pot, double* grad, double* hess, int nt,
                 const double* targ, int ifpghtarg, double* pottarg, double* gradtarg,
                 double* hesstarg, int* info, int nthreads);
int orc_fgt(int dim, int nd, double delta, double eps, int ns, const double* sources,
            int ifcharge, const double* charge, int ifdipole, int ifpgh, double* pot, int nt,
            const double* targ, int ifpghtarg, double* pottarg, int* info, int nthreads) {
  if (ifpgh > 1 || ifpghtarg > 1) return ORC_UNSUPPORTED;  // no gradient/Hessian arrays here
  return orc_fgt_pgh(dim, nd, delta, eps, ns, sources, ifcharge, charge, ifdipole, ifpgh, pot, nullptr,
                     nullptr, nt, targ, ifpghtarg, pottarg, nullptr, nullptr, info, nthreads);
}

// The same with the gradient and Hessian arrays (ifpgh, ifpghtarg up to 3):
// grad(nd, dim, ns), hess(nd, 3 or 6, ns) as in fgt2d / fgt3d.
int orc_fgt_pgh(int dim, int nd, double delta, double eps, int ns, const double* sources,
                int ifcharge, const double* charge, int ifdipole, int ifpgh, double* pot,
                double* grad, double* hess, int nt, const double* targ, int ifpghtarg,
                double* pottarg, double* gradtarg, double* hesstarg, int* info, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  if (ifdipole) return ORC_UNSUPPORTED;  // no dipole arrays here
  return orc_fgt_full(dim, nd, delta, eps, ns, sources, ifcharge, charge, 0, nullptr, nullptr, ifpgh,
                      pot, grad, hess, nt, targ, ifpghtarg, pottarg, gradtarg, hesstarg, info, nthreads);
}

// The reference's full argument list (fgt2d.f:19-22, less iper): charges
// and/or dipoles with rnormal(dim, ns), dipstr(nd, ns).
int orc_fgt_full(int dim, int nd, double delta, double eps, int ns, const double* sources,
                 int ifcharge, const double* charge, int ifdipole, const double* rnormal,
                 const double* dipstr, int ifpgh, double* pot, double* grad, double* hess, int nt,
                 const double* targ, int ifpghtarg, double* pottarg, double* gradtarg,
                 double* hesstarg, int* info, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  Result r;
  int rc = dim == 2 ? fgt_run<2>(nd, delta, eps, ns, sources, ifcharge, charge, ifdipole, rnormal, dipstr, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg, gradtarg, hesstarg, &r)
                    : fgt_run<3>(nd, delta, eps, ns, sources, ifcharge, charge, ifdipole, rnormal, dipstr, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg, gradtarg, hesstarg, &r);
  if (info) {
    info[0] = r.npwlevel; info[1] = r.nlevels; info[2] = r.nboxes; info[3] = r.npw;
    info[4] = r.nlmax; info[5] = (int)r.nleaf_direct; info[6] = 0; info[7] = 0;
  }
  return rc;
}

// The plane-wave scheme's expansions of chosen boxes (0-based ids): mp and
// lo receive nd * nexp complex values (re, im) per box after the shifts,
// has[i] = 1 where the box carries expansions (levels >= the cut).
int orc_fgt_expansions(int dim, int nd, double delta, double eps, int ns, const double* sources,
                       const double* charge, int nt, const double* targ, int ifpgh, int ifpghtarg, int nbox,
                       const int* boxes, double* mp, double* lo, int* has, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  Probe pr;
  pr.nbox = nbox;
  pr.boxes = boxes;
  pr.mp = reinterpret_cast<cplx*>(mp);
  pr.lo = reinterpret_cast<cplx*>(lo);
  pr.has = has;
  for (int i = 0; i < nbox; i++) has[i] = 0;
  const int NH = dim == 2 ? 3 : 6;
  std::vector<double> pot((size_t)nd * std::max(ns, 1)), pt((size_t)nd * std::max(nt, 1));
  std::vector<double> g((size_t)nd * dim * std::max(ns, 1)), h((size_t)nd * NH * std::max(ns, 1));
  std::vector<double> gt((size_t)nd * dim * std::max(nt, 1)), ht((size_t)nd * NH * std::max(nt, 1));
  Result r;
  return dim == 2 ? fgt_run<2>(nd, delta, eps, ns, sources, 1, charge, 0, nullptr, nullptr, ifpgh, pot.data(),
                               g.data(), h.data(), nt, targ, ifpghtarg, pt.data(), gt.data(), ht.data(), &r, 0, &pr)
                  : fgt_run<3>(nd, delta, eps, ns, sources, 1, charge, 0, nullptr, nullptr, ifpgh, pot.data(),
                               g.data(), h.data(), nt, targ, ifpghtarg, pt.data(), gt.data(), ht.data(), &r, 0, &pr);
}

// The NUFFT scheme (2d/nufft, 3d/nufft; see fgt_run) with the full argument
// list of orc_fgt_full.
int orc_fgt_nufft(int dim, int nd, double delta, double eps, int ns, const double* sources,
                  int ifcharge, const double* charge, int ifdipole, const double* rnormal,
                  const double* dipstr, int ifpgh, double* pot, double* grad, double* hess, int nt,
                  const double* targ, int ifpghtarg, double* pottarg, double* gradtarg,
                  double* hesstarg, int* info, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  Result r;
  int rc = dim == 2 ? fgt_run<2>(nd, delta, eps, ns, sources, ifcharge, charge, ifdipole, rnormal, dipstr, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg, gradtarg, hesstarg, &r, 1)
                    : fgt_run<3>(nd, delta, eps, ns, sources, ifcharge, charge, ifdipole, rnormal, dipstr, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg, gradtarg, hesstarg, &r, 1);
  if (info) {
    info[0] = r.npwlevel; info[1] = r.nlevels; info[2] = r.nboxes; info[3] = r.npw;
    info[4] = r.nlmax; info[5] = (int)r.nleaf_direct; info[6] = 0; info[7] = 0;
  }
  return rc;
}

// FP64 direct sum without cutoff (the reference test's check,
// test_fgt2d.f:161-169 with reps = 1e-100), at targets [0, nt).
void orc_direct(int dim, int nd, double delta, int ns, const double* src, const double* chg,
                int nt, const double* trg, double* pot, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 16)
  for (int it = 0; it < nt; it++) {
    for (int k = 0; k < nd; k++) {
      double acc = 0;
      for (int i = 0; i < ns; i++) {
        double rr = 0;
        for (int d = 0; d < dim; d++) {
          double df = trg[(size_t)dim * it + d] - src[(size_t)dim * i + d];
          rr += df * df;
        }
        acc += std::exp(-rr / delta) * chg[(size_t)nd * i + k];
      }
      pot[(size_t)nd * it + k] = acc;
    }
  }
}

// The FP64 direct sum at sampled targets for large N: sources binned on a
// uniform grid whose cells are at least `rcut` wide, each target summing the
// 3^d cells around its own.  Pairs farther apart than rcut are dropped; with
// rcut^2 = delta * ln(1e30) every dropped term is below 1e-30 of its charge,
// so the sum equals the plain one (orc_direct) to rounding for any workload
// whose potentials are not themselves below ~1e-25 of the charges.
void orc_direct_cut(int dim, int nd, double delta, double rcut, int ns, const double* src,
                    const double* chg, int nt, const double* trg, double* pot, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  if (ns <= 0) {
    for (size_t i = 0; i < (size_t)nt * nd; i++) pot[i] = 0;
    return;
  }
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  for (int d = 0; d < dim; d++) lo[d] = hi[d] = src[d];
  for (int i = 0; i < ns; i++)
    for (int d = 0; d < dim; d++) {
      lo[d] = std::min(lo[d], src[(size_t)dim * i + d]);
      hi[d] = std::max(hi[d], src[(size_t)dim * i + d]);
    }
  double ext = 0;
  for (int d = 0; d < dim; d++) ext = std::max(ext, hi[d] - lo[d]);
  const double maxcells = dim == 2 ? 4096.0 : 256.0;  // per dimension
  const double h = std::max(rcut, ext / maxcells) * (1 + 1e-12) + 1e-300;
  int nc[3] = {1, 1, 1};
  for (int d = 0; d < dim; d++) nc[d] = std::max(1, (int)std::floor((hi[d] - lo[d]) / h) + 1);
  const size_t ncell = (size_t)nc[0] * nc[1] * nc[2];
  auto cell_of = [&](const double* x, int* c) {
    for (int d = 0; d < 3; d++) c[d] = 0;
    for (int d = 0; d < dim; d++) c[d] = (int)std::floor((x[d] - lo[d]) / h);
  };
  std::vector<size_t> start(ncell + 1, 0);
  std::vector<int> order(ns);
  std::vector<size_t> cid(ns);
  for (int i = 0; i < ns; i++) {
    int c[3];
    cell_of(src + (size_t)dim * i, c);
    for (int d = 0; d < dim; d++) c[d] = std::min(std::max(c[d], 0), nc[d] - 1);
    cid[i] = ((size_t)c[2] * nc[1] + c[1]) * nc[0] + c[0];
    start[cid[i] + 1]++;
  }
  for (size_t c = 0; c < ncell; c++) start[c + 1] += start[c];
  {
    std::vector<size_t> fill(start.begin(), start.end() - 1);
    for (int i = 0; i < ns; i++) order[fill[cid[i]]++] = i;
  }
  const double r2 = rcut * rcut;
#pragma omp parallel for schedule(dynamic, 16)
  for (int it = 0; it < nt; it++) {
    const double* t = trg + (size_t)dim * it;
    int c[3];
    cell_of(t, c);
    std::vector<double> acc(nd, 0.0);
    const int zr = dim == 3 ? 1 : 0;
    for (int dz = -zr; dz <= zr; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          const int cx = c[0] + dx, cy = c[1] + dy, cz = c[2] + dz;
          if (cx < 0 || cy < 0 || cz < 0 || cx >= nc[0] || cy >= nc[1] || cz >= nc[2]) continue;
          const size_t cc = ((size_t)cz * nc[1] + cy) * nc[0] + cx;
          for (size_t k = start[cc]; k < start[cc + 1]; k++) {
            const int i = order[k];
            double rr = 0;
            for (int d = 0; d < dim; d++) {
              const double df = t[d] - src[(size_t)dim * i + d];
              rr += df * df;
            }
            if (rr > r2) continue;
            const double e = std::exp(-rr / delta);
            for (int m = 0; m < nd; m++) acc[m] += e * chg[(size_t)nd * i + m];
          }
        }
    for (int m = 0; m < nd; m++) pot[(size_t)nd * it + m] = acc[m];
  }
}

// The same direct sum with gradients and Hessians (pgh = 2, 3): the
// derivatives of exp(-r^2/delta) with respect to the target, per
// g2d_directch_vec / g3d_directch_vec without the cutoff.
void orc_direct_pgh(int dim, int nd, double delta, int ns, const double* src, const double* chg,
                    int nt, const double* trg, int pgh, double* pot, double* grad, double* hess,
                    int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  const int NH = dim == 2 ? 3 : 6;
  const double rfac = -2.0 / delta;
#pragma omp parallel for schedule(dynamic, 16)
  for (int it = 0; it < nt; it++) {
    for (int k = 0; k < nd; k++) {
      double a[10] = {0};
      for (int i = 0; i < ns; i++) {
        double rr = 0, g[3] = {0, 0, 0};
        for (int d = 0; d < dim; d++) {
          double df = trg[(size_t)dim * it + d] - src[(size_t)dim * i + d];
          rr += df * df;
          g[d] = rfac * df;
        }
        const double v = std::exp(-rr / delta) * chg[(size_t)nd * i + k];
        a[0] += v;
        for (int d = 0; d < dim; d++) a[1 + d] += g[d] * v;
        double* h = a + 1 + dim;
        if (dim == 2) {
          h[0] += (rfac + g[0] * g[0]) * v; h[1] += g[0] * g[1] * v; h[2] += (rfac + g[1] * g[1]) * v;
        } else {
          h[0] += (rfac + g[0] * g[0]) * v; h[1] += (rfac + g[1] * g[1]) * v;
          h[2] += (rfac + g[2] * g[2]) * v; h[3] += g[0] * g[1] * v;
          h[4] += g[0] * g[2] * v; h[5] += g[1] * g[2] * v;
        }
      }
      pot[(size_t)nd * it + k] = a[0];
      if (pgh >= 2)
        for (int d = 0; d < dim; d++) grad[k + nd * (d + (size_t)dim * it)] = a[1 + d];
      if (pgh >= 3)
        for (int c = 0; c < NH; c++) hess[k + nd * (c + (size_t)NH * it)] = a[1 + dim + c];
    }
  }
}

// Exact sums (no cutoff) with charges and/or dipoles, pot/grad/hess by pgh:
// the per-pair terms of g2d_directc*/d*_vec and the 3D twins.
void orc_direct_full(int dim, int nd, double delta, int ns, const double* src, int ifcharge,
                     const double* chg, int ifdipole, const double* rn, const double* ds, int nt,
                     const double* trg, int pgh, double* pot, double* grad, double* hess,
                     int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  const int NH = dim == 2 ? 3 : 6;
  const double inf = HUGE_VAL;
  std::fill(pot, pot + (size_t)nd * nt, 0.0);
  if (pgh >= 2) std::fill(grad, grad + (size_t)nd * dim * nt, 0.0);
  if (pgh >= 3) std::fill(hess, hess + (size_t)nd * NH * nt, 0.0);
#pragma omp parallel for schedule(dynamic, 4)
  for (int it = 0; it < nt; it++) {
    double* p = pot + (size_t)nd * it;
    double* g = pgh >= 2 ? grad + (size_t)nd * dim * it : nullptr;
    double* h = pgh >= 3 ? hess + (size_t)nd * NH * it : nullptr;
    const double* t = trg + (size_t)dim * it;
    if (dim == 2) {
      if (ifcharge) directc<2>(nd, delta, inf, src, ns, chg, t, 1, pgh, p, g, h);
      if (ifdipole) directd<2>(nd, delta, inf, src, ns, rn, ds, t, 1, pgh, p, g, h);
    } else {
      if (ifcharge) directc<3>(nd, delta, inf, src, ns, chg, t, 1, pgh, p, g, h);
      if (ifdipole) directd<3>(nd, delta, inf, src, ns, rn, ds, t, 1, pgh, p, g, h);
    }
  }
}

void* orc_tree_build(int dim, double delta, double eps, int ns, const double* src, int nt, const double* trg) {
  return dim == 2 ? (void*)tree_snapshot<2>(delta, eps, ns, src, nt, trg) : (void*)tree_snapshot<3>(delta, eps, ns, src, nt, trg);
}
void orc_tree_dims(void* h, int* out) {
  TreeOut* t = (TreeOut*)h;
  out[0] = t->dim; out[1] = t->nlevels; out[2] = t->nboxes; out[3] = t->npwlevel;
}
// field: 0 laddr, 1 ilevel, 2 iparent, 3 nchild, 4 ichild, 5 nnbors, 6 nbors,
// 7 isrc, 8 isrcse, 9 itarg, 10 itargse
long long orc_tree_int(void* h, int field, int* out) {
  TreeOut* t = (TreeOut*)h;
  std::vector<int>* v[] = {&t->laddr, &t->ilevel, &t->iparent, &t->nchild, &t->ichild, &t->nnbors,
                           &t->nbors, &t->isrc, &t->isrcse, &t->itarg, &t->itargse};
  if (field < 0 || field > 10) return -1;
  if (out) std::memcpy(out, v[field]->data(), v[field]->size() * sizeof(int));
  return (long long)v[field]->size();
}
// field: 0 centers, 1 boxsize
long long orc_tree_dbl(void* h, int field, double* out) {
  TreeOut* t = (TreeOut*)h;
  std::vector<double>& v = field == 0 ? t->centers : t->boxsize;
  if (out) std::memcpy(out, v.data(), v.size() * sizeof(double));
  return (long long)v.size();
}
void orc_tree_free(void* h) { delete (TreeOut*)h; }

}  // extern "C"
