// Host-side tree and lists; see fgt_tree.hpp.
//
// Point work (refinement bookkeeping, final point location and the stable
// sort into tree order) is data-parallel over points with OpenMP; box work
// (level restriction, colleagues, lists) follows the reference routines.
#include "fgt_tree.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace fgtb {

namespace {
// Default-real (single precision) literals of the reference.
const double F105 = (double)1.05f;  // tree_routs4.f:195, pts_tree2d4.f:959
const double F109 = (double)1.09f;  // g2dterms.f:54
inline double child_sign(int j, int d) { return ((j >> d) & 1) ? 1.0 : -1.0; }
}  // namespace

// g2dhlterms, g2dterms.f:19-64 (Wan-Karniadakis error bound)
int hlterms(int ndim, double bsize, double delta, double eps, int nterms_default) {
  double e1 = std::exp(1.0);
  double r = bsize / std::sqrt(2.0 * delta);
  int p0 = (int)(e1 * r * r) + 1;
  double rk = F109 * std::pow(8 * std::atan(1.0), -0.25);
  for (int p = p0; p <= 300; p++) {
    double rp = r * std::sqrt(e1 / p);
    double err = ndim * rk * std::pow((double)p, -0.25) * __builtin_powi(rp, p) / (1 - rp);
    if (err < eps) return p;
  }
  return nterms_default;
}

// g2dpwterms, g2dterms.f:71-133 (Poisson summation: h = 2pi/(rmax+sqrt(ln 1/eps)))
void pwterms(double bsize, double delta, double eps, double* pmax, int* npw) {
  double pi = 4.0 * std::atan(1.0);
  double rmax = bsize / std::sqrt(delta);
  double d = std::sqrt(std::log(1.0 / eps));
  *pmax = 2.0 * d;
  double h = 2 * pi / (rmax + d);
  *npw = 2 * (int)(*pmax / h);
}

void boxsize0(int dim, double delta, double eps, const double* src, int ns, const double* trg,
              int nt, int* levcut, double* bs0, double* cen0) {
  double mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
  const double* first = ns > 0 ? src : trg;
  for (int d = 0; d < dim; d++) mn[d] = mx[d] = first[d];
  auto scan = [&](const double* x, int n) {
    for (int d = 0; d < dim; d++) {
      double lo = mn[d], hi = mx[d];
#pragma omp parallel for reduction(min : lo) reduction(max : hi)
      for (int i = 0; i < n; i++) {
        double v = x[(size_t)dim * i + d];
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
      }
      mn[d] = lo;
      mx[d] = hi;
    }
  };
  scan(src, ns);
  scan(trg, nt);
  boxsize0_bbox(dim, delta, eps, mn, mx, levcut, bs0, cen0);
}

void boxsize0_bbox(int dim, double delta, double eps, const double* mn, const double* mx, int* levcut,
                   double* bs0, double* cen0) {
  double b = mx[0] - mn[0];
  for (int d = 1; d < dim; d++)
    if (mx[d] - mn[d] > b) b = mx[d] - mn[d];
  for (int d = 0; d < dim; d++) cen0[d] = (mn[d] + mx[d]) / 2;
  double dc = std::sqrt(delta * std::log(1.0 / eps));
  double dl = std::log(b / dc) / std::log(2.0);
  int lc = (int)dl;
  *bs0 = b;
  *levcut = lc;
  if (b < dc) return;
  *bs0 = std::ldexp(1.0, lc + 1) * dc;
  *levcut = lc + 1;
}

namespace {

struct Builder {
  Tree& t;
  int D, NCH, NCO;
  std::vector<int> idmap;  // box id before level restriction -> current id
  explicit Builder(Tree& tt) : t(tt), D(tt.dim), NCH(tt.nch), NCO(tt.nco) {}

  double& C(int b, int d) { return t.centers[(size_t)b * D + d]; }
  int& CH(int b, int j) { return t.child[(size_t)b * NCH + j]; }

  // Grows the box arrays to n boxes (the vectors grow their capacity
  // geometrically; only the new boxes are initialised).
  void reserve_boxes(int n) {
    if ((int)t.level.size() >= n) return;
    const size_t m = n;
    t.level.resize(m, 0);
    t.parent.resize(m, -1);
    t.nchild.resize(m, 0);
    t.child.resize(m * NCH, -1);
    t.centers.resize(m * D, 0.0);
  }

  // Appends the children of box b (tree_refine_boxes, tree_routs4.f:28-49).
  void make_children(int b, int first_child, int lev, double bs) {
    t.nchild[b] = NCH;
    for (int j = 0; j < NCH; j++) {
      int c = first_child + j;
      for (int d = 0; d < D; d++) C(c, d) = C(b, d) + child_sign(j, d) * bs / 2;
      t.parent[c] = b;
      t.nchild[c] = 0;
      for (int l = 0; l < NCH; l++) CH(c, l) = -1;
      CH(b, j) = c;
      t.level[c] = lev;
    }
  }

  // computecoll, tree_routs4.f:100-211, levels [l0, l1]
  // colleagues of box b at level l from its parent's list, into (nc, co)
  // The children of a refined box share their coordinate along d with every
  // sibling on the same side of d, so the test is made once per side and
  // dimension (child 0 and child 2^d) and a child passes when its sides do;
  // a box with a missing child takes the test child by child.
  void colleagues_box(int b, double lim, uvector<int>& nc, uvector<int>& co) {
    int dad = t.parent[b];
    int n = 0;
    for (int i = 0; i < nc[dad]; i++) {
      int jb = co[(size_t)dad * NCO + i];
      if (CH(jb, 0) < 0 && t.nchild[jb] == 0) continue;
      bool all = true;
      for (int j = 0; j < NCH; j++) all = all && CH(jb, j) >= 0;
      if (all) {
        unsigned pass[2] = {0u, 0u};  // bit d: side 0 / side 1 of dimension d is near
        for (int d = 0; d < D; d++) {
          if (std::fabs(C(CH(jb, 0), d) - C(b, d)) <= lim) pass[0] |= 1u << d;
          if (std::fabs(C(CH(jb, 1 << d), d) - C(b, d)) <= lim) pass[1] |= 1u << d;
        }
        for (int j = 0; j < NCH; j++) {
          const unsigned ok = (pass[1] & (unsigned)j) | (pass[0] & ~(unsigned)j);
          if ((ok & ((1u << D) - 1)) == (1u << D) - 1) co[(size_t)b * NCO + n++] = CH(jb, j);
        }
        continue;
      }
      for (int j = 0; j < NCH; j++) {
        int kb = CH(jb, j);
        if (kb < 0) continue;
        bool ok = true;
        for (int d = 0; d < D; d++)
          if (!(std::fabs(C(kb, d) - C(b, d)) <= lim)) ok = false;
        if (ok) co[(size_t)b * NCO + n++] = kb;
      }
    }
    nc[b] = n;
  }
  void colleagues_level(int l) {
    double lim = F105 * t.boxsize[l];
#pragma omp parallel for schedule(static) if (t.llast[l] - t.lfirst[l] > 512)
    for (int b = t.lfirst[l]; b <= t.llast[l]; b++) colleagues_box(b, lim, t.ncoll, t.coll);
  }
  // After a refinement pass and its reorg (map: id before -> id after; the
  // boxes that existed before the pass have ids < nold before it): the
  // lists of those boxes are carried over through map, and only the new
  // boxes and the old boxes next to them (children of a colleague of a box
  // refined in the pass) are computed again, level by level.  computecoll's
  // order is kept, so the result equals colleagues_all().
  std::vector<int> refined_ids;  // ids (before reorg) of the boxes refined in the pass
  std::vector<int> last_map;     // reorg's map
  void colleagues_after_pass(int nold) {
    const int nb = t.nboxes;
    const std::vector<int>& map = last_map;
    uvector<int> nc(nb, 0), co((size_t)nb * NCO, -1);
    std::vector<char> fresh(nb, 1), mark(nb, 0), refd(nb, 0);
#pragma omp parallel for schedule(static) if (nold > 16384)
    for (int o = 0; o < nold; o++) {
      const int b = map[o];
      fresh[b] = 0;
      nc[b] = t.ncoll[o];
      for (int i = 0; i < t.ncoll[o]; i++) co[(size_t)b * NCO + i] = map[t.coll[(size_t)o * NCO + i]];
    }
    for (int r : refined_ids) refd[map[r]] = 1;
    for (int l = 1; l <= t.nlevels; l++) {
      const double lim = F105 * t.boxsize[l];
#pragma omp parallel for schedule(static) if (t.llast[l] - t.lfirst[l] > 512)
      for (int b = t.lfirst[l]; b <= t.llast[l]; b++)
        if (fresh[b] || mark[b]) colleagues_box(b, lim, nc, co);
      // old boxes of level l + 1 whose parent has a refined colleague
      for (int b = t.lfirst[l]; b <= t.llast[l]; b++) {
        if (!refd[b]) continue;
        for (int i = 0; i < nc[b]; i++) {
          const int c = co[(size_t)b * NCO + i];
          for (int j = 0; j < NCH; j++) {
            const int e = CH(c, j);
            if (e >= 0 && !fresh[e]) mark[e] = 1;
          }
        }
      }
    }
    t.ncoll.swap(nc);
    t.coll.swap(co);
  }
  void colleagues_all() {
    t.ncoll.assign(t.nboxes, 0);
    t.coll.assign((size_t)t.nboxes * NCO, -1);
    t.ncoll[0] = 1;
    t.coll[0] = 0;
    for (int l = 1; l <= t.nlevels; l++) colleagues_level(l);
  }

  // tree_refine_boxes_flag, tree_routs4.f:334-388, over boxes ids[]
  void refine_flagged(std::vector<int>& iflag, int a, int b, int lev) {
    for (int box = a; box <= b; box++) {
      if (iflag[box] <= 0) continue;
      int c0 = t.nboxes;
      reserve_boxes(c0 + NCH);
      if ((int)iflag.size() < c0 + NCH) iflag.resize((size_t)(c0 + NCH) * 2, 0);
      make_children(box, c0, lev + 1, t.boxsize[lev + 1]);
      refined_ids.push_back(box);
      for (int j = 0; j < NCH; j++) iflag[c0 + j] = iflag[box] == 1 ? 3 : 0;
      t.nboxes += NCH;
    }
  }

  // pts_tree_reorg, pts_tree2d4.f:1001-1150: level l >= 2 becomes
  // [old boxes of l] ++ [tail boxes of l].
  void reorg(const std::vector<int>& tf, const std::vector<int>& tl, std::vector<int>& iflag) {
    int nb = t.nboxes;
    std::vector<int>& map = last_map;
    map.assign(nb, -1);
    std::vector<int> olevel(t.level.begin(), t.level.begin() + nb);
    std::vector<int> oparent(t.parent.begin(), t.parent.begin() + nb);
    std::vector<int> onchild(t.nchild.begin(), t.nchild.begin() + nb);
    std::vector<int> ochild(t.child.begin(), t.child.begin() + (size_t)nb * NCH);
    std::vector<double> ocent(t.centers.begin(), t.centers.begin() + (size_t)nb * D);
    std::vector<int> oflag(iflag.begin(), iflag.begin() + nb);
    for (int l = 0; l <= std::min(1, t.nlevels); l++)
      for (int b = t.lfirst[l]; b <= t.llast[l]; b++) map[b] = b;
    // the new position of every box: per level the old boxes, then the tail
    if (t.nlevels >= 2) {
      int cur = t.lfirst[2];
      for (int l = 2; l <= t.nlevels; l++) {
        const int a0 = t.lfirst[l], a1 = t.llast[l];
        t.lfirst[l] = cur;
        for (int pass = 0; pass < 2; pass++) {
          const int a = pass ? tf[l] : a0, b = pass ? tl[l] : a1, base = cur;
#pragma omp parallel for schedule(static) if (b - a > 16384)
          for (int box = a; box <= b; box++) map[box] = base + (box - a);
          cur += std::max(0, b - a + 1);
        }
        t.llast[l] = cur - 1;
      }
    }
#pragma omp parallel for schedule(static) if (nb > 16384)
    for (int box = 0; box < nb; box++) {
      const int nbx = map[box];
      t.level[nbx] = olevel[box];
      t.nchild[nbx] = onchild[box];
      for (int d = 0; d < D; d++) t.centers[(size_t)nbx * D + d] = ocent[(size_t)box * D + d];
      iflag[nbx] = oflag[box];
      t.parent[nbx] = oparent[box] >= 0 ? map[oparent[box]] : -1;
      for (int j = 0; j < NCH; j++) {
        int c = ochild[(size_t)box * NCH + j];
        CH(nbx, j) = c >= 0 ? map[c] : -1;
      }
    }
#pragma omp parallel for schedule(static) if (idmap.size() > 16384)
    for (size_t k = 0; k < idmap.size(); k++) idmap[k] = map[idmap[k]];
  }

  bool touching(int a, int b, double lim) {
    for (int d = 0; d < D; d++)
      if (!(std::fabs(C(a, d) - C(b, d)) <= lim)) return false;
    return true;
  }

  // pts_tree_fix_lr, pts_tree2d4.f:693-996
  void fix_lr() {
    auto T = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
    double tt[8];
    tt[0] = T();
    int nlev = t.nlevels;
    std::vector<int> iflag((size_t)t.nboxes * 2, 0);
    int* const fl = iflag.data();
    // Flag pass 1 only ever sets a flag from 0 to 1, so its outcome does not
    // depend on the order of the boxes: all levels at once, in parallel
    // (relaxed atomics: several boxes may flag the same colleague).
    if (nlev >= 2) {
      const int b0 = t.lfirst[2], b1 = t.llast[nlev];
#pragma omp parallel for schedule(dynamic, 1024) if (b1 - b0 > 4096)
      for (int b = b0; b <= b1; b++) {
        const int l = t.level[b];
        const double dist = 1.05 * (t.boxsize[l - 1] + t.boxsize[l - 2]) / 2.0;
        const int dad = t.parent[b], gd = t.parent[dad];
        for (int i = 0; i < t.ncoll[gd]; i++) {
          const int jb = t.coll[(size_t)gd * NCO + i];
          if (t.nchild[jb] == 0 && __atomic_load_n(fl + jb, __ATOMIC_RELAXED) == 0 && touching(jb, dad, dist))
            __atomic_store_n(fl + jb, 1, __ATOMIC_RELAXED);
        }
      }
    }
    // Pass 2 runs from the finest level up; a level reads its own flags and
    // only sets flags of the level above from 0 to 2, so each level is one
    // parallel step.
    for (int l = nlev; l >= 1; l--) {
      const double dist = 1.05 * (t.boxsize[l] + t.boxsize[l - 1]) / 2.0;
#pragma omp parallel for schedule(dynamic, 1024) if (t.llast[l] - t.lfirst[l] > 4096)
      for (int b = t.lfirst[l]; b <= t.llast[l]; b++) {
        const int f = __atomic_load_n(fl + b, __ATOMIC_RELAXED);
        if (f != 1 && f != 2) continue;
        const int dad = t.parent[b];
        for (int i = 0; i < t.ncoll[dad]; i++) {
          const int jb = t.coll[(size_t)dad * NCO + i];
          if (t.nchild[jb] == 0 && __atomic_load_n(fl + jb, __ATOMIC_RELAXED) == 0 && touching(jb, b, dist))
            __atomic_store_n(fl + jb, 2, __ATOMIC_RELAXED);
        }
      }
    }
    tt[1] = T();
    const int nb0_ = t.nboxes;
    std::vector<int> tf(nlev + 1, 0), tl(nlev + 1, -1);
    int nold = t.nboxes;
    refined_ids.clear();
    for (int l = 1; l <= nlev - 2; l++) {
      tf[l + 1] = t.nboxes;
      refine_flagged(iflag, t.lfirst[l], t.llast[l], l);
      tl[l + 1] = t.nboxes - 1;
    }
    tt[2] = T();
    const int nb1_ = t.nboxes;
    reorg(tf, tl, iflag);
    tt[3] = T();
    colleagues_after_pass(nold);
    tt[4] = T();
    for (int b = 0; b < t.nboxes; b++)
      if (iflag[b] != 3) iflag[b] = 0;
    std::fill(tf.begin(), tf.end(), 0);
    std::fill(tl.begin(), tl.end(), -1);
    nold = t.nboxes;
    refined_ids.clear();
    for (int l = 2; l <= nlev - 2; l++) {
      update_flags(l, t.lfirst[l], t.llast[l], iflag);
      update_flags(l, tf[l], tl[l], iflag);
      tf[l + 1] = t.nboxes;
      refine_flagged(iflag, t.lfirst[l], t.llast[l], l);
      refine_flagged(iflag, tf[l], tl[l], l);
      tl[l + 1] = t.nboxes - 1;
      t.ncoll.resize(t.nboxes, 0);
      t.coll.resize((size_t)t.nboxes * NCO, -1);
      double lim = F105 * t.boxsize[l + 1];
#pragma omp parallel for schedule(static) if (tl[l + 1] - tf[l + 1] > 4096)
      for (int b = tf[l + 1]; b <= tl[l + 1]; b++) {
        int dad = t.parent[b];
        int n = 0;
        for (int i = 0; i < t.ncoll[dad]; i++) {
          int jb = t.coll[(size_t)dad * NCO + i];
          for (int j = 0; j < NCH; j++) {
            int kb = CH(jb, j);
            if (kb >= 0 && touching(kb, b, lim)) t.coll[(size_t)b * NCO + n++] = kb;
          }
        }
        t.ncoll[b] = n;
      }
    }
    tt[5] = T();
    reorg(tf, tl, iflag);
    tt[6] = T();
    colleagues_after_pass(nold);
    tt[7] = T();
    if (getenv("FGT_TREE_TIMING"))
      fprintf(stderr, "fix_lr: flags %.4f refine1 %.4f reorg1 %.4f coll1 %.4f pass2 %.4f reorg2 %.4f coll2 %.4f nb %d nb0 %d nb1 %d\n",
              tt[1] - tt[0], tt[2] - tt[1], tt[3] - tt[2], tt[4] - tt[3], tt[5] - tt[4], tt[6] - tt[5], tt[7] - tt[6], t.nboxes, nb0_, nb1_);
  }

  // updateflags, tree_routs4.f:217-326
  void update_flags(int lev, int a, int b, std::vector<int>& iflag) {
    double dist = 1.05 * (t.boxsize[lev] + t.boxsize[lev + 1]) / 2.0;
    // each box decides its own flag from its colleagues' children
#pragma omp parallel for schedule(dynamic, 1024) if (b - a > 4096)
    for (int box = a; box <= b; box++) {
      if (iflag[box] != 3) continue;
      iflag[box] = 0;
      for (int i = 0; i < t.ncoll[box] && iflag[box] == 0; i++) {
        int jb = t.coll[(size_t)box * NCO + i];
        for (int j = 0; j < NCH; j++) {
          int kb = CH(jb, j);
          if (kb >= 0 && t.nchild[kb] > 0 && touching(kb, box, dist)) { iflag[box] = 1; break; }
        }
      }
    }
  }
};

// Child slot of point x in box centre c (sort_pts_to_children: coordinate
// minus centre < 0 goes to the lower child).
inline int child_slot(const double* x, const double* c, int D) {
  int j = 0;
  for (int d = 0; d < D; d++)
    if (!(x[d] - c[d] < 0)) j |= 1 << d;
  return j;
}

// Locates every point in its leaf, then stable-sorts points by the leaf's
// depth-first rank (the order pts_tree_sort produces) and fills the per-box
// ranges.
void sort_points(Tree& t, const double* x, int n, std::vector<int>& perm, std::vector<int>& r0,
                 std::vector<int>& r1, const std::vector<int>& dfs_rank, int nleafrank,
                 const std::vector<int>& leaf_of_rank, const int* start = nullptr) {
  int D = t.dim;
  std::vector<int> key(n);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    const double* p = x + (size_t)D * i;
    int b = start ? start[i] : 0;
    while (t.nchild[b] > 0) b = t.child[(size_t)b * t.nch + child_slot(p, &t.centers[(size_t)b * D], D)];
    key[i] = dfs_rank[b];
  }
  // stable counting sort by key (per-thread histograms keep it stable)
  int nth = 1;
#ifdef _OPENMP
  nth = omp_get_max_threads();
#endif
  if ((size_t)nth * nleafrank > (size_t)64 << 20) nth = std::max<int>(1, (64 << 20) / std::max(nleafrank, 1));
  std::vector<int> cnt((size_t)nth * nleafrank, 0);
  perm.assign(n, 0);
#pragma omp parallel num_threads(nth)
  {
    int tid = 0, nt = 1;
#ifdef _OPENMP
    tid = omp_get_thread_num();
    nt = omp_get_num_threads();
#endif
    int lo = (int)((long long)n * tid / nt), hi = (int)((long long)n * (tid + 1) / nt);
    int* c = cnt.data() + (size_t)tid * nleafrank;
    for (int i = lo; i < hi; i++) c[key[i]]++;
#pragma omp barrier
#pragma omp single
    {
      long long run = 0;
      for (int k = 0; k < nleafrank; k++)
        for (int th = 0; th < nt; th++) {
          int v = cnt[(size_t)th * nleafrank + k];
          cnt[(size_t)th * nleafrank + k] = (int)run;
          run += v;
        }
    }
    for (int i = lo; i < hi; i++) perm[c[key[i]]++] = i;
  }
  std::vector<int> leafcount(nleafrank, 0);
  for (int i = 0; i < n; i++) leafcount[key[i]]++;
  tree_ranges(t, leafcount, leaf_of_rank, r0, r1);
}

}  // namespace

void tree_ranges(const Tree& t, const std::vector<int>& leafcount, const std::vector<int>& leaf_of_rank,
                 std::vector<int>& r0, std::vector<int>& r1) {
  // leaf ranges from the per-leaf counts, then internal boxes bottom-up
  r0.assign(t.nboxes, 0);
  r1.assign(t.nboxes, 0);
  int pos = 0;
  for (size_t k = 0; k < leaf_of_rank.size(); k++) {
    int b = leaf_of_rank[k];
    r0[b] = pos;
    pos += leafcount[k];
    r1[b] = pos;
  }
  for (int l = t.nlevels; l >= 0; l--)
    for (int b = t.lfirst[l]; b <= t.llast[l]; b++)
      if (t.nchild[b] > 0) {
        r0[b] = r0[t.child[(size_t)b * t.nch]];
        r1[b] = r1[t.child[(size_t)b * t.nch + t.nch - 1]];
      }
}

void tree_init(Tree& t, int dim, double bs0, const double* cen0, int nlmax) {
  t = Tree();
  t.dim = dim;
  t.nch = 1 << dim;
  t.nco = dim == 2 ? 9 : 27;
  t.bs0 = bs0;
  for (int d = 0; d < dim; d++) t.cen0[d] = cen0[d];
  Builder B(t);
  int maxlev = std::max(nlmax, 0);
  t.boxsize.assign(maxlev + 2, 0.0);
  t.lfirst.assign(maxlev + 2, 0);
  t.llast.assign(maxlev + 2, -1);
  B.reserve_boxes(1024);
  t.boxsize[0] = bs0;
  for (int d = 0; d < dim; d++) B.C(0, d) = cen0[d];
  t.level[0] = 0;
  t.parent[0] = -1;
  t.nchild[0] = 0;
  t.lfirst[0] = 0;
  t.llast[0] = 0;
  t.nboxes = 1;
}

int tree_refine_level(Tree& t, int lev, int thr, const std::vector<int>& count, std::vector<int>& firstchild) {
  Builder B(t);
  const int a = t.lfirst[lev], b = t.llast[lev], NCH = t.nch;
  firstchild.assign(b - a + 1, -1);
  int nref = 0;
  for (int box = a; box <= b; box++)
    if (count[box] > thr) firstchild[box - a] = t.nboxes + NCH * nref++;
  if (nref == 0) return 0;
  t.boxsize[lev + 1] = t.boxsize[lev] / 2;
  B.reserve_boxes(t.nboxes + NCH * nref);
  t.lfirst[lev + 1] = t.nboxes;
  const double bs = t.boxsize[lev + 1];
#pragma omp parallel for schedule(static) if (nref > 2048)
  for (int box = a; box <= b; box++)
    if (firstchild[box - a] >= 0) B.make_children(box, firstchild[box - a], lev + 1, bs);
  t.nboxes += NCH * nref;
  t.llast[lev + 1] = t.nboxes - 1;
  return nref;
}

void tree_finish(Tree& t, int nlevels, std::vector<int>& idmap, bool have_colleagues) {
  t.nlevels = nlevels;
  t.boxsize.resize(t.nlevels + 1);
  t.lfirst.resize(t.nlevels + 1);
  t.llast.resize(t.nlevels + 1);
  Builder B(t);
  auto T = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
  const double q0 = T();
  if (!have_colleagues) B.colleagues_all();
  const double q1 = T();
  B.idmap.resize(t.nboxes);
  for (int k = 0; k < t.nboxes; k++) B.idmap[k] = k;
  if (t.nlevels >= 2) B.fix_lr();
  if (getenv("FGT_TREE_TIMING")) fprintf(stderr, "finish: nb %d colleagues %.4f fix_lr %.4f\n", t.nboxes, q1 - q0, T() - q1);
  idmap.swap(B.idmap);
  const int NCH = t.nch, D = t.dim;
  t.level.resize(t.nboxes);
  t.parent.resize(t.nboxes);
  t.nchild.resize(t.nboxes);
  t.child.resize((size_t)t.nboxes * NCH);
  t.centers.resize((size_t)t.nboxes * D);
}

void tree_leaf_ranks(const Tree& t, std::vector<int>& dfs_rank, std::vector<int>& leaf_of_rank) {
  const int NCH = t.nch;
  dfs_rank.assign(t.nboxes, -1);
  leaf_of_rank.clear();
  leaf_of_rank.reserve(t.nboxes);
  std::vector<int> stack;
  stack.push_back(0);
  while (!stack.empty()) {
    int b = stack.back();
    stack.pop_back();
    if (t.nchild[b] == 0) {
      dfs_rank[b] = (int)leaf_of_rank.size();
      leaf_of_rank.push_back(b);
    } else {
      for (int j = NCH - 1; j >= 0; j--) stack.push_back(t.child[(size_t)b * NCH + j]);
    }
  }
}

void compute_colleagues(Tree& t) {
  Builder B(t);
  B.colleagues_all();
}

void build_tree(Tree& t, int dim, const double* src, int ns, const double* trg, int nt, int ndiv,
                int ndiv0, int levcut, int nlmax, double bs0, const double* cen0, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  tree_init(t, dim, bs0, cen0, nlmax);
  const int D = dim;
  auto T = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
  bool dbg = getenv("FGT_TREE_TIMING") != nullptr;
  double tA = T();
  // refinement on source counts (idivflag = 0), pts_tree2d4.f:495-563
  std::vector<int> pbox(ns, 0);
  std::vector<int> count(1, ns), firstchild;
  int lev;
  for (lev = 0; lev <= nlmax - 1; lev++) {
    const int a = t.lfirst[lev], b = t.llast[lev];
    const int thr = lev < levcut ? ndiv0 : ndiv;
    if (tree_refine_level(t, lev, thr, count, firstchild) == 0) break;
    count.resize(t.nboxes, 0);
    const int* fc = firstchild.data();
    const int c0 = t.lfirst[lev + 1], nnew = t.nboxes - c0;
    // per-thread counts of the new boxes, summed afterwards (no atomics)
#pragma omp parallel
    {
      std::vector<int> loc(nnew, 0);
#pragma omp for schedule(static) nowait
      for (int i = 0; i < ns; i++) {
        int box = pbox[i];
        if (box < a || box > b || fc[box - a] < 0) continue;
        int c = fc[box - a] + child_slot(src + (size_t)D * i, &t.centers[(size_t)box * D], D);
        pbox[i] = c;
        loc[c - c0]++;
      }
#pragma omp critical
      for (int k = 0; k < nnew; k++) count[c0 + k] += loc[k];
    }
  }
  double tB = T();
  std::vector<int> idmap;
  tree_finish(t, lev, idmap);
  // each source continues its descent from its box before level restriction
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ns; i++) pbox[i] = idmap[pbox[i]];
  double tC = T();
  std::vector<int> dfs_rank, leaf_of_rank;
  tree_leaf_ranks(t, dfs_rank, leaf_of_rank);
  int nl = (int)leaf_of_rank.size();
  double tD = T();
  sort_points(t, src, ns, t.isrc, t.s0, t.s1, dfs_rank, nl, leaf_of_rank, pbox.data());
  double tE = T();
  if (trg == src && nt == ns) {  // targets given as the same array as the sources
    t.itarg = t.isrc;
    t.t0 = t.s0;
    t.t1 = t.s1;
  } else {
    sort_points(t, trg, nt, t.itarg, t.t0, t.t1, dfs_rank, nl, leaf_of_rank);
  }
  double tF = T();
  if (dbg) fprintf(stderr, "tree: refine %.3f lr %.3f dfs %.3f sort_s %.3f sort_t %.3f\n", tB - tA, tC - tB, tD - tC, tE - tD, tF - tE);
}

void build_lists(const Tree& t, Lists& L) {
  int nb = t.nboxes, NCO = t.nco, NCH = t.nch, D = t.dim;
  int npw = t.npwlevel;
  int nlevend = npw < t.nlevels ? npw : t.nlevels;
  L.ifhung.assign(nb, 0);
  for (int l = 0; l <= nlevend; l++)
    for (int b = t.lfirst[l]; b <= t.llast[l]; b++)
      if (t.nchild[b] == 0 && t.ns(b) > 0) L.ifhung[b] = 1;
  // modified list1: tree_routs4.f:715-879 (2D, symmetric insertion at
  // coarse levels) / tree_routs3d.f:511-619 (3D, coarser leaf neighbours).
  // The serial construction appends to list(X) first the symmetric entries
  // b (boxes of the level above, in increasing id), then X's own entries in
  // its loop order.  Here both are counted in parallel, the list is laid out
  // as [symmetric | own], own entries are written by X's iteration and
  // symmetric ones through atomic cursors, each symmetric block then sorted.
  // Only the lists of boxes at levels <= the cut are read (the near-field
  // sources are the leaves there); they receive entries from boxes of their
  // own level and, in 2D, of the level above, so the loops stop at the cut.
  auto cdist = [&](int a, int b, int d) { return std::fabs(t.c(a, d) - t.c(b, d)); };
  const int lmax = std::min(t.nlevels, nlevend);
  const int b_hi = lmax >= 1 ? t.llast[lmax] : -1, b_lo = t.nlevels >= 1 ? t.lfirst[1] : 1;
  // visit(b, own, sym): X's own entries in order, and (kb, b) symmetric pairs
  auto visit = [&](int b, auto&& own, auto&& sym) {
    const int l = t.level[b];
    if (t.nchild[b] != 0) return;
    for (int i = 0; i < t.ncoll[b]; i++) {
      int jb = t.coll[(size_t)b * NCO + i];
      if (l >= npw || t.nchild[jb] == 0) {
        own(jb);
        continue;
      }
      double dist = 1.05 * (t.boxsize[l] + t.boxsize[l + 1]) / 2.0;
      for (int j = 0; j < NCH; j++) {
        int kb = t.ch(jb, j);
        if (kb < 0) continue;
        bool near = true;
        for (int d = 0; d < D; d++)
          if (!(cdist(kb, b, d) < dist)) near = false;
        if (near) {
          own(kb);
          if (D == 2) sym(kb);
        }
      }
    }
    if (D == 3) {
      int dad = t.parent[b];
      double dist = 1.05 * (t.boxsize[l] + t.boxsize[l - 1]) / 2.0;
      for (int i = 0; i < t.ncoll[dad]; i++) {
        int jb = t.coll[(size_t)dad * NCO + i];
        if (t.nchild[jb] != 0) continue;
        bool near = true;
        for (int d = 0; d < D; d++)
          if (!(cdist(jb, b, d) < dist)) near = false;
        if (near) own(jb);
      }
    }
  };
  std::vector<int> nown(nb, 0), nsym(nb, 0);
  if (t.nchild[0] == 0) nown[0] = 1;  // the root leaf holds itself
#pragma omp parallel for schedule(dynamic, 512)
  for (int b = b_lo; b <= b_hi; b++) {
    int n = 0;
    visit(b, [&](int) { n++; }, [&](int kb) {
#pragma omp atomic
      nsym[kb]++;
    });
    nown[b] = n;
  }
  L.l1off.assign(nb + 1, 0);
  for (int b = 0; b < nb; b++) L.l1off[b + 1] = L.l1off[b] + nsym[b] + nown[b];
  L.l1.assign(L.l1off[nb], 0);
  std::vector<int> scur(L.l1off.begin(), L.l1off.end() - 1);
  if (t.nchild[0] == 0) L.l1[L.l1off[0] + nsym[0]] = 0;
#pragma omp parallel for schedule(dynamic, 512)
  for (int b = b_lo; b <= b_hi; b++) {
    int pos = L.l1off[b] + nsym[b];
    visit(b, [&](int v) { L.l1[pos++] = v; }, [&](int kb) {
      int q;
#pragma omp atomic capture
      q = scur[kb]++;
      L.l1[q] = b;
    });
  }
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; b++)
    if (nsym[b] > 1) std::sort(L.l1.begin() + L.l1off[b], L.l1.begin() + L.l1off[b] + nsym[b]);
}

}  // namespace fgtb
