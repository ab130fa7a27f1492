// Host-side adaptive tree and interaction lists for the plane-wave FGT.
//
// Same tree and list semantics as the reference's host layer
// (2d/planewave/src/common/pts_tree2d4.f, tree_routs4.f and the 3D twins
// pts_tree3d.f, tree_routs3d.f): level-restricted 2^d-tree refined on source
// counts, colleagues, modified list1, plane-wave list.  Box ids here are
// 0-based; the reference's numbering order is kept (level by level, children
// in parent order, level-restriction boxes appended per level), so box k here
// is box k+1 there.
#pragma once
#include <cstdint>
#include <memory>
#include <new>
#include <type_traits>
#include <utility>
#include <vector>

namespace fgtb {

// Allocator whose resize leaves new elements default-initialised (no
// zeroing), for arrays that are filled right after sizing (box arrays read
// back from the device, task arrays).
template <class T, class A = std::allocator<T>>
struct default_init_allocator : A {
  using A::A;
  template <class U>
  struct rebind {
    using other = default_init_allocator<U, typename std::allocator_traits<A>::template rebind_alloc<U>>;
  };
  template <class U>
  void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
    ::new (static_cast<void*>(p)) U;
  }
  template <class U, class... Args>
  void construct(U* p, Args&&... args) {
    std::allocator_traits<A>::construct(static_cast<A&>(*this), p, std::forward<Args>(args)...);
  }
};
template <class T>
using uvector = std::vector<T, default_init_allocator<T>>;

struct Tree {
  int dim = 2, nch = 4, nco = 9;
  int nlevels = 0, nboxes = 0;
  int npwlevel = 0;
  double bs0 = 0, cen0[3] = {0, 0, 0};
  std::vector<int> lfirst, llast;          // boxes of level l: [lfirst[l], llast[l]]
  uvector<int> level, parent, nchild;  // per box
  uvector<int> child;                  // nch per box, -1 when absent
  uvector<int> ncoll, coll;            // colleagues (self included), nco per box
  uvector<double> centers;             // dim per box
  std::vector<double> boxsize;             // per level
  // sorted order: position -> original index (0-based)
  std::vector<int> isrc, itarg;
  // per box point ranges in sorted order, [start, end)
  std::vector<int> s0, s1, t0, t1;

  int ns(int b) const { return s1[b] - s0[b]; }
  int nt(int b) const { return t1[b] - t0[b]; }
  int ch(int b, int j) const { return child[(size_t)b * nch + j]; }
  double c(int b, int d) const { return centers[(size_t)b * dim + d]; }
};

// Expansion-length rules, g2dterms.f:19-133 / g3dterms.f:13-127.
int hlterms(int ndim, double bsize, double delta, double eps, int nterms_default);
void pwterms(double bsize, double delta, double eps, double* pmax, int* npw);

// Bounding box, cut level and enlarged root size, pts_tree2d4.f:1187-1258.
void boxsize0(int dim, double delta, double eps, const double* src, int ns, const double* trg,
              int nt, int* levcut, double* bs0, double* cen0);
// The same from a bounding box already known (per-dimension min mn, max mx).
void boxsize0_bbox(int dim, double delta, double eps, const double* mn, const double* mx, int* levcut,
                   double* bs0, double* cen0);

// Builds the tree for sources/targets given as (n, dim) row-major arrays and
// sorts both point sets (pts_tree_mem/build/sort).  nthreads <= 0 uses all.
void build_tree(Tree& t, int dim, const double* src, int ns, const double* trg, int nt, int ndiv,
                int ndiv0, int levcut, int nlmax, double bs0, const double* cen0, int nthreads);

// Box-level steps of build_tree, shared by the host build and the build whose
// point work runs on the GPU (fgt_devtree.cu).
//   tree_init: the root box only.
//   tree_refine_level: refines the boxes of level lev whose source count
//     (count[box], every box so far) exceeds thr, appending their children;
//     firstchild[box - lfirst[lev]] receives the first child id or -1.
//     Returns the number of refined boxes (0 ends the refinement).
//   tree_finish: closes the refinement at nlevels, computes colleagues (unless
//     have_colleagues: t.ncoll / t.coll already hold them) and
//     applies the level restriction (pts_tree_fix_lr + reorg); idmap maps a
//     box id of the refinement to its final id.
//   tree_leaf_ranks: depth-first rank of the leaves (the pts_tree_sort order).
//   tree_ranges: per-box point ranges [r0, r1) from the per-leaf counts.
void tree_init(Tree& t, int dim, double bs0, const double* cen0, int nlmax);
int tree_refine_level(Tree& t, int lev, int thr, const std::vector<int>& count, std::vector<int>& firstchild);
void tree_finish(Tree& t, int nlevels, std::vector<int>& idmap, bool have_colleagues = false);
void tree_leaf_ranks(const Tree& t, std::vector<int>& dfs_rank, std::vector<int>& leaf_of_rank);
void tree_ranges(const Tree& t, const std::vector<int>& leafcount, const std::vector<int>& leaf_of_rank,
                 std::vector<int>& r0, std::vector<int>& r1);

// Interaction lists used by the transform (fgt2dmain / fgt3dmain set-up).
struct Lists {
  // modified list1 as CSR over boxes (compute_modified_list1); filled for
  // the boxes at levels <= the cut, the only ones whose lists are read.
  // (The plane-wave lists of the cut level are the colleagues filtered
  // where the far-field tasks are built.)
  std::vector<int> l1off, l1;
  std::vector<uint8_t> ifhung;
};
void build_lists(const Tree& t, Lists& L);

// Recomputes colleagues (computecoll) on a tree given from outside.
void compute_colleagues(Tree& t);

}  // namespace fgtb
