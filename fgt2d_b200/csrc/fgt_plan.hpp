// Execution plan of one plane-wave FGT on one GPU: the host tree and lists
// flattened into task arrays that the CUDA stages consume, plus the device
// copies of those arrays and of the expansion pools.
#pragma once
#include <cstdint>
#include <cstddef>
#include <functional>
#include <memory>
#include <new>
#include <type_traits>
#include <utility>
#include <vector>

#include "fgt_tree.hpp"

namespace fgtb {


enum Route { ROUTE_HERMITE = 0, ROUTE_PW = 1, ROUTE_TAYLOR = 0 };

// stage (a): one formed leaf
struct FormTask {
  int box, s0, n, slot, p, route;
};
// stage (a), 3D Hermite: a chunk of a leaf's sources and the offset (in
// doubles, per density) of its partial Hermite block
struct FormChunk {
  int task, s0, n;
  long long hoff;
};
// stage (b) merge / split: one (parent, child) shift
struct ShiftTask {
  int dst, src, table;  // dst slot, src slot, table row (level * nch + child slot)
};
// stage (b) mp->loc: one cut-level box, its sources in [off, off+cnt) of the
// neighbour array
struct M2LTask {
  int loc, self_mp, off, cnt;
};
struct M2LNbr {
  int mp, shift;  // neighbour mp slot, translation index (jx+1)+3(jy+1)+9(jz+1)
};
// stage (c): one evaluation leaf and point set
struct EvalTask {
  int box, set, i0, n, slot, p, route;
};
// stage (d): a chunk of evaluation points and its source ranges
struct DirTask {
  int set, i0, n, off, cnt;  // points [i0, i0+n) of set; source ranges [off, off+cnt)
};
struct SrcRange {
  int s0, n;
};

struct Params {
  int dim = 2, nd = 1;
  double delta = 0, eps = 0;
  int ns = 0, nt = 0, ifpgh = 0, ifpghtarg = 0;
  int ifcharge = 1, ifdipole = 0;  // source kinds (fgt2d.f:23-40)
  int npwlevel = 0, nlevels = 0, nlevstart = 0, nlmax = 0;
  int npw = 0, nexp = 0, ntermmax = 0;
  double pmax = 0, dsq = 0, dmax = 0;
  bool large_delta = false, all_direct = false;
  int nlocal0 = 0;  // large-delta local order
  double cen0[3] = {0, 0, 0};
  // 0: the plane-wave scheme (2d/planewave, 3d/planewave); 1: the NUFFT
  // scheme (2d/nufft, 3d/nufft): plane-wave expansions at the cut level
  // only, formed from and evaluated at every point of their box
  int scheme = 0;
};

// Host side of the plan.
struct HostPlan {
  Params P;
  int scheme = 0;  // Params.scheme of the next build (set before it)
  Tree tree;
  Lists lists;
  std::vector<int> nlocal;        // per level
  std::vector<double> ts, ws;     // reference node order for the dimension
  std::vector<double> h2x;        // [j * npw + k] = ws_k (-ts_k)^j / sqrt(j!)
  std::vector<double> x2l;        // [j * npw + k] = ts_k^j / j!
  // 1D factors of the diagonal translation tables (re, im): ww[j][k] =
  // exp(i t_j xmin2)^(2^(k-1)) for the merge / split rows of nms levels,
  // w1[j] = exp(i t_j xmin) for mp->loc; the device forms the nexp-long rows
  std::vector<double> ww, w1;
  int nms = 1;
  int nmp = 0, nloc = 0;
  std::vector<int> mp_slot, loc_slot;  // per box, -1 when absent
  uvector<double> box_centers;         // dim per box
  // tasks
  std::vector<FormTask> form;
  // merge / split tasks of parents at level l: [beg[l], end[l])
  std::vector<int> merge_beg, merge_end;
  std::vector<ShiftTask> merge;
  std::vector<int> split_beg, split_end;
  std::vector<ShiftTask> split;
  std::vector<M2LTask> m2l;
  std::vector<M2LNbr> m2l_nbr;
  std::vector<EvalTask> eval;
  uvector<DirTask> dir;
  uvector<SrcRange> dir_src;
  // The near-field arrays built on the GPU instead (build_near_tasks_device;
  // dir / dir_src then stay empty): one stream-ordered allocation, copied
  // into the plan's arena and released by the plan's creation.
  struct DevNear {
    DirTask* dir = nullptr;
    SrcRange* src = nullptr;
    long long ndir = 0, nsrc = 0;
    void* mem = nullptr;
  } dnear;
  bool defer_near = false;  // finish_plan leaves the near-field arrays to the device build
  bool near_built = false;  // the device build has run (beside the host tasks)
  bool same_points = false;  // the targets are the sources (their permutations agree)
  // The finished tree's box arrays as the device build left them (final ids;
  // kept for the near-field build when defer_near, else empty): one
  // stream-ordered allocation, released by the near-field build (or with
  // dnear when the plan's creation stops before it).
  struct DevTree {
    int *level = nullptr, *parent = nullptr, *nchild = nullptr, *child = nullptr, *ncoll = nullptr,
        *coll = nullptr, *s0 = nullptr, *s1 = nullptr;
    double* centers = nullptr;
    void* mem = nullptr;
  } dtree;
  // statistics
  long long direct_pairs = 0;
  long long form_sources = 0, eval_points = 0;
  long long shift_bytes[3] = {0, 0, 0};  // algorithmic bytes of merge, mp->loc, split
  double form_route_flops = 0, eval_route_flops = 0;
  double host_tree_s = 0, host_lists_s = 0, host_plan_s = 0;
};

// Plan building in two halves around the tree build (shared by the host tree
// and the tree whose point work runs on the GPU):
//   plan_begin: parameters from the bounding-box results; false for the
//     large-delta path (no tree).  ts receives the tree-build settings.
//   plan_end: expansion lengths, tables and tasks once H.tree is complete;
//     beside (if given) runs on a second thread while the tables and tasks
//     are built, after the parameters it may read are final (the device
//     build of the near-field tasks, which reads H.P and H.tree only).
struct TreeSetup {
  int ndiv = 0, ndiv0 = 0, levcut = 0, nlmax = 0;
  double bs0 = 0, cen0[3] = {0, 0, 0};
};
bool plan_begin(HostPlan& H, int dim, int nd, double delta, double eps, int ns, int nt, int ifpgh,
                int ifpghtarg, int npwlevel, double bs0, const double* cen0, TreeSetup& ts,
                int ifcharge = 1, int ifdipole = 0);
void plan_end(HostPlan& H, const std::function<void()>& beside = nullptr);

int build_host_plan(HostPlan& H, int dim, int nd, double delta, double eps, int ns,
                    const double* sources, int nt, const double* targ, int ifpgh, int ifpghtarg,
                    int nthreads, int ifcharge = 1, int ifdipole = 0);
// Fills the plan from a tree that was built outside (the fgt2dmain entry).
int build_host_plan_from_tree(HostPlan& H, const Params& P0, const std::vector<int>& nlocal,
                              double pmax, int npw);

}  // namespace fgtb
