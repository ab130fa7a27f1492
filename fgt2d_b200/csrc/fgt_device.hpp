// Device side of a plan: task arrays and tables resident in HBM, expansion
// pools, scratch, and the stage launcher.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "fgt_plan.hpp"

namespace fgtb {

enum Precision { PREC_FP64 = 0, PREC_MIXED = 1 };

// Outputs per point and density for ifpgh = pgh: 1 (pot), 1 + dim (+ grad),
// 1 + dim + H (+ Hessian; H = 3 in 2D, 6 in 3D); 0 for pgh = 0.
inline int out_comps(int dim, int pgh) {
  return pgh <= 0 ? 0 : pgh == 1 ? 1 : pgh == 2 ? 1 + dim : 1 + dim + (dim == 2 ? 3 : 6);
}

// Caller-order device inputs of one execute: charge (nd, ns) when the plan
// has charges, rnormal (dim, ns) and dipstr (nd, ns) when it has dipoles.
struct Inputs {
  const double* charge = nullptr;
  const double* rnormal = nullptr;
  const double* dipstr = nullptr;
};

// Caller-order device outputs of one execute: pot (nd, ns), grad (nd, dim, ns),
// hess (nd, H, ns) and the same at the targets; the ones the flags do not ask
// for are ignored.
struct Outputs {
  double* pot = nullptr;
  double* grad = nullptr;
  double* hess = nullptr;
  double* pottarg = nullptr;
  double* gradtarg = nullptr;
  double* hesstarg = nullptr;
};

struct MergeGroup {
  int dst, beg, cnt;
};

struct OrderGroup {
  int p, beg, end;     // tasks [beg, end) of expansion order p
  long long tab = -1;  // offset of the group's operand tables in DevicePlan::tables (doubles)
};

// 2D Taylor evaluation in two kernels: one plane wave -> Taylor conversion per
// evaluation leaf (its block of nd * P * E doubles at `off`, E = P rounded up
// to even), then point chunks of <= 256 that read the block.
struct ConvTask {
  int slot, p;
  long long off;
  // split fused into the conversion: slot is then the cut-level ancestor's
  // local expansion and sh the leaf centre minus the ancestor's, scaled by
  // 1/sqrt(delta); the conversion multiplies the ancestor's coefficients by
  // exp(i t . sh) (3D: t_m3 sh0 + t_m2 sh1 + t_m1 sh2; 2D: t_j2 sh0 + t_J
  // sh1), the product of the split factors from the ancestor to the leaf
  int fused = 0;
  double sh[3] = {0, 0, 0};
};
struct HornerTask {
  int box, set, i0, n, p;
  long long off;
};

struct StageTimes {
  float ms[8];  // gather, form, merge, m2l, split, eval, direct, scatter
  // the dominant tensor-core launch: the Hermite-block MMA kernel of the
  // form group with the most sources (k_form2d_mma / k_form3d_mma)
  float dom_ms = 0;
  double dom_flops = 0;      // executed: 2 n P^dim (x nd) for that group
  double dom_alg_flops = 0;  // algorithmic: 4 n npw^dim (x nd), n = the group's sources
  char dom_name[48] = {0};
};

struct DevicePlan {
  Params P;
  int nboxes = 0, nch = 4;
  // buffers (one allocation, carved)
  char* base = nullptr;
  size_t bytes = 0;
  cudaStream_t stream = 0;  // stream of the stream-ordered allocation
  double* centers = nullptr;
  double* h2x = nullptr;
  double* x2l = nullptr;
  double2* wms = nullptr;
  double2* wsh = nullptr;
  int* isrc = nullptr;       // sorted position -> caller index
  int* itarg = nullptr;
  int* isrc_inv = nullptr;   // caller index -> sorted position
  int* itarg_inv = nullptr;
  double* isq = nullptr;     // 1/sqrt(j), j = 0..ntermmax+1
  double* cfac = nullptr;    // 1/sqrt(j!), j < 32
  FormTask* form = nullptr;
  int nform = 0;
  std::vector<int> merge_beg, merge_end;  // host copies of group ranges per level
  MergeGroup* mgroups = nullptr;
  ShiftTask* merge = nullptr;
  ShiftTask* split = nullptr;
  std::vector<int> split_beg, split_end;
  M2LTask* m2l = nullptr;
  int nm2l = 0;
  M2LNbr* m2l_nbr = nullptr;
  EvalTask* eval = nullptr;
  int neval = 0;
  DirTask* dir = nullptr;
  int ndir = 0;
  SrcRange* dir_src = nullptr;
  // pools and sorted data
  double2* mp = nullptr;
  double2* loc = nullptr;
  int nmp = 0, nloc = 0;
  double* ssort = nullptr;  // sorted sources (ns, dim)
  double* csort = nullptr;  // sorted charges (ns, nd)
  double* nsort = nullptr;  // sorted dipole directions (ns, dim), dipole plans only
  double* dsort = nullptr;  // sorted dipole strengths (ns, nd), dipole plans only
  double* tsort = nullptr;  // sorted targets (nt, dim)
  // the mixed near field's coordinates: (x - cen0) sqrt(log2 e / delta) split
  // into FP32 (hi, lo) pairs, per point [dim][2], sorted order (plans with a
  // near field and no dipoles; null otherwise)
  float* fsrc = nullptr;
  float* ftrg = nullptr;
  double* psort = nullptr;  // sorted source outputs, per point [out_comps(dim, ifpgh)][nd]
  double* ptsort = nullptr; // sorted target outputs, per point [out_comps(dim, ifpghtarg)][nd]
  double* local0 = nullptr; // large-delta local expansion
  // 3D Hermite form in two kernels: source chunks and their partial blocks
  FormChunk* fchunks = nullptr;
  int nfchunks = 0;
  int* fcbeg = nullptr;      // per Hermite form task, first chunk (size n+1)
  double* hbuf = nullptr;    // partial Hermite blocks
  bool form3_smem = false, eval3_smem = false;
  bool eval3_split = false;  // 3D Taylor eval in two kernels (conversion, Horner)
  int eval3_nsplit = 0;      // 3D Taylor tasks [0, eval3_nsplit) take the two kernels
  int form3_nsplit = 0;      // 3D Hermite form tasks [0, form3_nsplit) take the shared-memory kernels
  size_t form3_shB = 0, eval3_sh = 0;
  std::vector<OrderGroup> fchunk_groups;  // chunk ranges of equal order
  // per-CTA scratch of the 3D separable transforms (fallback path)
  double2* scratch = nullptr;
  size_t scratch_per_cta = 0;  // in double2
  int scratch_ctas = 0;
  // U2 scratch of the persistent 3D PW -> Taylor conversion: conv3_ctas CTAs
  // per density, uscr_per_cta doubles each
  double* uscr = nullptr;
  size_t uscr_per_cta = 0;
  int conv3_ctas = 0;
  // launch shapes
  int form_hermite_n = 0, form_pw_n = 0;
  int eval_taylor_n = 0, eval_pw_n = 0;
  int form_pmax = 0, eval_pmax = 0;  // largest order among Hermite form / Taylor eval tasks
  std::vector<OrderGroup> form_groups;
  int dom_form_group = -1;        // 2D: form group with the most sources (MMA kernels)
  int dom_fchunk_group = -1;      // 3D: chunk group with the most sources
  std::vector<double> group_flops;      // 2 n P^dim per form group (2D) / chunk group (3D)
  std::vector<double> group_alg_flops;  // 4 n npw^dim per form group (2D) / chunk group (3D)
  // 2D Taylor evaluation (conversion per leaf, then Horner per point chunk)
  long long* form_hoff = nullptr;  // 2D MMA form: per form task, offset of its Hermite block in hbuf
  ConvTask* conv = nullptr;
  HornerTask* horner = nullptr;
  double* lo = nullptr;
  double* tables = nullptr;  // padded operand tables of the 2D MMA transforms
  std::vector<OrderGroup> conv_groups, horner_groups;
  int sm_count = 148;
  // SMs the persistent kernels of this plan size their grids for (0: all);
  // a server caps it so that a large request's persistent kernels leave SMs
  // to the requests that arrive while they run
  int persist_sms = 0;
  int psm() const { return persist_sms > 0 && persist_sms < sm_count ? persist_sms : sm_count; }
  // One CTA per task instead of persistent CTAs, in the kernels whose CTAs
  // hold no per-CTA scratch: CTAs of other streams (a server's small
  // requests, on higher-priority streams) are then scheduled as soon as any
  // CTA of this plan finishes, not after the whole launch.
  bool yield_grids = false;
  int pgrid(int ntask, int per_sm) const {
    return yield_grids ? ntask : (ntask < psm() * per_sm ? ntask : psm() * per_sm);
  }
  // statistics copied from the host plan
  long long direct_pairs = 0, form_sources = 0, eval_points = 0;
  long long launches = 0;
  // algorithmic bytes of the split tasks that run (the others are fused into
  // the conversion): each distinct expansion read or written once, 16 B per
  // complex coefficient
  long long split_bytes = 0;
};

// Makes freed stream-ordered allocations stay in the current device's default
// memory pool (once per device).
cudaError_t device_pool_setup();

// Uploads the host plan; returns cudaSuccess or the first error.  The point
// permutations come from H.tree (host) or, when d_isrc is given, from device
// arrays (d_isrc: ns, d_itarg: nt) copied on stream st.  With size_only, only
// the device bytes the plan needs are computed (nothing is allocated).
cudaError_t device_plan_create(const HostPlan& H, DevicePlan& D, const int* d_isrc = nullptr,
                               const int* d_itarg = nullptr, cudaStream_t st = 0,
                               size_t* size_only = nullptr);

// Tree and plan with the point work of the tree build on the GPU
// (fgt_devtree.cu).  d_src (ns, dim) and d_trg (nt, dim) are device arrays in
// the caller's order (same: targets are the sources); the permutations
// (position -> input index) are written to d_isrc / d_itarg.  With keep, the
// exact-key form leaves the finished tree's box arrays on the device there
// (keep->mem non-null; the caller frees it on the stream).
cudaError_t build_tree_device(Tree& t, int dim, const double* d_src, int ns, const double* d_trg, int nt,
                              bool same, const TreeSetup& ts, int* d_isrc, int* d_itarg, cudaStream_t st,
                              HostPlan::DevTree* keep = nullptr);
// The near-field task arrays of a built host plan on the GPU (H.dnear,
// H.direct_pairs), in the order of the host's build, with list1 built there
// too (from H.dtree when the tree build left it, else from the host tree);
// device_near_free releases them and H.dtree (after device_plan_create has
// copied them).
cudaError_t build_near_tasks_device(HostPlan& H, cudaStream_t st);
void device_near_free(HostPlan& H, cudaStream_t st);
// Bounding box (per-dimension min / max) of device point arrays.
cudaError_t build_plan_device_bbox(const double* d_src, int ns, const double* d_trg, int nt, int dim,
                                   double* mn, double* mx, cudaStream_t st);
cudaError_t build_plan_device(HostPlan& H, int dim, int nd, double delta, double eps, int ns,
                              const double* d_src, int nt, const double* d_trg, bool same, int ifpgh,
                              int ifpghtarg, int* d_isrc, int* d_itarg, cudaStream_t st,
                              int ifcharge = 1, int ifdipole = 0);
void device_plan_destroy(DevicePlan& D);

// Sorts the plan's points into tree order once: device arrays in the
// caller's order, sources (ns, dim) and targets (nt, dim).
cudaError_t device_plan_set_points(DevicePlan& D, const double* src, const double* trg,
                                   cudaStream_t stream);
// Runs charge gather -> stages -> scatter on `stream`.  Device pointers in
// the caller's order: charge (ns, nd) and the outputs.
// times (optional) receives per-stage milliseconds (synchronises).
// phase: 0 everything; 1 through the merge (every mp expansion up to the
// cut level), 2 from mp -> loc on (the caller may replace mp expansions of
// the cut level between the two).
cudaError_t device_plan_execute(DevicePlan& D, const Inputs& in, const Outputs& out,
                                int precision, cudaStream_t stream, StageTimes* times, int phase = 0);

// Sets *d_flag (device int, not cleared here) when any of x[0, n) is not
// finite; asynchronous on st.
cudaError_t device_check_finite(const double* x, size_t n, int* d_flag, cudaStream_t st);

// Measures the FP64 tensor-core (mma.m8n8k4.f64) throughput of the current
// device in TFLOP/s.
cudaError_t probe_fp64_mma(double* tflops);

// The tensor-core kernels' device error flag on the current device (set when
// a wait on an MMA completion gave up); cleared on request.
cudaError_t tc_error_flag(int* flag, bool clear);
// One BF16 x 3 tcgen05 tile (M = 128, K = 16, N) on the current device
// against an FP64 product on the host: the largest error relative to the
// largest entry.
cudaError_t tc_selftest(int N, double* max_rel_err);

// Large-delta path with its scratch in a fixed device array instead of
// `work`: no allocation.  cudaErrorInvalidValue when nd (nlocal0+1)^dim
// exceeds large_delta_noalloc_capacity() doubles.
cudaError_t large_delta_noalloc(const Params& P, const double* src, const double* chg,
                                const double* trg, double* pot, double* pottarg,
                                cudaStream_t stream);
size_t large_delta_noalloc_capacity();

// Large-delta path (one Taylor local about the root centre), no tree.
// deterministic: the sources' contributions are summed in a fixed order
// through per-CTA partial blocks (work must hold large_delta_work_doubles(P,
// true) doubles); otherwise they are added atomically (nd (nlocal0+1)^dim
// doubles of work; results can differ in the last bits from call to call).
cudaError_t large_delta_execute(const Params& P, const double* src, const Inputs& in,
                                const double* trg, const Outputs& out, double* work,
                                cudaStream_t stream, bool deterministic);
size_t large_delta_work_doubles(const Params& P, bool deterministic);

}  // namespace fgtb
