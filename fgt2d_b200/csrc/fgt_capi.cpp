// C ABI of the B200 plane-wave FGT (declared in include/fgt_b200.h).
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <condition_variable>
#include <functional>
#include <thread>
#include <unordered_map>
#include <memory>
#include <mutex>
#include <new>
#include <vector>

#include <malloc.h>
#include <omp.h>

#include "fgt_b200.h"
#include "fgt_device.hpp"
#include "fgt_plan.hpp"
#include "fgt_shard.hpp"

using namespace fgtb;

struct fgt_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int precision = FGT_PREC_AUTO;
  int tree = FGT_TREE_DEVICE;
  int nthreads = 0;
  int sm_budget = 0;  // SMs the persistent kernels of this context's plans size their grids for (0: all)
  bool yield_grids = false;  // one CTA per task where a kernel allows it (DevicePlan::yield_grids)
  int scheme = FGT_SCHEME_PLANEWAVE;  // the algorithm of the context's plans
  // uploads of a one-shot call's source strengths: they follow the points on
  // the copy engine while the tree build runs on `stream`
  cudaStream_t up_stream = nullptr;
  std::mutex mu;
};

struct fgt_plan {
  fgt_ctx* ctx = nullptr;
  HostPlan H;
  DevicePlan D;
  bool have_device = false;
  // device copies of the caller-order arrays for the host-array entry points
  double* d_io = nullptr;
  size_t io_bytes = 0;
  double* d_src = nullptr;
  double* d_chg = nullptr;
  double* d_trg = nullptr;
  double* d_pot = nullptr;
  double* d_pottarg = nullptr;
  double* d_rn = nullptr;        // dipole directions and strengths (dipole plans)
  double* d_ds = nullptr;
  double* d_grad = nullptr;      // gradients / Hessians when the flags ask for them
  double* d_hess = nullptr;
  double* d_gradtarg = nullptr;
  double* d_hesstarg = nullptr;
  double* d_work = nullptr;  // large-delta local expansion
  int* d_flag = nullptr;     // device-side argument checks
  int last_launches = 0;
  // host strengths of a one-shot call, uploaded with the points so the copy
  // overlaps the host part of the plan build (exec_host then skips it)
  const double* pre_q = nullptr;
  const double* pre_rn = nullptr;
  const double* pre_ds = nullptr;
  cudaEvent_t pre_done = nullptr;  // the strengths' uploads on the context's up_stream
  // recorded after every execute on the stream it used: the frees of
  // fgt_plan_destroy (stream-ordered on the context's stream) wait for it
  cudaEvent_t done = nullptr;
  // spatial shard (fgt_plan_create_shard): this rank's part of the tasks and
  // the cut-level mp slots it exchanges; d_xslots holds every peer's send
  // list, then every peer's receive list
  int shard_n = 1, shard_r = 0;
  ShardInfo shard;
  int* d_xslots = nullptr;
  std::vector<long long> xsend_off, xrecv_off;
};

namespace {
thread_local int g_last_cuda = 0;

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return FGT_OK;
  g_last_cuda = (int)e;
  if (e == cudaErrorMemoryAllocation) return FGT_ERR_NOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return FGT_ERR_NODEVICE;
  if (e == cudaErrorNotSupported) return FGT_ERR_UNSUPPORTED;
  return FGT_ERR_CUDA;
}
#define CKS(x)                                 \
  do {                                         \
    int s_ = cuda_status(x);                   \
    if (s_ != FGT_OK) return s_;               \
  } while (0)

int resolve_precision(const fgt_ctx* c, double eps) {
  if (c->precision == FGT_PREC_AUTO) return eps >= 1e-6 ? PREC_MIXED : PREC_FP64;
  return c->precision == FGT_PREC_MIXED ? PREC_MIXED : PREC_FP64;
}

bool finite_all(const double* a, size_t n) {
  if (!a) return n == 0;
  for (size_t i = 0; i < n; i++)
    if (!std::isfinite(a[i])) return false;
  return true;
}

// Argument checks; scan_points = false leaves the finiteness of the point
// coordinates to a device-side check after the upload.
int check_args(int dim, int nd, double delta, double eps, int ns, const double* sources,
               int ifcharge, int ifdipole, int ifpgh, int nt, const double* targ, int ifpghtarg,
               bool scan_points = true) {
  if (dim != 2 && dim != 3) return FGT_ERR_BADARG;
  if (nd < 1 || !(delta > 0) || !std::isfinite(delta) || !(eps > 0) || !(eps < 1)) return FGT_ERR_BADARG;
  if (ns < 0 || nt < 0) return FGT_ERR_BADARG;
  if (ns > 0 && !sources) return FGT_ERR_BADARG;
  if (nt > 0 && ifpghtarg > 0 && !targ) return FGT_ERR_BADARG;
  if (scan_points && !finite_all(sources, (size_t)ns * dim)) return FGT_ERR_BADARG;
  if (scan_points && nt > 0 && targ && !finite_all(targ, (size_t)nt * dim)) return FGT_ERR_BADARG;
  if (ifcharge < 0 || ifcharge > 1 || ifdipole < 0 || ifdipole > 1) return FGT_ERR_UNSUPPORTED;
  if (ifpgh < 0 || ifpgh > 3 || ifpghtarg < 0 || ifpghtarg > 3) return FGT_ERR_UNSUPPORTED;
  return FGT_OK;
}

// Device copies of the caller-order arrays (sources, charges, targets and
// the outputs the flags ask for) and n_work doubles of large-delta work in one
// allocation; uploads the points.
int alloc_io(fgt_plan* p, int dim, int nd, int ns, int nt, int ifpgh, int ifpghtarg, size_t n_work,
             const double* src_host, const double* trg_host, bool upload_trg, int ifdipole = 0) {
  const size_t nh = dim == 2 ? 3 : 6;
  size_t n_src = (size_t)ns * dim, n_chg = (size_t)ns * nd, n_trg = (size_t)nt * dim;
  size_t n_rn = ifdipole ? (size_t)ns * dim : 0, n_ds = ifdipole ? (size_t)ns * nd : 0;
  size_t n_pot = (size_t)ns * nd, n_pt = (size_t)nt * nd;
  size_t n_g = ifpgh >= 2 ? n_pot * dim : 0, n_h = ifpgh >= 3 ? n_pot * nh : 0;
  size_t n_gt = ifpghtarg >= 2 ? n_pt * dim : 0, n_ht = ifpghtarg >= 3 ? n_pt * nh : 0;
  auto al = [](size_t n) { return (n + 31) & ~size_t(31); };
  p->io_bytes = 8 * (al(n_src) + al(n_chg) + al(n_trg) + al(n_pot) + al(n_pt) + al(n_g) + al(n_h) +
                     al(n_gt) + al(n_ht) + al(n_rn) + al(n_ds) + al(n_work) + 32);
  CKS(device_pool_setup());
  CKS(cudaMallocAsync(reinterpret_cast<void**>(&p->d_io), p->io_bytes, p->ctx->stream));
  double* c = p->d_io;
  p->d_src = c; c += al(n_src);
  p->d_chg = c; c += al(n_chg);
  p->d_trg = c; c += al(n_trg);
  p->d_pot = c; c += al(n_pot);
  p->d_pottarg = c; c += al(n_pt);
  p->d_grad = n_g ? c : nullptr; c += al(n_g);
  p->d_hess = n_h ? c : nullptr; c += al(n_h);
  p->d_gradtarg = n_gt ? c : nullptr; c += al(n_gt);
  p->d_hesstarg = n_ht ? c : nullptr; c += al(n_ht);
  p->d_rn = n_rn ? c : nullptr; c += al(n_rn);
  p->d_ds = n_ds ? c : nullptr; c += al(n_ds);
  p->d_work = c; c += al(n_work);
  p->d_flag = reinterpret_cast<int*>(c);
  cudaStream_t st = p->ctx->stream;
  if (ns > 0) CKS(cudaMemcpyAsync(p->d_src, src_host, n_src * 8, cudaMemcpyHostToDevice, st));
  if (nt > 0 && upload_trg) CKS(cudaMemcpyAsync(p->d_trg, trg_host, n_trg * 8, cudaMemcpyHostToDevice, st));
  // the strengths go up on the side stream once the points are up, so the
  // tree build (which needs only the points) does not wait for them; the
  // execute waits for pre_done
  if (ns > 0 && (p->pre_q || (p->pre_rn && p->d_rn) || (p->pre_ds && p->d_ds))) {
    if (!p->ctx->up_stream) CKS(cudaStreamCreateWithFlags(&p->ctx->up_stream, cudaStreamNonBlocking));
    if (!p->pre_done) CKS(cudaEventCreateWithFlags(&p->pre_done, cudaEventDisableTiming));
    cudaStream_t us = p->ctx->up_stream;
    CKS(cudaEventRecord(p->pre_done, st));
    CKS(cudaStreamWaitEvent(us, p->pre_done, 0));
    if (p->pre_q) CKS(cudaMemcpyAsync(p->d_chg, p->pre_q, n_chg * 8, cudaMemcpyHostToDevice, us));
    if (p->pre_rn && p->d_rn) CKS(cudaMemcpyAsync(p->d_rn, p->pre_rn, n_rn * 8, cudaMemcpyHostToDevice, us));
    if (p->pre_ds && p->d_ds) CKS(cudaMemcpyAsync(p->d_ds, p->pre_ds, n_ds * 8, cudaMemcpyHostToDevice, us));
    CKS(cudaEventRecord(p->pre_done, us));
  }
  return FGT_OK;
}

// Device-side finiteness check of n doubles at d (synchronises).
int check_finite_device(fgt_plan* p, const double* d, size_t n) {
  if (n == 0) return FGT_OK;
  cudaStream_t st = p->ctx->stream;
  int bad = 0;
  CKS(cudaMemsetAsync(p->d_flag, 0, sizeof(int), st));
  CKS(device_check_finite(d, n, p->d_flag, st));
  CKS(cudaMemcpyAsync(&bad, p->d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKS(cudaStreamSynchronize(st));
  return bad ? FGT_ERR_BADARG : FGT_OK;
}

int plan_device(fgt_plan* p, const double* src_host, const double* trg_host) {
  const Params& P = p->H.P;
  const size_t n_work = P.large_delta ? large_delta_work_doubles(P, true) : 0;
  const int sa = alloc_io(p, P.dim, P.nd, P.ns, P.nt, P.ifpgh, P.ifpghtarg, n_work, src_host, trg_host,
                         P.ifpghtarg > 0, P.ifdipole);
  if (sa != FGT_OK) return sa;
  cudaStream_t st = p->ctx->stream;
  if (shard_filter(p->H, p->shard_n, p->shard_r, p->shard) != 0) return FGT_ERR_BADARG;
  if (!P.large_delta) {
    CKS(device_plan_create(p->H, p->D));
    p->have_device = true;
    p->D.persist_sms = p->ctx->sm_budget;
  p->D.yield_grids = p->ctx->yield_grids;
    CKS(device_plan_set_points(p->D, p->d_src, p->d_trg, st));
  }
  return FGT_OK;
}

// Plan whose tree build does its point work on the GPU (fgt_devtree.cu).  The
// largest large-delta order is not known before the bounding box, so that
// path re-allocates its work array once the order is.
// admit (optional) is called with the device bytes of the plan proper once
// the tree is built and before they are allocated; it may block, and a
// status other than FGT_OK abandons the plan.
// The OpenMP team of a plan's host work: the context's setting, else half
// the cores and at most 8.  On the 16-core benchmark host the full team lost
// time to threads descheduled at its barriers (the drop-in call 12.2-16 ms
// with 16 threads, 11.4-12.0 ms with 8).  The calling thread's setting comes
// back when the guard ends.
struct OmpTeam {
  int old;
  explicit OmpTeam(const fgt_ctx* c) : old(omp_get_max_threads()) {
    omp_set_num_threads(c && c->nthreads > 0 ? c->nthreads : std::max(1, std::min(8, omp_get_num_procs() / 2)));
  }
  ~OmpTeam() { omp_set_num_threads(old); }
};

int plan_create_device_tree(fgt_plan* p, int dim, int nd, double delta, double eps, int ns,
                            const double* sources, int nt, const double* targ, int ifpgh, int ifpghtarg,
                            const std::function<int(size_t)>* admit = nullptr, int ifcharge = 1,
                            int ifdipole = 0) {
  OmpTeam team(p->ctx);
  const bool same = targ == sources && nt == ns;
  int st = alloc_io(p, dim, nd, ns, nt, ifpgh, ifpghtarg, 0, sources, targ, !same, ifdipole);
  if (st != FGT_OK) return st;
  const double tq0 = now_s();
  st = check_finite_device(p, p->d_src, (size_t)ns * dim);
  if (st == FGT_OK && !same) st = check_finite_device(p, p->d_trg, (size_t)nt * dim);
  if (st != FGT_OK) return st;
  if (getenv("FGT_TREE_TIMING")) fprintf(stderr, "plan: points up and checked %.4f\n", now_s() - tq0);
  cudaStream_t s = p->ctx->stream;
  const double* d_trg = same ? p->d_src : p->d_trg;
  int* perms = nullptr;
  CKS(cudaMallocAsync(reinterpret_cast<void**>(&perms), sizeof(int) * ((size_t)ns + nt + 2), s));
  struct Free {
    int* q;
    cudaStream_t st;
    ~Free() { cudaFreeAsync(q, st); }
  } fr{perms, s};
  int *d_isrc = perms, *d_itarg = perms + ns + 1;
  // an unsharded plan builds its near-field task arrays on the GPU; a shard
  // filters them on the host
  p->H.defer_near = p->shard_n <= 1;
  struct NearFree {
    HostPlan& h;
    cudaStream_t st;
    ~NearFree() { device_near_free(h, st); }  // copied into the plan's arena, or abandoned
  } nf{p->H, s};
  try {
    CKS(build_plan_device(p->H, dim, nd, delta, eps, ns, p->d_src, nt, d_trg, same, ifpgh, ifpghtarg,
                          d_isrc, d_itarg, s, ifcharge, ifdipole));
  } catch (const std::bad_alloc&) {
    return FGT_ERR_NOMEM;
  }
  const Params& P = p->H.P;
  const double tP = now_s();
  if (P.large_delta) {
    // same layout as plan_device, with the work array of the known order
    std::vector<double> hs((size_t)ns * dim), ht(same ? 0 : (size_t)nt * dim);
    CKS(cudaMemcpyAsync(hs.data(), p->d_src, hs.size() * 8, cudaMemcpyDeviceToHost, s));
    if (!same && nt > 0) CKS(cudaMemcpyAsync(ht.data(), p->d_trg, ht.size() * 8, cudaMemcpyDeviceToHost, s));
    if (p->pre_done) CKS(cudaStreamWaitEvent(s, p->pre_done, 0));  // the strengths' uploads into d_io
    CKS(cudaStreamSynchronize(s));
    cudaFreeAsync(p->d_io, s);
    p->d_io = nullptr;
    return plan_device(p, hs.data(), same ? hs.data() : ht.data());
  }
  if (same && nt > 0) CKS(cudaMemcpyAsync(p->d_trg, p->d_src, (size_t)nt * dim * 8, cudaMemcpyDeviceToDevice, s));
  if (shard_filter(p->H, p->shard_n, p->shard_r, p->shard) != 0) return FGT_ERR_BADARG;
  if (p->H.defer_near && p->H.tree.nboxes > 0 && !p->H.near_built) {
    const double tn = now_s();
    const cudaError_t e = build_near_tasks_device(p->H, s);
    if (e != cudaSuccess) {
      device_near_free(p->H, s);
      return cuda_status(e);
    }
    p->H.host_plan_s += now_s() - tn;
    if (getenv("FGT_TREE_TIMING")) fprintf(stderr, "near-field tasks (device): %.4f\n", now_s() - tn);
  }
  if (admit) {
    size_t bytes = 0;
    DevicePlan probe;
    CKS(device_plan_create(p->H, probe, d_isrc, d_itarg, s, &bytes));
    st = (*admit)(bytes);
    if (st != FGT_OK) return st;
  }
  CKS(device_plan_create(p->H, p->D, d_isrc, d_itarg, s));
  p->have_device = true;
  p->D.persist_sms = p->ctx->sm_budget;
  p->D.yield_grids = p->ctx->yield_grids;
  CKS(device_plan_set_points(p->D, p->d_src, p->d_trg, s));
  CKS(cudaStreamSynchronize(s));
  if (getenv("FGT_TREE_TIMING"))
    fprintf(stderr, "plan: tree %.4f lists %.4f tasks %.4f device plan %.4f\n", p->H.host_tree_s,
            p->H.host_lists_s, p->H.host_plan_s, now_s() - tP);
  return FGT_OK;
}

// Outputs the plan's flags ask for must be non-null except gradients and
// Hessians, which are skipped when null.
int run_device(fgt_plan* p, const Inputs& in, const Outputs& o, cudaStream_t st, StageTimes* times,
               int phase = 0) {
  const Params& P = p->H.P;
  if ((P.ifpgh > 0 && P.ns > 0 && !o.pot) || (P.ifpghtarg > 0 && P.nt > 0 && !o.pottarg))
    return FGT_ERR_BADARG;
  if ((P.ifcharge && !in.charge) || (P.ifdipole && (!in.rnormal || !in.dipstr))) return FGT_ERR_BADARG;
  int prec = resolve_precision(p->ctx, P.eps);
  if (!p->done) CKS(cudaEventCreateWithFlags(&p->done, cudaEventDisableTiming));
  if (!P.ifcharge && !P.ifdipole) {  // no sources of either kind: zero fields
    const size_t nd = P.nd, nh = P.dim == 2 ? 3 : 6;
    auto z = [&](double* a, size_t n) { return a && n ? cudaMemsetAsync(a, 0, n * 8, st) : cudaSuccess; };
    if (P.ifpgh >= 1) CKS(z(o.pot, P.ns * nd));
    if (P.ifpgh >= 2) CKS(z(o.grad, P.ns * nd * P.dim));
    if (P.ifpgh >= 3) CKS(z(o.hess, P.ns * nd * nh));
    if (P.ifpghtarg >= 1) CKS(z(o.pottarg, P.nt * nd));
    if (P.ifpghtarg >= 2) CKS(z(o.gradtarg, P.nt * nd * P.dim));
    if (P.ifpghtarg >= 3) CKS(z(o.hesstarg, P.nt * nd * nh));
    p->last_launches = 0;
    CKS(cudaEventRecord(p->done, st));
    return FGT_OK;
  }
  if (P.large_delta && p->shard.large_delta_idle) {
    // a shard rank other than 0 of a large-delta plan: its part is zero
    const size_t nd = P.nd, nh = P.dim == 2 ? 3 : 6;
    auto z = [&](double* a, size_t n) { return a && n ? cudaMemsetAsync(a, 0, n * 8, st) : cudaSuccess; };
    if (P.ifpgh >= 1) CKS(z(o.pot, P.ns * nd));
    if (P.ifpgh >= 2) CKS(z(o.grad, P.ns * nd * P.dim));
    if (P.ifpgh >= 3) CKS(z(o.hess, P.ns * nd * nh));
    if (P.ifpghtarg >= 1) CKS(z(o.pottarg, P.nt * nd));
    if (P.ifpghtarg >= 2) CKS(z(o.gradtarg, P.nt * nd * P.dim));
    if (P.ifpghtarg >= 3) CKS(z(o.hesstarg, P.nt * nd * nh));
    p->last_launches = 0;
  } else if (P.large_delta) {
    Outputs lo = o;  // the large-delta kernels write every component they compute
    double* dg[4] = {p->d_grad, p->d_hess, p->d_gradtarg, p->d_hesstarg};
    double** og[4] = {&lo.grad, &lo.hess, &lo.gradtarg, &lo.hesstarg};
    for (int i = 0; i < 4; i++)
      if (!*og[i]) *og[i] = dg[i];
    CKS(large_delta_execute(P, p->d_src, in, p->d_trg, lo, p->d_work, st, true));
    p->last_launches = (P.ns > 0) + (P.ifpgh >= 1) + (P.ifpghtarg >= 1);
  } else {
    CKS(device_plan_execute(p->D, in, o, prec, st, times, phase));
    p->last_launches = (int)p->D.launches;
  }
  CKS(cudaEventRecord(p->done, st));
  return FGT_OK;
}

// Source strengths in from the host (charges and/or dipole directions and
// strengths, as the plan's flags say), every execute output the plan
// computes back to the non-null host arrays of `host`.
int exec_host(fgt_plan* p, const double* charge, const Outputs& host, const double* rnormal = nullptr,
              const double* dipstr = nullptr) {
  OmpTeam team(p->ctx);
  const Params& P = p->H.P;
  cudaStream_t st = p->ctx->stream;
  CKS(cudaSetDevice(p->ctx->device));
  const size_t ns = P.ns, nt = P.nt, nd = P.nd, nh = P.dim == 2 ? 3 : 6;
  if (p->pre_done) CKS(cudaStreamWaitEvent(st, p->pre_done, 0));  // strengths uploaded with the points
  Inputs in;
  if (P.ifcharge) {
    if (!charge && ns) return FGT_ERR_BADARG;
    if (charge != p->pre_q) CKS(cudaMemcpyAsync(p->d_chg, charge, ns * nd * 8, cudaMemcpyHostToDevice, st));
    int s = check_finite_device(p, p->d_chg, ns * nd);
    if (s != FGT_OK) return s;
    in.charge = p->d_chg;
  }
  if (P.ifdipole) {
    if ((!rnormal || !dipstr) && ns) return FGT_ERR_BADARG;
    if (rnormal != p->pre_rn) CKS(cudaMemcpyAsync(p->d_rn, rnormal, ns * P.dim * 8, cudaMemcpyHostToDevice, st));
    if (dipstr != p->pre_ds) CKS(cudaMemcpyAsync(p->d_ds, dipstr, ns * nd * 8, cudaMemcpyHostToDevice, st));
    int s = check_finite_device(p, p->d_rn, ns * P.dim);
    if (s == FGT_OK) s = check_finite_device(p, p->d_ds, ns * nd);
    if (s != FGT_OK) return s;
    in.rnormal = p->d_rn;
    in.dipstr = p->d_ds;
  }
  Outputs d;
  d.pot = p->d_pot; d.grad = p->d_grad; d.hess = p->d_hess;
  d.pottarg = p->d_pottarg; d.gradtarg = p->d_gradtarg; d.hesstarg = p->d_hesstarg;
  const double tx0 = now_s();
  if (getenv("FGT_TREE_TIMING")) cudaStreamSynchronize(st);
  const double tx1 = now_s();
  int s = run_device(p, in, d, st, nullptr);
  if (getenv("FGT_TREE_TIMING")) cudaStreamSynchronize(st);
  const double tx2 = now_s();
  if (getenv("FGT_TREE_TIMING")) fprintf(stderr, "exec_host: inputs %.4f run %.4f\n", tx1 - tx0, tx2 - tx1);
  if (s != FGT_OK) return s;
  auto back = [&](double* h, const double* dv, size_t n) -> cudaError_t {
    return h && dv && n ? cudaMemcpyAsync(h, dv, n * 8, cudaMemcpyDeviceToHost, st) : cudaSuccess;
  };
  if (P.ifpgh >= 1) CKS(back(host.pot, d.pot, ns * nd));
  if (P.ifpgh >= 2) CKS(back(host.grad, d.grad, ns * nd * P.dim));
  if (P.ifpgh >= 3) CKS(back(host.hess, d.hess, ns * nd * nh));
  if (P.ifpghtarg >= 1) CKS(back(host.pottarg, d.pottarg, nt * nd));
  if (P.ifpghtarg >= 2) CKS(back(host.gradtarg, d.gradtarg, nt * nd * P.dim));
  if (P.ifpghtarg >= 3) CKS(back(host.hesstarg, d.hesstarg, nt * nd * nh));
  CKS(cudaStreamSynchronize(st));
  if (getenv("FGT_TREE_TIMING")) fprintf(stderr, "exec_host: outputs down %.4f\n", now_s() - tx2);
  return FGT_OK;
}

int plan_create_impl(fgt_ctx* ctx, int dim, int nd, double delta, double eps, int ns,
                     const double* sources, int nt, const double* targ, int ifcharge, int ifdipole,
                     int ifpgh, int ifpghtarg, fgt_plan** out, const double* pre_q = nullptr,
                     const double* pre_rn = nullptr, const double* pre_ds = nullptr);

int transform_impl(fgt_ctx* ctx, int dim, int nd, double delta, double eps, int ns,
                   const double* sources, int ifcharge, const double* charge, int ifdipole,
                   const double* rnormal, const double* dipstr,
                   int ifpgh, double* pot, double* grad, double* hess, int nt, const double* targ,
                   int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg) {
  const bool on_device = ctx->tree == FGT_TREE_DEVICE;
  int st = check_args(dim, nd, delta, eps, ns, sources, ifcharge, ifdipole, ifpgh, nt, targ, ifpghtarg,
                      !on_device);
  if (st != FGT_OK) return st;
  if (ns > 0 && ((ifcharge && !charge) || (ifdipole && (!rnormal || !dipstr)))) return FGT_ERR_BADARG;
  if (!on_device && ns > 0 && ifcharge && !finite_all(charge, (size_t)ns * nd)) return FGT_ERR_BADARG;
  // outputs are written in full on success; zero them when nothing runs or
  // the call fails
  const size_t nh = dim == 2 ? 3 : 6;
  if ((ifpgh >= 1 && ns > 0 && !pot) || (ifpgh >= 2 && ns > 0 && !grad) || (ifpgh >= 3 && ns > 0 && !hess) ||
      (ifpghtarg >= 1 && nt > 0 && !pottarg) || (ifpghtarg >= 2 && nt > 0 && !gradtarg) ||
      (ifpghtarg >= 3 && nt > 0 && !hesstarg))
    return FGT_ERR_BADARG;
  auto zero = [&] {
    auto z = [](double* a, size_t n) { if (a && n) memset(a, 0, sizeof(double) * n); };
    if (ifpgh >= 1) z(pot, (size_t)ns * nd);
    if (ifpgh >= 2) z(grad, (size_t)ns * nd * dim);
    if (ifpgh >= 3) z(hess, (size_t)ns * nd * nh);
    if (ifpghtarg >= 1) z(pottarg, (size_t)nt * nd);
    if (ifpghtarg >= 2) z(gradtarg, (size_t)nt * nd * dim);
    if (ifpghtarg >= 3) z(hesstarg, (size_t)nt * nd * nh);
  };
  if (ns == 0) {
    zero();
    return FGT_OK;
  }
  fgt_plan* plan = nullptr;
  const double ta = now_s();
  st = plan_create_impl(ctx, dim, nd, delta, eps, ns, sources, nt, targ, ifcharge, ifdipole, ifpgh,
                        ifpghtarg, &plan, ifcharge ? charge : nullptr, ifdipole ? rnormal : nullptr,
                        ifdipole ? dipstr : nullptr);
  const double tb = now_s();
  if (st == FGT_OK) {
    Outputs h;
    h.pot = pot; h.grad = grad; h.hess = hess;
    h.pottarg = pottarg; h.gradtarg = gradtarg; h.hesstarg = hesstarg;
    st = exec_host(plan, charge, h, rnormal, dipstr);
    const double tc = now_s();
    fgt_plan_destroy(plan);
    if (getenv("FGT_TREE_TIMING"))
      fprintf(stderr, "transform: plan %.4f execute+outputs %.4f destroy %.4f\n", tb - ta, tc - tb, now_s() - tc);
  }
  if (st != FGT_OK) zero();
  return st;
}

std::once_flag g_default_once;
fgt_ctx* g_default = nullptr;

void report(const char* who, int st) {
  if (st != FGT_OK)
    fprintf(stderr, "%s: failed with status %d (%s), cuda error %d\n", who, st, fgt_status_string(st),
            g_last_cuda);
}
}  // namespace

extern "C" {

const char* fgt_status_string(int s) {
  switch (s) {
    case FGT_OK: return "ok";
    case FGT_ERR_BADARG: return "bad argument";
    case FGT_ERR_UNSUPPORTED: return "unsupported option";
    case FGT_ERR_NOMEM: return "out of memory";
    case FGT_ERR_CUDA: return "CUDA error";
    case FGT_ERR_NODEVICE: return "no CUDA device";
    case FGT_ERR_SCRATCH: return "problem exceeds the fixed scratch of the allocation-free call";
    default: return "unknown status";
  }
}
int fgt_last_cuda_error(void) { return g_last_cuda; }
const char* fgt_build_info(void) { return "fgt_b200 sm_100a FP64+mixed near field"; }

int fgt_ctx_create(int device, fgt_ctx** out) {
  if (!out) return FGT_ERR_BADARG;
  *out = nullptr;
  // The plan build's host arrays (tree, lists, task arrays: tens of MB for
  // 1e7 points) are allocated afresh per plan; glibc serves blocks that size
  // with mmap and returns them on free, so every plan paid a page fault per
  // 4 KB touched (about half of the host build time measured).  Keeping them
  // in the heap (mmap threshold at its 32 MB maximum, no trimming below
  // 1 GB) lets later plans reuse faulted pages.  Process-wide, set once;
  // FGT_KEEP_MALLOC=1 leaves glibc's defaults alone.
  static std::once_flag malloc_once;
  std::call_once(malloc_once, [] {
    const char* e = getenv("FGT_KEEP_MALLOC");
    if (!(e && e[0] == '1')) {
      mallopt(M_MMAP_THRESHOLD, 32 << 20);
      mallopt(M_TRIM_THRESHOLD, 1 << 30);
    }
  });
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return FGT_ERR_NODEVICE;
  if (device < 0 || device >= n) return FGT_ERR_BADARG;
  fgt_ctx* c = new (std::nothrow) fgt_ctx();
  if (!c) return FGT_ERR_NOMEM;
  c->device = device;
  int s = cuda_status(cudaSetDevice(device));
  if (s == FGT_OK) s = cuda_status(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  if (s != FGT_OK) {
    delete c;
    return s;
  }
  *out = c;
  return FGT_OK;
}
int fgt_ctx_destroy(fgt_ctx* c) {
  if (!c) return FGT_ERR_BADARG;
  if (c == g_default) return FGT_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->up_stream) cudaStreamDestroy(c->up_stream);
  delete c;
  return FGT_OK;
}
int fgt_ctx_set_precision(fgt_ctx* c, int precision) {
  if (!c || precision < 0 || precision > 2) return FGT_ERR_BADARG;
  c->precision = precision;
  return FGT_OK;
}
int fgt_ctx_set_tree(fgt_ctx* c, int where) {
  if (!c || (where != FGT_TREE_DEVICE && where != FGT_TREE_HOST)) return FGT_ERR_BADARG;
  c->tree = where;
  return FGT_OK;
}
int fgt_ctx_set_scheme(fgt_ctx* c, int scheme) {
  if (!c || (scheme != FGT_SCHEME_PLANEWAVE && scheme != FGT_SCHEME_NUFFT)) return FGT_ERR_BADARG;
  c->scheme = scheme;
  return FGT_OK;
}
int fgt_ctx_set_sm_budget(fgt_ctx* c, int sms) {
  if (!c || sms < 0) return FGT_ERR_BADARG;
  c->sm_budget = sms;
  return FGT_OK;
}
int fgt_ctx_set_grid_yield(fgt_ctx* c, int on) {
  if (!c) return FGT_ERR_BADARG;
  c->yield_grids = on != 0;
  return FGT_OK;
}
int fgt_ctx_set_host_threads(fgt_ctx* c, int nthreads) {
  if (!c) return FGT_ERR_BADARG;
  c->nthreads = nthreads;
  return FGT_OK;
}
int fgt_large_delta_noalloc(int dim, int nd, double delta, int ns, const double* sources,
                            const double* charge, int nlocal, const double* center, int ifpgh,
                            double* pot, int nt, const double* targ, int ifpghtarg,
                            double* pottarg, void* stream) {
  if ((dim != 2 && dim != 3) || nd < 1 || !(delta > 0) || !std::isfinite(delta) || ns < 0 ||
      nt < 0 || nlocal < 0 || !center)
    return FGT_ERR_BADARG;
  if (ifpgh < 0 || ifpgh > 1 || ifpghtarg < 0 || ifpghtarg > 1) return FGT_ERR_UNSUPPORTED;
  if ((ns > 0 && (!sources || !charge)) || (ifpgh == 1 && ns > 0 && !pot) ||
      (ifpghtarg == 1 && nt > 0 && (!targ || !pottarg)))
    return FGT_ERR_BADARG;
  for (int d = 0; d < dim; d++)
    if (!std::isfinite(center[d])) return FGT_ERR_BADARG;
  const size_t Pn = (size_t)nlocal + 1;
  if ((double)nd * std::pow((double)Pn, dim) > (double)large_delta_noalloc_capacity())
    return FGT_ERR_SCRATCH;
  Params P;
  P.dim = dim; P.nd = nd; P.delta = delta; P.dsq = 1.0 / std::sqrt(delta);
  P.ns = ns; P.nt = nt; P.ifpgh = ifpgh; P.ifpghtarg = ifpghtarg;
  P.large_delta = true; P.nlocal0 = nlocal;
  for (int d = 0; d < dim; d++) P.cen0[d] = center[d];
  CKS(large_delta_noalloc(P, sources, charge, targ, pot, pottarg, (cudaStream_t)stream));
  return FGT_OK;
}

int fgt_tc_selftest(int device, int n, double* max_rel_err) {
  if (!max_rel_err || n < 16 || n > 256 || n % 16) return FGT_ERR_BADARG;
  CKS(cudaSetDevice(device));
  CKS(tc_selftest(n, max_rel_err));
  return FGT_OK;
}
int fgt_tc_error(int device, int clear, int* flag) {
  if (!flag) return FGT_ERR_BADARG;
  CKS(cudaSetDevice(device));
  CKS(tc_error_flag(flag, clear != 0));
  return FGT_OK;
}

int fgt_probe_fp64_mma_tflops(fgt_ctx* c, double* tflops) {
  if (!c || !tflops) return FGT_ERR_BADARG;
  CKS(cudaSetDevice(c->device));
  CKS(probe_fp64_mma(tflops));
  return FGT_OK;
}
void* fgt_ctx_stream(fgt_ctx* c) { return c ? (void*)c->stream : nullptr; }
fgt_ctx* fgt_default_ctx(void) {
  std::call_once(g_default_once, [] {
    fgt_ctx* c = nullptr;
    if (fgt_ctx_create(0, &c) == FGT_OK) g_default = c;
  });
  return g_default;
}

int fgt_plan_create(fgt_ctx* ctx, int dim, int nd, double delta, double eps, int ns,
                    const double* sources, int nt, const double* targ, int ifpgh, int ifpghtarg,
                    fgt_plan** out) {
  return plan_create_impl(ctx, dim, nd, delta, eps, ns, sources, nt, targ, 1, 0, ifpgh, ifpghtarg, out);
}

int fgt_plan_create_cd(fgt_ctx* ctx, int dim, int nd, double delta, double eps, int ns,
                       const double* sources, int nt, const double* targ, int ifcharge, int ifdipole,
                       int ifpgh, int ifpghtarg, fgt_plan** out) {
  return plan_create_impl(ctx, dim, nd, delta, eps, ns, sources, nt, targ, ifcharge, ifdipole, ifpgh,
                          ifpghtarg, out);
}

}  // extern "C"

namespace {
int plan_create_impl(fgt_ctx* ctx, int dim, int nd, double delta, double eps, int ns,
                     const double* sources, int nt, const double* targ, int ifcharge, int ifdipole,
                     int ifpgh, int ifpghtarg, fgt_plan** out, const double* pre_q,
                     const double* pre_rn, const double* pre_ds) {
  if (!ctx || !out) return FGT_ERR_BADARG;
  *out = nullptr;
  int st = check_args(dim, nd, delta, eps, ns, sources, ifcharge, ifdipole, ifpgh, nt, targ, ifpghtarg,
                      ctx->tree != FGT_TREE_DEVICE);
  if (st != FGT_OK) return st;
  if (ns == 0) return FGT_ERR_BADARG;
  if (!targ) nt = 0;  // no target array: no targets in the tree either
  // the NUFFT scheme's 2D form takes charges only
  if (ctx->scheme == FGT_SCHEME_NUFFT && dim == 2 && ifdipole) return FGT_ERR_UNSUPPORTED;
  std::unique_ptr<fgt_plan> p(new (std::nothrow) fgt_plan());
  if (!p) return FGT_ERR_NOMEM;
  p->ctx = ctx;
  p->H.scheme = ctx->scheme;
  p->pre_q = pre_q;
  p->pre_rn = pre_rn;
  p->pre_ds = pre_ds;
  CKS(cudaSetDevice(ctx->device));
  if (ctx->tree == FGT_TREE_DEVICE) {
    st = plan_create_device_tree(p.get(), dim, nd, delta, eps, ns, sources, nt, targ, ifpgh, ifpghtarg,
                                 nullptr, ifcharge, ifdipole);
  } else {
    try {
      build_host_plan(p->H, dim, nd, delta, eps, ns, sources, nt, targ, ifpgh, ifpghtarg, ctx->nthreads,
                      ifcharge, ifdipole);
    } catch (const std::bad_alloc&) {
      return FGT_ERR_NOMEM;
    }
    st = plan_device(p.get(), sources, targ);
  }
  if (st != FGT_OK) {
    fgt_plan_destroy(p.release());
    return st;
  }
  *out = p.release();
  return FGT_OK;
}
}  // namespace

extern "C" {

int fgt_plan_destroy(fgt_plan* p) {
  if (!p) return FGT_ERR_BADARG;
  if (p->ctx) cudaSetDevice(p->ctx->device);
  if (p->done) {
    // the stream-ordered frees below follow the last execute, on any stream
    cudaStreamWaitEvent(p->ctx->stream, p->done, 0);
    cudaEventDestroy(p->done);
  }
  if (p->pre_done) {  // and the strengths' uploads
    cudaStreamWaitEvent(p->ctx->stream, p->pre_done, 0);
    cudaEventDestroy(p->pre_done);
  }
  if (p->have_device) {
    p->D.stream = p->ctx->stream;
    device_plan_destroy(p->D);
  }
  if (p->d_io) cudaFreeAsync(p->d_io, p->ctx->stream);
  if (p->d_xslots) cudaFreeAsync(p->d_xslots, p->ctx->stream);
  delete p;
  return FGT_OK;
}

int fgt_plan_execute_host(fgt_plan* p, const double* sources, const double* charge,
                          const double* targ, double* pot, double* pottarg) {
  if (!p) return FGT_ERR_BADARG;
  (void)sources; (void)targ;  // fixed at plan creation
  Outputs h;
  h.pot = pot;
  h.pottarg = pottarg;
  return exec_host(p, charge, h);
}

int fgt_plan_execute_host_pgh(fgt_plan* p, const double* charge, double* pot, double* grad,
                              double* hess, double* pottarg, double* gradtarg, double* hesstarg) {
  if (!p) return FGT_ERR_BADARG;
  Outputs h;
  h.pot = pot; h.grad = grad; h.hess = hess;
  h.pottarg = pottarg; h.gradtarg = gradtarg; h.hesstarg = hesstarg;
  return exec_host(p, charge, h);
}

int fgt_plan_execute_device(fgt_plan* p, const double* s, const double* q, const double* t,
                            double* pot, double* pt, void* stream) {
  if (!p) return FGT_ERR_BADARG;
  CKS(cudaSetDevice(p->ctx->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : p->ctx->stream;
  (void)s; (void)t;  // the points are fixed at plan creation
  Outputs o;
  o.pot = pot;
  o.pottarg = pt;
  Inputs in;
  in.charge = q;
  return run_device(p, in, o, st, nullptr);
}

int fgt_plan_create_shard(fgt_ctx* ctx, int dim, int nd, double delta, double eps, int ns,
                          const double* sources, int nt, const double* targ, int ifpgh, int ifpghtarg,
                          int nranks, int rank, fgt_plan** out) {
  if (!ctx || !out || nranks < 1 || rank < 0 || rank >= nranks) return FGT_ERR_BADARG;
  *out = nullptr;
  int st = check_args(dim, nd, delta, eps, ns, sources, 1, 0, ifpgh, nt, targ, ifpghtarg,
                      ctx->tree != FGT_TREE_DEVICE);
  if (st != FGT_OK) return st;
  if (ns == 0) return FGT_ERR_BADARG;
  if (!targ) nt = 0;
  std::unique_ptr<fgt_plan> p(new (std::nothrow) fgt_plan());
  if (!p) return FGT_ERR_NOMEM;
  p->ctx = ctx;
  p->H.scheme = ctx->scheme;
  p->shard_n = nranks;
  p->shard_r = rank;
  CKS(cudaSetDevice(ctx->device));
  if (ctx->tree == FGT_TREE_DEVICE) {
    st = plan_create_device_tree(p.get(), dim, nd, delta, eps, ns, sources, nt, targ, ifpgh, ifpghtarg);
  } else {
    try {
      build_host_plan(p->H, dim, nd, delta, eps, ns, sources, nt, targ, ifpgh, ifpghtarg, ctx->nthreads);
    } catch (const std::bad_alloc&) {
      return FGT_ERR_NOMEM;
    }
    st = plan_device(p.get(), sources, targ);
  }
  if (st == FGT_OK && nranks > 1) {
    // the exchange lists on the device: every peer's send list, then every peer's receive list
    std::vector<int> all;
    p->xsend_off.assign(nranks + 1, 0);
    p->xrecv_off.assign(nranks + 1, 0);
    for (int r = 0; r < nranks; r++) {
      all.insert(all.end(), p->shard.send[r].begin(), p->shard.send[r].end());
      p->xsend_off[r + 1] = (long long)all.size();
    }
    for (int r = 0; r < nranks; r++) {
      p->xrecv_off[r] = (long long)all.size();
      all.insert(all.end(), p->shard.recv[r].begin(), p->shard.recv[r].end());
    }
    p->xrecv_off[nranks] = (long long)all.size();
    if (!all.empty()) {
      cudaStream_t s = ctx->stream;
      if (cudaMallocAsync(reinterpret_cast<void**>(&p->d_xslots), all.size() * sizeof(int), s) != cudaSuccess ||
          cudaMemcpyAsync(p->d_xslots, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice, s) !=
              cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        st = FGT_ERR_CUDA;
    }
  }
  if (st != FGT_OK) {
    fgt_plan_destroy(p.release());
    return st;
  }
  *out = p.release();
  return FGT_OK;
}

int fgt_plan_shard_counts(fgt_plan* p, int peer, long long* nsend, long long* nrecv, long long* slot_doubles) {
  if (!p || peer < 0 || peer >= p->shard_n) return FGT_ERR_BADARG;
  if (nsend) *nsend = (long long)p->shard.send[peer].size();
  if (nrecv) *nrecv = (long long)p->shard.recv[peer].size();
  if (slot_doubles) *slot_doubles = 2LL * p->H.P.nd * p->H.P.nexp;
  return FGT_OK;
}

int fgt_plan_shard_owned(fgt_plan* p, long long* owned_sources, long long* owned_targets) {
  if (!p) return FGT_ERR_BADARG;
  const bool all = p->shard_n <= 1;
  if (owned_sources) *owned_sources = all ? p->H.P.ns : p->shard.owned_src;
  if (owned_targets) *owned_targets = all ? p->H.P.nt : p->shard.owned_trg;
  return FGT_OK;
}

int fgt_plan_execute_device_phase(fgt_plan* p, int phase, const double* q, double* pot, double* pt,
                                  void* stream) {
  if (!p || phase < 0 || phase > 2) return FGT_ERR_BADARG;
  CKS(cudaSetDevice(p->ctx->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : p->ctx->stream;
  Outputs o;
  o.pot = pot;
  o.pottarg = pt;
  Inputs in;
  in.charge = q;
  if (p->H.P.large_delta && phase == 1) return FGT_OK;  // one phase: all of it runs in phase 2
  return run_device(p, in, o, st, nullptr, p->H.P.large_delta ? 0 : phase);
}

int fgt_plan_mp_pack(fgt_plan* p, int peer, double* d_buf, void* stream) {
  if (!p || peer < 0 || peer >= p->shard_n) return FGT_ERR_BADARG;
  if (p->shard_n <= 1 || !p->have_device) return FGT_OK;
  const long long n = p->xsend_off[peer + 1] - p->xsend_off[peer];
  if (n > 0 && !d_buf) return FGT_ERR_BADARG;
  CKS(cudaSetDevice(p->ctx->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : p->ctx->stream;
  CKS(shard_mp_copy(p->D, p->d_xslots + p->xsend_off[peer], (int)n, d_buf, true, st));
  return FGT_OK;
}

int fgt_plan_mp_unpack(fgt_plan* p, int peer, const double* d_buf, void* stream) {
  if (!p || peer < 0 || peer >= p->shard_n) return FGT_ERR_BADARG;
  if (p->shard_n <= 1 || !p->have_device) return FGT_OK;
  const long long n = p->xrecv_off[peer + 1] - p->xrecv_off[peer];
  if (n > 0 && !d_buf) return FGT_ERR_BADARG;
  CKS(cudaSetDevice(p->ctx->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : p->ctx->stream;
  CKS(shard_mp_copy(p->D, p->d_xslots + p->xrecv_off[peer], (int)n, const_cast<double*>(d_buf), false, st));
  return FGT_OK;
}

// Host-only view of a shard (no GPU): the host tree and plan, filtered.
struct fgt_host_shard {
  HostPlan H;
  ShardInfo S;
  long long nform = 0, neval = 0, ndir = 0, nm2l = 0, nmerge = 0, nsplit = 0;
  int nmp = 0;
};

int fgt_host_shard_create(int dim, int nd, double delta, double eps, int ns, const double* sources, int nt,
                          const double* targ, int ifpgh, int ifpghtarg, int nranks, int rank,
                          fgt_host_shard** out) {
  if (!out || nranks < 1 || rank < 0 || rank >= nranks) return FGT_ERR_BADARG;
  *out = nullptr;
  int st = check_args(dim, nd, delta, eps, ns, sources, 1, 0, ifpgh, nt, targ, ifpghtarg, true);
  if (st != FGT_OK) return st;
  if (!targ) nt = 0;
  std::unique_ptr<fgt_host_shard> h(new (std::nothrow) fgt_host_shard());
  if (!h) return FGT_ERR_NOMEM;
  try {
    build_host_plan(h->H, dim, nd, delta, eps, ns, sources, nt, targ, ifpgh, ifpghtarg, 0);
  } catch (const std::bad_alloc&) {
    return FGT_ERR_NOMEM;
  }
  if (shard_filter(h->H, nranks, rank, h->S) != 0) return FGT_ERR_BADARG;
  h->nform = (long long)h->H.form.size();
  h->neval = (long long)h->H.eval.size();
  h->ndir = (long long)h->H.dir.size();
  h->nm2l = (long long)h->H.m2l.size();
  h->nmerge = (long long)h->H.merge.size();
  h->nsplit = (long long)h->H.split.size();
  h->nmp = h->H.nmp;
  *out = h.release();
  return FGT_OK;
}
int fgt_host_shard_counts(fgt_host_shard* h, int peer, long long* nsend, long long* nrecv) {
  if (!h || peer < 0 || peer >= h->S.nranks) return FGT_ERR_BADARG;
  if (nsend) *nsend = (long long)h->S.send[peer].size();
  if (nrecv) *nrecv = (long long)h->S.recv[peer].size();
  return FGT_OK;
}
int fgt_host_shard_slots(fgt_host_shard* h, int peer, int which, int* out) {
  if (!h || !out || peer < 0 || peer >= h->S.nranks || which < 0 || which > 1) return FGT_ERR_BADARG;
  const std::vector<int>& v = which == 0 ? h->S.send[peer] : h->S.recv[peer];
  std::copy(v.begin(), v.end(), out);
  return FGT_OK;
}
int fgt_host_shard_stats(fgt_host_shard* h, long long* out8) {
  if (!h || !out8) return FGT_ERR_BADARG;
  const bool all = h->S.nranks <= 1;
  out8[0] = all ? h->H.P.ns : h->S.owned_src;
  out8[1] = all ? h->H.P.nt : h->S.owned_trg;
  out8[2] = h->nform;
  out8[3] = h->neval;
  out8[4] = h->ndir;
  out8[5] = h->nm2l;
  out8[6] = h->nmerge + h->nsplit;
  out8[7] = h->nmp;
  return FGT_OK;
}
int fgt_host_shard_destroy(fgt_host_shard* h) {
  delete h;
  return FGT_OK;
}

int fgt_plan_execute_device_pgh(fgt_plan* p, const double* q, double* pot, double* grad, double* hess,
                                double* pottarg, double* gradtarg, double* hesstarg, void* stream) {
  if (!p) return FGT_ERR_BADARG;
  CKS(cudaSetDevice(p->ctx->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : p->ctx->stream;
  Outputs o;
  o.pot = pot; o.grad = grad; o.hess = hess;
  o.pottarg = pottarg; o.gradtarg = gradtarg; o.hesstarg = hesstarg;
  Inputs in;
  in.charge = q;
  return run_device(p, in, o, st, nullptr);
}

int fgt_plan_execute_host_full(fgt_plan* p, const double* charge, const double* rnormal,
                               const double* dipstr, double* pot, double* grad, double* hess,
                               double* pottarg, double* gradtarg, double* hesstarg) {
  if (!p) return FGT_ERR_BADARG;
  Outputs h;
  h.pot = pot; h.grad = grad; h.hess = hess;
  h.pottarg = pottarg; h.gradtarg = gradtarg; h.hesstarg = hesstarg;
  return exec_host(p, charge, h, rnormal, dipstr);
}

int fgt_plan_execute_device_full(fgt_plan* p, const double* q, const double* rnormal,
                                 const double* dipstr, double* pot, double* grad, double* hess,
                                 double* pottarg, double* gradtarg, double* hesstarg, void* stream) {
  if (!p) return FGT_ERR_BADARG;
  CKS(cudaSetDevice(p->ctx->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : p->ctx->stream;
  Outputs o;
  o.pot = pot; o.grad = grad; o.hess = hess;
  o.pottarg = pottarg; o.gradtarg = gradtarg; o.hesstarg = hesstarg;
  Inputs in;
  in.charge = q;
  in.rnormal = rnormal;
  in.dipstr = dipstr;
  return run_device(p, in, o, st, nullptr);
}

int fgt_plan_profile_dominant(fgt_plan* p, const double* q, double* pot, double* pt, double* ms,
                              double* flops, double* alg_flops, char* name, int name_len) {
  if (!p || !ms || !flops) return FGT_ERR_BADARG;
  CKS(cudaSetDevice(p->ctx->device));
  StageTimes T;
  memset(T.ms, 0, sizeof(T.ms));
  if (p->H.P.large_delta) return FGT_ERR_UNSUPPORTED;
  Outputs o;
  o.pot = pot;
  o.pottarg = pt;
  Inputs in;
  in.charge = q;
  int r = run_device(p, in, o, p->ctx->stream, &T);
  if (r != FGT_OK) return r;
  CKS(cudaStreamSynchronize(p->ctx->stream));
  *ms = T.dom_ms;
  *flops = T.dom_flops;
  if (alg_flops) *alg_flops = T.dom_alg_flops;
  if (name && name_len > 0) snprintf(name, name_len, "%s", T.dom_name);
  return T.dom_name[0] ? FGT_OK : FGT_ERR_UNSUPPORTED;
}

int fgt_plan_profile_device(fgt_plan* p, const double* s, const double* q, const double* t,
                            double* pot, double* pt, float* ms8) {
  if (!p || !ms8) return FGT_ERR_BADARG;
  CKS(cudaSetDevice(p->ctx->device));
  StageTimes T;
  memset(T.ms, 0, sizeof(T.ms));
  (void)s; (void)t;
  Outputs o;
  o.pot = pot;
  o.pottarg = pt;
  Inputs in;
  in.charge = q;
  int r = run_device(p, in, o, p->ctx->stream, p->H.P.large_delta ? nullptr : &T);
  if (r != FGT_OK) return r;
  CKS(cudaStreamSynchronize(p->ctx->stream));
  for (int i = 0; i < 8; i++) ms8[i] = T.ms[i];
  return FGT_OK;
}

int fgt_plan_expansion(fgt_plan* p, int which, int box, double* out) {
  if (!p || !out || (which != 0 && which != 1)) return FGT_ERR_BADARG;
  if (!p->have_device) return FGT_ERR_UNSUPPORTED;  // large-delta and all-direct plans hold none
  const HostPlan& H = p->H;
  if (box < 0 || box >= H.tree.nboxes) return FGT_ERR_BADARG;
  const std::vector<int>& slots = which == 0 ? H.mp_slot : H.loc_slot;
  if ((int)slots.size() <= box || slots[box] < 0) return FGT_ERR_BADARG;
  const double2* pool = which == 0 ? p->D.mp : p->D.loc;
  const size_t per = (size_t)H.P.nd * H.P.nexp;
  CKS(cudaSetDevice(p->ctx->device));
  if (p->done) CKS(cudaEventSynchronize(p->done));
  CKS(cudaMemcpyAsync(out, pool + (size_t)slots[box] * per, per * 16, cudaMemcpyDeviceToHost, p->ctx->stream));
  CKS(cudaStreamSynchronize(p->ctx->stream));
  return FGT_OK;
}

int fgt_plan_get_info(const fgt_plan* p, fgt_plan_info* o) {
  if (!p || !o) return FGT_ERR_BADARG;
  memset(o, 0, sizeof(*o));
  const Params& P = p->H.P;
  o->dim = P.dim; o->nd = P.nd; o->ns = P.ns; o->nt = P.nt;
  o->npwlevel = P.npwlevel; o->nlevels = P.nlevels; o->nboxes = p->H.tree.nboxes;
  o->npw = P.npw; o->nexp = P.nexp; o->nlmax = P.nlmax;
  o->nform = (int)p->H.form.size(); o->neval = (int)p->H.eval.size();
  o->ndirect_tasks = p->have_device ? p->D.ndir : (int)p->H.dir.size(); o->nmp = p->H.nmp; o->nloc = p->H.nloc;
  o->direct_pairs = p->H.direct_pairs; o->form_sources = p->H.form_sources;
  o->eval_points = p->H.eval_points;
  o->device_bytes = (long long)(p->D.bytes + p->io_bytes);
  o->host_tree_s = p->H.host_tree_s; o->host_lists_s = p->H.host_lists_s;
  o->host_plan_s = p->H.host_plan_s;
  o->large_delta = P.large_delta; o->all_direct = P.all_direct;
  o->kernel_launches = p->last_launches;
  for (int i = 0; i < 3; i++) o->shift_bytes[i] = p->H.shift_bytes[i];
  if (p->have_device) o->shift_bytes[2] = p->D.split_bytes;  // the splits that run
  o->form_route_flops = p->H.form_route_flops;
  o->eval_route_flops = p->H.eval_route_flops;
  double npwd = std::pow((double)P.npw, P.dim);
  o->form_flops = 4.0 * (double)p->H.form_sources * npwd;
  o->eval_flops = 4.0 * (double)p->H.eval_points * npwd;
  return FGT_OK;
}

struct fgt_host_tree {
  Tree t;
  int nlmax = 0;
  bool large = false;
};

int fgt_host_tree_create(int dim, double delta, double eps, int ns, const double* sources, int nt,
                         const double* targ, int nthreads, fgt_host_tree** out) {
  if (!out) return FGT_ERR_BADARG;
  *out = nullptr;
  int st = check_args(dim, 1, delta, eps, ns, sources, 1, 0, 0, nt, targ, 0);
  if (st != FGT_OK) return st;
  if (ns == 0) return FGT_ERR_BADARG;
  fgt_host_tree* h = new (std::nothrow) fgt_host_tree();
  if (!h) return FGT_ERR_NOMEM;
  try {
    HostPlan H;
    int lc;
    double bs0, cen0[3] = {0, 0, 0};
    boxsize0(dim, delta, eps, sources, ns, targ, nt, &lc, &bs0, cen0);
    if (lc < -2) {
      h->large = true;
      h->t.npwlevel = lc;
    } else {
      int ndiv0 = dim == 2 ? 10 : 40, ndiv = dim == 2 ? 80 : 100, hcap = dim == 2 ? 18 : 15;
      int nlmax = lc + 4, nls = lc > 0 ? lc : 0, nl0 = 0;
      double bsize = bs0 / std::ldexp(1.0, nls);
      for (int i = nls; i <= 100; i++) {
        nl0 = hlterms(dim, bsize, delta, eps, nl0);
        if (nl0 <= hcap) { nlmax = i; break; }
        bsize /= 2;
      }
      build_tree(h->t, dim, sources, ns, targ, nt, ndiv, ndiv0, lc, nlmax, bs0, cen0, nthreads);
      h->t.npwlevel = lc;
      h->nlmax = nlmax;
    }
  } catch (const std::bad_alloc&) {
    delete h;
    return FGT_ERR_NOMEM;
  }
  *out = h;
  return FGT_OK;
}
int fgt_device_tree_create(fgt_ctx* ctx, int dim, double delta, double eps, int ns, const double* sources,
                           int nt, const double* targ, fgt_host_tree** out) {
  if (!ctx || !out) return FGT_ERR_BADARG;
  *out = nullptr;
  int st = check_args(dim, 1, delta, eps, ns, sources, 1, 0, 0, nt, targ, 0);
  if (st != FGT_OK) return st;
  if (ns == 0) return FGT_ERR_BADARG;
  if (!targ) nt = 0;
  CKS(cudaSetDevice(ctx->device));
  std::unique_ptr<fgt_host_tree> h(new (std::nothrow) fgt_host_tree());
  if (!h) return FGT_ERR_NOMEM;
  cudaStream_t s = ctx->stream;
  const bool same = targ == sources && nt == ns;
  double *d_src = nullptr, *d_trg = nullptr;
  int* perms = nullptr;
  size_t nsd = (size_t)ns * dim, ntd = same ? 0 : (size_t)nt * dim;
  CKS(cudaMalloc(&d_src, 8 * (nsd + ntd + 2)));
  struct Free {
    void* a;
    void* b;
    ~Free() { cudaFree(a); cudaFree(b); }
  } fr{d_src, nullptr};
  CKS(cudaMalloc(&perms, sizeof(int) * ((size_t)ns + nt + 2)));
  fr.b = perms;
  d_trg = same ? d_src : d_src + nsd + 1;
  CKS(cudaMemcpyAsync(d_src, sources, nsd * 8, cudaMemcpyHostToDevice, s));
  if (!same && nt > 0) CKS(cudaMemcpyAsync(d_trg, targ, ntd * 8, cudaMemcpyHostToDevice, s));
  try {
    HostPlan H;
    double mn[3], mx[3];
    CKS(cudaStreamSynchronize(s));
    int lc;
    double bs0, cen0[3] = {0, 0, 0};
    // bounding box from the same reduction the plan uses
    CKS(build_plan_device_bbox(d_src, ns, d_trg, same ? 0 : nt, dim, mn, mx, s));
    boxsize0_bbox(dim, delta, eps, mn, mx, &lc, &bs0, cen0);
    TreeSetup ts;
    if (!plan_begin(H, dim, 1, delta, eps, ns, nt, 0, 0, lc, bs0, cen0, ts)) {
      h->large = true;
      h->t.npwlevel = lc;
    } else {
      CKS(build_tree_device(h->t, dim, d_src, ns, d_trg, nt, same, ts, perms, perms + ns + 1, s));
      h->t.npwlevel = lc;
      h->nlmax = ts.nlmax;
      h->t.isrc.resize(ns);
      h->t.itarg.resize(nt);
      CKS(cudaMemcpyAsync(h->t.isrc.data(), perms, sizeof(int) * ns, cudaMemcpyDeviceToHost, s));
      if (nt > 0)
        CKS(cudaMemcpyAsync(h->t.itarg.data(), perms + ns + 1, sizeof(int) * nt, cudaMemcpyDeviceToHost, s));
      CKS(cudaStreamSynchronize(s));
    }
  } catch (const std::bad_alloc&) {
    return FGT_ERR_NOMEM;
  }
  *out = h.release();
  return FGT_OK;
}
int fgt_host_tree_dims(const fgt_host_tree* h, int* dims) {
  if (!h || !dims) return FGT_ERR_BADARG;
  dims[0] = h->t.nlevels; dims[1] = h->t.nboxes; dims[2] = h->t.npwlevel; dims[3] = h->nlmax;
  return h->large ? FGT_ERR_UNSUPPORTED : FGT_OK;
}
long long fgt_host_tree_field(const fgt_host_tree* h, int field, void* out) {
  if (!h || h->large) return -1;
  const Tree& t = h->t;
  std::vector<int> v;
  int nb = t.nboxes;
  auto id = [](int b) { return b >= 0 ? b + 1 : -1; };
  switch (field) {
    case 0: for (int l = 0; l <= t.nlevels; l++) { v.push_back(t.lfirst[l] + 1); v.push_back(t.llast[l] + 1); } break;
    case 1: v.assign(t.level.begin(), t.level.begin() + nb); break;
    case 2: for (int b = 0; b < nb; b++) v.push_back(id(t.parent[b])); break;
    case 3: v.assign(t.nchild.begin(), t.nchild.begin() + nb); break;
    case 4: for (size_t i = 0; i < (size_t)nb * t.nch; i++) v.push_back(id(t.child[i])); break;
    case 5: v.assign(t.ncoll.begin(), t.ncoll.begin() + nb); break;
    case 6: for (size_t i = 0; i < (size_t)nb * t.nco; i++) v.push_back(id(t.coll[i])); break;
    case 7: for (int x : t.isrc) v.push_back(x + 1); break;
    case 8: for (int b = 0; b < nb; b++) { v.push_back(t.s0[b] + 1); v.push_back(t.s1[b]); } break;
    case 9: for (int x : t.itarg) v.push_back(x + 1); break;
    case 10: for (int b = 0; b < nb; b++) { v.push_back(t.t0[b] + 1); v.push_back(t.t1[b]); } break;
    case 11:
      if (out) memcpy(out, t.centers.data(), sizeof(double) * (size_t)nb * t.dim);
      return (long long)nb * t.dim;
    case 12:
      if (out) memcpy(out, t.boxsize.data(), sizeof(double) * (t.nlevels + 1));
      return t.nlevels + 1;
    default: return -1;
  }
  if (out) memcpy(out, v.data(), sizeof(int) * v.size());
  return (long long)v.size();
}
int fgt_host_tree_destroy(fgt_host_tree* h) {
  delete h;
  return FGT_OK;
}

int fgt_transform(fgt_ctx* ctx, int dim, int nd, double delta, double eps, int ns,
                  const double* sources, int ifcharge, const double* charge, int ifdipole,
                  const double* rnormal, const double* dipstr, int ifpgh, double* pot, double* grad,
                  double* hess, int nt, const double* targ, int ifpghtarg, double* pottarg,
                  double* gradtarg, double* hesstarg) {
  (void)rnormal; (void)dipstr;
  if (!ctx) return FGT_ERR_BADARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return transform_impl(ctx, dim, nd, delta, eps, ns, sources, ifcharge, charge, ifdipole, rnormal,
                        dipstr, ifpgh,
                        pot, grad, hess, nt, targ, ifpghtarg, pottarg, gradtarg, hesstarg);
}

static int fortran_call(int dim, const int* nd, const double* delta, const double* eps, const int* ns,
                        const double* sources, const int* ifcharge, const double* charge,
                        const int* ifdipole, const double* rnormal, const double* dipstr,
                        const int* ifpgh, double* pot, double* grad, double* hess, const int* nt,
                        const double* targ, const int* ifpghtarg, double* pottarg, double* gradtarg,
                        double* hesstarg) {
  if (!nd || !delta || !eps || !ns || !ifcharge || !ifdipole || !ifpgh || !nt || !ifpghtarg)
    return FGT_ERR_BADARG;
  fgt_ctx* c = fgt_default_ctx();
  if (!c) return FGT_ERR_NODEVICE;
  return fgt_transform(c, dim, *nd, *delta, *eps, *ns, sources, *ifcharge, charge, *ifdipole,
                       rnormal, dipstr, *ifpgh, pot, grad, hess, *nt, targ, *ifpghtarg, pottarg,
                       gradtarg, hesstarg);
}

void fgt2d_(const int* nd, const double* delta, const double* eps, const int* ns,
            const double* sources, const int* ifcharge, const double* charge, const int* ifdipole,
            const double* rnormal, const double* dipstr, const int* iper, const int* ifpgh,
            double* pot, double* grad, double* hess, const int* nt, const double* targ,
            const int* ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg) {
  (void)iper;
  report("fgt2d", fortran_call(2, nd, delta, eps, ns, sources, ifcharge, charge, ifdipole, rnormal,
                               dipstr, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg,
                               gradtarg, hesstarg));
}
void fgt3d_(const int* nd, const double* delta, const double* eps, const int* ns,
            const double* sources, const int* ifcharge, const double* charge, const int* ifdipole,
            const double* rnormal, const double* dipstr, const int* iper, const int* ifpgh,
            double* pot, double* grad, double* hess, const int* nt, const double* targ,
            const int* ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg) {
  (void)iper;
  report("fgt3d", fortran_call(3, nd, delta, eps, ns, sources, ifcharge, charge, ifdipole, rnormal,
                               dipstr, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg,
                               gradtarg, hesstarg));
}
void fgt2d_st_(const int* nd, const double* delta, const double* eps, const int* ns,
               const double* sources, const int* ifcharge, const double* charge,
               const int* ifdipole, const double* rnormal, const double* dipstr, const int* iper,
               const int* ifpgh, double* pot, double* grad, double* hess, const int* nt,
               const double* targ, const int* ifpghtarg, double* pottarg, double* gradtarg,
               double* hesstarg, int* ier) {
  (void)iper;
  int s = fortran_call(2, nd, delta, eps, ns, sources, ifcharge, charge, ifdipole, rnormal, dipstr,
                       ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg, gradtarg, hesstarg);
  if (ier) *ier = s;
}
void fgt3d_st_(const int* nd, const double* delta, const double* eps, const int* ns,
               const double* sources, const int* ifcharge, const double* charge,
               const int* ifdipole, const double* rnormal, const double* dipstr, const int* iper,
               const int* ifpgh, double* pot, double* grad, double* hess, const int* nt,
               const double* targ, const int* ifpghtarg, double* pottarg, double* gradtarg,
               double* hesstarg, int* ier) {
  (void)iper;
  int s = fortran_call(3, nd, delta, eps, ns, sources, ifcharge, charge, ifdipole, rnormal, dipstr,
                       ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg, gradtarg, hesstarg);
  if (ier) *ier = s;
}

}  // extern "C"

// ---- the fgt2dmain / fgt3dmain cut -----------------------------------------
template <typename IP>
static int main_gpu(int dim, const int* nd, const double* delta, const double* eps,
                    const int* nsource, const double* sourcesort, const int* ifcharge,
                    const double* chargesort, const int* ifdipole, const double* rnormalsort,
                    const double* dipstrsort, const int* ntarget,
                    const double* targetsort, const int* itree, const IP* iptr, const int* nlevels,
                    const int* npwlevel, const int* nboxes, const double* boxsize,
                    const double* centers, const int* laddr, const int* isrcse, const int* itargse,
                    const int* nlocal, const double* pmax, const int* npw, const int* ifpgh,
                    double* pot, double* grad, double* hess, const int* ifpghtarg, double* pottarg,
                    double* gradtarg, double* hesstarg) {
  if (!nd || !delta || !eps || !nsource || !ntarget || !itree || !iptr || !nlevels || !npwlevel ||
      !nboxes || !boxsize || !centers || !laddr || !isrcse || !itargse || !nlocal || !pmax || !npw ||
      !ifpgh || !ifpghtarg || !ifcharge || !ifdipole)
    return FGT_ERR_BADARG;
  int st = check_args(dim, *nd, *delta, *eps, *nsource, sourcesort, *ifcharge, *ifdipole, *ifpgh,
                      *ntarget, targetsort, *ifpghtarg);
  if (st != FGT_OK) return st;
  fgt_ctx* c = fgt_default_ctx();
  if (!c) return FGT_ERR_NODEVICE;
  std::lock_guard<std::mutex> lk(c->mu);
  std::unique_ptr<fgt_plan> p(new (std::nothrow) fgt_plan());
  if (!p) return FGT_ERR_NOMEM;
  p->ctx = c;
  int nb = *nboxes, nlev = *nlevels, ns = *nsource, nt = *ntarget, D = dim;
  int nch = 1 << dim, nco = dim == 2 ? 9 : 27;
  Tree& t = p->H.tree;
  t.dim = dim; t.nch = nch; t.nco = nco; t.nlevels = nlev; t.nboxes = nb; t.npwlevel = *npwlevel;
  t.lfirst.resize(nlev + 1);
  t.llast.resize(nlev + 1);
  for (int l = 0; l <= nlev; l++) {
    t.lfirst[l] = laddr[2 * l] - 1;
    t.llast[l] = laddr[2 * l + 1] - 1;
  }
  auto at = [&](int k, long long off) { return itree[(long long)iptr[k] - 1 + off]; };
  t.level.resize(nb); t.parent.resize(nb); t.nchild.resize(nb);
  t.child.assign((size_t)nb * nch, -1); t.ncoll.resize(nb); t.coll.assign((size_t)nb * nco, -1);
  for (int b = 0; b < nb; b++) {
    t.level[b] = at(1, b);
    int par = at(2, b);
    t.parent[b] = par > 0 ? par - 1 : -1;
    t.nchild[b] = at(3, b);
    for (int j = 0; j < nch; j++) {
      int cb = at(4, (long long)nch * b + j);
      t.child[(size_t)b * nch + j] = cb > 0 ? cb - 1 : -1;
    }
    t.ncoll[b] = at(5, b);
    for (int i = 0; i < t.ncoll[b] && i < nco; i++) {
      int cb = at(6, (long long)nco * b + i);
      t.coll[(size_t)b * nco + i] = cb > 0 ? cb - 1 : -1;
    }
  }
  t.centers.assign(centers, centers + (size_t)nb * D);
  t.boxsize.assign(boxsize, boxsize + nlev + 1);
  t.s0.resize(nb); t.s1.resize(nb); t.t0.resize(nb); t.t1.resize(nb);
  for (int b = 0; b < nb; b++) {
    t.s0[b] = isrcse[2 * b] - 1; t.s1[b] = isrcse[2 * b + 1];
    t.t0[b] = itargse[2 * b] - 1; t.t1[b] = itargse[2 * b + 1];
  }
  t.isrc.resize(ns); t.itarg.resize(nt);
  for (int i = 0; i < ns; i++) t.isrc[i] = i;
  for (int i = 0; i < nt; i++) t.itarg[i] = i;
  Params P0;
  P0.dim = dim; P0.nd = *nd; P0.delta = *delta; P0.eps = *eps; P0.ns = ns; P0.nt = nt;
  P0.ifpgh = *ifpgh; P0.ifpghtarg = *ifpghtarg; P0.npwlevel = *npwlevel;
  P0.ifcharge = *ifcharge; P0.ifdipole = *ifdipole;
  std::vector<int> nl(nlocal, nlocal + nlev + 1);
  try {
    build_host_plan_from_tree(p->H, P0, nl, *pmax, *npw);
  } catch (const std::bad_alloc&) {
    return FGT_ERR_NOMEM;
  }
  CKS(cudaSetDevice(c->device));
  st = plan_device(p.get(), sourcesort, targetsort);
  if (st != FGT_OK) {
    fgt_plan_destroy(p.release());
    return st;
  }
  // outputs are incremented (fgt2dmain adds into pot/grad/hess)
  const size_t nh = dim == 2 ? 3 : 6, n1 = (size_t)ns * *nd, n2 = (size_t)nt * *nd;
  std::vector<double> po(n1), go(*ifpgh >= 2 ? n1 * dim : 0), ho(*ifpgh >= 3 ? n1 * nh : 0);
  std::vector<double> pt(n2), gt(*ifpghtarg >= 2 ? n2 * dim : 0), ht(*ifpghtarg >= 3 ? n2 * nh : 0);
  Outputs h;
  h.pot = po.data(); h.grad = go.data(); h.hess = ho.data();
  h.pottarg = pt.data(); h.gradtarg = gt.data(); h.hesstarg = ht.data();
  st = exec_host(p.get(), chargesort, h, rnormalsort, dipstrsort);
  fgt_plan_destroy(p.release());
  if (st != FGT_OK) return st;
  auto add = [](double* out, const std::vector<double>& v) {
    if (out)
      for (size_t i = 0; i < v.size(); i++) out[i] += v[i];
  };
  if (*ifpgh >= 1) add(pot, po);
  if (*ifpgh >= 2) add(grad, go);
  if (*ifpgh >= 3) add(hess, ho);
  if (*ifpghtarg >= 1) add(pottarg, pt);
  if (*ifpghtarg >= 2) add(gradtarg, gt);
  if (*ifpghtarg >= 3) add(hesstarg, ht);
  return FGT_OK;
}

extern "C" {

int fgt2dmain_gpu_(const int* nd, const double* delta, const double* eps, const int* nsource,
                   const double* sourcesort, const int* ifcharge, const double* chargesort,
                   const int* ifdipole, const double* rnormalsort, const double* dipstrsort,
                   const int* ntarget, const double* targetsort, const int* iaddr,
                   const double* rmlexp, const int* itree, const int* ltree, const int* iptr,
                   const int* nlevels, const int* npwlevel, const int* nboxes, const int* iper,
                   const double* boxsize, const double* centers, const int* laddr,
                   const int* isrcse, const int* itargse, const int* ntermsh, const int* nlocal,
                   const int* ntermmax, const double* pmax, const int* npw, const int* ifpgh,
                   double* pot, double* grad, double* hess, const int* ifpghtarg, double* pottarg,
                   double* gradtarg, double* hesstarg) {
  (void)iaddr; (void)rmlexp; (void)ltree; (void)iper;
  (void)ntermsh; (void)ntermmax;
  return main_gpu<int>(2, nd, delta, eps, nsource, sourcesort, ifcharge, chargesort, ifdipole,
                       rnormalsort, dipstrsort, ntarget, targetsort, itree, iptr, nlevels, npwlevel, nboxes, boxsize,
                       centers, laddr, isrcse, itargse, nlocal, pmax, npw, ifpgh, pot, grad, hess,
                       ifpghtarg, pottarg, gradtarg, hesstarg);
}

int fgt3dmain_gpu_(const int* nd, const double* delta, const double* eps, const int* nsource,
                   const double* sourcesort, const int* ifcharge, const double* chargesort,
                   const int* ifdipole, const double* rnormalsort, const double* dipstrsort,
                   const int* ntarget, const double* targetsort, const int* iaddr,
                   const double* rmlexp, const int* itree, const long long* ltree,
                   const long long* iptr, const int* nlevels, const int* npwlevel, const int* ndiv,
                   const int* nboxes, const int* iper, const double* boxsize,
                   const double* centers, const int* laddr, const int* isrcse,
                   const int* itargse, const int* ntermsh, const int* nlocal, const int* ntermmax,
                   const double* pmax, const int* npw, const int* ifpgh, double* pot, double* grad,
                   double* hess, const int* ifpghtarg, double* pottarg, double* gradtarg,
                   double* hesstarg) {
  (void)iaddr; (void)rmlexp; (void)ltree; (void)iper;
  (void)ndiv; (void)ntermsh; (void)ntermmax;
  return main_gpu<long long>(3, nd, delta, eps, nsource, sourcesort, ifcharge, chargesort, ifdipole,
                             rnormalsort, dipstrsort, ntarget, targetsort, itree, iptr, nlevels, npwlevel, nboxes, boxsize,
                             centers, laddr, isrcse, itargse, nlocal, pmax, npw, ifpgh, pot, grad,
                             hess, ifpghtarg, pottarg, gradtarg, hesstarg);
}

}  // extern "C"

// ---------------------------------------------------------------- serving
// A transform server on one device: requests of any dimension, size, delta and
// eps are queued as they arrive; worker threads, each with its own context
// and CUDA stream, take the smallest pending request (the oldest once it has
// waited longer than kServerAgeS), build its plan and run it, so requests
// that arrive while others are on the GPU overlap with them.  Device memory
// is admitted by footprint from two pools that cannot deadlock: the point
// arrays and tree scratch of a request (a fixed share of the budget), then
// the exact bytes of its plan, computed before they are allocated.  A plan
// pool holder never waits for anything else, so point-pool holders waiting
// for plan memory always see it freed.

struct fgt_server {
  int device = 0;
  long long budget = 0, budget_pts = 0, budget_plan = 0;
  std::vector<fgt_ctx*> ctxs;
  // per worker, a stream of the device's highest priority for small requests
  // (their blocks are dispatched ahead of large requests' when SMs free up)
  std::vector<cudaStream_t> hi;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_q, cv_mem, cv_done;
  struct Job {
    fgt_request r;
    long long id = 0;
    double t_sub = 0, t_start = 0, t_end = 0;
    int status = FGT_OK;
    bool done = false;
  };
  std::vector<Job*> queue;
  std::unordered_map<long long, Job*> jobs;
  long long next_id = 1;
  long long in_pts = 0, in_plan = 0, peak = 0;
  bool stop = false;
  long long submitted = 0, completed = 0, failed = 0, points = 0, hi_priority = 0;
  int running = 0;  // requests taken by a worker and not yet done
  std::vector<double> lat;
  double t_first = -1, t_last = 0;
};

namespace {
constexpr double kServerAgeS = 0.05;
constexpr long long kServerSmall = 100000;  // points of a request on the high-priority stream

long long request_points(const fgt_request& r) {
  return (r.ifpgh >= 1 ? r.ns : 0) + (r.ifpghtarg >= 1 && r.targ ? r.nt : 0);
}

// blocks until b bytes fit in the pool (or the pool is idle), then takes them
void server_take(fgt_server* S, long long* in_use, long long cap, long long b) {
  std::unique_lock<std::mutex> lk(S->mu);
  S->cv_mem.wait(lk, [&] { return *in_use + b <= cap || *in_use == 0; });
  *in_use += b;
  S->peak = std::max(S->peak, S->in_pts + S->in_plan);
}
void server_give(fgt_server* S, long long* in_use, long long b) {
  std::lock_guard<std::mutex> lk(S->mu);
  *in_use -= b;
  S->cv_mem.notify_all();
}

int server_run(fgt_server* S, fgt_ctx* ctx, const fgt_request& r) {
  const int nt = r.targ ? r.nt : 0;
  const int ifcharge = r.charge != nullptr, ifdipole = r.ifdipole;
  int st = check_args(r.dim, r.nd, r.delta, r.eps, r.ns, r.sources, ifcharge, ifdipole, r.ifpgh, nt,
                      r.targ, r.ifpghtarg, false);
  if (st != FGT_OK) return st;
  if (ifdipole && r.ns > 0 && (!r.rnormal || !r.dipstr)) return FGT_ERR_BADARG;
  const size_t nh = r.dim == 2 ? 3 : 6;
  if ((r.ifpgh >= 1 && r.ns > 0 && !r.pot) || (r.ifpgh >= 2 && r.ns > 0 && !r.grad) ||
      (r.ifpgh >= 3 && r.ns > 0 && !r.hess) || (r.ifpghtarg >= 1 && nt > 0 && !r.pottarg) ||
      (r.ifpghtarg >= 2 && nt > 0 && !r.gradtarg) || (r.ifpghtarg >= 3 && nt > 0 && !r.hesstarg))
    return FGT_ERR_BADARG;
  auto zero = [&] {
    auto z = [](double* a, size_t n) { if (a && n) memset(a, 0, sizeof(double) * n); };
    if (r.ifpgh >= 1) z(r.pot, (size_t)r.ns * r.nd);
    if (r.ifpgh >= 2) z(r.grad, (size_t)r.ns * r.nd * r.dim);
    if (r.ifpgh >= 3) z(r.hess, (size_t)r.ns * r.nd * nh);
    if (r.ifpghtarg >= 1) z(r.pottarg, (size_t)nt * r.nd);
    if (r.ifpghtarg >= 2) z(r.gradtarg, (size_t)nt * r.nd * r.dim);
    if (r.ifpghtarg >= 3) z(r.hesstarg, (size_t)nt * r.nd * nh);
  };
  if (r.ns == 0) {
    zero();
    return FGT_OK;
  }
  CKS(cudaSetDevice(ctx->device));
  // point arrays (caller order, sorted copies, potentials) and tree scratch
  const long long npts = (long long)r.ns + nt;
  const long long nc = 2 + out_comps(r.dim, std::max(1, std::max(r.ifpgh, r.ifpghtarg)));
  const long long est_pts = 8LL * ((long long)r.ns * (2 * r.dim + nc * r.nd) + (long long)nt * (2 * r.dim + nc * r.nd)) +
                            64LL * npts + (1 << 20);
  server_take(S, &S->in_pts, S->budget_pts, est_pts);
  long long plan_bytes = 0;
  std::unique_ptr<fgt_plan> p(new (std::nothrow) fgt_plan());
  if (!p) {
    server_give(S, &S->in_pts, est_pts);
    return FGT_ERR_NOMEM;
  }
  p->ctx = ctx;
  p->pre_q = ifcharge ? r.charge : nullptr;
  p->pre_rn = ifdipole ? r.rnormal : nullptr;
  p->pre_ds = ifdipole ? r.dipstr : nullptr;
  std::function<int(size_t)> admit = [&](size_t b) {
    plan_bytes = (long long)b;
    server_take(S, &S->in_plan, S->budget_plan, plan_bytes);
    return FGT_OK;
  };
  st = plan_create_device_tree(p.get(), r.dim, r.nd, r.delta, r.eps, r.ns, r.sources, nt, r.targ, r.ifpgh,
                               r.ifpghtarg, &admit, ifcharge, ifdipole);
  if (st == FGT_OK) {
    Outputs h;
    h.pot = r.pot; h.grad = r.grad; h.hess = r.hess;
    h.pottarg = r.pottarg; h.gradtarg = r.gradtarg; h.hesstarg = r.hesstarg;
    st = exec_host(p.get(), r.charge, h, r.rnormal, r.dipstr);
  }
  fgt_plan_destroy(p.release());
  cudaStreamSynchronize(ctx->stream);  // the stream-ordered frees have run
  if (plan_bytes) server_give(S, &S->in_plan, plan_bytes);
  server_give(S, &S->in_pts, est_pts);
  if (st != FGT_OK) zero();
  return st;
}

// points of a request (sources and targets it carries)
long long job_points(const fgt_server::Job* J) { return (long long)J->r.ns + (J->r.targ ? J->r.nt : 0); }

void server_worker(fgt_server* S, int w) {
  fgt_ctx* ctx = S->ctxs[w];
  // the first quarter of the workers (at least one when there are two or
  // more) take only small requests, so that those never wait on the host for
  // a worker that holds a large one
  const int nsmall = S->ctxs.size() >= 2 ? std::max<int>(1, (int)S->ctxs.size() / 4) : 0;
  const bool small_only = w < nsmall;
  auto takeable = [&](const fgt_server::Job* J) { return !small_only || job_points(J) <= kServerSmall; };
  // the workers share the host cores: each builds its host-side plan parts
  // with its share of them
  omp_set_num_threads(std::max(1, omp_get_num_procs() / (int)S->ctxs.size()));
  for (;;) {
    fgt_server::Job* J = nullptr;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      auto any = [&] {
        for (const fgt_server::Job* J : S->queue)
          if (takeable(J)) return true;
        return false;
      };
      S->cv_q.wait(lk, [&] { return S->stop || any(); });
      if (!any()) return;  // stop requested and nothing left for this worker
      const double t = now_s();
      size_t pick = 0;
      while (!takeable(S->queue[pick])) pick++;
      for (size_t k = pick + 1; k < S->queue.size(); k++) {
        const fgt_server::Job* a = S->queue[k];
        const fgt_server::Job* b = S->queue[pick];
        if (!takeable(a)) continue;
        const bool a_old = t - a->t_sub > kServerAgeS, b_old = t - b->t_sub > kServerAgeS;
        if (a_old != b_old ? a_old
                           : (a_old ? a->t_sub < b->t_sub
                                    : (long long)a->r.ns + a->r.nt < (long long)b->r.ns + b->r.nt))
          pick = k;
      }
      J = S->queue[pick];
      S->queue.erase(S->queue.begin() + pick);
      J->t_start = t;
      S->running++;
    }
    // small requests run on the worker's high-priority stream
    const cudaStream_t base = ctx->stream;
    const bool on_hi = job_points(J) <= kServerSmall && S->hi[w];
    if (on_hi) ctx->stream = S->hi[w];
    int st = server_run(S, ctx, J->r);
    for (int retry = 0; st == FGT_ERR_NOMEM && retry < 50; retry++) {
      // the device memory is held (or fragmented) by requests in flight:
      // retry when one of them has finished (or after 0.1 s, so that workers
      // that all wait cannot block one another); alone, the failure stands
      (void)cudaGetLastError();
      {
        std::unique_lock<std::mutex> lk(S->mu);
        if (S->running <= 1) break;
        const long long c0 = S->completed;
        S->cv_done.wait_for(lk, std::chrono::milliseconds(100), [&] { return S->completed != c0; });
      }
      st = server_run(S, ctx, J->r);
    }
    ctx->stream = base;
    if (st == FGT_ERR_CUDA)  // an internal failure: say which
      fprintf(stderr, "fgt server: request %lld (dim %d, %d + %d points, delta %g, eps %g) failed: CUDA error %d (%s)\n",
              J->id, J->r.dim, J->r.ns, J->r.targ ? J->r.nt : 0, J->r.delta, J->r.eps, g_last_cuda,
              cudaGetErrorName((cudaError_t)g_last_cuda));
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->running--;
      J->t_end = now_s();
      J->status = st;
      J->done = true;
      S->completed++;
      if (on_hi) S->hi_priority++;
      if (st != FGT_OK) S->failed++;
      else S->points += request_points(J->r);
      S->lat.push_back(J->t_end - J->t_sub);
      S->t_last = std::max(S->t_last, J->t_end);
      S->cv_done.notify_all();
    }
  }
}
}  // namespace

extern "C" {

int fgt_server_create(int device, long long max_device_bytes, int nworkers, fgt_server** out) {
  if (!out || nworkers < 1 || nworkers > 64) return FGT_ERR_BADARG;
  *out = nullptr;
  std::unique_ptr<fgt_server> S(new (std::nothrow) fgt_server());
  if (!S) return FGT_ERR_NOMEM;
  S->device = device;
  if (max_device_bytes <= 0) {
    size_t fr = 0, tot = 0;
    CKS(cudaSetDevice(device));
    CKS(cudaMemGetInfo(&fr, &tot));
    max_device_bytes = (long long)(0.8 * fr);
  }
  S->budget = max_device_bytes;
  S->budget_pts = max_device_bytes / 4;
  S->budget_plan = max_device_bytes - S->budget_pts;
  for (int w = 0; w < nworkers; w++) {
    fgt_ctx* c = nullptr;
    int st = fgt_ctx_create(device, &c);
    if (st != FGT_OK) {
      for (fgt_ctx* x : S->ctxs) fgt_ctx_destroy(x);
      return st;
    }
    c->nthreads = std::max(1, omp_get_num_procs() / nworkers);  // the workers share the host cores
    S->ctxs.push_back(c);
  }
  {
    // reserve the budget in the device's stream-ordered pool once (it keeps
    // freed memory), so that a request's plan is carved from memory the pool
    // already holds instead of growing it (mapping tens of GB) inside the
    // request's latency; without the reservation the pool grows on demand
    CKS(cudaSetDevice(device));
    CKS(device_pool_setup());
    cudaStream_t s = S->ctxs[0]->stream;
    void* blk = nullptr;
    if (cudaMallocAsync(&blk, (size_t)max_device_bytes, s) == cudaSuccess) {
      CKS(cudaFreeAsync(blk, s));
      CKS(cudaStreamSynchronize(s));
    } else {
      (void)cudaGetLastError();
    }
  }
  {
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) greatest = least = 0;
    for (int w = 0; w < nworkers; w++) {
      cudaStream_t h = nullptr;
      if (greatest == least ||
          cudaStreamCreateWithPriority(&h, cudaStreamNonBlocking, greatest) != cudaSuccess) {
        (void)cudaGetLastError();
        h = nullptr;  // no priorities: small requests share the worker's stream
      }
      S->hi.push_back(h);
    }
  }
  fgt_server* raw = S.release();
  for (int w = 0; w < nworkers; w++) raw->workers.emplace_back(server_worker, raw, w);
  *out = raw;
  return FGT_OK;
}

int fgt_server_set_precision(fgt_server* s, int precision) {
  if (!s) return FGT_ERR_BADARG;
  for (fgt_ctx* c : s->ctxs) {
    int st = fgt_ctx_set_precision(c, precision);
    if (st != FGT_OK) return st;
  }
  return FGT_OK;
}

int fgt_server_set_sm_budget(fgt_server* s, int sms) {
  if (!s || sms < 0) return FGT_ERR_BADARG;
  for (fgt_ctx* c : s->ctxs) {
    int st = fgt_ctx_set_sm_budget(c, sms);
    if (st != FGT_OK) return st;
  }
  return FGT_OK;
}

int fgt_server_set_grid_yield(fgt_server* s, int on) {
  if (!s) return FGT_ERR_BADARG;
  for (fgt_ctx* c : s->ctxs) {
    int st = fgt_ctx_set_grid_yield(c, on);
    if (st != FGT_OK) return st;
  }
  return FGT_OK;
}

int fgt_server_submit(fgt_server* s, const fgt_request* req, long long* id) {
  if (!s || !req || !id) return FGT_ERR_BADARG;
  auto* J = new (std::nothrow) fgt_server::Job();
  if (!J) return FGT_ERR_NOMEM;
  J->r = *req;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) {
    delete J;
    return FGT_ERR_BADARG;
  }
  J->id = s->next_id++;
  J->t_sub = now_s();
  if (s->t_first < 0) s->t_first = J->t_sub;
  s->jobs[J->id] = J;
  s->queue.push_back(J);
  s->submitted++;
  *id = J->id;
  s->cv_q.notify_all();  // a worker that takes only small requests may not take this one
  return FGT_OK;
}

int fgt_server_wait(fgt_server* s, long long id, double* latency_s) {
  if (!s) return FGT_ERR_BADARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return FGT_ERR_BADARG;
  fgt_server::Job* J = it->second;
  s->cv_done.wait(lk, [&] { return J->done; });
  const int st = J->status;
  if (latency_s) *latency_s = J->t_end - J->t_sub;
  s->jobs.erase(it);
  delete J;
  return st;
}

int fgt_server_stats_get(fgt_server* s, fgt_server_stats* out) {
  if (!s || !out) return FGT_ERR_BADARG;
  std::lock_guard<std::mutex> lk(s->mu);
  memset(out, 0, sizeof(*out));
  out->submitted = s->submitted;
  out->completed = s->completed;
  out->failed = s->failed;
  out->points = s->points;
  out->peak_bytes = s->peak;
  out->budget_bytes = s->budget;
  if (!s->lat.empty()) {
    std::vector<double> v = s->lat;
    std::sort(v.begin(), v.end());
    auto q = [&](double f) { return v[std::min(v.size() - 1, (size_t)(f * (v.size() - 1) + 0.5))]; };
    out->p50_s = q(0.50);
    out->p99_s = q(0.99);
    out->max_s = v.back();
    double m = 0;
    for (double x : v) m += x;
    out->mean_s = m / v.size();
  }
  out->span_s = s->t_first >= 0 ? s->t_last - s->t_first : 0.0;
  out->hi_priority = s->hi_priority;
  return FGT_OK;
}

int fgt_server_destroy(fgt_server* s) {
  if (!s) return FGT_ERR_BADARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_q.notify_all();
  }
  for (auto& t : s->workers) t.join();
  for (auto& kv : s->jobs) delete kv.second;
  for (cudaStream_t h : s->hi)
    if (h) cudaStreamDestroy(h);
  for (fgt_ctx* c : s->ctxs) fgt_ctx_destroy(c);
  delete s;
  return FGT_OK;
}

}  // extern "C"
