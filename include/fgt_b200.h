/*
 * fgt_b200.h -- C ABI of the B200 plane-wave fast Gauss transform.
 *
 * The transform is the point-case plane-wave FGT of flatironinstitute/fgt2d
 * (2d/planewave, 3d/planewave):
 *
 *     pot(x_t) = sum_s charge_s exp(-|x_t - x_s|^2 / delta)
 *
 * at the sources (ifpgh = 1) and/or at separate targets (ifpghtarg = 1), to
 * precision eps.  Arrays follow the reference: column-major Fortran arrays,
 * i.e. sources(dim, ns) is ns consecutive dim-tuples, charge(nd, ns) is ns
 * consecutive nd-tuples, pot(nd, ns) likewise.  Every argument of the
 * Fortran-named entry points is passed by reference.
 *
 * with gradients (ifpgh / ifpghtarg = 2) and Hessians (3) in the reference's
 * layouts: grad(nd, dim, n); hess(nd, 3, n) in 2D ordered xx, xy, yy, and
 * hess(nd, 6, n) in 3D ordered xx, yy, zz, xy, xz, yz.
 *
 * Sources are charges (ifcharge = 1) and/or dipoles (ifdipole = 1: directions
 * rnormal(dim, ns), strengths dipstr(nd, ns), field dipstr n . grad_s of the
 * Gaussian, g2d_directdp_vec).  Supported: ifcharge, ifdipole in {0, 1},
 * ifpgh and ifpghtarg in {0..3}, any nd >= 1.  Other flag values return
 * FGT_ERR_UNSUPPORTED.
 *
 * All entry points return a status (FGT_OK or an error code below) except
 * fgt2d_ / fgt3d_, which keep the reference's subroutine signature and
 * report a failure on stderr; fgt2d_st_ / fgt3d_st_ add a trailing status.
 */
#ifndef FGT_B200_H
#define FGT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
  FGT_OK = 0,
  FGT_ERR_BADARG = 1,      /* nd < 1, delta <= 0, eps not in (0,1), n < 0, NaN */
  FGT_ERR_UNSUPPORTED = 2, /* flags out of range, orders too large */
  FGT_ERR_NOMEM = 3,       /* device or host allocation failed */
  FGT_ERR_CUDA = 4,        /* CUDA runtime error (see fgt_last_cuda_error) */
  FGT_ERR_NODEVICE = 5,    /* no CUDA device */
  FGT_ERR_SCRATCH = 6      /* problem larger than the fixed scratch of fgt_large_delta_noalloc */
};

enum {
  FGT_PREC_FP64 = 0,  /* everything in FP64 (the plain form) */
  FGT_PREC_MIXED = 1, /* FP32 SFU exponentials in the near field, FP64 accumulation */
  FGT_PREC_AUTO = 2   /* MIXED when eps >= 1e-6, FP64 otherwise (default) */
};

enum {
  FGT_TREE_DEVICE = 0, /* tree build with its point work on the GPU (default) */
  FGT_TREE_HOST = 1    /* tree build entirely on the host (OpenMP) */
};

/* Algorithm of a context's plans (fgt_ctx_set_scheme). */
enum {
  /* the plane-wave scheme of 2d/planewave and 3d/planewave (default):
   * Hermite / plane-wave / Taylor expansions on every level from the cut
   * level down */
  FGT_SCHEME_PLANEWAVE = 0,
  /* the NUFFT scheme of 2d/nufft and 3d/nufft: plane-wave expansions at the
   * cut level only, formed from and evaluated at every point of a cut-level
   * box; the reference computes them with type-1 / type-2 NUFFTs (FINUFFT),
   * this library with the exact sums those approximate.  2D: charges only. */
  FGT_SCHEME_NUFFT = 1
};

typedef struct fgt_ctx fgt_ctx;
typedef struct fgt_plan fgt_plan;

typedef struct fgt_plan_info {
  int dim, nd, ns, nt;
  int npwlevel, nlevels, nboxes, npw, nexp, nlmax;
  int nform, neval, ndirect_tasks, nmp, nloc;
  long long direct_pairs, form_sources, eval_points;
  long long device_bytes;
  double host_tree_s, host_lists_s, host_plan_s;
  int large_delta, all_direct;
  int kernel_launches;
  /* algorithmic work per execute: stage (b) bytes counting each distinct
   * expansion once (merge, mp->loc, split; the split's counts only the
   * split tasks that run, the rest being fused into the conversion to
   * Taylor form), stage (a)/(c) flops as 4 * points * npw^dim, stage (d)
   * source-target pairs */
  long long shift_bytes[3];
  double form_flops, eval_flops;
  /* flops of the routes actually taken (Hermite/Taylor or plane wave),
   * counting each multiply-add as 2 and complex ones as 8 */
  double form_route_flops, eval_route_flops;
} fgt_plan_info;

/* ---- context: one device, its stream and default precision -------------- */
int fgt_ctx_create(int device, fgt_ctx** out);
int fgt_ctx_destroy(fgt_ctx* ctx);
int fgt_ctx_set_precision(fgt_ctx* ctx, int precision);
/* OpenMP threads of the host parts of the context's plans (tree, lists,
 * task arrays, staging copies); 0 (the default) uses half the cores, at most
 * 8 (a server's contexts: the cores divided among its workers).  The calling
 * thread's own OpenMP setting is restored when each call returns. */
int fgt_ctx_set_host_threads(fgt_ctx* ctx, int nthreads);
/* where plans built with this context build their tree (FGT_TREE_DEVICE or
 * FGT_TREE_HOST); both give the same tree.  No counterpart in the reference,
 * whose tree is built on the host (pts_tree_build, pts_tree2d4.f:363-590). */
int fgt_ctx_set_tree(fgt_ctx* ctx, int where);
/* how many SMs the persistent kernels of the context's plans (created after
 * the call) size their grids for; 0 (the default) uses every SM.  A smaller
 * budget leaves SMs free for work that arrives while a large transform runs
 * (fgt_server_set_sm_budget).  No counterpart in the reference. */
int fgt_ctx_set_sm_budget(fgt_ctx* ctx, int sms);
/* on != 0: the context's plans (created after the call) launch one CTA per
 * task, instead of persistent CTAs, in the kernels that allow it, so that a
 * large transform's launches let work on other (higher-priority) streams
 * onto the SMs as soon as any of their CTAs finish.  Default off.  No
 * counterpart in the reference. */
int fgt_ctx_set_grid_yield(fgt_ctx* ctx, int on);
/* the algorithm of the plans created after the call (FGT_SCHEME_*): the
 * reference selects it by building 2d/planewave or 2d/nufft (3D likewise),
 * whose fgt2d / fgt3d share one signature (2d/nufft/src/fgt2d.f:19-22). */
int fgt_ctx_set_scheme(fgt_ctx* ctx, int scheme);
/* the context used by the Fortran-named entry points (device 0, created on
 * first use) */
fgt_ctx* fgt_default_ctx(void);
/* the context's CUDA stream (a cudaStream_t) */
void* fgt_ctx_stream(fgt_ctx* ctx);
/* measured FP64 tensor-core (mma.m8n8k4.f64) throughput of the context's
 * device, in TFLOP/s: the denominator of the FP64 form/eval roofline */
int fgt_probe_fp64_mma_tflops(fgt_ctx* ctx, double* tflops);
/* Diagnostics of the tcgen05 tensor-core path (no counterpart in the
 * reference).  fgt_tc_selftest runs one BF16 x 3 compensated tile (M = 128,
 * K = 16, N = n, n a multiple of 16 up to 256) on `device` and returns its
 * largest error relative to the largest entry of an FP64 product;
 * fgt_tc_error reads (and with clear != 0 resets) the flag the tensor-core
 * kernels set when a bounded wait on an MMA completion gave up. */
int fgt_tc_selftest(int device, int n, double* max_rel_err);
int fgt_tc_error(int device, int clear, int* flag);

/* ---- whole transform from host arrays ------------------------------------
 * Replaces fgt2d (2d/planewave/src/fgt2d.f:19-462) and fgt3d
 * (3d/planewave/src/fgt3d.f:19-477): argument meaning, array layouts and
 * output semantics are the reference's (outputs are overwritten). */
int fgt_transform(fgt_ctx* ctx, int dim, int nd, double delta, double eps, int ns,
                  const double* sources, int ifcharge, const double* charge, int ifdipole,
                  const double* rnormal, const double* dipstr, int ifpgh, double* pot, double* grad,
                  double* hess, int nt, const double* targ, int ifpghtarg, double* pottarg,
                  double* gradtarg, double* hesstarg);

/* gfortran-ABI drop-ins for `call fgt2d(...)` / `call fgt3d(...)`
 * (fgt2d.f:19-22, fgt3d.f:19-22); all arguments by reference. */
void fgt2d_(const int* nd, const double* delta, const double* eps, const int* ns,
            const double* sources, const int* ifcharge, const double* charge, const int* ifdipole,
            const double* rnormal, const double* dipstr, const int* iper, const int* ifpgh,
            double* pot, double* grad, double* hess, const int* nt, const double* targ,
            const int* ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg);
void fgt3d_(const int* nd, const double* delta, const double* eps, const int* ns,
            const double* sources, const int* ifcharge, const double* charge, const int* ifdipole,
            const double* rnormal, const double* dipstr, const int* iper, const int* ifpgh,
            double* pot, double* grad, double* hess, const int* nt, const double* targ,
            const int* ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg);
/* the same with a trailing status argument */
void fgt2d_st_(const int* nd, const double* delta, const double* eps, const int* ns,
               const double* sources, const int* ifcharge, const double* charge,
               const int* ifdipole, const double* rnormal, const double* dipstr, const int* iper,
               const int* ifpgh, double* pot, double* grad, double* hess, const int* nt,
               const double* targ, const int* ifpghtarg, double* pottarg, double* gradtarg,
               double* hesstarg, int* ier);
void fgt3d_st_(const int* nd, const double* delta, const double* eps, const int* ns,
               const double* sources, const int* ifcharge, const double* charge,
               const int* ifdipole, const double* rnormal, const double* dipstr, const int* iper,
               const int* ifpgh, double* pot, double* grad, double* hess, const int* nt,
               const double* targ, const int* ifpghtarg, double* pottarg, double* gradtarg,
               double* hesstarg, int* ier);

/* ---- the GPU main at the reference's host/device cut ---------------------
 * fgt2dmain (fgt2d.f:468-478) / fgt3dmain (fgt3d.f:483-493): tree-sorted
 * arrays and the reference's own tree (itree/iptr as built by pts_tree_build,
 * 1-based box ids).  iaddr/rmlexp are accepted and ignored: the device keeps
 * its own expansion pool.  Outputs are incremented, as in the reference.
 * 2D: iptr and ltree are default integers; 3D: integer*8 (fgt3d.f:643-645). */
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
                   double* gradtarg, double* hesstarg);
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
                   double* hesstarg);

/* ---- plans: build the tree once, apply many times ------------------------
 * A plan fixes the points (sources, targets), delta, eps and flags: it holds
 * the tree, the lists and the points sorted into tree order on the device.
 * The execute calls take charges and write the outputs; their point
 * arguments are accepted for symmetry with the reference call and ignored
 * (they may be NULL). */
int fgt_plan_create(fgt_ctx* ctx, int dim, int nd, double delta, double eps, int ns,
                    const double* sources, int nt, const double* targ, int ifpgh, int ifpghtarg,
                    fgt_plan** out);
/* The same for charges and/or dipoles (the orders grow by ifdipole as in
 * fgt2d.f:339-347); execute such plans with the _full calls below. */
int fgt_plan_create_cd(fgt_ctx* ctx, int dim, int nd, double delta, double eps, int ns,
                       const double* sources, int nt, const double* targ, int ifcharge,
                       int ifdipole, int ifpgh, int ifpghtarg, fgt_plan** out);
/* host arrays in and out; copies the charges in and the outputs back */
int fgt_plan_execute_host(fgt_plan* plan, const double* sources, const double* charge,
                          const double* targ, double* pot, double* pottarg);
/* device pointers in the caller's order; runs on `stream` (a cudaStream_t,
 * NULL for the context stream) and returns without synchronising */
int fgt_plan_execute_device(fgt_plan* plan, const double* d_sources, const double* d_charge,
                            const double* d_targ, double* d_pot, double* d_pottarg, void* stream);
/* The same two with the gradient and Hessian arrays of plans created with
 * ifpgh or ifpghtarg >= 2 (layouts as fgt_transform).  A NULL gradient or
 * Hessian array is skipped; the potentials of the flagged sets are required.
 * The reference has no plan API: these split fgt2d's one call
 * (fgt2d.f:19-462) into set-up and apply. */
int fgt_plan_execute_host_pgh(fgt_plan* plan, const double* charge, double* pot, double* grad,
                              double* hess, double* pottarg, double* gradtarg, double* hesstarg);
int fgt_plan_execute_device_pgh(fgt_plan* plan, const double* d_charge, double* d_pot,
                                double* d_grad, double* d_hess, double* d_pottarg,
                                double* d_gradtarg, double* d_hesstarg, void* stream);
/* Every input and output: charge (nd, ns) for plans with charges, rnormal
 * (dim, ns) and dipstr (nd, ns) for plans with dipoles (NULL otherwise). */
int fgt_plan_execute_host_full(fgt_plan* plan, const double* charge, const double* rnormal,
                               const double* dipstr, double* pot, double* grad, double* hess,
                               double* pottarg, double* gradtarg, double* hesstarg);
int fgt_plan_execute_device_full(fgt_plan* plan, const double* d_charge, const double* d_rnormal,
                                 const double* d_dipstr, double* d_pot, double* d_grad,
                                 double* d_hess, double* d_pottarg, double* d_gradtarg,
                                 double* d_hesstarg, void* stream);
/* per-stage device milliseconds of one synchronous execute on device data:
 * gather, form, merge, mp->loc, split, eval, direct, scatter */
int fgt_plan_profile_device(fgt_plan* plan, const double* d_sources, const double* d_charge,
                            const double* d_targ, double* d_pot, double* d_pottarg, float* ms8);
int fgt_plan_get_info(const fgt_plan* plan, fgt_plan_info* info);
/* The plane-wave expansion of one box after the last execute (which = 0:
 * its multipole expansion, formed or merged; 1: its local expansion at the
 * cut level after mp -> loc, or below it after the split), copied into
 * out[2 * nd * nexp] (complex, re/im interleaved) in the reference's layout
 * (2D pw(npw/2, npw, nd), 3D pw(npw, npw, npw/2, nd) with its node
 * orders, fgt2d.f:1518-1610 / fgt3d.f).  box is 0-based in the tree's
 * numbering (the reference's box - 1).  FGT_ERR_BADARG when the box holds
 * no such expansion (this library allocates them only where the transform
 * reads them).  For checking intermediate stages against the reference. */
int fgt_plan_expansion(fgt_plan* plan, int which, int box, double* out);
/* One execute with CUDA events around the plan's dominant tensor-core launch
 * (the Hermite-block MMA kernel of the form order group with the most
 * sources) on the context's stream: its device time (ms), the flops it
 * executes (2 n P^dim nd over the group's n sources), the plane-wave
 * algorithmic count of the same sources (4 n npw^dim nd; NULL to skip) and its
 * name.  FGT_ERR_UNSUPPORTED when the plan has no such launch (all-direct,
 * large-delta). */
int fgt_plan_profile_dominant(fgt_plan* plan, const double* d_charge, double* d_pot, double* d_pottarg,
                              double* ms, double* flops, double* alg_flops, char* name, int name_len);
int fgt_plan_destroy(fgt_plan* plan);

/* ---- spatial shard of one transform over several GPUs ----------------------
 * No counterpart in the reference (which runs on one node).  The cut-level
 * boxes are cut into `nranks` Morton ranges of nearly equal point counts;
 * rank `rank` computes the boxes of its range: their formation, merge,
 * mp -> loc, split, evaluation and near field.  The one exchange is the
 * cut-level multipole expansions that mp -> loc reads across a range
 * boundary (the coupling of fgt2d.f:1026-1064 / fgt3d.f:1172-1209); the
 * points are replicated on every rank.  Use:
 *   fgt_plan_create_shard(...)                  same arguments on every rank
 *   fgt_plan_execute_device_phase(plan, 1, ...)  form + merge
 *   for every peer: fgt_plan_mp_pack(plan, peer, sendbuf[peer]) and send it;
 *     receive recvbuf[peer], then fgt_plan_mp_unpack(plan, peer, recvbuf[peer])
 *   fgt_plan_execute_device_phase(plan, 2, ...)  mp -> loc .. scatter
 * Each rank's outputs hold its owned points and zeros elsewhere; their sum
 * is the one-GPU result bit for bit.  Buffers hold nsend (nrecv) expansions
 * of slot_doubles doubles each (fgt_plan_shard_counts).  A large-delta plan
 * runs whole on rank 0. */
int fgt_plan_create_shard(fgt_ctx* ctx, int dim, int nd, double delta, double eps, int ns,
                          const double* sources, int nt, const double* targ, int ifpgh, int ifpghtarg,
                          int nranks, int rank, fgt_plan** out);
int fgt_plan_shard_counts(fgt_plan* plan, int peer, long long* nsend, long long* nrecv,
                          long long* slot_doubles);
int fgt_plan_shard_owned(fgt_plan* plan, long long* owned_sources, long long* owned_targets);
/* phase 0: the whole execute; 1: through the merge; 2: from mp -> loc on */
int fgt_plan_execute_device_phase(fgt_plan* plan, int phase, const double* d_charge, double* d_pot,
                                  double* d_pottarg, void* stream);
int fgt_plan_mp_pack(fgt_plan* plan, int peer, double* d_buf, void* stream);
int fgt_plan_mp_unpack(fgt_plan* plan, int peer, const double* d_buf, void* stream);
/* Host-only view of a shard (no GPU needed): the host tree and plan of the
 * same points, filtered for (nranks, rank); the exchange lists as mp slot
 * numbers (which = 0: send to peer, 1: receive from peer) and statistics
 * out8 = {owned sources, owned targets, form tasks, eval tasks, near-field
 * tasks, mp -> loc tasks, merge + split tasks, mp slots}. */
typedef struct fgt_host_shard fgt_host_shard;
int fgt_host_shard_create(int dim, int nd, double delta, double eps, int ns, const double* sources, int nt,
                          const double* targ, int ifpgh, int ifpghtarg, int nranks, int rank,
                          fgt_host_shard** out);
int fgt_host_shard_counts(fgt_host_shard* h, int peer, long long* nsend, long long* nrecv);
int fgt_host_shard_slots(fgt_host_shard* h, int peer, int which, int* out);
int fgt_host_shard_stats(fgt_host_shard* h, long long* out8);
int fgt_host_shard_destroy(fgt_host_shard* h);

/* ---- host tree (no device needed) ----------------------------------------
 * The level-restricted tree the transform builds (pts_tree_boxsize0,
 * pts_tree_mem/build/sort: pts_tree2d4.f:34-1258, pts_tree3d.f:34-1685),
 * exposed in the reference's conventions: 1-based box ids, laddr(2,0:nlevels),
 * per-box ranges isrcse(2,nboxes) and the sort permutations isrc/itarg. */
typedef struct fgt_host_tree fgt_host_tree;
int fgt_host_tree_create(int dim, double delta, double eps, int ns, const double* sources, int nt,
                         const double* targ, int nthreads, fgt_host_tree** out);
/* The same tree built with its point work on the context's GPU (the build
 * the plans use by default); the handle is read with the calls below. */
int fgt_device_tree_create(fgt_ctx* ctx, int dim, double delta, double eps, int ns,
                           const double* sources, int nt, const double* targ, fgt_host_tree** out);
/* dims[0..3] = nlevels, nboxes, npwlevel, nlmax; returns FGT_ERR_UNSUPPORTED
 * for the large-delta case, which builds no tree */
int fgt_host_tree_dims(const fgt_host_tree* t, int* dims);
/* field: 0 laddr, 1 ilevel, 2 iparent, 3 nchild, 4 ichild, 5 nnbors, 6 nbors,
 * 7 isrc, 8 isrcse, 9 itarg, 10 itargse (int); 11 centers, 12 boxsize (double).
 * Returns the element count; copies when out != NULL. */
long long fgt_host_tree_field(const fgt_host_tree* t, int field, void* out);
int fgt_host_tree_destroy(fgt_host_tree* t);

/* ---- serving ----------------------------------------------------------------
 * No counterpart in the reference (a Fortran library call).  A server on one
 * device accepts transforms of any dimension, size, delta and eps as they
 * arrive and runs them on worker threads, each with its own stream, so
 * requests that arrive while others are on the GPU overlap with them.  The
 * smallest pending request goes first (the oldest once it has waited 50 ms);
 * a quarter of the workers (at least one of two or more) take only requests
 * of at most 1e5 points, and those run on high-priority streams.
 * Device memory is admitted by footprint: a quarter of max_device_bytes for
 * the requests' point arrays and tree scratch, the rest for their plans,
 * whose exact size is known before allocation; a request that does not fit
 * waits until memory frees up (or runs alone when nothing else is in
 * flight).  max_device_bytes <= 0 uses 80% of the free memory.
 * The request's host arrays must stay valid until fgt_server_wait returns;
 * outputs have fgt_transform's meaning (zeros on failure). */
typedef struct fgt_server fgt_server;
typedef struct fgt_request {
  int dim, nd;
  double delta, eps;
  int ns;
  const double* sources; /* (ns, dim) */
  const double* charge;  /* (ns, nd) */
  int nt;
  const double* targ;    /* (nt, dim), may be NULL */
  int ifpgh, ifpghtarg;
  double* pot;           /* (ns, nd) when ifpgh >= 1 */
  double* pottarg;       /* (nt, nd) when ifpghtarg >= 1 */
  double* grad;          /* (ns, dim, nd) when ifpgh >= 2, else may be NULL */
  double* hess;          /* (ns, H, nd) when ifpgh = 3 */
  double* gradtarg;      /* (nt, dim, nd) when ifpghtarg >= 2 */
  double* hesstarg;      /* (nt, H, nd) when ifpghtarg = 3 */
  int ifdipole;          /* 1: dipoles rnormal (ns, dim), dipstr (ns, nd); charge NULL: none */
  const double* rnormal;
  const double* dipstr;
} fgt_request;
typedef struct fgt_server_stats {
  long long submitted, completed, failed;
  long long points;            /* potentials evaluated by successful requests */
  long long peak_bytes, budget_bytes;
  double p50_s, p99_s, mean_s, max_s;  /* latency: submit -> result on the host */
  double span_s;               /* first submit -> last completion */
  long long hi_priority;       /* requests run on a worker's highest-priority stream
                                  (those of <= 1e5 points, when the device has priorities) */
} fgt_server_stats;
int fgt_server_create(int device, long long max_device_bytes, int nworkers, fgt_server** out);
int fgt_server_set_precision(fgt_server* server, int precision);
/* SMs the persistent kernels of the requests planned afterwards size their
 * grids for (0, the default: every SM); see fgt_ctx_set_sm_budget. */
int fgt_server_set_sm_budget(fgt_server* server, int sms);
/* fgt_ctx_set_grid_yield for the requests planned afterwards */
int fgt_server_set_grid_yield(fgt_server* server, int on);
int fgt_server_submit(fgt_server* server, const fgt_request* request, long long* id);
/* blocks until request id completes; returns its status (and frees its id) */
int fgt_server_wait(fgt_server* server, long long id, double* latency_s);
int fgt_server_stats_get(fgt_server* server, fgt_server_stats* out);
/* finishes the queued requests, then stops the workers */
int fgt_server_destroy(fgt_server* server);

/* ---- allocation-free large-delta transform ----------------------------------
 * No counterpart in the reference.  For callers that cannot let the library
 * allocate device memory -- codes that pass device arrays from their own
 * memory pool under a fixed budget, or latency-critical loops that must not
 * call cudaMalloc, which can synchronise the whole device.  It runs the
 * large-delta transform of fgt2d_large_delta / fgt3d_large_delta
 * (fgt2d.f:1616-1733, fgt3d.f:1783-1914): one Taylor expansion of order
 * `nlocal` about `center` (dim doubles, host memory), formed from all sources
 * and evaluated at the sources (ifpgh = 1) and/or targets (ifpghtarg = 1);
 * the fgt2d/fgt3d driver takes this path when the root box is far smaller
 * than the Gaussian (cut level < -2), with the box centre and nlocal =
 * hlterms(dim, box size, delta, eps) + max(ifpgh, ifpghtarg) - 1.
 * All arrays are device pointers in the caller's layout: sources (ns, dim),
 * charge (ns, nd), targ (nt, dim), pot (ns, nd), pottarg (nt, nd); outputs
 * are overwritten.  The work runs on `stream` (a cudaStream_t, NULL for the
 * default stream) and the call returns without synchronising.
 * Scratch: the local expansion lives in one fixed device array of
 * FGT_NOALLOC_MAX_DOUBLES doubles that every device which loads the library
 * holds until the process exits; nd * (nlocal+1)^dim larger than that returns
 * FGT_ERR_SCRATCH.  All calls share the array: calls that overlap on the GPU
 * race.  The first call on a device looks up the array's device address
 * (a one-time set-up). */
#define FGT_NOALLOC_MAX_DOUBLES 65536
int fgt_large_delta_noalloc(int dim, int nd, double delta, int ns, const double* sources,
                            const double* charge, int nlocal, const double* center, int ifpgh,
                            double* pot, int nt, const double* targ, int ifpghtarg,
                            double* pottarg, void* stream);

/* ---- status -------------------------------------------------------------- */
const char* fgt_status_string(int status);
int fgt_last_cuda_error(void);
const char* fgt_build_info(void);

#ifdef __cplusplus
}
#endif
#endif /* FGT_B200_H */
