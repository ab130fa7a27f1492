// Spatial shard of one transform over several GPUs (one rank each).
//
// The cut-level boxes are the independent units of the plane-wave FGT:
// formation, merge, split and evaluation below a cut-level box touch only
// its own subtree.  Boxes couple in two places only: mp -> loc, where a
// cut-level box reads the multipole expansions of its plane-wave list
// (colleagues, fgt2d.f:1026-1064 / fgt3d.f:1172-1209), and the near field,
// where a leaf reads the sources of its list1 neighbours (fgt2d.f:1287-1333).
//
// Partition: every box gets the Morton key of the cut-level cell holding its
// lower corner; the distinct keys, in Morton order, are cut into `nranks`
// contiguous ranges of nearly equal point counts (sources + targets), and a
// box belongs to the rank whose range holds its key, so a cut-level box and
// its whole subtree share one owner.  Every rank builds the same tree from
// the same (replicated) points, so all ranks compute the same partition
// without communicating.
//
// Each rank keeps only the tasks of the boxes it owns.  The one exchange:
// after phase 1 (form + merge) rank r sends the cut-level multipole
// expansions that other ranks' mp -> loc tasks read and receives the ones
// its own tasks read.  The near field needs no exchange because the source
// coordinates and charges are replicated.  Every owned point is computed by
// the same tasks in the same order as without the shard, so the sum of the
// ranks' outputs (zero at the points a rank does not own) equals the
// one-GPU result bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "fgt_device.hpp"
#include "fgt_plan.hpp"
#include "fgt_shard.hpp"

namespace fgtb {

namespace {

uint64_t morton(const int* c, int dim, int bits) {
  uint64_t k = 0;
  for (int b = bits - 1; b >= 0; b--)
    for (int d = dim - 1; d >= 0; d--) k = (k << 1) | (uint64_t)((c[d] >> b) & 1);
  return k;
}

// key of the cut-level cell holding the lower corner of box b
uint64_t box_key(const Tree& t, int b, int lc) {
  const int l = t.level[b];
  const double bs = t.boxsize[l];
  int c[3] = {0, 0, 0};
  for (int d = 0; d < t.dim; d++) {
    const double lo0 = t.cen0[d] - t.bs0 / 2;
    int ix = (int)std::floor((t.c(b, d) - lo0) / bs);  // integer box index at level l (centre at ix + 1/2)
    ix = std::max(0, std::min((1 << l) - 1, ix));
    c[d] = l >= lc ? ix >> (l - lc) : ix << (lc - l);
  }
  return morton(c, t.dim, std::max(lc, 1));
}

}  // namespace

int shard_filter(HostPlan& H, int nranks, int rank, ShardInfo& S) {
  S.nranks = nranks;
  S.rank = rank;
  S.send.assign(nranks, {});
  S.recv.assign(nranks, {});
  if (nranks <= 1) return 0;
  if (nranks < 1 || rank < 0 || rank >= nranks) return 1;
  const Tree& t = H.tree;
  const Params& P = H.P;
  if (P.large_delta) {  // no tree: rank 0 computes everything, the others write zeros
    S.large_delta_idle = rank != 0;
    return 0;
  }
  const int nb = t.nboxes;
  const int lc = std::max(0, std::min(P.npwlevel, t.nlevels));
  std::vector<uint64_t> key(nb);
  for (int b = 0; b < nb; b++) key[b] = box_key(t, b, lc);
  // weights: the points of every leaf, on its key
  std::vector<std::pair<uint64_t, long long>> kw;
  kw.reserve(nb);
  for (int b = 0; b < nb; b++)
    if (t.nchild[b] == 0) kw.push_back({key[b], (long long)t.ns(b) + t.nt(b)});
  std::sort(kw.begin(), kw.end());
  std::vector<uint64_t> keys;
  std::vector<long long> wsum;
  long long tot = 0;
  for (size_t i = 0; i < kw.size(); i++) {
    if (keys.empty() || keys.back() != kw[i].first) {
      keys.push_back(kw[i].first);
      wsum.push_back(0);
    }
    wsum.back() += kw[i].second;
    tot += kw[i].second;
  }
  // first key of each rank: the rank boundaries are where the running weight
  // crosses multiples of tot / nranks
  S.key_lo.assign(nranks + 1, UINT64_MAX);
  S.key_lo[0] = 0;
  {
    long long run = 0;
    int r = 1;
    for (size_t i = 0; i < keys.size() && r < nranks; i++) {
      while (r < nranks && run >= (long long)((double)tot * r / nranks)) S.key_lo[r++] = keys[i];
      run += wsum[i];
    }
  }
  auto owner_of_key = [&](uint64_t k) {
    int r = (int)(std::upper_bound(S.key_lo.begin(), S.key_lo.begin() + nranks, k) - S.key_lo.begin()) - 1;
    return std::max(0, r);
  };
  S.owner.resize(nb);
  for (int b = 0; b < nb; b++) S.owner[b] = owner_of_key(key[b]);
  // slot -> box maps
  std::vector<int> mp_box(H.nmp, -1), loc_box(H.nloc, -1);
  for (int b = 0; b < nb; b++) {
    if (H.mp_slot[b] >= 0) mp_box[H.mp_slot[b]] = b;
    if (H.loc_slot[b] >= 0) loc_box[H.loc_slot[b]] = b;
  }
  auto own = [&](int b) { return b >= 0 && S.owner[b] == rank; };
  // form
  {
    std::vector<FormTask> f;
    for (const FormTask& x : H.form)
      if (own(x.box)) f.push_back(x);
    H.form.swap(f);
  }
  // merge / split per level
  auto filter_shift = [&](std::vector<ShiftTask>& v, std::vector<int>& beg, std::vector<int>& end,
                          const std::vector<int>& dst_box) {
    std::vector<ShiftTask> out;
    for (size_t l = 0; l < beg.size(); l++) {
      const int b0 = (int)out.size();
      for (int i = beg[l]; i < end[l]; i++)
        if (own(dst_box[v[i].dst])) out.push_back(v[i]);
      beg[l] = b0;
      end[l] = (int)out.size();
    }
    v.swap(out);
  };
  filter_shift(H.merge, H.merge_beg, H.merge_end, mp_box);
  filter_shift(H.split, H.split_beg, H.split_end, loc_box);
  // mp -> loc, and the exchange lists: every rank's tasks are scanned so
  // that each side of a transfer lists the same slots
  {
    std::vector<std::vector<std::vector<int>>> need(nranks, std::vector<std::vector<int>>(nranks));
    std::vector<M2LTask> m;
    std::vector<M2LNbr> nbr;
    for (const M2LTask& x : H.m2l) {
      const int o = S.owner[loc_box[x.loc]];
      for (int i = x.off; i < x.off + x.cnt; i++) {
        const int so = S.owner[mp_box[H.m2l_nbr[i].mp]];
        if (so != o) need[o][so].push_back(H.m2l_nbr[i].mp);
      }
      if (o != rank) continue;
      M2LTask y = x;
      y.off = (int)nbr.size();
      for (int i = x.off; i < x.off + x.cnt; i++) nbr.push_back(H.m2l_nbr[i]);
      m.push_back(y);
    }
    H.m2l.swap(m);
    H.m2l_nbr.swap(nbr);
    for (int a = 0; a < nranks; a++)
      for (int b = 0; b < nranks; b++) {
        auto& v = need[a][b];
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
      }
    for (int peer = 0; peer < nranks; peer++) {
      S.recv[peer] = need[rank][peer];  // slots owned by peer that this rank reads
      S.send[peer] = need[peer][rank];  // slots of this rank that peer reads
    }
  }
  // evaluation leaves
  {
    std::vector<EvalTask> e;
    for (const EvalTask& x : H.eval)
      if (own(x.box)) e.push_back(x);
    H.eval.swap(e);
  }
  // near field: the box of a task is the leaf holding its first point
  {
    std::vector<int> lb[2], ls[2];  // per set: leaf boxes sorted by first point
    for (int b = 0; b < nb; b++) {
      if (t.nchild[b] != 0) continue;
      if (t.ns(b) > 0) { ls[0].push_back(t.s0[b]); lb[0].push_back(b); }
      if (t.nt(b) > 0) { ls[1].push_back(t.t0[b]); lb[1].push_back(b); }
    }
    for (int s = 0; s < 2; s++) {
      std::vector<int> idx(ls[s].size());
      for (size_t i = 0; i < idx.size(); i++) idx[i] = (int)i;
      std::sort(idx.begin(), idx.end(), [&](int a, int b) { return ls[s][a] < ls[s][b]; });
      std::vector<int> a2, b2;
      for (int i : idx) { a2.push_back(ls[s][i]); b2.push_back(lb[s][i]); }
      ls[s].swap(a2);
      lb[s].swap(b2);
    }
    uvector<DirTask> d;
    uvector<SrcRange> r;
    for (const DirTask& x : H.dir) {
      const int s = x.set ? 1 : 0;
      const auto it = std::upper_bound(ls[s].begin(), ls[s].end(), x.i0);
      const int box = it == ls[s].begin() ? -1 : lb[s][(it - ls[s].begin()) - 1];
      if (!own(box)) continue;
      DirTask y = x;
      y.off = (int)r.size();
      for (int i = x.off; i < x.off + x.cnt; i++) r.push_back(H.dir_src[i]);
      d.push_back(y);
    }
    H.dir.swap(d);
    H.dir_src.swap(r);
  }
  // owned points
  S.owned_src = S.owned_trg = 0;
  for (int b = 0; b < nb; b++)
    if (t.nchild[b] == 0 && own(b)) {
      S.owned_src += t.ns(b);
      S.owned_trg += t.nt(b);
    }
  return 0;
}

// ---- device side: copies of cut-level mp expansions between a plan's pool
// and a contiguous exchange buffer ([i][nd * nexp] complex per listed slot)
namespace {
__global__ void k_mp_pack(const double2* __restrict__ mp, const int* __restrict__ slots, int nslot,
                          size_t per, double2* __restrict__ buf) {
  const size_t n = (size_t)nslot * per;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t i = e / per, r = e - i * per;
    buf[e] = mp[(size_t)slots[i] * per + r];
  }
}
__global__ void k_mp_unpack(double2* __restrict__ mp, const int* __restrict__ slots, int nslot, size_t per,
                            const double2* __restrict__ buf) {
  const size_t n = (size_t)nslot * per;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t i = e / per, r = e - i * per;
    mp[(size_t)slots[i] * per + r] = buf[e];
  }
}
}  // namespace

cudaError_t shard_mp_copy(DevicePlan& D, const int* d_slots, int nslot, double* buf, bool pack,
                          cudaStream_t st) {
  if (nslot <= 0) return cudaSuccess;
  const size_t per = (size_t)D.P.nd * D.P.nexp;
  const size_t n = (size_t)nslot * per;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)8 * D.sm_count);
  if (pack) k_mp_pack<<<blocks, 256, 0, st>>>(D.mp, d_slots, nslot, per, reinterpret_cast<double2*>(buf));
  else k_mp_unpack<<<blocks, 256, 0, st>>>(D.mp, d_slots, nslot, per, reinterpret_cast<const double2*>(buf));
  return cudaGetLastError();
}

}  // namespace fgtb
