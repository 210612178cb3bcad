// slab.cuh -- device execution of the guard-fold slab operations (fold_ops.h).
#pragma once
#include <algorithm>

#include "common.cuh"
#include "fold_ops.h"

namespace emsesg {

struct SlabArgs {
  SlabOp o;
  FieldDesc f;
  int64_t count;  // depth * extent_a * extent_b * nc
};

// Element t of one slab operation (also run on the host by a test).
template <typename T>
__host__ __device__ __forceinline__ void slab_apply(T* __restrict__ a, const SlabArgs& s, int64_t t) {
  const SlabOp& o = s.o;
  int ax = o.axis, ea = ax == 0 ? 1 : 0, eb = ax == 2 ? 1 : 2;
  int na = o.hi[ea] - o.lo[ea] + 1, nb = o.hi[eb] - o.lo[eb] + 1;
  int cc = (int)(t % o.nc);
  int64_t r = t / o.nc;
  int ia = (int)(r % na);
  r /= na;
  int ib = (int)(r % nb);
  int p = (int)(r / nb);
  int idx[3], sidx[3];
  idx[ea] = o.lo[ea] + ia;
  idx[eb] = o.lo[eb] + ib;
  idx[ax] = o.dst0 + p;
  sidx[ea] = idx[ea];
  sidx[eb] = idx[eb];
  sidx[ax] = o.src0 + p;
  int comp = o.c0 + cc * o.cstride;
  int64_t d = s.f.at(comp, idx[0], idx[1], idx[2]);
  int64_t sr = s.f.at(comp, sidx[0], sidx[1], sidx[2]);
  switch (o.op) {
    case 0: a[d] = a[sr]; break;
    case 1: a[d] = a[d] + a[sr]; break;
    case 2: a[d] = a[d] * (T)2; break;
    case 3: a[d] = -a[sr]; break;
  }
}

template <typename T>
__global__ void k_slab(T* __restrict__ a, SlabArgs s) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= s.count) return;
  slab_apply(a, s, t);
}

// Up to SLAB_MULTI operations that touch no element another one of them
// reads or writes, in one launch: the threads are dealt out to them in turn.
constexpr int SLAB_MULTI = 4;
template <typename T>
struct SlabMulti {
  T* a[SLAB_MULTI];
  SlabArgs s[SLAB_MULTI];
  int64_t start[SLAB_MULTI + 1];  // first thread of each operation; start[n] = all
  int n;
};

template <typename T>
__global__ void k_slab_multi(SlabMulti<T> m) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m.start[m.n]) return;
  int q = 0;
  while (q + 1 < m.n && t >= m.start[q + 1]) q++;
  slab_apply(m.a[q], m.s[q], t - m.start[q]);
}

template <typename T>
int run_slab_ops(emsesg_ctx* ctx, T* a, const FieldDesc& f, const std::vector<SlabOp>& ops, const char* name) {
  for (const SlabOp& o : ops) {
    SlabArgs s;
    s.o = o;
    s.f = f;
    int ax = o.axis, ea = ax == 0 ? 1 : 0, eb = ax == 2 ? 1 : 2;
    int64_t na = o.hi[ea] - o.lo[ea] + 1, nb = o.hi[eb] - o.lo[eb] + 1;
    s.count = (int64_t)o.depth * na * nb * o.nc;
    if (s.count <= 0) continue;
    int threads = 256;
    int64_t blocks = (s.count + threads - 1) / threads;
    EMSESG_LAUNCH(ctx, name, k_slab<T>, (unsigned)blocks, threads, 0, a, s);
  }
  return EMSESG_OK;
}

// Elements an operation writes and reads, as boxes of (component-blind)
// node indices: w[axis] = its dst planes, r[axis] = its src planes, the other
// axes their ranges; ops 1 and 2 also read their dst.
struct SlabBox {
  int lo[3], hi[3];
};
inline void slab_boxes(const SlabOp& o, SlabBox& w, SlabBox& r) {
  for (int e = 0; e < 3; e++) {
    w.lo[e] = r.lo[e] = o.lo[e];
    w.hi[e] = r.hi[e] = o.hi[e];
  }
  w.lo[o.axis] = o.dst0; w.hi[o.axis] = o.dst0 + o.depth - 1;
  r.lo[o.axis] = o.src0; r.hi[o.axis] = o.src0 + o.depth - 1;
}
inline bool boxes_meet(const SlabBox& a, const SlabBox& b) {
  for (int e = 0; e < 3; e++)
    if (a.hi[e] < b.lo[e] || b.hi[e] < a.lo[e]) return false;
  return true;
}
// True when neither operation writes what the other reads or writes.
inline bool slab_independent(const SlabOp& x, const SlabOp& y) {
  SlabBox wx, rx, wy, ry;
  slab_boxes(x, wx, rx);
  slab_boxes(y, wy, ry);
  return !boxes_meet(wx, wy) && !boxes_meet(wx, ry) && !boxes_meet(wy, rx);
}

// Consecutive operations of a list grouped into stages of at most
// SLAB_MULTI / 2 pairwise independent ones, in list order.
inline std::vector<std::vector<SlabOp>> slab_stages(const std::vector<SlabOp>& ops) {
  std::vector<std::vector<SlabOp>> st;
  for (const SlabOp& o : ops) {
    bool join = !st.empty() && st.back().size() < SLAB_MULTI / 2;
    if (join)
      for (const SlabOp& p : st.back()) join = join && slab_independent(p, o);
    if (join) st.back().push_back(o);
    else st.push_back({o});
  }
  return st;
}

// Runs two operation lists on two arrays (each list in its order; the
// lists are unrelated) in few launches: the k-th stages of both lists share
// one launch.
template <typename T>
int run_slab_ops2(emsesg_ctx* ctx, T* a1, const FieldDesc& f1, const std::vector<SlabOp>& ops1, T* a2,
                  const FieldDesc& f2, const std::vector<SlabOp>& ops2, const char* name) {
  const auto s1 = slab_stages(ops1), s2 = slab_stages(ops2);
  const size_t ns = std::max(s1.size(), s2.size());
  for (size_t k = 0; k < ns; k++) {
    SlabMulti<T> m{};
    m.n = 0;
    int64_t total = 0;
    auto add = [&](T* a, const FieldDesc& f, const SlabOp& o) {
      int ax = o.axis, ea = ax == 0 ? 1 : 0, eb = ax == 2 ? 1 : 2;
      int64_t na = o.hi[ea] - o.lo[ea] + 1, nb = o.hi[eb] - o.lo[eb] + 1;
      int64_t count = (int64_t)o.depth * na * nb * o.nc;
      if (count <= 0) return;
      m.a[m.n] = a;
      m.s[m.n].o = o;
      m.s[m.n].f = f;
      m.s[m.n].count = count;
      m.start[m.n] = total;
      total += count;
      m.n++;
    };
    if (k < s1.size())
      for (const SlabOp& o : s1[k]) add(a1, f1, o);
    if (k < s2.size())
      for (const SlabOp& o : s2[k]) add(a2, f2, o);
    if (m.n == 0) continue;
    m.start[m.n] = total;
    const int threads = 256;
    EMSESG_LAUNCH(ctx, name, k_slab_multi<T>, (unsigned)((total + threads - 1) / threads), threads, 0, m);
  }
  return EMSESG_OK;
}

}  // namespace emsesg
