// slab.cuh -- device execution of the guard-fold slab operations (fold_ops.h).
#pragma once
#include "common.cuh"
#include "fold_ops.h"

namespace emsesg {

struct SlabArgs {
  SlabOp o;
  FieldDesc f;
  int64_t count;  // depth * extent_a * extent_b * nc
};

template <typename T>
__global__ void k_slab(T* __restrict__ a, SlabArgs s) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= s.count) return;
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

}  // namespace emsesg
