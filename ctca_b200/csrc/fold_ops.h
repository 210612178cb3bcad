// fold_ops.h -- the guard-cell reduction of rho / aj / ajdg as a list of
// slab operations, for one rank.
//
// On one rank, OhHelp's oh3_exchange_borders (ohhelp3.c:1011-1046) copies
// border slabs of a periodic axis onto the guard slabs of the same array
// (set_border_exchange / set_border_comm, ohhelp3.c:525-697), and then
// add_boundary_charge (charge.F90:214-412), add_boundary_current
// (psolve1.F90:859-1079) or add_boundary_current2 (psolve1.F90:1081-) fold
// the guards into the interior (periodic) or apply the x2 / mirror rules
// (non-periodic).  Every loop nest of those routines reads and writes
// disjoint planes, so each nest is one data-parallel slab operation; the
// nests run in the reference's order.
#pragma once
#include <vector>

#include "../../include/emses_gpu.h"

namespace emsesg {

struct SlabOp {
  int op;          // 0: dst = src, 1: dst += src, 2: dst *= 2, 3: dst = -src
  int axis;        // slab normal
  int dst0, src0;  // first plane index along the axis
  int depth;       // number of planes
  int lo[3], hi[3];  // inclusive ranges of the other two axes (axis entry unused)
  int c0, nc, cstride;  // components c0, c0+cstride, ... (nc of them)
};

// kind 0: rho-type arrays (ctypes CRH, add_boundary_charge), ncomp components.
// kind 1: aj / ajdg (ctypes CAJ / CJD, add_boundary_current{,2}), ncomp = 3*k.
// kind 2: eb (ctypes CEB): the border exchange only, ncomp = 6.
inline std::vector<SlabOp> fold_ops(const emsesg_config& c, int kind, int ncomp) {
  std::vector<SlabOp> ops;
  const int n[3] = {c.nx, c.ny, c.nz};
  // ctypes as (from, to, size) of the lower and upper sends (ohinit.F90:113-118)
  int fromL, toL, sizeL, fromU, toU, sizeU;
  if (kind == 0) { fromL = 0; toL = 1; sizeL = 1; fromU = 0; toU = -1; sizeU = 1; }
  else if (kind == 2) { fromL = 0; toL = 0; sizeL = 2; fromU = -1; toU = -1; sizeU = 1; }
  else { fromL = -1; toL = 2; sizeL = 3; fromU = -1; toU = -4; sizeU = 3; }
  // Exchange: x, then y, then z; the other axes span exti (inner) or exto
  // (outer) ranges.
  for (int d = 0; d < 3; d++) {
    if (c.nfbnd[d] != 0) continue;
    SlabOp o{};
    for (int e = 0; e < 3; e++) {
      if (e == d) continue;
      if (e < d) { o.lo[e] = toU; o.hi[e] = n[e] + toL + sizeL - 1; }
      else { o.lo[e] = fromL; o.hi[e] = n[e] + fromU + sizeU - 1; }
    }
    o.op = 0; o.axis = d; o.c0 = 0; o.nc = ncomp; o.cstride = 1;
    o.src0 = fromL; o.dst0 = n[d] + toL; o.depth = sizeL;
    ops.push_back(o);
    o.src0 = n[d] + fromU; o.dst0 = toU; o.depth = sizeU;
    ops.push_back(o);
  }
  if (kind == 2) return ops;
  const int sl = toU, su = toL, nl = sizeU, nu = sizeL;
  const int dl = sl + nl, du = su - nu;
  auto box = [&](int axis, int op, int dst0, int src0, int depth, int loa, int hia, int lob, int hib,
                 int c0, int nc, int cs) {
    SlabOp o{};
    o.op = op; o.axis = axis; o.dst0 = dst0; o.src0 = src0; o.depth = depth;
    int a = axis == 0 ? 1 : 0, b = axis == 2 ? 1 : 2;
    o.lo[a] = loa; o.hi[a] = hia; o.lo[b] = lob; o.hi[b] = hib;
    o.c0 = c0; o.nc = nc; o.cstride = cs;
    ops.push_back(o);
  };
  if (kind == 0) {
    // add_boundary_charge, charge.F90:265-409
    int fx = sl + c.nx + (su + nu - sl) - 1, fy = sl + c.ny + (su + nu - sl) - 1;
    int zk = dl + c.nz + (du + nu - dl) - 1, yk = dl + c.ny + (du + nu - dl) - 1;
    // z lower / upper: i, j over sl..sl+l+(su+nu-sl)-1
    if (c.nfbnd[2] == 0) box(2, 1, dl, sl, nl, sl, fx, sl, fy, 0, ncomp, 1);
    else box(2, 2, dl, dl, 1, sl, fx, sl, fy, 0, ncomp, 1);
    if (c.nfbnd[2] == 0) box(2, 1, c.nz + du, c.nz + su, nu, sl, fx, sl, fy, 0, ncomp, 1);
    else box(2, 2, c.nz + du, c.nz + du, 1, sl, fx, sl, fy, 0, ncomp, 1);
    // y lower / upper: i over sl..fx, k over dl..zk
    if (c.nfbnd[1] == 0) box(1, 1, dl, sl, nl, sl, fx, dl, zk, 0, ncomp, 1);
    else box(1, 2, dl, dl, 1, sl, fx, dl, zk, 0, ncomp, 1);
    if (c.nfbnd[1] == 0) box(1, 1, c.ny + du, c.ny + su, nu, sl, fx, dl, zk, 0, ncomp, 1);
    else box(1, 2, c.ny + du, c.ny + du, 1, sl, fx, dl, zk, 0, ncomp, 1);
    // x lower / upper: j over dl..yk, k over dl..zk
    if (c.nfbnd[0] == 0) box(0, 1, dl, sl, nl, dl, yk, dl, zk, 0, ncomp, 1);
    else box(0, 2, dl, dl, 1, dl, yk, dl, zk, 0, ncomp, 1);
    if (c.nfbnd[0] == 0) box(0, 1, c.nx + du, c.nx + su, nu, dl, yk, dl, zk, 0, ncomp, 1);
    else box(0, 2, c.nx + du, c.nx + du, 1, dl, yk, dl, zk, 0, ncomp, 1);
    return ops;
  }
  // add_boundary_current / add_boundary_current2 (psolve1.F90:902-1076),
  // applied to every component triple at once (the triples never mix).
  const int xu = c.nx, yu = c.ny, zu = c.nz;
  int fx = sl + xu + (su + nu - sl) - 1, fy = sl + yu + (su + nu - sl) - 1;
  int zk = dl + zu + (du + nu - dl) - 1, yk = dl + yu + (du + nu - dl) - 1;
  int nt = ncomp / 3;
  // z lower
  if (c.nfbnd[2] == 0) box(2, 1, dl, sl, nl, sl, fx, sl, fy, 0, ncomp, 1);
  else if (c.nfbnd[2] == 1) {
    box(2, 2, 0, 0, 1, sl, fx, sl, fy, 0, nt, 3);  // JX *= 2
    box(2, 2, 0, 0, 1, sl, fx, sl, fy, 1, nt, 3);  // JY *= 2
    box(2, 3, -1, 0, 1, sl, fx, sl, fy, 2, nt, 3); // JZ(k-1) = -JZ(-k)
  }
  // z upper
  if (c.nfbnd[2] == 0) box(2, 1, zu + du, zu + su, nu, sl, fx, sl, fy, 0, ncomp, 1);
  else if (c.nfbnd[2] == 1) {
    box(2, 2, zu, zu, 1, sl, fx, sl, fy, 0, nt, 3);
    box(2, 2, zu, zu, 1, sl, fx, sl, fy, 1, nt, 3);
    box(2, 3, zu, zu - 1, 1, sl, fx, sl, fy, 2, nt, 3);
    box(2, 0, zu + 1, zu - 1, 1, sl, fx, sl, fy, 0, nt, 3);
    box(2, 0, zu + 1, zu - 1, 1, sl, fx, sl, fy, 1, nt, 3);
    box(2, 3, zu + 1, zu - 2, 1, sl, fx, sl, fy, 2, nt, 3);
  }
  // y lower
  if (c.nfbnd[1] == 0) box(1, 1, dl, sl, nl, sl, fx, dl, zk, 0, ncomp, 1);
  else if (c.nfbnd[1] == 1) {
    box(1, 2, 0, 0, 1, sl, fx, dl, zk, 0, nt, 3);
    box(1, 3, -1, 0, 1, sl, fx, dl, zk, 1, nt, 3);
    box(1, 2, 0, 0, 1, sl, fx, dl, zk, 2, nt, 3);
  }
  // y upper
  if (c.nfbnd[1] == 0) box(1, 1, yu + du, yu + su, nu, sl, fx, dl, zk, 0, ncomp, 1);
  else if (c.nfbnd[1] == 1) {
    box(1, 2, yu, yu, 1, sl, fx, dl, zk, 0, nt, 3);
    box(1, 3, yu, yu - 1, 1, sl, fx, dl, zk, 1, nt, 3);
    box(1, 2, yu, yu, 1, sl, fx, dl, zk, 2, nt, 3);
    box(1, 0, yu + 1, yu - 1, 1, sl, fx, dl, zk, 0, nt, 3);
    box(1, 3, yu + 1, yu - 2, 1, sl, fx, dl, zk, 1, nt, 3);
    box(1, 0, yu + 1, yu - 1, 1, sl, fx, dl, zk, 2, nt, 3);
  }
  // x lower
  if (c.nfbnd[0] == 0) box(0, 1, dl, sl, nl, dl, yk, dl, zk, 0, ncomp, 1);
  else if (c.nfbnd[0] == 1) {
    box(0, 3, -1, 0, 1, dl, yk, dl, zk, 0, nt, 3);
    box(0, 2, 0, 0, 1, dl, yk, dl, zk, 1, nt, 3);
    box(0, 2, 0, 0, 1, dl, yk, dl, zk, 2, nt, 3);
  }
  // x upper
  if (c.nfbnd[0] == 0) box(0, 1, xu + du, xu + su, nu, dl, yk, dl, zk, 0, ncomp, 1);
  else if (c.nfbnd[0] == 1) {
    box(0, 3, xu, xu - 1, 1, dl, yk, dl, zk, 0, nt, 3);
    box(0, 2, xu, xu, 1, dl, yk, dl, zk, 1, nt, 3);
    box(0, 2, xu, xu, 1, dl, yk, dl, zk, 2, nt, 3);
    box(0, 3, xu + 1, xu - 2, 1, dl, yk, dl, zk, 0, nt, 3);
    box(0, 0, xu + 1, xu - 1, 1, dl, yk, dl, zk, 1, nt, 3);
    box(0, 0, xu + 1, xu - 1, 1, dl, yk, dl, zk, 2, nt, 3);
  }
  return ops;
}

}  // namespace emsesg
