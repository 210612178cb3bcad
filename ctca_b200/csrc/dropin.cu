// dropin.cu -- the plain FP64 GPU drop-in: one kernel per reference routine,
// keeping the 64-byte oh_particle records and the Fortran operation order.
//
// This file is compiled with --fmad=false so that no multiply-add is fused:
// positions, velocities, cell indices and counters of grdcrt / psolve1 /
// psolve2 are then bit-identical to an IEEE FP64 evaluation of the Fortran
// statements.  rho and J are summed with FP64 atomics, so their summation
// order (not their terms) differs from the reference's particle order.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "slab.cuh"

namespace emsesg {

namespace {

constexpr int EX = 0, EY = 1, EZ = 2, BX = 3, BY = 4, BZ = 5;
constexpr int JX = 0, JY = 1, JZ = 2;

struct W8 { double v1, v2, v3, v4, v5, v6, v7, v8; };

// Trilinear weights, psolve2.F90:166-183 / charge.F90:173-192.
__device__ __forceinline__ W8 weights(double x1, double y1, double z1) {
  W8 w;
  double xy1 = x1 * y1, xz1 = x1 * z1, yz1 = y1 * z1;
  double z2 = 1.0 - z1;
  double xz2 = x1 * z2, yz2 = y1 * z2;
  w.v3 = xy1 * z1;
  w.v2 = xz1 - w.v3;
  w.v4 = yz1 - w.v3;
  w.v1 = z1 - xz1 - w.v4;
  w.v7 = xy1 * z2;
  w.v6 = xz2 - w.v7;
  w.v8 = yz2 - w.v7;
  w.v5 = z2 - xz2 - w.v8;
  return w;
}

struct PushArgs {
  emsesg_particle* p;
  int64_t n;
  const int64_t* count;   // device count of this species
  int is;
  int64_t packed_base;    // index of the first particle in the packed pbuf
  const double* node;     // 8 doubles per node over (nx+1)(ny+1)(nz+1)
  const emsesg_config* cfg;
  int ustep;
  uint64_t seed, stream;
  const double* randoms;
  int64_t nrand;
  const int64_t* rand_pos;
  const uint32_t* ordinal;
  emsesg_counter* gc;
  int* status;
  long long* diag;
  double* tj;             // psolve1: per-species zigzag scratch (aj layout)
  FieldDesc fa;
};

// The drop-in node field covers nodes 0..n+1 per axis; grdcrt fills 0..n
// (grdcrt.F90:158-160) and node n+1 stays 0.  A particle that a periodic
// wrap leaves exactly on x = slx (x - slx + slx rounding) has i = n and gathers
// node n+1 with weight 0, as the reference reads wrk(n+1) with weight 0.
__device__ __forceinline__ int64_t node_index(const emsesg_config* c, int i, int j, int k) {
  return (int64_t)i + (int64_t)(c->nx + 2) * ((int64_t)j + (int64_t)(c->ny + 2) * k);
}

__device__ __forceinline__ bool cell_ok(const emsesg_config* c, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i <= c->nx && j <= c->ny && k <= c->nz;
}

// Gather + Buneman-Boris + move, psolve2.F90:185-318 (psolve1.F90:201-333).
__device__ __forceinline__ void gather_boris_move(const double* __restrict__ node, const emsesg_config* c,
                                                  emsesg_particle& p, int i, int j, int k, const W8& w,
                                                  double qmp, double gustep) {
  int64_t n1 = node_index(c, i, j, k + 1), n5 = node_index(c, i, j, k);
  int64_t sx = 1, sy = c->nx + 2;
  const double* c1 = node + 8 * n1;            // (i,  j,  k1)
  const double* c2 = node + 8 * (n1 + sx);     // (i1, j,  k1)
  const double* c3 = node + 8 * (n1 + sx + sy);// (i1, j1, k1)
  const double* c4 = node + 8 * (n1 + sy);     // (i,  j1, k1)
  const double* c5 = node + 8 * n5;            // (i,  j,  k)
  const double* c6 = node + 8 * (n5 + sx);
  const double* c7 = node + 8 * (n5 + sx + sy);
  const double* c8 = node + 8 * (n5 + sy);
  double eex = c1[EX] * w.v1 + c2[EX] * w.v2 + c3[EX] * w.v3 + c4[EX] * w.v4 + c5[EX] * w.v5 +
               c6[EX] * w.v6 + c7[EX] * w.v7 + c8[EX] * w.v8;
  double eey = c1[EY] * w.v1 + c2[EY] * w.v2 + c3[EY] * w.v3 + c4[EY] * w.v4 + c5[EY] * w.v5 +
               c6[EY] * w.v6 + c7[EY] * w.v7 + c8[EY] * w.v8;
  double eez = c1[EZ] * w.v1 + c2[EZ] * w.v2 + c3[EZ] * w.v3 + c4[EZ] * w.v4 + c5[EZ] * w.v5 +
               c6[EZ] * w.v6 + c7[EZ] * w.v7 + c8[EZ] * w.v8;
  double bbx = c1[BX] * w.v1 + c2[BX] * w.v2 + c3[BX] * w.v3 + c4[BX] * w.v4 + c5[BX] * w.v5 +
               c6[BX] * w.v6 + c7[BX] * w.v7 + c8[BX] * w.v8;
  double bby = c1[BY] * w.v1 + c2[BY] * w.v2 + c3[BY] * w.v3 + c4[BY] * w.v4 + c5[BY] * w.v5 +
               c6[BY] * w.v6 + c7[BY] * w.v7 + c8[BY] * w.v8;
  double bbz = c1[BZ] * w.v1 + c2[BZ] * w.v2 + c3[BZ] * w.v3 + c4[BZ] * w.v4 + c5[BZ] * w.v5 +
               c6[BZ] * w.v6 + c7[BZ] * w.v7 + c8[BZ] * w.v8;
  const double ewx = 0.0, ewy = 0.0;
  eex = (eex + ewx) * qmp;
  eey = (eey + ewy) * qmp;
  eez = eez * qmp;
  bbx = bbx * qmp;
  bby = bby * qmp;
  bbz = bbz * qmp;
  double boris = 2.0 / (1.0 + bbx * bbx + bby * bby + bbz * bbz);
  p.vx = p.vx + eex;
  p.vy = p.vy + eey;
  p.vz = p.vz + eez;
  double vxt = p.vx + p.vy * bbz - p.vz * bby;
  double vyt = p.vy + p.vz * bbx - p.vx * bbz;
  double vzt = p.vz + p.vx * bby - p.vy * bbx;
  p.vx = p.vx + boris * (vyt * bbz - vzt * bby);
  p.vy = p.vy + boris * (vzt * bbx - vxt * bbz);
  p.vz = p.vz + boris * (vxt * bby - vyt * bbx);
  p.vx = p.vx + eex;
  p.vy = p.vy + eey;
  p.vz = p.vz + eez;
  double xmove = p.vx * gustep, ymove = p.vy * gustep, zmove = p.vz * gustep;
  p.x = p.x + xmove;
  p.y = p.y + ymove;
  p.z = p.z + zmove;
}

// Single-rank nborps: -1 as soon as a crossed axis is neither periodic (0)
// nor reflecting (1), else the rank itself (0).  src/etc/nborps.F90:29-…
__device__ __forceinline__ int nborps_single(const int32_t* nb, bool cx, bool cy, bool cz) {
  if (cx && !(nb[0] == 0 || nb[0] == 1)) return -1;
  if (cy && !(nb[1] == 0 || nb[1] == 1)) return -1;
  if (cz && !(nb[2] == 0 || nb[2] == 1)) return -1;
  return 0;
}

__device__ __forceinline__ void absorb(emsesg_counter* gc, int is, int ipc, int pid) {
  atomicAdd(&gc->influx[is][ipc], 1);
  if (pid >= 0 && pid <= EMSESG_INPC) atomicAdd(&gc->infhist[is][ipc][pid], 1);
}

// Injected-particle random number (psolve2.F90:142-146).
__device__ __forceinline__ bool draw(const PushArgs& a, int64_t m, double& u) {
  if (a.cfg->rng_mode == 1) {
    int64_t k = *a.rand_pos + a.ordinal[m];
    if (k >= a.nrand) return false;
    u = a.randoms[k];
    return true;
  }
  u = hash_u01(a.seed, a.stream, (uint64_t)(a.packed_base + m));
  return true;
}

// Status handling at the top of the particle loop (psolve2.F90:138-152).
// Returns false when the particle is skipped.
__device__ __forceinline__ bool push_status(const PushArgs& a, int64_t m, emsesg_particle& p, double& gustep,
                                            double& qmp) {
  double qm = a.cfg->qm[a.is];
  gustep = 0.0;
  qmp = 0.0;
  if (p.preside < 0) {
    p.nid = -1;
    p.preside = 0;
  } else if (p.preside == EMSESG_PCL_INJECTED) {
    double u;
    if (!draw(a, m, u)) {
      atomicOr(a.status, ST_RANDOMS);
      u = 0.0;
    }
    gustep = (double)a.ustep * u;
    qmp = qm * gustep * 0.5;
    p.preside = 0;
  } else {
    gustep = (double)a.ustep;
    qmp = qm * gustep * 0.5;
  }
  return p.nid != -1;
}

// psolve2, src/pcl2field/psolve2.F90:137-533, one thread per particle.
__global__ void k_psolve2(PushArgs a) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.n || m >= *a.count) return;
  const emsesg_config* c = a.cfg;
  emsesg_particle p = a.p[m];
  double gustep, qmp;
  if (!push_status(a, m, p, gustep, qmp)) { a.p[m] = p; return; }
  const double dxl = 0.0, dyl = 0.0, dzl = 0.0;
  const double dxu = c->nx, dyu = c->ny, dzu = c->nz;
  const double slx = c->nx, sly = c->ny, slz = c->nz;
  const double tslx = 2.0 * slx, tsly = 2.0 * sly, tslz = 2.0 * slz;
  double xlocal = p.x - dxl, ylocal = p.y - dyl, zlocal = p.z - dzl;
  int i = (int)xlocal, j = (int)ylocal, k = (int)zlocal;
  if (!cell_ok(c, i, j, k) || !(xlocal >= 0.0 && ylocal >= 0.0 && zlocal >= 0.0)) {
    report_bad(a.status, a.diag, SITE_PSOLVE2, a.packed_base + m, i + 100000LL * j + 10000000000LL * k);
    return;
  }
  W8 w = weights(xlocal - i, ylocal - j, zlocal - k);
  gather_boris_move(a.node, c, p, i, j, k, w, qmp, gustep);

  int nud = 14;
  if (p.x < dxl) nud -= 1; else if (p.x >= dxu) nud += 1;
  if (p.y < dyl) nud -= 3; else if (p.y >= dyu) nud += 3;
  if (p.z < dzl) nud -= 9; else if (p.z >= dzu) nud += 9;
  if (nud != 14) {
    const int32_t* nb = c->npbnd[a.is];
    p.nid = nborps_single(nb, p.x < dxl || p.x >= dxu, p.y < dyl || p.y >= dyu, p.z < dzl || p.z >= dzu);
    if (p.x < 0.0) {
      if (nb[0] == 0) p.x = p.x + slx;
      else if (nb[0] == 1) { p.x = -p.x; p.vx = -p.vx; }
    } else if (p.x >= slx) {
      if (nb[0] == 0) p.x = p.x - slx;
      else if (nb[0] == 1) { p.x = tslx - p.x; p.vx = -p.vx; }
    }
    if (p.y < 0.0) {
      if (nb[1] == 0) p.y = p.y + sly;
      else if (nb[1] == 1) { p.y = -p.y; p.vy = -p.vy; }
    } else if (p.y >= sly) {
      if (nb[1] == 0) p.y = p.y - sly;
      else if (nb[1] == 1) { p.y = tsly - p.y; p.vy = -p.vy; }
    }
    if (p.z < 0.0) {
      if (nb[2] == 0) p.z = p.z + slz;
      else if (nb[2] == 1) { p.z = -p.z; p.vz = -p.vz; }
    } else if (p.z >= slz) {
      if (nb[2] == 0) p.z = p.z - slz;
      else if (nb[2] == 1) { p.z = tslz - p.z; p.vz = -p.vz; }
    }
    if (p.nid == -1) atomicAdd(&a.gc->nesc[a.is], 1);
  }
  // Internal boundary treatment 1, psolve2.F90:465-531.
  if (c->line_mode != 1) {
    for (int ipc = 0; ipc < c->npc; ipc++) {
      if (p.nid == -1) continue;
      const emsesg_body& b = c->body[ipc];
      bool kill = false;
      if ((b.geotype == 0 || b.geotype == 1) &&
          (p.x >= b.xlpc && p.x <= b.xupc && p.y >= b.ylpc && p.y <= b.yupc && p.z >= b.zlpc && p.z <= b.zupc)) {
        kill = true;
      } else if (b.geotype == 2) {
        double d1, d2, ax;
        if (b.cyl_align == 1) { d1 = p.y - b.cyl_axis[0]; d2 = p.z - b.cyl_axis[1]; ax = p.x; }
        else if (b.cyl_align == 2) { d1 = p.z - b.cyl_axis[0]; d2 = p.x - b.cyl_axis[1]; ax = p.y; }
        else if (b.cyl_align == 3) { d1 = p.x - b.cyl_axis[0]; d2 = p.y - b.cyl_axis[1]; ax = p.z; }
        else continue;
        if (ax >= b.cyl_edge[0] && ax <= b.cyl_edge[1] && d1 * d1 + d2 * d2 < b.radius * b.radius) kill = true;
      } else if (b.geotype == 3) {
        double d1 = p.x - b.sph_center[0], d2 = p.y - b.sph_center[1], d3 = p.z - b.sph_center[2];
        if (d1 * d1 + d2 * d2 + d3 * d3 < b.radius * b.radius) kill = true;
      }
      if (kill) {
        p.nid = -1;
        absorb(a.gc, a.is, ipc, p.pid);
      }
    }
  }
  a.p[m] = p;
}

// positn, src/pcl/positn.F90:50-355: position-only advance (x += v*ustep;
// injected particles still draw, :97-101), outer boundary with nesc counted
// per escaping axis (:228-268), body test with the box bounds as the
// cylinder's axial extent (:283-316).  One thread per particle.
__global__ void k_positn(PushArgs a) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.n || m >= *a.count) return;
  const emsesg_config* c = a.cfg;
  emsesg_particle p = a.p[m];
  double gustep, qmp;
  if (!push_status(a, m, p, gustep, qmp)) { a.p[m] = p; return; }
  const double dxl = 0.0, dyl = 0.0, dzl = 0.0;
  const double dxu = c->nx, dyu = c->ny, dzu = c->nz;
  const double slx = c->nx, sly = c->ny, slz = c->nz;
  const double tslx = 2.0 * slx, tsly = 2.0 * sly, tslz = 2.0 * slz;
  const double us = (double)a.ustep;
  double xmove = p.vx * us, ymove = p.vy * us, zmove = p.vz * us;
  p.x = p.x + xmove;
  p.y = p.y + ymove;
  p.z = p.z + zmove;
  int nud = 14;
  if (p.x < dxl) nud -= 1; else if (p.x >= dxu) nud += 1;
  if (p.y < dyl) nud -= 3; else if (p.y >= dyu) nud += 3;
  if (p.z < dzl) nud -= 9; else if (p.z >= dzu) nud += 9;
  if (nud != 14) {
    const int32_t* nb = c->npbnd[a.is];
    p.nid = nborps_single(nb, p.x < dxl || p.x >= dxu, p.y < dyl || p.y >= dyu, p.z < dzl || p.z >= dzu);
    int esc = 0;
    if (p.x < 0.0) {
      if (nb[0] == 0) p.x = p.x + slx;
      else if (nb[0] == 1) { p.x = -p.x; p.vx = -p.vx; }
      else esc++;
    } else if (p.x >= slx) {
      if (nb[0] == 0) p.x = p.x - slx;
      else if (nb[0] == 1) { p.x = tslx - p.x; p.vx = -p.vx; }
      else esc++;
    }
    if (p.y < 0.0) {
      if (nb[1] == 0) p.y = p.y + sly;
      else if (nb[1] == 1) { p.y = -p.y; p.vy = -p.vy; }
      else esc++;
    } else if (p.y >= sly) {
      if (nb[1] == 0) p.y = p.y - sly;
      else if (nb[1] == 1) { p.y = tsly - p.y; p.vy = -p.vy; }
      else esc++;
    }
    if (p.z < 0.0) {
      if (nb[2] == 0) p.z = p.z + slz;
      else if (nb[2] == 1) { p.z = -p.z; p.vz = -p.vz; }
      else esc++;
    } else if (p.z >= slz) {
      if (nb[2] == 0) p.z = p.z - slz;
      else if (nb[2] == 1) { p.z = tslz - p.z; p.vz = -p.vz; }
      else esc++;
    }
    if (esc) atomicAdd(&a.gc->nesc[a.is], esc);
  }
  if (c->line_mode != 1) {
    for (int ipc = 0; ipc < c->npc; ipc++) {
      if (p.nid == -1) continue;
      const emsesg_body& b = c->body[ipc];
      bool kill = false;
      if ((b.geotype == 0 || b.geotype == 1) &&
          (p.x >= b.xlpc && p.x <= b.xupc && p.y >= b.ylpc && p.y <= b.yupc && p.z >= b.zlpc && p.z <= b.zupc)) {
        kill = true;
      } else if (b.geotype == 2) {
        double d1, d2, ax, lo, hi;
        if (b.cyl_align == 1) { d1 = p.y - b.cyl_axis[0]; d2 = p.z - b.cyl_axis[1]; ax = p.x; lo = b.xlpc; hi = b.xupc; }
        else if (b.cyl_align == 2) { d1 = p.z - b.cyl_axis[0]; d2 = p.x - b.cyl_axis[1]; ax = p.y; lo = b.ylpc; hi = b.yupc; }
        else if (b.cyl_align == 3) { d1 = p.x - b.cyl_axis[0]; d2 = p.y - b.cyl_axis[1]; ax = p.z; lo = b.zlpc; hi = b.zupc; }
        else continue;
        if (ax >= lo && ax <= hi && d1 * d1 + d2 * d2 < b.radius * b.radius) kill = true;
      } else if (b.geotype == 3) {
        double d1 = p.x - b.sph_center[0], d2 = p.y - b.sph_center[1], d3 = p.z - b.sph_center[2];
        if (d1 * d1 + d2 * d2 + d3 * d3 < b.radius * b.radius) kill = true;
      }
      if (kill) {
        p.nid = -1;
        absorb(a.gc, a.is, ipc, p.pid);
      }
    }
  }
  a.p[m] = p;
}

// psolve1, src/pcl2field/psolve1.F90:146-789: push with floor() indices and
// the zigzag current into the per-species scratch tj (wrk(TJX:TJZ)).
__global__ void k_psolve1(PushArgs a) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.n || m >= *a.count) return;
  const emsesg_config* c = a.cfg;
  emsesg_particle p = a.p[m];
  double gustep, qmp;
  if (!push_status(a, m, p, gustep, qmp)) { a.p[m] = p; return; }
  const double dxl = 0.0, dyl = 0.0, dzl = 0.0;
  const double dxu = c->nx, dyu = c->ny, dzu = c->nz;
  const double slx = c->nx, sly = c->ny, slz = c->nz;
  const double tslx = 2.0 * slx, tsly = 2.0 * sly, tslz = 2.0 * slz;
  const int ngx = c->nx, ngy = c->ny, ngz = c->nz;
  const double dngx = ngx, dngy = ngy, dngz = ngz;
  const double rustep = 1.0 / a.ustep;

  double xlocalb = p.x - dxl, ylocalb = p.y - dyl, zlocalb = p.z - dzl;
  int ib = (int)floor(xlocalb), jb = (int)floor(ylocalb), kb = (int)floor(zlocalb);
  if (!cell_ok(c, ib, jb, kb)) {
    report_bad(a.status, a.diag, SITE_PSOLVE1, a.packed_base + m, ib + 100000LL * jb + 10000000000LL * kb);
    return;
  }
  double xb = ib, yb = jb, zb = kb;
  int i1b = ib + 1, j1b = jb + 1, k1b = kb + 1;
  W8 w = weights(xlocalb - xb, ylocalb - yb, zlocalb - zb);
  gather_boris_move(a.node, c, p, ib, jb, kb, w, qmp, gustep);

  double xlocala, ylocala, zlocala, xa, ya, za, xr, yr, zr;
  int ia, ja, ka, i1a, j1a, k1a;
  int nud = 14;
  if (p.x < dxl) nud -= 1; else if (p.x >= dxu) nud += 1;
  if (p.y < dyl) nud -= 3; else if (p.y >= dyu) nud += 3;
  if (p.z < dzl) nud -= 9; else if (p.z >= dzu) nud += 9;
  if (nud == 14) {
    xlocala = p.x - dxl; ylocala = p.y - dyl; zlocala = p.z - dzl;
    ia = (int)floor(xlocala); ja = (int)floor(ylocala); ka = (int)floor(zlocala);
    xa = ia; ya = ja; za = ka;
    i1a = ia + 1; j1a = ja + 1; k1a = ka + 1;
    xr = (ib == ia) ? (xlocalb + xlocala) * 0.5 : fmax(xb, xa);
    yr = (jb == ja) ? (ylocalb + ylocala) * 0.5 : fmax(yb, ya);
    zr = (kb == ka) ? (zlocalb + zlocala) * 0.5 : fmax(zb, za);
  } else {
    const int32_t* nb = c->npbnd[a.is];
    p.nid = nborps_single(nb, p.x < dxl || p.x >= dxu, p.y < dyl || p.y >= dyu, p.z < dzl || p.z >= dzu);
    if (p.x < 0.0) {
      if (nb[0] == 0) { xlocala = p.x; p.x = p.x + slx; ia = -1; xa = -1.0; i1a = 0; xr = 0.0; }
      else if (nb[0] == 1) { p.x = -p.x; p.vx = -p.vx; xlocala = p.x; ia = 0; xa = 0.0; i1a = 1; xr = 0.0; }
      else { xlocala = -1.0; ia = -1; xa = -1.0; i1a = 0; xr = 0.0; }
    } else if (p.x >= slx) {
      if (nb[0] == 0) { xlocala = p.x - dxl; p.x = p.x - slx; ia = ngx; xa = dngx; i1a = ngx + 1; xr = dngx; }
      else if (nb[0] == 1) { p.x = tslx - p.x; p.vx = -p.vx; xlocala = p.x - dxl; ia = ngx - 1; xa = dngx - 1.0; i1a = ngx; xr = dngx; }
      else { xlocala = dngx + 1.0; ia = ngx; xa = dngx; i1a = ngx + 1; xr = dngx; }
    } else {
      xlocala = p.x - dxl; ia = (int)floor(xlocala); xa = ia; i1a = ia + 1;
      xr = (ib == ia) ? (xlocalb + xlocala) * 0.5 : fmax(xb, xa);
    }
    if (p.y < 0.0) {
      if (nb[1] == 0) { ylocala = p.y; p.y = p.y + sly; ja = -1; ya = -1.0; j1a = 0; yr = 0.0; }
      else if (nb[1] == 1) { p.y = -p.y; p.vy = -p.vy; ylocala = p.y; ja = 0; ya = 0.0; j1a = 1; yr = 0.0; }
      else { ylocala = -1.0; ja = -1; ya = -1.0; j1a = 0; yr = 0.0; }
    } else if (p.y >= sly) {
      if (nb[1] == 0) { ylocala = p.y - dyl; p.y = p.y - sly; ja = ngy; ya = dngy; j1a = ngy + 1; yr = dngy; }
      else if (nb[1] == 1) { p.y = tsly - p.y; p.vy = -p.vy; ylocala = p.y - dyl; ja = ngy - 1; ya = dngy - 1.0; j1a = ngy; yr = dngy; }
      else { ylocala = dngy + 1.0; ja = ngy; ya = dngy; j1a = ngy + 1; yr = dngy; }
    } else {
      ylocala = p.y - dyl; ja = (int)floor(ylocala); ya = ja; j1a = ja + 1;
      yr = (jb == ja) ? (ylocalb + ylocala) * 0.5 : fmax(yb, ya);
    }
    if (p.z < 0.0) {
      if (nb[2] == 0) { zlocala = p.z; p.z = p.z + slz; ka = -1; za = -1.0; k1a = 0; zr = 0.0; }
      else if (nb[2] == 1) { p.z = -p.z; p.vz = -p.vz; zlocala = p.z; ka = 0; za = 0.0; k1a = 1; zr = 0.0; }
      else { zlocala = -1.0; ka = -1; za = -1.0; k1a = 0; zr = 0.0; }
    } else if (p.z >= slz) {
      if (nb[2] == 0) { zlocala = p.z - dzl; p.z = p.z - slz; ka = ngz; za = dngz; k1a = ngz + 1; zr = dngz; }
      else if (nb[2] == 1) { p.z = tslz - p.z; p.vz = -p.vz; zlocala = p.z - dzl; ka = ngz - 1; za = dngz - 1.0; k1a = ngz; zr = dngz; }
      else { zlocala = dngz + 1.0; ka = ngz; za = dngz; k1a = ngz + 1; zr = dngz; }
    } else {
      zlocala = p.z - dzl; ka = (int)floor(zlocala); za = ka; k1a = ka + 1;
      zr = (kb == ka) ? (zlocalb + zlocala) * 0.5 : fmax(zb, za);
    }
    if (p.nid == -1) atomicAdd(&a.gc->nesc[a.is], 1);
  }

  // Internal boundary treatment 1, psolve1.F90:639-715.
  if (c->line_mode != 1) {
    for (int ipc = 0; ipc < c->npc; ipc++) {
      if (p.nid == -1) continue;
      const emsesg_body& b = c->body[ipc];
      if (b.geotype == 0 || b.geotype == 1) {
        double xlc = b.xlpc - dxl, xuc = b.xupc - dxl, ylc = b.ylpc - dyl, yuc = b.yupc - dyl;
        double zlc = b.zlpc - dzl, zuc = b.zupc - dzl;
        if (xlocalb >= xlc && xlocalb <= xuc && ylocalb >= ylc && ylocalb <= yuc && zlocalb >= zlc && zlocalb <= zuc) {
          xlocalb = xr; ylocalb = yr; zlocalb = zr;
        }
        if (xlocala >= xlc && xlocala <= xuc && ylocala >= ylc && ylocala <= yuc && zlocala >= zlc && zlocala <= zuc) {
          p.nid = -1;
          absorb(a.gc, a.is, ipc, p.pid);
          xlocala = xr; ylocala = yr; zlocala = zr;
        }
      } else if (b.geotype == 2) {
        double d1, d2, ax;
        if (b.cyl_align == 1) { d1 = p.y - b.cyl_axis[0]; d2 = p.z - b.cyl_axis[1]; ax = p.x; }
        else if (b.cyl_align == 2) { d1 = p.z - b.cyl_axis[0]; d2 = p.x - b.cyl_axis[1]; ax = p.y; }
        else if (b.cyl_align == 3) { d1 = p.x - b.cyl_axis[0]; d2 = p.y - b.cyl_axis[1]; ax = p.z; }
        else continue;
        if (ax >= b.cyl_edge[0] && ax <= b.cyl_edge[1] && d1 * d1 + d2 * d2 < b.radius * b.radius) {
          p.nid = -1;
          absorb(a.gc, a.is, ipc, p.pid);
        }
      } else if (b.geotype == 3) {
        double d1 = p.x - b.sph_center[0], d2 = p.y - b.sph_center[1], d3 = p.z - b.sph_center[2];
        if (d1 * d1 + d2 * d2 + d3 * d3 < b.radius * b.radius) {
          p.nid = -1;
          absorb(a.gc, a.is, ipc, p.pid);
        }
      }
    }
  }

  // Zigzag weights, psolve1.F90:717-757.
  double xd1 = (xr + xlocalb) * 0.5 - xb, yd1 = (yr + ylocalb) * 0.5 - yb, zd1 = (zr + zlocalb) * 0.5 - zb;
  double vvx1 = (xr - xlocalb) * rustep, vvy1 = (yr - ylocalb) * rustep, vvz1 = (zr - zlocalb) * rustep;
  double vx1w4 = yd1 * zd1, vx1w2 = yd1 - vx1w4, vx1w3 = zd1 - vx1w4, vx1w1 = 1.0 - yd1 - vx1w3;
  double vy1w4 = xd1 * zd1, vy1w2 = xd1 - vy1w4, vy1w3 = zd1 - vy1w4, vy1w1 = 1.0 - xd1 - vy1w3;
  double vz1w4 = xd1 * yd1, vz1w2 = xd1 - vz1w4, vz1w3 = yd1 - vz1w4, vz1w1 = 1.0 - xd1 - vz1w3;
  double xd2 = (xlocala + xr) * 0.5 - xa, yd2 = (ylocala + yr) * 0.5 - ya, zd2 = (zlocala + zr) * 0.5 - za;
  double vvx2 = (xlocala - xr) * rustep, vvy2 = (ylocala - yr) * rustep, vvz2 = (zlocala - zr) * rustep;
  double vx2w4 = yd2 * zd2, vx2w2 = yd2 - vx2w4, vx2w3 = zd2 - vx2w4, vx2w1 = 1.0 - yd2 - vx2w3;
  double vy2w4 = xd2 * zd2, vy2w2 = xd2 - vy2w4, vy2w3 = zd2 - vy2w4, vy2w1 = 1.0 - xd2 - vy2w3;
  double vz2w4 = xd2 * yd2, vz2w2 = xd2 - vz2w4, vz2w3 = yd2 - vz2w4, vz2w1 = 1.0 - xd2 - vz2w3;

  const FieldDesc& f = a.fa;
  double* t = a.tj;
  // The 24 scatter-adds of psolve1.F90:759-789; all indices lie in -1..n+1.
  atomicAdd(&t[f.at(JX, ib, jb, kb)], vvx1 * vx1w1);
  atomicAdd(&t[f.at(JY, ib, jb, kb)], vvy1 * vy1w1);
  atomicAdd(&t[f.at(JZ, ib, jb, kb)], vvz1 * vz1w1);
  atomicAdd(&t[f.at(JX, ib, j1b, kb)], vvx1 * vx1w2);
  atomicAdd(&t[f.at(JY, i1b, jb, kb)], vvy1 * vy1w2);
  atomicAdd(&t[f.at(JZ, i1b, jb, kb)], vvz1 * vz1w2);
  atomicAdd(&t[f.at(JX, ib, jb, k1b)], vvx1 * vx1w3);
  atomicAdd(&t[f.at(JY, ib, jb, k1b)], vvy1 * vy1w3);
  atomicAdd(&t[f.at(JZ, ib, j1b, kb)], vvz1 * vz1w3);
  atomicAdd(&t[f.at(JX, ib, j1b, k1b)], vvx1 * vx1w4);
  atomicAdd(&t[f.at(JY, i1b, jb, k1b)], vvy1 * vy1w4);
  atomicAdd(&t[f.at(JZ, i1b, j1b, kb)], vvz1 * vz1w4);
  atomicAdd(&t[f.at(JX, ia, ja, ka)], vvx2 * vx2w1);
  atomicAdd(&t[f.at(JY, ia, ja, ka)], vvy2 * vy2w1);
  atomicAdd(&t[f.at(JZ, ia, ja, ka)], vvz2 * vz2w1);
  atomicAdd(&t[f.at(JX, ia, j1a, ka)], vvx2 * vx2w2);
  atomicAdd(&t[f.at(JY, i1a, ja, ka)], vvy2 * vy2w2);
  atomicAdd(&t[f.at(JZ, i1a, ja, ka)], vvz2 * vz2w2);
  atomicAdd(&t[f.at(JX, ia, ja, k1a)], vvx2 * vx2w3);
  atomicAdd(&t[f.at(JY, ia, ja, k1a)], vvy2 * vy2w3);
  atomicAdd(&t[f.at(JZ, ia, j1a, ka)], vvz2 * vz2w3);
  atomicAdd(&t[f.at(JX, ia, j1a, k1a)], vvx2 * vx2w4);
  atomicAdd(&t[f.at(JY, i1a, ja, k1a)], vvy2 * vy2w4);
  atomicAdd(&t[f.at(JZ, i1a, j1a, ka)], vvz2 * vz2w4);
  a.p[m] = p;
}

// aj += wrk(TJ)*q (and ajdg), psolve1.F90:793-817, over -1..n+1.
__global__ void k_flush_tj(const double* __restrict__ tj, double* aj, double* ajdg, FieldDesc fa, FieldDesc fj,
                           int nx, int ny, int nz, double qs, int iss, int do_dg) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t ex = nx + 3, ey = ny + 3, ez = nz + 3;
  if (t >= ex * ey * ez) return;
  int i = (int)(t % ex) - 1, j = (int)((t / ex) % ey) - 1, k = (int)(t / (ex * ey)) - 1;
  for (int d = 0; d < 3; d++) {
    double v = tj[fa.at(d, i, j, k)];
    aj[fa.at(d, i, j, k)] = aj[fa.at(d, i, j, k)] + v * qs;
    if (do_dg) ajdg[fj.at(iss + d, i, j, k)] = ajdg[fj.at(iss + d, i, j, k)] + v * qs;
  }
}

// chgacm update after the species loop, psolve2.F90:537-543.
__global__ void k_chgacm(const emsesg_config* c, emsesg_counter* gc) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int is = 0; is < c->nspec; is++)
    for (int ipc = 0; ipc < c->npc; ipc++)
      if (c->body[ipc].ncond > 0) {
        double add = (double)gc->influx[is][ipc] * c->q[is] * c->body[ipc].sqdscaled;
        gc->chgacm[ipc][0] = gc->chgacm[ipc][0] + add;
        gc->chgacm[ipc][1] = gc->chgacm[ipc][1] + add;
      }
}

// grdcrt, src/field/grdcrt.F90:156-169 and :214-230, one thread per node.
__global__ void k_grdcrt(const double* __restrict__ eb, double* __restrict__ node, FieldDesc fe, int nx, int ny,
                         int nz, double e0x, double e0y, double e0z, double b0x, double b0y, double b0z) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t ex = nx + 1, ey = ny + 1, ez = nz + 1;
  if (t >= ex * ey * ez) return;
  int i = (int)(t % ex), j = (int)((t / ex) % ey), k = (int)(t / (ex * ey));
  double* o = node + 8 * ((int64_t)i + (ex + 1) * ((int64_t)j + (ey + 1) * k));
  o[EX] = 0.5 * (eb[fe.at(EX, i, j, k)] + eb[fe.at(EX, i - 1, j, k)]) + e0x;
  o[EY] = 0.5 * (eb[fe.at(EY, i, j, k)] + eb[fe.at(EY, i, j - 1, k)]) + e0y;
  o[EZ] = 0.5 * (eb[fe.at(EZ, i, j, k)] + eb[fe.at(EZ, i, j, k - 1)]) + e0z;
  o[BX] = 0.25 * (eb[fe.at(BX, i, j, k)] + eb[fe.at(BX, i, j - 1, k)] + eb[fe.at(BX, i, j, k - 1)] +
                   eb[fe.at(BX, i, j - 1, k - 1)]) + b0x;
  o[BY] = 0.25 * (eb[fe.at(BY, i, j, k)] + eb[fe.at(BY, i - 1, j, k)] + eb[fe.at(BY, i, j, k - 1)] +
                   eb[fe.at(BY, i - 1, j, k - 1)]) + b0y;
  o[BZ] = 0.25 * (eb[fe.at(BZ, i, j, k)] + eb[fe.at(BZ, i - 1, j, k)] + eb[fe.at(BZ, i, j - 1, k)] +
                   eb[fe.at(BZ, i - 1, j - 1, k)]) + b0z;
  o[6] = 0.0;
  o[7] = 0.0;
}

// Writes the node field into the reference wrk layout (EX..BZ at 0..n).
__global__ void k_node_to_wrk(const double* __restrict__ node, double* wrk, FieldDesc fw, int nx, int ny, int nz) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t ex = nx + 1, ey = ny + 1, ez = nz + 1;
  if (t >= ex * ey * ez) return;
  int i = (int)(t % ex), j = (int)((t / ex) % ey), k = (int)(t / (ex * ey));
  int64_t nd = (int64_t)i + (ex + 1) * ((int64_t)j + (ey + 1) * k);
  for (int cc = 0; cc < 6; cc++) wrk[fw.at(cc, i, j, k)] = node[8 * nd + cc];
}

struct ChargeArgs {
  emsesg_particle* p;
  int64_t n;
  const int64_t* count;
  int is, nspec, func;
  double q;
  double *rho, *rhodg, *rhobk, *rhobksp;
  FieldDesc fr, fd;
  const emsesg_config* cfg;
  int* status;
  long long* diag;
};

__device__ __forceinline__ void distribute(double* rh, const FieldDesc& f, int cc, int i, int j, int k, double qc,
                                           const W8& w) {
  atomicAdd(&rh[f.at(cc, i, j, k + 1)], w.v1 * qc);
  atomicAdd(&rh[f.at(cc, i + 1, j, k + 1)], w.v2 * qc);
  atomicAdd(&rh[f.at(cc, i + 1, j + 1, k + 1)], w.v3 * qc);
  atomicAdd(&rh[f.at(cc, i, j + 1, k + 1)], w.v4 * qc);
  atomicAdd(&rh[f.at(cc, i, j, k)], w.v5 * qc);
  atomicAdd(&rh[f.at(cc, i + 1, j, k)], w.v6 * qc);
  atomicAdd(&rh[f.at(cc, i + 1, j + 1, k)], w.v7 * qc);
  atomicAdd(&rh[f.at(cc, i, j + 1, k)], w.v8 * qc);
}

// charge, src/pcl2field/charge.F90:53-146, one thread per particle.
__global__ void k_charge(ChargeArgs a) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.n || m >= *a.count) return;
  emsesg_particle& p = a.p[m];
  if (p.nid == -1) return;
  double xlocal = p.x, ylocal = p.y, zlocal = p.z;
  int i = (int)xlocal, j = (int)ylocal, k = (int)zlocal;
  const emsesg_config* c = a.cfg;
  if (i < -1 || j < -1 || k < -1 || i > c->nx || j > c->ny || k > c->nz) {
    report_bad(a.status, a.diag, SITE_CHARGE, m, i + 100000LL * j + 10000000000LL * k);
    return;
  }
  W8 w = weights(xlocal - i, ylocal - j, zlocal - k);
  int func = a.func;
  if (p.preside >= 0) {
    if (func == 0 || func == 2) distribute(a.rho, a.fr, 0, i, j, k, a.q, w);
    if (func == 1 || func == 2) distribute(a.rhodg, a.fd, a.is, i, j, k, a.q, w);
  } else if (p.preside == EMSESG_PCL_TO_BE_ACCUMULATED || p.preside == EMSESG_PCL_TO_BE_ACCUMULATED_AS_ANTIPCL) {
    double qq = p.preside == EMSESG_PCL_TO_BE_ACCUMULATED ? a.q : -a.q;
    distribute(a.rhobk, a.fr, 0, i, j, k, qq, w);
    distribute(a.rhobksp + (int64_t)a.is * a.fr.size(), a.fr, 0, i, j, k, qq, w);
    if (func == 1 || func == 2) {
      if (func == 2 && p.preside == EMSESG_PCL_TO_BE_ACCUMULATED_AS_ANTIPCL) distribute(a.rhodg, a.fd, a.is, i, j, k, qq, w);
      distribute(a.rhodg, a.fd, a.nspec + a.is, i, j, k, qq, w);
    }
    p.nid = -1;
    p.preside = 0;
  }
}

// rhoupd, src/field/rhoupd.F90:40-49.
__global__ void k_rhoupd(double* rho, const double* __restrict__ aj, FieldDesc fr, FieldDesc fa, int nx, int ny,
                         int nz) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t ex = nx + 1, ey = ny + 1, ez = nz + 1;
  if (t >= ex * ey * ez) return;
  int i = (int)(t % ex), j = (int)((t / ex) % ey), k = (int)(t / (ex * ey));
  rho[fr.at(0, i, j, k)] = rho[fr.at(0, i, j, k)] -
      (aj[fa.at(JX, i, j, k)] - aj[fa.at(JX, i - 1, j, k)] + aj[fa.at(JY, i, j, k)] - aj[fa.at(JY, i, j - 1, k)] +
       aj[fa.at(JZ, i, j, k)] - aj[fa.at(JZ, i, j, k - 1)]) * 2.0;
}

// bfield, src/field/bfield.F90:37-53: B(i,j,k) for i,j,k in -1..n, from E
// (the reference's statement order; B written, E read only).
__global__ void k_bfield(double* eb, FieldDesc f, int nx, int ny, int nz) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t ex = nx + 2, ey = ny + 2, ez = nz + 2;
  if (t >= ex * ey * ez) return;
  const int i = (int)(t % ex) - 1, j = (int)((t / ex) % ey) - 1, k = (int)(t / (ex * ey)) - 1;
  eb[f.at(BX, i, j, k)] = eb[f.at(BX, i, j, k)] + eb[f.at(EY, i, j, k + 1)] - eb[f.at(EY, i, j, k)] -
                          eb[f.at(EZ, i, j + 1, k)] + eb[f.at(EZ, i, j, k)];
  eb[f.at(BY, i, j, k)] = eb[f.at(BY, i, j, k)] + eb[f.at(EZ, i + 1, j, k)] - eb[f.at(EZ, i, j, k)] -
                          eb[f.at(EX, i, j, k + 1)] + eb[f.at(EX, i, j, k)];
  eb[f.at(BZ, i, j, k)] = eb[f.at(BZ, i, j, k)] + eb[f.at(EX, i, j + 1, k)] - eb[f.at(EX, i, j, k)] -
                          eb[f.at(EY, i + 1, j, k)] + eb[f.at(EY, i, j, k)];
}

// efield, src/field/efield.F90:54-70 (no lumped elements): E(i,j,k) for
// i,j,k in 0..n, from B and J (E written, B and J read only).
__global__ void k_efield(double* eb, const double* __restrict__ aj, FieldDesc f, FieldDesc fa, int nx, int ny,
                         int nz, double tcs, double dlt) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t ex = nx + 1, ey = ny + 1, ez = nz + 1;
  if (t >= ex * ey * ez) return;
  const int i = (int)(t % ex), j = (int)((t / ex) % ey), k = (int)(t / (ex * ey));
  eb[f.at(EX, i, j, k)] = eb[f.at(EX, i, j, k)] +
                          tcs * (eb[f.at(BZ, i, j, k)] - eb[f.at(BZ, i, j - 1, k)] - eb[f.at(BY, i, j, k)] +
                                 eb[f.at(BY, i, j, k - 1)]) -
                          dlt * aj[fa.at(JX, i, j, k)];
  eb[f.at(EY, i, j, k)] = eb[f.at(EY, i, j, k)] +
                          tcs * (eb[f.at(BX, i, j, k)] - eb[f.at(BX, i, j, k - 1)] - eb[f.at(BZ, i, j, k)] +
                                 eb[f.at(BZ, i - 1, j, k)]) -
                          dlt * aj[fa.at(JY, i, j, k)];
  eb[f.at(EZ, i, j, k)] = eb[f.at(EZ, i, j, k)] +
                          tcs * (eb[f.at(BY, i, j, k)] - eb[f.at(BY, i - 1, j, k)] - eb[f.at(BX, i, j, k)] +
                                 eb[f.at(BX, i, j - 1, k)]) -
                          dlt * aj[fa.at(JZ, i, j, k)];
}

// Sum of v_d^2 of live particles (energy.F90:38-43); FP64 block partials.
__global__ void k_energy(const emsesg_particle* __restrict__ p, int64_t n, const int64_t* count, double* out) {
  __shared__ double s[3][256];
  double t[3] = {0, 0, 0};
  int64_t nn = min(n, *count);
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < nn; m += (int64_t)gridDim.x * blockDim.x) {
    if (p[m].nid == -1) continue;
    t[0] += p[m].vx * p[m].vx;
    t[1] += p[m].vy * p[m].vy;
    t[2] += p[m].vz * p[m].vz;
  }
  for (int d = 0; d < 3; d++) s[d][threadIdx.x] = t[d];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int d = 0; d < 3; d++) s[d][threadIdx.x] += s[d][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; d++) atomicAdd(&out[d], s[d][0]);
}

// Canonical sort key: tile-major cell key of int() of the position, clamped.
__device__ __forceinline__ uint32_t sort_key(const emsesg_config* c, double x, double y, double z, const int* t,
                                             const int* nt) {
  int ci[3];
  double pos[3] = {x, y, z};
  int n[3] = {c->nx, c->ny, c->nz};
  for (int d = 0; d < 3; d++) {
    int v = pos[d] < 0.0 ? 0 : (int)fmin(pos[d], (double)(n[d] - 1));
    ci[d] = min(max(v, 0), n[d] - 1);
  }
  uint32_t tile = (uint32_t)(ci[0] / t[0]) + (uint32_t)nt[0] * ((uint32_t)(ci[1] / t[1]) + (uint32_t)nt[1] * (uint32_t)(ci[2] / t[2]));
  uint32_t in = (uint32_t)(ci[0] % t[0]) + (uint32_t)t[0] * ((uint32_t)(ci[1] % t[1]) + (uint32_t)t[1] * (uint32_t)(ci[2] % t[2]));
  return tile * (uint32_t)(t[0] * t[1] * t[2]) + in;
}

struct KeyArgs { int t[3], nt[3]; };

__global__ void k_make_keys(const emsesg_particle* __restrict__ p, int64_t n, const emsesg_config* c, KeyArgs ka,
                            uint32_t* keys, uint32_t* vals) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  keys[m] = sort_key(c, p[m].x, p[m].y, p[m].z, ka.t, ka.nt);
  vals[m] = (uint32_t)m;
}

__global__ void k_gather_particles(const emsesg_particle* __restrict__ src, emsesg_particle* __restrict__ dst,
                                   const uint32_t* __restrict__ idx, int64_t n) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  dst[m] = src[idx[m]];
}

__global__ void k_live_flags(const emsesg_particle* __restrict__ p, int64_t n, uint32_t* flags) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  flags[m] = p[m].nid != -1 ? 1u : 0u;
}

__global__ void k_compact_scatter(const emsesg_particle* __restrict__ src, emsesg_particle* __restrict__ dst,
                                  const uint32_t* __restrict__ pos, int64_t n) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  if (src[m].nid != -1) dst[pos[m]] = src[m];
}

__global__ void k_injected_flags(const emsesg_particle* __restrict__ p, int64_t n, const int64_t* count,
                                 uint32_t* flags) {
  int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  flags[m] = (m < *count && p[m].preside == EMSESG_PCL_INJECTED) ? 1u : 0u;
}

__global__ void k_advance(int64_t* pos, const uint32_t* total) { *pos += *total; }

__global__ void k_set_count(int64_t* count, const uint32_t* total) { *count = *total; }

// Synthetic plasma, same streams as orc_load_plasma (oracle/emses_oracle.cpp).
// Particles m0 .. m0+n-1 of species `is` into p[0 .. n).
__global__ void k_load_plasma(emsesg_particle* p, int64_t m0, int64_t n, int ppc, int nx, int ny, int is,
                              uint64_t seed, double vth, double vdx, double vdy, double vdz) {
  const int64_t loc = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (loc >= n) return;
  const int64_t m = m0 + loc;
  int64_t cell = m / ppc;
  int i = (int)(cell % nx), j = (int)((cell / nx) % ny), k = (int)(cell / ((int64_t)nx * ny));
  uint64_t st = 1000 + is;
  double u[8];
  for (int s = 0; s < 7; s++) u[s] = hash_u01(seed, st, (uint64_t)m * 8 + s);
  const double twopi = 6.283185307179586;
  emsesg_particle q;
  q.x = i + u[0];
  q.y = j + u[1];
  q.z = k + u[2];
  double r1 = sqrt(-2.0 * log(1.0 - u[3]));
  double r2 = sqrt(-2.0 * log(1.0 - u[5]));
  q.vx = vth * r1 * cos(twopi * u[4]) + vdx;
  q.vy = vth * r1 * sin(twopi * u[4]) + vdy;
  q.vz = vth * r2 * cos(twopi * u[6]) + vdz;
  q.pid = 0;
  q.preside = 0;
  q.nid = 0;
  q.spec = is + 1;
  p[loc] = q;
}

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

}  // namespace

int download_wrk(emsesg_ctx* ctx, double* host) {
  FieldDesc fw = field_desc(ctx->cfg, EMSESG_FIELD_WRK);
  EMSESG_CUDA(ctx, cudaMemsetAsync(ctx->field[EMSESG_FIELD_WRK], 0, fw.size() * sizeof(double), ctx->stream));
  int64_t nn = (int64_t)(ctx->cfg.nx + 1) * (ctx->cfg.ny + 1) * (ctx->cfg.nz + 1);
  EMSESG_LAUNCH(ctx, "node_to_wrk", k_node_to_wrk, nblk(nn), 256, 0, ctx->node64, ctx->field[EMSESG_FIELD_WRK], fw,
                ctx->cfg.nx, ctx->cfg.ny, ctx->cfg.nz);
  EMSESG_CUDA(ctx, cudaMemcpyAsync(host, ctx->field[EMSESG_FIELD_WRK], fw.size() * sizeof(double),
                                   cudaMemcpyDeviceToHost, ctx->stream));
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return EMSESG_OK;
}

}  // namespace emsesg

using namespace emsesg;


namespace {

int check_ps(emsesg_ctx* ctx, int ps) {
  if (!ctx) return EMSESG_ERR_ARG;
  if (ps == 2) return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "ps=2 (helper subdomain) is not supported on one rank");
  if (ps != 1) return set_error(ctx, EMSESG_ERR_ARG, "ps must be 1");
  return EMSESG_OK;
}

int64_t max_count(emsesg_ctx* ctx) {
  int64_t m = 0;
  for (int is = 0; is < ctx->cfg.nspec; is++) m = std::max(m, ctx->seg.capacity[is]);
  return m;
}

// Ordinals of injected particles for the pre-drawn random stream.
int prepare_ordinals(emsesg_ctx* ctx, int is, const uint32_t** ord) {
  *ord = nullptr;
  if (ctx->cfg.rng_mode != 1) return EMSESG_OK;
  int rc = ensure_sort_scratch(ctx, max_count(ctx));
  if (rc) return rc;
  int64_t n = ctx->totalp[is];
  uint32_t* flags = ctx->sort.keys[1];
  EMSESG_LAUNCH(ctx, "injected_flags", k_injected_flags, nblk(n), 256, 0, ctx->pbuf + ctx->seg.base[is], n,
                ctx->d_count + is, flags);
  rc = exclusive_scan_u32(ctx, flags, n);
  if (rc) return rc;
  *ord = flags;
  return EMSESG_OK;
}

int advance_randoms(emsesg_ctx* ctx, int is) {
  if (ctx->cfg.rng_mode != 1) return EMSESG_OK;
  // total injected = scan total, left by exclusive_scan_u32 in scan_tmp[0]
  EMSESG_LAUNCH(ctx, "advance_randoms", k_advance, 1, 1, 0, ctx->d_rand_pos, ctx->sort.scan_tmp);
  return EMSESG_OK;
}

PushArgs push_args(emsesg_ctx* ctx, int is, int ustep) {
  PushArgs a{};
  a.p = ctx->pbuf + ctx->seg.base[is];
  a.n = ctx->totalp[is];
  a.count = ctx->d_count + is;
  a.is = is;
  int64_t pb = 0;
  for (int s = 0; s < is; s++) pb += ctx->totalp[s];
  a.packed_base = pb;
  a.node = ctx->node64;
  a.cfg = ctx->d_cfg;
  a.ustep = ustep;
  a.seed = ctx->cfg.rng_seed;
  a.stream = ctx->rng_stream;
  a.randoms = ctx->d_randoms;
  a.nrand = ctx->n_randoms;
  a.rand_pos = ctx->d_rand_pos;
  a.gc = ctx->d_counter;
  a.status = ctx->d_status;
  a.diag = ctx->d_diag;
  a.tj = ctx->tj;
  a.fa = field_desc(ctx->cfg, EMSESG_FIELD_AJ);
  return a;
}

}  // namespace

extern "C" int emsesg_grdcrt(emsesg_ctx* ctx, int ps) {
  int rc = check_ps(ctx, ps);
  if (rc) return rc;
  if ((rc = apply_pending_eb(ctx))) return rc;
  const emsesg_config& c = ctx->cfg;
  int64_t nn = (int64_t)(c.nx + 1) * (c.ny + 1) * (c.nz + 1);
  EMSESG_LAUNCH(ctx, "grdcrt", k_grdcrt, nblk(nn), 256, 0, ctx->field[EMSESG_FIELD_EB], ctx->node64,
                field_desc(c, EMSESG_FIELD_EB), c.nx, c.ny, c.nz, c.e0[0], c.e0[1], c.e0[2], c.b0[0], c.b0[1],
                c.b0[2]);
  return EMSESG_OK;
}

static int finish_push(emsesg_ctx* ctx, emsesg_counter* gcount) {
  EMSESG_LAUNCH(ctx, "chgacm", k_chgacm, 1, 32, 0, ctx->d_cfg, ctx->d_counter);
  ctx->rng_stream++;
  if (gcount) {
    int rc = emsesg_get_counters(ctx, gcount);
    if (rc) return rc;
    return emsesg_synchronize(ctx);
  }
  return EMSESG_OK;
}

extern "C" int emsesg_psolve2(emsesg_ctx* ctx, int ps, int ustep, emsesg_counter* gcount) {
  int rc = check_ps(ctx, ps);
  if (rc) return rc;
  if (ustep < 1) return set_error(ctx, EMSESG_ERR_ARG, "ustep must be >= 1");
  if (gcount && (rc = emsesg_set_counters(ctx, gcount))) return rc;
  for (int is = 0; is < ctx->cfg.nspec; is++) {
    if (ctx->totalp[is] == 0) continue;
    const uint32_t* ord;
    if ((rc = prepare_ordinals(ctx, is, &ord))) return rc;
    PushArgs a = push_args(ctx, is, ustep);
    a.ordinal = ord;
    EMSESG_LAUNCH(ctx, "psolve2", k_psolve2, nblk(a.n), 256, 0, a);
    if ((rc = advance_randoms(ctx, is))) return rc;
  }
  return finish_push(ctx, gcount);
}

extern "C" int emsesg_positn(emsesg_ctx* ctx, int ps, int ustep, emsesg_counter* gcount) {
  int rc = check_ps(ctx, ps);
  if (rc) return rc;
  if (ustep < 1) return set_error(ctx, EMSESG_ERR_ARG, "ustep must be >= 1");
  if (gcount && (rc = emsesg_set_counters(ctx, gcount))) return rc;
  for (int is = 0; is < ctx->cfg.nspec; is++) {
    if (ctx->totalp[is] == 0) continue;
    const uint32_t* ord;
    if ((rc = prepare_ordinals(ctx, is, &ord))) return rc;
    PushArgs a = push_args(ctx, is, ustep);
    a.ordinal = ord;
    EMSESG_LAUNCH(ctx, "positn", k_positn, nblk(a.n), 256, 0, a);
    if ((rc = advance_randoms(ctx, is))) return rc;
  }
  ctx->rng_stream++;
  if (gcount) {
    if ((rc = emsesg_get_counters(ctx, gcount))) return rc;
    return emsesg_synchronize(ctx);
  }
  return EMSESG_OK;
}

extern "C" int emsesg_psolve1(emsesg_ctx* ctx, int ps, int ustep, int func, emsesg_counter* gcount) {
  int rc = check_ps(ctx, ps);
  if (rc) return rc;
  if (ustep < 1) return set_error(ctx, EMSESG_ERR_ARG, "ustep must be >= 1");
  if (gcount && (rc = emsesg_set_counters(ctx, gcount))) return rc;
  const emsesg_config& c = ctx->cfg;
  FieldDesc fa = field_desc(c, EMSESG_FIELD_AJ), fj = field_desc(c, EMSESG_FIELD_AJDG);
  int64_t ng = (int64_t)(c.nx + 3) * (c.ny + 3) * (c.nz + 3);
  for (int is = 0; is < c.nspec; is++) {
    // wrk(TJX:TJZ, :, :, :) = 0, psolve1.F90:143
    EMSESG_CUDA(ctx, cudaMemsetAsync(ctx->tj, 0, fa.size() * sizeof(double), ctx->stream));
    if (ctx->totalp[is] > 0) {
      const uint32_t* ord;
      if ((rc = prepare_ordinals(ctx, is, &ord))) return rc;
      PushArgs a = push_args(ctx, is, ustep);
      a.ordinal = ord;
      EMSESG_LAUNCH(ctx, "psolve1", k_psolve1, nblk(a.n), 256, 0, a);
      if ((rc = advance_randoms(ctx, is))) return rc;
    }
    EMSESG_LAUNCH(ctx, "flush_tj", k_flush_tj, nblk(ng), 256, 0, ctx->tj, ctx->field[EMSESG_FIELD_AJ],
                  ctx->field[EMSESG_FIELD_AJDG], fa, fj, c.nx, c.ny, c.nz, c.q[is], is * 3, func == 1 ? 1 : 0);
  }
  return finish_push(ctx, gcount);
}

extern "C" int emsesg_charge(emsesg_ctx* ctx, int ps, int func) {
  int rc = check_ps(ctx, ps);
  if (rc) return rc;
  if (func < 0 || func > 2) return set_error(ctx, EMSESG_ERR_ARG, "func must be 0, 1 or 2");
  const emsesg_config& c = ctx->cfg;
  if (func == 0 || func == 2) EMSESG_CUDA(ctx, cudaMemsetAsync(ctx->field[EMSESG_FIELD_RHO], 0,
                                                               field_desc(c, EMSESG_FIELD_RHO).size() * sizeof(double), ctx->stream));
  if (func == 1 || func == 2) EMSESG_CUDA(ctx, cudaMemsetAsync(ctx->field[EMSESG_FIELD_RHODG], 0,
                                                               field_desc(c, EMSESG_FIELD_RHODG).size() * sizeof(double), ctx->stream));
  for (int is = 0; is < c.nspec; is++) {
    if (ctx->totalp[is] == 0) continue;
    ChargeArgs a{};
    a.p = ctx->pbuf + ctx->seg.base[is];
    a.n = ctx->totalp[is];
    a.count = ctx->d_count + is;
    a.is = is;
    a.nspec = c.nspec;
    a.func = func;
    a.q = c.q[is];
    a.rho = ctx->field[EMSESG_FIELD_RHO];
    a.rhodg = ctx->field[EMSESG_FIELD_RHODG];
    a.rhobk = ctx->field[EMSESG_FIELD_RHOBK];
    a.rhobksp = ctx->field[EMSESG_FIELD_RHOBKSP];
    a.fr = field_desc(c, EMSESG_FIELD_RHO);
    a.fd = field_desc(c, EMSESG_FIELD_RHODG);
    a.cfg = ctx->d_cfg;
    a.status = ctx->d_status;
    a.diag = ctx->d_diag;
    EMSESG_LAUNCH(ctx, "charge", k_charge, nblk(a.n), 256, 0, a);
  }
  return EMSESG_OK;
}

extern "C" int emsesg_reduce_rho(emsesg_ctx* ctx, int field) {
  if (!ctx) return EMSESG_ERR_ARG;
  if (field != EMSESG_FIELD_RHO && field != EMSESG_FIELD_RHODG && field != EMSESG_FIELD_RHOBK &&
      field != EMSESG_FIELD_RHOBKSP)
    return set_error(ctx, EMSESG_ERR_ARG, "reduce_rho takes a rho-type field");
  FieldDesc f = field_desc(ctx->cfg, field);
  int narr = field == EMSESG_FIELD_RHOBKSP ? ctx->cfg.nspec : 1;
  std::vector<SlabOp> ops = fold_ops(ctx->cfg, 0, f.nc);
  for (int a = 0; a < narr; a++) {
    int rc = run_slab_ops(ctx, ctx->field[field] + (int64_t)a * f.size(), f, ops, "reduce_rho");
    if (rc) return rc;
  }
  return EMSESG_OK;
}

extern "C" int emsesg_reduce_aj(emsesg_ctx* ctx) {
  if (!ctx) return EMSESG_ERR_ARG;
  FieldDesc f = field_desc(ctx->cfg, EMSESG_FIELD_AJ);
  return run_slab_ops(ctx, ctx->field[EMSESG_FIELD_AJ], f, fold_ops(ctx->cfg, 1, 3), "reduce_aj");
}

extern "C" int emsesg_reduce_ajdg(emsesg_ctx* ctx) {
  if (!ctx) return EMSESG_ERR_ARG;
  FieldDesc f = field_desc(ctx->cfg, EMSESG_FIELD_AJDG);
  return run_slab_ops(ctx, ctx->field[EMSESG_FIELD_AJDG], f, fold_ops(ctx->cfg, 1, f.nc), "reduce_ajdg");
}

extern "C" int emsesg_rhoupd(emsesg_ctx* ctx, int ps) {
  int rc = check_ps(ctx, ps);
  if (rc) return rc;
  const emsesg_config& c = ctx->cfg;
  int64_t nn = (int64_t)(c.nx + 1) * (c.ny + 1) * (c.nz + 1);
  EMSESG_LAUNCH(ctx, "rhoupd", k_rhoupd, nblk(nn), 256, 0, ctx->field[EMSESG_FIELD_RHO],
                ctx->field[EMSESG_FIELD_AJ], field_desc(c, EMSESG_FIELD_RHO), field_desc(c, EMSESG_FIELD_AJ), c.nx,
                c.ny, c.nz);
  return EMSESG_OK;
}

extern "C" int emsesg_bfield(emsesg_ctx* ctx, int ps) {
  int rc = check_ps(ctx, ps);
  if (rc) return rc;
  if ((rc = apply_pending_eb(ctx))) return rc;
  const emsesg_config& c = ctx->cfg;
  const int64_t nn = (int64_t)(c.nx + 2) * (c.ny + 2) * (c.nz + 2);
  EMSESG_LAUNCH(ctx, "bfield", k_bfield, nblk(nn), 256, 0, ctx->field[EMSESG_FIELD_EB],
                field_desc(c, EMSESG_FIELD_EB), c.nx, c.ny, c.nz);
  return EMSESG_OK;
}

extern "C" int emsesg_efield(emsesg_ctx* ctx, int ps, double tcs, double dlt) {
  int rc = check_ps(ctx, ps);
  if (rc) return rc;
  if ((rc = apply_pending_eb(ctx))) return rc;
  const emsesg_config& c = ctx->cfg;
  const int64_t nn = (int64_t)(c.nx + 1) * (c.ny + 1) * (c.nz + 1);
  EMSESG_LAUNCH(ctx, "efield", k_efield, nblk(nn), 256, 0, ctx->field[EMSESG_FIELD_EB], ctx->field[EMSESG_FIELD_AJ],
                field_desc(c, EMSESG_FIELD_EB), field_desc(c, EMSESG_FIELD_AJ), c.nx, c.ny, c.nz, tcs, dlt);
  return EMSESG_OK;
}

extern "C" int emsesg_exchange_eb(emsesg_ctx* ctx) {
  if (!ctx) return EMSESG_ERR_ARG;
  int rc = apply_pending_eb(ctx);
  if (rc) return rc;
  const FieldDesc f = field_desc(ctx->cfg, EMSESG_FIELD_EB);
  return run_slab_ops(ctx, ctx->field[EMSESG_FIELD_EB], f, fold_ops(ctx->cfg, 2, 6), "exchange_eb");
}

extern "C" int emsesg_energy(emsesg_ctx* ctx, double* engk) {
  if (!ctx || !engk) return EMSESG_ERR_ARG;
  const emsesg_config& c = ctx->cfg;
  EMSESG_CUDA(ctx, cudaMemsetAsync(ctx->d_sum, 0, 3 * EMSESG_ISPEC * sizeof(double), ctx->stream));
  for (int is = 0; is < c.nspec; is++) {
    int64_t n = ctx->totalp[is];
    if (n == 0) continue;
    unsigned blocks = (unsigned)std::min<int64_t>(nblk(n), 148 * 8);
    EMSESG_LAUNCH(ctx, "energy", k_energy, blocks, 256, 0, ctx->pbuf + ctx->seg.base[is], n, ctx->d_count + is,
                  ctx->d_sum + 3 * is);
  }
  double s[3 * EMSESG_ISPEC];
  EMSESG_CUDA(ctx, cudaMemcpyAsync(s, ctx->d_sum, sizeof s, cudaMemcpyDeviceToHost, ctx->stream));
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  double vol = (double)c.nx * (double)c.ny * (double)c.nz;
  for (int is = 0; is < c.nspec; is++)
    for (int d = 0; d < 3; d++) engk[is * 3 + d] = 0.5 * c.rm[is] * s[3 * is + d] / vol;
  return emsesg_synchronize(ctx);
}

namespace {
KeyArgs key_args(const emsesg_config& c) {
  KeyArgs ka;
  int n[3] = {c.nx, c.ny, c.nz};
  for (int d = 0; d < 3; d++) {
    ka.t[d] = c.sort_tile[d] > 0 ? std::min(c.sort_tile[d], n[d]) : n[d];
    ka.nt[d] = (n[d] + ka.t[d] - 1) / ka.t[d];
  }
  return ka;
}
int key_bits_for(uint64_t maxkey) {
  int b = 1;
  while (b < 32 && (1ULL << b) <= maxkey) b++;
  return b;
}
int ensure_pbuf2(emsesg_ctx* ctx) {
  if (ctx->pbuf2) return EMSESG_OK;
  int64_t cap = 0;
  for (int is = 0; is < ctx->cfg.nspec; is++) cap += ctx->seg.capacity[is];
  EMSESG_CUDA(ctx, cudaMalloc(&ctx->pbuf2, std::max<int64_t>(cap, 1) * sizeof(emsesg_particle)));
  return EMSESG_OK;
}
}  // namespace

// spsort, src/etc/spsort.F90:29-35: every species segment sorted by the
// canonical key (stable), replacing particle_sort_ (psort-struct.c:7-9).
extern "C" int emsesg_spsort(emsesg_ctx* ctx, int ps) {
  int rc = check_ps(ctx, ps);
  if (rc) return rc;
  if ((rc = ensure_sort_scratch(ctx, max_count(ctx)))) return rc;
  if ((rc = ensure_pbuf2(ctx))) return rc;
  KeyArgs ka = key_args(ctx->cfg);
  uint64_t maxkey = (uint64_t)ka.nt[0] * ka.nt[1] * ka.nt[2] * ka.t[0] * ka.t[1] * ka.t[2];
  int bits = key_bits_for(maxkey);
  for (int is = 0; is < ctx->cfg.nspec; is++) {
    int64_t n = ctx->totalp[is];
    if (n <= 1) continue;
    emsesg_particle* p = ctx->pbuf + ctx->seg.base[is];
    EMSESG_LAUNCH(ctx, "sort_keys", k_make_keys, nblk(n), 256, 0, p, n, ctx->d_cfg, ka, ctx->sort.keys[0],
                  ctx->sort.vals[0]);
    uint32_t *ko, *vo;
    if ((rc = sort_pairs(ctx, ctx->sort.keys[0], ctx->sort.vals[0], n, bits, &ko, &vo))) return rc;
    emsesg_particle* q = ctx->pbuf2 + ctx->seg.base[is];
    EMSESG_LAUNCH(ctx, "sort_gather", k_gather_particles, nblk(n), 256, 0, p, q, vo, n);
    EMSESG_CUDA(ctx, cudaMemcpyAsync(p, q, n * sizeof(emsesg_particle), cudaMemcpyDeviceToDevice, ctx->stream));
  }
  return EMSESG_OK;
}

// Single-rank compaction (the part of oh3_transbound that one rank needs):
// drop nid == -1, keep order, update counts.
extern "C" int emsesg_compact(emsesg_ctx* ctx, int ps, int64_t* totalp) {
  int rc = check_ps(ctx, ps);
  if (rc) return rc;
  if ((rc = ensure_sort_scratch(ctx, max_count(ctx)))) return rc;
  if ((rc = ensure_pbuf2(ctx))) return rc;
  for (int is = 0; is < ctx->cfg.nspec; is++) {
    int64_t n = ctx->totalp[is];
    if (n == 0) continue;
    emsesg_particle* p = ctx->pbuf + ctx->seg.base[is];
    emsesg_particle* q = ctx->pbuf2 + ctx->seg.base[is];
    uint32_t* flags = ctx->sort.keys[0];
    EMSESG_LAUNCH(ctx, "live_flags", k_live_flags, nblk(n), 256, 0, p, n, flags);
    if ((rc = exclusive_scan_u32(ctx, flags, n))) return rc;
    EMSESG_LAUNCH(ctx, "compact_scatter", k_compact_scatter, nblk(n), 256, 0, p, q, flags, n);
    EMSESG_LAUNCH(ctx, "set_count", k_set_count, 1, 1, 0, ctx->d_count + is, ctx->sort.scan_tmp);
    EMSESG_CUDA(ctx, cudaMemcpyAsync(ctx->totalp + is, ctx->d_count + is, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                     ctx->stream));
    EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->totalp[is] > 0)
      EMSESG_CUDA(ctx, cudaMemcpyAsync(p, q, ctx->totalp[is] * sizeof(emsesg_particle), cudaMemcpyDeviceToDevice,
                                       ctx->stream));
  }
  if (totalp)
    for (int is = 0; is < ctx->cfg.nspec; is++) totalp[is] = ctx->totalp[is];
  return emsesg_synchronize(ctx);
}

int emsesg::plasma_records(emsesg_ctx* ctx, emsesg_particle* dst, int is, int64_t m0, int64_t n,
                           const emsesg_plasma* pl) {
  const emsesg_config& c = ctx->cfg;
  EMSESG_LAUNCH(ctx, "load_plasma", k_load_plasma, nblk(n), 256, 0, dst, m0, n, pl->ppc[is], c.nx, c.ny, is,
                pl->seed, pl->vth[is], pl->vdrift[is][0], pl->vdrift[is][1], pl->vdrift[is][2]);
  return EMSESG_OK;
}

extern "C" int emsesg_load_plasma(emsesg_ctx* ctx, const emsesg_plasma* pl) {
  if (!ctx || !pl) return EMSESG_ERR_ARG;
  if (ctx->cfg.flags & EMSESG_FLAG_FP32_ONLY)
    return set_error(ctx, EMSESG_ERR_STATE, "FP32-only context: use emsesg_fx_load_plasma");
  const emsesg_config& c = ctx->cfg;
  int64_t ncell = (int64_t)c.nx * c.ny * c.nz;
  for (int is = 0; is < c.nspec; is++) {
    int64_t n = ncell * pl->ppc[is];
    if (pl->ppc[is] < 0 || n > ctx->seg.capacity[is])
      return set_error(ctx, EMSESG_ERR_OVERFLOW, "species %d: %lld particles exceed capacity", is + 1, (long long)n);
  }
  for (int is = 0; is < c.nspec; is++) {
    int64_t n = ncell * pl->ppc[is];
    ctx->totalp[is] = n;
    if (n == 0) continue;
    int rc = plasma_records(ctx, ctx->pbuf + ctx->seg.base[is], is, 0, n, pl);
    if (rc) return rc;
  }
  EMSESG_CUDA(ctx, cudaMemcpyAsync(ctx->d_count, ctx->totalp, EMSESG_ISPEC * sizeof(int64_t), cudaMemcpyHostToDevice,
                                   ctx->stream));
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->fx.loaded = false;
  return EMSESG_OK;
}
