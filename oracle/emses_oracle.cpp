// emses_oracle.cpp -- TEST INFRASTRUCTURE ONLY (see emses_oracle.h).
//
// CPU FP64 restatement of the EMSES particle hot path for one rank
// (sdid(1) = 0, sdoms = [0, n] on every axis, so dxl = 0 and dxu = slx = n).
// Each function cites the Fortran it follows.  Build flags keep IEEE FP64
// without contraction: -O2 -ffp-contract=off -fno-fast-math.
#include "emses_oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>
#include <thread>

namespace {

// Fortran array descriptor: (nc, lo:n+hi) on every axis, component fastest.
struct FD {
  int nc, lo, ex, ey, ez;
  int64_t at(int c, int i, int j, int k) const {
    return c + (int64_t)nc * ((i - lo) + (int64_t)ex * ((j - lo) + (int64_t)ey * (k - lo)));
  }
  int64_t size() const { return (int64_t)nc * ex * ey * ez; }
};

// Guard extents from OhHelp's fsizes rule (ohhelp3.c:439-477) applied to the
// ftypes/ctypes of src/wrapper/ohinit.F90:98-122:
//   FEB: -1..n+1, FAJ (aj, wrk, ajdg): -4..n+4, FRH/FRD: -1..n+1.
FD fd_of(const emsesg_config* c, int field) {
  int nx = c->nx, ny = c->ny, nz = c->nz;
  switch (field) {
    case EMSESG_FIELD_EB: return {6, -1, nx + 3, ny + 3, nz + 3};
    case EMSESG_FIELD_WRK: return {9, -4, nx + 9, ny + 9, nz + 9};
    case EMSESG_FIELD_AJ: return {3, -4, nx + 9, ny + 9, nz + 9};
    case EMSESG_FIELD_AJDG: return {3 * c->nspec, -4, nx + 9, ny + 9, nz + 9};
    case EMSESG_FIELD_RHO: return {1, -1, nx + 3, ny + 3, nz + 3};
    case EMSESG_FIELD_RHODG: return {2 * c->nspec + 1, -1, nx + 3, ny + 3, nz + 3};
    case EMSESG_FIELD_RHOBK: return {1, -1, nx + 3, ny + 3, nz + 3};
    case EMSESG_FIELD_RHOBKSP: return {1, -1, nx + 3, ny + 3, nz + 3};
  }
  return {0, 0, 0, 0, 0};
}

// Component indices, src/main/paramt.F90:46-48 (0-based here).
enum { EX = 0, EY, EZ, BX, BY, BZ, TJX, TJY, TJZ };
enum { JX = 0, JY, JZ };

// SplitMix64 finaliser (Steele, Lea, Flood 2014): the counter hash of the
// project.  Used for injected-particle fractions and the synthetic loader.
inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// Single-rank nborps (src/etc/nborps.F90:29-…): with nodes = (1,1,1) every
// neighbour is the rank itself (sdid = 0) when the crossed axes are periodic
// or reflecting, and -1 as soon as one crossed axis has another npbnd.
inline int nborps_single(const emsesg_config* c, int is, bool cx, bool cy, bool cz) {
  const int32_t* nb = c->npbnd[is];
  if (cx && !(nb[0] == 0 || nb[0] == 1)) return -1;
  if (cy && !(nb[1] == 0 || nb[1] == 1)) return -1;
  if (cz && !(nb[2] == 0 || nb[2] == 1)) return -1;
  return 0;
}

struct RandSource {
  const emsesg_config* c;
  const double* ranu;
  int64_t nranu;
  int64_t* pos;
  uint64_t stream;
  bool ok = true;
  double draw(int64_t m) {
    if (c->rng_mode == 1) {
      if (*pos >= nranu) { ok = false; return 0.0; }
      return ranu[(*pos)++];
    }
    return orc_hash_u01(c->rng_seed, stream, (uint64_t)m);
  }
};

// Body test, internal boundary treatment 1 of psolve2.F90:465-531.  Returns
// true when the particle was absorbed (nid set to -1, counters updated).
void body_test_psolve2(const emsesg_config* c, int is, emsesg_particle& p,
                       const double* radsq, emsesg_counter* gc) {
  if (c->line_mode == 1) return;
  for (int ipc = 0; ipc < c->npc; ipc++) {
    if (p.nid == -1) continue;
    const emsesg_body& b = c->body[ipc];
    bool kill = false;
    if ((b.geotype == 0 || b.geotype == 1) &&
        (p.x >= b.xlpc && p.x <= b.xupc && p.y >= b.ylpc && p.y <= b.yupc &&
         p.z >= b.zlpc && p.z <= b.zupc)) {
      kill = true;
    } else if (b.geotype == 2) {
      double d1, d2, a;
      if (b.cyl_align == 1) { d1 = p.y - b.cyl_axis[0]; d2 = p.z - b.cyl_axis[1]; a = p.x; }
      else if (b.cyl_align == 2) { d1 = p.z - b.cyl_axis[0]; d2 = p.x - b.cyl_axis[1]; a = p.y; }
      else if (b.cyl_align == 3) { d1 = p.x - b.cyl_axis[0]; d2 = p.y - b.cyl_axis[1]; a = p.z; }
      else continue;
      if (a >= b.cyl_edge[0] && a <= b.cyl_edge[1] && d1 * d1 + d2 * d2 < radsq[ipc]) kill = true;
    } else if (b.geotype == 3) {
      double d1 = p.x - b.sph_center[0], d2 = p.y - b.sph_center[1], d3 = p.z - b.sph_center[2];
      if (d1 * d1 + d2 * d2 + d3 * d3 < radsq[ipc]) kill = true;
    }
    if (kill) {
      p.nid = -1;
      gc->influx[is][ipc] += 1;
      if (p.pid >= 0 && p.pid <= EMSESG_INPC) gc->infhist[is][ipc][p.pid] += 1;
    }
  }
}

// chgacm update after the species loop, psolve2.F90:537-543 / psolve1.F90:821-828.
void chgacm_update(const emsesg_config* c, emsesg_counter* gc) {
  for (int is = 0; is < c->nspec; is++)
    for (int ipc = 0; ipc < c->npc; ipc++)
      if (c->body[ipc].ncond > 0) {
        double add = (double)gc->influx[is][ipc] * c->q[is] * c->body[ipc].sqdscaled;
        gc->chgacm[ipc][0] = gc->chgacm[ipc][0] + add;
        gc->chgacm[ipc][1] = gc->chgacm[ipc][1] + add;
      }
}

void radsq_of(const emsesg_config* c, double* radsq) {
  for (int ipc = 0; ipc < c->npc; ipc++) {
    radsq[ipc] = 0.0;
    if (c->body[ipc].geotype == 2 || c->body[ipc].geotype == 3)
      radsq[ipc] = c->body[ipc].radius * c->body[ipc].radius;
  }
}

// Per-surface-cell absorbed-charge counts of the box bodies (a rule of this
// project; the reference's own per-cell absorbed charge comes from its
// finbound route only).  Bodies with geotype 0/1 and integer bounds have six
// faces -x,+x,-y,+y,-z,+z; a face's cells are numbered with its first
// tangential axis fastest (x faces: y then z; y faces: x then z; z faces:
// x then y).  A particle entering the box between its start point b and its
// end point a is counted on the face it crossed last (largest entry time
// along the segment; ties take the lower axis), in the cell that holds a's
// tangential coordinates.
bool box_surface(const emsesg_body& b) {
  if (!(b.geotype == 0 || b.geotype == 1)) return false;
  const double v[6] = {b.xlpc, b.xupc, b.ylpc, b.yupc, b.zlpc, b.zupc};
  for (int q = 0; q < 6; q++)
    if (v[q] != std::floor(v[q])) return false;
  return b.xupc > b.xlpc && b.yupc > b.ylpc && b.zupc > b.zlpc;
}

void body_bounds(const emsesg_body& b, int lo[3], int hi[3]) {
  lo[0] = (int)b.xlpc; hi[0] = (int)b.xupc;
  lo[1] = (int)b.ylpc; hi[1] = (int)b.yupc;
  lo[2] = (int)b.zlpc; hi[2] = (int)b.zupc;
}

const int TAN1[3] = {1, 0, 0}, TAN2[3] = {2, 2, 1};

int64_t face_cells(const int lo[3], const int hi[3], int d) {
  return (int64_t)(hi[TAN1[d]] - lo[TAN1[d]]) * (hi[TAN2[d]] - lo[TAN2[d]]);
}

int64_t face_index(const int lo[3], const int hi[3], int d, const double a[3]) {
  const int e1 = TAN1[d], e2 = TAN2[d];
  int u = (int)std::floor(a[e1]), v = (int)std::floor(a[e2]);
  u = std::min(std::max(u, lo[e1]), hi[e1] - 1) - lo[e1];
  v = std::min(std::max(v, lo[e2]), hi[e2] - 1) - lo[e2];
  return u + (int64_t)(hi[e1] - lo[e1]) * v;
}

}  // namespace

extern "C" int64_t orc_surface_layout(const emsesg_config* c, int64_t* offsets) {
  int64_t n = 0;
  for (int ipc = 0; ipc < c->npc; ipc++) {
    const emsesg_body& b = c->body[ipc];
    bool on = box_surface(b);
    int lo[3], hi[3];
    if (on) body_bounds(b, lo, hi);
    for (int f = 0; f < 6; f++) {
      if (offsets) offsets[ipc * 6 + f] = n;
      if (on) n += face_cells(lo, hi, f / 2);
    }
  }
  return n;
}

extern "C" int64_t orc_surface_cell(const emsesg_config* c, int ipc, const double* bp, const double* ap) {
  const emsesg_body& b = c->body[ipc];
  if (!box_surface(b)) return -1;
  int lo[3], hi[3];
  body_bounds(b, lo, hi);
  int64_t off[6 * EMSESG_INPC];
  orc_surface_layout(c, off);
  int best = -1, side = 0;
  double tb = -1.0;
  for (int d = 0; d < 3; d++) {
    double t = -1.0;
    int sd = 0;
    if (bp[d] < lo[d]) { t = (lo[d] - bp[d]) / (ap[d] - bp[d]); sd = 0; }
    else if (bp[d] > hi[d]) { t = (hi[d] - bp[d]) / (ap[d] - bp[d]); sd = 1; }
    if (t > tb) { tb = t; best = d; side = sd; }
  }
  if (best < 0) {  // start point inside: the nearest face of the end point
    double dm = 1e300;
    for (int d = 0; d < 3; d++) {
      if (ap[d] - lo[d] < dm) { dm = ap[d] - lo[d]; best = d; side = 0; }
      if (hi[d] - ap[d] < dm) { dm = hi[d] - ap[d]; best = d; side = 1; }
    }
  }
  return off[ipc * 6 + 2 * best + side] + face_index(lo, hi, best, ap);
}

// Background charge of the box bodies from the per-surface-cell counts
// surf[nspec][nsurf] (absorbed minus emitted particles): the node field
// rhobk(...,3) with a surface cell's charge q(is) * count in equal quarters
// on the four nodes of its face cell (the counts meeting at a node summed as
// integers per species, then scaled), species by species and body by body;
// then add_background_charge, charge.F90:440-448: rho(0:n) += rhobk, or
// rho(0:n) = rhobk with `replace` (nflag_testp == 1).  rhobk and rho have the
// rho layout.  The counts-to-nodes rule is the project's: the reference
// deposits absorbed charge into rhobk only along the finbound route.
extern "C" void orc_background(const emsesg_config* c, const int64_t* surf, double* rhobk, double* rho,
                               int replace) {
  const FD fr = fd_of(c, EMSESG_FIELD_RHO);
  for (int64_t x = 0; x < fr.size(); x++) rhobk[x] = 0.0;
  int64_t off[6 * EMSESG_INPC];
  const int64_t nsurf = orc_surface_layout(c, off);
  for (int is = 0; is < c->nspec; is++)
    for (int ipc = 0; ipc < c->npc; ipc++) {
      const emsesg_body& b = c->body[ipc];
      if (!box_surface(b)) continue;
      int lo[3], hi[3];
      body_bounds(b, lo, hi);
      for (int k = lo[2]; k <= hi[2]; k++)
        for (int j = lo[1]; j <= hi[1]; j++)
          for (int i = lo[0]; i <= hi[0]; i++) {
            const int nd[3] = {i, j, k};
            int64_t sum = 0;
            for (int f = 0; f < 6; f++) {
              const int d = f / 2, e1 = TAN1[d], e2 = TAN2[d];
              if (nd[d] != ((f & 1) ? hi[d] : lo[d])) continue;
              const int ext1 = hi[e1] - lo[e1], ext2 = hi[e2] - lo[e2];
              const int a = nd[e1] - lo[e1], bb = nd[e2] - lo[e2];
              for (int v = bb - 1; v <= bb; v++)
                for (int u = a - 1; u <= a; u++)
                  if (u >= 0 && v >= 0 && u < ext1 && v < ext2)
                    sum += surf[is * nsurf + off[ipc * 6 + f] + u + (int64_t)ext1 * v];
            }
            if (sum != 0) {
              const int64_t x = fr.at(0, i, j, k);
              rhobk[x] = rhobk[x] + c->q[is] * 0.25 * (double)sum;
            }
          }
    }
  for (int k = 0; k <= c->nz; k++)
    for (int j = 0; j <= c->ny; j++)
      for (int i = 0; i <= c->nx; i++) {
        const int64_t x = fr.at(0, i, j, k);
        rho[x] = replace ? rhobk[x] : rho[x] + rhobk[x];
      }
}

// Face cell of a point lying on a box face (an emitted particle's
// anti-particle), or -1.
extern "C" int64_t orc_surface_point(const emsesg_config* c, int ipc, const double* p) {
  const emsesg_body& b = c->body[ipc];
  if (!box_surface(b)) return -1;
  int lo[3], hi[3];
  body_bounds(b, lo, hi);
  int64_t off[6 * EMSESG_INPC];
  orc_surface_layout(c, off);
  for (int d = 0; d < 3; d++) {
    const int e1 = TAN1[d], e2 = TAN2[d];
    if (p[e1] < lo[e1] || p[e1] > hi[e1] || p[e2] < lo[e2] || p[e2] > hi[e2]) continue;
    if (p[d] == (double)lo[d]) return off[ipc * 6 + 2 * d] + face_index(lo, hi, d, p);
    if (p[d] == (double)hi[d]) return off[ipc * 6 + 2 * d + 1] + face_index(lo, hi, d, p);
  }
  return -1;
}

namespace {

// Trilinear weights v1..v8 (psolve2.F90:166-183, charge.F90:173-192).
struct W8 { double v1, v2, v3, v4, v5, v6, v7, v8; };
inline W8 weights(double x1, double y1, double z1) {
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

// Gather + Boris + move, psolve2.F90:185-318 (identical in psolve1.F90:201-333
// apart from the cell index).  Updates p.v*, p.x/y/z.
inline void gather_boris_move(const FD& fw, const double* wrk, emsesg_particle& p,
                              int i, int j, int k, const W8& w, double qmp,
                              double gustep) {
  int i1 = i + 1, j1 = j + 1, k1 = k + 1;
  double e[3][8];
  for (int d = 0; d < 3; d++) {
    e[d][0] = wrk[fw.at(EX + d, i, j, k1)];
    e[d][1] = wrk[fw.at(EX + d, i1, j, k1)];
    e[d][2] = wrk[fw.at(EX + d, i1, j1, k1)];
    e[d][3] = wrk[fw.at(EX + d, i, j1, k1)];
    e[d][4] = wrk[fw.at(EX + d, i, j, k)];
    e[d][5] = wrk[fw.at(EX + d, i1, j, k)];
    e[d][6] = wrk[fw.at(EX + d, i1, j1, k)];
    e[d][7] = wrk[fw.at(EX + d, i, j1, k)];
  }
  double eex = e[0][0] * w.v1 + e[0][1] * w.v2 + e[0][2] * w.v3 + e[0][3] * w.v4 +
               e[0][4] * w.v5 + e[0][5] * w.v6 + e[0][6] * w.v7 + e[0][7] * w.v8;
  double eey = e[1][0] * w.v1 + e[1][1] * w.v2 + e[1][2] * w.v3 + e[1][3] * w.v4 +
               e[1][4] * w.v5 + e[1][5] * w.v6 + e[1][6] * w.v7 + e[1][7] * w.v8;
  double eez = e[2][0] * w.v1 + e[2][1] * w.v2 + e[2][2] * w.v3 + e[2][3] * w.v4 +
               e[2][4] * w.v5 + e[2][5] * w.v6 + e[2][6] * w.v7 + e[2][7] * w.v8;
  double b[3];
  for (int d = 0; d < 3; d++) {
    int cc = BX + d;
    b[d] = wrk[fw.at(cc, i, j, k1)] * w.v1 + wrk[fw.at(cc, i1, j, k1)] * w.v2 +
           wrk[fw.at(cc, i1, j1, k1)] * w.v3 + wrk[fw.at(cc, i, j1, k1)] * w.v4 +
           wrk[fw.at(cc, i, j, k)] * w.v5 + wrk[fw.at(cc, i1, j, k)] * w.v6 +
           wrk[fw.at(cc, i1, j1, k)] * w.v7 + wrk[fw.at(cc, i, j1, k)] * w.v8;
  }
  const double ewx = 0.0, ewy = 0.0;  // ewmodel off (psolve2.F90:119-126)
  eex = (eex + ewx) * qmp;
  eey = (eey + ewy) * qmp;
  eez = eez * qmp;
  double bbx = b[0] * qmp, bby = b[1] * qmp, bbz = b[2] * qmp;
  // Buneman-Boris, psolve2.F90:241-257.
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
  // Position update, psolve2.F90:313-318.
  double xmove = p.vx * gustep, ymove = p.vy * gustep, zmove = p.vz * gustep;
  p.x = p.x + xmove;
  p.y = p.y + ymove;
  p.z = p.z + zmove;
}

// Exchange of one axis for a single periodic rank: OhHelp border exchange
// sends [from_L, from_L+size_L) to the receiver's [n+to_L, ...) and
// [n+from_U, n+from_U+size_U) to [to_U, ...)  (set_border_comm,
// ohhelp3.c:570-697); on one rank the neighbour is the rank itself.
struct CT { int fromL, toL, sizeL, fromU, toU, sizeU; };
// ctypes of ohinit.F90:111-122 as (from,to,size) for the lower and upper sends.
const CT CT_EB = {0, 0, 2, -1, -1, 1};
const CT CT_AJ = {-1, 2, 3, -1, -4, 3};
const CT CT_RH = {0, 1, 1, 0, -1, 1};

void exchange_single(const emsesg_config* c, const FD& f, double* a, const CT& ct) {
  int n[3] = {c->nx, c->ny, c->nz};
  // exti = [from_L, n+from_U+size_U-1], exto = [to_U, n+to_L+size_L-1]
  int tlo[3], thi[3], olo[3], ohi[3];
  for (int d = 0; d < 3; d++) {
    tlo[d] = ct.fromL; thi[d] = n[d] + ct.fromU + ct.sizeU - 1;
    olo[d] = ct.toU;   ohi[d] = n[d] + ct.toL + ct.sizeL - 1;
  }
  for (int d = 0; d < 3; d++) {
    if (c->nfbnd[d] != 0) continue;  // non-periodic: MPI_PROC_NULL, no copy
    // ranges of the other two axes: x-exchange uses exti for y,z; y uses exto
    // for x and exti for z; z uses exto for x,y.
    int lo[3], hi[3];
    for (int e = 0; e < 3; e++) {
      if (e == d) continue;
      bool outer = e < d;
      lo[e] = outer ? olo[e] : tlo[e];
      hi[e] = outer ? ohi[e] : thi[e];
    }
    for (int lu = 0; lu < 2; lu++) {
      int src0 = lu == 0 ? ct.fromL : n[d] + ct.fromU;
      int dst0 = lu == 0 ? n[d] + ct.toL : ct.toU;
      int sz = lu == 0 ? ct.sizeL : ct.sizeU;
      for (int s = 0; s < sz; s++) {
        int is = src0 + s, id = dst0 + s;
        int a0 = d == 0 ? 0 : lo[0], a1 = d == 0 ? 0 : hi[0];
        int b0 = d == 1 ? 0 : lo[1], b1 = d == 1 ? 0 : hi[1];
        int c0 = d == 2 ? 0 : lo[2], c1 = d == 2 ? 0 : hi[2];
        for (int k = c0; k <= c1; k++)
          for (int j = b0; j <= b1; j++)
            for (int i = a0; i <= a1; i++) {
              int si[3] = {i, j, k}, di[3] = {i, j, k};
              si[d] = is; di[d] = id;
              for (int cc = 0; cc < f.nc; cc++)
                a[f.at(cc, di[0], di[1], di[2])] = a[f.at(cc, si[0], si[1], si[2])];
            }
      }
    }
  }
}

}  // namespace

extern "C" {

int64_t orc_field_size(const emsesg_config* c, int field) {
  FD f = fd_of(c, field);
  if (field == EMSESG_FIELD_RHOBKSP) return f.size() * c->nspec;
  return f.size();
}

double orc_hash_u01(uint64_t seed, uint64_t stream, uint64_t index) {
  uint64_t a = mix64(seed ^ mix64(stream + 0x632BE59BD9B4E019ULL));
  uint64_t b = mix64(a ^ (index * 0xD1B54A32D192ED03ULL));
  return (double)(b >> 11) * (1.0 / 9007199254740992.0);
}

void orc_exchange_eb(const emsesg_config* c, double* eb) {
  exchange_single(c, fd_of(c, EMSESG_FIELD_EB), eb, CT_EB);
}

// bfield, src/field/bfield.F90:37-53 (statement order of the reference;
// the loop writes B only and reads E only).
void orc_bfield(const emsesg_config* c, double* eb) {
  FD f = fd_of(c, EMSESG_FIELD_EB);
  for (int k = -1; k <= c->nz; k++)
    for (int j = -1; j <= c->ny; j++)
      for (int i = -1; i <= c->nx; i++) {
        eb[f.at(BX, i, j, k)] = eb[f.at(BX, i, j, k)] + eb[f.at(EY, i, j, k + 1)] - eb[f.at(EY, i, j, k)] -
                                eb[f.at(EZ, i, j + 1, k)] + eb[f.at(EZ, i, j, k)];
        eb[f.at(BY, i, j, k)] = eb[f.at(BY, i, j, k)] + eb[f.at(EZ, i + 1, j, k)] - eb[f.at(EZ, i, j, k)] -
                                eb[f.at(EX, i, j, k + 1)] + eb[f.at(EX, i, j, k)];
        eb[f.at(BZ, i, j, k)] = eb[f.at(BZ, i, j, k)] + eb[f.at(EX, i, j + 1, k)] - eb[f.at(EX, i, j, k)] -
                                eb[f.at(EY, i + 1, j, k)] + eb[f.at(EY, i, j, k)];
      }
}

// efield, src/field/efield.F90:54-70 (mode_dipole != 3: no lumped
// elements; the loop writes E only and reads B and J).
void orc_efield(const emsesg_config* c, double* eb, const double* aj, double tcs, double dlt) {
  FD f = fd_of(c, EMSESG_FIELD_EB), fa = fd_of(c, EMSESG_FIELD_AJ);
  for (int k = 0; k <= c->nz; k++)
    for (int j = 0; j <= c->ny; j++)
      for (int i = 0; i <= c->nx; i++) {
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
}

// grdcrt main relocations, src/field/grdcrt.F90:156-169 (E) and :214-230 (B).
// The hole (zurechole) and sfecrrct surface corrections are not part of the
// path (off in every configuration).
void orc_grdcrt(const emsesg_config* c, const double* eb, double* wrk) {
  FD fe = fd_of(c, EMSESG_FIELD_EB), fw = fd_of(c, EMSESG_FIELD_WRK);
  for (int k = 0; k <= c->nz; k++)
    for (int j = 0; j <= c->ny; j++)
      for (int i = 0; i <= c->nx; i++) {
        wrk[fw.at(EX, i, j, k)] = 0.5 * (eb[fe.at(EX, i, j, k)] + eb[fe.at(EX, i - 1, j, k)]) + c->e0[0];
        wrk[fw.at(EY, i, j, k)] = 0.5 * (eb[fe.at(EY, i, j, k)] + eb[fe.at(EY, i, j - 1, k)]) + c->e0[1];
        wrk[fw.at(EZ, i, j, k)] = 0.5 * (eb[fe.at(EZ, i, j, k)] + eb[fe.at(EZ, i, j, k - 1)]) + c->e0[2];
      }
  for (int k = 0; k <= c->nz; k++)
    for (int j = 0; j <= c->ny; j++)
      for (int i = 0; i <= c->nx; i++) {
        wrk[fw.at(BX, i, j, k)] = 0.25 * (eb[fe.at(BX, i, j, k)] + eb[fe.at(BX, i, j - 1, k)] +
                                          eb[fe.at(BX, i, j, k - 1)] + eb[fe.at(BX, i, j - 1, k - 1)]) + c->b0[0];
        wrk[fw.at(BY, i, j, k)] = 0.25 * (eb[fe.at(BY, i, j, k)] + eb[fe.at(BY, i - 1, j, k)] +
                                          eb[fe.at(BY, i, j, k - 1)] + eb[fe.at(BY, i - 1, j, k - 1)]) + c->b0[1];
        wrk[fw.at(BZ, i, j, k)] = 0.25 * (eb[fe.at(BZ, i, j, k)] + eb[fe.at(BZ, i - 1, j, k)] +
                                          eb[fe.at(BZ, i, j - 1, k)] + eb[fe.at(BZ, i - 1, j - 1, k)]) + c->b0[2];
      }
}

// psolve2, src/pcl2field/psolve2.F90:101-544 (single rank, no collisions,
// no test charges, no wave field, empty finbound boundary list).
int orc_psolve2(const emsesg_config* c, int ustep, const double* wrk,
                emsesg_particle* pbuf, const int64_t* totalp, const double* ranu,
                int64_t nranu, int64_t* ranu_pos, uint64_t rng_stream,
                emsesg_counter* gc) {
  FD fw = fd_of(c, EMSESG_FIELD_WRK);
  double radsq[EMSESG_INPC];
  radsq_of(c, radsq);
  const double dxl = 0.0, dyl = 0.0, dzl = 0.0;
  const double dxu = c->nx, dyu = c->ny, dzu = c->nz;
  const double slx = c->nx, sly = c->ny, slz = c->nz;
  const double tslx = 2.0 * slx, tsly = 2.0 * sly, tslz = 2.0 * slz;
  RandSource rs{c, ranu, nranu, ranu_pos, rng_stream};
  int64_t nee = 0;
  for (int is = 0; is < c->nspec; is++) {
    int64_t ns = nee, ne = nee + totalp[is];
    nee = ne;
    for (int64_t m = ns; m < ne; m++) {
      emsesg_particle& p = pbuf[m];
      double gustep = 0.0, qmp = 0.0;
      if (p.preside < 0) {
        p.nid = -1;
        p.preside = 0;
      } else if (p.preside == EMSESG_PCL_INJECTED) {
        double u = rs.draw(m);
        gustep = (double)ustep * u;
        qmp = c->qm[is] * gustep * 0.5;
        p.preside = 0;
      } else {
        gustep = (double)ustep;
        qmp = c->qm[is] * gustep * 0.5;
      }
      if (p.nid == -1) continue;

      double xlocal = p.x - dxl, ylocal = p.y - dyl, zlocal = p.z - dzl;
      int i = (int)xlocal, j = (int)ylocal, k = (int)zlocal;  // int(): truncation
      double x1 = xlocal - i, y1 = ylocal - j, z1 = zlocal - k;
      W8 w = weights(x1, y1, z1);
      gather_boris_move(fw, wrk, p, i, j, k, w, qmp, gustep);

      // External boundary treatment, psolve2.F90:352-432.
      int nud = 14;
      if (p.x < dxl) nud -= 1; else if (p.x >= dxu) nud += 1;
      if (p.y < dyl) nud -= 3; else if (p.y >= dyu) nud += 3;
      if (p.z < dzl) nud -= 9; else if (p.z >= dzu) nud += 9;
      if (nud != 14) {
        bool cx = p.x < dxl || p.x >= dxu, cy = p.y < dyl || p.y >= dyu, cz = p.z < dzl || p.z >= dzu;
        p.nid = nborps_single(c, is, cx, cy, cz);
        const int32_t* nb = c->npbnd[is];
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
        if (p.nid == -1) gc->nesc[is] += 1;
      }
      body_test_psolve2(c, is, p, radsq, gc);
    }
  }
  chgacm_update(c, gc);
  return rs.ok ? 0 : EMSESG_ERR_ARG;
}

// positn, src/pcl/positn.F90:50-355: the position-only advance of the
// initial state.  x += v*ustep for every live particle (injected ones still
// draw their random number, :97-101, but move by ustep, :109-114); the outer
// boundary counts nesc once per escaping axis (:228-268); the body test takes
// the box bounds xlpc..zupc as the cylinder's axial extent (:283-316); there
// is no chgacm update.
int orc_positn(const emsesg_config* c, int ustep, emsesg_particle* pbuf, const int64_t* totalp,
               const double* ranu, int64_t nranu, int64_t* ranu_pos, uint64_t rng_stream, emsesg_counter* gc) {
  double radsq[EMSESG_INPC];
  radsq_of(c, radsq);
  const double dxl = 0.0, dyl = 0.0, dzl = 0.0;
  const double dxu = c->nx, dyu = c->ny, dzu = c->nz;
  const double slx = c->nx, sly = c->ny, slz = c->nz;
  const double tslx = 2.0 * slx, tsly = 2.0 * sly, tslz = 2.0 * slz;
  RandSource rs{c, ranu, nranu, ranu_pos, rng_stream};
  int64_t nee = 0;
  for (int is = 0; is < c->nspec; is++) {
    int64_t ns = nee, ne = nee + totalp[is];
    nee = ne;
    for (int64_t m = ns; m < ne; m++) {
      emsesg_particle& p = pbuf[m];
      if (p.preside < 0) {
        p.nid = -1;
        p.preside = 0;
      } else if (p.preside == EMSESG_PCL_INJECTED) {
        (void)rs.draw(m);
        p.preside = 0;
      }
      if (p.nid == -1) continue;
      double xmove = p.vx * ustep, ymove = p.vy * ustep, zmove = p.vz * ustep;
      p.x = p.x + xmove;
      p.y = p.y + ymove;
      p.z = p.z + zmove;
      int nud = 14;
      if (p.x < dxl) nud -= 1; else if (p.x >= dxu) nud += 1;
      if (p.y < dyl) nud -= 3; else if (p.y >= dyu) nud += 3;
      if (p.z < dzl) nud -= 9; else if (p.z >= dzu) nud += 9;
      if (nud != 14) {
        bool cx = p.x < dxl || p.x >= dxu, cy = p.y < dyl || p.y >= dyu, cz = p.z < dzl || p.z >= dzu;
        p.nid = nborps_single(c, is, cx, cy, cz);
        const int32_t* nb = c->npbnd[is];
        if (p.x < 0.0) {
          if (nb[0] == 0) p.x = p.x + slx;
          else if (nb[0] == 1) { p.x = -p.x; p.vx = -p.vx; }
          else gc->nesc[is] += 1;
        } else if (p.x >= slx) {
          if (nb[0] == 0) p.x = p.x - slx;
          else if (nb[0] == 1) { p.x = tslx - p.x; p.vx = -p.vx; }
          else gc->nesc[is] += 1;
        }
        if (p.y < 0.0) {
          if (nb[1] == 0) p.y = p.y + sly;
          else if (nb[1] == 1) { p.y = -p.y; p.vy = -p.vy; }
          else gc->nesc[is] += 1;
        } else if (p.y >= sly) {
          if (nb[1] == 0) p.y = p.y - sly;
          else if (nb[1] == 1) { p.y = tsly - p.y; p.vy = -p.vy; }
          else gc->nesc[is] += 1;
        }
        if (p.z < 0.0) {
          if (nb[2] == 0) p.z = p.z + slz;
          else if (nb[2] == 1) { p.z = -p.z; p.vz = -p.vz; }
          else gc->nesc[is] += 1;
        } else if (p.z >= slz) {
          if (nb[2] == 0) p.z = p.z - slz;
          else if (nb[2] == 1) { p.z = tslz - p.z; p.vz = -p.vz; }
          else gc->nesc[is] += 1;
        }
      }
      if (c->line_mode == 1) continue;
      for (int ipc = 0; ipc < c->npc; ipc++) {
        if (p.nid == -1) continue;
        const emsesg_body& b = c->body[ipc];
        bool kill = false;
        if ((b.geotype == 0 || b.geotype == 1) &&
            (p.x >= b.xlpc && p.x <= b.xupc && p.y >= b.ylpc && p.y <= b.yupc && p.z >= b.zlpc && p.z <= b.zupc)) {
          kill = true;
        } else if (b.geotype == 2) {
          double d1, d2, a, lo, hi;
          if (b.cyl_align == 1) { d1 = p.y - b.cyl_axis[0]; d2 = p.z - b.cyl_axis[1]; a = p.x; lo = b.xlpc; hi = b.xupc; }
          else if (b.cyl_align == 2) { d1 = p.z - b.cyl_axis[0]; d2 = p.x - b.cyl_axis[1]; a = p.y; lo = b.ylpc; hi = b.yupc; }
          else if (b.cyl_align == 3) { d1 = p.x - b.cyl_axis[0]; d2 = p.y - b.cyl_axis[1]; a = p.z; lo = b.zlpc; hi = b.zupc; }
          else continue;
          if (a >= lo && a <= hi && d1 * d1 + d2 * d2 < radsq[ipc]) kill = true;
        } else if (b.geotype == 3) {
          double d1 = p.x - b.sph_center[0], d2 = p.y - b.sph_center[1], d3 = p.z - b.sph_center[2];
          if (d1 * d1 + d2 * d2 + d3 * d3 < radsq[ipc]) kill = true;
        }
        if (kill) {
          p.nid = -1;
          gc->influx[is][ipc] += 1;
          if (p.pid >= 0 && p.pid <= EMSESG_INPC) gc->infhist[is][ipc][p.pid] += 1;
        }
      }
    }
  }
  return rs.ok ? 0 : EMSESG_ERR_ARG;
}

// psolve1, src/pcl2field/psolve1.F90:85-828: the push of psolve2 with floor()
// cell indices and the zigzag current (Umeda 2003) into wrk(TJX:TJZ), flushed
// into aj (and ajdg when func == 1) with q(is) per species.
int orc_psolve1(const emsesg_config* c, int ustep, int func, double* wrk,
                emsesg_particle* pbuf, const int64_t* totalp, const double* ranu,
                int64_t nranu, int64_t* ranu_pos, uint64_t rng_stream,
                double* aj, double* ajdg, emsesg_counter* gc, int64_t* surf) {
  const int64_t nsurf = orc_surface_layout(c, nullptr);
  FD fw = fd_of(c, EMSESG_FIELD_WRK), fa = fd_of(c, EMSESG_FIELD_AJ), fj = fd_of(c, EMSESG_FIELD_AJDG);
  double radsq[EMSESG_INPC];
  radsq_of(c, radsq);
  const double dxl = 0.0, dyl = 0.0, dzl = 0.0;
  const double dxu = c->nx, dyu = c->ny, dzu = c->nz;
  const double slx = c->nx, sly = c->ny, slz = c->nz;
  const double tslx = 2.0 * slx, tsly = 2.0 * sly, tslz = 2.0 * slz;
  const int ngx = c->nx, ngy = c->ny, ngz = c->nz;
  const double dngx = ngx, dngy = ngy, dngz = ngz;
  double xlc[EMSESG_INPC], ylc[EMSESG_INPC], zlc[EMSESG_INPC];
  double xuc[EMSESG_INPC], yuc[EMSESG_INPC], zuc[EMSESG_INPC];
  for (int ipc = 0; ipc < c->npc; ipc++) {  // psolve1.F90:86-90
    xlc[ipc] = c->body[ipc].xlpc - dxl; xuc[ipc] = c->body[ipc].xupc - dxl;
    ylc[ipc] = c->body[ipc].ylpc - dyl; yuc[ipc] = c->body[ipc].yupc - dyl;
    zlc[ipc] = c->body[ipc].zlpc - dzl; zuc[ipc] = c->body[ipc].zupc - dzl;
  }
  const double rustep = 1.0 / ustep;
  RandSource rs{c, ranu, nranu, ranu_pos, rng_stream};
  int64_t nee = 0;
  for (int is = 0; is < c->nspec; is++) {
    int64_t ns = nee, ne = nee + totalp[is];
    nee = ne;
    // wrk(TJX:TJZ, :, :, :) = 0 (psolve1.F90:143)
    for (int k = fw.lo; k < fw.lo + fw.ez; k++)
      for (int j = fw.lo; j < fw.lo + fw.ey; j++)
        for (int i = fw.lo; i < fw.lo + fw.ex; i++)
          for (int cc = TJX; cc <= TJZ; cc++) wrk[fw.at(cc, i, j, k)] = 0.0;
    for (int64_t m = ns; m < ne; m++) {
      emsesg_particle& p = pbuf[m];
      double gustep = 0.0, qmp = 0.0;
      if (p.preside < 0) {
        p.nid = -1;
        p.preside = 0;
      } else if (p.preside == EMSESG_PCL_INJECTED) {
        double u = rs.draw(m);
        gustep = (double)ustep * u;
        qmp = c->qm[is] * gustep * 0.5;
        p.preside = 0;
      } else {
        gustep = (double)ustep;
        qmp = c->qm[is] * gustep * 0.5;
      }
      if (p.nid == -1) continue;

      double xlocalb = p.x - dxl, ylocalb = p.y - dyl, zlocalb = p.z - dzl;
      const double xlocalb0 = xlocalb, ylocalb0 = ylocalb, zlocalb0 = zlocalb;
      int ib = (int)std::floor(xlocalb), jb = (int)std::floor(ylocalb), kb = (int)std::floor(zlocalb);
      double xb = ib, yb = jb, zb = kb;
      int i1b = ib + 1, j1b = jb + 1, k1b = kb + 1;
      double x1 = xlocalb - xb, y1 = ylocalb - yb, z1 = zlocalb - zb;
      W8 w = weights(x1, y1, z1);
      gather_boris_move(fw, wrk, p, ib, jb, kb, w, qmp, gustep);

      double xlocala, ylocala, zlocala, xa, ya, za, xr, yr, zr;
      int ia, ja, ka, i1a, j1a, k1a;
      int nud = 14;
      if (p.x < dxl) nud -= 1; else if (p.x >= dxu) nud += 1;
      if (p.y < dyl) nud -= 3; else if (p.y >= dyu) nud += 3;
      if (p.z < dzl) nud -= 9; else if (p.z >= dzu) nud += 9;
      if (nud == 14) {  // psolve1.F90:382-415
        xlocala = p.x - dxl; ylocala = p.y - dyl; zlocala = p.z - dzl;
        ia = (int)std::floor(xlocala); ja = (int)std::floor(ylocala); ka = (int)std::floor(zlocala);
        xa = ia; ya = ja; za = ka;
        i1a = ia + 1; j1a = ja + 1; k1a = ka + 1;
        xr = (ib == ia) ? (xlocalb + xlocala) * 0.5 : std::max(xb, xa);
        yr = (jb == ja) ? (ylocalb + ylocala) * 0.5 : std::max(yb, ya);
        zr = (kb == ka) ? (zlocalb + zlocala) * 0.5 : std::max(zb, za);
      } else {  // psolve1.F90:416-606
        bool cx = p.x < dxl || p.x >= dxu, cy = p.y < dyl || p.y >= dyu, cz = p.z < dzl || p.z >= dzu;
        p.nid = nborps_single(c, is, cx, cy, cz);
        const int32_t* nb = c->npbnd[is];
        // x
        if (p.x < 0.0) {
          if (nb[0] == 0) { xlocala = p.x; p.x = p.x + slx; ia = -1; xa = -1.0; i1a = 0; xr = 0.0; }
          else if (nb[0] == 1) { p.x = -p.x; p.vx = -p.vx; xlocala = p.x; ia = 0; xa = 0.0; i1a = 1; xr = 0.0; }
          else { xlocala = -1.0; ia = -1; xa = -1.0; i1a = 0; xr = 0.0; }
        } else if (p.x >= slx) {
          if (nb[0] == 0) { xlocala = p.x - dxl; p.x = p.x - slx; ia = ngx; xa = dngx; i1a = ngx + 1; xr = dngx; }
          else if (nb[0] == 1) { p.x = tslx - p.x; p.vx = -p.vx; xlocala = p.x - dxl; ia = ngx - 1; xa = dngx - 1.0; i1a = ngx; xr = dngx; }
          else { xlocala = dngx + 1.0; ia = ngx; xa = dngx; i1a = ngx + 1; xr = dngx; }
        } else {
          xlocala = p.x - dxl; ia = (int)std::floor(xlocala); xa = ia; i1a = ia + 1;
          xr = (ib == ia) ? (xlocalb + xlocala) * 0.5 : std::max(xb, xa);
        }
        // y
        if (p.y < 0.0) {
          if (nb[1] == 0) { ylocala = p.y; p.y = p.y + sly; ja = -1; ya = -1.0; j1a = 0; yr = 0.0; }
          else if (nb[1] == 1) { p.y = -p.y; p.vy = -p.vy; ylocala = p.y; ja = 0; ya = 0.0; j1a = 1; yr = 0.0; }
          else { ylocala = -1.0; ja = -1; ya = -1.0; j1a = 0; yr = 0.0; }
        } else if (p.y >= sly) {
          if (nb[1] == 0) { ylocala = p.y - dyl; p.y = p.y - sly; ja = ngy; ya = dngy; j1a = ngy + 1; yr = dngy; }
          else if (nb[1] == 1) { p.y = tsly - p.y; p.vy = -p.vy; ylocala = p.y - dyl; ja = ngy - 1; ya = dngy - 1.0; j1a = ngy; yr = dngy; }
          else { ylocala = dngy + 1.0; ja = ngy; ya = dngy; j1a = ngy + 1; yr = dngy; }
        } else {
          ylocala = p.y - dyl; ja = (int)std::floor(ylocala); ya = ja; j1a = ja + 1;
          yr = (jb == ja) ? (ylocalb + ylocala) * 0.5 : std::max(yb, ya);
        }
        // z
        if (p.z < 0.0) {
          if (nb[2] == 0) { zlocala = p.z; p.z = p.z + slz; ka = -1; za = -1.0; k1a = 0; zr = 0.0; }
          else if (nb[2] == 1) { p.z = -p.z; p.vz = -p.vz; zlocala = p.z; ka = 0; za = 0.0; k1a = 1; zr = 0.0; }
          else { zlocala = -1.0; ka = -1; za = -1.0; k1a = 0; zr = 0.0; }
        } else if (p.z >= slz) {
          if (nb[2] == 0) { zlocala = p.z - dzl; p.z = p.z - slz; ka = ngz; za = dngz; k1a = ngz + 1; zr = dngz; }
          else if (nb[2] == 1) { p.z = tslz - p.z; p.vz = -p.vz; zlocala = p.z - dzl; ka = ngz - 1; za = dngz - 1.0; k1a = ngz; zr = dngz; }
          else { zlocala = dngz + 1.0; ka = ngz; za = dngz; k1a = ngz + 1; zr = dngz; }
        } else {
          zlocala = p.z - dzl; ka = (int)std::floor(zlocala); za = ka; k1a = ka + 1;
          zr = (kb == ka) ? (zlocalb + zlocala) * 0.5 : std::max(zb, za);
        }
        if (p.nid == -1) gc->nesc[is] += 1;
      }

      // Internal boundary treatment 1, psolve1.F90:639-715.
      if (c->line_mode != 1) {
        for (int ipc = 0; ipc < c->npc; ipc++) {
          if (p.nid == -1) continue;
          const emsesg_body& b = c->body[ipc];
          if (b.geotype == 0 || b.geotype == 1) {
            if (xlocalb >= xlc[ipc] && xlocalb <= xuc[ipc] && ylocalb >= ylc[ipc] &&
                ylocalb <= yuc[ipc] && zlocalb >= zlc[ipc] && zlocalb <= zuc[ipc]) {
              xlocalb = xr; ylocalb = yr; zlocalb = zr;
            }
            if (xlocala >= xlc[ipc] && xlocala <= xuc[ipc] && ylocala >= ylc[ipc] &&
                ylocala <= yuc[ipc] && zlocala >= zlc[ipc] && zlocala <= zuc[ipc]) {
              p.nid = -1;
              gc->influx[is][ipc] += 1;
              if (p.pid >= 0 && p.pid <= EMSESG_INPC) gc->infhist[is][ipc][p.pid] += 1;
              if (surf) {
                const double bp[3] = {xlocalb0 + dxl, ylocalb0 + dyl, zlocalb0 + dzl};
                const double ap[3] = {xlocala + dxl, ylocala + dyl, zlocala + dzl};
                const int64_t sc = orc_surface_cell(c, ipc, bp, ap);
                if (sc >= 0) surf[(int64_t)is * nsurf + sc] += 1;
              }
              xlocala = xr; ylocala = yr; zlocala = zr;
            }
          } else if (b.geotype == 2) {
            double d1, d2, a;
            if (b.cyl_align == 1) { d1 = p.y - b.cyl_axis[0]; d2 = p.z - b.cyl_axis[1]; a = p.x; }
            else if (b.cyl_align == 2) { d1 = p.z - b.cyl_axis[0]; d2 = p.x - b.cyl_axis[1]; a = p.y; }
            else if (b.cyl_align == 3) { d1 = p.x - b.cyl_axis[0]; d2 = p.y - b.cyl_axis[1]; a = p.z; }
            else continue;
            if (a >= b.cyl_edge[0] && a <= b.cyl_edge[1] && d1 * d1 + d2 * d2 < radsq[ipc]) {
              p.nid = -1;
              gc->influx[is][ipc] += 1;
              if (p.pid >= 0 && p.pid <= EMSESG_INPC) gc->infhist[is][ipc][p.pid] += 1;
            }
          } else if (b.geotype == 3) {
            double d1 = p.x - b.sph_center[0], d2 = p.y - b.sph_center[1], d3 = p.z - b.sph_center[2];
            if (d1 * d1 + d2 * d2 + d3 * d3 < radsq[ipc]) {
              p.nid = -1;
              gc->influx[is][ipc] += 1;
              if (p.pid >= 0 && p.pid <= EMSESG_INPC) gc->infhist[is][ipc][p.pid] += 1;
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

      // 24 scatter-adds, psolve1.F90:759-789 (same statement order).
      auto add = [&](int cc, int i, int j, int k, double v) { wrk[fw.at(cc, i, j, k)] = wrk[fw.at(cc, i, j, k)] + v; };
      add(TJX, ib, jb, kb, vvx1 * vx1w1);
      add(TJY, ib, jb, kb, vvy1 * vy1w1);
      add(TJZ, ib, jb, kb, vvz1 * vz1w1);
      add(TJX, ib, j1b, kb, vvx1 * vx1w2);
      add(TJY, i1b, jb, kb, vvy1 * vy1w2);
      add(TJZ, i1b, jb, kb, vvz1 * vz1w2);
      add(TJX, ib, jb, k1b, vvx1 * vx1w3);
      add(TJY, ib, jb, k1b, vvy1 * vy1w3);
      add(TJZ, ib, j1b, kb, vvz1 * vz1w3);
      add(TJX, ib, j1b, k1b, vvx1 * vx1w4);
      add(TJY, i1b, jb, k1b, vvy1 * vy1w4);
      add(TJZ, i1b, j1b, kb, vvz1 * vz1w4);
      add(TJX, ia, ja, ka, vvx2 * vx2w1);
      add(TJY, ia, ja, ka, vvy2 * vy2w1);
      add(TJZ, ia, ja, ka, vvz2 * vz2w1);
      add(TJX, ia, j1a, ka, vvx2 * vx2w2);
      add(TJY, i1a, ja, ka, vvy2 * vy2w2);
      add(TJZ, i1a, ja, ka, vvz2 * vz2w2);
      add(TJX, ia, ja, k1a, vvx2 * vx2w3);
      add(TJY, ia, ja, k1a, vvy2 * vy2w3);
      add(TJZ, ia, j1a, ka, vvz2 * vz2w3);
      add(TJX, ia, j1a, k1a, vvx2 * vx2w4);
      add(TJY, i1a, ja, k1a, vvy2 * vy2w4);
      add(TJZ, i1a, j1a, ka, vvz2 * vz2w4);
    }
    // Flush, psolve1.F90:793-817.
    double qs = c->q[is];
    for (int k = -1; k <= c->nz + 1; k++)
      for (int j = -1; j <= c->ny + 1; j++)
        for (int i = -1; i <= c->nx + 1; i++) {
          aj[fa.at(JX, i, j, k)] = aj[fa.at(JX, i, j, k)] + wrk[fw.at(TJX, i, j, k)] * qs;
          aj[fa.at(JY, i, j, k)] = aj[fa.at(JY, i, j, k)] + wrk[fw.at(TJY, i, j, k)] * qs;
          aj[fa.at(JZ, i, j, k)] = aj[fa.at(JZ, i, j, k)] + wrk[fw.at(TJZ, i, j, k)] * qs;
        }
    if (func == 1 && ajdg) {
      int iss = is * 3;
      for (int k = -1; k <= c->nz + 1; k++)
        for (int j = -1; j <= c->ny + 1; j++)
          for (int i = -1; i <= c->nx + 1; i++)
            for (int d = 0; d < 3; d++)
              ajdg[fj.at(iss + d, i, j, k)] = ajdg[fj.at(iss + d, i, j, k)] + wrk[fw.at(TJX + d, i, j, k)] * qs;
    }
  }
  chgacm_update(c, gc);
  return rs.ok ? 0 : EMSESG_ERR_ARG;
}

// charge, src/pcl2field/charge.F90:40-146, with get_interpolation_weight
// (:152-194) and distribute_charge (:197-210).
void orc_charge(const emsesg_config* c, int func, emsesg_particle* pbuf,
                const int64_t* totalp, double* rho, double* rhodg, double* rhobk,
                double* rhobksp) {
  FD fr = fd_of(c, EMSESG_FIELD_RHO), fd = fd_of(c, EMSESG_FIELD_RHODG);
  int64_t rsz = fr.size();
  if (func == 0 || func == 2) std::fill(rho, rho + rsz, 0.0);
  if ((func == 1 || func == 2) && rhodg) std::fill(rhodg, rhodg + fd.size(), 0.0);
  const int nspec = c->nspec;
  auto distribute = [&](double* rh, const FD& f, int cc, int i, int j, int k, double qc, const W8& w) {
    // rh(1:2,1:2,1:2) view at (i,j,k): rh(a,b,c) -> (i+a-1, j+b-1, k+c-1)
    rh[f.at(cc, i, j, k + 1)] = rh[f.at(cc, i, j, k + 1)] + w.v1 * qc;
    rh[f.at(cc, i + 1, j, k + 1)] = rh[f.at(cc, i + 1, j, k + 1)] + w.v2 * qc;
    rh[f.at(cc, i + 1, j + 1, k + 1)] = rh[f.at(cc, i + 1, j + 1, k + 1)] + w.v3 * qc;
    rh[f.at(cc, i, j + 1, k + 1)] = rh[f.at(cc, i, j + 1, k + 1)] + w.v4 * qc;
    rh[f.at(cc, i, j, k)] = rh[f.at(cc, i, j, k)] + w.v5 * qc;
    rh[f.at(cc, i + 1, j, k)] = rh[f.at(cc, i + 1, j, k)] + w.v6 * qc;
    rh[f.at(cc, i + 1, j + 1, k)] = rh[f.at(cc, i + 1, j + 1, k)] + w.v7 * qc;
    rh[f.at(cc, i, j + 1, k)] = rh[f.at(cc, i, j + 1, k)] + w.v8 * qc;
  };
  int64_t nee = 0;
  for (int is = 0; is < nspec; is++) {
    int64_t ns = nee, ne = nee + totalp[is];
    nee = ne;
    double* rbsp = rhobksp ? rhobksp + (int64_t)is * rsz : nullptr;
    int cis = is, cnis = nspec + is;  // rhodg(is) and rhodg(nspec+is), 0-based
    for (int64_t m = ns; m < ne; m++) {
      emsesg_particle& p = pbuf[m];
      if (p.nid == -1) continue;
      double xlocal = p.x, ylocal = p.y, zlocal = p.z;  // xl = yl = zl = 0
      int i = (int)xlocal, j = (int)ylocal, k = (int)zlocal;
      W8 w = weights(xlocal - i, ylocal - j, zlocal - k);
      double q = c->q[is];
      if (p.preside >= 0) {
        if (func == 0 || func == 2) distribute(rho, fr, 0, i, j, k, q, w);
        if ((func == 1 || func == 2) && rhodg) distribute(rhodg, fd, cis, i, j, k, q, w);
      } else if (p.preside == EMSESG_PCL_TO_BE_ACCUMULATED ||
                 p.preside == EMSESG_PCL_TO_BE_ACCUMULATED_AS_ANTIPCL) {
        double qq = p.preside == EMSESG_PCL_TO_BE_ACCUMULATED ? q : -q;
        if (rhobk) distribute(rhobk, fr, 0, i, j, k, qq, w);
        if (rbsp) distribute(rbsp, fr, 0, i, j, k, qq, w);
        if ((func == 1 || func == 2) && rhodg) {
          if (func == 2 && p.preside == EMSESG_PCL_TO_BE_ACCUMULATED_AS_ANTIPCL)
            distribute(rhodg, fd, cis, i, j, k, qq, w);  // charge.F90:134
          distribute(rhodg, fd, cnis, i, j, k, qq, w);
        }
        p.nid = -1;
        p.preside = 0;
      }
    }
  }
}

// oh3_exchange_borders(CRH) + add_boundary_charge, charge.F90:214-412, with
// sl=-1, su=1, nl=nu=1, dl=du=0 (ctypes CRH, ohinit.F90:115).
void orc_reduce_rho(const emsesg_config* c, double* rh, int ncomp) {
  FD f = fd_of(c, EMSESG_FIELD_RHO);
  f.nc = ncomp;
  exchange_single(c, f, rh, CT_RH);
  const int sl = -1, su = 1, nl = 1, nu = 1, dl = sl + nl, du = su - nu;
  const int lx = c->nx, ly = c->ny, lz = c->nz;
  auto R = [&](int e, int i, int j, int k) -> double& { return rh[f.at(e, i, j, k)]; };
  bool per[3] = {c->nfbnd[0] == 0, c->nfbnd[1] == 0, c->nfbnd[2] == 0};
  // z lower / upper
  if (per[2]) {
    for (int k = 0; k <= nl - 1; k++) for (int j = 0; j <= ly + (su + nu - sl) - 1; j++)
      for (int i = 0; i <= lx + (su + nu - sl) - 1; i++) for (int e = 0; e < ncomp; e++)
        R(e, sl + i, sl + j, dl + k) = R(e, sl + i, sl + j, dl + k) + R(e, sl + i, sl + j, sl + k);
  } else {
    for (int j = 0; j <= ly + (su + nu - sl) - 1; j++) for (int i = 0; i <= lx + (su + nu - sl) - 1; i++)
      for (int e = 0; e < ncomp; e++) R(e, sl + i, sl + j, dl) = R(e, sl + i, sl + j, dl) * 2.0;
  }
  if (per[2]) {
    for (int k = 0; k <= nu - 1; k++) for (int j = 0; j <= ly + (su + nu - sl) - 1; j++)
      for (int i = 0; i <= lx + (su + nu - sl) - 1; i++) for (int e = 0; e < ncomp; e++)
        R(e, sl + i, sl + j, lz + du + k) = R(e, sl + i, sl + j, lz + du + k) + R(e, sl + i, sl + j, lz + su + k);
  } else {
    for (int j = 0; j <= ly + (su + nu - sl) - 1; j++) for (int i = 0; i <= lx + (su + nu - sl) - 1; i++)
      for (int e = 0; e < ncomp; e++) R(e, sl + i, sl + j, lz + du) = R(e, sl + i, sl + j, lz + du) * 2.0;
  }
  // y lower / upper
  if (per[1]) {
    for (int k = 0; k <= lz + (du + nu - dl) - 1; k++) for (int j = 0; j <= nl - 1; j++)
      for (int i = 0; i <= lx + (su + nu - sl) - 1; i++) for (int e = 0; e < ncomp; e++)
        R(e, sl + i, dl + j, dl + k) = R(e, sl + i, dl + j, dl + k) + R(e, sl + i, sl + j, dl + k);
  } else {
    for (int k = 0; k <= lz + (du + nu - dl) - 1; k++) for (int i = 0; i <= lx + (su + nu - sl) - 1; i++)
      for (int e = 0; e < ncomp; e++) R(e, sl + i, dl, dl + k) = R(e, sl + i, dl, dl + k) * 2.0;
  }
  if (per[1]) {
    for (int k = 0; k <= lz + (du + nu - dl) - 1; k++) for (int j = 0; j <= nu - 1; j++)
      for (int i = 0; i <= lx + (su + nu - sl) - 1; i++) for (int e = 0; e < ncomp; e++)
        R(e, sl + i, ly + du + j, dl + k) = R(e, sl + i, ly + du + j, dl + k) + R(e, sl + i, ly + su + j, dl + k);
  } else {
    for (int k = 0; k <= lz + (du + nu - dl) - 1; k++) for (int i = 0; i <= lx + (su + nu - sl) - 1; i++)
      for (int e = 0; e < ncomp; e++) R(e, sl + i, ly + du, dl + k) = R(e, sl + i, ly + du, dl + k) * 2.0;
  }
  // x lower / upper
  if (per[0]) {
    for (int k = 0; k <= lz + (du + nu - dl) - 1; k++) for (int j = 0; j <= ly + (du + nu - dl) - 1; j++)
      for (int i = 0; i <= nl - 1; i++) for (int e = 0; e < ncomp; e++)
        R(e, dl + i, dl + j, dl + k) = R(e, dl + i, dl + j, dl + k) + R(e, sl + i, dl + j, dl + k);
  } else {
    for (int k = 0; k <= lz + (du + nu - dl) - 1; k++) for (int j = 0; j <= ly + (du + nu - dl) - 1; j++)
      for (int e = 0; e < ncomp; e++) R(e, dl, dl + j, dl + k) = R(e, dl, dl + j, dl + k) * 2.0;
  }
  if (per[0]) {
    for (int k = 0; k <= lz + (du + nu - dl) - 1; k++) for (int j = 0; j <= ly + (du + nu - dl) - 1; j++)
      for (int i = 0; i <= nu - 1; i++) for (int e = 0; e < ncomp; e++)
        R(e, lx + du + i, dl + j, dl + k) = R(e, lx + du + i, dl + j, dl + k) + R(e, lx + su + i, dl + j, dl + k);
  } else {
    for (int k = 0; k <= lz + (du + nu - dl) - 1; k++) for (int j = 0; j <= ly + (du + nu - dl) - 1; j++)
      for (int e = 0; e < ncomp; e++) R(e, lx + du, dl + j, dl + k) = R(e, lx + du, dl + j, dl + k) * 2.0;
  }
}

namespace {
// add_boundary_current (psolve1.F90:859-1079) on one component triple
// (e0 = offset of JX), with sl=-4, su=2, nl=nu=3, dl=du=-1 (ctypes CAJ).
void add_boundary_current_triple(const emsesg_config* c, const FD& f, double* aj, int e0) {
  const int sl = -4, su = 2, nl = 3, nu = 3, dl = sl + nl, du = su - nu;
  const int xu = c->nx, yu = c->ny, zu = c->nz;
  auto A = [&](int d, int i, int j, int k) -> double& { return aj[f.at(e0 + d, i, j, k)]; };
  // z lower
  if (c->nfbnd[2] == 0) {
    for (int k = 0; k <= nl - 1; k++) for (int j = 0; j <= yu + (su + nu - sl) - 1; j++)
      for (int i = 0; i <= xu + (su + nu - sl) - 1; i++) for (int d = 0; d < 3; d++)
        A(d, sl + i, sl + j, dl + k) = A(d, sl + i, sl + j, dl + k) + A(d, sl + i, sl + j, sl + k);
  } else if (c->nfbnd[2] == 1) {
    int k = 0;
    for (int j = 0; j <= yu + (su + nu - sl) - 1; j++) for (int i = 0; i <= xu + (su + nu - sl) - 1; i++) {
      A(JX, sl + i, sl + j, k) = A(JX, sl + i, sl + j, k) * 2.0;
      A(JY, sl + i, sl + j, k) = A(JY, sl + i, sl + j, k) * 2.0;
      A(JZ, sl + i, sl + j, k - 1) = -A(JZ, sl + i, sl + j, -k);
    }
  }
  // z upper
  if (c->nfbnd[2] == 0) {
    for (int k = 0; k <= nu - 1; k++) for (int j = 0; j <= yu + (su + nu - sl) - 1; j++)
      for (int i = 0; i <= xu + (su + nu - sl) - 1; i++) for (int d = 0; d < 3; d++)
        A(d, sl + i, sl + j, zu + du + k) = A(d, sl + i, sl + j, zu + du + k) + A(d, sl + i, sl + j, zu + su + k);
  } else if (c->nfbnd[2] == 1) {
    for (int k = 0; k <= 0; k++) for (int j = 0; j <= yu + (su + nu - sl) - 1; j++)
      for (int i = 0; i <= xu + (su + nu - sl) - 1; i++) {
        A(JX, sl + i, sl + j, zu + k) = A(JX, sl + i, sl + j, zu + k) * 2.0;
        A(JY, sl + i, sl + j, zu + k) = A(JY, sl + i, sl + j, zu + k) * 2.0;
        A(JZ, sl + i, sl + j, zu + k) = -A(JZ, sl + i, sl + j, zu - k - 1);
      }
    for (int k = 1; k <= 1; k++) for (int j = 0; j <= yu + (su + nu - sl) - 1; j++)
      for (int i = 0; i <= xu + (su + nu - sl) - 1; i++) {
        A(JX, sl + i, sl + j, zu + k) = A(JX, sl + i, sl + j, zu - k);
        A(JY, sl + i, sl + j, zu + k) = A(JY, sl + i, sl + j, zu - k);
        A(JZ, sl + i, sl + j, zu + k) = -A(JZ, sl + i, sl + j, zu - k - 1);
      }
  }
  // y lower
  if (c->nfbnd[1] == 0) {
    for (int k = 0; k <= zu + (du + nu - dl) - 1; k++) for (int j = 0; j <= nl - 1; j++)
      for (int i = 0; i <= xu + (su + nu - sl) - 1; i++) for (int d = 0; d < 3; d++)
        A(d, sl + i, dl + j, dl + k) = A(d, sl + i, dl + j, dl + k) + A(d, sl + i, sl + j, dl + k);
  } else if (c->nfbnd[1] == 1) {
    int j = 0;
    for (int k = 0; k <= zu + (du + nu - dl) - 1; k++) for (int i = 0; i <= xu + (su + nu - sl) - 1; i++) {
      A(JX, sl + i, j, dl + k) = A(JX, sl + i, j, dl + k) * 2.0;
      A(JY, sl + i, j - 1, dl + k) = -A(JY, sl + i, -j, dl + k);
      A(JZ, sl + i, j, dl + k) = A(JZ, sl + i, j, dl + k) * 2.0;
    }
  }
  // y upper
  if (c->nfbnd[1] == 0) {
    for (int k = 0; k <= zu + (du + nu - dl) - 1; k++) for (int j = 0; j <= nu - 1; j++)
      for (int i = 0; i <= xu + (su + nu - sl) - 1; i++) for (int d = 0; d < 3; d++)
        A(d, sl + i, yu + du + j, dl + k) = A(d, sl + i, yu + du + j, dl + k) + A(d, sl + i, yu + su + j, dl + k);
  } else if (c->nfbnd[1] == 1) {
    for (int k = 0; k <= zu + (du + nu - dl) - 1; k++) {
      for (int j = 0; j <= 0; j++) for (int i = 0; i <= xu + (su + nu - sl) - 1; i++) {
        A(JX, sl + i, yu + j, dl + k) = A(JX, sl + i, yu + j, dl + k) * 2.0;
        A(JY, sl + i, yu + j, dl + k) = -A(JY, sl + i, yu - j - 1, dl + k);
        A(JZ, sl + i, yu + j, dl + k) = A(JZ, sl + i, yu + j, dl + k) * 2.0;
      }
      for (int j = 1; j <= 1; j++) for (int i = 0; i <= xu + (su + nu - sl) - 1; i++) {
        A(JX, sl + i, yu + j, dl + k) = A(JX, sl + i, yu - j, dl + k);
        A(JY, sl + i, yu + j, dl + k) = -A(JY, sl + i, yu - j - 1, dl + k);
        A(JZ, sl + i, yu + j, dl + k) = A(JZ, sl + i, yu - j, dl + k);
      }
    }
  }
  // x lower
  if (c->nfbnd[0] == 0) {
    for (int k = 0; k <= zu + (du + nu - dl) - 1; k++) for (int j = 0; j <= yu + (du + nu - dl) - 1; j++)
      for (int i = 0; i <= nl - 1; i++) for (int d = 0; d < 3; d++)
        A(d, dl + i, dl + j, dl + k) = A(d, dl + i, dl + j, dl + k) + A(d, sl + i, dl + j, dl + k);
  } else if (c->nfbnd[0] == 1) {
    int i = 0;
    for (int k = 0; k <= zu + (du + nu - dl) - 1; k++) for (int j = 0; j <= yu + (du + nu - dl) - 1; j++) {
      A(JX, i - 1, dl + j, dl + k) = -A(JX, -i, dl + j, dl + k);
      A(JY, i, dl + j, dl + k) = A(JY, i, dl + j, dl + k) * 2.0;
      A(JZ, i, dl + j, dl + k) = A(JZ, i, dl + j, dl + k) * 2.0;
    }
  }
  // x upper
  if (c->nfbnd[0] == 0) {
    for (int k = 0; k <= zu + (du + nu - dl) - 1; k++) for (int j = 0; j <= yu + (du + nu - dl) - 1; j++)
      for (int i = 0; i <= nu - 1; i++) for (int d = 0; d < 3; d++)
        A(d, xu + du + i, dl + j, dl + k) = A(d, xu + du + i, dl + j, dl + k) + A(d, xu + su + i, dl + j, dl + k);
  } else if (c->nfbnd[0] == 1) {
    for (int k = 0; k <= zu + (du + nu - dl) - 1; k++) for (int j = 0; j <= yu + (du + nu - dl) - 1; j++) {
      for (int i = 0; i <= 0; i++) {
        A(JX, xu + i, dl + j, dl + k) = -A(JX, xu - i - 1, dl + j, dl + k);
        A(JY, xu + i, dl + j, dl + k) = A(JY, xu + i, dl + j, dl + k) * 2.0;
        A(JZ, xu + i, dl + j, dl + k) = A(JZ, xu + i, dl + j, dl + k) * 2.0;
      }
      for (int i = 1; i <= 1; i++) {
        A(JX, xu + i, dl + j, dl + k) = -A(JX, xu - i - 1, dl + j, dl + k);
        A(JY, xu + i, dl + j, dl + k) = A(JY, xu - i, dl + j, dl + k);
        A(JZ, xu + i, dl + j, dl + k) = A(JZ, xu - i, dl + j, dl + k);
      }
    }
  }
}
}  // namespace

void orc_reduce_aj(const emsesg_config* c, double* aj) {
  FD f = fd_of(c, EMSESG_FIELD_AJ);
  exchange_single(c, f, aj, CT_AJ);
  add_boundary_current_triple(c, f, aj, 0);
}

// add_boundary_current2 (psolve1.F90:1081-) applies the same folds to every
// species triple of ajdg; doing the triples one after another gives the same
// values because the triples never mix.
void orc_reduce_ajdg(const emsesg_config* c, double* ajdg) {
  FD f = fd_of(c, EMSESG_FIELD_AJDG);
  exchange_single(c, f, ajdg, CT_AJ);
  for (int is = 0; is < c->nspec; is++) add_boundary_current_triple(c, f, ajdg, 3 * is);
}

// rhoupd, src/field/rhoupd.F90:40-49.
void orc_rhoupd(const emsesg_config* c, double* rho, const double* aj) {
  FD fr = fd_of(c, EMSESG_FIELD_RHO), fa = fd_of(c, EMSESG_FIELD_AJ);
  for (int k = 0; k <= c->nz; k++)
    for (int j = 0; j <= c->ny; j++)
      for (int i = 0; i <= c->nx; i++)
        rho[fr.at(0, i, j, k)] = rho[fr.at(0, i, j, k)] -
            (aj[fa.at(JX, i, j, k)] - aj[fa.at(JX, i - 1, j, k)] + aj[fa.at(JY, i, j, k)] -
             aj[fa.at(JY, i, j - 1, k)] + aj[fa.at(JZ, i, j, k)] - aj[fa.at(JZ, i, j, k - 1)]) * 2.0;
}

// Kinetic energy, src/etc/energy.F90:29-47 (ps = 1 only).
void orc_energy(const emsesg_config* c, const emsesg_particle* pbuf,
                const int64_t* totalp, double* engk) {
  double vol = (double)c->nx * (double)c->ny * (double)c->nz;
  int64_t nee = 0;
  for (int is = 0; is < c->nspec; is++) {
    int64_t ns = nee, ne = nee + totalp[is];
    nee = ne;
    double tkx = 0.0, tky = 0.0, tkz = 0.0;
    for (int64_t m = ns; m < ne; m++) {
      if (pbuf[m].nid == -1) continue;
      tkx = tkx + pbuf[m].vx * pbuf[m].vx;
      tky = tky + pbuf[m].vy * pbuf[m].vy;
      tkz = tkz + pbuf[m].vz * pbuf[m].vz;
    }
    engk[is * 3 + 0] = 0.5 * c->rm[is] * tkx / vol;
    engk[is * 3 + 1] = 0.5 * c->rm[is] * tky / vol;
    engk[is * 3 + 2] = 0.5 * c->rm[is] * tkz / vol;
  }
}

// Canonical sort key.  The reference sorts each species segment with libc
// qsort on (int)(a->z - b->z) (lib/psort/psort-struct.c:15-20), a truncated,
// non-transitive comparator with an unspecified (unstable) result order.
// The project fixes the order as a stable sort by the tile-major cell key:
//   tile = (i/tx, j/ty, k/tz) in x-fastest order, then the cell inside the
//   tile in x-fastest order; cell indices int() of the position, clamped to
//   the grid.  With the tile equal to the whole grid (the default) the key is
//   k*ny*nx + j*nx + i.  Within a species segment, consecutive particles in
//   this order satisfy the reference comparator's (int)(z_a - z_b) <= 0.
int64_t orc_sort_key(const emsesg_config* c, const emsesg_particle* p) {
  int n[3] = {c->nx, c->ny, c->nz};
  int t[3];
  for (int d = 0; d < 3; d++) t[d] = c->sort_tile[d] > 0 ? c->sort_tile[d] : n[d];
  double pos[3] = {p->x, p->y, p->z};
  int ci[3];
  for (int d = 0; d < 3; d++) {
    int v = (int)pos[d];
    if (pos[d] < 0.0) v = 0;
    ci[d] = std::min(std::max(v, 0), n[d] - 1);
  }
  int nt[3];
  for (int d = 0; d < 3; d++) nt[d] = (n[d] + t[d] - 1) / t[d];
  int64_t tile = (int64_t)(ci[0] / t[0]) + (int64_t)nt[0] * ((ci[1] / t[1]) + (int64_t)nt[1] * (ci[2] / t[2]));
  int64_t in = (int64_t)(ci[0] % t[0]) + (int64_t)t[0] * ((ci[1] % t[1]) + (int64_t)t[1] * (ci[2] % t[2]));
  return tile * ((int64_t)t[0] * t[1] * t[2]) + in;
}

void orc_spsort(const emsesg_config* c, emsesg_particle* pbuf, const int64_t* totalp) {
  int64_t nee = 0;
  for (int is = 0; is < c->nspec; is++) {
    int64_t ns = nee, n = totalp[is];
    nee += n;
    std::vector<std::pair<int64_t, int64_t>> keys(n);
    for (int64_t m = 0; m < n; m++) keys[m] = {orc_sort_key(c, &pbuf[ns + m]), m};
    std::stable_sort(keys.begin(), keys.end(),
                     [](const std::pair<int64_t, int64_t>& a, const std::pair<int64_t, int64_t>& b) { return a.first < b.first; });
    std::vector<emsesg_particle> tmp(n);
    for (int64_t m = 0; m < n; m++) tmp[m] = pbuf[ns + keys[m].second];
    std::copy(tmp.begin(), tmp.end(), pbuf + ns);
  }
}

// Single-rank compaction: particles with nid == -1 leave, the rest keep
// their buffer order; species segments stay back to back.
void orc_compact(const emsesg_config* c, emsesg_particle* pbuf, int64_t* totalp) {
  int64_t rd = 0, wr = 0;
  for (int is = 0; is < c->nspec; is++) {
    int64_t kept = 0;
    for (int64_t m = 0; m < totalp[is]; m++, rd++) {
      if (pbuf[rd].nid == -1) continue;
      pbuf[wr++] = pbuf[rd];
      kept++;
    }
    totalp[is] = kept;
  }
}

// Synthetic plasma: for every cell (x fastest) and species, ppc particles at
// cell + U[0,1)^3, velocities N(0, vth^2) per component + drift by
// Box-Muller.  Uniforms come from the counter hash with stream 1000+is and
// index 8*m + slot, so any slice can be regenerated independently.
void orc_load_plasma(const emsesg_config* c, const emsesg_plasma* pl,
                     emsesg_particle* pbuf, int64_t* totalp) {
  int64_t ncell = (int64_t)c->nx * c->ny * c->nz;
  int64_t base = 0;
  const double twopi = 6.283185307179586;
  for (int is = 0; is < c->nspec; is++) {
    int64_t n = ncell * pl->ppc[is];
    for (int64_t m = 0; m < n; m++) {
      int64_t cell = m / pl->ppc[is];
      int i = (int)(cell % c->nx), j = (int)((cell / c->nx) % c->ny), k = (int)(cell / ((int64_t)c->nx * c->ny));
      uint64_t st = 1000 + is;
      double u[8];
      for (int s = 0; s < 8; s++) u[s] = orc_hash_u01(pl->seed, st, (uint64_t)m * 8 + s);
      emsesg_particle& p = pbuf[base + m];
      p.x = i + u[0];
      p.y = j + u[1];
      p.z = k + u[2];
      double r1 = std::sqrt(-2.0 * std::log(1.0 - u[3]));
      double r2 = std::sqrt(-2.0 * std::log(1.0 - u[5]));
      p.vx = pl->vth[is] * r1 * std::cos(twopi * u[4]) + pl->vdrift[is][0];
      p.vy = pl->vth[is] * r1 * std::sin(twopi * u[4]) + pl->vdrift[is][1];
      p.vz = pl->vth[is] * r2 * std::cos(twopi * u[6]) + pl->vdrift[is][2];
      p.pid = 0;
      p.preside = 0;
      p.nid = 0;
      p.spec = is + 1;
    }
    totalp[is] = n;
    base += n;
  }
}

}  // extern "C"
