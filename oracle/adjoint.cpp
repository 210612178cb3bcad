/*
 * adjoint.cpp -- TEST INFRASTRUCTURE ONLY: the FP64 CPU adjoint of K steps of
 * the particle path on a periodic grid, the checker of the GPU adjoint.
 *
 * Forward step (psolve1.F90:186-333 and :717-789, all particles alive,
 * periodic axes): trilinear gather of the node fields E, B (+ e0, b0) at
 * x_n, Buneman-Boris with qmp = qm*ustep/2, move a = x_n + v_{n+1}*ustep,
 * zigzag current J_n of the segment x_n -> a (relay point r = (a+b)/2 in one
 * cell, else the shared cell face), deposited with q(is) and folded
 * periodically; x_{n+1} = a wrapped into [0, n).
 *
 * Loss: sum over steps and over the probe nodes of Jx(node)^2.
 *
 * Reverse sweep by hand, step by step from the last (orc_adjoint_ckpt keeps
 * the state every ckpt steps and recomputes each segment's states, moves
 * only, before its reverse steps; orc_adjoint keeps every state): the J-loss gradient
 * g = 2 Jx on the probe nodes gives dS/da and dS/db of each particle's
 * deposit S = sum_nodes g . J; the move gives lambda_v += lambda_a*ustep and
 * lambda_b += lambda_a; the Boris rotation is transposed term by term; the
 * gather scatters w_c*lambda_E and w_c*lambda_B into the node-field
 * gradients and adds sum_c grad(w_c) (E_c.lambda_E + B_c.lambda_B) to
 * lambda_x.  The gradient of the uniform e0 / b0 is the sum of the node
 * gradients.  Gradients of the initial velocities are lambda_v after the
 * sweep.
 */
#include <cmath>
#include <cstdint>
#include <algorithm>
#include <cstring>
#include <vector>

#include "emses_oracle.h"

namespace {

struct Grid {
  int n[3];
  int64_t idx(int i, int j, int k) const {
    i %= n[0]; if (i < 0) i += n[0];
    j %= n[1]; if (j < 0) j += n[1];
    k %= n[2]; if (k < 0) k += n[2];
    return (int64_t)i + (int64_t)n[0] * ((int64_t)j + (int64_t)n[1] * k);
  }
};

struct V3 { double x, y, z; };
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

// Corner c = (di,dj,dk) of the trilinear gather: weight and its gradient
// with respect to the in-cell offsets (x1, y1, z1).
inline void corner(int c, double x1, double y1, double z1, int& di, int& dj, int& dk, double& w, double g[3]) {
  di = c & 1; dj = (c >> 1) & 1; dk = c >> 2;
  const double X = di ? x1 : 1.0 - x1, Y = dj ? y1 : 1.0 - y1, Z = dk ? z1 : 1.0 - z1;
  const double dX = di ? 1.0 : -1.0, dY = dj ? 1.0 : -1.0, dZ = dk ? 1.0 : -1.0;
  w = X * Y * Z;
  g[0] = dX * Y * Z; g[1] = X * dY * Z; g[2] = X * Y * dZ;
}

struct Seg {     // per axis of one zigzag step
  int cb, ca;    // cells of b and a
  double r;      // relay point
  double drda, drdb;
};

inline Seg relay(double b, double a) {
  Seg s;
  s.cb = (int)std::floor(b);
  s.ca = (int)std::floor(a);
  if (s.cb == s.ca) { s.r = 0.5 * (a + b); s.drda = 0.5; s.drdb = 0.5; }
  else { s.r = (double)std::max(s.cb, s.ca); s.drda = 0.0; s.drdb = 0.0; }
  return s;
}

// The zigzag deposit of one particle with charge q: J(node) += ...; when g
// is given, also dS/da, dS/db for S = sum_nodes g.J.
void zigzag(const Grid& G, const Seg ax[3], const double b[3], const double a[3], double q, double rustep,
            double* J, const double* g, double dSda[3], double dSdb[3]) {
  // segment s = 0: b -> r in cell cb; s = 1: r -> a in cell ca
  for (int s = 0; s < 2; s++) {
    double F[3], d[3], dF_da[3], dF_db[3], dd_da[3], dd_db[3];
    int cell[3];
    for (int k = 0; k < 3; k++) {
      const Seg& z = ax[k];
      if (s == 0) {
        F[k] = (z.r - b[k]) * rustep;
        d[k] = 0.5 * (z.r + b[k]) - z.cb;
        dF_da[k] = z.drda * rustep; dF_db[k] = (z.drdb - 1.0) * rustep;
        dd_da[k] = 0.5 * z.drda; dd_db[k] = 0.5 * (z.drdb + 1.0);
        cell[k] = z.cb;
      } else {
        F[k] = (a[k] - z.r) * rustep;
        d[k] = 0.5 * (a[k] + z.r) - z.ca;
        dF_da[k] = (1.0 - z.drda) * rustep; dF_db[k] = -z.drdb * rustep;
        dd_da[k] = 0.5 * (1.0 + z.drda); dd_db[k] = 0.5 * z.drdb;
        cell[k] = z.ca;
      }
    }
    for (int comp = 0; comp < 3; comp++) {
      const int p1 = comp == 0 ? 1 : 0, p2 = comp == 2 ? 1 : 2;
      double Gv = 0.0, dG1 = 0.0, dG2 = 0.0;
      for (int e = 0; e < 4; e++) {
        const int u = e & 1, v = e >> 1;
        int o[3] = {cell[0], cell[1], cell[2]};
        o[p1] += u; o[p2] += v;
        const double W1 = u ? d[p1] : 1.0 - d[p1], W2 = v ? d[p2] : 1.0 - d[p2];
        const double D1 = u ? 1.0 : -1.0, D2 = v ? 1.0 : -1.0;
        const int64_t node = G.idx(o[0], o[1], o[2]);
        if (J) J[3 * node + comp] += q * F[comp] * W1 * W2;
        if (g) {
          const double gn = g[3 * node + comp];
          Gv += gn * W1 * W2;
          dG1 += gn * D1 * W2;
          dG2 += gn * W1 * D2;
        }
      }
      if (g) {
        // S += q * F[comp] * G(d[p1], d[p2])
        for (int k = 0; k < 3; k++) {
          dSda[k] += q * Gv * (k == comp ? dF_da[k] : 0.0);
          dSdb[k] += q * Gv * (k == comp ? dF_db[k] : 0.0);
        }
        dSda[p1] += q * F[comp] * dG1 * dd_da[p1];
        dSdb[p1] += q * F[comp] * dG1 * dd_db[p1];
        dSda[p2] += q * F[comp] * dG2 * dd_da[p2];
        dSdb[p2] += q * F[comp] * dG2 * dd_db[p2];
      }
    }
  }
}

struct Fwd {  // forward quantities of one particle-step
  double x1, y1, z1;
  int ci[3];
  V3 E, B, e, t, u, w, c, p, vnew;
  double s, qmp;
};

Fwd forward(const Grid& G, const double* en, const double* bn, const double e0b0[6], const double x[3], V3 v,
            double qmp) {
  Fwd f;
  for (int k = 0; k < 3; k++) f.ci[k] = (int)std::floor(x[k]);
  f.x1 = x[0] - f.ci[0]; f.y1 = x[1] - f.ci[1]; f.z1 = x[2] - f.ci[2];
  f.E = {e0b0[0], e0b0[1], e0b0[2]};
  f.B = {e0b0[3], e0b0[4], e0b0[5]};
  for (int c = 0; c < 8; c++) {
    int di, dj, dk;
    double w, gw[3];
    corner(c, f.x1, f.y1, f.z1, di, dj, dk, w, gw);
    const int64_t node = G.idx(f.ci[0] + di, f.ci[1] + dj, f.ci[2] + dk);
    f.E = f.E + w * V3{en[3 * node], en[3 * node + 1], en[3 * node + 2]};
    f.B = f.B + w * V3{bn[3 * node], bn[3 * node + 1], bn[3 * node + 2]};
  }
  f.qmp = qmp;
  f.e = qmp * f.E;
  f.t = qmp * f.B;
  f.s = 2.0 / (1.0 + dot(f.t, f.t));
  f.u = v + f.e;
  f.w = f.u + cross(f.u, f.t);
  f.c = cross(f.w, f.t);
  f.p = f.u + f.s * f.c;
  f.vnew = f.p + f.e;
  return f;
}

double wrap(double x, int n) {
  x = std::fmod(x, (double)n);
  if (x < 0) x += n;
  if (x >= n) x -= n;
  return x;
}

}  // namespace

// The zigzag current q * J(b -> a) of one segment on the periodic grid, added
// into J[nn][3] (node index i + nx*(j + ny*k)): b the start point, a the
// unwrapped end point.  The checker uses it to follow a particle that FP32
// rounding put on the other side of a cell face.
extern "C" void orc_zigzag_one(const emsesg_config* c, int ustep, double q, const double* b, const double* a,
                               double* J) {
  const Grid G{{c->nx, c->ny, c->nz}};
  const Seg ax[3] = {relay(b[0], a[0]), relay(b[1], a[1]), relay(b[2], a[2])};
  zigzag(G, ax, b, a, q, 1.0 / ustep, J, nullptr, nullptr, nullptr);
}

extern "C" double orc_adjoint_ckpt(const emsesg_config* c, int K, int ckpt, int ustep, const double* enode,
                                   const double* bnode, const double* e0b0, emsesg_particle* p, int64_t np,
                                   const int* probe_lo, const int* probe_hi, double* gE, double* gB, double* g0,
                                   double* gv) {
  const Grid G{{c->nx, c->ny, c->nz}};
  const int64_t nn = (int64_t)c->nx * c->ny * c->nz;
  const double rustep = 1.0 / ustep;
  const bool grad = gE != nullptr;
  if (ckpt < 1 || ckpt > K || K % ckpt != 0) ckpt = K;
  const int nseg = K / ckpt;
  // checkpoints (state before steps 0, ckpt, 2 ckpt, ...) and the states of
  // one segment, recomputed from its checkpoint in the reverse sweep
  std::vector<double> ckx((size_t)(grad ? nseg * np * 3 : 0)), ckv((size_t)(grad ? nseg * np * 3 : 0));
  std::vector<double> xs((size_t)(grad ? ckpt * np * 3 : 0)), vs((size_t)(grad ? ckpt * np * 3 : 0));
  std::vector<double> J((size_t)(3 * nn)), Jx((size_t)(grad ? K * nn : 0));
  auto probe = [&](int64_t node) {
    const int i = (int)(node % c->nx), j = (int)((node / c->nx) % c->ny), k = (int)(node / ((int64_t)c->nx * c->ny));
    return i >= probe_lo[0] && i < probe_hi[0] && j >= probe_lo[1] && j < probe_hi[1] && k >= probe_lo[2] &&
           k < probe_hi[2];
  };
  // one forward step of every particle of p in place; the states before it
  // go to (sx, sv) when given, the current into J when `deposit`
  auto step = [&](double* sx, double* sv, bool deposit) {
    if (deposit) std::memset(J.data(), 0, J.size() * sizeof(double));
    for (int64_t m = 0; m < np; m++) {
      emsesg_particle& q = p[m];
      const int is = q.spec - 1;
      const double x[3] = {q.x, q.y, q.z};
      if (sx) {
        for (int k = 0; k < 3; k++) sx[3 * m + k] = x[k];
        sv[3 * m + 0] = q.vx;
        sv[3 * m + 1] = q.vy;
        sv[3 * m + 2] = q.vz;
      }
      const Fwd f = forward(G, enode, bnode, e0b0, x, V3{q.vx, q.vy, q.vz}, c->qm[is] * ustep * 0.5);
      const double a[3] = {x[0] + f.vnew.x * ustep, x[1] + f.vnew.y * ustep, x[2] + f.vnew.z * ustep};
      if (deposit) {
        const Seg ax[3] = {relay(x[0], a[0]), relay(x[1], a[1]), relay(x[2], a[2])};
        zigzag(G, ax, x, a, c->q[is], rustep, J.data(), nullptr, nullptr, nullptr);
      }
      q.vx = f.vnew.x; q.vy = f.vnew.y; q.vz = f.vnew.z;
      q.x = wrap(a[0], c->nx); q.y = wrap(a[1], c->ny); q.z = wrap(a[2], c->nz);
    }
  };
  double loss = 0.0;
  for (int n = 0; n < K; n++) {
    double* sx = (grad && n % ckpt == 0) ? &ckx[(size_t)((n / ckpt) * np * 3)] : nullptr;
    double* sv = (grad && n % ckpt == 0) ? &ckv[(size_t)((n / ckpt) * np * 3)] : nullptr;
    step(sx, sv, true);
    for (int64_t node = 0; node < nn; node++)
      if (probe(node)) loss += J[3 * node] * J[3 * node];
    if (grad)
      for (int64_t node = 0; node < nn; node++) Jx[(size_t)(n * nn + node)] = J[3 * node];
  }
  if (!grad) return loss;
  // the state after K steps is given back at the end
  std::vector<emsesg_particle> pend(p, p + np);
  std::memset(gE, 0, 3 * nn * sizeof(double));
  std::memset(gB, 0, 3 * nn * sizeof(double));
  std::memset(g0, 0, 6 * sizeof(double));
  std::vector<double> lx((size_t)(3 * np), 0.0), lv((size_t)(3 * np), 0.0), gJ((size_t)(3 * nn), 0.0);
  for (int sg = nseg - 1; sg >= 0; sg--) {
    // recompute the segment's states from its checkpoint (moves only)
    for (int64_t m = 0; m < np; m++) {
      const double* x = &ckx[(size_t)((sg * np + m) * 3)];
      const double* v = &ckv[(size_t)((sg * np + m) * 3)];
      p[m].x = x[0]; p[m].y = x[1]; p[m].z = x[2];
      p[m].vx = v[0]; p[m].vy = v[1]; p[m].vz = v[2];
    }
    for (int j = 0; j < ckpt; j++) step(&xs[(size_t)(j * np * 3)], &vs[(size_t)(j * np * 3)], false);
  for (int j = ckpt - 1; j >= 0; j--) {
    const int n = sg * ckpt + j;
    for (int64_t node = 0; node < nn; node++) gJ[3 * node] = probe(node) ? 2.0 * Jx[(size_t)(n * nn + node)] : 0.0;
    for (int64_t m = 0; m < np; m++) {
      const int is = p[m].spec - 1;
      const double* x = &xs[(size_t)((j * np + m) * 3)];
      const double* v = &vs[(size_t)((j * np + m) * 3)];
      const Fwd f = forward(G, enode, bnode, e0b0, x, V3{v[0], v[1], v[2]}, c->qm[is] * ustep * 0.5);
      const double a[3] = {x[0] + f.vnew.x * ustep, x[1] + f.vnew.y * ustep, x[2] + f.vnew.z * ustep};
      const Seg ax[3] = {relay(x[0], a[0]), relay(x[1], a[1]), relay(x[2], a[2])};
      double dSda[3] = {0, 0, 0}, dSdb[3] = {0, 0, 0};
      zigzag(G, ax, x, a, c->q[is], rustep, nullptr, gJ.data(), dSda, dSdb);
      double* LX = &lx[(size_t)(3 * m)];
      double* LV = &lv[(size_t)(3 * m)];
      // a = b + v_{n+1}*ustep; x_{n+1} = wrap(a)
      const V3 la = {LX[0] + dSda[0], LX[1] + dSda[1], LX[2] + dSda[2]};
      const V3 lvnew = V3{LV[0], LV[1], LV[2]} + (double)ustep * la;
      V3 lb = V3{dSdb[0], dSdb[1], dSdb[2]} + la;
      // Boris, reversed: vnew = p + e; p = u + s*c; c = w x t; w = u + u x t; u = v + e
      V3 le = lvnew, lp = lvnew;
      V3 lu = lp;
      const double ls = dot(lp, f.c);
      const V3 lc = f.s * lp;
      const V3 lw = cross(f.t, lc);
      V3 lt = cross(lc, f.w);
      lu = lu + lw + cross(f.t, lw);
      lt = lt + cross(lw, f.u);
      lt = lt + (-ls * f.s * f.s) * f.t;
      const V3 lvold = lu;
      le = le + lu;
      const V3 lE = f.qmp * le, lB = f.qmp * lt;
      g0[0] += lE.x; g0[1] += lE.y; g0[2] += lE.z;
      g0[3] += lB.x; g0[4] += lB.y; g0[5] += lB.z;
      // gather, reversed
      for (int cc = 0; cc < 8; cc++) {
        int di, dj, dk;
        double w, gw[3];
        corner(cc, f.x1, f.y1, f.z1, di, dj, dk, w, gw);
        const int64_t node = G.idx(f.ci[0] + di, f.ci[1] + dj, f.ci[2] + dk);
        gE[3 * node] += w * lE.x; gE[3 * node + 1] += w * lE.y; gE[3 * node + 2] += w * lE.z;
        gB[3 * node] += w * lB.x; gB[3 * node + 1] += w * lB.y; gB[3 * node + 2] += w * lB.z;
        const V3 Ec = {enode[3 * node], enode[3 * node + 1], enode[3 * node + 2]};
        const V3 Bc = {bnode[3 * node], bnode[3 * node + 1], bnode[3 * node + 2]};
        const double s = dot(Ec, lE) + dot(Bc, lB);
        lb = lb + s * V3{gw[0], gw[1], gw[2]};
      }
      LX[0] = lb.x; LX[1] = lb.y; LX[2] = lb.z;
      LV[0] = lvold.x; LV[1] = lvold.y; LV[2] = lvold.z;
    }
  }
  }
  for (int64_t m = 0; m < np; m++)
    for (int k = 0; k < 3; k++) gv[3 * m + k] = lv[(size_t)(3 * m + k)];
  std::copy(pend.begin(), pend.end(), p);
  return loss;
}

extern "C" double orc_adjoint(const emsesg_config* c, int K, int ustep, const double* enode, const double* bnode,
                              const double* e0b0, emsesg_particle* p, int64_t np, const int* probe_lo,
                              const int* probe_hi, double* gE, double* gB, double* g0, double* gv) {
  return orc_adjoint_ckpt(c, K, K, ustep, enode, bnode, e0b0, p, np, probe_lo, probe_hi, gE, gB, g0, gv);
}
