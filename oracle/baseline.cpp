// baseline.cpp -- TEST INFRASTRUCTURE ONLY: the timed CPU baseline.
//
// The reference runs its particle step with one MPI rank per core, each rank
// owning a block of the grid with its own field arrays (OhHelp's subdomains,
// lib/ohhelp/ohhelp-1.1.1/ohhelp1.c) and pushing the particles that sit in
// it with psolve1 + charge (src/pcl2field/psolve1.F90:143-828,
// src/pcl2field/charge.F90:40-212).  This file models that on the host's
// threads: the particles given are split into blocks of whole x rows
// (ranges of y rows x ranges of z layers), one block per thread; a block has
// its own sub-grid (its cells plus `margin` cells on each split side), its
// own wrk (E/B copied from the global node field once, at set-up), aj and
// rho; every step each thread runs the oracle's orc_psolve1 (zigzag J) and
// orc_charge (func 0) on its block.  The per-particle arithmetic is the
// oracle's statement-for-statement restatement: positions are shifted by a
// whole number of cells into the sub-grid, which is exact in FP64.
//
// A step may start from the block's initial particles (restored before the
// timer starts), so that every timed step is the same bounded sample of the
// workload, or go on from the last one.  The exchange of guard layers
// between ranks is not timed (it costs the reference a surface's worth of
// data per step).
// orc_blocks_result adds the blocks' aj / rho into the global periodic
// arrays (interior nodes), which lets tests compare this path with the
// single-threaded oracle.
#include <chrono>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "emses_oracle.h"

namespace {

struct Block {
  emsesg_config c;                  // the block's sub-grid
  int y0, z0;                       // global index of the sub-grid's node 0
  int64_t np;                       // particles of the block
  int64_t tp[EMSESG_ISPEC];
  std::vector<emsesg_particle> p0;  // initial state
  std::vector<emsesg_particle> p;   // state of the step
  std::vector<double> wrk, aj, rho;
};

// Index of a FAJ / FRH / wrk layout: nc components, lower guard lo, extents.
struct Lay {
  int nc, lo, ex, ey, ez;
  int64_t at(int c, int i, int j, int k) const {
    return c + (int64_t)nc * ((i - lo) + (int64_t)ex * ((j - lo) + (int64_t)ey * (k - lo)));
  }
};
Lay lay_wrk(const emsesg_config& c) { return {9, -4, c.nx + 9, c.ny + 9, c.nz + 9}; }
Lay lay_aj(const emsesg_config& c) { return {3, -4, c.nx + 9, c.ny + 9, c.nz + 9}; }
Lay lay_rho(const emsesg_config& c) { return {1, -1, c.nx + 3, c.ny + 3, c.nz + 3}; }

inline int wrapi(int a, int n) { return ((a % n) + n) % n; }

template <class F>
void parallel(int n, F f) {
  std::vector<std::thread> pool;
  for (int t = 1; t < n; t++) pool.emplace_back(f, t);
  f(0);
  for (auto& th : pool) th.join();
}

}  // namespace

struct orc_blocks {
  emsesg_config c;  // the global grid
  std::vector<Block> b;
};

extern "C" {

orc_blocks* orc_blocks_create(const emsesg_config* c, const double* wrk, const emsesg_particle* p,
                              const int64_t* totalp, int threads, int margin) {
  auto* h = new orc_blocks;
  h->c = *c;
  int64_t n = 0;
  for (int is = 0; is < c->nspec; is++) n += totalp[is];
  // the z layers and y rows the particles occupy
  int kmin = c->nz, kmax = -1, jmin = c->ny, jmax = -1;
  for (int64_t m = 0; m < n; m++) {
    int k = (int)std::floor(p[m].z), j = (int)std::floor(p[m].y);
    kmin = std::min(kmin, k); kmax = std::max(kmax, k);
    jmin = std::min(jmin, j); jmax = std::max(jmax, j);
  }
  if (n == 0) { kmin = kmax = jmin = jmax = 0; }
  const int nzl = kmax - kmin + 1, nyl = jmax - jmin + 1;
  if (threads < 1) threads = 1;
  const int zs = std::min(threads, nzl);
  const int ys = std::max(1, std::min(threads / zs, nyl));
  const Lay gw = lay_wrk(*c);
  for (int bz = 0; bz < zs; bz++)
    for (int by = 0; by < ys; by++) {
      Block B;
      const int za = kmin + (int)((int64_t)nzl * bz / zs), zb = kmin + (int)((int64_t)nzl * (bz + 1) / zs);
      const int ya = jmin + (int)((int64_t)nyl * by / ys), yb = jmin + (int)((int64_t)nyl * (by + 1) / ys);
      const bool fully = (yb - ya) == c->ny, fullz = (zb - za) == c->nz;
      B.c = *c;
      B.c.ny = fully ? c->ny : (yb - ya) + 2 * margin;
      B.c.nz = fullz ? c->nz : (zb - za) + 2 * margin;
      B.y0 = fully ? 0 : ya - margin;
      B.z0 = fullz ? 0 : za - margin;
      // the block's particles, per species, shifted into the sub-grid
      B.np = 0;
      int64_t base = 0;
      for (int is = 0; is < c->nspec; is++) {
        int64_t cnt = 0;
        for (int64_t m = base; m < base + totalp[is]; m++) {
          const int k = (int)std::floor(p[m].z), j = (int)std::floor(p[m].y);
          if (k < za || k >= zb || j < ya || j >= yb) continue;
          emsesg_particle q = p[m];
          q.y -= (double)B.y0;
          q.z -= (double)B.z0;
          B.p0.push_back(q);
          cnt++;
        }
        B.tp[is] = cnt;
        B.np += cnt;
        base += totalp[is];
      }
      for (int is = c->nspec; is < EMSESG_ISPEC; is++) B.tp[is] = 0;
      B.p = B.p0;
      // E/B of the sub-grid's nodes from the global node field (periodic)
      const Lay w = lay_wrk(B.c);
      B.wrk.assign((size_t)w.nc * w.ex * w.ey * w.ez, 0.0);
      for (int k = -4; k <= B.c.nz + 4; k++)
        for (int j = -4; j <= B.c.ny + 4; j++)
          for (int i = -4; i <= B.c.nx + 4; i++) {
            const int gi = wrapi(i, c->nx), gj = wrapi(j + B.y0, c->ny), gk = wrapi(k + B.z0, c->nz);
            for (int q = 0; q < 6; q++) B.wrk[w.at(q, i, j, k)] = wrk[gw.at(q, gi, gj, gk)];
          }
      const Lay a = lay_aj(B.c), r = lay_rho(B.c);
      B.aj.assign((size_t)a.nc * a.ex * a.ey * a.ez, 0.0);
      B.rho.assign((size_t)r.nc * r.ex * r.ey * r.ez, 0.0);
      h->b.push_back(std::move(B));
    }
  return h;
}

int orc_blocks_threads(const orc_blocks* h) { return (int)h->b.size(); }

int64_t orc_blocks_particles(const orc_blocks* h) {
  int64_t n = 0;
  for (const Block& B : h->b) n += B.np;
  return n;
}

// One step of every block, from its initial particles when `restore` (the
// restore runs before the timer) or else from where the last step left
// them; returns the wall time of psolve1 + charge on all threads.
double orc_blocks_step(orc_blocks* h, int ustep, int restore) {
  const int nt = (int)h->b.size();
  if (restore)
    parallel(nt, [&](int t) {
      Block& B = h->b[t];
      std::memcpy(B.p.data(), B.p0.data(), B.p0.size() * sizeof(emsesg_particle));
    });
  const auto t0 = std::chrono::steady_clock::now();
  parallel(nt, [&](int t) {
    Block& B = h->b[t];
    std::fill(B.aj.begin(), B.aj.end(), 0.0);
    std::fill(B.rho.begin(), B.rho.end(), 0.0);
    emsesg_counter gc;
    std::memset(&gc, 0, sizeof(gc));
    int64_t pos = 0;
    orc_psolve1(&B.c, ustep, 0, B.wrk.data(), B.p.data(), B.tp, nullptr, 0, &pos, 0, B.aj.data(), nullptr, &gc,
                nullptr);
    orc_charge(&B.c, 0, B.p.data(), B.tp, B.rho.data(), nullptr, nullptr, nullptr);
  });
  const auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

// The blocks' aj and rho of the last step added into the global arrays
// (layouts of the global grid, zeroed here) at the interior nodes 0..n-1,
// every sub-grid node wrapped periodically: the guard fold of a periodic
// run.
void orc_blocks_result(const orc_blocks* h, double* aj, double* rho) {
  const emsesg_config& c = h->c;
  const Lay ga = lay_aj(c), gr = lay_rho(c);
  std::memset(aj, 0, sizeof(double) * (size_t)ga.nc * ga.ex * ga.ey * ga.ez);
  std::memset(rho, 0, sizeof(double) * (size_t)gr.nc * gr.ex * gr.ey * gr.ez);
  for (const Block& B : h->b) {
    const Lay a = lay_aj(B.c), r = lay_rho(B.c);
    for (int k = -4; k <= B.c.nz + 4; k++)
      for (int j = -4; j <= B.c.ny + 4; j++)
        for (int i = -4; i <= B.c.nx + 4; i++) {
          const int gi = wrapi(i, c.nx), gj = wrapi(j + B.y0, c.ny), gk = wrapi(k + B.z0, c.nz);
          for (int q = 0; q < 3; q++) aj[ga.at(q, gi, gj, gk)] += B.aj[a.at(q, i, j, k)];
          if (i >= -1 && j >= -1 && k >= -1 && i <= B.c.nx + 1 && j <= B.c.ny + 1 && k <= B.c.nz + 1)
            rho[gr.at(0, gi, gj, gk)] += B.rho[r.at(0, i, j, k)];
        }
  }
}

void orc_blocks_destroy(orc_blocks* h) { delete h; }

}  // extern "C"
