/*
 * emses_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU FP64 restatement of the reference's particle hot path, written
 * statement for statement from the Fortran sources and used only as the
 * checker of the CUDA path (by tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arm of bench.py).  Nothing in the product links
 * or calls it.
 *
 * Parity status: the reference Fortran cannot be compiled in this
 * environment (no Fortran compiler, MPI, HDF5 or FFTW), and the reference
 * has no tests or golden vectors for this path.  The parts of the reference
 * that are C (lib/mtarm/mt19937arm.c, lib/psort/psort-struct.c) are compiled
 * from their own sources into oracle/_ref and checked against this file;
 * the Fortran statements are pinned by the golden fixtures that
 * tests/golden/make_golden.py produces by executing the reference's own
 * Fortran source text with a small interpreter (see that script).
 *
 * Arithmetic: IEEE FP64, no FMA contraction (-ffp-contract=off), Fortran
 * left-to-right expression order.  Fortran int() truncates toward zero,
 * floor() rounds down; both are kept where the reference uses them.
 */
#ifndef EMSES_ORACLE_H
#define EMSES_ORACLE_H
#include "../include/emses_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Size in doubles of a field array (same layouts as emses_gpu.h). */
int64_t orc_field_size(const emsesg_config* c, int field);

/* Single-rank guard fill of eb (oh3_exchange_borders with CEB), periodic axes. */
void orc_exchange_eb(const emsesg_config* c, double* eb);
// bfield, src/field/bfield.F90:37-53: B += curl-E step (half time step).
void orc_bfield(const emsesg_config* c, double* eb);
// efield, src/field/efield.F90:54-70 (no lumped elements): E += tcs curl B - dlt J.
void orc_efield(const emsesg_config* c, double* eb, const double* aj, double tcs, double dlt);

void orc_grdcrt(const emsesg_config* c, const double* eb, double* wrk);

/* Random numbers for injected particles: rng_mode 1 consumes ranu[*ranu_pos]
 * in buffer order; rng_mode 0 uses the counter hash of (seed, stream, m). */
int orc_psolve2(const emsesg_config* c, int ustep, const double* wrk,
                emsesg_particle* pbuf, const int64_t* totalp, const double* ranu,
                int64_t nranu, int64_t* ranu_pos, uint64_t rng_stream,
                emsesg_counter* gc);
int orc_positn(const emsesg_config* c, int ustep, emsesg_particle* pbuf, const int64_t* totalp,
               const double* ranu, int64_t nranu, int64_t* ranu_pos, uint64_t rng_stream,
               emsesg_counter* gc);
int orc_psolve1(const emsesg_config* c, int ustep, int func, double* wrk,
                emsesg_particle* pbuf, const int64_t* totalp, const double* ranu,
                int64_t nranu, int64_t* ranu_pos, uint64_t rng_stream,
                double* aj, double* ajdg, emsesg_counter* gc, int64_t* surf);
/* Per-surface-cell counts of box bodies (geotype 0/1, integer bounds):
 * layout (faces -x,+x,-y,+y,-z,+z per body, first tangential axis fastest)
 * and the cell of an entering particle (b -> a) or of a point on a face.
 * surf in orc_psolve1 may be NULL; else [nspec][nsurf] counts are added. */
int64_t orc_surface_layout(const emsesg_config* c, int64_t* offsets);
int64_t orc_surface_cell(const emsesg_config* c, int ipc, const double* b, const double* a);
int64_t orc_surface_point(const emsesg_config* c, int ipc, const double* p);
/* Background charge from the surface counts surf[nspec][nsurf]: rhobk
 * (node field, rho layout) and rho(0:n) += rhobk, or = rhobk with
 * `replace` (add_background_charge, charge.F90:414-449). */
void orc_background(const emsesg_config* c, const int64_t* surf, double* rhobk, double* rho, int replace);
void orc_charge(const emsesg_config* c, int func, emsesg_particle* pbuf,
                const int64_t* totalp, double* rho, double* rhodg, double* rhobk,
                double* rhobksp);
/* oh3_exchange_borders(CRH) + add_boundary_charge on an array of ncomp
 * components with the rho layout. */
void orc_reduce_rho(const emsesg_config* c, double* rh, int ncomp);
/* oh3_exchange_borders(CAJ) + add_boundary_current; ncomp = 3. */
void orc_reduce_aj(const emsesg_config* c, double* aj);
/* oh3_exchange_borders(CJD) + add_boundary_current2; ncomp = 3*nspec. */
void orc_reduce_ajdg(const emsesg_config* c, double* ajdg);
void orc_rhoupd(const emsesg_config* c, double* rho, const double* aj);
void orc_energy(const emsesg_config* c, const emsesg_particle* pbuf,
                const int64_t* totalp, double* engk);

/* Canonical sort key of a particle and the stable sort by it. */
int64_t orc_sort_key(const emsesg_config* c, const emsesg_particle* p);
void orc_spsort(const emsesg_config* c, emsesg_particle* pbuf, const int64_t* totalp);
void orc_compact(const emsesg_config* c, emsesg_particle* pbuf, int64_t* totalp);

/* Counter hash used for injected particles (rng_mode 0). */
double orc_hash_u01(uint64_t seed, uint64_t stream, uint64_t index);

/* Synthetic plasma loader, same hash streams as emsesg_load_plasma. */
void orc_load_plasma(const emsesg_config* c, const emsesg_plasma* pl,
                     emsesg_particle* pbuf, int64_t* totalp);

/* Timed CPU baseline in the reference's one-rank-per-core model
 * (baseline.cpp): the particles are split into blocks of x rows (y rows x z
 * layers), one per thread, each with its own sub-grid (margin cells on its
 * split sides), wrk, aj and rho; a step runs orc_psolve1 + orc_charge on
 * every block in parallel (from the blocks' initial particles when
 * `restore`) and returns the wall time.  orc_blocks_result sums the blocks' aj / rho into the global
 * periodic arrays (interior nodes). */
typedef struct orc_blocks orc_blocks;
orc_blocks* orc_blocks_create(const emsesg_config* c, const double* wrk, const emsesg_particle* p,
                              const int64_t* totalp, int threads, int margin);
int orc_blocks_threads(const orc_blocks* h);
int64_t orc_blocks_particles(const orc_blocks* h);
double orc_blocks_step(orc_blocks* h, int ustep, int restore);
void orc_blocks_result(const orc_blocks* h, double* aj, double* rho);
void orc_blocks_destroy(orc_blocks* h);

/* Loss sum_steps sum_probe Jx^2 of K periodic steps and, when gE is not
 * NULL, its gradients with respect to the node fields (gE, gB: [n^3][3],
 * x fastest), the uniform e0 / b0 (g0[6]) and the initial velocities
 * (gv[np][3]); particles are advanced in place.  Node fields exclude e0/b0.
 * adjoint.cpp. */
double orc_adjoint(const emsesg_config* c, int K, int ustep, const double* enode, const double* bnode,
                   const double* e0b0, emsesg_particle* p, int64_t np, const int* probe_lo,
                   const int* probe_hi, double* gE, double* gB, double* g0, double* gv);
/* q * the zigzag current of one segment b -> a (a unwrapped) on the periodic
 * grid, added into J[nn][3] (x fastest). */
void orc_zigzag_one(const emsesg_config* c, int ustep, double q, const double* b, const double* a, double* J);
/* The same with the state kept every ckpt steps (K a multiple of ckpt) and
 * each segment recomputed in the reverse sweep; same result. */
double orc_adjoint_ckpt(const emsesg_config* c, int K, int ckpt, int ustep, const double* enode,
                        const double* bnode, const double* e0b0, emsesg_particle* p, int64_t np,
                        const int* probe_lo, const int* probe_hi, double* gE, double* gB, double* g0, double* gv);

#ifdef __cplusplus
}
#endif
#endif
