/*
 * emses_gpu.h -- C ABI of the B200 (sm_100a) particle hot path of EMSES
 * (MPIEMSES3D): Buneman-Boris push with trilinear E/B gather and
 * boundary/body handling, the particle cell sort, CIC charge deposition and
 * the charge-conserving zigzag current deposition.
 *
 * The entry points keep the argument meaning of the reference's external
 * Fortran subroutines so that an ISO_C_BINDING shim with the same subroutine
 * names (grdcrt, psolve1, psolve2, charge, spsort) can forward to them:
 *
 *   emsesg_grdcrt    <- subroutine grdcrt(ps)            src/field/grdcrt.F90:125
 *   emsesg_psolve2   <- subroutine psolve2(ps, ustep)     src/pcl2field/psolve2.F90:4
 *   emsesg_psolve1   <- subroutine psolve1(ps,ustep,func) src/pcl2field/psolve1.F90:4
 *   emsesg_positn    <- subroutine positn(ps, ustep)     src/pcl/positn.F90:3
 *   emsesg_charge    <- subroutine charge(ps, func)       src/pcl2field/charge.F90:4
 *   emsesg_spsort    <- subroutine spsort(ps)             src/etc/spsort.F90:4
 *                       (and the C symbol particle_sort_,  lib/psort/psort-struct.c:7)
 *   emsesg_compact   <- single-rank part of oh3_transbound
 *                       lib/ohhelp/ohhelp-1.1.1/ohhelp2.c:103-123
 *   emsesg_reduce_rho / emsesg_reduce_aj / emsesg_reduce_ajdg
 *                    <- oh3_exchange_borders (ohhelp3.c:1011) on one rank
 *                       followed by add_boundary_charge (charge.F90:214),
 *                       add_boundary_current (psolve1.F90:859) and
 *                       add_boundary_current2 (psolve1.F90:1081)
 *   emsesg_rhoupd    <- subroutine rhoupd(ps)             src/field/rhoupd.F90:4
 *   emsesg_energy    <- kinetic part of energy            src/etc/energy.F90:29-47
 *
 * Single rank, one GPU: ps must be 1 (the helper subdomain ps=2 of OhHelp is
 * not supported and returns EMSESG_ERR_UNSUPPORTED).  There is no CPU
 * fallback: every compute entry point launches CUDA kernels.
 *
 * Data ownership: the context owns persistent device mirrors of pbuf, eb,
 * wrk, rho, rhodg, rhobk, rhobksp, aj and ajdg.  Between calls the device
 * copy is authoritative; host arrays are read or written only by the
 * explicit upload/download calls.  Compute calls are asynchronous on the
 * context's CUDA stream, except where a host output argument is given.
 *
 * Array layouts are the reference's Fortran (column-major) layouts with the
 * guard extents that OhHelp gives them (ohhelp3.c:439-477, ftypes/ctypes in
 * src/wrapper/ohinit.F90:98-122), for a subdomain of nx*ny*nz cells:
 *
 *   eb     (6,        -1:nx+1, -1:ny+1, -1:nz+1)   EMSESG_FIELD_EB
 *   wrk    (9,        -4:nx+4, -4:ny+4, -4:nz+4)   EMSESG_FIELD_WRK
 *   aj     (3,        -4:nx+4, -4:ny+4, -4:nz+4)   EMSESG_FIELD_AJ
 *   ajdg   (3*nspec,  -4:nx+4, -4:ny+4, -4:nz+4)   EMSESG_FIELD_AJDG
 *   rho    (1,        -1:nx+1, -1:ny+1, -1:nz+1)   EMSESG_FIELD_RHO
 *   rhodg  (2*nspec+1,-1:nx+1, -1:ny+1, -1:nz+1)   EMSESG_FIELD_RHODG
 *   rhobk  (1,        -1:nx+1, -1:ny+1, -1:nz+1)   EMSESG_FIELD_RHOBK
 *   rhobksp(1,        -1:nx+1, -1:ny+1, -1:nz+1, nspec) EMSESG_FIELD_RHOBKSP
 *   phi    (1,        -1:nx+1, -1:ny+1, -1:nz+1)   EMSESG_FIELD_PHI
 *
 * Error convention: every function returns an int status (EMSESG_OK == 0);
 * none of them exits, aborts or traps.  emsesg_last_error() gives the text.
 * A context is not thread-safe; use one context per host thread.
 */
#ifndef EMSES_GPU_H
#define EMSES_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Array caps of the reference, src/main/paramt.F90:55-60 (ispec, inpc). */
#define EMSESG_ISPEC 10
#define EMSESG_INPC 15

/* Status codes. */
#define EMSESG_OK 0
#define EMSESG_ERR_ARG 1          /* bad argument or configuration */
#define EMSESG_ERR_UNSUPPORTED 2  /* ps=2, disabled physics options */
#define EMSESG_ERR_CUDA 3         /* a CUDA runtime call failed */
#define EMSESG_ERR_OVERFLOW 4     /* particle capacity exceeded */
#define EMSESG_ERR_NOMEM 5        /* device allocation failed */
#define EMSESG_ERR_TIMEOUT 6      /* a bounded device wait gave up */
#define EMSESG_ERR_DEVICE 7       /* a kernel reported a bad index */
#define EMSESG_ERR_STATE 8        /* call out of order (e.g. no fixed state) */

/* Particle states, lib/ohhelp/ohhelp-1.1.1/oh_type.F90:31-34. */
#define EMSESG_PCL_ALIVE 0
#define EMSESG_PCL_INJECTED 1
#define EMSESG_PCL_TO_BE_ACCUMULATED (-1)
#define EMSESG_PCL_TO_BE_ACCUMULATED_AS_ANTIPCL (-2)

/* Field identifiers for upload/download. */
#define EMSESG_FIELD_EB 0
#define EMSESG_FIELD_WRK 1
#define EMSESG_FIELD_AJ 2
#define EMSESG_FIELD_AJDG 3
#define EMSESG_FIELD_RHO 4
#define EMSESG_FIELD_RHODG 5
#define EMSESG_FIELD_RHOBK 6
#define EMSESG_FIELD_RHOBKSP 7
#define EMSESG_FIELD_PHI 8
#define EMSESG_NFIELDS 9

/* The OhHelp particle record oh_particle (oh_type.F90:15-28, oh_part.h:23-28,
 * OH_BIG_SPACE off): 64 bytes. */
typedef struct emsesg_particle {
  double x, y, z, vx, vy, vz;
  int32_t pid;
  int32_t preside;
  int32_t nid;
  int32_t spec;
} emsesg_particle;

/* The Fortran sequence type `counter` (src/main/paramt.F90:76-83) with the
 * same memory layout: Fortran (a,b,c) arrays appear as C [c][b][a]. */
typedef struct emsesg_counter {
  int64_t globalp[2][EMSESG_ISPEC];
  int32_t influx[EMSESG_ISPEC][EMSESG_INPC];
  int32_t outflux[EMSESG_ISPEC][EMSESG_INPC];
  int32_t infhist[EMSESG_ISPEC][EMSESG_INPC][EMSESG_INPC + 1];
  int32_t nesc[(EMSESG_ISPEC + 1) / 2 * 2];
  double chgacm[EMSESG_INPC][2];
} emsesg_counter;

/* One internal body (&ptcond), as tested by psolve2.F90:465-531. */
typedef struct emsesg_body {
  int32_t geotype;   /* 0 or 1: box; 2: cylinder; 3: sphere; <0: none */
  int32_t ncond;     /* >0: conductor, chgacm is accumulated */
  int32_t cyl_align; /* cylinder axis 1=x 2=y 3=z */
  int32_t reserved_;
  double xlpc, xupc, ylpc, yupc, zlpc, zupc; /* box bounds, inclusive */
  double cyl_axis[2];
  double cyl_edge[2];
  double radius;     /* cylinder / sphere radius */
  double sph_center[3];
  double sqdscaled;  /* chgacm weight (allcom.F90:132) */
} emsesg_body;

/* Run configuration in the reference's internal units (rescal.F90:47-81). */
typedef struct emsesg_config {
  int32_t nx, ny, nz;               /* subdomain cells = sdoms(2,d)-sdoms(1,d) */
  int32_t nspec;                    /* number of species, <= EMSESG_ISPEC */
  int32_t nfbnd[3];                 /* field BC per axis: 0 periodic */
  int32_t npbnd[EMSESG_ISPEC][3];   /* particle BC per species, axis: 0 wrap,
                                       1 reflect, 2 escape (npbnd(3,ispec)) */
  int32_t npc;                      /* number of bodies, <= EMSESG_INPC */
  int32_t line_mode;                /* 1 disables the body test */
  int32_t rng_mode;                 /* 0 counter hash, 1 pre-drawn uniforms */
  int32_t sort_tile[3];             /* cell tile of the sort key (0: whole grid) */
  int32_t flags;                    /* EMSESG_FLAG_* (0: none) */
  uint64_t rng_seed;                /* seed of the counter hash */
  double q[EMSESG_ISPEC];           /* charge per macro-particle */
  double qm[EMSESG_ISPEC];          /* charge-to-mass ratio */
  double rm[EMSESG_ISPEC];          /* mass (energy.F90:44) */
  double e0[3], b0[3];              /* background fields added by grdcrt */
  emsesg_body body[EMSESG_INPC];
  int64_t capacity[EMSESG_ISPEC];   /* device particle capacity per species */
} emsesg_config;

/* Config flags.  EMSESG_FLAG_FP32_ONLY: the context keeps no FP64 particle
 * buffer (64 bytes a particle); particles live in the FP32 form only, loaded
 * by emsesg_fx_load_plasma and added by emsesg_fx_inject, so that runs of
 * some 1.6e9 particles fit one GPU.  The calls that move FP64 particle
 * records (emsesg_upload/download_particles, emsesg_load_plasma,
 * emsesg_fx_load, emsesg_fx_store) then return EMSESG_ERR_STATE. */
#define EMSESG_FLAG_FP32_ONLY 1

typedef struct emsesg_ctx emsesg_ctx;

/* ---- context ------------------------------------------------------------ */
/* Makes `device` the CUDA device of the contexts created next by this host
 * thread (one process per GPU: call it with the local rank). */
int emsesg_select_device(int device);
int emsesg_create(const emsesg_config* cfg, emsesg_ctx** out);
int emsesg_destroy(emsesg_ctx* ctx);
/* Copies the last error text (NUL-terminated) into buf. */
int emsesg_last_error(const emsesg_ctx* ctx, char* buf, size_t len);
/* The context's cudaStream_t, as an opaque pointer. */
void* emsesg_stream(emsesg_ctx* ctx);
int emsesg_synchronize(emsesg_ctx* ctx);
/* Number of doubles of a field array in the layout above. */
int emsesg_field_size(const emsesg_ctx* ctx, int field, int64_t* ndoubles);

/* ---- explicit sync points (host <-> device) ---------------------------- */
/* pbuf holds the species segments back to back (pbase = 0); totalp[is] is
 * the count of species is (totalp(is,ps)). */
int emsesg_upload_particles(emsesg_ctx* ctx, int ps, const emsesg_particle* pbuf,
                            const int64_t* totalp);
int emsesg_download_particles(emsesg_ctx* ctx, int ps, emsesg_particle* pbuf,
                              int64_t* totalp);
int emsesg_upload_field(emsesg_ctx* ctx, int field, const double* host);
int emsesg_download_field(emsesg_ctx* ctx, int field, double* host);
/* Sets a whole field array to 0.0, as `aj(:,:,:,:,1:2) = 0.0d0` at the start
 * of a step (src/main/esses.F90:318-321, src/pcl/psuper1.F90:88-90). */
int emsesg_zero_field(emsesg_ctx* ctx, int field);
/* Counters (gcount(1)): set before a push, read after it. */
int emsesg_set_counters(emsesg_ctx* ctx, const emsesg_counter* gcount);
int emsesg_get_counters(emsesg_ctx* ctx, emsesg_counter* gcount);
/* Pre-drawn U[0,1) numbers for injected particles (rng_mode 1): the k-th
 * injected particle met by a push, in buffer order, takes u[k]; the index
 * carries over from call to call until emsesg_set_randoms is called again. */
int emsesg_set_randoms(emsesg_ctx* ctx, const double* u, int64_t n);

/* ---- the reference subroutines (plain FP64 drop-in) --------------------- */
int emsesg_grdcrt(emsesg_ctx* ctx, int ps);
/* gcount may be NULL: counters then stay on the device (emsesg_get_counters). */
int emsesg_psolve2(emsesg_ctx* ctx, int ps, int ustep, emsesg_counter* gcount);
/* Position-only advance of the initial state (no fields, no deposit). */
int emsesg_positn(emsesg_ctx* ctx, int ps, int ustep, emsesg_counter* gcount);
int emsesg_psolve1(emsesg_ctx* ctx, int ps, int ustep, int func,
                   emsesg_counter* gcount);
int emsesg_charge(emsesg_ctx* ctx, int ps, int func);
int emsesg_reduce_rho(emsesg_ctx* ctx, int field);
int emsesg_reduce_aj(emsesg_ctx* ctx);
int emsesg_reduce_ajdg(emsesg_ctx* ctx);
int emsesg_spsort(emsesg_ctx* ctx, int ps);
/* Drops particles with nid == -1, keeps species segments contiguous and the
 * survivors in buffer order; totalp (may be NULL) receives the new counts. */
int emsesg_compact(emsesg_ctx* ctx, int ps, int64_t* totalp);
int emsesg_rhoupd(emsesg_ctx* ctx, int ps);

/* Compaction that allocates nothing (no counterpart in the reference).  For
 * hosts that cannot call cudaMalloc (device memory owned by their own pool or
 * framework): copies the particles of d_in[0..n) with nid != -1, in buffer
 * order, into d_out and writes their number to *d_kept; all three are device
 * pointers owned by the caller and must not overlap (EMSESG_ERR_ARG).  No
 * context is needed.  Scratch is a fixed file-scope device array, so
 * n <= EMSESG_NOALLOC_MAX_PARTICLES (else EMSESG_ERR_ARG), every GPU that
 * loads the library holds it (about 4 MB) until exit, and calls whose kernels
 * overlap on a GPU race on it: order them on one stream.  Each call outside a
 * stream capture looks up the scratch address of the current device; a call
 * inside a capture reuses the last one, so make the first call on a device
 * before any stream capture.  A CUDA error left pending by earlier work is
 * not consumed.  Asynchronous on `stream` (a cudaStream_t, NULL = default). */
#define EMSESG_NOALLOC_MAX_PARTICLES (1 << 20)
int emsesg_compact_noalloc(const emsesg_particle* d_in, int64_t n, emsesg_particle* d_out, int64_t* d_kept,
                           void* stream);
/* The EM field step around the push (src/main/emses.F90:365-430, 536-540):
 * bfield (src/field/bfield.F90:4) advances B by half a step from E;
 * efield (src/field/efield.F90:4, no lumped elements) advances E from B and
 * the reduced aj, E += tcs curl B - dlt J (tcs of inital.F90:78 /
 * rescal.F90:132; dlt = 2, or 0 for test-particle runs); exchange_eb is
 * oh3_exchange_borders(eb, CEB) on one rank.  FP64 on the eb mirror,
 * bit-identical to the reference's statement order. */
int emsesg_bfield(emsesg_ctx* ctx, int ps);
int emsesg_efield(emsesg_ctx* ctx, int ps, double tcs, double dlt);
int emsesg_exchange_eb(emsesg_ctx* ctx);
/* One EM step of the FP32 form with the fields on the device (periodic
 * fields, no bodies): bfield, emsesg_fx_step (push, J, rho), bfield,
 * efield, exchange_eb -- the order of the reference's main loop. */
int emsesg_fx_em_step(emsesg_ctx* ctx, int ustep, int do_sort, double tcs);

/* emsesg_esfield: the electrostatic field from rho on the device.
 * Replaces esfld1(0) with poisson(3) (src/field/esfild.F90:5-236,
 * src/field/poisson/poissn.F90:4-890 with the set-up of
 * src/field/poisson/inifft.F90:389-470), the guards of phi and esfld2
 * (src/field/esfild.F90:351-435).  mtd_vbnd[3] (x, y, z; NULL: all 0) is the
 * reference's Poisson boundary per axis: 0 periodic (nodes 0..n-1 solved),
 * 1 phi = 0 on the faces (nodes 1..n-1), 2 Neumann (nodes 0..n, with
 * bcond[2 axis + side] = boundary_conditions(side+1, axis+1) * rene added as
 * -2 bcond on the node-0 plane and +2 bcond on the node-n plane of rho;
 * bcond NULL: zeros).  phi (EMSESG_FIELD_PHI, nodes -1..n+1) solves
 * rho + (sum of the six neighbours of phi) - 6 phi = 0 on the solved nodes
 * (less the mean when no axis has a face), by cuFFT transforms divided by
 * the reference's eigenvalues -- (2 sin(pi m / n))^2 on periodic axes,
 * 2 (1 - cos(i pi / n)) on the others -- and mfactor (n per periodic axis,
 * 2n per other); it is zero outside the solved nodes and keeps the periodic
 * copies on periodic axes.  EX..EZ of eb become (phi(i) - phi(i+1)) * mltstp
 * on their staggered positions and zero elsewhere, the normal component at
 * -1 and n copied from 0 and n-1 on a mtd_vbnd 1 axis and negated on a 2
 * axis; BX..BZ are left as they are.  FP64.  With resid non-null it also
 * returns poichk's residual (src/field/poisson/poissn.F90:921-961):
 * sqrt(sum of (rho + sum of neighbours - 6 phi)^2 over its nodes -- the
 * solved ones up to n-1 -- ) divided by their count (synchronises).
 * Asynchronous otherwise. */
int emsesg_esfield(emsesg_ctx* ctx, const int* mtd_vbnd, const double* bcond, int mltstp, double* resid);
/* engk[is*3 + d] = 0.5*rm(is)*sum(v_d^2)/(slx*sly*slz), FP64. */
int emsesg_energy(emsesg_ctx* ctx, double* engk);

/* ---- FP32 / fixed-point form -------------------------------------------
 * Particle state as SoA {packed int32 cell, 3 x FP32 in-cell offset,
 * 3 x FP32 velocity} = 28 bytes, species segments, sorted by the tile-major
 * cell key.  rho and J accumulate in int64 fixed point (scale 2^40), so the
 * sums do not depend on the order in which threads add them. */
/* Converts the FP64 pbuf mirror into the FP32 form and sorts it. */
/* Slots per row of the FP32 form's thread-major tile regions: after a sort
 * the particle of sorted rank q of a tile of n particles sits in row q % L,
 * column q / L of its region, L = ceil(n / EMSESG_FX_ROW_SLOTS). */
#define EMSESG_FX_ROW_SLOTS 736
int emsesg_fx_load(emsesg_ctx* ctx);
/* Converts the FP32 form back into the FP64 pbuf mirror (for download), in
 * the current buffer order; particles that died since the last sort come
 * out in place with nid = -1. */
int emsesg_fx_store(emsesg_ctx* ctx);
/* One step of the FP32 form: push of the tile regions and of the tail zone,
 * zigzag J and CIC rho into int64 fixed point, guard folds, FP64 rho / aj;
 * with do_sort, the re-sort after the push. */
int emsesg_fx_step(emsesg_ctx* ctx, int ustep, int do_sort);
int emsesg_fx_sort(emsesg_ctx* ctx);
/* emsesg_fx_step followed by the downloads of rho and aj (the arrays a field
 * solver takes), made on a side stream as soon as the step's fields are
 * final, so that they overlap with the re-sort; returns once rho and aj are
 * in host memory (pinned memory for the overlap), the sort may still run.
 * emsesg_upload_field_async(ctx, EMSESG_FIELD_EB, host) copies the eb of
 * the next step on the side stream into a second buffer, which replaces the
 * field before the next work that reads eb (an FP32 step, grdcrt, the field
 * step, a download of eb); the copy starts once the last step has read eb,
 * so it overlaps with that step's sort.  With the FP32 form loaded the copy
 * goes in z chunks and the next FP32 step pushes its tile layers in parts,
 * each once its chunk is there; a particle outside its tile's box whose
 * node planes are not there yet is pushed after the last part, by a kernel
 * that may round its kick otherwise in the last bit (such a step agrees
 * with the step after a synchronous upload in counts, cells and liveness,
 * and up to those particles' last bits).  A synchronous emsesg_upload_field
 * of eb replaces a pending asynchronous one.  The two buffers change roles
 * with every asynchronous upload: emsesg_fx_run takes a pending upload
 * before it captures or replays its graph and captures again when the eb
 * buffer changed; a batch (emsesg_batch_create) takes pending uploads before
 * its capture, and emsesg_batch_launch refuses (EMSESG_ERR_STATE) a run whose
 * eb was uploaded asynchronously since. */
int emsesg_fx_step_download(emsesg_ctx* ctx, int ustep, int do_sort, double* rho, double* aj);
/* emsesg_fx_step_es: the electrostatic step of the FP32 form, the
 * reference's psolve2 + charge (src/pcl2field/psolve2.F90:4-548,
 * src/pcl2field/charge.F90:4-212, as its ES main loop calls them,
 * src/main/esses.F90:341-367,530-560): the push with the outer boundary
 * rules, bodies and injected particles of emsesg_fx_step, rho deposited
 * and folded, no current (J's accumulator and the aj field are left as
 * they are, and the step has no continuity residual); then the re-sort when
 * do_sort.  rho is the one emsesg_fx_step deposits for the same particles.
 * Not in slab mode.  Asynchronous. */
int emsesg_fx_step_es(emsesg_ctx* ctx, int ustep, int do_sort);
int emsesg_upload_field_async(emsesg_ctx* ctx, int field, const double* host);
/* nsteps steps of the FP32 form, re-sorting every sort_every steps
 * (emsesg_fx_step with do_sort on every sort_every-th step).  With use_graph,
 * a block of 2*sort_every steps is captured once into a CUDA graph (cached
 * per ustep and sort_every) and replayed; the remaining steps run one by one.
 * Inside the graph a tile sort that meets a particle outside its tile's sort
 * box cannot switch to the global sort: it keeps the current order for that
 * species (the push handles such particles on its general path), so rho/J
 * stay the same physics, though their FP32 partial sums may round in a
 * different order than emsesg_fx_step's.  Injected particles waiting in the
 * tail zone, or an unsorted layout, make it run step by step.  Asynchronous
 * on the context's stream. */
int emsesg_fx_run(emsesg_ctx* ctx, int ustep, int nsteps, int sort_every, int use_graph);

/* Rows of a tile region that one push CTA takes (default 256; a tile of
 * more rows is pushed by several CTAs that add their sums into the same
 * accumulators).  Fewer rows per CTA spread a small grid over more SMs at
 * the cost of more field-tile loads and accumulator flushes; the ensemble's
 * autotuner picks it per grid size.  Kept until the FP32 form is released. */
int emsesg_fx_chunk_rows(emsesg_ctx* ctx, int rows);

/* Domain decomposition in z slabs (replaces, for slabs of one periodic z
 * axis, OhHelp's particle migration, oh2_transbound / exchange_particles,
 * lib/ohhelp/ohhelp-1.1.1/ohhelp2.c:103-123, 333-384, and the border
 * exchange of oh3_exchange_borders, ohhelp3.c:959-1046, between ranks).
 * The context's grid is one slab of nz cells of a grid cut into slabs of
 * equal thickness; its eb holds the slab's field with its guards.
 * emsesg_fx_slab(ctx, 1, cap) turns slab mode on (periodic z particles and
 * fields, no bodies; cap: room for the particles leaving a slab through one
 * face per species and step).  A step is then
 *   emsesg_fx_slab_begin(ctx, ustep, counts): the push; particles leaving
 *     through z = 0 / z = nz go to the outbox of direction 0 / 1 (their
 *     positions in the neighbour's frame, their current in this slab's
 *     guard planes), counts[2 (spec - 1) + dir] of them, in the order of
 *     their slots; synchronous;
 *   the exchange of particles: the outbox of direction 1 of a rank goes to
 *     the rank above, direction 0 to the rank below (emsesg_fx_slab_outbox
 *     gives its device address);
 *   emsesg_fx_slab_arrive(ctx, spec, dev, n), for the particles from below,
 *     then from above: into the tail zone, their charge into rho;
 *   emsesg_fx_slab_border(ctx): the x / y border exchange of rho and J (the
 *     z border planes then hold what goes to the neighbours); synchronous;
 *   the exchange of planes: the z border planes of the int64 rho and J
 *     accumulators (emsesg_fx_slab_planes: which 0 / 1 the planes sent
 *     down / up, 2 / 3 the planes that receive them from below / above,
 *     device addresses and counts of int64) are copied from the sending
 *     planes of the neighbours;
 *   emsesg_fx_slab_end(ctx, do_sort): the guard folds (z, y, x), FP64 rho
 *     and aj, with do_sort the re-sort.
 * The nodes 0..nz of each slab then hold what one grid of all slabs holds
 * on them (rho and J as sums of the same int64 contributions). */
int emsesg_fx_slab(emsesg_ctx* ctx, int on, int64_t outbox_cap);
int emsesg_fx_slab_begin(emsesg_ctx* ctx, int ustep, int64_t* counts);
int emsesg_fx_slab_outbox(emsesg_ctx* ctx, int spec, int dir, emsesg_particle** dev);
int emsesg_fx_slab_planes(emsesg_ctx* ctx, int which, int64_t** rho, int64_t* nrho, int64_t** j, int64_t* nj);
int emsesg_fx_slab_arrive(emsesg_ctx* ctx, int spec, const emsesg_particle* dev, int64_t n);
int emsesg_fx_slab_border(emsesg_ctx* ctx);
int emsesg_fx_slab_end(emsesg_ctx* ctx, int do_sort);

/* Ensembles (no counterpart in the reference, which runs one job per run):
 * one CUDA graph holding `block` steps of each of n independent runs
 * (contexts on one device, FP32 form loaded, no injected particles
 * waiting), run r re-sorting every sort_every[r] steps; block must be a
 * multiple of 2*sort_every[r] for every r.  The runs are independent
 * branches of the graph, so the GPU runs their kernels side by side. */
typedef struct emsesg_batch emsesg_batch;
int emsesg_batch_create(emsesg_ctx* const* ctxs, int n, int ustep, int block, const int* sort_every,
                        emsesg_batch** out);
/* Replays the graph nrep times (nrep*block steps of every run) on the
 * batch's own stream, after the earlier work of every run's stream and
 * before its later work.  Errors are reported through the run contexts
 * (emsesg_last_error of the first one for launch errors). */
int emsesg_batch_launch(emsesg_batch* b, int nrep);
/* The batch's cudaStream_t, as an opaque pointer (for timing events). */
void* emsesg_batch_stream(emsesg_batch* b);
/* Kernel launches in one replay of the batch's graph. */
int emsesg_batch_kernels(const emsesg_batch* b, int64_t* n);
/* Waits for the batch's work and releases it (the runs stay). */
int emsesg_batch_destroy(emsesg_batch* b);
/* Particle counts of the FP32 form (nspec entries). */
int emsesg_fx_counts(emsesg_ctx* ctx, int64_t* totalp);
/* Raw fixed-point accumulators after the guard folding, int64 at 2^40:
 * rho in the rho layout followed by (jx, jy, jz) in the aj layout. */
int emsesg_fx_download_accum(emsesg_ctx* ctx, int64_t* host);
/* Injected particles of species `spec` (1-based), oh2_inject_particle
 * (lib/ohhelp/ohhelp-1.1.1/ohhelp2.c:549) for the FP32 form: the records go
 * to a tail zone that the next emsesg_fx_step pushes with the general path
 * (preside +1: a random fraction U of the first step, psolve1.F90:150-156;
 * drawn in buffer order after the species before it); an anti-particle
 * (preside -2, the image of an emitted particle on a body face,
 * psuper3.F90:203-206) removes one count from that face cell.  The next
 * sort merges the tail into the tile regions (sorting with particles still
 * waiting for their first push is an error). */
/* Asynchronous: from pinned host memory the upload overlaps the GPU's work
 * (keep the records unchanged until the stream has passed the call); from
 * pageable memory the call returns once the records are copied. */
int emsesg_fx_inject(emsesg_ctx* ctx, int spec, const emsesg_particle* host, int64_t n);
/* The injection supervisors on the device (records drawn, converted and
 * put into the tail zone without a host round trip).  U[0,1) numbers come
 * from a counter hash of (seed, stream, index0 + k) per particle k;
 * ctca_b200/inject.py computes the same records on the host
 * (hash_uniforms), to which these are bit-identical.
 * emsesg_fx_emit: n emitted pairs from the face nemd (+-1: x, +-2: y, +-3:
 * z) at grd, extents b1 / b2 along its first / second tangential axis:
 * an anti-particle (preside -2) on the face and its twin 1e-5 off it
 * (preside 1), normal speed vnorm[int(npr*u0)], tangential vtang[int(npr*u1)],
 * vtang[int(npr*u2)] (psuper3.F90:142-208).  emsesg_fx_inflow_z: n
 * particles through z = 0 (front) or z = nz: x, y uniform on the face, z =
 * the distance vz * injctisw * u4 from it, vz = vz_t[int(npr*u0)],
 * vx / vy = vx_t / vy_t[int(npr*u1)], preside 0 (psuper2.F90:236-292). */
int emsesg_fx_emit(emsesg_ctx* ctx, int spec, int nemd, double grd, const double* b1, const double* b2, int64_t n,
                   const double* vnorm, const double* vtang, int npr, uint64_t seed, uint64_t stream,
                   uint64_t index0);
int emsesg_fx_inflow_z(emsesg_ctx* ctx, int spec, int front, int64_t n, const double* vz_t, const double* vx_t,
                       const double* vy_t, int npr, double injctisw, uint64_t seed, uint64_t stream,
                       uint64_t index0);
/* emsesg_fx_inflow: the same through the lower (front) or upper face of
 * any axis (0: x, 1: y, 2: z; psuper2.F90:114-173 x faces, :175-233 y
 * faces, :236-292 z faces): u2 / u3 / u4 give x / y / z, uniform on the
 * face along the tangential axes, the distance vn * injctisw * u from the
 * face along the normal; vn = vn_t[int(npr*u0)], the tangential speeds of
 * the two other axes in increasing order va_t / vb_t[int(npr*u1)].
 * emsesg_fx_inflow_z(..., vz_t, vx_t, vy_t, ...) is
 * emsesg_fx_inflow(..., 2, ..., vz_t, vx_t, vy_t, ...). */
int emsesg_fx_inflow(emsesg_ctx* ctx, int spec, int axis, int front, int64_t n, const double* vn_t, const double* va_t,
                     const double* vb_t, int npr, double injctisw, uint64_t seed, uint64_t stream, uint64_t index0);
/* emsesg_fx_inflow_current: emsesg_fx_inflow with the injection current of
 * psuper1 (replaces psuper1's outer-face blocks, src/pcl/psuper1.F90:120-323,
 * and current_deposition, :859-988): each particle also deposits, times its
 * species' charge, the zigzag current of its path from b outside the face
 * (-1 below the lower face, n + 0.99999999 above the upper one, along the
 * normal; its position minus v * ustep along the other axes) to its
 * injection point, into the J of the next emsesg_fx_step (the step adds its
 * own deposit to these currents instead of starting J from zero; the
 * reference zeroes aj, runs psuper1, then psolve1).  Contributions are
 * rounded to the int64 accumulator (scale 2^40) one by one. */
int emsesg_fx_inflow_current(emsesg_ctx* ctx, int spec, int axis, int front, int64_t n, const double* vn_t,
                             const double* va_t, const double* vb_t, int npr, double injctisw, int ustep,
                             uint64_t seed, uint64_t stream, uint64_t index0);
/* emsesg_fx_emit_plane: n particles from a rectangular plane of body pid
 * (psuper2.F90:330-360 with emit_from_rectangular_surf, :554-576): six
 * uniforms each; normal speed ud * vnorm[int(npr*u0)], tangential
 * vtang[int(npr*u1)], vtang[int(npr*u2)]; normal coordinate
 * grd + vnorm * injctisw * u3, tangential b1 / b2 uniform (u4, u5) plus
 * vtang * injctisw * u3; one record each, preside 0.  The outflux and
 * chgacm bookkeeping of psuper2.F90:494-498 (n per call) is the caller's. */
int emsesg_fx_emit_plane(emsesg_ctx* ctx, int spec, int nemd, double grd, const double* b1, const double* b2,
                         int64_t n, const double* vnorm, const double* vtang, int npr, double injctisw, int pid,
                         uint64_t seed, uint64_t stream, uint64_t index0);
/* emsesg_fx_emit_cylinder: n particles from a face of a cylindrical body
 * (replaces emit_from_cylinder with emit_from_circular_surf and
 * emit_from_cylindrical_surf1/2/3, src/pcl/psuper3.F90:241-528).  align:
 * the cylinder's axis (1..3); axis: its two axis coordinates as the
 * reference's cylinder%axis; radius; omni: the reference's omniemit.
 * |nemd| = align: the end cap at grd (normal ud * vnormf[int(npr u0)],
 * tangential vtangf[int(npr u1)], vtangf[int(npr u2)], the point radius *
 * runiform[int(npr u3)] from the axis at the angle 2 pi u4).  Other nemd:
 * the side, between hl and hu along the axis: omni 0 and radius >= 1
 * turns vnormc / vtangc by psicos[int(npr u2)] + psi, omni 0 and radius < 1
 * by psi (five uniforms a particle), omni 1 by the azimuth 2 pi u2; psi is
 * the reference's psizy / psizx / psixy for align 1 / 2 / 3.  Uniform c of
 * particle k is the hash of index0 * 6 + per * k + c (per: 5 or 6), the
 * flat RANU0(dranu, 6n) of the reference.  Each particle gives a record
 * with preside 1 and, with anti (the reference's ncond <= 0), its
 * anti-particle (preside -2) at the same place; the FP32 form counts
 * anti-particles on box-body face cells only, so these are dropped.  The
 * tables (npr entries each) are the species' vnormf, vtangf, runiform,
 * vnormc, vtangc, psicos (inipin.F90:996-1097).  ctca_b200/inject.py
 * (emit_cylinder) computes the same records on the host; they agree to the
 * last bits of cos / sin. */
int emsesg_fx_emit_cylinder(emsesg_ctx* ctx, int spec, int nemd, int align, double radius, const double* axis,
                            int omni, double grd, double hl, double hu, double psi, int64_t n, const double* vnormf,
                            const double* vtangf, const double* runiform, const double* vnormc,
                            const double* vtangc, const double* psicos, int npr, int anti, uint64_t seed,
                            uint64_t stream, uint64_t index0);
/* Absorbed minus emitted particles per surface cell of the box bodies
 * (geotype 0/1, integer bounds), int64 [nspec][nsurf]: body by body, faces
 * -x,+x,-y,+y,-z,+z, each face's cells with its first tangential axis
 * fastest (x faces: y then z; y faces: x then z; z faces: x then y).  A
 * particle entering a box between two positions counts on the face it
 * crossed last, in the cell holding its end point.  counts may be NULL to
 * query nsurf. */
int emsesg_fx_surface(emsesg_ctx* ctx, int64_t* counts, int64_t* nsurf);
/* Background charge from the surface counts (replaces add_background_charge,
 * src/pcl2field/charge.F90:414-449, with rhobk(...,3) += rhobk(...,1) of
 * src/main/emses.F90:249-251): the field EMSESG_FIELD_RHOBK becomes the
 * cumulative absorbed minus emitted charge of the box bodies as node values
 * -- a surface cell's charge q(is) * count goes in equal quarters to the four
 * nodes of its face cell, the counts meeting at a node summed in int64 per
 * species, then scaled once in FP64 -- and rho(0:nx,0:ny,0:nz) += rhobk, or
 * = rhobk with replace != 0 (the reference's nflag_testp == 1).  Call it
 * after a step, as the reference calls add_background_charge after charge. */
int emsesg_fx_background(emsesg_ctx* ctx, int replace);
/* Kinetic energy of the FP32 state in FP64 (replaces energy,
 * src/etc/energy.F90:29-47): engk[is*3 + d] = 0.5*rm(is)*sum(v_d^2)/(nx*ny*nz)
 * over the live particles, the sums in a fixed order (reproducible bit for
 * bit).  Works with EMSESG_FLAG_FP32_ONLY. */
int emsesg_fx_energy(emsesg_ctx* ctx, double* engk);
/* Charge continuity of the last FP32 step in FP64 (the check of rhoupd,
 * src/field/rhoupd.F90:41-49): res[0] = max over the nodes 0..n of
 * |rho_new - rho_old + 2 (div J)|, rho_old the rho field the step before
 * left; res[1] = max |rho_new|.  res[0] is NaN when no step deposited rho
 * before the last one (after a load).  Works with EMSESG_FLAG_FP32_ONLY. */
int emsesg_fx_continuity(emsesg_ctx* ctx, double* res);
/* Reverse mode through K steps of the FP32 form on a periodic grid (no
 * bodies, no injection): runs the K forward steps (re-sort every sort_every
 * steps), then the adjoint sweep with the particle state checkpointed every
 * ckpt steps (K a multiple of ckpt, ckpt <= 64) and recomputed in between.
 * Loss: L = sum over the K steps and the probe nodes lo <= (i,j,k) < hi of
 * aj_x(i,j,k)^2 (the folded current).  Gradients, each optional: gE, gB of
 * the FP32 node fields E, B used by the push, [nx*ny*nz][3] with x fastest;
 * g0[6] of the uniform e0, b0 (the node sums); gv[N][3] of the initial
 * velocities, in the order emsesg_fx_store writes the particles (species by
 * species, tile-major sorted ranks).  The state ends as after the forward. */
int emsesg_fx_adjoint(emsesg_ctx* ctx, int K, int ustep, int ckpt, int sort_every, const int32_t* probe_lo,
                      const int32_t* probe_hi, double* loss, double* gE, double* gB, double* g0, double* gv);

/* ---- synthetic plasma loader (seeded, on the device) -------------------- */
typedef struct emsesg_plasma {
  int32_t ppc[EMSESG_ISPEC];     /* particles per cell per species */
  double vth[EMSESG_ISPEC];      /* thermal speed (internal units) */
  double vdrift[EMSESG_ISPEC][3];/* drift velocity (internal units) */
  uint64_t seed;
} emsesg_plasma;
/* Fills the FP64 pbuf mirror: ppc particles uniform in every cell,
 * Maxwellian velocities (Box-Muller on a SplitMix64 counter hash). */
int emsesg_load_plasma(emsesg_ctx* ctx, const emsesg_plasma* pl);
/* The same plasma (the same draws, particle for particle) straight into the
 * FP32 form, tile-sorted, without the FP64 records: emsesg_load_plasma then
 * emsesg_fx_load give the same state.  Works with EMSESG_FLAG_FP32_ONLY. */
int emsesg_fx_load_plasma(emsesg_ctx* ctx, const emsesg_plasma* pl);

/* ---- profiling ----------------------------------------------------------- */
/* When on, every kernel launch is bracketed by CUDA events on the context
 * stream and its duration is summed per kernel name. */
int emsesg_set_profiling(emsesg_ctx* ctx, int on);
/* Writes "name total_ms launches\n" lines; returns EMSESG_OK. */
int emsesg_profile_report(emsesg_ctx* ctx, char* buf, size_t len);
int emsesg_profile_reset(emsesg_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* EMSES_GPU_H */
