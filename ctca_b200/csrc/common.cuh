// common.cuh -- shared internals of libemsesg (the B200 EMSES particle path).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

#include "../../include/emses_gpu.h"

// z chunks of an asynchronous eb upload for the FP32 step (parts of its push)
constexpr int EMSESG_EB_PARTS = 4;

namespace emsesg {

// Fortran-layout field descriptor (nc, lo:n+hi per axis), component fastest.
struct FieldDesc {
  int nc, lo, ex, ey, ez;
  __host__ __device__ int64_t at(int c, int i, int j, int k) const {
    return c + (int64_t)nc * ((i - lo) + (int64_t)ex * ((j - lo) + (int64_t)ey * (k - lo)));
  }
  __host__ __device__ int64_t size() const { return (int64_t)nc * ex * ey * ez; }
};

// Guard extents from OhHelp's fsizes rule (ohhelp3.c:439-477) applied to
// ftypes/ctypes of src/wrapper/ohinit.F90:98-122.
FieldDesc field_desc(const emsesg_config& c, int field);

// Per-species device segment: particles [base, base + count) of a region of
// `capacity` slots.  The device keeps one region per species (the host
// buffer packs them back to back, as pbuf/pbase/totalp do).
struct Segments {
  int64_t base[EMSESG_ISPEC];
  int64_t capacity[EMSESG_ISPEC];
};

// Kernel launch timing (CUDA events on the context stream).
struct KernelTimer {
  bool on = false;
  struct Entry { double ms = 0; int64_t launches = 0; };
  std::map<std::string, Entry> total;
  struct Pending { std::string name; cudaEvent_t a, b; };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> pool;
};

struct SortScratch {
  // Radix sort buffers sized for the largest species region.
  uint32_t* keys[2] = {nullptr, nullptr};
  uint32_t* vals[2] = {nullptr, nullptr};
  uint32_t* hist = nullptr;       // digit-major block histograms
  uint32_t* scan_tmp = nullptr;   // partial sums of the scans
  int64_t cap = 0;
  int64_t hist_cap = 0;
  int64_t scan_tmp_cap = 0;
};

// FP32 / fixed-point particle state.
struct AdjWork;  // reverse-mode workspace (fx.cu), kept between calls
struct FxState;
void adj_free(FxState& f);

// Arrays a move-only step reads instead of the live ones (see FxPushArgs).
struct FxSrc {
  const float4* pos = nullptr;
  const float* vx = nullptr;
  const float* vy = nullptr;
  const float* vz = nullptr;
};

struct FxState {
  bool loaded = false;
  FxSrc move_src;          // set around the adjoint's recompute steps only
  float4* pos = nullptr;   // {ox, oy, oz, __int_as_float(cell)}
  float* vx = nullptr;
  float* vy = nullptr;
  float* vz = nullptr;
  float4* pos2 = nullptr;  // sort double buffer
  float* vx2 = nullptr;
  float* vy2 = nullptr;
  float* vz2 = nullptr;
  int64_t* count_d = nullptr;       // device live-particle counts per species (last sort)
  int64_t* slots_d = nullptr;       // device slot counts per species (padded regions)
  int64_t* tile_start = nullptr;    // [nspec][ntiles+1] sorted ranks of each tile's first particle
  int64_t* tile_pad = nullptr;      // [nspec][ntiles+1] first slot of each tile's padded region
  int64_t* chunk_start = nullptr;   // [nspec][ntiles+1] first push CTA of each tile
  int64_t base[EMSESG_ISPEC] = {};  // species region offsets in pos / vx / vy / vz
  int64_t cap[EMSESG_ISPEC] = {};   // species region sizes (capacity + tile padding)
  bool tiled = false;               // regions hold the thread-major layout of a sort
  bool box_inside = false;          // loaded particles start inside a box body (until the next push)
  // tile-local counting sort (fx_sort.cuh): per species
  int64_t* tile_start2 = nullptr;   // the new tile_start / tile_pad, swapped in after
  int64_t* tile_pad2 = nullptr;
  uint32_t* lcs_cnt = nullptr;      // [nspec][ntiles][nbc]
  uint32_t* lcs_base = nullptr;     // [nspec][ntiles][nbc]
  uint32_t* lcs_wcnt = nullptr;     // [ntiles][warps][nbc] of the species being sorted
  uint32_t* lcs_celltot = nullptr;  // [ntiles][tile cells]
  int64_t* lcs_tiletot = nullptr;   // [ntiles]
  int* lcs_stray = nullptr;         // [nspec]
  uint32_t* lcs_inv = nullptr;      // per slot: the old slot of its particle
  // box bodies: absorbed minus emitted particles per surface cell
  unsigned long long* surf = nullptr;  // [nspec][nsurf]
  int64_t nsurf = 0;
  // injected particles (oh2_inject_particle): a tail zone at the end of each
  // species region, pushed by the general path until the next sort
  int64_t tail0[EMSESG_ISPEC] = {};    // first slot of the tail zone
  int64_t tailcap[EMSESG_ISPEC] = {};
  int64_t ntail[EMSESG_ISPEC] = {};
  int32_t* tailord = nullptr;          // per tail slot: 1 + ordinal of a pending random step, or 0
  int64_t tailord_base[EMSESG_ISPEC] = {};  // offset of each species' tail in tailord
  int64_t pending[EMSESG_ISPEC] = {};  // injected particles still to take their random step
  bool inj_j_pending = false;          // the J accumulator holds injection currents for the next step
  // slab mode (emsesg_fx_slab): records of the particles leaving through the
  // z faces, [2 nspec][outbox_cap], and their counts
  bool slab = false;
  bool slab_open = false;              // between emsesg_fx_slab_begin and emsesg_fx_slab_end
  emsesg_particle* outbox = nullptr;
  emsesg_particle* outbox2 = nullptr;  // the sort of a region by source slot
  unsigned long long* outbox_n = nullptr;
  int64_t outbox_cap = 0;
  emsesg_particle* stage = nullptr;    // device staging of injected records
  int32_t* stage_ord = nullptr;
  int64_t stage_cap = 0;
  double* inj_tab = nullptr;           // velocity tables of the device supervisors
  int64_t inj_tab_cap = 0;
  int32_t* ord_host = nullptr;         // pinned host staging of the ordinals
  int64_t ord_host_cap = 0;
  cudaEvent_t ord_ev = nullptr;        // the last upload from ord_host
  // CUDA graph of a block of steps (emsesg_fx_run)
  bool capture = false;                // inside a stream capture: no host syncs
  cudaGraphExec_t gexec = nullptr;
  int g_ustep = 0, g_sort = 0;
  const float4* g_pos = nullptr;       // buffers and configuration it was captured with
  const int64_t* g_ts = nullptr;
  const double* g_eb = nullptr;        // (an asynchronous eb upload swaps the eb buffer)
  emsesg_config g_cfg{};
  AdjWork* adj = nullptr;
  uint32_t* defer = nullptr;        // one bit per slot: left for k_fx_deferred by the parts of a step
  int64_t defer_words = 0;
  int64_t* accum = nullptr;         // int64 (rho, jx, jy, jz) on the rho layout
  double* diag = nullptr;           // FP64 checks: energy partials, sums, continuity maxima
  bool rho_prev = false;            // the rho field holds the deposit of the step before
  bool cont_valid = false;          // ... so the last step's continuity residual is meaningful
  float4* fnode = nullptr;          // node field {ex, ey, ez, bx} over (n+1)^3 nodes
  float4* fnode2 = nullptr;         // {by, bz, 0, 0}
  int bits[3] = {0, 0, 0};          // packed cell bit widths
  int tile[3] = {8, 8, 8};
  int chunk_rows = 256;             // rows of a tile region per push CTA (emsesg_fx_chunk_rows)
  int ntile[3] = {0, 0, 0};
  int64_t ntiles = 0;
};

}  // namespace emsesg

// Electrostatic field step (esfield.cu): cuFFT plans (cufftHandle values),
// the dense rho / phi of the nodes 0..n-1, its spectrum, the eigenvalues of
// the three axes and the residual sum.
struct EsState {
  int fwd = 0, inv = 0;
  bool has_fwd = false, has_inv = false;
  double* r = nullptr;
  void* c = nullptr;
  double* lam = nullptr;
  double* sum = nullptr;
  bool ready = false;
  // any field boundary (axis by axis): the mtd_vbnd it was set up for, one
  // batched complex plan per axis, the solved nodes, the complex lines and
  // the eigenvalues over the solved nodes
  int gt[3] = {-1, -1, -1};
  int gplan[3] = {0, 0, 0};
  bool has_gplan[3] = {false, false, false};
  double* w = nullptr;
  void* z = nullptr;
  double* glam = nullptr;
};

struct emsesg_ctx {
  emsesg_config cfg;
  emsesg_config* d_cfg = nullptr;      // device copy of cfg for the kernels
  int device = 0;
  cudaStream_t stream = nullptr;
  // host transfers beside the step (emsesg_fx_step_download,
  // emsesg_upload_field_async): a side stream, the event after a step's
  // field phase, the next eb (double buffer) and its copy event
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fields = nullptr;
  cudaEvent_t ev_eb = nullptr;
  double* eb_next = nullptr;
  bool eb_next_pending = false;
  // the pending eb copied in z chunks for the FP32 step (eb_parts > 1):
  // chunk p holds what the node planes 0..eb_zready[p] read, and part p of
  // the push (tiles eb_tile[p] .. eb_tile[p+1] - 1) runs once it is there
  int eb_parts = 0;
  int eb_zready[EMSESG_EB_PARTS] = {0};
  int64_t eb_tile[EMSESG_EB_PARTS + 1] = {0};
  cudaEvent_t ev_ebp[EMSESG_EB_PARTS] = {nullptr};
  std::string err;
  emsesg::Segments seg;
  int64_t totalp[EMSESG_ISPEC] = {0};  // host mirror of the species counts
  int64_t* d_count = nullptr;          // device species counts (drop-in)
  emsesg_particle* pbuf = nullptr;     // device pbuf, one region per species
  emsesg_particle* pbuf2 = nullptr;    // scratch for sort / compaction
  double* field[EMSESG_NFIELDS] = {nullptr};
  EsState es;
  double* node64 = nullptr;            // drop-in node field: 8 doubles / node
  double* tj = nullptr;                // per-species zigzag scratch (aj layout)
  emsesg_counter* d_counter = nullptr;
  double* d_randoms = nullptr;
  int64_t n_randoms = 0;
  int64_t* d_rand_pos = nullptr;       // next pre-drawn number (device)
  uint64_t rng_stream = 0;             // push call counter for the hash
  int* d_status = nullptr;             // device error word
  long long* d_diag = nullptr;         // first bad-index report {site, index, what, 0}
  int64_t* d_scratch64 = nullptr;      // small scratch (counts, sums)
  double* d_sum = nullptr;
  emsesg::SortScratch sort;
  emsesg::FxState fx;
  emsesg::KernelTimer timer;
};

namespace emsesg {

int set_error(emsesg_ctx* ctx, int code, const char* fmt, ...);
// The side stream of host transfers (created on first use), and the eb of
// an asynchronous upload put in place (the context's stream waits for its
// copy) before the work that reads eb.
int side_stream(emsesg_ctx* ctx);
int apply_pending_eb(emsesg_ctx* ctx);
// The z chunks of an eb upload for the FP32 step (fx.cu): per part the last
// node plane it needs and its first tile; returns the number of parts (0:
// one copy).
int fx_eb_plan(const emsesg_ctx* ctx, int* zready, int64_t* tile);
// Records m0 .. m0+n-1 of species `is` of the seeded plasma of
// emsesg_load_plasma, into the device array dst (n records).
int plasma_records(emsesg_ctx* ctx, emsesg_particle* dst, int is, int64_t m0, int64_t n, const emsesg_plasma* pl);
int check_cuda(emsesg_ctx* ctx, cudaError_t e, const char* what);
// Launch bracketing for the per-kernel profile.
void timer_begin(emsesg_ctx* ctx, const char* name);
void timer_end(emsesg_ctx* ctx);
void timer_collect(emsesg_ctx* ctx);

// Device status word codes.
enum { ST_OK = 0, ST_BAD_INDEX = 1, ST_RANDOMS = 2, ST_OVERFLOW = 4 };

// Sites that report ST_BAD_INDEX; the first report also leaves
// {site, particle index, packed or truncated cell, 0} in the diag record.
enum { SITE_PSOLVE2 = 1, SITE_PSOLVE1, SITE_CHARGE, SITE_FX_LOAD, SITE_FX_PUSH, SITE_FX_DEPOSIT, SITE_FX_FLUSH, SITE_FX_SORT };

__device__ __forceinline__ void report_bad(int* status, long long* diag, int site, long long index,
                                           long long what) {
  atomicOr(status, ST_BAD_INDEX);
  if (diag && atomicCAS((unsigned long long*)&diag[0], 0ull, (unsigned long long)site) == 0ull) {
    diag[1] = index;
    diag[2] = what;
  }
}

// SplitMix64 finaliser (Steele, Lea, Flood 2014).
__host__ __device__ inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
// U[0,1) with 53 random bits from (seed, stream, index).
__host__ __device__ inline double hash_u01(uint64_t seed, uint64_t stream, uint64_t index) {
  uint64_t a = mix64(seed ^ mix64(stream + 0x632BE59BD9B4E019ULL));
  uint64_t b = mix64(a ^ (index * 0xD1B54A32D192ED03ULL));
  return (double)(b >> 11) * (1.0 / 9007199254740992.0);
}

// Internal entry points shared between translation units.
int sort_pairs(emsesg_ctx* ctx, uint32_t* keys, uint32_t* vals, int64_t n, int key_bits,
               uint32_t** keys_out, uint32_t** vals_out);
int exclusive_scan_u32(emsesg_ctx* ctx, uint32_t* data, int64_t n);
int exclusive_scan_i64(emsesg_ctx* ctx, int64_t* data, int64_t n);
int ensure_sort_scratch(emsesg_ctx* ctx, int64_t n);

int fx_alloc(emsesg_ctx* ctx);
void fx_free(emsesg_ctx* ctx);
void es_free(emsesg_ctx* ctx);

}  // namespace emsesg

#define EMSESG_CUDA(ctx, call)                                               \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) return emsesg::check_cuda((ctx), e_, #call);      \
  } while (0)

#define EMSESG_LAUNCH(ctx, name, kernel, grid, block, smem, ...)             \
  do {                                                                       \
    emsesg::timer_begin((ctx), (name));                                      \
    kernel<<<(grid), (block), (smem), (ctx)->stream>>>(__VA_ARGS__);         \
    emsesg::timer_end((ctx));                                                \
    cudaError_t e_ = cudaGetLastError();                                     \
    if (e_ != cudaSuccess) return emsesg::check_cuda((ctx), e_, name);       \
  } while (0)
