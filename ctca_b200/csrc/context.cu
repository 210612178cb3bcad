// context.cu -- context life cycle, explicit host<->device sync points,
// error reporting and the per-kernel profile of libemsesg.
#include <algorithm>
#include <cstring>

#include "common.cuh"

namespace emsesg {

FieldDesc field_desc(const emsesg_config& c, int field) {
  int nx = c.nx, ny = c.ny, nz = c.nz;
  switch (field) {
    case EMSESG_FIELD_EB: return {6, -1, nx + 3, ny + 3, nz + 3};
    case EMSESG_FIELD_WRK: return {9, -4, nx + 9, ny + 9, nz + 9};
    case EMSESG_FIELD_AJ: return {3, -4, nx + 9, ny + 9, nz + 9};
    case EMSESG_FIELD_AJDG: return {3 * c.nspec, -4, nx + 9, ny + 9, nz + 9};
    case EMSESG_FIELD_RHO: return {1, -1, nx + 3, ny + 3, nz + 3};
    case EMSESG_FIELD_RHODG: return {2 * c.nspec + 1, -1, nx + 3, ny + 3, nz + 3};
    case EMSESG_FIELD_RHOBK: return {1, -1, nx + 3, ny + 3, nz + 3};
    case EMSESG_FIELD_RHOBKSP: return {1, -1, nx + 3, ny + 3, nz + 3};
    case EMSESG_FIELD_PHI: return {1, -1, nx + 3, ny + 3, nz + 3};
  }
  return {0, 0, 0, 0, 0};
}

static int64_t field_doubles(const emsesg_config& c, int field) {
  FieldDesc f = field_desc(c, field);
  return field == EMSESG_FIELD_RHOBKSP ? f.size() * c.nspec : f.size();
}

int set_error(emsesg_ctx* ctx, int code, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return code;
}

int check_cuda(emsesg_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return EMSESG_OK;
  int code = (e == cudaErrorMemoryAllocation) ? EMSESG_ERR_NOMEM : EMSESG_ERR_CUDA;
  return set_error(ctx, code, "%s: %s", what, cudaGetErrorString(e));
}

void timer_begin(emsesg_ctx* ctx, const char* name) {
  if (!ctx->timer.on) return;
  KernelTimer::Pending p;
  p.name = name;
  auto take = [&]() {
    cudaEvent_t e;
    if (!ctx->timer.pool.empty()) { e = ctx->timer.pool.back(); ctx->timer.pool.pop_back(); }
    else cudaEventCreate(&e);
    return e;
  };
  p.a = take();
  p.b = take();
  cudaEventRecord(p.a, ctx->stream);
  ctx->timer.pending.push_back(p);
}

void timer_end(emsesg_ctx* ctx) {
  if (!ctx->timer.on || ctx->timer.pending.empty()) return;
  cudaEventRecord(ctx->timer.pending.back().b, ctx->stream);
  if (ctx->timer.pending.size() > 4096) timer_collect(ctx);
}

void timer_collect(emsesg_ctx* ctx) {
  if (ctx->timer.pending.empty()) return;
  cudaStreamSynchronize(ctx->stream);
  for (auto& p : ctx->timer.pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.a, p.b);
    auto& e = ctx->timer.total[p.name];
    e.ms += ms;
    e.launches += 1;
    ctx->timer.pool.push_back(p.a);
    ctx->timer.pool.push_back(p.b);
  }
  ctx->timer.pending.clear();
}

}  // namespace emsesg

using namespace emsesg;

static int validate_config(emsesg_ctx* ctx, const emsesg_config* c) {
  if (c->nx < 2 || c->ny < 2 || c->nz < 2) return set_error(ctx, EMSESG_ERR_ARG, "grid must be at least 2 cells per axis");
  if ((int64_t)c->nx * c->ny * c->nz >= (1LL << 31)) return set_error(ctx, EMSESG_ERR_ARG, "grid too large");
  if (c->nspec < 1 || c->nspec > EMSESG_ISPEC) return set_error(ctx, EMSESG_ERR_ARG, "nspec out of range");
  if (c->npc < 0 || c->npc > EMSESG_INPC) return set_error(ctx, EMSESG_ERR_ARG, "npc out of range");
  if (c->rng_mode != 0 && c->rng_mode != 1) return set_error(ctx, EMSESG_ERR_ARG, "rng_mode must be 0 or 1");
  for (int is = 0; is < c->nspec; is++) {
    if (c->capacity[is] < 0 || c->capacity[is] >= (1LL << 31))
      return set_error(ctx, EMSESG_ERR_ARG, "capacity[%d] out of range (0 .. 2^31-1)", is);
  }
  for (int d = 0; d < 3; d++)
    if (c->sort_tile[d] < 0) return set_error(ctx, EMSESG_ERR_ARG, "sort_tile must be >= 0");
  if (c->flags & ~EMSESG_FLAG_FP32_ONLY) return set_error(ctx, EMSESG_ERR_ARG, "unknown config flags");
  return EMSESG_OK;
}

extern "C" int emsesg_select_device(int device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return EMSESG_ERR_ARG;
  return cudaSetDevice(device) == cudaSuccess ? EMSESG_OK : EMSESG_ERR_CUDA;
}

extern "C" int emsesg_create(const emsesg_config* cfg, emsesg_ctx** out) {
  if (!cfg || !out) return EMSESG_ERR_ARG;
  *out = nullptr;
  emsesg_ctx* ctx = new emsesg_ctx();
  ctx->cfg = *cfg;
  int rc = validate_config(ctx, cfg);
  if (rc) { delete ctx; return rc; }
  cudaError_t e = cudaGetDevice(&ctx->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    rc = check_cuda(ctx, e, "stream");
    delete ctx;
    return rc;
  }
  int64_t cap = 0;
  for (int is = 0; is < cfg->nspec; is++) {
    ctx->seg.base[is] = cap;
    ctx->seg.capacity[is] = cfg->capacity[is];
    cap += cfg->capacity[is];
  }
  auto fail = [&](cudaError_t err, const char* what) {
    int r = check_cuda(ctx, err, what);
    std::string msg = ctx->err;
    emsesg_destroy(ctx);
    return r;
  };
  if ((e = cudaMalloc(&ctx->d_cfg, sizeof(emsesg_config)))) return fail(e, "cfg");
  if ((e = cudaMemcpyAsync(ctx->d_cfg, &ctx->cfg, sizeof(emsesg_config), cudaMemcpyHostToDevice, ctx->stream)))
    return fail(e, "cfg");
  // no FP64 particle buffer in FP32-only contexts (a one-record placeholder)
  const int64_t cap64 = (cfg->flags & EMSESG_FLAG_FP32_ONLY) ? 1 : std::max<int64_t>(cap, 1);
  if ((e = cudaMalloc(&ctx->pbuf, cap64 * sizeof(emsesg_particle)))) return fail(e, "pbuf");
  for (int f = 0; f < EMSESG_NFIELDS; f++) {
    int64_t n = field_doubles(ctx->cfg, f);
    if ((e = cudaMalloc(&ctx->field[f], n * sizeof(double)))) return fail(e, "field");
    if ((e = cudaMemsetAsync(ctx->field[f], 0, n * sizeof(double), ctx->stream))) return fail(e, "field");
  }
  int64_t nn = (int64_t)(cfg->nx + 2) * (cfg->ny + 2) * (cfg->nz + 2);
  if ((e = cudaMalloc(&ctx->node64, nn * 8 * sizeof(double)))) return fail(e, "node64");
  if ((e = cudaMemsetAsync(ctx->node64, 0, nn * 8 * sizeof(double), ctx->stream))) return fail(e, "node64");
  if ((e = cudaMalloc(&ctx->tj, field_doubles(ctx->cfg, EMSESG_FIELD_AJ) * sizeof(double)))) return fail(e, "tj");
  if ((e = cudaMalloc(&ctx->d_counter, sizeof(emsesg_counter)))) return fail(e, "counter");
  if ((e = cudaMemsetAsync(ctx->d_counter, 0, sizeof(emsesg_counter), ctx->stream))) return fail(e, "counter");
  if ((e = cudaMalloc(&ctx->d_count, EMSESG_ISPEC * sizeof(int64_t)))) return fail(e, "count");
  if ((e = cudaMemsetAsync(ctx->d_count, 0, EMSESG_ISPEC * sizeof(int64_t), ctx->stream))) return fail(e, "count");
  if ((e = cudaMalloc(&ctx->d_rand_pos, sizeof(int64_t)))) return fail(e, "rand");
  if ((e = cudaMemsetAsync(ctx->d_rand_pos, 0, sizeof(int64_t), ctx->stream))) return fail(e, "rand");
  if ((e = cudaMalloc(&ctx->d_status, sizeof(int)))) return fail(e, "status");
  if ((e = cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream))) return fail(e, "status");
  if ((e = cudaMalloc(&ctx->d_diag, 4 * sizeof(long long)))) return fail(e, "diag");
  if ((e = cudaMemsetAsync(ctx->d_diag, 0, 4 * sizeof(long long), ctx->stream))) return fail(e, "diag");
  if ((e = cudaMalloc(&ctx->d_scratch64, 64 * sizeof(int64_t)))) return fail(e, "scratch");
  if ((e = cudaMalloc(&ctx->d_sum, 64 * sizeof(double)))) return fail(e, "sum");
  if ((e = cudaStreamSynchronize(ctx->stream))) return fail(e, "create");
  *out = ctx;
  return EMSESG_OK;
}

extern "C" int emsesg_destroy(emsesg_ctx* ctx) {
  if (!ctx) return EMSESG_OK;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  timer_collect(ctx);
  cudaFree(ctx->d_cfg);
  cudaFree(ctx->pbuf);
  cudaFree(ctx->pbuf2);
  for (int f = 0; f < EMSESG_NFIELDS; f++) cudaFree(ctx->field[f]);
  cudaFree(ctx->node64);
  cudaFree(ctx->tj);
  cudaFree(ctx->d_counter);
  cudaFree(ctx->d_count);
  cudaFree(ctx->d_randoms);
  cudaFree(ctx->d_rand_pos);
  cudaFree(ctx->d_status);
  cudaFree(ctx->d_diag);
  cudaFree(ctx->d_scratch64);
  cudaFree(ctx->d_sum);
  for (int b = 0; b < 2; b++) { cudaFree(ctx->sort.keys[b]); cudaFree(ctx->sort.vals[b]); }
  cudaFree(ctx->sort.hist);
  cudaFree(ctx->sort.scan_tmp);
  fx_free(ctx);
  es_free(ctx);
  for (auto e : ctx->timer.pool) cudaEventDestroy(e);
  if (ctx->side) cudaStreamSynchronize(ctx->side);
  cudaFree(ctx->eb_next);
  if (ctx->ev_fields) cudaEventDestroy(ctx->ev_fields);
  if (ctx->ev_eb) cudaEventDestroy(ctx->ev_eb);
  for (auto e : ctx->ev_ebp)
    if (e) cudaEventDestroy(e);
  if (ctx->side) cudaStreamDestroy(ctx->side);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return EMSESG_OK;
}

extern "C" int emsesg_last_error(const emsesg_ctx* ctx, char* buf, size_t len) {
  if (!ctx || !buf || len == 0) return EMSESG_ERR_ARG;
  size_t n = std::min(len - 1, ctx->err.size());
  std::memcpy(buf, ctx->err.data(), n);
  buf[n] = 0;
  return EMSESG_OK;
}

extern "C" void* emsesg_stream(emsesg_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

extern "C" int emsesg_synchronize(emsesg_ctx* ctx) {
  if (!ctx) return EMSESG_ERR_ARG;
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  int st = 0;
  EMSESG_CUDA(ctx, cudaMemcpy(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st) {
    long long diag[4] = {0, 0, 0, 0};
    cudaMemcpy(diag, ctx->d_diag, sizeof diag, cudaMemcpyDeviceToHost);
    cudaMemset(ctx->d_status, 0, sizeof(int));
    cudaMemset(ctx->d_diag, 0, sizeof diag);
    if (st & ST_RANDOMS) return set_error(ctx, EMSESG_ERR_ARG, "pre-drawn random numbers exhausted");
    if (st & ST_OVERFLOW) return set_error(ctx, EMSESG_ERR_OVERFLOW, "particle capacity exceeded");
    static const char* sites[] = {"?", "psolve2", "psolve1", "charge", "fx_load", "fx_push", "fx_deposit",
                                  "fx_flush", "fx_sort"};
    int site = (diag[0] >= 0 && diag[0] <= 8) ? (int)diag[0] : 0;
    return set_error(ctx, EMSESG_ERR_DEVICE,
                     "a kernel met a particle outside the field arrays (status %d, site %s, index %lld, cell %lld)",
                     st, sites[site], diag[1], diag[2]);
  }
  return EMSESG_OK;
}

extern "C" int emsesg_field_size(const emsesg_ctx* ctx, int field, int64_t* n) {
  if (!ctx || !n || field < 0 || field >= EMSESG_NFIELDS) return EMSESG_ERR_ARG;
  *n = field_doubles(ctx->cfg, field);
  return EMSESG_OK;
}

static int check_ps(emsesg_ctx* ctx, int ps) {
  if (!ctx) return EMSESG_ERR_ARG;
  if (ps == 2) return set_error(ctx, EMSESG_ERR_UNSUPPORTED, "ps=2 (helper subdomain) is not supported on one rank");
  if (ps != 1) return set_error(ctx, EMSESG_ERR_ARG, "ps must be 1");
  return EMSESG_OK;
}

extern "C" int emsesg_upload_particles(emsesg_ctx* ctx, int ps, const emsesg_particle* pbuf,
                                       const int64_t* totalp) {
  int rc = check_ps(ctx, ps);
  if (rc) return rc;
  if (!pbuf || !totalp) return set_error(ctx, EMSESG_ERR_ARG, "null argument");
  if (ctx->cfg.flags & EMSESG_FLAG_FP32_ONLY)
    return set_error(ctx, EMSESG_ERR_STATE, "FP32-only context: no FP64 particle records");
  for (int is = 0; is < ctx->cfg.nspec; is++)
    if (totalp[is] < 0 || totalp[is] > ctx->seg.capacity[is])
      return set_error(ctx, EMSESG_ERR_OVERFLOW, "species %d: %lld particles exceed capacity %lld", is + 1,
                       (long long)totalp[is], (long long)ctx->seg.capacity[is]);
  int64_t off = 0;
  for (int is = 0; is < ctx->cfg.nspec; is++) {
    if (totalp[is])
      EMSESG_CUDA(ctx, cudaMemcpyAsync(ctx->pbuf + ctx->seg.base[is], pbuf + off, totalp[is] * sizeof(emsesg_particle),
                                       cudaMemcpyHostToDevice, ctx->stream));
    off += totalp[is];
    ctx->totalp[is] = totalp[is];
  }
  EMSESG_CUDA(ctx, cudaMemcpyAsync(ctx->d_count, ctx->totalp, EMSESG_ISPEC * sizeof(int64_t), cudaMemcpyHostToDevice,
                                   ctx->stream));
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->fx.loaded = false;
  return EMSESG_OK;
}

extern "C" int emsesg_download_particles(emsesg_ctx* ctx, int ps, emsesg_particle* pbuf, int64_t* totalp) {
  int rc = check_ps(ctx, ps);
  if (rc) return rc;
  if (ctx->cfg.flags & EMSESG_FLAG_FP32_ONLY)
    return set_error(ctx, EMSESG_ERR_STATE, "FP32-only context: no FP64 particle records");
  EMSESG_CUDA(ctx, cudaMemcpyAsync(ctx->totalp, ctx->d_count, EMSESG_ISPEC * sizeof(int64_t), cudaMemcpyDeviceToHost,
                                   ctx->stream));
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  int64_t off = 0;
  for (int is = 0; is < ctx->cfg.nspec; is++) {
    if (pbuf && ctx->totalp[is])
      EMSESG_CUDA(ctx, cudaMemcpyAsync(pbuf + off, ctx->pbuf + ctx->seg.base[is], ctx->totalp[is] * sizeof(emsesg_particle),
                                       cudaMemcpyDeviceToHost, ctx->stream));
    off += ctx->totalp[is];
    if (totalp) totalp[is] = ctx->totalp[is];
  }
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return emsesg_synchronize(ctx);
}

extern "C" int emsesg_upload_field(emsesg_ctx* ctx, int field, const double* host) {
  if (!ctx || !host || field < 0 || field >= EMSESG_NFIELDS) return set_error(ctx, EMSESG_ERR_ARG, "bad field");
  if (field == EMSESG_FIELD_WRK) return set_error(ctx, EMSESG_ERR_ARG, "wrk is produced by grdcrt");
  if (field == EMSESG_FIELD_EB && ctx->eb_next_pending) {  // this upload replaces a pending one
    EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->side));
    ctx->eb_next_pending = false;
  }
  int64_t n = field_doubles(ctx->cfg, field);
  EMSESG_CUDA(ctx, cudaMemcpyAsync(ctx->field[field], host, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  return EMSESG_OK;
}

namespace emsesg {
int side_stream(emsesg_ctx* ctx) {
  if (ctx->side) return EMSESG_OK;
  EMSESG_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
  EMSESG_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_fields, cudaEventDisableTiming));
  EMSESG_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_eb, cudaEventDisableTiming));
  // no step yet: the first copy waits for the work queued so far
  EMSESG_CUDA(ctx, cudaEventRecord(ctx->ev_fields, ctx->stream));
  return EMSESG_OK;
}

int apply_pending_eb(emsesg_ctx* ctx) {
  if (!ctx->eb_next_pending) return EMSESG_OK;
  EMSESG_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_eb, 0));
  std::swap(ctx->field[EMSESG_FIELD_EB], ctx->eb_next);
  ctx->eb_next_pending = false;
  return EMSESG_OK;
}
}  // namespace emsesg

extern "C" int emsesg_upload_field_async(emsesg_ctx* ctx, int field, const double* host) {
  if (!ctx || !host) return EMSESG_ERR_ARG;
  if (field != EMSESG_FIELD_EB) return set_error(ctx, EMSESG_ERR_ARG, "asynchronous upload: eb only");
  int rc = side_stream(ctx);
  if (rc) return rc;
  const int64_t n = field_doubles(ctx->cfg, field);
  if (!ctx->eb_next) EMSESG_CUDA(ctx, cudaMalloc(&ctx->eb_next, n * sizeof(double)));
  // the buffer was last read before the last step's field phase ended
  EMSESG_CUDA(ctx, cudaStreamWaitEvent(ctx->side, ctx->ev_fields, 0));
  // for the FP32 step: in z chunks, each with its event, so that the push's
  // parts start while the later planes are still on their way
  ctx->eb_parts = emsesg::fx_eb_plan(ctx, ctx->eb_zready, ctx->eb_tile);
  if (ctx->eb_parts > 1) {
    const emsesg::FieldDesc fe = emsesg::field_desc(ctx->cfg, EMSESG_FIELD_EB);
    const int64_t plane = (int64_t)fe.nc * fe.ex * fe.ey;  // doubles of one z plane
    int64_t done = 0;
    for (int p = 0; p < ctx->eb_parts; p++) {
      if (!ctx->ev_ebp[p]) EMSESG_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_ebp[p], cudaEventDisableTiming));
      // node plane k reads the eb planes k - 1 and k
      const int64_t upto =
          p + 1 == ctx->eb_parts ? n : std::min(n, (int64_t)(ctx->eb_zready[p] - fe.lo + 1) * plane);
      if (upto > done) {
        EMSESG_CUDA(ctx, cudaMemcpyAsync(ctx->eb_next + done, host + done, (upto - done) * sizeof(double),
                                         cudaMemcpyHostToDevice, ctx->side));
        done = upto;
      }
      EMSESG_CUDA(ctx, cudaEventRecord(ctx->ev_ebp[p], ctx->side));
    }
  } else {
    EMSESG_CUDA(ctx, cudaMemcpyAsync(ctx->eb_next, host, n * sizeof(double), cudaMemcpyHostToDevice, ctx->side));
  }
  EMSESG_CUDA(ctx, cudaEventRecord(ctx->ev_eb, ctx->side));
  ctx->eb_next_pending = true;
  return EMSESG_OK;
}

extern "C" int emsesg_zero_field(emsesg_ctx* ctx, int field) {
  if (!ctx || field < 0 || field >= EMSESG_NFIELDS) return set_error(ctx, EMSESG_ERR_ARG, "bad field");
  int64_t n = field_doubles(ctx->cfg, field);
  EMSESG_CUDA(ctx, cudaMemsetAsync(ctx->field[field], 0, n * sizeof(double), ctx->stream));
  return EMSESG_OK;
}

namespace emsesg {
int download_wrk(emsesg_ctx* ctx, double* host);  // dropin.cu
}

extern "C" int emsesg_download_field(emsesg_ctx* ctx, int field, double* host) {
  if (!ctx || !host || field < 0 || field >= EMSESG_NFIELDS) return set_error(ctx, EMSESG_ERR_ARG, "bad field");
  if (field == EMSESG_FIELD_EB) {
    int rc = apply_pending_eb(ctx);
    if (rc) return rc;
  }
  if (field == EMSESG_FIELD_WRK) return download_wrk(ctx, host);
  int64_t n = field_doubles(ctx->cfg, field);
  EMSESG_CUDA(ctx, cudaMemcpyAsync(host, ctx->field[field], n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return EMSESG_OK;
}

extern "C" int emsesg_set_counters(emsesg_ctx* ctx, const emsesg_counter* gc) {
  if (!ctx || !gc) return EMSESG_ERR_ARG;
  EMSESG_CUDA(ctx, cudaMemcpyAsync(ctx->d_counter, gc, sizeof(emsesg_counter), cudaMemcpyHostToDevice, ctx->stream));
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return EMSESG_OK;
}

extern "C" int emsesg_get_counters(emsesg_ctx* ctx, emsesg_counter* gc) {
  if (!ctx || !gc) return EMSESG_ERR_ARG;
  EMSESG_CUDA(ctx, cudaMemcpyAsync(gc, ctx->d_counter, sizeof(emsesg_counter), cudaMemcpyDeviceToHost, ctx->stream));
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return EMSESG_OK;
}

extern "C" int emsesg_set_randoms(emsesg_ctx* ctx, const double* u, int64_t n) {
  if (!ctx || (n > 0 && !u) || n < 0) return EMSESG_ERR_ARG;
  EMSESG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  cudaFree(ctx->d_randoms);
  ctx->d_randoms = nullptr;
  ctx->n_randoms = n;
  if (n > 0) {
    EMSESG_CUDA(ctx, cudaMalloc(&ctx->d_randoms, n * sizeof(double)));
    EMSESG_CUDA(ctx, cudaMemcpy(ctx->d_randoms, u, n * sizeof(double), cudaMemcpyHostToDevice));
  }
  EMSESG_CUDA(ctx, cudaMemset(ctx->d_rand_pos, 0, sizeof(int64_t)));
  return EMSESG_OK;
}

extern "C" int emsesg_set_profiling(emsesg_ctx* ctx, int on) {
  if (!ctx) return EMSESG_ERR_ARG;
  if (!on) timer_collect(ctx);
  ctx->timer.on = on != 0;
  return EMSESG_OK;
}

extern "C" int emsesg_profile_reset(emsesg_ctx* ctx) {
  if (!ctx) return EMSESG_ERR_ARG;
  timer_collect(ctx);
  ctx->timer.total.clear();
  return EMSESG_OK;
}

extern "C" int emsesg_profile_report(emsesg_ctx* ctx, char* buf, size_t len) {
  if (!ctx || !buf || len == 0) return EMSESG_ERR_ARG;
  timer_collect(ctx);
  std::string s;
  for (auto& kv : ctx->timer.total) {
    char line[256];
    snprintf(line, sizeof line, "%s %.6f %lld\n", kv.first.c_str(), kv.second.ms, (long long)kv.second.launches);
    s += line;
  }
  size_t n = std::min(len - 1, s.size());
  std::memcpy(buf, s.data(), n);
  buf[n] = 0;
  return EMSESG_OK;
}
