// C ABI of keldy_b200 (declared in include/keldy_b200.h): argument checks, device
// memory, and the launch sequences of the kernels in tree.cu / misc_kernels.cu.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "kb_host.h"

namespace kb {
void sobol_setup(int dim, int m, bool do_shift, bool do_scramble, int seed_shift, uint32_t *Csr, uint32_t *shfr);
}

using namespace kb;

namespace kb {
namespace {
thread_local std::string g_last_error;
}
int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}
} // namespace kb

extern "C" {

const char *kb_last_error(void) { return g_last_error.c_str(); }

int kb_version(void) { return 100; }

uint64_t kb_device_allocations(void) { return device_allocations().load(); }

int kb_context_create(int device, kb_context **out) {
  KB_CHECK(out, "kb_context_create: out is NULL");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(KB_E_NODEVICE, "keldy_b200 needs a CUDA device and found none (" +
                                   std::string(cudaGetErrorString(e)) + "); the library has no CPU path");
  KB_CHECK(device >= 0 && device < n, "kb_context_create: device index out of range");
  KB_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  KB_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return fail(KB_E_NODEVICE, std::string("keldy_b200 is built for sm_100a; device is ") + prop.name);
  KB_CUDA(configure_kernels());
  KB_CUDA(flow_configure());
  auto *ctx = new kb_context;
  ctx->device = device;
  ctx->sm_count = prop.multiProcessorCount;
  for (int n = 0; n <= MAX_ORDER; ++n) ctx->chunk_points[n] = CHUNK_POINTS;
  e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete ctx;
    return fail(KB_E_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  }
  // Every upload goes through the library's stream: it does not synchronise with the
  // legacy default stream, and a plain cudaMemcpy from pageable memory may return before
  // its data has landed.
  e = device_malloc(&ctx->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return fail(KB_E_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  // Persistent tree kernel: as many CTAs as fit on the device at once.
  int per_sm = 4;
  ctx->tree_grid = ctx->sm_count * per_sm;
  *out = ctx;
  return KB_OK;
}

int kb_context_destroy(kb_context *ctx) {
  if (!ctx) return KB_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto &e : ctx->ev)
    if (e) cudaEventDestroy(e);
  cudaFree(ctx->d_err);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return KB_OK;
}

int kb_context_synchronize(kb_context *ctx) {
  KB_CHECK(ctx, "null context");
  KB_CUDA(cudaStreamSynchronize(ctx->stream));
  return KB_OK;
}

void *kb_context_stream(kb_context *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int kb_context_set_timing(kb_context *ctx, int enable) {
  KB_CHECK(ctx, "null context");
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  if (enable && !ctx->ev[0])
    for (auto &e : ctx->ev) KB_CUDA(cudaEventCreate(&e));
  ctx->timing = enable != 0;
  return KB_OK;
}

int kb_context_last_timing(kb_context *ctx, double *integrand_ms, double *fallback_ms, double *reduce_ms,
                           int *launches) {
  KB_CHECK(ctx, "null context");
  if (integrand_ms) *integrand_ms = ctx->last_ms[0];
  if (fallback_ms) *fallback_ms = ctx->last_ms[1];
  if (reduce_ms) *reduce_ms = ctx->last_ms[2];
  if (launches) *launches = ctx->last_launches;
  return KB_OK;
}

// ------------------------------------------------------------------ Sobol
int kb_sobol_create(kb_context *ctx, int dim, int log_max_points, int do_shift, int do_scramble, int seed_shift,
                    kb_sobol **out) {
  KB_CHECK(ctx && out, "kb_sobol_create: null argument");
  KB_CHECK(dim >= 1 && dim <= 250, "Sobol dimension must be in [1, 250]");
  if (log_max_points > 31) return fail(KB_E_INVALID, "To many points requested from Sobol generator.");
  KB_CHECK(log_max_points >= 1, "log_max_points must be >= 1");
  std::vector<uint32_t> Csr(static_cast<size_t>(dim) * log_max_points), shfr(static_cast<size_t>(dim));
  sobol_setup(dim, log_max_points, do_shift != 0, do_scramble != 0, seed_shift, Csr.data(), shfr.data());
  auto *s = new kb_sobol;
  s->ctx = ctx;
  s->device = ctx->device;
  s->dim = dim;
  s->m = log_max_points;
  std::lock_guard<std::mutex> lk(ctx->mu); // the upload uses the context's stream
  cudaSetDevice(ctx->device);
  cudaError_t e = device_malloc(&s->d_Csr, Csr.size() * sizeof(uint32_t));
  if (e == cudaSuccess) e = device_malloc(&s->d_shfr, shfr.size() * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_Csr, Csr.data(), Csr.size() * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->d_shfr, shfr.data(), shfr.size() * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    cudaFree(s->d_Csr);
    cudaFree(s->d_shfr);
    delete s;
    return fail(KB_E_CUDA, std::string("kb_sobol_create: ") + cudaGetErrorString(e));
  }
  *out = s;
  return KB_OK;
}

int kb_sobol_matrices(int dim, int log_max_points, int do_shift, int do_scramble, int seed_shift, uint32_t *Csr,
                      uint32_t *shfr) {
  KB_CHECK(Csr && shfr, "kb_sobol_matrices: null argument");
  KB_CHECK(dim >= 1 && dim <= 250, "Sobol dimension must be in [1, 250]");
  if (log_max_points > 31) return fail(KB_E_INVALID, "To many points requested from Sobol generator.");
  KB_CHECK(log_max_points >= 1, "log_max_points must be >= 1");
  sobol_setup(dim, log_max_points, do_shift != 0, do_scramble != 0, seed_shift, Csr, shfr);
  return KB_OK;
}

int kb_sobol_destroy(kb_sobol *s) {
  if (!s) return KB_OK;
  cudaSetDevice(s->device); // cudaFree waits for the device's pending work
  cudaFree(s->d_Csr);
  cudaFree(s->d_shfr);
  delete s;
  return KB_OK;
}

} // extern "C"

SobolDev kb::sobol_dev(const kb_sobol *s) {
  SobolDev d;
  d.Csr = s->d_Csr;
  d.shfr = s->d_shfr;
  d.dim = s->dim;
  d.m = s->m;
  return d;
}

int kb::check_sobol_range(const kb_sobol *s, uint32_t k_first, int64_t count) {
  if (k_first < 1) return fail(KB_E_INVALID, "Sobol point index must be >= 1 (first draw of sobol(dim, seed) is seed+1)");
  // the last point keldy's generator hands out is k = 2^m (past_end() is checked before next())
  uint64_t last = (uint64_t)k_first + (uint64_t)(count > 0 ? count - 1 : 0);
  if (count > 0 && last > (1ull << s->m))
    return fail(KB_E_EXHAUSTED, "More sample points requested then generator can hold.");
  return KB_OK;
}

extern "C" {

int kb_sobol_points_dev(kb_context *ctx, const kb_sobol *s, uint32_t k_first, int64_t count, double *out_dev) {
  KB_CHECK(ctx && s, "kb_sobol_points: null argument");
  KB_CHECK(count >= 0, "count must be >= 0");
  int st = check_sobol_range(s, k_first, count);
  if (st) return st;
  KB_CUDA(cudaSetDevice(ctx->device));
  KB_CUDA(launch_sobol_points(sobol_dev(s), k_first, count, out_dev, ctx->stream));
  return KB_OK;
}

int kb_sobol_points(kb_context *ctx, const kb_sobol *s, uint32_t k_first, int64_t count, double *out) {
  KB_CHECK(ctx && s && (out || count == 0), "kb_sobol_points: null argument");
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  DevBuf d;
  size_t bytes = (size_t)count * s->dim * sizeof(double);
  KB_CUDA(d.alloc(bytes, ctx->stream));
  int st = kb_sobol_points_dev(ctx, s, k_first, count, d.as<double>());
  if (st) return st;
  KB_CUDA(cudaMemcpyAsync(out, d.p, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  KB_CUDA(cudaStreamSynchronize(ctx->stream));
  return KB_OK;
}

// ---------------------------------------------------------------- warpers
// Maker constants, evaluated as keldy's makers do (long double norms) and rounded.
static int make_warper_dev(const kb_warper &w, WarperDev &d) {
  memset(&d, 0, sizeof(d));
  d.kind = w.kind;
  d.power = w.power;
  d.u_max = w.u_max;
  d.w = w.w;
  switch (w.kind) {
  case KB_WARPER_IDENTITY:
    return KB_OK;
  case KB_WARPER_PLASMA_UV:
    return KB_OK;
  case KB_WARPER_UNIFORM:
    if (!(w.u_max > 0.0)) return fail(KB_E_INVALID, "coord_domain_u coordinates must be ordered.");
    return KB_OK;
  case KB_WARPER_EXPONENTIAL: {
    if (!(w.u_max > 0.0)) return fail(KB_E_INVALID, "coord_domain_u coordinates must be ordered.");
    if (!(w.w > 0.0)) return fail(KB_E_INVALID, "w_scale must be > 0");
    long double norm = -std::expm1(-static_cast<long double>(w.u_max) / w.w);
    d.c[0] = std::expm1(w.u_max / w.w);
    d.c[1] = static_cast<double>(static_cast<long double>(w.w) * norm);
    return KB_OK;
  }
  case KB_WARPER_INVERSE: {
    if (!(w.u_max > 0.0)) return fail(KB_E_INVALID, "coord_domain_u coordinates must be ordered.");
    if (!(w.w > 0.0)) return fail(KB_E_INVALID, "w_scale must be > 0");
    d.c[0] = static_cast<double>(std::log1p(static_cast<long double>(w.u_max) / w.w));
    return KB_OK;
  }
  case KB_WARPER_INVERSE_SQUARE: {
    if (!(w.u_max > 0.0)) return fail(KB_E_INVALID, "coord_domain_u coordinates must be ordered.");
    if (!(w.w > 0.0)) return fail(KB_E_INVALID, "w_scale must be > 0");
    d.c[0] = static_cast<double>(static_cast<long double>(w.u_max) / (w.w + w.u_max));
    return KB_OK;
  }
  case KB_WARPER_INVERSE_POWER: {
    if (!(w.u_max > 0.0)) return fail(KB_E_INVALID, "coord_domain_u coordinates must be ordered.");
    if (!(w.w > 0.0)) return fail(KB_E_INVALID, "w_scale must be > 0");
    if (w.power < 1) return fail(KB_E_INVALID, "inverse_power warper needs power >= 1");
    if (w.power == 1) { // make_product_1d_simple_inverse_power(1, ...) is the inverse maker
      kb_warper v = w;
      v.kind = KB_WARPER_INVERSE;
      return make_warper_dev(v, d);
    }
    long double u_max = w.u_max;
    int p = w.power;
    long double den = std::pow(u_max / w.w + 1, p - 1) - 1;
    d.c[0] = static_cast<double>((p - 1) * std::pow(u_max + w.w, p - 1) / den);
    d.c[1] = static_cast<double>(std::pow(u_max + w.w, p - 1) / den);
    d.c[2] = static_cast<double>(std::pow(w.w / (u_max + w.w), p - 1) - 1);
    return KB_OK;
  }
  case KB_WARPER_TABLE:
    if (!w.table) return fail(KB_E_INVALID, "tabulated warper without a table");
    d.tab = w.table->d_dims;
    d.ntab = w.table->ndims;
    d.u_max = w.table->u_max;
    return KB_OK;
  default:
    return fail(KB_E_INVALID, "unknown warper kind " + std::to_string(w.kind));
  }
}

} // extern "C"

namespace kb {
int simple_dev(const kb_warper &w, SimpleDev &out) {
  WarperDev d;
  int st = make_warper_dev(w, d);
  if (st) return st;
  out.kind = d.kind;
  out.power = d.power;
  out.u_max = d.u_max;
  out.w = d.w;
  for (int i = 0; i < 3; ++i) out.c[i] = d.c[i];
  return KB_OK;
}
} // namespace kb

extern "C" {

// A product warper with one 1D warper per coordinate maps coordinate i with warper i
// (keldy's ui_from_li enumerates the point's coordinates, product_1d.hpp and
// projection.hpp:330-344): it needs at least as many warpers as coordinates; one 1D
// warper maps every coordinate.
static int check_chain_dims(const kb_warper *chain, int len, int n) {
  for (int i = 0; i < len; ++i)
    if (chain[i].kind == KB_WARPER_TABLE && chain[i].table && chain[i].table->ndims != 1 &&
        chain[i].table->ndims < n)
      return fail(KB_E_INVALID, "the tabulated warper has " + std::to_string(chain[i].table->ndims) +
                                    " tables for " + std::to_string(n) + " coordinates");
  return KB_OK;
}

static int make_chain(const kb_warper *chain, int len, WarperDev *out) {
  if (len < 0 || len > KB_MAX_CHAIN) return fail(KB_E_INVALID, "warper chain longer than KB_MAX_CHAIN");
  if (len > 0 && !chain) return fail(KB_E_INVALID, "null warper chain");
  for (int i = 0; i < KB_MAX_CHAIN; ++i) memset(&out[i], 0, sizeof(WarperDev));
  for (int i = 0; i < len; ++i) {
    int st = make_warper_dev(chain[i], out[i]);
    if (st) return st;
  }
  return KB_OK;
}

int kb_warp(kb_context *ctx, const kb_warper *chain, int chain_len, int direction, int start, int end, int n,
            int64_t count, const double *in, double *out, double *jac) {
  KB_CHECK(ctx, "null context");
  if (chain_len > 0 && chain) {
    int cd = check_chain_dims(chain, chain_len, n);
    if (cd) return cd;
  }
  KB_CHECK(n >= 0 && n <= MAX_ORDER, "number of coordinates must be in [0, 16]");
  KB_CHECK(count >= 0 && (count == 0 || (in && out)), "kb_warp: null buffer");
  KB_CHECK(direction == KB_REVERSE || direction == KB_FORWARD, "direction must be KB_REVERSE or KB_FORWARD");
  if (direction == KB_REVERSE)
    KB_CHECK(0 <= end && end <= start && start <= chain_len, "map_reverse needs 0 <= end <= start <= size");
  else
    KB_CHECK(0 <= start && start <= end && end <= chain_len, "map_forward needs 0 <= start <= end <= size");
  WarperDev w[KB_MAX_CHAIN];
  int st = make_chain(chain, chain_len, w);
  if (st) return st;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  size_t bytes = (size_t)count * n * sizeof(double);
  DevBuf dw, din, dout, djac;
  KB_CUDA(dw.alloc(sizeof(w), ctx->stream));
  KB_CUDA(din.alloc(bytes, ctx->stream));
  KB_CUDA(dout.alloc(bytes, ctx->stream));
  KB_CUDA(djac.alloc((size_t)count * sizeof(double), ctx->stream));
  KB_CUDA(cudaMemcpyAsync(dw.p, w, sizeof(w), cudaMemcpyHostToDevice, ctx->stream));
  KB_CUDA(cudaMemcpyAsync(din.p, in, bytes, cudaMemcpyHostToDevice, ctx->stream));
  KB_CUDA(launch_warp(dw.as<WarperDev>(), start, end, direction, n, count, din.as<double>(), dout.as<double>(),
                      djac.as<double>(), ctx->stream));
  KB_CUDA(cudaMemcpyAsync(out, dout.p, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (jac) KB_CUDA(cudaMemcpyAsync(jac, djac.p, (size_t)count * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  KB_CUDA(cudaStreamSynchronize(ctx->stream));
  return KB_OK;
}

// ---------------------------------------------------------------- model
int kb_model_create(kb_context *ctx, int npts, double time_max, double alpha, kb_model **out) {
  KB_CHECK(ctx && out, "kb_model_create: null argument");
  KB_CHECK(npts >= 2, "g0 tables need at least 2 mesh points");
  KB_CHECK(time_max > 0.0 && std::isfinite(time_max), "time_max must be > 0");
  auto *m = new kb_model;
  m->ctx = ctx;
  m->device = ctx->device;
  m->npts = npts;
  m->tmax = time_max;
  m->alpha = alpha;
  *out = m;
  return KB_OK;
}

int kb_model_destroy(kb_model *m) {
  if (!m) return KB_OK;
  cudaSetDevice(m->device); // cudaFree waits for the device's pending work
  for (int s = 0; s < 2; ++s)
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        if (!(m->slab && s == 0 && a == 0 && b == 0)) cudaFree(m->tab[s][a][b]);
  delete m; // releases its share of a slab
  return KB_OK;
}

static int set_table(kb_model *m, int spin, int o1, int o2, const double *lesser, const double *greater,
                     cudaMemcpyKind kind) {
  KB_CHECK(m && lesser && greater, "kb_model_set_table: null argument");
  KB_CHECK(spin >= 0 && spin < 2 && o1 >= 0 && o1 < 2 && o2 >= 0 && o2 < 2, "spin/orbital index out of range");
  kb_context *ctx = m->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  const size_t n = (size_t)m->npts;
  if (!m->tab[spin][o1][o2]) KB_CUDA(device_malloc(&m->tab[spin][o1][o2], n * 2 * sizeof(double2)));
  double2 *dst = m->tab[spin][o1][o2];
  // interleave lesser/greater per mesh point
  KB_CUDA(cudaMemcpy2DAsync(dst, 2 * sizeof(double2), lesser, sizeof(double2), sizeof(double2), n, kind,
                            ctx->stream));
  KB_CUDA(cudaMemcpy2DAsync(dst + 1, 2 * sizeof(double2), greater, sizeof(double2), sizeof(double2), n, kind,
                            ctx->stream));
  double tmax_tab = 0.0;
  if (kind == cudaMemcpyHostToDevice) {
    double mx = 0.0;
    for (size_t i = 0; i < n; ++i) {
      mx = std::max(mx, fabs(lesser[2 * i]) + fabs(lesser[2 * i + 1]));
      mx = std::max(mx, fabs(greater[2 * i]) + fabs(greater[2 * i + 1]));
    }
    tmax_tab = mx;
    m->hash[spin][o1][o2] = fnv1a(lesser, n * 16) ^ (fnv1a(greater, n * 16) * 31ULL) ^ 1ULL;
  } else {
    DevBuf d;
    KB_CUDA(d.alloc(sizeof(double), ctx->stream));
    KB_CUDA(launch_table_max(dst, m->npts, d.as<double>(), ctx->stream));
    KB_CUDA(cudaMemcpyAsync(&tmax_tab, d.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    m->hash[spin][o1][o2] = 0;
  }
  KB_CUDA(cudaStreamSynchronize(ctx->stream));
  if (!std::isfinite(tmax_tab)) return fail(KB_E_INVALID, "g0 table contains non-finite values");
  m->tabmax = std::max(m->tabmax, tmax_tab);
  return KB_OK;
}

int kb_model_set_table(kb_model *m, int spin, int o1, int o2, const double *lesser, const double *greater) {
  return set_table(m, spin, o1, o2, lesser, greater, cudaMemcpyHostToDevice);
}

int kb_model_set_table_dev(kb_model *m, int spin, int o1, int o2, const double *lesser_dev,
                           const double *greater_dev) {
  return set_table(m, spin, o1, o2, lesser_dev, greater_dev, cudaMemcpyDeviceToDevice);
}

} // extern "C"

namespace {
// Gauss-Legendre rule of n nodes on [-1, 1]: Newton iteration on P_n from the
// Chebyshev-like first guesses, P_n and P_n' by the three-term recurrence.
void gauss_legendre(int n, double *x, double *w) {
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = std::cos(pi * (i + 0.75) / (n + 0.5)), dp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = 0.0;
      for (int j = 1; j <= n; ++j) {
        const double p2 = p1;
        p1 = p0;
        p0 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p2) / j;
      }
      dp = n * (z * p0 - p1) / (z * z - 1.0);
      const double dz = p0 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = -z;
    x[n - 1 - i] = z;
    w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}
} // namespace

extern "C" {

int kb_model_get_table(kb_model *m, int spin, int o1, int o2, double *lesser, double *greater) {
  KB_CHECK(m && lesser && greater, "kb_model_get_table: null argument");
  KB_CHECK(spin >= 0 && spin < 2 && o1 >= 0 && o1 < 2 && o2 >= 0 && o2 < 2, "spin/orbital index out of range");
  const double2 *src = m->tab[spin][o1][o2] ? m->tab[spin][o1][o2] : m->tab[1 - spin][o1][o2];
  if (!src) return fail(KB_E_INVALID, "kb_model_get_table: no table for this block");
  kb_context *ctx = m->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  const size_t n = (size_t)m->npts;
  KB_CUDA(cudaMemcpy2DAsync(lesser, sizeof(double2), src, 2 * sizeof(double2), sizeof(double2), n,
                            cudaMemcpyDeviceToHost, ctx->stream));
  KB_CUDA(cudaMemcpy2DAsync(greater, sizeof(double2), src + 1, 2 * sizeof(double2), sizeof(double2), n,
                            cudaMemcpyDeviceToHost, ctx->stream));
  KB_CUDA(cudaStreamSynchronize(ctx->stream));
  return KB_OK;
}

int kb_models_set_flatband(int n, kb_model *const *models, const double *params) {
  KB_CHECK(n >= 0 && (n == 0 || (models && params)), "kb_models_set_flatband: null argument");
  if (n == 0) return KB_OK;
  kb_context *ctx = models[0] ? models[0]->ctx : nullptr;
  KB_CHECK(ctx, "kb_models_set_flatband: null model");
  const int npts = models[0]->npts;
  const double tmax = models[0]->tmax;
  KB_CHECK(npts % 2 == 1 && npts >= 3, "the flat-band builder needs an odd number of mesh points (t = 0 on the mesh)");
  for (int i = 0; i < n; ++i) {
    KB_CHECK(models[i] && models[i]->ctx == ctx, "all models of one call must belong to one context");
    KB_CHECK(models[i]->npts == npts && models[i]->tmax == tmax, "all models of one call must share their time mesh");
    const double *p = params + 4 * i;
    KB_CHECK(p[0] > 0.0 && std::isfinite(p[0]), "Gamma must be > 0");
    KB_CHECK(std::isfinite(p[1]) && std::isfinite(p[2]), "eps_d and V must be finite");
    KB_CHECK(p[3] > 0.0, "beta must be > 0 (INFINITY: zero temperature)");
  }
  constexpr int NODES = 240;
  std::vector<double> gx(NODES), gw(NODES);
  gauss_legendre(NODES, gx.data(), gw.data());
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  std::vector<double2 *> tabs((size_t)n);
  // models without a dot table get slices of one allocation (one cudaMalloc for the call,
  // not one per model)
  size_t fresh = 0;
  for (int i = 0; i < n; ++i) fresh += models[i]->tab[0][0][0] ? 0 : 1;
  if (fresh) {
    const size_t per = (size_t)npts * 2;
    double2 *block = nullptr;
    KB_CUDA(device_malloc(&block, fresh * per * sizeof(double2)));
    const int dev = ctx->device;
    std::shared_ptr<void> slab(block, [dev](void *q) {
      cudaSetDevice(dev);
      cudaFree(q);
    });
    size_t k = 0;
    for (int i = 0; i < n; ++i)
      if (!models[i]->tab[0][0][0]) {
        models[i]->tab[0][0][0] = block + (k++) * per;
        models[i]->slab = slab;
      }
  }
  for (int i = 0; i < n; ++i) tabs[(size_t)i] = models[i]->tab[0][0][0];
  DevBuf dpar, dtab, dx, dw, dmax;
  KB_CUDA(dpar.alloc((size_t)n * 4 * sizeof(double), st));
  KB_CUDA(dtab.alloc((size_t)n * sizeof(double2 *), st));
  KB_CUDA(dx.alloc(NODES * sizeof(double), st));
  KB_CUDA(dw.alloc(NODES * sizeof(double), st));
  KB_CUDA(dmax.alloc((size_t)n * sizeof(double), st));
  KB_CUDA(cudaMemcpyAsync(dpar.p, params, (size_t)n * 4 * sizeof(double), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemcpyAsync(dtab.p, tabs.data(), (size_t)n * sizeof(double2 *), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemcpyAsync(dx.p, gx.data(), NODES * sizeof(double), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemcpyAsync(dw.p, gw.data(), NODES * sizeof(double), cudaMemcpyHostToDevice, st));
  KB_CUDA(launch_flatband_tables(n, dpar.as<double>(), dtab.as<double2 *>(), npts, tmax, dx.as<double>(),
                                 dw.as<double>(), NODES, st));
  KB_CUDA(launch_tables_max(dtab.as<double2 *>(), n, npts, dmax.as<double>(), st));
  std::vector<double> mx((size_t)n);
  KB_CUDA(cudaMemcpyAsync(mx.data(), dmax.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaStreamSynchronize(st));
  for (int i = 0; i < n; ++i) {
    if (!std::isfinite(mx[(size_t)i])) return fail(KB_E_INVALID, "flat-band table has non-finite values");
    models[i]->hash[0][0][0] = 0;
    models[i]->tabmax = std::max(models[i]->tabmax, mx[(size_t)i]);
  }
  return KB_OK;
}

int kb_model_set_interpolation(kb_model *m, int order) {
  KB_CHECK(m, "null model");
  KB_CHECK(order == KB_INTERP_LINEAR || order == KB_INTERP_CUBIC, "interpolation order must be 1 or 3");
  KB_CHECK(order == KB_INTERP_LINEAR || m->npts >= 4, "cubic interpolation needs at least 4 mesh points");
  m->interp = order;
  return KB_OK;
}

int kb_model_set_fourier(kb_model *m, int o1, int o2, int n_nodes, const double *w, const double *cl,
                         const double *cg, int flags) {
  KB_CHECK(m && w && cl && cg, "kb_model_set_fourier: null argument");
  KB_CHECK(o1 >= 0 && o1 < 2 && o2 >= 0 && o2 < 2, "orbital index out of range");
  KB_CHECK(n_nodes >= 1 && n_nodes <= (1 << 24), "n_nodes must be in [1, 2^24]");
  KB_CHECK(!(flags & KB_FT_SYMMETRIC) || (m->npts % 2 == 1 && m->npts >= 3),
           "a symmetric block needs an odd number of mesh points (t = 0 on the mesh)");
  KB_CHECK(!(flags & KB_FT_MIRROR) || o1 != o2, "KB_FT_MIRROR needs an off-diagonal block");
  for (int k = 0; k < n_nodes; ++k)
    KB_CHECK(std::isfinite(w[k]) && std::isfinite(cl[2 * k]) && std::isfinite(cl[2 * k + 1]) &&
                 std::isfinite(cg[2 * k]) && std::isfinite(cg[2 * k + 1]),
             "quadrature nodes and weights must be finite");
  kb_context *ctx = m->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const size_t n = (size_t)m->npts;
  const bool mirror = (flags & KB_FT_MIRROR) != 0;
  if (!m->tab[0][o1][o2]) KB_CUDA(device_malloc(&m->tab[0][o1][o2], n * 2 * sizeof(double2)));
  if (mirror && !m->tab[0][o2][o1]) KB_CUDA(device_malloc(&m->tab[0][o2][o1], n * 2 * sizeof(double2)));
  DevBuf dw, dl, dg, dbad, dmax;
  KB_CUDA(dw.alloc((size_t)n_nodes * sizeof(double), st));
  KB_CUDA(dl.alloc((size_t)n_nodes * sizeof(double2), st));
  KB_CUDA(dg.alloc((size_t)n_nodes * sizeof(double2), st));
  KB_CUDA(dbad.alloc(sizeof(int), st));
  KB_CUDA(dmax.alloc(2 * sizeof(double), st));
  KB_CUDA(cudaMemcpyAsync(dw.p, w, (size_t)n_nodes * sizeof(double), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemcpyAsync(dl.p, cl, (size_t)n_nodes * sizeof(double2), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemcpyAsync(dg.p, cg, (size_t)n_nodes * sizeof(double2), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemsetAsync(dbad.p, 0, sizeof(int), st));
  KB_CUDA(launch_fourier_table(dw.as<double>(), dl.as<double2>(), dg.as<double2>(), n_nodes, m->tab[0][o1][o2],
                               m->npts, m->tmax, (flags & KB_FT_SYMMETRIC) ? 1 : 0, dbad.as<int>(), st));
  KB_CUDA(launch_table_max(m->tab[0][o1][o2], m->npts, dmax.as<double>(), st));
  if (mirror) KB_CUDA(launch_mirror_block(m->tab[0][o1][o2], m->tab[0][o2][o1], m->npts, st));
  int bad = 0;
  double mx = 0.0;
  KB_CUDA(cudaMemcpyAsync(&bad, dbad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaMemcpyAsync(&mx, dmax.p, sizeof(double), cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaStreamSynchronize(st));
  if (bad) return fail(KB_E_INVALID, "g0 table contains non-finite values");
  // spin down uses the spin-up blocks (model.cpp:209-211): drop any spin-down copy
  const int blocks[2][2] = {{o1, o2}, {o2, o1}};
  for (int k = 0; k < (mirror ? 2 : 1); ++k) {
    const int a = blocks[k][0], b = blocks[k][1];
    cudaFree(m->tab[1][a][b]);
    m->tab[1][a][b] = nullptr;
    m->hash[0][a][b] = 0;
    m->hash[1][a][b] = 0;
  }
  m->tabmax = std::max(m->tabmax, mx);
  return KB_OK;
}

int kb_model_set_rational(kb_model *m, int o1, int o2, int n_terms, const double *mu, const int *n_poles,
                          const double *poles, const double *residues, double beta, int flags) {
  KB_CHECK(m && mu && n_poles && poles && residues, "kb_model_set_rational: null argument");
  KB_CHECK(o1 >= 0 && o1 < 2 && o2 >= 0 && o2 < 2, "orbital index out of range");
  KB_CHECK(n_terms >= 1 && n_terms <= RATIONAL_MAX_TERMS, "n_terms must be in [1, 4]");
  KB_CHECK(beta > 0.0, "beta must be > 0 (INFINITY: zero temperature)");
  KB_CHECK(m->npts % 2 == 1 && m->npts >= 3,
           "the rational builder needs an odd number of mesh points (t = 0 on the mesh)");
  KB_CHECK(!(flags & KB_FT_MIRROR) || o1 != o2, "KB_FT_MIRROR needs an off-diagonal block");
  std::vector<RationalTermDev> terms((size_t)n_terms);
  int off = 0;
  for (int l = 0; l < n_terms; ++l) {
    RationalTermDev &T = terms[(size_t)l];
    memset(&T, 0, sizeof(T));
    KB_CHECK(n_poles[l] >= 1 && n_poles[l] <= RATIONAL_MAX_POLES, "each term has 1..8 poles");
    KB_CHECK(std::isfinite(mu[l]), "chemical potentials must be finite");
    T.mu = mu[l];
    T.n = n_poles[l];
    for (int k = 0; k < T.n; ++k, ++off) {
      T.z[k] = make_double2(poles[2 * off], poles[2 * off + 1]);
      T.r[k] = make_double2(residues[2 * off], residues[2 * off + 1]);
      KB_CHECK(std::isfinite(T.z[k].x) && std::isfinite(T.z[k].y) && std::isfinite(T.r[k].x) &&
                   std::isfinite(T.r[k].y),
               "poles and residues must be finite");
      KB_CHECK(T.z[k].y != 0.0, "poles must lie off the real axis");
    }
  }
  constexpr int NODES = 240;
  std::vector<double> gx(NODES), gw(NODES);
  gauss_legendre(NODES, gx.data(), gw.data());
  kb_context *ctx = m->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const size_t n = (size_t)m->npts;
  const bool mirror = (flags & KB_FT_MIRROR) != 0;
  if (!m->tab[0][o1][o2]) KB_CUDA(device_malloc(&m->tab[0][o1][o2], n * 2 * sizeof(double2)));
  if (mirror && !m->tab[0][o2][o1]) KB_CUDA(device_malloc(&m->tab[0][o2][o1], n * 2 * sizeof(double2)));
  DevBuf dterms, dx, dw, dbad, dmax;
  KB_CUDA(dterms.alloc(terms.size() * sizeof(RationalTermDev), st));
  KB_CUDA(dx.alloc(NODES * sizeof(double), st));
  KB_CUDA(dw.alloc(NODES * sizeof(double), st));
  KB_CUDA(dbad.alloc(sizeof(int), st));
  KB_CUDA(dmax.alloc(2 * sizeof(double), st));
  KB_CUDA(cudaMemcpyAsync(dterms.p, terms.data(), terms.size() * sizeof(RationalTermDev), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemcpyAsync(dx.p, gx.data(), NODES * sizeof(double), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemcpyAsync(dw.p, gw.data(), NODES * sizeof(double), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemsetAsync(dbad.p, 0, sizeof(int), st));
  KB_CUDA(launch_rational_table(dterms.as<RationalTermDev>(), n_terms, beta, dx.as<double>(), dw.as<double>(), NODES,
                                m->tab[0][o1][o2], m->npts, m->tmax, (flags & KB_FT_SYMMETRIC) ? 1 : 0,
                                dbad.as<int>(), st));
  KB_CUDA(launch_table_max(m->tab[0][o1][o2], m->npts, dmax.as<double>(), st));
  if (mirror) KB_CUDA(launch_mirror_block(m->tab[0][o1][o2], m->tab[0][o2][o1], m->npts, st));
  int bad = 0;
  double mx = 0.0;
  KB_CUDA(cudaMemcpyAsync(&bad, dbad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaMemcpyAsync(&mx, dmax.p, sizeof(double), cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaStreamSynchronize(st));
  if (bad) return fail(KB_E_INVALID, "g0 table contains non-finite values");
  const int blocks[2][2] = {{o1, o2}, {o2, o1}};
  for (int k = 0; k < (mirror ? 2 : 1); ++k) { // spin down uses the spin-up blocks (model.cpp:209-211)
    const int a = blocks[k][0], b = blocks[k][1];
    cudaFree(m->tab[1][a][b]);
    m->tab[1][a][b] = nullptr;
    m->hash[0][a][b] = 0;
    m->hash[1][a][b] = 0;
  }
  m->tabmax = std::max(m->tabmax, mx);
  return KB_OK;
}

int kb_model_set_fft(kb_model *m, int o1, int o2, const double *gl, const double *gg, int flags) {
  KB_CHECK(m && gl && gg, "kb_model_set_fft: null argument");
  KB_CHECK(o1 >= 0 && o1 < 2 && o2 >= 0 && o2 < 2, "orbital index out of range");
  KB_CHECK(m->npts % 2 == 1 && m->npts >= 3, "the fft method needs an odd number of mesh points (t = 0 on the mesh)");
  KB_CHECK(!(flags & KB_FT_MIRROR) || o1 != o2, "KB_FT_MIRROR needs an off-diagonal block");
  KB_CHECK((flags & ~KB_FT_MIRROR) == 0, "kb_model_set_fft takes only the KB_FT_MIRROR flag");
  const size_t n = (size_t)m->npts;
  for (size_t k = 0; k < 2 * n; ++k)
    KB_CHECK(std::isfinite(gl[k]) && std::isfinite(gg[k]), "frequency values must be finite");
  kb_context *ctx = m->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const bool mirror = (flags & KB_FT_MIRROR) != 0;
  if (!m->tab[0][o1][o2]) KB_CUDA(device_malloc(&m->tab[0][o1][o2], n * 2 * sizeof(double2)));
  if (mirror && !m->tab[0][o2][o1]) KB_CUDA(device_malloc(&m->tab[0][o2][o1], n * 2 * sizeof(double2)));
  DevBuf dl, dg, dbad, dmax;
  KB_CUDA(dl.alloc(n * sizeof(double2), st));
  KB_CUDA(dg.alloc(n * sizeof(double2), st));
  KB_CUDA(dbad.alloc(sizeof(int), st));
  KB_CUDA(dmax.alloc(2 * sizeof(double), st));
  KB_CUDA(cudaMemcpyAsync(dl.p, gl, n * sizeof(double2), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemcpyAsync(dg.p, gg, n * sizeof(double2), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemsetAsync(dbad.p, 0, sizeof(int), st));
  // the 1/w^2 tail coefficient of each function: the mean of w^2 g(w) at the mesh's two ends
  const double dt = 2.0 * m->tmax / (double)(n - 1), wmax = M_PI * (double)(n - 1) / ((double)n * dt);
  const double w2 = wmax * wmax;
  const double2 ml = make_double2(0.5 * w2 * (gl[0] + gl[2 * n - 2]), 0.5 * w2 * (gl[1] + gl[2 * n - 1]));
  const double2 mg = make_double2(0.5 * w2 * (gg[0] + gg[2 * n - 2]), 0.5 * w2 * (gg[1] + gg[2 * n - 1]));
  KB_CUDA(launch_dft_table(dl.as<double2>(), dg.as<double2>(), ml, mg, m->tab[0][o1][o2], m->npts, m->tmax,
                           dbad.as<int>(), st));
  KB_CUDA(launch_table_max(m->tab[0][o1][o2], m->npts, dmax.as<double>(), st));
  if (mirror) KB_CUDA(launch_mirror_block(m->tab[0][o1][o2], m->tab[0][o2][o1], m->npts, st));
  int bad = 0;
  double mx = 0.0;
  KB_CUDA(cudaMemcpyAsync(&bad, dbad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaMemcpyAsync(&mx, dmax.p, sizeof(double), cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaStreamSynchronize(st));
  if (bad) return fail(KB_E_INVALID, "g0 table contains non-finite values");
  const int blocks[2][2] = {{o1, o2}, {o2, o1}};
  for (int k = 0; k < (mirror ? 2 : 1); ++k) { // spin down uses the spin-up blocks (model.cpp:209-211)
    const int a = blocks[k][0], b = blocks[k][1];
    cudaFree(m->tab[1][a][b]);
    m->tab[1][a][b] = nullptr;
    m->hash[0][a][b] = 0;
    m->hash[1][a][b] = 0;
  }
  m->tabmax = std::max(m->tabmax, mx);
  return KB_OK;
}

// Device view of a model. A spin whose (o1,o2) block was never uploaded uses the
// other spin's block (keldy's models are spin symmetric, model.cpp:209-211).
static ModelDev model_dev(const kb_model *m, bool *spin_symmetric) {
  ModelDev d;
  memset(&d, 0, sizeof(d));
  bool sym = true;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) {
      double2 *up = m->tab[0][a][b], *dn = m->tab[1][a][b];
      d.tab[0][a][b] = up ? up : dn;
      d.tab[1][a][b] = dn ? dn : up;
      if (up && dn && !(m->hash[0][a][b] != 0 && m->hash[0][a][b] == m->hash[1][a][b])) sym = false;
    }
  d.npts = m->npts;
  d.tmax = m->tmax;
  d.xmin = -m->tmax;
  d.delta = (m->tmax - d.xmin) / (double)(m->npts - 1);
  d.alpha = m->alpha;
  d.pivot_floor = 1e-8 * (m->tabmax > 0 ? m->tabmax : 1.0);
  d.interp = m->interp;
  if (spin_symmetric) *spin_symmetric = sym;
  return d;
}

int kb_g0_eval(kb_context *ctx, const kb_model *m, const kb_gf_index *a, const kb_gf_index *b, const int *internal,
               int64_t count, double *out) {
  KB_CHECK(ctx && m && (count == 0 || (a && b && out)), "kb_g0_eval: null argument");
  for (int64_t i = 0; i < count; ++i) {
    KB_CHECK(a[i].spin >= 0 && a[i].spin < 2 && b[i].spin >= 0 && b[i].spin < 2, "spin must be 0 or 1");
    KB_CHECK(a[i].orbital >= 0 && a[i].orbital < 2 && b[i].orbital >= 0 && b[i].orbital < 2, "orbital must be 0 or 1");
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  DevBuf da, db, di, dout;
  KB_CUDA(da.alloc(count * sizeof(kb_gf_index), ctx->stream));
  KB_CUDA(db.alloc(count * sizeof(kb_gf_index), ctx->stream));
  KB_CUDA(dout.alloc(count * sizeof(double2), ctx->stream));
  KB_CUDA(cudaMemcpyAsync(da.p, a, count * sizeof(kb_gf_index), cudaMemcpyHostToDevice, ctx->stream));
  KB_CUDA(cudaMemcpyAsync(db.p, b, count * sizeof(kb_gf_index), cudaMemcpyHostToDevice, ctx->stream));
  if (internal) {
    KB_CUDA(di.alloc(count * sizeof(int), ctx->stream));
    KB_CUDA(cudaMemcpyAsync(di.p, internal, count * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  }
  KB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
  KB_CUDA(launch_g0_eval(model_dev(m, nullptr), da.as<kb_gf_index>(), db.as<kb_gf_index>(),
                         internal ? di.as<int>() : nullptr, count, dout.as<double2>(), ctx->d_err, ctx->stream));
  int err = 0;
  KB_CUDA(cudaMemcpyAsync(out, dout.p, count * sizeof(double2), cudaMemcpyDeviceToHost, ctx->stream));
  KB_CUDA(cudaMemcpyAsync(&err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  KB_CUDA(cudaStreamSynchronize(ctx->stream));
  if (err & 1) return fail(KB_E_RANGE, "g0 evaluated outside its tabulated time window");
  return KB_OK;
}

// ------------------------------------------------------------- integrand
static int check_integrand(const kb_model *m, const kb_integrand *f, int order) {
  KB_CHECK(m && f, "null model or integrand");
  KB_CHECK(order >= 0 && order <= MAX_ORDER, "order must be in [0, 16]");
  const kb_gf_index *e[2] = {&f->A, &f->B};
  for (auto *x : e) {
    KB_CHECK(x->spin >= 0 && x->spin < 2, "spin must be 0 or 1");
    KB_CHECK(x->k_idx >= 0 && x->k_idx < 2, "keldysh index must be 0 or 1");
    KB_CHECK(x->orbital >= 0 && x->orbital < 2, "orbital must be 0 or 1");
    // integrand_g_direct's constructor checks (wick_direct.hpp:50-56)
    if (x->time < 0.0) return fail(KB_E_INVALID, "An external point has negative time.");
    if (x->time > m->tmax) return fail(KB_E_INVALID, "An external point is out of g0 time window.");
  }
  return KB_OK;
}

static ItemDev make_item(const kb_model *m, const kb_integrand *f, int order) {
  ItemDev it;
  memset(&it, 0, sizeof(it));
  bool sym = true;
  it.model = model_dev(m, &sym);
  it.spin_symmetric = sym ? 1 : 0;
  it.f = *f;
  it.order = order;
  it.chunk_points = CHUNK_POINTS;
  return it;
}

// Runs the tree (or direct) kernel over `count` points of one item in an evaluation
// mode, then re-evaluates points the tree flagged with the pivoted-LU kernel.
static int run_eval(kb_context *ctx, ItemDev it, int mode, int64_t count, const double *in_host, int keep,
                    int algo, double *out, double *jac, int *in_domain, double *scale) {
  KB_CHECK(algo == KB_ALGO_AUTO || algo == KB_ALGO_TREE || algo == KB_ALGO_DIRECT, "unknown algorithm");
  if (count == 0) return KB_OK;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  it.n_points = count;
  const int N = it.order;
  const bool use_tree = (algo == KB_ALGO_TREE) || (algo == KB_ALGO_AUTO && it.spin_symmetric);
  if (algo == KB_ALGO_TREE && !it.spin_symmetric)
    return fail(KB_E_INVALID, "the tree algorithm needs equal spin-up and spin-down g0 tables");
  long long nchunks = (count + CHUNK_POINTS - 1) / CHUNK_POINTS;
  long long offs[2] = {0, nchunks};
  DevBuf ditem, doff, dcnt, din, dval, djac, ddom, dscale, dflag;
  KB_CUDA(ditem.alloc(sizeof(ItemDev), st));
  KB_CUDA(doff.alloc(sizeof(offs), st));
  KB_CUDA(dcnt.alloc(sizeof(int), st));
  size_t inbytes = (size_t)count * N * sizeof(double);
  KB_CUDA(din.alloc(inbytes, st));
  KB_CUDA(dval.alloc(count * sizeof(double2), st));
  KB_CUDA(djac.alloc(count * sizeof(double), st));
  KB_CUDA(ddom.alloc(count * sizeof(int), st));
  KB_CUDA(dflag.alloc(count * sizeof(int), st));
  if (scale) KB_CUDA(dscale.alloc(count * sizeof(double), st));
  KB_CUDA(cudaMemcpyAsync(ditem.p, &it, sizeof(ItemDev), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemcpyAsync(doff.p, offs, sizeof(offs), cudaMemcpyHostToDevice, st));
  if (inbytes) KB_CUDA(cudaMemcpyAsync(din.p, in_host, inbytes, cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemsetAsync(dcnt.p, 0, sizeof(int), st));
  KB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), st));
  Launch L;
  memset(&L, 0, sizeof(L));
  L.items = ditem.as<ItemDev>();
  L.n_items = 1;
  L.any_cubic = items_any_cubic(&it, 1);
  L.chunk_offsets = doff.as<long long>();
  L.n_chunks = (int)nchunks;
  L.chunk_counter = dcnt.as<int>();
  L.mode = mode;
  L.keep_u_hypercube = keep;
  L.in = din.as<double>();
  L.out_val = dval.as<double2>();
  L.out_jac = djac.as<double>();
  L.out_dom = ddom.as<int>();
  L.out_scale = scale ? dscale.as<double>() : nullptr;
  L.out_flag = dflag.as<int>();
  L.err = ctx->d_err;
  int grid = (int)std::min<long long>(nchunks, use_tree ? ctx->tree_grid : ctx->sm_count * 4);
  if (use_tree) {
    DevBuf dpts;
    KB_CUDA(dpts.alloc((size_t)grid * PTS_SLOT * sizeof(double), st));
    L.pts = dpts.as<double>();
    KB_CUDA(launch_tree(L, grid, st));
    std::vector<int> flags((size_t)count);
    KB_CUDA(cudaMemcpyAsync(flags.data(), dflag.p, count * sizeof(int), cudaMemcpyDeviceToHost, st));
    KB_CUDA(cudaStreamSynchronize(st));
    std::vector<int> idx;
    for (int64_t i = 0; i < count; ++i)
      if (flags[(size_t)i]) idx.push_back((int)i);
    if (!idx.empty()) {
      DevBuf didx;
      KB_CUDA(didx.alloc(idx.size() * sizeof(int), st));
      KB_CUDA(cudaMemcpyAsync(didx.p, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, st));
      long long nc2 = ((long long)idx.size() + CHUNK_POINTS - 1) / CHUNK_POINTS;
      long long offs2[2] = {0, nc2};
      KB_CUDA(cudaMemcpyAsync(doff.p, offs2, sizeof(offs2), cudaMemcpyHostToDevice, st));
      KB_CUDA(cudaMemsetAsync(dcnt.p, 0, sizeof(int), st));
      Launch L2 = L;
      L2.index = didx.as<int>();
      L2.n_index = (int)idx.size();
      L2.n_chunks = (int)nc2;
      KB_CUDA(launch_direct(L2, (int)std::min<long long>(nc2, ctx->sm_count * 4), st));
      KB_CUDA(cudaStreamSynchronize(st));
    }
  } else {
    KB_CUDA(launch_direct(L, grid, st));
  }
  int err = 0;
  KB_CUDA(cudaMemcpyAsync(out, dval.p, count * sizeof(double2), cudaMemcpyDeviceToHost, st));
  if (jac) KB_CUDA(cudaMemcpyAsync(jac, djac.p, count * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (in_domain) KB_CUDA(cudaMemcpyAsync(in_domain, ddom.p, count * sizeof(int), cudaMemcpyDeviceToHost, st));
  if (scale) KB_CUDA(cudaMemcpyAsync(scale, dscale.p, count * sizeof(double), cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaMemcpyAsync(&err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaStreamSynchronize(st));
  if (err & 1) return fail(KB_E_RANGE, "g0 evaluated outside its tabulated time window");
  return KB_OK;
}

int kb_integrand_eval(kb_context *ctx, const kb_model *m, const kb_integrand *f, int order, int64_t count,
                      const double *times, int keep_u_hypercube, int algo, double *out, int *in_domain,
                      double *scale) {
  KB_CHECK(ctx, "null context");
  int st = check_integrand(m, f, order);
  if (st) return st;
  KB_CHECK(count >= 0 && (count == 0 || (out && (times || order == 0))), "kb_integrand_eval: null buffer");
  ItemDev it = make_item(m, f, order);
  return run_eval(ctx, it, IN_TIMES, count, times, keep_u_hypercube, algo, out, nullptr, in_domain, scale);
}

int kb_evaluate_warped(kb_context *ctx, const kb_model *m, const kb_integrand *f, const kb_warper *chain,
                       int chain_len, int start_domain_nr, int order, int64_t count, const double *li,
                       int keep_u_hypercube, int algo, double *out, double *jac, int *in_domain) {
  KB_CHECK(ctx, "null context");
  int st = check_integrand(m, f, order);
  if (st) return st;
  KB_CHECK(count >= 0 && (count == 0 || (out && (li || order == 0))), "kb_evaluate_warped: null buffer");
  KB_CHECK(0 <= start_domain_nr && start_domain_nr <= chain_len, "start_domain_nr must be in [0, chain size]");
  ItemDev it = make_item(m, f, order);
  st = make_chain(chain, chain_len, it.chain);
  if (st) return st;
  st = check_chain_dims(chain, chain_len, order);
  if (st) return st;
  it.chain_len = chain_len;
  it.chain_start = start_domain_nr;
  return run_eval(ctx, it, IN_LI, count, li, keep_u_hypercube, algo, out, jac, in_domain, nullptr);
}

int kb_integrand_eval_no_det(kb_context *ctx, const kb_model *m, const kb_integrand *f, int order, int64_t count,
                             const double *times, int keep_u_hypercube, double *out, int *in_domain) {
  KB_CHECK(ctx, "null context");
  int st = check_integrand(m, f, order);
  if (st) return st;
  if (order > 2) return fail(KB_E_INVALID, "Not supported for order > 2");
  if (count == 0) return KB_OK;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  DevBuf dt, dv, dd;
  size_t tb = (size_t)count * order * sizeof(double);
  KB_CUDA(dt.alloc(tb, s));
  KB_CUDA(dv.alloc(count * sizeof(double2), s));
  KB_CUDA(dd.alloc(count * sizeof(int), s));
  if (tb) KB_CUDA(cudaMemcpyAsync(dt.p, times, tb, cudaMemcpyHostToDevice, s));
  KB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), s));
  KB_CUDA(launch_no_det(model_dev(m, nullptr), *f, order, count, dt.as<double>(), keep_u_hypercube,
                        dv.as<double2>(), dd.as<int>(), ctx->d_err, s));
  int err = 0;
  KB_CUDA(cudaMemcpyAsync(out, dv.p, count * sizeof(double2), cudaMemcpyDeviceToHost, s));
  if (in_domain) KB_CUDA(cudaMemcpyAsync(in_domain, dd.p, count * sizeof(int), cudaMemcpyDeviceToHost, s));
  KB_CUDA(cudaMemcpyAsync(&err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  KB_CUDA(cudaStreamSynchronize(s));
  if (err & 1) return fail(KB_E_RANGE, "g0 evaluated outside its tabulated time window");
  return KB_OK;
}

// ------------------------------------------------------------- integrator
} // extern "C"

namespace kb {
std::atomic<unsigned long long> &device_allocations() {
  static std::atomic<unsigned long long> n{0};
  return n;
}

cudaMemPool_t kb_pool() {
  constexpr int MAX_DEVICES = 64;
  static std::mutex mu;
  static cudaMemPool_t pools[MAX_DEVICES] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= MAX_DEVICES) { // beyond the table: that device's default pool
    cudaMemPool_t p = nullptr;
    cudaDeviceGetDefaultMemPool(&p, dev);
    return p;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) == cudaSuccess) {
      unsigned long long keep = KB_POOL_KEEP_BYTES;
      cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    } else {
      cudaGetLastError();
      cudaDeviceGetDefaultMemPool(&p, dev);
    }
    pools[dev] = p;
  }
  return pools[dev];
}
} // namespace kb

namespace {
// Time bins of an integration (integrand_g_direct_time) and the caller's outputs.
struct TimeBins {
  int nbins;
  double xmin, xmax;
  double *sums;      // [n_work][nbins] interleaved complex, added to
  uint64_t *counts;  // [n_work][nbins], added to
  uint64_t *dropped; // [n_work], added to
};

// One batched pass over `items`: two groups (tree / pivoted LU), each one persistent
// launch over its items, heaviest orders first. Sums are added to acc[acc_index[i]]
// (and to the time bins of that work item when `bins` is given).
int run_integrate(kb_context *ctx, const std::vector<ItemDev> &items, const std::vector<int> &use_tree,
                  const std::vector<int> &acc_index, kb_accum *acc, const TimeBins *bins = nullptr) {
  cudaStream_t st = ctx->stream;
  const int n_work = (int)items.size();
  for (int group = 0; group < 2; ++group) {
    std::vector<int> ids;
    for (int i = 0; i < n_work; ++i)
      if (use_tree[(size_t)i] == (group == 0) && items[(size_t)i].n_points > 0) ids.push_back(i);
    if (ids.empty()) continue;
    std::stable_sort(ids.begin(), ids.end(), [&](int a, int b) { return items[(size_t)a].order > items[(size_t)b].order; });
    std::vector<ItemDev> sorted;
    std::vector<long long> offs(1, 0);
    for (int i : ids) {
      sorted.push_back(items[(size_t)i]);
      const long long cp = items[(size_t)i].chunk_points;
      offs.push_back(offs.back() + (items[(size_t)i].n_points + cp - 1) / cp);
    }
    const long long nchunks = offs.back();
    if (nchunks > INT32_MAX) return fail(KB_E_INVALID, "too many points in one kb_integrate call");
    DevBuf ditems, doff, dcnt, dpart, dacc_s;
    KB_CUDA(ditems.alloc(sorted.size() * sizeof(ItemDev), st));
    KB_CUDA(doff.alloc(offs.size() * sizeof(long long), st));
    KB_CUDA(dcnt.alloc(sizeof(int), st));
    KB_CUDA(dpart.alloc((size_t)nchunks * sizeof(ChunkPartial), st));
    KB_CUDA(dacc_s.alloc(sorted.size() * sizeof(kb_accum), st));
    KB_CUDA(cudaMemcpyAsync(ditems.p, sorted.data(), sorted.size() * sizeof(ItemDev), cudaMemcpyHostToDevice, st));
    KB_CUDA(cudaMemcpyAsync(doff.p, offs.data(), offs.size() * sizeof(long long), cudaMemcpyHostToDevice, st));
    KB_CUDA(cudaMemsetAsync(dcnt.p, 0, sizeof(int), st));
    KB_CUDA(cudaMemsetAsync(dacc_s.p, 0, sorted.size() * sizeof(kb_accum), st));
    Launch L;
    memset(&L, 0, sizeof(L));
    L.items = ditems.as<ItemDev>();
    L.n_items = (int)sorted.size();
    L.any_cubic = items_any_cubic(sorted.data(), sorted.size());
    L.chunk_offsets = doff.as<long long>();
    L.n_chunks = (int)nchunks;
    L.chunk_counter = dcnt.as<int>();
    L.mode = IN_SOBOL;
    L.partials = dpart.as<ChunkPartial>();
    L.err = ctx->d_err;
    DevBuf dbs, dbc, dbd, dos, doc, dod;
    if (bins) {
      const size_t nb = (size_t)bins->nbins;
      KB_CUDA(dbs.alloc((size_t)nchunks * nb * sizeof(double2), st));
      KB_CUDA(dbc.alloc((size_t)nchunks * nb * sizeof(unsigned), st));
      KB_CUDA(dbd.alloc((size_t)nchunks * sizeof(unsigned), st));
      KB_CUDA(dos.alloc(sorted.size() * nb * sizeof(double2), st));
      KB_CUDA(doc.alloc(sorted.size() * nb * sizeof(unsigned long long), st));
      KB_CUDA(dod.alloc(sorted.size() * sizeof(unsigned long long), st));
      L.nbins = bins->nbins;
      L.bin_cols = 1;
      L.bin_xmin = bins->xmin;
      L.bin_xmax = bins->xmax;
      L.bin_size = (bins->xmax - bins->xmin) / bins->nbins;
      L.bin_sums = dbs.as<double2>();
      L.bin_counts = dbc.as<unsigned>();
      L.bin_dropped = dbd.as<unsigned>();
    }
    DevBuf dpts;
    const int tgrid = (int)std::min<long long>(nchunks, (long long)ctx->sm_count * ctx->ctas_per_sm);
    if (group == 0) {
      KB_CUDA(dpts.alloc((size_t)tgrid * PTS_SLOT * sizeof(double), st));
      L.pts = dpts.as<double>();
    }
    if (ctx->timing) KB_CUDA(cudaEventRecord(ctx->ev[0], st));
    if (group == 0)
      KB_CUDA(launch_tree(L, tgrid, st));
    else
      KB_CUDA(launch_direct(L, (int)std::min<long long>(nchunks, ctx->sm_count * 4), st));
    if (ctx->timing) KB_CUDA(cudaEventRecord(ctx->ev[1], st));
    if (group == 0) {
      KB_CUDA(launch_fallback(L, ctx->sm_count * 4, st));
      ctx->last_launches++;
    }
    if (ctx->timing) KB_CUDA(cudaEventRecord(ctx->ev[2], st));
    KB_CUDA(launch_reduce(L, dacc_s.as<kb_accum>(), st));
    if (bins) {
      KB_CUDA(launch_reduce_bins(L, dos.as<double2>(), doc.as<unsigned long long>(), dod.as<unsigned long long>(), st));
      ctx->last_launches++;
    }
    if (ctx->timing) KB_CUDA(cudaEventRecord(ctx->ev[3], st));
    ctx->last_launches += 2;
    std::vector<kb_accum> part(sorted.size());
    KB_CUDA(cudaMemcpyAsync(part.data(), dacc_s.p, part.size() * sizeof(kb_accum), cudaMemcpyDeviceToHost, st));
    std::vector<double> hbs;
    std::vector<unsigned long long> hbc, hbd;
    if (bins) {
      const size_t nb = (size_t)bins->nbins;
      hbs.resize(sorted.size() * nb * 2);
      hbc.resize(sorted.size() * nb);
      hbd.resize(sorted.size());
      KB_CUDA(cudaMemcpyAsync(hbs.data(), dos.p, hbs.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
      KB_CUDA(cudaMemcpyAsync(hbc.data(), doc.p, hbc.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
      KB_CUDA(cudaMemcpyAsync(hbd.data(), dod.p, hbd.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    }
    KB_CUDA(cudaStreamSynchronize(st));
    if (ctx->timing) {
      float a = 0, b = 0, c = 0;
      KB_CUDA(cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]));
      KB_CUDA(cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[2]));
      KB_CUDA(cudaEventElapsedTime(&c, ctx->ev[2], ctx->ev[3]));
      ctx->last_ms[0] += a;
      ctx->last_ms[1] += b;
      ctx->last_ms[2] += c;
    }
    for (size_t j = 0; j < ids.size(); ++j) {
      const int w = acc_index[(size_t)ids[j]];
      kb_accum &a = acc[w];
      a.sum_re += part[j].sum_re;
      a.sum_im += part[j].sum_im;
      a.n_points += part[j].n_points;
      a.n_in_domain += part[j].n_in_domain;
      a.n_fallback += part[j].n_fallback;
      if (bins) {
        const size_t nb = (size_t)bins->nbins;
        for (size_t b = 0; b < nb; ++b) {
          bins->sums[2 * ((size_t)w * nb + b)] += hbs[2 * (j * nb + b)];
          bins->sums[2 * ((size_t)w * nb + b) + 1] += hbs[2 * (j * nb + b) + 1];
          bins->counts[(size_t)w * nb + b] += hbc[j * nb + b];
        }
        bins->dropped[w] += hbd[j];
      }
    }
  }
  return KB_OK;
}

constexpr int64_t FLOW_PIECE = 1 << 22;            // points per flow-mapped piece
constexpr size_t FLOW_ROUND_BYTES = (size_t)1 << 30; // flow-mapped points held at once

// Points per scheduling chunk of a work item of n points: the context's chunk size for its
// order (autotuned or kb_context_set_launch), halved (down to 8) while the item would have
// fewer chunks than half the resident tree CTAs, so that a small item is spread over the
// GPU instead of a few CTAs walking long chunks one point after another (a batch of many
// small items keeps larger chunks than one small item alone would need). It depends on
// the item alone: a batch adds each item's points in the order of a call of its own.
int item_chunk(const kb_context *ctx, int order, int64_t n) {
  int c = ctx->chunk_points[order];
  const int64_t want = (int64_t)ctx->sm_count * ctx->ctas_per_sm / 2;
  while (c > 8 && (n + c - 1) / c < want) c >>= 1;
  return c;
}

// Checks of a work item shared by kb_integrate and kb_plan_create; fills `it`.
int work_item(kb_context *ctx, const kb_work &w, int algo, ItemDev &it, int &tree) {
  int st = check_integrand(w.m, &w.f, w.order);
  if (st) return st;
  KB_CHECK(w.rng, "work item without a Sobol generator");
  KB_CHECK(w.n_points >= 0, "n_points must be >= 0");
  KB_CHECK(w.order >= 1, "integrator dimension must be > 0 (Dimension of the integration space must be > 0.)");
  if (w.rng->dim < w.order) return fail(KB_E_INVALID, "Sobol generator has fewer dimensions than the order");
  st = check_sobol_range(w.rng, w.k_first, w.n_points);
  if (st) return st;
  if (w.flow) {
    KB_CHECK(w.flow->dim == w.order, "the flow's dimension differs from the work item's order");
    KB_CHECK(w.flow->device == ctx->device, "the flow lives on another device");
  }
  it = make_item(w.m, &w.f, w.order);
  st = make_chain(w.chain, w.chain_len, it.chain);
  if (st) return st;
  st = check_chain_dims(w.chain, w.chain_len, w.order);
  if (st) return st;
  it.chain_len = w.chain_len;
  it.chain_start = w.chain_len;
  it.rng = sobol_dev(w.rng);
  it.k_first = w.k_first;
  it.n_points = w.n_points;
  it.chunk_points = item_chunk(ctx, w.order, w.n_points);
  if (w.flow && w.flow->layout.kind == FLOW_KIND_SPLINE) it.spline_knots = w.flow->knots; // mapped in line
  if (w.flow && w.flow->layout.kind == FLOW_KIND_AR_SPLINE) it.ar_spline = w.flow->master; // mapped in line
  if (algo == KB_ALGO_TREE && !it.spin_symmetric)
    return fail(KB_E_INVALID, "the tree algorithm needs equal spin-up and spin-down g0 tables");
  tree = ((algo == KB_ALGO_TREE) || (algo == KB_ALGO_AUTO && it.spin_symmetric)) ? 1 : 0;
  return KB_OK;
}

int integrate_impl(kb_context *ctx, const kb_work *work, int n_work, int algo, kb_accum *acc, const TimeBins *tb);

// A flow whose points come from its own map kernel before the integration pass (the
// coupling flow); the spline flows are applied in line by the integrand kernels.
bool mapped_flow(const kb_work &w) { return w.flow && w.flow->layout.kind == FLOW_KIND_COUPLING; }

// The knots of every distinct spline flow among the work items, made from its current
// parameters on stream st (ahead of the kernels that read them).
int spline_knots_for(const kb_work *work, int n_work, cudaStream_t st, int *launches) {
  std::vector<const kb_flow *> done;
  for (int i = 0; i < n_work; ++i) {
    const kb_flow *f = work[i].flow;
    if (!f || f->layout.kind != FLOW_KIND_SPLINE || std::find(done.begin(), done.end(), f) != done.end()) continue;
    done.push_back(f);
    KB_CUDA(launch_spline_knots(f->master, f->dim, f->knots, st));
    ++*launches;
  }
  return KB_OK;
}
} // namespace

extern "C" {

int kb_integrate(kb_context *ctx, const kb_work *work, int n_work, int algo, kb_accum *acc) {
  return integrate_impl(ctx, work, n_work, algo, acc, nullptr);
}

int kb_integrate_binned(kb_context *ctx, const kb_work *work, int n_work, int algo, const kb_time_bins *bins,
                        kb_accum *acc, double *bin_sums, uint64_t *bin_counts, uint64_t *dropped) {
  KB_CHECK(bins && (n_work == 0 || (bin_sums && bin_counts && dropped)), "kb_integrate_binned: null argument");
  KB_CHECK(bins->nbins >= 1 && bins->nbins <= 4096, "the number of time bins must be in [1, 4096]");
  if (!(bins->xmin < bins->xmax))
    return fail(KB_E_INVALID, "Boundaries of binning range are in wrong order (" + std::to_string(bins->xmin) +
                                  " >= " + std::to_string(bins->xmax) + ")");
  TimeBins tb{bins->nbins, bins->xmin, bins->xmax, bin_sums, bin_counts, dropped};
  return integrate_impl(ctx, work, n_work, algo, acc, &tb);
}

} // extern "C"

namespace {
// The kernel method's integration: binned by (vertex time, Keldysh index) (bins given,
// compute_gf_kernel) or summed with the weight e^{i omega t} of each term's vertex (omega
// given, compute_gf_kernel_single_omega).
int integrate_kernel_impl(kb_context *ctx, const kb_work *work, int n_work, const kb_time_bins *bins,
                          const double *omega, kb_accum *acc, double *bin_sums, uint64_t *bin_counts,
                          uint64_t *dropped) {
  if (n_work == 0) return KB_OK;
  std::vector<ItemDev> items((size_t)n_work);
  std::vector<long long> offs(1, 0);
  for (int i = 0; i < n_work; ++i) {
    int tree = 0;
    kb_work w = work[i];
    w.f.B = w.f.A; // the fixed point X (integrand_g_kernel has one external point and no cutoff)
    w.f.cutoff = 0.0;
    int st = work_item(ctx, w, KB_ALGO_AUTO, items[(size_t)i], tree);
    if (st) return st;
    KB_CHECK(work[i].order <= KM_MAX_ORDER, "the kernel method runs orders 1..10");
    KB_CHECK(!work[i].flow, "the kernel method does not take a learned flow");
    items[(size_t)i].chunk_points = 16; // a CTA evaluates its chunk's points one after another
    offs.push_back(offs.back() + (items[(size_t)i].n_points + 15) / 16);
  }
  const long long nchunks = offs.back();
  if (nchunks > INT32_MAX) return fail(KB_E_INVALID, "too many points in one call");
  if (nchunks == 0) return KB_OK;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const size_t nb = bins ? 2 * (size_t)bins->nbins : 0;
  DevBuf ditems, doff, dcnt, dpart, dacc, dbs, dbc, dbd, dos, doc, dod;
  KB_CUDA(ditems.alloc(items.size() * sizeof(ItemDev), st));
  KB_CUDA(doff.alloc(offs.size() * sizeof(long long), st));
  KB_CUDA(dcnt.alloc(sizeof(int), st));
  KB_CUDA(dpart.alloc((size_t)nchunks * sizeof(ChunkPartial), st));
  KB_CUDA(dacc.alloc(items.size() * sizeof(kb_accum), st));
  if (nb) {
    KB_CUDA(dbs.alloc((size_t)nchunks * nb * sizeof(double2), st));
    KB_CUDA(dbc.alloc((size_t)nchunks * nb * sizeof(unsigned), st));
    KB_CUDA(dbd.alloc((size_t)nchunks * sizeof(unsigned), st));
    KB_CUDA(dos.alloc(items.size() * nb * sizeof(double2), st));
    KB_CUDA(doc.alloc(items.size() * nb * sizeof(unsigned long long), st));
    KB_CUDA(dod.alloc(items.size() * sizeof(unsigned long long), st));
  }
  KB_CUDA(cudaMemcpyAsync(ditems.p, items.data(), items.size() * sizeof(ItemDev), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemcpyAsync(doff.p, offs.data(), offs.size() * sizeof(long long), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemsetAsync(dcnt.p, 0, sizeof(int), st));
  KB_CUDA(cudaMemsetAsync(dacc.p, 0, items.size() * sizeof(kb_accum), st));
  KB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), st));
  Launch L;
  memset(&L, 0, sizeof(L));
  L.items = ditems.as<ItemDev>();
  L.n_items = n_work;
  L.chunk_offsets = doff.as<long long>();
  L.n_chunks = (int)nchunks;
  L.chunk_counter = dcnt.as<int>();
  L.mode = IN_SOBOL;
  L.partials = dpart.as<ChunkPartial>();
  if (bins) {
    L.nbins = bins->nbins;
    L.bin_cols = 2;
    L.bin_xmin = bins->xmin;
    L.bin_xmax = bins->xmax;
    L.bin_size = (bins->xmax - bins->xmin) / bins->nbins;
    L.bin_sums = dbs.as<double2>();
    L.bin_counts = dbc.as<unsigned>();
    L.bin_dropped = dbd.as<unsigned>();
  } else {
    L.km_fourier = 1;
    L.km_omega = *omega;
  }
  L.err = ctx->d_err;
  const int kgrid = (int)std::min<long long>(nchunks, (long long)ctx->sm_count * KM_CTAS_PER_SM);
  DevBuf dpts;
  KB_CUDA(dpts.alloc((size_t)kgrid * KM_SLOT * sizeof(double), st));
  L.pts = dpts.as<double>();
  if (ctx->timing) KB_CUDA(cudaEventRecord(ctx->ev[0], st));
  KB_CUDA(launch_kernel_method(L, kgrid, st));
  if (ctx->timing) KB_CUDA(cudaEventRecord(ctx->ev[1], st));
  KB_CUDA(launch_reduce(L, dacc.as<kb_accum>(), st));
  if (nb)
    KB_CUDA(launch_reduce_bins(L, dos.as<double2>(), doc.as<unsigned long long>(), dod.as<unsigned long long>(), st));
  if (ctx->timing) KB_CUDA(cudaEventRecord(ctx->ev[2], st));
  ctx->last_launches = nb ? 3 : 2;
  std::vector<kb_accum> part(items.size());
  std::vector<double> hbs(items.size() * nb * 2);
  std::vector<unsigned long long> hbc(items.size() * nb), hbd(items.size());
  KB_CUDA(cudaMemcpyAsync(part.data(), dacc.p, part.size() * sizeof(kb_accum), cudaMemcpyDeviceToHost, st));
  if (nb) {
    KB_CUDA(cudaMemcpyAsync(hbs.data(), dos.p, hbs.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    KB_CUDA(cudaMemcpyAsync(hbc.data(), doc.p, hbc.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    KB_CUDA(cudaMemcpyAsync(hbd.data(), dod.p, hbd.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  }
  int err = 0;
  KB_CUDA(cudaMemcpyAsync(&err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaStreamSynchronize(st));
  if (ctx->timing) {
    float a = 0, c = 0;
    KB_CUDA(cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]));
    KB_CUDA(cudaEventElapsedTime(&c, ctx->ev[1], ctx->ev[2]));
    ctx->last_ms[0] = a;
    ctx->last_ms[1] = 0.0;
    ctx->last_ms[2] = c;
  }
  if (err & 1) return fail(KB_E_RANGE, "g0 evaluated outside its tabulated time window");
  for (int w = 0; w < n_work; ++w) {
    acc[w].sum_re += part[(size_t)w].sum_re;
    acc[w].sum_im += part[(size_t)w].sum_im;
    acc[w].n_points += part[(size_t)w].n_points;
    acc[w].n_in_domain += part[(size_t)w].n_in_domain;
    if (!nb) continue;
    for (size_t b = 0; b < nb; ++b) {
      bin_sums[2 * ((size_t)w * nb + b)] += hbs[2 * ((size_t)w * nb + b)];
      bin_sums[2 * ((size_t)w * nb + b) + 1] += hbs[2 * ((size_t)w * nb + b) + 1];
      bin_counts[(size_t)w * nb + b] += hbc[(size_t)w * nb + b];
    }
    dropped[w] += hbd[(size_t)w];
  }
  return KB_OK;
}
} // namespace

extern "C" {

int kb_integrate_kernel(kb_context *ctx, const kb_work *work, int n_work, const kb_time_bins *bins, kb_accum *acc,
                        double *bin_sums, uint64_t *bin_counts, uint64_t *dropped) {
  KB_CHECK(ctx && bins && (n_work == 0 || (work && acc && bin_sums && bin_counts && dropped)),
           "kb_integrate_kernel: null argument");
  KB_CHECK(bins->nbins >= 1 && bins->nbins <= 4096, "the number of time bins must be in [1, 4096]");
  if (!(bins->xmin < bins->xmax))
    return fail(KB_E_INVALID, "Boundaries of binning range are in wrong order (" + std::to_string(bins->xmin) +
                                  " >= " + std::to_string(bins->xmax) + ")");
  return integrate_kernel_impl(ctx, work, n_work, bins, nullptr, acc, bin_sums, bin_counts, dropped);
}

int kb_integrate_kernel_single_omega(kb_context *ctx, const kb_work *work, int n_work, double omega,
                                     kb_accum *acc) {
  KB_CHECK(ctx && (n_work == 0 || (work && acc)), "kb_integrate_kernel_single_omega: null argument");
  KB_CHECK(std::isfinite(omega), "omega must be finite");
  return integrate_kernel_impl(ctx, work, n_work, nullptr, &omega, acc, nullptr, nullptr, nullptr);
}

int kb_integrand_kernel_eval(kb_context *ctx, const kb_model *m, const kb_gf_index *X, int order, int64_t count,
                             const double *times, int keep_u_hypercube, double *out, int *in_domain) {
  KB_CHECK(ctx && m && X, "kb_integrand_kernel_eval: null argument");
  KB_CHECK(order >= 1 && order <= KM_MAX_ORDER, "the kernel method runs orders 1..10");
  KB_CHECK(count >= 0 && (count == 0 || (times && out)), "kb_integrand_kernel_eval: null buffer");
  kb_integrand f{*X, *X, 0.0};
  int st = check_integrand(m, &f, order);
  if (st) return st;
  if (count == 0) return KB_OK;
  ItemDev it = make_item(m, &f, order);
  it.n_points = count;
  it.chunk_points = 16;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const long long nchunks = (count + 15) / 16;
  long long offs[2] = {0, nchunks};
  DevBuf ditem, doff, dcnt, din, dout, ddom;
  KB_CUDA(ditem.alloc(sizeof(ItemDev), s));
  KB_CUDA(doff.alloc(sizeof(offs), s));
  KB_CUDA(dcnt.alloc(sizeof(int), s));
  KB_CUDA(din.alloc((size_t)count * order * sizeof(double), s));
  KB_CUDA(dout.alloc((size_t)count * 2 * order * sizeof(double2), s));
  KB_CUDA(ddom.alloc((size_t)count * sizeof(int), s));
  KB_CUDA(cudaMemcpyAsync(ditem.p, &it, sizeof(ItemDev), cudaMemcpyHostToDevice, s));
  KB_CUDA(cudaMemcpyAsync(doff.p, offs, sizeof(offs), cudaMemcpyHostToDevice, s));
  KB_CUDA(cudaMemcpyAsync(din.p, times, (size_t)count * order * sizeof(double), cudaMemcpyHostToDevice, s));
  KB_CUDA(cudaMemsetAsync(dcnt.p, 0, sizeof(int), s));
  KB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), s));
  Launch L;
  memset(&L, 0, sizeof(L));
  L.items = ditem.as<ItemDev>();
  L.n_items = 1;
  L.any_cubic = items_any_cubic(&it, 1);
  L.chunk_offsets = doff.as<long long>();
  L.n_chunks = (int)nchunks;
  L.chunk_counter = dcnt.as<int>();
  L.mode = IN_TIMES;
  L.keep_u_hypercube = keep_u_hypercube;
  L.in = din.as<double>();
  L.out_kvals = dout.as<double2>();
  L.out_dom = ddom.as<int>();
  L.err = ctx->d_err;
  const int kgrid = (int)std::min<long long>(nchunks, (long long)ctx->sm_count * KM_CTAS_PER_SM);
  DevBuf dpts;
  KB_CUDA(dpts.alloc((size_t)kgrid * KM_SLOT * sizeof(double), s));
  L.pts = dpts.as<double>();
  KB_CUDA(launch_kernel_method(L, kgrid, s));
  int err = 0;
  KB_CUDA(cudaMemcpyAsync(out, dout.p, (size_t)count * 2 * order * sizeof(double2), cudaMemcpyDeviceToHost, s));
  if (in_domain) KB_CUDA(cudaMemcpyAsync(in_domain, ddom.p, (size_t)count * sizeof(int), cudaMemcpyDeviceToHost, s));
  KB_CUDA(cudaMemcpyAsync(&err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  KB_CUDA(cudaStreamSynchronize(s));
  if (err & 1) return fail(KB_E_RANGE, "g0 evaluated outside its tabulated time window");
  return KB_OK;
}

} // extern "C"

namespace {
int integrate_impl(kb_context *ctx, const kb_work *work, int n_work, int algo, kb_accum *acc, const TimeBins *tb) {
  KB_CHECK(ctx && (n_work == 0 || (work && acc)), "kb_integrate: null argument");
  KB_CHECK(algo == KB_ALGO_AUTO || algo == KB_ALGO_TREE || algo == KB_ALGO_DIRECT, "unknown algorithm");
  if (n_work == 0) return KB_OK;
  std::vector<ItemDev> items((size_t)n_work);
  std::vector<int> use_tree((size_t)n_work), index((size_t)n_work);
  bool any_flow = false;
  for (int i = 0; i < n_work; ++i) {
    int st = work_item(ctx, work[i], algo, items[(size_t)i], use_tree[(size_t)i]);
    if (st) return st;
    index[(size_t)i] = i;
    any_flow = any_flow || (mapped_flow(work[i]) && work[i].n_points > 0);
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  ctx->last_ms[0] = ctx->last_ms[1] = ctx->last_ms[2] = 0.0;
  ctx->last_launches = 0;
  KB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), st));
  {
    int rc = spline_knots_for(work, n_work, st, &ctx->last_launches);
    if (rc) return rc;
  }
  if (!any_flow) {
    int rc = run_integrate(ctx, items, use_tree, index, acc, tb);
    if (rc) return rc;
  } else {
    // Items with a flow run in pieces whose flow-mapped points (li, Jacobian) are made by
    // the flow's sampling kernel right before the pass that integrates them.
    struct Piece {
      ItemDev it;
      int tree, acc;
      const kb_flow *flow;
      size_t bytes;
    };
    std::vector<Piece> plain, flowed;
    for (int i = 0; i < n_work; ++i) {
      const ItemDev &it = items[(size_t)i];
      if (!mapped_flow(work[i])) {
        plain.push_back({it, use_tree[(size_t)i], i, nullptr, 0});
        continue;
      }
      for (int64_t off = 0; off < it.n_points; off += FLOW_PIECE) {
        Piece p{it, use_tree[(size_t)i], i, work[i].flow, 0};
        p.it.k_first = it.k_first + (uint32_t)off;
        p.it.n_points = std::min<int64_t>(FLOW_PIECE, it.n_points - off);
        p.bytes = (size_t)p.it.n_points * (size_t)(it.order + 1) * sizeof(double);
        flowed.push_back(p);
      }
    }
    size_t next = 0;
    bool first_round = true;
    while (first_round || next < flowed.size()) {
      std::vector<Piece> round = first_round ? plain : std::vector<Piece>();
      size_t bytes = 0;
      const size_t begin = next;
      while (next < flowed.size() && (next == begin || bytes + flowed[next].bytes <= FLOW_ROUND_BYTES))
        bytes += flowed[next++].bytes;
      DevBuf fbuf;
      if (bytes) KB_CUDA(fbuf.alloc(bytes, st));
      size_t off = 0;
      for (size_t j = begin; j < next; ++j) {
        Piece p = flowed[j];
        double *x = reinterpret_cast<double *>(fbuf.as<unsigned char>() + off);
        double *jac = x + (size_t)p.it.n_points * p.it.order;
        KB_CUDA(launch_flow_map(p.flow->layout, 1, p.it.n_points, nullptr, p.it.rng, p.it.k_first, nullptr, 1, x, jac,
                                ctx->d_err, ctx->sm_count, st));
        ctx->last_launches++;
        p.it.flow_x = x;
        p.it.flow_jac = jac;
        off += p.bytes;
        round.push_back(p);
      }
      std::vector<ItemDev> ritems;
      std::vector<int> rtree, racc;
      for (const Piece &p : round) {
        ritems.push_back(p.it);
        rtree.push_back(p.tree);
        racc.push_back(p.acc);
      }
      int rc = run_integrate(ctx, ritems, rtree, racc, acc, tb);
      if (rc) return rc;
      first_round = false;
    }
  }
  int err = 0;
  KB_CUDA(cudaMemcpyAsync(&err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaStreamSynchronize(st));
  if (err & 1) return fail(KB_E_RANGE, "g0 evaluated outside its tabulated time window");
  if (err & 2) return fail(KB_E_CUDA, "a flow kernel's wait on the tensor cores ran out");
  return KB_OK;
}
} // namespace

extern "C" {

// ------------------------------------------------------------------ plans
struct kb_plan {
  struct Group {
    int n_items = 0;
    std::vector<int> ids;      // original work index of each sorted item
    std::vector<ItemDev> items; // host copy (k_first updates)
    long long n_chunks = 0;
    int grid = 0;
    ItemDev *d_items = nullptr;
    long long *d_offs = nullptr;
    int *d_cnt = nullptr;
    ChunkPartial *d_part = nullptr;
    double *d_pts = nullptr;
    kb_accum *d_acc = nullptr;
  } g[2];
  int n_work = 0;
  std::vector<int> where_group, where_pos; // work index -> (group, sorted position)
  std::vector<const kb_sobol *> rng;
  // items with a learned flow: their points are mapped into `buf` at every launch
  struct Fill {
    FlowDev layout;
    SobolDev rng;
    int gi, pos;
    int64_t n;
    int order;
    double *buf = nullptr; // [n][order] points, then [n] Jacobians
  };
  std::vector<Fill> fills;
  std::vector<const kb_flow *> splines; // spline flows of the items: knots made at every launch
  cudaGraphExec_t exec = nullptr;
  int device = 0;
};

static void plan_free(kb_plan *p) {
  cudaSetDevice(p->device);
  if (p->exec) cudaGraphExecDestroy(p->exec);
  for (auto &g : p->g) {
    cudaFree(g.d_items);
    cudaFree(g.d_offs);
    cudaFree(g.d_cnt);
    cudaFree(g.d_part);
    cudaFree(g.d_pts);
    cudaFree(g.d_acc);
  }
  for (auto &f : p->fills) cudaFree(f.buf);
  delete p;
}

int kb_plan_destroy(kb_plan *plan) {
  if (plan) plan_free(plan);
  return KB_OK;
}

int kb_plan_create(kb_context *ctx, const kb_work *work, int n_work, int algo, kb_plan **out) {
  KB_CHECK(ctx && out && (n_work == 0 || work), "kb_plan_create: null argument");
  KB_CHECK(algo == KB_ALGO_AUTO || algo == KB_ALGO_TREE || algo == KB_ALGO_DIRECT, "unknown algorithm");
  std::vector<ItemDev> items((size_t)n_work);
  std::vector<int> grp((size_t)n_work);
  for (int i = 0; i < n_work; ++i) {
    int tree = 0;
    int st = work_item(ctx, work[i], algo, items[(size_t)i], tree);
    if (st) return st;
    grp[(size_t)i] = tree ? 0 : 1;
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  auto *p = new kb_plan;
  p->device = ctx->device;
  p->n_work = n_work;
  p->where_group.assign((size_t)n_work, -1);
  p->where_pos.assign((size_t)n_work, -1);
  for (int i = 0; i < n_work; ++i) p->rng.push_back(work[i].rng);
  for (int i = 0; i < n_work; ++i) {
    const kb_work &w = work[i];
    if (w.flow && w.flow->layout.kind == FLOW_KIND_SPLINE &&
        std::find(p->splines.begin(), p->splines.end(), w.flow) == p->splines.end())
      p->splines.push_back(w.flow);
    if (!mapped_flow(w) || w.n_points == 0) continue;
    kb_plan::Fill f;
    f.layout = w.flow->layout;
    f.rng = items[(size_t)i].rng;
    f.n = w.n_points;
    f.order = w.order;
    f.gi = grp[(size_t)i];
    f.pos = -1;
    cudaError_t e = device_malloc(&f.buf, (size_t)f.n * (size_t)(f.order + 1) * sizeof(double));
    if (e != cudaSuccess) {
      plan_free(p);
      return fail(KB_E_NOMEM, std::string("kb_plan_create: ") + cudaGetErrorString(e));
    }
    items[(size_t)i].flow_x = f.buf;
    items[(size_t)i].flow_jac = f.buf + (size_t)f.n * f.order;
    f.pos = i; // work index until the groups are sorted
    p->fills.push_back(f);
  }
  for (int gi = 0; gi < 2; ++gi) {
    auto &g = p->g[gi];
    for (int i = 0; i < n_work; ++i)
      if (grp[(size_t)i] == gi && items[(size_t)i].n_points > 0) g.ids.push_back(i);
    std::stable_sort(g.ids.begin(), g.ids.end(),
                     [&](int a, int b) { return items[(size_t)a].order > items[(size_t)b].order; });
    g.n_items = (int)g.ids.size();
    if (!g.n_items) continue;
    std::vector<long long> offs(1, 0);
    for (int j = 0; j < g.n_items; ++j) {
      const ItemDev &it = items[(size_t)g.ids[(size_t)j]];
      g.items.push_back(it);
      offs.push_back(offs.back() + (it.n_points + it.chunk_points - 1) / it.chunk_points);
      p->where_group[(size_t)g.ids[(size_t)j]] = gi;
      p->where_pos[(size_t)g.ids[(size_t)j]] = j;
    }
    g.n_chunks = offs.back();
    if (g.n_chunks > INT32_MAX) {
      plan_free(p);
      return fail(KB_E_INVALID, "too many points in one plan");
    }
    g.grid = (int)std::min<long long>(g.n_chunks, gi == 0 ? (long long)ctx->sm_count * ctx->ctas_per_sm
                                                          : (long long)ctx->sm_count * 4);
    cudaError_t e = device_malloc(&g.d_items, sizeof(ItemDev) * g.n_items);
    if (e == cudaSuccess) e = device_malloc(&g.d_offs, sizeof(long long) * offs.size());
    if (e == cudaSuccess) e = device_malloc(&g.d_cnt, sizeof(int));
    if (e == cudaSuccess) e = device_malloc(&g.d_part, sizeof(ChunkPartial) * (size_t)g.n_chunks);
    if (e == cudaSuccess && gi == 0) e = device_malloc(&g.d_pts, sizeof(double) * PTS_SLOT * (size_t)g.grid);
    if (e == cudaSuccess) e = device_malloc(&g.d_acc, sizeof(kb_accum) * g.n_items);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(g.d_items, g.items.data(), sizeof(ItemDev) * g.n_items, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(g.d_offs, offs.data(), sizeof(long long) * offs.size(), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      plan_free(p);
      return fail(KB_E_NOMEM, std::string("kb_plan_create: ") + cudaGetErrorString(e));
    }
  }
  for (auto &f : p->fills) f.pos = p->where_pos[(size_t)f.pos];
  *out = p;
  return KB_OK;
}

// The launch sequence of one run (captured into the plan's graph).
static int plan_enqueue(kb_context *ctx, kb_plan *p, cudaStream_t st) {
  for (const kb_flow *f : p->splines) KB_CUDA(launch_spline_knots(f->master, f->dim, f->knots, st));
  for (const auto &f : p->fills) {
    const uint32_t *kf = &p->g[f.gi].d_items[f.pos].k_first;
    KB_CUDA(launch_flow_map(f.layout, 1, f.n, nullptr, f.rng, 0, kf, 1, f.buf, f.buf + (size_t)f.n * f.order, ctx->d_err,
                            ctx->sm_count, st));
  }
  for (int gi = 0; gi < 2; ++gi) {
    auto &g = p->g[gi];
    if (!g.n_items) continue;
    KB_CUDA(cudaMemsetAsync(g.d_acc, 0, sizeof(kb_accum) * g.n_items, st));
    KB_CUDA(cudaMemsetAsync(g.d_cnt, 0, sizeof(int), st));
    Launch L;
    memset(&L, 0, sizeof(L));
    L.items = g.d_items;
    L.n_items = g.n_items;
    L.any_cubic = items_any_cubic(g.items.data(), g.items.size());
    L.chunk_offsets = g.d_offs;
    L.n_chunks = (int)g.n_chunks;
    L.chunk_counter = g.d_cnt;
    L.mode = IN_SOBOL;
    L.partials = g.d_part;
    L.pts = g.d_pts;
    L.err = ctx->d_err;
    if (gi == 0) {
      KB_CUDA(launch_tree(L, g.grid, st));
      KB_CUDA(launch_fallback(L, ctx->sm_count * 4, st));
    } else {
      KB_CUDA(launch_direct(L, g.grid, st));
    }
    KB_CUDA(launch_reduce(L, g.d_acc, st));
  }
  return KB_OK;
}

int kb_plan_launch(kb_context *ctx, kb_plan *plan) {
  KB_CHECK(ctx && plan, "kb_plan_launch: null argument");
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  if (!plan->exec) {
    cudaGraph_t graph = nullptr;
    KB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = plan_enqueue(ctx, plan, st);
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return fail(KB_E_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&plan->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(KB_E_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  }
  KB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), st));
  if (ctx->timing) KB_CUDA(cudaEventRecord(ctx->ev[0], st));
  KB_CUDA(cudaGraphLaunch(plan->exec, st));
  if (ctx->timing) KB_CUDA(cudaEventRecord(ctx->ev[1], st));
  return KB_OK;
}

int kb_plan_result(kb_context *ctx, kb_plan *plan, kb_accum *acc) {
  KB_CHECK(ctx && plan && (plan->n_work == 0 || acc), "kb_plan_result: null argument");
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  std::vector<kb_accum> part[2];
  for (int gi = 0; gi < 2; ++gi) {
    part[gi].resize((size_t)plan->g[gi].n_items);
    if (plan->g[gi].n_items)
      KB_CUDA(cudaMemcpyAsync(part[gi].data(), plan->g[gi].d_acc, sizeof(kb_accum) * plan->g[gi].n_items,
                              cudaMemcpyDeviceToHost, st));
  }
  int err = 0;
  KB_CUDA(cudaMemcpyAsync(&err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaStreamSynchronize(st));
  if (ctx->timing) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]) == cudaSuccess) {
      ctx->last_ms[0] = ms;
      ctx->last_ms[1] = ctx->last_ms[2] = 0.0;
    }
  }
  if (err & 1) return fail(KB_E_RANGE, "g0 evaluated outside its tabulated time window");
  if (err & 2) return fail(KB_E_CUDA, "a flow kernel's wait on the tensor cores ran out");
  for (int gi = 0; gi < 2; ++gi)
    for (int j = 0; j < plan->g[gi].n_items; ++j) {
      kb_accum &a = acc[plan->g[gi].ids[(size_t)j]];
      const kb_accum &q = part[gi][(size_t)j];
      a.sum_re += q.sum_re;
      a.sum_im += q.sum_im;
      a.n_points += q.n_points;
      a.n_in_domain += q.n_in_domain;
      a.n_fallback += q.n_fallback;
    }
  return KB_OK;
}

int kb_plan_set_k_first(kb_context *ctx, kb_plan *plan, int item, uint32_t k_first) {
  KB_CHECK(ctx && plan, "kb_plan_set_k_first: null argument");
  KB_CHECK(item >= 0 && item < plan->n_work, "work item index out of range");
  const int gi = plan->where_group[(size_t)item], pos = plan->where_pos[(size_t)item];
  if (gi < 0) return KB_OK; // no points
  ItemDev &it = plan->g[gi].items[(size_t)pos];
  int st = check_sobol_range(plan->rng[(size_t)item], k_first, it.n_points);
  if (st) return st;
  it.k_first = k_first;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  KB_CUDA(cudaMemcpyAsync(&plan->g[gi].d_items[pos].k_first, &it.k_first, sizeof(uint32_t), cudaMemcpyHostToDevice,
                          ctx->stream));
  KB_CUDA(cudaStreamSynchronize(ctx->stream));
  return KB_OK;
}

int kb_context_set_launch(kb_context *ctx, int order, int chunk_points, int ctas_per_sm) {
  KB_CHECK(ctx, "null context");
  KB_CHECK(order == -1 || (order >= 0 && order <= MAX_ORDER), "order must be -1 or in [0, 16]");
  KB_CHECK(chunk_points >= 1 && chunk_points <= CHUNK_POINTS, "chunk_points must be in [1, 128]");
  KB_CHECK(ctas_per_sm >= 0 && ctas_per_sm <= 4, "ctas_per_sm must be 0 (keep) or 1..4");
  std::lock_guard<std::mutex> lk(ctx->mu);
  for (int n = 0; n <= MAX_ORDER; ++n)
    if (order == -1 || order == n) ctx->chunk_points[n] = chunk_points;
  if (ctas_per_sm) ctx->ctas_per_sm = ctas_per_sm;
  return KB_OK;
}

int kb_context_get_launch(kb_context *ctx, int order, int *chunk_points, int *ctas_per_sm) {
  KB_CHECK(ctx && order >= 0 && order <= MAX_ORDER, "kb_context_get_launch: bad argument");
  if (chunk_points) *chunk_points = ctx->chunk_points[order];
  if (ctas_per_sm) *ctas_per_sm = ctx->ctas_per_sm;
  return KB_OK;
}

// ------------------------------------------------------------------ peaks
int kb_fp64_peak(kb_context *ctx, int iters, double *flops_per_s) {
  KB_CHECK(ctx && flops_per_s && iters > 0, "kb_fp64_peak: bad argument");
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  const int block = 256, grid = ctx->sm_count * 8;
  DevBuf sink;
  KB_CUDA(sink.alloc(grid * sizeof(double), ctx->stream));
  cudaEvent_t e0, e1;
  KB_CUDA(cudaEventCreate(&e0));
  KB_CUDA(cudaEventCreate(&e1));
  KB_CUDA(launch_fp64_peak(iters, sink.as<double>(), grid, block, ctx->stream)); // warm-up
  KB_CUDA(cudaEventRecord(e0, ctx->stream));
  KB_CUDA(launch_fp64_peak(iters, sink.as<double>(), grid, block, ctx->stream));
  KB_CUDA(cudaEventRecord(e1, ctx->stream));
  KB_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  KB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *flops_per_s = 2.0 * 8.0 * (double)iters * grid * block / (ms * 1e-3);
  return KB_OK;
}

} // extern "C"

// ------------------------------------------------- integrate without allocating
// kb_integrate_noalloc: the integrate path with its scratch (item descriptors, chunk
// offsets, the scheduling counter, per-chunk partial sums and the per-item sums) in one
// file-scope device array instead of memory allocated per call. It serves callers that
// cannot call cudaMalloc: a host application whose own allocator owns all of the
// device's memory, or a latency-bound loop that must not pay cudaMalloc's implicit
// device synchronisation.
//
// The array is KB_NOALLOC_SCRATCH_BYTES per device, held by every GPU that loads the
// library until the process exits. All calls share it and it keeps the last call's
// contents: each call clears the counter and the sums it needs, and two calls whose
// work overlaps on the GPU (different streams, contexts or threads on one device) race
// on it. The device address of the array is looked up with cudaGetSymbolAddress the
// first time the entry point runs on a device (with that device current); make that
// first call before any stream capture.
namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
constexpr size_t NOALLOC_ITEMS_OFF = 0;
constexpr size_t NOALLOC_OFFS_OFF = NOALLOC_ITEMS_OFF + sizeof(ItemDev) * KB_NOALLOC_MAX_ITEMS;
constexpr size_t NOALLOC_ACC_OFF = ((NOALLOC_OFFS_OFF + sizeof(long long) * (KB_NOALLOC_MAX_ITEMS + 1)) + 255) / 256 * 256;
constexpr size_t NOALLOC_CNT_OFF = NOALLOC_ACC_OFF + sizeof(kb_accum) * 2 * KB_NOALLOC_MAX_ITEMS;
constexpr size_t NOALLOC_PART_OFF = (NOALLOC_CNT_OFF + sizeof(int) + 255) / 256 * 256;
constexpr size_t NOALLOC_PTS_OFF =
    (NOALLOC_PART_OFF + sizeof(ChunkPartial) * (size_t)KB_NOALLOC_MAX_CHUNKS + 255) / 256 * 256;
constexpr size_t NOALLOC_PTS_SLOTS = (KB_NOALLOC_SCRATCH_BYTES - NOALLOC_PTS_OFF) / (PTS_SLOT * sizeof(double));
// one set-up slot per resident tree CTA of a 148-SM B200 at the most CTAs per SM the
// launch shape allows; a device with more SMs runs the tree with a grid capped at the slots
constexpr size_t NOALLOC_B200_TREE_CTAS = 148 * 4;
static_assert(NOALLOC_PTS_SLOTS >= NOALLOC_B200_TREE_CTAS, "scratch too small for one set-up slot per resident CTA");

static __device__ __align__(256) unsigned char kb_noalloc_scratch[KB_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mu;
unsigned char *g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};

// Device address of kb_noalloc_scratch on the current device (looked up once per device).
int noalloc_scratch(int device, unsigned char **out) {
  if (device < 0 || device >= NOALLOC_MAX_DEVICES) return fail(KB_E_INVALID, "device index too large for kb_integrate_noalloc");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, kb_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(KB_E_CUDA, std::string("cudaGetSymbolAddress(kb_noalloc_scratch): ") + cudaGetErrorString(e));
    g_noalloc_addr[device] = static_cast<unsigned char *>(p);
  }
  *out = g_noalloc_addr[device];
  return KB_OK;
}
} // namespace

extern "C" int kb_integrate_noalloc(kb_context *ctx, const kb_work *work, int n_work, kb_accum *acc) {
  KB_CHECK(ctx && (n_work == 0 || (work && acc)), "kb_integrate_noalloc: null argument");
  if (n_work < 0 || n_work > KB_NOALLOC_MAX_ITEMS)
    return fail(KB_E_INVALID, "kb_integrate_noalloc takes at most KB_NOALLOC_MAX_ITEMS (64) work items");
  if (n_work == 0) return KB_OK;
  ItemDev items[KB_NOALLOC_MAX_ITEMS];
  int group_of[KB_NOALLOC_MAX_ITEMS];
  long long chunks_total = 0;
  for (int i = 0; i < n_work; ++i) {
    const kb_work &w = work[i];
    int st = check_integrand(w.m, &w.f, w.order);
    if (st) return st;
    KB_CHECK(w.rng, "work item without a Sobol generator");
    KB_CHECK(w.n_points >= 0, "n_points must be >= 0");
    KB_CHECK(w.order >= 1, "integrator dimension must be > 0 (Dimension of the integration space must be > 0.)");
    if (w.rng->dim < w.order) return fail(KB_E_INVALID, "Sobol generator has fewer dimensions than the order");
    st = check_sobol_range(w.rng, w.k_first, w.n_points);
    if (st) return st;
    KB_CHECK(!w.flow, "kb_integrate_noalloc does not take work items with a learned flow");
    ItemDev &it = items[i];
    it = make_item(w.m, &w.f, w.order);
    st = make_chain(w.chain, w.chain_len, it.chain);
    if (st) return st;
    st = check_chain_dims(w.chain, w.chain_len, w.order);
    if (st) return st;
    it.chain_len = w.chain_len;
    it.chain_start = w.chain_len;
    it.rng = sobol_dev(w.rng);
    it.k_first = w.k_first;
    it.n_points = w.n_points;
    group_of[i] = it.spin_symmetric ? 0 : 1;
    // the same scheduling chunks as kb_integrate (the context's launch shape of the order,
    // smaller for a small item), so that the sums are added in the same order
    it.chunk_points = item_chunk(ctx, w.order, w.n_points);
    chunks_total += (w.n_points + it.chunk_points - 1) / it.chunk_points;
  }
  if (chunks_total > KB_NOALLOC_MAX_CHUNKS)
    return fail(KB_E_INVALID, "kb_integrate_noalloc: more than KB_NOALLOC_MAX_CHUNKS (65,536) scheduling chunks in "
                              "one call (8,388,608 points with the default 128-point chunks)");
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  unsigned char *base = nullptr;
  int st = noalloc_scratch(ctx->device, &base);
  if (st) return st;
  cudaStream_t stream = ctx->stream;
  ItemDev *d_items = reinterpret_cast<ItemDev *>(base + NOALLOC_ITEMS_OFF);
  long long *d_offs = reinterpret_cast<long long *>(base + NOALLOC_OFFS_OFF);
  kb_accum *d_acc = reinterpret_cast<kb_accum *>(base + NOALLOC_ACC_OFF);
  int *d_cnt = reinterpret_cast<int *>(base + NOALLOC_CNT_OFF);
  ChunkPartial *d_part = reinterpret_cast<ChunkPartial *>(base + NOALLOC_PART_OFF);
  double *d_pts = reinterpret_cast<double *>(base + NOALLOC_PTS_OFF);
  KB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), stream));
  KB_CUDA(cudaMemsetAsync(d_acc, 0, sizeof(kb_accum) * 2 * KB_NOALLOC_MAX_ITEMS, stream));
  // Group 0 (tree) and group 1 (pivoted LU), heaviest orders first within a group; the
  // groups use the item and chunk regions in turn, their sums land in separate halves.
  int ids[2][KB_NOALLOC_MAX_ITEMS];
  int nids[2] = {0, 0};
  for (int g = 0; g < 2; ++g) {
    for (int i = 0; i < n_work; ++i)
      if (group_of[i] == g && items[i].n_points > 0) ids[g][nids[g]++] = i;
    for (int a = 1; a < nids[g]; ++a) // stable insertion sort by order, descending
      for (int b = a; b > 0 && items[ids[g][b]].order > items[ids[g][b - 1]].order; --b) {
        int t = ids[g][b];
        ids[g][b] = ids[g][b - 1];
        ids[g][b - 1] = t;
      }
  }
  ItemDev sorted[KB_NOALLOC_MAX_ITEMS];
  long long offs[KB_NOALLOC_MAX_ITEMS + 1];
  for (int g = 0; g < 2; ++g) {
    if (nids[g] == 0) continue;
    offs[0] = 0;
    for (int j = 0; j < nids[g]; ++j) {
      sorted[j] = items[ids[g][j]];
      offs[j + 1] = offs[j] + (sorted[j].n_points + sorted[j].chunk_points - 1) / sorted[j].chunk_points;
    }
    KB_CUDA(cudaMemcpyAsync(d_items, sorted, sizeof(ItemDev) * nids[g], cudaMemcpyHostToDevice, stream));
    KB_CUDA(cudaMemcpyAsync(d_offs, offs, sizeof(long long) * (nids[g] + 1), cudaMemcpyHostToDevice, stream));
    KB_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(int), stream));
    Launch L;
    memset(&L, 0, sizeof(L));
    L.items = d_items;
    L.n_items = nids[g];
    L.any_cubic = items_any_cubic(sorted, (size_t)nids[g]);
    L.chunk_offsets = d_offs;
    L.n_chunks = (int)offs[nids[g]];
    L.chunk_counter = d_cnt;
    L.mode = IN_SOBOL;
    L.partials = d_part;
    L.pts = d_pts;
    L.err = ctx->d_err;
    if (g == 0) {
      // the tree grid of kb_integrate, capped at the set-up slots the array holds
      const long long slots = (long long)NOALLOC_PTS_SLOTS;
      const long long tgrid = std::min<long long>(L.n_chunks, (long long)ctx->sm_count * ctx->ctas_per_sm);
      KB_CUDA(launch_tree(L, (int)std::min<long long>(tgrid, slots), stream));
      KB_CUDA(launch_fallback(L, ctx->sm_count * 4, stream));
    } else {
      KB_CUDA(launch_direct(L, (int)std::min<long long>(L.n_chunks, ctx->sm_count * 4), stream));
    }
    KB_CUDA(launch_reduce(L, d_acc + g * KB_NOALLOC_MAX_ITEMS, stream));
  }
  kb_accum part[2][KB_NOALLOC_MAX_ITEMS];
  int err = 0;
  KB_CUDA(cudaMemcpyAsync(part, d_acc, sizeof(part), cudaMemcpyDeviceToHost, stream));
  KB_CUDA(cudaMemcpyAsync(&err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
  KB_CUDA(cudaStreamSynchronize(stream));
  if (err & 1) return fail(KB_E_RANGE, "g0 evaluated outside its tabulated time window");
  for (int g = 0; g < 2; ++g)
    for (int j = 0; j < nids[g]; ++j) {
      kb_accum &a = acc[ids[g][j]];
      const kb_accum &p = part[g][j];
      a.sum_re += p.sum_re;
      a.sum_im += p.sum_im;
      a.n_points += p.n_points;
      a.n_in_domain += p.n_in_domain;
      a.n_fallback += p.n_fallback;
    }
  return KB_OK;
}

