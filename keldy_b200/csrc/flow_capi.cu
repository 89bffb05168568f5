// C ABI of the learned coupling-flow warper (kb_flow_* in include/keldy_b200.h): weights,
// the sampling and density maps, gradients and Adam training on the kernels of flow.cu.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <vector>

#include "kb_host.h"
#include "kb_spline.cuh"

using namespace kb;

namespace {

constexpr int TRAIN_BATCH_MAX = 1 << 16;

// API order [matrix][out][in] <-> internal order [matrix][in][out]
void api_to_internal(const float *api, float *inr) {
  for (int m = 0; m < FLOW_NMAT; ++m)
    for (int r = 0; r < FLOW_W; ++r)
      for (int k = 0; k < FLOW_W; ++k) inr[(size_t)m * FLOW_MAT + k * FLOW_W + r] = api[(size_t)m * FLOW_MAT + r * FLOW_W + k];
}
void internal_to_api(const float *inr, float *api) {
  for (int m = 0; m < FLOW_NMAT; ++m)
    for (int r = 0; r < FLOW_W; ++r)
      for (int k = 0; k < FLOW_W; ++k) api[(size_t)m * FLOW_MAT + r * FLOW_W + k] = inr[(size_t)m * FLOW_MAT + k * FLOW_W + r];
}

int flow_error(kb_context *ctx) {
  int err = 0;
  KB_CUDA(cudaMemcpyAsync(&err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  KB_CUDA(cudaStreamSynchronize(ctx->stream));
  if (err & 2) return fail(KB_E_CUDA, "a flow kernel's wait on the tensor cores ran out");
  return KB_OK;
}

// Loss partials and weight-gradient partials of `count` points (device x, w, index).
int train_pass(kb_flow *f, long long count, const float *dx, const float *dw, const int *dindex, float *partials,
               float *loss_part, float *xs, int grid) {
  kb_context *ctx = f->ctx;
  KB_CUDA(launch_flow_train(f->layout, count, dx, dw, dindex, 1.0f / (float)count, partials, loss_part, xs, ctx->d_err,
                            grid, ctx->stream));
  return KB_OK;
}

int train_grid(const kb_flow *f, long long count) {
  const long long tiles = (count + FLOW_TILE - 1) / FLOW_TILE;
  return (int)std::min<long long>(tiles, f->ctx->sm_count);
}

// CTAs of the spline flow's gradient kernel (256 threads each, grid-stride over the batch).
int spline_grid(const kb_flow *f, long long count) {
  return (int)std::max<long long>(1, std::min<long long>((count + 255) / 256, 2LL * f->ctx->sm_count));
}

// The flows whose parameters are a plain fp32 vector trained by their own gradient and Adam
// kernels (the separable and the autoregressive spline flows), and those kernels by kind.
bool param_flow(const kb_flow *f) { return f->layout.kind != FLOW_KIND_COUPLING; }
int param_grid(const kb_flow *f, long long count) {
  return f->layout.kind == FLOW_KIND_AR_SPLINE ? ar_grad_grid(count, f->ctx->sm_count) : spline_grid(f, count);
}
size_t param_partial(const kb_flow *f) {
  return f->layout.kind == FLOW_KIND_AR_SPLINE ? (size_t)ar_num_params(f->dim)
                                                : (size_t)f->dim * spline_grad_per_dim();
}
cudaError_t param_grad(const kb_flow *f, long long count, const float *x, const float *w, const int *index,
                       double inv_batch, double *partials, double *loss_part, int grid, cudaStream_t st) {
  if (f->layout.kind == FLOW_KIND_AR_SPLINE)
    return launch_ar_grad(f->master, f->dim, count, x, w, index, inv_batch, partials, loss_part, grid, st);
  return launch_spline_grad(f->master, f->dim, count, x, w, index, inv_batch, partials, loss_part, grid, st);
}
cudaError_t param_adam(kb_flow *f, const double *partials, int nparts, const double *loss_part, double *loss_out,
                       float *grad_out, float lr, float beta1, float beta2, float eps, float bc1, float bc2,
                       cudaStream_t st) {
  if (f->layout.kind == FLOW_KIND_AR_SPLINE)
    return launch_ar_adam(f->master, f->adam_m, f->adam_v, f->dim, partials, nparts, loss_part, loss_out, grad_out,
                          lr, beta1, beta2, eps, bc1, bc2, st);
  return launch_spline_adam(f->master, f->adam_m, f->adam_v, f->dim, partials, nparts, loss_part, loss_out, grad_out,
                            lr, beta1, beta2, eps, bc1, bc2, st);
}

// kb_flow_train for the spline flows (the caller holds the context's lock): per step the
// batch's derivative partials, then the gradient and the Adam step, cosine-decayed
// learning rate as for the coupling flow.
int spline_train(kb_flow *f, int64_t count, const std::vector<float> &hx, const std::vector<float> &hw,
                 const kb_flow_train_cfg *cfg, int64_t batch, int64_t per_epoch, int64_t steps, double *loss_hist,
                 int *n_steps) {
  kb_context *ctx = f->ctx;
  cudaStream_t st = ctx->stream;
  const int N = f->dim;
  const int sg = param_grid(f, batch);
  (void)N;
  DevBuf dx, dw, di, dpart, dlp, dhist;
  KB_CUDA(dx.alloc(hx.size() * sizeof(float), st));
  KB_CUDA(dw.alloc(hw.size() * sizeof(float), st));
  KB_CUDA(di.alloc((size_t)count * sizeof(int), st));
  KB_CUDA(dpart.alloc((size_t)sg * param_partial(f) * sizeof(double), st));
  KB_CUDA(dlp.alloc((size_t)sg * sizeof(double), st));
  KB_CUDA(dhist.alloc((size_t)steps * sizeof(double), st));
  KB_CUDA(cudaMemcpyAsync(dx.p, hx.data(), hx.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemcpyAsync(dw.p, hw.data(), hw.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  std::vector<int> perm((size_t)count);
  std::iota(perm.begin(), perm.end(), 0);
  std::mt19937_64 shuffler(cfg->seed);
  const double pi = 3.14159265358979323846;
  int64_t s = 0;
  for (int ep = 0; ep < cfg->epochs; ++ep) {
    std::shuffle(perm.begin(), perm.end(), shuffler);
    KB_CUDA(cudaStreamSynchronize(st)); // the previous epoch's steps read the old order
    KB_CUDA(cudaMemcpyAsync(di.p, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    for (int64_t b = 0; b < per_epoch; ++b, ++s) {
      KB_CUDA(param_grad(f, batch, dx.as<float>(), dw.as<float>(), di.as<int>() + b * batch, 1.0 / (double)batch,
                         dpart.as<double>(), dlp.as<double>(), sg, st));
      const int64_t t = ++f->adam_step;
      const double lr = cfg->lr_final + 0.5 * (cfg->lr - cfg->lr_final) * (1.0 + std::cos(pi * (double)s / (double)steps));
      const float bc1 = (float)(1.0 - std::pow((double)cfg->beta1, (double)t));
      const float bc2 = (float)(1.0 - std::pow((double)cfg->beta2, (double)t));
      KB_CUDA(param_adam(f, dpart.as<double>(), sg, dlp.as<double>(), dhist.as<double>() + s, nullptr, (float)lr,
                         cfg->beta1, cfg->beta2, cfg->eps, bc1, bc2, st));
    }
  }
  std::vector<double> hist((size_t)steps);
  KB_CUDA(cudaMemcpyAsync(hist.data(), dhist.p, hist.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaStreamSynchronize(st));
  if (loss_hist)
    for (int64_t i = 0; i < steps; ++i) loss_hist[i] = hist[(size_t)i];
  if (n_steps) *n_steps = (int)steps;
  return KB_OK;
}

} // namespace

extern "C" {

int kb_flow_create(kb_context *ctx, int dim, uint64_t seed, kb_flow **out) {
  KB_CHECK(ctx && out, "kb_flow_create: null argument");
  KB_CHECK(dim >= 2 && dim <= FLOW_MAX_DIM, "flow dimension must be in [2, 8]");
  std::vector<float> api((size_t)FLOW_NPARAM, 0.0f), inr((size_t)FLOW_NPARAM);
  std::mt19937_64 gen(seed);
  const double a = std::sqrt(6.0 / FLOW_W);
  for (int l = 0; l < FLOW_LAYERS; ++l)
    for (int m = 0; m < 2; ++m)
      for (int i = 0; i < FLOW_MAT; ++i) {
        const double u = (double)(gen() >> 11) * (1.0 / 9007199254740992.0);
        api[(size_t)(3 * l + m) * FLOW_MAT + i] = (float)(a * (2.0 * u - 1.0));
      }
  api_to_internal(api.data(), inr.data());
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  auto *f = new kb_flow;
  f->ctx = ctx;
  f->device = ctx->device;
  f->dim = dim;
  flow_layout(dim, f->layout);
  const size_t nb = (size_t)FLOW_NPARAM * sizeof(float);
  cudaError_t e = device_malloc(&f->master, nb);
  if (e == cudaSuccess) e = device_malloc(&f->adam_m, nb);
  if (e == cudaSuccess) e = device_malloc(&f->adam_v, nb);
  if (e == cudaSuccess) e = device_malloc(&f->img, (size_t)FLOW_NPARAM * sizeof(uint16_t));
  // on the library's stream, which does not synchronise with the legacy default stream
  if (e == cudaSuccess) e = cudaMemcpyAsync(f->master, inr.data(), nb, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(f->adam_m, 0, nb, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(f->adam_v, 0, nb, ctx->stream);
  if (e == cudaSuccess) e = launch_flow_pack(f->master, f->img, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    cudaFree(f->master);
    cudaFree(f->adam_m);
    cudaFree(f->adam_v);
    cudaFree(f->img);
    delete f;
    return fail(KB_E_CUDA, std::string("kb_flow_create: ") + cudaGetErrorString(e));
  }
  f->layout.img = f->img;
  *out = f;
  return KB_OK;
}

int kb_flow_create_kind(kb_context *ctx, int dim, int kind, uint64_t seed, kb_flow **out) {
  if (kind == KB_FLOW_COUPLING) return kb_flow_create(ctx, dim, seed, out);
  KB_CHECK(ctx && out, "kb_flow_create_kind: null argument");
  KB_CHECK(kind == KB_FLOW_SPLINE || kind == KB_FLOW_AR_SPLINE,
           "flow kind must be KB_FLOW_COUPLING, KB_FLOW_SPLINE or KB_FLOW_AR_SPLINE");
  KB_CHECK(dim >= 1 && dim <= FLOW_MAX_DIM, "flow dimension must be in [1, 8]");
  // identity map: equal bins, knot derivatives 1 (softplus(c) = 1 - SPL_MIN_DERIV); the
  // autoregressive flow holds them in each dimension's constant feature, the other
  // features' weights zero
  std::vector<float> init((size_t)FLOW_NPARAM, 0.0f);
  const float c0 = (float)std::log(std::expm1(1.0 - SPL_MIN_DERIV));
  for (int d = 0; d < dim; ++d)
    for (int k = 0; k <= SPL_BINS; ++k) {
      if (kind == KB_FLOW_SPLINE)
        init[(size_t)d * SPL_PER_DIM + 2 * SPL_BINS + k] = c0;
      else
        init[(size_t)ar_offset(d) + (size_t)(2 * SPL_BINS + k) * ar_features(d)] = c0;
    }
  (void)seed;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  auto *f = new kb_flow;
  f->ctx = ctx;
  f->device = ctx->device;
  f->dim = dim;
  f->layout.kind = kind == KB_FLOW_SPLINE ? FLOW_KIND_SPLINE : FLOW_KIND_AR_SPLINE;
  f->layout.dim = dim;
  const size_t nb = (size_t)FLOW_NPARAM * sizeof(float);
  cudaError_t e = device_malloc(&f->master, nb);
  if (e == cudaSuccess) e = device_malloc(&f->adam_m, nb);
  if (e == cudaSuccess) e = device_malloc(&f->adam_v, nb);
  if (e == cudaSuccess) e = device_malloc(&f->knots, (size_t)FLOW_MAX_DIM * SPL_KNOT_DOUBLES * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyAsync(f->master, init.data(), nb, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(f->adam_m, 0, nb, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(f->adam_v, 0, nb, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    cudaFree(f->master);
    cudaFree(f->adam_m);
    cudaFree(f->adam_v);
    cudaFree(f->knots);
    delete f;
    return fail(KB_E_CUDA, std::string("kb_flow_create_kind: ") + cudaGetErrorString(e));
  }
  f->layout.spline = f->master;
  f->layout.knots = f->knots;
  *out = f;
  return KB_OK;
}

int kb_flow_num_params(const kb_flow *f) {
  if (!f) return 0;
  if (f->layout.kind == FLOW_KIND_AR_SPLINE) return ar_num_params(f->dim);
  return f->layout.kind == FLOW_KIND_SPLINE ? f->dim * SPL_PER_DIM : FLOW_NPARAM;
}

int kb_flow_destroy(kb_flow *f) {
  if (!f) return KB_OK;
  cudaSetDevice(f->device);
  cudaFree(f->master);
  cudaFree(f->adam_m);
  cudaFree(f->adam_v);
  cudaFree(f->img);
  cudaFree(f->knots);
  delete f;
  return KB_OK;
}

int kb_flow_dim(const kb_flow *f) { return f ? f->dim : 0; }

int kb_flow_get_params(kb_flow *f, float *params) {
  KB_CHECK(f && params, "kb_flow_get_params: null argument");
  if (param_flow(f)) {
    std::lock_guard<std::mutex> lk(f->ctx->mu);
    KB_CUDA(cudaSetDevice(f->device));
    KB_CUDA(cudaMemcpyAsync(params, f->master, (size_t)kb_flow_num_params(f) * sizeof(float), cudaMemcpyDeviceToHost,
                            f->ctx->stream));
    KB_CUDA(cudaStreamSynchronize(f->ctx->stream));
    return KB_OK;
  }
  std::vector<float> inr((size_t)FLOW_NPARAM);
  std::lock_guard<std::mutex> lk(f->ctx->mu);
  KB_CUDA(cudaSetDevice(f->device));
  KB_CUDA(cudaMemcpyAsync(inr.data(), f->master, inr.size() * sizeof(float), cudaMemcpyDeviceToHost, f->ctx->stream));
  KB_CUDA(cudaStreamSynchronize(f->ctx->stream));
  internal_to_api(inr.data(), params);
  return KB_OK;
}

// Resets the Adam moments: new weights start a new optimisation.
int kb_flow_set_params(kb_flow *f, const float *params) {
  KB_CHECK(f && params, "kb_flow_set_params: null argument");
  for (int i = 0; i < kb_flow_num_params(f); ++i)
    if (!std::isfinite(params[i])) return fail(KB_E_INVALID, "flow parameters must be finite");
  if (param_flow(f)) {
    std::lock_guard<std::mutex> lk(f->ctx->mu);
    KB_CUDA(cudaSetDevice(f->device));
    cudaStream_t st = f->ctx->stream;
    const size_t nb = (size_t)kb_flow_num_params(f) * sizeof(float);
    KB_CUDA(cudaMemcpyAsync(f->master, params, nb, cudaMemcpyHostToDevice, st));
    KB_CUDA(cudaMemsetAsync(f->adam_m, 0, nb, st));
    KB_CUDA(cudaMemsetAsync(f->adam_v, 0, nb, st));
    KB_CUDA(cudaStreamSynchronize(st));
    f->adam_step = 0;
    return KB_OK;
  }
  std::vector<float> inr((size_t)FLOW_NPARAM);
  api_to_internal(params, inr.data());
  std::lock_guard<std::mutex> lk(f->ctx->mu);
  KB_CUDA(cudaSetDevice(f->device));
  cudaStream_t st = f->ctx->stream;
  const size_t nb = inr.size() * sizeof(float);
  KB_CUDA(cudaMemcpyAsync(f->master, inr.data(), nb, cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemsetAsync(f->adam_m, 0, nb, st));
  KB_CUDA(cudaMemsetAsync(f->adam_v, 0, nb, st));
  KB_CUDA(launch_flow_pack(f->master, f->img, st));
  KB_CUDA(cudaStreamSynchronize(st));
  f->adam_step = 0;
  return KB_OK;
}

int kb_flow_map(kb_flow *f, int direction, int64_t count, const double *in, double *out, double *out2) {
  KB_CHECK(f, "kb_flow_map: null flow");
  KB_CHECK(direction == 0 || direction == 1, "direction must be 0 (density) or 1 (sampling)");
  KB_CHECK(count >= 0 && (count == 0 || (in && out && out2)), "kb_flow_map: null buffer");
  if (count == 0) return KB_OK;
  for (int64_t i = 0; i < count * f->dim; ++i)
    if (!(in[i] >= 0.0 && in[i] <= 1.0)) return fail(KB_E_INVALID, "flow inputs must lie in [0, 1]");
  kb_context *ctx = f->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const size_t nb = (size_t)count * f->dim * sizeof(double);
  DevBuf din, dout, dout2;
  KB_CUDA(din.alloc(nb, st));
  KB_CUDA(dout.alloc(nb, st));
  KB_CUDA(dout2.alloc((size_t)count * sizeof(double), st));
  KB_CUDA(cudaMemcpyAsync(din.p, in, nb, cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), st));
  SobolDev none;
  memset(&none, 0, sizeof(none));
  KB_CUDA(launch_flow_map(f->layout, direction, count, din.as<double>(), none, 0, nullptr, 0, dout.as<double>(),
                          dout2.as<double>(), ctx->d_err, ctx->sm_count, st));
  KB_CUDA(cudaMemcpyAsync(out, dout.p, nb, cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaMemcpyAsync(out2, dout2.p, (size_t)count * sizeof(double), cudaMemcpyDeviceToHost, st));
  return flow_error(ctx);
}

int kb_flow_sample(kb_flow *f, const kb_sobol *rng, uint32_t k_first, int64_t count, double *x, double *jac) {
  KB_CHECK(f && rng, "kb_flow_sample: null argument");
  KB_CHECK(count >= 0 && (count == 0 || (x && jac)), "kb_flow_sample: null buffer");
  KB_CHECK(rng->dim >= f->dim, "Sobol generator has fewer dimensions than the flow");
  int rc = check_sobol_range(rng, k_first, count);
  if (rc) return rc;
  if (count == 0) return KB_OK;
  kb_context *ctx = f->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const size_t nb = (size_t)count * f->dim * sizeof(double);
  DevBuf dx, dj;
  KB_CUDA(dx.alloc(nb, st));
  KB_CUDA(dj.alloc((size_t)count * sizeof(double), st));
  KB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), st));
  KB_CUDA(launch_flow_map(f->layout, 1, count, nullptr, sobol_dev(rng), k_first, nullptr, 1, dx.as<double>(),
                          dj.as<double>(), ctx->d_err, ctx->sm_count, st));
  KB_CUDA(cudaMemcpyAsync(x, dx.p, nb, cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaMemcpyAsync(jac, dj.p, (size_t)count * sizeof(double), cudaMemcpyDeviceToHost, st));
  return flow_error(ctx);
}

int kb_flow_gradient(kb_flow *f, int64_t count, const double *x, const double *w, float *grad, double *loss) {
  KB_CHECK(f && x && w && grad, "kb_flow_gradient: null argument");
  KB_CHECK(count >= 1 && count <= (int64_t)1 << 24, "kb_flow_gradient: count must be in [1, 2^24]");
  const int N = f->dim;
  std::vector<float> hx((size_t)count * N), hw((size_t)count);
  for (int64_t i = 0; i < count * N; ++i) {
    if (!(x[i] >= 0.0 && x[i] <= 1.0)) return fail(KB_E_INVALID, "flow inputs must lie in [0, 1]");
    hx[(size_t)i] = (float)x[i];
  }
  for (int64_t i = 0; i < count; ++i) {
    if (!(w[i] >= 0.0) || !std::isfinite(w[i])) return fail(KB_E_INVALID, "weights must be finite and >= 0");
    hw[(size_t)i] = (float)w[i];
  }
  std::vector<int> idx((size_t)count);
  std::iota(idx.begin(), idx.end(), 0);
  kb_context *ctx = f->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  if (param_flow(f)) {
    const int sg = param_grid(f, count);
    DevBuf dx, dw, di, dpart, dlp, dloss, dgrad;
    KB_CUDA(dx.alloc(hx.size() * sizeof(float), st));
    KB_CUDA(dw.alloc(hw.size() * sizeof(float), st));
    KB_CUDA(di.alloc(idx.size() * sizeof(int), st));
    KB_CUDA(dpart.alloc((size_t)sg * param_partial(f) * sizeof(double), st));
    KB_CUDA(dlp.alloc((size_t)sg * sizeof(double), st));
    KB_CUDA(dloss.alloc(sizeof(double), st));
    KB_CUDA(dgrad.alloc((size_t)kb_flow_num_params(f) * sizeof(float), st));
    KB_CUDA(cudaMemcpyAsync(dx.p, hx.data(), hx.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    KB_CUDA(cudaMemcpyAsync(dw.p, hw.data(), hw.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    KB_CUDA(cudaMemcpyAsync(di.p, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    KB_CUDA(param_grad(f, count, dx.as<float>(), dw.as<float>(), di.as<int>(), 1.0 / (double)count,
                       dpart.as<double>(), dlp.as<double>(), sg, st));
    KB_CUDA(param_adam(f, dpart.as<double>(), sg, dlp.as<double>(), dloss.as<double>(), dgrad.as<float>(), 0.0f, 0.0f,
                       0.0f, 1.0f, 1.0f, 1.0f, st));
    double lsum = 0.0;
    KB_CUDA(cudaMemcpyAsync(grad, dgrad.p, (size_t)kb_flow_num_params(f) * sizeof(float), cudaMemcpyDeviceToHost, st));
    KB_CUDA(cudaMemcpyAsync(&lsum, dloss.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    KB_CUDA(cudaStreamSynchronize(st));
    if (loss) *loss = lsum;
    return KB_OK;
  }
  const int grid = train_grid(f, count);
  DevBuf dx, dw, di, dpart, dloss, dxs, dgrad;
  KB_CUDA(dx.alloc(hx.size() * sizeof(float), st));
  KB_CUDA(dw.alloc(hw.size() * sizeof(float), st));
  KB_CUDA(di.alloc(idx.size() * sizeof(int), st));
  KB_CUDA(dpart.alloc((size_t)grid * FLOW_NPARAM * sizeof(float), st));
  KB_CUDA(dloss.alloc((size_t)grid * sizeof(float), st));
  KB_CUDA(dxs.alloc((size_t)count * FLOW_LAYERS * FLOW_MAX_DIM * sizeof(float), st));
  KB_CUDA(dgrad.alloc((size_t)FLOW_NPARAM * sizeof(float), st));
  KB_CUDA(cudaMemcpyAsync(dx.p, hx.data(), hx.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemcpyAsync(dw.p, hw.data(), hw.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemcpyAsync(di.p, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), st));
  int rc = train_pass(f, count, dx.as<float>(), dw.as<float>(), di.as<int>(), dpart.as<float>(), dloss.as<float>(),
                      dxs.as<float>(), grid);
  if (rc) return rc;
  KB_CUDA(launch_flow_reduce(dpart.as<float>(), grid, dgrad.as<float>(), st));
  std::vector<float> inr((size_t)FLOW_NPARAM), lp((size_t)grid);
  KB_CUDA(cudaMemcpyAsync(inr.data(), dgrad.p, inr.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
  KB_CUDA(cudaMemcpyAsync(lp.data(), dloss.p, lp.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
  rc = flow_error(ctx);
  if (rc) return rc;
  internal_to_api(inr.data(), grad);
  if (loss) {
    double s = 0.0;
    for (float v : lp) s += v;
    *loss = s;
  }
  return KB_OK;
}

int kb_flow_train(kb_flow *f, int64_t count, const double *x, const double *w, const kb_flow_train_cfg *cfg,
                  double *loss_hist, int *n_steps) {
  KB_CHECK(f && x && w && cfg, "kb_flow_train: null argument");
  KB_CHECK(count >= 1 && count <= (int64_t)1 << 26, "kb_flow_train: count must be in [1, 2^26]");
  KB_CHECK(cfg->epochs >= 1, "epochs must be >= 1");
  KB_CHECK(cfg->batch >= 1 && cfg->batch <= TRAIN_BATCH_MAX, "batch must be in [1, 65536]");
  KB_CHECK(cfg->lr > 0.0f && cfg->lr_final >= 0.0f && cfg->beta1 >= 0.0f && cfg->beta1 < 1.0f &&
               cfg->beta2 >= 0.0f && cfg->beta2 < 1.0f && cfg->eps > 0.0f,
           "invalid Adam settings");
  const int N = f->dim;
  std::vector<float> hx((size_t)count * N), hw((size_t)count);
  double wsum = 0.0;
  for (int64_t i = 0; i < count * N; ++i) {
    if (!(x[i] >= 0.0 && x[i] <= 1.0)) return fail(KB_E_INVALID, "flow inputs must lie in [0, 1]");
    hx[(size_t)i] = (float)x[i];
  }
  for (int64_t i = 0; i < count; ++i) {
    if (!(w[i] >= 0.0) || !std::isfinite(w[i])) return fail(KB_E_INVALID, "weights must be finite and >= 0");
    wsum += w[i];
  }
  if (!(wsum > 0.0)) return fail(KB_E_INVALID, "all weights are zero");
  for (int64_t i = 0; i < count; ++i) hw[(size_t)i] = (float)(w[i] * (double)count / wsum);
  const int64_t batch = std::min<int64_t>(cfg->batch, count);
  const int64_t per_epoch = std::max<int64_t>(1, count / batch);
  const int64_t steps = per_epoch * cfg->epochs;
  if (steps > (int64_t)1 << 24) return fail(KB_E_INVALID, "too many training steps");
  kb_context *ctx = f->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  if (param_flow(f)) return spline_train(f, count, hx, hw, cfg, batch, per_epoch, steps, loss_hist,
                                                               n_steps);
  const int grid = train_grid(f, batch);
  DevBuf dx, dw, di, dpart, dlp, dxs, dhist;
  KB_CUDA(dx.alloc(hx.size() * sizeof(float), st));
  KB_CUDA(dw.alloc(hw.size() * sizeof(float), st));
  KB_CUDA(di.alloc((size_t)count * sizeof(int), st));
  KB_CUDA(dpart.alloc((size_t)grid * FLOW_NPARAM * sizeof(float), st));
  KB_CUDA(dlp.alloc((size_t)grid * sizeof(float), st));
  KB_CUDA(dxs.alloc((size_t)batch * FLOW_LAYERS * FLOW_MAX_DIM * sizeof(float), st));
  KB_CUDA(dhist.alloc((size_t)steps * sizeof(float), st));
  KB_CUDA(cudaMemcpyAsync(dx.p, hx.data(), hx.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemcpyAsync(dw.p, hw.data(), hw.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  KB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), st));
  std::vector<int> perm((size_t)count);
  std::iota(perm.begin(), perm.end(), 0);
  std::mt19937_64 shuffler(cfg->seed);
  const double pi = 3.14159265358979323846;
  int64_t s = 0;
  for (int ep = 0; ep < cfg->epochs; ++ep) {
    std::shuffle(perm.begin(), perm.end(), shuffler);
    // the previous epoch's steps read the old order: wait before overwriting it
    KB_CUDA(cudaStreamSynchronize(st));
    KB_CUDA(cudaMemcpyAsync(di.p, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    for (int64_t b = 0; b < per_epoch; ++b, ++s) {
      int rc = train_pass(f, batch, dx.as<float>(), dw.as<float>(), di.as<int>() + b * batch, dpart.as<float>(),
                          dlp.as<float>(), dxs.as<float>(), grid);
      if (rc) return rc;
      const int64_t t = ++f->adam_step;
      const double lr = cfg->lr_final + 0.5 * (cfg->lr - cfg->lr_final) * (1.0 + std::cos(pi * (double)s / (double)steps));
      const float bc1 = (float)(1.0 - std::pow((double)cfg->beta1, (double)t));
      const float bc2 = (float)(1.0 - std::pow((double)cfg->beta2, (double)t));
      KB_CUDA(launch_flow_adam(f->master, f->adam_m, f->adam_v, f->img, dpart.as<float>(), grid, dlp.as<float>(),
                               dhist.as<float>() + s, (float)lr, cfg->beta1, cfg->beta2, cfg->eps, bc1, bc2, st));
    }
  }
  std::vector<float> hist((size_t)steps);
  KB_CUDA(cudaMemcpyAsync(hist.data(), dhist.p, hist.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
  int rc = flow_error(ctx);
  if (rc) return rc;
  if (loss_hist)
    for (int64_t i = 0; i < steps; ++i) loss_hist[i] = hist[(size_t)i];
  if (n_steps) *n_steps = (int)steps;
  return KB_OK;
}

int kb_flow_fit(kb_flow *f, const kb_model *m, const kb_integrand *fi, const kb_warper *chain, int chain_len,
                const kb_sobol *rng, uint32_t k_first, int64_t n_samples, const kb_flow_train_cfg *cfg,
                double *final_loss) {
  KB_CHECK(f && m && fi && rng && cfg, "kb_flow_fit: null argument");
  KB_CHECK(n_samples >= 1, "n_samples must be >= 1");
  KB_CHECK(rng->dim >= f->dim, "Sobol generator has fewer dimensions than the flow");
  const int N = f->dim;
  std::vector<double> li((size_t)n_samples * N), val((size_t)n_samples * 2), w((size_t)n_samples);
  int rc = kb_sobol_points(f->ctx, rng, k_first, n_samples, li.data());
  if (rc) return rc;
  rc = kb_evaluate_warped(f->ctx, m, fi, chain, chain_len, chain_len, N, n_samples, li.data(), 1, KB_ALGO_AUTO,
                          val.data(), nullptr, nullptr);
  if (rc) return rc;
  for (int64_t i = 0; i < n_samples; ++i) w[(size_t)i] = std::hypot(val[2 * i], val[2 * i + 1]);
  const int64_t steps = std::max<int64_t>(1, n_samples / std::min<int64_t>(cfg->batch, n_samples)) * cfg->epochs;
  std::vector<double> hist((size_t)std::max<int64_t>(steps, 1));
  int ns = 0;
  rc = kb_flow_train(f, n_samples, li.data(), w.data(), cfg, hist.data(), &ns);
  if (rc) return rc;
  if (final_loss) {
    const int64_t per_epoch = ns / cfg->epochs;
    double s = 0.0;
    for (int i = ns - (int)per_epoch; i < ns; ++i) s += hist[(size_t)i];
    *final_loss = per_epoch > 0 ? s / (double)per_epoch : 0.0;
  }
  return KB_OK;
}

} // extern "C"
