// C ABI of the tabulated product warpers (kb_warper_table_*, include/keldy_b200.h):
// keldy's warper_product_1d_simple_interp_nearest_t tables (integrate_and_inverse,
// product_1d_simple.hpp:219-253) and make_warper_from_proj (make_warper_from_proj.hpp),
// built on the host; the warper chain evaluates them on the device (kb_device.cuh).
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "kb_host.h"

using namespace kb;

namespace {

// One table from points u (u[0] = 0, increasing) and f1 values: F, fm, cut, as keldy's
// integrate_and_inverse: F[n-1] = 0, F[i] = F[i+1] - (f1[i+1] + f1[i]) / 2 (u[i+1] - u[i]),
// normalised by -F[0] (F[0] then set to -1 exactly); the inverse runs on F[0..cut].
int build_table(const double *u, const double *f1, int n, std::vector<double> &F, std::vector<double> &fm,
                int &cut) {
  if (n < 3) return fail(KB_E_INVALID, "Expect nr_sample_points to be >= 3. Given was " + std::to_string(n));
  if (u[0] != 0.0) return fail(KB_E_INVALID, "times_u_pts should start at 0");
  for (int i = 0; i < n; ++i) {
    if (!std::isfinite(u[i]) || !std::isfinite(f1[i])) return fail(KB_E_INVALID, "warper table values must be finite");
    if (i > 0 && !(u[i] > u[i - 1])) return fail(KB_E_INVALID, "times_u_pts must be strictly increasing");
  }
  F.assign((size_t)n, 0.0);
  std::vector<double> f((size_t)n);
  for (int i = 0; i < n; ++i) f[(size_t)i] = f1[i];
  cut = n - 1;
  bool found = false;
  for (int i = n - 2; i >= 0; --i) {
    F[(size_t)i] = F[(size_t)i + 1] - 0.5 * (f[(size_t)i + 1] + f[(size_t)i]) * (u[i + 1] - u[i]);
    found = found || (F[(size_t)i] != 0);
    if (!found) cut = i;
  }
  if (!found) return fail(KB_E_INVALID, "Model function is flat zero.");
  const double norm = -F[0];
  for (auto &v : F) v /= norm;
  for (auto &v : f) v /= norm;
  F[0] = -1;
  for (int i = 0; i < cut; ++i)
    if (!(F[(size_t)i + 1] > F[(size_t)i]))
      return fail(KB_E_INVALID, "the integral of f1 is not strictly increasing on the warper's support "
                                "(f1 must be > 0 there)");
  fm.assign((size_t)n - 1, 0.0);
  for (int i = 0; i + 1 < n; ++i) fm[(size_t)i] = 0.5 * (f[(size_t)i] + f[(size_t)i + 1]);
  return KB_OK;
}

// Weighted least-squares line y = c0 + c1 x over the points with weight > 0; y_out at x0.
double wlinear_at(const double *x, const double *y, const double *w, int n, double x0) {
  double W = 0.0, mx = 0.0, my = 0.0;
  for (int i = 0; i < n; ++i)
    if (w[i] > 0.0) {
      W += w[i];
      mx += w[i] * x[i];
      my += w[i] * y[i];
    }
  mx /= W;
  my /= W;
  double sxx = 0.0, sxy = 0.0;
  for (int i = 0; i < n; ++i)
    if (w[i] > 0.0) {
      const double dx = x[i] - mx;
      sxx += w[i] * dx * dx;
      sxy += w[i] * dx * (y[i] - my);
    }
  const double c1 = sxy / sxx;
  return (my - mx * c1) + x0 * c1;
}

// kernel_smoothing (make_warper_from_proj.hpp:40-66): exp of a local linear fit of log y
// at every bin, Gaussian weights exp(-((j - H) / sigma)^2 / 2) on the bins i - H .. i + H
// (H = max(min(3 sigma, N), 1)), the bins with y <= 0 left out.
std::vector<double> kernel_smoothing(const std::vector<double> &y, double sigma) {
  const int N = (int)y.size();
  const int H = std::max(std::min((int)(3 * sigma), N), 1);
  const int K = 2 * H + 1;
  std::vector<double> ker((size_t)K), logy((size_t)N), x((size_t)N), out((size_t)N);
  for (int j = 0; j < K; ++j) ker[(size_t)j] = std::exp(-std::pow((j - H) / sigma, 2) / 2);
  for (int i = 0; i < N; ++i) {
    x[(size_t)i] = i;
    logy[(size_t)i] = std::log(y[(size_t)i]);
  }
  std::vector<double> w((size_t)K);
  for (int i = 0; i < N; ++i) {
    const int start_ker = std::max(0, H - i);
    const int end_ker = std::min(N + H - i - 1, K - 1);
    const int size = end_ker - start_ker + 1;
    const int start_x = start_ker - H + i;
    for (int j = 0; j < size; ++j) {
      const int xi = start_x + j;
      w[(size_t)j] = (y[(size_t)xi] <= 0.0) ? 0.0 : ker[(size_t)(start_ker + j)];
    }
    out[(size_t)i] = std::exp(wlinear_at(x.data() + start_x, logy.data() + start_x, w.data(), size, x[(size_t)i]));
  }
  return out;
}

} // namespace

extern "C" {

int kb_warper_table_create(kb_context *ctx, int ndims, const int *npts, const double *u_pts, const double *f1_pts,
                           kb_warper_table **out) {
  KB_CHECK(ctx && npts && u_pts && f1_pts && out, "kb_warper_table_create: null argument");
  KB_CHECK(ndims >= 1 && ndims <= MAX_ORDER, "a tabulated warper has 1 to 16 tables");
  std::vector<std::vector<double>> Fs((size_t)ndims), fms((size_t)ndims);
  std::vector<int> cuts((size_t)ndims);
  size_t off = 0, total = 0;
  for (int d = 0; d < ndims; ++d) {
    int st = build_table(u_pts + off, f1_pts + off, npts[d], Fs[(size_t)d], fms[(size_t)d], cuts[(size_t)d]);
    if (st) return st;
    off += (size_t)npts[d];
    total += 3 * (size_t)npts[d] - 1;
  }
  std::vector<double> host(total);
  std::vector<size_t> base((size_t)ndims);
  off = 0;
  size_t pos = 0;
  for (int d = 0; d < ndims; ++d) {
    const int n = npts[d];
    base[(size_t)d] = pos;
    std::copy(u_pts + off, u_pts + off + n, host.begin() + (long)pos);
    std::copy(Fs[(size_t)d].begin(), Fs[(size_t)d].end(), host.begin() + (long)pos + n);
    std::copy(fms[(size_t)d].begin(), fms[(size_t)d].end(), host.begin() + (long)pos + 2 * n);
    pos += 3 * (size_t)n - 1;
    off += (size_t)n;
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  KB_CUDA(cudaSetDevice(ctx->device));
  auto *t = new kb_warper_table;
  t->ctx = ctx;
  t->device = ctx->device;
  t->ndims = ndims;
  t->u_max = u_pts[npts[0] - 1];
  cudaError_t e = cudaMalloc(&t->d_data, total * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&t->d_dims, (size_t)ndims * sizeof(TableDimDev));
  std::vector<TableDimDev> dims((size_t)ndims);
  if (e == cudaSuccess) {
    for (int d = 0; d < ndims; ++d) {
      const int n = npts[d];
      dims[(size_t)d].u = t->d_data + base[(size_t)d];
      dims[(size_t)d].F = t->d_data + base[(size_t)d] + n;
      dims[(size_t)d].fm = t->d_data + base[(size_t)d] + 2 * n;
      dims[(size_t)d].n = n;
      dims[(size_t)d].cut = cuts[(size_t)d];
    }
    e = cudaMemcpy(t->d_data, host.data(), total * sizeof(double), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMemcpy(t->d_dims, dims.data(), dims.size() * sizeof(TableDimDev), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(t->d_data);
    cudaFree(t->d_dims);
    delete t;
    return fail(KB_E_CUDA, std::string("kb_warper_table_create: ") + cudaGetErrorString(e));
  }
  *out = t;
  return KB_OK;
}

int kb_warper_table_destroy(kb_warper_table *t) {
  if (!t) return KB_OK;
  cudaSetDevice(t->device);
  cudaFree(t->d_data);
  cudaFree(t->d_dims);
  delete t;
  return KB_OK;
}

int kb_warper_table_from_projection(kb_context *ctx, const kb_model *m, const kb_integrand *f,
                                    const kb_warper *chain, int chain_len, int order, int num_bins, int nr_samples,
                                    double sigma, int keep_u_hypercube, kb_warper_table **out) {
  KB_CHECK(ctx && m && f && out, "kb_warper_table_from_projection: null argument");
  KB_CHECK(order >= 1 && order <= MAX_ORDER, "order must be in [1, 16]");
  KB_CHECK(num_bins >= 2 && nr_samples >= 1 && sigma > 0.0, "need num_bins >= 2, nr_samples >= 1, sigma > 0");
  kb_sobol *g = nullptr;
  int st = kb_sobol_create(ctx, order, 31, 0, 0, 0, &g);
  if (st) return st;
  std::vector<double> li((size_t)nr_samples * order), val(2 * (size_t)nr_samples);
  st = kb_sobol_points(ctx, g, 1, nr_samples, li.data());
  kb_sobol_destroy(g);
  if (st) return st;
  st = kb_evaluate_warped(ctx, m, f, chain, chain_len, chain_len, order, nr_samples, li.data(), keep_u_hypercube,
                          KB_ALGO_AUTO, val.data(), nullptr, nullptr);
  if (st) return st;
  // gather_data (make_warper_from_proj.hpp:68-98): per axis, the mean |f J| of each bin
  const double bin_size = 1.0 / num_bins;
  std::vector<double> tu((size_t)num_bins + 1), f1all, uall;
  for (int i = 0; i <= num_bins; ++i) tu[(size_t)i] = i * bin_size;
  tu[(size_t)num_bins] = 1.0;
  std::vector<int> npts((size_t)order, num_bins + 1);
  for (int axis = 0; axis < order; ++axis) {
    std::vector<double> sum((size_t)num_bins, 0.0);
    std::vector<long> cnt((size_t)num_bins, 0);
    for (int p = 0; p < nr_samples; ++p) {
      const double x = li[(size_t)p * order + axis];
      if (!(0.0 <= x && x <= 1.0)) continue;
      const int b = (x == 1.0) ? num_bins - 1 : std::min((int)((x - 0.0) / bin_size), num_bins - 1);
      sum[(size_t)b] += std::hypot(val[2 * (size_t)p], val[2 * (size_t)p + 1]);
      cnt[(size_t)b]++;
    }
    for (int b = 0; b < num_bins; ++b)
      if (cnt[(size_t)b] > 0) sum[(size_t)b] /= (double)cnt[(size_t)b];
    const std::vector<double> sm = kernel_smoothing(sum, sigma / bin_size);
    std::vector<double> f1((size_t)num_bins + 1);
    f1[0] = 0;
    for (int i = 0; i < num_bins; ++i) f1[(size_t)i + 1] = 2 * sm[(size_t)i] - f1[(size_t)i];
    f1all.insert(f1all.end(), f1.begin(), f1.end());
    uall.insert(uall.end(), tu.begin(), tu.end());
  }
  return kb_warper_table_create(ctx, order, npts.data(), uall.data(), f1all.data(), out);
}

} // extern "C"
