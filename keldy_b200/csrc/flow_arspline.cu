// Learned autoregressive spline warper (sm_100a), the third learned first stage of the
// warper chain (no keldy counterpart): a triangular (Knothe-Rosenblatt) map in which
// dimension d goes through the separable spline flow's monotone rational-quadratic CDF
// with parameters theta_d = A_d phi_d(x_0..x_{d-1}), a linear function of smooth features
// (Legendre polynomials of degree 1..3) of the coordinates before it. The density is
// q(x) = prod_d F_d'(x_d | x_<d) and stays smooth in every coordinate, so the map keeps what
// quasi-Monte Carlo needs while modelling how each vertex time depends on the earlier
// ones. With only the constant feature it is the separable spline flow, from which it is
// warm-started.
//
// Training: Adam on the weighted negative log-likelihood. Per sample and dimension the
// derivative of log F' with respect to theta_d (through the active bin's width, left knot,
// height and knot derivatives, then softmax, cumulative sums and softplus) times phi_d is
// the sample's contribution to d loss / d A_d; each CTA sums its tile's contributions
// with a small product in shared memory (no atomics: the sums are deterministic) and a
// second kernel adds the CTAs' partials in CTA order and takes the Adam step.
#include <cuda_runtime.h>
#include <math.h>

#include "kb_device.cuh"
#include "kb_flow.h"
#include "kb_spline.cuh"

namespace kb {

namespace {

constexpr double MW = SPL_MIN_BIN, MH = SPL_MIN_BIN;
constexpr int AR_TILE = 128; // samples per tile = threads per CTA of the gradient kernel

// DIR 1: z -> x = F^{-1}(z), out2 = dx/dz; DIR 0: x -> z = F(x), out2 = log q(x).
template <int DIR>
__global__ void ar_map_kernel(const float *params, int dim, long long count, const double *in, SobolDev rng,
                              uint32_t k_first, const uint32_t *k_first_dev, int use_sobol, double *out,
                              double *out2) {
  if (k_first_dev) k_first = *k_first_dev;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < count;
       p += (long long)gridDim.x * blockDim.x) {
    double x[FLOW_MAX_DIM];
    for (int d = 0; d < dim; ++d) x[d] = use_sobol ? sobol_coord(rng, k_first + (uint32_t)p, d) : in[p * dim + d];
    double acc;
    if (DIR == 1) {
      acc = ar_spline_point(params, dim, x, 1);
    } else {
      double phi[AR_MAX_FEAT], theta[SPL_PER_DIM];
      SplineKnots k;
      phi[0] = 1.0;
      acc = 0.0;
      double xin = 0.0;
      for (int d = 0; d < dim; ++d) {
        const double v = x[d];
        if (d > 0) ar_append_features(phi, d - 1, xin);
        xin = v; // the next dimension is conditioned on this input coordinate
        ar_theta(params + ar_offset(d), phi, ar_features(d), theta);
        spline_make_knots(theta, k);
        const int j = spline_find_bin(k.x, v);
        const double w = k.x[j + 1] - k.x[j], h = k.y[j + 1] - k.y[j], s = h / w;
        const double xi = fmin(fmax((v - k.x[j]) / w, 0.0), 1.0), e = xi * (1.0 - xi);
        const double d0 = k.d[j], d1 = k.d[j + 1];
        x[d] = k.y[j] + h * (s * xi * xi + d0 * e) / (s + (d1 + d0 - 2.0 * s) * e);
        acc += log(spline_deriv(k, j, xi));
      }
    }
    for (int d = 0; d < dim; ++d) out[p * dim + d] = x[d];
    out2[p] = acc;
  }
}

// One sample's d(-wn log F_d') / d theta_d into g[SPL_PER_DIM]; returns -wn log F_d'.
__device__ double ar_sample_grad(const double *theta, double v, double wn, double *g) {
  SplineKnots k;
  spline_make_knots(theta, k);
  const int j = spline_find_bin(k.x, v);
  const double wj = k.x[j + 1] - k.x[j], h = k.y[j + 1] - k.y[j], s = h / wj;
  const double xi = fmin(fmax((v - k.x[j]) / wj, 0.0), 1.0), e = xi * (1.0 - xi);
  const double d0 = k.d[j], d1 = k.d[j + 1];
  const double N = d1 * xi * xi + 2.0 * s * e + d0 * (1.0 - xi) * (1.0 - xi);
  const double D = s + (d1 + d0 - 2.0 * s) * e;
  // derivatives of log F' = 2 log s + log N - 2 log D
  const double ls = 2.0 / s + 2.0 * e / N - 2.0 * (1.0 - 2.0 * e) / D;
  const double ld0 = (1.0 - xi) * (1.0 - xi) / N - 2.0 * e / D;
  const double ld1 = xi * xi / N - 2.0 * e / D;
  const double lxi = (2.0 * d1 * xi + 2.0 * s * (1.0 - 2.0 * xi) - 2.0 * d0 * (1.0 - xi)) / N -
                     2.0 * (d1 + d0 - 2.0 * s) * (1.0 - 2.0 * xi) / D;
  // loss = -wn log F'; s = h / w, xi = (x - x_j) / w
  const double gh = -wn * ls / wj;
  const double gw = -wn * (ls * (-s / wj) + lxi * (-xi / wj));
  const double gx = -wn * lxi * (-1.0 / wj);
  // softmaxes of the width and height logits
  double mxa = -1e300, mxb = -1e300;
  for (int i = 0; i < SPL_BINS; ++i) {
    mxa = fmax(mxa, theta[i]);
    mxb = fmax(mxb, theta[SPL_BINS + i]);
  }
  double sa[SPL_BINS], sb[SPL_BINS], za = 0.0, zb = 0.0;
  for (int i = 0; i < SPL_BINS; ++i) {
    sa[i] = exp(theta[i] - mxa);
    sb[i] = exp(theta[SPL_BINS + i] - mxb);
    za += sa[i];
    zb += sb[i];
  }
  // widths: w_i enters bin j's width (i = j) and its left knot x_j (i < j)
  double dota = 0.0;
  for (int i = 0; i < SPL_BINS; ++i) {
    sa[i] /= za;
    sb[i] /= zb;
    dota += sa[i] * ((i == j ? gw : 0.0) + (i < j ? gx : 0.0));
  }
  const double dotb = sb[j] * gh;
  for (int i = 0; i < SPL_BINS; ++i) {
    g[i] = (1.0 - SPL_BINS * MW) * sa[i] * ((i == j ? gw : 0.0) + (i < j ? gx : 0.0) - dota);
    g[SPL_BINS + i] = (1.0 - SPL_BINS * MH) * sb[i] * ((i == j ? gh : 0.0) - dotb);
  }
  for (int q = 0; q <= SPL_BINS; ++q) {
    const double gd = q == j ? -wn * ld0 : (q == j + 1 ? -wn * ld1 : 0.0);
    g[2 * SPL_BINS + q] = gd / (1.0 + exp(-theta[2 * SPL_BINS + q])); // softplus' = sigmoid
  }
  return -wn * (2.0 * log(s) + log(N) - 2.0 * log(D));
}

// Per CTA: its tiles' sum_i wn_i (-log q(x_i)) and the derivatives with respect to every
// parameter; wn_i = w[index[i]] * inv_batch. partials [grid][ar_num_params(dim)],
// loss_part [grid]. Dynamic shared memory: ar_grad_smem_bytes(dim).
__global__ void __launch_bounds__(AR_TILE) ar_grad_kernel(const float *params, int dim, long long count,
                                                          const float *x, const float *w, const int *index,
                                                          double inv_batch, double *partials, double *loss_part) {
  extern __shared__ __align__(16) double ar_smem[];
  const int T = ar_num_params(dim);
  double *part = ar_smem;                   // [T]
  double *gt = part + T;                    // [AR_TILE][SPL_PER_DIM]
  double *ph = gt + AR_TILE * SPL_PER_DIM;  // [AR_TILE][AR_MAX_FEAT]
  __shared__ double sloss[AR_TILE];
  const int tid = threadIdx.x;
  for (int i = tid; i < T; i += AR_TILE) part[i] = 0.0;
  double lsum = 0.0;
  const long long ntiles = (count + AR_TILE - 1) / AR_TILE;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long p = tile * AR_TILE + tid;
    double xs[FLOW_MAX_DIM], wn = 0.0;
    if (p < count) {
      const long long src = index[p];
      wn = (double)w[src] * inv_batch;
      for (int d = 0; d < dim; ++d) xs[d] = (double)x[src * dim + d];
    }
    double phi[AR_MAX_FEAT], theta[SPL_PER_DIM];
    phi[0] = 1.0;
    for (int d = 0; d < dim; ++d) {
      if (d > 0) ar_append_features(phi, d - 1, p < count ? xs[d - 1] : 0.5);
      const int F = ar_features(d);
      double *g = gt + tid * SPL_PER_DIM;
      if (wn != 0.0) {
        ar_theta(params + ar_offset(d), phi, F, theta);
        lsum += ar_sample_grad(theta, xs[d], wn, g);
      } else {
        for (int q = 0; q < SPL_PER_DIM; ++q) g[q] = 0.0;
      }
      for (int f = 0; f < F; ++f) ph[tid * AR_MAX_FEAT + f] = phi[f];
      __syncthreads();
      // d loss / d A_d[q][f] += sum over the tile's samples of g[s][q] phi[s][f]
      double *pd = part + ar_offset(d);
      for (int e = tid; e < SPL_PER_DIM * F; e += AR_TILE) {
        const int q = e / F, f = e - q * F;
        double s = 0.0;
        for (int smp = 0; smp < AR_TILE; ++smp) s = fma(gt[smp * SPL_PER_DIM + q], ph[smp * AR_MAX_FEAT + f], s);
        pd[e] += s;
      }
      __syncthreads();
    }
  }
  sloss[tid] = lsum;
  __syncthreads();
  for (int i = tid; i < T; i += AR_TILE) partials[(size_t)blockIdx.x * T + i] = part[i];
  if (tid == 0) {
    double s = 0.0;
    for (int i = 0; i < AR_TILE; ++i) s += sloss[i];
    loss_part[blockIdx.x] = s;
  }
}

// The CTAs' partials summed in CTA order into grad_out (optional) and, with lr > 0, the
// Adam step on params; loss_out (optional) gets the loss.
__global__ void ar_adam_kernel(float *params, float *m, float *v, int T, const double *partials, int nparts,
                               const double *loss_part, double *loss_out, float *grad_out, float lr, float beta1,
                               float beta2, float eps, float bc1, float bc2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && loss_out) {
    double s = 0.0;
    for (int c = 0; c < nparts; ++c) s += loss_part[c];
    *loss_out = s;
  }
  if (i >= T) return;
  double g = 0.0;
  for (int c = 0; c < nparts; ++c) g += partials[(size_t)c * T + i];
  if (grad_out) grad_out[i] = (float)g;
  if (lr > 0.0f) {
    const float gi = (float)g;
    m[i] = beta1 * m[i] + (1.0f - beta1) * gi;
    v[i] = beta2 * v[i] + (1.0f - beta2) * gi * gi;
    params[i] -= lr * (m[i] / bc1) / (sqrtf(v[i] / bc2) + eps);
  }
}

} // namespace

size_t ar_grad_smem_bytes(int dim) {
  return sizeof(double) * ((size_t)ar_num_params(dim) + (size_t)AR_TILE * (SPL_PER_DIM + AR_MAX_FEAT));
}

cudaError_t ar_configure() {
  return cudaFuncSetAttribute(ar_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)ar_grad_smem_bytes(FLOW_MAX_DIM));
}

int ar_grad_grid(long long count, int sm_count) {
  const long long tiles = (count + AR_TILE - 1) / AR_TILE;
  return (int)(tiles < 2LL * sm_count ? (tiles > 0 ? tiles : 1) : 2LL * sm_count);
}

cudaError_t launch_ar_map(const float *params, int dim, int direction, long long count, const double *in,
                          SobolDev rng, uint32_t k_first, const uint32_t *k_first_dev, int use_sobol, double *out,
                          double *out2, int grid, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  const long long blocks = (count + 127) / 128;
  const int g = (int)(blocks < grid ? blocks : grid);
  if (direction == 0)
    ar_map_kernel<0><<<g, 128, 0, st>>>(params, dim, count, in, rng, k_first, k_first_dev, use_sobol, out, out2);
  else
    ar_map_kernel<1><<<g, 128, 0, st>>>(params, dim, count, in, rng, k_first, k_first_dev, use_sobol, out, out2);
  return cudaGetLastError();
}

cudaError_t launch_ar_grad(const float *params, int dim, long long count, const float *x, const float *w,
                           const int *index, double inv_batch, double *partials, double *loss_part, int grid,
                           cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  ar_grad_kernel<<<grid, AR_TILE, ar_grad_smem_bytes(dim), st>>>(params, dim, count, x, w, index, inv_batch, partials,
                                                                 loss_part);
  return cudaGetLastError();
}

cudaError_t launch_ar_adam(float *params, float *m, float *v, int dim, const double *partials, int nparts,
                           const double *loss_part, double *loss_out, float *grad_out, float lr, float beta1,
                           float beta2, float eps, float bc1, float bc2, cudaStream_t st) {
  const int T = ar_num_params(dim);
  ar_adam_kernel<<<(T + 255) / 256, 256, 0, st>>>(params, m, v, T, partials, nparts, loss_part, loss_out, grad_out, lr,
                                                  beta1, beta2, eps, bc1, bc2);
  return cudaGetLastError();
}

} // namespace kb
