// Learned separable spline warper (sm_100a), the second learned first stage of the warper
// chain (no keldy counterpart): per dimension d a monotone rational-quadratic spline CDF F_d
// on [0, 1] (Gregory & Delbourgo's rational-quadratic interpolant, in the parameterisation
// of Durkan et al., "Neural Spline Flows", 2019) with SPL_BINS bins. Its density is
// q(x) = prod_d F_d'(x_d); sampling maps the Sobol point z to x_d = F_d^{-1}(z_d) with
// dx/dz = 1 / q(x). The map is smooth (C^1 density) and acts on each axis alone, so it keeps
// the low-dimensional, nearly separable structure that quasi-Monte Carlo exploits, unlike
// the coupling layers' mixing of dimensions.
//
// Parameters per dimension (fp32, the flow's master array): SPL_BINS width logits a,
// SPL_BINS height logits b, SPL_BINS + 1 knot-derivative pre-activations c:
//   w_j = mw + (1 - K mw) softmax(a)_j, x_0 = 0, x_{j+1} = x_j + w_j (x_K = 1),
//   h_j = mh + (1 - K mh) softmax(b)_j, y likewise, delta_k = md + spline_softplus(c_k).
// In bin j with xi = (x - x_j)/w_j, s = h_j/w_j:
//   F(x) = y_j + h_j (s xi^2 + d0 xi (1 - xi)) / (s + (d1 + d0 - 2s) xi (1 - xi)),
//   F'(x) = s^2 (d1 xi^2 + 2 s xi (1 - xi) + d0 (1 - xi)^2) / (s + (d1 + d0 - 2s) xi (1 - xi))^2,
// d0 = delta_j, d1 = delta_{j+1}; the inverse solves the quadratic in xi.
// Training: Adam on the weighted negative log-likelihood sum_i w_i (-log q(x_i)), the
// gradient by hand: per sample the derivatives of log F' with respect to s, xi, d0, d1,
// chained to (w_j, x_j, h_j, delta_k) and summed per CTA in shared memory; one small
// kernel then chains those to the logits (softmax, cumulative sum, softplus) and takes the
// Adam step.
#include <cuda_runtime.h>
#include <math.h>

#include "kb_device.cuh"
#include "kb_flow.h"
#include "kb_spline.cuh"

namespace kb {

namespace {

constexpr double MW = SPL_MIN_BIN, MH = SPL_MIN_BIN;
// per-dimension gradient accumulators: dL/dw_j, dL/dx_j (bin j's left knot), dL/dh_j, dL/ddelta_k
constexpr int G_W = 0, G_X = SPL_BINS, G_H = 2 * SPL_BINS, G_D = 3 * SPL_BINS;
constexpr int G_PER_DIM = 4 * SPL_BINS + 1;

// Knots of every dimension (one thread per dimension), for the tree kernel's in-line map.
__global__ void spline_knots_kernel(const float *params, int dim, SplineKnots *knots) {
  const int d = threadIdx.x;
  if (d < dim) spline_make_knots(params + d * SPL_PER_DIM, knots[d]);
}

// DIR 1: z -> x = F^{-1}(z), out2 = dx/dz; DIR 0: x -> z = F(x), out2 = log q(x).
template <int DIR>
__global__ void spline_map_kernel(const float *params, int dim, long long count, const double *in, SobolDev rng,
                                  uint32_t k_first, const uint32_t *k_first_dev, int use_sobol, double *out,
                                  double *out2) {
  __shared__ SplineKnots K[FLOW_MAX_DIM];
  if (threadIdx.x < dim) spline_make_knots(params + threadIdx.x * SPL_PER_DIM, K[threadIdx.x]);
  __syncthreads();
  if (k_first_dev) k_first = *k_first_dev;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < count;
       p += (long long)gridDim.x * blockDim.x) {
    double acc = DIR == 0 ? 0.0 : 1.0;
    for (int d = 0; d < dim; ++d) {
      const SplineKnots &k = K[d];
      const double v = use_sobol ? sobol_coord(rng, k_first + (uint32_t)p, d) : in[p * dim + d];
      double r;
      if (DIR == 1) {
        double der;
        r = spline_inverse(k, v, der);
        acc /= der;
      } else {
        const int j = spline_find_bin(k.x, v);
        const double w = k.x[j + 1] - k.x[j], h = k.y[j + 1] - k.y[j], s = h / w;
        const double xi = fmin(fmax((v - k.x[j]) / w, 0.0), 1.0), e = xi * (1.0 - xi);
        const double d0 = k.d[j], d1 = k.d[j + 1];
        r = k.y[j] + h * (s * xi * xi + d0 * e) / (s + (d1 + d0 - 2.0 * s) * e);
        acc += log(spline_deriv(k, j, xi));
      }
      out[p * dim + d] = r;
    }
    out2[p] = acc;
  }
}

// Per CTA: sum_i wn_i (-log q(x_i)) and its derivatives with respect to every dimension's
// (w_j, x_j, h_j, delta_k); wn_i = w[index[i]] * inv_batch. partials [grid][dim * G_PER_DIM],
// loss_part [grid]. Samples in fp32 as the coupling flow's training takes them.
__global__ void spline_grad_kernel(const float *params, int dim, long long count, const float *x, const float *w,
                                   const int *index, double inv_batch, double *partials, double *loss_part) {
  __shared__ SplineKnots K[FLOW_MAX_DIM];
  __shared__ double G[FLOW_MAX_DIM * G_PER_DIM];
  __shared__ double sloss;
  for (int i = threadIdx.x; i < dim * G_PER_DIM; i += blockDim.x) G[i] = 0.0;
  if (threadIdx.x == 0) sloss = 0.0;
  if (threadIdx.x < dim) spline_make_knots(params + threadIdx.x * SPL_PER_DIM, K[threadIdx.x]);
  __syncthreads();
  double lsum = 0.0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < count;
       p += (long long)gridDim.x * blockDim.x) {
    const long long src = index[p];
    const double wn = (double)w[src] * inv_batch;
    if (wn == 0.0) continue;
    for (int d = 0; d < dim; ++d) {
      const SplineKnots &k = K[d];
      const double v = (double)x[src * dim + d];
      const int j = spline_find_bin(k.x, v);
      const double wj = k.x[j + 1] - k.x[j], h = k.y[j + 1] - k.y[j], s = h / wj;
      const double xi = fmin(fmax((v - k.x[j]) / wj, 0.0), 1.0), e = xi * (1.0 - xi);
      const double d0 = k.d[j], d1 = k.d[j + 1];
      const double N = d1 * xi * xi + 2.0 * s * e + d0 * (1.0 - xi) * (1.0 - xi);
      const double D = s + (d1 + d0 - 2.0 * s) * e;
      lsum -= wn * (2.0 * log(s) + log(N) - 2.0 * log(D));
      // derivatives of log F' = 2 log s + log N - 2 log D
      const double ls = 2.0 / s + 2.0 * e / N - 2.0 * (1.0 - 2.0 * e) / D;
      const double ld0 = (1.0 - xi) * (1.0 - xi) / N - 2.0 * e / D;
      const double ld1 = xi * xi / N - 2.0 * e / D;
      const double lxi = (2.0 * d1 * xi + 2.0 * s * (1.0 - 2.0 * xi) - 2.0 * d0 * (1.0 - xi)) / N -
                         2.0 * (d1 + d0 - 2.0 * s) * (1.0 - 2.0 * xi) / D;
      double *g = G + d * G_PER_DIM;
      // loss = -wn log F'; s = h / w, xi = (x - x_j) / w
      atomicAdd(&g[G_H + j], -wn * ls / wj);
      atomicAdd(&g[G_W + j], -wn * (ls * (-s / wj) + lxi * (-xi / wj)));
      atomicAdd(&g[G_X + j], -wn * lxi * (-1.0 / wj));
      atomicAdd(&g[G_D + j], -wn * ld0);
      atomicAdd(&g[G_D + j + 1], -wn * ld1);
    }
  }
  atomicAdd(&sloss, lsum);
  __syncthreads();
  for (int i = threadIdx.x; i < dim * G_PER_DIM; i += blockDim.x)
    partials[(size_t)blockIdx.x * dim * G_PER_DIM + i] = G[i];
  if (threadIdx.x == 0) loss_part[blockIdx.x] = sloss;
}

// The CTAs' partials summed in CTA order, chained to the logits, into grad[dim][SPL_PER_DIM]
// (one thread per dimension); with lr > 0 also the Adam step on params (m, v moments).
__global__ void spline_adam_kernel(float *params, float *m, float *v, int dim, const double *partials, int nparts,
                                   const double *loss_part, double *loss_out, float *grad_out, float lr, float beta1,
                                   float beta2, float eps, float bc1, float bc2) {
  const int d = threadIdx.x;
  if (d == 0 && loss_out) {
    double s = 0.0;
    for (int c = 0; c < nparts; ++c) s += loss_part[c];
    *loss_out = s;
  }
  if (d >= dim) return;
  double g[G_PER_DIM];
  for (int i = 0; i < G_PER_DIM; ++i) g[i] = 0.0;
  for (int c = 0; c < nparts; ++c)
    for (int i = 0; i < G_PER_DIM; ++i) g[i] += partials[((size_t)c * dim + d) * G_PER_DIM + i];
  float *p = params + d * SPL_PER_DIM;
  double gp[SPL_PER_DIM];
  // widths: dL/dw_j plus the knots x_k = sum_{i<k} w_i to the right of bin j (k = j+1 .. K-1)
  double gw[SPL_BINS], sa[SPL_BINS], sb[SPL_BINS];
  double tail = 0.0;
  for (int j = SPL_BINS - 1; j >= 0; --j) {
    gw[j] = g[G_W + j] + tail;
    tail += g[G_X + j];
  }
  double mxa = -1e300, mxb = -1e300, za = 0.0, zb = 0.0;
  for (int j = 0; j < SPL_BINS; ++j) {
    mxa = fmax(mxa, (double)p[j]);
    mxb = fmax(mxb, (double)p[SPL_BINS + j]);
  }
  for (int j = 0; j < SPL_BINS; ++j) {
    sa[j] = exp((double)p[j] - mxa);
    sb[j] = exp((double)p[SPL_BINS + j] - mxb);
    za += sa[j];
    zb += sb[j];
  }
  double dota = 0.0, dotb = 0.0;
  for (int j = 0; j < SPL_BINS; ++j) {
    sa[j] /= za;
    sb[j] /= zb;
    dota += sa[j] * gw[j];
    dotb += sb[j] * g[G_H + j];
  }
  for (int j = 0; j < SPL_BINS; ++j) {
    gp[j] = (1.0 - SPL_BINS * MW) * sa[j] * (gw[j] - dota);
    gp[SPL_BINS + j] = (1.0 - SPL_BINS * MH) * sb[j] * (g[G_H + j] - dotb);
  }
  for (int k = 0; k <= SPL_BINS; ++k) {
    const double c = (double)p[2 * SPL_BINS + k];
    gp[2 * SPL_BINS + k] = g[G_D + k] / (1.0 + exp(-c)); // softplus' = sigmoid
  }
  for (int i = 0; i < SPL_PER_DIM; ++i) {
    if (grad_out) grad_out[d * SPL_PER_DIM + i] = (float)gp[i];
    if (lr > 0.0f) {
      const int q = d * SPL_PER_DIM + i;
      const float gi = (float)gp[i];
      m[q] = beta1 * m[q] + (1.0f - beta1) * gi;
      v[q] = beta2 * v[q] + (1.0f - beta2) * gi * gi;
      p[i] -= lr * (m[q] / bc1) / (sqrtf(v[q] / bc2) + eps);
    }
  }
}

} // namespace

cudaError_t launch_spline_map(const float *params, int dim, int direction, long long count, const double *in,
                              SobolDev rng, uint32_t k_first, const uint32_t *k_first_dev, int use_sobol, double *out,
                              double *out2, int grid, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  const long long blocks = (count + 127) / 128;
  const int g = (int)(blocks < grid ? blocks : grid);
  if (direction == 0)
    spline_map_kernel<0><<<g, 128, 0, st>>>(params, dim, count, in, rng, k_first, k_first_dev, use_sobol, out, out2);
  else
    spline_map_kernel<1><<<g, 128, 0, st>>>(params, dim, count, in, rng, k_first, k_first_dev, use_sobol, out, out2);
  return cudaGetLastError();
}

cudaError_t launch_spline_knots(const float *params, int dim, double *knots, cudaStream_t st) {
  spline_knots_kernel<<<1, 32, 0, st>>>(params, dim, reinterpret_cast<SplineKnots *>(knots));
  return cudaGetLastError();
}

int spline_grad_per_dim() { return G_PER_DIM; }

cudaError_t launch_spline_grad(const float *params, int dim, long long count, const float *x, const float *w,
                               const int *index, double inv_batch, double *partials, double *loss_part, int grid,
                               cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  spline_grad_kernel<<<grid, 256, 0, st>>>(params, dim, count, x, w, index, inv_batch, partials, loss_part);
  return cudaGetLastError();
}

cudaError_t launch_spline_adam(float *params, float *m, float *v, int dim, const double *partials, int nparts,
                               const double *loss_part, double *loss_out, float *grad_out, float lr, float beta1,
                               float beta2, float eps, float bc1, float bc2, cudaStream_t st) {
  spline_adam_kernel<<<1, 32, 0, st>>>(params, m, v, dim, partials, nparts, loss_part, loss_out, grad_out, lr, beta1,
                                       beta2, eps, bc1, bc2);
  return cudaGetLastError();
}

} // namespace kb
