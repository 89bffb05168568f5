// The separable spline flow's per-dimension knots and its sampling map z -> x = F^{-1}(z),
// shared by the flow's own map kernel (flow_spline.cu) and the tree kernel's point set-up,
// which applies the flow in line when a work item carries one (so both give bit-identical
// points and Jacobians). The spline is Gregory & Delbourgo's monotone rational-quadratic
// interpolant in the parameterisation of Durkan et al., "Neural Spline Flows" (2019).
#pragma once

#include <math.h>

#include "kb_flow.h"

namespace kb {

// Knots of one dimension: bin edges x (inputs), y (outputs), derivatives d at the edges.
struct SplineKnots {
  double x[SPL_BINS + 1], y[SPL_BINS + 1], d[SPL_BINS + 1];
};
static_assert(sizeof(SplineKnots) == SPL_KNOT_DOUBLES * sizeof(double), "knots layout");

__device__ __forceinline__ double spline_softplus(double v) { return v > 30.0 ? v : log1p(exp(v)); }

// Knots of one dimension from its SPL_PER_DIM parameters (width logits, height logits,
// knot-derivative pre-activations): the flow's fp32 parameters, or the autoregressive
// flow's fp64 conditioner output.
template <typename T>
__device__ inline void spline_make_knots(const T *p, SplineKnots &k) {
  constexpr double MW = SPL_MIN_BIN, MH = SPL_MIN_BIN, MD = SPL_MIN_DERIV;
  double mxa = -1e300, mxb = -1e300;
  for (int j = 0; j < SPL_BINS; ++j) {
    mxa = fmax(mxa, (double)p[j]);
    mxb = fmax(mxb, (double)p[SPL_BINS + j]);
  }
  double ea[SPL_BINS], eb[SPL_BINS], sa = 0.0, sb = 0.0;
  for (int j = 0; j < SPL_BINS; ++j) {
    ea[j] = exp((double)p[j] - mxa);
    eb[j] = exp((double)p[SPL_BINS + j] - mxb);
    sa += ea[j];
    sb += eb[j];
  }
  k.x[0] = k.y[0] = 0.0;
  for (int j = 0; j < SPL_BINS; ++j) {
    k.x[j + 1] = k.x[j] + (MW + (1.0 - SPL_BINS * MW) * ea[j] / sa);
    k.y[j + 1] = k.y[j] + (MH + (1.0 - SPL_BINS * MH) * eb[j] / sb);
  }
  k.x[SPL_BINS] = k.y[SPL_BINS] = 1.0;
  for (int j = 0; j <= SPL_BINS; ++j) k.d[j] = MD + spline_softplus((double)p[2 * SPL_BINS + j]);
}

// Bin of v among the edges e[0..SPL_BINS] (the last bin takes v >= e[SPL_BINS - 1]).
__device__ __forceinline__ int spline_find_bin(const double *e, double v) {
  int j = 0;
#pragma unroll
  for (int q = 1; q < SPL_BINS; ++q) j += (v >= e[q]) ? 1 : 0;
  return j;
}

// F'(x) of bin j at xi = (x - x_j) / w_j.
__device__ __forceinline__ double spline_deriv(const SplineKnots &k, int j, double xi) {
  const double w = k.x[j + 1] - k.x[j], h = k.y[j + 1] - k.y[j], s = h / w;
  const double d0 = k.d[j], d1 = k.d[j + 1], e = xi * (1.0 - xi);
  const double den = s + (d1 + d0 - 2.0 * s) * e;
  return s * s * (d1 * xi * xi + 2.0 * s * e + d0 * (1.0 - xi) * (1.0 - xi)) / (den * den);
}

// Sampling direction: x = F^{-1}(v) (the root of the bin's quadratic in xi that lies in
// [0, 1], in the cancellation-free form), and F'(x) into `deriv` (dx/dv = 1 / F'(x)).
__device__ __forceinline__ double spline_inverse(const SplineKnots &k, double v, double &deriv) {
  const int j = spline_find_bin(k.y, v);
  const double w = k.x[j + 1] - k.x[j], h = k.y[j + 1] - k.y[j], s = h / w;
  const double d0 = k.d[j], d1 = k.d[j + 1], t = v - k.y[j], g = d1 + d0 - 2.0 * s;
  const double qa = h * (s - d0) + t * g, qb = h * d0 - t * g, qc = -s * t;
  const double disc = fmax(qb * qb - 4.0 * qa * qc, 0.0);
  double xi = (2.0 * qc) / (-qb - sqrt(disc));
  xi = fmin(fmax(xi, 0.0), 1.0);
  deriv = spline_deriv(k, j, xi);
  return fmin(fmax(k.x[j] + xi * w, 0.0), 1.0);
}

// ---- the autoregressive (Knothe-Rosenblatt) spline flow: dimension d's SPL_PER_DIM
// parameters are theta_d = A_d phi_d, phi_d = [1, P1(x_k), P2(x_k), P3(x_k) for k < d]
// (Legendre polynomials on [0, 1]); A_d is [SPL_PER_DIM][ar_features(d)] row-major and the
// flow's parameters hold A_0, A_1, ... in order.
constexpr int AR_NFEAT = 3;
constexpr int AR_MAX_FEAT = 1 + AR_NFEAT * (FLOW_MAX_DIM - 1);
__host__ __device__ inline int ar_features(int d) { return 1 + AR_NFEAT * d; }
__host__ __device__ inline int ar_offset(int d) { return SPL_PER_DIM * (d + AR_NFEAT * d * (d - 1) / 2); }
__host__ __device__ inline int ar_num_params(int dim) { return ar_offset(dim); }

// Appends coordinate x_k's features to phi (phi[1 + 3k .. 3 + 3k]).
__device__ __forceinline__ void ar_append_features(double *phi, int k, double xk) {
  const double u = 2.0 * xk - 1.0;
  phi[1 + AR_NFEAT * k] = u;
  phi[2 + AR_NFEAT * k] = 1.5 * u * u - 0.5;
  phi[3 + AR_NFEAT * k] = (2.5 * u * u - 1.5) * u;
}

// theta = A phi, A [SPL_PER_DIM][F] (fp32), sums over the features in order.
__device__ __forceinline__ void ar_theta(const float *A, const double *phi, int F, double *theta) {
  for (int q = 0; q < SPL_PER_DIM; ++q) {
    double s = 0.0;
    for (int f = 0; f < F; ++f) s = fma((double)A[q * F + f], phi[f], s);
    theta[q] = s;
  }
}

// Sampling direction of the autoregressive flow on one point: x (stride st) holds the
// Sobol coordinates z on entry and x = F^{-1}(z) on return, dimension by dimension (each
// conditioned on the ones before); returns dx/dz = prod_d 1 / F_d'(x_d).
static __device__ __noinline__ double ar_spline_point(const float *params, int N, double *x, int st) {
  double phi[AR_MAX_FEAT], theta[SPL_PER_DIM];
  SplineKnots k;
  phi[0] = 1.0;
  double jac = 1.0;
  for (int d = 0; d < N; ++d) {
    if (d > 0) ar_append_features(phi, d - 1, x[(d - 1) * st]);
    ar_theta(params + ar_offset(d), phi, ar_features(d), theta);
    spline_make_knots(theta, k);
    double der;
    x[d * st] = spline_inverse(k, x[d * st], der);
    jac /= der;
  }
  return jac;
}

} // namespace kb
