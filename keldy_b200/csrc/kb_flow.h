// Learned coupling-flow warper: device descriptors and kernel launchers (flow.cu).
//
// The flow maps the Sobol point z in [0,1]^n (n = 2..8) to the input li of the plain
// warper chain; the integrand is then f(chain(li)) * J_chain(li) * J_flow(z). Six
// coupling layers; layer l redraws the dims T_l (bit (l/2) % ceil(log2 n) of the dim
// index equal to l % 2) through piecewise-linear CDFs of 32 bins whose logits come
// from an MLP (128 hat features -> 128 -> 128 -> 4 x 32 logits, ReLU, bf16 weights,
// fp32 accumulation on the tensor cores) of the other dims. Biases are folded into the
// matrices: input feature 16*T_l[0] and hidden unit 127 are constant 1.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kb_types.h"

namespace kb {

constexpr int FLOW_LAYERS = 6;
constexpr int FLOW_W = 128;      // features = hidden units = logits per layer
constexpr int FLOW_BLOB = 16;    // hat features per conditioning dim
constexpr int FLOW_BINS = 32;    // bins of each piecewise-linear CDF
constexpr int FLOW_SLOTS = 4;    // transformed dims per layer (at most)
constexpr int FLOW_MAX_DIM = 8;
constexpr int FLOW_CONST = 127;  // hidden unit fixed to 1 (bias carrier)
constexpr float FLOW_EPS = 0.01f; // uniform share mixed into every bin distribution
constexpr int FLOW_MAT = FLOW_W * FLOW_W;
constexpr int FLOW_NMAT = 3 * FLOW_LAYERS;
constexpr int FLOW_NPARAM = FLOW_NMAT * FLOW_MAT;
constexpr int FLOW_TILE = 128;   // points per CTA tile (one TMEM lane each)

// Element (r, k) of a 128x128 bf16 matrix in the tensor-core image layout: 8x8 core
// matrices (8 rows of 16 bytes), K-adjacent core matrices 128 bytes apart, 8-row groups
// 2048 bytes apart. The same bytes are a K-major operand with rows r and an MN-major
// operand with rows k.
__host__ __device__ inline int flow_img_index(int r, int k) {
  return (r >> 3) * 1024 + (k >> 3) * 64 + (r & 7) * 8 + (k & 7);
}

// The separable spline flow (flow_spline.cu): per dimension a rational-quadratic spline CDF
// of SPL_BINS bins, SPL_PER_DIM parameters (width logits, height logits, knot-derivative
// pre-activations); bins at least SPL_MIN_BIN wide and high, knot derivatives at least
// SPL_MIN_DERIV.
constexpr int FLOW_KIND_COUPLING = 0;
constexpr int FLOW_KIND_SPLINE = 1;
constexpr int FLOW_KIND_AR_SPLINE = 2; // autoregressive spline flow (flow_arspline.cu)
constexpr int SPL_BINS = 16;
constexpr int SPL_PER_DIM = 3 * SPL_BINS + 1;
constexpr double SPL_MIN_BIN = 1e-3;
constexpr double SPL_MIN_DERIV = 1e-3;
constexpr int SPL_KNOT_DOUBLES = 3 * (SPL_BINS + 1); // x, y and derivative at each bin edge

struct FlowDev {
  int kind;            // FLOW_KIND_*
  const float *spline; // FLOW_KIND_SPLINE: [dim][SPL_PER_DIM] parameters
  double *knots;       // FLOW_KIND_SPLINE: [dim][SPL_KNOT_DOUBLES] knots made from them (launch_spline_knots)
  const uint16_t *img; // [FLOW_NMAT][FLOW_MAT] bf16 bit patterns, image layout
  int dim;
  int ntr[FLOW_LAYERS];              // number of transformed dims
  int tdim[FLOW_LAYERS][FLOW_SLOTS]; // transformed dims in slot order (-1: unused)
  unsigned tmask[FLOW_LAYERS];       // bit i set: dim i transformed
};

void flow_layout(int dim, FlowDev &f);
size_t flow_map_smem_bytes();
size_t flow_train_smem_bytes();
cudaError_t flow_configure();

// direction 0: x -> z with log q(x) in out2; direction 1: z -> x with dx/dz in out2.
// Inputs from `in` ([count][dim]) or, with use_sobol, Sobol points k_first.. of rng
// (k_first read from k_first_dev when that is not null: graph-captured launches). grid:
// the SM count (the coupling flow runs two CTAs per SM).
cudaError_t launch_flow_map(const FlowDev &f, int direction, long long count, const double *in, SobolDev rng,
                            uint32_t k_first, const uint32_t *k_first_dev, int use_sobol, double *out, double *out2,
                            int *err, int grid, cudaStream_t st);
// Loss and gradient partials of one batch: point p of the batch is index[p] of x/w
// (x: [*][dim] float, w: weights). partials [grid][FLOW_NPARAM] in the internal order
// [matrix][in][out]; loss_part[grid] = sum w (-log q) * inv_batch; xs: 48 floats per point.
cudaError_t launch_flow_train(const FlowDev &f, long long count, const float *x, const float *w, const int *index,
                              float inv_batch, float *partials, float *loss_part, float *xs, int *err, int grid,
                              cudaStream_t st);
// Sum of the partials (grid rows) into grad [FLOW_NPARAM] (internal order).
cudaError_t launch_flow_reduce(const float *partials, int nparts, float *grad, cudaStream_t st);
// Adam step on the fp32 master weights (internal order) from the summed partials; writes
// the bf16 images; block 0 stores sum(loss_part) into *loss_out.
cudaError_t launch_flow_adam(float *master, float *m, float *v, uint16_t *img, const float *partials, int nparts,
                             const float *loss_part, float *loss_out, float lr, float beta1, float beta2, float eps,
                             float bc1, float bc2, cudaStream_t st);
// bf16 images from the fp32 master weights.
cudaError_t launch_flow_pack(const float *master, uint16_t *img, cudaStream_t st);

// Spline flow: the maps (as launch_flow_map), the per-CTA loss and derivative partials of a
// batch ([grid][dim * spline_grad_per_dim()] and [grid], fp64), and the step that sums them
// in CTA order, chains them to the parameters (grad_out, optional) and, with lr > 0, takes
// the Adam step.
cudaError_t launch_spline_map(const float *params, int dim, int direction, long long count, const double *in,
                              SobolDev rng, uint32_t k_first, const uint32_t *k_first_dev, int use_sobol, double *out,
                              double *out2, int grid, cudaStream_t st);
// The autoregressive spline flow (flow_arspline.cu; parameters: kb_spline.cuh's layout,
// ar_num_params(dim) floats): its maps, the per-CTA partial derivatives of the weighted
// negative log-likelihood over a batch ([grid][ar_num_params(dim)] and [grid], fp64; grid
// from ar_grad_grid), and the step that sums them in CTA order and takes the Adam step.
cudaError_t ar_configure();
size_t ar_grad_smem_bytes(int dim);
int ar_grad_grid(long long count, int sm_count);
cudaError_t launch_ar_map(const float *params, int dim, int direction, long long count, const double *in,
                          SobolDev rng, uint32_t k_first, const uint32_t *k_first_dev, int use_sobol, double *out,
                          double *out2, int grid, cudaStream_t st);
cudaError_t launch_ar_grad(const float *params, int dim, long long count, const float *x, const float *w,
                           const int *index, double inv_batch, double *partials, double *loss_part, int grid,
                           cudaStream_t st);
cudaError_t launch_ar_adam(float *params, float *m, float *v, int dim, const double *partials, int nparts,
                           const double *loss_part, double *loss_out, float *grad_out, float lr, float beta1,
                           float beta2, float eps, float bc1, float bc2, cudaStream_t st);

// Knots of the spline flow's dimensions from its parameters, [dim][SPL_KNOT_DOUBLES]: what a
// work item's in-line map reads (ItemDev::spline_knots).
cudaError_t launch_spline_knots(const float *params, int dim, double *knots, cudaStream_t st);
int spline_grad_per_dim();
cudaError_t launch_spline_grad(const float *params, int dim, long long count, const float *x, const float *w,
                               const int *index, double inv_batch, double *partials, double *loss_part, int grid,
                               cudaStream_t st);
cudaError_t launch_spline_adam(float *params, float *m, float *v, int dim, const double *partials, int nparts,
                               const double *loss_part, double *loss_out, float *grad_out, float lr, float beta1,
                               float beta2, float eps, float bc1, float bc2, cudaStream_t st);

} // namespace kb
