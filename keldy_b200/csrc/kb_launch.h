// Host-side launch interface of the kernels (implemented in tree.cu and misc_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "kb_types.h"

namespace kb {

enum InputMode {
  IN_TIMES = 0, // vertex times given: integrand_g_direct::operator()
  IN_LI = 1,    // hypercube points given, warped: evaluate_warped_integrand
  IN_SOBOL = 2, // Sobol points generated and warped, summed per chunk: integrator::run
};

// Per-chunk partial sums of the integrate mode. fb_mask marks the chunk's points whose
// tree pivots were guarded; the pivoted-LU pass adds them to sum_re/sum_im.
struct ChunkPartial {
  double sum_re;
  double sum_im;
  unsigned long long n_in_domain;
  unsigned long long n_fallback;
  unsigned long long fb_mask[2];
};

constexpr int CHUNK_POINTS = 128; // points per scheduling chunk (<= 128: two 64-bit masks)
// Per-CTA slot of the tree kernel in global memory (L2-resident): the chunk's set-up,
// PTS_ROWS doubles (coordinates [MAX_ORDER][CHUNK_POINTS], then the Jacobians and the
// domain flags of the chunk's points; with time bins also each point's bin code (2 bin + 1
// when its value is added, 2 bin when only counted, -1 when dropped) and its f*J (re,
// im)), then G_STAGE complex entries of staged G matrices (a G-batch, tree_gbatch).
constexpr int PTS_ROWS = CHUNK_POINTS * (MAX_ORDER + 5);
constexpr int G_STAGE = 4096;
// Frontier entries at the start of a buffer that the tree's fused bottom uses for its
// per-point sums (CTA_THREADS double2 and CTA_THREADS / 2 double2 of doubles).
constexpr int BOTTOM_SCRATCH = CTA_THREADS + CTA_THREADS / 2;
constexpr int PTS_SLOT = PTS_ROWS + 2 * G_STAGE;
// Per-CTA slot of the kernel-method tree: the chunk's set-up rows only.
constexpr int KM_SLOT = PTS_ROWS;
// Resident CTAs per SM of the kernel-method tree (256 threads, ~114 KB of shared memory).
constexpr int KM_CTAS_PER_SM = 2;
static_assert(PTS_ROWS % 2 == 0 && PTS_SLOT % 2 == 0, "staged G on 16-byte boundaries");

// Points per G-batch of the tree kernel at order N: their (2N+1)^2 matrices G fit the
// staging area, their coordinates the kernel's 256-entry shared array, and the count is a
// multiple of the sub-batch size tree_points_per_chunk(N).
__host__ __device__ inline int tree_gbatch(int N) {
  const int P = tree_points_per_chunk(N);
  const int M = 2 * N + 1;
  // orders above TREE_MAX_SUB keep up to four subtree roots (17 x 17) and their prefix
  // determinants after the batch's G matrices
  const int R = 2 * TREE_MAX_SUB + 1, reserve = N > TREE_MAX_SUB ? 4 * R * R + 4 : 0;
  int g = CHUNK_POINTS;
  if (N > 0 && 256 / N < g) g = 256 / N;
  if ((G_STAGE - reserve) / (M * M) < g) g = (G_STAGE - reserve) / (M * M);
  g -= g % P;
  return g > 0 ? g : P;
}

// Orders whose G-batch is a single sub-batch (1..4) gain nothing from staging G in global
// memory: the tree kernel builds their G directly in shared memory.
__host__ __device__ inline bool tree_direct(int N) {
  return N <= TREE_MAX_SUB && tree_gbatch(N) <= tree_points_per_chunk(N);
}

struct Launch {
  const ItemDev *items; // device
  int n_items;
  const long long *chunk_offsets; // device [n_items+1]: first chunk of each item (items sorted by cost)
  int n_chunks;
  int *chunk_counter; // device, zeroed before the launch (dynamic scheduling)
  int mode;
  int keep_u_hypercube;
  // IN_TIMES / IN_LI
  const double *in;     // [count][order]
  const int *index;     // optional list of point indices to evaluate (direct kernel, fallback)
  int n_index;
  double2 *out_val;     // f*J (or f)
  double *out_jac;
  int *out_dom;
  double *out_scale;
  int *out_flag;        // tree: 1 = point needs the pivoted-LU kernel
  // tree kernel: gridDim.x * PTS_SLOT doubles of set-up and staging scratch (kernel-method
  // tree: gridDim.x * KM_SLOT)
  double *pts;
  // IN_SOBOL
  ChunkPartial *partials; // [n_chunks]
  // IN_SOBOL with time bins (integrand_g_direct_time): every point's f*J also goes to the
  // bin of its earliest vertex time; per chunk: sums [n_chunks][nbins], counts, dropped
  int nbins; // 0: no bins
  int bin_cols; // values per time bin: 1 (time-binned direct integrand), 2 (kernel method: Keldysh index)
  double bin_xmin, bin_xmax, bin_size;
  double2 *out_kvals; // kernel method, IN_TIMES: per point the 2n sums (vertex i, Keldysh index k) at [2i + k]
  double2 *bin_sums;
  unsigned *bin_counts;
  unsigned *bin_dropped; // [n_chunks]
  // errors
  int *err; // bit 0: g0 evaluated outside its window
  // some item's model interpolates its tables cubically: the tree kernel's instantiation
  // that carries both interpolations (the default one has the linear lookup only)
  int any_cubic;
  // kernel method at a single frequency (integrand_g_kernel_single_omega), IN_SOBOL with no
  // bins: each point adds sum_i e^{i omega t_i} (its vertex i's terms of both Keldysh
  // indices) times its Jacobian to the chunk partials
  int km_fourier;
  double km_omega;
};

// any_cubic of a launch over items[0..n)
inline int items_any_cubic(const ItemDev *items, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (items[i].model.interp == 3) return 1;
  return 0;
}

size_t tree_smem_bytes();
// sets the kernels' shared-memory attributes (before any stream capture)
cudaError_t configure_kernels();
cudaError_t launch_tree(const Launch &L, int grid, cudaStream_t st);
cudaError_t launch_direct(const Launch &L, int grid, cudaStream_t st);
// pivoted-LU evaluation of the points marked in the chunk partials' fb_mask
cudaError_t launch_fallback(const Launch &L, int grid, cudaStream_t st);
// acc[item] += sum over the item's chunks in chunk order
cudaError_t launch_reduce(const Launch &L, kb_accum *acc_dev, cudaStream_t st);
// per item: bin sums [n_items][nbins], counts [n_items][nbins], dropped [n_items] summed
// over the item's chunks in chunk order (written, not added)
// keldy's kernel-method integrand (integrand_g_kernel): IN_SOBOL with time bins of 2
// columns, or IN_TIMES into out_kvals. Orders 1..KM_MAX_ORDER.
constexpr int KM_MAX_ORDER = 10;
cudaError_t launch_kernel_method(const Launch &L, int grid, cudaStream_t st);
cudaError_t launch_reduce_bins(const Launch &L, double2 *sums, unsigned long long *counts,
                               unsigned long long *dropped, cudaStream_t st);

cudaError_t launch_sobol_points(SobolDev s, uint32_t k_first, long long count, double *out, cudaStream_t st);
cudaError_t launch_warp(const WarperDev *chain_dev, int start, int end, int direction, int n, long long count,
                        const double *in, double *out, double *jac, cudaStream_t st);
cudaError_t launch_g0_eval(ModelDev m, const kb_gf_index *a, const kb_gf_index *b, const int *internal,
                           long long count, double2 *out, int *err, cudaStream_t st);
cudaError_t launch_no_det(ModelDev m, kb_integrand f, int order, long long count, const double *times, int keep,
                          double2 *out, int *dom, int *err, cudaStream_t st);
cudaError_t launch_table_max(const double2 *tab, int npts, double *out, cudaStream_t st);
// the same for n tables (device array of their pointers): out[i] for table i, one launch
cudaError_t launch_tables_max(double2 *const *tabs, int n, int npts, double *out, cudaStream_t st);
cudaError_t launch_fp64_peak(int iters, double *sink, int grid, int block, cudaStream_t st);
// Flat-band dot g0 tables of n models ({Gamma, eps_d, V, beta} each) on the mesh of
// npts points over [-tmax, tmax] (g0_build.cu); Gauss-Legendre rule on [-1, 1].
cudaError_t launch_fourier_table(const double *w, const double2 *cl, const double2 *cg, int n_nodes, double2 *tab,
                                 int npts, double tmax, int symmetric, int *bad, cudaStream_t st);
cudaError_t launch_mirror_block(const double2 *src, double2 *dst, int npts, cudaStream_t st);
// Tables of a bath with a rational hybridisation in closed form: n_terms terms, each a
// chemical potential and a rational function given by its simple poles and residues.
constexpr int RATIONAL_MAX_POLES = 8;
constexpr int RATIONAL_MAX_TERMS = 4;
struct RationalTermDev {
  double mu;
  int n;
  double2 z[RATIONAL_MAX_POLES], r[RATIONAL_MAX_POLES];
};
cudaError_t launch_rational_table(const RationalTermDev *terms, int n_terms, double beta, const double *nodes,
                                  const double *weights, int n_nodes, double2 *tab, int npts, double tmax, int symmetric,
                                  int *bad, cudaStream_t st);
// keldy's "fft" tables: the discrete transform of npts frequency values on the adjoint mesh,
// the 1/w^2 tails ml, mg beyond it transformed exactly
cudaError_t launch_dft_table(const double2 *gl, const double2 *gg, double2 ml, double2 mg, double2 *tab, int npts,
                             double tmax, int *bad, cudaStream_t st);
cudaError_t launch_flatband_tables(int n_models, const double *params_dev, double2 *const *tabs_dev, int npts,
                                   double tmax, const double *nodes_dev, const double *weights_dev, int n_nodes,
                                   cudaStream_t st);

} // namespace kb
