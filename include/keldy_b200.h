/*
 * keldy_b200 C ABI: the boundary between keldy's host classes and the sm_100a kernels.
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes. Every function
 * returns KB_OK (0) or a negative KB_E* code; kb_last_error() gives the message of the
 * calling thread's last failure. Host-pointer entry points copy their inputs to the
 * device, run on the context's CUDA stream and copy results back before returning;
 * the *_dev entry points take device pointers and only enqueue work on the stream.
 *
 * Each entry point names the keldy interface it replaces (paths relative to keldy's
 * c++/keldy/ source tree).
 */
#ifndef KELDY_B200_H
#define KELDY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KB_OK 0
#define KB_E_INVALID -1   /* bad argument (keldy raises TRIQS_RUNTIME_ERROR for these) */
#define KB_E_CUDA -2      /* a CUDA call failed */
#define KB_E_NOMEM -3     /* device or host allocation failed */
#define KB_E_RANGE -4     /* g0 evaluated outside its tabulated window */
#define KB_E_EXHAUSTED -5 /* Sobol generator past its last point */
#define KB_E_NODEVICE -6  /* no CUDA device: the library has no CPU path */

typedef struct kb_context kb_context;
typedef struct kb_model kb_model;
typedef struct kb_sobol kb_sobol;

/* ---------------------------------------------------------------- context --- */
const char *kb_last_error(void);
int kb_version(void);
/* One context per device: a CUDA stream plus reusable device buffers. */
int kb_context_create(int device, kb_context **out);
int kb_context_destroy(kb_context *ctx);
int kb_context_synchronize(kb_context *ctx);
/* The context's CUDA stream, as a cudaStream_t cast to void*. */
void *kb_context_stream(kb_context *ctx);
/* Kernel timing (measurement aid, off by default): when enabled, kb_integrate brackets
 * its integrand, pivoted-LU and reduction launches with CUDA events on the context's
 * stream; kb_context_last_timing returns the last call's times in milliseconds
 * (summed over its launch groups). */
int kb_context_set_timing(kb_context *ctx, int enable);
int kb_context_last_timing(kb_context *ctx, double *integrand_ms, double *fallback_ms, double *reduce_ms,
                           int *launches);

/* ------------------------------------------------------------------ Sobol --- */
/* keldy::sobol(dim, seed, do_shift, do_scramble, seed_shift, log_max_points)
 * (qrng.hpp:77-109; the unshifted qrng.hpp:69-75 is do_shift = do_scramble = 0).
 * Generating matrices of the Joe-Kuo 2008 sequence, optional random digital shift and
 * linear scramble from std::mt19937_64(seed_shift). The generator state (the index of
 * the last point drawn) stays with the caller: point number k (k >= 1) is the point
 * digitalseq_b2g::next() returns when its counter becomes k. */
int kb_sobol_create(kb_context *ctx, int dim, int log_max_points, int do_shift, int do_scramble, int seed_shift,
                    kb_sobol **out);
int kb_sobol_destroy(kb_sobol *s);
/* Host only (no device needed): the generator's bit-reversed generating matrices
 * Csr[dim * log_max_points] and shift vector shfr[dim], in digitalseq_b2g's Csr/shfr
 * layout (digitalseq_b2g.hpp:307-312, 486-513; qmc::JK2008_sobol_matrices and
 * qmc::scramble, digitalseq_b2g.hpp:178-186, 598-861). */
int kb_sobol_matrices(int dim, int log_max_points, int do_shift, int do_scramble, int seed_shift, uint32_t *Csr,
                      uint32_t *shfr);
/* Points k_first .. k_first+count-1, row-major [count][dim] doubles
 * (replaces digitalseq_b2g::next/set_state, digitalseq_b2g.hpp:415-471, and
 * sobol::operator()/seed/discard, qrng.hpp:51-67). KB_E_EXHAUSTED past 2^log_max_points. */
int kb_sobol_points(kb_context *ctx, const kb_sobol *s, uint32_t k_first, int64_t count, double *out);
int kb_sobol_points_dev(kb_context *ctx, const kb_sobol *s, uint32_t k_first, int64_t count, double *out_dev);

/* ---------------------------------------------------------------- warpers --- */
#define KB_WARPER_IDENTITY 0       /* warper_identity_t (warpers/identity.hpp:30-49) */
#define KB_WARPER_PLASMA_UV 1      /* warper_plasma_uv_t(t_max) (warpers/plasma_uv.hpp:55-81) */
#define KB_WARPER_EXPONENTIAL 2    /* make_product_1d_simple_exponential(u_max, w) (product_1d_simple.hpp:560-576) */
#define KB_WARPER_INVERSE 3        /* make_product_1d_simple_inverse(u_max, w) (:578-592) */
#define KB_WARPER_INVERSE_SQUARE 4 /* make_product_1d_simple_inverse_square(u_max, w) (:594-608) */
#define KB_WARPER_INVERSE_POWER 5  /* make_product_1d_simple_inverse_power(power, u_max, w) (:610-630) */
#define KB_WARPER_UNIFORM 6        /* warper_product_1d_simple_t with f1 = 1/u_max (product_1d_simple_test.cpp:10-23) */
#define KB_WARPER_TABLE 7          /* device-resident product warper: kb_warper_table (see below) */
#define KB_MAX_CHAIN 8

typedef struct {
  int kind;
  int power;    /* KB_WARPER_INVERSE_POWER only */
  double u_max; /* domain_u_max, or t_max for the plasma warper */
  double w;     /* w_scale of the product makers */
  const struct kb_warper_table *table; /* KB_WARPER_TABLE only */
} kb_warper;

/* Device-resident product warpers, used in a chain as {KB_WARPER_TABLE, .table = t}. A
 * table object holds one 1D warper per coordinate (ndims = the order) or one for every
 * coordinate (ndims = 1). Its type:
 * KB_TABLE_NEAREST: warper_product_1d_simple_interp_nearest_t (product_1d_simple.hpp:
 *   174-330; ndims = 1) and warper_product_1d_interp_nearest_t (product_1d.hpp:164-211).
 *   kb_warper_table_create: table d has npts[d] >= 3 points u (u[0] = 0, strictly
 *   increasing, the last one the domain's u_max) with values f1 >= 0 there; the arrays of
 *   all tables are concatenated. As keldy's integrate_and_inverse (:219-253): F is f1's
 *   trapezoid integral from u_max, normalised to 1; u = F^-1(l) and the Jacobian 1/f1(u)
 *   use linear interpolation on the points (f1 on an interval: the mean of its ends).
 *   Errors as keldy: "Model function is flat zero.", fewer than 3 points, u[0] != 0.
 * KB_TABLE_PROJECTION: warper_projection_t (projection.hpp:176-382), see below.
 * KB_TABLE_ANALYTIC: warper_product_1d_t (product_1d.hpp:110-160): dims[d] one of the
 *   product makers (KB_WARPER_EXPONENTIAL .. KB_WARPER_UNIFORM) for coordinate d
 *   (make_product_1d_inverse_cube_alternate, :253-266).
 * KB_TABLE_HYBRID: warper_product_1d_simple_interp_hybrid_t (product_1d_simple.hpp:
 *   381-554) per coordinate: f1[d].kind names the closed form of f1 up to a factor
 *   (EXPONENTIAL exp(-u/w), INVERSE w/(w+u), INVERSE_SQUARE (w/(w+u))^2, INVERSE_POWER
 *   (w/(w+u))^power, UNIFORM 1), f1[d].u_max the domain, npts[d] >= 3 equidistant points;
 *   F by Simpson's rule, Steffen splines of F and of its inverse, Jacobian from the closed
 *   form (make_product_1d_inverse_cube_alternate_interp_hybrid, product_1d.hpp:290-309). */
#define KB_TABLE_NEAREST 0
#define KB_TABLE_PROJECTION 1
#define KB_TABLE_ANALYTIC 2
#define KB_TABLE_HYBRID 3
typedef struct kb_warper_table kb_warper_table;
int kb_warper_table_create(kb_context *ctx, int ndims, const int *npts, const double *u_pts, const double *f1_pts,
                           kb_warper_table **out);
int kb_warper_table_analytic(kb_context *ctx, int ndims, const kb_warper *dims, kb_warper_table **out);
int kb_warper_table_hybrid(kb_context *ctx, int ndims, const kb_warper *f1, const int *npts, kb_warper_table **out);
int kb_warper_table_destroy(kb_warper_table *t);
/* type, number of coordinates and (npts, optional, [ndims]) the points of each one's table */
int kb_warper_table_info(const kb_warper_table *t, int *type, int *ndims, int *npts);
/* KB_TABLE_NEAREST: the points u and the f1 values (as given, before normalisation) of
 * coordinate d's table (npts[d] each). */
int kb_warper_table_points(const kb_warper_table *t, int d, double *u, double *f1);

/* make_warper_from_proj (warpers/make_warper_from_proj.hpp:118-153) from samples the
 * caller computed: li [n][order] (keldy uses Sobol points 1..n of dimension order,
 * unshifted) and values[n] = |f J| there. Per axis the mean value in each of num_bins
 * bins of [0, 1], smoothed by a local linear fit of its logarithm with a Gaussian kernel
 * of width sigma (kernel_smoothing, :40-66), turned into f1 points (f1[0] = 0,
 * f1[i+1] = 2 s_i - f1[i]) of a KB_TABLE_NEAREST table per axis. */
int kb_warper_table_from_samples(kb_context *ctx, int order, int num_bins, int64_t n, const double *li,
                                 const double *values, double sigma, kb_warper_table **out);

/* warper_projection_t(warped_integrand, order, num_bins, nr_samples, sigma, optimize_sigma)
 * (projection.hpp:225-332) from samples li [n][order] with values |f J|: per axis the
 * mean value in num_bins bins centred on the points i/(num_bins-1), smoothed with width
 * sigma or, with optimize_sigma, the width (>= 0.3 bins) minimising the leave-one-out
 * error (optimize_sigma, :82-128); fn = the smoothed projection on num_bins mesh points,
 * its normalised integral, and the integral's inverse (Akima interpolation) on
 * 1 + 5 (num_bins - 1) points. Reverse map u = inverse(l) with Jacobian norm / fn(u),
 * forward l = integral(u) with Jacobian fn(u), all linearly interpolated on the meshes.
 * num_bins >= 5. */
int kb_warper_projection_create(kb_context *ctx, int order, int num_bins, int64_t n, const double *li,
                                const double *values, double sigma, int optimize_sigma, kb_warper_table **out);
/* One axis of a projection warper: its smoothing width (natural units), the binned mean
 * |f J| and counts (num_bins each; get_xi) and fn on the mesh (num_bins; get_fi). Any
 * output may be null. */
int kb_warper_projection_axis(const kb_warper_table *t, int axis, double *sigma, double *xi, uint64_t *xi_count,
                              double *fn);

/* warper_train_t::map_reverse(li, start, end) (warpers.hpp:72-85; direction 0) or
 * map_forward(ui, start, end) (warpers.hpp:88-101; direction 1) on count points of n
 * coordinates each. Warpers are applied last-to-first in reverse, first-to-last
 * forward. jac may be NULL (ui_from_li / li_from_ui). */
#define KB_REVERSE 0
#define KB_FORWARD 1
int kb_warp(kb_context *ctx, const kb_warper *chain, int chain_len, int direction, int start, int end, int n,
            int64_t count, const double *in, double *out, double *jac);

/* ---------------------------------------------------------------- g0 model --- */
/* g0 tables on the uniform mesh t_i = -time_max + i*2*time_max/(npts-1), i < npts
 * (keldy's g0_model::g0_lesser / g0_greater, model.hpp:183-190): complex values as
 * interleaved (re, im) doubles. One table pair per (spin, orbital a, orbital b); the
 * Keldysh adaptor (model.hpp:244-265) picks lesser or greater by contour order. */
int kb_model_create(kb_context *ctx, int npts, double time_max, double alpha, kb_model **out);
int kb_model_destroy(kb_model *m);
/* Upload the (spin, o1, o2) block; lesser/greater: npts interleaved complex values. */
int kb_model_set_table(kb_model *m, int spin, int o1, int o2, const double *lesser, const double *greater);
/* Same from device memory. */
int kb_model_set_table_dev(kb_model *m, int spin, int o1, int o2, const double *lesser_dev,
                           const double *greater_dev);
/* Copies a model's g0^< and g0^> table of (spin, o1, o2) to the host (interleaved complex,
 * npts each): keldy's public g0_model::g0_lesser / g0_greater members (model.hpp:184-188).
 * A spin never uploaded reads the other spin's table. */
int kb_model_get_table(kb_model *m, int spin, int o1, int o2, double *lesser, double *greater);
/* Builds the spin-up orbital (0,0) tables of n models on the GPU, the single-level dot
 * coupled to two flat-band leads (keldy's make_g0_flat_band with the contour/fft
 * methods' functions, impurity_oneband/model.hpp:100-130, model.cpp:107-111, evaluated
 * in closed form through the exponential integral plus a quadrature of the
 * finite-temperature correction; the same functions as the package's host builder
 * g0_tables.flatband). params [n][4] = {Gamma, eps_d, V, beta} (beta = INFINITY: zero
 * temperature; mu_left = -V/2, mu_right = +V/2). All models share one context and one
 * time mesh (odd npts). */
int kb_models_set_flatband(int n, kb_model *const *models, const double *params);
/* Interpolation of the tables between mesh points: KB_INTERP_LINEAR (keldy's, TRIQS
 * gf<retime> evaluation; the default) or KB_INTERP_CUBIC, an extension with no keldy
 * counterpart: Lagrange interpolation through the 4 mesh points around the interval (the
 * window moved inside the mesh at its ends). Needs npts >= 4 for cubic. */
#define KB_INTERP_LINEAR 1
#define KB_INTERP_CUBIC 3
int kb_model_set_interpolation(kb_model *m, int order);

/* Fourier sums by quadrature, the GPU form of keldy's finite-contour construction
 * (make_g0_by_finite_contour, model.cpp:220-319, which integrates g^{</>}(w) e^{-iwt}/2pi
 * over the band by adaptive quadrature) with the nodes and weights chosen by the caller:
 * block (o1, o2) of model m (used for both spins) gets
 *   g^<(t) = sum_k cl[k] e^{-i w[k] t},   g^>(t) = sum_k cg[k] e^{-i w[k] t}
 * at every mesh point (cl, cg: n_nodes interleaved complex, the quadrature weights and
 * 1/2pi included). KB_FT_SYMMETRIC: only t >= 0 is summed (t = 0 exactly at the middle
 * point; odd npts) and g(-t) = -conj(g(t)) fills the rest (the dot block, model.cpp:302-310).
 * KB_FT_MIRROR: block (o2, o1) is also set, to -conj(g_{o1 o2}(-t)) (model.cpp:311-313).
 * KB_E_INVALID if a value is not finite. */
#define KB_FT_SYMMETRIC 1
#define KB_FT_MIRROR 2
int kb_model_set_fourier(kb_model *m, int o1, int o2, int n_nodes, const double *w, const double *cl,
                         const double *cg, int flags);

/* keldy's ft_method "fft" (make_g0_by_fft, model.cpp:179-212, which transforms with TRIQS's
 * make_gf_from_fourier) on the GPU: block (o1, o2) of model m (both spins) from its values
 * gl = g^<(w_j), gg = g^>(w_j) (npts interleaved complex each) on the frequency mesh adjoint
 * to the model's time mesh: w_j = (j - c) dw, c = (npts - 1)/2, dw = 2 pi/(npts dt), dt the
 * time step (npts odd). Every mesh point gets the discrete transform
 *   g(t_k) = dw/(2 pi) sum_j g(w_j) e^{-i w_j t_k},
 * with the functions' 1/w^2 tails beyond the mesh transformed exactly: m2 = the mean of
 * w^2 g(w) at the mesh's two ends, g - m2/(w^2 + a^2) summed discretely (a = dw sqrt(npts)),
 * m2 e^{-a|t|}/(2a) added (the subtraction TRIQS's real-frequency transform makes).
 * KB_FT_MIRROR also sets block (o2, o1) = -conj(g_{o1 o2}(-t)), the transform of the
 * frequency values -conj(g_{o1 o2}(w)) keldy gives that block (model.cpp:196-199).
 * KB_E_INVALID if a value is not finite. */
int kb_model_set_fft(kb_model *m, int o1, int o2, const double *gl, const double *gg, int flags);

/* keldy's ft_method "contour" for the baths whose hybridisation is rational (flat band,
 * Lorentzian: make_g0_by_contour, model.cpp:326-426, integrates their Fourier transforms
 * along a contour in the complex plane) in closed form on the GPU. The block's functions are
 * given as sums over n_terms leads of a Fermi function times a rational function with
 * simple poles: g^<(w) = sum_l n_F(w - mu[l]) R_l(w), g^>(w) = -sum_l (1 - n_F(w - mu[l]))
 * R_l(w), R_l(w) = sum_k r_lk / (w - z_lk) (n_poles[l] <= 8 poles z off the real axis,
 * residues r; poles/residues interleaved complex, term after term; R_l decaying at least as
 * 1/w^2). Every mesh point gets g(t) = int dw/2pi e^{-iwt} g(w): the zero-temperature part
 * through the exponential integral E1 at each pole, the finite-temperature correction by
 * Gauss-Legendre quadrature within 36/beta of each mu (beta = INFINITY: none).
 * KB_FT_SYMMETRIC: t >= 0 only, g(-t) = -conj(g(t)); KB_FT_MIRROR: block (o2, o1) too. */
int kb_model_set_rational(kb_model *m, int o1, int o2, int n_terms, const double *mu, const int *n_poles,
                          const double *poles, const double *residues, double beta, int flags);

/* A point of the Keldysh contour with spin and orbital: keldy's gf_index_t (model.hpp:55-78). */
typedef struct {
  double time;
  int spin;      /* 0 = up, 1 = down */
  int k_idx;     /* 0 = forward, 1 = backward */
  int timesplit; /* orders equal-time points */
  int orbital;
} kb_gf_index;

/* g0_keldysh_contour_t::operator()(a[i], b[i], internal[i]) (model.hpp:244-265);
 * out: count interleaved complex values. internal may be NULL (all true). */
int kb_g0_eval(kb_context *ctx, const kb_model *m, const kb_gf_index *a, const kb_gf_index *b, const int *internal,
               int64_t count, double *out);

/* ------------------------------------------------------------- integrand --- */
/* integrand_g_direct(g0, external_A, external_B, cutoff) (wick_direct.hpp:34-65). */
typedef struct {
  kb_gf_index A;
  kb_gf_index B;
  double cutoff;
} kb_integrand;

#define KB_ALGO_AUTO 0   /* Schur-complement tree, pivoted per-configuration LU where the tree cannot run */
#define KB_ALGO_TREE 1   /* Schur-complement tree over the Keldysh bits */
#define KB_ALGO_DIRECT 2 /* one partial-pivot LU pair per Keldysh configuration (keldy's own algorithm) */

/* integrand_g_direct::operator()(times, keep_u_hypercube) (wick_direct.cpp:43-158) on
 * count time vectors of `order` entries. out: interleaved complex; in_domain: int per
 * point; scale (optional, may be NULL): sum over Keldysh configurations of
 * |det up * det down| (error scale of the alternating sum). */
int kb_integrand_eval(kb_context *ctx, const kb_model *m, const kb_integrand *f, int order, int64_t count,
                      const double *times, int keep_u_hypercube, int algo, double *out, int *in_domain,
                      double *scale);
/* integrand_g_direct::eval_no_det (wick_direct.cpp:161-228), orders 0..2. */
int kb_integrand_eval_no_det(kb_context *ctx, const kb_model *m, const kb_integrand *f, int order, int64_t count,
                             const double *times, int keep_u_hypercube, double *out, int *in_domain);

/* integrator::evaluate_warped_integrand(li, start_domain_nr, keep_u_hypercube)
 * (integrator.hpp:68-79): out = f(map_reverse(li, start, 0)) * J as interleaved
 * complex; jac (optional): J; in_domain: int per point. */
int kb_evaluate_warped(kb_context *ctx, const kb_model *m, const kb_integrand *f, const kb_warper *chain,
                       int chain_len, int start_domain_nr, int order, int64_t count, const double *li,
                       int keep_u_hypercube, int algo, double *out, double *jac, int *in_domain);

/* make_warper_from_proj (warpers/make_warper_from_proj.hpp:118-153) for the integrand f
 * on model m through `chain`: |f J| at Sobol points 1..nr_samples of dimension order
 * (unshifted), evaluated on the GPU, then as kb_warper_table_from_samples. The table maps
 * the Sobol point before `chain` (append it to the chain's end). */
int kb_warper_table_from_projection(kb_context *ctx, const kb_model *m, const kb_integrand *f,
                                    const kb_warper *chain, int chain_len, int order, int num_bins, int nr_samples,
                                    double sigma, int keep_u_hypercube, kb_warper_table **out);
/* warper_projection_t for the integrand f on model m through `chain` (Sobol points
 * 1..nr_samples, unshifted, evaluated on the GPU). */
int kb_warper_projection_from_integrand(kb_context *ctx, const kb_model *m, const kb_integrand *f,
                                        const kb_warper *chain, int chain_len, int order, int num_bins,
                                        int nr_samples, double sigma, int optimize_sigma, int keep_u_hypercube,
                                        kb_warper_table **out);

/* ------------------------------------------------------------- integrator --- */
/* Running sums of integrator::run (integrator.hpp:50-52). */
typedef struct {
  double sum_re;        /* sum of f*J */
  double sum_im;
  uint64_t n_points;    /* points run */
  uint64_t n_in_domain; /* integrand evaluations in domain */
  uint64_t n_fallback;  /* points the tree handed to the pivoted-LU kernel (guarded pivots) */
} kb_accum;

typedef struct kb_flow kb_flow;

/* One unit of QMC work: `n_points` Sobol points k_first.. of `rng` through `chain` into
 * the integrand of `order` on model `m`. `flow` (optional, NULL = none): a learned
 * coupling flow of dimension `order` applied to each Sobol point before the chain, its
 * Jacobian multiplying the chain's (see kb_flow_create). */
typedef struct {
  const kb_model *m;
  const kb_sobol *rng;
  const kb_warper *chain;
  int chain_len;
  kb_integrand f;
  int order;
  uint32_t k_first;
  int64_t n_points;
  const kb_flow *flow;
} kb_work;

/* integrator::run(nr_steps) (integrator.hpp:81-95) for every work item, summed into
 * acc[i] (acc is added to, not overwritten). All items run in one batched launch
 * sequence on the context's stream; sums are deterministic (fixed reduction order). */
int kb_integrate(kb_context *ctx, const kb_work *work, int n_work, int algo, kb_accum *acc);

/* Time bins of integrand_g_direct_time (wick_direct_time.cpp:42-163): each point's f*J
 * goes to the bin of its earliest vertex time in the binner (xmin, xmax, nbins) of
 * binner_t (binner.hpp:163-176, 241-260: points outside [xmin, xmax] are dropped, xmax
 * itself falls in the last bin); out-of-domain points add 0 to their bin's sum and count.
 * compute_charge_Q_direct_time (compute_obs.hpp:85-101) bins [0, t] in nr_time_slices. */
typedef struct {
  int nbins;
  double xmin, xmax;
} kb_time_bins;
/* kb_integrate plus, per work item, the binned sums bin_sums[n_work][nbins] (interleaved
 * complex), the counts bin_counts[n_work][nbins] of values added and dropped[n_work]: all
 * added to. nbins in [1, 4096]. */
int kb_integrate_binned(kb_context *ctx, const kb_work *work, int n_work, int algo, const kb_time_bins *bins,
                        kb_accum *acc, double *bin_sums, uint64_t *bin_counts, uint64_t *dropped);

/* The kernel method (integrand_g_kernel, impurity_oneband/wick_kernel.cpp:42-138, with
 * first_row_expansion, det_expansion.hpp:44-74; compute_gf_kernel, compute_obs.hpp:105-117):
 * the fixed point X = work[i].f.A (f.B and the cutoff are not used). For every Keldysh
 * configuration a, the first-row cofactors x of s1 (X first, then the vertices picked by
 * a; keldy's zeroed entry (n, n) kept) times (-1)^|a| det(s2_a); vertex i's term goes to
 * the bin of (its time, a_i) of binner_t<1, 1>(xmin, xmax, nbins) x {forward, backward}.
 * bin_sums[n_work][nbins][2] (interleaved complex), bin_counts[n_work][nbins][2] (values
 * added), dropped[n_work]: added to; acc: the sum of all terms and the point counts.
 * Orders 1..10; no learned flows. */
int kb_integrate_kernel(kb_context *ctx, const kb_work *work, int n_work, const kb_time_bins *bins, kb_accum *acc,
                        double *bin_sums, uint64_t *bin_counts, uint64_t *dropped);
/* The kernel method at a single frequency (integrand_g_kernel_single_omega,
 * impurity_oneband/wick_kernel_single_omega.cpp:42-140; compute_gf_kernel_single_omega,
 * compute_obs.hpp:119-133): per point, the terms of kb_integrate_kernel (fixed point X =
 * work[i].f.A; first-row cofactors of s1 times (-1)^|a| det(s2_a)) summed with the weight
 * e^{i omega t} of their vertex's time t; acc[i] += the sum of those values times the
 * warper Jacobian, and the point counts. Orders 1..10; no learned flows. */
int kb_integrate_kernel_single_omega(kb_context *ctx, const kb_work *work, int n_work, double omega,
                                     kb_accum *acc);
/* integrand_g_kernel::operator()(times, keep_u_hypercube) for count points of `order` vertex
 * times: out[count][order][2] (interleaved complex) = the point's terms summed per (vertex i,
 * Keldysh index k), the sums of the pairs keldy's wick_kernel_test compares; in_domain. */
int kb_integrand_kernel_eval(kb_context *ctx, const kb_model *m, const kb_gf_index *X, int order, int64_t count,
                             const double *times, int keep_u_hypercube, double *out, int *in_domain);

/* Integrate without allocating device memory. No counterpart in keldy: this entry point
 * is for callers that cannot call cudaMalloc (a host application whose own allocator
 * owns the device's memory, or a latency-bound loop that must not pay cudaMalloc's
 * implicit synchronisation). Same work and sums as kb_integrate with KB_ALGO_AUTO, but
 * its scratch lives in one file-scope device array of KB_NOALLOC_SCRATCH_BYTES (held by
 * every GPU that loads the library until exit) instead of per-call allocations; the
 * model tables and Sobol matrices are the caller's existing objects. Limits: at most
 * KB_NOALLOC_MAX_ITEMS work items and KB_NOALLOC_MAX_CHUNKS scheduling chunks per call
 * (8,388,608 points with the default 128-point chunks; KB_E_INVALID beyond). The chunk
 * size and CTAs per SM are the context's launch shape (kb_context_set_launch), as in
 * kb_integrate; the tree grid is also capped at the per-CTA slots the array holds (more
 * than the 592 resident CTAs of a B200). All calls share the array: calls that overlap on
 * the GPU race. The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make it before any stream capture. */
#define KB_NOALLOC_MAX_ITEMS 64
#define KB_NOALLOC_MAX_CHUNKS 65536
#define KB_NOALLOC_SCRATCH_BYTES (56u << 20)
int kb_integrate_noalloc(kb_context *ctx, const kb_work *work, int n_work, kb_accum *acc);

/* Number of device allocations (cudaMalloc and stream-ordered pool allocations) the
 * library has made in this process. A diagnostic with no keldy counterpart: it lets a
 * caller check that kb_integrate_noalloc allocates nothing. */
uint64_t kb_device_allocations(void);

/* ------------------------------------------------------------------ plans --- */
/* A batched integration set up once and launched many times: the work items' descriptors
 * and scratch stay on the device, and the launch sequence (tree or pivoted-LU kernel,
 * guarded-pivot pass, reduction) is captured into a CUDA graph on the first launch and
 * replayed after. Replaces keldy's per-point integrator::run loop (integrator.hpp:81-95)
 * for a fixed set of (model, order, generator, warper chain) runs. */
typedef struct kb_plan kb_plan;
int kb_plan_create(kb_context *ctx, const kb_work *work, int n_work, int algo, kb_plan **out);
int kb_plan_destroy(kb_plan *plan);
/* Enqueue one run on the context's stream; the sums of this run land in the plan's device
 * accumulators (read them with kb_plan_result). */
int kb_plan_launch(kb_context *ctx, kb_plan *plan);
/* Wait for the last launch and add its sums to acc[n_work]. */
int kb_plan_result(kb_context *ctx, kb_plan *plan, kb_accum *acc);
/* Move work item i to Sobol points k_first .. k_first + n_points - 1 for the next launch
 * (the generator state advances without rebuilding the plan). */
int kb_plan_set_k_first(kb_context *ctx, kb_plan *plan, int item, uint32_t k_first);

/* Launch shape of the tree kernel: points per scheduling chunk for `order` (1..128;
 * order -1 sets every order) and resident CTAs per SM (1 to 4; 0 keeps the value). A work
 * item with fewer chunks than half the resident CTAs runs in chunks halved (down to 8
 * points) until it has that many, so that it spreads over the GPU; the chunking depends on
 * the item alone. */
int kb_context_set_launch(kb_context *ctx, int order, int chunk_points, int ctas_per_sm);
int kb_context_get_launch(kb_context *ctx, int order, int *chunk_points, int *ctas_per_sm);

/* ------------------------------------------------------ learned flow warper --- */
/* No counterpart in keldy: a learned first stage of the warper chain. A flow of
 * dimension n (2..8) maps the Sobol point z in [0,1]^n to the chain's input li with an
 * exact Jacobian; six coupling layers, each redrawing half of the dims through 32-bin
 * piecewise-linear CDFs whose logits come from a 128-wide two-hidden-layer ReLU MLP of
 * the other half (bf16 weights, fp32 accumulation on the tensor cores, CDFs in fp64 when
 * sampling). Trained by weighted maximum likelihood on points li with weights |f(li) J|
 * of the plain warper chain, its density approaches |integrand|, which lowers the
 * variance of the estimate; the plain chain alone remains the method without it.
 * Parameters: KB_FLOW_PARAMS floats, [layer][matrix W1, W2, W3][out][in], 128 x 128
 * each; the biases are column 16*T_l[0] of W1 (constant input) and column 127 of W2, W3
 * (hidden unit 127 is fixed to 1). */
#define KB_FLOW_LAYERS 6
#define KB_FLOW_WIDTH 128
#define KB_FLOW_MAX_DIM 8
#define KB_FLOW_PARAMS (KB_FLOW_LAYERS * 3 * KB_FLOW_WIDTH * KB_FLOW_WIDTH)
/* W1, W2 uniform in +-sqrt(6/128) from mt19937_64(seed), W3 = 0 (identity flow). */
int kb_flow_create(kb_context *ctx, int dim, uint64_t seed, kb_flow **out);
/* No counterpart in keldy: the second learned first stage, a separable spline flow. Per
 * dimension d (1..8) a monotone rational-quadratic spline CDF F_d on [0, 1] with 16 bins
 * (widths and heights from softmaxes of 16 logits each, at least 1e-3; knot derivatives
 * 1e-3 + softplus of 17 parameters); density q(x) = prod_d F_d'(x_d), sampling
 * x_d = F_d^{-1}(z_d). Smooth and acting on each axis alone, it keeps the structure that
 * quasi-Monte Carlo exploits. Same calls as the coupling flow (map, sample, gradient,
 * train, fit, work items); parameters: kb_flow_num_params = dim * 49 floats, [dim][16 width
 * logits, 16 height logits, 17 derivative parameters]; created as the identity map. In
 * kb_integrate and plans its map runs in line in the integrand kernel's point set-up (its
 * knots made from the current parameters at every call or replay): no mapped-point buffer
 * and no extra pass, results equal to mapping by kb_flow_sample first. */
#define KB_FLOW_COUPLING 0
#define KB_FLOW_SPLINE 1
/* No counterpart in keldy: the third learned first stage, an autoregressive
 * (Knothe-Rosenblatt) spline flow. Dimension d goes through the spline CDF above with its
 * 49 parameters theta_d = A_d phi_d, phi_d = [1, P1(x_k), P2(x_k), P3(x_k) for k < d]
 * (Legendre polynomials on [0, 1] of the dimensions before it), so each vertex time's
 * density is conditioned smoothly on the earlier ones. Parameters: kb_flow_num_params =
 * 49 * (dim + 3 dim (dim - 1) / 2) floats, A_0, A_1, ... each [49][1 + 3 d] row-major;
 * created as the identity map; with only the constant column set it is the separable flow
 * of those parameters. Mapped in line like the separable flow. */
#define KB_FLOW_AR_SPLINE 2
int kb_flow_create_kind(kb_context *ctx, int dim, int kind, uint64_t seed, kb_flow **out);
/* Parameters of the flow: KB_FLOW_PARAMS (coupling), dim * 49 (spline) or
 * 49 * (dim + 3 dim (dim - 1) / 2) (autoregressive spline). */
int kb_flow_num_params(const kb_flow *flow);
int kb_flow_destroy(kb_flow *flow);
int kb_flow_dim(const kb_flow *flow);
int kb_flow_get_params(kb_flow *flow, float *params);
int kb_flow_set_params(kb_flow *flow, const float *params);
/* direction 0 (density): x [count][dim] -> z, out2 = log q(x); direction 1 (sampling):
 * z -> x, out2 = dx/dz = 1/q(x). Host arrays. */
int kb_flow_map(kb_flow *flow, int direction, int64_t count, const double *in, double *out, double *out2);
/* Sampling direction on Sobol points k_first.. of rng (host outputs). */
int kb_flow_sample(kb_flow *flow, const kb_sobol *rng, uint32_t k_first, int64_t count, double *x, double *jac);
/* Loss sum_p w_p (-log q(x_p)) / count and its gradient (KB_FLOW_PARAMS floats, layout of
 * kb_flow_get_params) on the GPU's own forward and backward kernels. */
int kb_flow_gradient(kb_flow *flow, int64_t count, const double *x, const double *w, float *grad, double *loss);
typedef struct {
  int epochs;       /* passes over the samples */
  int batch;        /* points per step (multiple of 128 recommended) */
  float lr;         /* Adam step size, cosine-decayed to lr_final */
  float lr_final;
  float beta1, beta2, eps;
  uint64_t seed;    /* shuffling of the samples per epoch */
} kb_flow_train_cfg;
/* Adam on the weighted negative log-likelihood of samples x [count][dim] (in [0,1]) with
 * weights w >= 0 (normalised to mean 1 internally). loss_hist (optional): the loss of
 * every step, *n_steps of them. */
int kb_flow_train(kb_flow *flow, int64_t count, const double *x, const double *w, const kb_flow_train_cfg *cfg,
                  double *loss_hist, int *n_steps);
/* Generates n_samples points with the plain method (Sobol points k_first.. of rng,
 * weights |f(chain(li)) J_chain|) and trains the flow on them. */
int kb_flow_fit(kb_flow *flow, const kb_model *m, const kb_integrand *f, const kb_warper *chain, int chain_len,
                const kb_sobol *rng, uint32_t k_first, int64_t n_samples, const kb_flow_train_cfg *cfg,
                double *final_loss);

/* ----------------------------------------------------------------- peaks --- */
/* Measures the FP64 FMA rate of this device (FLOP/s, 2 per FMA) with a dependent-chain
 * kernel of `iters` FMAs per thread; used as the roofline denominator. */
int kb_fp64_peak(kb_context *ctx, int iters, double *flops_per_s);

#ifdef __cplusplus
}
#endif
#endif /* KELDY_B200_H */
