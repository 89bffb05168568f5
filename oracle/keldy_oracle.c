/*
 * keldy CPU oracle: a plain-C restatement of keldy's quasi-Monte-Carlo hot path.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the keldy_b200 package links, loads or calls
 * this file; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * it, and only as the checker (or the timed CPU baseline), never as the thing measured
 * or shipped.
 *
 * What it restates (paths relative to the keldy source tree):
 *   - Sobol digital sequence: qrng_details/digitalseq_b2g.hpp (next 415-426,
 *     set_state 455-471, bitreverse 45-66, bit_depth 139-146, random linear scramble
 *     156-186 / 209-237) and the keldy::sobol wrapper in qrng.hpp:49-114 (first draw is
 *     k = seed + 1; shifts are mt19937_64 draws narrowed to 32 bits).
 *   - Warpers: identity.hpp:30-49, plasma_uv.hpp:35-81, product_1d_simple.hpp:44-168
 *     and its makers 560-630; the chain order of warpers.hpp:72-101.
 *   - g0 contour adaptor: model.hpp:244-265 with compare_3way (common.cpp:47-57) and
 *     linear interpolation on the uniform time mesh (TRIQS gf<retime> evaluation).
 *   - Wick-determinant integrand: impurity_oneband/wick_direct.cpp:43-158 with a
 *     partial-pivot complex LU determinant (LAPACK zgetf2 order of operations, pivot =
 *     first maximum of |re|+|im|), and eval_no_det (wick_direct.cpp:161-228).
 *   - Integrator loop: integrator.hpp:68-95, 123-131.
 *
 * Parity anchors: Sobol points and warper outputs are pinned by the compiled reference
 * (oracle/_ref, built from keldy's own sources) and the fixtures in tests/golden/; the
 * integrand is pinned by keldy's order-1/order-2 closed-form Wick sums (the
 * eval_no_det restatement below) and by the compiled reference integrand.
 *
 * Compiled with -ffp-contract=off so that every product and sum rounds exactly once.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../keldy_b200/csrc/sobol_joe_kuo.h"

/* ------------------------------------------------------------------------- */
/* Complex arithmetic (explicit, so the rounding sequence is fixed).         */
/* ------------------------------------------------------------------------- */
typedef struct {
  double re, im;
} cplx;

static inline cplx c_make(double re, double im) {
  cplx z = {re, im};
  return z;
}
static inline cplx c_add(cplx a, cplx b) { return c_make(a.re + b.re, a.im + b.im); }
static inline cplx c_sub(cplx a, cplx b) { return c_make(a.re - b.re, a.im - b.im); }
static inline cplx c_mul(cplx a, cplx b) { return c_make(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cplx c_scale(cplx a, double s) { return c_make(a.re * s, a.im * s); }
static inline double c_abs1(cplx a) { return fabs(a.re) + fabs(a.im); }
static inline double c_abs(cplx a) { return hypot(a.re, a.im); }
static inline cplx c_div(cplx a, cplx b) {
  /* Smith's algorithm (the usual Fortran/C++ complex division) */
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re, d = b.re + b.im * r;
    return c_make((a.re + a.im * r) / d, (a.im - a.re * r) / d);
  }
  double r = b.re / b.im, d = b.re * r + b.im;
  return c_make((a.re * r + a.im) / d, (a.im * r - a.re) / d);
}

/* ------------------------------------------------------------------------- */
/* Sobol sequence                                                             */
/* ------------------------------------------------------------------------- */

/* Generating matrices of the Joe-Kuo 2008 sequence: dim x m columns, least
 * significant bit = first binary digit (digitalseq_b2g.hpp:598-861). */
int or_sobol_matrices(int dim, int m, uint32_t *Cs) {
  if (dim < 1 || dim > KB_SOBOL_MAX_DIM || m < 1 || m > 32) return -1;
  uint32_t mk[32];
  for (int j = 0; j < dim; ++j) {
    if (j == 0) {
      for (int k = 0; k < m; ++k) mk[k] = 1u;
    } else {
      const kb_joe_kuo_row *row = &kb_joe_kuo_rows[j - 1];
      int s = row->degree;
      for (int k = 0; k < m && k < s; ++k) mk[k] = row->m_init[k];
      for (int k = s; k < m; ++k) {
        uint32_t v = mk[k - s] ^ (mk[k - s] << s);
        for (int i = 1; i < s; ++i)
          if ((row->poly >> (s - 1 - i)) & 1u) v ^= mk[k - i] << i;
        mk[k] = v;
      }
    }
    for (int k = 0; k < m; ++k) {
      /* reverse the k+1 low bits of m_{k+1} */
      uint32_t r = 0;
      for (int b = 0; b <= k; ++b)
        if ((mk[k] >> b) & 1u) r |= 1u << (k - b);
      Cs[j * m + k] = r;
    }
  }
  return 0;
}

static uint32_t or_bitreverse32(uint32_t v) {
  uint32_t r = 0;
  for (int b = 0; b < 32; ++b)
    if ((v >> b) & 1u) r |= 1u << (31 - b);
  return r;
}

/* mt19937_64 (Matsumoto & Nishimura; the C++ <random> engine std::mt19937_64). */
typedef struct {
  uint64_t mt[312];
  int idx;
} or_mt64;

static void or_mt64_seed(or_mt64 *g, uint64_t seed) {
  g->mt[0] = seed;
  for (int i = 1; i < 312; ++i) g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
  g->idx = 312;
}

static uint64_t or_mt64_next(or_mt64 *g) {
  const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL, MATRIX_A = 0xB5026F5AA96619E9ULL;
  if (g->idx >= 312) {
    for (int i = 0; i < 312; ++i) {
      uint64_t x = (g->mt[i] & UM) | (g->mt[(i + 1) % 312] & LM);
      uint64_t xa = x >> 1;
      if (x & 1ULL) xa ^= MATRIX_A;
      g->mt[i] = g->mt[(i + 156) % 312] ^ xa;
    }
    g->idx = 0;
  }
  uint64_t x = g->mt[g->idx++];
  x ^= (x >> 29) & 0x5555555555555555ULL;
  x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
  x ^= (x << 37) & 0xFFF7EEE000000000ULL;
  x ^= x >> 43;
  return x;
}

/* Bit depth of the generating matrices (digitalseq_b2g.hpp:139-146). */
static unsigned or_bit_depth(const uint32_t *Cs, int count) {
  uint32_t mx = 0;
  for (int i = 0; i < count; ++i)
    if (Cs[i] > mx) mx = Cs[i];
  unsigned t = 31;
  while (t && !((1u << (t - 1)) & mx)) t--;
  return t;
}

/* Radical-inverse generating matrices Csr (dim x m) and shift vector shfr (dim) of
 * keldy::sobol (qrng.hpp:69-109). Unshifted: do_shift = do_scramble = 0. */
int or_sobol_setup(int dim, int m, int do_shift, int do_scramble, int seed_shift, uint32_t *Csr, uint32_t *shfr) {
  if (dim < 1 || dim > KB_SOBOL_MAX_DIM || m < 1 || m > 31) return -1;
  uint32_t *Cs = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)dim * (size_t)m);
  uint32_t *shifts = (uint32_t *)calloc((size_t)dim, sizeof(uint32_t));
  if (!Cs || !shifts) return -2;
  or_sobol_matrices(dim, m, Cs);
  if (do_shift || do_scramble) {
    /* std::generate_n and generate_random_linear_scramble both take the engine by
     * value, so both start from the freshly seeded state (qrng.hpp:95-103). */
    or_mt64 g;
    or_mt64_seed(&g, (uint64_t)(int64_t)seed_shift);
    for (int j = 0; j < dim; ++j) shifts[j] = (uint32_t)or_mt64_next(&g);
    if (!do_shift) memset(shifts, 0, sizeof(uint32_t) * (size_t)dim);
    if (do_scramble) {
      unsigned t = or_bit_depth(Cs, dim * m), t2 = t;
      uint32_t *M = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)dim * t);
      uint32_t *Cout = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)dim * (size_t)m);
      or_mt64 g2;
      or_mt64_seed(&g2, (uint64_t)(int64_t)seed_shift);
      for (int j = 0; j < dim; ++j)
        for (unsigned k = 0; k < t; ++k) {
          uint64_t r = or_mt64_next(&g2);
          uint32_t top = (uint32_t)1u << (t2 - k - 1);
          r &= (uint64_t)((top - 1u) | top);
          r |= 1u;
          r <<= k;
          M[j * t + k] = (uint32_t)r;
        }
      for (int j = 0; j < dim; ++j)
        for (int k = 0; k < m; ++k) {
          uint32_t c = 0;
          for (unsigned i = 0; i < t; ++i)
            if ((Cs[j * m + k] >> i) & 1u) c ^= M[j * t + i];
          Cout[j * m + k] = c;
        }
      memcpy(Cs, Cout, sizeof(uint32_t) * (size_t)dim * (size_t)m);
      free(M);
      free(Cout);
    }
  }
  for (int i = 0; i < dim * m; ++i) Csr[i] = or_bitreverse32(Cs[i]);
  for (int j = 0; j < dim; ++j) shfr[j] = or_bitreverse32(shifts[j]);
  free(Cs);
  free(shifts);
  return 0;
}

/* Points number k_first .. k_first+count-1 of the sequence, k >= 1 (the point that
 * digitalseq_b2g::next() returns after its counter became k). The keldy::sobol wrapper
 * constructed with seed s returns k = s+1, s+2, ... (qrng.hpp:51-58, 69-75). Each point
 * is advanced by the Gray-code step of next() from the state set_state(k_first - 1). */
int or_sobol_points(int dim, int m, const uint32_t *Csr, const uint32_t *shfr, uint32_t k_first, int64_t count,
                    double *out) {
  if (k_first < 1) return -1;
  uint32_t cur[KB_SOBOL_MAX_DIM];
  const double recipd = 1.0 / 4294967296.0;
  uint32_t k = k_first - 1;
  uint32_t gk = (k >> 1) ^ k;
  for (int j = 0; j < dim; ++j) {
    cur[j] = 0;
    for (int i = 0; i < m; ++i)
      if ((1u << i) & gk) cur[j] ^= Csr[j * m + i];
  }
  for (int64_t p = 0; p < count; ++p) {
    k += 1;
    unsigned c = 0;
    while (c < 32 && !((k >> c) & 1u)) ++c;
    c %= (unsigned)m;
    for (int j = 0; j < dim; ++j) {
      cur[j] ^= Csr[j * m + c];
      out[p * dim + j] = recipd * (double)(cur[j] ^ shfr[j]);
    }
  }
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Warpers                                                                    */
/* ------------------------------------------------------------------------- */
enum {
  OR_W_IDENTITY = 0,
  OR_W_PLASMA_UV = 1,
  OR_W_EXPONENTIAL = 2,
  OR_W_INVERSE = 3,
  OR_W_INVERSE_SQUARE = 4,
  OR_W_INVERSE_POWER = 5,
  OR_W_UNIFORM = 6,
};

typedef struct {
  int kind;
  int power;
  double u_max; /* domain_u_max, or t_max for the plasma warper */
  double w;     /* w_scale */
} or_warper;

/* f1, f1_integrated, f1_integrated_inverse of the analytic product makers
 * (product_1d_simple.hpp:560-630; the norms are long double there as here). */
static double or_f1(const or_warper *w, double t) {
  switch (w->kind) {
  case OR_W_EXPONENTIAL: {
    long double norm = -expm1l(-(long double)w->u_max / w->w);
    return (double)((long double)exp(-t / w->w) / ((long double)w->w * norm));
  }
  case OR_W_INVERSE: {
    long double norm = log1pl((long double)w->u_max / w->w);
    return (double)(1.0L / (norm * (long double)(w->w + t)));
  }
  case OR_W_INVERSE_SQUARE: {
    long double norm = (long double)w->u_max / (w->w + w->u_max);
    return (double)((long double)w->w / ((long double)((w->w + t) * (w->w + t)) * norm));
  }
  case OR_W_INVERSE_POWER: {
    int p = w->power;
    long double u_max = w->u_max;
    long double norm = (p - 1) * powl(u_max + w->w, p - 1) / (powl(u_max / w->w + 1, p - 1) - 1);
    return (double)(norm / (long double)pow(w->w + t, p));
  }
  case OR_W_UNIFORM:
    return 1.0 / w->u_max;
  default:
    return 1.0;
  }
}

static double or_f1_integrated(const or_warper *w, double t) {
  switch (w->kind) {
  case OR_W_EXPONENTIAL:
    return expm1((w->u_max - t) / w->w) / expm1(w->u_max / w->w);
  case OR_W_INVERSE: {
    long double norm = log1pl((long double)w->u_max / w->w);
    return (double)((long double)log1p(t / w->w) / norm);
  }
  case OR_W_INVERSE_SQUARE: {
    long double norm = (long double)w->u_max / (w->w + w->u_max);
    return (double)((long double)t / ((long double)(w->w + t) * norm));
  }
  case OR_W_INVERSE_POWER: {
    int p = w->power;
    long double u_max = w->u_max;
    long double norm = powl(u_max + w->w, p - 1) / (powl(u_max / w->w + 1, p - 1) - 1);
    return (double)(norm * (long double)(pow(t / w->w + 1, p - 1) - 1) / (long double)pow(t + w->w, p - 1));
  }
  case OR_W_UNIFORM:
    return t / w->u_max;
  default:
    return t;
  }
}

static double or_f1_integrated_inverse(const or_warper *w, double l) {
  switch (w->kind) {
  case OR_W_EXPONENTIAL:
    return w->u_max - w->w * log1p(expm1(w->u_max / w->w) * l);
  case OR_W_INVERSE: {
    long double norm = log1pl((long double)w->u_max / w->w);
    return (double)((long double)w->w * expm1l((long double)l * norm));
  }
  case OR_W_INVERSE_SQUARE: {
    long double norm = (long double)w->u_max / (w->w + w->u_max);
    return (double)(norm * l * w->w / (1.0L - norm * l));
  }
  case OR_W_INVERSE_POWER: {
    int p = w->power;
    long double u_max = w->u_max;
    long double denom = powl(1 + l * (powl(w->w / (u_max + w->w), p - 1) - 1), 1.0L / (p - 1.0));
    return (double)((long double)w->w * (1 - denom) / denom);
  }
  case OR_W_UNIFORM:
    return w->u_max * l;
  default:
    return l;
  }
}

/* One warper's map_reverse (l -> u, Jacobian) on a vector of n coordinates. */
static void or_warper_reverse(const or_warper *w, int n, double *x, double *jac) {
  switch (w->kind) {
  case OR_W_IDENTITY:
    return;
  case OR_W_PLASMA_UV: {
    /* ui_from_vi (plasma_uv.hpp:46-51): u0 = t_max - v0, then a running difference */
    if (n == 0) return;
    x[0] = w->u_max - x[0];
    for (int i = 1; i < n; ++i) x[i] = x[i - 1] - x[i];
    return;
  }
  default: {
    /* product_1d_simple.hpp:109-117 */
    double j = 1.0;
    for (int i = 0; i < n; ++i) {
      x[i] = or_f1_integrated_inverse(w, x[i]);
      j *= 1.0 / or_f1(w, x[i]);
    }
    *jac *= j;
  }
  }
}

static int or_cmp_desc(const void *a, const void *b) {
  double x = *(const double *)a, y = *(const double *)b;
  return (x < y) - (x > y);
}

/* One warper's map_forward (u -> l, Jacobian). */
static void or_warper_forward(const or_warper *w, int n, double *x, double *jac) {
  switch (w->kind) {
  case OR_W_IDENTITY:
    return;
  case OR_W_PLASMA_UV: {
    /* vi_from_ui (plasma_uv.hpp:35-44): sort descending, consecutive differences */
    if (n == 0) return;
    qsort(x, (size_t)n, sizeof(double), or_cmp_desc);
    for (int i = n - 1; i > 0; i--) x[i] = x[i - 1] - x[i];
    x[0] = w->u_max - x[0];
    return;
  }
  default: {
    /* product_1d_simple.hpp:119-127 */
    double j = 1.0;
    for (int i = 0; i < n; ++i) {
      j *= or_f1(w, x[i]);
      x[i] = or_f1_integrated(w, x[i]);
    }
    *jac *= j;
  }
  }
}

/* warper_train_t::map_reverse(li, start, end) (warpers.hpp:72-85): warpers
 * start-1 down to end, i.e. the last warper first. */
int or_map_reverse(const or_warper *chain, int len, int start, int end, int n, const double *li, double *ui,
                   double *jac) {
  if (start < 0 || start > len || end < 0 || end > start) return -1;
  memcpy(ui, li, sizeof(double) * (size_t)n);
  double j = 1.0;
  for (int i = start - 1; i >= end; --i) {
    double jw = 1.0;
    or_warper_reverse(&chain[i], n, ui, &jw);
    j *= jw;
  }
  *jac = j;
  return 0;
}

/* warper_train_t::map_forward(ui, start, end) (warpers.hpp:88-101). */
int or_map_forward(const or_warper *chain, int len, int start, int end, int n, const double *ui, double *li,
                   double *jac) {
  if (start < 0 || end > len || start > end) return -1;
  memcpy(li, ui, sizeof(double) * (size_t)n);
  double j = 1.0;
  for (int i = start; i < end; ++i) {
    double jw = 1.0;
    or_warper_forward(&chain[i], n, li, &jw);
    j *= jw;
  }
  *jac = j;
  return 0;
}

/* ------------------------------------------------------------------------- */
/* g0 model and Keldysh-contour adaptor                                       */
/* ------------------------------------------------------------------------- */

/* Tabulated g^<(t), g^>(t) on the uniform mesh t_i = -time_max + i*delta,
 * i = 0..npts-1, delta = 2 time_max/(npts-1); complex values interleaved (re, im).
 * tab[spin][o1][o2][0 = lesser, 1 = greater]; a NULL entry is an all-zero block. */
typedef struct {
  int npts;
  double time_max;
  double alpha;
  const double *tab[2][2][2][2];
  int interp; /* 3: cubic (4-point Lagrange, an extension with no keldy counterpart); else linear */
} or_model;

typedef struct {
  double time;
  int spin;
  int k_idx;
  int timesplit;
  int orbital;
} or_gf_index;

/* compare_3way (common.cpp:47-57) */
int or_compare_3way(double ta, int ka, int sa, double tb, int kb, int sb) {
  int k3 = ka - kb;
  if (k3 != 0) return k3;
  double d = ta - tb;
  if (d != 0.0) return (1 - 2 * ka) * (2 * (!signbit(d)) - 1);
  return (1 - 2 * ka) * (sa - sb);
}

/* Linear (or, interp = 3, cubic) interpolation on the uniform mesh. Returns -1 outside
 * [-time_max, time_max]. */
static int or_interp(const or_model *mdl, const double *tab, double x, cplx *out) {
  if (!tab) {
    *out = c_make(0.0, 0.0);
    return 0;
  }
  double xmin = -mdl->time_max;
  double delta = (mdl->time_max - xmin) / (double)(mdl->npts - 1);
  double a = (x - xmin) / delta;
  double fi = floor(a);
  long i = (long)fi;
  if (i == mdl->npts - 1) i = mdl->npts - 2;
  if (i < 0 || i > mdl->npts - 2) return -1;
  double w = a - (double)i;
  if (mdl->interp == 3) {
    /* cubic Lagrange interpolation through the 4 mesh points s0..s0+3 around the interval
     * [i, i+1] (s0 = i-1, moved inside the mesh at its ends), evaluated at u = x/delta - s0 */
    long s0 = i - 1;
    if (s0 < 0) s0 = 0;
    if (s0 > mdl->npts - 4) s0 = mdl->npts - 4;
    double u = (double)(i - s0) + w;
    double am = u - 1.0, bm = u - 2.0, cm = u - 3.0;
    double L[4];
    L[0] = -((am * bm) * cm) / 6.0;
    L[1] = ((u * bm) * cm) / 2.0;
    L[2] = -((u * am) * cm) / 2.0;
    L[3] = ((u * am) * bm) / 6.0;
    double re = 0.0, im = 0.0;
    for (int k = 0; k < 4; ++k) {
      re = re + L[k] * tab[2 * (s0 + k)];
      im = im + L[k] * tab[2 * (s0 + k) + 1];
    }
    *out = c_make(re, im);
    return 0;
  }
  cplx g0 = c_make(tab[2 * i], tab[2 * i + 1]);
  cplx g1 = c_make(tab[2 * i + 2], tab[2 * i + 3]);
  *out = c_add(c_scale(g0, 1.0 - w), c_scale(g1, w));
  return 0;
}

/* g0_keldysh_contour_t::operator() (model.hpp:244-265) */
int or_g0(const or_model *mdl, const or_gf_index *a, const or_gf_index *b, int internal, double *out) {
  cplx r = c_make(0.0, 0.0);
  int st = 0;
  if (a->spin == b->spin) {
    int ord = or_compare_3way(a->time, a->k_idx, a->timesplit, b->time, b->k_idx, b->timesplit);
    const double *const *blk = mdl->tab[a->spin][a->orbital][b->orbital];
    if (ord > 0)
      st = or_interp(mdl, blk[1], a->time - b->time, &r);
    else if (ord < 0)
      st = or_interp(mdl, blk[0], a->time - b->time, &r);
    else if (a->orbital != b->orbital)
      st = or_interp(mdl, blk[0], 0.0, &r);
    else {
      st = or_interp(mdl, mdl->tab[a->spin][a->orbital][a->orbital][0], 0.0, &r);
      r = c_sub(r, c_make(0.0, (double)internal * mdl->alpha));
    }
  }
  out[0] = r.re;
  out[1] = r.im;
  return st;
}

static cplx or_g0c(const or_model *mdl, const or_gf_index *a, const or_gf_index *b, int internal, int *err) {
  double v[2];
  if (or_g0(mdl, a, b, internal, v) != 0) *err = 1;
  return c_make(v[0], v[1]);
}

/* ------------------------------------------------------------------------- */
/* Determinant: partial-pivot LU in the order of LAPACK zgetf2.               */
/* ------------------------------------------------------------------------- */
static cplx or_det(cplx *A, int n) {
  cplx det = c_make(1.0, 0.0);
  int swaps = 0;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = c_abs1(A[k * n + k]);
    for (int i = k + 1; i < n; ++i) {
      double v = c_abs1(A[i * n + k]);
      if (v > best) {
        best = v;
        p = i;
      }
    }
    if (best == 0.0) return c_make(0.0, 0.0);
    if (p != k) {
      for (int j = 0; j < n; ++j) {
        cplx t = A[k * n + j];
        A[k * n + j] = A[p * n + j];
        A[p * n + j] = t;
      }
      swaps++;
    }
    cplx piv = A[k * n + k];
    det = c_mul(det, piv);
    cplx inv = c_div(c_make(1.0, 0.0), piv);
    for (int i = k + 1; i < n; ++i) A[i * n + k] = c_mul(A[i * n + k], inv);
    for (int i = k + 1; i < n; ++i) {
      cplx l = A[i * n + k];
      for (int j = k + 1; j < n; ++j) A[i * n + j] = c_sub(A[i * n + j], c_mul(l, A[k * n + j]));
    }
  }
  return (swaps & 1) ? c_make(-det.re, -det.im) : det;
}

/* integrand_g_direct::operator() (wick_direct.cpp:43-158).
 * out[0..1] = integrand, *in_domain, *scale = sum over Keldysh configurations of
 * |det(s1) det(s2)| (the natural error scale of the alternating sum).
 * Returns 0, or -1 if a g0 evaluation left the tabulated window. */
int or_integrand(const or_model *mdl, const or_gf_index *A, const or_gf_index *B, double cutoff, int n,
                 const double *times, int keep_u_hypercube, double *out, int *in_domain, double *scale) {
  int err = 0;
  out[0] = out[1] = 0.0;
  *scale = 0.0;
  *in_domain = 0;
  if (A->spin != B->spin) return 0;
  if (keep_u_hypercube)
    for (int i = 0; i < n; ++i)
      if (times[i] < 0.0) return 0;
  or_gf_index a = *A, b = *B;
  a.timesplit = n;
  b.timesplit = n;
  if (n == 0) {
    cplx v = or_g0c(mdl, &a, &b, 0, &err);
    out[0] = v.re;
    out[1] = v.im;
    *scale = c_abs(v);
    *in_domain = 1;
    return err ? -1 : 0;
  }
  int N1 = 2 * n + 1, N2 = 2 * n;
  cplx *s1 = (cplx *)malloc(sizeof(cplx) * (size_t)(N1 * N1));
  cplx *s2 = (cplx *)malloc(sizeof(cplx) * (size_t)(N2 * N2));
  cplx *t1 = (cplx *)malloc(sizeof(cplx) * (size_t)((n + 1) * (n + 1)));
  cplx *t2 = (cplx *)malloc(sizeof(cplx) * (size_t)(n * n));
  or_gf_index *c1 = (or_gf_index *)malloc(sizeof(or_gf_index) * (size_t)N2);
  or_gf_index *c2 = (or_gf_index *)malloc(sizeof(or_gf_index) * (size_t)N2);
  for (int i = 0; i < n; ++i) {
    or_gf_index p = {times[i], a.spin, 0, i, 0};
    c1[i] = p;
    p.k_idx = 1;
    c1[i + n] = p;
    or_gf_index q = {times[i], 1 - a.spin, 0, i, 0};
    c2[i] = q;
    q.k_idx = 1;
    c2[i + n] = q;
  }
  int ext = 2 * n;
  s1[ext * N1 + ext] = or_g0c(mdl, &a, &b, 0, &err);
  for (int i = 0; i < N2; ++i) {
    s1[ext * N1 + i] = or_g0c(mdl, &a, &c1[i], 1, &err);
    s1[i * N1 + ext] = or_g0c(mdl, &c1[i], &b, 1, &err);
    for (int j = 0; j < N2; ++j) {
      s1[i * N1 + j] = or_g0c(mdl, &c1[i], &c1[j], 1, &err);
      s2[i * N2 + j] = or_g0c(mdl, &c2[i], &c2[j], 1, &err);
    }
  }
  cplx acc = c_make(0.0, 0.0);
  double sc = 0.0;
  int pick[64];
  uint64_t nconf = (uint64_t)1 << n;
  for (uint64_t kel = 0; kel < nconf; ++kel) {
    for (int i = 0; i < n; ++i) pick[i] = i + (int)((kel >> i) & 1u) * n;
    pick[n] = ext;
    for (int i = 0; i <= n; ++i)
      for (int j = 0; j <= n; ++j) t1[i * (n + 1) + j] = s1[pick[i] * N1 + pick[j]];
    t1[n * (n + 1) + n] = c_make(0.0, 0.0);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) t2[i * n + j] = s2[pick[i] * N2 + pick[j]];
    cplx d = c_mul(or_det(t1, n + 1), or_det(t2, n));
    int parity = 1 - 2 * __builtin_parityll(kel);
    acc = c_add(acc, c_scale(d, (double)parity));
    sc += c_abs(d);
  }
  if (c_abs(acc) < cutoff) acc = c_make(0.0, 0.0);
  out[0] = acc.re;
  out[1] = acc.im;
  *scale = sc;
  *in_domain = 1;
  free(s1);
  free(s2);
  free(t1);
  free(t2);
  free(c1);
  free(c2);
  return err ? -1 : 0;
}

/* integrand_g_direct::eval_no_det (wick_direct.cpp:161-228): closed-form connected
 * Wick sums at orders 1 and 2. Returns -2 for other orders. */
int or_integrand_no_det(const or_model *mdl, const or_gf_index *A, const or_gf_index *B, double cutoff, int n,
                        const double *times, int keep_u_hypercube, double *out, int *in_domain) {
  int err = 0;
  out[0] = out[1] = 0.0;
  *in_domain = 0;
  if (A->spin != B->spin) return 0;
  if (keep_u_hypercube)
    for (int i = 0; i < n; ++i)
      if (times[i] < 0.0) return 0;
  or_gf_index a = *A, b = *B;
  a.timesplit = n;
  b.timesplit = n;
  cplx acc = c_make(0.0, 0.0);
  if (n == 0) {
    acc = or_g0c(mdl, &a, &b, 0, &err);
  } else if (n == 1) {
    for (int k0 = 0; k0 < 2; ++k0) {
      or_gf_index pu = {times[0], 0, k0, 0, 0}, pd = {times[0], 1, k0, 0, 0};
      int sign = (k0 == 0) ? 1 : -1;
      cplx t = c_mul(c_mul(or_g0c(mdl, &pd, &pd, 1, &err), or_g0c(mdl, &a, &pu, 1, &err)),
                     or_g0c(mdl, &pu, &b, 1, &err));
      acc = c_add(acc, c_scale(t, (double)(-sign)));
    }
  } else if (n == 2) {
    for (int k0 = 0; k0 < 2; ++k0)
      for (int k1 = 0; k1 < 2; ++k1) {
        or_gf_index u0 = {times[0], 0, k0, 0, 0}, u1 = {times[1], 0, k1, 1, 0};
        or_gf_index d0 = {times[0], 1, k0, 0, 0}, d1 = {times[1], 1, k1, 1, 0};
        int sign = (((k0 + k1) % 2) == 0) ? 1 : -1;
        cplx x1 = c_add(c_mul(c_mul(or_g0c(mdl, &u0, &u0, 1, &err), or_g0c(mdl, &a, &u1, 1, &err)),
                              or_g0c(mdl, &u1, &b, 1, &err)),
                        c_mul(c_mul(or_g0c(mdl, &a, &u0, 1, &err), or_g0c(mdl, &u1, &u1, 1, &err)),
                              or_g0c(mdl, &u0, &b, 1, &err)));
        cplx y1 = c_mul(or_g0c(mdl, &d1, &d0, 1, &err), or_g0c(mdl, &d0, &d1, 1, &err));
        acc = c_add(acc, c_scale(c_mul(x1, y1), (double)sign));
        cplx x2 = c_add(c_mul(c_mul(or_g0c(mdl, &a, &u0, 1, &err), or_g0c(mdl, &u0, &u1, 1, &err)),
                              or_g0c(mdl, &u1, &b, 1, &err)),
                        c_mul(c_mul(or_g0c(mdl, &u1, &u0, 1, &err), or_g0c(mdl, &a, &u1, 1, &err)),
                              or_g0c(mdl, &u0, &b, 1, &err)));
        cplx y2 = c_sub(c_mul(or_g0c(mdl, &d0, &d0, 1, &err), or_g0c(mdl, &d1, &d1, 1, &err)),
                        c_mul(or_g0c(mdl, &d1, &d0, 1, &err), or_g0c(mdl, &d0, &d1, 1, &err)));
        acc = c_add(acc, c_scale(c_mul(x2, y2), (double)sign));
      }
  } else {
    return -2;
  }
  if (c_abs(acc) < cutoff) acc = c_make(0.0, 0.0);
  out[0] = acc.re;
  out[1] = acc.im;
  *in_domain = 1;
  return err ? -1 : 0;
}

/* ------------------------------------------------------------------------- */
/* Integrator                                                                 */
/* ------------------------------------------------------------------------- */

/* evaluate_warped_integrand (integrator.hpp:68-79): out[0..1] = f(warp(li)) * J,
 * out[2] = J, *in_domain, *scale = integrand scale * |J|. */
int or_evaluate_warped(const or_model *mdl, const or_gf_index *A, const or_gf_index *B, double cutoff,
                       const or_warper *chain, int len, int n, const double *li, double *out, int *in_domain,
                       double *scale) {
  double ui[64];
  double jac = 1.0;
  or_map_reverse(chain, len, len, 0, n, li, ui, &jac);
  double f[2];
  int st = or_integrand(mdl, A, B, cutoff, n, ui, 1, f, in_domain, scale);
  out[0] = f[0] * jac;
  out[1] = f[1] * jac;
  out[2] = jac;
  *scale *= fabs(jac);
  return st;
}

/* integrator::run (integrator.hpp:81-95) on one rank of `world` ranks, drawing
 * Sobol points k_first, k_first+1, ... (k_first = seed + 1 for a fresh generator)
 * and keeping point i when i % world == rank. result[0..1] = sum of f*J,
 * result[2] = points run, result[3] = points in domain, result[4] = sum of the
 * per-point scales (for tolerances). */
int or_integrate(const or_model *mdl, const or_gf_index *A, const or_gf_index *B, double cutoff,
                 const or_warper *chain, int len, int n, const uint32_t *Csr, const uint32_t *shfr, int m,
                 uint32_t k_first, int64_t nr_steps, int rank, int world, double *result) {
  double li[64], v[3], sc;
  int dom;
  double sre = 0.0, sim = 0.0, ssc = 0.0;
  uint64_t npts = 0, ndom = 0;
  int st = 0;
  for (int64_t i = 0; i < nr_steps; ++i) {
    or_sobol_points(n, m, Csr, shfr, k_first + (uint32_t)i, 1, li);
    if (i % world != rank) continue;
    if (or_evaluate_warped(mdl, A, B, cutoff, chain, len, n, li, v, &dom, &sc) != 0) st = -1;
    sre += v[0];
    sim += v[1];
    ssc += sc;
    npts++;
    ndom += (uint64_t)dom;
  }
  result[0] = sre;
  result[1] = sim;
  result[2] = (double)npts;
  result[3] = (double)ndom;
  result[4] = ssc;
  return st;
}

/* integrator<binner_t<1>, integrand_g_direct_time>::run: as or_integrate, each point's
 * f*J also added to the bin of its earliest warped vertex time
 * (wick_direct_time.cpp:55, 160; binner_t<1>(xmin, xmax, nbins), binner.hpp:163-176,
 * 241-260: in_bounds xmin <= x <= xmax, index (x - xmin) / bin_size truncated, x == xmax
 * in the last bin, out-of-bounds values counted as dropped). Out-of-domain points add 0.
 * bins[2 * nbins] (complex sums), counts[nbins], *dropped: added to. */
int or_integrate_binned(const or_model *mdl, const or_gf_index *A, const or_gf_index *B, double cutoff,
                        const or_warper *chain, int len, int n, const uint32_t *Csr, const uint32_t *shfr, int m,
                        uint32_t k_first, int64_t nr_steps, int nbins, double xmin, double xmax, double *result,
                        double *bins, double *counts, double *dropped) {
  double li[64], ui[64], v[3], sc, jac;
  int dom;
  const double bin_size = (xmax - xmin) / nbins;
  double sre = 0.0, sim = 0.0, ssc = 0.0;
  uint64_t npts = 0, ndom = 0;
  int st = 0;
  for (int64_t i = 0; i < nr_steps; ++i) {
    or_sobol_points(n, m, Csr, shfr, k_first + (uint32_t)i, 1, li);
    if (or_evaluate_warped(mdl, A, B, cutoff, chain, len, n, li, v, &dom, &sc) != 0) st = -1;
    jac = 1.0;
    or_map_reverse(chain, len, len, 0, n, li, ui, &jac);
    double t = ui[0];
    for (int j = 1; j < n; ++j)
      if (ui[j] < t) t = ui[j];
    if (xmin <= t && t <= xmax) {
      int b = (t == xmax) ? nbins - 1 : (int)((t - xmin) / bin_size);
      if (b > nbins - 1) b = nbins - 1;
      bins[2 * b] += v[0];
      bins[2 * b + 1] += v[1];
      counts[b] += 1.0;
    } else {
      *dropped += 1.0;
    }
    sre += v[0];
    sim += v[1];
    ssc += sc;
    npts++;
    ndom += (uint64_t)dom;
  }
  result[0] = sre;
  result[1] = sim;
  result[2] = (double)npts;
  result[3] = (double)ndom;
  result[4] = ssc;
  return st;
}

/* first_row_expansion (det_expansion.hpp:44-74): LU with partial pivoting (zgetrf: pivot =
 * first maximum of |re|+|im|, multipliers from the pivot's reciprocal), det(a) from the
 * diagonal and the interchanges, then zgetrs on b = det(a) e_0: row interchanges, unit
 * lower and upper triangular solves. x = the first row of a's cofactor matrix. */
static void or_first_row_expansion(cplx *a, int m, cplx *x) {
  int piv[64];
  cplx det = c_make(1.0, 0.0);
  int neg = 0;
  for (int k = 0; k < m; ++k) {
    int p = k;
    double best = c_abs1(a[k * m + k]);
    for (int i = k + 1; i < m; ++i)
      if (c_abs1(a[i * m + k]) > best) {
        best = c_abs1(a[i * m + k]);
        p = i;
      }
    piv[k] = p;
    if (p != k) {
      for (int j = 0; j < m; ++j) {
        cplx t = a[k * m + j];
        a[k * m + j] = a[p * m + j];
        a[p * m + j] = t;
      }
      neg = !neg;
    }
    det = c_mul(det, a[k * m + k]);
    if (best == 0.0) continue;
    cplx inv = c_div(c_make(1.0, 0.0), a[k * m + k]);
    for (int i = k + 1; i < m; ++i) {
      cplx l = c_mul(a[i * m + k], inv);
      a[i * m + k] = l;
      for (int j = k + 1; j < m; ++j) a[i * m + j] = c_sub(a[i * m + j], c_mul(l, a[k * m + j]));
    }
  }
  if (neg) det = c_scale(det, -1.0);
  for (int i = 0; i < m; ++i) x[i] = c_make(0.0, 0.0);
  x[0] = det;
  for (int k = 0; k < m; ++k)
    if (piv[k] != k) {
      cplx t = x[k];
      x[k] = x[piv[k]];
      x[piv[k]] = t;
    }
  for (int i = 1; i < m; ++i)
    for (int j = 0; j < i; ++j) x[i] = c_sub(x[i], c_mul(a[i * m + j], x[j]));
  for (int i = m - 1; i >= 0; --i) {
    for (int j = i + 1; j < m; ++j) x[i] = c_sub(x[i], c_mul(a[i * m + j], x[j]));
    x[i] = c_div(x[i], a[i * m + i]);
  }
}

/* integrand_g_kernel::operator() (impurity_oneband/wick_kernel.cpp:42-138) for one point:
 * out[2 * (2 i + k)], out[2 * (2 i + k) + 1] = the sum over the Keldysh configurations with
 * a_i = k of vertex i's term x_{i+1} (-1)^|a| det(s2_a) (keldy accumulates each term at
 * (u_i, a_i)); *scale = sum of the terms' moduli. X's timesplit is set to n. */
int or_integrand_kernel(const or_model *mdl, const or_gf_index *X, int n, const double *times, int keep_u_hypercube,
                        double *out, int *in_domain, double *scale) {
  int err = 0;
  for (int q = 0; q < 4 * n; ++q) out[q] = 0.0;
  *scale = 0.0;
  *in_domain = 0;
  if (keep_u_hypercube)
    for (int i = 0; i < n; ++i)
      if (times[i] < 0.0) return 0;
  or_gf_index a = *X;
  a.timesplit = n;
  int N1 = 2 * n + 1, N2 = 2 * n;
  cplx *s1 = (cplx *)malloc(sizeof(cplx) * (size_t)(N1 * N1));
  cplx *s2 = (cplx *)malloc(sizeof(cplx) * (size_t)(N2 * N2));
  cplx *t1 = (cplx *)malloc(sizeof(cplx) * (size_t)((n + 1) * (n + 1)));
  cplx *t2 = (cplx *)malloc(sizeof(cplx) * (size_t)(n * n));
  cplx *x = (cplx *)malloc(sizeof(cplx) * (size_t)(n + 1));
  or_gf_index *c1 = (or_gf_index *)malloc(sizeof(or_gf_index) * (size_t)N2);
  or_gf_index *c2 = (or_gf_index *)malloc(sizeof(or_gf_index) * (size_t)N2);
  for (int i = 0; i < n; ++i) {
    or_gf_index p = {times[i], a.spin, 0, i, 0};
    c1[i] = p;
    p.k_idx = 1;
    c1[i + n] = p;
    or_gf_index q = {times[i], 1 - a.spin, 0, i, 0};
    c2[i] = q;
    q.k_idx = 1;
    c2[i + n] = q;
  }
  int ext = 2 * n;
  s1[ext * N1 + ext] = or_g0c(mdl, &a, &a, 0, &err);
  for (int i = 0; i < N2; ++i) {
    s1[ext * N1 + i] = or_g0c(mdl, &a, &c1[i], 1, &err);
    s1[i * N1 + ext] = or_g0c(mdl, &c1[i], &a, 1, &err);
    for (int j = 0; j < N2; ++j) {
      s1[i * N1 + j] = or_g0c(mdl, &c1[i], &c1[j], 1, &err);
      s2[i * N2 + j] = or_g0c(mdl, &c2[i], &c2[j], 1, &err);
    }
  }
  int pick[65];
  uint64_t nconf = (uint64_t)1 << n;
  for (uint64_t kel = 0; kel < nconf; ++kel) {
    pick[0] = ext;
    for (int i = 0; i < n; ++i) pick[i + 1] = i + (int)((kel >> i) & 1u) * n;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) t2[i * n + j] = s2[pick[i + 1] * N2 + pick[j + 1]];
    for (int i = 0; i <= n; ++i)
      for (int j = 0; j <= n; ++j) t1[i * (n + 1) + j] = s1[pick[i] * N1 + pick[j]];
    t1[n * (n + 1) + n] = c_make(0.0, 0.0); /* wick_kernel.cpp:121 */
    or_first_row_expansion(t1, n + 1, x);
    cplx d2 = or_det(t2, n);
    if (__builtin_parityll(kel)) d2 = c_scale(d2, -1.0);
    for (int i = 0; i < n; ++i) {
      cplx v = c_mul(x[i + 1], d2);
      int k = (int)((kel >> i) & 1u);
      out[2 * (2 * i + k)] += v.re;
      out[2 * (2 * i + k) + 1] += v.im;
      *scale += c_abs(v);
    }
  }
  free(s1);
  free(s2);
  free(t1);
  free(t2);
  free(x);
  free(c1);
  free(c2);
  *in_domain = 1;
  return err ? -1 : 0;
}

/* integrator<binner_t<1, 1>, integrand_g_kernel>::run (integrator.hpp:81-95): Sobol points
 * k_first.., chain, per point the terms times the Jacobian into bins[nbins][2] (complex,
 * (time bin, Keldysh index)), counts[nbins][2] (values added, 2^(n-1) per (vertex, index)),
 * *dropped; result[0..1] = sum of all terms, [2] points, [3] in domain, [4] sum of moduli. */
int or_integrate_kernel(const or_model *mdl, const or_gf_index *X, const or_warper *chain, int len, int n,
                        const uint32_t *Csr, const uint32_t *shfr, int m, uint32_t k_first, int64_t nr_steps, int nbins,
                        double xmin, double xmax, double *result, double *bins, double *counts, double *dropped) {
  double li[64], ui[64], out[256], jac, sc;
  int dom;
  const double bin_size = (xmax - xmin) / nbins;
  double sre = 0.0, sim = 0.0, ssc = 0.0;
  uint64_t npts = 0, ndom = 0;
  int st = 0;
  for (int64_t s = 0; s < nr_steps; ++s) {
    or_sobol_points(n, m, Csr, shfr, k_first + (uint32_t)s, 1, li);
    jac = 1.0;
    or_map_reverse(chain, len, len, 0, n, li, ui, &jac);
    if (or_integrand_kernel(mdl, X, n, ui, 1, out, &dom, &sc) != 0) st = -1;
    npts++;
    if (!dom) continue;
    ndom++;
    ssc += sc * fabs(jac);
    for (int i = 0; i < n; ++i) {
      double t = ui[i];
      int b = -1;
      if (xmin <= t && t <= xmax) {
        b = (t == xmax) ? nbins - 1 : (int)((t - xmin) / bin_size);
        if (b > nbins - 1) b = nbins - 1;
      }
      for (int k = 0; k < 2; ++k) {
        double vr = out[2 * (2 * i + k)] * jac, vi = out[2 * (2 * i + k) + 1] * jac;
        sre += vr;
        sim += vi;
        if (b < 0) {
          *dropped += (double)((uint64_t)1 << (n - 1));
        } else {
          bins[2 * (2 * b + k)] += vr;
          bins[2 * (2 * b + k) + 1] += vi;
          counts[2 * b + k] += (double)((uint64_t)1 << (n - 1));
        }
      }
    }
  }
  result[0] = sre;
  result[1] = sim;
  result[2] = (double)npts;
  result[3] = (double)ndom;
  result[4] = ssc;
  return st;
}
