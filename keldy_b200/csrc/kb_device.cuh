// Device building blocks of the QMC pipeline: complex arithmetic, g0 lookup on the
// Keldysh contour, Sobol points and the warper chain.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <math_constants.h>

#include "kb_types.h"

namespace kb {

// ------------------------------------------------------------------ complex
__device__ __forceinline__ double2 c2(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return c2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return c2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// c - a*b with four fused multiply-adds
__device__ __forceinline__ double2 cfms(double2 c, double2 a, double2 b) {
  return c2(fma(-a.x, b.x, fma(a.y, b.y, c.x)), fma(-a.x, b.y, fma(-a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 crcp(double2 a) {
  double r = 1.0 / fma(a.x, a.x, a.y * a.y);
  return c2(a.x * r, -a.y * r);
}
__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }
__device__ __forceinline__ double cabs(double2 a) { return hypot(a.x, a.y); }

// --------------------------------------------------------------- g0 lookup
// Linear interpolation on the uniform mesh [xmin, xmin + (npts-1) delta], the last
// interval closed at the right end. Every product and sum is rounded separately
// (no contraction), so the values equal the CPU oracle's bit for bit.
// Returns false outside the tabulated window.
__device__ __forceinline__ bool interp_index(const ModelDev &m, double x, int &i, double &w) {
  double a = __ddiv_rn(__dsub_rn(x, m.xmin), m.delta);
  double fi = floor(a);
  if (!(fi >= 0.0) || fi > (double)(m.npts - 1)) return false;
  i = (int)fi;
  if (i == m.npts - 1) i = m.npts - 2;
  w = __dsub_rn(a, (double)i);
  return true;
}

// g^<(x) and g^>(x) of one table (interleaved lesser/greater per mesh point): mesh points
// i and i + 1 as two 32-byte read-only loads (the tables are cudaMalloc'd, so 256-byte
// aligned, and a mesh point's pair starts on a 32-byte boundary). The loads are volatile
// so that they are never hoisted above the callers' checks of the table pointer.
__device__ __forceinline__ void interp_pair(const double2 *tab, int i, double w, double2 &gl, double2 &gg) {
  double2 l0, g0, l1, g1;
  asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
               : "=d"(l0.x), "=d"(l0.y), "=d"(g0.x), "=d"(g0.y)
               : "l"(tab + 2 * i));
  asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
               : "=d"(l1.x), "=d"(l1.y), "=d"(g1.x), "=d"(g1.y)
               : "l"(tab + 2 * i + 2));
  double v = __dsub_rn(1.0, w);
  gl = c2(__dadd_rn(__dmul_rn(v, l0.x), __dmul_rn(w, l1.x)), __dadd_rn(__dmul_rn(v, l0.y), __dmul_rn(w, l1.y)));
  gg = c2(__dadd_rn(__dmul_rn(v, g0.x), __dmul_rn(w, g1.x)), __dadd_rn(__dmul_rn(v, g0.y), __dmul_rn(w, g1.y)));
}

// Cubic Lagrange interpolation (an extension: keldy interpolates linearly) through the 4
// mesh points s0..s0+3 around the interval [i, i+1] (s0 = i-1, moved inside the mesh at
// its ends) at u = i + w - s0; every operation rounded separately, as the CPU oracle.
__device__ __forceinline__ void interp_pair_cubic(const double2 *tab, int npts, int i, double w, double2 &gl,
                                                  double2 &gg) {
  const int s0 = max(0, min(i - 1, npts - 4));
  const double u = __dadd_rn((double)(i - s0), w);
  const double am = __dsub_rn(u, 1.0), bm = __dsub_rn(u, 2.0), cm = __dsub_rn(u, 3.0);
  double L[4];
  L[0] = -__ddiv_rn(__dmul_rn(__dmul_rn(am, bm), cm), 6.0);
  L[1] = __ddiv_rn(__dmul_rn(__dmul_rn(u, bm), cm), 2.0);
  L[2] = -__ddiv_rn(__dmul_rn(__dmul_rn(u, am), cm), 2.0);
  L[3] = __ddiv_rn(__dmul_rn(__dmul_rn(u, am), bm), 6.0);
  gl = gg = c2(0.0, 0.0);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double2 l = __ldg(tab + 2 * (s0 + k)), g = __ldg(tab + 2 * (s0 + k) + 1);
    gl = c2(__dadd_rn(gl.x, __dmul_rn(L[k], l.x)), __dadd_rn(gl.y, __dmul_rn(L[k], l.y)));
    gg = c2(__dadd_rn(gg.x, __dmul_rn(L[k], g.x)), __dadd_rn(gg.y, __dmul_rn(L[k], g.y)));
  }
}

// The model's interpolation of both tables at mesh interval i, weight w.
__device__ __forceinline__ void interp_model(const ModelDev &m, const double2 *tab, int i, double w, double2 &gl,
                                             double2 &gg) {
  if (m.interp == 3)
    interp_pair_cubic(tab, m.npts, i, w, gl, gg);
  else
    interp_pair(tab, i, w, gl, gg);
}

// Both tables at x; zero when the block is absent. Sets *bad outside the window.
__device__ __forceinline__ void g0_pair(const ModelDev &m, const double2 *tab, double x, double2 &gl, double2 &gg,
                                        int *bad) {
  if (!tab) {
    gl = gg = c2(0.0, 0.0);
    return;
  }
  int i;
  double w;
  if (!interp_index(m, x, i, w)) {
    *bad = 1;
    i = 0;
    w = 0.0;
  }
  interp_model(m, tab, i, w, gl, gg);
}

// keldy::compare_3way (common.cpp:47-57) on (time, keldysh index, timesplit).
__device__ __forceinline__ int compare_3way(double ta, int ka, int sa, double tb, int kb, int sb) {
  int k3 = ka - kb;
  if (k3 != 0) return k3;
  double d = ta - tb;
  if (d != 0.0) return (1 - 2 * ka) * (2 * (!signbit(d)) - 1);
  return (1 - 2 * ka) * (sa - sb);
}

// g0_keldysh_contour_t::operator() (model.hpp:244-265) for general indices.
__device__ inline double2 g0_contour(const ModelDev &m, const kb_gf_index &a, const kb_gf_index &b, int internal,
                                     int *bad) {
  if (a.spin != b.spin) return c2(0.0, 0.0);
  int ord = compare_3way(a.time, a.k_idx, a.timesplit, b.time, b.k_idx, b.timesplit);
  double2 gl, gg;
  if (ord != 0) {
    g0_pair(m, m.tab[a.spin][a.orbital][b.orbital], a.time - b.time, gl, gg, bad);
    return ord > 0 ? gg : gl;
  }
  if (a.orbital != b.orbital) {
    g0_pair(m, m.tab[a.spin][a.orbital][b.orbital], 0.0, gl, gg, bad);
    return gl;
  }
  g0_pair(m, m.tab[a.spin][a.orbital][a.orbital], 0.0, gl, gg, bad);
  return c2(gl.x, gl.y - (double)internal * m.alpha);
}

// ------------------------------------------------------------------ Sobol
// Point number k (k >= 1) of the digital sequence: the state digitalseq_b2g::set_state
// builds for Gray code gray(k), x_j = 2^-32 (cur_j ^ shift_j) (digitalseq_b2g.hpp:455-471).
// k runs up to 2^m inclusive: keldy checks past_end() before next(), so the point
// k = 2^m is drawn once, with next()'s column ctz(2^m) % m = 0 for the Gray-code bit m.
__device__ __forceinline__ double sobol_coord(const SobolDev &s, uint32_t k, int j) {
  const uint32_t g = k ^ (k >> 1);
  const uint32_t *C = s.Csr + j * s.m;
  uint32_t cur = 0;
#pragma unroll
  for (int b = 0; b < SOBOL_COLS; ++b)
    if (b < s.m && ((g >> b) & 1u)) cur ^= __ldg(C + b);
  if (s.m < 32 && ((g >> s.m) & 1u)) cur ^= __ldg(C);
  return 2.3283064365386963e-10 * (double)(cur ^ __ldg(s.shfr + j));
}

// ---------------------------------------------------------------- warpers
// f1, f1_integrated and f1_integrated_inverse of the analytic product makers
// (product_1d_simple.hpp:560-630). The constants c[] are the makers' normalisations,
// evaluated once on the host in long double and rounded to double. W is WarperDev or
// SimpleDev (the same fields).
template <class W>
__device__ __forceinline__ double warper_f1(const W &w, double t) {
  switch (w.kind) {
  case KB_WARPER_EXPONENTIAL: return exp(-t / w.w) / w.c[1];
  case KB_WARPER_INVERSE: return 1.0 / (w.c[0] * (w.w + t));
  case KB_WARPER_INVERSE_SQUARE: return w.w / ((w.w + t) * (w.w + t) * w.c[0]);
  case KB_WARPER_INVERSE_POWER: return w.c[0] / pow(w.w + t, (double)w.power);
  case KB_WARPER_UNIFORM: return 1.0 / w.u_max;
  default: return 1.0;
  }
}

template <class W>
__device__ __forceinline__ double warper_F(const W &w, double t) {
  switch (w.kind) {
  case KB_WARPER_EXPONENTIAL: return expm1((w.u_max - t) / w.w) / w.c[0];
  case KB_WARPER_INVERSE: return log1p(t / w.w) / w.c[0];
  case KB_WARPER_INVERSE_SQUARE: return t / ((w.w + t) * w.c[0]);
  case KB_WARPER_INVERSE_POWER:
    return w.c[1] * (pow(t / w.w + 1.0, (double)(w.power - 1)) - 1.0) / pow(t + w.w, (double)(w.power - 1));
  case KB_WARPER_UNIFORM: return t / w.u_max;
  default: return t;
  }
}

template <class W>
__device__ __forceinline__ double warper_Finv(const W &w, double l) {
  switch (w.kind) {
  case KB_WARPER_EXPONENTIAL: return w.u_max - w.w * log1p(w.c[0] * l);
  case KB_WARPER_INVERSE: return w.w * expm1(l * w.c[0]);
  case KB_WARPER_INVERSE_SQUARE: return w.c[0] * l * w.w / (1.0 - w.c[0] * l);
  case KB_WARPER_INVERSE_POWER: {
    double d = pow(1.0 + l * w.c[2], 1.0 / (w.power - 1.0));
    return w.w * (1.0 - d) / d;
  }
  case KB_WARPER_UNIFORM: return w.u_max * l;
  default: return l;
  }
}

// The unnormalised f1 shapes of the hybrid warpers (make_product_1d_inverse_cube_alternate_
// interp_hybrid, product_1d.hpp:293-300): exp(-t/w), w/(w+t), (w/(w+t))^2, w^p/(w+t)^p
// (products in keldy's order), 1.
__device__ __forceinline__ double hybrid_f1(const SimpleDev &f, double t) {
  switch (f.kind) {
  case KB_WARPER_EXPONENTIAL: return exp(-t / f.w);
  case KB_WARPER_INVERSE: return f.w / (f.w + t);
  case KB_WARPER_INVERSE_SQUARE: return f.w * f.w / ((f.w + t) * (f.w + t));
  case KB_WARPER_INVERSE_POWER: {
    double num = f.w, den = f.w + t;
    for (int k = 1; k < f.power; ++k) {
      num *= f.w;
      den *= f.w + t;
    }
    return num / den;
  }
  default: return 1.0;
  }
}

// Interval i of the increasing points a[lo..hi] holding v: a[i] <= v < a[i+1], i in
// [lo, hi-1] (GSL's bisection: the last point falls in the last interval).
__device__ __forceinline__ int table_interval(const double *a, int lo, int hi, double v) {
  while (hi > lo + 1) {
    const int m = (lo + hi) >> 1;
    if (a[m] > v)
      hi = m;
    else
      lo = m;
  }
  return lo;
}

// Linear interpolation y(x) on the interval [x0, x1] (GSL's linear spline: y0 when the
// interval is empty).
__device__ __forceinline__ double table_lerp(double x, double x0, double x1, double y0, double y1) {
  const double dx = x1 - x0;
  return dx > 0.0 ? y0 + (x - x0) / dx * (y1 - y0) : y0;
}

// Cubic Hermite interpolation on [x0, x1] from the end values y0, y1 and slopes d0, d1
// (the form of GSL's Steffen spline between two knots).
__device__ __forceinline__ double table_hermite(double x, double x0, double x1, double y0, double y1, double d0,
                                                double d1) {
  const double h = x1 - x0;
  const double s = (y1 - y0) / h;
  const double c2 = (3.0 * s - 2.0 * d0 - d1) / h;
  const double c3 = (d0 + d1 - 2.0 * s) / (h * h);
  const double dx = x - x0;
  return y0 + dx * (d0 + dx * (c2 + dx * c3));
}

// A real function on the uniform mesh of [0, 1] with n points, linearly interpolated
// (TRIQS gf<retime> evaluation): NaN outside the mesh (out of window).
__device__ __forceinline__ double mesh_eval(const double *g, int n, double x) {
  const double delta_inv = 1.0 / (1.0 / (n - 1));
  const double a = x * delta_inv;
  double fi = floor(a);
  double w = a - fi;
  long i = (long)fi;
  if (i == n - 1 && fabs(w) < 1e-14) {
    i = n - 2;
    w = 1.0;
  }
  if (!(i >= 0 && i < n - 1) || !(x == x)) return CUDART_NAN;
  return (1.0 - w) * g[i] + w * g[i + 1];
}

// One coordinate of a device-resident product warper. reverse: u from l and the Jacobian
// of u(l); forward: l from u and the Jacobian of l(u). Outside a table's range the values
// are NaN (GSL's and TRIQS's evaluations fail there).
__device__ inline double table_reverse(const TableDimDev &t, double l, double &u) {
  switch (t.type) {
  case TAB_NEAREST: { // product_1d_simple.hpp:206-217, 270-278
    const double y = -l;
    if (!(t.p1[0] <= y && y <= t.p1[t.cut])) break;
    const int i = table_interval(t.p1, 0, t.cut, y);
    u = table_lerp(y, t.p1[i], t.p1[i + 1], t.p0[i], t.p0[i + 1]);
    if (!(t.p0[0] <= u && u <= t.p0[t.n - 1])) return CUDART_NAN;
    return 1.0 / t.p2[table_interval(t.p0, 0, t.n - 1, u)];
  }
  case TAB_PROJECTION: // projection.hpp:330-344, 361-363
    u = mesh_eval(t.p2, t.m, l);
    return t.norm / mesh_eval(t.p0, t.n, u);
  case TAB_ANALYTIC:
    u = warper_Finv(t.f, l);
    return 1.0 / warper_f1(t.f, u);
  case TAB_HYBRID: { // product_1d_simple.hpp:411-415, 484-492
    const double y = -l;
    if (!(t.p1[0] <= y && y <= t.p1[t.cut])) break;
    const int i = table_interval(t.p1, 0, t.cut, y);
    u = table_hermite(y, t.p1[i], t.p1[i + 1], t.p0[i], t.p0[i + 1], t.p3[i], t.p3[i + 1]);
    return 1.0 / (hybrid_f1(t.f, u) / t.norm);
  }
  }
  u = CUDART_NAN;
  return CUDART_NAN;
}

__device__ inline double table_forward(const TableDimDev &t, double u, double &l) {
  switch (t.type) {
  case TAB_NEAREST: {
    if (!(t.p0[0] <= u && u <= t.p0[t.n - 1])) break;
    const int i = table_interval(t.p0, 0, t.n - 1, u);
    l = -table_lerp(u, t.p0[i], t.p0[i + 1], t.p1[i], t.p1[i + 1]);
    return t.p2[i];
  }
  case TAB_PROJECTION: // projection.hpp:338-345, 352-358
    l = mesh_eval(t.p1, t.n, u);
    return mesh_eval(t.p0, t.n, u);
  case TAB_ANALYTIC: {
    const double f = warper_f1(t.f, u);
    l = warper_F(t.f, u);
    return f;
  }
  case TAB_HYBRID: {
    if (!(t.p0[0] <= u && u <= t.p0[t.n - 1])) break;
    const int i = table_interval(t.p0, 0, t.n - 1, u);
    const double f = hybrid_f1(t.f, u) / t.norm;
    l = -table_hermite(u, t.p0[i], t.p0[i + 1], t.p1[i], t.p1[i + 1], t.p2[i], t.p2[i + 1]);
    return f;
  }
  }
  l = CUDART_NAN;
  return CUDART_NAN;
}

// One warper's map_reverse on x[0..n) (identity.hpp:34-48, plasma_uv.hpp:46-51,
// product_1d_simple.hpp:109-117); returns its Jacobian.
__device__ inline double warp_reverse_one(const WarperDev &w, int n, double *x, int stride) {
  if (w.kind == KB_WARPER_IDENTITY) return 1.0;
  if (w.kind == KB_WARPER_TABLE) {
    double jac = 1.0;
    for (int i = 0; i < n; ++i) {
      double u;
      jac *= table_reverse(w.tab[w.ntab == 1 ? 0 : i], x[i * stride], u);
      x[i * stride] = u;
    }
    return jac;
  }
  if (w.kind == KB_WARPER_PLASMA_UV) {
    if (n > 0) {
      double u = w.u_max - x[0];
      x[0] = u;
      for (int i = 1; i < n; ++i) {
        u = u - x[i * stride];
        x[i * stride] = u;
      }
    }
    return 1.0;
  }
  double jac = 1.0;
  for (int i = 0; i < n; ++i) {
    double u = warper_Finv(w, x[i * stride]);
    x[i * stride] = u;
    jac *= 1.0 / warper_f1(w, u);
  }
  return jac;
}

// One warper's map_forward (plasma_uv.hpp:35-44, product_1d_simple.hpp:119-127).
__device__ inline double warp_forward_one(const WarperDev &w, int n, double *x, int stride) {
  if (w.kind == KB_WARPER_IDENTITY) return 1.0;
  if (w.kind == KB_WARPER_TABLE) {
    double jac = 1.0;
    for (int i = 0; i < n; ++i) {
      double l;
      jac *= table_forward(w.tab[w.ntab == 1 ? 0 : i], x[i * stride], l);
      x[i * stride] = l;
    }
    return jac;
  }
  if (w.kind == KB_WARPER_PLASMA_UV) {
    if (n > 0) {
      // sort descending (insertion sort; n <= MAX_ORDER), then consecutive differences
      for (int i = 1; i < n; ++i) {
        double v = x[i * stride];
        int j = i - 1;
        while (j >= 0 && x[j * stride] < v) {
          x[(j + 1) * stride] = x[j * stride];
          --j;
        }
        x[(j + 1) * stride] = v;
      }
      for (int i = n - 1; i > 0; --i) x[i * stride] = x[(i - 1) * stride] - x[i * stride];
      x[0] = w.u_max - x[0];
    }
    return 1.0;
  }
  double jac = 1.0;
  for (int i = 0; i < n; ++i) {
    double u = x[i * stride];
    jac *= warper_f1(w, u);
    x[i * stride] = warper_F(w, u);
  }
  return jac;
}

// warper_train_t::map_reverse(li, start, end) (warpers.hpp:72-85): warpers start-1
// down to end.
__device__ inline double chain_reverse(const WarperDev *chain, int start, int end, int n, double *x, int stride) {
  double jac = 1.0;
  for (int i = start - 1; i >= end; --i) jac *= warp_reverse_one(chain[i], n, x, stride);
  return jac;
}

__device__ inline double chain_forward(const WarperDev *chain, int start, int end, int n, double *x, int stride) {
  double jac = 1.0;
  for (int i = start; i < end; ++i) jac *= warp_forward_one(chain[i], n, x, stride);
  return jac;
}

} // namespace kb
