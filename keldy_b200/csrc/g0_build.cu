// g0 tables of the single-level dot with flat-band leads, built on the GPU: the step
// before the hot path when many models run at once (parameter sweeps).
//
// Same functions as the host builder (keldy_b200/g0_tables.py: flatband), restated per
// mesh point: keldy's flat-band dot (impurity_oneband/model.hpp:100-112, 129-130;
// Delta^R = -i Gamma/2 per lead, model.cpp:107-111) Fourier-transformed as
//   g^<(t) = i Gamma/(2 pi) sum_mu [K_mu(t) + C_mu(t)],
//   g^>(t) = -i Gamma/(2 pi) sum_mu [pi/Gamma e^{-i eps t - Gamma t} - K_mu(t) - C_mu(t)],
// K_mu(t) = int_{-inf}^{mu} e^{-i w t} / ((w - eps)^2 + Gamma^2) dw in closed form through
// the exponential integral E1 (complex argument), C_mu(t) the finite-temperature
// correction int e^{-i w t} (n_F - theta)(w - mu) / ((w - eps)^2 + Gamma^2) dw by
// Gauss-Legendre quadrature on [mu - 36/beta, mu + 36/beta]. t = 0 in closed form
// (arctan), t < 0 from g(-t) = -conj(g(t)) (model.cpp:302-314).
//
// E1: power series E1(z) = -gamma - ln z - sum_k (-z)^k / (k k!) for small |z| or near
// the negative real axis, otherwise the even continued fraction
// E1(z) = e^{-z} / (z + 1 - 1/(z + 3 - 4/(z + 5 - ...))) evaluated by the modified Lentz
// method (Abramowitz & Stegun 5.1.11 and 5.1.22; Press et al., Numerical Recipes 6.3).
#include <cuda_runtime.h>
#include <math.h>

#include "kb_device.cuh"
#include "kb_launch.h"

namespace kb {

namespace {

constexpr double EULER_GAMMA = 0.57721566490153286061;
constexpr double PI = 3.14159265358979323846;

__device__ __forceinline__ double2 cdiv(double2 a, double2 b) { return cmul(a, crcp(b)); }
__device__ __forceinline__ double2 cexpd(double2 z) {
  double s, c;
  sincos(z.y, &s, &c);
  const double e = exp(z.x);
  return c2(e * c, e * s);
}
__device__ __forceinline__ double2 clogd(double2 z) { return c2(log(hypot(z.x, z.y)), atan2(z.y, z.x)); }

// E1(z), principal branch (cut on the negative real axis).
__device__ double2 e1_complex(double2 z) {
  const double az = hypot(z.x, z.y);
  const bool series = az < 1.5 || (z.x < 0.0 && fabs(z.y) < 0.6 * fabs(z.x));
  if (series) {
    // sum_{k>=1} (-z)^k / (k k!)
    double2 term = c2(1.0, 0.0), sum = c2(0.0, 0.0);
    const double2 mz = c2(-z.x, -z.y);
    for (int k = 1; k < 400; ++k) {
      term = cmul(term, mz);
      term = c2(term.x / k, term.y / k); // (-z)^k / k!
      const double2 t = c2(term.x / k, term.y / k);
      sum = cadd(sum, t);
      if (k > az && hypot(t.x, t.y) <= 1e-17 * hypot(sum.x, sum.y)) break;
    }
    const double2 lz = clogd(z);
    return c2(-EULER_GAMMA - lz.x - sum.x, -lz.y - sum.y);
  }
  double2 b = c2(z.x + 1.0, z.y);
  double2 c = c2(1e300, 0.0);
  double2 d = crcp(b);
  double2 h = d;
  for (int i = 1; i < 2000; ++i) {
    const double an = -(double)i * (double)i;
    b = c2(b.x + 2.0, b.y);
    d = crcp(c2(an * d.x + b.x, an * d.y + b.y));
    const double2 q = cdiv(c2(an, 0.0), c);
    c = c2(b.x + q.x, b.y + q.y);
    const double2 del = cmul(c, d);
    h = cmul(h, del);
    if (fabs(del.x - 1.0) + fabs(del.y) < 1e-16) break;
  }
  return cmul(h, cexpd(c2(-z.x, -z.y)));
}

// Ei(x) for real x > 0: gamma + ln x + sum x^k / (k k!) (all terms positive).
__device__ double ei_positive(double x) {
  double term = 1.0, sum = 0.0;
  for (int k = 1; k < 600; ++k) {
    term *= x / k;
    const double t = term / k;
    sum += t;
    if (k > x && t <= 1e-17 * sum) break;
  }
  return EULER_GAMMA + log(x) + sum;
}

// K_mu(t) for t > 0 (the host builder's _lorentz_below).
__device__ double2 lorentz_below(double t, double mu, double eps, double gamma) {
  double2 out = c2(0.0, 0.0);
  for (int sgn = 1; sgn >= -1; sgn -= 2) {
    const double2 z = c2(eps, sgn * gamma);
    const double2 v = c2(sgn * gamma * t, (mu - eps) * t); // i (mu - z) t
    double2 e1;
    if (sgn < 0 && mu == eps) {
      e1 = c2(-ei_positive(gamma * t), PI); // the path ends on the cut: limit from below
    } else {
      e1 = e1_complex(v);
      if (sgn < 0 && mu > eps) e1.y += 2.0 * PI; // continuation across the cut
    }
    const double2 ez = cexpd(c2(z.y * t, -z.x * t)); // exp(-i z t)
    const double2 J = cmul(c2(-ez.x, -ez.y), e1);
    out = c2(out.x + sgn * J.x, out.y + sgn * J.y);
  }
  // / (2 i gamma)
  return c2(out.y / (2.0 * gamma), -out.x / (2.0 * gamma));
}

struct FlatbandParams {
  double gamma, eps, bias, beta;
};

// One table per blockIdx.y; thread k >= 1 of the positive half builds mesh point mid+k
// and its mirror mid-k; k = 0 builds t = 0.
__global__ void flatband_kernel(const FlatbandParams *params, double2 *const *tabs, int npts, double tmax,
                                const double *nodes, const double *weights, int n_nodes) {
  const FlatbandParams P = params[blockIdx.y];
  double2 *tab = tabs[blockIdx.y];
  const int mid = npts / 2;
  const double delta = (tmax - (-tmax)) / (double)(npts - 1);
  const double pref = P.gamma / (2.0 * PI);
  const double mus[2] = {-P.bias / 2.0, P.bias / 2.0};
  const bool finite = isfinite(P.beta);
  const double W = 36.0 / P.beta;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= npts - 1 - mid; k += gridDim.x * blockDim.x) {
    const int i = mid + k;
    const double t = -tmax + i * delta;
    double2 less = c2(0.0, 0.0), great = c2(0.0, 0.0);
    double occ = 0.0;
    for (int l = 0; l < 2; ++l) {
      const double mu = mus[l];
      // finite-temperature correction: two Gauss-Legendre panels [-W, 0], [0, W]
      double2 corr = c2(0.0, 0.0);
      if (finite) {
        for (int pnl = 0; pnl < 2; ++pnl) {
          const double a = pnl == 0 ? -W : 0.0, b = pnl == 0 ? 0.0 : W;
          for (int q = 0; q < n_nodes; ++q) {
            const double x = 0.5 * (b - a) * nodes[q] + 0.5 * (b + a);
            const double wq = 0.5 * (b - a) * weights[q];
            const double ax = fabs(x);
            const double e = exp(-P.beta * ax);
            const double d = (x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0)) * e / (1.0 + e);
            const double dx = x + mu - P.eps;
            const double f = wq * d / (dx * dx + P.gamma * P.gamma);
            double s, c;
            sincos(-(x + mu) * (k == 0 ? 0.0 : t), &s, &c);
            corr = c2(corr.x + f * c, corr.y + f * s);
          }
        }
      }
      if (k == 0) {
        occ += (atan((mu - P.eps) / P.gamma) + PI / 2.0) / P.gamma + corr.x;
      } else {
        const double2 below = lorentz_below(t, mu, P.eps, P.gamma);
        const double2 full = cmul(c2(PI / P.gamma, 0.0), cexpd(c2(-P.gamma * t, -P.eps * t)));
        less = cadd(less, cadd(below, corr));
        great = c2(great.x + full.x - below.x - corr.x, great.y + full.y - below.y - corr.y);
      }
    }
    if (k == 0) {
      tab[2 * mid] = c2(0.0, pref * occ);
      tab[2 * mid + 1] = c2(0.0, -pref * (2.0 * PI / P.gamma - occ));
    } else {
      const double2 gl = c2(-pref * less.y, pref * less.x);   // i pref less
      const double2 gg = c2(pref * great.y, -pref * great.x); // -i pref great
      tab[2 * i] = gl;
      tab[2 * i + 1] = gg;
      const int j = npts - 1 - i; // mirror point of -t
      tab[2 * j] = c2(-gl.x, gl.y);
      tab[2 * j + 1] = c2(-gg.x, gg.y);
    }
  }
}

// Fourier sums by quadrature: keldy's finite-contour construction (model.cpp:220-319,
// qagp over the band of the semicircular bath) with the nodes and weights chosen by the
// caller: per mesh point t, g^<(t) = sum_k cl_k e^{-i w_k t}, g^>(t) = sum_k cg_k e^{-i w_k t}.
// symmetric: the dot block, summed on t >= 0 only (t = 0 exactly at the middle point) with
// g(-t) = -conj(g(t)) (model.cpp:302-310); otherwise every mesh point. One thread per
// summed point; the nodes are staged through shared memory in tiles of FT_TILE.
constexpr int FT_TILE = 256;

__global__ void fourier_kernel(const double *w, const double2 *cl, const double2 *cg, int n_nodes, double2 *tab,
                               int npts, double tmax, int symmetric, int *bad) {
  __shared__ double sw[FT_TILE];
  __shared__ double2 sl[FT_TILE], sg[FT_TILE];
  const int mid = npts / 2;
  const double delta = (tmax - (-tmax)) / (double)(npts - 1);
  const int count = symmetric ? npts - mid : npts;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = idx < count;
  const int i = symmetric ? mid + idx : idx;
  const double t = (symmetric && idx == 0) ? 0.0 : -tmax + i * delta;
  double2 gl = c2(0.0, 0.0), gg = c2(0.0, 0.0);
  for (int base = 0; base < n_nodes; base += FT_TILE) {
    const int nt = min(FT_TILE, n_nodes - base);
    __syncthreads();
    for (int k = threadIdx.x; k < nt; k += blockDim.x) {
      sw[k] = w[base + k];
      sl[k] = cl[base + k];
      sg[k] = cg[base + k];
    }
    __syncthreads();
    if (active) {
      for (int k = 0; k < nt; ++k) {
        double sn, cs;
        sincos(t * sw[k], &sn, &cs);
        // c e^{-i theta} = (c.x cos + c.y sin) + i (c.y cos - c.x sin)
        gl.x += sl[k].x * cs + sl[k].y * sn;
        gl.y += sl[k].y * cs - sl[k].x * sn;
        gg.x += sg[k].x * cs + sg[k].y * sn;
        gg.y += sg[k].y * cs - sg[k].x * sn;
      }
    }
  }
  if (!active) return;
  if (!isfinite(gl.x) || !isfinite(gl.y) || !isfinite(gg.x) || !isfinite(gg.y)) atomicOr(bad, 1);
  tab[2 * i] = gl;
  tab[2 * i + 1] = gg;
  if (symmetric && idx > 0) {
    const int j = npts - 1 - i; // mirror point of -t
    tab[2 * j] = c2(-gl.x, gl.y);
    tab[2 * j + 1] = c2(-gg.x, gg.y);
  }
}

// keldy's ft_method "fft" (make_g0_by_fft, model.cpp:179-212): TRIQS's make_gf_from_fourier
// of frequency values on the mesh adjoint to the time mesh. With L mesh points (odd),
// c = (L-1)/2, t_k = (k-c) dt and w_j = (j-c) dw, dw = 2 pi/(L dt), the discrete transform
//   g(t_k) = dw/(2 pi) sum_j G_j e^{-i w_j t_k} = dw/(2 pi) sum_j G_j e^{-2 pi i (j-c)(k-c)/L}
// summed directly, one thread per k, lesser and greater together. Within a tile of DFT_TILE
// frequencies the twiddle advances by the factor e^{-2 pi i (k-c)/L}; each tile starts from
// the exact twiddle of the integer phase (j-c)(k-c) mod L, so rounding does not build up.
// The 1/w^2 tails beyond the mesh: m2/(w^2 + a^2) (a = dw sqrt(L), m2 per function) is
// subtracted from G before the sum and its exact transform m2 e^{-a|t|}/(2a) added after.
constexpr int DFT_TILE = 256;

__device__ __forceinline__ double2 twiddle(long long phase, long long L) {
  long long r = phase % L;
  if (r < 0) r += L;
  double s, c;
  sincospi(-2.0 * (double)r / (double)L, &s, &c);
  return c2(c, s);
}

struct DftTail {
  double2 ml, mg; // 1/w^2 coefficients of the lesser and greater functions
  double a;
};

__global__ void dft_kernel(const double2 *Gl, const double2 *Gg, double2 *tab, int L, double dw, double dt,
                           DftTail tail, int *bad) {
  __shared__ double2 sl[DFT_TILE], sg[DFT_TILE];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const long long c = (L - 1) / 2;
  const long long kc = (long long)k - c;
  const double2 step = twiddle(kc, L);
  double2 al = c2(0.0, 0.0), ag = c2(0.0, 0.0);
  for (int base = 0; base < L; base += DFT_TILE) {
    const int nt = min(DFT_TILE, L - base);
    __syncthreads();
    for (int j = threadIdx.x; j < nt; j += blockDim.x) {
      const double w = (double)((long long)(base + j) - c) * dw;
      const double lz = 1.0 / (w * w + tail.a * tail.a);
      sl[j] = c2(Gl[base + j].x - tail.ml.x * lz, Gl[base + j].y - tail.ml.y * lz);
      sg[j] = c2(Gg[base + j].x - tail.mg.x * lz, Gg[base + j].y - tail.mg.y * lz);
    }
    __syncthreads();
    if (k < L) {
      double2 w = twiddle(((long long)base - c) * kc, L);
      for (int j = 0; j < nt; ++j) {
        al = c2(fma(sl[j].x, w.x, fma(-sl[j].y, w.y, al.x)), fma(sl[j].x, w.y, fma(sl[j].y, w.x, al.y)));
        ag = c2(fma(sg[j].x, w.x, fma(-sg[j].y, w.y, ag.x)), fma(sg[j].x, w.y, fma(sg[j].y, w.x, ag.y)));
        w = cmul(w, step);
      }
    }
  }
  if (k >= L) return;
  const double scale = dw / (2.0 * PI);
  const double e = exp(-tail.a * fabs((double)kc * dt)) / (2.0 * tail.a);
  al = c2(al.x * scale + tail.ml.x * e, al.y * scale + tail.ml.y * e);
  ag = c2(ag.x * scale + tail.mg.x * e, ag.y * scale + tail.mg.y * e);
  if (!isfinite(al.x) || !isfinite(al.y) || !isfinite(ag.x) || !isfinite(ag.y)) atomicOr(bad, 1);
  tab[2 * k] = al;
  tab[2 * k + 1] = ag;
}

// Baths with a rational hybridisation (flat band, Lorentzian; model.cpp:107-118): keldy's
// dot functions are sums over the leads of Fermi functions times rational functions R_l
// with simple poles z_k and residues r_k (g0_tables.rational_terms):
//   g^<(w) = sum_l n_F(w - mu_l) R_l(w),   g^>(w) = -sum_l (1 - n_F(w - mu_l)) R_l(w).
// Their transforms g(t) = int dw/2pi e^{-iwt} g(w), the exact quantity keldy's contour
// method integrates numerically (model.cpp:326-426), in closed form for t > 0:
//   K_mu(t) = int_{-inf}^{mu} e^{-iwt} R dw = sum_k r_k J(z_k), J(z) = -e^{-izt} E1(i (mu - z) t)
//     (E1 continued across its cut when Im z < 0 and mu > Re z: + 2 pi i),
//   F(t) = int e^{-iwt} R dw = -2 pi i sum_{Im z_k < 0} r_k e^{-i z_k t},
// the finite-temperature part C_mu(t) = int e^{-iwt} (n_F - theta)(w - mu) R dw by
// Gauss-Legendre quadrature on [mu - 36/beta, mu + 36/beta], t = 0 by the logarithms
// K_mu(0) = sum_k r_k (Log(mu - z_k) - i pi s_k) (s_k = +1 below the real axis, -1 above),
// and t < 0 as the conjugate of the same formulas for the conjugate poles and residues.
// E1 is evaluated scaled, e^v E1(v), so that e^{-izt} E1 does not overflow.
using RationalTerm = RationalTermDev;

__device__ double2 e1_scaled(double2 v) {
  const double av = hypot(v.x, v.y);
  const bool series = av < 1.5 || (v.x < 0.0 && fabs(v.y) < 0.6 * fabs(v.x));
  if (series) return cmul(cexpd(v), e1_complex(v));
  double2 b = c2(v.x + 1.0, v.y), c = c2(1e300, 0.0), d = crcp(b), h = d;
  for (int i = 1; i < 2000; ++i) { // the continued fraction of e1_complex without its e^{-v}
    const double an = -(double)i * (double)i;
    b = c2(b.x + 2.0, b.y);
    d = crcp(c2(an * d.x + b.x, an * d.y + b.y));
    const double2 q = cdiv(c2(an, 0.0), c);
    c = c2(b.x + q.x, b.y + q.y);
    const double2 del = cmul(c, d);
    h = cmul(h, del);
    if (fabs(del.x - 1.0) + fabs(del.y) < 1e-16) break;
  }
  return h;
}

// K, F and C of one term at t >= 0 (poles and residues conjugated when conj).
__device__ void rational_term(const RationalTerm &T, bool conj, double t, bool finite, double beta,
                              const double *nodes, const double *weights, int n_nodes, double2 &K, double2 &F,
                              double2 &C) {
  K = F = C = c2(0.0, 0.0);
  const double mu = T.mu;
  for (int k = 0; k < T.n; ++k) {
    const double2 z = conj ? c2(T.z[k].x, -T.z[k].y) : T.z[k];
    const double2 r = conj ? c2(T.r[k].x, -T.r[k].y) : T.r[k];
    if (t == 0.0) {
      const double2 lg = clogd(c2(mu - z.x, -z.y));
      const double s = z.y < 0.0 ? 1.0 : -1.0;
      K = cadd(K, cmul(r, c2(lg.x, lg.y - PI * s)));
      if (z.y < 0.0) F = cadd(F, cmul(r, c2(0.0, -2.0 * PI)));
      continue;
    }
    const double2 v = c2(z.y * t, (mu - z.x) * t); // i (mu - z) t
    double2 J;
    if (z.y < 0.0 && mu == z.x) { // the path ends on E1's cut: the limit from below
      const double2 e1 = c2(-ei_positive(-z.y * t), PI);
      J = cmul(c2(-1.0, 0.0), cmul(cexpd(c2(z.y * t, -z.x * t)), e1));
    } else {
      J = cmul(c2(-1.0, 0.0), cmul(cexpd(c2(0.0, -mu * t)), e1_scaled(v)));
      if (z.y < 0.0 && mu > z.x) // continuation across the cut: -2 pi i e^{-izt}
        J = cadd(J, cmul(c2(0.0, -2.0 * PI), cexpd(c2(z.y * t, -z.x * t))));
    }
    K = cadd(K, cmul(r, J));
    if (z.y < 0.0) F = cadd(F, cmul(cmul(r, c2(0.0, -2.0 * PI)), cexpd(c2(z.y * t, -z.x * t))));
  }
  if (!finite) return;
  const double W = 36.0 / beta;
  for (int pnl = 0; pnl < 2; ++pnl) {
    const double a = pnl == 0 ? -W : 0.0, b = pnl == 0 ? 0.0 : W;
    for (int q = 0; q < n_nodes; ++q) {
      const double x = 0.5 * (b - a) * nodes[q] + 0.5 * (b + a);
      const double wq = 0.5 * (b - a) * weights[q];
      const double e = exp(-beta * fabs(x));
      const double dn = (x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0)) * e / (1.0 + e); // n_F(x) - theta(-x)
      const double w = mu + x;
      double2 R = c2(0.0, 0.0);
      for (int k = 0; k < T.n; ++k) {
        const double2 z = conj ? c2(T.z[k].x, -T.z[k].y) : T.z[k];
        const double2 r = conj ? c2(T.r[k].x, -T.r[k].y) : T.r[k];
        R = cadd(R, cdiv(r, c2(w - z.x, -z.y)));
      }
      double s, c;
      sincos(-w * t, &s, &c);
      C = cadd(C, cmul(c2(wq * dn * R.x, wq * dn * R.y), c2(c, s)));
    }
  }
}

// One thread per mesh point (the t >= 0 half when symmetric, mirrored by g(-t) = -conj(g(t))).
__global__ void rational_kernel(const RationalTerm *terms, int n_terms, double beta, const double *nodes,
                                const double *weights, int n_nodes, double2 *tab, int npts, double tmax,
                                int symmetric, int *bad) {
  const int mid = npts / 2;
  const double delta = (tmax - (-tmax)) / (double)(npts - 1);
  const int count = symmetric ? npts - mid : npts;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= count) return;
  const int i = symmetric ? mid + idx : idx;
  const double t = (i == mid) ? 0.0 : -tmax + i * delta;
  const bool neg = t < 0.0;
  const bool finite = isfinite(beta);
  double2 less = c2(0.0, 0.0), great = c2(0.0, 0.0);
  for (int l = 0; l < n_terms; ++l) {
    double2 K, F, C;
    rational_term(terms[l], neg, fabs(t), finite, beta, nodes, weights, n_nodes, K, F, C);
    if (neg) { // g(t) for t < 0: the conjugate of the conjugate function's value at |t|
      K = c2(K.x, -K.y);
      F = c2(F.x, -F.y);
      C = c2(C.x, -C.y);
    }
    less = cadd(less, cadd(K, C));
    great = c2(great.x - (F.x - K.x - C.x), great.y - (F.y - K.y - C.y));
  }
  const double s = 1.0 / (2.0 * PI);
  const double2 gl = c2(less.x * s, less.y * s), gg = c2(great.x * s, great.y * s);
  if (!isfinite(gl.x) || !isfinite(gl.y) || !isfinite(gg.x) || !isfinite(gg.y)) atomicOr(bad, 1);
  tab[2 * i] = gl;
  tab[2 * i + 1] = gg;
  if (symmetric && i != mid) {
    const int j = npts - 1 - i;
    tab[2 * j] = c2(-gl.x, gl.y);
    tab[2 * j + 1] = c2(-gg.x, gg.y);
  }
}

// Block (o2, o1) from block (o1, o2): g_{o2 o1}(t) = -conj(g_{o1 o2}(-t)) (model.cpp:311-313).
__global__ void mirror_block_kernel(const double2 *src, double2 *dst, int npts) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += gridDim.x * blockDim.x) {
    const int j = npts - 1 - i;
    const double2 l = src[2 * j], g = src[2 * j + 1];
    dst[2 * i] = c2(-l.x, l.y);
    dst[2 * i + 1] = c2(-g.x, g.y);
  }
}

} // namespace

cudaError_t launch_fourier_table(const double *w, const double2 *cl, const double2 *cg, int n_nodes, double2 *tab,
                                 int npts, double tmax, int symmetric, int *bad, cudaStream_t st) {
  const int count = symmetric ? npts - npts / 2 : npts;
  fourier_kernel<<<(count + 127) / 128, 128, 0, st>>>(w, cl, cg, n_nodes, tab, npts, tmax, symmetric, bad);
  return cudaGetLastError();
}

cudaError_t launch_dft_table(const double2 *gl, const double2 *gg, double2 ml, double2 mg, double2 *tab, int npts,
                             double tmax, int *bad, cudaStream_t st) {
  const double dt = (tmax - (-tmax)) / (double)(npts - 1);
  const double dw = 2.0 * PI / ((double)npts * dt);
  DftTail tail{ml, mg, dw * sqrt((double)npts)};
  dft_kernel<<<(npts + 127) / 128, 128, 0, st>>>(gl, gg, tab, npts, dw, dt, tail, bad);
  return cudaGetLastError();
}

cudaError_t launch_rational_table(const RationalTermDev *terms, int n_terms, double beta, const double *nodes,
                                  const double *weights, int n_nodes, double2 *tab, int npts, double tmax, int symmetric,
                                  int *bad, cudaStream_t st) {
  const int count = symmetric ? npts - npts / 2 : npts;
  rational_kernel<<<(count + 127) / 128, 128, 0, st>>>(terms, n_terms, beta, nodes, weights, n_nodes, tab, npts, tmax,
                                                       symmetric, bad);
  return cudaGetLastError();
}

cudaError_t launch_mirror_block(const double2 *src, double2 *dst, int npts, cudaStream_t st) {
  mirror_block_kernel<<<(npts + 255) / 256, 256, 0, st>>>(src, dst, npts);
  return cudaGetLastError();
}

cudaError_t launch_flatband_tables(int n_models, const double *params_dev, double2 *const *tabs_dev, int npts,
                                   double tmax, const double *nodes_dev, const double *weights_dev, int n_nodes,
                                   cudaStream_t st) {
  if (n_models <= 0) return cudaSuccess;
  const int half = npts - npts / 2;
  dim3 grid((half + 127) / 128, n_models);
  flatband_kernel<<<grid, 128, 0, st>>>(reinterpret_cast<const FlatbandParams *>(params_dev), tabs_dev, npts, tmax,
                                        nodes_dev, weights_dev, n_nodes);
  return cudaGetLastError();
}

} // namespace kb
