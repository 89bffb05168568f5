// Descriptors shared by the host side of the library (capi.cu) and the kernels.
#pragma once
#include <stdint.h>

#include "../../include/keldy_b200.h"

namespace kb {

constexpr int MAX_ORDER = 16;      // 2^16 Keldysh configurations per point
constexpr int SOBOL_COLS = 31;     // columns of the generating matrices (log_max_points <= 31)
constexpr int CTA_THREADS = 128;   // threads per CTA of the tree kernel (four CTAs per SM)
constexpr int TREE_MAX_SUB = 8;    // largest order solved breadth-first in one pass

// g0 tables of one model on the device: per mesh point {lesser.re, lesser.im,
// greater.re, greater.im} (32 bytes), one array per (spin, orbital a, orbital b); null
// = zero block.
struct ModelDev {
  const double2 *tab[2][2][2]; // [spin][o1][o2] -> 2*npts double2 (lesser, greater interleaved)
  int npts;
  double tmax;
  double xmin;
  double delta;
  double alpha;
  double pivot_floor; // |re|+|im| below which a tree pivot hands the point to the pivoted-LU kernel
  int interp;         // 1: linear (keldy, TRIQS gf<retime>); 3: cubic Lagrange through 4 mesh points
};

// One analytic 1D warper of the product makers (product_1d_simple.hpp:560-630): kind
// (KB_WARPER_*), power, u_max, w and the constants c[] computed on the host.
struct SimpleDev {
  int kind;
  int power;
  double u_max;
  double w;
  double c[3];
};

// What one coordinate of a device-resident product warper (kb_warper_table) holds.
enum TableType : int {
  // warper_product_1d_simple_interp_nearest_t (product_1d_simple.hpp:174-330): p0 = the
  // points u[n] (u[0] = 0, increasing), p1 = F[n], the normalised integral of f1 from u to
  // u_max, negated (F[0] = -1 ... F[n-1] = 0), p2 = f1 on each of the n-1 intervals (the
  // mean of its ends); the inverse interpolates F[0..cut] (cut: the last point before F's
  // trailing zeros).
  TAB_NEAREST = 0,
  // warper_projection_t (projection.hpp:176-382): uniform meshes of [0, 1]: p0 = fn[n],
  // p1 = its normalised integral fint[n], p2 = the inverse of fint on m points; norm = the
  // integral before normalisation.
  TAB_PROJECTION = 1,
  // one analytic warper_product_1d_simple_t per coordinate (warper_product_1d_t,
  // product_1d.hpp:110-160): f.
  TAB_ANALYTIC = 2,
  // warper_product_1d_simple_interp_hybrid_t (product_1d_simple.hpp:381-554): p0 = u[n],
  // p1 = F[n] (Simpson's rule), p2 = Steffen slopes dF/du at the n points, p3 = Steffen
  // slopes du/dF of the inverse at F[0..cut]; the Jacobian uses the closed form f.kind of
  // f1 divided by norm.
  TAB_HYBRID = 3,
};

struct TableDimDev {
  int type;
  int n;
  int m;
  int cut;
  const double *p0;
  const double *p1;
  const double *p2;
  const double *p3;
  double norm;
  SimpleDev f;
};

struct WarperDev {
  int kind;
  int power;
  double u_max;
  double w;
  double c[3];             // constants of the product makers, computed on the host (see make_warper_dev)
  const TableDimDev *tab;  // KB_WARPER_TABLE: ntab tables (1: every coordinate; n: one per coordinate)
  int ntab;
};

struct SobolDev {
  const uint32_t *Csr; // [dim][SOBOL_COLS] bit-reversed generating matrices
  const uint32_t *shfr;
  int dim;
  int m; // log_max_points
};

// Everything a kernel needs to evaluate one integrand configuration.
struct ItemDev {
  ModelDev model;
  SobolDev rng;
  WarperDev chain[KB_MAX_CHAIN];
  int chain_len;
  int chain_start; // map_reverse(li, chain_start, 0)
  kb_integrand f;
  int order;
  int spin_symmetric; // spin-down tables equal spin-up ones: det(s2) = det of s1's vertex block
  uint32_t k_first;
  int chunk_points; // points per scheduling chunk of this item (<= 128)
  int64_t n_points;
  // learned flow (integrate mode): point gp of the item is flow_x[gp*order..] with flow
  // Jacobian flow_jac[gp] instead of its Sobol point; null = plain Sobol points
  const double *flow_x;
  const double *flow_jac;
  // learned separable spline flow applied in line (integrate mode): [order][3 * 17] knots
  // (bin edges x, y and derivatives, kb_spline.cuh) of its dimensions; null = none
  const double *spline_knots;
  // learned autoregressive spline flow applied in line: its fp32 parameters (the
  // conditioners A_d, kb_spline.cuh); null = none
  const float *ar_spline;
};

// One chunk of points of one item, processed by one CTA iteration.
struct ChunkDev {
  int item;
  int order;
  int64_t first; // offset of the first point within the item
  int count;
};

// Per-chunk partial sums (deterministic reduction afterwards).
struct PartialDev {
  double sum_re;
  double sum_im;
  unsigned long long n_in_domain;
  unsigned long long n_fallback;
};

// A point the tree handed to the pivoted-LU kernel.
struct FallbackDev {
  int item;
  int pad;
  int64_t index; // point offset within the item
};

// Points per sub-batch of the tree kernel for each order: the widest breadth-first level
// fits a frontier buffer, and the fused bottom's nodes (9x9: eight threads each, 7x7: four)
// fit the CTA's 128 threads (16 nodes of 9x9 for orders 5..8, up to 32 of 7x7 for 3 and 4).
__host__ __device__ inline int tree_points_per_chunk(int n) {
  switch (n) {
  case 0: return 128;
  case 1: return 128;
  case 2: return 32;
  case 3: return 16;
  case 4: return 8;
  case 5: return 8;
  case 6: return 4;
  case 7: return 2;
  case 8: return 1;
  default: return 1;
  }
}

// Complex entries per frontier buffer: enough for the widest breadth-first level of
// every order (P * max_k 2^k (2(R-k)+1)^2 <= 1296 for every P, R pair above: 16 nodes of
// 9x9 at orders 5..8), so that four CTAs (two buffers each) fit an SM's shared memory.
constexpr int FRONTIER = 1296;

} // namespace kb
