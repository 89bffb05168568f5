// Wick-determinant integrand kernels (sm_100a).
//
// keldy's integrand (impurity_oneband/wick_direct.cpp:43-158) sums, over the 2^n
// Keldysh configurations a, (-1)^|a| det(s1_a) det(s2_a), where s1_a is the (n+1)^2
// matrix of g0 between the chosen vertex copies and the two external points (corner
// set to 0) and s2_a the n^2 matrix of the opposite spin. Every s1_a/s2_a is a
// principal submatrix of one (2n+1)^2 matrix G (vertex j forward = row 2j, backward =
// row 2j+1, external = row 2n).
//
// Tree kernel: Gaussian elimination of G with the pivot of vertex k taken on the
// diagonal entry of the chosen copy (2k or 2k+1) visits all 2^n configurations as the
// leaves of a binary tree; the Schur complement of a node is shared by its whole
// subtree. At a leaf, det(s2_a) is the product of the pivots along the path (spin
// symmetric models) and the remaining 1x1 Schur complement of the external corner is
// det(s1_a)/det(s2_a). Cost O(2^n) complex FMAs per point instead of O(2^n n^3).
// The top levels run breadth-first in shared memory (two 20.7 KB frontier buffers,
// ping-pong), the last three (two at orders 3 and 4) per thread in registers. Orders above
// 8 walk their first n-8 levels one root-to-subtree path at a time. Per G-batch of points
// every table lookup is issued at once and G staged in global memory; each sub-batch's G
// is copied into shared memory asynchronously while the previous sub-batch's bottom runs.
//
// Direct kernel: keldy's own algorithm, one partial-pivot LU pair per configuration
// (pivot = first maximum of |re|+|im|, as LAPACK's zgetf2). It serves models whose
// spin-down tables differ from spin-up ones, points whose tree pivots fall below the
// guard, and cross-checks.
#include <cuda_runtime.h>
#include <stdio.h>

#include "kb_device.cuh"
#include "kb_launch.h"
#include "kb_spline.cuh"

namespace kb {

namespace {

constexpr int NT = CTA_THREADS;
// first of the set-up slot's three rows of per-point bin data (after the coordinates,
// the Jacobians and the flags)
constexpr int BIN_CODE_ROW = MAX_ORDER + 2;
// Threads of a tree-kernel CTA: eight per 9x9 node (16 nodes per sub-batch at orders 5..8),
// four per 7x7 node (up to 32 at orders 3 and 4).
constexpr int TREE_THREADS = CTA_THREADS;

struct TreeShared {
  double2 buf[2][FRONTIER];
  double2 D[2][NT];  // prefix determinant per node (ping-pong with the frontier)
  double2 tmp[NT];   // pivot reciprocals during a level; per-node partial sums after the bottom
  double u[256];     // vertex times, u[j * np + p]
  double jac[NT];
  double2 fval[NT];
  double fscale[NT];
  int flag[NT];      // bit 0: out of domain, bit 1: needs the pivoted-LU kernel
  double2 wsum[TREE_THREADS / 32]; // per-warp partial sums of the per-point reduction
  double wscale[TREE_THREADS / 32];
};

__device__ __forceinline__ int find_item(const long long *off, int n_items, long long c) {
  int lo = 0, hi = n_items; // off[lo] <= c < off[hi]
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (off[mid] <= c)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// The learned spline flow in line: the Sobol point x (stride `st`) to x_j = F_j^{-1}(x_j),
// returning the flow's Jacobian prod_j 1 / F_j'(x_j), formed as the flow's own map kernel
// forms it (same operations, same order).
__device__ __forceinline__ double spline_flow_point(const double *knots, int N, double *x, int st) {
  const SplineKnots *k = reinterpret_cast<const SplineKnots *>(knots);
  double jac = 1.0;
  for (int j = 0; j < N; ++j) {
    double der;
    x[j * st] = spline_inverse(k[j], x[j * st], der);
    jac /= der;
  }
  return jac;
}

// Inputs of np points (thread p < np): vertex times into u[j*np+p], Jacobian and
// domain flag. keep: drop points with a negative time (keep_u_hypercube).
__device__ void load_points(const Launch &L, const ItemDev &it, int N, int np, long long gp0, double *u,
                            double *jac_out, int *flag_out, bool keep) {
  int p = threadIdx.x;
  if (p >= np) return;
  long long gp = gp0 + p;
  double *x = u + p;
  double jac = 1.0;
  if (L.mode == IN_SOBOL) {
    if (it.flow_x) { // Sobol point already mapped by the learned flow
      for (int j = 0; j < N; ++j) x[j * np] = it.flow_x[gp * N + j];
      jac = it.flow_jac[gp];
    } else {
      uint32_t k = it.k_first + (uint32_t)gp;
      for (int j = 0; j < N; ++j) x[j * np] = sobol_coord(it.rng, k, j);
      if (it.spline_knots) jac = spline_flow_point(it.spline_knots, N, x, np);
      if (it.ar_spline) jac = ar_spline_point(it.ar_spline, N, x, np);
    }
    jac *= chain_reverse(it.chain, it.chain_len, 0, N, x, np);
  } else {
    long long src = L.index ? (long long)L.index[gp] : gp;
    for (int j = 0; j < N; ++j) x[j * np] = L.in[src * N + j];
    if (L.mode == IN_LI) jac = chain_reverse(it.chain, it.chain_start, 0, N, x, np);
  }
  int dom = 1;
  if (it.f.A.spin != it.f.B.spin) dom = 0;
  if (keep)
    for (int j = 0; j < N; ++j)
      if (x[j * np] < 0.0) dom = 0;
  jac_out[p] = jac;
  flag_out[p] = dom ? 0 : 1;
}

// Bin of the earliest vertex time (binner_t::in_bounds and coord2index, binner.hpp:163-176:
// in [xmin, xmax], xmax itself in the last bin); -1: dropped. An index that rounds up to
// nbins just below xmax goes to the last bin.
__device__ __forceinline__ int time_bin(const Launch &L, const double *u, int stride, int N) {
  double t = u[0];
  for (int j = 1; j < N; ++j) t = fmin(t, u[j * stride]);
  if (!(L.bin_xmin <= t && t <= L.bin_xmax)) return -1;
  if (t == L.bin_xmax) return L.nbins - 1;
  return min((int)((t - L.bin_xmin) / L.bin_size), L.nbins - 1);
}

// One point of a chunk, on one thread: Sobol coordinates (or the given inputs), the
// warper chain, the domain flag; written to the CTA's set-up slot at column t.
__device__ void prepare_point(const Launch &L, const ItemDev &it, int N, long long gp, bool keep, double *slot,
                              int t) {
  double x[MAX_ORDER];
  double jac = 1.0;
  if (L.mode == IN_SOBOL) {
    if (it.flow_x) { // Sobol point already mapped by the learned flow
      for (int j = 0; j < N; ++j) x[j] = it.flow_x[gp * N + j];
      jac = it.flow_jac[gp];
    } else {
      const uint32_t k = it.k_first + (uint32_t)gp;
      for (int j = 0; j < N; ++j) x[j] = sobol_coord(it.rng, k, j);
      if (it.spline_knots) jac = spline_flow_point(it.spline_knots, N, x, 1);
      if (it.ar_spline) jac = ar_spline_point(it.ar_spline, N, x, 1);
    }
    jac *= chain_reverse(it.chain, it.chain_len, 0, N, x, 1);
  } else {
    const long long src = L.index ? (long long)L.index[gp] : gp;
    for (int j = 0; j < N; ++j) x[j] = L.in[src * N + j];
    if (L.mode == IN_LI) jac = chain_reverse(it.chain, it.chain_start, 0, N, x, 1);
  }
  int dom = (it.f.A.spin == it.f.B.spin) ? 1 : 0;
  if (keep)
    for (int j = 0; j < N; ++j)
      if (x[j] < 0.0) dom = 0;
  for (int j = 0; j < N; ++j) slot[j * CHUNK_POINTS + t] = x[j];
  slot[MAX_ORDER * CHUNK_POINTS + t] = jac;
  slot[(MAX_ORDER + 1) * CHUNK_POINTS + t] = dom ? 0.0 : 1.0;
  if (L.nbins) { // the time bin of the earliest vertex: code 2 bin, or -1 when dropped
    const int bin = time_bin(L, x, 1, N);
    slot[BIN_CODE_ROW * CHUNK_POINTS + t] = bin < 0 ? -1.0 : (double)(2 * bin);
  }
}

// G (row-major, M = 2N+1) of np points: G[p*M*M + r*M + c]. Out-of-domain points get
// the identity (their values are discarded; this keeps every pivot finite).
// Items per point: the N(N-1) ordered vertex pairs, the N external-row and N
// external-column entries (one table lookup each: g^< and g^> at one time difference),
// the N diagonal blocks (g(0)) and the corner. Each thread computes the lookup positions
// of GK items before issuing their loads, so that GK L2 round trips overlap.
template <bool CUBIC, int GK>
__device__ void build_G(const ItemDev &it, int N, int np, const double *u, const int *flag, double2 *buf,
                        int spin, int *bad) {
  const ModelDev &m = it.model;
  const int M = 2 * N + 1;
  const int npair = N * (N - 1), nlook = npair + 2 * N, per = nlook + N + 1;
  const kb_gf_index &A = it.f.A, &B = it.f.B;
  const double2 *t00 = m.tab[spin][0][0];
  const double2 *trow = m.tab[spin][A.orbital][0];
  const double2 *tcol = m.tab[spin][0][B.orbital];
  const int total = np * per;
  // r / per and q / (N - 1) as a multiply-high by 2^32 / d rounded up (exact for the
  // quotients here: r < 2^16, d <= 289); mn1 wraps to 0 for N - 1 = 1 (q / 1 = q)
  const unsigned mper = 0xFFFFFFFFu / (unsigned)per + 1u;
  const unsigned mn1 = N > 1 ? 0xFFFFFFFFu / (unsigned)(N - 1) + 1u : 0u;
  for (int base = threadIdx.x; base < total; base += GK * blockDim.x) {
    int kind[GK], pi[GK], qi[GK], ix[GK];
    double wt[GK], dt[GK];
    const double2 *tb[GK];
#pragma unroll
    for (int k = 0; k < GK; ++k) {
      const int r = base + k * blockDim.x;
      kind[k] = 0; // 0: none, 1: pair, 2: row, 3: col, 4: diagonal, 5: corner, 6: out of domain
      tb[k] = nullptr;
      ix[k] = 0;
      wt[k] = 0.0;
      dt[k] = 0.0;
      pi[k] = 0;
      qi[k] = 0;
      if (r >= total) continue;
      const int p = (int)__umulhi((unsigned)r, mper), q = r - p * per;
      pi[k] = p;
      qi[k] = q;
      const double *x = u + p;
      if (flag[p] & 1) {
        kind[k] = 6;
        continue;
      }
      if (q < npair) {
        const int i = mn1 ? (int)__umulhi((unsigned)q, mn1) : q, r2 = q - i * (N - 1), j = r2 + (r2 >= i ? 1 : 0);
        kind[k] = 1;
        dt[k] = x[i * np] - x[j * np];
        tb[k] = t00;
      } else if (q < npair + N) {
        kind[k] = 2;
        dt[k] = A.time - x[(q - npair) * np];
        tb[k] = trow;
      } else if (q < nlook) {
        kind[k] = 3;
        dt[k] = x[(q - npair - N) * np] - B.time;
        tb[k] = tcol;
      } else if (q < nlook + N) {
        kind[k] = 4;
        tb[k] = t00;
      } else {
        kind[k] = 5;
      }
      if (tb[k] && !interp_index(m, dt[k], ix[k], wt[k])) {
        *bad = 1;
        ix[k] = 0;
        wt[k] = 0.0;
      }
    }
    double2 gl[GK], gg[GK];
#pragma unroll
    for (int k = 0; k < GK; ++k) {
      if (tb[k] && CUBIC)
        interp_pair_cubic(tb[k], m.npts, ix[k], wt[k], gl[k], gg[k]);
      else if (tb[k])
        interp_pair(tb[k], ix[k], wt[k], gl[k], gg[k]);
      else
        gl[k] = gg[k] = c2(0.0, 0.0);
    }
#pragma unroll
    for (int k = 0; k < GK; ++k) {
      if (kind[k] == 0) continue;
      double2 *G = buf + (size_t)pi[k] * M * M;
      const int q = qi[k];
      const double *x = u + pi[k];
      if (kind[k] == 1) {
        const int i = mn1 ? (int)__umulhi((unsigned)q, mn1) : q, r2 = q - i * (N - 1), j = r2 + (r2 >= i ? 1 : 0);
        double2 *g = G + (2 * i) * M + 2 * j;
        const double d = dt[k];
        const bool later = (d != 0.0) ? (d > 0.0) : (i > j);
        g[0] = later ? gg[k] : gl[k];     // forward-forward
        g[M + 1] = later ? gl[k] : gg[k]; // backward-backward
        g[1] = gl[k];                     // forward-backward
        g[M] = gg[k];                     // backward-forward
      } else if (kind[k] == 2) {
        const int j = q - npair;
        const double uj = x[j * np];
        double2 *row = G + (2 * N) * M + 2 * j;
        row[0] = compare_3way(A.time, A.k_idx, N, uj, 0, j) > 0 ? gg[k] : gl[k];
        row[1] = compare_3way(A.time, A.k_idx, N, uj, 1, j) > 0 ? gg[k] : gl[k];
      } else if (kind[k] == 3) {
        const int j = q - npair - N;
        const double uj = x[j * np];
        double2 *col = G + (2 * j) * M + 2 * N;
        col[0] = compare_3way(uj, 0, j, B.time, B.k_idx, N) > 0 ? gg[k] : gl[k];
        col[M] = compare_3way(uj, 1, j, B.time, B.k_idx, N) > 0 ? gg[k] : gl[k];
      } else if (kind[k] == 4) {
        const int i = q - nlook;
        double2 *g = G + (2 * i) * M + 2 * i;
        const double2 eq = c2(gl[k].x, gl[k].y - m.alpha); // equal contour points, internal
        g[0] = eq;
        g[M + 1] = eq;
        g[1] = gl[k];
        g[M] = gg[k];
      } else if (kind[k] == 5) {
        G[(2 * N) * M + 2 * N] = c2(0.0, 0.0);
      } else { // out of domain: identity blocks, zero externals
        const double2 z = c2(0.0, 0.0), one = c2(1.0, 0.0);
        if (q < npair) {
          const int i = mn1 ? (int)__umulhi((unsigned)q, mn1) : q, r2 = q - i * (N - 1), j = r2 + (r2 >= i ? 1 : 0);
          double2 *g = G + (2 * i) * M + 2 * j;
          g[0] = g[1] = g[M] = g[M + 1] = z;
        } else if (q < npair + N) {
          double2 *row = G + (2 * N) * M + 2 * (q - npair);
          row[0] = row[1] = z;
        } else if (q < nlook) {
          double2 *col = G + (2 * (q - npair - N)) * M + 2 * N;
          col[0] = col[M] = z;
        } else if (q < nlook + N) {
          const int i = q - nlook;
          double2 *g = G + (2 * i) * M + 2 * i;
          g[0] = g[M + 1] = one;
          g[1] = g[M] = z;
        } else {
          G[(2 * N) * M + 2 * N] = one;
        }
      }
    }
  }
}

// build_G with the model's interpolation chosen once per call; ANY_CUBIC = false compiles
// the linear lookup only (launches whose models all interpolate linearly).
template <bool ANY_CUBIC, int GK = 2>
__device__ void build_G_any(const ItemDev &it, int N, int np, const double *u, const int *flag, double2 *buf,
                            int spin, int *bad) {
  if (ANY_CUBIC && it.model.interp == 3)
    build_G<true, GK>(it, N, np, u, flag, buf, spin, bad);
  else
    build_G<false, GK>(it, N, np, u, flag, buf, spin, bad);
}

// 16-byte asynchronous copies global -> shared (the L2-only variant: the source was
// written by this CTA moments before), and the wait for the calling thread's copies.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Copies n complex entries (the staged G of a sub-batch) into shared memory, spread over
// the CTA's threads; completed by cp_async_wait_all and a barrier.
__device__ __forceinline__ void copy_roots(double2 *dst, const double2 *src, int n) {
  for (int e = threadIdx.x; e < n; e += blockDim.x) cp_async16(dst + e, src + e);
}

// One breadth-first level, both children of a node from one read of its rows: thread r
// takes row i of parent `par` and writes row i of children 2 par (pivot on row 0) and
// 2 par + 1 (pivot on row 1). Nodes per point = 2^lg_npp; m >= 9.
__device__ void tree_level2(const double2 *cur, double2 *nxt, const double2 *Dc, double2 *Dn, double2 *inv,
                            int *flag, int nodes, int lg_npp, int m, double floor_) {
  const int mc = m - 2, mm = m * m, mcc = mc * mc;
  for (int c = threadIdx.x; c < 2 * nodes; c += blockDim.x) {
    int par = c >> 1, b = c & 1;
    double2 piv = cur[par * mm + b * (m + 1)];
    if (!(cabs1(piv) >= floor_)) flag[par >> lg_npp] |= 2;
    inv[c] = crcp(piv);
    Dn[c] = cmul(Dc[par], piv);
  }
  __syncthreads();
  const unsigned rows = (unsigned)(nodes * mc);
  const unsigned magic = 0xFFFFFFFFu / (unsigned)mc + 1u; // r / mc == umulhi(r, magic) for r < 2^20, mc <= 31
  // split rows into column segments of at least 4 columns while the CTA has idle threads
  int lgseg = 0;
  while ((rows << (lgseg + 1)) <= blockDim.x && (mc >> (lgseg + 1)) >= 4) ++lgseg;
  const int seglen = (mc + (1 << lgseg) - 1) >> lgseg;
  const unsigned items = rows << lgseg;
  for (unsigned t = threadIdx.x; t < items; t += blockDim.x) {
    const unsigned r = t >> lgseg;
    const int j0 = (int)(t & ((1u << lgseg) - 1)) * seglen, j1 = min(mc, j0 + seglen);
    const unsigned par = __umulhi(r, magic);
    const unsigned i = r - par * (unsigned)mc;
    const double2 *S = cur + par * mm;
    const double2 L0 = cmul(S[(i + 2) * m], inv[2 * par]);
    const double2 L1 = cmul(S[(i + 2) * m + 1], inv[2 * par + 1]);
    const double2 *srow = S + (i + 2) * m + 2, *p0 = S + 2, *p1 = S + m + 2;
    double2 *o0 = nxt + (2 * par) * mcc + i * mc, *o1 = o0 + mcc;
#pragma unroll 4
    for (int j = j0; j < j1; ++j) {
      const double2 v = srow[j];
      o0[j] = cfms(v, L0, p0[j]);
      o1[j] = cfms(v, L1, p1[j]);
    }
  }
  __syncthreads();
}

// Two breadth-first levels at once: node `par` (m x m) into its four grandchildren
// 4 par + 2 b + bp (pivot on row b, then on row bp of that child), (m-4) x (m-4) each,
// every entry formed exactly as two tree_level2 steps form it. A pre-pass forms each
// parent's pivot quantities once (one thread per (parent, b, b'), into pv); then each item
// (grandchild row i of a parent, one first pivot b, a column segment) forms the entries of
// child b it needs itself and writes row i of grandchildren (b, 0) and (b, 1), so the pair
// takes two barriers and never stores the children. (Items of both first pivots, twice the
// work per item and half the items, were 6 % slower at order 8 and 3-5 % at orders 6, 7,
// 9 and 10: the first pair of a one-point sub-batch had 26 busy threads of 128. Items
// that formed the pivot quantities themselves, six reciprocals each, with one barrier per
// pair, were slower again, 4-13 % at orders 6-10. A pre-pass that also formed the
// grandchildren's pivot rows, three complex products per column and item instead of five,
// was slower as well: four loads per three products, less work in flight per thread.)
__device__ void tree_level4(const double2 *cur, double2 *nxt, const double2 *Dc, double2 *Dn, int *flag, int nodes,
                            int lg_npp, int m, double floor_, double2 *pv) {
  const int mg = m - 4, mm = m * m, mgg = mg * mg;
  // the pivot quantities of every (parent, b, b') once, before the rows (pv: 12 entries
  // per parent): the first pivot's reciprocal, child row b''s factor and the second
  // pivot's reciprocal; the guard flags and the grandchildren's prefix determinants
  for (int c = threadIdx.x; c < nodes * 4; c += blockDim.x) {
    const int par = c >> 2, b = (c >> 1) & 1, bp = c & 1;
    const double2 *S = cur + par * mm;
    const double2 piv = S[b * (m + 1)];
    const double2 ibv = crcp(piv);
    const double2 Lpv = cmul(S[(2 + bp) * m + b], ibv); // child row bp's factor
    const double2 cpv = cfms(S[(2 + bp) * m + 2 + bp], Lpv, S[b * m + 2 + bp]);
    pv[c * 3 + 0] = ibv;
    pv[c * 3 + 1] = Lpv;
    pv[c * 3 + 2] = crcp(cpv);
    if (!(cabs1(piv) >= floor_) || !(cabs1(cpv) >= floor_)) flag[par >> lg_npp] |= 2;
    Dn[c] = cmul(cmul(Dc[par], piv), cpv);
  }
  __syncthreads();
  if (nodes == 1) {
    // a single parent (the first pair of a one-point sub-batch, orders 8 and up): items of
    // one row, one b and one b', each writing one grandchild's row, so that 104 threads
    // work at order 8 instead of 52 (order 8 -0.7 %, order 10 -3 %)
    int lgs = 0;
    while (((4 * mg) << (lgs + 1)) <= (int)blockDim.x && (mg >> (lgs + 1)) >= 4) ++lgs;
    const int sl = (mg + (1 << lgs) - 1) >> lgs;
    const int nit = (4 * mg) << lgs;
    for (int t = threadIdx.x; t < nit; t += blockDim.x) {
      const int q4 = t >> lgs;
      const int j0 = (t & ((1 << lgs) - 1)) * sl, j1 = min(mg, j0 + sl);
      const int c = q4 & 3, b = c >> 1, bp = c & 1, i = q4 >> 2;
      const double2 *S = cur;
      const double2 Lr = cmul(S[(i + 4) * m + b], pv[(2 * b) * 3]);
      const double2 Lp = pv[c * 3 + 1];
      const double2 Lg = cmul(cfms(S[(i + 4) * m + 2 + bp], Lr, S[b * m + 2 + bp]), pv[c * 3 + 2]);
      const double2 *sr = S + (i + 4) * m + 4, *sb = S + b * m + 4, *sa = S + (2 + bp) * m + 4;
      double2 *o = nxt + c * mgg + i * mg;
#pragma unroll 3
      for (int j = j0; j < j1; ++j) {
        const double2 pb = sb[j];
        const double2 cij = cfms(sr[j], Lr, pb); // child b, row i + 2
        const double2 cc = cfms(sa[j], Lp, pb);  // child b, row b' (the second pivot row)
        o[j] = cfms(cij, Lg, cc);
      }
    }
    __syncthreads();
    return;
  }
  const unsigned rows = (unsigned)(nodes * mg);
  const unsigned magic = 0xFFFFFFFFu / (unsigned)mg + 1u; // r / mg == umulhi(r, magic) for r < 2^20, mg <= 31
  // column segments of at least two columns while the CTA has idle threads; four for a
  // single node (a one-point sub-batch's first pair, orders 8 and up), where fewer, longer
  // segments repeat each item's own quantities (Lr, the child-row entries, Lg) less often
  const int minc = nodes == 1 ? 4 : 2;
  int lgseg = 0;
  while (((2 * rows) << (lgseg + 1)) <= blockDim.x && (mg >> (lgseg + 1)) >= minc) ++lgseg;
  const int seglen = (mg + (1 << lgseg) - 1) >> lgseg;
  const unsigned items = (2 * rows) << lgseg;
  for (unsigned t = threadIdx.x; t < items; t += blockDim.x) {
    const unsigned rb2 = t >> lgseg;
    const int j0 = (int)(t & ((1u << lgseg) - 1)) * seglen, j1 = min(mg, j0 + seglen);
    const int b = (int)(rb2 & 1u);
    const unsigned r = rb2 >> 1;
    const unsigned par = __umulhi(r, magic);
    const int i = (int)(r - par * (unsigned)mg);
    const double2 *S = cur + par * mm;
    const double2 ib = pv[(par * 4 + 2 * b) * 3];
    const double2 Lr = cmul(S[(i + 4) * m + b], ib);
    const double2 Lp0 = pv[(par * 4 + 2 * b) * 3 + 1], Lp1 = pv[(par * 4 + 2 * b + 1) * 3 + 1];
    const double2 Lg0 = cmul(cfms(S[(i + 4) * m + 2], Lr, S[b * m + 2]), pv[(par * 4 + 2 * b) * 3 + 2]);
    const double2 Lg1 = cmul(cfms(S[(i + 4) * m + 3], Lr, S[b * m + 3]), pv[(par * 4 + 2 * b + 1) * 3 + 2]);
    const double2 *sr = S + (i + 4) * m + 4, *sb = S + b * m + 4, *s2 = S + 2 * m + 4, *s3 = S + 3 * m + 4;
    double2 *o = nxt + (4 * par + 2 * b) * mgg + i * mg;
    // (unrolled by 2 the kernel spilled five times as many bytes and ran 3-16 % slower)
#pragma unroll 3
    for (int j = j0; j < j1; ++j) {
      const double2 v = sr[j], pb = sb[j], a2 = s2[j], a3 = s3[j];
      const double2 cij = cfms(v, Lr, pb);  // child b, row i + 2
      const double2 c0 = cfms(a2, Lp0, pb); // child b, row 0 (pivot row of b' = 0)
      const double2 c1 = cfms(a3, Lp1, pb); // child b, row 1
      o[j] = cfms(cij, Lg0, c0);
      o[mgg + j] = cfms(cij, Lg1, c1);
    }
  }
  __syncthreads();
}


// One step down a fixed path (single point): pivot on row b, drop rows 0 and 1.
__device__ void tree_path_step(const double2 *cur, double2 *nxt, const double2 *Dc, double2 *Dn, int *flag, int m,
                               int b, double floor_) {
  const int mc = m - 2;
  // every thread forms the pivot's reciprocal itself: no barrier before the row updates
  const double2 piv = cur[b * m + b];
  const double2 inv = crcp(piv);
  if (threadIdx.x == 0) {
    if (!(cabs1(piv) >= floor_)) flag[0] |= 2;
    Dn[0] = cmul(Dc[0], piv);
  }
  const unsigned magic = 0xFFFFFFFFu / (unsigned)mc + 1u; // r / mc == umulhi(r, magic) for r < 2^20, mc >= 2
  for (int r = threadIdx.x; r < mc * mc; r += blockDim.x) {
    const int i = (int)__umulhi((unsigned)r, magic), j = r - i * mc;
    double2 Lf = cmul(cur[(i + 2) * m + b], inv);
    nxt[r] = cfms(cur[(i + 2) * m + j + 2], Lf, cur[b * m + j + 2]);
  }
  __syncthreads();
}

// Last two levels of a 5x5 node in registers: children on pivots 0/1, then the four
// leaves, each leaf term (-1)^|a| det(s2)^2 * (1x1 Schur complement) written without
// division as Db^2 T_cc (T_cc T_ee - T_ce T_ec).
__device__ __forceinline__ void tree_bottom5r(const double2 (&s)[25], double2 D, int parity, double floor_,
                                              bool want_scale, double2 &sum, double &scale, bool &guard) {
  sum = c2(0.0, 0.0);
  scale = 0.0;
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    double2 piv = s[b * 6];
    if (!(cabs1(piv) >= floor_)) guard = true;
    double2 inv = crcp(piv);
    double2 Db = cmul(D, piv);
    double2 T[9];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double2 Lf = cmul(s[(i + 2) * 5 + b], inv);
#pragma unroll
      for (int j = 0; j < 3; ++j) T[i * 3 + j] = cfms(s[(i + 2) * 5 + j + 2], Lf, s[b * 5 + j + 2]);
    }
    double2 Db2 = cmul(Db, Db);
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      double2 q = cmul(T[c * 4], cfms(cmul(T[c * 4], T[8]), T[c * 3 + 2], T[6 + c]));
      double2 term = cmul(Db2, q);
      if ((b ^ c) & 1)
        sum = c2(sum.x - term.x, sum.y - term.y);
      else
        sum = cadd(sum, term);
      if (want_scale) scale += cabs(term);
    }
  }
  if (parity & 1) sum = c2(-sum.x, -sum.y);
}

__device__ __forceinline__ void tree_bottom5(const double2 *R, double2 D, int parity, double floor_, bool want_scale,
                                             double2 &sum, double &scale, bool &guard) {
  double2 s[25];
#pragma unroll
  for (int i = 0; i < 25; ++i) s[i] = R[i];
  tree_bottom5r(s, D, parity, floor_, want_scale, sum, scale, guard);
}

// Grandchild (b, bp) of a 7x7 node (shared memory; rows 0,1: vertex k, 2,3: vertex k+1,
// 4,5: vertex k+2, 6: external) in registers: eliminate row b, then row 2 + bp of the
// child, leaving the 3x3 Schur complement T over rows {4, 5, 6}; then its two leaves,
// each (-1)^|a| det(s2)^2 T_cc (T_cc T_ee - T_ce T_ec). Only the child's entries that T
// needs are formed (rows and columns 2 + bp, 4, 5, 6), each as the two-level scheme forms it.
__device__ __forceinline__ void tree_bottom7q(const double2 *S, double2 D, int b, int bp, int parity, double floor_,
                                              bool want_scale, double2 &sum, double &scale, bool &guard) {
  const double2 p1 = S[b * 8];
  if (!(cabs1(p1) >= floor_)) guard = true;
  const double2 i1 = crcp(p1);
  const int c0 = 2 + bp;
  // child row c0 at columns c0, 4, 5, 6
  double2 a0[4];
  {
    const double2 Lf = cmul(S[c0 * 7 + b], i1);
    a0[0] = cfms(S[c0 * 7 + c0], Lf, S[b * 7 + c0]);
#pragma unroll
    for (int j = 0; j < 3; ++j) a0[j + 1] = cfms(S[c0 * 7 + 4 + j], Lf, S[b * 7 + 4 + j]);
  }
  const double2 p2 = a0[0];
  if (!(cabs1(p2) >= floor_)) guard = true;
  const double2 i2 = crcp(p2);
  double2 T[9];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const int ri = 4 + r;
    const double2 Lf = cmul(S[ri * 7 + b], i1);
    const double2 ar0 = cfms(S[ri * 7 + c0], Lf, S[b * 7 + c0]);
    const double2 L2 = cmul(ar0, i2);
#pragma unroll
    for (int j = 0; j < 3; ++j) T[r * 3 + j] = cfms(cfms(S[ri * 7 + 4 + j], Lf, S[b * 7 + 4 + j]), L2, a0[j + 1]);
  }
  const double2 Db = cmul(cmul(D, p1), p2);
  const double2 Db2 = cmul(Db, Db);
  sum = c2(0.0, 0.0);
  scale = 0.0;
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const double2 q = cmul(T[c * 4], cfms(cmul(T[c * 4], T[8]), T[c * 3 + 2], T[6 + c]));
    const double2 term = cmul(Db2, q);
    if ((b ^ bp ^ c) & 1)
      sum = c2(sum.x - term.x, sum.y - term.y);
    else
      sum = cadd(sum, term);
    if (want_scale) scale += cabs(term);
  }
  if (parity & 1) sum = c2(-sum.x, -sum.y);
}

// Sums (v, sc) over aligned groups of G consecutive threads (G a power of two <= TREE_THREADS)
// and adds group g's sum to fval[g], fscale[g] for g < ngroups. Fixed shuffle pattern:
// deterministic. Every thread of the CTA calls it.
__device__ void group_sum(double2 v, double sc, int G, int ngroups, double2 *fval, double *fscale, double2 *wsum,
                          double *wscale) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gw = G < 32 ? G : 32;
  for (int off = 1; off < gw; off <<= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
    sc += __shfl_xor_sync(0xffffffffu, sc, off);
  }
  if (G <= 32) {
    const int g = tid / G;
    if ((lane & (G - 1)) == 0 && g < ngroups) {
      fval[g] = cadd(fval[g], v);
      fscale[g] += sc;
    }
    __syncthreads();
  } else {
    if (lane == 0) {
      wsum[warp] = v;
      wscale[warp] = sc;
    }
    __syncthreads();
    const int wpg = G / 32;
    if (tid < ngroups) {
      double2 f = fval[tid];
      double s2 = fscale[tid];
      for (int w = tid * wpg; w < (tid + 1) * wpg; ++w) {
        f = cadd(f, wsum[w]);
        s2 += wscale[w];
      }
      fval[tid] = f;
      fscale[tid] = s2;
    }
    __syncthreads();
  }
}

// Great-grandchild (b, bp, bq) of a 9x9 node (shared memory; rows 0,1: vertex k, 2,3:
// vertex k+1, 4,5: vertex k+2, 6,7: vertex k+3, 8: external) in registers: the
// eliminations of row b, then 2 + bp, then 4 + bq, every entry formed as the breadth-first
// levels and tree_bottom7q form it (so each leaf term is the same number), leaving the
// 3x3 Schur complement T over rows {6, 7, 8}; then its two leaves,
// each (-1)^|a| det(s2)^2 T_cc (T_cc T_ee - T_ce T_ec).
__device__ __forceinline__ void tree_bottom9(const double2 *S, double2 D, int b, int bp, int bq, int parity,
                                             double floor_, bool want_scale, double2 &sum, double &scale,
                                             bool &guard) {
  constexpr int W = 9;
  const int c = 2 + bp, d = 4 + bq;
  const int cols[5] = {c, d, 6, 7, 8};
  const double2 p1 = S[b * W + b];
  if (!(cabs1(p1) >= floor_)) guard = true;
  const double2 i1 = crcp(p1);
  double2 rb[5]; // row b at the columns that remain needed
#pragma unroll
  for (int k = 0; k < 5; ++k) rb[k] = S[b * W + cols[k]];
  // child row c (first elimination) at columns {c, d, 6, 7, 8}
  double2 rc[5];
  {
    const double2 Lf = cmul(S[c * W + b], i1);
#pragma unroll
    for (int k = 0; k < 5; ++k) rc[k] = cfms(S[c * W + cols[k]], Lf, rb[k]);
  }
  const double2 p2 = rc[0];
  if (!(cabs1(p2) >= floor_)) guard = true;
  const double2 i2 = crcp(p2);
  // grandchild row d (second elimination) at columns {d, 6, 7, 8}
  double2 rd[4];
  {
    const double2 Lf = cmul(S[d * W + b], i1);
    const double2 a = cfms(S[d * W + c], Lf, rb[0]);
    const double2 L2 = cmul(a, i2);
#pragma unroll
    for (int k = 0; k < 4; ++k) rd[k] = cfms(cfms(S[d * W + cols[k + 1]], Lf, rb[k + 1]), L2, rc[k + 1]);
  }
  const double2 p3 = rd[0];
  if (!(cabs1(p3) >= floor_)) guard = true;
  const double2 i3 = crcp(p3);
  // T row r - 6 at columns {6, 7, 8} (third elimination)
  double2 T[9];
#pragma unroll
  for (int rr = 0; rr < 3; ++rr) {
    const int r = 6 + rr;
    const double2 Lf = cmul(S[r * W + b], i1);
    const double2 a0 = cfms(S[r * W + c], Lf, rb[0]);
    const double2 L2 = cmul(a0, i2);
    const double2 a1 = cfms(cfms(S[r * W + d], Lf, rb[1]), L2, rc[1]);
    const double2 L3 = cmul(a1, i3);
#pragma unroll
    for (int j = 0; j < 3; ++j)
      T[rr * 3 + j] = cfms(cfms(cfms(S[r * W + 6 + j], Lf, rb[2 + j]), L2, rc[2 + j]), L3, rd[1 + j]);
  }
  const double2 Db = cmul(cmul(cmul(D, p1), p2), p3);
  const double2 Db2 = cmul(Db, Db);
  sum = c2(0.0, 0.0);
  scale = 0.0;
#pragma unroll
  for (int cc = 0; cc < 2; ++cc) {
    const double2 q = cmul(T[cc * 4], cfms(cmul(T[cc * 4], T[8]), T[cc * 3 + 2], T[6 + cc]));
    const double2 term = cmul(Db2, q);
    if ((b ^ bp ^ bq ^ cc) & 1)
      sum = c2(sum.x - term.x, sum.y - term.y);
    else
      sum = cadd(sum, term);
    if (want_scale) scale += cabs(term);
  }
  if (parity & 1) sum = c2(-sum.x, -sum.y);
}

// Per-point sums of the fused bottom (thread q * NODES + node, 2^lg nodes per point): lane
// groups of consecutive nodes by shuffles, then each point's groups and the
// TREE_THREADS / NODES descendant slots q in a fixed order by thread p; adds to fval[p],
// fscale[p]. Every thread calls it; scratch: 256 double2 + 256 double of free shared memory
// (BOTTOM_SCRATCH entries), read until the caller's next barrier.
template <int NODES>
__device__ void bottom_sum(double2 v, double sc, int lg, int np, double2 *fval, double *fscale, double2 *scratch) {
  static_assert(NODES >= 16 && NODES * (TREE_THREADS / NODES) == TREE_THREADS, "descendant slots of the CTA");
  const int tid = threadIdx.x, lane = tid & 31;
  const int g = lg < 5 ? (1 << lg) : 32;
  for (int off = 1; off < g; off <<= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
    sc += __shfl_xor_sync(0xffffffffu, sc, off);
  }
  double *sscale = reinterpret_cast<double *>(scratch + TREE_THREADS);
  if ((lane & (g - 1)) == 0) {
    scratch[tid] = v;
    sscale[tid] = sc;
  }
  __syncthreads();
  if (tid < np) {
    const int per = 1 << lg;
    double2 f = fval[tid];
    double s2 = fscale[tid];
    for (int q = 0; q < TREE_THREADS / NODES; ++q)
      for (int nd = tid * per; nd < (tid + 1) * per; nd += g) {
        f = cadd(f, scratch[q * NODES + nd]);
        s2 += sscale[q * NODES + nd];
      }
    fval[tid] = f;
    fscale[tid] = s2;
  }
}

// Order 1: the 3x3 root's two leaves directly.
__device__ __forceinline__ void tree_bottom3(const double2 *R, double2 &sum, double &scale, bool want_scale) {
  sum = c2(0.0, 0.0);
  scale = 0.0;
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    double2 piv = R[b * 4];
    double2 term = cmul(piv, cfms(cmul(piv, R[8]), R[b * 3 + 2], R[6 + b]));
    if (b)
      sum = c2(sum.x - term.x, sum.y - term.y);
    else
      sum = cadd(sum, term);
    if (want_scale) scale += cabs(term);
  }
}

// One sub-batch of np points (N <= TREE_MAX_SUB, or the subtree of a path pass) whose
// root matrices sit at `root` in frontier buffer rb, with S.D[rb][node] their prefix
// determinants: the breadth-first levels, then the fused bottom, each point's sum added
// to fval[p] (fscale[p]) and bit 1 of flag[p] set where a pivot fell below the guard.
// pf_n > 0: copies pf_n staged entries from pf_src to the buffer the bottom does not read
// (at offset roff, past the bottom's scratch) while the bottom runs, for the next
// sub-batch. Returns the buffer the bottom read. The per-point sums are read from the
// bottom's scratch until the caller's next barrier.
__device__ int tree_sub(TreeShared &S, int N, int np, int rb, const double2 *root, int *flag, double2 *fval,
                        double *fscale, double floor_, bool want_scale, int parity0, const double2 *pf_src,
                        int pf_n, int roff) {
  const int tid = threadIdx.x;
  // breadth-first levels down to 9x9 nodes, then the fused bottom of three eliminations;
  // orders 3 and 4 go down to 7x7 nodes and a bottom of two (three were 4 % slower at 4)
  const int LB = N >= 5 ? N - 4 : (N >= 3 ? N - 3 : 0);
  int m = 2 * N + 1, cur = rb, nodes = np, lg = 0;
  const double2 *src = root;
  for (int k = 0; k + 1 < LB; k += 2) { // pairs of levels, then a last single one
    tree_level4(src, S.buf[cur ^ 1], S.D[cur], S.D[cur ^ 1], flag, nodes, lg, m, floor_, S.tmp);
    nodes *= 4;
    lg += 2;
    m -= 4;
    cur ^= 1;
    src = S.buf[cur];
  }
  if (LB & 1) {
    tree_level2(src, S.buf[cur ^ 1], S.D[cur], S.D[cur ^ 1], S.tmp, flag, nodes, lg, m, floor_);
    nodes *= 2;
    lg += 1;
    m -= 2;
    cur ^= 1;
    src = S.buf[cur];
  }
  if (pf_n > 0) copy_roots(S.buf[cur ^ 1] + roff, pf_src, pf_n);
  double2 v = c2(0.0, 0.0);
  double sc = 0.0;
  bool guard = false;
  int p = 0;
  if (m == 7) { // four threads per 7x7 node: grandchild tid >> 5 of node tid & 31, so that a
                // warp's lanes read consecutive nodes (49-entry stride: no bank conflicts)
    const int node = tid & 31, q = tid >> 5;
    if (node < nodes) {
      p = node >> lg;
      const int parity = __popc(node & ((1 << lg) - 1)) + parity0;
      tree_bottom7q(src + node * 49, S.D[cur][node], q >> 1, q & 1, parity, floor_, want_scale, v, sc, guard);
    }
    if (guard) flag[p] |= 2;
    bottom_sum<32>(v, sc, lg, np, fval, fscale, S.buf[cur ^ 1]);
  } else if (m == 9) { // eight threads per 9x9 node: great-grandchild tid >> 4 of node tid & 15
    const int node = tid & 15, q = tid >> 4;
    if (node < nodes) {
      p = node >> lg;
      const int parity = __popc(node & ((1 << lg) - 1)) + parity0;
      tree_bottom9(src + node * 81, S.D[cur][node], q >> 2, (q >> 1) & 1, q & 1, parity, floor_, want_scale, v, sc,
                   guard);
    }
    if (guard) flag[p] |= 2;
    bottom_sum<16>(v, sc, lg, np, fval, fscale, S.buf[cur ^ 1]);
  } else { // orders 1 and 2: the root itself, one thread per point
    if (tid < nodes) {
      p = tid;
      if (m == 5)
        tree_bottom5(src + tid * 25, S.D[cur][tid], parity0, floor_, want_scale, v, sc, guard);
      else
        tree_bottom3(src + tid * 9, v, sc, want_scale);
    }
    if (guard) flag[p] |= 2;
    group_sum(v, sc, 1, np, fval, fscale, S.wsum, S.wscale);
  }
  return cur;
}

// Where a sub-batch's roots go when they are copied while the previous sub-batch's bottom
// runs: past the bottom's scratch (orders 3 and up) of the buffer the bottom does not read.
// -1: they do not fit beside it (order 3); those sub-batches copy theirs after a barrier.
__device__ __forceinline__ int tree_prefetch_offset(int N, int P) {
  const int off = N >= 3 ? BOTTOM_SCRATCH : 0;
  return off + P * (2 * N + 1) * (2 * N + 1) <= FRONTIER ? off : -1;
}

// The G-batch's points (gb, staged G at gst: point p at p M^2): the integrand of each,
// added to S.fval[p] (S.fscale[p]) with bit 1 of S.flag[p] set where a pivot fell below
// the guard. S.D and the frontier buffers are free on entry; the caller's barrier follows.
__device__ void tree_gbatch_points(TreeShared &S, const ItemDev &it, int N, int gb, double2 *gst,
                                   bool want_scale, bool direct, int *bad) {
  const int tid = threadIdx.x;
  const int M = 2 * N + 1, MM = M * M;
  const double floor_ = it.model.pivot_floor;
  if (N == 0) {
    if (tid < gb && !(S.flag[tid] & 1)) {
      kb_gf_index a = it.f.A, b = it.f.B;
      a.timesplit = 0;
      b.timesplit = 0;
      double2 v = g0_contour(it.model, a, b, 0, bad);
      S.fval[tid] = v;
      S.fscale[tid] = cabs(v);
    }
    return;
  }
  if (N > TREE_MAX_SUB) {
    // one point at a time: the K0 = N - 8 levels above the order-8 subtrees. The last one
    // (order 9) or two of them run breadth-first (tree_level2 / tree_level4 on one node) into
    // the staging area after the batch's G matrices, 2^Kb subtree roots of 17 x 17 and their
    // prefix determinants; the Kp levels before them are walked one root-to-node path at a
    // time (2^Kp passes, the point's G copied again for each). Against walking all K0 levels
    // by paths: orders 10 / 12 -4 / -20 %, order 9 +7 % (its one breadth-first level computes
    // what its two paths did, through the staging area; the code that kept paths for order 9
    // compiled into a kernel 13 % slower at order 10). Each subtree root is copied into shared memory
    // asynchronously while the previous subtree's bottom runs. Subtrees are summed in the
    // order of their path bits, first level first, as walking all K0 levels by paths would.
    const int K0 = N - TREE_MAX_SUB;
    const int Kb = K0 >= 2 ? 2 : 1, Kp = K0 - Kb, NS = 1 << Kb;
    constexpr int R = 2 * TREE_MAX_SUB + 1, RR = R * R;
    double2 *gsub = gst + (size_t)gb * MM;
    double2 *gD = gsub + (size_t)NS * RR;
    const int pf = tree_prefetch_offset(TREE_MAX_SUB, 1);
    for (int p = 0; p < gb; ++p) {
      for (int sub = 0; sub < (1 << Kp); ++sub) {
        copy_roots(S.buf[0], gst + (size_t)p * MM, MM);
        if (tid == 0) S.D[0][0] = c2(1.0, 0.0);
        cp_async_wait_all();
        __syncthreads();
        int m = M, cur = 0;
        for (int k = 0; k < Kp; ++k) {
          const int b = (sub >> (Kp - 1 - k)) & 1;
          tree_path_step(S.buf[cur], S.buf[cur ^ 1], S.D[cur], S.D[cur ^ 1], S.flag + p, m, b, floor_);
          m -= 2;
          cur ^= 1;
        }
        if (Kb == 2)
          tree_level4(S.buf[cur], gsub, S.D[cur], gD, S.flag + p, 1, 0, m, floor_, S.tmp);
        else
          tree_level2(S.buf[cur], gsub, S.D[cur], gD, S.tmp, S.flag + p, 1, 0, m, floor_);
        int rb = 0, roff = 0;
        for (int g = 0; g < NS; ++g) {
          if (g == 0) {
            copy_roots(S.buf[0], gsub, RR);
            if (tid == 0) S.D[0][0] = gD[0];
            cp_async_wait_all();
            __syncthreads();
          }
          const bool prefetch = pf >= 0 && g + 1 < NS;
          const int bot = tree_sub(S, TREE_MAX_SUB, 1, rb, S.buf[rb] + roff, S.flag + p, S.fval + p, S.fscale + p,
                                   floor_, want_scale, __popc(sub) + __popc(g), gsub + (size_t)(g + 1) * RR,
                                   prefetch ? RR : 0, pf);
          if (prefetch) {
            rb = bot ^ 1;
            roff = pf;
            if (tid == 0) S.D[rb][0] = gD[g + 1];
            cp_async_wait_all();
          }
          __syncthreads();
        }
      }
    }
    return;
  }
  const int P = tree_points_per_chunk(N);
  const int pf = tree_prefetch_offset(N, P);
  int rb = 0, roff = 0;
  for (int sb = 0; sb < gb; sb += P) {
    const int np = min(P, gb - sb);
    if (sb == 0 || pf < 0) { // copy this sub-batch's roots now (direct: built there already)
      rb = 0;
      roff = 0;
      if (!direct) copy_roots(S.buf[0], gst + (size_t)sb * MM, np * MM);
      if (tid < np) S.D[0][tid] = c2(1.0, 0.0);
      cp_async_wait_all();
      __syncthreads();
    }
    const int nsb = sb + P, nnp = min(P, gb - nsb);
    const bool prefetch = pf >= 0 && nnp > 0;
    const int bot = tree_sub(S, N, np, rb, S.buf[rb] + roff, S.flag + sb, S.fval + sb, S.fscale + sb, floor_,
                             want_scale, 0, gst + (size_t)nsb * MM, prefetch ? nnp * MM : 0, pf);
    if (prefetch) {
      rb = bot ^ 1;
      roff = pf;
      if (tid < nnp) S.D[rb][tid] = c2(1.0, 0.0);
      cp_async_wait_all();
    }
    __syncthreads();
  }
}

__device__ __forceinline__ double2 apply_cutoff(double2 f, double cutoff) {
  return (cabs(f) < cutoff) ? c2(0.0, 0.0) : f;
}

// Zeroes chunk c's bins (all threads of the CTA; a barrier follows before their use).
__device__ __forceinline__ void clear_bins(const Launch &L, int c) {
  if (!L.nbins) return;
  for (int b = threadIdx.x; b < L.nbins; b += blockDim.x) {
    L.bin_sums[(size_t)c * L.nbins + b] = c2(0.0, 0.0);
    L.bin_counts[(size_t)c * L.nbins + b] = 0u;
  }
  if (threadIdx.x == 0) L.bin_dropped[c] = 0u;
}

// Persistent CTAs pull chunks of up to 128 points. Per chunk: the points' set-up (Sobol
// coordinates or given inputs, warper chain, domain flag: one thread per point) into the
// CTA's global slot; then per G-batch of tree_gbatch(N) points: every table lookup of the
// batch in flight at once (build_G into the slot's staging area), then the trees of its
// sub-batches, each sub-batch's G copied into shared memory asynchronously while the
// previous sub-batch's bottom runs; then the batch's values in point order.
template <bool EVAL, bool ANY_CUBIC>
__global__ void __launch_bounds__(TREE_THREADS, 4) tree_kernel(Launch L) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TreeShared &S = *reinterpret_cast<TreeShared *>(smem_raw);
  __shared__ int s_chunk;
  __shared__ int s_bad;
  // the chunk's partial sums and dropped count (thread 0), in shared memory so that they
  // hold no registers through the tree
  __shared__ ChunkPartial s_part;
  __shared__ unsigned s_drop;
  __shared__ unsigned s_bal[3][TREE_THREADS / 32]; // per warp: in-domain, guarded and dropped points of a batch
  const int tid = threadIdx.x;
  if (tid == 0) s_bad = 0;
  for (;;) {
    if (tid == 0) {
      s_chunk = atomicAdd(L.chunk_counter, 1);
      s_part.sum_re = s_part.sum_im = 0.0;
      s_part.n_in_domain = s_part.n_fallback = 0;
      s_part.fb_mask[0] = s_part.fb_mask[1] = 0;
      s_drop = 0;
    }
    __syncthreads();
    const int c = s_chunk;
    if (c >= L.n_chunks) break;
    const int item = find_item(L.chunk_offsets, L.n_items, c);
    const ItemDev &it = L.items[item];
    const long long cfirst = (long long)(c - L.chunk_offsets[item]) * it.chunk_points;
    const long long total = EVAL ? (L.index ? (long long)L.n_index : it.n_points) : it.n_points;
    const int ccount = (int)min((long long)it.chunk_points, total - cfirst);
    const int N = it.order;
    const int GB = tree_gbatch(N);
    const bool keep = (L.mode == IN_SOBOL) ? true : (L.keep_u_hypercube != 0);
    const bool want_scale = EVAL && L.out_scale != nullptr;
    double *slot = L.pts + (size_t)blockIdx.x * PTS_SLOT;
    double2 *gst = reinterpret_cast<double2 *>(slot + PTS_ROWS);
    if (tid < ccount) prepare_point(L, it, N, cfirst + tid, keep, slot, tid);
    __syncthreads();
    for (int g0 = 0; g0 < ccount; g0 += GB) {
      const int gb = min(GB, ccount - g0);
      if (tid < gb) {
        for (int j = 0; j < N; ++j) S.u[j * gb + tid] = slot[j * CHUNK_POINTS + g0 + tid];
        S.jac[tid] = slot[MAX_ORDER * CHUNK_POINTS + g0 + tid];
        S.flag[tid] = (int)slot[(MAX_ORDER + 1) * CHUNK_POINTS + g0 + tid];
        S.fval[tid] = c2(0.0, 0.0);
        S.fscale[tid] = 0.0;
      }
      __syncthreads();
      const bool direct = tree_direct(N);
      if (N > 0) {
        if (direct) // the batch is one sub-batch: G straight into the frontier buffer
          build_G_any<ANY_CUBIC, 2>(it, N, gb, S.u, S.flag, S.buf[0], it.f.A.spin, &s_bad);
        else
          build_G_any<ANY_CUBIC, 4>(it, N, gb, S.u, S.flag, gst, it.f.A.spin, &s_bad);
        __syncthreads();
      }
      tree_gbatch_points(S, it, N, gb, gst, want_scale, direct, &s_bad);
      if (EVAL) {
        if (tid < gb) {
          const long long o = cfirst + g0 + tid;
          int fl = S.flag[tid];
          const double2 fv = S.fval[tid];
          if (!isfinite(fv.x) || !isfinite(fv.y)) fl |= 2;
          const bool dom = !(fl & 1);
          const double2 f = dom ? apply_cutoff(fv, it.f.cutoff) : c2(0.0, 0.0);
          const double j = S.jac[tid];
          L.out_val[o] = c2(f.x * j, f.y * j);
          if (L.out_jac) L.out_jac[o] = j;
          if (L.out_dom) L.out_dom[o] = dom ? 1 : 0;
          if (L.out_scale) L.out_scale[o] = dom ? S.fscale[tid] * fabs(j) : 0.0;
          if (L.out_flag) L.out_flag[o] = (dom && (fl & 2)) ? 1 : 0;
        }
      } else {
        // the batch's point values, one thread per point; then each warp's sum in a fixed
        // shuffle order, and thread 0 adds the warps in order (deterministic)
        const int lane = tid & 31, w = tid >> 5;
        bool dom = false, fb = false, drop = false;
        double2 fj = c2(0.0, 0.0);
        if (tid < gb) {
          int fl = S.flag[tid];
          const double2 fv = S.fval[tid];
          if (!isfinite(fv.x) || !isfinite(fv.y)) fl |= 2;
          const int q = g0 + tid;
          int bin = -2;
          if (L.nbins) { // the code prepare_point stored: 2 bin, or -1 when dropped
            const double code = slot[BIN_CODE_ROW * CHUNK_POINTS + q];
            bin = code < 0.0 ? -1 : (int)code >> 1;
            drop = bin < 0;
          }
          if (!(fl & 1)) {
            dom = true;
            fb = (fl & 2) != 0;
            if (!fb) {
              const double2 f = apply_cutoff(fv, it.f.cutoff);
              const double j = S.jac[tid];
              fj = c2(f.x * j, f.y * j);
              if (bin >= 0) {
                slot[BIN_CODE_ROW * CHUNK_POINTS + q] = (double)(2 * bin + 1);
                slot[(BIN_CODE_ROW + 1) * CHUNK_POINTS + q] = fj.x;
                slot[(BIN_CODE_ROW + 2) * CHUNK_POINTS + q] = fj.y;
              }
            }
          }
        }
        for (int off = 16; off > 0; off >>= 1) {
          fj.x += __shfl_xor_sync(0xffffffffu, fj.x, off);
          fj.y += __shfl_xor_sync(0xffffffffu, fj.y, off);
        }
        const unsigned bdom = __ballot_sync(0xffffffffu, dom), bfb = __ballot_sync(0xffffffffu, fb);
        const unsigned bdrop = __ballot_sync(0xffffffffu, drop);
        if (lane == 0) {
          S.wsum[w] = fj;
          s_bal[0][w] = bdom;
          s_bal[1][w] = bfb;
          s_bal[2][w] = bdrop;
        }
        __syncthreads();
        if (tid == 0) {
          double2 csum = c2(s_part.sum_re, s_part.sum_im);
          unsigned long long cdom = s_part.n_in_domain, cfb = s_part.n_fallback;
          unsigned long long mask0 = s_part.fb_mask[0], mask1 = s_part.fb_mask[1];
          unsigned cdrop = s_drop;
          for (int k = 0; k < TREE_THREADS / 32; ++k) {
            csum = cadd(csum, S.wsum[k]);
            cdom += __popc(s_bal[0][k]);
            cfb += __popc(s_bal[1][k]);
            cdrop += __popc(s_bal[2][k]);
            // guarded points' chunk bits: point q = g0 + 32 k + lane
            const unsigned long long m = s_bal[1][k];
            const int b0 = g0 + 32 * k;
            if (m && b0 < 64) {
              mask0 |= m << b0;
              if (b0 > 32) mask1 |= m >> (64 - b0);
            } else if (m) {
              mask1 |= m << (b0 - 64);
            }
          }
          s_part.sum_re = csum.x;
          s_part.sum_im = csum.y;
          s_part.n_in_domain = cdom;
          s_part.n_fallback = cfb;
          s_part.fb_mask[0] = mask0;
          s_part.fb_mask[1] = mask1;
          s_drop = cdrop;
        }
      }
      __syncthreads();
    }
    if (!EVAL && L.nbins) {
      // the chunk's bins with its points added in point order (the order of one thread
      // walking the chunk): one thread per bin for up to 512 bins, else one thread over the
      // points; the pivoted-LU pass adds its points later
      const double *code = slot + BIN_CODE_ROW * CHUNK_POINTS;
      const double *vre = code + CHUNK_POINTS, *vim = vre + CHUNK_POINTS;
      if (L.nbins <= 512) {
        for (int b = tid; b < L.nbins; b += blockDim.x) {
          double2 bs = c2(0.0, 0.0);
          unsigned cnt = 0;
          for (int q = 0; q < ccount; ++q) {
            if (code[q] < 0.0 || (int)code[q] >> 1 != b) continue;
            cnt++;
            if ((int)code[q] & 1) bs = c2(bs.x + vre[q], bs.y + vim[q]);
          }
          L.bin_sums[(size_t)c * L.nbins + b] = bs;
          L.bin_counts[(size_t)c * L.nbins + b] = cnt;
        }
      } else {
        clear_bins(L, c);
        __syncthreads();
        if (tid == 0)
          for (int q = 0; q < ccount; ++q) {
            if (code[q] < 0.0) continue;
            const int b = (int)code[q] >> 1;
            L.bin_counts[(size_t)c * L.nbins + b]++;
            if ((int)code[q] & 1) {
              double2 &bs = L.bin_sums[(size_t)c * L.nbins + b];
              bs = c2(bs.x + vre[q], bs.y + vim[q]);
            }
          }
      }
      if (tid == 0) L.bin_dropped[c] = s_drop;
    }
    if (!EVAL && tid == 0) L.partials[c] = s_part;
  }
  if (tid == 0 && s_bad) atomicOr(L.err, 1);
}

// ---------------------------------------------------------------- direct kernel

struct DirectShared {
  double2 G1[(2 * MAX_ORDER + 1) * (2 * MAX_ORDER + 1)];
  double2 G2[(2 * MAX_ORDER + 1) * (2 * MAX_ORDER + 1)];
  double u[MAX_ORDER];
  double jac[1];
  int flag[1];
  double2 red[NT];
  double reds[NT];
};

// det of the n x n row-major matrix a (destroyed): partial pivoting on the first
// maximum of |re|+|im| in the column, multipliers with the pivot's reciprocal.
__device__ double2 lu_det(double2 *a, int n) {
  double2 det = c2(1.0, 0.0);
  bool neg = false;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = cabs1(a[k * n + k]);
    for (int i = k + 1; i < n; ++i) {
      double v = cabs1(a[i * n + k]);
      if (v > best) {
        best = v;
        p = i;
      }
    }
    if (best == 0.0) return c2(0.0, 0.0);
    if (p != k) {
      for (int j = 0; j < n; ++j) {
        double2 t = a[k * n + j];
        a[k * n + j] = a[p * n + j];
        a[p * n + j] = t;
      }
      neg = !neg;
    }
    double2 piv = a[k * n + k];
    det = cmul(det, piv);
    double2 inv = crcp(piv);
    for (int i = k + 1; i < n; ++i) {
      double2 l = cmul(a[i * n + k], inv);
      for (int j = k + 1; j < n; ++j) a[i * n + j] = cfms(a[i * n + j], l, a[k * n + j]);
    }
  }
  return neg ? c2(-det.x, -det.y) : det;
}

// The integrand of one point (inputs in D.u / D.flag): keldy's algorithm.
__device__ __forceinline__ void direct_point(DirectShared &D, const ItemDev &it, int N, bool want_scale, double2 &f_out,
                             double &scale_out, int *bad) {
  const int tid = threadIdx.x;
  if (D.flag[0] & 1) {
    f_out = c2(0.0, 0.0);
    scale_out = 0.0;
    return;
  }
  if (N == 0) {
    if (tid == 0) {
      kb_gf_index a = it.f.A, b = it.f.B;
      a.timesplit = 0;
      b.timesplit = 0;
      D.red[0] = g0_contour(it.model, a, b, 0, bad);
      D.reds[0] = cabs(D.red[0]);
    }
    __syncthreads();
    f_out = D.red[0];
    scale_out = D.reds[0];
    __syncthreads();
    return;
  }
  const int M = 2 * N + 1;
  const int spin = it.f.A.spin;
  build_G_any<true>(it, N, 1, D.u, D.flag, D.G1, spin, bad);
  const double2 *G2 = D.G1;
  if (!it.spin_symmetric) {
    build_G_any<true>(it, N, 1, D.u, D.flag, D.G2, 1 - spin, bad);
    G2 = D.G2;
  }
  __syncthreads();
  double2 acc = c2(0.0, 0.0);
  double sc = 0.0;
  double2 m1[(MAX_ORDER + 1) * (MAX_ORDER + 1)];
  double2 m2[MAX_ORDER * MAX_ORDER];
  int pick[MAX_ORDER + 1];
  const unsigned nconf = 1u << N;
  for (unsigned cfg = tid; cfg < nconf; cfg += blockDim.x) {
    for (int i = 0; i < N; ++i) pick[i] = 2 * i + ((cfg >> i) & 1u);
    pick[N] = 2 * N;
    for (int i = 0; i <= N; ++i)
      for (int j = 0; j <= N; ++j) m1[i * (N + 1) + j] = D.G1[pick[i] * M + pick[j]];
    m1[N * (N + 1) + N] = c2(0.0, 0.0);
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) m2[i * N + j] = G2[pick[i] * M + pick[j]];
    double2 d = cmul(lu_det(m1, N + 1), lu_det(m2, N));
    if (__popc(cfg) & 1)
      acc = c2(acc.x - d.x, acc.y - d.y);
    else
      acc = cadd(acc, d);
    if (want_scale) sc += cabs(d);
  }
  D.red[tid] = acc;
  D.reds[tid] = sc;
  __syncthreads();
  if (tid == 0) {
    double2 s = c2(0.0, 0.0);
    double ss = 0.0;
    for (int t = 0; t < (int)blockDim.x; ++t) {
      s = cadd(s, D.red[t]);
      ss += D.reds[t];
    }
    D.red[0] = s;
    D.reds[0] = ss;
  }
  __syncthreads();
  f_out = D.red[0];
  scale_out = D.reds[0];
  __syncthreads();
}

__device__ void direct_load_point(const Launch &L, const ItemDev &it, int N, long long gp, bool keep,
                                  DirectShared &D) {
  load_points(L, it, N, 1, gp, D.u, D.jac, D.flag, keep);
  __syncthreads();
}

// Modes: IN_TIMES / IN_LI (every point, or the points of L.index), IN_SOBOL (per-chunk
// partial sums, as the tree kernel).
__global__ void __launch_bounds__(NT) direct_kernel(Launch L) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  DirectShared &D = *reinterpret_cast<DirectShared *>(smem_raw);
  __shared__ int s_chunk;
  __shared__ int s_bad;
  const int tid = threadIdx.x;
  if (tid == 0) s_bad = 0;
  const bool eval = L.mode != IN_SOBOL;
  for (;;) {
    if (tid == 0) s_chunk = atomicAdd(L.chunk_counter, 1);
    __syncthreads();
    const int c = s_chunk;
    if (c >= L.n_chunks) break;
    const int item = find_item(L.chunk_offsets, L.n_items, c);
    const ItemDev &it = L.items[item];
    const long long cfirst = (long long)(c - L.chunk_offsets[item]) * it.chunk_points;
    const long long total = eval ? (L.index ? (long long)L.n_index : it.n_points) : it.n_points;
    const int ccount = (int)min((long long)it.chunk_points, total - cfirst);
    const int N = it.order;
    const bool keep = eval ? (L.keep_u_hypercube != 0) : true;
    double2 csum = c2(0.0, 0.0);
    unsigned long long cdom = 0;
    if (!eval) {
      clear_bins(L, c);
      __syncthreads();
    }
    for (int p = 0; p < ccount; ++p) {
      long long gp = cfirst + p;
      direct_load_point(L, it, N, gp, keep, D);
      double2 f;
      double sc;
      direct_point(D, it, N, eval && L.out_scale != nullptr, f, sc, &s_bad);
      if (tid == 0) {
        bool dom = !(D.flag[0] & 1);
        double j = D.jac[0];
        f = dom ? apply_cutoff(f, it.f.cutoff) : c2(0.0, 0.0);
        if (eval) {
          long long o = L.index ? (long long)L.index[gp] : gp;
          L.out_val[o] = c2(f.x * j, f.y * j);
          if (L.out_jac) L.out_jac[o] = j;
          if (L.out_dom) L.out_dom[o] = dom ? 1 : 0;
          if (L.out_scale) L.out_scale[o] = dom ? sc * fabs(j) : 0.0;
          if (L.out_flag) L.out_flag[o] = 0;
        } else {
          csum.x += f.x * j;
          csum.y += f.y * j;
          cdom += dom ? 1 : 0;
          if (L.nbins) {
            const int bin = time_bin(L, D.u, 1, N);
            if (bin < 0) {
              L.bin_dropped[c]++;
            } else {
              L.bin_counts[(size_t)c * L.nbins + bin]++;
              double2 &bs = L.bin_sums[(size_t)c * L.nbins + bin];
              bs = c2(bs.x + f.x * j, bs.y + f.y * j);
            }
          }
        }
      }
      __syncthreads();
    }
    if (!eval && tid == 0) {
      ChunkPartial pr;
      pr.sum_re = csum.x;
      pr.sum_im = csum.y;
      pr.n_in_domain = cdom;
      pr.n_fallback = 0;
      pr.fb_mask[0] = pr.fb_mask[1] = 0;
      L.partials[c] = pr;
    }
  }
  if (tid == 0 && s_bad) atomicOr(L.err, 1);
}

// Points the tree marked in a chunk's fb_mask, evaluated with keldy's algorithm and
// added to that chunk's partial sum in point order.
__global__ void __launch_bounds__(NT) fallback_kernel(Launch L) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  DirectShared &D = *reinterpret_cast<DirectShared *>(smem_raw);
  __shared__ int s_bad;
  const int tid = threadIdx.x;
  if (tid == 0) s_bad = 0;
  __syncthreads();
  for (int c = blockIdx.x; c < L.n_chunks; c += gridDim.x) {
    ChunkPartial pr = L.partials[c];
    if (pr.n_fallback == 0) continue;
    const int item = find_item(L.chunk_offsets, L.n_items, c);
    const ItemDev &it = L.items[item];
    const long long cfirst = (long long)(c - L.chunk_offsets[item]) * it.chunk_points;
    for (int bit = 0; bit < it.chunk_points; ++bit) {
      unsigned long long w = pr.fb_mask[bit >> 6];
      if (!((w >> (bit & 63)) & 1ull)) continue;
      direct_load_point(L, it, it.order, cfirst + bit, true, D);
      double2 f;
      double sc;
      direct_point(D, it, it.order, false, f, sc, &s_bad);
      if (tid == 0) {
        f = apply_cutoff(f, it.f.cutoff);
        pr.sum_re += f.x * D.jac[0];
        pr.sum_im += f.y * D.jac[0];
        if (L.nbins) { // counted by the tree kernel; the value is added here
          const int bin = time_bin(L, D.u, 1, it.order);
          if (bin >= 0) {
            double2 &bs = L.bin_sums[(size_t)c * L.nbins + bin];
            bs = c2(bs.x + f.x * D.jac[0], bs.y + f.y * D.jac[0]);
          }
        }
      }
      __syncthreads();
    }
    if (tid == 0) L.partials[c] = pr;
    __syncthreads();
  }
  if (tid == 0 && s_bad) atomicOr(L.err, 1);
}

// acc[item] += sum of the item's chunk partials: each thread adds a contiguous run of
// chunks in order, then the threads' sums are added in thread order (deterministic).
__global__ void __launch_bounds__(NT) reduce_kernel(Launch L, kb_accum *acc) {
  __shared__ double s_re[NT], s_im[NT];
  __shared__ unsigned long long s_dom[NT], s_fb[NT];
  const int item = blockIdx.x;
  const long long c0 = L.chunk_offsets[item], c1 = L.chunk_offsets[item + 1];
  const long long nc = c1 - c0;
  const long long per = (nc + NT - 1) / NT;
  const long long a = c0 + threadIdx.x * per, b = min(c1, a + per);
  double re = 0.0, im = 0.0;
  unsigned long long dom = 0, fb = 0;
  for (long long c = a; c < b; ++c) {
    ChunkPartial pr = L.partials[c];
    re += pr.sum_re;
    im += pr.sum_im;
    dom += pr.n_in_domain;
    fb += pr.n_fallback;
  }
  s_re[threadIdx.x] = re;
  s_im[threadIdx.x] = im;
  s_dom[threadIdx.x] = dom;
  s_fb[threadIdx.x] = fb;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int t = 1; t < NT; ++t) {
      re += s_re[t];
      im += s_im[t];
      dom += s_dom[t];
      fb += s_fb[t];
    }
    acc[item].sum_re += re;
    acc[item].sum_im += im;
    acc[item].n_points += (uint64_t)L.items[item].n_points;
    acc[item].n_in_domain += dom;
    acc[item].n_fallback += fb;
  }
}

// ------------------------------------------------------------ kernel method
// keldy's integrand_g_kernel (impurity_oneband/wick_kernel.cpp:42-138): with the fixed
// point X in the external slot, for every Keldysh configuration a the matrix s1 (X first,
// then the vertex copies picked by a; keldy zeroes its entry (n, n)) is factored with
// partial pivoting and the first row of its cofactor matrix is found by solving
// s1 x = det(s1) e_0 (first_row_expansion, det_expansion.hpp:44-74). Vertex i's term is
// x_{i+1} (-1)^|a| det(s2_a), accumulated at (vertex time, a_i). Here the terms of a point
// are summed per (vertex i, Keldysh index k) in configuration order (2n sums), then
// binned; keldy accumulates them one by one into the same bins.
// Threads of a km_tree_kernel CTA (two CTAs per SM: 16 warps); the points per pass stay
// sized for 128 (km_points_per_pass), the extra warps hide the levels' latency.
constexpr int KM_THREADS = 256;
struct KernelShared {
  double2 G1[(2 * KM_MAX_ORDER + 1) * (2 * KM_MAX_ORDER + 1)];
  double2 G2[(2 * KM_MAX_ORDER) * (2 * KM_MAX_ORDER)];
  double u[KM_MAX_ORDER];
  double jac[1];
  int flag[1];
  double2 X[KM_THREADS][KM_MAX_ORDER];
  double2 S[2 * KM_MAX_ORDER];
};

// LU with partial pivoting (first maximum of |re|+|im|) of the m x m matrix a, then the
// solve a x = det(a) e_0 (row interchanges, unit-lower then upper substitution).
__device__ void first_row_cofactors(double2 *a, int m, double2 *x) {
  int piv[KM_MAX_ORDER + 1];
  double2 det = c2(1.0, 0.0);
  bool neg = false;
  for (int k = 0; k < m; ++k) {
    int p = k;
    double best = cabs1(a[k * m + k]);
    for (int i = k + 1; i < m; ++i) {
      const double v = cabs1(a[i * m + k]);
      if (v > best) {
        best = v;
        p = i;
      }
    }
    piv[k] = p;
    if (p != k) {
      for (int j = 0; j < m; ++j) {
        const double2 t = a[k * m + j];
        a[k * m + j] = a[p * m + j];
        a[p * m + j] = t;
      }
      neg = !neg;
    }
    const double2 pv = a[k * m + k];
    det = cmul(det, pv);
    if (best == 0.0) continue;
    const double2 inv = crcp(pv);
    for (int i = k + 1; i < m; ++i) {
      const double2 l = cmul(a[i * m + k], inv);
      a[i * m + k] = l;
      for (int j = k + 1; j < m; ++j) a[i * m + j] = cfms(a[i * m + j], l, a[k * m + j]);
    }
  }
  if (neg) det = c2(-det.x, -det.y);
  for (int i = 0; i < m; ++i) x[i] = c2(0.0, 0.0);
  x[0] = det;
  for (int k = 0; k < m; ++k)
    if (piv[k] != k) {
      const double2 t = x[k];
      x[k] = x[piv[k]];
      x[piv[k]] = t;
    }
  for (int i = 1; i < m; ++i)
    for (int j = 0; j < i; ++j) x[i] = cfms(x[i], a[i * m + j], x[j]);
  for (int i = m - 1; i >= 0; --i) {
    for (int j = i + 1; j < m; ++j) x[i] = cfms(x[i], a[i * m + j], x[j]);
    x[i] = cmul(x[i], crcp(a[i * m + i]));
  }
}

// The 2n sums of one point (inputs in K.u, K.flag): thread t < 2n returns sum (i = t/2, k = t%2).
__device__ double2 kernel_point(KernelShared &K, const ItemDev &it, int N, int *bad) {
  const int tid = threadIdx.x;
  const kb_gf_index X = it.f.A;
  const int spin = X.spin;
  const int M1 = 2 * N + 1, M2 = 2 * N;
  for (int e = tid; e < M1 * M1 + M2 * M2; e += blockDim.x) {
    const bool first = e < M1 * M1;
    const int q = first ? e : e - M1 * M1, M = first ? M1 : M2;
    const int r = q / M, c = q - r * M;
    kb_gf_index a, b;
    const int sp = first ? spin : 1 - spin;
    if (first && r == 2 * N) {
      a = X;
      a.timesplit = N;
    } else {
      a.time = K.u[r % N];
      a.spin = sp;
      a.k_idx = r >= N ? 1 : 0;
      a.timesplit = r % N;
      a.orbital = 0;
    }
    if (first && c == 2 * N) {
      b = X;
      b.timesplit = N;
    } else {
      b.time = K.u[c % N];
      b.spin = sp;
      b.k_idx = c >= N ? 1 : 0;
      b.timesplit = c % N;
      b.orbital = 0;
    }
    const double2 g = g0_contour(it.model, a, b, (first && r == 2 * N && c == 2 * N) ? 0 : 1, bad);
    if (first)
      K.G1[q] = g;
    else
      K.G2[q] = g;
  }
  __syncthreads();
  const unsigned nconf = 1u << N;
  const int ti = tid >> 1, tk = tid & 1;
  double2 acc = c2(0.0, 0.0);
  for (unsigned base = 0; base < nconf; base += blockDim.x) {
    const unsigned cfg = base + tid;
    if (cfg < nconf) {
      double2 m1[(KM_MAX_ORDER + 1) * (KM_MAX_ORDER + 1)], m2[KM_MAX_ORDER * KM_MAX_ORDER];
      double2 x[KM_MAX_ORDER + 1];
      int pick[KM_MAX_ORDER + 1];
      pick[0] = 2 * N;
      for (int i = 0; i < N; ++i) pick[i + 1] = i + (int)((cfg >> i) & 1u) * N;
      for (int r = 0; r <= N; ++r)
        for (int c = 0; c <= N; ++c) m1[r * (N + 1) + c] = K.G1[pick[r] * M1 + pick[c]];
      m1[N * (N + 1) + N] = c2(0.0, 0.0);
      for (int r = 0; r < N; ++r)
        for (int c = 0; c < N; ++c) m2[r * N + c] = K.G2[pick[r + 1] * M2 + pick[c + 1]];
      first_row_cofactors(m1, N + 1, x);
      double2 d2 = lu_det(m2, N);
      if (__popc(cfg) & 1) d2 = c2(-d2.x, -d2.y);
      for (int i = 0; i < N; ++i) K.X[tid][i] = cmul(x[i + 1], d2);
    }
    __syncthreads();
    if (tid < 2 * N) {
      const unsigned cnt = min((unsigned)blockDim.x, nconf - base);
      for (unsigned c = 0; c < cnt; ++c)
        if ((int)(((base + c) >> ti) & 1u) == tk) acc = cadd(acc, K.X[c][ti]);
    }
    __syncthreads();
  }
  return acc;
}

// ------------------------------------------------------------ kernel method, tree form
// For spin-symmetric models det(s2_a) = det(V_a), V_a the vertex block of G picked by a,
// and keldy's s1_a = [[g_XX, r], [c, W_a]] with W_a = V_a except its last vertex's
// diagonal entry set to 0. The first-row cofactors of s1_a are x_0 = det(W_a) and
// x_{i+1} = -det(W_a) (W_a^-1 c)_i (block inverse), so only the vertex block and the X
// column enter. Gauss-Jordan elimination of the vertices in order 0..n-1, pivoting on the
// diagonal entry of the chosen copy and carrying the X column, visits the 2^n
// configurations as the leaves of a binary tree that shares its prefixes, as the direct
// integrand's tree does; a node after j eliminations holds the j eliminated rows (pivot
// rows normalised by their pivots), both copies' rows of the remaining vertices, and the
// columns of the remaining copies plus the X column. At a leaf (copy b of the last
// vertex), with D the product of the earlier pivots, p the last pivot and p_W = p minus
// that copy's original diagonal entry (the Schur complement is affine in it with
// coefficient 1), c_b the carried X entry of the last row and (e_j, f_j) an eliminated
// row's last-copy and X entries:
//   x_n = -D c_b,  x_{j+1} = -D (p_W f_j - e_j c_b),  det(V_a) = D p,
// with no division by p_W (W_a may be singular, as for n = 1). Cost O(2^n n) per point
// after the shared levels, instead of 2^n pivoted LU pairs. A point whose pivot falls
// below the guard (or a model whose spins differ) takes keldy's pivoted-LU path,
// kernel_point above, with the same per-(vertex, index) sums.

// Sized for two CTAs per SM: at most 64 points per pass, 64 nodes per level, 128 vertex
// times; the per-warp partial sums of the leaves' reduction live in the frontier buffer
// that the last level leaves free.
constexpr int KM_MAX_PASS = 64;
// Complex entries per frontier buffer of the kernel-method tree: its widest level (64 nodes
// of 10 x 5 at order 8, one point per pass) is larger than the direct tree's.
constexpr int KM_FRONTIER = 3200;

struct KMTreeShared {
  union {
    double2 buf[2][KM_FRONTIER];
    KernelShared K; // the pivoted-LU path of a guarded point (after the tree pass)
  };
  double2 D[2][KM_MAX_PASS];
  double2 inv[KM_MAX_PASS];
  double u[2 * KM_MAX_PASS];   // vertex times, u[j * np + p]
  double jac[KM_MAX_PASS];
  int flag[KM_MAX_PASS];       // bit 0: out of domain, bit 1: a guarded pivot
  double2 gd[KM_MAX_PASS][2];  // original diagonal entries of the last vertex's two copies, per point
  double2 S[256];              // per point the 2n sums, S[p * 2n + 2i + k]
  int bidx[256];               // per (point, vertex) the time bin (-1 dropped, -2 out of domain)
};

// Points per pass of the tree form: 2^(n-1) threads per point (one per configuration of
// the first n-1 vertices; two for n = 1) up to the CTA's 128; orders 9 and 10 walk their first 2 and 3
// levels one path at a time so that the widest level fits a frontier buffer.
__host__ __device__ inline int km_points_per_pass(int n) { return n == 1 ? 64 : n <= 8 ? (128 >> (n - 1)) : 1; }
__host__ __device__ inline int km_path_levels(int n) { return n <= 8 ? 0 : n - 7; }

// Orders with path levels run 2^K0 passes from the same G (one point per pass). It stays
// at the end of the frontier buffer that no level of a pass writes that far (level j
// writes buffer (j + 1) & 1 from its start; the leaves' reduction scratch takes the first
// 160 entries of the free buffer). Returns that buffer, or -1 (single pass, or no room).
__host__ __device__ inline int km_root_buffer(int N) {
  const int K0 = km_path_levels(N);
  if (K0 == 0) return -1;
  const int root = (2 * N + 1) * (2 * N + 1);
  int use[2] = {0, 0}, nodes = 1;
  for (int j = 0; j < N - 2; ++j) {
    if (j >= K0) nodes *= 2;
    const int sz = nodes * (2 * N - j - 1) * (2 * (N - j) - 1);
    if (use[(j + 1) & 1] < sz) use[(j + 1) & 1] = sz;
  }
  const int b = use[0] <= use[1] ? 0 : 1;
  return (use[b] + root <= KM_FRONTIER && root + 160 <= KM_FRONTIER) ? b : -1;
}

// One elimination level: vertex j of every node (rows 2n - j, columns 2(n - j) + 1,
// stride `cs` elements per node) into its children (rows 2n - j - 1, columns
// 2(n - j) - 1). bsel < 0: both children (child 2 par + b pivots on copy b); otherwise
// the single child on copy bsel. inv and Dn get the children's pivot reciprocals and
// prefix determinants. (Each item forming its own reciprocals instead, without the
// barrier after them, was 2-5 % slower at orders 6-8; levels fused in pairs as in the
// direct tree, with a pivot pre-pass and the children never stored, were 6-16 % slower at
// orders 5-8: the kept rows make each grandchild entry cost 2.5 complex FMAs there
// against 1.5 in two single levels.)
__device__ void km_level(const double2 *cur, int cs, double2 *nxt, const double2 *Dc, double2 *Dn, double2 *inv,
                         int *flag, int nodes, int lg_npp, int j, int n, int bsel, double floor_) {
  const int R = 2 * n - j, C = 2 * (n - j) + 1;
  const int R1 = R - 1, C1 = C - 2;
  const int nch = bsel < 0 ? 2 : 1;
  for (int c = threadIdx.x; c < nodes * nch; c += blockDim.x) {
    const int par = bsel < 0 ? c >> 1 : c, b = bsel < 0 ? (c & 1) : bsel;
    const double2 piv = cur[par * cs + (j + b) * C + b];
    if (!(cabs1(piv) >= floor_)) flag[par >> lg_npp] |= 2;
    inv[c] = crcp(piv);
    Dn[c] = cmul(Dc[par], piv);
  }
  __syncthreads();
  // rows split into column segments while the CTA has idle threads: of at least 4 columns,
  // down to single columns when a pass holds at most 4 points (orders 6 and up, whose top
  // levels have few rows: order 8 7 % faster, orders 9 / 10 6 / 5 %; orders 4-5 2 % slower)
  const int rows = nodes * R1;
  const int minc = (nodes >> lg_npp) <= 4 ? 1 : 4;
  int lgseg = 0;
  while ((rows << (lgseg + 1)) <= (int)blockDim.x && (C1 >> (lgseg + 1)) >= minc) ++lgseg;
  const int seglen = (C1 + (1 << lgseg) - 1) >> lgseg;
  const unsigned magic = 0xFFFFFFFFu / (unsigned)R1 + 1u; // r / R1 == umulhi(r, magic) for r < 2^20, R1 >= 3
  for (int t = threadIdx.x; t < (rows << lgseg); t += blockDim.x) {
    const int r = t >> lgseg;
    const int q0 = (t & ((1 << lgseg) - 1)) * seglen, q1 = min(C1, q0 + seglen);
    const int par = (int)__umulhi((unsigned)r, magic), ri = r - par * R1;
    const double2 *S = cur + par * cs;
    for (int k = 0; k < nch; ++k) {
      const int b = bsel < 0 ? k : bsel;
      const int ci = par * nch + k;
      const double2 *prow = S + (j + b) * C + 2;
      double2 *o = nxt + (size_t)ci * (R1 * C1) + ri * C1;
      const double2 iv = inv[ci];
      if (ri == j) {
        for (int q = q0; q < q1; ++q) o[q] = cmul(prow[q], iv);
      } else {
        const int old = ri < j ? ri : ri + 1;
        const double2 *srow = S + old * C;
        const double2 Lf = cmul(srow[b], iv);
#pragma unroll 4
        for (int q = q0; q < q1; ++q) o[q] = cfms(srow[q + 2], Lf, prow[q]);
      }
    }
  }
  __syncthreads();
}

// The leaves under a node after n-2 eliminations (rows: n-2 eliminated, then vertex
// n-2's two copies, then vertex n-1's; columns: the four copies, then X), on thread b
// (copy of vertex n-2): the last elimination in registers, then both leaves. Adds the
// terms into v[2i + k] (vertex i, Keldysh index k). path: the copies of vertices
// 0..n-3 (bit n-3-i for vertex i), parity their count.
template <int n>
__device__ __forceinline__ void km_leaves2(const double2 *S, double2 D, const double2 *gd, int b, unsigned path,
                                           int parity, double floor_, bool &guard, double2 (&v)[2 * n]) {
  const int C = 5;
  const double2 p1 = S[(n - 2 + b) * C + b];
  if (!(cabs1(p1) >= floor_)) guard = true;
  const double2 i1 = crcp(p1);
  const double2 D1 = cmul(D, p1);
  double2 prow[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) prow[q] = cmul(S[(n - 2 + b) * C + 2 + q], i1);
  // rows of vertex n-1's copies after the elimination: pivot, X entry, W pivot
  double2 p[2], cb[2], pw[2];
#pragma unroll
  for (int bp = 0; bp < 2; ++bp) {
    const double2 *r = S + (n + bp) * C;
    const double2 Lf = r[b]; // prow is normalised by the pivot already
    p[bp] = cfms(r[2 + bp], Lf, prow[bp]);
    cb[bp] = cfms(r[4], Lf, prow[2]);
    pw[bp] = c2(p[bp].x - gd[bp].x, p[bp].y - gd[bp].y);
    if (!(cabs1(p[bp]) >= floor_)) guard = true;
  }
  // coefficient of each leaf: -D1 * det(V) * sign = -D1^2 p (-1)^(parity + b + bp)
  double2 coef[2];
#pragma unroll
  for (int bp = 0; bp < 2; ++bp) {
    double2 t = cmul(cmul(D1, D1), p[bp]);
    if ((parity + b + bp) & 1) t = c2(-t.x, -t.y);
    coef[bp] = c2(-t.x, -t.y);
  }
  // vertex n-1: x_n = -D1 c_b (the D1 factor is in coef)
#pragma unroll
  for (int bp = 0; bp < 2; ++bp) {
    const double2 t = cmul(coef[bp], cb[bp]);
    v[2 * (n - 1) + bp] = cadd(v[2 * (n - 1) + bp], t);
  }
  // eliminated rows: vertices 0..n-3 (rows 0..n-3), then vertex n-2 (the pivot row)
#pragma unroll
  for (int i = 0; i <= n - 2; ++i) {
    double2 r0, r1, rx; // the child's row i at vertex n-1's copies and X
    if (i == n - 2) {
      r0 = prow[0];
      r1 = prow[1];
      rx = prow[2];
    } else {
      const double2 *r = S + i * C;
      const double2 Lf = r[b];
      r0 = cfms(r[2], Lf, prow[0]);
      r1 = cfms(r[3], Lf, prow[1]);
      rx = cfms(r[4], Lf, prow[2]);
    }
    const int k = (i == n - 2) ? b : (int)((path >> (n - 3 - i)) & 1u);
    double2 acc = c2(0.0, 0.0);
#pragma unroll
    for (int bp = 0; bp < 2; ++bp) {
      // x_{i+1} / D1 = p_W f - e c_b
      const double2 x = cfms(cmul(pw[bp], rx), bp ? r1 : r0, cb[bp]);
      acc = cadd(acc, cmul(coef[bp], x));
    }
    // to (i, k), written without a dynamic index so that v stays in registers
    v[2 * i] = cadd(v[2 * i], k ? c2(0.0, 0.0) : acc);
    v[2 * i + 1] = cadd(v[2 * i + 1], k ? acc : c2(0.0, 0.0));
  }
}

// Sums the 2n values v[] over aligned groups of G consecutive threads (G a power of two)
// into S[g * 2n + q] for group g < ngroups; fixed shuffle pattern (deterministic).
template <int n2>
__device__ void km_group_sum(double2 (&v)[n2], int G, int ngroups, double2 *S, double2 (*red)[2 * KM_MAX_ORDER]) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gw = G < 32 ? G : 32;
#pragma unroll
  for (int q = 0; q < n2; ++q)
    for (int off = 1; off < gw; off <<= 1) {
      v[q].x += __shfl_xor_sync(0xffffffffu, v[q].x, off);
      v[q].y += __shfl_xor_sync(0xffffffffu, v[q].y, off);
    }
  if (G <= 32) {
    const int g = tid / G;
    if ((lane & (G - 1)) == 0 && g < ngroups)
#pragma unroll
      for (int q = 0; q < n2; ++q) S[g * n2 + q] = cadd(S[g * n2 + q], v[q]);
    __syncthreads();
  } else {
    if (lane == 0)
#pragma unroll
      for (int q = 0; q < n2; ++q) red[warp][q] = v[q];
    __syncthreads();
    const int wpg = G / 32;
    for (int e = tid; e < ngroups * n2; e += blockDim.x) {
      const int g = e / n2, q = e - g * n2;
      double2 s = S[e];
      for (int w = g * wpg; w < (g + 1) * wpg; ++w) s = cadd(s, red[w][q]);
      S[e] = s;
    }
    __syncthreads();
  }
}

// Per-point sums S of np points whose inputs are in K.u, K.flag (tree form; flag bit 1
// marks points to redo on the pivoted-LU path).
template <int N>
__device__ void km_tree_points(KMTreeShared &K, const ItemDev &it, int np, int *bad) {
  const int tid = threadIdx.x;
  const int n2 = 2 * N;
  for (int e = tid; e < np * n2; e += blockDim.x) K.S[e] = c2(0.0, 0.0);
  __syncthreads();
  const double floor_ = it.model.pivot_floor;
  const int spin = it.f.A.spin;
  const int K0 = km_path_levels(N);
  const int M = 2 * N + 1;
  // G built once for all passes (one point per pass) when it fits at a buffer's end
  const int rb = km_root_buffer(N);
  double2 *root = rb >= 0 ? K.buf[rb] + (KM_FRONTIER - M * M) : K.buf[0];
  for (int sub = 0; sub < (1 << K0); ++sub) {
    if (rb < 0 || sub == 0) build_G_any<true>(it, N, np, K.u, K.flag, root, spin, bad);
    __syncthreads();
    for (int p = tid; p < np; p += blockDim.x) {
      K.D[0][p] = c2(1.0, 0.0);
      const double2 *G = root + (size_t)p * M * M;
      K.gd[p][0] = G[(2 * N - 2) * M + 2 * N - 2];
      K.gd[p][1] = G[(2 * N - 1) * M + 2 * N - 1];
    }
    __syncthreads();
    double2 v[2 * N];
#pragma unroll
    for (int q = 0; q < 2 * N; ++q) v[q] = c2(0.0, 0.0);
    if (N == 1) {
      // the leaves of the root itself: x_1 = -c_b, det(V) = p
      if (tid < 2 * np) {
        const int p = tid >> 1, b = tid & 1;
        const double2 *G = K.buf[0] + (size_t)p * M * M;
        const double2 piv = G[b * M + b], cb = G[b * M + 2];
        double2 t = cmul(piv, cb);
        if (!b) t = c2(-t.x, -t.y); // -(-1)^b p c_b
        v[0] = b ? c2(0.0, 0.0) : t;
        v[1] = b ? t : c2(0.0, 0.0);
      }
      km_group_sum<2 * N>(v, 2, np, K.S, reinterpret_cast<double2(*)[2 * KM_MAX_ORDER]>(K.buf[1]));
      continue;
    }
    int cur = 0, cs = M * M, nodes = np, lg = 0;
    for (int j = 0; j < N - 2; ++j) {
      const int bsel = j < K0 ? (int)((sub >> (K0 - 1 - j)) & 1u) : -1;
      km_level(j == 0 ? root : K.buf[cur], cs, K.buf[cur ^ 1], K.D[cur], K.D[cur ^ 1], K.inv, K.flag, nodes, lg, j,
               N, bsel, floor_);
      if (bsel < 0) {
        nodes *= 2;
        lg += 1;
      }
      cur ^= 1;
      cs = (2 * N - j - 1) * (2 * (N - j) - 1);
    }
    // nodes after N-2 eliminations: 2 threads each
    bool guard = false;
    int p = 0;
    if (tid < 2 * nodes) {
      const int node = tid >> 1, b = tid & 1;
      p = node >> lg;
      const unsigned pathbits = ((unsigned)sub << lg) | (unsigned)(node & ((1 << lg) - 1));
      if constexpr (N >= 2)
        km_leaves2<N>(K.buf[cur] + (size_t)node * cs, K.D[cur][node], K.gd[p], b, pathbits, __popc(pathbits), floor_,
                      guard, v);
    }
    if (guard) K.flag[p] |= 2;
    km_group_sum<2 * N>(v, 2 << lg, np, K.S, reinterpret_cast<double2(*)[2 * KM_MAX_ORDER]>(K.buf[cur ^ 1]));
  }
}

__device__ void km_tree_points_any(KMTreeShared &K, const ItemDev &it, int N, int np, int *bad) {
  switch (N) {
  case 1: km_tree_points<1>(K, it, np, bad); break;
  case 2: km_tree_points<2>(K, it, np, bad); break;
  case 3: km_tree_points<3>(K, it, np, bad); break;
  case 4: km_tree_points<4>(K, it, np, bad); break;
  case 5: km_tree_points<5>(K, it, np, bad); break;
  case 6: km_tree_points<6>(K, it, np, bad); break;
  case 7: km_tree_points<7>(K, it, np, bad); break;
  case 8: km_tree_points<8>(K, it, np, bad); break;
  case 9: km_tree_points<9>(K, it, np, bad); break;
  default: km_tree_points<10>(K, it, np, bad); break;
  }
}

// A pass's point values (one per thread, f, in the domain or not, with its dropped bin
// terms) into the chunk's sums: each warp's by a fixed xor-shuffle pattern, then thread 0
// adds the warps in order (deterministic). Every thread calls it; the caller's barrier
// follows before the next pass.
__device__ __noinline__ void km_pass_sum(double2 f, bool dom, unsigned long long drop, double2 &csum,
                                         unsigned long long &cdom, unsigned *dropped) {
  __shared__ double2 wsum[KM_THREADS / 32];
  __shared__ unsigned wdom[KM_THREADS / 32];
  __shared__ unsigned long long wdrop[KM_THREADS / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int off = 16; off > 0; off >>= 1) {
    f.x += __shfl_xor_sync(0xffffffffu, f.x, off);
    f.y += __shfl_xor_sync(0xffffffffu, f.y, off);
    drop += __shfl_xor_sync(0xffffffffu, drop, off);
  }
  const unsigned bdom = __ballot_sync(0xffffffffu, dom);
  if (lane == 0) {
    wsum[w] = f;
    wdom[w] = bdom;
    wdrop[w] = drop;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long d = 0;
    for (int k = 0; k < KM_THREADS / 32; ++k) {
      csum = cadd(csum, wsum[k]);
      cdom += __popc(wdom[k]);
      d += wdrop[k];
    }
    if (dropped) *dropped += (unsigned)d;
  }
}

// integrand_g_kernel_single_omega (wick_kernel_single_omega.cpp:126-135): point p's terms
// weighted by e^{i omega t} of their vertex, in vertex order, times its Jacobian.
__device__ __forceinline__ double2 km_fourier_value(const KMTreeShared &K, const Launch &L, int p, int np, int N) {
  const int n2 = 2 * N;
  double2 f = c2(0.0, 0.0);
  for (int i = 0; i < N; ++i) {
    double sn, cs;
    sincos(L.km_omega * K.u[i * np + p], &sn, &cs);
    const double2 sv = cadd(K.S[p * n2 + 2 * i], K.S[p * n2 + 2 * i + 1]);
    f = cadd(f, cmul(sv, c2(cs, sn)));
  }
  const double j = K.jac[p];
  return c2(f.x * j, f.y * j);
}

__global__ void __launch_bounds__(KM_THREADS, KM_CTAS_PER_SM) km_tree_kernel(Launch L) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  KMTreeShared &K = *reinterpret_cast<KMTreeShared *>(smem_raw);
  __shared__ int s_chunk;
  __shared__ int s_bad;
  const int tid = threadIdx.x;
  if (tid == 0) s_bad = 0;
  const bool eval = L.mode != IN_SOBOL;
  const int nb = L.nbins * L.bin_cols;
  for (;;) {
    if (tid == 0) s_chunk = atomicAdd(L.chunk_counter, 1);
    __syncthreads();
    const int c = s_chunk;
    if (c >= L.n_chunks) break;
    const int item = find_item(L.chunk_offsets, L.n_items, c);
    const ItemDev &it = L.items[item];
    const long long cfirst = (long long)(c - L.chunk_offsets[item]) * it.chunk_points;
    const int ccount = (int)min((long long)it.chunk_points, it.n_points - cfirst);
    const int N = it.order;
    const int n2 = 2 * N;
    const bool keep = L.mode == IN_SOBOL ? true : (L.keep_u_hypercube != 0);
    if (!eval && nb) {
      for (int b = tid; b < nb; b += blockDim.x) {
        L.bin_sums[(size_t)c * nb + b] = c2(0.0, 0.0);
        L.bin_counts[(size_t)c * nb + b] = 0u;
      }
      if (tid == 0) L.bin_dropped[c] = 0u;
    }
    double2 csum = c2(0.0, 0.0);
    unsigned long long cdom = 0;
    const int P = it.spin_symmetric ? km_points_per_pass(N) : 1;
    // passes of at most 8 points (orders 5 and up): the chunk's points are set up at once
    // (Sobol coordinates or given inputs, warper chain, domain flag: one thread per point)
    // into the CTA's slot and each pass reads its own, instead of a pass's few threads
    // walking the chain for its points while the others wait
    const bool staged = P <= 8;
    double *slot = L.pts + (size_t)blockIdx.x * KM_SLOT;
    if (staged) {
      if (tid < ccount) prepare_point(L, it, N, cfirst + tid, keep, slot, tid);
      __syncthreads();
    }
    for (int sb = 0; sb < ccount; sb += P) {
      const int np = min(P, ccount - sb);
      if (!staged) {
        load_points(L, it, N, np, cfirst + sb, K.u, K.jac, K.flag, keep);
      } else if (tid < np) {
        for (int j = 0; j < N; ++j) K.u[j * np + tid] = slot[j * CHUNK_POINTS + sb + tid];
        K.jac[tid] = slot[MAX_ORDER * CHUNK_POINTS + sb + tid];
        K.flag[tid] = (int)slot[(MAX_ORDER + 1) * CHUNK_POINTS + sb + tid];
      }
      __syncthreads();
      if (it.spin_symmetric) {
        km_tree_points_any(K, it, N, np, &s_bad);
      } else {
        for (int e = tid; e < np * n2; e += blockDim.x) K.S[e] = c2(0.0, 0.0);
        if (tid < np) K.flag[tid] |= (K.flag[tid] & 1) ? 0 : 2;
        __syncthreads();
      }
      // guarded points (and the spin-asymmetric ones): keldy's pivoted-LU path, one by one
      bool g = false; // any guarded point (every warp finds the same answer, no barrier)
      for (int p = tid & 31; p < np; p += 32) g = g || (K.flag[p] & 3) == 2;
      const bool any_guarded = __any_sync(0xffffffffu, g);
      for (int p = 0; any_guarded && p < np; ++p) {
        if ((K.flag[p] & 3) != 2) continue;
        double ut[KM_MAX_ORDER];
        for (int j = 0; j < N; ++j) ut[j] = K.u[j * np + p];
        __syncthreads();
        if (tid < N) K.K.u[tid] = ut[tid];
        if (tid == 0) K.K.flag[0] = 0;
        __syncthreads();
        const double2 s = kernel_point(K.K, it, N, &s_bad);
        if (tid < n2) K.S[p * n2 + tid] = s;
        __syncthreads();
      }
      if (eval) {
        for (int e = tid; e < np * n2; e += blockDim.x) {
          const int p = e / n2, q = e - p * n2;
          const long long gp = cfirst + sb + p;
          const bool dom = !(K.flag[p] & 1);
          const double j = K.jac[p];
          L.out_kvals[gp * n2 + q] = dom ? c2(K.S[e].x * j, K.S[e].y * j) : c2(0.0, 0.0);
          if (q == 0) {
            if (L.out_jac) L.out_jac[gp] = j;
            if (L.out_dom) L.out_dom[gp] = dom ? 1 : 0;
          }
        }
      } else if (L.km_fourier) {
        // integrand_g_kernel_single_omega (wick_kernel_single_omega.cpp:126-135): the
        // point's terms weighted by e^{i omega t} of their vertex, in point and vertex order
        // passes of more than two points: one thread per point, then km_pass_sum; one or
        // two points: thread 0 in point order (no extra barrier)
        if (P > 2) {
          const bool dom = tid < np && !(K.flag[tid] & 1);
          const double2 f = dom ? km_fourier_value(K, L, tid, np, N) : c2(0.0, 0.0);
          km_pass_sum(f, dom, 0ull, csum, cdom, nullptr);
        } else if (tid == 0) {
          for (int p = 0; p < np; ++p) {
            if (K.flag[p] & 1) continue;
            cdom++;
            csum = cadd(csum, km_fourier_value(K, L, p, np, N));
          }
        }
      } else {
        // bin of every (point, vertex); then one thread per (bin, index) adds the pass's
        // terms in point and vertex order, as one thread walking them would
        for (int e = tid; e < np * N; e += blockDim.x) {
          const int p = e / N, i = e - p * N;
          K.bidx[e] = (K.flag[p] & 1) ? -2 : time_bin(L, K.u + i * np + p, 1, 1);
        }
        __syncthreads();
        const unsigned half = 1u << (N - 1);
        for (int bk = tid; bk < nb; bk += blockDim.x) {
          const int bin = bk >> 1, k = bk & 1;
          double2 bs = L.bin_sums[(size_t)c * nb + bk];
          unsigned cnt = 0;
          bool any = false;
          for (int p = 0; p < np; ++p) {
            const double j = K.jac[p];
            for (int i = 0; i < N; ++i)
              if (K.bidx[p * N + i] == bin) {
                const double2 sv = K.S[p * n2 + 2 * i + k];
                bs = c2(bs.x + sv.x * j, bs.y + sv.y * j);
                cnt += half;
                any = true;
              }
          }
          if (any) {
            L.bin_sums[(size_t)c * nb + bk] = bs;
            L.bin_counts[(size_t)c * nb + bk] += cnt;
          }
        }
        if (P > 2) { // as above: one thread per point, then km_pass_sum
          double2 f = c2(0.0, 0.0);
          unsigned long long drop = 0;
          const bool dom = tid < np && !(K.flag[tid] & 1);
          if (dom) {
            const double j = K.jac[tid];
            for (int i = 0; i < N; ++i) {
              if (K.bidx[tid * N + i] < 0) drop += 2 * half;
              for (int k = 0; k < 2; ++k) {
                const double2 sv = K.S[tid * n2 + 2 * i + k];
                f = c2(f.x + sv.x * j, f.y + sv.y * j);
              }
            }
          }
          km_pass_sum(f, dom, drop, csum, cdom, L.bin_dropped + c);
        } else if (tid == 0) {
          for (int p = 0; p < np; ++p) {
            if (K.flag[p] & 1) continue;
            cdom++;
            const double j = K.jac[p];
            for (int i = 0; i < N; ++i) {
              if (K.bidx[p * N + i] < 0) L.bin_dropped[c] += 2 * half;
              for (int k = 0; k < 2; ++k) {
                const double2 sv = K.S[p * n2 + 2 * i + k];
                csum = c2(csum.x + sv.x * j, csum.y + sv.y * j);
              }
            }
          }
        }
      }
      __syncthreads();
    }
    if (!eval && tid == 0) {
      ChunkPartial pr;
      pr.sum_re = csum.x;
      pr.sum_im = csum.y;
      pr.n_in_domain = cdom;
      pr.n_fallback = 0;
      pr.fb_mask[0] = pr.fb_mask[1] = 0;
      L.partials[c] = pr;
    }
  }
  if (tid == 0 && s_bad) atomicOr(L.err, 1);
}

// Thread t of block `item` sums bins t, t + NT, ... over the item's chunks in chunk order.
__global__ void __launch_bounds__(NT) reduce_bins_kernel(Launch L, double2 *sums, unsigned long long *counts,
                                                         unsigned long long *dropped) {
  const int item = blockIdx.x;
  const long long c0 = L.chunk_offsets[item], c1 = L.chunk_offsets[item + 1];
  const int nb = L.nbins * max(1, L.bin_cols);
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    double2 s = c2(0.0, 0.0);
    unsigned long long n = 0;
    for (long long c = c0; c < c1; ++c) {
      s = cadd(s, L.bin_sums[(size_t)c * nb + b]);
      n += L.bin_counts[(size_t)c * nb + b];
    }
    sums[(size_t)item * nb + b] = s;
    counts[(size_t)item * nb + b] = n;
  }
  if (threadIdx.x == 0) {
    unsigned long long d = 0;
    for (long long c = c0; c < c1; ++c) d += L.bin_dropped[c];
    dropped[item] = d;
  }
}

} // namespace

// The launchers rely on configure_kernels() having set the kernels' shared-memory limits
// on the launching device: kb_context_create calls it, with the context's device current,
// for every context (the attribute belongs to each device's context, not to the process).
cudaError_t launch_kernel_method(const Launch &L, int grid, cudaStream_t st) {
  km_tree_kernel<<<grid, KM_THREADS, (int)sizeof(KMTreeShared), st>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_reduce_bins(const Launch &L, double2 *sums, unsigned long long *counts,
                               unsigned long long *dropped, cudaStream_t st) {
  if (L.n_items == 0 || L.nbins == 0) return cudaSuccess;
  reduce_bins_kernel<<<L.n_items, NT, 0, st>>>(L, sums, counts, dropped);
  return cudaGetLastError();
}

size_t tree_smem_bytes() { return sizeof(TreeShared); }

// Shared-memory limit of the four tree-kernel instantiations.
static cudaError_t configure_tree(int smem) {
  cudaError_t e = cudaFuncSetAttribute(tree_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(tree_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(tree_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(tree_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  return e;
}

cudaError_t configure_kernels() {
  cudaError_t e = configure_tree((int)sizeof(TreeShared));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(direct_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DirectShared));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fallback_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DirectShared));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(km_tree_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(KMTreeShared));
  return e;
}

static size_t direct_smem_bytes() { return sizeof(DirectShared); }

cudaError_t launch_tree(const Launch &L, int grid, cudaStream_t st) {
  const size_t smem = tree_smem_bytes();
  if (L.mode == IN_SOBOL) {
    if (L.any_cubic)
      tree_kernel<false, true><<<grid, TREE_THREADS, smem, st>>>(L);
    else
      tree_kernel<false, false><<<grid, TREE_THREADS, smem, st>>>(L);
  } else {
    if (L.any_cubic)
      tree_kernel<true, true><<<grid, TREE_THREADS, smem, st>>>(L);
    else
      tree_kernel<true, false><<<grid, TREE_THREADS, smem, st>>>(L);
  }
  return cudaGetLastError();
}

cudaError_t launch_direct(const Launch &L, int grid, cudaStream_t st) {
  direct_kernel<<<grid, NT, direct_smem_bytes(), st>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_fallback(const Launch &L, int grid, cudaStream_t st) {
  fallback_kernel<<<grid, NT, direct_smem_bytes(), st>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_reduce(const Launch &L, kb_accum *acc_dev, cudaStream_t st) {
  if (L.n_items == 0) return cudaSuccess;
  reduce_kernel<<<L.n_items, NT, 0, st>>>(L, acc_dev);
  return cudaGetLastError();
}

} // namespace kb
