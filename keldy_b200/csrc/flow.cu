// Learned coupling-flow warper kernels (sm_100a): sampling / density maps and the
// fused training step, with every MLP product on the 5th-generation tensor cores.
//
// One CTA = 128 threads = one tile of 128 points; thread t owns point t of the tile and
// TMEM lane t. Each 128x128x128 product is 8 tcgen05.mma (kind::f16, bf16 operands,
// fp32 accumulator in TMEM) issued by thread 0 from shared-memory descriptors and
// completed through tcgen05.commit on an mbarrier. Activations and weights live in
// shared memory in one image layout (kb_flow.h: flow_img_index) that serves as a
// K-major operand in the forward products and, unchanged, as the MN-major operand of the
// backward products (dX = dY W, dW = dY^T X), so nothing is transposed. Weight images
// (32 KB each) stream from global memory with cp.async.bulk into three slots; the slot
// of W_j is refilled with the next layer's W_j as soon as the product reading it ends.
//
// Waits on mbarriers are bounded (about two seconds of SM clock); a CTA whose wait runs
// out sets bit 1 of the error word, skips the rest of its work, frees its TMEM and exits.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "kb_device.cuh"
#include "kb_flow.h"

namespace kb {

namespace {

constexpr int NT = FLOW_TILE;
constexpr uint32_t MAT_BYTES = FLOW_MAT * 2;
constexpr long long WAIT_CYCLES = 4000000000LL;
constexpr int FLOW_ERR_TIMEOUT = 2;

// ------------------------------------------------------------ PTX primitives
__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}\n"
               : "=r"(ok)
               : "r"(bar), "r"(parity)
               : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_test(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_test(bar, parity))
    if (clock64() - t0 > WAIT_CYCLES) return false;
  return true;
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Untiled bulk copy global -> shared (no multicast), completion counted on `bar`.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Shared-memory matrix descriptor, no swizzle (start, leading and stride byte offsets
// in 16-byte units; version 1 at bits 46-47).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: fp32 accumulator, bf16 A and B, M = N = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t a_mn, uint32_t b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn << 15) | (b_mn << 16) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void umma_issue(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
               "l"(a), "l"(b), "r"(idesc), "r"(acc)
               : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
               "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                 "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                 "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                 "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&h);
}
__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

template <typename T> __device__ __forceinline__ T get_dim(const T (&x)[FLOW_MAX_DIM], int d) {
  T r = x[0];
#pragma unroll
  for (int i = 1; i < FLOW_MAX_DIM; ++i) r = (d == i) ? x[i] : r;
  return r;
}
template <typename T> __device__ __forceinline__ void set_dim(T (&x)[FLOW_MAX_DIM], int d, T v) {
#pragma unroll
  for (int i = 0; i < FLOW_MAX_DIM; ++i)
    if (d == i) x[i] = v;
}

// ------------------------------------------------------------ CTA pipeline state
struct Pipe {
  uint32_t sW, sA;     // shared addresses of the weight slots and activation buffers
  uint32_t mbar;       // MMA completion
  uint32_t wbar[3];    // weight slot fills
  uint32_t tmem;       // TMEM base
  uint32_t mphase;     // parity of the next MMA completion (all threads)
  uint32_t wphase[3];  // parity of the next fill of each slot (thread 0)
  int pending[3];      // fill issued and not yet waited (thread 0)
  const uint16_t *img; // global weight images
};

__device__ __forceinline__ uint32_t act_addr(const Pipe &P, int i) { return P.sA + (uint32_t)i * MAT_BYTES; }
__device__ __forceinline__ uint32_t w_addr(const Pipe &P, int j) { return P.sW + (uint32_t)j * MAT_BYTES; }

// Thread 0: refill slot j with weight matrix `mat`.
__device__ __forceinline__ void load_weight(Pipe &P, int j, int mat) {
  mbar_expect_tx(P.wbar[j], MAT_BYTES);
  bulk_g2s(w_addr(P, j), P.img + (size_t)mat * FLOW_MAT, MAT_BYTES, P.wbar[j]);
  P.pending[j] = 1;
}

struct Mma {
  uint32_t d, a, b;
  uint32_t a_mn, b_mn;
  uint32_t acc;
};

// Thread 0: one 128x128x128 product, D (+)= A B^T, as 8 MMAs of K = 16.
__device__ __forceinline__ void issue_mma(const Mma &m) {
  const uint32_t id = idesc_bf16(m.a_mn, m.b_mn);
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const uint64_t ad = m.a_mn ? sdesc(m.a + s * 4096, 2048, 128) : sdesc(m.a + s * 256, 128, 2048);
    const uint64_t bd = m.b_mn ? sdesc(m.b + s * 4096, 2048, 128) : sdesc(m.b + s * 256, 128, 2048);
    umma_issue(m.d, ad, bd, id, (m.acc || s > 0) ? 1u : 0u);
  }
}

// All threads: publish this thread's shared-memory writes to the tensor core, run n
// products (thread 0; weight slot `wslot` waited first if a fill is pending) and wait
// for them. Returns false (uniformly) when a wait ran out.
__device__ bool mma_step(Pipe &P, int wslot, const Mma &m0, const Mma &m1, int n) {
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  int bad = 0;
  if (threadIdx.x == 0) {
    tc_fence_after();
    if (wslot >= 0 && P.pending[wslot]) {
      if (!mbar_wait(P.wbar[wslot], P.wphase[wslot])) bad = 1;
      P.wphase[wslot] ^= 1;
      P.pending[wslot] = 0;
    }
    if (!bad) {
      issue_mma(m0);
      if (n > 1) issue_mma(m1);
      umma_commit(P.mbar);
    }
  }
  if (__syncthreads_or(bad)) return false;
  const int tmo = mbar_wait(P.mbar, P.mphase) ? 0 : 1;
  P.mphase ^= 1;
  tc_fence_after();
  return !__syncthreads_or(tmo);
}

__device__ __forceinline__ unsigned char *row_ptr(unsigned char *buf, int t) {
  return buf + (t >> 3) * 2048 + (t & 7) * 16;
}

// Hat features of the conditioning dims of x into row t of buffer `buf`; feature
// 16*T_l[0] is the constant 1.
__device__ void encode_row(const FlowDev &f, int l, const float (&x)[FLOW_MAX_DIM], unsigned char *buf, int t) {
  unsigned char *row = row_ptr(buf, t);
  const unsigned tm = f.tmask[l];
  const int t0 = f.tdim[l][0];
#pragma unroll
  for (int i = 0; i < FLOW_MAX_DIM; ++i) {
    const bool cond = i < f.dim && !((tm >> i) & 1u);
    float u = x[i] * (float)FLOW_BLOB - 0.5f;
    const float fl = floorf(u);
    const int j0 = cond ? (int)fl : -100;
    const float fr = u - fl;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      uint32_t w[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int ja = 8 * h + 2 * e, jb = ja + 1;
        float a = (ja == j0) ? 1.0f - fr : ((ja == j0 + 1) ? fr : 0.0f);
        const float b = (jb == j0) ? 1.0f - fr : ((jb == j0 + 1) ? fr : 0.0f);
        if (ja == 0 && i == t0) a = 1.0f;
        w[e] = pack_bf16(a, b);
      }
      *reinterpret_cast<uint4 *>(row + (2 * i + h) * 128) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// Accumulator row -> ReLU -> bf16 row t of `buf`, hidden unit 127 set to 1.
__device__ void epi_relu(uint32_t trow, unsigned char *buf, int t) {
  unsigned char *row = row_ptr(buf, t);
#pragma unroll
  for (int c4 = 0; c4 < 4; ++c4) {
    float v[32];
    tmem_ld32(trow + 32 * c4, v);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t w[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float a = fmaxf(v[8 * q + 2 * e], 0.0f);
        float b = fmaxf(v[8 * q + 2 * e + 1], 0.0f);
        if (c4 == 3 && q == 3 && e == 3) b = 1.0f;
        w[e] = pack_bf16(a, b);
      }
      *reinterpret_cast<uint4 *>(row + (4 * c4 + q) * 128) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// The three conditioner products of layer l on the features already in act[0]:
// h1 -> act[1], h2 -> act[h2buf], logits left in the accumulator. Weight slots are
// refilled with matrix j of layer `next` (-1: none) after product j.
__device__ bool conditioner(Pipe &P, unsigned char *act, int h2buf, int next, uint32_t trow) {
  const int t = threadIdx.x;
  Mma none = {};
  Mma m = {P.tmem, act_addr(P, 0), w_addr(P, 0), 0, 0, 0};
  if (!mma_step(P, 0, m, none, 1)) return false;
  if (t == 0 && next >= 0) load_weight(P, 0, 3 * next + 0);
  epi_relu(trow, act + MAT_BYTES, t);
  m.a = act_addr(P, 1);
  m.b = w_addr(P, 1);
  if (!mma_step(P, 1, m, none, 1)) return false;
  if (t == 0 && next >= 0) load_weight(P, 1, 3 * next + 1);
  epi_relu(trow, act + (size_t)h2buf * MAT_BYTES, t);
  m.a = act_addr(P, h2buf);
  m.b = w_addr(P, 2);
  if (!mma_step(P, 2, m, none, 1)) return false;
  if (t == 0 && next >= 0) load_weight(P, 2, 3 * next + 2);
  return true;
}

struct SmemHead {
  unsigned long long bars[4];
  uint32_t tmem_slot;
  int pad;
  float red[NT / 32];
};

__device__ unsigned char *aligned_smem(unsigned char *raw) {
  return (unsigned char *)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
}

__device__ void pipe_init(Pipe &P, unsigned char *base, int n_act, SmemHead *&head, const uint16_t *img,
                          uint32_t ncols) {
  head = reinterpret_cast<SmemHead *>(base + (3 + n_act) * MAT_BYTES);
  P.sW = su32(base);
  P.sA = P.sW + 3 * MAT_BYTES;
  P.mbar = su32(&head->bars[0]);
  for (int j = 0; j < 3; ++j) {
    P.wbar[j] = su32(&head->bars[1 + j]);
    P.wphase[j] = 0;
    P.pending[j] = 0;
  }
  P.mphase = 0;
  P.img = img;
  if (threadIdx.x == 0) {
    mbar_init(P.mbar, 1);
    for (int j = 0; j < 3; ++j) mbar_init(P.wbar[j], 1);
    mbar_init_fence();
  }
  if (threadIdx.x < 32) tmem_alloc(su32(&head->tmem_slot), ncols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  P.tmem = head->tmem_slot;
}

// Waits for fills still in flight, then frees the TMEM columns.
__device__ void pipe_finish(Pipe &P, uint32_t ncols, int *err) {
  if (threadIdx.x == 0) {
    for (int j = 0; j < 3; ++j)
      if (P.pending[j]) {
        if (!mbar_wait(P.wbar[j], P.wphase[j])) atomicOr(err, FLOW_ERR_TIMEOUT);
        P.pending[j] = 0;
      }
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    tc_fence_after();
    tmem_dealloc(P.tmem, ncols);
  }
}

// ------------------------------------------------------------ sampling / density map
// Two CTAs per SM, each with one activation buffer and two weight slots: while one CTA runs
// its epilogues (ReLU, the CDF of the logits) on the CUDA cores, the other's products run on
// the tensor core. The CTA's products are numbered q = 0, 1, ... over its tiles (18 per
// tile: three per layer); product q reads weight slot q & 1, which is refilled with the
// matrix of product q + 2 as soon as product q completes. Each epilogue writes its output
// over the activation buffer the product just read (the product has completed).
template <int DIR>
__global__ void __launch_bounds__(NT, 2)
    flow_map_kernel(FlowDev f, long long count, const double *in, SobolDev rng, uint32_t k_first,
                    const uint32_t *k_first_dev, int use_sobol, double *out, double *out2, int *err) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char *base = aligned_smem(smem_raw);
  unsigned char *act = base + 2 * MAT_BYTES;
  SmemHead *head = reinterpret_cast<SmemHead *>(base + 3 * MAT_BYTES);
  Pipe P;
  P.sW = su32(base);
  P.sA = P.sW + 2 * MAT_BYTES;
  P.mbar = su32(&head->bars[0]);
  for (int j = 0; j < 3; ++j) {
    P.wbar[j] = su32(&head->bars[1 + j]);
    P.wphase[j] = 0;
    P.pending[j] = 0;
  }
  P.mphase = 0;
  P.img = f.img;
  if (threadIdx.x == 0) {
    mbar_init(P.mbar, 1);
    for (int j = 0; j < 2; ++j) mbar_init(P.wbar[j], 1);
    mbar_init_fence();
  }
  if (threadIdx.x < 32) tmem_alloc(su32(&head->tmem_slot), 128);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  P.tmem = head->tmem_slot;
  const int t = threadIdx.x, warp = t >> 5;
  const uint32_t trow = P.tmem + ((uint32_t)(warp * 32) << 16);
  const long long ntiles = (count + NT - 1) / NT;
  const long long my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const long long nq = my_tiles * 3 * FLOW_LAYERS;
  const int N = f.dim;
  if (k_first_dev) k_first = *k_first_dev;
  auto layer_at = [](int i) { return DIR == 0 ? i : FLOW_LAYERS - 1 - i; };
  // weight matrix read by product q
  auto mat_of = [&](long long q) { return 3 * layer_at((int)((q / 3) % FLOW_LAYERS)) + (int)(q % 3); };
  if (t == 0)
    for (int j = 0; j < 2 && j < nq; ++j) load_weight(P, j, mat_of(j));
  long long q = 0;
  bool ok = true;
  Mma none = {};
  for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const long long p = tile * NT + t;
    const bool valid = p < count;
    double x[FLOW_MAX_DIM];
#pragma unroll
    for (int d = 0; d < FLOW_MAX_DIM; ++d) {
      double v = 0.5;
      if (valid && d < N) v = use_sobol ? sobol_coord(rng, k_first + (uint32_t)p, d) : in[p * N + d];
      x[d] = v;
    }
    double acc = DIR == 0 ? 0.0 : 1.0;
    for (int li = 0; li < FLOW_LAYERS && ok; ++li) {
      const int l = layer_at(li);
      float xf[FLOW_MAX_DIM];
#pragma unroll
      for (int d = 0; d < FLOW_MAX_DIM; ++d) xf[d] = (float)x[d];
      encode_row(f, l, xf, act, t);
      // the layer's three products: features -> h1 -> h2 -> logits, all in one buffer
      for (int j = 0; j < 3 && ok; ++j, ++q) {
        const int slot = (int)(q & 1);
        Mma m = {P.tmem, act_addr(P, 0), w_addr(P, slot), 0, 0, 0};
        ok = mma_step(P, slot, m, none, 1);
        if (!ok) break;
        if (t == 0 && q + 2 < nq) load_weight(P, slot, mat_of(q + 2));
        if (j < 2) epi_relu(trow, act, t);
      }
      if (!ok) break;
#pragma unroll
      for (int s = 0; s < FLOW_SLOTS; ++s) {
        if (s >= f.ntr[l]) break;
        const int d = f.tdim[l][s];
        float v[32];
        tmem_ld32(trow + 32 * s, v);
        float mx = v[0];
#pragma unroll
        for (int j = 1; j < 32; ++j) mx = fmaxf(mx, v[j]);
        float e[32];
        double S = 0.0;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          e[j] = __expf(v[j] - mx);
          S += (double)e[j];
        }
        const double inv = (1.0 - (double)FLOW_EPS) / S, floor_p = (double)FLOW_EPS / FLOW_BINS;
        const double xd = get_dim(x, d);
        double cb = 0.0, pb = 1.0, cum = 0.0;
        int b = 0;
        if (DIR == 1) {
          bool found = false;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const double pj = (double)e[j] * inv + floor_p;
            const bool take = !found && (xd < cum + pj || j == 31);
            if (take) {
              b = j;
              cb = cum;
              pb = pj;
              found = true;
            }
            cum += pj;
          }
          double xn = ((double)b + (xd - cb) / pb) * (1.0 / FLOW_BINS);
          xn = fmin(fmax(xn, 0.0), 1.0);
          set_dim(x, d, xn);
          acc /= (double)FLOW_BINS * pb;
        } else {
          const double u = xd * FLOW_BINS;
          b = min(max((int)floor(u), 0), FLOW_BINS - 1);
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const double pj = (double)e[j] * inv + floor_p;
            if (j < b) cb += pj;
            if (j == b) pb = pj;
          }
          set_dim(x, d, cb + (u - (double)b) * pb);
          acc += log((double)FLOW_BINS * pb);
        }
      }
    }
    if (ok && valid) {
      for (int d = 0; d < N; ++d) out[p * N + d] = x[d];
      out2[p] = acc;
    }
  }
  if (!ok && t == 0) atomicOr(err, FLOW_ERR_TIMEOUT);
  pipe_finish(P, 128, err);
}

// ------------------------------------------------------------ training step
// TMEM columns: [0,128) working accumulator, [128,256) dW1, [256,384) dW2, [384,512) dW3.
__global__ void __launch_bounds__(NT, 1)
    flow_train_kernel(FlowDev f, long long count, const float *xin, const float *win, const int *index,
                      float inv_batch, float *partials, float *loss_part, float *xs, int *err) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char *base = aligned_smem(smem_raw);
  unsigned char *act = base + 3 * MAT_BYTES;
  SmemHead *head;
  Pipe P;
  pipe_init(P, base, 3, head, f.img, 512);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const uint32_t trow = P.tmem + ((uint32_t)(warp * 32) << 16);
  const long long ntiles = (count + NT - 1) / NT;
  const int N = f.dim;
  if (t == 0 && blockIdx.x < ntiles)
    for (int j = 0; j < 3; ++j) load_weight(P, j, j);
  bool ok = true;
  bool first = true;
  for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, first = false) {
    const long long p = tile * NT + t;
    const bool valid = p < count;
    const long long src = valid ? (long long)index[p] : 0;
    float x[FLOW_MAX_DIM];
#pragma unroll
    for (int d = 0; d < FLOW_MAX_DIM; ++d) x[d] = (valid && d < N) ? xin[src * N + d] : 0.5f;
    const float w = valid ? win[src] : 0.0f;
    const float glq = -w * inv_batch;
    float lq = 0.0f;
    // forward, saving each layer's input
    for (int l = 0; l < FLOW_LAYERS && ok; ++l) {
      if (valid)
#pragma unroll
        for (int d = 0; d < FLOW_MAX_DIM; ++d) xs[((size_t)l * FLOW_MAX_DIM + d) * count + p] = x[d];
      encode_row(f, l, x, act, t);
      ok = conditioner(P, act, 2, l + 1 < FLOW_LAYERS ? l + 1 : -1, trow);
      if (!ok) break;
#pragma unroll
      for (int s = 0; s < FLOW_SLOTS; ++s) {
        if (s >= f.ntr[l]) break;
        const int d = f.tdim[l][s];
        float v[32];
        tmem_ld32(trow + 32 * s, v);
        float mx = v[0];
#pragma unroll
        for (int j = 1; j < 32; ++j) mx = fmaxf(mx, v[j]);
        float S = 0.0f;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          v[j] = __expf(v[j] - mx);
          S += v[j];
        }
        const float inv = (1.0f - FLOW_EPS) / S, floor_p = FLOW_EPS / FLOW_BINS;
        const float u = get_dim(x, d) * FLOW_BINS;
        const int b = min(max((int)floorf(u), 0), FLOW_BINS - 1);
        float cb = 0.0f, pb = 1.0f;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const float pj = v[j] * inv + floor_p;
          if (j < b) cb += pj;
          if (j == b) pb = pj;
        }
        set_dim(x, d, cb + (u - (float)b) * pb);
        lq += logf(FLOW_BINS * pb);
      }
    }
    if (!ok) break;
    // loss of the tile
    float lv = valid ? -w * lq * inv_batch : 0.0f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lv += __shfl_xor_sync(0xffffffffu, lv, o);
    if (lane == 0) head->red[warp] = lv;
    __syncthreads();
    if (t == 0) {
      const float tot = head->red[0] + head->red[1] + head->red[2] + head->red[3];
      loss_part[blockIdx.x] = first ? tot : loss_part[blockIdx.x] + tot;
    }
    // backward
    float gx[FLOW_MAX_DIM];
#pragma unroll
    for (int d = 0; d < FLOW_MAX_DIM; ++d) gx[d] = 0.0f;
    for (int l = FLOW_LAYERS - 1; l >= 0 && ok; --l) {
      if (valid)
#pragma unroll
        for (int d = 0; d < FLOW_MAX_DIM; ++d) x[d] = xs[((size_t)l * FLOW_MAX_DIM + d) * count + p];
      encode_row(f, l, x, act, t);
      ok = conditioner(P, act, 2, -1, trow);
      if (!ok) break;
      // logit gradients -> act[0] (the features are no longer needed)
      unsigned char *row0 = row_ptr(act, t);
#pragma unroll
      for (int s = 0; s < FLOW_SLOTS; ++s) {
        float g[32];
        if (s < f.ntr[l]) {
          const int d = f.tdim[l][s];
          float v[32];
          tmem_ld32(trow + 32 * s, v);
          float mx = v[0];
#pragma unroll
          for (int j = 1; j < 32; ++j) mx = fmaxf(mx, v[j]);
          float S = 0.0f;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            v[j] = __expf(v[j] - mx);
            S += v[j];
          }
          const float invS = 1.0f / S;
          const float u = get_dim(x, d) * FLOW_BINS;
          const int b = min(max((int)floorf(u), 0), FLOW_BINS - 1);
          const float fr = u - (float)b;
          float pb = 1.0f;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            v[j] *= invS; // softmax
            if (j == b) pb = (1.0f - FLOW_EPS) * v[j] + FLOW_EPS / FLOW_BINS;
          }
          const float gz = get_dim(gx, d);
          float dot = 0.0f;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            float dp = (j < b) ? gz : ((j == b) ? gz * fr + glq / pb : 0.0f);
            g[j] = (1.0f - FLOW_EPS) * dp;
            dot += v[j] * g[j];
          }
#pragma unroll
          for (int j = 0; j < 32; ++j) g[j] = v[j] * (g[j] - dot);
          set_dim(gx, d, gz * FLOW_BINS * pb);
        } else {
#pragma unroll
          for (int j = 0; j < 32; ++j) g[j] = 0.0f;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
          *reinterpret_cast<uint4 *>(row0 + (4 * s + q) * 128) =
              make_uint4(pack_bf16(g[8 * q], g[8 * q + 1]), pack_bf16(g[8 * q + 2], g[8 * q + 3]),
                         pack_bf16(g[8 * q + 4], g[8 * q + 5]), pack_bf16(g[8 * q + 6], g[8 * q + 7]));
      }
      // dW3 = dL^T h2 ; dh2 = dL W3
      Mma mw = {P.tmem + 384, act_addr(P, 0), act_addr(P, 2), 1, 1, 0};
      Mma mx_ = {P.tmem, act_addr(P, 0), w_addr(P, 2), 0, 1, 0};
      if (!(ok = mma_step(P, 2, mw, mx_, 2))) break;
      if (t == 0 && l > 0) load_weight(P, 2, 3 * (l - 1) + 2);
      // g2 = dh2 * [h2 > 0] (unit 127: 0) -> act[2]
      unsigned char *row2 = row_ptr(act + 2 * MAT_BYTES, t);
      unsigned char *row1 = row_ptr(act + MAT_BYTES, t);
#pragma unroll
      for (int pass = 0; pass < 2; ++pass) {
        unsigned char *rowh = pass == 0 ? row2 : row1;
#pragma unroll
        for (int c4 = 0; c4 < 4; ++c4) {
          float v[32];
          tmem_ld32(trow + 32 * c4, v);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            uint4 hv = *reinterpret_cast<const uint4 *>(rowh + (4 * c4 + q) * 128);
            const uint32_t hw[4] = {hv.x, hv.y, hv.z, hv.w};
            uint32_t o[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const float a = bf16_lo(hw[e]) > 0.0f ? v[8 * q + 2 * e] : 0.0f;
              float b = bf16_hi(hw[e]) > 0.0f ? v[8 * q + 2 * e + 1] : 0.0f;
              if (c4 == 3 && q == 3 && e == 3) b = 0.0f;
              o[e] = pack_bf16(a, b);
            }
            *reinterpret_cast<uint4 *>(rowh + (4 * c4 + q) * 128) = make_uint4(o[0], o[1], o[2], o[3]);
          }
        }
        if (pass == 0) {
          // dW2 = g2^T h1 ; dh1 = g2 W2
          Mma a = {P.tmem + 256, act_addr(P, 2), act_addr(P, 1), 1, 1, 0};
          Mma b = {P.tmem, act_addr(P, 2), w_addr(P, 1), 0, 1, 0};
          if (!(ok = mma_step(P, 1, a, b, 2))) break;
          if (t == 0 && l > 0) load_weight(P, 1, 3 * (l - 1) + 1);
        }
      }
      if (!ok) break;
      // the features again -> act[0]; dW1 = g1^T e ; de = g1 W1
      encode_row(f, l, x, act, t);
      Mma a = {P.tmem + 128, act_addr(P, 1), act_addr(P, 0), 1, 1, 0};
      Mma b = {P.tmem, act_addr(P, 1), w_addr(P, 0), 0, 1, 0};
      if (!(ok = mma_step(P, 0, a, b, l > 0 ? 2 : 1))) break;
      if (t == 0 && l > 0) load_weight(P, 0, 3 * (l - 1) + 0);
      if (l > 0) {
        // gradient of the conditioning dims through the hat features
        const unsigned tm = f.tmask[l];
#pragma unroll
        for (int c4 = 0; c4 < 4; ++c4) {
          float v[32];
          tmem_ld32(trow + 32 * c4, v);
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int i = 2 * c4 + h;
            if (i < N && !((tm >> i) & 1u)) {
              const float u = x[i] * (float)FLOW_BLOB - 0.5f;
              const int j0 = (int)floorf(u);
              float gsum = 0.0f;
#pragma unroll
              for (int j = 0; j < 16; ++j) {
                if (j == j0) gsum -= v[16 * h + j];
                if (j == j0 + 1) gsum += v[16 * h + j];
              }
              gx[i] += (float)FLOW_BLOB * gsum;
            }
          }
        }
      }
      // this tile's weight gradients of layer l -> the CTA's partial sums
#pragma unroll 1
      for (int mtx = 0; mtx < 3; ++mtx) {
        float *dst = partials + (size_t)blockIdx.x * FLOW_NPARAM + (size_t)(3 * l + mtx) * FLOW_MAT;
#pragma unroll 1
        for (int c4 = 0; c4 < 4; ++c4) {
          float v[32];
          tmem_ld32(trow + 128 * (1 + mtx) + 32 * c4, v);
#pragma unroll
          for (int e = 0; e < 32; ++e) {
            const size_t idx = (size_t)(32 * c4 + e) * FLOW_W + t;
            dst[idx] = first ? v[e] : dst[idx] + v[e];
          }
        }
      }
    }
  }
  if (!ok && t == 0) atomicOr(err, FLOW_ERR_TIMEOUT);
  pipe_finish(P, 512, err);
}

__device__ __forceinline__ uint16_t bf16_bits(float x) {
  __nv_bfloat16 h = __float2bfloat16_rn(x);
  return *reinterpret_cast<uint16_t *>(&h);
}

// internal order [matrix][in k][out r] -> image element (r, k)
__device__ __forceinline__ size_t img_of(int i) {
  const int mat = i / FLOW_MAT, rem = i - mat * FLOW_MAT, k = rem / FLOW_W, r = rem - k * FLOW_W;
  return (size_t)mat * FLOW_MAT + flow_img_index(r, k);
}

__global__ void flow_reduce_kernel(const float *partials, int nparts, float *grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= FLOW_NPARAM) return;
  float g = 0.0f;
  for (int c = 0; c < nparts; ++c) g += partials[(size_t)c * FLOW_NPARAM + i];
  grad[i] = g;
}

__global__ void flow_adam_kernel(float *master, float *m, float *v, uint16_t *img, const float *partials, int nparts,
                                 const float *loss_part, float *loss_out, float lr, float b1, float b2, float eps,
                                 float bc1, float bc2) {
  if (blockIdx.x == 0 && loss_out && threadIdx.x < 32) {
    float s = 0.0f;
    for (int c = threadIdx.x; c < nparts; c += 32) s += loss_part[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) *loss_out = s;
  }
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= FLOW_NPARAM) return;
  float g = 0.0f;
  for (int c = 0; c < nparts; ++c) g += partials[(size_t)c * FLOW_NPARAM + i];
  const float mm = b1 * m[i] + (1.0f - b1) * g;
  const float vv = b2 * v[i] + (1.0f - b2) * g * g;
  m[i] = mm;
  v[i] = vv;
  const float th = master[i] - lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
  master[i] = th;
  img[img_of(i)] = bf16_bits(th);
}

__global__ void flow_pack_kernel(const float *master, uint16_t *img) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < FLOW_NPARAM) img[img_of(i)] = bf16_bits(master[i]);
}

} // namespace

void flow_layout(int dim, FlowDev &f) {
  f.dim = dim;
  int nb = 1;
  while ((1 << nb) < dim) ++nb;
  for (int l = 0; l < FLOW_LAYERS; ++l) {
    const int b = (l >> 1) % nb;
    f.ntr[l] = 0;
    f.tmask[l] = 0;
    for (int s = 0; s < FLOW_SLOTS; ++s) f.tdim[l][s] = -1;
    for (int i = 0; i < dim; ++i)
      if (((i >> b) & 1) == (l & 1)) {
        f.tdim[l][f.ntr[l]++] = i;
        f.tmask[l] |= 1u << i;
      }
  }
}

size_t flow_map_smem_bytes() { return 3 * (size_t)MAT_BYTES + sizeof(SmemHead) + 1024; }
size_t flow_train_smem_bytes() { return 6 * (size_t)MAT_BYTES + sizeof(SmemHead) + 1024; }

cudaError_t flow_configure() {
  cudaError_t e = cudaFuncSetAttribute(flow_map_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)flow_map_smem_bytes());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(flow_map_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)flow_map_smem_bytes());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(flow_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)flow_train_smem_bytes());
  if (e != cudaSuccess) return e;
  return ar_configure();
}

cudaError_t launch_flow_map(const FlowDev &f, int direction, long long count, const double *in, SobolDev rng,
                            uint32_t k_first, const uint32_t *k_first_dev, int use_sobol, double *out, double *out2,
                            int *err, int grid, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  if (f.kind == FLOW_KIND_SPLINE)
    return launch_spline_map(f.spline, f.dim, direction, count, in, rng, k_first, k_first_dev, use_sobol, out, out2,
                             4 * grid, st);
  if (f.kind == FLOW_KIND_AR_SPLINE)
    return launch_ar_map(f.spline, f.dim, direction, count, in, rng, k_first, k_first_dev, use_sobol, out, out2,
                         4 * grid, st);
  grid *= 2; // two resident CTAs per SM (grid is given as the SM count)
  const long long tiles = (count + NT - 1) / NT;
  if (grid > tiles) grid = (int)tiles;
  const size_t smem = flow_map_smem_bytes();
  if (direction == 0)
    flow_map_kernel<0><<<grid, NT, smem, st>>>(f, count, in, rng, k_first, k_first_dev, use_sobol, out, out2, err);
  else
    flow_map_kernel<1><<<grid, NT, smem, st>>>(f, count, in, rng, k_first, k_first_dev, use_sobol, out, out2, err);
  return cudaGetLastError();
}

cudaError_t launch_flow_train(const FlowDev &f, long long count, const float *x, const float *w, const int *index,
                              float inv_batch, float *partials, float *loss_part, float *xs, int *err, int grid,
                              cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  const long long tiles = (count + NT - 1) / NT;
  if (grid > tiles) grid = (int)tiles;
  flow_train_kernel<<<grid, NT, flow_train_smem_bytes(), st>>>(f, count, x, w, index, inv_batch, partials, loss_part,
                                                               xs, err);
  return cudaGetLastError();
}

cudaError_t launch_flow_reduce(const float *partials, int nparts, float *grad, cudaStream_t st) {
  flow_reduce_kernel<<<(FLOW_NPARAM + 255) / 256, 256, 0, st>>>(partials, nparts, grad);
  return cudaGetLastError();
}

cudaError_t launch_flow_adam(float *master, float *m, float *v, uint16_t *img, const float *partials, int nparts,
                             const float *loss_part, float *loss_out, float lr, float beta1, float beta2, float eps,
                             float bc1, float bc2, cudaStream_t st) {
  flow_adam_kernel<<<(FLOW_NPARAM + 255) / 256, 256, 0, st>>>(master, m, v, img, partials, nparts, loss_part, loss_out,
                                                              lr, beta1, beta2, eps, bc1, bc2);
  return cudaGetLastError();
}

cudaError_t launch_flow_pack(const float *master, uint16_t *img, cudaStream_t st) {
  flow_pack_kernel<<<(FLOW_NPARAM + 255) / 256, 256, 0, st>>>(master, img);
  return cudaGetLastError();
}

} // namespace kb
