// Host-side objects of the C ABI shared by capi.cu and flow_capi.cu: error
// reporting, stream-ordered device buffers, and the opaque handle types of
// include/keldy_b200.h.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <atomic>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "kb_flow.h"
#include "kb_launch.h"
#include "kb_types.h"

namespace kb {
// Records msg as the calling thread's last error (kb_last_error) and returns code.
int fail(int code, const std::string &msg);

// The current device's memory pool of the library's stream-ordered allocations: unlike the
// device's default pool, which hands freed memory back to the driver at every
// synchronisation (so that the next call maps it again), it keeps up to
// KB_POOL_KEEP_BYTES of freed memory cached for the next call.
constexpr unsigned long long KB_POOL_KEEP_BYTES = 256ull << 20;
cudaMemPool_t kb_pool();

// Every device allocation of the library goes through device_malloc or DevBuf::alloc,
// which count it (kb_device_allocations reads the count).
std::atomic<unsigned long long> &device_allocations();
template <typename T> cudaError_t device_malloc(T **p, size_t bytes) {
  device_allocations().fetch_add(1, std::memory_order_relaxed);
  return cudaMalloc(reinterpret_cast<void **>(p), bytes);
}

// Stream-ordered device buffer released at scope exit (on the same stream).
struct DevBuf {
  void *p = nullptr;
  cudaStream_t st = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  cudaError_t alloc(size_t bytes, cudaStream_t s) {
    st = s;
    device_allocations().fetch_add(1, std::memory_order_relaxed);
    return cudaMallocFromPoolAsync(&p, bytes ? bytes : 16, kb_pool(), s);
  }
  ~DevBuf() {
    if (p) cudaFreeAsync(p, st);
  }
  template <typename T> T *as() const { return static_cast<T *>(p); }
};

// Content hash of a table (equality test of spin blocks): four independent lanes of
// 64-bit words, each an FNV-1a step on the word followed by a xor-shift, then the lanes
// and the tail bytes combined.
inline uint64_t fnv1a(const void *data, size_t n) {
  const unsigned char *c = static_cast<const unsigned char *>(data);
  const uint64_t P = 1099511628211ULL;
  uint64_t h[4] = {1469598103934665603ULL, 0x9E3779B97F4A7C15ULL, 0xC2B2AE3D27D4EB4FULL, 0x165667B19E3779F9ULL};
  size_t i = 0;
  for (; i + 32 <= n; i += 32)
    for (int k = 0; k < 4; ++k) {
      uint64_t w;
      memcpy(&w, c + i + 8 * k, 8);
      h[k] = (h[k] ^ w) * P;
      h[k] ^= h[k] >> 29;
    }
  uint64_t r = h[0] ^ (h[1] * 3) ^ (h[2] * 5) ^ (h[3] * 7);
  for (; i < n; ++i) r = (r ^ c[i]) * P;
  return r ^ n;
}

} // namespace kb

#define KB_CUDA(call)                                                                                        \
  do {                                                                                                       \
    cudaError_t e_ = (call);                                                                                 \
    if (e_ != cudaSuccess) return kb::fail(KB_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
  } while (0)

#define KB_CHECK(cond, msg)                                                                                  \
  do {                                                                                                       \
    if (!(cond)) return kb::fail(KB_E_INVALID, msg);                                                        \
  } while (0)

struct kb_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sm_count = 0;
  int tree_grid = 0;
  int *d_err = nullptr; // error flags written by kernels
  int chunk_points[kb::MAX_ORDER + 1]; // scheduling chunk of each order (autotuned; default 128)
  int ctas_per_sm = 4;                 // resident tree CTAs per SM
  bool timing = false;
  cudaEvent_t ev[4] = {};
  double last_ms[3] = {0, 0, 0};
  int last_launches = 0;
  std::mutex mu;
};

// Models, generators and flows belong to a context and must be destroyed before it;
// their destroy functions touch only the device they live on.
struct kb_model {
  kb_context *ctx = nullptr;
  int device = 0;
  int npts = 0;
  double tmax = 0, alpha = 0;
  double2 *tab[2][2][2] = {};
  uint64_t hash[2][2][2] = {}; // 0 = unknown (device upload)
  double tabmax = 0;
  int interp = 1; // 1 linear, 3 cubic
  // tab[0][0][0] lies in a device block shared with the other models of one
  // kb_models_set_flatband call (freed with its last owner) instead of its own allocation
  std::shared_ptr<void> slab;
};

struct kb_sobol {
  kb_context *ctx = nullptr;
  int device = 0;
  int dim = 0, m = 0;
  uint32_t *d_Csr = nullptr;
  uint32_t *d_shfr = nullptr;
};

namespace kb {
SobolDev sobol_dev(const kb_sobol *s);
// KB_E_EXHAUSTED when points k_first .. k_first+count-1 pass the generator's end
int check_sobol_range(const kb_sobol *s, uint32_t k_first, int64_t count);
} // namespace kb

// Device-resident product warper (tabulated, projection, hybrid or per-coordinate
// analytic): the per-coordinate descriptors and their arrays on the device, and what the
// projection warper reports back (its widths, binned projections and smoothed fn).
struct kb_warper_table {
  kb_context *ctx = nullptr;
  int device = 0;
  int ndims = 0;
  int type = KB_TABLE_NEAREST;
  double u_max = 0.0;
  kb::TableDimDev *d_dims = nullptr; // [ndims]
  double *d_data = nullptr;          // all coordinates' arrays
  std::vector<int> npts;             // points of each coordinate's first table
  std::vector<std::vector<double>> pts_u, pts_f1; // nearest tables: the points and f1 as given
  std::vector<double> sigmas;        // projection: smoothing width per axis (natural units)
  std::vector<std::vector<double>> xi;
  std::vector<std::vector<uint64_t>> xi_count;
  std::vector<std::vector<double>> fn;
};

namespace kb {
// The device form of one analytic product maker (the constants of make_warper_dev).
int simple_dev(const kb_warper &w, SimpleDev &out);
} // namespace kb

// Learned coupling-flow warper: fp32 master weights and Adam moments in the internal
// order [matrix][in][out], bf16 images for the tensor cores.
struct kb_flow {
  kb_context *ctx = nullptr;
  int device = 0;
  int dim = 0;
  kb::FlowDev layout{};    // img set to `img`
  float *master = nullptr; // [FLOW_NPARAM]
  float *adam_m = nullptr;
  float *adam_v = nullptr;
  uint16_t *img = nullptr; // [FLOW_NPARAM] bf16
  double *knots = nullptr; // spline flows: [FLOW_MAX_DIM][SPL_KNOT_DOUBLES], made at each integration
  int64_t adam_step = 0;
};
