// Host-side set-up of a Sobol generator: generating matrices of the Joe-Kuo 2008
// sequence, optional random digital shift and linear scramble, in the form the device
// kernels consume (bit-reversed columns, "radical inverse" order).
#include <stdint.h>

#include <algorithm>
#include <random>
#include <vector>

#include "sobol_joe_kuo.h"

namespace kb {

static uint32_t bit_reverse32(uint32_t v) {
  v = ((v >> 1) & 0x55555555u) | ((v & 0x55555555u) << 1);
  v = ((v >> 2) & 0x33333333u) | ((v & 0x33333333u) << 2);
  v = ((v >> 4) & 0x0F0F0F0Fu) | ((v & 0x0F0F0F0Fu) << 4);
  v = ((v >> 8) & 0x00FF00FFu) | ((v & 0x00FF00FFu) << 8);
  return (v >> 16) | (v << 16);
}

// Columns 0..m-1 of the generating matrix of every dimension < dim, least significant
// bit = first binary digit (the layout of digitalseq_b2g.hpp:598-861): column k is the
// direction integer m_{k+1} with its k+1 low bits reversed.
void sobol_generating_matrices(int dim, int m, uint32_t *Cs) {
  std::vector<uint32_t> mk(static_cast<size_t>(m));
  for (int j = 0; j < dim; ++j) {
    if (j == 0) {
      std::fill(mk.begin(), mk.end(), 1u); // van der Corput
    } else {
      const kb_joe_kuo_row &row = kb_joe_kuo_rows[j - 1];
      const int s = row.degree;
      for (int k = 0; k < std::min(s, m); ++k) mk[static_cast<size_t>(k)] = row.m_init[k];
      for (int k = s; k < m; ++k) {
        uint32_t v = mk[static_cast<size_t>(k - s)];
        v ^= v << s;
        for (int i = 1; i < s; ++i)
          if ((row.poly >> (s - 1 - i)) & 1u) v ^= mk[static_cast<size_t>(k - i)] << i;
        mk[static_cast<size_t>(k)] = v;
      }
    }
    for (int k = 0; k < m; ++k) Cs[j * m + k] = bit_reverse32(mk[static_cast<size_t>(k)]) >> (31 - k);
  }
}

// keldy::sobol's construction (qrng.hpp:77-109): shifts are the first `dim` outputs of
// std::mt19937_64(seed_shift) narrowed to 32 bits; the scramble matrices are drawn from
// another copy of the freshly seeded engine (std::generate_n and
// generate_random_linear_scramble take it by value), lower triangular with unit
// diagonal (digitalseq_b2g.hpp:209-237), and multiply the generating matrices over Z_2
// (digitalseq_b2g.hpp:156-186). Outputs Csr[dim*m] and shfr[dim] bit-reversed.
void sobol_setup(int dim, int m, bool do_shift, bool do_scramble, int seed_shift, uint32_t *Csr, uint32_t *shfr) {
  std::vector<uint32_t> Cs(static_cast<size_t>(dim) * m);
  sobol_generating_matrices(dim, m, Cs.data());
  std::vector<uint32_t> shifts(static_cast<size_t>(dim), 0u);
  if (do_shift || do_scramble) {
    std::mt19937_64 engine(static_cast<std::mt19937_64::result_type>(static_cast<int64_t>(seed_shift)));
    if (do_shift) {
      std::mt19937_64 g = engine;
      for (int j = 0; j < dim; ++j) shifts[static_cast<size_t>(j)] = static_cast<uint32_t>(g());
    }
    if (do_scramble) {
      uint32_t mx = *std::max_element(Cs.begin(), Cs.end());
      unsigned t = 31;
      while (t && !((1u << (t - 1)) & mx)) t--;
      std::mt19937_64 g = engine;
      std::vector<uint32_t> M(static_cast<size_t>(dim) * t);
      for (int j = 0; j < dim; ++j)
        for (unsigned k = 0; k < t; ++k) {
          uint64_t r = g();
          r &= (uint64_t)((1u << (t - k)) - 1u);
          r |= 1u;
          r <<= k;
          M[static_cast<size_t>(j) * t + k] = static_cast<uint32_t>(r);
        }
      for (int j = 0; j < dim; ++j)
        for (int k = 0; k < m; ++k) {
          uint32_t col = Cs[static_cast<size_t>(j) * m + k], acc = 0;
          for (unsigned i = 0; i < t; ++i)
            if ((col >> i) & 1u) acc ^= M[static_cast<size_t>(j) * t + i];
          Cs[static_cast<size_t>(j) * m + k] = acc;
        }
    }
  }
  for (size_t i = 0; i < Cs.size(); ++i) Csr[i] = bit_reverse32(Cs[i]);
  for (int j = 0; j < dim; ++j) shfr[j] = bit_reverse32(shifts[static_cast<size_t>(j)]);
}

} // namespace kb
