// Stand-in for itertools/omp_chunk.hpp (test infrastructure; not used on the hot path).
#pragma once
