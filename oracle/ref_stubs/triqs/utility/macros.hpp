// Stand-in for TRIQS's macros.hpp (test infrastructure).
#pragma once
#include "exceptions.hpp"
