// Shim: math functions live in Kokkos_Core.hpp (test infrastructure).
#include "Kokkos_Core.hpp"
