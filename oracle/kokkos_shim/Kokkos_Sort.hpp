// Shim: sort / sort_by_key live in Kokkos_Core.hpp (test infrastructure).
#include "Kokkos_Core.hpp"
