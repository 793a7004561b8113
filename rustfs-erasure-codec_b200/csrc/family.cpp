// family.cpp -- codec family selection and Leopard shape validation.
#include "codec.hpp"
#include "leopard.hpp"

namespace rsgpu {

// src/core/leopard.rs:191-223: only an untouched Classic request on the byte
// field is eligible for automatic Leopard selection.
int resolve_family(int requested, int mode, size_t total, size_t parity) {
  if (requested != RSGPU_FAMILY_CLASSIC) return requested;
  switch (mode) {
    case RSGPU_LEOPARD_AS_NEEDED:
      return total <= 256 ? RSGPU_FAMILY_CLASSIC : RSGPU_FAMILY_LEOPARD_GF16;
    case RSGPU_LEOPARD_PREFER_GF16:
      return RSGPU_FAMILY_LEOPARD_GF16;
    case RSGPU_LEOPARD_PREFER_LEOPARD:
      return (total <= 256 && parity <= 128) ? RSGPU_FAMILY_LEOPARD_GF8 : RSGPU_FAMILY_LEOPARD_GF16;
    default:
      return RSGPU_FAMILY_CLASSIC;
  }
}

static size_t pow2_ceil(size_t n) {
  size_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

// src/core/leopard.rs:225-237: ceil(k/m)*m must fit in order - m.
static bool combo_fits(size_t k, size_t p, size_t order) {
  size_t m = pow2_ceil(p);
  if (k == 0 || p == 0 || m > order) return false;
  size_t rounded = (k + m - 1) / m * m;
  return rounded <= (order > m ? order - m : 0);
}

int validate_leopard_family(int family, size_t k, size_t m) {
  if (family == RSGPU_FAMILY_LEOPARD_GF8 && !combo_fits(k, m, 256)) return RSGPU_ERR_TOO_MANY_SHARDS;
  if (family == RSGPU_FAMILY_LEOPARD_GF16 && !combo_fits(k, m, 65536)) return RSGPU_ERR_TOO_MANY_SHARDS;
  return RSGPU_OK;
}

}  // namespace rsgpu
