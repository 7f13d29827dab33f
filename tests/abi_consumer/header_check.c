/* The ABI header is plain C: this translation unit includes it with a C compiler and
 * takes the address of every entry point through a pointer of its declared type. */
#include "litho_b200.h"

int header_check_main(void) {
  int (*create)(int, void*, litho_ctx**) = litho_ctx_create;
  int (*imaging)(litho_ctx*, const litho_cache*, const float*, double, double, float*, float*,
                 litho_field*) = litho_imaging_compute;
  int (*rk2)(void*, int, int, const float*, const float*, double, double, double, double, float*,
             float*, double*) = litho_lsm_rk2_update_noalloc;
  return create != 0 && imaging != 0 && rk2 != 0;
}
