/* Layout of the public structs of the C ABI -- TEST INFRASTRUCTURE ONLY.
 *
 * oracle/build.py compiles this file twice:
 *   -DLAYOUT_EMIT against the reference's header (src/fast_hankel_nufht.h:21-97): a program
 *     that prints every struct size and field offset as a #define; its output is written to
 *     oracle/_ref/abi_layout_ref.h;
 *   without it, against include/nufht_b200.h plus that generated header: a program that
 *     compiles only when every size and offset equals the reference's (C11 _Static_assert).
 * A mismatch therefore fails the build instead of surfacing as corrupted plans at run time.
 */
#include <stddef.h>
#include <stdio.h>

#ifdef LAYOUT_EMIT
#include "fast_hankel_nufht.h"
#else
#include "nufht_b200.h"
#include "abi_layout_ref.h"
#endif

#define ABI_TYPES(X) X(NufhtOptions) X(Box) X(BoxVector) X(Boxes) X(NufhtPlan) X(NufhtScratch)

#define ABI_FIELDS(X)                                                                      \
    X(NufhtOptions, tol) X(NufhtOptions, max_levels) X(NufhtOptions, min_dim_prod)         \
    X(NufhtOptions, z_split) X(NufhtOptions, K_asy) X(NufhtOptions, K_loc)                 \
    X(Box, i0) X(Box, i1) X(Box, j0) X(Box, j1)                                            \
    X(BoxVector, data) X(BoxVector, length) X(BoxVector, capacity)                         \
    X(Boxes, loc) X(Boxes, asy) X(Boxes, dir)                                              \
    X(NufhtPlan, nu) X(NufhtPlan, tol) X(NufhtPlan, z_split) X(NufhtPlan, K_asy)           \
    X(NufhtPlan, K_loc) X(NufhtPlan, asy_coef) X(NufhtPlan, m) X(NufhtPlan, n)             \
    X(NufhtPlan, rs) X(NufhtPlan, ws) X(NufhtPlan, max_levels) X(NufhtPlan, min_dim_prod)  \
    X(NufhtPlan, boxes) X(NufhtPlan, tables_loaded)                                        \
    X(NufhtScratch, in_buffer) X(NufhtScratch, out_buffer) X(NufhtScratch, real_buffer_1)  \
    X(NufhtScratch, real_buffer_2) X(NufhtScratch, cheb_buffer)                            \
    X(NufhtScratch, bessel_buffer_1) X(NufhtScratch, bessel_buffer_2)                      \
    X(NufhtScratch, m_alloc) X(NufhtScratch, n_alloc) X(NufhtScratch, Kloc_alloc)          \
    X(NufhtScratch, extra_alloc)

#ifdef LAYOUT_EMIT

#define EMIT_SIZE(T) printf("#define REF_SIZEOF_%s %zu\n", #T, sizeof(T));
#define EMIT_OFFSET(T, f) printf("#define REF_OFFSET_%s_%s %zu\n", #T, #f, offsetof(T, f));

int main(void)
{
    ABI_TYPES(EMIT_SIZE)
    ABI_FIELDS(EMIT_OFFSET)
    return 0;
}

#else

#define CHECK_SIZE(T) _Static_assert(sizeof(T) == REF_SIZEOF_##T, "sizeof(" #T ") differs from the reference");
#define CHECK_OFFSET(T, f) \
    _Static_assert(offsetof(T, f) == REF_OFFSET_##T##_##f, "offset of " #T "." #f " differs from the reference");

ABI_TYPES(CHECK_SIZE)
ABI_FIELDS(CHECK_OFFSET)

int main(void)
{
    int n = 0;
#define COUNT(...) ++n;
    ABI_TYPES(COUNT)
    ABI_FIELDS(COUNT)
    printf("abi layout matches the reference header: %d sizes and offsets\n", n);
    return 0;
}

#endif
