/*
 * oracle/ref_layout.cpp -- ORACLE (test infrastructure only).
 *
 * Layout check of include/bte/launch_params.h against the reference's own headers.
 * Compiled twice by oracle/Makefile into one library: with -DBTE_LAYOUT_REFERENCE
 * it includes the reference's include/optix_launch_params.h (through the OptiX and
 * CUDA shims) and exports ref_layout(); otherwise it includes the library's header
 * and exports bte_layout().  Each fills a table of (offset, size) per field plus the
 * four struct sizes; tests/test_abi.py compares the two tables.
 */
#include <cstddef>
#ifdef BTE_LAYOUT_REFERENCE
#include "optix_launch_params.h"
#define BTE_LAYOUT_FN ref_layout
#else
#include "bte/launch_params.h"
#define BTE_LAYOUT_FN bte_layout
#endif
#include "ref_layout_fields.h"

extern "C" __attribute__((visibility("default"))) int BTE_LAYOUT_FN(long long* out, int capacity)
{
    static const long long table[] = BTE_LAYOUT_TABLE;
    const int n = (int)(sizeof(table) / sizeof(table[0]));
    for (int i = 0; i < n && i < capacity; ++i) out[i] = table[i];
    return n;
}
