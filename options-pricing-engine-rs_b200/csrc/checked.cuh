// Bounds-checked build (make CHECKED=1, the library at lib/checked/): device
// invariants of the pricing and adjoint kernels -- panel-list indices and
// counts, surface indices, panel-list slots -- are tested at run time.  A
// failed test sets a bit of a device-wide check word and the kernel avoids
// the bad access (clamps or skips); it never traps.  The host reads and
// clears the word with ope_check_word().  In the ordinary build the tests
// compile to nothing.
#pragma once

#ifndef OPE_CHECKED
#define OPE_CHECKED 0
#endif

namespace ope {

enum : unsigned {
    CHK_PANEL_INDEX = 1u,  // argmax index outside the live panel list
    CHK_PANEL_COUNT = 2u,  // a bisection with the list already full
    CHK_SURFACE = 4u,      // parameter-set index outside [0, n_surf)
    CHK_SLOT = 8u,         // panel-list slot outside [0, n_slots)
    CHK_PANEL_LEN = 16u,   // stored bisection count outside [0, kMaxPanels)
    CHK_RUN_ENTRY = 32u,   // run-cache entry outside the run's allocated entries
};

#if OPE_CHECKED
extern __device__ unsigned int g_ope_check_word;
// true when `ok`; otherwise records `bit` and returns false.
__device__ __forceinline__ bool ope_check(bool ok, unsigned bit) {
    if (!ok) atomicOr(&g_ope_check_word, bit);
    return ok;
}
#else
__device__ __forceinline__ bool ope_check(bool, unsigned) { return true; }
#endif

}  // namespace ope
