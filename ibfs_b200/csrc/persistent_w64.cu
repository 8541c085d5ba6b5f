// persistent_w64.cu -- the persistent kernel for 64-bit status words
// (persistent.cuh), in a translation unit of its own so that the four widths
// compile in parallel.
#include "internal.h"
#include "persistent.cuh"

namespace ibfs {
const void* persistent_fn_w64(int level) { return persistent_fn<2>(level); }
}  // namespace ibfs
