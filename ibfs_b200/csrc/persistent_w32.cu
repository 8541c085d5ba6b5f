// persistent_w32.cu -- the persistent kernel for 32-bit status words
// (persistent.cuh), in a translation unit of its own so that the four widths
// compile in parallel.
#include "internal.h"
#include "persistent.cuh"

namespace ibfs {
const void* persistent_fn_w32(int level) { return persistent_fn<1>(level); }
}  // namespace ibfs
