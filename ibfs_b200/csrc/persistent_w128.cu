// persistent_w128.cu -- the persistent kernel for 128-bit status words
// (persistent.cuh), in a translation unit of its own so that the four widths
// compile in parallel.
#include "internal.h"
#include "persistent.cuh"

namespace ibfs {
const void* persistent_fn_w128(int level) { return persistent_fn<4>(level); }
}  // namespace ibfs
