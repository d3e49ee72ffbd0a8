// rms_walk_split.cu -- placeholder until the split-precision walk lands.
#include <cuda_runtime.h>
#include "rms_internal.h"
namespace rms {
int launch_walk_split(const WalkArgs&, int, int, void*) { return (int)cudaErrorNotSupported; }
int walk_split_blocks_per_sm(int, int) { return 1; }
}  // namespace rms
