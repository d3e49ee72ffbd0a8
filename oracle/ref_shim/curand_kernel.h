/* oracle/ref_shim/curand_kernel.h -- TEST INFRASTRUCTURE: stand-in header so the reference simulator source compiles for the host; everything lives in rms_ref_shim.hpp (force-included). */
#include "rms_ref_shim.hpp"
