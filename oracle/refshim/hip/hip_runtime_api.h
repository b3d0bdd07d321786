/* Names-only shim: see hip_runtime.h (test infrastructure only). */
#include "hip_runtime.h"
