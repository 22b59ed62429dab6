// Shared constants between the public C header and the device code.
#pragma once
#include "mpm_capi.h"

#define MPM_GHOST 3

// device-side error flag bits, OR-ed into a per-handle word
#define MPM_FLAG_NAN 1u
#define MPM_FLAG_DOMAIN 2u
#define MPM_FLAG_NOT_CONVERGED 4u
#define MPM_FLAG_TIMEOUT 8u
#define MPM_FLAG_ORDER 16u       // the fast path's per-block counts were out of step (nothing written)
