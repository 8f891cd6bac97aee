// cgb_internal.h -- shared host-side declarations of libcgb.
#pragma once

#include "../../include/cgb.h"

namespace cgb {

// Records a formatted message as the calling thread's last error and returns
// `status` unchanged, so call sites read `return set_error(...)`.
int set_error(int status, const char *fmt, ...);

// Odd integer in (1, 2^46): the LCG's admissible seeds (c_randdp.cpp:70-71).
bool valid_seed(double seed);

// Generator (makea.cpp).
int makea(int n, int nonzer, double rcond, double shift, double seed, int *rowstr, int *colidx,
          double *a, long long cap, long long *nnz_out);

}  // namespace cgb
