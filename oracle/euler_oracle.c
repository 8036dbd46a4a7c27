/* euler_oracle.c -- binary64 and binary32 instantiations of the Euler
 * sibling's oracle (euler_oracle.h), plus .dat writers in the reference's
 * format.  TEST INFRASTRUCTURE ONLY (loaded by tests/ through ctypes). */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#define ET double
#define EF f64
#include "euler_oracle.h"
#undef ET
#undef EF
#define ET float
#define EF f32
#include "euler_oracle.h"
#undef ET
#undef EF
