/* Forced include for compiling the reference's own test driver
 * (tests/test.c), which calls sp_norm_f (src/norm.c:37) without a
 * declaration; with an implicit int return the driver crashes.  The
 * reference header has no include guard, so the declaration is K&R style.
 * Test infrastructure only. */
#include <stdlib.h>
double sp_norm_f();
