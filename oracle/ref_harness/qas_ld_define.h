/* Forced include for the extended-precision build of the reference's 2D stepping code: every
 * system header first (qas_dual.h lists them), mixed-precision min/max beside the reference's
 * templates (common/common_func.h:4-14 deduce one TYPE, so max(0.0, x) with x long double needs
 * an overload), then `double` means long double (x87 80-bit: 64-bit significand).  The
 * constants of the sources stay the double literals they are.  Test infrastructure: the
 * finite differences of the adjoint's gradient check are taken on this build. */
#include "qas_dual.h"
inline long double max(long double a, long double b) { return (a >= b) ? a : b; }
inline long double min(long double a, long double b) { return (a >= b) ? b : a; }
#define double long double
