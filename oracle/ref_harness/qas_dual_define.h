/* Forced include for the dual-number build of the reference sources: the dual
 * type and every system header first, then `double` means qd.  Test infrastructure. */
#include "qas_dual.h"
#define double qd
