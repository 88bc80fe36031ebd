/* Reference header name (csrc/test.h) mapped onto this library's C ABI,
 * so the reference's csrc/module.c builds unchanged against it. */
#include "cuacd_b200.h"
