/* Reference header name (csrc/preprocess.h) mapped onto this library's C ABI,
 * so the reference's csrc/module.c builds unchanged against it. */
#include "cuacd_b200.h"
