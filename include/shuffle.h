/* Compatibility header: callers of the reference's include/shuffle.h keep
 * compiling; the declarations live in inplace_detail.h. */
#pragma once
#include "inplace_detail.h"
