/* Compatibility header: callers of the reference's include/skinny.h keep
 * compiling; the declarations live in inplace_detail.h. */
#pragma once
#include "inplace_detail.h"
