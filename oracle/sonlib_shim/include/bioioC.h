/* Stand-in for sonLib's bioioC.h: the hot-path sources need nothing from it. */
#ifndef MP_SHIM_BIOIOC_H_
#define MP_SHIM_BIOIOC_H_
#include "sonLib.h"
#endif
