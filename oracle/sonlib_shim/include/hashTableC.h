/* Stand-in for sonLib's hashTableC.h: only `struct hashtable` is named. */
#ifndef MP_SHIM_HASHTABLEC_H_
#define MP_SHIM_HASHTABLEC_H_
#include "sonLib.h"
struct hashtable;
#endif
