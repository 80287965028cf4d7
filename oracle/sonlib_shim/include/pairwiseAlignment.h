/* Stand-in for sonLib's pairwiseAlignment.h: only the struct name is referenced
 * (in a prototype of inc/pairwiseAligner.h). */
#ifndef MP_SHIM_PAIRWISEALIGNMENT_H_
#define MP_SHIM_PAIRWISEALIGNMENT_H_
#include "sonLib.h"
struct PairwiseAlignment;
#endif
