/*
 * Stand-in for sonLib's private list header, which impl/polisher.c includes but whose
 * contents it does not use beyond the public stList API (TEST INFRASTRUCTURE ONLY).
 */
#ifndef MP_SONLIB_LIST_PRIVATE_SHIM_H_
#define MP_SONLIB_LIST_PRIVATE_SHIM_H_
#include "sonLib.h"
#endif
