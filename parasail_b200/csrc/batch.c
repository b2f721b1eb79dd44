/*
 * batch.c -- parasail-b200 batch API (include/parasail_b200.h).
 */
#include "pb_internal.h"
