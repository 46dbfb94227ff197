/* Compiles the reference He-Ar plugin header (PES-IDS/HeAr.h) as-is into
 * oracle/_ref/libref_hear.so.  Test infrastructure only. */
#define HEAR_IMPLEMENTATION
#include "HeAr.h"
