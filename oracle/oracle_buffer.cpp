/* CPU FP64 oracle, distance and erosion joins (buffer.cuh restatements) - TEST INFRASTRUCTURE ONLY. */
#include "oracle.h"
