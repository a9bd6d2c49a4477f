/* Host-only stand-in for <cuda.h> used to compile the reference's FisherInfo_IO sources
 * as plain C++ on a machine without a GPU (test infrastructure; built by oracle/build.sh). */
#pragma once
#include "cuda_runtime.h"
