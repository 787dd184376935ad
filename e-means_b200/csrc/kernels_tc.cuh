// tcgen05 (5th-generation tensor core) fused assign kernels.
#pragma once
#include "common.cuh"
