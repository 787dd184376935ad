// Device kernels of the training update path.
#pragma once
#include "common.cuh"
