// Batched SVD of many small matrices in one persistent launch (batched.cu).
#pragma once

#include "common.cuh"
