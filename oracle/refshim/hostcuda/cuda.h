// Host-compiler stand-in for <cuda.h>, used only to compile the reference's
// device code as plain C++ for the CPU parity oracle (TEST INFRASTRUCTURE).
#pragma once
#include "cuda_runtime.h"
