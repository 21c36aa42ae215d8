/* Stand-in for the CUDA-SDK helper_cuda.h: the CPU path needs nothing from it. */
#pragma once
