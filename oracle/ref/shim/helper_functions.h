/* Stand-in for the CUDA-SDK helper_functions.h: the CPU path needs nothing from it. */
#pragma once
