/* Stand-in for the CUDA-SDK cutil.h: the CPU path needs nothing from it. */
#pragma once
