/* Stand-in for the CUDA-SDK cutil_inline_runtime.h: the CPU path needs nothing from it. */
#pragma once
