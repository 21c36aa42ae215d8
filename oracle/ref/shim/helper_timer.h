/* Stand-in for the CUDA-SDK helper_timer.h: the CPU path needs nothing from it. */
#pragma once
