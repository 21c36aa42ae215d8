"""medusa_b200 -- Medusa's BSP superstep (BFS, SSSP, PageRank) on B200 / sm_100a.

The product is libmedusa_b200.so behind the C ABI in include/medusa_b200.h
(built by ``python -m medusa_b200.build``); ``medusa_b200.api`` is its ctypes
binding and include/medusa/*.h the reference-named C++ API on top of it.
Import ``medusa_b200.api`` explicitly: importing the package alone loads
nothing, so the build step works before the library exists.
"""
