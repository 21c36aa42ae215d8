/* Stand-in for cudpp.h (CUDPP 2.x is not installed).  Only the enum and
 * handle types named by the reference's headers are declared; the CPU path
 * makes no CUDPP call, and the GPU combiner that does is not compiled. */
#pragma once
typedef enum { CUDPP_ADD, CUDPP_MULTIPLY, CUDPP_MIN, CUDPP_MAX } CUDPPOperator;
typedef enum { CUDPP_CHAR, CUDPP_UCHAR, CUDPP_SHORT, CUDPP_USHORT, CUDPP_INT,
               CUDPP_UINT, CUDPP_FLOAT, CUDPP_DOUBLE } CUDPPDatatype;
typedef enum { CUDPP_SCAN, CUDPP_SEGMENTED_SCAN } CUDPPAlgorithm;
typedef size_t CUDPPHandle;
typedef int CUDPPResult;
typedef struct { CUDPPAlgorithm algorithm; CUDPPOperator op;
                 CUDPPDatatype datatype; unsigned int options; } CUDPPConfiguration;
