// wos_pipe.cuh -- persistent, double-buffered variants of the specialised
// power-of-two sweeps.  Each CTA walks a strided list of work units (row
// groups, or tiles of W columns); the unit after next is fetched by the Tensor
// Memory Accelerator into the stage the current unit has just released, so the
// HBM latency of a unit is covered by the computation of the one before it.
#pragma once
#include <cuda_runtime.h>

#include "wos_fast.cuh"

namespace wos {

// Error bits of the pipelined kernels' device error word.
constexpr unsigned kPipeErrWait = 1u;  // a bounded wait on a copy expired

// Rows: native-precision input and output (no complex128 conversion), the
// input 16-byte aligned with 16-byte multiple row and batch strides.
// Returns cudaErrorNotSupported when the arguments do not meet these
// requirements; *nblocks receives the number of per-CTA reduction records.
cudaError_t pipe_rows(int fp64, int L, int E, bool inv, const FastRows& a, cudaStream_t st, int* nblocks);

// Columns (in place): the data 16-byte aligned with 16-byte multiple row and
// batch strides, and, for complex64, at least two columns per tile (a tile's
// first column then starts on a 16-byte boundary).
cudaError_t pipe_cols(int fp64, int L, int E, const FastCols& a, cudaStream_t st, int* nblocks);

}  // namespace wos
