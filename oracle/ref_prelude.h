/* Host-C++ prelude that lets the reference's CUDA sources compile as plain C++ so that they
 * can be run on the CPU as a parity oracle (test infrastructure only).  A CUDA "launch" is
 * emulated by ref_launch.cpp, which walks blockIdx/threadIdx one thread at a time. */
#pragma once
#include <cmath>
#include <algorithm>
using std::fmax; using std::fmin; using std::sqrt; using std::acos;
using std::max; using std::min; using std::abs; using std::lgamma; using std::pow; using std::exp;
#define __global__
#define __device__
#define __forceinline__ inline
#define __restrict__
/* block-shared tables become function statics (filled by emulated threads before use) */
#define __shared__ static
#define __syncthreads() ((void)0)
struct hb_dim3 { long long x, y, z; };
extern hb_dim3 blockIdx, threadIdx, blockDim, gridDim;
