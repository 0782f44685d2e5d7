// Ahead-of-time layout kernels shared by the C ABI (xs_aot.cu).
#pragma once
#include <cuda_runtime.h>

// Block means: device [block][time][stride] -> MATLAB av{o}(lines, time, space)
// per block, observables one after another (complex FP64).
struct XsAvMap {
  int nobs, npts, NS, nout_site, stride, pad;
  long long per_block;  // complex values per block in the MATLAB layout
  int lines[32], spatial[32], out_off[32];
  long long o_off[32];  // first complex value of each observable within a block
};

extern "C" int xs_aot_reorder_launch(const void* src, void* dst, int F, int NS, long long E, int to_device,
                                      cudaStream_t st);
extern "C" int xs_aot_av_matlab_launch(const void* src, void* dst, const XsAvMap* m, int nblocks, cudaStream_t st);
extern "C" int xs_aot_block_moments_launch(const void* av, long long n, int nblocks, double scale, void* mom,
                                            int accumulate, cudaStream_t st);
