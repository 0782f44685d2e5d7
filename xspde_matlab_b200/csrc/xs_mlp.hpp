// Control-variate MLP kernels (xs_mlp.cu).
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

size_t xs_mlp_layout(int in, int hidden, int batch, size_t* nparams);
int xs_mlp_forward_impl(int B, int in, int H, const float* x, const float* P, float* work, float* y, cudaStream_t st,
                        bool train);
int xs_mlp_status(cudaStream_t st);
int xs_mlp_uses_tensor_memory(int in, int hidden);
int xs_mlp_backward_impl(int B, int in, int H, const float* x, const float* P, float* work, const float* target,
                         float* grad, double* loss, cudaStream_t st);
int xs_mlp_adam_impl(size_t n, float* P, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
                     int step, float wd, cudaStream_t st);
