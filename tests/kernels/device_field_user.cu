// An application kernel that evaluates a reconstructed field through psr_field.cuh, as a
// warp-psr user kernel calls evaluate_field(field, point) (the reference's
// tests/test_device_field.py query kernel).  Built without --fmad=false on purpose.
#include <cuda_runtime.h>

#include "psr_field.cuh"

template <class T>
__global__ void query_kernel(psr_field_handle field, const T* queries, int64_t n, T* values, T* gradients,
                             int32_t* valid) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const auto r = psr_evaluate_field(field, queries[3 * i], queries[3 * i + 1], queries[3 * i + 2]);
  values[i] = r.value;
  for (int a = 0; a < 3; ++a) gradients[3 * i + a] = r.gradient[a];
  valid[i] = r.valid;
}

extern "C" int user_evaluate(const psr_field_handle* field, const void* queries, int64_t n, void* values,
                             void* gradients, int32_t* valid, void* stream) {
  if (n <= 0) return 0;
  const unsigned blocks = unsigned((n + 127) / 128);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (field->dtype == PSR_FLOAT64)
    query_kernel<double><<<blocks, 128, 0, s>>>(*field, static_cast<const double*>(queries), n,
                                                static_cast<double*>(values), static_cast<double*>(gradients), valid);
  else
    query_kernel<float><<<blocks, 128, 0, s>>>(*field, static_cast<const float*>(queries), n,
                                               static_cast<float*>(values), static_cast<float*>(gradients), valid);
  return int(cudaGetLastError());
}
