// FP32 instantiation of the fused CSR Clenshaw step (csr_clenshaw.cuh).
#include "csr_clenshaw.cuh"

template void sma::csr_clenshaw_step<float>(const sma_op *, cudaStream_t, int64_t, const float *,
                                            int64_t, const float *, const float *, int64_t, float *,
                                            int64_t, double, double, double, bool);
template void sma::csr_clenshaw_step_untuned<float>(const sma_op *, cudaStream_t, int64_t,
                                                    const float *, int64_t, const float *,
                                                    const float *, int64_t, float *, int64_t,
                                                    double, double, double, bool);
template void sma::csr_clenshaw_step_seg<float>(const sma_op *, cudaStream_t, int64_t,
                                                 const float *, int64_t, const float *, const float *,
                                                 int64_t, float *, int64_t, const float *, const int *,
                                                 double, double, bool);
