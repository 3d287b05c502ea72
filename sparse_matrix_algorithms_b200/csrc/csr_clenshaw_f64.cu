// FP64 instantiation of the fused CSR Clenshaw step (csr_clenshaw.cuh).
#include "csr_clenshaw.cuh"

template void sma::csr_clenshaw_step<double>(const sma_op *, cudaStream_t, int64_t, const double *,
                                             int64_t, const double *, const double *, int64_t,
                                             double *, int64_t, double, double, double, bool);
template void sma::csr_clenshaw_step_untuned<double>(const sma_op *, cudaStream_t, int64_t,
                                                     const double *, int64_t, const double *,
                                                     const double *, int64_t, double *, int64_t,
                                                     double, double, double, bool);
template void sma::csr_clenshaw_step_seg<double>(const sma_op *, cudaStream_t, int64_t,
                                                 const double *, int64_t, const double *, const double *,
                                                 int64_t, double *, int64_t, const double *, const int *,
                                                 double, double, bool);
