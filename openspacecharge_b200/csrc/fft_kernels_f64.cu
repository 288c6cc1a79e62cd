// fft_kernels_f64.cu -- FP64 instantiations of the FFT kernels (fft_kernels_impl.cuh).
#include "fft_kernels_impl.cuh"

namespace osc {
template int launch_lines<double>(const cplx<double> *, cplx<double> *, const LineArgs &, int, int, bool,
                                  const TwPair<cplx<double>> &, cudaStream_t);
template int launch_r2c_rows<double, double>(const double *, cplx<double> *, const R2CArgs &,
                                             const TwPair<cplx<double>> &, cudaStream_t);
template int launch_c2r_rows<double>(const cplx<double> *, const C2RArgs &, const TwPair<cplx<double>> &,
                                     cudaStream_t);
template int launch_zconv<double>(const cplx<double> *, cplx<double> *, const ZConvArgs &,
                                  const TwPair<cplx<double>> &, int, cudaStream_t);
template int launch_sym_lines<double, double, double>(const double *, double *, const SymArgs &,
                                                      const TwPair<cplx<double>> &, bool, bool, cudaStream_t);
}  // namespace osc
