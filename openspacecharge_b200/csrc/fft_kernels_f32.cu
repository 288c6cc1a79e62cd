// fft_kernels_f32.cu -- FP32 instantiations of the FFT kernels (fft_kernels_impl.cuh).
#define OSC_FFT_DEFINE_PLAN
#include "fft_kernels_impl.cuh"

namespace osc {
template int launch_lines<float>(const cplx<float> *, cplx<float> *, const LineArgs &, int, int, bool,
                                 const TwPair<cplx<float>> &, cudaStream_t);
template int launch_r2c_rows<float, float>(const float *, cplx<float> *, const R2CArgs &, const TwPair<cplx<float>> &,
                                           cudaStream_t);
template int launch_r2c_rows<float, float4>(const float4 *, cplx<float> *, const R2CArgs &,
                                            const TwPair<cplx<float>> &, cudaStream_t);
template int launch_r2c_rows<float, double>(const double *, cplx<float> *, const R2CArgs &,
                                            const TwPair<cplx<float>> &, cudaStream_t);
template int launch_c2r_rows<float>(const cplx<float> *, const C2RArgs &, const TwPair<cplx<float>> &, cudaStream_t);
template int launch_zconv<float>(const cplx<float> *, cplx<float> *, const ZConvArgs &, const TwPair<cplx<float>> &,
                                 int, cudaStream_t);
template int launch_sym_lines<float, float, float>(const float *, float *, const SymArgs &,
                                                   const TwPair<cplx<float>> &, bool, bool, cudaStream_t);
}  // namespace osc
