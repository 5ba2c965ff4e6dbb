// Stencil kernels instantiated for one element type (cplx<float>).
#include "stencil_launch.cuh"

namespace gfd {

int star_c64(const gfd_operator* op, int mode, const void* in, void* out, const void* rho,
               int64_t nin, const double* ph, double w, double* partials, cudaStream_t s) {
  return launch_star_typed<cplx<float>>(op, mode, in, out, rho, nin, ph, w, partials, s);
}

int general_c64(const gfd_operator* op, int mode, const void* in, void* out, const void* rho,
                  int64_t nin, const double* ph, double w, double* partials, cudaStream_t s) {
  return launch_general_typed<cplx<float>>(op, mode, in, out, rho, nin, ph, w, partials, s);
}

}  // namespace gfd
