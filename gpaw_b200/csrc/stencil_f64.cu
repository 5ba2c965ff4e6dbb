// Stencil kernels instantiated for one element type (double).
#include "stencil_launch.cuh"

namespace gfd {

int star_f64(const gfd_operator* op, int mode, const void* in, void* out, const void* rho,
               int64_t nin, const double* ph, double w, double* partials, cudaStream_t s) {
  return launch_star_typed<double>(op, mode, in, out, rho, nin, ph, w, partials, s);
}

int general_f64(const gfd_operator* op, int mode, const void* in, void* out, const void* rho,
                  int64_t nin, const double* ph, double w, double* partials, cudaStream_t s) {
  return launch_general_typed<double>(op, mode, in, out, rho, nin, ph, w, partials, s);
}

}  // namespace gfd
