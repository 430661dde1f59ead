// backward.cu -- vector-Jacobian product of the LETKF analysis (placeholder).
#include "point.cuh"

namespace sbl {
int launch_backward(sbletkf_workspace *, const sbletkf_params *, const GridView &, const void *, const void *, int,
                    const void *, const void *, double *, double *, double *, double *, cudaStream_t) {
  return SBLETKF_ERR_UNSUPPORTED;
}
}  // namespace sbl
