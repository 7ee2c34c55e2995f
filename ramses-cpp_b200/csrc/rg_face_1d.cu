// rg_face_1d.cu -- instantiation of the tiled face kernel for ndim = 1
// (separate translation unit so the variants compile in parallel).
#include "rg_face.cuh"

namespace rg {
int launch_face_nd1(rg_ctx* c, const Plan& P, const StepK& K, int variant, int batch, const double* uold,
                    const double* prim, double* flux, double* fsum) {
    return launch_face_nd<1>(c, P, K, variant, batch, uold, prim, flux, fsum);
}
}  // namespace rg
