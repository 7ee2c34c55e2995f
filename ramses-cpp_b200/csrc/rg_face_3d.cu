// rg_face_3d.cu -- instantiation of the face kernels for ndim = 3 (separate
// translation unit so the variants compile in parallel): the tiled kernel's
// variants 0..6, the software-pipelined kernel's variants 7..8 and the brick
// kernel's variants 9..10.
#include "rg_face_brick.cuh"
#include "rg_face_pipe.cuh"

namespace rg {

namespace {
template <int RS>
int launch_pipe_rs(rg_ctx* c, const Plan& P, const StepK& K, int variant, const double* prim, double* flux,
                   double* fsum) {
    if (P.nbox > 0) return launch_face_pipe<3, RS, 4, true>(c, P, K, prim, flux, fsum);
    if (variant == kFirstPipeVariant) return launch_face_pipe<3, RS, 4>(c, P, K, prim, flux, fsum);
    return launch_face_pipe<3, RS, 3>(c, P, K, prim, flux, fsum);
}
template <int RS>
int launch_brick_rs(rg_ctx* c, const Plan& P, const StepK& K, int variant, const double* prim, double* flux,
                    double* fsum) {
    if (P.nbox > 0) return launch_face_brick<RS, 2, true>(c, P, K, prim, flux, fsum);
    if (variant == kFirstBrickVariant) return launch_face_brick<RS, 3>(c, P, K, prim, flux, fsum);
    return launch_face_brick<RS, 2>(c, P, K, prim, flux, fsum);
}
}  // namespace

int launch_face_nd3(rg_ctx* c, const Plan& P, const StepK& K, int variant, int batch, const double* uold,
                    const double* prim, double* flux, double* fsum) {
    if (variant >= kFirstBrickVariant) {
        const bool ok = P.nbox > 0 ? P.box_lattice != 0 : P.lattice != 0;
        if (!ok) return launch_face_nd<3>(c, P, K, kDefaultFaceVariant, batch, uold, prim, flux, fsum);
        switch (c->params.riemann) {
            case RG_RIEMANN_HLLC: return launch_brick_rs<RG_RIEMANN_HLLC>(c, P, K, variant, prim, flux, fsum);
            case RG_RIEMANN_HLL: return launch_brick_rs<RG_RIEMANN_HLL>(c, P, K, variant, prim, flux, fsum);
            case RG_RIEMANN_EXACT: return launch_brick_rs<RG_RIEMANN_EXACT>(c, P, K, variant, prim, flux, fsum);
            case RG_RIEMANN_ACOUSTIC: return launch_brick_rs<RG_RIEMANN_ACOUSTIC>(c, P, K, variant, prim, flux, fsum);
            default: return launch_brick_rs<RG_RIEMANN_LLF>(c, P, K, variant, prim, flux, fsum);
        }
    }
    if (variant >= kFirstPipeVariant) {
        if (P.level0) return launch_face_nd<3>(c, P, K, kDefaultFaceVariant, batch, uold, prim, flux, fsum);
        switch (c->params.riemann) {
            case RG_RIEMANN_HLLC: return launch_pipe_rs<RG_RIEMANN_HLLC>(c, P, K, variant, prim, flux, fsum);
            case RG_RIEMANN_HLL: return launch_pipe_rs<RG_RIEMANN_HLL>(c, P, K, variant, prim, flux, fsum);
            case RG_RIEMANN_EXACT: return launch_pipe_rs<RG_RIEMANN_EXACT>(c, P, K, variant, prim, flux, fsum);
            case RG_RIEMANN_ACOUSTIC: return launch_pipe_rs<RG_RIEMANN_ACOUSTIC>(c, P, K, variant, prim, flux, fsum);
            default: return launch_pipe_rs<RG_RIEMANN_LLF>(c, P, K, variant, prim, flux, fsum);
        }
    }
    return launch_face_nd<3>(c, P, K, variant, batch, uold, prim, flux, fsum);
}

}  // namespace rg
