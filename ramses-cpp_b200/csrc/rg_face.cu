// rg_face.cu -- launch of the persistent tiled face kernel (rg_face.cuh) and
// its autotuner: every (variant, batch) pair is timed once per level plan on
// the level's own data and the fastest is kept.
#include <algorithm>

#include "rg_face.cuh"

namespace rg {

namespace {
constexpr int kBatches[] = {1, 4, 16};

int launch_variant(rg_ctx* c, const Plan& P, const StepK& K, int v, int b, const double* uold, const double* prim,
                   double* flux, double* fsum) {
    if (c->params.ndim == 1) return launch_face_nd1(c, P, K, v, b, uold, prim, flux, fsum);
    return launch_face_nd3(c, P, K, v, b, uold, prim, flux, fsum);
}
}  // namespace

int launch_face_tiles(rg_ctx* c, const Plan& P, const StepK& K, const double* uold, const double* prim,
                      double* flux, double* fsum) {
    if (P.ncells == 0) return RG_OK;
    int v = P.face_variant >= 0 ? P.face_variant : kDefaultFaceVariant;
    int b = P.face_batch > 0 ? P.face_batch : 1;
    return launch_variant(c, P, K, v, b, uold, prim, flux, fsum);
}

// Times every (variant, batch) on the level's current data (the face kernel
// only writes the flux scratch, so repeating it changes no state) and keeps
// the fastest.  Levels below 2^17 cells are not timed.  Must run outside a
// capture.
int autotune_face(rg_ctx* c, Plan& P, const StepK& K) {
    if (P.face_variant >= 0) return RG_OK;
    P.face_variant = kDefaultFaceVariant;
    P.face_batch = 1;
    // small levels are not timed (75 launches would cost more than any shape
    // can save, and AMR rebuilds its small levels whenever the tree changes).
    // A level whose tiles (one block each) outnumber the default shape's
    // resident blocks (8 per SM) takes the shape with the fewest resident
    // blocks per SM that still holds them all in one wave -- 9 (variant 3)
    // or 10 (variant 2), the fewer the more registers a thread keeps -- and
    // variant 2 beyond that (on the finest level of the Sedov AMR run, 1,272
    // tiles: face 0.373 instead of 0.409 ms per coarse step with variant 2)
    if (c->no_autotune) return RG_OK;
    if (P.ncells < (1 << 17)) {
        const int ntiles = (P.ncells + TILE - 1) / TILE;
        if (c->params.ndim == 3 && P.nbox == 0 && !P.lattice && ntiles > 8 * c->sm_count)
            P.face_variant = ntiles <= 9 * c->sm_count ? 3 : 2;
        return RG_OK;
    }
    const int ns = 2 * c->params.ndim, nv = c->params.ndim + 2;
    double* fsum = c->d_flux + (size_t)ns * nv * P.ncells;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int bv = kDefaultFaceVariant, bb = 1;
    for (int v = 0; v < kNumFaceVariants; ++v) {
        for (int b : kBatches) {
            if (v >= kFirstPipeVariant && b != 1) continue;  // round-robin tiles / bricks: no batch
            if (v >= kFirstBrickVariant && !(P.nbox > 0 ? P.box_lattice : P.lattice)) continue;
            if (v > kFirstBrickVariant && P.nbox > 0) continue;  // one boxed brick shape
            if (P.nbox > 0 && !boxed_variant_distinct(v)) continue;
            float tmin = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {
                cudaEventRecord(e0, c->stream);
                if (int rc = launch_variant(c, P, K, v, b, c->d_uold, c->d_prim, c->d_flux, fsum)) {
                    cudaEventDestroy(e0);
                    cudaEventDestroy(e1);
                    return rc;
                }
                cudaEventRecord(e1, c->stream);
                cudaEventSynchronize(e1);
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0) tmin = std::min(tmin, ms);  // the first launch warms caches and code
            }
            if (tmin < best) {
                best = tmin;
                bv = v;
                bb = b;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    P.face_variant = bv;
    P.face_batch = bb;
    P.face_ms = best;
    remember_shape(c, P);
    return check_cuda(c, cudaGetLastError(), "face autotune");
}

}  // namespace rg
