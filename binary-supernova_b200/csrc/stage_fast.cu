// stage_fast.cu -- FP32-stencil variants of the fused stage kernel (the fast
// path): FP32 staging, WENO5-Z, pressures and HLLC with FMA and approximate
// reciprocals/square roots; FP64 state, floors, divergence, sources, RK3
// combine and CFL.  Built with --ftz=true --prec-div=false --prec-sqrt=false.
#include "hydro_f64.cuh"
#include "physics_f32.cuh"
#include "stage_f32.cuh"
#include "stage_launch.cuh"
#include "stage_tile.cuh"

namespace bsn {

namespace {
const TileVariant kF32Variants[] = {{8, 8, 8, 256, 3}, {16, 8, 4, 256, 3}, {8, 8, 4, 128, 6}, {16, 8, 8, 256, 2},
                                     {16, 16, 4, 256, 2}, {16, 16, 8, 512, 1}};

template <class P, int TX, int TY, int TZ, int NT, int MINB>
bsn_status launch_f32_policy(bsn_ctx* ctx, const f64::StageArgs& A) {
    static_assert(tile::smem_bytes<P, TX, TY, TZ>() <= 200 * 1024, "tile's shared memory exceeds the per-CTA limit");
    bool tma_used = false;
    BSN_TRY((tile::launch_tma<P, TX, TY, TZ, NT, MINB>(ctx, A, "stage_kernel_f32_tma", &tma_used)));
    if (tma_used) return BSN_OK;
    return tile::launch_plain<P, TX, TY, TZ, NT, MINB>(ctx, A, tile::smem_bytes<P, TX, TY, TZ>(), "stage_kernel_f32");
}
template <int TX, int TY, int TZ, int NT, int MINB>
bsn_status launch_f32(bsn_ctx* ctx, const f64::StageArgs& A) {
    return A.stiff_guard ? launch_f32_policy<tile::F32Guarded, TX, TY, TZ, NT, MINB>(ctx, A)
                         : launch_f32_policy<tile::F32Physics, TX, TY, TZ, NT, MINB>(ctx, A);
}
template <class P>
bsn_status launch_f32_batch(bsn_ctx* ctx, int idx, const f64::StageBatch& B) {
    const char* nm = "stage_kernel_batch_f32";
    switch (idx) {
        case 0: return tile::launch_batch<P, 8, 8, 8, 256, 3>(ctx, B, tile::smem_bytes<P, 8, 8, 8>(), nm);
        case 1: return tile::launch_batch<P, 16, 8, 4, 256, 3>(ctx, B, tile::smem_bytes<P, 16, 8, 4>(), nm);
        case 2: return tile::launch_batch<P, 8, 8, 4, 128, 6>(ctx, B, tile::smem_bytes<P, 8, 8, 4>(), nm);
        case 3: return tile::launch_batch<P, 16, 8, 8, 256, 2>(ctx, B, tile::smem_bytes<P, 16, 8, 8>(), nm);
        case 4: return tile::launch_batch<P, 16, 16, 4, 256, 2>(ctx, B, tile::smem_bytes<P, 16, 16, 4>(), nm);
        case 5: return tile::launch_batch<P, 16, 16, 8, 512, 1>(ctx, B, tile::smem_bytes<P, 16, 16, 8>(), nm);
        default: return set_err(ctx, BSN_ERR_ARG, "no FP32 tile variant %d", idx);
    }
}
}  // namespace

int f32_variant_count() { return (int)(sizeof(kF32Variants) / sizeof(kF32Variants[0])); }
TileVariant f32_variant(int idx) { return kF32Variants[idx]; }
bsn_status f32_launch_variant(bsn_ctx* ctx, int idx, const f64::StageArgs& A) {
    switch (idx) {
        case 0: return launch_f32<8, 8, 8, 256, 3>(ctx, A);
        case 1: return launch_f32<16, 8, 4, 256, 3>(ctx, A);
        case 2: return launch_f32<8, 8, 4, 128, 6>(ctx, A);
        case 3: return launch_f32<16, 8, 8, 256, 2>(ctx, A);
        case 4: return launch_f32<16, 16, 4, 256, 2>(ctx, A);
        case 5: return launch_f32<16, 16, 8, 512, 1>(ctx, A);   // one CTA of 512 threads: a smaller halo share
        default: return set_err(ctx, BSN_ERR_ARG, "no FP32 tile variant %d", idx);
    }
}

bsn_status f32_launch_batch_variant(bsn_ctx* ctx, int idx, const f64::StageBatch& B) {
    bool guard = false;
    for (int l = 0; l < B.nlev && l < f64::MAXLEV; ++l) guard = guard || B.lv[l].stiff_guard;
    return guard ? launch_f32_batch<tile::F32Guarded>(ctx, idx, B) : launch_f32_batch<tile::F32Physics>(ctx, idx, B);
}

}  // namespace bsn
