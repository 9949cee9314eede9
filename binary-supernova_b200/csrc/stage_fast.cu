// stage_fast.cu -- FP32-stencil variants of the fused stage kernel (the fast
// path): FP32 staging, WENO5-Z, pressures and HLLC with FMA and approximate
// reciprocals/square roots; FP64 state, floors, divergence, sources, RK3
// combine and CFL.  Built with --ftz=true --prec-div=false --prec-sqrt=false.
#include "hydro_f64.cuh"
#include "physics_f32.cuh"
#include "stage_launch.cuh"
#include "stage_tile.cuh"

namespace bsn {
namespace tile {
struct F32Physics {
    using real = float;
    static constexpr bool kCross = true;
    static constexpr int kCols = 5;                  // rho, m, P: the epilogue reloads the FP64 state
    static constexpr bool kCenterFromSmem = false;  // smem holds FP32 copies: reload FP64 state
    static constexpr bool kWarpFaces = false;
    static constexpr bool kQuiescentSkip = false;
    __device__ static bool same(float, float) { return true; }
    static constexpr int kExtraSmem(int) { return 0; }
    __device__ static void prologue(unsigned char*, const f64::StageArgs&, int) {}
    struct Consts { float g, gm1, inv_gm1, gg; };
    __device__ static Consts consts(const f64::StageArgs& A) {
        float g = (float)A.g;
        return {g, (float)A.gm1, 1.0f / (float)A.gm1, (g + 1.0f) / (2.0f * g)};
    }
    __device__ static float pressure(const float v[5], const Consts& k) {
        return f32::cell_pressure(v[0], v[1], v[2], v[3], v[4], k.gm1);
    }
    __device__ static void floor(double (&v)[5], const f64::StageArgs& A) {
        f32::floor_screened(v, A.rho_floor, A.P_floor, A.Pfl_gm1, A.gm1);
    }
    __device__ static void stage(double (&v)[5], bool act, const f64::StageArgs& A, float (&w)[5]) {
        f32::stage_floored(v, act, A.rho_floor, A.P_floor, A.Pfl_gm1, A.gm1, w);
    }
    template <int D>
    __device__ static void flux(const float (&c)[6][6], const Consts& k, float F[5]) {
        f32::interface_flux<D>(c, k.g, k.gm1, k.inv_gm1, k.gg, F);
    }
};

}  // namespace tile

namespace {
const TileVariant kF32Variants[] = {{8, 8, 8, 256, 3}, {16, 8, 4, 256, 3}, {8, 8, 4, 128, 6}, {16, 8, 8, 256, 2},
                                     {16, 16, 4, 256, 2}};

template <int TX, int TY, int TZ, int NT, int MINB>
bsn_status launch_f32(bsn_ctx* ctx, const f64::StageArgs& A) {
    auto fn = tile::stage_kernel<tile::F32Physics, TX, TY, TZ, NT, MINB>;
    constexpr int smem = tile::smem_bytes<tile::F32Physics, TX, TY, TZ>();
    static bool attr_done[64] = {false};
    int dev = ctx->device & 63;
    if (!attr_done[dev]) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return cuda_check(ctx, e, "cudaFuncSetAttribute(stage_kernel_f32)");
        attr_done[dev] = true;
    }
    dim3 grid((A.nx + TX - 1) / TX, (A.ny + TY - 1) / TY, (A.nz + TZ - 1) / TZ);
    prof_begin(ctx);
    fn<<<grid, NT, smem, ctx->stream>>>(A);
    return launch_check(ctx, "stage_kernel_f32");
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
        default: return set_err(ctx, BSN_ERR_ARG, "no FP32 tile variant %d", idx);
    }
}

bsn_status f32_launch_batch_variant(bsn_ctx* ctx, int idx, const f64::StageBatch& B) {
    using P = tile::F32Physics;
    const char* nm = "stage_kernel_batch_f32";
    switch (idx) {
        case 0: return tile::launch_batch<P, 8, 8, 8, 256, 3>(ctx, B, tile::smem_bytes<P, 8, 8, 8>(), nm);
        case 1: return tile::launch_batch<P, 16, 8, 4, 256, 3>(ctx, B, tile::smem_bytes<P, 16, 8, 4>(), nm);
        case 2: return tile::launch_batch<P, 8, 8, 4, 128, 6>(ctx, B, tile::smem_bytes<P, 8, 8, 4>(), nm);
        case 3: return tile::launch_batch<P, 16, 8, 8, 256, 2>(ctx, B, tile::smem_bytes<P, 16, 8, 8>(), nm);
        case 4: return tile::launch_batch<P, 16, 16, 4, 256, 2>(ctx, B, tile::smem_bytes<P, 16, 16, 4>(), nm);
        default: return set_err(ctx, BSN_ERR_ARG, "no FP32 tile variant %d", idx);
    }
}

}  // namespace bsn
