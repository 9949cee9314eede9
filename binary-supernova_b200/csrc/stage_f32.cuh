// stage_f32.cuh -- the FP32-stencil physics policy of the fused stage kernel
// (the fast path): FP32 staging, WENO5-Z, pressures and HLLC; FP64 state,
// floors, divergence, sources, RK3 combine and CFL.  Included by the
// translation units built with the fast-path flags (stage_fast.cu, and
// learned.cu for the screening launch of the learned stage).
#pragma once

#include "physics_f32.cuh"
#include "stage_tile.cuh"

namespace bsn {
namespace tile {

struct F32Physics {
    using real = float;
    static constexpr bool kStiffFallback = false;
    static constexpr bool kCross = true;
    static constexpr int kCols = 5;                  // rho, m, P: the epilogue reloads the FP64 state
    static constexpr bool kCenterFromSmem = false;  // smem holds FP32 copies: reload FP64 state
    static constexpr bool kWarpFaces = false;
    static constexpr bool kQuiescentSkip = false;
    static constexpr bool kScreen = false;
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

// The FP32 policy with stiff faces in FP64: a face whose density stencil
// spans more than three decades is computed from the FP64 state by the FP64
// path's arithmetic (stage_tile.cuh face_flux_f64).  Launched where
// A.stiff_guard is set: the coupled driver loops with sinks (near-vacuum
// cells beside dense gas), or any loop on request.
struct F32Guarded : F32Physics {
    static constexpr bool kStiffFallback = true;
};

}  // namespace tile
}  // namespace bsn
