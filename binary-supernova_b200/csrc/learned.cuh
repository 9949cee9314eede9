// learned.cuh -- the learned WENO-weight network shared by the sample
// collector, the training kernels and the stencil-kernel inference.
//
// Two MLPs (one for the left-biased, one for the right-biased reconstruction
// of src/weno5.jl:25-61), each 5 -> 32 -> 32 -> 3 with ReLU and a softmax
// output, map a normalised 5-point stencil
//     u_i = (v_i - v_c) / max_j |v_j - v_c|,   v_c = the stencil's centre cell,
// to the three nonlinear weights (omega_0, omega_1, omega_2).  WENO-Z weights
// are invariant to v -> a v + b (up to its 1e-36 epsilon), so the normalised
// stencil carries all the information they depend on.
//
// Fallback: a reconstruction uses the network only where the WENO-Z
// smoothness indicators of the normalised stencil say the data is smooth,
//     tau5 <= THETA * (min_k beta_k + BETA_EPS),
// and the stencil's spread is above rounding level (SPREAD_*); elsewhere
// (discontinuities, strong extrema, quiescent gas) it uses plain WENO5-Z.
#pragma once

#include <cstdint>

namespace bsn {
namespace learned {

constexpr int NIN = 5, NH = 32, NOUT = 3;
// parameter layout of one network (FP32): W1[NH][NIN], b1[NH], W2[NH][NH], b2[NH], W3[NOUT][NH], b3[NOUT]
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NH * NIN, OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + NH * NH,
              OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + NOUT * NH, NPARAM = OFF_B3 + NOUT;
constexpr float THETA = 4.0f, BETA_EPS = 1e-3f;
// Minimum stencil spread max|v_i - v_c| for the network: below it the
// weights cannot change the reconstruction beyond rounding.  Training
// samples (FP64) need spread > SPREAD_ABS and > SPREAD_REL_F64 |v_c|; the
// FP32 stencil kernel uses SPREAD_REL_F32 (FP32 rounding level).
constexpr float SPREAD_ABS = 1e-15f;
constexpr double SPREAD_REL_F64 = 1e-12;
constexpr float SPREAD_REL_F32 = 1e-6f;
constexpr int SAMPLE = 8;   // floats per training sample: u[5], target omega[3]

// Normalised stencil and the fallback flag.  side 0: left-biased stencil
// (v0..v4 = cells i-2..i+2, centre v2); side 1: right-biased (v0..v4 = cells
// i-1..i+3, centre v1).  Smoothness indicators follow the reference formulas
// of that side.  Returns true where the network may be used.
template <typename T>
__host__ __device__ inline bool normalise(const T v[5], int side, T u[5]) {
    T c = side == 0 ? v[2] : v[1];
    T s = T(0);
    for (int i = 0; i < 5; ++i) {
        T d = v[i] - c;
        d = d < T(0) ? -d : d;
        s = d > s ? d : s;
    }
    T inv = s > T(0) ? T(1) / s : T(0);
    for (int i = 0; i < 5; ++i) u[i] = (v[i] - c) * inv;
    T b0, b1, b2;
    const T k = T(13) / T(12), q = T(0.25);
    if (side == 0) {
        b0 = k * (u[0] - 2 * u[1] + u[2]) * (u[0] - 2 * u[1] + u[2]) + q * (u[0] - 4 * u[1] + 3 * u[2]) * (u[0] - 4 * u[1] + 3 * u[2]);
        b1 = k * (u[1] - 2 * u[2] + u[3]) * (u[1] - 2 * u[2] + u[3]) + q * (u[1] - u[3]) * (u[1] - u[3]);
        b2 = k * (u[2] - 2 * u[3] + u[4]) * (u[2] - 2 * u[3] + u[4]) + q * (3 * u[2] - 4 * u[3] + u[4]) * (3 * u[2] - 4 * u[3] + u[4]);
    } else {
        b0 = k * (u[0] - 2 * u[1] + u[2]) * (u[0] - 2 * u[1] + u[2]) + q * (u[0] - u[2]) * (u[0] - u[2]);
        b1 = k * (u[1] - 2 * u[2] + u[3]) * (u[1] - 2 * u[2] + u[3]) + q * (u[1] - 4 * u[2] + 3 * u[3]) * (u[1] - 4 * u[2] + 3 * u[3]);
        b2 = k * (u[2] - 2 * u[3] + u[4]) * (u[2] - 2 * u[3] + u[4]) + q * (3 * u[2] - 4 * u[3] + u[4]) * (3 * u[2] - 4 * u[3] + u[4]);
    }
    T tau = b0 - b2;
    tau = tau < T(0) ? -tau : tau;
    T bmin = b0 < b1 ? b0 : b1;
    bmin = bmin < b2 ? bmin : b2;
    return tau <= T(THETA) * (bmin + T(BETA_EPS));
}

}  // namespace learned
}  // namespace bsn
