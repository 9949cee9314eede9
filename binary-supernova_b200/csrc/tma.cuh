// tma.cuh -- TMA (cp.async.bulk.tensor) staging of the fused stage kernel's
// cross region.
//
// The state array U[q,i,j,k] (FP64, q fastest) is described to the tensor
// memory accelerator as a 3-D tensor of doubles: x = 5 i + q (the whole
// ghosted row of cells, 5 NXT doubles), y = j, z = k, with the reference
// layout's strides (40 NXT and 40 NXT NYT bytes, multiples of 16 when nx is
// even).  Three box shapes cover a TX x TY x TZ block's cross region:
//
//   A  the block with its x halos: cells a0-3 .. a0+TX+2 (5 (TX+6) doubles),
//      AY rows x AZ planes per copy;
//   Y  a y halo: cells a0-1 .. a0+TX (5 (TX+2) doubles, the row start
//      rounded down to an even cell so every copy starts on a 16-byte
//      boundary: a0 is even), 3 rows, YZ planes per copy;
//   Z  a z halo: the same cells, ZY rows, 3 planes per copy.
//
// Every box lies inside the ghosted array (x from ghosted cell a0 to at
// most a0+TX+5 <= nx+5), so no copy reads out of bounds.  The copies land in
// two raw buffers of at most CAP bytes (kChunkCap, or less where the face
// buffer must hold both); each buffer has an mbarrier,
// and the block's cells are converted from one buffer (floors, pressure,
// precision of the policy) while the copy into the other is in flight.  Halo
// cells outside the active domain are not taken from the copy: they come
// through the boundary map (or ghost buffer) as in the plain loader.
//
// No copy here uses .multicast::cluster; every tensor map describes this
// GPU's own buffer.
#pragma once

#include <cuda.h>
#include <cstdint>

#include "stage_f64.cuh"

namespace bsn {
namespace tma {

constexpr int kChunkCap = 18432;   // bytes of one staged copy where the smem budget allows

// Box shapes and copy counts of a tile for copies of at most CAP bytes,
// fixed at compile time.
template <int TX, int TY, int TZ, int CAP>
struct Chunks {
    static constexpr int RA = 5 * (TX + 6), RH = 5 * (TX + 2);   // doubles per row of A / of Y and Z
    static constexpr int best_div(int n, int per) {
        int b = 1;
        for (int d = 1; d <= n; ++d)
            if (n % d == 0 && d * per <= CAP) b = d;
        return b;
    }
    // A: whole planes when one fits, else AY rows of one plane
    static constexpr int AY = RA * TY * 8 <= CAP ? TY : best_div(TY, RA * 8);
    static constexpr int AZ = AY == TY ? best_div(TZ, RA * TY * 8) : 1;
    static constexpr int YZ = best_div(TZ, RH * 3 * 8);      // planes per Y copy
    static constexpr int ZY = best_div(TY, RH * 3 * 8);      // rows per Z copy
    static constexpr int NAY = TY / AY;                      // A copies per plane group
    static constexpr int NA = (TZ / AZ) * NAY, NY = 2 * (TZ / YZ), NZ = 2 * (TY / ZY);
    static constexpr int N = NA + NY + NZ;                    // copies per block
    static constexpr int BA = RA * AY * AZ * 8, BY = RH * 3 * YZ * 8, BZ = RH * ZY * 3 * 8;
    static constexpr int RAWB = ((BA > BY ? (BA > BZ ? BA : BZ) : (BY > BZ ? BY : BZ)) + 127) / 128 * 128;
    static_assert(TX % 2 == 0, "TMA staging needs an even tile width (16-byte aligned row starts)");
    static_assert(BA <= CAP && BY <= CAP && BZ <= CAP, "a copy exceeds the raw buffer");
    static_assert(RA <= 256 && RH <= 256 && TY <= 256, "TMA box dimensions are limited to 256");
};

// Tensor maps of one stage input (the three box shapes) and the flag a
// bounded wait sets when a copy does not arrive.  Passed to the kernel as a
// __grid_constant__ parameter.
struct alignas(64) Maps {
    CUtensorMap a, y, z;
    unsigned int* err;       // device word: bit 0 set by a timed-out wait
};

// Host (tma_host.cu): the three tensor maps of A.Uin for a TX x TY x TZ tile
// with the given copy extents (A boxes of AY rows x AZ planes), when the grid
// qualifies -- TMA staging on for the context, no ghost buffer, the tile
// dividing the grid, nx even (row strides multiples of 16 bytes), Uin
// 16-byte aligned -- else false.
bool build_maps(bsn_ctx* ctx, const f64::StageArgs& A, int TX, int TY, int TZ, int AY, int AZ, int YZ, int ZY,
                Maps& M);

#ifdef __CUDACC__
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// make initialised barriers visible to the async proxy (the copy engine)
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// order this CTA's generic-proxy accesses of shared memory before later
// async-proxy writes (a raw buffer refilled by a copy after threads read it)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity to complete, at most `limit`
// polls (each try_wait suspends for a bounded, implementation-defined time).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, unsigned limit = 1u << 24) {
    for (unsigned i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// One 3-D tile copy global -> shared, completing on `bar` (bytes counted by
// the barrier's transaction count).  Coordinates in elements; x * 8 bytes is
// a multiple of 16 by construction of the boxes.
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
#endif

}  // namespace tma
}  // namespace bsn
