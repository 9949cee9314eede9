// stage_launch.cuh -- tile variants of the fused stage kernel, the autotuner
// that picks one per grid, and the launch dispatch (autotune.cu).
#pragma once

#include <functional>

#include "stage_f64.cuh"

namespace bsn {

enum Precision { PREC_F64 = 0, PREC_F32 = 1, PREC_LEARNED = 2 };

struct TileVariant {
    int tx, ty, tz, nt, minb;   // block tile, threads per CTA, min CTAs per SM (register cap)
};

// Bytes of the split learned stage's block list (count + one index per
// block) for the tile variant with the most blocks on an nx x ny x nz grid.
size_t learned_split_bytes(int nx, int ny, int nz);

// per-precision variant tables (hydro_f64.cu: FP64, stage_fast.cu: FP32)
int f64_variant_count();
TileVariant f64_variant(int idx);
bsn_status f64_launch_variant(bsn_ctx* ctx, int idx, const f64::StageArgs& A);
int f32_variant_count();
TileVariant f32_variant(int idx);
bsn_status f32_launch_variant(bsn_ctx* ctx, int idx, const f64::StageArgs& A);
int learned_variant_count();
TileVariant learned_variant(int idx);
bsn_status learned_launch_variant(bsn_ctx* ctx, int idx, const f64::StageArgs& A);
// batched (several grids in one persistent launch) counterparts
bsn_status f64_launch_batch_variant(bsn_ctx* ctx, int idx, const f64::StageBatch& B);
bsn_status f32_launch_batch_variant(bsn_ctx* ctx, int idx, const f64::StageBatch& B);
bsn_status learned_launch_batch_variant(bsn_ctx* ctx, int idx, const f64::StageBatch& B);

// Driver classes of StageArgs::tune_class: each keeps its own tile choices.
enum TuneClass {
    TUNE_GENERIC = 0,    // single stages and steps through the C ABI
    TUNE_RUN = 1,        // uniform-grid device time loop (run_steps.cu)
    TUNE_COUPLED = 2,    // uniform coupled driver loop (coupled_run.cu)
    TUNE_NESTED = 3,     // nested-level coupled driver loop (coupled_run.cu)
    TUNE_FMR = 4,        // two-level FMR loop (fmr_f64.cu)
    TUNE_FMR_N = 5,      // N-level FMR loop (fmr_nlevel.cu)
    TUNE_RELAX = 6,      // relaxation loop (relax.cu)
};
// The tile-choice code recorded for A's driver class and grid (-1: none yet).
int tile_code(bsn_ctx* ctx, int precision, const f64::StageArgs& A);

// Launch one stage with the tile chosen for (precision, A.tune_class, nx, ny,
// nz); the first call for a grid runs the autotuner unless a tile was forced.
bsn_status stage_launch(bsn_ctx* ctx, int precision, const f64::StageArgs& A);
// One stage on all levels of B in one launch, with the tile variant chosen
// for the last level's grid (autotuned on first use unless forced).
bsn_status stage_launch_batch(bsn_ctx* ctx, int precision, const f64::StageBatch& B);
// Autotune explicitly (must not run during stream capture): times every
// variant on stage-1 work writing to `scratch` and records the fastest.
bsn_status stage_autotune(bsn_ctx* ctx, int precision, const f64::StageArgs& probe, double* scratch);

// Device loops tune on the state they are first called with.  From an
// initial condition (gas at rest) every tile variant can time within a
// percent of the others while one of them is 20 % faster on the flow the loop
// then evolves, so a loop whose (driver class, precision) is not settled yet
// replays its first step alone and then calls tile_retime: `tune` runs the
// loop's own probes again, each grid of that class is re-timed once on the
// state the step reached, and the pair is marked settled.  Every variant gives
// the same results, so the split changes no result.
bool tile_settled(bsn_ctx* ctx, int tune_class, int precision);
bsn_status tile_retime(bsn_ctx* ctx, int tune_class, int precision, const std::function<bsn_status()>& tune);

}  // namespace bsn
