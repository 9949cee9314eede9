// autotune.cu -- picks the tile shape of the fused stage kernel per grid,
// and whether its block is staged by TMA copies or by the plain loader.
//
// On the first stage of a new (precision, driver class, nx, ny, nz) the
// autotuner launches
// every tile variant on stage-1 work (reading the caller's state, writing a
// scratch array), with each staging the grid allows, times two launches of
// each with CUDA events after one warm-up, and keeps the fastest for the life
// of the context.  Every variant and staging gives bit-identical results (FP64
// by the reference's arithmetic, FP32 by its written-out multiply-adds), so
// the choice never changes a result.  The choice is stored as a code: the
// variant index plus kTmaBit when the TMA form won.
#include "hydro_f64.cuh"
#include "stage_launch.cuh"

namespace bsn {

static int variant_count(int prec) {
    return prec == PREC_F64 ? f64_variant_count() : (prec == PREC_F32 ? f32_variant_count() : learned_variant_count());
}
static TileVariant variant(int prec, int idx) {
    return prec == PREC_F64 ? f64_variant(idx) : (prec == PREC_F32 ? f32_variant(idx) : learned_variant(idx));
}
constexpr int kTmaBit = 256;   // tile-choice code: variant index | kTmaBit when TMA staging is chosen

// One launch of variant `code & 255`, TMA-staged where the code asks for it
// (and the grid allows it); ctx->tma_used_last tells whether it was.
static bsn_status launch_variant(bsn_ctx* ctx, int prec, int code, const f64::StageArgs& A) {
    const int idx = code & (kTmaBit - 1);
    ctx->tma_now = (code & kTmaBit) ? 1 : 0;
    ctx->tma_used_last = 0;
    bsn_status st = prec == PREC_F64 ? f64_launch_variant(ctx, idx, A)
                    : prec == PREC_F32 ? f32_launch_variant(ctx, idx, A)
                                       : learned_launch_variant(ctx, idx, A);
    ctx->tma_now = 0;
    return st;
}
// the code of a forced variant: TMA wherever the context allows it
static int forced_code(bsn_ctx* ctx, int prec) {
    const int v = ctx->forced_tile[prec] >= 0 ? ctx->forced_tile[prec] : 0;
    return v | (ctx->tma_on ? kTmaBit : 0);
}
static bsn_status launch_batch_variant(bsn_ctx* ctx, int prec, int idx, const f64::StageBatch& B) {
    if (prec == PREC_F64) return f64_launch_batch_variant(ctx, idx, B);
    if (prec == PREC_F32) return f32_launch_batch_variant(ctx, idx, B);
    return learned_launch_batch_variant(ctx, idx, B);
}
static bool prec_ok(int p) { return p == PREC_F64 || p == PREC_F32 || p == PREC_LEARNED; }
// Drivers whose stages run in batched launches over several grids: the batch
// kernel has no TMA form, so their choices are timed with the plain loader only
// (a TMA variant timed alone can win and then run plain, and slower, in the batch).
static bool batched_class(int c) { return c == TUNE_FMR || c == TUNE_FMR_N || c == TUNE_NESTED; }
static std::tuple<int, int, int, int, int> tile_key(int prec, const f64::StageArgs& A) {
    return std::make_tuple(prec, A.tune_class, A.nx, A.ny, A.nz);
}
static void record(bsn_ctx* ctx, int prec, const f64::StageArgs& A, int code) {
    ctx->tile_choice[tile_key(prec, A)] = code;
    ctx->tile_last[std::make_tuple(prec, A.nx, A.ny, A.nz)] = code;
}

int tile_code(bsn_ctx* ctx, int prec, const f64::StageArgs& A) {
    auto it = ctx->tile_choice.find(tile_key(prec, A));
    return it == ctx->tile_choice.end() ? -1 : it->second;
}

bsn_status stage_autotune(bsn_ctx* ctx, int prec, const f64::StageArgs& probe, double* scratch) {
    if (prec == PREC_LEARNED) {   // the split learned stage's block list, allocated before any capture
        bsn_status st;
        slot(ctx, SLOT_SPLIT, learned_split_bytes(probe.nx, probe.ny, probe.nz), &st);
        BSN_TRY(st);
    }
    const auto key = tile_key(prec, probe);
    if (ctx->tile_choice.count(key) && (probe.tune_class != ctx->retime_class || ctx->retimed.count(key)))
        return BSN_OK;
    if (probe.tune_class == ctx->retime_class) ctx->retimed.insert(key);
    int nv = variant_count(prec);
    if (ctx->forced_tile[prec] >= 0) {
        record(ctx, prec, probe, forced_code(ctx, prec));
        return BSN_OK;
    }
    f64::StageArgs a = probe;
    a.Un = probe.Uin;
    a.Uout = scratch;
    a.mode = 0;
    a.stage = 1;
    a.dt = 0.0;
    a.cfl_max = nullptr;
    a.cfl_nan = nullptr;
    a.use_reg = 0;
    a.use_bnd = 0;
    a.F[0] = a.F[1] = a.F[2] = nullptr;
    a.dt_dev = nullptr;
    a.done_dev = nullptr;
    a.ledger = nullptr;
    cudaEvent_t e0, e1;
    BSN_CUDA(ctx, cudaEventCreate(&e0));
    BSN_CUDA(ctx, cudaEventCreate(&e1));
    int best = 0;
    float best_ms = 1e30f;
    bool prof = ctx->profiling;
    ctx->profiling = false;
    bsn_status st = BSN_OK;
    for (int v = 0; v < nv && st == BSN_OK; ++v) {
        for (int tma = 0; tma < (ctx->tma_on && !batched_class(probe.tune_class) ? 2 : 1) && st == BSN_OK; ++tma) {
            const int code = v | (tma ? kTmaBit : 0);
            st = launch_variant(ctx, prec, code, a);   // warm-up (sets smem attributes)
            if (st != BSN_OK) break;
            if (tma && !ctx->tma_used_last) break;      // the grid does not allow TMA staging of this tile
            float ms = 1e30f;
            for (int r = 0; r < 2 && st == BSN_OK; ++r) {
                cudaEventRecord(e0, ctx->stream);
                st = launch_variant(ctx, prec, code, a);
                cudaEventRecord(e1, ctx->stream);
                st = st != BSN_OK ? st : cuda_check(ctx, cudaEventSynchronize(e1), "cudaEventSynchronize(autotune)");
                float t = 0.f;
                cudaEventElapsedTime(&t, e0, e1);
                ms = t < ms ? t : ms;
            }
            if (ms < best_ms) { best_ms = ms; best = code; }
        }
    }
    ctx->profiling = prof;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    BSN_TRY(st);
    record(ctx, prec, probe, best);
    return BSN_OK;
}

bool tile_settled(bsn_ctx* ctx, int tune_class, int prec) {
    return ctx->forced_tile[prec] >= 0 || ctx->settled.count(std::make_pair(tune_class, prec)) > 0;
}

bsn_status tile_retime(bsn_ctx* ctx, int tune_class, int prec, const std::function<bsn_status()>& tune) {
    ctx->retime_class = tune_class;
    ctx->retimed.clear();
    bsn_status st = tune();
    ctx->retime_class = -1;
    ctx->retimed.clear();
    if (st == BSN_OK) ctx->settled.insert(std::make_pair(tune_class, prec));
    return st;
}

bsn_status stage_launch(bsn_ctx* ctx, int prec, const f64::StageArgs& A) {
    auto it = ctx->tile_choice.find(tile_key(prec, A));
    if (it == ctx->tile_choice.end()) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(ctx->stream, &cs);
        if (ctx->forced_tile[prec] >= 0 || cs != cudaStreamCaptureStatusNone)
            return launch_variant(ctx, prec, forced_code(ctx, prec), A);
        Geom G(A.nx, A.ny, A.nz);
        bsn_status st;
        double* scratch = (double*)slot(ctx, SLOT_UN, sizeof(double) * (size_t)G.nelem(), &st);
        BSN_TRY(st);
        BSN_TRY(stage_autotune(ctx, prec, A, scratch));
        it = ctx->tile_choice.find(tile_key(prec, A));
    }
    return launch_variant(ctx, prec, it->second, A);
}

// The variant of a batch is the one chosen for its last level's grid (for
// two-level FMR the fine level, the larger share of the work per step).
static bsn_status choose(bsn_ctx* ctx, int prec, const f64::StageArgs& A, int& v) {
    auto it = ctx->tile_choice.find(tile_key(prec, A));
    if (it != ctx->tile_choice.end()) { v = it->second & (kTmaBit - 1); return BSN_OK; }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(ctx->stream, &cs);
    if (ctx->forced_tile[prec] >= 0 || cs != cudaStreamCaptureStatusNone) {
        v = ctx->forced_tile[prec] >= 0 ? ctx->forced_tile[prec] : 0;
        return BSN_OK;
    }
    Geom G(A.nx, A.ny, A.nz);
    bsn_status st;
    double* scratch = (double*)slot(ctx, SLOT_UN, sizeof(double) * (size_t)G.nelem(), &st);
    BSN_TRY(st);
    BSN_TRY(stage_autotune(ctx, prec, A, scratch));
    v = ctx->tile_choice[tile_key(prec, A)] & (kTmaBit - 1);   // several grids in one launch: the plain loader
    return BSN_OK;
}

bsn_status stage_launch_batch(bsn_ctx* ctx, int prec, const f64::StageBatch& B) {
    if (B.nlev < 1 || B.nlev > f64::MAXLEV) return set_err(ctx, BSN_ERR_ARG, "batch of %d levels", B.nlev);
    int v = 0;
    BSN_TRY(choose(ctx, prec, B.lv[B.nlev - 1], v));
    return launch_batch_variant(ctx, prec, v, B);
}

}  // namespace bsn

using namespace bsn;

extern "C" bsn_status bsn_ctx_set_tile(bsn_ctx* ctx, int precision, int variant) {
    if (!ctx) return BSN_ERR_ARG;
    if (!prec_ok(precision)) return set_err(ctx, BSN_ERR_ARG, "bad precision %d", precision);
    if (variant >= variant_count(precision)) return set_err(ctx, BSN_ERR_ARG, "no tile variant %d", variant);
    ctx->forced_tile[precision] = variant < 0 ? -1 : variant;
    for (auto it = ctx->tile_choice.begin(); it != ctx->tile_choice.end();)
        it = std::get<0>(it->first) == precision ? ctx->tile_choice.erase(it) : std::next(it);
    for (auto it = ctx->tile_last.begin(); it != ctx->tile_last.end();)
        it = std::get<0>(it->first) == precision ? ctx->tile_last.erase(it) : std::next(it);
    for (auto it = ctx->settled.begin(); it != ctx->settled.end();)
        it = it->second == precision ? ctx->settled.erase(it) : std::next(it);
    return BSN_OK;
}

extern "C" bsn_status bsn_ctx_get_tile(bsn_ctx* ctx, int precision, int nx, int ny, int nz, int out[5]) {
    if (!ctx || !out) return BSN_ERR_ARG;
    auto it = ctx->tile_last.find(std::make_tuple(precision, nx, ny, nz));
    if (it == ctx->tile_last.end()) return set_err(ctx, BSN_ERR_ARG, "no tile chosen yet for this grid");
    if (!prec_ok(precision)) return set_err(ctx, BSN_ERR_ARG, "bad precision %d", precision);
    TileVariant v = variant(precision, it->second & (kTmaBit - 1));
    out[0] = v.tx; out[1] = v.ty; out[2] = v.tz; out[3] = v.nt; out[4] = v.minb;
    return BSN_OK;
}

extern "C" int bsn_ctx_get_tile_tma(bsn_ctx* ctx, int precision, int nx, int ny, int nz) {
    if (!ctx) return -1;
    auto it = ctx->tile_last.find(std::make_tuple(precision, nx, ny, nz));
    if (it == ctx->tile_last.end()) return -1;
    return (it->second & kTmaBit) ? 1 : 0;
}

extern "C" int bsn_tile_variant_count(int precision) {
    return prec_ok(precision) ? variant_count(precision) : 0;
}
