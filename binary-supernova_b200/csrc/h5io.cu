// h5io.cu -- checkpoints, snapshots and BH trajectories in the reference's
// HDF5 layouts (src/checkpoint.jl, src/io.jl) through the writer and reader
// of h5file.h, with the state copied from the device; the uniform
// checkpoint's asynchronous form snapshots the state on the context's stream
// and copies and writes it while the stream runs on.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "bsn_internal.cuh"
#include "h5file.h"

namespace bsn {

namespace {

constexpr int64_t FORMAT_VERSION = 1;   // CHECKPOINT_FORMAT_VERSION (src/checkpoint.jl:30)

long long state_elems(int nx, int ny, int nz) { return 5LL * (nx + 2 * BSN_NG) * (ny + 2 * BSN_NG) * (nz + 2 * BSN_NG); }
std::vector<uint64_t> state_dims(int nx, int ny, int nz) {   // HDF5 order of the Julia (NQ, nx+2NG, ny+2NG, nz+2NG)
    return {(uint64_t)nz + 2 * BSN_NG, (uint64_t)ny + 2 * BSN_NG, (uint64_t)nx + 2 * BSN_NG, 5};
}

bsn_status io_err(bsn_ctx* ctx, const std::string& what) {
    if (ctx) return set_err(ctx, BSN_ERR_IO, "%s", what.c_str());
    return BSN_ERR_IO;
}

// host copy of a state array (device or host source)
bsn_status fetch(bsn_ctx* ctx, const double* U, int on_device, long long n, std::vector<double>& out,
                 const double** host) {
    if (!on_device) { *host = U; return BSN_OK; }
    if (!ctx) return BSN_ERR_ARG;
    out.resize((size_t)n);
    BSN_CUDA(ctx, cudaMemcpyAsync(out.data(), U, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *host = out.data();
    return BSN_OK;
}

// the BH group (src/checkpoint.jl:205-222): n, and pos/vel (3, n), mass ... (n)
struct BHArrays { std::vector<double> pos, vel, mass, eps, c_code, r_floor; };
h5::Group bh_group(const bsn_bh* bhs, int nbh, BHArrays& A) {
    h5::Group b;
    b.name = "bhs";
    b.attrs.push_back(h5::attr_i64("n", nbh));
    if (nbh <= 0) return b;
    for (int i = 0; i < nbh; ++i) {
        for (int d = 0; d < 3; ++d) { A.pos.push_back(bhs[i].pos[d]); A.vel.push_back(bhs[i].vel[d]); }
        A.mass.push_back(bhs[i].mass); A.eps.push_back(bhs[i].eps);
        A.c_code.push_back(bhs[i].c_code); A.r_floor.push_back(bhs[i].r_floor);
    }
    auto ds = [&](const char* name, const std::vector<double>& v, std::vector<uint64_t> dims) {
        h5::Dataset d;
        d.name = name; d.kind = h5::F64; d.dims = dims; d.data = v.data();
        b.dsets.push_back(d);
    };
    ds("pos", A.pos, {(uint64_t)nbh, 3});
    ds("vel", A.vel, {(uint64_t)nbh, 3});
    ds("mass", A.mass, {(uint64_t)nbh});
    ds("eps", A.eps, {(uint64_t)nbh});
    ds("c_code", A.c_code, {(uint64_t)nbh});
    ds("r_floor", A.r_floor, {(uint64_t)nbh});
    return b;
}

bool read_bhs(const h5::Reader& R, bsn_bh* bhs, int cap, int* nbh, std::string* err) {
    const h5::RGroup* b = R.group("bhs");
    int64_t n = 0;
    if (!b || !h5::get_i64(b->attrs, "n", &n) || n < 0) { *err = "no /bhs group with its count n"; return false; }
    *nbh = (int)n;
    if (!bhs || n == 0) return true;
    if (n > cap) { *err = "more BHs in the file than room for them"; return false; }
    std::vector<double> pos(3 * n), vel(3 * n), mass(n), eps(n), cc(n), rf(n);
    struct { const char* name; std::vector<double>* v; } f[] = {{"pos", &pos}, {"vel", &vel}, {"mass", &mass},
                                                                {"eps", &eps}, {"c_code", &cc}, {"r_floor", &rf}};
    for (auto& x : f) {
        auto it = b->dsets.find(x.name);
        if (it == b->dsets.end() || it->second.kind != h5::F64 || it->second.count() != x.v->size()) {
            *err = std::string("bad /bhs/") + x.name;
            return false;
        }
        if (!R.read_data(it->second, x.v->data(), 8 * x.v->size(), err)) return false;
    }
    for (int i = 0; i < n; ++i) {
        for (int d = 0; d < 3; ++d) { bhs[i].pos[d] = pos[3 * i + d]; bhs[i].vel[d] = vel[3 * i + d]; }
        bhs[i].mass = mass[i]; bhs[i].eps = eps[i]; bhs[i].c_code = cc[i]; bhs[i].r_floor = rf[i];
    }
    return true;
}

// the uniform checkpoint's tree over a host state (src/checkpoint.jl:222-265)
bool write_uniform(const std::string& path, const double* U, const bsn_bh* bhs, int nbh, const bsn_grid_meta& g,
                   const bsn_ckpt_meta& m, std::string* err) {
    h5::Group root;
    h5::Group man;
    man.name = "manifest";
    man.attrs = {h5::attr_i64("format_version", FORMAT_VERSION), h5::attr_str("kind", "uniform"),
                 h5::attr_f64("t", m.t), h5::attr_i64("step", m.step), h5::attr_f64("dt_last", m.dt_last),
                 h5::attr_f64("t_snap", m.t_snap), h5::attr_f64("t_bh2_sink_on", m.t_bh2_sink_on)};
    h5::Group grid;
    grid.name = "grid";
    grid.attrs = {h5::attr_i64("nx", g.nx), h5::attr_i64("ny", g.ny), h5::attr_i64("nz", g.nz),
                  h5::attr_f64("dx", g.dx), h5::attr_f64("dy", g.dy), h5::attr_f64("dz", g.dz),
                  h5::attr_f64("gamma", g.gamma), h5::attr_f64("x0", g.x0), h5::attr_f64("y0", g.y0),
                  h5::attr_f64("z0", g.z0), h5::attr_f64("rho_floor", g.rho_floor),
                  h5::attr_f64("P_floor", g.P_floor)};
    h5::Dataset u;
    u.name = "U"; u.kind = h5::F64; u.dims = state_dims(g.nx, g.ny, g.nz); u.data = U;
    grid.dsets.push_back(u);
    BHArrays A;
    root.groups = {man, grid, bh_group(bhs, nbh, A)};
    return h5::write_file(path, root, err);
}

bool valid_grid(const bsn_grid_meta& g) { return g.nx >= 1 && g.ny >= 1 && g.nz >= 1; }

// asynchronous uniform checkpoint: device snapshot, pinned host copy, writer thread
struct CkptState {
    int device = 0;
    double* snap = nullptr;
    double* host = nullptr;
    size_t bytes = 0;
    cudaStream_t copy = nullptr;
    cudaEvent_t snapped = nullptr, copied = nullptr;
    std::thread th;
    bool active = false;
    bsn_status result = BSN_OK;
    std::string err;
};

CkptState* ckpt(bsn_ctx* ctx) {
    if (!ctx->ckpt_state) ctx->ckpt_state = new CkptState();
    return (CkptState*)ctx->ckpt_state;
}

}  // namespace

void ckpt_state_free(bsn_ctx* ctx) {
    if (!ctx->ckpt_state) return;
    CkptState* S = (CkptState*)ctx->ckpt_state;
    if (S->th.joinable()) S->th.join();
    if (S->snap) cudaFree(S->snap);
    if (S->host) cudaFreeHost(S->host);
    if (S->copy) cudaStreamDestroy(S->copy);
    if (S->snapped) cudaEventDestroy(S->snapped);
    if (S->copied) cudaEventDestroy(S->copied);
    delete S;
    ctx->ckpt_state = nullptr;
}

}  // namespace bsn

using namespace bsn;

extern "C" bsn_status bsn_save_checkpoint_uniform(bsn_ctx* ctx, const char* path, const double* U, int on_device,
                                                  const bsn_bh* bhs, int nbh, const bsn_grid_meta* g,
                                                  const bsn_ckpt_meta* m) {
    try {
        if (!path || !U || !g || !m || nbh < 0 || (nbh > 0 && !bhs) || !valid_grid(*g) || (on_device && !ctx))
            return ctx ? set_err(ctx, BSN_ERR_ARG, "invalid checkpoint arguments") : BSN_ERR_ARG;
        std::vector<double> tmp;
        const double* h = nullptr;
        BSN_TRY(fetch(ctx, U, on_device, state_elems(g->nx, g->ny, g->nz), tmp, &h));
        std::string err;
        if (!write_uniform(path, h, bhs, nbh, *g, *m, &err)) return io_err(ctx, err);
        return BSN_OK;
    } catch (const std::bad_alloc&) {
        return ctx ? set_err(ctx, BSN_ERR_NOMEM, "host memory exhausted") : BSN_ERR_NOMEM;
    } catch (...) {
        return ctx ? set_err(ctx, BSN_ERR_IO, "unexpected error") : BSN_ERR_IO;
    }
}

extern "C" bsn_status bsn_save_checkpoint_uniform_async(bsn_ctx* ctx, const char* path, const double* U,
                                                        const bsn_bh* bhs, int nbh, const bsn_grid_meta* g,
                                                        const bsn_ckpt_meta* m) {
    try {
        if (!ctx) return BSN_ERR_ARG;
        if (!path || !U || !g || !m || nbh < 0 || (nbh > 0 && !bhs) || !valid_grid(*g))
            return set_err(ctx, BSN_ERR_ARG, "invalid checkpoint arguments");
        BSN_TRY(bsn_checkpoint_wait(ctx));   // one checkpoint in flight per context
        CkptState* S = ckpt(ctx);
        const size_t bytes = sizeof(double) * (size_t)state_elems(g->nx, g->ny, g->nz);
        if (S->bytes < bytes) {
            if (S->snap) cudaFree(S->snap);
            if (S->host) cudaFreeHost(S->host);
            S->snap = nullptr; S->host = nullptr; S->bytes = 0;
            BSN_CUDA(ctx, cudaMalloc(&S->snap, bytes));
            BSN_CUDA(ctx, cudaMallocHost(&S->host, bytes));
            S->bytes = bytes;
        }
        if (!S->copy) {
            BSN_CUDA(ctx, cudaStreamCreateWithFlags(&S->copy, cudaStreamNonBlocking));
            BSN_CUDA(ctx, cudaEventCreateWithFlags(&S->snapped, cudaEventDisableTiming));
            BSN_CUDA(ctx, cudaEventCreateWithFlags(&S->copied, cudaEventDisableTiming));
        }
        // the snapshot is ordered on the caller's stream: later work there may change U at once
        BSN_CUDA(ctx, cudaMemcpyAsync(S->snap, U, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        BSN_CUDA(ctx, cudaEventRecord(S->snapped, ctx->stream));
        BSN_CUDA(ctx, cudaStreamWaitEvent(S->copy, S->snapped, 0));
        BSN_CUDA(ctx, cudaMemcpyAsync(S->host, S->snap, bytes, cudaMemcpyDeviceToHost, S->copy));
        BSN_CUDA(ctx, cudaEventRecord(S->copied, S->copy));
        std::vector<bsn_bh> b(bhs, bhs + nbh);
        const bsn_grid_meta gm = *g;
        const bsn_ckpt_meta mm = *m;
        const std::string p = path;
        S->device = ctx->device;
        S->active = true;
        S->result = BSN_OK;
        S->err.clear();
        S->th = std::thread([S, b, gm, mm, p]() {
            cudaSetDevice(S->device);
            if (cudaEventSynchronize(S->copied) != cudaSuccess) {
                S->result = BSN_ERR_CUDA;
                S->err = "checkpoint copy failed";
                return;
            }
            std::string err;
            if (!write_uniform(p, S->host, b.data(), (int)b.size(), gm, mm, &err)) {
                S->result = BSN_ERR_IO;
                S->err = err;
            }
        });
        return BSN_OK;
    } catch (const std::bad_alloc&) {
        return ctx ? set_err(ctx, BSN_ERR_NOMEM, "host memory exhausted") : BSN_ERR_NOMEM;
    } catch (...) {
        return ctx ? set_err(ctx, BSN_ERR_IO, "unexpected error") : BSN_ERR_IO;
    }
}

extern "C" bsn_status bsn_checkpoint_wait(bsn_ctx* ctx) {
    try {
        if (!ctx) return BSN_ERR_ARG;
        if (!ctx->ckpt_state) return BSN_OK;
        CkptState* S = (CkptState*)ctx->ckpt_state;
        if (!S->active) return BSN_OK;
        if (S->th.joinable()) S->th.join();
        S->active = false;
        if (S->result != BSN_OK) return set_err(ctx, S->result, "asynchronous checkpoint: %s", S->err.c_str());
        return BSN_OK;
    } catch (const std::bad_alloc&) {
        return ctx ? set_err(ctx, BSN_ERR_NOMEM, "host memory exhausted") : BSN_ERR_NOMEM;
    } catch (...) {
        return ctx ? set_err(ctx, BSN_ERR_IO, "unexpected error") : BSN_ERR_IO;
    }
}

extern "C" bsn_status bsn_load_checkpoint_uniform(bsn_ctx* ctx, const char* path, double* U, int on_device,
                                                  bsn_bh* bhs, int cap_bh, int* nbh, bsn_grid_meta* g,
                                                  bsn_ckpt_meta* m) {
    try {
        if (!path || !nbh || !g || !m || (U && on_device && !ctx)) return ctx ? set_err(ctx, BSN_ERR_ARG, "null argument") : BSN_ERR_ARG;
        h5::Reader R;
        std::string err;
        if (!R.open(path, &err)) return io_err(ctx, err);
        const h5::RGroup* man = R.group("manifest");
        const h5::RGroup* gr = R.group("grid");
        int64_t fv = 0, step = 0, nx = 0, ny = 0, nz = 0;
        std::string kind;
        if (!man || !gr || !h5::get_i64(man->attrs, "format_version", &fv))
            return io_err(ctx, std::string(path) + ": no checkpoint manifest");
        if (fv != FORMAT_VERSION) return io_err(ctx, "checkpoint format_version " + std::to_string(fv) + ", expected 1");
        if (!h5::get_str(man->attrs, "kind", &kind) || kind != "uniform")
            return io_err(ctx, std::string(path) + " is not a uniform-grid checkpoint (kind != \"uniform\")");
        bool ok = h5::get_f64(man->attrs, "t", &m->t) && h5::get_i64(man->attrs, "step", &step) &&
                  h5::get_f64(man->attrs, "dt_last", &m->dt_last) && h5::get_f64(man->attrs, "t_snap", &m->t_snap) &&
                  h5::get_f64(man->attrs, "t_bh2_sink_on", &m->t_bh2_sink_on) &&
                  h5::get_i64(gr->attrs, "nx", &nx) && h5::get_i64(gr->attrs, "ny", &ny) && h5::get_i64(gr->attrs, "nz", &nz) &&
                  h5::get_f64(gr->attrs, "dx", &g->dx) && h5::get_f64(gr->attrs, "dy", &g->dy) &&
                  h5::get_f64(gr->attrs, "dz", &g->dz) && h5::get_f64(gr->attrs, "gamma", &g->gamma) &&
                  h5::get_f64(gr->attrs, "x0", &g->x0) && h5::get_f64(gr->attrs, "y0", &g->y0) &&
                  h5::get_f64(gr->attrs, "z0", &g->z0) && h5::get_f64(gr->attrs, "rho_floor", &g->rho_floor) &&
                  h5::get_f64(gr->attrs, "P_floor", &g->P_floor);
        if (!ok) return io_err(ctx, std::string(path) + ": checkpoint attributes missing");
        m->step = step;
        g->nx = (int)nx; g->ny = (int)ny; g->nz = (int)nz;
        if (!read_bhs(R, bhs, cap_bh, nbh, &err)) return io_err(ctx, err);
        if (!U) return BSN_OK;
        const h5::RDataset* d = R.dataset("grid/U");
        if (!d || d->kind != h5::F64 || d->dims != state_dims(g->nx, g->ny, g->nz))
            return io_err(ctx, std::string(path) + ": /grid/U does not match the grid");
        const size_t bytes = sizeof(double) * (size_t)state_elems(g->nx, g->ny, g->nz);
        if (!on_device) return R.read_data(*d, U, bytes, &err) ? BSN_OK : io_err(ctx, err);
        std::vector<double> h(bytes / 8);
        if (!R.read_data(*d, h.data(), bytes, &err)) return io_err(ctx, err);
        BSN_CUDA(ctx, cudaMemcpyAsync(U, h.data(), bytes, cudaMemcpyHostToDevice, ctx->stream));
        BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        return BSN_OK;
    } catch (const std::bad_alloc&) {
        return ctx ? set_err(ctx, BSN_ERR_NOMEM, "host memory exhausted") : BSN_ERR_NOMEM;
    } catch (...) {
        return ctx ? set_err(ctx, BSN_ERR_IO, "unexpected error") : BSN_ERR_IO;
    }
}

// ---- two-level FMR checkpoint (src/checkpoint.jl:39-119) ---------------------

extern "C" bsn_status bsn_save_checkpoint_fmr(bsn_ctx* ctx, const char* path, const bsn_fmr2* G, int on_device,
                                              const bsn_bh* bhs, int nbh, double t, long long step, double dt_last) {
    try {
        if (!path || !G || !G->Uc || !G->Uf || nbh < 0 || (nbh > 0 && !bhs) || (on_device && !ctx))
            return ctx ? set_err(ctx, BSN_ERR_ARG, "invalid checkpoint arguments") : BSN_ERR_ARG;
        std::vector<double> tc, tf;
        const double *hc = nullptr, *hf = nullptr;
        BSN_TRY(fetch(ctx, G->Uc, on_device, state_elems(G->ncx, G->ncy, G->ncz), tc, &hc));
        BSN_TRY(fetch(ctx, G->Uf, on_device, state_elems(G->nfx, G->nfy, G->nfz), tf, &hf));
        h5::Group root, man, grid;
        man.name = "manifest";
        man.attrs = {h5::attr_i64("format_version", FORMAT_VERSION), h5::attr_f64("t", t), h5::attr_i64("step", step),
                     h5::attr_f64("dt_last", dt_last)};
        grid.name = "grid";
        grid.attrs = {h5::attr_i64("ratio", G->ratio), h5::attr_f64("gamma", G->gamma),
                      h5::attr_str("bc", G->bc == BSN_BC_PERIODIC ? "periodic" : "outflow"),
                      h5::attr_f64("rho_floor", G->rho_floor), h5::attr_f64("P_floor", G->P_floor),
                      h5::attr_i64("ci_lo", G->ci_lo), h5::attr_i64("ci_hi", G->ci_hi),
                      h5::attr_i64("cj_lo", G->cj_lo), h5::attr_i64("cj_hi", G->cj_hi),
                      h5::attr_i64("ck_lo", G->ck_lo), h5::attr_i64("ck_hi", G->ck_hi)};
        auto level = [](const char* name, int nx, int ny, int nz, double dx, double dy, double dz, const double* U) {
            h5::Group l;
            l.name = name;
            l.attrs = {h5::attr_i64("nx", nx), h5::attr_i64("ny", ny), h5::attr_i64("nz", nz), h5::attr_f64("dx", dx),
                       h5::attr_f64("dy", dy), h5::attr_f64("dz", dz)};
            h5::Dataset u;
            u.name = "U"; u.kind = h5::F64; u.dims = state_dims(nx, ny, nz); u.data = U;
            l.dsets.push_back(u);
            return l;
        };
        grid.groups = {level("coarse", G->ncx, G->ncy, G->ncz, G->dxc, G->dyc, G->dzc, hc),
                       level("fine", G->nfx, G->nfy, G->nfz, G->dxf, G->dyf, G->dzf, hf)};
        BHArrays A;
        root.groups = {man, grid, bh_group(bhs, nbh, A)};
        std::string err;
        if (!h5::write_file(path, root, &err)) return io_err(ctx, err);
        return BSN_OK;
    } catch (const std::bad_alloc&) {
        return ctx ? set_err(ctx, BSN_ERR_NOMEM, "host memory exhausted") : BSN_ERR_NOMEM;
    } catch (...) {
        return ctx ? set_err(ctx, BSN_ERR_IO, "unexpected error") : BSN_ERR_IO;
    }
}

extern "C" bsn_status bsn_load_checkpoint_fmr(bsn_ctx* ctx, const char* path, bsn_fmr2* G, int on_device,
                                              bsn_bh* bhs, int cap_bh, int* nbh, double* t, long long* step,
                                              double* dt_last) {
    try {
        if (!path || !G || !nbh || !t || !step || !dt_last || (on_device && (G->Uc || G->Uf) && !ctx))
            return ctx ? set_err(ctx, BSN_ERR_ARG, "null argument") : BSN_ERR_ARG;
        h5::Reader R;
        std::string err;
        if (!R.open(path, &err)) return io_err(ctx, err);
        const h5::RGroup *man = R.group("manifest"), *gr = R.group("grid");
        const h5::RGroup *co = R.group("grid/coarse"), *fi = R.group("grid/fine");
        int64_t fv = 0, st = 0, v[7];
        std::string bc;
        if (!man || !gr || !co || !fi || !h5::get_i64(man->attrs, "format_version", &fv))
            return io_err(ctx, std::string(path) + ": no FMR checkpoint manifest");
        if (fv != FORMAT_VERSION) return io_err(ctx, "checkpoint format_version " + std::to_string(fv) + ", expected 1");
        const char* keys[7] = {"ratio", "ci_lo", "ci_hi", "cj_lo", "cj_hi", "ck_lo", "ck_hi"};
        bool ok = h5::get_f64(man->attrs, "t", t) && h5::get_i64(man->attrs, "step", &st) &&
                  h5::get_f64(man->attrs, "dt_last", dt_last) && h5::get_f64(gr->attrs, "gamma", &G->gamma) &&
                  h5::get_str(gr->attrs, "bc", &bc) && h5::get_f64(gr->attrs, "rho_floor", &G->rho_floor) &&
                  h5::get_f64(gr->attrs, "P_floor", &G->P_floor);
        for (int i = 0; i < 7; ++i) ok = ok && h5::get_i64(gr->attrs, keys[i], &v[i]);
        int64_t c3[3], f3[3];
        ok = ok && h5::get_i64(co->attrs, "nx", &c3[0]) && h5::get_i64(co->attrs, "ny", &c3[1]) &&
             h5::get_i64(co->attrs, "nz", &c3[2]) && h5::get_i64(fi->attrs, "nx", &f3[0]) &&
             h5::get_i64(fi->attrs, "ny", &f3[1]) && h5::get_i64(fi->attrs, "nz", &f3[2]) &&
             h5::get_f64(co->attrs, "dx", &G->dxc) && h5::get_f64(co->attrs, "dy", &G->dyc) &&
             h5::get_f64(co->attrs, "dz", &G->dzc) && h5::get_f64(fi->attrs, "dx", &G->dxf) &&
             h5::get_f64(fi->attrs, "dy", &G->dyf) && h5::get_f64(fi->attrs, "dz", &G->dzf);
        if (!ok) return io_err(ctx, std::string(path) + ": checkpoint attributes missing");
        *step = st;
        G->ratio = (int)v[0]; G->ci_lo = (int)v[1]; G->ci_hi = (int)v[2]; G->cj_lo = (int)v[3]; G->cj_hi = (int)v[4];
        G->ck_lo = (int)v[5]; G->ck_hi = (int)v[6];
        G->bc = bc == "periodic" ? BSN_BC_PERIODIC : BSN_BC_OUTFLOW;
        G->ncx = (int)c3[0]; G->ncy = (int)c3[1]; G->ncz = (int)c3[2];
        G->nfx = (int)f3[0]; G->nfy = (int)f3[1]; G->nfz = (int)f3[2];
        if (!read_bhs(R, bhs, cap_bh, nbh, &err)) return io_err(ctx, err);
        struct { const char* p; double* U; int nx, ny, nz; } lv[2] = {{"grid/coarse/U", G->Uc, G->ncx, G->ncy, G->ncz},
                                                                     {"grid/fine/U", G->Uf, G->nfx, G->nfy, G->nfz}};
        for (auto& l : lv) {
            if (!l.U) continue;
            const h5::RDataset* d = R.dataset(l.p);
            if (!d || d->kind != h5::F64 || d->dims != state_dims(l.nx, l.ny, l.nz))
                return io_err(ctx, std::string(path) + ": /" + l.p + " does not match its level");
            const size_t bytes = sizeof(double) * (size_t)state_elems(l.nx, l.ny, l.nz);
            if (!on_device) {
                if (!R.read_data(*d, l.U, bytes, &err)) return io_err(ctx, err);
                continue;
            }
            std::vector<double> h(bytes / 8);
            if (!R.read_data(*d, h.data(), bytes, &err)) return io_err(ctx, err);
            BSN_CUDA(ctx, cudaMemcpyAsync(l.U, h.data(), bytes, cudaMemcpyHostToDevice, ctx->stream));
            BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        }
        return BSN_OK;
    } catch (const std::bad_alloc&) {
        return ctx ? set_err(ctx, BSN_ERR_NOMEM, "host memory exhausted") : BSN_ERR_NOMEM;
    } catch (...) {
        return ctx ? set_err(ctx, BSN_ERR_IO, "unexpected error") : BSN_ERR_IO;
    }
}

// ---- snapshots (src/io.jl:29-83) ----------------------------------------------

extern "C" bsn_status bsn_write_snapshot(bsn_ctx* ctx, const char* path, const double* U, int on_device, int nx,
                                         int ny, int nz, double dx, double dy, double dz, double t, double gamma) {
    try {
        if (!path || !U || nx < 1 || ny < 1 || nz < 1 || (on_device && !ctx))
            return ctx ? set_err(ctx, BSN_ERR_ARG, "invalid snapshot arguments") : BSN_ERR_ARG;
        std::vector<double> tmp;
        const double* h = nullptr;
        BSN_TRY(fetch(ctx, U, on_device, state_elems(nx, ny, nz), tmp, &h));
        // the five active-cell fields, each (nx, ny, nz) column-major
        const size_t nc = (size_t)nx * ny * nz;
        std::vector<double> F(5 * nc);
        const long long X = nx + 2 * BSN_NG, Y = ny + 2 * BSN_NG;
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const double* c = h + 5 * ((i + BSN_NG) + X * ((j + BSN_NG) + Y * (long long)(k + BSN_NG)));
                    const size_t o = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
                    for (int q = 0; q < 5; ++q) F[q * nc + o] = c[q];
                }
        h5::Group root, gas;
        gas.name = "gas";
        const char* names[5] = {"rho", "rhovx", "rhovy", "rhovz", "E"};
        for (int q = 0; q < 5; ++q) {
            h5::Dataset d;
            d.name = names[q]; d.kind = h5::F64; d.dims = {(uint64_t)nz, (uint64_t)ny, (uint64_t)nx};
            d.data = F.data() + q * nc;
            gas.dsets.push_back(d);
        }
        root.groups = {gas};
        root.attrs = {h5::attr_f64("t", t), h5::attr_i64("nx", nx), h5::attr_i64("ny", ny), h5::attr_i64("nz", nz),
                      h5::attr_f64("dx", dx), h5::attr_f64("dy", dy), h5::attr_f64("dz", dz),
                      h5::attr_f64("gamma", gamma)};
        std::string err;
        if (!h5::write_file(path, root, &err)) return io_err(ctx, err);
        return BSN_OK;
    } catch (const std::bad_alloc&) {
        return ctx ? set_err(ctx, BSN_ERR_NOMEM, "host memory exhausted") : BSN_ERR_NOMEM;
    } catch (...) {
        return ctx ? set_err(ctx, BSN_ERR_IO, "unexpected error") : BSN_ERR_IO;
    }
}

extern "C" bsn_status bsn_read_snapshot(const char* path, double* U_active, long long cap, int* nx, int* ny, int* nz,
                                        double* dx, double* dy, double* dz, double* t, double* gamma) {
    try {
        if (!path || !nx || !ny || !nz || !dx || !dy || !dz || !t || !gamma) return BSN_ERR_ARG;
        h5::Reader R;
        std::string err;
        if (!R.open(path, &err)) return BSN_ERR_IO;
        const auto& a = R.root().attrs;
        int64_t n3[3];
        if (!h5::get_i64(a, "nx", &n3[0]) || !h5::get_i64(a, "ny", &n3[1]) || !h5::get_i64(a, "nz", &n3[2]) ||
            !h5::get_f64(a, "dx", dx) || !h5::get_f64(a, "dy", dy) || !h5::get_f64(a, "dz", dz) ||
            !h5::get_f64(a, "t", t) || !h5::get_f64(a, "gamma", gamma))
            return BSN_ERR_IO;
        *nx = (int)n3[0]; *ny = (int)n3[1]; *nz = (int)n3[2];
        if (!U_active) return BSN_OK;
        const size_t nc = (size_t)n3[0] * n3[1] * n3[2];
        if ((long long)(5 * nc) > cap) return BSN_ERR_ARG;
        const char* names[5] = {"gas/rho", "gas/rhovx", "gas/rhovy", "gas/rhovz", "gas/E"};
        std::vector<double> f(nc);
        for (int q = 0; q < 5; ++q) {
            const h5::RDataset* d = R.dataset(names[q]);
            if (!d || d->kind != h5::F64 || d->count() != nc || !R.read_data(*d, f.data(), 8 * nc, &err)) return BSN_ERR_IO;
            for (size_t o = 0; o < nc; ++o) U_active[5 * o + q] = f[o];   // U_active[q, i, j, k]
        }
        return BSN_OK;
    } catch (const std::bad_alloc&) {
        return BSN_ERR_NOMEM;
    } catch (...) {
        return BSN_ERR_IO;
    }
}

// ---- BH trajectories (src/io.jl:96-180) -----------------------------------------
// The reference extends chunked datasets per dump; here every append rewrites
// the file with contiguous datasets one record longer (same names, shapes
// and values; a trajectory is a few hundred bytes per dump).

namespace {
struct Traj {
    std::vector<double> t;
    struct B { std::vector<double> mass, rsink, pos, vel; };   // pos/vel: (N, 3) column-major
    std::vector<B> bh;
};

bool traj_write(const std::string& path, Traj& T, std::string* err) {
    h5::Group root;
    const uint64_t N = T.t.size();
    h5::Dataset td;
    td.name = "time"; td.kind = h5::F64; td.dims = {N}; td.data = T.t.data();
    root.dsets.push_back(td);
    for (size_t i = 0; i < T.bh.size(); ++i) {
        h5::Group g;
        g.name = "bh" + std::to_string(i + 1);
        auto add = [&](const char* n, const std::vector<double>& v, std::vector<uint64_t> dims) {
            h5::Dataset d;
            d.name = n; d.kind = h5::F64; d.dims = dims; d.data = v.data();
            g.dsets.push_back(d);
        };
        add("mass", T.bh[i].mass, {N});
        add("rsink", T.bh[i].rsink, {N});
        add("pos", T.bh[i].pos, {3, N});
        add("vel", T.bh[i].vel, {3, N});
        root.groups.push_back(g);
    }
    return h5::write_file(path, root, err);
}

bool traj_read(const std::string& path, Traj& T, std::string* err) {
    h5::Reader R;
    if (!R.open(path, err)) return false;
    const h5::RDataset* td = R.dataset("time");
    if (!td || td->dims.size() != 1) { *err = path + ": no /time"; return false; }
    const uint64_t N = td->dims[0];
    T.t.resize(N);
    if (N && !R.read_data(*td, T.t.data(), 8 * N, err)) return false;
    for (int i = 1;; ++i) {
        const h5::RGroup* g = R.group("bh" + std::to_string(i));
        if (!g) break;
        Traj::B b;
        struct { const char* n; std::vector<double>* v; uint64_t cnt; } f[] = {
            {"mass", &b.mass, N}, {"rsink", &b.rsink, N}, {"pos", &b.pos, 3 * N}, {"vel", &b.vel, 3 * N}};
        for (auto& x : f) {
            auto it = g->dsets.find(x.n);
            if (it == g->dsets.end() || it->second.count() != x.cnt) { *err = path + ": bad bh dataset"; return false; }
            x.v->resize(x.cnt);
            if (x.cnt && !R.read_data(it->second, x.v->data(), 8 * x.cnt, err)) return false;
        }
        T.bh.push_back(b);
    }
    return true;
}
}  // namespace

extern "C" bsn_status bsn_trajectory_init(const char* path, int n_bh) {
    try {
        if (!path || n_bh < 0) return BSN_ERR_ARG;
        Traj T;
        T.bh.resize((size_t)n_bh);
        std::string err;
        return traj_write(path, T, &err) ? BSN_OK : BSN_ERR_IO;
    } catch (const std::bad_alloc&) {
        return BSN_ERR_NOMEM;
    } catch (...) {
        return BSN_ERR_IO;
    }
}

extern "C" bsn_status bsn_trajectory_append(const char* path, double t, const bsn_bh* bhs, int nbh) {
    try {
        if (!path || nbh < 0 || (nbh > 0 && !bhs)) return BSN_ERR_ARG;
        Traj T;
        std::string err;
        if (!traj_read(path, T, &err)) return BSN_ERR_IO;
        if ((int)T.bh.size() != nbh) return BSN_ERR_ARG;
        const size_t N = T.t.size();
        T.t.push_back(t);
        for (int i = 0; i < nbh; ++i) {
            Traj::B& b = T.bh[i];
            b.mass.push_back(bhs[i].mass);
            b.rsink.push_back(jmax(6.0 * bhs[i].mass / sq(bhs[i].c_code), bhs[i].r_floor));   // r_sink(bh)
            // (N+1, 3) column-major: insert the new row's entry at the end of each column
            std::vector<double> p(3 * (N + 1)), v(3 * (N + 1));
            for (int d = 0; d < 3; ++d) {
                for (size_t r = 0; r < N; ++r) { p[d * (N + 1) + r] = b.pos[d * N + r]; v[d * (N + 1) + r] = b.vel[d * N + r]; }
                p[d * (N + 1) + N] = bhs[i].pos[d];
                v[d * (N + 1) + N] = bhs[i].vel[d];
            }
            b.pos.swap(p);
            b.vel.swap(v);
        }
        return traj_write(path, T, &err) ? BSN_OK : BSN_ERR_IO;
    } catch (const std::bad_alloc&) {
        return BSN_ERR_NOMEM;
    } catch (...) {
        return BSN_ERR_IO;
    }
}

extern "C" bsn_status bsn_trajectory_read(const char* path, int* n_dumps, int* n_bh, double* t, double* mass,
                                          double* pos, double* vel, double* rsink, long long cap) {
    try {
        if (!path || !n_dumps || !n_bh) return BSN_ERR_ARG;
        Traj T;
        std::string err;
        if (!traj_read(path, T, &err)) return BSN_ERR_IO;
        const long long N = (long long)T.t.size(), nb = (long long)T.bh.size();
        *n_dumps = (int)N;
        *n_bh = (int)nb;
        if (!t) return BSN_OK;
        if (N > cap) return BSN_ERR_ARG;
        // t[N]; mass/rsink[b][N]; pos/vel[b][N][3] (row per dump)
        for (long long r = 0; r < N; ++r) t[r] = T.t[r];
        for (long long b = 0; b < nb; ++b)
            for (long long r = 0; r < N; ++r) {
                if (mass) mass[b * N + r] = T.bh[b].mass[r];
                if (rsink) rsink[b * N + r] = T.bh[b].rsink[r];
                for (int d = 0; d < 3; ++d) {
                    if (pos) pos[(b * N + r) * 3 + d] = T.bh[b].pos[d * N + r];
                    if (vel) vel[(b * N + r) * 3 + d] = T.bh[b].vel[d * N + r];
                }
            }
        return BSN_OK;
    } catch (const std::bad_alloc&) {
        return BSN_ERR_NOMEM;
    } catch (...) {
        return BSN_ERR_IO;
    }
}
