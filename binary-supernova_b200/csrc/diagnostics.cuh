// diagnostics.cuh -- the conserved-total and bound-mass reduction (diagnostics.cu).
#pragma once

#include "hydro_f64.cuh"

namespace bsn {
namespace diag {

constexpr int NDIAG = 10;     // E_gas, KE_gas, Px, Py, Pz, Lx, Ly, Lz, M_bound, M_gas
constexpr int NREC = NDIAG + 2 + f64::LEDT_COUNT;   // per-step record: t, dt, totals, mass ledger
constexpr int BLOCKS = 148 * 2;

// One reduction over the active cells of U.  bhs_dev: device BHs (nbh of
// them, or *nbh_dev when non-null).  part: 2 NDIAG BLOCKS doubles of scratch.
// Without `steps`: out[0..NDIAG) = the totals.  With the device loop's t, dt,
// steps (and done: nothing once the loop has finished): record {t, dt, totals,
// ledger[0..LEDT_COUNT) (zeros when ledger is null)} at out + NREC (steps - 1)
// when steps - 1 < cap.
bsn_status launch(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx, double dy, double dz, double x0,
                  double y0, double z0, const bsn_bh* bhs_dev, const int* nbh_dev, int nbh, double gamma,
                  double* part, double* out, const double* t, const double* dt, const int* steps, const int* done,
                  int cap, const double* ledger = nullptr);

}  // namespace diag
}  // namespace bsn
