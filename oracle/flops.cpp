/*
 * flops.cpp -- algorithmic floating-point operation count of the reference's
 * SSP-RK3 step (TEST INFRASTRUCTURE ONLY; used by tests/ and by
 * oracle/count_flops.py, never by the product path).
 *
 * hydro.inc, the oracle's restatement of euler3d_step! (src/euler3d.jl:220-260
 * with src/weno5.jl, src/hllc.jl, src/gpu_kernels.jl), is compiled here over
 * FD: a double that counts every +, -, *, /, sqrt and comparison it takes
 * part in, one each whatever the operands.  The values computed are the
 * oracle's own (FD does the same IEEE double operation), so the count follows
 * the branches the reference takes on the given state.  Unary minus, fabs,
 * copies and the compile-time constants (1.0/3.0 and the like) are not
 * counted.  Single-threaded: the OpenMP pragmas of hydro.inc are ignored.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace flopcount {
unsigned long long n_add, n_mul, n_div, n_sqrt, n_cmp;
}

struct FD {
    double v;
    FD() = default;
    constexpr FD(double x) : v(x) {}
    FD(int x) : v((double)x) {}
    FD(long x) : v((double)x) {}
    FD operator-() const { return FD(-v); }
    FD& operator*=(FD o) { ++flopcount::n_mul; v *= o.v; return *this; }
    FD& operator+=(FD o) { ++flopcount::n_add; v += o.v; return *this; }
};
static_assert(sizeof(FD) == sizeof(double), "FD is a double");

inline FD operator+(FD a, FD b) { ++flopcount::n_add; return FD(a.v + b.v); }
inline FD operator-(FD a, FD b) { ++flopcount::n_add; return FD(a.v - b.v); }
inline FD operator*(FD a, FD b) { ++flopcount::n_mul; return FD(a.v * b.v); }
inline FD operator/(FD a, FD b) { ++flopcount::n_div; return FD(a.v / b.v); }
inline bool operator<(FD a, FD b) { ++flopcount::n_cmp; return a.v < b.v; }
inline bool operator>(FD a, FD b) { ++flopcount::n_cmp; return a.v > b.v; }
inline bool operator<=(FD a, FD b) { ++flopcount::n_cmp; return a.v <= b.v; }
inline bool operator>=(FD a, FD b) { ++flopcount::n_cmp; return a.v >= b.v; }
inline bool operator==(FD a, FD b) { ++flopcount::n_cmp; return a.v == b.v; }
inline bool operator!=(FD a, FD b) { ++flopcount::n_cmp; return a.v != b.v; }

namespace std {
inline FD sqrt(FD x) { ++flopcount::n_sqrt; return FD(std::sqrt(x.v)); }
inline FD fabs(FD x) { return FD(std::fabs(x.v)); }
inline bool signbit(FD x) { return std::signbit(x.v); }
}  // namespace std

#define double FD
#include "hydro.inc"
#undef double

extern "C" __attribute__((visibility("default"))) void orc_count_step(
    double* U, int nx, int ny, int nz, double dx, double dy, double dz, double dt, double g, int bc,
    double rho_floor, double P_floor, unsigned long long out[5]) {
    const long n = 5L * (nx + 2 * NG) * (ny + 2 * NG) * (nz + 2 * NG);
    std::vector<FD> V(n);
    std::memcpy(V.data(), U, sizeof(double) * n);
    flopcount::n_add = flopcount::n_mul = flopcount::n_div = flopcount::n_sqrt = flopcount::n_cmp = 0;
    orc_euler3d_step(V.data(), nx, ny, nz, FD(dx), FD(dy), FD(dz), FD(dt), FD(g), bc, FD(rho_floor),
                     FD(P_floor));
    out[0] = flopcount::n_add;
    out[1] = flopcount::n_mul;
    out[2] = flopcount::n_div;
    out[3] = flopcount::n_sqrt;
    out[4] = flopcount::n_cmp;
    std::memcpy(U, V.data(), sizeof(double) * n);
}
