"""The hand-written batched FFTs of the isolated Poisson solve against cuFFT.

The reference's GPU path runs solve_poisson_isolated (src/self_gravity.jl:35-76)
through AbstractFFTs on a CuArray, i.e. cuFFT: Phi = dV * real(ifft(fft(K) .*
fft(rho_pad)))[1:nx, 1:ny, 1:nz] with K = -1/sqrt(r^2 + eps^2) on the (2n)^3
grid with folded indices and eps^2 = (dx dy dz)^(2/3).  Here the same
expression runs through torch.fft on a CUDA tensor (cuFFT, complex128), and
bsn_solve_poisson_isolated_f64 / _f32 (the library's own line FFTs) are
compared with it: FP64 within 1e-12 relative L-inf (max |dPhi| / max |Phi|),
FP32 transforms within 1e-5.
"""
import numpy as np
import pytest

from gpu_util import dev

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _green(nx, ny, nz, dx, dy, dz):
    """K on the padded grid, as src/self_gravity.jl:43-55 builds it."""
    Nx, Ny, Nz = 2 * nx, 2 * ny, 2 * nz
    eps2 = (dx * dy * dz) ** (2.0 / 3.0)
    fi = np.where(np.arange(Nx) < nx, np.arange(Nx), np.arange(Nx) - Nx).astype(np.float64)
    fj = np.where(np.arange(Ny) < ny, np.arange(Ny), np.arange(Ny) - Ny).astype(np.float64)
    fk = np.where(np.arange(Nz) < nz, np.arange(Nz), np.arange(Nz) - Nz).astype(np.float64)
    r2 = ((fi * dx)[:, None, None] ** 2 + (fj * dy)[None, :, None] ** 2) + (fk * dz)[None, None, :] ** 2
    return -1.0 / np.sqrt(r2 + eps2)


def _cufft_phi(rho, dx, dy, dz):
    nx, ny, nz = rho.shape
    K = torch.from_numpy(_green(nx, ny, nz, dx, dy, dz)).cuda()
    pad = torch.zeros((2 * nx, 2 * ny, 2 * nz), dtype=torch.float64, device="cuda")
    pad[:nx, :ny, :nz] = rho
    assert pad.is_cuda and K.is_cuda     # torch.fft on CUDA tensors runs cuFFT
    phi = torch.fft.ifftn(torch.fft.fftn(K) * torch.fft.fftn(pad)).real * (dx * dy * dz)
    return phi[:nx, :ny, :nz]


def _density(nx, ny, nz, dx, dy, dz, seed):
    """A centrally condensed star (n=1 polytrope profile) in a 1e-8 floor plus
    a seeded random component: smooth and sharp structure at once."""
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5 - nx / 2) * dx
    y = (np.arange(ny) + 0.5 - ny / 2) * dy
    z = (np.arange(nz) + 0.5 - nz / 2) * dz
    r = np.sqrt(x[:, None, None] ** 2 + y[None, :, None] ** 2 + z[None, None, :] ** 2)
    R = 0.3 * min(nx * dx, ny * dy, nz * dz)
    xi = np.pi * r / R
    star = np.where(r < R, np.sinc(xi / np.pi), 0.0)
    rho = 1e-8 + star + 0.05 * rng.random((nx, ny, nz))
    return np.asfortranarray(rho)


@pytest.mark.parametrize("shape,d", [((128, 128, 128), (4.0 / 128,) * 3),
                                     ((32, 64, 16), (0.05, 0.03, 0.11)),
                                     ((16, 16, 64), (0.1, 0.1, 0.025)),
                                     # every line length of the transforms, 4 .. 4096 points
                                     ((2, 4, 8), (0.3, 0.2, 0.1)),
                                     ((512, 4, 2), (0.004, 0.2, 0.3)),
                                     ((4, 2048, 2), (0.2, 0.001, 0.3)),
                                     ((2, 2, 1024), (0.3, 0.3, 0.002)),
                                     ((256, 16, 32), (0.01, 0.1, 0.05))])
def test_poisson_solve_matches_cufft(shape, d):
    import bsn
    rho = dev(_density(*shape, *d, seed=sum(shape)))
    ref = _cufft_phi(rho, *d)
    scale = float(ref.abs().max())
    got64 = bsn.solve_poisson_isolated(rho, *shape, *d, precision="f64")
    err64 = float((got64 - ref).abs().max()) / scale
    assert err64 <= 1e-12, err64
    got32 = bsn.solve_poisson_isolated(rho, *shape, *d, precision="f32")
    err32 = float((got32 - ref).abs().max()) / scale
    assert err32 <= 1e-5, err32


def test_self_gravity_source_matches_cufft_potential(orc):
    """add_self_gravity_source! (src/self_gravity.jl:93-115) with the
    library's solve against the same gradient of the cuFFT potential (the
    oracle's gradient arithmetic on the cuFFT Phi): within 1e-12 of the
    largest source term."""
    import bsn
    from gpu_util import host, random_state
    n, d = 32, (0.05, 0.05, 0.05)
    U = random_state(n, n, n, seed=41, gamma=5 / 3, jumps=False)
    orc.fill_ghost_3d_outflow(U)
    Ud = dev(U)
    dU = torch.zeros_like(Ud)
    bsn.add_self_gravity_source(dU, Ud, n, n, n, *d)
    rho = Ud[0, 3:3 + n, 3:3 + n, 3:3 + n]
    phi = np.asfortranarray(_cufft_phi(rho, *d).cpu().numpy())
    dU_ref = np.zeros_like(U, order="F")
    orc.sg_gradient(dU_ref, U, phi, *d)
    got = host(dU)
    for q in range(1, 5):
        scale = np.abs(dU_ref[q]).max()
        assert np.abs(got[q] - dU_ref[q]).max() <= 1e-12 * scale, q
