"""Helpers shared by the GPU parity tests: host<->device transfer in the
reference layout and seeded test states."""
import numpy as np
import torch

NG = 3


def dev(a: np.ndarray) -> torch.Tensor:
    """F-ordered numpy array -> CUDA tensor with the same (column-major) strides."""
    assert a.flags.f_contiguous
    t = torch.from_numpy(a).cuda()
    assert t.stride() == tuple(s // 8 for s in a.strides)
    return t


def host(t: torch.Tensor) -> np.ndarray:
    a = t.cpu().numpy()
    return np.asfortranarray(a)


def random_state(nx, ny, nz, seed=0, gamma=1.4, jumps=True, vacuum=False):
    """Smooth random state plus optional discontinuities / near-vacuum cells,
    so every WENO, floor and HLLC branch is exercised."""
    rng = np.random.default_rng(seed)
    X, Y, Z = nx + 2 * NG, ny + 2 * NG, nz + 2 * NG
    U = np.zeros((5, X, Y, Z), order="F")
    rho = 1.0 + 0.3 * rng.standard_normal((X, Y, Z))
    rho = np.abs(rho) + 0.05
    v = 0.5 * rng.standard_normal((3, X, Y, Z))
    P = np.abs(1.0 + 0.3 * rng.standard_normal((X, Y, Z))) + 0.01
    if jumps:
        i = np.arange(X)[:, None, None]
        j = np.arange(Y)[None, :, None]
        k = np.arange(Z)[None, None, :]
        blob = ((i - X / 2) ** 2 + (j - Y / 3) ** 2 + (k - Z / 2) ** 2) < (min(X, Y, Z) / 3) ** 2
        rho = np.where(blob, rho * 10.0, rho)
        P = np.where(blob, P * 100.0, P)
        v[0] = np.where(i > X // 2, v[0] + 3.0, v[0])
    if vacuum:
        m = rng.random((X, Y, Z)) < 0.02
        rho = np.where(m, 1e-9, rho)
        P = np.where(rng.random((X, Y, Z)) < 0.02, -1e-3, P)
    U[0] = rho
    U[1:4] = rho * v
    U[4] = P / (gamma - 1) + 0.5 * rho * (v ** 2).sum(0)
    return U


def assert_bitwise(a: np.ndarray, b: np.ndarray, what=""):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    if not same.all():
        idx = np.argwhere(~same)[:5]
        rel = np.max(np.abs(a - b)[~same] / np.maximum(np.abs(b[~same]), 1e-300))
        raise AssertionError(f"{what}: {(~same).sum()} of {a.size} differ (max rel {rel:.3e}); first {idx.tolist()}")
