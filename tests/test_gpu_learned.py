"""GPU tests of the learned WENO weights (no reference counterpart; plain
WENO5-Z is the yardstick):

* the hand-written training kernels' loss and gradient agree with a numpy
  FP64 forward/backward (tests/mlp_ref.py) to 1e-4 relative;
* the BF16 tensor-core inference used in the stencil kernel agrees with the
  FP32 arithmetic of the training kernels to BF16 accuracy;
* trained on stencils collected from the method's own Sedov and Sod runs, the
  network's reconstructions are closer to WENO5-Z than those of the linear
  (ideal) weights on held-out smooth stencils -- the gain the network brings;
* a Sedov run with the learned stencil path stays close to the FP64 solution.
"""
import numpy as np
import pytest

from gpu_util import NG, dev, host
from mlp_ref import candidates, loss_and_grad

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def bsn():
    import bsn as b
    return b


@pytest.fixture(scope="module")
def L():
    import bsn.learned as l
    return l


def _random_samples(n, seed):
    rng = np.random.default_rng(seed)
    u = rng.uniform(-1, 1, (n, 5))
    t = rng.dirichlet([1.0, 1.0, 1.0], n)
    return np.concatenate([u, t], axis=1).astype(np.float32)


def test_training_gradient_matches_cpu(L):
    S = _random_samples(1000, 1)
    p = L.init_params(seed=2)
    g, loss = L.grad(torch.from_numpy(S).cuda(), p)
    loss_ref, g_ref = loss_and_grad(p.cpu().numpy(), S)
    assert abs(loss - loss_ref) <= 1e-5 * loss_ref
    g = g.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(g - g_ref) <= 1e-4 * np.linalg.norm(g_ref)


def test_tensor_core_inference_matches_fp32(L):
    u = torch.from_numpy(_random_samples(4096, 3)[:, :5].copy()).cuda()
    p = L.init_params(seed=4)
    w32 = L.evaluate(u, p, tensor_cores=False)
    wtc = L.evaluate(u, p, tensor_cores=True)
    d = (w32 - wtc).abs()
    assert torch.allclose(w32.sum(1), torch.ones(4096, device="cuda"), atol=1e-5)
    assert d.mean().item() < 5e-3 and d.max().item() < 5e-2


def _sedov(orc, n, L_=1.0, g=5 / 3):
    dx = 2 * L_ / n
    U = orc.state(n, n, n)
    orc.sedov_ic_3d(U, dx, dx, dx, g, E_blast=1.0, r_inject=3.5 * dx, rho_bg=1.0, P_floor=1e-5,
                    x_offset=-L_, y_offset=-L_, z_offset=-L_)
    return U, dx


@pytest.fixture(scope="module")
def trained(orc, bsn, L):
    buf = L.SampleBuffers(4_000_000)
    U, dx = _sedov(orc, 48)
    Ud = dev(U)
    for k in range(8):
        bsn.run_steps(Ud, 48, 48, 48, dx, dx, dx, 5 / 3, 0.4, n_steps=3, rho_floor=1e-6, P_floor=1e-6)
        buf.collect(Ud, 48, 48, 48, 5 / 3, stride=1, seed=k)
    Us, dims, (dx, dy, dz) = orc.sod_ic_3d("x", n_normal=64, n_trans=16)
    Usd = dev(Us)
    for k in range(3):
        bsn.run_steps(Usd, *dims, dx, dy, dz, 1.4, 0.4, n_steps=10)
        buf.collect(Usd, *dims, 1.4, stride=1, seed=10 + k)
    nl, nr = buf.stored
    assert nl > 100_000 and nr > 100_000
    out = []
    for side, S in ((0, buf.left()), (1, buf.right())):
        perm = torch.randperm(S.shape[0], device="cuda", generator=torch.Generator(device="cuda").manual_seed(5))
        S = S[perm]
        nt = int(0.9 * S.shape[0])
        train_S, test_S = S[:nt].contiguous(), S[nt:].contiguous()
        p = L.init_params(seed=6 + side, side=side)
        l0 = L.grad(test_S, p)[1] / test_S.shape[0]
        L.train(train_S, p, steps=4000, batch=4096, lr=2e-3, seed=7 + side)
        last = L.grad(test_S, p)[1] / test_S.shape[0]
        out.append((side, p, test_S, l0, last))
    return out


def test_trained_network_beats_linear_weights(L, trained):
    for side, p, test_S, l0, last in trained:
        assert last < 0.5 * l0, (side, l0, last)   # held-out loss, starting from the linear weights
        u = test_S[:, :5].contiguous()
        t = test_S[:, 5:].cpu().numpy().astype(np.float64)
        w = L.evaluate(u, p, tensor_cores=True).cpu().numpy().astype(np.float64)
        q = candidates(u.cpu().numpy(), side)
        d = np.array([0.1, 0.6, 0.3]) if side == 0 else np.array([0.3, 0.6, 0.1])
        err_net = np.abs(((w - t) * q).sum(1)).mean()
        err_lin = np.abs(((d[None, :] - t) * q).sum(1)).mean()
        print(f"side {side}: mean |reconstruction - WENO-Z| network {err_net:.3e}, linear weights {err_lin:.3e}, "
              f"gain {err_lin / max(err_net, 1e-300):.1f}x; loss {l0:.3e} -> {last:.3e}")
        assert err_net < 0.5 * err_lin


def test_learned_stencil_run_close_to_fp64(orc, bsn, L, trained):
    L.install(trained[0][1], trained[1][1])
    U, dx = _sedov(orc, 32)
    Ud32, Udl = dev(U), dev(U)
    g, tend = 5 / 3, 0.05
    t = 0.0
    while t < tend:
        dt = min(orc.cfl_dt_3d(U, dx, dx, dx, g, 0.4), tend - t)
        orc.euler3d_step(U, dx, dx, dx, dt, g, rho_floor=1e-6, P_floor=1e-6)
        t += dt
    kw = dict(n_steps=10000, t_end=tend, rho_floor=1e-6, P_floor=1e-6)
    bsn.run_steps(Ud32, 32, 32, 32, dx, dx, dx, g, 0.4, precision="f32", **kw)
    tl, nl = bsn.run_steps(Udl, 32, 32, 32, dx, dx, dx, g, 0.4, precision="learned", **kw)
    assert abs(tl - tend) < 1e-12
    a = (0,) + (slice(NG, -NG),) * 3
    ref = U[a]
    e32 = np.abs(host(Ud32)[a] - ref).sum() / np.abs(ref).sum()
    el = np.abs(host(Udl)[a] - ref).sum() / np.abs(ref).sum()
    print(f"Sedov 32^3 t=0.05 L1(rho) vs FP64: FP32 {e32:.3e}, learned {el:.3e} ({nl} steps)")
    assert np.isfinite(host(Udl)).all()
    assert el < 1e-2
