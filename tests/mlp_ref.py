"""CPU (numpy, FP64) forward and backward of the learned-WENO network, the
checker for the GPU training kernels.  Same layout as include/bsn.h:
W1[32][5] b1[32] W2[32][32] b2[32] W3[3][32] b3[3]; ReLU hidden layers,
softmax output, loss = sum over samples of |softmax(z) - target|^2."""
import numpy as np

NIN, NH, NOUT = 5, 32, 3


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    out = []
    for shape in ((NH, NIN), (NH,), (NH, NH), (NH,), (NOUT, NH), (NOUT,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    return out


def forward(p, U):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    h1 = np.maximum(U @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    z = h2 @ W3.T + b3
    z = z - z.max(axis=1, keepdims=True)
    e = np.exp(z)
    return e / e.sum(axis=1, keepdims=True), (h1, h2)


def loss_and_grad(p, samples):
    samples = np.asarray(samples, dtype=np.float64)
    U, T = samples[:, :NIN], samples[:, NIN:NIN + NOUT]
    W1, b1, W2, b2, W3, b3 = unpack(p)
    w, (h1, h2) = forward(p, U)
    err = w - T
    loss = float((err ** 2).sum())
    g = 2.0 * err
    dz = w * (g - (w * g).sum(axis=1, keepdims=True))
    dW3, db3 = dz.T @ h2, dz.sum(0)
    dh2 = (dz @ W3) * (h2 > 0)
    dW2, db2 = dh2.T @ h1, dh2.sum(0)
    dh1 = (dh2 @ W2) * (h1 > 0)
    dW1, db1 = dh1.T @ U, dh1.sum(0)
    return loss, np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])


def candidates(U, side):
    """Candidate polynomials (q0, q1, q2) of src/weno5.jl:25-61 on stencils U[:,5]."""
    u = np.asarray(U, dtype=np.float64)
    if side == 0:
        return np.stack([u[:, 0] / 3 - 7 * u[:, 1] / 6 + 11 * u[:, 2] / 6,
                         -u[:, 1] / 6 + 5 * u[:, 2] / 6 + u[:, 3] / 3,
                         u[:, 2] / 3 + 5 * u[:, 3] / 6 - u[:, 4] / 6], axis=1)
    return np.stack([-u[:, 0] / 6 + 5 * u[:, 1] / 6 + u[:, 2] / 3,
                     u[:, 1] / 3 + 5 * u[:, 2] / 6 - u[:, 3] / 6,
                     11 * u[:, 2] / 6 - 7 * u[:, 3] / 6 + u[:, 4] / 3], axis=1)
