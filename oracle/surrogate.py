"""CPU reference (FP64 numpy) of the learned dipolar surrogate's network,
forward and backward.  Test infrastructure only: the surrogate has no
counterpart in the reference (it stands in for the LongRange convolution of
M/cpu/longrange/spinoperationlongrange.cpp:354-440 between exact
evaluations), so this module states the network the CUDA kernels evaluate
and is the oracle for their outputs and gradients.

Layout: x has shape (3, nx*ny*nz) in SpinSystem order (x fastest, then y,
then z); channel ch = c * nz + z on the in-plane grid (ny, nx).

  out[co](s) = sum_{o, ci} W[o, co, ci] X[ci](s + o)                 o = (dy, dx), |dy|,|dx| <= rad,
                                                                     index o = (dy + rad) (2 rad + 1) + dx + rad
             + Re( ifft2( S ) )[co](s),  S[co, ky_j, kx] = w_kx sum_ci R[kx, j, co, ci] fft2(X)[ci, ky_j, kx]
with kx < mx, ky_j = j (j < my/2) or ny - my + j, w_0 = 1, w_kx = 2 otherwise,
periodic in x and y.
"""
import numpy as np


def ky_list(ny, my):
    return [j if j < my // 2 else ny - my + j for j in range(my)]


def to_channels(v, dims):
    nx, ny, nz = dims
    return np.asarray(v, dtype=np.float64).reshape(3, nz, ny, nx).reshape(3 * nz, ny, nx)


def from_channels(X, dims):
    nx, ny, nz = dims
    return X.reshape(3, nz, ny, nx).reshape(3, nx * ny * nz)


def _shift(A, dy, dx):
    # A(s + o) for every s, periodic
    return np.roll(A, (-dy, -dx), axis=(-2, -1))


def forward(x, W, R, dims, mx, my, rad):
    """x (3, n); W (dia^2, C, C); R complex (mx, my, C, C) -> dH (3, n)."""
    X = to_channels(x, dims)
    C, ny, nx = X.shape
    dia = 2 * rad + 1
    out = np.zeros_like(X)
    for o in range(dia * dia):
        dy, dx = o // dia - rad, o % dia - rad
        out += np.einsum('ab,byx->ayx', W[o], _shift(X, dy, dx))
    Xh = np.fft.fft2(X)
    S = np.zeros_like(Xh)
    for kx in range(mx):
        w = 1.0 if kx == 0 else 2.0
        for j, ky in enumerate(ky_list(ny, my)):
            S[:, ky, kx] += w * (R[kx, j] @ Xh[:, ky, kx])
    out += np.real(np.fft.ifft2(S))
    return from_channels(out, dims)


def gradients(x, G, dims, mx, my, rad):
    """dL/dW and dL/dR for dL/dout = G (3, n); R's gradient as complex
    (d/dRe + i d/dIm)."""
    X = to_channels(x, dims)
    Gc = to_channels(G, dims)
    C, ny, nx = X.shape
    dia = 2 * rad + 1
    dW = np.zeros((dia * dia, C, C))
    for o in range(dia * dia):
        dy, dx = o // dia - rad, o % dia - rad
        dW[o] = np.einsum('ayx,byx->ab', Gc, _shift(X, dy, dx))
    Xh = np.fft.fft2(X)
    Gh = np.fft.fft2(Gc)
    dR = np.zeros((mx, my, C, C), complex)
    for kx in range(mx):
        w = (1.0 if kx == 0 else 2.0) / (nx * ny)
        for j, ky in enumerate(ky_list(ny, my)):
            dR[kx, j] = w * np.outer(Gh[:, ky, kx], np.conj(Xh[:, ky, kx]))
    return dW, dR


def loss_and_gradients(x, t, W, R, dims, mx, my, rad, pred=None):
    """L = |P - t|^2 / |t|^2 with P = forward(x) (or the given prediction)."""
    P = forward(x, W, R, dims, mx, my, rad) if pred is None else np.asarray(pred, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    st = float(np.sum(t * t))
    G = 2.0 * (P - t) / st
    dW, dR = gradients(x, G, dims, mx, my, rad)
    return float(np.sum((P - t) ** 2) / st), dW, dR, P
