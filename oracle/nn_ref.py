"""CPU restatement (numpy, float64) of the warm-start network's layers -- test infrastructure only.

Checks the CUDA kernels of ptychopy_b200/csrc/kernels_nn.cu: 3x3 convolution (stride 1, zero padding 1) with its
data and weight gradients, ReLU, 2x2 average pooling, 2x nearest upsampling, mean-squared error.  Its own gradients
are checked against finite differences in tests/test_nn.py."""
import numpy as np


def conv3x3(x, w, b=None):
    """x (B, Cin, H, W), w (Cout, Cin, 3, 3) -> (B, Cout, H, W)."""
    B, Cin, H, W = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    y = np.zeros((B, w.shape[0], H, W))
    for ky in range(3):
        for kx in range(3):
            y += np.einsum("oc,bchw->bohw", w[:, :, ky, kx], xp[:, :, ky:ky + H, kx:kx + W])
    if b is not None:
        y += b[None, :, None, None]
    return y


def conv3x3_bwd(x, w, dy):
    """(dx, dw, db) of conv3x3 for the output gradient dy."""
    B, Cin, H, W = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    dw = np.zeros_like(w)
    dxp = np.zeros_like(xp)
    for ky in range(3):
        for kx in range(3):
            dw[:, :, ky, kx] = np.einsum("bohw,bchw->oc", dy, xp[:, :, ky:ky + H, kx:kx + W])
            dxp[:, :, ky:ky + H, kx:kx + W] += np.einsum("oc,bohw->bchw", w[:, :, ky, kx], dy)
    return dxp[:, :, 1:-1, 1:-1], dw, dy.sum(axis=(0, 2, 3))


def relu(a):
    return np.maximum(a, 0)


def relu_bwd(y, g):
    return np.where(y > 0, g, 0.0)


def pool2(x):
    B, C, H, W = x.shape
    return x.reshape(B, C, H // 2, 2, W // 2, 2).mean(axis=(3, 5))


def pool2_bwd(dy):
    return np.repeat(np.repeat(dy, 2, axis=2), 2, axis=3) / 4.0


def up2(x):
    return np.repeat(np.repeat(x, 2, axis=2), 2, axis=3)


def up2_bwd(dy):
    B, C, H2, W2 = dy.shape
    return dy.reshape(B, C, H2 // 2, 2, W2 // 2, 2).sum(axis=(3, 5))


def mse(p, t):
    d = p - t
    return float(np.mean(d * d)), 2.0 * d / d.size


def adam(p, g, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One bias-corrected Adam step (Kingma & Ba, 2015); returns the new (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v


# ---- warm-start assembly (ptychopy_b200/csrc/kernels_warm.cu) ----------------------------------------------------

def warm_input(amp, scale):
    """scale * log1p(amplitude) with the zero frequency moved to the centre (even N)."""
    return scale * np.log1p(np.fft.fftshift(np.asarray(amp, np.float64), axes=(-2, -1)))


def warm_stitch(out, pos, weight, N, X, Y, amp_mean, amp_scale, grad_scale):
    """(4, X, Y) probe-weighted sums of the decoded outputs of the central S x S windows at rounded positions."""
    P, _, S, _ = out.shape
    off = (N - S) // 2
    acc = np.zeros((4, X, Y))
    for p in range(P):
        r0 = int(np.rint(np.float32(pos[p, 0]))) + off
        c0 = int(np.rint(np.float32(pos[p, 1]))) + off
        i0, i1 = max(r0, 0), min(r0 + S, X)
        j0, j1 = max(c0, 0), min(c0 + S, Y)
        if i0 >= i1 or j0 >= j1:
            continue
        w = weight[i0 - r0:i1 - r0, j0 - c0:j1 - c0]
        o = out[p, :, i0 - r0:i1 - r0, j0 - c0:j1 - c0].astype(np.float64)
        acc[0, i0:i1, j0:j1] += w * (amp_mean + o[0] * amp_scale)
        acc[1, i0:i1, j0:j1] += w * o[1] * grad_scale
        acc[2, i0:i1, j0:j1] += w * o[2] * grad_scale
        acc[3, i0:i1, j0:j1] += w
    return acc


def warm_object(acc, wmin, amp_fill, probe, pos, amp):
    """Object from the stitched sums: weighted mean amplitude, least-squares integral of the mean forward phase
    differences on the periodic M x M grid (M the power of two >= max(X, Y), at least 32), then the energy match
    sum_p sum |P O_p|^2 N^2 = sum amp^2 (rounded positions, window clamped to the object)."""
    _, X, Y = acc.shape
    M = 32
    while M < max(X, Y):
        M *= 2
    ws = acc[3]
    cov = ws > wmin
    gx = np.zeros((M, M))
    gy = np.zeros((M, M))
    gx[:X, :Y][cov] = acc[1][cov] / ws[cov]
    gy[:X, :Y][cov] = acc[2][cov] / ws[cov]
    u = np.arange(M)
    dx = (np.exp(2j * np.pi * u / M) - 1)[:, None]
    dy = (np.exp(2j * np.pi * u / M) - 1)[None, :]
    den = np.abs(dx) ** 2 + np.abs(dy) ** 2
    num = np.conj(dx) * np.fft.fft2(gx) + np.conj(dy) * np.fft.fft2(gy)
    spec = np.where(den > 0, num / np.where(den > 0, den, 1), 0)
    phi = np.real(np.fft.ifft2(spec))[:X, :Y]
    A = np.where(cov, acc[0] / np.where(cov, ws, 1), amp_fill)
    obj = A * np.exp(1j * phi)
    N = probe.shape[0]
    pw = np.abs(probe.astype(np.complex128)) ** 2
    model = 0.0
    ii = np.arange(N)
    for p in range(pos.shape[0]):
        r0 = int(np.rint(np.float32(pos[p, 0])))
        c0 = int(np.rint(np.float32(pos[p, 1])))
        ri = np.clip(r0 + ii, 0, X - 1)
        ci = np.clip(c0 + ii, 0, Y - 1)
        model += float((pw * np.abs(obj[np.ix_(ri, ci)]) ** 2).sum())
    data = float((np.asarray(amp, np.float64) ** 2).sum())
    k = np.sqrt(data / (model * N * N)) if model > 0 else 1.0
    return obj * k
