"""Learned warm start: a convolutional encoder-decoder that maps one diffraction amplitude to the object under the
probe, trained on the GPU by the library's own kernels, and the assembly of its per-position predictions into an
initial object for ePIE / DM / MLs.

No counterpart in the reference, which starts every reconstruction from a constant object (``src/Sample.cpp:216-220``)
or from a user-supplied ``objectNP`` (``src/ptychopy.cpp``); the object made here is handed over exactly like
``objectNP`` (``Session.set_object`` before ``init``).

Network (NCHW float32, 3x3 convolutions with zero padding, ReLU, 2x2 average pooling, 2x nearest upsampling; about
1.15 M parameters at width 16 for 128^2 patterns):

    input  log1p(amplitude), zero frequency centred, x 0.25          1 x N x N
    encoder conv 1->w, 2w, 4w, 8w with a pool after each, conv 8w->16w, 16w->16w at N/16
    decoder up, conv 16w->4w; up, conv 4w->2w; conv 2w->3 at N/4     3 x N/4 x N/4

The three output planes describe the central N/4 x N/4 window of the object patch: amplitude, encoded as
(|O| - 0.9) * 10, and the phase differences phi(i+1,j) - phi(i,j) and phi(i,j+1) - phi(i,j), encoded x 5.  Phase
differences instead of the phase itself because a diffraction pattern does not see the patch's mean phase; the
differences agree between neighbouring positions, and their least-squares integral over the whole scan is one FFT
Poisson solve (``pty_warm_object``).

Everything that computes runs in the library's CUDA kernels through the C ABI (``pty_nn_*``, ``pty_warm_*``,
``pty_simulate``); torch only allocates device memory and orders work on its current stream.
"""
import ctypes

import numpy as np

from . import abi, synth

AMP_MEAN, AMP_SCALE, GRAD_SCALE = 0.9, 0.1, 0.2  # decode: |O| = 0.9 + o * 0.1, difference = o * 0.2
INPUT_SCALE = 0.25


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def layer_plan(N=128, width=16):
    """[(Cin, Cout, H, relu, after)] with H the side at which the convolution runs and after in {pool, up, None}."""
    if N % 16:
        raise ValueError("pattern size must be a multiple of 16")
    w = width
    return [(1, w, N, True, "pool"), (w, 2 * w, N // 2, True, "pool"), (2 * w, 4 * w, N // 4, True, "pool"),
            (4 * w, 8 * w, N // 8, True, "pool"), (8 * w, 16 * w, N // 16, True, None),
            (16 * w, 16 * w, N // 16, True, "up"), (16 * w, 4 * w, N // 8, True, "up"),
            (4 * w, 2 * w, N // 4, True, None), (2 * w, 3, N // 4, False, None)]


class Net:
    """The encoder-decoder with its parameters, gradients and Adam moments in flat device buffers."""

    def __init__(self, N=128, width=16, seed=0, device=None):
        import torch

        self.N, self.width, self.S = N, width, N // 4
        self.plan = layer_plan(N, width)
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        sizes = []
        for cin, cout, *_ in self.plan:
            sizes += [cout * cin * 9, cout]
        self.n_params = int(sum(sizes))
        rng = np.random.default_rng(seed)
        host = np.zeros(self.n_params, np.float32)
        off, self.views = 0, []
        for cin, cout, *_ in self.plan:  # He initialisation, zero biases
            nw = cout * cin * 9
            host[off:off + nw] = rng.standard_normal(nw) * np.sqrt(2.0 / (cin * 9))
            self.views.append((off, off + nw))
            off += nw + cout
        self.params = torch.from_numpy(host).to(self.device)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step_count = 0
        self._bufs, self._bufs_B = None, 0

    # ---- parameter views -------------------------------------------------------------------------------------
    def _w(self, t, l):
        a, b = self.views[l]
        return t[a:b]

    def _b(self, t, l):
        a, b = self.views[l]
        return t[b:b + self.plan[l][1]]

    def state(self):
        return self.params.cpu().numpy().copy()

    def load(self, host):
        import torch

        host = np.ascontiguousarray(host, np.float32)
        if host.size != self.n_params:
            raise ValueError("parameter count differs")
        self.params.copy_(torch.from_numpy(host))

    # ---- activations -----------------------------------------------------------------------------------------
    def _buffers(self, B):
        import torch

        if self._bufs is not None and self._bufs_B >= B:
            return self._bufs
        f = dict(dtype=torch.float32, device=self.device)
        bufs = []
        for cin, cout, H, relu, after in self.plan:
            y = torch.empty((B, cout, H, H), **f)
            post = None
            if after == "pool":
                post = torch.empty((B, cout, H // 2, H // 2), **f)
            elif after == "up":
                post = torch.empty((B, cout, 2 * H, 2 * H), **f)
            gy = torch.empty_like(y)
            gpost = torch.empty_like(post) if post is not None else None
            bufs.append(dict(y=y, post=post, gy=gy, gpost=gpost))
        self._bufs, self._bufs_B = bufs, B
        return bufs

    def forward(self, x, B, out=None):
        """x: device tensor holding B x 1 x N x N inputs (contiguous).  Returns the B x 3 x S x S output view (or writes
        into `out`, a contiguous device tensor with room for B outputs)."""
        L = abi.lib()
        bufs = self._buffers(B)
        st = _stream()
        cur = x
        for l, (cin, cout, H, relu, after) in enumerate(self.plan):
            y = bufs[l]["y"]
            if out is not None and l == len(self.plan) - 1:
                y = out
            abi.check(L.pty_nn_conv3x3(_p(cur), _p(self._w(self.params, l)), _p(self._b(self.params, l)), _p(y), B,
                                       cin, cout, H, H, int(relu), st))
            cur = y
            if after == "pool":
                cur = bufs[l]["post"]
                abi.check(L.pty_nn_pool2(_p(y), _p(cur), B * cout, H // 2, H // 2, st))
            elif after == "up":
                cur = bufs[l]["post"]
                abi.check(L.pty_nn_up2(_p(y), _p(cur), B * cout, H, H, st))
        self._x = x
        if out is not None:
            return out
        return cur[:B]

    def backward(self, g_out, B):
        """Parameter gradients (into self.grads) for the output gradient g_out (B x 3 x S x S) of the last forward."""
        L = abi.lib()
        bufs = self._bufs
        st = _stream()
        g = g_out
        for l in range(len(self.plan) - 1, -1, -1):
            cin, cout, H, relu, after = self.plan[l]
            gy = bufs[l]["gy"]
            if after == "pool":
                abi.check(L.pty_nn_pool2_bwd(_p(g), _p(gy), B * cout, H // 2, H // 2, st))
            elif after == "up":
                abi.check(L.pty_nn_up2_bwd(_p(g), _p(gy), B * cout, H, H, st))
            else:
                gy = g
            if relu:
                abi.check(L.pty_nn_relu_bwd(_p(bufs[l]["y"]), _p(gy), B * cout * H * H, st))
            if l > 0:
                prev = bufs[l - 1]
                x_in = prev["post"] if prev["post"] is not None else prev["y"]
                g_in = prev["gpost"] if prev["gpost"] is not None else prev["gy"]
            else:
                x_in, g_in = self._x, None
            abi.check(L.pty_nn_conv3x3_bwd(_p(x_in), _p(self._w(self.params, l)), _p(gy), _p(g_in),
                                           _p(self._w(self.grads, l)), _p(self._b(self.grads, l)), B, cin, cout, H, H,
                                           st))
            g = g_in

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        abi.check(abi.lib().pty_nn_adam(_p(self.params), _p(self.grads), _p(self.m), _p(self.v), self.n_params, lr,
                                        b1, b2, eps, self.step_count, _stream()))


class TcNet:
    """BF16 tensor-core (tcgen05) inference copy of a trained Net: weights packed once, activations NHWC BF16,
    FP32 accumulation, the output planes in FP32 NCHW like Net.forward."""

    def __init__(self, net):
        import torch

        L = abi.lib()
        self.net, self.plan, self.S, self.N = net, net.plan, net.S, net.N
        self.device = net.device
        self.wpk = []
        st = _stream()
        for l, (cin, cout, *_rest) in enumerate(self.plan):
            n = L.pty_tc_weights_size(cin, cout)
            if n < 0:
                raise ValueError("layer %d not supported by the tensor-core path" % l)
            w = torch.empty(n, dtype=torch.bfloat16, device=self.device)
            abi.check(L.pty_tc_pack_weights(_p(net._w(net.params, l)), cin, cout, _p(w), st))
            self.wpk.append(w)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._bufs, self._bufs_B = None, 0

    def _buffers(self, B):
        import torch

        if self._bufs is not None and self._bufs_B >= B:
            return self._bufs
        f = dict(dtype=torch.bfloat16, device=self.device)
        bufs = []
        for cin, cout, H, relu, after in self.plan[:-1]:
            side = H // 2 if after == "pool" else H  # pooling is fused into the convolution's epilogue
            bufs.append(torch.empty((B, side, side, cout), **f))
        self._bufs, self._bufs_B = bufs, B
        return bufs

    def forward_amp(self, amp, B, out):
        """amp: B x N x N FP32 measured amplitudes (device); out: B x 3 x S x S FP32 (device), written.  The first
        layer reads the amplitudes directly (log1p, centred zero frequency), pooling is fused into the epilogues and
        upsampling into the next layer's loads."""
        L = abi.lib()
        bufs = self._buffers(B)
        st = _stream()
        cur, in_mode = amp, 2
        last = len(self.plan) - 1
        net = self.net
        for l, (cin, cout, H, relu, after) in enumerate(self.plan):
            y = out if l == last else bufs[l]
            if l == 0 and cout == 16 and after == "pool" and relu:  # K = 9: CUDA cores
                abi.check(L.pty_tc_first_layer(_p(cur), _p(net._w(net.params, l)), _p(net._b(net.params, l)), _p(y),
                                               B, cout, H, H, INPUT_SCALE, st))
            elif l == last and cin == 32 and cout <= 4 and in_mode == 0 and not relu and H % 16:  # N = 3: CUDA cores
                # (at H a multiple of 16 the output layer runs on the tensor cores in the shifted-GEMM form)
                abi.check(L.pty_tc_last_layer(_p(cur), _p(net._w(net.params, l)), _p(net._b(net.params, l)), _p(y),
                                              B, cin, cout, H, H, st))
            else:
                out_mode = 1 if l == last else (2 if after == "pool" else 0)
                abi.check(L.pty_tc_conv3x3(_p(cur), _p(self.wpk[l]), _p(net._b(net.params, l)), _p(y), B, cin,
                                           cout, H, H, int(relu), in_mode, out_mode, INPUT_SCALE, _p(self.err), st))
            cur, in_mode = y, (1 if after == "up" else 0)
        return out

    def check(self):
        """Raises if a tensor-core pipeline wait timed out since the last check."""
        e = int(self.err.item())
        if e:
            self.err.zero_()
            raise abi.PtyError(abi.PTY_ERR_CUDA, "tensor-core convolution: pipeline wait timed out (code %d)" % e)


def loss_weight(probe, S):
    """Loss weight of the S x S output window: 0.1 + |P|^2 / max |P|^2 over the window, normalised to mean 1."""
    p = np.asarray(probe)
    if p.ndim == 3:
        p = p[0]
    N = p.shape[0]
    o = (N - S) // 2
    w = np.abs(p[o:o + S, o:o + S]) ** 2
    w = 0.1 + w / w.max()
    return (w / w.mean()).astype(np.float32)


def stitch_weight(probe, S):
    """Stitching weight of the S x S output window: |P|^2 / max |P|^2."""
    p = np.asarray(probe)
    if p.ndim == 3:
        p = p[0]
    N = p.shape[0]
    o = (N - S) // 2
    w = np.abs(p[o:o + S, o:o + S]) ** 2
    return (w / w.max()).astype(np.float32)


def patch_targets(obj, starts, N, S):
    """Encoded targets (P x 3 x S x S float32) of the central S x S windows at integer window starts."""
    o = (N - S) // 2
    out = np.empty((len(starts), 3, S, S), np.float32)
    for k, (r, c) in enumerate(starts):
        win = obj[r + o:r + o + S + 1, c + o:c + o + S + 1].astype(np.complex128)
        a = win[:S, :S]
        out[k, 0] = (np.abs(a) - AMP_MEAN) / AMP_SCALE
        out[k, 1] = np.angle(win[1:, :S] * np.conj(a)) / GRAD_SCALE
        out[k, 2] = np.angle(win[:S, 1:] * np.conj(a)) / GRAD_SCALE
    return out


def simulate_device(obj, probe, pos_px, amp_out):
    """|FFT2(O(pos) P)| into a device tensor amp_out (P x N x N) through pty_simulate."""
    o = np.ascontiguousarray(obj, np.complex64)
    p = np.ascontiguousarray(probe, np.complex64)
    q = np.ascontiguousarray(pos_px, np.float32)
    abi.check(abi.lib().pty_simulate(o.ctypes.data_as(ctypes.c_void_p), o.shape[0], o.shape[1],
                                     p.ctypes.data_as(ctypes.c_void_p), p.shape[0],
                                     q.ctypes.data_as(ctypes.c_void_p), q.shape[0], _p(amp_out)))


def training_set(probe, n_patterns=20480, N=128, nx=64, step=50e-9, lambd=2.48e-10, z=1.0, dx_d=172e-6,
                 photons=1e5, seed=1000, device=None):
    """Network inputs (n x 1 x N x N) and encoded targets (n x 3 x S x S) on the device, from objects of the
    synthetic generator (amplitude uniform in [0.8, 1], phase a Gaussian random field of correlation length 8 px
    over [-pi/2, pi/2]) with seeds seed, seed+1, ...: nx x nx raster scans at integer positions, amplitudes from
    the forward model pty_simulate with Poisson noise at `photons` per pattern, the samples shuffled across scans."""
    import torch

    S = N // 4
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    dx_s = synth.sample_pixel(lambd, z, dx_d, N)
    pos, X, Y = synth.raster_positions(nx, nx, step, step, dx_s, N)
    starts = np.rint(pos).astype(np.int64)
    x = torch.empty((n_patterns, 1, N, N), dtype=torch.float32, device=dev)
    t = np.empty((n_patterns, 3, S, S), np.float32)
    order = np.random.default_rng(seed).permutation(n_patterns)
    amp = torch.empty((len(starts), N, N), dtype=torch.float32, device=dev)
    L = abi.lib()
    k, s = 0, seed
    while k < n_patterns:
        rng = np.random.default_rng(s)
        obj = synth.make_object(X, Y, rng)
        n = min(len(starts), n_patterns - k)
        simulate_device(obj, probe, starts[:n].astype(np.float32), amp[:n])
        g = torch.Generator(device=dev)
        g.manual_seed(int(s))
        I = amp[:n] ** 2
        scale = photons / float(I.sum(dim=(1, 2)).mean())
        noisy = torch.sqrt(torch.poisson(I * scale, generator=g))
        idx = order[k:k + n]
        xs = torch.empty((n, 1, N, N), dtype=torch.float32, device=dev)
        abi.check(L.pty_warm_input(_p(noisy), _p(xs), n, N, INPUT_SCALE, _stream()))
        x[torch.from_numpy(idx).to(dev)] = xs
        t[idx] = patch_targets(obj, starts[:n], N, S)
        k += n
        s += 1
    return x, torch.from_numpy(t).to(dev)


def train(net, x, t, weight, epochs=6, batch=64, lr=1e-3, seed=0, log=None):
    """Adam on the weighted MSE over contiguous minibatches of the (pre-shuffled) set, batch order reshuffled each
    epoch.  Returns the mean loss of every epoch."""
    import torch

    L = abi.lib()
    n = x.shape[0]
    S = net.S
    w = torch.from_numpy(np.ascontiguousarray(weight, np.float32)).to(x.device)
    g = torch.empty((batch, 3, S, S), dtype=torch.float32, device=x.device)
    loss = torch.zeros(len(range(0, n - batch + 1, batch)), dtype=torch.float64, device=x.device)
    rng = np.random.default_rng(seed)
    history = []
    starts = np.arange(0, n - batch + 1, batch)
    for ep in range(epochs):
        for k, s0 in enumerate(rng.permutation(starts)):
            out = net.forward(x[s0:s0 + batch], batch)
            abi.check(L.pty_nn_mse(_p(out), _p(t[s0:s0 + batch]), _p(w), S * S, _p(g), batch * 3 * S * S,
                                   ctypes.c_void_p(loss.data_ptr() + 8 * k), _stream()))
            net.backward(g, batch)
            net.adam(lr)
        history.append(float(loss.mean()))
        if log:
            log(ep, history[-1])
    return history


def predict(net, amp, chunk=256, out=None):
    """Network outputs (P x 3 x S x S device tensor) for the amplitudes amp (P x N x N device tensor); `net` is a
    Net (FP32 CUDA-core kernels) or a TcNet (BF16 tensor cores)."""
    import torch

    L = abi.lib()
    P, N = amp.shape[0], amp.shape[1]
    S = net.S
    if out is None:
        out = torch.empty((P, 3, S, S), dtype=torch.float32, device=amp.device)
    if isinstance(net, TcNet):
        for c0 in range(0, P, chunk):
            cnt = min(chunk, P - c0)
            net.forward_amp(amp[c0:c0 + cnt], cnt, out[c0:c0 + cnt])
        net.check()
        return out
    xb = torch.empty((min(chunk, P), 1, N, N), dtype=torch.float32, device=amp.device)
    for c0 in range(0, P, chunk):
        cnt = min(chunk, P - c0)
        abi.check(L.pty_warm_input(_p(amp[c0:c0 + cnt]), _p(xb), cnt, N, INPUT_SCALE, _stream()))
        net.forward(xb, cnt, out=out[c0:c0 + cnt])
    return out


def assemble(out, pos_px, probe, X, Y, amp, wmin=1e-3, amp_fill=AMP_MEAN):
    """Initial object (X x Y complex64 device tensor) from the network outputs `out` at pixel positions pos_px
    (P x 2, the session's), the probe (N x N) and the measured amplitudes amp (P x N x N device tensor)."""
    import torch

    L = abi.lib()
    dev = out.device
    P, S = out.shape[0], out.shape[2]
    pr = np.asarray(probe, np.complex64)
    if pr.ndim == 3:
        pr = pr[0]
    N = pr.shape[0]
    pos_d = torch.from_numpy(np.ascontiguousarray(pos_px, np.float32)).to(dev)
    w_d = torch.from_numpy(stitch_weight(pr, S)).to(dev)
    pr_d = torch.from_numpy(np.ascontiguousarray(pr).view(np.float32)).to(dev)
    acc = torch.empty((4, X, Y), dtype=torch.float32, device=dev)
    M = 32
    while M < max(X, Y):
        M *= 2
    work = torch.empty(6 * M * M + 4, dtype=torch.float32, device=dev)
    obj = torch.empty((X, Y, 2), dtype=torch.float32, device=dev)
    st = _stream()
    abi.check(L.pty_warm_stitch(_p(out), _p(pos_d), P, _p(w_d), S, N, AMP_MEAN, AMP_SCALE, GRAD_SCALE, _p(acc), X, Y,
                                st))
    abi.check(L.pty_warm_object(_p(acc), X, Y, wmin, amp_fill, _p(pr_d), N, _p(pos_d), P, _p(amp), _p(work), _p(obj),
                                st))
    return obj


def initial_object(net, amp, pos_px, probe, X, Y, chunk=256):
    """predict + assemble: the warm-start object (X x Y complex64, host numpy) for a scan."""
    out = predict(net, amp, chunk=chunk)
    obj = assemble(out, pos_px, probe, X, Y, amp)
    return obj.cpu().numpy().view(np.complex64)[..., 0]
