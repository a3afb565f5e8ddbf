"""The learned constitutive surrogate of law 160: data, training and
inference through the library's CUDA kernels (include/alya_sma.h,
``sma_sur_*``).

The reference has no surrogate; its adjacent hook is the ANN framework's
libtorch forward pass (src/alya-ann/mod_ann_framework.f90:421-446), and the
law the network stands in for is compute_kirchoff_stress
(sld_stress_model_160.f90:212-500).  Everything that computes runs in the
library: the plain-law load paths that make the data (FP64), the BF16
tensor-core forward/backward/weight-gradient pass, Adam, the weight packing
and the tcgen05 inference.  PyTorch only holds the device buffers, shuffles
the sample order and computes the normalisation statistics.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _check, lib

NIN, NOUT, NPARAM, IMAGE_BYTES = 14, 13, 14608, 35904
OFF = dict(W1=0, b1=1024, W2=1088, b2=5184, W3=5248, b3=9344, W4=9408, b4=13504, W5=13568, b5=14592)


class Stats(C.Structure):
    """sma_sur_stats: normalisation and the out-of-envelope gate."""
    _fields_ = [("mu_x", C.c_float * NIN), ("sd_x", C.c_float * NIN), ("mu_y", C.c_float * NOUT),
                ("sd_y", C.c_float * NOUT), ("linv", C.c_float * (NIN * NIN)),
                ("lo_x", C.c_float * NIN), ("hi_x", C.c_float * NIN)]


def _bind():
    L = lib()
    if getattr(L, "_sur_bound", False):
        return L
    vp, i64, i32, f32, f64 = C.c_void_p, C.c_int64, C.c_int32, C.c_float, C.c_double
    L.sma_sur_generate.argtypes = [i64, i32, C.c_uint64, vp, f64, f64, f64, f64, f64, f64, f64, i32, vp, vp, vp]
    L.sma_sur_train_step.argtypes = [vp, vp, vp, i64, vp, vp, vp, vp, vp]
    L.sma_sur_adam.argtypes = [vp, vp, vp, vp, vp, f32, f32, f32, f32, i32, vp]
    L.sma_sur_pack.argtypes = [vp, vp, vp, vp]
    L.sma_sur_forward.argtypes = [vp, vp, i64, vp, vp, vp, vp, vp]
    L.sma_sur_wait_check.argtypes = [i32, C.POINTER(C.c_int32)]
    L._sur_bound = True
    return L


def wait_check(tries=1000):
    """sma_sur_wait_check: 1 if the network kernels' bounded mbarrier wait
    gives up on a phase that never completes (as it must), 0 otherwise."""
    st = C.c_int32(-1)
    _check(_bind().sma_sur_wait_check(int(tries), C.byref(st)))
    return int(st.value)


def generate(props, e_mart, npath, nstep=512, seed=0, spread=0.10, t_range=(300.0, 320.0),
             e_range=(-0.09, 0.06), shear=0.006, nseg=4, device=0, inactive_only=False):
    """Randomised plain-law load paths on the GPU: (x, y) float32 tensors of
    npath * nstep samples (see sma_sur_generate).  inactive_only keeps the
    samples where the law's return map left xS unchanged: the points the
    network stands in for (a transforming point's martensite and
    transformation-strain increments depend on the strain increment, which
    is not an input, and the gate sends such points to the plain law)."""
    import torch
    L = _bind()
    dev = torch.device("cuda", device)
    n = int(npath) * int(nstep)
    x = torch.empty((n, NIN), dtype=torch.float32, device=dev)
    y = torch.empty((n, NOUT), dtype=torch.float32, device=dev)
    p = np.ascontiguousarray(props, dtype=np.float64).reshape(18)
    s = torch.cuda.current_stream(dev).cuda_stream
    _check(L.sma_sur_generate(int(npath), int(nstep), int(seed), p.ctypes.data, float(e_mart), float(spread),
                              float(t_range[0]), float(t_range[1]), float(e_range[0]), float(e_range[1]),
                              float(shear), int(nseg), x.data_ptr(), y.data_ptr(), s))
    if inactive_only:
        keep = y[:, 6] == 0.0
        x, y = x[keep].contiguous(), y[keep].contiguous()
    return x, y


def init_params(seed=0):
    """Uniform initialisation with the fan-in scale of the layer (He et al.,
    ICCV 2015, for ReLU-like units), biases zero; padding zero."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NPARAM, np.float32)

    def fill(off, nout, nin, nin_used, nout_used):
        lim = math.sqrt(6.0 / nin_used)
        blk = rng.uniform(-lim, lim, size=(nout, nin)).astype(np.float32)
        blk[:, nin_used:] = 0.0
        blk[nout_used:, :] = 0.0
        w[off:off + nout * nin] = blk.ravel()

    fill(OFF["W1"], 64, 16, NIN, 64)
    for l in (2, 3, 4):
        fill(OFF[f"W{l}"], 64, 64, 64, 64)
    fill(OFF["W5"], 16, 64, 64, NOUT)
    w[OFF["W5"]:OFF["b5"]] *= 0.5
    return w


class Surrogate:
    """The network's device state: FP32 master weights, their BF16 copy, Adam
    moments, the gradient, the tcgen05 weight image and the statistics."""

    def __init__(self, device=0, seed=0):
        import torch
        self.device = torch.device("cuda", device)
        dev = self.device
        self.w = torch.from_numpy(init_params(seed)).to(dev)
        self.wb = torch.zeros(NPARAM, dtype=torch.int16, device=dev)
        self.m = torch.zeros(NPARAM, dtype=torch.float32, device=dev)
        self.v = torch.zeros(NPARAM, dtype=torch.float32, device=dev)
        self.grad = torch.zeros(NPARAM, dtype=torch.float32, device=dev)
        self.loss = torch.zeros(1, dtype=torch.float32, device=dev)
        # 16-byte aligned weight image (torch allocations are 256-aligned)
        self.img = torch.zeros(IMAGE_BYTES, dtype=torch.uint8, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.stats_host = Stats()
        self.stats = torch.zeros(C.sizeof(Stats), dtype=torch.uint8, device=dev)
        self.t = 0
        self.history = []
        self.pack()

    @property
    def _s(self):
        import torch
        return torch.cuda.current_stream(self.device).cuda_stream

    # -- statistics ---------------------------------------------------------
    def fit_stats(self, x, y):
        """Per-feature mean and standard deviation of inputs and outputs, and
        the inverse Cholesky factor of the normalised inputs' covariance."""
        import torch
        xd, yd = x.double(), y.double()
        mx, sx = xd.mean(0), xd.std(0).clamp_min(1e-12)
        # an output that is constant in the data (the xS increment of
        # inactive points) keeps a unit of 1e-6, so the network's noise on it
        # stays far below the gate's tolerance
        my, sy = yd.mean(0), yd.std(0).clamp_min(1e-6)
        # The transformation-strain increment of an inactive point is its
        # direction turning with the step's strain increment: a few 1e-3 of
        # eps_tr, below what BF16 activations resolve, so its six outputs
        # weigh 1e-2 in the loss (a unit 10x their spread) and the stress,
        # which they would otherwise swamp, is learned to its target.
        sy[7:13] *= 10.0
        xh = (xd - mx) / sx
        cov = (xh.T @ xh) / (xh.shape[0] - 1)
        cov = cov + 1e-9 * torch.eye(NIN, dtype=torch.float64, device=cov.device)
        Lc = np.linalg.cholesky(cov.cpu().numpy())
        Linv = np.linalg.inv(Lc)
        st = self.stats_host
        for arr, src in ((st.mu_x, mx), (st.sd_x, sx), (st.mu_y, my), (st.sd_y, sy)):
            v = src.cpu().numpy()
            for i in range(len(arr)):
                arr[i] = float(v[i])
        lv = Linv.astype(np.float32).ravel()
        for i in range(NIN * NIN):
            st.linv[i] = float(lv[i])
        lo, hi = x.min(0).values.cpu().numpy(), x.max(0).values.cpu().numpy()
        for i in range(NIN):
            st.lo_x[i], st.hi_x[i] = float(lo[i]), float(hi[i])
        self._upload_stats()

    def _upload_stats(self):
        import torch
        raw = bytes(self.stats_host)
        self.stats.copy_(torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(self.device))

    def stats_array(self):
        """mu_x, sd_x, mu_y, sd_y as one float64 array (the oracle's layout)."""
        st = self.stats_host
        return np.concatenate([np.array(st.mu_x[:]), np.array(st.sd_x[:]), np.array(st.mu_y[:]),
                               np.array(st.sd_y[:])]).astype(np.float64)

    def linv(self):
        return np.array(self.stats_host.linv[:], dtype=np.float64).reshape(NIN, NIN)

    # -- training -----------------------------------------------------------
    def pack(self):
        _check(_bind().sma_sur_pack(self.w.data_ptr(), self.wb.data_ptr(), self.img.data_ptr(), self._s))

    def gradient(self, x, y):
        """(loss, gradient) of one batch from the tensor-core training kernel."""
        self.grad.zero_()
        self.loss.zero_()
        _check(_bind().sma_sur_train_step(self.wb.data_ptr(), self.w.data_ptr(), self.stats.data_ptr(),
                                          int(x.shape[0]), x.data_ptr(), y.data_ptr(), self.grad.data_ptr(),
                                          self.loss.data_ptr(), self._s))
        return float(self.loss.item()), self.grad.cpu().numpy()

    def train(self, x, y, epochs=4, batch=8192, lr=2e-3, lr_end=1e-4, b1=0.9, b2=0.999, eps=1e-8, seed=0):
        """Adam over shuffled batches (cosine learning-rate decay from lr to
        lr_end); returns the mean training loss of each epoch."""
        import torch
        L = _bind()
        n = x.shape[0]
        nb = (n + batch - 1) // batch
        total = epochs * nb
        gen = torch.Generator(device=self.device)
        gen.manual_seed(seed)
        s = self._s
        losses = []
        step = 0
        for ep in range(epochs):
            perm = torch.randperm(n, device=self.device, generator=gen)
            xs, ys = x[perm].contiguous(), y[perm].contiguous()
            acc = torch.zeros(1, dtype=torch.float32, device=self.device)
            for b in range(nb):
                lo, hi = b * batch, min(n, (b + 1) * batch)
                self.grad.zero_()
                self.loss.zero_()
                _check(L.sma_sur_train_step(self.wb.data_ptr(), self.w.data_ptr(), self.stats.data_ptr(),
                                            hi - lo, xs[lo:hi].data_ptr(), ys[lo:hi].data_ptr(),
                                            self.grad.data_ptr(), self.loss.data_ptr(), s))
                acc += self.loss
                self.t += 1
                step += 1
                lr_t = lr_end + 0.5 * (lr - lr_end) * (1.0 + math.cos(math.pi * step / total))
                _check(L.sma_sur_adam(self.w.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
                                      self.grad.data_ptr(), self.wb.data_ptr(), float(lr_t), float(b1),
                                      float(b2), float(eps), int(self.t), s))
            losses.append(float(acc.item()) / nb)
        self.history += losses
        self.pack()
        return losses

    # -- inference ----------------------------------------------------------
    def forward(self, x):
        """The network on the tcgen05 tensor cores: raw outputs (n, 13) and
        the out-of-envelope score (n,)."""
        import torch
        n = x.shape[0]
        y = torch.empty((n, NOUT), dtype=torch.float32, device=self.device)
        sc = torch.empty(n, dtype=torch.float32, device=self.device)
        self.status.zero_()
        _check(_bind().sma_sur_forward(self.img.data_ptr(), self.stats.data_ptr(), int(n), x.contiguous().data_ptr(),
                                       y.data_ptr(), sc.data_ptr(), self.status.data_ptr(), self._s))
        if int(self.status.item()) != 0:
            raise RuntimeError("surrogate forward: a wait for the tensor cores ran out")
        return y, sc

    def params(self):
        return self.w.cpu().numpy()

    def params_bf16(self):
        """The master weights rounded to BF16 as the tensor cores see them
        (biases stay FP32)."""
        import torch
        w = self.w.clone()
        wb = w.to(torch.bfloat16).float()
        for l in (1, 2, 3, 4, 5):
            a, b = OFF[f"W{l}"], OFF[f"b{l}"]
            w[a:b] = wb[a:b]
        return w.cpu().numpy()


class ZeroResidual:
    """The surrogate's element loop with the network's output held at zero:
    the analytic part alone (the law's elastic response on a third-order
    logarithmic strain), with the same gates and plain-law fallback -- the
    method without the learned part, for comparisons.  It keeps a trained
    network's statistics (input box and envelope), so the same points go to
    the plain law; zero weights and a zero output mean make every stress
    residual and predicted martensite increment zero."""

    def __init__(self, net):
        self.stats_host = Stats.from_buffer_copy(bytes(net.stats_host))
        for i in range(7):
            self.stats_host.mu_y[i] = 0.0

    def params(self):
        return np.zeros(NPARAM, np.float32)


def training_setup(prob):
    """The generator's material, spread and temperature range for a problem:
    the mean of its per-element materials (sampled symmetrically around a
    base), their largest relative spread, and its temperature range."""
    props = np.atleast_2d(prob.props)
    base = props.mean(axis=0)
    em = float(np.mean(prob.e_mart)) if prob.e_mart is not None else 0.0
    spread = 0.0
    if len(props) > 1:
        for k in (0, 2, 3, 4, 9, 10):
            if base[k] != 0.0:
                spread = max(spread, float(np.abs(props[:, k] / base[k] - 1.0).max()))
    t = (float(np.min(prob.tempe)), float(np.max(prob.tempe))) if prob.tempe is not None else (0.0, 0.0)
    return base, em, spread, t


def train_for(prob, nsamples=20_000_000, epochs=4, seed=0, device=0, batch=8192, lr=3e-3):
    """Generate nsamples plain-law samples for the problem's materials (the
    inactive ones kept), fit the statistics, train; returns (net, info)."""
    import time
    import torch
    base, em, spread, t = training_setup(prob)
    nstep = 256
    npath = max(1, nsamples // nstep)
    t0 = time.perf_counter()
    x, y = generate(base, em, npath, nstep=nstep, seed=seed, spread=spread, t_range=t, device=device,
                    inactive_only=True)
    torch.cuda.synchronize(device)
    t1 = time.perf_counter()
    net = Surrogate(device=device, seed=seed + 1)
    net.fit_stats(x, y)
    losses = net.train(x, y, epochs=epochs, batch=batch, lr=lr, seed=seed)
    torch.cuda.synchronize(device)
    t2 = time.perf_counter()
    info = {"samples_generated": npath * nstep, "samples_kept_inactive": int(x.shape[0]), "epochs": epochs,
            "batch": batch, "loss_per_epoch": [round(v, 6) for v in losses],
            "generate_s": round(t1 - t0, 3), "train_s": round(t2 - t1, 3),
            "material_spread": spread, "temperature_range": list(t)}
    del x, y
    return net, info
