"""Training the soft-shadow denoiser on the library's own kernels.

`Trainer` wraps the rt_dn_train_* entry points: FP32 master weights and Adam
moments on the device, the forward pass on the inference kernels, weight
gradients as tcgen05 implicit GEMMs and data gradients as transposed
convolutions on the same kernels (rtrace_b200/csrc/dn_train.cu).  PyTorch
only holds the training set in device memory and draws the batches.
"""
import ctypes
import math
import time

import numpy as np

from . import _capi, denoiser


class Trainer:
    """Training state for batches of `planes` feature images of height x
    width, starting from a Net (version 3: visibility and error outputs)."""

    def __init__(self, ctx, net, planes, height, width):
        self.ctx = ctx
        self.net = net
        self.shape = (planes, height, width)
        blob = denoiser.pack_net(net)
        buf = ctypes.create_string_buffer(blob, len(blob))
        h = ctypes.c_void_p()
        L = _capi.lib()
        st = L.rt_dn_train_create(ctx.handle, buf, len(blob), planes, height, width, ctypes.byref(h))
        if st != _capi.RT_OK:
            from . import _raise
            _raise(st, ctx.handle)
        self.handle = h

    def _check(self, st):
        if st != _capi.RT_OK:
            from . import _raise
            _raise(st, self.ctx.handle)

    def _args(self, feats, targs):
        if tuple(feats.shape) != self.shape + (denoiser.FEAT_CHANNELS,) or feats.dtype.itemsize != 2:
            raise ValueError("features must be FP16 of shape %s" % ((self.shape + (16,)),))
        if tuple(targs.shape) != (self.shape[0], 2) + self.shape[1:] or targs.dtype.itemsize != 2:
            raise ValueError("targets must be FP16 of shape %s" % (((self.shape[0], 2) + self.shape[1:]),))
        if not (feats.is_contiguous() and targs.is_contiguous()):
            raise ValueError("features and targets must be contiguous")
        return feats.data_ptr(), targs.data_ptr()

    def step(self, feats, targs, lr, beta1=0.9, beta2=0.999, eps=1e-8, want_loss=False):
        """One Adam step on a batch (device tensors).  With want_loss, returns
        (masked count, visibility loss sum, error loss sum, non-finite
        gradient entries: the step was skipped when this is not 0)."""
        f, t = self._args(feats, targs)
        loss = (ctypes.c_float * 4)() if want_loss else None
        self._check(_capi.lib().rt_dn_train_step(self.handle, f, t, lr, beta1, beta2, eps, loss))
        return tuple(loss) if want_loss else None

    def grads(self, feats, targs):
        """(per convolution (dW [cout][3][3][cin], db [cout]) of the summed
        loss, (count, visibility loss, error loss)) without an update."""
        f, t = self._args(feats, targs)
        n = sum(w.size + b.size for w, b in self.net.params)
        g = np.zeros(n, np.float32)
        loss = (ctypes.c_float * 3)()
        self._check(_capi.lib().rt_dn_train_grads(self.handle, f, t, g.ctypes.data, loss))
        out, k = [], 0
        for w, b in self.net.params:
            dw = g[k:k + w.size].reshape(w.shape)
            k += w.size
            out.append((dw, g[k:k + b.size].copy()))
            k += b.size
        return out, tuple(loss)

    def export(self, threshold=None):
        """The current weights as a Net."""
        L = _capi.lib()
        if threshold is not None:
            self._check(L.rt_dn_train_set_threshold(self.handle, float(threshold)))
        n = ctypes.c_size_t(0)
        self._check(L.rt_dn_train_export(self.handle, None, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        self._check(L.rt_dn_train_export(self.handle, buf, ctypes.byref(n)))
        return denoiser.unpack_net(buf.raw[:n.value])

    def close(self):
        if self.handle:
            _capi.lib().rt_dn_train_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fit_native(ctx, net, feats, targs, iters=8000, batch=16, lr=1e-3, seed=0, log=print):
    """Adam on the library's training kernels with a one-cycle learning-rate
    schedule (5% warm-up, cosine decay); returns the fitted Net."""
    import torch
    crop = feats.shape[1]
    tr = Trainer(ctx, net, batch, crop, crop)
    g = torch.Generator(device="cpu").manual_seed(seed)
    warm = max(1, int(0.05 * iters))
    t0 = time.time()
    for it in range(iters):
        if it < warm:
            a = lr * (0.04 + 0.96 * it / warm)
        else:
            a = lr * (1e-4 + 0.5 * (1 - 1e-4) * (1 + math.cos(math.pi * (it - warm) / max(1, iters - warm))))
        idx = torch.randint(0, feats.shape[0], (batch,), generator=g).to(feats.device)
        fb = feats[idx].contiguous()
        tb = targs[idx].contiguous()
        torch.cuda.synchronize(feats.device)  # the batch is gathered on torch's stream
        report = it % 500 == 0 or it == iters - 1
        loss = tr.step(fb, tb, a, want_loss=report)
        if report:
            cnt, lv, lc, bad = loss
            log("iter %d loss %.6f vis-mse %.6f%s (%.1f s, native kernels)" %
                (it, (lv + lc) / max(cnt, 1), lv / max(cnt, 1), " (step skipped: non-finite gradient)" if bad else "",
                 time.time() - t0))
    out = tr.export()
    tr.close()
    return out
