"""The learned RVE surrogate (include/akb_fe2.h: akb_mlp_*).

MLPSurrogate maps a macroscopic displacement gradient H to the homogenised
first Piola-Kirchhoff stress P with a SiLU perceptron (3 hidden layers of
256) whose GEMMs run on the tensor cores (tcgen05, BF16 operands, FP32
accumulation). Training, gradients and inference all run in libakb.so; torch
only holds the device arrays. Tensors are (nb, 3, 3) with [b, i, j] =
du_i/dX_j (inputs) or P_ij (outputs); features are their column-major
flattening, the library's layout of grad_u and stress.

Features: with r = |H| (Frobenius), the network reads (H / r, log r) (10
inputs) and predicts P / r (9 outputs), so P = r net(H / r, log r). P is
homogeneous of degree 1 in H at small strain, so this keeps the relative
error uniform from r = 1e-4 to the envelope's edge (a network on raw H has
an absolute error floor that dominates small-strain stresses).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib
from .model import torch_stream


def _torch():
    import torch
    return torch


R_MIN = 1e-8


def _flat(t, torch):
    """(nb, 3, 3) -> (nb, 9) column-major features, FP64, contiguous."""
    return t.reshape(-1, 3, 3).transpose(1, 2).reshape(-1, 9).to(torch.float64).contiguous()


def scaled_features(h, p=None):
    """(nb, 9) column-major H (and P) -> network inputs (nb, 10) = (H / r,
    log r) and targets P / r, r = |H| clamped to R_MIN."""
    import torch
    r = torch.linalg.norm(h, dim=1, keepdim=True).clamp_min(R_MIN)
    x = torch.cat([h / r, torch.log(r)], dim=1).contiguous()
    return (x, None) if p is None else (x, (p / r).contiguous())


class MLPSurrogate:
    def __init__(self, nb_inputs=10, nb_outputs=9, width=256, nb_hidden=3, device=0, seed=0):
        self.shape = (nb_inputs, nb_outputs, width, nb_hidden)
        self.device = device
        h = C.c_void_p()
        # on torch's stream, so the device arrays torch fills are ordered with it
        check(lib().akb_mlp_create(nb_inputs, nb_outputs, width, nb_hidden, device,
                                   torch_stream(device), C.byref(h)))
        self._h = h
        n = C.c_int64()
        check(lib().akb_mlp_get_parameter_count(h, C.byref(n)))
        self.nb_parameters = n.value
        self.scaling = dict(in_shift=np.zeros(nb_inputs, np.float32),
                            in_scale=np.ones(nb_inputs, np.float32),
                            out_shift=np.zeros(nb_outputs, np.float32),
                            out_scale=np.ones(nb_outputs, np.float32))
        self.set_parameters(self.initial_parameters(seed))

    def close(self):
        if getattr(self, "_h", None):
            lib().akb_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def layer_shapes(self):
        nin, nout, w, nh = self.shape
        return [(w if l else nin, nout if l == nh else w) for l in range(nh + 1)]

    def initial_parameters(self, seed):
        """Uniform +-sqrt(6 / (fan_in + fan_out)) weights (Glorot & Bengio
        2010), zero biases."""
        rng = np.random.default_rng(seed)
        out = []
        for k, n in self.layer_shapes():
            a = np.sqrt(6.0 / (k + n))
            out += [rng.uniform(-a, a, n * k), np.zeros(n)]
        return np.concatenate(out).astype(np.float32)

    def set_parameters(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib().akb_mlp_set_parameters(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))

    def get_parameters(self):
        p = np.zeros(self.nb_parameters, np.float32)
        check(lib().akb_mlp_get_parameters(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))
        return p

    def set_scaling(self, in_shift, in_scale, out_shift, out_scale):
        s = {k: np.ascontiguousarray(v, dtype=np.float32) for k, v in
             dict(in_shift=in_shift, in_scale=in_scale, out_shift=out_shift,
                  out_scale=out_scale).items()}
        nin, nout = self.shape[0], self.shape[1]
        if any(s[k].shape != (nin,) for k in ("in_shift", "in_scale")) or \
                any(s[k].shape != (nout,) for k in ("out_shift", "out_scale")):
            raise ValueError("scaling needs %d input and %d output entries" % (nin, nout))
        F = C.POINTER(C.c_float)
        check(lib().akb_mlp_set_scaling(self._h, *[s[k].ctypes.data_as(F) for k in
                                                   ("in_shift", "in_scale", "out_shift",
                                                    "out_scale")]))
        self.scaling = s

    def fit_scaling(self, x, y):
        """Per-feature shift/scale from training data ((nb, d) FP64 features)."""
        x = np.asarray(x)
        y = np.asarray(y)
        xs = x.std(0)
        ys = y.std(0)
        self.set_scaling(x.mean(0), 1.0 / np.where(xs > 0, xs, 1.0), y.mean(0),
                         np.where(ys > 0, ys, 1.0))

    # -- device features (nb, d) FP64 --------------------------------------
    def forward_features(self, x, stream=None):
        torch = _torch()
        x = x.to(torch.float64).contiguous()
        y = torch.empty((x.shape[0], self.shape[1]), dtype=torch.float64, device=x.device)
        s = stream if stream is not None else torch_stream(x.device)
        check(lib().akb_mlp_forward(self._h, x.shape[0], x.data_ptr(), y.data_ptr(), s))
        return y

    def gradients_features(self, x, t):
        torch = _torch()
        torch.cuda.synchronize()
        g = np.zeros(self.nb_parameters, np.float32)
        loss = C.c_float()
        check(lib().akb_mlp_gradients(self._h, x.shape[0], x.data_ptr(), t.data_ptr(),
                                      g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)))
        return loss.value, g

    def train_step_features(self, x, t, lr):
        loss = C.c_float()
        check(lib().akb_mlp_train_step(self._h, x.shape[0], x.data_ptr(), t.data_ptr(),
                                       float(lr), C.byref(loss)))
        return loss.value

    # -- data-parallel halves of a training step (akb_mlp_compute_gradients,
    #    akb_mlp_apply_gradients) ------------------------------------------
    def compute_gradients(self, x, t):
        """Gradient of the mean loss over (x, t) into the network's device
        gradient array (gradient_tensor); returns the loss."""
        loss = C.c_float()
        check(lib().akb_mlp_compute_gradients(self._h, x.shape[0], x.data_ptr(), t.data_ptr(),
                                              C.byref(loss)))
        return loss.value

    def gradient_tensor(self):
        """Zero-copy float32 torch view of the device gradient array."""
        torch = _torch()
        ptr = C.c_void_p()
        check(lib().akb_mlp_gradient_device_pointer(self._h, C.byref(ptr)))

        class _Cai:
            __cuda_array_interface__ = dict(shape=(self.nb_parameters,), typestr="<f4",
                                            data=(int(ptr.value), False), version=3,
                                            strides=None, stream=None)
        return torch.as_tensor(_Cai(), device="cuda:%d" % self.device)

    def apply_gradients(self, lr):
        check(lib().akb_mlp_apply_gradients(self._h, float(lr)))

    def train(self, x, t, epochs=20, batch=4096, lr=1e-3, lr_final=1e-5, seed=0, log=None,
              group=None):
        """Adam over shuffled minibatches with a cosine-decayed learning
        rate; x, t device (nb, d) FP64 features. Returns the epoch losses.
        With a torch.distributed group of several processes (one GPU each,
        every rank holding the same x and t), each minibatch is split over
        the ranks and their gradients averaged (data_parallel_train)."""
        torch = _torch()
        import torch.distributed as dist
        if group is not None or (dist.is_available() and dist.is_initialized()
                                 and dist.get_world_size() > 1):
            return data_parallel_train(self, x, t, epochs, batch, lr, lr_final, seed, log, group)
        torch.cuda.synchronize()
        n = x.shape[0]
        g = torch.Generator(device=x.device)
        g.manual_seed(seed)
        steps = epochs * max(1, n // batch)
        k = 0
        losses = []
        for ep in range(epochs):
            perm = torch.randperm(n, device=x.device, generator=g)
            tot = 0.0
            nbat = max(1, n // batch)
            for b in range(nbat):
                idx = perm[b * batch:(b + 1) * batch]
                xb = x[idx].contiguous()
                tb = t[idx].contiguous()
                lr_k = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * k / steps))
                tot += self.train_step_features(xb, tb, lr_k)
                k += 1
            losses.append(tot / nbat)
            if log:
                log("epoch %d loss %.3e" % (ep, losses[-1]))
        return losses

    # -- stresses ------------------------------------------------------------
    def predict_flat(self, h, stream=None):
        """(nb, 9) column-major H -> (nb, 9) column-major P."""
        torch = _torch()
        if self.shape[0] == 9:  # raw features
            return self.forward_features(h, stream)
        x, _ = scaled_features(h)
        r = torch.linalg.norm(h, dim=1, keepdim=True)
        return r * self.forward_features(x, stream)

    def stress_into(self, grad_u, stress, envelope=None, fallback=None, stream=None):
        """MaterialFE2's stress map in one launch (akb_mlp_stress): grad_u and
        stress are contiguous (nb, 9) FP64 device tensors, column-major per
        point; stress <- |H| net(H / r, log r). With envelope = (amplitude,
        min_det) and fallback = (index (nb,) int32, count (1,) int32) device
        tensors, the points outside the envelope are listed in index[:count]
        (no host round trip)."""
        torch = _torch()
        for t in (grad_u, stress):
            if t.dtype != torch.float64 or not t.is_contiguous() or t.shape[-1] != 9:
                raise ValueError("grad_u and stress must be contiguous (nb, 9) float64 tensors")
        amp, det = envelope if envelope is not None else (0.0, 0.0)
        idx, cnt = fallback if fallback is not None else (None, None)
        s = stream if stream is not None else torch_stream(grad_u.device)
        check(lib().akb_mlp_stress(self._h, grad_u.shape[0], grad_u.data_ptr(), stress.data_ptr(),
                                   float(amp), float(det),
                                   idx.data_ptr() if idx is not None else None,
                                   cnt.data_ptr() if cnt is not None else None, s))
        return stress

    def __call__(self, grad_u, stream=None):
        torch = _torch()
        y = self.predict_flat(_flat(torch.as_tensor(grad_u), torch), stream)
        return y.reshape(-1, 3, 3).transpose(1, 2)

    def save(self, path):
        np.savez(path, params=self.get_parameters(), shape=np.array(self.shape), **self.scaling)

    @classmethod
    def load(cls, path, device=0):
        d = np.load(path)
        s = tuple(int(v) for v in d["shape"])
        m = cls(*s, device=device)
        m.set_parameters(d["params"])
        m.set_scaling(d["in_shift"], d["in_scale"], d["out_shift"], d["out_scale"])
        return m


def data_parallel_train(model, x, t, epochs=20, batch=4096, lr=1e-3, lr_final=1e-5, seed=0,
                        log=None, group=None):
    """Data-parallel Adam (one process and GPU per rank): every rank draws the
    same shuffled minibatches (same seed), takes its share (rank r: samples
    r, r + world, ... of each minibatch; batch must be a multiple of the
    world size), computes its gradient on its GPU, and the gradients are
    averaged by one all-reduce per step (NCCL on the network's stream, or
    gloo), so every rank applies the same Adam step and the replicas stay
    equal. model: compute_gradients(x, t) -> loss, gradient_tensor() (reduced
    in place), apply_gradients(lr). Returns the epoch losses (averaged over
    ranks)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if batch % world:
        raise ValueError("batch (%d) must be a multiple of the world size (%d)" % (batch, world))
    n = x.shape[0]
    g = torch.Generator(device=x.device)
    g.manual_seed(seed)
    nbat = max(1, n // batch)
    steps = epochs * nbat
    k = 0
    losses = []
    grad = model.gradient_tensor()
    loss_t = torch.zeros(1, dtype=torch.float64, device=grad.device)
    for ep in range(epochs):
        perm = torch.randperm(n, device=x.device, generator=g)
        tot = 0.0
        for b in range(nbat):
            idx = perm[b * batch:(b + 1) * batch][rank::world]
            loss = model.compute_gradients(x[idx].contiguous(), t[idx].contiguous())
            if world > 1:
                dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
                grad.div_(world)
                loss_t.fill_(loss)
                dist.all_reduce(loss_t, op=dist.ReduceOp.SUM, group=group)
                loss = float(loss_t.item()) / world
            lr_k = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * k / steps))
            model.apply_gradients(lr_k)
            tot += loss
            k += 1
        losses.append(tot / nbat)
        if log:
            log("epoch %d loss %.3e" % (ep, losses[-1]))
    return losses
