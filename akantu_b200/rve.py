"""Batched periodic RVE solves (include/akb_fe2.h: akb_rve_*).

SolidMechanicsModelRVE relaxes many copies of one voxel microstructure, each
under its own macroscopic displacement gradient, in one launch, and returns
their homogenised first Piola-Kirchhoff stresses -- the micro side of FE^2
(the reference's SolidMechanicsModelRVE,
extra_packages/extra-materials/src/material_FE2/solid_mechanics_model_RVE.hh:
44-93, applies the macroscopic gradient to one RVE at a time and averages its
stress). Device buffers are torch tensors; tensors here are (nb, 3, 3) with
[b, i, j] = du_i/dX_j (the library's column-major layout is handled here).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._lib import check, lib
from .model import material_from_dict, torch_stream


def _torch():
    import torch
    return torch


class SolidMechanicsModelRVE:
    def __init__(self, cells, voxel_material, materials, length=1.0,
                 precision=_abi.MODE_FP32_BULK, device=0, max_iterations=0, check_interval=0,
                 tolerance=0.0, time_step_factor=0.0, damping_factor=0.0):
        self.cells = int(cells)
        self.length = float(length)
        vm = np.ascontiguousarray(voxel_material, dtype=np.uint8).ravel()
        if vm.size != self.cells ** 3:
            raise ValueError("voxel_material needs cells^3 entries")
        mats = [material_from_dict(m) if isinstance(m, dict) else m for m in materials]
        self._mats = (_abi.MaterialDesc * len(mats))(*[m.desc() for m in mats])
        self._vm = vm
        desc = _abi.RveDesc(self.cells, len(mats), self.length,
                            vm.ctypes.data_as(C.POINTER(C.c_uint8)), self._mats)
        opt = _abi.RveOptions(precision, device, None, max_iterations, check_interval,
                              tolerance, time_step_factor, damping_factor)
        h = C.c_void_p()
        check(lib().akb_rve_create(C.byref(desc), C.byref(opt), C.byref(h)))
        self._h = h
        self.precision = precision
        self.device = device
        info = _abi.RveInfo()
        check(lib().akb_rve_get_info(h, C.byref(info)))
        self.volume_fraction = list(info.volume_fraction)[:len(mats)]
        self.shared_bytes = info.shared_bytes
        self.nb_nodes = info.nb_nodes

    def close(self):
        if getattr(self, "_h", None):
            lib().akb_rve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def fluctuation_dtype(self):
        torch = _torch()
        return torch.float64 if self.precision == _abi.MODE_FP64 else torch.float32

    def zero_fluctuation(self, nb):
        torch = _torch()
        return torch.zeros((nb, self.nb_nodes, 3), dtype=self.fluctuation_dtype,
                           device="cuda:%d" % self.device)

    def _grad_u(self, grad_u):
        torch = _torch()
        g = torch.as_tensor(grad_u, dtype=torch.float64)
        g = g.to("cuda:%d" % self.device).reshape(-1, 3, 3)
        return g.transpose(1, 2).contiguous()  # column-major per point

    def solve(self, grad_u, fluctuation=None):
        """Relaxes one RVE per gradient. grad_u: (nb, 3, 3); fluctuation: an
        (nb, n^3, 3) device tensor used as the start and overwritten (None:
        start from zero). Returns dict(stress (nb, 3, 3) FP64 device tensor,
        iterations, residual, fluctuation)."""
        torch = _torch()
        H = self._grad_u(grad_u)
        nb = H.shape[0]
        dev = H.device
        if fluctuation is not None:
            if (fluctuation.dtype != self.fluctuation_dtype or not fluctuation.is_contiguous()
                    or tuple(fluctuation.shape) != (nb, self.nb_nodes, 3)):
                raise ValueError("fluctuation must be a contiguous (nb, n^3, 3) %s tensor"
                                 % self.fluctuation_dtype)
        P = torch.empty((nb, 3, 3), dtype=torch.float64, device=dev)
        it = torch.empty(nb, dtype=torch.int32, device=dev)
        res = torch.empty(nb, dtype=torch.float64, device=dev)
        stream = torch_stream(dev)
        check(lib().akb_rve_solve(self._h, nb, H.data_ptr(),
                                  fluctuation.data_ptr() if fluctuation is not None else None,
                                  P.data_ptr(), it.data_ptr(), res.data_ptr(), stream))
        return dict(stress=P.transpose(1, 2), iterations=it, residual=res,
                    fluctuation=fluctuation)

    def solve_indexed(self, index, count, grad_u, stress, fluctuation=None):
        """Relaxes the RVEs of the points index[:count] (device int32
        tensors; count is read on the device) of (capacity, 9) column-major
        FP64 gradient and stress tensors, writing those points' stresses
        (and fluctuations, warm-started from fluctuation if given)."""
        torch = _torch()
        cap = grad_u.shape[0]
        for t in (grad_u, stress):
            if t.dtype != torch.float64 or not t.is_contiguous() or tuple(t.shape) != (cap, 9):
                raise ValueError("grad_u and stress must be contiguous (capacity, 9) float64")
        if fluctuation is not None and (fluctuation.dtype != self.fluctuation_dtype
                                        or not fluctuation.is_contiguous()
                                        or tuple(fluctuation.shape) != (cap, self.nb_nodes, 3)):
            raise ValueError("fluctuation must be a contiguous (capacity, n^3, 3) %s tensor"
                             % self.fluctuation_dtype)
        check(lib().akb_rve_solve_indexed(self._h, cap, index.data_ptr(), count.data_ptr(),
                                          grad_u.data_ptr(),
                                          fluctuation.data_ptr() if fluctuation is not None else None,
                                          stress.data_ptr(), None, None,
                                          torch_stream(grad_u.device)))
        return stress

    def stress(self, grad_u, fluctuation):
        """Homogenised stress and internal force (nb, n^3, 3) of given states."""
        torch = _torch()
        H = self._grad_u(grad_u)
        nb = H.shape[0]
        P = torch.empty((nb, 3, 3), dtype=torch.float64, device=H.device)
        f = torch.empty((nb, self.nb_nodes, 3), dtype=torch.float64, device=H.device)
        w = fluctuation.to(self.fluctuation_dtype).contiguous()
        stream = torch_stream(H.device)
        check(lib().akb_rve_stress(self._h, nb, H.data_ptr(), w.data_ptr(), P.data_ptr(),
                                   f.data_ptr(), stream))
        return P.transpose(1, 2), f
