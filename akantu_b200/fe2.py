"""FE^2 building blocks: periodic voxel RVEs and their macroscopic samples.

The micro problem is a cube of n^3 hexahedron_8 voxels with periodic nodes,
loaded by a macroscopic displacement gradient H (F = I + H); its homogenised
first Piola-Kirchhoff stress is what the macroscopic material
(MaterialFE2, extra_packages/extra-materials/src/material_FE2/material_FE2.hh:
40-101 in the reference, which linearises the same micro-macro coupling)
returns at each quadrature point.
"""
from __future__ import annotations

import math

import numpy as np

from . import _abi

SEED = 20261203


def sphere_inclusion_rve(cells=16, volume_fraction=0.2, length=1.0):
    """Voxel materials of a cube with one centred spherical inclusion of the
    given volume fraction (radius (vf 3 / 4 pi)^(1/3) L), voxelised by
    element centroid: 0 = matrix, 1 = inclusion. Returns (voxel_material
    uint8 n^3 with x fastest, actual voxel volume fraction)."""
    n = int(cells)
    r = (volume_fraction * 3.0 / (4.0 * math.pi)) ** (1.0 / 3.0) * length
    c = (np.arange(n) + 0.5) * (length / n) - 0.5 * length
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    inside = (x * x + y * y + z * z) <= r * r
    vm = inside.astype(np.uint8).ravel()  # index x + n (y + n z)
    return vm, float(vm.mean())


def matrix_inclusion_materials(lam=1.0e6, mu=0.4e6, contrast=10.0, rho=1100.0):
    """Neo-Hookean matrix (lambda, mu) and an inclusion `contrast` times
    stiffer, as material descriptors (E, nu derived from the Lame moduli)."""
    def nh(l, m):
        return dict(kind=_abi.MATERIAL_NEOHOOKEAN, rho=rho, E=m * (3 * l + 2 * m) / (l + m),
                    nu=l / (2 * (l + m)), lam=l, mu=m)
    return [nh(lam, mu), nh(contrast * lam, contrast * mu)]


def sample_gradients(count, seed=SEED, amplitude=0.3, min_det=0.5):
    """Macroscopic displacement gradients H with H_ij ~ U[-a, a], rejecting
    det(I + H) < min_det. Returns (count, 3, 3) FP64."""
    rng = np.random.default_rng(seed)
    out = np.empty((0, 3, 3))
    while out.shape[0] < count:
        H = rng.uniform(-amplitude, amplitude, (2 * (count - out.shape[0]) + 16, 3, 3))
        ok = np.linalg.det(np.eye(3) + H) >= min_det
        out = np.concatenate([out, H[ok]])
    return out[:count].copy()


def sample_small_gradients(count, seed=SEED, r_min=1e-4, r_max=0.3):
    """Gradients of log-uniform magnitude |H| in [r_min, r_max] (Frobenius)
    and uniformly distributed direction: the small strains a macro model
    passes through, which the uniform envelope sampling almost never draws."""
    rng = np.random.default_rng(seed)
    D = rng.normal(size=(count, 3, 3))
    D /= np.linalg.norm(D.reshape(count, 9), axis=1)[:, None, None]
    r = np.exp(rng.uniform(np.log(r_min), np.log(r_max), count))
    return D * r[:, None, None]


def in_envelope(H, amplitude=0.3, min_det=0.5):
    """The training envelope of the surrogate: |H_ij| <= a and det F >= d."""
    H = np.asarray(H).reshape(-1, 3, 3)
    return (np.abs(H).max(axis=(1, 2)) <= amplitude) & \
           (np.linalg.det(np.eye(3) + H) >= min_det)


# --------------------------------------------------------------- the macro side
def voigt_material(mats, fractions, rho=1100.0):
    """Material descriptor with the Voigt (upper-bound) Lame moduli of the
    mixture: its wave speed bounds the macroscopic one, so the stable time
    step computed from it is safe for the homogenised material."""
    lam = sum(f * m["lam"] for f, m in zip(fractions, mats))
    mu = sum(f * m["mu"] for f, m in zip(fractions, mats))
    return dict(rho=rho, E=mu * (3 * lam + 2 * mu) / (lam + mu), nu=lam / (2 * (lam + mu)))


def spec_rve(cells=16, precision=None, **options):
    """The periodic RVE of the FE^2 workload: 16^3 voxels, centred sphere of
    voxel fraction ~0.2, neo-Hookean matrix lambda = 1 MPa, mu = 0.4 MPa and
    an inclusion 10 times stiffer."""
    from .rve import SolidMechanicsModelRVE
    vm, vf = sphere_inclusion_rve(cells)
    mats = matrix_inclusion_materials()
    kw = dict(options)
    if precision is not None:
        kw["precision"] = precision
    return SolidMechanicsModelRVE(cells, vm, mats, **kw), mats, vf


def generate_dataset(rve, count, seed=SEED, chunk=32768, amplitude=0.3, min_det=0.5,
                     small=False):
    """count samples (H, P) with H drawn in the envelope (or, small=True,
    with log-uniform magnitude) and P the relaxed RVE's homogenised stress.
    Returns device FP64 X, Y (count, 9) (column-major flattening), the
    iteration counts and the final relative residuals."""
    import torch
    H = (sample_small_gradients(count, seed=seed) if small else
         sample_gradients(count, seed=seed, amplitude=amplitude, min_det=min_det))
    X, Y, its, res = [], [], [], []
    for k in range(0, count, chunk):
        Hc = torch.as_tensor(H[k:k + chunk], device="cuda:%d" % rve.device)
        out = rve.solve(Hc)
        X.append(Hc.transpose(1, 2).reshape(-1, 9))
        Y.append(out["stress"].transpose(1, 2).reshape(-1, 9))
        its.append(out["iterations"])
        res.append(out["residual"])
    return (torch.cat(X).contiguous(), torch.cat(Y).contiguous(), torch.cat(its),
            torch.cat(res))


def surrogate_error(net, X, Y):
    """Relative stress errors of the surrogate on (H, P) column-major
    samples: the global relative L2 error, the median and the 99th
    percentile of the per-sample relative error ||P_net - P|| / ||P||."""
    import torch
    P = net.predict_flat(X)
    d = torch.linalg.norm(P - Y, dim=1)
    r = torch.linalg.norm(Y, dim=1)
    per = (d / r.clamp_min(1e-30)).cpu().numpy()
    return dict(relative_l2=float(torch.linalg.norm(P - Y) / torch.linalg.norm(Y)),
                median=float(np.median(per)), p99=float(np.percentile(per, 99)))


class MaterialFE2:
    """Stress provider of the FE^2 macro material: the homogenised stress of a
    periodic RVE per quadrature point (warm-started from that point's previous
    fluctuation), or the learned surrogate inside its training envelope with
    RVE solves for the points outside it. Plugged into a SolidMechanicsModel
    through MaterialUser (the reference's MaterialFE2::computeStress,
    extra_packages/extra-materials/src/material_FE2/material_FE2.cc:116-157)."""

    def __init__(self, rve, surrogate=None, amplitude=0.3, min_det=0.5, chunk=32768,
                 warm_start=True):
        self.rve = rve
        self.surrogate = surrogate
        self.amplitude = amplitude
        self.min_det = min_det
        self.chunk = chunk
        self.warm_start = warm_start
        self.fluct = None
        self._stats = dict(rve_solves=0, fallback=0, iterations=0)
        self._fb = None  # device buffers of the learned path: index, count, running total

    @property
    def stats(self):
        """RVE solves, fallback points (learned path) and RVE updates (plain
        path) so far; reading it waits for the queued steps."""
        out = dict(self._stats)
        if self._fb is not None:
            n = int(self._fb[2].item())
            out["fallback"] += n
            out["rve_solves"] += n
        return out

    def material(self, mats, fractions, rho=1100.0):
        from .model import MaterialUser
        outer = self

        class _M(MaterialUser):
            def computeStress(self, grad_u, stress):
                outer.compute(grad_u, stress)
        d = voigt_material(mats, fractions, rho)
        return _M(rho=d["rho"], E=d["E"], nu=d["nu"], finite_deformation=True)

    def _ensure_fluct(self):
        if self.warm_start and (self.fluct is None or self.fluct.shape[0] != self.nq):
            self.fluct = self.rve.zero_fluctuation(self.nq)

    def _rve(self, H):
        """Plain FE^2: every point's RVE, in chunks; a point's warm start is
        its row of self.fluct, solved in place."""
        import torch
        n = H.shape[0]
        self._ensure_fluct()
        P = torch.empty((n, 3, 3), dtype=torch.float64, device=H.device)
        for k in range(0, n, self.chunk):
            sl = slice(k, min(n, k + self.chunk))
            out = self.rve.solve(H[sl], self.fluct[sl] if self.warm_start else None)
            P[sl] = out["stress"]
            self._stats["iterations"] += int(out["iterations"].sum())
        self._stats["rve_solves"] += n
        return P

    def compute(self, grad_u, stress):
        """The stresses of every Gauss point. With a surrogate: one kernel
        forms the features, runs the network, writes |H| net(.) and lists the
        points outside the envelope; one kernel relaxes the RVEs of the
        listed points (it reads the list's length on the device, so the step
        never waits for the host)."""
        import torch
        self.nq = grad_u.shape[0]
        if self.surrogate is None:
            stress.copy_(self._rve(grad_u))
            return
        # [k, i, j] views of column-major storage: transposed back, they are
        # the (nq, 9) column-major arrays the kernels take
        H = grad_u.transpose(1, 2).reshape(-1, 9)
        P = stress.transpose(1, 2).reshape(-1, 9)
        direct = H.is_contiguous() and P.is_contiguous() and \
            P.data_ptr() == stress.data_ptr() and H.dtype == P.dtype == torch.float64
        if not direct:
            H = H.to(torch.float64).contiguous()
            P = torch.empty_like(H)
        if self._fb is None or self._fb[0].shape[0] != self.nq:
            dev = grad_u.device
            self._fb = (torch.empty(self.nq, dtype=torch.int32, device=dev),
                        torch.zeros(1, dtype=torch.int32, device=dev),
                        torch.zeros(1, dtype=torch.int64, device=dev))
        idx, cnt, total = self._fb
        self.surrogate.stress_into(H, P, envelope=(self.amplitude, self.min_det),
                                   fallback=(idx, cnt))
        self._ensure_fluct()
        self.rve.solve_indexed(idx, cnt, H, P, self.fluct if self.warm_start else None)
        total += cnt
        if not direct:
            stress.copy_(P.reshape(-1, 3, 3).transpose(1, 2))


def macro_block(material, cells=32, length=1.0, precision=None):
    """The FE^2 macro problem: a cube of cells^3 hexahedron_8, face x = 0
    fixed, face x = L pulled along x (its x displacement prescribed)."""
    from . import _abi
    from .mesh import block_hexahedron8
    from .model import SolidMechanicsModel
    mesh = block_hexahedron8(cells, length)
    m = SolidMechanicsModel(mesh, [material], precision=_abi.MODE_FP64)
    m.initFull()
    x = mesh.nodes
    left = np.nonzero(np.isclose(x[:, 0], 0.0))[0]
    right = np.nonzero(np.isclose(x[:, 0], length))[0]
    blocked = np.zeros_like(x, dtype=np.uint8)
    blocked[left] = 1
    blocked[right, 0] = 1
    m.setBlockedDOFs(blocked)
    m.fe2_right = right
    m.fe2_length = length
    return m


def macro_step(model, step, ramp_steps=200, stretch=0.05):
    """One macro step with the pulled face at stretch * L * min(step / ramp, 1)."""
    ux = stretch * model.fe2_length * min(step / ramp_steps, 1.0)
    model.applyDirichlet(model.fe2_right, 0, ux)
    model.solveStep()
