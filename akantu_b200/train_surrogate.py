"""Trains the learned RVE surrogate of the FE^2 workload and writes its
weights (python -m akantu_b200.train_surrogate --samples N --out PATH).

1. Macroscopic gradients H with H_ij ~ U[-0.3, 0.3], det(I + H) >= 0.5,
   plus gradients of log-uniform magnitude 1e-4..0.3 (the small strains a
   macro model passes through), each relaxed on the 16^3 periodic
   sphere-inclusion RVE (batched RVE kernel, FP32, residual 1e-4) for its
   homogenised stress P.
2. Held-out sets of both kinds from other seeds.
3. The SiLU MLP (inputs H/|H| and log|H|, outputs P/|H|, 3 hidden layers of
   256) trained with Adam on the tensor cores (normalised inputs and
   outputs, cosine learning-rate decay).
Prints one JSON line: sizes, RVE solve rate, training time, held-out errors.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time


HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "data", "rve_surrogate.npz")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=2_000_000)
    ap.add_argument("--small-samples", type=int, default=1_000_000,
                    help="extra samples of log-uniform magnitude 1e-4..0.3")
    ap.add_argument("--heldout", type=int, default=16384)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--inference-samples", type=int, default=262144,
                    help="one timed inference pass over this many gradients (the Gauss "
                         "points of the 32^3 macro block)")
    a = ap.parse_args(argv)
    import torch
    from . import fe2
    from .surrogate import MLPSurrogate, scaled_features
    rve, mats, vf = fe2.spec_rve(16)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    X, Y, it, res = fe2.generate_dataset(rve, a.samples, seed=a.seed)
    if a.small_samples:
        Xs, Ys, its, rs = fe2.generate_dataset(rve, a.small_samples, seed=a.seed + 3, small=True)
        X, Y, it, res = (torch.cat([X, Xs]), torch.cat([Y, Ys]), torch.cat([it, its]),
                         torch.cat([res, rs]))
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    # labels of relaxations that did not reach the tolerance are left out
    keep = torch.isfinite(res) & (res <= 10 * 1e-4)
    X, Y = X[keep].contiguous(), Y[keep].contiguous()
    held = {}
    for name, small in (("envelope", False), ("small_strain", True)):
        Xh, Yh, _, rh = fe2.generate_dataset(rve, a.heldout, seed=a.seed + 1, small=small)
        kh = torch.isfinite(rh) & (rh <= 10 * 1e-4)
        held[name] = (Xh[kh].contiguous(), Yh[kh].contiguous())
    net = MLPSurrogate(seed=a.seed)
    x, y = scaled_features(X, Y)
    net.fit_scaling(x.cpu().numpy(), y.cpu().numpy())
    t1 = time.perf_counter()
    losses = net.train(x, y, epochs=a.epochs, batch=a.batch, lr=a.lr, lr_final=a.lr * 1e-3,
                       seed=a.seed, log=lambda s: print(s, file=sys.stderr, flush=True))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    err = {k: fe2.surrogate_error(net, *v) for k, v in held.items()}
    Hq = torch.as_tensor(fe2.sample_gradients(a.inference_samples, seed=a.seed + 2), device="cuda")
    Xq = Hq.transpose(1, 2).reshape(-1, 9).contiguous()
    net.predict_flat(Xq)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    net.predict_flat(Xq)
    e1.record()
    torch.cuda.synchronize()
    inf_ms = e0.elapsed_time(e1)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    net.save(a.out)
    print(json.dumps(dict(samples=a.samples, small_samples=a.small_samples,
                          kept=int(keep.sum()), heldout=a.heldout,
                          voxel_fraction=vf,
                          rve_solves_per_s=(a.samples + a.small_samples) / t_data,
                          mean_iterations=float(it.float().mean()), data_s=t_data,
                          train_s=t_train, epochs=a.epochs, final_loss=losses[-1],
                          heldout_error=err, inference_ms=inf_ms,
                          inference_samples=a.inference_samples, out=a.out)))


if __name__ == "__main__":
    main()
