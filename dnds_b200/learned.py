"""Learned warm start for the VR coefficients (no counterpart in the reference).

A per-cell network (64 -> 64 -> 64 -> 64 -> 20, SiLU; BF16 weights and
activations, FP32 accumulation) extrapolates the Jacobi sequence: from the
starting coefficients x0 and two plain sweeps x1, x2 it proposes the converged
coefficients, using the sweep increments, the neighbour mean differences and
the slot geometry in the cell's own polynomial frame.  Training,
inference and the per-cell gate all run in ``libdndsg.so``
(``dndsg_mlp_*``, ``dndsg_vr_to_tolerance``, ``dndsg_ssprk3_step_tol``);
this module only drives them:

* ``WarmStartNet``   one network on one GPU (create / params / forward /
                     gradient / Adam step / save / load)
* ``harvest``        (feature, target) pairs from tolerance-mode SSP-RK3 runs:
                     the target is (converged - x2) / r
* ``train``          minibatch Adam over harvested pairs, on the GPU
* ``sweep_counts``   Jacobi sweeps per stage to a tolerance, with or without
                     the network, for the sweeps-saved comparison

The plain Jacobi sweep (ReconstructionJacobiStep, DNDS_FV_VR.hpp:1474-1713)
decides: it iterates to the same tolerance either way, and per cell
the learned start is kept only where the Jacobi increment from it is smaller
than from the plain start.  Device arrays are torch CUDA tensors (plumbing
only); no computation of the path runs in torch.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import _lib
from .solver import DndsgError, Solver

N_IN, N_OUT, N_PARAM = _lib.MLP_IN, _lib.MLP_OUT, _lib.MLP_NPARAM
HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "weights", "vr_warm_start.npz")


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def _stream_ptr():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class WarmStartNet:
    """One network on one GPU; parameters are FP32 masters with a BF16 copy for the MMAs."""

    def __init__(self, device: int = 0, seed: int = 0, params: np.ndarray | None = None, features: int = 0):
        self.L = _lib.lib()
        self.device = device
        h = C.c_void_p()
        rc = self.L.dndsg_mlp_create(int(device), C.c_uint64(seed), C.byref(h))
        if rc != 0:
            raise DndsgError(rc, "dndsg_mlp_create failed")
        self.h = h
        self.features = int(features)
        self._check(self.L.dndsg_mlp_set_features(self.h, self.features))
        if params is not None:
            self.params = params

    def close(self):
        if getattr(self, "h", None):
            self.L.dndsg_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            raise DndsgError(rc, self.L.dndsg_mlp_last_error(self.h).decode())

    @property
    def params(self) -> np.ndarray:
        p = np.empty(N_PARAM, dtype=np.float32)
        self._check(self.L.dndsg_mlp_get_params(self.h, p.ctypes.data_as(C.c_void_p)))
        return p

    @params.setter
    def params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32).reshape(N_PARAM)
        self._check(self.L.dndsg_mlp_set_params(self.h, p.ctypes.data_as(C.c_void_p)))

    def forward(self, X):
        """Y [n][20] for features X [n][64] (float32 CUDA tensors)."""
        import torch
        X = X.contiguous()
        Y = torch.empty((X.shape[0], N_OUT), dtype=torch.float32, device=X.device)
        self._check(self.L.dndsg_mlp_forward(self.h, _ptr(X), X.shape[0], _ptr(Y), _stream_ptr()))
        return Y

    def gradient(self, X, T):
        """(mean-square loss, gradient [N_PARAM] float32) on the batch."""
        X, T = X.contiguous(), T.contiguous()
        g = np.empty(N_PARAM, dtype=np.float32)
        loss = C.c_double()
        self._check(self.L.dndsg_mlp_gradient(self.h, _ptr(X), _ptr(T), X.shape[0], C.byref(loss),
                                              g.ctypes.data_as(C.c_void_p), _stream_ptr()))
        return loss.value, g

    def train_step(self, X, T, lr: float, want_loss: bool = False):
        loss = C.c_double()
        self._check(self.L.dndsg_mlp_train_step(self.h, _ptr(X), _ptr(T), X.shape[0], C.c_float(lr),
                                                C.byref(loss) if want_loss else None, _stream_ptr()))
        return loss.value if want_loss else None

    def save(self, path: str, **meta):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez(path, params=self.params, **{k: np.asarray(v) for k, v in meta.items()})

    @classmethod
    def load(cls, path: str = WEIGHTS, device: int = 0) -> "WarmStartNet":
        with np.load(path) as z:
            return cls(device=device, params=z["params"])


def harvest(solver: Solver, steps: int, cfl: float, tol: float, max_sweeps: int = 200, net=None,
            t_end: float = 1e300):
    """Runs `steps` tolerance-mode SSP-RK3 steps and returns the (X, T) pairs of every stage
    as float32 CUDA tensors [3*steps*N][64], [3*steps*N][20], and the sweeps taken per step."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    N = solver.N
    Xs, Ts, sweeps = [], [], []
    for _ in range(steps):
        X = torch.empty((3, N, N_IN), dtype=torch.float32, device=dev)
        T = torch.empty((3, N, N_OUT), dtype=torch.float32, device=dev)
        sweeps.append(solver.ssprk3_step_tol(cfl, tol, max_sweeps, net, t_end, X.data_ptr(), T.data_ptr()))
        Xs.append(X.view(-1, N_IN))
        Ts.append(T.view(-1, N_OUT))
    return torch.cat(Xs), torch.cat(Ts), sweeps


def bounded_pairs(X, T, bound: float = 10.0):
    """The pairs whose targets all lie within +-bound, and the fraction kept.  Targets are coefficient
    changes in units of the cell's own feature scale; where that scale sits at its floor (a nearly
    uniform neighbourhood) a rounding-level change becomes a huge target, yet the network's output is
    multiplied by that same tiny scale when it is applied, so such pairs carry nothing for inference
    and would only dominate the mean-square loss."""
    keep = T.abs().amax(dim=1) <= bound
    return X[keep].contiguous(), T[keep].contiguous(), float(keep.float().mean())


def train(net: WarmStartNet, X, T, epochs: int = 20, batch: int = 65536, lr: float = 2e-3,
          lr_end: float = 5e-5, seed: int = 0, val_frac: float = 0.05, log=None):
    """Minibatch Adam with a cosine learning-rate decay; returns (train losses per epoch, validation loss)."""
    import torch
    g = torch.Generator(device=X.device)
    g.manual_seed(seed)
    n = X.shape[0]
    perm = torch.randperm(n, generator=g, device=X.device)
    nval = max(1, int(n * val_frac))
    Xv, Tv = X[perm[:nval]].contiguous(), T[perm[:nval]].contiguous()
    tr = perm[nval:]
    nb = max(1, (tr.numel() + batch - 1) // batch)
    total = epochs * nb
    it = 0
    hist = []
    for ep in range(epochs):
        p = tr[torch.randperm(tr.numel(), generator=g, device=X.device)]
        acc = 0.0
        for b in range(nb):
            idx = p[b * batch:(b + 1) * batch]
            xb, tb = X[idx].contiguous(), T[idx].contiguous()
            cur = lr_end + 0.5 * (lr - lr_end) * (1 + math.cos(math.pi * it / total))
            want = b == nb - 1
            l = net.train_step(xb, tb, cur, want_loss=want)
            if want:
                acc = l
            it += 1
        hist.append(acc)
        if log:
            log(f"epoch {ep}: batch loss {acc:.4e}")
    val, _ = net.gradient(Xv, Tv)
    return hist, val


def sweep_counts(solver: Solver, steps: int, cfl: float, tol: float, net=None, max_sweeps: int = 200,
                 t_end: float = 1e300):
    """Jacobi sweeps taken per SSP-RK3 step in tolerance mode (the warm start's two gated sweeps count)."""
    return [solver.ssprk3_step_tol(cfl, tol, max_sweeps, net, t_end) for _ in range(steps)]


def training_set(tol: float = 1e-7, steps: int = 8, n: int = 256, seeds=(11, 12), log=None, features: int = 0):
    """(X, T) harvested from tolerance-mode runs of the three explicit workloads on small meshes:
    the isentropic vortex on 40x40 quads, on jittered n x n x 2 triangles (one run per seed), and
    the four-quadrant Riemann problem with the limiter on jittered n x n x 2 triangles; features of
    the given design (0 Jacobi extrapolation, 1 previous-step coefficients)."""
    import torch

    from .geometry import isentropic_vortex, quadrant_states
    from .mesh import riemann_mesh, vortex_mesh
    from .settings import RIEMANN_2D_STATES, preset

    runs = [("vortex quads 40x40", vortex_mesh(40, False), "vortex", 0.5, isentropic_vortex)]
    for sd in seeds:
        runs.append((f"vortex tri {n}x{n}x2 seed {sd}", vortex_mesh(n, True, jitter=0.2, seed=sd), "vortex", 0.5,
                     isentropic_vortex))
    runs.append((f"riemann tri {n}x{n}x2", riemann_mesh(n, seed=seeds[0]), "riemann", 0.4,
                  lambda m, t: quadrant_states(m, RIEMANN_2D_STATES)))
    Xs, Ts = [], []
    for name, m, pre, cfl, init in runs:
        s = Solver(m, preset(pre), precision=1)
        s.set_warm_start_features(features)
        s.set_u(init(m, 0.0))
        s.vr_to_tolerance(tol, 2000)
        X, T, sw = harvest(s, steps, cfl, tol, 2000)
        Xs.append(X)
        Ts.append(T)
        if log:
            log(f"{name}: {X.shape[0]} pairs, sweeps per step {sw}")
        s.close()
    return torch.cat(Xs), torch.cat(Ts)


def evaluate(nets: dict, tol: float = 1e-7, grid: int = 1448, steps: int = 3, seed: int = 9999, log=None):
    """Jacobi sweeps per SSP-RK3 step to the same rms-increment tolerance, without a network and with
    each network of `nets` (name -> WarmStartNet), on fresh-seed jittered grid x grid x 2 meshes of the
    vortex and of the Riemann problem (with the CWBAP limiter), FP32 bulk: sweeps per step, ms per step
    (wall time of the steps), and the density difference to the plain run after the steps (L2 relative
    to the density's L2)."""
    import time

    import torch

    from .geometry import cell_quadrature, isentropic_vortex, quadrant_states
    from .mesh import riemann_mesh, vortex_mesh
    from .settings import RIEMANN_2D_STATES, preset

    out = {}
    cases = (("vortex", lambda: vortex_mesh(grid, True, jitter=0.2, seed=seed), "vortex", 0.5,
              lambda m: isentropic_vortex(m)),
             ("riemann", lambda: riemann_mesh(grid, seed=seed), "riemann", 0.4,
              lambda m: quadrant_states(m, RIEMANN_2D_STATES)))
    for name, mk, pre, cfl, init in cases:
        m = mk()
        vol = cell_quadrature(m)[1].sum(1)
        r, us = {"cells": m.n_cells}, {}
        for label, net in [("plain", None)] + list(nets.items()):
            s = Solver(m, preset(pre), precision=1)
            s.set_warm_start_features(net.features if net is not None else 0)
            s.set_u(init(m))
            s.vr_to_tolerance(tol, 2000)
            s.ssprk3_step_tol(cfl, tol, 2000, net)  # warm-up step
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sw = [s.ssprk3_step_tol(cfl, tol, 2000, net) for _ in range(steps)]
            torch.cuda.synchronize()
            r[label] = {"sweeps_per_step": sw, "ms_per_step": (time.perf_counter() - t0) / steps * 1e3}
            us[label] = s.get_u()
            s.close()
            if label != "plain":
                d = us[label][:, 0] - us["plain"][:, 0]
                r[label]["rho_l2_vs_plain"] = float(np.sqrt((d * d * vol).sum() / (us["plain"][:, 0] ** 2 * vol).sum()))
                r[label]["sweeps_saved_per_step"] = float(np.mean(r["plain"]["sweeps_per_step"]) - np.mean(sw))
        out[name] = r
        if log:
            log(name, r)
    return out


def time_forward(rows_list=(1 << 20, 1 << 22), reps: int = 5, seed: int = 7):
    """CUDA-event time of the tensor-core forward on random features; returns [(rows, ms)]."""
    import torch

    net = WarmStartNet(0, seed=seed)
    dev = torch.device("cuda:0")
    out = []
    for rows in rows_list:
        X = torch.randn((rows, N_IN), device=dev)
        net.forward(X)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            net.forward(X)
        e1.record()
        torch.cuda.synchronize()
        out.append((rows, e0.elapsed_time(e1) / reps))
    return out


def time_train_step(rows: int = 1 << 20, reps: int = 10, seed: int = 7):
    """CUDA-event time of one training step (forward, backward, Adam) on random features and
    targets; returns ms per step."""
    import torch

    net = WarmStartNet(0, seed=seed)
    dev = torch.device("cuda:0")
    X = torch.randn((rows, N_IN), device=dev)
    T = 0.1 * torch.randn((rows, N_OUT), device=dev)
    net.train_step(X, T, 1e-4)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        net.train_step(X, T, 1e-4)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def main(argv=None):
    import argparse
    import time

    import torch

    if argv is None:
        import sys

        argv = sys.argv[1:]
    if "--time-train" in argv:
        rows = 1 << 20
        ms = time_train_step(rows)
        flop = 3 * 2 * (N_IN * 64 + 64 * 64 * 2 + 64 * N_OUT) * rows
        print(f"{rows} rows: {ms:.4f} ms per training step, {rows / ms / 1e6:.3f}e9 samples/s, "
              f"{flop / ms / 1e9:.1f} TFLOP/s (forward + backward, 3x the forward)")
        return
    if "--time-forward" in argv:
        for rows, ms in time_forward():
            flop = 2 * (N_IN * 64 + 64 * 64 * 2 + 64 * N_OUT) * rows
            print(f"{rows} rows: {ms:.4f} ms, {rows / ms / 1e6:.3f}e9 rows/s, {flop / ms / 1e9:.1f} TFLOP/s, "
                  f"{rows * (4 * N_IN + 4 * N_OUT) / ms / 1e6:.0f} GB/s")
        return
    ap = argparse.ArgumentParser(description="harvest, train and save the VR warm-start network "
                                             "(--time-forward: time the tensor-core forward instead)")
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--tol", type=float, default=1e-7)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--seed", type=int, default=7)
    a = ap.parse_args(argv)
    t0 = time.time()
    X, T = training_set(a.tol, a.steps, a.n, log=print)
    torch.cuda.synchronize()
    print(f"harvested {X.shape[0]} pairs in {time.time() - t0:.1f} s")
    net = WarmStartNet(0, seed=a.seed)
    t0 = time.time()
    hist, val = train(net, X, T, epochs=a.epochs, log=print)
    torch.cuda.synchronize()
    print(f"trained in {time.time() - t0:.1f} s: validation loss {val:.4e}, "
          f"target mean square {float((T ** 2).mean()):.4e}")
    net.save(a.out, tol=a.tol, val_loss=val, n_pairs=X.shape[0])
    print(a.out)


if __name__ == "__main__":
    main()
