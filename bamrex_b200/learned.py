"""The learned preconditioner of the pressure solve over the C ABI: the
network (``PrecNet``), training data from the plain solver, training with
the library's own forward/backward/Adam kernels, and the FGMRES solve that
falls back to the plain one.  This part has no counterpart in the reference;
the solve it serves is solve_pressure (Source/IMEX/IMEX_O1.cpp:616-640)."""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import problems
from ._abi import PRECOND_NETWORK, PRECOND_NETWORK_VCYCLE, PRECOND_VCYCLE, BamrexError, check, lib
from .helmholtz import Helmholtz, _ptr


class PrecNet:
    def __init__(self, nx, ny, batch=1, seed=1234, stream=None):
        self._h = ctypes.c_void_p()
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        check(lib().bamrex_precnet_create(ctypes.byref(self._h), nx, ny, batch, seed, st))
        self.nx, self.ny, self.batch = nx, ny, batch

    def close(self):
        if self._h:
            lib().bamrex_precnet_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        if rc != 0:
            m = lib().bamrex_precnet_last_error(self._h)
            raise BamrexError(rc, (m or b"").decode() or lib().bamrex_last_error().decode())

    @property
    def num_params(self):
        return lib().bamrex_precnet_num_params(self._h)

    def resize(self, nx, ny, batch=1):
        self._ck(lib().bamrex_precnet_resize(self._h, nx, ny, batch))
        self.nx, self.ny, self.batch = nx, ny, batch

    def set_tensor_cores(self, on=True):
        """Where the 16 -> 16 convolutions of inference run: True / 1 the
        tensor cores (tcgen05 on levels whose width is a multiple of 128,
        mma.sync elsewhere), 2 mma.sync only, False / 0 the FP32 CUDA cores
        (bamrex_precnet_set_tensor_cores)."""
        mode = int(on) if not isinstance(on, bool) else (1 if on else 0)
        self._ck(lib().bamrex_precnet_set_tensor_cores(self._h, mode))

    def get_weights(self):
        w = np.empty(self.num_params, dtype=np.float32)
        self._ck(lib().bamrex_precnet_get_weights(self._h, ctypes.c_void_p(w.ctypes.data)))
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._ck(lib().bamrex_precnet_set_weights(self._h, ctypes.c_void_p(w.ctypes.data)))

    def forward(self, inp):
        inp = np.ascontiguousarray(inp, dtype=np.float32)
        out = np.empty((self.batch, self.ny, self.nx), dtype=np.float32)
        self._ck(lib().bamrex_precnet_forward(self._h, ctypes.c_void_p(inp.ctypes.data), ctypes.c_void_p(out.ctypes.data)))
        return out

    def backward(self, dout):
        dout = np.ascontiguousarray(dout, dtype=np.float32)
        g = np.empty(self.num_params, dtype=np.float32)
        self._ck(lib().bamrex_precnet_backward(self._h, ctypes.c_void_p(dout.ctypes.data), ctypes.c_void_p(g.ctypes.data)))
        return g

    def train_step(self, inp, target, lr):
        inp = np.ascontiguousarray(inp, dtype=np.float32)
        target = np.ascontiguousarray(target, dtype=np.float32)
        loss = ctypes.c_double()
        self._ck(lib().bamrex_precnet_train_step(self._h, ctypes.c_void_p(inp.ctypes.data),
                                                 ctypes.c_void_p(target.ctypes.data), lr, ctypes.byref(loss)))
        return loss.value


def network_input(r, beta_cc):
    """(r / rms(r), log beta) as the network's two input channels."""
    r = np.asarray(r, dtype=np.float64).reshape(beta_cc.shape[-2:])
    s = np.sqrt(np.mean(r * r))
    return np.stack([r / s, np.log(beta_cc.reshape(r.shape))]).astype(np.float32), s


def make_training_pairs(count, n=256, seed=7, tol=1e-7, corr_cells=32, log_sigma=1.0, mach=0.01, dx=1.0 / 2048,
                        log=None, after_vcycle=False):
    """(input, target) pairs from the plain solver on n^2 periodic patches
    with the pressure problem's scalars at cell size dx: a fresh lognormal
    beta and a random right-hand side per pair (white noise blended with a
    smooth field); target = solution * B / (rms(r) dx^2).

    after_vcycle: the pair is what one multigrid V-cycle leaves of that
    right-hand side instead, r' = r - A V(r) and its error A^-1 r' (the
    network of the PRECOND_VCYCLE_NETWORK mode corrects the V-cycle: it sees
    the V-cycle's residual and should return the error the V-cycle left)."""
    rng = np.random.default_rng(seed)
    eps = mach * mach
    a = eps / 0.4
    dt = 0.8 * dx / mach
    B = dt * dt
    h = Helmholtz(2, (n, n), [0.0, 0.0], [n * dx, n * dx])
    h.setScalars(1.0, B, 0.0)
    h.setACoeffs(a)
    X = np.empty((count, 2, n, n), dtype=np.float32)
    Y = np.empty((count, n, n), dtype=np.float32)
    t0 = time.time()
    for k in range(count):
        if k % 8 == 0:
            g = problems.gaussian_random_field((n, n), corr_cells, None, rng)
            beta = np.exp(-log_sigma * g)[None]
            h.setBCoeffsFromCell(beta)
        w = rng.uniform(0.0, 1.0)
        r = w * rng.standard_normal((1, n, n)) + (1 - w) * problems.gaussian_random_field((n, n), rng.uniform(1, 16),
                                                                                          None, rng)[None]
        if after_vcycle:
            r = r - h.apply(h.vcycle(r))
        e, it, rr = h.solve(r, tol_rel=tol)
        inp, s = network_input(r[0], beta[0])
        X[k] = inp
        Y[k] = (e[0] * B / (s * dx * dx)).astype(np.float32)
        if log and k % 250 == 0:
            log("pair %d/%d (%.1fs, %d iterations)" % (k, count, time.time() - t0, it))
    h.close()
    return X, Y


def train(net: PrecNet, X, Y, epochs=4, batch=8, lr=2e-3, seed=3, log=None):
    """Adam on the relative squared error with the library's kernels."""
    rng = np.random.default_rng(seed)
    n = X.shape[0]
    net.resize(X.shape[3], X.shape[2], batch)
    losses = []
    steps = 0
    total = epochs * (n // batch)
    for ep in range(epochs):
        order = rng.permutation(n)
        for q in range(n // batch):
            idx = order[q * batch:(q + 1) * batch]
            cur_lr = lr * 0.5 * (1 + np.cos(np.pi * steps / total))
            losses.append(net.train_step(X[idx], Y[idx], cur_lr))
            steps += 1
        if log:
            log("epoch %d: mean loss %.4f" % (ep, float(np.mean(losses[-(n // batch):]))))
    return losses


def solve_learned(h: Helmholtz, net, rhs, x0=None, tol_rel=1e-8, tol_abs=0.0, max_iter=60, restart=30,
                  mode=PRECOND_NETWORK_VCYCLE):
    """FGMRES with the chosen preconditioner, falling back to the plain
    solve: returns (x, fgmres iterations, fallback iterations, rel residual,
    fell_back).  net may be None for PRECOND_VCYCLE."""
    x = np.zeros(h.shape) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    rp, kr = _ptr(rhs)
    it, pit, fb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rr = ctypes.c_double()
    h._ck(lib().bamrex_helmholtz_solve_learned(h._h, net._h if net is not None else None, mode,
                                               ctypes.c_void_p(x.ctypes.data), rp, tol_rel, tol_abs, max_iter, restart,
                                               ctypes.byref(it), ctypes.byref(pit), ctypes.byref(rr), ctypes.byref(fb)))
    return x, it.value, pit.value, rr.value, bool(fb.value)


def solve_learned_device(h: Helmholtz, net, x, rhs, tol_rel=1e-8, tol_abs=0.0, max_iter=60, restart=30,
                         mode=PRECOND_NETWORK_VCYCLE):
    it, pit, fb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rr = ctypes.c_double()
    h._ck(lib().bamrex_helmholtz_solve_learned(h._h, net._h if net is not None else None, mode,
                                               ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(rhs.data_ptr()), tol_rel,
                                               tol_abs, max_iter, restart, ctypes.byref(it), ctypes.byref(pit),
                                               ctypes.byref(rr), ctypes.byref(fb)))
    return it.value, pit.value, rr.value, bool(fb.value)


def _main(argv=None):
    """python -m bamrex_b200.learned [--n N] [--forwards K] [--mode M]:
    forward passes of the preconditioner network (untrained weights) on an
    N x N grid."""
    import argparse

    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--forwards", type=int, default=3)
    ap.add_argument("--mode", type=int, default=1,
                    help="16 -> 16 convolutions: 1 tensor cores (tcgen05 / mma.sync), 2 mma.sync, 0 FP32 CUDA cores")
    a = ap.parse_args(argv)
    net = PrecNet(a.n, a.n, batch=1, seed=1)
    net.set_tensor_cores(a.mode)
    inp = np.random.default_rng(0).standard_normal((1, 2, a.n, a.n)).astype(np.float32)
    for k in range(a.forwards):
        t0 = time.perf_counter()
        out = net.forward(inp)
        torch.cuda.synchronize()
        print("forward %d: %.2f ms (host copies included), |out| %.3e" % (k, 1e3 * (time.perf_counter() - t0),
                                                                         float(np.abs(out).mean())))
    net.close()


if __name__ == "__main__":
    _main()
