"""Exact Riemann solver with a learned star-pressure guess (C-ABI wrapper).

Device arrays are torch tensors (device memory plumbing only); the solver,
the tensor-core network inference (tcgen05 with TMEM accumulators, or
per-warp mma.sync) and the training all run in the CUDA library
(flash5_b200/csrc/riemann_exact.cu).
"""
import ctypes as C

import numpy as np

from . import abi

_SIGS = {
    "flash_hy_rsolver_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "flash_hy_rsolver_destroy": (C.c_int, [C.c_void_p]),
    "flash_hy_rsolver_stream": (C.c_void_p, [C.c_void_p]),
    "flash_hy_rsolver_generate": (C.c_int, [C.c_void_p, C.c_ulonglong, C.c_long, C.c_void_p]),
    "flash_hy_rsolver_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_int, C.c_double, C.c_int]),
    "flash_hy_rsolver_predict": (C.c_int, [C.c_void_p, C.c_void_p, C.c_long, C.c_void_p]),
    "flash_hy_rsolver_make_samples": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_void_p,
                                                C.c_void_p, C.c_long, C.POINTER(C.c_long)]),
    "flash_hy_rsolver_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                        C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "flash_hy_rsolver_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_int, C.c_int,
                                         C.c_float, C.POINTER(C.c_float)]),
    "flash_hy_rsolver_get_weights": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int]),
    "flash_hy_rsolver_set_weights": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int]),
    "flash_hy_rsolver_num_params": (C.c_int, []),
    "flash_hy_rsolver_sync": (C.c_int, [C.c_void_p]),
    "flash_hy_rsolver_set_inference": (C.c_int, [C.c_void_p, C.c_int]),
}

INFER_TCGEN05 = 0     # network on the tcgen05 tensor cores, 128 interfaces per MMA tile (default)
INFER_WARP_MMA = 1    # network per warp on mma.sync (the form inlined in the hydro kernels)


def _lib():
    L = abi.load_library()
    if not getattr(L, "_rs_sigs", False):
        for n, (res, args) in _SIGS.items():
            f = getattr(L, n)
            f.restype = res
            f.argtypes = args
        L._rs_sigs = True
    return L


class RiemannError(RuntimeError):
    pass


class ExactRiemann:
    def __init__(self, device=0):
        import torch
        self.torch = torch
        self.device = device
        self.L = _lib()
        self.h = C.c_void_p()
        st = self.L.flash_hy_rsolver_create(device, C.byref(self.h))
        if st:
            raise RiemannError(f"create failed: {st}")
        self.nparam = self.L.flash_hy_rsolver_num_params()
        self.stream = self.torch.cuda.ExternalStream(self.L.flash_hy_rsolver_stream(self.h), device=f"cuda:{device}")

    def close(self):
        if self.h:
            self.L.flash_hy_rsolver_destroy(self.h)
            self.h = C.c_void_p()

    def _check(self, st):
        if st:
            raise RiemannError(f"status {st:#x}")

    def _enter(self):
        # the library works on its own stream: order it after torch's work
        self.stream.wait_stream(self.torch.cuda.current_stream())

    def _leave(self):
        self.torch.cuda.current_stream().wait_stream(self.stream)

    def empty(self, *shape, dtype=None):
        return self.torch.empty(*shape, dtype=dtype or self.torch.float64, device=f"cuda:{self.device}")

    def generate(self, seed, n):
        S = self.empty(7, n)
        self._enter()
        self._check(self.L.flash_hy_rsolver_generate(self.h, seed, n, S.data_ptr()))
        self._leave()
        return S

    def solve(self, S, learned, tol=1e-12, max_iter=50, out=None, iters=None, flags=None):
        n = S.shape[1]
        out = self.empty(2, n) if out is None else out
        iters = self.empty(n, dtype=self.torch.uint8) if iters is None else iters
        flags = self.empty(n, dtype=self.torch.uint8) if flags is None else flags
        self._enter()
        self._check(self.L.flash_hy_rsolver_solve(self.h, S.data_ptr(), n, out.data_ptr(), iters.data_ptr(),
                                                  flags.data_ptr(), int(learned), tol, max_iter))
        self._leave()
        return out, iters, flags

    def predict(self, S):
        n = S.shape[1]
        y = self.empty(n, dtype=self.torch.float32)
        self._enter()
        self._check(self.L.flash_hy_rsolver_predict(self.h, S.data_ptr(), n, y.data_ptr()))
        self._leave()
        return y

    def make_samples(self, S, star, cap=None):
        n = S.shape[1]
        cap = n if cap is None else cap
        X = self.empty(cap, 8, dtype=self.torch.float32)
        T = self.empty(cap, dtype=self.torch.float32)
        cnt = C.c_long()
        self._enter()
        self._check(self.L.flash_hy_rsolver_make_samples(self.h, S.data_ptr(), star.data_ptr(), n, X.data_ptr(),
                                                         T.data_ptr(), cap, C.byref(cnt)))
        return X, T, cnt.value

    def grad(self, X, T, idx):
        g = np.zeros(self.nparam, np.float32)
        loss = C.c_float()
        self._enter()
        self._check(self.L.flash_hy_rsolver_grad(self.h, X.data_ptr(), T.data_ptr(), idx.data_ptr(), idx.numel(),
                                                 g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)))
        return g, loss.value

    def train(self, X, T, ns, epochs=4, batch=4096, lr=2e-3):
        loss = C.c_float()
        self._enter()
        self._check(self.L.flash_hy_rsolver_train(self.h, X.data_ptr(), T.data_ptr(), ns, epochs, batch, lr,
                                                  C.byref(loss)))
        return loss.value

    def fit(self, S, epochs=8, batch=4096, lr=2e-3):
        """Train the guess on interface states S ([7, n] CUDA tensor, e.g. the
        face states harvested by Hydro.harvest_fetch): solve them from the
        two-rarefaction guess, build (features, ln(p*/p_TR)) samples where
        that guess is inexact, run the Adam training kernels.  Returns
        (final loss, number of samples)."""
        out, _, _ = self.solve(S, learned=False)
        X, T, ns = self.make_samples(S, out)
        if ns < batch:
            raise RiemannError(f"only {ns} training samples (batch {batch})")
        return self.train(X, T, ns, epochs=epochs, batch=batch, lr=lr), ns

    def weights(self):
        w = np.zeros(self.nparam, np.float32)
        self._check(self.L.flash_hy_rsolver_get_weights(self.h, w.ctypes.data_as(C.POINTER(C.c_float)), self.nparam))
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._check(self.L.flash_hy_rsolver_set_weights(self.h, w.ctypes.data_as(C.POINTER(C.c_float)), self.nparam))

    def set_inference(self, mode):
        """Run the network of solve(learned=True) and predict() on the tcgen05
        tensor cores (INFER_TCGEN05, default) or per warp on mma.sync
        (INFER_WARP_MMA)."""
        self._check(self.L.flash_hy_rsolver_set_inference(self.h, int(mode)))

    def sync(self):
        return self.L.flash_hy_rsolver_sync(self.h)
