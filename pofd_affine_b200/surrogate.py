"""Online-trained MLP surrogate of the log-likelihood (BF16 tensor cores)
and the delayed-acceptance stretch move built on it.

The reference has no surrogate: this is the learned first stage of a
two-stage delayed-acceptance step (Christen & Fox 2005) on top of the
reference's stretch move, so the exact P(D) likelihood still decides every
accepted step.

  * Surrogate     pairs buffer, train (Adam), predict, parameters, gradients
  * bf16_gemm     the tensor-core GEMM main loop on torch tensors
"""
import ctypes as C

import numpy as np

from ._lib import PofdError, check, lib  # noqa: F401

NUM_TENSORS = 8
TENSOR_NAMES = ["W1", "b1", "W2", "b2", "W3", "b3", "w4", "b4"]


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise PofdError(-11, "the surrogate needs a CUDA device")
    return torch


def bf16_gemm(A, B, stream=None):
    """C = A @ B.T in FP32 on the tensor cores; A [M, K], B [N, K] bf16 CUDA
    tensors (contiguous)."""
    torch = _torch()
    M, K = A.shape
    N = B.shape[0]
    Cm = torch.empty((M, N), dtype=torch.float32, device=A.device)
    st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    check(lib().pofd_bf16_gemm(M, N, K, C.c_void_p(A.data_ptr()), A.stride(0),
                               C.c_void_p(B.data_ptr()), B.stride(0),
                               C.c_void_p(Cm.data_ptr()), Cm.stride(0),
                               C.c_void_p(st)))
    return Cm


class Surrogate:
    """MLP logL surrogate over the parameters listed in `inputs`."""

    def __init__(self, ctx, nparams, inputs, hidden=256, capacity=65536,
                 seed=0):
        idx = np.ascontiguousarray(inputs, dtype=np.int32)
        h = C.c_void_p()
        check(lib().pofd_surrogate_create(ctx.h, int(nparams), idx, idx.size,
                                          int(hidden), int(capacity),
                                          int(seed), C.byref(h)))
        self.h, self.ctx = h, ctx
        self.nparams, self.nin, self.hidden = int(nparams), idx.size, int(hidden)

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().pofd_surrogate_destroy(self.h)
            except Exception:  # interpreter shutdown: the library is gone
                pass
            self.h = None

    # ------------------------------------------------------------ pairs
    def addPairs(self, theta, logl, status=None):
        torch = _torch()
        th = torch.as_tensor(np.ascontiguousarray(theta, np.float32)).cuda()
        ll = torch.as_tensor(np.ascontiguousarray(logl, np.float64)).cuda()
        st = None
        if status is not None:
            st = torch.as_tensor(np.ascontiguousarray(status, np.int32)).cuda()
        torch.cuda.synchronize()
        check(lib().pofd_surrogate_add_pairs(
            self.h, th.shape[0], C.c_void_p(th.data_ptr()), th.shape[1],
            C.c_void_p(ll.data_ptr()),
            C.c_void_p(st.data_ptr()) if st is not None else None, None))
        self.nPairs()  # synchronises

    def nPairs(self):
        n = C.c_uint()
        check(lib().pofd_surrogate_npairs(self.h, C.byref(n)))
        return n.value

    def getPairs(self, n=None):
        """The training pairs held (buffer order): (theta [n][nparams]
        float32, logl [n] float64)."""
        n = self.nPairs() if n is None else int(n)
        th = np.empty((n, self.nparams), np.float32)
        ll = np.empty(n, np.float64)
        check(lib().pofd_surrogate_get_pairs(self.h, n,
                                             th.ctypes.data_as(C.c_void_p),
                                             ll.ctypes.data_as(C.c_void_p)))
        return th, ll

    # ---------------------------------------------------------- training
    def train(self, iters, batch=1024, lr=1e-3):
        loss = C.c_float()
        check(lib().pofd_surrogate_train(self.h, int(iters), int(batch),
                                         float(lr), C.byref(loss)))
        return loss.value

    def predict(self, theta):
        torch = _torch()
        th = torch.as_tensor(np.ascontiguousarray(theta, np.float32)).cuda()
        out = torch.empty(th.shape[0], dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        check(lib().pofd_surrogate_predict_device(
            self.h, th.shape[0], C.c_void_p(th.data_ptr()), th.shape[1],
            C.c_void_p(out.data_ptr()), None, None))
        lib().pofd_ctx_synchronize(self.ctx.h)
        return out.cpu().numpy()

    def rms(self, theta, logl):
        p = self.predict(theta)
        return float(np.sqrt(np.mean((p - np.asarray(logl)) ** 2)))

    # -------------------------------------------------------- parameters
    def getParams(self):
        out = []
        for t in range(NUM_TENSORS):
            n = C.c_size_t()
            check(lib().pofd_surrogate_get_params(self.h, t, None, C.byref(n)))
            a = np.empty(n.value, np.float32)
            check(lib().pofd_surrogate_get_params(
                self.h, t, a.ctypes.data_as(C.c_void_p), C.byref(n)))
            out.append(a)
        return out

    def setParams(self, tensors):
        arrs = [np.ascontiguousarray(a, np.float32) for a in tensors]
        ptrs = (C.c_void_p * NUM_TENSORS)(*[a.ctypes.data_as(C.c_void_p)
                                            for a in arrs])
        check(lib().pofd_surrogate_set_params(self.h, ptrs))

    def gradients(self, n):
        sizes = [p.size for p in self.getParams()]
        grads = [np.empty(s, np.float32) for s in sizes]
        ptrs = (C.c_void_p * NUM_TENSORS)(*[g.ctypes.data_as(C.c_void_p)
                                            for g in grads])
        loss = C.c_float()
        check(lib().pofd_surrogate_gradients(self.h, int(n), ptrs,
                                             C.byref(loss)))
        return grads, loss.value

    def scaling(self):
        """Input transform x = W (theta_free - mu) and target scaling of the
        last training."""
        o = np.empty(276)
        check(lib().pofd_surrogate_scaling(self.h, o))
        return {"mu": o[:16], "W": o[16:272].reshape(16, 16), "ymax": o[272],
                "ys": o[273], "clip": o[274], "whitened": bool(o[275])}
