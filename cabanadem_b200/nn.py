"""Dense layers of the learned surrogate, run by the library's tensor-core kernels
(``dem_nn_mlp_forward`` / ``dem_nn_mlp_backward``).  torch tensors only hold device memory
here; every multiply-accumulate of a layer happens in the library.

A layer is the two-layer perceptron y = W2 relu(W1 x + b1) + b2 with hidden width 128.  The
FP32 master weights are kept with their BF16 copies in both layouts the kernels read
(W^T for the forward pass, W for the input gradient)."""
from __future__ import annotations

import ctypes as C

import torch

from ._lib import NnMlp, NnRows, check, lib

HIDDEN = 128
SHAPES = ((16, 128), (128, 128), (256, 128), (384, 128), (128, 16))


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class Mlp:
    def __init__(self, kin: int, nout: int, device, gen: torch.Generator | None = None, out_scale: float = 1.0):
        if (kin, nout) not in SHAPES:
            raise ValueError("unsupported layer shape %r" % ((kin, nout),))
        self.kin, self.nout = kin, nout
        f32 = dict(device=device, dtype=torch.float32)
        self.w1t = torch.randn(HIDDEN, kin, generator=gen, device="cpu").mul_((2.0 / kin) ** 0.5).to(**f32)
        self.b1 = torch.zeros(HIDDEN, **f32)
        self.w2t = torch.randn(nout, HIDDEN, generator=gen, device="cpu").mul_(out_scale * (1.0 / HIDDEN) ** 0.5).to(**f32)
        self.b2 = torch.zeros(nout, **f32)
        self.grads = [torch.zeros_like(p) for p in self.params()]
        self.sync_bf16()

    def params(self):
        return [self.w1t, self.b1, self.w2t, self.b2]

    def sync_bf16(self):
        """Refresh the BF16 operand copies from the FP32 master weights."""
        self.w1t_bf = self.w1t.to(torch.bfloat16).contiguous()
        self.w1_bf = self.w1t.t().to(torch.bfloat16).contiguous()
        self.w2t_bf = self.w2t.to(torch.bfloat16).contiguous()
        self.w2_bf = self.w2t.t().to(torch.bfloat16).contiguous()
        self._desc = NnMlp(self.kin, self.nout, self.w1t_bf.data_ptr(), self.w1_bf.data_ptr(), self.b1.data_ptr(),
                           self.w2t_bf.data_ptr(), self.w2_bf.data_ptr(), self.b2.data_ptr())

    def zero_grad(self):
        for g in self.grads:
            g.zero_()

    @staticmethod
    def _rows(srcs):
        arr = (NnRows * len(srcs))()
        for k, (data, index) in enumerate(srcs):
            arr[k] = NnRows(data.data_ptr(), index.data_ptr() if index is not None else None, data.shape[1])
        return arr

    def forward(self, ctx, rows: int, srcs, resid=None, out=None, out_f32=None, h1=None):
        """srcs: sequence of (bf16 [*, width] tensor, int32 row index or None)."""
        arr = self._rows(srcs)
        st = lib().dem_nn_mlp_forward(ctx.h, C.byref(self._desc), rows, arr, len(srcs), _ptr(resid), _ptr(out),
                                      _ptr(out_f32), _ptr(h1))
        check(st, ctx.h, "dem_nn_mlp_forward")

    def backward(self, ctx, rows: int, srcs, dy, h1, dz1, dx=None):
        arr = self._rows(srcs)
        g = self.grads
        st = lib().dem_nn_mlp_backward(ctx.h, C.byref(self._desc), rows, arr, len(srcs), _ptr(dy), _ptr(h1),
                                       _ptr(dz1), _ptr(dx), _ptr(g[0]), _ptr(g[1]), _ptr(g[2]), _ptr(g[3]))
        check(st, ctx.h, "dem_nn_mlp_backward")


def status(ctx) -> int:
    """Error word of the tensor-core kernels (synchronises and clears it)."""
    v = C.c_int(0)
    check(lib().dem_nn_status(ctx.h, C.byref(v)), ctx.h, "dem_nn_status")
    return v.value


def edge_forward(ctx, e, pq, recv, send, w1e_t, b1, w2t, b2, out, h1=None, form: int = 0):
    """The factorised message layer (``dem_nn_edge_forward``): out = e + b2 + W2 relu(W1e e + b1
    + P[recv] + Q[send]), PQ = [W1i h | W1j h] per node.  Tensors on the context's device: e, out
    bf16 [rows][128], pq bf16 [nodes][256], recv/send int32 [rows], w1e_t/w2t bf16 [128][128],
    b1/b2 float32 [128], h1 bf16 [rows][128] or None.  form 0: tensor-copy tiles and the hidden
    tile in tensor memory; 1: per-thread staged copies (same results)."""
    st = lib().dem_nn_edge_forward(ctx.h, int(e.shape[0]), _ptr(e), _ptr(pq), _ptr(recv), _ptr(send), _ptr(w1e_t),
                                   _ptr(b1), _ptr(w2t), _ptr(b2), _ptr(out), _ptr(h1), int(form))
    check(st, ctx.h, "dem_nn_edge_forward")
