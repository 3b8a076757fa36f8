"""Differentiable float32 SGM: the CUDA forward/backward kernels (csrc/float_sgm.cu) behind a
torch.autograd.Function, plus a plain-PyTorch restatement used by the tests as the autograd and
finite-difference reference.

    disp = float_sgm(cost, p1, p2, temperature=1.0)   # cost [B,H,W,D] float32 CUDA, p1/p2 [B,H,W]
"""
from __future__ import annotations

import ctypes as C

import torch

from . import load_library

_PATHS = ((1, False), (2, False), (1, True), (2, True))  # (scan dim, reversed): T->B, L->R, B->T, R->L


def _lib():
    lib = load_library()
    if not hasattr(lib, "_float_sgm_bound"):
        vp, i32, f32 = C.c_void_p, C.c_int32, C.c_float
        lib.sgm_float_checkpoint_elems.argtypes = [i32, i32, i32, i32]
        lib.sgm_float_checkpoint_elems.restype = C.c_size_t
        lib.sgm_float_workspace_elems.argtypes = [i32, i32, i32, i32]
        lib.sgm_float_workspace_elems.restype = C.c_size_t
        lib.sgm_float_forward.argtypes = [vp, vp, vp, i32, i32, i32, i32, f32, vp, vp, vp, vp, vp]
        lib.sgm_float_forward.restype = i32
        lib.sgm_float_backward.argtypes = [vp, vp, vp, i32, i32, i32, i32, f32, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        lib.sgm_float_backward.restype = i32
        lib._float_sgm_bound = True
    return lib


def _aligned(t):
    """the kernels read the cost volume with 16-byte vector loads"""
    return t if t.data_ptr() % 16 == 0 else t.clone()


class FloatSGM(torch.autograd.Function):
    @staticmethod
    def forward(ctx, cost, p1, p2, temperature=1.0):
        if not (cost.is_cuda and cost.dtype == torch.float32 and cost.dim() == 4):
            raise ValueError("cost must be a float32 CUDA tensor [B,H,W,D]")
        cost, p1, p2 = _aligned(cost.contiguous()), p1.contiguous().float(), p2.contiguous().float()
        B, H, W, D = cost.shape
        lib = _lib()
        sum_ = torch.empty_like(cost)
        ckpt = torch.empty(lib.sgm_float_checkpoint_elems(B, H, W, D), dtype=torch.float32, device=cost.device)
        work = torch.empty(lib.sgm_float_workspace_elems(B, H, W, D), dtype=torch.float32, device=cost.device)
        disp = torch.empty((B, H, W), dtype=torch.float32, device=cost.device)
        st = lib.sgm_float_forward(cost.data_ptr(), p1.data_ptr(), p2.data_ptr(), B, H, W, D, float(temperature),
                                   sum_.data_ptr(), ckpt.data_ptr(), work.data_ptr(), disp.data_ptr(),
                                   torch.cuda.current_stream(cost.device).cuda_stream)
        if st != 0:
            raise RuntimeError(f"float SGM forward failed: {lib.sgm_last_error(None).decode()}")
        ctx.save_for_backward(cost, p1, p2, sum_, ckpt)
        ctx.temperature = float(temperature)
        return disp

    @staticmethod
    def backward(ctx, grad_disp):
        cost, p1, p2, sum_, ckpt = ctx.saved_tensors
        B, H, W, D = cost.shape
        lib = _lib()
        g = grad_disp.contiguous().float()
        gsum = torch.empty_like(cost)
        gcost = torch.empty_like(cost)
        gp1 = torch.empty_like(p1)
        gp2 = torch.empty_like(p2)
        work = torch.empty(lib.sgm_float_workspace_elems(B, H, W, D), dtype=torch.float32, device=cost.device)
        st = lib.sgm_float_backward(cost.data_ptr(), p1.data_ptr(), p2.data_ptr(), B, H, W, D, ctx.temperature,
                                    sum_.data_ptr(), ckpt.data_ptr(), g.data_ptr(), gsum.data_ptr(),
                                    work.data_ptr(), gcost.data_ptr(), gp1.data_ptr(), gp2.data_ptr(),
                                    torch.cuda.current_stream(cost.device).cuda_stream)
        if st != 0:
            raise RuntimeError(f"float SGM backward failed: {lib.sgm_last_error(None).decode()}")
        return gcost, gp1, gp2, None


def float_sgm(cost, p1, p2, temperature: float = 1.0):
    return FloatSGM.apply(cost, p1, p2, temperature)


def reference_sgm(cost, p1, p2, temperature: float = 1.0, return_sum: bool = False):
    """The same function in plain PyTorch ops (any device / dtype; differentiable by autograd)."""
    B, H, W, D = cost.shape
    inf = torch.full(cost.shape[:-1] + (1,), float("inf"), dtype=cost.dtype, device=cost.device)
    total = 0
    for dim, rev in _PATHS:
        n = cost.shape[dim]
        idx = range(n - 1, -1, -1) if rev else range(n)
        outs = [None] * n
        L = None
        for s, k in enumerate(idx):
            c = cost.select(dim, k)
            if s == 0:
                L = c
            else:
                P1 = p1.select(dim, k).unsqueeze(-1)
                P2 = p2.select(dim, k).unsqueeze(-1)
                m = L.min(-1, keepdim=True).values
                ninf = inf.select(dim, 0)
                lm = torch.cat([ninf, L[..., :-1]], -1) + P1
                lp = torch.cat([L[..., 1:], ninf], -1) + P1
                t = torch.minimum(torch.minimum(torch.minimum(L, lm), lp), m + P2)
                L = c + t - m
            outs[k] = L
        total = total + torch.stack(outs, dim)
    w = torch.softmax(-total / temperature, dim=-1)
    d = torch.arange(D, dtype=cost.dtype, device=cost.device)
    disp = (w * d).sum(-1)
    return (disp, total) if return_sum else disp
