"""Learned SGS closure: host side of the tensor-core MLP (include/diablo_b200.h,
db_sgs_*).  Feature vectors, targets and outputs live in device memory
(torch CUDA tensors are used for the plumbing); parameters cross as FP32
host arrays in the packed order W1[64][16] b1 W2[64][64] b2 W3[64][64] b3
W4[2][64] b4.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import lib as _L

NFEAT = 16
NHID = 64
NOUT = 2
NPARAMS = 9538
OFFSETS = {"W1": (0, (64, 16)), "b1": (1024, (64,)), "W2": (1088, (64, 64)), "b2": (5184, (64,)),
           "W3": (5248, (64, 64)), "b3": (9344, (64,)), "W4": (9408, (2, 64)), "b4": (9536, (2,))}


def unpack(params: np.ndarray) -> dict:
    return {k: params[o:o + int(np.prod(sh))].reshape(sh) for k, (o, sh) in OFFSETS.items()}


def pack(d: dict) -> np.ndarray:
    out = np.zeros(NPARAMS, np.float32)
    for k, (o, sh) in OFFSETS.items():
        out[o:o + int(np.prod(sh))] = np.asarray(d[k], np.float32).reshape(-1)
    return out


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation (zero biases)."""
    rng = np.random.default_rng(seed)
    d = {}
    for k, (o, sh) in OFFSETS.items():
        if k.startswith("W"):
            d[k] = rng.standard_normal(sh) * np.sqrt(2.0 / sh[1])
        else:
            d[k] = np.zeros(sh)
    return pack(d)


def _vp(t):
    """Device pointer of a contiguous torch CUDA tensor."""
    assert t.is_cuda and t.is_contiguous()
    return ctypes.c_void_p(t.data_ptr())


class SgsNet:
    def __init__(self, stream: int | None = None):
        self.L = _L.load()
        h = ctypes.c_void_p()
        _L.check(self.L.db_sgs_create(ctypes.c_void_p(stream) if stream else None, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.db_sgs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set(self, params, feat_mean, feat_std, out_scale):
        p = np.ascontiguousarray(params, np.float32)
        m = np.ascontiguousarray(feat_mean, np.float32)
        sd = np.ascontiguousarray(feat_std, np.float32)
        os_ = np.ascontiguousarray(out_scale, np.float32)
        assert p.shape == (NPARAMS,) and m.shape == (NFEAT,) and sd.shape == (NFEAT,) and os_.shape == (NOUT,)
        _L.check(self.L.db_sgs_set(self.h, _L.fptr(p), _L.fptr(m), _L.fptr(sd), _L.fptr(os_)))

    def set_range(self, lo, hi):
        """Training range of the raw features; outside it the channel step
        keeps AMD's coefficients."""
        a = np.ascontiguousarray(lo, np.float32)
        b = np.ascontiguousarray(hi, np.float32)
        _L.check(self.L.db_sgs_set_range(self.h, _L.fptr(a), _L.fptr(b)))

    def get(self) -> np.ndarray:
        p = np.zeros(NPARAMS, np.float32)
        _L.check(self.L.db_sgs_get(self.h, _L.fptr(p)))
        return p

    def forward(self, feat, out=None):
        """feat: CUDA float32 tensor [n][16] -> [n][2] (nu_t, kappa_t)."""
        import torch
        n = feat.shape[0]
        if out is None:
            out = torch.empty((n, NOUT), dtype=torch.float32, device=feat.device)
        _L.check(self.L.db_sgs_forward(self.h, _vp(feat), _vp(out), n))
        return out

    def gradient(self, feat, target):
        g = np.zeros(NPARAMS, np.float32)
        loss = ctypes.c_double()
        _L.check(self.L.db_sgs_gradient(self.h, _vp(feat), _vp(target), feat.shape[0], _L.fptr(g),
                                        ctypes.byref(loss)))
        return g, loss.value

    def train_step(self, feat, target, lr: float = 1e-3) -> float:
        loss = ctypes.c_double()
        _L.check(self.L.db_sgs_train_step(self.h, _vp(feat), _vp(target), feat.shape[0], ctypes.c_float(lr),
                                          ctypes.byref(loss)))
        return loss.value


def gemm_check(a_bits: np.ndarray, b_bits: np.ndarray) -> np.ndarray:
    """D[128][N] = A[128][K] B[N][K]^T through the tensor-core path; A, B as
    uint16 BF16 bit patterns."""
    L = _L.load()
    a = np.ascontiguousarray(a_bits, np.uint16)
    b = np.ascontiguousarray(b_bits, np.uint16)
    K = a.shape[1]
    N = b.shape[0]
    assert a.shape == (128, K) and b.shape == (N, K)
    d = np.zeros((128, N), np.float32)
    _L.check(L.db_sgs_gemm_check(a.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p),
                                 _L.fptr(d), K, N))
    return d
