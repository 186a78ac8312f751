"""Host-side interface of the learned per-block preconditioner
(include/bx200.h, bx_learned_*): a new #PRECONDITIONER value LEARNED for the
implicit step's FGMRES, trained on (Krylov vector, BILU correction) pairs
that the BILU-preconditioned solver generates."""
import ctypes

import numpy as np

from . import capi
from .capi import check, dptr, fptr


class LearnedPreconditioner:
    def __init__(self, nSampleMax=32768, seed=2024, relu=False):
        self.L = capi.load()
        check(self.L.bx_learned_init(int(nSampleMax), int(seed)))
        if relu:
            check(self.L.bx_learned_set_activation(1))
        n = ctypes.c_int(0)
        check(self.L.bx_learned_nparam(ctypes.byref(n)))
        self.nparam = n.value

    def set_blend(self, blend):
        """weight of the learned remainder at inference (0: identity part only)"""
        check(self.L.bx_learned_set_blend(float(blend)))

    def close(self):
        self.L.bx_learned_finalize()

    def params(self):
        p = np.empty(self.nparam, dtype=np.float32)
        check(self.L.bx_learned_get_params(fptr(p), self.nparam))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(self.L.bx_learned_set_params(fptr(p), p.size))

    def collect(self, blocksPerPair):
        check(self.L.bx_learned_collect(int(blocksPerPair)))

    def collect_probes(self, nProbe, blocksPerPair, seed=1):
        """(v, BILU(v)) pairs of seeded probe vectors; call after an implicit
        step with the BILU preconditioner"""
        check(self.L.bx_learned_collect_probes(int(nProbe), int(blocksPerPair), int(seed)))

    def num_samples(self):
        n = ctypes.c_longlong(0)
        check(self.L.bx_learned_num_samples(ctypes.byref(n)))
        return n.value

    def set_samples(self, in16, tgt):
        in16 = np.ascontiguousarray(in16, dtype=np.float32)
        tgt = np.ascontiguousarray(tgt, dtype=np.float32)
        n = in16.shape[0]
        assert in16.size == n * 512 * 16 and tgt.size == n * 512 * 8
        check(self.L.bx_learned_set_samples(fptr(in16), fptr(tgt), n))

    def gradient(self, s0, nS):
        g = np.empty(self.nparam, dtype=np.float32)
        loss = ctypes.c_double(0)
        check(self.L.bx_learned_gradient(int(s0), int(nS), fptr(g), ctypes.byref(loss)))
        return loss.value, g

    def train(self, nEpoch=4, batch=256, lr=2e-3):
        a, b = ctypes.c_double(0), ctypes.c_double(0)
        check(self.L.bx_learned_train(int(nEpoch), int(batch), float(lr), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def apply_blocks(self, v, feat):
        v = np.ascontiguousarray(v, dtype=np.float64)
        feat = np.ascontiguousarray(feat, dtype=np.float32)
        nb = v.shape[0]
        z = np.empty_like(v)
        check(self.L.bx_learned_apply_blocks(dptr(v), fptr(feat), nb, dptr(z)))
        return z
