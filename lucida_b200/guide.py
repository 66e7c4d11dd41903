"""Host side of the learned path-guiding proposal (no counterpart in Lucida's
pt_gpu; the model is described in include/luc_cuda.h).

    guide = Guide(gpu)                  # seeded init, box = uploaded scene's bounds
    guide.configure(train=True, records_per_step=1 << 18, lr=1e-2)
    render_accum(gpu, scene, params, guided=True)   # one Adam step per batch

Everything runs through the C ABI of liblucida_cuda.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .native import GuideInfo, check, lib, ptr

NPARAMS = 19176
RECORD_FLOATS = 20


def records_array(x, n, wo, wi, F) -> np.ndarray:
    """Pack training records (N, 20): position, F, normal, -, outgoing
    direction, -, sampled direction, -, 4 unused."""
    x, n, wo, wi = (np.asarray(a, np.float32).reshape(-1, 3) for a in (x, n, wo, wi))
    r = np.zeros((len(x), RECORD_FLOATS), np.float32)
    r[:, 0:3], r[:, 3] = x, np.asarray(F, np.float32)
    r[:, 4:7], r[:, 8:11], r[:, 12:15] = n, wo, wi
    return r


class Guide:
    """The context's guide network: initialise, configure, inspect, train on
    host records, evaluate; renders use it through `guided=True`."""

    def __init__(self, gpu, params: np.ndarray | None = None, seed: int = 0, lo=None, hi=None):
        self.gpu = gpu
        self.reset(params, seed, lo, hi)

    def reset(self, params=None, seed: int = 0, lo=None, hi=None):
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        if p is not None and p.size != NPARAMS:
            raise ValueError(f"expected {NPARAMS} parameters, got {p.size}")
        lo_a = None if lo is None else np.ascontiguousarray(lo, np.float32)
        hi_a = None if hi is None else np.ascontiguousarray(hi, np.float32)
        check(self.gpu.handle, lib().luc_guide_init(self.gpu.handle, ptr(p), int(seed) & (2**64 - 1), ptr(lo_a),
                                                    ptr(hi_a)))

    def configure(self, train: bool = True, records_per_step: int = 1 << 18, lr: float = 1e-2):
        check(self.gpu.handle, lib().luc_guide_configure(self.gpu.handle, int(bool(train)), int(records_per_step),
                                                         float(lr)))

    def params(self) -> np.ndarray:
        out = np.zeros(NPARAMS, np.float32)
        check(self.gpu.handle, lib().luc_guide_get_params(self.gpu.handle, ptr(out)))
        return out

    def stats(self) -> GuideInfo:
        s = GuideInfo()
        check(self.gpu.handle, lib().luc_guide_stats(self.gpu.handle, C.byref(s)))
        return s

    def forward(self, x, n, wo, path: str = "tcgen05") -> np.ndarray:
        """Raw outputs (N, 40) for positions, shading normals and outgoing
        directions, through the tcgen05 tensor-core kernel or the mma.sync one."""
        a = np.ascontiguousarray(np.concatenate([np.asarray(v, np.float32).reshape(-1, 3) for v in (x, n, wo)], 1))
        out = np.zeros((len(a), 40), np.float32)
        code = {"tcgen05": 0, "mma.sync": 1}[path]
        check(self.gpu.handle, lib().luc_guide_forward_ex(self.gpu.handle, ptr(a), len(a), code, ptr(out)))
        return out

    def gradient(self, records: np.ndarray):
        """(gradient (NPARAMS,), loss) at the current parameters."""
        r = np.ascontiguousarray(records, np.float32).reshape(-1, RECORD_FLOATS)
        g = np.zeros(NPARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        check(self.gpu.handle, lib().luc_guide_train_records(self.gpu.handle, ptr(r), len(r), 0, ptr(g), ptr(loss)))
        return g, float(loss[0])

    def train(self, records: np.ndarray, steps: int = 1) -> float:
        """Take `steps` Adam steps on the records; returns the last loss."""
        if steps < 1:
            raise ValueError("steps must be positive")
        r = np.ascontiguousarray(records, np.float32).reshape(-1, RECORD_FLOATS)
        loss = np.zeros(1, np.float32)
        check(self.gpu.handle, lib().luc_guide_train_records(self.gpu.handle, ptr(r), len(r), int(steps), None,
                                                             ptr(loss)))
        return float(loss[0])

    def mixture_sample(self, raw: np.ndarray, u3: np.ndarray):
        raw = np.ascontiguousarray(raw, np.float32).reshape(-1, 40)
        u = np.ascontiguousarray(u3, np.float32).reshape(-1, 3)
        d = np.zeros((len(u), 3), np.float32)
        pdf = np.zeros(len(u), np.float32)
        check(self.gpu.handle, lib().luc_guide_mixture(self.gpu.handle, ptr(raw), ptr(u), len(u), 0, ptr(d), ptr(pdf)))
        return d, pdf

    def mixture_pdf(self, raw: np.ndarray, dirs: np.ndarray) -> np.ndarray:
        raw = np.ascontiguousarray(raw, np.float32).reshape(-1, 40)
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
        pdf = np.zeros(len(d), np.float32)
        check(self.gpu.handle, lib().luc_guide_mixture(self.gpu.handle, ptr(raw), ptr(d), len(d), 1, None, ptr(pdf)))
        return pdf
