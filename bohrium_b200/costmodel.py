"""The learned fusion cost model: feature scaling, training and the model file.

The network (an MLP of 16 features -> 64 -> 64 -> 1, float32) is trained and evaluated on the
GPU by the hand-written kernels of libbh_ve_cuda.so (bh_ve_cuda_costmodel_*, declared in
include/bh_b200.h). Its input is the feature vector of a fused block that the engine computes
(bohrium_b200/csrc/jitk/costmodel.cpp) and records, with the block's measured device time, when
recording is on (message "CUDA: record on"). The target is log(time in microseconds), and features
and target are standardised with the training set's mean and deviation.

Model file (little endian), read by the engine with message "CUDA: costmodel load <path>":
    8 bytes  magic b"BHCM0001"
    int32    number of features F, int32 number of parameters P
    float32  feature mean[F], feature std[F], target mean, target std
    float32  parameters[P] (W1[64][F], b1[64], W2[64][64], b2[64], W3[64], b3)
"""
from __future__ import annotations

import ctypes
import os
import struct

import numpy as np

from .runtime import LIB_DIR, load_library

MAGIC = b"BHCM0001"
_ve = None


def _lib():
    global _ve
    if _ve is None:
        load_library()  # libbh_core.so (bhb_last_error) first, with global symbols
        lib = ctypes.CDLL(os.path.join(LIB_DIR, "libbh_ve_cuda.so"))
        P, I64, F32P = ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_float)
        sig = {
            "bh_ve_cuda_costmodel_nfeatures": (ctypes.c_int, []),
            "bh_ve_cuda_costmodel_nparams": (I64, []),
            "bh_ve_cuda_costmodel_create": (P, [ctypes.c_uint64]),
            "bh_ve_cuda_costmodel_destroy": (None, [P]),
            "bh_ve_cuda_costmodel_get_params": (ctypes.c_int, [P, P]),
            "bh_ve_cuda_costmodel_set_params": (ctypes.c_int, [P, P]),
            "bh_ve_cuda_costmodel_predict": (ctypes.c_int, [P, P, I64, P]),
            "bh_ve_cuda_costmodel_gradient": (ctypes.c_int, [P, P, P, I64, P, F32P]),
            "bh_ve_cuda_costmodel_train": (ctypes.c_int, [P, P, P, I64, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                                          ctypes.c_uint64, F32P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _ve = lib
    return _ve


def _err() -> str:
    return (load_library().bhb_last_error() or b"").decode(errors="replace")


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


class Network:
    """The GPU network on the current device (raw inputs and outputs, no scaling)."""

    def __init__(self, seed: int = 0):
        self.lib = _lib()
        self.nfeat = int(self.lib.bh_ve_cuda_costmodel_nfeatures())
        self.nparams = int(self.lib.bh_ve_cuda_costmodel_nparams())
        self.h = self.lib.bh_ve_cuda_costmodel_create(seed)
        if not self.h:
            raise RuntimeError("bh_ve_cuda_costmodel_create: " + _err())

    def close(self):
        if self.h:
            self.lib.bh_ve_cuda_costmodel_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _rows(self, X) -> np.ndarray:
        X = _f32(X)
        if X.ndim != 2 or X.shape[1] != self.nfeat:
            raise ValueError(f"features must have shape (rows, {self.nfeat})")
        return X

    @property
    def params(self) -> np.ndarray:
        out = np.zeros(self.nparams, dtype=np.float32)
        if self.lib.bh_ve_cuda_costmodel_get_params(self.h, out.ctypes.data) != 0:
            raise RuntimeError(_err())
        return out

    @params.setter
    def params(self, p) -> None:
        p = _f32(p).reshape(-1)
        if p.size != self.nparams:
            raise ValueError("parameter count mismatch")
        if self.lib.bh_ve_cuda_costmodel_set_params(self.h, p.ctypes.data) != 0:
            raise RuntimeError(_err())

    def predict(self, X) -> np.ndarray:
        X = self._rows(X)
        y = np.zeros(X.shape[0], dtype=np.float32)
        if self.lib.bh_ve_cuda_costmodel_predict(self.h, X.ctypes.data, X.shape[0], y.ctypes.data) != 0:
            raise RuntimeError(_err())
        return y

    def gradient(self, X, t):
        X, t = self._rows(X), _f32(t)
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = ctypes.c_float()
        if self.lib.bh_ve_cuda_costmodel_gradient(self.h, X.ctypes.data, t.ctypes.data, X.shape[0], g.ctypes.data,
                                                  ctypes.byref(loss)) != 0:
            raise RuntimeError(_err())
        return float(loss.value), g

    def train(self, X, t, epochs: int = 100, batch: int = 256, lr: float = 1e-3, seed: int = 0) -> float:
        X, t = self._rows(X), _f32(t)
        loss = ctypes.c_float()
        if self.lib.bh_ve_cuda_costmodel_train(self.h, X.ctypes.data, t.ctypes.data, X.shape[0], epochs, batch, lr,
                                               seed, ctypes.byref(loss)) != 0:
            raise RuntimeError(_err())
        return float(loss.value)


class CostModel:
    """Network plus the feature and target scaling of its training set."""

    def __init__(self, seed: int = 0):
        self.net = Network(seed)
        self.mean = np.zeros(self.net.nfeat, dtype=np.float32)
        self.std = np.ones(self.net.nfeat, dtype=np.float32)
        self.tmean, self.tstd = 0.0, 1.0

    def fit(self, features, times_us, epochs: int = 200, batch: int = 256, lr: float = 2e-3, seed: int = 0) -> float:
        X = np.asarray(features, dtype=np.float64)
        y = np.log(np.maximum(np.asarray(times_us, dtype=np.float64), 1e-3))
        self.mean = X.mean(axis=0).astype(np.float32)
        self.std = np.maximum(X.std(axis=0), 1e-6).astype(np.float32)
        # float32, as stored in the model file and used by the engine
        self.tmean, self.tstd = float(np.float32(y.mean())), float(np.float32(max(y.std(), 1e-6)))
        return self.net.train(self.scale(X), (y - self.tmean) / self.tstd, epochs=epochs, batch=batch, lr=lr,
                              seed=seed)

    def scale(self, features) -> np.ndarray:
        return ((np.asarray(features, dtype=np.float32) - self.mean) / self.std).astype(np.float32)

    def predict_us(self, features) -> np.ndarray:
        z = self.net.predict(self.scale(features)).astype(np.float64)
        return np.exp(z * self.tstd + self.tmean)

    def save(self, path: str) -> None:
        p = self.net.params
        with open(path, "wb") as f:
            f.write(MAGIC)
            f.write(struct.pack("<ii", self.net.nfeat, p.size))
            f.write(self.mean.astype("<f4").tobytes())
            f.write(self.std.astype("<f4").tobytes())
            f.write(struct.pack("<ff", self.tmean, self.tstd))
            f.write(p.astype("<f4").tobytes())

    @classmethod
    def load(cls, path: str) -> "CostModel":
        m = cls()
        with open(path, "rb") as f:
            if f.read(8) != MAGIC:
                raise ValueError(f"{path}: not a cost model file")
            nf, npar = struct.unpack("<ii", f.read(8))
            if nf != m.net.nfeat or npar != m.net.nparams:
                raise ValueError(f"{path}: shape mismatch")
            m.mean = np.frombuffer(f.read(4 * nf), dtype="<f4").astype(np.float32)
            m.std = np.frombuffer(f.read(4 * nf), dtype="<f4").astype(np.float32)
            m.tmean, m.tstd = struct.unpack("<ff", f.read(8))
            m.net.params = np.frombuffer(f.read(4 * npar), dtype="<f4")
        return m


def read_records(path: str):
    """Training records dumped by the engine (message "CUDA: records dump <path>"): float32 rows
    of F features followed by the measured device time in microseconds."""
    raw = np.fromfile(path, dtype="<f4")
    nf = 16
    raw = raw.reshape(-1, nf + 1)
    return raw[:, :nf].copy(), raw[:, nf].astype(np.float64)
