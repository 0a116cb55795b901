"""Python handle on the proposal network of include/mbs_mlp.h (BF16
tensor-core forward/backward kernels and Adam training on the device)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi

N_PARAMS = 128 * 4 + 128 + 128 * 128 + 128 + 128 * 128 + 128 + 128 + 1
_fp = C.POINTER(C.c_float)
_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = abi.load("libmbs_po_b200.so")
        vp = C.c_void_p
        L.mbs_mlp_create.argtypes = [C.POINTER(vp), C.c_int, C.c_uint64]
        L.mbs_mlp_destroy.argtypes = [vp]
        L.mbs_mlp_last_error.argtypes = [vp]
        L.mbs_mlp_last_error.restype = C.c_char_p
        L.mbs_mlp_get_params.argtypes = [vp, _fp]
        L.mbs_mlp_set_params.argtypes = [vp, _fp]
        L.mbs_mlp_forward.argtypes = [vp, _fp, C.c_int, _fp]
        L.mbs_mlp_loss_grad.argtypes = [vp, _fp, _fp, C.c_int, _fp, _fp]
        L.mbs_mlp_train.argtypes = [vp, _fp, _fp, C.c_int, C.c_int, C.c_int, C.c_float,
                                    C.c_uint64, _fp]
        L.mbs_mlp_set_watchdog.argtypes = [vp, C.c_int, C.c_int]
        _lib = L
    return _lib


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


class ProposalNet:
    """4 -> 128 -> 128 -> 128 -> 1 GELU network on one device."""

    def __init__(self, device: int = 0, seed: int = 1):
        self.h = C.c_void_p()
        rc = lib().mbs_mlp_create(C.byref(self.h), device, seed)
        if rc:
            raise RuntimeError(f"mbs_mlp_create failed ({rc})")

    def _call(self, rc: int, what: str) -> None:
        if rc:
            msg = lib().mbs_mlp_last_error(self.h)
            raise RuntimeError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")

    def close(self) -> None:
        if self.h:
            lib().mbs_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(N_PARAMS, np.float32)
        self._call(lib().mbs_mlp_get_params(self.h, abi.ptr(p, C.c_float)), "mbs_mlp_get_params")
        return p

    @params.setter
    def params(self, p) -> None:
        p = _f32(p)
        assert p.shape == (N_PARAMS,)
        self._call(lib().mbs_mlp_set_params(self.h, abi.ptr(p, C.c_float)), "mbs_mlp_set_params")

    def set_watchdog(self, poll_limit: int = 0, skip_mma: bool = False) -> None:
        """Poll limit of the GEMMs' barrier waits (0: default); skip_mma is
        the test hook that makes the waits run out (mbs_mlp_set_watchdog)."""
        self._call(lib().mbs_mlp_set_watchdog(self.h, poll_limit, int(skip_mma)),
                   "mbs_mlp_set_watchdog")

    def forward(self, q) -> np.ndarray:
        q = _f32(q).reshape(-1, 4)
        y = np.zeros(len(q), np.float32)
        self._call(lib().mbs_mlp_forward(self.h, abi.ptr(q, C.c_float), len(q),
                                         abi.ptr(y, C.c_float)), "mbs_mlp_forward")
        return y

    def loss_grad(self, q, t):
        q, t = _f32(q).reshape(-1, 4), _f32(t)
        loss = C.c_float()
        g = np.zeros(N_PARAMS, np.float32)
        self._call(lib().mbs_mlp_loss_grad(self.h, abi.ptr(q, C.c_float), abi.ptr(t, C.c_float),
                                           len(t), C.byref(loss), abi.ptr(g, C.c_float)),
                   "mbs_mlp_loss_grad")
        return float(loss.value), g

    def train(self, q, t, epochs: int = 200, batch: int = 256, lr: float = 2e-3,
              seed: int = 7) -> float:
        q, t = _f32(q).reshape(-1, 4), _f32(t)
        loss = C.c_float()
        self._call(lib().mbs_mlp_train(self.h, abi.ptr(q, C.c_float), abi.ptr(t, C.c_float), len(t),
                                       epochs, batch, lr, seed, C.byref(loss)), "mbs_mlp_train")
        return float(loss.value)
