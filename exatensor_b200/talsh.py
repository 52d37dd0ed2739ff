"""Python mirror of the talsh.h C API (TALSH/talsh.h, TALSH/talshxx.hpp).

``Tensor`` wraps a ``talsh_tens_t`` handle the way the reference's C++
``talsh::Tensor`` does (TALSH/talshxx.hpp:99): a dense tensor with images on
the Host and on GPUs.  Operations call the library's ``talshTensor*``
functions, so copy control, tasks and error codes behave as in TAL-SH.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib as _lib, R4, R8, C4, C8

TALSH_SUCCESS = 0
TALSH_NOT_AVAILABLE = -888
TALSH_NOT_IMPLEMENTED = -999
TALSH_INVALID_ARGS = 1000002
TALSH_TASK_COMPLETED = 2000005
DEV_NULL, DEV_DEFAULT, DEV_HOST, DEV_NVIDIA_GPU = -1, -1, 0, 1
COPY_D, COPY_M, COPY_T, COPY_K = 0, 1, 2, 3
COPY_MT, COPY_TT, COPY_MTT, COPY_TTT, COPY_KKK = 6, 10, 26, 42, 63
NP_DTYPE = {R4: np.float32, R8: np.float64, C4: np.complex64, C8: np.complex128}


class TalshError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what} returned {code}")
        self.code = code


_bound = False


def api() -> C.CDLL:
    global _bound
    L = _lib()
    if not _bound:
        vp, ip, d = C.c_void_p, C.c_int, C.c_double
        L.talshInit.argtypes = [C.POINTER(C.c_size_t), C.POINTER(C.c_int), ip, C.POINTER(C.c_int), ip, vp, ip, vp]
        L.talshTensorCreate.argtypes = [C.POINTER(vp)]
        L.talshTensorConstruct.argtypes = [vp, ip, ip, C.POINTER(C.c_int), ip, vp, ip, vp, d, d]
        L.talshTensorDestroy.argtypes = [vp]
        L.talshTensorVolume.argtypes = [vp]
        L.talshTensorVolume.restype = C.c_size_t
        L.talshTensorGetBodyAccess.argtypes = [vp, C.POINTER(vp), ip, ip, ip]
        L.talshTensorGetBodyAccessConst.argtypes = [vp, C.POINTER(vp), ip, ip, ip]
        L.talshTensorPlace.argtypes = [vp, ip, ip, vp, ip, vp]
        L.talshTensorPresence.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), ip, ip]
        L.talshTensorImageNorm1_cpu.argtypes = [vp]
        L.talshTensorImageNorm1_cpu.restype = d
        L.talshTensorGetScalar.argtypes = [vp, C.POINTER(d), C.POINTER(d)]
        L.talshTensorInit.argtypes = [vp, d, d, ip, ip, ip, vp]
        L.talshTensorScale.argtypes = [vp, d, d, ip, ip, ip, vp]
        L.talshTensorCopy.argtypes = [C.c_char_p, vp, vp, ip, ip, ip, vp]
        L.talshTensorAdd.argtypes = [C.c_char_p, vp, vp, d, d, ip, ip, ip, vp]
        L.talshTensorContract.argtypes = [C.c_char_p, vp, vp, vp, d, d, ip, ip, ip, ip, vp]
        L.talshTensorContractXL.argtypes = [C.c_char_p, vp, vp, vp, d, d, ip, ip, ip]
        L.tb_xl_last_split.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.talshTaskCreate.argtypes = [C.POINTER(vp)]
        L.talshTaskDestroy.argtypes = [vp]
        L.talshTaskWait.argtypes = [vp, C.POINTER(C.c_int)]
        L.talshTaskComplete.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.talshTaskTime.argtypes = [vp, C.POINTER(d), C.POINTER(d), C.POINTER(d), C.POINTER(d), C.POINTER(d)]
        L.talshEnableFastMath.argtypes = [ip, ip]
        L.talshDisableFastMath.argtypes = [ip, ip]
        _bound = True
    return L


def check(code, what):
    if code != TALSH_SUCCESS:
        raise TalshError(code, what)


def init(gpus=(0,)):
    n = len(gpus)
    arr = (C.c_int * max(1, n))(*gpus)
    hb, ha = C.c_size_t(1 << 20), C.c_int(0)
    return api().talshInit(C.byref(hb), C.byref(ha), n, arr, 0, None, 0, None)


def shutdown():
    return api().talshShutdown()


class Task:
    def __init__(self):
        self.h = C.c_void_p()
        check(api().talshTaskCreate(C.byref(self.h)), "talshTaskCreate")

    def wait(self) -> int:
        st = C.c_int()
        check(api().talshTaskWait(self.h, C.byref(st)), "talshTaskWait")
        return st.value

    def time(self):
        t = [C.c_double() for _ in range(5)]
        check(api().talshTaskTime(self.h, *[C.byref(x) for x in t]), "talshTaskTime")
        return [x.value for x in t]

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            api().talshTaskDestroy(self.h)
            self.h = C.c_void_p()


class Tensor:
    """A TAL-SH tensor block (dims first-fastest) with Host/GPU images."""

    def __init__(self, dims, data_kind=R8, init_val=0.0, dev_id=0, ext: np.ndarray | None = None):
        self.dims = list(dims)
        self.data_kind = data_kind
        self.h = C.c_void_p()
        self._ext = ext
        check(api().talshTensorCreate(C.byref(self.h)), "talshTensorCreate")
        v = complex(init_val)
        dims_arr = (C.c_int * max(1, len(self.dims)))(*self.dims)
        ext_p = C.c_void_p(ext.ctypes.data) if ext is not None else None
        check(api().talshTensorConstruct(self.h, data_kind, len(self.dims), dims_arr, dev_id, ext_p, -1, None,
                                         v.real, v.imag), "talshTensorConstruct")

    @property
    def volume(self) -> int:
        return api().talshTensorVolume(self.h)

    def host_array(self) -> np.ndarray:
        """A numpy view of the Host image (place the tensor on the Host first)."""
        p = C.c_void_p()
        check(api().talshTensorGetBodyAccessConst(self.h, C.byref(p), self.data_kind, 0, DEV_HOST),
              "talshTensorGetBodyAccessConst")
        dt = np.dtype(NP_DTYPE[self.data_kind])
        buf = (C.c_char * (self.volume * dt.itemsize)).from_address(p.value)
        return np.frombuffer(buf, dtype=dt)

    def place(self, dev_id=0, dev_kind=DEV_HOST, copy_ctrl=COPY_M):
        check(api().talshTensorPlace(self.h, dev_id, dev_kind, None, copy_ctrl, None), "talshTensorPlace")

    def presence(self):
        n = C.c_int()
        copies = (C.c_int * 16)()
        kinds = (C.c_int * 16)()
        check(api().talshTensorPresence(self.h, C.byref(n), copies, kinds, DEV_NULL, -1), "talshTensorPresence")
        return list(copies[:n.value])

    def norm1_host(self) -> float:
        return api().talshTensorImageNorm1_cpu(self.h)

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            api().talshTensorDestroy(self.h)
            self.h = C.c_void_p()


def contract(pattern, d: Tensor, l: Tensor, r: Tensor, alpha=1.0, dev_id=0, dev_kind=DEV_NVIDIA_GPU,
             copy_ctrl=COPY_MTT, accumulative=True, task: Task | None = None) -> int:
    a = complex(alpha)
    return api().talshTensorContract(pattern.encode(), d.h, l.h, r.h, a.real, a.imag, dev_id, dev_kind, copy_ctrl,
                                     int(accumulative), task.h if task else None)


def contract_xl(pattern, d: Tensor, l: Tensor, r: Tensor, alpha=1.0, dev_id=0, dev_kind=DEV_NVIDIA_GPU,
                accumulative=True) -> int:
    """talshTensorContractXL: a blocking contraction whose arguments may exceed
    the GPU's memory (host-resident D, L, R are decomposed into D slabs)."""
    a = complex(alpha)
    return api().talshTensorContractXL(pattern.encode(), d.h, l.h, r.h, a.real, a.imag, dev_id, dev_kind,
                                       int(accumulative))


def xl_last_split():
    """(D dimension, slabs) of this thread's last contract_xl; (-1, 0) if undecomposed."""
    dd, ns = C.c_int(), C.c_int()
    api().tb_xl_last_split(C.byref(dd), C.byref(ns))
    return dd.value, ns.value


def copy(pattern, d: Tensor, l: Tensor, dev_id=0, dev_kind=DEV_NVIDIA_GPU, copy_ctrl=COPY_MT, task=None) -> int:
    return api().talshTensorCopy(pattern.encode(), d.h, l.h, dev_id, dev_kind, copy_ctrl, task.h if task else None)


def add(pattern, d: Tensor, l: Tensor, scale=1.0, dev_id=0, dev_kind=DEV_NVIDIA_GPU, copy_ctrl=COPY_MT,
        task=None) -> int:
    s = complex(scale)
    return api().talshTensorAdd(pattern.encode(), d.h, l.h, s.real, s.imag, dev_id, dev_kind, copy_ctrl,
                                task.h if task else None)
