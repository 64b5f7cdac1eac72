"""ctypes binding of libcusmic_b200.so (the C ABI of include/cusmic.h and
include/cusmic_b200.h).

The library is built in-tree by ``cusmic_b200.build``; there is no fallback:
importing the Python API without it raises immediately.
"""

import ctypes
import json
from pathlib import Path

LIB_PATH = Path(__file__).with_name("libcusmic_b200.so")

CUSMIC_OK, CUSMIC_INVALID, CUSMIC_CUDA_ERROR, CUSMIC_NO_MEMORY = range(4)
BORDERS = {"reflect": 0, "constant": 1, "nearest": 2, "mirror": 3, "wrap": 4}
PLAN_GRAPH, PLAN_KEEP = 1, 2
FAULT_PREPARE_WAIT, FAULT_DETECT_WAIT, FAULT_NO_MEMORY = 1, 2, 3

# Every symbol declared in include/cusmic.h and include/cusmic_b200.h.
EXPORTS = (
    "cusmic_version", "cusmic_cuda_version", "cusmic_default_options", "remove_cosmics",
    "remove_cosmics_device", "remove_cosmics_batch_device", "cusmic_ragged_batch_device",
    "cusmic_plan_create", "cusmic_plan_bind", "cusmic_plan_execute", "cusmic_plan_wait",
    "cusmic_plan_passes", "cusmic_plan_profile", "cusmic_plan_backward", "cusmic_plan_destroy",
    "remove_cosmics_device_noalloc", "cusmic_set_tuning", "cusmic_get_tuning",
    "cusmic_inject_fault", "cusmic_batch_host",
)
TUNING_PATH = Path(__file__).with_name("tuning.json")
KERNEL_KINDS = ("init", "prepare", "fill", "sigraw", "cand", "seed", "grow", "control",
                "replace", "restore", "copy", "low", "classify", "floor", "reclass", "dirty",
                "sigmap")


class Image(ctypes.Structure):
    """struct cusmic_image."""
    _fields_ = [("data", ctypes.c_void_p), ("error", ctypes.c_void_p), ("gain", ctypes.c_void_p),
                ("readnoise", ctypes.c_void_p), ("background", ctypes.c_void_p),
                ("mask", ctypes.c_void_p), ("width", ctypes.c_size_t), ("height", ctypes.c_size_t)]


class Options(ctypes.Structure):
    """struct cusmic_options."""
    _fields_ = [("contrast", ctypes.c_double), ("cr_threshold", ctypes.c_double),
                ("neighbor_threshold", ctypes.c_double), ("gain", ctypes.c_double),
                ("readnoise", ctypes.c_double), ("background", ctypes.c_double),
                ("maxiter", ctypes.c_int), ("border", ctypes.c_int)]


class FrameScalars(ctypes.Structure):
    """struct cusmic_frame_scalars."""
    _fields_ = [("gain", ctypes.c_double), ("readnoise", ctypes.c_double),
                ("background", ctypes.c_double)]


class Tuning(ctypes.Structure):
    """struct cusmic_tuning."""
    _fields_ = [("max_pixels", ctypes.c_size_t), ("dense_rows", ctypes.c_int),
                ("dense_blocks_per_sm", ctypes.c_int), ("sparse_blocks_per_sm", ctypes.c_int),
                ("row_blocks_per_sm", ctypes.c_int)]

    FIELDS = ("max_pixels", "dense_rows", "dense_blocks_per_sm", "sparse_blocks_per_sm",
              "row_blocks_per_sm")

    def as_dict(self):
        return {k: int(getattr(self, k)) for k in self.FIELDS}


class CusmicError(RuntimeError):
    pass


_lib = None


def lib():
    """Load the native library (once); raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cusmic_b200.build`")
    L = ctypes.CDLL(str(LIB_PATH))
    vp, sz, cp, ip = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_int
    img, opt, sca = ctypes.POINTER(Image), ctypes.POINTER(Options), ctypes.POINTER(FrameScalars)
    L.cusmic_version.restype = ctypes.c_char_p
    L.cusmic_version.argtypes = []
    L.cusmic_cuda_version.restype = ip
    L.cusmic_cuda_version.argtypes = []
    L.cusmic_default_options.restype = None
    L.cusmic_default_options.argtypes = [opt]
    L.remove_cosmics.restype = ip
    L.remove_cosmics.argtypes = [img, opt, vp, vp, cp, sz]
    L.remove_cosmics_device.restype = ip
    L.remove_cosmics_device.argtypes = [img, opt, vp, vp, vp, cp, sz]
    L.remove_cosmics_batch_device.restype = ip
    L.remove_cosmics_batch_device.argtypes = [img, sz, opt, vp, vp, vp, cp, sz]
    L.cusmic_ragged_batch_device.restype = ip
    L.cusmic_ragged_batch_device.argtypes = [img, sz, opt, sca, vp, vp, vp, cp, sz]
    L.cusmic_plan_create.restype = ip
    L.cusmic_plan_create.argtypes = [ctypes.POINTER(vp), img, sz, opt, sca, vp, vp, ip, cp, sz]
    L.cusmic_plan_bind.restype = ip
    L.cusmic_plan_bind.argtypes = [vp, img, vp, vp, cp, sz]
    L.cusmic_plan_execute.restype = ip
    L.cusmic_plan_execute.argtypes = [vp, vp, cp, sz]
    L.cusmic_plan_wait.restype = ip
    L.cusmic_plan_wait.argtypes = [vp, cp, sz]
    L.cusmic_plan_passes.restype = ip
    L.cusmic_plan_passes.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.cusmic_plan_profile.restype = ip
    L.cusmic_plan_profile.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_int), ip, cp, sz]
    L.cusmic_plan_backward.restype = ip
    L.cusmic_plan_backward.argtypes = [vp, vp, vp, vp, vp, cp, sz]
    L.cusmic_plan_destroy.restype = None
    L.cusmic_plan_destroy.argtypes = [vp]
    L.remove_cosmics_device_noalloc.restype = ip
    L.remove_cosmics_device_noalloc.argtypes = [img, opt, vp, vp, vp, cp, sz]
    L.cusmic_set_tuning.restype = ip
    L.cusmic_set_tuning.argtypes = [ctypes.POINTER(Tuning), sz, cp, sz]
    L.cusmic_get_tuning.restype = ip
    L.cusmic_get_tuning.argtypes = [sz, ctypes.POINTER(Tuning)]
    L.cusmic_batch_host.restype = ip
    L.cusmic_batch_host.argtypes = [img, sz, opt, sca, vp, vp, cp, sz]
    L.cusmic_inject_fault.restype = ip
    L.cusmic_inject_fault.argtypes = [ip, ctypes.c_longlong]
    _lib = L
    if TUNING_PATH.exists():
        set_tuning(json.loads(TUNING_PATH.read_text())["table"])
    return L


def set_tuning(entries):
    """Install a tuning table: a list of dicts with Tuning's fields (max_pixels
    may be null for "no limit"); an empty list restores the built-in defaults."""
    arr = (Tuning * max(1, len(entries)))()
    for i, e in enumerate(entries):
        mp = e.get("max_pixels")
        arr[i] = Tuning(2 ** 64 - 1 if mp is None else int(mp), int(e["dense_rows"]),
                        int(e["dense_blocks_per_sm"]), int(e["sparse_blocks_per_sm"]),
                        int(e["row_blocks_per_sm"]))
    msg = ctypes.create_string_buffer(256)
    raise_for(lib().cusmic_set_tuning(arr, len(entries), msg, 256), msg)


def get_tuning(total_pixels):
    t = Tuning()
    raise_for(lib().cusmic_get_tuning(int(total_pixels), ctypes.byref(t)), "invalid tuning query")
    return t.as_dict()


def default_options():
    o = Options()
    lib().cusmic_default_options(ctypes.byref(o))
    return o


def raise_for(status, msg):
    """Map a status code to the exception the reference's Python API raises."""
    if status == CUSMIC_OK:
        return
    text = msg.value.decode(errors="replace") if hasattr(msg, "value") else str(msg)
    if status == CUSMIC_INVALID:
        raise ValueError(text)
    if status == CUSMIC_NO_MEMORY:
        raise MemoryError(text)
    raise CusmicError(text)
