"""ctypes binding of the C ABI in include/ds2d.h (library ds2d_b200/libds2d_b200.so).

The product path has no fallback: if the CUDA library is missing or cannot be loaded, every
entry point raises instead of computing anything on the host.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libds2d_b200.so")

DS2D_OK = 0
DS2D_E_ARG = -1
DS2D_E_CUDA = -2
DS2D_E_NOMEM = -3
DS2D_E_STATE = -4
DS2D_E_NUMERIC = -5

BOUNDARY = {"pml": 0, "random": 1}
STRIPS = {"f32": 0, "f16": 1, "bf16": 2}

# Every symbol include/ds2d.h declares (checked by the CPU test suite).
EXPORTS = [
    "ds2d_create", "ds2d_destroy", "ds2d_last_error", "ds2d_set_stream", "ds2d_set_models",
    "ds2d_set_wavelet", "ds2d_set_image", "ds2d_forward", "ds2d_elsrtm", "ds2d_rtm",
    "ds2d_rtm_device", "ds2d_read_images", "ds2d_last_cell_updates", "ds2d_last_launches",
    "ds2d_profile", "ds2d_profile_report", "ds2d_set_option", "ds2d_ac_born",
    "ds2d_ac_born_adj", "ds2d_lsrtm", "ds2d_dot_f64", "ds2d_dot_f64_noalloc",
    "ds2d_ac_normal", "ds2d_lsrtm_pcg", "ds2d_unet_create", "ds2d_unet_destroy", "ds2d_unet_last_error", "ds2d_unet_set_stream",
    "ds2d_unet_num_params", "ds2d_unet_set_params", "ds2d_unet_get_params", "ds2d_unet_forward",
    "ds2d_unet_loss_grad", "ds2d_unet_adam_step", "ds2d_unet_set_option",
]


class Grid(ctypes.Structure):
    _fields_ = [("allnx", ctypes.c_int), ("allnz", ctypes.c_int), ("nx", ctypes.c_int),
                ("pml", ctypes.c_int), ("nt", ctypes.c_int), ("dx", ctypes.c_float),
                ("dz", ctypes.c_float), ("dt", ctypes.c_float)]


class Opts(ctypes.Structure):
    _fields_ = [("boundary", ctypes.c_int), ("strip_precision", ctypes.c_int),
                ("max_shots", ctypes.c_int), ("max_ntr", ctypes.c_int),
                ("seed", ctypes.c_ulonglong), ("device", ctypes.c_int)]


class Shot(ctypes.Structure):
    _fields_ = [("win_left", ctypes.c_int), ("isx", ctypes.c_int), ("isz", ctypes.c_int),
                ("igz", ctypes.c_int), ("ntr", ctypes.c_int),
                ("igx", ctypes.POINTER(ctypes.c_int)), ("nx", ctypes.c_int)]


class DS2DError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"ds2d error {code}: {msg}")
        self.code = code


_lib = None


def load():
    """Loads the CUDA library; raises if it is absent (there is no host fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python ds2d_b200/build.py` "
                          "(the DS2D path has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    fp = ctypes.POINTER(ctypes.c_float)
    dp = ctypes.POINTER(ctypes.c_double)
    sig = {
        "ds2d_create": ([ctypes.POINTER(Grid), ctypes.POINTER(Opts), ctypes.POINTER(P)], ctypes.c_int),
        "ds2d_destroy": ([P], ctypes.c_int),
        "ds2d_last_error": ([P], ctypes.c_char_p),
        "ds2d_set_stream": ([P, P], ctypes.c_int),
        "ds2d_set_models": ([P, fp, fp, fp], ctypes.c_int),
        "ds2d_set_wavelet": ([P, fp], ctypes.c_int),
        "ds2d_set_image": ([P, fp, fp], ctypes.c_int),
        "ds2d_forward": ([P, ctypes.POINTER(Shot), ctypes.c_int, fp, fp], ctypes.c_int),
        "ds2d_elsrtm": ([P, ctypes.POINTER(Shot), ctypes.c_int, fp, fp, ctypes.c_int, dp, fp, fp,
                         fp, fp], ctypes.c_int),
        "ds2d_rtm": ([P, ctypes.POINTER(Shot), ctypes.c_int, fp, fp], ctypes.c_int),
        "ds2d_rtm_device": ([P, ctypes.POINTER(Shot), ctypes.c_int, P, P], ctypes.c_int),
        "ds2d_read_images": ([P, ctypes.POINTER(fp), ctypes.c_int], ctypes.c_int),
        "ds2d_read_images_device": ([P, ctypes.POINTER(P), ctypes.c_int], ctypes.c_int),
        "ds2d_last_cell_updates": ([P], ctypes.c_double),
        "ds2d_last_launches": ([P], ctypes.c_longlong),
        "ds2d_profile": ([P, ctypes.c_int], ctypes.c_int),
        "ds2d_set_option": ([P, ctypes.c_char_p, ctypes.c_longlong], ctypes.c_int),
        "ds2d_dot_f64": ([P, P, P, ctypes.c_longlong, dp], ctypes.c_int),
        "ds2d_dot_f64_noalloc": ([P, P, ctypes.c_longlong, P, dp], ctypes.c_int),
        "ds2d_ac_normal": ([P, ctypes.POINTER(Shot), ctypes.c_int, P, P], ctypes.c_int),
        "ds2d_lsrtm_pcg": ([P, P, ctypes.POINTER(Shot), ctypes.c_int, P, P, ctypes.c_int,
                            ctypes.c_double, P, dp, dp, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "ds2d_unet_create": ([ctypes.c_int] * 5 + [ctypes.POINTER(P)], ctypes.c_int),
        "ds2d_unet_destroy": ([P], ctypes.c_int),
        "ds2d_unet_last_error": ([P], ctypes.c_char_p),
        "ds2d_unet_set_stream": ([P, P], ctypes.c_int),
        "ds2d_unet_num_params": ([P], ctypes.c_longlong),
        "ds2d_unet_set_params": ([P, fp, ctypes.c_longlong], ctypes.c_int),
        "ds2d_unet_get_params": ([P, fp, ctypes.c_longlong], ctypes.c_int),
        "ds2d_unet_forward": ([P, P, P] + [ctypes.c_int] * 3, ctypes.c_int),
        "ds2d_unet_loss_grad": ([P, P, P] + [ctypes.c_int] * 3 + [dp, fp], ctypes.c_int),
        "ds2d_unet_adam_step": ([P] + [ctypes.c_float] * 4, ctypes.c_int),
        "ds2d_unet_set_option": ([P, ctypes.c_char_p, ctypes.c_longlong], ctypes.c_int),
        "ds2d_ac_born": ([P, ctypes.POINTER(Shot), ctypes.c_int, fp, fp, fp], ctypes.c_int),
        "ds2d_ac_born_adj": ([P, ctypes.POINTER(Shot), ctypes.c_int, fp, fp, fp], ctypes.c_int),
        "ds2d_lsrtm": ([P, ctypes.POINTER(Shot), ctypes.c_int, fp, fp, ctypes.c_int,
                        ctypes.c_double, fp, dp, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        "ds2d_profile_report": ([P, ctypes.c_char_p, ctypes.c_int], ctypes.c_int),
        "ds2d_bandpass_filter": ([ctypes.c_int] * 6 + [fp, fp], ctypes.c_int),
        "ds2d_bandpass_filter_device": ([ctypes.c_int] * 6 + [P, P, P], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib
