"""ctypes binding of libcpm_cuda.so (the C ABI declared in include/cpm.h).

The library is loaded from this package directory only. There is no CPU fallback: when the
library is missing the first call raises, and every non-zero status code raises CpmError with
the library's error text.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libcpm_cuda.so"
HEADER = HERE.parent / "include" / "cpm.h"

CPM_OK = 0
ERROR_NAMES = {
    -1: "CPM_E_INVALID", -2: "CPM_E_MESH_MISMATCH", -3: "CPM_E_CAPACITY", -4: "CPM_E_UNSUPPORTED",
    -5: "CPM_E_CUDA", -6: "CPM_E_NONFINITE", -7: "CPM_E_NOMEM", -8: "CPM_E_DEVICE", -9: "CPM_E_NO_DEVICE",
}
SIM_FIXED_POINT = 0x1
SIM_DECONVOLVE = 0x2
SIM_TIMING = 0x4
SIM_NO_GRAPH = 0x8
SIM_QUADRUPOLE = 0x10
SIM_NO_AUTOTUNE = 0x20


class CpmError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {message}")
        self.code = code
        self.message = message


class Cosmology(C.Structure):
    """cosmology.rs:9-16 `Cosmology`."""
    _fields_ = [("omega_r", C.c_float), ("omega_m", C.c_float), ("omega_l", C.c_float), ("h0", C.c_float)]

    @staticmethod
    def lcdm_default() -> "Cosmology":
        """cosmology.rs:21-29, evaluated in f32."""
        omega_r = np.float32(9.14e-5)
        omega_l = np.float32(np.float32(np.float32(1.0) - np.float32(0.315)) - omega_r)
        return Cosmology(float(omega_r), 0.315, float(omega_l), 67.4)

    def __repr__(self):
        return f"Cosmology(omega_r={self.omega_r}, omega_m={self.omega_m}, omega_l={self.omega_l}, h0={self.h0})"


class ForceSplitC(C.Structure):
    _fields_ = [("r_split", C.c_float), ("r_cut", C.c_float), ("softening", C.c_float), ("theta", C.c_float)]


class SimParams(C.Structure):
    _fields_ = [("cosmo", Cosmology), ("box_size", C.c_float), ("mesh_n", C.c_int), ("n_particles", C.c_size_t),
                ("use_tree", C.c_int), ("split", ForceSplitC), ("flags", C.c_uint32)]


def exported_symbols() -> list[str]:
    """Every function name declared in include/cpm.h."""
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(cpm_[a-z0-9_]+)\s*\(", text)
    seen, out = set(), []
    for n in names:
        if n not in seen:
            seen.add(n)
            out.append(n)
    return out


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is not built: run `python {HERE / 'build.py'}` (needs nvcc)")
    L = C.CDLL(str(LIB_PATH))
    vp, sz, fl, i, u32, u64 = C.c_void_p, C.c_size_t, C.c_float, C.c_int, C.c_uint32, C.c_uint64
    sig = {
        "cpm_version": (C.c_char_p, []),
        "cpm_last_error": (C.c_char_p, [vp]),
        "cpm_ctx_create": (i, [i, fl, sz, u32, C.POINTER(vp)]),
        "cpm_ctx_destroy": (i, [vp]),
        "cpm_mesh_deposit": (i, [vp, vp, sz, fl, vp]),
        "cpm_density_contrast": (i, [vp, vp, sz, vp]),
        "cpm_mesh_interpolate": (i, [vp, vp, vp, sz, vp]),
        "cpm_mesh_interpolate3": (i, [vp, vp, vp, vp, vp, sz, vp]),
        "cpm_fft3": (i, [vp, vp, i, i]),
        "cpm_wavenumber": (fl, [sz, sz, fl]),
        "cpm_poisson_accel": (i, [vp, vp, i, C.POINTER(Cosmology), fl, fl, vp, vp, vp]),
        "cpm_force_split_with": (ForceSplitC, [fl, sz, sz, fl, fl]),
        "cpm_short_range_factor": (fl, [fl, fl]),
        "cpm_tree_accel": (i, [vp, vp, sz, fl, C.POINTER(ForceSplitC), fl, vp]),
        "cpm_octant_keys": (i, [vp, vp, sz, fl, i, vp, vp]),
        "cpm_tree_stats": (i, [vp, C.POINTER(u64), C.POINTER(u64), C.POINTER(u64), C.POINTER(u32)]),
        "cpm_ics_zeldovich": (i, [i, fl, C.POINTER(Cosmology), fl, fl, fl, u64, vp, vp]),
        "cpm_power_spectrum": (i, [vp, vp, sz, i, vp, vp, vp]),
        "cpm_fft_supported": (i, [i]),
        "cpm_sim_power_spectrum": (i, [vp, i, vp, vp, vp]),
        "cpm_sim_create": (i, [C.POINTER(SimParams), vp, vp, fl, C.POINTER(vp)]),
        "cpm_sim_create_zeldovich": (i, [C.POINTER(SimParams), i, fl, fl, fl, u64, C.POINTER(vp)]),
        "cpm_sim_step_to": (i, [vp, fl]),
        "cpm_sim_step_host": (i, [vp, fl, vp, vp]),
        "cpm_sim_get_state": (i, [vp, vp, vp, vp, vp, C.POINTER(fl)]),
        "cpm_sim_set_state": (i, [vp, vp, vp]),
        "cpm_sim_phase_times": (i, [vp, vp, C.POINTER(u64), i]),
        "cpm_sim_counters": (i, [vp, C.POINTER(u64), C.POINTER(u64), C.POINTER(u64), C.POINTER(u32)]),
        "cpm_sim_walk_candidates": (i, [vp, C.POINTER(u64)]),
        "cpm_walk_kernel_fit_error": (i, [fl, fl, i, C.POINTER(C.c_double)]),
        "cpm_hilbert_fsm_check": (i, [i, u64, u64, C.POINTER(u64), C.POINTER(i)]),
        "cpm_sim_stream": (vp, [vp]),
        "cpm_sim_graphs": (i, [vp]),
        "cpm_sim_snapshot": (i, [vp, vp, vp, vp, vp, C.POINTER(i), C.POINTER(fl)]),
        "cpm_density_grid": (i, [vp, vp, i, vp, C.POINTER(i)]),
        "cpm_sim_destroy": (i, [vp]),
        "cpm_sim_set_learned": (i, [vp, vp, fl, fl]),
        "cpm_sim_learned_walked": (i, [vp, C.POINTER(u64)]),
        "cpm_sim_short_range": (i, [vp, vp]),
        "cpm_sim_save": (i, [vp, C.c_char_p]),
        "cpm_sim_autotune_report": (i, [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i), vp]),
        "cpm_sim_set_tuning": (i, [vp, i, i, i]),
        "cpm_step_factors": (i, [C.POINTER(Cosmology), C.c_double, C.c_double, i, C.POINTER(C.c_double),
                                 C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "cpm_sim_load": (i, [C.c_char_p, u32, C.POINTER(vp)]),
        "cpm_sim_tree_depth": (i, [vp, C.POINTER(u32), C.POINTER(u64)]),
        "cpm_ensemble_create": (i, [C.POINTER(Cosmology), fl, fl, fl, fl, i, vp, u32, C.POINTER(vp)]),
        "cpm_ensemble_step_to": (i, [vp, fl]),
        "cpm_ensemble_get_state": (i, [vp, i, i, vp, vp, vp]),
        "cpm_ensemble_power_spectrum": (i, [vp, i, i, i, vp, vp, vp]),
        "cpm_ensemble_graphs": (i, [vp]),
        "cpm_ensemble_stream": (vp, [vp]),
        "cpm_ensemble_last_error": (C.c_char_p, [vp]),
        "cpm_ensemble_destroy": (i, [vp]),
        "cpm_net_weight_count": (i, []),
        "cpm_net_create": (i, [i, C.POINTER(vp)]),
        "cpm_net_destroy": (i, [vp]),
        "cpm_net_last_error": (C.c_char_p, [vp]),
        "cpm_net_set_weights": (i, [vp, vp]),
        "cpm_net_get_weights": (i, [vp, vp]),
        "cpm_net_get_grads": (i, [vp, vp]),
        "cpm_net_forward": (i, [vp, vp, fl, fl, vp, vp]),
        "cpm_net_backward": (i, [vp, vp, fl, vp]),
        "cpm_net_activations": (i, [vp, i, vp, vp]),
        "cpm_net_train_step": (i, [vp, vp, fl, vp, vp, vp, sz, fl, fl, fl, C.POINTER(C.c_double), vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error(handle=None) -> str:
    msg = lib().cpm_last_error(handle)
    return msg.decode() if msg else ""


def check(rc: int, handle=None, sim: bool = False) -> None:
    if rc != CPM_OK:
        # cpm_last_error takes a context; simulations keep their text in the thread-local slot too.
        raise CpmError(rc, last_error(None if sim else handle))


def ptr(a: np.ndarray | None):
    return None if a is None else C.c_void_p(a.ctypes.data)


def f32c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)
