"""B200-native solve path of SemiSim 3D (kotmariusz/Semiconductor_devices_simulator).

The product is the shared library lib/libsemisim_b200.so: the reference core's C ABI
(the 89 ``api3_*`` entry points of semiconductor_3d.c) over CUDA kernels built for
sm_100a.  main.py and validate.py of the reference load it unchanged through
``SEMISIM_SO=<path to libsemisim_b200.so>``.

``load()`` returns the library bound with the ABI's ctypes signatures (abi.API3) and the
kernel-level test hooks; it raises if the library has not been built
(``python -m semiconductor_devices_simulator_b200.build``).
"""
import ctypes
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libsemisim_b200.so")

_I, _D, _LL = ctypes.c_int, ctypes.c_double, ctypes.c_longlong
_DP, _IP = ctypes.POINTER(_D), ctypes.POINTER(_I)
_VP = ctypes.c_void_p
HOOKS = {
    "b200x_prepare": (_I, []),
    "b200x_masks": (_I, [_IP, _IP, _IP, _DP]),
    "b200x_ion": (_I, [_DP]),
    "b200x_te_update": (_I, []),
    "b200x_set_qc": (_I, [_DP, _DP]),
    "b200x_tun_update": (_I, []),
    "b200x_tun": (_I, [_IP, _DP, _DP, ctypes.POINTER(_LL), ctypes.POINTER(_LL)]),
    "b200x_gmg_plan": (_I, [_I, _IP, _IP, _DP, _DP, _I, _IP, _IP, _IP, _IP, _IP]),
    "b200x_gmg_vals": (_I, [_I, _I, _DP, _DP]),
    "b200x_te": (_I, [_IP, _DP, _DP, _DP, _DP, _DP, _DP, _DP]),
    "b200x_set": (_I, [_I, _DP]),
    "b200x_get": (_I, [_I, _DP]),
    "b200x_vlo": (_D, []),
    "b200x_vhi": (_D, []),
    "b200x_apply_bc": (None, []),
    "b200x_rebuild_np": (None, []),
    "b200x_init_state": (None, []),
    "b200x_upd_mob": (None, []),
    "b200x_clamp_qf": (None, []),
    "b200x_poisson": (_D, [_DP, _DP, _DP, _DP]),
    "b200x_cont_assemble": (None, [_I, _DP, _DP, _DP, _DP]),
    "b200x_cont_update": (_D, [_I, _DP, _D, _D, _DP]),
    "b200x_currents": (None, [_DP, _DP, _DP]),
    "b200x_mg_setup": (_I, [_I]),
    "b200x_mg_level": (_I, [_I, _IP, _DP, _DP]),
    "b200x_bicgstab": (_I, [_I, _D, _D, _I, _DP, _DP, _DP, _DP]),
    "b200x_pcg": (_I, [_I, _D, _DP]),
    "b200x_persist_probe": (_I, [_I, _D, _IP]),
    "b200x_persist_trace": (_I, [_I, ctypes.POINTER(ctypes.c_ulonglong), _IP]),
    "b200x_persist_tblocks": (_I, [_I]),
    "b200x_float_fix": (_I, [_I, _DP]),
    "b200x_device_bytes": (_LL, []),
    "b200x_stream_timer": (_D, [_I]),
    "b200x_set_device": (_I, [_I]),
    "b200x_bench": (_D, [_I, _I]),
    "api3b_stencil_residual_noalloc": (_I, [_DP, _DP, _DP, _I, _I, _I, _DP, _DP]),
    "b200x_prof": (_I, [_I]),
    "b200x_prof_read": (_I, [_I, _DP, _DP, _DP]),
    "b200x_prof_name": (ctypes.c_char_p, [_I]),
    "b200x_prof_detail": (_I, [_I, _IP, _DP, _DP, _DP]),
    "b200x_launches": (ctypes.c_ulonglong, []),
    "b200x_ir_stats": (None, [ctypes.POINTER(_LL), ctypes.POINTER(_LL)]),
    "b200x_seed_run": (_I, [_D, _DP]),
    "b200x_vtref": (_D, []),
    # training kernels of the learned predictor (device pointers as integers)
    "b200m_seed_features": (_I, [_VP] * 6 + [_D, _DP, _VP, _VP]),
    "b200m_mlp_pack": (_I, [_VP, _VP, _VP, _VP]),
    "b200m_mlp_forward": (_I, [_VP, _I, _VP, _VP, _VP, _VP, _VP, _VP]),
    "b200m_mlp_backward": (_I, [_VP, _I, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "b200m_mlp_adam": (_I, [_VP, _VP, _VP, _VP, ctypes.c_float, _I, _VP, _VP, _VP]),
    "b200m_mlp_sizes": (_I, [_IP, _IP, _IP]),
}
# state arrays reachable through b200x_set / b200x_get
ST_PHI, ST_PHIN, ST_PHIP, ST_N, ST_P, ST_MU0N, ST_MU0P, ST_SOL, ST_RHS, ST_SC, ST_DSC = range(11)
ST_FMU = 16
ST_H1, ST_E2 = 22, 25                 # sweep history: solution now (h1) and one step back (e2)

_lib = None


def load(path=None):
    """The solver library with every ABI signature declared (loaded once)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("SEMISIM_B200_SO") or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"solver library not built: {p} (python -m semiconductor_devices_simulator_b200.build)")
    lib = abi.bind(ctypes.CDLL(p), HOOKS)
    if path is None:
        _lib = lib
    return lib
