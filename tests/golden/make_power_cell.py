"""Golden sweeps of the vertical power cell (the large-device configuration's device,
devices.power_cell) on a reduced mesh, from the reference core itself.

The unmodified reference core (oracle/_ref/libsemisim_ref.so, built from the reference's
semiconductor_3d.c by oracle/Makefile) sweeps the drain 0..50 V in 5 V steps at
Vg = 10 V on a 40x64x3 mesh of the 10 x 60 x 10 um cell, once at the production
tolerances (the GUI's solver tuple) and once converged tightly (validate.py's inner
tolerances and a 1e-12 V Gummel tolerance).  Stored per sweep: the drain voltages, every
terminal current and its round-off floor, the converged flags and psi at every point.
The reference's thread count is recorded (its threaded reductions move the last digits).

Usage (needs `make -C oracle`):
    python tests/golden/make_power_cell.py
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from semiconductor_devices_simulator_b200 import abi, devices as D   # noqa: E402
from make_golden import TIGHT_ENV, TIGHT_SOLVER                        # noqa: E402

MESH = (40, 64, 3)
VD_MAX, DVD, VG = 50.0, 5.0, 10.0


def build(lib, solver=D.GUI_SOLVER):
    return D.power_cell(lib, n=MESH, vgs=(VG,), vd_max=VD_MAX, dvd=DVD, solver=solver)


def sweep(lib, w, tag):
    s = w.sweeps[0]
    ok0 = D.start_sweep(lib, w, s)
    psi = []
    V, I, F, conv = D.run_sweep(lib, w, s, on_point=lambda q, v: psi.append(D.field(lib, 0, w.shape).ravel()))
    return {f"{tag}_V": V, f"{tag}_I": I, f"{tag}_Iflr": F, f"{tag}_conv": conv, f"{tag}_start_ok": np.array(ok0),
            f"{tag}_psi": np.array(psi)}


def main():
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_ref.so")
    lib = abi.bind(ctypes.CDLL(path))
    threads = os.cpu_count() or 1
    lib.api3_set_threads(threads)
    out = {"mesh": np.array(MESH), "threads": np.array(threads), "vg": np.array(VG)}
    out.update(sweep(lib, build(lib), "sw"))
    os.environ.update(TIGHT_ENV)                   # read by api3_init
    try:
        out.update(sweep(lib, build(lib, TIGHT_SOLVER), "swt"))
    finally:
        for k in TIGHT_ENV:
            del os.environ[k]
    dst = os.path.join(HERE, "power_cell_small.npz")
    np.savez_compressed(dst, **out)
    print(f"power_cell_small: {MESH} -> {os.path.relpath(dst, ROOT)} ({os.path.getsize(dst) // 1024} KiB)")


if __name__ == "__main__":
    main()
