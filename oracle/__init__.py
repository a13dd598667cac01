"""The FP64 CPU oracle: test infrastructure, never part of the product path.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this package.  It restates ryoung48/web-exoplasim's GCM set-up
(setup_f64.py, model_f64.py) and timestep (oracle.cpp) in double precision,
and drives the timestep in the reference's run order
(runner/webgpu/gcm.worker.ts:53-176: start-up steps at the start step's date,
then the main loop).

Oracle(model, precision=32) steps the same loops in sequential f32
(liboracle32.so): the comparator of the reference's "<= 2x sequential f32"
and V3 gates (scripts/exoplasim-webgpu/verify-kernels.mjs:273,
verify-dynamics.mjs:179-181).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from . import model_f64, setup_f64

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liboracle.so")
LIB32_PATH = os.path.join(HERE, "build", "liboracle32.so")
_libs = {}


def build():
    """Compile liboracle.so (f64) and liboracle32.so (sequential f32) from
    oracle.cpp (g++, C++17)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(precision=64):
    if precision not in _libs:
        path = {64: LIB_PATH, 32: LIB32_PATH}[precision]
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.ora_create.restype = ctypes.c_void_p
        L.ora_create.argtypes = [ctypes.c_int, ctypes.c_int]
        L.ora_destroy.argtypes = [ctypes.c_void_p]
        L.ora_set_const.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double]
        L.ora_size.restype = ctypes.c_long
        L.ora_size.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p]
        dp = ctypes.POINTER(ctypes.c_double)
        L.ora_set.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, dp, ctypes.c_long]
        L.ora_get.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, dp, ctypes.c_long]
        L.ora_run.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.ora_last_error.restype = ctypes.c_char_p
        _libs[precision] = L
    return _libs[precision]


class Oracle:
    """One planet stepped in FP64 (or sequential f32) on the CPU."""

    def __init__(self, model: dict, precision: int = 64):
        self.model = model
        self.precision = precision
        self.L = L = lib(precision)
        self.h = L.ora_create(model["truncation"], model["levels"])
        if not self.h:
            raise RuntimeError(L.ora_last_error().decode())
        for name, values in model["tables"].items():
            self.set_table(name, values)
        for name, values in model["state"].items():
            if self.size(name) >= 0:
                self.set(name, values)
        self.step = model["start_step"]
        self.carbon_step = 0
        self.started = False
        sigma = model["tables"]["sigma"]
        jet = 0
        for l in range(1, len(sigma)):
            if abs(sigma[l] - 0.25) < abs(sigma[jet] - 0.25):
                jet = l
        self._extra = dict(JET=float(jet), SIGMA_LOW=float(sigma[-1]))
        self.set_phase(model["nkits"])

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ora_destroy(self.h)
            self.h = None

    # -- raw access --------------------------------------------------------
    def size(self, name, kind=0):
        return self.L.ora_size(self.h, kind, name.encode())

    def set(self, name, values, kind=0):
        arr = np.ascontiguousarray(np.asarray(values, dtype=np.float64).reshape(-1))
        if self.L.ora_set(self.h, kind, name.encode(), arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                         arr.size) != 0:
            raise RuntimeError(self.L.ora_last_error().decode())

    def set_table(self, name, values):
        self.set(name, values, kind=1)

    def get(self, name, kind=0):
        n = self.size(name, kind)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n)
        if self.L.ora_get(self.h, kind, name.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n) != 0:
            raise RuntimeError(self.L.ora_last_error().decode())
        return out

    def set_const(self, name, value):
        if self.L.ora_set_const(self.h, name.encode(), float(value)) != 0:
            raise RuntimeError(self.L.ora_last_error().decode())

    def run(self, stage):
        if self.L.ora_run(self.h, stage.encode()) != 0:
            raise RuntimeError(self.L.ora_last_error().decode())

    # -- schedule ----------------------------------------------------------
    def set_phase(self, kits):
        for k, v in self.model["phases"][kits].items():
            self.set_const(k, v)
        for k, v in self._extra.items():
            self.set_const(k, v)
        self.set_table("bm1", self.model["bm1"][kits])

    def write_step_values(self, step, publish=False):
        values, cstep = setup_f64.step_values(step, self.carbon_step, self.model["calendar"])
        for name, arr in values.items():
            if name == "snapshot_step":
                arr = arr.copy()
                arr[2] = 1.0 if publish else 0.0
            self.set(name, arr)
        return cstep

    def startup(self):
        """master's nkits start-up steps, all at the start step's date."""
        for kits in range(self.model["nkits"], 0, -1):
            self.set_phase(kits)
            self.carbon_step = self.write_step_values(self.step)
            self.run("step")
        self.set_phase(0)
        self.started = True

    def advance(self, steps=1, publish_every=0):
        if not self.started:
            self.startup()
        for _ in range(steps):
            publish = publish_every > 0 and self.step % publish_every == 0
            self.carbon_step = self.write_step_values(self.step, publish)
            self.run("step")
            self.step += 1


def model_for(planet):
    """The FP64 model for a planets.Planet."""
    return model_f64.build(planet.config, planet.boundary, planet.t_grid, planet.q_grid)
