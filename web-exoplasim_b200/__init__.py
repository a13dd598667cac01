"""exogcm: B200-native ExoPlaSim timestep behind the reference's engine interface.

The product is the CUDA library libexogcm.so (csrc/, C ABI in include/exogcm.h).
This package binds it with ctypes and mirrors the reference's host-side engine
interface (src/model/climate/gcm/runner/{types,index}.ts): ``Engine`` is the
configure/step/readback/checkpoint surface of one batch of planet slots, and
``runner.GCM_RUNNER.start`` the GcmRun control handle on top of it.

There is no CPU fallback: loading fails loudly when the library or a CUDA
device is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libexogcm.so")

EXOGCM_OK = 0
ERRORS = {-1: "invalid argument", -2: "out of memory", -3: "unstable", -4: "layout mismatch",
          -5: "device error", -6: "invalid state"}


class ExogcmError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


class Planet(ctypes.Structure):
    """exogcm_planet (include/exogcm.h)."""
    _fields_ = [
        ("truncation", ctypes.c_int), ("levels", ctypes.c_int), ("radius_earth", ctypes.c_double),
        ("gravity", ctypes.c_double), ("flux", ctypes.c_double), ("eccentricity", ctypes.c_double),
        ("obliquity_deg", ctypes.c_double), ("fixed_orbit", ctypes.c_int), ("keplerian", ctypes.c_int),
        ("synchronous", ctypes.c_int), ("substellar_longitude_deg", ctypes.c_double),
        ("ocean_depth_m", ctypes.c_double), ("year_days", ctypes.c_double),
        ("rotation_period_days", ctypes.c_double), ("timestep_minutes", ctypes.c_double),
        ("pressure_bar", ctypes.c_double), ("gas_constant", ctypes.c_double), ("co2_ppm", ctypes.c_double),
        ("ozone", ctypes.c_int), ("wet_soil", ctypes.c_int), ("vegetation", ctypes.c_int),
        ("initial_growth", ctypes.c_double), ("glaciers", ctypes.c_int), ("glacier_min_depth_m", ctypes.c_double),
        ("glacier_initial_height_m", ctypes.c_double), ("filter_gp", ctypes.c_int), ("filter_sp", ctypes.c_int),
        ("filter_kind", ctypes.c_int), ("soil_depth_scale", ctypes.c_double),
        ("star_temperature_k", ctypes.c_double), ("storm_diagnostics", ctypes.c_int),
        ("storm_ckcd", ctypes.c_double), ("storm_vithresh", ctypes.c_double),
    ]


_DP = ctypes.POINTER(ctypes.c_double)


class Boundary(ctypes.Structure):
    """exogcm_boundary (include/exogcm.h)."""
    _fields_ = [("land_mask", _DP), ("orography", _DP), ("sst", _DP), ("sst_months", ctypes.c_int),
                ("ice_cover", _DP), ("ice_cover_months", ctypes.c_int), ("t_init", _DP), ("q_init", _DP)]


class ServerOptions(ctypes.Structure):
    """exogcm_server_options (include/exogcm.h)."""
    _fields_ = [("budget_bytes", ctypes.c_double), ("block_slots", ctypes.c_int), ("chunk_steps", ctypes.c_int),
                ("mode", ctypes.c_int)]


_lib = None

# Every entry point include/exogcm.h declares: name -> (restype, argtypes).
_VP = ctypes.c_void_p
_FP = ctypes.POINTER(ctypes.c_float)
SIGNATURES = {
    "exogcm_last_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
    "exogcm_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(_VP)]),
    "exogcm_destroy": (None, [_VP]),
    "exogcm_configure": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(Planet), ctypes.POINTER(Boundary)]),
    "exogcm_setup_preview": (ctypes.c_int, [ctypes.POINTER(Planet), ctypes.POINTER(Boundary), ctypes.c_char_p,
                                            _DP, ctypes.POINTER(ctypes.c_size_t)]),
    "exogcm_setup_preview_device": (ctypes.c_int, [ctypes.POINTER(Planet), ctypes.POINTER(Boundary),
                                                   ctypes.c_char_p, _DP, ctypes.POINTER(ctypes.c_size_t)]),
    "exogcm_setup_on_device": (ctypes.c_int, [_VP, ctypes.c_int]),
    "exogcm_slot_date": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_long, ctypes.POINTER(ctypes.c_int)]),
    "exogcm_release": (ctypes.c_int, [_VP, ctypes.c_int]),
    "exogcm_server_create": (ctypes.c_int, [ctypes.POINTER(ServerOptions), ctypes.POINTER(_VP)]),
    "exogcm_server_destroy": (None, [_VP]),
    "exogcm_server_submit": (ctypes.c_int, [_VP, ctypes.POINTER(Planet), ctypes.POINTER(Boundary), ctypes.c_long,
                                            ctypes.POINTER(ctypes.c_long)]),
    "exogcm_server_pump": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int)]),
    "exogcm_server_poll": (ctypes.c_int, [_VP, ctypes.c_long, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_long)]),
    "exogcm_server_result": (ctypes.c_int, [_VP, ctypes.c_long, ctypes.c_char_p, _FP, ctypes.c_size_t]),
    "exogcm_server_release": (ctypes.c_int, [_VP, ctypes.c_long]),
    "exogcm_step": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int]),
    "exogcm_step_async": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int]),
    "exogcm_poll": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int)]),
    "exogcm_wait": (ctypes.c_int, [_VP]),
    "exogcm_group_step": (ctypes.c_int, [ctypes.POINTER(_VP), ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                         _FP]),
    "exogcm_snapshots_begin": (ctypes.c_int, [_VP, _FP, ctypes.c_size_t]),
    "exogcm_snapshots_wait": (ctypes.c_int, [_VP]),
    "exogcm_budgets": (ctypes.c_int, [_VP, ctypes.c_int, _DP, _DP, ctypes.POINTER(ctypes.c_long), ctypes.c_int]),
    "exogcm_averages_enable": (ctypes.c_int, [_VP, ctypes.c_int]),
    "exogcm_averages_read": (ctypes.c_int, [_VP, ctypes.c_int, _FP, ctypes.c_size_t, ctypes.POINTER(ctypes.c_long),
                                            ctypes.c_int]),
    "exogcm_read_snapshot": (ctypes.c_int, [_VP, ctypes.c_int, _FP, ctypes.c_size_t,
                                            ctypes.POINTER(ctypes.c_long)]),
    "exogcm_set_stop": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_long]),
    "exogcm_slot_info": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_long),
                                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "exogcm_field_size": (ctypes.c_int, [_VP, ctypes.c_char_p, ctypes.POINTER(ctypes.c_size_t)]),
    "exogcm_read_field": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_char_p, _FP, ctypes.c_size_t]),
    "exogcm_write_field": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_char_p, _FP, ctypes.c_size_t]),
    "exogcm_read_table": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_char_p, _FP, ctypes.c_size_t]),
    "exogcm_checkpoint_save": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(_VP),
                                              ctypes.POINTER(ctypes.c_size_t)]),
    "exogcm_checkpoint_load": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]),
    "exogcm_free": (None, [_VP]),
    "exogcm_unstable": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
    "exogcm_run_stage": (ctypes.c_int, [_VP, ctypes.c_char_p]),
    "exogcm_last_step_ms": (ctypes.c_int, [_VP, _FP]),
    "exogcm_device_field": (ctypes.c_int, [_VP, ctypes.c_char_p, ctypes.POINTER(_VP),
                                           ctypes.POINTER(ctypes.c_size_t)]),
    "exogcm_stream": (_VP, [_VP]),
    "exogcm_time_kernel": (ctypes.c_int, [_VP, ctypes.c_char_p, ctypes.c_int, _FP, _DP]),
    "exogcm_tuning": (ctypes.c_int, [_VP, _VP, ctypes.c_int]),
    "exogcm_slot_sums_noalloc": (ctypes.c_int, [_VP, _VP, ctypes.c_int, ctypes.c_int, _VP, _VP]),
    "exogcm_graph_launches": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
}


def load_library(path: str = LIB_PATH):
    """Loads libexogcm.so and binds every declared entry point. Raises when the
    library is missing: there is no fallback implementation."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with web-exoplasim_b200/build.py")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _check(code):
    if code != EXOGCM_OK:
        buf = ctypes.create_string_buffer(1024)
        _lib.exogcm_last_error(buf, 1024)
        raise ExogcmError(code, buf.value.decode())


FILTER_KINDS = {"none": 0, "cesaro": 1, "exp": 2, "lh": 3}


def planet_struct(config: dict) -> Planet:
    """exogcm_planet from a GcmConfig-like dict (planets.BASE_CONFIG keys)."""
    kind = 0
    gp = sp = 0
    for f in config.get("physicsFilter", ()):
        if f == "gp":
            gp = 1
        elif f == "sp":
            sp = 1
        else:
            kind = FILTER_KINDS[f]
    return Planet(
        truncation=int(config["truncation"]), levels=int(config["layers"]), radius_earth=config["radiusEarth"],
        gravity=config["gravityMs2"], flux=config["fluxWm2"], eccentricity=config["eccentricity"],
        obliquity_deg=config["obliquityDeg"], fixed_orbit=int(bool(config["fixedOrbit"])),
        keplerian=int(bool(config["keplerian"])), synchronous=int(bool(config["synchronous"])),
        substellar_longitude_deg=config["substellarLongitudeDeg"], ocean_depth_m=config["oceanDepthM"],
        year_days=float(config["yearDays"]), rotation_period_days=float(config["rotationPeriodDays"]),
        timestep_minutes=float(config["timestepMinutes"]), pressure_bar=float(config["pressureBar"]),
        gas_constant=float(config["gasConstant"]), co2_ppm=float(config["co2Ppm"]),
        ozone=int(bool(config["ozone"])), wet_soil=int(bool(config["wetSoil"])),
        vegetation=int(config["vegetation"]), initial_growth=float(config["initialGrowth"]),
        glaciers=int(bool(config["glaciersEnabled"])), glacier_min_depth_m=float(config["glaciersMinDepthM"]),
        glacier_initial_height_m=float(config["glaciersInitialHeightM"]), filter_gp=gp, filter_sp=sp,
        filter_kind=kind, soil_depth_scale=float(config["soilDepthScale"]),
        star_temperature_k=float(config["starTemperatureK"]),
        storm_diagnostics=int(bool(config.get("stormclim", False))),
        storm_ckcd=float(config.get("stormCkcd", 0.0)), storm_vithresh=float(config.get("stormVithresh", 0.0)))


def boundary_struct(planet, nhor: int, keep: dict) -> Boundary:
    """exogcm_boundary for a planets.Planet; `keep` holds the arrays alive."""
    def ptr(name, a):
        if a is None:
            return None
        arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
        keep[name] = arr
        return arr.ctypes.data_as(_DP)
    bd = planet.boundary
    sst, ice = bd.get(169), bd.get(210)
    return Boundary(land_mask=ptr("mask", bd[172]), orography=ptr("oro", bd.get(129)),
                    sst=ptr("sst", sst), sst_months=0 if sst is None else int(np.size(sst) // nhor),
                    ice_cover=ptr("ice", ice), ice_cover_months=0 if ice is None else int(np.size(ice) // nhor),
                    t_init=ptr("t", planet.t_grid), q_init=ptr("q", planet.q_grid))


def group_step(engines, steps, publish_every: int | None = None) -> float:
    """Steps several engines (any resolutions) as one CUDA graph launch
    (exogcm_group_step): engine i runs steps[i] model steps. Returns the
    launch's device time in ms."""
    lib = load_library()
    n = len(engines)
    handles = (_VP * n)(*[e.h for e in engines])
    counts = (ctypes.c_int * n)(*steps)
    ms = ctypes.c_float()
    _check(lib.exogcm_group_step(handles, n, counts, publish_every or max(max(steps), 1 << 20), ctypes.byref(ms)))
    return ms.value


def setup_preview(planet, name: str, on_device: bool = False) -> np.ndarray:
    """The FP64 set-up array `name` (see exogcm_setup_preview) for a planet,
    computed on the host without a device, or with the heavy loops on the
    current device as exogcm_configure runs them (`on_device`)."""
    lib = load_library()
    call = lib.exogcm_setup_preview_device if on_device else lib.exogcm_setup_preview
    nhor = 2 * {21: 32, 42: 64, 63: 96}[planet.config["truncation"]] ** 2
    keep = {}
    p = planet_struct(planet.config)
    b = boundary_struct(planet, nhor, keep)
    n = ctypes.c_size_t(0)
    _check(call(ctypes.byref(p), ctypes.byref(b), name.encode(), None, ctypes.byref(n)))
    out = np.zeros(n.value)
    _check(call(ctypes.byref(p), ctypes.byref(b), name.encode(), out.ctypes.data_as(_DP), ctypes.byref(n)))
    return out


class NativeServer:
    """The C ABI's batched server (exogcm_server_*): continuous batching of
    planet runs within a device-byte budget, driven by pump()."""

    STATUS = ("queued", "running", "finished", "failed", "rejected")

    def __init__(self, budget_bytes: float, block_slots: int = 32, chunk_steps: int = 32, mode: int = 1):
        lib = load_library()
        opt = ServerOptions(budget_bytes=float(budget_bytes), block_slots=block_slots, chunk_steps=chunk_steps,
                            mode=mode)
        self.h = _VP()
        _check(lib.exogcm_server_create(ctypes.byref(opt), ctypes.byref(self.h)))

    def submit(self, planet, steps: int) -> int:
        """Queues `steps` main-loop steps of a planets.Planet; returns the request id."""
        nhor = 2 * {21: 32, 42: 64, 63: 96}[planet.config["truncation"]] ** 2
        keep = {}
        p = planet_struct(planet.config)
        b = boundary_struct(planet, nhor, keep)
        rid = ctypes.c_long()
        _check(_lib.exogcm_server_submit(self.h, ctypes.byref(p), ctypes.byref(b), int(steps), ctypes.byref(rid)))
        return rid.value

    def pump(self) -> int:
        """One scheduling round; returns the runs still queued or running."""
        active = ctypes.c_int()
        _check(_lib.exogcm_server_pump(self.h, ctypes.byref(active)))
        return active.value

    def poll(self, request: int):
        """(status name, main-loop steps done) of a request."""
        status, done = ctypes.c_int(), ctypes.c_long()
        _check(_lib.exogcm_server_poll(self.h, request, ctypes.byref(status), ctypes.byref(done)))
        return self.STATUS[status.value], done.value

    def result(self, request: int, field: str, size: int) -> np.ndarray:
        out = np.zeros(size, dtype=np.float32)
        _check(_lib.exogcm_server_result(self.h, request, field.encode(), out.ctypes.data_as(_FP), size))
        return out

    def release(self, request: int) -> None:
        _check(_lib.exogcm_server_release(self.h, request))

    def close(self):
        if _lib is None:
            return
        if getattr(self, "h", None):
            _lib.exogcm_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class Engine:
    """One batch of `slots` planets at one resolution on the current device."""

    def __init__(self, truncation: int, levels: int, slots: int = 1, mode: int = 0):
        lib = load_library()
        h = _VP()
        _check(lib.exogcm_create(truncation, levels, slots, mode, ctypes.byref(h)))
        self.h = h
        self.truncation, self.levels, self.slots = truncation, levels, slots
        self.nlat = {21: 32, 42: 64, 63: 96}[truncation]
        self.nhor = 2 * self.nlat * self.nlat
        self._keep = []

    def close(self):
        if _lib is None:  # interpreter shutdown: the library is gone already
            return
        if getattr(self, "h", None):
            _lib.exogcm_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def setup_on_device(self, enable: bool = True) -> None:
        """Where configure runs its heavy FP64 set-up loops (device by default)."""
        _check(_lib.exogcm_setup_on_device(self.h, int(bool(enable))))

    def configure(self, slot: int, planet) -> None:
        """SETUP + LAYOUT.write for a planets.Planet."""
        keep = {}
        p = planet_struct(planet.config)
        b = boundary_struct(planet, self.nhor, keep)
        _check(_lib.exogcm_configure(self.h, slot, ctypes.byref(p), ctypes.byref(b)))

    def release(self, slot: int) -> None:
        _check(_lib.exogcm_release(self.h, slot))

    def step(self, steps: int = 1, publish_every: int | None = None) -> None:
        _check(_lib.exogcm_step(self.h, steps, publish_every or max(steps, 1 << 20)))

    def step_async(self, steps: int = 1, publish_every: int | None = None) -> None:
        """Submits a batch and returns at once (at most two in flight)."""
        _check(_lib.exogcm_step_async(self.h, steps, publish_every or max(steps, 1 << 20)))

    def poll(self) -> bool:
        """True when no batch is in flight; never blocks."""
        done = ctypes.c_int()
        _check(_lib.exogcm_poll(self.h, ctypes.byref(done)))
        return bool(done.value)

    def wait(self) -> None:
        _check(_lib.exogcm_wait(self.h))

    BUDGETS = ("surface_pressure", "toa_net", "surface_net", "surface_temperature", "precipitation", "evaporation",
               "water_vapour", "weight")

    def budgets(self, slot: int, reset: bool = False) -> dict:
        """The slot's FP64 global budgets: {'last': {...}, 'mean': {...}, 'samples': n} (exogcm_budgets)."""
        last = (ctypes.c_double * 8)()
        mean = (ctypes.c_double * 8)()
        n = ctypes.c_long()
        _check(_lib.exogcm_budgets(self.h, slot, last, mean, ctypes.byref(n), 1 if reset else 0))
        return {"last": dict(zip(self.BUDGETS, last[:])), "mean": dict(zip(self.BUDGETS, mean[:])),
                "samples": n.value}

    def averages_enable(self, enable: bool = True) -> None:
        _check(_lib.exogcm_averages_enable(self.h, 1 if enable else 0))

    def averages_read(self, slot: int, reset: bool = False):
        """(mean snapshot [planes][NHOR] float32, samples) since the last reset."""
        out = np.zeros(self.field_size("snapshot"), dtype=np.float32)
        n = ctypes.c_long()
        _check(_lib.exogcm_averages_read(self.h, slot, out.ctypes.data_as(_FP), out.size, ctypes.byref(n),
                                         1 if reset else 0))
        return out.reshape(-1, self.nhor), n.value

    def run_stage(self, stage: str) -> None:
        _check(_lib.exogcm_run_stage(self.h, stage.encode()))

    def field_size(self, name: str) -> int:
        n = ctypes.c_size_t()
        _check(_lib.exogcm_field_size(self.h, name.encode(), ctypes.byref(n)))
        return n.value

    def read(self, slot: int, name: str) -> np.ndarray:
        out = np.zeros(self.field_size(name), dtype=np.float32)
        _check(_lib.exogcm_read_field(self.h, slot, name.encode(), out.ctypes.data_as(_FP), out.size))
        return out

    def write(self, slot: int, name: str, values) -> None:
        arr = np.ascontiguousarray(np.asarray(values, dtype=np.float32).reshape(-1))
        _check(_lib.exogcm_write_field(self.h, slot, name.encode(), arr.ctypes.data_as(_FP), arr.size))

    def read_table(self, slot: int, name: str, count: int) -> np.ndarray:
        out = np.zeros(count, dtype=np.float32)
        _check(_lib.exogcm_read_table(self.h, slot, name.encode(), out.ctypes.data_as(_FP), count))
        return out

    def snapshot(self, slot: int):
        """(step, values [fields][NHOR]) of the slot's snapshot published in
        the last step() call, or (-1, None)."""
        step = ctypes.c_long()
        _check(_lib.exogcm_read_snapshot(self.h, slot, None, 0, ctypes.byref(step)))
        if step.value < 0:
            return -1, None
        n = self.field_size("snapshot")
        out = np.zeros(n, dtype=np.float32)
        _check(_lib.exogcm_read_snapshot(self.h, slot, out.ctypes.data_as(_FP), n, ctypes.byref(step)))
        return step.value, out.reshape(-1, self.nhor)

    def set_stop(self, slot: int, step: int) -> None:
        """The slot stops advancing at model step `step` (-1: no limit)."""
        _check(_lib.exogcm_set_stop(self.h, slot, step))

    def read_snapshot_into(self, slot: int, out: np.ndarray) -> int:
        """Copies the slot's last published snapshot into a float32 host
        array; returns its step, or -1 (and leaves `out`) if none."""
        step = ctypes.c_long()
        _check(_lib.exogcm_read_snapshot(self.h, slot, out.ctypes.data_as(_FP), out.size, ctypes.byref(step)))
        return step.value

    def snapshots_begin(self, out: np.ndarray) -> None:
        """Starts copying every slot's snapshot field ([plane][slot][point],
        float32, pinned for overlap) as the last submitted batch leaves it,
        without waiting for batches in flight, while the caller goes on
        stepping; see snapshots_wait. `out` must stay alive until then."""
        _check(_lib.exogcm_snapshots_begin(self.h, out.ctypes.data_as(_FP), out.size))

    def snapshots_wait(self) -> None:
        _check(_lib.exogcm_snapshots_wait(self.h))

    def slot_info(self, slot: int):
        step, left, active = ctypes.c_long(), ctypes.c_int(), ctypes.c_int()
        _check(_lib.exogcm_slot_info(self.h, slot, ctypes.byref(step), ctypes.byref(left), ctypes.byref(active)))
        return dict(step=step.value, startup_left=left.value, active=bool(active.value))

    def unstable(self) -> np.ndarray:
        flags = (ctypes.c_int * self.slots)()
        _check(_lib.exogcm_unstable(self.h, flags, self.slots))
        return np.array(flags[:], dtype=bool)

    def last_step_ms(self) -> float:
        ms = ctypes.c_float()
        _check(_lib.exogcm_last_step_ms(self.h, ctypes.byref(ms)))
        return ms.value

    def time_kernel(self, kernel: str, reps: int = 10):
        """(ms per launch, algorithmic bytes per launch) of one step kernel."""
        ms, nbytes = ctypes.c_float(), ctypes.c_double()
        _check(_lib.exogcm_time_kernel(self.h, kernel.encode(), reps, ctypes.byref(ms), ctypes.byref(nbytes)))
        return ms.value, nbytes.value

    def device_field(self, name: str):
        """(device pointer, floats across all slots) of a state field."""
        ptr, n = _VP(), ctypes.c_size_t()
        _check(_lib.exogcm_device_field(self.h, name.encode(), ctypes.byref(ptr), ctypes.byref(n)))
        return ptr.value, n.value

    def tuning(self) -> dict:
        """The transform launch shapes chosen at the first configure."""
        v = (ctypes.c_int * 16)()
        _check(_lib.exogcm_tuning(self.h, v, 16))
        kinds = ("fc2sp", "uv2dv", "mktend", "qtend")
        return {"fft_rows": v[0], "sp2fc": (v[1], v[2]), "dv2uv": (v[3], v[4]),
                "forward_tiles": dict(zip(kinds, v[5:9])), "forward_buffers": dict(zip(kinds, v[9:13])),
                "sp2gp_planes": v[13], "fft_persistent": {"forward": v[14], "inverse": v[15]}}

    def graph_launches(self, steps: int) -> int:
        n = ctypes.c_size_t()
        _check(_lib.exogcm_graph_launches(self.h, steps, ctypes.byref(n)))
        return n.value

    def date(self, slot: int, step: int = -1) -> dict:
        """GcmDate (year, month, day, hour, minute) of a model step of the
        slot's planet; the slot's current step by default."""
        out = (ctypes.c_int * 5)()
        _check(_lib.exogcm_slot_date(self.h, slot, step, out))
        return dict(zip(("year", "month", "day", "hour", "minute"), list(out)))

    def checkpoint_save(self, slot: int) -> bytes:
        buf, size = _VP(), ctypes.c_size_t()
        _check(_lib.exogcm_checkpoint_save(self.h, slot, ctypes.byref(buf), ctypes.byref(size)))
        try:
            return ctypes.string_at(buf, size.value)
        finally:
            _lib.exogcm_free(buf)

    def checkpoint_load(self, slot: int, data: bytes) -> None:
        _check(_lib.exogcm_checkpoint_load(self.h, slot, data, len(data)))
