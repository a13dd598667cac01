"""GCM_RUNNER: the reference's run-control interface over the CUDA engine.

Mirrors src/model/climate/gcm/runner/index.ts:61-78 (GCM_RUNNER.start),
runner/types.ts:34-74 (GcmRunRequest, GcmRun, the status enum) and the
WebGPU worker's loop (runner/webgpu/gcm.worker.ts:53-367): a run owns one
engine slot on a worker thread, pumps batches of whole publish intervals,
posts each published snapshot, pauses and resumes between batches, takes a
checkpoint (the format-21 container, checkpoint.py) once the device is
idle, and fails with the reference's messages
("GPU device lost: ...", "The model became unstable at step N",
"This checkpoint's model state does not match ...").
"""
from __future__ import annotations

import importlib
import threading
import time
from dataclasses import dataclass, field
from typing import Callable, Optional

STATUSES = ("loading", "running", "paused", "checkpointing", "finished", "failed")
# runner/webgpu/gcm.worker.ts and stepper/index.ts:168-184: a batch is a whole
# number of publish intervals, at most MAX_INTERVALS of them.
MAX_INTERVALS = 16


@dataclass
class GcmRunRequest:
    """runner/types.ts:47-67, for the GPU engine."""
    planet: object                      # planets.Planet: config + boundary + initial state
    publish_every: int = 32
    restart: Optional[bytes] = None
    start_paused: bool = False
    max_steps: Optional[int] = None     # stop after this many main-loop steps (None: until stop())
    on_snapshot: Callable = lambda snapshot: None
    on_status: Callable = lambda update: None
    on_device: Callable = lambda description: None
    on_checkpoint: Callable = lambda saved: None


@dataclass
class GcmSnapshot:
    """types.ts:74-79: layers, step and the packed field values."""
    layers: int
    step: int
    values: object


@dataclass
class GcmStatusUpdate:
    status: str
    message: str = ""


class GcmRun:
    """runner/types.ts:69-74: the control handle of a started run."""

    def __init__(self, request: GcmRunRequest):
        self.request = request
        self._paused = threading.Event()
        if request.start_paused:
            self._paused.set()
        self._stop = threading.Event()
        self._checkpoint = threading.Event()
        self._thread = threading.Thread(target=self._work, daemon=True)
        self.status = "loading"
        self.error: Optional[str] = None
        self.step = 0
        self._thread.start()

    # -- GcmRun -------------------------------------------------------------
    def pause(self):
        self._paused.set()

    def resume(self):
        self._paused.clear()

    def checkpoint(self):
        self._checkpoint.set()

    def stop(self):
        self._stop.set()

    def join(self, timeout=None):
        self._thread.join(timeout)

    # -- worker ---------------------------------------------------------------
    def _status(self, status, message=""):
        self.status = status
        self.request.on_status(GcmStatusUpdate(status, message))

    def _fail(self, message):
        self.error = message
        self._status("failed", message)

    def _work(self):
        pkg = importlib.import_module("web-exoplasim_b200")
        checkpoint = importlib.import_module("web-exoplasim_b200.checkpoint")
        req = self.request
        cfg = req.planet.config
        try:
            engine = pkg.Engine(cfg["truncation"], cfg["layers"], 1)
            engine.configure(0, req.planet)
            if req.restart is not None:
                engine.step(3)  # a restarted run resumes in the main loop
                if bytes(req.restart[:len(checkpoint.MAGIC)]) == checkpoint.MAGIC:
                    checkpoint.load(engine, 0, req.restart)  # the format-21 container
                else:
                    engine.checkpoint_load(0, req.restart)  # a bare restart file
            else:
                engine.step(3)  # master's start-up steps at the start step's date
            info = engine.slot_info(0)
            start = info["step"]
            if req.max_steps is not None:
                engine.set_stop(0, start + req.max_steps)
            req.on_device("NVIDIA B200 (CUDA, sm_100a)")
        except (pkg.ExogcmError, checkpoint.CheckpointError) as err:
            self._fail(str(err))
            return
        except Exception as err:  # device unavailable and the like
            self._fail(f"GPU device lost: {err}")
            return
        publish = max(1, req.publish_every)
        self._status("paused" if self._paused.is_set() else "running")
        try:
            while not self._stop.is_set():
                if self._checkpoint.is_set():
                    self._status("checkpointing")
                    req.on_checkpoint(checkpoint.save(engine, 0, req.planet))
                    self._checkpoint.clear()
                    self._status("paused" if self._paused.is_set() else "running")
                if self._paused.is_set():
                    time.sleep(0.01)
                    continue
                info = engine.slot_info(0)
                self.step = info["step"]
                if req.max_steps is not None and self.step >= start + req.max_steps:
                    self._status("finished")
                    break
                # one publish interval per engine call, ending on a publishing step
                first = self.step + ((publish - self.step % publish) % publish)
                count = min(first - self.step + 1, publish, 64)
                engine.step(count, publish_every=publish)
                if engine.unstable()[0]:
                    self._fail(f"The model became unstable at step {engine.slot_info(0)['step'] - 1}")
                    return
                step, values = engine.snapshot(0)
                if step >= 0:
                    req.on_snapshot(GcmSnapshot(layers=cfg["layers"], step=step, values=values))
            else:
                self._status("finished")
        except pkg.ExogcmError as err:
            self._fail(str(err))
        finally:
            engine.close()


class _Runner:
    """runner/index.ts:61-78: GCM_RUNNER.start routes to the GPU engine."""

    resolutions = ((21, 5), (21, 10), (42, 5), (42, 10), (63, 5), (63, 10))

    def start(self, request: GcmRunRequest) -> GcmRun:
        return GcmRun(request)


GCM_RUNNER = _Runner()
