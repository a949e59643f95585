"""Shared pytest setup.

Markers: ``gpu`` -- needs a CUDA device (a B200 for the parity and timing
tests).  Everything else runs on a CPU-only host.

GPU availability is decided once per session, before any test touches CUDA,
by a probe in a child process that calls the driver directly (``cuInit`` and
``cuDeviceGetCount`` through ``libcuda.so.1``).  The probe runs in a child
because a failed initialisation is remembered for the life of a process, both
by the driver and by torch, which would turn a device that is merely slow to
come up into a whole session without CUDA.

* When the ``gpu`` marker was asked for explicitly (``-m gpu``) the probe is
  retried for up to ``MCKL_B200_GPU_PROBE_S`` seconds (default 120) and, if the
  device never answers, the session FAILS with the driver's return code and
  the environment it saw.  A GPU run never passes by skipping its tests.
* Otherwise (a plain ``pytest tests/`` on a CPU-only host) the GPU tests are
  skipped with the probe's reason.

GPU test modules call :func:`require_cuda` in their fixtures; once the probe
has said yes, a torch that still cannot see the device is an error, not a skip.
"""
import os
import subprocess
import sys
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

_PROBE = r"""
import ctypes, sys
try:
    cu = ctypes.CDLL("libcuda.so.1")
except OSError as e:
    print("dlopen(libcuda.so.1) failed: %s" % e)
    sys.exit(2)
rc = cu.cuInit(0)
if rc != 0:
    print("cuInit(0) returned %d" % rc)
    sys.exit(3)
n = ctypes.c_int(0)
rc = cu.cuDeviceGetCount(ctypes.byref(n))
if rc != 0 or n.value < 1:
    print("cuDeviceGetCount returned %d, count %d" % (rc, n.value))
    sys.exit(4)
print("ok: %d device(s)" % n.value)
"""

_STATE = {"ok": None, "reason": ""}


def _probe_once():
    try:
        r = subprocess.run([sys.executable, "-c", _PROBE], capture_output=True, text=True, timeout=120)
    except subprocess.TimeoutExpired:
        return False, "driver probe did not finish within 120 s"
    out = (r.stdout + r.stderr).strip()
    return r.returncode == 0, out


def _environment_report():
    keys = ("CUDA_VISIBLE_DEVICES", "NVIDIA_VISIBLE_DEVICES", "CUDA_DEVICE_ORDER", "LD_LIBRARY_PATH",
            "LD_PRELOAD", "PYTHONPATH")
    lines = [f"{k}={os.environ.get(k, '<unset>')}" for k in keys]
    try:
        lines.append("device nodes: " + " ".join(sorted(n for n in os.listdir("/dev") if n.startswith("nvidia"))))
    except OSError as e:
        lines.append(f"device nodes: {e}")
    try:
        smi = subprocess.run(["nvidia-smi", "-L"], capture_output=True, text=True, timeout=30)
        lines.append("nvidia-smi -L: " + (smi.stdout + smi.stderr).strip().replace("\n", " | "))
    except (OSError, subprocess.TimeoutExpired) as e:
        lines.append(f"nvidia-smi -L: {e}")
    return "\n  ".join(lines)


def _gpu_explicitly_selected(config):
    expr = (config.option.markexpr or "").replace("(", " ").replace(")", " ").split()
    return "gpu" in expr and "not" not in expr


def probe_gpu(config):
    """Decide once whether this session has a CUDA device (see module doc)."""
    if _STATE["ok"] is not None:
        return _STATE["ok"]
    explicit = _gpu_explicitly_selected(config)
    limit = float(os.environ.get("MCKL_B200_GPU_PROBE_S", "120")) if explicit else 0.0
    t0 = time.monotonic()
    attempts = 0
    while True:
        attempts += 1
        ok, out = _probe_once()
        if ok or time.monotonic() - t0 >= limit:
            break
        time.sleep(3.0)
    _STATE["ok"] = ok
    _STATE["reason"] = out
    if not ok and explicit:
        msg = (f"GPU tests were selected but the CUDA driver did not initialise after {attempts} attempt(s) "
               f"over {time.monotonic() - t0:.0f} s: {out}\n  {_environment_report()}")
        pytest.exit(msg, returncode=1)
    return ok


def require_cuda():
    """For GPU test fixtures: the device the session probe found must be
    usable from torch; anything else fails the test with the reason."""
    import torch

    if not _STATE["ok"]:
        pytest.skip("no CUDA device: " + (_STATE["reason"] or "probe not run"))
    if not torch.cuda.is_available():
        pytest.fail("the driver probe found a device but torch cannot initialise CUDA in this process "
                    f"({_STATE['reason']})\n  {_environment_report()}")
    torch.cuda.set_device(0)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run on a B200)")


@pytest.hookimpl(trylast=True)
def pytest_collection_modifyitems(session, config, items):
    """Runs after the marker expression has deselected items: probe the device
    only when GPU tests remain, and skip them on a host without one (unless
    they were asked for explicitly, in which case the session fails)."""
    gpu_items = [it for it in items if it.get_closest_marker("gpu") is not None]
    if not gpu_items:
        return
    if not probe_gpu(config):
        skip = pytest.mark.skip(reason="no CUDA device: " + _STATE["reason"])
        for it in gpu_items:
            it.add_marker(skip)
