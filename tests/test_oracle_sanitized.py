"""The oracle under AddressSanitizer and UndefinedBehaviorSanitizer.

The reference has no sanitizer runs and one known out-of-bounds read (the
RAV walk of 2phase_n-tau-leaping.cu:1870); compute-sanitizer is not used on
the GPU side here.  The oracle, which every parity test trusts, is rebuilt
from oracle/ctl_oracle.c with -fsanitize=address,undefined (any report
aborts) and run on the small networks of the parity tests -- every reaction
order, feed species, per-simulation rates -- in dynamics, forced-SSA and
all-quirks-off modes, plus the exact Gillespie method and the Poisson
sampler on both of its branches.  CPU only.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r'''
import numpy as np
import oracle
from tests.netutil import oracle_run, oracle_model, small_networks
for name, net in small_networks():
    for flags in (0, oracle.FORCE_SSA, oracle.ALL_QUIRKS_OFF):
        oracle_run(net, seed=3, flags=flags)
    oracle_model(net, seed=3).gillespie(net.X0[:8], np.asarray(net.c[:8], np.float32))
for lam in (0.0, 0.5, 9.9, 10.0, 37.5, 2.5e6):
    oracle.poisson(lam, 1, 2, 3, 0, 5)
assert oracle._lib._name == __import__("os").environ["CTL_ORACLE_LIB"]
print("sanitized oracle ok")
'''


def _runtime(name):
    p = subprocess.run(["gcc", f"-print-file-name={name}"], capture_output=True, text=True)
    path = p.stdout.strip()
    return path if p.returncode == 0 and os.path.isabs(path) and os.path.exists(path) else None


def test_oracle_clean_under_asan_and_ubsan(tmp_path):
    asan = _runtime("libasan.so")
    if asan is None:
        pytest.skip("no AddressSanitizer runtime for gcc on this host")
    lib = str(tmp_path / "libctl_oracle_san.so")
    subprocess.run(["gcc", "-O1", "-g", "-std=c11", "-fPIC", "-ffp-contract=off", "-fno-omit-frame-pointer",
                    "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined", "-shared", "-o", lib,
                    os.path.join(ROOT, "oracle", "ctl_oracle.c"), "-lm", "-lpthread"], check=True)
    env = dict(os.environ, CTL_ORACLE_LIB=lib, LD_PRELOAD=asan, ASAN_OPTIONS="detect_leaks=0:abort_on_error=1",
               UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1")
    p = subprocess.run([sys.executable, "-c", DRIVER], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0 and "sanitized oracle ok" in p.stdout, p.stderr[-4000:]
