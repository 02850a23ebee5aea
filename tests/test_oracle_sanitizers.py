"""The oracle under AddressSanitizer and UndefinedBehaviorSanitizer (CPU).

The checker is C, so an out-of-bounds index or an overflow in it would make
every parity claim built on it suspect.  This test builds the same source with
-fsanitize=address,undefined (every UB report fatal), runs each oracle routine
once on small cells in a child process with libasan preloaded, and requires a
clean exit with no sanitizer report.
"""
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))

CHILD = r"""
import sys
sys.path[:0] = [sys.argv[1], sys.argv[1] + "/oracle", sys.argv[1] + "/tests"]
import numpy as np
import helpers as H
import oracle as O
import ctypes

assert O.lib()._name.endswith("libfp4_oracle_san.so"), O.lib()._name
assert hasattr(ctypes.CDLL(None), "__asan_report_load8")  # the runtime is preloaded

for kind, grid in (("diamond", (3, 3, 3)), ("layered", (2, 2, 2))):
    s = H.cached_solve(kind, grid, temperatures=(300.0,))
    o = O.Oracle(s, T=300.0)
    n_p, n_m, _, _ = o.np3()
    n4, _ = o.np4()
    r3 = o.rta3()
    r4 = o.rta4()
    o.rta4_range(s.nb, 2 * s.nb, 0, 2)
    o.rta4_pairs(np.arange(4, dtype=np.int64), np.arange(4, dtype=np.int64))
    mm = s.nb + 2
    o.ind_only3(mm, 0, int(n_p[mm - 1]))
    o.ind_only4(mm, 1, int(n4[1][mm - 1]))
    lists = o.ind3(n_p, n_m)
    ind4 = o.ind4(*n4)
    rate = lists["rate_plus"] + lists["rate_minus"] + ind4["rate_pp"] + ind4["rate_pm"] + ind4["rate_mm"]
    tau = np.zeros_like(rate)
    tau[rate != 0] = 1.0 / rate[rate != 0]
    F = o.iteration0(tau)
    F = o.iteration(F, tau, n_p, n_m, lists, ind4=ind4)
    F = o.symmetrize_fn(F)
    o.tconduct(F)
    o.cumulative_tconduct(F)
    o.cumulative_tconduct(F, omega_mode=True)
    o.sample4(2000, 11, mode=2, mm0=s.nb, mm1=2 * s.nb)
    o.sample3(2000, 11, mode=2, mm0=s.nb, mm1=2 * s.nb)
    o.vp4(0, 1, 1, 1, 1, 1, 2, 3, 4)
    o.vp3(0, 1, 1, 1, 1, 2, 3)
    assert np.isfinite(r3[0]).all() and np.isfinite(r4[0]).all()
print("SANITIZED ORACLE OK")
"""


def test_oracle_is_clean_under_asan_and_ubsan():
    if shutil.which("make") is None or not os.path.exists("/usr/bin/gcc"):
        pytest.skip("no C toolchain")
    asan = subprocess.run(["/usr/bin/gcc", "-print-file-name=libasan.so"], capture_output=True, text=True).stdout.strip()
    if not asan or not os.path.isabs(asan) or not os.path.exists(asan):
        pytest.skip("libasan is not available")
    b = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "sanitize"], capture_output=True, text=True)
    assert b.returncode == 0, b.stderr
    env = dict(os.environ)
    env.update(LD_PRELOAD=asan, ASAN_OPTIONS="detect_leaks=0:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1", OMP_NUM_THREADS=str(min(8, os.cpu_count() or 1)),
               FP4_ORACLE_LIB=os.path.join(ROOT, "oracle", "_san", "libfp4_oracle_san.so"))
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT], capture_output=True, text=True, env=env, timeout=900)
    report = r.stderr[-4000:]
    assert r.returncode == 0, report
    assert "SANITIZED ORACLE OK" in r.stdout, report
    assert "runtime error" not in r.stderr and "AddressSanitizer" not in r.stderr, report
