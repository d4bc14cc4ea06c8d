"""The bounds-checked build (libspearhed_b200_check.so, compiled with
-DSPH_CHECK).

Its kernels check the indices they read through (stencil cell ids, cell
source ranges, staged candidates, target ranges, list entries read back,
permutation indices, sorted cell keys, drift cells) and, on a failed check,
set that site's bit in a status word and skip the access; the host turns the
word into SPH_ERR_STATE.  It is the substitute for compute-sanitizer, which is
closed on this pool.

Without a GPU: the checked library loads and exports every declared entry
point.  With one: the parity, ensemble, species and configuration tests run
on the checked library (a child pytest with SPEARHED_B200_VARIANT=check) and
pass, i.e. no check fires and every result still matches the oracle.
"""
import os
import re
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK_LIB = os.path.join(ROOT, "spearhed_b200", "_lib", "libspearhed_b200_check.so")


def _env():
    env = dict(os.environ)
    env["SPEARHED_B200_VARIANT"] = "check"
    return env


def test_checked_library_loads_and_exports_the_boundary():
    assert os.path.exists(CHECK_LIB), "build() makes the checked twin"
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from spearhed_b200 import abi\n"
            "import tests.test_abi_symbols as t\n"
            "assert abi.LIB_PATH.endswith('libspearhed_b200_check.so'), abi.LIB_PATH\n"
            "L = abi.lib()\n"
            "missing = [n for n in t.declared() if not hasattr(L, n)]\n"
            "assert not missing, missing\n"
            "print('ok', len(t.declared()))\n") % ROOT
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=_env(), capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("ok")


@pytest.mark.gpu
def test_parity_suites_pass_on_the_checked_build():
    files = ["tests/test_gpu_parity.py", "tests/test_gpu_ensemble.py", "tests/test_gpu_species.py",
             "tests/test_gpu_configs.py"]
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider"] + files,
                       cwd=ROOT, env=_env(), capture_output=True, text=True, timeout=1800)
    tail = "\n".join(r.stdout.splitlines()[-15:])
    assert r.returncode == 0, tail + r.stderr[-2000:]
    # every selected test ran and passed on the checked library: none skipped
    summary = r.stdout.strip().splitlines()[-1]
    m = re.search(r"(\d+) passed", summary)
    assert m and int(m.group(1)) >= 50, summary  # 82 selected at the time of writing
    assert not re.search(r"skipped|failed|error", summary), summary
