"""The bounds-checked build (lib/libgrn_b200_checked.so, GRN_BOUNDS_CHECK):
every state access of the simulation kernel is checked against its block's
shared-memory state area and the launch's global slots (and float4 accesses
for 16-byte alignment), with a bad access redirected to a scratch word and
reported as GRN_ERR_KERNEL instead of faulting.  This is the memory check
the tests can run on a GPU without a sanitizer.

CPU: the checked library is built and exports what the normal one does.
GPU: every schedule on small grids (tests/bounds_cases.py) runs clean
through the checked library -- no access outside its buffer -- and gives
bit-identical states and errors to the normal library."""
import os
import subprocess
import sys

import numpy as np
import pytest

import grn_b200 as grn

HERE = os.path.dirname(os.path.abspath(__file__))
CHECKED = os.path.join(os.path.dirname(grn.LIB_PATH), "libgrn_b200_checked.so")


def _exports(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return set(line.split()[-1] for line in out.splitlines() if line.strip())


def test_checked_library_is_built_with_the_same_entry_points(built_libs):
    assert os.path.exists(CHECKED)
    want = set(n for n in _exports(grn.LIB_PATH) if n.startswith("grn_"))
    assert want and want <= _exports(CHECKED)


@pytest.mark.gpu
def test_every_schedule_is_in_bounds_and_unchanged(built_libs, tmp_path):
    out = tmp_path / "checked.npz"
    r = subprocess.run([sys.executable, os.path.join(HERE, "bounds_cases.py"), CHECKED,
                        str(out)], capture_output=True, text=True, timeout=900)
    # A bad access shows up as GrnError(GRN_ERR_KERNEL, "bounds check: ...").
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    checked = np.load(out)
    import bounds_cases
    normal = bounds_cases.run_cases()
    assert set(checked.files) == set(normal)
    for name, value in normal.items():
        assert np.array_equal(checked[name], value, equal_nan=True), name
