"""The two executables' argument and input checks, which run before any device
work, so these run without a GPU: usage on too few arguments, unknown forms,
the active-dims range, missing files, binary files of the wrong size, CSV
files with too few rows (comment lines do not count), and engine rejections
reported as "join failed" with the engine's message."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "hilbertjoin_b200", "bin")
SELF = os.path.join(BIN, "hilbertSelfJoinCardinality")
JOIN = os.path.join(BIN, "hilbertJoinCardinality")

pytestmark = pytest.mark.skipif(not (os.path.exists(SELF) and os.path.exists(JOIN)),
                                reason="executables not built")


def run(args):
    r = subprocess.run(args, capture_output=True, text=True, timeout=120)
    return r.returncode, r.stderr


def test_usage_on_too_few_arguments():
    for exe, flags in ((SELF, "-n N -e EPS -d D"), (JOIN, "-n N -m M -e EPS -d D")):
        rc, err = run([exe, "-n", "10"])
        assert rc == 1 and "Usage" in err and flags in err


def test_unknown_form_and_active_dims():
    rc, err = run([SELF, "-n", "16", "-e", "0.1", "-d", "4", "-F", "int8"])
    assert rc == 1 and "unknown form 'int8'" in err
    rc, err = run([SELF, "-n", "16", "-e", "0.1", "-d", "4", "-s", "6"])
    assert rc == 1 and "active dimensions must be in [0, 5]" in err


def test_missing_file(tmp_path):
    p = str(tmp_path / "nope.csv")
    rc, err = run([SELF, "-n", "16", "-e", "0.1", "-d", "4", "-f", p])
    assert rc == 1 and f"File '{p}' does not exist!" in err
    a = tmp_path / "a.bin"
    np.zeros((16, 4)).tofile(a)
    rc, err = run([JOIN, "-n", "16", "-m", "16", "-e", "0.1", "-d", "4", "-f", str(a), "-g", p])
    assert rc == 1 and "does not exist" in err


@pytest.mark.parametrize("ext,dtype", [("bin", np.float64), ("f32", np.float32)])
def test_binary_size_checked(tmp_path, ext, dtype):
    p = tmp_path / f"x.{ext}"
    np.zeros(10, dtype).tofile(p)
    rc, err = run([SELF, "-n", "12", "-e", "0.1", "-d", "4", "-f", str(p)])
    assert rc == 1 and "holds 10 values, 48 expected" in err


def test_csv_rows_counted_without_comments(tmp_path):
    p = tmp_path / "x.csv"
    p.write_text("% header\n1,2,3\n% another comment\n4,5,6\n")
    rc, err = run([SELF, "-n", "3", "-e", "0.1", "-d", "3", "-f", str(p)])
    assert rc == 1 and "holds 2 rows, 3 expected" in err


def test_engine_rejection_is_reported(tmp_path):
    rc, err = run([SELF, "-n", "64", "-e", "-0.5", "-d", "4"])
    assert rc == 2 and "join failed: invalid argument" in err and "eps" in err
    rc, err = run([JOIN, "-n", "64", "-m", "64", "-e", "0.5", "-d", "1100"])
    assert rc == 2 and "join failed: invalid argument" in err and "d must be" in err


def test_no_device_is_reported():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    rc, err = run([SELF, "-n", "64", "-e", "0.5", "-d", "4"])
    assert rc == 2 and "join failed" in err
