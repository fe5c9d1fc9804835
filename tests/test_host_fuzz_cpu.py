"""The input-folder parsers under malformed input (CPU only).

The reference exits on some malformed files and reads past buffers on others
(2phase_n-tau-leaping.cu read_stoichiometry 122-457, read_time_series
1056-1261).  Here every parser returns a status: seeded random mutations of
a valid folder -- deleted, inserted, repeated and truncated bytes, huge and
out-of-range numbers, empty and missing files -- must load or fail with a
CtlError, in a child process so that a crash fails the test instead of
ending the run.  One regression case came from such a run: a huge ts_rep
made the target loader attempt a multi-terabyte allocation and abort.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import cutauleaping_b200 as ctl
from cutauleaping_b200 import inputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

FUZZ = r'''
import os, random, shutil, sys
import numpy as np
import cutauleaping_b200 as ctl
from cutauleaping_b200 import inputs
base, seed, count = sys.argv[1], int(sys.argv[2]), int(sys.argv[3])
src = os.path.join(base, "src")
net = inputs.schlogl(8, samples=6, t_end=1.0)
inputs.write_folder(src, net, {"ts_rep": 2, "p_rep": 2, "ts_numtgt": 3, "tts_vector": [4, 8],
                               "ts_matrix": np.arange(6 * 2 * 2 * 3).reshape(6, 2, 2, 3)})
files = sorted(os.listdir(src))
tokens = ["\t", "\n", "\r", " ", "-", ".", "e", "+", "x", "0", "1", "9", "4294967296", "-2147483649",
          "1e309", "nan", "inf", "\x00", "99999999999999999999", "127", "128", "-1"]
rng = random.Random(seed)
case = os.path.join(base, "case")
for it in range(count):
    shutil.rmtree(case, ignore_errors=True)
    shutil.copytree(src, case)
    p = os.path.join(case, rng.choice(files))
    data = open(p, "rb").read().decode("latin-1")
    for _ in range(rng.randint(1, 4)):
        op, i = rng.randrange(7), rng.randrange(len(data) + 1)
        if op == 0 and data:
            data = data[:i] + data[i + 1:]
        elif op == 1:
            data = data[:i] + rng.choice(tokens) + data[i:]
        elif op == 2:
            data = data[:i]
        elif op == 3:
            lines = data.split("\n"); j = rng.randrange(len(lines)); lines.insert(j, lines[j])
            data = "\n".join(lines)
        elif op == 4:
            data = data[:i] + rng.choice(tokens) * rng.randint(1, 3000) + data[i:]
        elif op == 5:
            data = ""
        else:
            os.remove(p); data = None; break
    if data is not None:
        open(p, "wb").write(data.encode("latin-1"))
    try:
        m = ctl.Model.load(case)
        ctl.load_rows(case, m, 0, 8)
        ctl.Target(case, m, threads=2, blocks=4)
    except ctl.CtlError:
        pass
print("fuzz ok", count)
'''


def _target_folder(tmp_path, **edits):
    net = inputs.schlogl(8, samples=6, t_end=1.0)
    folder = inputs.write_folder(str(tmp_path / "f"), net, {
        "ts_rep": 2, "p_rep": 2, "ts_numtgt": 3, "tts_vector": [4, 8],
        "ts_matrix": np.arange(6 * 2 * 2 * 3).reshape(6, 2, 2, 3)})
    for name, text in edits.items():
        with open(os.path.join(folder, name), "w") as f:
            f.write(text)
    return folder


@pytest.mark.parametrize("ts_rep,status", [("4294967295\n", ctl.ERR_SHAPE), ("16777217\n", ctl.ERR_SHAPE),
                                           ("99999999999999999999999\n", ctl.ERR_PARSE)])
def test_huge_target_counts_fail_cleanly(tmp_path, ts_rep, status):
    folder = _target_folder(tmp_path, ts_rep=ts_rep)
    m = ctl.Model.load(folder)
    with pytest.raises(ctl.CtlError) as e:
        ctl.Target(folder, m, threads=2, blocks=4)
    assert e.value.status == status


def test_out_of_range_integers_are_parse_errors(tmp_path):
    folder = _target_folder(tmp_path, left_side="99999999999999999999\t2\t0\n0\t3\t0\n0\t0\t1\n0\t1\t0\n")
    with pytest.raises(ctl.CtlError) as e:
        ctl.Model.load(folder)
    assert e.value.status == ctl.ERR_PARSE


def test_mutated_folders_load_or_fail_with_a_status(tmp_path):
    p = subprocess.run([sys.executable, "-c", FUZZ, str(tmp_path), "11", "600"], cwd=ROOT, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0 and "fuzz ok" in p.stdout, p.stderr[-3000:]
