"""Host logic of the product on CPU: the C ABI loads and exports every symbol
include/ctl.h declares, the input-folder parsers (2phase_n-tau-leaping.cu
first_pass 90-120, read_stoichiometry 122-457, read_quantities_offset 570-649,
read_parameters_offset 717-782, read_instants 932-1053) produce the same
tables as the oracle, their error paths return statuses instead of exiting,
the dynamics writer is byte-compatible with WriteDynamics2 (3431-3469), and
the CLI's early exits keep the reference's exit codes.  No GPU calls."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

import cutauleaping_b200 as ctl
import oracle
from cutauleaping_b200 import inputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "ctl.h")).read()
    declared = set(re.findall(r"\b(ctl_[a-z_]+)\s*\(", hdr))
    assert declared == set(ctl.EXPORTS)
    L = ctl.lib()
    for name in declared:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", ctl.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (ctl_\w+)", out))
    assert declared <= exported


def test_schlogl_folder_roundtrip(tmp_path):
    net = inputs.schlogl(32)
    folder = inputs.write_folder(str(tmp_path / "schlogl"), net)
    m = ctl.Model.load(folder)
    assert (m.S, m.R, m.P, m.ns, m.s_out) == (3, 4, 4, 100, 3)
    assert m.tmax == 5.0
    X0, c = ctl.load_rows(folder, m, 0, 32)
    assert np.array_equal(X0, net.X0)
    assert np.array_equal(c, net.c.astype(np.float32))
    X0b, _ = ctl.load_rows(folder, m, 5, 3)
    assert np.array_equal(X0b, net.X0[5:8])


@pytest.mark.parametrize("seed", range(6))
def test_hor_tables_match_oracle(seed):
    left, right, _, _ = inputs.random_network(10, 24, seed, max_order=3)
    tvec = np.linspace(0.1, 1, 10)
    m = ctl.Model.create(left, right, None, tvec)
    om = oracle.OracleModel(left, right, None, tvec)
    h1, t1 = m.hor()
    h2, t2 = om.hor()
    assert np.array_equal(h1, h2) and np.array_equal(t1, t2)


def test_schlogl_hor_is_the_reference_value():
    net = inputs.schlogl(1)
    hor, hort = ctl.Model.create(net.left, net.right, net.feed, net.tvec).hor()
    # A: order-3 reaction with coefficient 1; X: order 3, max coefficient 3; B: order 1.
    assert list(hor) == [3, 3, 1] and list(hort) == [1, 3, 1]


def _folder(tmp_path, **edits):
    net = inputs.schlogl(8)
    folder = inputs.write_folder(str(tmp_path / "m"), net)
    for name, text in edits.items():
        path = os.path.join(folder, name)
        if text is None:
            os.remove(path)
        else:
            with open(path, "w") as f:
                f.write(text)
    return folder


@pytest.mark.parametrize("edit,status", [
    ({"left_side": None}, ctl.ERR_IO),
    ({"t_vector": None}, ctl.ERR_IO),
    ({"left_side": "1\t2\t0\n0\t3\n0\t0\t1\n0\t1\t0\n"}, ctl.ERR_SHAPE),
    ({"right_side": "0\t3\t0\n1\t2\t0\n"}, ctl.ERR_SHAPE),
    ({"left_side": "1\tx\t0\n0\t3\t0\n0\t0\t1\n0\t1\t0\n"}, ctl.ERR_PARSE),
    ({"left_side": "-1\t2\t0\n0\t3\t0\n0\t0\t1\n0\t1\t0\n"}, ctl.ERR_SHAPE),
    ({"cs_vector": "0\n7\n"}, ctl.ERR_SHAPE),
])
def test_model_load_errors(tmp_path, edit, status):
    folder = _folder(tmp_path, **edit)
    with pytest.raises(ctl.CtlError) as e:
        ctl.Model.load(folder)
    assert e.value.status == status


def test_missing_optional_files(tmp_path):
    folder = _folder(tmp_path, M_feed=None, cs_vector=None)
    m = ctl.Model.load(folder)
    assert m.s_out == 3


# ctl_error_detail codes (include/ctl.h): the CLI maps them to the
# reference's exit codes -4, -5, -6 and -10.
DETAIL_NONE, DETAIL_MX0_UNREADABLE, DETAIL_ROWS_SHORT, DETAIL_MX0_ROW, DETAIL_TARGET_ASSIGN = range(5)


@pytest.mark.parametrize("edit,n,status,detail", [
    ({}, 9, ctl.ERR_SHAPE, DETAIL_ROWS_SHORT),                               # read_quantities_offset exit(-4)
    ({"MX_0": "1\t2\n" * 8}, 8, ctl.ERR_SHAPE, DETAIL_MX0_ROW),              # exit(-5)
    ({"MX_0": None}, 8, ctl.ERR_IO, DETAIL_MX0_UNREADABLE),                  # exit(-6)
    ({"c_matrix": "1\t2\t3\n" * 8}, 8, ctl.ERR_SHAPE, DETAIL_NONE),          # too many / few parameters
    ({"c_matrix": "1\t2\t3\t4\n" * 4}, 8, ctl.ERR_SHAPE, DETAIL_NONE),       # fewer rows than requested
    ({"MX_0": "1\t-2\t3\n" * 8}, 8, ctl.ERR_SHAPE, DETAIL_MX0_ROW),          # negative population
])
def test_rows_load_errors(tmp_path, edit, n, status, detail):
    folder = _folder(tmp_path, **edit)
    m = ctl.Model.create(*[np.array(x) for x in ([[1, 2, 0], [0, 3, 0], [0, 0, 1], [0, 1, 0]],
                                                  [[0, 3, 0], [1, 2, 0], [0, 1, 0], [0, 0, 1]])],
                         [1, 0, 1], np.arange(1, 11) * 0.5)
    with pytest.raises(ctl.CtlError) as e:
        ctl.load_rows(folder, m, 0, n)
    assert e.value.status == status
    assert e.value.detail == detail


def test_write_dynamics_format(tmp_path):
    net = inputs.schlogl(3, samples=7, t_end=1e-4 * 7)
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    rng = np.random.default_rng(0)
    samples = rng.integers(0, 2**32 - 1, size=(3, 7, 3), dtype=np.uint64).astype(np.uint32)
    prefix = str(tmp_path / "pref")
    m.write_dynamics(prefix, samples, threads=2)
    for gid in range(3):
        got = open(f"{prefix}_{gid}").read()
        # std::ostream default formatting of a double == printf("%g")
        exp = "".join("%g" % t + "".join(f"\t{v}" for v in samples[gid, i]) + "\n"
                      for i, t in enumerate(net.tvec))
        assert got == exp


def test_fitness_target_load(tmp_path):
    net = inputs.schlogl(8, samples=5, t_end=1.0)
    ts = np.arange(5 * 2 * 3 * 3).reshape(5, 2, 3, 3)
    target = {"ts_rep": 3, "p_rep": 2, "ts_numtgt": 3, "tts_vector": [4, 8], "ts_matrix": ts}
    folder = inputs.write_folder(str(tmp_path / "f"), net, target)
    m = ctl.Model.load(folder)
    t = ctl.Target(folder, m, threads=2, blocks=4)
    assert (t.repetitions, t.p_rep, t.target_quantities, t.experiments) == (3, 2, 3, 2)
    with pytest.raises(ctl.CtlError):
        ctl.Target(folder, m, threads=2, blocks=3)   # p_rep does not divide blocks
    with pytest.raises(ctl.CtlError) as e:
        ctl.Target(folder, m, threads=2, blocks=6)   # tts_vector covers 8 of 12 simulations
    assert e.value.detail == DETAIL_TARGET_ASSIGN


def _cli(*args, cwd=None):
    return subprocess.run([ctl.CLI_PATH, *map(str, args)], capture_output=True, text=True,
                          cwd=cwd, timeout=60)


def test_cli_usage_and_early_exit_codes(tmp_path):
    p = _cli("only", "three", "args")
    assert p.returncode == 255 and "ERROR: please specify" in p.stdout
    folder = _folder(tmp_path)
    p = _cli(folder, 4, 4, 0, 0, tmp_path / "out", "pref", 0, 0, 0)     # 16 rows > 8 in MX_0
    assert p.returncode == 256 - 4, p.stderr
    p = _cli(tmp_path / "nope", 2, 2, 0, 0, tmp_path / "out", "pref", 0, 0, 0)
    assert p.returncode == 255
    folder2 = _folder(tmp_path / "x", MX_0=None)
    p = _cli(folder2, 2, 2, 0, 0, tmp_path / "out", "pref", 0, 0, 0)
    assert p.returncode == 256 - 6
    # negative counts and threads*blocks beyond 32 bits are refused before any work
    for args in ((-4, 4, 0), (4, -4, 0), (4, 4, -1), (70000, 70000, 0)):
        p = _cli(folder, args[0], args[1], 0, args[2], tmp_path / "out", "pref", 0, 0, 0)
        assert p.returncode == 255 and "threads*blocks" in p.stderr, (args, p.stderr)
    # a batch far beyond the rows of MX_0 is refused before its buffers are allocated
    p = _cli(folder, 65536, 65535, 0, 0, tmp_path / "out", "pref", 0, 0, 0)
    assert p.returncode == 256 - 4 and "do not fit" in p.stderr


@pytest.mark.parametrize("kw", [{"min_blocks": -1}, {"min_blocks": 5}, {"ssa_steps": 0}, {"sched": 3},
                                {"sched": -1}, {"warp_sims": 33}, {"warp_sims": -2},
                                {"spec": 2}, {"spec": -2}])
def test_run_cfg_rejected_before_any_device_work(kw):
    """Invalid run configurations fail with CTL_ERR_ARG in host code, before
    the library selects or touches a device."""
    net = inputs.schlogl(4, samples=5, t_end=0.1)
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    with pytest.raises(ctl.CtlError) as e:
        m.run(net.X0, net.c, **kw)
    assert e.value.status == ctl.ERR_ARG


@pytest.mark.parametrize("with_cs", [True, False])
def test_binary_samples_roundtrip(tmp_path, with_cs):
    """ctl_write_samples_binary: header (instants, sampled species, first id),
    16-byte aligned payload identical to the samples given, and the reader's
    checks on foreign or truncated files."""
    net = inputs.schlogl(5, samples=9, t_end=1.0)
    cs = net.cs if with_cs else None
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, cs)
    so = m.s_out
    rng = np.random.default_rng(1)
    samples = rng.integers(0, 2**32 - 1, size=(5, 9, so), dtype=np.uint64).astype(np.uint32)
    path = str(tmp_path / "batch.ctlbin")
    m.write_samples_binary(path, samples, first_id=40)
    d = ctl.read_samples_binary(path)
    assert d["first_id"] == 40
    assert np.array_equal(d["t"], np.asarray(net.tvec, np.float64))
    assert np.array_equal(d["species"], np.asarray(cs if with_cs else np.arange(so), np.uint32))
    assert np.array_equal(np.asarray(d["samples"]), samples)
    raw = open(path, "rb").read()
    off = (24 + 8 * 9 + 4 * so + 15) // 16 * 16
    assert len(raw) == off + samples.nbytes and raw[off:] == samples.tobytes()
    assert ctl.read_samples_binary(path, mmap=False)["samples"].tolist() == samples.tolist()
    open(tmp_path / "short", "wb").write(raw[:-4])
    with pytest.raises(ValueError):
        ctl.read_samples_binary(str(tmp_path / "short"))
    open(tmp_path / "text", "wb").write(b"0.1\t5\n" * 10)
    with pytest.raises(ValueError):
        ctl.read_samples_binary(str(tmp_path / "text"))
    with pytest.raises(ctl.CtlError):
        m.write_samples_binary(str(tmp_path / "no_such_dir" / "x"), samples)
    empty = np.zeros((0, 9, so), np.uint32)
    m.write_samples_binary(str(tmp_path / "empty.ctlbin"), empty)
    e = ctl.read_samples_binary(str(tmp_path / "empty.ctlbin"))
    assert e["samples"].shape == (0, 9, so) and np.array_equal(e["t"], d["t"])


def test_bench_io_timing_reports_both_writers():
    import bench
    net = inputs.schlogl(6, samples=5, t_end=1.0)
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    samples = np.arange(6 * 5 * m.s_out, dtype=np.uint32).reshape(6, 5, m.s_out)
    io = bench.io_timing(m, samples, threads=2)
    assert io["sample_sims"] == 6 and io["threads"] == 2
    assert io["text_s_per_sim"] > 0 and io["binary_s_per_sim"] > 0
    assert io["binary_bytes_per_sim"] > 5 * m.s_out * 4 - 1
    assert io["text_bytes_per_sim"] > 0


def _bench(*args, env_extra=None):
    env = dict(os.environ, **(env_extra or {}))
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True,
                          text=True, env=env, timeout=600, cwd=ROOT)


def test_bench_reference_arm_line():
    """`bench.py --impl reference` times the CPU restatement on the host
    cores and prints one JSON line in the contract's shape; under torchrun
    only rank 0 works and prints."""
    import json
    p = _bench("--impl", "reference", "--config", "1", "--steps", "1", "--warmup", "0")
    assert p.returncode == 0, p.stderr
    lines = [x for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "sims/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["e2e"] == {"value": d["value"], "unit": "sims/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    p1 = _bench("--impl", "reference", "--config", "1", "--steps", "1", "--warmup", "0",
                env_extra={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p1.returncode == 0 and not [x for x in p1.stdout.splitlines() if x.startswith("{")]


def test_run_report_json(tmp_path):
    """ctl_write_run_report: rates, sums, per-status counts and launch shape
    as one JSON object (host code; records made up here)."""
    import json
    net = inputs.schlogl(4, samples=10, t_end=1.0)
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    info = np.zeros(4, dtype=ctl.INFO_DTYPE)
    info["firings"] = [10, 20, 30, 40]
    info["steps"] = [5, 6, 7, 8]
    info["leaps"] = [1, 2, 3, 4]
    info["ssa_steps"] = [4, 4, 4, 4]
    info["rejections"] = [0, 1, 0, 1]
    info["status"] = [ctl.SIM_OK, ctl.SIM_OK, ctl.SIM_STEP_LIMIT, 7]
    li = ctl.LaunchInfo()
    li.group, li.threads, li.blocks, li.min_blocks, li.sched, li.ssa_budget, li.dec_budget = 4, 96, 2, 2, 1, 8, 1
    path = str(tmp_path / "report.json")
    m.write_run_report(path, info, 0.5, li)
    r = json.load(open(path))
    assert r["simulations"] == 4 and r["seconds"] == 0.5 and r["sims_per_s"] == 8.0
    assert r["firings"] == 100 and r["firings_per_s"] == 200.0
    assert (r["steps"], r["leaps"], r["ssa_steps"], r["rejections"]) == (26, 10, 16, 2)
    assert r["status"] == {"ok": 2, "step_limit": 1, "overflow": 0, "attempt_limit": 0, "other": 1}
    assert r["hbm_bytes_per_sim"] == 4 * m.S + 4 * m.R + 4 * m.ns * m.s_out + 40
    assert r["launch"] == {"group": 4, "threads": 96, "blocks": 2, "min_blocks": 2, "sched": 1,
                           "ssa_budget": 8, "dec_budget": 1}
    m.write_run_report(str(tmp_path / "nolaunch.json"), info, 2.0)
    assert "launch" not in json.load(open(tmp_path / "nolaunch.json"))
    with pytest.raises(ctl.CtlError):
        m.write_run_report(str(tmp_path / "bad.json"), info, 0.0)


@pytest.mark.parametrize("bad", ["nan_rate", "inf_rate", "negative_rate", "negative_count"])
def test_host_rows_rejected_before_device_work(bad):
    """ctl_run refuses rows that would make a simulation run to its step cap
    (non-finite rates) or that are not counts, before touching a device."""
    net = inputs.schlogl(4, samples=5, t_end=1.0)
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    X0 = np.array(net.X0, np.int32)
    c = np.array(net.c, np.float32)
    if bad == "nan_rate":
        c[2, 1] = np.nan
    elif bad == "inf_rate":
        c[3, 0] = np.inf
    elif bad == "negative_rate":
        c[1, 3] = -1e-3
    else:
        X0[2, 0] = -5
    with pytest.raises(ctl.CtlError) as e:
        m.run(X0, c, seed=1)
    assert e.value.status == ctl.ERR_ARG and ("c:" in str(e.value) or "X0:" in str(e.value))


def test_model_instants_must_be_finite_and_non_negative():
    left, right = np.array([[1, 0]], np.int32), np.array([[0, 1]], np.int32)
    for tv in ([0.5, np.nan], [0.5, np.inf], [-1.0, 0.5]):
        with pytest.raises(ctl.CtlError) as e:
            ctl.Model.create(left, right, None, np.array(tv))
        assert e.value.status == ctl.ERR_SHAPE
    ctl.Model.create(left, right, None, np.array([0.0, 0.5, 0.2]))  # zero and unsorted instants stay valid
