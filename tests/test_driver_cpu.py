"""The harness driver's host side and the wenoss golden workflow.  CPU only.

* the driver binary's namelist handling (s_read_input, f90:111-144): run with
  no visible GPU it prints what it read and stops at the first device call;
* the wenoss test / test-update / sweep logic (wenoss.sh:330-414 and
  toolchain/optimize_amdflang.sh:70-108) against a stand-in driver that
  prints chosen checksum lines;
* the committed driver goldens: the oracle-made weno5.txt against the
  reference's published golden, and the FP32-bulk goldens against the FP64
  ones.
"""
import csv
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "driver")


@pytest.fixture(scope="module")
def driver():
    from wenostandalone_b200 import build
    build.build_lib()
    return build.build_driver()


def _run_driver(driver, nml, tmp_path, extra_env=None):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", WENO_WARMUP_ITERS="0", WENO_BENCH_ITERS="1")
    env.update(extra_env or {})
    return subprocess.run([driver, str(nml)], env=env, capture_output=True, text=True, cwd=tmp_path)


def _from_input(out):
    vals = {}
    for line in out.splitlines():
        if "(from input)" in line:
            key = line.split("(")[0].strip()
            vals[key] = int(line.split(":")[1])
    return vals


def test_driver_missing_namelist_keeps_defaults(driver, tmp_path):
    p = _run_driver(driver, tmp_path / "absent.nml", tmp_path)
    assert 'Input file "' in p.stdout and 'not found; using defaults.' in p.stdout
    # f90:121-124 returns before echoing the values (the defaults stay)
    assert _from_input(p.stdout) == {}
    # no GPU visible: the first device call fails loudly, with status 2
    assert p.returncode == 2 and "ERROR" in p.stderr


def test_driver_reads_the_namelist(driver, tmp_path):
    nml = tmp_path / "g.nml"
    nml.write_text("&GRID_PARAMS\n  m_cells = 31, n_cells=17 ! comment\n  p_cells = 9, v_size = 3,\n"
                   "  buff_size = 6, weno_eps = 1d-16, wenojs = .false., teno_CT = 2.5e-5 /\n")
    p = _run_driver(driver, nml, tmp_path)
    assert "WARNING" not in p.stdout
    assert _from_input(p.stdout) == {"m_cells": 31, "n_cells": 17, "p_cells": 9, "v_size": 3}


@pytest.mark.parametrize("body", [
    "&grid_params\n  m_cells = 31, n_cells = x /\n",         # unreadable value
    "&grid_params\n  m_cells = 31, unknown_key = 3 /\n",     # unknown key
    "&other_group\n  m_cells = 31 /\n",                      # no grid_params group
])
def test_driver_bad_namelist_warns_and_keeps_defaults(driver, tmp_path, body):
    nml = tmp_path / "bad.nml"
    nml.write_text(body)
    p = _run_driver(driver, nml, tmp_path)
    assert "WARNING: error reading namelist grid_params; using defaults." in p.stdout
    assert _from_input(p.stdout)["m_cells"] == 199


def test_driver_echoes_the_switches(driver, tmp_path):
    p = _run_driver(driver, tmp_path / "absent.nml", tmp_path,
                    {"WENO_KERNEL_MODE": "weno3", "WENO5_BENCH_SCOPE": "kernel", "WENO5_SPLIT_KERNELS": "1",
                     "WENO_WARMUP_ITERS": "-4", "WENO_BENCH_ITERS": "junk"})
    out = p.stdout
    assert "Kernel mode              : weno3" in out
    assert "WENO5 benchmark scope    : kernel" in out
    assert "WENO5 split kernels      : T" in out
    # f90:1757-1758: max(0, warmup), max(1, bench); unparsable -> default 5
    assert "Warmup iterations        : 0" in out
    assert "Benchmark iterations     : 5" in out


# ---------------------------------------------------------------------------
# wenoss workflow with a stand-in driver
# ---------------------------------------------------------------------------
FAKE = r'''
import os, sys
t = os.environ.get("FAKE_T", "1.5000000000E+00")
print("  Kernel mode              : " + os.environ.get("WENO_KERNEL_MODE", "?"))
print("  Precision seen           : " + os.environ.get("WENO_PRECISION", "?"))
if os.environ.get("FAKE_NO_T") != "1":
    print("  Checksum X :   5.0000000000E-01")
    print("  Checksum Y :   5.0000000000E-01")
    print("  Checksum Z :   5.0000000000E-01")
    print("  Checksum T : " + t)
per = {"1": "0.200000", "fp32": "0.100000"}.get(os.environ.get("WENO5_FUSED_MP", ""), "0.300000")
if os.environ.get("WENO_PRECISION") == "fp32":
    per = "0.050000"
print("  Kernel time total        :     1.000000 s")
print("  Kernel time per iter     :     " + per + " s")
sys.exit(int(os.environ.get("FAKE_RC", "0")))
'''


@pytest.fixture
def fake(tmp_path, monkeypatch):
    p = tmp_path / "fake_driver.py"
    p.write_text(FAKE)
    monkeypatch.setenv("WENOSS_BIN", str(p))
    monkeypatch.setenv("TEST_GOLDEN_DIR", str(tmp_path / "golden"))
    monkeypatch.setenv("INPUT_NML", str(tmp_path / "in.nml"))
    (tmp_path / "in.nml").write_text("&grid_params\n wenojs = T /\n")
    for k in ("WENO_TEST_PRECISION", "WENO_TEST_KERNEL_MODE", "FAKE_T", "FAKE_NO_T", "FAKE_RC"):
        monkeypatch.delenv(k, raising=False)
    return tmp_path


def test_wenoss_update_then_test(fake, monkeypatch, capsys):
    from wenostandalone_b200 import wenoss
    assert wenoss.main(["test"]) == 1                      # no golden yet
    assert wenoss.main(["test-update"]) == 0
    g = (fake / "golden" / "weno5.txt").read_text().split()
    assert g == ["X", "5.0000000000E-01", "Y", "5.0000000000E-01", "Z", "5.0000000000E-01",
                 "T", "1.5000000000E+00"]
    assert wenoss.main(["test"]) == 0
    monkeypatch.setenv("FAKE_T", "1.5000000002E+00")          # 1.3e-10 > rtol 1e-10
    assert wenoss.main(["check"]) == 1
    monkeypatch.setenv("WENO_TEST_RTOL", "1e-9")
    assert wenoss.main(["check"]) == 0
    monkeypatch.setenv("FAKE_T", "NaN")
    assert wenoss.main(["test"]) == 1                      # NaN fails whatever the rtol
    out = capsys.readouterr().out
    assert "FAIL" in out and "OK" in out


@pytest.mark.parametrize("t", ["NaN", "Infinity", "0.0000000000E+00"])
def test_wenoss_update_refuses_bad_totals(fake, monkeypatch, t):
    from wenostandalone_b200 import wenoss
    monkeypatch.setenv("FAKE_T", t)
    assert wenoss.main(["test-update"]) == 1
    assert not (fake / "golden" / "weno5.txt").exists()


def test_wenoss_update_refuses_missing_total_and_failed_runs(fake, monkeypatch):
    from wenostandalone_b200 import wenoss
    monkeypatch.setenv("FAKE_NO_T", "1")
    assert wenoss.main(["test-update"]) == 1
    monkeypatch.delenv("FAKE_NO_T")
    monkeypatch.setenv("FAKE_RC", "2")
    assert wenoss.main(["test-update"]) == 1
    assert not (fake / "golden" / "weno5.txt").exists()


def test_wenoss_golden_names(fake, monkeypatch):
    from wenostandalone_b200 import wenoss
    s = wenoss.settings()
    assert os.path.basename(wenoss.golden_file(s)) == "weno5.txt"
    monkeypatch.setenv("WENO_TEST_PRECISION", "fp32")
    monkeypatch.setenv("WENO_TEST_KERNEL_MODE", "all")
    (fake / "in.nml").write_text("&grid_params\n m_cells = 9, wenojs = .false. ! TENO\n/\n")
    assert os.path.basename(wenoss.golden_file(wenoss.settings())) == "all_fp32_teno.txt"
    # the pinned run passes the precision and pins the extensions off
    env = wenoss.pinned_env(wenoss.settings())
    assert env["WENO_PRECISION"] == "fp32" and env["WENO5_FUSED_MP"] == "0" and env["WENO5_BENCH_SCOPE"] == "full"
    assert env["WENO_WARMUP_ITERS"] == "0" and env["WENO_BENCH_ITERS"] == "1"


def test_wenoss_sweep_csv(fake, monkeypatch):
    from wenostandalone_b200 import wenoss
    out = fake / "res" / "v.csv"
    monkeypatch.setenv("RESULT_CSV", str(out))
    monkeypatch.setenv("WENOSS_VARIANTS", "weno5_fp64,weno5_fp64_fused_mp,weno5_fp32")
    assert wenoss.main(["sweep"]) == 0
    rows = list(csv.reader(out.open()))
    assert rows[0] == ["variant", "binary", "compile_status", "run_status", "checksum_total",
                       "kernel_time_total_s", "kernel_time_per_iter_s", "flags"]
    by = {r[0]: r for r in rows[1:]}
    assert set(by) == {"weno5_fp64", "weno5_fp64_fused_mp", "weno5_fp32"}
    assert by["weno5_fp32"][3] == "ok" and by["weno5_fp32"][6] == "0.050000"
    assert by["weno5_fp64_fused_mp"][7] == "WENO5_FUSED_MP=1"
    assert float(by["weno5_fp64"][4]) == 1.5


# ---------------------------------------------------------------------------
# committed goldens
# ---------------------------------------------------------------------------
def test_oracle_made_golden_is_the_reference_golden():
    import test_oracle_golden as tg
    from wenostandalone_b200 import wenoss
    exp = tg.reference_checksums()["weno5_full"]
    got = wenoss.read_golden(os.path.join(GOLDEN, "weno5.txt"))
    for k in "XYZT":
        assert abs(got[k] - exp[k]) <= 1e-10 * exp[k], (k, got[k], exp[k])


@pytest.mark.parametrize("mode", ["weno5", "all"])
def test_fp32_goldens_are_near_the_fp64_goldens(mode):
    from wenostandalone_b200 import wenoss
    p32 = os.path.join(GOLDEN, f"{mode}_fp32.txt")
    if not os.path.exists(p32):
        pytest.skip(f"{p32} not generated yet")
    g32 = wenoss.read_golden(p32)
    g64 = wenoss.read_golden(os.path.join(GOLDEN, f"{mode}.txt"))
    for k in "XYZT":
        assert abs(g32[k] - g64[k]) <= 1e-6 * g64[k], (k, g32[k], g64[k])
