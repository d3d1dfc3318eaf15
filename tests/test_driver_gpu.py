"""The harness driver (weno_standalone_b200, the B200 counterpart of the
reference's weno_test_driver, f90:1734-1861) run end to end on the GPU.

* the golden workflow: `wenoss test` (wenoss.sh:351-387 -- pinned
  environment, `  Checksum [XYZT] :` lines, rtol 1e-10, NaN fails) against
  every committed golden under tests/golden/driver/ (FP64 goldens made by the
  oracle, FP32-bulk goldens by the driver itself);
* the reference's own golden (tests/golden/weno5.txt of the reference) with
  the namelist file missing altogether, so the defaults of f90:120-124 apply;
* WENO_KERNEL_MODE values other than weno5 run every family (f90:1805-1808);
* WENO5_BENCH_SCOPE=kernel prepares the inputs once and repeats only the
  reconstruction (f90:1795-1799, 1814-1817).
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "driver")
NML = os.path.join(ROOT, "wenostandalone_b200", "inputs")


@pytest.fixture(scope="module")
def driver():
    from wenostandalone_b200 import build
    build.build_lib()
    return build.build_driver()


def _wenoss(args, env_over):
    env = dict(os.environ)
    env.update(env_over)
    return subprocess.run([sys.executable, "-m", "wenostandalone_b200.wenoss", *args], env=env,
                          capture_output=True, text=True, cwd=ROOT)


CASES = [  # (golden, kernel mode, precision, namelist)
    ("weno5", "weno5", "fp64", "weno_input.nml"),
    ("all", "all", "fp64", "weno_input.nml"),
    ("weno5_teno", "weno5", "fp64", "weno_input_teno.nml"),
    ("weno5_fp32", "weno5", "fp32", "weno_input.nml"),
    ("all_fp32", "all", "fp32", "weno_input.nml"),
]


@pytest.mark.parametrize("golden,mode,precision,nml", CASES)
def test_wenoss_test_against_committed_golden(driver, golden, mode, precision, nml):
    if not os.path.exists(os.path.join(GOLDEN, golden + ".txt")):
        pytest.skip(f"no golden {golden}.txt")
    p = _wenoss(["test"], {"WENO_TEST_KERNEL_MODE": mode, "WENO_TEST_PRECISION": precision,
                           "INPUT_NML": os.path.join(NML, nml), "TEST_GOLDEN_DIR": GOLDEN})
    print(p.stdout)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "test passed" in p.stderr


def _run(driver, nml_path, cwd, **env):
    e = dict(os.environ, WENO_WARMUP_ITERS="0", WENO_BENCH_ITERS="1")
    e.update({k: str(v) for k, v in env.items()})
    p = subprocess.run([driver, str(nml_path)], env=e, capture_output=True, text=True, cwd=cwd)
    assert p.returncode == 0, p.stdout + p.stderr
    from wenostandalone_b200 import wenoss
    return p.stdout, wenoss.extract_checksums(p.stdout)


def test_missing_namelist_runs_the_defaults_to_the_reference_golden(driver, tmp_path):
    import test_oracle_golden as tg
    exp = tg.reference_checksums()["weno5_full"]
    out, chk = _run(driver, tmp_path / "no_such_file.nml", tmp_path, WENO_KERNEL_MODE="weno5")
    assert "not found; using defaults." in out
    for k in "XYZT":
        assert abs(chk[k] - exp[k]) <= 1e-10 * exp[k], (k, chk[k], exp[k])
    assert "All kernel families executed with finite non-zero output." in out


def _small_nml(tmp_path, m=47, nv=4, wenojs="T"):
    p = tmp_path / "small.nml"
    p.write_text(f"&grid_params\n m_cells = {m}, n_cells = {m}, p_cells = {m}, v_size = {nv},\n"
                 f" buff_size = 6, weno_eps = 1e-16, wenojs = {wenojs}, teno_CT = 1e-5\n/\n")
    return p


@pytest.mark.parametrize("mode", ["weno3", "all", "anything"])
def test_modes_other_than_weno5_run_every_family(driver, oracle_mod, tmp_path, mode):
    exp = oracle_mod.harness_run(47, 47, 47, 4, 6, all_mode=True)
    out, chk = _run(driver, _small_nml(tmp_path), tmp_path, WENO_KERNEL_MODE=mode, WENO_WARMUP_ITERS=1)
    assert f"Kernel mode              : {mode}" in out
    for k, e in zip("XYZ", exp):
        assert abs(chk[k] - e) <= 1e-10 * e, (mode, k, chk[k], e)   # the printed 11 digits


@pytest.mark.parametrize("split,specialized", [(0, 0), (1, 0), (0, 1)])
def test_kernel_scope_repeats_only_the_reconstruction(driver, oracle_mod, tmp_path, split, specialized):
    exp = oracle_mod.harness_run(47, 47, 47, 4, 6, all_mode=False)
    out, chk = _run(driver, _small_nml(tmp_path), tmp_path, WENO_KERNEL_MODE="weno5",
                    WENO5_BENCH_SCOPE="kernel", WENO_WARMUP_ITERS=2, WENO_BENCH_ITERS=3,
                    WENO5_SPLIT_KERNELS=split, WENO5_SPECIALIZED_COMBINED=specialized)
    assert "WENO5 benchmark scope    : kernel" in out
    for k, e in zip("XYZ", exp):
        assert abs(chk[k] - e) <= 1e-10 * e, (k, chk[k], e)   # the printed 11 digits


def test_all_mode_with_teno_reports_non_finite_output(driver, tmp_path):
    """wenojs = F in all mode: WENO3 has no TENO branch, so its faces outside
    the WENO5/7 core stay NaN, and the driver says so (f90:1841-1842)."""
    out, chk = _run(driver, _small_nml(tmp_path, m=15, nv=2, wenojs="F"), tmp_path, WENO_KERNEL_MODE="all")
    assert chk["T"] != chk["T"]
    assert "WARNING: non-finite values detected in standalone output." in out
