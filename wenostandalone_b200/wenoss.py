"""Build, run, golden-test and sweep the B200 WENO harness driver.

    python -m wenostandalone_b200.wenoss build|run|test|test-update|sweep|help

The command-line front end of the harness driver ``weno_standalone_b200``
(``csrc/weno_driver.cpp``), with the subcommands, environment variables and
defaults of the reference's ``wenoss.sh`` (wilfonba/WenoStandalone) for the
parts that concern the WENO path:

* ``run`` / ``benchmark`` (wenoss.sh:209-213): the driver on ``INPUT_NML`` with
  the run environment (``WENO_KERNEL_MODE`` default ``weno5``,
  ``WENO5_BENCH_SCOPE`` ``full``, ``WENO5_SPLIT_KERNELS`` /
  ``WENO5_SPECIALIZED_COMBINED`` ``0``, ``WENO_WARMUP_ITERS`` 5,
  ``WENO_BENCH_ITERS`` 10; wenoss.sh:143-148).
* ``test`` / ``check`` (wenoss.sh:351-387): a pinned run (scope full, split 0,
  specialised 0, ``WENO_TEST_WARMUP_ITERS`` 0, ``WENO_TEST_BENCH_ITERS`` 1,
  mode ``WENO_TEST_KERNEL_MODE``), its ``  Checksum [XYZT] :`` lines compared
  with the golden file at ``WENO_TEST_RTOL`` (1e-10); a NaN fails.
* ``test-update`` (wenoss.sh:389-414): the same pinned run written as the
  golden, refused when ``Checksum T`` is missing, non-finite or zero.
* ``sweep``: the driver over a list of variants, one CSV row each with the
  columns of the reference's variant sweep (toolchain/optimize_amdflang.sh:70-108:
  ``variant,binary,compile_status,run_status,checksum_total,
  kernel_time_total_s,kernel_time_per_iter_s,flags``), and the fastest
  variant named.  The reference's variants are compiler flags; here they
  are the driver's run-time switches (kernel mode, precision, fused MP,
  folded reshape, split / specialised WENO5).

Goldens are kept per kernel mode, precision and weight family: the file is
``<TEST_GOLDEN_DIR>/<mode>[_fp32][_teno].txt`` (``weno5.txt`` is the
reference's own name for its FP64 JS golden); ``_fp32`` comes from
``WENO_TEST_PRECISION=fp32`` and ``_teno`` from ``wenojs = F`` in the
namelist.  The AMD profiler, CMake and module-loading subcommands of
wenoss.sh have no counterpart on this hardware.
"""
from __future__ import annotations

import csv
import math
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
DEFAULT_BIN = os.path.join(HERE, "weno_standalone_b200")
DEFAULT_NML = os.path.join(HERE, "inputs", "weno_input.nml")

CHECK_RE = re.compile(r"^  Checksum ([XYZT]) :\s*(\S+)", re.M)


def _env(name: str, default: str) -> str:
    v = os.environ.get(name)
    return default if v is None or v == "" else v


def settings() -> dict:
    """The knobs of wenoss.sh:140-155 (environment, with its defaults)."""
    return {
        "BIN": _env("WENOSS_BIN", DEFAULT_BIN),
        "INPUT_NML": _env("INPUT_NML", DEFAULT_NML),
        "WENO_KERNEL_MODE": _env("WENO_KERNEL_MODE", "weno5"),
        "WENO5_BENCH_SCOPE": _env("WENO5_BENCH_SCOPE", "full"),
        "WENO5_SPLIT_KERNELS": _env("WENO5_SPLIT_KERNELS", "0"),
        "WENO5_SPECIALIZED_COMBINED": _env("WENO5_SPECIALIZED_COMBINED", "0"),
        "WENO_WARMUP_ITERS": _env("WENO_WARMUP_ITERS", "5"),
        "WENO_BENCH_ITERS": _env("WENO_BENCH_ITERS", "10"),
        "TEST_GOLDEN_DIR": _env("TEST_GOLDEN_DIR", os.path.join(ROOT, "tests", "golden", "driver")),
        "WENO_TEST_RTOL": float(_env("WENO_TEST_RTOL", "1e-10")),
        "WENO_TEST_KERNEL_MODE": _env("WENO_TEST_KERNEL_MODE", "weno5"),
        "WENO_TEST_WARMUP_ITERS": _env("WENO_TEST_WARMUP_ITERS", "0"),
        "WENO_TEST_BENCH_ITERS": _env("WENO_TEST_BENCH_ITERS", "1"),
        "WENO_TEST_PRECISION": _env("WENO_TEST_PRECISION", "fp64").lower(),
        "RESULT_CSV": _env("RESULT_CSV", os.path.join(os.getcwd(), "results", "weno_variants.csv")),
    }


# extensions of the B200 driver passed through to every run when set
PASS_THROUGH = ("WENO_PRECISION", "WENO_TENO", "WENO5_FUSED_MP", "WENO5_FOLDED", "CUDA_VISIBLE_DEVICES")


def log(msg: str) -> None:
    print(f">> {msg}", file=sys.stderr, flush=True)


def namelist_wenojs(path: str) -> bool:
    """wenojs of the &grid_params group (True when absent, the default)."""
    try:
        txt = open(path).read()
    except OSError:
        return True
    txt = re.sub(r"!.*", "", txt)
    m = re.search(r"\bwenojs\s*=\s*\.?\s*([tTfF])", txt)
    return True if m is None else m.group(1).lower() == "t"


def golden_file(s: dict) -> str:
    name = s["WENO_TEST_KERNEL_MODE"]
    if s["WENO_TEST_PRECISION"] == "fp32":
        name += "_fp32"
    if not namelist_wenojs(s["INPUT_NML"]):
        name += "_teno"
    return os.path.join(s["TEST_GOLDEN_DIR"], name + ".txt")


def extract_checksums(text: str) -> dict:
    """The wenoss.sh:347-349 rule: '<label> <value>' from '  Checksum X : v'."""
    out = {}
    for lab, val in CHECK_RE.findall(text):
        try:
            out[lab] = float(val)
        except ValueError:
            out[lab] = float("nan")
    return out


def extract_metric(text: str, key: str) -> str:
    """Value of the last '<key> : <value> s' line (optimize_amdflang.sh:60-63)."""
    val = ""
    for line in text.splitlines():
        if ":" in line and key in line.split(":", 1)[0]:
            val = line.split(":", 1)[1].strip()
            if val.endswith(" s"):
                val = val[:-2].strip()
    return val


def read_golden(path: str) -> dict:
    with open(path) as f:
        return {k: float(v) for k, v in (line.split() for line in f if line.strip())}


def compare(actual: dict, expected: dict, rtol: float) -> bool:
    """wenoss.sh:364-383: per label rel = |a - e| / max(|e|, 1e-300); fail
    past rtol or on NaN.  Prints one line per label; True when all pass."""
    ok = True
    for key in ("X", "Y", "Z", "T"):
        a = actual.get(key, float("nan"))
        e = expected.get(key, float("nan"))
        rel = abs(a - e) / max(abs(e), 1e-300)
        good = rel <= rtol and a == a
        print(f"  {key}  expected={e: .10e}  actual={a: .10e}  rel_err={rel:.3e}  {'OK  ' if good else 'FAIL'}")
        ok = ok and good
    return ok


def _run(s: dict, env_over: dict) -> subprocess.CompletedProcess:
    env = dict(os.environ)
    env.update({k: str(v) for k, v in env_over.items()})
    binary = s["BIN"]
    cmd = [sys.executable, binary] if binary.endswith(".py") else [binary]
    return subprocess.run(cmd + [s["INPUT_NML"]], env=env, capture_output=True, text=True)


def run_env(s: dict) -> dict:
    env = {k: s[k] for k in ("WENO_KERNEL_MODE", "WENO5_BENCH_SCOPE", "WENO5_SPLIT_KERNELS",
                             "WENO5_SPECIALIZED_COMBINED", "WENO_WARMUP_ITERS", "WENO_BENCH_ITERS")}
    for k in PASS_THROUGH:
        if os.environ.get(k):
            env[k] = os.environ[k]
    return env


def pinned_env(s: dict) -> dict:
    """wenoss.sh:331-345: the test's pinned run."""
    env = {"WENO_KERNEL_MODE": s["WENO_TEST_KERNEL_MODE"], "WENO5_BENCH_SCOPE": "full",
           "WENO5_SPLIT_KERNELS": "0", "WENO5_SPECIALIZED_COMBINED": "0",
           "WENO_WARMUP_ITERS": s["WENO_TEST_WARMUP_ITERS"], "WENO_BENCH_ITERS": s["WENO_TEST_BENCH_ITERS"],
           "WENO_PRECISION": s["WENO_TEST_PRECISION"], "WENO5_FUSED_MP": "0", "WENO5_FOLDED": "0"}
    for k in ("WENO_TENO", "CUDA_VISIBLE_DEVICES"):
        if os.environ.get(k):
            env[k] = os.environ[k]
    return env


def cmd_build(s: dict) -> int:
    from wenostandalone_b200 import build
    build.build(verbose=True)
    return 0


def cmd_run(s: dict) -> int:
    log(f"running {s['BIN']}")
    p = _run(s, run_env(s))
    sys.stdout.write(p.stdout)
    sys.stderr.write(p.stderr)
    return p.returncode


def _pinned_output(s: dict):
    log(f"running test: kernel_mode={s['WENO_TEST_KERNEL_MODE']} precision={s['WENO_TEST_PRECISION']} "
        f"warmup={s['WENO_TEST_WARMUP_ITERS']} bench={s['WENO_TEST_BENCH_ITERS']}")
    p = _run(s, pinned_env(s))
    if p.returncode != 0:
        sys.stderr.write(p.stdout + p.stderr)
        log(f"driver exited with status {p.returncode}")
    return p


def cmd_test(s: dict) -> int:
    golden = golden_file(s)
    if not os.path.isfile(golden):
        log(f"golden file not found: {golden}. Generate with: python -m wenostandalone_b200.wenoss test-update")
        return 1
    p = _pinned_output(s)
    actual = extract_checksums(p.stdout)
    log(f"comparing against {golden} (rtol={s['WENO_TEST_RTOL']})")
    if not compare(actual, read_golden(golden), s["WENO_TEST_RTOL"]) or p.returncode != 0:
        log("test FAILED")
        return 1
    log("test passed")
    return 0


def cmd_test_update(s: dict) -> int:
    golden = golden_file(s)
    p = _pinned_output(s)
    if p.returncode != 0:
        return 1
    chk = extract_checksums(p.stdout)
    if "T" not in chk:
        log("no 'Checksum T' line in binary output -- did the run succeed?")
        return 1
    t = chk["T"]
    if not math.isfinite(t) or t == 0.0:
        log(f"refusing to write golden: Checksum T = {t!r}")
        return 1
    os.makedirs(os.path.dirname(golden) or ".", exist_ok=True)
    with open(golden, "w") as f:
        for lab, val in CHECK_RE.findall(p.stdout):
            f.write(f"{lab} {val}\n")
    log(f"wrote golden: {golden}")
    sys.stdout.write(open(golden).read())
    return 0


# The run-time variants of the sweep (name -> environment overrides).
VARIANTS = [
    ("weno5_fp64", {}),
    ("weno5_fp64_split", {"WENO5_SPLIT_KERNELS": "1"}),
    ("weno5_fp64_specialized", {"WENO5_SPECIALIZED_COMBINED": "1"}),
    ("weno5_fp64_fused_mp", {"WENO5_FUSED_MP": "1"}),
    ("weno5_fp64_fused_mp_folded", {"WENO5_FUSED_MP": "1", "WENO5_FOLDED": "1"}),
    ("weno5_fp32", {"WENO_PRECISION": "fp32"}),
    ("weno5_fp32_fused_mp", {"WENO_PRECISION": "fp32", "WENO5_FUSED_MP": "1"}),
    ("all_fp64", {"WENO_KERNEL_MODE": "all"}),
    ("all_fp32", {"WENO_KERNEL_MODE": "all", "WENO_PRECISION": "fp32"}),
]


def cmd_sweep(s: dict) -> int:
    """One driver run per variant, a CSV row each (RESULT_CSV)."""
    compile_status = "ok"
    if not os.environ.get("WENOSS_BIN"):
        try:
            cmd_build(s)
        except Exception as e:  # the build's own output already explains it
            log(f"build failed: {e}")
            compile_status = "fail"
    out = s["RESULT_CSV"]
    os.makedirs(os.path.dirname(out) or ".", exist_ok=True)
    best, best_t = "", None
    only = [v for v in os.environ.get("WENOSS_VARIANTS", "").split(",") if v]
    with open(out, "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(["variant", "binary", "compile_status", "run_status", "checksum_total",
                    "kernel_time_total_s", "kernel_time_per_iter_s", "flags"])
        for name, over in VARIANTS:
            if only and name not in only:
                continue
            flags = " ".join(f"{k}={v}" for k, v in over.items())
            if compile_status != "ok":
                w.writerow([name, s["BIN"], compile_status, "not-run", "", "", "", flags])
                continue
            log(f"running {name}")
            env = run_env(s)
            env.update(over)
            p = _run(s, env)
            status = "ok" if p.returncode == 0 else "fail"
            chk = extract_checksums(p.stdout).get("T")
            tot = extract_metric(p.stdout, "Kernel time total")
            per = extract_metric(p.stdout, "Kernel time per iter")
            w.writerow([name, s["BIN"], compile_status, status, "" if chk is None else f"{chk:.10E}", tot, per,
                        flags])
            if status == "ok" and per:
                t = float(per)
                if best_t is None or t < best_t:
                    best, best_t = name, t
    log(f"wrote {out}")
    if best:
        log(f"fastest variant: {best} ({best_t:.6f} s per iteration)")
    return 0


def cmd_help(s: dict) -> int:
    print(__doc__)
    return 0


COMMANDS = {"build": cmd_build, "run": cmd_run, "benchmark": cmd_run, "test": cmd_test, "check": cmd_test,
            "test-update": cmd_test_update, "sweep": cmd_sweep, "help": cmd_help, "-h": cmd_help,
            "--help": cmd_help}


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    sub = argv[0] if argv else "help"
    fn = COMMANDS.get(sub)
    if fn is None:
        log(f"unknown subcommand: {sub}. Try 'help'.")
        return 1
    return fn(settings())


if __name__ == "__main__":
    sys.exit(main())
