"""Generate the driver goldens under tests/golden/driver/ (test infrastructure).

    python tests/golden/make_driver_goldens.py           # FP64 goldens from the oracle

FP64 goldens come from the CPU oracle's harness run (oracle/weno_oracle.c
wo_harness_run, the restatement of inputs/weno_standalone.f90:1734-1861 with
the harness field and coefficients of f90:221-279) at the driver's namelist
(wenostandalone_b200/inputs/weno_input.nml, 200^3 cells x 8 variables):

    weno5.txt        WENO_KERNEL_MODE=weno5, wenojs = T  (the reference's own
                     golden case, tests/golden/weno5.txt of the reference;
                     test_driver_cpu checks the two agree to 1e-10)
    all.txt          WENO_KERNEL_MODE=all (reshape, copy, WENO3/5/7, MP)
    weno5_teno.txt   WENO_KERNEL_MODE=weno5, wenojs = F (TENO, CT = 1e-5)

(all-mode with wenojs = F has no golden: WENO3 has no TENO branch, so its
faces outside the WENO5/7 core stay NaN, as in the reference, and
test-update refuses a non-finite Checksum T.)

FP32-bulk goldens (weno5_fp32.txt, all_fp32.txt) have no CPU oracle: they are
written by the driver itself on a B200 with the golden workflow,

    WENO_TEST_PRECISION=fp32 WENO_TEST_KERNEL_MODE=weno5 \\
        python -m wenostandalone_b200.wenoss test-update

(and WENO_TEST_KERNEL_MODE=all), then copied here; test_driver_cpu checks
that they lie within FP32-storage error of the FP64 ones.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402

CASES = {
    "weno5": dict(scheme=oracle.JS, all_mode=False),
    "all": dict(scheme=oracle.JS, all_mode=True),
    "weno5_teno": dict(scheme=oracle.TENO, all_mode=False),
}


def main():
    oracle.build()
    out_dir = os.path.join(HERE, "driver")
    os.makedirs(out_dir, exist_ok=True)
    for name, kw in CASES.items():
        x, y, z, t = oracle.harness_run(199, 199, 199, 8, 6, eps=1e-16, teno_ct=1e-5, **kw)
        with open(os.path.join(out_dir, name + ".txt"), "w") as f:
            for lab, val in zip("XYZT", (x, y, z, t)):
                f.write(f"{lab} {val:.10E}\n")
        print(name, x, y, z, t, flush=True)


if __name__ == "__main__":
    main()
