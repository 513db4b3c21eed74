"""Run the reference's own driver (test/full_example.cu) twice on one system:
linked against the reference library (oracle/_ref/full_example_ref) and,
unchanged, against this engine (oracle/_ref/full_example_b200); both built by
``make -C oracle drivers``.  Test infrastructure (needs a CUDA GPU).

The driver reads ``<sys>.psf``/``<sys>.cor`` and the t-designs from
``SS31-Mar-2016/`` in its working directory; this script writes the seeded
water box in CHARMM format and renders the project's t-design store there, so
both builds run on the same atoms and nodes.  Logs (the driver's stdout) go
to ``--out``; utils/parse_glst_results.py of the reference reads them.

    python oracle/run_drivers.py --workload water10k --out DIR
"""
import argparse
import math
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="water10k")
    ap.add_argument("--out", required=True)
    args = ap.parse_args()
    g = __graft_entry__.load_package()
    from glst_b200 import systems
    sys.path.insert(0, os.path.dirname(g.TDESIGN_STORE))
    import make_tdesigns
    s = systems.config_system(args.workload, seed=0)
    os.makedirs(args.out, exist_ok=True)
    rc = 0
    with tempfile.TemporaryDirectory() as work:
        make_tdesigns.write_reference_dir(g.TDESIGN_STORE, os.path.join(work, "SS31-Mar-2016"))
        systems.write_charmm(os.path.join(work, args.workload), s["x"], s["y"], s["z"], s["q"])
        for build in ("ref", "b200"):
            exe = os.path.join(HERE, "_ref", "full_example_" + build)
            env = dict(os.environ, GLST_BENCH_TERMINAL="1", GLST_BENCH_SWEEP="drivers",
                       GLST_BENCH_SYS=args.workload, GLST_BENCH_GPUS="1")
            cmd = [exe, args.workload, repr(s["tol"]), "%.17g" % s["box"][0], "%.17g" % s["rcut"]]
            with open(os.path.join(args.out, "full_example_%s_%s.log" % (args.workload, build)), "w") as fh:
                r = subprocess.run(cmd, cwd=work, stdout=fh, stderr=subprocess.DEVNULL, env=env)
            print(build, "exit", r.returncode, flush=True)
            rc = rc or r.returncode
    return rc


if __name__ == "__main__":
    raise SystemExit(main())
