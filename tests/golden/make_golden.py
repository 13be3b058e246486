"""Regenerate the golden fixtures in tests/golden from the reference checkout.

Run where the reference sources are checked out, after building the oracle
(`make -C oracle REF=<checkout>`):

    python tests/golden/make_golden.py --ref <reference checkout>

Fixtures written:
  ref_0128_<Re>.txt, ref_0256_<Re>.txt
      the reference's own shipped stdout histories (0128/<Re>, 0256/<Re>):
      Taylor-Green, dt = 0.0025, T = 10, nu = 1/Re, at 128^3 and 256^3.
  tgv_l<L>.sha256
      sha256 of the .raw file the reference tgv.py writes for level L.
  refrun_tgv64_nu0.01_dt0.01_T1.txt
      stdout of the reference main.c (compiled unchanged against the oracle's
      FFTW-subset shim, oracle/_ref/dns) for config "64^3 Taylor-Green,
      nu = 0.01, dt = 0.01, T = 1".
  refrun_tgv32_nu0.01_dt0.01_T0.2.txt
      same at 32^3, T = 0.2, used by the CLI parity test.
  refrun_tgv128_re0100_dt0.0025_T5.txt
      the reference main.c at 128^3, nu = 1/100 (written "%.16e" as run.sh
      passes it), dt = 0.0025, T = 5 (2000 steps): main.c's own 128^3 history
      where the published 0128/0100 file no longer follows it.
  refrun_tgv128_re3000_dt0.0025_T2.5.txt
      the same at nu = 1/3000, T = 2.5 (1000 steps), for the GPU test of the
      128^3 path against main.c past t = 1.
  refrun_tgv128_re1600_dt0.005_T10.txt
      the 128^3 configuration of the mixed-precision comparison: nu = 1/1600,
      dt = 0.005, T = 10 (2000 steps).
"""
import argparse
import hashlib
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_DNS = os.path.join(ROOT, "oracle", "_ref", "dns")
RES = ("0100", "0200", "0400", "0800", "1600", "3000")


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="reference checkout (holds main.c, tgv.py, 0128/, 0256/)")
    a = ap.parse_args()
    if not os.path.exists(os.path.join(a.ref, "main.c")):
        ap.error(f"{a.ref} has no main.c")
    if not os.path.exists(REF_DNS):
        ap.error(f"{REF_DNS} is missing: run make -C oracle REF={a.ref} first")
    for size in ("0128", "0256"):
        for re_ in RES:
            shutil.copyfile(os.path.join(a.ref, size, re_), os.path.join(HERE, f"ref_{size}_{re_}.txt"))
    with tempfile.TemporaryDirectory() as tmp:
        for level in (3, 4, 5, 6):
            raw = os.path.join(tmp, f"tgv{level}.raw")
            subprocess.run([sys.executable, os.path.join(a.ref, "tgv.py"), "-l", str(level), "-o", raw],
                           check=True, stderr=subprocess.DEVNULL)
            digest = hashlib.sha256(open(raw, "rb").read()).hexdigest()
            with open(os.path.join(HERE, f"tgv_l{level}.sha256"), "w") as f:
                f.write(digest + "\n")
        runs = ((6, "0.01", "0.01", "1", "refrun_tgv64_nu0.01_dt0.01_T1.txt"),
                (5, "0.01", "0.01", "0.2", "refrun_tgv32_nu0.01_dt0.01_T0.2.txt"),
                (7, "%.16e" % (1 / 100), "0.0025", "5", "refrun_tgv128_re0100_dt0.0025_T5.txt"),
                (7, "%.16e" % (1 / 3000), "0.0025", "2.5", "refrun_tgv128_re3000_dt0.0025_T2.5.txt"),
                (7, "%.16e" % (1 / 1600), "0.005", "10", "refrun_tgv128_re1600_dt0.005_T10.txt"))
        for level, nu, dt, T, name in runs:
            raw = os.path.join(tmp, f"tgv{level}.raw")
            if not os.path.exists(raw):
                subprocess.run([sys.executable, os.path.join(a.ref, "tgv.py"), "-l", str(level), "-o", raw],
                               check=True, stderr=subprocess.DEVNULL)
            env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
            out = subprocess.run([REF_DNS, "-i", raw, "-n", nu, "-s", dt, "-t", T],
                                 check=True, capture_output=True, text=True, env=env).stdout
            with open(os.path.join(HERE, name), "w") as f:
                f.write(out)
    print("golden fixtures written to", HERE)
    return 0


if __name__ == "__main__":
    sys.exit(main())
