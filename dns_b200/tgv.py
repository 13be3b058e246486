#!/usr/bin/env python
"""Generate the Taylor-Green initial condition: drop-in for slitvinov/dns
tgv.py (same flags, same .raw output byte for byte).

    python -m dns_b200.tgv -l <level> -o <file.raw>      # n = 2**level
"""
import argparse
import sys

from dns_b200 import tgv_fields, write_raw


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="Generate initial conditions for Taylor–Green vortex")
    ap.add_argument("-l", "--level", type=int, required=True)
    ap.add_argument("-o", "--output", type=str, required=True)
    a = ap.parse_args(argv)
    n = 1 << a.level
    sys.stderr.write(f"tgv.py: {n=}\n")
    write_raw(a.output, tgv_fields(n))
    return 0


if __name__ == "__main__":
    sys.exit(main())
