"""The ``arma`` programme: ``python -m arma_b200 [-h] [-C DIR] INPUTFILE``.

Reads a ``.arma`` configuration, generates the wavy surface on the GPU,
computes the velocity potentials and writes the output files into the
working directory (or DIR), like the reference's ``arma`` binary
(src/arma_main.cc:80-112, src/common_main.hh).
"""
from __future__ import annotations

import sys

from . import capi as A


def usage(argv0: str = "arma") -> str:
    return f"usage: {argv0} [-h] [-C DIR] INPUTFILE\n"


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    outdir = ""
    if "-C" in argv:
        k = argv.index("-C")
        if k + 1 >= len(argv):
            sys.stdout.write(usage())
            return 1
        outdir = argv[k + 1]
        del argv[k:k + 2]
    if len(argv) != 1 or argv[0] in ("-h", "--help"):
        sys.stdout.write(usage())
        return 0 if argv and argv[0] in ("-h", "--help") else 1
    try:
        with A.Context(0) as ctx, A.Driver.open(argv[0]) as drv:
            info = drv.info()
            sys.stderr.write(f"Input file = {argv[0]}\nOutput grid = {info['shape']}\n")
            drv.set_output_dir(outdir)
            drv.generate_wavy_surface(ctx)
            drv.compute_velocity_potentials(ctx)
            drv.write_all(outdir)
    except A.ArmaError as e:
        if e.code == -6:  # ARMA_EPRNG
            sys.stderr.write("No parallel Mersenne Twisters configuration is found. "
                             "Please, generate sufficient number of MTs with dcmt programme.\n")
        sys.stderr.write(f"ERROR: {e}\n")
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
