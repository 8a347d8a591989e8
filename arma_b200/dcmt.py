"""The ``arma-dcmt`` programme: ``python -m arma_b200.dcmt [-n N] [-p P] [-o PATH] [-s SEED]``.

Creates N dcmt Mersenne Twister parameter sets of period 2^P - 1 (w = 32)
with consecutive ids and writes them to PATH in the mt.dat layout that
``arma_mt_file_read`` and the driver's ``mt_file`` read, like the reference's
``arma-dcmt -n N -o PATH`` (src/dcmt.cc:15-33, which creates p = 521 sets from
a clock seed).  The creation itself is ``arma_mt_create`` in the library.
Extensions: ``-p`` chooses the period, ``-s`` makes the file reproducible, and
an id for which no twist vector gives a primitive polynomial is skipped (the
reference throws "bad MT"); ``--first-id`` sets the first id.
"""
from __future__ import annotations

import argparse
import sys
import time

from . import capi as A


def create_sets(n: int, p: int, seed: int, first_id: int = 0, log=None):
    """n parameter sets with consecutive ids from `first_id`, skipping ids
    without a primitive set; returns [(id, params)]."""
    out = []
    i = first_id
    while len(out) < n:
        if i >= 65536:
            raise A.ArmaError(-7, "ran out of generator ids")
        t0 = time.time()
        try:
            out.append((i, A.mt_create(p, i, seed)))
            if log:
                log(f"Finished [{len(out)}/{n}] id {i} in {time.time() - t0:.1f} s")
        except A.ArmaError as e:
            if e.code != -7:
                raise
            if log:
                log(f"id {i}: {e}")
        i += 1
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m arma_b200.dcmt")
    ap.add_argument("-n", type=int, default=128, help="number of generators")
    ap.add_argument("-o", default="mt.dat", help="output file")
    ap.add_argument("-p", type=int, default=521, help="Mersenne exponent of the period")
    ap.add_argument("-s", "--seed", type=int, default=None, help="search seed (default: clock)")
    ap.add_argument("--first-id", type=int, default=0)
    args = ap.parse_args(argv)
    if args.n <= 0:
        sys.stderr.write(f"Bad no. of generators: {args.n}\n")
        return 1
    seed = args.seed if args.seed is not None else time.time_ns() & 0xffffffff
    sets = create_sets(args.n, args.p, seed, args.first_id,
                       log=lambda m: sys.stderr.write(m + "\n"))
    A.mt_file_write(args.o, [s for _, s in sets])
    sys.stderr.write(f"Saved {args.n} MT configuration(s) in \"{args.o}\" "
                     f"(p = {args.p}, seed = {seed}, ids {[i for i, _ in sets]})\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
