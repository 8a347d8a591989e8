"""Regenerate the committed golden fixtures in this directory.

    python tests/golden/make_golden.py --reference /path/to/arma

Two kinds of fixtures:

* ``reference_known_answers.json`` -- the known answers that the reference's
  own unit tests assert (Owen T, the skew-normal CDF, the 3x3 symmetric solve,
  the config-syntax strings).  When the reference source tree is available
  they are parsed out of its test files (read as text); otherwise the
  committed file is kept.
* ``oracle_cases.npz`` -- small seeded cases computed by the CPU oracle
  (``oracle/``): MT19937 draws, white noise, AR filter outputs, the
  renormalisation, NIT and velocity results.  The GPU parity tests compare the
  device path against these, and the CPU tests check that the oracle still
  reproduces them.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def parse_reference(ref: str) -> dict:
    t = os.path.join(ref, "src", "test")
    out = {}
    txt = open(os.path.join(t, "owen-t-test.cc")).read()
    txt = txt[txt.index("TEST(OwenT, ExactValues)"):]
    out["owen_t"] = [
        [float(h), float(a), float(v)]
        for h, a, v in re.findall(
            r"owen_t<T>\(([-\d.]+),\s*(?:T\()?([-\d.]+)\)?\),\s*T\(([-\d.e]+)\)", txt)
    ]
    txt = open(os.path.join(t, "skew-normal-test.cc")).read()
    m = re.search(r"Skew_normal<T> sn\(T\(([-\d.]+)\), T\(([-\d.]+)\), T\(([-\d.]+)\)\)", txt)
    out["skew_normal"] = {
        "params": [float(m.group(i)) for i in (1, 2, 3)],
        "cdf": [[float(x), float(v)] for x, v in
                re.findall(r"sn\.cdf\((-?\d+)\),\s*T\(([-\d.e]+)\)", txt)],
        "tolerance": 1e-5,
    }
    txt = open(os.path.join(t, "linalg-test.cc")).read()
    blk = txt[txt.index("TEST(Cholesky, Matrix3)"):]
    blk = blk[:blk.index("TEST(Inverse")]
    mat = [float(v) for v in re.search(r"lhs = ([-\d., ]+);", blk).group(1).split(",")]
    exp = [float(v) for v in re.findall(r"EXPECT_NEAR\(rhs\(\d\), T\(([-\d.]+)\)", blk)]
    out["sysv_3x3"] = {"a": mat, "b": [1.0, 1.0, 1.0], "x": exp, "tolerance": 1e-3}
    txt = open(os.path.join(t, "output-flags-test.cc")).read()
    blk = txt[txt.index("::testing::Values("):]
    out["output_flags_inputs"] = [
        s.encode().decode("unicode_escape") for s in re.findall(r'"((?:[^"\\]|\\.)*)"', blk)
    ]
    out["source"] = "reference src/test/{owen-t,skew-normal,linalg,output-flags}-test.cc"
    return out


def oracle_cases() -> dict:
    import oracle as O

    cases = {}
    p = O.mt19937_params()
    cases["mt19937_seed42"] = O.std_mt19937(42, 4096)
    cases["mt19937_seed5489_10000"] = O.std_mt19937(5489, 10000)[-1:]
    # white noise: 5000 values, stddev 0.5, seed 42
    cases["wn_seed42"] = O.white_noise(p, 42, 0.5, 5001)
    cases["wn_words_seed42"] = np.array([O.white_noise_words(p, 42, 5001)], np.int64)
    # AR filter: standing-wave model of order 3^3 on a ragged 23x17x29 grid
    acf = O.acf("standing_wave", (3, 3, 3), 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    phi, var = O.ar_fit(acf, (3, 3, 3), "cholesky")
    eps = O.white_noise(p, 7, np.sqrt(var), 23 * 17 * 29).reshape(23, 17, 29)
    cases["ar_phi_333"] = phi
    cases["ar_eps_333"] = eps
    cases["ar_zeta_333"] = O.ar_filter(eps, phi)
    # order 7^3 standing wave (the 200x40x40 model) on a 24x20x20 grid
    acf = O.acf("standing_wave", (7, 7, 7), 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
    phi7, var7 = O.ar_fit(acf, (7, 7, 7), "cholesky")
    eps7 = O.white_noise(p, 42, np.sqrt(var7), 24 * 20 * 20).reshape(24, 20, 20)
    cases["ar_phi_777"] = phi7
    cases["ar_var_777"] = np.array([var7])
    cases["ar_eps_777"] = eps7
    z7 = O.ar_filter(eps7, phi7)
    cases["ar_zeta_777"] = z7
    zr, sc = O.variance_renorm(z7, acf[0, 0, 0])
    cases["renorm_zeta_777"] = zr
    cases["renorm_scale_777"] = np.array([sc])
    # NIT by bisection on a slice of the renormalised surface
    vals = zr.ravel()[:2000]
    sd = np.sqrt(acf[0, 0, 0])
    cases["nit_in"] = vals
    cases["nit_gc"] = O.nit_transform(vals, sd, "gram_charlier", [0.3, 3.2], (-5, 5))
    cases["nit_sn"] = O.nit_transform(vals, sd, "skew_normal", [0.0, 1.0, 1.5], (-5, 5))
    # linear velocity potential on a 16x32x32 surface, 2 slices, 3 depths
    zsurf = zr[:16, :16, :16]
    zsurf = np.ascontiguousarray(np.concatenate([zsurf, zsurf], axis=1))
    zsurf = np.ascontiguousarray(np.concatenate([zsurf, zsurf], axis=2))
    cases["vel_zeta"] = zsurf
    cases["vel_phi"] = O.velocity_linear(zsurf, (1.0, 1.0, 1.0), 12.0, [0.0, -1.0, -2.0],
                                         [3, 10])
    return cases


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="checkout of the reference (read-only); its src/test/*-test.cc "
                         "give the known answers")
    args = ap.parse_args()
    ka = os.path.join(HERE, "reference_known_answers.json")
    if os.path.isdir(args.reference):
        with open(ka, "w") as f:
            json.dump(parse_reference(args.reference), f, indent=1)
        print("wrote", ka)
    np.savez_compressed(os.path.join(HERE, "oracle_cases.npz"), **oracle_cases())
    print("wrote", os.path.join(HERE, "oracle_cases.npz"))


if __name__ == "__main__":
    main()
