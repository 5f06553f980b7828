"""Copies the reference's golden data into tests/golden/ and records their SHA-256.

Sources (read from a checkout of the reference project):
  tests/fixtures/cpp_{analytic_layers,mc_aniso,mc_layers,mc_footprint2,particles_c3r,
  particles_c1_lin}.f64 -- 48x48x3 little-endian f64 images written by the original C++
  oracle (loaded by crates/gps-core/tests/cpp_crosscheck.rs:36-45);
  tests/fixtures/synthetic_sh1.ply -- a small binary SH-degree-1 3DGS file
  (generator tests/gen_synthetic_ply.py).
Usage: python tests/golden/make_fixtures.py <reference_root>
"""
import hashlib
import json
import os
import shutil
import sys

NAMES = ["cpp_analytic_layers.f64", "cpp_mc_aniso.f64", "cpp_mc_layers.f64", "cpp_mc_footprint2.f64",
         "cpp_particles_c3r.f64", "cpp_particles_c1_lin.f64", "synthetic_sh1.ply"]


def main(root):
    here = os.path.dirname(os.path.abspath(__file__))
    manifest = {}
    for n in NAMES:
        src = os.path.join(root, "tests", "fixtures", n)
        dst = os.path.join(here, n)
        shutil.copyfile(src, dst)
        manifest[n] = hashlib.sha256(open(dst, "rb").read()).hexdigest()
    with open(os.path.join(here, "MANIFEST.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print(json.dumps(manifest, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <reference_root>")
    main(sys.argv[1])
