"""Copies the reference's own regression fixtures into tests/golden/.

The reference (davecats/homogenenousShearTurbulence) keeps three final
fields of 50-step runs in tests/reference/*.fld together with the decks that
made them (tests/decks/*.in); tests/regression.sh compares a fresh run with
them at 1e-10.  They are the golden vectors of this path.  This script
copies them unchanged (data, not code) and writes their sha256 sums to
SHA256SUMS so that a test can check the copies.

    python tests/golden/make_fixtures.py /path/to/reference
"""
import hashlib
import pathlib
import shutil
import sys

HERE = pathlib.Path(__file__).resolve().parent
NAMES = ["small", "small_s2x", "small_stokes"]
EXTRA_DECKS = ["kelvin", "kelvin_exact", "kelvin_s2const", "kelvin_s2osc", "kelvin_s2mean",
               "kelvin_stretched", "kelvin_damped", "kelvin_hard", "kelvin_outside", "pressure"]


def main(ref):
    ref = pathlib.Path(ref)
    lines = []
    for n in NAMES:
        for src, dst in ((ref / "tests/reference" / f"{n}.fld", HERE / f"{n}.fld"),
                         (ref / "tests/decks" / f"{n}.in", HERE / f"{n}.in")):
            shutil.copyfile(src, dst)
            lines.append(f"{hashlib.sha256(dst.read_bytes()).hexdigest()}  {dst.name}")
    for n in EXTRA_DECKS:
        src, dst = ref / "tests/decks" / f"{n}.in", HERE / f"{n}.in"
        shutil.copyfile(src, dst)
        lines.append(f"{hashlib.sha256(dst.read_bytes()).hexdigest()}  {dst.name}")
    (HERE / "SHA256SUMS").write_text("\n".join(lines) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py /path/to/reference (a checkout of the reference project)")
    main(sys.argv[1])
