"""Copies the reference's own test fixtures into tests/golden/.

Source: StanfordLegion/pennant-legion test/ (decks of every problem and the
one known-answer output set, test/sedov/sedov.{xy,geo,zr,ze,zp}).  The files
are copied byte for byte; the test suite reads only these copies.

Usage: python tests/golden/copy_reference_fixtures.py REFERENCE_ROOT

(REFERENCE_ROOT is the checked-out StanfordLegion/pennant-legion tree.)
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref: str) -> None:
    test = os.path.join(ref, "test")
    for prob in sorted(os.listdir(test)):
        src = os.path.join(test, prob, prob + ".pnt")
        if os.path.exists(src):
            shutil.copyfile(src, os.path.join(HERE, prob + ".pnt"))
    for ext in ("xy", "geo", "zr", "ze", "zp"):
        shutil.copyfile(os.path.join(test, "sedov", "sedov." + ext), os.path.join(HERE, "sedov." + ext))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
