"""Run the reference's own input-deck executable on every deck under tests/decks/ and keep its
output as a golden fixture (tests/golden/<deck>.ref.out), timestamp lines removed.

    make -C oracle ref REF_SRC=<reference>/src/lib/accel && python tests/golden/make_deck_golden.py

oracle/_ref/accel+ref is the reference's process.cpp compiled with its library sources; the decks
name their lattice files relative to the repository root, so the decks run from there.
"""
from __future__ import annotations

import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def strip_times(text: str) -> str:
    return "".join(l for l in text.splitlines(keepends=True) if not l.startswith("#UTC"))


def main():
    exe = os.path.join(ROOT, "oracle", "_ref", "accel+ref")
    for deck in sorted(glob.glob(os.path.join(ROOT, "tests", "decks", "*.in"))):
        out = subprocess.run([exe, deck], cwd=ROOT, capture_output=True, text=True, check=True).stdout
        name = os.path.splitext(os.path.basename(deck))[0]
        with open(os.path.join(HERE, name + ".ref.out"), "w") as f:
            f.write(strip_times(out))
        print("wrote", name + ".ref.out", len(out.splitlines()), "lines")


if __name__ == "__main__":
    main()
