"""Copies the reference's input decks (input/*.in) here as test fixtures.

The decks are the reference's own problem descriptions (namelist text read
by Snap::parse_arguments, snap.cc:1032-1168); the GPU box has no reference
tree, so the deck tests read these copies.  Run in a container that has the
reference: python tests/decks/make_decks.py [reference root]
"""
import pathlib
import shutil
import sys

HERE = pathlib.Path(__file__).resolve().parent


def main():
    root = pathlib.Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    for src in sorted((root / "input").glob("*.in")):
        shutil.copyfile(src, HERE / src.name)
        print("copied", src.name)


if __name__ == "__main__":
    main()
