"""Locate the libzstd 1.5.7 shared library bundled on this image (inside Pillow's wheel).

The reference pins zstd 1.5.7 (conanfile.py:14); the system libzstd is 1.5.5, whose
level-3 output may differ, so the 1.5.7 copy is preferred.  Prints the path.
"""
import glob
import os
import sys
import sysconfig


def find_zstd() -> str:
    env = os.environ.get("XNYZ_ZSTD_LIBRARY")
    if env:
        return env
    roots = {sysconfig.get_paths()["purelib"], sysconfig.get_paths()["platlib"]}
    for root in sorted(roots):
        hits = sorted(glob.glob(os.path.join(root, "pillow.libs", "libzstd-*.so.1.5.7")))
        if hits:
            return hits[0]
    raise FileNotFoundError("libzstd 1.5.7 not found (set XNYZ_ZSTD_LIBRARY)")


if __name__ == "__main__":
    try:
        print(find_zstd())
    except FileNotFoundError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
