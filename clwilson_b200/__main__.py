"""python -m clwilson_b200 -p # -P # [-s] [-r]: runs the clwilson command-line program.

The flags, messages and results.txt are those of the reference program
(main.cpp:27-159); all work happens in libwilson.so.
"""
import os
import sys

from clwilson_b200 import build as _build

if __name__ == "__main__":
    exe = _build.CLI
    if not os.path.exists(exe):
        raise SystemExit(f"{exe} is not built; run `python -m clwilson_b200.build`")
    os.execv(exe, [exe] + sys.argv[1:])
