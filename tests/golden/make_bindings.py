"""Regenerate tests/golden/reference_bindings.json: the C entry points that the
reference's own Python modules bind at import time (python/mesh/*.py,
python/numerics/*.py), found as `lib<name>.<Symbol>` attribute accesses.

Usage: STREAM_REFERENCE=<reference root> python tests/golden/make_bindings.py
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ref = os.environ.get("STREAM_REFERENCE")
    if not ref:
        sys.exit("set STREAM_REFERENCE to the reference tree")
    out = {}
    for sub in ("mesh", "numerics"):
        d = os.path.join(ref, "python", sub)
        for f in sorted(os.listdir(d)):
            if not f.endswith(".py") or f == "__init__.py":
                continue
            names = sorted(set(re.findall(r"\blib(?:mesh|num|geo)\.([A-Za-z_][A-Za-z0-9_]*)", open(os.path.join(d, f)).read())))
            out[f"python/{sub}/{f}"] = names
    with open(os.path.join(HERE, "reference_bindings.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
        fh.write("\n")
    print({k: len(v) for k, v in out.items()})


if __name__ == "__main__":
    main()
