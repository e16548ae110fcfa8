"""Committed C headers of the pipelines shipped prebuilt (include/)."""

import os

from .apps import catalog

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def expected_headers():
    out = {}
    for name, builder in catalog.default_builds():
        mod = builder().generate_code()
        out["pipeline_%s.h" % mod.name] = mod.header
    return out


def write_headers():
    for fn, text in expected_headers().items():
        with open(os.path.join(INCLUDE, fn), "w") as f:
            f.write(text)


if __name__ == "__main__":
    write_headers()
