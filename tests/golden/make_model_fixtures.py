"""Writes tests/golden/models/l3k3.mtp: the seeded l3k3 Cu-Zr model of the
benchmark workload (preset "l3k3" of sus2sh.models, written by
sus2sh_write_synthetic_model in libsus2sh_tools.so).

The benchmark's reference arm reads this file instead of calling the writer,
so that it loads no library of this repository; tests/test_capi.py checks
that the writer still produces it byte for byte.

    python tests/golden/make_model_fixtures.py
"""
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "gpumd-sus2-sh_b200"))

FIXTURES = {"l3k3": os.path.join(HERE, "models", "l3k3.mtp")}


def write_fresh(name: str, directory: str) -> str:
    from sus2sh import models
    return models.preset_model(name, directory)


if __name__ == "__main__":
    with tempfile.TemporaryDirectory() as d:
        for name, dst in FIXTURES.items():
            os.makedirs(os.path.dirname(dst), exist_ok=True)
            with open(write_fresh(name, d), "rb") as f, open(dst, "wb") as g:
                g.write(f.read())
            print(dst)
