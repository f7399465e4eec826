"""Regenerate the committed fixtures under tests/golden/.

Run in the build container, where the reference tree is mounted:

    python tests/golden/make_fixtures.py /root/reference

* models/*.json: the reference's earth-model input files used by the
  configurations and by the reference's own model-reader known-answer test
  (f90/testReadNodeEarthmodel.f90).  They are input data, copied verbatim so
  the GPU tests and the bench can run where the reference is absent.
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
MODELS = ["prem-no-ocean_si.json", "ak135q.json"]


def main(ref):
    os.makedirs(os.path.join(HERE, "models"), exist_ok=True)
    for m in MODELS:
        shutil.copyfile(os.path.join(ref, "earthmodels", m), os.path.join(HERE, "models", m))
        print("wrote", m)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
