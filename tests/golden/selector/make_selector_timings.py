"""Regenerates selector_timings.npz beside this file (needs a GPU, about two minutes on one
B200): 2,200 seeded matrices generated on the device, their structural features and the
timings of the six engine variants.

    python tests/golden/selector/make_selector_timings.py
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))

if __name__ == "__main__":
    sys.exit(subprocess.call([sys.executable, "-m", "pava_b200.selector", "generate", "--out",
                              os.path.join(HERE, "selector_timings.npz")], cwd=ROOT))
