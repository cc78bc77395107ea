"""bench.py's data generator on the CPU: SynthRng (Python Xoshiro256++ with the
reference's unit and Box–Muller draws) gives the pinned sequences of gprx
src/rng.rs and the same draws, bit for bit, as the library's gprx_rng_*, so
both arms of the benchmark see identical data although the reference arm never
loads the CUDA library.  Also checks that the reference arm's data path does
not import the package.
"""

import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
import gprx_b200 as gx  # noqa: E402


def test_synth_rng_matches_pins_and_library():
    with open(os.path.join(ROOT, "tests", "golden", "rng_pins.json")) as fh:
        pins = json.load(fh)["seeds"]
    for seed, vals in pins.items():
        r = bench.SynthRng(int(seed))
        assert [r.next_u64() for _ in range(4)] == [int(v) for v in vals]
    for seed in (0, 1, 3, 10):
        a, b = bench.SynthRng(seed), gx.SeededRng(seed)
        assert np.array_equal(a.unit(500), b.unit(500))
        assert np.array_equal(a.normal(5000), b.normal(5000))


def test_reference_arm_data_does_not_load_the_package():
    code = ("import sys; import numpy as np; sys.path.insert(0, %r); import bench; x, y, th = bench.synth(64, 8); "
            "bench.perturbations(th); bench.c1_synth(); print('gprx_b200' in sys.modules)") % ROOT
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True)
    assert out.stdout.strip() == "False"
