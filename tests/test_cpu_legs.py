"""The CPU legs of bench.py: the host-side generator of the checkers and the
reference arm, which must never load the CUDA library."""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from gaffa_b200 import configs, synth  # noqa: E402
from oracle import oracle  # noqa: E402


@pytest.mark.parametrize("name,kw", [("plain_end_to_end", dict(nsamples=1 << 13)),
                                     ("survey_size", dict(nsamples=1 << 11)),
                                     ("wide_subband", dict(nsamples=1 << 11))])
def test_host_generator_matches_numpy_generator(name, kw):
    """oracle/synth_oracle.c gives the numpy generator's bytes, pulsars, RFI and
    2-bit packing included, for a row range that starts mid-observation."""
    obs = configs.CONFIGS[name](seed=11, **kw).obs
    want = synth.generate(obs, 100, 1500)
    if obs.nbits == 2:
        want = synth.pack_2bit(want)
    got = oracle.synth_generate(obs, 100, 1500)
    assert np.array_equal(got, want)


def test_host_generator_counts_each_sample_once_in_wide_windows():
    """Pulses wider than half a period (windows of neighbouring pulses overlap)
    and very narrow ones."""
    obs = configs.plain_end_to_end(seed=2, nsamples=1 << 13, nchans=64).obs
    obs.pulsars += [synth.Pulsar(0.011, 50.0, 0.12, 20.0), synth.Pulsar(0.0101, 10.0, 0.09, 20.0),
                    synth.Pulsar(0.3, 20.0, 0.001, 40.0)]
    assert np.array_equal(oracle.synth_generate(obs), synth.generate(obs))


def test_reference_arm_runs_without_the_cuda_library():
    """bench.py --impl reference on a small case: one JSON line, a sample of at
    least five DM trials (the reference's parallel DM loop), and no
    libgaffa_b200.so mapped into the process."""
    if not oracle.Oracle.available("port"):
        pytest.skip("oracle not built")
    code = (
        "import sys, json, argparse; sys.path.insert(0, %r)\n"
        "import bench\n"
        "bench.set_cpu_threads()\n"
        "args = argparse.Namespace(workload='survey_size', ndm=64, nsamples_log2=16, steps=1, warmup=1)\n"
        "bench.run_reference(args, 0, 1)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'cuda_library_loaded': 'libgaffa_b200' in maps}))\n" % str(ROOT))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    line, maps = lines[0], lines[1]
    assert line["impl"] == "reference" and line["value"] > 0
    assert "DM trials" in line["cpu_baseline"]["sample"]
    first, last = line["cpu_baseline"]["sample"].split("DM trials ")[1].split(" ")[0].split("-")
    assert int(last) - int(first) + 1 >= 5
    assert line["cpu_baseline"]["cores"] >= 1 and line["cpu_baseline"]["cpu"]["model"]
    assert maps["cuda_library_loaded"] is False
