"""Aligned single-DM spectrum (dedisperse_spectrum_cpu, src/gaffa/dedispersion.cpp:249-289).

tests/golden/ref_spectrum.npz holds the reference's own outputs
(tests/golden/make_golden.py); the CUDA path must match them byte for byte.
"""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_spectrum.npz"
CASES = [("sp_full", 60.0, 0, None), ("sp_sub", 37.5, 5, 41), ("sp_zero", 0.0, 0, None)]


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(GOLDEN))


@pytest.mark.parametrize("key,dm,cb,ce", CASES)
def test_oracle_matches_reference(port, golden, key, dm, cb, ce):
    f = golden["sp_freq"]
    out = port.dedisperse_spectrum(golden["sp_data"], f, dm, f.max(), 1e-3, cb, ce)
    assert np.array_equal(out, golden[key])


def test_oracle_rejects_empty_output(port, golden):
    from oracle.oracle import OracleError
    f = golden["sp_freq"]
    with pytest.raises(OracleError):
        port.dedisperse_spectrum(golden["sp_data"][:10], f, 60.0, f.max(), 1e-3)


@pytest.mark.gpu
@pytest.mark.parametrize("key,dm,cb,ce", CASES)
def test_cuda_spectrum_matches_reference(golden, key, dm, cb, ce):
    import torch
    from gaffa_b200 import core
    f = golden["sp_freq"]
    x = torch.from_numpy(golden["sp_data"]).cuda()
    out = core.dedisperse_spectrum(x, f, dm, 1e-3, chan_begin=cb, chan_end=ce)
    assert np.array_equal(out.cpu().numpy(), golden[key])


@pytest.mark.gpu
def test_cuda_spectrum_float_and_errors(golden):
    import torch
    from gaffa_b200 import core
    f = golden["sp_freq"]
    x = torch.from_numpy(golden["sp_data"].astype(np.float32)).cuda()
    out = core.dedisperse_spectrum(x, f, 60.0, 1e-3)
    assert np.array_equal(out.cpu().numpy(), golden["sp_full"].astype(np.float32))
    with pytest.raises(ValueError):
        core.dedisperse_spectrum(x[:10], f, 60.0, 1e-3)           # empty output range
    with pytest.raises(ValueError):
        core.dedisperse_spectrum(x, f, -1.0, 1e-3)                 # negative DM
    with pytest.raises(ValueError):
        core.dedisperse_spectrum(x, f, 60.0, 1e-3, ref_frequency_mhz=1300.0)


FOLD_RTOL = 1e-6  # FP64 sums in a different order from the reference


@pytest.mark.gpu
@pytest.mark.parametrize("tag,kw", [("fold", dict(nbin=32, tsubint=0.5)),
                                    ("fold_ch", dict(nbin=24, tsubint=0.7, output_channels=12))])
def test_cuda_fold_dedispersed_spectrum_matches_reference(golden, tag, kw):
    """fold_dedispersed_spectrum_view_cpu of the aligned spectrum (folding.cpp:408-438):
    cube and exposure, then the profile / frequency-phase / time-phase projections."""
    import torch
    from gaffa_b200 import core
    x = torch.from_numpy(golden["sp_data"]).cuda()
    r = core.fold_dedispersed_spectrum(x, golden["sp_freq"], 60.0, 0.2, 1e-3, **kw)
    np.testing.assert_allclose(r["exposure"].cpu().numpy(), golden[f"{tag}_exposure"], rtol=1e-12)
    for k in ("cube", "profile", "freq_phase", "time_phase"):
        np.testing.assert_allclose(r[k].cpu().numpy(), golden[f"{tag}_{k}"], rtol=FOLD_RTOL, atol=1e-5)


@pytest.mark.gpu
def test_cuda_fold_spectrum_rejects_bad_arguments(golden):
    import torch
    from gaffa_b200 import core
    x = torch.from_numpy(golden["sp_full"]).cuda()
    with pytest.raises(ValueError):
        core.fold_spectrum(x, 0.2, 1e-3, 32, 0)                          # subint_samples == 0
    with pytest.raises(ValueError):
        core.fold_spectrum(x, 0.2, 1e-3, 32, 100, output_channels=7)     # 48 % 7 != 0
    with pytest.raises(ValueError):
        core.fold_spectrum(x, -0.2, 1e-3, 32, 100)
    bad = x.float()
    bad[3, 5] = float("nan")
    with pytest.raises(ValueError, match="finite"):
        core.fold_spectrum(bad, 0.2, 1e-3, 32, 100)
