"""The wide-range subband workload at its configured size, against the
reference CPU path on sampled DM groups.

Configuration: 2-bit samples, 4096 channels over 300-400 MHz, 81.92 us,
2^22 samples, 64 subbands, nominal DMs every 20 pc cm^-3, 8192 DM trials over
0-3000, 16 pulsars, 50 Hz narrowband RFI in 5 % of the channels and 0.1 Hz
zero-DM impulses.  The RFI drives ~10^8 raw peaks, so the search selects
candidates on the device.

* The whole search runs through DmSearch; for the first, a middle and the
  last nominal-DM group, the dedispersed rows equal the reference's
  dedisperse_subband_cpu (dedispersion.cpp:331-453) on the unpacked levels
  bit for bit, and one group's raw peaks equal the reference's
  find_dm_peaks_cpu (dm_search.cpp:142-199) byte for byte.
* On a shorter observation of the same configuration (2^20 samples, 1024
  DM trials, millions of raw peaks) the device candidate selection equals
  the host selection of the expanded, sorted peaks.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _cpu_checker():
    from oracle.oracle import Oracle
    return Oracle("reference" if Oracle.available("reference") else "port")


def test_wide_subband_at_size_matches_reference_on_sampled_groups():
    psutil = pytest.importorskip("psutil")
    from gaffa_b200 import configs, core, search, synth
    cfg = configs.wide_subband()
    obs = cfg.obs
    if psutil.virtual_memory().available < 6 * obs.nsamples * obs.nchans:
        pytest.skip("not enough host memory for the unpacked levels")
    raw = core.synth_generate(obs)
    ds = search.from_config(cfg)
    assert ds.device_candidates
    res = ds.run(raw)
    assert res.peak_count > 10_000_000 and len(res.candidates) > 0 and len(res.peaks) == 0
    npn, nout = cfg.ndm_per_nominal, ds.nout
    first = [0, (cfg.ndm // npn // 2) * npn, ((cfg.ndm - 1) // npn) * npn]
    staged = ds.stage(raw)
    ws = torch.empty(ds.dedisp.workspace_bytes(npn), dtype=torch.uint8, device="cuda")
    gpu = {}
    for g0 in first:
        cnt = min(npn, cfg.ndm - g0)
        gpu[g0] = ds.dedisp.run(staged, g0, cnt, workspace=ws)[:, :nout].cpu().numpy().view(np.uint32).copy()
    # one group's raw peaks through the host path of the same search
    g0 = first[1]
    ds.device_candidates = False
    peaks, _ = ds.search_staged(staged, dm_ranges=[(g0, g0 + npn)])
    peaks = core.sort_peaks(peaks)
    del staged, ws
    levels = synth.unpack_2bit(raw.cpu().numpy(), obs.nchans)
    del raw
    torch.cuda.empty_cache()
    ref = _cpu_checker()
    freq = obs.frequencies
    want = {}
    for g in first:
        cnt = min(npn, cfg.ndm - g)
        want[g] = ref.dedisperse_subband(levels, freq, cfg.dm_low + g * cfg.dm_step, cfg.dm_step, cnt,
                                         obs.ref_frequency, obs.tsamp, subband_channels=cfg.subband_channels,
                                         ndm_per_nominal=npn)[:, :nout]
        assert np.array_equal(gpu[g], want[g]), f"dedispersed rows of the group at DM trial {g} differ"
    del levels
    ref_peaks = ref.find_dm_peaks(np.ascontiguousarray(want[g0]), cfg.dms[g0:g0 + npn], obs.tsamp,
                                  cfg.plan_options(), cfg.preprocess_options(), cfg.snr_threshold)
    ref_peaks["dm_index"] += np.uint64(g0)
    assert len(peaks) == len(ref_peaks) > 0
    assert np.array_equal(peaks, ref_peaks)


def test_wide_subband_device_candidates_equal_host_candidates():
    from gaffa_b200 import configs, core, search
    cfg = configs.wide_subband(nsamples=1 << 20, ndm=1024)
    raw = core.synth_generate(cfg.obs)
    ds = search.from_config(cfg, device_candidates=False)
    host = ds.run(raw)
    assert len(host.peaks) > 1_000_000
    ds.device_candidates = True
    dev = ds.run(raw)
    assert dev.peak_count == len(host.peaks)
    assert np.array_equal(dev.candidates, host.candidates)
    assert np.array_equal(dev.ranked, host.ranked) and np.array_equal(dev.harmonics, host.harmonics)
    if dev.fold_profile is not None:
        np.testing.assert_allclose(dev.fold_profile, host.fold_profile, rtol=1e-6)
