"""gaffa's Python API on the B200 path: a drop-in for ``import gaffa``.

    from gaffa_b200 import gaffa
    fb = gaffa.io.Filterbank(path)
    dd = gaffa.dedispersion.dedisperse_multi_dm(fb, dm_low=0.0, dm_step=0.5, ndm=512)
    plan = gaffa.ffa.make_riptide_plan(nsamples=n, tsamp=fb.header.tsamp, period_min=0.2, period_max=2.0)
    peaks = gaffa.ffa.ffa_search(series, plan, snr_threshold=6.0)

Modules and names follow the reference package (python/gaffa/__init__.py):
``dedispersion``, ``ffa``, ``io``, ``pfold`` and ``_core``.  Everything runs on
the GPU through libgaffa_b200.so; ``backend`` defaults to ``"cuda"`` and
``backend="cpu"`` raises ValueError (there is no CPU path).
"""
from . import _core, dedispersion, ffa, io, pfold
from ._core import cuda_device_count, cuda_runtime_version

__all__ = ["cuda_device_count", "cuda_runtime_version", "dedispersion", "ffa", "io", "pfold"]
