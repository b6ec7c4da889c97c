"""Dedispersion returning host NumPy results (python/gaffa/dedispersion.py)."""
from ._core import (DedispersedResult, DedispersedSpectrum, dedisperse_multi_dm, dedisperse_single_dm,
                    dedisperse_spectrum, dedisperse_subband)

__all__ = ["DedispersedResult", "DedispersedSpectrum", "dedisperse_multi_dm", "dedisperse_single_dm",
           "dedisperse_spectrum", "dedisperse_subband"]
